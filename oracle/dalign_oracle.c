/* dalign_oracle.c -- TEST INFRASTRUCTURE ONLY (the parity oracle; never shipped).
 *
 * Single-threaded CPU restatement of MARVEL daligner's overlap path.  Each function
 * names the reference code it restates.  Threading, buffer growth and in-place vector
 * moves of the reference are left out: they do not change any output.
 */
#include "dalign_oracle.h"

#include <limits.h>
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

typedef uint64_t u64;

/* ------------------------------------------------------------------------------------ */
/*  K-mer index: tuple extraction + stable sort by code (dalign/filter.c:400-490,698-903) */
/* ------------------------------------------------------------------------------------ */

typedef struct
{
    u64 code;
    int32_t rpos, read;
} KPos;

/* stable LSD radix sort of KPos by the low `nbytes` bytes of code */
static void sort_kpos(KPos* x, int64_t n, int nbytes)
{
    KPos* t = (KPos*)malloc(sizeof(KPos) * (n + 1));
    int64_t cnt[256];
    for (int byte = 0; byte < nbytes; byte++)
    {
        int sh = 8 * byte;
        memset(cnt, 0, sizeof(cnt));
        for (int64_t i = 0; i < n; i++)
            cnt[(x[i].code >> sh) & 0xff]++;
        int64_t s = 0;
        for (int d = 0; d < 256; d++)
        {
            int64_t c = cnt[d];
            cnt[d] = s;
            s += c;
        }
        for (int64_t i = 0; i < n; i++)
            t[cnt[(x[i].code >> sh) & 0xff]++] = x[i];
        memcpy(x, t, sizeof(KPos) * n);
    }
    free(t);
}

/* Extraction over the unmasked segments of each read (tuple_thread, filter.c:400-490):
 * a k-mer is kept when it lies wholly inside [0,rlen) minus the mask intervals. */
static int64_t extract_kmers(const or_block* b, int K, KPos* list)
{
    u64 kmask = (K >= 32) ? ~0ull : ((1ull << (2 * K)) - 1);
    int64_t n = 0;
    for (int i = 0; i < b->nreads; i++)
    {
        const uint8_t* s = b->bases + b->boff[i];
        int rlen = b->rlen[i];
        int64_t f0 = 0, f1 = 0;
        if (b->mask_anno)
        {
            f0 = b->mask_anno[i];
            f1 = b->mask_anno[i + 1];
        }
        for (int64_t a = f0; a <= f1; a += 2)
        {
            int p = (a == f0) ? 0 : b->mask_data[a - 1];
            int q = (a == f1) ? rlen : b->mask_data[a];
            if (p + K <= q)
            {
                u64 c = 0;
                for (int x = 1; x < K; x++)
                    c = (c << 2) | s[p++];
                while (p < q)
                {
                    c = ((c << 2) | s[p]) & kmask;
                    list[n].code = c;
                    list[n].read = i;
                    list[n].rpos = p++;
                    n++;
                }
            }
            if (!b->mask_anno)
                break;
        }
    }
    return n;
}

/* daligner -b: frequency-weighted tuples (biased_tuple_thread, filter.c:492-633, with the
 * tables of Sort_Kmers, filter.c:718-733).  A base x carries the information
 * w[x] = ceil(-10000 log4 freq[x]); a window of k <= K bases is grown to the right while its
 * information is below 10000 K (and k < K), trimmed from the left while what remains still
 * reaches 10000 K, and kept when its information exceeds 10000 (K - 2), as a K-mer code with
 * its k bases at the top and zeros below.  The window then slides one base (same length).
 * The tables are made once, from the frequencies of the first block indexed: daligner's A
 * block, whose frequencies are the ones New_Align_Spec receives. */
typedef struct
{
    int w[5], norm, thresh, K; /* w[4] = 0: see bias_scan */
    u64 kmask;
} Bias;

static void bias_tables(const float freq[4], int K, Bias* B)
{
    double scale = -10000. / log(4.);
    for (int i = 0; i < 4; i++)
        B->w[i] = (int)ceil(scale * log(freq[i]));
    B->w[4] = 0;
    B->norm = 10000 * K;
    B->thresh = 10000 * (K - 2); /* MAX_BIAS = 2 (filter.c:18) */
    B->K = K;
    B->kmask = (K >= 32) ? ~0ull : ((1ull << (2 * K)) - 1);
}

/* One scan of read s from p: over [p, q) when the block has a mask track (tracked), else up
 * to the read's 4 terminator.  The two loops differ where growing meets the end: untracked
 * stops, tracked still tests the window s[q-k, q) and keeps it at position q
 * (filter.c:545-551 against 591-592).  There the trim finds the window below 10000 K and
 * stops at once; it would read the base after the segment only for a one-base window, which
 * needs a frequency below 4^-K (the reference then reads past its table; w[4] = 0 here). */
static int64_t bias_scan(const Bias* B, const uint8_t* s, int p, int q, int tracked, int read, KPos* list, int64_t n)
{
    u64 c = 0;
    int a = 0, k = 1;
    while (tracked ? p < q : s[p] != 4)
    {
        int x = s[p];
        a += B->w[x];
        c = (c << 2) | x;
        while (a < B->norm && k < B->K)
        {
            p += 1;
            if (tracked ? p >= q : s[p] == 4)
            {
                if (!tracked)
                    return n;
                break;
            }
            k += 1;
            x = s[p];
            a += B->w[x];
            c = (c << 2) | x;
        }
        /* trim: the window's first base is s[p - k + 1] */
        while (a - B->w[s[p - k + 1]] >= B->norm)
        {
            a -= B->w[s[p - k + 1]];
            k -= 1;
        }
        if (a > B->thresh)
        {
            list[n].code = (c << (2 * (B->K - k))) & B->kmask;
            list[n].read = read;
            list[n].rpos = p;
            n++;
        }
        p += 1;
        a -= B->w[s[p - k]];
    }
    return n;
}

/* All reads in order; the untracked scan needs no segment test, a tracked segment needs
 * K bases (filter.c:533). */
static int64_t extract_biased(const or_block* b, const Bias* B, KPos* list)
{
    int64_t n = 0;
    for (int i = 0; i < b->nreads; i++)
    {
        const uint8_t* s = b->bases + b->boff[i];
        int rlen = b->rlen[i];
        if (!b->mask_anno)
        {
            n = bias_scan(B, s, 0, rlen, 0, i, list, n);
            continue;
        }
        int64_t f0 = b->mask_anno[i], f1 = b->mask_anno[i + 1];
        for (int64_t a = f0; a <= f1; a += 2)
        {
            int p = (a == f0) ? 0 : b->mask_data[a - 1];
            int q = (a == f1) ? rlen : b->mask_data[a];
            if (p + B->K <= q)
                n = bias_scan(B, s, p, q, 1, i, list, n);
        }
    }
    return n;
}

static KPos* build_index(const or_block* b, const or_params* p, int64_t* len)
{
    int K = p->kmer;
    /* a biased scan keeps at most one tuple per position, plus one per segment end */
    int64_t cap = b->totlen + 1 + (p->biased ? b->nreads + (b->mask_anno ? b->mask_anno[b->nreads] : 0) : 0);
    KPos* list = (KPos*)malloc(sizeof(KPos) * (cap + 1));
    int64_t n;
    if (p->biased)
    {
        Bias B;
        bias_tables(p->freq, K, &B);
        n = extract_biased(b, &B, list);
    }
    else
        n = extract_kmers(b, K, list);
    sort_kpos(list, n, (2 * K + 7) / 8); /* mersort bytes (filter.c:713-716) */
    list[n].code = 1ull << (2 * K);      /* Kpowr sentinel (filter.c:796) */
    if (p->suppress > 0 && n > 0)        /* -t: drop codes occurring >= t times (filter.c:645-696) */
    {
        int64_t w = 0, i = 0;
        while (i < n)
        {
            int64_t j = i + 1;
            while (j < n && list[j].code == list[i].code)
                j++;
            if (j - i < p->suppress)
                for (int64_t q = i; q < j; q++)
                    list[w++] = list[q];
            i = j;
        }
        n = w;
        list[n].code = 1ull << (2 * K);
    }
    *len = n;
    return list;
}

int64_t or_sort_kmers(const or_block* b, const or_params* p, uint64_t* code, int32_t* read, int32_t* rpos)
{
    int64_t n;
    KPos* l = build_index(b, p, &n);
    for (int64_t i = 0; i < n; i++)
    {
        code[i] = l[i].code;
        read[i] = l[i].read;
        rpos[i] = l[i].rpos;
    }
    free(l);
    return n;
}

/* ------------------------------------------------------------------------------------ */
/*  A x B merge (count_thread/merge_thread, filter.c:948-1231) + hit sort (2030-2267)    */
/* ------------------------------------------------------------------------------------ */

#define MAXGRAM 10000

typedef struct
{
    int32_t diag, apos, aread, bread;
} Hit;

/* Number of B entries of one code that pair with an A entry of read ar: all of them
 * across blocks, only those with read < ar within a block (or <= / same-read-earlier
 * with -I, filter.c:984-998). */
static int64_t pair_limit(const KPos* bl, int64_t jb, int64_t je, int self, int identity, int comp, int ar, int ap)
{
    int64_t ib = jb;
    if (!self)
        return je;
    if (identity)
    {
        if (comp)
            while (ib < je && bl[ib].read <= ar)
                ib++;
        else
        {
            while (ib < je && bl[ib].read < ar)
                ib++;
            while (ib < je && bl[ib].read == ar && bl[ib].rpos < ap)
                ib++;
        }
    }
    else
        while (ib < je && bl[ib].read < ar)
            ib++;
    return ib;
}

static Hit* merge_hits(const KPos* al, int64_t alen, const KPos* bl, int64_t blen, const or_params* p, int self,
                       int comp, int same_index, int64_t* nhits_out, int* limit_out)
{
    int64_t hist[MAXGRAM];
    memset(hist, 0, sizeof(hist));
    int64_t total = 0;
    /* pass 1: per code product counts (count_thread) */
    int64_t ia = 0, ib = 0;
    while (ia < alen && ib < blen)
    {
        u64 ca = al[ia].code, cb = bl[ib].code;
        if (cb < ca)
        {
            ib++;
            continue;
        }
        if (cb > ca)
        {
            ia++;
            continue;
        }
        int64_t ja = ia, jb = ib;
        while (ia < alen && al[ia].code == ca)
            ia++;
        while (ib < blen && bl[ib].code == cb)
            ib++;
        int64_t ct = 0;
        if (self)
        {
            /* The reference -I self-complement count adds nothing (filter.c:1108-1124); the
             * count pass does add (filter.c:984-998).  Both are restated as they are. */
            for (int64_t a = ja; a < ia; a++)
                ct += pair_limit(bl, jb, ib, 1, p->identity, comp, al[a].read, al[a].rpos) - jb;
        }
        else
            ct = (ia - ja) * (ib - jb);
        total += ct;
        if (ct < MAXGRAM)
            hist[ct]++;
    }
    /* cap from the memory limit (filter.c:2107-2174) */
    int limit;
    if (p->mem_limit > 0)
    {
        int64_t avail;
        u64 dsz = p->mem_limit / 16;
        if (same_index || (int64_t)dsz > alen + 2 * blen)
            avail = ((int64_t)dsz - alen) / 2;
        else
            avail = (int64_t)dsz - (alen + blen);
        avail = (int64_t)(avail * .98);
        int64_t tom = 0;
        int j;
        for (j = 0; j < MAXGRAM; j++)
        {
            tom += j * hist[j];
            if (tom > avail)
                break;
        }
        limit = j;
        if (limit == 1)
        {
            fprintf(stderr, "oracle: insufficient memory limit\n");
            limit = 1;
        }
    }
    else
        limit = INT_MAX;
    *limit_out = limit;

    /* pass 2: emit hits of codes whose count is under the cap (merge_thread) */
    int64_t cap = 0;
    {
        /* exact size: sum of ct over codes with ct < limit */
        int64_t xa = 0, xb = 0;
        while (xa < alen && xb < blen)
        {
            u64 ca = al[xa].code, cb = bl[xb].code;
            if (cb < ca)
            {
                xb++;
                continue;
            }
            if (cb > ca)
            {
                xa++;
                continue;
            }
            int64_t ja = xa, jb = xb;
            while (xa < alen && al[xa].code == ca)
                xa++;
            while (xb < blen && bl[xb].code == cb)
                xb++;
            int64_t ct = 0;
            if (self)
                for (int64_t a = ja; a < xa; a++)
                    ct += pair_limit(bl, jb, xb, 1, p->identity, comp, al[a].read, al[a].rpos) - jb;
            else
                ct = (xa - ja) * (xb - jb);
            if (self && p->identity && comp)
                ; /* merge_thread's -I comp branch never adds to ct: compare ct(=0) < limit */
            if ((self && p->identity && comp ? 0 : ct) < limit)
                cap += ct;
        }
    }
    Hit* hits = (Hit*)malloc(sizeof(Hit) * (cap + 1));
    int64_t nh = 0;
    ia = ib = 0;
    while (ia < alen && ib < blen)
    {
        u64 ca = al[ia].code, cb = bl[ib].code;
        if (cb < ca)
        {
            ib++;
            continue;
        }
        if (cb > ca)
        {
            ia++;
            continue;
        }
        int64_t ja = ia, jb = ib;
        while (ia < alen && al[ia].code == ca)
            ia++;
        while (ib < blen && bl[ib].code == cb)
            ib++;
        int64_t ct = 0;
        if (self)
        {
            if (!(p->identity && comp))
                for (int64_t a = ja; a < ia; a++)
                    ct += pair_limit(bl, jb, ib, 1, p->identity, comp, al[a].read, al[a].rpos) - jb;
        }
        else
            ct = (ia - ja) * (ib - jb);
        if (ct >= limit)
            continue;
        for (int64_t a = ja; a < ia; a++)
        {
            int64_t e = self ? pair_limit(bl, jb, ib, 1, p->identity, comp, al[a].read, al[a].rpos) : ib;
            for (int64_t q = jb; q < e; q++)
            {
                hits[nh].bread = bl[q].read;
                hits[nh].aread = al[a].read;
                hits[nh].apos = al[a].rpos;
                hits[nh].diag = al[a].rpos - bl[q].rpos;
                nh++;
            }
        }
    }
    *nhits_out = nh;
    return hits;
}

static int nbytes_for(int64_t v)
{
    int64_t powr = 1;
    int n = 0;
    while (powr < v)
    {
        powr <<= 8;
        n++;
    }
    return n;
}

/* stable LSD sort of hits on apos, aread, bread bytes (pairsort, filter.c:2030-2054) */
static void sort_hits(Hit* h, int64_t n, int abytes_pos, int abytes_read, int bbytes_read)
{
    Hit* t = (Hit*)malloc(sizeof(Hit) * (n + 1));
    int64_t cnt[256];
    for (int field = 0; field < 3; field++)
    {
        int nb = field == 0 ? abytes_pos : field == 1 ? abytes_read : bbytes_read;
        for (int byte = 0; byte < nb; byte++)
        {
            int sh = 8 * byte;
            memset(cnt, 0, sizeof(cnt));
#define KEYOF(x) ((uint32_t)(field == 0 ? (x).apos : field == 1 ? (x).aread : (x).bread) >> sh & 0xff)
            for (int64_t i = 0; i < n; i++)
                cnt[KEYOF(h[i])]++;
            int64_t s = 0;
            for (int d = 0; d < 256; d++)
            {
                int64_t c = cnt[d];
                cnt[d] = s;
                s += c;
            }
            for (int64_t i = 0; i < n; i++)
                t[cnt[KEYOF(h[i])]++] = h[i];
#undef KEYOF
            memcpy(h, t, sizeof(Hit) * n);
        }
    }
    free(t);
}

static Hit* sorted_hits(const or_block* a, const or_block* b, const KPos* al, int64_t alen, const KPos* bl,
                        int64_t blen, const or_params* p, int self, int comp, int same_index, int64_t* nh,
                        int* limit)
{
    Hit* h = merge_hits(al, alen, bl, blen, p, self, comp, same_index, nh, limit);
    sort_hits(h, *nh, nbytes_for(a->maxlen), nbytes_for(a->nreads), nbytes_for(b->nreads));
    h[*nh].aread = h[*nh].bread = h[*nh].diag = 0x7fffffff; /* sentinel (filter.c:2254-2257) */
    h[*nh].apos = 0;
    return h;
}

int64_t or_match_hits(const or_block* a, const or_block* b, const or_params* p, int self, int32_t** out,
                      int32_t* limit_out)
{
    int64_t alen, blen, nh;
    int limit;
    KPos* al = build_index(a, p, &alen);
    KPos* bl = self ? al : build_index(b, p, &blen);
    if (self)
        blen = alen;
    Hit* h = sorted_hits(a, b, al, alen, bl, blen, p, self, 0, self, &nh, &limit);
    *out = (int32_t*)h;
    *limit_out = limit;
    free(al);
    if (!self)
        free(bl);
    return nh;
}

/* ------------------------------------------------------------------------------------ */
/*  Adaptive wave (forward_wave/reverse_wave/Local_Alignment, align.c:145-2060)          */
/* ------------------------------------------------------------------------------------ */

#define TRIM_LEN 15
#define PATH_LEN 60
#define PATH_TOP 0x1000000000000000ull
#define PATH_INT 0x0fffffffffffffffull
#define TRIM_MASK 0x7fff
#define TRIM_MLAG 200
#define WAVE_LAG 30

static const double Bias_Factor[10] = {.690, .690, .690, .690, .780, .850, .900, .933, .966, 1.000};

typedef struct
{
    int tspace, ave_path;
    int16_t score[TRIM_MASK + 1];
    int16_t table[TRIM_MASK + 1];
} Spec;

/* trim tables (set_table, align.c:196-210) */
static void fill_table(Spec* s, int bit, int prefix, int score, int max, int mscore, int dscore)
{
    if (bit >= TRIM_LEN)
    {
        s->table[prefix] = (int16_t)(score - max);
        s->score[prefix] = (int16_t)score;
    }
    else
    {
        if (score > max)
            max = score;
        fill_table(s, bit + 1, prefix << 1, score - dscore, max, mscore, dscore);
        fill_table(s, bit + 1, (prefix << 1) | 1, score + mscore, max, mscore, dscore);
    }
}

/* New_Align_Spec (align.c:214-279) */
static void make_spec(Spec* s, const or_params* p)
{
    double match = p->freq[0] + p->freq[3];
    if (match > .5)
        match = 1. - match;
    int bias = (int)((match + .025) * 20. - 1.);
    if (match < .2)
        bias = 3;
    s->tspace = p->tspace;
    s->ave_path = (int)(PATH_LEN * (1. - Bias_Factor[bias] * (1. - p->ave_corr)));
    int mscore = (int)(1000 * Bias_Factor[bias] * (1. - p->ave_corr));
    int dscore = 1000 - mscore;
    fill_table(s, 0, 0, 0, 0, mscore, dscore);
}

typedef struct
{
    int ptr, diag, diff, mark;
} Peb;

typedef struct
{
    /* wave vectors indexed by diagonal, valid over [dlo, dhi] */
    int *V, *M, *HA, *HB, *NA, *NB;
    u64* T;
    void* mem;
    int dlo, dhi;
    Peb* cells;
    int64_t ncell, cmax;
    uint16_t* pts; /* trace point buffer: [maxtp | A (2 maxtp) | B ...] */
    int64_t ptsmax;
    int64_t cells_count; /* sum of wave widths (WAVE_STATS TOT, align.c:957-963) */
    int64_t max_width, max_cells, waves, snakes;
} Work;

typedef struct
{
    uint16_t* trace;
    int tlen, diffs, abpos, bbpos, aepos, bepos;
} WPath;

static void work_vectors(Work* w, int lo, int hi)
{
    if (w->mem && lo >= w->dlo && hi <= w->dhi)
        return;
    free(w->mem);
    int span = hi - lo + 1;
    w->mem = malloc((size_t)span * (6 * sizeof(int) + sizeof(u64)));
    u64* T = (u64*)w->mem;
    int* base = (int*)(T + span);
    w->T = T - lo;
    w->V = base - lo;
    w->M = base + span - lo;
    w->HA = base + 2 * span - lo;
    w->HB = base + 3 * span - lo;
    w->NA = base + 4 * span - lo;
    w->NB = base + 5 * span - lo;
    w->dlo = lo;
    w->dhi = hi;
}

static int new_cell(Work* w, int ptr, int diag, int diff, int mark)
{
    if (w->ncell >= w->cmax)
    {
        w->cmax = w->cmax * 2 + 10000;
        w->cells = (Peb*)realloc(w->cells, sizeof(Peb) * w->cmax);
    }
    Peb* c = w->cells + w->ncell;
    c->ptr = ptr;
    c->diag = diag;
    c->diff = diff;
    c->mark = mark;
    return (int)(w->ncell++);
}

#define CHECK_DIAG(k)                                                                 \
    do                                                                                \
    {                                                                                 \
        if ((k) < w->dlo || (k) > w->dhi)                                             \
        {                                                                             \
            fprintf(stderr, "oracle: diagonal %d outside [%d,%d]\n", k, w->dlo, w->dhi); \
            abort();                                                                  \
        }                                                                             \
    } while (0)

/* forward_wave (align.c:369-1110) */
static void fwd_wave(Work* w, const Spec* sp, const uint8_t* aseq, const uint8_t* bseq, int alen, int blen, int comp,
                     WPath* apath, WPath* bpath, int* mind, int maxd, int mida, int minp, int maxp)
{
    int *V = w->V, *M = w->M, *HA = w->HA, *HB = w->HB, *NA = w->NA, *NB = w->NB;
    u64* T = w->T;
    const int TS = sp->tspace, PATH_AVE = sp->ave_path;
    const int16_t *SCORE = sp->score, *TABLE = sp->table;
    int hgh = maxd, low = *mind, dif = 0;
    int boff = comp ? blen % TS : 0;
    int besta, besty, trima, trimy, trimd, trimha, trimhb;
    int morea, morey, mored, moreha, morehb, more, morem, lasta;
    int aclip, bclip;

    w->ncell = 0;
    more = 1;
    aclip = INT32_MAX;
    bclip = -INT32_MAX;
    besta = trima = morea = lasta = mida;
    besty = trimy = morey = (mida - hgh) >> 1;
    trimd = mored = 0;
    trimha = moreha = 0;
    trimhb = morehb = 1;
    morem = -1;

    for (int k = hgh; k >= low; k--)
    {
        CHECK_DIAG(k);
        int y = (mida - k) >> 1, c, d, ha, hb, na, nb;
        const uint8_t* a = aseq + k;
        na = ((y + k) / TS) * TS;
        ha = new_cell(w, -1, k, 0, na);
        na += TS;
        nb = ((y + (TS - boff)) / TS - 1) * TS + boff;
        hb = new_cell(w, -1, k, 0, nb);
        nb += TS;
        while (1)
        {
            c = bseq[y];
            if (c == 4)
            {
                more = 0;
                if (bclip < k)
                    bclip = k;
                break;
            }
            d = a[y];
            if (c != d)
            {
                if (d == 4)
                {
                    more = 0;
                    aclip = k;
                }
                break;
            }
            y += 1;
        }
        c = (y << 1) + k;
        while (y + k >= na)
        {
            ha = new_cell(w, ha, k, 0, na);
            na += TS;
        }
        while (y >= nb)
        {
            hb = new_cell(w, hb, k, 0, nb);
            nb += TS;
        }
        if (c > besta)
        {
            besta = trima = lasta = c;
            besty = trimy = y;
            trimha = ha;
            trimhb = hb;
        }
        V[k] = c;
        T[k] = PATH_INT;
        M[k] = PATH_LEN;
        HA[k] = ha;
        HB[k] = hb;
        NA[k] = na;
        NB[k] = nb;
    }

    if (more == 0)
    {
        if (bseq[besty] != 4 && aseq[besta - besty] != 4)
            more = 1;
        if (hgh >= aclip)
        {
            hgh = aclip - 1;
            if (morem <= M[aclip])
            {
                morem = M[aclip];
                morea = V[aclip];
                morey = (morea - aclip) / 2;
                moreha = HA[aclip];
                morehb = HB[aclip];
            }
        }
        if (low <= bclip)
        {
            low = bclip + 1;
            if (morem <= M[bclip])
            {
                morem = M[bclip];
                morea = V[bclip];
                morey = (morea - bclip) / 2;
                moreha = HA[bclip];
                morehb = HB[bclip];
            }
        }
        aclip = INT32_MAX;
        bclip = -INT32_MAX;
    }

    while (more && lasta >= besta - TRIM_MLAG)
    {
        int k, n, ua, ub, am, ac, ap;
        u64 t;
        low -= 1;
        hgh += 1;
        CHECK_DIAG(low - 1);
        CHECK_DIAG(hgh + 1);
        if (low >= minp)
        {
            NA[low] = NA[low + 1];
            NB[low] = NB[low + 1];
            V[low] = -1;
        }
        else
            low += 1;
        if (hgh <= maxp)
        {
            NA[hgh] = NA[hgh - 1];
            NB[hgh] = NB[hgh - 1];
            V[hgh] = am = -1;
        }
        else
            am = V[--hgh];
        dif += 1;
        ac = V[hgh + 1] = V[low - 1] = -1;
        t = PATH_INT;
        n = PATH_LEN;
        ua = ub = -1;
        for (k = hgh; k >= low; k--)
        {
            int y, m, ha, hb, c, d;
            u64 b;
            const uint8_t* a = aseq + k;
            ap = ac;
            ac = am;
            am = V[d = k - 1];
            if (ac < am)
                if (am < ap)
                {
                    c = ap + 1;
                    m = n;
                    b = t;
                    ha = ua;
                    hb = ub;
                }
                else
                {
                    c = am + 1;
                    m = M[d];
                    b = T[d];
                    ha = HA[d];
                    hb = HB[d];
                }
            else if (ac < ap)
            {
                c = ap + 1;
                m = n;
                b = t;
                ha = ua;
                hb = ub;
            }
            else
            {
                c = ac + 2;
                m = M[k];
                b = T[k];
                ha = HA[k];
                hb = HB[k];
            }
            if ((b & PATH_TOP) != 0)
                m -= 1;
            b <<= 1;
            y = (c - k) >> 1;
            while (1)
            {
                c = bseq[y];
                if (c == 4)
                {
                    more = 0;
                    if (bclip < k)
                        bclip = k;
                    break;
                }
                d = a[y];
                if (c != d)
                {
                    if (d == 4)
                    {
                        more = 0;
                        aclip = k;
                    }
                    break;
                }
                y += 1;
                w->snakes++;
                if ((b & PATH_TOP) == 0)
                    m += 1;
                b = (b << 1) | 1;
            }
            c = (y << 1) + k;
            while (y + k >= NA[k])
            {
                if (w->cells[ha].mark < NA[k])
                    ha = new_cell(w, ha, k, dif, NA[k]);
                NA[k] += TS;
            }
            while (y >= NB[k])
            {
                if (w->cells[hb].mark < NB[k])
                    hb = new_cell(w, hb, k, dif, NB[k]);
                NB[k] += TS;
            }
            if (c > besta)
            {
                besta = c;
                besty = y;
                if (m >= PATH_AVE)
                {
                    lasta = c;
                    if (TABLE[b & TRIM_MASK] >= 0)
                        if (TABLE[(b >> TRIM_LEN) & TRIM_MASK] + SCORE[b & TRIM_MASK] >= 0)
                        {
                            trima = c;
                            trimy = y;
                            trimd = dif;
                            trimha = ha;
                            trimhb = hb;
                        }
                }
            }
            t = T[k];
            n = M[k];
            ua = HA[k];
            ub = HB[k];
            V[k] = c;
            T[k] = b;
            M[k] = m;
            HA[k] = ha;
            HB[k] = hb;
        }
        if (more == 0)
        {
            if (bseq[besty] != 4 && aseq[besta - besty] != 4)
                more = 1;
            if (hgh >= aclip)
            {
                hgh = aclip - 1;
                if (morem <= M[aclip])
                {
                    morem = M[aclip];
                    morea = V[aclip];
                    morey = (morea - aclip) / 2;
                    mored = dif;
                    moreha = HA[aclip];
                    morehb = HB[aclip];
                }
            }
            if (low <= bclip)
            {
                low = bclip + 1;
                if (morem <= M[bclip])
                {
                    morem = M[bclip];
                    morea = V[bclip];
                    morey = (morea - bclip) / 2;
                    mored = dif;
                    moreha = HA[bclip];
                    morehb = HB[bclip];
                }
            }
            aclip = INT32_MAX;
            bclip = -INT32_MAX;
        }
        n = besta - WAVE_LAG;
        while (hgh >= low)
            if (V[hgh] < n)
                hgh -= 1;
            else
            {
                while (V[low] < n)
                    low += 1;
                break;
            }
        w->cells_count += (hgh - low) + 1;
        w->waves++;
        if (hgh - low + 1 > w->max_width) w->max_width = hgh - low + 1;
        if (w->ncell > w->max_cells) w->max_cells = w->ncell;
    }

    {
        uint16_t* atrace = apath->trace;
        uint16_t* btrace = bpath->trace;
        Peb* cells = w->cells;
        int atlen = 0, btlen = 0, trimx, a, b, k, h, d, e;
        if (morem >= 0)
        {
            trimx = morea - morey;
            trimy = morey;
            trimd = mored;
            trimha = moreha;
            trimhb = morehb;
        }
        else
            trimx = trima - trimy;

        a = -1;
        for (h = trimha; h >= 0; h = b)
        {
            b = cells[h].ptr;
            cells[h].ptr = a;
            a = h;
        }
        h = a;
        k = cells[h].diag;
        b = (mida - k) / 2;
        e = 0;
        for (h = cells[h].ptr; h >= 0; h = cells[h].ptr)
        {
            k = cells[h].diag;
            a = cells[h].mark - k;
            d = cells[h].diff;
            atrace[atlen++] = (uint16_t)(d - e);
            atrace[atlen++] = (uint16_t)(a - b);
            b = a;
            e = d;
        }
        if (b + k != trimx)
        {
            atrace[atlen++] = (uint16_t)(trimd - e);
            atrace[atlen++] = (uint16_t)(trimy - b);
        }
        else if (b != trimy)
        {
            atrace[atlen - 1] = (uint16_t)(atrace[atlen - 1] + (trimy - b));
            atrace[atlen - 2] = (uint16_t)(atrace[atlen - 2] + (trimd - e));
        }

        a = -1;
        for (h = trimhb; h >= 0; h = b)
        {
            b = cells[h].ptr;
            cells[h].ptr = a;
            a = h;
        }
        h = a;
        k = cells[h].diag;
        b = (mida + k) / 2;
        e = 0;
        low = k;
        for (h = cells[h].ptr; h >= 0; h = cells[h].ptr)
        {
            k = cells[h].diag;
            a = cells[h].mark + k;
            d = cells[h].diff;
            btrace[btlen++] = (uint16_t)(d - e);
            btrace[btlen++] = (uint16_t)(a - b);
            b = a;
            e = d;
        }
        if (b - k != trimy)
        {
            btrace[btlen++] = (uint16_t)(trimd - e);
            btrace[btlen++] = (uint16_t)(trimx - b);
        }
        else if (b != trimx)
        {
            btrace[btlen - 1] = (uint16_t)(btrace[btlen - 1] + (trimx - b));
            btrace[btlen - 2] = (uint16_t)(btrace[btlen - 2] + (trimd - e));
        }

        apath->aepos = trimx;
        apath->bepos = trimy;
        apath->diffs = trimd;
        apath->tlen = atlen;
        if (comp)
        {
            bpath->abpos = blen - apath->bepos;
            bpath->bbpos = alen - apath->aepos;
        }
        else
        {
            bpath->aepos = apath->bepos;
            bpath->bepos = apath->aepos;
        }
        bpath->diffs = trimd;
        bpath->tlen = btlen;
    }
    *mind = low;
}

/* reverse_wave (align.c:1114-1916) */
static void rev_wave(Work* w, const Spec* sp, const uint8_t* aseq0, const uint8_t* bseq0, int alen, int blen, int comp,
                     WPath* apath, WPath* bpath, int mind, int maxd, int mida, int minp, int maxp)
{
    const uint8_t* aseq = aseq0 - 1;
    const uint8_t* bseq = bseq0 - 1;
    int *V = w->V, *M = w->M, *HA = w->HA, *HB = w->HB, *NA = w->NA, *NB = w->NB;
    u64* T = w->T;
    const int TS = sp->tspace, PATH_AVE = sp->ave_path;
    const int16_t *SCORE = sp->score, *TABLE = sp->table;
    int hgh = maxd, low = mind, dif = 0;
    int boff = comp ? blen % TS : 0;
    int besta, besty, trima, trimy, trimd, trimha, trimhb;
    int morea, morey, mored, moreha, morehb, more, morem, lasta;
    int aclip, bclip;

    w->ncell = 0;
    more = 1;
    aclip = -INT32_MAX;
    bclip = INT32_MAX;
    besta = trima = morea = lasta = mida;
    besty = trimy = morey = (mida - hgh) >> 1;
    trimd = mored = 0;
    trimha = moreha = 0;
    trimhb = morehb = 1;
    morem = -1;

    for (int k = low; k <= hgh; k++)
    {
        CHECK_DIAG(k);
        int y = (mida - k) >> 1, c, d, ha, hb, na, nb;
        const uint8_t* a = aseq + k;
        na = ((y + k + TS - 1) / TS - 1) * TS;
        ha = new_cell(w, -1, k, 0, y + k);
        nb = ((y + (TS - boff) - 1) / TS - 1) * TS + boff;
        hb = new_cell(w, -1, k, 0, y);
        while (1)
        {
            c = bseq[y];
            if (c == 4)
            {
                more = 0;
                if (bclip > k)
                    bclip = k;
                break;
            }
            d = a[y];
            if (c != d)
            {
                if (d == 4)
                {
                    more = 0;
                    aclip = k;
                }
                break;
            }
            y -= 1;
        }
        c = (y << 1) + k;
        while (y + k <= na)
        {
            ha = new_cell(w, ha, k, 0, na);
            na -= TS;
        }
        while (y <= nb)
        {
            hb = new_cell(w, hb, k, 0, nb);
            nb -= TS;
        }
        if (c < besta)
        {
            besta = trima = lasta = c;
            besty = trimy = y;
            trimha = ha;
            trimhb = hb;
        }
        V[k] = c;
        T[k] = PATH_INT;
        M[k] = PATH_LEN;
        HA[k] = ha;
        HB[k] = hb;
        NA[k] = na;
        NB[k] = nb;
    }

    if (more == 0)
    {
        if (bseq[besty] != 4 && aseq[besta - besty] != 4)
            more = 1;
        if (low <= aclip)
        {
            low = aclip + 1;
            if (morem <= M[aclip])
            {
                morem = M[aclip];
                morea = V[aclip];
                morey = (morea - aclip) / 2;
                moreha = HA[aclip];
                morehb = HB[aclip];
            }
        }
        if (hgh >= bclip)
        {
            hgh = bclip - 1;
            if (morem <= M[bclip])
            {
                morem = M[bclip];
                morea = V[bclip];
                morey = (morea - bclip) / 2;
                moreha = HA[bclip];
                morehb = HB[bclip];
            }
        }
        aclip = -INT32_MAX;
        bclip = INT32_MAX;
    }

    while (more && lasta <= besta + TRIM_MLAG)
    {
        int k, n, ua, ub, am, ac, ap;
        u64 t;
        low -= 1;
        hgh += 1;
        CHECK_DIAG(low - 1);
        CHECK_DIAG(hgh + 1);
        if (low >= minp)
        {
            NA[low] = NA[low + 1];
            NB[low] = NB[low + 1];
            V[low] = ap = INT32_MAX;
        }
        else
            ap = V[++low];
        if (hgh <= maxp)
        {
            NA[hgh] = NA[hgh - 1];
            NB[hgh] = NB[hgh - 1];
            V[hgh] = INT32_MAX;
        }
        else
            hgh -= 1;
        dif += 1;
        ac = V[hgh + 1] = V[low - 1] = INT32_MAX;
        t = PATH_INT;
        n = PATH_LEN;
        ua = ub = -1;
        for (k = low; k <= hgh; k++)
        {
            int y, m, ha, hb, c, d;
            u64 b;
            const uint8_t* a = aseq + k;
            am = ac;
            ac = ap;
            ap = V[d = k + 1];
            if (ac > ap)
                if (ap > am)
                {
                    c = am - 1;
                    m = n;
                    b = t;
                    ha = ua;
                    hb = ub;
                }
                else
                {
                    c = ap - 1;
                    m = M[d];
                    b = T[d];
                    ha = HA[d];
                    hb = HB[d];
                }
            else if (ac > am)
            {
                c = am - 1;
                m = n;
                b = t;
                ha = ua;
                hb = ub;
            }
            else
            {
                c = ac - 2;
                m = M[k];
                b = T[k];
                ha = HA[k];
                hb = HB[k];
            }
            if ((b & PATH_TOP) != 0)
                m -= 1;
            b <<= 1;
            y = (c - k) >> 1;
            while (1)
            {
                c = bseq[y];
                if (c == 4)
                {
                    more = 0;
                    if (bclip > k)
                        bclip = k;
                    break;
                }
                d = a[y];
                if (c != d)
                {
                    if (d == 4)
                    {
                        more = 0;
                        aclip = k;
                    }
                    break;
                }
                y -= 1;
                if ((b & PATH_TOP) == 0)
                    m += 1;
                b = (b << 1) | 1;
            }
            c = (y << 1) + k;
            while (y + k <= NA[k])
            {
                if (w->cells[ha].mark > NA[k])
                    ha = new_cell(w, ha, k, dif, NA[k]);
                NA[k] -= TS;
            }
            while (y <= NB[k])
            {
                if (w->cells[hb].mark > NB[k])
                    hb = new_cell(w, hb, k, dif, NB[k]);
                NB[k] -= TS;
            }
            if (c < besta)
            {
                besta = c;
                besty = y;
                if (m >= PATH_AVE)
                {
                    lasta = c;
                    if (TABLE[b & TRIM_MASK] >= 0)
                        if (TABLE[(b >> TRIM_LEN) & TRIM_MASK] + SCORE[b & TRIM_MASK] >= 0)
                        {
                            trima = c;
                            trimy = y;
                            trimd = dif;
                            trimha = ha;
                            trimhb = hb;
                        }
                }
            }
            t = T[k];
            n = M[k];
            ua = HA[k];
            ub = HB[k];
            V[k] = c;
            T[k] = b;
            M[k] = m;
            HA[k] = ha;
            HB[k] = hb;
        }
        if (more == 0)
        {
            if (bseq[besty] != 4 && aseq[besta - besty] != 4)
                more = 1;
            if (low <= aclip)
            {
                low = aclip + 1;
                if (morem <= M[aclip])
                {
                    morem = M[aclip];
                    morea = V[aclip];
                    morey = (morea - aclip) / 2;
                    mored = dif;
                    moreha = HA[aclip];
                    morehb = HB[aclip];
                }
            }
            if (hgh >= bclip)
            {
                hgh = bclip - 1;
                if (morem <= M[bclip])
                {
                    morem = M[bclip];
                    morea = V[bclip];
                    morey = (morea - bclip) / 2;
                    mored = dif;
                    moreha = HA[bclip];
                    morehb = HB[bclip];
                }
            }
            aclip = -INT32_MAX;
            bclip = INT32_MAX;
        }
        n = besta + WAVE_LAG;
        while (hgh >= low)
            if (V[hgh] > n)
                hgh -= 1;
            else
            {
                while (V[low] > n)
                    low += 1;
                break;
            }
        w->cells_count += (hgh - low) + 1;
        w->waves++;
        if (hgh - low + 1 > w->max_width) w->max_width = hgh - low + 1;
        if (w->ncell > w->max_cells) w->max_cells = w->ncell;
    }

    {
        uint16_t* atrace = apath->trace;
        uint16_t* btrace = bpath->trace;
        Peb* cells = w->cells;
        int atlen = 0, btlen = 0, trimx, a, b, k, h, d, e;
        if (morem >= 0)
        {
            trimx = morea - morey;
            trimy = morey;
            trimd = mored;
            trimha = moreha;
            trimhb = morehb;
        }
        else
            trimx = trima - trimy;

        a = -1;
        for (h = trimha; h >= 0; h = b)
        {
            b = cells[h].ptr;
            cells[h].ptr = a;
            a = h;
        }
        h = a;
        k = cells[h].diag;
        b = cells[h].mark - k;
        e = 0;
        if ((b + k) % TS != 0)
        {
            h = cells[h].ptr;
            if (h < 0)
            {
                a = trimy;
                d = trimd;
            }
            else
            {
                k = cells[h].diag;
                a = cells[h].mark - k;
                d = cells[h].diff;
            }
            if (apath->tlen == 0)
            {
                atrace[--atlen] = (uint16_t)(b - a);
                atrace[--atlen] = (uint16_t)(d - e);
            }
            else
            {
                atrace[1] = (uint16_t)(atrace[1] + (b - a));
                atrace[0] = (uint16_t)(atrace[0] + (d - e));
            }
            b = a;
            e = d;
        }
        if (h >= 0)
        {
            for (h = cells[h].ptr; h >= 0; h = cells[h].ptr)
            {
                k = cells[h].diag;
                a = cells[h].mark - k;
                atrace[--atlen] = (uint16_t)(b - a);
                d = cells[h].diff;
                atrace[--atlen] = (uint16_t)(d - e);
                b = a;
                e = d;
            }
            if (b + k != trimx)
            {
                atrace[--atlen] = (uint16_t)(b - trimy);
                atrace[--atlen] = (uint16_t)(trimd - e);
            }
            else if (b != trimy)
            {
                atrace[atlen + 1] = (uint16_t)(atrace[atlen + 1] + (b - trimy));
                atrace[atlen] = (uint16_t)(atrace[atlen] + (trimd - e));
            }
        }

        a = -1;
        for (h = trimhb; h >= 0; h = b)
        {
            b = cells[h].ptr;
            cells[h].ptr = a;
            a = h;
        }
        h = a;
        k = cells[h].diag;
        b = cells[h].mark + k;
        e = 0;
        if ((b - k) % TS != boff)
        {
            h = cells[h].ptr;
            if (h < 0)
            {
                a = trimx;
                d = trimd;
            }
            else
            {
                k = cells[h].diag;
                a = cells[h].mark + k;
                d = cells[h].diff;
            }
            if (bpath->tlen == 0)
            {
                btrace[--btlen] = (uint16_t)(b - a);
                btrace[--btlen] = (uint16_t)(b - a); /* sic: the reference stores b-a twice here */
            }
            else
            {
                btrace[1] = (uint16_t)(btrace[1] + (b - a));
                btrace[0] = (uint16_t)(btrace[0] + (d - e));
            }
            b = a;
            e = d;
        }
        if (h >= 0)
        {
            for (h = cells[h].ptr; h >= 0; h = cells[h].ptr)
            {
                k = cells[h].diag;
                a = cells[h].mark + k;
                btrace[--btlen] = (uint16_t)(b - a);
                d = cells[h].diff;
                btrace[--btlen] = (uint16_t)(d - e);
                b = a;
                e = d;
            }
            if (b - k != trimy)
            {
                btrace[--btlen] = (uint16_t)(b - trimx);
                btrace[--btlen] = (uint16_t)(trimd - e);
            }
            else if (b != trimx)
            {
                btrace[btlen + 1] = (uint16_t)(btrace[btlen + 1] + (b - trimx));
                btrace[btlen] = (uint16_t)(btrace[btlen] + (trimd - e));
            }
        }

        apath->abpos = trimx;
        apath->bbpos = trimy;
        apath->diffs = apath->diffs + trimd;
        apath->tlen = apath->tlen - atlen;
        apath->trace = atrace + atlen;
        if (comp)
        {
            bpath->aepos = blen - apath->bbpos;
            bpath->bepos = alen - apath->abpos;
        }
        else
        {
            bpath->abpos = apath->bbpos;
            bpath->bbpos = apath->abpos;
        }
        bpath->diffs = bpath->diffs + trimd;
        bpath->tlen = bpath->tlen - btlen;
        bpath->trace = btrace + btlen;
    }
}

/* Local_Alignment (align.c:1922-2060) for daligner's use: a single start diagonal,
 * no borders (lbord = hbord = -1). */
static void local_alignment(Work* w, const Spec* sp, const uint8_t* aseq, const uint8_t* bseq, int alen, int blen,
                            int comp, int diag, int anti, WPath* apath, WPath* bpath)
{
    int low = diag, hgh = diag, minp, maxp;
    int maxtp = 2 * (((alen < blen) ? blen : alen) / sp->tspace + 2);
    if (w->ptsmax < 4 * maxtp + 8)
    {
        w->ptsmax = 4 * maxtp + 8;
        free(w->pts);
        w->pts = (uint16_t*)calloc(w->ptsmax, sizeof(uint16_t));
    }
    apath->trace = w->pts + maxtp;
    bpath->trace = apath->trace + 2 * maxtp;
    work_vectors(w, -(blen + 8), alen + 8);

    int selfie = (aseq == bseq);
    minp = (selfie && low >= 0) ? 1 : -INT32_MAX;
    maxp = (selfie && hgh <= 0) ? -1 : INT32_MAX;

    fwd_wave(w, sp, aseq, bseq, alen, blen, comp, apath, bpath, &low, hgh, anti, minp, maxp);
    rev_wave(w, sp, aseq, bseq, alen, blen, comp, apath, bpath, low, low, anti, minp, maxp);

    if (comp)
    {
        uint16_t* tr = bpath->trace;
        int i = bpath->tlen - 2, j = 0;
        while (j < i)
        {
            uint16_t p = tr[i];
            tr[i] = tr[j];
            tr[j] = p;
            p = tr[i + 1];
            tr[i + 1] = tr[j + 1];
            tr[j + 1] = p;
            i -= 2;
            j += 2;
        }
    }
}

int or_local_alignment(const uint8_t* aseq, const uint8_t* bseq, int alen, int blen, int comp, int diag, int anti,
                       const or_params* p, int32_t* out, uint16_t* atrace, uint16_t* btrace, int64_t* cells)
{
    Spec sp;
    Work w;
    WPath ap, bp;
    memset(&w, 0, sizeof(w));
    memset(&ap, 0, sizeof(ap));
    memset(&bp, 0, sizeof(bp));
    make_spec(&sp, p);
    local_alignment(&w, &sp, aseq, bseq, alen, blen, comp, diag, anti, &ap, &bp);
    WPath* ps[2] = {&ap, &bp};
    for (int i = 0; i < 2; i++)
    {
        out[6 * i + 0] = ps[i]->abpos;
        out[6 * i + 1] = ps[i]->bbpos;
        out[6 * i + 2] = ps[i]->aepos;
        out[6 * i + 3] = ps[i]->bepos;
        out[6 * i + 4] = ps[i]->diffs;
        out[6 * i + 5] = ps[i]->tlen;
    }
    memcpy(atrace, ap.trace, sizeof(uint16_t) * ap.tlen);
    memcpy(btrace, bp.trace, sizeof(uint16_t) * bp.tlen);
    if (cells)
        *cells = w.cells_count;
    free(w.mem);
    free(w.cells);
    free(w.pts);
    return 0;
}

/* ------------------------------------------------------------------------------------ */
/*  Seed scan and overlap assembly (report_thread & co, filter.c:1249-1989)              */
/* ------------------------------------------------------------------------------------ */

#define PANEL_SIZE 50000
#define PANEL_OVERLAP 10000

typedef struct
{
    int64_t toff; /* offset into the pair trace buffer */
    int tlen, diffs, abpos, bbpos, aepos, bepos;
} MPath;

typedef struct
{
    uint16_t* tr;
    int64_t top, max;
} TBuf;

static void tbuf_reserve(TBuf* t, int64_t extra)
{
    if (t->top + extra >= t->max)
    {
        t->max = (t->top + extra) * 2 + 1000;
        t->tr = (uint16_t*)realloc(t->tr, sizeof(uint16_t) * t->max);
    }
}

/* Entwine (filter.c:1249-1342).  d2: daligner2's version (dalign2/filter.c:1707-1825),
 * which also compares the B coordinates at a common start and a common end point. */
static int entwine(MPath* jpath, MPath* kpath, TBuf* tb, int TS, int* where, int d2)
{
    int ac, b2, y2, ae, i, j, k, num = 0, den = 0, min = 10000;
    uint16_t* ktrace = tb->tr + kpath->toff;
    uint16_t* jtrace = tb->tr + jpath->toff;
    y2 = jpath->bbpos;
    j = jpath->abpos / TS;
    b2 = kpath->bbpos;
    k = kpath->abpos / TS;
    if (d2 && jpath->abpos == kpath->abpos)
    {
        min = abs(y2 - b2);
        if (min == 0)
            *where = kpath->abpos;
    }
    if (j < k)
    {
        ac = k * TS;
        j = 1 + 2 * (k - j);
        k = 1;
        for (i = 1; i < j; i += 2)
            y2 += jtrace[i];
    }
    else
    {
        ac = j * TS;
        k = 1 + 2 * (j - k);
        j = 1;
        for (i = 1; i < k; i += 2)
            b2 += ktrace[i];
    }
    ae = jpath->aepos;
    if (ae > kpath->aepos)
        ae = kpath->aepos;
    while (1)
    {
        ac += TS;
        if (ac >= ae)
            break;
        y2 += jtrace[j];
        b2 += ktrace[k];
        j += 2;
        k += 2;
        i = abs(y2 - b2);
        if (i <= min)
        {
            min = i;
            if (i == 0)
                *where = ac;
        }
        num += i;
        den += 1;
    }
    if (d2 && jpath->aepos == kpath->aepos)
    {
        i = abs(jpath->bepos - kpath->bepos);
        if (i <= min)
        {
            min = i;
            if (i == 0)
                *where = kpath->aepos;
        }
    }
    return den == 0 ? -1 : min;
}

/* Fusion (filter.c:1347-1401) */
static void fusion(MPath* p1, int ap, MPath* p2, TBuf* tb, int TS)
{
    int k1 = 2 * ((ap / TS) - (p1->abpos / TS));
    int k2 = 2 * ((ap / TS) - (p2->abpos / TS));
    int len = k1 + (p2->tlen - k2), diff = 0, k;
    tbuf_reserve(tb, len);
    int64_t base = tb->top;
    tb->top += len;
    uint16_t* trace = tb->tr + base;
    len = 0;
    if (k1 > 0)
    {
        uint16_t* t = tb->tr + p1->toff;
        for (k = 0; k < k1; k += 2)
        {
            trace[len++] = t[k];
            trace[len++] = t[k + 1];
            diff += t[k];
        }
    }
    if (k2 < p2->tlen)
    {
        uint16_t* t = tb->tr + p2->toff;
        for (k = k2; k < p2->tlen; k += 2)
        {
            trace[len++] = t[k];
            trace[len++] = t[k + 1];
            diff += t[k];
        }
    }
    p1->aepos = p2->aepos;
    p1->bepos = p2->bepos;
    p1->diffs = diff;
    p1->toff = base;
    p1->tlen = len;
}

/* Handle_Redundancies (filter.c:1403-1566) */
static int handle_redundancies(MPath* amatch, int novls, MPath* bmatch, TBuf* tb, int TS, int comp)
{
    int j, k, no = 0, dist, awhen = 0, bwhen = 0;
    int hasB = (bmatch != NULL);
    for (j = 1; j < novls; j++)
    {
        MPath* jpath = amatch + j;
        for (k = no; k >= 0; k--)
        {
            MPath* kpath = amatch + k;
            if (jpath->abpos < kpath->abpos)
            {
                if (kpath->abpos <= jpath->aepos && kpath->bbpos <= jpath->bepos)
                {
                    dist = entwine(jpath, kpath, tb, TS, &awhen, 0);
                    if (dist == 0)
                    {
                        if (kpath->aepos > jpath->aepos)
                        {
                            if (hasB)
                            {
                                if (comp)
                                {
                                    dist = entwine(bmatch + k, bmatch + j, tb, TS, &bwhen, 0);
                                    if (dist != 0)
                                        continue;
                                    fusion(jpath, awhen, kpath, tb, TS);
                                    amatch[k] = *jpath;
                                    fusion(bmatch + k, bwhen, bmatch + j, tb, TS);
                                }
                                else
                                {
                                    dist = entwine(bmatch + j, bmatch + k, tb, TS, &bwhen, 0);
                                    if (dist != 0)
                                        continue;
                                    fusion(jpath, awhen, kpath, tb, TS);
                                    amatch[k] = *jpath;
                                    fusion(bmatch + j, bwhen, bmatch + k, tb, TS);
                                    bmatch[k] = bmatch[j];
                                }
                            }
                            else
                            {
                                fusion(jpath, awhen, kpath, tb, TS);
                                amatch[k] = *jpath;
                            }
                        }
                        else
                        {
                            amatch[k] = *jpath;
                            if (hasB)
                                bmatch[k] = bmatch[j];
                        }
                        break;
                    }
                }
            }
            else
            {
                if (jpath->abpos <= kpath->aepos && jpath->bbpos <= kpath->bepos)
                {
                    dist = entwine(kpath, jpath, tb, TS, &awhen, 0);
                    if (dist == 0)
                    {
                        if (kpath->abpos == jpath->abpos)
                        {
                            if (kpath->aepos < jpath->aepos)
                            {
                                amatch[k] = *jpath;
                                if (hasB)
                                    bmatch[k] = bmatch[j];
                            }
                        }
                        else if (jpath->aepos > kpath->aepos)
                        {
                            if (hasB)
                            {
                                if (comp)
                                {
                                    dist = entwine(bmatch + j, bmatch + k, tb, TS, &bwhen, 0);
                                    if (dist != 0)
                                        continue;
                                    fusion(kpath, awhen, jpath, tb, TS);
                                    fusion(bmatch + j, bwhen, bmatch + k, tb, TS);
                                    bmatch[k] = bmatch[j];
                                }
                                else
                                {
                                    dist = entwine(bmatch + k, bmatch + j, tb, TS, &bwhen, 0);
                                    if (dist != 0)
                                        continue;
                                    fusion(kpath, awhen, jpath, tb, TS);
                                    fusion(bmatch + k, bwhen, bmatch + j, tb, TS);
                                }
                            }
                            else
                                fusion(kpath, awhen, jpath, tb, TS);
                        }
                        break;
                    }
                }
            }
        }
        if (k < 0)
        {
            no += 1;
            amatch[no] = *jpath;
            if (hasB)
                bmatch[no] = bmatch[j];
        }
    }
    return no + 1;
}

/* ---- daligner2 bridging (DO_BRIDGING, dalign2/filter.c:1479-1705, 2124-2262) ---------- */

/* split_nd (dalign2/align.c:4355-4523): bidirectional O(nd) waves over A[0,M) x B[0,N) until
 * they meet; returns the edit distance D and the meeting point (x, y).  VF/VB as the
 * reference places them in its vector (Compute_Alignment, :4815-4826). */
static int split_nd(const uint8_t* A, int M, const uint8_t* B, int N, int* VF, int* VB, int* px, int* py)
{
    int x, y, D, flow, blow, bhgh;
    const uint8_t* a;
    y = 0;
    if (N < M)
        while (y < N && B[y] == A[y])
            y += 1;
    else
    {
        while (y < M && B[y] == A[y])
            y += 1;
        if (y >= M && N == M)
        {
            *px = *py = M;
            return 0;
        }
    }
    flow = 0;
    VF[0] = y;
    VF[-1] = -2;
    x = N - M;
    a = A - x;
    y = N - 1;
    if (N > M)
        while (y >= x && B[y] == a[y])
            y -= 1;
    else
        while (y >= 0 && B[y] == a[y])
            y -= 1;
    blow = bhgh = -x;
    VB += x;
    VB[blow] = y;
    VB[blow - 1] = N + 1;
    for (D = 1;; D += 1)
    {
        int k, r, am, ac, ap;
        flow -= 1;
        am = ac = VF[flow - 1] = -2;
        a = A + D;
        x = M - D;
        for (k = D; k >= flow; k--)
        {
            ap = ac;
            ac = am + 1;
            am = VF[k - 1];
            if (ac < am)
                y = (ap < am) ? am : ap;
            else
                y = (ap < ac) ? ac : ap;
            if (blow <= k && k <= bhgh)
            {
                r = VB[k];
                if (y > r)
                {
                    D = (D << 1) - 1;
                    if (ap > r)
                        y = ap;
                    else if (ac > r)
                        y = ac;
                    else
                        y = r + 1;
                    *px = k + y;
                    *py = y;
                    return D;
                }
            }
            if (N < x)
                while (y < N && B[y] == a[y])
                    y += 1;
            else
                while (y < x && B[y] == a[y])
                    y += 1;
            VF[k] = y;
            a -= 1;
            x += 1;
        }
        bhgh += 1;
        blow -= 1;
        am = ac = VB[blow - 1] = N + 1;
        a = A + bhgh;
        x = -bhgh;
        for (k = bhgh; k >= blow; k--)
        {
            ap = ac + 1;
            ac = am;
            am = VB[k - 1];
            if (ac > am)
                y = (ap > am) ? am : ap;
            else
                y = (ap > ac) ? ac : ap;
            if (flow <= k && k <= D)
            {
                r = VF[k];
                if (y <= r)
                {
                    D = (D << 1);
                    if (ap <= r)
                        y = ap;
                    else if (ac <= r)
                        y = ac;
                    else
                        y = r;
                    *px = k + y;
                    *py = y;
                    return D;
                }
            }
            y -= 1;
            if (x > 0)
                while (y >= x && B[y] == a[y])
                    y -= 1;
            else
                while (y >= 0 && B[y] == a[y])
                    y -= 1;
            VB[k] = y;
            a -= 1;
            x += 1;
        }
    }
}

typedef struct
{
    const uint8_t* Aabs;
    uint16_t* Trace; /* indexed by 2 * (absolute A position / tspace) */
    int *VF, *VB;
} TWave;

/* trace_nd (dalign2/align.c:4525-4679): the trace-point counts (diffs, b-advance) of an
 * optimal alignment of A[0,M) x B[0,N), split at midpoints until a piece lies inside one
 * trace interval.  Every update is an addition, so the order of the pieces is free. */
static int trace_nd(const uint8_t* A, int M, const uint8_t* B, int N, TWave* w, int tspace)
{
    int x, y, D, s;
    if (M <= 0)
    {
        y = (int)(((A - w->Aabs) / tspace) << 1);
        w->Trace[y] += N;
        w->Trace[y + 1] += N;
        return N;
    }
    if (N <= 0)
    {
        x = (int)(A - w->Aabs);
        y = x / tspace;
        x = (y + 1) * tspace - x;
        y <<= 1;
        for (s = M; s > 0; s -= x, x = tspace)
        {
            if (x > s)
                x = s;
            w->Trace[y] += x;
            y += 2;
        }
        return M;
    }
    D = split_nd(A, M, B, N, w->VF, w->VB, &x, &y);
    if (D > 1)
    {
        s = (int)(A - w->Aabs);
        if ((s / tspace + 1) * tspace - s >= x)
        {
            s = ((s / tspace) << 1);
            w->Trace[s] += (D + 1) / 2;
            w->Trace[s + 1] += y;
        }
        else
            trace_nd(A, x, B, y, w, tspace);
        s = (int)((A + x) - w->Aabs);
        if ((s / tspace + 1) * tspace - s >= M - x)
        {
            s = ((s / tspace) << 1);
            w->Trace[s] += D / 2;
            w->Trace[s + 1] += N - y;
        }
        else
            trace_nd(A + x, M - x, B + y, N - y, w, tspace);
    }
    else
    {
        int u, v;
        s = (D == 0 || M < N) ? x : x - 1;
        if (s > 0)
        {
            u = (int)(A - w->Aabs);
            v = u / tspace;
            u = (v + 1) * tspace - u;
            for (v <<= 1; s > 0; s -= u, u = tspace)
            {
                if (u > s)
                    u = s;
                w->Trace[v + 1] += u;
                v += 2;
            }
        }
        if (D == 0)
            return D;
        if (M < N)
            y = (int)((((A + x) - w->Aabs) / tspace) << 1);
        else
            y = (int)((((A + (x - 1)) - w->Aabs) / tspace) << 1);
        w->Trace[y] += 1;
        if (M <= N)
            w->Trace[y + 1] += 1;
        s = M - x;
        if (s > 0)
        {
            u = (int)((A + x) - w->Aabs);
            v = u / tspace;
            u = (v + 1) * tspace - u;
            for (v <<= 1; s > 0; s -= u, u = tspace)
            {
                if (u > s)
                    u = s;
                w->Trace[v + 1] += u;
                v += 2;
            }
        }
    }
    return D;
}

/* A bridge path: coordinates, diffs and its own trace (Compute_Alignment's alnpts). */
typedef struct
{
    int abpos, bbpos, aepos, bepos, diffs, tlen;
    uint16_t* trace;
    int cap;
} BPath;

/* Compute_Alignment(align, work, DIFF_TRACE, tspace) (dalign2/align.c:4762-4913) for the box
 * of p over aseq (its absolute base) and bseq. */
static void compute_alignment_trace(const uint8_t* aseq, const uint8_t* bseq, BPath* p, int tspace)
{
    int asub = p->aepos - p->abpos, bsub = p->bepos - p->bbpos;
    int n = 2 * (((p->aepos + (tspace - 1)) / tspace - p->abpos / tspace) + 1);
    if (n > p->cap)
    {
        p->cap = 2 * n + 64;
        p->trace = (uint16_t*)realloc(p->trace, sizeof(uint16_t) * p->cap);
    }
    int m = asub > bsub ? asub : bsub;
    int* vec = (int*)malloc(sizeof(int) * (4 * (size_t)m + 6 + 8));
    TWave w;
    w.VF = vec + (m + 1);
    w.VB = w.VF + (2 * m + 3);
    w.Aabs = aseq;
    w.Trace = p->trace - 2 * (p->abpos / tspace);
    memset(p->trace, 0, sizeof(uint16_t) * n);
    p->diffs = trace_nd(aseq + p->abpos, asub, bseq + p->bbpos, bsub, &w, tspace);
    if (p->trace[n - 1] != 0)
    {
        p->trace[n - 3] += p->trace[n - 1];
        p->trace[n - 4] += p->trace[n - 2];
    }
    p->tlen = n - 2;
    free(vec);
}

/* MapToTPAbove / MapToTPBelow (dalign2/filter.c:1481-1563): the first trace point of path at
 * or past *x (above) or at or before *x (below), in A (isA) or B; *x becomes it, the other
 * coordinate is returned. */
static int map_tp_above(const MPath* path, int* x, int isA, const TBuf* tb, int TS)
{
    const uint16_t* trace = tb->tr + path->toff;
    int a = (path->abpos / TS) * TS, b = path->bbpos;
    for (int i = 1; i < path->tlen; i += 2)
    {
        a += TS;
        b += trace[i];
        if (a > path->aepos)
            a = path->aepos;
        if (isA ? a >= *x : b >= *x)
        {
            int r = isA ? b : a;
            *x = isA ? a : b;
            return r;
        }
    }
    int r = isA ? b : a;
    *x = isA ? a : b;
    return r;
}

static int map_tp_below(const MPath* path, int* x, int isA, const TBuf* tb, int TS)
{
    const uint16_t* trace = tb->tr + path->toff;
    int a = ((path->aepos + (TS - 1)) / TS) * TS, b = path->bepos;
    for (int i = path->tlen - 1; i >= 0; i -= 2)
    {
        a -= TS;
        b -= trace[i];
        if (a < path->abpos)
            a = path->abpos;
        if (isA ? a <= *x : b <= *x)
        {
            int r = isA ? b : a;
            *x = isA ? a : b;
            return r;
        }
    }
    int r = isA ? b : a;
    *x = isA ? a : b;
    return r;
}

/* Compute_Bridge_Path (dalign2/filter.c:1579-1705): the box from two trace points before
 * path2's start to two after path1's end, aligned afresh with trace points; with comp the
 * box is aligned in the complemented frame, shifted so its trace points fall on multiples of
 * the spacing.  (The bin/bout/err tail of the reference only feeds its debug print.) */
static void compute_bridge_path(const MPath* path1, const MPath* path2, const uint8_t* aseq, const uint8_t* bseq,
                                int alen, int blen, int comp, int aovl, int bovl, const TBuf* tb, int TS, BPath* ap)
{
    int ain, aout, bin, bout, boff = 0, p;
    if (bovl > aovl)
    {
        bin = path2->bbpos;
        bout = path1->bepos;
        ain = map_tp_below(path1, &bin, 0, tb, TS);
        aout = map_tp_above(path2, &bout, 0, tb, TS);
    }
    else
    {
        ain = path2->abpos;
        aout = path1->aepos;
        bin = map_tp_below(path1, &ain, 1, tb, TS);
        bout = map_tp_above(path2, &aout, 1, tb, TS);
    }
    (void)bin;
    (void)bout;
    ap->abpos = ain - 2 * TS;
    ap->aepos = aout + 2 * TS;
    ap->bbpos = map_tp_below(path1, &ap->abpos, 1, tb, TS);
    ap->bepos = map_tp_above(path2, &ap->aepos, 1, tb, TS);
    const uint8_t* A = aseq;
    if (comp)
    {
        boff = TS - ap->aepos % TS;
        p = alen - ap->abpos;
        ap->abpos = alen - ap->aepos;
        ap->aepos = p;
        p = blen - ap->bbpos;
        ap->bbpos = blen - ap->bepos;
        ap->bepos = p;
        boff = boff - ap->abpos % TS;
        A -= boff;
        ap->abpos += boff;
        ap->aepos += boff;
    }
    compute_alignment_trace(A, bseq, ap, TS);
    if (comp)
    {
        uint16_t* trk = ap->trace;
        int j = ap->tlen - 2, i = 0;
        while (i < j)
        {
            uint16_t t = trk[i];
            trk[i] = trk[j];
            trk[j] = t;
            t = trk[i + 1];
            trk[i + 1] = trk[j + 1];
            trk[j + 1] = t;
            i += 2;
            j -= 2;
        }
        ap->abpos -= boff;
        ap->aepos -= boff;
        p = alen - ap->abpos;
        ap->abpos = alen - ap->aepos;
        ap->aepos = p;
        p = blen - ap->bbpos;
        ap->bbpos = blen - ap->bepos;
        ap->bepos = p;
    }
}

/* Check_Bridge (dalign2/filter.c:1565-1577) */
static int check_bridge(const BPath* p, int TS)
{
    if (TS <= 125)
        for (int i = 0; i < p->tlen; i++)
            if (p->trace[i] > 250)
                return 1;
    return 0;
}

/* Bridge (dalign2/filter.c:1885-1948): path1 up to the bridge, the bridge, path3 after it */
static void bridge(MPath* path1, const BPath* path2, const MPath* path3, TBuf* tb, int TS)
{
    int k, k1, k2, len, diff;
    k1 = 2 * ((path2->abpos / TS) - (path1->abpos / TS));
    if (path2->aepos == path3->aepos)
        k2 = path3->tlen;
    else
        k2 = 2 * ((path2->aepos / TS) - (path3->abpos / TS));
    len = k1 + path2->tlen + (path3->tlen - k2);
    tbuf_reserve(tb, len);
    int64_t base = tb->top;
    tb->top += len;
    uint16_t* trace = tb->tr + base;
    diff = 0;
    len = 0;
    if (k1 > 0)
    {
        const uint16_t* t = tb->tr + path1->toff;
        for (k = 0; k < k1; k += 2)
        {
            trace[len++] = t[k];
            trace[len++] = t[k + 1];
            diff += t[k];
        }
    }
    for (k = 0; k < path2->tlen; k += 2)
    {
        trace[len++] = path2->trace[k];
        trace[len++] = path2->trace[k + 1];
        diff += path2->trace[k];
    }
    if (k2 < path3->tlen)
    {
        const uint16_t* t = tb->tr + path3->toff;
        for (k = k2; k < path3->tlen; k += 2)
        {
            trace[len++] = t[k];
            trace[len++] = t[k + 1];
            diff += t[k];
        }
    }
    path1->aepos = path3->aepos;
    path1->bepos = path3->bepos;
    path1->diffs = diff;
    path1->toff = base;
    path1->tlen = len;
}

/* The sequences of a pair as Handle_Redundancies sees them: align (A against B, B
 * complemented for a complement pair) and blign (the roles swapped). */
typedef struct
{
    const uint8_t *aseq, *bseq;
    int alen, blen, comp;
} PairSeq;

/* daligner2's Handle_Redundancies (dalign2/filter.c:1952-2272): paths fused into the later
 * index j, the absorbed one marked with abpos = -1 and the scan restarted after a fusion;
 * then the bridging pass; then compaction. */
static int handle_redundancies_d2(MPath* amatch, int novls, MPath* bmatch, TBuf* tb, int TS, int comp,
                                  const PairSeq* ps)
{
    int j, k, no, dist, awhen = 0, bwhen = 0;
    int hasB = (bmatch != NULL);
    for (j = 1; j < novls; j++)
    {
        MPath* jpath = amatch + j;
        for (k = j - 1; k >= 0; k--)
        {
            MPath* kpath = amatch + k;
            if (kpath->abpos < 0)
                continue;
            if (jpath->abpos < kpath->abpos)
            {
                if (kpath->abpos <= jpath->aepos && kpath->bbpos <= jpath->bepos)
                {
                    dist = entwine(jpath, kpath, tb, TS, &awhen, 1);
                    if (dist == 0)
                    {
                        if (kpath->aepos > jpath->aepos)
                        {
                            if (hasB)
                            {
                                if (comp)
                                {
                                    dist = entwine(bmatch + k, bmatch + j, tb, TS, &bwhen, 1);
                                    if (dist != 0)
                                        continue;
                                    fusion(jpath, awhen, kpath, tb, TS);
                                    fusion(bmatch + k, bwhen, bmatch + j, tb, TS);
                                    bmatch[j] = bmatch[k];
                                }
                                else
                                {
                                    dist = entwine(bmatch + j, bmatch + k, tb, TS, &bwhen, 1);
                                    if (dist != 0)
                                        continue;
                                    fusion(jpath, awhen, kpath, tb, TS);
                                    fusion(bmatch + j, bwhen, bmatch + k, tb, TS);
                                }
                            }
                            else
                                fusion(jpath, awhen, kpath, tb, TS);
                            kpath->abpos = -1;
                            k = j;
                            continue;
                        }
                        kpath->abpos = -1;
                    }
                }
            }
            else
            {
                if (jpath->abpos <= kpath->aepos && jpath->bbpos <= kpath->bepos)
                {
                    dist = entwine(kpath, jpath, tb, TS, &awhen, 1);
                    if (dist == 0)
                    {
                        int restart = 0;
                        if (kpath->abpos == jpath->abpos)
                        {
                            if (kpath->aepos > jpath->aepos)
                            {
                                *jpath = *kpath;
                                if (hasB)
                                    bmatch[j] = bmatch[k];
                            }
                        }
                        else if (jpath->aepos > kpath->aepos)
                        {
                            if (hasB)
                            {
                                if (comp)
                                {
                                    dist = entwine(bmatch + j, bmatch + k, tb, TS, &bwhen, 1);
                                    if (dist != 0)
                                        continue;
                                    fusion(kpath, awhen, jpath, tb, TS);
                                    *jpath = *kpath;
                                    fusion(bmatch + j, bwhen, bmatch + k, tb, TS);
                                }
                                else
                                {
                                    dist = entwine(bmatch + k, bmatch + j, tb, TS, &bwhen, 1);
                                    if (dist != 0)
                                        continue;
                                    fusion(kpath, awhen, jpath, tb, TS);
                                    *jpath = *kpath;
                                    fusion(bmatch + k, bwhen, bmatch + j, tb, TS);
                                    bmatch[j] = bmatch[k];
                                }
                            }
                            else
                            {
                                fusion(kpath, awhen, jpath, tb, TS);
                                *jpath = *kpath;
                            }
                            restart = 1;
                        }
                        else
                        {
                            *jpath = *kpath;
                            if (hasB)
                                bmatch[j] = bmatch[k];
                        }
                        kpath->abpos = -1;
                        if (restart)
                            k = j;
                    }
                }
            }
        }
    }
    /* the bridging pass (dalign2/filter.c:2124-2262): a pair of paths with a narrow
     * parallel overlap is joined through a fresh alignment of the overlap's box; the A-side
     * box is aligned uncomplemented, the B side in its pair's orientation */
    BPath bp = {0, 0, 0, 0, 0, 0, NULL, 0};
    for (j = 1; j < novls; j++)
    {
        MPath* jpath = amatch + j;
        if (jpath->abpos < 0)
            continue;
        for (k = j - 1; k >= 0; k--)
        {
            MPath* kpath = amatch + k;
            if (kpath->abpos < 0)
                continue;
            MPath *path1, *path2, *bath1 = NULL, *bath2 = NULL;
            if (jpath->abpos < kpath->abpos)
            {
                path1 = jpath;
                path2 = kpath;
            }
            else
            {
                path1 = kpath;
                path2 = jpath;
            }
            if (path2->abpos >= path1->aepos || path1->aepos >= path2->aepos || path1->bbpos >= path2->bbpos ||
                path2->bbpos >= path1->bepos || path1->bepos >= path2->bepos)
                continue;
            int aovl = path1->aepos - path2->abpos;
            int bovl = path1->bepos - path2->bbpos;
            if (abs(aovl - bovl) > .2 * (aovl + bovl))
                continue;
            if (hasB)
            {
                if (comp == (jpath->abpos < kpath->abpos))
                {
                    bath1 = bmatch + k;
                    bath2 = bmatch + j;
                }
                else
                {
                    bath1 = bmatch + j;
                    bath2 = bmatch + k;
                }
                if (bath1->abpos > bath2->abpos)
                    continue;
            }
            compute_bridge_path(path1, path2, ps->aseq, ps->bseq, ps->alen, ps->blen, 0, aovl, bovl, tb, TS, &bp);
            if (check_bridge(&bp, TS))
                continue;
            MPath jback = *jpath, kback = *kpath;
            bridge(path1, &bp, path2, tb, TS);
            *jpath = *path1;
            kpath->abpos = -1;
            if (hasB)
            {
                compute_bridge_path(bath1, bath2, ps->bseq, ps->aseq, ps->blen, ps->alen, comp, bovl, aovl, tb, TS,
                                    &bp);
                if (check_bridge(&bp, TS))
                {
                    *jpath = jback;
                    *kpath = kback;
                    continue;
                }
                bridge(bath1, &bp, bath2, tb, TS);
                bmatch[j] = *bath1;
            }
        }
    }
    free(bp.trace);
    no = 0;
    for (j = 0; j < novls; j++)
        if (amatch[j].abpos >= 0)
        {
            if (hasB)
                bmatch[no] = bmatch[j];
            amatch[no++] = amatch[j];
        }
    return no;
}

/* Diagonal_Span (filter.c:1568-1599) */
static void diagonal_span(const WPath* path, int TS, int binshift, int* mind, int* maxd)
{
    const uint16_t* points = path->trace;
    int tlen = path->tlen, dd, low, hgh, i;
    dd = path->abpos - path->bbpos;
    low = hgh = dd;
    dd = path->aepos - path->bepos;
    if (dd < low)
        low = dd;
    else if (dd > hgh)
        hgh = dd;
    dd = (path->abpos / TS) * TS - path->bbpos;
    tlen -= 2;
    for (i = 1; i < tlen; i += 2)
    {
        dd += TS - points[i];
        if (dd < low)
            low = dd;
        else if (dd > hgh)
            hgh = dd;
    }
    *mind = (low >> binshift) - 1;
    *maxd = (hgh >> binshift) + 1;
}

typedef struct
{
    or_overlap* o;
    int64_t n, max;
    uint8_t* tr;
    int64_t ttop, tmax;
    int tbytes;
} OBuf;

static void obuf_add(OBuf* ob, const MPath* mp, const uint16_t* trace, uint32_t flags, int aread, int bread, int no_trace)
{
    if (ob->n >= ob->max)
    {
        ob->max = ob->max * 2 + 1000;
        ob->o = (or_overlap*)realloc(ob->o, sizeof(or_overlap) * ob->max);
    }
    or_overlap* o = ob->o + ob->n++;
    o->tlen = no_trace ? 0 : mp->tlen;
    o->diffs = mp->diffs;
    o->abpos = mp->abpos;
    o->bbpos = mp->bbpos;
    o->aepos = mp->aepos;
    o->bepos = mp->bepos;
    o->flags = flags;
    o->aread = aread;
    o->bread = bread;
    o->toff = ob->ttop;
    if (no_trace)
        return;
    int64_t need = (int64_t)mp->tlen * ob->tbytes;
    if (ob->ttop + need >= ob->tmax)
    {
        ob->tmax = (ob->ttop + need) * 2 + 1000;
        ob->tr = (uint8_t*)realloc(ob->tr, ob->tmax);
    }
    if (ob->tbytes == 1)
        for (int i = 0; i < mp->tlen; i++)
            ob->tr[ob->ttop + i] = (uint8_t)trace[i]; /* Compress_TraceTo8 (align.c:3352-3360) */
    else
        memcpy(ob->tr + ob->ttop, trace, need);
    ob->ttop += need;
}

/* report_thread (filter.c:1617-1989) over the whole sorted hit list */
/* p->variant == 2: daligner2's report_thread (dalign2/filter_reporter_cpu.c:16-411): the last
 * group of the list is scanned too (nidx <= eidx), -H is live, the B-side record of a read
 * against itself is dropped in both orientations, its Handle_Redundancies, and the 8-bit
 * trace compression checked.  *status receives the daligner2 failure codes of or_result. */
static void report(const or_block* A, const or_block* B, const Hit* hits, int64_t nhits, const or_params* p,
                   const Spec* sp, Work* w, int self, int comp, OBuf* ob, int64_t* nseed, int32_t* status)
{
    const int d2 = p->variant == 2;
    const int K = p->kmer, BS = p->binshift, TS = sp->tspace;
    int maxdiag = (A->maxlen >> BS);
    int mindiag = ((-B->maxlen) >> BS);
    int wdt = maxdiag - mindiag + 1;
    /* score | lastp | lasta laid out back to back as the reference lays them out
     * (filter.c:2296-2311), so out-of-range band writes land where they land there. */
    int* counters = (int*)calloc(3 * (size_t)wdt + 2, sizeof(int));
    int* score = counters + 1 - mindiag;
    int* lastp = score + wdt;
    int* lasta = lastp + wdt;
    int minhit = (p->hitmin - 1) / K + 1;
    /* daligner: -H is a no-op, main() shadows the global (daligner.c:63 vs 641) */
    int HGAP_MIN = d2 ? p->hgap : 0;
    int64_t AOmax = 100, BOmax = 100;
    MPath* amatch = (MPath*)malloc(sizeof(MPath) * AOmax);
    MPath* bmatch = (MPath*)malloc(sizeof(MPath) * BOmax);
    TBuf tb = {0, 0, 0};
    tbuf_reserve(&tb, 40000);
    WPath apath, bpath;
    int64_t nfilt = 0;

#define PAIR(i) (((u64)(uint32_t)hits[i].bread << 32) | (uint32_t)hits[i].aread)
    int64_t nidx = 0, eidx = nhits - minhit;
    u64 cpair, npair = 0;
    for (cpair = PAIR(0); d2 ? nidx <= eidx : nidx < eidx; cpair = npair)
    {
        if (PAIR(nidx + minhit - 1) != cpair)
        {
            nidx += 1;
            while ((npair = PAIR(nidx)) == cpair)
                nidx += 1;
            continue;
        }
        int ar = hits[nidx].aread, br = hits[nidx].bread;
        int alen = A->rlen[ar], blen = B->rlen[br];
        if (alen < HGAP_MIN && blen < HGAP_MIN)
        {
            nidx += 1;
            while ((npair = PAIR(nidx)) == cpair)
                nidx += 1;
            continue;
        }
        const uint8_t* aseq = A->bases + A->boff[ar];
        const uint8_t* bseq = B->bases + B->boff[br];
        int setaln = 1, doA = 0, doB = 0, amark, amark2 = 0, novla = 0, novlb = 0;
        int64_t sidx, lidx, f, h2;
        tb.top = 0;
        for (sidx = nidx; PAIR(nidx) == cpair; nidx = h2)
        {
            amark = amark2 + PANEL_SIZE;
            amark2 = amark - PANEL_OVERLAP;
            h2 = lidx = nidx;
            int apos;
            do
            {
                apos = hits[nidx].apos;
                ++nidx;
                npair = PAIR(nidx);
                if (apos <= amark2)
                    h2 = nidx;
            } while (npair == cpair && apos <= amark);
            if (nidx - lidx < minhit)
                continue;
            for (f = lidx; f < nidx; f++)
            {
                int ap = hits[f].apos, dg = hits[f].diag >> BS;
                if (ap - lastp[dg] >= K)
                    score[dg] += K;
                else
                    score[dg] += ap - lastp[dg];
                lastp[dg] = ap;
            }
            for (f = lidx; f < nidx; f++)
            {
                int ap = hits[f].apos, dg = hits[f].diag, bp = ap - dg;
                dg >>= BS;
                if (ap > lasta[dg] && (score[dg] + score[dg + 1] >= p->hitmin || score[dg] + score[dg - 1] >= p->hitmin))
                {
                    if (setaln)
                    {
                        setaln = 0;
                        doA = (alen >= HGAP_MIN);
                        if (d2)
                            doB = (p->symmetric && blen >= HGAP_MIN && !(ar == br && self));
                        else
                            doB = (p->symmetric && blen >= HGAP_MIN && (ar != br || !self || !comp));
                    }
                    nfilt += 1;
                    local_alignment(w, sp, aseq, bseq, alen, blen, comp, ap - bp, ap + bp, &apath, &bpath);
                    {
                        int lo, hi, ae = apath.aepos;
                        diagonal_span(&apath, TS, BS, &lo, &hi);
                        if (dg < lo)
                            lo = dg;
                        else if (dg > hi)
                            hi = dg;
                        for (int d2 = lo; d2 <= hi; d2++)
                            if (ae > lasta[d2])
                                lasta[d2] = ae;
                    }
                    if ((apath.aepos - apath.abpos) + (apath.bepos - apath.bbpos) >= p->minover)
                    {
                        if (doA)
                        {
                            if (novla >= AOmax)
                            {
                                AOmax = AOmax * 2 + 100;
                                amatch = (MPath*)realloc(amatch, sizeof(MPath) * AOmax);
                            }
                            tbuf_reserve(&tb, apath.tlen);
                            MPath* m = amatch + novla++;
                            m->toff = tb.top;
                            m->tlen = apath.tlen;
                            m->diffs = apath.diffs;
                            m->abpos = apath.abpos;
                            m->bbpos = apath.bbpos;
                            m->aepos = apath.aepos;
                            m->bepos = apath.bepos;
                            memcpy(tb.tr + tb.top, apath.trace, sizeof(uint16_t) * apath.tlen);
                            tb.top += apath.tlen;
                        }
                        if (doB)
                        {
                            if (novlb >= BOmax)
                            {
                                BOmax = BOmax * 2 + 100;
                                bmatch = (MPath*)realloc(bmatch, sizeof(MPath) * BOmax);
                            }
                            tbuf_reserve(&tb, bpath.tlen);
                            MPath* m = bmatch + novlb++;
                            m->toff = tb.top;
                            m->tlen = bpath.tlen;
                            m->diffs = bpath.diffs;
                            m->abpos = bpath.abpos;
                            m->bbpos = bpath.bbpos;
                            m->aepos = bpath.aepos;
                            m->bepos = bpath.bepos;
                            memcpy(tb.tr + tb.top, bpath.trace, sizeof(uint16_t) * bpath.tlen);
                            tb.top += bpath.tlen;
                        }
                    }
                }
            }
            for (f = lidx; f < nidx; f++)
            {
                int dg = hits[f].diag >> BS;
                score[dg] = lastp[dg] = 0;
            }
        }
        for (f = sidx; f < nidx; f++)
        {
            int dg = hits[f].diag >> BS, d2;
            for (d2 = dg; d2 <= maxdiag; d2++)
                if (lasta[d2] == 0)
                    break;
                else
                    lasta[d2] = 0;
            for (d2 = dg - 1; d2 >= mindiag; d2--)
                if (lasta[d2] == 0)
                    break;
                else
                    lasta[d2] = 0;
        }
        if (d2)
        {
            int r1 = novla, r2 = novlb;
            /* the pair's align (B complemented for a complement pair); a B-only call is
             * handed the same align, as the reference does (filter_reporter_cpu.c:392-400) */
            PairSeq ps = {aseq, bseq, alen, blen, comp};
            if (novla > 1)
            {
                if (novlb > 1)
                    r1 = r2 = handle_redundancies_d2(amatch, novla, bmatch, &tb, TS, comp, &ps);
                else
                    r1 = handle_redundancies_d2(amatch, novla, NULL, &tb, TS, comp, &ps);
            }
            else if (novlb > 1)
                r2 = handle_redundancies_d2(bmatch, novlb, NULL, &tb, TS, comp, &ps);
            if (r1 < 0 || r2 < 0)
            {
                *status = 1;
                break;
            }
            novla = r1;
            novlb = r2;
            if (ob->tbytes == 1 && !p->no_trace)
            {
                int big = 0;
                for (int i = 0; i < novla; i++)
                    for (int t = 0; t < amatch[i].tlen; t++)
                        big |= tb.tr[amatch[i].toff + t] > 255;
                for (int i = 0; i < novlb; i++)
                    for (int t = 0; t < bmatch[i].tlen; t++)
                        big |= tb.tr[bmatch[i].toff + t] > 255;
                if (big)
                {
                    *status = 2;
                    break;
                }
            }
        }
        else if (novla > 1)
        {
            if (novlb > 1)
                novla = novlb = handle_redundancies(amatch, novla, bmatch, &tb, TS, comp);
            else
                novla = handle_redundancies(amatch, novla, NULL, &tb, TS, comp);
        }
        else if (novlb > 1)
            novlb = handle_redundancies(bmatch, novlb, NULL, &tb, TS, comp);
        for (int i = 0; i < novla; i++)
            obuf_add(ob, amatch + i, tb.tr + amatch[i].toff, comp, ar + A->ufirst, br + B->ufirst, p->no_trace);
        for (int i = 0; i < novlb; i++)
            obuf_add(ob, bmatch + i, tb.tr + bmatch[i].toff, comp, br + B->ufirst, ar + A->ufirst, p->no_trace);
    }
#undef PAIR
    *nseed = nfilt;
    free(counters);
    free(amatch);
    free(bmatch);
    free(tb.tr);
}

static int cmp_ovl(const void* x, const void* y)
{
    const or_overlap* l = (const or_overlap*)x;
    const or_overlap* r = (const or_overlap*)y;
    if (l->aread != r->aread)
        return l->aread < r->aread ? -1 : 1;
    if (l->bread != r->bread)
        return l->bread < r->bread ? -1 : 1;
    if ((l->flags & 1) != (r->flags & 1))
        return (l->flags & 1) < (r->flags & 1) ? -1 : 1;
    if (l->abpos != r->abpos)
        return l->abpos < r->abpos ? -1 : 1;
    /* ties are unordered in the reference (qsort); order them fully here */
    if (l->aepos != r->aepos)
        return l->aepos < r->aepos ? -1 : 1;
    if (l->bbpos != r->bbpos)
        return l->bbpos < r->bbpos ? -1 : 1;
    return l->toff < r->toff ? -1 : (l->toff > r->toff);
}

int or_daligner(const or_block* a, const or_block* b, const or_block* bc, const or_params* p, int self,
                or_result* res)
{
    Spec sp;
    Work w;
    OBuf ob;
    memset(res, 0, sizeof(*res));
    memset(&w, 0, sizeof(w));
    memset(&ob, 0, sizeof(ob));
    make_spec(&sp, p);
    ob.tbytes = (p->tspace <= 125) ? 1 : 2;

    int64_t alen, blen, nh;
    int limit;
    KPos* al = build_index(a, p, &alen);
    res->kmers_a = alen;
    if (alen > 0)
    {
        KPos* bl = self ? al : build_index(b, p, &blen);
        if (self)
            blen = alen;
        res->kmers_b = blen;
        if (blen > 0)
        {
            Hit* h = sorted_hits(a, b, al, alen, bl, blen, p, self, 0, self, &nh, &limit);
            res->hits_n = nh;
            if (nh > 0)
                report(a, b, h, nh, p, &sp, &w, self, 0, &ob, &res->seeds_n, &res->status);
            free(h);
        }
        if (!self)
            free(bl);
        /* complemented B block (complement_DB, daligner.c:474-573) */
        bl = build_index(bc, p, &blen);
        if (blen > 0)
        {
            Hit* h = sorted_hits(a, bc, al, alen, bl, blen, p, self, 1, 0, &nh, &limit);
            res->hits_c = nh;
            if (nh > 0)
                report(a, bc, h, nh, p, &sp, &w, self, 1, &ob, &res->seeds_c, &res->status);
            free(h);
        }
        free(bl);
    }
    free(al);

    /* only-identity filter and sort (Write_Overlap_Buffer, align.c:5815-5853) */
    if (p->only_identity)
    {
        int64_t c = 0;
        for (int64_t i = 0; i < ob.n; i++)
            if (ob.o[i].aread == ob.o[i].bread)
                ob.o[c++] = ob.o[i];
        ob.n = c;
    }
    qsort(ob.o, ob.n, sizeof(or_overlap), cmp_ovl);
    res->novl = ob.n;
    res->ovl = ob.o;
    res->trace = ob.tr;
    res->tbytes_total = ob.ttop;
    res->tbytes = ob.tbytes;
    res->cells = w.cells_count;
    res->snake_steps = w.snakes;
    fprintf(stderr, "oracle stats: max_width %lld max_cells %lld waves %lld snakes %lld\n", (long long)w.max_width, (long long)w.max_cells, (long long)w.waves, (long long)w.snakes);
    free(w.mem);
    free(w.cells);
    free(w.pts);
    return 0;
}

/* ------------------------------------------------------------------------------------ */
/*  daligner2 (dalign2/): modimizer index, one join for both orientations                */
/* ------------------------------------------------------------------------------------ */

#define D2_MODULUS 101
#define D2_MODTHR 28

/* The k-mer list (mask_thread/tuple_thread, dalign2/filter.c:147-769, MODIFER on): at every
 * position p of an unmasked segment, after k-1 bases of warm-up, two codes: the canonical
 * k-mer min(c, u) of the forward code c and the reverse-complement code u, and the
 * "half-shifted" code min(d, v) whose high half comes from the previous code.  A code is
 * listed when code % 101 < 28, with read = (i << 1) | (1 if the complement code won). */
static int64_t extract_kmers2(const or_block* b, int K, KPos* list)
{
    const int Kshift = K >= 32 ? 64 : 2 * K;
    const u64 Kmask = K >= 32 ? ~0ull : ((1ull << Kshift) - 1);
    const u64 LFmask = (1ull << (Kshift / 2)) - 1, HFmask = Kmask - LFmask;
    const u64 LRmask = (1ull << ((Kshift + 1) / 2)) - 1, HRmask = Kmask - LRmask;
    u64 cumber[4];
    for (int x = 0; x < 4; x++)
        cumber[x] = (u64)(3 - x) << (Kshift - 2);
    int64_t n = 0;
    for (int i = 0; i < b->nreads; i++)
    {
        const uint8_t* s = b->bases + b->boff[i];
        const int rlen = b->rlen[i], r = i << 1;
        int64_t f0 = 0, f1 = 0;
        if (b->mask_anno)
        {
            f0 = b->mask_anno[i];
            f1 = b->mask_anno[i + 1];
        }
        for (int64_t a = f0; a <= f1; a += 2)
        {
            int p = (a == f0) ? 0 : b->mask_data[a - 1];
            int q = (a == f1) ? rlen : b->mask_data[a];
            if (q - p > K - 1)
            {
                u64 c = 0, u = 0, d, v;
                for (int x = 1; x < K; x++)
                {
                    c = (c << 2) | s[p];
                    u = (u >> 2) | cumber[s[p]];
                    p++;
                }
                for (; p < q; p++)
                {
                    int x = s[p];
                    d = c & HFmask;
                    c = ((c << 2) | (u64)x) & Kmask;
                    d |= c & LFmask;
                    v = u & LRmask;
                    u = (u >> 2) | cumber[x];
                    v |= u & HRmask;
                    if (u < c)
                    {
                        if (u % D2_MODULUS < D2_MODTHR)
                        {
                            list[n].code = u;
                            list[n].read = r | 1;
                            list[n++].rpos = p;
                        }
                    }
                    else if (c % D2_MODULUS < D2_MODTHR)
                    {
                        list[n].code = c;
                        list[n].read = r;
                        list[n++].rpos = p;
                    }
                    if (v < d)
                    {
                        if (v % D2_MODULUS < D2_MODTHR)
                        {
                            list[n].code = v;
                            list[n].read = r | 1;
                            list[n++].rpos = p;
                        }
                    }
                    else if (d % D2_MODULUS < D2_MODTHR)
                    {
                        list[n].code = d;
                        list[n].read = r;
                        list[n++].rpos = p;
                    }
                }
            }
            if (!b->mask_anno)
                break;
        }
    }
    return n;
}

/* Sort_Kmers (dalign2/filter.c:834-1106): stable radix sort on (k-1)/4+1 code bytes, -t */
static KPos* build_index2(const or_block* b, const or_params* p, int64_t* len)
{
    int K = p->kmer;
    KPos* list = (KPos*)malloc(sizeof(KPos) * (2 * (size_t)b->totlen + 2));
    int64_t n = extract_kmers2(b, K, list);
    sort_kpos(list, n, (K - 1) / 4 + 1);
    if (p->suppress > 0 && n > 0)
    {
        int64_t w = 0, i = 0;
        while (i < n)
        {
            int64_t j = i + 1;
            while (j < n && list[j].code == list[i].code)
                j++;
            if (j - i < p->suppress)
                for (int64_t q = i; q < j; q++)
                    list[w++] = list[q];
            i = j;
        }
        n = w;
    }
    list[n].code = ~0ull; /* MAX_CODE_64 sentinel (dalign2/filter.c:991) */
    *len = n;
    return list;
}

int64_t or_sort_kmers2(const or_block* b, const or_params* p, uint64_t* code, int32_t* read, int32_t* rpos)
{
    int64_t n;
    KPos* l = build_index2(b, p, &n);
    for (int64_t i = 0; i < n; i++)
    {
        code[i] = l[i].code;
        read[i] = l[i].read;
        rpos[i] = l[i].rpos;
    }
    free(l);
    return n;
}

/* count_thread + the -M cap + merge_thread (dalign2/filter.c:1136-1466, 2401-2520).
 * Within a block, entry ka of a code run pairs with the run's earlier entries of a smaller
 * read (all earlier entries with -I); across blocks every A entry with every B entry.  A
 * pair is a forward hit when both strands agree, else a complement hit whose B position is
 * reflected (rlen - bpos + k - 2).  Hits of each orientation are returned in the
 * reference's generation order. */
static void merge_hits2(const or_block* B, const KPos* al, int64_t alen, const KPos* bl, int64_t blen,
                        const or_params* p, int self, Hit** hf, int64_t* nf, Hit** hc, int64_t* nc,
                        int* limit_out)
{
    const int Koff = p->kmer - 2;
    int64_t hist[MAXGRAM];
    memset(hist, 0, sizeof(hist));
    int64_t total = 0;
#define RUN_CT(ja, ia, jb, ib, ct)                                                \
    do                                                                            \
    {                                                                             \
        ct = 0;                                                                   \
        if (self)                                                                 \
        {                                                                         \
            for (int64_t ka = ja + 1; ka < ia; ka++)                              \
                if (p->identity)                                                  \
                    ct += ka - ja;                                                \
                else                                                              \
                {                                                                 \
                    int64_t a = ja;                                               \
                    while (a < ka && (al[a].read >> 1) < (al[ka].read >> 1))      \
                        a++;                                                      \
                    ct += a - ja;                                                 \
                }                                                                 \
        }                                                                         \
        else                                                                      \
            ct = (ia - ja) * (ib - jb);                                           \
    } while (0)
    /* pass 1: the histogram of per-code pair counts */
    {
        int64_t ia = 0, ib = 0;
        while (ia < alen)
        {
            int64_t ja = ia;
            u64 ca = al[ia].code;
            while (ia < alen && al[ia].code == ca)
                ia++;
            int64_t jb = 0, ct;
            if (!self)
            {
                while (ib < blen && bl[ib].code < ca)
                    ib++;
                if (ib >= blen || bl[ib].code != ca)
                    continue;
                jb = ib;
                while (ib < blen && bl[ib].code == ca)
                    ib++;
            }
            RUN_CT(ja, ia, jb, ib, ct);
            total += ct;
            if (ct < MAXGRAM)
                hist[ct]++;
        }
    }
    int limit = INT_MAX;
    if (p->mem_limit > 0)
    {
        int64_t avail = (int64_t)(p->mem_limit / 16);
        if (self || avail > alen + 2 * blen)
            avail = (avail - alen) / 2;
        else
            avail = avail - (alen + blen);
        avail = (int64_t)(avail * .98);
        int64_t tom = 0;
        int j;
        for (j = 0; j < MAXGRAM; j++)
        {
            tom += j * hist[j];
            if (tom > avail)
                break;
        }
        limit = j;
    }
    *limit_out = limit;
    /* pass 2: emission; sizes first */
    int64_t cap = total + 1;
    Hit* F = (Hit*)malloc(sizeof(Hit) * (cap + 1));
    Hit* Cm = (Hit*)malloc(sizeof(Hit) * (cap + 1));
    int64_t n1 = 0, n2 = 0;
    int64_t ia = 0, ib = 0;
    while (ia < alen)
    {
        int64_t ja = ia;
        u64 ca = al[ia].code;
        while (ia < alen && al[ia].code == ca)
            ia++;
        int64_t jb = 0, ct;
        if (!self)
        {
            while (ib < blen && bl[ib].code < ca)
                ib++;
            if (ib >= blen || bl[ib].code != ca)
                continue;
            jb = ib;
            while (ib < blen && bl[ib].code == ca)
                ib++;
        }
        RUN_CT(ja, ia, jb, ib, ct);
        if (ct >= limit)
            continue;
#define EMIT(A_, B_)                                                                 \
    do                                                                               \
    {                                                                                \
        int ar = (A_).read >> 1, as = (A_).read & 1, ap = (A_).rpos;                 \
        int br = (B_).read >> 1, bs = (B_).read & 1, bp = (B_).rpos;                 \
        Hit* h;                                                                      \
        if (bs == as)                                                                \
            h = F + n1++;                                                            \
        else                                                                         \
        {                                                                            \
            bp = (B->rlen[br] - bp) + Koff;                                          \
            h = Cm + n2++;                                                           \
        }                                                                            \
        h->aread = ar;                                                               \
        h->bread = br;                                                               \
        h->apos = ap;                                                                \
        h->diag = ap - bp;                                                           \
    } while (0)
        if (self)
        {
            for (int64_t ka = ja + 1; ka < ia; ka++)
                for (int64_t a = ja; a < ka; a++)
                {
                    if (!p->identity && (al[a].read >> 1) >= (al[ka].read >> 1))
                        break;
                    EMIT(al[ka], al[a]);
                }
        }
        else
            for (int64_t a = ja; a < ia; a++)
                for (int64_t q = jb; q < ib; q++)
                    EMIT(al[a], bl[q]);
#undef EMIT
    }
#undef RUN_CT
    *hf = F;
    *nf = n1;
    *hc = Cm;
    *nc = n2;
}

int or_handle_redundancies_d2(const uint8_t* aseq, const uint8_t* bseq, int alen, int blen, int tspace, int comp,
                              int novls, int hasB, const int32_t* hdr, const uint16_t* traces, int32_t* out_hdr,
                              uint16_t* out_traces, int64_t tcap)
{
    TBuf tb = {0, 0, 0};
    int npath = novls * (hasB ? 2 : 1);
    MPath* m = (MPath*)malloc(sizeof(MPath) * (size_t)(npath + 1));
    int64_t off = 0;
    for (int i = 0; i < npath; i++)
    {
        const int32_t* h = hdr + 6 * i;
        m[i].abpos = h[0];
        m[i].bbpos = h[1];
        m[i].aepos = h[2];
        m[i].bepos = h[3];
        m[i].diffs = h[4];
        m[i].tlen = h[5];
        tbuf_reserve(&tb, h[5] + 16);
        memcpy(tb.tr + tb.top, traces + off, sizeof(uint16_t) * h[5]);
        m[i].toff = tb.top;
        tb.top += h[5];
        off += h[5];
    }
    PairSeq ps = {aseq, bseq, alen, blen, comp};
    int n = handle_redundancies_d2(m, novls, hasB ? m + novls : NULL, &tb, tspace, comp, &ps);
    int64_t o = 0;
    for (int side = 0; side < (hasB ? 2 : 1); side++)
        for (int i = 0; i < n; i++)
        {
            const MPath* q = m + side * novls + i;
            int32_t* h = out_hdr + 6 * (side * n + i);
            h[0] = q->abpos;
            h[1] = q->bbpos;
            h[2] = q->aepos;
            h[3] = q->bepos;
            h[4] = q->diffs;
            h[5] = q->tlen;
            if (o + q->tlen > tcap)
            {
                free(m);
                free(tb.tr);
                return -1;
            }
            memcpy(out_traces + o, tb.tr + q->toff, sizeof(uint16_t) * q->tlen);
            o += q->tlen;
        }
    free(m);
    free(tb.tr);
    return n;
}

int or_daligner2(const or_block* a, const or_block* b, const or_block* bc, const or_params* p, int self,
                 or_result* res)
{
    Spec sp;
    Work w;
    OBuf ob;
    memset(res, 0, sizeof(*res));
    memset(&w, 0, sizeof(w));
    memset(&ob, 0, sizeof(ob));
    if (p->variant != 2)
        return -1;
    make_spec(&sp, p);
    ob.tbytes = (p->tspace <= 125) ? 1 : 2;
    int64_t alen, blen;
    KPos* al = build_index2(a, p, &alen);
    KPos* bl = self ? al : build_index2(b, p, &blen);
    if (self)
        blen = alen;
    res->kmers_a = alen;
    res->kmers_b = blen;
    if (alen > 0 && blen > 0)
    {
        Hit *hf, *hc;
        int64_t nf, nc;
        int limit;
        merge_hits2(b, al, alen, bl, blen, p, self, &hf, &nf, &hc, &nc, &limit);
        res->hits_n = nf;
        res->hits_c = nc;
        /* the hit sort orders (aread', bread, apos) with aread' = aread + nreads(A) for the
         * complement; per orientation that is (aread, bread, apos), and groups are
         * independent, so each orientation is sorted and scanned on its own */
        sort_hits(hf, nf, nbytes_for(a->maxlen), nbytes_for(a->nreads), nbytes_for(b->nreads));
        sort_hits(hc, nc, nbytes_for(a->maxlen), nbytes_for(a->nreads), nbytes_for(b->nreads));
        hf[nf].aread = hf[nf].bread = hf[nf].diag = 0x7fffffff;
        hf[nf].apos = 0;
        hc[nc].aread = hc[nc].bread = hc[nc].diag = 0x7fffffff;
        hc[nc].apos = 0;
        if (nf > 0)
            report(a, b, hf, nf, p, &sp, &w, self, 0, &ob, &res->seeds_n, &res->status);
        if (nc > 0 && res->status == 0)
            report(a, bc, hc, nc, p, &sp, &w, self, 1, &ob, &res->seeds_c, &res->status);
        free(hf);
        free(hc);
    }
    if (!self)
        free(bl);
    free(al);
    qsort(ob.o, ob.n, sizeof(or_overlap), cmp_ovl);
    res->novl = ob.n;
    res->ovl = ob.o;
    res->trace = ob.tr;
    res->tbytes_total = ob.ttop;
    res->tbytes = ob.tbytes;
    res->cells = w.cells_count;
    res->snake_steps = w.snakes;
    free(w.mem);
    free(w.cells);
    free(w.pts);
    return res->status ? -1 : 0;
}

/* iter_np (align.c:4556-4917), the distance part: the O(np) waves between A[0..M) and
 * B[0..N) with substitutions.  F0/F1/F2 are waves D, D-1, D-2 indexed by diagonal (the
 * reference keeps every wave for its traceback; the distance needs three).  A and B are
 * separate buffers here, as LAcheck and LAshow load them, so no self-comparison borders.
 * Each of the three buffers holds 2*R+1 diagonals centred on 0, R >= M + N + 4. */
static int iter_np_dist(const uint8_t* A, int M, const uint8_t* B, int N, int* b0, int* b1, int* b2)
{
    int del = M - N, low, hgh, D, k, j, i, am, ac, ap;
    int *F0, *F1, *F2, *nf;
    if (del >= 0)
    {
        low = 0;
        hgh = del;
    }
    else
    {
        low = del;
        hgh = 0;
    }
    F1 = b1;
    F0 = b2;
    nf = b0;
    for (k = low - 1; k <= hgh + 1; k++)
        F1[k] = F0[k] = -2;
    F0[0] = -1;
    low += 1;
    hgh -= 1;
    for (D = 0;; D++)
    {
        int* t = nf;
        F2 = F1;
        F1 = F0;
        F0 = t;
        nf = F2;
        if ((D & 1) == 0)
        {
            low -= 1;
            hgh += 1;
        }
        F0[hgh + 1] = F0[low - 1] = -2;
#define FS(AP, AM)                                    \
    ap = (AP);                                        \
    am = (AM);                                        \
    ac = F1[k] + 1;                                   \
    if (ac < am)                                      \
        j = (ap < am) ? am : ap;                      \
    else if (ap < ac)                                 \
        j = ac;                                       \
    else                                              \
        j = ap;                                       \
    i = M - k;                                        \
    {                                                 \
        int lim = (N < i) ? N : i;                    \
        while (j < lim && B[j] == A[j + k])           \
            j += 1;                                   \
    }                                                 \
    F0[k] = j;
        j = -2;
        for (k = hgh; k > del; k--)
        {
            FS(j + 1, F2[k - 1])
        }
        j = -2;
        for (k = low; k < del; k++)
        {
            FS(F2[k + 1] + 1, j)
        }
        k = del;
        FS(F0[del + 1] + 1, j)
#undef FS
        if (F0[del] >= N)
            break;
    }
    return D + abs(del);
}

/* Compute_Trace_PTS (align.c:5286-5397): exact differences of a .las record, segment by
 * segment between its trace points.  aseq/bseq point at the reads' first bases (bseq
 * already complemented for a COMP record). */
int or_trace_pts_diffs(const uint8_t* aseq, const uint8_t* bseq, int alen, int blen, int abpos, int bbpos, int aepos,
                       int bepos, const uint8_t* trace8, const uint16_t* trace16, int tlen, int tspace,
                       int32_t* diffs_out)
{
    (void)alen;
    (void)blen;
    int nmax = 0, dmax = 0;
    for (int d = 1; d < tlen; d += 2)
    {
        int dv = trace8 ? trace8[d - 1] : trace16[d - 1];
        int nv = trace8 ? trace8[d] : trace16[d];
        if (dv > dmax)
            dmax = dv;
        if (nv > nmax)
            nmax = nv;
    }
    if (tlen <= 1)
        nmax = bepos - bbpos;
    int R = tspace + nmax + (aepos - abpos) + (bepos - bbpos) + 16;
    int* mem = (int*)malloc(sizeof(int) * 3 * (2 * R + 1));
    int *b0 = mem + R, *b1 = mem + (2 * R + 1) + R, *b2 = mem + 2 * (2 * R + 1) + R;
    int diffs = 0, ab = abpos, ae = (abpos / tspace) * tspace, bb = bbpos, be;
    for (int i = 1; i < tlen - 2; i += 2)
    {
        ae = ae + tspace;
        be = bb + (trace8 ? trace8[i] : trace16[i]);
        diffs += iter_np_dist(aseq + ab, ae - ab, bseq + bb, be - bb, b0, b1, b2);
        ab = ae;
        bb = be;
    }
    diffs += iter_np_dist(aseq + ab, aepos - ab, bseq + bb, bepos - bb, b0, b1, b2);
    free(mem);
    *diffs_out = diffs;
    return 0;
}

void or_free(void* p)
{
    free(p);
}

void or_free_result(or_result* r)
{
    free(r->ovl);
    free(r->trace);
    memset(r, 0, sizeof(*r));
}
