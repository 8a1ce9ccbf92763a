/* compat.c -- MARVEL's daligner library interface under its own names, over the B200 path.
 *
 * These are the entry points dalign/filter.h:67-71 and dalign/align.h:131-344 declare, with
 * the reference's signatures, so that a program written against the reference's filter.c
 * and align.c -- dalign/daligner.c itself -- links against libgpudalign.so unchanged:
 *
 *   Set_Filter_Params, Sort_Kmers, Match_Filter       (dalign/filter.c:119-139, 698-903, 1997-2407)
 *   New_Align_Spec, Free_Align_Spec                   (dalign/align.c:214-279)
 *   New_Work_Data, Free_Work_Data                     (dalign/align.h:131-133)
 *   Local_Alignment                                   (dalign/align.c:1922-2060)
 *   Compute_Trace_PTS                                 (dalign/align.c:5286-5397)
 *   Write_Overlap_Buffer, Reset_Overlap_Buffer        (dalign/align.c:5815-6056)
 *
 * The filter state the reference keeps in file statics lives in one process-wide
 * gd_context on the current CUDA device, created by the first of these calls.  The
 * reference's driver globals (VERBOSE, BIASED, MINOVER, IDENTITY, MEM_LIMIT, MEM_PHYSICAL,
 * defined by dalign/daligner.c:60-71) are read through weak references: a program that
 * defines them is read, one that does not gets 0.
 *
 * Index handles: Sort_Kmers loads the block into a device slot (the first block it sees
 * into slot 0, the A slot; others alternately into slots 1 and 2), builds its index there
 * and returns a small handle naming the slot instead of the reference's host KmerPos
 * array -- callers only pass it back to Match_Filter.  As in the reference, Match_Filter
 * frees the B handle when it differs from the A handle (dalign/filter.c:2194-2204,
 * 2358-2359), and NULL stands for an empty index.
 *
 * Errors: like the reference, a failing call prints a message and exits with status 1
 * (EXIT, db/DB.h:36), except Local_Alignment, which returns NULL as documented
 * (dalign/align.h:186-187).
 *
 * Local_Alignment and Compute_Trace_PTS run one alignment per call on the device (the
 * batch entry points gd_local_alignment_batch and gd_compute_trace_pts are the fast way);
 * Local_Alignment takes the single-diagonal seeds without borders that daligner's filter
 * passes (low == hgh, lbord = hbord = -1, dalign/filter.c:1805), and Compute_Trace_PTS
 * sets path->diffs (the exact difference count between the trace points, what LAcheck -a
 * checks) without building the full trace of the alignment.
 */
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "gd_report.h"
#include "gpudalign.h"
#include "gpudalign_compat.h"

/* the reference's records under their own names (layouts in gpudalign_compat.h) */
typedef gdc_HITS_READ HITS_READ;
typedef gdc_HITS_TRACK HITS_TRACK;
typedef gdc_HITS_DB HITS_DB;
typedef gdc_Path Path;
typedef gdc_Alignment Alignment;

_Static_assert(sizeof(HITS_READ) == 32, "HITS_READ layout");
_Static_assert(sizeof(HITS_TRACK) == 40, "HITS_TRACK layout");
_Static_assert(sizeof(HITS_DB) == 88, "HITS_DB layout");
_Static_assert(sizeof(Path) == 32, "Path layout");
_Static_assert(sizeof(Alignment) == 40, "Alignment layout");

/* ---- the reference driver's globals, when the program defines them */
extern int VERBOSE __attribute__((weak));
extern int BIASED __attribute__((weak));
extern int MINOVER __attribute__((weak));
extern int IDENTITY __attribute__((weak));
extern uint64_t MEM_LIMIT __attribute__((weak));
extern uint64_t MEM_PHYSICAL __attribute__((weak));

#define GLOBAL(x, dflt) (&(x) ? (x) : (dflt))

#define INDEX_MAGIC 0x6764784bu  /* "Kxdg" */
#define SPEC_MAGIC 0x67647370u
#define WORK_MAGIC 0x6764776bu

typedef struct
{
    uint32_t magic;
    int slot;
} KmerIndex;

typedef struct
{
    uint32_t magic;
    gd_context* ctx;
    int tspace;
} SpecHandle;

typedef struct
{
    uint32_t magic;
    Path bpath;        /* the B-path Local_Alignment returns */
    uint16_t* atrace;  /* the A-path's trace points (align->path->trace) */
    uint16_t* btrace;
    int32_t* out;      /* one seed's batch output */
    uint16_t* tbuf;    /* the batch's trace rows */
    int64_t cap;       /* uint16 capacity of atrace / btrace, half of tbuf */
    gd_context* vctx;  /* Compute_Trace_PTS's own context (two one-read blocks) */
    int vtspace;
    uint8_t* seq;      /* sentinel-bounded copies of the reads for the verifier */
    int64_t seqcap;
} WorkHandle;

static gd_context* g_ctx;
static const HITS_DB* g_ablock;
static int g_next = 1;
static int g_biased = -1;
static int g_kmer = 14, g_suppress = 0;

static void die(const char* where)
{
    fprintf(stderr, "%s: %s\n", where, gd_last_error());
    exit(1);
}

static gd_context* filter_ctx(void)
{
    if (!g_ctx)
    {
        g_ctx = gd_create();
        if (!g_ctx)
            die("daligner");
    }
    return g_ctx;
}

int Set_Filter_Params(int kmer, int binshift, int suppress, int hitmin)
{
    if (kmer <= 1)
        return 1;
    if (gd_set_filter_params(filter_ctx(), kmer, binshift, suppress, hitmin) < 0)
        return 1;
    g_kmer = kmer;
    g_suppress = suppress;
    return 0;
}

void* New_Align_Spec(double ave_corr, int trace_space, float* freq, int nthreads, int symmetric, int only_identity,
                     int no_trace_points)
{
    (void)nthreads;  /* the device path has no host thread count */
    gd_context* ctx = filter_ctx();
    if (gd_new_align_spec(ctx, ave_corr, trace_space, freq, symmetric, only_identity, no_trace_points) < 0)
        die("New_Align_Spec");
    SpecHandle* h = (SpecHandle*)malloc(sizeof(SpecHandle));
    if (!h)
    {
        fprintf(stderr, "New_Align_Spec: out of memory\n");
        exit(1);
    }
    h->magic = SPEC_MAGIC;
    h->ctx = ctx;
    h->tspace = trace_space;
    return h;
}

void Free_Align_Spec(void* spec)
{
    SpecHandle* h = (SpecHandle*)spec;
    if (h && h->magic == SPEC_MAGIC)
    {
        h->magic = 0;
        free(h);
    }
}

static SpecHandle* spec_of(void* spec, const char* where)
{
    SpecHandle* h = (SpecHandle*)spec;
    if (!h || h->magic != SPEC_MAGIC)
    {
        fprintf(stderr, "%s: not an Align_Spec made by New_Align_Spec\n", where);
        exit(1);
    }
    return h;
}

void* Sort_Kmers(HITS_DB* block, int* len)
{
    gd_context* ctx = filter_ctx();
    const int biased = GLOBAL(BIASED, 0) != 0;
    if (biased != g_biased)
    {
        if (gd_set_biased(ctx, biased) < 0)
            die("Sort_Kmers");
        g_biased = biased;
    }
    int slot;
    if (g_ablock == NULL || block == g_ablock)
    {
        g_ablock = block;
        slot = 0;
    }
    else
    {
        slot = g_next;
        g_next = 3 - g_next;
    }
    const int n = block->nreads;
    int64_t* boff = (int64_t*)malloc(sizeof(int64_t) * (n + 1));
    int32_t* rlen = (int32_t*)malloc(sizeof(int32_t) * (n + 1));
    if (!boff || !rlen)
    {
        fprintf(stderr, "Sort_Kmers: out of memory\n");
        exit(1);
    }
    for (int i = 0; i <= n; i++)
        boff[i] = block->reads[i].boff;
    for (int i = 0; i < n; i++)
        rlen[i] = block->reads[i].rlen;
    gd_block g;
    g.bases = (const uint8_t*)block->bases;
    g.boff = boff;
    g.rlen = rlen;
    g.nreads = n;
    g.maxlen = block->maxlen;
    g.totlen = block->totlen;
    g.ufirst = block->ufirst;
    /* the first track is the (merged) mask, its anno already in int units
       (dalign/daligner.c:425-440, dalign/filter.c:764) */
    g.mask_anno = block->tracks ? (const int64_t*)block->tracks->anno : NULL;
    g.mask_data = block->tracks ? (const int32_t*)block->tracks->data : NULL;
    if (gd_load_block(ctx, slot, &g) < 0 || gd_sort_kmers(ctx, slot) < 0)
        die("Sort_Kmers");
    const int64_t slots = boff[n] - (int64_t)g_kmer * n;
    free(boff);
    free(rlen);
    const uint64_t mem_limit = GLOBAL(MEM_LIMIT, 0);
    gd_report_index(ctx, slot, slots, g_suppress, (int64_t)mem_limit, mem_limit == GLOBAL(MEM_PHYSICAL, 0),
                    GLOBAL(VERBOSE, 0));
    gd_stats st;
    gd_get_stats(ctx, &st);
    if (slots <= 0 || st.kmers[slot] <= 0)
    {
        *len = 0;
        return NULL;
    }
    *len = (int)st.kmers[slot];
    KmerIndex* h = (KmerIndex*)malloc(sizeof(KmerIndex));
    if (!h)
    {
        fprintf(stderr, "Sort_Kmers: out of memory\n");
        exit(1);
    }
    h->magic = INDEX_MAGIC;
    h->slot = slot;
    return h;
}

static int slot_of(void* table)
{
    KmerIndex* h = (KmerIndex*)table;
    if (h->magic != INDEX_MAGIC)
    {
        fprintf(stderr, "Match_Filter: not an index made by Sort_Kmers\n");
        exit(1);
    }
    return h->slot;
}

void Match_Filter(char* aname, HITS_DB* ablock, char* bname, HITS_DB* bblock, void* atable, int alen, void* btable,
                  int blen, int comp, void* asettings)
{
    SpecHandle* sp = spec_of(asettings, "Match_Filter");
    gd_context* ctx = sp->ctx;
    const int self = aname == bname;  /* MG_self, dalign/filter.c:2076 */
    const int verbose = GLOBAL(VERBOSE, 0);
    const uint64_t mem_limit = GLOBAL(MEM_LIMIT, 0);
    if (gd_set_globals(ctx, GLOBAL(MINOVER, 0), GLOBAL(IDENTITY, 0), mem_limit) < 0)
        die("Match_Filter");
    if (atable == NULL || btable == NULL || alen == 0 || blen == 0)
    {
        if (verbose)  /* the zero-work report (dalign/filter.c:2058-2066, 2388-2405) */
        {
            const double atot = (double)ablock->totlen, btot = (double)bblock->totlen;
            printf(comp ? "\nComparing %s to c(%s)\n" : "\nComparing %s to %s\n", aname, bname);
            printf("\n     0 %d-mers (%e of matrix)\n     0 seed hits (%e of matrix)\n     0 confirmed hits (%e of "
                   "matrix)\n",
                   g_kmer, 0. / atot / btot, 0. / atot / btot, 0. / atot / btot);
            fflush(stdout);
        }
    }
    else
    {
        const int bslot = slot_of(btable);
        slot_of(atable);
        int64_t tb = 0;
        const int64_t r0 = gd_num_overlaps(ctx, &tb);
        if (gd_match_filter(ctx, bslot, comp, self) < 0)
            die("Match_Filter");
        if (verbose)
            gd_report_match(ctx, aname, bname, comp, atable == btable, bslot, r0, (double)ablock->totlen,
                            (double)bblock->totlen, g_kmer, (int64_t)mem_limit);
    }
    if (btable != atable && btable != NULL)
    {
        ((KmerIndex*)btable)->magic = 0;
        free(btable);
    }
}

void Write_Overlap_Buffer(void* spec, int RUN_ID, char* ablock, char* bblock, int lastRead)
{
    SpecHandle* sp = spec_of(spec, "Write_Overlap_Buffer");
    if (gd_write_overlap_buffer(sp->ctx, RUN_ID, ablock, bblock, lastRead) < 0)
        die("Write_Overlap_Buffer");
}

void Reset_Overlap_Buffer(void* spec)
{
    SpecHandle* sp = spec_of(spec, "Reset_Overlap_Buffer");
    if (gd_reset_overlap_buffer(sp->ctx) < 0)
        die("Reset_Overlap_Buffer");
}

/* ---- single alignments */

void* New_Work_Data(void)
{
    WorkHandle* w = (WorkHandle*)calloc(1, sizeof(WorkHandle));
    if (w)
        w->magic = WORK_MAGIC;
    return w;
}

void Free_Work_Data(void* work)
{
    WorkHandle* w = (WorkHandle*)work;
    if (!w || w->magic != WORK_MAGIC)
        return;
    if (w->vctx)
        gd_destroy(w->vctx);
    free(w->atrace);
    free(w->btrace);
    free(w->out);
    free(w->tbuf);
    free(w->seq);
    w->magic = 0;
    free(w);
}

static int work_room(WorkHandle* w, int64_t half)
{
    if (half <= w->cap)
        return 0;
    uint16_t* a = (uint16_t*)realloc(w->atrace, sizeof(uint16_t) * half);
    if (a)
        w->atrace = a;
    uint16_t* b = (uint16_t*)realloc(w->btrace, sizeof(uint16_t) * half);
    if (b)
        w->btrace = b;
    uint16_t* t = (uint16_t*)realloc(w->tbuf, sizeof(uint16_t) * 2 * half);
    if (t)
        w->tbuf = t;
    if (!w->out)
        w->out = (int32_t*)malloc(sizeof(int32_t) * 12);
    if (!a || !b || !t || !w->out)
        return -1;
    w->cap = half;
    return 0;
}

Path* Local_Alignment(Alignment* align, void* work, void* spec, int low, int hgh, int anti, int lbord, int hbord)
{
    WorkHandle* w = (WorkHandle*)work;
    SpecHandle* sp = (SpecHandle*)spec;
    if (!w || w->magic != WORK_MAGIC || !sp || sp->magic != SPEC_MAGIC)
    {
        fprintf(stderr, "Local_Alignment: work or spec not made by New_Work_Data / New_Align_Spec\n");
        return NULL;
    }
    if (low != hgh || lbord >= 0 || hbord >= 0)
    {
        fprintf(stderr, "Local_Alignment: this build takes single-diagonal seeds without borders "
                        "(low == hgh, lbord = hbord = -1)\n");
        return NULL;
    }
    const int alen = align->alen, blen = align->blen;
    const int maxlen = alen > blen ? alen : blen;
    const int64_t half = 4 * ((int64_t)maxlen / sp->tspace + 2) + 16;
    if (work_room(w, half))
    {
        fprintf(stderr, "Local_Alignment: out of memory\n");
        return NULL;
    }
    /* the reads with their sentinels: aseq[-1] and aseq[alen] are 4, as in a loaded block */
    const int64_t aoff = 1, boff = 1;
    const int32_t al = alen, bl = blen, diag = low, an = anti;
    int64_t cells = 0;
    if (gd_local_alignment_batch(sp->ctx, (const uint8_t*)align->aseq - 1, alen + 2, (const uint8_t*)align->bseq - 1,
                                 blen + 2, &aoff, &al, &boff, &bl, &diag, &an, 1, (int)(align->flags & 1), w->out,
                                 w->tbuf, (int)(2 * half), &cells) < 0)
    {
        fprintf(stderr, "Local_Alignment: %s\n", gd_last_error());
        return NULL;
    }
    const int32_t* o = w->out;
    Path* ap = align->path;
    ap->abpos = o[0];
    ap->bbpos = o[1];
    ap->aepos = o[2];
    ap->bepos = o[3];
    ap->diffs = o[4];
    ap->tlen = o[5];
    memcpy(w->atrace, w->tbuf, sizeof(uint16_t) * o[5]);
    ap->trace = w->atrace;
    Path* bp = &w->bpath;
    bp->abpos = o[6];
    bp->bbpos = o[7];
    bp->aepos = o[8];
    bp->bepos = o[9];
    bp->diffs = o[10];
    bp->tlen = o[11];
    memcpy(w->btrace, w->tbuf + half, sizeof(uint16_t) * o[11]);
    bp->trace = w->btrace;
    return bp;
}

/* a one-read block: [4, read, 4] in w->seq at offset at */
static gd_block one_read(WorkHandle* w, int64_t at, const char* seq, int len, int64_t* boff, int32_t* rlen)
{
    uint8_t* s = w->seq + at;
    s[0] = 4;
    memcpy(s + 1, seq, (size_t)len);
    s[len + 1] = 4;
    boff[0] = 0;
    boff[1] = len + 1;
    rlen[0] = len;
    gd_block g;
    g.bases = s + 1;
    g.boff = boff;
    g.rlen = rlen;
    g.nreads = 1;
    g.maxlen = len;
    g.totlen = len;
    g.ufirst = 0;
    g.mask_anno = NULL;
    g.mask_data = NULL;
    return g;
}

int Compute_Trace_PTS(Alignment* align, void* work, int trace_spacing, int mode, int debug)
{
    (void)mode;  /* the difference count of an optimal alignment does not depend on the tie rule */
    (void)debug;
    WorkHandle* w = (WorkHandle*)work;
    if (!w || w->magic != WORK_MAGIC)
    {
        fprintf(stderr, "Compute_Trace_PTS: work not made by New_Work_Data\n");
        exit(1);
    }
    Path* p = align->path;
    if (!w->vctx)
    {
        w->vctx = gd_create();
        if (!w->vctx || gd_set_filter_params(w->vctx, 2, 0, 0, 0) < 0)
            die("Compute_Trace_PTS");
    }
    if (w->vtspace != trace_spacing)
    {
        float freq[4] = {.25f, .25f, .25f, .25f};
        if (gd_new_align_spec(w->vctx, .70, trace_spacing, freq, 1, 0, 0) < 0)
            die("Compute_Trace_PTS");
        w->vtspace = trace_spacing;
    }
    const int64_t need = (int64_t)align->alen + align->blen + 4 + 2 * (int64_t)p->tlen + 16;
    if (need > w->seqcap)
    {
        uint8_t* s = (uint8_t*)realloc(w->seq, (size_t)need);
        if (!s)
        {
            fprintf(stderr, "Compute_Trace_PTS: out of memory\n");
            exit(1);
        }
        w->seq = s;
        w->seqcap = need;
    }
    int64_t aboff[2], bboff[2];
    int32_t arlen[1], brlen[1];
    gd_block A = one_read(w, 0, align->aseq, align->alen, aboff, arlen);
    /* the caller has complemented bseq for a COMP alignment (dalign/align.h:96-101) */
    gd_block B = one_read(w, align->alen + 2, align->bseq, align->blen, bboff, brlen);
    if (gd_load_block(w->vctx, 0, &A) < 0 || gd_load_block(w->vctx, 1, &B) < 0)
        die("Compute_Trace_PTS");
    /* the trace points as the .las file stores them */
    const int tbytes = trace_spacing <= 125 ? 1 : 2;
    uint8_t* tb = w->seq + align->alen + align->blen + 4;
    const uint16_t* pts = (const uint16_t*)p->trace;
    for (int i = 0; i < p->tlen; i++)
    {
        if (tbytes == 1)
            tb[i] = (uint8_t)pts[i];
        else
        {
            tb[2 * i] = (uint8_t)(pts[i] & 0xff);
            tb[2 * i + 1] = (uint8_t)(pts[i] >> 8);
        }
    }
    gd_overlap o;
    memset(&o, 0, sizeof o);
    o.tlen = p->tlen;
    o.diffs = p->diffs;
    o.abpos = p->abpos;
    o.bbpos = p->bbpos;
    o.aepos = p->aepos;
    o.bepos = p->bepos;
    o.flags = align->flags & 1;
    o.toff = 0;
    int32_t diffs = 0;
    if (gd_compute_trace_pts(w->vctx, 0, 1, 1, &o, tb, 1, &diffs) < 0)
        die("Compute_Trace_PTS");
    p->diffs = diffs;
    return 0;
}
