/* dazz_db.c -- Dazzler DB blocks and mask tracks (see dazz_db.h). */
#include "dazz_db.h"

#include <stdarg.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <sys/stat.h>

#define HITS_DB_BYTES 88
#define HITS_READ_BYTES 32

static int fail(char* err, size_t n, const char* fmt, ...)
{
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(err, n, fmt, ap);
    va_end(ap);
    return -1;
}

/* split "dir/X.n.db" into dir, root X and block n (0 = whole DB), as Open_DB_Block does
 * (db/DB.c:365-416): a trailing ".<positive int>" names a block */
static void split_name(const char* path, char* dir, size_t dn, char* root, size_t rn, int* part)
{
    const char* slash = strrchr(path, '/');
    const char* base = slash ? slash + 1 : path;
    if (slash)
    {
        size_t l = (size_t)(slash - path);
        if (l >= dn)
            l = dn - 1;
        memcpy(dir, path, l);
        dir[l] = 0;
        if (l == 0)
            strcpy(dir, "/");
    }
    else
        snprintf(dir, dn, ".");
    snprintf(root, rn, "%s", base);
    size_t L = strlen(root);
    if (L > 3 && strcmp(root + L - 3, ".db") == 0)
        root[L - 3] = 0;
    *part = 0;
    char* dot = strrchr(root, '.');
    if (dot && dot[1] && dot[1] != '-')
    {
        char* end;
        long v = strtol(dot + 1, &end, 10);
        if (*end == 0 && v > 0)
        {
            *part = (int)v;
            *dot = 0;
        }
    }
}

int dz_open_block(const char* path, dz_block* b, char* err, size_t errlen)
{
    memset(b, 0, sizeof(*b));
    char fn[8192];
    split_name(path, b->dir, sizeof b->dir, b->root, sizeof b->root, &b->part);

    /* stub: files = N / N file lines / blocks = M / size = S / M+1 boundaries */
    snprintf(fn, sizeof fn, "%s/%s.db", b->dir, b->root);
    FILE* f = fopen(fn, "r");
    if (!f)
        return fail(err, errlen, "Could not open database %s", path);
    int nfiles = 0, nblocks = 0, ulast = 0, ufirst = 0;
    long long size = 0;
    char a[4096], c[4096];
    if (fscanf(f, "files = %d\n", &nfiles) != 1)
    {
        fclose(f);
        return fail(err, errlen, "Stub file (.db) of %s is junk", b->root);
    }
    for (int i = 0; i < nfiles; i++)
        if (fscanf(f, " %d %4095s %4095s\n", &ulast, a, c) != 3)
        {
            fclose(f);
            return fail(err, errlen, "Stub file (.db) of %s is junk", b->root);
        }
    int have_blocks = fscanf(f, "blocks = %d\n", &nblocks) == 1;
    if (have_blocks && fscanf(f, "size = %lld\n", &size) != 1)
    {
        fclose(f);
        return fail(err, errlen, "Stub file (.db) of %s is junk", b->root);
    }
    if (b->part > 0)
    {
        if (!have_blocks)
        {
            fclose(f);
            return fail(err, errlen, "DB %s has not yet been partitioned, cannot request a block !", b->root);
        }
        if (b->part > nblocks)
        {
            fclose(f);
            return fail(err, errlen, "DB %s has only %d blocks", b->root, nblocks);
        }
        for (int p = 1; p <= b->part; p++)
            if (fscanf(f, " %d\n", &ufirst) != 1)
            {
                fclose(f);
                return fail(err, errlen, "Stub file (.db) of %s is junk", b->root);
            }
        if (fscanf(f, " %d\n", &ulast) != 1)
        {
            fclose(f);
            return fail(err, errlen, "Stub file (.db) of %s is junk", b->root);
        }
    }
    fclose(f);

    snprintf(fn, sizeof fn, "%s/.%s.idx", b->dir, b->root);
    f = fopen(fn, "rb");
    if (!f)
        return fail(err, errlen, "Cannot open %s", fn);
    unsigned char hdr[HITS_DB_BYTES];
    if (fread(hdr, 1, HITS_DB_BYTES, f) != HITS_DB_BYTES)
    {
        fclose(f);
        return fail(err, errlen, "Index file (.idx) of %s is junk", b->root);
    }
    memcpy(&b->ureads, hdr + 0, 4);
    memcpy(b->freq, hdr + 4, 16);
    memcpy(&b->maxlen, hdr + 20, 4);
    memcpy(&b->totlen, hdr + 24, 8);
    float sum = b->freq[0] + b->freq[1] + b->freq[2] + b->freq[3];
    if (sum < 0.99f || sum > 1.01f)
    {
        fclose(f);
        return fail(err, errlen, "Index file frequencies sum to %.2f. File corrupt.", sum);
    }
    if (b->part <= 0)
    {
        ufirst = 0;
        ulast = b->ureads;
    }
    int n = ulast - ufirst;
    b->nreads = n;
    b->ufirst = ufirst;
    int64_t* foff = (int64_t*)malloc(sizeof(int64_t) * (n + 1));
    b->rlen = (int32_t*)malloc(sizeof(int32_t) * (n + 1));
    b->boff = (int64_t*)malloc(sizeof(int64_t) * (n + 1));
    if (!foff || !b->rlen || !b->boff)
    {
        fclose(f);
        free(foff);
        return fail(err, errlen, "out of memory");
    }
    if (fseeko(f, (off_t)HITS_DB_BYTES + (off_t)HITS_READ_BYTES * ufirst, SEEK_SET))
    {
        fclose(f);
        free(foff);
        return fail(err, errlen, "Index file (.idx) of %s is junk", b->root);
    }
    unsigned char rec[HITS_READ_BYTES];
    int64_t tot = 0;
    int maxlen = 0;
    for (int i = 0; i < n; i++)
    {
        if (fread(rec, 1, HITS_READ_BYTES, f) != HITS_READ_BYTES)
        {
            fclose(f);
            free(foff);
            return fail(err, errlen, "Index file (.idx) of %s is junk", b->root);
        }
        memcpy(&b->rlen[i], rec + 0, 4);
        memcpy(&foff[i], rec + 8, 8);
        tot += b->rlen[i];
        if (b->rlen[i] > maxlen)
            maxlen = b->rlen[i];
    }
    fclose(f);
    if (b->part > 0)
    {
        /* a block's maxlen and totlen come from its own reads (db/DB.c:519-536) */
        b->maxlen = maxlen;
        b->totlen = tot;
    }

    /* bases: decode 2-bit, a 4 before read 0 and after every read (db/DB.c:1349-1410) */
    b->boff[0] = 0;
    for (int i = 0; i < n; i++)
        b->boff[i + 1] = b->boff[i] + b->rlen[i] + 1;
    size_t total = (size_t)b->boff[n] + 1 + 64;
    b->buf = (uint8_t*)malloc(total);
    if (!b->buf)
    {
        free(foff);
        return fail(err, errlen, "out of memory for %zu bases", total);
    }
    memset(b->buf, 4, total);
    b->bases = b->buf + 33;
    snprintf(fn, sizeof fn, "%s/.%s.bps", b->dir, b->root);
    f = fopen(fn, "rb");
    if (!f)
    {
        free(foff);
        return fail(err, errlen, "Cannot open %s", fn);
    }
    size_t cap = 0;
    unsigned char* packed = NULL;
    for (int i = 0; i < n; i++)
    {
        int len = b->rlen[i];
        size_t clen = (size_t)(len + 3) / 4;
        if (clen > cap)
        {
            cap = clen * 2 + 1024;
            packed = (unsigned char*)realloc(packed, cap);
        }
        if (fseeko(f, (off_t)foff[i], SEEK_SET) || (clen && fread(packed, 1, clen, f) != clen))
        {
            fclose(f);
            free(foff);
            free(packed);
            return fail(err, errlen, "Read of .bps file failed");
        }
        uint8_t* s = b->bases + b->boff[i];
        for (int p = 0; p < len; p++)
            s[p] = (packed[p >> 2] >> (6 - 2 * (p & 3))) & 3;
        s[len] = 4;
    }
    fclose(f);
    free(packed);
    free(foff);
    return 0;
}

static int read_track_file(dz_block* b, const char* track, int64_t** anno_out, int32_t** data_out, char* err,
                           size_t errlen)
{
    char an[8192], dn[8192];
    FILE *af = NULL, *df = NULL;
    int ispart = 0;
    if (b->part > 0)
    {
        snprintf(an, sizeof an, "%s/.%s.%d.%s.anno", b->dir, b->root, b->part, track);
        snprintf(dn, sizeof dn, "%s/.%s.%d.%s.data", b->dir, b->root, b->part, track);
        af = fopen(an, "rb");
        ispart = af != NULL;
    }
    if (!af)
    {
        snprintf(an, sizeof an, "%s/.%s.%s.anno", b->dir, b->root, track);
        snprintf(dn, sizeof dn, "%s/.%s.%s.data", b->dir, b->root, track);
        af = fopen(an, "rb");
    }
    if (!af)
        return fail(err, errlen, "Unable to load track %s!", track);
    df = fopen(dn, "rb");
    int tracklen = 0, size = 0;
    if (fread(&tracklen, 4, 1, af) != 1 || fread(&size, 4, 1, af) != 1 || (size != 4 && size != 8) || !df)
    {
        fclose(af);
        if (df)
            fclose(df);
        return fail(err, errlen, "Track '%s' annotation file is junk", track);
    }
    int want = ispart ? b->nreads : b->ureads;
    if (tracklen != want)
    {
        fclose(af);
        fclose(df);
        return fail(err, errlen, "Track '%s' not same size as database (track: %d, db: %d)!", track, tracklen, want);
    }
    if (!ispart && b->part > 0)
        fseeko(af, (off_t)size * b->ufirst, SEEK_CUR);
    int n = b->nreads;
    int64_t* anno = (int64_t*)malloc(sizeof(int64_t) * (n + 1));
    for (int i = 0; i <= n; i++)
    {
        int64_t v = 0;
        if (size == 8)
        {
            if (fread(&v, 8, 1, af) != 1)
                goto junk;
        }
        else
        {
            int32_t v4;
            if (fread(&v4, 4, 1, af) != 1)
                goto junk;
            v = v4;
        }
        anno[i] = v;
    }
    {
        int64_t off = anno[0];
        /* byte offsets of (begin, end) int pairs: non-decreasing, whole pairs per read */
        for (int i = 0; i < n; i++)
            if (anno[i + 1] < anno[i] || (anno[i + 1] - anno[i]) % 8 != 0)
                goto junk;
        if (off < 0)
            goto junk;
        for (int i = 0; i <= n; i++)
            anno[i] = (anno[i] - off) / 4; /* bytes -> ints (dalign/daligner.c:425-428) */
        int64_t cnt = anno[n];
        int32_t* data = (int32_t*)malloc(sizeof(int32_t) * (cnt + 1));
        if (fseeko(df, (off_t)off, SEEK_SET) || (cnt && fread(data, 4, (size_t)cnt, df) != (size_t)cnt))
        {
            free(data);
            goto junk;
        }
        fclose(af);
        fclose(df);
        *anno_out = anno;
        *data_out = data;
        return 0;
    }
junk:
    free(anno);
    fclose(af);
    fclose(df);
    return fail(err, errlen, "Track '%s' data file is junk", track);
}

typedef struct
{
    int32_t b, e;
} Iv;

static int iv_cmp(const void* x, const void* y)
{
    const Iv* a = (const Iv*)x;
    const Iv* c = (const Iv*)y;
    return a->b != c->b ? (a->b < c->b ? -1 : 1) : (a->e < c->e ? -1 : a->e > c->e);
}

int dz_add_mask(dz_block* b, const char* track, char* err, size_t errlen)
{
    int64_t* anno;
    int32_t* data;
    if (read_track_file(b, track, &anno, &data, err, errlen))
        return -1;
    if (!b->mask_anno)
    {
        b->mask_anno = anno;
        b->mask_data = data;
        return 0;
    }
    /* union with the masks so far (Merge_Tracks, dalign/daligner.c:275-370): touching or
     * overlapping intervals merge; k-mers that span a boundary are masked either way */
    int n = b->nreads;
    int64_t cap = b->mask_anno[n] + anno[n] + 2;
    int64_t* na = (int64_t*)malloc(sizeof(int64_t) * (n + 1));
    int32_t* nd = (int32_t*)malloc(sizeof(int32_t) * cap);
    Iv* tmp = (Iv*)malloc(sizeof(Iv) * (cap / 2 + 2));
    int64_t top = 0;
    for (int r = 0; r < n; r++)
    {
        na[r] = top;
        int m = 0;
        for (int64_t j = b->mask_anno[r]; j < b->mask_anno[r + 1]; j += 2)
            tmp[m++] = (Iv){b->mask_data[j], b->mask_data[j + 1]};
        for (int64_t j = anno[r]; j < anno[r + 1]; j += 2)
            tmp[m++] = (Iv){data[j], data[j + 1]};
        qsort(tmp, m, sizeof(Iv), iv_cmp);
        int k = 0;
        for (int i = 0; i < m; i++)
        {
            if (k > 0 && tmp[i].b <= tmp[k - 1].e)
            {
                if (tmp[i].e > tmp[k - 1].e)
                    tmp[k - 1].e = tmp[i].e;
            }
            else
                tmp[k++] = tmp[i];
        }
        for (int i = 0; i < k; i++)
        {
            nd[top++] = tmp[i].b;
            nd[top++] = tmp[i].e;
        }
    }
    na[n] = top;
    free(tmp);
    free(anno);
    free(data);
    free(b->mask_anno);
    free(b->mask_data);
    b->mask_anno = na;
    b->mask_data = nd;
    return 0;
}

void dz_free(dz_block* b)
{
    free(b->buf);
    free(b->boff);
    free(b->rlen);
    free(b->mask_anno);
    free(b->mask_data);
    memset(b, 0, sizeof(*b));
}
