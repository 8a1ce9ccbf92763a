/* daligner2_main.c -- the daligner2 (modimizer seeds) command line over the B200 path.
 *
 * Same options, defaults, validation and output files as MARVEL's daligner2
 * (dalign2/daligner.c:454-801, the .las writer dalign2/ovlbuffer.c:226-421): targets after
 * the subject are blocks or, when a bare number, blocks of the subject's DB; -P<dir> roots the
 * per-block output folders <dir>_<block>/; -S skips a comparison whose .las files exist and
 * read through.  -T is validated and otherwise unused (the GPU path has no host threads).
 */
#include <errno.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <sys/stat.h>
#include <unistd.h>

#include "dazz_db.h"
#include "gpudalign.h"

static const char* Prog = "daligner";

static void usage(void)
{
    fprintf(stderr, "Usage: daligner [-vAIS] [-k<int(16)>] [-w<int(6)>] [-h<int(50)>] [-t<int>] [-M<int>]\n");
    fprintf(stderr, "                [-e<double(.75)] [-l<int(1500)>] [-s<int(100)>] [-H<int>]\n");
    fprintf(stderr, "                [-T<int(4)>] [-P<dir(/tmp)>] [-m<track>]+\n");
    fprintf(stderr, "                <subject:db> <target:db> ...\n");
    exit(1);
}

static int64_t physical_memory(void)
{
    long pages = sysconf(_SC_PHYS_PAGES), psz = sysconf(_SC_PAGESIZE);
    return (pages > 0 && psz > 0) ? (int64_t)pages * psz : 0;
}

#define GPU(call)                                               \
    do                                                          \
    {                                                           \
        if ((call) < 0)                                         \
        {                                                       \
            fprintf(stderr, "%s: %s\n", Prog, gd_last_error()); \
            exit(1);                                            \
        }                                                       \
    } while (0)

/* the argument parsers of the reference's DB.h (ARG_POSITIVE, ARG_NON_NEGATIVE, ARG_REAL) */
static int arg_int(const char* a, const char* name, int positive)
{
    char* e;
    long v = strtol(a + 2, &e, 10);
    if (*e != '\0' || a[2] == '\0')
    {
        fprintf(stderr, "%s: -%c argument is not an integer\n", Prog, a[1]);
        exit(1);
    }
    if (positive ? v <= 0 : v < 0)
    {
        fprintf(stderr, "%s: %s must be %s (%d)\n", Prog, name, positive ? "positive" : "non-negative", (int)v);
        exit(1);
    }
    return (int)v;
}

/* Root(path, ".db") and split_blockname (dalign2/ovlbuffer.c:409-421) */
static void root_of(const char* path, char* out, size_t n)
{
    const char* s = strrchr(path, '/');
    snprintf(out, n, "%s", s ? s + 1 : path);
    size_t L = strlen(out);
    if (L > 3 && strcmp(out + L - 3, ".db") == 0)
        out[L - 3] = 0;
}

static int split_blockname(const char* block, char* root, size_t n)
{
    const char* dot = strrchr(block, '.');
    if (dot == NULL)
    {
        snprintf(root, n, "%s", block);
        return 0;
    }
    snprintf(root, n, "%.*s", (int)(dot - block), block);
    return atoi(dot + 1);
}

static int mkdir_p(const char* path)
{
    char p[4096];
    snprintf(p, sizeof p, "%s", path);
    for (char* c = p + 1; *c; c++)
        if (*c == '/')
        {
            *c = '\0';
            if (mkdir(p, S_IRWXU) != 0 && errno != EEXIST)
                return -1;
            *c = '/';
        }
    return (mkdir(p, S_IRWXU) != 0 && errno != EEXIST) ? -1 : 0;
}

/* pathLas (dalign2/ovlbuffer.c:226-266) */
static void path_las(const char* base, const char* ar, int ai, const char* br, int bi, char* out, size_t n)
{
    if (ai > 0 && bi > 0)
    {
        char prefix[4096];
        size_t L = strlen(base);
        if (L > 0 && base[L - 1] == '/')
            snprintf(prefix, sizeof prefix, "%s%05d", base, ai);
        else
            snprintf(prefix, sizeof prefix, "%s_%05d", base, ai);
        if (mkdir_p(prefix) != 0)
        {
            fprintf(stderr, "failed to create %s\n", prefix);
            exit(1);
        }
        snprintf(out, n, "%s/%s.%d.%s.%d.las", prefix, ar, ai, br, bi);
    }
    else if (ai > 0)
        snprintf(out, n, "%s/%s.%d.%s.las", base, ar, ai, br);
    else if (bi > 0)
        snprintf(out, n, "%s/%s.%s.%d.las", base, ar, br, bi);
    else
        snprintf(out, n, "%s/%s.%s.las", base, ar, br);
}

/* a .las file that opens and whose records run exactly to its end (is_valid_las's test) */
static int valid_las(const char* path)
{
    FILE* f = fopen(path, "rb");
    if (f == NULL)
        return 0;
    int64_t n;
    int32_t ts;
    int ok = fread(&n, 8, 1, f) == 1 && fread(&ts, 4, 1, f) == 1 && n >= 0 && ts > 0;
    int tb = ts <= 125 ? 1 : 2;
    for (int64_t i = 0; ok && i < n; i++)
    {
        int32_t rec[10];
        ok = fread(rec, 40, 1, f) == 1 && rec[0] >= 0 && fseek(f, (long)rec[0] * tb, SEEK_CUR) == 0;
    }
    if (ok)
    {
        long here = ftell(f);
        fseek(f, 0, SEEK_END);
        ok = ftell(f) == here;
    }
    fclose(f);
    return ok;
}

static void write_las(const char* path, const gd_overlap* r, int64_t from, int64_t to, const uint8_t* trace,
                      int tspace)
{
    FILE* f = fopen(path, "wb");
    if (f == NULL)
    {
        fprintf(stderr, "[ERROR] - Write_Overlap_Buffer: Cannot open file %s for writing\n", path);
        exit(1);
    }
    int64_t n = to - from;
    int32_t ts = tspace;
    int tb = tspace <= 125 ? 1 : 2;
    fwrite(&n, 8, 1, f);
    fwrite(&ts, 4, 1, f);
    for (int64_t i = from; i < to; i++)
    {
        fwrite(r + i, 40, 1, f);
        fwrite(trace + r[i].toff, tb, (size_t)r[i].tlen, f);
    }
    fclose(f);
}

/* Write_Overlap_Buffer (dalign2/ovlbuffer.c:282-421) from the device's sorted buffer */
static void write_buffer(gd_context* ctx, const char* base, const char* ablock, const char* bblock, int last_read,
                         int symmetric, int tspace)
{
    int64_t tbytes = 0;
    int64_t n = gd_sort_overlaps(ctx, &tbytes);
    GPU(n);
    gd_overlap* r = (gd_overlap*)malloc(sizeof(gd_overlap) * (size_t)(n + 1));
    uint8_t* tr = (uint8_t*)malloc((size_t)tbytes + 16);
    if (n > 0)
        GPU(gd_get_overlaps(ctx, r, tr, n, tbytes));
    char ar[1024], br[1024], p1[8192], p2[8192];
    int ai = split_blockname(ablock, ar, sizeof ar), bi = split_blockname(bblock, br, sizeof br);
    if (strcmp(ablock, bblock) == 0 || !symmetric)
    {
        path_las(base, ar, ai, br, bi, p1, sizeof p1);
        write_las(p1, r, 0, n, tr, tspace);
    }
    else
    {
        p1[0] = p2[0] = 0;
        if (ai > 0)
            path_las(base, ar, ai, br, bi, p1, sizeof p1);
        if (bi > 0)
            path_las(base, br, bi, ar, ai, p2, sizeof p2);
        if (bi < ai)
        {
            char t[8192];
            strcpy(t, p1);
            strcpy(p1, p2);
            strcpy(p2, t);
        }
        int64_t j = 0;
        while (j < n && r[j].aread <= last_read)
            j++;
        write_las(p1, r, 0, j, tr, tspace);
        write_las(p2, r, j, n, tr, tspace);
    }
    free(r);
    free(tr);
}

static gd_block as_gd(const dz_block* b)
{
    gd_block g = {b->bases, b->boff, b->rlen, b->nreads, b->maxlen, b->totlen, b->ufirst, b->mask_anno, b->mask_data};
    return g;
}

static void load(dz_block* b, const char* name, char** mask, int mtop, int kmer)
{
    char err[1024];
    if (dz_open_block(name, b, err, sizeof err))
    {
        fprintf(stderr, "%s: %s\n", Prog, err);
        exit(1);
    }
    for (int i = 0; i < mtop; i++)
        if (dz_add_mask(b, mask[i], err, sizeof err))
        {
            printf("unable to load track %s\n", mask[i]);
            exit(1);
        }
    for (int i = 0; i < b->nreads; i++)
        if (b->rlen[i] < kmer)
        {
            fprintf(stderr, "%s: Block %s contains reads < %dbp long !  Run DBsplit.\n", Prog, name, kmer);
            exit(1);
        }
}

int main(int argc, char* argv[])
{
    int VERBOSE = 0, SYMMETRIC = 1, IDENTITY = 0, SKIP_VALID = 0;
    int KMER_LEN = 16, HIT_MIN = 50, BIN_SHIFT = 6, MAX_REPS = 0, HGAP_MIN = 0, SPACING = 100, MINOVER = 1500;
    double AVE_ERROR = .75;
    int64_t MEM_LIMIT = physical_memory();
    const char* SORT_PATH = "/tmp";
    int MTOP = 0;
    char** MASK = (char**)malloc(sizeof(char*) * (size_t)(argc + 1));
    char** pos = (char**)malloc(sizeof(char*) * (size_t)(argc + 1));
    int npos = 0;

    for (int i = 1; i < argc; i++)
    {
        const char* a = argv[i];
        if (a[0] != '-')
        {
            pos[npos++] = argv[i];
            continue;
        }
        char* e;
        switch (a[1])
        {
        case 'k':
            KMER_LEN = arg_int(a, "K-mer length", 1);
            if (KMER_LEN > 32)
            {
                fprintf(stderr, "%s: K-mer length must be 32 or less\n", Prog);
                exit(1);
            }
            break;
        case 'w': BIN_SHIFT = arg_int(a, "Log of bin width", 1); break;
        case 'h': HIT_MIN = arg_int(a, "Hit threshold (in bp.s)", 1); break;
        case 't': MAX_REPS = arg_int(a, "Tuple supression frequency", 1); break;
        case 'H': HGAP_MIN = arg_int(a, "HGAP threshold (in bp.s)", 1); break;
        case 'e':
            AVE_ERROR = strtod(a + 2, &e);
            if (*e != '\0' || a[2] == '\0')
            {
                fprintf(stderr, "%s: -%c argument is not a real number\n", Prog, a[1]);
                exit(1);
            }
            if (AVE_ERROR < .7 || AVE_ERROR >= 1.)
            {
                fprintf(stderr, "%s: Average correlation must be in [.7,1.) (%g)\n", Prog, AVE_ERROR);
                exit(1);
            }
            break;
        case 'l': MINOVER = arg_int(a, "Minimum alignment length", 1); break;
        case 's': SPACING = arg_int(a, "Trace spacing", 1); break;
        case 'M': MEM_LIMIT = (int64_t)arg_int(a, "Memory allocation (in Gb)", 0) * 0x40000000ll; break;
        case 'm': MASK[MTOP++] = argv[i] + 2; break;
        case 'P': SORT_PATH = argv[i] + 2; break;
        case 'T': (void)arg_int(a, "Number of threads", 1); break;
        default:
            for (int k = 1; a[k] != '\0'; k++)
            {
                if (strchr("vAIS", a[k]) == NULL)
                {
                    fprintf(stderr, "%s: -%c is an illegal option\n", Prog, a[k]);
                    exit(1);
                }
                VERBOSE |= a[k] == 'v';
                SYMMETRIC &= a[k] != 'A';
                IDENTITY |= a[k] == 'I';
                SKIP_VALID |= a[k] == 'S';
            }
        }
    }
    if (npos < 2)
        usage();
    MINOVER *= 2;
    if (mkdir(SORT_PATH, S_IRWXU) != 0 && errno != EEXIST)
    {
        fprintf(stderr, "%s: Could not create directory %s\n", Prog, SORT_PATH);
        exit(1);
    }

    gd_context* ctx = gd_create();
    if (!ctx)
    {
        fprintf(stderr, "%s: %s\n", Prog, gd_last_error());
        exit(1);
    }
    GPU(gd_set_variant(ctx, 2, HGAP_MIN));
    GPU(gd_set_filter_params(ctx, KMER_LEN, BIN_SHIFT, MAX_REPS, HIT_MIN));
    GPU(gd_set_globals(ctx, MINOVER, IDENTITY, (uint64_t)MEM_LIMIT));

    const char* afile = pos[0];
    dz_block A, B;
    load(&A, afile, MASK, MTOP, KMER_LEN);
    char aroot[1024], broot[1024], adir[4096];
    root_of(afile, aroot, sizeof aroot);
    snprintf(adir, sizeof adir, "%s", afile);
    char* sl = strrchr(adir, '/');
    if (sl)
        sl[0] = 0;
    else
        strcpy(adir, ".");
    GPU(gd_new_align_spec(ctx, AVE_ERROR, SPACING, A.freq, SYMMETRIC, 0, 0));
    gd_block ga = as_gd(&A);
    GPU(gd_load_block(ctx, 0, &ga));
    int indexed = 0;

    for (int i = 1; i < npos; i++)
    {
        /* a bare number names a block of the subject's DB (dalign2/daligner.c:668-679) */
        char bfile[4096];
        char* endp;
        strtol(pos[i], &endp, 10);
        if (*endp == '\0')
        {
            snprintf(bfile, sizeof bfile, "%s", afile);
            char* dot = strrchr(bfile, '.');
            if (dot)
                snprintf(dot + 1, sizeof bfile - (size_t)(dot + 1 - bfile), "%s", pos[i]);
        }
        else
            snprintf(bfile, sizeof bfile, "%s", pos[i]);
        root_of(bfile, broot, sizeof broot);
        char bdir[4096];
        snprintf(bdir, sizeof bdir, "%s", bfile);
        sl = strrchr(bdir, '/');
        if (sl)
            sl[0] = 0;
        else
            strcpy(bdir, ".");
        const int same = strcmp(adir, bdir) == 0 && strcmp(aroot, broot) == 0;
        if (!indexed)
        {
            if (VERBOSE)
                printf("\nBuilding index for %s\n", aroot);
            GPU(gd_sort_kmers(ctx, 0));
            indexed = 1;
        }
        if (SKIP_VALID)
        {
            char ar[1024], br[1024], p1[8192], p2[8192];
            int ai = split_blockname(aroot, ar, sizeof ar), bi = split_blockname(broot, br, sizeof br);
            path_las(SORT_PATH, ar, ai, br, bi, p1, sizeof p1);
            if (!same)
            {
                path_las(SORT_PATH, br, bi, ar, ai, p2, sizeof p2);
                if (valid_las(p1) && valid_las(p2))
                    continue;
            }
            else if (valid_las(p1))
                continue;
        }
        if (!same)
        {
            load(&B, bfile, MASK, MTOP, KMER_LEN);
            gd_block gb = as_gd(&B);
            GPU(gd_load_block(ctx, 1, &gb));
            if (VERBOSE)
                printf("\nBuilding index for %s\n", broot);
            GPU(gd_sort_kmers(ctx, 1));
            GPU(gd_complement_block(ctx, 1, 2));
            GPU(gd_match_filter2(ctx, 1, 2, 0));
            int lastRead = (B.part < A.part) ? B.ufirst + B.nreads - 1 : A.ufirst + A.nreads - 1;
            write_buffer(ctx, SORT_PATH, aroot, broot, lastRead, SYMMETRIC, SPACING);
            dz_free(&B);
        }
        else
        {
            GPU(gd_complement_block(ctx, 0, 2));
            GPU(gd_match_filter2(ctx, 0, 2, 1));
            write_buffer(ctx, SORT_PATH, aroot, aroot, A.ufirst + A.nreads - 1, SYMMETRIC, SPACING);
        }
        if (VERBOSE)
        {
            gd_stats st;
            gd_get_stats(ctx, &st);
            printf("\n   %lld + %lld hits, %lld + %lld seed hits, %lld overlaps\n", (long long)st.hits[0],
                   (long long)st.hits[1], (long long)st.seeds[0], (long long)st.seeds[1], (long long)st.records);
        }
        GPU(gd_reset_overlap_buffer(ctx));
    }
    dz_free(&A);
    gd_destroy(ctx);
    free(MASK);
    free(pos);
    exit(0);
}
