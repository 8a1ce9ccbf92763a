/* daligner_main.c -- the daligner command line over the B200 overlap path.
 *
 * Same options, defaults, validation, output directories and .las names as MARVEL's
 * daligner (dalign/daligner.c:27-58, 615-1029); the filter and aligner run on the GPU
 * through include/gpudalign.h.  Not supported: -D (dynamic mask server), rejected with a
 * message.  -j is validated and otherwise unused.
 */
#include <errno.h>
#include <getopt.h>
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <sys/stat.h>
#include <unistd.h>

#include "dazz_db.h"
#include "gpudalign.h"

static void usage(void)
{
    fprintf(stderr, "usage:  \n");
    fprintf(stderr, "daligner [-vbAIOT] [-k<int(14)>] [-w<int(6)>] [-h<int(35)>] [-t<int>] [-M<int>]\n");
    fprintf(stderr, "         [-e<double(.70)] [-l<int(1000)>] [-s<int(100)>] [-H<int>] [-j<int>]\n");
    fprintf(stderr, "         [-m<track>]+ <subject:db|dam> <target:db|dam> ...\n");
    fprintf(stderr, "         [-r<int()1>]\n");
}

/* Print_Number (db/DB.c:193-240): the number with its digits grouped by commas, right-aligned
 * in width characters (0: no padding) */
static void print_number(int64_t num, int width)
{
    char t[48];
    long long n = (long long)num;
    if (n < 1000ll)
        snprintf(t, sizeof t, "%lld", n);
    else if (n < 1000000ll)
        snprintf(t, sizeof t, "%lld,%03lld", n / 1000ll, n % 1000ll);
    else if (n < 1000000000ll)
        snprintf(t, sizeof t, "%lld,%03lld,%03lld", n / 1000000ll, (n % 1000000ll) / 1000ll, n % 1000ll);
    else
        snprintf(t, sizeof t, "%lld,%03lld,%03lld,%03lld", n / 1000000000ll, (n % 1000000000ll) / 1000000ll,
                 (n % 1000000ll) / 1000ll, n % 1000ll);
    printf("%*s", width, t);
}

/* Sort_Kmers' report under -v and its memory warning (dalign/filter.c:754-759, 865-892):
 * the k-mer slots of the block, the index left after masking and -t. */
static void report_index(gd_context* ctx, int slot, const dz_block* b, int kmer, int suppress, int64_t mem_limit,
                         int mem_physical, int verbose)
{
    const int64_t slots = b->boff[b->nreads] - (int64_t)kmer * b->nreads;
    if (slots <= 0)
        return;
    gd_stats st;
    gd_get_stats(ctx, &st);
    const int64_t kmers = st.kmers[slot];
    if (verbose)
    {
        printf("\n   Kmer count = ");
        print_number(slots, 0);
        printf("\n   Using %.2fGb of space\n", (1. * slots) / 33554432);
        if (suppress > 0)
        {
            printf("   Revised kmer count = ");
            print_number(kmers, 0);
            printf("\n");
        }
        printf("   Index occupies %.2fGb\n", (1. * kmers) / 67108864);
        fflush(stdout);
    }
    if (kmers > 0 && mem_limit > 0 && kmers > mem_limit / 64)
    {
        fprintf(stderr, "Warning: Block size too big, index occupies more than 1/4 of");
        if (mem_physical)
            fprintf(stderr, " physical memory (%.1fGb)\n", (1. * mem_limit) / 0x40000000ll);
        else
            fprintf(stderr, " desired memory allocation (%.1fGb)\n", (1. * mem_limit) / 0x40000000ll);
        fflush(stderr);
    }
}

/* Match_Filter's report under -v (dalign/filter.c:2058-2063, 2105-2106, 2158-2162, 2180-2189,
 * 2388-2405): the pair cap, the hits, the Local_Alignment calls (seed hits) and the overlaps
 * they added (confirmed hits).  same_index: A's index also served as B's. */
static void report_match(gd_context* ctx, const char* aname, const char* bname, int comp, int same_index, int bslot,
                         int64_t recs_before, const dz_block* a, const dz_block* b, int kmer, int64_t mem_limit)
{
    gd_stats st;
    gd_get_stats(ctx, &st);
    int64_t tb = 0;
    const int64_t recs = gd_num_overlaps(ctx, &tb);
    const int64_t alen = st.kmers[0], blen = st.kmers[bslot];
    int64_t nhits = 0, nfilt = 0, ncheck = 0;
    if (comp)
        printf("\nComparing %s to c(%s)\n", aname, bname);
    else
        printf("\nComparing %s to %s\n", aname, bname);
    if (alen > 0 && blen > 0)
    {
        printf("\n");
        if (mem_limit > 0)
            printf("   Capping mutual k-mer matches over %d (effectively -t%d)\n", st.limit[comp],
                   (int)sqrt(1. * st.limit[comp]));
        nhits = st.hits[comp];
        printf("   Hit count = ");
        print_number(nhits, 0);
        if (same_index || nhits >= blen)
            printf("\n   Highwater of %.2fGb space\n", (1. * (alen + 2 * nhits)) / 67108864);
        else
            printf("\n   Highwater of %.2fGb space\n", (1. * (alen + blen + nhits)) / 67108864);
        if (nhits > 0)
        {
            nfilt = st.seeds[comp];
            ncheck = recs - recs_before;
        }
    }
    const double atot = (double)a->totlen, btot = (double)b->totlen;
    int width = nhits <= 0 ? 1 : (int)log10((double)nhits) + 1;
    width += (width - 1) / 3;
    printf("\n     ");
    print_number(nhits, width);
    printf(" %d-mers (%e of matrix)\n     ", kmer, (1. * nhits / atot) / btot);
    print_number(nfilt, width);
    printf(" seed hits (%e of matrix)\n     ", (1. * nfilt / atot) / btot);
    print_number(ncheck, width);
    printf(" confirmed hits (%e of matrix)\n", (1. * ncheck / atot) / btot);
    fflush(stdout);
}

static int64_t num_overlaps(gd_context* ctx)
{
    int64_t tb = 0;
    return gd_num_overlaps(ctx, &tb);
}

static int64_t physical_memory(void)
{
    long pages = sysconf(_SC_PHYS_PAGES), psz = sysconf(_SC_PAGESIZE);
    return (pages > 0 && psz > 0) ? (int64_t)pages * psz : 0;
}

/* the block's output directory RRR_BBBBB (createSubdir, dalign/daligner.c:583-613) */
static int make_subdir(int run_id, int part)
{
    if (part == 0)
        return 0;
    char out[64];
    snprintf(out, sizeof out, "%03d_%05d", run_id, part);
    struct stat s;
    if (stat(out, &s) == -1)
    {
        if (errno == ENOENT)
            mkdir(out, S_IRWXU | S_IRGRP | S_IXGRP | S_IROTH | S_IXOTH);
        else
        {
            fprintf(stderr, "Cannot create output directory: %s\n", out);
            return -1;
        }
    }
    else if (!S_ISDIR(s.st_mode))
    {
        fprintf(stderr, "Output directory name: \"%s\" exist - but its not a directory\n", out);
        return -1;
    }
    return 0;
}

/* Root(file, ".db"): the name without directory and .db suffix */
static void root_of(const char* path, char* out, size_t n)
{
    const char* s = strrchr(path, '/');
    snprintf(out, n, "%s", s ? s + 1 : path);
    size_t L = strlen(out);
    if (L > 3 && strcmp(out + L - 3, ".db") == 0)
        out[L - 3] = 0;
}

static gd_block as_gd(const dz_block* b)
{
    gd_block g;
    g.bases = b->bases;
    g.boff = b->boff;
    g.rlen = b->rlen;
    g.nreads = b->nreads;
    g.maxlen = b->maxlen;
    g.totlen = b->totlen;
    g.ufirst = b->ufirst;
    g.mask_anno = b->mask_anno;
    g.mask_data = b->mask_data;
    return g;
}

#define GPU(call)                                                \
    do                                                           \
    {                                                            \
        if ((call) < 0)                                          \
        {                                                        \
            fprintf(stderr, "daligner: %s\n", gd_last_error());  \
            exit(1);                                             \
        }                                                        \
    } while (0)

static void load(dz_block* b, const char* name, char** mask, int mtop, int kmer)
{
    char err[1024];
    if (dz_open_block(name, b, err, sizeof err))
    {
        fprintf(stderr, "daligner: %s\n", err);
        exit(1);
    }
    for (int i = 0; i < mtop; i++)
        if (dz_add_mask(b, mask[i], err, sizeof err))
        {
            printf("[ERROR] - Unable to load track %s!\n", mask[i]);
            exit(1);
        }
    for (int i = 0; i < b->nreads; i++)
        if (b->rlen[i] < kmer)
        {
            fprintf(stderr, "[ERROR] - daligner: Block %s contains reads < %dbp long !  Run DBsplit.\n", name, kmer);
            exit(1);
        }
}

int main(int argc, char* argv[])
{
    int VERBOSE = 0, SYMMETRIC = 1, IDENTITY = 0, ONLY_IDENTITY = 0, NO_TRACE_POINTS = 0, BIASED = 0;
    int KMER_LEN = 14, HIT_MIN = 35, BIN_SHIFT = 6, MAX_REPS = 0, HGAP_MIN = 0, SPACING = 100, RUN_ID = 1;
    int MINOVER = 1000;
    double AVE_ERROR = .70;
    const int64_t MEM_PHYSICAL_BYTES = physical_memory();
    int64_t MEM_LIMIT = MEM_PHYSICAL_BYTES;
    int MTOP = 0, MMAX = 10;
    char** MASK = (char**)malloc(MMAX * sizeof(char*));
    int c;

    opterr = 0;
    while ((c = getopt(argc, argv, "vbOTAIk:w:h:t:M:e:l:s:H:D:m:r:j:")) != -1)
    {
        switch (c)
        {
        case 'v': VERBOSE = 1; break;
        case 'b': BIASED = 1; break;
        case 'T': NO_TRACE_POINTS = 1; break;
        case 'I': IDENTITY = 1; break;
        case 'O': IDENTITY = 1; ONLY_IDENTITY = 1; break;
        case 'A': SYMMETRIC = 0; break;
        case 'k': KMER_LEN = atoi(optarg); break;
        case 'w': BIN_SHIFT = atoi(optarg); break;
        case 'h': HIT_MIN = atoi(optarg); break;
        case 't': MAX_REPS = atoi(optarg); break;
        case 'H': HGAP_MIN = atoi(optarg); break;  /* accepted and, as in the reference, unused */
        case 'e': AVE_ERROR = atof(optarg); break;
        case 'l': MINOVER = atoi(optarg); break;
        case 's': SPACING = atoi(optarg); break;
        case 'j':
        {
            int tmp = atoi(optarg);
            if (tmp < 1)
            {
                fprintf(stderr, "invalid number of threads: %d. Must be a positive number.\n", tmp);
                exit(1);
            }
            if (tmp & (tmp - 1))
            {
                fprintf(stderr, "invalid number of threads: %d. Must be a power of 2.\n", tmp);
                exit(1);
            }
            break;
        }
        case 'D':
            fprintf(stderr, "daligner: -D (dynamic mask server) is not supported by the GPU path\n");
            exit(1);
        case 'M':
        {
            int tmp = atoi(optarg);
            if (tmp < 0)
                fprintf(stderr, "invalid memory limit of (%d)\n", tmp);
            MEM_LIMIT = (int64_t)tmp * 0x40000000ll;
            break;
        }
        case 'm':
            if (MTOP >= MMAX)
            {
                MMAX = (int)(1.2 * MTOP + 10);
                MASK = (char**)realloc(MASK, MMAX * sizeof(char*));
            }
            MASK[MTOP++] = optarg;
            break;
        case 'r':
            RUN_ID = atoi(optarg);
            if (RUN_ID < 0)
            {
                fprintf(stderr, "invalid run id of %d\n", RUN_ID);
                exit(1);
            }
            break;
        default:
            fprintf(stderr, "Unsupported option: %s\n", argv[optind - 1]);
            usage();
            exit(1);
        }
    }
    if (KMER_LEN < 0) { fprintf(stderr, "invalid kmer length of %d\n", KMER_LEN); exit(1); }
    if (BIN_SHIFT < 0) { fprintf(stderr, "invalid log of bin width of %d\n", BIN_SHIFT); exit(1); }
    if (HIT_MIN < 0) { fprintf(stderr, "invalid hit threshold of %d\n", HIT_MIN); exit(1); }
    if (MAX_REPS < 0) { fprintf(stderr, "invalid tuple supression frequency of %d\n", MAX_REPS); exit(1); }
    if (HGAP_MIN < 0) { fprintf(stderr, "invalid HGAP threshold of %d\n", HGAP_MIN); exit(1); }
    if (AVE_ERROR < .5 || AVE_ERROR >= 1.)
    {
        fprintf(stderr, "Average correlation must be in [.5,1.) (%g)\n", AVE_ERROR);
        exit(1);
    }
    if (MINOVER < 0) { fprintf(stderr, "invalid minimum alignmnet length of (%d)\n", MINOVER); exit(1); }
    if (SPACING < 0) { fprintf(stderr, "invalid trace spacing of (%d)\n", SPACING); exit(1); }
    if (optind + 2 > argc)
    {
        fprintf(stderr, "[ERROR] - at least one target and one subject block are required\n\n");
        usage();
        exit(1);
    }
    MINOVER *= 2;

    const int MEM_PHYSICAL = MEM_LIMIT == MEM_PHYSICAL_BYTES;
    gd_context* ctx = gd_create();
    if (!ctx)
    {
        fprintf(stderr, "daligner: %s\n", gd_last_error());
        exit(1);
    }
    GPU(gd_set_filter_params(ctx, KMER_LEN, BIN_SHIFT, MAX_REPS, HIT_MIN));
    GPU(gd_set_globals(ctx, MINOVER, IDENTITY, (uint64_t)MEM_LIMIT));
    GPU(gd_set_biased(ctx, BIASED));

    const char* afile = argv[optind];
    dz_block A, B;
    load(&A, afile, MASK, MTOP, KMER_LEN);
    char aroot[1024], broot[1024];
    root_of(afile, aroot, sizeof aroot);
    optind++;

    /* targets from another DB switch SYMMETRIC off (dalign/daligner.c:886-921) */
    if (SYMMETRIC)
        for (int i = optind; i < argc; i++)
            if (strcmp(afile, argv[i]) != 0)
            {
                root_of(argv[i], broot, sizeof broot);
                const char* adot = strrchr(aroot, '.');
                const char* bdot = strrchr(broot, '.');
                size_t al = adot ? (size_t)(adot - aroot + 1) : strlen(aroot);
                size_t bl = bdot ? (size_t)(bdot - broot + 1) : strlen(broot);
                if (strncmp(aroot, broot, al > bl ? al : bl) != 0)
                {
                    if (VERBOSE)
                        printf("[WARNING] - Daligner is performed on different databases (%s - %s). SYMMETRIC option "
                               "is disabled!\n",
                               aroot, broot);
                    SYMMETRIC = 0;
                    break;
                }
            }

    if (make_subdir(RUN_ID, A.part))
        exit(1);
    GPU(gd_new_align_spec(ctx, AVE_ERROR, SPACING, A.freq, SYMMETRIC, ONLY_IDENTITY, NO_TRACE_POINTS));
    gd_block ga = as_gd(&A);
    GPU(gd_load_block(ctx, 0, &ga));

    for (int i = optind; i < argc; i++)
    {
        const char* bfile = argv[i];
        if (i == optind)
        {
            if (VERBOSE)
                printf("\nBuilding index for %s\n", aroot);
            GPU(gd_sort_kmers(ctx, 0));
            report_index(ctx, 0, &A, KMER_LEN, MAX_REPS, MEM_LIMIT, MEM_PHYSICAL, VERBOSE);
        }
        if (strcmp(afile, bfile) != 0)
        {
            load(&B, bfile, MASK, MTOP, KMER_LEN);
            root_of(bfile, broot, sizeof broot);
            if (SYMMETRIC && make_subdir(RUN_ID, B.part))
                exit(1);
            gd_block gb = as_gd(&B);
            GPU(gd_load_block(ctx, 1, &gb));
            if (VERBOSE)
                printf("\nBuilding index for %s\n", broot);
            GPU(gd_sort_kmers(ctx, 1));
            report_index(ctx, 1, &B, KMER_LEN, MAX_REPS, MEM_LIMIT, MEM_PHYSICAL, VERBOSE);
            int64_t r0 = num_overlaps(ctx);
            GPU(gd_match_filter(ctx, 1, 0, 0));
            if (VERBOSE)
                report_match(ctx, aroot, broot, 0, 0, 1, r0, &A, &B, KMER_LEN, MEM_LIMIT);
            GPU(gd_complement_block(ctx, 1, 2));
            if (VERBOSE)
                printf("\nBuilding index for c(%s)\n", broot);
            GPU(gd_sort_kmers(ctx, 2));
            report_index(ctx, 2, &B, KMER_LEN, MAX_REPS, MEM_LIMIT, MEM_PHYSICAL, VERBOSE);
            r0 = num_overlaps(ctx);
            GPU(gd_match_filter(ctx, 2, 1, 0));
            if (VERBOSE)
                report_match(ctx, aroot, broot, 1, 0, 2, r0, &A, &B, KMER_LEN, MEM_LIMIT);
            int lastRead = (B.part < A.part) ? B.ufirst + B.nreads - 1 : A.ufirst + A.nreads - 1;
            GPU(gd_write_overlap_buffer(ctx, RUN_ID, aroot, broot, lastRead));
            dz_free(&B);
        }
        else
        {
            int64_t r0 = num_overlaps(ctx);
            GPU(gd_match_filter(ctx, 0, 0, 1));
            if (VERBOSE)
                report_match(ctx, aroot, aroot, 0, 1, 0, r0, &A, &A, KMER_LEN, MEM_LIMIT);
            GPU(gd_complement_block(ctx, 0, 2));
            if (VERBOSE)
                printf("\nBuilding index for c(%s)\n", aroot);
            GPU(gd_sort_kmers(ctx, 2));
            report_index(ctx, 2, &A, KMER_LEN, MAX_REPS, MEM_LIMIT, MEM_PHYSICAL, VERBOSE);
            r0 = num_overlaps(ctx);
            GPU(gd_match_filter(ctx, 2, 1, 1));
            if (VERBOSE)
                report_match(ctx, aroot, aroot, 1, 0, 2, r0, &A, &A, KMER_LEN, MEM_LIMIT);
            GPU(gd_write_overlap_buffer(ctx, RUN_ID, aroot, aroot, A.ufirst + A.nreads - 1));
        }
        GPU(gd_reset_overlap_buffer(ctx));
    }
    dz_free(&A);
    gd_destroy(ctx);
    free(MASK);
    exit(0);
}
