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
#include "gd_report.h"
#include "gpudalign.h"

static void usage(void)
{
    fprintf(stderr, "usage:  \n");
    fprintf(stderr, "daligner [-vbAIOT] [-k<int(14)>] [-w<int(6)>] [-h<int(35)>] [-t<int>] [-M<int>]\n");
    fprintf(stderr, "         [-e<double(.70)] [-l<int(1000)>] [-s<int(100)>] [-H<int>] [-j<int>]\n");
    fprintf(stderr, "         [-m<track>]+ <subject:db|dam> <target:db|dam> ...\n");
    fprintf(stderr, "         [-r<int()1>]\n");
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
            fprintf(stderr, "daligner: %s\n", err);
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
    /* the subject block is read before the device is touched: a malformed DB or track is
       reported (exit 1) on any machine */
    const char* afile = argv[optind];
    dz_block A, B;
    load(&A, afile, MASK, MTOP, KMER_LEN);
    gd_context* ctx = gd_create();
    if (!ctx)
    {
        fprintf(stderr, "daligner: %s\n", gd_last_error());
        exit(1);
    }
    GPU(gd_set_filter_params(ctx, KMER_LEN, BIN_SHIFT, MAX_REPS, HIT_MIN));
    GPU(gd_set_globals(ctx, MINOVER, IDENTITY, (uint64_t)MEM_LIMIT));
    GPU(gd_set_biased(ctx, BIASED));

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
            gd_report_index(ctx, 0, A.boff[A.nreads] - (int64_t)KMER_LEN * A.nreads, MAX_REPS, MEM_LIMIT, MEM_PHYSICAL, VERBOSE);
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
            gd_report_index(ctx, 1, B.boff[B.nreads] - (int64_t)KMER_LEN * B.nreads, MAX_REPS, MEM_LIMIT, MEM_PHYSICAL, VERBOSE);
            int64_t r0 = num_overlaps(ctx);
            GPU(gd_match_filter(ctx, 1, 0, 0));
            if (VERBOSE)
                gd_report_match(ctx, aroot, broot, 0, 0, 1, r0, (double)A.totlen, (double)B.totlen, KMER_LEN, MEM_LIMIT);
            GPU(gd_complement_block(ctx, 1, 2));
            if (VERBOSE)
                printf("\nBuilding index for c(%s)\n", broot);
            GPU(gd_sort_kmers(ctx, 2));
            gd_report_index(ctx, 2, B.boff[B.nreads] - (int64_t)KMER_LEN * B.nreads, MAX_REPS, MEM_LIMIT, MEM_PHYSICAL, VERBOSE);
            r0 = num_overlaps(ctx);
            GPU(gd_match_filter(ctx, 2, 1, 0));
            if (VERBOSE)
                gd_report_match(ctx, aroot, broot, 1, 0, 2, r0, (double)A.totlen, (double)B.totlen, KMER_LEN, MEM_LIMIT);
            int lastRead = (B.part < A.part) ? B.ufirst + B.nreads - 1 : A.ufirst + A.nreads - 1;
            GPU(gd_write_overlap_buffer(ctx, RUN_ID, aroot, broot, lastRead));
            dz_free(&B);
        }
        else
        {
            int64_t r0 = num_overlaps(ctx);
            GPU(gd_match_filter(ctx, 0, 0, 1));
            if (VERBOSE)
                gd_report_match(ctx, aroot, aroot, 0, 1, 0, r0, (double)A.totlen, (double)A.totlen, KMER_LEN, MEM_LIMIT);
            GPU(gd_complement_block(ctx, 0, 2));
            if (VERBOSE)
                printf("\nBuilding index for c(%s)\n", aroot);
            GPU(gd_sort_kmers(ctx, 2));
            gd_report_index(ctx, 2, A.boff[A.nreads] - (int64_t)KMER_LEN * A.nreads, MAX_REPS, MEM_LIMIT, MEM_PHYSICAL, VERBOSE);
            r0 = num_overlaps(ctx);
            GPU(gd_match_filter(ctx, 2, 1, 1));
            if (VERBOSE)
                gd_report_match(ctx, aroot, aroot, 1, 0, 2, r0, (double)A.totlen, (double)A.totlen, KMER_LEN, MEM_LIMIT);
            GPU(gd_write_overlap_buffer(ctx, RUN_ID, aroot, aroot, A.ufirst + A.nreads - 1));
        }
        GPU(gd_reset_overlap_buffer(ctx));
    }
    dz_free(&A);
    gd_destroy(ctx);
    free(MASK);
    exit(0);
}
