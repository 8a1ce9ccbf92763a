/* gpudalign_compat.h -- MARVEL's daligner library interface, by its own names, served by
 * libgpudalign.so (marvel_b200/csrc/host/compat.c).
 *
 * A program written against the reference's dalign/filter.h and dalign/align.h -- the
 * reference's own driver dalign/daligner.c included -- links against libgpudalign.so in
 * place of the reference's filter.c and align.c, unchanged: C links by name, and the
 * records passed by pointer below have the reference's layouts (x86-64).  Such a program
 * keeps including the reference's headers; this header states the same interface for
 * programs that do not have them, with the records under gdc_ names.
 *
 * The reference's driver globals VERBOSE, BIASED, MINOVER, IDENTITY, MEM_LIMIT and
 * MEM_PHYSICAL (dalign/daligner.c:60-71, read by dalign/filter.c) are read from the program
 * when it defines them (weak references), else taken as 0.
 *
 * Differences of contract: Sort_Kmers returns a handle to an index built in device memory
 * (not a host KmerPos array); only Match_Filter may be given it.  Local_Alignment takes the
 * seeds daligner's filter gives it (low == hgh, lbord = hbord = -1).  Compute_Trace_PTS sets
 * path->diffs, the exact difference count through the trace points, and leaves path->trace
 * as given.  Errors print a message and exit with status 1, like the reference's EXIT
 * (db/DB.h:36); Local_Alignment returns NULL instead.
 */
#ifndef GPUDALIGN_COMPAT_H
#define GPUDALIGN_COMPAT_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* HITS_READ, HITS_TRACK, HITS_DB (db/DB.h:163-236): a block as Read_All_Sequences leaves it */
typedef struct
{
    int rlen;
    int64_t boff;
    int64_t coff;
    int flags;
} gdc_HITS_READ;

typedef struct gdc_HITS_TRACK_s
{
    struct gdc_HITS_TRACK_s* next;
    char* name;
    int size;
    void* anno;
    void* data;
} gdc_HITS_TRACK;

typedef struct
{
    int ureads;
    float freq[4];
    int maxlen;
    int64_t totlen;
    int nreads;
    int part;
    int ufirst;
    char* path;
    int loaded;
    void* bases;
    gdc_HITS_READ* reads;
    gdc_HITS_TRACK* tracks;
} gdc_HITS_DB;

/* Path and Alignment (dalign/align.h:76-117) */
typedef struct
{
    void* trace;
    int tlen;
    int diffs;
    int abpos, bbpos;
    int aepos, bepos;
} gdc_Path;

typedef struct
{
    gdc_Path* path;
    uint32_t flags;
    char* aseq;
    char* bseq;
    int alen;
    int blen;
} gdc_Alignment;

/* Set_Filter_Params (dalign/filter.h:67, dalign/filter.c:119-139): 1 for an illegal k. */
int Set_Filter_Params(int kmer, int binshift, int suppress, int hitmin);

/* Sort_Kmers (dalign/filter.h:69, dalign/filter.c:698-903): builds the block's k-mer index
 * on the device; *len = its size; NULL for an empty index. */
void* Sort_Kmers(gdc_HITS_DB* block, int* len);

/* Match_Filter (dalign/filter.h:71-73, dalign/filter.c:1997-2407): A's index against B's,
 * aligning every pair group into the overlap buffer of asettings; comp: B is complemented;
 * aname == bname (the same pointer) marks a block against itself; frees btable when it is
 * not atable. */
void Match_Filter(char* aname, gdc_HITS_DB* ablock, char* bname, gdc_HITS_DB* bblock, void* atable, int alen,
                  void* btable, int blen, int comp, void* asettings);

/* New_Align_Spec / Free_Align_Spec (dalign/align.h:160-162, dalign/align.c:214-279). */
void* New_Align_Spec(double ave_corr, int trace_space, float* freq, int nthreads, int symmetric, int only_identity,
                     int no_trace_points);
void Free_Align_Spec(void* spec);

/* New_Work_Data / Free_Work_Data (dalign/align.h:131-133). */
void* New_Work_Data(void);
void Free_Work_Data(void* work);

/* Local_Alignment (dalign/align.h:195, dalign/align.c:1922-2060): fills align->path (trace
 * points in work storage) and returns the B-path, valid until the next call on work. */
gdc_Path* Local_Alignment(gdc_Alignment* align, void* work, void* spec, int low, int hgh, int anti, int lbord,
                          int hbord);

/* Compute_Trace_PTS (dalign/align.h:224, dalign/align.c:5286-5397): path->diffs. */
int Compute_Trace_PTS(gdc_Alignment* align, void* work, int trace_spacing, int mode, int debug);

/* Write_Overlap_Buffer / Reset_Overlap_Buffer (dalign/align.h:336-344,
 * dalign/align.c:5815-6056). */
void Write_Overlap_Buffer(void* spec, int RUN_ID, char* ablock, char* bblock, int lastRead);
void Reset_Overlap_Buffer(void* spec);

#ifdef __cplusplus
}
#endif
#endif
