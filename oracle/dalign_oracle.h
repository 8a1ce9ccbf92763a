/* dalign_oracle.h -- TEST INFRASTRUCTURE ONLY.
 *
 * A single-threaded CPU restatement of MARVEL daligner's overlap path (dalign/filter.c,
 * dalign/align.c), written as a parity checker for the sm_100a implementation.  It is
 * never linked into the product library and is only loaded by tests/, by the smoke check
 * and by bench.py's CPU-baseline leg.
 *
 * Parity of this restatement is pinned against the reference binary built from source
 * (oracle/Makefile -> oracle/_ref/daligner) on seeded synthetic DBs, and against the
 * committed golden .las fixtures in tests/golden/.
 */
#ifndef DALIGN_ORACLE_H
#define DALIGN_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* A loaded DB block, laid out like Read_All_Sequences (db/DB.c:1349-1410):
 * bases[-1] == 4, read i occupies bases[boff[i] .. boff[i]+rlen[i]) and bases[boff[i]+rlen[i]] == 4. */
typedef struct
{
    const uint8_t* bases;
    const int64_t* boff;    /* [nreads+1] */
    const int32_t* rlen;    /* [nreads]   */
    int32_t nreads;
    int32_t maxlen;
    int64_t totlen;
    int32_t ufirst;
    const int64_t* mask_anno; /* [nreads+1] int index into mask_data, or NULL */
    const int32_t* mask_data; /* (beg,end) pairs of masked intervals */
} or_block;

typedef struct
{
    int32_t kmer, binshift, suppress, hitmin; /* -k -w -t -h */
    double ave_corr;                          /* -e */
    int32_t tspace;                           /* -s */
    int32_t minover;                          /* 2 * -l (dalign/daligner.c:836) */
    int32_t symmetric, identity, only_identity, no_trace;
    uint64_t mem_limit;                       /* bytes (-M << 30), 0 = no cap */
    float freq[4];                            /* A-block base frequencies */
    int32_t hgap;                             /* daligner2 -H (its HGAP_MIN is live) */
    int32_t variant;                          /* 1 = daligner, 2 = daligner2 (dalign2/) */
    int32_t biased;                           /* daligner -b: frequency-weighted tuples */
} or_params;

typedef struct
{
    int32_t tlen, diffs, abpos, bbpos, aepos, bepos;
    uint32_t flags;
    int32_t aread, bread;
    int64_t toff; /* offset of this record's trace bytes in or_result.trace */
} or_overlap;

typedef struct
{
    int64_t novl;
    or_overlap* ovl;
    uint8_t* trace;   /* tbytes per trace value */
    int64_t tbytes_total;
    int32_t tbytes;
    /* statistics */
    int64_t kmers_a, kmers_b, hits_n, hits_c, seeds_n, seeds_c, cells, snake_steps;
    /* 0, or daligner2 only: 2 = a trace value above 255 met the 8-bit compression check
     * (Compress_TraceTo8) */
    int32_t status;
} or_result;

/* Sorted k-mer index of a block (Sort_Kmers, dalign/filter.c:698-903).
 * Fills code/read/rpos (capacity >= totlen) and returns the number of entries. */
int64_t or_sort_kmers(const or_block* b, const or_params* p, uint64_t* code, int32_t* read, int32_t* rpos);

/* Hits of one orientation after the hit sort (Match_Filter up to dalign/filter.c:2267).
 * self != 0 for a block against itself.  Returns the number of hits; *out points at
 * malloc'ed int32[4*n] rows (diag, apos, aread, bread); free with or_free. */
int64_t or_match_hits(const or_block* a, const or_block* b, const or_params* p, int self, int32_t** out,
                      int32_t* limit_out);

/* One Local_Alignment call from (diag, anti) (dalign/align.c:1922-2060).
 * out8 = {abpos, bbpos, aepos, bepos, diffs, tlen} of the A-path then of the B-path;
 * atrace/btrace receive the uint16 trace values (capacity >= 4*(maxlen/tspace+2)). */
int or_local_alignment(const uint8_t* aseq, const uint8_t* bseq, int alen, int blen, int comp, int diag,
                       int anti, const or_params* p, int32_t* out12, uint16_t* atrace, uint16_t* btrace,
                       int64_t* cells);

/* The whole overlap path for block A against block B (both orientations), like
 * daligner's main loop body (dalign/daligner.c:957-1014): returns every overlap record
 * sorted as Write_Overlap_Buffer sorts them (dalign/align.c:5786-5853). */
int or_daligner(const or_block* a, const or_block* b, const or_block* bc, const or_params* p, int self,
                or_result* res);

/* daligner2's overlap path for block A against block B (dalign2/daligner.c:654-790): the
 * modimizer index of both blocks, one join giving both orientations, the seed scan and
 * alignment per orientation (bc = the complemented B block), records sorted as
 * Write_Overlap_Buffer sorts them (dalign2/ovlbuffer.c:160-312).  p->variant must be 2. */
int or_daligner2(const or_block* a, const or_block* b, const or_block* bc, const or_params* p, int self,
                 or_result* res);

/* daligner2's Handle_Redundancies (fusion, bridging, compaction; dalign2/filter.c:1952-2272)
 * on one pair's paths: aseq/bseq with a 4 before and after, bseq complemented when comp;
 * hdr = 6 ints per path (abpos, bbpos, aepos, bepos, diffs, tlen) of the novls A-side paths
 * and, with hasB, the novls B-side paths; traces = their trace values back to back.
 * Returns the number of paths kept and writes them the same way (A side, then B side). */
int or_handle_redundancies_d2(const uint8_t* aseq, const uint8_t* bseq, int alen, int blen, int tspace, int comp,
                              int novls, int hasB, const int32_t* hdr, const uint16_t* traces, int32_t* out_hdr,
                              uint16_t* out_traces, int64_t tcap);

/* daligner2's sorted k-mer index (dalign2/filter.c:834-1106): read = (read << 1) | strand. */
int64_t or_sort_kmers2(const or_block* b, const or_params* p, uint64_t* code, int32_t* read, int32_t* rpos);

/* Exact diffs between trace points (Compute_Trace_PTS, dalign/align.c:5286-5397). */
int or_trace_pts_diffs(const uint8_t* aseq, const uint8_t* bseq, int alen, int blen, int abpos, int bbpos,
                       int aepos, int bepos, const uint8_t* trace8, const uint16_t* trace16, int tlen,
                       int tspace, int32_t* diffs_out);

void or_free(void* p);
void or_free_result(or_result* r);

#ifdef __cplusplus
}
#endif
#endif
