/* gpudalign.h -- C ABI of the sm_100a daligner overlap path (libgpudalign.so).
 *
 * The entry points mirror the reference's inner C interface of the path, so that the
 * reference driver (dalign/daligner.c main) or any FFI can call the GPU path in place of
 * dalign/filter.c + dalign/align.c.  All pointers are plain host pointers; no CUDA or
 * torch types cross this boundary.  Every function returns 0 (or a count >= 0) on
 * success and -1 on failure, with the message in gd_last_error(); nothing exits the
 * process (the reference calls exit(1) instead, dalign/filter.c:2135-2145).
 *
 * One context = one GPU (the device current at gd_create) and one host thread.
 */
#ifndef GPUDALIGN_H
#define GPUDALIGN_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct gd_context gd_context;

/* A DB block in host memory, laid out like the reference's Read_All_Sequences result
 * (db/DB.c:1349-1410): bases[-1] == 4, read i at bases[boff[i]] .. bases[boff[i]+rlen[i]-1],
 * bases[boff[i]+rlen[i]] == 4.  mask_anno/mask_data (optional) give per read the masked
 * (begin,end) intervals of the -m tracks: read i's pairs are mask_data[mask_anno[i] ..
 * mask_anno[i+1]) (the converted track layout of dalign/daligner.c:425-428). */
typedef struct
{
    const uint8_t* bases;
    const int64_t* boff; /* [nreads+1] */
    const int32_t* rlen; /* [nreads]   */
    int32_t nreads;
    int32_t maxlen;
    int64_t totlen;
    int32_t ufirst;
    const int64_t* mask_anno;
    const int32_t* mask_data;
} gd_block;

/* One overlap as the .las file stores it (Overlap minus its trace pointer,
 * dalign/align.h:307-312, written by Write_Overlap dalign/align.c:3345-3350). */
typedef struct
{
    int32_t tlen, diffs, abpos, bbpos, aepos, bepos;
    uint32_t flags;
    int32_t aread, bread, pad;
    uint64_t toff; /* offset of this record's trace bytes in the trace array */
} gd_overlap;

typedef struct
{
    int64_t kmers[3];     /* index sizes of slots A, B, complement-B */
    int64_t hits[2];      /* hits of the last N and C Match_Filter calls */
    int64_t groups[2];    /* pair groups with >= ceil(h/k) hits */
    int64_t seeds[2];     /* Local_Alignment calls */
    int64_t cells[2];     /* wave cells (sum of wave widths, dalign/align.c:957-963) */
    int64_t records;      /* overlaps in the buffer */
    int32_t limit[2];     /* k-mer pair cap used (dalign/filter.c:2107-2174) */
    double ms_index[3];   /* device time of Sort_Kmers per slot */
    double ms_merge[2];   /* device time of merge + hit sort */
    double ms_align[2];   /* device time of seed scan + alignment */
    int64_t skipped[2];   /* pair groups the learned triage skipped (0 with no model set) */
    int64_t wide[2];      /* pair groups whose band outgrew 128 diagonals (aligned by the wide kernel) */
    int64_t reruns[2];    /* aligner re-runs after a scratch or output buffer was grown */
} gd_stats;

/* Context on the current CUDA device. */
gd_context* gd_create(void);
void gd_destroy(gd_context* ctx);
const char* gd_last_error(void);

/* Set_Filter_Params (dalign/filter.c:119-139). */
int gd_set_filter_params(gd_context* ctx, int kmer, int binshift, int suppress, int hitmin);

/* New_Align_Spec (dalign/align.c:214-279) with the HEIDELBERG flags it takes. */
int gd_new_align_spec(gd_context* ctx, double ave_corr, int trace_space, const float freq[4], int symmetric,
                      int only_identity, int no_trace_points);

/* The globals daligner's main shares with filter.c (dalign/daligner.c:60-71):
 * MINOVER (already doubled, :836), IDENTITY, MEM_LIMIT in bytes (0 = uncapped). */
int gd_set_globals(gd_context* ctx, int minover, int identity, uint64_t mem_limit);

/* Copy a block to the device into slot 0 (A), 1 (B) or 2 (complemented B). */
int gd_load_block(gd_context* ctx, int slot, const gd_block* block);

/* complement_DB (dalign/daligner.c:474-573) on the device: slot dst becomes the
 * reverse complement of slot src (reads, and mask intervals mirrored). */
int gd_complement_block(gd_context* ctx, int src, int dst);

/* Sort_Kmers (dalign/filter.c:698-903): builds the sorted k-mer index of a loaded slot on
 * the device; returns its length. */
int64_t gd_sort_kmers(gd_context* ctx, int slot);

/* Copies the sorted index of a slot to the host (code, read, rpos); returns its length. */
int64_t gd_get_kmers(gd_context* ctx, int slot, uint64_t* code, int32_t* read, int32_t* rpos, int64_t cap);

/* Match_Filter (dalign/filter.c:1997-2407): A (slot 0) against bslot in orientation comp;
 * self != 0 when A and B are the same block (aname == bname in the reference).
 * Appends the overlaps it finds to the context's overlap buffer. */
int gd_match_filter(gd_context* ctx, int bslot, int comp, int self);

/* daligner's -b (BIASED, dalign/daligner.c:61,681-683): gd_sort_kmers then builds the
 * frequency-weighted index of biased_tuple_thread (dalign/filter.c:492-633): per read a window
 * of at most k bases, grown until its information (sum of ceil(-10000 log4 freq[base]))
 * reaches 10000 k, kept when above 10000 (k - 2), coded with its bases at the top of the k-mer
 * code.  The weights come from the frequencies of gd_new_align_spec (daligner gives the A
 * block's, which is also the first block it indexes); they must lie in (0, 1].  Not
 * available with variant 2.  Changing the flag drops the slots' indices. */
int gd_set_biased(gd_context* ctx, int biased);

/* daligner2 mode (the reference's dalign2/, modimizer seeds).  variant 1 = daligner (the
 * default), 2 = daligner2; hgap = daligner2's -H (HGAP_MIN, dalign2/daligner.c:29,570: pairs
 * whose reads are both shorter are skipped, shorter reads get no record of their own).
 * In mode 2, gd_sort_kmers builds daligner2's index (Sort_Kmers, dalign2/filter.c:834-1106:
 * canonical and half-shifted codes with code % 101 < 28; read = (read << 1) | strand) and
 * Match_Filter is gd_match_filter2.  Changing the mode drops the slots' indices. */
int gd_set_variant(gd_context* ctx, int variant, int hgap);

/* daligner2's Match_Filter (dalign2/filter.c:2344-2700 with report_thread,
 * dalign2/filter_reporter_cpu.c:16-411): A (slot 0) against bslot in both orientations from
 * one join; cslot holds the complemented B block (gd_complement_block) the complement pairs
 * are aligned against.  Two paths of a pair with a narrow parallel overlap are bridged as
 * daligner2 bridges them (Compute_Bridge_Path, dalign2/filter.c:1579-1705); the call fails
 * where a trace value above 255 meets the 8-bit compression check (Compress_TraceTo8). */
int gd_match_filter2(gd_context* ctx, int bslot, int cslot, int self);

/* Test hook, no counterpart in the reference: daligner2's Handle_Redundancies (fusion, bridging,
 * compaction; dalign2/filter.c:1952-2272) of one pair on the device, with the calling
 * convention of the oracle's or_handle_redundancies_d2: aseq/bseq point at the first base
 * with a 4 before and after (bseq complemented when comp); hdr = 6 ints per path (abpos,
 * bbpos, aepos, bepos, diffs, tlen) of the novls A-side paths and, with hasB, the B-side
 * paths; traces back to back.  Returns the number of paths kept (written the same way). */
int gd_test_handle_redundancies_d2(gd_context* ctx, const uint8_t* aseq, const uint8_t* bseq, int alen, int blen,
                                   int tspace, int comp, int novls, int hasB, const int32_t* hdr,
                                   const uint16_t* traces, int32_t* out_hdr, uint16_t* out_traces, int64_t tcap);

/* The sorted hits of the last gd_match_filter (rows diag, apos, aread, bread), for tests. */
int64_t gd_get_hits(gd_context* ctx, int32_t* rows4, int64_t cap);

/* Overlap buffer (kept in device memory): count, sort, copy out, write .las files as
 * Write_Overlap_Buffer does (dalign/align.c:5815-6043), reset.
 * gd_num_overlaps: records and trace bytes in the buffer (before the -I identity filter).
 * gd_sort_overlaps: sorts the buffer on the device in SORT_OVL order (aread, bread,
 * orientation, abpos; dalign/align.c:5786-5813; ties by aepos, bbpos) with the identity
 * filter applied; returns the records kept and their trace bytes.  Later reads reuse it.
 * gd_get_overlaps: copies up to rcap sorted records and their traces (at most tcap bytes;
 * toff = offset in trace) to host memory; returns the number of records copied. */
int64_t gd_num_overlaps(gd_context* ctx, int64_t* trace_bytes);
int64_t gd_sort_overlaps(gd_context* ctx, int64_t* trace_bytes);
int64_t gd_get_overlaps(gd_context* ctx, gd_overlap* recs, uint8_t* trace, int64_t rcap, int64_t tcap);

/* DBdust (db/DBdust.c:92-530) on the device for the block in slot: low-complexity
 * intervals of every read with scan window `window` (-w, 3..128), threshold `thresh` (-t),
 * intervals of at least `mflag` bases (-m), `biased` (-b, weights from freq, the DB's base
 * frequencies).  Returns the number of ints of interval data (pairs begin, end); when
 * anno (nreads + 1 int64) and data (cap int32) are given and cap suffices, fills them in
 * the .dust.anno / .dust.data layout: anno[r] = byte offset of read r's pairs in data. */
int64_t gd_dust(gd_context* ctx, int slot, int window, double thresh, int mflag, int biased, const float freq[4],
                int64_t* anno, int32_t* data, int64_t cap);

/* Test hook, no counterpart in the reference: the widest band (in diagonals) the main
 * aligner kernel takes before it hands a pair group to the wide kernel: 128 (default) or
 * 32 (a narrow kernel instance that routes most groups through the wide kernel; the
 * output must not change). */
int gd_set_wave_limit(gd_context* ctx, int limit);

/* The aligner's schedule, no counterpart in the reference (its threads split the hits by
 * b-read, dalign/filter.c:2282-2294).  nedges = 0 (the default): every pair group of a
 * Match_Filter in one persistent launch, taken longest first from a device queue.  Else one
 * launch per length class, the classes split at the given alen + blen edges (bp), longest
 * class first.  kind (nedges + 1 entries, longest class first, or NULL for all 0) picks each
 * class's kernel instance: 0 = a warp per alignment with 128-diagonal wave rings, 4 warps
 * per CTA (a group whose band outgrows 128 is redone by the wide instance), 1 = the wide
 * instance, 512-diagonal rings, one warp per CTA, 2 = the duo instance, two 16-lane teams
 * per warp, each aligning its own pair group with 128-diagonal rings (wider bands are redone
 * by the wide instance; daligner2's report runs instance 0 in its place).  The autotuner
 * (marvel_b200/autotune.py) sets it; the output is the same for every schedule. */
int gd_set_align_schedule(gd_context* ctx, int nedges, const int32_t* edges, const int32_t* kind);

/* Test hook, no counterpart in the reference: the aligner's starting capacities -- pebbles
 * and pair-trace values per warp, paths per pair, overlap records and trace bytes per
 * Match_Filter.  Each one the aligner outgrows is reported by the device, grown on the host
 * and the alignment stage re-run (gd_stats.reruns); small values force that path, and the
 * output must not change.  Values <= 0 keep the current capacity. */
int gd_set_capacities(gd_context* ctx, int pebbles, int traces, int paths, int64_t records, int64_t trace_bytes);

/* Test hook, no counterpart in the reference: one block of the radix sort's bounded wait on
 * an mbarrier armed for a copy that is never issued (nothing is in flight), with polls
 * tries; the wait must give up, raise the sort's wait flag and return, and the check every
 * sort makes afterwards must report it (-1, gd_last_error set) and clear it. */
int gd_test_wait_expiry(gd_context* ctx, int polls);

/* LAsort (dalign/LAsort.c:65-90, 139-256) of one .las file on the device: writes out_path
 * with the records of in_path ordered by (aread, bread, abpos) -- ties, which the
 * reference's qsort leaves unordered, by (aepos, bbpos) and then file order -- each record's
 * bytes (trace and pad word included) unchanged.  Returns the number of records. */
int64_t gd_las_sort(gd_context* ctx, const char* in_path, const char* out_path);

/* LAmerge's result (utils/LAmerge.c, heap merge ordered by SORT_OVL of
 * utils/LAmergeUtils.c:50-79: aread, bread, orientation, abpos) for nin .las files of one
 * trace spacing, in one device sort of all their records; ties by (aepos, bbpos), then
 * input order.  Record bytes are kept.  Returns the number of records. */
int64_t gd_las_merge(gd_context* ctx, const char* const* in_paths, int nin, const char* out_path);
int gd_write_overlap_buffer(gd_context* ctx, int run_id, const char* ablock, const char* bblock, int last_read);
int gd_reset_overlap_buffer(gd_context* ctx);

int gd_get_stats(gd_context* ctx, gd_stats* st);

/* Compute_Trace_PTS (dalign/align.c:5286-5397) over n .las records: the exact number of
 * differences of each record, aligning every trace-point interval with iter_np's O(np)
 * waves (dalign/align.c:4556-4917) -- the check LAcheck -a makes (utils/LAcheck.c:236-252).
 * Records and trace bytes as gd_get_overlaps returns them; A reads come from aslot, B reads
 * from bslot, or from cslot (the complemented B block) for records with the COMP flag.
 * diffs_out[i] receives record i's exact diffs. */
int gd_compute_trace_pts(gd_context* ctx, int aslot, int bslot, int cslot, const gd_overlap* recs,
                         const uint8_t* trace, int64_t n, int32_t* diffs_out);

/* Device timer on the context's stream: mark 0 = start, mark 1 = stop; elapsed in ms. */
int gd_timer_mark(gd_context* ctx, int which);
double gd_timer_elapsed_ms(gd_context* ctx);

/* Kernels this library has launched since it was loaded (launch accounting). */
unsigned long long gd_kernel_launches(void);

/* Local_Alignment (dalign/align.c:1922-2060) for a batch of seeds on the device.
 * Sequences are host buffers in gd_block layout; per seed: read offsets into abases /
 * bbases, lengths, diagonal and anti-diagonal.  out12 receives per seed the A-path
 * {abpos,bbpos,aepos,bepos,diffs,tlen} then the B-path; traces land at
 * trace + seed*trstride (A) and + trstride/2 (B); cells per seed in cells. */
int gd_local_alignment_batch(gd_context* ctx, const uint8_t* abases, int64_t alen_total, const uint8_t* bbases,
                             int64_t blen_total, const int64_t* aoff, const int32_t* alen, const int64_t* boff,
                             const int32_t* blen, const int32_t* diag, const int32_t* anti, int nseeds, int comp,
                             int32_t* out12, uint16_t* trace, int trstride, int64_t* cells);

/* Local_Alignment batch that allocates nothing, for callers that may not call cudaMalloc
 * once they run (an application that gives all HBM to its own pool, or a latency-critical
 * loop where an allocation's implicit device synchronization is not allowed).  It has no
 * counterpart in the reference.  All array arguments are DEVICE pointers owned by the
 * caller, in the layout of gd_local_alignment_batch (sequence buffers need 16 readable
 * bytes before the first base and after the last 4); maxlen is the longest read among the
 * seeds; stream is a cudaStream_t (NULL = legacy default stream).  ctx must have had
 * gd_new_align_spec called (that call may allocate; do it during set-up).
 * Working memory is one file-scope device array of 17,301,760 bytes (16 warps, 65,536
 * pebbles and 16,384 trace-point slots per warp) that every GPU loading the library keeps
 * until exit; maxlen / tspace may be at most 2044 (reads up to 204,499 bp at trace
 * spacing 100), larger batches are rejected up front with an error.  The pebbles bound the
 * band: a wave over L bases of A whose band averages W diagonals needs up to about
 * 2 * W * L / tspace of them (65,536 hold 150 kbp at W = 21, spacing 100); a seed that
 * needs more fails the call with an error naming it, as does a seed whose trace is longer
 * than trstride / 2.  The first call on a device looks up that array's device address
 * (cudaGetSymbolAddress) with the device current, so make the first call before any
 * stream capture.  Calls share the array: two calls that overlap on the GPU (different
 * streams or threads) race and must be serialised by the caller.  The call synchronizes
 * its stream to read the status word. */
int gd_local_alignment_batch_noalloc(gd_context* ctx, const uint8_t* d_abases, const uint8_t* d_bbases,
                                     const int64_t* d_aoff, const int32_t* d_alen, const int64_t* d_boff,
                                     const int32_t* d_blen, const int32_t* d_diag, const int32_t* d_anti, int nseeds,
                                     int maxlen, int comp, int32_t* d_out12, uint16_t* d_trace, int trstride,
                                     int64_t* d_cells, void* stream);

/* ------------------------------------------------------------------------------------
 * Learned triage of pair groups.  No counterpart in the reference: an addition in front of
 * the aligner (report_thread, dalign/filter.c:1656-1995, aligns every pair group that has
 * >= ceil(h/k) hits).  Each pair group is described by 12 features of its hits (TRI_NF);
 * a 12-64-64-1 MLP (BF16 tensor-core kernels, FP32 accumulate, FP32 Adam state) predicts
 * whether the group yields an overlap.  A group is skipped or aligned as a whole, so every
 * record of the triaged path is a record of the plain path.
 * Parameter vector (GD_TRI_NPARAM floats): mean[12], scale[12] (features are standardised
 * as (f - mean) / scale), W1[64][12], b1[64], W2[64][64], b2[64], W3[64], b3.
 * ------------------------------------------------------------------------------------ */
#define GD_TRI_NF 12
#define GD_TRI_NPARAM 5081

/* Collect, per pair group of every following gd_match_filter, its features and the plain
 * path's outcome (records emitted, wave cells); on != 0 turns collection on. */
int gd_triage_collect(gd_context* ctx, int on);

/* Copies up to cap collected rows (feat: cap x 12 floats, records, cells; any may be NULL);
 * returns the number of rows collected. */
int64_t gd_triage_get_groups(gd_context* ctx, float* feat, uint32_t* records, uint32_t* cells, int64_t cap);

int gd_triage_reset(gd_context* ctx);

/* Sets the model used inside gd_match_filter: groups whose predicted probability is below
 * threshold are not aligned.  params == NULL turns the triage off. */
int gd_triage_set_model(gd_context* ctx, const float* params, float threshold);

/* Feature scales (mean / standard deviation over feat's n rows) and seeded He-uniform
 * initial weights, zero biases.  Host only. */
int gd_mlp_init(const float* feat, int64_t n, uint64_t seed, float* params);

/* prob[i] = sigmoid(MLP(feat[i])) on the device, host buffers in and out. */
int gd_mlp_forward(gd_context* ctx, const float* params, const float* feat, int64_t n, float* prob);

/* Gradient (GD_TRI_NPARAM floats; mean and scale entries 0) and value of the batch-mean
 * binary cross-entropy with positives weighted pos_weight, over n rows, on the device. */
int gd_mlp_grad(gd_context* ctx, const float* params, const float* feat, const float* label, int n, float pos_weight,
                float* grad, float* loss);

/* Mini-batch Adam (beta 0.9 / 0.999, eps 1e-8) on the device for epochs passes over the n
 * rows in a seeded shuffled order; params holds the initial model on entry and the trained
 * one on return; epoch_loss (optional, epochs floats) receives each pass's mean loss. */
int gd_mlp_train(gd_context* ctx, const float* feat, const float* label, int64_t n, int epochs, int batch, float lr,
                 float pos_weight, uint64_t seed, float* params, float* epoch_loss);

#ifdef __cplusplus
}
#endif
#endif
