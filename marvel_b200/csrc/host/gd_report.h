/* gd_report.h -- daligner's -v report lines and its index-size warning, shared by the
 * command line (daligner_main.c) and the reference-named entry points (compat.c).  Built
 * into libgpudalign.so; not part of include/gpudalign.h. */
#ifndef GD_REPORT_H
#define GD_REPORT_H
#include <stdint.h>

#include "gpudalign.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Print_Number (db/DB.c:193-240): digits grouped by commas, right-aligned in width. */
void gd_report_number(int64_t num, int width);

/* Sort_Kmers' report under -v and its memory warning (dalign/filter.c:754-759, 865-892):
 * slots = the block's k-mer positions (boff[nreads] - k * nreads); the index size comes
 * from the context's statistics of that slot. */
void gd_report_index(gd_context* ctx, int slot, int64_t slots, int suppress, int64_t mem_limit, int mem_physical,
                     int verbose);

/* Match_Filter's report under -v (dalign/filter.c:2058-2063, 2105-2106, 2158-2162,
 * 2180-2189, 2388-2405): the pair cap, the hits, the Local_Alignment calls (seed hits) and
 * the overlaps they added (confirmed hits).  same_index: A's index also served as B's;
 * recs_before: the overlap count before the call; atot/btot: the blocks' base counts. */
void gd_report_match(gd_context* ctx, const char* aname, const char* bname, int comp, int same_index, int bslot,
                     int64_t recs_before, double atot, double btot, int kmer, int64_t mem_limit);

#ifdef __cplusplus
}
#endif
#endif
