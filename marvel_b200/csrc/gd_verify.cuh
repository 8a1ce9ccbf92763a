// gd_verify.cuh -- Compute_Trace_PTS (exact diffs between trace points) on the device.
#pragma once
#include "gd_common.cuh"

namespace gd
{

// One trace-point interval of one .las record: A[ab..ae) against B[bb..be) (block-relative
// read indices; comp selects the complemented B block).
struct Segment
{
    int32_t aread, bread;
    int32_t ab, ae, bb, be;
    int32_t rec, comp;
};

// Per segment: threads need 3 * (2R + 1) ints of scratch each, R >= segment M + N + 4.
int launch_trace_pts(const DevBlock& A, const DevBlock& B, const DevBlock& C, const Segment* seg, int64_t nseg,
                     int* scratch, int R, int nthreads, int* diffs, DevStatus* st, cudaStream_t s);

}  // namespace gd
