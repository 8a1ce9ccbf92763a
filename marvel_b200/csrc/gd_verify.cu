// gd_verify.cu -- Compute_Trace_PTS on the device: exact differences of .las records.
//
// Restates dalign/align.c Compute_Trace_PTS (:5286-5397) with the distance part of iter_np
// (:4556-4917): each record is cut at its trace points (one segment per trace-spacing
// interval of the A read), every segment is aligned exactly with the O(np) waves, and the
// segment distances add up to the record's diffs.  GPU mapping: one thread per segment
// (segments are independent, ~100 bases each), three rolling wave vectors per thread in
// L1-resident scratch, distances summed per record with atomics.  This is the check
// LAcheck -a runs (utils/LAcheck.c:236-252), for a whole overlap buffer at once.
#include "gd_verify.cuh"

namespace gd
{

constexpr int VT = 128;

__device__ int iter_np_dist(const uint8_t* A, int M, const uint8_t* B, int N, int* b0, int* b1, int* b2)
{
    int del = M - N, low, hgh, D, k, j, i, am, ac, ap;
    int *F0, *F1, *F2, *nf;
    if (del >= 0)
    {
        low = 0;
        hgh = del;
    }
    else
    {
        low = del;
        hgh = 0;
    }
    F1 = b1;
    F0 = b2;
    nf = b0;
    for (k = low - 1; k <= hgh + 1; k++)
        F1[k] = F0[k] = -2;
    F0[0] = -1;
    low += 1;
    hgh -= 1;
    for (D = 0; D <= M + N + 2; D++)
    {
        int* t = nf;
        F2 = F1;
        F1 = F0;
        F0 = t;
        nf = F2;
        if ((D & 1) == 0)
        {
            low -= 1;
            hgh += 1;
        }
        F0[hgh + 1] = F0[low - 1] = -2;
        // one furthest-reaching step (FS_MOVE, align.c:4640-4672): the best of the two
        // waves back, the previous wave plus a substitution, and the neighbour on this wave
#define GD_FS(AP, AM)                                       \
    ap = (AP);                                              \
    am = (AM);                                              \
    ac = F1[k] + 1;                                         \
    if (ac < am)                                            \
        j = (ap < am) ? am : ap;                            \
    else if (ap < ac)                                       \
        j = ac;                                             \
    else                                                    \
        j = ap;                                             \
    i = M - k;                                              \
    {                                                       \
        int lim = (N < i) ? N : i;                          \
        while (j < lim && __ldg(B + j) == __ldg(A + j + k)) \
            j += 1;                                         \
    }                                                       \
    F0[k] = j;
        j = -2;
        for (k = hgh; k > del; k--)
        {
            GD_FS(j + 1, F2[k - 1])
        }
        j = -2;
        for (k = low; k < del; k++)
        {
            GD_FS(F2[k + 1] + 1, j)
        }
        k = del;
        GD_FS(F0[del + 1] + 1, j)
#undef GD_FS
        if (F0[del] >= N)
            return D + abs(del);
    }
    return -1;
}

__global__ void __launch_bounds__(VT) k_trace_pts(DevBlock A, DevBlock B, DevBlock C, const Segment* __restrict__ seg,
                                                 int64_t nseg, int* scratch, int R, int* diffs, DevStatus* st)
{
    const int64_t nthreads = (int64_t)gridDim.x * VT;
    const int64_t tid = (int64_t)blockIdx.x * VT + threadIdx.x;
    int* mem = scratch + tid * 3 * (2 * R + 1);
    int* b0 = mem + R;
    int* b1 = mem + (2 * R + 1) + R;
    int* b2 = mem + 2 * (2 * R + 1) + R;
    for (int64_t s = tid; s < nseg; s += nthreads)
    {
        Segment g = seg[s];
        if ((g.ae - g.ab) + (g.be - g.bb) + 4 > R || g.ae < g.ab || g.be < g.bb)
        {
            gd_fail(st, GD_ERR_TRACE, (int)g.rec, R);
            continue;
        }
        const DevBlock& bb = g.comp ? C : B;
        const uint8_t* a = A.bases + A.boff[g.aread] + g.ab;
        const uint8_t* b = bb.bases + bb.boff[g.bread] + g.bb;
        int d = iter_np_dist(a, g.ae - g.ab, b, g.be - g.bb, b0, b1, b2);
        if (d < 0)
        {
            gd_fail(st, GD_ERR_TRACE, (int)g.rec, -1);
            continue;
        }
        atomicAdd(diffs + g.rec, d);
    }
}

int launch_trace_pts(const DevBlock& A, const DevBlock& B, const DevBlock& C, const Segment* seg, int64_t nseg,
                     int* scratch, int R, int nthreads, int* diffs, DevStatus* st, cudaStream_t s)
{
    if (nseg <= 0)
        return 0;
    k_trace_pts<<<nthreads / VT, VT, 0, s>>>(A, B, C, seg, nseg, scratch, R, diffs, st);
    GD_LAUNCHED(1);
    GD_CUDA(cudaGetLastError());
    return 0;
}

}  // namespace gd
