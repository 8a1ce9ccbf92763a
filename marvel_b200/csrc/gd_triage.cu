// gd_triage.cu -- learned triage of pair groups on sm_100a.
//
// A pair group (the hits of one aread x bread x orientation that reach the aligner) is
// described by 12 features; a 12-64-64-1 MLP predicts whether the plain path will emit an
// overlap for it.  Training and inference run on hand-written BF16 tensor-core kernels
// (mma.sync m16n8k16, FP32 accumulate): forward layers 1-3; backward dW2, dH1 and dW1 as
// tensor-core GEMMs over the batch rows; bias / last-layer reductions in FP32; Adam in FP32.
// The decision is per group, so every record the triaged path emits is a record of the
// plain path (the group is aligned exactly as the plain path aligns it).
#include <algorithm>
#include <climits>
#include <cuda_bf16.h>

#include "gd_triage.cuh"

namespace gd
{

// ------------------------------------------------------------------------------------------
// features
// ------------------------------------------------------------------------------------------

// f0 log2 #hits            f1 log2 |A read|        f2 log2 |B read|
// f3 apos span / |A|       f4 log2(1+diag range)   f5 mean diagonal / |A|
// f6 log2(1+diag sd)       f7 overlap length on the mean diagonal / (2*minover)
// f8 hits per 64 bp of apos span                   f9 fraction of hits within one band of the mean diagonal
// f10 orientation (comp)   f11 masked fraction of the A read
// The twelve features from a group's sums: hits n, read lengths, a-position extent, the
// diagonals' mean, variance, range and the hits near the mean, the masked bases of the A read.
__device__ __forceinline__ void features_out(int n, float alen, float blen, int amin, int amax, double mean, double var,
                                             int dmin, int dmax, int near, long long masked_bases, bool has_mask,
                                             int comp, int minover, float f[TRI_NF])
{
    const double ovl = fmin((double)alen, (double)blen + mean) - fmax(0.0, mean);
    f[0] = log2f((float)n);
    f[1] = log2f(alen);
    f[2] = log2f(blen);
    f[3] = (float)(amax - amin) / alen;
    f[4] = log2f(1.f + (float)(dmax - dmin));
    f[5] = (float)(mean / alen);
    f[6] = log2f(1.f + (float)sqrt(var));
    f[7] = (float)(ovl / (2.0 * minover));
    f[8] = 64.f * n / (float)(amax - amin + 1);
    f[9] = (float)near / n;
    f[10] = (float)comp;
    f[11] = has_mask ? (float)masked_bases / alen : 0.f;
}

__device__ void group_features(const uint64_t* __restrict__ hkey, const uint32_t* __restrict__ hdiag, uint2 gr,
                               const HitBits& hb, const DevBlock& A, const DevBlock& B, int comp, int minover,
                               int binshift, const int64_t* __restrict__ anno, const int32_t* __restrict__ mdata,
                               float f[TRI_NF])
{
    int s = (int)gr.x, e = (int)gr.y, n = e - s;
    uint64_t k0 = hkey[s];
    int ar = (int)((k0 >> hb.pbits) & ((1ull << hb.abits) - 1));
    int br = (int)(k0 >> (hb.pbits + hb.abits));
    float alen = (float)A.rlen[ar], blen = (float)B.rlen[br];
    uint64_t pmask = (1ull << hb.pbits) - 1;
    int amin = (int)(k0 & pmask), amax = (int)(hkey[e - 1] & pmask);
    double sum = 0, sq = 0;
    int dmin = INT_MAX, dmax = INT_MIN;
    for (int i = s; i < e; i++)
    {
        int d = (int)hdiag[i];
        sum += d;
        sq += (double)d * d;
        dmin = min(dmin, d);
        dmax = max(dmax, d);
    }
    double mean = sum / n, var = fmax(sq / n - mean * mean, 0.0);
    int band = 1 << binshift, near = 0;
    for (int i = s; i < e; i++)
        near += fabs((double)(int)hdiag[i] - mean) <= band;
    long long mb = 0;
    if (anno)
        for (int64_t j = anno[ar]; j < anno[ar + 1]; j += 2)
            mb += mdata[j + 1] - mdata[j];
    features_out(n, alen, blen, amin, amax, mean, var, dmin, dmax, near, mb, anno != nullptr, comp, minover, f);
}

// group_features with a warp's lanes over the group's hits (every lane returns the features).
// The diagonal sums are integer sums, exact in any order, so the result equals
// group_features' wherever its double sums are exact (below 2^53).
__device__ void group_features_warp(const uint64_t* __restrict__ hkey, const uint32_t* __restrict__ hdiag, uint2 gr,
                                    const HitBits& hb, const DevBlock& A, const DevBlock& B, int comp, int minover,
                                    int binshift, const int64_t* __restrict__ anno, const int32_t* __restrict__ mdata,
                                    float f[TRI_NF])
{
    const int lane = lane_id();
    int s = (int)gr.x, e = (int)gr.y, n = e - s;
    uint64_t k0 = hkey[s];
    int ar = (int)((k0 >> hb.pbits) & ((1ull << hb.abits) - 1));
    int br = (int)(k0 >> (hb.pbits + hb.abits));
    float alen = (float)A.rlen[ar], blen = (float)B.rlen[br];
    uint64_t pmask = (1ull << hb.pbits) - 1;
    int amin = (int)(k0 & pmask), amax = (int)(hkey[e - 1] & pmask);
    long long isum = 0;
    unsigned long long isq = 0;
    int dmin = INT_MAX, dmax = INT_MIN;
    for (int i = s + lane; i < e; i += 32)
    {
        int d = (int)hdiag[i];
        isum += d;
        isq += (unsigned long long)((long long)d * d);
        dmin = min(dmin, d);
        dmax = max(dmax, d);
    }
    for (int o = 16; o; o >>= 1)
    {
        isum += __shfl_xor_sync(GD_FULL, isum, o);
        isq += __shfl_xor_sync(GD_FULL, isq, o);
    }
    dmin = __reduce_min_sync(GD_FULL, dmin);
    dmax = __reduce_max_sync(GD_FULL, dmax);
    double sum = (double)isum, sq = (double)isq;
    double mean = sum / n, var = fmax(sq / n - mean * mean, 0.0);
    int band = 1 << binshift, near = 0;
    for (int i = s + lane; i < e; i += 32)
        near += fabs((double)(int)hdiag[i] - mean) <= band;
    near = __reduce_add_sync(GD_FULL, near);
    long long mb = 0;
    if (anno)
    {
        for (int64_t j = anno[ar] + 2 * lane; j < anno[ar + 1]; j += 64)
            mb += mdata[j + 1] - mdata[j];
        for (int o = 16; o; o >>= 1)
            mb += __shfl_xor_sync(GD_FULL, mb, o);
    }
    features_out(n, alen, blen, amin, amax, mean, var, dmin, dmax, near, mb, anno != nullptr, comp, minover, f);
}

// groups of more hits than this get their features from a whole warp (group_features_warp)
constexpr int TRI_WARP_FEATURES = 32;

// ------------------------------------------------------------------------------------------
// MLP on tensor cores
// ------------------------------------------------------------------------------------------

constexpr int MT = 128;   // threads per CTA (4 warps)
constexpr int MR = 64;    // batch rows per CTA (16 per warp)

typedef __nv_bfloat16 bf16;

__device__ __forceinline__ void mma_bf16(float c[4], unsigned a0, unsigned a1, unsigned a2, unsigned a3, unsigned b0,
                                         unsigned b1)
{
    asm volatile("mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
                 "{%0,%1,%2,%3};\n"
                 : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
                 : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b0), "r"(b1));
}

__device__ __forceinline__ unsigned ld2(const bf16* p)
{
    return *reinterpret_cast<const unsigned*>(p);
}

// A fragment of a row-major bf16 tile (16 x 16) at (r0, k0), leading dimension ld
__device__ __forceinline__ void frag_a(const bf16* M, int ld, int r0, int k0, unsigned a[4])
{
    int g = lane_id() >> 2, t = lane_id() & 3;
    a[0] = ld2(M + (r0 + g) * ld + k0 + 2 * t);
    a[1] = ld2(M + (r0 + g + 8) * ld + k0 + 2 * t);
    a[2] = ld2(M + (r0 + g) * ld + k0 + 8 + 2 * t);
    a[3] = ld2(M + (r0 + g + 8) * ld + k0 + 8 + 2 * t);
}

// B fragment (16 x 8, K x N) from a matrix stored as [n][k] with leading dimension ldk
__device__ __forceinline__ void frag_b(const bf16* Wt, int ldk, int n0, int k0, unsigned b[2])
{
    int g = lane_id() >> 2, t = lane_id() & 3;
    b[0] = ld2(Wt + (n0 + g) * ldk + k0 + 2 * t);
    b[1] = ld2(Wt + (n0 + g) * ldk + k0 + 8 + 2 * t);
}

struct MlpSmem
{
    bf16 W1[TRI_H][16];      // [out][in], inputs 12..15 zero
    bf16 W2[TRI_H][TRI_H];   // [out][in]
    bf16 W2T[TRI_H][TRI_H];  // [in][out]
    bf16 W3[8][TRI_H];       // row 0 = W3, rows 1..7 zero
    bf16 X[MR][16];
    bf16 XT[16][MR];
    bf16 H1[MR][TRI_H];
    bf16 H1T[TRI_H][MR];
    bf16 H2[MR][TRI_H];
    bf16 dH2[MR][TRI_H];
    bf16 dH2T[TRI_H][MR];
    bf16 dH1T[TRI_H][MR];
    float b1[TRI_H], b2[TRI_H], w3[TRI_H];
    float z[MR], dz[MR];
    float b3;
};

__device__ void mlp_load(MlpSmem& S, const float* __restrict__ P, const float* __restrict__ x,
                         const int* __restrict__ perm, int64_t base, int64_t n)
{
    for (int i = threadIdx.x; i < TRI_H * 16; i += MT)
    {
        int o = i >> 4, f = i & 15;
        S.W1[o][f] = __float2bfloat16(f < TRI_NF ? P[TRI_OFF_W1 + o * TRI_NF + f] : 0.f);
    }
    for (int i = threadIdx.x; i < TRI_H * TRI_H; i += MT)
    {
        int o = i >> 6, k = i & 63;
        bf16 w = __float2bfloat16(P[TRI_OFF_W2 + i]);
        S.W2[o][k] = w;
        S.W2T[k][o] = w;
    }
    for (int i = threadIdx.x; i < 8 * TRI_H; i += MT)
        S.W3[i >> 6][i & 63] = __float2bfloat16((i >> 6) == 0 ? P[TRI_OFF_W3 + (i & 63)] : 0.f);
    for (int i = threadIdx.x; i < TRI_H; i += MT)
    {
        S.b1[i] = P[TRI_OFF_B1 + i];
        S.b2[i] = P[TRI_OFF_B2 + i];
        S.w3[i] = P[TRI_OFF_W3 + i];
    }
    if (threadIdx.x == 0)
        S.b3 = P[TRI_OFF_B3];
    for (int i = threadIdx.x; i < MR * 16; i += MT)
    {
        int r = i >> 4, f = i & 15;
        int64_t row = base + r;
        float v = 0.f;
        if (row < n && f < TRI_NF)
        {
            int64_t src = perm ? perm[row] : row;
            v = (x[src * TRI_NF + f] - P[TRI_OFF_MEAN + f]) / P[TRI_OFF_STD + f];
        }
        bf16 h = __float2bfloat16(v);
        S.X[r][f] = h;
        S.XT[f][r] = h;
    }
}

// forward of the warp's 16 rows: H1, H2 (bf16) and z (fp32) in shared memory
__device__ void mlp_forward_warp(MlpSmem& S)
{
    const int w = threadIdx.x >> 5, r0 = 16 * w;
    const int g = lane_id() >> 2, t = lane_id() & 3;
    unsigned a[4], b[2];
    frag_a(&S.X[0][0], 16, r0, 0, a);
#pragma unroll
    for (int nt = 0; nt < 8; nt++)
    {
        float c[4] = {0.f, 0.f, 0.f, 0.f};
        frag_b(&S.W1[0][0], 16, nt * 8, 0, b);
        mma_bf16(c, a[0], a[1], a[2], a[3], b[0], b[1]);
        int col = nt * 8 + 2 * t;
#pragma unroll
        for (int q = 0; q < 4; q++)
        {
            int r = r0 + g + (q >= 2 ? 8 : 0), cc = col + (q & 1);
            bf16 h = __float2bfloat16(fmaxf(c[q] + S.b1[cc], 0.f));
            S.H1[r][cc] = h;
            S.H1T[cc][r] = h;
        }
    }
    __syncwarp();
#pragma unroll
    for (int nt = 0; nt < 8; nt++)
    {
        float c[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll
        for (int ks = 0; ks < 4; ks++)
        {
            frag_a(&S.H1[0][0], TRI_H, r0, ks * 16, a);
            frag_b(&S.W2[0][0], TRI_H, nt * 8, ks * 16, b);
            mma_bf16(c, a[0], a[1], a[2], a[3], b[0], b[1]);
        }
        int col = nt * 8 + 2 * t;
#pragma unroll
        for (int q = 0; q < 4; q++)
        {
            int r = r0 + g + (q >= 2 ? 8 : 0), cc = col + (q & 1);
            S.H2[r][cc] = __float2bfloat16(fmaxf(c[q] + S.b2[cc], 0.f));
        }
    }
    __syncwarp();
    {
        float c[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll
        for (int ks = 0; ks < 4; ks++)
        {
            frag_a(&S.H2[0][0], TRI_H, r0, ks * 16, a);
            frag_b(&S.W3[0][0], TRI_H, 0, ks * 16, b);
            mma_bf16(c, a[0], a[1], a[2], a[3], b[0], b[1]);
        }
        if (t == 0)
        {
            S.z[r0 + g] = c[0] + S.b3;
            S.z[r0 + g + 8] = c[2] + S.b3;
        }
    }
    __syncwarp();
}

// ------------------------------------------------------------------------------------------
// inference: forward only, persistent CTAs (weights staged once), 128 rows per tile
// ------------------------------------------------------------------------------------------

constexpr int IR = 128;  // rows per tile: 32 per warp, two 16-row MMA tiles

struct InferSmem
{
    bf16 W1[TRI_H][16];
    bf16 W2[TRI_H][TRI_H];
    bf16 W3[8][TRI_H];
    bf16 X[IR][16];
    bf16 H[IR][TRI_H];  // layer-1 output, overwritten in place by layer 2
    float b1[TRI_H], b2[TRI_H], mean[16], stdv[16];
    float z[IR];
    float b3;
};

__device__ void infer_load_weights(InferSmem& S, const float* __restrict__ P)
{
    for (int i = threadIdx.x; i < TRI_H * 16; i += MT)
    {
        int o = i >> 4, f = i & 15;
        S.W1[o][f] = __float2bfloat16(f < TRI_NF ? P[TRI_OFF_W1 + o * TRI_NF + f] : 0.f);
    }
    for (int i = threadIdx.x; i < TRI_H * TRI_H; i += MT)
        S.W2[i >> 6][i & 63] = __float2bfloat16(P[TRI_OFF_W2 + i]);
    for (int i = threadIdx.x; i < 8 * TRI_H; i += MT)
        S.W3[i >> 6][i & 63] = __float2bfloat16((i >> 6) == 0 ? P[TRI_OFF_W3 + (i & 63)] : 0.f);
    for (int i = threadIdx.x; i < TRI_H; i += MT)
    {
        S.b1[i] = P[TRI_OFF_B1 + i];
        S.b2[i] = P[TRI_OFF_B2 + i];
    }
    if (threadIdx.x < 16)
    {
        int f = threadIdx.x;
        S.mean[f] = f < TRI_NF ? P[TRI_OFF_MEAN + f] : 0.f;
        S.stdv[f] = f < TRI_NF ? P[TRI_OFF_STD + f] : 1.f;
    }
    if (threadIdx.x == 0)
        S.b3 = P[TRI_OFF_B3];
}

// standardised bf16 input row r from raw features (the same arithmetic as mlp_load)
__device__ __forceinline__ void infer_put_row(InferSmem& S, int r, const float f[TRI_NF], bool valid)
{
#pragma unroll
    for (int j = 0; j < 16; j++)
    {
        float v = (j < TRI_NF && valid) ? (f[j] - S.mean[j]) / S.stdv[j] : 0.f;
        S.X[r][j] = __float2bfloat16(v);
    }
}

// z of the warp's 32 rows; the MMA sequence per row is the one of mlp_forward_warp, so both
// give bit-identical z for the same inputs
__device__ void infer_rows(InferSmem& S)
{
    const int w = threadIdx.x >> 5, g = lane_id() >> 2, t = lane_id() & 3;
    unsigned a[4], b[2];
#pragma unroll 1
    for (int mt = 0; mt < 2; mt++)
    {
        const int r0 = 32 * w + 16 * mt;
        frag_a(&S.X[0][0], 16, r0, 0, a);
#pragma unroll
        for (int nt = 0; nt < 8; nt++)
        {
            float c[4] = {0.f, 0.f, 0.f, 0.f};
            frag_b(&S.W1[0][0], 16, nt * 8, 0, b);
            mma_bf16(c, a[0], a[1], a[2], a[3], b[0], b[1]);
            int col = nt * 8 + 2 * t;
#pragma unroll
            for (int q = 0; q < 4; q++)
                S.H[r0 + g + (q >= 2 ? 8 : 0)][col + (q & 1)] = __float2bfloat16(fmaxf(c[q] + S.b1[col + (q & 1)], 0.f));
        }
        __syncwarp();
        float acc[8][4];
#pragma unroll
        for (int nt = 0; nt < 8; nt++)
        {
            acc[nt][0] = acc[nt][1] = acc[nt][2] = acc[nt][3] = 0.f;
#pragma unroll
            for (int ks = 0; ks < 4; ks++)
            {
                frag_a(&S.H[0][0], TRI_H, r0, ks * 16, a);
                frag_b(&S.W2[0][0], TRI_H, nt * 8, ks * 16, b);
                mma_bf16(acc[nt], a[0], a[1], a[2], a[3], b[0], b[1]);
            }
        }
        __syncwarp();
#pragma unroll
        for (int nt = 0; nt < 8; nt++)
        {
            int col = nt * 8 + 2 * t;
#pragma unroll
            for (int q = 0; q < 4; q++)
                S.H[r0 + g + (q >= 2 ? 8 : 0)][col + (q & 1)] =
                    __float2bfloat16(fmaxf(acc[nt][q] + S.b2[col + (q & 1)], 0.f));
        }
        __syncwarp();
        float c[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll
        for (int ks = 0; ks < 4; ks++)
        {
            frag_a(&S.H[0][0], TRI_H, r0, ks * 16, a);
            frag_b(&S.W3[0][0], TRI_H, 0, ks * 16, b);
            mma_bf16(c, a[0], a[1], a[2], a[3], b[0], b[1]);
        }
        if (t == 0)
        {
            S.z[r0 + g] = c[0] + S.b3;
            S.z[r0 + g + 8] = c[2] + S.b3;
        }
        __syncwarp();
    }
}

__global__ void __launch_bounds__(MT) k_mlp_forward(const float* __restrict__ P, const float* __restrict__ x, int64_t n,
                                                   float* p)
{
    extern __shared__ __align__(16) unsigned char infer_smem_f[];
    InferSmem& S = *reinterpret_cast<InferSmem*>(infer_smem_f);
    infer_load_weights(S, P);
    __syncthreads();
    const int64_t ntiles = (n + IR - 1) / IR;
    for (int64_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x)
    {
        const int64_t row = tile * IR + threadIdx.x;
        float f[TRI_NF];
#pragma unroll
        for (int j = 0; j < TRI_NF; j++)
            f[j] = row < n ? x[row * TRI_NF + j] : 0.f;
        infer_put_row(S, threadIdx.x, f, row < n);
        __syncthreads();
        infer_rows(S);
        __syncthreads();
        if (row < n)
            p[row] = 1.f / (1.f + __expf(-S.z[threadIdx.x]));
        __syncthreads();
    }
}

// The learned triage of the pair groups that selection kept (groups[0, ng), after
// k_select_groups): a CTA per tile of IR groups -- each group's features (a thread per short
// group, the lanes of its warp together over a long one), the MLP over the tile on tensor
// cores, the skip flag (p < thr) at the group's slot and, when feat is given, its raw
// features.  With P == nullptr only the features are computed.  Selection keeps its own
// full-occupancy kernel: the MLP's shared memory would hold the selection's latency-bound
// candidate tests to a third of the resident warps.
struct TriArgs
{
    const uint64_t* hkey;
    const uint32_t* hdiag;
    HitBits hb;
    DevBlock A, B;
    int comp, minover, binshift;
    const int64_t* anno;
    const int32_t* mdata;
    const float* P;
    float thr;
    float* feat;
    const uint2* groups;
    uint8_t* skip;
};

__global__ void __launch_bounds__(MT) k_triage_groups(unsigned ng, TriArgs a, unsigned* nskip)
{
    extern __shared__ __align__(16) unsigned char infer_smem_t[];
    InferSmem& S = *reinterpret_cast<InferSmem*>(infer_smem_t);
    if (a.P)
        infer_load_weights(S, a.P);
    __syncthreads();
    unsigned cnt = 0;
    const int64_t ntiles = ((int64_t)ng + IR - 1) / IR;
    for (int64_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x)
    {
        const int r = threadIdx.x;
        const int64_t slot = tile * IR + r;
        const bool mine = slot < (int64_t)ng;
        float f[TRI_NF];
#pragma unroll
        for (int j = 0; j < TRI_NF; j++)
            f[j] = 0.f;
        const uint2 gr = mine ? a.groups[slot] : make_uint2(0u, 0u);
        if (mine && gr.y - gr.x <= TRI_WARP_FEATURES)
            group_features(a.hkey, a.hdiag, gr, a.hb, a.A, a.B, a.comp, a.minover, a.binshift, a.anno, a.mdata, f);
        // a long group is walked by its warp's lanes together, not by one thread while the CTA
        // waits for it at the next barrier
        unsigned big = __ballot_sync(GD_FULL, mine && gr.y - gr.x > TRI_WARP_FEATURES);
        while (big)
        {
            const int j = __ffs(big) - 1;
            big &= big - 1;
            const uint2 gj = make_uint2(__shfl_sync(GD_FULL, gr.x, j), __shfl_sync(GD_FULL, gr.y, j));
            float fj[TRI_NF];
            group_features_warp(a.hkey, a.hdiag, gj, a.hb, a.A, a.B, a.comp, a.minover, a.binshift, a.anno, a.mdata,
                                fj);
            if (lane_id() == j)
#pragma unroll
                for (int k = 0; k < TRI_NF; k++)
                    f[k] = fj[k];
        }
        bool drop = false;
        if (a.P)
        {
            infer_put_row(S, r, f, mine);
            __syncthreads();
            infer_rows(S);
            __syncthreads();
            drop = mine && 1.f / (1.f + __expf(-S.z[r])) < a.thr;
        }
        if (mine)
        {
            a.skip[slot] = drop ? 1 : 0;
            cnt += drop;
            if (a.feat)
#pragma unroll
                for (int j = 0; j < TRI_NF; j++)
                    a.feat[slot * TRI_NF + j] = f[j];
        }
        __syncthreads();  // S.X / S.z are rewritten by the next tile
    }
    if (a.P)
    {
        for (int o = 16; o; o >>= 1)
            cnt += __shfl_xor_sync(GD_FULL, cnt, o);
        if (lane_id() == 0 && cnt)
            atomicAdd(nskip, cnt);
    }
}

__global__ void __launch_bounds__(MT) k_mlp_grad(const float* __restrict__ P, const float* __restrict__ x,
                                                const float* __restrict__ y, const int* __restrict__ perm, int64_t n0,
                                                int n, float pos_weight, float* grad, float* loss)
{
    extern __shared__ __align__(16) unsigned char mlp_smem_g[];
    MlpSmem& S = *reinterpret_cast<MlpSmem*>(mlp_smem_g);
    const int64_t base = n0 + (int64_t)blockIdx.x * MR;
    const int64_t end = n0 + n;
    mlp_load(S, P, x, perm, base, end);
    __syncthreads();
    mlp_forward_warp(S);
    __syncthreads();
    // dL/dz of the weighted binary cross-entropy, mean over the batch
    if (threadIdx.x < MR)
    {
        int r = threadIdx.x;
        int64_t row = base + r;
        float dz = 0.f, l = 0.f;
        if (row < end)
        {
            int64_t src = perm ? perm[row] : row;
            float yy = y[src], z = S.z[r];
            float wgt = yy > 0.5f ? pos_weight : 1.f;
            float pz = 1.f / (1.f + __expf(-z));
            dz = wgt * (pz - yy) / (float)n;
            // log(1 + e^-|z|) + max(z,0) - z*y, numerically stable
            l = wgt * (fmaxf(z, 0.f) - z * yy + log1pf(__expf(-fabsf(z)))) / (float)n;
        }
        S.dz[r] = dz;
        for (int o = 16; o; o >>= 1)
            l += __shfl_xor_sync(GD_FULL, l, o);
        if ((r & 31) == 0)
            atomicAdd(loss, l);
    }
    __syncthreads();
    for (int i = threadIdx.x; i < MR * TRI_H; i += MT)
    {
        int r = i >> 6, o = i & 63;
        float h2 = __bfloat162float(S.H2[r][o]);
        bf16 d = __float2bfloat16(h2 > 0.f ? S.dz[r] * S.w3[o] : 0.f);
        S.dH2[r][o] = d;
        S.dH2T[o][r] = d;
    }
    if (threadIdx.x < TRI_H)
    {
        int o = threadIdx.x;
        float gw3 = 0.f, gb2 = 0.f;
        for (int r = 0; r < MR; r++)
        {
            float h2 = __bfloat162float(S.H2[r][o]);
            gw3 += S.dz[r] * h2;
            gb2 += h2 > 0.f ? S.dz[r] * S.w3[o] : 0.f;
        }
        atomicAdd(grad + TRI_OFF_W3 + o, gw3);
        atomicAdd(grad + TRI_OFF_B2 + o, gb2);
    }
    else if (threadIdx.x == TRI_H)
    {
        float gb3 = 0.f;
        for (int r = 0; r < MR; r++)
            gb3 += S.dz[r];
        atomicAdd(grad + TRI_OFF_B3, gb3);
    }
    __syncthreads();
    const int w = threadIdx.x >> 5, g = lane_id() >> 2, t = lane_id() & 3;
    unsigned a[4], b[2];
    // dW2[o][i] = sum_r dH2[r][o] H1[r][i]: warp w owns o in [16w, 16w+16)
#pragma unroll
    for (int it = 0; it < 8; it++)
    {
        float c[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll
        for (int ks = 0; ks < 4; ks++)
        {
            frag_a(&S.dH2T[0][0], MR, 16 * w, ks * 16, a);
            frag_b(&S.H1T[0][0], MR, it * 8, ks * 16, b);
            mma_bf16(c, a[0], a[1], a[2], a[3], b[0], b[1]);
        }
#pragma unroll
        for (int q = 0; q < 4; q++)
        {
            int o = 16 * w + g + (q >= 2 ? 8 : 0), i = it * 8 + 2 * t + (q & 1);
            atomicAdd(grad + TRI_OFF_W2 + o * TRI_H + i, c[q]);
        }
    }
    // dH1[r][i] = (sum_o dH2[r][o] W2[o][i]) * [H1 > 0]: warp w owns rows [16w, 16w+16)
#pragma unroll
    for (int it = 0; it < 8; it++)
    {
        float c[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll
        for (int ks = 0; ks < 4; ks++)
        {
            frag_a(&S.dH2[0][0], TRI_H, 16 * w, ks * 16, a);
            frag_b(&S.W2T[0][0], TRI_H, it * 8, ks * 16, b);
            mma_bf16(c, a[0], a[1], a[2], a[3], b[0], b[1]);
        }
#pragma unroll
        for (int q = 0; q < 4; q++)
        {
            int r = 16 * w + g + (q >= 2 ? 8 : 0), i = it * 8 + 2 * t + (q & 1);
            float h1 = __bfloat162float(S.H1[r][i]);
            S.dH1T[i][r] = __float2bfloat16(h1 > 0.f ? c[q] : 0.f);
        }
    }
    __syncthreads();
    if (threadIdx.x < TRI_H)
    {
        int i = threadIdx.x;
        float gb1 = 0.f;
        for (int r = 0; r < MR; r++)
            gb1 += __bfloat162float(S.dH1T[i][r]);
        atomicAdd(grad + TRI_OFF_B1 + i, gb1);
    }
    // dW1[i][f] = sum_r dH1[r][i] X[r][f]: warp w owns i in [16w, 16w+16), features in 2 tiles
#pragma unroll
    for (int ft = 0; ft < 2; ft++)
    {
        float c[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll
        for (int ks = 0; ks < 4; ks++)
        {
            frag_a(&S.dH1T[0][0], MR, 16 * w, ks * 16, a);
            frag_b(&S.XT[0][0], MR, ft * 8, ks * 16, b);
            mma_bf16(c, a[0], a[1], a[2], a[3], b[0], b[1]);
        }
#pragma unroll
        for (int q = 0; q < 4; q++)
        {
            int i = 16 * w + g + (q >= 2 ? 8 : 0), f = ft * 8 + 2 * t + (q & 1);
            if (f < TRI_NF)
                atomicAdd(grad + TRI_OFF_W1 + i * TRI_NF + f, c[q]);
        }
    }
}

__global__ void k_adam(float* P, const float* __restrict__ G, float* M, float* V, int step, float lr)
{
    int i = TRI_OFF_W1 + blockIdx.x * 256 + threadIdx.x;
    if (i >= TRI_NPARAM)
        return;
    const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
    float g = G[i];
    float m = M[i] = b1 * M[i] + (1.f - b1) * g;
    float v = V[i] = b2 * V[i] + (1.f - b2) * g * g;
    float mh = m / (1.f - powf(b1, (float)step)), vh = v / (1.f - powf(b2, (float)step));
    P[i] -= lr * mh / (sqrtf(vh) + eps);
}

static int mlp_smem_attr(const void* fn)
{
    GD_CUDA(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(MlpSmem)));
    return 0;
}

static int infer_grid(int64_t ntiles)
{
    static int grids[GD_MAX_DEVICES] = {};
    const int dv = gd_device();
    if (dv < 0)
        return -1;
    int& blocks = grids[dv];
    if (!blocks)
    {
        int dev = 0, nsm = 0, per = 0;
        GD_CUDA(cudaGetDevice(&dev));
        GD_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
        GD_CUDA(cudaFuncSetAttribute((const void*)k_triage_groups, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)sizeof(InferSmem)));
        GD_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_triage_groups, MT, sizeof(InferSmem)));
        blocks = nsm * std::max(per, 1);
    }
    return (int)std::min<int64_t>(ntiles, blocks);
}

int launch_mlp_forward(const float* params, const float* x, int64_t n, float* p, cudaStream_t s)
{
    if (n <= 0)
        return 0;
    int grid = infer_grid((n + IR - 1) / IR);
    if (grid <= 0)
        return -1;
    k_mlp_forward<<<grid, MT, sizeof(InferSmem), s>>>(params, x, n, p);
    GD_LAUNCHED(1);
    GD_CUDA(cudaGetLastError());
    return 0;
}

int launch_mlp_grad_perm(const float* params, const float* x, const float* y, const int* perm, int64_t n0, int n,
                         float pos_weight, float* grad, float* loss, cudaStream_t s)
{
    static bool done[GD_MAX_DEVICES] = {};
    const int dv = gd_device();
    if (dv < 0)
        return -1;
    if (!done[dv])
    {
        if (mlp_smem_attr((const void*)k_mlp_grad))
            return -1;
        done[dv] = true;
    }
    GD_CUDA(cudaMemsetAsync(grad, 0, sizeof(float) * TRI_NPARAM, s));
    GD_CUDA(cudaMemsetAsync(loss, 0, sizeof(float), s));
    if (n <= 0)
        return 0;
    k_mlp_grad<<<gd_cdiv(n, MR), MT, sizeof(MlpSmem), s>>>(params, x, y, perm, n0, n, pos_weight, grad, loss);
    GD_LAUNCHED(1);
    GD_CUDA(cudaGetLastError());
    return 0;
}

int launch_mlp_grad(const float* params, const float* x, const float* y, int n, float pos_weight, float* grad,
                    float* loss, cudaStream_t s)
{
    return launch_mlp_grad_perm(params, x, y, nullptr, 0, n, pos_weight, grad, loss, s);
}

int launch_adam(float* params, const float* grad, float* m, float* v, int step, float lr, cudaStream_t s)
{
    k_adam<<<gd_cdiv(TRI_NPARAM - TRI_OFF_W1, 256), 256, 0, s>>>(params, grad, m, v, step, lr);
    GD_LAUNCHED(1);
    GD_CUDA(cudaGetLastError());
    return 0;
}

int launch_triage_groups(const uint2* groups, unsigned ng, const uint64_t* hkey, const uint32_t* hdiag, HitBits hb,
                         const DevBlock& A, const DevBlock& B, int comp, int minover, int binshift,
                         const int64_t* amask_anno, const int32_t* amask_data, const float* params, float threshold,
                         float* feat, uint8_t* skip, unsigned* nskip, cudaStream_t s)
{
    if (ng == 0)
        return 0;
    int grid = infer_grid(((int64_t)ng + IR - 1) / IR);
    if (grid <= 0)
        return -1;
    TriArgs a{hkey, hdiag, hb, A, B, comp, minover, binshift, amask_anno, amask_data, params, threshold, feat, groups,
              skip};
    k_triage_groups<<<grid, MT, sizeof(InferSmem), s>>>(ng, a, nskip);
    GD_LAUNCHED(1);
    GD_CUDA(cudaGetLastError());
    return 0;
}

}  // namespace gd
