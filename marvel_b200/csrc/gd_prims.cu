// gd_prims.cu -- exclusive scan and stable LSD radix sort (see gd_prims.cuh).
#include "gd_prims.cuh"

#include <algorithm>

namespace gd
{

template <typename T>
__global__ void __launch_bounds__(SCAN_THREADS) k_scan_reduce(const T* __restrict__ in, int64_t n, T* partial)
{
    __shared__ T red[SCAN_THREADS / 32];
    int64_t base = (int64_t)blockIdx.x * SCAN_TILE;
    T acc = 0;
#pragma unroll
    for (int i = 0; i < SCAN_ITEMS; i++)
    {
        int64_t idx = base + i * SCAN_THREADS + threadIdx.x;
        if (idx < n)
            acc += in[idx];
    }
    for (int o = 16; o; o >>= 1)
        acc += __shfl_xor_sync(GD_FULL, acc, o);
    if ((threadIdx.x & 31) == 0)
        red[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x == 0)
    {
        T t = 0;
        for (int w = 0; w < SCAN_THREADS / 32; w++)
            t += red[w];
        partial[blockIdx.x] = t;
    }
}

// Single-CTA exclusive scan of the tile partials (in place); writes the grand total.
template <typename T>
__global__ void __launch_bounds__(1024) k_scan_partials(T* partial, int64_t m, T* total)
{
    __shared__ T warp_tot[32];
    __shared__ T carry_s;
    if (threadIdx.x == 0)
        carry_s = 0;
    __syncthreads();
    int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    for (int64_t base = 0; base < m; base += 1024)
    {
        int64_t idx = base + threadIdx.x;
        T v = idx < m ? partial[idx] : 0;
        T x = v;
        for (int o = 1; o < 32; o <<= 1)
        {
            T y = __shfl_up_sync(GD_FULL, x, o);
            if (lane >= o)
                x += y;
        }
        if (lane == 31)
            warp_tot[wid] = x;
        __syncthreads();
        if (wid == 0)
        {
            T w = warp_tot[lane];
            T z = w;
            for (int o = 1; o < 32; o <<= 1)
            {
                T y = __shfl_up_sync(GD_FULL, z, o);
                if (lane >= o)
                    z += y;
            }
            warp_tot[lane] = z - w;  // exclusive over warps
        }
        __syncthreads();
        T carry = carry_s;
        T excl = carry + warp_tot[wid] + x - v;
        if (idx < m)
            partial[idx] = excl;
        __syncthreads();
        if (threadIdx.x == 1023)
            carry_s = excl + v;
        __syncthreads();
    }
    if (threadIdx.x == 0 && total)
        *total = carry_s;
}

template <typename T>
__global__ void __launch_bounds__(SCAN_THREADS) k_scan_down(const T* in, T* out, int64_t n, const T* partial)
{
    __shared__ T tile[SCAN_TILE];
    __shared__ T warp_tot[SCAN_THREADS / 32];
    int64_t base = (int64_t)blockIdx.x * SCAN_TILE;
#pragma unroll
    for (int i = 0; i < SCAN_ITEMS; i++)
    {
        int64_t idx = base + i * SCAN_THREADS + threadIdx.x;
        tile[i * SCAN_THREADS + threadIdx.x] = idx < n ? in[idx] : 0;
    }
    __syncthreads();
    T loc[SCAN_ITEMS];
    T sum = 0;
#pragma unroll
    for (int i = 0; i < SCAN_ITEMS; i++)
    {
        loc[i] = sum;
        sum += tile[threadIdx.x * SCAN_ITEMS + i];
    }
    int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    T x = sum;
    for (int o = 1; o < 32; o <<= 1)
    {
        T y = __shfl_up_sync(GD_FULL, x, o);
        if (lane >= o)
            x += y;
    }
    if (lane == 31)
        warp_tot[wid] = x;
    __syncthreads();
    T wpre = 0;
    for (int w = 0; w < wid; w++)
        wpre += warp_tot[w];
    T pre = partial[blockIdx.x] + wpre + x - sum;
#pragma unroll
    for (int i = 0; i < SCAN_ITEMS; i++)
        tile[threadIdx.x * SCAN_ITEMS + i] = pre + loc[i];
    __syncthreads();
#pragma unroll
    for (int i = 0; i < SCAN_ITEMS; i++)
    {
        int64_t idx = base + i * SCAN_THREADS + threadIdx.x;
        if (idx < n)
            out[idx] = tile[i * SCAN_THREADS + threadIdx.x];
    }
}

template <typename T>
int exclusive_scan(const T* in, T* out, int64_t n, T* total, void* scratch, cudaStream_t s)
{
    int64_t tiles = gd_cdiv<int64_t>(n, SCAN_TILE);
    T* partial = (T*)scratch;
    if (n <= 0)
    {
        if (total)
            GD_CUDA(cudaMemsetAsync(total, 0, sizeof(T), s));
        return 0;
    }
    k_scan_reduce<T><<<(unsigned)tiles, SCAN_THREADS, 0, s>>>(in, n, partial);
    GD_LAUNCHED(1);
    k_scan_partials<T><<<1, 1024, 0, s>>>(partial, tiles, total);
    GD_LAUNCHED(1);
    k_scan_down<T><<<(unsigned)tiles, SCAN_THREADS, 0, s>>>(in, out, n, partial);
    GD_LAUNCHED(1);
    GD_CUDA(cudaGetLastError());
    return 0;
}

template int exclusive_scan<uint32_t>(const uint32_t*, uint32_t*, int64_t, uint32_t*, void*, cudaStream_t);
template int exclusive_scan<uint64_t>(const uint64_t*, uint64_t*, int64_t, uint64_t*, void*, cudaStream_t);

// ---------------------------------------------------------------------------------------
// radix sort
// ---------------------------------------------------------------------------------------

template <typename K>
__global__ void __launch_bounds__(RS_THREADS) k_rs_hist(const K* __restrict__ keys, int64_t n, int shift,
                                                       uint32_t* counts, int ntiles)
{
    // one histogram per warp, plain shared-memory atomics; full tiles of 16-byte aligned keys
    // are read as 16-byte vectors
    __shared__ uint32_t h[RS_WARPS][256];
    const int w = threadIdx.x >> 5;
#pragma unroll
    for (int i = 0; i < RS_WARPS; i++)
        h[i][threadIdx.x] = 0;
    __syncthreads();
    const int64_t base = (int64_t)blockIdx.x * RS_TILE;
    constexpr int PER = 16 / sizeof(K);  // keys per vector
    if (base + RS_TILE <= n && ((uintptr_t)keys & 15) == 0)
    {
        const uint4* v = reinterpret_cast<const uint4*>(keys + base);
        uint4 x[RS_TILE / PER / RS_THREADS];
#pragma unroll
        for (int i = 0; i < RS_TILE / PER / RS_THREADS; i++)
            x[i] = v[i * RS_THREADS + threadIdx.x];
#pragma unroll
        for (int i = 0; i < RS_TILE / PER / RS_THREADS; i++)
        {
            if (sizeof(K) == 4)
            {
                atomicAdd(&h[w][(x[i].x >> shift) & 255u], 1u);
                atomicAdd(&h[w][(x[i].y >> shift) & 255u], 1u);
                atomicAdd(&h[w][(x[i].z >> shift) & 255u], 1u);
                atomicAdd(&h[w][(x[i].w >> shift) & 255u], 1u);
            }
            else
            {
                const uint64_t k0 = ((uint64_t)x[i].y << 32) | x[i].x, k1 = ((uint64_t)x[i].w << 32) | x[i].z;
                atomicAdd(&h[w][(unsigned)(k0 >> shift) & 255u], 1u);
                atomicAdd(&h[w][(unsigned)(k1 >> shift) & 255u], 1u);
            }
        }
    }
    else
    {
        for (int i = 0; i < RS_ROUNDS; i++)
        {
            int64_t idx = base + i * RS_THREADS + threadIdx.x;
            if (idx < n)
                atomicAdd(&h[w][(unsigned)(keys[idx] >> shift) & 255u], 1u);
        }
    }
    __syncthreads();
    uint32_t t = 0;
#pragma unroll
    for (int i = 0; i < RS_WARPS; i++)
        t += h[i][threadIdx.x];
    counts[(int64_t)threadIdx.x * ntiles + blockIdx.x] = t;
}

// Shared memory of one scatter tile: the tile's items re-ordered by digit (stable), the
// per-warp digit counts, the tile's digit starts and its global digit offsets.
template <typename K>
struct RsTile
{
    K key[RS_TILE];
    uint32_t val[RS_TILE];
    uint32_t wcnt[RS_WARPS][256];
    uint32_t lstart[256];
    uint32_t toff[256];
};

// Ranks every item of the tile (warps own contiguous sub-tiles, rounds walk them in order,
// match-any groups within a round: stable), places it in a digit-sorted copy of the tile in
// shared memory, and then writes the copy out in tile order: items of one digit leave as a
// contiguous run, so the global writes coalesce.
template <typename K>
__global__ void __launch_bounds__(RS_THREADS) k_rs_scatter(const K* __restrict__ kin, const uint32_t* __restrict__ vin,
                                                          K* __restrict__ kout, uint32_t* __restrict__ vout, int64_t n,
                                                          int shift, const uint32_t* __restrict__ offs, int ntiles)
{
    extern __shared__ __align__(16) unsigned char rs_smem[];
    RsTile<K>& S = *reinterpret_cast<RsTile<K>*>(rs_smem);
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
    for (int i = 0; i < RS_WARPS; i++)
        S.wcnt[i][threadIdx.x] = 0;
    S.toff[threadIdx.x] = offs[(int64_t)threadIdx.x * ntiles + blockIdx.x];
    __syncthreads();

    const int64_t tbase = (int64_t)blockIdx.x * RS_TILE;
    const int64_t base = tbase + (int64_t)w * (RS_ROUNDS * 32);
    K key[RS_ROUNDS];
    uint32_t val[RS_ROUNDS];
    uint32_t rank[RS_ROUNDS];
    const unsigned lt = lanemask_lt();
    // all of the sub-tile's loads in flight before the ranking
#pragma unroll
    for (int r = 0; r < RS_ROUNDS; r++)
    {
        int64_t idx = base + r * 32 + lane;
        if (idx < n)
        {
            key[r] = kin[idx];
            val[r] = vin[idx];
        }
    }
#pragma unroll
    for (int r = 0; r < RS_ROUNDS; r++)
    {
        int64_t idx = base + r * 32 + lane;
        bool valid = idx < n;
        unsigned d = valid ? (unsigned)(key[r] >> shift) & 255u : 256u;
        unsigned peers = __match_any_sync(GD_FULL, d);
        unsigned c = valid ? S.wcnt[w][d] : 0;
        rank[r] = c + __popc(peers & lt);
        __syncwarp();
        if (valid && (peers & lt) == 0)
            S.wcnt[w][d] = c + __popc(peers);
        __syncwarp();
    }
    __syncthreads();
    // per digit: warp offsets within the digit's run, and the run's length
    uint32_t tot = 0;
#pragma unroll
    for (int i = 0; i < RS_WARPS; i++)
    {
        uint32_t t = S.wcnt[i][threadIdx.x];
        S.wcnt[i][threadIdx.x] = tot;
        tot += t;
    }
    // exclusive scan of the run lengths over the 256 digits (one per thread)
    {
        uint32_t x = tot;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1)
        {
            uint32_t t = __shfl_up_sync(GD_FULL, x, o);
            if (lane >= o)
                x += t;
        }
        __shared__ uint32_t wsum[RS_WARPS];
        if (lane == 31)
            wsum[w] = x;
        __syncthreads();
        uint32_t wo = 0;
#pragma unroll
        for (int i = 0; i < RS_WARPS; i++)
            wo += i < w ? wsum[i] : 0;
        S.lstart[threadIdx.x] = wo + x - tot;
    }
    __syncthreads();
#pragma unroll
    for (int r = 0; r < RS_ROUNDS; r++)
    {
        int64_t idx = base + r * 32 + lane;
        if (idx < n)
        {
            unsigned d = (unsigned)(key[r] >> shift) & 255u;
            uint32_t pos = S.lstart[d] + S.wcnt[w][d] + rank[r];
            S.key[pos] = key[r];
            S.val[pos] = val[r];
        }
    }
    __syncthreads();
    const int tn = (int)min((int64_t)RS_TILE, n - tbase);
    for (int i = threadIdx.x; i < tn; i += RS_THREADS)
    {
        K k = S.key[i];
        unsigned d = (unsigned)(k >> shift) & 255u;
        uint32_t dest = S.toff[d] + (uint32_t)i - S.lstart[d];
        kout[dest] = k;
        vout[dest] = S.val[i];
    }
}

// ---------------------------------------------------------------------------------------
// pipelined scatter: a persistent CTA streams its tiles' keys and values into shared memory
// with bulk asynchronous copies (two stages, one mbarrier each), so the next tile arrives
// while this one is ranked, re-ordered in place and written out.  Same ranking as
// k_rs_scatter, so the same (stable) order.
// ---------------------------------------------------------------------------------------

__device__ int g_rs_wait_failed;  // set when a stage's copy did not complete within the wait limit

__device__ __forceinline__ uint32_t smem_addr(const void* p)
{
    return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, unsigned count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, unsigned bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes)
                 : "memory");
}

// bounded wait for the phase with the given parity; false if the limit ran out
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, unsigned parity, int polls = 1 << 22)
{
    const uint32_t a = smem_addr(bar);
    for (int it = 0; it < polls; it++)
    {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}"
            : "=r"(done)
            : "r"(a), "r"(parity)
            : "memory");
        if (done)
            return true;
    }
    return false;
}

// global -> this CTA's shared memory; both addresses 16-byte aligned, bytes a multiple of 16
__device__ __forceinline__ void bulk_load(void* dst, const void* src, unsigned bytes, uint64_t* bar)
{
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_addr(dst)),
                 "l"(src), "r"(bytes), "r"(smem_addr(bar))
                 : "memory");
}

template <bool V>
struct RsPipeVals
{
    uint32_t val[2][RS_TILE];
};
template <>
struct RsPipeVals<false>
{
};

// V = false: a keys-only sort (no value arrays)
template <typename K, bool V = true>
struct RsPipe : RsPipeVals<V>
{
    K key[2][RS_TILE];
    uint32_t wcnt[RS_WARPS][256];
    uint32_t lstart[256];
    uint32_t toff[256];
    uint32_t wsum[RS_WARPS];
    uint64_t full[2];
};

template <typename K, bool V>
constexpr int rs_pipe_ctas()
{
    return (sizeof(K) == 4 || !V) ? 3 : 2;
}

// Full tiles (all but possibly the last) arrive by bulk copy; a ragged last tile is read
// with plain loads.  Requires 16-byte aligned kin and vin.  V = false: keys only.
template <typename K, bool V = true, int F = RsFinal::NONE>
__global__ void __launch_bounds__(RS_THREADS, rs_pipe_ctas<K, V>())
    k_rs_scatter_pipe(const K* __restrict__ kin, const uint32_t* __restrict__ vin, K* __restrict__ kout,
                      uint32_t* __restrict__ vout, int64_t n, int shift, const uint32_t* __restrict__ offs, int ntiles,
                      RsFinal fin)
{
    extern __shared__ __align__(128) unsigned char rs_pipe_smem[];
    RsPipe<K, V>& S = *reinterpret_cast<RsPipe<K, V>*>(rs_pipe_smem);
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int nfull = (int)(n / RS_TILE);
    constexpr unsigned TILE_BYTES = RS_TILE * (sizeof(K) + (V ? sizeof(uint32_t) : 0));
    if (threadIdx.x == 0)
    {
        mbar_init(&S.full[0], 1);
        mbar_init(&S.full[1], 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    int tile = blockIdx.x;
    if (threadIdx.x == 0 && tile < nfull)
    {
        mbar_expect_tx(&S.full[0], TILE_BYTES);
        bulk_load(S.key[0], kin + (int64_t)tile * RS_TILE, RS_TILE * sizeof(K), &S.full[0]);
        if constexpr (V)
            bulk_load(S.val[0], vin + (int64_t)tile * RS_TILE, RS_TILE * 4, &S.full[0]);
    }
    uint32_t toff = tile < ntiles ? offs[(int64_t)threadIdx.x * ntiles + tile] : 0;
    unsigned parity = 0;  // bit st: phase of stage st's barrier
    const unsigned lt = lanemask_lt();
    for (int st = 0; tile < ntiles; tile += gridDim.x, st ^= 1)
    {
        const int next = tile + gridDim.x;
        // the other stage was released by the barrier that ended the previous tile
        if (threadIdx.x == 0 && next < nfull)
        {
            mbar_expect_tx(&S.full[st ^ 1], TILE_BYTES);
            bulk_load(S.key[st ^ 1], kin + (int64_t)next * RS_TILE, RS_TILE * sizeof(K), &S.full[st ^ 1]);
            if constexpr (V)
                bulk_load(S.val[st ^ 1], vin + (int64_t)next * RS_TILE, RS_TILE * 4, &S.full[st ^ 1]);
        }
        const uint32_t toff_next = next < ntiles ? offs[(int64_t)threadIdx.x * ntiles + next] : 0;
        S.toff[threadIdx.x] = toff;
#pragma unroll
        for (int i = 0; i < RS_WARPS; i++)
            S.wcnt[i][threadIdx.x] = 0;
        const int64_t tbase = (int64_t)tile * RS_TILE;
        const int tn = (int)min((int64_t)RS_TILE, n - tbase);
        K* skey = S.key[st];
        uint32_t* sval = nullptr;
        if constexpr (V)
            sval = S.val[st];
        bool ok = true;
        if (tile < nfull)
        {
            ok = mbar_wait(&S.full[st], (parity >> st) & 1u);
            parity ^= 1u << st;
        }
        else
            for (int i = threadIdx.x; i < tn; i += RS_THREADS)
            {
                skey[i] = kin[tbase + i];
                if constexpr (V)
                    sval[i] = vin[tbase + i];
            }
        if (__syncthreads_or(!ok))
        {
            // all threads leave; wait (bounded) for the copies still in flight first
            if (threadIdx.x == 0)
                atomicExch(&g_rs_wait_failed, 1);
            if (ok == false)
                mbar_wait(&S.full[st], ((parity >> st) & 1u) ^ 1u);
            if (next < nfull)
                mbar_wait(&S.full[st ^ 1], (parity >> (st ^ 1)) & 1u);
            return;
        }

        K key[RS_ROUNDS];
        uint32_t val[RS_ROUNDS];
        uint32_t rank2[RS_ROUNDS / 2];  // two 16-bit ranks per register (a rank is < RS_TILE)
#pragma unroll
        for (int r = 0; r < RS_ROUNDS; r++)
        {
            const int i = w * (RS_ROUNDS * 32) + r * 32 + lane;
            const bool valid = i < tn;
            key[r] = valid ? skey[i] : (K)0;
            if constexpr (V)
                val[r] = valid ? sval[i] : 0u;
            unsigned d = valid ? (unsigned)(key[r] >> shift) & 255u : 256u;
            unsigned peers = __match_any_sync(GD_FULL, d);
            unsigned c = valid ? S.wcnt[w][d] : 0;
            const uint32_t rk = c + __popc(peers & lt);
            if (r & 1)
                rank2[r >> 1] |= rk << 16;
            else
                rank2[r >> 1] = rk;
            __syncwarp();
            if (valid && (peers & lt) == 0)
                S.wcnt[w][d] = c + __popc(peers);
            __syncwarp();
        }
        __syncthreads();
        uint32_t tot = 0;
#pragma unroll
        for (int i = 0; i < RS_WARPS; i++)
        {
            uint32_t t = S.wcnt[i][threadIdx.x];
            S.wcnt[i][threadIdx.x] = tot;
            tot += t;
        }
        {
            uint32_t x = tot;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1)
            {
                uint32_t t = __shfl_up_sync(GD_FULL, x, o);
                if (lane >= o)
                    x += t;
            }
            if (lane == 31)
                S.wsum[w] = x;
            __syncthreads();
            uint32_t wo = 0;
#pragma unroll
            for (int i = 0; i < RS_WARPS; i++)
                wo += i < w ? S.wsum[i] : 0;
            S.lstart[threadIdx.x] = wo + x - tot;
        }
        __syncthreads();
        // the stage's tile is in registers: re-order it in place
#pragma unroll
        for (int r = 0; r < RS_ROUNDS; r++)
        {
            const int i = w * (RS_ROUNDS * 32) + r * 32 + lane;
            if (i < tn)
            {
                unsigned d = (unsigned)(key[r] >> shift) & 255u;
                uint32_t pos = S.lstart[d] + S.wcnt[w][d] + ((rank2[r >> 1] >> (16 * (r & 1))) & 0xffffu);
                skey[pos] = key[r];
                if constexpr (V)
                    sval[pos] = val[r];
            }
        }
        __syncthreads();
        for (int i = threadIdx.x; i < tn; i += RS_THREADS)
        {
            K k = skey[i];
            unsigned d = (unsigned)(k >> shift) & 255u;
            uint32_t dest = S.toff[d] + (uint32_t)i - S.lstart[d];
            if constexpr (F == RsFinal::INDEX)
            {
                const uint32_t v = sval[i];
                static_cast<K*>(fin.a)[dest] = k;
                fin.b[dest] = (int32_t)(v >> fin.bits);
                fin.c[dest] = (int32_t)(v & ((1u << fin.bits) - 1u)) + fin.kmer - 1;
            }
            else if constexpr (F == RsFinal::HITS)
            {
                const uint64_t hk = (uint64_t)k >> fin.bits;
                const int bpos = (int)((uint64_t)k & ((1ull << fin.bits) - 1));
                static_cast<uint64_t*>(fin.a)[dest] = hk;
                fin.b[dest] = (int32_t)((int)(hk & ((1ull << fin.pbits) - 1)) - bpos);
            }
            else
            {
                kout[dest] = k;
                if constexpr (V)
                    vout[dest] = sval[i];
            }
        }
        // this stage is refilled by the bulk copy engine two tiles on: order these generic
        // accesses before it
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        __syncthreads();
        toff = toff_next;
    }
}

// Test of the wait's expiry path: an mbarrier armed for 16 bytes that no copy will bring
// (none is issued, so nothing is in flight when the block leaves), waited on with a short
// limit; the expiry raises the same flag a stalled tile copy raises.
__global__ void k_test_wait_expiry(int polls)
{
    __shared__ __align__(8) uint64_t bar;
    if (threadIdx.x == 0)
    {
        mbar_init(&bar, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    if (threadIdx.x == 0)
        mbar_expect_tx(&bar, 16);
    __syncthreads();
    const bool ok = mbar_wait(&bar, 0, polls);
    if (__syncthreads_or(!ok) && threadIdx.x == 0)
        atomicExch(&g_rs_wait_failed, 1);
    __syncthreads();
    if (threadIdx.x == 0)
        asm volatile("mbarrier.inval.shared::cta.b64 [%0];" ::"r"(smem_addr(&bar)) : "memory");
}

int radix_sort_test_wait_expiry(int polls, cudaStream_t s)
{
    k_test_wait_expiry<<<1, 32, 0, s>>>(polls);
    GD_LAUNCHED(1);
    GD_CUDA(cudaGetLastError());
    return 0;
}

int radix_sort_wait_check(cudaStream_t s)
{
    int h = 0;
    GD_CUDA(cudaMemcpyFromSymbolAsync(&h, g_rs_wait_failed, sizeof(int), 0, cudaMemcpyDeviceToHost, s));
    GD_CUDA(cudaStreamSynchronize(s));
    if (h)
    {
        int z = 0;
        GD_CUDA(cudaMemcpyToSymbolAsync(g_rs_wait_failed, &z, sizeof(int), 0, cudaMemcpyHostToDevice, s));
        GD_CUDA(cudaStreamSynchronize(s));
        gd_set_error("radix sort: a tile copy did not complete within the wait limit");
        return -1;
    }
    return 0;
}

template <typename K>
int radix_sort_pairs(K* k0, uint32_t* v0, K* k1, uint32_t* v1, int64_t n, int begin_bit, int end_bit, void* scratch,
                     cudaStream_t s, const RsFinal* fin)
{
    if (n <= 1 || end_bit <= begin_bit)
        return 0;
    int64_t tiles64 = gd_cdiv<int64_t>(n, RS_TILE);
    if (tiles64 > (1 << 30) || n > 0xffffffffll)
    {
        gd_set_error("radix sort of %lld items exceeds 32-bit offsets", (long long)n);
        return -1;
    }
    int ntiles = (int)tiles64;
    static int pipe_grids[GD_MAX_DEVICES] = {};
    const int dv = gd_device();
    if (dv < 0)
    {
        gd_set_error("radix sort: no usable current device");
        return -1;
    }
    int& pipe_grid = pipe_grids[dv];
    if (!pipe_grid)
    {
        GD_CUDA(cudaFuncSetAttribute((const void*)k_rs_scatter<K>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)sizeof(RsTile<K>)));
        GD_CUDA(cudaFuncSetAttribute((const void*)k_rs_scatter_pipe<K>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)sizeof(RsPipe<K>)));
        GD_CUDA(cudaFuncSetAttribute((const void*)k_rs_scatter_pipe<K, true, RsFinal::INDEX>,
                                     cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(RsPipe<K>)));
        int dev = 0, sms = 0, per = 0;
        GD_CUDA(cudaGetDevice(&dev));
        GD_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
        GD_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_rs_scatter_pipe<K>, RS_THREADS,
                                                              sizeof(RsPipe<K>)));
        pipe_grid = sms * std::max(per, 1);
    }
    // the bulk copies need 16-byte aligned sources (tile starts are then aligned too)
    const bool pipe = ((uintptr_t)k0 & 15) == 0 && ((uintptr_t)k1 & 15) == 0 && ((uintptr_t)v0 & 15) == 0 &&
                      ((uintptr_t)v1 & 15) == 0;
    if (fin && (fin->kind != RsFinal::INDEX || !pipe))
    {
        gd_set_error("radix sort: this final pass needs the pipelined kernel and an index target");
        return -1;
    }
    int64_t ncnt = (int64_t)ntiles * 256;
    uint32_t* counts = (uint32_t*)scratch;
    void* sscr = (void*)(((uintptr_t)(counts + ncnt) + 255) & ~(uintptr_t)255);
    int cur = 0;
    for (int b = begin_bit; b < end_bit; b += 8)
    {
        K* kin = cur ? k1 : k0;
        uint32_t* vin = cur ? v1 : v0;
        K* kout = cur ? k0 : k1;
        uint32_t* vout = cur ? v0 : v1;
        k_rs_hist<K><<<ntiles, RS_THREADS, 0, s>>>(kin, n, b, counts, ntiles);
        GD_LAUNCHED(1);
        if (exclusive_scan<uint32_t>(counts, counts, ncnt, (uint32_t*)nullptr, sscr, s))
            return -1;
        if (fin && b + 8 >= end_bit)
            k_rs_scatter_pipe<K, true, RsFinal::INDEX><<<std::min(ntiles, pipe_grid), RS_THREADS, sizeof(RsPipe<K>),
                                                         s>>>(kin, vin, kout, vout, n, b, counts, ntiles, *fin);
        else if (pipe)
            k_rs_scatter_pipe<K><<<std::min(ntiles, pipe_grid), RS_THREADS, sizeof(RsPipe<K>), s>>>(
                kin, vin, kout, vout, n, b, counts, ntiles, RsFinal{});
        else
            k_rs_scatter<K><<<ntiles, RS_THREADS, sizeof(RsTile<K>), s>>>(kin, vin, kout, vout, n, b, counts, ntiles);
        GD_LAUNCHED(1);
        cur ^= 1;
    }
    GD_CUDA(cudaGetLastError());
    if (pipe && radix_sort_wait_check(s))
        return -1;
    return cur;
}

template <typename K>
int radix_sort_keys(K* k0, K* k1, int64_t n, int begin_bit, int end_bit, void* scratch, cudaStream_t s,
                    const RsFinal* fin)
{
    if (n <= 1 || end_bit <= begin_bit)
        return 0;
    int64_t tiles64 = gd_cdiv<int64_t>(n, RS_TILE);
    if (tiles64 > (1 << 30) || n > 0xffffffffll)
    {
        gd_set_error("radix sort of %lld items exceeds 32-bit offsets", (long long)n);
        return -1;
    }
    if (((uintptr_t)k0 & 15) || ((uintptr_t)k1 & 15))
    {
        gd_set_error("keys-only radix sort needs 16-byte aligned arrays");
        return -1;
    }
    if (fin && fin->kind != RsFinal::HITS)
    {
        gd_set_error("keys-only radix sort: this final pass needs a hit target");
        return -1;
    }
    const int ntiles = (int)tiles64;
    static int grids[GD_MAX_DEVICES] = {};
    const int dv = gd_device();
    if (dv < 0)
    {
        gd_set_error("radix sort: no usable current device");
        return -1;
    }
    int& grid = grids[dv];
    if (!grid)
    {
        GD_CUDA(cudaFuncSetAttribute((const void*)k_rs_scatter_pipe<K, false>,
                                     cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(RsPipe<K, false>)));
        GD_CUDA(cudaFuncSetAttribute((const void*)k_rs_scatter_pipe<K, false, RsFinal::HITS>,
                                     cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(RsPipe<K, false>)));
        int sms = 0, per = 0;
        GD_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dv));
        GD_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_rs_scatter_pipe<K, false>, RS_THREADS,
                                                              sizeof(RsPipe<K, false>)));
        grid = sms * std::max(per, 1);
    }
    int64_t ncnt = (int64_t)ntiles * 256;
    uint32_t* counts = (uint32_t*)scratch;
    void* sscr = (void*)(((uintptr_t)(counts + ncnt) + 255) & ~(uintptr_t)255);
    int cur = 0;
    for (int b = begin_bit; b < end_bit; b += 8)
    {
        K* kin = cur ? k1 : k0;
        K* kout = cur ? k0 : k1;
        k_rs_hist<K><<<ntiles, RS_THREADS, 0, s>>>(kin, n, b, counts, ntiles);
        GD_LAUNCHED(1);
        if (exclusive_scan<uint32_t>(counts, counts, ncnt, (uint32_t*)nullptr, sscr, s))
            return -1;
        if (fin && b + 8 >= end_bit)
            k_rs_scatter_pipe<K, false, RsFinal::HITS><<<std::min(ntiles, grid), RS_THREADS,
                                                         sizeof(RsPipe<K, false>), s>>>(kin, nullptr, kout, nullptr,
                                                                                        n, b, counts, ntiles, *fin);
        else
            k_rs_scatter_pipe<K, false><<<std::min(ntiles, grid), RS_THREADS, sizeof(RsPipe<K, false>), s>>>(
                kin, nullptr, kout, nullptr, n, b, counts, ntiles, RsFinal{});
        GD_LAUNCHED(1);
        cur ^= 1;
    }
    GD_CUDA(cudaGetLastError());
    if (radix_sort_wait_check(s))
        return -1;
    return cur;
}

template int radix_sort_keys<uint64_t>(uint64_t*, uint64_t*, int64_t, int, int, void*, cudaStream_t,
                                       const RsFinal*);
template int radix_sort_pairs<uint32_t>(uint32_t*, uint32_t*, uint32_t*, uint32_t*, int64_t, int, int, void*,
                                        cudaStream_t, const RsFinal*);
template int radix_sort_pairs<uint64_t>(uint64_t*, uint32_t*, uint64_t*, uint32_t*, int64_t, int, int, void*,
                                        cudaStream_t, const RsFinal*);

}  // namespace gd
