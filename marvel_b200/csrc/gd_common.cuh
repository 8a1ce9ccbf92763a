// gd_common.cuh -- shared device types and helpers of the sm_100a overlap path.
#pragma once
#include <cstdint>
#include <cstdio>
#include <cuda_runtime.h>

#define GD_WARP 32
#define GD_FULL 0xffffffffu

#define GD_CUDA(call)                                                                          \
    do                                                                                         \
    {                                                                                          \
        cudaError_t e_ = (call);                                                               \
        if (e_ != cudaSuccess)                                                                 \
        {                                                                                      \
            gd_set_error("%s:%d: CUDA error %s: %s", __FILE__, __LINE__, cudaGetErrorName(e_), \
                         cudaGetErrorString(e_));                                              \
            return -1;                                                                         \
        }                                                                                      \
    } while (0)

void gd_set_error(const char* fmt, ...);

// Number of kernels this library has launched (all contexts), for launch accounting.
extern unsigned long long g_gd_launches;
#define GD_LAUNCHED(n) (g_gd_launches += (n))

// A DB block resident in HBM, laid out like the reference's in-memory block
// (db/DB.c:1349-1410): one byte per base (0..3), a 4 before read 0 and after every read,
// read i at bases[boff[i]].  The allocation carries 16 bytes of slack on each side so
// that 8-byte windows around any base stay in bounds.
struct DevBlock
{
    const uint8_t* bases;
    const int64_t* boff;
    const int32_t* rlen;
    int32_t nreads;
    int32_t maxlen;
    int32_t ufirst;
    // the block's bases 2 bits each, 16 per word (base i at index PK_BIAS + i, a 4 packed as
    // 0): the aligner's match extension reads 16 bases per word
    const uint32_t* pk;
};

// index in DevBlock::pk of bases[0] (the byte buffer's slack before it plus its leading 4)
constexpr int PK_BIAS = 33;

// k-mer slots of a block: read r owns slots [kstart(r), kstart(r+1)), one per position p of
// its last k-mer base (p >= k-1); slot kstart(r) + p - (k-1).  A block's reads are >= k long.
__device__ __forceinline__ int64_t kstart_of(const DevBlock& b, int r, int K)
{
    return b.boff[r] - (int64_t)K * r;
}

// largest r in [0, nreads) with kstart(r) <= s
__device__ __forceinline__ int read_of_slot(const DevBlock& b, int64_t s, int K)
{
    int lo = 0, hi = b.nreads - 1;
    while (lo < hi)
    {
        int mid = (lo + hi + 1) >> 1;
        if (kstart_of(b, mid, K) <= s)
            lo = mid;
        else
            hi = mid - 1;
    }
    return lo;
}

// Device-side error status shared by all kernels of a context.  Kernels never trap:
// they record the first failure here and skip the remaining work.
struct DevStatus
{
    int32_t code;   // 0 = ok
    int32_t where;  // pair index or item that failed
    int32_t info;
    int32_t pad;
};

enum
{
    GD_ERR_OK = 0,
    GD_ERR_BAND_WIDTH = 1,   // wave band wider than the register tile
    GD_ERR_PEBBLES = 2,      // pebble arena exhausted
    GD_ERR_TRACE = 3,        // trace scratch exhausted
    GD_ERR_MATCHES = 4,      // per-pair path list exhausted
    GD_ERR_OUTPUT = 5,       // overlap output buffer exhausted
    GD_ERR_EMPTY_BAND = 6,   // wave band emptied while the wave continues
    GD_ERR_RING = 7,         // band left the ring window
    GD_ERR_BRIDGE = 8,       // daligner2: bridging scratch exhausted (info: ints needed)
    GD_ERR_TRACE8 = 9,       // daligner2: a trace value above 255 fails the 8-bit compression check
    GD_ERR_TRACE_STRIDE = 10,  // Local_Alignment batch: a trace longer than half the caller's stride (info: stride needed)
};

__device__ __forceinline__ void gd_fail(DevStatus* st, int code, int where, int info)
{
    if (atomicCAS(&st->code, 0, code) == 0)
    {
        st->where = where;
        st->info = info;
    }
}

__device__ __forceinline__ unsigned lanemask_lt()
{
    unsigned m;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}

__device__ __forceinline__ int lane_id()
{
    int l;
    asm("mov.u32 %0, %%laneid;" : "=r"(l));
    return l;
}

// Per-device one-time set-up (kernel attributes, occupancy-derived grids) is kept in arrays
// indexed by the current device, so that contexts on several GPUs of one process each get it.
constexpr int GD_MAX_DEVICES = 64;

// the current device, or -1 if it cannot be had or is beyond GD_MAX_DEVICES
inline int gd_device()
{
    int d = 0;
    return (cudaGetDevice(&d) == cudaSuccess && d >= 0 && d < GD_MAX_DEVICES) ? d : -1;
}

template <typename T>
__host__ __device__ inline T gd_cdiv(T a, T b)
{
    return (a + b - 1) / b;
}
