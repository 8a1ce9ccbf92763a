// gd_output.cu -- the overlap buffer in HBM and its sort (Write_Overlap_Buffer's SORT_OVL
// order, dalign/align.c:5786-5813: aread, bread, orientation, abpos).
//
// The records of every Match_Filter call stay on the device.  Read-out sorts them with two
// stable LSD radix sorts -- first by (orientation, abpos, aepos, bbpos), then by (dropped,
// aread, bread) -- so the final order is (aread, bread, orientation, abpos) with ties broken
// by aepos and bbpos, the same total order the host comparator used.  An exclusive scan of
// the records' trace lengths gives the compacted trace offsets, and one warp per record
// moves each record and its trace bytes into a contiguous, sorted buffer that the host
// copies out in one transfer.
#include "gd_output.cuh"

namespace gd
{

__global__ void k_ovl_append(const OutRec* __restrict__ src, uint64_t n, uint64_t t0, OutRec* __restrict__ dst)
{
    uint64_t i = (uint64_t)blockIdx.x * 256 + threadIdx.x;
    if (i >= n)
        return;
    OutRec o = src[i];
    o.toff += t0;
    dst[i] = o;
}

__global__ void k_ovl_extent(const OutRec* __restrict__ r, uint64_t n, unsigned* ext)
{
    uint64_t i = (uint64_t)blockIdx.x * 256 + threadIdx.x;
    unsigned lo = 0xffffffffu, hi = 0, pos = 0;
    if (i < n)
    {
        const OutRec& o = r[i];
        lo = (unsigned)min(o.aread, o.bread);
        hi = (unsigned)max(o.aread, o.bread);
        pos = (unsigned)max(max(o.aepos, o.bepos), max(o.abpos, o.bbpos));
    }
    lo = __reduce_min_sync(GD_FULL, lo);
    hi = __reduce_max_sync(GD_FULL, hi);
    pos = __reduce_max_sync(GD_FULL, pos);
    if (lane_id() == 0)
    {
        atomicMin(ext, lo);
        atomicMax(ext + 1, hi);
        atomicMax(ext + 2, pos);
    }
}

__global__ void k_ovl_key_lo(const OutRec* __restrict__ r, uint64_t n, int pbits, int with_comp,
                             uint64_t* __restrict__ key, uint32_t* __restrict__ val)
{
    uint64_t i = (uint64_t)blockIdx.x * 256 + threadIdx.x;
    if (i >= n)
        return;
    const OutRec& o = r[i];
    key[i] = ((uint64_t)(with_comp ? o.flags & 1 : 0) << (3 * pbits)) | ((uint64_t)o.abpos << (2 * pbits)) |
             ((uint64_t)o.aepos << pbits) | (uint64_t)o.bbpos;
    val[i] = (uint32_t)i;
}

__global__ void k_ovl_key_hi(const OutRec* __restrict__ r, const uint32_t* __restrict__ perm, uint64_t n, int rbits,
                             unsigned rmin, int only_identity, uint64_t* __restrict__ key, unsigned long long* nkept)
{
    uint64_t i = (uint64_t)blockIdx.x * 256 + threadIdx.x;
    bool keep = false;
    if (i < n)
    {
        const OutRec& o = r[perm[i]];
        bool drop = only_identity && o.aread != o.bread;
        keep = !drop;
        key[i] = ((uint64_t)drop << (2 * rbits)) | ((uint64_t)((unsigned)o.aread - rmin) << rbits) |
                 (uint64_t)((unsigned)o.bread - rmin);
    }
    unsigned m = __ballot_sync(GD_FULL, keep);
    if (lane_id() == 0 && m)
        atomicAdd(nkept, (unsigned long long)__popc(m));
}

__global__ void k_ovl_len(const OutRec* __restrict__ r, const uint32_t* __restrict__ perm, uint64_t n, int tbytes,
                          uint64_t* __restrict__ len)
{
    uint64_t i = (uint64_t)blockIdx.x * 256 + threadIdx.x;
    if (i < n)
        len[i] = (uint64_t)r[perm[i]].tlen * tbytes;
}

// one warp per record: the record, then its trace bytes (8-byte words where both ends allow)
__global__ void k_ovl_gather(const OutRec* __restrict__ r, const uint8_t* __restrict__ tr,
                             const uint32_t* __restrict__ perm, const uint64_t* __restrict__ off, uint64_t n,
                             int tbytes, OutRec* __restrict__ out, uint8_t* __restrict__ outtr)
{
    const uint64_t w = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = lane_id();
    if (w >= n)
        return;
    OutRec o = r[perm[w]];
    const uint8_t* src = tr + o.toff;
    uint8_t* dst = outtr + off[w];
    const uint64_t len = (uint64_t)o.tlen * tbytes;
    if (lane == 0)
    {
        o.toff = off[w];
        o.pad = 0;
        out[w] = o;
    }
    if (((uintptr_t)src & 7) == ((uintptr_t)dst & 7))
    {
        // head bytes up to 8-byte alignment, aligned words, tail bytes
        uint64_t head = (8 - ((uintptr_t)dst & 7)) & 7;
        if (head > len)
            head = len;
        if ((uint64_t)lane < head)
            dst[lane] = src[lane];
        const uint64_t nw = (len - head) >> 3;
        const uint64_t* s8 = reinterpret_cast<const uint64_t*>(src + head);
        uint64_t* d8 = reinterpret_cast<uint64_t*>(dst + head);
        for (uint64_t j = lane; j < nw; j += 32)
            d8[j] = s8[j];
        for (uint64_t j = head + nw * 8 + lane; j < len; j += 32)
            dst[j] = src[j];
    }
    else
    {
        for (uint64_t j = lane; j < len; j += 32)
            dst[j] = src[j];
    }
}

// .las record header: tlen, diffs, abpos, bbpos, aepos, bepos, flags, aread, bread, pad
// (Overlap without its trace pointer, dalign/align.h:307-312), 40 little-endian bytes.  A
// record starts at any even byte offset (1-byte trace points), so headers are read and
// written byte by byte.
__device__ __forceinline__ int32_t rd32(const uint8_t* q)
{
    return (int32_t)((uint32_t)q[0] | ((uint32_t)q[1] << 8) | ((uint32_t)q[2] << 16) | ((uint32_t)q[3] << 24));
}

__global__ void k_las_parse(const uint8_t* __restrict__ raw, const int64_t* __restrict__ off, uint64_t n,
                            OutRec* __restrict__ rec)
{
    uint64_t i = (uint64_t)blockIdx.x * 256 + threadIdx.x;
    if (i >= n)
        return;
    const uint8_t* h = raw + off[i];
    OutRec o;
    o.tlen = rd32(h);
    o.diffs = rd32(h + 4);
    o.abpos = rd32(h + 8);
    o.bbpos = rd32(h + 12);
    o.aepos = rd32(h + 16);
    o.bepos = rd32(h + 20);
    o.flags = (uint32_t)rd32(h + 24);
    o.aread = rd32(h + 28);
    o.bread = rd32(h + 32);
    o.pad = rd32(h + 36);
    o.toff = (uint64_t)off[i] + 40;
    rec[i] = o;
}

// one warp per record: lanes write the 40 header bytes, then the trace bytes
__global__ void k_las_emit(const OutRec* __restrict__ r, const uint8_t* __restrict__ tr,
                           const uint32_t* __restrict__ perm, const uint64_t* __restrict__ toff, uint64_t n,
                           int tbytes, uint8_t* __restrict__ out)
{
    const uint64_t w = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = lane_id();
    if (w >= n)
        return;
    const OutRec o = r[perm[w]];
    uint8_t* dst = out + 40 * w + toff[w];
    const int32_t f[10] = {o.tlen, o.diffs, o.abpos, o.bbpos, o.aepos, o.bepos, (int32_t)o.flags, o.aread, o.bread,
                           o.pad};
    for (int j = lane; j < 40; j += 32)
        dst[j] = (uint8_t)((uint32_t)f[j >> 2] >> (8 * (j & 3)));
    const uint8_t* src = tr + o.toff;
    const uint64_t len = (uint64_t)o.tlen * tbytes;
    for (uint64_t j = lane; j < len; j += 32)
        dst[40 + j] = src[j];
}

int launch_las_parse(const uint8_t* raw, const int64_t* off, uint64_t n, OutRec* rec, cudaStream_t s)
{
    if (n == 0)
        return 0;
    k_las_parse<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(raw, off, n, rec);
    GD_LAUNCHED(1);
    GD_CUDA(cudaGetLastError());
    return 0;
}

int launch_las_emit(const OutRec* r, const uint8_t* tr, const uint32_t* perm, const uint64_t* toff, uint64_t n,
                    int tbytes, uint8_t* out, cudaStream_t s)
{
    if (n == 0)
        return 0;
    const uint64_t threads = n * 32;
    k_las_emit<<<(unsigned)((threads + 255) / 256), 256, 0, s>>>(r, tr, perm, toff, n, tbytes, out);
    GD_LAUNCHED(1);
    GD_CUDA(cudaGetLastError());
    return 0;
}

static inline unsigned grid256(uint64_t n)
{
    return (unsigned)((n + 255) / 256);
}

int launch_ovl_append(const OutRec* src, uint64_t n, uint64_t t0, OutRec* dst, cudaStream_t s)
{
    if (n == 0)
        return 0;
    k_ovl_append<<<grid256(n), 256, 0, s>>>(src, n, t0, dst);
    GD_LAUNCHED(1);
    GD_CUDA(cudaGetLastError());
    return 0;
}

int launch_ovl_extent(const OutRec* r, uint64_t n, unsigned* ext, cudaStream_t s)
{
    if (n == 0)
        return 0;
    k_ovl_extent<<<grid256(n), 256, 0, s>>>(r, n, ext);
    GD_LAUNCHED(1);
    GD_CUDA(cudaGetLastError());
    return 0;
}

int launch_ovl_key_lo(const OutRec* r, uint64_t n, int pbits, int with_comp, uint64_t* key, uint32_t* val,
                      cudaStream_t s)
{
    if (n == 0)
        return 0;
    k_ovl_key_lo<<<grid256(n), 256, 0, s>>>(r, n, pbits, with_comp, key, val);
    GD_LAUNCHED(1);
    GD_CUDA(cudaGetLastError());
    return 0;
}

int launch_ovl_key_hi(const OutRec* r, const uint32_t* perm, uint64_t n, int rbits, unsigned rmin, int only_identity,
                      uint64_t* key, unsigned long long* nkept, cudaStream_t s)
{
    if (n == 0)
        return 0;
    k_ovl_key_hi<<<grid256(n), 256, 0, s>>>(r, perm, n, rbits, rmin, only_identity, key, nkept);
    GD_LAUNCHED(1);
    GD_CUDA(cudaGetLastError());
    return 0;
}

int launch_ovl_len(const OutRec* r, const uint32_t* perm, uint64_t n, int tbytes, uint64_t* len, cudaStream_t s)
{
    if (n == 0)
        return 0;
    k_ovl_len<<<grid256(n), 256, 0, s>>>(r, perm, n, tbytes, len);
    GD_LAUNCHED(1);
    GD_CUDA(cudaGetLastError());
    return 0;
}

int launch_ovl_gather(const OutRec* r, const uint8_t* tr, const uint32_t* perm, const uint64_t* off, uint64_t n,
                      int tbytes, OutRec* out, uint8_t* outtr, cudaStream_t s)
{
    if (n == 0)
        return 0;
    const uint64_t threads = n * 32;
    k_ovl_gather<<<(unsigned)((threads + 255) / 256), 256, 0, s>>>(r, tr, perm, off, n, tbytes, out, outtr);
    GD_LAUNCHED(1);
    GD_CUDA(cudaGetLastError());
    return 0;
}

}  // namespace gd
