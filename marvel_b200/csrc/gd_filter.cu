// gd_filter.cu -- k-mer filter kernels for sm_100a.
//
// Restates dalign/filter.c's index build (tuple_thread :400-490, Sort_Kmers :698-903) and
// A x B merge (count_thread :948-1056, merge_thread :1061-1231) as data-parallel passes
// over HBM-resident arrays: one thread per k-mer slot for extraction, one thread per index
// entry for the join, with binary searches replacing the reference's merge cursors.
#include "gd_filter.cuh"
#include "gd_prims.cuh"

namespace gd
{

constexpr int FT = 256;

// Four consecutive slots per thread: one read lookup, the codes rolled base by base within
// a read, keys and values stored as 16-byte vectors.  The value is the slot index, or with
// pbits >= 0 the packed (read << pbits | first position), so that no search is needed after
// the sort (the packed values keep the slots' order, so the sort's ties come out the same).
template <typename K>
__global__ void __launch_bounds__(FT) k_extract(DevBlock b, const int64_t* __restrict__ mask_anno,
                                               const int32_t* __restrict__ mask_data, int kmer, K* keys, uint32_t* vals,
                                               int64_t nslots, uint32_t* nmasked, int pbits)
{
    const int64_t s0 = ((int64_t)blockIdx.x * FT + threadIdx.x) * 4;
    unsigned nm = 0;
    if (s0 < nslots)
    {
        const K kmask = (2 * kmer >= (int)(8 * sizeof(K))) ? ~(K)0 : (((K)1 << (2 * kmer)) - 1);
        int r = read_of_slot(b, s0, kmer);
        int64_t kst = kstart_of(b, r, kmer), knext = kstart_of(b, r + 1, kmer);
        K kv[4], code = 0;
        uint32_t vv[4];
        int have = -2;  // first position whose code is in `code`
        const int nj = (int)min((int64_t)4, nslots - s0);
#pragma unroll
        for (int j = 0; j < 4; j++)
        {
            if (j >= nj)
                break;
            const int64_t s = s0 + j;
            while (s >= knext)
            {
                r++;
                kst = knext;
                knext = kstart_of(b, r + 1, kmer);
                have = -2;
            }
            const int p0 = (int)(s - kst);
            const int rpos = p0 + kmer - 1;
            const uint8_t* src = b.bases + b.boff[r];
            if (have == p0 - 1)
                code = ((code << 2) | (K)src[rpos]) & kmask;
            else
            {
                code = 0;
                for (int t = 0; t < kmer; t++)
                    code = (code << 2) | (K)src[p0 + t];
            }
            have = p0;
            bool masked = false;
            if (mask_anno)
            {
                // the segment of unmasked bases containing p0 must also contain rpos
                // (segments [0,b0) [e0,b1) ... [e_last,rlen), tuple_thread's loop :428-457)
                int64_t f0 = mask_anno[r], f1 = mask_anno[r + 1];
                int q = b.rlen[r];
                int p = 0;
                for (int64_t a = f0; a < f1; a += 2)
                {
                    int ib = mask_data[a], ie = mask_data[a + 1];
                    if (p0 < ib)
                    {
                        q = ib;
                        break;
                    }
                    p = ie;
                    q = b.rlen[r];
                }
                masked = !(p0 >= p && rpos < q);
            }
            nm += masked;
            kv[j] = masked ? (K)~(K)0 : code;
            vv[j] = pbits >= 0 ? ((uint32_t)r << pbits) | (uint32_t)p0 : (uint32_t)s;
        }
        if (nj == 4)
        {
            if (sizeof(K) == 4)
                *reinterpret_cast<uint4*>(keys + s0) = make_uint4((uint32_t)kv[0], (uint32_t)kv[1], (uint32_t)kv[2],
                                                                  (uint32_t)kv[3]);
            else
            {
                *reinterpret_cast<ulonglong2*>(keys + s0) = make_ulonglong2((unsigned long long)kv[0],
                                                                            (unsigned long long)kv[1]);
                *reinterpret_cast<ulonglong2*>(keys + s0 + 2) = make_ulonglong2((unsigned long long)kv[2],
                                                                                (unsigned long long)kv[3]);
            }
            *reinterpret_cast<uint4*>(vals + s0) = make_uint4(vv[0], vv[1], vv[2], vv[3]);
        }
        else
            for (int j = 0; j < nj; j++)
            {
                keys[s0 + j] = kv[j];
                vals[s0 + j] = vv[j];
            }
    }
    for (int o = 16; o; o >>= 1)
        nm += __shfl_xor_sync(GD_FULL, nm, o);
    if (nm && lane_id() == 0)
        atomicAdd(nmasked, nm);
}

template <typename K>
int launch_extract(const DevBlock& b, const int64_t* mask_anno, const int32_t* mask_data, int kmer, K* keys,
                   uint32_t* vals, int64_t nslots, uint32_t* nmasked, int pbits, cudaStream_t s)
{
    GD_CUDA(cudaMemsetAsync(nmasked, 0, sizeof(uint32_t), s));
    if (nslots <= 0)
        return 0;
    const int64_t threads = (nslots + 3) / 4;
    k_extract<K><<<(unsigned)gd_cdiv<int64_t>(threads, FT), FT, 0, s>>>(b, mask_anno, mask_data, kmer, keys, vals,
                                                                         nslots, nmasked, pbits);
    GD_LAUNCHED(1);
    GD_CUDA(cudaGetLastError());
    return 0;
}

// code/read/rpos of the sorted index from packed values (read << pbits | first position)
template <typename K>
__global__ void __launch_bounds__(FT) k_unpack(const K* __restrict__ skeys, const uint32_t* __restrict__ svals,
                                              int64_t n, int pbits, int kmer, K* __restrict__ code,
                                              int32_t* __restrict__ read, int32_t* __restrict__ rpos)
{
    const int64_t i = (int64_t)blockIdx.x * FT + threadIdx.x;
    if (i >= n)
        return;
    const uint32_t v = svals[i];
    code[i] = skeys[i];
    read[i] = (int32_t)(v >> pbits);
    rpos[i] = (int32_t)(v & ((1u << pbits) - 1u)) + kmer - 1;
}

template <typename K>
int launch_unpack(const K* skeys, const uint32_t* svals, int64_t n, int pbits, int kmer, K* code, int32_t* read,
                  int32_t* rpos, cudaStream_t s)
{
    if (n <= 0)
        return 0;
    k_unpack<K><<<(unsigned)gd_cdiv<int64_t>(n, FT), FT, 0, s>>>(skeys, svals, n, pbits, kmer, code, read, rpos);
    GD_LAUNCHED(1);
    GD_CUDA(cudaGetLastError());
    return 0;
}

__global__ void __launch_bounds__(FT) k_decode(DevBlock b, int kmer, const uint32_t* __restrict__ slots, int64_t n,
                                              int32_t* read, int32_t* rpos)
{
    int64_t i = (int64_t)blockIdx.x * FT + threadIdx.x;
    if (i >= n)
        return;
    int64_t s = slots[i];
    int r = read_of_slot(b, s, kmer);
    read[i] = r;
    rpos[i] = (int)(s - kstart_of(b, r, kmer)) + kmer - 1;
}

template <typename K>
int launch_decode(const DevBlock& b, int kmer, const uint32_t* slots, int64_t n, int32_t* read, int32_t* rpos,
                  cudaStream_t s)
{
    if (n <= 0)
        return 0;
    k_decode<<<(unsigned)gd_cdiv<int64_t>(n, FT), FT, 0, s>>>(b, kmer, slots, n, read, rpos);
    GD_LAUNCHED(1);
    GD_CUDA(cudaGetLastError());
    return 0;
}

// ---- -b: frequency-weighted tuples ---------------------------------------------------

constexpr int BT = 128;

// The bases of one read, read forward through a cached aligned 8-byte word (the block
// buffer has slack on both sides, so the word around any base is in bounds).
struct BaseStream
{
    const uint8_t* s;
    uintptr_t word;
    uint64_t w;
    __device__ __forceinline__ int at(int p)
    {
        const uintptr_t a = (uintptr_t)(s + p);
        if ((a >> 3) != word)
        {
            word = a >> 3;
            w = __ldg(reinterpret_cast<const unsigned long long*>(a & ~(uintptr_t)7));
        }
        return (int)(w >> (8 * (a & 7))) & 0xff;
    }
};

// One scan of bases [p, q) of a read: the loop of biased_tuple_thread (dalign/filter.c:536-570
// over a mask track's unmasked segment, :583-612 over a whole read), left at the first
// iteration that starts at or after pend.  The window s[p-k+1..p] is the low 2k bits of c, so
// the trim and the slide take the leaving base from c.  When growing runs into q the
// untracked scan stops, the tracked one still tests the window (now s[q-k..q-1]) and keeps it
// at position q; its trim is skipped there, as it cannot remove a base from a window below
// norm when every weight is >= 0.
template <typename F>
__device__ __forceinline__ void bias_scan(BaseStream& bs, int p, int q, int pend, bool tracked, const BiasParams& bp,
                                          uint64_t kmask, F&& keep)
{
    uint64_t c = 0;
    int a = 0, k = 1;
    while (p < q && p < pend)
    {
        int x = bs.at(p);
        a += bp.w[x];
        c = (c << 2) | (uint64_t)x;
        bool cut = false;
        while (a < bp.norm && k < bp.kmer)
        {
            if (++p >= q)
            {
                cut = true;
                break;
            }
            k += 1;
            x = bs.at(p);
            a += bp.w[x];
            c = (c << 2) | (uint64_t)x;
        }
        if (cut && !tracked)
            return;
        if (!cut)
            while (true)
            {
                const int u = a - bp.w[(int)(c >> (2 * (k - 1))) & 3];
                if (u < bp.norm)
                    break;
                a = u;
                k -= 1;
            }
        if (a > bp.thresh)
            keep(p, (c << (2 * (bp.kmer - k))) & kmask);
        a -= bp.w[(int)(c >> (2 * (k - 1))) & 3];
        p += 1;
    }
}

// Chunks: chunk t of read r keeps the tuples at positions [t*BCHUNK, (t+1)*BCHUNK); a read has
// rlen / BCHUNK + 1 of them (a tracked tuple can sit at rlen).
//
// A chunk's thread starts its scan of a segment that began before c0 - 3K afresh at
// x = c0 - 3K (k = 1, nothing summed), and the tuples it keeps from c0 on are the reference's.
// With weights >= 0, the window length at any kept-or-tested position p >= x + K - 1 is
// min(K, shortest suffix ending at p that reaches norm), the same in both scans, and from a
// position both scans test they go on alike.  A scan tests a position at least every K bases
// (growing stops at length K).  Let p1 <= x + 2K - 2 be the fresh scan's first tested position
// at or after x + K - 1.  If the true scan skips p1, it is growing a window [L, .] that is below
// norm and shorter than K there; the fresh scan's window then always starts left of L (a
// shortest suffix reaching norm, or K bases), so when the true scan next tests a position
// r <= p1 + K - 1 -- its window reached norm, or K bases -- the fresh window ending at r
// contains it and is tested too.  Both scans test r <= x + 3K - 3 < c0 with the same window.
constexpr int BCHUNK = 512;

__global__ void __launch_bounds__(BT) k_bias_nchunks(DevBlock b, uint32_t* nch)
{
    const int r = blockIdx.x * BT + threadIdx.x;
    if (r < b.nreads)
        nch[r] = (uint32_t)(b.rlen[r] / BCHUNK + 1);
}

// EMIT: count[] holds the chunks' output offsets
template <typename K, bool EMIT>
__global__ void __launch_bounds__(BT) k_bias(DevBlock b, const int64_t* __restrict__ mask_anno,
                                            const int32_t* __restrict__ mask_data, BiasParams bp,
                                            const uint32_t* __restrict__ cfirst, uint32_t nchunks,
                                            uint32_t* __restrict__ count, K* __restrict__ keys,
                                            uint32_t* __restrict__ vals, int32_t* __restrict__ eread,
                                            int32_t* __restrict__ erpos, int pbits)
{
    const uint32_t i = blockIdx.x * BT + threadIdx.x;
    if (i >= nchunks)
        return;
    int lo = 0, hi = b.nreads - 1;  // the read: largest r with cfirst[r] <= i
    while (lo < hi)
    {
        const int md = (lo + hi + 1) >> 1;
        if (cfirst[md] <= i)
            lo = md;
        else
            hi = md - 1;
    }
    const int r = lo;
    const int c0 = (int)(i - cfirst[r]) * BCHUNK, c1 = c0 + BCHUNK;
    const int back = 3 * bp.kmer;
    BaseStream bs{b.bases + b.boff[r], ~(uintptr_t)0, 0};
    const int rlen = b.rlen[r];
    const uint64_t kmask = bp.kmer >= 32 ? ~0ull : (1ull << (2 * bp.kmer)) - 1;
    uint32_t n = EMIT ? count[i] : 0;
    auto keep = [&](int p, uint64_t code) {
        if (p < c0 || p >= c1)
            return;
        if constexpr (EMIT)
        {
            keys[n] = (K)code;
            if (pbits >= 0)
                vals[n] = ((uint32_t)r << pbits) | (uint32_t)p;
            else
            {
                vals[n] = n;
                eread[n] = r;
                erpos[n] = p;
            }
        }
        n += 1;
    };
    if (!mask_anno)
    {
        if (c0 < rlen)
            bias_scan(bs, max(0, c0 - back), rlen, c1, false, bp, kmask, keep);
    }
    else
    {
        const int64_t f0 = mask_anno[r], f1 = mask_anno[r + 1];
        for (int64_t j = f0; j <= f1; j += 2)
        {
            const int p = j == f0 ? 0 : mask_data[j - 1];
            if (p >= c1)
                break;
            const int q = j == f1 ? rlen : mask_data[j];
            if (p + bp.kmer <= q && q >= c0)
                bias_scan(bs, max(p, c0 - back), q, c1, true, bp, kmask, keep);
        }
    }
    if constexpr (!EMIT)
        count[i] = n;
}

int bias_chunks(const DevBlock& b, uint32_t* cfirst, uint32_t* total, void* scratch, cudaStream_t s)
{
    if (b.nreads <= 0)
        return 0;
    k_bias_nchunks<<<gd_cdiv(b.nreads, BT), BT, 0, s>>>(b, cfirst);
    GD_LAUNCHED(1);
    GD_CUDA(cudaGetLastError());
    return exclusive_scan<uint32_t>(cfirst, cfirst, b.nreads, total, scratch, s);
}

int launch_bias_count(const DevBlock& b, const int64_t* mask_anno, const int32_t* mask_data, const BiasParams& bp,
                      const uint32_t* cfirst, uint32_t nchunks, uint32_t* count, cudaStream_t s)
{
    if (nchunks == 0)
        return 0;
    k_bias<uint32_t, false><<<gd_cdiv(nchunks, (uint32_t)BT), BT, 0, s>>>(b, mask_anno, mask_data, bp, cfirst, nchunks,
                                                                          count, nullptr, nullptr, nullptr, nullptr, 0);
    GD_LAUNCHED(1);
    GD_CUDA(cudaGetLastError());
    return 0;
}

template <typename K>
int launch_bias_emit(const DevBlock& b, const int64_t* mask_anno, const int32_t* mask_data, const BiasParams& bp,
                     const uint32_t* cfirst, uint32_t nchunks, const uint32_t* offs, K* keys, uint32_t* vals,
                     int32_t* eread, int32_t* erpos, int pbits, cudaStream_t s)
{
    if (nchunks == 0)
        return 0;
    k_bias<K, true><<<gd_cdiv(nchunks, (uint32_t)BT), BT, 0, s>>>(b, mask_anno, mask_data, bp, cfirst, nchunks,
                                                                  const_cast<uint32_t*>(offs), keys, vals, eread, erpos,
                                                                  pbits);
    GD_LAUNCHED(1);
    GD_CUDA(cudaGetLastError());
    return 0;
}

__global__ void __launch_bounds__(FT) k_gather_read_pos(const uint32_t* __restrict__ idx, int64_t n,
                                                       const int32_t* __restrict__ eread,
                                                       const int32_t* __restrict__ erpos, int32_t* read, int32_t* rpos)
{
    const int64_t i = (int64_t)blockIdx.x * FT + threadIdx.x;
    if (i >= n)
        return;
    const uint32_t j = idx[i];
    read[i] = eread[j];
    rpos[i] = erpos[j];
}

int launch_gather_read_pos(const uint32_t* idx, int64_t n, const int32_t* eread, const int32_t* erpos, int32_t* read,
                           int32_t* rpos, cudaStream_t s)
{
    if (n <= 0)
        return 0;
    k_gather_read_pos<<<(unsigned)gd_cdiv<int64_t>(n, FT), FT, 0, s>>>(idx, n, eread, erpos, read, rpos);
    GD_LAUNCHED(1);
    GD_CUDA(cudaGetLastError());
    return 0;
}

template <typename K>
__global__ void __launch_bounds__(FT) k_suppress(const K* __restrict__ code, int64_t n, int t, uint32_t* keep)
{
    int64_t i = (int64_t)blockIdx.x * FT + threadIdx.x;
    if (i >= n)
        return;
    K c = code[i];
    int64_t lo = lower_code(code, n, c), hi = upper_code(code, n, c);
    keep[i] = (hi - lo) < t;
}

template <typename K>
int launch_suppress_flags(const K* code, int64_t n, int t, uint32_t* keep, cudaStream_t s)
{
    if (n <= 0)
        return 0;
    k_suppress<K><<<(unsigned)gd_cdiv<int64_t>(n, FT), FT, 0, s>>>(code, n, t, keep);
    GD_LAUNCHED(1);
    GD_CUDA(cudaGetLastError());
    return 0;
}

template <typename K>
__global__ void __launch_bounds__(FT) k_compact_index(const K* code, const int32_t* read, const int32_t* rpos,
                                                     const uint32_t* keep, const uint32_t* pos, int64_t n, K* code2,
                                                     int32_t* read2, int32_t* rpos2)
{
    int64_t i = (int64_t)blockIdx.x * FT + threadIdx.x;
    if (i >= n || !keep[i])
        return;
    uint32_t d = pos[i];
    code2[d] = code[i];
    read2[d] = read[i];
    rpos2[d] = rpos[i];
}

template <typename K>
int launch_compact_index(const K* code, const int32_t* read, const int32_t* rpos, const uint32_t* keep,
                         const uint32_t* pos, int64_t n, K* code2, int32_t* read2, int32_t* rpos2, cudaStream_t s)
{
    if (n <= 0)
        return 0;
    k_compact_index<K><<<(unsigned)gd_cdiv<int64_t>(n, FT), FT, 0, s>>>(code, read, rpos, keep, pos, n, code2, read2,
                                                                         rpos2);
    GD_LAUNCHED(1);
    GD_CUDA(cudaGetLastError());
    return 0;
}

template <typename K>
__global__ void __launch_bounds__(FT) k_run_flags(const K* __restrict__ code, int64_t n, uint32_t* flags)
{
    int64_t i = (int64_t)blockIdx.x * FT + threadIdx.x;
    if (i < n)
        flags[i] = (i == 0 || code[i] != code[i - 1]) ? 1u : 0u;
}

template <typename K>
__global__ void __launch_bounds__(FT) k_code_buckets(const K* __restrict__ code, int64_t n, int shift, uint32_t nb,
                                                    uint32_t* table)
{
    // entry i opens the buckets (prefix of entry i-1, prefix of entry i]; the last entry also
    // closes the ones after it
    const int64_t i = (int64_t)blockIdx.x * FT + threadIdx.x;
    if (i >= n)
        return;
    const uint32_t pc = code_bucket(code[i], shift, nb);
    const uint32_t p0 = i == 0 ? 0u : code_bucket(code[i - 1], shift, nb) + 1u;
    for (uint32_t p = p0; p <= pc; p++)
        table[p] = (uint32_t)i;
    if (i == n - 1)
        for (uint32_t p = pc + 1; p <= nb + 1; p++)
            table[p] = (uint32_t)n;
}

template <typename K>
int launch_code_buckets(const K* code, int64_t n, int shift, uint32_t nb, uint32_t* table, cudaStream_t s)
{
    if (n <= 0)
    {
        GD_CUDA(cudaMemsetAsync(table, 0, ((size_t)nb + 2) * 4, s));
        return 0;
    }
    k_code_buckets<K><<<(unsigned)gd_cdiv<int64_t>(n, FT), FT, 0, s>>>(code, n, shift, nb, table);
    GD_LAUNCHED(1);
    GD_CUDA(cudaGetLastError());
    return 0;
}

__global__ void __launch_bounds__(FT) k_run_starts(const uint32_t* __restrict__ flags,
                                                  const uint32_t* __restrict__ excl, int64_t n, uint32_t nruns,
                                                  uint32_t* runstart)
{
    int64_t i = (int64_t)blockIdx.x * FT + threadIdx.x;
    if (i < n && flags[i])
        runstart[excl[i]] = (uint32_t)i;
    if (i == 0)
        runstart[nruns] = (uint32_t)n;
}

int launch_run_starts(const uint32_t* flags, const uint32_t* excl, int64_t n, uint32_t nruns, uint32_t* runstart,
                      cudaStream_t s)
{
    if (n <= 0)
        return 0;
    k_run_starts<<<(unsigned)gd_cdiv<int64_t>(n, FT), FT, 0, s>>>(flags, excl, n, nruns, runstart);
    GD_LAUNCHED(1);
    GD_CUDA(cudaGetLastError());
    return 0;
}

template <typename K>
int launch_run_flags(const K* code, int64_t n, uint32_t* flags, cudaStream_t s)
{
    if (n <= 0)
        return 0;
    k_run_flags<K><<<(unsigned)gd_cdiv<int64_t>(n, FT), FT, 0, s>>>(code, n, flags);
    GD_LAUNCHED(1);
    GD_CUDA(cudaGetLastError());
    return 0;
}

// For A entry i: the B range with the same code and how many of its entries pair with i.
template <typename K>
__global__ void __launch_bounds__(FT) k_pair_count(const K* __restrict__ acode, const int32_t* __restrict__ aread,
                                                  const int32_t* __restrict__ arpos, const uint32_t* __restrict__ arun_excl,
                                                  const uint32_t* __restrict__ arun_flag, const K* __restrict__ bcode,
                                                  const int32_t* __restrict__ bread, const int32_t* __restrict__ brpos,
                                                  MergeArgs m, uint32_t* jb_out, uint64_t* cnt_out,
                                                  unsigned long long* ctrun)
{
    int64_t i = (int64_t)blockIdx.x * FT + threadIdx.x;
    bool act = i < m.na;
    uint64_t n = 0;
    uint32_t run = 0;
    if (act && m.runstart)
    {
        // B is A's own index: the run is i's own run; the entries pairing with i are the
        // run's earlier entries of smaller reads (of any earlier entry with -I, filter.c:984-998)
        run = arun_excl[i] + arun_flag[i] - 1;
        const int64_t jb = m.runstart[run];
        const int64_t e = m.identity ? i : same_read_start(aread, jb, i, 0);
        n = (uint64_t)(e - jb);
        jb_out[i] = (uint32_t)jb;
        cnt_out[i] = n;
    }
    else if (act)
    {
        // the B run of the code: a search inside the code's bucket
        K c = acode[i];
        const uint32_t bk = code_bucket(c, m.bshift, m.nbuckets);
        const int64_t lo = m.btable[bk], hi = m.btable[bk + 1];
        int64_t jb = lower_code_in(bcode, lo, hi, c);
        int64_t je = jb;
        if (jb < hi && bcode[jb] == c)
            je = upper_code_from(bcode, jb, hi, c);
        int ar = aread[i], ap = arpos[i];
        int64_t e = je;
        if (m.self)
        {
            // prefix of the B run pairing with this A entry (dalign/filter.c:984-998)
            int64_t l = jb, r = je;
            if (m.identity && m.comp)
            {
                while (l < r)
                {
                    int64_t md = (l + r) >> 1;
                    if (bread[md] <= ar)
                        l = md + 1;
                    else
                        r = md;
                }
            }
            else if (m.identity)
            {
                while (l < r)
                {
                    int64_t md = (l + r) >> 1;
                    int br = bread[md];
                    if (br < ar || (br == ar && brpos[md] < ap))
                        l = md + 1;
                    else
                        r = md;
                }
            }
            else
            {
                while (l < r)
                {
                    int64_t md = (l + r) >> 1;
                    if (bread[md] < ar)
                        l = md + 1;
                    else
                        r = md;
                }
            }
            e = l;
        }
        n = (uint64_t)(e - jb);
        jb_out[i] = (uint32_t)jb;
        cnt_out[i] = n;
        run = arun_excl[i] + arun_flag[i] - 1;
    }
    // per-run sums: the entries are sorted by code, so a run's lanes are contiguous.  When every
    // lane holds its own run (the common case) each adds its count; else a segmented sum over
    // the warp, added by each run's last lane
    const int lane = threadIdx.x & 31;
    const uint32_t rkey = act ? run : 0xffffffffu;
    const uint32_t prev = __shfl_up_sync(GD_FULL, rkey, 1);
    const unsigned heads = __ballot_sync(GD_FULL, lane == 0 || prev != rkey);
    if (heads == GD_FULL)
    {
        if (act && n)
            atomicAdd(&ctrun[run], (unsigned long long)n);
        return;
    }
    const uint32_t next = __shfl_down_sync(GD_FULL, rkey, 1);
    const int seg0 = 31 - __clz((int)(heads & (0xffffffffu >> (31 - lane))));  // this lane's run head
    unsigned long long tot = n;
    for (int o = 1; o < 32; o <<= 1)
    {
        const unsigned long long t = __shfl_up_sync(GD_FULL, tot, o);
        if (lane - o >= seg0)
            tot += t;
    }
    if (act && (lane == 31 || next != rkey) && tot)
        atomicAdd(&ctrun[run], tot);
}

template <typename K>
int launch_pair_count(const K* acode, const int32_t* aread, const int32_t* arpos, const uint32_t* arun_excl,
                      const uint32_t* arun_flag, const K* bcode, const int32_t* bread, const int32_t* brpos,
                      MergeArgs m, uint32_t* jb, uint64_t* cnt, unsigned long long* ctrun, cudaStream_t s)
{
    if (m.na <= 0)
        return 0;
    k_pair_count<K><<<(unsigned)gd_cdiv<int64_t>(m.na, FT), FT, 0, s>>>(acode, aread, arpos, arun_excl, arun_flag,
                                                                         bcode, bread, brpos, m, jb, cnt, ctrun);
    GD_LAUNCHED(1);
    GD_CUDA(cudaGetLastError());
    return 0;
}

// Histogram of per-code pair counts (< MAXGRAM): block-local shared bins, match-any
// aggregation of equal counts inside a warp, one global add per non-empty bin per block.
__global__ void __launch_bounds__(FT) k_gram(const unsigned long long* __restrict__ ctrun, int64_t nruns,
                                            unsigned long long* gram)
{
    __shared__ unsigned int h[MAXGRAM];
    for (int i = threadIdx.x; i < MAXGRAM; i += FT)
        h[i] = 0;
    __syncthreads();
    for (int64_t base = (int64_t)blockIdx.x * FT; base < nruns; base += (int64_t)gridDim.x * FT)
    {
        int64_t r = base + threadIdx.x;
        unsigned c = MAXGRAM;
        if (r < nruns)
        {
            unsigned long long x = ctrun[r];
            c = x < (unsigned long long)MAXGRAM ? (unsigned)x : MAXGRAM;
        }
        unsigned peers = __match_any_sync(GD_FULL, c);
        if (c < MAXGRAM && (peers & lanemask_lt()) == 0)
            atomicAdd(&h[c], (unsigned)__popc(peers));
    }
    __syncthreads();
    for (int i = threadIdx.x; i < MAXGRAM; i += FT)
        if (h[i])
            atomicAdd(&gram[i], (unsigned long long)h[i]);
}

int launch_gram(const unsigned long long* ctrun, int64_t nruns, unsigned long long* gram, cudaStream_t s)
{
    GD_CUDA(cudaMemsetAsync(gram, 0, sizeof(unsigned long long) * MAXGRAM, s));
    if (nruns <= 0)
        return 0;
    int dev = 0, nsm = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    int64_t want = gd_cdiv<int64_t>(nruns, FT);
    int grid = (int)(want < 4 * nsm ? want : 4 * nsm);
    k_gram<<<grid, FT, 0, s>>>(ctrun, nruns, gram);
    GD_LAUNCHED(1);
    GD_CUDA(cudaGetLastError());
    return 0;
}

__global__ void __launch_bounds__(FT) k_cnt_mask(const uint32_t* arun_excl, const uint32_t* arun_flag,
                                                const unsigned long long* ctrun, int64_t na, int limit, int always,
                                                uint64_t* cnt)
{
    int64_t i = (int64_t)blockIdx.x * FT + threadIdx.x;
    if (i >= na)
        return;
    uint32_t run = arun_excl[i] + arun_flag[i] - 1;
    if (!always && ctrun[run] >= (unsigned long long)limit)
        cnt[i] = 0;
}

int launch_cnt_mask(const uint32_t* arun_excl, const uint32_t* arun_flag, const unsigned long long* ctrun, int64_t na,
                    int limit, int always, uint64_t* cnt, cudaStream_t s)
{
    if (na <= 0)
        return 0;
    k_cnt_mask<<<(unsigned)gd_cdiv<int64_t>(na, FT), FT, 0, s>>>(arun_excl, arun_flag, ctrun, na, limit, always, cnt);
    GD_LAUNCHED(1);
    GD_CUDA(cudaGetLastError());
    return 0;
}

__global__ void __launch_bounds__(FT) k_emit(const int32_t* __restrict__ aread, const int32_t* __restrict__ arpos,
                                            const int32_t* __restrict__ bread, const int32_t* __restrict__ brpos,
                                            const uint32_t* __restrict__ jb, const uint64_t* __restrict__ cnt,
                                            const uint64_t* __restrict__ hoff, int64_t na, HitBits hb,
                                            uint64_t* hkey, uint32_t* hdiag)
{
    int64_t i = (int64_t)blockIdx.x * FT + threadIdx.x;
    if (i >= na)
        return;
    uint64_t n = cnt[i];
    if (!n)
        return;
    uint64_t o = hoff[i];
    int ar = aread[i], ap = arpos[i];
    uint64_t akey = ((uint64_t)ar << hb.pbits) | (uint64_t)ap;
    int sh = hb.pbits + hb.abits;
    uint32_t b0 = jb[i];
    if (hb.qbits > 0)
        for (uint64_t j = 0; j < n; j++)
        {
            uint32_t b = b0 + (uint32_t)j;
            hkey[o + j] = ((((uint64_t)bread[b] << sh) | akey) << hb.qbits) | (uint64_t)(uint32_t)brpos[b];
        }
    else
        for (uint64_t j = 0; j < n; j++)
        {
            uint32_t b = b0 + (uint32_t)j;
            hkey[o + j] = ((uint64_t)bread[b] << sh) | akey;
            hdiag[o + j] = (uint32_t)(ap - brpos[b]);
        }
}

__global__ void __launch_bounds__(FT) k_hit_unpack(const uint64_t* __restrict__ packed, int64_t n, HitBits hb,
                                                  uint64_t* __restrict__ hkey, uint32_t* __restrict__ hdiag)
{
    const int64_t i = (int64_t)blockIdx.x * FT + threadIdx.x;
    if (i >= n)
        return;
    const uint64_t v = packed[i];
    const uint64_t k = v >> hb.qbits;
    const int bpos = (int)(v & ((1ull << hb.qbits) - 1));
    const int apos = (int)(k & ((1ull << hb.pbits) - 1));
    hkey[i] = k;
    hdiag[i] = (uint32_t)(apos - bpos);
}

int launch_hit_unpack(const uint64_t* packed, int64_t n, HitBits hb, uint64_t* hkey, uint32_t* hdiag, cudaStream_t s)
{
    if (n <= 0)
        return 0;
    k_hit_unpack<<<(unsigned)gd_cdiv<int64_t>(n, FT), FT, 0, s>>>(packed, n, hb, hkey, hdiag);
    GD_LAUNCHED(1);
    GD_CUDA(cudaGetLastError());
    return 0;
}

int launch_emit(const int32_t* aread, const int32_t* arpos, const int32_t* bread, const int32_t* brpos,
                const uint32_t* jb, const uint64_t* cnt, const uint64_t* hoff, int64_t na, HitBits hb,
                uint64_t* hkey, uint32_t* hdiag, cudaStream_t s)
{
    if (na <= 0)
        return 0;
    k_emit<<<(unsigned)gd_cdiv<int64_t>(na, FT), FT, 0, s>>>(aread, arpos, bread, brpos, jb, cnt, hoff, na, hb, hkey,
                                                             hdiag);
    GD_LAUNCHED(1);
    GD_CUDA(cudaGetLastError());
    return 0;
}

__global__ void __launch_bounds__(FT) k_pair_flags(const uint64_t* __restrict__ hkey, int64_t n, int pbits,
                                                  uint32_t* flags)
{
    int64_t i = (int64_t)blockIdx.x * FT + threadIdx.x;
    if (i < n)
        flags[i] = (i == 0 || (hkey[i] >> pbits) != (hkey[i - 1] >> pbits)) ? 1u : 0u;
}

int launch_pair_flags(const uint64_t* hkey, int64_t n, int pbits, uint32_t* flags, cudaStream_t s)
{
    if (n <= 0)
        return 0;
    k_pair_flags<<<(unsigned)gd_cdiv<int64_t>(n, FT), FT, 0, s>>>(hkey, n, pbits, flags);
    GD_LAUNCHED(1);
    GD_CUDA(cudaGetLastError());
    return 0;
}

__global__ void __launch_bounds__(FT) k_pair_scatter(const uint32_t* flags, const uint32_t* pos, int64_t n,
                                                    uint32_t* starts)
{
    int64_t i = (int64_t)blockIdx.x * FT + threadIdx.x;
    if (i < n && flags[i])
        starts[pos[i]] = (uint32_t)i;
}

int launch_pair_scatter(const uint32_t* flags, const uint32_t* pos, int64_t n, uint32_t* starts, cudaStream_t s)
{
    if (n <= 0)
        return 0;
    k_pair_scatter<<<(unsigned)gd_cdiv<int64_t>(n, FT), FT, 0, s>>>(flags, pos, n, starts);
    GD_LAUNCHED(1);
    GD_CUDA(cudaGetLastError());
    return 0;
}

__global__ void __launch_bounds__(FT) k_select_groups(const uint32_t* __restrict__ starts, int64_t nstarts,
                                                     int64_t nhits, int minhit, const uint64_t* __restrict__ hkey,
                                                     const uint32_t* __restrict__ hdiag, int binshift, int kmer,
                                                     int hitmin, HitBits hb, const int32_t* __restrict__ arlen,
                                                     const int32_t* __restrict__ brlen, uint2* groups, uint32_t* cost,
                                                     uint32_t* idx, unsigned int* ngroups)
{
    int64_t g = (int64_t)blockIdx.x * FT + threadIdx.x;
    bool take = false;
    uint32_t s = 0, e = 0, c = 0;
    if (g < nstarts)
    {
        s = starts[g];
        e = (g + 1 < nstarts) ? starts[g + 1] : (uint32_t)nhits;
        take = (int64_t)(e - s) >= minhit && group_can_fire(hkey, hdiag, s, e, hb.pbits, binshift, kmer, hitmin, minhit);
        if (take)
        {
            uint64_t k = hkey[s];
            int ar = (int)((k >> hb.pbits) & ((1ull << hb.abits) - 1));
            int br = (int)(k >> (hb.pbits + hb.abits));
            c = (uint32_t)(arlen[ar] + brlen[br]);
        }
    }
    // slots for the block's kept groups: one atomic per block (a per-warp atomic on the one
    // counter serialised millions of times on the large block pairs)
    __shared__ unsigned wn[FT / 32];
    __shared__ unsigned bbase;
    const unsigned m = __ballot_sync(GD_FULL, take);
    const int w = threadIdx.x >> 5;
    if (lane_id() == 0)
        wn[w] = __popc(m);
    __syncthreads();
    if (threadIdx.x == 0)
    {
        unsigned tot = 0;
        for (int i = 0; i < FT / 32; i++)
            tot += wn[i];
        bbase = tot ? atomicAdd(ngroups, tot) : 0u;
    }
    __syncthreads();
    if (take)
    {
        unsigned slot = bbase + __popc(m & lanemask_lt());
        for (int i = 0; i < w; i++)
            slot += wn[i];
        groups[slot] = make_uint2(s, e);
        cost[slot] = ~c;  // ascending sort of ~cost = longest pairs first
        idx[slot] = slot;
    }
}

int launch_select_groups(const uint32_t* starts, int64_t nstarts, int64_t nhits, int minhit, const uint64_t* hkey,
                         const uint32_t* hdiag, int binshift, int kmer, int hitmin, HitBits hb, const int32_t* arlen,
                         const int32_t* brlen, uint2* groups, uint32_t* cost, uint32_t* idx, unsigned int* ngroups,
                         cudaStream_t s)
{
    GD_CUDA(cudaMemsetAsync(ngroups, 0, sizeof(unsigned), s));
    if (nstarts <= 0)
        return 0;
    k_select_groups<<<(unsigned)gd_cdiv<int64_t>(nstarts, FT), FT, 0, s>>>(
        starts, nstarts, nhits, minhit, hkey, hdiag, binshift, kmer, hitmin, hb, arlen, brlen, groups, cost, idx, ngroups);
    GD_LAUNCHED(1);
    GD_CUDA(cudaGetLastError());
    return 0;
}

__global__ void __launch_bounds__(FT) k_pack2(const uint8_t* __restrict__ buf, int64_t nbytes, uint32_t* pk,
                                             int64_t nwords)
{
    const int64_t i = (int64_t)blockIdx.x * FT + threadIdx.x;
    if (i >= nwords)
        return;
    const int64_t o = 16 * i;
    uint32_t w = 0;
    if (o + 16 <= nbytes)
    {
        const uint4 v = *reinterpret_cast<const uint4*>(buf + o);
        const uint32_t q[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
        for (int j = 0; j < 4; j++)
#pragma unroll
            for (int t = 0; t < 4; t++)
                w |= ((q[j] >> (8 * t)) & 3u) << (2 * (4 * j + t));
    }
    else
        for (int j = 0; j < 16 && o + j < nbytes; j++)
            w |= (uint32_t)(buf[o + j] & 3) << (2 * j);
    pk[i] = w;
}

int launch_pack2(const uint8_t* buf, int64_t nbytes, uint32_t* pk, int64_t nwords, cudaStream_t s)
{
    if (nwords <= 0)
        return 0;
    k_pack2<<<(unsigned)gd_cdiv<int64_t>(nwords, FT), FT, 0, s>>>(buf, nbytes, pk, nwords);
    GD_LAUNCHED(1);
    GD_CUDA(cudaGetLastError());
    return 0;
}

__global__ void __launch_bounds__(FT) k_complement(DevBlock b, uint8_t* dst)
{
    int r = blockIdx.x;
    int len = b.rlen[r];
    const uint8_t* s = b.bases + b.boff[r];
    uint8_t* d = dst + b.boff[r];
    for (int p = threadIdx.x; p < len; p += FT)
        d[p] = (uint8_t)(3 - s[len - 1 - p]);
}

__global__ void __launch_bounds__(FT) k_complement_mask(DevBlock b, const int64_t* anno, const int32_t* src,
                                                       int32_t* dst)
{
    int r = blockIdx.x * FT + threadIdx.x;
    if (r >= b.nreads)
        return;
    int64_t a0 = anno[r], a1 = anno[r + 1];
    int len = b.rlen[r];
    int64_t npair = (a1 - a0) / 2;
    for (int64_t j = 0; j < npair; j++)
    {
        int64_t q = a0 + 2 * (npair - 1 - j);
        dst[a0 + 2 * j] = len - src[q + 1];
        dst[a0 + 2 * j + 1] = len - src[q];
    }
}

int launch_complement(const DevBlock& src, uint8_t* dst_bases, const int64_t* anno, const int32_t* mdata,
                      int32_t* mdata_dst, cudaStream_t s)
{
    if (src.nreads <= 0)
        return 0;
    k_complement<<<src.nreads, FT, 0, s>>>(src, dst_bases);
    GD_LAUNCHED(1);
    if (anno)
    {
        k_complement_mask<<<(unsigned)gd_cdiv(src.nreads, FT), FT, 0, s>>>(src, anno, mdata, mdata_dst);
        GD_LAUNCHED(1);
    }
    GD_CUDA(cudaGetLastError());
    return 0;
}

#define INST(K)                                                                                                  \
    template int launch_extract<K>(const DevBlock&, const int64_t*, const int32_t*, int, K*, uint32_t*, int64_t, \
                                   uint32_t*, int, cudaStream_t);                                                \
    template int launch_unpack<K>(const K*, const uint32_t*, int64_t, int, int, K*, int32_t*, int32_t*,          \
                                  cudaStream_t);                                                                 \
    template int launch_decode<K>(const DevBlock&, int, const uint32_t*, int64_t, int32_t*, int32_t*,            \
                                  cudaStream_t);                                                                 \
    template int launch_bias_emit<K>(const DevBlock&, const int64_t*, const int32_t*, const BiasParams&,         \
                                     const uint32_t*, uint32_t, const uint32_t*, K*, uint32_t*, int32_t*,        \
                                     int32_t*, int, cudaStream_t);                                               \
    template int launch_suppress_flags<K>(const K*, int64_t, int, uint32_t*, cudaStream_t);                      \
    template int launch_compact_index<K>(const K*, const int32_t*, const int32_t*, const uint32_t*,              \
                                         const uint32_t*, int64_t, K*, int32_t*, int32_t*, cudaStream_t);        \
    template int launch_run_flags<K>(const K*, int64_t, uint32_t*, cudaStream_t);                                \
    template int launch_code_buckets<K>(const K*, int64_t, int, uint32_t, uint32_t*, cudaStream_t);              \
    template int launch_pair_count<K>(const K*, const int32_t*, const int32_t*, const uint32_t*, const uint32_t*, \
                                      const K*, const int32_t*, const int32_t*, MergeArgs, uint32_t*, uint64_t*, \
                                      unsigned long long*, cudaStream_t);
INST(uint32_t)
INST(uint64_t)
#undef INST

}  // namespace gd
