// gd_filter2.cu -- daligner2's modimizer filter (dalign2/filter.c) on sm_100a.
//
// Index build: one thread per k-mer slot evaluates the slot's two candidate codes from the
// bases alone (no per-read serial state), a scan of the per-slot counts places them in the
// reference's list order (read, position, canonical before half-shifted), and the shared LSD
// radix sort orders them by code.  Join: one thread per A entry finds its B range by binary
// search, splits it by orientation with a prefix count of strands, and writes its hits of
// each orientation into that orientation's own list in the reference's generation order.
#include "gd_filter2.cuh"

namespace gd
{

constexpr int F2T = 256;
constexpr unsigned D2_MODULUS = 101;  // MODULUS / MODTHR (dalign2/filter.c:47-48)
constexpr unsigned D2_MODTHR = 28;

D2Masks d2_masks(int kmer)
{
    D2Masks m;
    m.kshift = kmer >= 32 ? 64 : 2 * kmer;
    m.kmask = kmer >= 32 ? ~0ull : ((1ull << m.kshift) - 1);
    m.lf = (1ull << (m.kshift / 2)) - 1;
    m.hf = m.kmask - m.lf;
    m.lr = (1ull << ((m.kshift + 1) / 2)) - 1;
    m.hr = m.kmask - m.lr;
    return m;
}

__device__ __forceinline__ bool d2_keep(uint64_t code, int kshift)
{
    if (kshift <= 32)
        return (uint32_t)code % D2_MODULUS < D2_MODTHR;
    return code % D2_MODULUS < D2_MODTHR;
}

// The slot's two candidates (tuple_thread's loop body, dalign2/filter.c:485-565).  For the
// k-mer ending at p of the unmasked segment starting at ps: c / u are the forward /
// reverse-complement codes of bases [p-k+1, p]; the codes one step earlier cover bases
// [max(ps, p-k), p-1] (k-1 bases at the segment's first k-mer, where the reference's
// warm-up leaves them).  d = high half of the earlier c | low half of c, v likewise from u.
// A thread takes four consecutive slots: within one read and segment the codes roll base by
// base (the earlier codes are the previous slot's), otherwise they are built from the bases.
struct D2Codes
{
    uint64_t code1, code2;
    unsigned strand1, strand2;
    bool keep1, keep2;
};

// the unmasked segment [ps, q) holding the k-mer [p0, p], or false (tuple_thread :436-460)
__device__ __forceinline__ bool d2_segment(const DevBlock& b, const int64_t* __restrict__ manno,
                                           const int32_t* __restrict__ mdata, int r, int p0, int p, int& ps)
{
    ps = 0;
    if (!manno)
        return true;
    const int64_t f0 = manno[r], f1 = manno[r + 1];
    int q = b.rlen[r];
    for (int64_t a = f0; a < f1; a += 2)
    {
        const int ib = mdata[a], ie = mdata[a + 1];
        if (p0 < ib)
        {
            q = ib;
            break;
        }
        ps = ie;
        q = b.rlen[r];
    }
    return p0 >= ps && p < q;
}

__device__ __forceinline__ void d2_pick(uint64_t c, uint64_t u, uint64_t cp, uint64_t up, const D2Masks& M,
                                        D2Codes& o)
{
    const uint64_t d = (cp & M.hf) | (c & M.lf);
    const uint64_t v = (up & M.lr) | (u & M.hr);
    o.code1 = u < c ? u : c;
    o.strand1 = u < c;
    o.code2 = v < d ? v : d;
    o.strand2 = v < d;
    o.keep1 = d2_keep(o.code1, M.kshift);
    o.keep2 = d2_keep(o.code2, M.kshift);
}

// EMIT = false: count[s] = codes the slot lists; EMIT = true: the slot's entries at off[s]
template <bool EMIT, typename K>
__global__ void __launch_bounds__(F2T) k_d2_slots(DevBlock b, const int64_t* __restrict__ manno,
                                                 const int32_t* __restrict__ mdata, int kmer, D2Masks M,
                                                 int64_t nslots, uint32_t* count, const uint32_t* __restrict__ off,
                                                 K* keys, uint32_t* vals, int32_t* rd, int32_t* rp)
{
    const int64_t s0 = ((int64_t)blockIdx.x * F2T + threadIdx.x) * 4;
    if (s0 >= nslots)
        return;
    const int nj = (int)min((int64_t)4, nslots - s0);
    const int top = M.kshift - 2;
    int r = read_of_slot(b, s0, kmer);
    int64_t kst = kstart_of(b, r, kmer), knext = kstart_of(b, r + 1, kmer);
    uint64_t c = 0, u = 0;
    int have = -2, seg = -1;  // position whose codes are in (c, u), and its segment start
    unsigned cnt[4] = {0, 0, 0, 0};
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
        const int p0 = (int)(s - kst), p = p0 + kmer - 1;
        int ps;
        if (!d2_segment(b, manno, mdata, r, p0, p, ps))
        {
            have = -2;
            continue;
        }
        const uint8_t* src = b.bases + b.boff[r];
        uint64_t cp, up;
        if (have == p - 1 && seg == ps)
        {
            const uint64_t x = src[p];
            cp = c;
            up = u;
            c = ((c << 2) | x) & M.kmask;
            u = (u >> 2) | ((3ull - x) << top);
        }
        else
        {
            cp = up = c = u = 0;
            for (int t = max(ps, p - kmer); t < p; t++)
            {
                const uint64_t x = src[t];
                cp = (cp << 2) | x;
                up = (up >> 2) | ((3ull - x) << top);
            }
            for (int t = p - kmer + 1; t <= p; t++)
            {
                const uint64_t x = src[t];
                c = (c << 2) | x;
                u = (u >> 2) | ((3ull - x) << top);
            }
            c &= M.kmask;
            cp &= M.kmask;
        }
        have = p;
        seg = ps;
        D2Codes o;
        d2_pick(c, u, cp, up, M, o);
        if (!EMIT)
            cnt[j] = (unsigned)o.keep1 + (unsigned)o.keep2;
        else
        {
            uint32_t e = off[s];
            if (o.keep1)
            {
                keys[e] = (K)o.code1;
                vals[e] = e;
                rd[e] = (r << 1) | (int)o.strand1;
                rp[e] = p;
                e++;
            }
            if (o.keep2)
            {
                keys[e] = (K)o.code2;
                vals[e] = e;
                rd[e] = (r << 1) | (int)o.strand2;
                rp[e] = p;
            }
        }
    }
    if (!EMIT)
    {
        if (nj == 4)
            *reinterpret_cast<uint4*>(count + s0) = make_uint4(cnt[0], cnt[1], cnt[2], cnt[3]);
        else
            for (int j = 0; j < nj; j++)
                count[s0 + j] = cnt[j];
    }
}

int launch_d2_count(const DevBlock& b, const int64_t* mask_anno, const int32_t* mask_data, int kmer,
                    const D2Masks& m, int64_t nslots, uint32_t* count, cudaStream_t s)
{
    if (nslots <= 0)
        return 0;
    const int64_t threads = (nslots + 3) / 4;
    k_d2_slots<false, uint32_t><<<(unsigned)gd_cdiv<int64_t>(threads, F2T), F2T, 0, s>>>(
        b, mask_anno, mask_data, kmer, m, nslots, count, nullptr, nullptr, nullptr, nullptr, nullptr);
    GD_LAUNCHED(1);
    GD_CUDA(cudaGetLastError());
    return 0;
}

template <typename K>
int launch_d2_emit(const DevBlock& b, const int64_t* mask_anno, const int32_t* mask_data, int kmer,
                   const D2Masks& m, int64_t nslots, const uint32_t* off, K* keys, uint32_t* vals, int32_t* rd,
                   int32_t* rp, cudaStream_t s)
{
    if (nslots <= 0)
        return 0;
    const int64_t threads = (nslots + 3) / 4;
    k_d2_slots<true, K><<<(unsigned)gd_cdiv<int64_t>(threads, F2T), F2T, 0, s>>>(
        b, mask_anno, mask_data, kmer, m, nslots, nullptr, off, keys, vals, rd, rp);
    GD_LAUNCHED(1);
    GD_CUDA(cudaGetLastError());
    return 0;
}

template <typename K>
__global__ void __launch_bounds__(F2T) k_d2_gather(const K* __restrict__ skeys, const uint32_t* __restrict__ svals,
                                                  int64_t n, const int32_t* __restrict__ rd,
                                                  const int32_t* __restrict__ rp, K* code, int32_t* read,
                                                  int32_t* rpos)
{
    const int64_t i = (int64_t)blockIdx.x * F2T + threadIdx.x;
    if (i >= n)
        return;
    const uint32_t e = svals[i];
    code[i] = skeys[i];
    read[i] = rd[e];
    rpos[i] = rp[e];
}

template <typename K>
int launch_d2_gather(const K* skeys, const uint32_t* svals, int64_t n, const int32_t* rd, const int32_t* rp, K* code,
                     int32_t* read, int32_t* rpos, cudaStream_t s)
{
    if (n <= 0)
        return 0;
    k_d2_gather<K><<<(unsigned)gd_cdiv<int64_t>(n, F2T), F2T, 0, s>>>(skeys, svals, n, rd, rp, code, read, rpos);
    GD_LAUNCHED(1);
    GD_CUDA(cudaGetLastError());
    return 0;
}

__global__ void __launch_bounds__(F2T) k_d2_strand_flags(const int32_t* __restrict__ read, int64_t n,
                                                        uint32_t* flags)
{
    const int64_t i = (int64_t)blockIdx.x * F2T + threadIdx.x;
    if (i < n)
        flags[i] = (uint32_t)read[i] & 1u;
}

int launch_d2_strand_flags(const int32_t* read, int64_t n, uint32_t* flags, cudaStream_t s)
{
    if (n <= 0)
        return 0;
    k_d2_strand_flags<<<(unsigned)gd_cdiv<int64_t>(n, F2T), F2T, 0, s>>>(read, n, flags);
    GD_LAUNCHED(1);
    GD_CUDA(cudaGetLastError());
    return 0;
}

// count_thread (dalign2/filter.c:1136-1256), per A entry.  Within a block (self) the entry
// pairs with the earlier entries of its code run whose read is smaller (all earlier entries
// with -I); across blocks with the whole B run of its code.  bstrand_excl[j] = number of
// complement-strand entries among B[0, j).
template <typename K>
__global__ void __launch_bounds__(F2T) k_d2_pair_count(const K* __restrict__ acode, const int32_t* __restrict__ aread,
                                                      const uint32_t* __restrict__ arun_excl,
                                                      const uint32_t* __restrict__ arun_flag,
                                                      const uint32_t* __restrict__ runstart,
                                                      const uint32_t* __restrict__ btable, int bshift,
                                                      uint32_t nbuckets,
                                                      const K* __restrict__ bcode, const int32_t* __restrict__ bread,
                                                      const uint32_t* __restrict__ bstrand_excl, int64_t na,
                                                      int64_t nb, int self, int identity, uint32_t* jb_out,
                                                      uint64_t* cnt_f, uint64_t* cnt_c, unsigned long long* ctrun)
{
    const int64_t i = (int64_t)blockIdx.x * F2T + threadIdx.x;
    const bool act = i < na;
    uint64_t n = 0;
    uint32_t run = 0;
    if (act)
    {
        const int ar = aread[i];
        int64_t jb, e;
        if (runstart)
        {
            // B is A's own index: i's own run; the earlier entries of smaller reads (any
            // earlier entry with -I), found by galloping back over i's read
            jb = runstart[arun_excl[i] + arun_flag[i] - 1];
            e = identity ? i : same_read_start(aread, jb, i, 1);
        }
        else
        {
            const K c = acode[i];
            const uint32_t bk = code_bucket(c, bshift, nbuckets);
            const int64_t lo = btable[bk], hi = btable[bk + 1];
            jb = lower_code_in(bcode, lo, hi, c);
            int64_t je = jb;
            if (jb < hi && bcode[jb] == c)
                je = upper_code_from(bcode, jb, hi, c);
            e = je;
            if (self)
            {
                if (identity)
                    e = i;  // every earlier entry of the run (A and B are the same index)
                else
                {
                    int64_t l = jb, r = je;
                    while (l < r)
                    {
                        const int64_t md = (l + r) >> 1;
                        if ((bread[md] >> 1) < (ar >> 1))
                            l = md + 1;
                        else
                            r = md;
                    }
                    e = l;
                }
            }
        }
        n = (uint64_t)(e - jb);
        const uint64_t ncomp_strand = bstrand_excl[e] - bstrand_excl[jb];
        const uint64_t fwd = (ar & 1) ? ncomp_strand : n - ncomp_strand;
        jb_out[i] = (uint32_t)jb;
        cnt_f[i] = fwd;
        cnt_c[i] = n - fwd;
        run = arun_excl[i] + arun_flag[i] - 1;
    }
    // per-run sums over contiguous runs: each lane alone when every lane holds its own run,
    // else a segmented shuffle sum added by each run's last lane
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
    const int seg0 = 31 - __clz((int)(heads & (0xffffffffu >> (31 - lane))));
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
int launch_d2_pair_count(const K* acode, const int32_t* aread, const uint32_t* arun_excl, const uint32_t* arun_flag,
                         const uint32_t* runstart, const uint32_t* btable, int bshift, uint32_t nbuckets,
                         const K* bcode, const int32_t* bread, const uint32_t* bstrand_excl, int64_t na, int64_t nb,
                         int self, int identity, uint32_t* jb, uint64_t* cnt_f, uint64_t* cnt_c,
                         unsigned long long* ctrun, cudaStream_t s)
{
    if (na <= 0)
        return 0;
    k_d2_pair_count<K><<<(unsigned)gd_cdiv<int64_t>(na, F2T), F2T, 0, s>>>(
        acode, aread, arun_excl, arun_flag, runstart, btable, bshift, nbuckets, bcode, bread, bstrand_excl, na, nb,
        self, identity, jb, cnt_f, cnt_c, ctrun);
    GD_LAUNCHED(1);
    GD_CUDA(cudaGetLastError());
    return 0;
}

// merge_thread's emission (dalign2/filter.c:1358-1463) for one A entry: its B entries in
// index order, each to the list of its orientation; a complement hit's B position is
// reflected into the complemented read (rlen - bpos + k - 2).
__global__ void __launch_bounds__(F2T) k_d2_emit_hits(const int32_t* __restrict__ aread,
                                                     const int32_t* __restrict__ arpos,
                                                     const int32_t* __restrict__ bread,
                                                     const int32_t* __restrict__ brpos,
                                                     const int32_t* __restrict__ brlen,
                                                     const uint32_t* __restrict__ jb,
                                                     const uint64_t* __restrict__ cnt_f,
                                                     const uint64_t* __restrict__ cnt_c,
                                                     const uint64_t* __restrict__ foff,
                                                     const uint64_t* __restrict__ coff, int64_t na, int koff,
                                                     HitBits hb, uint64_t* fkey, uint32_t* fdiag, uint64_t* ckey,
                                                     uint32_t* cdiag)
{
    const int64_t i = (int64_t)blockIdx.x * F2T + threadIdx.x;
    if (i >= na)
        return;
    const uint64_t n = cnt_f[i] + cnt_c[i];
    if (!n)
        return;
    uint64_t of = foff[i], oc = coff[i];
    const int ar = aread[i] >> 1, as = aread[i] & 1, ap = arpos[i];
    const uint64_t akey = ((uint64_t)ar << hb.pbits) | (uint64_t)ap;
    const int sh = hb.pbits + hb.abits;
    const uint32_t b0 = jb[i];
    for (uint64_t j = 0; j < n; j++)
    {
        const uint32_t q = b0 + (uint32_t)j;
        const int br = bread[q] >> 1, bs = bread[q] & 1;
        const uint64_t key = ((uint64_t)br << sh) | akey;
        const int bp = (bs == as) ? brpos[q] : (brlen[br] - brpos[q]) + koff;
        uint64_t* dk = (bs == as) ? fkey + of : ckey + oc;
        if (hb.qbits > 0)
            *dk = (key << hb.qbits) | (uint64_t)(uint32_t)bp;
        else
        {
            *dk = key;
            ((bs == as) ? fdiag + of : cdiag + oc)[0] = (uint32_t)(ap - bp);
        }
        if (bs == as)
            of++;
        else
            oc++;
    }
}

int launch_d2_emit_hits(const int32_t* aread, const int32_t* arpos, const int32_t* bread, const int32_t* brpos,
                        const int32_t* brlen, const uint32_t* jb, const uint64_t* cnt_f, const uint64_t* cnt_c,
                        const uint64_t* foff, const uint64_t* coff, int64_t na, int kmer, HitBits hb, uint64_t* fkey,
                        uint32_t* fdiag, uint64_t* ckey, uint32_t* cdiag, cudaStream_t s)
{
    if (na <= 0)
        return 0;
    k_d2_emit_hits<<<(unsigned)gd_cdiv<int64_t>(na, F2T), F2T, 0, s>>>(aread, arpos, bread, brpos, brlen, jb, cnt_f,
                                                                       cnt_c, foff, coff, na, kmer - 2, hb, fkey,
                                                                       fdiag, ckey, cdiag);
    GD_LAUNCHED(1);
    GD_CUDA(cudaGetLastError());
    return 0;
}

#define INST2(K)                                                                                                 \
    template int launch_d2_emit<K>(const DevBlock&, const int64_t*, const int32_t*, int, const D2Masks&, int64_t, \
                                   const uint32_t*, K*, uint32_t*, int32_t*, int32_t*, cudaStream_t);            \
    template int launch_d2_gather<K>(const K*, const uint32_t*, int64_t, const int32_t*, const int32_t*, K*,     \
                                     int32_t*, int32_t*, cudaStream_t);                                          \
    template int launch_d2_pair_count<K>(const K*, const int32_t*, const uint32_t*, const uint32_t*,             \
                                         const uint32_t*, const uint32_t*, int, uint32_t, const K*,              \
                                         const int32_t*,                                                         \
                                         const uint32_t*, int64_t, int64_t, int, int, uint32_t*, uint64_t*,      \
                                         uint64_t*, unsigned long long*, cudaStream_t);
INST2(uint32_t)
INST2(uint64_t)
#undef INST2

}  // namespace gd
