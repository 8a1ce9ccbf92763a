// gd_filter.cuh -- device kernels of the k-mer filter (dalign/filter.c restated for sm_100a).
#pragma once
#include <climits>
#include "gd_common.cuh"

namespace gd
{

constexpr int MAXGRAM = 10000;  // cap on per-code pair counts (dalign/filter.c:20)

// k-mer slots: read r owns slots [kstart[r], kstart[r+1]) with kstart[r] = boff[r] - K*r,
// slot s of read r ends at rpos = s - kstart[r] + K - 1 (the tuple_thread layout,
// dalign/filter.c:410-425).
// keys (code, or all ones where masked) and values (slot index, or with pbits >= 0 the
// packed read << pbits | first position) of every slot
template <typename K>
int launch_extract(const DevBlock& b, const int64_t* mask_anno, const int32_t* mask_data, int kmer, K* keys,
                   uint32_t* vals, int64_t nslots, uint32_t* nmasked, int pbits, cudaStream_t s);

// the index arrays from sorted keys and packed values
template <typename K>
int launch_unpack(const K* skeys, const uint32_t* svals, int64_t n, int pbits, int kmer, K* code, int32_t* read,
                  int32_t* rpos, cudaStream_t s);

template <typename K>
int launch_decode(const DevBlock& b, int kmer, const uint32_t* slots, int64_t n, int32_t* read, int32_t* rpos,
                  cudaStream_t s);

// daligner -b (biased_tuple_thread, dalign/filter.c:492-633, tables :718-733): per read, a
// window of k <= K bases whose information (sum of w[base]) is grown to reach norm, trimmed
// from the left while it stays at norm, kept when above thresh, then slid one base.
struct BiasParams
{
    int w[4];    // ceil(-10000 log4 freq[base]), all >= 0
    int norm;    // 10000 K
    int thresh;  // 10000 (K - MAX_BIAS), MAX_BIAS = 2
    int kmer;
};

// The scan works in chunks of positions (one thread each): cfirst[r] = the read's first chunk
// (exclusive scan over the reads; *total = the number of chunks).
int bias_chunks(const DevBlock& b, uint32_t* cfirst, uint32_t* total, void* scratch, cudaStream_t s);

// Tuples each chunk keeps (count[chunk]).
int launch_bias_count(const DevBlock& b, const int64_t* mask_anno, const int32_t* mask_data, const BiasParams& bp,
                      const uint32_t* cfirst, uint32_t nchunks, uint32_t* count, cudaStream_t s);

// The kept tuples at offs[chunk] (exclusive offsets), in (read, position) order: keys = K-mer
// codes (the window's k bases at the top), vals = read << pbits | position with pbits >= 0,
// else the entry index with (read, position) in eread/erpos.
template <typename K>
int launch_bias_emit(const DevBlock& b, const int64_t* mask_anno, const int32_t* mask_data, const BiasParams& bp,
                     const uint32_t* cfirst, uint32_t nchunks, const uint32_t* offs, K* keys, uint32_t* vals,
                     int32_t* eread, int32_t* erpos, int pbits, cudaStream_t s);

// read[i] = eread[idx[i]], rpos[i] = erpos[idx[i]]
int launch_gather_read_pos(const uint32_t* idx, int64_t n, const int32_t* eread, const int32_t* erpos, int32_t* read,
                           int32_t* rpos, cudaStream_t s);

// Keep flags for -t suppression: 1 where the entry's code run is shorter than t.
template <typename K>
int launch_suppress_flags(const K* code, int64_t n, int t, uint32_t* keep, cudaStream_t s);

template <typename K>
int launch_compact_index(const K* code, const int32_t* read, const int32_t* rpos, const uint32_t* keep,
                         const uint32_t* pos, int64_t n, K* code2, int32_t* read2, int32_t* rpos2, cudaStream_t s);

// Merge-join of the A and B indices (count_thread / merge_thread, dalign/filter.c:948-1231).
struct MergeArgs
{
    int64_t na, nb;
    int self, identity, comp;
    // non-null when B is A's own index (a block against itself, forward): the start of every
    // code run of A (nruns + 1 entries, the last = na), so no searches are needed
    const uint32_t* runstart;
    // otherwise: btable[p] = the first B entry whose code >> bshift is >= p (code_buckets)
    const uint32_t* btable;
    int bshift;
    uint32_t nbuckets;
};

// Bucket table of a sorted code array: with bucket(code) = min(code >> shift, nb), table[p] =
// the first index whose bucket is >= p, for p in [0, nb + 1]: a code's run lies in
// [table[b], table[b + 1]).  Bucket nb holds codes beyond 4^k (the all-ones code of a masked
// slot that the 4-byte sort for k = 16 can leave inside the index).  bucket_shift: the shift
// that gives at most 2^20 buckets for k-mers of length kmer.
inline int bucket_shift(int kmer)
{
    return 2 * kmer > 20 ? 2 * kmer - 20 : 0;
}
inline uint32_t bucket_count(int kmer)
{
    return 1u << (2 * kmer - bucket_shift(kmer));
}
template <typename K>
int launch_code_buckets(const K* code, int64_t n, int shift, uint32_t nb, uint32_t* table, cudaStream_t s);

template <typename K>
__device__ __forceinline__ uint32_t code_bucket(K code, int shift, uint32_t nb)
{
    const K b = code >> shift;
    return b < (K)nb ? (uint32_t)b : nb;
}

// runstart[excl[i]] = i for every run head i, runstart[nruns] = n
int launch_run_starts(const uint32_t* flags, const uint32_t* excl, int64_t n, uint32_t nruns, uint32_t* runstart,
                      cudaStream_t s);

template <typename K>
int launch_run_flags(const K* code, int64_t n, uint32_t* flags, cudaStream_t s);

template <typename K>
int launch_pair_count(const K* acode, const int32_t* aread, const int32_t* arpos, const uint32_t* arun_excl,
                      const uint32_t* arun_flag, const K* bcode, const int32_t* bread, const int32_t* brpos,
                      MergeArgs m, uint32_t* jb, uint64_t* cnt, unsigned long long* ctrun, cudaStream_t s);

int launch_gram(const unsigned long long* ctrun, int64_t nruns, unsigned long long* gram, cudaStream_t s);

int launch_cnt_mask(const uint32_t* arun_excl, const uint32_t* arun_flag, const unsigned long long* ctrun, int64_t na,
                    int limit, int always, uint64_t* cnt, cudaStream_t s);

struct HitBits
{
    int pbits, abits, bbits;
    // > 0: the emitted hits are packed keys (bread, aread, apos, bpos) with the B position in
    // the low qbits (no separate diag array), sorted keys-only on the upper bits and then
    // unpacked by launch_hit_unpack; 0: (key, diag) pairs
    int qbits;
};

int launch_emit(const int32_t* aread, const int32_t* arpos, const int32_t* bread, const int32_t* brpos,
                const uint32_t* jb, const uint64_t* cnt, const uint64_t* hoff, int64_t na, HitBits hb,
                uint64_t* hkey, uint32_t* hdiag, cudaStream_t s);

// sorted packed hits -> hkey (bread, aread, apos) and hdiag (apos - bpos)
int launch_hit_unpack(const uint64_t* packed, int64_t n, HitBits hb, uint64_t* hkey, uint32_t* hdiag, cudaStream_t s);

// Pair groups of the sorted hits: start flags, then (start, end) of groups with >= minhit hits.
// With hitmin > 0 a group of at most GD_FIRE_TEST_MAX hits is also dropped when the seed scan would find no
// candidate seed in it (group_can_fire): such a group fires no Local_Alignment and yields
// nothing, the scan would only have read its hits.  hitmin = 0 keeps every group with >=
// minhit hits.
int launch_pair_flags(const uint64_t* hkey, int64_t n, int pbits, uint32_t* flags, cudaStream_t s);
int launch_pair_scatter(const uint32_t* flags, const uint32_t* pos, int64_t n, uint32_t* starts, cudaStream_t s);
int launch_select_groups(const uint32_t* starts, int64_t nstarts, int64_t nhits, int minhit, const uint64_t* hkey,
                         const uint32_t* hdiag, int binshift, int kmer, int hitmin, HitBits hb, const int32_t* arlen,
                         const int32_t* brlen, uint2* groups, uint32_t* cost, uint32_t* idx, unsigned int* ngroups,
                         cudaStream_t s);

// groups longer than this pass selection untested (the test is quadratic in the hits, and a
// thread's long group would hold up its warp); nearly all groups without a candidate are shorter
constexpr int GD_FIRE_TEST_MAX = 16;

// the seed scan's panels: a-position windows of 50,000 overlapping by 10,000 (filter.c:1717-1745)
constexpr int GD_PANEL_SIZE = 50000;
constexpr int GD_PANEL_OVERLAP = 10000;

// Whether the seed scan of report_thread (dalign/filter.c:1717-1781) finds a candidate seed in
// the group [s, e) of the sorted hits: per panel (a panel with fewer than minhit hits is
// skipped), each diagonal band (diag >> binshift) scores the sum over its hits of min(k,
// apos - the band's previous apos in the panel, 0 for its first), and a hit is a candidate when
// its band and a neighbouring band together reach hitmin.  The same panel bounds and sums as
// k_align_pairs forms; a group without a candidate aligns nothing.  Groups of more than
// GD_FIRE_TEST_MAX hits are passed without the test.
__device__ __forceinline__ bool group_can_fire(const uint64_t* __restrict__ hkey, const uint32_t* __restrict__ hdiag,
                                               uint32_t s, uint32_t e, int pbits, int binshift, int kmer, int hitmin,
                                               int minhit)
{
    const int n = (int)(e - s);
    if (hitmin <= 0 || n > GD_FIRE_TEST_MAX)
        return true;
    // a band scores at most k per hit, so a candidate needs minhit hits in its band and a
    // neighbouring one: most groups (hits on unrelated diagonals) fail this count at once
    // (a loop over the few hits, left at the first band that passes: a fully unrolled count
    // over GD_FIRE_TEST_MAX slots in registers made the selection kernels 2-3x slower)
    bool maybe = false;
    for (int i = 0; i < n && !maybe; i++)
    {
        const int d = ((int)__ldg(hdiag + s + i)) >> binshift;
        int lo = 0, hi = 0;  // hits in bands {d - 1, d} and {d, d + 1}
        for (int j = 0; j < n; j++)
        {
            const int x = ((int)__ldg(hdiag + s + j)) >> binshift;
            lo += (x == d) | (x == d - 1);
            hi += (x == d) | (x == d + 1);
        }
        maybe = lo >= minhit || hi >= minhit;
    }
    if (!maybe)
        return false;
    int ap[GD_FIRE_TEST_MAX], bd[GD_FIRE_TEST_MAX], dl[GD_FIRE_TEST_MAX];
    const uint64_t pm = (1ull << pbits) - 1;
    for (int i = 0; i < n; i++)
    {
        ap[i] = (int)(__ldg(hkey + s + i) & pm);
        bd[i] = ((int)__ldg(hdiag + s + i)) >> binshift;
    }
    int nidx = 0, amark2 = 0;
    while (nidx < n)
    {
        const int amark = amark2 + GD_PANEL_SIZE;
        amark2 = amark - GD_PANEL_OVERLAP;
        const int lidx = nidx;
        int q = lidx;
        while (q < n && ap[q] <= amark)
            q++;
        const int nend = q < n ? q + 1 : n;
        int h2 = lidx;
        while (h2 < nend && ap[h2] <= amark2)
            h2++;
        if (nend - lidx >= minhit)
        {
            // each hit's contribution to its band's score in this panel
            for (int j = lidx; j < nend; j++)
            {
                int prev = 0;
                for (int i = lidx; i < j; i++)
                    if (bd[i] == bd[j])
                        prev = ap[i];
                dl[j] = (ap[j] - prev >= kmer) ? kmer : ap[j] - prev;
            }
            for (int i = lidx; i < nend; i++)
            {
                int sc0 = 0, up = 0, dn = 0;  // scores of bands bd[i], bd[i] + 1, bd[i] - 1
                for (int j = lidx; j < nend; j++)
                {
                    sc0 += bd[j] == bd[i] ? dl[j] : 0;
                    up += bd[j] == bd[i] + 1 ? dl[j] : 0;
                    dn += bd[j] == bd[i] - 1 ? dl[j] : 0;
                }
                if (sc0 + up >= hitmin || sc0 + dn >= hitmin)
                    return true;
            }
        }
        nidx = h2;
    }
    return false;
}

// DevBlock::pk from a block's byte buffer (buf 16-byte aligned): word i holds bytes
// [16 i, 16 i + 16), byte j of them in bits 2j..2j+1 (low two bits: a 4 packs as 0)
int launch_pack2(const uint8_t* buf, int64_t nbytes, uint32_t* pk, int64_t nwords, cudaStream_t s);

// complement_DB (dalign/daligner.c:474-573) on the device: reverse-complement every read of
// src into dst (same offsets, 4s kept), and mirror the mask intervals if there are any.
int launch_complement(const DevBlock& src, uint8_t* dst_bases, const int64_t* anno, const int32_t* mdata,
                      int32_t* mdata_dst, cudaStream_t s);

// binary searches over a sorted code array: first index with a[i] >= x (lower) / > x (upper)
template <typename K>
__device__ __forceinline__ int64_t lower_code(const K* a, int64_t n, K x)
{
    int64_t l = 0, r = n;
    while (l < r)
    {
        int64_t m = (l + r) >> 1;
        if (a[m] < x)
            l = m + 1;
        else
            r = m;
    }
    return l;
}

template <typename K>
__device__ __forceinline__ int64_t upper_code(const K* a, int64_t n, K x)
{
    int64_t l = 0, r = n;
    while (l < r)
    {
        int64_t m = (l + r) >> 1;
        if (a[m] <= x)
            l = m + 1;
        else
            r = m;
    }
    return l;
}

// the same searches restricted to [l, r), for keys known to lie in that window
template <typename K>
__device__ __forceinline__ int64_t lower_code_in(const K* a, int64_t l, int64_t r, K x)
{
    while (l < r)
    {
        int64_t m = (l + r) >> 1;
        if (a[m] < x)
            l = m + 1;
        else
            r = m;
    }
    return l;
}

template <typename K>
__device__ __forceinline__ int64_t upper_code_in(const K* a, int64_t l, int64_t r, K x)
{
    while (l < r)
    {
        int64_t m = (l + r) >> 1;
        if (a[m] <= x)
            l = m + 1;
        else
            r = m;
    }
    return l;
}

// First index of the run end after jb (the first entry > x), galloping from jb: runs are short.
template <typename K>
__device__ __forceinline__ int64_t upper_code_from(const K* a, int64_t jb, int64_t r, K x)
{
    int64_t l = jb, step = 1;  // a[l] <= x
    while (true)
    {
        const int64_t j = l + step;
        if (j >= r || a[j] > x)
            return upper_code_in(a, l + 1, min(j, r), x);
        l = j;
        step <<= 1;
    }
}

// The first index j in [lo, i] from which read[j] >> shift equals read[i] >> shift (the
// entries are sorted by read within their code run), galloping back from i.
__device__ __forceinline__ int64_t same_read_start(const int32_t* __restrict__ read, int64_t lo, int64_t i,
                                                   int shift)
{
    const int key = read[i] >> shift;
    int64_t l = i, step = 1;  // read[l] matches
    int64_t j;
    while (true)
    {
        j = l - step;
        if (j < lo)
        {
            if ((read[lo] >> shift) == key)
                return lo;
            j = lo;
            break;
        }
        if ((read[j] >> shift) != key)
            break;
        l = j;
        step <<= 1;
    }
    // read[j] does not match, read[l] does
    while (l - j > 1)
    {
        const int64_t md = (j + l) >> 1;
        if ((read[md] >> shift) == key)
            l = md;
        else
            j = md;
    }
    return l;
}

}  // namespace gd
