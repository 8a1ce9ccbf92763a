// gd_prims.cuh -- scans and the LSD radix sort used by the k-mer filter.
//
// The k-mer index and the hit list are sorted by stable least-significant-digit radix
// passes with 8-bit digits, as the reference's lex_sort does (dalign/filter.c:147-377),
// but restructured for the GPU: per pass one kernel builds per-tile digit histograms,
// one exclusive scan turns them into tile offsets (digit-major), and one kernel ranks
// every item inside its tile with warp match-any groups (stable: warps own contiguous
// sub-tiles, rounds walk them in order), re-orders the tile by digit in shared memory and
// writes each digit's items out as one contiguous run (coalesced scatter).
#pragma once
#include "gd_common.cuh"

namespace gd
{

constexpr int SCAN_THREADS = 256;
constexpr int SCAN_ITEMS = 8;
constexpr int SCAN_TILE = SCAN_THREADS * SCAN_ITEMS;

constexpr int RS_THREADS = 256;
constexpr int RS_WARPS = RS_THREADS / 32;
constexpr int RS_ROUNDS = 16;
constexpr int RS_TILE = RS_THREADS * RS_ROUNDS;  // 4096 items per tile

// Scratch bytes the exclusive scan of n elements of T needs.
template <typename T>
inline size_t scan_scratch_bytes(int64_t n)
{
    int64_t tiles = gd_cdiv<int64_t>(n, SCAN_TILE);
    return (size_t)(tiles + 1) * sizeof(T) + 256;
}

// out[i] = sum(in[0..i-1]); *total (device, may be null) = sum of all.  in may equal out.
template <typename T>
int exclusive_scan(const T* in, T* out, int64_t n, T* total, void* scratch, cudaStream_t s);

// What the last pass of a radix sort writes instead of the sorted arrays:
//   INDEX: the k-mer index from (code, packed value = read << bits | first position):
//          code[], read[] = v >> bits, rpos[] = (v & mask) + kmer - 1
//   HITS:  the hit list from keys-only packed hits (key << bits | bpos): hkey[] = k >> bits,
//          hdiag[] = apos - bpos with apos = hkey & ((1 << pbits) - 1)
struct RsFinal
{
    enum Kind
    {
        NONE = 0,
        INDEX = 1,
        HITS = 2
    } kind = NONE;
    void* a = nullptr;       // code[] / hkey[]
    int32_t* b = nullptr;    // read[] / hdiag[]
    int32_t* c = nullptr;    // rpos[]
    int bits = 0, pbits = 0, kmer = 0;
};

// Bytes of scratch a radix sort of n items needs (tile histograms + their scan).
inline size_t radix_scratch_bytes(int64_t n)
{
    int64_t tiles = gd_cdiv<int64_t>(n, RS_TILE);
    int64_t cnt = tiles * 256;
    return (size_t)cnt * 4 + scan_scratch_bytes<uint32_t>(cnt) + 256;
}

// Stable sort of (key, val) pairs by key bits [begin_bit, end_bit).  Ping-pongs between
// (k0,v0) and (k1,v1); returns 0 if the result is in (k0,v0), 1 if in (k1,v1), -1 on error.
// fin (optional): the last pass writes fin's arrays instead (the return value then only
// says where the sorted pairs would have been; with fewer than 2 items nothing is written).
template <typename K>
int radix_sort_pairs(K* k0, uint32_t* v0, K* k1, uint32_t* v1, int64_t n, int begin_bit, int end_bit, void* scratch,
                     cudaStream_t s, const RsFinal* fin = nullptr);

// The same for keys alone (16-byte aligned k0 and k1).
template <typename K>
int radix_sort_keys(K* k0, K* k1, int64_t n, int begin_bit, int end_bit, void* scratch, cudaStream_t s,
                    const RsFinal* fin = nullptr);

// 0, or -1 with the error set when a sort's bounded tile-copy wait ran out since the last
// check (the flag is cleared); synchronizes s.
int radix_sort_wait_check(cudaStream_t s);

// Test hook: the wait's expiry path on an mbarrier no copy completes (see gd_test_wait_expiry).
int radix_sort_test_wait_expiry(int polls, cudaStream_t s);

}  // namespace gd
