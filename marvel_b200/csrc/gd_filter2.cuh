// gd_filter2.cuh -- daligner2's modimizer filter (dalign2/filter.c) on sm_100a.
//
// daligner2 lists, at every k-mer position of a read, up to two codes -- the canonical k-mer
// (the smaller of the forward code and its reverse complement) and a "half-shifted" code whose
// high half comes from the previous position -- keeping a code when code % 101 < 28.  One
// sorted index per block then serves both orientations: an A entry and a B entry of the same
// code pair forward when their strands agree, and complemented otherwise.
#pragma once
#include "gd_filter.cuh"

namespace gd
{

// the bit masks of Set_Filter_Params (dalign2/filter.c:83-128)
struct D2Masks
{
    uint64_t kmask, lf, hf, lr, hr;
    int kshift;
};

D2Masks d2_masks(int kmer);

// Per slot: how many codes the slot lists (0..2).
int launch_d2_count(const DevBlock& b, const int64_t* mask_anno, const int32_t* mask_data, int kmer,
                    const D2Masks& m, int64_t nslots, uint32_t* count, cudaStream_t s);

// Per slot, at off[slot]: keys (code), vals (entry index), rd ((read << 1) | strand), rp (position).
template <typename K>
int launch_d2_emit(const DevBlock& b, const int64_t* mask_anno, const int32_t* mask_data, int kmer,
                   const D2Masks& m, int64_t nslots, const uint32_t* off, K* keys, uint32_t* vals, int32_t* rd,
                   int32_t* rp, cudaStream_t s);

// The index arrays from sorted (code, entry index) pairs.
template <typename K>
int launch_d2_gather(const K* skeys, const uint32_t* svals, int64_t n, const int32_t* rd, const int32_t* rp, K* code,
                     int32_t* read, int32_t* rpos, cudaStream_t s);

// flags[i] = strand bit of entry i (for the exclusive scan of strands over the B index).
int launch_d2_strand_flags(const int32_t* read, int64_t n, uint32_t* flags, cudaStream_t s);

// Per A entry: the B range [jb, jb + n) it pairs with, split by orientation (cnt_f forward,
// cnt_c complement), and the per-code-run totals (count_thread, dalign2/filter.c:1136-1256).
// runstart (non-null when B is A's own index): the start of every code run of A; otherwise
// btable / bshift: B's bucket table (launch_code_buckets).
template <typename K>
int launch_d2_pair_count(const K* acode, const int32_t* aread, const uint32_t* arun_excl, const uint32_t* arun_flag,
                         const uint32_t* runstart, const uint32_t* btable, int bshift, uint32_t nbuckets,
                         const K* bcode, const int32_t* bread, const uint32_t* bstrand_excl, int64_t na, int64_t nb,
                         int self, int identity, uint32_t* jb, uint64_t* cnt_f, uint64_t* cnt_c,
                         unsigned long long* ctrun, cudaStream_t s);

// The hits of each orientation in generation order (merge_thread, dalign2/filter.c:1259-1466):
// forward into (fkey, fdiag) at foff, complement -- B position reflected -- into (ckey, cdiag)
// at coff.  Keys are (bread, aread, apos) packed as HitBits says.
int launch_d2_emit_hits(const int32_t* aread, const int32_t* arpos, const int32_t* bread, const int32_t* brpos,
                        const int32_t* brlen, const uint32_t* jb, const uint64_t* cnt_f, const uint64_t* cnt_c,
                        const uint64_t* foff, const uint64_t* coff, int64_t na, int kmer, HitBits hb, uint64_t* fkey,
                        uint32_t* fdiag, uint64_t* ckey, uint32_t* cdiag, cudaStream_t s);

}  // namespace gd
