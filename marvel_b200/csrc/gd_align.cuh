// gd_align.cuh -- warp-per-pair seed scan and adaptive-wave aligner for sm_100a.
#pragma once
#include "gd_common.cuh"
#include "gd_filter.cuh"

struct gd_context;

// The alignment spec of a context (trim tables, trace spacing, PATH_AVE) for entry points
// outside gd_pipeline.cu; null until gd_new_align_spec has been called.
const int16_t* gd_context_align_tables(gd_context* ctx, int* tspace, int* ave_path, int* mscore, int* dscore);

namespace gd
{

constexpr int RING = 128;           // wave-vector rings per warp, one for the previous and one for the
                                     // current wave (diagonal k lives at k & (RING-1)): the widest band
constexpr int WIDE_RING = 512;      // the same for the wide instance, for pair groups whose band outgrows RING
constexpr int TEST_RING = 32;       // a narrow instance for tests only: most groups then go to the wide one
constexpr int ALIGN_WARPS = 4;      // warps per CTA of the aligner (the wide instance: 1)
constexpr int DUO = (1 << 16) | 128; // the two-teams-per-warp instance: its id carries the team split
                                     // (bit 16: half-warp teams of 16 lanes) and the ring (128 per team)
#ifndef GD_DUO_WARPS
#define GD_DUO_WARPS 2
#endif
constexpr int DUO_WARPS = GD_DUO_WARPS;  // warps per CTA of the duo instance
constexpr int TRIM_TABLE = 1 << 15; // TRIM_MASK + 1 (dalign/align.c:154)

// One path as Local_Alignment returns it (dalign/align.h:76-83); trace is an offset into
// the owning buffer.
struct MPath
{
    int32_t toff, tlen, diffs, abpos, bbpos, aepos, bepos, pad;
};

// One output overlap record (the 40-byte .las record plus where its trace bytes are).
struct OutRec
{
    int32_t tlen, diffs, abpos, bbpos, aepos, bepos;
    uint32_t flags;
    int32_t aread, bread, pad;
    uint64_t toff;
};

struct AlignParams
{
    int tspace, ave_path, kmer, binshift, hitmin, minover;
    int symmetric, self, comp, trace8, no_trace;
    int mindiag, maxdiag;  // band range of the block pair: (-maxlen_B >> w) .. (maxlen_A >> w)
    HitBits hb;
    const int16_t* table;  // TABLE and SCORE trim tables (set_table, dalign/align.c:196-210)
    const int16_t* score;
    int mscore, dscore;    // match / edit weights the tables are built from (align.c:238-240)
    int test_narrow;       // tests only: the main pass runs the TEST_RING instance
    int d2, hgap;          // daligner2's report (dalign2/filter_reporter_cpu.c) and its -H
};

// Per-warp global scratch, carved from one allocation.
struct AlignScratch
{
    int4* peb;         // pebbles {ptr, diag, diff, mark}
    int pcap;
    uint16_t* pts;     // Local_Alignment trace points (4 * maxtp + 16 per warp)
    int ptscap;
    MPath* match;      // amatch | bmatch, mcap each
    int mcap;
    uint16_t* tbuf;    // per-pair trace buffer
    int tcap;
    int* bands;        // score | lastp | lasta, each nbands ints
    int nbands;
    int nwarps;
    int* bvec;         // daligner2 bridging: the O(nd) wave vectors of Compute_Alignment (bvcap ints
    int bvcap;         //   per warp; 0 outside daligner2 mode)
    uint16_t* btr;     //   and the bridge's trace (btcap values per warp)
    int btcap;
};

struct AlignOut
{
    OutRec* rec;
    uint8_t* trace;
    unsigned long long* counters;  // [0] records, [1] trace bytes, [2] cells, [3] seeds, [4] LA calls kept
    uint64_t rcap, tcap;
    const uint8_t* skip;  // per pair group: 1 = triaged away (may be null)
    uint2* gstat;         // per pair group: (records emitted, wave cells) (may be null)
    unsigned* wide_list;  // groups handed to the wide instance (null: a too-wide band is an error)
    unsigned* nwide;      // their count
};

size_t align_scratch_bytes(int nwarps, int pcap, int ptscap, int mcap, int tcap, int nbands, int bvcap = 0,
                           int btcap = 0);
void align_scratch_carve(AlignScratch* s, void* base, int nwarps, int pcap, int ptscap, int mcap, int tcap, int nbands,
                         int bvcap = 0, int btcap = 0);

// Persistent seed-scan + alignment over the ordered pair groups on one instance (wide): 0 the
// warp instance (RING), 1 the wide instance (WIDE_RING, one warp per CTA), 2 the duo instance
// (two half-warp teams per warp, 128-diagonal rings each; sc holds a slot per team,
// align_slots_per_warp).  The
// duo instance aligns daligner's report; daligner2's (p.d2) and the tests' narrow instance
// (p.test_narrow) take the warp instance in its place.
int launch_align_pairs(const DevBlock& A, const DevBlock& B, const uint64_t* hkey, const uint32_t* hdiag,
                       const uint2* groups, const uint32_t* order, unsigned ngroups, AlignParams p, AlignScratch sc,
                       AlignOut out, unsigned* queue, DevStatus* st, int grid, cudaStream_t s, int wide = 0);

// One Local_Alignment per seed (for parity tests of the wave alone).  out12 per seed:
// A-path {abpos,bbpos,aepos,bepos,diffs,tlen}, B-path the same; traces at
// tr + seed * trstride (A) and tr + seed * trstride + trstride/2 (B).
int launch_la_batch(const uint8_t* aseq_base, const int64_t* aoff, const int32_t* alen, const uint8_t* bseq_base,
                    const int64_t* boff, const int32_t* blen, const int32_t* diag, const int32_t* anti, int nseeds,
                    AlignParams p, AlignScratch sc, int32_t* out12, uint16_t* tr, int trstride, int64_t* cells,
                    DevStatus* st, cudaStream_t s);

// Test hook: daligner2's Handle_Redundancies of one pair on one device thread (see gd_align.cu).
int launch_test_hr_d2(const uint8_t* aseq, const uint8_t* bseq, int alen, int blen, int tspace, int comp, int novls,
                      int hasB, const int32_t* hdr, MPath* paths, uint16_t* tbuf, int ttop, int tcap, int* vec,
                      int vcap, uint16_t* btr, int btcap, int32_t* out_hdr, int* out_n, cudaStream_t s);

// CTAs for a persistent launch of an instance (wide as in launch_align_pairs), its warps per CTA
int align_grid(int* grid_out, int wide = 0);
int align_warps_per_cta(int wide);
// scratch slots per warp of an instance: 2 for the duo instance, else 1
int align_slots_per_warp(int wide);

}  // namespace gd
