// gd_align.cu -- seed scan and adaptive-wave local alignment, one warp per (aread, bread) pair.
//
// Restates dalign/filter.c report_thread (:1617-1989) and dalign/align.c Local_Alignment
// (:1922-2060) with forward_wave (:369-1110) and reverse_wave (:1114-1916).
//
// GPU mapping.  A warp owns one pair group of the sorted hit list.  The panel band scores
// are built lane-parallel (match-any groups per diagonal band), candidate seeds are taken
// in hit order, and each fired seed runs the O(ND) wave with lanes over diagonals: the
// wave vectors V (furthest anti-diagonal), T (60-column match bit vector; its popcount
// is the reference's M), HA/HB (pebble heads), NA/NB (next trace-point marks) live in two
// per-warp shared-memory rings indexed by diagonal, one per wave parity: each wave reads
// the previous wave for diagonals k-1, k, k+1 and writes the other ring, which is the
// reference's in-place update order.  The reference's sequential "c > besta" scan over
// diagonals becomes a warp prefix-max in scan order; its clip bookkeeping becomes ballots.
// Pebbles go to a per-warp global arena; the two trace-point chains are unwound by lane 0.
// Match extension compares 4 bases per step with 32-bit XOR windows.
//
// Instances by ring size: RING (128 diagonals, 4 warps per CTA) aligns every pair group; a
// group whose band grows wider is abandoned there (nothing emitted, its counts dropped) and
// listed for the WIDE_RING instance (512 diagonals, 1 warp per CTA), which aligns it from
// scratch.  TEST_RING (32) replaces RING in tests so that most groups take that route.  The
// duo instance (k_align_duo, DUO) splits each warp into two 16-lane teams with 128-diagonal
// rings each, one pair group per team; the wave functions are written over a team (WarpCtx
// with team collectives), and wave_step_duo runs both teams' waves in lockstep.
#include "gd_align.cuh"

#include <climits>
#include <type_traits>

namespace gd
{

#define PATH_TOP 0x1000000000000000ull
#define PATH_INT 0x0fffffffffffffffull
#define MASK61 0x1fffffffffffffffull
#define TRIM_LEN 15
#define TRIM_MASK 0x7fff
#define TRIM_MLAG 200
#define WAVE_LAG 30
#define PANEL_SIZE 50000
#define PANEL_OVERLAP 10000
#define RM (ring_of<RG>() - 1)  // ring index mask of the instance
#define SENT4 0x0404040404040404ull

// An instance id RG is its ring size (diagonals per wave ring), with bit 16 set for the duo
// instance's half-warp teams.
template <int RG>
constexpr int ring_of()
{
    return RG & 0xffff;
}

// Wave vectors by diagonal (k & RM).  The warp instances keep one ring per warp and update it
// in place: within a chunk of 32 diagonals every lane reads its three predecessors before any
// lane writes (the reads come before the chunk's first warp vote, the writes after a warp
// barrier), and the one diagonal a chunk's first lane reads from the chunk before it (its kP,
// and for a new band edge its NA/NB) is saved by that chunk's last lane before it writes
// (ChunkEdge).  One ring instead of two halves the shared memory of a warp, which leaves the
// SM a larger L1 for the reads' 2-bit words and the pebbles.  The duo instance's teams keep
// two rings, [dif & 1] holding wave dif.
template <int RG>
constexpr int parities_of()
{
    return (RG >> 16) ? 2 : 1;
}

template <int RG>
__device__ __forceinline__ int par(int dif)
{
    if constexpr (parities_of<RG>() == 2)
        return dif & 1;
    else
        return 0;
}

template <int RG>
struct WaveSmem
{
    unsigned long long T[parities_of<RG>()][ring_of<RG>()];
    int V[parities_of<RG>()][ring_of<RG>()], HA[parities_of<RG>()][ring_of<RG>()], HB[parities_of<RG>()][ring_of<RG>()],
        NA[parities_of<RG>()][ring_of<RG>()], NB[parities_of<RG>()][ring_of<RG>()];
};

// The previous wave's values at the last diagonal of a 32-lane chunk, for the next chunk's
// first lane (single-ring instances only)
struct ChunkEdge
{
    unsigned long long t;
    int v, ha, hb, na, nb, pad;
};

struct LAPath
{
    int abpos, bbpos, aepos, bepos, diffs, tlen, toff, pad;
};

template <int RG>
struct WarpSmem
{
    WaveSmem<RG> ws;
    LAPath ap, bp;
    int span_lo, span_hi;
    int trim[5];  // the trim point (anti-diagonal, y, diffs, A and B pebble heads), written by its lane
    int clipm[6];  // the clip fallback: M count, anti-diagonal, y, diffs, A and B pebble heads
    int besty;    // y of the best anti-diagonal
    ChunkEdge edge[ring_of<RG>() / 32 > 1 ? ring_of<RG>() / 32 - 1 : 1];  // [ch]: chunk ch's last diagonal
};

// The lanes that align one pair group together: a whole warp, or in the duo instance a
// half-warp team of 16 (two pair groups per warp).
template <int RG>
constexpr int team_width()
{
    return (RG >> 16) ? 16 : 32;
}

template <int RG>
struct WarpCtx
{
    WarpSmem<RG>* sm;
    int4* peb;
    int pcap;
    uint16_t* pts;
    int ptscap;
    DevStatus* st;
    int lane;        // lane within the team
    int err;         // 1: failed (status set); 2: the band outgrew this instance (the caller decides)
    int item;
    unsigned cells;  // wave cells of the current pair group (or seed)
    unsigned tmask;  // the team's lanes in the warp (half-warp teams only)
    int tbase;       // the team's first lane in the warp (half-warp teams only)
};

// Warp collectives over a team: the whole warp (constant masks, as plain warp code) or a
// half-warp (its mask; ballots and match masks shifted to the team's 16 bits).
template <int RG>
__device__ __forceinline__ unsigned tmask(const WarpCtx<RG>& w)
{
    if constexpr (team_width<RG>() == 32)
        return GD_FULL;
    else
        return w.tmask;
}

template <int RG>
__device__ __forceinline__ unsigned tballot(const WarpCtx<RG>& w, bool p)
{
    if constexpr (team_width<RG>() == 32)
        return __ballot_sync(GD_FULL, p);
    else
        return (__ballot_sync(w.tmask, p) >> w.tbase) & 0xffffu;
}

template <int RG>
__device__ __forceinline__ bool tany(const WarpCtx<RG>& w, bool p)
{
    return __any_sync(tmask(w), p);
}

template <int RG, typename T>
__device__ __forceinline__ T tshfl(const WarpCtx<RG>& w, T v, int src)
{
    return __shfl_sync(tmask(w), v, src, team_width<RG>());
}

template <int RG, typename T>
__device__ __forceinline__ T tshfl_up(const WarpCtx<RG>& w, T v, int o)
{
    return __shfl_up_sync(tmask(w), v, o, team_width<RG>());
}

template <int RG>
__device__ __forceinline__ int tmax(const WarpCtx<RG>& w, int v)
{
    return __reduce_max_sync(tmask(w), v);
}

template <int RG>
__device__ __forceinline__ int tmin(const WarpCtx<RG>& w, int v)
{
    return __reduce_min_sync(tmask(w), v);
}

template <int RG>
__device__ __forceinline__ int tadd(const WarpCtx<RG>& w, int v)
{
    return __reduce_add_sync(tmask(w), v);
}

template <int RG>
__device__ __forceinline__ unsigned tmatch(const WarpCtx<RG>& w, unsigned v)
{
    if constexpr (team_width<RG>() == 32)
        return __match_any_sync(GD_FULL, v);
    else
        return (__match_any_sync(w.tmask, v) >> w.tbase) & 0xffffu;
}

template <int RG>
__device__ __forceinline__ void tsync(const WarpCtx<RG>& w)
{
    __syncwarp(tmask(w));
}

// lanes of the team below this one
template <int RG>
__device__ __forceinline__ unsigned tlt(const WarpCtx<RG>& w)
{
    if constexpr (team_width<RG>() == 32)
        return lanemask_lt();
    else
        return (1u << w.lane) - 1u;
}

__device__ __forceinline__ unsigned ld4u(const uint8_t* p)
{
    uintptr_t a = (uintptr_t)p;
    const unsigned* q = (const unsigned*)(a & ~(uintptr_t)3);
    return __funnelshift_r(__ldg(q), __ldg(q + 1), (unsigned)(a & 3) * 8);
}

// Extend the match on diagonal k from b-position y forward (FWD) or backward.
// Returns the new y; sets bend/aend like the reference's snake loop (align.c:798-824).
__device__ __forceinline__ int snake(const bool FWD, const uint8_t* aseq, const uint8_t* bseq, int y, int k, int lim, bool& bend,
                                     bool& aend)
{
    if (FWD)
    {
        // the 4 after every read stops the extension; the cap only guards against a bad pointer
        for (int guard = (lim >> 2) + 2; guard > 0; guard--)
        {
            unsigned wb = ld4u(bseq + y), wa = ld4u(aseq + y + k);
            unsigned stop = (wa ^ wb) | (wb & 0x04040404u);
            if (stop)
            {
                int i = (__ffs((int)stop) - 1) >> 3;
                y += i;
                int cb = (int)(wb >> (8 * i)) & 0xff;
                bend = (cb == 4);
                aend = !bend && (((int)(wa >> (8 * i)) & 0xff) == 4);
                return y;
            }
            y += 4;
        }
        bend = aend = true;  // unreachable with well-formed blocks (every read ends with a 4)
    }
    else
    {
        for (int guard = (lim >> 2) + 2; guard > 0; guard--)
        {
            unsigned wb = ld4u(bseq + y - 4), wa = ld4u(aseq + y + k - 4);
            unsigned stop = (wa ^ wb) | (wb & 0x04040404u);
            if (stop)
            {
                int i = __clz((int)stop) >> 3;
                y -= i;
                int sh = 8 * (3 - i);
                int cb = (int)(wb >> sh) & 0xff;
                bend = (cb == 4);
                aend = !bend && (((int)(wa >> sh) & 0xff) == 4);
                return y;
            }
            y -= 4;
        }
        bend = aend = true;
    }
    return y;
}

// The same from the 2-bit copies: A's base i at apk index ag + i, B's at bpk index bg + i; 16
// bases per step (one funnel shift per sequence), the read ends found from the lengths
// instead of the 4s: the extension stops at the first mismatch, the end of b (bend, also when
// both end there) or the end of a (aend), as the 4s stop the byte loop.
__device__ __forceinline__ int snake_pk(const bool FWD, const uint32_t* __restrict__ apk, uint32_t ag,
                                        const uint32_t* __restrict__ bpk, uint32_t bg, int y, int k, int alen,
                                        int blen, bool& bend, bool& aend)
{
    int eb = FWD ? blen - y : y;  // bases left before the end of b / a in the direction of travel
    int ea = FWD ? alen - (y + k) : y + k;
    while (true)
    {
        const uint32_t sb = FWD ? bg + y : bg + y - 16, sa = FWD ? ag + y + k : ag + y + k - 16;
        const uint32_t wb = __funnelshift_r(__ldg(bpk + (sb >> 4)), __ldg(bpk + (sb >> 4) + 1), 2 * (sb & 15));
        const uint32_t wa = __funnelshift_r(__ldg(apk + (sa >> 4)), __ldg(apk + (sa >> 4) + 1), 2 * (sa & 15));
        const uint32_t x = wa ^ wb;
        // matching bases from the start of travel: low bits first forward, high bits first back
        const int m = FWD ? (x ? (__ffs((int)x) - 1) >> 1 : 16) : (__clz((int)x) >> 1);
        const int s = min(m, min(ea, eb));
        if (s < 16)
        {
            bend = s == eb;
            aend = !bend && s == ea;
            return FWD ? y + s : y - s;
        }
        y += FWD ? 16 : -16;
        ea -= 16;
        eb -= 16;
    }
}

// The trim test of forward_wave/reverse_wave (align.c:884-896): the newest 15 columns are
// suffix-positive and so are the newest 30 (TABLE / SCORE built by set_table, align.c:196-210).
__device__ __forceinline__ bool trim_ok(unsigned long long b, const int16_t* table, const int16_t* score)
{
    int lo15 = (int)(b & TRIM_MASK), hi15 = (int)((b >> TRIM_LEN) & TRIM_MASK);
    return (__ldg(table + lo15) >= 0) && (__ldg(table + hi15) + __ldg(score + lo15) >= 0);
}

// uniform single-pebble allocation (all lanes call, lane 0 writes)
template <int RG>
__device__ __forceinline__ int peb_one(WarpCtx<RG>& w, int& npeb, int ptr, int diag, int diff, int mark)
{
    int idx = npeb++;
    if (idx >= w.pcap)
    {
        if (!w.err && w.lane == 0)
            gd_fail(w.st, GD_ERR_PEBBLES, w.item, w.pcap);
        w.err = 1;
        return 0;
    }
    if (w.lane == 0)
        w.peb[idx] = make_int4(ptr, diag, diff, mark);
    return idx;
}

// The wave's state between waves (forward_wave / reverse_wave's loop-carried locals).
struct WaveVars
{
    int hgh, low, dif, more, aclip, bclip, besta, lasta, npeb;
};

// forward_wave (FWD) / reverse_wave (!FWD) restated, with lanes over diagonals, in three
// parts so that a caller can run it a wave at a time: wave_begin (the 0-wave from the seed
// point), wave_step (one wave; false when the wave loop ends, or on an error in w.err) and
// wave_end (the trace points of both paths from the pebble chains).
template <int RG, bool PK>
__device__ __forceinline__ void wave_begin(const bool FWD, WarpCtx<RG>& w, WaveVars& wvars, const AlignParams& P, const uint8_t* aseq0, const uint8_t* bseq0,
    const uint32_t* apk, uint32_t ag, const uint32_t* bpk, uint32_t bg, int alen, int blen, int comp, int low0, int maxd, int mida)
{
    WaveSmem<RG>& R = w.sm->ws;
    const int lane = w.lane;
    const int TS = P.tspace;
    const int S = FWD ? 1 : -1;
    const int VNONE = FWD ? -1 : INT_MAX;
    const int boff = comp ? blen % TS : 0;
    int* const trim = w.sm->trim;
    int* const clipm = w.sm->clipm;
    const uint8_t* as = FWD ? aseq0 : aseq0 - 1;
    const uint8_t* bs = FWD ? bseq0 : bseq0 - 1;
    (void)S; (void)VNONE; (void)boff; (void)as; (void)bs; (void)trim; (void)clipm; (void)R; (void)TS; (void)lane;
    int hgh = maxd, low = low0, dif = 0;
    int more = 1;
    int aclip = FWD ? INT_MAX : -INT_MAX;
    int bclip = FWD ? -INT_MAX : INT_MAX;
    int besta, lasta;
    besta = lasta = mida;
    if (lane == 0)
    {
        trim[0] = mida;
        trim[1] = (mida - hgh) >> 1;
        trim[2] = 0;
        trim[3] = 0;
        trim[4] = 1;
        clipm[0] = -1;
        w.sm->besty = (mida - hgh) >> 1;
    }
    int npeb = 0;

    if (low != hgh)
    {
        if (lane == 0)
            gd_fail(w.st, GD_ERR_BAND_WIDTH, w.item, -1);
        w.err = 1;
        wvars.hgh = hgh; wvars.low = low; wvars.dif = dif; wvars.more = more; wvars.aclip = aclip; wvars.bclip = bclip; wvars.besta = besta; wvars.lasta = lasta; wvars.npeb = npeb;
        return;
    }

    // ---- 0-wave from the seed point on its single diagonal
    {
        int k = hgh;
        int y = (mida - k) >> 1;
        int ha, hb, na, nb;
        if (FWD)
        {
            na = ((y + k) / TS) * TS;
            ha = peb_one(w, npeb, -1, k, 0, na);
            na += TS;
            nb = ((y + (TS - boff)) / TS - 1) * TS + boff;
            hb = peb_one(w, npeb, -1, k, 0, nb);
            nb += TS;
        }
        else
        {
            na = ((y + k + TS - 1) / TS - 1) * TS;
            ha = peb_one(w, npeb, -1, k, 0, y + k);
            nb = ((y + (TS - boff) - 1) / TS - 1) * TS + boff;
            hb = peb_one(w, npeb, -1, k, 0, y);
        }
        bool bend, aend;
        y = PK ? snake_pk(FWD, apk, ag, bpk, bg, y, k, alen, blen, bend, aend)
               : snake(FWD, aseq0, bseq0, y, k, blen + 16, bend, aend);
        if (bend)
        {
            more = 0;
            bclip = FWD ? max(bclip, k) : min(bclip, k);
        }
        if (aend)
        {
            more = 0;
            aclip = k;
        }
        int c = (y << 1) + k;
        if (FWD)
        {
            while (y + k >= na)
            {
                ha = peb_one(w, npeb, ha, k, 0, na);
                na += TS;
            }
            while (y >= nb)
            {
                hb = peb_one(w, npeb, hb, k, 0, nb);
                nb += TS;
            }
        }
        else
        {
            while (y + k <= na)
            {
                ha = peb_one(w, npeb, ha, k, 0, na);
                na -= TS;
            }
            while (y <= nb)
            {
                hb = peb_one(w, npeb, hb, k, 0, nb);
                nb -= TS;
            }
        }
        if (FWD ? (c > besta) : (c < besta))
        {
            besta = lasta = c;
            if (lane == 0)
            {
                trim[0] = c;
                trim[1] = y;
                trim[3] = ha;
                trim[4] = hb;
                w.sm->besty = y;
            }
        }
        if (lane == 0)
        {
            R.V[0][k & RM] = c;
            R.T[0][k & RM] = PATH_INT;
            R.HA[0][k & RM] = ha;
            R.HB[0][k & RM] = hb;
            R.NA[0][k & RM] = na;
            R.NB[0][k & RM] = nb;
        }
        tsync(w);
    }
    if (w.err)
    {
        wvars.hgh = hgh; wvars.low = low; wvars.dif = dif; wvars.more = more; wvars.aclip = aclip; wvars.bclip = bclip; wvars.besta = besta; wvars.lasta = lasta; wvars.npeb = npeb;
        return;
    }

    auto clip_block = [&]() {
        if (!more)
        {
            const int besty = w.sm->besty;
            // the best point is not at a read end (the bytes there are 4s)
            if (PK ? (FWD ? (besty < blen && besta - besty < alen) : (besty > 0 && besta - besty > 0))
                   : (__ldg(bs + besty) != 4 && __ldg(as + besta - besty) != 4))
                more = 1;
            if (FWD ? (hgh >= aclip) : (low <= aclip))
            {
                if (FWD)
                    hgh = aclip - 1;
                else
                    low = aclip + 1;
                int Mc = __popcll(R.T[par<RG>(dif)][aclip & RM] & MASK61);
                if (lane == 0 && clipm[0] <= Mc)
                {
                    clipm[0] = Mc;
                    clipm[1] = R.V[par<RG>(dif)][aclip & RM];
                    clipm[2] = (clipm[1] - aclip) / 2;
                    clipm[3] = dif;
                    clipm[4] = R.HA[par<RG>(dif)][aclip & RM];
                    clipm[5] = R.HB[par<RG>(dif)][aclip & RM];
                }
                tsync(w);
            }
            if (FWD ? (low <= bclip) : (hgh >= bclip))
            {
                if (FWD)
                    low = bclip + 1;
                else
                    hgh = bclip - 1;
                int Mc = __popcll(R.T[par<RG>(dif)][bclip & RM] & MASK61);
                if (lane == 0 && clipm[0] <= Mc)
                {
                    clipm[0] = Mc;
                    clipm[1] = R.V[par<RG>(dif)][bclip & RM];
                    clipm[2] = (clipm[1] - bclip) / 2;
                    clipm[3] = dif;
                    clipm[4] = R.HA[par<RG>(dif)][bclip & RM];
                    clipm[5] = R.HB[par<RG>(dif)][bclip & RM];
                }
                tsync(w);
            }
            aclip = FWD ? INT_MAX : -INT_MAX;
            bclip = FWD ? -INT_MAX : INT_MAX;
        }
    };
    clip_block();
    wvars.hgh = hgh; wvars.low = low; wvars.dif = dif; wvars.more = more; wvars.aclip = aclip; wvars.bclip = bclip; wvars.besta = besta; wvars.lasta = lasta; wvars.npeb = npeb;
}

template <int RG, bool PK>
__device__ __forceinline__ bool wave_step(const bool FWD, WarpCtx<RG>& w, WaveVars& wvars, const AlignParams& P, const uint8_t* aseq0, const uint8_t* bseq0,
    const uint32_t* apk, uint32_t ag, const uint32_t* bpk, uint32_t bg, int alen, int blen, int comp, int minp, int maxp)
{
    WaveSmem<RG>& R = w.sm->ws;
    const int lane = w.lane;
    const int TS = P.tspace;
    const int S = FWD ? 1 : -1;
    const int VNONE = FWD ? -1 : INT_MAX;
    const int boff = comp ? blen % TS : 0;
    int* const trim = w.sm->trim;
    int* const clipm = w.sm->clipm;
    const uint8_t* as = FWD ? aseq0 : aseq0 - 1;
    const uint8_t* bs = FWD ? bseq0 : bseq0 - 1;
    (void)S; (void)VNONE; (void)boff; (void)as; (void)bs; (void)trim; (void)clipm; (void)R; (void)TS; (void)lane;
    int hgh = wvars.hgh, low = wvars.low, dif = wvars.dif, more = wvars.more;
    int aclip = wvars.aclip, bclip = wvars.bclip, besta = wvars.besta, lasta = wvars.lasta, npeb = wvars.npeb;
    auto clip_block = [&]() {
        if (!more)
        {
            const int besty = w.sm->besty;
            // the best point is not at a read end (the bytes there are 4s)
            if (PK ? (FWD ? (besty < blen && besta - besty < alen) : (besty > 0 && besta - besty > 0))
                   : (__ldg(bs + besty) != 4 && __ldg(as + besta - besty) != 4))
                more = 1;
            if (FWD ? (hgh >= aclip) : (low <= aclip))
            {
                if (FWD)
                    hgh = aclip - 1;
                else
                    low = aclip + 1;
                int Mc = __popcll(R.T[par<RG>(dif)][aclip & RM] & MASK61);
                if (lane == 0 && clipm[0] <= Mc)
                {
                    clipm[0] = Mc;
                    clipm[1] = R.V[par<RG>(dif)][aclip & RM];
                    clipm[2] = (clipm[1] - aclip) / 2;
                    clipm[3] = dif;
                    clipm[4] = R.HA[par<RG>(dif)][aclip & RM];
                    clipm[5] = R.HB[par<RG>(dif)][aclip & RM];
                }
                tsync(w);
            }
            if (FWD ? (low <= bclip) : (hgh >= bclip))
            {
                if (FWD)
                    low = bclip + 1;
                else
                    hgh = bclip - 1;
                int Mc = __popcll(R.T[par<RG>(dif)][bclip & RM] & MASK61);
                if (lane == 0 && clipm[0] <= Mc)
                {
                    clipm[0] = Mc;
                    clipm[1] = R.V[par<RG>(dif)][bclip & RM];
                    clipm[2] = (clipm[1] - bclip) / 2;
                    clipm[3] = dif;
                    clipm[4] = R.HA[par<RG>(dif)][bclip & RM];
                    clipm[5] = R.HB[par<RG>(dif)][bclip & RM];
                }
                tsync(w);
            }
            aclip = FWD ? INT_MAX : -INT_MAX;
            bclip = FWD ? -INT_MAX : INT_MAX;
        }
    };

    const unsigned lt = tlt(w);
    const int PATH_AVE = P.ave_path;
    if (!(more && (FWD ? (lasta >= besta - TRIM_MLAG) : (lasta <= besta + TRIM_MLAG))))
        return false;
    // widen the band by one each side (align.c:636-745).  Diagonals outside the previous
    // band read as VNONE and new end diagonals take their inner neighbour's NA/NB: the
    // reference writes those values into its vectors first, here they are read that way.
    const int olow = low, ohgh = hgh;
    if (olow > ohgh)  // every diagonal fell WAVE_LAG behind: the reference would read stale vectors
    {
        if (lane == 0)
            gd_fail(w.st, GD_ERR_EMPTY_BAND, w.item, dif);
        w.err = 1;
        wvars.hgh = hgh; wvars.low = low; wvars.dif = dif; wvars.more = more; wvars.aclip = aclip; wvars.bclip = bclip; wvars.besta = besta; wvars.lasta = lasta; wvars.npeb = npeb;
        return false;
    }
    low -= 1;
    hgh += 1;
    if (low < minp)
        low += 1;
    if (hgh > maxp)
        hgh -= 1;
    dif += 1;
    if (dif > alen + blen + 2)  // the edit distance cannot exceed alen + blen
    {
        if (lane == 0)
            gd_fail(w.st, GD_ERR_EMPTY_BAND, w.item, dif);
        w.err = 1;
        wvars.hgh = hgh; wvars.low = low; wvars.dif = dif; wvars.more = more; wvars.aclip = aclip; wvars.bclip = bclip; wvars.besta = besta; wvars.lasta = lasta; wvars.npeb = npeb;
        return false;
    }
    const int width = hgh - low + 1;
    if ((unsigned)(width - 1) >= (unsigned)ring_of<RG>())  // empty, or wider than this instance
    {
        if (width > ring_of<RG>())
            w.err = 2;  // a wider instance may take this pair (the caller decides)
        else
        {
            if (lane == 0)
                gd_fail(w.st, GD_ERR_EMPTY_BAND, w.item, width);
            w.err = 1;
        }
        wvars.hgh = hgh; wvars.low = low; wvars.dif = dif; wvars.more = more; wvars.aclip = aclip; wvars.bclip = bclip; wvars.besta = besta; wvars.lasta = lasta; wvars.npeb = npeb;
        return false;
    }
    constexpr int TW = team_width<RG>();
    const int nch = (width + TW - 1) / TW;
    const int hgh0 = hgh, low0 = low;
    constexpr int NP = parities_of<RG>();
    const int cur = par<RG>(dif), prv = par<RG>(dif - 1);
    int c0 = 0;  // chunk 0's new V, for the WAVE_LAG test
    // one chunk of 32 diagonals; true: the wave failed (w.err set, wvars stored).  Chunk 0 is
    // specialised, the rare later chunks share one non-unrolled copy
    auto chunk = [&](const int ch, auto first) -> bool {
        constexpr bool FIRST = decltype(first)::value;
        const int p = ch * TW + lane;
        const bool valid = p < width;
        const int k = FWD ? hgh - p : low + p;
        int c = 0, y = 0, ha = 0, hb = 0, na = 0, nb = 0;
        unsigned long long b = 0;
        bool bend = false, aend = false;
        // single ring: the chunk before this one has written its diagonals, so the first lane
        // takes its kP values from that chunk's saved edge
        const bool fromedge = NP == 1 && !FIRST && lane == 0;
        if (NP == 1 && !FIRST)
            tsync(w);
        if (valid)
        {
            // choose the furthest of the three predecessors (align.c:748-797)
            const int kP = k + S, kN = k - S;
            int vP = (kP >= olow && kP <= ohgh) ? R.V[prv][kP & RM] : VNONE;
            int vC = (k >= olow && k <= ohgh) ? R.V[prv][k & RM] : VNONE;
            int vN = (kN >= olow && kN <= ohgh) ? R.V[prv][kN & RM] : VNONE;
            if (fromedge)
                vP = w.sm->edge[ch > 0 ? ch - 1 : 0].v;
            int wP = FWD ? vP : -vP, wC = FWD ? vC : -vC, wN = FWD ? vN : -vN;
            int ks, vs, step;
            if (wC < wN)
            {
                if (wN < wP)
                {
                    ks = k + S;
                    vs = vP;
                }
                else
                {
                    ks = k - S;
                    vs = vN;
                }
                step = 1;
            }
            else if (wC < wP)
            {
                ks = k + S;
                vs = vP;
                step = 1;
            }
            else
            {
                ks = k;
                vs = vC;
                step = 2;
            }
            c = vs + S * step;
            b = R.T[prv][ks & RM] << 1;
            ha = R.HA[prv][ks & RM];
            hb = R.HB[prv][ks & RM];
            if (fromedge && ks == kP)
            {
                const ChunkEdge& e = w.sm->edge[ch > 0 ? ch - 1 : 0];
                b = e.t << 1;
                ha = e.ha;
                hb = e.hb;
            }
            y = (c - k) >> 1;
            int y0 = y;
            y = PK ? snake_pk(FWD, apk, ag, bpk, bg, y, k, alen, blen, bend, aend)
           : snake(FWD, aseq0, bseq0, y, k, blen + 16, bend, aend);
            int L = FWD ? (y - y0) : (y0 - y);
            b = (L >= 61) ? ~0ull : ((b << L) | ((1ull << L) - 1ull));
            c = (y << 1) + k;
            const int kn = k < olow ? olow : (k > ohgh ? ohgh : k);
            na = R.NA[prv][kn & RM];
            nb = R.NB[prv][kn & RM];
            if (fromedge && kn == kP)  // a new band edge next to the chunk before
            {
                const ChunkEdge& e = w.sm->edge[ch > 0 ? ch - 1 : 0];
                na = e.na;
                nb = e.nb;
            }
            if (NP == 1 && ch + 1 < ring_of<RG>() / TW && lane == TW - 1 && ch + 1 < nch)
            {
                // the last lane saves its diagonal's previous values for the next chunk
                ChunkEdge& e = w.sm->edge[ch];
                e.v = vC;
                e.t = R.T[prv][k & RM];
                e.ha = R.HA[prv][k & RM];
                e.hb = R.HB[prv][k & RM];
                e.na = na;
                e.nb = nb;
            }
        }
        // trace points of A and B crossed by this extension (align.c:826-878)
        while (true)
        {
            bool needA = valid && (FWD ? (y + k >= na) : (y + k <= na));
            bool needB = valid && (FWD ? (y >= nb) : (y <= nb));
            if (!tany(w, needA || needB))
                break;
            bool cA = needA && (FWD ? (w.peb[ha].w < na) : (w.peb[ha].w > na));
            bool cB = needB && (FWD ? (w.peb[hb].w < nb) : (w.peb[hb].w > nb));
            unsigned ma = tballot(w, cA), mbb = tballot(w, cB);
            if (ma | mbb)
            {
                int base = npeb;
                npeb += __popc(ma) + __popc(mbb);
                if (npeb > w.pcap)
                {
                    if (lane == 0)
                        gd_fail(w.st, GD_ERR_PEBBLES, w.item, w.pcap);
                    w.err = 1;
                    wvars.hgh = hgh; wvars.low = low; wvars.dif = dif; wvars.more = more; wvars.aclip = aclip; wvars.bclip = bclip; wvars.besta = besta; wvars.lasta = lasta; wvars.npeb = npeb;
                    return true;
                }
                if (cA)
                {
                    int idx = base + __popc(ma & lt);
                    w.peb[idx] = make_int4(ha, k, dif, na);
                    ha = idx;
                }
                if (cB)
                {
                    int idx = base + __popc(ma) + __popc(mbb & lt);
                    w.peb[idx] = make_int4(hb, k, dif, nb);
                    hb = idx;
                }
            }
            if (needA)
                na += FWD ? TS : -TS;
            if (needB)
                nb += FWD ? TS : -TS;
        }
        if (FIRST)
            c0 = c;
        if (NP == 1)
            tsync(w);  // every lane of the chunk has read the ring
        if (valid)
        {
            R.V[cur][k & RM] = c;
            R.T[cur][k & RM] = b;
            R.HA[cur][k & RM] = ha;
            R.HB[cur][k & RM] = hb;
            R.NA[cur][k & RM] = na;
            R.NB[cur][k & RM] = nb;
        }

        // clip bookkeeping: bclip = first B-end in scan order, aclip = last A-end (a read end
        // is rare: one vote for both first)
        if (tany(w, valid && (bend || aend)))
        {
            unsigned bm = tballot(w, valid && bend);
            if (bm)
            {
                int pb = ch * TW + __ffs(bm) - 1;
                int kb = FWD ? hgh - pb : low + pb;
                bclip = FWD ? max(bclip, kb) : min(bclip, kb);
                more = 0;
            }
            unsigned amk = tballot(w, valid && aend);
            if (amk)
            {
                int pa = ch * TW + 31 - __clz(amk);
                aclip = FWD ? hgh - pa : low + pa;
                more = 0;
            }
        }

        // best point: every new maximum in scan order is a record (align.c:880-897).  The
        // last record is the first lane holding the chunk maximum; when it also passes the
        // PATH_AVE and trim-table tests it decides besta, lasta and trim at once, otherwise
        // the records are enumerated with a prefix-max scan.
        int wv = valid ? (FWD ? c : -c) : INT_MIN;
        int wbest = FWD ? besta : -besta;
        // the PATH_AVE and trim tests, in parallel with the reduction, of the lanes that can be
        // records (above the best so far): only records read them, so the others skip the
        // table lookups
        const bool q1 = valid && wv > wbest && __popcll(b & MASK61) >= PATH_AVE;
        const bool q2 = q1 && trim_ok(b, P.table, P.score);
        int wmax = tmax(w, wv);
        if (wmax > wbest)
        {
            int jm = __ffs(tballot(w, wv == wmax)) - 1;
            const unsigned mq1 = tballot(w, q1), mq2 = tballot(w, q2);
            besta = tshfl(w, c, jm);
            if (lane == jm)
                w.sm->besty = y;
            bool p1j = (mq1 >> jm) & 1;
            bool p2j = (mq2 >> jm) & 1;
            if (p1j)
                lasta = besta;
            if (p2j)
            {
                if (lane == jm)
                {
                    trim[0] = c;
                    trim[1] = y;
                    trim[2] = dif;
                    trim[3] = ha;
                    trim[4] = hb;
                }
            }
            else if ((mq1 & ((1u << jm) - 1u)) && (!p1j || (mq2 & ((1u << jm) - 1u))))
            {
                // only a q1 lane before jm can be a record that matters here (lasta when jm
                // itself fails q1; the trim point when a q2 lane precedes it): without one the
                // scan would change nothing, and that is most waves (on a 6 Mbp sample of the
                // 1 Mbp model, every forward wave whose maximum fails the trim test)
                // prefix max over the lanes before jm only (records lie before the maximum)
                int incl = wv;
                for (int o = 1; o < jm; o <<= 1)
                {
                    int t = tshfl_up(w, incl, o);
                    if (lane >= o)
                        incl = max(incl, t);
                }
                int excl = tshfl_up(w, incl, 1);
                if (lane == 0)
                    excl = INT_MIN;
                bool rec = valid && wv > max(wbest, excl) && lane < jm;
                unsigned mrec = tballot(w, rec);
                unsigned m1 = mrec & mq1;
                if (m1 && !p1j)
                    lasta = tshfl(w, c, 31 - __clz(m1));
                unsigned m2 = mrec & mq2;
                if (m2)
                {
                    int j2 = 31 - __clz(m2);
                    if (lane == j2)
                    {
                        trim[0] = c;
                        trim[1] = y;
                        trim[2] = dif;
                        trim[3] = ha;
                        trim[4] = hb;
                    }
                }
            }
            tsync(w);  // a later chunk's best point and trim point overwrite these
        }        return false;
    };
    if (chunk(0, std::true_type{}))
        return false;
#pragma unroll 1
    for (int ch = 1; ch < nch; ch++)
        if (chunk(ch, std::false_type{}))
            return false;
    tsync(w);
    clip_block();

    // drop diagonals more than WAVE_LAG behind the best (align.c:946-955), from this
    // wave's ring; k runs monotonically with the lane position
    {
        const int n = FWD ? besta - WAVE_LAG : besta + WAVE_LAG;
        const int hw = FWD ? hgh0 : low0;  // wave origin before clipping
        int nl = INT_MAX, nh = INT_MIN;
#pragma unroll
        for (int ch = 0; ch < ring_of<RG>() / TW; ch++)
        {
            if (ch >= nch)
                break;
            int p = ch * TW + lane;
            int k = FWD ? hw - p : hw + p;
            bool good = p < width && k >= low && k <= hgh;
            if (good)
            {
                const int v = ch == 0 ? c0 : R.V[cur][k & RM];
                good = FWD ? (v >= n) : (v <= n);
            }
            unsigned gm = tballot(w, good);
            if (gm)
            {
                int pf = ch * TW + __ffs(gm) - 1, pl = ch * TW + 31 - __clz(gm);
                int k1 = FWD ? hw - pf : hw + pf, k2 = FWD ? hw - pl : hw + pl;
                nl = min(nl, min(k1, k2));
                nh = max(nh, max(k1, k2));
            }
        }
        if (nh != INT_MIN)
        {
            hgh = nh;
            low = nl;
        }
        else
            hgh = low - 1;
    }
    w.cells += hgh - low + 1;
    wvars.hgh = hgh; wvars.low = low; wvars.dif = dif; wvars.more = more; wvars.aclip = aclip; wvars.bclip = bclip; wvars.besta = besta; wvars.lasta = lasta; wvars.npeb = npeb;
    return true;
}

// One wave of both teams of a duo warp at once: wave_step's work, for each team on its own
// diagonals, with every instruction run by all 32 lanes.  Every collective is whole-warp (a
// team reads its half of a ballot, shuffles within its 16 lanes, reduces by a 16-lane
// butterfly) and every branch around one is taken when either team needs it, with the
// team's own effects predicated, so that the two teams' waves share each issue slot instead
// of taking turns.  go: this team is in a wave.  Returns whether the team's wave loop goes on
// (false: it ended, or an error in w.err); a team that was not in a wave keeps its state.
__device__ __forceinline__ bool wave_step_duo(bool go, const bool FWD, WarpCtx<DUO>& w, WaveVars& wvars,
                                              const AlignParams& P, const uint32_t* apk, uint32_t ag,
                                              const uint32_t* bpk, uint32_t bg, int alen, int blen, int minp,
                                              int maxp)
{
    constexpr int RG = DUO;
    constexpr int TW = 16;
    constexpr int NR = ring_of<RG>();
    WaveSmem<RG>& R = w.sm->ws;
    const int lane = w.lane;
    const int tb = w.tbase;
    const int TS = P.tspace;
    const int S = FWD ? 1 : -1;
    const int VNONE = FWD ? -1 : INT_MAX;
    int* const trim = w.sm->trim;
    int* const clipm = w.sm->clipm;
    int hgh = wvars.hgh, low = wvars.low, dif = wvars.dif, more = wvars.more;
    int aclip = wvars.aclip, bclip = wvars.bclip, besta = wvars.besta, lasta = wvars.lasta, npeb = wvars.npeb;
    const int PATH_AVE = P.ave_path;
    auto half = [&](bool p) { return (__ballot_sync(GD_FULL, p) >> tb) & 0xffffu; };

    go = go && more && (FWD ? (lasta >= besta - TRIM_MLAG) : (lasta <= besta + TRIM_MLAG));
    if (!__any_sync(GD_FULL, go))
        return false;
    // widen the band by one each side (align.c:636-745); the checks of wave_step
    const int olow = low, ohgh = hgh;
    if (go && olow > ohgh)
    {
        if (lane == 0)
            gd_fail(w.st, GD_ERR_EMPTY_BAND, w.item, dif);
        w.err = 1;
        go = false;
    }
    if (go)
    {
        low -= 1;
        hgh += 1;
        if (low < minp)
            low += 1;
        if (hgh > maxp)
            hgh -= 1;
        dif += 1;
        if (dif > alen + blen + 2)
        {
            if (lane == 0)
                gd_fail(w.st, GD_ERR_EMPTY_BAND, w.item, dif);
            w.err = 1;
            go = false;
        }
    }
    int width = go ? hgh - low + 1 : 0;
    if (go && (unsigned)(width - 1) >= (unsigned)NR)
    {
        if (width > NR)
            w.err = 2;
        else
        {
            if (lane == 0)
                gd_fail(w.st, GD_ERR_EMPTY_BAND, w.item, width);
            w.err = 1;
        }
        go = false;
        width = 0;
    }
    const int nch = (width + TW - 1) / TW;
    const int nchw = max(nch, __shfl_xor_sync(GD_FULL, nch, 16));  // chunks of the wider team
    const int hgh0 = hgh, low0 = low;
    const int cur = dif & 1, prv = cur ^ 1;
    const unsigned lt = (1u << lane) - 1u;
    int c0 = 0;
#pragma unroll
    for (int ch = 0; ch < NR / TW; ch++)
    {
        if (ch >= nchw)
            break;
        const int p = ch * TW + lane;
        const bool valid = p < width;
        const int k = FWD ? hgh - p : low + p;
        int c = 0, y = 0, ha = 0, hb = 0, na = 0, nb = 0;
        unsigned long long b = 0;
        bool bend = false, aend = false;
        if (valid)
        {
            // choose the furthest of the three predecessors (align.c:748-797)
            const int kP = k + S, kN = k - S;
            int vP = (kP >= olow && kP <= ohgh) ? R.V[prv][kP & RM] : VNONE;
            int vC = (k >= olow && k <= ohgh) ? R.V[prv][k & RM] : VNONE;
            int vN = (kN >= olow && kN <= ohgh) ? R.V[prv][kN & RM] : VNONE;
            int wP = FWD ? vP : -vP, wC = FWD ? vC : -vC, wN = FWD ? vN : -vN;
            int ks, vs, step;
            if (wC < wN)
            {
                if (wN < wP)
                {
                    ks = k + S;
                    vs = vP;
                }
                else
                {
                    ks = k - S;
                    vs = vN;
                }
                step = 1;
            }
            else if (wC < wP)
            {
                ks = k + S;
                vs = vP;
                step = 1;
            }
            else
            {
                ks = k;
                vs = vC;
                step = 2;
            }
            c = vs + S * step;
            b = R.T[prv][ks & RM] << 1;
            ha = R.HA[prv][ks & RM];
            hb = R.HB[prv][ks & RM];
            y = (c - k) >> 1;
            const int y0 = y;
            y = snake_pk(FWD, apk, ag, bpk, bg, y, k, alen, blen, bend, aend);
            const int L = FWD ? (y - y0) : (y0 - y);
            b = (L >= 61) ? ~0ull : ((b << L) | ((1ull << L) - 1ull));
            c = (y << 1) + k;
            const int kn = k < olow ? olow : (k > ohgh ? ohgh : k);
            na = R.NA[prv][kn & RM];
            nb = R.NB[prv][kn & RM];
        }
        // trace points of A and B crossed by this extension (align.c:826-878)
        while (true)
        {
            const bool needA = valid && go && (FWD ? (y + k >= na) : (y + k <= na));
            const bool needB = valid && go && (FWD ? (y >= nb) : (y <= nb));
            if (!__any_sync(GD_FULL, needA || needB))
                break;
            const bool cA = needA && (FWD ? (w.peb[ha].w < na) : (w.peb[ha].w > na));
            const bool cB = needB && (FWD ? (w.peb[hb].w < nb) : (w.peb[hb].w > nb));
            const unsigned ma = half(cA), mbb = half(cB);
            if (ma | mbb)
            {
                const int base = npeb;
                npeb += __popc(ma) + __popc(mbb);
                if (npeb > w.pcap)
                {
                    if (lane == 0)
                        gd_fail(w.st, GD_ERR_PEBBLES, w.item, w.pcap);
                    w.err = 1;
                    go = false;  // the team stops here; its lanes only join the warp's collectives
                }
                else
                {
                    if (cA)
                    {
                        const int idx = base + __popc(ma & lt);
                        w.peb[idx] = make_int4(ha, k, dif, na);
                        ha = idx;
                    }
                    if (cB)
                    {
                        const int idx = base + __popc(ma) + __popc(mbb & lt);
                        w.peb[idx] = make_int4(hb, k, dif, nb);
                        hb = idx;
                    }
                }
            }
            if (needA)
                na += FWD ? TS : -TS;
            if (needB)
                nb += FWD ? TS : -TS;
        }
        const bool live = valid && go;
        if (ch == 0)
            c0 = c;
        if (live)
        {
            R.V[cur][k & RM] = c;
            R.T[cur][k & RM] = b;
            R.HA[cur][k & RM] = ha;
            R.HB[cur][k & RM] = hb;
            R.NA[cur][k & RM] = na;
            R.NB[cur][k & RM] = nb;
        }

        // clip bookkeeping: bclip = first B-end in scan order, aclip = last A-end
        const unsigned bm = half(live && bend);
        if (bm)
        {
            const int pb = ch * TW + __ffs(bm) - 1;
            const int kb = FWD ? hgh - pb : low + pb;
            bclip = FWD ? max(bclip, kb) : min(bclip, kb);
            more = 0;
        }
        const unsigned amk = half(live && aend);
        if (amk)
        {
            const int pa = ch * TW + 31 - __clz(amk);
            aclip = FWD ? hgh - pa : low + pa;
            more = 0;
        }

        // best point: the records of wave_step, per team
        const int wv = live ? (FWD ? c : -c) : INT_MIN;
        const int wbest = FWD ? besta : -besta;
        const bool q1 = live && wv > wbest && __popcll(b & MASK61) >= PATH_AVE;
        const bool q2 = q1 && trim_ok(b, P.table, P.score);
        int wmax = wv;
#pragma unroll
        for (int o = 8; o >= 1; o >>= 1)
            wmax = max(wmax, __shfl_xor_sync(GD_FULL, wmax, o, 16));
        const bool recT = go && wmax > wbest;
        if (__any_sync(GD_FULL, recT))
        {
            const int jm = __ffs(half(wv == wmax)) - 1;
            const unsigned mq1 = half(q1), mq2 = half(q2);
            const int cj = __shfl_sync(GD_FULL, c, jm, 16);
            const bool p1j = (mq1 >> jm) & 1;
            const bool p2j = (mq2 >> jm) & 1;
            if (recT)
            {
                besta = cj;
                if (lane == jm)
                    w.sm->besty = y;
                if (p1j)
                    lasta = besta;
                if (p2j && lane == jm)
                {
                    trim[0] = c;
                    trim[1] = y;
                    trim[2] = dif;
                    trim[3] = ha;
                    trim[4] = hb;
                }
            }
            // the records before jm, when the maximum itself does not settle the trim point
            const bool scan = recT && !p2j;
            if (__any_sync(GD_FULL, scan))
            {
                const int js = scan ? jm : 0;
                const int jmw = max(js, __shfl_xor_sync(GD_FULL, js, 16));
                int incl = wv;
                for (int o = 1; o < jmw; o <<= 1)  // lanes at or past a team's jm are not read
                {
                    const int t = __shfl_up_sync(GD_FULL, incl, o, 16);
                    if (lane >= o)
                        incl = max(incl, t);
                }
                int excl = __shfl_up_sync(GD_FULL, incl, 1, 16);
                if (lane == 0)
                    excl = INT_MIN;
                const bool rec = scan && live && wv > max(wbest, excl) && lane < jm;
                const unsigned mrec = half(rec);
                const unsigned m1 = mrec & mq1;
                const int c1 = __shfl_sync(GD_FULL, c, m1 ? 31 - __clz(m1) : 0, 16);
                if (scan && m1 && !p1j)
                    lasta = c1;
                const unsigned m2 = mrec & mq2;
                if (scan && m2)
                {
                    const int j2 = 31 - __clz(m2);
                    if (lane == j2)
                    {
                        trim[0] = c;
                        trim[1] = y;
                        trim[2] = dif;
                        trim[3] = ha;
                        trim[4] = hb;
                    }
                }
            }
            __syncwarp();  // a later chunk's best point and trim point overwrite these
        }
    }
    __syncwarp();
    // clip_block of wave_step (lane 0 alone writes and reads the clip fallback)
    if (go && !more)
    {
        const int besty = w.sm->besty;
        if (FWD ? (besty < blen && besta - besty < alen) : (besty > 0 && besta - besty > 0))
            more = 1;
        if (FWD ? (hgh >= aclip) : (low <= aclip))
        {
            if (FWD)
                hgh = aclip - 1;
            else
                low = aclip + 1;
            const int Mc = __popcll(R.T[dif & 1][aclip & RM] & MASK61);
            if (lane == 0 && clipm[0] <= Mc)
            {
                clipm[0] = Mc;
                clipm[1] = R.V[dif & 1][aclip & RM];
                clipm[2] = (clipm[1] - aclip) / 2;
                clipm[3] = dif;
                clipm[4] = R.HA[dif & 1][aclip & RM];
                clipm[5] = R.HB[dif & 1][aclip & RM];
            }
        }
        if (FWD ? (low <= bclip) : (hgh >= bclip))
        {
            if (FWD)
                low = bclip + 1;
            else
                hgh = bclip - 1;
            const int Mc = __popcll(R.T[dif & 1][bclip & RM] & MASK61);
            if (lane == 0 && clipm[0] <= Mc)
            {
                clipm[0] = Mc;
                clipm[1] = R.V[dif & 1][bclip & RM];
                clipm[2] = (clipm[1] - bclip) / 2;
                clipm[3] = dif;
                clipm[4] = R.HA[dif & 1][bclip & RM];
                clipm[5] = R.HB[dif & 1][bclip & RM];
            }
        }
        aclip = FWD ? INT_MAX : -INT_MAX;
        bclip = FWD ? -INT_MAX : INT_MAX;
    }

    // drop diagonals more than WAVE_LAG behind the best (align.c:946-955)
    {
        const int n = FWD ? besta - WAVE_LAG : besta + WAVE_LAG;
        const int hw = FWD ? hgh0 : low0;
        int nl = INT_MAX, nh = INT_MIN;
#pragma unroll
        for (int ch = 0; ch < NR / TW; ch++)
        {
            if (ch >= nchw)
                break;
            const int p = ch * TW + lane;
            const int k = FWD ? hw - p : hw + p;
            bool good = go && p < width && k >= low && k <= hgh;
            if (good)
            {
                const int v = ch == 0 ? c0 : R.V[cur][k & RM];
                good = FWD ? (v >= n) : (v <= n);
            }
            const unsigned gm = half(good);
            if (gm)
            {
                const int pf = ch * TW + __ffs(gm) - 1, pl = ch * TW + 31 - __clz(gm);
                const int k1 = FWD ? hw - pf : hw + pf, k2 = FWD ? hw - pl : hw + pl;
                nl = min(nl, min(k1, k2));
                nh = max(nh, max(k1, k2));
            }
        }
        if (go)
        {
            if (nh != INT_MIN)
            {
                hgh = nh;
                low = nl;
            }
            else
                hgh = low - 1;
            w.cells += hgh - low + 1;
        }
    }
    wvars.hgh = hgh;
    wvars.low = low;
    wvars.dif = dif;
    wvars.more = more;
    wvars.aclip = aclip;
    wvars.bclip = bclip;
    wvars.besta = besta;
    wvars.lasta = lasta;
    wvars.npeb = npeb;
    return go;
}

template <int RG, bool PK>
__device__ __forceinline__ void wave_end(const bool FWD, WarpCtx<RG>& w, WaveVars& wvars, const AlignParams& P, const uint8_t* aseq0, const uint8_t* bseq0,
    const uint32_t* apk, uint32_t ag, const uint32_t* bpk, uint32_t bg, int alen, int blen, int comp, LAPath* apath, LAPath* bpath, int* mind, int mida,
    uint16_t* atrace, uint16_t* btrace)
{
    WaveSmem<RG>& R = w.sm->ws;
    const int lane = w.lane;
    const int TS = P.tspace;
    const int S = FWD ? 1 : -1;
    const int VNONE = FWD ? -1 : INT_MAX;
    const int boff = comp ? blen % TS : 0;
    int* const trim = w.sm->trim;
    int* const clipm = w.sm->clipm;
    const uint8_t* as = FWD ? aseq0 : aseq0 - 1;
    const uint8_t* bs = FWD ? bseq0 : bseq0 - 1;
    (void)S; (void)VNONE; (void)boff; (void)as; (void)bs; (void)trim; (void)clipm; (void)R; (void)TS; (void)lane;
    int low = wvars.low;
    // ---- trace points of both paths from the pebble chains (align.c:970-1106, 1710-1902)
    tsync(w);
    if (lane == 0)
    {
        int4* cells = w.peb;
        int atlen = 0, btlen = 0, trimx, a, b, k, h, d, e;
        int trima = trim[0], trimy = trim[1], trimd = trim[2], trimha = trim[3], trimhb = trim[4];
        if (clipm[0] >= 0)
        {
            trimx = clipm[1] - clipm[2];
            trimy = clipm[2];
            trimd = clipm[3];
            trimha = clipm[4];
            trimhb = clipm[5];
        }
        else
            trimx = trima - trimy;

        a = -1;
        for (h = trimha; h >= 0; h = b)
        {
            b = cells[h].x;
            cells[h].x = a;
            a = h;
        }
        h = a;
        if (FWD)
        {
            k = cells[h].y;
            b = (mida - k) / 2;
            e = 0;
            for (h = cells[h].x; h >= 0; h = cells[h].x)
            {
                k = cells[h].y;
                a = cells[h].w - k;
                d = cells[h].z;
                atrace[atlen++] = (uint16_t)(d - e);
                atrace[atlen++] = (uint16_t)(a - b);
                b = a;
                e = d;
            }
            if (b + k != trimx)
            {
                atrace[atlen++] = (uint16_t)(trimd - e);
                atrace[atlen++] = (uint16_t)(trimy - b);
            }
            else if (b != trimy)
            {
                atrace[atlen - 1] = (uint16_t)(atrace[atlen - 1] + (trimy - b));
                atrace[atlen - 2] = (uint16_t)(atrace[atlen - 2] + (trimd - e));
            }
        }
        else
        {
            k = cells[h].y;
            b = cells[h].w - k;
            e = 0;
            if ((b + k) % TS != 0)
            {
                h = cells[h].x;
                if (h < 0)
                {
                    a = trimy;
                    d = trimd;
                }
                else
                {
                    k = cells[h].y;
                    a = cells[h].w - k;
                    d = cells[h].z;
                }
                if (apath->tlen == 0)
                {
                    atrace[--atlen] = (uint16_t)(b - a);
                    atrace[--atlen] = (uint16_t)(d - e);
                }
                else
                {
                    atrace[1] = (uint16_t)(atrace[1] + (b - a));
                    atrace[0] = (uint16_t)(atrace[0] + (d - e));
                }
                b = a;
                e = d;
            }
            if (h >= 0)
            {
                for (h = cells[h].x; h >= 0; h = cells[h].x)
                {
                    k = cells[h].y;
                    a = cells[h].w - k;
                    atrace[--atlen] = (uint16_t)(b - a);
                    d = cells[h].z;
                    atrace[--atlen] = (uint16_t)(d - e);
                    b = a;
                    e = d;
                }
                if (b + k != trimx)
                {
                    atrace[--atlen] = (uint16_t)(b - trimy);
                    atrace[--atlen] = (uint16_t)(trimd - e);
                }
                else if (b != trimy)
                {
                    atrace[atlen + 1] = (uint16_t)(atrace[atlen + 1] + (b - trimy));
                    atrace[atlen] = (uint16_t)(atrace[atlen] + (trimd - e));
                }
            }
        }

        a = -1;
        for (h = trimhb; h >= 0; h = b)
        {
            b = cells[h].x;
            cells[h].x = a;
            a = h;
        }
        h = a;
        if (FWD)
        {
            k = cells[h].y;
            b = (mida + k) / 2;
            e = 0;
            low = k;
            for (h = cells[h].x; h >= 0; h = cells[h].x)
            {
                k = cells[h].y;
                a = cells[h].w + k;
                d = cells[h].z;
                btrace[btlen++] = (uint16_t)(d - e);
                btrace[btlen++] = (uint16_t)(a - b);
                b = a;
                e = d;
            }
            if (b - k != trimy)
            {
                btrace[btlen++] = (uint16_t)(trimd - e);
                btrace[btlen++] = (uint16_t)(trimx - b);
            }
            else if (b != trimx)
            {
                btrace[btlen - 1] = (uint16_t)(btrace[btlen - 1] + (trimx - b));
                btrace[btlen - 2] = (uint16_t)(btrace[btlen - 2] + (trimd - e));
            }
            apath->aepos = trimx;
            apath->bepos = trimy;
            apath->diffs = trimd;
            apath->tlen = atlen;
            apath->toff = (int)(atrace - w.pts);
            if (comp)
            {
                bpath->abpos = blen - apath->bepos;
                bpath->bbpos = alen - apath->aepos;
            }
            else
            {
                bpath->aepos = apath->bepos;
                bpath->bepos = apath->aepos;
            }
            bpath->diffs = trimd;
            bpath->tlen = btlen;
            bpath->toff = (int)(btrace - w.pts);
            w.sm->span_lo = low;
        }
        else
        {
            k = cells[h].y;
            b = cells[h].w + k;
            e = 0;
            if ((b - k) % TS != boff)
            {
                h = cells[h].x;
                if (h < 0)
                {
                    a = trimx;
                    d = trimd;
                }
                else
                {
                    k = cells[h].y;
                    a = cells[h].w + k;
                    d = cells[h].z;
                }
                if (bpath->tlen == 0)
                {
                    btrace[--btlen] = (uint16_t)(b - a);
                    btrace[--btlen] = (uint16_t)(b - a);  // sic: align.c:1861-1862 stores b-a twice
                }
                else
                {
                    btrace[1] = (uint16_t)(btrace[1] + (b - a));
                    btrace[0] = (uint16_t)(btrace[0] + (d - e));
                }
                b = a;
                e = d;
            }
            if (h >= 0)
            {
                for (h = cells[h].x; h >= 0; h = cells[h].x)
                {
                    k = cells[h].y;
                    a = cells[h].w + k;
                    btrace[--btlen] = (uint16_t)(b - a);
                    d = cells[h].z;
                    btrace[--btlen] = (uint16_t)(d - e);
                    b = a;
                    e = d;
                }
                if (b - k != trimy)
                {
                    btrace[--btlen] = (uint16_t)(b - trimx);
                    btrace[--btlen] = (uint16_t)(trimd - e);
                }
                else if (b != trimx)
                {
                    btrace[btlen + 1] = (uint16_t)(btrace[btlen + 1] + (b - trimx));
                    btrace[btlen] = (uint16_t)(btrace[btlen] + (trimd - e));
                }
            }
            apath->abpos = trimx;
            apath->bbpos = trimy;
            apath->diffs = apath->diffs + trimd;
            apath->tlen = apath->tlen - atlen;
            apath->toff = (int)(atrace + atlen - w.pts);
            if (comp)
            {
                bpath->aepos = blen - apath->bbpos;
                bpath->bepos = alen - apath->abpos;
            }
            else
            {
                bpath->abpos = apath->bbpos;
                bpath->bbpos = apath->abpos;
            }
            bpath->diffs = bpath->diffs + trimd;
            bpath->tlen = bpath->tlen - btlen;
            bpath->toff = (int)(btrace + btlen - w.pts);
        }
    }
    tsync(w);
    if (FWD)
        *mind = w.sm->span_lo;
}

template <bool FWD, int RG, bool PK>
__device__ void wave(WarpCtx<RG>& w, const AlignParams& P, const uint8_t* aseq0, const uint8_t* bseq0,
                     const uint32_t* apk, uint32_t ag, const uint32_t* bpk, uint32_t bg, int alen, int blen,
                     int comp, LAPath* apath, LAPath* bpath, int* mind, int maxd, int mida, int minp, int maxp,
                     uint16_t* atrace, uint16_t* btrace)
{
    WaveVars v;
    wave_begin<RG, PK>(FWD, w, v, P, aseq0, bseq0, apk, ag, bpk, bg, alen, blen, comp, *mind, maxd, mida);
    if (w.err)
        return;
    while (wave_step<RG, PK>(FWD, w, v, P, aseq0, bseq0, apk, ag, bpk, bg, alen, blen, comp, minp, maxp))
        ;
    if (w.err)
        return;
    wave_end<RG, PK>(FWD, w, v, P, aseq0, bseq0, apk, ag, bpk, bg, alen, blen, comp, apath, bpath, mind, mida, atrace,
                          btrace);
}

// Local_Alignment from one seed (diag, anti) with lbord = hbord = -1 (align.c:1922-2060).
template <int RG, bool PK>
__device__ void local_alignment(WarpCtx<RG>& w, const AlignParams& P, const uint8_t* aseq, const uint8_t* bseq,
                                const uint32_t* apk, uint32_t ag, const uint32_t* bpk, uint32_t bg, int alen,
                                int blen, int comp, int diag, int anti)
{
    const int TS = P.tspace;
    int maxtp = 2 * (max(alen, blen) / TS + 2);
    if (4 * maxtp + 16 > w.ptscap)
    {
        if (w.lane == 0)
            gd_fail(w.st, GD_ERR_TRACE, w.item, maxtp);
        w.err = 1;
        return;
    }
    uint16_t* atrace = w.pts + maxtp;
    uint16_t* btrace = atrace + 2 * maxtp;
    LAPath* ap = &w.sm->ap;
    LAPath* bp = &w.sm->bp;
    int low = diag, hgh = diag;
    bool selfie = (aseq == bseq);
    int minp = (selfie && low >= 0) ? 1 : -INT_MAX;
    int maxp = (selfie && hgh <= 0) ? -1 : INT_MAX;
    if (w.lane == 0)
    {
        ap->tlen = bp->tlen = 0;
        ap->diffs = bp->diffs = 0;
    }
    tsync(w);
    wave<true, RG, PK>(w, P, aseq, bseq, apk, ag, bpk, bg, alen, blen, comp, ap, bp, &low, hgh, anti, minp, maxp,
                       atrace, btrace);
    if (w.err)
        return;
    wave<false, RG, PK>(w, P, aseq, bseq, apk, ag, bpk, bg, alen, blen, comp, ap, bp, &low, low, anti, minp, maxp,
                        atrace, btrace);
    if (w.err)
        return;
    if (comp && w.lane == 0)
    {
        uint16_t* tr = w.pts + bp->toff;
        int i = bp->tlen - 2, j = 0;
        while (j < i)
        {
            uint16_t t = tr[i];
            tr[i] = tr[j];
            tr[j] = t;
            t = tr[i + 1];
            tr[i + 1] = tr[j + 1];
            tr[j + 1] = t;
            i -= 2;
            j += 2;
        }
    }
    tsync(w);
}

// ------------------------------------------------------------------------------------------
// per-pair redundancy handling (Entwine / Fusion / Handle_Redundancies, filter.c:1249-1566),
// lane 0 only: O(n^2) over the few paths of one pair.
// ------------------------------------------------------------------------------------------

struct PairBuf
{
    MPath* am;
    MPath* bm;
    uint16_t* tb;
    int ttop, tcap;
    int err;
};

// Entwine (filter.c:1249-1342); d2: daligner2's version (dalign2/filter.c:1707-1825), which
// also compares the B coordinates at a common start and a common end point
__device__ int entwine(const MPath* jpath, const MPath* kpath, const uint16_t* tb, int TS, int* where, bool d2 = false)
{
    int ac, b2, y2, ae, i, j, k, den = 0, min = 10000;
    const uint16_t* ktrace = tb + kpath->toff;
    const uint16_t* jtrace = tb + jpath->toff;
    y2 = jpath->bbpos;
    j = jpath->abpos / TS;
    b2 = kpath->bbpos;
    k = kpath->abpos / TS;
    if (d2 && jpath->abpos == kpath->abpos)
    {
        min = abs(y2 - b2);
        if (min == 0)
            *where = kpath->abpos;
    }
    if (j < k)
    {
        ac = k * TS;
        j = 1 + 2 * (k - j);
        k = 1;
        for (i = 1; i < j; i += 2)
            y2 += jtrace[i];
    }
    else
    {
        ac = j * TS;
        k = 1 + 2 * (j - k);
        j = 1;
        for (i = 1; i < k; i += 2)
            b2 += ktrace[i];
    }
    ae = jpath->aepos;
    if (ae > kpath->aepos)
        ae = kpath->aepos;
    while (1)
    {
        ac += TS;
        if (ac >= ae)
            break;
        y2 += jtrace[j];
        b2 += ktrace[k];
        j += 2;
        k += 2;
        i = abs(y2 - b2);
        if (i <= min)
        {
            min = i;
            if (i == 0)
                *where = ac;
        }
        den += 1;
    }
    if (d2 && jpath->aepos == kpath->aepos)
    {
        i = abs(jpath->bepos - kpath->bepos);
        if (i <= min)
        {
            min = i;
            if (i == 0)
                *where = kpath->aepos;
        }
    }
    return den == 0 ? -1 : min;
}

__device__ void fusion(MPath* p1, int ap, const MPath* p2, PairBuf& pb, int TS)
{
    int k1 = 2 * ((ap / TS) - (p1->abpos / TS));
    int k2 = 2 * ((ap / TS) - (p2->abpos / TS));
    int len = k1 + (p2->tlen - k2), diff = 0, k;
    if (pb.ttop + len > pb.tcap)
    {
        pb.err = 1;
        return;
    }
    int base = pb.ttop;
    pb.ttop += len;
    uint16_t* trace = pb.tb + base;
    len = 0;
    if (k1 > 0)
    {
        const uint16_t* t = pb.tb + p1->toff;
        for (k = 0; k < k1; k += 2)
        {
            trace[len++] = t[k];
            trace[len++] = t[k + 1];
            diff += t[k];
        }
    }
    if (k2 < p2->tlen)
    {
        const uint16_t* t = pb.tb + p2->toff;
        for (k = k2; k < p2->tlen; k += 2)
        {
            trace[len++] = t[k];
            trace[len++] = t[k + 1];
            diff += t[k];
        }
    }
    p1->aepos = p2->aepos;
    p1->bepos = p2->bepos;
    p1->diffs = diff;
    p1->toff = base;
    p1->tlen = len;
}

__device__ int handle_redundancies(MPath* amatch, int novls, MPath* bmatch, PairBuf& pb, int TS, int comp)
{
    int j, k, no = 0, dist, awhen = 0, bwhen = 0;
    bool hasB = (bmatch != nullptr);
    for (j = 1; j < novls; j++)
    {
        MPath* jpath = amatch + j;
        for (k = no; k >= 0; k--)
        {
            MPath* kpath = amatch + k;
            if (jpath->abpos < kpath->abpos)
            {
                if (kpath->abpos <= jpath->aepos && kpath->bbpos <= jpath->bepos)
                {
                    dist = entwine(jpath, kpath, pb.tb, TS, &awhen);
                    if (dist == 0)
                    {
                        if (kpath->aepos > jpath->aepos)
                        {
                            if (hasB)
                            {
                                if (comp)
                                {
                                    dist = entwine(bmatch + k, bmatch + j, pb.tb, TS, &bwhen);
                                    if (dist != 0)
                                        continue;
                                    fusion(jpath, awhen, kpath, pb, TS);
                                    amatch[k] = *jpath;
                                    fusion(bmatch + k, bwhen, bmatch + j, pb, TS);
                                }
                                else
                                {
                                    dist = entwine(bmatch + j, bmatch + k, pb.tb, TS, &bwhen);
                                    if (dist != 0)
                                        continue;
                                    fusion(jpath, awhen, kpath, pb, TS);
                                    amatch[k] = *jpath;
                                    fusion(bmatch + j, bwhen, bmatch + k, pb, TS);
                                    bmatch[k] = bmatch[j];
                                }
                            }
                            else
                            {
                                fusion(jpath, awhen, kpath, pb, TS);
                                amatch[k] = *jpath;
                            }
                        }
                        else
                        {
                            amatch[k] = *jpath;
                            if (hasB)
                                bmatch[k] = bmatch[j];
                        }
                        break;
                    }
                }
            }
            else
            {
                if (jpath->abpos <= kpath->aepos && jpath->bbpos <= kpath->bepos)
                {
                    dist = entwine(kpath, jpath, pb.tb, TS, &awhen);
                    if (dist == 0)
                    {
                        if (kpath->abpos == jpath->abpos)
                        {
                            if (kpath->aepos < jpath->aepos)
                            {
                                amatch[k] = *jpath;
                                if (hasB)
                                    bmatch[k] = bmatch[j];
                            }
                        }
                        else if (jpath->aepos > kpath->aepos)
                        {
                            if (hasB)
                            {
                                if (comp)
                                {
                                    dist = entwine(bmatch + j, bmatch + k, pb.tb, TS, &bwhen);
                                    if (dist != 0)
                                        continue;
                                    fusion(kpath, awhen, jpath, pb, TS);
                                    fusion(bmatch + j, bwhen, bmatch + k, pb, TS);
                                    bmatch[k] = bmatch[j];
                                }
                                else
                                {
                                    dist = entwine(bmatch + k, bmatch + j, pb.tb, TS, &bwhen);
                                    if (dist != 0)
                                        continue;
                                    fusion(kpath, awhen, jpath, pb, TS);
                                    fusion(bmatch + k, bwhen, bmatch + j, pb, TS);
                                }
                            }
                            else
                                fusion(kpath, awhen, jpath, pb, TS);
                        }
                        break;
                    }
                }
            }
        }
        if (k < 0)
        {
            no += 1;
            amatch[no] = *jpath;
            if (hasB)
                bmatch[no] = bmatch[j];
        }
    }
    return no + 1;
}

// ---- daligner2 bridging (DO_BRIDGING, dalign2/filter.c:1479-1705, 2124-2262), lane 0 ------

// The bridge scratch of one warp and the sequences of its pair.
struct BridgeCtx
{
    const uint8_t *aseq, *bseq;  // the pair's align: A, and B complemented for a complement pair
    int alen, blen;
    int* vec;                    // Compute_Alignment's wave vectors
    int vcap;
    uint16_t* tr;                // the bridge's trace
    int tcap;
    int need;                    // > 0: ints of vec (or values of tr) a bridge needed but did not have
};

// split_nd (dalign2/align.c:4355-4523): bidirectional O(nd) waves over A[0,M) x B[0,N) until
// they meet; the edit distance and the meeting point (x, y)
__device__ int d2_split_nd(const uint8_t* A, int M, const uint8_t* B, int N, int* VF, int* VB, int* px, int* py)
{
    int x, y, D, flow, blow, bhgh;
    const uint8_t* a;
    y = 0;
    if (N < M)
        while (y < N && B[y] == A[y])
            y += 1;
    else
    {
        while (y < M && B[y] == A[y])
            y += 1;
        if (y >= M && N == M)
        {
            *px = *py = M;
            return 0;
        }
    }
    flow = 0;
    VF[0] = y;
    VF[-1] = -2;
    x = N - M;
    a = A - x;
    y = N - 1;
    if (N > M)
        while (y >= x && B[y] == a[y])
            y -= 1;
    else
        while (y >= 0 && B[y] == a[y])
            y -= 1;
    blow = bhgh = -x;
    VB += x;
    VB[blow] = y;
    VB[blow - 1] = N + 1;
    for (D = 1;; D += 1)
    {
        int k, r, am, ac, ap;
        flow -= 1;
        am = ac = VF[flow - 1] = -2;
        a = A + D;
        x = M - D;
        for (k = D; k >= flow; k--)
        {
            ap = ac;
            ac = am + 1;
            am = VF[k - 1];
            if (ac < am)
                y = (ap < am) ? am : ap;
            else
                y = (ap < ac) ? ac : ap;
            if (blow <= k && k <= bhgh)
            {
                r = VB[k];
                if (y > r)
                {
                    D = (D << 1) - 1;
                    y = (ap > r) ? ap : ((ac > r) ? ac : r + 1);
                    *px = k + y;
                    *py = y;
                    return D;
                }
            }
            if (N < x)
                while (y < N && B[y] == a[y])
                    y += 1;
            else
                while (y < x && B[y] == a[y])
                    y += 1;
            VF[k] = y;
            a -= 1;
            x += 1;
        }
        bhgh += 1;
        blow -= 1;
        am = ac = VB[blow - 1] = N + 1;
        a = A + bhgh;
        x = -bhgh;
        for (k = bhgh; k >= blow; k--)
        {
            ap = ac + 1;
            ac = am;
            am = VB[k - 1];
            if (ac > am)
                y = (ap > am) ? am : ap;
            else
                y = (ap > ac) ? ac : ap;
            if (flow <= k && k <= D)
            {
                r = VF[k];
                if (y <= r)
                {
                    D = (D << 1);
                    y = (ap <= r) ? ap : ((ac <= r) ? ac : r);
                    *px = k + y;
                    *py = y;
                    return D;
                }
            }
            y -= 1;
            if (x > 0)
                while (y >= x && B[y] == a[y])
                    y -= 1;
            else
                while (y >= 0 && B[y] == a[y])
                    y -= 1;
            VB[k] = y;
            a -= 1;
            x += 1;
        }
    }
}

// adds s bases of one side, from absolute A position u on, to the trace intervals they fall in
__device__ __forceinline__ void d2_spread(uint16_t* Trace, int u, int s, int tspace, int side)
{
    int v = u / tspace;
    u = (v + 1) * tspace - u;
    for (v <<= 1; s > 0; s -= u, u = tspace)
    {
        if (u > s)
            u = s;
        Trace[v + side] += u;
        v += 2;
    }
}

// trace_nd (dalign2/align.c:4525-4679) without recursion: every update is an addition to a
// trace interval, so the pieces go on a small stack in any order.  Returns the top-level
// distance, or -1 if the stack ran out.
__device__ int d2_trace_nd(const uint8_t* Aabs, int a0, int M0, const uint8_t* B0, int N0, uint16_t* Trace, int* VF,
                           int* VB, int tspace)
{
    struct Piece
    {
        int a, M, N;
        const uint8_t* B;
    };
    Piece stk[48];
    int top = 0, D0 = -1;
    stk[top++] = Piece{a0, M0, N0, B0};
    while (top > 0)
    {
        const Piece pc = stk[--top];
        const uint8_t* A = Aabs + pc.a;
        const int M = pc.M, N = pc.N;
        int x, y, D, s;
        if (M <= 0)
        {
            y = ((pc.a / tspace) << 1);
            Trace[y] += N;
            Trace[y + 1] += N;
            D = N;
        }
        else if (N <= 0)
        {
            x = pc.a;
            y = x / tspace;
            x = (y + 1) * tspace - x;
            y <<= 1;
            for (s = M; s > 0; s -= x, x = tspace)
            {
                if (x > s)
                    x = s;
                Trace[y] += x;
                y += 2;
            }
            D = M;
        }
        else
        {
            D = d2_split_nd(A, M, pc.B, N, VF, VB, &x, &y);
            if (D > 1)
            {
                s = pc.a;
                if ((s / tspace + 1) * tspace - s >= x)
                {
                    s = ((s / tspace) << 1);
                    Trace[s] += (D + 1) / 2;
                    Trace[s + 1] += y;
                }
                else
                {
                    if (top >= 48)
                        return -1;
                    stk[top++] = Piece{pc.a, x, y, pc.B};
                }
                s = pc.a + x;
                if ((s / tspace + 1) * tspace - s >= M - x)
                {
                    s = ((s / tspace) << 1);
                    Trace[s] += D / 2;
                    Trace[s + 1] += N - y;
                }
                else
                {
                    if (top >= 48)
                        return -1;
                    stk[top++] = Piece{pc.a + x, M - x, N - y, pc.B + y};
                }
            }
            else
            {
                s = (D == 0 || M < N) ? x : x - 1;
                if (s > 0)
                    d2_spread(Trace, pc.a, s, tspace, 1);
                if (D != 0)
                {
                    y = (((M < N) ? pc.a + x : pc.a + (x - 1)) / tspace) << 1;
                    Trace[y] += 1;
                    if (M <= N)
                        Trace[y + 1] += 1;
                    s = M - x;
                    if (s > 0)
                        d2_spread(Trace, pc.a + x, s, tspace, 1);
                }
            }
        }
        if (D0 < 0)
            D0 = D;
    }
    return D0;
}

// A bridge path: coordinates, diffs and its trace in the warp's bridge buffer.
struct BPath
{
    int abpos, bbpos, aepos, bepos, diffs, tlen;
};

// Compute_Alignment(align, work, DIFF_TRACE, tspace) (dalign2/align.c:4762-4913) for the box of
// p over aseq (its absolute base) and bseq; false if the scratch is too small (bc.need set)
__device__ bool d2_compute_alignment(const uint8_t* aseq, const uint8_t* bseq, BPath* p, int tspace, BridgeCtx& bc)
{
    const int asub = p->aepos - p->abpos, bsub = p->bepos - p->bbpos;
    const int n = 2 * (((p->aepos + (tspace - 1)) / tspace - p->abpos / tspace) + 1);
    const int m = asub > bsub ? asub : bsub;
    if (4 * m + 6 > bc.vcap || n > bc.tcap)
    {
        bc.need = max(4 * m + 6 > bc.vcap ? 4 * m + 6 : 0, n > bc.tcap ? n : 0);
        return false;
    }
    int* VF = bc.vec + (m + 1);
    int* VB = VF + (2 * m + 3);
    uint16_t* strace = bc.tr;
    for (int i = 0; i < n; i++)
        strace[i] = 0;
    uint16_t* Trace = strace - 2 * (p->abpos / tspace);
    const int d = d2_trace_nd(aseq, p->abpos, asub, bseq + p->bbpos, bsub, Trace, VF, VB, tspace);
    if (d < 0)
    {
        bc.need = 1;  // the piece stack ran out: reported like a scratch shortage
        return false;
    }
    p->diffs = d;
    if (strace[n - 1] != 0)
    {
        strace[n - 3] += strace[n - 1];
        strace[n - 4] += strace[n - 2];
    }
    p->tlen = n - 2;
    return true;
}

// MapToTPAbove / MapToTPBelow (dalign2/filter.c:1481-1563)
__device__ int d2_map_tp_above(const MPath* path, int* x, bool isA, const uint16_t* tb, int TS)
{
    const uint16_t* trace = tb + path->toff;
    int a = (path->abpos / TS) * TS, b = path->bbpos;
    for (int i = 1; i < path->tlen; i += 2)
    {
        a += TS;
        b += trace[i];
        if (a > path->aepos)
            a = path->aepos;
        if (isA ? a >= *x : b >= *x)
            break;
    }
    const int r = isA ? b : a;
    *x = isA ? a : b;
    return r;
}

__device__ int d2_map_tp_below(const MPath* path, int* x, bool isA, const uint16_t* tb, int TS)
{
    const uint16_t* trace = tb + path->toff;
    int a = ((path->aepos + (TS - 1)) / TS) * TS, b = path->bepos;
    for (int i = path->tlen - 1; i >= 0; i -= 2)
    {
        a -= TS;
        b -= trace[i];
        if (a < path->abpos)
            a = path->abpos;
        if (isA ? a <= *x : b <= *x)
            break;
    }
    const int r = isA ? b : a;
    *x = isA ? a : b;
    return r;
}

// Compute_Bridge_Path (dalign2/filter.c:1579-1705): the box from two trace points before
// path2's start to two after path1's end, aligned afresh with trace points; with comp in the
// complemented frame, shifted so its trace points fall on multiples of the spacing
__device__ bool d2_bridge_path(const MPath* path1, const MPath* path2, const uint8_t* aseq, const uint8_t* bseq,
                               int alen, int blen, int comp, int aovl, int bovl, const uint16_t* tb, int TS, BPath* ap,
                               BridgeCtx& bc)
{
    int ain, aout, bin, bout, boff = 0, p;
    if (bovl > aovl)
    {
        bin = path2->bbpos;
        bout = path1->bepos;
        ain = d2_map_tp_below(path1, &bin, false, tb, TS);
        aout = d2_map_tp_above(path2, &bout, false, tb, TS);
    }
    else
    {
        ain = path2->abpos;
        aout = path1->aepos;
        bin = d2_map_tp_below(path1, &ain, true, tb, TS);
        bout = d2_map_tp_above(path2, &aout, true, tb, TS);
    }
    ap->abpos = ain - 2 * TS;
    ap->aepos = aout + 2 * TS;
    ap->bbpos = d2_map_tp_below(path1, &ap->abpos, true, tb, TS);
    ap->bepos = d2_map_tp_above(path2, &ap->aepos, true, tb, TS);
    const uint8_t* A = aseq;
    if (comp)
    {
        boff = TS - ap->aepos % TS;
        p = alen - ap->abpos;
        ap->abpos = alen - ap->aepos;
        ap->aepos = p;
        p = blen - ap->bbpos;
        ap->bbpos = blen - ap->bepos;
        ap->bepos = p;
        boff = boff - ap->abpos % TS;
        A -= boff;
        ap->abpos += boff;
        ap->aepos += boff;
    }
    if (!d2_compute_alignment(A, bseq, ap, TS, bc))
        return false;
    if (comp)
    {
        uint16_t* trk = bc.tr;
        int j = ap->tlen - 2, i = 0;
        while (i < j)
        {
            uint16_t t = trk[i];
            trk[i] = trk[j];
            trk[j] = t;
            t = trk[i + 1];
            trk[i + 1] = trk[j + 1];
            trk[j + 1] = t;
            i += 2;
            j -= 2;
        }
        ap->abpos -= boff;
        ap->aepos -= boff;
        p = alen - ap->abpos;
        ap->abpos = alen - ap->aepos;
        ap->aepos = p;
        p = blen - ap->bbpos;
        ap->bbpos = blen - ap->bepos;
        ap->bepos = p;
    }
    return true;
}

// Check_Bridge (dalign2/filter.c:1565-1577)
__device__ bool d2_check_bridge(const BPath* p, const BridgeCtx& bc, int TS)
{
    if (TS <= 125)
        for (int i = 0; i < p->tlen; i++)
            if (bc.tr[i] > 250)
                return true;
    return false;
}

// Bridge (dalign2/filter.c:1885-1948): path1 up to the bridge, the bridge, path3 after it
__device__ void d2_bridge(MPath* path1, const BPath* path2, const uint16_t* btr, const MPath* path3, PairBuf& pb,
                          int TS)
{
    int k, k1, k2, len, diff;
    k1 = 2 * ((path2->abpos / TS) - (path1->abpos / TS));
    k2 = (path2->aepos == path3->aepos) ? path3->tlen : 2 * ((path2->aepos / TS) - (path3->abpos / TS));
    len = k1 + path2->tlen + (path3->tlen - k2);
    if (len < 0 || pb.ttop + len > pb.tcap)
    {
        pb.err = 1;
        return;
    }
    const int base = pb.ttop;
    pb.ttop += len;
    uint16_t* trace = pb.tb + base;
    diff = 0;
    len = 0;
    if (k1 > 0)
    {
        const uint16_t* t = pb.tb + path1->toff;
        for (k = 0; k < k1; k += 2)
        {
            trace[len++] = t[k];
            trace[len++] = t[k + 1];
            diff += t[k];
        }
    }
    for (k = 0; k < path2->tlen; k += 2)
    {
        trace[len++] = btr[k];
        trace[len++] = btr[k + 1];
        diff += btr[k];
    }
    if (k2 < path3->tlen)
    {
        const uint16_t* t = pb.tb + path3->toff;
        for (k = k2; k < path3->tlen; k += 2)
        {
            trace[len++] = t[k];
            trace[len++] = t[k + 1];
            diff += t[k];
        }
    }
    path1->aepos = path3->aepos;
    path1->bepos = path3->bepos;
    path1->diffs = diff;
    path1->toff = base;
    path1->tlen = len;
}

// daligner2's Handle_Redundancies (dalign2/filter.c:1952-2272): the surviving path of a fused
// or contained pair stays at the later index j, the other is marked abpos = -1, a fusion
// restarts j's scan; then the bridging pass; compaction at the end.  Returns -1 when the
// bridge scratch was too small (bc.need says how much), or the pair trace buffer filled.
__device__ int handle_redundancies_d2(MPath* amatch, int novls, MPath* bmatch, PairBuf& pb, int TS, int comp,
                                      BridgeCtx& bc)
{
    int j, k, dist, awhen = 0, bwhen = 0;
    const bool hasB = (bmatch != nullptr);
    for (j = 1; j < novls; j++)
    {
        MPath* jpath = amatch + j;
        for (k = j - 1; k >= 0; k--)
        {
            MPath* kpath = amatch + k;
            if (kpath->abpos < 0)
                continue;
            if (jpath->abpos < kpath->abpos)
            {
                if (kpath->abpos <= jpath->aepos && kpath->bbpos <= jpath->bepos)
                {
                    dist = entwine(jpath, kpath, pb.tb, TS, &awhen, true);
                    if (dist == 0)
                    {
                        if (kpath->aepos > jpath->aepos)
                        {
                            if (hasB)
                            {
                                if (comp)
                                {
                                    dist = entwine(bmatch + k, bmatch + j, pb.tb, TS, &bwhen, true);
                                    if (dist != 0)
                                        continue;
                                    fusion(jpath, awhen, kpath, pb, TS);
                                    fusion(bmatch + k, bwhen, bmatch + j, pb, TS);
                                    bmatch[j] = bmatch[k];
                                }
                                else
                                {
                                    dist = entwine(bmatch + j, bmatch + k, pb.tb, TS, &bwhen, true);
                                    if (dist != 0)
                                        continue;
                                    fusion(jpath, awhen, kpath, pb, TS);
                                    fusion(bmatch + j, bwhen, bmatch + k, pb, TS);
                                }
                            }
                            else
                                fusion(jpath, awhen, kpath, pb, TS);
                            kpath->abpos = -1;
                            k = j;
                            continue;
                        }
                        kpath->abpos = -1;
                    }
                }
            }
            else
            {
                if (jpath->abpos <= kpath->aepos && jpath->bbpos <= kpath->bepos)
                {
                    dist = entwine(kpath, jpath, pb.tb, TS, &awhen, true);
                    if (dist == 0)
                    {
                        bool restart = false;
                        if (kpath->abpos == jpath->abpos)
                        {
                            if (kpath->aepos > jpath->aepos)
                            {
                                *jpath = *kpath;
                                if (hasB)
                                    bmatch[j] = bmatch[k];
                            }
                        }
                        else if (jpath->aepos > kpath->aepos)
                        {
                            if (hasB)
                            {
                                if (comp)
                                {
                                    dist = entwine(bmatch + j, bmatch + k, pb.tb, TS, &bwhen, true);
                                    if (dist != 0)
                                        continue;
                                    fusion(kpath, awhen, jpath, pb, TS);
                                    *jpath = *kpath;
                                    fusion(bmatch + j, bwhen, bmatch + k, pb, TS);
                                }
                                else
                                {
                                    dist = entwine(bmatch + k, bmatch + j, pb.tb, TS, &bwhen, true);
                                    if (dist != 0)
                                        continue;
                                    fusion(kpath, awhen, jpath, pb, TS);
                                    *jpath = *kpath;
                                    fusion(bmatch + k, bwhen, bmatch + j, pb, TS);
                                    bmatch[j] = bmatch[k];
                                }
                            }
                            else
                            {
                                fusion(kpath, awhen, jpath, pb, TS);
                                *jpath = *kpath;
                            }
                            restart = true;
                        }
                        else
                        {
                            *jpath = *kpath;
                            if (hasB)
                                bmatch[j] = bmatch[k];
                        }
                        kpath->abpos = -1;
                        if (restart)
                            k = j;
                    }
                }
            }
        }
    }
    // the bridging pass (dalign2/filter.c:2124-2262): a pair of paths with a narrow parallel
    // overlap joined through a fresh alignment of the overlap's box; the A side's box is
    // aligned uncomplemented, the B side's in the pair's orientation
    for (j = 1; j < novls; j++)
    {
        MPath* jpath = amatch + j;
        if (jpath->abpos < 0)
            continue;
        for (k = j - 1; k >= 0; k--)
        {
            MPath* kpath = amatch + k;
            if (kpath->abpos < 0)
                continue;
            MPath* path1 = jpath->abpos < kpath->abpos ? jpath : kpath;
            MPath* path2 = jpath->abpos < kpath->abpos ? kpath : jpath;
            if (path2->abpos >= path1->aepos || path1->aepos >= path2->aepos || path1->bbpos >= path2->bbpos ||
                path2->bbpos >= path1->bepos || path1->bepos >= path2->bepos)
                continue;
            const int aovl = path1->aepos - path2->abpos;
            const int bovl = path1->bepos - path2->bbpos;
            if (abs(aovl - bovl) > .2 * (aovl + bovl))
                continue;
            MPath *bath1 = nullptr, *bath2 = nullptr;
            if (hasB)
            {
                const bool first = (comp != 0) == (jpath->abpos < kpath->abpos);
                bath1 = first ? bmatch + k : bmatch + j;
                bath2 = first ? bmatch + j : bmatch + k;
                if (bath1->abpos > bath2->abpos)
                    continue;
            }
            BPath bp;
            if (!d2_bridge_path(path1, path2, bc.aseq, bc.bseq, bc.alen, bc.blen, 0, aovl, bovl, pb.tb, TS, &bp, bc))
                return -1;
            if (d2_check_bridge(&bp, bc, TS))
                continue;
            const MPath jback = *jpath, kback = *kpath;
            d2_bridge(path1, &bp, bc.tr, path2, pb, TS);
            if (pb.err)
                return -1;
            *jpath = *path1;
            kpath->abpos = -1;
            if (hasB)
            {
                if (!d2_bridge_path(bath1, bath2, bc.bseq, bc.aseq, bc.blen, bc.alen, comp, bovl, aovl, pb.tb, TS, &bp,
                                    bc))
                    return -1;
                if (d2_check_bridge(&bp, bc, TS))
                {
                    *jpath = jback;
                    *kpath = kback;
                    continue;
                }
                d2_bridge(bath1, &bp, bc.tr, bath2, pb, TS);
                if (pb.err)
                    return -1;
                bmatch[j] = *bath1;
            }
        }
    }
    int no = 0;
    for (j = 0; j < novls; j++)
        if (amatch[j].abpos >= 0)
        {
            if (hasB)
                bmatch[no] = bmatch[j];
            amatch[no++] = amatch[j];
        }
    return no;
}

// daligner2's end of a pair (filter_reporter_cpu.c:330-371): Handle_Redundancies, then the
// check of Compress_TraceTo8 (dalign2/align.c:3391-3412).  Returns (paths kept on the A side,
// on the B side, 0 or the GD_ERR_ code the pair fails with, the bridging scratch it needed).
// Kept out of line and given everything by value, so that the pair kernel's own registers
// and hot loop stay as they are.
__device__ __noinline__ int4 finish_pair_d2(MPath* amatch, int novla, MPath* bmatch, int novlb, PairBuf pb, int TS,
                                            int comp, bool check8, const uint8_t* aseq, const uint8_t* bseq, int alen,
                                            int blen, int* bvec, int bvcap, uint16_t* btr, int btcap)
{
    BridgeCtx bc{aseq, bseq, alen, blen, bvec, bvcap, btr, btcap, 0};
    int r1 = novla, r2 = novlb;
    // a B-only call gets the pair's align too, as the reference hands it (filter_reporter_cpu.c:392-400)
    if (r1 > 1)
    {
        if (r2 > 1)
            r1 = r2 = handle_redundancies_d2(amatch, r1, bmatch, pb, TS, comp, bc);
        else
            r1 = handle_redundancies_d2(amatch, r1, nullptr, pb, TS, comp, bc);
    }
    else if (r2 > 1)
        r2 = handle_redundancies_d2(bmatch, r2, nullptr, pb, TS, comp, bc);
    if (r1 < 0 || r2 < 0)
        return make_int4(novla, novlb, pb.err ? GD_ERR_TRACE : GD_ERR_BRIDGE, bc.need);
    if (check8)
    {
        for (int i = 0; i < r1; i++)
            for (int t = 0; t < amatch[i].tlen; t++)
                if (pb.tb[amatch[i].toff + t] > 255)
                    return make_int4(r1, r2, GD_ERR_TRACE8, 0);
        for (int i = 0; i < r2; i++)
            for (int t = 0; t < bmatch[i].tlen; t++)
                if (pb.tb[bmatch[i].toff + t] > 255)
                    return make_int4(r1, r2, GD_ERR_TRACE8, 0);
    }
    return make_int4(r1, r2, 0, 0);
}

// ------------------------------------------------------------------------------------------
// the pair kernel
// ------------------------------------------------------------------------------------------

__device__ __forceinline__ int hit_apos(uint64_t key, const HitBits& hb)
{
    return (int)(key & ((1ull << hb.pbits) - 1));
}

// first index in [lo, hi) whose apos exceeds x (apos ascending within a pair)
__device__ __forceinline__ int first_above(const uint64_t* hkey, int lo, int hi, int x, const HitBits& hb)
{
    while (lo < hi)
    {
        int m = (lo + hi) >> 1;
        if (hit_apos(hkey[m], hb) <= x)
            lo = m + 1;
        else
            hi = m;
    }
    return lo;
}

template <int RG>
__device__ void store_path(WarpCtx<RG>& w, const LAPath& lp, MPath* dst, PairBuf& pb)
{
    // all lanes: copy the trace into the pair buffer
    if (pb.ttop + lp.tlen > pb.tcap)
    {
        pb.err = 1;
        return;
    }
    for (int i = w.lane; i < lp.tlen; i += team_width<RG>())
        pb.tb[pb.ttop + i] = w.pts[lp.toff + i];
    if (w.lane == 0)
    {
        dst->toff = pb.ttop;
        dst->tlen = lp.tlen;
        dst->diffs = lp.diffs;
        dst->abpos = lp.abpos;
        dst->bbpos = lp.bbpos;
        dst->aepos = lp.aepos;
        dst->bepos = lp.bepos;
    }
    pb.ttop += lp.tlen;
}

template <int RG>
__device__ void emit_paths(WarpCtx<RG>& w, const AlignParams& P, const MPath* m, int n, const uint16_t* tb, int aread,
                           int bread, AlignOut& out)
{
    if (n <= 0)
        return;
    int tlen_tot = 0;
    if (!P.no_trace)
        for (int i = 0; i < n; i++)
            tlen_tot += m[i].tlen;
    int tbytes = P.trace8 ? 1 : 2;
    unsigned long long r0 = 0, t0 = 0;
    if (w.lane == 0)
    {
        r0 = atomicAdd(&out.counters[0], (unsigned long long)n);
        t0 = atomicAdd(&out.counters[1], (unsigned long long)tlen_tot * tbytes);
    }
    r0 = tshfl(w, r0, 0);
    t0 = tshfl(w, t0, 0);
    if (r0 + n > out.rcap || t0 + (unsigned long long)tlen_tot * tbytes > out.tcap)
        return;  // the host sees the counters past capacity and re-runs with more room
    unsigned long long toff = t0;
    for (int i = 0; i < n; i++)
    {
        int tl = P.no_trace ? 0 : m[i].tlen;
        if (w.lane == 0)
        {
            OutRec o;
            o.tlen = tl;
            o.diffs = m[i].diffs;
            o.abpos = m[i].abpos;
            o.bbpos = m[i].bbpos;
            o.aepos = m[i].aepos;
            o.bepos = m[i].bepos;
            o.flags = (uint32_t)P.comp;
            o.aread = aread;
            o.bread = bread;
            o.pad = 0;
            o.toff = toff;
            out.rec[r0 + i] = o;
        }
        const uint16_t* src = tb + m[i].toff;
        constexpr int TW = team_width<RG>();
        if (P.trace8)
            for (int j = w.lane; j < tl; j += TW)
                out.trace[toff + j] = (uint8_t)src[j];  // Compress_TraceTo8 (align.c:3352-3360)
        else
            for (int j = w.lane; j < tl; j += TW)
            {
                out.trace[toff + 2 * j] = (uint8_t)(src[j] & 0xff);
                out.trace[toff + 2 * j + 1] = (uint8_t)(src[j] >> 8);
            }
        toff += (unsigned long long)tl * tbytes;
    }
}

template <int RG>
constexpr int warps_of()
{
    return RG == WIDE_RING ? 1 : ALIGN_WARPS;
}

// D2: daligner2's report (dalign2/filter_reporter_cpu.c) -- its -H, its rule for the B-side
// record of a read against itself, its Handle_Redundancies; a separate instance, so that
// daligner's keeps its code layout.
#ifndef GD_ALIGN_MINB
#define GD_ALIGN_MINB 6  // CTAs per SM the warp instance is compiled for (80 registers; 7, at 72, spills and runs 9 % slower)
#endif

template <int RG, bool D2 = false>
__global__ void __launch_bounds__(warps_of<RG>() * 32, RG == WIDE_RING ? 1 : GD_ALIGN_MINB)
    k_align_pairs(DevBlock A, DevBlock B, const uint64_t* __restrict__ hkey, const uint32_t* __restrict__ hdiag,
                  const uint2* __restrict__ groups, const uint32_t* __restrict__ order, unsigned ngroups, AlignParams P,
                  AlignScratch sc, AlignOut out, unsigned* queue, DevStatus* st)
{
    constexpr int NW = warps_of<RG>();
    __shared__ WarpSmem<RG> smem[NW];
    const int lane = threadIdx.x & 31;
    const int wib = threadIdx.x >> 5;
    const int gw = blockIdx.x * NW + wib;
    if (gw >= sc.nwarps)
        return;
    WarpCtx<RG> w;
    w.sm = &smem[wib];
    w.peb = sc.peb + (size_t)gw * sc.pcap;
    w.pcap = sc.pcap;
    w.pts = sc.pts + (size_t)gw * sc.ptscap;
    w.ptscap = sc.ptscap;
    w.st = st;
    w.lane = lane;
    w.err = 0;
    w.cells = 0;
    MPath* amatch = sc.match + (size_t)gw * 2 * sc.mcap;
    MPath* bmatch = amatch + sc.mcap;
    uint16_t* tbuf = sc.tbuf + (size_t)gw * sc.tcap;
    int* score = sc.bands + (size_t)gw * 3 * sc.nbands - (P.mindiag - 2);
    int* lastp = score + sc.nbands;
    int* lasta = lastp + sc.nbands;
    const int K = P.kmer, BS = P.binshift, TS = P.tspace;
    const int minhit = (P.hitmin - 1) / K + 1;
    const unsigned lt = lanemask_lt();
    unsigned long long tcells = 0, tseeds = 0;  // this warp's totals over the groups it completed

    while (true)
    {
        unsigned g = 0;
        if (lane == 0)
            g = atomicAdd(queue, 1u);
        g = __shfl_sync(GD_FULL, g, 0);
        if (g >= ngroups || st->code != 0)
            break;
        const unsigned item = order[g];
        if (out.skip && out.skip[item])
            continue;
        uint2 grp = groups[item];
        const int s = (int)grp.x, e = (int)grp.y;
        w.item = (int)item;
        w.cells = 0;
        unsigned nseeds = 0;
        uint64_t k0 = hkey[s];
        const int ar = (int)((k0 >> P.hb.pbits) & ((1ull << P.hb.abits) - 1));
        const int br = (int)(k0 >> (P.hb.pbits + P.hb.abits));
        const int alen = A.rlen[ar], blen = B.rlen[br];
        const uint8_t* aseq = A.bases + A.boff[ar];
        const uint8_t* bseq = B.bases + B.boff[br];
        const uint32_t ag = PK_BIAS + (uint32_t)A.boff[ar], bg = PK_BIAS + (uint32_t)B.boff[br];
        if (D2 && alen < P.hgap && blen < P.hgap)
            continue;  // daligner2 -H: neither read is long enough (filter_reporter_cpu.c:156-162)
        const bool doA = !D2 || alen >= P.hgap;
        const bool doB = D2 ? (P.symmetric && blen >= P.hgap && !(ar == br && P.self))
                            : (P.symmetric && (ar != br || !P.self || !P.comp));
        PairBuf pb;
        pb.am = amatch;
        pb.bm = bmatch;
        pb.tb = tbuf;
        pb.ttop = 0;
        pb.tcap = sc.tcap;
        pb.err = 0;
        int novla = 0, novlb = 0;
        int tlo = INT_MAX, thi = INT_MIN;  // lasta bands touched in this pair

        int nidx = s, amark2 = 0;
        while (nidx < e && !w.err && !pb.err)
        {
            int amark = amark2 + PANEL_SIZE;
            amark2 = amark - PANEL_OVERLAP;
            const int lidx = nidx;
            int q = first_above(hkey, lidx, e, amark, P.hb);
            const int nend = (q < e) ? q + 1 : e;
            const int h2 = first_above(hkey, lidx, nend, amark2, P.hb);
            if (nend - lidx < minhit)
            {
                nidx = h2;
                continue;
            }
            // panel band scores (filter.c:1754-1766)
            for (int base = lidx; base < nend; base += 32)
            {
                int i = base + lane;
                bool valid = i < nend;
                int ap = 0, dg = 0;
                if (valid)
                {
                    ap = hit_apos(hkey[i], P.hb);
                    dg = ((int)hdiag[i]) >> BS;
                }
                unsigned key = valid ? (unsigned)dg : (0x80000000u | (unsigned)lane);
                unsigned peers = __match_any_sync(GD_FULL, key);
                unsigned lower = peers & lt;
                int src = lower ? 31 - __clz(lower) : lane;
                int prevap = __shfl_sync(GD_FULL, ap, src);
                int delta = 0;
                if (valid)
                {
                    int prev = lower ? prevap : lastp[dg];
                    delta = (ap - prev >= K) ? K : ap - prev;
                }
                unsigned todo = __ballot_sync(GD_FULL, valid);
                while (todo)
                {
                    int leader = __ffs(todo) - 1;
                    unsigned grpm = __shfl_sync(GD_FULL, peers, leader);
                    int sum = __reduce_add_sync(GD_FULL, ((grpm >> lane) & 1) ? delta : 0);
                    int last = 31 - __clz(grpm);
                    int lastap = __shfl_sync(GD_FULL, ap, last);
                    int gdg = __shfl_sync(GD_FULL, dg, leader);
                    if (lane == 0)
                    {
                        score[gdg] += sum;
                        lastp[gdg] = lastap;
                    }
                    todo &= ~grpm;
                }
                __syncwarp();
            }
            // seeds in hit order (filter.c:1776-1893)
            for (int base = lidx; base < nend && !w.err && !pb.err; base += 32)
            {
                int i = base + lane;
                bool valid = i < nend;
                int ap = 0, d = 0, dg = 0;
                bool cand = false;
                if (valid)
                {
                    ap = hit_apos(hkey[i], P.hb);
                    d = (int)hdiag[i];
                    dg = d >> BS;
                    int sc0 = score[dg];
                    cand = (sc0 + score[dg + 1] >= P.hitmin) || (sc0 + score[dg - 1] >= P.hitmin);
                }
                unsigned cm = __ballot_sync(GD_FULL, cand);
                while (cm && !w.err && !pb.err)
                {
                    int j = __ffs(cm) - 1;
                    cm &= cm - 1;
                    int apj = __shfl_sync(GD_FULL, ap, j);
                    int dj = __shfl_sync(GD_FULL, d, j);
                    int dgj = dj >> BS;
                    if (!(apj > lasta[dgj]))
                        continue;
                    nseeds++;
                    int bpj = apj - dj;
                    local_alignment<RG, true>(w, P, aseq, bseq, A.pk, ag, B.pk, bg, alen, blen, P.comp, dj,
                                              apj + bpj);
                    if (w.err)
                        break;
                    const LAPath apth = w.sm->ap;
                    const LAPath bpth = w.sm->bp;
                    // Diagonal_Span (filter.c:1568-1599) of the A path, then widen lasta
                    int lo, hi;
                    {
                        const uint16_t* points = w.pts + apth.toff;
                        int dd = apth.abpos - apth.bbpos, low = dd, hgh = dd;
                        dd = apth.aepos - apth.bepos;
                        if (dd < low)
                            low = dd;
                        else if (dd > hgh)
                            hgh = dd;
                        dd = (apth.abpos / TS) * TS - apth.bbpos;
                        int tl = apth.tlen - 2;
                        // prefix sums of (TS - points[2i+1]) in lane chunks
                        for (int b0 = 1; b0 < tl; b0 += 64)
                        {
                            int idx = b0 + 2 * lane;
                            int v = (idx < tl) ? (TS - (int)points[idx]) : 0;
                            int x = v;
#pragma unroll
                            for (int o = 1; o < 32; o <<= 1)
                            {
                                int t = __shfl_up_sync(GD_FULL, x, o);
                                if (lane >= o)
                                    x += t;
                            }
                            int val = dd + x;
                            int vlo = (idx < tl) ? val : INT_MAX, vhi = (idx < tl) ? val : INT_MIN;
                            vlo = __reduce_min_sync(GD_FULL, vlo);
                            vhi = __reduce_max_sync(GD_FULL, vhi);
                            low = min(low, vlo);
                            hgh = max(hgh, vhi);
                            dd = __shfl_sync(GD_FULL, val, 31);
                        }
                        lo = (low >> BS) - 1;
                        hi = (hgh >> BS) + 1;
                    }
                    if (dgj < lo)
                        lo = dgj;
                    else if (dgj > hi)
                        hi = dgj;
                    // the reference's band arrays end one band past each side (filter.c:2296-2311)
                    lo = max(lo, P.mindiag - 1);
                    hi = min(hi, P.maxdiag + 1);
                    const int ae = apth.aepos;
                    for (int dd2 = lo + lane; dd2 <= hi; dd2 += 32)
                        if (ae > lasta[dd2])
                            lasta[dd2] = ae;
                    tlo = min(tlo, lo);
                    thi = max(thi, hi);
                    __syncwarp();
                    if ((apth.aepos - apth.abpos) + (apth.bepos - apth.bbpos) >= P.minover)
                    {
                        if ((doA && novla >= sc.mcap) || (doB && novlb >= sc.mcap))
                        {
                            if (lane == 0)
                                gd_fail(st, GD_ERR_MATCHES, w.item, sc.mcap);
                            w.err = 1;
                            break;
                        }
                        if (doA)
                        {
                            store_path(w, apth, amatch + novla, pb);
                            novla++;
                        }
                        if (doB)
                        {
                            store_path(w, bpth, bmatch + novlb, pb);
                            novlb++;
                        }
                        __syncwarp();
                        if (pb.err)
                        {
                            if (lane == 0)
                                gd_fail(st, GD_ERR_TRACE, w.item, sc.tcap);
                            w.err = 1;
                            break;
                        }
                    }
                }
            }
            // reset the panel's band scores (filter.c:1895-1899)
            for (int i = lidx + lane; i < nend; i += 32)
            {
                int dg = ((int)hdiag[i]) >> BS;
                score[dg] = 0;
                lastp[dg] = 0;
            }
            __syncwarp();
            nidx = h2;
        }
        // reset lasta (filter.c:1902-1920): every band this pair raised
        if (tlo <= thi)
            for (int dd2 = tlo + lane; dd2 <= thi; dd2 += 32)
                lasta[dd2] = 0;
        if (nidx < e)  // aborted pair: clear score/lastp of all its hits
            for (int i = s + lane; i < e; i += 32)
            {
                int dg = ((int)hdiag[i]) >> BS;
                score[dg] = 0;
                lastp[dg] = 0;
            }
        __syncwarp();
        if (w.err == 2)
        {
            if (!out.wide_list)
            {
                if (lane == 0)
                    gd_fail(st, GD_ERR_BAND_WIDTH, w.item, ring_of<RG>());
                break;
            }
            // the band outgrew this instance: the group goes to the wide instance as if this
            // warp had never seen it (its band arrays are clean again, nothing was emitted)
            if (lane == 0)
                out.wide_list[atomicAdd(out.nwide, 1u)] = item;
            w.err = 0;
            __syncwarp();
            continue;
        }
        if (w.err)
            break;
        // merge redundant paths (filter.c:1922-1938), lane 0
        int d2fail = 0;
        if (lane == 0)
        {
            if (D2)
            {
                const int4 f = finish_pair_d2(amatch, novla, bmatch, novlb, pb, TS, P.comp, P.trace8 && !P.no_trace,
                                              aseq, bseq, alen, blen, sc.bvec + (size_t)gw * sc.bvcap, sc.bvcap,
                                              sc.btr + (size_t)gw * sc.btcap, sc.btcap);
                novla = f.x;
                novlb = f.y;
                d2fail = f.z;
                if (d2fail)
                    gd_fail(st, d2fail, w.item, d2fail == GD_ERR_BRIDGE ? f.w : sc.tcap);
            }
            else if (novla > 1)
            {
                if (novlb > 1)
                    novla = novlb = handle_redundancies(amatch, novla, bmatch, pb, TS, P.comp);
                else
                    novla = handle_redundancies(amatch, novla, nullptr, pb, TS, P.comp);
            }
            else if (novlb > 1)
                novlb = handle_redundancies(bmatch, novlb, nullptr, pb, TS, P.comp);
            if (pb.err)
                gd_fail(st, GD_ERR_TRACE, w.item, sc.tcap);
        }
        novla = __shfl_sync(GD_FULL, novla, 0);
        novlb = __shfl_sync(GD_FULL, novlb, 0);
        d2fail = __shfl_sync(GD_FULL, d2fail, 0);
        __syncwarp();
        if (d2fail)
            break;
        emit_paths(w, P, amatch, novla, tbuf, ar + A.ufirst, br + B.ufirst, out);
        emit_paths(w, P, bmatch, novlb, tbuf, br + B.ufirst, ar + A.ufirst, out);
        if (out.gstat && lane == 0)
            out.gstat[item] = make_uint2((unsigned)(novla + novlb), w.cells);
        tcells += w.cells;
        tseeds += nseeds;
        __syncwarp();
    }
    if (lane == 0)
    {
        atomicAdd(&out.counters[2], tcells);
        atomicAdd(&out.counters[3], tseeds);
    }
}

// ------------------------------------------------------------------------------------------
// The duo instance: two pair groups per warp, one per half-warp team of 16 lanes.
//
// Most waves are narrow (a few to 20 diagonals), so a warp with lanes over diagonals leaves
// most of its lanes idle; two teams of 16 are meant to keep them busy.  Each team runs its
// pair group as a state machine: the warp takes one wave of every team that is in a wave in
// lockstep (wave_step_duo: the teams run the same instructions on their own data, in either
// direction), then lets each team that left its wave do everything up to its next wave --
// the end of the wave, the next seed, the next panel or pair group -- on its own.  Records,
// cells and seeds are those of k_align_pairs: the per-team work is the same code at team
// width.  A group whose band outgrows 128 diagonals goes to the wide list.  Measured, it is
// slower than k_align_pairs: a lockstep step of two waves issues about twice a warp wave's
// instructions, and two rings per warp halve the resident warps.
// ------------------------------------------------------------------------------------------
enum DuoState : int
{
    D_NEXT,    // take the next pair group from the queue
    D_PANEL,   // the next panel of the group: its band scores
    D_SEEDS,   // the next seed of the panel that passes the lasta test
    D_BEGIN,   // the 0-wave of the forward (then reverse) wave from the seed
    D_WAVE,    // one wave per warp step
    D_WAVED,   // the wave ended: its trace points, the reverse wave, the path's bookkeeping
    D_FINISH,  // the group ended: band resets, Handle_Redundancies, the records
    D_DONE
};

#ifndef GD_DUO_MINB
#define GD_DUO_MINB 7  // CTAs per SM the duo instance is compiled for (shared memory allows 7)
#endif

__global__ void __launch_bounds__(DUO_WARPS * 32, GD_DUO_MINB)
    k_align_duo(DevBlock A, DevBlock B, const uint64_t* __restrict__ hkey, const uint32_t* __restrict__ hdiag,
                const uint2* __restrict__ groups, const uint32_t* __restrict__ order, unsigned ngroups, AlignParams P,
                AlignScratch sc, AlignOut out, unsigned* queue, DevStatus* st)
{
    constexpr int RG = DUO;
    constexpr int TW = team_width<RG>();
    __shared__ WarpSmem<RG> smem[DUO_WARPS][2];
    const int wlane = threadIdx.x & 31;
    const int wib = threadIdx.x >> 5;
    const int team = wlane >> 4;
    const int gt = (blockIdx.x * DUO_WARPS + wib) * 2 + team;  // the team's scratch slot
    if ((blockIdx.x * DUO_WARPS + wib) * 2 >= sc.nwarps)
        return;
    WarpCtx<RG> w;
    w.sm = &smem[wib][team];
    w.peb = sc.peb + (size_t)gt * sc.pcap;
    w.pcap = sc.pcap;
    w.pts = sc.pts + (size_t)gt * sc.ptscap;
    w.ptscap = sc.ptscap;
    w.st = st;
    w.lane = wlane & 15;
    w.tbase = team * 16;
    w.tmask = 0xffffu << w.tbase;
    w.err = 0;
    w.cells = 0;
    w.item = 0;
    const int lane = w.lane;
    MPath* amatch = sc.match + (size_t)gt * 2 * sc.mcap;
    MPath* bmatch = amatch + sc.mcap;
    uint16_t* tbuf = sc.tbuf + (size_t)gt * sc.tcap;
    int* score = sc.bands + (size_t)gt * 3 * sc.nbands - (P.mindiag - 2);
    int* lastp = score + sc.nbands;
    int* lasta = lastp + sc.nbands;
    const int K = P.kmer, BS = P.binshift, TS = P.tspace;
    const int minhit = (P.hitmin - 1) / K + 1;
    const unsigned lt = tlt(w);
    unsigned long long tcells = 0, tseeds = 0;

    // the team's pair group, panel and seed
    int state = D_NEXT;
    unsigned item = 0, nseeds = 0;
    int s = 0, e = 0, ar = 0, br = 0, alen = 0, blen = 0;
    bool doA = false, doB = false;
    const uint8_t* aseq = nullptr;
    const uint8_t* bseq = nullptr;
    uint32_t ag = 0, bg = 0;
    PairBuf pb;
    pb.am = amatch;
    pb.bm = bmatch;
    pb.tb = tbuf;
    pb.tcap = sc.tcap;
    pb.ttop = 0;
    pb.err = 0;
    int novla = 0, novlb = 0, tlo = INT_MAX, thi = INT_MIN;
    int nidx = 0, amark2 = 0, lidx = 0, nend = 0, h2 = 0, base = 0;
    unsigned cm = 0;
    // the alignment: its direction, seed, and wave state
    bool fwd = true;
    int dj = 0, anti = 0, low = 0, minp = 0, maxp = 0, maxtp = 0;
    WaveVars wv{};

    while (true)
    {
        const bool act = state == D_WAVE;
        if (__any_sync(GD_FULL, act))
        {
            const bool cont = wave_step_duo(act, fwd, w, wv, P, A.pk, ag, B.pk, bg, alen, blen, minp, maxp);
            if (act && !cont)
                state = D_WAVED;
        }
        // everything up to the team's next wave
        while (state != D_WAVE && state != D_DONE)
        {
            if (state == D_NEXT)
            {
                unsigned g = 0;
                if (lane == 0)
                    g = atomicAdd(queue, 1u);
                g = tshfl(w, g, 0);
                if (g >= ngroups || st->code != 0)
                {
                    state = D_DONE;
                    break;
                }
                item = order[g];
                if (out.skip && out.skip[item])
                    continue;
                const uint2 grp = groups[item];
                s = (int)grp.x;
                e = (int)grp.y;
                w.item = (int)item;
                w.cells = 0;
                nseeds = 0;
                const uint64_t k0 = hkey[s];
                ar = (int)((k0 >> P.hb.pbits) & ((1ull << P.hb.abits) - 1));
                br = (int)(k0 >> (P.hb.pbits + P.hb.abits));
                alen = A.rlen[ar];
                blen = B.rlen[br];
                aseq = A.bases + A.boff[ar];
                bseq = B.bases + B.boff[br];
                ag = PK_BIAS + (uint32_t)A.boff[ar];
                bg = PK_BIAS + (uint32_t)B.boff[br];
                doA = true;
                doB = P.symmetric && (ar != br || !P.self || !P.comp);
                pb.ttop = 0;
                pb.err = 0;
                novla = novlb = 0;
                tlo = INT_MAX;
                thi = INT_MIN;
                nidx = s;
                amark2 = 0;
                state = D_PANEL;
            }
            else if (state == D_PANEL)
            {
                if (!(nidx < e && !w.err && !pb.err))
                {
                    state = D_FINISH;
                    continue;
                }
                const int amark = amark2 + PANEL_SIZE;
                amark2 = amark - PANEL_OVERLAP;
                lidx = nidx;
                const int q = first_above(hkey, lidx, e, amark, P.hb);
                nend = (q < e) ? q + 1 : e;
                h2 = first_above(hkey, lidx, nend, amark2, P.hb);
                if (nend - lidx < minhit)
                {
                    nidx = h2;
                    continue;
                }
                // panel band scores (filter.c:1754-1766)
                for (int b0 = lidx; b0 < nend; b0 += TW)
                {
                    const int i = b0 + lane;
                    const bool valid = i < nend;
                    int ap = 0, dg = 0;
                    if (valid)
                    {
                        ap = hit_apos(hkey[i], P.hb);
                        dg = ((int)hdiag[i]) >> BS;
                    }
                    const unsigned key = valid ? (unsigned)dg : (0x80000000u | (unsigned)lane);
                    const unsigned peers = tmatch(w, key);
                    const unsigned lower = peers & lt;
                    const int src = lower ? 31 - __clz(lower) : lane;
                    const int prevap = tshfl(w, ap, src);
                    int delta = 0;
                    if (valid)
                    {
                        const int prev = lower ? prevap : lastp[dg];
                        delta = (ap - prev >= K) ? K : ap - prev;
                    }
                    unsigned todo = tballot(w, valid);
                    while (todo)
                    {
                        const int leader = __ffs(todo) - 1;
                        const unsigned grpm = tshfl(w, peers, leader);
                        const int sum = tadd(w, ((grpm >> lane) & 1) ? delta : 0);
                        const int last = 31 - __clz(grpm);
                        const int lastap = tshfl(w, ap, last);
                        const int gdg = tshfl(w, dg, leader);
                        if (lane == 0)
                        {
                            score[gdg] += sum;
                            lastp[gdg] = lastap;
                        }
                        todo &= ~grpm;
                    }
                    tsync(w);
                }
                base = lidx - TW;
                cm = 0;
                state = D_SEEDS;
            }
            else if (state == D_SEEDS)
            {
                // seeds in hit order (filter.c:1776-1893)
                if (w.err || pb.err || (cm == 0 && base + TW >= nend))
                {
                    // reset the panel's band scores (filter.c:1895-1899)
                    for (int i = lidx + lane; i < nend; i += TW)
                    {
                        const int dg = ((int)hdiag[i]) >> BS;
                        score[dg] = 0;
                        lastp[dg] = 0;
                    }
                    tsync(w);
                    nidx = h2;
                    state = D_PANEL;
                    continue;
                }
                if (cm == 0)
                {
                    base += TW;
                    const int i = base + lane;
                    bool cand = false;
                    if (i < nend)
                    {
                        const int dg = ((int)hdiag[i]) >> BS;
                        const int sc0 = score[dg];
                        cand = (sc0 + score[dg + 1] >= P.hitmin) || (sc0 + score[dg - 1] >= P.hitmin);
                    }
                    cm = tballot(w, cand);
                    continue;
                }
                const int j = __ffs(cm) - 1;
                cm &= cm - 1;
                const int apj = hit_apos(hkey[base + j], P.hb);
                dj = (int)hdiag[base + j];
                if (!(apj > lasta[dj >> BS]))
                    continue;
                nseeds++;
                // Local_Alignment from (dj, apj + bpj) with lbord = hbord = -1 (align.c:1922-2060)
                anti = 2 * apj - dj;
                maxtp = 2 * (max(alen, blen) / TS + 2);
                if (4 * maxtp + 16 > w.ptscap)
                {
                    if (lane == 0)
                        gd_fail(w.st, GD_ERR_TRACE, w.item, maxtp);
                    w.err = 1;
                    continue;
                }
                low = dj;
                const bool selfie = (aseq == bseq);
                minp = (selfie && dj >= 0) ? 1 : -INT_MAX;
                maxp = (selfie && dj <= 0) ? -1 : INT_MAX;
                if (lane == 0)
                {
                    w.sm->ap.tlen = w.sm->bp.tlen = 0;
                    w.sm->ap.diffs = w.sm->bp.diffs = 0;
                }
                tsync(w);
                fwd = true;
                state = D_BEGIN;
            }
            else if (state == D_BEGIN)
            {
                wave_begin<RG, true>(fwd, w, wv, P, aseq, bseq, A.pk, ag, B.pk, bg, alen, blen, P.comp, low, low, anti);
                state = w.err ? D_SEEDS : D_WAVE;
            }
            else if (state == D_WAVED)
            {
                if (w.err)
                {
                    state = D_SEEDS;
                    continue;
                }
                uint16_t* atrace = w.pts + maxtp;
                uint16_t* btrace = atrace + 2 * maxtp;
                wave_end<RG, true>(fwd, w, wv, P, aseq, bseq, A.pk, ag, B.pk, bg, alen, blen, P.comp, &w.sm->ap,
                                   &w.sm->bp, &low, anti, atrace, btrace);
                if (fwd)
                {
                    fwd = false;
                    state = D_BEGIN;
                    continue;
                }
                if (P.comp && lane == 0)
                {
                    uint16_t* tr = w.pts + w.sm->bp.toff;
                    int i = w.sm->bp.tlen - 2, jj = 0;
                    while (jj < i)
                    {
                        uint16_t t = tr[i];
                        tr[i] = tr[jj];
                        tr[jj] = t;
                        t = tr[i + 1];
                        tr[i + 1] = tr[jj + 1];
                        tr[jj + 1] = t;
                        i -= 2;
                        jj += 2;
                    }
                }
                tsync(w);
                state = D_SEEDS;
                const LAPath apth = w.sm->ap;
                const LAPath bpth = w.sm->bp;
                // Diagonal_Span (filter.c:1568-1599) of the A path, then widen lasta
                int lo, hi;
                {
                    const uint16_t* points = w.pts + apth.toff;
                    int dd = apth.abpos - apth.bbpos, dlo = dd, dhi = dd;
                    dd = apth.aepos - apth.bepos;
                    if (dd < dlo)
                        dlo = dd;
                    else if (dd > dhi)
                        dhi = dd;
                    dd = (apth.abpos / TS) * TS - apth.bbpos;
                    const int tl = apth.tlen - 2;
                    for (int b0 = 1; b0 < tl; b0 += 2 * TW)
                    {
                        const int idx = b0 + 2 * lane;
                        int x = (idx < tl) ? (TS - (int)points[idx]) : 0;
#pragma unroll
                        for (int o = 1; o < TW; o <<= 1)
                        {
                            const int t = tshfl_up(w, x, o);
                            if (lane >= o)
                                x += t;
                        }
                        const int val = dd + x;
                        dlo = min(dlo, tmin(w, (idx < tl) ? val : INT_MAX));
                        dhi = max(dhi, tmax(w, (idx < tl) ? val : INT_MIN));
                        dd = tshfl(w, val, TW - 1);
                    }
                    lo = (dlo >> BS) - 1;
                    hi = (dhi >> BS) + 1;
                }
                const int dgj = dj >> BS;
                if (dgj < lo)
                    lo = dgj;
                else if (dgj > hi)
                    hi = dgj;
                // the reference's band arrays end one band past each side (filter.c:2296-2311)
                lo = max(lo, P.mindiag - 1);
                hi = min(hi, P.maxdiag + 1);
                const int ae = apth.aepos;
                for (int dd2 = lo + lane; dd2 <= hi; dd2 += TW)
                    if (ae > lasta[dd2])
                        lasta[dd2] = ae;
                tlo = min(tlo, lo);
                thi = max(thi, hi);
                tsync(w);
                if ((apth.aepos - apth.abpos) + (apth.bepos - apth.bbpos) >= P.minover)
                {
                    if ((doA && novla >= sc.mcap) || (doB && novlb >= sc.mcap))
                    {
                        if (lane == 0)
                            gd_fail(st, GD_ERR_MATCHES, w.item, sc.mcap);
                        w.err = 1;
                        continue;
                    }
                    if (doA)
                    {
                        store_path(w, apth, amatch + novla, pb);
                        novla++;
                    }
                    if (doB)
                    {
                        store_path(w, bpth, bmatch + novlb, pb);
                        novlb++;
                    }
                    tsync(w);
                    if (pb.err)
                    {
                        if (lane == 0)
                            gd_fail(st, GD_ERR_TRACE, w.item, sc.tcap);
                        w.err = 1;
                    }
                }
            }
            else  // D_FINISH
            {
                // reset lasta (filter.c:1902-1920): every band this pair raised
                if (tlo <= thi)
                    for (int dd2 = tlo + lane; dd2 <= thi; dd2 += TW)
                        lasta[dd2] = 0;
                if (nidx < e)  // aborted pair: clear score/lastp of all its hits
                    for (int i = s + lane; i < e; i += TW)
                    {
                        const int dg = ((int)hdiag[i]) >> BS;
                        score[dg] = 0;
                        lastp[dg] = 0;
                    }
                tsync(w);
                if (w.err == 2)
                {
                    if (!out.wide_list)
                    {
                        if (lane == 0)
                            gd_fail(st, GD_ERR_BAND_WIDTH, w.item, ring_of<RG>());
                        state = D_DONE;
                        break;
                    }
                    // the band outgrew this instance: the group goes to the wide instance as if
                    // this team had never seen it (its band arrays are clean again)
                    if (lane == 0)
                        out.wide_list[atomicAdd(out.nwide, 1u)] = item;
                    w.err = 0;
                    tsync(w);
                    state = D_NEXT;
                    continue;
                }
                if (w.err)
                {
                    state = D_DONE;
                    break;
                }
                // merge redundant paths (filter.c:1922-1938), lane 0
                if (lane == 0)
                {
                    if (novla > 1)
                    {
                        if (novlb > 1)
                            novla = novlb = handle_redundancies(amatch, novla, bmatch, pb, TS, P.comp);
                        else
                            novla = handle_redundancies(amatch, novla, nullptr, pb, TS, P.comp);
                    }
                    else if (novlb > 1)
                        novlb = handle_redundancies(bmatch, novlb, nullptr, pb, TS, P.comp);
                    if (pb.err)
                        gd_fail(st, GD_ERR_TRACE, w.item, sc.tcap);
                }
                novla = tshfl(w, novla, 0);
                novlb = tshfl(w, novlb, 0);
                tsync(w);
                emit_paths(w, P, amatch, novla, tbuf, ar + A.ufirst, br + B.ufirst, out);
                emit_paths(w, P, bmatch, novlb, tbuf, br + B.ufirst, ar + A.ufirst, out);
                if (out.gstat && lane == 0)
                    out.gstat[item] = make_uint2((unsigned)(novla + novlb), w.cells);
                tcells += w.cells;
                tseeds += nseeds;
                tsync(w);
                state = D_NEXT;
            }
        }
        if (__all_sync(GD_FULL, state == D_DONE))
            break;
    }
    if (lane == 0)
    {
        atomicAdd(&out.counters[2], tcells);
        atomicAdd(&out.counters[3], tseeds);
    }
}

// Test hook: daligner2's Handle_Redundancies (fusion, bridging, compaction) of one pair on
// the device, single thread.  hdr = 6 ints per path (A side, then B side with hasB), trace =
// their trace values back to back (capacity tcap in the pair buffer, which also receives
// fusions and bridges); out_hdr receives the kept paths, out_n their count (or -code).
__global__ void k_test_hr_d2(const uint8_t* aseq, const uint8_t* bseq, int alen, int blen, int tspace, int comp,
                             int novls, int hasB, const int32_t* hdr, MPath* paths, uint16_t* tbuf, int ttop,
                             int tcap, int* vec, int vcap, uint16_t* btr, int btcap, int32_t* out_hdr, int* out_n)
{
    const int npath = novls * (hasB ? 2 : 1);
    int off = 0;
    for (int i = 0; i < npath; i++)
    {
        const int32_t* h = hdr + 6 * i;
        paths[i] = MPath{off, h[5], h[4], h[0], h[1], h[2], h[3], 0};
        off += h[5];
    }
    PairBuf pb{paths, hasB ? paths + novls : nullptr, tbuf, ttop, tcap, 0};
    BridgeCtx bc{aseq, bseq, alen, blen, vec, vcap, btr, btcap, 0};
    const int n = handle_redundancies_d2(paths, novls, hasB ? paths + novls : nullptr, pb, tspace, comp, bc);
    if (n < 0)
    {
        *out_n = pb.err ? -GD_ERR_TRACE : -GD_ERR_BRIDGE;
        return;
    }
    for (int side = 0; side < (hasB ? 2 : 1); side++)
        for (int i = 0; i < n; i++)
        {
            const MPath& q = paths[side * novls + i];
            int32_t* h = out_hdr + 6 * (side * n + i);
            h[0] = q.abpos;
            h[1] = q.bbpos;
            h[2] = q.aepos;
            h[3] = q.bepos;
            h[4] = q.diffs;
            h[5] = q.tlen;
        }
    // the kept paths' trace offsets, for the host to gather
    for (int side = 0; side < (hasB ? 2 : 1); side++)
        for (int i = 0; i < n; i++)
            out_hdr[6 * npath + side * n + i] = paths[side * novls + i].toff;
    *out_n = n;
}

int launch_test_hr_d2(const uint8_t* aseq, const uint8_t* bseq, int alen, int blen, int tspace, int comp, int novls,
                      int hasB, const int32_t* hdr, MPath* paths, uint16_t* tbuf, int ttop, int tcap, int* vec,
                      int vcap, uint16_t* btr, int btcap, int32_t* out_hdr, int* out_n, cudaStream_t s)
{
    k_test_hr_d2<<<1, 1, 0, s>>>(aseq, bseq, alen, blen, tspace, comp, novls, hasB, hdr, paths, tbuf, ttop, tcap, vec,
                                 vcap, btr, btcap, out_hdr, out_n);
    GD_LAUNCHED(1);
    GD_CUDA(cudaGetLastError());
    return 0;
}

size_t align_scratch_bytes(int nwarps, int pcap, int ptscap, int mcap, int tcap, int nbands, int bvcap, int btcap)
{
    size_t per = (size_t)pcap * sizeof(int4) + (size_t)ptscap * 2 + (size_t)2 * mcap * sizeof(MPath) +
                 (size_t)tcap * 2 + (size_t)3 * nbands * 4 + (size_t)bvcap * 4 + (size_t)btcap * 2 + 6 * 256;
    return per * nwarps + 4096;
}

static inline char* align_up(char* p, size_t a)
{
    return (char*)(((uintptr_t)p + a - 1) & ~(uintptr_t)(a - 1));
}

void align_scratch_carve(AlignScratch* s, void* base, int nwarps, int pcap, int ptscap, int mcap, int tcap, int nbands,
                         int bvcap, int btcap)
{
    char* p = align_up((char*)base, 256);
    s->nwarps = nwarps;
    s->pcap = pcap;
    s->peb = (int4*)p;
    p = align_up(p + (size_t)pcap * sizeof(int4) * nwarps, 256);
    s->ptscap = ptscap;
    s->pts = (uint16_t*)p;
    p = align_up(p + (size_t)ptscap * 2 * nwarps, 256);
    s->mcap = mcap;
    s->match = (MPath*)p;
    p = align_up(p + (size_t)2 * mcap * sizeof(MPath) * nwarps, 256);
    s->tcap = tcap;
    s->tbuf = (uint16_t*)p;
    p = align_up(p + (size_t)tcap * 2 * nwarps, 256);
    s->nbands = nbands;
    s->bands = (int*)p;
    p = align_up(p + (size_t)3 * nbands * 4 * nwarps, 256);
    s->bvcap = bvcap;
    s->bvec = bvcap ? (int*)p : nullptr;
    p = align_up(p + (size_t)bvcap * 4 * nwarps, 256);
    s->btcap = btcap;
    s->btr = btcap ? (uint16_t*)p : nullptr;
}

// Prefer the smallest shared-memory carveout that holds ctas CTAs of kern: the rest of the SM's
// 256 KB stays L1, which the aligner's reads of the 2-bit words, the pebbles and the trim tables
// depend on
static int prefer_l1(const void* kern, int ctas)
{
    cudaFuncAttributes fa;
    int dev = 0, smsm = 0;
    GD_CUDA(cudaFuncGetAttributes(&fa, kern));
    GD_CUDA(cudaGetDevice(&dev));
    GD_CUDA(cudaDeviceGetAttribute(&smsm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev));
    const long need = (long)ctas * ((long)fa.sharedSizeBytes + 1024);  // 1 KB per CTA is reserved
    int pct = (int)((need * 100 + smsm - 1) / smsm);
    pct = pct < 1 ? 1 : (pct > 100 ? 100 : pct);
    GD_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributePreferredSharedMemoryCarveout, pct));
    return 0;
}

int align_grid(int* grid_out, int wide)
{
    static bool carved = false;  // once per process (the attribute stays with the kernel)
    if (!carved)
    {
        if (prefer_l1((const void*)k_align_pairs<RING>, GD_ALIGN_MINB) ||
            prefer_l1((const void*)k_align_pairs<RING, true>, GD_ALIGN_MINB) ||
            prefer_l1((const void*)k_align_pairs<TEST_RING>, GD_ALIGN_MINB))
            return -1;
        carved = true;
    }
    int dev = 0, nsm = 0, per = 0;
    GD_CUDA(cudaGetDevice(&dev));
    GD_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
    if (wide == 1)
        GD_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_align_pairs<WIDE_RING>,
                                                              warps_of<WIDE_RING>() * 32, 0));
    else if (wide == 2)
        GD_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_align_duo, DUO_WARPS * 32, 0));
    else  // the narrow instances (RING, TEST_RING) have the same shape
        GD_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_align_pairs<RING>, ALIGN_WARPS * 32, 0));
    if (per < 1)
        per = 1;
    *grid_out = nsm * per;
    return 0;
}

int align_warps_per_cta(int wide)
{
    return wide == 1 ? warps_of<WIDE_RING>() : (wide == 2 ? DUO_WARPS : ALIGN_WARPS);
}

int align_slots_per_warp(int wide)
{
    return wide == 2 ? 2 : 1;
}

int launch_align_pairs(const DevBlock& A, const DevBlock& B, const uint64_t* hkey, const uint32_t* hdiag,
                       const uint2* groups, const uint32_t* order, unsigned ngroups, AlignParams p, AlignScratch sc,
                       AlignOut out, unsigned* queue, DevStatus* st, int grid, cudaStream_t s, int wide)
{
    GD_CUDA(cudaMemsetAsync(queue, 0, sizeof(unsigned), s));
    if (ngroups == 0)
        return 0;
    if (wide == 2 && !p.d2 && !p.test_narrow)
        k_align_duo<<<grid, DUO_WARPS * 32, 0, s>>>(A, B, hkey, hdiag, groups, order, ngroups, p, sc, out, queue, st);
    else if (p.d2)
    {
        if (wide == 1)
            k_align_pairs<WIDE_RING, true><<<grid, warps_of<WIDE_RING>() * 32, 0, s>>>(A, B, hkey, hdiag, groups, order,
                                                                                      ngroups, p, sc, out, queue, st);
        else
            k_align_pairs<RING, true><<<grid, ALIGN_WARPS * 32, 0, s>>>(A, B, hkey, hdiag, groups, order, ngroups, p,
                                                                        sc, out, queue, st);
    }
    else if (wide == 1)
        k_align_pairs<WIDE_RING><<<grid, warps_of<WIDE_RING>() * 32, 0, s>>>(A, B, hkey, hdiag, groups, order, ngroups,
                                                                            p, sc, out, queue, st);
    else if (p.test_narrow)
        k_align_pairs<TEST_RING><<<grid, ALIGN_WARPS * 32, 0, s>>>(A, B, hkey, hdiag, groups, order, ngroups, p, sc,
                                                                   out, queue, st);
    else
        k_align_pairs<RING><<<grid, ALIGN_WARPS * 32, 0, s>>>(A, B, hkey, hdiag, groups, order, ngroups, p, sc, out,
                                                              queue, st);
    GD_LAUNCHED(1);
    GD_CUDA(cudaGetLastError());
    return 0;
}

// ------------------------------------------------------------------------------------------
// Local_Alignment batch (tests)
// ------------------------------------------------------------------------------------------

__global__ void __launch_bounds__(ALIGN_WARPS * 32)
    k_la_batch(const uint8_t* abase, const int64_t* aoff, const int32_t* alen, const uint8_t* bbase,
               const int64_t* boff, const int32_t* blen, const int32_t* diag, const int32_t* anti, int nseeds,
               AlignParams P, AlignScratch sc, int32_t* out12, uint16_t* tr, int trstride, int64_t* cells,
               DevStatus* st)
{
    __shared__ WarpSmem<RING> smem[ALIGN_WARPS];
    const int lane = threadIdx.x & 31;
    const int wib = threadIdx.x >> 5;
    const int gw = blockIdx.x * ALIGN_WARPS + wib;
    if (gw >= sc.nwarps)
        return;
    WarpCtx<RING> w;
    w.sm = &smem[wib];
    w.peb = sc.peb + (size_t)gw * sc.pcap;
    w.pcap = sc.pcap;
    w.pts = sc.pts + (size_t)gw * sc.ptscap;
    w.ptscap = sc.ptscap;
    w.st = st;
    w.lane = lane;
    for (int sd = gw; sd < nseeds; sd += sc.nwarps)
    {
        w.err = 0;
        w.cells = 0;
        w.item = sd;
        const uint8_t* aseq = abase + aoff[sd];
        const uint8_t* bseq = bbase + boff[sd];
        local_alignment<RING, false>(w, P, aseq, bseq, nullptr, 0, nullptr, 0, alen[sd], blen[sd], P.comp, diag[sd],
                                     anti[sd]);
        if (w.err)
        {
            if (w.err == 2 && lane == 0)
                gd_fail(st, GD_ERR_BAND_WIDTH, sd, RING);
            continue;
        }
        LAPath a = w.sm->ap, b = w.sm->bp;
        if (a.tlen > trstride / 2 || b.tlen > trstride / 2)
        {
            // the caller's trace stride cannot hold this seed's traces: an error, not a
            // silently shortened trace
            if (lane == 0)
                gd_fail(st, GD_ERR_TRACE_STRIDE, sd, 2 * max(a.tlen, b.tlen));
            continue;
        }
        if (lane == 0)
        {
            int32_t* o = out12 + 12 * (size_t)sd;
            o[0] = a.abpos;
            o[1] = a.bbpos;
            o[2] = a.aepos;
            o[3] = a.bepos;
            o[4] = a.diffs;
            o[5] = a.tlen;
            o[6] = b.abpos;
            o[7] = b.bbpos;
            o[8] = b.aepos;
            o[9] = b.bepos;
            o[10] = b.diffs;
            o[11] = b.tlen;
            cells[sd] = w.cells;
        }
        uint16_t* ta = tr + (size_t)sd * trstride;
        uint16_t* tb = ta + trstride / 2;
        for (int i = lane; i < a.tlen; i += 32)
            ta[i] = w.pts[a.toff + i];
        for (int i = lane; i < b.tlen; i += 32)
            tb[i] = w.pts[b.toff + i];
        __syncwarp();
    }
}

int launch_la_batch(const uint8_t* aseq_base, const int64_t* aoff, const int32_t* alen, const uint8_t* bseq_base,
                    const int64_t* boff, const int32_t* blen, const int32_t* diag, const int32_t* anti, int nseeds,
                    AlignParams p, AlignScratch sc, int32_t* out12, uint16_t* tr, int trstride, int64_t* cells,
                    DevStatus* st, cudaStream_t s)
{
    if (nseeds <= 0)
        return 0;
    int grid = gd_cdiv(sc.nwarps, ALIGN_WARPS);
    k_la_batch<<<grid, ALIGN_WARPS * 32, 0, s>>>(aseq_base, aoff, alen, bseq_base, boff, blen, diag, anti, nseeds, p, sc,
                                                 out12, tr, trstride, cells, st);
    GD_LAUNCHED(1);
    GD_CUDA(cudaGetLastError());
    return 0;
}

}  // namespace gd
