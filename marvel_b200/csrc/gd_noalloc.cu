// gd_noalloc.cu -- Local_Alignment batch whose call path allocates nothing.
//
// Who needs it: a caller that owns all device memory up front and may not allocate once
// it is running -- e.g. a stage inside an application that hands every byte of HBM to its
// own pool allocator, or a latency-critical service loop where cudaMalloc/cudaFree would
// stall on an implicit device synchronization.  Such a caller creates its gd_context and
// sets the alignment spec during initialisation, allocates its own input and output device
// buffers, and then calls gd_local_alignment_batch_noalloc for every batch.
//
// The working memory of the aligner (per-warp pebble arenas and trace-point buffers, and
// the device status word) lives in the file-scope array below, sized once at load time.
// Every GPU that loads the library holds it until the process exits.
#include <mutex>

#include "../../include/gpudalign.h"
#include "gd_align.cuh"

namespace
{

// Two resources bound what one seed may need.  The trace-point slots bound the read length
// up front (checked before launch).  The pebbles -- one per band diagonal each time the
// wave's furthest point on that diagonal crosses an A or a B trace point -- depend on how
// wide the band grows, which no caller knows in advance: a wave spanning L bases of A with
// a band of W diagonals on average needs at most about 2 * W * L / tspace of them, so 65,536
// hold a 150 kbp wave at spacing 100 whose band averages up to ~21 diagonals.  A seed that
// needs more fails the call with GD_ERR_PEBBLES, nothing of that seed written; the
// allocating entry point grows its arena instead.
constexpr int NOALLOC_WARPS = 16;      // 4 CTAs of 4 warps
constexpr int NOALLOC_PCAP = 65536;    // pebbles per warp (each wave of a seed starts it afresh)
constexpr int NOALLOC_PTSCAP = 16384;  // trace-point slots per warp (uint16)
constexpr size_t NOALLOC_STATUS = 256;
constexpr size_t NOALLOC_PEB_BYTES = (size_t)NOALLOC_WARPS * NOALLOC_PCAP * sizeof(int4);
constexpr size_t NOALLOC_PTS_BYTES = (size_t)NOALLOC_WARPS * NOALLOC_PTSCAP * sizeof(uint16_t);
constexpr size_t NOALLOC_BYTES = NOALLOC_STATUS + NOALLOC_PEB_BYTES + NOALLOC_PTS_BYTES;  // 17,301,760 bytes

// The scratch.  Host code must not take its address directly: the name is only a host-side
// stand-in; the device address comes from cudaGetSymbolAddress below.
static __device__ __align__(256) unsigned char gd_noalloc_scratch[NOALLOC_BYTES];

std::mutex g_setup_lock;
void* g_scratch_addr[256] = {nullptr};  // per device ordinal, filled on the first call

}  // namespace

extern "C" int gd_local_alignment_batch_noalloc(gd_context* ctx, const uint8_t* d_abases, const uint8_t* d_bbases,
                                                const int64_t* d_aoff, const int32_t* d_alen, const int64_t* d_boff,
                                                const int32_t* d_blen, const int32_t* d_diag, const int32_t* d_anti,
                                                int nseeds, int maxlen, int comp, int32_t* d_out12, uint16_t* d_trace,
                                                int trstride, int64_t* d_cells, void* stream)
{
    if (!ctx)
    {
        gd_set_error("gd_local_alignment_batch_noalloc: null context");
        return -1;
    }
    int tspace = 0, ave_path = 0, mscore = 0, dscore = 0;
    const int16_t* tables = gd_context_align_tables(ctx, &tspace, &ave_path, &mscore, &dscore);
    if (!tables)
    {
        gd_set_error("gd_local_alignment_batch_noalloc: gd_new_align_spec has not been called on this context");
        return -1;
    }
    if (nseeds < 0 || maxlen < 0 || trstride < 2)
    {
        gd_set_error("gd_local_alignment_batch_noalloc: bad sizes (nseeds %d, maxlen %d, trstride %d)", nseeds, maxlen,
                     trstride);
        return -1;
    }
    // the trace-point buffer of one warp bounds the read length: 4 * maxtp + 16 slots with
    // maxtp = 2 * (maxlen / tspace + 2) (the reference's bound, dalign/align.c:1946-1953)
    long need = 4L * (2L * (maxlen / tspace + 2)) + 16;
    int limit = ((NOALLOC_PTSCAP - 16) / 8 - 2) * tspace + tspace - 1;
    if (need > NOALLOC_PTSCAP)
    {
        gd_set_error("gd_local_alignment_batch_noalloc: reads of %d bp exceed the %d bp this entry point supports "
                     "at trace spacing %d (static scratch of %zu bytes)",
                     maxlen, limit, tspace, NOALLOC_BYTES);
        return -1;
    }
    if (nseeds == 0)
        return 0;

    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 256)
    {
        gd_set_error("gd_local_alignment_batch_noalloc: no current CUDA device");
        return -1;
    }
    void* base = nullptr;
    {
        // once per device, with that device current: the device address of the scratch
        std::lock_guard<std::mutex> g(g_setup_lock);
        if (!g_scratch_addr[dev])
        {
            void* p = nullptr;
            cudaError_t e = cudaGetSymbolAddress(&p, gd_noalloc_scratch);
            if (e != cudaSuccess || !p)
            {
                gd_set_error("gd_local_alignment_batch_noalloc: cudaGetSymbolAddress failed: %s", cudaGetErrorString(e));
                return -1;
            }
            g_scratch_addr[dev] = p;
        }
        base = g_scratch_addr[dev];
    }
    cudaStream_t s = (cudaStream_t)stream;
    DevStatus* st = (DevStatus*)base;
    // the status word must start at zero; pebbles and trace points need no clearing
    if (cudaMemsetAsync(st, 0, sizeof(DevStatus), s) != cudaSuccess)
    {
        gd_set_error("gd_local_alignment_batch_noalloc: status reset failed");
        return -1;
    }
    gd::AlignScratch sc{};
    sc.nwarps = NOALLOC_WARPS;
    sc.pcap = NOALLOC_PCAP;
    sc.peb = (int4*)((unsigned char*)base + NOALLOC_STATUS);
    sc.ptscap = NOALLOC_PTSCAP;
    sc.pts = (uint16_t*)((unsigned char*)base + NOALLOC_STATUS + NOALLOC_PEB_BYTES);
    gd::AlignParams ap{};
    ap.tspace = tspace;
    ap.ave_path = ave_path;
    ap.comp = comp;
    ap.trace8 = tspace <= 125;
    ap.table = tables;
    ap.score = tables + gd::TRIM_TABLE;
    ap.mscore = mscore;
    ap.dscore = dscore;
    if (gd::launch_la_batch(d_abases, d_aoff, d_alen, d_bbases, d_boff, d_blen, d_diag, d_anti, nseeds, ap, sc, d_out12,
                            d_trace, trstride, d_cells, st, s))
        return -1;
    DevStatus hs;
    if (cudaMemcpyAsync(&hs, st, sizeof(hs), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
        cudaStreamSynchronize(s) != cudaSuccess)
    {
        gd_set_error("gd_local_alignment_batch_noalloc: %s", cudaGetErrorString(cudaGetLastError()));
        return -1;
    }
    if (hs.code == GD_ERR_PEBBLES)
    {
        gd_set_error("gd_local_alignment_batch_noalloc: seed %d needs more than the %d pebbles per warp of the static "
                     "scratch (its band is too wide for its length)",
                     hs.where, NOALLOC_PCAP);
        return -1;
    }
    if (hs.code == GD_ERR_TRACE_STRIDE)
    {
        gd_set_error("gd_local_alignment_batch_noalloc: seed %d has a trace longer than trstride / 2 (trstride %d, "
                     "needs %d)",
                     hs.where, trstride, hs.info);
        return -1;
    }
    if (hs.code)
    {
        gd_set_error("gd_local_alignment_batch_noalloc: seed %d failed with code %d (info %d)", hs.where, hs.code,
                     hs.info);
        return -1;
    }
    return 0;
}
