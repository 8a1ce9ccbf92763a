// gd_pipeline.cu -- host orchestration of the overlap path and its C ABI (include/gpudalign.h).
//
// Per Match_Filter call the device runs: run flags + scan over the A index, per-entry pair
// counts against the B index, the count histogram (the host derives the pair cap from it
// exactly as dalign/filter.c:2107-2174 does), per-entry hit counts + scan, hit emission,
// the stable radix sort of hits by (bread, aread, apos), pair-group detection, groups
// ordered longest-first, and the persistent seed-scan/alignment kernel.  The overlaps it
// writes come back to host memory, where Write_Overlap_Buffer's sort and file layout are
// applied.
#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstring>
#include <functional>
#include <string>
#include <vector>

#include "../../include/gpudalign.h"
#include "gd_align.cuh"
#include "gd_filter.cuh"
#include "gd_filter2.cuh"
#include "gd_dust.cuh"
#include "gd_output.cuh"
#include "gd_prims.cuh"
#include "gd_verify.cuh"
#include "gd_triage.cuh"

static_assert(GD_TRI_NPARAM == gd::TRI_NPARAM && GD_TRI_NF == gd::TRI_NF, "triage parameter layout");

static thread_local char g_err[1024] = "";
unsigned long long g_gd_launches = 0;

void gd_set_error(const char* fmt, ...)
{
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_err, sizeof(g_err), fmt, ap);
    va_end(ap);
}

namespace
{

struct DevBuf
{
    void* p = nullptr;
    size_t n = 0;
};

int ensure(DevBuf& b, size_t bytes)
{
    if (bytes == 0)
        bytes = 16;
    if (bytes <= b.n)
        return 0;
    if (b.p)
        cudaFree(b.p);
    b.p = nullptr;
    b.n = 0;
    size_t want = bytes + bytes / 8;
    cudaError_t e = cudaMalloc(&b.p, want);
    if (e != cudaSuccess)
    {
        b.p = nullptr;
        gd_set_error("cudaMalloc of %zu bytes failed: %s", want, cudaGetErrorString(e));
        return -1;
    }
    b.n = want;
    return 0;
}

void release(DevBuf& b)
{
    if (b.p)
        cudaFree(b.p);
    b.p = nullptr;
    b.n = 0;
}

template <typename T>
T* P(DevBuf& b)
{
    return (T*)b.p;
}

// grows b to at least bytes, keeping its first used bytes
int ensure_keep(DevBuf& b, size_t bytes, size_t used, cudaStream_t s)
{
    if (bytes <= b.n)
        return 0;
    size_t want = bytes + bytes / 2;
    void* p = nullptr;
    cudaError_t e = cudaMalloc(&p, want);
    if (e != cudaSuccess)
    {
        gd_set_error("cudaMalloc of %zu bytes failed: %s", want, cudaGetErrorString(e));
        return -1;
    }
    if (used)
    {
        GD_CUDA(cudaMemcpyAsync(p, b.p, used, cudaMemcpyDeviceToDevice, s));
        GD_CUDA(cudaStreamSynchronize(s));
    }
    if (b.p)
        cudaFree(b.p);
    b.p = p;
    b.n = want;
    return 0;
}

struct HostBuf
{
    void* p = nullptr;
    size_t n = 0;
};

int ensure_host(HostBuf& b, size_t bytes)
{
    if (bytes == 0)
        bytes = 16;
    if (bytes <= b.n)
        return 0;
    if (b.p)
        cudaFreeHost(b.p);
    b.p = nullptr;
    b.n = 0;
    size_t want = bytes + bytes / 8;
    cudaError_t e = cudaMallocHost(&b.p, want);
    if (e != cudaSuccess)
    {
        b.p = nullptr;
        gd_set_error("cudaMallocHost of %zu bytes failed: %s", want, cudaGetErrorString(e));
        return -1;
    }
    b.n = want;
    return 0;
}

struct Slot
{
    DevBuf bases, boff, rlen, manno, mdata, pk;
    DevBlock blk{};
    int64_t totlen = 0, nslots = 0;
    int64_t nmask = 0;  // ints of mask interval data
    int has_mask = 0, loaded = 0;
    DevBuf code, read, rpos;
    int64_t nk = -1;
    std::vector<int32_t> hrlen;
};

int bits_for(int64_t maxval)
{
    int b = 1;
    while (b < 63 && (1ll << b) <= maxval)
        b++;
    return b;
}

}  // namespace

struct gd_context
{
    cudaStream_t s = nullptr;
    int kmer = 14, binshift = 6, suppress = 0, hitmin = 35;
    double ave_corr = .70;
    int tspace = 100;
    float freq[4] = {.25f, .25f, .25f, .25f};
    int symmetric = 1, only_identity = 0, no_trace = 0;
    int minover = 2000, identity = 0;
    uint64_t mem_limit = 0;
    int ave_path = 0, mscore = 0, dscore = 0;
    int spec_set = 0;
    DevBuf tables;
    Slot slot[3];
    DevBuf k0, v0, k1, v1, scratch, flags, excl, jb, cnt, hoff, ctrun, gram, misc;
    DevBuf hk0, hd0, hk1, hd1, starts, groups, gcost, gidx, gcost2, gidx2;
    uint64_t* hkey = nullptr;
    uint32_t* hdiag = nullptr;
    int64_t nhits = 0;
    gd::HitBits hb{};
    DevBuf ascr, outrec, outtr, counters, status, queue;
    int agrid = 0;
    DevBuf ascr_w, wide;  // the wide aligner instance's scratch, and its group list + count
    int agrid_w = 0;
    DevBuf ascr_d;        // the duo instance's scratch
    int agrid_d = 0;
    int test_narrow = 0;  // tests only: the main aligner pass with the 32-diagonal instance
    // aligner schedule: empty = every pair group in one persistent launch (longest first from
    // the device queue); else one launch per length class, split at these alen + blen edges
    std::vector<int32_t> sched_edges;
    std::vector<int32_t> sched_kind;  // per length class (longest first): 0 = RING instance, 1 = WIDE_RING
    int variant = 1, hgap = 0;  // 2 = daligner2 (modimizer seeds, dalign2/), its -H
    int biased = 0;             // daligner -b: frequency-weighted tuples
    // -b: the reads' first chunks, tuples per chunk (then offsets), unpacked (read, position)
    DevBuf bchunk, bcount, brp;
    DevBuf d2rd, d2rp, d2sgn, cnt2, hoff2, hk2, hd2, runstart, btable;
    int pcap = 32768, mcap = 1024, tcap = 1 << 17;
    int bvcap = 8192, btcap = 1024;  // daligner2 bridging scratch per warp (ints, trace values)
    uint64_t rcap = 1 << 22, tbcap = 512ull << 20;
    // the overlap buffer: records and trace bytes of every Match_Filter since the last reset,
    // in HBM in emission order (acc_*), and its sorted, compacted copy (srt_*)
    DevBuf acc_rec, acc_tr, srt_rec, srt_tr, okey0, okey1, oval0, oval1, olen;
    uint64_t acc_n = 0, acc_tb = 0, srt_n = 0, srt_tb = 0;
    bool srt_valid = false;
    HostBuf h_rec, h_tr;  // pinned staging for file writes
    DevBuf las_raw, las_off, las_rec, las_out;  // gd_las_sort
    gd_stats stats;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr, tev0 = nullptr, tev1 = nullptr;
    // learned triage: model (on), per-group feature/outcome collection (collect)
    int tri_on = 0, tri_collect = 0;
    float tri_thr = 0.f;
    DevBuf tri_params, tri_feat, tri_prob, tri_skip, tri_gstat, tri_misc;
    DevBuf tri_x, tri_y, tri_perm, tri_grad, tri_m, tri_v, tri_loss, tri_w;
    std::vector<float> tri_hfeat;
    std::vector<uint32_t> tri_hrec, tri_hcells;
};

// ----------------------------------------------------------------------------------------
// align spec: trim tables (set_table / New_Align_Spec, dalign/align.c:196-279)
// ----------------------------------------------------------------------------------------

static const double kBias[10] = {.690, .690, .690, .690, .780, .850, .900, .933, .966, 1.000};

static void set_table(int bit, int prefix, int score, int max, int mscore, int dscore, int16_t* table, int16_t* sc)
{
    if (bit >= 15)
    {
        table[prefix] = (int16_t)(score - max);
        sc[prefix] = (int16_t)score;
    }
    else
    {
        if (score > max)
            max = score;
        set_table(bit + 1, prefix << 1, score - dscore, max, mscore, dscore, table, sc);
        set_table(bit + 1, (prefix << 1) | 1, score + mscore, max, mscore, dscore, table, sc);
    }
}

static int upload_spec(gd_context* c)
{
    double match = c->freq[0] + c->freq[3];
    if (match > .5)
        match = 1. - match;
    int bias = (int)((match + .025) * 20. - 1.);
    if (match < .2)
    {
        fprintf(stderr, "Warning: Base bias worse than 80/20%% ! (New_Align_Spec)\n");
        fprintf(stderr, "         Capping bias at this ratio.\n");
        bias = 3;
    }
    c->ave_path = (int)(60 * (1. - kBias[bias] * (1. - c->ave_corr)));
    int mscore = (int)(1000 * kBias[bias] * (1. - c->ave_corr));
    int dscore = 1000 - mscore;
    c->mscore = mscore;
    c->dscore = dscore;
    std::vector<int16_t> t(2 * gd::TRIM_TABLE);
    set_table(0, 0, 0, 0, mscore, dscore, t.data(), t.data() + gd::TRIM_TABLE);
    if (ensure(c->tables, t.size() * 2))
        return -1;
    // on the context's stream: its kernels must see the tables (the stream does not order
    // against the legacy default stream)
    GD_CUDA(cudaMemcpyAsync(c->tables.p, t.data(), t.size() * 2, cudaMemcpyHostToDevice, c->s));
    GD_CUDA(cudaStreamSynchronize(c->s));
    return 0;
}

// ----------------------------------------------------------------------------------------
// k-mer index (Sort_Kmers)
// ----------------------------------------------------------------------------------------

template <typename K>
static int suppress_index(gd_context* c, Slot& sl, int64_t& n);

template <typename K>
static int64_t index_slot_t(gd_context* c, Slot& sl)
{
    using namespace gd;
    const int Kmer = c->kmer;
    int64_t nslots = sl.nslots;
    cudaStream_t s = c->s;
    sl.nk = 0;
    if (nslots <= 0)
        return 0;
    if (ensure(c->k0, nslots * sizeof(K)) || ensure(c->k1, nslots * 8) || ensure(c->v0, nslots * 4) ||
        ensure(c->v1, nslots * 4) || ensure(c->scratch, radix_scratch_bytes(nslots)) || ensure(c->misc, 64))
        return -1;
    uint32_t* nmasked = P<uint32_t>(c->misc);
    // sort values carry (read, first position) when both fit in 32 bits, else the slot index
    const int pb = bits_for(std::max(sl.blk.maxlen - Kmer, 1));
    const int pbits = (bits_for(std::max(sl.blk.nreads - 1, 1)) + pb <= 32) ? pb : -1;
    if (launch_extract<K>(sl.blk, sl.has_mask ? P<int64_t>(sl.manno) : nullptr,
                          sl.has_mask ? P<int32_t>(sl.mdata) : nullptr, Kmer, P<K>(c->k0), P<uint32_t>(c->v0), nslots,
                          nmasked, pbits, s))
        return -1;
    int sort_bits = 8 * ((2 * Kmer + 7) / 8);  // mersort bytes (filter.c:713-716)
    // A masked slot's key is all ones.  When the sorted bytes end at the code's top bit (k a
    // multiple of 4) that ties with the poly-T code, and cutting the masked count off the end
    // could then keep masked slots and drop real k-mers (the reference's own result there
    // depends on its thread split: its pads sit at the end of each thread's part of the list).
    // One more byte puts every masked slot behind every k-mer.
    if (sl.has_mask && (2 * Kmer) % 8 == 0)
        sort_bits += 8;
    if (sort_bits > (int)(8 * sizeof(K)))
        sort_bits = 8 * sizeof(K);
    // with packed values the last pass writes the index arrays itself (masked slots, sorted to
    // the end, included: the arrays hold every slot)
    const bool fused = pbits >= 0 && nslots > 1;
    RsFinal fin;
    if (fused)
    {
        if (ensure(sl.code, (nslots + 1) * sizeof(K)) || ensure(sl.read, (nslots + 1) * 4) ||
            ensure(sl.rpos, (nslots + 1) * 4))
            return -1;
        fin.kind = RsFinal::INDEX;
        fin.a = sl.code.p;
        fin.b = P<int32_t>(sl.read);
        fin.c = P<int32_t>(sl.rpos);
        fin.bits = pbits;
        fin.kmer = Kmer;
    }
    int which = radix_sort_pairs<K>(P<K>(c->k0), P<uint32_t>(c->v0), P<K>(c->k1), P<uint32_t>(c->v1), nslots, 0,
                                    sort_bits, c->scratch.p, s, fused ? &fin : nullptr);
    if (which < 0)
        return -1;
    K* skeys = which ? P<K>(c->k1) : P<K>(c->k0);
    uint32_t* svals = which ? P<uint32_t>(c->v1) : P<uint32_t>(c->v0);
    uint32_t hmask = 0;
    GD_CUDA(cudaMemcpyAsync(&hmask, nmasked, 4, cudaMemcpyDeviceToHost, s));
    GD_CUDA(cudaStreamSynchronize(s));
    int64_t n = nslots - hmask;
    if (ensure(sl.code, (n + 1) * sizeof(K)) || ensure(sl.read, (n + 1) * 4) || ensure(sl.rpos, (n + 1) * 4))
        return -1;
    if (fused)
    {
        // the sort's last pass wrote the index arrays
    }
    else if (pbits >= 0)
    {
        if (launch_unpack<K>(skeys, svals, n, pbits, Kmer, P<K>(sl.code), P<int32_t>(sl.read), P<int32_t>(sl.rpos), s))
            return -1;
    }
    else
    {
        GD_CUDA(cudaMemcpyAsync(sl.code.p, skeys, n * sizeof(K), cudaMemcpyDeviceToDevice, s));
        if (launch_decode<K>(sl.blk, Kmer, svals, n, P<int32_t>(sl.read), P<int32_t>(sl.rpos), s))
            return -1;
    }
    if (suppress_index<K>(c, sl, n))
        return -1;
    GD_CUDA(cudaStreamSynchronize(s));
    sl.nk = n;
    return n;
}

// -b weights from the frequencies of the align spec (Sort_Kmers, dalign/filter.c:718-733: the
// reference takes them once, from the first block it indexes, daligner's A block, whose
// frequencies are the ones New_Align_Spec gets).  The table is made on the host with the
// reference's own double expression.
static int bias_params(const gd_context* c, gd::BiasParams& bp)
{
    const double scale = -10000. / ::log(4.);
    for (int i = 0; i < 4; i++)
    {
        if (!(c->freq[i] > 0.f && c->freq[i] <= 1.f))
        {
            gd_set_error("-b needs base frequencies in (0, 1], got %g for base %d", (double)c->freq[i], i);
            return -1;
        }
        bp.w[i] = (int)::ceil(scale * ::log((double)c->freq[i]));  // the float widened, as in C
    }
    bp.norm = 10000 * c->kmer;
    bp.thresh = 10000 * (c->kmer - 2);
    bp.kmer = c->kmer;
    return 0;
}

// Sort_Kmers with -b: the reads cut into chunks of positions, one scan per chunk counts its
// tuples, a scan of the counts places them, a second scan writes them; then the sort and -t as
// for the plain index.  Entries come out in (read, position) order before the sort, as the
// reference's threads list them.
template <typename K>
static int64_t index_slot_bias_t(gd_context* c, Slot& sl)
{
    using namespace gd;
    const int Kmer = c->kmer;
    const int nr = sl.blk.nreads;
    cudaStream_t s = c->s;
    sl.nk = 0;
    if (nr <= 0)
        return 0;
    BiasParams bp;
    if (bias_params(c, bp))
        return -1;
    // chunk counts, tuple counts and offsets are 32-bit: at most one tuple per position and
    // one more per unmasked segment
    if (sl.totlen + 2 * (int64_t)nr + (sl.has_mask ? sl.nmask : 0) > 0xffffffffll)
    {
        gd_set_error("-b index of a %lld-base block exceeds this build's 32-bit tuple offsets",
                     (long long)sl.totlen);
        return -1;
    }
    const int64_t* manno = sl.has_mask ? P<int64_t>(sl.manno) : nullptr;
    const int32_t* mdata = sl.has_mask ? P<int32_t>(sl.mdata) : nullptr;
    if (ensure(c->bchunk, (nr + 1) * 4) || ensure(c->misc, 64) ||
        ensure(c->scratch, scan_scratch_bytes<uint32_t>(nr)))
        return -1;
    uint32_t* cfirst = P<uint32_t>(c->bchunk);
    uint32_t* total = P<uint32_t>(c->misc);
    uint32_t hn = 0;
    if (bias_chunks(sl.blk, cfirst, total, c->scratch.p, s))
        return -1;
    GD_CUDA(cudaMemcpyAsync(&hn, total, 4, cudaMemcpyDeviceToHost, s));
    GD_CUDA(cudaStreamSynchronize(s));
    const uint32_t nchunks = hn;
    if (ensure(c->bcount, ((int64_t)nchunks + 1) * 4) || ensure(c->scratch, scan_scratch_bytes<uint32_t>(nchunks)))
        return -1;
    uint32_t* count = P<uint32_t>(c->bcount);
    if (launch_bias_count(sl.blk, manno, mdata, bp, cfirst, nchunks, count, s) ||
        exclusive_scan<uint32_t>(count, count, nchunks, total, c->scratch.p, s))
        return -1;
    GD_CUDA(cudaMemcpyAsync(&hn, total, 4, cudaMemcpyDeviceToHost, s));
    GD_CUDA(cudaStreamSynchronize(s));
    int64_t n = hn;
    if (n == 0)
        return 0;
    // positions run to maxlen (a tracked tuple can sit at rlen)
    const int pb = bits_for(std::max(sl.blk.maxlen, 1));
    const int pbits = (bits_for(std::max(nr - 1, 1)) + pb <= 32) ? pb : -1;
    if (ensure(c->k0, n * sizeof(K)) || ensure(c->k1, n * 8) || ensure(c->v0, n * 4) || ensure(c->v1, n * 4) ||
        ensure(c->scratch, radix_scratch_bytes(n)) || ensure(sl.code, (n + 1) * sizeof(K)) ||
        ensure(sl.read, (n + 1) * 4) || ensure(sl.rpos, (n + 1) * 4) || (pbits < 0 && ensure(c->brp, n * 8)))
        return -1;
    int32_t* eread = pbits < 0 ? P<int32_t>(c->brp) : nullptr;
    int32_t* erpos = pbits < 0 ? eread + n : nullptr;
    if (launch_bias_emit<K>(sl.blk, manno, mdata, bp, cfirst, nchunks, count, P<K>(c->k0), P<uint32_t>(c->v0), eread,
                            erpos, pbits, s))
        return -1;
    int sort_bits = 8 * ((2 * Kmer + 7) / 8);  // mersort bytes (filter.c:713-716)
    if (sort_bits > (int)(8 * sizeof(K)))
        sort_bits = 8 * sizeof(K);
    const bool fused = pbits >= 0 && n > 1;
    RsFinal fin;
    if (fused)
    {
        fin.kind = RsFinal::INDEX;
        fin.a = sl.code.p;
        fin.b = P<int32_t>(sl.read);
        fin.c = P<int32_t>(sl.rpos);
        fin.bits = pbits;
        fin.kmer = 1;  // the value holds the position itself
    }
    int which = radix_sort_pairs<K>(P<K>(c->k0), P<uint32_t>(c->v0), P<K>(c->k1), P<uint32_t>(c->v1), n, 0,
                                    sort_bits, c->scratch.p, s, fused ? &fin : nullptr);
    if (which < 0)
        return -1;
    K* skeys = which ? P<K>(c->k1) : P<K>(c->k0);
    uint32_t* svals = which ? P<uint32_t>(c->v1) : P<uint32_t>(c->v0);
    if (fused)
    {
        // the sort's last pass wrote the index arrays
    }
    else if (pbits >= 0)
    {
        if (launch_unpack<K>(skeys, svals, n, pbits, 1, P<K>(sl.code), P<int32_t>(sl.read), P<int32_t>(sl.rpos), s))
            return -1;
    }
    else
    {
        GD_CUDA(cudaMemcpyAsync(sl.code.p, skeys, n * sizeof(K), cudaMemcpyDeviceToDevice, s));
        if (launch_gather_read_pos(svals, n, eread, erpos, P<int32_t>(sl.read), P<int32_t>(sl.rpos), s))
            return -1;
    }
    if (suppress_index<K>(c, sl, n))
        return -1;
    GD_CUDA(cudaStreamSynchronize(s));
    sl.nk = n;
    return n;
}

// -t: drop codes occurring >= t times (compsize/compress_thread, filter.c:645-696 and
// dalign2/filter.c:771-832); k0, k1 (2n int32), v0 and v1 hold at least n entries
template <typename K>
static int suppress_index(gd_context* c, Slot& sl, int64_t& n)
{
    using namespace gd;
    cudaStream_t s = c->s;
    if (c->suppress > 0 && n > 0)
    {
        uint32_t* keep = P<uint32_t>(c->v0);
        uint32_t* pos = P<uint32_t>(c->v1);
        if (ensure(c->misc, 64))
            return -1;
        uint32_t* tot = P<uint32_t>(c->misc) + 4;
        if (launch_suppress_flags<K>(P<K>(sl.code), n, c->suppress, keep, s) ||
            exclusive_scan<uint32_t>(keep, pos, n, tot, c->scratch.p, s))
            return -1;
        uint32_t kept = 0;
        GD_CUDA(cudaMemcpyAsync(&kept, tot, 4, cudaMemcpyDeviceToHost, s));
        // compact into k0 / v-buffers then copy back
        K* code2 = P<K>(c->k0);
        int32_t* read2 = (int32_t*)P<K>(c->k1);
        int32_t* rpos2 = read2 + n;
        if (launch_compact_index<K>(P<K>(sl.code), P<int32_t>(sl.read), P<int32_t>(sl.rpos), keep, pos, n, code2,
                                    read2, rpos2, s))
            return -1;
        GD_CUDA(cudaStreamSynchronize(s));
        GD_CUDA(cudaMemcpyAsync(sl.code.p, code2, kept * sizeof(K), cudaMemcpyDeviceToDevice, s));
        GD_CUDA(cudaMemcpyAsync(sl.read.p, read2, kept * 4ull, cudaMemcpyDeviceToDevice, s));
        GD_CUDA(cudaMemcpyAsync(sl.rpos.p, rpos2, kept * 4ull, cudaMemcpyDeviceToDevice, s));
        n = kept;
    }
    return 0;
}

// daligner2's Sort_Kmers (dalign2/filter.c:834-1106): the modimizer list in the reference's
// order (per slot counts, their scan, emission), the stable radix sort on (k-1)/4+1 code
// bytes, the gather of (read << 1 | strand, position), -t.
template <typename K>
static int64_t index_slot_d2_t(gd_context* c, Slot& sl)
{
    using namespace gd;
    const int Kmer = c->kmer;
    const int64_t nslots = sl.nslots;
    cudaStream_t s = c->s;
    sl.nk = 0;
    if (nslots <= 0)
        return 0;
    const D2Masks M = d2_masks(Kmer);
    const int64_t* manno = sl.has_mask ? P<int64_t>(sl.manno) : nullptr;
    const int32_t* mdata = sl.has_mask ? P<int32_t>(sl.mdata) : nullptr;
    if (ensure(c->flags, nslots * 4) || ensure(c->excl, nslots * 4 + 4) ||
        ensure(c->scratch, scan_scratch_bytes<uint32_t>(nslots)) || ensure(c->misc, 64))
        return -1;
    uint32_t* d_tot = P<uint32_t>(c->misc) + 4;
    if (launch_d2_count(sl.blk, manno, mdata, Kmer, M, nslots, P<uint32_t>(c->flags), s) ||
        exclusive_scan<uint32_t>(P<uint32_t>(c->flags), P<uint32_t>(c->excl), nslots, d_tot, c->scratch.p, s))
        return -1;
    uint32_t ne = 0;
    GD_CUDA(cudaMemcpyAsync(&ne, d_tot, 4, cudaMemcpyDeviceToHost, s));
    GD_CUDA(cudaStreamSynchronize(s));
    int64_t n = ne;
    if (n == 0)
        return 0;
    if (ensure(c->k0, n * sizeof(K)) || ensure(c->k1, n * 8) || ensure(c->v0, n * 4) || ensure(c->v1, n * 4) ||
        ensure(c->d2rd, n * 4) || ensure(c->d2rp, n * 4) || ensure(c->scratch, radix_scratch_bytes(n)) ||
        ensure(sl.code, (n + 1) * sizeof(K)) || ensure(sl.read, (n + 1) * 4) || ensure(sl.rpos, (n + 1) * 4))
        return -1;
    if (launch_d2_emit<K>(sl.blk, manno, mdata, Kmer, M, nslots, P<uint32_t>(c->excl), P<K>(c->k0),
                          P<uint32_t>(c->v0), P<int32_t>(c->d2rd), P<int32_t>(c->d2rp), s))
        return -1;
    int sort_bits = 8 * ((Kmer - 1) / 4 + 1);  // mersort bytes (dalign2/filter.c:942-953)
    if (sort_bits > (int)(8 * sizeof(K)))
        sort_bits = 8 * sizeof(K);
    int which = radix_sort_pairs<K>(P<K>(c->k0), P<uint32_t>(c->v0), P<K>(c->k1), P<uint32_t>(c->v1), n, 0,
                                    sort_bits, c->scratch.p, s);
    if (which < 0)
        return -1;
    if (launch_d2_gather<K>(which ? P<K>(c->k1) : P<K>(c->k0), which ? P<uint32_t>(c->v1) : P<uint32_t>(c->v0), n,
                            P<int32_t>(c->d2rd), P<int32_t>(c->d2rp), P<K>(sl.code), P<int32_t>(sl.read),
                            P<int32_t>(sl.rpos), s))
        return -1;
    if (suppress_index<K>(c, sl, n))
        return -1;
    GD_CUDA(cudaStreamSynchronize(s));
    sl.nk = n;
    return n;
}

// ----------------------------------------------------------------------------------------
// Match_Filter
// ----------------------------------------------------------------------------------------

// appends the features and plain-path outcome (records, cells) of the last call's groups
static int tri_append(gd_context* c, unsigned ng)
{
    size_t f0 = c->tri_hfeat.size(), g0 = c->tri_hrec.size();
    c->tri_hfeat.resize(f0 + (size_t)ng * gd::TRI_NF);
    std::vector<uint2> st(ng);
    GD_CUDA(cudaMemcpy(c->tri_hfeat.data() + f0, c->tri_feat.p, (size_t)ng * gd::TRI_NF * 4, cudaMemcpyDeviceToHost));
    GD_CUDA(cudaMemcpy(st.data(), c->tri_gstat.p, (size_t)ng * 8, cudaMemcpyDeviceToHost));
    c->tri_hrec.resize(g0 + ng);
    c->tri_hcells.resize(g0 + ng);
    for (unsigned i = 0; i < ng; i++)
    {
        c->tri_hrec[g0 + i] = st[i].x;
        c->tri_hcells[g0 + i] = st[i].y;
    }
    return 0;
}

static int align_hits(gd_context* c, Slot& A, Slot& B, uint64_t nhits, gd::HitBits hb, int comp, int self);

// bits of a tuple position in a block: at most maxlen - 1, or maxlen with -b (a tuple that
// growing pushed to the end of an unmasked segment, dalign/filter.c:545-551)
static int pos_bits(const gd_context* c, const Slot& S)
{
    return bits_for(std::max(S.blk.maxlen - (c->biased ? 0 : 1), 1));
}

// bits of the B position when (bread, aread, apos, bpos) fits one 64-bit word, else 0
static int hit_qbits(const gd_context* c, const gd::HitBits& hb, const Slot& B)
{
    const int q = pos_bits(c, B);
    return hb.pbits + hb.abits + hb.bbits + q <= 64 ? q : 0;
}
static int pair_cap(gd_context* c, int64_t na, int64_t nb, int same_index, int* limit_out);
template <typename K>
static int match_emit_t(gd_context* c, Slot& A, Slot& B, int64_t na, uint64_t* d_nhits, int comp, int self);

template <typename K>
static int match_filter_t(gd_context* c, int bslot, int comp, int self)
{
    using namespace gd;
    cudaStream_t s = c->s;
    Slot& A = c->slot[0];
    Slot& B = c->slot[bslot];
    int oi = comp ? 1 : 0;
    c->stats.hits[oi] = c->stats.groups[oi] = c->stats.seeds[oi] = c->stats.cells[oi] = 0;
    c->stats.skipped[oi] = 0;
    c->stats.wide[oi] = 0;
    c->stats.ms_merge[oi] = c->stats.ms_align[oi] = 0;
    c->nhits = 0;
    int64_t na = A.nk, nb = B.nk;
    if (na <= 0 || nb <= 0)
        return 0;
    GD_CUDA(cudaEventRecord(c->ev0, s));
    // run ids of the A index
    if (ensure(c->flags, na * 4) || ensure(c->excl, na * 4) || ensure(c->jb, na * 4) || ensure(c->cnt, na * 8) ||
        ensure(c->hoff, na * 8) || ensure(c->scratch, std::max(scan_scratch_bytes<uint64_t>(na), (size_t)4096)) ||
        ensure(c->misc, 256) || ensure(c->gram, MAXGRAM * 8))
        return -1;
    uint32_t* d_nruns = P<uint32_t>(c->misc) + 8;
    if (launch_run_flags<K>(P<K>(A.code), na, P<uint32_t>(c->flags), s) ||
        exclusive_scan<uint32_t>(P<uint32_t>(c->flags), P<uint32_t>(c->excl), na, d_nruns, c->scratch.p, s))
        return -1;
    uint32_t nruns = 0;
    GD_CUDA(cudaMemcpyAsync(&nruns, d_nruns, 4, cudaMemcpyDeviceToHost, s));
    GD_CUDA(cudaStreamSynchronize(s));
    if (ensure(c->ctrun, (size_t)nruns * 8 + 8))
        return -1;
    GD_CUDA(cudaMemsetAsync(c->ctrun.p, 0, (size_t)nruns * 8, s));
    MergeArgs m{na, nb, self, c->identity, comp, nullptr, nullptr, 0, 0};
    if (&B == &A)  // the block against its own index: run bounds without searches
    {
        if (ensure(c->runstart, ((size_t)nruns + 1) * 4) ||
            launch_run_starts(P<uint32_t>(c->flags), P<uint32_t>(c->excl), na, nruns, P<uint32_t>(c->runstart), s))
            return -1;
        m.runstart = P<uint32_t>(c->runstart);
    }
    else  // the B index's bucket table: each search stays inside its code's bucket
    {
        m.bshift = bucket_shift(c->kmer);
        m.nbuckets = bucket_count(c->kmer);
        const uint32_t nbk = m.nbuckets;
        if (ensure(c->btable, ((size_t)nbk + 2) * 4) ||
            launch_code_buckets<K>(P<K>(B.code), nb, m.bshift, nbk, P<uint32_t>(c->btable), s))
            return -1;
        m.btable = P<uint32_t>(c->btable);
    }
    if (launch_pair_count<K>(P<K>(A.code), P<int32_t>(A.read), P<int32_t>(A.rpos), P<uint32_t>(c->excl),
                             P<uint32_t>(c->flags), P<K>(B.code), P<int32_t>(B.read), P<int32_t>(B.rpos), m,
                             P<uint32_t>(c->jb), P<uint64_t>(c->cnt), P<unsigned long long>(c->ctrun), s) ||
        launch_gram(P<unsigned long long>(c->ctrun), nruns, P<unsigned long long>(c->gram), s))
        return -1;
    int limit;
    if (pair_cap(c, na, nb, self && !comp, &limit))  // asort == bsort only for the self N call
        return -1;
    c->stats.limit[oi] = limit;
    uint64_t* d_nhits = (uint64_t*)(P<uint32_t>(c->misc) + 16);
    if (launch_cnt_mask(P<uint32_t>(c->excl), P<uint32_t>(c->flags), P<unsigned long long>(c->ctrun), na, limit,
                        self && c->identity && comp, P<uint64_t>(c->cnt), s) ||
        exclusive_scan<uint64_t>(P<uint64_t>(c->cnt), P<uint64_t>(c->hoff), na, d_nhits, c->scratch.p, s))
        return -1;
    return match_emit_t<K>(c, A, B, na, d_nhits, comp, self);
}

// The pair cap from the memory limit (filter.c:2107-2174, dalign2/filter.c:2430-2480), from
// the histogram of per-code pair counts in c->gram.
static int pair_cap(gd_context* c, int64_t na, int64_t nb, int same_index, int* limit_out)
{
    using namespace gd;
    cudaStream_t s = c->s;
    std::vector<unsigned long long> gram(MAXGRAM);
    GD_CUDA(cudaMemcpyAsync(gram.data(), c->gram.p, MAXGRAM * 8, cudaMemcpyDeviceToHost, s));
    GD_CUDA(cudaStreamSynchronize(s));
    int limit = INT32_MAX;
    if (c->mem_limit > 0)
    {
        int64_t avail;
        uint64_t dsz = c->mem_limit / 16;
        if (same_index || (int64_t)dsz > na + 2 * nb)
            avail = ((int64_t)dsz - na) / 2;
        else
            avail = (int64_t)dsz - (na + nb);
        avail = (int64_t)(avail * .98);
        int64_t tom = 0;
        int j;
        for (j = 0; j < MAXGRAM; j++)
        {
            tom += (int64_t)j * (int64_t)gram[j];
            if (tom > avail)
                break;
        }
        limit = j;
        if (limit == 1)
        {
            gd_set_error("Insufficient memory allocation (%.1fGb), reduce block size or increase allocation",
                         (1. * c->mem_limit) / 0x40000000ll);
            return -1;
        }
        if (limit < 10)
            fprintf(stderr, "\nWarning: Sensitivity hampered by low memory allocation (%.1fGb)\n",
                    (1. * c->mem_limit) / 0x40000000ll);
    }
    *limit_out = limit;
    return 0;
}

// daligner's emission of one orientation's hits (merge_thread, filter.c:1061-1231) after the
// per-entry counts are capped and scanned, then the hit sort, groups and alignment.
template <typename K>
static int match_emit_t(gd_context* c, Slot& A, Slot& B, int64_t na, uint64_t* d_nhits, int comp, int self)
{
    using namespace gd;
    cudaStream_t s = c->s;
    const int oi = comp ? 1 : 0;
    uint64_t nhits = 0;
    GD_CUDA(cudaMemcpyAsync(&nhits, d_nhits, 8, cudaMemcpyDeviceToHost, s));
    GD_CUDA(cudaStreamSynchronize(s));
    c->stats.hits[oi] = (int64_t)nhits;
    if (nhits == 0)
        return 0;
    if (nhits > 0xffffffffull)
    {
        gd_set_error("%llu hits exceed the 32-bit hit index of this build", (unsigned long long)nhits);
        return -1;
    }
    HitBits hb;
    hb.pbits = pos_bits(c, A);
    hb.abits = bits_for(std::max(A.blk.nreads - 1, 1));
    hb.bbits = bits_for(std::max(B.blk.nreads - 1, 1));
    int hbits = hb.pbits + hb.abits + hb.bbits;
    if (hbits > 64)
    {
        gd_set_error("hit key needs %d bits (> 64): block too large for this build", hbits);
        return -1;
    }
    hb.qbits = hit_qbits(c, hb, B);
    if (ensure(c->hk0, nhits * 8) || ensure(c->hk1, nhits * 8) || ensure(c->hd0, nhits * 4) ||
        ensure(c->hd1, nhits * 4) || ensure(c->scratch, radix_scratch_bytes(nhits)))
        return -1;
    if (launch_emit(P<int32_t>(A.read), P<int32_t>(A.rpos), P<int32_t>(B.read), P<int32_t>(B.rpos),
                    P<uint32_t>(c->jb), P<uint64_t>(c->cnt), P<uint64_t>(c->hoff), na, hb, P<uint64_t>(c->hk0),
                    P<uint32_t>(c->hd0), s))
        return -1;
    return align_hits(c, A, B, nhits, hb, comp, self);
}

// daligner2's Match_Filter (dalign2/filter.c:2344-2700) for A (slot 0) against B (bslot),
// both orientations from one join: per A entry the B range of its code split by strand
// agreement, the pair cap over both, and the hits of each orientation in generation order;
// then each orientation's hit sort, groups and alignment (complement groups against the
// complemented B block in cslot).
template <typename K>
static int match_filter_d2_t(gd_context* c, int bslot, int cslot, int self)
{
    using namespace gd;
    cudaStream_t s = c->s;
    Slot& A = c->slot[0];
    Slot& B = c->slot[bslot];
    Slot& C = c->slot[cslot];
    for (int oi = 0; oi < 2; oi++)
    {
        c->stats.hits[oi] = c->stats.groups[oi] = c->stats.seeds[oi] = c->stats.cells[oi] = 0;
        c->stats.skipped[oi] = 0;
        c->stats.wide[oi] = 0;
        c->stats.ms_merge[oi] = c->stats.ms_align[oi] = 0;
    }
    c->nhits = 0;
    const int64_t na = A.nk, nb = B.nk;
    if (na <= 0 || nb <= 0)
        return 0;
    GD_CUDA(cudaEventRecord(c->ev0, s));
    if (ensure(c->flags, na * 4) || ensure(c->excl, na * 4) || ensure(c->jb, na * 4) || ensure(c->cnt, na * 8) ||
        ensure(c->cnt2, na * 8) || ensure(c->hoff, na * 8) || ensure(c->hoff2, na * 8) ||
        ensure(c->d2sgn, (nb + 1) * 4) ||
        ensure(c->scratch, std::max(std::max(scan_scratch_bytes<uint64_t>(na), scan_scratch_bytes<uint32_t>(nb)),
                                    (size_t)4096)) ||
        ensure(c->misc, 256) || ensure(c->gram, MAXGRAM * 8))
        return -1;
    uint32_t* d_nruns = P<uint32_t>(c->misc) + 8;
    uint32_t* sgn = P<uint32_t>(c->d2sgn);
    if (launch_run_flags<K>(P<K>(A.code), na, P<uint32_t>(c->flags), s) ||
        exclusive_scan<uint32_t>(P<uint32_t>(c->flags), P<uint32_t>(c->excl), na, d_nruns, c->scratch.p, s) ||
        launch_d2_strand_flags(P<int32_t>(B.read), nb, sgn, s) ||
        exclusive_scan<uint32_t>(sgn, sgn, nb, sgn + nb, c->scratch.p, s))
        return -1;
    uint32_t nruns = 0;
    GD_CUDA(cudaMemcpyAsync(&nruns, d_nruns, 4, cudaMemcpyDeviceToHost, s));
    GD_CUDA(cudaStreamSynchronize(s));
    if (ensure(c->ctrun, (size_t)nruns * 8 + 8))
        return -1;
    GD_CUDA(cudaMemsetAsync(c->ctrun.p, 0, (size_t)nruns * 8, s));
    const uint32_t* runstart = nullptr;
    const uint32_t* btable = nullptr;
    const int bshift = bucket_shift(c->kmer);
    const uint32_t nbk = bucket_count(c->kmer);
    if (&B == &A)  // the block against its own index: run bounds without searches
    {
        if (ensure(c->runstart, ((size_t)nruns + 1) * 4) ||
            launch_run_starts(P<uint32_t>(c->flags), P<uint32_t>(c->excl), na, nruns, P<uint32_t>(c->runstart), s))
            return -1;
        runstart = P<uint32_t>(c->runstart);
    }
    else  // the B index's bucket table: each search stays inside its code's bucket
    {
        if (ensure(c->btable, ((size_t)nbk + 2) * 4) ||
            launch_code_buckets<K>(P<K>(B.code), nb, bshift, nbk, P<uint32_t>(c->btable), s))
            return -1;
        btable = P<uint32_t>(c->btable);
    }
    if (launch_d2_pair_count<K>(P<K>(A.code), P<int32_t>(A.read), P<uint32_t>(c->excl), P<uint32_t>(c->flags),
                                runstart, btable, bshift, nbk, P<K>(B.code), P<int32_t>(B.read), sgn, na, nb, self, c->identity,
                                P<uint32_t>(c->jb), P<uint64_t>(c->cnt), P<uint64_t>(c->cnt2),
                                P<unsigned long long>(c->ctrun), s) ||
        launch_gram(P<unsigned long long>(c->ctrun), nruns, P<unsigned long long>(c->gram), s))
        return -1;
    int limit;
    if (pair_cap(c, na, nb, self, &limit))
        return -1;
    c->stats.limit[0] = c->stats.limit[1] = limit;
    uint64_t* d_nf = (uint64_t*)(P<uint32_t>(c->misc) + 16);
    uint64_t* d_nc = (uint64_t*)(P<uint32_t>(c->misc) + 20);
    if (launch_cnt_mask(P<uint32_t>(c->excl), P<uint32_t>(c->flags), P<unsigned long long>(c->ctrun), na, limit, 0,
                        P<uint64_t>(c->cnt), s) ||
        launch_cnt_mask(P<uint32_t>(c->excl), P<uint32_t>(c->flags), P<unsigned long long>(c->ctrun), na, limit, 0,
                        P<uint64_t>(c->cnt2), s) ||
        exclusive_scan<uint64_t>(P<uint64_t>(c->cnt), P<uint64_t>(c->hoff), na, d_nf, c->scratch.p, s) ||
        exclusive_scan<uint64_t>(P<uint64_t>(c->cnt2), P<uint64_t>(c->hoff2), na, d_nc, c->scratch.p, s))
        return -1;
    uint64_t nf = 0, nc = 0;
    GD_CUDA(cudaMemcpyAsync(&nf, d_nf, 8, cudaMemcpyDeviceToHost, s));
    GD_CUDA(cudaMemcpyAsync(&nc, d_nc, 8, cudaMemcpyDeviceToHost, s));
    GD_CUDA(cudaStreamSynchronize(s));
    c->stats.hits[0] = (int64_t)nf;
    c->stats.hits[1] = (int64_t)nc;
    if (nf == 0 && nc == 0)
        return 0;
    const uint64_t nmax = std::max(nf, nc);
    if (nmax > 0xffffffffull)
    {
        gd_set_error("%llu hits exceed the 32-bit hit index of this build", (unsigned long long)nmax);
        return -1;
    }
    HitBits hb;
    hb.pbits = bits_for(std::max(A.blk.maxlen - 1, 1));
    hb.abits = bits_for(std::max(A.blk.nreads - 1, 1));
    hb.bbits = bits_for(std::max(B.blk.nreads - 1, 1));
    if (hb.pbits + hb.abits + hb.bbits > 64)
    {
        gd_set_error("hit key needs %d bits (> 64): block too large for this build", hb.pbits + hb.abits + hb.bbits);
        return -1;
    }
    hb.qbits = hit_qbits(c, hb, B);
    if (ensure(c->hk0, nmax * 8 + 8) || ensure(c->hk1, nmax * 8 + 8) || ensure(c->hd0, nmax * 4 + 4) ||
        ensure(c->hd1, nmax * 4 + 4) || ensure(c->hk2, nc * 8 + 8) || ensure(c->hd2, nc * 4 + 4) ||
        ensure(c->scratch, radix_scratch_bytes(nmax)))
        return -1;
    if (launch_d2_emit_hits(P<int32_t>(A.read), P<int32_t>(A.rpos), P<int32_t>(B.read), P<int32_t>(B.rpos),
                            P<int32_t>(B.rlen), P<uint32_t>(c->jb), P<uint64_t>(c->cnt), P<uint64_t>(c->cnt2),
                            P<uint64_t>(c->hoff), P<uint64_t>(c->hoff2), na, c->kmer, hb, P<uint64_t>(c->hk0),
                            P<uint32_t>(c->hd0), P<uint64_t>(c->hk2), P<uint32_t>(c->hd2), s))
        return -1;
    if (nf > 0 && align_hits(c, A, B, nf, hb, 0, self))
        return -1;
    if (nc > 0)
    {
        GD_CUDA(cudaEventRecord(c->ev0, s));
        GD_CUDA(cudaMemcpyAsync(c->hk0.p, c->hk2.p, nc * 8, cudaMemcpyDeviceToDevice, s));
        if (hb.qbits == 0)
            GD_CUDA(cudaMemcpyAsync(c->hd0.p, c->hd2.p, nc * 4, cudaMemcpyDeviceToDevice, s));
        if (align_hits(c, A, C, nc, hb, 1, self))
            return -1;
    }
    return 0;
}

// The hits of one orientation in (hk0, hd0), in generation order, through the hit sort, the
// pair groups, the learned triage and the seed scan + alignment; records are appended to the
// overlap buffer in HBM.  c->ev0 marks the start of this orientation's merge stage.
static int align_hits(gd_context* c, Slot& A, Slot& B, uint64_t nhits, gd::HitBits hb, int comp, int self)
{
    using namespace gd;
    cudaStream_t s = c->s;
    const int oi = comp ? 1 : 0;
    const int hbits = hb.pbits + hb.abits + hb.bbits;
    // hit sort by (bread, aread, apos), stable (pairsort, filter.c:2030-2054, 2239-2252)
    uint64_t* hkey;
    uint32_t *hdiag, *pflags, *ppos;  // pflags / ppos: free ping-pong halves
    if (hb.qbits > 0)
    {
        // packed hits: keys alone through the passes, the B position riding below the key; the
        // last pass writes the key and diag arrays (with no pass to run, a separate unpack)
        const int passes = (hbits + 7) / 8;
        uint64_t* out = (passes & 1) ? P<uint64_t>(c->hk1) : P<uint64_t>(c->hk0);  // the last pass's target
        uint64_t* in = (passes & 1) ? P<uint64_t>(c->hk0) : P<uint64_t>(c->hk1);   // and its source
        hdiag = P<uint32_t>(c->hd0);
        if (nhits > 1)
        {
            RsFinal fin;
            fin.kind = RsFinal::HITS;
            fin.a = out;
            fin.b = (int32_t*)hdiag;
            fin.bits = hb.qbits;
            fin.pbits = hb.pbits;
            if (radix_sort_keys<uint64_t>(P<uint64_t>(c->hk0), P<uint64_t>(c->hk1), nhits, hb.qbits,
                                          hb.qbits + hbits, c->scratch.p, s, &fin) < 0)
                return -1;
            hkey = out;
            ppos = (uint32_t*)in;
        }
        else
        {
            hkey = P<uint64_t>(c->hk1);
            if (launch_hit_unpack(P<uint64_t>(c->hk0), nhits, hb, hkey, hdiag, s))
                return -1;
            ppos = (uint32_t*)P<uint64_t>(c->hk0);
        }
        pflags = P<uint32_t>(c->hd1);
    }
    else
    {
        int which = radix_sort_pairs<uint64_t>(P<uint64_t>(c->hk0), P<uint32_t>(c->hd0), P<uint64_t>(c->hk1),
                                               P<uint32_t>(c->hd1), nhits, 0, hbits, c->scratch.p, s);
        if (which < 0)
            return -1;
        hkey = which ? P<uint64_t>(c->hk1) : P<uint64_t>(c->hk0);
        hdiag = which ? P<uint32_t>(c->hd1) : P<uint32_t>(c->hd0);
        pflags = which ? P<uint32_t>(c->hd0) : P<uint32_t>(c->hd1);
        ppos = (uint32_t*)(which ? P<uint64_t>(c->hk0) : P<uint64_t>(c->hk1));
    }
    c->hkey = hkey;
    c->hdiag = hdiag;
    c->nhits = (int64_t)nhits;
    c->hb = hb;
    // pair groups with >= ceil(h/k) hits (report_thread's minhit test, filter.c:1699-1709)
    uint32_t* d_nst = P<uint32_t>(c->misc) + 24;
    if (launch_pair_flags(hkey, nhits, hb.pbits, pflags, s) ||
        exclusive_scan<uint32_t>(pflags, ppos, nhits, d_nst, c->scratch.p, s))
        return -1;
    uint32_t nst = 0;
    GD_CUDA(cudaMemcpyAsync(&nst, d_nst, 4, cudaMemcpyDeviceToHost, s));
    GD_CUDA(cudaStreamSynchronize(s));
    if (ensure(c->starts, (size_t)nst * 4 + 8) || ensure(c->groups, (size_t)nst * 8 + 8) ||
        ensure(c->gcost, (size_t)nst * 4 + 8) || ensure(c->gidx, (size_t)nst * 4 + 8) ||
        ensure(c->gcost2, (size_t)nst * 4 + 8) || ensure(c->gidx2, (size_t)nst * 4 + 8))
        return -1;
    unsigned* d_ng = P<unsigned>(c->misc) + 28;
    // with the learned triage on (or its features collected), the kept groups' features, MLP
    // and skip flags follow selection
    const bool triage = c->tri_on || c->tri_collect;
    unsigned* d_nskip = P<unsigned>(c->misc) + 32;
    if (triage)
    {
        if (ensure(c->tri_skip, (size_t)nst + 8) || ensure(c->tri_gstat, (size_t)nst * 8 + 8) ||
            (c->tri_collect && ensure(c->tri_feat, (size_t)nst * TRI_NF * 4 + 64)))
            return -1;
        GD_CUDA(cudaMemsetAsync(d_nskip, 0, 4, s));
    }
    if (launch_pair_scatter(pflags, ppos, nhits, P<uint32_t>(c->starts), s))
        return -1;
    // groups in which daligner's seed scan would find no candidate are dropped here, exactly
    // (daligner2's report keeps its own selection)
    const int minhit = (c->hitmin - 1) / c->kmer + 1;
    const int seed_test = c->variant == 1 ? c->hitmin : 0;
    if (launch_select_groups(P<uint32_t>(c->starts), nst, nhits, minhit, hkey, hdiag, c->binshift, c->kmer, seed_test,
                             hb, P<int32_t>(A.rlen), P<int32_t>(B.rlen), P<uint2>(c->groups), P<uint32_t>(c->gcost),
                             P<uint32_t>(c->gidx), d_ng, s))
        return -1;
    unsigned ng = 0;
    GD_CUDA(cudaMemcpyAsync(&ng, d_ng, 4, cudaMemcpyDeviceToHost, s));
    GD_CUDA(cudaStreamSynchronize(s));
    c->stats.groups[oi] = ng;
    if (triage &&
        launch_triage_groups(P<uint2>(c->groups), ng, hkey, hdiag, hb, A.blk, B.blk, comp, c->minover, c->binshift,
                             A.has_mask ? P<int64_t>(A.manno) : nullptr, A.has_mask ? P<int32_t>(A.mdata) : nullptr,
                             c->tri_on ? P<float>(c->tri_params) : nullptr, c->tri_thr,
                             c->tri_collect ? P<float>(c->tri_feat) : nullptr, P<uint8_t>(c->tri_skip), d_nskip, s))
        return -1;
    if (ensure(c->scratch, std::max(c->scratch.n, radix_scratch_bytes(ng) + 4096)))
        return -1;
    int gw = radix_sort_pairs<uint32_t>(P<uint32_t>(c->gcost), P<uint32_t>(c->gidx), P<uint32_t>(c->gcost2),
                                        P<uint32_t>(c->gidx2), ng, 0, 32, c->scratch.p, s);
    if (gw < 0)
        return -1;
    uint32_t* order = gw ? P<uint32_t>(c->gidx2) : P<uint32_t>(c->gidx);
    // per-length-class launches (the comparison schedule): each class is a contiguous range of
    // the cost-sorted order, found from the sorted keys ~(alen + blen)
    std::vector<unsigned> bucket{0u};
    std::vector<int> bclass{0};  // the length class of each bucket (empty classes have none)
    if (!c->sched_edges.empty() && ng > 0)
    {
        std::vector<uint32_t> keys(ng);
        GD_CUDA(cudaMemcpyAsync(keys.data(), gw ? P<uint32_t>(c->gcost2) : P<uint32_t>(c->gcost), (size_t)ng * 4,
                                cudaMemcpyDeviceToHost, s));
        GD_CUDA(cudaStreamSynchronize(s));
        std::vector<int32_t> edges = c->sched_edges;
        std::sort(edges.begin(), edges.end(), std::greater<int32_t>());
        for (size_t i = 0; i < edges.size(); i++)
        {
            unsigned p = (unsigned)(std::upper_bound(keys.begin(), keys.end(), ~(uint32_t)edges[i]) - keys.begin());
            if (p >= ng)
                break;
            if (p > bucket.back())
            {
                bucket.push_back(p);
                bclass.push_back((int)i + 1);
            }
            else
                bclass.back() = (int)i + 1;  // the classes before this edge are empty
        }
    }
    bucket.push_back(ng);
    // the learned triage's skip flags came with the groups
    const uint8_t* skip = nullptr;
    if (triage && ng > 0)
    {
        if (c->tri_on)
            skip = P<uint8_t>(c->tri_skip);
        if (c->tri_collect)
            GD_CUDA(cudaMemsetAsync(c->tri_gstat.p, 0, (size_t)ng * 8, s));
    }
    GD_CUDA(cudaEventRecord(c->ev1, s));
    GD_CUDA(cudaEventSynchronize(c->ev1));
    float ms = 0;
    cudaEventElapsedTime(&ms, c->ev0, c->ev1);
    c->stats.ms_merge[oi] = ms;
    if (ng == 0)
        return 0;

    // seed scan + alignment
    AlignParams ap{};
    ap.tspace = c->tspace;
    ap.ave_path = c->ave_path;
    ap.kmer = c->kmer;
    ap.binshift = c->binshift;
    ap.hitmin = c->hitmin;
    ap.minover = c->minover;
    ap.symmetric = c->symmetric;
    ap.self = self;
    ap.comp = comp;
    ap.trace8 = c->tspace <= 125;
    ap.no_trace = c->no_trace;
    ap.maxdiag = A.blk.maxlen >> c->binshift;
    ap.mindiag = (-B.blk.maxlen) >> c->binshift;
    ap.hb = hb;
    ap.table = P<int16_t>(c->tables);
    ap.score = P<int16_t>(c->tables) + TRIM_TABLE;
    ap.mscore = c->mscore;
    ap.dscore = c->dscore;
    ap.test_narrow = c->test_narrow;
    ap.d2 = c->variant == 2;
    ap.hgap = c->hgap;
    if ((!c->agrid && align_grid(&c->agrid, 0)) || (!c->agrid_w && align_grid(&c->agrid_w, 1)) ||
        (!c->agrid_d && align_grid(&c->agrid_d, 2)))
        return -1;
    const int nwarps_w = c->agrid_w * align_warps_per_cta(1);
    int maxlen = std::max(A.blk.maxlen, B.blk.maxlen);
    int ptscap = 4 * (2 * (maxlen / c->tspace + 2)) + 32;
    int nbands = ap.maxdiag - ap.mindiag + 8;
    // the instance of each length class (0 warp, 1 wide, 2 duo); daligner2's report has no duo
    // instance and takes the warp instance there
    std::vector<int> kind(bucket.size() - 1, 0);
    for (size_t b = 0; b < kind.size(); b++)
        if ((size_t)bclass[b] < c->sched_kind.size())
            kind[b] = (c->sched_kind[bclass[b]] == 2 && ap.d2) ? 0 : c->sched_kind[bclass[b]];
    DevBuf* const kbuf[3] = {&c->ascr, &c->ascr_w, &c->ascr_d};
    const int kgrid[3] = {c->agrid, c->agrid_w, c->agrid_d};
    c->stats.reruns[oi] = 0;
    for (int attempt = 0; attempt < 48; attempt++)
    {
        if (attempt)
            c->stats.reruns[oi]++;
        const int bvcap = ap.d2 ? c->bvcap : 0, btcap = ap.d2 ? c->btcap : 0;
        // each instance in use gets its scratch: a slot per warp (per team of the duo instance).
        // The band arrays (score, lastp, lasta per slot) start at zero on every launch: their
        // place in the scratch moves with maxlen and the capacities, so an earlier launch's
        // clean-up does not cover them
        AlignScratch ks[3]{};
        for (int k = 0; k < 3; k++)
        {
            if (std::find(kind.begin(), kind.end(), k) == kind.end())
                continue;
            const int slots = kgrid[k] * align_warps_per_cta(k) * align_slots_per_warp(k);
            if (ensure(*kbuf[k], align_scratch_bytes(slots, c->pcap, ptscap, c->mcap, c->tcap, nbands, bvcap, btcap)))
                return -1;
            align_scratch_carve(&ks[k], kbuf[k]->p, slots, c->pcap, ptscap, c->mcap, c->tcap, nbands, bvcap, btcap);
            GD_CUDA(cudaMemsetAsync(ks[k].bands, 0, (size_t)slots * 3 * nbands * 4, s));
        }
        if (ensure(c->outrec, c->rcap * sizeof(OutRec)) || ensure(c->outtr, c->tbcap) ||
            ensure(c->counters, 8 * 8) || ensure(c->status, sizeof(DevStatus)) || ensure(c->queue, 16))
            return -1;
        GD_CUDA(cudaMemsetAsync(c->counters.p, 0, 64, s));
        GD_CUDA(cudaMemsetAsync(c->status.p, 0, sizeof(DevStatus), s));
        if (ensure(c->wide, (size_t)ng * 4 + 16))
            return -1;
        unsigned* wide_list = P<unsigned>(c->wide);
        unsigned* d_nwide = wide_list + ng;
        GD_CUDA(cudaMemsetAsync(d_nwide, 0, 4, s));
        AlignOut out{P<OutRec>(c->outrec), P<uint8_t>(c->outtr), P<unsigned long long>(c->counters), c->rcap,
                     c->tbcap, skip, c->tri_collect ? P<uint2>(c->tri_gstat) : nullptr, wide_list, d_nwide};
        GD_CUDA(cudaEventRecord(c->ev0, s));
        for (size_t b = 0; b < kind.size(); b++)
        {
            // a class on the wide instance has no wider one to hand groups to
            AlignOut o2 = out;
            if (kind[b] == 1)
            {
                o2.wide_list = nullptr;
                o2.nwide = nullptr;
            }
            if (launch_align_pairs(A.blk, B.blk, hkey, hdiag, P<uint2>(c->groups), order + bucket[b],
                                   bucket[b + 1] - bucket[b], ap, ks[kind[b]], o2, P<unsigned>(c->queue),
                                   P<DevStatus>(c->status), kgrid[kind[b]], s, kind[b]))
                return -1;
        }
        // pair groups whose band outgrew the main instance: the wide one, appending to the same
        // output with its own scratch (a band wider than WIDE_RING is an error there)
        unsigned nwide = 0;
        GD_CUDA(cudaMemcpyAsync(&nwide, d_nwide, 4, cudaMemcpyDeviceToHost, s));
        GD_CUDA(cudaStreamSynchronize(s));
        c->stats.wide[oi] = nwide;
        if (nwide > 0)
        {
            AlignScratch scw{};
            const size_t need_w =
                align_scratch_bytes(nwarps_w, c->pcap, ptscap, c->mcap, c->tcap, nbands, bvcap, btcap);
            if (ensure(c->ascr_w, need_w))
                return -1;
            align_scratch_carve(&scw, c->ascr_w.p, nwarps_w, c->pcap, ptscap, c->mcap, c->tcap, nbands, bvcap,
                                btcap);
            GD_CUDA(cudaMemsetAsync(scw.bands, 0, (size_t)nwarps_w * 3 * nbands * 4, s));
            AlignOut outw = out;
            outw.wide_list = nullptr;
            outw.nwide = nullptr;
            if (launch_align_pairs(A.blk, B.blk, hkey, hdiag, P<uint2>(c->groups), wide_list, nwide, ap, scw, outw,
                                   P<unsigned>(c->queue), P<DevStatus>(c->status), c->agrid_w, s, 1))
                return -1;
        }
        GD_CUDA(cudaEventRecord(c->ev1, s));
        GD_CUDA(cudaEventSynchronize(c->ev1));
        cudaEventElapsedTime(&ms, c->ev0, c->ev1);
        c->stats.ms_align[oi] = ms;
        DevStatus st;
        unsigned long long cnt[8];
        GD_CUDA(cudaMemcpy(&st, c->status.p, sizeof(st), cudaMemcpyDeviceToHost));
        GD_CUDA(cudaMemcpy(cnt, c->counters.p, sizeof(cnt), cudaMemcpyDeviceToHost));
        if (st.code != 0)
        {
            if (st.code == GD_ERR_PEBBLES)
                c->pcap *= 2;
            else if (st.code == GD_ERR_TRACE)
                c->tcap *= 2;
            else if (st.code == GD_ERR_MATCHES)
                c->mcap *= 2;
            else if (st.code == GD_ERR_BRIDGE && st.info > 1)
            {
                // a daligner2 bridge box larger than the bridging scratch: grow both and re-run
                c->bvcap = std::max(2 * c->bvcap, st.info + 64);
                c->btcap = std::max(2 * c->btcap, st.info + 64);
                continue;
            }
            else
            {
                gd_set_error("aligner failed on pair group %d: code %d info %d", st.where, st.code, st.info);
                return -1;
            }
            continue;
        }
        if (cnt[0] > c->rcap || cnt[1] > c->tbcap)
        {
            c->rcap = std::max(c->rcap, (uint64_t)(cnt[0] * 5 / 4 + 1024));
            c->tbcap = std::max(c->tbcap, (uint64_t)(cnt[1] * 5 / 4 + 65536));
            continue;
        }
        c->stats.cells[oi] = (int64_t)cnt[2];
        c->stats.seeds[oi] = (int64_t)cnt[3];
        if (c->tri_on)
        {
            unsigned nskip = 0;
            GD_CUDA(cudaMemcpy(&nskip, d_nskip, 4, cudaMemcpyDeviceToHost));
            c->stats.skipped[oi] = nskip;
        }
        if (c->tri_collect && tri_append(c, ng))
            return -1;
        // append to the overlap buffer in HBM
        if (ensure_keep(c->acc_rec, (c->acc_n + cnt[0]) * sizeof(OutRec), c->acc_n * sizeof(OutRec), s) ||
            ensure_keep(c->acc_tr, c->acc_tb + cnt[1] + 16, c->acc_tb, s))
            return -1;
        if (launch_ovl_append(P<OutRec>(c->outrec), cnt[0], c->acc_tb, P<OutRec>(c->acc_rec) + c->acc_n, s))
            return -1;
        if (cnt[1])
            GD_CUDA(cudaMemcpyAsync(P<uint8_t>(c->acc_tr) + c->acc_tb, c->outtr.p, cnt[1], cudaMemcpyDeviceToDevice, s));
        c->acc_n += cnt[0];
        c->acc_tb += cnt[1];
        c->srt_valid = false;
        return 0;
    }
    gd_set_error("aligner scratch could not be grown enough");
    return -1;
}

// ----------------------------------------------------------------------------------------
// overlap sort + .las writing (Write_Overlap_Buffer, dalign/align.c:5786-6043)
// ----------------------------------------------------------------------------------------

// The order of n records on the device: two stable radix sorts, by (orientation if
// with_comp, abpos, aepos, bbpos) and then by (dropped, aread, bread).  Returns the
// permutation (in oval0 or oval1) in *perm, the records kept (not dropped by the identity
// filter; they come first) in *kept, and in olen the exclusive scan of their trace bytes
// (olen[n] = total); *kbytes = trace bytes of the kept records.
static int sort_perm(gd_context* c, const gd::OutRec* rec, uint64_t n, int with_comp, int only_identity, int tbytes,
                     const uint32_t** perm_out, uint64_t* kept_out, uint64_t* kbytes_out)
{
    using namespace gd;
    cudaStream_t s = c->s;
    if (n > 0xffffffffull)
    {
        gd_set_error("%llu overlaps exceed the 32-bit sort index", (unsigned long long)n);
        return -1;
    }
    if (ensure(c->okey0, n * 8) || ensure(c->okey1, n * 8) || ensure(c->oval0, n * 4) || ensure(c->oval1, n * 4) ||
        ensure(c->olen, n * 8 + 8) ||
        ensure(c->scratch, std::max(radix_scratch_bytes((int64_t)n), scan_scratch_bytes<uint64_t>((int64_t)n))) ||
        ensure(c->misc, 256))
        return -1;
    unsigned* d_ext = P<unsigned>(c->misc) + 40;
    unsigned long long* d_kept = (unsigned long long*)(P<unsigned>(c->misc) + 44);
    uint64_t* d_total = (uint64_t*)(P<unsigned>(c->misc) + 46);
    static const unsigned ext0[3] = {0xffffffffu, 0u, 0u};
    GD_CUDA(cudaMemcpyAsync(d_ext, ext0, sizeof ext0, cudaMemcpyHostToDevice, s));
    GD_CUDA(cudaMemsetAsync(d_kept, 0, 8, s));
    if (launch_ovl_extent(rec, n, d_ext, s))
        return -1;
    unsigned ext[3];
    GD_CUDA(cudaMemcpyAsync(ext, d_ext, sizeof ext, cudaMemcpyDeviceToHost, s));
    GD_CUDA(cudaStreamSynchronize(s));
    const int pbits = bits_for(std::max(ext[2], 1u));
    const int rbits = bits_for(std::max(ext[1] - ext[0], 1u));
    if (3 * pbits + 1 > 64 || 2 * rbits + 1 > 64)
    {
        gd_set_error("overlap sort keys need %d / %d bits", 3 * pbits + 1, 2 * rbits + 1);
        return -1;
    }
    if (launch_ovl_key_lo(rec, n, pbits, with_comp, P<uint64_t>(c->okey0), P<uint32_t>(c->oval0), s))
        return -1;
    int w1 = radix_sort_pairs<uint64_t>(P<uint64_t>(c->okey0), P<uint32_t>(c->oval0), P<uint64_t>(c->okey1),
                                        P<uint32_t>(c->oval1), n, 0, 3 * pbits + 1, c->scratch.p, s);
    if (w1 < 0)
        return -1;
    uint64_t* ka = w1 ? P<uint64_t>(c->okey1) : P<uint64_t>(c->okey0);
    uint32_t* va = w1 ? P<uint32_t>(c->oval1) : P<uint32_t>(c->oval0);
    uint64_t* kb = w1 ? P<uint64_t>(c->okey0) : P<uint64_t>(c->okey1);
    uint32_t* vb = w1 ? P<uint32_t>(c->oval0) : P<uint32_t>(c->oval1);
    if (launch_ovl_key_hi(rec, va, n, rbits, ext[0], only_identity, ka, d_kept, s))
        return -1;
    int w2 = radix_sort_pairs<uint64_t>(ka, va, kb, vb, n, 0, 2 * rbits + 1, c->scratch.p, s);
    if (w2 < 0)
        return -1;
    const uint32_t* perm = w2 ? vb : va;
    uint64_t* off = P<uint64_t>(c->olen);
    if (launch_ovl_len(rec, perm, n, tbytes, off, s) ||
        exclusive_scan<uint64_t>(off, off, (int64_t)n, d_total, c->scratch.p, s))
        return -1;
    unsigned long long kept = 0;
    GD_CUDA(cudaMemcpyAsync(&kept, d_kept, 8, cudaMemcpyDeviceToHost, s));
    GD_CUDA(cudaStreamSynchronize(s));
    uint64_t kbytes = 0;
    GD_CUDA(cudaMemcpyAsync(&kbytes, kept < n ? off + kept : d_total, 8, cudaMemcpyDeviceToHost, s));
    GD_CUDA(cudaStreamSynchronize(s));
    *perm_out = perm;
    *kept_out = kept;
    *kbytes_out = kbytes;
    return 0;
}

// Write_Overlap_Buffer's sort (SORT_OVL, dalign/align.c:5786-5813) of the overlap buffer:
// order (aread, bread, orientation, abpos), ties by (aepos, bbpos) -- the reference's qsort
// leaves ties unordered -- with -I's identity filter (only_identity) applied as a drop bit;
// the kept records and their traces are gathered into srt_rec / srt_tr.
static int sort_overlaps(gd_context* c)
{
    using namespace gd;
    if (c->srt_valid)
        return 0;
    const uint64_t n = c->acc_n;
    c->srt_n = c->srt_tb = 0;
    if (n == 0)
    {
        c->srt_valid = true;
        return 0;
    }
    const int tbytes = c->tspace <= 125 ? 1 : 2;
    const uint32_t* perm = nullptr;
    uint64_t kept = 0, kbytes = 0;
    if (sort_perm(c, P<OutRec>(c->acc_rec), n, 1, c->only_identity, tbytes, &perm, &kept, &kbytes))
        return -1;
    if (ensure(c->srt_rec, kept * sizeof(OutRec)) || ensure(c->srt_tr, kbytes + 16))
        return -1;
    if (launch_ovl_gather(P<OutRec>(c->acc_rec), P<uint8_t>(c->acc_tr), perm, P<uint64_t>(c->olen), kept, tbytes,
                          P<OutRec>(c->srt_rec), P<uint8_t>(c->srt_tr), c->s))
        return -1;
    GD_CUDA(cudaStreamSynchronize(c->s));
    c->srt_n = kept;
    c->srt_tb = kbytes;
    c->srt_valid = true;
    return 0;
}

// the sorted buffer in pinned host memory (h_rec, h_tr)
static int stage_sorted(gd_context* c)
{
    if (sort_overlaps(c) || ensure_host(c->h_rec, c->srt_n * sizeof(gd_overlap)) || ensure_host(c->h_tr, c->srt_tb))
        return -1;
    if (c->srt_n)
        GD_CUDA(cudaMemcpyAsync(c->h_rec.p, c->srt_rec.p, c->srt_n * sizeof(gd_overlap), cudaMemcpyDeviceToHost, c->s));
    if (c->srt_tb)
        GD_CUDA(cudaMemcpyAsync(c->h_tr.p, c->srt_tr.p, c->srt_tb, cudaMemcpyDeviceToHost, c->s));
    GD_CUDA(cudaStreamSynchronize(c->s));
    return 0;
}

static int write_las(gd_context* c, const char* path, size_t from, size_t to)
{
    FILE* f = fopen(path, "w");
    if (!f)
    {
        gd_set_error("Cannot open file %s for writing", path);
        return -1;
    }
    const gd_overlap* recs = (const gd_overlap*)c->h_rec.p;
    const uint8_t* trace = (const uint8_t*)c->h_tr.p;
    int tbytes = c->tspace <= 125 ? 1 : 2;
    int64_t n = (int64_t)(to - from);
    int32_t ts = c->tspace;
    fwrite(&n, 8, 1, f);
    fwrite(&ts, 4, 1, f);
    std::vector<uint8_t> buf;
    buf.reserve(1 << 21);
    for (size_t i = from; i < to; i++)
    {
        const gd_overlap& o = recs[i];
        int32_t r[10] = {o.tlen, o.diffs, o.abpos, o.bbpos, o.aepos, o.bepos, (int32_t)o.flags, o.aread, o.bread, 0};
        const uint8_t* rb = (const uint8_t*)r;
        buf.insert(buf.end(), rb, rb + 40);
        if (o.tlen > 0)
            buf.insert(buf.end(), trace + o.toff, trace + o.toff + (size_t)o.tlen * tbytes);
        if (buf.size() > (1 << 20))
        {
            fwrite(buf.data(), 1, buf.size(), f);
            buf.clear();
        }
    }
    fwrite(buf.data(), 1, buf.size(), f);
    if (fclose(f))
    {
        gd_set_error("write to %s failed", path);
        return -1;
    }
    return 0;
}

static std::string dirname_of(int run_id, int block)
{
    // getDir (db/DB.c:1661-1675)
    if (block == 0)
        return ".";
    char b[64];
    snprintf(b, sizeof b, "%03d_%05d", run_id, block);
    return b;
}

const int16_t* gd_context_align_tables(gd_context* c, int* tspace, int* ave_path, int* mscore, int* dscore)
{
    if (!c || !c->spec_set)
        return nullptr;
    *tspace = c->tspace;
    *ave_path = c->ave_path;
    *mscore = c->mscore;
    *dscore = c->dscore;
    return P<int16_t>(c->tables);
}

// ----------------------------------------------------------------------------------------
// C ABI
// ----------------------------------------------------------------------------------------

extern "C" {

const char* gd_last_error(void)
{
    return g_err;
}

gd_context* gd_create(void)
{
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0)
    {
        gd_set_error("no CUDA device: the overlap path runs on the GPU only");
        return nullptr;
    }
    gd_context* c = new gd_context();
    memset(&c->stats, 0, sizeof(c->stats));
    if (cudaStreamCreateWithFlags(&c->s, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreate(&c->ev0) != cudaSuccess || cudaEventCreate(&c->ev1) != cudaSuccess ||
        cudaEventCreate(&c->tev0) != cudaSuccess || cudaEventCreate(&c->tev1) != cudaSuccess)
    {
        gd_set_error("stream/event creation failed");
        delete c;
        return nullptr;
    }
    return c;
}

void gd_destroy(gd_context* c)
{
    if (!c)
        return;
    cudaStreamSynchronize(c->s);
    DevBuf* bufs[] = {&c->tables, &c->k0,     &c->v0,    &c->k1,     &c->v1,     &c->scratch, &c->flags,
                      &c->excl,   &c->jb,     &c->cnt,   &c->hoff,   &c->ctrun,  &c->gram,    &c->misc,
                      &c->hk0,    &c->hd0,    &c->hk1,   &c->hd1,    &c->starts, &c->groups,  &c->gcost,
                      &c->gidx,   &c->gcost2, &c->gidx2, &c->ascr,   &c->outrec, &c->outtr,   &c->counters,
                      &c->status, &c->queue,  &c->tri_params, &c->tri_feat, &c->tri_prob, &c->tri_skip,
                      &c->tri_gstat, &c->tri_misc, &c->tri_x, &c->tri_y, &c->tri_perm, &c->tri_grad, &c->tri_m,
                      &c->tri_v, &c->tri_loss, &c->tri_w, &c->acc_rec, &c->acc_tr, &c->srt_rec, &c->srt_tr,
                      &c->okey0, &c->okey1, &c->oval0, &c->oval1, &c->olen, &c->las_raw, &c->las_off,
                      &c->las_rec, &c->las_out, &c->ascr_w, &c->wide, &c->ascr_d};
    for (DevBuf* b : bufs)
        release(*b);
    for (HostBuf* h : {&c->h_rec, &c->h_tr})
        if (h->p)
            cudaFreeHost(h->p);
    for (Slot& s : c->slot)
    {
        DevBuf* sb[] = {&s.bases, &s.boff, &s.rlen, &s.manno, &s.mdata, &s.code, &s.read, &s.rpos};
        for (DevBuf* b : sb)
            release(*b);
    }
    cudaEventDestroy(c->ev0);
    cudaEventDestroy(c->ev1);
    cudaEventDestroy(c->tev0);
    cudaEventDestroy(c->tev1);
    cudaStreamDestroy(c->s);
    delete c;
}

int gd_set_filter_params(gd_context* c, int kmer, int binshift, int suppress, int hitmin)
{
    if (kmer <= 1)
    {
        gd_set_error("Illegal combination of filter parameters");
        return -1;
    }
    if (kmer > 32)
    {
        gd_set_error("k-mer length %d exceeds 32", kmer);
        return -1;
    }
    c->kmer = kmer;
    c->binshift = binshift;
    c->suppress = suppress;
    c->hitmin = hitmin;
    for (Slot& s : c->slot)
        s.nk = -1;
    return 0;
}

int gd_new_align_spec(gd_context* c, double ave_corr, int trace_space, const float freq[4], int symmetric,
                      int only_identity, int no_trace_points)
{
    if (trace_space <= 0)
    {
        gd_set_error("invalid trace spacing of (%d)", trace_space);
        return -1;
    }
    c->ave_corr = ave_corr;
    c->tspace = trace_space;
    for (int i = 0; i < 4; i++)
        c->freq[i] = freq[i];
    c->symmetric = symmetric;
    c->only_identity = only_identity;
    c->no_trace = no_trace_points;
    c->spec_set = 1;
    c->srt_valid = false;  // the identity filter and trace width enter the sorted copy
    return upload_spec(c);
}

int gd_set_globals(gd_context* c, int minover, int identity, uint64_t mem_limit)
{
    c->minover = minover;
    c->identity = identity;
    c->mem_limit = mem_limit;
    return 0;
}

static int pack_slot(gd_context* c, Slot& s, int64_t nbytes);

int gd_load_block(gd_context* c, int slot, const gd_block* b)
{
    if (slot < 0 || slot > 2)
    {
        gd_set_error("slot %d out of range", slot);
        return -1;
    }
    Slot& s = c->slot[slot];
    if (!b->bases || !b->boff || !b->rlen || b->nreads < 0 || (b->mask_anno == nullptr) != (b->mask_data == nullptr))
    {
        gd_set_error("gd_load_block: bases, boff and rlen are required (mask_anno and mask_data together)");
        return -1;
    }
    int64_t nb = b->boff[b->nreads];  // bytes after bases[-1], through the last 4
    for (int i = 0; i < b->nreads; i++)
        if (b->rlen[i] < c->kmer)
        {
            gd_set_error("Block contains reads < %dbp long !  Run DBsplit.", c->kmer);
            return -1;
        }
    // the kernels index the block by these offsets: read i ends with a 4 right before read i+1
    if (b->nreads > 0 && b->boff[0] != 0)
    {
        gd_set_error("gd_load_block: read 0 must start at offset 0 (boff[0] = %lld)", (long long)b->boff[0]);
        return -1;
    }
    for (int i = 0; i < b->nreads; i++)
        if (b->boff[i + 1] != b->boff[i] + b->rlen[i] + 1 || b->rlen[i] > b->maxlen)
        {
            gd_set_error("gd_load_block: read %d is not laid out as Read_All_Sequences leaves it (boff %lld, rlen %d, "
                         "next boff %lld, maxlen %d)",
                         i, (long long)b->boff[i], b->rlen[i], (long long)b->boff[i + 1], b->maxlen);
            return -1;
        }
    if (b->mask_anno)
        for (int i = 0; i < b->nreads; i++)
        {
            const int64_t lo = b->mask_anno[i], hi = b->mask_anno[i + 1];
            if (lo < 0 || hi < lo || ((hi - lo) & 1))
            {
                gd_set_error("gd_load_block: mask intervals of read %d are malformed (anno %lld .. %lld)", i,
                             (long long)lo, (long long)hi);
                return -1;
            }
        }
    if (ensure(s.bases, nb + 1 + 64) || ensure(s.boff, (b->nreads + 1) * 8) || ensure(s.rlen, b->nreads * 4 + 4))
        return -1;
    GD_CUDA(cudaMemsetAsync(s.bases.p, 4, nb + 1 + 64, c->s));
    GD_CUDA(cudaMemcpyAsync((uint8_t*)s.bases.p + 32, b->bases - 1, nb + 1, cudaMemcpyHostToDevice, c->s));
    GD_CUDA(cudaMemcpyAsync(s.boff.p, b->boff, (b->nreads + 1) * 8, cudaMemcpyHostToDevice, c->s));
    GD_CUDA(cudaMemcpyAsync(s.rlen.p, b->rlen, b->nreads * 4, cudaMemcpyHostToDevice, c->s));
    s.has_mask = b->mask_anno != nullptr;
    s.nmask = 0;
    if (s.has_mask)
    {
        int64_t nd = b->mask_anno[b->nreads];
        s.nmask = nd;
        if (ensure(s.manno, (b->nreads + 1) * 8) || ensure(s.mdata, nd * 4 + 8))
            return -1;
        GD_CUDA(cudaMemcpyAsync(s.manno.p, b->mask_anno, (b->nreads + 1) * 8, cudaMemcpyHostToDevice, c->s));
        if (nd)
            GD_CUDA(cudaMemcpyAsync(s.mdata.p, b->mask_data, nd * 4, cudaMemcpyHostToDevice, c->s));
    }
    s.blk.bases = (const uint8_t*)s.bases.p + 33;
    s.blk.boff = P<int64_t>(s.boff);
    s.blk.rlen = P<int32_t>(s.rlen);
    s.blk.nreads = b->nreads;
    s.blk.maxlen = b->maxlen;
    s.blk.ufirst = b->ufirst;
    if (pack_slot(c, s, nb + 1 + 64))
        return -1;
    s.totlen = b->totlen;
    s.nslots = nb - (int64_t)c->kmer * b->nreads;
    s.hrlen.assign(b->rlen, b->rlen + b->nreads);
    s.loaded = 1;
    s.nk = -1;
    GD_CUDA(cudaStreamSynchronize(c->s));
    return 0;
}

// The 2-bit copy of a slot's byte buffer (its first nbytes) for the aligner: the buffer's
// base index must fit 32 bits; one word more than the bytes cover, for the two-word reads
static int pack_slot(gd_context* c, Slot& s, int64_t nbytes)
{
    const int64_t nwords = (nbytes + 15) / 16 + 1;
    if (nbytes + 32 > 0xffffffffll)
    {
        gd_set_error("block of %lld bytes exceeds this build's 32-bit base index", (long long)nbytes);
        return -1;
    }
    if (ensure(s.pk, nwords * 4) || gd::launch_pack2((const uint8_t*)s.bases.p, nbytes, P<uint32_t>(s.pk), nwords, c->s))
        return -1;
    s.blk.pk = P<uint32_t>(s.pk);
    return 0;
}

int gd_complement_block(gd_context* c, int src, int dst)
{
    if (src < 0 || src > 2 || dst < 0 || dst > 2 || src == dst || !c->slot[src].loaded)
    {
        gd_set_error("bad complement slots %d -> %d", src, dst);
        return -1;
    }
    Slot& S = c->slot[src];
    Slot& D = c->slot[dst];
    int64_t nb = S.blk.boff ? 0 : 0;
    int n = S.blk.nreads;
    std::vector<int64_t> boff_last(1);
    GD_CUDA(cudaMemcpy(boff_last.data(), S.blk.boff + n, 8, cudaMemcpyDeviceToHost));
    nb = boff_last[0];
    if (ensure(D.bases, nb + 1 + 64) || ensure(D.boff, (n + 1) * 8) || ensure(D.rlen, n * 4 + 4))
        return -1;
    GD_CUDA(cudaMemsetAsync(D.bases.p, 4, nb + 1 + 64, c->s));
    GD_CUDA(cudaMemcpyAsync(D.boff.p, S.boff.p, (n + 1) * 8, cudaMemcpyDeviceToDevice, c->s));
    GD_CUDA(cudaMemcpyAsync(D.rlen.p, S.rlen.p, n * 4, cudaMemcpyDeviceToDevice, c->s));
    D.has_mask = S.has_mask;
    D.nmask = S.nmask;
    int32_t* mdst = nullptr;
    if (S.has_mask)
    {
        int64_t nd = 0;
        GD_CUDA(cudaMemcpy(&nd, P<int64_t>(S.manno) + n, 8, cudaMemcpyDeviceToHost));
        if (ensure(D.manno, (n + 1) * 8) || ensure(D.mdata, nd * 4 + 8))
            return -1;
        GD_CUDA(cudaMemcpyAsync(D.manno.p, S.manno.p, (n + 1) * 8, cudaMemcpyDeviceToDevice, c->s));
        mdst = P<int32_t>(D.mdata);
    }
    D.blk = S.blk;
    D.blk.bases = (const uint8_t*)D.bases.p + 33;
    D.blk.boff = P<int64_t>(D.boff);
    D.blk.rlen = P<int32_t>(D.rlen);
    if (gd::launch_complement(S.blk, (uint8_t*)D.bases.p + 33, S.has_mask ? P<int64_t>(S.manno) : nullptr,
                              S.has_mask ? P<int32_t>(S.mdata) : nullptr, mdst, c->s))
        return -1;
    if (pack_slot(c, D, nb + 1 + 64))
        return -1;
    D.totlen = S.totlen;
    D.nslots = S.nslots;
    D.hrlen = S.hrlen;
    D.loaded = 1;
    D.nk = -1;
    GD_CUDA(cudaStreamSynchronize(c->s));
    return 0;
}

int gd_timer_mark(gd_context* c, int which)
{
    if (which < 0 || which > 1)
        return -1;
    GD_CUDA(cudaEventRecord(which ? c->tev1 : c->tev0, c->s));
    return 0;
}

double gd_timer_elapsed_ms(gd_context* c)
{
    float ms = -1.f;
    if (cudaEventSynchronize(c->tev1) != cudaSuccess || cudaEventElapsedTime(&ms, c->tev0, c->tev1) != cudaSuccess)
    {
        gd_set_error("timer events not recorded");
        return -1.0;
    }
    return ms;
}

unsigned long long gd_kernel_launches(void)
{
    return g_gd_launches;
}

int64_t gd_sort_kmers(gd_context* c, int slot)
{
    if (slot < 0 || slot > 2 || !c->slot[slot].loaded)
    {
        gd_set_error("slot %d not loaded", slot);
        return -1;
    }
    GD_CUDA(cudaEventRecord(c->ev0, c->s));
    int64_t n;
    if (c->variant == 2)
        n = c->kmer <= 15 ? index_slot_d2_t<uint32_t>(c, c->slot[slot]) : index_slot_d2_t<uint64_t>(c, c->slot[slot]);
    else if (c->biased)
        n = c->kmer <= 15 ? index_slot_bias_t<uint32_t>(c, c->slot[slot])
                          : index_slot_bias_t<uint64_t>(c, c->slot[slot]);
    else
        n = c->kmer <= 15 ? index_slot_t<uint32_t>(c, c->slot[slot]) : index_slot_t<uint64_t>(c, c->slot[slot]);
    GD_CUDA(cudaEventRecord(c->ev1, c->s));
    GD_CUDA(cudaEventSynchronize(c->ev1));
    float ms = 0;
    cudaEventElapsedTime(&ms, c->ev0, c->ev1);
    c->stats.ms_index[slot] = ms;
    c->stats.kmers[slot] = n;
    return n;
}

int64_t gd_get_kmers(gd_context* c, int slot, uint64_t* code, int32_t* read, int32_t* rpos, int64_t cap)
{
    Slot& s = c->slot[slot];
    if (s.nk < 0)
    {
        gd_set_error("slot %d has no index", slot);
        return -1;
    }
    int64_t n = std::min(s.nk, cap);
    if (c->kmer <= 15)
    {
        std::vector<uint32_t> t(n);
        GD_CUDA(cudaMemcpy(t.data(), s.code.p, n * 4, cudaMemcpyDeviceToHost));
        for (int64_t i = 0; i < n; i++)
            code[i] = t[i];
    }
    else
        GD_CUDA(cudaMemcpy(code, s.code.p, n * 8, cudaMemcpyDeviceToHost));
    GD_CUDA(cudaMemcpy(read, s.read.p, n * 4, cudaMemcpyDeviceToHost));
    GD_CUDA(cudaMemcpy(rpos, s.rpos.p, n * 4, cudaMemcpyDeviceToHost));
    return s.nk;
}

int gd_match_filter(gd_context* c, int bslot, int comp, int self)
{
    if (c->variant != 1)
    {
        gd_set_error("gd_match_filter runs daligner's filter; daligner2 mode uses gd_match_filter2");
        return -1;
    }
    if (!c->spec_set)
    {
        gd_set_error("gd_new_align_spec has not been called");
        return -1;
    }
    if (c->slot[0].nk < 0 || bslot < 0 || bslot > 2 || c->slot[bslot].nk < 0)
    {
        gd_set_error("both indices must be built before Match_Filter");
        return -1;
    }
    return c->kmer <= 15 ? match_filter_t<uint32_t>(c, bslot, comp, self)
                         : match_filter_t<uint64_t>(c, bslot, comp, self);
}

int gd_set_biased(gd_context* c, int biased)
{
    if (biased && c->variant == 2)
    {
        gd_set_error("daligner2 has no -b (biased tuples)");
        return -1;
    }
    c->biased = biased != 0;
    for (int i = 0; i < 3; i++)
        c->slot[i].nk = -1;  // an index of the other kind must be rebuilt
    return 0;
}

int gd_set_variant(gd_context* c, int variant, int hgap)
{
    if (variant != 1 && variant != 2)
    {
        gd_set_error("variant must be 1 (daligner) or 2 (daligner2), got %d", variant);
        return -1;
    }
    if (variant == 2 && c->biased)
    {
        gd_set_error("daligner2 has no -b (biased tuples)");
        return -1;
    }
    c->variant = variant;
    c->hgap = variant == 2 ? std::max(hgap, 0) : 0;
    for (int i = 0; i < 3; i++)
        c->slot[i].nk = -1;  // an index of the other kind must be rebuilt
    return 0;
}

int gd_match_filter2(gd_context* c, int bslot, int cslot, int self)
{
    if (c->variant != 2)
    {
        gd_set_error("gd_match_filter2 needs gd_set_variant(ctx, 2, ...)");
        return -1;
    }
    if (!c->spec_set)
    {
        gd_set_error("gd_new_align_spec has not been called");
        return -1;
    }
    if (bslot < 0 || bslot > 2 || cslot < 0 || cslot > 2 || cslot == bslot || c->slot[0].nk < 0 ||
        c->slot[bslot].nk < 0 || !c->slot[cslot].loaded)
    {
        gd_set_error("gd_match_filter2: both indices must be built and the complemented B block loaded");
        return -1;
    }
    return c->kmer <= 15 ? match_filter_d2_t<uint32_t>(c, bslot, cslot, self)
                         : match_filter_d2_t<uint64_t>(c, bslot, cslot, self);
}

int gd_test_handle_redundancies_d2(gd_context* c, const uint8_t* aseq, const uint8_t* bseq, int alen, int blen,
                                   int tspace, int comp, int novls, int hasB, const int32_t* hdr,
                                   const uint16_t* traces, int32_t* out_hdr, uint16_t* out_traces, int64_t tcap)
{
    using namespace gd;
    cudaStream_t s = c->s;
    const int npath = novls * (hasB ? 2 : 1);
    if (novls <= 0 || alen <= 0 || blen <= 0 || tspace <= 0)
    {
        gd_set_error("gd_test_handle_redundancies_d2: empty case");
        return -1;
    }
    int64_t ttot = 0;
    for (int i = 0; i < npath; i++)
        ttot += hdr[6 * i + 5];
    const int m = std::max(alen, blen);
    const int pcap_tr = (int)(ttot + 8 * (int64_t)(m / tspace + 8) * npath + 4096);
    const int vcap = 4 * m + 64, btcap = 2 * (m / tspace + 8) + 64;
    DevBuf da, db, dh, dp, dt, dv, dbt, doh, dn;
    struct Frees  // the hook's buffers are its own; cudaFree waits for the device
    {
        DevBuf* b[9];
        ~Frees()
        {
            for (DevBuf* x : b)
                if (x->p)
                    cudaFree(x->p);
        }
    } frees{{&da, &db, &dh, &dp, &dt, &dv, &dbt, &doh, &dn}};
    if (ensure(da, alen + 2) || ensure(db, blen + 2) || ensure(dh, npath * 24) ||
        ensure(dp, (npath + 1) * sizeof(MPath)) || ensure(dt, (size_t)pcap_tr * 2) || ensure(dv, (size_t)vcap * 4) ||
        ensure(dbt, (size_t)btcap * 2) || ensure(doh, (size_t)npath * 7 * 4) || ensure(dn, 4))
        return -1;
    GD_CUDA(cudaMemcpyAsync(da.p, aseq - 1, alen + 2, cudaMemcpyHostToDevice, s));
    GD_CUDA(cudaMemcpyAsync(db.p, bseq - 1, blen + 2, cudaMemcpyHostToDevice, s));
    GD_CUDA(cudaMemcpyAsync(dh.p, hdr, npath * 24, cudaMemcpyHostToDevice, s));
    if (ttot)
        GD_CUDA(cudaMemcpyAsync(dt.p, traces, ttot * 2, cudaMemcpyHostToDevice, s));
    if (launch_test_hr_d2((const uint8_t*)da.p + 1, (const uint8_t*)db.p + 1, alen, blen, tspace, comp, novls, hasB,
                          P<int32_t>(dh), P<MPath>(dp), P<uint16_t>(dt), (int)ttot, pcap_tr, P<int>(dv), vcap,
                          P<uint16_t>(dbt), btcap, P<int32_t>(doh), P<int>(dn), s))
        return -1;
    int n = 0;
    std::vector<int32_t> oh((size_t)npath * 7);
    GD_CUDA(cudaMemcpyAsync(&n, dn.p, 4, cudaMemcpyDeviceToHost, s));
    GD_CUDA(cudaMemcpyAsync(oh.data(), doh.p, oh.size() * 4, cudaMemcpyDeviceToHost, s));
    std::vector<uint16_t> tb((size_t)pcap_tr);
    GD_CUDA(cudaMemcpyAsync(tb.data(), dt.p, tb.size() * 2, cudaMemcpyDeviceToHost, s));
    GD_CUDA(cudaStreamSynchronize(s));
    if (n < 0)
    {
        gd_set_error("gd_test_handle_redundancies_d2: device code %d", -n);
        return -1;
    }
    const int nk = n * (hasB ? 2 : 1);
    int64_t o = 0;
    for (int i = 0; i < nk; i++)
    {
        memcpy(out_hdr + 6 * i, oh.data() + 6 * i, 24);
        const int tl = oh[6 * i + 5], toff = oh[6 * npath + i];
        if (o + tl > tcap || toff < 0 || toff + tl > pcap_tr)
        {
            gd_set_error("gd_test_handle_redundancies_d2: output trace capacity");
            return -1;
        }
        memcpy(out_traces + o, tb.data() + toff, (size_t)tl * 2);
        o += tl;
    }
    return n;
}

int64_t gd_get_hits(gd_context* c, int32_t* rows4, int64_t cap)
{
    int64_t n = std::min(c->nhits, cap);
    if (n <= 0)
        return c->nhits;
    std::vector<uint64_t> k(n);
    std::vector<uint32_t> d(n);
    GD_CUDA(cudaMemcpy(k.data(), c->hkey, n * 8, cudaMemcpyDeviceToHost));
    GD_CUDA(cudaMemcpy(d.data(), c->hdiag, n * 4, cudaMemcpyDeviceToHost));
    for (int64_t i = 0; i < n; i++)
    {
        rows4[4 * i + 0] = (int32_t)d[i];
        rows4[4 * i + 1] = (int32_t)(k[i] & ((1ull << c->hb.pbits) - 1));
        rows4[4 * i + 2] = (int32_t)((k[i] >> c->hb.pbits) & ((1ull << c->hb.abits) - 1));
        rows4[4 * i + 3] = (int32_t)(k[i] >> (c->hb.pbits + c->hb.abits));
    }
    return c->nhits;
}

int64_t gd_num_overlaps(gd_context* c, int64_t* trace_bytes)
{
    if (trace_bytes)
        *trace_bytes = (int64_t)c->acc_tb;
    return (int64_t)c->acc_n;
}

int64_t gd_sort_overlaps(gd_context* c, int64_t* trace_bytes)
{
    if (sort_overlaps(c))
        return -1;
    if (trace_bytes)
        *trace_bytes = (int64_t)c->srt_tb;
    return (int64_t)c->srt_n;
}

// LAsort / LAmerge core: the records of all input files, ordered on the device by (aread,
// bread, [orientation,] abpos), ties by (aepos, bbpos) and then input order, written to
// out_path with every record's bytes unchanged.
static int64_t las_sort_files(gd_context* c, const char* const* in_paths, int nin, const char* out_path, int with_comp)
{
    using namespace gd;
    int64_t novl = 0;
    int32_t tspace = 0;
    std::vector<uint64_t> bodies(nin);
    uint64_t body = 0;
    for (int f = 0; f < nin; f++)
    {
        FILE* fp = fopen(in_paths[f], "rb");
        if (!fp)
        {
            gd_set_error("Cannot open %s for reading", in_paths[f]);
            return -1;
        }
        int64_t nf = 0;
        int32_t ts = 0;
        fseek(fp, 0, SEEK_END);
        long fsize = ftell(fp);
        fclose(fp);
        fp = fopen(in_paths[f], "rb");
        if (fsize < 12 || fread(&nf, 8, 1, fp) != 1 || fread(&ts, 4, 1, fp) != 1 || nf < 0 || ts <= 0)
        {
            fclose(fp);
            gd_set_error("%s: not a .las file", in_paths[f]);
            return -1;
        }
        fclose(fp);
        if (f > 0 && ts != tspace)
        {
            gd_set_error("%s: trace spacing %d differs from %d of the first input", in_paths[f], ts, tspace);
            return -1;
        }
        tspace = ts;
        novl += nf;
        bodies[f] = (uint64_t)fsize - 12;
        body += bodies[f];
    }
    if (ensure_host(c->h_tr, body + 16) || ensure_host(c->h_rec, body + 16))
        return -1;
    uint8_t* raw = (uint8_t*)c->h_tr.p;
    const int tbytes = tspace <= 125 ? 1 : 2;  // TRACE_XOVR
    if ((uint64_t)novl > body / 40)
    {
        gd_set_error("%s: headers claim %lld records, the files hold at most %llu", in_paths[0], (long long)novl,
                     (unsigned long long)(body / 40));
        return -1;
    }
    // record offsets: records are variable length (LAsort.c:209-218), a sequential walk per file
    std::vector<int64_t> off((size_t)novl);
    uint64_t base = 0, used = 0;
    int64_t k = 0;
    for (int f = 0; f < nin; f++)
    {
        FILE* fp = fopen(in_paths[f], "rb");
        int64_t nf = 0;
        int32_t ts = 0;
        if (!fp || fread(&nf, 8, 1, fp) != 1 || fread(&ts, 4, 1, fp) != 1 ||
            (bodies[f] && fread(raw + base, 1, bodies[f], fp) != bodies[f]))
        {
            if (fp)
                fclose(fp);
            gd_set_error("%s: short read", in_paths[f]);
            return -1;
        }
        fclose(fp);
        uint64_t o = 0;
        for (int64_t i = 0; i < nf; i++, k++)
        {
            int32_t tlen;
            if (o + 40 > bodies[f])
            {
                gd_set_error("%s: record %lld runs past the end of the file", in_paths[f], (long long)i);
                return -1;
            }
            memcpy(&tlen, raw + base + o, 4);
            if (tlen < 0 || o + 40 + (uint64_t)tlen * tbytes > bodies[f])
            {
                gd_set_error("%s: record %lld has a bad trace length %d", in_paths[f], (long long)i, tlen);
                return -1;
            }
            off[(size_t)k] = (int64_t)(base + o);
            o += 40 + (uint64_t)tlen * tbytes;
        }
        // bytes after a file's last record are never referenced (the reference ignores them too)
        base += bodies[f];
        used = base;
    }
    cudaStream_t s = c->s;
    if (ensure(c->las_raw, used + 16) || ensure(c->las_off, (size_t)novl * 8 + 8) ||
        ensure(c->las_rec, (size_t)novl * sizeof(OutRec) + 16) || ensure(c->las_out, used + 16))
        return -1;
    if (used)
        GD_CUDA(cudaMemcpyAsync(c->las_raw.p, raw, used, cudaMemcpyHostToDevice, s));
    if (novl)
        GD_CUDA(cudaMemcpyAsync(c->las_off.p, off.data(), (size_t)novl * 8, cudaMemcpyHostToDevice, s));
    uint64_t outbytes = 0;
    if (novl)
    {
        const uint32_t* perm = nullptr;
        uint64_t kept = 0, kbytes = 0;
        if (launch_las_parse(P<uint8_t>(c->las_raw), P<int64_t>(c->las_off), (uint64_t)novl, P<OutRec>(c->las_rec), s) ||
            sort_perm(c, P<OutRec>(c->las_rec), (uint64_t)novl, with_comp, 0, tbytes, &perm, &kept, &kbytes) ||
            launch_las_emit(P<OutRec>(c->las_rec), P<uint8_t>(c->las_raw), perm, P<uint64_t>(c->olen), kept, tbytes,
                            P<uint8_t>(c->las_out), s))
            return -1;
        outbytes = 40 * kept + kbytes;
        GD_CUDA(cudaMemcpyAsync(c->h_rec.p, c->las_out.p, outbytes, cudaMemcpyDeviceToHost, s));
    }
    GD_CUDA(cudaStreamSynchronize(s));
    FILE* g = fopen(out_path, "wb");
    if (!g)
    {
        gd_set_error("Cannot open %s for writing", out_path);
        return -1;
    }
    bool ok = fwrite(&novl, 8, 1, g) == 1 && fwrite(&tspace, 4, 1, g) == 1 &&
              (outbytes == 0 || fwrite(c->h_rec.p, 1, outbytes, g) == outbytes);
    if (fclose(g) || !ok)
    {
        gd_set_error("write to %s failed", out_path);
        return -1;
    }
    return novl;
}

int64_t gd_las_sort(gd_context* c, const char* in_path, const char* out_path)
{
    return las_sort_files(c, &in_path, 1, out_path, 0);
}

int64_t gd_las_merge(gd_context* c, const char* const* in_paths, int nin, const char* out_path)
{
    if (nin <= 0)
    {
        gd_set_error("gd_las_merge: no input files");
        return -1;
    }
    return las_sort_files(c, in_paths, nin, out_path, 1);
}

int64_t gd_dust(gd_context* c, int slot, int window, double thresh, int mflag, int biased, const float freq[4],
                int64_t* anno, int32_t* data, int64_t cap)
{
    using namespace gd;
    if (slot < 0 || slot > 2 || !c->slot[slot].loaded)
    {
        gd_set_error("gd_dust: slot %d not loaded", slot);
        return -1;
    }
    if (!(thresh > 0.) || mflag - 1 <= 0)
    {
        gd_set_error("gd_dust: threshold must be positive and -m at least 2");
        return -1;
    }
    Slot& S = c->slot[slot];
    const int n = S.blk.nreads;
    cudaStream_t s = c->s;
    // 64 triplet weights for -b, in the reference's precision: the product of three float
    // frequencies in float, then .015625 / product in double (db/DBdust.c:244-252)
    double skew[64];
    for (int a = 0, p = 0; a < 4; a++)
        for (int b = 0; b < 4; b++)
            for (int e = 0; e < 4; e++)
            {
                float q = freq[a] * freq[b];
                q = q * freq[e];
                skew[p++] = .015625 / (double)q;
            }
    int64_t boff_end = 0;
    GD_CUDA(cudaMemcpyAsync(&boff_end, S.blk.boff + n, 8, cudaMemcpyDeviceToHost, s));
    GD_CUDA(cudaStreamSynchronize(s));
    const size_t outints = (size_t)boff_end + 4ull * n + 8;
    // scratch: per-read slices (k0), counts (flags), offsets (hoff), packed data (k1), weights (misc)
    if (ensure(c->k0, outints * 4) || ensure(c->flags, (size_t)n * 4 + 4) || ensure(c->hoff, (size_t)n * 8 + 8) ||
        ensure(c->misc, 1024))
        return -1;
    GD_CUDA(cudaMemcpyAsync(c->misc.p, skew, sizeof skew, cudaMemcpyHostToDevice, s));
    if (launch_dust(S.blk, window, thresh, mflag - 1, biased != 0, P<double>(c->misc), P<int>(c->k0),
                    P<int>(c->flags), s))
        return -1;
    std::vector<int> cnt(n);
    GD_CUDA(cudaMemcpyAsync(cnt.data(), c->flags.p, (size_t)n * 4, cudaMemcpyDeviceToHost, s));
    GD_CUDA(cudaStreamSynchronize(s));
    std::vector<int64_t> off(n + 1);
    int64_t total = 0;
    for (int r = 0; r < n; r++)
    {
        if (cnt[r] < 0)
        {
            gd_set_error("gd_dust: read %d overflowed the candidate list", r);
            return -1;
        }
        off[r] = total;
        total += cnt[r];
    }
    off[n] = total;
    if (!anno || !data || cap < total)
        return total;
    if (ensure(c->k1, (size_t)total * 4 + 16))
        return -1;
    GD_CUDA(cudaMemcpyAsync(c->hoff.p, off.data(), (size_t)n * 8, cudaMemcpyHostToDevice, s));
    if (launch_dust_gather(S.blk, P<int>(c->k0), P<int>(c->flags), P<int64_t>(c->hoff), P<int>(c->k1), s))
        return -1;
    if (total)
        GD_CUDA(cudaMemcpyAsync(data, c->k1.p, (size_t)total * 4, cudaMemcpyDeviceToHost, s));
    GD_CUDA(cudaStreamSynchronize(s));
    for (int r = 0; r <= n; r++)
        anno[r] = off[r] * 4;  // the .anno file holds byte offsets
    return total;
}

int64_t gd_get_overlaps(gd_context* c, gd_overlap* recs, uint8_t* trace, int64_t rcap, int64_t tcap)
{
    if (sort_overlaps(c))
        return -1;
    int64_t m = std::min<int64_t>(rcap, (int64_t)c->srt_n);
    if (m <= 0)
        return 0;
    if (m == (int64_t)c->srt_n && (uint64_t)tcap >= c->srt_tb)
    {
        // everything fits: the records and the trace bytes (laid out in record order) in two
        // back-to-back copies
        GD_CUDA(cudaMemcpyAsync(recs, c->srt_rec.p, (size_t)m * sizeof(gd_overlap), cudaMemcpyDeviceToHost, c->s));
        if (c->srt_tb)
            GD_CUDA(cudaMemcpyAsync(trace, c->srt_tr.p, c->srt_tb, cudaMemcpyDeviceToHost, c->s));
        GD_CUDA(cudaStreamSynchronize(c->s));
        return m;
    }
    // the leading records whose traces fit in tcap
    GD_CUDA(cudaMemcpyAsync(recs, c->srt_rec.p, (size_t)m * sizeof(gd_overlap), cudaMemcpyDeviceToHost, c->s));
    GD_CUDA(cudaStreamSynchronize(c->s));
    int tbytes = c->tspace <= 125 ? 1 : 2;
    int64_t n = 0;
    uint64_t end = 0;
    for (; n < m; n++)
    {
        uint64_t e2 = recs[n].toff + (uint64_t)recs[n].tlen * tbytes;
        if ((int64_t)e2 > tcap)
            break;
        end = e2;
    }
    if (end)
    {
        GD_CUDA(cudaMemcpyAsync(trace, c->srt_tr.p, end, cudaMemcpyDeviceToHost, c->s));
        GD_CUDA(cudaStreamSynchronize(c->s));
    }
    return n;
}

int gd_write_overlap_buffer(gd_context* c, int run_id, const char* ablock, const char* bblock, int last_read)
{
    if (stage_sorted(c))
        return -1;
    const size_t nsrt = c->srt_n;
    const gd_overlap* srt = (const gd_overlap*)c->h_rec.p;
    // block ids and roots from the names (dalign/align.c:5858-5877)
    auto split = [](const char* name, std::string& root, int& id) {
        const char* dot = strrchr(name, '.');
        id = 0;
        root = name;
        if (dot)
        {
            id = atoi(dot + 1);
            root = std::string(name, dot - name);
        }
    };
    std::string aroot, broot;
    int aid, bid;
    split(ablock, aroot, aid);
    split(bblock, broot, bid);
    char path1[4096], path2[4096];
    if (strcmp(ablock, bblock) == 0 || c->symmetric == 0)
    {
        std::string dir = dirname_of(run_id, aid);
        if (aid > 0 && bid > 0)
            snprintf(path1, sizeof path1, "%s/%s.%d.%s.%d.las", dir.c_str(), aroot.c_str(), aid, broot.c_str(), bid);
        else if (aid > 0)
            snprintf(path1, sizeof path1, "%s/%s.%d.%s.las", dir.c_str(), aroot.c_str(), aid, broot.c_str());
        else if (bid > 0)
            snprintf(path1, sizeof path1, "%s.%s.%d.las", aroot.c_str(), broot.c_str(), bid);
        else
            snprintf(path1, sizeof path1, "%s.%s.las", aroot.c_str(), broot.c_str());
        return write_las(c, path1, 0, nsrt);
    }
    std::string d1 = dirname_of(run_id, aid), d2 = dirname_of(run_id, bid);
    if (aid > 0)
    {
        if (bid > 0)
        {
            snprintf(path1, sizeof path1, "%s/%s.%d.%s.%d.las", d1.c_str(), aroot.c_str(), aid, broot.c_str(), bid);
            snprintf(path2, sizeof path2, "%s/%s.%d.%s.%d.las", d2.c_str(), broot.c_str(), bid, aroot.c_str(), aid);
        }
        else
        {
            snprintf(path1, sizeof path1, "%s/%s.%d.%s.las", d1.c_str(), aroot.c_str(), aid, broot.c_str());
            snprintf(path2, sizeof path2, "%s.%s.%d.las", broot.c_str(), aroot.c_str(), aid);
        }
    }
    else
    {
        if (bid > 0)
        {
            snprintf(path1, sizeof path1, "%s.%s.%d.las", aroot.c_str(), broot.c_str(), bid);
            snprintf(path2, sizeof path2, "%s/%s.%d.%s.las", d2.c_str(), broot.c_str(), bid, aroot.c_str());
        }
        else
        {
            snprintf(path1, sizeof path1, "%s.%s.las", aroot.c_str(), broot.c_str());
            snprintf(path2, sizeof path2, "%s.%s.las", broot.c_str(), aroot.c_str());
        }
    }
    const char* p1 = path1;
    const char* p2 = path2;
    if (bid < aid)
        std::swap(p1, p2);
    size_t j = 0;
    while (j < nsrt && srt[j].aread <= last_read)
        j++;
    if (write_las(c, p1, 0, j))
        return -1;
    return write_las(c, p2, j, nsrt);
}

int gd_compute_trace_pts(gd_context* c, int aslot, int bslot, int cslot, const gd_overlap* recs, const uint8_t* trace,
                         int64_t n, int32_t* diffs_out)
{
    using namespace gd;
    if (aslot < 0 || aslot > 2 || bslot < 0 || bslot > 2 || cslot < 0 || cslot > 2 || !c->slot[aslot].loaded ||
        !c->slot[bslot].loaded)
    {
        gd_set_error("gd_compute_trace_pts: bad or unloaded slots");
        return -1;
    }
    if (n <= 0)
        return 0;
    Slot& A = c->slot[aslot];
    Slot& B = c->slot[bslot];
    Slot& Cc = c->slot[cslot];
    const int TS = c->tspace;
    const int tbytes = TS <= 125 ? 1 : 2;
    bool any_comp = false;
    std::vector<Segment> seg;
    int R = 8;
    for (int64_t r = 0; r < n; r++)
    {
        const gd_overlap& o = recs[r];
        int ar = o.aread - A.blk.ufirst, br = o.bread - B.blk.ufirst;
        if (ar < 0 || ar >= A.blk.nreads || br < 0 || br >= B.blk.nreads)
        {
            gd_set_error("gd_compute_trace_pts: record %lld names reads outside the loaded blocks", (long long)r);
            return -1;
        }
        if (o.aepos > A.hrlen[ar] || o.bepos > B.hrlen[br] || o.abpos < 0 || o.bbpos < 0 || o.abpos > o.aepos ||
            o.bbpos > o.bepos)
        {
            gd_set_error("gd_compute_trace_pts: record %lld has positions outside its reads", (long long)r);
            return -1;
        }
        int comp = o.flags & 1;
        any_comp |= comp != 0;
        const uint8_t* t = trace + o.toff;
        auto pt = [&](int i) { return tbytes == 1 ? (int)t[i] : (int)(t[2 * i] | (t[2 * i + 1] << 8)); };
        // segments between consecutive trace points (align.c:5355-5389)
        int ab = o.abpos, ae = (o.abpos / TS) * TS, bb = o.bbpos, be;
        for (int i = 1; i < o.tlen - 2; i += 2)
        {
            ae += TS;
            be = bb + pt(i);
            seg.push_back(Segment{ar, br, ab, ae, bb, be, (int32_t)r, comp});
            R = std::max(R, (ae - ab) + (be - bb) + 8);
            ab = ae;
            bb = be;
        }
        seg.push_back(Segment{ar, br, ab, o.aepos, bb, o.bepos, (int32_t)r, comp});
        R = std::max(R, (o.aepos - ab) + (o.bepos - bb) + 8);
    }
    if (any_comp && !Cc.loaded)
    {
        gd_set_error("gd_compute_trace_pts: complemented records need the complemented block in slot %d", cslot);
        return -1;
    }
    int64_t nseg = (int64_t)seg.size();
    int64_t nthreads = std::min<int64_t>(nseg, 148 * 512);
    nthreads = (nthreads + 127) / 128 * 128;
    DevBuf dseg, dscr, ddiff, dst;
    int rc = -1;
    do
    {
        if (ensure(dseg, nseg * sizeof(Segment)) || ensure(dscr, (size_t)nthreads * 3 * (2 * R + 1) * 4) ||
            ensure(ddiff, n * 4) || ensure(dst, sizeof(DevStatus)))
            break;
        // all on the context's stream, which the kernel runs on: a plain cudaMemcpy/cudaMemset
        // goes to the legacy stream, which a non-blocking stream does not wait for
        if (cudaMemcpyAsync(dseg.p, seg.data(), nseg * sizeof(Segment), cudaMemcpyHostToDevice, c->s) != cudaSuccess ||
            cudaMemsetAsync(ddiff.p, 0, n * 4, c->s) != cudaSuccess ||
            cudaMemsetAsync(dst.p, 0, sizeof(DevStatus), c->s) != cudaSuccess)
        {
            gd_set_error("gd_compute_trace_pts: copies failed");
            break;
        }
        if (launch_trace_pts(A.blk, B.blk, Cc.loaded ? Cc.blk : B.blk, P<Segment>(dseg), nseg, P<int>(dscr), R,
                             (int)nthreads, P<int>(ddiff), P<DevStatus>(dst), c->s))
            break;
        DevStatus st;
        if (cudaStreamSynchronize(c->s) != cudaSuccess ||
            cudaMemcpy(&st, dst.p, sizeof st, cudaMemcpyDeviceToHost) != cudaSuccess ||
            cudaMemcpy(diffs_out, ddiff.p, n * 4, cudaMemcpyDeviceToHost) != cudaSuccess)
        {
            gd_set_error("gd_compute_trace_pts: %s", cudaGetErrorString(cudaGetLastError()));
            break;
        }
        if (st.code)
        {
            gd_set_error("gd_compute_trace_pts: record %d failed (code %d)", st.where, st.code);
            break;
        }
        rc = 0;
    } while (0);
    DevBuf* all[] = {&dseg, &dscr, &ddiff, &dst};
    for (DevBuf* b : all)
        release(*b);
    return rc;
}

int gd_reset_overlap_buffer(gd_context* c)
{
    c->acc_n = c->acc_tb = 0;
    c->srt_n = c->srt_tb = 0;
    c->srt_valid = false;
    return 0;
}

int gd_set_wave_limit(gd_context* c, int limit)
{
    if (limit != gd::RING && limit != gd::TEST_RING)
    {
        gd_set_error("gd_set_wave_limit: %d is neither %d nor %d", limit, gd::RING, gd::TEST_RING);
        return -1;
    }
    c->test_narrow = limit == gd::TEST_RING;
    return 0;
}

int gd_set_capacities(gd_context* c, int pebbles, int traces, int paths, int64_t records, int64_t trace_bytes)
{
    if (pebbles > 0)
        c->pcap = pebbles;
    if (traces > 0)
        c->tcap = traces;
    if (paths > 0)
        c->mcap = paths;
    if (records > 0)
        c->rcap = (uint64_t)records;
    if (trace_bytes > 0)
        c->tbcap = (uint64_t)trace_bytes;
    return 0;
}

int gd_set_align_schedule(gd_context* c, int nedges, const int32_t* edges, const int32_t* kind)
{
    if (nedges < 0 || (nedges > 0 && !edges))
    {
        gd_set_error("gd_set_align_schedule: bad edge list");
        return -1;
    }
    for (int i = 0; kind && i <= nedges; i++)
        if (kind[i] < 0 || kind[i] > 2)
        {
            gd_set_error("gd_set_align_schedule: instance %d of class %d is not 0, 1 or 2", kind[i], i);
            return -1;
        }
    c->sched_edges.assign(edges, edges + nedges);
    c->sched_kind.clear();
    if (kind)
        c->sched_kind.assign(kind, kind + nedges + 1);
    return 0;
}

int gd_test_wait_expiry(gd_context* c, int polls)
{
    if (polls < 1)
    {
        gd_set_error("gd_test_wait_expiry: polls must be positive");
        return -2;
    }
    if (gd::radix_sort_test_wait_expiry(polls, c->s))
        return -2;
    return gd::radix_sort_wait_check(c->s);
}

int gd_get_stats(gd_context* c, gd_stats* st)
{
    c->stats.records = (int64_t)c->acc_n;
    *st = c->stats;
    return 0;
}

int gd_local_alignment_batch(gd_context* c, const uint8_t* abases, int64_t alen_total, const uint8_t* bbases,
                             int64_t blen_total, const int64_t* aoff, const int32_t* alen, const int64_t* boff,
                             const int32_t* blen, const int32_t* diag, const int32_t* anti, int nseeds, int comp,
                             int32_t* out12, uint16_t* trace, int trstride, int64_t* cells)
{
    using namespace gd;
    if (!c->spec_set)
    {
        gd_set_error("gd_new_align_spec has not been called");
        return -1;
    }
    if (nseeds <= 0)
        return 0;
    DevBuf da, db, dao, dal, dbo, dbl, dd, dn, dout, dtr, dc, dst;
    int rc = -1;
    int maxlen = 0;
    for (int i = 0; i < nseeds; i++)
        maxlen = std::max(maxlen, std::max(alen[i], blen[i]));
    AlignParams ap{};
    ap.tspace = c->tspace;
    ap.ave_path = c->ave_path;
    ap.comp = comp;
    ap.trace8 = c->tspace <= 125;
    ap.table = P<int16_t>(c->tables);
    ap.score = P<int16_t>(c->tables) + TRIM_TABLE;
    ap.mscore = c->mscore;
    ap.dscore = c->dscore;
    int grid = 0;
    if (align_grid(&grid))
        return -1;
    int nwarps = std::min(grid * ALIGN_WARPS, ((nseeds + ALIGN_WARPS - 1) / ALIGN_WARPS) * ALIGN_WARPS);
    int ptscap = 4 * (2 * (maxlen / c->tspace + 2)) + 32;
    AlignScratch sc{};
    DevBuf scr;
    do
    {
        if (ensure(da, alen_total + 128) || ensure(db, blen_total + 128) || ensure(dao, nseeds * 8) ||
            ensure(dal, nseeds * 4) || ensure(dbo, nseeds * 8) || ensure(dbl, nseeds * 4) ||
            ensure(dd, nseeds * 4) || ensure(dn, nseeds * 4) || ensure(dout, (size_t)nseeds * 48) ||
            ensure(dtr, (size_t)nseeds * trstride * 2) || ensure(dc, nseeds * 8) || ensure(dst, sizeof(DevStatus)) ||
            ensure(scr, align_scratch_bytes(nwarps, c->pcap, ptscap, 4, 4, 4)))
            break;
        align_scratch_carve(&sc, scr.p, nwarps, c->pcap, ptscap, 4, 4, 4);
        // sequences: caller buffers hold [4, read, 4, read, ...] with offsets relative to index 0
        if (cudaMemset(da.p, 4, alen_total + 128) != cudaSuccess || cudaMemset(db.p, 4, blen_total + 128) != cudaSuccess)
            break;
        cudaMemcpy((uint8_t*)da.p + 64, abases, alen_total, cudaMemcpyHostToDevice);
        cudaMemcpy((uint8_t*)db.p + 64, bbases, blen_total, cudaMemcpyHostToDevice);
        cudaMemcpy(dao.p, aoff, nseeds * 8, cudaMemcpyHostToDevice);
        cudaMemcpy(dal.p, alen, nseeds * 4, cudaMemcpyHostToDevice);
        cudaMemcpy(dbo.p, boff, nseeds * 8, cudaMemcpyHostToDevice);
        cudaMemcpy(dbl.p, blen, nseeds * 4, cudaMemcpyHostToDevice);
        cudaMemcpy(dd.p, diag, nseeds * 4, cudaMemcpyHostToDevice);
        cudaMemcpy(dn.p, anti, nseeds * 4, cudaMemcpyHostToDevice);
        cudaMemset(dst.p, 0, sizeof(DevStatus));
        cudaMemset(dout.p, 0, (size_t)nseeds * 48);
        if (launch_la_batch((const uint8_t*)da.p + 64, P<int64_t>(dao), P<int32_t>(dal), (const uint8_t*)db.p + 64,
                            P<int64_t>(dbo), P<int32_t>(dbl), P<int32_t>(dd), P<int32_t>(dn), nseeds, ap, sc,
                            P<int32_t>(dout), P<uint16_t>(dtr), trstride, P<int64_t>(dc), P<DevStatus>(dst), 0))
            break;
        if (cudaDeviceSynchronize() != cudaSuccess)
        {
            gd_set_error("Local_Alignment batch failed: %s", cudaGetErrorString(cudaGetLastError()));
            break;
        }
        DevStatus st;
        cudaMemcpy(&st, dst.p, sizeof st, cudaMemcpyDeviceToHost);
        if (st.code)
        {
            gd_set_error("Local_Alignment batch: seed %d failed with code %d (info %d)", st.where, st.code, st.info);
            break;
        }
        cudaMemcpy(out12, dout.p, (size_t)nseeds * 48, cudaMemcpyDeviceToHost);
        cudaMemcpy(trace, dtr.p, (size_t)nseeds * trstride * 2, cudaMemcpyDeviceToHost);
        cudaMemcpy(cells, dc.p, nseeds * 8, cudaMemcpyDeviceToHost);
        rc = 0;
    } while (0);
    DevBuf* all[] = {&da, &db, &dao, &dal, &dbo, &dbl, &dd, &dn, &dout, &dtr, &dc, &dst, &scr};
    for (DevBuf* b : all)
        release(*b);
    return rc;
}

// ---------------------------------------------------------------------------------------
// learned triage (no counterpart in the reference)
// ---------------------------------------------------------------------------------------

int gd_triage_collect(gd_context* c, int on)
{
    c->tri_collect = on ? 1 : 0;
    return 0;
}

int64_t gd_triage_get_groups(gd_context* c, float* feat, uint32_t* records, uint32_t* cells, int64_t cap)
{
    int64_t n = (int64_t)c->tri_hrec.size();
    int64_t m = std::min(n, cap);
    if (m > 0)
    {
        if (feat)
            memcpy(feat, c->tri_hfeat.data(), (size_t)m * gd::TRI_NF * 4);
        if (records)
            memcpy(records, c->tri_hrec.data(), (size_t)m * 4);
        if (cells)
            memcpy(cells, c->tri_hcells.data(), (size_t)m * 4);
    }
    return n;
}

int gd_triage_reset(gd_context* c)
{
    c->tri_hfeat.clear();
    c->tri_hrec.clear();
    c->tri_hcells.clear();
    return 0;
}

int gd_triage_set_model(gd_context* c, const float* params, float threshold)
{
    if (!params)
    {
        c->tri_on = 0;
        return 0;
    }
    for (int i = 0; i < gd::TRI_NF; i++)
        if (!(params[gd::TRI_OFF_STD + i] > 0.f))
        {
            gd_set_error("triage model: feature %d has a non-positive scale", i);
            return -1;
        }
    if (ensure(c->tri_params, gd::TRI_NPARAM * 4) || ensure(c->tri_misc, 64))
        return -1;
    GD_CUDA(cudaMemcpyAsync(c->tri_params.p, params, gd::TRI_NPARAM * 4, cudaMemcpyHostToDevice, c->s));
    GD_CUDA(cudaStreamSynchronize(c->s));
    c->tri_thr = threshold;
    c->tri_on = 1;
    return 0;
}

int gd_mlp_forward(gd_context* c, const float* params, const float* feat, int64_t n, float* prob)
{
    if (n < 0)
    {
        gd_set_error("gd_mlp_forward: negative row count");
        return -1;
    }
    if (n == 0)
        return 0;
    if (ensure(c->tri_w, gd::TRI_NPARAM * 4) || ensure(c->tri_x, (size_t)n * gd::TRI_NF * 4) ||
        ensure(c->tri_prob, (size_t)n * 4))
        return -1;
    cudaStream_t s = c->s;
    GD_CUDA(cudaMemcpyAsync(c->tri_w.p, params, gd::TRI_NPARAM * 4, cudaMemcpyHostToDevice, s));
    GD_CUDA(cudaMemcpyAsync(c->tri_x.p, feat, (size_t)n * gd::TRI_NF * 4, cudaMemcpyHostToDevice, s));
    if (gd::launch_mlp_forward(P<float>(c->tri_w), P<float>(c->tri_x), n, P<float>(c->tri_prob), s))
        return -1;
    GD_CUDA(cudaMemcpyAsync(prob, c->tri_prob.p, (size_t)n * 4, cudaMemcpyDeviceToHost, s));
    GD_CUDA(cudaStreamSynchronize(s));
    return 0;
}

int gd_mlp_grad(gd_context* c, const float* params, const float* feat, const float* label, int n, float pos_weight,
                float* grad, float* loss)
{
    if (n <= 0)
    {
        gd_set_error("gd_mlp_grad: empty batch");
        return -1;
    }
    if (ensure(c->tri_w, gd::TRI_NPARAM * 4) || ensure(c->tri_x, (size_t)n * gd::TRI_NF * 4) ||
        ensure(c->tri_y, (size_t)n * 4) || ensure(c->tri_grad, gd::TRI_NPARAM * 4) || ensure(c->tri_loss, 16))
        return -1;
    cudaStream_t s = c->s;
    GD_CUDA(cudaMemcpyAsync(c->tri_w.p, params, gd::TRI_NPARAM * 4, cudaMemcpyHostToDevice, s));
    GD_CUDA(cudaMemcpyAsync(c->tri_x.p, feat, (size_t)n * gd::TRI_NF * 4, cudaMemcpyHostToDevice, s));
    GD_CUDA(cudaMemcpyAsync(c->tri_y.p, label, (size_t)n * 4, cudaMemcpyHostToDevice, s));
    if (gd::launch_mlp_grad(P<float>(c->tri_w), P<float>(c->tri_x), P<float>(c->tri_y), n, pos_weight,
                            P<float>(c->tri_grad), P<float>(c->tri_loss), s))
        return -1;
    GD_CUDA(cudaMemcpyAsync(grad, c->tri_grad.p, gd::TRI_NPARAM * 4, cudaMemcpyDeviceToHost, s));
    GD_CUDA(cudaMemcpyAsync(loss, c->tri_loss.p, 4, cudaMemcpyDeviceToHost, s));
    GD_CUDA(cudaStreamSynchronize(s));
    return 0;
}

static uint64_t splitmix64(uint64_t& x)
{
    uint64_t z = (x += 0x9e3779b97f4a7c15ull);
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
    return z ^ (z >> 31);
}

int gd_mlp_init(const float* feat, int64_t n, uint64_t seed, float* params)
{
    using namespace gd;
    if (n <= 0)
    {
        gd_set_error("gd_mlp_init: no rows");
        return -1;
    }
    memset(params, 0, TRI_NPARAM * 4);
    for (int f = 0; f < TRI_NF; f++)
    {
        double s = 0, q = 0;
        for (int64_t i = 0; i < n; i++)
        {
            double v = feat[i * TRI_NF + f];
            s += v;
            q += v * v;
        }
        double mean = s / n, var = q / n - mean * mean;
        params[TRI_OFF_MEAN + f] = (float)mean;
        params[TRI_OFF_STD + f] = (float)(var > 1e-12 ? sqrt(var) : 1.0);
    }
    // He-uniform weights, zero biases
    uint64_t st = seed;
    auto uni = [&](double bound) {
        double u = (double)(splitmix64(st) >> 11) * (1.0 / 9007199254740992.0);
        return (float)((2 * u - 1) * bound);
    };
    for (int i = 0; i < TRI_H * TRI_NF; i++)
        params[TRI_OFF_W1 + i] = uni(sqrt(6.0 / TRI_NF));
    for (int i = 0; i < TRI_H * TRI_H; i++)
        params[TRI_OFF_W2 + i] = uni(sqrt(6.0 / TRI_H));
    for (int i = 0; i < TRI_H; i++)
        params[TRI_OFF_W3 + i] = uni(sqrt(3.0 / TRI_H));
    return 0;
}

int gd_mlp_train(gd_context* c, const float* feat, const float* label, int64_t n, int epochs, int batch, float lr,
                 float pos_weight, uint64_t seed, float* params, float* epoch_loss)
{
    using namespace gd;
    if (n <= 0 || batch <= 0 || epochs <= 0 || n > INT32_MAX)
    {
        gd_set_error("gd_mlp_train: bad sizes (n %lld, batch %d, epochs %d)", (long long)n, batch, epochs);
        return -1;
    }
    const int64_t nb = (n + batch - 1) / batch;
    cudaStream_t s = c->s;
    if (ensure(c->tri_w, TRI_NPARAM * 4) || ensure(c->tri_x, (size_t)n * TRI_NF * 4) || ensure(c->tri_y, (size_t)n * 4) ||
        ensure(c->tri_perm, (size_t)n * 4) || ensure(c->tri_grad, TRI_NPARAM * 4) || ensure(c->tri_m, TRI_NPARAM * 4) ||
        ensure(c->tri_v, TRI_NPARAM * 4) || ensure(c->tri_loss, (size_t)nb * 4))
        return -1;
    GD_CUDA(cudaMemcpyAsync(c->tri_w.p, params, TRI_NPARAM * 4, cudaMemcpyHostToDevice, s));
    GD_CUDA(cudaMemcpyAsync(c->tri_x.p, feat, (size_t)n * TRI_NF * 4, cudaMemcpyHostToDevice, s));
    GD_CUDA(cudaMemcpyAsync(c->tri_y.p, label, (size_t)n * 4, cudaMemcpyHostToDevice, s));
    GD_CUDA(cudaMemsetAsync(c->tri_m.p, 0, TRI_NPARAM * 4, s));
    GD_CUDA(cudaMemsetAsync(c->tri_v.p, 0, TRI_NPARAM * 4, s));
    std::vector<int> perm(n);
    std::vector<float> bl(nb);
    uint64_t st = seed ^ 0x5bd1e995ull;
    int step = 0;
    for (int ep = 0; ep < epochs; ep++)
    {
        for (int64_t i = 0; i < n; i++)
            perm[i] = (int)i;
        for (int64_t i = n - 1; i > 0; i--)
            std::swap(perm[i], perm[splitmix64(st) % (uint64_t)(i + 1)]);
        GD_CUDA(cudaMemcpyAsync(c->tri_perm.p, perm.data(), (size_t)n * 4, cudaMemcpyHostToDevice, s));
        for (int64_t b = 0; b < nb; b++)
        {
            int64_t r0 = b * batch;
            int rows = (int)std::min<int64_t>(batch, n - r0);
            if (launch_mlp_grad_perm(P<float>(c->tri_w), P<float>(c->tri_x), P<float>(c->tri_y), P<int>(c->tri_perm),
                                     r0, rows, pos_weight, P<float>(c->tri_grad), P<float>(c->tri_loss) + b, s) ||
                launch_adam(P<float>(c->tri_w), P<float>(c->tri_grad), P<float>(c->tri_m), P<float>(c->tri_v), ++step,
                            lr, s))
                return -1;
        }
        GD_CUDA(cudaMemcpyAsync(bl.data(), c->tri_loss.p, (size_t)nb * 4, cudaMemcpyDeviceToHost, s));
        GD_CUDA(cudaStreamSynchronize(s));
        if (epoch_loss)
        {
            double sum = 0, w = 0;
            for (int64_t b = 0; b < nb; b++)
            {
                double rows = (double)std::min<int64_t>(batch, n - b * batch);
                sum += bl[b] * rows;
                w += rows;
            }
            epoch_loss[ep] = (float)(sum / w);
        }
    }
    GD_CUDA(cudaMemcpyAsync(params, c->tri_w.p, TRI_NPARAM * 4, cudaMemcpyDeviceToHost, s));
    GD_CUDA(cudaStreamSynchronize(s));
    return 0;
}

}  // extern "C"
