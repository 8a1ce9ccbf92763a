// gd_dust.cu -- DBdust's low-complexity scan (db/DBdust.c:219-487) on the device.
//
// The scan of one read is a sequential state machine (a window of triplet counts, a
// left-trimmed run with its own counts, a short list of candidate intervals), so the GPU
// runs one read per thread: a block of a few thousand to tens of thousands of reads keeps
// the SMs busy, the counts and candidate list live in the thread's local memory (L1), and
// each read's mask is written to its own slice of a device buffer.  Arithmetic follows the
// reference's types: integer pair-count sums, doubles for the thresholds, and with -b
// (biased) double sums of count * skew, computed with explicit round-to-nearest operations
// so that no multiply-add is fused (the reference's x86-64 build has none either).
#include <cmath>

#include "gd_dust.cuh"

namespace gd
{

struct DustCand
{
    int beg, end;
    double score;
    int prev, next;
};

__device__ __forceinline__ int dtrip(const uint8_t* b, int x)
{
    return (b[x] << 4) | (b[x + 1] << 2) | b[x + 2];
}

__device__ __forceinline__ void dust_retire(int* mask, int& mtop, int beg, int end)
{
    const int c = end + 2;
    if (mask[mtop] + 1 >= beg)
    {
        if (mask[mtop] < c)
            mask[mtop] = c;
    }
    else
    {
        mask[++mtop] = beg;
        mask[++mtop] = c;
    }
}

template <bool BIASED>
__global__ void __launch_bounds__(64) k_dust(DevBlock blk, int W, double T, int thr2i, double thr2r,
                                             const double* __restrict__ skew, int minlen, int* out,
                                             int* __restrict__ nout)
{
    const int r = blockIdx.x * 64 + threadIdx.x;
    if (r >= blk.nreads)
        return;
    const int rlen = blk.rlen[r];
    const uint8_t* b = blk.bases + blk.boff[r];
    int* mask = out + blk.boff[r] + 4ll * r;  // room for rlen + 4 ints
    int mtop = 0;
    mask[0] = -2;
    const int len = rlen - 2;
    if (len > 0)
    {
        DustCand cd[DUST_MAXW + 1];
        int wcount[64], lcount[64];
        for (int e = 0; e < 64; e++)
            wcount[e] = lcount[e] = 0;
        cd[0].beg = -2;
        cd[0].prev = cd[0].next = 0;
        for (int i = 1; i <= W; i++)
            cd[i].next = (i < W) ? i + 1 : -1;
        int freel = 1, wb = -1, lb = -1;
        long long wsi = 0, lsi = 0;
        double wsr = 0., lsr = 0.;
        auto add = [&](int* cnt, int e, long long& si, double& sr) {
            if (BIASED)
                sr = __dadd_rn(sr, __dmul_rn((double)cnt[e], skew[e]));
            else
                si += cnt[e];
            cnt[e]++;
        };
        auto del = [&](int* cnt, int e, long long& si, double& sr) {
            cnt[e]--;
            if (BIASED)
                sr = __dsub_rn(sr, __dmul_rn((double)cnt[e], skew[e]));
            else
                si -= cnt[e];
        };
        for (int j = 0; j < len; j++)
        {
            const int c = dtrip(b, j);
            int d;
            if (j > W - 3)
            {
                d = dtrip(b, ++wb);
                del(wcount, d, wsi, wsr);
            }
            add(wcount, c, wsi, wsr);
            if (lb < wb)
            {
                d = dtrip(b, ++lb);
                del(lcount, d, lsi, lsr);
            }
            bool cut;
            if (BIASED)
            {
                const double tr = __dmul_rn((double)lcount[c], skew[c]);
                lcount[c]++;
                lsr = __dadd_rn(lsr, tr);
                cut = tr >= thr2r;
            }
            else
            {
                const int tr = lcount[c]++;
                lsi += tr;
                cut = tr >= thr2i;
            }
            if (cut)
                while (lb < j)
                {
                    d = dtrip(b, ++lb);
                    del(lcount, d, lsi, lsr);
                    if (d == c)
                        break;
                }
            // retire the oldest candidate once its start has left the window
            const int t = cd[0].prev;
            if (t != 0 && cd[t].beg <= wb)
            {
                dust_retire(mask, mtop, cd[t].beg, cd[t].end);
                const int p = cd[t].prev;
                cd[0].prev = p;
                cd[p].next = 0;
                cd[t].next = freel;
                freel = t;
            }
            double lsq = BIASED ? lsr : (double)lsi;
            const double wsq = BIASED ? wsr : (double)wsi;
            if (wsq <= __dmul_rn(lsq, T))
                continue;
            int jp = cd[0].next, lp = 0, x;
            double ms = 0.;
            for (x = lb; x > wb; x--)
            {
                d = dtrip(b, x);
                add(lcount, d, lsi, lsr);
                lsq = BIASED ? lsr : (double)lsi;
                if (lsq >= __dmul_rn(T, (double)(j - x)))
                {
                    for (; cd[jp].beg >= x; lp = jp, jp = cd[jp].next)
                        if (cd[jp].score > ms)
                            ms = cd[jp].score;
                    if (lsq >= __dmul_rn(ms, (double)(j - x)))
                    {
                        ms = __ddiv_rn(lsq, (double)(j - x));
                        if (cd[lp].beg == x)
                        {
                            cd[lp].end = j;
                            cd[lp].score = ms;
                        }
                        else
                        {
                            const int n = freel;
                            if (n < 0)
                            {
                                nout[r] = -1;  // candidate pool exhausted
                                return;
                            }
                            freel = cd[n].next;
                            cd[n].beg = x;
                            cd[n].end = j;
                            cd[n].score = ms;
                            cd[n].prev = lp;
                            cd[lp].next = n;
                            cd[n].next = jp;
                            cd[jp].prev = n;
                            lp = n;
                        }
                    }
                }
            }
            for (x++; x <= lb; x++)
            {
                d = dtrip(b, x);
                del(lcount, d, lsi, lsr);
            }
        }
        int t;
        while ((t = cd[0].prev) != 0)
        {
            dust_retire(mask, mtop, cd[t].beg, cd[t].end);
            const int p = cd[t].prev;
            cd[0].prev = p;
            cd[p].next = 0;
        }
    }
    // keep intervals of more than minlen positions, as [beg, end + 1), in place
    int n = 0;
    for (int k = 1; k < mtop; k += 2)
        if (mask[k + 1] - mask[k] >= minlen)
        {
            const int bg = mask[k], en = mask[k + 1] + 1;
            mask[n++] = bg;
            mask[n++] = en;
        }
    nout[r] = n;
}

// packs read r's nout[r] ints to dst + off[r] (one warp per read)
__global__ void k_dust_gather(DevBlock blk, const int* __restrict__ out, const int* __restrict__ nout,
                              const int64_t* __restrict__ off, int* __restrict__ dst)
{
    const int64_t w = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (w >= blk.nreads)
        return;
    const int* src = out + blk.boff[w] + 4 * w;
    for (int j = lane_id(); j < nout[w]; j += 32)
        dst[off[w] + j] = src[j];
}

int launch_dust_gather(const DevBlock& blk, const int* out, const int* nout, const int64_t* off, int* dst,
                       cudaStream_t s)
{
    if (blk.nreads <= 0)
        return 0;
    const int64_t threads = (int64_t)blk.nreads * 32;
    k_dust_gather<<<(unsigned)((threads + 255) / 256), 256, 0, s>>>(blk, out, nout, off, dst);
    GD_LAUNCHED(1);
    GD_CUDA(cudaGetLastError());
    return 0;
}

int launch_dust(const DevBlock& blk, int window, double thresh, int minlen, bool biased, const double* skew, int* out,
                int* nout, cudaStream_t s)
{
    if (blk.nreads <= 0)
        return 0;
    if (window < 3 || window > DUST_MAXW)
    {
        gd_set_error("DUST window %d outside [3, %d]", window, DUST_MAXW);
        return -1;
    }
    const int thr2i = (int)std::ceil(2. * thresh);
    const double thr2r = 2. * thresh;
    const unsigned grid = (unsigned)((blk.nreads + 63) / 64);
    if (biased)
        k_dust<true><<<grid, 64, 0, s>>>(blk, window, thresh, thr2i, thr2r, skew, minlen, out, nout);
    else
        k_dust<false><<<grid, 64, 0, s>>>(blk, window, thresh, thr2i, thr2r, skew, minlen, out, nout);
    GD_LAUNCHED(1);
    GD_CUDA(cudaGetLastError());
    return 0;
}

}  // namespace gd
