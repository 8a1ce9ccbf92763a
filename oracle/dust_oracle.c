/* dust_oracle.c -- CPU restatement of DBdust's low-complexity scan (db/DBdust.c:219-487).
 *
 * TEST INFRASTRUCTURE ONLY: the checker for the device DUST kernel, pinned against the
 * reference DBdust's own track files (tests/golden/dust).
 *
 * Per read, over the triplet codes t(x) = 16 b[x] + 4 b[x+1] + b[x+2] (x < len - 2):
 *   * a window of the last W-2 triplets, with its count table and sum of pair counts
 *     (wsqr: sum over codes of count*(count-1)/2, kept incrementally);
 *   * a left-trimmed run [lb+1, j] with the same kind of count table (lsqr), cut back so
 *     that no code in it reaches a pair count of ceil(2*T);
 *   * a list of candidate "perfect intervals" (start, end, score), newest start first,
 *     retired into the read's mask when their start leaves the window;
 *   * when the window scores above T, the run is scanned right to left for starts whose
 *     run score beats T and every candidate it contains.
 * Intervals of at least minlen+1 triplet positions are reported as [beg, end+3).
 * -b weights pair counts by the inverse triplet frequency (skew).  Arithmetic follows the
 * reference's types: integer sums without -b, doubles with it (no fused multiply-add).
 */
#include <math.h>
#include <stdint.h>
#include <string.h>

#define DUST_MAXW 256

typedef struct
{
    int beg, end;
    double score;
    int prev, next;
} Cand;

static inline int trip(const uint8_t* b, int x)
{
    return (b[x] << 4) | (b[x + 1] << 2) | b[x + 2];
}

/* mask[0] is a sentinel; merges [beg, end+2] into the last mask interval or appends it */
static inline void retire(int* mask, int* mtop, int beg, int end)
{
    int c = end + 2;
    if (mask[*mtop] + 1 >= beg)
    {
        if (mask[*mtop] < c)
            mask[*mtop] = c;
    }
    else
    {
        mask[++*mtop] = beg;
        mask[++*mtop] = c;
    }
}

/* One read: writes (beg, end) pairs into out (room for rlen + 4 ints); returns the number of
 * ints written.  work needs rlen + 4 ints. */
int or_dust_read(const uint8_t* b, int rlen, int W, double T, int minlen, int biased, const double* skew, int* out,
                 int* work)
{
    if (W > DUST_MAXW || W < 3)
        return -1;
    int len = rlen - 2;
    int* mask = work;
    int mtop = 0;
    mask[0] = -2;
    if (len > 0)
    {
        Cand cd[DUST_MAXW + 1];
        int wcount[64], lcount[64];
        int freel, i, j, x, d;
        memset(wcount, 0, sizeof wcount);
        memset(lcount, 0, sizeof lcount);
        cd[0].beg = -2;
        cd[0].prev = cd[0].next = 0;
        for (i = 1; i <= W; i++)
            cd[i].next = (i < W) ? i + 1 : -1;
        freel = 1;
        int wb = -1, lb = -1;
        const int thr2i = (int)ceil(2. * T);
        const double thr2r = 2. * T;
        long long wsi = 0, lsi = 0; /* integer sums (no -b) */
        double wsr = 0., lsr = 0.;  /* weighted sums (-b) */
#define ADD(cnt, e, si, sr)                                 \
    do                                                      \
    {                                                       \
        if (biased)                                         \
            sr = sr + (double)(cnt[e]) * skew[e];           \
        else                                                \
            si += cnt[e];                                   \
        cnt[e]++;                                           \
    } while (0)
#define DEL(cnt, e, si, sr)                                 \
    do                                                      \
    {                                                       \
        cnt[e]--;                                           \
        if (biased)                                         \
            sr = sr - (double)(cnt[e]) * skew[e];           \
        else                                                \
            si -= cnt[e];                                   \
    } while (0)
        for (j = 0; j < len; j++)
        {
            int c = trip(b, j);
            if (j > W - 3)
            {
                d = trip(b, ++wb);
                DEL(wcount, d, wsi, wsr);
            }
            ADD(wcount, c, wsi, wsr);
            if (lb < wb)
            {
                d = trip(b, ++lb);
                DEL(lcount, d, lsi, lsr);
            }
            int cut;
            if (biased)
            {
                double tr = (double)lcount[c] * skew[c];
                lcount[c]++;
                lsr = lsr + tr;
                cut = tr >= thr2r;
            }
            else
            {
                int tr = lcount[c]++;
                lsi += tr;
                cut = tr >= thr2i;
            }
            if (cut)
                while (lb < j)
                {
                    d = trip(b, ++lb);
                    DEL(lcount, d, lsi, lsr);
                    if (d == c)
                        break;
                }
            /* retire the oldest candidate once its start has left the window */
            int t = cd[0].prev;
            if (t != 0 && cd[t].beg <= wb)
            {
                retire(mask, &mtop, cd[t].beg, cd[t].end);
                int p = cd[t].prev;
                cd[0].prev = p;
                cd[p].next = 0;
                cd[t].next = freel;
                freel = t;
            }
            double lsq = biased ? lsr : (double)lsi, wsq = biased ? wsr : (double)wsi;
            if (wsq <= lsq * T)
                continue;
            int jp = cd[0].next, lp = 0;
            double ms = 0.;
            for (x = lb; x > wb; x--)
            {
                d = trip(b, x);
                ADD(lcount, d, lsi, lsr);
                lsq = biased ? lsr : (double)lsi;
                if (lsq >= T * (j - x))
                {
                    for (; cd[jp].beg >= x; lp = jp, jp = cd[jp].next)
                        if (cd[jp].score > ms)
                            ms = cd[jp].score;
                    if (lsq >= ms * (j - x))
                    {
                        ms = lsq / (j - x);
                        if (cd[lp].beg == x)
                        {
                            cd[lp].end = j;
                            cd[lp].score = ms;
                        }
                        else
                        {
                            int n = freel;
                            if (n < 0)
                                return -2;
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
                d = trip(b, x);
                DEL(lcount, d, lsi, lsr);
            }
        }
#undef ADD
#undef DEL
        /* remaining candidates, oldest first */
        int t;
        while ((t = cd[0].prev) != 0)
        {
            retire(mask, &mtop, cd[t].beg, cd[t].end);
            int p = cd[t].prev;
            cd[0].prev = p;
            cd[p].next = 0;
        }
    }
    int n = 0;
    for (int k = 1; k < mtop; k += 2)
        if (mask[k + 1] - mask[k] >= minlen)
        {
            out[n++] = mask[k];
            out[n++] = mask[k + 1] + 1;
        }
    return n;
}
