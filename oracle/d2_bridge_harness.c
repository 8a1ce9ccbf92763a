/* d2_bridge_harness.c -- TEST INFRASTRUCTURE ONLY: drives the reference daligner2's own
 * Handle_Redundancies (dalign2/filter.c:1952-2272, bridging included) on path sets read from
 * stdin, so that the restatement of its fusion and bridging passes can be pinned against it.
 * Built by oracle/Makefile against the reference sources into oracle/_ref/; never shipped.
 *
 * Input, repeated until EOF (little-endian int32 unless noted):
 *   alen blen tspace comp novls hasB
 *   aseq[alen] bseq[blen]              (bytes 0..3; bseq already complemented when comp)
 *   novls x { abpos bbpos aepos bepos diffs tlen trace[tlen] (uint16) }      amatch
 *   hasB ? novls x { ... }                                                   bmatch
 * Output per case, to the file named by argv[1] (the reference prints notes to stdout): n,
 * then n x { abpos bbpos aepos bepos diffs tlen trace[tlen] } of amatch and, with hasB, of
 * bmatch.
 */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "filter.h"

/* the daligner2 globals filter.c expects from its main (dalign2/daligner.c:24-40) */
int BIASED = 0, VERBOSE = 0, MINOVER = 0, HGAP_MIN = 0, SYMMETRIC = 1, IDENTITY = 0;
char* SORT_PATH = "/tmp";
uint64_t MEM_LIMIT = 0, MEM_PHYSICAL = 0;

static int rd(void* p, size_t n)
{
    return fread(p, 1, n, stdin) == n;
}

static int read_paths(Path* p, int n, Trace_Buffer* tb)
{
    for (int i = 0; i < n; i++)
    {
        int h[6];
        if (!rd(h, sizeof h))
            return 0;
        p[i].abpos = h[0];
        p[i].bbpos = h[1];
        p[i].aepos = h[2];
        p[i].bepos = h[3];
        p[i].diffs = h[4];
        p[i].tlen = h[5];
        if (tb->top + h[5] + 16 > tb->max)
        {
            tb->max = 2 * (tb->top + h[5]) + 1000;
            tb->trace = (uint16*)realloc(tb->trace, sizeof(uint16) * tb->max);
        }
        if (!rd(tb->trace + tb->top, sizeof(uint16) * h[5]))
            return 0;
        p[i].trace = (void*)(uint64)tb->top;
        tb->top += h[5];
    }
    return 1;
}

static void write_paths(FILE* out, const Path* p, int n, const Trace_Buffer* tb)
{
    for (int i = 0; i < n; i++)
    {
        int h[6] = {p[i].abpos, p[i].bbpos, p[i].aepos, p[i].bepos, p[i].diffs, p[i].tlen};
        fwrite(h, sizeof h, 1, out);
        fwrite(tb->trace + (uint64)p[i].trace, sizeof(uint16), p[i].tlen, out);
    }
}

int main(int argc, char** argv)
{
    if (argc < 2)
        return 2;
    FILE* out = fopen(argv[1], "wb");
    if (out == NULL)
        return 2;
    Work_Data* work = New_Work_Data();
    Trace_Buffer tb = {0, 0, NULL};
    for (;;)
    {
        int h[6];
        if (!rd(h, sizeof h))
            break;
        int alen = h[0], blen = h[1], novls = h[4], hasB = h[5];
        MR_tspace = h[2];
        char* abuf = (char*)malloc(alen + 2);
        char* bbuf = (char*)malloc(blen + 2);
        abuf[0] = abuf[alen + 1] = 4;
        bbuf[0] = bbuf[blen + 1] = 4;
        Path* am = (Path*)malloc(sizeof(Path) * (novls + 1));
        Path* bm = (Path*)malloc(sizeof(Path) * (novls + 1));
        tb.top = 0;
        if (!rd(abuf + 1, alen) || !rd(bbuf + 1, blen) || !read_paths(am, novls, &tb) ||
            (hasB && !read_paths(bm, novls, &tb)))
            return 1;
        Path scratch;
        memset(&scratch, 0, sizeof scratch);
        Alignment align;
        memset(&align, 0, sizeof align);
        align.path = &scratch;
        align.flags = h[3] ? COMP_FLAG : 0;
        align.aseq = abuf + 1;
        align.bseq = bbuf + 1;
        align.alen = alen;
        align.blen = blen;
        int n = Handle_Redundancies(am, novls, hasB ? bm : NULL, &align, work, &tb);
        fwrite(&n, sizeof n, 1, out);
        write_paths(out, am, n, &tb);
        if (hasB)
            write_paths(out, bm, n, &tb);
        free(abuf);
        free(bbuf);
        free(am);
        free(bm);
    }
    fclose(out);
    return 0;
}
