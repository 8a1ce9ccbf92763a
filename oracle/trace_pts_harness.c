/* trace_pts_harness.c -- the reference's Compute_Trace_PTS on every record of a .las file.
 *
 * Test infrastructure only: oracle/Makefile links this file with the reference's own
 * dalign/align.c and DB sources into oracle/_ref/trace_pts_harness; nothing of it ships.
 * For each record of the file, in file order, it loads the A read and the B read
 * (complemented for a COMP record, as LAcheck -a does, utils/LAcheck.c:232-248), hands the
 * record's trace points (widened to uint16 when the file stores bytes) to
 * Compute_Trace_PTS (dalign/align.c:5286-5397, mode 0 = GREEDIEST) and prints the diffs it
 * computes, one line per record.  The fixtures it makes pin the restatement of iter_np
 * (oracle/dalign_oracle.c) and the device verifier (gd_compute_trace_pts).
 *
 * usage: trace_pts_harness <db> <file.las>
 */
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "dalign/align.h"
#include "db/DB.h"

int main(int argc, char* argv[])
{
    if (argc != 3)
    {
        fprintf(stderr, "usage: %s <db> <file.las>\n", argv[0]);
        return 1;
    }
    HITS_DB db;
    if (Open_DB(argv[1], &db) < 0)
    {
        fprintf(stderr, "cannot open %s\n", argv[1]);
        return 1;
    }
    FILE* f = fopen(argv[2], "rb");
    if (!f)
    {
        fprintf(stderr, "cannot open %s\n", argv[2]);
        return 1;
    }
    int64_t novl;
    int32_t tspace;
    if (fread(&novl, 8, 1, f) != 1 || fread(&tspace, 4, 1, f) != 1)
    {
        fprintf(stderr, "truncated header\n");
        return 1;
    }
    int tbytes = tspace <= TRACE_XOVR ? 1 : 2;
    char* aseq = New_Read_Buffer(&db);
    char* bseq = New_Read_Buffer(&db);
    Work_Data* work = New_Work_Data();
    Path path;
    Alignment align;
    align.path = &path;
    align.aseq = aseq;
    align.bseq = bseq;
    size_t cap = 0;
    uint8_t* raw = NULL;
    uint16_t* pts = NULL;
    for (int64_t i = 0; i < novl; i++)
    {
        int32_t r[10];  // tlen, diffs, abpos, bbpos, aepos, bepos, flags, aread, bread, pad
        if (fread(r, 4, 10, f) != 10)
        {
            fprintf(stderr, "truncated record %lld\n", (long long)i);
            return 1;
        }
        int tlen = r[0];
        if ((size_t)tlen + 1 > cap)
        {
            cap = 2 * (size_t)tlen + 16;
            raw = realloc(raw, cap * 2);
            pts = realloc(pts, cap * 2);
        }
        if (tlen > 0 && fread(raw, tbytes, tlen, f) != (size_t)tlen)
        {
            fprintf(stderr, "truncated trace %lld\n", (long long)i);
            return 1;
        }
        for (int j = 0; j < tlen; j++)
            pts[j] = tbytes == 1 ? raw[j] : ((uint16_t*)raw)[j];
        int aread = r[7], bread = r[8];
        Load_Read(&db, aread, aseq, 0);
        Load_Read(&db, bread, bseq, 0);
        align.alen = db.reads[aread].rlen;
        align.blen = db.reads[bread].rlen;
        align.flags = (uint32)r[6];
        if (COMP(align.flags))
            Complement_Seq(bseq, align.blen);
        path.trace = pts;
        path.tlen = tlen;
        path.diffs = r[1];
        path.abpos = r[2];
        path.bbpos = r[3];
        path.aepos = r[4];
        path.bepos = r[5];
        Compute_Trace_PTS(&align, work, tspace, 0, 0);
        printf("%d\n", path.diffs);
    }
    fclose(f);
    Free_Work_Data(work);
    Close_DB(&db);
    return 0;
}
