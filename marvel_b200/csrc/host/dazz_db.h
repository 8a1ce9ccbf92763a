/* dazz_db.h -- Dazzler DB blocks and mask tracks for the daligner driver (host C).
 *
 * Reads the formats MARVEL's DB library writes: the .db stub (db/DB.h:239-249), .idx
 * (raw HITS_DB header + HITS_READ records, db/DB.c:424-450), .bps (2-bit bases, MSB
 * first, db/DB.c:261-309) and interval tracks in the .anno/.data layout Load_Track reads
 * (db/DB.c:967-1120).  A loaded block has the in-memory layout of Read_All_Sequences
 * (db/DB.c:1349-1410), which is what gd_load_block takes.
 */
#ifndef DAZZ_DB_H
#define DAZZ_DB_H
#include <stddef.h>
#include <stdint.h>

typedef struct
{
    int32_t nreads, maxlen, ufirst, part, ureads;
    int64_t totlen;
    float freq[4];
    uint8_t* buf;      /* allocation: 32 bytes slack | 4 | read0 | 4 | ... | 4 | slack */
    uint8_t* bases;    /* read 0's first base; bases[-1] == 4 */
    int64_t* boff;     /* [nreads+1] */
    int32_t* rlen;     /* [nreads] */
    int64_t* mask_anno; /* [nreads+1] index into mask_data, or NULL */
    int32_t* mask_data; /* (begin,end) pairs */
    char dir[4096];    /* directory of the DB */
    char root[1024];   /* DB name without .db and block suffix */
} dz_block;

/* Opens "X", "X.db", "X.n" or "X.n.db" (n = block number) and loads its bases. */
int dz_open_block(const char* path, dz_block* b, char* err, size_t errlen);

/* Adds the named interval track as a mask (the per-block file ".X.n.track.anno" if it
 * exists, else the whole-DB ".X.track.anno" restricted to the block); several calls take
 * the union of the tracks' intervals. */
int dz_add_mask(dz_block* b, const char* track, char* err, size_t errlen);

void dz_free(dz_block* b);

#endif
