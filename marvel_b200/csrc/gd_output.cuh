// gd_output.cuh -- the overlap buffer in HBM: append per Match_Filter, sort and compact on
// the device for Write_Overlap_Buffer / read-out.
#pragma once
#include "gd_align.cuh"
#include "gd_common.cuh"

namespace gd
{

// dst[i] = src[i] with toff += t0 (appending one Match_Filter's records to the buffer)
int launch_ovl_append(const OutRec* src, uint64_t n, uint64_t t0, OutRec* dst, cudaStream_t s);

// ext[0] = min read id, ext[1] = max read id, ext[2] = max position over a and b
// coordinates (ext must hold {UINT_MAX, 0, 0} on entry)
int launch_ovl_extent(const OutRec* r, uint64_t n, unsigned* ext, cudaStream_t s);

// low sort key (orientation, abpos, aepos, bbpos) with pbits bits per position -- without
// the orientation when with_comp is 0 (LAsort's key); val[i] = i
int launch_ovl_key_lo(const OutRec* r, uint64_t n, int pbits, int with_comp, uint64_t* key, uint32_t* val,
                      cudaStream_t s);

// high sort key of r[perm[i]]: (dropped, aread - rmin, bread - rmin) with rbits per read id;
// a record is dropped when only_identity and aread != bread; *nkept counts the others
int launch_ovl_key_hi(const OutRec* r, const uint32_t* perm, uint64_t n, int rbits, unsigned rmin, int only_identity,
                      uint64_t* key, unsigned long long* nkept, cudaStream_t s);

// len[i] = trace bytes of r[perm[i]]
int launch_ovl_len(const OutRec* r, const uint32_t* perm, uint64_t n, int tbytes, uint64_t* len, cudaStream_t s);

// out[i] = r[perm[i]] with its trace moved to outtr + off[i] (toff = off[i]); first n records
int launch_ovl_gather(const OutRec* r, const uint8_t* tr, const uint32_t* perm, const uint64_t* off, uint64_t n,
                      int tbytes, OutRec* out, uint8_t* outtr, cudaStream_t s);

// .las records at byte offsets off[i] of raw (the 40-byte header of each) -> rec[i], with
// toff = off[i] + 40 (its trace bytes in raw) and the header's pad word kept in pad
int launch_las_parse(const uint8_t* raw, const int64_t* off, uint64_t n, OutRec* rec, cudaStream_t s);

// the .las byte stream of r[perm[0..n)]: record i's 40-byte header (pad kept) at
// out + 40 * i + toff[i], its trace bytes right after
int launch_las_emit(const OutRec* r, const uint8_t* tr, const uint32_t* perm, const uint64_t* toff, uint64_t n,
                    int tbytes, uint8_t* out, cudaStream_t s);

}  // namespace gd
