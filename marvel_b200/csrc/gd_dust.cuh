// gd_dust.cuh -- DBdust's low-complexity scan on the device (one read per thread).
#pragma once
#include "gd_common.cuh"

namespace gd
{

constexpr int DUST_MAXW = 128;  // largest scan window (-w) of the device scan

// For every read of blk: the reported intervals as (beg, end) pairs at out + boff[r] + 4 r
// (room for rlen + 4 ints per read) and their int count in nout[r] (-1: candidate list
// overflow).  minlen is DBdust's MINLEN (-m value - 1); skew (64 doubles) is used with biased.
int launch_dust(const DevBlock& blk, int window, double thresh, int minlen, bool biased, const double* skew, int* out,
                int* nout, cudaStream_t s);

// packs the per-read results: read r's nout[r] ints to dst + off[r]
int launch_dust_gather(const DevBlock& blk, const int* out, const int* nout, const int64_t* off, int* dst,
                       cudaStream_t s);

}  // namespace gd
