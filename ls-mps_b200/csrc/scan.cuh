// Device-wide exclusive prefix sums (reduce -> scan of tile sums -> downsweep) used for
// cell starts, CSR row pointers and unknown numbering.
#pragma once
#include "common.cuh"

namespace lsmps_gpu {

// out[i] = sum_{j<i} in[i] for i in [0, n], out[n] the total. The total must fit in int32:
// otherwise the DFLAG_INDEX bit of *dflag is set (the caller turns it into
// LSMPS_ERR_OVERFLOW). `in` may alias `out` only when InT is int. tmp is grow-only scratch.
template <class InT>
void scan_exclusive(const InT* in, int* out, long long n, cudaStream_t s, DevBuf& tmp, int* dflag);

// Same, with the input given as a predicate: in[i] = pred(i) != 0 via a 0/1 byte array.
// (A byte array input is just scan_exclusive<uint8_t>.)

// Sum of an int array (n entries) into *out (device, int64), deterministic.
void reduce_sum_i32(const int* in, long long n, long long* out, cudaStream_t s);

}  // namespace lsmps_gpu
