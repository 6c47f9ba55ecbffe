// Sample preparation on the device (see prep.cu).
#pragma once

#include <cuda_runtime.h>

#include <vector>

#include "common.h"

namespace fereg {

// factor.rs:38 factorize: dense codes of a column in ascending value order (NaN: 198); returns
// the level count.
u32 prep_factorize(const double* x, size_t n, u32* codes_out);
// factor.rs:255 combine: codes of the interaction of code columns (lexicographic order).
u32 prep_combine(const std::vector<const u32*>& parts, const std::vector<u32>& nl, size_t n, u32* codes_out);

struct DropCounts {
    u64 singletons = 0, separated = 0;
};
// sample.rs:44-72 drop_singletons: cyclic passes over the terms until none drops; with a family
// (1 Poisson, 2 logit) and its outcome y, the `fe` rule drops levels without variation.
DropCounts prep_drop(const std::vector<const u32*>& codes, const std::vector<u32>& g, size_t n, const double* fw,
                     const double* y, int family, bool singletons, uint8_t* alive);
// Exclusive scan of n device u32 values into out (device) on `st`; returns the total (the host
// waits for it).
u32 device_excl_scan(const u32* in, size_t n, u32* out, cudaStream_t st);
// Stable LSD radix sort of n (key, value) pairs in device memory over the low `bits` bits of the
// keys, 8 bits a pass, ping-ponging with the *_alt buffers: on return keys / vals point at
// whichever pair of buffers holds the sorted data.
void device_sort_pairs(u64*& keys, u32*& vals, u64* keys_alt, u32* vals_alt, size_t n, int bits, cudaStream_t st);

// factor.rs:281 restrict: the kept rows' codes renumbered densely in order; returns the level
// count, and the number of kept rows in *kept.
u32 prep_restrict(const u32* codes, u32 g, const uint8_t* alive, size_t n, u32* out, size_t* kept);

}  // namespace fereg
