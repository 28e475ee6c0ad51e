// egg_sort.h -- device sort, scan and segmented-sum primitives (egg_sort.cu),
// used by the eps search's coding cost.  All run on the given stream and
// take their scratch from the caller (sizes from the *_scratch_bytes calls).
#pragma once

#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>

namespace egg {
namespace prim {

// Stable ascending sort of n 32-bit keys; vals (optional, with vals_out)
// travel with their keys.  keys_out / vals_out must not alias the inputs.
size_t sort_scratch_bytes(int n);
void sort_pairs(const uint32_t* keys, const int* vals, uint32_t* keys_out, int* vals_out, int n, void* scratch,
                cudaStream_t st);

// out[i] = in[0] + ... + in[i]
size_t scan_scratch_bytes(int m);
void inclusive_scan(const int* in, int* out, int m, void* scratch, cudaStream_t st);

// out[s] = sum of v[begin[s] .. begin[s+1]) for s < K, added in a fixed order
void segment_sums(const double* v, const int* begin, int K, double* out, cudaStream_t st);

}  // namespace prim
}  // namespace egg
