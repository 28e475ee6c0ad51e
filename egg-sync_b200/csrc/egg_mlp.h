// egg_mlp.h -- learned warm start (egg_mlp.cu), internal declarations.
#pragma once

#include <cuda_runtime.h>

#include <cstddef>

#include "eggsync.h"

namespace egg {
namespace mlp {

constexpr int kHidden = 128;      // width of both hidden layers
constexpr int kMaxWarmDims = 3;   // 3^d neighbour cells in the features

// features per point: the offset in its coarse cell (d values), then per
// neighbour cell log1p(count)/8, centroid offset (d) and spread (d)
__host__ __device__ inline int feat_dim(int d) {
    int c = 1;
    for (int l = 0; l < d; l++) c *= 3;
    return d + c * (1 + 2 * d);
}
// feature row width, padded to the tensor-core k step
__host__ __device__ inline int feat_pad(int d) { return (feat_dim(d) + 15) & ~15; }

// device buffers of the warm start, grown on demand
struct Buffers {
    void* grid = nullptr;
    size_t grid_cap = 0;
    void* feats = nullptr;
    size_t feats_cap = 0;
    void* w = nullptr;
    size_t w_cap = 0;
    float* delta = nullptr;
    size_t delta_cap = 0;
};

// x <- clamp(x + eps * MLP(features(x)), 0, 1) on the SoA positions X
// (stride ns) of the loop
void warm_start(const egg_mlp& m, float* X, size_t ns, int n, int d, float eps, Buffers& B, cudaStream_t st);
void release(Buffers& B);
void release_all();

}  // namespace mlp
}  // namespace egg
