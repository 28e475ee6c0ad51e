// egg_kernels.h -- host-side launchers of the EGG-SynC kernels (internal).
#pragma once

#include <cuda_runtime.h>

#include "egg_common.cuh"

namespace egg {

// LSD radix passes over the cell digits: pass p sorts on
// (cell_dim(x[dim[p]]) >> shift[p]) & 255, least significant pass first;
// dim[p] < 0 is the within-cell sub-cell key.
struct SortPlan {
    int count = 0;
    int dim[2 * kMaxDims + 1];
    int shift[2 * kMaxDims + 1];
};

// grid (egg_grid.cu)
void launch_sort(const Geom& g, const Work& w, const SortPlan& plan, cudaStream_t st);
void launch_build(const Geom& g, const Work& w, const SortPlan& plan, cudaStream_t st);
void launch_cell_sums(const Geom& g, const Work& w, cudaStream_t st);
void launch_transpose_in(const Geom& g, const Work& w, const float* x, cudaStream_t st);
void launch_unsort_positions(const Geom& g, const Work& w, const float* src, float* out, cudaStream_t st);
void launch_labels(const Geom& g, const Work& w, int* out, cudaStream_t st);
// union-find labelling (egg_labels.cu): same partition and values as launch_labels
void launch_labels_uf(const Geom& g, const Work& w, int* out, cudaStream_t st);
void launch_unsort_int(const Geom& g, const Work& w, const int* src, int* out, cudaStream_t st);

// update + flag (egg_update.cu); counts (nullable) receives |N_eps(p)| per
// sorted point
void launch_update(const Geom& g, const Work& w, int* counts, cudaStream_t st);
// stencil dilation of the outer cells touched by moved points (incremental update)
void launch_need(const Geom& g, const Work& w, cudaStream_t st);

// FP64 local order parameter (egg_order.cu): final_slot < 0 = this iteration
void launch_order_param(const Geom& g, const Work& w, int final_slot, cudaStream_t st);

// extra convergence check (egg_extra.cu)
void launch_extra_check(const Geom& g, const Work& w, cudaStream_t st);

// loop control (egg_host.cu)
void launch_iter_begin(const Geom& g, const Work& w, cudaStream_t st);

}  // namespace egg
