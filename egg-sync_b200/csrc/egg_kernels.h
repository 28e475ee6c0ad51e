// egg_kernels.h -- host-side launchers of the EGG-SynC kernels (internal).
//
// Every launcher takes an Exec: either one instance (its geometry and
// workspace, passed to the kernels by value) or a batch of instances (device
// arrays of geometries and workspaces plus per-shape block-offset tables; one
// launch covers every instance, see egg_batch.cuh).
#pragma once

#include <cuda_runtime.h>

#include "egg_batch.cuh"
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

struct BatchTables {
    const Geom* geoms = nullptr;  // device [ninst]
    const Work* works = nullptr;  // device [ninst]
    const int* boff = nullptr;    // device [kShapeCount][ninst + 1]
    int total[kShapeCount] = {};  // blocks per shape over the batch
    int ninst = 0;
    int max_table_k = 0;
};

struct Exec {
    const Geom* g = nullptr;           // single instance (host objects)
    const Work* w = nullptr;
    const BatchTables* bt = nullptr;   // batch
    int skip_done = 1;                 // batch: blocks of finished instances return at once
    int d = 0;                         // dimensions (kernel template)
    bool batch() const { return bt != nullptr; }
    int blocks(int shape) const { return bt ? bt->total[shape] : shape_blocks(shape, *g); }
    BatchArgs args(int shape) const {
        return BatchArgs{bt->geoms, bt->works, bt->boff + (size_t)shape * (bt->ninst + 1), bt->ninst};
    }
    int table_k() const { return bt ? bt->max_table_k : g->table_k; }
};

inline Exec single(const Geom& g, const Work& w) {
    Exec e;
    e.g = &g;
    e.w = &w;
    e.d = g.d;
    return e;
}

// grid (egg_grid.cu)
void launch_build(const Exec& ex, const SortPlan& plan, cudaStream_t st);
void launch_cell_sums(const Exec& ex, cudaStream_t st);
void launch_transpose_in(const Geom& g, const Work& w, const float* x, cudaStream_t st);
void launch_unsort_positions(const Geom& g, const Work& w, const float* src, float* out, cudaStream_t st);
void launch_labels(const Geom& g, const Work& w, int* out, cudaStream_t st);
void launch_unsort_int(const Geom& g, const Work& w, const int* src, int* out, cudaStream_t st);
// union-find labelling (egg_labels.cu): same partition and values as launch_labels
void launch_labels_uf(const Geom& g, const Work& w, int* out, cudaStream_t st);

// update + flag (egg_update.cu); counts (nullable, single instance only)
// receives |N_eps(p)| per sorted point
void launch_update(const Exec& ex, int* counts, cudaStream_t st);
// stencil dilation of the outer cells touched by moved points (incremental update)
void launch_need(const Exec& ex, cudaStream_t st);

// FP64 local order parameter (egg_order.cu, single instance): final_slot < 0 = this iteration
void launch_order_param(const Geom& g, const Work& w, int final_slot, cudaStream_t st);

// extra convergence check (egg_extra.cu)
void launch_extra_check(const Exec& ex, cudaStream_t st);

}  // namespace egg
