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

// A batch of instances: device descriptors plus one active list with its
// per-shape virtual-block offsets (egg_batch.cuh).
struct BatchTables {
    const Geom* geoms = nullptr;  // device [instances]
    const Work* works = nullptr;  // device [instances]
    const int* boff = nullptr;    // device [kShapeCount][cap + 1]
    const int* active = nullptr;  // device [cap]
    const int* nact = nullptr;    // device [1]
    int cap = 0;                  // list capacity
    int total[kShapeCount] = {};  // virtual blocks per shape over all instances
    int max_passes = 0;           // radix passes of the instance with the most
    int max_table_k = 0;
    int occ = 8;                  // persistent blocks per SM of a 256-thread kernel
    int update_threads = 128;     // block size of the update kernel: 64, 128 or 256
};

struct Exec {
    const Geom* g = nullptr;           // single instance (host objects)
    const Work* w = nullptr;
    const BatchTables* bt = nullptr;   // batch
    int d = 0;                         // dimensions (kernel template)
    bool batch() const { return bt != nullptr; }
    // single: the shape's block count; batch: a persistent grid
    int blocks(int shape, int threads) const {
        if (!bt) return shape_blocks(shape, *g);
        int per_sm = bt->occ * 256 / threads;
        if (per_sm < 1) per_sm = 1;
        const int cap = 148 * per_sm;
        const int t = bt->total[shape];
        return t < 1 ? 1 : (t < cap ? t : cap);
    }
    BatchArgs args(int shape) const {
        return BatchArgs{bt->geoms, bt->works, bt->boff + (size_t)shape * (bt->cap + 1), bt->active, bt->nact};
    }
    int table_k() const { return bt ? bt->max_table_k : g->table_k; }
    int update_threads() const { return bt ? bt->update_threads : 128; }
};

inline Exec single(const Geom& g, const Work& w) {
    Exec e;
    e.g = &g;
    e.w = &w;
    e.d = g.d;
    return e;
}

inline Exec batched(const BatchTables& bt, int d) {
    Exec e;
    e.bt = &bt;
    e.d = d;
    return e;
}

// grid (egg_grid.cu)
// the grid of the current positions Xn (radix passes: plan_count/plan_pass)
void launch_build(const Exec& ex, cudaStream_t st);
// its two halves: has any point left its cell (copies the positions), and
// the sort and cell tables, whose kernels return at once when none has.
// begin = false: the caller's loop control already cleared the changed word.
void launch_build_check(const Exec& ex, cudaStream_t st, bool begin = true);
void launch_build_sort(const Exec& ex, cudaStream_t st);
void launch_cell_sums(const Exec& ex, cudaStream_t st);
void launch_transpose_in(const Geom& g, const Work& w, const float* x, cudaStream_t st);
void launch_unsort_positions(const Geom& g, const Work& w, const float* src, float* out, cudaStream_t st);
void launch_labels(const Geom& g, const Work& w, int* out, cudaStream_t st);
void launch_unsort_int(const Geom& g, const Work& w, const int* src, int* out, cudaStream_t st);
// union-find labelling (egg_labels.cu): same partition and values as
// launch_labels; a batch writes each instance's labels to its w.labels
void launch_labels_uf(const Geom& g, const Work& w, int* out, cudaStream_t st);
void launch_labels_uf(const Exec& ex, cudaStream_t st);

// update + flag (egg_update.cu); counts (nullable, single instance only)
// receives |N_eps(p)| per sorted point
void launch_update(const Exec& ex, int* counts, cudaStream_t st);
// stencil dilation of the outer cells touched by moved points (incremental update)
void launch_need(const Exec& ex, cudaStream_t st);

// FP64 local order parameter (egg_order.cu, single instance): final_slot < 0 = this iteration
void launch_order_param(const Geom& g, const Work& w, int final_slot, cudaStream_t st);

// extra convergence check (egg_extra.cu)
void launch_extra_check(const Exec& ex, cudaStream_t st, bool gated = false);
// loop graph of one instance: opens the conditional node of the extra check
// when the update left the flag at 1 (stage stamp and run count included)
void launch_gate_extra(const Work& w, cudaGraphConditionalHandle h, cudaStream_t st);
// loop graph of a batch: the same per dimension group (any active instance flagged)
void launch_batch_gate_extra(const Exec& ex, cudaGraphConditionalHandle h, cudaStream_t st);
// ... and its grid sort (any active instance with a point that changed cell;
// *opened counts the openings)
void launch_batch_gate_sort(const Exec& ex, cudaGraphConditionalHandle h, int* opened, cudaStream_t st);

}  // namespace egg
