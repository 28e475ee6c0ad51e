// egg_labels.cu -- cluster extraction by GPU union-find.
//
// The reference labels a point with the compacted index of its final cell
// when that cell holds more than one point, else -1
// (src/algorithms/EGG_SynC.cu:1205-1227, 1504-1522).  Here the collapsed
// points are joined into components by a lock-free union-find: every point
// is joined to the first cell-sorted point of its final cell (a star per
// cell: one hook per point, where a chain of consecutive points made finds
// walk paths as long as the cluster); a link hooks the larger root onto the
// smaller one with atomicCAS, so every component's root is its smallest
// sorted index, i.e. the first point of the cell, whatever the order of the
// atomics.  Component sizes are counted with one atomic per warp and root.  After full path compression a
// point's label is the cell index of its root when the component holds more
// than one point: the reference's partition and label values, deterministic.
#include "egg_common.cuh"
#include "egg_kernels.h"

namespace egg {

namespace {

__device__ __forceinline__ int uf_find(int* parent, int x) {
    int p = parent[x];
    while (p != x) {
        const int gp = parent[p];
        if (gp != p) parent[x] = gp;  // path halving; any order of these writes is safe
        x = p;
        p = gp;
    }
    return x;
}

__device__ __forceinline__ void uf_union(int* parent, int a, int b) {
    for (;;) {
        a = uf_find(parent, a);
        b = uf_find(parent, b);
        if (a == b) return;
        if (a < b) {
            const int t = a;
            a = b;
            b = t;
        }
        // hook root a (larger) below root b; retry if a stopped being a root
        if (atomicCAS(parent + a, a, b) == a) return;
    }
}

}  // namespace

__device__ __forceinline__ void uf_init_body(const Geom& g, const Work& w, int bx, int gx) {
    for (int i = bx * blockDim.x + threadIdx.x; i < g.n; i += gx * blockDim.x) {
        w.uf_parent[i] = i;
        w.uf_size[i] = 0;
    }
}

// edge (first point of i's final cell, i)
__device__ __forceinline__ void uf_link_body(const Geom& g, const Work& w, int bx, int gx) {
    for (int i = bx * blockDim.x + threadIdx.x; i < g.n; i += gx * blockDim.x) {
        const int f = w.cell_start[w.cell_of[i]];
        if (f != i) uf_union(w.uf_parent, f, i);
    }
}

__device__ __forceinline__ void uf_compress_body(const Geom& g, const Work& w, int bx, int gx) {
    for (int i = bx * blockDim.x + threadIdx.x; i < g.n; i += gx * blockDim.x) {
        const int r = uf_find(w.uf_parent, i);
        // lanes with the same root add once (sorted points share roots)
        const unsigned peers = __match_any_sync(__activemask(), r);
        if ((threadIdx.x & 31) == __ffs(peers) - 1) atomicAdd(w.uf_size + r, __popc(peers));
    }
}

__device__ __forceinline__ void uf_labels_body(const Geom& g, const Work& w, int* __restrict__ out, int bx, int gx) {
    const int* parent = w.uf_parent;
    for (int i = bx * blockDim.x + threadIdx.x; i < g.n; i += gx * blockDim.x) {
        // parent[i] may still point to a non-root after compress (halving),
        // so follow it to the root without writing
        int r = parent[i];
        while (parent[r] != r) r = parent[r];
        const bool multi = w.uf_size[r] > 1;
        out[w.orig[i]] = multi ? w.cell_of[r] : -1;
        if (multi && r == i) atomicAdd(w.ctrl + kCtrlClusters, 1);
    }
}

__global__ void k_uf_init(Geom g, Work w) { uf_init_body(g, w, blockIdx.x, gridDim.x); }
__global__ void k_uf_link(Geom g, Work w) { uf_link_body(g, w, blockIdx.x, gridDim.x); }
__global__ void k_uf_compress(Geom g, Work w) { uf_compress_body(g, w, blockIdx.x, gridDim.x); }
__global__ void k_uf_labels(Geom g, Work w, int* out) { uf_labels_body(g, w, out, blockIdx.x, gridDim.x); }

__global__ void kb_uf_init(BatchArgs B) {
    batch_for(B, [&](const Geom& g, const Work& w, int bx, int gx) { uf_init_body(g, w, bx, gx); });
}
__global__ void kb_uf_link(BatchArgs B) {
    batch_for(B, [&](const Geom& g, const Work& w, int bx, int gx) { uf_link_body(g, w, bx, gx); });
}
__global__ void kb_uf_compress(BatchArgs B) {
    batch_for(B, [&](const Geom& g, const Work& w, int bx, int gx) { uf_compress_body(g, w, bx, gx); });
}
__global__ void kb_uf_labels(BatchArgs B) {
    batch_for(B, [&](const Geom& g, const Work& w, int bx, int gx) { uf_labels_body(g, w, w.labels, bx, gx); });
}

void launch_labels_uf(const Geom& g, const Work& w, int* out, cudaStream_t st) {
    const int blocks = shape_blocks(kShapeCapN256L, g);
    k_uf_init<<<blocks, 256, 0, st>>>(g, w);
    k_uf_link<<<blocks, 256, 0, st>>>(g, w);
    k_uf_compress<<<blocks, 256, 0, st>>>(g, w);
    k_uf_labels<<<blocks, 256, 0, st>>>(g, w, out);
}

void launch_labels_uf(const Exec& ex, cudaStream_t st) {
    const int blocks = ex.blocks(kShapeCapN256L, 256);
    const BatchArgs B = ex.args(kShapeCapN256L);
    kb_uf_init<<<blocks, 256, 0, st>>>(B);
    kb_uf_link<<<blocks, 256, 0, st>>>(B);
    kb_uf_compress<<<blocks, 256, 0, st>>>(B);
    kb_uf_labels<<<blocks, 256, 0, st>>>(B);
}

}  // namespace egg
