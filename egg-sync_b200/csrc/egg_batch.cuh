// egg_batch.cuh -- one launch for many instances.
//
// Every per-iteration kernel is written as a device body over a block index
// bx of gx blocks.  The single-instance kernel calls it with (blockIdx.x,
// gridDim.x).  The batched kernel is persistent: its blocks stride over the
// virtual blocks of all instances still in the active list (for a launch
// shape s, instance k of the list owns virtual blocks [boff[k], boff[k+1])),
// copy that instance's geometry and workspace descriptor to shared memory and
// run the same body.  The active list and its offset tables are rebuilt on
// the device after every iteration, so the cost of a launch follows the
// instances that still iterate, and one CUDA graph replays the loop of the
// whole batch.
#pragma once

#include "egg_common.cuh"

namespace egg {

constexpr int kScanSmallTiles = 64;  // radix digit scan: one block per instance up to this many tiles
constexpr int kMaxBatch = 1024;      // instances of one batched call

// launch shapes: how many blocks a kernel uses for one instance
enum Shape : int {
    kShapeN128 = 0,    // ceil(n / 128)
    kShapeN256,        // ceil(n / 256)
    kShapeN1024,       // ceil(n / 1024)
    kShapeTiles,       // ceil(n / kSortTile)
    kShapeDigits,      // 1 (few tiles: one thread per digit) or 256 (one block per digit)
    kShapeOne,         // 1
    kShapeOuter,       // ceil((n_outer + 1) / 256)
    kShapeCapN256,     // min(ceil(n / 256), 148 * 8)
    kShapeCapN128,     // min(ceil(n / 128), 148 * 8)
    kShapeCapOuter,    // min(ceil(n_outer / 64), 148 * 8): 8 outer cells per warp
    kShapeFix,         // min(ceil(ceil(n / 32) / 8), 148 * 8)
    kShapeCapN256L,    // min(ceil(n / 256), 148 * 16)
    kShapeN64,         // ceil(n / 64)
    kShapeCount
};

__host__ __device__ inline int sort_tiles(const Geom& g) { return (g.n + kSortTile - 1) / kSortTile; }

__host__ __device__ inline int shape_blocks(int shape, const Geom& g) {
    auto cdiv = [](long a, long b) { return (int)((a + b - 1) / b); };
    auto cap = [](int v, int c) { return v < c ? v : c; };
    switch (shape) {
        case kShapeN128: return cdiv(g.n, 128);
        case kShapeN256: return cdiv(g.n, 256);
        case kShapeN1024: return cdiv(g.n, kHeadsBlock);
        case kShapeTiles: return sort_tiles(g);
        case kShapeDigits: return sort_tiles(g) <= kScanSmallTiles ? 1 : 256;
        case kShapeOne: return 1;
        case kShapeOuter: return cdiv((long)g.n_outer + 1, 256);
        case kShapeCapN256: return cap(cdiv(g.n, 256), 148 * 8);
        case kShapeCapN128: return cap(cdiv(g.n, 128), 148 * 8);
        case kShapeCapOuter: return cap(cdiv(g.n_outer, 64) > 0 ? cdiv(g.n_outer, 64) : 1, 148 * 8);
        case kShapeFix: return cap(cdiv(cdiv(g.n, 32), 8), 148 * 8);
        case kShapeCapN256L: return cap(cdiv(g.n, 256), 148 * 16);
        case kShapeN64: return cdiv(g.n, 64);
        default: return 1;
    }
}

// Radix passes of an instance, least significant first: the sub-cell key,
// then g_{d-1}, ..., g_od, then g_0, ..., g_{od-1}; two 8-bit passes per
// dimension when there are more than 256 cells per dimension.  The last
// pass must write perm (selector 0); pass p reads what pass p-1 wrote.
__host__ __device__ inline int plan_count(const Geom& g) { return 1 + g.d * (g.width > 256 ? 2 : 1); }

__host__ __device__ inline void plan_pass(const Geom& g, int p, int& dim, int& shift) {
    if (p == 0) {
        dim = -1;
        shift = 0;
        return;
    }
    const int per = g.width > 256 ? 2 : 1;
    const int k = (p - 1) / per;
    const int nin = g.d - g.od;
    dim = k < nin ? g.d - 1 - k : k - nin;
    shift = 8 * ((p - 1) % per);
}

__host__ __device__ inline int plan_out_sel(int count, int p) { return ((count - p) & 1) ? 0 : 1; }

struct BatchArgs {
    const Geom* geoms;   // [instances]
    const Work* works;   // [instances]
    const int* boff;     // [list + 1] virtual-block offsets of this launch's shape
    const int* active;   // [list] instance ids
    const int* nact;     // list length
};

// Runs body(g, w, bx, gx) for every virtual block of the listed instances.
// Virtual blocks are dealt out with stride gridDim.x, which spreads the
// dense regions of every instance over all SMs.  Each block copies the
// offset table to shared memory once and the descriptors of an instance only
// when its next virtual block belongs to another instance.
template <typename F>
__device__ __forceinline__ void batch_for(const BatchArgs& B, F&& body) {
    static_assert(sizeof(Geom) % 4 == 0 && sizeof(Work) % 4 == 0, "descriptor copy by words");
    __shared__ Geom s_g;
    __shared__ Work s_w;
    __shared__ int s_boff[kMaxBatch + 1];
    __shared__ int s_act[kMaxBatch];
    __shared__ int s_info[4];  // list entry, its first virtual block, its block count, entry loaded
    // the offset table and the list in one round of loads after the list length
    const int na = *B.nact;
    for (int t = threadIdx.x; t <= na; t += blockDim.x) {
        s_boff[t] = B.boff[t];
        if (t < na) s_act[t] = B.active[t];
    }
    if (threadIdx.x == 0) s_info[3] = -1;
    __syncthreads();
    const int tot = s_boff[na];
    for (int vb = blockIdx.x; vb < tot; vb += gridDim.x) {
        if (threadIdx.x == 0) {
            int lo = 0, hi = na - 1;
            while (lo < hi) {
                const int m = (lo + hi + 1) >> 1;
                if (s_boff[m] <= vb) lo = m; else hi = m - 1;
            }
            s_info[0] = lo;
            s_info[1] = s_boff[lo];
            s_info[2] = s_boff[lo + 1] - s_boff[lo];
        }
        __syncthreads();
        if (s_info[0] != s_info[3]) {
            const int inst = s_act[s_info[0]];
            const int* sg = reinterpret_cast<const int*>(B.geoms + inst);
            const int* sw = reinterpret_cast<const int*>(B.works + inst);
            int* dg = reinterpret_cast<int*>(&s_g);
            int* dw = reinterpret_cast<int*>(&s_w);
            for (int t = threadIdx.x; t < (int)(sizeof(Geom) / 4); t += blockDim.x) dg[t] = sg[t];
            for (int t = threadIdx.x; t < (int)(sizeof(Work) / 4); t += blockDim.x) dw[t] = sw[t];
            __syncthreads();
            if (threadIdx.x == 0) s_info[3] = s_info[0];
        }
        body(static_cast<const Geom&>(s_g), static_cast<const Work&>(s_w), vb - s_info[1], s_info[2]);
        __syncthreads();
    }
}

}  // namespace egg
