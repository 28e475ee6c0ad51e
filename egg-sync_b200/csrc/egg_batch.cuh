// egg_batch.cuh -- one launch for many instances.
//
// Every per-iteration kernel is written as a device body taking its block
// index bx and block count gx.  The single-instance kernel calls it with
// (blockIdx.x, gridDim.x); the batched kernel maps blockIdx.x to (instance,
// local block) through a prefix table of per-instance block counts and runs
// the same body on that instance's geometry and workspace, copied to shared
// memory.  Blocks of instances whose loop has finished return at once.
#pragma once

#include "egg_common.cuh"

namespace egg {

// launch shapes: how many blocks a kernel uses for one instance
enum Shape : int {
    kShapeN128 = 0,    // ceil(n / 128)
    kShapeN256,        // ceil(n / 256)
    kShapeN1024,       // ceil(n / 1024)
    kShapeTiles,       // ceil(n / kSortTile)
    kShapeDigits,      // 256
    kShapeOne,         // 1
    kShapeOuter,       // ceil((n_outer + 1) / 256)
    kShapeCapN256,     // min(ceil(n / 256), 148 * 8)
    kShapeCapN128,     // min(ceil(n / 128), 148 * 8)
    kShapeCapOuter,    // min(ceil(n_outer / 256), 148 * 8)
    kShapeFix,         // min(ceil(ceil(n / 32) / 8), 148 * 8)
    kShapeCapN256L,    // min(ceil(n / 256), 148 * 16)
    kShapeCount
};

__host__ __device__ inline int shape_blocks(int shape, const Geom& g) {
    auto cdiv = [](long a, long b) { return (int)((a + b - 1) / b); };
    auto cap = [](int v, int c) { return v < c ? v : c; };
    switch (shape) {
        case kShapeN128: return cdiv(g.n, 128);
        case kShapeN256: return cdiv(g.n, 256);
        case kShapeN1024: return cdiv(g.n, kHeadsBlock);
        case kShapeTiles: return cdiv(g.n, kSortTile);
        case kShapeDigits: return 256;
        case kShapeOne: return 1;
        case kShapeOuter: return cdiv((long)g.n_outer + 1, 256);
        case kShapeCapN256: return cap(cdiv(g.n, 256), 148 * 8);
        case kShapeCapN128: return cap(cdiv(g.n, 128), 148 * 8);
        case kShapeCapOuter: return cap(cdiv(g.n_outer, 256) > 0 ? cdiv(g.n_outer, 256) : 1, 148 * 8);
        case kShapeFix: return cap(cdiv(cdiv(g.n, 32), 8), 148 * 8);
        case kShapeCapN256L: return cap(cdiv(g.n, 256), 148 * 16);
        default: return 1;
    }
}

struct BatchArgs {
    const Geom* geoms;  // [ninst]
    const Work* works;  // [ninst]
    const int* boff;    // [ninst + 1] block offsets of this launch's shape
    int ninst;
};

// Declares `g`, `w`, `bx`, `gx` for the block's instance (shared-memory
// copies) and returns for instances whose loop is done when skip_done.
#define EGG_BATCH_ENTRY(B, skip_done)                                                          \
    __shared__ Geom _bg;                                                                       \
    __shared__ Work _bw;                                                                       \
    __shared__ int _bbx, _bgx, _bskip;                                                         \
    if (threadIdx.x == 0) {                                                                    \
        int lo_ = 0, hi_ = (B).ninst - 1;                                                      \
        while (lo_ < hi_) {                                                                    \
            const int m_ = (lo_ + hi_ + 1) >> 1;                                               \
            if ((B).boff[m_] <= (int)blockIdx.x) lo_ = m_; else hi_ = m_ - 1;                  \
        }                                                                                      \
        _bg = (B).geoms[lo_];                                                                  \
        _bw = (B).works[lo_];                                                                  \
        _bbx = (int)blockIdx.x - (B).boff[lo_];                                                \
        _bgx = (B).boff[lo_ + 1] - (B).boff[lo_];                                              \
        _bskip = (skip_done) && _bw.ctrl[kCtrlDone] != 0;                                      \
    }                                                                                          \
    __syncthreads();                                                                           \
    if (_bskip) return;                                                                        \
    const Geom& g = _bg;                                                                       \
    const Work& w = _bw;                                                                       \
    const int bx = _bbx, gx = _bgx;

}  // namespace egg
