// egg_common.cuh -- shared definitions for the EGG-SynC sm_100a kernels.
//
// Geometry, workspace layout and the discrete decision primitives (cell ids,
// border rule, box distance, point distance) used by every kernel.  The
// decision primitives are written with explicit round-to-nearest intrinsics
// so that the compiler cannot contract them; the CPU oracle uses the same
// operation order, which makes every discrete decision (cell membership,
// full/partial/none classification, eps tests, the convergence flag)
// bit-identical between the two.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace egg {

constexpr int kMaxDims = 64;        // generic kernels support d <= kMaxDims
constexpr int kMaxTable = 64;       // sin/cos table half-width: |k| <= kMaxTable
constexpr int kSortTile = 2048;     // points per radix-sort tile (2048: 489 blocks at 1M points, 3.3 per SM)
constexpr int kSortThreads = 256;
constexpr int kHeadsBlock = 1024;   // points per block in the cell-boundary scan

// Status word bits set by kernels (read by the host after the run).
enum : int {
    kErrNonFinite = 1,       // input holds NaN/Inf
    kErrTable = 2,           // a cell offset fell outside the sin/cos table
    kErrStencil = 4,
};

// The update kernel's point-by-point walks read a candidate point's
// coordinates and its sin / 1 - cos offsets as whole 16-byte records when
// d <= kPackDims: pack_w(d) float4 of coordinates, pack_s(d) float4 of the
// 2d offsets, zero-padded.
constexpr int kPackDims = 8;
__host__ __device__ constexpr int pack_w(int d) { return (d + 3) / 4; }
__host__ __device__ constexpr int pack_s(int d) { return (2 * d + 3) / 4; }

// Per-instance geometry, exactly as the reference computes it
// (src/algorithms/EGG_SynC.cu:1249-1260, 1430, 563, 779, 1045).
struct Geom {
    int n;             // points
    int d;             // dimensions
    int ns;            // SoA stride (n rounded up to 32)
    int od;            // outer grid dimensions
    int width;         // cells per dimension
    int n_outer;       // width^od
    int r;             // ceil(eps / side)                 (float)
    int r_extra;       // ceil(eps_extra / side)           (float)
    int r_half;        // ceil((eps / 2.) / side)          (double)
    int table_k;       // sin/cos table covers k in [-table_k, table_k]
    float side;        // inner = outer cell side
    float eps;
    float eps_extra;
    float t_eps;       // largest v with sqrtf(v) <= eps
    float t_half;      // ... <= eps/2
    float t_extra;     // ... <= eps_extra
    int sub_dims;      // dimensions in the within-cell (sub-cell) sort key
    int sub_bits;      // bits per dimension of the sub-cell key (sub_dims*sub_bits <= 8)
    int stop_rule;     // 0 = the reference's convergence flag, 1 = order parameter >= lam
    int order_mode;    // 0 = no order parameter, 1 = final only, 2 = every iteration
    float lam;         // order-parameter threshold of stop rule 1
    int zblk;          // incremental update: cells of dimension od per block (1 block when od == d)
    int nzb;           // ... number of blocks (<= 64: one bit each)
    int wpow[32];      // width^l for l < od
};

// Device workspace.  All arrays are SoA with stride g.ns where per-point or
// per-cell with a dimension index.
struct Work {
    // points, in the current cell-sorted order
    float* X;          // [d][ns] positions (current grid)
    float* Xn;         // [d][ns] positions after the update (same order as X)
    float* sd;         // [d][ns] sin(delta), delta = x - cell corner (d > kPackDims)
    float* md;         // [d][ns] 1 - cos(delta) (= 2 sin^2(delta/2))  (d > kPackDims)
    float4* xp;        // [ns][pack_w(d)] positions packed per point (d <= kPackDims)
    float4* smp;       // [ns][pack_s(d)] sin(delta) then 1 - cos(delta), packed per point (d <= kPackDims)
    float* qlo;        // [d][ns] eps/2-ball extremes (extra check)
    float* qhi;        // [d][ns]
    float* ulo;        // [d][ns] per cell: union of its points' eps/2-ball extremes
    float* uhi;        // [d][ns]
    int* orig;         // [ns]   original index of sorted point i
    int* orig_tmp;     // [ns]
    int* perm;         // [ns]   radix sort output: new position -> previous position
    int* perm_tmp;     // [ns]
    unsigned* skey[2]; // [ns] each: whole 32-bit sort keys of the one-key grid sort (d <= 3 and at most
                       // 256 cells per dimension; nullptr otherwise: the per-dimension passes)
    int* cell_of;      // [ns]   cell index of sorted point i
    // cells (index < M, M only known on the device)
    int* cell_start;   // [ns+1]
    int* cell_dims;    // [d][ns]
    unsigned long long* cell_key;  // [ns] the cell's dims packed 16 bits each (d <= 4): one load per box test
    int* cell_outer;   // [ns]
    float* css;        // [d][ns] sum sin(delta) per cell
    float* csm;        // [d][ns] sum (1 - cos(delta)) per cell
    float* cbmin;      // [d][ns] tight bounding box of the cell's points
    float* cbmax;      // [d][ns]
    int* outer_begin;  // [n_outer + 1]
    unsigned long long* colmask;  // [n_outer] per outer cell: the blocks of zblk cells of dimension od holding a cell
    // scratch for scans / sorts
    int* hist;         // [256 * tiles]
    int* digit_total;  // [256]
    int* block_sums;   // [blocks]
    double* wpart;     // [(2d values + 2d bbox) * 2 * warps] warp partials for spanning cells
    float* gpart;      // the same records in FP32: the 32-point groups of spanning cells
    // stencils (host-built tables)
    int* st_delta;     // [3][st_cap] linear outer-id offset
    signed char* st_off;  // [3][st_cap * od] per-dimension offsets
    int st_count[3];   // entries per stencil: 0 = update (r), 1 = annulus (r_extra), 2 = ball (r_half)
    int st_cap;
    float* table;      // [3][2*table_k+1]: sin(ks), cos(ks), 1-cos(ks)
    // control words
    int* ctrl;         // [16]: see kCtrl* below
    unsigned long long* stamps;  // [max_iter+1] globaltimer at iteration start
    int* labels;       // [ns] output labels (original order)
    int* iter_flags;   // [max_iter] flag after each iteration
    unsigned long long* ustats;  // [kUStats] interaction counters of the update kernel (stats build)
    // incremental update, per outer cell a bit mask over blocks of cells of
    // dimension od: the blocks holding a moved point (old or new position) in
    // the last update, ping-pong by iteration parity; their dilation over
    // the update's candidate region; the last violation bit of every point
    unsigned long long* dirty[2];  // [n_outer]
    unsigned long long* need;      // [n_outer]
    unsigned char* viol_orig;  // [ns] by original index
    unsigned char* warp_moved; // [ns/32 + 1] the warp's points changed in the last update (grid check)
    unsigned* warp_viol;       // [ns/32 + 1] the warp's violation bits (lane mask) as of its last update
    int* span_list;            // [ns/32 + 1] cells whose points span 2-3 warps
    int* big_list;             // [ns/128 + 1] cells whose points span 4 or more warps
    int* span_mark;            // [ns] per spanning cell: the last iteration that re-summed one of its warps
    // local order parameter (FP64): per-block partials, per-iteration [lo, hi]
    double* rpart;             // [2 * blocks]
    double* rvals;             // [2 * (max_iter + 2)]; slot max_iter + 1 = final value
    // union-find labelling
    int* uf_parent;            // [ns]
    int* uf_size;              // [ns]
    // batched runs: this instance's input (device, row-major n x d)
    const float* src;
};

enum : int {
    kCtrlM = 0,        // number of non-empty cells
    kCtrlFlag = 1,     // 1 = converged so far in this iteration
    kCtrlIter = 2,     // iterations done
    kCtrlDone = 3,     // loop finished
    kCtrlStatus = 4,   // kErr* bits
    kCtrlMaxIter = 5,
    kCtrlExtraRuns = 6,   // number of extra checks run
    kCtrlPairs = 7,       // annulus pairs examined in the last extra check
    kCtrlClusters = 8,    // final cells holding more than one point
    kCtrlChanged = 9,     // some point left its cell since the last grid build
    kCtrlGridValid = 10,  // the grid arrays describe the current sorted order
    kCtrlBuilds = 11,     // grid builds actually performed (statistics)
    kCtrlForce = 12,      // recompute every point (first iteration of a run)
    kCtrlComputed = 13,   // points recomputed by the update (statistics)
    kCtrlFullUpdate = 14, // recompute every point in every iteration
    kCtrlSpanCount = 15,  // cells over 2-3 warps listed in span_list by the cell-sums kernel
    kCtrlBigCount = 16,   // cells over 4 or more warps listed in big_list
    kCtrlLamReached = 17, // the order parameter's lower bound reached lambda this iteration
    kCtrlWords = 32,      // size of the control-word array
};

// Interaction counters of the update kernel, summed over a run.  Collected
// only in the stats build (EGG_UPDATE_STATS, libeggsync_stats.so); they give
// the kernel's algorithmic work: cells examined and how each was decided,
// point pairs tested.
enum : int {
    kUsPoints = 0,     // point updates computed
    kUsCells,          // candidate cells examined (box test)
    kUsSmallPass,      // ... passing the reference's small box test
    kUsFull,           // ... fully covered (box), aggregated
    kUsTightIn,        // ... all points within eps by their tight box, aggregated
    kUsTightOut,       // ... no point within eps by their tight box, skipped
    kUsGroupsIn,       // 32-point groups of spanning cells aggregated
    kUsGroupsOut,      // 32-point groups skipped
    kUsPairs,          // point-pair distance tests
    kUsPairsIn,        // ... within eps
    kUsLaneWarps,      // warps whose lanes span several outer cells
    kUsHalfCount,      // border points that needed the half count
    kUsNeighbors,      // sum of |N(p)|
    kUsCyclesShared,   // SM cycles of the candidate walk, warps whose lanes share one outer cell
    kUsCyclesLane,     // SM cycles of the candidate walk, warps whose lanes span several outer cells
    kUsWarpVisits,     // candidate cells visited by lockstep warps (once per warp)
    kUsCyclesVisits,   // SM cycles of those visits (box tests, aggregates, walks): the rest of
                       // cycles_shared is the stencil enumeration
    kUsWalkSteps,      // warp steps of the point walks (one per loop iteration a warp executes)
    kUStats = 20
};

// ------------------------------------------------------------------------
// decision primitives (identical operation order on the CPU oracle)
// ------------------------------------------------------------------------
__device__ __forceinline__ int cell_dim(float x, const Geom& g) {
    int t = (int)__fdiv_rn(x, g.side);
    if (t == g.width) t--;
    t = t < 0 ? 0 : t;
    t = t > g.width - 1 ? g.width - 1 : t;
    return t;
}

// reference border rule, EGG_SynC.cu:590-596 (the +-1e-5 probes are double).
// A point whose cell coordinate x/side is farther than 1e-5/side from every
// integer, with margins for the float rounding of x/side, gives
// idm == id == idp; only points near a face take the exact double path.
__device__ __forceinline__ bool on_border_dim(float x, float side) {
    const float q = __fdiv_rn(x, side);
    const int id = (int)q;
    const float f = q - floorf(q);
    const float a = 1.001e-5f / side + 2.5e-7f * fabsf(q) + 1e-6f;
    if (q >= 0.0f && f > a && f < 1.0f - a) return false;
    int idm = (int)__ddiv_rn((double)x - 0.00001, (double)side);
    int idp = (int)__ddiv_rn((double)x + 0.00001, (double)side);
    return (id != idm) || (id != idp);
}

// reference box distance terms for one dimension, EGG_SynC.cu:613-630.  The
// face offsets are one fused multiply-add each: the reference's
// `dim_id * side` followed by `-= x` is contracted by nvcc, and only this
// rounding reproduces the reference's own results for points lying exactly
// on cell faces.
__device__ __forceinline__ void box_terms(float x, int cd, float side, float& sm, float& lg) {
    float left = __fmaf_rn((float)cd, side, -x);
    float right = __fmaf_rn((float)(cd + 1), side, -x);
    left = __fmul_rn(left, left);
    right = __fmul_rn(right, right);
    if (left < right) {
        sm = __fadd_rn(sm, left);
        lg = __fadd_rn(lg, right);
    } else {
        sm = __fadd_rn(sm, right);
        lg = __fadd_rn(lg, left);
    }
}

__device__ __forceinline__ float dist_step(float a, float b, float acc) {
    float diff = __fsub_rn(a, b);
    return __fmaf_rn(diff, diff, acc);
}

// largest of |lo - x|, |hi - x| (tight bounding box, farthest face)
__device__ __forceinline__ float far_gap(float x, float lo, float hi) {
    float a = fabsf(__fsub_rn(lo, x));
    float b = fabsf(__fsub_rn(hi, x));
    return a > b ? a : b;
}

// distance from x to [lo, hi] in one dimension (0 inside)
__device__ __forceinline__ float near_gap(float x, float lo, float hi) {
    if (x < lo) return __fsub_rn(lo, x);
    if (x > hi) return __fsub_rn(x, hi);
    return 0.0f;
}

// Squared distances from x to the nearest and to the farthest point of the
// tight bounding box [lo, hi] of a cell's points, accumulated with the same
// fused operation order as dist_step.  Every float step is monotone, so for
// each point q of the cell near2 <= dist2(x, q) <= far2 holds exactly as the
// kernels compute dist2: near2 > T proves no point passes "dist2 <= T", and
// far2 <= T proves all of them do.
__device__ __forceinline__ void tight_box_dist2(const float* x, const float* __restrict__ lo,
                                                const float* __restrict__ hi, size_t stride, int d, float& near2,
                                                float& far2) {
    float a2 = 0.f, b2 = 0.f;
    for (int l = 0; l < d; l++) {
        const float L = __ldg(lo + (size_t)l * stride), H = __ldg(hi + (size_t)l * stride);
        const float a = near_gap(x[l], L, H), b = far_gap(x[l], L, H);
        a2 = __fmaf_rn(a, a, a2);
        b2 = __fmaf_rn(b, b, b2);
    }
    near2 = a2;
    far2 = b2;
}

// index of a warp-partial record: ((field * d + l) * 2 + rec) * warps + warp,
// field in {sum sin, sum 1-cos, min, max}; rec 0 = the segment holding the
// warp's lane 0, rec 1 = the segment holding lane 31
__device__ __forceinline__ size_t wp_idx_f(int field, int l, int d, int rec, int nw, int warp) {
    return ((size_t)(field * d + l) * 2 + rec) * nw + warp;
}

__device__ __forceinline__ unsigned long long globaltimer() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// first index in [b, e) whose key >= v (keys non-decreasing)
__device__ __forceinline__ int lower_bound_i(const int* __restrict__ keys, int b, int e, int v) {
    while (b < e) {
        int m = (b + e) >> 1;
        if (__ldg(keys + m) < v) b = m + 1; else e = m;
    }
    return b;
}

}  // namespace egg
