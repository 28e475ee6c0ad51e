// egg_grid.cu -- double-grid spatial index for EGG-SynC on sm_100a.
//
// Replaces build_the_grid + kernel_inner_grid_stats of the reference
// (src/algorithms/EGG_SynC.cu:78-341, 344-366) and its recursive
// Brent-Kung scan (src/utils/GPU_utils.cu:12-238).
//
// The reference keeps a dense outer grid over the first `od` dimensions and,
// inside each outer cell, a list of inner cells found by a linear search.
// Here the same structure is obtained by one stable LSD radix sort of the
// points on their cell tuple, ordered (outer id, g_od, ..., g_{d-1}), so:
//   * every inner cell is a contiguous run of sorted points,
//   * the inner cells of one outer cell are contiguous and sorted by g_od
//     (the update kernel binary-searches that dimension),
//   * outer cell o owns cells [outer_begin[o], outer_begin[o+1]).
// The sort never materialises keys: each pass recomputes one dimension's
// cell digit from the positions through the current permutation.  All
// passes are stable and run in a fixed order, so the whole index (and the
// cell sums below) is bit-reproducible from run to run.
//
// Every kernel is a device body over its block index (bx, gx) with a
// single-instance wrapper and a batched wrapper (egg_batch.cuh).
#include "egg_common.cuh"
#include "egg_kernels.h"

namespace egg {

namespace {

__device__ __forceinline__ unsigned lanemask_lt() {
    unsigned m;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}

// block-wide exclusive scan of one int per thread (blockDim.x <= 1024)
__device__ int block_exclusive_scan(int v, int* total) {
    __shared__ int warp_sums[33];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const int nw = (blockDim.x + 31) >> 5;
    int incl = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        int t = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += t;
    }
    if (lane == 31) warp_sums[wid] = incl;
    __syncthreads();
    if (wid == 0) {
        int s = lane < nw ? warp_sums[lane] : 0;
        int si = s;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            int t = __shfl_up_sync(0xffffffffu, si, o);
            if (lane >= o) si += t;
        }
        if (lane < nw) warp_sums[lane] = si - s;
        if (lane == 31) warp_sums[32] = si;  // lanes >= nw add 0: lane 31 holds the total
    }
    __syncthreads();
    int excl = incl - v + warp_sums[wid];
    if (total) *total = warp_sums[32];
    __syncthreads();
    return excl;
}

// Sort digit of point j.  dim >= 0: bits [shift, shift+8) of the point's cell
// index in that dimension.  dim < 0: the sub-cell key, a Morton interleave of
// the top sub_bits bits of the point's offset inside its cell in the first
// sub_dims dimensions; sorted first (least significant), it orders the points
// of every cell along a space-filling curve, so consecutive runs of a cell's
// points (its 32-point groups) are spatially compact.
__device__ __forceinline__ int digit_of(const Geom& g, const float* __restrict__ Xs, int j, int dim, int shift) {
    if (dim >= 0) {
        float x = __ldg(Xs + (size_t)dim * g.ns + j);
        return (cell_dim(x, g) >> shift) & 255;
    }
    const int b = g.sub_bits;
    const float scale = (float)(1 << b) / g.side;
    int t[8];
    for (int l = 0; l < g.sub_dims; l++) {
        const float x = __ldg(Xs + (size_t)l * g.ns + j);
        const float off = x - __fmul_rn((float)cell_dim(x, g), g.side);
        int v = (int)(off * scale);
        t[l] = v < 0 ? 0 : (v > (1 << b) - 1 ? (1 << b) - 1 : v);
    }
    int dig = 0;
    for (int k = b - 1; k >= 0; k--)
        for (int l = 0; l < g.sub_dims; l++) dig = (dig << 1) | ((t[l] >> k) & 1);
    return dig;
}

// permutation buffer of a sort pass: 0 = perm, 1 = perm_tmp
__device__ __forceinline__ int* perm_buf(const Work& w, int sel) { return sel ? w.perm_tmp : w.perm; }

struct TwoSum {
    float hi, lo;
};

__device__ __forceinline__ TwoSum ts_add(TwoSum a, TwoSum b) {
    float s = __fadd_rn(a.hi, b.hi);
    float bb = __fsub_rn(s, a.hi);
    float err = __fadd_rn(__fsub_rn(a.hi, __fsub_rn(s, bb)), __fsub_rn(b.hi, bb));
    return {s, __fadd_rn(__fadd_rn(a.lo, b.lo), err)};
}

__device__ __forceinline__ size_t wp_idx(int field, int l, int d, int rec, int nw, int warp) {
    return wp_idx_f(field, l, d, rec, nw, warp);
}

}  // namespace

#define EGG_SKIP_IF_UNCHANGED(ctrl) \
    if ((ctrl)[kCtrlChanged] == 0) return;

// ---------------------------------------------------------------------------
// has any point left its cell?  A stable sort of unchanged keys is the
// identity, so when no point changed cell the previous grid (order, cells,
// outer ranges) is exactly the grid a rebuild would produce and every build
// kernel below returns at once.  Also copies the positions into X (with a
// valid grid only for the warps the last update marked as moved: the
// others hold Xn == X already).
// ---------------------------------------------------------------------------
template <int D>
__device__ __forceinline__ void check_cells_body(const Geom& g, const Work& w, int bx, int gx) {
    const int d = D > 0 ? D : g.d;
    const bool valid = w.ctrl[kCtrlGridValid] != 0;
    bool changed = false;
    // d <= 4: the cell's coordinates packed 16 bits each, one load per point
    constexpr bool kKeyed = D >= 1 && D <= 4;
    const bool keyed = kKeyed && w.cell_key != nullptr;
    for (int i = bx * blockDim.x + threadIdx.x; i < g.n; i += gx * blockDim.x) {
        // with a valid grid, only the warps whose points the last update
        // moved (it marks them) can differ from X: the others are skipped
        // (blockDim is a multiple of 32, so the test is warp-uniform)
        if (valid && w.warp_moved && w.warp_moved[i >> 5] == 0) continue;
        const int c = valid ? w.cell_of[i] : 0;
        bool moved = false;
        unsigned long long key = 0;
        for (int l = 0; l < d; l++) {
            const float x = w.Xn[(size_t)l * g.ns + i];
            moved |= __float_as_uint(x) != __float_as_uint(w.X[(size_t)l * g.ns + i]);
            w.X[(size_t)l * g.ns + i] = x;
            if (valid) {
                if (keyed) key |= (unsigned long long)cell_dim(x, g) << (16 * l);
                else changed |= cell_dim(x, g) != w.cell_dims[(size_t)l * g.ns + c];
            }
        }
        if (valid && keyed) changed |= key != w.cell_key[c];
        // per warp of sorted points: did any of them move?  (lane 0 of the
        // warp is active whenever any lane is: the warp's first index is < n)
        const unsigned m = __ballot_sync(__activemask(), moved);
        if ((threadIdx.x & 31) == 0 && w.warp_moved) w.warp_moved[i >> 5] = m != 0;
    }
    if (!valid) changed = true;
    // the incremental update's need marks are rebuilt after every grid check
    for (int o = bx * blockDim.x + threadIdx.x; o < g.n_outer; o += gx * blockDim.x) w.need[o] = 0;
    if (__syncthreads_or(changed) && threadIdx.x == 0) w.ctrl[kCtrlChanged] = 1;
}

__device__ __forceinline__ void build_begin_body(const Work& w) { w.ctrl[kCtrlChanged] = 0; }

// radix sort pass: tile histograms
__device__ __forceinline__ void radix_hist_body(const Geom& g, const Work& w, int in_sel, int first, int dim, int shift, int bx) {
    EGG_SKIP_IF_UNCHANGED(w.ctrl);
    __shared__ int h[256];
    const int tiles = (g.n + kSortTile - 1) / kSortTile;
    const int* pin = perm_buf(w, in_sel);
    for (int t = threadIdx.x; t < 256; t += blockDim.x) h[t] = 0;
    __syncthreads();
    const int base = bx * kSortTile;
    const int end = min(base + kSortTile, g.n);
    for (int i = base + threadIdx.x; i < end; i += blockDim.x) {
        int j = first ? i : __ldg(pin + i);
        int dg = digit_of(g, w.Xn, j, dim, shift);
        unsigned act = __activemask();
        unsigned peers = __match_any_sync(act, dg);
        if ((peers & lanemask_lt()) == 0) atomicAdd(&h[dg], __popc(peers));
    }
    __syncthreads();
    for (int t = threadIdx.x; t < 256; t += blockDim.x) w.hist[(size_t)t * tiles + bx] = h[t];
}

// per-digit exclusive scan over tiles (one block per digit)
__device__ __forceinline__ void radix_scan_body(const Geom& g, const Work& w, int bx) {
    EGG_SKIP_IF_UNCHANGED(w.ctrl);
    const int tiles = (g.n + kSortTile - 1) / kSortTile;
    if (tiles <= kScanSmallTiles) {
        // one block for all digits: a thread walks its digit's tiles
        const int t = threadIdx.x;
        if (t < 256) {
            int* h = w.hist + (size_t)t * tiles;
            int run = 0;
            for (int k = 0; k < tiles; k++) {
                const int v = h[k];
                h[k] = run;
                run += v;
            }
            w.digit_total[t] = run;
        }
        return;
    }
    int* h = w.hist + (size_t)bx * tiles;
    const int per = (tiles + blockDim.x - 1) / blockDim.x;
    const int b = threadIdx.x * per;
    const int e = min(b + per, tiles);
    int s = 0;
    for (int k = b; k < e; k++) s += h[k];
    int total;
    int run = block_exclusive_scan(s, &total);
    for (int k = b; k < e; k++) {
        int v = h[k];
        h[k] = run;
        run += v;
    }
    if (threadIdx.x == 0) w.digit_total[bx] = total;
}

// stable scatter of one tile
__device__ __forceinline__ void radix_scatter_body(const Geom& g, const Work& w, int in_sel, int out_sel, int first, int dim, int shift,
                                   int bx) {
    EGG_SKIP_IF_UNCHANGED(w.ctrl);
    constexpr int kWarps = kSortThreads / 32;
    __shared__ int base[256];
    __shared__ int run[256];
    __shared__ int wcnt[kWarps][256];
    const int tiles = (g.n + kSortTile - 1) / kSortTile;
    const int* pin = perm_buf(w, in_sel);
    int* pout = perm_buf(w, out_sel);
    const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
    {
        int v = w.digit_total[tid];
        int db = block_exclusive_scan(v, nullptr);
        base[tid] = db + w.hist[(size_t)tid * tiles + bx];
        run[tid] = 0;
#pragma unroll
        for (int k = 0; k < kWarps; k++) wcnt[k][tid] = 0;
    }
    __syncthreads();
    const int tile0 = bx * kSortTile;
    for (int round = 0; round < kSortTile / kSortThreads; round++) {
        const int i = tile0 + round * kSortThreads + tid;
        if (tile0 + round * kSortThreads >= g.n) break;  // uniform across the block
        const bool valid = i < g.n;
        int j = 0, dg = 0;
        if (valid) {
            j = first ? i : __ldg(pin + i);
            dg = digit_of(g, w.Xn, j, dim, shift);
        }
        unsigned peers = __match_any_sync(0xffffffffu, valid ? dg : 256 + lane);
        int rank = __popc(peers & lanemask_lt());
        if (valid && rank == 0) wcnt[wid][dg] = __popc(peers);
        __syncthreads();
        {
            int r = run[tid];
#pragma unroll
            for (int k = 0; k < kWarps; k++) {
                int c = wcnt[k][tid];
                wcnt[k][tid] = r;
                r += c;
            }
            run[tid] = r;
        }
        __syncthreads();
        if (valid) pout[base[dg] + wcnt[wid][dg] + rank] = j;
        __syncthreads();
#pragma unroll
        for (int k = 0; k < kWarps; k++) wcnt[k][tid] = 0;
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------
// One-key grid sort (d <= 3, at most 256 cells per dimension): the whole sort
// key of a point -- the sub-cell digit in bits 0-7, then the cell
// coordinates in the order of the per-dimension passes (plan_pass), 8 bits
// each -- fits in 32 bits, so it is computed once and the LSD passes move
// (key, previous position) pairs with coalesced reads instead of recomputing
// every pass's digit through the permutation.  The digits and their order
// are those of the per-dimension passes and every pass is stable, so the
// resulting permutation is the same.
// ---------------------------------------------------------------------------
__device__ __forceinline__ int onekey_passes(const Geom& g) { return 1 + g.d; }

// keys of the points in their current order; the first pass's payload (the
// identity) goes to the buffer that makes the last pass end in perm
__device__ __forceinline__ void onekey_keys_body(const Geom& g, const Work& w, int bx, int gx) {
    EGG_SKIP_IF_UNCHANGED(w.ctrl);
    const int P = onekey_passes(g);
    int* v0 = (P & 1) ? w.perm_tmp : w.perm;
    for (int i = bx * blockDim.x + threadIdx.x; i < g.n; i += gx * blockDim.x) {
        unsigned key = (unsigned)digit_of(g, w.Xn, i, -1, 0);
        for (int p = 1; p < P; p++) {
            int dim, shift;
            plan_pass(g, p, dim, shift);
            key |= (unsigned)(cell_dim(__ldg(w.Xn + (size_t)dim * g.ns + i), g) & 255) << (8 * p);
        }
        w.skey[0][i] = key;
        v0[i] = i;
    }
}

__device__ __forceinline__ void onekey_hist_body(const Geom& g, const Work& w, int p, int bx) {
    EGG_SKIP_IF_UNCHANGED(w.ctrl);
    __shared__ int h[256];
    const int tiles = (g.n + kSortTile - 1) / kSortTile;
    const unsigned* kin = w.skey[p & 1];
    for (int t = threadIdx.x; t < 256; t += blockDim.x) h[t] = 0;
    __syncthreads();
    const int b = bx * kSortTile, e = min(b + kSortTile, g.n);
    for (int i = b + threadIdx.x; i < e; i += blockDim.x) atomicAdd(&h[(__ldg(kin + i) >> (8 * p)) & 255u], 1);
    __syncthreads();
    for (int t = threadIdx.x; t < 256; t += blockDim.x) w.hist[(size_t)t * tiles + bx] = h[t];
}

// stable scatter of one tile of (key, previous position) pairs
__device__ __forceinline__ void onekey_scatter_body(const Geom& g, const Work& w, int p, int bx) {
    EGG_SKIP_IF_UNCHANGED(w.ctrl);
    constexpr int kWarps = kSortThreads / 32;
    __shared__ int base[256];
    __shared__ int run[256];
    __shared__ int wcnt[kWarps][256];
    const int P = onekey_passes(g);
    const int tiles = (g.n + kSortTile - 1) / kSortTile;
    const unsigned* kin = w.skey[p & 1];
    unsigned* kout = w.skey[(p + 1) & 1];
    // payload ping-pong that ends in perm: pass p writes perm when P - 1 - p is even
    const int* vin = ((P - p) & 1) ? w.perm_tmp : w.perm;
    int* vout = ((P - 1 - p) & 1) ? w.perm_tmp : w.perm;
    const int shift = 8 * p;
    const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
    {
        const int v = w.digit_total[tid];
        const int db = block_exclusive_scan(v, nullptr);
        base[tid] = db + w.hist[(size_t)tid * tiles + bx];
        run[tid] = 0;
#pragma unroll
        for (int k = 0; k < kWarps; k++) wcnt[k][tid] = 0;
    }
    __syncthreads();
    const int tile0 = bx * kSortTile;
    for (int round = 0; round < kSortTile / kSortThreads; round++) {
        if (tile0 + round * kSortThreads >= g.n) break;  // uniform across the block
        const int i = tile0 + round * kSortThreads + tid;
        const bool valid = i < g.n;
        unsigned key = 0;
        int dg = 0;
        if (valid) {
            key = __ldg(kin + i);
            dg = (int)((key >> shift) & 255u);
        }
        const unsigned peers = __match_any_sync(0xffffffffu, valid ? dg : 256 + lane);
        const int rank = __popc(peers & lanemask_lt());
        if (valid && rank == 0) wcnt[wid][dg] = __popc(peers);
        __syncthreads();
        {
            int r = run[tid];
#pragma unroll
            for (int k = 0; k < kWarps; k++) {
                const int c = wcnt[k][tid];
                wcnt[k][tid] = r;
                r += c;
            }
            run[tid] = r;
        }
        __syncthreads();
        if (valid) {
            const int pos = base[dg] + wcnt[wid][dg] + rank;
            if (p + 1 < P) kout[pos] = key;
            vout[pos] = __ldg(vin + i);
        }
        __syncthreads();
#pragma unroll
        for (int k = 0; k < kWarps; k++) wcnt[k][tid] = 0;
        __syncthreads();
    }
}

// gather into the new order and count cell heads per block
template <int D>
__device__ __forceinline__ void gather_heads_body(const Geom& g, const Work& w, int identity, int bx) {
    EGG_SKIP_IF_UNCHANGED(w.ctrl);
    const int d = D > 0 ? D : g.d;
    const int i = bx * blockDim.x + threadIdx.x;
    int head = 0;
    if (i < g.n) {
        const int j = identity ? i : __ldg(w.perm + i);
        const int jp = i > 0 ? (identity ? i - 1 : __ldg(w.perm + i - 1)) : 0;
        head = (i == 0);
        for (int l = 0; l < d; l++) {
            float x = __ldg(w.Xn + (size_t)l * g.ns + j);
            w.X[(size_t)l * g.ns + i] = x;
            if (i > 0) {
                float xp = __ldg(w.Xn + (size_t)l * g.ns + jp);
                head |= (cell_dim(x, g) != cell_dim(xp, g));
            }
        }
        w.orig_tmp[i] = __ldg(w.orig + j);
    }
    int total;
    block_exclusive_scan(head, &total);
    if (threadIdx.x == 0) w.block_sums[bx] = total;
}

// single-block exclusive scan of the per-block head counts; M = total
__device__ __forceinline__ void scan_block_sums_body(const Geom& g, const Work& w) {
    EGG_SKIP_IF_UNCHANGED(w.ctrl);
    const int nb = (g.n + kHeadsBlock - 1) / kHeadsBlock;
    int* bs = w.block_sums;
    const int per = (nb + blockDim.x - 1) / blockDim.x;
    const int b = threadIdx.x * per;
    const int e = min(b + per, nb);
    int s = 0;
    for (int k = b; k < e; k++) s += bs[k];
    int total;
    int run = block_exclusive_scan(s, &total);
    for (int k = b; k < e; k++) {
        int v = bs[k];
        bs[k] = run;
        run += v;
    }
    if (threadIdx.x == 0) {
        w.ctrl[kCtrlM] = total;
        w.ctrl[kCtrlGridValid] = 1;
        w.ctrl[kCtrlBuilds] += 1;
        // the spanning-cell lists describe the grid: rebuilt with it
        w.ctrl[kCtrlSpanCount] = 0;
        w.ctrl[kCtrlBigCount] = 0;
    }
}

template <int D>
__device__ __forceinline__ void heads_finalize_body(const Geom& g, const Work& w, int bx) {
    EGG_SKIP_IF_UNCHANGED(w.ctrl);
    const int d = D > 0 ? D : g.d;
    const int i = bx * blockDim.x + threadIdx.x;
    // the outer-ranges kernel that follows ORs the column masks in
    // (n_outer = width^od <= n: one thread per point covers every column)
    if (g.od < d && w.colmask != nullptr && i < g.n_outer) w.colmask[i] = 0ull;
    int head = 0;
    if (i < g.n) {
        head = (i == 0);
        if (i > 0)
            for (int l = 0; l < d && !head; l++)
                head = cell_dim(w.X[(size_t)l * g.ns + i], g) != cell_dim(w.X[(size_t)l * g.ns + i - 1], g);
    }
    int excl = block_exclusive_scan(head, nullptr) + w.block_sums[bx];
    if (i < g.n) {
        const int c = excl + head - 1;
        w.cell_of[i] = c;
        w.orig[i] = w.orig_tmp[i];
        if (head) {
            w.cell_start[c] = i;
            int outer = 0;
            unsigned long long key = 0;
            for (int l = 0; l < d; l++) {
                int gl = cell_dim(w.X[(size_t)l * g.ns + i], g);
                w.cell_dims[(size_t)l * g.ns + c] = gl;
                if (l < g.od) outer += gl * g.wpow[l];
                if (l < 4) key |= (unsigned long long)gl << (16 * l);
            }
            w.cell_outer[c] = outer;
            if (d <= 4 && w.cell_key) w.cell_key[c] = key;
        }
        if (i == g.n - 1) w.cell_start[c + 1] = g.n;
    }
}

// outer_begin[o] = first cell whose outer id >= o, o in [0, n_outer]; with
// od < d, colmask[o] = the blocks of dimension od (zblk cells each, bit
// z / zblk) that hold a cell of outer cell o
__device__ __forceinline__ void outer_ranges_body(const Geom& g, const Work& w, int bx, int gx) {
    EGG_SKIP_IF_UNCHANGED(w.ctrl);
    const int M = w.ctrl[kCtrlM];
    const bool cols = g.od < g.d && w.colmask != nullptr;
    const int* z = w.cell_dims + (size_t)g.od * g.ns;
    // A thread per cell: cell c is the first cell of every column o with
    // cell_outer[c - 1] < o <= cell_outer[c] (columns in between are empty;
    // c = M closes the last one), so outer_begin[o] is the first cell of a
    // column at or after o, each entry written once.  A column's mask of
    // occupied blocks of dimension od is the OR over its cells: one atomic
    // per column and warp (the heads kernel zeroed the masks).
    for (int c = bx * blockDim.x + threadIdx.x; c <= M; c += gx * blockDim.x) {
        const int oc = c < M ? w.cell_outer[c] : g.n_outer;
        const int op = c > 0 ? w.cell_outer[c - 1] : -1;
        for (int o = op + 1; o <= oc; o++) w.outer_begin[o] = c;
        if (cols && c < M) {
            const unsigned long long bit = 1ull << (z[c] / g.zblk);
            const unsigned peers = __match_any_sync(__activemask(), oc);
            const unsigned lo = __reduce_or_sync(peers, (unsigned)bit);
            const unsigned hi = __reduce_or_sync(peers, (unsigned)(bit >> 32));
            if ((threadIdx.x & 31) == __ffs(peers) - 1)
                atomicOr(w.colmask + oc, ((unsigned long long)hi << 32) | lo);
        }
    }
}

// ---------------------------------------------------------------------------
// per-cell sums of sin(delta) and 1 - cos(delta), delta = x - cell corner,
// plus the tight bounding box of each cell's points
// ---------------------------------------------------------------------------
template <int D>
__device__ __forceinline__ void cell_sums_body(const Geom& g, const Work& w, int bx) {
    const int d = D > 0 ? D : g.d;
    const int i = bx * blockDim.x + threadIdx.x;
    const int lane = threadIdx.x & 31;
    const int warp = i >> 5;
    const int nw = (g.n + 31) >> 5;
    if ((i & ~31) >= g.n) return;  // whole warp beyond n
    // Unchanged grid and none of the warp's points moved: every output of
    // this warp (point offsets, complete-cell sums, warp partials of
    // spanning cells) is what the last launch wrote.  The spanning-cell
    // lists are kept from the last rebuild.
    const bool rebuilt = w.ctrl[kCtrlChanged] != 0;
    if (!rebuilt && w.warp_moved[i >> 5] == 0) return;
    const bool valid = i < g.n;
    const int c = valid ? w.cell_of[i] : 0x7fffffff - lane;
    const int cnext = __shfl_down_sync(0xffffffffu, c, 1);
    const bool seg_end = valid && (lane == 31 || cnext != c);
    const int wb = i & ~31;
    int cs = 0, ce = 0;
    if (seg_end) {
        cs = w.cell_start[c];
        ce = w.cell_start[c + 1];
    }
    const bool complete = seg_end && cs >= wb && ce <= wb + 32;
    // a spanning cell with a warp re-summed in this iteration: its warp
    // partials are combined again (every warp holding a point of the cell
    // has a segment end for it)
    if (seg_end && !complete) w.span_mark[c] = w.ctrl[kCtrlIter];
    // a cell that starts in this warp and continues past it: list it once
    // for the FP64 combination of its warp partials
    if (rebuilt && seg_end && cs >= wb && ce > wb + 32) {
        if (((ce - 1) >> 5) - (cs >> 5) > 2) w.big_list[atomicAdd(w.ctrl + kCtrlBigCount, 1)] = c;
        else w.span_list[atomicAdd(w.ctrl + kCtrlSpanCount, 1)] = c;
    }
    constexpr bool kPacked = D >= 1 && D <= kPackDims;
    constexpr int PW = kPacked ? pack_w(D) : 1, PS = kPacked ? pack_s(D) : 1;
    float pk_x[4 * PW], pk_s[4 * PS];
    if constexpr (kPacked) {
#pragma unroll
        for (int k = 0; k < 4 * PW; k++) pk_x[k] = 0.f;
#pragma unroll
        for (int k = 0; k < 4 * PS; k++) pk_s[k] = 0.f;
    }
    for (int l = 0; l < d; l++) {
        float s = 0.f, m = 0.f, x = 0.f;
        if (valid) {
            x = w.X[(size_t)l * g.ns + i];
            int cd = w.cell_dims[(size_t)l * g.ns + c];
            float corner = __fmul_rn((float)cd, g.side);
            float delta = __fsub_rn(x, corner);
            float sh, ch;
            sincosf(0.5f * delta, &sh, &ch);
            s = 2.0f * sh * ch;
            m = 2.0f * sh * sh;
            if constexpr (kPacked) {
                pk_x[l] = x;
                pk_s[l] = s;
                pk_s[d + l] = m;
            } else {
                w.sd[(size_t)l * g.ns + i] = s;
                w.md[(size_t)l * g.ns + i] = m;
            }
        }
        TwoSum vs{s, 0.f}, vm{m, 0.f};
        float mn = x, mx = x;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            TwoSum us{__shfl_up_sync(0xffffffffu, vs.hi, o), __shfl_up_sync(0xffffffffu, vs.lo, o)};
            TwoSum um{__shfl_up_sync(0xffffffffu, vm.hi, o), __shfl_up_sync(0xffffffffu, vm.lo, o)};
            float umn = __shfl_up_sync(0xffffffffu, mn, o);
            float umx = __shfl_up_sync(0xffffffffu, mx, o);
            int uc = __shfl_up_sync(0xffffffffu, c, o);
            if (lane >= o && uc == c) {
                vs = ts_add(us, vs);
                vm = ts_add(um, vm);
                mn = fminf(mn, umn);
                mx = fmaxf(mx, umx);
            }
        }
        if (complete) {
            w.css[(size_t)l * g.ns + c] = __fadd_rn(vs.hi, vs.lo);
            w.csm[(size_t)l * g.ns + c] = __fadd_rn(vm.hi, vm.lo);
            w.cbmin[(size_t)l * g.ns + c] = mn;
            w.cbmax[(size_t)l * g.ns + c] = mx;
        } else if (seg_end) {
            // partial of a cell spanning several warps: rec 0 = segment holding
            // lane 0 (continues from the previous warp), rec 1 = segment holding
            // lane 31 (continues into the next warp); a warp inside one cell
            // writes both.  The FP32 copy (gpart) is the record of this
            // 32-point group of the cell, used to decide groups wholesale.
            const double S = (double)vs.hi + (double)vs.lo;
            const double Mm = (double)vm.hi + (double)vm.lo;
            const float Sf = __fadd_rn(vs.hi, vs.lo), Mf = __fadd_rn(vm.hi, vm.lo);
            for (int rec = 0; rec < 2; rec++) {
                if (rec == 0 ? !(cs < wb) : !(ce > wb + 32)) continue;
                w.wpart[wp_idx(0, l, d, rec, nw, warp)] = S;
                w.wpart[wp_idx(1, l, d, rec, nw, warp)] = Mm;
                w.wpart[wp_idx(2, l, d, rec, nw, warp)] = mn;
                w.wpart[wp_idx(3, l, d, rec, nw, warp)] = mx;
                w.gpart[wp_idx(0, l, d, rec, nw, warp)] = Sf;
                w.gpart[wp_idx(1, l, d, rec, nw, warp)] = Mf;
                w.gpart[wp_idx(2, l, d, rec, nw, warp)] = mn;
                w.gpart[wp_idx(3, l, d, rec, nw, warp)] = mx;
            }
        }
    }
    if constexpr (kPacked) {
        if (!valid) return;
#pragma unroll
        for (int k = 0; k < PW; k++)
            w.xp[(size_t)i * PW + k] = make_float4(pk_x[4 * k], pk_x[4 * k + 1], pk_x[4 * k + 2], pk_x[4 * k + 3]);
#pragma unroll
        for (int k = 0; k < PS; k++)
            w.smp[(size_t)i * PS + k] = make_float4(pk_s[4 * k], pk_s[4 * k + 1], pk_s[4 * k + 2], pk_s[4 * k + 3]);
    }
}

// one big spanning cell, the whole warp: lanes stride over its warp partials
template <int D>
__device__ void combine_big(const Geom& g, const Work& w, int c, int wh, int wt, int lane, int nw) {
    constexpr int DM = D > 0 ? D : 1;
    const int d = D > 0 ? D : g.d;
    if (D > 0) {
        // every dimension in one pass: 4*D independent loads per partial
        double S[DM], Mm[DM], mn[DM], mx[DM];
#pragma unroll
        for (int l = 0; l < DM; l++) { S[l] = 0.0; Mm[l] = 0.0; mn[l] = 1e300; mx[l] = -1e300; }
        // kBatch partials per lane in flight: all their loads first, then
        // the accumulation in the lane's order k = wh + lane, +32, ...
        // (wide d: one at a time, the accumulators fill the registers)
        constexpr int kBatch = DM <= 4 ? 4 : 1;
        if constexpr (kBatch == 1) {
            for (int k = wh + lane; k <= wt; k += 32) {
                const int rec = (k == wh) ? 1 : 0;
#pragma unroll
                for (int l = 0; l < DM; l++) {
                    S[l] += w.wpart[wp_idx(0, l, d, rec, nw, k)];
                    Mm[l] += w.wpart[wp_idx(1, l, d, rec, nw, k)];
                    mn[l] = fmin(mn[l], w.wpart[wp_idx(2, l, d, rec, nw, k)]);
                    mx[l] = fmax(mx[l], w.wpart[wp_idx(3, l, d, rec, nw, k)]);
                }
            }
        } else {
            for (int k0 = wh + lane; k0 <= wt; k0 += 32 * kBatch) {
                double v[kBatch][4][DM];
#pragma unroll
                for (int u = 0; u < kBatch; u++) {
                    const int k = k0 + 32 * u;
                    const int kk = k <= wt ? k : k0;  // in-range stand-in, not accumulated
                    const int rec = (kk == wh) ? 1 : 0;
#pragma unroll
                    for (int l = 0; l < DM; l++)
#pragma unroll
                        for (int f = 0; f < 4; f++) v[u][f][l] = w.wpart[wp_idx(f, l, d, rec, nw, kk)];
                }
#pragma unroll
                for (int u = 0; u < kBatch; u++) {
                    if (k0 + 32 * u > wt) break;
#pragma unroll
                    for (int l = 0; l < DM; l++) {
                        S[l] += v[u][0][l];
                        Mm[l] += v[u][1][l];
                        mn[l] = fmin(mn[l], v[u][2][l]);
                        mx[l] = fmax(mx[l], v[u][3][l]);
                    }
                }
            }
        }
#pragma unroll
        for (int l = 0; l < DM; l++) {
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
                S[l] += __shfl_xor_sync(0xffffffffu, S[l], o);
                Mm[l] += __shfl_xor_sync(0xffffffffu, Mm[l], o);
                mn[l] = fmin(mn[l], __shfl_xor_sync(0xffffffffu, mn[l], o));
                mx[l] = fmax(mx[l], __shfl_xor_sync(0xffffffffu, mx[l], o));
            }
            if (lane == 0) {
                w.css[(size_t)l * g.ns + c] = (float)S[l];
                w.csm[(size_t)l * g.ns + c] = (float)Mm[l];
                w.cbmin[(size_t)l * g.ns + c] = (float)mn[l];
                w.cbmax[(size_t)l * g.ns + c] = (float)mx[l];
            }
        }
    } else {
        for (int l = 0; l < d; l++) {
            double S = 0.0, Mm = 0.0, mn = 1e300, mx = -1e300;
            for (int k = wh + lane; k <= wt; k += 32) {
                const int rec = (k == wh) ? 1 : 0;
                S += w.wpart[wp_idx(0, l, d, rec, nw, k)];
                Mm += w.wpart[wp_idx(1, l, d, rec, nw, k)];
                mn = fmin(mn, w.wpart[wp_idx(2, l, d, rec, nw, k)]);
                mx = fmax(mx, w.wpart[wp_idx(3, l, d, rec, nw, k)]);
            }
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
                S += __shfl_xor_sync(0xffffffffu, S, o);
                Mm += __shfl_xor_sync(0xffffffffu, Mm, o);
                mn = fmin(mn, __shfl_xor_sync(0xffffffffu, mn, o));
                mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
            }
            if (lane == 0) {
                w.css[(size_t)l * g.ns + c] = (float)S;
                w.csm[(size_t)l * g.ns + c] = (float)Mm;
                w.cbmin[(size_t)l * g.ns + c] = (float)mn;
                w.cbmax[(size_t)l * g.ns + c] = (float)mx;
            }
        }
    }
}

// One field of one big spanning cell (0: sum sin, 1: sum 1 - cos, 2: min,
// 3: max), the whole warp: lane L accumulates the partials of warps
// wh + L, wh + L + 32, ... in that order, then a butterfly over the lanes --
// the order combine_big uses, so the result is the same bit for bit.  The
// four fields of a cell go to four warps, and each lane keeps kB partials
// per dimension in flight: a cell over thousands of warps no longer holds
// the launch on one warp's chain of loads.
template <int D>
__device__ void combine_big_field(const Geom& g, const Work& w, int c, int wh, int wt, int lane, int nw, int f) {
    constexpr int kB = 48 / D > 0 ? 48 / D : 1;
    const int d = D;
    double acc[D];
#pragma unroll
    for (int l = 0; l < D; l++) acc[l] = f < 2 ? 0.0 : (f == 2 ? 1e300 : -1e300);
    for (int k0 = wh + lane; k0 <= wt; k0 += 32 * kB) {
        double v[kB][D];
#pragma unroll
        for (int u = 0; u < kB; u++) {
            const int k = k0 + 32 * u;
            const int kk = k <= wt ? k : k0;  // in-range stand-in, not accumulated
            const int rec = (kk == wh) ? 1 : 0;
#pragma unroll
            for (int l = 0; l < D; l++) v[u][l] = w.wpart[wp_idx(f, l, d, rec, nw, kk)];
        }
#pragma unroll
        for (int u = 0; u < kB; u++) {
            if (k0 + 32 * u > wt) break;
#pragma unroll
            for (int l = 0; l < D; l++)
                acc[l] = f < 2 ? acc[l] + v[u][l] : (f == 2 ? fmin(acc[l], v[u][l]) : fmax(acc[l], v[u][l]));
        }
    }
    float* out = f == 0 ? w.css : (f == 1 ? w.csm : (f == 2 ? w.cbmin : w.cbmax));
#pragma unroll
    for (int l = 0; l < D; l++) {
        double a = acc[l];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            const double b = __shfl_xor_sync(0xffffffffu, a, o);
            a = f < 2 ? a + b : (f == 2 ? fmin(a, b) : fmax(a, b));
        }
        if (lane == 0) out[(size_t)l * g.ns + c] = (float)a;
    }
}

// Cells spanning more than one warp: combine the warp partials in FP64 in a
// fixed order.  Cells over four or more warps (the heavily populated ones)
// get a warp each; the others (nearly all: a small cell straddling a warp
// boundary) a thread each.  The list order depends on scheduling, the result
// of every cell does not.
template <int D>
__device__ __forceinline__ void cell_sums_fix_body(const Geom& g, const Work& w, int bx, int gx) {
    const int d = D > 0 ? D : g.d;
    const int lane = threadIdx.x & 31;
    const int nw = (g.n + 31) >> 5;
    // with the grid unchanged, a cell none of whose warps moved keeps its sums
    // (marked by the cell-sums kernel of this iteration)
    const bool rebuilt = w.ctrl[kCtrlChanged] != 0;
    const int it = w.ctrl[kCtrlIter];
    const int big = w.ctrl[kCtrlBigCount];
    const int warps = (gx * blockDim.x) >> 5;
    if constexpr (D > 0) {
        // a warp per (cell, field)
        for (int e = (bx * blockDim.x + threadIdx.x) >> 5; e < 4 * big; e += warps) {
            const int c = w.big_list[e >> 2];
            if (!rebuilt && w.span_mark[c] != it) continue;  // uniform across the warp
            const int wh = w.cell_start[c] >> 5, wt = (w.cell_start[c + 1] - 1) >> 5;
            combine_big_field<D>(g, w, c, wh, wt, lane, nw, e & 3);
        }
    } else {
        for (int e = (bx * blockDim.x + threadIdx.x) >> 5; e < big; e += warps) {
            const int c = w.big_list[e];
            if (!rebuilt && w.span_mark[c] != it) continue;  // uniform across the warp
            const int wh = w.cell_start[c] >> 5, wt = (w.cell_start[c + 1] - 1) >> 5;
            combine_big<D>(g, w, c, wh, wt, lane, nw);
        }
    }
    const int count = w.ctrl[kCtrlSpanCount];
    for (int e = bx * blockDim.x + threadIdx.x; e < count; e += gx * blockDim.x) {
        const int c = w.span_list[e];
        if (!rebuilt && w.span_mark[c] != it) continue;
        const int wh = w.cell_start[c] >> 5, wt = (w.cell_start[c + 1] - 1) >> 5;
        for (int l = 0; l < d; l++) {
            double S = 0.0, Mm = 0.0, mn = 1e300, mx = -1e300;
            for (int k = wh; k <= wt; k++) {
                const int rec = (k == wh) ? 1 : 0;
                S += w.wpart[wp_idx(0, l, d, rec, nw, k)];
                Mm += w.wpart[wp_idx(1, l, d, rec, nw, k)];
                mn = fmin(mn, w.wpart[wp_idx(2, l, d, rec, nw, k)]);
                mx = fmax(mx, w.wpart[wp_idx(3, l, d, rec, nw, k)]);
            }
            w.css[(size_t)l * g.ns + c] = (float)S;
            w.csm[(size_t)l * g.ns + c] = (float)Mm;
            w.cbmin[(size_t)l * g.ns + c] = (float)mn;
            w.cbmax[(size_t)l * g.ns + c] = (float)mx;
        }
    }
}

// ---------------------------------------------------------------------------
// single-instance and batched wrappers
// ---------------------------------------------------------------------------
#define EGG_WRAP0(NAME, BOUNDS, BODYCALL)                                            \
    __global__ void __launch_bounds__(BOUNDS) k_##NAME(Geom g, Work w) {             \
        const int bx = blockIdx.x, gx = gridDim.x;                                   \
        (void)bx; (void)gx;                                                          \
        BODYCALL;                                                                    \
    }                                                                                \
    __global__ void __launch_bounds__(BOUNDS) kb_##NAME(BatchArgs B) {               \
        batch_for(B, [&](const Geom& g, const Work& w, int bx, int gx) {             \
            (void)bx; (void)gx;                                                      \
            BODYCALL;                                                                \
        });                                                                          \
    }

#define EGG_WRAPD(NAME, BOUNDS, BODYCALL)                                                \
    template <int D>                                                                     \
    __global__ void __launch_bounds__(BOUNDS) k_##NAME(Geom g, Work w) {                 \
        const int bx = blockIdx.x, gx = gridDim.x;                                       \
        (void)bx; (void)gx;                                                              \
        BODYCALL;                                                                        \
    }                                                                                    \
    template <int D>                                                                     \
    __global__ void __launch_bounds__(BOUNDS) kb_##NAME(BatchArgs B) {                   \
        batch_for(B, [&](const Geom& g, const Work& w, int bx, int gx) {                 \
            (void)bx; (void)gx;                                                          \
            BODYCALL;                                                                    \
        });                                                                              \
    }

EGG_WRAPD(check_cells, 256, check_cells_body<D>(g, w, bx, gx))
EGG_WRAP0(build_begin, 32, (void)g; if (threadIdx.x == 0) build_begin_body(w))
EGG_WRAP0(scan_block_sums, 1024, scan_block_sums_body(g, w))
__global__ void __launch_bounds__(256) k_radix_scan(Geom g, Work w) { radix_scan_body(g, w, blockIdx.x); }
EGG_WRAPD(heads_finalize, kHeadsBlock, heads_finalize_body<D>(g, w, bx))
EGG_WRAP0(outer_ranges, 256, outer_ranges_body(g, w, bx, gx))
// single instance: a grid capped at 148 x 8 blocks strides over the
// 256-point blocks (late in a run nearly every warp returns at once, and a
// full-size grid would be mostly block scheduling); batched: one virtual
// block each
template <int D>
__global__ void __launch_bounds__(256) k_cell_sums(Geom g, Work w) {
    const int nblk = (g.n + 255) / 256;
    for (int bx = blockIdx.x; bx < nblk; bx += gridDim.x) cell_sums_body<D>(g, w, bx);
}
template <int D>
__global__ void __launch_bounds__(256) kb_cell_sums(BatchArgs B) {
    batch_for(B, [&](const Geom& g, const Work& w, int bx, int gx) {
        (void)gx;
        cell_sums_body<D>(g, w, bx);
    });
}
EGG_WRAPD(cell_sums_fix, 256, cell_sums_fix_body<D>(g, w, bx, gx))

__global__ void __launch_bounds__(kSortThreads) k_radix_hist(Geom g, Work w, int in_sel, int first, int dim,
                                                             int shift) {
    radix_hist_body(g, w, in_sel, first, dim, shift, blockIdx.x);
}
__global__ void __launch_bounds__(kSortThreads) k_radix_scatter(Geom g, Work w, int in_sel, int out_sel, int first,
                                                                int dim, int shift) {
    radix_scatter_body(g, w, in_sel, out_sel, first, dim, shift, blockIdx.x);
}
// batched radix passes: pass p of each instance's own plan
__global__ void __launch_bounds__(kSortThreads) kb_radix_hist(BatchArgs B, int p) {
    batch_for(B, [&](const Geom& g, const Work& w, int bx, int) {
        const int count = plan_count(g);
        if (p >= count) return;
        int dim, shift;
        plan_pass(g, p, dim, shift);
        radix_hist_body(g, w, p > 0 ? plan_out_sel(count, p - 1) : 0, p == 0, dim, shift, bx);
    });
}
__global__ void __launch_bounds__(256) kb_radix_scan(BatchArgs B, int p) {
    batch_for(B, [&](const Geom& g, const Work& w, int bx, int) {
        if (p >= plan_count(g)) return;
        radix_scan_body(g, w, bx);
    });
}
__global__ void __launch_bounds__(kSortThreads) kb_radix_scatter(BatchArgs B, int p) {
    batch_for(B, [&](const Geom& g, const Work& w, int bx, int) {
        const int count = plan_count(g);
        if (p >= count) return;
        int dim, shift;
        plan_pass(g, p, dim, shift);
        radix_scatter_body(g, w, p > 0 ? plan_out_sel(count, p - 1) : 0, plan_out_sel(count, p), p == 0, dim, shift,
                           bx);
    });
}
__global__ void __launch_bounds__(256) k_onekey_keys(Geom g, Work w) { onekey_keys_body(g, w, blockIdx.x, gridDim.x); }
__global__ void __launch_bounds__(kSortThreads) k_onekey_hist(Geom g, Work w, int p) {
    onekey_hist_body(g, w, p, blockIdx.x);
}
__global__ void __launch_bounds__(kSortThreads) k_onekey_scatter(Geom g, Work w, int p) {
    onekey_scatter_body(g, w, p, blockIdx.x);
}
template <int D>
__global__ void __launch_bounds__(kHeadsBlock) k_gather_heads(Geom g, Work w) {
    gather_heads_body<D>(g, w, 0, blockIdx.x);
}
template <int D>
__global__ void __launch_bounds__(kHeadsBlock) kb_gather_heads(BatchArgs B) {
    batch_for(B, [&](const Geom& g, const Work& w, int bx, int) { gather_heads_body<D>(g, w, 0, bx); });
}

// ---------------------------------------------------------------------------
// misc: input transpose, labels
// ---------------------------------------------------------------------------
__global__ void k_transpose_in(Geom g, Work w, const float* __restrict__ x_aos) {
    for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < (size_t)g.n * g.d;
         t += (size_t)gridDim.x * blockDim.x) {
        const int p = (int)(t / g.d), l = (int)(t % g.d);
        float v = x_aos[t];
        if (!isfinite(v)) atomicOr(w.ctrl + kCtrlStatus, kErrNonFinite);
        w.Xn[(size_t)l * g.ns + p] = v;
        if (l == 0) w.orig[p] = p;
    }
}

// positions of the sorted points back to original order (row-major n x d)
__global__ void k_unsort_positions(Geom g, Work w, const float* __restrict__ src, float* __restrict__ out) {
    for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < (size_t)g.n * g.d;
         t += (size_t)gridDim.x * blockDim.x) {
        const int i = (int)(t % g.n), l = (int)(t / g.n);
        out[(size_t)w.orig[i] * g.d + l] = src[(size_t)l * g.ns + i];
    }
}

// GPU_synCluster_float_grid semantics, EGG_SynC.cu:1205-1227: the compacted
// cell index when the cell holds more than one point, else -1.
__global__ void k_labels(Geom g, Work w, int* __restrict__ out) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < g.n; i += gridDim.x * blockDim.x) {
        const int c = w.cell_of[i];
        const int cs = w.cell_start[c];
        const int cnt = w.cell_start[c + 1] - cs;
        out[w.orig[i]] = cnt > 1 ? c : -1;
        if (i == cs && cnt > 1) atomicAdd(w.ctrl + kCtrlClusters, 1);
    }
}

__global__ void k_unsort_int(Geom g, Work w, const int* __restrict__ src, int* __restrict__ out) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < g.n; i += gridDim.x * blockDim.x)
        out[w.orig[i]] = src[i];
}

// ---------------------------------------------------------------------------
// launchers
// ---------------------------------------------------------------------------
#define EGG_DISPATCH_D(d, KERNEL, ...)                \
    switch (d) {                                      \
        case 1: KERNEL<1> __VA_ARGS__; break;         \
        case 2: KERNEL<2> __VA_ARGS__; break;         \
        case 3: KERNEL<3> __VA_ARGS__; break;         \
        case 4: KERNEL<4> __VA_ARGS__; break;         \
        case 5: KERNEL<5> __VA_ARGS__; break;         \
        case 6: KERNEL<6> __VA_ARGS__; break;         \
        case 8: KERNEL<8> __VA_ARGS__; break;         \
        case 16: KERNEL<16> __VA_ARGS__; break;       \
        default: KERNEL<0> __VA_ARGS__; break;        \
    }

// launch NAME (plain) or its batched twin with the same extra arguments
#define EGG_GO(ex, shape, threads, st, NAME, ...)                                                     \
    do {                                                                                             \
        if ((ex).batch())                                                                            \
            kb_##NAME<<<(ex).blocks(shape, threads), threads, 0, st>>>((ex).args(shape), ##__VA_ARGS__); \
        else                                                                                         \
            k_##NAME<<<(ex).blocks(shape, threads), threads, 0, st>>>(*(ex).g, *(ex).w, ##__VA_ARGS__); \
    } while (0)

#define EGG_GO_D(ex, shape, threads, st, NAME, ...)                                                   \
    do {                                                                                             \
        if ((ex).batch()) {                                                                          \
            EGG_DISPATCH_D((ex).d, kb_##NAME,                                                        \
                           <<<(ex).blocks(shape, threads), threads, 0, st>>>((ex).args(shape), ##__VA_ARGS__)); \
        } else {                                                                                     \
            EGG_DISPATCH_D((ex).d, k_##NAME,                                                         \
                           <<<(ex).blocks(shape, threads), threads, 0, st>>>(*(ex).g, *(ex).w, ##__VA_ARGS__)); \
        }                                                                                            \
    } while (0)

void launch_build_check(const Exec& ex, cudaStream_t st, bool begin) {
    if (begin) EGG_GO(ex, kShapeOne, 32, st, build_begin);
    EGG_GO_D(ex, kShapeCapN256, 256, st, check_cells);
}

void launch_build(const Exec& ex, cudaStream_t st) {
    launch_build_check(ex, st);
    launch_build_sort(ex, st);
}

void launch_build_sort(const Exec& ex, cudaStream_t st) {
    if (ex.batch()) {
        for (int p = 0; p < ex.bt->max_passes; p++) {
            kb_radix_hist<<<ex.blocks(kShapeTiles, kSortThreads), kSortThreads, 0, st>>>(ex.args(kShapeTiles), p);
            kb_radix_scan<<<ex.blocks(kShapeDigits, 256), 256, 0, st>>>(ex.args(kShapeDigits), p);
            kb_radix_scatter<<<ex.blocks(kShapeTiles, kSortThreads), kSortThreads, 0, st>>>(ex.args(kShapeTiles), p);
        }
    } else if (ex.w->skey[0] != nullptr && ex.g->d <= 3 && ex.g->width <= 256) {
        // one 32-bit key per point, 1 + d coalesced (key, position) passes
        const Geom& g = *ex.g;
        const int tiles = shape_blocks(kShapeTiles, g);
        const int kb = std::min((g.n + 255) / 256, 148 * 16);
        k_onekey_keys<<<kb, 256, 0, st>>>(g, *ex.w);
        for (int p = 0; p < 1 + g.d; p++) {
            k_onekey_hist<<<tiles, kSortThreads, 0, st>>>(g, *ex.w, p);
            k_radix_scan<<<shape_blocks(kShapeDigits, g), 256, 0, st>>>(g, *ex.w);
            k_onekey_scatter<<<tiles, kSortThreads, 0, st>>>(g, *ex.w, p);
        }
    } else {
        const Geom& g = *ex.g;
        const int count = plan_count(g);
        for (int p = 0; p < count; p++) {
            int dim, shift;
            plan_pass(g, p, dim, shift);
            const int in = p > 0 ? plan_out_sel(count, p - 1) : 0, out = plan_out_sel(count, p);
            const int tiles = shape_blocks(kShapeTiles, g);
            k_radix_hist<<<tiles, kSortThreads, 0, st>>>(g, *ex.w, in, p == 0, dim, shift);
            k_radix_scan<<<shape_blocks(kShapeDigits, g), 256, 0, st>>>(g, *ex.w);
            k_radix_scatter<<<tiles, kSortThreads, 0, st>>>(g, *ex.w, in, out, p == 0, dim, shift);
        }
    }
    EGG_GO_D(ex, kShapeN1024, kHeadsBlock, st, gather_heads);
    EGG_GO(ex, kShapeOne, 1024, st, scan_block_sums);
    EGG_GO_D(ex, kShapeN1024, kHeadsBlock, st, heads_finalize);
    EGG_GO(ex, kShapeOuter, 256, st, outer_ranges);
}

void launch_cell_sums(const Exec& ex, cudaStream_t st) {
    if (ex.batch()) {
        EGG_DISPATCH_D(ex.d, kb_cell_sums, <<<ex.blocks(kShapeN256, 256), 256, 0, st>>>(ex.args(kShapeN256)));
    } else {
        const int blocks = std::min(shape_blocks(kShapeN256, *ex.g), 148 * 8);
        EGG_DISPATCH_D(ex.d, k_cell_sums, <<<blocks, 256, 0, st>>>(*ex.g, *ex.w));
    }
    EGG_GO_D(ex, kShapeFix, 256, st, cell_sums_fix);
}

void launch_transpose_in(const Geom& g, const Work& w, const float* x, cudaStream_t st) {
    size_t tot = (size_t)g.n * g.d;
    int blocks = (int)((tot + 255) / 256);
    if (blocks > 148 * 16) blocks = 148 * 16;
    k_transpose_in<<<blocks, 256, 0, st>>>(g, w, x);
}

void launch_unsort_positions(const Geom& g, const Work& w, const float* src, float* out, cudaStream_t st) {
    size_t tot = (size_t)g.n * g.d;
    int blocks = (int)((tot + 255) / 256);
    if (blocks > 148 * 16) blocks = 148 * 16;
    k_unsort_positions<<<blocks, 256, 0, st>>>(g, w, src, out);
}

void launch_unsort_int(const Geom& g, const Work& w, const int* src, int* out, cudaStream_t st) {
    int blocks = (g.n + 255) / 256;
    if (blocks > 148 * 16) blocks = 148 * 16;
    k_unsort_int<<<blocks, 256, 0, st>>>(g, w, src, out);
}

void launch_labels(const Geom& g, const Work& w, int* out, cudaStream_t st) {
    int blocks = (g.n + 255) / 256;
    if (blocks > 148 * 16) blocks = 148 * 16;
    k_labels<<<blocks, 256, 0, st>>>(g, w, out);
}

}  // namespace egg
