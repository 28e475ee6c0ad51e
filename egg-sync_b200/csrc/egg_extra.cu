// egg_extra.cu -- extra convergence check of EGG-SynC.
//
// Replaces kernel_float_grid_extra_check_part1_count / part1 / part2 and
// MBR_in_eps of the reference (src/algorithms/EGG_SynC.cu:767-1203, host
// 1425-1489).  It runs only in iterations whose update left the flag at 1
// (both kernels return at once otherwise) and clears the flag when some pair
// (p, q) with eps < |p - q| <= eps_extra has the per-dimension closest corner
// of q's eps/2 group (its "MBR") within eps of p.
//
// The reference counts the pairs, reads the count back, allocates a pair
// list, lists the pairs and checks each one by walking q's eps/2 group.
// Here one pass walks the pairs and decides each one on the spot:
//   * k_ball_bbox first records, for every point q, the extremes of its eps/2
//     group per dimension.  When p lies outside [lo, hi] in a dimension, the
//     group's coordinate closest to p there is the extreme itself, so the MBR
//     is known without a walk; only dimensions where p falls inside [lo, hi]
//     need the reference's walk (mbr_exact).
//   * Cells are skipped wholesale with the tight bounding box of their points
//     when no point of theirs can lie in the (eps, eps_extra] annulus.
// Both shortcuts are exact under the shared float conventions (every
// comparison is monotone in the coordinates).
#include "egg_common.cuh"
#include "egg_kernels.h"

namespace egg {

namespace {

template <typename F>
__device__ __forceinline__ void for_stencil_cells(const Geom& g, const Work& w, int which, int rad, const int* gi,
                                                  int obase, int d, F&& fn) {
    const int nst = w.st_count[which];
    const int* st_delta = w.st_delta + (size_t)which * w.st_cap;
    const signed char* st_off = w.st_off + (size_t)which * w.st_cap * (g.od > 0 ? g.od : 1);
    for (int s = 0; s < nst; s++) {
        bool inb = true;
        for (int l = 0; l < g.od; l++) {
            int v = gi[l] + __ldg(st_off + (size_t)s * g.od + l);
            inb = inb && (unsigned)v < (unsigned)g.width;
        }
        if (!inb) continue;
        const int o = obase + __ldg(st_delta + s);
        int cb = __ldg(w.outer_begin + o), ce = __ldg(w.outer_begin + o + 1);
        if (cb >= ce) continue;
        if (g.od < d) {
            const int* keys = w.cell_dims + (size_t)g.od * g.ns;
            cb = lower_bound_i(keys, cb, ce, gi[g.od] - rad - 1);
            ce = lower_bound_i(keys, cb, ce, gi[g.od] + rad + 2);
        }
        for (int c = cb; c < ce; c++)
            if (!fn(c)) return;
    }
}

// MBR_in_eps (EGG_SynC.cu:1037-1159) by the reference's walk: per dimension
// the coordinate of q's eps/2 group with the smallest squared distance to p.
template <int D>
__device__ bool mbr_exact(const Geom& g, const Work& w, int qi, const float* xp) {
    constexpr int DM = D > 0 ? D : kMaxDims;
    const int d = D > 0 ? D : g.d;
    float xq[DM], mbr[DM];
    int gq[DM];
    int obase = 0;
    for (int l = 0; l < d; l++) {
        xq[l] = w.X[(size_t)l * g.ns + qi];
        mbr[l] = xq[l];
        gq[l] = cell_dim(xq[l], g);
        if (l < g.od) obase += gq[l] * g.wpow[l];
    }
    for_stencil_cells(g, w, 2, g.r_half, gq, obase, d, [&](int c) {
        float sm2 = 0.f, lg2 = 0.f;
        for (int l = 0; l < d; l++) box_terms(xq[l], __ldg(w.cell_dims + (size_t)l * g.ns + c), g.side, sm2, lg2);
        if (!(sm2 <= g.t_half)) return true;
        const int qb = __ldg(w.cell_start + c), qe = __ldg(w.cell_start + c + 1);
        for (int r = qb; r < qe; r++) {
            float d2 = 0.f;
            for (int l = 0; l < d; l++) d2 = dist_step(xq[l], __ldg(w.X + (size_t)l * g.ns + r), d2);
            if (d2 <= g.t_half) {
                for (int l = 0; l < d; l++) {
                    const float xr = __ldg(w.X + (size_t)l * g.ns + r);
                    float od_ = __fsub_rn(mbr[l], xp[l]);
                    od_ = __fmul_rn(od_, od_);
                    float nd = __fsub_rn(xr, xp[l]);
                    nd = __fmul_rn(nd, nd);
                    if (nd < od_) mbr[l] = xr;
                }
            }
        }
        return true;
    });
    float acc = 0.f;
    for (int l = 0; l < d; l++) acc = dist_step(mbr[l], xp[l], acc);
    return acc <= g.t_eps;
}

}  // namespace

// Every point of cell c has the same coordinates (its tight box is a
// point): they take the same steps in each kernel of the check, so one of
// them (the cell's first) stands for all.  Near convergence nearly every
// cell is such a collapsed cluster (1M x 3D: 41,646 of 41,660 final cells,
// holding all but 44 points).
__device__ __forceinline__ bool cell_degenerate(const Geom& g, const Work& w, int c, int d) {
    for (int l = 0; l < d; l++)
        if (__ldg(w.cbmin + (size_t)l * g.ns + c) != __ldg(w.cbmax + (size_t)l * g.ns + c)) return false;
    return true;
}

// extremes of each point's eps/2 group (itself included)
template <int D>
__device__ __forceinline__ void ball_bbox_body(const Geom& g, const Work& w, int bx, int gx, int mark = 1) {
    constexpr int DM = D > 0 ? D : kMaxDims;
    const int d = D > 0 ? D : g.d;
    if (mark && bx == 0 && threadIdx.x == 0) {
        const int it = w.ctrl[kCtrlIter];
        w.stamps[4 * it + 2] = globaltimer();
        // the extra check runs in this iteration when the flag reached it
        // (only the annulus kernel, launched after this one, clears the flag)
        if (w.ctrl[kCtrlFlag] != 0) atomicAdd(w.ctrl + kCtrlExtraRuns, 1);
    }
    if (w.ctrl[kCtrlFlag] == 0) return;
    for (int i = bx * blockDim.x + threadIdx.x; i < g.n; i += gx * blockDim.x) {
        // in a collapsed cell only the first point's extremes are read
        const int ci = w.cell_of[i];
        if (i != w.cell_start[ci] && cell_degenerate(g, w, ci, d)) continue;
        float xq[DM], lo[DM], hi[DM];
        int gq[DM];
        int obase = 0;
        for (int l = 0; l < d; l++) {
            xq[l] = w.X[(size_t)l * g.ns + i];
            lo[l] = hi[l] = xq[l];
            gq[l] = cell_dim(xq[l], g);
            if (l < g.od) obase += gq[l] * g.wpow[l];
        }
        for_stencil_cells(g, w, 2, g.r_half, gq, obase, d, [&](int c) {
            float sm2 = 0.f, lg2 = 0.f;
            for (int l = 0; l < d; l++)
                box_terms(xq[l], __ldg(w.cell_dims + (size_t)l * g.ns + c), g.side, sm2, lg2);
            if (!(sm2 <= g.t_half)) return true;
            // none / all of the cell's points inside the eps/2 ball?
            float near2, far2;
            tight_box_dist2(xq, w.cbmin + c, w.cbmax + c, g.ns, d, near2, far2);
            if (near2 > g.t_half) return true;
            if (far2 <= g.t_half) {
                for (int l = 0; l < d; l++) {
                    lo[l] = fminf(lo[l], __ldg(w.cbmin + (size_t)l * g.ns + c));
                    hi[l] = fmaxf(hi[l], __ldg(w.cbmax + (size_t)l * g.ns + c));
                }
                return true;
            }
            const int qb = __ldg(w.cell_start + c), qe = __ldg(w.cell_start + c + 1);
            for (int r = qb; r < qe; r++) {
                float d2 = 0.f;
                for (int l = 0; l < d; l++) d2 = dist_step(xq[l], __ldg(w.X + (size_t)l * g.ns + r), d2);
                if (d2 <= g.t_half)
                    for (int l = 0; l < d; l++) {
                        const float v = __ldg(w.X + (size_t)l * g.ns + r);
                        lo[l] = fminf(lo[l], v);
                        hi[l] = fmaxf(hi[l], v);
                    }
            }
            return true;
        });
        for (int l = 0; l < d; l++) {
            w.qlo[(size_t)l * g.ns + i] = lo[l];
            w.qhi[(size_t)l * g.ns + i] = hi[l];
        }
    }
}

// Union over a cell's points of their eps/2-group extremes.  The MBR of any
// pair (p, q) with q in the cell lies inside it, so its distance to p is a
// lower bound for every pair of the cell.  One warp per cell (collapsed
// clusters hold tens of thousands of points); min and max do not depend on
// the order of their operands, so the result is the serial one.
__device__ __forceinline__ void cell_ballbox_body(const Geom& g, const Work& w, int bx, int gx) {
    if (w.ctrl[kCtrlFlag] == 0) return;
    const int M = w.ctrl[kCtrlM];
    const int lane = threadIdx.x & 31, wpb = blockDim.x >> 5;
    for (int c = bx * wpb + (threadIdx.x >> 5); c < M; c += gx * wpb) {
        const int qb = w.cell_start[c], qe = w.cell_start[c + 1];
        const bool deg = cell_degenerate(g, w, c, g.d);
        for (int l = 0; l < g.d; l++) {
            float lo, hi;
            if (deg) {
                lo = w.qlo[(size_t)l * g.ns + qb];
                hi = w.qhi[(size_t)l * g.ns + qb];
            } else {
                lo = 3.0e38f;
                hi = -3.0e38f;
                for (int q = qb + lane; q < qe; q += 32) {
                    lo = fminf(lo, w.qlo[(size_t)l * g.ns + q]);
                    hi = fmaxf(hi, w.qhi[(size_t)l * g.ns + q]);
                }
#pragma unroll
                for (int o = 16; o > 0; o >>= 1) {
                    lo = fminf(lo, __shfl_xor_sync(0xffffffffu, lo, o));
                    hi = fmaxf(hi, __shfl_xor_sync(0xffffffffu, hi, o));
                }
            }
            if (lane == 0) {
                w.ulo[(size_t)l * g.ns + c] = lo;
                w.uhi[(size_t)l * g.ns + c] = hi;
            }
        }
    }
}

template <int D>
__device__ __forceinline__ void annulus_body(const Geom& g, const Work& w, int bx, int gx) {
    constexpr int DM = D > 0 ? D : kMaxDims;
    const int d = D > 0 ? D : g.d;
    volatile int* flag = w.ctrl + kCtrlFlag;
    if (*flag == 0) return;
    int pairs = 0;
    for (int i = bx * blockDim.x + threadIdx.x; i < g.n; i += gx * blockDim.x) {
        // a point of a collapsed cell finds what the cell's first point finds
        const int cp = w.cell_of[i];
        const int pb = w.cell_start[cp];
        const bool pdeg = cell_degenerate(g, w, cp, d);
        if (pdeg && i != pb) continue;
        const int pw = pdeg ? w.cell_start[cp + 1] - pb : 1;  // points it stands for (pair count)
        float xp[DM];
        int gp[DM];
        int obase = 0;
        for (int l = 0; l < d; l++) {
            xp[l] = w.X[(size_t)l * g.ns + i];
            gp[l] = cell_dim(xp[l], g);
            if (l < g.od) obase += gp[l] * g.wpow[l];
        }
        bool violated = false;
        for_stencil_cells(g, w, 1, g.r_extra, gp, obase, d, [&](int c) {
            if (*flag == 0) return false;
            float sm2 = 0.f, lg2 = 0.f;
            for (int l = 0; l < d; l++)
                box_terms(xp[l], __ldg(w.cell_dims + (size_t)l * g.ns + c), g.side, sm2, lg2);
            const bool included = sm2 <= g.t_extra;
            const bool fully = lg2 <= g.t_eps;
            if (!included || fully) return true;
            float near2, far2;
            tight_box_dist2(xp, w.cbmin + c, w.cbmax + c, g.ns, d, near2, far2);
            if (near2 > g.t_extra || far2 <= g.t_eps) return true;
            float lb2, ub2;
            tight_box_dist2(xp, w.ulo + c, w.uhi + c, g.ns, d, lb2, ub2);
            if (lb2 > g.t_eps) return true;  // no pair of this cell can have its MBR within eps
            const int qb = __ldg(w.cell_start + c), qe = __ldg(w.cell_start + c + 1);
            // a collapsed cell: its first point decides for all of them
            const bool qdeg = cell_degenerate(g, w, c, d);
            const int qend = qdeg ? qb + 1 : qe;
            for (int q = qb; q < qend; q++) {
                float d2 = 0.f;
                for (int l = 0; l < d; l++) d2 = dist_step(xp[l], __ldg(w.X + (size_t)l * g.ns + q), d2);
                if (!(d2 > g.t_eps && d2 <= g.t_extra)) continue;
                pairs += pw * (qdeg ? qe - qb : 1);
                bool resolved = true;
                float acc = 0.f;
                for (int l = 0; l < d; l++) {
                    const float lo = __ldg(w.qlo + (size_t)l * g.ns + q), hi = __ldg(w.qhi + (size_t)l * g.ns + q);
                    float m;
                    if (xp[l] >= hi) m = hi;
                    else if (xp[l] <= lo) m = lo;
                    else { resolved = false; break; }
                    acc = dist_step(m, xp[l], acc);
                }
                const bool in_eps = resolved ? (acc <= g.t_eps) : mbr_exact<D>(g, w, q, xp);
                if (in_eps) {
                    violated = true;
                    *flag = 0;
                    return false;
                }
            }
            return true;
        });
        if (violated || *flag == 0) break;
    }
    if (pairs) atomicAdd(w.ctrl + kCtrlPairs, pairs);
}

template <int D>
__global__ void __launch_bounds__(128) k_ball_bbox(Geom g, Work w, int mark) {
    ball_bbox_body<D>(g, w, blockIdx.x, gridDim.x, mark);
}
template <int D>
__global__ void __launch_bounds__(128) kb_ball_bbox(BatchArgs B, int mark) {
    batch_for(B, [&](const Geom& g, const Work& w, int bx, int gx) { ball_bbox_body<D>(g, w, bx, gx, mark); });
}
__global__ void __launch_bounds__(256) k_cell_ballbox(Geom g, Work w) { cell_ballbox_body(g, w, blockIdx.x, gridDim.x); }
__global__ void __launch_bounds__(256) kb_cell_ballbox(BatchArgs B) {
    batch_for(B, [&](const Geom& g, const Work& w, int bx, int gx) { cell_ballbox_body(g, w, bx, gx); });
}
template <int D>
__global__ void __launch_bounds__(128) k_annulus(Geom g, Work w) { annulus_body<D>(g, w, blockIdx.x, gridDim.x); }
template <int D>
__global__ void __launch_bounds__(128) kb_annulus(BatchArgs B) {
    batch_for(B, [&](const Geom& g, const Work& w, int bx, int gx) { annulus_body<D>(g, w, bx, gx); });
}

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

// Opens the conditional node holding the extra check when the update left
// the flag at 1 (the loop graph of a single instance), with the stage stamp
// and the run count the first extra-check kernel keeps otherwise.
__global__ void k_gate_extra(Work w, cudaGraphConditionalHandle h) {
    const int it = w.ctrl[kCtrlIter];
    w.stamps[4 * it + 2] = globaltimer();
    const int flag = w.ctrl[kCtrlFlag];
    if (flag != 0) atomicAdd(w.ctrl + kCtrlExtraRuns, 1);
    cudaGraphSetConditional(h, flag != 0 ? 1u : 0u);
}

void launch_gate_extra(const Work& w, cudaGraphConditionalHandle h, cudaStream_t st) {
    k_gate_extra<<<1, 1, 0, st>>>(w, h);
}

// The same for one dimension group of a batched loop: one thread per active
// instance stamps the stage and counts a flagged instance's extra check; the
// node opens when any of them has its flag at 1.
__global__ void __launch_bounds__(1024) k_batch_gate_extra(const Work* __restrict__ works,
                                                           const int* __restrict__ active, const int* __restrict__ nact,
                                                           cudaGraphConditionalHandle h) {
    const int na = *nact;
    const unsigned long long now = globaltimer();
    int flagged = 0;
    for (int t = threadIdx.x; t < na; t += blockDim.x) {
        const Work& w = works[active[t]];
        const int it = w.ctrl[kCtrlIter];
        w.stamps[4 * it + 2] = now;
        if (w.ctrl[kCtrlFlag] != 0) {
            atomicAdd(w.ctrl + kCtrlExtraRuns, 1);
            flagged = 1;
        }
    }
    const int any = __syncthreads_or(flagged);
    if (threadIdx.x == 0) cudaGraphSetConditional(h, any ? 1u : 0u);
}

void launch_batch_gate_extra(const Exec& ex, cudaGraphConditionalHandle h, cudaStream_t st) {
    k_batch_gate_extra<<<1, 1024, 0, st>>>(ex.bt->works, ex.bt->active, ex.bt->nact, h);
}

// Opens the grid-sort node of one dimension group when the grid check found
// a point that left its cell in any of the group's active instances (for
// the others the sort kernels would return at once); counts the openings.
__global__ void __launch_bounds__(1024) k_batch_gate_sort(const Work* __restrict__ works,
                                                          const int* __restrict__ active, const int* __restrict__ nact,
                                                          int* __restrict__ opened, cudaGraphConditionalHandle h) {
    const int na = *nact;
    int changed = 0;
    for (int t = threadIdx.x; t < na; t += blockDim.x) changed |= works[active[t]].ctrl[kCtrlChanged] != 0;
    const int any = __syncthreads_or(changed);
    if (threadIdx.x == 0) {
        if (any) *opened += 1;
        cudaGraphSetConditional(h, any ? 1u : 0u);
    }
}

void launch_batch_gate_sort(const Exec& ex, cudaGraphConditionalHandle h, int* opened, cudaStream_t st) {
    k_batch_gate_sort<<<1, 1024, 0, st>>>(ex.bt->works, ex.bt->active, ex.bt->nact, opened, h);
}

// The kernels return at once unless the update left the flag at 1; the
// grids are bounded so that the common early exit costs little.  gated: the
// call sits behind k_gate_extra, which did the stage stamp and the count.
void launch_extra_check(const Exec& ex, cudaStream_t st, bool gated) {
    const int blocks = ex.blocks(kShapeCapN128, 128);
    if (ex.batch()) {
        const BatchArgs B = ex.args(kShapeCapN128);
        EGG_DISPATCH_D(ex.d, kb_ball_bbox, <<<blocks, 128, 0, st>>>(B, gated ? 0 : 1));
        kb_cell_ballbox<<<ex.blocks(kShapeCapN128, 256), 256, 0, st>>>(B);
        EGG_DISPATCH_D(ex.d, kb_annulus, <<<blocks, 128, 0, st>>>(B));
    } else {
        EGG_DISPATCH_D(ex.d, k_ball_bbox, <<<blocks, 128, 0, st>>>(*ex.g, *ex.w, gated ? 0 : 1));
        k_cell_ballbox<<<blocks, 256, 0, st>>>(*ex.g, *ex.w);
        EGG_DISPATCH_D(ex.d, k_annulus, <<<blocks, 128, 0, st>>>(*ex.g, *ex.w));
    }
}

}  // namespace egg
