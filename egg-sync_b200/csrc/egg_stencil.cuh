// egg_stencil.cuh -- candidate-cell enumeration shared by the per-point kernels.
//
// For a point with cell dims gi (outer id obase) the candidate cells are the
// inner cells of the outer cells in the box stencil [-r, r]^od (the
// reference's pre-grid, EGG_SynC.cu:386-536), restricted in dimension od to
// [gi_od - r - 1, gi_od + r + 1]: cells beyond fail the reference's box test
// in exact and rounded arithmetic alike (their gap exceeds (r+1)*side > eps).
//
// Must be called by all 32 lanes of a warp.  When every lane has the same
// outer cell and their cells in dimension od lie within kLockZSpan of each
// other, the warp resolves the stencil entries in parallel (lane = entry)
// and visits each candidate cell with all lanes in lockstep (the cell
// records become broadcast loads); otherwise each lane walks its own stencil
// (the lockstep window in dimension od is the union of the lanes' windows, so
// lanes spread along od would each test many cells that only others need).
// Both paths give every lane the same results bit for bit: the extra cells
// of the union fail that lane's box test.
// fn(c) is called once per candidate cell per lane, in increasing stencil
// entry then increasing cell order in both paths.  A lane for which
// active() is false needs no result: it rides along in the lockstep path
// and skips its own walk in the other (active() is evaluated there only, so
// the lockstep path carries nothing extra).
//
// In a lane's own walk with od < d, an outer cell none of whose blocks of
// dimension od (colmask) meets the lane's z-window holds no candidate: it is
// passed over without the two binary searches (the same empty range they
// would give).

#pragma once

#include "egg_common.cuh"

namespace egg {

// warps whose cells in dimension od span more than this take the per-lane walk
// (1M x 3D: 96.4 -> 95.5 ms against lockstep for every single-column warp)
constexpr int kLockZSpan = 4;

// colmask bits of the blocks meeting the cells [zl, zh] of dimension od
__device__ __forceinline__ unsigned long long zwindow_mask(const Geom& g, int zl, int zh) {
    const int bl = max(0, zl) / g.zblk, bh = min(g.width - 1, zh) / g.zblk;
    return (2ull << bh) - (1ull << bl);  // bits bl..bh (bh = 63 wraps to the right value)
}

template <typename A, typename F>
__device__ __forceinline__ void for_candidates(const Geom& g, const Work& w, const int* gi, int obase, int lane,
                                               int d, A&& active, F&& fn) {
    const int nst = w.st_count[0];
    const int ob0 = __shfl_sync(0xffffffffu, obase, 0);
    int zlo = 0, zhi = 0;
    if (g.od < d) {
        zlo = zhi = gi[g.od];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            zlo = min(zlo, __shfl_xor_sync(0xffffffffu, zlo, o));
            zhi = max(zhi, __shfl_xor_sync(0xffffffffu, zhi, o));
        }
    }
    if (__all_sync(0xffffffffu, obase == ob0) && zhi - zlo <= kLockZSpan) {
        for (int s0 = 0; s0 < nst; s0 += 32) {
            const int s = s0 + lane;
            int cb = 0, ce = 0;
            if (s < nst) {
                bool inb = true;
                for (int l = 0; l < g.od; l++) {
                    const int v = gi[l] + __ldg(w.st_off + (size_t)s * g.od + l);
                    inb = inb && (unsigned)v < (unsigned)g.width;
                }
                if (inb) {
                    const int o = obase + __ldg(w.st_delta + s);
                    cb = __ldg(w.outer_begin + o);
                    ce = __ldg(w.outer_begin + o + 1);
                    if (cb < ce && g.od < d) {
                        const int* keys = w.cell_dims + (size_t)g.od * g.ns;
                        cb = lower_bound_i(keys, cb, ce, zlo - g.r - 1);
                        ce = lower_bound_i(keys, cb, ce, zhi + g.r + 2);
                    }
                }
            }
            unsigned live = __ballot_sync(0xffffffffu, cb < ce);
            while (live) {
                const int src = __ffs(live) - 1;
                live &= live - 1;
                const int b = __shfl_sync(0xffffffffu, cb, src);
                const int e = __shfl_sync(0xffffffffu, ce, src);
                for (int c = b; c < e; c++) fn(c);
            }
        }
    } else {
        if (!active()) return;  // no warp-wide operation below
        // each lane walks its own stencil; the column masks of four entries
        // are loaded together, so most columns cost a quarter of a load
        constexpr int kAhead = 4;
        const bool zs = g.od < d && w.colmask != nullptr;
        const unsigned long long wm = zs ? zwindow_mask(g, gi[g.od] - g.r - 1, gi[g.od] + g.r + 1) : 0ull;
        for (int s0 = 0; s0 < nst; s0 += kAhead) {
            int ol[kAhead];
#pragma unroll
            for (int k = 0; k < kAhead; k++) {
                const int s = s0 + k;
                ol[k] = -1;
                if (s < nst) {
                    bool inb = true;
                    for (int l = 0; l < g.od; l++) {
                        const int v = gi[l] + __ldg(w.st_off + (size_t)s * g.od + l);
                        inb = inb && (unsigned)v < (unsigned)g.width;
                    }
                    const int o = obase + __ldg(w.st_delta + s);
                    if (inb && zs) inb = (__ldg(w.colmask + o) & wm) != 0;
                    if (inb) ol[k] = o;
                }
            }
#pragma unroll 1
            for (int k = 0; k < kAhead; k++) {
                const int o = ol[k];
                if (o < 0) continue;
                int cb = __ldg(w.outer_begin + o), ce = __ldg(w.outer_begin + o + 1);
                if (cb >= ce) continue;
                if (g.od < d) {
                    const int* keys = w.cell_dims + (size_t)g.od * g.ns;
                    cb = lower_bound_i(keys, cb, ce, gi[g.od] - g.r - 1);
                    ce = lower_bound_i(keys, cb, ce, gi[g.od] + g.r + 2);
                }
                for (int c = cb; c < ce; c++) fn(c);
            }
        }
    }
}

}  // namespace egg
