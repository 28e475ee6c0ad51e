// egg_update.cu -- eps-ball synchronisation update + convergence flag.
//
// Replaces kernel_itr_grid_STAD5_5_1 of the reference
// (src/algorithms/EGG_SynC.cu:551-763) together with its pre-grid of
// neighbour outer cells (EGG_SynC.cu:368-536), which the dense outer_begin
// array makes unnecessary.
//
// For point p with own-cell corner c (c_l = g_l * side) and phi = x_p - c:
//   sum_{q in N(p)} sin(x_q - x_p) = cos(phi) * S - sin(phi) * (N - Cm)
// with S = sum sin(x_q - c), Cm = sum (1 - cos(x_q - c)), N = |N(p)|.
// A neighbour cell with dim ids g' (k = g' - g) whose points have offsets
// delta_q = x_q - g' * side contributes, through sin/cos tables of k * side,
//   S  += sin(k s) * (m - SM) + cos(k s) * SS
//   Cm += m * (1 - cos(k s)) + cos(k s) * SM + sin(k s) * SS
// where SS = sum sin(delta), SM = sum (1 - cos(delta)) over the counted
// points (the whole cell when it lies inside the eps-ball, the points that
// pass the distance test otherwise).  Every term is a small, well-conditioned
// quantity, so the FP32 result stays within ~1e-7 of the exact FP64 update.
//
// Cell classification, distance tests, the border rule and the flag follow
// the reference exactly (EGG_SynC.cu:583-597, 613-636, 666-681, 706-709).
#include "egg_common.cuh"
#include "egg_kernels.h"
#include "egg_stencil.cuh"

namespace egg {

namespace {

// reference half_count (EGG_SynC.cu:666-681) for a border point whose
// neighbourhood holds other fully covered cells: own cell plus the points
// within eps/2 in the other fully covered cells.
template <int D>
__device__ int half_count(const Geom& g, const Work& w, const float* x, const int* gi, int obase, int own, int own_cnt) {
    constexpr int DM = D > 0 ? D : kMaxDims;
    const int d = D > 0 ? D : g.d;
    int half = own_cnt;
    const int nst = w.st_count[0];
    for (int s = 0; s < nst; s++) {
        bool inb = true;
        for (int l = 0; l < g.od; l++) {
            int v = gi[l] + w.st_off[(size_t)s * g.od + l];
            inb = inb && (unsigned)v < (unsigned)g.width;
        }
        if (!inb) continue;
        const int o = obase + w.st_delta[s];
        int cb = w.outer_begin[o], ce = w.outer_begin[o + 1];
        if (cb >= ce) continue;
        if (g.od < d) {
            const int* keys = w.cell_dims + (size_t)g.od * g.ns;
            cb = lower_bound_i(keys, cb, ce, gi[g.od] - g.r - 1);
            ce = lower_bound_i(keys, cb, ce, gi[g.od] + g.r + 2);
        }
        for (int c = cb; c < ce; c++) {
            if (c == own) continue;
            float sm2 = 0.f, lg2 = 0.f;
            for (int l = 0; l < d; l++) box_terms(x[l], __ldg(w.cell_dims + (size_t)l * g.ns + c), g.side, sm2, lg2);
            if (!(lg2 <= g.t_eps)) continue;
            const int qb = __ldg(w.cell_start + c), qe = __ldg(w.cell_start + c + 1);
            float near2, far2;
            tight_box_dist2(x, w.cbmin + c, w.cbmax + c, g.ns, d, near2, far2);
            if (near2 > g.t_half) continue;
            if (far2 <= g.t_half) {
                half += qe - qb;
                continue;
            }
            for (int q = qb; q < qe; q++) {
                float d2 = 0.f;
                for (int l = 0; l < d; l++) d2 = dist_step(__ldg(w.X + (size_t)l * g.ns + q), x[l], d2);
                half += (d2 <= g.t_half);
            }
        }
    }
    (void)DM;
    return half;
}

}  // namespace

namespace {

#ifdef EGG_UPDATE_STATS
#define EGG_STAT(a, k, v) ((a).st[k] += (v))
#else
#define EGG_STAT(a, k, v) ((void)0)
#endif

template <int D>
struct Acc {
    float S[D > 0 ? D : kMaxDims];
    float Cm[D > 0 ? D : kMaxDims];
    int N;
    int partial_in;
    bool tab_err;
#ifdef EGG_UPDATE_STATS
    unsigned st[kUStats];
#endif
};

// m counted points of a cell at offsets k (= cell dims - own dims) with
// SS = sum sin(delta), SM = sum (1 - cos(delta)) into the own-cell frame.
template <int D>
__device__ __forceinline__ void add_counted(Acc<D>& a, int d, const int* kk, float m, const float* SS, const float* SM,
                                            const float* Ts, const float* Tc, const float* Tm, int K, int TW) {
    for (int l = 0; l < d; l++) {
        int k = kk[l] + K;
        if ((unsigned)k >= (unsigned)TW) { a.tab_err = true; k = K; }
        const float ts = Ts[k], tc = Tc[k], tm = Tm[k];
        a.S[l] += ts * (m - SM[l]) + tc * SS[l];
        a.Cm[l] += m * tm + tc * SM[l] + ts * SS[l];
    }
}

// One candidate cell for one point: the reference's box test
// (EGG_SynC.cu:613-636), then the aggregate (fully covered, or all points
// provably within eps), nothing (no point provably within eps), or a walk.
template <int D>
__device__ __forceinline__ void visit_cell(const Geom& g, const Work& w, int c, const float* x, const int* gi,
                                           Acc<D>& a, const float* Ts, const float* Tc, const float* Tm, int K, int TW) {
    constexpr int DM = D > 0 ? D : kMaxDims;
    const int d = D > 0 ? D : g.d;
    float sm2 = 0.f, lg2 = 0.f;
    int kk[DM];
    if constexpr (D >= 1 && D <= 4) {
        // the cell's dims from one packed word
        const unsigned long long key = __ldg(w.cell_key + c);
#pragma unroll
        for (int l = 0; l < D; l++) {
            const int cd = (int)((key >> (16 * l)) & 0xffffu);
            box_terms(x[l], cd, g.side, sm2, lg2);
            kk[l] = cd - gi[l];
        }
    } else {
        for (int l = 0; l < d; l++) {
            const int cd = __ldg(w.cell_dims + (size_t)l * g.ns + c);
            box_terms(x[l], cd, g.side, sm2, lg2);
            kk[l] = cd - gi[l];
        }
    }
    EGG_STAT(a, kUsCells, 1);
    if (!(sm2 <= g.t_eps)) return;
    EGG_STAT(a, kUsSmallPass, 1);
    const int qb = __ldg(w.cell_start + c), qe = __ldg(w.cell_start + c + 1);
    bool all_in = lg2 <= g.t_eps;
    const bool full = all_in;
    if (!full) {
        float near2, far2;
        tight_box_dist2(x, w.cbmin + c, w.cbmax + c, g.ns, d, near2, far2);
        if (near2 > g.t_eps) {
            EGG_STAT(a, kUsTightOut, 1);
            return;
        }
        all_in = far2 <= g.t_eps;
        if (all_in) EGG_STAT(a, kUsTightIn, 1);
    } else {
        EGG_STAT(a, kUsFull, 1);
    }
    if (all_in) {
        float SS[DM], SM[DM];
        for (int l = 0; l < d; l++) {
            SS[l] = __ldg(w.css + (size_t)l * g.ns + c);
            SM[l] = __ldg(w.csm + (size_t)l * g.ns + c);
        }
        add_counted<D>(a, d, kk, (float)(qe - qb), SS, SM, Ts, Tc, Tm, K, TW);
        a.N += qe - qb;
        if (!full) a.partial_in += qe - qb;
        return;
    }
    float as[DM], am[DM];
    for (int l = 0; l < d; l++) { as[l] = 0.f; am[l] = 0.f; }
    int cnt = 0;
    const int kh = qb >> 5, kt = (qe - 1) >> 5;
    for (int k = kh; k <= kt; k++) {
        // the cell's points in warp k: one 32-point group of a cell ordered
        // along the sub-cell curve; its tight box decides it wholesale when
        // all or none of its points are within eps
        const int sb = max(qb, k << 5), se = min(qe, (k << 5) + 32);
        if (kh != kt) {
            const int nw = (g.n + 31) >> 5;
            const int rec = (k == kh) ? 1 : 0;
            float n2 = 0.f, f2 = 0.f;
            for (int l = 0; l < d; l++) {
                const float L = __ldg(w.gpart + wp_idx_f(2, l, d, rec, nw, k));
                const float H = __ldg(w.gpart + wp_idx_f(3, l, d, rec, nw, k));
                const float a0 = near_gap(x[l], L, H), b0 = far_gap(x[l], L, H);
                n2 = __fmaf_rn(a0, a0, n2);
                f2 = __fmaf_rn(b0, b0, f2);
            }
            if (n2 > g.t_eps) {
                EGG_STAT(a, kUsGroupsOut, 1);
                continue;
            }
            if (f2 <= g.t_eps) {
                EGG_STAT(a, kUsGroupsIn, 1);
                for (int l = 0; l < d; l++) {
                    as[l] += __ldg(w.gpart + wp_idx_f(0, l, d, rec, nw, k));
                    am[l] += __ldg(w.gpart + wp_idx_f(1, l, d, rec, nw, k));
                }
                cnt += se - sb;
                continue;
            }
        }
        EGG_STAT(a, kUsPairs, se - sb);
        if constexpr (D >= 1 && D <= kPackDims) {
            // packed records: one or two 16-byte loads per candidate point
            constexpr int PW = pack_w(D > 0 ? D : 1), PS = pack_s(D > 0 ? D : 1);
            const float4* xp = w.xp + (size_t)sb * PW;
            const float4* sp = w.smp + (size_t)sb * PS;
            for (int q = sb; q < se; q++, xp += PW, sp += PS) {
#ifdef EGG_UPDATE_STATS
                {
                    const unsigned am_ = __activemask();
                    if ((threadIdx.x & 31) == __ffs(am_) - 1) a.st[kUsWalkSteps] += 1;
                }
#endif
                float xq[4 * PW];
#pragma unroll
                for (int k = 0; k < PW; k++) {
                    const float4 v = __ldg(xp + k);
                    xq[4 * k] = v.x;
                    xq[4 * k + 1] = v.y;
                    xq[4 * k + 2] = v.z;
                    xq[4 * k + 3] = v.w;
                }
                float d2 = 0.f;
#pragma unroll
                for (int l = 0; l < DM; l++) d2 = dist_step(xq[l], x[l], d2);
                if (d2 <= g.t_eps) {
                    float v[4 * PS];
#pragma unroll
                    for (int k = 0; k < PS; k++) {
                        const float4 t = __ldg(sp + k);
                        v[4 * k] = t.x;
                        v[4 * k + 1] = t.y;
                        v[4 * k + 2] = t.z;
                        v[4 * k + 3] = t.w;
                    }
#pragma unroll
                    for (int l = 0; l < DM; l++) {
                        as[l] += v[l];
                        am[l] += v[DM + l];
                    }
                    cnt++;
                }
            }
        } else {
            for (int q = sb; q < se; q++) {
                float d2 = 0.f;
                for (int l = 0; l < d; l++) d2 = dist_step(__ldg(w.X + (size_t)l * g.ns + q), x[l], d2);
                if (d2 <= g.t_eps) {
                    for (int l = 0; l < d; l++) {
                        as[l] += __ldg(w.sd + (size_t)l * g.ns + q);
                        am[l] += __ldg(w.md + (size_t)l * g.ns + q);
                    }
                    cnt++;
                }
            }
        }
    }
    if (cnt) {
        add_counted<D>(a, d, kk, (float)cnt, as, am, Ts, Tc, Tm, K, TW);
        a.N += cnt;
        a.partial_in += cnt;
    }
    EGG_STAT(a, kUsPairsIn, cnt);
}

}  // namespace

// One thread per cell-sorted point.  When the 32 points of a warp share one
// outer cell (the common case: sorted points are grouped by outer cell), the
// warp resolves the stencil's outer cells in parallel (lane = stencil entry)
// and then visits every candidate cell with all lanes in lockstep, so cell
// records are broadcast loads and the dependent-load chain of the stencil
// walk is paid once per warp instead of once per point.  Otherwise each lane
// walks the stencil on its own.  Both paths visit a superset of the cells
// the reference visits and apply the reference's per-point box test to each.
template <int D>
__device__ __forceinline__ void update_body(const Geom& g, const Work& w, int* __restrict__ counts, int bx) {
    constexpr int DM = D > 0 ? D : kMaxDims;
    const int d = D > 0 ? D : g.d;
    extern __shared__ float s_tab[];
    const int K = g.table_k, TW = 2 * K + 1;
    const int i = bx * blockDim.x + threadIdx.x;
    const int lane = threadIdx.x & 31;
    const bool valid = i < g.n;
    const int iv = valid ? i : g.n - 1;  // lanes past n shadow the last point; their results are dropped
    // the point and its warp's last violation bits are loaded before the
    // table's barrier, so their latency overlaps it (most warps late in a
    // run need nothing else)
    float x[DM];
    for (int l = 0; l < d; l++) x[l] = w.X[(size_t)l * g.ns + iv];
    const unsigned wv_last = (w.warp_viol && (i & ~31) < g.n) ? w.warp_viol[i >> 5] : 0u;
    for (int t = threadIdx.x; t < 3 * TW; t += blockDim.x) s_tab[t] = w.table[t];
    if (bx == 0 && threadIdx.x == 0) {
        const int it = w.ctrl[kCtrlIter];
        w.stamps[4 * it + 1] = globaltimer();
    }
    __syncthreads();
    if ((i & ~31) >= g.n) return;  // whole warp beyond n
    const float* Ts = s_tab;
    const float* Tc = s_tab + TW;
    const float* Tm = s_tab + 2 * TW;

    const int it = w.ctrl[kCtrlIter];
    int gi[DM];
    int obase = 0;
    for (int l = 0; l < d; l++) {
        gi[l] = cell_dim(x[l], g);
        if (l < g.od) obase += gi[l] * g.wpow[l];
    }

    // Incremental update: when no point of this warp has a moved point (old
    // or new position) anywhere in its stencil region since the last update,
    // every input of its update is unchanged, so the result is the same bit
    // for bit: keep the position and the last violation bit.
    const int zb = g.od < d ? gi[g.od] / g.zblk : 0;
    const bool need_me = w.ctrl[kCtrlForce] != 0 || ((w.need[obase] >> zb) & 1ull) != 0;
    // Xn equals X here unless this iteration rebuilt the grid (the grid check
    // copied Xn into X; a rebuild reorders X only): a kept position is
    // written back only after a rebuild (the control word is read where it
    // is used, so nothing extra stays live over the walk)
    // Without a rebuild the warp holds the same points as at its last update
    // and its violation bits stand; a rebuild reorders the points, so the
    // bits are gathered by original index and the warp's word rewritten.
    if (!__any_sync(0xffffffffu, need_me)) {
        unsigned vb = wv_last;
        if (w.ctrl[kCtrlChanged] != 0 || !w.warp_viol) {
            bool viol = false;
            if (valid) {
                for (int l = 0; l < d; l++) w.Xn[(size_t)l * g.ns + i] = x[l];
                viol = w.viol_orig[w.orig[i]] != 0;
            }
            vb = __ballot_sync(0xffffffffu, viol);
            if (lane == 0 && w.warp_viol) w.warp_viol[i >> 5] = vb;
        }
        if (lane == 0) {
            if (w.warp_moved) w.warp_moved[i >> 5] = 0;
            if (vb != 0) {
                volatile int* f = w.ctrl + kCtrlFlag;
                if (*f != 0) *f = 0;
            }
        }
        return;
    }
    // Within a warp that recomputes, a lane whose own region is clean keeps
    // its result too (same argument, per point): it does not walk when the
    // lanes walk separately (lanes in several outer cells), where the walks
    // of a warp's lanes run one after another.  The lane's need bit is read
    // again where it is used, so nothing extra stays live over the walk.
    auto lane_needs = [&]() {
        return counts != nullptr || w.ctrl[kCtrlForce] != 0 ||
               ((w.need[obase] >> (g.od < d ? gi[g.od] / g.zblk : 0)) & 1ull) != 0;
    };
    {
        const unsigned vm = __ballot_sync(0xffffffffu, valid && (need_me || counts != nullptr));
        if (lane == 0) atomicAdd(w.ctrl + kCtrlComputed, __popc(vm));
    }

    bool border = false;
    Acc<D> a;
    for (int l = 0; l < d; l++) {
        border |= on_border_dim(x[l], g.side);
        a.S[l] = 0.f;
        a.Cm[l] = 0.f;
    }
    a.N = 0;
    a.partial_in = 0;
    a.tab_err = false;
#ifdef EGG_UPDATE_STATS
    for (int k = 0; k < kUStats; k++) a.st[k] = 0;
    {
        // every lane takes part in the vote (a full-mask vote by one lane never completes)
        const int ob0 = __shfl_sync(0xffffffffu, obase, 0);
        const bool uniform = __all_sync(0xffffffffu, obase == ob0);
        if (lane == 0 && !uniform) a.st[kUsLaneWarps] = 1;
    }
#endif
    const int own = w.cell_of[iv];
    const int own_cnt = w.cell_start[own + 1] - w.cell_start[own];

#ifdef EGG_UPDATE_STATS
    const long long t_walk0 = clock64();
#endif
#ifdef EGG_UPDATE_STATS
    const bool ls_warp = a.st[kUsLaneWarps] == 0;  // meaningful in lane 0, which counts
    for_candidates(g, w, gi, obase, lane, d, lane_needs, [&](int c) {
        const long long tv = clock64();
        visit_cell<D>(g, w, c, x, gi, a, Ts, Tc, Tm, K, TW);
        if (lane == 0 && ls_warp) {
            a.st[kUsWarpVisits] += 1;
            a.st[kUsCyclesVisits] += (unsigned)(clock64() - tv);
        }
    });
#else
    for_candidates(g, w, gi, obase, lane, d, lane_needs,
                   [&](int c) { visit_cell<D>(g, w, c, x, gi, a, Ts, Tc, Tm, K, TW); });
#endif
#ifdef EGG_UPDATE_STATS
    {
        const long long dt = clock64() - t_walk0;
        const long long warp_dt = __reduce_max_sync(0xffffffffu, (unsigned)min(dt, 0x7fffffffLL));
        if (lane == 0) a.st[a.st[kUsLaneWarps] ? kUsCyclesLane : kUsCyclesShared] += (unsigned)warp_dt;
    }
#endif

    const bool walk = lane_needs();
    const int N = a.N;
    const float fN = (float)N;
    bool moved = false;
    int onew = 0, zbnew = 0;
    if (valid && !walk) {
        if (w.ctrl[kCtrlChanged] != 0)
            for (int l = 0; l < d; l++) w.Xn[(size_t)l * g.ns + i] = x[l];
    } else if (valid) {
        for (int l = 0; l < d; l++) {
            const float corner = __fmul_rn((float)gi[l], g.side);
            const float phi = x[l] - corner;
            float sp, cp;
            sincosf(phi, &sp, &cp);
            const float A = cp * a.S[l] - sp * (fN - a.Cm[l]);
            const float xn = x[l] + A / fN;
            w.Xn[(size_t)l * g.ns + i] = xn;
            moved |= __float_as_uint(xn) != __float_as_uint(x[l]);
            if (l < g.od) onew += cell_dim(xn, g) * g.wpow[l];
            if (l == g.od) zbnew = cell_dim(xn, g) / g.zblk;
        }
        if (counts) counts[i] = N;
    }

    // convergence flag, EGG_SynC.cu:706-709.  half_count <= N - partial_in,
    // so a border point with neighbours in a partial cell always violates.
    bool viol = false;
    if (valid && !walk) {
        viol = (w.ctrl[kCtrlChanged] != 0 || !w.warp_viol) ? w.viol_orig[w.orig[i]] != 0
                                                           : ((w.warp_viol[i >> 5] >> lane) & 1u) != 0;
    } else if (valid) {
        if (!border) viol = (N != own_cnt);
        else if (a.partial_in > 0) viol = true;
        else if (N == own_cnt) viol = false;
        else {
            viol = (N != half_count<D>(g, w, x, gi, obase, own, own_cnt));
            EGG_STAT(a, kUsHalfCount, 1);
        }
        w.viol_orig[w.orig[i]] = viol ? 1 : 0;
        if (moved) {
            unsigned long long* dcur = w.dirty[it & 1];
            atomicOr(dcur + obase, 1ull << zb);
            atomicOr(dcur + onew, 1ull << zbnew);
        }
    }
    // the warps whose points moved: the next grid check reads only those
    const bool warp_mv = __any_sync(0xffffffffu, moved);
    if (lane == 0 && w.warp_moved) w.warp_moved[i >> 5] = warp_mv ? 1 : 0;
    const unsigned vb = __ballot_sync(0xffffffffu, viol);
    if (lane == 0) {
        if (w.warp_viol) w.warp_viol[i >> 5] = vb;
        if (vb != 0) {
            volatile int* f = w.ctrl + kCtrlFlag;
            if (*f != 0) *f = 0;
        }
    }
    if (a.tab_err) atomicOr(w.ctrl + kCtrlStatus, kErrTable);
#ifdef EGG_UPDATE_STATS
    if (valid && walk) {
        a.st[kUsPoints] += 1;
        a.st[kUsNeighbors] += N;
    } else {
        // shadow lanes, and lanes that kept their result (their lockstep
        // visits are not work of the update)
        for (int k = 0; k < kUStats; k++)
            if (k != kUsLaneWarps && k != kUsCyclesShared && k != kUsCyclesLane && k != kUsWarpVisits &&
                k != kUsCyclesVisits && k != kUsWalkSteps)
                a.st[k] = 0;
    }
    for (int k = 0; k < kUStats; k++) {
        unsigned long long v = a.st[k];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        if (lane == 0 && v) atomicAdd(w.ustats + k, v);
    }
#endif
}

template <int D>
__global__ void __launch_bounds__(128) k_update(Geom g, Work w, int* __restrict__ counts) {
    update_body<D>(g, w, counts, blockIdx.x);
}

template <int D, int T>
__global__ void __launch_bounds__(T) kb_update(BatchArgs B) {
    batch_for(B, [&](const Geom& g, const Work& w, int bx, int) { update_body<D>(g, w, nullptr, bx); });
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

// need[] (zeroed by the grid-build check of this iteration) receives, over
// the stencil of every outer cell that the previous update marked dirty, the
// dirty blocks of dimension od widened by r + 1 cells on each side: exactly
// the points whose candidate cells (outer stencil, dimension od within
// r + 1 cells, for_candidates) can hold a moved point's old or new position.
// The dirty marks are cleared as they are consumed, so the array is clean
// again when the update after next writes it.
// A warp reads kNeedChunk outer cells at once; the lanes share the stencil
// entries of each dirty one (dirty cells cluster around the regions still
// moving, so a long run of them per warp would hold the whole launch).
// The dilation is closed-form: block b covers the blocks
// [b - ceil((r+1)/zblk), b + 1 + floor(r/zblk)], clipped to [0, nzb).
constexpr int kNeedChunk = 8;

__device__ __forceinline__ void need_body(const Geom& g, const Work& w, int bx, int gx) {
    const int it = w.ctrl[kCtrlIter];
    unsigned long long* prev = w.dirty[(it + 1) & 1];
    const int nst = w.st_count[0];
    const int lane = threadIdx.x & 31;
    const int wpb = blockDim.x >> 5;
    const int lo_sh = min(63, (g.r + g.zblk) / g.zblk), hi_sh = min(63, 1 + g.r / g.zblk);
    const unsigned long long full = g.nzb >= 64 ? ~0ull : (1ull << g.nzb) - 1ull;
    const long long stride = (long long)gx * wpb * kNeedChunk;
    // warp-uniform loop over chunks of outer cells
    for (long long o0 = ((long long)bx * wpb + (threadIdx.x >> 5)) * kNeedChunk; o0 < g.n_outer; o0 += stride) {
        const long long o = o0 + lane;
        const unsigned long long mine = (lane < kNeedChunk && o < g.n_outer) ? prev[o] : 0ull;
        if (mine) prev[o] = 0;
        unsigned todo = __ballot_sync(0xffffffffu, mine != 0);
        while (todo) {
            const int src = __ffs(todo) - 1;
            todo &= todo - 1;
            const unsigned long long m = __shfl_sync(0xffffffffu, mine, src);
            const int oc = (int)o0 + src;
            unsigned long long dil = 0;
            for (int s = 0; s <= lo_sh; s++) dil |= m >> s;
            for (int s = 1; s <= hi_sh; s++) dil |= m << s;
            dil &= full;
            int co[32];
            int rem = oc;
            for (int l = 0; l < g.od; l++) {
                co[l] = rem % g.width;
                rem /= g.width;
            }
            for (int s = lane; s < nst; s += 32) {
                bool inb = true;
                for (int l = 0; l < g.od; l++) {
                    const int v = co[l] + __ldg(w.st_off + (size_t)s * g.od + l);
                    inb = inb && (unsigned)v < (unsigned)g.width;
                }
                if (inb) atomicOr(w.need + oc + __ldg(w.st_delta + s), dil);
            }
        }
    }
}

__global__ void k_need(Geom g, Work w) { need_body(g, w, blockIdx.x, gridDim.x); }

__global__ void kb_need(BatchArgs B) {
    batch_for(B, [&](const Geom& g, const Work& w, int bx, int gx) { need_body(g, w, bx, gx); });
}

void launch_need(const Exec& ex, cudaStream_t st) {
    if (ex.batch())
        kb_need<<<ex.blocks(kShapeCapOuter, 256), 256, 0, st>>>(ex.args(kShapeCapOuter));
    else
        k_need<<<ex.blocks(kShapeCapOuter, 256), 256, 0, st>>>(*ex.g, *ex.w);
}

#define EGG_DISPATCH_DT(d, KERNEL, T, ...)            \
    switch (d) {                                      \
        case 1: KERNEL<1, T> __VA_ARGS__; break;      \
        case 2: KERNEL<2, T> __VA_ARGS__; break;      \
        case 3: KERNEL<3, T> __VA_ARGS__; break;      \
        case 4: KERNEL<4, T> __VA_ARGS__; break;      \
        case 5: KERNEL<5, T> __VA_ARGS__; break;      \
        case 6: KERNEL<6, T> __VA_ARGS__; break;      \
        case 8: KERNEL<8, T> __VA_ARGS__; break;      \
        case 16: KERNEL<16, T> __VA_ARGS__; break;    \
        default: KERNEL<0, T> __VA_ARGS__; break;     \
    }

template <int T>
void launch_update_batch(const Exec& ex, size_t smem, cudaStream_t st) {
    const int shape = T == 64 ? kShapeN64 : (T == 128 ? kShapeN128 : kShapeN256);
    EGG_DISPATCH_DT(ex.d, kb_update, T, <<<ex.blocks(shape, T), T, smem, st>>>(ex.args(shape)));
}

void launch_update(const Exec& ex, int* counts, cudaStream_t st) {
    const size_t smem = sizeof(float) * 3 * (2 * ex.table_k() + 1);
    if (ex.batch()) {
        switch (ex.update_threads()) {
            case 64: launch_update_batch<64>(ex, smem, st); break;
            case 256: launch_update_batch<256>(ex, smem, st); break;
            default: launch_update_batch<128>(ex, smem, st); break;
        }
    } else {
        EGG_DISPATCH_D(ex.d, k_update, <<<ex.blocks(kShapeN128, 128), 128, smem, st>>>(*ex.g, *ex.w, counts));
    }
}

}  // namespace egg
