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

template <int D>
__global__ void __launch_bounds__(128) k_update(Geom g, Work w, int* __restrict__ counts) {
    constexpr int DM = D > 0 ? D : kMaxDims;
    const int d = D > 0 ? D : g.d;
    extern __shared__ float s_tab[];
    const int K = g.table_k, TW = 2 * K + 1;
    for (int t = threadIdx.x; t < 3 * TW; t += blockDim.x) s_tab[t] = w.table[t];
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        const int it = w.ctrl[kCtrlIter];
        w.stamps[4 * it + 1] = globaltimer();
    }
    __syncthreads();
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= g.n) return;
    const float* Ts = s_tab;
    const float* Tc = s_tab + TW;
    const float* Tm = s_tab + 2 * TW;

    float x[DM], S[DM], Cm[DM];
    int gi[DM];
    bool border = false;
    int obase = 0;
    for (int l = 0; l < d; l++) {
        x[l] = w.X[(size_t)l * g.ns + i];
        gi[l] = cell_dim(x[l], g);
        border |= on_border_dim(x[l], g.side);
        S[l] = 0.f;
        Cm[l] = 0.f;
        if (l < g.od) obase += gi[l] * g.wpow[l];
    }
    int N = 0, partial_in = 0;
    bool tab_err = false;
    const int own = w.cell_of[i];
    const int own_cnt = w.cell_start[own + 1] - w.cell_start[own];

    const int nst = w.st_count[0];
    for (int s = 0; s < nst; s++) {
        bool inb = true;
        for (int l = 0; l < g.od; l++) {
            int v = gi[l] + __ldg(w.st_off + (size_t)s * g.od + l);
            inb = inb && (unsigned)v < (unsigned)g.width;
        }
        if (!inb) continue;
        const int o = obase + __ldg(w.st_delta + s);
        int cb = __ldg(w.outer_begin + o), ce = __ldg(w.outer_begin + o + 1);
        if (cb >= ce) continue;
        if (g.od < d) {
            // cells beyond r+1 in dimension od fail the box test (their gap
            // exceeds (r+1)*side > eps), so the search keeps the visiting set
            const int* keys = w.cell_dims + (size_t)g.od * g.ns;
            cb = lower_bound_i(keys, cb, ce, gi[g.od] - g.r - 1);
            ce = lower_bound_i(keys, cb, ce, gi[g.od] + g.r + 2);
        }
        for (int c = cb; c < ce; c++) {
            float sm2 = 0.f, lg2 = 0.f;
            int kk[DM];
            for (int l = 0; l < d; l++) {
                const int cd = __ldg(w.cell_dims + (size_t)l * g.ns + c);
                box_terms(x[l], cd, g.side, sm2, lg2);
                kk[l] = cd - gi[l];
            }
            if (!(sm2 <= g.t_eps)) continue;
            const int qb = __ldg(w.cell_start + c), qe = __ldg(w.cell_start + c + 1);
            if (lg2 <= g.t_eps) {
                // fully inside the eps-ball: aggregate
                const float m = (float)(qe - qb);
                for (int l = 0; l < d; l++) {
                    int k = kk[l] + K;
                    if ((unsigned)k >= (unsigned)TW) { tab_err = true; k = K; }
                    const float ss = __ldg(w.css + (size_t)l * g.ns + c);
                    const float sm = __ldg(w.csm + (size_t)l * g.ns + c);
                    const float ts = Ts[k], tc = Tc[k], tm = Tm[k];
                    S[l] += ts * (m - sm) + tc * ss;
                    Cm[l] += m * tm + tc * sm + ts * ss;
                }
                N += qe - qb;
            } else {
                // boundary cell.  The tight box of its points decides it
                // wholesale when all or none of them are within eps (the
                // usual case once clusters have collapsed); otherwise walk.
                float near2, far2;
                tight_box_dist2(x, w.cbmin + c, w.cbmax + c, g.ns, d, near2, far2);
                if (near2 > g.t_eps) continue;
                if (far2 <= g.t_eps) {
                    const float m = (float)(qe - qb);
                    for (int l = 0; l < d; l++) {
                        int k = kk[l] + K;
                        if ((unsigned)k >= (unsigned)TW) { tab_err = true; k = K; }
                        const float ss = __ldg(w.css + (size_t)l * g.ns + c);
                        const float sm = __ldg(w.csm + (size_t)l * g.ns + c);
                        const float ts = Ts[k], tc = Tc[k], tm = Tm[k];
                        S[l] += ts * (m - sm) + tc * ss;
                        Cm[l] += m * tm + tc * sm + ts * ss;
                    }
                    N += qe - qb;
                    partial_in += qe - qb;
                    continue;
                }
                float as[DM], am[DM];
                for (int l = 0; l < d; l++) { as[l] = 0.f; am[l] = 0.f; }
                int cnt = 0;
                for (int q = qb; q < qe; q++) {
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
                if (cnt) {
                    const float m = (float)cnt;
                    for (int l = 0; l < d; l++) {
                        int k = kk[l] + K;
                        if ((unsigned)k >= (unsigned)TW) { tab_err = true; k = K; }
                        const float ts = Ts[k], tc = Tc[k], tm = Tm[k];
                        S[l] += ts * (m - am[l]) + tc * as[l];
                        Cm[l] += m * tm + tc * am[l] + ts * as[l];
                    }
                    N += cnt;
                    partial_in += cnt;
                }
            }
        }
    }

    const float fN = (float)N;
    for (int l = 0; l < d; l++) {
        const float corner = __fmul_rn((float)gi[l], g.side);
        const float phi = x[l] - corner;
        float sp, cp;
        sincosf(phi, &sp, &cp);
        const float A = cp * S[l] - sp * (fN - Cm[l]);
        w.Xn[(size_t)l * g.ns + i] = x[l] + A / fN;
    }
    if (counts) counts[i] = N;

    // convergence flag, EGG_SynC.cu:706-709.  half_count <= N - partial_in,
    // so a border point with neighbours in a partial cell always violates.
    bool viol;
    if (!border) viol = (N != own_cnt);
    else if (partial_in > 0) viol = true;
    else if (N == own_cnt) viol = false;
    else viol = (N != half_count<D>(g, w, x, gi, obase, own, own_cnt));
    const unsigned act = __activemask();
    const unsigned vb = __ballot_sync(act, viol);
    if (vb && (threadIdx.x & 31) == __ffs(act) - 1) {
        volatile int* f = w.ctrl + kCtrlFlag;
        if (*f != 0) *f = 0;
    }
    if (tab_err) atomicOr(w.ctrl + kCtrlStatus, kErrTable);
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

void launch_update(const Geom& g, const Work& w, int* counts, cudaStream_t st) {
    const int threads = 128;
    const int blocks = (g.n + threads - 1) / threads;
    const size_t smem = sizeof(float) * 3 * (2 * g.table_k + 1);
    EGG_DISPATCH_D(g.d, k_update, <<<blocks, threads, smem, st>>>(g, w, counts));
}

}  // namespace egg
