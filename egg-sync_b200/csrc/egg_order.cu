// egg_order.cu -- FP64 local order parameter of the current positions.
//
// r = mean_p ( mean_{q in N(p)} exp(-|x_p - x_q|) ), the quantity the
// reference's CPU SynC computes before each move and stops on once it reaches
// lambda (src/algorithms/SynC.cpp:42-56, 277-303), evaluated here over the
// neighbourhoods N(p) of the EGG-SynC update (same cells, same tests).
//
// Walked neighbours contribute exp(-|x_p - x_q|) exactly in FP64.  Cells and
// 32-point groups whose points are all within eps (fully covered cells, or
// tight boxes provably inside) are aggregated, as in the update; each of
// their m points lies between the tight box's nearest and farthest corner
// from p, so the group adds m*exp(-far) to the lower and m*exp(-near) to the
// upper bound.  The result is a certified interval [r_lo, r_hi] (tight once
// clusters have collapsed); the lambda stop rule requires r_lo >= lambda.
// Reductions run in a fixed order: the interval is bit-reproducible.
#include "egg_common.cuh"
#include "egg_kernels.h"
#include "egg_stencil.cuh"

namespace egg {

namespace {

// distance bounds from float squared-distance bounds: the exact distance of
// every point of the box lies in [sqrt(near2)*(1-1e-5), sqrt(far2)*(1+1e-5)]
// (the float sums carry a relative error far below 1e-5 for d <= 64)
__device__ __forceinline__ void add_interval(double& lo, double& hi, int m, float near2, float far2) {
    const double dn = sqrt((double)near2) * (1.0 - 1e-5);
    const double df = sqrt((double)far2) * (1.0 + 1e-5);
    lo += (double)m * exp(-df);
    hi += (double)m * exp(-dn);
}

template <int D>
__device__ __forceinline__ void order_cell(const Geom& g, const Work& w, int c, const float* x, double& lo,
                                           double& hi, int& N) {
    constexpr int DM = D > 0 ? D : kMaxDims;
    const int d = D > 0 ? D : g.d;
    float sm2 = 0.f, lg2 = 0.f;
    for (int l = 0; l < d; l++) box_terms(x[l], __ldg(w.cell_dims + (size_t)l * g.ns + c), g.side, sm2, lg2);
    if (!(sm2 <= g.t_eps)) return;
    const int qb = __ldg(w.cell_start + c), qe = __ldg(w.cell_start + c + 1);
    float near2, far2;
    tight_box_dist2(x, w.cbmin + c, w.cbmax + c, g.ns, d, near2, far2);
    const bool full = lg2 <= g.t_eps;
    if (!full && near2 > g.t_eps) return;
    if (full || far2 <= g.t_eps) {
        add_interval(lo, hi, qe - qb, near2, far2);
        N += qe - qb;
        return;
    }
    const int kh = qb >> 5, kt = (qe - 1) >> 5;
    const int nw = (g.n + 31) >> 5;
    for (int k = kh; k <= kt; k++) {
        const int sb = max(qb, k << 5), se = min(qe, (k << 5) + 32);
        if (kh != kt) {
            const int rec = (k == kh) ? 1 : 0;
            float n2 = 0.f, f2 = 0.f;
            for (int l = 0; l < d; l++) {
                const float L = __ldg(w.gpart + wp_idx_f(2, l, d, rec, nw, k));
                const float H = __ldg(w.gpart + wp_idx_f(3, l, d, rec, nw, k));
                const float a0 = near_gap(x[l], L, H), b0 = far_gap(x[l], L, H);
                n2 = __fmaf_rn(a0, a0, n2);
                f2 = __fmaf_rn(b0, b0, f2);
            }
            if (n2 > g.t_eps) continue;
            if (f2 <= g.t_eps) {
                add_interval(lo, hi, se - sb, n2, f2);
                N += se - sb;
                continue;
            }
        }
        for (int q = sb; q < se; q++) {
            float d2 = 0.f;
            double dd = 0.0;
            for (int l = 0; l < d; l++) {
                const float xq = __ldg(w.X + (size_t)l * g.ns + q);
                d2 = dist_step(xq, x[l], d2);
                const double df = (double)xq - (double)x[l];
                dd += df * df;
            }
            if (d2 <= g.t_eps) {
                const double e = exp(-sqrt(dd));
                lo += e;
                hi += e;
                N++;
            }
        }
    }
    (void)DM;
}

}  // namespace

template <int D>
__global__ void __launch_bounds__(128) k_order_param(Geom g, Work w) {
    constexpr int DM = D > 0 ? D : kMaxDims;
    const int d = D > 0 ? D : g.d;
    __shared__ double s_lo[4], s_hi[4];
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    double rlo = 0.0, rhi = 0.0;
    if ((i & ~31) < g.n) {
        const bool valid = i < g.n;
        const int iv = valid ? i : g.n - 1;
        float x[DM];
        int gi[DM];
        int obase = 0;
        for (int l = 0; l < d; l++) {
            x[l] = w.X[(size_t)l * g.ns + iv];
            gi[l] = cell_dim(x[l], g);
            if (l < g.od) obase += gi[l] * g.wpow[l];
        }
        double lo = 0.0, hi = 0.0;
        int N = 0;
        for_candidates(g, w, gi, obase, lane, d, [] { return true; }, [&](int c) { order_cell<D>(g, w, c, x, lo, hi, N); });
        if (valid && N > 0) {
            rlo = lo / (double)N;
            rhi = hi / (double)N;
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        rlo += __shfl_xor_sync(0xffffffffu, rlo, o);
        rhi += __shfl_xor_sync(0xffffffffu, rhi, o);
    }
    if (lane == 0) {
        s_lo[wid] = rlo;
        s_hi[wid] = rhi;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double a = 0.0, b = 0.0;
        for (int k = 0; k < (int)(blockDim.x >> 5); k++) {
            a += s_lo[k];
            b += s_hi[k];
        }
        w.rpart[2 * blockIdx.x] = a;
        w.rpart[2 * blockIdx.x + 1] = b;
    }
}

// sum of the block partials in a fixed order; r = sum / n into rvals[slot]
__global__ void __launch_bounds__(256) k_order_reduce(Geom g, Work w, int nblocks, int final_slot) {
    __shared__ double s_lo[256], s_hi[256];
    double a = 0.0, b = 0.0;
    for (int k = threadIdx.x; k < nblocks; k += blockDim.x) {
        a += w.rpart[2 * k];
        b += w.rpart[2 * k + 1];
    }
    s_lo[threadIdx.x] = a;
    s_hi[threadIdx.x] = b;
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
        if ((int)threadIdx.x < s) {
            s_lo[threadIdx.x] += s_lo[threadIdx.x + s];
            s_hi[threadIdx.x] += s_hi[threadIdx.x + s];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        const int slot = final_slot >= 0 ? final_slot : w.ctrl[kCtrlIter];
        const double lo = s_lo[0] / (double)g.n, hi = s_hi[0] / (double)g.n;
        w.rvals[2 * slot] = lo;
        w.rvals[2 * slot + 1] = hi;
        if (final_slot < 0) w.ctrl[kCtrlLamReached] = lo >= (double)g.lam ? 1 : 0;
    }
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

// final_slot < 0: the value of the current iteration (slot = iteration);
// otherwise written to rvals[final_slot].  Needs the grid and the cell sums
// of the current positions.
void launch_order_param(const Geom& g, const Work& w, int final_slot, cudaStream_t st) {
    const int blocks = (g.n + 127) / 128;
    EGG_DISPATCH_D(g.d, k_order_param, <<<blocks, 128, 0, st>>>(g, w));
    k_order_reduce<<<1, 256, 0, st>>>(g, w, blocks, final_slot);
}

}  // namespace egg
