// egg_simple.cu -- brute-force GPU SynC, the second drop-in.
//
// Replaces GPU_DynamicalClustering (src/algorithms/simple_GPU_SynC.cu:29-238,
// reached from GPU_DynamicalClustering_wrapper, src/maps/map.cpp:27-29): every
// iteration updates each point from all points within eps (itself included),
//   x_p += (1/N) sum_q sin(x_q - x_p),
// and the loop stops once the mean local order parameter
// r_local = mean_p (1/N) sum_q exp(-|x_p - x_q|) reaches lam, or after max_iter
// iterations (the reference's cap is 100).  Labels: a point whose eps-ball
// holds more than one point gets the rank of the smallest index in that ball
// among all such smallest indices (simple_GPU_SynC.cu:70-100), else -1.
//
// The neighbour test is the reference's `sqrt(sum of diff^2) <= eps` with the
// square sum accumulated by fused multiply-adds, i.e. d2 <= the largest float
// whose sqrtf is <= eps.  A block stages tiles of source points in shared
// memory and every thread visits them in index order, so each point's sums
// are formed in the reference's order.  r_local is summed in FP64 in a fixed
// order (the reference adds per-point floats with atomics, in no fixed order).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "eggsync.h"
#include "egg_common.cuh"
#include "egg_host_common.h"

namespace egg {

namespace {

constexpr int kSimpleBlock = 128;

// one iteration; part[blockIdx.x] = sum over the block's points of r_p
template <int D>
__global__ void __launch_bounds__(kSimpleBlock) k_simple_iter(const float* __restrict__ cur, float* __restrict__ next,
                                                              int n, int dd, float t_eps, double* part) {
    constexpr int DM = D > 0 ? D : kMaxDims;
    const int d = D > 0 ? D : dd;
    extern __shared__ float tile[];  // [kSimpleBlock][d]
    __shared__ double s_r[kSimpleBlock];
    const int p = blockIdx.x * kSimpleBlock + threadIdx.x;
    const bool valid = p < n;
    float x[DM], s[DM];
    for (int l = 0; l < d; l++) {
        x[l] = valid ? cur[(size_t)p * d + l] : 0.f;
        s[l] = 0.f;
    }
    float r = 0.f;
    int cnt = 0;
    for (int t0 = 0; t0 < n; t0 += kSimpleBlock) {
        const int m = min(kSimpleBlock, n - t0);
        __syncthreads();
        for (int k = threadIdx.x; k < m * d; k += kSimpleBlock) tile[k] = cur[(size_t)t0 * d + k];
        __syncthreads();
        if (valid) {
            for (int j = 0; j < m; j++) {
                const float* q = tile + j * d;
                float d2 = 0.f;
                for (int l = 0; l < d; l++) d2 = dist_step(x[l], q[l], d2);
                if (d2 <= t_eps) {
                    cnt++;
                    for (int l = 0; l < d; l++) s[l] += sinf(__fsub_rn(q[l], x[l]));
                    r += expf(-sqrtf(d2));
                }
            }
        }
    }
    double rp = 0.0;
    if (valid) {
        for (int l = 0; l < d; l++) next[(size_t)p * d + l] = x[l] + s[l] / (float)cnt;
        rp = (double)(r / (float)cnt);
    }
    s_r[threadIdx.x] = rp;
    __syncthreads();
    for (int o = kSimpleBlock / 2; o > 0; o >>= 1) {
        if (threadIdx.x < o) s_r[threadIdx.x] += s_r[threadIdx.x + o];
        __syncthreads();
    }
    if (threadIdx.x == 0) part[blockIdx.x] = s_r[0];
}

__global__ void k_simple_rsum(const double* __restrict__ part, int blocks, int n, double* r) {
    if (threadIdx.x == 0 && blockIdx.x == 0) {
        double s = 0.0;
        for (int b = 0; b < blocks; b++) s += part[b];
        *r = s / n;
    }
}

// smallest index within eps (count > 1): rep[p], and mark that index
template <int D>
__global__ void __launch_bounds__(kSimpleBlock) k_simple_reps(const float* __restrict__ X, int n, int dd, float t_eps,
                                                              int* rep, int* incl) {
    constexpr int DM = D > 0 ? D : kMaxDims;
    const int d = D > 0 ? D : dd;
    extern __shared__ float tile[];
    const int p = blockIdx.x * kSimpleBlock + threadIdx.x;
    const bool valid = p < n;
    float x[DM];
    for (int l = 0; l < d; l++) x[l] = valid ? X[(size_t)p * d + l] : 0.f;
    int mn = p, cnt = 0;
    for (int t0 = 0; t0 < n; t0 += kSimpleBlock) {
        const int m = min(kSimpleBlock, n - t0);
        __syncthreads();
        for (int k = threadIdx.x; k < m * d; k += kSimpleBlock) tile[k] = X[(size_t)t0 * d + k];
        __syncthreads();
        if (valid) {
            for (int j = 0; j < m; j++) {
                float d2 = 0.f;
                for (int l = 0; l < d; l++) d2 = dist_step(x[l], tile[j * d + l], d2);
                if (d2 <= t_eps) {
                    cnt++;
                    mn = min(mn, t0 + j);
                }
            }
        }
    }
    if (valid) {
        rep[p] = cnt > 1 ? mn : -1;
        if (cnt > 1) incl[mn] = 1;
    }
}

// ranks of the marked indices: exclusive prefix counts, one block of 1024
// threads walking the array in chunks
__global__ void __launch_bounds__(1024) k_simple_rank(const int* __restrict__ incl, int n, int* rank) {
    __shared__ int ws[32];
    __shared__ int carry;
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    for (int base = 0; base < n; base += 1024) {
        const int i = base + threadIdx.x;
        const int v = i < n ? incl[i] : 0;
        int x = v;
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, x, o);
            if (lane >= o) x += y;
        }
        if (lane == 31) ws[wid] = x;
        __syncthreads();
        if (wid == 0) {
            int s = ws[lane], t = s;
            for (int o = 1; o < 32; o <<= 1) {
                const int y = __shfl_up_sync(0xffffffffu, t, o);
                if (lane >= o) t += y;
            }
            ws[lane] = t - s;
        }
        __syncthreads();
        if (i < n) rank[i] = carry + ws[wid] + x - v;
        __syncthreads();
        if (threadIdx.x == 1023) carry += ws[wid] + x;
        __syncthreads();
    }
}

__global__ void k_simple_labels(const int* __restrict__ rep, const int* __restrict__ rank, int n, int* out) {
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += gridDim.x * blockDim.x)
        out[p] = rep[p] >= 0 ? rank[rep[p]] : -1;
}

#define EGG_SIMPLE_D(d, KERNEL, ...)                  \
    switch (d) {                                      \
        case 1: KERNEL<1> __VA_ARGS__; break;         \
        case 2: KERNEL<2> __VA_ARGS__; break;         \
        case 3: KERNEL<3> __VA_ARGS__; break;         \
        case 4: KERNEL<4> __VA_ARGS__; break;         \
        case 5: KERNEL<5> __VA_ARGS__; break;         \
        case 8: KERNEL<8> __VA_ARGS__; break;         \
        case 16: KERNEL<16> __VA_ARGS__; break;       \
        default: KERNEL<0> __VA_ARGS__; break;        \
    }

float sq_threshold_f(float e) {
    float t = e * e;
    while (t > 0.0f && sqrtf(t) > e) t = nextafterf(t, 0.0f);
    for (;;) {
        const float u = nextafterf(t, INFINITY);
        if (sqrtf(u) <= e) t = u; else break;
    }
    return t;
}

}  // namespace

int simple_run(const float* x, int64_t n64, int32_t d, float eps, float lam, int32_t max_iter, int32_t* labels,
               float* positions_out, egg_stats* stats, void* stream) {
    if (!x || !labels) throw ArgError{EGG_ERR_ARG, "x and labels must not be NULL"};
    if (n64 < 1 || n64 > (1 << 26)) throw ArgError{EGG_ERR_ARG, "n out of range"};
    if (d < 1 || d > kMaxDims) throw ArgError{EGG_ERR_ARG, "d must be in [1, 64]"};
    if (!(eps > 0.f) || !std::isfinite(eps)) throw ArgError{EGG_ERR_ARG, "eps must be positive and finite"};
    if (max_iter < 0) throw ArgError{EGG_ERR_ARG, "max_iter must be >= 0"};
    const int n = (int)n64;
    const int cap = max_iter > 0 ? max_iter : 100;
    const float t_eps = sq_threshold_f(eps);
    cudaStream_t st = (cudaStream_t)stream;
    const int blocks = (n + kSimpleBlock - 1) / kSimpleBlock;
    const size_t smem = sizeof(float) * kSimpleBlock * d;
    std::vector<void*> tmp;
    auto alloc = [&](size_t bytes) {
        void* p = nullptr;
        EGG_CHECK(dev_alloc((void**)&p, std::max<size_t>(bytes, 4)));
        tmp.push_back(p);
        return p;
    };
    cudaEvent_t ev[6] = {};
    int iters = 0;
    double r_local = 0.0;
    std::vector<float> itr;
    try {
        for (auto& e : ev) EGG_CHECK(cudaEventCreate(&e));
        EGG_CHECK(cudaEventRecord(ev[0], st));
        float* cur = (float*)alloc(4 * (size_t)n * d);
        float* nxt = (float*)alloc(4 * (size_t)n * d);
        double* part = (double*)alloc(8 * (size_t)blocks);
        double* rd = (double*)alloc(8);
        EGG_CHECK(cudaMemcpyAsync(cur, x, 4 * (size_t)n * d, cudaMemcpyDefault, st));
        {
            std::vector<float> h((size_t)n * d);
            EGG_CHECK(cudaMemcpyAsync(h.data(), cur, 4 * h.size(), cudaMemcpyDeviceToHost, st));
            EGG_CHECK(cudaStreamSynchronize(st));
            for (float v : h)
                if (!std::isfinite(v)) throw ArgError{EGG_ERR_INPUT, "input holds NaN or Inf"};
        }
        EGG_CHECK(cudaEventRecord(ev[1], st));
        while (r_local < (double)lam && iters < cap) {
            EGG_CHECK(cudaEventRecord(ev[4], st));
            EGG_SIMPLE_D(d, k_simple_iter, <<<blocks, kSimpleBlock, smem, st>>>(cur, nxt, n, d, t_eps, part));
            k_simple_rsum<<<1, 32, 0, st>>>(part, blocks, n, rd);
            EGG_CHECK(cudaMemcpyAsync(&r_local, rd, 8, cudaMemcpyDeviceToHost, st));
            EGG_CHECK(cudaEventRecord(ev[5], st));
            EGG_CHECK(cudaStreamSynchronize(st));
            float ms = 0.f;
            EGG_CHECK(cudaEventElapsedTime(&ms, ev[4], ev[5]));
            itr.push_back(ms);
            std::swap(cur, nxt);
            iters++;
        }
        EGG_CHECK(cudaEventRecord(ev[2], st));
        int* rep = (int*)alloc(4 * (size_t)n);
        int* incl = (int*)alloc(4 * (size_t)n);
        int* rank = (int*)alloc(4 * (size_t)n);
        const bool dev_out = is_device_ptr(labels);
        int* lab = dev_out ? labels : (int*)alloc(4 * (size_t)n);
        EGG_CHECK(cudaMemsetAsync(incl, 0, 4 * (size_t)n, st));
        EGG_SIMPLE_D(d, k_simple_reps, <<<blocks, kSimpleBlock, smem, st>>>(cur, n, d, t_eps, rep, incl));
        k_simple_rank<<<1, 1024, 0, st>>>(incl, n, rank);
        k_simple_labels<<<std::min(blocks, 148 * 16), kSimpleBlock, 0, st>>>(rep, rank, n, lab);
        EGG_CHECK(cudaEventRecord(ev[3], st));
        if (!dev_out) EGG_CHECK(cudaMemcpyAsync(labels, lab, 4 * (size_t)n, cudaMemcpyDeviceToHost, st));
        if (positions_out)
            EGG_CHECK(cudaMemcpyAsync(positions_out, cur, 4 * (size_t)n * d, cudaMemcpyDefault, st));
        EGG_CHECK(cudaStreamSynchronize(st));
        EGG_CHECK(cudaGetLastError());
        if (stats) {
            float t01, t12, t23, t03;
            EGG_CHECK(cudaEventElapsedTime(&t01, ev[0], ev[1]));
            EGG_CHECK(cudaEventElapsedTime(&t12, ev[1], ev[2]));
            EGG_CHECK(cudaEventElapsedTime(&t23, ev[2], ev[3]));
            EGG_CHECK(cudaEventElapsedTime(&t03, ev[0], ev[3]));
            std::vector<int> hl((size_t)n);
            EGG_CHECK(cudaMemcpy(hl.data(), lab, 4 * (size_t)n, cudaMemcpyDefault));
            int k = 0;
            for (int v : hl) k = std::max(k, v + 1);
            stats->iterations = iters;
            stats->converged = r_local >= (double)lam;
            stats->n_clusters = k;
            stats->order_param = r_local;
            stats->order_param_lo = stats->order_param_hi = r_local;
            stats->workspace_bytes = (int64_t)(4 * (size_t)n * d * 2 + 8 * (size_t)blocks + 16 * (size_t)n);
            stats->stage_ms[0] = t01;
            stats->stage_ms[2] = t12;
            stats->stage_ms[4] = t23;
            stats->total_ms = t03;
            stats->launches = 2 * iters + 4;
            if (stats->itr_ms)
                for (int i = 0; i < std::min(iters, stats->itr_cap); i++) stats->itr_ms[i] = itr[i];
        }
    } catch (...) {
        for (void* p : tmp) cudaFree(p);
        for (auto e : ev)
            if (e) cudaEventDestroy(e);
        throw;
    }
    for (void* p : tmp) cudaFree(p);
    for (auto e : ev) cudaEventDestroy(e);
    return r_local >= (double)lam ? EGG_OK : EGG_MAX_ITER;
}

}  // namespace egg

extern "C" __attribute__((visibility("default"))) int egg_simple_sync_run(const float* x, int64_t n, int32_t d,
                                                                          float eps, float lam, int32_t max_iter,
                                                                          int32_t* labels, float* positions_out,
                                                                          egg_stats* stats, void* stream) {
    return egg::guarded(
        [&] { return egg::simple_run(x, n, d, eps, lam, max_iter, labels, positions_out, stats, stream); });
}
