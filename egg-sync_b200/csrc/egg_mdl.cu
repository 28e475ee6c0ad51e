// egg_mdl.cu -- eps search by minimum description length, on the GPU.
//
// Replaces the reference's full-SynC driver Sync(D, k)
// (python/SynCTorch.py:349-372) and its two cost pieces:
//   * NN(k, D) (SynCTorch.py:112-137): mean over the points of the distance
//     to the k-th nearest other point (brute force, O(n^2 d));
//   * L_Clust_Outl(D, M) (SynCTorch.py:265-314): the coding cost of a
//     clustering, a model term over the cluster sizes and outliers plus the
//     negative log-likelihood of every clustered point under a Gaussian
//     product-kernel density estimate of its own cluster (O(sum |C|^2 d)).
// The search starts at eps = NN(k), steps by NN(k+1) - NN(k) in float32 as
// the reference does, clusters each eps, stops at the first clustering with
// a single cluster and returns the clustering of least cost.  The
// clusterings come from this library's EGG-SynC loop, run as batches of eps
// candidates (egg_sync_batch semantics: each one identical to egg_sync_run).
//
// Kernels: brute-force k-NN (the k+1 smallest squared distances per point in
// registers, candidate points staged through shared memory), column
// statistics (FP64, fixed reduction order), and the per-cluster density
// sums (FP32 exponent, FP64 accumulation; clusters laid out contiguously by
// a stable sort on the label, sums reduced per cluster in a fixed order), so
// every cost is reproducible bit for bit from run to run.
#include <cuda_runtime.h>


#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "eggsync.h"
#include "egg_common.cuh"
#include "egg_host_common.h"
#include "egg_sort.h"

namespace egg {

namespace {

constexpr int kKnnThreads = 128;
constexpr int kKnnMaxK = 31;  // k + 1 <= 32 distances kept per point
constexpr int kSumBlocks = 256;
constexpr int kMdlBatch = 8;  // eps candidates clustered per batched call

// ------------------------------------------------------------------------
// k-NN: the (k)-th and (k+1)-th smallest distance of every point to the
// other points (the reference's NN keeps the k smallest, distances[0] being
// the k-th).  Squared distances are compared; the two kept are rooted.
// ------------------------------------------------------------------------
template <int KM, int D>
__global__ void __launch_bounds__(kKnnThreads) k_knn(const float* __restrict__ x, int n, int dd, int k,
                                                     float* __restrict__ kth, float* __restrict__ kth1) {
    constexpr int DM = D > 0 ? D : 1;
    const int d = D > 0 ? D : dd;
    extern __shared__ float tile[];  // [kKnnThreads][d]
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const bool valid = i < n;
    float xi[DM];
    if constexpr (D > 0) {
#pragma unroll
        for (int l = 0; l < D; l++) xi[l] = valid ? x[(size_t)i * D + l] : 0.f;
    }
    float best[KM];
#pragma unroll
    for (int t = 0; t < KM; t++) best[t] = INFINITY;
    for (int j0 = 0; j0 < n; j0 += kKnnThreads) {
        const int cnt = min(kKnnThreads, n - j0);
        __syncthreads();
        for (int t = threadIdx.x; t < cnt * d; t += blockDim.x) tile[t] = x[(size_t)j0 * d + t];
        __syncthreads();
        if (!valid) continue;
        for (int jj = 0; jj < cnt; jj++) {
            float s = 0.f;
            if constexpr (D > 0) {
#pragma unroll
                for (int l = 0; l < D; l++) {
                    const float df = xi[l] - tile[jj * D + l];
                    s = fmaf(df, df, s);
                }
            } else {
                for (int l = 0; l < d; l++) {
                    const float df = __ldg(x + (size_t)i * d + l) - tile[jj * d + l];
                    s = fmaf(df, df, s);
                }
            }
            if (j0 + jj == i || !(s < best[KM - 1])) continue;
            // insertion into the ascending list
#pragma unroll
            for (int t = 0; t < KM; t++) {
                const float a = best[t];
                const bool sw = s < a;
                best[t] = sw ? s : a;
                s = sw ? a : s;
            }
        }
    }
    if (!valid) return;
    float a = best[0], b = best[0];
#pragma unroll
    for (int t = 0; t < KM; t++) {
        if (t == k - 1) a = best[t];
        if (t == k) b = best[t];
    }
    kth[i] = sqrtf(a);
    kth1[i] = sqrtf(b);
}

// ------------------------------------------------------------------------
// deterministic FP64 sums: per-block partials in a fixed tree, then one block
// ------------------------------------------------------------------------
__device__ double block_sum_d(double v) {
    __shared__ double ws[32];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    if (lane == 0) ws[wid] = v;
    __syncthreads();
    const int nw = (blockDim.x + 31) >> 5;
    double r = 0.0;
    if (wid == 0) {
        r = lane < nw ? ws[lane] : 0.0;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) r += __shfl_down_sync(0xffffffffu, r, o);
    }
    __syncthreads();
    return r;  // valid in thread 0
}

// sum over i < n of (v[i*stride] - center)^power (power 1 or 2)
__global__ void __launch_bounds__(256) k_sum_partial(const float* __restrict__ v, int n, int stride,
                                                     const double* __restrict__ center, int power,
                                                     double* __restrict__ part) {
    const double c = center ? *center : 0.0;
    double s = 0.0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const double t = (double)v[(size_t)i * stride] - c;
        s += power == 2 ? t * t : t;
    }
    const double r = block_sum_d(s);
    if (threadIdx.x == 0) part[blockIdx.x] = r;
}

__global__ void __launch_bounds__(256) k_sum_final(const double* __restrict__ part, int nb, double scale,
                                                   double* __restrict__ out) {
    double s = 0.0;
    for (int t = threadIdx.x; t < nb; t += blockDim.x) s += part[t];
    const double r = block_sum_d(s);
    if (threadIdx.x == 0) *out = r * scale;
}

// row-major n x d -> column l (contiguous), with a non-finite check
__global__ void k_column(const float* __restrict__ x, int n, int d, int l, float* __restrict__ col, int* bad) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const float v = x[(size_t)i * d + l];
        if (!isfinite(v)) *bad = 1;
        col[i] = v;
    }
}

// ------------------------------------------------------------------------
// clusters of a labelling: keys = label as unsigned (outliers, -1, last),
// stably sorted with the point indices; segment heads of the clustered part
// ------------------------------------------------------------------------
__global__ void k_label_keys(const int* __restrict__ labels, int n, unsigned* __restrict__ keys,
                             int* __restrict__ idx, int* bad) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const int l = labels[i];
        if (l < -1) *bad = 1;
        keys[i] = (unsigned)l;  // -1 -> 0xffffffff: after every cluster
        idx[i] = i;
    }
}

__global__ void k_heads(const unsigned* __restrict__ keys, int m, int* __restrict__ head) {
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < m; j += gridDim.x * blockDim.x)
        head[j] = (j == 0 || keys[j] != keys[j - 1]) ? 1 : 0;
}

// first sorted position holding an outlier key (the clustered count)
__global__ void k_first_outlier(const unsigned* __restrict__ keys, int n, int* __restrict__ m) {
    int lo = 0, hi = n;
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (keys[mid] < 0xffffffffu) lo = mid + 1;
        else hi = mid;
    }
    *m = lo;
}

// clustered points in sorted order, coordinates by dimension (SoA, stride m)
__global__ void k_gather_sorted(const float* __restrict__ x, int d, const int* __restrict__ idx, int m,
                                float* __restrict__ xs) {
    for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < (size_t)m * d;
         t += (size_t)gridDim.x * blockDim.x) {
        const int j = (int)(t % m), l = (int)(t / m);
        xs[t] = x[(size_t)idx[j] * d + l];
    }
}

// segment of every clustered point: seg[j] = (inclusive count of heads) - 1
// float32 bits -> unsigned keys in the same order (negative values flipped)
__global__ void k_float_keys(const float* __restrict__ v, int n, unsigned* __restrict__ keys) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const unsigned u = __float_as_uint(v[i]);
        keys[i] = (u & 0x80000000u) ? ~u : (u | 0x80000000u);
    }
}

// first sorted position of every segment: begin[incl[j] - 1] = j at heads
__global__ void k_seg_begin(const int* __restrict__ head, const int* __restrict__ incl, int m, int* __restrict__ begin) {
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < m; j += gridDim.x * blockDim.x)
        if (head[j]) begin[incl[j] - 1] = j;
}

__global__ void k_seg_of(const int* __restrict__ incl, int m, int* __restrict__ seg) {
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < m; j += gridDim.x * blockDim.x) seg[j] = incl[j] - 1;
}

// Density of every clustered point within its own cluster (f_hat,
// SynCTorch.py:144-154, over D[C]): s = sum over the cluster's points y of
// exp(-1/2 sum_l ((x_l - y_l) / h_l)^2), f = s * norm / |C| with
// norm = (2 pi)^(-d/2) / prod h_l.  Writes f and log2 f.
template <int D>
__global__ void __launch_bounds__(256) k_kde(const float* __restrict__ xs, int m, int dd,
                                             const int* __restrict__ seg, const int* __restrict__ begin,
                                             const float* __restrict__ invh, double norm,
                                             double* __restrict__ f, double* __restrict__ lf) {
    constexpr int DM = D > 0 ? D : 1;
    const int d = D > 0 ? D : dd;
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= m) return;
    const int sg = seg[j];
    const int b = begin[sg], e = begin[sg + 1];
    float xj[DM], ih[DM];
    if constexpr (D > 0) {
#pragma unroll
        for (int l = 0; l < D; l++) {
            xj[l] = xs[(size_t)l * m + j];
            ih[l] = invh[l];
        }
    }
    double s = 0.0;
    for (int y = b; y < e; y++) {
        float u = 0.f;
        if constexpr (D > 0) {
#pragma unroll
            for (int l = 0; l < D; l++) {
                const float t = (xj[l] - __ldg(xs + (size_t)l * m + y)) * ih[l];
                u = fmaf(t, t, u);
            }
        } else {
            for (int l = 0; l < d; l++) {
                const float t = (__ldg(xs + (size_t)l * m + j) - __ldg(xs + (size_t)l * m + y)) * __ldg(invh + l);
                u = fmaf(t, t, u);
            }
        }
        s += (double)expf(-0.5f * u);
    }
    const double fv = s * norm / (double)(e - b);
    f[j] = fv;
    lf[j] = log2(fv);
}

#define EGG_MDL_DISPATCH_D(d, KERNEL, ...)         \
    switch (d) {                                   \
        case 1: KERNEL<1> __VA_ARGS__; break;      \
        case 2: KERNEL<2> __VA_ARGS__; break;      \
        case 3: KERNEL<3> __VA_ARGS__; break;      \
        case 4: KERNEL<4> __VA_ARGS__; break;      \
        case 5: KERNEL<5> __VA_ARGS__; break;      \
        case 8: KERNEL<8> __VA_ARGS__; break;      \
        default: KERNEL<0> __VA_ARGS__; break;     \
    }

int grid_for(size_t work, int threads, int cap = 148 * 16) {
    return (int)std::max<size_t>(1, std::min<size_t>((work + threads - 1) / threads, (size_t)cap));
}

// device memory of one call, freed on every exit
struct Arena {
    std::vector<void*> ptrs;
    template <typename T>
    T* get(size_t count) {
        void* p = nullptr;
        EGG_CHECK(dev_alloc((void**)&p, std::max<size_t>(1, count * sizeof(T))));
        ptrs.push_back(p);
        return (T*)p;
    }
    ~Arena() {
        for (void* p : ptrs) cudaFree(p);
    }
};

// the input on the device (a copy when it is in host memory)
const float* device_input(Arena& A, const float* x, size_t count, cudaStream_t st) {
    if (is_device_ptr(x)) return x;
    float* d = A.get<float>(count);
    EGG_CHECK(cudaMemcpyAsync(d, x, 4 * count, cudaMemcpyHostToDevice, st));
    return d;
}

void check_nd(int64_t n, int32_t d, int64_t min_n) {
    if (n < min_n || n > ((int64_t)1 << 30)) throw ArgError{EGG_ERR_ARG, "n out of range"};
    if (d < 1 || d > kMaxDims) throw ArgError{EGG_ERR_ARG, "d must be in [1, 64]"};
}

template <int KM>
void launch_knn(int d, int blocks, size_t smem, cudaStream_t st, const float* x, int n, int k, float* kth,
                float* kth1) {
    switch (d) {
        case 1: k_knn<KM, 1><<<blocks, kKnnThreads, smem, st>>>(x, n, d, k, kth, kth1); break;
        case 2: k_knn<KM, 2><<<blocks, kKnnThreads, smem, st>>>(x, n, d, k, kth, kth1); break;
        case 3: k_knn<KM, 3><<<blocks, kKnnThreads, smem, st>>>(x, n, d, k, kth, kth1); break;
        case 4: k_knn<KM, 4><<<blocks, kKnnThreads, smem, st>>>(x, n, d, k, kth, kth1); break;
        case 5: k_knn<KM, 5><<<blocks, kKnnThreads, smem, st>>>(x, n, d, k, kth, kth1); break;
        case 8: k_knn<KM, 8><<<blocks, kKnnThreads, smem, st>>>(x, n, d, k, kth, kth1); break;
        default: k_knn<KM, 0><<<blocks, kKnnThreads, smem, st>>>(x, n, d, k, kth, kth1); break;
    }
}

// mean of the k-th and (k+1)-th nearest-neighbour distances, FP64
void knn_mean(Arena& A, const float* xd, int n, int d, int k, double out[2], cudaStream_t st) {
    float* kth = A.get<float>(n);
    float* kth1 = A.get<float>(n);
    const int blocks = (n + kKnnThreads - 1) / kKnnThreads;
    const size_t smem = sizeof(float) * kKnnThreads * d;  // <= 32 KB (d <= 64)
    if (k + 1 <= 8) launch_knn<8>(d, blocks, smem, st, xd, n, k, kth, kth1);
    else if (k + 1 <= 16) launch_knn<16>(d, blocks, smem, st, xd, n, k, kth, kth1);
    else launch_knn<32>(d, blocks, smem, st, xd, n, k, kth, kth1);
    EGG_CHECK(cudaGetLastError());
    double* part = A.get<double>(kSumBlocks);
    double* res = A.get<double>(2);
    const int nb = grid_for((size_t)n, 256, kSumBlocks);
    k_sum_partial<<<nb, 256, 0, st>>>(kth, n, 1, nullptr, 1, part);
    k_sum_final<<<1, 256, 0, st>>>(part, nb, 1.0 / n, res);
    k_sum_partial<<<nb, 256, 0, st>>>(kth1, n, 1, nullptr, 1, part);
    k_sum_final<<<1, 256, 0, st>>>(part, nb, 1.0 / n, res + 1);
    EGG_CHECK(cudaMemcpyAsync(out, res, 16, cudaMemcpyDeviceToHost, st));
    EGG_CHECK(cudaStreamSynchronize(st));
}

// The bandwidths of L_Clust_Outl (SynCTorch.py:284-286): per dimension,
// h = 0.9 n^(-1/(d+4)) min(var, IQR / 1.34), var the unbiased variance (the
// reference's "sigma" is torch.var) and IQR the 75th minus the 25th
// percentile with linear interpolation (scipy.stats.iqr).
std::vector<double> bandwidths(Arena& A, const float* xd, int n, int d, cudaStream_t st) {
    float* col = A.get<float>(n);
    unsigned* ckeys = A.get<unsigned>(n);
    unsigned* sorted = A.get<unsigned>(n);  // the column's order-preserving keys, sorted
    void* sort_tmp = A.get<char>(prim::sort_scratch_bytes(n));
    double* part = A.get<double>(kSumBlocks);
    double* res = A.get<double>(2);
    int* bad = A.get<int>(1);
    EGG_CHECK(cudaMemsetAsync(bad, 0, 4, st));
    std::vector<double> h(d);
    const int nb = grid_for((size_t)n, 256, kSumBlocks);
    const double c = 0.9 * std::pow((double)n, -1.0 / (d + 4));
    for (int l = 0; l < d; l++) {
        k_column<<<grid_for((size_t)n, 256), 256, 0, st>>>(xd, n, d, l, col, bad);
        k_sum_partial<<<nb, 256, 0, st>>>(col, n, 1, nullptr, 1, part);
        k_sum_final<<<1, 256, 0, st>>>(part, nb, 1.0 / n, res);
        k_sum_partial<<<nb, 256, 0, st>>>(col, n, 1, res, 2, part);
        k_sum_final<<<1, 256, 0, st>>>(part, nb, 1.0 / (n - 1), res + 1);
        k_float_keys<<<grid_for((size_t)n, 256), 256, 0, st>>>(col, n, ckeys);
        prim::sort_pairs(ckeys, nullptr, sorted, nullptr, n, sort_tmp, st);
        double mv[2];
        EGG_CHECK(cudaMemcpyAsync(mv, res, 16, cudaMemcpyDeviceToHost, st));
        auto pct = [&](double q) {
            const double pos = q * (double)(n - 1);
            const int lo = (int)std::floor(pos);
            const int hi = std::min(lo + 1, n - 1);
            unsigned ka = 0, kb = 0;
            EGG_CHECK(cudaMemcpyAsync(&ka, sorted + lo, 4, cudaMemcpyDeviceToHost, st));
            EGG_CHECK(cudaMemcpyAsync(&kb, sorted + hi, 4, cudaMemcpyDeviceToHost, st));
            EGG_CHECK(cudaStreamSynchronize(st));
            auto unkey = [](unsigned k) {
                const unsigned u = (k & 0x80000000u) ? (k & 0x7fffffffu) : ~k;
                float f;
                memcpy(&f, &u, 4);
                return f;
            };
            const float a = unkey(ka), b = unkey(kb);
            const double t = pos - lo;
            // numpy's linear interpolation, from the nearer end
            return t >= 0.5 ? (double)b - ((double)b - a) * (1.0 - t) : (double)a + ((double)b - a) * t;
        };
        const double iqr = pct(0.75) - pct(0.25);
        EGG_CHECK(cudaStreamSynchronize(st));
        h[l] = c * std::min(mv[1], iqr / 1.34);
        if (!(h[l] > 0.0) || !std::isfinite(h[l]))
            throw ArgError{EGG_ERR_INPUT, "dimension " + std::to_string(l) + " has no spread (zero KDE bandwidth)"};
    }
    int hbad = 0;
    EGG_CHECK(cudaMemcpyAsync(&hbad, bad, 4, cudaMemcpyDeviceToHost, st));
    EGG_CHECK(cudaStreamSynchronize(st));
    if (hbad) throw ArgError{EGG_ERR_INPUT, "input holds NaN or Inf"};
    return h;
}

// Coding cost of one labelling (device labels, original order), L_Clust_Outl:
//   L_M = sum_C |C| log2(n / |C|) + d/2 log2 |C|  +  outliers * log2 n
//   L_D = -( sum_C sum_{x in C} log2(f(x) / sum_{y in C} f(y))
//            + outliers * (2 pi)^(-1/2) * prod h )
// Returns L_M + L_D; *clusters = number of clusters.
// Device arrays of the cost of labellings of one n x d input, sized once
// (the search costs every candidate with the same arrays).
struct CostWs {
    Arena A;
    int n, d;
    unsigned *keys, *keys_s;
    int *idx, *idx_s, *head, *incl, *seg, *begin, *scal;  // scal: bad flag, m
    float *xs, *invh;
    double *f, *lf, *sf, *slf;
    void* sort_tmp = nullptr;  // scratch of the label sort
    void* scan_tmp = nullptr;  // scratch of the head scan
    CostWs(int n_, int d_) : n(n_), d(d_) {
        sort_tmp = A.get<char>(prim::sort_scratch_bytes(n));
        scan_tmp = A.get<char>(prim::scan_scratch_bytes(n));
        keys = A.get<unsigned>(n);
        keys_s = A.get<unsigned>(n);
        idx = A.get<int>(n);
        idx_s = A.get<int>(n);
        head = A.get<int>(n);
        incl = A.get<int>(n);
        seg = A.get<int>(n);
        begin = A.get<int>((size_t)n + 1);
        scal = A.get<int>(4);
        xs = A.get<float>((size_t)n * d);
        invh = A.get<float>(d);
        f = A.get<double>(n);
        lf = A.get<double>(n);
        sf = A.get<double>(n);
        slf = A.get<double>(n);
    }
};

// Coding cost of one labelling (device labels, original order), L_Clust_Outl:
//   L_M = sum_C |C| log2(n / |C|) + d/2 log2 |C|  +  outliers * log2 n
//   L_D = -( sum_C sum_{x in C} log2(f(x) / sum_{y in C} f(y))
//            + outliers * (2 pi)^(-1/2) * prod h )
// Returns L_M + L_D; *clusters = number of clusters.
double mdl_cost(CostWs& W, const float* xd, const int* labels_d, const std::vector<double>& h, int* clusters,
                cudaStream_t st) {
    const int n = W.n, d = W.d;
    int* bad = W.scal;
    int* dm = W.scal + 1;
    EGG_CHECK(cudaMemsetAsync(bad, 0, 4, st));
    k_label_keys<<<grid_for((size_t)n, 256), 256, 0, st>>>(labels_d, n, W.keys, W.idx, bad);
    prim::sort_pairs(W.keys, W.idx, W.keys_s, W.idx_s, n, W.sort_tmp, st);
    // clustered points: keys below 0xffffffff
    k_first_outlier<<<1, 1, 0, st>>>(W.keys_s, n, dm);
    int hs2[2];
    EGG_CHECK(cudaMemcpyAsync(hs2, bad, 8, cudaMemcpyDeviceToHost, st));
    EGG_CHECK(cudaStreamSynchronize(st));
    if (hs2[0]) throw ArgError{EGG_ERR_ARG, "labels must be -1 (outlier) or a cluster id >= 0"};
    const int m = hs2[1];
    const int outliers = n - m;
    double LM = (double)outliers * std::log2((double)n);
    double prodh = 1.0;
    for (double v : h) prodh *= v;
    double LD = (double)outliers * std::pow(2.0 * M_PI, -0.5) * prodh;
    *clusters = 0;
    if (m > 0) {
        k_heads<<<grid_for((size_t)m, 256), 256, 0, st>>>(W.keys_s, m, W.head);
        prim::inclusive_scan(W.head, W.incl, m, W.scan_tmp, st);
        k_seg_begin<<<grid_for((size_t)m, 256), 256, 0, st>>>(W.head, W.incl, m, W.begin);
        k_seg_of<<<grid_for((size_t)m, 256), 256, 0, st>>>(W.incl, m, W.seg);
        k_gather_sorted<<<grid_for((size_t)m * d, 256), 256, 0, st>>>(xd, d, W.idx_s, m, W.xs);
        int K = 0;
        EGG_CHECK(cudaMemcpyAsync(&K, W.incl + (m - 1), 4, cudaMemcpyDeviceToHost, st));
        EGG_CHECK(cudaStreamSynchronize(st));
        // begin[K] = m and the inverse bandwidths, one small upload
        std::vector<int> up(1 + d);
        up[0] = m;
        for (int l = 0; l < d; l++) {
            const float ih = (float)(1.0 / h[l]);
            memcpy(&up[1 + l], &ih, 4);
        }
        EGG_CHECK(cudaMemcpyAsync(W.begin + K, up.data(), 4, cudaMemcpyHostToDevice, st));
        EGG_CHECK(cudaMemcpyAsync(W.invh, up.data() + 1, 4 * (size_t)d, cudaMemcpyHostToDevice, st));
        const double norm = std::pow(2.0 * M_PI, -0.5 * d) / prodh;
        EGG_MDL_DISPATCH_D(d, k_kde, <<<(m + 255) / 256, 256, 0, st>>>(W.xs, m, d, W.seg, W.begin, W.invh, norm,
                                                                         W.f, W.lf));
        EGG_CHECK(cudaGetLastError());
        prim::segment_sums(W.f, W.begin, K, W.sf, st);
        prim::segment_sums(W.lf, W.begin, K, W.slf, st);
        std::vector<int> hb(K + 1);
        std::vector<double> hs(K), hl(K);
        EGG_CHECK(cudaMemcpyAsync(hb.data(), W.begin, 4 * (size_t)(K + 1), cudaMemcpyDeviceToHost, st));
        EGG_CHECK(cudaMemcpyAsync(hs.data(), W.sf, 8 * (size_t)K, cudaMemcpyDeviceToHost, st));
        EGG_CHECK(cudaMemcpyAsync(hl.data(), W.slf, 8 * (size_t)K, cudaMemcpyDeviceToHost, st));
        EGG_CHECK(cudaStreamSynchronize(st));
        for (int c = 0; c < K; c++) {
            const double sz = (double)(hb[c + 1] - hb[c]);
            LM += sz * std::log2((double)n / sz) + d / 2.0 * std::log2(sz);
            LD += hl[c] - sz * std::log2(hs[c]);
        }
        *clusters = K;
    }
    return LM - LD;
}

// The search (Sync, SynCTorch.py:349-372).
struct SearchOut {
    double nn[2];
    float step = 0.f, eps_best = 0.f;
    int candidates = 0, best = -1, clusters = 0, end_reason = 1;
    double cost_best = 0.0;
    std::vector<double> costs;
    std::vector<float> eps;
    std::vector<int> ks;
};

void mdl_search(const float* x, int n, int d, int k, int max_cand, int* labels, SearchOut& R, cudaStream_t st) {
    Arena A;
    const float* xd = device_input(A, x, (size_t)n * d, st);
    knn_mean(A, xd, n, d, k, R.nn, st);
    const std::vector<double> h = bandwidths(A, xd, n, d, st);
    // eps = NN(k); delta = NN(k+1) - eps; eps += delta, in float32 as the
    // reference's tensors are
    const float e0 = (float)R.nn[0];
    R.step = (float)R.nn[1] - e0;
    if (!(R.step > 0.f))
        throw ArgError{EGG_ERR_INPUT, "NN(k+1) equals NN(k): the eps schedule does not advance"};
    int* lab = A.get<int>((size_t)kMdlBatch * n);
    int* best_lab = A.get<int>(n);
    CostWs W(n, d);
    float eps = e0;
    bool done = false;
    while (!done && R.candidates < max_cand) {
        std::vector<egg_batch_item> items;
        for (int b = 0; b < kMdlBatch && R.candidates + b < max_cand; b++) {
            try {
                make_geom(n, d, eps);
            } catch (const ArgError&) {
                R.end_reason = 2;  // eps beyond what the grid takes: the schedule ends here
                done = true;
                break;
            }
            egg_batch_item it;
            memset(&it, 0, sizeof(it));
            it.x = xd;
            it.n = n;
            it.d = d;
            it.eps = eps;
            it.labels = lab + (size_t)b * n;
            items.push_back(it);
            eps = eps + R.step;
        }
        if (items.empty()) break;
        egg_opts o;
        memset(&o, 0, sizeof(o));
        o.batch_tune = 1;  // default launch configuration: every batch has new eps values
        run_batch(items.data(), (int)items.size(), &o, nullptr, st);
        for (size_t b = 0; b < items.size(); b++) {
            const egg_batch_item& it = items[b];
            if (it.status < 0) throw ArgError{it.status, "clustering at eps " + std::to_string(it.eps) + " failed"};
            int K = 0;
            const double cost = mdl_cost(W, xd, it.labels, h, &K, st);
            R.costs.push_back(cost);
            R.eps.push_back(it.eps);
            R.ks.push_back(K);
            if (R.best < 0 || cost < R.cost_best) {
                R.best = R.candidates;
                R.cost_best = cost;
                R.eps_best = it.eps;
                R.clusters = K;
                EGG_CHECK(cudaMemcpyAsync(best_lab, it.labels, 4 * (size_t)n, cudaMemcpyDeviceToDevice, st));
            }
            R.candidates++;
            if (K == 1) {
                R.end_reason = 0;
                done = true;
                break;
            }
        }
    }
    if (R.best < 0) throw ArgError{EGG_ERR_GEOMETRY, "eps = NN(k) is beyond what the grid takes"};
    EGG_CHECK(cudaMemcpyAsync(labels, best_lab, 4 * (size_t)n, cudaMemcpyDefault, st));
    EGG_CHECK(cudaStreamSynchronize(st));
}

}  // namespace

}  // namespace egg

using egg::ArgError;

extern "C" __attribute__((visibility("default"))) int egg_knn_mean(const float* x, int64_t n, int32_t d, int32_t k,
                                                                   double* out, void* stream) {
    return egg::guarded([&] {
        if (!x || !out) throw ArgError{EGG_ERR_ARG, "x and out must not be NULL"};
        if (k < 1 || k > egg::kKnnMaxK) throw ArgError{EGG_ERR_ARG, "k must be in [1, 31]"};
        egg::check_nd(n, d, (int64_t)k + 2);
        cudaStream_t st = (cudaStream_t)stream;
        egg::Arena A;
        const float* xd = egg::device_input(A, x, (size_t)n * d, st);
        egg::knn_mean(A, xd, (int)n, d, k, out, st);
        return EGG_OK;
    });
}

extern "C" __attribute__((visibility("default"))) int egg_mdl_cost(const float* x, int64_t n, int32_t d,
                                                                   const int32_t* labels, double* cost,
                                                                   int32_t* clusters, void* stream) {
    return egg::guarded([&] {
        if (!x || !labels || !cost) throw ArgError{EGG_ERR_ARG, "x, labels and cost must not be NULL"};
        egg::check_nd(n, d, 2);
        cudaStream_t st = (cudaStream_t)stream;
        egg::Arena A;
        const float* xd = egg::device_input(A, x, (size_t)n * d, st);
        const int* ld = labels;
        if (!egg::is_device_ptr(labels)) {
            int* t = A.get<int>((size_t)n);
            EGG_CHECK(cudaMemcpyAsync(t, labels, 4 * (size_t)n, cudaMemcpyHostToDevice, st));
            ld = t;
        }
        const std::vector<double> h = egg::bandwidths(A, xd, (int)n, d, st);
        egg::CostWs W((int)n, d);
        int K = 0;
        *cost = egg::mdl_cost(W, xd, ld, h, &K, st);
        if (clusters) *clusters = K;
        return EGG_OK;
    });
}

extern "C" __attribute__((visibility("default"))) int egg_mdl_search(const float* x, int64_t n, int32_t d, int32_t k,
                                                                     int32_t max_candidates, int32_t* labels,
                                                                     egg_mdl_stats* stats, void* stream) {
    return egg::guarded([&] {
        if (!x || !labels) throw ArgError{EGG_ERR_ARG, "x and labels must not be NULL"};
        if (k < 1 || k > egg::kKnnMaxK) throw ArgError{EGG_ERR_ARG, "k must be in [1, 31]"};
        if (max_candidates < 0 || max_candidates > 4096) throw ArgError{EGG_ERR_ARG, "max_candidates must be in [0, 4096]"};
        egg::check_nd(n, d, (int64_t)k + 2);
        cudaStream_t st = (cudaStream_t)stream;
        cudaEvent_t e0, e1;
        EGG_CHECK(cudaEventCreate(&e0));
        EGG_CHECK(cudaEventCreate(&e1));
        EGG_CHECK(cudaEventRecord(e0, st));
        egg::SearchOut R;
        try {
            egg::mdl_search(x, (int)n, d, k, max_candidates > 0 ? max_candidates : 256, labels, R, st);
        } catch (...) {
            cudaEventDestroy(e0);
            cudaEventDestroy(e1);
            throw;
        }
        EGG_CHECK(cudaEventRecord(e1, st));
        EGG_CHECK(cudaEventSynchronize(e1));
        float ms = 0.f;
        cudaEventElapsedTime(&ms, e0, e1);
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        if (stats) {
            const egg_mdl_stats in = *stats;
            memset(stats, 0, sizeof(*stats));
            stats->eps0 = R.nn[0];
            stats->eps1 = R.nn[1];
            stats->eps_step = R.step;
            stats->eps_best = R.eps_best;
            stats->candidates = R.candidates;
            stats->best = R.best;
            stats->n_clusters = R.clusters;
            stats->end_reason = R.end_reason;
            stats->cost_best = R.cost_best;
            stats->total_ms = ms;
            stats->cap = in.cap;
            stats->costs = in.costs;
            stats->eps = in.eps;
            stats->clusters = in.clusters;
            for (int c = 0; c < R.candidates && c < in.cap; c++) {
                if (in.costs) in.costs[c] = R.costs[c];
                if (in.eps) in.eps[c] = R.eps[c];
                if (in.clusters) in.clusters[c] = R.ks[c];
            }
        }
        return EGG_OK;
    });
}
