// egg_mlp.cu -- learned warm start for the synchronisation loop (no
// counterpart in the reference).
//
// A small MLP reads, for every point, its offset inside a coarse cell of side
// eps and summaries of the 3^d coarse cells around it (point count, centroid
// relative to the point, spread), and predicts the point's displacement over
// the next K iterations of the plain loop, in units of eps.  The plain loop
// then runs from the displaced positions to convergence.
//
//   features   k_fgrid_accum + k_features: a dense coarse grid filled with
//              64-bit fixed-point sums (integer atomics: the result does not
//              depend on the order of the additions), then one row of
//              feat_dim(d) values per point (192 for d = 3).
//   inference  k_mlp_infer: the three layers fused in one kernel on the
//              tensor cores (BF16 operands, FP32 accumulation, mma.sync
//              m16n8k16); a warp owns 16 points, a layer's accumulators stay
//              in registers and become the next layer's operand fragments.
//   training   FP32 kernels: tiled SGEMM, bias/ReLU, ReLU backward, column
//              sums (fixed order), MSE gradient, Adam.  The gradient of one
//              batch is exported (egg_mlp_grad) so that tests can check it
//              against a CPU computation.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <numeric>
#include <random>
#include <string>
#include <vector>

#include "eggsync.h"
#include "egg_common.cuh"
#include "egg_host_common.h"
#include "egg_mlp.h"

namespace egg {
namespace mlp {

namespace {

constexpr float kFix = 16777216.0f;  // 2^24: fixed-point scale of in-cell offsets

// ---------------------------------------------------------------------------
// features
// ---------------------------------------------------------------------------
struct FGrid {
    int d, width, ncell;
    float f;  // coarse side (= eps)
    int* cnt;
    long long* su;  // [ncell][d] sum of offsets (fixed point)
    long long* sq;  // [ncell][d] sum of squared offsets (fixed point)
};

__device__ __forceinline__ float load_x(const float* X, size_t sp, size_t sl, int p, int l) {
    return X[(size_t)p * sp + (size_t)l * sl];
}

__device__ __forceinline__ int coarse_of(float x, float f, int width, float& u) {
    const float q = __fdiv_rn(x, f);
    int c = (int)q;
    c = c < 0 ? 0 : (c > width - 1 ? width - 1 : c);
    u = __fsub_rn(q, (float)c);
    return c;
}

__global__ void k_fgrid_clear(FGrid G) {
    for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < (size_t)G.ncell;
         t += (size_t)gridDim.x * blockDim.x) {
        G.cnt[t] = 0;
        for (int l = 0; l < G.d; l++) {
            G.su[t * G.d + l] = 0;
            G.sq[t * G.d + l] = 0;
        }
    }
}

__global__ void k_fgrid_accum(FGrid G, const float* __restrict__ X, size_t sp, size_t sl, int n) {
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += gridDim.x * blockDim.x) {
        int cell = 0, mul = 1;
        long long U[kMaxWarmDims], Q[kMaxWarmDims];
        for (int l = 0; l < G.d; l++) {
            float u;
            const int c = coarse_of(load_x(X, sp, sl, p, l), G.f, G.width, u);
            cell += c * mul;
            mul *= G.width;
            U[l] = __float2ll_rn(u * kFix);
            Q[l] = __float2ll_rn(u * u * kFix);
        }
        atomicAdd(G.cnt + cell, 1);
        for (int l = 0; l < G.d; l++) {
            atomicAdd(reinterpret_cast<unsigned long long*>(G.su + (size_t)cell * G.d + l), (unsigned long long)U[l]);
            atomicAdd(reinterpret_cast<unsigned long long*>(G.sq + (size_t)cell * G.d + l), (unsigned long long)Q[l]);
        }
    }
}

// One feature row per point: [u_0..u_{d-1}], then for every neighbour offset
// o in {-1,0,1}^d (o_0 fastest): log1p(count)/8, centroid - point (d values,
// eps units), standard deviation of the offsets (d values); zeros for empty
// or outside cells; zero padding up to the row width fp.
template <typename T>
__global__ void k_features(FGrid G, const float* __restrict__ X, size_t sp, size_t sl, int n, T* __restrict__ out,
                           int fp) {
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += gridDim.x * blockDim.x) {
        T* row = out + (size_t)p * fp;
        float u[kMaxWarmDims];
        int c[kMaxWarmDims];
        const int d = G.d;
        for (int l = 0; l < d; l++) c[l] = coarse_of(load_x(X, sp, sl, p, l), G.f, G.width, u[l]);
        int k = 0;
        for (int l = 0; l < d; l++) row[k++] = (T)u[l];
        int nb = 1;
        for (int l = 0; l < d; l++) nb *= 3;
        for (int s = 0; s < nb; s++) {
            int o[kMaxWarmDims];
            int rem = s, cell = 0, mul = 1;
            bool inb = true;
            for (int l = 0; l < d; l++) {
                o[l] = rem % 3 - 1;
                rem /= 3;
                const int v = c[l] + o[l];
                inb = inb && v >= 0 && v < G.width;
                cell += v * mul;
                mul *= G.width;
            }
            const int cnt = inb ? G.cnt[cell] : 0;
            if (cnt == 0) {
                for (int j = 0; j < 1 + 2 * d; j++) row[k++] = (T)0.f;
                continue;
            }
            row[k++] = (T)(log1pf((float)cnt) * 0.125f);
            double var[kMaxWarmDims];
            for (int l = 0; l < d; l++) {
                const double m = (double)G.su[(size_t)cell * d + l] / ((double)cnt * kFix);
                const double e2 = (double)G.sq[(size_t)cell * d + l] / ((double)cnt * kFix);
                var[l] = fmax(0.0, e2 - m * m);
                row[k++] = (T)(float)(m + (double)o[l] - (double)u[l]);
            }
            for (int l = 0; l < d; l++) row[k++] = (T)(float)sqrt(var[l]);
        }
        for (; k < fp; k++) row[k] = (T)0.f;
    }
}

// ---------------------------------------------------------------------------
// inference: fused 3-layer MLP on the tensor cores
// ---------------------------------------------------------------------------
__device__ __forceinline__ void mma_bf16(float (&c)[4], unsigned a0, unsigned a1, unsigned a2, unsigned a3,
                                         unsigned b0, unsigned b1) {
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
        "{%0,%1,%2,%3};\n"
        : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
        : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b0), "r"(b1));
}

__device__ __forceinline__ unsigned pack_bf16(float lo, float hi) {
    __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
    return *reinterpret_cast<unsigned*>(&v);
}

// packed weights on the device: W1t [kHidden][fp], W2t [kHidden][kHidden],
// W3t [8][kHidden] (bf16, output-major so that a B fragment's k pairs are
// adjacent), biases FP32 [kHidden], [kHidden], [8]
struct Packed {
    __nv_bfloat16* w1t;
    __nv_bfloat16* w2t;
    __nv_bfloat16* w3t;
    float* b1;
    float* b2;
    float* b3;
    int fp;
    int dout;
};

constexpr int kInferWarps = 4;

__host__ __device__ inline int w1_stride(int fp) { return fp + 8; }
constexpr int kW2Stride = kHidden + 8;

__host__ __device__ inline size_t infer_smem(int fp) {
    return sizeof(__nv_bfloat16) * ((size_t)kHidden * w1_stride(fp) + (size_t)kHidden * kW2Stride + 8 * kW2Stride) +
           sizeof(float) * (2 * kHidden + 8);
}

__global__ void __launch_bounds__(32 * kInferWarps) k_mlp_infer(Packed P, const __nv_bfloat16* __restrict__ feats,
                                                                 int n, float* __restrict__ out) {
    extern __shared__ __align__(16) unsigned char smem[];
    const int fp = P.fp, s1 = w1_stride(fp);
    __nv_bfloat16* W1 = reinterpret_cast<__nv_bfloat16*>(smem);
    __nv_bfloat16* W2 = W1 + (size_t)kHidden * s1;
    __nv_bfloat16* W3 = W2 + (size_t)kHidden * kW2Stride;
    float* B1 = reinterpret_cast<float*>(W3 + 8 * kW2Stride);
    float* B2 = B1 + kHidden;
    float* B3 = B2 + kHidden;
    for (int t = threadIdx.x; t < kHidden * fp; t += blockDim.x) W1[(t / fp) * s1 + t % fp] = P.w1t[t];
    for (int t = threadIdx.x; t < kHidden * kHidden; t += blockDim.x)
        W2[(t / kHidden) * kW2Stride + t % kHidden] = P.w2t[t];
    for (int t = threadIdx.x; t < 8 * kHidden; t += blockDim.x) W3[(t / kHidden) * kW2Stride + t % kHidden] = P.w3t[t];
    for (int t = threadIdx.x; t < kHidden; t += blockDim.x) {
        B1[t] = P.b1[t];
        B2[t] = P.b2[t];
    }
    if (threadIdx.x < 8) B3[threadIdx.x] = P.b3[threadIdx.x];
    __syncthreads();

    const int lane = threadIdx.x & 31, g = lane >> 2, t4 = lane & 3;
    const int warp = blockIdx.x * kInferWarps + (threadIdx.x >> 5);
    const int nwarps = gridDim.x * kInferWarps;
    const int tiles = (n + 15) / 16;
    for (int tile = warp; tile < tiles; tile += nwarps) {
        const int r0 = tile * 16 + g, r1 = r0 + 8;
        const bool v0 = r0 < n, v1 = r1 < n;
        const unsigned* f0 = reinterpret_cast<const unsigned*>(feats + (size_t)(v0 ? r0 : 0) * fp);
        const unsigned* f1 = reinterpret_cast<const unsigned*>(feats + (size_t)(v1 ? r1 : 0) * fp);
        // layer 1
        float acc[kHidden / 8][4];
#pragma unroll
        for (int j = 0; j < kHidden / 8; j++) acc[j][0] = acc[j][1] = acc[j][2] = acc[j][3] = 0.f;
        for (int kc = 0; kc < fp / 16; kc++) {
            const int kw = kc * 8 + t4;  // 32-bit word index of columns 16kc + 2t4
            const unsigned a0 = v0 ? __ldg(f0 + kw) : 0u, a1 = v1 ? __ldg(f1 + kw) : 0u;
            const unsigned a2 = v0 ? __ldg(f0 + kw + 4) : 0u, a3 = v1 ? __ldg(f1 + kw + 4) : 0u;
#pragma unroll
            for (int j = 0; j < kHidden / 8; j++) {
                const unsigned* wr = reinterpret_cast<const unsigned*>(W1 + (size_t)(8 * j + g) * s1 + 16 * kc);
                mma_bf16(acc[j], a0, a1, a2, a3, wr[t4], wr[t4 + 4]);
            }
        }
        unsigned A[kHidden / 16][4];
#pragma unroll
        for (int j = 0; j < kHidden / 8; j++) {
            const float bx = B1[8 * j + 2 * t4], by = B1[8 * j + 2 * t4 + 1];
            const unsigned lo = pack_bf16(fmaxf(acc[j][0] + bx, 0.f), fmaxf(acc[j][1] + by, 0.f));
            const unsigned hi = pack_bf16(fmaxf(acc[j][2] + bx, 0.f), fmaxf(acc[j][3] + by, 0.f));
            A[j >> 1][(j & 1) * 2 + 0] = lo;
            A[j >> 1][(j & 1) * 2 + 1] = hi;
        }
        // layer 2
#pragma unroll
        for (int j = 0; j < kHidden / 8; j++) acc[j][0] = acc[j][1] = acc[j][2] = acc[j][3] = 0.f;
#pragma unroll
        for (int kc = 0; kc < kHidden / 16; kc++) {
#pragma unroll
            for (int j = 0; j < kHidden / 8; j++) {
                const unsigned* wr = reinterpret_cast<const unsigned*>(W2 + (size_t)(8 * j + g) * kW2Stride + 16 * kc);
                mma_bf16(acc[j], A[kc][0], A[kc][1], A[kc][2], A[kc][3], wr[t4], wr[t4 + 4]);
            }
        }
#pragma unroll
        for (int j = 0; j < kHidden / 8; j++) {
            const float bx = B2[8 * j + 2 * t4], by = B2[8 * j + 2 * t4 + 1];
            A[j >> 1][(j & 1) * 2 + 0] = pack_bf16(fmaxf(acc[j][0] + bx, 0.f), fmaxf(acc[j][1] + by, 0.f));
            A[j >> 1][(j & 1) * 2 + 1] = pack_bf16(fmaxf(acc[j][2] + bx, 0.f), fmaxf(acc[j][3] + by, 0.f));
        }
        // layer 3 (outputs padded to 8)
        float o[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll
        for (int kc = 0; kc < kHidden / 16; kc++) {
            const unsigned* wr = reinterpret_cast<const unsigned*>(W3 + (size_t)g * kW2Stride + 16 * kc);
            mma_bf16(o, A[kc][0], A[kc][1], A[kc][2], A[kc][3], wr[t4], wr[t4 + 4]);
        }
        const int c0 = 2 * t4, c1 = 2 * t4 + 1;
        if (v0 && c0 < P.dout) out[(size_t)r0 * P.dout + c0] = o[0] + B3[c0];
        if (v0 && c1 < P.dout) out[(size_t)r0 * P.dout + c1] = o[1] + B3[c1];
        if (v1 && c0 < P.dout) out[(size_t)r1 * P.dout + c0] = o[2] + B3[c0];
        if (v1 && c1 < P.dout) out[(size_t)r1 * P.dout + c1] = o[3] + B3[c1];
    }
}

// fp32 [in][out] (row-major, as trained) -> bf16 [out_pad][in_pad], zero padded
__global__ void k_pack_t(const float* __restrict__ w, int in, int outn, __nv_bfloat16* __restrict__ wt, int in_pad,
                         int out_pad) {
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < in_pad * out_pad; t += gridDim.x * blockDim.x) {
        const int o = t / in_pad, i = t % in_pad;
        wt[t] = __float2bfloat16_rn(o < outn && i < in ? w[(size_t)i * outn + o] : 0.f);
    }
}

__global__ void k_to_bf16(const float* __restrict__ a, __nv_bfloat16* __restrict__ b, size_t cnt) {
    for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < cnt; t += (size_t)gridDim.x * blockDim.x)
        b[t] = __float2bfloat16_rn(a[t]);
}

// x <- clamp(x + eps * delta, 0, 1) on the SoA positions of the loop, for
// the points with at least min_count points in their 3^d coarse cells
__global__ void k_apply(FGrid G, float* X, size_t ns, int n, const float* __restrict__ delta, float eps,
                        int min_count) {
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += gridDim.x * blockDim.x) {
        const int d = G.d;
        int c[kMaxWarmDims];
        for (int l = 0; l < d; l++) {
            float u;
            c[l] = coarse_of(X[(size_t)l * ns + p], G.f, G.width, u);
        }
        int nb = 1;
        for (int l = 0; l < d; l++) nb *= 3;
        int total = 0;
        for (int s = 0; s < nb && total < min_count; s++) {
            int rem = s, cell = 0, mul = 1;
            bool inb = true;
            for (int l = 0; l < d; l++) {
                const int v = c[l] + rem % 3 - 1;
                rem /= 3;
                inb = inb && v >= 0 && v < G.width;
                cell += v * mul;
                mul *= G.width;
            }
            if (inb) total += G.cnt[cell];
        }
        if (total < min_count) continue;
        for (int l = 0; l < d; l++) {
            float* x = X + (size_t)l * ns + p;
            *x = fminf(fmaxf(__fmaf_rn(eps, delta[(size_t)p * d + l], *x), 0.f), 1.f);
        }
    }
}

// ---------------------------------------------------------------------------
// training (FP32)
// ---------------------------------------------------------------------------
// C[M][N] = op(A)[M][K] . op(B)[K][N] (+ beta C); op(A)[m][k] = TA ? A[k][m] : A[m][k]
template <bool TA, bool TB>
__global__ void __launch_bounds__(256) k_sgemm(int M, int N, int K, const float* __restrict__ A, int lda,
                                               const float* __restrict__ B, int ldb, float* __restrict__ C, int ldc,
                                               float beta) {
    __shared__ float As[16][65];
    __shared__ float Bs[16][65];
    const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
    const int m0 = blockIdx.y * 64, n0 = blockIdx.x * 64;
    float acc[4][4] = {};
    for (int k0 = 0; k0 < K; k0 += 16) {
        for (int i = 0; i < 4; i++) {
            const int idx = threadIdx.x + 256 * i;
            const int kk = TA ? idx / 64 : idx % 16, mm = TA ? idx % 64 : idx / 16;
            const int m = m0 + mm, k = k0 + kk;
            float v = 0.f;
            if (m < M && k < K) v = TA ? A[(size_t)k * lda + m] : A[(size_t)m * lda + k];
            As[kk][mm] = v;
            const int kb = TB ? idx % 16 : idx / 64, nn = TB ? idx / 16 : idx % 64;
            const int nb = n0 + nn, kb2 = k0 + kb;
            float u = 0.f;
            if (nb < N && kb2 < K) u = TB ? B[(size_t)nb * ldb + kb2] : B[(size_t)kb2 * ldb + nb];
            Bs[kb][nn] = u;
        }
        __syncthreads();
#pragma unroll
        for (int kk = 0; kk < 16; kk++) {
            float a[4], b[4];
#pragma unroll
            for (int i = 0; i < 4; i++) {
                a[i] = As[kk][ty + 16 * i];
                b[i] = Bs[kk][tx + 16 * i];
            }
#pragma unroll
            for (int i = 0; i < 4; i++)
#pragma unroll
                for (int j = 0; j < 4; j++) acc[i][j] = fmaf(a[i], b[j], acc[i][j]);
        }
        __syncthreads();
    }
    for (int i = 0; i < 4; i++)
        for (int j = 0; j < 4; j++) {
            const int m = m0 + ty + 16 * i, nn = n0 + tx + 16 * j;
            if (m < M && nn < N) {
                float* c = C + (size_t)m * ldc + nn;
                *c = acc[i][j] + (beta != 0.f ? beta * *c : 0.f);
            }
        }
}

__global__ void k_bias_act(float* H, int M, int N, const float* __restrict__ b, int relu) {
    for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < (size_t)M * N;
         t += (size_t)gridDim.x * blockDim.x) {
        const float v = H[t] + b[t % N];
        H[t] = relu ? fmaxf(v, 0.f) : v;
    }
}

__global__ void k_relu_back(float* dH, const float* __restrict__ H, size_t cnt) {
    for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < cnt; t += (size_t)gridDim.x * blockDim.x)
        if (!(H[t] > 0.f)) dH[t] = 0.f;
}

// out[n] = sum_m X[m][n], each column summed in row order
__global__ void k_colsum(const float* __restrict__ X, int M, int N, float* out) {
    const int nn = blockIdx.x * blockDim.x + threadIdx.x;
    if (nn >= N) return;
    float s = 0.f;
    for (int m = 0; m < M; m++) s += X[(size_t)m * N + nn];
    out[nn] = s;
}

// dY = 2 (Y - T) / (M * N); per-block partial sums of (Y - T)^2
__global__ void k_mse(const float* __restrict__ Y, const float* __restrict__ T, int M, int N, float* dY,
                      double* partial) {
    __shared__ double s[256];
    double acc = 0.0;
    const float scale = 2.f / ((float)M * (float)N);
    for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < (size_t)M * N;
         t += (size_t)gridDim.x * blockDim.x) {
        const float e = Y[t] - T[t];
        dY[t] = scale * e;
        acc += (double)e * e;
    }
    s[threadIdx.x] = acc;
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
        if (threadIdx.x < o) s[threadIdx.x] += s[threadIdx.x + o];
        __syncthreads();
    }
    if (threadIdx.x == 0) partial[blockIdx.x] = s[0];
}

__global__ void k_adam(float* p, const float* __restrict__ gr, float* m, float* v, size_t cnt, float lr, float b1,
                       float b2, float c1, float c2) {
    for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < cnt; t += (size_t)gridDim.x * blockDim.x) {
        const float gg = gr[t];
        m[t] = b1 * m[t] + (1.f - b1) * gg;
        v[t] = b2 * v[t] + (1.f - b2) * gg * gg;
        p[t] -= lr * (m[t] / c1) / (sqrtf(v[t] / c2) + 1e-8f);
    }
}

__global__ void k_gather(const float* __restrict__ src, const int* __restrict__ idx, int rows, int cols,
                         float* __restrict__ dst) {
    for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < (size_t)rows * cols;
         t += (size_t)gridDim.x * blockDim.x) {
        const int r = (int)(t / cols), c = (int)(t % cols);
        dst[t] = src[(size_t)idx[r] * cols + c];
    }
}

int grid_for(size_t cnt, int threads = 256) {
    size_t b = (cnt + threads - 1) / threads;
    return (int)std::max<size_t>(1, std::min<size_t>(b, 148 * 16));
}

template <bool TA, bool TB>
void sgemm(int M, int N, int K, const float* A, int lda, const float* B, int ldb, float* C, int ldc, float beta,
           cudaStream_t st) {
    dim3 grid((N + 63) / 64, (M + 63) / 64);
    k_sgemm<TA, TB><<<grid, 256, 0, st>>>(M, N, K, A, lda, B, ldb, C, ldc, beta);
}

// parameter block on the device: w1 [F][H], b1 [H], w2 [H][H], b2 [H], w3 [H][D], b3 [D]
struct Params {
    int F, H, D;
    float* base;
    size_t count() const { return (size_t)F * H + H + (size_t)H * H + H + (size_t)H * D + D; }
    float* w1() const { return base; }
    float* b1() const { return w1() + (size_t)F * H; }
    float* w2() const { return b1() + H; }
    float* b2() const { return w2() + (size_t)H * H; }
    float* w3() const { return b2() + H; }
    float* b3() const { return w3() + (size_t)H * D; }
};

void check_model(const egg_mlp& m) {
    if (m.d < 1 || m.d > kMaxWarmDims) throw ArgError{EGG_ERR_ARG, "warm-start model: d must be 1, 2 or 3"};
    if (m.d_in != feat_dim(m.d)) throw ArgError{EGG_ERR_ARG, "warm-start model: d_in must be egg_mlp_feature_dim(d)"};
    if (m.hidden != kHidden) throw ArgError{EGG_ERR_ARG, "warm-start model: hidden must be 128"};
    if (!m.w1 || !m.b1 || !m.w2 || !m.b2 || !m.w3 || !m.b3) throw ArgError{EGG_ERR_ARG, "warm-start model: NULL weight"};
}

void upload_params(const egg_mlp& m, const Params& P, cudaStream_t st) {
    auto up = [&](float* dst, const float* src, size_t cnt) {
        EGG_CHECK(cudaMemcpyAsync(dst, src, 4 * cnt, is_device_ptr(src) ? cudaMemcpyDeviceToDevice
                                                                          : cudaMemcpyHostToDevice, st));
    };
    up(P.w1(), m.w1, (size_t)P.F * P.H);
    up(P.b1(), m.b1, P.H);
    up(P.w2(), m.w2, (size_t)P.H * P.H);
    up(P.b2(), m.b2, P.H);
    up(P.w3(), m.w3, (size_t)P.H * P.D);
    up(P.b3(), m.b3, P.D);
}

void download_params(const Params& P, egg_mlp& m, cudaStream_t st) {
    auto dn = [&](float* dst, const float* src, size_t cnt) {
        EGG_CHECK(cudaMemcpyAsync(dst, src, 4 * cnt, cudaMemcpyDefault, st));
    };
    dn(m.w1, P.w1(), (size_t)P.F * P.H);
    dn(m.b1, P.b1(), P.H);
    dn(m.w2, P.w2(), (size_t)P.H * P.H);
    dn(m.b2, P.b2(), P.H);
    dn(m.w3, P.w3(), (size_t)P.H * P.D);
    dn(m.b3, P.b3(), P.D);
}

// device scratch of the training and gradient entry points
struct Scratch {
    std::vector<void*> ptrs;
    ~Scratch() {
        for (void* p : ptrs) cudaFree(p);
    }
    template <typename T>
    T* get(size_t cnt) {
        void* p = nullptr;
        EGG_CHECK(dev_alloc((void**)&p, std::max<size_t>(cnt, 1) * sizeof(T)));
        ptrs.push_back(p);
        return (T*)p;
    }
};

// forward + backward of one batch X [M][F], T [M][D]; grads into G (same
// layout as P); returns the batch's sum of squared errors on the device
void batch_grad(const Params& P, const Params& G, const float* X, const float* T, int M, float* H1, float* H2,
                float* Y, float* dY, float* dH2, float* dH1, double* partial, int nparts, cudaStream_t st) {
    const int F = P.F, H = P.H, D = P.D;
    sgemm<false, false>(M, H, F, X, F, P.w1(), H, H1, H, 0.f, st);
    k_bias_act<<<grid_for((size_t)M * H), 256, 0, st>>>(H1, M, H, P.b1(), 1);
    sgemm<false, false>(M, H, H, H1, H, P.w2(), H, H2, H, 0.f, st);
    k_bias_act<<<grid_for((size_t)M * H), 256, 0, st>>>(H2, M, H, P.b2(), 1);
    sgemm<false, false>(M, D, H, H2, H, P.w3(), D, Y, D, 0.f, st);
    k_bias_act<<<grid_for((size_t)M * D), 256, 0, st>>>(Y, M, D, P.b3(), 0);
    k_mse<<<nparts, 256, 0, st>>>(Y, T, M, D, dY, partial);
    // layer 3
    sgemm<true, false>(H, D, M, H2, H, dY, D, G.w3(), D, 0.f, st);
    k_colsum<<<(D + 127) / 128, 128, 0, st>>>(dY, M, D, G.b3());
    sgemm<false, true>(M, H, D, dY, D, P.w3(), D, dH2, H, 0.f, st);
    k_relu_back<<<grid_for((size_t)M * H), 256, 0, st>>>(dH2, H2, (size_t)M * H);
    // layer 2
    sgemm<true, false>(H, H, M, H1, H, dH2, H, G.w2(), H, 0.f, st);
    k_colsum<<<(H + 127) / 128, 128, 0, st>>>(dH2, M, H, G.b2());
    sgemm<false, true>(M, H, H, dH2, H, P.w2(), H, dH1, H, 0.f, st);
    k_relu_back<<<grid_for((size_t)M * H), 256, 0, st>>>(dH1, H1, (size_t)M * H);
    // layer 1
    sgemm<true, false>(F, H, M, X, F, dH1, H, G.w1(), H, 0.f, st);
    k_colsum<<<(H + 127) / 128, 128, 0, st>>>(dH1, M, H, G.b1());
}

constexpr int kLossParts = 64;

}  // namespace

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------
FGrid features(const float* X, size_t sp, size_t sl, int n, int d, float eps, void* out, bool bf16, int fp,
               Buffers& B, cudaStream_t st) {
    FGrid G;
    G.d = d;
    G.f = eps;
    G.width = std::max(1, (int)std::ceil(1.0 / (double)eps));
    double nc = std::pow((double)G.width, (double)d);
    if (nc > 3.0e7) throw ArgError{EGG_ERR_GEOMETRY, "warm start: eps too small for the coarse feature grid"};
    G.ncell = (int)nc;
    const size_t need = (size_t)G.ncell * (4 + 16 * (size_t)d);
    if (need > B.grid_cap) {
        if (B.grid) EGG_CHECK(cudaFree(B.grid));
        B.grid = nullptr;
        B.grid_cap = 0;
        EGG_CHECK(dev_alloc((void**)&B.grid, need));
        B.grid_cap = need;
    }
    G.su = (long long*)B.grid;
    G.sq = G.su + (size_t)G.ncell * d;
    G.cnt = (int*)(G.sq + (size_t)G.ncell * d);
    k_fgrid_clear<<<grid_for(G.ncell), 256, 0, st>>>(G);
    k_fgrid_accum<<<grid_for(n), 256, 0, st>>>(G, X, sp, sl, n);
    if (bf16)
        k_features<__nv_bfloat16><<<grid_for(n, 128), 128, 0, st>>>(G, X, sp, sl, n, (__nv_bfloat16*)out, fp);
    else
        k_features<float><<<grid_for(n, 128), 128, 0, st>>>(G, X, sp, sl, n, (float*)out, fp);
    return G;
}

void infer(const egg_mlp& m, const __nv_bfloat16* feats, int n, float* out, Buffers& B, cudaStream_t st) {
    check_model(m);
    const int fp = feat_pad(m.d), F = feat_dim(m.d);
    // weights: fp32 on the device, then packed bf16
    Params P{F, kHidden, m.d, nullptr};
    const size_t pcount = P.count();
    const size_t wbytes = 4 * pcount + 2 * ((size_t)kHidden * fp + (size_t)kHidden * kHidden + 8 * kHidden) + 4 * 8;
    if (wbytes > B.w_cap) {
        if (B.w) EGG_CHECK(cudaFree(B.w));
        B.w = nullptr;
        B.w_cap = 0;
        EGG_CHECK(dev_alloc((void**)&B.w, wbytes));
        B.w_cap = wbytes;
    }
    P.base = (float*)B.w;
    upload_params(m, P, st);
    Packed K;
    K.w1t = (__nv_bfloat16*)(P.base + pcount);
    K.w2t = K.w1t + (size_t)kHidden * fp;
    K.w3t = K.w2t + (size_t)kHidden * kHidden;
    K.b3 = (float*)(K.w3t + 8 * kHidden);
    K.b1 = P.b1();
    K.b2 = P.b2();
    K.fp = fp;
    K.dout = m.d;
    k_pack_t<<<grid_for((size_t)kHidden * fp), 256, 0, st>>>(P.w1(), F, kHidden, K.w1t, fp, kHidden);
    k_pack_t<<<grid_for((size_t)kHidden * kHidden), 256, 0, st>>>(P.w2(), kHidden, kHidden, K.w2t, kHidden, kHidden);
    k_pack_t<<<grid_for(8 * kHidden), 256, 0, st>>>(P.w3(), kHidden, m.d, K.w3t, kHidden, 8);
    EGG_CHECK(cudaMemsetAsync(K.b3, 0, 4 * 8, st));
    EGG_CHECK(cudaMemcpyAsync(K.b3, P.b3(), 4 * m.d, cudaMemcpyDeviceToDevice, st));
    const size_t smem = infer_smem(fp);
    EGG_CHECK(cudaFuncSetAttribute(k_mlp_infer, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    const int tiles = (n + 15) / 16;
    const int blocks = std::max(1, std::min((tiles + kInferWarps - 1) / kInferWarps, 148 * 2));
    k_mlp_infer<<<blocks, 32 * kInferWarps, smem, st>>>(K, feats, n, out);
}


void release(Buffers& B) {
    if (B.grid) cudaFree(B.grid);
    if (B.feats) cudaFree(B.feats);
    if (B.w) cudaFree(B.w);
    if (B.delta) cudaFree(B.delta);
    B = Buffers();
}

void ensure(void** p, size_t* cap, size_t bytes) {
    if (bytes <= *cap) return;
    if (*p) EGG_CHECK(cudaFree(*p));
    *p = nullptr;
    *cap = 0;
    EGG_CHECK(dev_alloc((void**)p, bytes));
    *cap = bytes;
}

void warm_start(const egg_mlp& m, float* Xn, size_t ns, int n, int d, float eps, Buffers& B, cudaStream_t st) {
    check_model(m);
    if (m.d != d) throw ArgError{EGG_ERR_ARG, "warm-start model was trained for another dimension"};
    const int fp = feat_pad(d);
    ensure(&B.feats, &B.feats_cap, 2 * (size_t)n * fp);
    ensure((void**)&B.delta, &B.delta_cap, 4 * (size_t)n * d);
    const FGrid G = features(Xn, 1, ns, n, d, eps, B.feats, true, fp, B, st);
    infer(m, (const __nv_bfloat16*)B.feats, n, B.delta, B, st);
    k_apply<<<grid_for(n), 256, 0, st>>>(G, Xn, ns, n, B.delta, eps, std::max(0, m.min_count));
}

namespace {

Buffers g_buf;  // entry points below (serialised by the library mutex)

const float* to_device(const float* p, size_t cnt, Scratch& S, cudaStream_t st) {
    if (is_device_ptr(p)) return p;
    float* d = S.get<float>(cnt);
    EGG_CHECK(cudaMemcpyAsync(d, p, 4 * cnt, cudaMemcpyHostToDevice, st));
    return d;
}

}  // namespace

int api_features(const float* x, int64_t n, int32_t d, float eps, float* feats) {
    if (!x || !feats) throw ArgError{EGG_ERR_ARG, "x and feats must not be NULL"};
    if (n < 1 || n > (1 << 28)) throw ArgError{EGG_ERR_ARG, "n out of range"};
    if (d < 1 || d > kMaxWarmDims) throw ArgError{EGG_ERR_ARG, "d must be 1, 2 or 3"};
    if (!(eps > 0.f) || !std::isfinite(eps)) throw ArgError{EGG_ERR_ARG, "eps must be positive and finite"};
    cudaStream_t st = 0;
    Scratch S;
    const int fp = feat_pad(d);
    const float* xd = to_device(x, (size_t)n * d, S, st);
    const bool dev_out = is_device_ptr(feats);
    float* fo = dev_out ? feats : S.get<float>((size_t)n * fp);
    features(xd, d, 1, (int)n, d, eps, fo, false, fp, g_buf, st);
    if (!dev_out) EGG_CHECK(cudaMemcpyAsync(feats, fo, 4 * (size_t)n * fp, cudaMemcpyDeviceToHost, st));
    EGG_CHECK(cudaStreamSynchronize(st));
    EGG_CHECK(cudaGetLastError());
    return EGG_OK;
}

int api_forward(const egg_mlp* m, const float* feats, int64_t n, float* out) {
    if (!m || !feats || !out) throw ArgError{EGG_ERR_ARG, "NULL argument"};
    check_model(*m);
    if (n < 1 || n > (1 << 28)) throw ArgError{EGG_ERR_ARG, "n out of range"};
    cudaStream_t st = 0;
    Scratch S;
    const int fp = feat_pad(m->d);
    const float* fd = to_device(feats, (size_t)n * fp, S, st);
    __nv_bfloat16* fb = S.get<__nv_bfloat16>((size_t)n * fp);
    k_to_bf16<<<grid_for((size_t)n * fp), 256, 0, st>>>(fd, fb, (size_t)n * fp);
    const bool dev_out = is_device_ptr(out);
    float* od = dev_out ? out : S.get<float>((size_t)n * m->d);
    infer(*m, fb, (int)n, od, g_buf, st);
    if (!dev_out) EGG_CHECK(cudaMemcpyAsync(out, od, 4 * (size_t)n * m->d, cudaMemcpyDeviceToHost, st));
    EGG_CHECK(cudaStreamSynchronize(st));
    EGG_CHECK(cudaGetLastError());
    return EGG_OK;
}

int api_grad(const egg_mlp* m, const float* feats, const float* targets, int64_t n, egg_mlp* grad, double* loss) {
    if (!m || !feats || !targets || !grad) throw ArgError{EGG_ERR_ARG, "NULL argument"};
    check_model(*m);
    if (n < 1 || n > (1 << 20)) throw ArgError{EGG_ERR_ARG, "n out of range"};
    cudaStream_t st = 0;
    Scratch S;
    const int F = feat_dim(m->d), fp = feat_pad(m->d), H = kHidden, D = m->d, M = (int)n;
    // the host feature rows are padded to fp: compact them to F columns
    const float* fd = to_device(feats, (size_t)n * fp, S, st);
    float* X = S.get<float>((size_t)M * F);
    EGG_CHECK(cudaMemcpy2DAsync(X, 4 * F, fd, 4 * fp, 4 * F, M, cudaMemcpyDeviceToDevice, st));
    const float* T = to_device(targets, (size_t)n * D, S, st);
    Params P{F, H, D, S.get<float>(Params{F, H, D, nullptr}.count())};
    Params G{F, H, D, S.get<float>(P.count())};
    upload_params(*m, P, st);
    float* H1 = S.get<float>((size_t)M * H);
    float* H2 = S.get<float>((size_t)M * H);
    float* Y = S.get<float>((size_t)M * D);
    float* dY = S.get<float>((size_t)M * D);
    float* dH2 = S.get<float>((size_t)M * H);
    float* dH1 = S.get<float>((size_t)M * H);
    double* part = S.get<double>(kLossParts);
    batch_grad(P, G, X, T, M, H1, H2, Y, dY, dH2, dH1, part, kLossParts, st);
    download_params(G, *grad, st);
    std::vector<double> hp(kLossParts);
    EGG_CHECK(cudaMemcpyAsync(hp.data(), part, 8 * kLossParts, cudaMemcpyDeviceToHost, st));
    EGG_CHECK(cudaStreamSynchronize(st));
    EGG_CHECK(cudaGetLastError());
    if (loss) {
        double s = 0.0;
        for (double v : hp) s += v;
        *loss = s / ((double)M * D);
    }
    return EGG_OK;
}

int api_train(egg_mlp* m, const float* feats, const float* targets, int64_t n, const egg_mlp_train_opts* o,
              double* epoch_loss) {
    if (!m || !feats || !targets || !o) throw ArgError{EGG_ERR_ARG, "NULL argument"};
    check_model(*m);
    if (n < 1 || n > (1 << 27)) throw ArgError{EGG_ERR_ARG, "n out of range"};
    if (o->epochs < 1 || o->batch < 16 || o->batch > 65536 || !(o->lr > 0.f))
        throw ArgError{EGG_ERR_ARG, "train options: epochs >= 1, 16 <= batch <= 65536, lr > 0"};
    cudaStream_t st = 0;
    Scratch S;
    const int F = feat_dim(m->d), fp = feat_pad(m->d), H = kHidden, D = m->d;
    const float* fd = to_device(feats, (size_t)n * fp, S, st);
    float* Xall = S.get<float>((size_t)n * F);
    EGG_CHECK(cudaMemcpy2DAsync(Xall, 4 * F, fd, 4 * fp, 4 * F, n, cudaMemcpyDeviceToDevice, st));
    const float* Tall = to_device(targets, (size_t)n * D, S, st);
    Params P{F, H, D, S.get<float>(Params{F, H, D, nullptr}.count())};
    Params G{F, H, D, S.get<float>(P.count())};
    float* mom = S.get<float>(P.count());
    float* vel = S.get<float>(P.count());
    EGG_CHECK(cudaMemsetAsync(mom, 0, 4 * P.count(), st));
    EGG_CHECK(cudaMemsetAsync(vel, 0, 4 * P.count(), st));
    upload_params(*m, P, st);
    const int Bm = o->batch;
    float* X = S.get<float>((size_t)Bm * F);
    float* T = S.get<float>((size_t)Bm * D);
    float* H1 = S.get<float>((size_t)Bm * H);
    float* H2 = S.get<float>((size_t)Bm * H);
    float* Y = S.get<float>((size_t)Bm * D);
    float* dY = S.get<float>((size_t)Bm * D);
    float* dH2 = S.get<float>((size_t)Bm * H);
    float* dH1 = S.get<float>((size_t)Bm * H);
    const int nb = (int)(n / Bm);
    if (nb < 1) throw ArgError{EGG_ERR_ARG, "fewer samples than one batch"};
    double* part = S.get<double>((size_t)kLossParts * nb);
    int* idx = S.get<int>((size_t)nb * Bm);
    std::vector<int> perm(n);
    std::mt19937_64 rng((unsigned long long)o->seed);
    std::vector<double> hp((size_t)kLossParts * nb);
    int step = 0;
    for (int e = 0; e < o->epochs; e++) {
        std::iota(perm.begin(), perm.end(), 0);
        std::shuffle(perm.begin(), perm.end(), rng);
        EGG_CHECK(cudaMemcpyAsync(idx, perm.data(), 4 * (size_t)nb * Bm, cudaMemcpyHostToDevice, st));
        // cosine decay of the learning rate over the run
        for (int b = 0; b < nb; b++) {
            k_gather<<<grid_for((size_t)Bm * F), 256, 0, st>>>(Xall, idx + (size_t)b * Bm, Bm, F, X);
            k_gather<<<grid_for((size_t)Bm * D), 256, 0, st>>>(Tall, idx + (size_t)b * Bm, Bm, D, T);
            batch_grad(P, G, X, T, Bm, H1, H2, Y, dY, dH2, dH1, part + (size_t)kLossParts * b, kLossParts, st);
            step++;
            const double frac = (double)(step - 1) / std::max(1, o->epochs * nb - 1);
            const float lr = (float)(o->lr * (0.05 + 0.95 * 0.5 * (1.0 + std::cos(M_PI * frac))));
            const float c1 = 1.f - std::pow(0.9f, (float)step), c2 = 1.f - std::pow(0.999f, (float)step);
            k_adam<<<grid_for(P.count()), 256, 0, st>>>(P.base, G.base, mom, vel, P.count(), lr, 0.9f, 0.999f, c1,
                                                         c2);
        }
        EGG_CHECK(cudaMemcpyAsync(hp.data(), part, 8 * hp.size(), cudaMemcpyDeviceToHost, st));
        EGG_CHECK(cudaStreamSynchronize(st));
        EGG_CHECK(cudaGetLastError());
        if (epoch_loss) {
            double s = 0.0;
            for (double v : hp) s += v;
            epoch_loss[e] = s / ((double)nb * Bm * D);
        }
    }
    download_params(P, *m, st);
    EGG_CHECK(cudaStreamSynchronize(st));
    EGG_CHECK(cudaGetLastError());
    return EGG_OK;
}

void release_all() { release(g_buf); }

}  // namespace mlp
}  // namespace egg

// ---------------------------------------------------------------------------
// C ABI
// ---------------------------------------------------------------------------
extern "C" {

__attribute__((visibility("default"))) int egg_mlp_feature_dim(int32_t d) {
    return d >= 1 && d <= egg::mlp::kMaxWarmDims ? egg::mlp::feat_pad(d) : -1;
}

__attribute__((visibility("default"))) int egg_mlp_features(const float* x, int64_t n, int32_t d, float eps,
                                                            float* feats) {
    return egg::guarded([&] { return egg::mlp::api_features(x, n, d, eps, feats); });
}

__attribute__((visibility("default"))) int egg_mlp_forward(const egg_mlp* m, const float* feats, int64_t n,
                                                           float* out) {
    return egg::guarded([&] { return egg::mlp::api_forward(m, feats, n, out); });
}

__attribute__((visibility("default"))) int egg_mlp_grad(const egg_mlp* m, const float* feats, const float* targets,
                                                        int64_t n, egg_mlp* grad, double* loss) {
    return egg::guarded([&] { return egg::mlp::api_grad(m, feats, targets, n, grad, loss); });
}

__attribute__((visibility("default"))) int egg_mlp_train(egg_mlp* m, const float* feats, const float* targets,
                                                         int64_t n, const egg_mlp_train_opts* opts,
                                                         double* epoch_loss) {
    return egg::guarded([&] { return egg::mlp::api_train(m, feats, targets, n, opts, epoch_loss); });
}

}  // extern "C"
