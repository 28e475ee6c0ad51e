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
//   inference  k_mlp_infer_tc: the three layers fused in one kernel on the
//              5th-generation tensor cores (tcgen05.mma, BF16 operands from
//              shared memory, FP32 accumulators in TMEM); a CTA owns
//              128-point tiles, the next tile's features arrive by cp.async
//              while the current one runs.
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

// ---------------------------------------------------------------------------
// inference on the 5th-generation tensor cores (tcgen05, TMEM accumulators)
// ---------------------------------------------------------------------------
// A CTA of four warps owns 128-point tiles (the MMA's M).  The three layers
// run as chains of tcgen05.mma (K = 16 per instruction, BF16 operands from
// shared memory, FP32 accumulation in 128 TMEM columns) issued by one
// thread and committed to an mbarrier; after each layer every warp reads its
// 32 TMEM lanes (rows) with tcgen05.ld, adds the bias, applies the ReLU and
// writes the rounded BF16 row as the next layer's A operand.  Operands use
// the no-swizzle K-major layout: a core matrix of 8 rows x 8 elements is 128
// contiguous bytes, the core matrices of one 8-element chunk of K follow each
// other down the rows (stride 128 bytes) and chunks are rows / 8 * 128 bytes
// apart.  Each output row depends on its own features only (the MMA sums K
// in the same order for every row), whatever the tile around it.
namespace tc {

constexpr int kRows = 128;     // points per tile
constexpr int kThreads = 128;  // warp w reads TMEM lanes 32w .. 32w + 31
constexpr int kN3 = 16;        // layer 3 padded to the smallest N of an M = 128 MMA
constexpr int kCols = 128;     // TMEM columns (FP32 accumulators of 128 outputs)
constexpr long kWaitLimit = 1L << 20;

__device__ __forceinline__ uint32_t cm_offset(int row, int kchunk, int rows) {
    return (uint32_t)kchunk * (uint32_t)(rows / 8) * 128u + (uint32_t)(row >> 3) * 128u + (uint32_t)(row & 7) * 16u;
}

// shared-memory matrix descriptor: start, leading (K) and stride (M/N) byte
// offsets >> 4, descriptor version 1, no swizzle
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
    return (uint64_t)((addr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

// instruction descriptor: F32 accumulator, BF16 A and B, both K-major, M = 128
__device__ __forceinline__ uint32_t idesc_bf16(int n) {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(kRows >> 4) << 24);
}

__device__ __forceinline__ void fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// bounded wait for the mbarrier's phase; false when the limit ran out
__device__ __forceinline__ bool wait_phase(uint32_t bar, uint32_t phase) {
    for (long it = 0; it < kWaitLimit; it++) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred P1;\n\tmbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2;\n\t"
            "selp.b32 %0, 1, 0, P1;\n\t}"
            : "=r"(done)
            : "r"(bar), "r"(phase)
            : "memory");
        if (done) return true;
    }
    return false;
}

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float* v) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 16; i++) v[i] = __uint_as_float(r[i]);
}

__host__ inline size_t smem_bytes(int fp) {
    const size_t ka = (size_t)std::max(fp, kHidden);
    return 1024 + 2 * ((size_t)kHidden * fp + (size_t)kHidden * kHidden + (size_t)kN3 * kHidden + 2 * (size_t)kRows * ka) +
           4 * (2 * kHidden + kN3) + 16;
}

}  // namespace tc

// status: set to 1 (and the tile's outputs to NaN) if an MMA never completed
__global__ void __launch_bounds__(tc::kThreads, 1) k_mlp_infer_tc(Packed P, const __nv_bfloat16* __restrict__ feats,
                                                                  int n, float* __restrict__ out, int* status) {
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    unsigned char* smem = reinterpret_cast<unsigned char*>(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
    const int fp = P.fp, ka = max(fp, kHidden);
    unsigned char* W1 = smem;
    unsigned char* W2 = W1 + (size_t)kHidden * fp * 2;
    unsigned char* W3 = W2 + (size_t)kHidden * kHidden * 2;
    // two operand tiles: a tile's features (then its hidden layers), and the
    // next tile's features arriving by cp.async meanwhile
    unsigned char* Abuf[2] = {W3 + (size_t)tc::kN3 * kHidden * 2, W3 + (size_t)tc::kN3 * kHidden * 2 + (size_t)tc::kRows * ka * 2};
    unsigned char* A = Abuf[0];
    float* B1 = reinterpret_cast<float*>(Abuf[1] + (size_t)tc::kRows * ka * 2);
    float* B2 = B1 + kHidden;
    float* B3 = B2 + kHidden;
    uint64_t* barp = reinterpret_cast<uint64_t*>(B3 + tc::kN3);
    uint32_t* slot = reinterpret_cast<uint32_t*>(barp + 1);
    const int tid = threadIdx.x, warp = tid >> 5;

    // weights in the canonical layout (rows of B are the layer's outputs);
    // 4-byte loads: the packed weights are only 4-byte aligned
    auto put_rows = [&](unsigned char* dst, const __nv_bfloat16* src, int rows, int valid_rows, int K) {
        for (int t = tid; t < rows * (K / 8); t += tc::kThreads) {
            const int r = t / (K / 8), kc = t % (K / 8);
            uint4 v = make_uint4(0u, 0u, 0u, 0u);
            if (r < valid_rows) {
                const uint32_t* s = reinterpret_cast<const uint32_t*>(src + (size_t)r * K + kc * 8);
                v = make_uint4(s[0], s[1], s[2], s[3]);
            }
            *reinterpret_cast<uint4*>(dst + tc::cm_offset(r, kc, rows)) = v;
        }
    };
    put_rows(W1, P.w1t, kHidden, kHidden, fp);
    put_rows(W2, P.w2t, kHidden, kHidden, kHidden);
    put_rows(W3, P.w3t, tc::kN3, 8, kHidden);
    for (int t = tid; t < kHidden; t += tc::kThreads) {
        B1[t] = P.b1[t];
        B2[t] = P.b2[t];
    }
    if (tid < tc::kN3) B3[tid] = tid < 8 ? P.b3[tid] : 0.f;
    const uint32_t sbase = (uint32_t)__cvta_generic_to_shared(smem);
    const uint32_t sW1 = sbase, sW2 = sbase + (uint32_t)(W2 - smem), sW3 = sbase + (uint32_t)(W3 - smem);
    uint32_t sA = sbase + (uint32_t)(A - smem);
    const uint32_t bar = (uint32_t)__cvta_generic_to_shared(barp);
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                         (uint32_t)__cvta_generic_to_shared(slot)),
                     "r"(tc::kCols));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    if (tid == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(1));
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    tc::fence_before();
    __syncthreads();
    tc::fence_after();
    const uint32_t tmem = *slot;
    const uint32_t lanes = tmem + ((uint32_t)(warp * 32) << 16);  // this warp's TMEM lanes, column 0
    const int row = tid;                                          // the tile row this thread's lane holds
    uint32_t phase = 0;

    // one layer: D (TMEM) = A (shared, 128 x K) x B (shared, N x K)^T
    auto layer = [&](uint32_t b_addr, int K, int N) -> bool {
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");  // A written by these threads
        tc::fence_before();
        __syncthreads();
        tc::fence_after();
        if (tid == 0) {
            const uint32_t lbo_a = (tc::kRows / 8) * 128u, lbo_b = (uint32_t)(N / 8) * 128u;
            const uint32_t id = tc::idesc_bf16(N);
            for (int kk = 0; kk < K / 16; kk++) {
                const uint64_t da = tc::smem_desc(sA + 2u * kk * lbo_a, lbo_a, 128u);
                const uint64_t db = tc::smem_desc(b_addr + 2u * kk * lbo_b, lbo_b, 128u);
                const uint32_t acc = kk > 0 ? 1u : 0u;
                asm volatile(
                    "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
                    "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem),
                    "l"(da), "l"(db), "r"(id), "r"(acc));
            }
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar)
                         : "memory");
        }
        const bool ok = tc::wait_phase(bar, phase);
        if (!ok) (void)tc::wait_phase(bar, phase);  // let an MMA still in flight finish before TMEM is freed
        phase ^= 1u;
        tc::fence_after();
        return __syncthreads_and(ok) != 0;
    };
    // hidden layer epilogue: bias, ReLU, BF16 into A as the next operand
    auto hidden = [&](const float* bias) {
        for (int c0 = 0; c0 < kHidden; c0 += 16) {
            float v[16];
            tc::tmem_ld16(lanes + (uint32_t)c0, v);
            uint32_t p[8];
#pragma unroll
            for (int i = 0; i < 8; i++)
                p[i] = pack_bf16(fmaxf(v[2 * i] + bias[c0 + 2 * i], 0.f), fmaxf(v[2 * i + 1] + bias[c0 + 2 * i + 1], 0.f));
            *reinterpret_cast<uint4*>(A + tc::cm_offset(row, c0 / 8, tc::kRows)) = make_uint4(p[0], p[1], p[2], p[3]);
            *reinterpret_cast<uint4*>(A + tc::cm_offset(row, c0 / 8 + 1, tc::kRows)) = make_uint4(p[4], p[5], p[6], p[7]);
        }
    };

    const bool al16 = ((uintptr_t)feats & 15) == 0;
    const int tiles = (n + tc::kRows - 1) / tc::kRows;
    // a tile's features into buf by 16-byte cp.async (rows past n zero-filled)
    auto prefetch = [&](int tile, unsigned char* buf) {
        const int r0 = tile * tc::kRows;
        for (int t = tid; t < tc::kRows * (fp / 8); t += tc::kThreads) {
            const int r = t / (fp / 8), kc = t % (fp / 8);
            const bool in = r0 + r < n;
            const __nv_bfloat16* src = feats + (in ? (size_t)(r0 + r) * fp + kc * 8 : 0);
            const uint32_t dst = (uint32_t)__cvta_generic_to_shared(buf + tc::cm_offset(r, kc, tc::kRows));
            asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(dst), "l"(src), "r"(in ? 16 : 0)
                         : "memory");
        }
        asm volatile("cp.async.commit_group;" ::: "memory");
    };
    if (al16 && blockIdx.x < tiles) prefetch(blockIdx.x, Abuf[0]);
    int cur = 0;
    for (int tile = blockIdx.x; tile < tiles; tile += gridDim.x, cur ^= 1) {
        const int r0 = tile * tc::kRows;
        A = Abuf[cur];
        sA = sbase + (uint32_t)(A - smem);
        if (al16) {
            asm volatile("cp.async.wait_all;" ::: "memory");
            // the other buffer's last reader (the previous tile's layer 3)
            // completed before this tile began
            if (tile + (int)gridDim.x < tiles) prefetch(tile + gridDim.x, Abuf[cur ^ 1]);
        }
        for (int t = tid; !al16 && t < tc::kRows * (fp / 8); t += tc::kThreads) {
            const int r = t / (fp / 8), kc = t % (fp / 8);
            uint4 v = make_uint4(0u, 0u, 0u, 0u);
            if (r0 + r < n) {
                // feature rows not 16-byte aligned: 2-byte loads, synchronously
                const unsigned short* h = reinterpret_cast<const unsigned short*>(feats + (size_t)(r0 + r) * fp + kc * 8);
                v = make_uint4(h[0] | ((uint32_t)h[1] << 16), h[2] | ((uint32_t)h[3] << 16),
                               h[4] | ((uint32_t)h[5] << 16), h[6] | ((uint32_t)h[7] << 16));
            }
            *reinterpret_cast<uint4*>(A + tc::cm_offset(r, kc, tc::kRows)) = v;
        }
        bool ok = layer(sW1, fp, kHidden);
        if (ok) {
            hidden(B1);
            ok = layer(sW2, kHidden, kHidden);
        }
        if (ok) {
            hidden(B2);
            ok = layer(sW3, kHidden, tc::kN3);
        }
        float v[16];
        if (ok) tc::tmem_ld16(lanes, v);
        if (r0 + row < n)
            for (int c = 0; c < P.dout; c++) out[(size_t)(r0 + row) * P.dout + c] = ok ? v[c] + B3[c] : __int_as_float(0x7fc00000);
        if (!ok) {
            if (tid == 0) atomicExch(status, 1);
            break;
        }
    }
    asm volatile("cp.async.wait_all;" ::: "memory");  // a prefetch left by a failed tile
    tc::fence_before();
    __syncthreads();
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(tc::kCols));
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
            // a NaN displacement (inference that did not complete) leaves the point in place
            const float dl = delta[(size_t)p * d + l];
            if (dl != dl) continue;
            float* x = X + (size_t)l * ns + p;
            *x = fminf(fmaxf(__fmaf_rn(eps, dl, *x), 0.f), 1.f);
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
    const size_t wbytes =
        4 * pcount + 2 * ((size_t)kHidden * fp + (size_t)kHidden * kHidden + 8 * kHidden) + 4 * 8 + 16;
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
    int* status = reinterpret_cast<int*>(K.b3 + 8);
    EGG_CHECK(cudaMemsetAsync(status, 0, sizeof(int), st));
    const size_t smem = tc::smem_bytes(fp);
    EGG_CHECK(cudaFuncSetAttribute(k_mlp_infer_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    const int tiles = (n + tc::kRows - 1) / tc::kRows;
    const int blocks = std::max(1, std::min(tiles, 148));
    k_mlp_infer_tc<<<blocks, tc::kThreads, smem, st>>>(K, feats, n, out, status);
}

// the status word of the last inference (1: an MMA never completed)
int infer_status(Buffers& B, const egg_mlp& m, cudaStream_t st) {
    const int fp = feat_pad(m.d), F = feat_dim(m.d);
    const size_t pcount = Params{F, kHidden, m.d, nullptr}.count();
    const char* base = (const char*)B.w + 4 * pcount + 2 * ((size_t)kHidden * fp + (size_t)kHidden * kHidden + 8 * kHidden) + 4 * 8;
    int v = 0;
    EGG_CHECK(cudaMemcpyAsync(&v, base, sizeof(int), cudaMemcpyDeviceToHost, st));
    EGG_CHECK(cudaStreamSynchronize(st));
    return v;
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
    if (infer_status(g_buf, *m, st) != 0)
        throw ArgError{EGG_ERR_INTERNAL, "tensor-core inference did not complete (mbarrier wait limit)"};
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
