// egg_normalize.cu -- per-dimension min-max normalisation on the GPU.
//
// The reference normalises on the host before clustering
// (python/data.py:100-103: (X - X.min(0)) / (X.max(0) - X.min(0))).  Here the
// same arithmetic runs on the device, in float32 with explicit
// round-to-nearest subtraction and division, so the result equals numpy's
// float32 evaluation of that expression bit for bit.  A dimension whose
// values are all equal maps to 0 (the reference divides by zero there).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <string>
#include <vector>

#include "eggsync.h"
#include "egg_common.cuh"
#include "egg_host_common.h"

namespace egg {

namespace {

constexpr int kNormBlocks = 148 * 4;
constexpr int kNormThreads = 256;

// per-block minimum and maximum of every dimension; non-finite values set *bad
__global__ void __launch_bounds__(kNormThreads) k_minmax_partial(const float* __restrict__ x, size_t n, int d,
                                                                  float* part, int* bad) {
    __shared__ float s_lo[kNormThreads], s_hi[kNormThreads];
    for (int l = 0; l < d; l++) {
        float lo = INFINITY, hi = -INFINITY;
        for (size_t p = blockIdx.x * (size_t)blockDim.x + threadIdx.x; p < n; p += (size_t)gridDim.x * blockDim.x) {
            const float v = x[p * d + l];
            if (!isfinite(v)) *bad = 1;
            lo = fminf(lo, v);
            hi = fmaxf(hi, v);
        }
        s_lo[threadIdx.x] = lo;
        s_hi[threadIdx.x] = hi;
        __syncthreads();
        for (int o = blockDim.x / 2; o > 0; o >>= 1) {
            if (threadIdx.x < o) {
                s_lo[threadIdx.x] = fminf(s_lo[threadIdx.x], s_lo[threadIdx.x + o]);
                s_hi[threadIdx.x] = fmaxf(s_hi[threadIdx.x], s_hi[threadIdx.x + o]);
            }
            __syncthreads();
        }
        if (threadIdx.x == 0) {
            part[((size_t)blockIdx.x * d + l) * 2] = s_lo[0];
            part[((size_t)blockIdx.x * d + l) * 2 + 1] = s_hi[0];
        }
        __syncthreads();
    }
}

__global__ void k_minmax_final(const float* __restrict__ part, int blocks, int d, float* lohi) {
    for (int l = threadIdx.x; l < d; l += blockDim.x) {
        float lo = INFINITY, hi = -INFINITY;
        for (int b = 0; b < blocks; b++) {
            lo = fminf(lo, part[((size_t)b * d + l) * 2]);
            hi = fmaxf(hi, part[((size_t)b * d + l) * 2 + 1]);
        }
        lohi[2 * l] = lo;
        lohi[2 * l + 1] = hi;
    }
}

__global__ void k_scale(const float* __restrict__ x, size_t n, int d, const float* __restrict__ lohi,
                        float* __restrict__ out) {
    for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < n * d; t += (size_t)gridDim.x * blockDim.x) {
        const int l = (int)(t % d);
        const float lo = lohi[2 * l], hi = lohi[2 * l + 1];
        const float span = __fsub_rn(hi, lo);
        out[t] = span > 0.f ? __fdiv_rn(__fsub_rn(x[t], lo), span) : 0.f;
    }
}

}  // namespace

int minmax_normalize(const float* x, int64_t n, int32_t d, float* out, float* lo_out, float* hi_out,
                     void* stream) {
    if (!x || !out) throw ArgError{EGG_ERR_ARG, "x and out must not be NULL"};
    if (n < 1 || n > ((int64_t)1 << 33)) throw ArgError{EGG_ERR_ARG, "n out of range"};
    if (d < 1 || d > kMaxDims) throw ArgError{EGG_ERR_ARG, "d must be in [1, 64]"};
    cudaStream_t st = (cudaStream_t)stream;
    const size_t cnt = (size_t)n * d;
    const bool dev_in = is_device_ptr(x), dev_out = is_device_ptr(out);
    std::vector<void*> tmp;
    auto alloc = [&](size_t bytes) {
        void* p = nullptr;
        EGG_CHECK(dev_alloc((void**)&p, bytes));
        tmp.push_back(p);
        return p;
    };
    try {
        const float* xd = x;
        if (!dev_in) {
            float* b = (float*)alloc(4 * cnt);
            EGG_CHECK(cudaMemcpyAsync(b, x, 4 * cnt, cudaMemcpyHostToDevice, st));
            xd = b;
        }
        // device output, else a device buffer copied back (the staged input when the input is on the host)
        float* od = dev_out ? out : (dev_in ? (float*)alloc(4 * cnt) : const_cast<float*>(xd));
        const int blocks =
            (int)std::max<int64_t>(1, std::min<int64_t>(kNormBlocks, (n + kNormThreads - 1) / kNormThreads));
        float* part = (float*)alloc(8 * (size_t)blocks * d);
        float* lohi = (float*)alloc(8 * (size_t)d);
        int* bad = (int*)alloc(4);
        EGG_CHECK(cudaMemsetAsync(bad, 0, 4, st));
        k_minmax_partial<<<blocks, kNormThreads, 0, st>>>(xd, (size_t)n, d, part, bad);
        k_minmax_final<<<1, 64, 0, st>>>(part, blocks, d, lohi);
        k_scale<<<(int)std::min<size_t>((cnt + 255) / 256, 148 * 16), 256, 0, st>>>(xd, (size_t)n, d, lohi, od);
        std::vector<float> hl(2 * (size_t)d);
        int hbad = 0;
        EGG_CHECK(cudaMemcpyAsync(hl.data(), lohi, 8 * (size_t)d, cudaMemcpyDeviceToHost, st));
        EGG_CHECK(cudaMemcpyAsync(&hbad, bad, 4, cudaMemcpyDeviceToHost, st));
        if (!dev_out) EGG_CHECK(cudaMemcpyAsync(out, od, 4 * cnt, cudaMemcpyDeviceToHost, st));
        EGG_CHECK(cudaStreamSynchronize(st));
        EGG_CHECK(cudaGetLastError());
        for (void* p : tmp) cudaFree(p);
        tmp.clear();
        if (hbad) throw ArgError{EGG_ERR_INPUT, "input holds NaN or Inf"};
        for (int l = 0; l < d; l++) {
            if (lo_out) lo_out[l] = hl[2 * l];
            if (hi_out) hi_out[l] = hl[2 * l + 1];
        }
    } catch (...) {
        for (void* p : tmp) cudaFree(p);
        throw;
    }
    return EGG_OK;
}

}  // namespace egg

extern "C" __attribute__((visibility("default"))) int egg_minmax_normalize(const float* x, int64_t n, int32_t d,
                                                                           float* out, float* lo, float* hi,
                                                                           void* stream) {
    return egg::guarded([&] { return egg::minmax_normalize(x, n, d, out, lo, hi, stream); });
}
