// ref_egg_driver.cu -- C-ABI driver around the reference's own EGG-SynC.
//
// TEST INFRASTRUCTURE ONLY (parity checker).  Compiled together with the
// unmodified reference sources src/algorithms/EGG_SynC.cu,
// src/utils/GPU_utils.cu and src/utils/CPU_math.cpp (see oracle/build.py)
// into oracle/_ref/libref_egg.so.  It converts the reference's result
// tensors (EGG_SynC.cu:1587-1600) into plain arrays.
//
// The reference calls exit() on any CUDA error and has no iteration cap
// (EGG_SynC.cu:20-26, 1322), so callers run it in a child process with a
// wall-clock timeout.  Its pre-grid kernels allocate from the device heap
// with `new` and no null check (EGG_SynC.cu:394-395, 467-468); the heap is
// raised before the first call so those allocations cannot fail.
#include <ATen/ATen.h>
#include <cuda_runtime.h>
#include <vector>

#include "EGG_SynC.cuh"

extern "C" {

// labels[n] (int, -1 = noise), *iters = number of iterations,
// stage_times[6] (reference Timer<6>, process CPU seconds).
__attribute__((visibility("default"))) int ref_egg_run(const float *D, int n, int d, float eps, int *labels,
                                                       int *iters, float *stage_times) {
    cudaError_t e = cudaDeviceSetLimit(cudaLimitMallocHeapSize, (size_t)256 << 20);
    if (e != cudaSuccess) return (int)e;
    std::vector<at::Tensor> r = EGG_SynC(const_cast<float *>(D), n, d, eps);
    at::Tensor C = r[0].contiguous();
    const float *c = C.data_ptr<float>();
    for (int i = 0; i < n; i++) labels[i] = (int)c[i];
    if (iters) *iters = (int)r[1].size(0);
    if (stage_times) {
        at::Tensor s = r[2].contiguous();
        for (int i = 0; i < 6 && i < s.size(0); i++) stage_times[i] = s.data_ptr<float>()[i];
    }
    return 0;
}

}  // extern "C"
