// ref_simple_driver.cu -- C-ABI driver around the reference's own brute-force
// GPU SynC.
//
// TEST INFRASTRUCTURE ONLY (parity checker).  Compiled together with the
// unmodified reference sources src/algorithms/simple_GPU_SynC.cu,
// src/utils/GPU_utils.cu and src/utils/CPU_math.cpp (see oracle/build.py)
// into oracle/_ref/libref_simple.so.  It converts the reference's result
// tensors (simple_GPU_SynC.cu:207-218) into plain arrays.  The reference calls
// exit() on CUDA errors (simple_GPU_SynC.cu:19-25), so callers run it in a
// child process.
#include <ATen/ATen.h>
#include <cuda_runtime.h>
#include <vector>

#include "simple_GPU_SynC.cuh"

extern "C" {

// labels[n] (int, -1 = noise), *iters = number of iterations
__attribute__((visibility("default"))) int ref_simple_run(const float *D, int n, int d, float eps, float lam,
                                                          int *labels, int *iters) {
    std::vector<at::Tensor> r = GPU_DynamicalClustering(const_cast<float *>(D), n, d, eps, lam);
    at::Tensor C = r[0].contiguous();
    const float *c = C.data_ptr<float>();
    for (int i = 0; i < n; i++) labels[i] = (int)c[i];
    if (iters) *iters = (int)r[1].size(0);
    return 0;
}

}  // extern "C"
