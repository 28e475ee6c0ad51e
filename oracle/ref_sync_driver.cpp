// ref_sync_driver.cpp -- C-ABI driver around the reference's own CPU SynC.
//
// TEST INFRASTRUCTURE ONLY (parity checker and timed CPU baseline).  It is
// compiled together with the unmodified reference sources
// src/algorithms/SynC.cpp and src/utils/CPU_math.cpp (see oracle/build.py)
// into oracle/_ref/libref_sync.so.  Nothing here re-implements the
// reference: every function only converts between plain pointers and the
// reference's interfaces.
//
//   ref_sync_run          -> DynamicalClustering_parallel  (SynC.cpp:328-399)
//   ref_sync_serial_run   -> DynamicalClustering           (SynC.cpp:268-326)
//   ref_sync_step_sample  -> ComputeNeighborhood + UpdatePoint +
//                            ComputeLocationOrder           (SynC.cpp:16-56)
#include <ATen/ATen.h>
#include <omp.h>
#include <cstdio>
#include <cstring>
#include <vector>

#include "SynC.h"

static void copy_result(const std::vector<at::Tensor> &r, int n, int *labels, int *iters) {
    at::Tensor C = r[0].to(at::kInt).contiguous();
    const int *c = C.data_ptr<int>();
    for (int i = 0; i < n; i++) labels[i] = c[i];
    if (iters) *iters = (int)r[1].size(0);
}

extern "C" {

__attribute__((visibility("default"))) int ref_sync_run(const float *D, int n, int d, float eps, float lam,
                                                         int *labels, int *iters) {
    std::vector<at::Tensor> r = DynamicalClustering_parallel(const_cast<float *>(D), n, d, eps, lam);
    copy_result(r, n, labels, iters);
    return 0;
}

__attribute__((visibility("default"))) int ref_sync_serial_run(const float *D, int n, int d, float eps, float lam,
                                                                int *labels, int *iters) {
    std::vector<at::Tensor> r = DynamicalClustering(const_cast<float *>(D), n, d, eps, lam);
    copy_result(r, n, labels, iters);
    return 0;
}

// One reference SynC iteration for the sampled points idx[0..m): the updated
// coordinates, |N_eps(p)| and the local order parameter r_p, computed on the
// unmodified D exactly as the reference's parallel loop body does.
__attribute__((visibility("default"))) int ref_sync_step_sample(const float *D, int n, int d, float eps,
                                                                const int *idx, int m, float *out, int *counts,
                                                                float *r_out) {
    float *Dc = const_cast<float *>(D);
    std::vector<float> Dn((size_t)n * d);
#pragma omp parallel for schedule(dynamic, 4)
    for (int k = 0; k < m; k++) {
        int p = idx[k];
        const neighborhood N = ComputeNeighborhood(p, eps, Dc, n, d);
        UpdatePoint(p, N, Dc, Dn.data(), n, d);
        for (int l = 0; l < d; l++) out[(size_t)k * d + l] = Dn[(size_t)p * d + l];
        if (counts) counts[k] = (int)N.size();
        if (r_out) r_out[k] = ComputeLocationOrder(p, N, Dc, n, d);
    }
    return 0;
}

__attribute__((visibility("default"))) int ref_sync_threads(void) { return omp_get_max_threads(); }

}  // extern "C"
