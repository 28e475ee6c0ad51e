// egg_host_common.h -- host helpers shared by the single-instance and the
// batched runners (internal).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <mutex>
#include <string>
#include <vector>

#include "eggsync.h"
#include "egg_common.cuh"

namespace egg {

struct CudaError {
    cudaError_t code;
    std::string where;
};

struct ArgError {
    int status;
    std::string msg;
};

#define EGG_CHECK(call)                                                              \
    do {                                                                             \
        cudaError_t _e = (call);                                                     \
        if (_e != cudaSuccess) throw ::egg::CudaError{_e, std::string(#call) + " @" + \
                                                            std::to_string(__LINE__)}; \
    } while (0)

// Every device allocation of the library goes through dev_alloc.  For tests
// of the error paths, egg_inject_alloc_failures(k) makes the next k calls
// fail as cudaMalloc does when the device is out of memory
// (cudaErrorMemoryAllocation), without allocating anything.
extern int g_fail_allocs;
inline cudaError_t dev_alloc(void** p, size_t bytes) {
    if (g_fail_allocs > 0) {
        g_fail_allocs--;
        *p = nullptr;
        return cudaErrorMemoryAllocation;
    }
    return cudaMalloc(p, bytes);
}

// geometry exactly as the reference computes it (EGG_SynC.cu:1249-1260, 1430, 563, 779, 1045)
Geom make_geom(int64_t n64, int d, float eps);

struct Stencil {
    std::vector<int> delta;
    std::vector<signed char> off;
};
Stencil make_stencil(const Geom& g, int rad);

inline size_t align_up(size_t v) { return (v + 255) & ~(size_t)255; }

bool is_device_ptr(const void* p);

// Device arrays of one instance, carved from `base` (nullptr: sizes only).
// With own_io, the workspace also holds the input staging area (*xin), the
// label staging area and the stencil/table constants; a batch places those
// in shared arenas instead.  Returns the bytes used.
size_t layout_work(const Geom& g, int max_iter, char* base, Work& w, float** xin, bool own_io);

// stencils (update, annulus, ball) and sin/cos tables of one instance
struct Consts {
    std::vector<int> st_delta;
    std::vector<signed char> st_off;
    std::vector<float> table;
    int st_cap = 1;
    int st_count[3] = {0, 0, 0};
};
Consts make_consts(const Geom& g);

// serialises the entry points and turns exceptions into status codes
extern std::mutex g_mutex;
extern thread_local std::string g_last_error;

inline int fail(int status, const std::string& msg) {
    g_last_error = msg;
    return status;
}

template <typename F>
int guarded(F&& fn) {
    std::lock_guard<std::mutex> lock(g_mutex);
    g_last_error.clear();
    try {
        return fn();
    } catch (const ArgError& e) {
        return fail(e.status, e.msg);
    } catch (const CudaError& e) {
        cudaGetLastError();
        return fail(e.code == cudaErrorNoDevice || e.code == cudaErrorInsufficientDriver ? EGG_ERR_NO_DEVICE
                                                                                          : EGG_ERR_CUDA,
                    std::string(cudaGetErrorString(e.code)) + " in " + e.where);
    } catch (const std::bad_alloc&) {
        return fail(EGG_ERR_INTERNAL, "host allocation failed");
    }
}

// batched runner (egg_batch_host.cu)
int run_batch(egg_batch_item* items, int count, const egg_opts* opts, egg_batch_stats* stats, void* stream);
void release_batch();

}  // namespace egg
