// egg_sort.cu -- device sort, scan and segmented-sum primitives of the eps
// search's coding cost (egg_mdl.cu): a stable LSD radix sort of 32-bit keys
// with an optional int payload (four 8-bit passes: tile histograms, per-digit
// scan over the tiles, stable scatter with warp match-any ranks), an
// inclusive scan of ints (block scans, a scan of the block totals, offsets),
// and per-segment sums of doubles with one warp per segment in a fixed order.
// Every result is deterministic: the sort is stable and the sums add in an
// order fixed by the segment layout.
#include <cuda_runtime.h>

#include <cstdint>

#include "egg_host_common.h"
#include "egg_sort.h"

namespace egg {
namespace prim {

namespace {

constexpr int kTile = 2048;   // keys per sort tile
constexpr int kThreads = 256; // threads per sort block (one per digit in the digit scans)
constexpr int kScanItems = 4; // ints per thread in the block scans
constexpr int kScanThreads = 1024;

__device__ __forceinline__ unsigned lanemask_lt() {
    unsigned m;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}

// block-wide exclusive scan of one int per thread; *total = the sum
__device__ int block_excl(int v, int* total) {
    __shared__ int ws[33];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
    int incl = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int t = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += t;
    }
    if (lane == 31) ws[wid] = incl;
    __syncthreads();
    if (wid == 0) {
        const int s = lane < nw ? ws[lane] : 0;
        int si = s;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int t = __shfl_up_sync(0xffffffffu, si, o);
            if (lane >= o) si += t;
        }
        if (lane < nw) ws[lane] = si - s;
        if (lane == 31) ws[32] = si;
    }
    __syncthreads();
    const int r = incl - v + ws[wid];
    if (total) *total = ws[32];
    __syncthreads();
    return r;
}

__global__ void __launch_bounds__(kThreads) k_tile_hist(const uint32_t* __restrict__ keys, int n, int shift,
                                                        int* __restrict__ hist, int tiles) {
    __shared__ int h[256];
    for (int t = threadIdx.x; t < 256; t += blockDim.x) h[t] = 0;
    __syncthreads();
    const int b = blockIdx.x * kTile, e = min(b + kTile, n);
    for (int i = b + threadIdx.x; i < e; i += blockDim.x) atomicAdd(&h[(keys[i] >> shift) & 255u], 1);
    __syncthreads();
    for (int t = threadIdx.x; t < 256; t += blockDim.x) hist[(size_t)t * tiles + blockIdx.x] = h[t];
}

// one block per digit: exclusive scan of the digit's tile counts, total per digit
__global__ void __launch_bounds__(kThreads) k_digit_scan(int* __restrict__ hist, int tiles, int* __restrict__ total) {
    int* h = hist + (size_t)blockIdx.x * tiles;
    const int per = (tiles + blockDim.x - 1) / blockDim.x;
    const int b = threadIdx.x * per, e = min(b + per, tiles);
    int s = 0;
    for (int k = b; k < e; k++) s += h[k];
    int tot;
    int run = block_excl(s, &tot);
    for (int k = b; k < e; k++) {
        const int v = h[k];
        h[k] = run;
        run += v;
    }
    if (threadIdx.x == 0) total[blockIdx.x] = tot;
}

// stable scatter of one tile (blockDim == kThreads == 256: one thread per digit)
__global__ void __launch_bounds__(kThreads) k_tile_scatter(const uint32_t* __restrict__ kin, const int* __restrict__ vin,
                                                           uint32_t* __restrict__ kout, int* __restrict__ vout, int n,
                                                           int shift, const int* __restrict__ hist, int tiles,
                                                           const int* __restrict__ total) {
    constexpr int W = kThreads / 32;
    __shared__ int base[256], run[256], wcnt[W][256];
    const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
    base[tid] = block_excl(total[tid], nullptr) + hist[(size_t)tid * tiles + blockIdx.x];
    run[tid] = 0;
#pragma unroll
    for (int k = 0; k < W; k++) wcnt[k][tid] = 0;
    __syncthreads();
    const int t0 = blockIdx.x * kTile;
    for (int r = 0; r < kTile / kThreads; r++) {
        if (t0 + r * kThreads >= n) break;  // uniform across the block
        const int i = t0 + r * kThreads + tid;
        const bool valid = i < n;
        uint32_t key = 0;
        int dg = 0;
        if (valid) {
            key = kin[i];
            dg = (int)((key >> shift) & 255u);
        }
        const unsigned peers = __match_any_sync(0xffffffffu, valid ? dg : 256 + lane);
        const int rank = __popc(peers & lanemask_lt());
        if (valid && rank == 0) wcnt[wid][dg] = __popc(peers);
        __syncthreads();
        {
            int rr = run[tid];
#pragma unroll
            for (int k = 0; k < W; k++) {
                const int c = wcnt[k][tid];
                wcnt[k][tid] = rr;
                rr += c;
            }
            run[tid] = rr;
        }
        __syncthreads();
        if (valid) {
            const int pos = base[dg] + wcnt[wid][dg] + rank;
            kout[pos] = key;
            if (vout) vout[pos] = vin[i];
        }
        __syncthreads();
#pragma unroll
        for (int k = 0; k < W; k++) wcnt[k][tid] = 0;
        __syncthreads();
    }
}

// inclusive scan of kScanItems consecutive ints per thread; block totals
__global__ void __launch_bounds__(kScanThreads) k_block_incl(const int* __restrict__ in, int* __restrict__ out, int m,
                                                             int* __restrict__ totals) {
    const size_t b = (size_t)blockIdx.x * kScanThreads * kScanItems + (size_t)threadIdx.x * kScanItems;
    int v[kScanItems];
    int s = 0;
#pragma unroll
    for (int k = 0; k < kScanItems; k++) {
        v[k] = b + k < (size_t)m ? in[b + k] : 0;
        s += v[k];
    }
    int tot;
    int run = block_excl(s, &tot);
#pragma unroll
    for (int k = 0; k < kScanItems; k++) {
        run += v[k];
        if (b + k < (size_t)m) out[b + k] = run;
    }
    if (threadIdx.x == 0) totals[blockIdx.x] = tot;
}

// single block: exclusive scan of the block totals (any count)
__global__ void __launch_bounds__(kScanThreads) k_totals_excl(int* __restrict__ t, int nb) {
    const int per = (nb + blockDim.x - 1) / blockDim.x;
    const int b = threadIdx.x * per, e = min(b + per, nb);
    int s = 0;
    for (int k = b; k < e; k++) s += t[k];
    int run = block_excl(s, nullptr);
    for (int k = b; k < e; k++) {
        const int v = t[k];
        t[k] = run;
        run += v;
    }
}

__global__ void k_add_offsets(int* __restrict__ out, int m, const int* __restrict__ off) {
    const size_t per = (size_t)kScanThreads * kScanItems;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < (size_t)m; i += (size_t)gridDim.x * blockDim.x)
        out[i] += off[i / per];
}

// one warp per segment: lane j adds elements j, j + 32, ... in order, then a
// fixed butterfly; the result depends only on the segment's values and length
__global__ void k_seg_sum(const double* __restrict__ v, const int* __restrict__ begin, int K, double* __restrict__ out) {
    const int lane = threadIdx.x & 31;
    const int wpb = blockDim.x >> 5;
    for (int s = blockIdx.x * wpb + (threadIdx.x >> 5); s < K; s += gridDim.x * wpb) {
        const int b = begin[s], e = begin[s + 1];
        double acc = 0.0;
        for (int i = b + lane; i < e; i += 32) acc += v[i];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
        if (lane == 0) out[s] = acc;
    }
}

}  // namespace

size_t sort_scratch_bytes(int n) {
    const size_t tiles = ((size_t)n + kTile - 1) / kTile;
    return 2 * align_up(4 * (size_t)n) + 2 * align_up(4 * (size_t)n) + align_up(4 * 256 * tiles) + align_up(4 * 256);
}

void sort_pairs(const uint32_t* keys, const int* vals, uint32_t* keys_out, int* vals_out, int n, void* scratch,
                cudaStream_t st) {
    if (n <= 0) return;
    const int tiles = (n + kTile - 1) / kTile;
    char* p = (char*)scratch;
    uint32_t* ka = (uint32_t*)p;
    p += align_up(4 * (size_t)n);
    uint32_t* kb = (uint32_t*)p;
    p += align_up(4 * (size_t)n);
    int* va = (int*)p;
    p += align_up(4 * (size_t)n);
    int* vb = (int*)p;
    p += align_up(4 * (size_t)n);
    int* hist = (int*)p;
    p += align_up(4 * 256 * (size_t)tiles);
    int* total = (int*)p;
    const bool pay = vals != nullptr && vals_out != nullptr;
    const uint32_t* kin = keys;
    const int* vin = vals;
    for (int pass = 0; pass < 4; pass++) {
        const int shift = 8 * pass;
        uint32_t* kout = pass == 3 ? keys_out : (pass % 2 == 0 ? ka : kb);
        int* vout = pay ? (pass == 3 ? vals_out : (pass % 2 == 0 ? va : vb)) : nullptr;
        k_tile_hist<<<tiles, kThreads, 0, st>>>(kin, n, shift, hist, tiles);
        k_digit_scan<<<256, kThreads, 0, st>>>(hist, tiles, total);
        k_tile_scatter<<<tiles, kThreads, 0, st>>>(kin, pay ? vin : nullptr, kout, vout, n, shift, hist, tiles,
                                                   total);
        kin = kout;
        vin = vout;
    }
    EGG_CHECK(cudaGetLastError());
}

size_t scan_scratch_bytes(int m) {
    const size_t per = (size_t)kScanThreads * kScanItems;
    return align_up(4 * (((size_t)m + per - 1) / per + 1));
}

void inclusive_scan(const int* in, int* out, int m, void* scratch, cudaStream_t st) {
    if (m <= 0) return;
    const size_t per = (size_t)kScanThreads * kScanItems;
    const int nb = (int)(((size_t)m + per - 1) / per);
    int* totals = (int*)scratch;
    k_block_incl<<<nb, kScanThreads, 0, st>>>(in, out, m, totals);
    if (nb > 1) {
        k_totals_excl<<<1, kScanThreads, 0, st>>>(totals, nb);
        const int blocks = (int)std::min<size_t>(((size_t)m + 255) / 256, 148 * 16);
        k_add_offsets<<<blocks, 256, 0, st>>>(out, m, totals);
    }
    EGG_CHECK(cudaGetLastError());
}

void segment_sums(const double* v, const int* begin, int K, double* out, cudaStream_t st) {
    if (K <= 0) return;
    const int wpb = 8;
    const int blocks = (int)std::min<long long>(((long long)K + wpb - 1) / wpb, 148 * 32);
    k_seg_sum<<<blocks, 32 * wpb, 0, st>>>(v, begin, K, out);
    EGG_CHECK(cudaGetLastError());
}

}  // namespace prim
}  // namespace egg
