// egg_host.cu -- host orchestration and C ABI of libeggsync.so.
//
// Replaces the host driver of the reference, EGG_SynC(float*, n, d, eps)
// (src/algorithms/EGG_SynC.cu:1229-1601).  Differences in how, not what:
//   * one device workspace per GPU, allocated once and grown on demand
//     (the reference allocates ~20 buffers per call and cudaMallocs inside
//     every scan and every extra check);
//   * the whole while-loop runs on the device: one CUDA graph whose
//     conditional while node repeats the iteration body until the
//     convergence flag (or the iteration cap) stops it, so there is no host
//     synchronisation between iterations (the reference has at least seven
//     device syncs and two to four readbacks per iteration);
//   * stage and iteration times come from %globaltimer stamps written by the
//     kernels, in the reference's six stage slots;
//   * failures are returned as status codes (the reference calls exit()).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "eggsync.h"
#include "egg_common.cuh"
#include "egg_host_common.h"
#include "egg_kernels.h"
#include "egg_mlp.h"

namespace egg {

std::mutex g_mutex;
thread_local std::string g_last_error;
int g_fail_allocs = 0;  // injected allocation failures still to deliver (egg_inject_alloc_failures)
// interaction counters of the last run (stats build)
unsigned long long g_counters[kUStats] = {};

namespace {

// ------------------------------------------------------------------------
// geometry, stencils, tables
// ------------------------------------------------------------------------
float sq_threshold(float e) {
    float t = e * e;
    while (t > 0.0f && sqrtf(t) > e) t = nextafterf(t, 0.0f);
    for (;;) {
        float u = nextafterf(t, INFINITY);
        if (sqrtf(u) <= e) t = u; else break;
    }
    return t;
}

}  // namespace

// EGG_SynC.cu:1249-1260, 1430, 563, 779, 1045
Geom make_geom(int64_t n64, int d, float eps) {
    if (n64 < 1 || n64 > (int64_t)0x7ffffff0 / 4) throw ArgError{EGG_ERR_ARG, "n out of range"};
    if (d < 1 || d > kMaxDims) throw ArgError{EGG_ERR_ARG, "d must be in [1, 64]"};
    if (!(eps > 0.0f) || !std::isfinite(eps)) throw ArgError{EGG_ERR_ARG, "eps must be positive and finite"};
    const int n = (int)n64;
    Geom g;
    memset(&g, 0, sizeof(g));
    g.n = n;
    g.d = d;
    g.ns = (n + 31) & ~31;
    g.eps = eps;
    g.side = (float)sqrt(pow((double)eps / 2., 2.) / (double)d);
    g.width = (int)(1.0f / g.side);
    if (g.width < 2) throw ArgError{EGG_ERR_GEOMETRY, "eps too large: fewer than 2 cells per dimension"};
    if (g.width > 65535) throw ArgError{EGG_ERR_GEOMETRY, "eps too small: more than 65535 cells per dimension"};
    int od = (int)(log((double)n) / log((double)g.width));
    od = std::min(d, std::max(od, 0));
    g.od = od;
    const double no = pow((double)g.width, (double)od);
    if (no > 2.0e9) throw ArgError{EGG_ERR_GEOMETRY, "outer grid too large"};
    g.n_outer = (int)no;
    int p = 1;
    for (int l = 0; l < od && l < 32; l++) {
        g.wpow[l] = p;
        p *= g.width;
    }
    g.r = (int)ceilf(eps / g.side);
    g.eps_extra = (float)((double)(2.0f * eps) - (double)eps * sqrt(15. / 16.) + (double)eps / 2. -
                          sin((double)eps / 2.));
    g.r_extra = (int)ceilf(g.eps_extra / g.side);
    g.r_half = (int)ceil(((double)eps / 2.) / (double)g.side);
    g.t_eps = sq_threshold(eps);
    g.t_half = sq_threshold(eps / 2.0f);
    g.t_extra = sq_threshold(g.eps_extra);
    g.table_k = std::max(g.r, std::max(g.r_extra, g.r_half)) + 2;
    if (g.table_k > kMaxTable) throw ArgError{EGG_ERR_GEOMETRY, "stencil radius too large"};
    if (od < d) {
        g.zblk = std::max(1, (g.width + 63) / 64);
        g.nzb = (g.width + g.zblk - 1) / g.zblk;
    } else {
        g.zblk = g.width;
        g.nzb = 1;
    }
    g.sub_dims = std::min(d, 8);
    g.sub_bits = std::max(1, 8 / g.sub_dims);
    return g;
}

Stencil make_stencil(const Geom& g, int rad) {
    Stencil S;
    const int od = g.od;
    if (od == 0) {
        S.delta.push_back(0);
        return S;
    }
    double cnt = pow(2.0 * rad + 1.0, (double)od);
    if (cnt > 4.0e6 || rad > 127) throw ArgError{EGG_ERR_GEOMETRY, "stencil too large"};
    std::vector<int> idx(od, -rad);
    for (;;) {
        int delta = 0;
        for (int l = 0; l < od; l++) {
            delta += idx[l] * g.wpow[l];
            S.off.push_back((signed char)idx[l]);
        }
        S.delta.push_back(delta);
        int l = 0;
        idx[0]++;
        while (l < od - 1 && idx[l] > rad) {
            idx[l] = -rad;
            l++;
            idx[l]++;
        }
        if (idx[od - 1] > rad) break;
    }
    return S;
}

bool is_device_ptr(const void* p) {
    cudaPointerAttributes a;
    cudaError_t e = cudaPointerGetAttributes(&a, p);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
}

size_t layout_work(const Geom& g, int max_iter, char* base, Work& w, float** xin, bool own_io) {
    const int d = g.d;
    const size_t ns = (size_t)g.ns;
    const int tiles = (g.n + kSortTile - 1) / kSortTile;
    const int nb = (g.n + kHeadsBlock - 1) / kHeadsBlock;
    const int nw = (g.n + 31) / 32;
    size_t off = 0;
    auto add = [&](void** p, size_t bytes) {
        *p = base ? base + off : nullptr;
        off += align_up(bytes);
    };
    add((void**)&w.X, 4 * d * ns);
    add((void**)&w.Xn, 4 * d * ns);
    const bool packed = d <= kPackDims;
    add((void**)&w.sd, packed ? 0 : 4 * d * ns);
    add((void**)&w.md, packed ? 0 : 4 * d * ns);
    add((void**)&w.xp, packed ? 16 * (size_t)pack_w(d) * ns : 0);
    add((void**)&w.smp, packed ? 16 * (size_t)pack_s(d) * ns : 0);
    add((void**)&w.qlo, 4 * d * ns);
    add((void**)&w.qhi, 4 * d * ns);
    add((void**)&w.ulo, 4 * d * ns);
    add((void**)&w.uhi, 4 * d * ns);
    add((void**)&w.orig, 4 * ns);
    add((void**)&w.orig_tmp, 4 * ns);
    add((void**)&w.perm, 4 * ns);
    add((void**)&w.perm_tmp, 4 * ns);
    const bool one_key = d <= 3 && g.width <= 256;
    add((void**)&w.skey[0], one_key ? 4 * ns : 0);
    add((void**)&w.skey[1], one_key ? 4 * ns : 0);
    if (!one_key) w.skey[0] = w.skey[1] = nullptr;  // the per-dimension passes
    add((void**)&w.cell_of, 4 * ns);
    add((void**)&w.cell_start, 4 * (ns + 1));
    add((void**)&w.cell_dims, 4 * d * ns);
    add((void**)&w.cell_key, d <= 4 ? 8 * ns : 0);
    add((void**)&w.cell_outer, 4 * ns);
    add((void**)&w.css, 4 * d * ns);
    add((void**)&w.csm, 4 * d * ns);
    add((void**)&w.cbmin, 4 * d * ns);
    add((void**)&w.cbmax, 4 * d * ns);
    add((void**)&w.outer_begin, 4 * ((size_t)g.n_outer + 1));
    add((void**)&w.colmask, g.od < d ? 8 * ((size_t)g.n_outer + 1) : 0);
    add((void**)&w.hist, 4 * 256 * (size_t)tiles);
    add((void**)&w.digit_total, 4 * 256);
    add((void**)&w.block_sums, 4 * (size_t)nb);
    add((void**)&w.wpart, 8 * 4 * (size_t)d * 2 * nw);
    add((void**)&w.gpart, 4 * 4 * (size_t)d * 2 * nw);
    add((void**)&w.ctrl, 4 * kCtrlWords);
    add((void**)&w.ustats, 8 * kUStats);
    add((void**)&w.stamps, 8 * 4 * ((size_t)max_iter + 2));
    add((void**)&w.iter_flags, 4 * ((size_t)max_iter + 2));
    add((void**)&w.dirty[0], 8 * ((size_t)g.n_outer + 1));
    add((void**)&w.dirty[1], 8 * ((size_t)g.n_outer + 1));
    add((void**)&w.need, 8 * ((size_t)g.n_outer + 1));
    add((void**)&w.viol_orig, ns);
    add((void**)&w.warp_moved, (size_t)nw + 1);
    add((void**)&w.warp_viol, 4 * ((size_t)nw + 1));
    add((void**)&w.span_list, 4 * ((size_t)nw + 1));
    add((void**)&w.big_list, 4 * ((size_t)nw / 4 + 1));
    add((void**)&w.span_mark, 4 * ns);
    add((void**)&w.rpart, 8 * 2 * (size_t)((g.n + 127) / 128));
    add((void**)&w.rvals, 8 * 2 * ((size_t)max_iter + 2));
    add((void**)&w.uf_parent, 4 * ns);
    add((void**)&w.uf_size, 4 * ns);
    if (own_io) {
        const Consts c = make_consts(g);
        add((void**)&w.st_delta, 4 * c.st_delta.size());
        add((void**)&w.st_off, c.st_off.size());
        add((void**)&w.table, 4 * c.table.size());
        add((void**)&w.labels, 4 * ns);
        add((void**)xin, 4 * (size_t)g.n * d);
    }
    return off;
}

// The update stencil keeps only the outer columns that can hold a cell
// passing the reference's small box test (EGG_SynC.cu:613-636).  For a cell
// at offset k from the point's own cell, the nearer face in dimension l is
// at least (|k_l| - 1) cells away (the point lies inside its own cell), so
// the test sum_l min(left_l^2, right_l^2) <= eps^2 needs
// sum_{l < od} ((|k_l| - 1)+)^2 <= eps^2 / side^2 (the other dimensions add
// terms >= 0).  The bound is applied with a 1e-3 margin in cells and in the
// squared radius, far above the float rounding of the cell ids and of the
// test, so every cell the test can pass stays a candidate: the results do
// not change, the corner columns are not visited.  (For d = 3 this drops 12
// of the 81 columns of r = 4.)
static Stencil screen_update_stencil(const Geom& g, const Stencil& full) {
    const int od = g.od;
    if (od == 0) return full;
    Stencil S;
    const double R2 = (double)g.t_eps / ((double)g.side * (double)g.side) * (1.0 + 1e-3);
    auto excess = [](int k) {
        const double v = std::abs(k) - 1.001;
        return v > 0.0 ? v * v : 0.0;
    };
    for (size_t s = 0; s < full.delta.size(); s++) {
        double a = 0.0;
        for (int l = 0; l < od; l++) a += excess(full.off[s * od + l]);
        if (a > R2) continue;
        S.delta.push_back(full.delta[s]);
        for (int l = 0; l < od; l++) S.off.push_back(full.off[s * od + l]);
    }
    return S;
}

Consts make_consts(const Geom& g) {
    Consts c;
    Stencil st[3] = {screen_update_stencil(g, make_stencil(g, g.r)), make_stencil(g, g.r_extra),
                     make_stencil(g, g.r_half)};
    for (auto& s : st) c.st_cap = std::max(c.st_cap, (int)s.delta.size());
    const int odp = std::max(g.od, 1);
    const int TW = 2 * g.table_k + 1;
    c.st_delta.assign(3 * (size_t)c.st_cap, 0);
    c.st_off.assign(3 * (size_t)c.st_cap * odp, 0);
    for (int k = 0; k < 3; k++) {
        c.st_count[k] = (int)st[k].delta.size();
        std::copy(st[k].delta.begin(), st[k].delta.end(), c.st_delta.begin() + (size_t)k * c.st_cap);
        std::copy(st[k].off.begin(), st[k].off.end(), c.st_off.begin() + (size_t)k * c.st_cap * odp);
    }
    c.table.resize(3 * (size_t)TW);
    for (int k = -g.table_k; k <= g.table_k; k++) {
        const double a = (double)k * (double)g.side;
        const double sh = sin(0.5 * a);
        c.table[k + g.table_k] = (float)sin(a);
        c.table[TW + k + g.table_k] = (float)cos(a);
        c.table[2 * TW + k + g.table_k] = (float)(2.0 * sh * sh);
    }
    return c;
}

namespace {

// ------------------------------------------------------------------------
// per-device instance: workspace, stream, graph
// ------------------------------------------------------------------------
struct Instance {
    int dev = -1;
    cudaStream_t st = nullptr;
    cudaStream_t side = nullptr;           // second branch of the loop graph (need dilation)
    cudaEvent_t fork = nullptr, join = nullptr;
    cudaEvent_t ev[6] = {};
    cudaEvent_t prof[8] = {};              // kernel-group timing (opts.profile)
    void* base = nullptr;
    size_t cap = 0;
    int* h_ctrl = nullptr;                 // pinned mirror of ctrl
    unsigned long long* h_stamps = nullptr;
    int h_stamps_cap = 0;
    // current layout
    Geom g;
    Work w;
    float* xin = nullptr;                  // staging for host input (n*d)
    int max_iter = 0;
    size_t used = 0;
    mlp::Buffers warm;                     // learned warm start
    cudaEvent_t wev[2] = {};
    // graph cache
    cudaGraphExec_t exec = nullptr;
    std::vector<char> graph_key;
    bool graph_failed = false;
};

std::map<int, Instance*> g_inst;

void destroy_graph(Instance& I) {
    if (I.exec) cudaGraphExecDestroy(I.exec);
    I.exec = nullptr;
    I.graph_key.clear();
}

Instance& instance() {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) throw CudaError{e, "cudaGetDevice"};
    auto it = g_inst.find(dev);
    if (it != g_inst.end()) return *it->second;
    Instance* I = new Instance();
    I->dev = dev;
    EGG_CHECK(cudaStreamCreateWithFlags(&I->st, cudaStreamNonBlocking));
    EGG_CHECK(cudaStreamCreateWithFlags(&I->side, cudaStreamNonBlocking));
    EGG_CHECK(cudaEventCreateWithFlags(&I->fork, cudaEventDisableTiming));
    EGG_CHECK(cudaEventCreateWithFlags(&I->join, cudaEventDisableTiming));
    for (auto& e2 : I->ev) EGG_CHECK(cudaEventCreate(&e2));
    EGG_CHECK(cudaMallocHost((void**)&I->h_ctrl, kCtrlWords * sizeof(int)));
    g_inst[dev] = I;
    return *I;
}

// Lay out the workspace for geometry g (allocating or growing it) and
// upload the stencils and tables.
void prepare(Instance& I, const Geom& g, int max_iter) {
    Work w;
    memset(&w, 0, sizeof(w));
    float* xin = nullptr;
    const size_t off = layout_work(g, max_iter, nullptr, w, &xin, true);
    if (off > I.cap) {
        destroy_graph(I);
        if (I.base) EGG_CHECK(cudaFree(I.base));
        I.base = nullptr;
        I.cap = 0;
        size_t want = off + off / 8;
        EGG_CHECK(dev_alloc((void**)&I.base, want));
        I.cap = want;
    }
    layout_work(g, max_iter, (char*)I.base, w, &xin, true);
    I.used = off;
    const Consts c = make_consts(g);
    w.st_cap = c.st_cap;
    for (int k = 0; k < 3; k++) w.st_count[k] = c.st_count[k];
    // pageable copies are synchronous; sizes are small
    EGG_CHECK(cudaMemcpyAsync(w.st_delta, c.st_delta.data(), c.st_delta.size() * 4, cudaMemcpyHostToDevice, I.st));
    EGG_CHECK(cudaMemcpyAsync(w.st_off, c.st_off.data(), c.st_off.size(), cudaMemcpyHostToDevice, I.st));
    EGG_CHECK(cudaMemcpyAsync(w.table, c.table.data(), c.table.size() * 4, cudaMemcpyHostToDevice, I.st));
    EGG_CHECK(cudaStreamSynchronize(I.st));

    if ((int)((max_iter + 2) * 4) > I.h_stamps_cap) {
        if (I.h_stamps) cudaFreeHost(I.h_stamps);
        I.h_stamps_cap = (max_iter + 2) * 4;
        EGG_CHECK(cudaMallocHost((void**)&I.h_stamps, 8 * (size_t)I.h_stamps_cap));
    }
    I.g = g;
    I.w = w;
    I.xin = xin;
    I.max_iter = max_iter;
}

// ------------------------------------------------------------------------
// loop control kernels
// ------------------------------------------------------------------------
__global__ void k_ctrl_reset(Work w, int max_iter, int full_update) {
    for (int t = threadIdx.x; t < kCtrlWords; t += blockDim.x) w.ctrl[t] = 0;
    for (int t = threadIdx.x; t < kUStats; t += blockDim.x) w.ustats[t] = 0;
    __syncwarp();
    if (threadIdx.x == 0) {
        w.ctrl[kCtrlMaxIter] = max_iter;
        w.ctrl[kCtrlForce] = 1;
        w.ctrl[kCtrlFullUpdate] = full_update;
    }
}

// also opens the grid check (the build-begin step: no point seen leaving its cell yet)
__global__ void k_iter_begin(Work w) {
    const int it = w.ctrl[kCtrlIter];
    w.ctrl[kCtrlFlag] = 1;
    w.ctrl[kCtrlChanged] = 0;
    w.stamps[4 * it + 0] = globaltimer();
}

__global__ void k_iter_end(Work w, cudaGraphConditionalHandle h, int in_graph, int stop_rule) {
    const int it = w.ctrl[kCtrlIter];
    const int flag = w.ctrl[kCtrlFlag];
    w.iter_flags[it] = flag;
    w.stamps[4 * it + 3] = globaltimer();
    const int next = it + 1;
    w.ctrl[kCtrlIter] = next;
    w.ctrl[kCtrlForce] = w.ctrl[kCtrlFullUpdate];
    // stop rule 0: the reference's flag (EGG_SynC.cu:1322); 1: the order
    // parameter's certified lower bound reached lambda (SynC.cpp:277 semantics)
    const int stop = stop_rule ? w.ctrl[kCtrlLamReached] : flag;
    const int done = stop != 0 || next >= w.ctrl[kCtrlMaxIter];
    w.ctrl[kCtrlDone] = done;
    if (in_graph && done) cudaGraphSetConditional(h, 0);
}


// One iteration of the loop body.  With prof (8 events), the four kernel
// groups are bracketed by CUDA events on the launching stream.
// Parts of one iteration: 0 = begin + grid check, 1 = grid sort (skippable
// when no point changed cell), 2 = the rest.  In the loop graph part 2 ends
// at the update (part 3 = the extra check, behind a conditional node; part 4
// = the loop control).
void enqueue_part(Instance& I, int part, cudaGraphConditionalHandle h, int in_graph, cudaEvent_t* prof = nullptr) {
    cudaStream_t st = I.st;
    auto mark = [&](int k) {
        if (prof) EGG_CHECK(cudaEventRecord(prof[k], st));
    };
    if (part == 0) {
        k_iter_begin<<<1, 1, 0, st>>>(I.w);
        mark(0);
        launch_build_check(single(I.g, I.w), st, false);
        return;
    }
    if (part == 1) {
        launch_build_sort(single(I.g, I.w), st);
        return;
    }
    if (part == 3) {
        launch_extra_check(single(I.g, I.w), st, true);
        return;
    }
    if (part == 4) {
        k_iter_end<<<1, 1, 0, st>>>(I.w, h, in_graph, I.g.stop_rule);
        return;
    }
    mark(1);
    mark(2);
    if (in_graph) {
        // the need dilation reads only the dirty marks of the last update: a
        // parallel branch of the graph beside the cell sums
        EGG_CHECK(cudaEventRecord(I.fork, st));
        EGG_CHECK(cudaStreamWaitEvent(I.side, I.fork, 0));
        launch_need(single(I.g, I.w), I.side);
        EGG_CHECK(cudaEventRecord(I.join, I.side));
        launch_cell_sums(single(I.g, I.w), st);
        EGG_CHECK(cudaStreamWaitEvent(st, I.join, 0));
    } else {
        launch_cell_sums(single(I.g, I.w), st);
        launch_need(single(I.g, I.w), st);
    }
    if (I.g.order_mode == 2 || I.g.stop_rule == 1) launch_order_param(I.g, I.w, -1, st);
    mark(3);
    mark(4);
    launch_update(single(I.g, I.w), nullptr, st);
    mark(5);
    if (in_graph) return;  // parts 3 and 4 follow behind the extra check's conditional node
    mark(6);
    launch_extra_check(single(I.g, I.w), st);
    mark(7);
    k_iter_end<<<1, 1, 0, st>>>(I.w, h, in_graph, I.g.stop_rule);
}

// one iteration outside the loop graph (host-driven loop): parts 0-2, the
// last of which runs the extra check and the loop control itself
void enqueue_iteration(Instance& I, cudaGraphConditionalHandle h, int in_graph, cudaEvent_t* prof = nullptr) {
    for (int part = 0; part < 3; part++) enqueue_part(I, part, h, in_graph, prof);
}

// opens the grid-sort node of the loop graph when some point changed cell
__global__ void k_gate_sort(Work w, cudaGraphConditionalHandle hs) {
    cudaGraphSetConditional(hs, w.ctrl[kCtrlChanged] != 0 ? 1u : 0u);
}

std::vector<char> graph_key(const Instance& I) {
    std::vector<char> k(sizeof(Geom) + sizeof(Work) + sizeof(int));
    memcpy(k.data(), &I.g, sizeof(Geom));
    memcpy(k.data() + sizeof(Geom), &I.w, sizeof(Work));
    memcpy(k.data() + sizeof(Geom) + sizeof(Work), &I.max_iter, sizeof(int));
    return k;
}

bool ensure_graph(Instance& I) {
    auto key = graph_key(I);
    if (I.exec && key == I.graph_key) return true;
    destroy_graph(I);
    cudaGraph_t graph = nullptr;
    cudaGraphConditionalHandle h;
    cudaError_t e = cudaGraphCreate(&graph, 0);
    if (e == cudaSuccess) e = cudaGraphConditionalHandleCreate(&h, graph, 1, cudaGraphCondAssignDefault);
    cudaGraph_t body = nullptr;
    if (e == cudaSuccess) {
        cudaGraphNodeParams p = {cudaGraphNodeTypeConditional};
        p.conditional.handle = h;
        p.conditional.type = cudaGraphCondTypeWhile;
        p.conditional.size = 1;
        cudaGraphNode_t node;
        e = cudaGraphAddNode(&node, graph, nullptr, 0, &p);
        if (e == cudaSuccess) body = p.conditional.phGraph_out[0];
    }
    // body: [begin, grid check, gate] -> IF(changed) [grid sort] -> [rest of the iteration]
    cudaGraphConditionalHandle hs;
    cudaGraphNode_t tail = nullptr, ifnode = nullptr;
    if (e == cudaSuccess) e = cudaGraphConditionalHandleCreate(&hs, body, 1, 0);
    if (e == cudaSuccess) e = cudaStreamBeginCaptureToGraph(I.st, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal);
    if (e == cudaSuccess) {
        enqueue_part(I, 0, h, 1);
        k_gate_sort<<<1, 1, 0, I.st>>>(I.w, hs);
        cudaStreamCaptureStatus cs;
        const cudaGraphNode_t* deps = nullptr;
        size_t nd = 0;
        e = cudaStreamGetCaptureInfo(I.st, &cs, nullptr, nullptr, &deps, &nd);
        if (e == cudaSuccess && nd == 1) tail = deps[0];
        cudaGraph_t captured = nullptr;
        const cudaError_t e2 = cudaStreamEndCapture(I.st, &captured);
        if (e == cudaSuccess) e = e2;
        if (e == cudaSuccess && !tail) e = cudaErrorUnknown;
    }
    if (e == cudaSuccess) {
        cudaGraphNodeParams cp = {cudaGraphNodeTypeConditional};
        cp.conditional.handle = hs;
        cp.conditional.type = cudaGraphCondTypeIf;
        cp.conditional.size = 1;
        e = cudaGraphAddNode(&ifnode, body, &tail, 1, &cp);
        if (e == cudaSuccess)
            e = cudaStreamBeginCaptureToGraph(I.st, cp.conditional.phGraph_out[0], nullptr, nullptr, 0,
                                              cudaStreamCaptureModeThreadLocal);
        if (e == cudaSuccess) {
            enqueue_part(I, 1, h, 1);
            cudaGraph_t captured = nullptr;
            e = cudaStreamEndCapture(I.st, &captured);
        }
    }
    // ... -> [rest of the iteration up to the update, gate] -> IF(flag) [extra check] -> [loop control]
    cudaGraphConditionalHandle hx;
    cudaGraphNode_t tail2 = nullptr, ifx = nullptr;
    if (e == cudaSuccess) e = cudaGraphConditionalHandleCreate(&hx, body, 0, 0);
    if (e == cudaSuccess) e = cudaStreamBeginCaptureToGraph(I.st, body, &ifnode, nullptr, 1, cudaStreamCaptureModeThreadLocal);
    if (e == cudaSuccess) {
        enqueue_part(I, 2, h, 1);
        launch_gate_extra(I.w, hx, I.st);
        cudaStreamCaptureStatus cs;
        const cudaGraphNode_t* deps = nullptr;
        size_t nd = 0;
        e = cudaStreamGetCaptureInfo(I.st, &cs, nullptr, nullptr, &deps, &nd);
        if (e == cudaSuccess && nd == 1) tail2 = deps[0];
        cudaGraph_t captured = nullptr;
        const cudaError_t e2 = cudaStreamEndCapture(I.st, &captured);
        if (e == cudaSuccess) e = e2;
        if (e == cudaSuccess && !tail2) e = cudaErrorUnknown;
    }
    if (e == cudaSuccess) {
        cudaGraphNodeParams cp = {cudaGraphNodeTypeConditional};
        cp.conditional.handle = hx;
        cp.conditional.type = cudaGraphCondTypeIf;
        cp.conditional.size = 1;
        e = cudaGraphAddNode(&ifx, body, &tail2, 1, &cp);
        if (e == cudaSuccess)
            e = cudaStreamBeginCaptureToGraph(I.st, cp.conditional.phGraph_out[0], nullptr, nullptr, 0,
                                              cudaStreamCaptureModeThreadLocal);
        if (e == cudaSuccess) {
            enqueue_part(I, 3, h, 1);
            cudaGraph_t captured = nullptr;
            e = cudaStreamEndCapture(I.st, &captured);
        }
    }
    if (e == cudaSuccess) e = cudaStreamBeginCaptureToGraph(I.st, body, &ifx, nullptr, 1, cudaStreamCaptureModeThreadLocal);
    if (e == cudaSuccess) {
        enqueue_part(I, 4, h, 1);
        cudaGraph_t captured = nullptr;
        e = cudaStreamEndCapture(I.st, &captured);
    }
    if (e == cudaSuccess) e = cudaGraphInstantiate(&I.exec, graph, 0);
    if (graph) cudaGraphDestroy(graph);
    if (e != cudaSuccess) {
        cudaGetLastError();
        I.exec = nullptr;
        I.graph_failed = true;
        return false;
    }
    I.graph_key = key;
    return true;
}

// load x (host or device, row-major n x d) into Xn and reset the control words
void load_input(Instance& I, const float* x, int full_update = 0) {
    const Geom& g = I.g;
    const float* src = x;
    if (!is_device_ptr(x)) {
        EGG_CHECK(cudaMemcpyAsync(I.xin, x, sizeof(float) * (size_t)g.n * g.d, cudaMemcpyHostToDevice, I.st));
        src = I.xin;
    }
    k_ctrl_reset<<<1, 32, 0, I.st>>>(I.w, I.max_iter, full_update);
    EGG_CHECK(cudaMemsetAsync(I.w.dirty[0], 0, 8 * ((size_t)g.n_outer + 1), I.st));
    EGG_CHECK(cudaMemsetAsync(I.w.dirty[1], 0, 8 * ((size_t)g.n_outer + 1), I.st));
    launch_transpose_in(g, I.w, src, I.st);
}

void check_status_bits(Instance& I) {
    EGG_CHECK(cudaMemcpyAsync(I.h_ctrl, I.w.ctrl, kCtrlWords * sizeof(int), cudaMemcpyDeviceToHost, I.st));
    EGG_CHECK(cudaStreamSynchronize(I.st));
    if (I.h_ctrl[kCtrlStatus] & kErrNonFinite) throw ArgError{EGG_ERR_INPUT, "input holds NaN or Inf"};
}

void order_after(Instance& I, void* stream) {
    // the internal stream waits for work the caller queued on `stream`
    cudaStream_t cs = (cudaStream_t)stream;
    EGG_CHECK(cudaEventRecord(I.ev[5], cs));
    EGG_CHECK(cudaStreamWaitEvent(I.st, I.ev[5], 0));
}

}  // namespace

// ------------------------------------------------------------------------
// entry points
// ------------------------------------------------------------------------
int run(const float* x, int64_t n, int32_t d, float eps, float lam, const egg_opts* opts_in, int32_t* labels,
        egg_stats* stats, void* stream) {
    if (!x || !labels) throw ArgError{EGG_ERR_ARG, "x and labels must not be NULL"};
    egg_opts opts;
    memset(&opts, 0, sizeof(opts));
    if (opts_in) opts = *opts_in;
    int max_iter = opts.max_iter > 0 ? opts.max_iter : 1000;
    if (max_iter > 1000000) throw ArgError{EGG_ERR_ARG, "max_iter too large"};
    if (opts.stop_rule < 0 || opts.stop_rule > 1) throw ArgError{EGG_ERR_ARG, "stop_rule must be 0 or 1"};
    if (opts.order_param < 0 || opts.order_param > 2) throw ArgError{EGG_ERR_ARG, "order_param must be 0, 1 or 2"};
    if (opts.stop_rule == 1 && !(lam > 0.0f && lam <= 1.0f)) throw ArgError{EGG_ERR_ARG, "lam must be in (0, 1]"};
    Geom g = make_geom(n, d, eps);
    g.stop_rule = opts.stop_rule;
    g.order_mode = opts.stop_rule == 1 ? 2 : opts.order_param;
    g.lam = lam;
    Instance& I = instance();
    EGG_CHECK(cudaEventRecord(I.ev[0], I.st));
    order_after(I, stream);
    prepare(I, g, max_iter);
    load_input(I, x, opts.full_update ? 1 : 0);
    check_status_bits(I);
    float warm_ms = 0.f;
    if (opts.warm_start) {
        // displace the input by the network's prediction; the loop starts there
        if (!I.wev[0])
            for (auto& e : I.wev) EGG_CHECK(cudaEventCreate(&e));
        EGG_CHECK(cudaEventRecord(I.wev[0], I.st));
        mlp::warm_start(*opts.warm_start, I.w.Xn, (size_t)g.ns, g.n, g.d, eps, I.warm, I.st);
        EGG_CHECK(cudaEventRecord(I.wev[1], I.st));
    }
    EGG_CHECK(cudaEventRecord(I.ev[1], I.st));

    float kms[4] = {0, 0, 0, 0};
    int kl[4] = {0, 0, 0, 0};
    bool use_graph = opts.loop == 0 && opts.profile == 0 && ensure_graph(I);
    if (use_graph) {
        EGG_CHECK(cudaGraphLaunch(I.exec, I.st));
    } else {
        cudaEvent_t* prof = opts.profile ? I.prof : nullptr;
        if (prof && !I.prof[0])
            for (auto& e : I.prof) EGG_CHECK(cudaEventCreate(&e));
        for (;;) {
            enqueue_iteration(I, 0, 0, prof);
            EGG_CHECK(cudaMemcpyAsync(I.h_ctrl, I.w.ctrl, kCtrlWords * sizeof(int), cudaMemcpyDeviceToHost, I.st));
            EGG_CHECK(cudaStreamSynchronize(I.st));
            if (prof) {
                for (int k = 0; k < 4; k++) {
                    float t = 0;
                    EGG_CHECK(cudaEventElapsedTime(&t, prof[2 * k], prof[2 * k + 1]));
                    kms[k] += t;
                    kl[k]++;
                }
            }
            if (I.h_ctrl[kCtrlDone]) break;
        }
    }
    EGG_CHECK(cudaEventRecord(I.ev[2], I.st));
    // final grid and labels (EGG_SynC.cu:1503-1522)
    launch_build(single(I.g, I.w), I.st);
    const bool dev_out = is_device_ptr(labels);
    int* lab = dev_out ? labels : I.w.labels;
    if (opts.labels_mode == 1) launch_labels(I.g, I.w, lab, I.st);
    else launch_labels_uf(I.g, I.w, lab, I.st);
    if (g.order_mode == 1) {
        // the final positions' order parameter needs their cell sums
        launch_cell_sums(single(I.g, I.w), I.st);
        launch_order_param(I.g, I.w, max_iter + 1, I.st);
    }
    if (opts.positions_out) {
        const bool dev_p = is_device_ptr(opts.positions_out);
        float* po = dev_p ? opts.positions_out : I.xin;
        launch_unsort_positions(I.g, I.w, I.w.X, po, I.st);
        if (!dev_p)
            EGG_CHECK(cudaMemcpyAsync(opts.positions_out, po, sizeof(float) * (size_t)g.n * g.d,
                                      cudaMemcpyDeviceToHost, I.st));
    }
    EGG_CHECK(cudaEventRecord(I.ev[3], I.st));
    if (!dev_out) EGG_CHECK(cudaMemcpyAsync(labels, lab, sizeof(int) * (size_t)g.n, cudaMemcpyDeviceToHost, I.st));
    EGG_CHECK(cudaMemcpyAsync(I.h_ctrl, I.w.ctrl, kCtrlWords * sizeof(int), cudaMemcpyDeviceToHost, I.st));
    EGG_CHECK(cudaEventRecord(I.ev[4], I.st));
    EGG_CHECK(cudaStreamSynchronize(I.st));
    EGG_CHECK(cudaGetLastError());

    const int iters = I.h_ctrl[kCtrlIter];
    const int converged = (g.stop_rule ? I.h_ctrl[kCtrlLamReached] : I.h_ctrl[kCtrlFlag]) != 0;
#ifdef EGG_UPDATE_STATS
    EGG_CHECK(cudaMemcpy(g_counters, I.w.ustats, sizeof(g_counters), cudaMemcpyDeviceToHost));
#endif
    if (stats) {
        const int M = I.h_ctrl[kCtrlM];
        stats->iterations = iters;
        stats->converged = converged;
        stats->n_cells = M;
        stats->extra_checks = I.h_ctrl[kCtrlExtraRuns];
        stats->status_bits = I.h_ctrl[kCtrlStatus];
        stats->workspace_bytes = (int64_t)I.used;
        stats->order_param = -1.0;
        stats->order_param_lo = stats->order_param_hi = -1.0;
        if (g.order_mode != 0) {
            const int slot = g.order_mode == 1 ? max_iter + 1 : iters - 1;
            double r[2];
            EGG_CHECK(cudaMemcpy(r, I.w.rvals + 2 * slot, sizeof(r), cudaMemcpyDeviceToHost));
            stats->order_param_lo = r[0];
            stats->order_param_hi = r[1];
            stats->order_param = 0.5 * (r[0] + r[1]);
            if (g.order_mode == 2 && stats->itr_order_param) {
                const int cnt = std::min(iters, stats->itr_cap);
                EGG_CHECK(cudaMemcpy(stats->itr_order_param, I.w.rvals, sizeof(double) * 2 * (size_t)cnt,
                                     cudaMemcpyDeviceToHost));
            }
        }
        stats->n_clusters = I.h_ctrl[kCtrlClusters];
        EGG_CHECK(cudaMemcpy(I.h_stamps, I.w.stamps, 8 * 4 * (size_t)iters, cudaMemcpyDeviceToHost));
        double st1 = 0, st2 = 0, st3 = 0;
        for (int it = 0; it < iters; it++) {
            const unsigned long long* s = I.h_stamps + 4 * it;
            st1 += (double)(s[1] - s[0]);
            st2 += (double)(s[2] - s[1]);
            st3 += (double)(s[3] - s[2]);
            if (stats->itr_ms && it < stats->itr_cap) stats->itr_ms[it] = (float)((s[3] - s[0]) * 1e-6);
        }
        float t01, t23, t34, t04;
        EGG_CHECK(cudaEventElapsedTime(&t01, I.ev[0], I.ev[1]));
        EGG_CHECK(cudaEventElapsedTime(&t23, I.ev[2], I.ev[3]));
        EGG_CHECK(cudaEventElapsedTime(&t34, I.ev[3], I.ev[4]));
        EGG_CHECK(cudaEventElapsedTime(&t04, I.ev[0], I.ev[4]));
        stats->stage_ms[0] = t01;
        stats->stage_ms[1] = (float)(st1 * 1e-6);
        stats->stage_ms[2] = (float)(st2 * 1e-6);
        stats->stage_ms[3] = (float)(st3 * 1e-6);
        stats->stage_ms[4] = t23;
        stats->stage_ms[5] = t34;
        stats->total_ms = t04;
        for (int k = 0; k < 4; k++) {
            stats->kernel_ms[k] = kms[k];
            stats->kernel_launches[k] = kl[k];
        }
        // launches: reset + transpose; per iteration: begin, grid check,
        // grid sort (3 per radix pass + 4; with one 32-bit key, 1 + 3 per
        // pass + 4), 2 cell sums, need, [2 order parameter], update, 3 extra
        // check, end; then the final build (begin, check, sort), labels (1
        // or 4 kernels), [2 cell sums + 2 order parameter], [positions].  In
        // the loop graph two gate kernels run every iteration, the grid sort
        // only in iterations where some point changed cell and the extra
        // check only where the update left the flag at 1.
        const bool onekey = I.w.skey[0] != nullptr && g.d <= 3 && g.width <= 256;
        const int sort_l = onekey ? 3 * (1 + g.d) + 5 : 3 * plan_count(g) + 4;
        const int build_l = sort_l + 2;
        const int order_l = (g.order_mode == 2 || g.stop_rule == 1) ? 2 : 0;
        const int final_l = build_l + (opts.labels_mode == 1 ? 1 : 4) + (g.order_mode == 1 ? 4 : 0) +
                            (opts.positions_out ? 1 : 0);
        long long loop_l = (long long)iters * (sort_l + 10 + order_l);
        if (use_graph) {
            // grid builds in the loop: all builds but the final one when it rebuilt
            const int loop_builds = I.h_ctrl[kCtrlBuilds] - (I.h_ctrl[kCtrlChanged] ? 1 : 0);
            loop_l = (long long)iters * (9 + order_l) + 3LL * I.h_ctrl[kCtrlExtraRuns] +
                     (long long)loop_builds * sort_l;
        }
        stats->launches = (int32_t)(2 + loop_l + final_l + (opts.warm_start ? 10 : 0));
        stats->grid_builds = I.h_ctrl[kCtrlBuilds];
        stats->points_updated = (int64_t)(unsigned)I.h_ctrl[kCtrlComputed];
        stats->warm_started = opts.warm_start ? 1 : 0;
        stats->warm_fallback = 0;
        stats->warm_same = 0;
        if (opts.warm_start) EGG_CHECK(cudaEventElapsedTime(&warm_ms, I.wev[0], I.wev[1]));
        stats->warm_ms = warm_ms;
    }
    if (I.h_ctrl[kCtrlStatus] & ~kErrNonFinite)
        throw ArgError{EGG_ERR_INTERNAL, "kernel consistency check failed (status bits " +
                                             std::to_string(I.h_ctrl[kCtrlStatus]) + ")"};
    return converged ? EGG_OK : EGG_MAX_ITER;
}

// identical partitions: -1 in the same places and a bijection between the
// other label values
bool same_partition(const std::vector<int32_t>& a, const std::vector<int32_t>& b) {
    if (a.size() != b.size()) return false;
    std::map<int32_t, int32_t> ab, ba;
    for (size_t i = 0; i < a.size(); i++) {
        if ((a[i] < 0) != (b[i] < 0)) return false;
        if (a[i] < 0) continue;
        auto x = ab.emplace(a[i], b[i]);
        if (x.first->second != b[i]) return false;
        auto y = ba.emplace(b[i], a[i]);
        if (y.first->second != a[i]) return false;
    }
    return true;
}

// Warm start with verification: run from the network's positions and from
// the input, return the warm run when both give the same partition, else
// the plain run (the fallback).
int run_verified(const float* x, int64_t n, int32_t d, float eps, float lam, const egg_opts* opts_in, int32_t* labels,
                 egg_stats* stats, void* stream) {
    if (!x || !labels) throw ArgError{EGG_ERR_ARG, "x and labels must not be NULL"};
    if (n < 1 || n > (int64_t)0x7ffffff0 / 4 || d < 1 || d > kMaxDims) throw ArgError{EGG_ERR_ARG, "n or d out of range"};
    const egg_opts opts = *opts_in;
    const int cap = stats && stats->itr_cap > 0 ? stats->itr_cap : 0;
    struct Leg {
        std::vector<int32_t> lab;
        std::vector<float> pos, itr;
        std::vector<double> itr_r;
        egg_stats st;
        int status;
    } leg[2];
    for (int k = 0; k < 2; k++) {
        Leg& L = leg[k];
        L.lab.resize((size_t)n);
        if (opts.positions_out) L.pos.resize((size_t)n * d);
        L.itr.resize(std::max(cap, 1));
        L.itr_r.resize(2 * (size_t)std::max(cap, 1));
        memset(&L.st, 0, sizeof(L.st));
        L.st.itr_ms = stats && stats->itr_ms ? L.itr.data() : nullptr;
        L.st.itr_order_param = stats && stats->itr_order_param ? L.itr_r.data() : nullptr;
        L.st.itr_cap = cap;
        egg_opts o = opts;
        o.warm_verify = 0;
        if (k == 1) o.warm_start = nullptr;
        o.positions_out = opts.positions_out ? L.pos.data() : nullptr;
        L.status = run(x, n, d, eps, lam, &o, L.lab.data(), &L.st, stream);
    }
    const bool same = same_partition(leg[0].lab, leg[1].lab);
    Leg& R = leg[same ? 0 : 1];
    EGG_CHECK(cudaMemcpy(labels, R.lab.data(), 4 * (size_t)n, cudaMemcpyDefault));
    if (opts.positions_out)
        EGG_CHECK(cudaMemcpy(opts.positions_out, R.pos.data(), 4 * (size_t)n * d, cudaMemcpyDefault));
    if (stats) {
        float* itr = stats->itr_ms;
        double* itr_r = stats->itr_order_param;
        const int icap = stats->itr_cap;
        *stats = R.st;
        stats->itr_ms = itr;
        stats->itr_order_param = itr_r;
        stats->itr_cap = icap;
        const int m = std::min(R.st.iterations, icap);
        if (itr && m > 0) memcpy(itr, R.itr.data(), 4 * (size_t)m);
        if (itr_r && m > 0) memcpy(itr_r, R.itr_r.data(), 16 * (size_t)m);
        stats->warm_same = same ? 1 : 0;
        stats->warm_fallback = same ? 0 : 1;
        stats->warm_started = same ? 1 : 0;
        stats->warm_ms = leg[0].st.warm_ms;
    }
    return R.status;
}

int step(const float* x, int64_t n, int32_t d, float eps, float* x_next, int32_t* counts, int32_t* flags,
         void* stream) {
    if (!x || !x_next || !flags) throw ArgError{EGG_ERR_ARG, "x, x_next and flags must not be NULL"};
    Geom g = make_geom(n, d, eps);
    Instance& I = instance();
    order_after(I, stream);
    prepare(I, g, 4);
    load_input(I, x);
    check_status_bits(I);
    cudaStream_t st = I.st;
    k_iter_begin<<<1, 1, 0, st>>>(I.w);
    launch_build(single(I.g, I.w), st);
    launch_cell_sums(single(I.g, I.w), st);
    launch_need(single(I.g, I.w), st);
    int* cnt_sorted = I.w.orig_tmp;  // free once the grid is built
    launch_update(single(I.g, I.w), cnt_sorted, st);
    EGG_CHECK(cudaMemcpyAsync(I.h_ctrl, I.w.ctrl, kCtrlWords * sizeof(int), cudaMemcpyDeviceToHost, st));
    EGG_CHECK(cudaStreamSynchronize(st));
    flags[0] = I.h_ctrl[kCtrlFlag];
    launch_extra_check(single(I.g, I.w), st);
    EGG_CHECK(cudaMemcpyAsync(I.h_ctrl, I.w.ctrl, kCtrlWords * sizeof(int), cudaMemcpyDeviceToHost, st));
    // updated positions back to the original order (staged in qlo, free now)
    const bool dev_x = is_device_ptr(x_next);
    float* xo = dev_x ? x_next : I.xin;
    launch_unsort_positions(I.g, I.w, I.w.Xn, xo, st);
    if (!dev_x) EGG_CHECK(cudaMemcpyAsync(x_next, xo, sizeof(float) * (size_t)g.n * g.d, cudaMemcpyDeviceToHost, st));
    if (counts) {
        const bool dev_c = is_device_ptr(counts);
        int* co = dev_c ? counts : I.w.labels;
        launch_unsort_int(I.g, I.w, cnt_sorted, co, st);
        if (!dev_c) EGG_CHECK(cudaMemcpyAsync(counts, co, sizeof(int) * (size_t)g.n, cudaMemcpyDeviceToHost, st));
    }
    EGG_CHECK(cudaStreamSynchronize(st));
    EGG_CHECK(cudaGetLastError());
    flags[1] = I.h_ctrl[kCtrlFlag];
    if (I.h_ctrl[kCtrlStatus] & ~kErrNonFinite)
        throw ArgError{EGG_ERR_INTERNAL, "kernel consistency check failed"};
    return EGG_OK;
}

int grid(const float* x, int64_t n, int32_t d, float eps, int32_t* order, int32_t* cell_of, int32_t* cell_start,
         int32_t* n_cells, void* stream) {
    if (!x || !order || !cell_of || !cell_start || !n_cells) throw ArgError{EGG_ERR_ARG, "NULL argument"};
    Geom g = make_geom(n, d, eps);
    Instance& I = instance();
    order_after(I, stream);
    prepare(I, g, 4);
    load_input(I, x);
    check_status_bits(I);
    launch_build(single(I.g, I.w), I.st);
    EGG_CHECK(cudaMemcpyAsync(I.h_ctrl, I.w.ctrl, kCtrlWords * sizeof(int), cudaMemcpyDeviceToHost, I.st));
    EGG_CHECK(cudaStreamSynchronize(I.st));
    const int M = I.h_ctrl[kCtrlM];
    auto out = [&](int32_t* dst, const int* src, size_t cnt) {
        EGG_CHECK(cudaMemcpyAsync(dst, src, sizeof(int) * cnt, cudaMemcpyDefault, I.st));
    };
    out(order, I.w.orig, (size_t)g.n);
    out(cell_of, I.w.cell_of, (size_t)g.n);
    out(cell_start, I.w.cell_start, (size_t)M + 1);
    EGG_CHECK(cudaStreamSynchronize(I.st));
    EGG_CHECK(cudaGetLastError());
    *n_cells = M;
    return EGG_OK;
}

// ------------------------------------------------------------------------
// Grid build without any device allocation.
//
// Some callers cannot allocate device memory: a host framework that has
// reserved the device through its own memory pool (cudaMalloc then fails or
// escapes the framework's accounting), or a latency-critical caller for
// which the implicit device synchronisation of cudaMalloc/cudaFree is not
// acceptable.  egg_sync_grid_noalloc serves them: it runs the same grid
// build as egg_sync_grid, with every scratch buffer carved out of one
// statically sized device array that belongs to this library.
// ------------------------------------------------------------------------
namespace {

constexpr int kNoAllocMaxN = 65536;
constexpr int kNoAllocMaxD = 4;
constexpr size_t kNoAllocBytes = (size_t)8 << 20;  // 8 MiB

// Every GPU on which libeggsync.so is loaded holds this array until the
// process exits.  In host code its name is only a stand-in: the device
// address comes from cudaGetSymbolAddress.
__device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocBytes];

// Device address of g_noalloc_scratch for each device, looked up on the first
// call on that device (with that device current).
void* g_noalloc_addr[256] = {};

__global__ void k_noalloc_reset(int* ctrl) {
    for (int t = threadIdx.x; t < kCtrlWords; t += blockDim.x) ctrl[t] = 0;
}

}  // namespace

int grid_noalloc(const float* x, int64_t n, int32_t d, float eps, int32_t* order, int32_t* cell_of,
                 int32_t* cell_start, int32_t* n_cells, void* stream) {
    if (!x || !order || !cell_of || !cell_start || !n_cells) throw ArgError{EGG_ERR_ARG, "NULL argument"};
    if (n < 1 || n > kNoAllocMaxN || d < 1 || d > kNoAllocMaxD)
        throw ArgError{EGG_ERR_ARG, "egg_sync_grid_noalloc supports 1 <= n <= 65536 and 1 <= d <= 4 (got n = " +
                                        std::to_string(n) + ", d = " + std::to_string(d) + ")"};
    const Geom g = make_geom(n, d, eps);
    int dev = 0;
    EGG_CHECK(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 256) throw ArgError{EGG_ERR_INTERNAL, "device ordinal out of range"};
    if (!g_noalloc_addr[dev]) {
        void* p = nullptr;
        EGG_CHECK(cudaGetSymbolAddress(&p, g_noalloc_scratch));
        g_noalloc_addr[dev] = p;
    }

    // carve the grid build's buffers out of the static array
    const size_t ns = (size_t)g.ns;
    const int tiles = (g.n + kSortTile - 1) / kSortTile;
    const int nb = (g.n + kHeadsBlock - 1) / kHeadsBlock;
    Work w;
    memset(&w, 0, sizeof(w));
    float* xin = nullptr;
    char* base = (char*)g_noalloc_addr[dev];
    size_t off = 0;
    auto take = [&](void** ptr, size_t bytes) {
        *ptr = base + off;
        off += align_up(bytes);
    };
    take((void**)&w.X, 4 * d * ns);
    take((void**)&w.Xn, 4 * d * ns);
    take((void**)&w.orig, 4 * ns);
    take((void**)&w.orig_tmp, 4 * ns);
    take((void**)&w.perm, 4 * ns);
    take((void**)&w.perm_tmp, 4 * ns);
    take((void**)&w.cell_of, 4 * ns);
    take((void**)&w.cell_start, 4 * (ns + 1));
    take((void**)&w.cell_dims, 4 * d * ns);
    take((void**)&w.cell_outer, 4 * ns);
    take((void**)&w.outer_begin, 4 * ((size_t)g.n_outer + 1));
    take((void**)&w.hist, 4 * 256 * (size_t)tiles);
    take((void**)&w.digit_total, 4 * 256);
    take((void**)&w.block_sums, 4 * (size_t)nb);
    take((void**)&w.ctrl, 4 * kCtrlWords);
    take((void**)&w.need, 8 * ((size_t)g.n_outer + 1));
    take((void**)&xin, 4 * (size_t)g.n * d);
    if (off > kNoAllocBytes) throw ArgError{EGG_ERR_INTERNAL, "static scratch too small for this geometry"};

    cudaStream_t st = (cudaStream_t)stream;
    // the array keeps the previous call's contents: the control words must
    // start at zero (every other buffer is fully written before it is read)
    k_noalloc_reset<<<1, 32, 0, st>>>(w.ctrl);
    const float* src = x;
    if (!is_device_ptr(x)) {
        EGG_CHECK(cudaMemcpyAsync(xin, x, sizeof(float) * (size_t)g.n * d, cudaMemcpyHostToDevice, st));
        src = xin;
    }
    launch_transpose_in(g, w, src, st);
    // non-finite input is rejected before the build runs on it (as egg_sync_grid does)
    int ctrl_h[kCtrlWords];
    EGG_CHECK(cudaMemcpyAsync(ctrl_h, w.ctrl, sizeof(ctrl_h), cudaMemcpyDeviceToHost, st));
    EGG_CHECK(cudaStreamSynchronize(st));
    if (ctrl_h[kCtrlStatus] & kErrNonFinite) throw ArgError{EGG_ERR_INPUT, "input holds NaN or Inf"};
    launch_build(single(g, w), st);
    EGG_CHECK(cudaMemcpyAsync(ctrl_h, w.ctrl, sizeof(ctrl_h), cudaMemcpyDeviceToHost, st));
    EGG_CHECK(cudaStreamSynchronize(st));
    const int M = ctrl_h[kCtrlM];
    EGG_CHECK(cudaMemcpyAsync(order, w.orig, sizeof(int) * (size_t)g.n, cudaMemcpyDefault, st));
    EGG_CHECK(cudaMemcpyAsync(cell_of, w.cell_of, sizeof(int) * (size_t)g.n, cudaMemcpyDefault, st));
    EGG_CHECK(cudaMemcpyAsync(cell_start, w.cell_start, sizeof(int) * ((size_t)M + 1), cudaMemcpyDefault, st));
    EGG_CHECK(cudaStreamSynchronize(st));
    EGG_CHECK(cudaGetLastError());
    *n_cells = M;
    return EGG_OK;
}

int release() {
    release_batch();
    mlp::release_all();
    // a device reset after this call may place the static scratch elsewhere:
    // the next allocation-free call looks its address up again
    for (auto& p : g_noalloc_addr) p = nullptr;
    for (auto& kv : g_inst) {
        Instance* I = kv.second;
        int cur = 0;
        cudaGetDevice(&cur);
        cudaSetDevice(I->dev);
        destroy_graph(*I);
        mlp::release(I->warm);
        for (auto e : I->wev)
            if (e) cudaEventDestroy(e);
        if (I->base) cudaFree(I->base);
        if (I->h_ctrl) cudaFreeHost(I->h_ctrl);
        if (I->h_stamps) cudaFreeHost(I->h_stamps);
        for (auto e : I->ev)
            if (e) cudaEventDestroy(e);
        for (auto e : I->prof)
            if (e) cudaEventDestroy(e);
        if (I->st) cudaStreamDestroy(I->st);
        if (I->side) cudaStreamDestroy(I->side);
        if (I->fork) cudaEventDestroy(I->fork);
        if (I->join) cudaEventDestroy(I->join);
        cudaSetDevice(cur);
        delete I;
    }
    g_inst.clear();
    return EGG_OK;
}

}  // namespace egg

// ---------------------------------------------------------------------------
// C ABI
// ---------------------------------------------------------------------------
extern "C" {

__attribute__((visibility("default"))) void egg_opts_default(egg_opts* opts) {
    if (opts) memset(opts, 0, sizeof(*opts));
}

__attribute__((visibility("default"))) int egg_sync_run(const float* x, int64_t n, int32_t d, float eps, float lam,
                                                        const egg_opts* opts, int32_t* labels, egg_stats* stats,
                                                        void* stream) {
    return egg::guarded([&] {
        if (opts && opts->warm_start && opts->warm_verify)
            return egg::run_verified(x, n, d, eps, lam, opts, labels, stats, stream);
        return egg::run(x, n, d, eps, lam, opts, labels, stats, stream);
    });
}

__attribute__((visibility("default"))) int egg_sync_step(const float* x, int64_t n, int32_t d, float eps,
                                                         float* x_next, int32_t* counts, int32_t* flags,
                                                         void* stream) {
    return egg::guarded([&] { return egg::step(x, n, d, eps, x_next, counts, flags, stream); });
}

__attribute__((visibility("default"))) int egg_sync_grid(const float* x, int64_t n, int32_t d, float eps,
                                                         int32_t* order, int32_t* cell_of, int32_t* cell_start,
                                                         int32_t* n_cells, void* stream) {
    return egg::guarded([&] { return egg::grid(x, n, d, eps, order, cell_of, cell_start, n_cells, stream); });
}

__attribute__((visibility("default"))) int egg_sync_grid_noalloc(const float* x, int64_t n, int32_t d, float eps,
                                                                 int32_t* order, int32_t* cell_of,
                                                                 int32_t* cell_start, int32_t* n_cells,
                                                                 void* stream) {
    return egg::guarded(
        [&] { return egg::grid_noalloc(x, n, d, eps, order, cell_of, cell_start, n_cells, stream); });
}

__attribute__((visibility("default"))) const char* egg_status_str(int s) {
    switch (s) {
        case EGG_OK: return "EGG_OK";
        case EGG_MAX_ITER: return "EGG_MAX_ITER";
        case EGG_ERR_ARG: return "EGG_ERR_ARG";
        case EGG_ERR_GEOMETRY: return "EGG_ERR_GEOMETRY";
        case EGG_ERR_INPUT: return "EGG_ERR_INPUT";
        case EGG_ERR_CUDA: return "EGG_ERR_CUDA";
        case EGG_ERR_NO_DEVICE: return "EGG_ERR_NO_DEVICE";
        case EGG_ERR_INTERNAL: return "EGG_ERR_INTERNAL";
        default: return "EGG_UNKNOWN_STATUS";
    }
}

__attribute__((visibility("default"))) const char* egg_last_error(void) { return egg::g_last_error.c_str(); }

__attribute__((visibility("default"))) int egg_release(void) {
    return egg::guarded([&] { return egg::release(); });
}

__attribute__((visibility("default"))) int egg_abi_version(void) { return EGG_SYNC_ABI_VERSION; }

__attribute__((visibility("default"))) int egg_inject_alloc_failures(int32_t count) {
    return egg::guarded([&] {
        if (count < 0) throw egg::ArgError{EGG_ERR_ARG, "count must be >= 0"};
        egg::g_fail_allocs = count;
        return (int)EGG_OK;
    });
}

__attribute__((visibility("default"))) int egg_update_counters(int64_t* out, int32_t cap) {
#ifdef EGG_UPDATE_STATS
    std::lock_guard<std::mutex> lock(egg::g_mutex);
    for (int k = 0; k < egg::kUStats && k < cap; k++) out[k] = (int64_t)egg::g_counters[k];
    return egg::kUStats;
#else
    (void)out;
    (void)cap;
    return 0;
#endif
}

}  // extern "C"
