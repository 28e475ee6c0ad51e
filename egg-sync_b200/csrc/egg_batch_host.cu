// egg_batch_host.cu -- many EGG-SynC instances in one CUDA graph.
//
// The instances of a call (datasets of uneven size and dimension, eps
// sweeps) are grouped by dimension d, since the kernels are specialised on
// it.  One CUDA graph holds the loop: a conditional while node whose body
// runs, for every group on its own branch, the iteration's kernels as
// persistent launches over the group's active instances (egg_batch.cuh),
// then one control kernel that ends the iteration of every instance with
// the reference's stop rule (EGG_SynC.cu:1322), rebuilds each group's active
// list and offset tables, and stops the loop when no instance is left.
// Every instance runs exactly the kernels, in the same order, that a
// single-instance run gives it, so its labels and iteration count are the
// same bits.
//
// Launch configuration (update block size, persistent blocks per SM, the
// order in which instances are listed) is chosen by a small autotuner that
// times the first iterations of the actual batch under each candidate and
// caches the winner per workload signature.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cstring>
#include <map>
#include <numeric>
#include <string>
#include <vector>

#include "eggsync.h"
#include "egg_batch.cuh"
#include "egg_common.cuh"
#include "egg_host_common.h"
#include "egg_kernels.h"

namespace egg {

namespace {

constexpr int kTuneIters = 4;
constexpr int kNumSlots = kShapeCount + 1;  // active flag + one count per launch shape

// ---------------------------------------------------------------------------
// device side
// ---------------------------------------------------------------------------
struct CtlArgs {
    const Geom* geoms;
    const Work* works;
    int count;             // instances
    int ngroups;
    const int* gstart;     // [ngroups + 1] instance ranges of the groups
    const int* sblocks;    // [count][kShapeCount] virtual blocks of each instance per shape
    int* boff;             // group k: [kShapeCount][cap + 1] at boff + k * kShapeCount * (cap + 1)
    int* active;           // group k: [cap] at active + k * cap
    int* nact;             // [ngroups]
    int cap;
    int* loop;             // [2]: loop iterations, any instance active
    unsigned long long* loop_stamps;  // [max_iter + 1] globaltimer at each loop iteration's end
    int max_iter;
};

// exclusive block scan of K ints per thread (blockDim.x <= 1024); tot = totals
template <int K>
__device__ void block_scan_multi(int (&v)[K], int (&tot)[K]) {
    __shared__ int ws[33][K];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const int nw = (blockDim.x + 31) >> 5;
    int incl[K];
#pragma unroll
    for (int k = 0; k < K; k++) {
        int x = v[k];
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, x, o);
            if (lane >= o) x += y;
        }
        incl[k] = x;
        if (lane == 31) ws[wid][k] = x;
    }
    __syncthreads();
    if (wid == 0) {
#pragma unroll
        for (int k = 0; k < K; k++) {
            const int s = lane < nw ? ws[lane][k] : 0;
            int x = s;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const int y = __shfl_up_sync(0xffffffffu, x, o);
                if (lane >= o) x += y;
            }
            if (lane < nw) ws[lane][k] = x - s;
            if (lane == 31) ws[32][k] = x;
        }
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < K; k++) {
        v[k] = incl[k] - v[k] + ws[wid][k];
        tot[k] = ws[32][k];
    }
    __syncthreads();
}

// phase 0: start iteration 0 of every instance with a finite input;
// phase 1: end the iteration of every instance that ran it, start the next
// one of those that go on.  Then rebuild the active lists.
__global__ void __launch_bounds__(1024) k_batch_ctl(CtlArgs a, int phase, cudaGraphConditionalHandle h,
                                                    int in_graph) {
    const int t = threadIdx.x;
    const unsigned long long now = globaltimer();
    bool act = false;
    bool left = false;  // this instance finished in this call
    if (t < a.count) {
        const Work& w = a.works[t];
        int* ctrl = w.ctrl;
        if (phase == 0) {
            act = (ctrl[kCtrlStatus] & kErrNonFinite) == 0;
            if (!act) ctrl[kCtrlDone] = 1;
        } else if (ctrl[kCtrlDone] == 0) {
            // k_iter_end of the single-instance loop, stop rule 0
            const int it = ctrl[kCtrlIter];
            const int flag = ctrl[kCtrlFlag];
            w.iter_flags[it] = flag;
            w.stamps[4 * it + 3] = now;
            const int next = it + 1;
            ctrl[kCtrlIter] = next;
            ctrl[kCtrlForce] = ctrl[kCtrlFullUpdate];
            const int done = flag != 0 || next >= ctrl[kCtrlMaxIter];
            ctrl[kCtrlDone] = done;
            act = !done;
            left = done;
        }
        if (act) {
            // k_iter_begin (with the grid check's begin step)
            ctrl[kCtrlFlag] = 1;
            ctrl[kCtrlChanged] = 0;
            w.stamps[4 * ctrl[kCtrlIter] + 0] = now;
        }
    }
    // The active lists and block offsets change only when an instance
    // finishes: otherwise those of the last call stand.
    const bool rebuild = __syncthreads_or(phase == 0 || left) != 0;
    int any = 0;
    if (!rebuild)
        for (int k = 0; k < a.ngroups; k++) any += a.nact[k];
    for (int k = 0; rebuild && k < a.ngroups; k++) {
        const bool mine = act && t >= a.gstart[k] && t < a.gstart[k + 1];
        int v[kNumSlots], tot[kNumSlots];
        v[0] = mine ? 1 : 0;
#pragma unroll
        for (int s = 0; s < kShapeCount; s++) v[s + 1] = mine ? a.sblocks[(size_t)t * kShapeCount + s] : 0;
        block_scan_multi<kNumSlots>(v, tot);
        int* boff = a.boff + (size_t)k * kShapeCount * (a.cap + 1);
        if (mine) {
            a.active[(size_t)k * a.cap + v[0]] = t;
#pragma unroll
            for (int s = 0; s < kShapeCount; s++) boff[(size_t)s * (a.cap + 1) + v[0]] = v[s + 1];
        }
        if (t == 0) {
            a.nact[k] = tot[0];
#pragma unroll
            for (int s = 0; s < kShapeCount; s++) boff[(size_t)s * (a.cap + 1) + tot[0]] = tot[s + 1];
        }
        any += tot[0];
    }
    if (t == 0) {
        const int li = a.loop[0] + (phase == 1 ? 1 : 0);
        a.loop[0] = li;
        if (li <= a.max_iter) a.loop_stamps[li] = now;
        a.loop[1] = any;
        if (in_graph && any == 0) cudaGraphSetConditional(h, 0);
    }
}

// Opens the conditional node of every group that still has active
// instances (run at the start of each loop iteration).
constexpr int kMaxGroups = 16;
struct GateHandles {
    cudaGraphConditionalHandle h[kMaxGroups];
};

__global__ void k_batch_gate(const int* nact, int ngroups, GateHandles hs) {
    const int k = threadIdx.x;
    if (k < ngroups) cudaGraphSetConditional(hs.h[k], nact[k] > 0 ? 1u : 0u);
}

__global__ void k_batch_reset(const Work* works, int count, int max_iter, int full_update) {
    const int i = blockIdx.x;
    if (i >= count) return;
    int* ctrl = works[i].ctrl;
    for (int t = threadIdx.x; t < kCtrlWords; t += blockDim.x) ctrl[t] = 0;
    for (int t = threadIdx.x; t < kUStats; t += blockDim.x) works[i].ustats[t] = 0;
    __syncwarp();
    if (threadIdx.x == 0) {
        ctrl[kCtrlMaxIter] = max_iter;
        ctrl[kCtrlForce] = 1;
        ctrl[kCtrlFullUpdate] = full_update;
    }
}

// the single-instance load: transpose to SoA, original indices, clear the
// incremental-update marks
__device__ __forceinline__ void load_body(const Geom& g, const Work& w, int bx, int gx) {
    for (size_t t = bx * (size_t)blockDim.x + threadIdx.x; t < (size_t)g.n * g.d; t += (size_t)gx * blockDim.x) {
        const int p = (int)(t / g.d), l = (int)(t % g.d);
        const float v = w.src[t];
        if (!isfinite(v)) atomicOr(w.ctrl + kCtrlStatus, kErrNonFinite);
        w.Xn[(size_t)l * g.ns + p] = v;
        if (l == 0) w.orig[p] = p;
    }
    for (int o = bx * blockDim.x + threadIdx.x; o <= g.n_outer; o += gx * blockDim.x) {
        w.dirty[0][o] = 0;
        w.dirty[1][o] = 0;
    }
}

__global__ void __launch_bounds__(256) kb_load(BatchArgs B) {
    batch_for(B, [&](const Geom& g, const Work& w, int bx, int gx) { load_body(g, w, bx, gx); });
}

__global__ void k_batch_results(const Work* works, int count, int* out) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < count; i += gridDim.x * blockDim.x) {
        const int* c = works[i].ctrl;
        out[5 * i + 0] = c[kCtrlIter];
        out[5 * i + 1] = c[kCtrlFlag];
        out[5 * i + 2] = c[kCtrlClusters];
        out[5 * i + 3] = c[kCtrlStatus];
        out[5 * i + 4] = c[kCtrlM];
    }
}

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------
struct Config {
    int update_threads = 128;
    int occ = 8;
    int order = 1;
    bool operator<(const Config& o) const {
        return std::tie(update_threads, occ, order) < std::tie(o.update_threads, o.occ, o.order);
    }
};

struct Group {
    int d = 0;
    int begin = 0, end = 0;          // positions in the listed order
    BatchTables act, all;            // active list (rebuilt every iteration), every instance
};

struct State {
    int dev = -1;
    cudaStream_t st = nullptr;
    cudaEvent_t ev[4] = {};
    cudaEvent_t fork = nullptr;
    std::vector<cudaStream_t> gstreams;
    std::vector<cudaEvent_t> gjoins;
    void* base = nullptr;
    size_t cap = 0;
    void* h_pinned = nullptr;        // host staging (inputs, labels, results)
    size_t h_cap = 0;
    std::map<Config, cudaGraphExec_t> graphs;
    std::vector<char> graph_key;
    std::map<std::vector<char>, Config> tuned;  // workload signature -> configuration
};

std::map<int, State*> g_states;

void drop_graphs(State& S) {
    for (auto& kv : S.graphs) cudaGraphExecDestroy(kv.second);
    S.graphs.clear();
    S.graph_key.clear();
}

State& state() {
    int dev = 0;
    EGG_CHECK(cudaGetDevice(&dev));
    auto it = g_states.find(dev);
    if (it != g_states.end()) return *it->second;
    State* S = new State();
    S->dev = dev;
    EGG_CHECK(cudaStreamCreateWithFlags(&S->st, cudaStreamNonBlocking));
    for (auto& e : S->ev) EGG_CHECK(cudaEventCreate(&e));
    EGG_CHECK(cudaEventCreateWithFlags(&S->fork, cudaEventDisableTiming));
    g_states[dev] = S;
    return *S;
}

void ensure_group_streams(State& S, int n) {
    while ((int)S.gstreams.size() < n) {
        cudaStream_t s;
        cudaEvent_t e;
        EGG_CHECK(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
        EGG_CHECK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
        S.gstreams.push_back(s);
        S.gjoins.push_back(e);
    }
}

// Everything one call needs, laid out in one device arena.
struct Plan {
    int count = 0;
    int max_iter = 0;
    int full_update = 0;
    std::vector<Geom> geoms;          // by item index
    std::vector<Work> works;          // by item index
    std::vector<size_t> ws_off;       // workspace offset per item
    std::vector<int> order;           // listed order: position -> item
    std::vector<Group> groups;
    std::vector<int> gstart;
    int cap = 0;                      // largest group
    // device pointers
    Geom* d_geoms = nullptr;
    Work* d_works = nullptr;
    int* d_gstart = nullptr;
    int* d_sblocks = nullptr;
    int* d_boff = nullptr;
    int* d_active = nullptr;
    int* d_nact = nullptr;
    int* d_boff_all = nullptr;
    int* d_active_all = nullptr;
    int* d_nact_all = nullptr;
    int* d_loop = nullptr;            // [2 + groups]: iterations, any active, sort openings per group
    int* d_results = nullptr;
    unsigned long long* d_loop_stamps = nullptr;
    float* d_in = nullptr;            // staged host inputs
    int* d_out = nullptr;             // staged host labels
    char* d_consts = nullptr;
    size_t bytes = 0;
    size_t in_floats = 0, out_ints = 0;
    std::vector<size_t> in_off, out_off;  // per item (SIZE_MAX = caller's device memory)
    std::vector<Consts> consts;
    std::vector<size_t> const_off;
    size_t const_bytes = 0;
};

CtlArgs ctl_args(const Plan& P) {
    CtlArgs a;
    a.geoms = P.d_geoms;
    a.works = P.d_works;
    a.count = P.count;
    a.ngroups = (int)P.groups.size();
    a.gstart = P.d_gstart;
    a.sblocks = P.d_sblocks;
    a.boff = P.d_boff;
    a.active = P.d_active;
    a.nact = P.d_nact;
    a.cap = P.cap;
    a.loop = P.d_loop;
    a.loop_stamps = P.d_loop_stamps;
    a.max_iter = P.max_iter;
    return a;
}

// Host-side tables of the listed order for configuration c: descriptors,
// per-shape block counts and the static every-instance tables.
void upload_order(State& S, Plan& P, const Config& c) {
    const int G = (int)P.groups.size();
    P.order.clear();
    for (int k = 0; k < G; k++) {
        std::vector<int> items;
        for (int i = 0; i < P.count; i++)
            if (P.geoms[i].d == P.groups[k].d) items.push_back(i);
        if (c.order == 1)
            std::stable_sort(items.begin(), items.end(),
                             [&](int a, int b) { return P.geoms[a].n > P.geoms[b].n; });
        P.groups[k].begin = (int)P.order.size();
        P.order.insert(P.order.end(), items.begin(), items.end());
        P.groups[k].end = (int)P.order.size();
        P.gstart[k] = P.groups[k].begin;
        P.gstart[k + 1] = P.groups[k].end;
    }
    std::vector<Geom> hg(P.count);
    std::vector<Work> hw(P.count);
    std::vector<int> sb((size_t)P.count * kShapeCount);
    for (int pos = 0; pos < P.count; pos++) {
        const int i = P.order[pos];
        hg[pos] = P.geoms[i];
        hw[pos] = P.works[i];
        for (int s = 0; s < kShapeCount; s++) sb[(size_t)pos * kShapeCount + s] = shape_blocks(s, P.geoms[i]);
    }
    const size_t tab = (size_t)kShapeCount * (P.cap + 1);
    std::vector<int> boff_all((size_t)G * tab, 0), active_all((size_t)G * P.cap, 0), nact_all(G, 0);
    for (int k = 0; k < G; k++) {
        const Group& gr = P.groups[k];
        const int m = gr.end - gr.begin;
        nact_all[k] = m;
        for (int j = 0; j < m; j++) active_all[(size_t)k * P.cap + j] = gr.begin + j;
        for (int s = 0; s < kShapeCount; s++) {
            int run = 0;
            for (int j = 0; j <= m; j++) {
                boff_all[(size_t)k * tab + (size_t)s * (P.cap + 1) + j] = run;
                if (j < m) run += sb[(size_t)(gr.begin + j) * kShapeCount + s];
            }
        }
    }
    cudaStream_t st = S.st;
    EGG_CHECK(cudaMemcpyAsync(P.d_geoms, hg.data(), sizeof(Geom) * P.count, cudaMemcpyHostToDevice, st));
    EGG_CHECK(cudaMemcpyAsync(P.d_works, hw.data(), sizeof(Work) * P.count, cudaMemcpyHostToDevice, st));
    EGG_CHECK(cudaMemcpyAsync(P.d_sblocks, sb.data(), 4 * sb.size(), cudaMemcpyHostToDevice, st));
    EGG_CHECK(cudaMemcpyAsync(P.d_gstart, P.gstart.data(), 4 * P.gstart.size(), cudaMemcpyHostToDevice, st));
    EGG_CHECK(cudaMemcpyAsync(P.d_boff_all, boff_all.data(), 4 * boff_all.size(), cudaMemcpyHostToDevice, st));
    EGG_CHECK(cudaMemcpyAsync(P.d_active_all, active_all.data(), 4 * active_all.size(), cudaMemcpyHostToDevice, st));
    EGG_CHECK(cudaMemcpyAsync(P.d_nact_all, nact_all.data(), 4 * nact_all.size(), cudaMemcpyHostToDevice, st));
    EGG_CHECK(cudaStreamSynchronize(st));  // the host vectors go out of scope
}

void set_tables(Plan& P, const Config& c) {
    const size_t tab = (size_t)kShapeCount * (P.cap + 1);
    for (int k = 0; k < (int)P.groups.size(); k++) {
        Group& gr = P.groups[k];
        for (BatchTables* bt : {&gr.act, &gr.all}) {
            bt->geoms = P.d_geoms;
            bt->works = P.d_works;
            bt->cap = P.cap;
            bt->occ = c.occ;
            bt->update_threads = c.update_threads;
            bt->max_passes = 0;
            bt->max_table_k = 0;
            for (int s = 0; s < kShapeCount; s++) bt->total[s] = 0;
            for (int i = 0; i < P.count; i++) {
                if (P.geoms[i].d != gr.d) continue;
                bt->max_passes = std::max(bt->max_passes, plan_count(P.geoms[i]));
                bt->max_table_k = std::max(bt->max_table_k, P.geoms[i].table_k);
                for (int s = 0; s < kShapeCount; s++) bt->total[s] += shape_blocks(s, P.geoms[i]);
            }
        }
        gr.act.boff = P.d_boff + k * tab;
        gr.act.active = P.d_active + (size_t)k * P.cap;
        gr.act.nact = P.d_nact + k;
        gr.all.boff = P.d_boff_all + k * tab;
        gr.all.active = P.d_active_all + (size_t)k * P.cap;
        gr.all.nact = P.d_nact_all + k;
    }
}

// one iteration of group k's instances.  Parts, in order: 0 = grid check,
// 1 = grid sort, 2 = cell sums, need, update, 3 = extra check; in the loop
// graph parts 1 and 3 sit behind conditional nodes (gated: the extra
// check's gate did the stage stamp and count).  -1 = all four, ungated.
void enqueue_group(Plan& P, int k, cudaStream_t st, int part = -1) {
    Group& gr = P.groups[k];
    const Exec ex = batched(gr.act, gr.d);
    const bool all = part < 0;
    if (all || part == 0) launch_build_check(ex, st, false);  // the control kernel cleared the changed words
    if (all || part == 1) launch_build_sort(ex, st);
    if (all || part == 2) {
        launch_cell_sums(ex, st);
        launch_need(ex, st);
        launch_update(ex, nullptr, st);
    }
    if (all || part == 3) launch_extra_check(ex, st, part == 3);
}

void enqueue_iteration(State& S, Plan& P, cudaGraphConditionalHandle h, int in_graph) {
    const int G = (int)P.groups.size();
    if (G > 1) EGG_CHECK(cudaEventRecord(S.fork, S.st));
    for (int k = 0; k < G; k++) {
        cudaStream_t st = G > 1 ? S.gstreams[k] : S.st;
        if (G > 1) EGG_CHECK(cudaStreamWaitEvent(st, S.fork, 0));
        enqueue_group(P, k, st);
        if (G > 1) {
            EGG_CHECK(cudaEventRecord(S.gjoins[k], st));
            EGG_CHECK(cudaStreamWaitEvent(S.st, S.gjoins[k], 0));
        }
    }
    k_batch_ctl<<<1, 1024, 0, S.st>>>(ctl_args(P), 1, h, in_graph);
}

// What a captured loop depends on besides the configuration: the arena's
// pointers and, per group, its dimension and launch sizes.  The contents of
// the descriptor arrays (instance order included) are read at run time.
std::vector<char> graph_key(const Plan& P) {
    std::vector<char> k;
    auto put = [&](const void* p, size_t b) { k.insert(k.end(), (const char*)p, (const char*)p + b); };
    put(&P.d_geoms, sizeof(void*));
    put(&P.d_boff, sizeof(void*));
    put(&P.count, sizeof(int));
    put(&P.cap, sizeof(int));
    for (const Group& g : P.groups) {
        put(&g.d, sizeof(int));
        put(g.act.total, sizeof(g.act.total));
        put(&g.act.max_passes, sizeof(int));
        put(&g.act.max_table_k, sizeof(int));
    }
    return k;
}

cudaGraphExec_t get_graph(State& S, Plan& P, const Config& c) {
    auto key = graph_key(P);
    if (key != S.graph_key) {
        drop_graphs(S);
        S.graph_key = key;
    }
    auto it = S.graphs.find(c);
    if (it != S.graphs.end()) return it->second;
    cudaGraph_t graph = nullptr;
    cudaGraphConditionalHandle h;
    cudaGraphExec_t exec = nullptr;
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
    const int G = (int)P.groups.size();
    if (e == cudaSuccess && G <= kMaxGroups) {
        // body: gate kernel -> one conditional IF node per group (siblings, so
        // the groups run concurrently and an idle group launches nothing) ->
        // control kernel
        GateHandles hs = {};
        for (int k = 0; k < G && e == cudaSuccess; k++)
            e = cudaGraphConditionalHandleCreate(&hs.h[k], body, 1, 0);
        cudaGraphNode_t gate = nullptr;
        if (e == cudaSuccess) {
            int ng = G;
            void* gargs[] = {&P.d_nact, &ng, &hs};
            cudaKernelNodeParams kp = {};
            kp.func = (void*)k_batch_gate;
            kp.gridDim = dim3(1);
            kp.blockDim = dim3(32);
            kp.kernelParams = gargs;
            e = cudaGraphAddKernelNode(&gate, body, nullptr, 0, &kp);
        }
        std::vector<cudaGraphNode_t> ifs(G);
        for (int k = 0; k < G && e == cudaSuccess; k++) {
            cudaGraphNodeParams cp = {cudaGraphNodeTypeConditional};
            cp.conditional.handle = hs.h[k];
            cp.conditional.type = cudaGraphCondTypeIf;
            cp.conditional.size = 1;
            e = cudaGraphAddNode(&ifs[k], body, &gate, 1, &cp);
            if (e != cudaSuccess) break;
            // group body: [check, gate] -> IF(some point changed cell) [sort] ->
            // [cell sums .. update, gate] -> IF(some instance flagged) [extra check]
            cudaGraph_t gbody = cp.conditional.phGraph_out[0];
            const Exec gex = batched(P.groups[k].act, P.groups[k].d);
            cudaGraphNode_t prev = nullptr;  // last node so far (nullptr: none)
            bool ok = true;
            // capture `fn` into graph `into` after the dependency `dep`; its last node -> *last
            auto seg = [&](cudaGraph_t into, cudaGraphNode_t dep, cudaGraphNode_t* last, auto&& fn) {
                cudaError_t r = cudaStreamBeginCaptureToGraph(S.st, into, dep ? &dep : nullptr, nullptr, dep ? 1 : 0,
                                                              cudaStreamCaptureModeThreadLocal);
                if (r != cudaSuccess) return r;
                try {
                    fn();
                    if (last) {
                        cudaStreamCaptureStatus cs;
                        const cudaGraphNode_t* deps = nullptr;
                        size_t nd = 0;
                        EGG_CHECK(cudaStreamGetCaptureInfo(S.st, &cs, nullptr, nullptr, &deps, &nd));
                        *last = nd == 1 ? deps[0] : nullptr;
                    }
                } catch (const CudaError& ce) {
                    ok = false;
                    r = ce.code;
                }
                cudaGraph_t captured = nullptr;
                const cudaError_t r2 = cudaStreamEndCapture(S.st, &captured);
                if (r == cudaSuccess) r = r2;
                if (r == cudaSuccess && last && !*last) r = cudaErrorUnknown;
                return r;
            };
            // an IF node after `dep` whose body is `fn`; the node -> *node
            auto cond = [&](cudaGraphConditionalHandle hc, cudaGraphNode_t dep, cudaGraphNode_t* node, auto&& fn) {
                cudaGraphNodeParams xp = {cudaGraphNodeTypeConditional};
                xp.conditional.handle = hc;
                xp.conditional.type = cudaGraphCondTypeIf;
                xp.conditional.size = 1;
                cudaError_t r = cudaGraphAddNode(node, gbody, &dep, 1, &xp);
                if (r == cudaSuccess) r = seg(xp.conditional.phGraph_out[0], nullptr, nullptr, fn);
                return r;
            };
            cudaGraphConditionalHandle hsort, hx;
            e = cudaGraphConditionalHandleCreate(&hsort, gbody, 0, 0);
            if (e == cudaSuccess) e = cudaGraphConditionalHandleCreate(&hx, gbody, 0, 0);
            if (e == cudaSuccess)
                e = seg(gbody, nullptr, &prev, [&] {
                    enqueue_group(P, k, S.st, 0);
                    launch_batch_gate_sort(gex, hsort, P.d_loop + 2 + k, S.st);
                });
            cudaGraphNode_t ifs_sort = nullptr, ifs_x = nullptr;
            if (e == cudaSuccess) e = cond(hsort, prev, &ifs_sort, [&] { enqueue_group(P, k, S.st, 1); });
            if (e == cudaSuccess)
                e = seg(gbody, ifs_sort, &prev, [&] {
                    enqueue_group(P, k, S.st, 2);
                    launch_batch_gate_extra(gex, hx, S.st);
                });
            if (e == cudaSuccess) e = cond(hx, prev, &ifs_x, [&] { enqueue_group(P, k, S.st, 3); });
            if (!ok && e == cudaSuccess) e = cudaErrorUnknown;
        }
        if (e == cudaSuccess) {
            CtlArgs a = ctl_args(P);
            int phase = 1, in_graph = 1;
            void* cargs[] = {&a, &phase, &h, &in_graph};
            cudaKernelNodeParams kp = {};
            kp.func = (void*)k_batch_ctl;
            kp.gridDim = dim3(1);
            kp.blockDim = dim3(1024);
            kp.kernelParams = cargs;
            cudaGraphNode_t ctl;
            e = cudaGraphAddKernelNode(&ctl, body, ifs.data(), G, &kp);
        }
    } else if (e == cudaSuccess) {
        e = cudaStreamBeginCaptureToGraph(S.st, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal);
        if (e == cudaSuccess) {
            bool ok = true;
            try {
                enqueue_iteration(S, P, h, 1);
            } catch (const CudaError& ce) {
                ok = false;
                e = ce.code;
            }
            cudaGraph_t captured = nullptr;
            const cudaError_t e2 = cudaStreamEndCapture(S.st, &captured);
            if (ok) e = e2;
        }
    }
    if (e == cudaSuccess) e = cudaGraphInstantiate(&exec, graph, 0);
    if (graph) cudaGraphDestroy(graph);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return nullptr;
    }
    S.graphs[c] = exec;
    return exec;
}

// Lay the call out: validation, geometry, arena offsets (no device work).
void make_plan(State& S, Plan& P, egg_batch_item* items, int count, const egg_opts& opts) {
    P.count = count;
    P.max_iter = opts.max_iter > 0 ? opts.max_iter : 1000;
    P.full_update = opts.full_update ? 1 : 0;
    P.geoms.resize(count);
    P.works.resize(count);
    P.ws_off.resize(count);
    P.in_off.assign(count, SIZE_MAX);
    P.out_off.assign(count, SIZE_MAX);
    P.consts.resize(count);
    P.const_off.resize(count);
    std::vector<int> ds;
    size_t off = 0;
    for (int i = 0; i < count; i++) {
        egg_batch_item& it = items[i];
        if (!it.x || !it.labels)
            throw ArgError{EGG_ERR_ARG, "item " + std::to_string(i) + ": x and labels must not be NULL"};
        try {
            P.geoms[i] = make_geom(it.n, it.d, it.eps);
        } catch (ArgError& e) {
            e.msg = "item " + std::to_string(i) + ": " + e.msg;
            throw;
        }
        Geom& g = P.geoms[i];
        g.stop_rule = 0;
        g.order_mode = 0;
        Work w;
        memset(&w, 0, sizeof(w));
        P.ws_off[i] = off;
        off += layout_work(g, P.max_iter, nullptr, w, nullptr, false);
        P.consts[i] = make_consts(g);
        if (std::find(ds.begin(), ds.end(), g.d) == ds.end()) ds.push_back(g.d);
    }
    std::sort(ds.begin(), ds.end());
    P.groups.assign(ds.size(), Group());
    P.gstart.assign(ds.size() + 1, 0);
    P.cap = 1;
    for (size_t k = 0; k < ds.size(); k++) {
        P.groups[k].d = ds[k];
        int m = 0;
        for (int i = 0; i < count; i++) m += P.geoms[i].d == ds[k];
        P.cap = std::max(P.cap, m);
    }
    const size_t ws_bytes = off;
    // inputs and labels in host memory are staged in two arenas
    P.in_floats = 0;
    P.out_ints = 0;
    for (int i = 0; i < count; i++) {
        const size_t nd = (size_t)P.geoms[i].n * P.geoms[i].d;
        if (!is_device_ptr(items[i].x)) {
            P.in_off[i] = P.in_floats;
            P.in_floats += (nd + 63) & ~(size_t)63;
        }
        if (!is_device_ptr(items[i].labels)) {
            P.out_off[i] = P.out_ints;
            P.out_ints += ((size_t)P.geoms[i].n + 63) & ~(size_t)63;
        }
    }
    P.const_bytes = 0;
    for (int i = 0; i < count; i++) {
        const Consts& c = P.consts[i];
        P.const_off[i] = P.const_bytes;
        P.const_bytes += align_up(4 * c.st_delta.size()) + align_up(c.st_off.size()) + align_up(4 * c.table.size());
    }
    const int G = (int)P.groups.size();
    const size_t tab = (size_t)G * kShapeCount * (P.cap + 1);
    size_t total = 0;
    auto reserve = [&](size_t b) {
        const size_t o = total;
        total += align_up(b);
        return o;
    };
    const size_t o_ws = reserve(ws_bytes);
    const size_t o_geoms = reserve(sizeof(Geom) * count);
    const size_t o_works = reserve(sizeof(Work) * count);
    const size_t o_gstart = reserve(4 * (G + 1));
    const size_t o_sb = reserve(4 * (size_t)count * kShapeCount);
    const size_t o_boff = reserve(4 * tab);
    const size_t o_act = reserve(4 * (size_t)G * P.cap);
    const size_t o_nact = reserve(4 * G);
    const size_t o_boff_all = reserve(4 * tab);
    const size_t o_act_all = reserve(4 * (size_t)G * P.cap);
    const size_t o_nact_all = reserve(4 * G);
    const size_t o_loop = reserve(4 * (2 + (size_t)G));
    const size_t o_res = reserve(4 * 5 * (size_t)count);
    const size_t o_ls = reserve(8 * ((size_t)P.max_iter + 2));
    const size_t o_in = reserve(4 * P.in_floats);
    const size_t o_out = reserve(4 * P.out_ints);
    const size_t o_consts = reserve(P.const_bytes);
    if (total > S.cap) {
        drop_graphs(S);
        if (S.base) EGG_CHECK(cudaFree(S.base));
        S.base = nullptr;
        S.cap = 0;
        const size_t want = total + total / 8;
        EGG_CHECK(dev_alloc((void**)&S.base, want));
        S.cap = want;
    }
    char* b = (char*)S.base;
    P.bytes = total;
    P.d_geoms = (Geom*)(b + o_geoms);
    P.d_works = (Work*)(b + o_works);
    P.d_gstart = (int*)(b + o_gstart);
    P.d_sblocks = (int*)(b + o_sb);
    P.d_boff = (int*)(b + o_boff);
    P.d_active = (int*)(b + o_act);
    P.d_nact = (int*)(b + o_nact);
    P.d_boff_all = (int*)(b + o_boff_all);
    P.d_active_all = (int*)(b + o_act_all);
    P.d_nact_all = (int*)(b + o_nact_all);
    P.d_loop = (int*)(b + o_loop);
    P.d_results = (int*)(b + o_res);
    P.d_loop_stamps = (unsigned long long*)(b + o_ls);
    P.d_in = (float*)(b + o_in);
    P.d_out = (int*)(b + o_out);
    P.d_consts = b + o_consts;
    for (int i = 0; i < count; i++) {
        Work& w = P.works[i];
        memset(&w, 0, sizeof(w));
        layout_work(P.geoms[i], P.max_iter, b + o_ws + P.ws_off[i], w, nullptr, false);
        const Consts& c = P.consts[i];
        char* cb = P.d_consts + P.const_off[i];
        w.st_delta = (int*)cb;
        cb += align_up(4 * c.st_delta.size());
        w.st_off = (signed char*)cb;
        cb += align_up(c.st_off.size());
        w.table = (float*)cb;
        w.st_cap = c.st_cap;
        for (int k = 0; k < 3; k++) w.st_count[k] = c.st_count[k];
        w.src = P.in_off[i] == SIZE_MAX ? items[i].x : P.d_in + P.in_off[i];
        w.labels = P.out_off[i] == SIZE_MAX ? items[i].labels : P.d_out + P.out_off[i];
    }
}

void ensure_pinned(State& S, size_t bytes) {
    if (bytes <= S.h_cap) return;
    if (S.h_pinned) EGG_CHECK(cudaFreeHost(S.h_pinned));
    S.h_pinned = nullptr;
    S.h_cap = 0;
    EGG_CHECK(cudaMallocHost(&S.h_pinned, bytes + bytes / 8));
    S.h_cap = bytes + bytes / 8;
}

// constants and staged inputs to the device
void upload_inputs(State& S, Plan& P, egg_batch_item* items) {
    const size_t in_b = 4 * P.in_floats;
    char* h = (char*)S.h_pinned;
    for (int i = 0; i < P.count; i++) {
        const Consts& c = P.consts[i];
        char* cb = h + P.const_off[i];
        memcpy(cb, c.st_delta.data(), 4 * c.st_delta.size());
        cb += align_up(4 * c.st_delta.size());
        memcpy(cb, c.st_off.data(), c.st_off.size());
        cb += align_up(c.st_off.size());
        memcpy(cb, c.table.data(), 4 * c.table.size());
    }
    EGG_CHECK(cudaMemcpyAsync(P.d_consts, h, P.const_bytes, cudaMemcpyHostToDevice, S.st));
    EGG_CHECK(cudaStreamSynchronize(S.st));
    if (in_b) {
        float* hf = (float*)S.h_pinned;
        for (int i = 0; i < P.count; i++)
            if (P.in_off[i] != SIZE_MAX)
                memcpy(hf + P.in_off[i], items[i].x, 4 * (size_t)P.geoms[i].n * P.geoms[i].d);
        EGG_CHECK(cudaMemcpyAsync(P.d_in, hf, in_b, cudaMemcpyHostToDevice, S.st));
    }
}

// reset + load + control phase 0 (start iteration 0)
int enqueue_prologue(State& S, Plan& P, int max_iter) {
    k_batch_reset<<<P.count, 32, 0, S.st>>>(P.d_works, P.count, max_iter, P.full_update);
    int launches = 1;
    for (Group& gr : P.groups) {
        const Exec ex = batched(gr.all, gr.d);
        kb_load<<<ex.blocks(kShapeCapN256L, 256), 256, 0, S.st>>>(ex.args(kShapeCapN256L));
        launches++;
    }
    EGG_CHECK(cudaMemsetAsync(P.d_loop, 0, 4 * (2 + P.groups.size()), S.st));
    k_batch_ctl<<<1, 1024, 0, S.st>>>(ctl_args(P), 0, 0, 0);
    return launches + 1;
}

// kernels of one group's iteration: grid check, sort (radix passes, 4
// tables), cell sums (2), need, update, extra check (3)
int sort_launches(const Group& gr) { return 3 * gr.act.max_passes + 4; }
int group_launches(const Group& gr) { return 1 + sort_launches(gr) + 2 + 1 + 1 + 3; }

// Kernels of the loop graph: gate and control every iteration, and each
// group's kernels in the iterations where it had active instances (the
// largest iteration count among its instances; an idle group's conditional
// node launches nothing): the two gates every such iteration, the sort
// where its gate opened (counted on the device), the three extra-check
// kernels only where an instance's flag reached it (counted once per
// instance: its final iteration).
long long loop_launches(const Plan& P, int loop_iters, const std::vector<int>& res) {
    long long l = 2LL * loop_iters;
    const int* opened = res.data() + 5 * (size_t)P.count + 2;
    for (size_t k = 0; k < P.groups.size(); k++) {
        const Group& gr = P.groups[k];
        int m = 0;
        for (int pos = gr.begin; pos < gr.end; pos++) m = std::max(m, res[5 * (size_t)pos]);
        l += (long long)m * (group_launches(gr) - 3 - sort_launches(gr) + 2) +
             (long long)opened[k] * sort_launches(gr) + 3LL * (gr.end - gr.begin);
    }
    return l;
}

// the loop: the graph, or (fallback) host-driven iterations
int enqueue_loop(State& S, Plan& P, const Config& c, bool host_loop) {
    cudaGraphExec_t exec = host_loop ? nullptr : get_graph(S, P, c);
    if (exec) {
        EGG_CHECK(cudaGraphLaunch(exec, S.st));
        return -1;
    }
    int iters = 0;
    int any = 1;
    while (any) {
        enqueue_iteration(S, P, 0, 0);
        EGG_CHECK(cudaMemcpyAsync(&any, P.d_loop + 1, 4, cudaMemcpyDeviceToHost, S.st));
        EGG_CHECK(cudaStreamSynchronize(S.st));
        iters++;
    }
    return iters;
}

float time_trial(State& S, Plan& P, const Config& c) {
    upload_order(S, P, c);
    set_tables(P, c);
    EGG_CHECK(cudaEventRecord(S.ev[0], S.st));
    // per-instance stamps and flags are sized for P.max_iter iterations
    enqueue_prologue(S, P, std::min(kTuneIters, P.max_iter));
    enqueue_loop(S, P, c, false);
    EGG_CHECK(cudaEventRecord(S.ev[1], S.st));
    EGG_CHECK(cudaEventSynchronize(S.ev[1]));
    float ms = 0;
    EGG_CHECK(cudaEventElapsedTime(&ms, S.ev[0], S.ev[1]));
    return ms;
}

// Coordinate descent over the three knobs on the first iterations of the
// batch itself.  Every candidate computes the same bits; only time differs.
// A candidate's time is the better of two trials (single trials of a few
// milliseconds differ by several percent from one to the next).
Config autotune(State& S, Plan& P) {
    Config best;
    time_trial(S, P, best);  // warm-up: graph instantiation, caches
    auto trial2 = [&](const Config& c) { return std::min(time_trial(S, P, c), time_trial(S, P, c)); };
    float tb = trial2(best);
    auto consider = [&](Config c) {
        const float t = trial2(c);
        if (t < tb) {
            tb = t;
            best = c;
        }
    };
    consider(Config{best.update_threads, best.occ, 1 - best.order});
    const Config b1 = best;
    for (int ut : {64, 256}) consider(Config{ut, b1.occ, b1.order});
    const Config b2 = best;
    for (int occ : {4, 16}) consider(Config{b2.update_threads, occ, b2.order});
    return best;
}

std::vector<char> signature(const Plan& P, const egg_opts& opts) {
    std::vector<char> k;
    auto put = [&](const void* p, size_t b) { k.insert(k.end(), (const char*)p, (const char*)p + b); };
    put(&P.count, sizeof(int));
    put(&opts.full_update, sizeof(int));
    for (const Geom& g : P.geoms) {
        put(&g.n, sizeof(int));
        put(&g.d, sizeof(int));
        put(&g.eps, sizeof(float));
    }
    return k;
}

}  // namespace

int run_batch(egg_batch_item* items, int count, const egg_opts* opts_in, egg_batch_stats* stats, void* stream) {
    if (!items) throw ArgError{EGG_ERR_ARG, "items must not be NULL"};
    if (count < 1 || count > kMaxBatch) throw ArgError{EGG_ERR_ARG, "count must be in [1, 1024]"};
    egg_opts opts;
    memset(&opts, 0, sizeof(opts));
    if (opts_in) opts = *opts_in;
    if (opts.max_iter > 1000000) throw ArgError{EGG_ERR_ARG, "max_iter too large"};
    if (opts.stop_rule != 0 || opts.order_param != 0)
        throw ArgError{EGG_ERR_ARG, "egg_sync_batch supports stop_rule 0 and order_param 0 only"};
    if (opts.batch_tune < 0 || opts.batch_tune > 2) throw ArgError{EGG_ERR_ARG, "batch_tune must be 0, 1 or 2"};
    // every argument error is reported before the first CUDA call
    for (int i = 0; i < count; i++) {
        if (!items[i].x || !items[i].labels)
            throw ArgError{EGG_ERR_ARG, "item " + std::to_string(i) + ": x and labels must not be NULL"};
        try {
            make_geom(items[i].n, items[i].d, items[i].eps);
        } catch (ArgError& e) {
            e.msg = "item " + std::to_string(i) + ": " + e.msg;
            throw;
        }
    }
    State& S = state();
    {
        cudaStream_t cs = (cudaStream_t)stream;
        EGG_CHECK(cudaEventRecord(S.ev[3], cs));
        EGG_CHECK(cudaStreamWaitEvent(S.st, S.ev[3], 0));
    }
    Plan P;
    make_plan(S, P, items, count, opts);
    ensure_group_streams(S, (int)P.groups.size());
    ensure_pinned(S, std::max(std::max(4 * P.in_floats, P.const_bytes),
                              std::max(4 * P.out_ints, 4 * 5 * (size_t)count + 16)));
    upload_inputs(S, P, items);

    // launch configuration
    Config cfg;
    bool tuned_now = false;
    float tune_ms = 0.f;
    if (opts.batch_tune != 1 && opts.loop == 0) {
        const auto sig = signature(P, opts);
        auto it = S.tuned.find(sig);
        if (it != S.tuned.end() && opts.batch_tune == 0) {
            cfg = it->second;
        } else {
            const auto t0 = std::chrono::steady_clock::now();
            cfg = autotune(S, P);
            tune_ms = std::chrono::duration<float, std::milli>(std::chrono::steady_clock::now() - t0).count();
            S.tuned[sig] = cfg;
            tuned_now = true;
        }
    }
    upload_order(S, P, cfg);
    set_tables(P, cfg);

    EGG_CHECK(cudaEventRecord(S.ev[0], S.st));
    int launches = enqueue_prologue(S, P, P.max_iter);
    EGG_CHECK(cudaEventRecord(S.ev[1], S.st));
    const bool graph_loop = enqueue_loop(S, P, cfg, opts.loop == 1) < 0;
    EGG_CHECK(cudaEventRecord(S.ev[2], S.st));
    // final grid and labels of every instance (EGG_SynC.cu:1503-1522)
    for (Group& gr : P.groups) {
        const Exec ex = batched(gr.all, gr.d);
        launch_build(ex, S.st);
        launch_labels_uf(ex, S.st);
        launches += 3 * gr.all.max_passes + 6 + 4;
    }
    k_batch_results<<<(count + 255) / 256, 256, 0, S.st>>>(P.d_works, count, P.d_results);
    launches++;
    const size_t out_b = 4 * P.out_ints;
    if (out_b) EGG_CHECK(cudaMemcpyAsync(S.h_pinned, P.d_out, out_b, cudaMemcpyDeviceToHost, S.st));
    const size_t nloop = 2 + P.groups.size();
    std::vector<int> res(5 * (size_t)count + nloop);
    EGG_CHECK(cudaMemcpyAsync(res.data(), P.d_results, 4 * 5 * (size_t)count, cudaMemcpyDeviceToHost, S.st));
    EGG_CHECK(cudaMemcpyAsync(res.data() + 5 * (size_t)count, P.d_loop, 4 * nloop, cudaMemcpyDeviceToHost, S.st));
    EGG_CHECK(cudaEventRecord(S.ev[3], S.st));
    EGG_CHECK(cudaStreamSynchronize(S.st));
    EGG_CHECK(cudaGetLastError());

    int bad = 0;
    for (int pos = 0; pos < count; pos++) {
        const int i = P.order[pos];  // results are in listed order
        const int* r = res.data() + 5 * (size_t)pos;
        egg_batch_item& it = items[i];
        it.iterations = r[0];
        it.converged = r[1] != 0;
        it.n_clusters = r[2];
        if (r[3] & kErrNonFinite) {
            it.status = EGG_ERR_INPUT;
            it.iterations = 0;
            it.converged = 0;
            it.n_clusters = 0;
            continue;
        }
        bad |= r[3];
        it.status = it.converged ? EGG_OK : EGG_MAX_ITER;
        if (P.out_off[i] != SIZE_MAX)
            memcpy(it.labels, (const int*)S.h_pinned + P.out_off[i], 4 * (size_t)P.geoms[i].n);
    }
    const int loop_iters = res[5 * (size_t)count];
    if (stats) {
        const egg_batch_stats stats_in = *stats;
        memset(stats, 0, sizeof(*stats));
        stats->loop_iterations = loop_iters;
        stats->groups = (int)P.groups.size();
        long long ll = loop_launches(P, loop_iters, res);
        if (!graph_loop || (int)P.groups.size() > kMaxGroups) {
            // host-driven loop, or a graph without gates: every group launches in every iteration
            ll = loop_iters;
            for (const Group& gr : P.groups) ll += (long long)loop_iters * group_launches(gr);
        }
        stats->launches = (int32_t)std::min<long long>(0x7fffffff, launches + ll);
        stats->tuned = tuned_now ? 1 : 0;
        stats->update_threads = cfg.update_threads;
        stats->blocks_per_sm = cfg.occ;
        stats->order = cfg.order;
        stats->workspace_bytes = (int64_t)P.bytes;
        EGG_CHECK(cudaEventElapsedTime(&stats->total_ms, S.ev[0], S.ev[3]));
        EGG_CHECK(cudaEventElapsedTime(&stats->loop_ms, S.ev[1], S.ev[2]));
        stats->tune_ms = tune_ms;
        if (stats_in.itr_ms && stats_in.itr_cap > 0 && loop_iters > 0) {
            std::vector<unsigned long long> ls((size_t)loop_iters + 1);
            EGG_CHECK(cudaMemcpy(ls.data(), P.d_loop_stamps, 8 * ls.size(), cudaMemcpyDeviceToHost));
            const int m = std::min(loop_iters, stats_in.itr_cap);
            for (int k = 0; k < m; k++) stats_in.itr_ms[k] = (float)((ls[k + 1] - ls[k]) * 1e-6);
        }
        stats->itr_cap = stats_in.itr_cap;
        stats->itr_ms = stats_in.itr_ms;
    }
    if (bad & ~kErrNonFinite)
        throw ArgError{EGG_ERR_INTERNAL, "kernel consistency check failed (status bits " + std::to_string(bad) + ")"};
    return EGG_OK;
}

void release_batch() {
    for (auto& kv : g_states) {
        State* S = kv.second;
        int cur = 0;
        cudaGetDevice(&cur);
        cudaSetDevice(S->dev);
        drop_graphs(*S);
        if (S->base) cudaFree(S->base);
        if (S->h_pinned) cudaFreeHost(S->h_pinned);
        for (auto e : S->ev)
            if (e) cudaEventDestroy(e);
        if (S->fork) cudaEventDestroy(S->fork);
        for (auto e : S->gjoins) cudaEventDestroy(e);
        for (auto s : S->gstreams) cudaStreamDestroy(s);
        if (S->st) cudaStreamDestroy(S->st);
        cudaSetDevice(cur);
        delete S;
    }
    g_states.clear();
}

}  // namespace egg

extern "C" __attribute__((visibility("default"))) int egg_sync_batch(egg_batch_item* items, int32_t count,
                                                                     const egg_opts* opts, egg_batch_stats* stats,
                                                                     void* stream) {
    return egg::guarded([&] { return egg::run_batch(items, count, opts, stats, stream); });
}
