/*
 * eggsync.h -- C ABI of libeggsync.so, the B200 (sm_100a) implementation of
 * the EGG-SynC synchronisation-clustering loop.
 *
 * Every entry point takes plain pointers and sizes.  Point arrays are n x d
 * float32, row-major (point-major), values normalised to [0, 1] as the
 * reference expects.  Input and output pointers may be host or device
 * memory (detected per pointer).  Calls are synchronous: they return when
 * the outputs are written.  Calls from several host threads are serialised
 * inside the library.  No entry point exits the process; failures are
 * returned as negative egg_status values with a message in egg_last_error().
 */
#ifndef EGGSYNC_H
#define EGGSYNC_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define EGG_SYNC_ABI_VERSION 5

typedef enum egg_status {
    EGG_OK = 0,
    EGG_MAX_ITER = 1,        /* warning: stopped at opts->max_iter before convergence; labels are valid */
    EGG_ERR_ARG = -1,        /* bad argument (null pointer, n < 1, d out of range, eps not positive) */
    EGG_ERR_GEOMETRY = -2,   /* eps gives a grid the kernels do not support (width < 2 or > 65535) */
    EGG_ERR_INPUT = -3,      /* input holds NaN or Inf */
    EGG_ERR_CUDA = -4,       /* a CUDA call failed; see egg_last_error() */
    EGG_ERR_NO_DEVICE = -5,  /* no CUDA device */
    EGG_ERR_INTERNAL = -6    /* an internal consistency check failed */
} egg_status;

/* A trained warm-start network (see egg_mlp_train): 3 dense layers,
 * d_in -> hidden -> hidden -> d, ReLU after the two hidden layers.  It maps
 * a point's features (egg_mlp_features) to its displacement over the next
 * k_steps iterations of the plain loop, in units of eps.  Weights are
 * float32 row-major [in][out], host or device memory. */
typedef struct egg_mlp {
    int32_t d;        /* point dimension, 1..3 */
    int32_t d_in;     /* d + 3^d (1 + 2d): 192 for d = 3 */
    int32_t hidden;   /* 128 */
    int32_t k_steps;  /* iterations the network was trained to predict (informational) */
    int32_t min_count; /* only points with at least this many points in their 3^d coarse cells are
                          displaced; sparse points keep their input positions */
    int32_t reserved0;
    float *w1, *b1;   /* [d_in][hidden], [hidden] */
    float *w2, *b2;   /* [hidden][hidden], [hidden] */
    float *w3, *b3;   /* [hidden][d], [d] */
} egg_mlp;

typedef struct egg_mlp_train_opts {
    int32_t epochs;
    int32_t batch;    /* rows per Adam step, 16..65536 */
    float lr;         /* peak learning rate (cosine decay to 5% of it) */
    int32_t reserved0;
    int64_t seed;     /* shuffling seed */
} egg_mlp_train_opts;

typedef struct egg_opts {
    int32_t max_iter;     /* iteration cap; 0 = default (1000).  The reference has none. */
    int32_t loop;         /* 0 = device-resident loop (one CUDA graph, conditional while node),
                             1 = host-driven loop (one 4-byte readback per iteration) */
    int32_t stop_rule;    /* 0 = the reference's convergence flag (EGG_SynC.cu:1322),
                             1 = local order parameter >= lam (SynC.cpp:277-303 semantics) */
    int32_t order_param;  /* FP64 local order parameter r = mean_p mean_{q in N(p)} exp(-|p-q|)
                             (SynC.cpp:42-56) over the update's neighbourhoods, as certified bounds:
                             0 = off, 1 = of the final positions, 2 = every iteration */
    int32_t profile;      /* 1 = time every kernel group with CUDA events (host-driven loop) */
    int32_t full_update;  /* 1 = recompute every point in every iteration.  By default a point whose
                             whole stencil region held no moved point since the last update keeps
                             its previous result, which is bit-identical to recomputing it. */
    float *positions_out; /* optional n x d buffer (host or device): final positions, input order */
    int32_t labels_mode;  /* 0 = GPU union-find over the points of each final cell (default),
                             1 = direct per-cell labelling; both give identical labels */
    int32_t batch_tune;   /* egg_sync_batch only: 0 = autotune the launch configuration once per
                             workload signature (cached for later calls), 1 = default configuration,
                             2 = tune again */
    const egg_mlp *warm_start;  /* optional (egg_sync_run, d <= 3): displace the input by the network's
                                   prediction, then run the plain loop from there to convergence */
    int32_t warm_verify;  /* with warm_start: also run the plain loop from the input and return its
                             result (stats->warm_fallback = 1) when the two partitions differ */
    int32_t reserved[3];
} egg_opts;

typedef struct egg_stats {
    int32_t iterations;    /* loop iterations run (the reference's #itr) */
    int32_t converged;     /* 1 when the stop rule ended the loop */
    int32_t n_cells;       /* non-empty inner cells of the final grid */
    int32_t n_clusters;    /* final cells holding more than one point */
    int32_t extra_checks;  /* iterations that ran the extra convergence check */
    int32_t status_bits;   /* kernel-side warning bits (0 normally) */
    int64_t workspace_bytes;
    double order_param;    /* final local order parameter (FP64) when requested, else -1 */
    float stage_ms[6];     /* the reference's stage slots (run_experiment.py:20): allocating,
                              build structure, update, extra check, clustering, copy-out */
    float total_ms;
    float *itr_ms;         /* optional caller array of itr_cap entries: device time per iteration */
    int32_t itr_cap;
    float kernel_ms[4];    /* with opts->profile: summed CUDA-event time of the grid build, cell
                              sums, update and extra-check kernel groups */
    int32_t kernel_launches[4];  /* launches of each group's main kernel */
    int32_t launches;      /* kernels the call launched (all groups, loop control included) */
    double order_param_lo; /* certified FP64 bounds of the local order parameter (final value with
                              opts->order_param == 1, last iteration's with 2 or stop_rule 1), else -1 */
    double order_param_hi;
    double *itr_order_param; /* optional caller array of 2*itr_cap doubles: [lo, hi] per iteration
                                (opts->order_param == 2 or stop_rule == 1) */
    int32_t warm_started;  /* 1 when the returned result started from the network's positions */
    int32_t warm_fallback; /* 1 when warm_verify found a different partition and returned the plain run */
    float warm_ms;         /* device time of the warm start (features + network + displacement) */
    int32_t warm_same;     /* warm_verify: 1 when the two partitions were identical */
    int32_t grid_builds;   /* grid builds performed (iterations where some point changed cell, the
                              first and the final build included) */
    int64_t points_updated; /* point updates computed; the rest reused their previous result */
} egg_stats;

/* Fill *opts with the defaults (all zero). */
void egg_opts_default(egg_opts *opts);

/* Cluster n points of dimension d with radius eps.
 * Replaces EGG_SynC(float *h_D, int n, int d, float eps)
 * (src/algorithms/EGG_SynC.cuh:11, EGG_SynC.cu:1229-1601), reached from
 * EGG_SynC_wrapper(at::Tensor &D, float eps) (src/maps/map.cpp:31-33).
 * lam is the order-parameter threshold; it is only used with
 * opts->stop_rule == 1 (the reference ignores it, EGG_SynC.cu:1233).
 * labels[n] receives the compacted final cell index of every point whose
 * final cell holds more than one point, else -1 (EGG_SynC.cu:1205-1227).
 * opts and stats may be NULL.  stream: a cudaStream_t the call orders
 * itself after (NULL = legacy default stream). */
int egg_sync_run(const float *x, int64_t n, int32_t d, float eps, float lam, const egg_opts *opts,
                 int32_t *labels, egg_stats *stats, void *stream);

/* One iteration of the loop from the given positions (inspection and
 * parity testing).  Mirrors one pass of the while body at
 * src/algorithms/EGG_SynC.cu:1322-1495: x_next[n*d] receives the updated
 * positions (original point order), counts[n] (may be NULL) |N_eps(p)|,
 * flags[0] the update kernel's convergence flag (EGG_SynC.cu:706-709) and
 * flags[1] the flag after the extra check (EGG_SynC.cu:1425-1489). */
int egg_sync_step(const float *x, int64_t n, int32_t d, float eps, float *x_next, int32_t *counts,
                  int32_t *flags, void *stream);

/* The double grid built from x (inspection and parity testing).  Replaces
 * build_the_grid (src/algorithms/EGG_SynC.cu:248-341): order[i] = original
 * index of the i-th cell-sorted point, cell_of[i] = its cell, cell_start
 * (n+1 entries) = first sorted position of each cell plus the end,
 * *n_cells = number of non-empty cells. */
int egg_sync_grid(const float *x, int64_t n, int32_t d, float eps, int32_t *order, int32_t *cell_of,
                  int32_t *cell_start, int32_t *n_cells, void *stream);

/* The grid build of egg_sync_grid, for callers that must not allocate device
 * memory.  No counterpart in the reference.  Callers whose device memory is
 * owned by their own pool (a framework that has reserved the device, where
 * cudaMalloc fails or escapes its accounting) or that cannot afford the
 * device synchronisation cudaMalloc/cudaFree imply can use this entry point:
 * it calls no cudaMalloc, cudaFree or allocating library routine.  All of its
 * scratch lives in one file-scope device array of 8 MiB that every GPU which
 * loads the library holds until the process exits; inputs and outputs are
 * still the caller's (host or device pointers).
 * Limits: 1 <= n <= 65536 and 1 <= d <= 4; larger inputs return EGG_ERR_ARG.
 * The first call on a device looks up the array's device address
 * (cudaGetSymbolAddress) with that device current; make that first call
 * before any stream capture.  egg_release() forgets the address, so the
 * first call after it looks it up again: call egg_release() before a device
 * reset (cudaDeviceReset), after which the array may sit elsewhere.  Input
 * holding NaN or Inf returns EGG_ERR_INPUT before the build runs.  Every
 * call reuses the same array and finds the
 * previous call's contents in it (the call clears what must start at zero);
 * two calls overlapping on the GPU would race on it.  Calls through this
 * library are serialised and each one has finished on the GPU before it
 * returns.  stream: the cudaStream_t the work runs on (NULL = legacy default
 * stream).  Outputs as for egg_sync_grid. */
int egg_sync_grid_noalloc(const float *x, int64_t n, int32_t d, float eps, int32_t *order, int32_t *cell_of,
                          int32_t *cell_start, int32_t *n_cells, void *stream);

/* One instance of a batched run (egg_sync_batch). */
typedef struct egg_batch_item {
    const float *x;       /* n x d float32, row-major, host or device */
    int64_t n;
    int32_t d;
    float eps;
    int32_t *labels;      /* n int32 (host or device), as egg_sync_run's labels */
    int32_t iterations;   /* out: loop iterations of this instance */
    int32_t converged;    /* out: 1 when the reference's flag ended its loop */
    int32_t n_clusters;   /* out: final cells holding more than one point */
    int32_t status;       /* out: EGG_OK, EGG_MAX_ITER, or EGG_ERR_INPUT (NaN/Inf in x, labels not written) */
} egg_batch_item;

typedef struct egg_batch_stats {
    int32_t loop_iterations;  /* iterations of the batch loop (the largest instance's count) */
    int32_t groups;           /* instance groups: one per dimension d present */
    int32_t launches;         /* kernels the call launched, graph replays included */
    int32_t tuned;            /* 1 when this call ran the autotuner */
    int32_t update_threads;   /* configuration used: update kernel block size */
    int32_t blocks_per_sm;    /* persistent blocks per SM of a 256-thread kernel */
    int32_t order;            /* 0 = input order, 1 = instances by decreasing size */
    int32_t reserved0;
    int64_t workspace_bytes;
    float total_ms;           /* device time of the call (CUDA events), tuning excluded */
    float loop_ms;            /* device time of the batch loop */
    float tune_ms;            /* host time spent autotuning (0 when cached or off) */
    int32_t itr_cap;          /* entries of itr_ms */
    float *itr_ms;            /* optional caller array: device time of each batch-loop iteration */
    int32_t reserved[2];
} egg_batch_stats;

/* Run EGG-SynC on many independent instances at once: datasets of uneven
 * size and dimension, eps sweeps.  No counterpart in the reference, whose
 * wrapper runs one instance per call (src/maps/map.cpp:31-33).  Every
 * instance gets exactly the labels and iteration count that egg_sync_run
 * gives it alone.  All instances iterate inside one CUDA graph (one
 * conditional while loop, one persistent launch per kernel for all
 * instances of a dimension); finished instances drop out of the launches.
 * opts: max_iter, full_update and batch_tune are used; stop_rule and
 * order_param must be 0.  1 <= count <= 1024.  stats may be NULL.
 * Returns EGG_OK when every instance was processed (see each item's status),
 * else an error for the whole call. */
int egg_sync_batch(egg_batch_item *items, int32_t count, const egg_opts *opts, egg_batch_stats *stats,
                   void *stream);

/* Brute-force SynC on the GPU, the second drop-in.  Replaces
 * GPU_DynamicalClustering (src/algorithms/simple_GPU_SynC.cu:29-238), reached
 * from GPU_DynamicalClustering_wrapper (src/maps/map.cpp:27-29).  Every
 * iteration updates each point from all points within eps (itself included);
 * the loop stops when the mean local order parameter reaches lam, or after
 * max_iter iterations (0 = the reference's 100).  labels[n] receives, for a
 * point whose final eps-ball holds more than one point, the rank of the
 * smallest index in that ball, else -1.  positions_out (optional, n x d,
 * host or device) receives the final positions.  stats (optional) receives
 * the iteration count, converged, the number of labels, the final order
 * parameter (order_param) and the per-iteration times (itr_ms). */
int egg_simple_sync_run(const float *x, int64_t n, int32_t d, float eps, float lam, int32_t max_iter,
                        int32_t *labels, float *positions_out, egg_stats *stats, void *stream);

/* Per-dimension min-max normalisation of n x d float32 points on the GPU:
 * out = (x - min) / (max - min), evaluated in float32 as python/data.py:100-103
 * computes it on the host (0 where max == min; the reference divides by zero
 * there).  x and out may be host or device memory and may be the same
 * buffer.  lo and hi (optional host arrays of d floats) receive the minima
 * and maxima.  NaN or Inf in x returns EGG_ERR_INPUT. */
int egg_minmax_normalize(const float *x, int64_t n, int32_t d, float *out, float *lo, float *hi, void *stream);

/* Learned warm start (no counterpart in the reference).  Width of one
 * feature row: feat_dim(d) = d + 3^d (1 + 2d) rounded up to a multiple of
 * 16 (192 for d = 3); -1 for d outside 1..3. */
int egg_mlp_feature_dim(int32_t d);

/* Features of n points x (row-major n x d, host or device): feats receives
 * n rows of egg_mlp_feature_dim(d) float32 values (zero padded).  A coarse
 * grid of side eps; per point its offset in its coarse cell and, for each of
 * the 3^d cells around it, log1p(count)/8, centroid minus point and the
 * spread of the offsets (eps units). */
int egg_mlp_features(const float *x, int64_t n, int32_t d, float eps, float *feats);

/* The network on n feature rows (BF16 tensor-core inference, FP32
 * accumulation): out receives n x d displacements in eps units. */
int egg_mlp_forward(const egg_mlp *m, const float *feats, int64_t n, float *out);

/* Mean squared error of the network on n rows (FP32) and its gradient:
 * grad's weight arrays (float32, caller-owned) receive d loss / d weight. */
int egg_mlp_grad(const egg_mlp *m, const float *feats, const float *targets, int64_t n, egg_mlp *grad,
                 double *loss);

/* Train m in place (FP32, Adam, minibatches of opts->batch rows, shuffled
 * with opts->seed) on n rows of features and target displacements (n x d,
 * eps units).  epoch_loss (optional, opts->epochs entries) receives each
 * epoch's mean squared error. */
int egg_mlp_train(egg_mlp *m, const float *feats, const float *targets, int64_t n,
                  const egg_mlp_train_opts *opts, double *epoch_loss);

/* Human-readable name of a status value. */
const char *egg_status_str(int status);

/* Message of the last failure on the calling thread ("" if none). */
const char *egg_last_error(void);

/* Free the cached device workspaces and graphs of every device. */
int egg_release(void);

/* EGG_SYNC_ABI_VERSION of the loaded library. */
int egg_abi_version(void);

/* Testing aid for the error paths; no counterpart in the reference, whose
 * failed allocations exit the process (gpuAssert, EGG_SynC.cu:20-26).  The
 * next `count` device allocations made by any entry point fail as cudaMalloc
 * does on an exhausted device, without allocating: the call returns
 * EGG_ERR_CUDA ("out of memory" in egg_last_error()), holds no device memory
 * from the failed attempt, and the next call allocates again.  Workspaces
 * are cached, so a call that needs no new workspace allocates nothing (call
 * egg_release() first to force one).  count 0 clears it; count < 0 is
 * EGG_ERR_ARG. */
int egg_inject_alloc_failures(int32_t count);

/* Interaction counters of the update kernel summed over the last
 * egg_sync_run: point updates computed, candidate cells examined, cells
 * passing the reference's small box test, cells aggregated as fully covered,
 * cells aggregated / skipped by their points' tight box, 32-point groups
 * aggregated / skipped, point-pair distance tests, pairs within eps, warps
 * that walked the stencil lane by lane, half-count evaluations, sum of
 * |N(p)|, SM cycles of the candidate walk in warps whose lanes share one
 * outer cell and in warps that walked lane by lane (in this order; 16
 * slots).  Only the stats build
 * (libeggsync_stats.so) collects them; it writes min(cap, 16) values and
 * returns 16.  The normal build returns 0.  No counterpart in the reference. */
int egg_update_counters(int64_t *out, int32_t cap);

/* ---- eps search by minimum description length ------------------------- */

/* Mean distance of the points to their k-th and (k+1)-th nearest other
 * point, out[0] and out[1] (FP64 means of FP32 distances).  Replaces
 * NN(k, D) (python/SynCTorch.py:112-137), which the reference calls for k
 * and k+1.  1 <= k <= 31, n >= k + 2; x n x d float32 row-major, host or
 * device.  Brute force on the GPU, O(n^2 d). */
int egg_knn_mean(const float *x, int64_t n, int32_t d, int32_t k, double *out, void *stream);

/* Coding cost of a clustering, L_Clust_Outl(D, M)
 * (python/SynCTorch.py:265-314): clusters are the points sharing a label
 * >= 0, label -1 marks an outlier (the labels egg_sync_run returns).  With
 * h_l = 0.9 n^(-1/(d+4)) min(var_l, IQR_l / 1.34) (var the unbiased
 * variance of dimension l, IQR its 75th minus 25th percentile) and f(x) the
 * Gaussian product-kernel density of x among its own cluster's points:
 *   cost = sum_C (|C| log2(n/|C|) + d/2 log2|C|) + outliers log2 n
 *          - sum_C sum_{x in C} log2(f(x) / sum_{y in C} f(y))
 *          - outliers (2 pi)^(-1/2) prod_l h_l.
 * Writes *cost and (optional) *clusters.  x and labels host or device. */
int egg_mdl_cost(const float *x, int64_t n, int32_t d, const int32_t *labels, double *cost, int32_t *clusters,
                 void *stream);

typedef struct egg_mdl_stats {
    double eps0;          /* NN(k) */
    double eps1;          /* NN(k+1) */
    float eps_step;       /* float32 NN(k+1) - NN(k): the eps schedule's step */
    float eps_best;       /* eps of the returned clustering */
    int32_t candidates;   /* eps values clustered and costed */
    int32_t best;         /* index of the returned candidate */
    int32_t n_clusters;   /* clusters of the returned clustering */
    int32_t end_reason;   /* 0: a clustering had one cluster (the reference's stop), 1: candidate cap,
                             2: the next eps is beyond what the grid takes */
    double cost_best;     /* its coding cost */
    float total_ms;       /* device time of the call */
    int32_t cap;          /* in: entries of the optional arrays below */
    double *costs;        /* optional [cap]: cost of every candidate, in order */
    float *eps;           /* optional [cap]: eps of every candidate */
    int32_t *clusters;    /* optional [cap]: clusters of every candidate */
} egg_mdl_stats;

/* The full-SynC eps search, Sync(D, k) (python/SynCTorch.py:349-372):
 * eps starts at NN(k) and grows by NN(k+1) - NN(k) (float32 arithmetic);
 * every eps is clustered with the EGG-SynC loop (eight candidates per
 * batched call, each identical to egg_sync_run with default options) and
 * costed with egg_mdl_cost; the search stops after the first clustering
 * with a single cluster (or max_candidates, 0 = 256) and writes the labels
 * of the clustering of least cost (the first on ties).  The reference
 * clusters with its Python SynC instead (DynamicalClustering, allclose
 * grouping); stats optional. */
int egg_mdl_search(const float *x, int64_t n, int32_t d, int32_t k, int32_t max_candidates, int32_t *labels,
                   egg_mdl_stats *stats, void *stream);

#ifdef __cplusplus
}
#endif

#endif /* EGGSYNC_H */
