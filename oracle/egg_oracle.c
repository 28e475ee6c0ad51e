/*
 * egg_oracle.c -- CPU restatement of the EGG-SynC synchronisation-clustering loop.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the parity checker for the CUDA
 * path in egg-sync_b200/csrc.  Only tests/, __graft_entry__.smoke() and the
 * cpu_baseline leg of bench.py may load it, and only to check or time; the
 * product never links or calls it.
 *
 * It restates, in plain C (FP64 for the update arithmetic, FP32 with a fixed
 * operation order for every decision), the reference's algorithm:
 *
 *   geometry ........ src/algorithms/EGG_SynC.cu:1249-1260 (+ 1430 eps_extra)
 *   cell ids ......... src/algorithms/EGG_SynC.cu:63-76, 102-108
 *   border rule ...... src/algorithms/EGG_SynC.cu:583-597
 *   box distances .... src/algorithms/EGG_SynC.cu:613-636
 *   update ........... src/algorithms/EGG_SynC.cu:605-703 (full cells through
 *                      the cell aggregate, partial cells point by point; both
 *                      equal sum_{q in N_eps(p)} sin(x_q - x_p), which is
 *                      what this oracle evaluates, in double precision)
 *   half-count flag .. src/algorithms/EGG_SynC.cu:666-681, 706-709
 *   extra check ...... src/algorithms/EGG_SynC.cu:767-1034 (pairs), 1037-1159
 *                      (MBR_in_eps), 1162-1203 (part 2), host 1425-1489
 *   loop + labels .... src/algorithms/EGG_SynC.cu:1322-1522, 1205-1227
 *
 * Parity status: pinned.  The one-step update is checked against the
 * reference's own CPU SynC (src/algorithms/SynC.cpp:16-40, built from the
 * reference sources into oracle/_ref) and the full-run labels against the
 * reference EGG-SynC run on a B200 (fixtures under tests/golden/).
 *
 * Floating-point conventions shared with the CUDA kernels (both sides use the
 * same operation order so that every discrete decision is bit-identical):
 *   - cell id:        (int)(x / side), value == width -> width-1, then clamp
 *                     into [0, width-1] (the reference is undefined outside
 *                     [0,1]; inside it the clamp never fires)
 *   - box distance:   left = fmaf(g, side, -x), right = fmaf(g+1, side, -x),
 *                     each squared (rounded), the smaller/larger added per
 *                     dimension (the fused face offset is the convention the
 *                     reference's own B200 run reproduces, see g_face_fma)
 *   - point distance: acc = fmaf(diff, diff, acc) over l = 0..d-1
 *   - "sqrt(v) <= e": v <= T(e), T(e) the largest float whose sqrtf is <= e
 *                     (sqrtf is correctly rounded and monotone, so the two
 *                     tests are equivalent)
 * Compile with -ffp-contract=off so the compiler does not fuse anything else.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <float.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define ORACLE_API __attribute__((visibility("default")))

typedef struct {
    int n, d;
    float eps;
    float side;        /* inner (= outer) cell side          EGG_SynC.cu:1249,1254 */
    int width;         /* cells per dimension                EGG_SynC.cu:1250,1255 */
    int od;            /* outer grid dimensions              EGG_SynC.cu:1256 */
    int64_t n_outer;   /* width^od                           EGG_SynC.cu:1257 */
    int r;             /* ceil(eps/side), float              EGG_SynC.cu:1259,563 */
    float eps_extra;   /*                                    EGG_SynC.cu:1430 */
    int r_extra;       /* ceil(eps_extra/side), float        EGG_SynC.cu:779 */
    int r_half;        /* ceil((eps/2.)/side), double        EGG_SynC.cu:1045 */
    float t_eps, t_half, t_extra; /* squared-distance thresholds */
} egg_geom;

/* largest float t >= 0 with sqrtf(t) <= e */
static float sq_threshold(float e) {
    float t = e * e;
    while (t > 0.0f && sqrtf(t) > e) t = nextafterf(t, 0.0f);
    for (;;) {
        float u = nextafterf(t, INFINITY);
        if (sqrtf(u) <= e) t = u; else break;
    }
    return t;
}

ORACLE_API float egg_oracle_sq_threshold(float e) { return sq_threshold(e); }

/* Returns 0 on success, -1 when the geometry is degenerate (width < 2). */
ORACLE_API int egg_oracle_geometry(int n, int d, float eps, egg_geom *g) {
    memset(g, 0, sizeof(*g));
    g->n = n; g->d = d; g->eps = eps;
    /* float inner_cell_size = sqrt(pow((eps / 2.), 2.) / d); */
    g->side = (float)sqrt(pow(((double)eps / 2.), 2.) / (double)d);
    /* int inner_grid_width = 1 / inner_cell_size;  (float division) */
    g->width = (int)(1.0f / g->side);
    if (g->width < 2) return -1;
    /* int outer_grid_dims = min(d, (int) (log(n) / log(outer_grid_width))); */
    int od = (int)(log((double)n) / log((double)g->width));
    if (od > d) od = d;
    if (od < 0) od = 0;
    g->od = od;
    g->n_outer = (int64_t)pow((double)g->width, (double)od);
    g->r = (int)ceilf(eps / g->side);
    /* float eps_extra = 2 * eps - eps * sqrt(15. / 16.) + eps / 2. - sin(eps / 2.); */
    g->eps_extra = (float)((double)(2.0f * eps) - (double)eps * sqrt(15. / 16.) + (double)eps / 2. -
                           sin((double)eps / 2.));
    g->r_extra = (int)ceilf(g->eps_extra / g->side);
    g->r_half = (int)ceil(((double)eps / 2.) / (double)g->side);
    g->t_eps = sq_threshold(eps);
    g->t_half = sq_threshold(eps / 2.0f);
    g->t_extra = sq_threshold(g->eps_extra);
    return 0;
}

static inline int cell_dim(float x, const egg_geom *g) {
    int t = (int)(x / g->side);
    if (t == g->width) t--;
    if (t < 0) t = 0;
    if (t > g->width - 1) t = g->width - 1;
    return t;
}

/* reference border rule, EGG_SynC.cu:590-596 (the +-1e-5 probes are in double) */
static inline int on_border_dim(float x, float side) {
    int idm = (int)(((double)x - 0.00001) / (double)side);
    int id = (int)(x / side);
    int idp = (int)(((double)x + 0.00001) / (double)side);
    return (id != idm || id != idp);
}

static inline float pdist2(const float *a, const float *b, int d) {
    float acc = 0.0f;
    for (int l = 0; l < d; l++) {
        float diff = a[l] - b[l];
        acc = fmaf(diff, diff, acc);
    }
    return acc;
}

/* Box-distance mode.  0 (default) = the reference's formula; 1 = the true
 * minimum distance (a dimension in which x lies inside the cell's extent
 * contributes 0).  The reference's "small" distance (EGG_SynC.cu:622-631)
 * adds the nearer face's distance in every dimension, also when x lies
 * inside the cell's extent there, so it over-estimates and the reference
 * skips some cells that hold points within eps.  Mode 1 exists only to pin
 * the grid machinery against the reference's brute-force CPU SynC. */
static int g_box_mode = 0;

ORACLE_API void egg_oracle_set_box_mode(int exact) { g_box_mode = exact ? 1 : 0; }

/* Rounding convention of the box-distance face offsets: 0 = product rounded,
 * then the subtraction (g*side rounded, minus x); 1 = one fused multiply-add
 * fmaf(g, side, -x).  The two differ only when x sits (almost) exactly on a
 * cell face.  Only 1 reproduces the reference EGG-SynC run on a B200 for
 * points placed exactly on cell faces (tests/golden/ref_egg_borders.npz:
 * 20 iterations and the same partition; 0 gives 16 iterations), i.e. nvcc
 * contracts the reference's `g * side` followed by `-= x` into one FMA. */
static int g_face_fma = 1;

ORACLE_API void egg_oracle_set_face_fma(int on) { g_face_fma = on ? 1 : 0; }

/* reference box distance of point x to the cell with dim ids cd, EGG_SynC.cu:613-633.
 * In mode 1 the last cell of a dimension is also open-ended: the clamp
 * (value == width -> width-1, EGG_SynC.cu:69-71) puts points up to 1.0 in a
 * cell whose box ends at width*side. */
static inline void box_dist2(const float *x, const int *cd, int d, const egg_geom *g, float *small2, float *large2) {
    const float side = g->side;
    float s = 0.0f, L = 0.0f;
    for (int l = 0; l < d; l++) {
        float left, right;
        if (g_face_fma) {
            left = fmaf((float)cd[l], side, -x[l]);
            right = fmaf((float)(cd[l] + 1), side, -x[l]);
        } else {
            left = (float)cd[l] * side;
            right = (float)(cd[l] + 1) * side;
            left = left - x[l];
            right = right - x[l];
        }
        const int last = cd[l] == g->width - 1;
        const int inside = (left <= 0.0f && (right >= 0.0f || last));
        left = left * left;
        right = right * right;
        if (g_box_mode) {
            s = s + (inside ? 0.0f : (left < right || last ? left : right));
            L = last ? INFINITY : L + (left < right ? right : left);
            continue;
        }
        if (left < right) { s = s + left; L = L + right; }
        else { s = s + right; L = L + left; }
    }
    *small2 = s; *large2 = L;
}

/* ------------------------------------------------------------------------ */
/* grid: points sorted by (outer id, g_od, ..., g_{d-1}), stable in index    */
/* ------------------------------------------------------------------------ */
typedef struct {
    egg_geom g;
    int n, d;
    const float *X;      /* n*d row-major */
    int *gid;            /* n*d dim ids per point */
    int64_t *outer;      /* per point outer id */
    int *sub;            /* per point sub-cell key (order inside a cell) */
    int *order;          /* sorted position -> point */
    int *cell_of_pt;     /* point -> cell */
    int M;               /* number of non-empty cells */
    int *cell_start;     /* M+1 */
    int *cell_dims;      /* M*d */
    int64_t *cell_outer; /* M */
    int *outer_begin;    /* n_outer+1 */
} grid_t;

static const grid_t *g_sort_ctx;
static int cmp_points(const void *pa, const void *pb) {
    int a = *(const int *)pa, b = *(const int *)pb;
    const grid_t *G = g_sort_ctx;
    if (G->outer[a] != G->outer[b]) return G->outer[a] < G->outer[b] ? -1 : 1;
    for (int l = G->g.od; l < G->d; l++) {
        int ga = G->gid[(size_t)a * G->d + l], gb = G->gid[(size_t)b * G->d + l];
        if (ga != gb) return ga < gb ? -1 : 1;
    }
    if (G->sub[a] != G->sub[b]) return G->sub[a] < G->sub[b] ? -1 : 1;
    return a < b ? -1 : (a > b);
}

/* Order of the points inside a cell (the GPU path's choice, not the
 * reference's; it only changes summation order): a Morton interleave of the
 * top `bits` bits of the point's offset inside its cell in the first
 * min(d, 8) dimensions, bits = max(1, 8 / min(d, 8)). */
static int sub_key(const float *x, const int *gid, const egg_geom *g) {
    const int nd = g->d < 8 ? g->d : 8;
    const int b = 8 / nd > 1 ? 8 / nd : 1;
    const float scale = (float)(1 << b) / g->side;
    int t[8];
    for (int l = 0; l < nd; l++) {
        const float off = x[l] - (float)gid[l] * g->side;
        int v = (int)(off * scale);
        t[l] = v < 0 ? 0 : (v > (1 << b) - 1 ? (1 << b) - 1 : v);
    }
    int dig = 0;
    for (int k = b - 1; k >= 0; k--)
        for (int l = 0; l < nd; l++) dig = (dig << 1) | ((t[l] >> k) & 1);
    return dig;
}

static int grid_build(grid_t *G, const float *X, int n, int d, float eps) {
    memset(G, 0, sizeof(*G));
    if (egg_oracle_geometry(n, d, eps, &G->g) != 0) return -1;
    G->n = n; G->d = d; G->X = X;
    G->gid = (int *)malloc(sizeof(int) * (size_t)n * d);
    G->outer = (int64_t *)malloc(sizeof(int64_t) * (size_t)n);
    G->sub = (int *)malloc(sizeof(int) * (size_t)n);
    G->order = (int *)malloc(sizeof(int) * (size_t)n);
    G->cell_of_pt = (int *)malloc(sizeof(int) * (size_t)n);
    G->cell_start = (int *)malloc(sizeof(int) * ((size_t)n + 1));
    G->cell_dims = (int *)malloc(sizeof(int) * (size_t)n * d);
    G->cell_outer = (int64_t *)malloc(sizeof(int64_t) * (size_t)n);
    G->outer_begin = (int *)malloc(sizeof(int) * ((size_t)G->g.n_outer + 1));
    for (int p = 0; p < n; p++) {
        int64_t o = 0, mul = 1;
        for (int l = 0; l < d; l++) {
            int t = cell_dim(X[(size_t)p * d + l], &G->g);
            G->gid[(size_t)p * d + l] = t;
            if (l < G->g.od) { o += (int64_t)t * mul; mul *= G->g.width; }
        }
        G->outer[p] = o;
        G->sub[p] = sub_key(&X[(size_t)p * d], &G->gid[(size_t)p * d], &G->g);
        G->order[p] = p;
    }
    g_sort_ctx = G;
    qsort(G->order, (size_t)n, sizeof(int), cmp_points);
    int M = 0;
    for (int i = 0; i < n; i++) {
        int p = G->order[i];
        int head = (i == 0);
        if (!head) {
            int q = G->order[i - 1];
            for (int l = 0; l < d && !head; l++)
                if (G->gid[(size_t)p * d + l] != G->gid[(size_t)q * d + l]) head = 1;
        }
        if (head) {
            G->cell_start[M] = i;
            for (int l = 0; l < d; l++) G->cell_dims[(size_t)M * d + l] = G->gid[(size_t)p * d + l];
            G->cell_outer[M] = G->outer[p];
            M++;
        }
        G->cell_of_pt[p] = M - 1;
    }
    G->M = M;
    G->cell_start[M] = n;
    /* outer_begin[o] = first cell whose outer id >= o */
    int c = 0;
    for (int64_t o = 0; o <= G->g.n_outer; o++) {
        while (c < M && G->cell_outer[c] < o) c++;
        G->outer_begin[o] = c;
    }
    return 0;
}

static void grid_free(grid_t *G) {
    free(G->gid); free(G->outer); free(G->sub); free(G->order); free(G->cell_of_pt);
    free(G->cell_start); free(G->cell_dims); free(G->cell_outer); free(G->outer_begin);
}

/* Iterate over the outer cells of the box stencil [-rad, rad]^od around the
 * outer cell of point dims gp, calling body(cell range) for the inner cells
 * that can be within reach in dimension od (dim-od pruning by rad+1 keeps the
 * reference's visiting set: cells beyond it fail the box test in exact and in
 * rounded arithmetic alike). */
typedef void (*cell_visit_fn)(const grid_t *G, int c, void *ctx);

static void visit_stencil(const grid_t *G, const int *gp, int rad, cell_visit_fn fn, void *ctx) {
    const int od = G->g.od, d = G->d, W = G->g.width;
    int idx[64];
    for (int l = 0; l < od; l++) idx[l] = -rad;
    for (;;) {
        int ok = 1;
        int64_t o = 0, mul = 1;
        for (int l = 0; l < od; l++) {
            int v = gp[l] + idx[l];
            if (v < 0 || v >= W) { ok = 0; break; }
            o += (int64_t)v * mul; mul *= W;
        }
        if (ok) {
            int b = G->outer_begin[o], e = G->outer_begin[o + 1];
            if (od < d) {
                int lo = gp[od] - rad - 1, hi = gp[od] + rad + 1;
                while (b < e && G->cell_dims[(size_t)b * d + od] < lo) b++;
                while (e > b && G->cell_dims[(size_t)(e - 1) * d + od] > hi) e--;
            }
            for (int c = b; c < e; c++) fn(G, c, ctx);
        }
        if (od == 0) break;
        int l = 0;
        idx[0]++;
        while (l < od - 1 && idx[l] > rad) { idx[l] = -rad; l++; idx[l]++; }
        if (idx[od - 1] > rad) break;
    }
}

/* ---------------------------- one update step ---------------------------- */
typedef struct {
    const float *xp;
    int p_cell;
    int border;
    double sum[64];
    int count;        /* |N_eps(p)| */
    int half;         /* reference half_count */
    int partial_in;   /* neighbours found in partial cells */
    double rsum;      /* sum over N_eps(p) of exp(-|x_p - x_q|) (FP64) */
} step_ctx;

static inline double exp_neg_dist(const float *a, const float *b, int d) {
    double s = 0.0;
    for (int l = 0; l < d; l++) {
        double df = (double)a[l] - (double)b[l];
        s += df * df;
    }
    return exp(-sqrt(s));
}

static void step_visit(const grid_t *G, int c, void *vctx) {
    step_ctx *s = (step_ctx *)vctx;
    const int d = G->d;
    float sm2, lg2;
    box_dist2(s->xp, &G->cell_dims[(size_t)c * d], d, &G->g, &sm2, &lg2);
    int b = G->cell_start[c], e = G->cell_start[c + 1];
    if (lg2 <= G->g.t_eps) {
        /* fully included: every point of the cell is a neighbour */
        for (int i = b; i < e; i++) {
            const float *xq = &G->X[(size_t)G->order[i] * d];
            for (int l = 0; l < d; l++) s->sum[l] += sin((double)xq[l] - (double)s->xp[l]);
            s->rsum += exp_neg_dist(s->xp, xq, d);
        }
        s->count += e - b;
        if (s->border) {
            if (c == s->p_cell) s->half += e - b;
            else
                for (int i = b; i < e; i++)
                    if (pdist2(s->xp, &G->X[(size_t)G->order[i] * d], d) <= G->g.t_half) s->half++;
        }
    } else if (sm2 <= G->g.t_eps) {
        for (int i = b; i < e; i++) {
            const float *xq = &G->X[(size_t)G->order[i] * d];
            if (pdist2(s->xp, xq, d) <= G->g.t_eps) {
                for (int l = 0; l < d; l++) s->sum[l] += sin((double)xq[l] - (double)s->xp[l]);
                s->rsum += exp_neg_dist(s->xp, xq, d);
                s->count++;
                s->partial_in++;
            }
        }
    }
}

/* One EGG-SynC iteration on X (n*d row-major, original order).
 * Xnext   <- updated positions (original order), FP64 arithmetic rounded to float
 * counts  <- |N_eps(p)| per point (may be NULL)
 * returns the update kernel's convergence flag (1 = every point passed the
 *         reference neighbourhood test), or -1 on a geometry error. */
ORACLE_API int egg_oracle_step(const float *X, int n, int d, float eps, float *Xnext, int *counts, double *delta64) {
    grid_t G;
    if (d > 64 || grid_build(&G, X, n, d, eps) != 0) return -1;
    int flag = 1;
#pragma omp parallel for schedule(dynamic, 64) reduction(&& : flag)
    for (int p = 0; p < n; p++) {
        step_ctx s;
        memset(&s, 0, sizeof(s));
        s.xp = &X[(size_t)p * d];
        s.p_cell = G.cell_of_pt[p];
        for (int l = 0; l < d; l++) s.border |= on_border_dim(s.xp[l], G.g.side);
        visit_stencil(&G, &G.gid[(size_t)p * d], G.g.r, step_visit, &s);
        for (int l = 0; l < d; l++) {
            double dl = s.sum[l] / (double)s.count;
            if (delta64) delta64[(size_t)p * d + l] = dl;
            Xnext[(size_t)p * d + l] = (float)((double)s.xp[l] + dl);
        }
        if (counts) counts[p] = s.count;
        int own = G.cell_start[s.p_cell + 1] - G.cell_start[s.p_cell];
        if ((!s.border && s.count != own) || (s.border && s.count != s.half)) flag = 0;
    }
    grid_free(&G);
    return flag;
}

/* The same iteration for the sampled points idx[0..m) only (for inputs too
 * large for a full oracle step): Xs[m*d], counts[m] and the per-point
 * convergence verdict viol[m] (1 = this point clears the flag). */
ORACLE_API int egg_oracle_step_sample(const float *X, int n, int d, float eps, const int *idx, int m, float *Xs,
                                      int *counts, int *viol) {
    grid_t G;
    if (d > 64 || grid_build(&G, X, n, d, eps) != 0) return -1;
#pragma omp parallel for schedule(dynamic, 4)
    for (int k = 0; k < m; k++) {
        const int p = idx[k];
        step_ctx s;
        memset(&s, 0, sizeof(s));
        s.xp = &X[(size_t)p * d];
        s.p_cell = G.cell_of_pt[p];
        for (int l = 0; l < d; l++) s.border |= on_border_dim(s.xp[l], G.g.side);
        visit_stencil(&G, &G.gid[(size_t)p * d], G.g.r, step_visit, &s);
        for (int l = 0; l < d; l++) Xs[(size_t)k * d + l] = (float)((double)s.xp[l] + s.sum[l] / (double)s.count);
        if (counts) counts[k] = s.count;
        int own = G.cell_start[s.p_cell + 1] - G.cell_start[s.p_cell];
        if (viol) viol[k] = (!s.border && s.count != own) || (s.border && s.count != s.half);
    }
    grid_free(&G);
    return 0;
}

/* Local order parameter over the EGG-SynC neighbourhoods (the update's cells
 * and tests), exact in FP64: mean_p mean_{q in N(p)} exp(-|x_p - x_q|), the
 * quantity of SynC.cpp:42-56 on the neighbourhoods the loop actually uses. */
ORACLE_API double egg_oracle_order_parameter_egg(const float *X, int n, int d, float eps) {
    grid_t G;
    if (d > 64 || grid_build(&G, X, n, d, eps) != 0) return -1.0;
    double total = 0.0;
#pragma omp parallel for schedule(dynamic, 64) reduction(+ : total)
    for (int p = 0; p < n; p++) {
        step_ctx s;
        memset(&s, 0, sizeof(s));
        s.xp = &X[(size_t)p * d];
        s.p_cell = G.cell_of_pt[p];
        visit_stencil(&G, &G.gid[(size_t)p * d], G.g.r, step_visit, &s);
        total += s.rsum / (double)s.count;
    }
    grid_free(&G);
    return total / n;
}

/* ------------------------------ extra check ------------------------------ */
typedef struct {
    const float *xq;      /* ball centre */
    const float *xp;      /* the far point (p_mark) */
    float mbr[64];
} mbr_ctx;

static void mbr_visit(const grid_t *G, int c, void *vctx) {
    mbr_ctx *m = (mbr_ctx *)vctx;
    const int d = G->d;
    float sm2, lg2;
    box_dist2(m->xq, &G->cell_dims[(size_t)c * d], d, &G->g, &sm2, &lg2);
    if (!(sm2 <= G->g.t_half)) return;
    for (int i = G->cell_start[c]; i < G->cell_start[c + 1]; i++) {
        const float *xr = &G->X[(size_t)G->order[i] * d];
        if (pdist2(m->xq, xr, d) <= G->g.t_half) {
            for (int l = 0; l < d; l++) {
                float od_ = m->mbr[l] - m->xp[l];
                od_ = od_ * od_;
                float nd = xr[l] - m->xp[l];
                nd = nd * nd;
                if (nd < od_) m->mbr[l] = xr[l];
            }
        }
    }
}

/* MBR_in_eps, EGG_SynC.cu:1037-1159: is the per-dimension closest corner of
 * q's eps/2 group within eps of p? */
static int mbr_in_eps(const grid_t *G, int p, int q) {
    const int d = G->d;
    mbr_ctx m;
    m.xq = &G->X[(size_t)q * d];
    m.xp = &G->X[(size_t)p * d];
    for (int l = 0; l < d; l++) m.mbr[l] = m.xq[l];
    visit_stencil(G, &G->gid[(size_t)q * d], G->g.r_half, mbr_visit, &m);
    float acc = 0.0f;
    for (int l = 0; l < d; l++) {
        float diff = m.mbr[l] - m.xp[l];
        acc = fmaf(diff, diff, acc);
    }
    return acc <= G->g.t_eps;
}

typedef struct {
    int p;
    int violated;
    int64_t pairs;
} extra_ctx;

static void extra_visit(const grid_t *G, int c, void *vctx) {
    extra_ctx *x = (extra_ctx *)vctx;
    if (x->violated) return;
    const int d = G->d;
    const float *xp = &G->X[(size_t)x->p * d];
    float sm2, lg2;
    box_dist2(xp, &G->cell_dims[(size_t)c * d], d, &G->g, &sm2, &lg2);
    int included = sm2 <= G->g.t_extra;
    int fully = lg2 <= G->g.t_eps;
    if (!included || fully) return;
    for (int i = G->cell_start[c]; i < G->cell_start[c + 1] && !x->violated; i++) {
        int q = G->order[i];
        float d2 = pdist2(xp, &G->X[(size_t)q * d], d);
        if (d2 > G->g.t_eps && d2 <= G->g.t_extra) {
            x->pairs++;
            if (mbr_in_eps(G, x->p, q)) x->violated = 1;
        }
    }
}

/* Extra convergence check on X; returns 1 if still converged, 0 if some pair
 * (p, q) with eps < |p-q| <= eps_extra has q's eps/2 MBR within eps of p.
 * *pairs_out (optional) receives the number of annulus pairs examined before
 * the first violation (all of them when none). */
ORACLE_API int egg_oracle_extra_check(const float *X, int n, int d, float eps, int64_t *pairs_out) {
    grid_t G;
    if (d > 64 || grid_build(&G, X, n, d, eps) != 0) return -1;
    int ok = 1;
    int64_t pairs = 0;
#pragma omp parallel for schedule(dynamic, 64) reduction(&& : ok) reduction(+ : pairs)
    for (int p = 0; p < n; p++) {
        extra_ctx x = {p, 0, 0};
        visit_stencil(&G, &G.gid[(size_t)p * d], G.g.r_extra, extra_visit, &x);
        pairs += x.pairs;
        if (x.violated) ok = 0;
    }
    if (pairs_out) *pairs_out = pairs;
    grid_free(&G);
    return ok;
}

/* Number of (p, q) pairs the reference's extra check lists on X: the counter
 * of kernel_float_grid_extra_check_part1_count (EGG_SynC.cu:767-878), i.e.
 * for every p, over the cells of its eps_extra stencil that pass the small
 * box test against eps_extra and are not fully inside eps (EGG_SynC.cu:
 * 848-866), the points q with eps < |p - q| <= eps_extra (EGG_SynC.cu:
 * 870-878).  The reference sizes its pair list from this count with int
 * arithmetic (EGG_SynC.cu:878, 1010, 1449-1450), so it must stay below
 * 2^30 and below n*n mod 2^32 (the wrap limit of its atomicInc).
 * Cells are decided wholesale by the tight box of their points where that
 * box proves all or none of their points lie in the (eps, eps_extra]
 * annulus; only straddling cells are walked.  *max_per_point (optional)
 * receives the largest count of a single p. */
ORACLE_API int64_t egg_oracle_ref_annulus_pairs(const float *X, int n, int d, float eps, int64_t *max_per_point) {
    grid_t G;
    if (d > 64 || grid_build(&G, X, n, d, eps) != 0) return -1;
    float *lo = (float *)malloc(sizeof(float) * (size_t)G.M * d);
    float *hi = (float *)malloc(sizeof(float) * (size_t)G.M * d);
    for (int c = 0; c < G.M; c++) {
        for (int l = 0; l < d; l++) { lo[(size_t)c * d + l] = FLT_MAX; hi[(size_t)c * d + l] = -FLT_MAX; }
        for (int i = G.cell_start[c]; i < G.cell_start[c + 1]; i++) {
            const float *xq = &X[(size_t)G.order[i] * d];
            for (int l = 0; l < d; l++) {
                if (xq[l] < lo[(size_t)c * d + l]) lo[(size_t)c * d + l] = xq[l];
                if (xq[l] > hi[(size_t)c * d + l]) hi[(size_t)c * d + l] = xq[l];
            }
        }
    }
    int64_t total = 0, worst = 0;
    const egg_geom *g = &G.g;
#pragma omp parallel for schedule(dynamic, 256) reduction(+ : total) reduction(max : worst)
    for (int p = 0; p < n; p++) {
        const float *xp = &X[(size_t)p * d];
        const int *gp = &G.gid[(size_t)p * d];
        const int od = g->od, W = g->width, rad = g->r_extra;
        int idx[64];
        int64_t mine = 0;
        for (int l = 0; l < od; l++) idx[l] = -rad;
        for (;;) {
            int ok = 1;
            int64_t o = 0, mul = 1;
            for (int l = 0; l < od; l++) {
                int v = gp[l] + idx[l];
                if (v < 0 || v >= W) { ok = 0; break; }
                o += (int64_t)v * mul; mul *= W;
            }
            if (ok) {
                for (int c = G.outer_begin[o]; c < G.outer_begin[o + 1]; c++) {
                    float sm2, lg2;
                    box_dist2(xp, &G.cell_dims[(size_t)c * d], d, g, &sm2, &lg2);
                    if (!(sm2 <= g->t_extra) || lg2 <= g->t_eps) continue;
                    float n2 = 0.f, f2 = 0.f;
                    for (int l = 0; l < d; l++) {
                        const float L = lo[(size_t)c * d + l], H = hi[(size_t)c * d + l];
                        float a = xp[l] < L ? L - xp[l] : (xp[l] > H ? xp[l] - H : 0.0f);
                        float b1 = fabsf(L - xp[l]), b2 = fabsf(H - xp[l]);
                        float b = b1 > b2 ? b1 : b2;
                        n2 = fmaf(a, a, n2);
                        f2 = fmaf(b, b, f2);
                    }
                    if (n2 > g->t_extra || f2 <= g->t_eps) continue;
                    if (n2 > g->t_eps && f2 <= g->t_extra) {
                        mine += G.cell_start[c + 1] - G.cell_start[c];
                        continue;
                    }
                    for (int i = G.cell_start[c]; i < G.cell_start[c + 1]; i++) {
                        float d2 = pdist2(xp, &X[(size_t)G.order[i] * d], d);
                        mine += (d2 > g->t_eps && d2 <= g->t_extra);
                    }
                }
            }
            if (od == 0) break;
            int l = 0;
            idx[0]++;
            while (l < od - 1 && idx[l] > rad) { idx[l] = -rad; l++; idx[l]++; }
            if (idx[od - 1] > rad) break;
        }
        total += mine;
        if (mine > worst) worst = mine;
    }
    free(lo);
    free(hi);
    grid_free(&G);
    if (max_per_point) *max_per_point = worst;
    return total;
}

/* -------------------------------- labels -------------------------------- */
/* GPU_synCluster_float_grid, EGG_SynC.cu:1205-1227: label = compacted cell
 * index when the cell holds more than one point, else -1.  Cells are ranked
 * by (outer id, g_od, ..., g_{d-1}). */
ORACLE_API int egg_oracle_labels(const float *X, int n, int d, float eps, int *labels) {
    grid_t G;
    if (d > 64 || grid_build(&G, X, n, d, eps) != 0) return -1;
    for (int p = 0; p < n; p++) {
        int c = G.cell_of_pt[p];
        labels[p] = (G.cell_start[c + 1] - G.cell_start[c] > 1) ? c : -1;
    }
    grid_free(&G);
    return 0;
}

/* grid inspection: order[i] (sorted position -> point), cell_of[p], number of
 * cells, cell_start[0..M] (caller provides n+1 entries). */
ORACLE_API int egg_oracle_grid(const float *X, int n, int d, float eps, int *order, int *cell_of, int *cell_start,
                               int *M_out) {
    grid_t G;
    if (d > 64 || grid_build(&G, X, n, d, eps) != 0) return -1;
    memcpy(order, G.order, sizeof(int) * (size_t)n);
    memcpy(cell_of, G.cell_of_pt, sizeof(int) * (size_t)n);
    memcpy(cell_start, G.cell_start, sizeof(int) * ((size_t)G.M + 1));
    *M_out = G.M;
    grid_free(&G);
    return 0;
}

/* ------------------------------- full loop ------------------------------- */
/* EGG_SynC.cu:1322-1522.  Returns the number of iterations, or -1 on error.
 * X0 is not modified; Xfinal (optional) receives the final positions.
 * max_iter <= 0 means no cap (the reference has none). */
ORACLE_API int egg_oracle_run(const float *X0, int n, int d, float eps, int max_iter, int *labels, float *Xfinal,
                              int *flags_out) {
    size_t nd = (size_t)n * d;
    float *cur = (float *)malloc(sizeof(float) * nd);
    float *nxt = (float *)malloc(sizeof(float) * nd);
    memcpy(cur, X0, sizeof(float) * nd);
    int itr = 0, flag = 0;
    while (!flag) {
        itr++;
        flag = egg_oracle_step(cur, n, d, eps, nxt, NULL, NULL);
        if (flag < 0) { free(cur); free(nxt); return -1; }
        if (flag) flag = egg_oracle_extra_check(cur, n, d, eps, NULL);
        if (flags_out) flags_out[itr - 1] = flag;
        float *t = cur; cur = nxt; nxt = t;
        if (max_iter > 0 && itr >= max_iter) break;
    }
    if (labels) egg_oracle_labels(cur, n, d, eps, labels);
    if (Xfinal) memcpy(Xfinal, cur, sizeof(float) * nd);
    free(cur); free(nxt);
    return itr;
}

/* ---------------------- brute-force sampled update ----------------------- */
/* For large inputs: the FP64 update of the sampled points only, with the
 * neighbourhood found by testing every point (SynC.cpp:16-40 semantics with
 * the shared distance convention). */
ORACLE_API void egg_oracle_update_sample(const float *X, int n, int d, float eps, const int *idx, int m, float *out,
                                         int *counts) {
    float t = sq_threshold(eps);
#pragma omp parallel for schedule(dynamic, 4)
    for (int k = 0; k < m; k++) {
        const float *xp = &X[(size_t)idx[k] * d];
        double s[64] = {0};
        int c = 0;
        for (int j = 0; j < n; j++) {
            const float *xq = &X[(size_t)j * d];
            if (pdist2(xp, xq, d) <= t) {
                c++;
                for (int l = 0; l < d; l++) s[l] += sin((double)xq[l] - (double)xp[l]);
            }
        }
        for (int l = 0; l < d; l++) out[(size_t)k * d + l] = (float)((double)xp[l] + s[l] / (double)c);
        if (counts) counts[k] = c;
    }
}

/* Local order parameter r = mean_p mean_{q in N_eps(p)} exp(-|x_p - x_q|),
 * SynC.cpp:42-56, evaluated exactly in FP64 with brute-force neighbourhoods. */
ORACLE_API double egg_oracle_order_parameter(const float *X, int n, int d, float eps) {
    float t = sq_threshold(eps);
    double total = 0.0;
#pragma omp parallel for schedule(dynamic, 16) reduction(+ : total)
    for (int p = 0; p < n; p++) {
        const float *xp = &X[(size_t)p * d];
        double s = 0.0;
        int c = 0;
        for (int j = 0; j < n; j++) {
            const float *xq = &X[(size_t)j * d];
            if (pdist2(xp, xq, d) <= t) {
                double a = 0.0;
                for (int l = 0; l < d; l++) {
                    double df = (double)xp[l] - (double)xq[l];
                    a += df * df;
                }
                s += exp(-sqrt(a));
                c++;
            }
        }
        total += c ? s / c : 1.0;
    }
    return total / n;
}

ORACLE_API int egg_oracle_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}
