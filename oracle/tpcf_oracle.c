/*
 * TEST INFRASTRUCTURE ONLY — CPU restatement of the reference's grid-binned
 * pair-counting algorithm (lstothert/two_pcf), written from its source as the
 * parity checker for the CUDA path.  Only tests/, __graft_entry__.smoke() and
 * the cpu_baseline leg of bench.py load it; the product never does.
 *
 * It restates, with the same float/double operation sequence:
 *   - Axis (src/hist.cpp:15-62): bin parameters and bin_num;
 *   - JKHists::add_pair / JKHists2D::add_pair (src/hist.cpp:246-260, :484-502);
 *   - the 3-D pair loops for monopole, sigma-pi and s-mu
 *     (src/correlators.cpp:11-125, :156-278, :309-430) and their inverse-p
 *     variants (src/correlators_invpweight.cpp:14-709);
 *   - the angular loops (src/correlators_invpweight.cpp:713-982);
 *   - invert_jk_hists / multiply_hists (src/hist.cpp:270-288, :464-482);
 *   - JKHists::interp (src/hist.cpp:369-391);
 *   - the d_comov < 0 partition loop (src/boxes.cpp:15-26).
 * The spatial index is its own uniform grid: any decomposition that visits
 * every pair within the maximum separation gives the same counts (a pair with
 * float s^2 < max^2 has every |dx_m| below max).  Histogram sums are
 * accumulated in double in a different order from the reference's OpenMP
 * reduction, so weighted sums agree to rounding and unit-weight counts agree
 * exactly.
 *
 * Build: gcc -O3 -fopenmp -ffp-contract=off -fPIC -shared tpcf_oracle.c -lm
 * (oracle/build_oracle.sh).  -ffp-contract=off is required: the reference's
 * arithmetic is singly rounded x86-64 SSE code.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

typedef struct {
    int n_bins;
    int log_binning;
    float min, minus_min, max, step, inv_step, base, inv_log_of_base, inv_log_step;
} orc_axis;

typedef struct {
    int n;
    const double *xyz;      /* n x 3 */
    const double *unit;     /* n x 3 (x_norm) */
    const double *dcom;     /* n or NULL (then all >= 0) */
    const float *w;         /* n or NULL (1.0) — Galaxy::weight */
    const float *iw;        /* n or NULL (w) — Galaxy::input_weight (inverse-p build) */
    const int *jk;          /* n or NULL (0) */
    const long long *masks; /* n x n_mask or NULL (all bits set) */
    int n_mask;
    const long long *dmasks; /* n x n_mask dither masks (Galaxy::dither_mask) or NULL */
} orc_cat;

/* Build variants of the reference, selected at run time here:
 *   los_midpoint — pi without _ANGULAR_PI_DEFN (src/correlators.cpp:172-182);
 *   dither       — _USE_DITHER_WEIGHTS: the popcount of the two dither masks
 *                  replaces n_bitwise_runs in the inverse-p DD weights
 *                  (src/correlators_invpweight.cpp:62-71, :749-757). */
static int g_los_midpoint = 0, g_dither = 0;

void orc_set_variant(int los_midpoint, int dither) {
    g_los_midpoint = los_midpoint;
    g_dither = dither;
}

/* Angular up-weight table for JKHists::interp: the ratio histogram's full
 * bins, its axis, and the bin centres the reference computes with exp(). */
typedef struct {
    orc_axis ax;
    const double *bins;
    const double *centre;
} orc_upweight;

enum { ORC_MONOPOLE = 0, ORC_SIGMA_PI = 1, ORC_S_MU = 2 };
enum { ORC_W_PLAIN = 0, ORC_W_INVP_DD = 1, ORC_W_INVP_DR = 2 };

/* Axis::Axis (src/hist.cpp:15-36).  The parameters are the Params doubles,
 * narrowed to float at the constructor call; log(float) resolves to logf and
 * pow(float, int) to pow(double, double) under C++11 overloading. */
void orc_axis_init(orc_axis *ax, double input_min, double input_max, int n_bins, double log_base) {
    float fmin = (float)input_min, fmax = (float)input_max, fbase = (float)log_base;
    ax->min = fmin;
    ax->minus_min = -fmin;
    ax->max = fmax;
    ax->n_bins = n_bins;
    ax->step = (fmax - fmin) / (float)n_bins;
    ax->inv_step = (float)(1.0 / (double)ax->step);
    ax->base = fbase;
    if ((double)ax->base > 1.02) {
        ax->inv_log_of_base = (float)(1.0 / (double)logf(fbase));
        ax->inv_log_step = (float)((pow((double)fbase, (double)n_bins) - 1) / (double)(fmax - fmin));
        ax->log_binning = 1;
    } else {
        ax->inv_log_of_base = 0.0f;
        ax->inv_log_step = 0.0f;
        ax->log_binning = 0;
    }
}

/* Axis::bin_num (src/hist.cpp:46-53). */
float orc_axis_bin_num(const orc_axis *ax, float value) {
    if (ax->log_binning) return ax->inv_log_of_base * log1pf(ax->inv_log_step * (value - ax->min));
    return (value + ax->minus_min) * ax->inv_step;
}

/* float -> int as x86-64 cvttss2si does it: truncation, and INT_MIN for NaN
 * or out-of-range values (which the range checks then reject). */
int orc_to_int(float f) {
    if (!(f > -2147483648.0f && f < 2147483648.0f)) return INT32_MIN;
    return (int)f;
}

/* Axis::value_from_bin / bin_centre (src/hist.cpp:38-40, :55-62). */
double orc_axis_value_from_bin(const orc_axis *ax, double b) {
    if (ax->log_binning) return (exp(b / ax->inv_log_of_base) - 1.0) / ax->inv_log_step + ax->min;
    return ax->min + b * ax->step;
}

double orc_axis_bin_centre(const orc_axis *ax, int b) {
    return (orc_axis_value_from_bin(ax, b + 1.0) + orc_axis_value_from_bin(ax, b)) / 2.0;
}

/* JKHists::interp (src/hist.cpp:369-391). */
double orc_interp(const orc_upweight *up, double value) {
    const orc_axis *ax = &up->ax;
    int n = ax->n_bins;
    if (value < ax->min) return up->bins[0];
    if (value > ax->max) return up->bins[n - 1];
    float bn = (float)((double)orc_axis_bin_num(ax, (float)value) - 0.5);
    if (bn < 0) return up->bins[0];
    if (bn > n - 1) return up->bins[n - 1];
    int b = (int)bn;
    /* b == n - 1 would read bins[n] in the reference (undefined); callers keep
     * the table one entry longer so the read stays in bounds. */
    return up->bins[b] + (up->bins[b + 1] - up->bins[b]) * (value - up->centre[b]) / (up->centre[b + 1] - up->centre[b]);
}

/* The d_comov < 0 partition loop of GalaxyBoxes / GalaxyPixels
 * (src/boxes.cpp:15-26, :222-234), applied to an index permutation.  Returns
 * how many points the reference keeps; perm[0..ret) are their indices. */
int orc_partition(const double *dcom, int n, int *perm) {
    for (int i = 0; i < n; ++i) perm[i] = i;
    if (!dcom) return n;
    int n_gals = 0;
    for (int ii = 0; ii < n - ii + n_gals; ++ii) {
        if (dcom[perm[n_gals]] < 0.0) {
            int b = perm[n_gals];
            perm[n_gals] = perm[n - 1 - ii + n_gals];
            perm[n - 1 - ii + n_gals] = b;
        } else {
            ++n_gals;
        }
    }
    return n_gals;
}

/* ---------------------------------------------------------------- grid --- */

typedef struct {
    double lo[3], side;
    int dim[3];
    int *start; /* ncell + 1 */
    int *idx;   /* sorted point indices (into the kept subset's perm) */
} orc_grid;

static void grid_build(orc_grid *g, const double *pts, const int *perm, int n, const double lo[3],
                       const double hi[3], double side) {
    g->side = side;
    for (int m = 0; m < 3; ++m) {
        g->lo[m] = lo[m];
        g->dim[m] = (int)((hi[m] - lo[m]) / side) + 1;
        if (g->dim[m] < 1) g->dim[m] = 1;
    }
    long long nc = (long long)g->dim[0] * g->dim[1] * g->dim[2];
    g->start = (int *)calloc((size_t)nc + 1, sizeof(int));
    g->idx = (int *)malloc(sizeof(int) * (size_t)(n > 0 ? n : 1));
    int *cid = (int *)malloc(sizeof(int) * (size_t)(n > 0 ? n : 1));
    for (int i = 0; i < n; ++i) {
        const double *p = pts + 3 * (size_t)perm[i];
        int c[3];
        for (int m = 0; m < 3; ++m) {
            c[m] = (int)floor((p[m] - lo[m]) / side);
            if (c[m] < 0) c[m] = 0;
            if (c[m] >= g->dim[m]) c[m] = g->dim[m] - 1;
        }
        cid[i] = (c[0] * g->dim[1] + c[1]) * g->dim[2] + c[2];
        g->start[cid[i] + 1]++;
    }
    for (long long c = 0; c < nc; ++c) g->start[c + 1] += g->start[c];
    int *fill = (int *)calloc((size_t)nc, sizeof(int));
    for (int i = 0; i < n; ++i) g->idx[g->start[cid[i]] + fill[cid[i]]++] = perm[i];
    free(fill);
    free(cid);
}

static void grid_free(orc_grid *g) {
    free(g->start);
    free(g->idx);
}

/* ------------------------------------------------------- pair kernels --- */

typedef struct {
    int mode;
    orc_axis ax1, ax2;
    float min_r_sq, max_r_sq;
    int nb, n_jk;
    int weight_kind;
    const orc_upweight *up;
    int n_runs;
} orc_setup;

/* Per-thread accumulators of a pair loop: histograms (full[nb], sub[n_jk*nb])
 * for counts; per-object gradients ga[n_a], gb[n_b] and the per-bin
 * derivative G[nb] for the adjoint. */
typedef struct {
    double *full, *sub;
    double *ga, *gb;
    const double *G;
} orc_acc;

static inline void add_pair(const orc_setup *s, double *full, double *sub, int jk1, int jk2, int b, float w) {
    full[b] += w;
    sub[(size_t)jk1 * s->nb + b] += w;
    if (jk1 != jk2) sub[(size_t)jk2 * s->nb + b] += w;
}

static inline float popc_weight(const long long *m1, const long long *m2, int n_mask) {
    /* src/correlators_invpweight.cpp:56-60: float accumulation of popcounts,
     * then +1 when no bit is shared. */
    float weight = 0.0f;
    for (int k = 0; k < n_mask; ++k) weight += (float)__builtin_popcountll((unsigned long long)(m1[k] & m2[k]));
    if (weight < 0.5) weight += 1.0f;
    return weight;
}

static inline double one_minus_cos(const double *n1, const double *n2) {
    /* src/correlators_invpweight.cpp:51-54 */
    double v = 1.0;
    for (int m = 0; m < 3; ++m) v -= n1[m] * n2[m];
    return v;
}

/* One candidate pair (i from catalogue a, j from catalogue b): the flat bin
 * it is added to, or -1, and its weight. */
static inline int pair_bin_3d(const orc_setup *s, const orc_cat *a, int i, const orc_cat *b, int j, float *w_out) {
    const double *x1 = a->xyz + 3 * (size_t)i, *x2 = b->xyz + 3 * (size_t)j;
    float d[3];
    for (int m = 0; m < 3; ++m) d[m] = (float)(x1[m] - x2[m]);
    float s2 = d[0] * d[0] + d[1] * d[1] + d[2] * d[2];
    if (!(s2 < s->max_r_sq && s2 > s->min_r_sq)) return -1;
    float w1 = a->w ? a->w[i] : 1.0f, w2 = b->w ? b->w[j] : 1.0f;
    const double *n1 = a->unit + 3 * (size_t)i, *n2 = b->unit + 3 * (size_t)j;

    float weight;
    if (s->weight_kind == ORC_W_PLAIN) {
        weight = w1 * w2;
    } else if (s->weight_kind == ORC_W_INVP_DD) {
        /* src/correlators_invpweight.cpp:51-77 */
        double omct = one_minus_cos(n1, n2);
        float pw = popc_weight(a->masks + (size_t)i * a->n_mask, b->masks + (size_t)j * b->n_mask, a->n_mask);
        if (g_dither) {
            float dw = popc_weight(a->dmasks + (size_t)i * a->n_mask, b->dmasks + (size_t)j * b->n_mask, a->n_mask);
            pw = (float)(orc_interp(s->up, omct) * dw / pw);
        } else {
            pw = (float)(orc_interp(s->up, omct) * s->n_runs / pw);
        }
        float iw1 = a->iw ? a->iw[i] : w1, iw2 = b->iw ? b->iw[j] : w2;
        weight = iw1 * iw2 * pw;
    } else {
        /* src/correlators_invpweight.cpp:184-189 */
        double omct = one_minus_cos(n1, n2);
        weight = (float)((double)(w1 * w2) * orc_interp(s->up, omct));
    }

    *w_out = weight;
    if (s->mode == ORC_MONOPOLE) {
        int bin = orc_to_int(orc_axis_bin_num(&s->ax1, sqrtf(s2)));
        return (bin < s->ax1.n_bins && bin >= 0) ? bin : -1;
    }
    float pi;
    if (g_los_midpoint) {
        /* src/correlators.cpp:172-182 */
        float sum[3], inv = 0.0f;
        for (int m = 0; m < 3; ++m) {
            sum[m] = (float)(x1[m] + x2[m]);
            inv += sum[m] * sum[m];
        }
        inv = (float)(1.0 / (double)sqrtf(inv));
        pi = d[0] * sum[0] * inv;
        pi += d[1] * sum[1] * inv;
        pi += d[2] * sum[2] * inv;
    } else {
        /* pi, _ANGULAR_PI_DEFN (src/correlators.cpp:166-170) */
        pi = (float)((double)d[0] * (n1[0] + n2[0]));
        pi = (float)((double)pi + (double)d[1] * (n1[1] + n2[1]));
        pi = (float)((double)pi + (double)d[2] * (n1[2] + n2[2]));
        pi = (float)((double)pi * 0.5);
    }
    float v1, v2;
    if (s->mode == ORC_SIGMA_PI) {
        v1 = sqrtf(s2 - pi * pi);
        v2 = fabsf(pi);
    } else {
        float sv = sqrtf(s2);
        v1 = sv;
        v2 = fabsf(pi) / sv;
    }
    int b1 = orc_to_int(orc_axis_bin_num(&s->ax1, v1));
    if (b1 < s->ax1.n_bins && b1 >= 0) {
        int b2 = orc_to_int(orc_axis_bin_num(&s->ax2, v2));
        if (b2 < s->ax2.n_bins && b2 >= 0) return b1 * s->ax2.n_bins + b2;
    }
    return -1;
}

static void eval_pair(const orc_setup *s, const orc_cat *a, int i, const orc_cat *b, int j, orc_acc *acc) {
    float w;
    int bin = pair_bin_3d(s, a, i, b, j, &w);
    if (bin < 0) return;
    add_pair(s, acc->full, acc->sub, a->jk ? a->jk[i] : 0, b->jk ? b->jk[j] : 0, bin, w);
}

/* Adjoint of one pair of a plain-weight count: the pair adds w_i w_j to its
 * bin, so dL/dw_i += G[bin] w_j and dL/dw_j += G[bin] w_i. */
static void eval_pair_grad(const orc_setup *s, const orc_cat *a, int i, const orc_cat *b, int j, orc_acc *acc) {
    float w;
    int bin = pair_bin_3d(s, a, i, b, j, &w);
    if (bin < 0) return;
    const double w1 = a->w ? a->w[i] : 1.0f, w2 = b->w ? b->w[j] : 1.0f;
    acc->ga[i] += acc->G[bin] * w2;
    acc->gb[j] += acc->G[bin] * w1;
}

static void setup_3d(orc_setup *s, int mode, const double axp[6], int nb1, int nb2, int n_jk) {
    memset(s, 0, sizeof(*s));
    s->mode = mode;
    s->n_jk = n_jk;
    if (mode == ORC_MONOPOLE) {
        orc_axis_init(&s->ax1, axp[0], axp[1], nb1, axp[2]);
        s->max_r_sq = s->ax1.max * s->ax1.max;
        s->min_r_sq = s->ax1.min * s->ax1.min;
        s->nb = nb1;
    } else if (mode == ORC_SIGMA_PI) {
        orc_axis_init(&s->ax1, axp[0], axp[1], nb1, axp[2]);
        orc_axis_init(&s->ax2, axp[3], axp[4], nb2, axp[5]);
        s->max_r_sq = s->ax1.max * s->ax1.max + s->ax2.max * s->ax2.max;
        s->min_r_sq = s->ax1.min * s->ax1.min;
        if (s->ax1.min > s->ax2.min) s->min_r_sq = s->ax2.min * s->ax2.min;
        s->nb = nb1 * nb2;
    } else {
        orc_axis_init(&s->ax1, axp[0], axp[1], nb1, axp[2]);
        orc_axis_init(&s->ax2, 0.0, 1.0, nb2, 0.0);
        s->max_r_sq = s->ax1.max * s->ax1.max;
        s->min_r_sq = s->ax1.min * s->ax1.min;
        s->nb = nb1 * nb2;
    }
}

static void finish(const orc_setup *s, int is_auto, double *full, double *sub) {
    /* invert_jk_hists (src/hist.cpp:270-277) then x2 for auto counts */
    for (int r = 0; r < s->n_jk; ++r)
        for (int b = 0; b < s->nb; ++b) sub[(size_t)r * s->nb + b] = full[b] - sub[(size_t)r * s->nb + b];
    if (is_auto) {
        for (int b = 0; b < s->nb; ++b) full[b] *= 2.0;
        for (size_t k = 0; k < (size_t)s->n_jk * s->nb; ++k) sub[k] *= 2.0;
    }
}

/* Pair loop over a uniform grid of the given side.  "pts" are the positions
 * the grid is built from (xyz for 3-D, x_norm for angular counts). */
typedef void (*orc_eval_fn)(const orc_setup *, const orc_cat *, int, const orc_cat *, int, orc_acc *);

/* out: the accumulators the per-thread ones are added into; histograms
 * always, gradients (indexed by catalogue index) when out->ga is set. */
static void pair_loop(const orc_setup *s, int is_auto, const orc_cat *a, const int *pa, int na, const orc_cat *b,
                      const int *pb, int nb_pts, int use_unit, double side, orc_eval_fn fn, int n_threads,
                      orc_acc *out) {
    const double *ptsa = use_unit ? a->unit : a->xyz;
    const double *ptsb = use_unit ? b->unit : b->xyz;
    double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
    for (int i = 0; i < na; ++i)
        for (int m = 0; m < 3; ++m) {
            double v = ptsa[3 * (size_t)pa[i] + m];
            if (v < lo[m]) lo[m] = v;
            if (v > hi[m]) hi[m] = v;
        }
    if (!is_auto)
        for (int i = 0; i < nb_pts; ++i)
            for (int m = 0; m < 3; ++m) {
                double v = ptsb[3 * (size_t)pb[i] + m];
                if (v < lo[m]) lo[m] = v;
                if (v > hi[m]) hi[m] = v;
            }
    if (na == 0 || (!is_auto && nb_pts == 0)) return;
    orc_grid ga, gb;
    grid_build(&ga, ptsa, pa, na, lo, hi, side);
    if (!is_auto) grid_build(&gb, ptsb, pb, nb_pts, lo, hi, side);
    const orc_grid *g2 = is_auto ? &ga : &gb;
    int dim[3] = {ga.dim[0], ga.dim[1], ga.dim[2]};
    long long ncell = (long long)dim[0] * dim[1] * dim[2];
    size_t hsz = (size_t)s->nb * (1 + s->n_jk);
#ifdef _OPENMP
    if (n_threads <= 0) n_threads = omp_get_max_threads();
#else
    n_threads = 1;
#endif
#pragma omp parallel num_threads(n_threads)
    {
        double *h = (double *)calloc(hsz, sizeof(double));
        orc_acc acc = {h, h + s->nb, NULL, NULL, out->G};
        if (out->ga) {
            acc.ga = (double *)calloc((size_t)(a->n > 0 ? a->n : 1), sizeof(double));
            acc.gb = is_auto ? acc.ga : (double *)calloc((size_t)(b->n > 0 ? b->n : 1), sizeof(double));
        }
#pragma omp for schedule(dynamic)
        for (long long c = 0; c < ncell; ++c) {
            int cx = (int)(c / ((long long)dim[1] * dim[2])), cy = (int)((c / dim[2]) % dim[1]), cz = (int)(c % dim[2]);
            for (int i0 = ga.start[c]; i0 < ga.start[c + 1]; ++i0) {
                int i = ga.idx[i0];
                for (int ox = -1; ox <= 1; ++ox)
                    for (int oy = -1; oy <= 1; ++oy)
                        for (int oz = -1; oz <= 1; ++oz) {
                            int nx = cx + ox, ny = cy + oy, nz = cz + oz;
                            if (nx < 0 || ny < 0 || nz < 0 || nx >= dim[0] || ny >= dim[1] || nz >= dim[2]) continue;
                            long long c2 = ((long long)nx * dim[1] + ny) * dim[2] + nz;
                            if (is_auto && c2 < c) continue;
                            for (int j0 = g2->start[c2]; j0 < g2->start[c2 + 1]; ++j0) {
                                if (is_auto && c2 == c && j0 <= i0) continue;
                                fn(s, a, i, b, g2->idx[j0], &acc);
                            }
                        }
            }
        }
#pragma omp critical
        {
            for (size_t k = 0; k < (size_t)s->nb; ++k) out->full[k] += acc.full[k];
            for (size_t k = 0; k < (size_t)s->nb * s->n_jk; ++k) out->sub[k] += acc.sub[k];
            if (out->ga) {
                for (int k = 0; k < a->n; ++k) out->ga[k] += acc.ga[k];
                if (!is_auto)
                    for (int k = 0; k < b->n; ++k) out->gb[k] += acc.gb[k];
            }
        }
        free(h);
        if (out->ga) {
            free(acc.ga);
            if (!is_auto) free(acc.gb);
        }
    }
    grid_free(&ga);
    if (!is_auto) grid_free(&gb);
}

/* 3-D count.  is_auto: DD-style count of catalogue a with itself (each
 * unordered pair once, then x2); otherwise the cross count of a with b.
 * weight_kind selects plain weight products or the inverse-p DD/DR weights;
 * up/n_runs are used only by the latter.  full[nb] and sub[n_jk*nb] receive
 * the histograms after invert_jk_hists and (auto) x2.  n_used (optional)
 * receives the number of points kept by the d_comov partition. */
int orc_count_3d(int mode, int is_auto, const orc_cat *a, const orc_cat *b, int n_jk, const double axp[6], int nb1,
                 int nb2, int weight_kind, const orc_upweight *up, int n_runs, int n_threads, double *full, double *sub,
                 int *n_used) {
    orc_setup s;
    setup_3d(&s, mode, axp, nb1, nb2, n_jk);
    s.weight_kind = weight_kind;
    s.up = up;
    s.n_runs = n_runs;
    memset(full, 0, sizeof(double) * s.nb);
    memset(sub, 0, sizeof(double) * s.nb * n_jk);
    int *pa = (int *)malloc(sizeof(int) * (size_t)(a->n > 0 ? a->n : 1));
    int na = orc_partition(a->dcom, a->n, pa);
    int *pb = NULL, nbp = 0;
    if (!is_auto) {
        pb = (int *)malloc(sizeof(int) * (size_t)(b->n > 0 ? b->n : 1));
        nbp = orc_partition(b->dcom, b->n, pb);
    }
    if (n_used) {
        n_used[0] = na;
        n_used[1] = nbp;
    }
    /* Grid side: every pair with float s^2 < max_r_sq has |x1_m - x2_m| below
     * sqrt(max_r_sq) * (1 + 2^-22); the extra margin absorbs the rounding of
     * the cell-index division. */
    double side = sqrt((double)s.max_r_sq) * (1.0 + 1e-5) + 1e-12;
    orc_acc out = {full, sub, NULL, NULL, NULL};
    pair_loop(&s, is_auto, a, pa, na, is_auto ? a : b, is_auto ? pa : pb, nbp, 0, side, eval_pair, n_threads, &out);
    finish(&s, is_auto, full, sub);
    free(pa);
    free(pb);
    return 0;
}

/* Adjoint of a plain-weight 3-D count (the FP64 CPU gradient of the weight
 * derivative): with G[nb] = dL/d(raw full histogram) — the unordered-pair
 * sums before the auto-count doubling — grad_a[i] = sum over the pairs (i, j)
 * in a binned range of G[bin] * w_j, and grad_b likewise for catalogue b
 * (auto: every pair adds to both ends in grad_a).  Arrays are indexed by
 * catalogue index; points dropped by the d_comov partition get 0. */
int orc_count_backward(int mode, int is_auto, const orc_cat *a, const orc_cat *b, const double axp[6], int nb1,
                       int nb2, const double *G, int n_threads, double *grad_a, double *grad_b) {
    orc_setup s;
    setup_3d(&s, mode, axp, nb1, nb2, 1);
    s.weight_kind = ORC_W_PLAIN;
    double *full = (double *)calloc((size_t)s.nb, sizeof(double));
    double *sub = (double *)calloc((size_t)s.nb, sizeof(double));
    memset(grad_a, 0, sizeof(double) * (size_t)a->n);
    if (!is_auto) memset(grad_b, 0, sizeof(double) * (size_t)b->n);
    int *pa = (int *)malloc(sizeof(int) * (size_t)(a->n > 0 ? a->n : 1));
    int na = orc_partition(a->dcom, a->n, pa);
    int *pb = NULL, nbp = 0;
    if (!is_auto) {
        pb = (int *)malloc(sizeof(int) * (size_t)(b->n > 0 ? b->n : 1));
        nbp = orc_partition(b->dcom, b->n, pb);
    }
    double side = sqrt((double)s.max_r_sq) * (1.0 + 1e-5) + 1e-12;
    orc_acc out = {full, sub, grad_a, is_auto ? grad_a : grad_b, G};
    pair_loop(&s, is_auto, a, pa, na, is_auto ? a : b, is_auto ? pa : pb, nbp, 0, side, eval_pair_grad, n_threads,
              &out);
    free(pa);
    free(pb);
    free(full);
    free(sub);
    return 0;
}

/* ------------------------------------------------------------ angular --- */

typedef struct {
    orc_setup base;
    int kind;
} orc_ang_setup;

static void eval_angular(const orc_setup *s, const orc_cat *a, int i, const orc_cat *b, int j, orc_acc *acc) {
    const orc_ang_setup *as = (const orc_ang_setup *)s;
    const double *n1 = a->unit + 3 * (size_t)i, *n2 = b->unit + 3 * (size_t)j;
    double omct = one_minus_cos(n1, n2);
    int jk1 = a->jk ? a->jk[i] : 0, jk2 = b->jk ? b->jk[j] : 0;
    float w1 = a->w ? a->w[i] : 1.0f, w2 = b->w ? b->w[j] : 1.0f;
    float iw1 = a->iw ? a->iw[i] : w1, iw2 = b->iw ? b->iw[j] : w2;
    float weight;
    switch (as->kind) {
    case 0: /* auto_pair_count_angular (:901, :919) */
    case 2: /* cross_pair_count_angular (:968) */
        weight = iw1 * iw2;
        break;
    case 1: { /* auto_pair_count_angular_invpweights (:743-764) */
        float pw = popc_weight(a->masks + (size_t)i * a->n_mask, b->masks + (size_t)j * b->n_mask, a->n_mask);
        if (g_dither)
            pw = popc_weight(a->dmasks + (size_t)i * a->n_mask, b->dmasks + (size_t)j * b->n_mask, a->n_mask) / pw;
        else
            pw = (float)s->n_runs / pw;
        weight = iw1 * iw2 * pw;
        break;
    }
    default: /* cross_pair_count_angular_invpweights (:853) */
        weight = w1 * w2;
        break;
    }
    /* JKHists::add_pair takes the value as float (src/hist.cpp:246). */
    int bin = orc_to_int(orc_axis_bin_num(&s->ax1, (float)omct));
    if (bin < s->ax1.n_bins && bin >= 0) add_pair(s, acc->full, acc->sub, jk1, jk2, bin, weight);
}

/* Angular count.  kind 0 = DD (all points), 1 = DD with inverse-p weights
 * (points with d_comov >= 0 via the partition loop), 2 = DR, 3 = DR with
 * inverse-p weights (both partitioned).  Axis: Hist(0, 1 - cos(theta_max),
 * n_theta, theta_log_base) (src/correlators_invpweight.cpp:991). */
int orc_count_angular(int kind, const orc_cat *a, const orc_cat *b, int n_jk, double theta_max, int n_theta,
                      double theta_log_base, int n_runs, int n_threads, double *full, double *sub) {
    orc_ang_setup as;
    memset(&as, 0, sizeof(as));
    as.kind = kind;
    orc_setup *s = &as.base;
    s->n_jk = n_jk;
    s->n_runs = n_runs;
    orc_axis_init(&s->ax1, 0.0, 1.0 - cos(theta_max), n_theta, theta_log_base);
    s->nb = n_theta;
    memset(full, 0, sizeof(double) * s->nb);
    memset(sub, 0, sizeof(double) * s->nb * n_jk);
    int req = (kind == 1 || kind == 3);
    int is_auto = (kind == 0 || kind == 1);
    int *pa = (int *)malloc(sizeof(int) * (size_t)(a->n > 0 ? a->n : 1));
    int na = orc_partition(req ? a->dcom : NULL, a->n, pa);
    int *pb = NULL, nbp = 0;
    if (!is_auto) {
        pb = (int *)malloc(sizeof(int) * (size_t)(b->n > 0 ? b->n : 1));
        nbp = orc_partition(req ? b->dcom : NULL, b->n, pb);
    }
    /* Pairs in a valid bin have float(1 - cos) below the axis maximum up to
     * rounding, so unit vectors closer than sqrt(2 * 1.5 * max) in chord
     * include them all. */
    double side = sqrt(3.0 * (double)s->ax1.max) + 1e-9;
    orc_acc out = {full, sub, NULL, NULL, NULL};
    pair_loop(s, is_auto, a, pa, na, is_auto ? a : b, is_auto ? pa : pb, nbp, 1, side, eval_angular, n_threads, &out);
    finish(s, is_auto, full, sub);
    free(pa);
    free(pb);
    return 0;
}

/* ----------------------------------------------------- finalisation --- */

/* JKHists::normalise, one-catalogue form (src/hist.cpp:290-321). */
void orc_normalise_auto(const float *w, const int *jk, int n, int n_jk, int nb, double *full, double *sub) {
    double sw = 0.0;
    double *swj = (double *)calloc((size_t)n_jk, sizeof(double));
    int *nj = (int *)calloc((size_t)n_jk, sizeof(int));
    for (int i = 0; i < n; ++i) {
        float wi = w ? w[i] : 1.0f;
        int r = jk ? jk[i] : 0;
        sw += wi;
        swj[r] += wi;
        ++nj[r];
    }
    for (int r = 0; r < n_jk; ++r) swj[r] = sw - swj[r];
    sw = sw * sw * (1.0 - 1.0 / (double)n);
    for (int r = 0; r < n_jk; ++r) swj[r] = swj[r] * swj[r] * (1.0 - 1.0 / nj[r]);
    for (int b = 0; b < nb; ++b) full[b] /= sw;
    for (int r = 0; r < n_jk; ++r)
        for (int b = 0; b < nb; ++b) sub[(size_t)r * nb + b] /= swj[r];
    free(swj);
    free(nj);
}

/* JKHists::normalise, two-catalogue form (src/hist.cpp:323-367). */
void orc_normalise_cross(const float *w1, const int *jk1, int n1, const float *w2, const int *jk2, int n2, int n_jk,
                         int nb, double *full, double *sub) {
    double s1 = 0.0, s2 = 0.0;
    double *j1 = (double *)calloc((size_t)n_jk, sizeof(double));
    double *j2 = (double *)calloc((size_t)n_jk, sizeof(double));
    for (int i = 0; i < n1; ++i) {
        float wi = w1 ? w1[i] : 1.0f;
        s1 += wi;
        j1[jk1 ? jk1[i] : 0] += wi;
    }
    for (int r = 0; r < n_jk; ++r) j1[r] = s1 - j1[r];
    for (int i = 0; i < n2; ++i) {
        float wi = w2 ? w2[i] : 1.0f;
        s2 += wi;
        j2[jk2 ? jk2[i] : 0] += wi;
    }
    for (int r = 0; r < n_jk; ++r) j2[r] = s2 - j2[r];
    s1 *= s2;
    for (int r = 0; r < n_jk; ++r) j1[r] *= j2[r];
    for (int b = 0; b < nb; ++b) full[b] /= s1;
    for (int r = 0; r < n_jk; ++r)
        for (int b = 0; b < nb; ++b) sub[(size_t)r * nb + b] /= j1[r];
    free(j1);
    free(j2);
}

/* ls_estimator (src/io.cpp:643-651). */
double orc_ls(double dd, double dr, double rr) {
    if (rr == 0) return 0;
    return dd / rr - 2.0 * dr / rr + 1.0;
}

/* ------------------------------------------------ binning monotonicity --- */

/* Exhaustive check that the reference binning is non-decreasing over every
 * float in [lo, hi] (non-negative lo): the engine's threshold tables rely on
 * it.  sqrt_space applies sqrtf first (s from s^2, sigma from s^2 - pi^2).
 * Returns the first offending float's bit pattern, or 0xffffffff. */
unsigned orc_axis_check_monotone(const orc_axis *ax, int sqrt_space, float lo, float hi) {
    unsigned ulo, uhi;
    memcpy(&ulo, &lo, 4);
    memcpy(&uhi, &hi, 4);
    unsigned bad = 0xffffffffu;
    const unsigned chunk = 1u << 20;
#pragma omp parallel for schedule(dynamic) reduction(min : bad)
    for (long long c = ulo; c <= (long long)uhi; c += chunk) {
        unsigned end = (unsigned)((c + chunk - 1 < (long long)uhi) ? c + chunk - 1 : uhi);
        float x;
        unsigned u = (unsigned)c;
        memcpy(&x, &u, 4);
        int prev = orc_to_int(orc_axis_bin_num(ax, sqrt_space ? sqrtf(x) : x));
        for (unsigned v = u + 1; v <= end && v > u - 1; ++v) {
            memcpy(&x, &v, 4);
            int cur = orc_to_int(orc_axis_bin_num(ax, sqrt_space ? sqrtf(x) : x));
            if (cur < prev && v < bad) bad = v;
            prev = cur;
            if (v == 0xffffffffu) break;
        }
    }
    return bad;
}
