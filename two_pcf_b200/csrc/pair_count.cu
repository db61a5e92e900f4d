// K2 (FP32 + guard) and K7 (plain FP64) 3-D pair counting: the replacement
// for auto_/cross_pair_count_{monopole,sigma_pi,s_mu}
// (src/correlators.cpp:11-125, :156-278, :309-430).
//
// Persistent CTAs pull work items — a chunk of one (cell, jackknife region)
// run of catalogue A against one run of catalogue B — from a device queue.
// Each thread holds R points of A in registers; B streams through shared
// memory in tiles staged by one-dimensional bulk copies (cp.async.bulk with
// mbarrier completion) into a ring of buffers; the last warp to finish a
// buffer stages the next tile into it, so no block barrier separates tiles.
//
// Producer/consumer inside every warp: the candidate loop evaluates s^2 in
// FP32 from cell-relative coordinates and pushes the pairs that pass the
// (guard-widened) range test into a per-warp queue with a ballot; whenever 32
// are queued the whole warp bins them together, so the binning path never
// runs divergent.  Binning uses host-built lookup tables over the float value
// (s^2, sigma^2) or a linear bucket index (mu, |pi|); buckets within the
// proven FP32 error bound of a bin edge are marked ambiguous and resolved by
// threshold search, and a pair that is still within the bound is re-evaluated
// with the reference's exact float/double sequence (exact_pair).  Counts go to
// one privatised 64-bit fixed-point histogram per CTA (two 32-bit shared
// words with carry), added to the global full histogram and to both regions'
// rows at the end of each item.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <limits>
#include <memory>
#include <mutex>
#include <string>
#include <type_traits>
#include <vector>

#include "engine.h"
#include "pair_kernels.cuh"

namespace tpcf {
namespace {

constexpr int NT = 256;        // threads per CTA
constexpr int NWARP = NT / 32;
constexpr int R = 4;           // A points per thread
constexpr int TA = NT * R;     // A chunk
constexpr int TB = 256;        // B points per staged tile (FP32 path)
constexpr int TB_EXACT = 256;  // B points per staged tile (FP64 path)
constexpr int TB_ALT = 512;    // the alternative configuration of the FP32 jackknife kernels
constexpr int kTileMax = TB_ALT > TB_EXACT ? TB_ALT : TB_EXACT;
// Staged tile buffers (warps may run up to NBUF - 1 tiles apart): FP32 path,
// FP64 path (whose per-pair loads of the double arrays lose L1 to a third
// buffer; measured on the survey benchmark, each path at its faster depth)
constexpr int NBUF = 3;
constexpr int NBUF_EXACT = 2;
constexpr int kNbufMax = NBUF > NBUF_EXACT ? NBUF : NBUF_EXACT;
// Count kernels without jackknife regions keep the lighter settings (two
// buffers, a push width of 2) so that their shared memory allows three CTAs
// per SM (the adjoint runs two CTAs per SM either way and keeps the others).
//
// Kernel configuration `cfg` (plain-weight FP32+guard kernels; the autotuner
// picks it per count class): 0 is the setting above for each kind; 1 swaps
// the kinds' settings -- the jackknife kernels take the light ring (two
// buffers, push width 2) with tiles of TB_ALT points, the kernels without
// regions the heavy one (three buffers, push width 4).
constexpr int NBUF_NOJK = 2;
__host__ __device__ constexpr bool light_fast(bool exact, bool jk, bool adj, int cfg = 0) {
    return !exact && !adj && (cfg == 0 ? !jk : jk);
}
__host__ __device__ constexpr int n_buffers(bool exact, bool jk, bool adj, int cfg = 0) {
    return exact ? NBUF_EXACT : (light_fast(exact, jk, adj, cfg) ? NBUF_NOJK : NBUF);
}
// B points per staged tile
__host__ __device__ constexpr int tile_points(bool exact, bool jk, bool adj, int cfg = 0) {
    return exact ? TB_EXACT : ((cfg == 1 && jk && !adj) ? TB_ALT : TB);
}
// queue entries pack (A chunk index << kTileShift | tile index)
constexpr int kTileShift = kTileMax <= 256 ? 8 : (kTileMax <= 512 ? 9 : 10);
constexpr int kTileMask = (1 << kTileShift) - 1;
static_assert(16 + 12 * kNbufMax <= 64 && kTileMax <= 1024 && (size_t)TA << kTileShift < (1u << 31), "queue entry packing");
// A slots pushed between two consume checks: FP32 path, FP64 path by mode
// (measured on the survey benchmark: s-mu counts run faster at 4, sigma-pi
// counts at 2); the warp's queue holds a partial round plus 4 ballots
constexpr int QPUSH = 4;
constexpr int QPUSH_NOJK = 2;
__host__ __device__ constexpr int qpush_exact(int mode) { return mode == MODE_S_MU ? 4 : 2; }
__host__ __device__ constexpr int queue_cap(bool exact, bool jk, bool adj, int cfg = 0) {
    return 32 + 32 * (light_fast(exact, jk, adj, cfg) ? QPUSH_NOJK : 4);
}
static_assert(R % QPUSH == 0 && R % QPUSH_NOJK == 0 && R % 2 == 0 && QPUSH <= 4 && QPUSH_NOJK <= 4,
              "the push loops consume after every QPUSH A slots");
// Table 1 over the float bits of its value: 2^bits buckets per octave (8,
// over 32 octaves; 9 over 16 for the linear sigma axis, whose edges crowd
// less toward 0 but sit closer together in sigma^2 at large sigma)
constexpr int LUT1_N = 8192;
constexpr int LUT1_N_T2 = 6144;  // when table 2 is staged too (the shared-memory footprint of both stays 10 KB)
constexpr int LUT2_N = 4096;
constexpr unsigned char LUT_INV = 254;  // every value of the bucket is dropped
constexpr unsigned char LUT_AMB = 255;  // bucket within the guard of an edge
// Edge-coded tables (axes of at most 126 bins): LUT_EDGE + k marks a bucket
// whose guarded range holds exactly one threshold, T[k + 1], with bin k below
// it and bin k + 1 above; the kernel compares the value with T[k + 1] and
// only a value within its guard of it needs the exact path.
constexpr unsigned char LUT_EDGE = 128;
constexpr int kLutEdgeMaxBins = 126;
constexpr uint32_t kWaitLimit = 1u << 22;

// A count's error record on the device: [0] the flag (0 none, kErrTimeout: a
// bounded wait gave up, kErrCheck: a device bounds check failed), then for a
// failed check its id, the value and the limit it broke.  Any flag stops the
// CTAs from taking further work items and the host discards the results.
constexpr int kErrWords = 4;
constexpr int kErrTimeout = 4;
constexpr int kErrCheck = 8;
// Device bounds checks of the checked build (TPCF_DEVICE_CHECKS)
enum DeviceCheck {
    DC_BIN = 1,       // bin index < bins
    DC_JOB,           // work item's job < jobs of the launch
    DC_SEGMENTS,      // work item's segments within the segment list
    DC_A_CHUNK,       // A chunk length within 0..kChunkA
    DC_A_POINTS,      // A chunk within grid A's points
    DC_A_CELL,        // A cell < cells of grid A
    DC_A_REGION,      // A region < regions
    DC_B_POINTS,      // segment's B run within grid B's points
    DC_B_CELL,        // B cell < cells of grid B
    DC_B_REGION,      // segment's region < regions
    DC_QUEUE,         // warp queue fill within its capacity
    DC_SIDE_QUEUE,    // side queue fill within its capacity
};
static_assert(TA == kChunkA, "work items are built for chunks of kChunkA points");

struct GridK {
    const float4 *pos;
    const float4 *aux;
    const int *idx;
    const double4 *xyz_s;
    const double4 *unit_s;
    const int3 *coord;
    int kmin0, kmin1, kmin2;
    int n_pts, n_cells;  // points and dense cells of the grid
    const double *xyz;   // original catalogue arrays (exact path)
    const double *unit;
};

// One (catalogue A, catalogue B, output histogram) of a launch; a batched
// launch runs the work items of many jobs.
struct JobK {
    GridK a, b;
    int out;  // output slot: histograms at g_full + 2 nb out, g_sub + 2 nb n_jk out
    int pad[3];
};

struct KParams {
    const JobK *jobs;  // jackknife kernels: the job of each work item (batched launches)
    JobK job0;         // kernels without jackknife regions: the launch's only job
    const WorkItem *items;
    const Segment *segs;
    int n_items;
    int n_segs, n_jobs;
    int *head;
    double side;
    int n1, n2, nb;
    float min_r_sq, max_r_sq, lo_cut, hi_cut;
    float cut_mid, cut_half;  // |s^2 - cut_mid| < cut_half covers [lo_cut, hi_cut]
    float s2_test;            // FP32 candidate test s^2 < s2_test (the upper side of the one above)
    float g_s2, g_pi, g_a, c1_mu, c2_mu, g_mu0;
    float s2_lut_min;   // below this s^2 the mu table's guard does not hold
    int lut_edge1, lut_edge2;  // tables carry LUT_EDGE codes
    const float *t1g, *t2g;
    const unsigned char *lut1g, *lut2g;
    unsigned lut1_base;  // (bits of the lowest bucket) >> lut1_shift
    unsigned lut1_shift;  // 23 - bits per octave
    int lut1_n;           // buckets of table 1 (LUT1_N, or LUT1_N_T2 beside table 2)
    float lut2_scale;    // bucket = (int)(value * lut2_scale)
    int direct2;         // axis 2 binned directly (linear, from 0): bin = floor(value * inv2)
    float inv2, k2;      // the axis's float 1 / step and the constant part of its guard (in bins)
    float c1y, c2y, g0y;  // mu guard in bins: c2y / s^2 + c1y / s + g0y (k2 included)
    unsigned long long *g_full, *g_sub;  // 128-bit fixed-point sums (low, high word pairs)
    int n_jk;
    float wscale;
    unsigned long long *counters;  // candidates, in_range, guard, flushes
    int *err;
    // inverse-p weights and the angular up-weight
    const long long *a_masks, *b_masks;  // original catalogue bitmasks, object-major
    const long long *a_dmasks, *b_dmasks;  // dither masks (dither != 0), same layout
    int n_mask;
    int mask_vec;  // mask words per load: 4 (n_mask % 4 == 0, 32-byte aligned), 2 (even, 16-byte aligned) or 1
    int dither;    // _USE_DITHER_WEIGHTS: popc of the dither masks replaces n_runs
    int los_mid;   // pi along x1 + x2 (src/correlators.cpp:172-182), exact path only
    float n_runs_f;
    double n_runs_d;
    const float *up_thr;                 // n_up + 1 interval thresholds
    const double *up_bins, *up_centre;   // n_up + 1 each
    int n_up;
    double up_min, up_max;
    float g_ang;       // error bound of the FP32 1 - cos(theta)
    unsigned *flags;   // (1 + n_jk) * nb: non-finite weights met per bin (1 NaN, 2 +inf, 4 -inf)
    // adjoint (W_ADJ): dL/d(full histogram) and the per-point gradients,
    // indexed by catalogue index (grad_b == grad_a for auto counts)
    const double *adj_G;
    double *grad_a, *grad_b;
    double adj_scale, adj_inv;  // gradient terms are summed as round(term * adj_scale) in 64-bit fixed point
    int force_timeout;          // tests: raise the timeout flag after a (completed) wait for a tile
};

// Shared-memory views the binning steps use.
struct Shm {
    const float *t1, *t2;          // threshold tables
    const unsigned char *l1, *l2;  // lookup tables
    uint32_t *lo, *hi;             // 64-bit fixed-point histogram as two 32-bit words per bin
    const double *G;               // adjoint: dL/d(full histogram) (aliases lo/hi)
    uint32_t *ga_lo, *ga_hi;       // adjoint: fixed-point gradient sums of the A chunk (two words per point)
    uint32_t *gb_lo, *gb_hi;       // and of the B tile
};

struct SmemLayout {
    size_t lo, hi, alo, ahi, t1, t2, lut1, lut2, queue, slow, achunk, ga, gb, tile0, tile1, misc, total;
};

// Per-warp side queue of the FP32 path: the packed (A chunk index, tile
// index) of pairs whose bin the tables leave ambiguous (bin_fast); at most
// 31 wait between rounds and a round adds at most 32.
constexpr int kSlowCap = 64;

// FP32 path: pos and aux float4 per point; FP64 path: one double4 per point
__host__ __device__ inline size_t tile_bytes(bool exact, bool jk, bool adj, int cfg) {
    return (size_t)tile_points(exact, jk, adj, cfg) * 32;
}

// lo/hi: the histogram pairs are added to (per segment region when there
// are jackknife regions); alo/ahi: the item's A-side total (jackknife only).
__host__ __device__ inline SmemLayout smem_layout(int nb, int n1, int n2, bool exact, bool jk, bool adj = false,
                                                  int cfg = 0, bool lut2 = true) {
    SmemLayout L;
    size_t o = 0;
    L.lo = o;
    o += 4 * (size_t)nb;
    L.hi = o;
    o += 4 * (size_t)nb;
    L.alo = o;
    if (jk) o += 4 * (size_t)nb;
    L.ahi = o;
    if (jk) o += 4 * (size_t)nb;
    L.t1 = o;
    o += 4 * (size_t)(n1 + 1);
    L.t2 = o;
    o += 4 * (size_t)(n2 + 1);
    L.lut1 = o;
    o += lut2 ? LUT1_N_T2 : LUT1_N;
    L.lut2 = o;  // table 2 only where an axis 2 is binned by table
    if (lut2) o += LUT2_N;
    o = (o + 15) / 16 * 16;
    L.queue = o;
    o += (size_t)NWARP * queue_cap(exact, jk, adj, cfg) * 16;
    L.slow = o;
    if (!exact) o += (size_t)NWARP * kSlowCap * 4;
    L.achunk = o;  // FP32 path: (x_norm, weight) of the item's A chunk
    if (!exact) o += (size_t)TA * 16;
    L.ga = o;      // adjoint: per-point gradient sums (64-bit fixed point as two 32-bit words)
    if (adj) o += (size_t)TA * 8;
    L.gb = o;
    if (adj) o += (size_t)TB * 8;
    o = (o + 127) / 128 * 128;
    L.tile0 = o;
    o += tile_bytes(exact, jk, adj, cfg);
    L.tile1 = o;
    o += (size_t)(n_buffers(exact, jk, adj, cfg) - 1) * tile_bytes(exact, jk, adj, cfg);
    o = (o + 15) / 16 * 16;
    L.misc = o;  // item index, mbarriers, tile-done counters, the item's job
    o += 64 + sizeof(JobK);
    L.total = o;
    return L;
}

// Exact evaluation of one pair with the reference's operation sequence
// (src/correlators.cpp:33-40 separation and range test; :166-170 pi with
// _ANGULAR_PI_DEFN; :185 sigma; :338-340 s and mu; src/hist.cpp:484-502
// binning), bins looked up in the threshold tables.  Returns the flat bin or
// -1; *in_range receives the range-test result.
struct ExactArgs {
    const double *a_xyz, *a_unit, *b_xyz, *b_unit;
    float min_r_sq, max_r_sq;
    int n1, n2;
    int los_mid;
};

// With mid set, (n1*, n2*) are the positions x1, x2 and pi follows the
// reference's build without _ANGULAR_PI_DEFN (src/correlators.cpp:172-182):
// sum = (float)(x1 + x2), inv = (float)(1.0 / sqrtf(|sum|^2)) in double,
// pi = sum_m (d_m sum_m) inv, all in float.
template <int MODE>
__device__ __forceinline__ int exact_bin(const ExactArgs &E, const float *t1, const float *t2, float d0, float d1,
                                         float d2, double n1x, double n1y, double n1z, double n2x, double n2y,
                                         double n2z, bool *in_range, bool mid = false) {
    float s2 = __fadd_rn(__fadd_rn(__fmul_rn(d0, d0), __fmul_rn(d1, d1)), __fmul_rn(d2, d2));
    *in_range = (s2 < E.max_r_sq) && (s2 > E.min_r_sq);
    if (!*in_range) return -1;
    if (MODE == MODE_MONOPOLE) {
        int b = dev::locate_exact(t1, E.n1, s2);
        return (b >= 0 && b < E.n1) ? b : -1;
    }
    float pi;
    if (mid) {
        const float sx = __double2float_rn(__dadd_rn(n1x, n2x));
        const float sy = __double2float_rn(__dadd_rn(n1y, n2y));
        const float sz = __double2float_rn(__dadd_rn(n1z, n2z));
        const float r2 = __fadd_rn(__fadd_rn(__fmul_rn(sx, sx), __fmul_rn(sy, sy)), __fmul_rn(sz, sz));
        const float inv = __double2float_rn(__ddiv_rn(1.0, (double)__fsqrt_rn(r2)));
        pi = __fmul_rn(__fmul_rn(d0, sx), inv);
        pi = __fadd_rn(pi, __fmul_rn(__fmul_rn(d1, sy), inv));
        pi = __fadd_rn(pi, __fmul_rn(__fmul_rn(d2, sz), inv));
    } else {
        pi = __double2float_rn(__dmul_rn((double)d0, __dadd_rn(n1x, n2x)));
        pi = __double2float_rn(__dadd_rn((double)pi, __dmul_rn((double)d1, __dadd_rn(n1y, n2y))));
        pi = __double2float_rn(__dadd_rn((double)pi, __dmul_rn((double)d2, __dadd_rn(n1z, n2z))));
        pi = __double2float_rn(__dmul_rn((double)pi, 0.5));
    }
    int b1, b2;
    if (MODE == MODE_S_MU) {
        b1 = dev::locate_exact(t1, E.n1, s2);
        if (b1 < 0 || b1 >= E.n1) return -1;
        float mu = __fdiv_rn(fabsf(pi), __fsqrt_rn(s2));
        b2 = dev::locate_exact(t2, E.n2, mu);
    } else {
        float a = __fsub_rn(s2, __fmul_rn(pi, pi));
        if (a < 0.0f) return -1;  // sqrtf of a negative number: NaN, never binned
        b1 = dev::locate_exact(t1, E.n1, a);
        if (b1 < 0 || b1 >= E.n1) return -1;
        b2 = dev::locate_exact(t2, E.n2, fabsf(pi));
    }
    if (b2 < 0 || b2 >= E.n2) return -1;
    return b1 * E.n2 + b2;
}

// Guard-band re-evaluation from the original double arrays.
// 1 - cos(theta) of two unit vectors with the reference's sequence
// (src/correlators_invpweight.cpp:51-54, :738-741): ((1 - a0 b0) - a1 b1) -
// a2 b2 in double, each product and difference rounded once.
__device__ __forceinline__ double omct_exact(double a0, double a1, double a2, double b0, double b1, double b2) {
    double v = __dsub_rn(1.0, __dmul_rn(a0, b0));
    v = __dsub_rn(v, __dmul_rn(a1, b1));
    return __dsub_rn(v, __dmul_rn(a2, b2));
}

template <int MODE>
__device__ __forceinline__ int exact_pair(const ExactArgs E, const float *t1, const float *t2, int ia, int jb,
                                       bool *in_range) {
    if (MODE == MODE_ANGULAR) {
        // The angular histogram takes (float)(1 - cos(theta)) with no range
        // test (JKHists::add_pair's float value, src/hist.cpp:246).
        const double *u1 = E.a_unit + 3 * (size_t)ia, *u2 = E.b_unit + 3 * (size_t)jb;
        const float v = __double2float_rn(omct_exact(u1[0], u1[1], u1[2], u2[0], u2[1], u2[2]));
        const int b = dev::locate_exact(t1, E.n1, v);
        *in_range = b >= 0 && b < E.n1;
        return *in_range ? b : -1;
    }
    const double *x1 = E.a_xyz + 3 * (size_t)ia, *x2 = E.b_xyz + 3 * (size_t)jb;
    float d0 = __double2float_rn(__dsub_rn(x1[0], x2[0]));
    float d1 = __double2float_rn(__dsub_rn(x1[1], x2[1]));
    float d2 = __double2float_rn(__dsub_rn(x1[2], x2[2]));
    double n1x = 0, n1y = 0, n1z = 0, n2x = 0, n2y = 0, n2z = 0;
    if (MODE != MODE_MONOPOLE) {
        const double *u1 = E.los_mid ? x1 : E.a_unit + 3 * (size_t)ia;
        const double *u2 = E.los_mid ? x2 : E.b_unit + 3 * (size_t)jb;
        n1x = u1[0];
        n1y = u1[1];
        n1z = u1[2];
        n2x = u2[0];
        n2y = u2[1];
        n2z = u2[2];
    }
    return exact_bin<MODE>(E, t1, t2, d0, d1, d2, n1x, n1y, n1z, n2x, n2y, n2z, in_range,
                           MODE != MODE_MONOPOLE && E.los_mid);
}

// Parameters of the threshold-search path (passed by value to the
// non-inlined function).
struct PreciseArgs {
    int n1, n2;
    float min_r_sq, max_r_sq, g_s2, g_pi, g_a, c1_mu, c2_mu, g_mu0;
};

// Threshold search with the FP32 error bounds; falls back to exact_pair when
// a value lies within its bound of an edge.  Used for table buckets marked
// ambiguous.
template <int MODE>
__device__ __forceinline__ int precise_bin(const PreciseArgs P, const ExactArgs E, const float *t1, const float *t2,
                                        float s2, float pi, int ia, int jb, bool *in_range, bool *guarded) {
    *guarded = false;
    const dev::AxisK ax1{t1, P.n1, 0, 0.f, 0.f, 0.f, 0.f};
    const dev::AxisK ax2{t2, P.n2, 0, 0.f, 0.f, 0.f, 0.f};
    bool ex = (fabsf(s2 - P.max_r_sq) <= P.g_s2) || (fabsf(s2 - P.min_r_sq) <= P.g_s2);
    int bin = -1;
    bool inr = false;
    if (!ex) {
        inr = (s2 < P.max_r_sq) && (s2 > P.min_r_sq);
        if (inr) {
            if (MODE == MODE_MONOPOLE) {
                const int b1 = dev::locate_exact(t1, P.n1, s2);
                ex = dev::near_edge(ax1, s2, b1, P.g_s2);
                bin = (b1 >= 0 && b1 < P.n1) ? b1 : -1;
            } else if (MODE == MODE_S_MU) {
                const float inv_s = rsqrtf(s2);
                const int b1 = dev::locate_exact(t1, P.n1, s2);
                const float mu = fabsf(pi) * inv_s;
                const int b2 = dev::locate_exact(t2, P.n2, mu);
                const float gmu = fmaf(P.c2_mu * inv_s, inv_s, fmaf(P.c1_mu, inv_s, P.g_mu0));
                ex = dev::near_edge(ax1, s2, b1, P.g_s2) || dev::near_edge(ax2, mu, b2, gmu);
                bin = (b1 >= 0 && b1 < P.n1 && b2 >= 0 && b2 < P.n2) ? b1 * P.n2 + b2 : -1;
            } else {
                const float a = fmaf(-pi, pi, s2);
                const float api = fabsf(pi);
                const int b2 = dev::locate_exact(t2, P.n2, api);
                ex = dev::near_edge(ax2, api, b2, P.g_pi);
                int b1 = -1;
                if (a <= P.g_a) {
                    ex = ex || (a >= -P.g_a);  // near zero: sqrtf of a value of unknown sign
                } else {
                    b1 = dev::locate_exact(t1, P.n1, a);
                    ex = ex || dev::near_edge(ax1, a, b1, P.g_a);
                }
                bin = (b1 >= 0 && b1 < P.n1 && b2 >= 0 && b2 < P.n2) ? b1 * P.n2 + b2 : -1;
            }
        }
    }
    if (ex) {
        *guarded = true;
        bin = exact_pair<MODE>(E, t1, t2, ia, jb, &inr);
    }
    *in_range = inr;
    return bin;
}

__device__ __forceinline__ int lut1_index(unsigned base, unsigned shift, int n, float x) {
    const int i = (int)((__float_as_uint(x) >> shift) - base);
    return min(max(i, 0), n - 1);
}

__device__ __forceinline__ int lut2_index(float scale, float x) {
    const int i = (int)(x * scale);
    return min(max(i, 0), LUT2_N - 1);
}

struct Counters {
    unsigned in_range = 0, guard = 0;  // per thread, folded into 64-bit totals per item
};

// Table entry -> bin for value x: a plain bin, LUT_INV (returned as is), or
// for an edge-coded bucket the side of its threshold; *amb is set when x is
// within its guard g of that threshold (or the bucket is ambiguous).
__device__ __forceinline__ unsigned lut_decode(unsigned c, float x, const float *t, float g, int edge, bool *amb) {
    *amb = (c == LUT_AMB);
    if (edge && c >= LUT_EDGE && c < LUT_INV) {
        const unsigned k = c - LUT_EDGE;
        const float tk = t[k + 1];
        *amb = fabsf(x - tk) <= g;
        return k + (x >= tk ? 1u : 0u);
    }
    return c;
}

// Direct binning of a linear axis starting at 0 from y = value * (1 / step),
// the reference's own float product (Axis::bin_num, src/hist.cpp:46-53):
// the nearest integer r of y and its distance d come from the 2^23 shift
// (exact for 0 <= y < 2^22), the bin is floor(y), and *amb is set unless y is
// farther than gy (bins) from r, the only threshold it can be near; NaN and
// infinite y are ambiguous.  Bins at or above n are returned as LUT_INV.
__device__ __forceinline__ unsigned direct_bin(float y, float gy, int n, bool *amb) {
    const float t = y + 8388608.0f;
    const int r = __float_as_int(t) - 0x4B000000;
    const float d = y - (t - 8388608.0f);
    *amb = !(fabsf(d) > gy);
    const int b = r - (d < 0.0f ? 1 : 0);
    return b < n ? (unsigned)b : (unsigned)LUT_INV;
}

// Approximate 1 / sqrt(x) (the MUFU reciprocal square root rsqrtf also
// uses, same error bound) with a subnormal x flushed to zero (+inf out): a
// pair that close has an infinite mu guard and goes to the exact path.
__device__ __forceinline__ float rsqrt_ftz(float x) {
    float r;
    asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}

// JKHists::interp (src/hist.cpp:369-391) of the angular up-weight at
// v = 1 - cos(theta): the interval comes from the host-built thresholds on
// (float)v (the reference's bin_num runs on glibc log1pf), the
// interpolation is the reference's double expression.
__device__ __forceinline__ double upweight(const KParams &P, double v) {
    if (v < P.up_min) return __ldg(P.up_bins);
    if (v > P.up_max) return __ldg(P.up_bins + P.n_up - 1);
    const int c = dev::locate_exact(P.up_thr, P.n_up, __double2float_rn(v));
    if (c < 0) return __ldg(P.up_bins);
    if (c >= P.n_up) return __ldg(P.up_bins + P.n_up - 1);
    const double b0 = __ldg(P.up_bins + c), b1 = __ldg(P.up_bins + c + 1);
    const double c0 = __ldg(P.up_centre + c), c1 = __ldg(P.up_centre + c + 1);
    return __dadd_rn(b0, __ddiv_rn(__dmul_rn(__dsub_rn(b1, b0), __dsub_rn(v, c0)), __dsub_rn(c1, c0)));
}

// Pair weight of the inverse-p kinds from the product of the two grid
// weights (input weights for W_INVP_DD / W_ANG_INVP, weights for
// W_INVP_DR) and the original indices i (catalogue A), j (catalogue B):
//   W_INVP_DD  (iw1 iw2) (float)(interp(1-cos) n_runs / popc)
//              (src/correlators_invpweight.cpp:51-77)
//   W_INVP_DR  (float)((w1 w2) interp(1-cos))         (:184-189)
//   W_ANG_INVP (iw1 iw2) (n_runs / popc), float division (:742-764)
// popc = float sum of the popcounts of mask1 & mask2, plus 1 when zero.
// 32-byte read-only load of four mask words (sm_100 vector load).
__device__ __forceinline__ void ldg_u64x4(const long long *p, unsigned long long &a, unsigned long long &b,
                                          unsigned long long &c, unsigned long long &d) {
    asm("ld.global.nc.v4.u64 {%0, %1, %2, %3}, [%4];" : "=l"(a), "=l"(b), "=l"(c), "=l"(d) : "l"(p));
}

// Sum over the mask words of popc(m1 & m2): exact integer work, read 32 or
// 16 bytes at a time where the rows allow it (a quarter or half of the load
// instructions and L1 requests of word-by-word loads).
__device__ __forceinline__ int and_popc(const long long *m1, const long long *m2, int n, int vec) {
    int c = 0;
    if (vec == 4) {
#pragma unroll 2
        for (int k = 0; k < n; k += 4) {
            unsigned long long a0, a1, a2, a3, b0, b1, b2, b3;
            ldg_u64x4(m1 + k, a0, a1, a2, a3);
            ldg_u64x4(m2 + k, b0, b1, b2, b3);
            c += __popcll(a0 & b0) + __popcll(a1 & b1) + __popcll(a2 & b2) + __popcll(a3 & b3);
        }
    } else if (vec == 2) {
        const longlong2 *a = reinterpret_cast<const longlong2 *>(m1);
        const longlong2 *b = reinterpret_cast<const longlong2 *>(m2);
#pragma unroll 4
        for (int k = 0; k < n / 2; ++k) {
            const longlong2 x = __ldg(a + k), y = __ldg(b + k);
            c += __popcll((unsigned long long)(x.x & y.x)) + __popcll((unsigned long long)(x.y & y.y));
        }
    } else {
        for (int k = 0; k < n; ++k) c += __popcll((unsigned long long)(__ldg(m1 + k) & __ldg(m2 + k)));
    }
    return c;
}

template <int WK>
__device__ __forceinline__ float pair_weight(const KParams &P, const JobK &J, float wprod, int i, int j) {
    auto omct = [&]() {
        const double *u1 = J.a.unit + 3 * (size_t)i, *u2 = J.b.unit + 3 * (size_t)j;
        return omct_exact(u1[0], u1[1], u1[2], u2[0], u2[1], u2[2]);
    };
    if (WK == W_INVP_DR) return __double2float_rn(__dmul_rn((double)wprod, upweight(P, omct())));
    const long long *m1 = P.a_masks + (size_t)i * P.n_mask;
    const long long *m2 = P.b_masks + (size_t)j * P.n_mask;
    const int c = and_popc(m1, m2, P.n_mask, P.mask_vec);
    float pw = (float)c;  // exact: at most 64 * kMaxMaskInts
    if (pw < 0.5f) pw += 1.0f;
    // numerator: n_runs, or with _USE_DITHER_WEIGHTS the same float popcount
    // of the two dither masks (src/correlators_invpweight.cpp:62-71, :749-757)
    float num = P.n_runs_f;
    if (P.dither) {
        const long long *d1 = P.a_dmasks + (size_t)i * P.n_mask;
        const long long *d2 = P.b_dmasks + (size_t)j * P.n_mask;
        const int dc = and_popc(d1, d2, P.n_mask, P.mask_vec);
        num = (float)dc;
        if (num < 0.5f) num += 1.0f;
    }
    if (WK == W_ANG_INVP) return __fmul_rn(wprod, __fdiv_rn(num, pw));
    const float f = __double2float_rn(__ddiv_rn(__dmul_rn(upweight(P, omct()), (double)num), (double)pw));
    return __fmul_rn(wprod, f);
}

// A non-finite pair weight (an up-weight from an empty angular bin) cannot
// go into the fixed-point sums: record it for the bin in the full histogram
// and in the rows of both regions; the host turns the flags into the NaN or
// infinity that double accumulation gives.
__device__ __noinline__ void flag_nonfinite(const KParams &P, int bin, int ra, int rb, float w) {
    const unsigned f = isnan(w) ? 1u : (w > 0 ? 2u : 4u);
    atomicOr(&P.flags[bin], f);
    atomicOr(&P.flags[(size_t)(1 + ra) * P.nb + bin], f);
    if (rb != ra) atomicOr(&P.flags[(size_t)(1 + rb) * P.nb + bin], f);
}

#ifdef TPCF_DEVICE_CHECKS
// Checked build (TPCF_DEVICE_CHECKS): the first index found outside its
// range is recorded in the count's error record (check id, value, limit)
// with the flag kErrCheck, which stops further work items and makes the host
// discard the results and report TPCF_E_DEVICE_CHECK.
__device__ __noinline__ void dcheck_record(int *err, int id, long long v, long long lim) {
    if (atomicCAS(err, 0, kErrCheck) == 0) {
        err[1] = id;
        err[2] = (int)max(min(v, (long long)INT_MAX), (long long)INT_MIN);
        err[3] = (int)max(min(lim, (long long)INT_MAX), (long long)INT_MIN);
    }
}
// True when lo <= v <= hi; else records the failure.
__device__ __forceinline__ bool dcheck(int *err, int id, long long v, long long lo, long long hi) {
    if (v >= lo && v <= hi) return true;
    dcheck_record(err, id, v, hi);
    return false;
}
// Every index a work item and its segments carry, against the bounds of the
// arrays it selects from, before any of its tiles is staged: the item's
// segment range, A chunk, cell and region, and each segment's B run, cell and
// region.  Each thread checks the item and every NT-th segment.
__device__ bool item_in_bounds(const KParams &P, const JobK &J, const WorkItem &it, int tid) {
    int *e = P.err;
    bool ok = dcheck(e, DC_SEGMENTS, it.seg_end, 0, P.n_segs) && dcheck(e, DC_SEGMENTS, it.seg_begin, 0, it.seg_end);
    ok = ok && dcheck(e, DC_A_CHUNK, it.a_len, 0, kChunkA);
    ok = ok && dcheck(e, DC_A_POINTS, it.a_start, 0, J.a.n_pts) &&
         dcheck(e, DC_A_POINTS, (long long)it.a_start + it.a_len, 0, J.a.n_pts);
    ok = ok && dcheck(e, DC_A_CELL, it.a_cell, 0, J.a.n_cells - 1);
    ok = ok && dcheck(e, DC_A_REGION, it.a_region, 0, P.n_jk - 1);
    if (!ok) return false;
    for (int k = it.seg_begin + tid; k < it.seg_end; k += NT) {
        const Segment sg = P.segs[k];
        ok = ok && dcheck(e, DC_B_POINTS, sg.b_len, 0, J.b.n_pts) && dcheck(e, DC_B_POINTS, sg.b_start, 0, J.b.n_pts) &&
             dcheck(e, DC_B_POINTS, (long long)sg.b_start + sg.b_len, 0, J.b.n_pts);
        ok = ok && dcheck(e, DC_B_CELL, sg.b_cell, 0, J.b.n_cells - 1);
        ok = ok && dcheck(e, DC_B_REGION, sg.meta & 0xffff, 0, P.n_jk - 1);
    }
    return ok;
}
#endif

// Add one binned pair: weight from the queue (product of the grid weights)
// or, for the inverse-p kinds, formed here; fixed-point shared add.
template <bool UNITW, int WK, bool WA_SCALED = false>
__device__ __forceinline__ void add_binned(const KParams &P, const JobK &J, const Shm &S, int bin, float wa, float wb,
                                           int ia, int jb, int ka, int jl, int ra, int rb) {
#ifdef TPCF_DEVICE_CHECKS
    if (WK == W_ADJ && !dcheck(P.err, DC_BIN, bin, 0, P.nb - 1)) return;
#endif
    if constexpr (WK == W_ADJ) {
        // the pair adds wa * wb to its bin: dL/dwa += G wb, dL/dwb += G wa
        const double g = S.G[bin];
        dev::acc_add(S.ga_lo, S.ga_hi, ka, __double2ll_rn(g * (double)wb * P.adj_scale));
        dev::acc_add(S.gb_lo, S.gb_hi, jl, __double2ll_rn(g * (double)wa * P.adj_scale));
        return;
    }
#ifdef TPCF_DEVICE_CHECKS
    if (!dcheck(P.err, DC_BIN, bin, 0, P.nb - 1)) return;
#endif
    float w = UNITW ? 1.0f : __fmul_rn(wa, wb);
    if (WK != W_PLAIN) {
        w = pair_weight<WK>(P, J, w, J.a.idx[ia], J.b.idx[jb]);
        if (!isfinite(w)) {
            flag_nonfinite(P, bin, ra, rb, w);
            return;
        }
    }
    const long long q = (UNITW && WK == W_PLAIN) ? 1LL
                        : __float2ll_rn(WA_SCALED ? w : __fmul_rn(w, P.wscale));
    dev::acc_add(S.lo, S.hi, bin, q);
}

// Bin one pair that passed the guard-widened range test, from its FP32
// separation in the B cell's frame: s^2 (the squared chord for angular
// counts), pi from the two unit vectors and the grid-weight product.  The
// pair's positions in the sorted grids (the exact path follows them back to
// the original arrays) come from the queue entry; ra/rb are the regions of
// its two points.
//
// A pair whose table entries leave its bin ambiguous needs the threshold
// search and possibly the exact sequence.  Resolved inline, that rare path
// (well under 1 % of the pairs) would run for the whole warp in every round
// where any lane met such a pair; so the first pass (SLOW = false) returns
// true for it without binning it, the caller parks it in the warp's side
// queue, and a second pass (SLOW = true) over 32 parked pairs at a time
// resolves them.  Returns false otherwise.
template <int MODE, bool UNITW, int WK, bool SLOW>
__device__ __forceinline__ bool bin_fast(const KParams &P, const JobK &J, const PreciseArgs &PA, const ExactArgs &E,
                                         const Shm &S, const float4 *s_pos, const float4 *s_aux,
                                         const float4 *s_achunk, const float4 e, int a_start, int jbase, int ra,
                                         int rb, Counters &cnt) {
    // queue entry: (dx, dy, dz, A chunk index << kTileShift | tile index)
    const int pk = __float_as_int(e.w);
    const int ka = pk >> kTileShift, jl = pk & kTileMask;
    const int ia = a_start + ka, jb = jbase + jl;
    const float dx = e.x, dy = e.y, dz = e.z;
    const float s2 = fmaf(dz, dz, fmaf(dy, dy, dx * dx));  // as in the candidate test
    const float4 qa = s_achunk[ka];
    const float wa = qa.w;
    float wb, pi = 0.f;
    if constexpr (MODE == MODE_SIGMA_PI || MODE == MODE_S_MU) {
        const float4 ab = s_aux[jl];  // half the unit vector and the weight of the B point
        wb = ab.w;
        pi = fmaf(dz, qa.z + ab.z, fmaf(dy, qa.y + ab.y, dx * (qa.x + ab.x)));  // halved unit vectors
    } else {
        wb = s_pos[jl].w;
    }
    int bin;
    bool amb;
    if constexpr (MODE == MODE_ANGULAR) {
        // v = |n1 - n2|^2 / 2 approximates 1 - cos(theta) within g_ang
        const float v = 0.5f * s2;
        bool amb1;
        const unsigned c1 =
            lut_decode(S.l1[lut1_index(P.lut1_base, P.lut1_shift, P.lut1_n, v)], v, S.t1, P.g_ang, P.lut_edge1, &amb1);
        if (c1 == LUT_INV) return false;
        if (!amb1) {
            cnt.in_range += 1;
            bin = (int)c1;
        } else {
            if constexpr (!SLOW) return true;
            const dev::AxisK ax1{S.t1, P.n1, 0, 0.f, 0.f, 0.f, 0.f};
            int b = dev::locate_exact(S.t1, P.n1, v);
            bool inr;
            if (dev::near_edge(ax1, v, b, P.g_ang)) {
                cnt.guard += 1;
                b = exact_pair<MODE_ANGULAR>(E, S.t1, S.t2, J.a.idx[ia], J.b.idx[jb], &inr);
            } else {
                inr = b >= 0 && b < P.n1;
            }
            cnt.in_range += inr ? 1 : 0;
            if (!inr) return false;
            bin = b;
        }
        add_binned<UNITW, WK, WK == W_PLAIN>(P, J, S, bin, wa, wb, ia, jb, ka, jl, ra, rb);
        return false;
    } else {
        if (MODE == MODE_SIGMA_PI) {
            if (s2 >= P.max_r_sq + P.g_s2 || s2 <= P.min_r_sq - P.g_s2) return false;  // certainly out of range
            amb = (fabsf(s2 - P.max_r_sq) <= P.g_s2) || (fabsf(s2 - P.min_r_sq) <= P.g_s2);
            const float a = fmaf(-pi, pi, s2);
            const float api = fabsf(pi);
            bool amb1, amb2;
            unsigned c1 =
                lut_decode(S.l1[lut1_index(P.lut1_base, P.lut1_shift, P.lut1_n, a)], a, S.t1, P.g_a, P.lut_edge1, &amb1);
            if (a <= P.g_a) {
                c1 = LUT_AMB;
                amb1 = true;
            }
            if (a < -P.g_a) {
                c1 = LUT_INV;  // sqrtf(negative) is NaN: never binned
                amb1 = false;
            }
            const unsigned c2 = P.direct2 ? direct_bin(api * P.inv2, P.k2, P.n2, &amb2)
                                          : lut_decode(S.l2[lut2_index(P.lut2_scale, api)], api, S.t2, P.g_pi,
                                                       P.lut_edge2, &amb2);
            if (!amb && ((c1 == LUT_INV && !amb1) || (c2 == LUT_INV && !amb2))) {
                cnt.in_range += 1;
                return false;
            }
            amb = amb || amb1 || amb2 || c1 == LUT_INV || c2 == LUT_INV;
            if (!amb) cnt.in_range += 1;
            bin = (int)(c1 * P.n2 + c2);
        } else {
            // both table lookups first: the two load chains overlap
            // s^2 passed the candidate test, so it lies below the table's top
            const unsigned raw1 = S.l1[max((int)((__float_as_uint(s2) >> P.lut1_shift) - P.lut1_base), 0)];
            unsigned raw2 = 0;
            float mu = 0.f, gmu = 0.f;
            if (MODE == MODE_S_MU && P.direct2) {
                // mu binned directly, its guard taken in bins
                const float inv_s = rsqrt_ftz(s2);
                bool amb2;
                const unsigned c2 = direct_bin(fabsf(pi) * inv_s * P.inv2,
                                               fmaf(P.c2y * inv_s, inv_s, fmaf(P.c1y, inv_s, P.g0y)), P.n2, &amb2);
                // a plain bin (the common case) needs no decoding
                unsigned c1 = raw1;
                amb = false;
                if (raw1 >= LUT_EDGE) {
                    c1 = lut_decode(raw1, s2, S.t1, P.g_s2, P.lut_edge1, &amb);
                    if (c1 == LUT_INV) {
                        cnt.in_range += (s2 < P.max_r_sq && s2 > P.min_r_sq) ? 1 : 0;
                        return false;
                    }
                }
                if (amb || amb2 || c2 == LUT_INV) {
                    // rare: ambiguous, or mu certainly beyond the last bin
                    if (!amb && !amb2) {
                        cnt.in_range += 1;
                        return false;
                    }
                    amb = true;
                } else {
                    cnt.in_range += 1;
                }
                bin = (int)(c1 * P.n2 + c2);
                goto binned;
            }
            if (MODE == MODE_S_MU) {
                const float inv_s = rsqrtf(s2);
                mu = fabsf(pi) * inv_s;
                gmu = fmaf(P.c2_mu * inv_s, inv_s, fmaf(P.c1_mu, inv_s, P.g_mu0));
                raw2 = S.l2[lut2_index(P.lut2_scale, mu)];
            }
            const unsigned c1 = lut_decode(raw1, s2, S.t1, P.g_s2, P.lut_edge1, &amb);
            bool amb2 = false;
            unsigned c2 = 0;
            if (MODE == MODE_S_MU) c2 = lut_decode(raw2, mu, S.t2, gmu, P.lut_edge2, &amb2);
            if (c1 == LUT_INV) {
                // certainly outside the range or the bins; the range status is
                // the same for every value of the widened bucket
                cnt.in_range += (s2 < P.max_r_sq && s2 > P.min_r_sq) ? 1 : 0;
                return false;
            }
            if (MODE == MODE_S_MU) {
                if (c2 == LUT_INV && !amb2 && !amb && s2 >= P.s2_lut_min) {
                    cnt.in_range += 1;
                    return false;
                }
                amb = amb || amb2 || c2 == LUT_INV || s2 < P.s2_lut_min;
            }
            if (!amb) cnt.in_range += 1;
            bin = (int)(MODE == MODE_S_MU ? c1 * P.n2 + c2 : c1);
        }
    binned:
        if (amb) {
            if constexpr (!SLOW) return true;
            bool inr, guarded;
            bin = precise_bin<MODE>(PA, E, S.t1, S.t2, s2, pi, J.a.idx[ia], J.b.idx[jb], &inr, &guarded);
            cnt.in_range += inr ? 1 : 0;
            cnt.guard += guarded ? 1 : 0;
            if (bin < 0) return false;
        }
        add_binned<UNITW, WK, WK == W_PLAIN>(P, J, S, bin, wa, wb, ia, jb, ka, jl, ra, rb);
        return false;
    }
}

// Bin one pair of the plain FP64 path: from its exact separation (d0, d1,
// d2), or for angular counts from its exact (float)(1 - cos(theta)) in d0;
// ia/jb are its positions in the sorted grids.
template <int MODE, bool UNITW, int WK>
__device__ __forceinline__ void bin_exact(const KParams &P, const JobK &J, const ExactArgs &E, const Shm &S, float d0,
                                          float d1,
                                          float d2, int ia, int jb, int ka, int jl, int ra, int rb, Counters &cnt) {
    int bin;
    if constexpr (MODE == MODE_ANGULAR) {
        bin = dev::locate_exact(S.t1, P.n1, d0);  // in [0, n1): the candidate test checked it
        cnt.in_range += 1;
    } else {
        double n1x = 0, n1y = 0, n1z = 0, n2x = 0, n2y = 0, n2z = 0;
        if (MODE != MODE_MONOPOLE) {
            const double4 u1 = J.a.unit_s[ia];
            const double4 u2 = J.b.unit_s[jb];
            n1x = u1.x;
            n1y = u1.y;
            n1z = u1.z;
            n2x = u2.x;
            n2y = u2.y;
            n2z = u2.z;
        }
        if (MODE != MODE_MONOPOLE && P.los_mid) {
            const double4 x1 = J.a.xyz_s[ia];
            const double4 x2 = J.b.xyz_s[jb];
            n1x = x1.x;
            n1y = x1.y;
            n1z = x1.z;
            n2x = x2.x;
            n2y = x2.y;
            n2z = x2.z;
        }
        bool inr;
        bin = exact_bin<MODE>(E, S.t1, S.t2, d0, d1, d2, n1x, n1y, n1z, n2x, n2y, n2z, &inr,
                              MODE != MODE_MONOPOLE && P.los_mid);
        cnt.in_range += inr ? 1 : 0;
        if (bin < 0) return;
    }
    const float wa = (float)J.a.xyz_s[ia].w, wb = (float)J.b.xyz_s[jb].w;
    add_binned<UNITW, WK>(P, J, S, bin, wa, wb, ia, jb, ka, jl, ra, rb);
}


// Add a 64-bit value held as two 32-bit words into another such pair (the
// caller owns the bin: no atomics).
__device__ __forceinline__ void add64_owned(uint32_t *lo, uint32_t *hi, int i, unsigned long long v) {
    const uint32_t vl = (uint32_t)v, vh = (uint32_t)(v >> 32);
    const uint32_t old = lo[i];
    lo[i] = old + vl;
    hi[i] = hi[i] + vh + ((old + vl) < old ? 1u : 0u);
}

template <int MODE, bool UNITW, bool JK, bool EXACT, int WK, int CFG = 0>
__global__ void __launch_bounds__(NT, (JK || CFG == 1) ? 2 : 3) pair_count_kernel(const KParams P) {
    extern __shared__ __align__(128) unsigned char smem[];
    constexpr bool kNeedAux = (MODE == MODE_SIGMA_PI || MODE == MODE_S_MU);
    constexpr bool ADJ = (WK == W_ADJ);
    constexpr int TBK = tile_points(EXACT, JK, ADJ, CFG);                     // B points per tile
    constexpr int NB = n_buffers(EXACT, JK, ADJ, CFG);                        // tile buffers
    constexpr int QPF = light_fast(EXACT, JK, ADJ, CFG) ? QPUSH_NOJK : QPUSH;  // FP32 path push width
    const bool need_lut2 = kNeedAux && !P.direct2;
    const SmemLayout L = smem_layout(P.nb, P.n1, P.n2, EXACT, JK, ADJ, CFG, need_lut2);
    uint32_t *s_lo = (uint32_t *)(smem + L.lo);
    uint32_t *s_hi = (uint32_t *)(smem + L.hi);
    uint32_t *s_alo = (uint32_t *)(smem + L.alo);
    uint32_t *s_ahi = (uint32_t *)(smem + L.ahi);
    float *s_t1 = (float *)(smem + L.t1);
    float *s_t2 = (float *)(smem + L.t2);
    unsigned char *s_l1 = smem + L.lut1;
    unsigned char *s_l2 = smem + L.lut2;
    unsigned char *const tile_base = smem + L.tile0;
    const size_t tile_stride = L.tile1 - L.tile0;
    float4 *s_achunk = (float4 *)(smem + L.achunk);
    int *s_item = (int *)(smem + L.misc);
    uint64_t *bar = (uint64_t *)(smem + L.misc + 16);                  // one per tile buffer
    unsigned *s_done = (unsigned *)(smem + L.misc + 16 + 8 * kNbufMax);  // warps done with each buffer (running count)
    JobK *s_job = (JobK *)(smem + L.misc + 64);
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    constexpr int QCAP = queue_cap(EXACT, JK, ADJ, CFG);  // entries of each warp's queue
    float4 *s_q = (float4 *)(smem + L.queue) + warp * QCAP;
    int *s_slow = (int *)(smem + L.slow) + warp * kSlowCap;
    const unsigned lt_mask = (1u << lane) - 1u;
    const Shm S{s_t1, s_t2, s_l1, s_l2, s_lo, s_hi, (const double *)(smem + L.lo),
                (uint32_t *)(smem + L.ga), (uint32_t *)(smem + L.ga) + TA,
                (uint32_t *)(smem + L.gb), (uint32_t *)(smem + L.gb) + TB};

    if (ADJ) {
        // the histogram words hold dL/d(full histogram) instead
        for (int i = tid; i < P.nb; i += NT) ((double *)(smem + L.lo))[i] = P.adj_G[i];
        for (int i = tid; i < TA; i += NT) S.ga_lo[i] = S.ga_hi[i] = 0u;
        for (int i = tid; i < TB; i += NT) S.gb_lo[i] = S.gb_hi[i] = 0u;
    } else {
        for (int i = tid; i < P.nb; i += NT) {
            s_lo[i] = 0;
            s_hi[i] = 0;
            if (JK) {
                s_alo[i] = 0;
                s_ahi[i] = 0;
            }
        }
    }
    for (int i = tid; i <= P.n1; i += NT) s_t1[i] = P.t1g[i];
    for (int i = tid; i <= P.n2; i += NT) s_t2[i] = P.t2g[i];
    for (int i = tid; i < P.lut1_n; i += NT) s_l1[i] = P.lut1g[i];
    if (need_lut2)
        for (int i = tid; i < LUT2_N; i += NT) s_l2[i] = P.lut2g[i];
    if (tid == 0) {
        for (int b = 0; b < NB; ++b) {
            dev::mbar_init(&bar[b], 1);
            s_done[b] = 0;
        }
        dev::mbar_init_fence();
    }
    __syncthreads();

    const PreciseArgs PA{P.n1, P.n2, P.min_r_sq, P.max_r_sq, P.g_s2, P.g_pi, P.g_a, P.c1_mu, P.c2_mu, P.g_mu0};
    Counters cnt;
    unsigned long long n_cand = 0, n_flush = 0, tot_in = 0, tot_guard = 0;
    unsigned tcount = 0;  // tiles staged so far by this CTA (selects buffer and phase)

    for (;;) {
        if (tid == 0) {
            int item = atomicAdd(P.head, 1);
            if (*(volatile int *)P.err != 0) item = P.n_items;
            s_item[0] = item;
        }
        __syncthreads();
        const int item = s_item[0];
        if (item >= P.n_items) break;
        const WorkItem it = P.items[item];
#ifdef TPCF_DEVICE_CHECKS
        // a barrier before skipping: every thread has read the item index
        if (__syncthreads_or(JK && !dcheck(P.err, DC_JOB, it.job, 0, P.n_jobs - 1))) continue;
#endif
        if constexpr (JK) {
            // the item's job (grids and output slot), staged for every thread
            const int *src = (const int *)(P.jobs + it.job);
            int *dst = (int *)s_job;
            for (int k = tid; k < (int)(sizeof(JobK) / 4); k += NT) dst[k] = src[k];
            __syncthreads();
        }
        const JobK &J = JK ? *s_job : P.job0;
#ifdef TPCF_DEVICE_CHECKS
        if (__syncthreads_or(!item_in_bounds(P, J, it, tid))) continue;
#endif
        const ExactArgs EA{J.a.xyz, J.a.unit, J.b.xyz, J.b.unit, P.min_r_sq, P.max_r_sq, P.n1, P.n2, P.los_mid};
    auto issue = [&](unsigned tc, int start, int len) {
        const unsigned buf = tc % NB;
        unsigned char *dst = tile_base + buf * tile_stride;
        dev::fence_proxy_async();
        if (EXACT) {
            const uint32_t by = (uint32_t)len * 32u;
            dev::mbar_expect_tx(&bar[buf], by);
            dev::bulk_g2s(dst, J.b.xyz_s + start, by, &bar[buf]);
        } else {
            const uint32_t by = (uint32_t)len * 16u;
            dev::mbar_expect_tx(&bar[buf], kNeedAux ? 2 * by : by);
            dev::bulk_g2s(dst, J.b.pos + start, by, &bar[buf]);
            if (kNeedAux) dev::bulk_g2s(dst + (size_t)TBK * 16, J.b.aux + start, by, &bar[buf]);
        }
    };

        tot_in += cnt.in_range;
        tot_guard += cnt.guard;
        cnt.in_range = cnt.guard = 0;

        // ---- phase mapping: Pn groups of G threads; each group holds the
        // whole A chunk (G * R slots) and takes every Pn-th B point, so short
        // runs still occupy every thread
        int Pn = min(32, max(1, TA / max(it.a_len, 1)));
        while (Pn > 1 && (NT / Pn) * R < it.a_len) --Pn;
        const int G = NT / Pn;
        const int grp = tid / G, loc = tid - grp * G;
        const bool thr_on = grp < Pn;

        // ---- A points: validity and indices; FP32 coordinates are
        // (re)loaded per segment in that segment's cell frame
        const int3 ca = J.a.coord[it.a_cell];
        double dax[R], day[R], daz[R];
        int ai[R], apack[R];
#pragma unroll
        for (int r = 0; r < R; ++r) {
            const int k = loc + r * G;
            const bool valid = thr_on && k < it.a_len;
            const int gi = it.a_start + k;
            apack[r] = k << kTileShift;  // queue entry: A chunk index << kTileShift | tile index
            ai[r] = valid ? gi : 0x7fffffff;
            dax[r] = day[r] = daz[r] = 1e300;
            if (EXACT && valid) {
                const double4 p = J.a.xyz_s[gi];
                dax[r] = p.x;
                day[r] = p.y;
                daz[r] = p.z;
            }
        }

        if (!EXACT) {
            // half the unit vector and the weight of every A point of the
            // chunk, read by the consume step (pi, pair weight) at full warp
            // occupancy
            for (int k = tid; k < it.a_len; k += NT) {
                const int gi = it.a_start + k;
                // plain weights: the A weight times the fixed-point scale 2^S
                // (exact), so the pair's fixed-point value is one product
                const float wk = (WK == W_PLAIN && !UNITW) ? J.a.pos[gi].w * P.wscale : J.a.pos[gi].w;
                if (kNeedAux) {
                    const float4 q = J.a.aux[gi];
                    s_achunk[k] = make_float4(q.x, q.y, q.z, wk);
                } else {
                    s_achunk[k] = make_float4(0.f, 0.f, 0.f, wk);
                }
            }
            __syncthreads();
        }
        // The item's tiles in order: (segment, tile within it).  Tiles 0 to
        // NB - 1 are staged here; each later tile by the last warp to
        // finish the tile NB before it, so no warp waits for the others
        // between tiles.
        auto tile_next = [&](int &psi, int &pt) -> bool {
            if (pt + 1 < (P.segs[psi].b_len + TBK - 1) / TBK) {
                ++pt;
                return true;
            }
            if (psi + 1 < it.seg_end) {
                ++psi;
                pt = 0;
                return true;
            }
            return false;
        };
        auto issue_at = [&](unsigned tc, int psi, int pt) {
            const Segment sx = P.segs[psi];
            const int st = pt * TBK;
            issue(tc, sx.b_start + st, min(TBK, sx.b_len - st));
        };
        if (tid == 0) {
            int psi = it.seg_begin, pt = 0;
            issue_at(tcount, psi, pt);
            for (int b = 1; b < NB && tile_next(psi, pt); ++b) issue_at(tcount + b, psi, pt);
        }
        for (int si = it.seg_begin; si < it.seg_end; ++si) {
            const Segment sg = P.segs[si];
            const int rb = sg.meta & 0xffff;
            const bool self = (sg.meta >> 16) != 0;
            if (tid == 0) {
                const long long al = it.a_len, bl = sg.b_len;
                n_cand += self ? (unsigned long long)(al * bl - al * (al + 1) / 2) : (unsigned long long)(al * bl);
            }
            // A coordinates in the frame of this segment's cell
            const int3 cb = J.b.coord[sg.b_cell];
            const float offx = (float)((double)((J.a.kmin0 + ca.x) - (J.b.kmin0 + cb.x)) * P.side);
            const float offy = (float)((double)((J.a.kmin1 + ca.y) - (J.b.kmin1 + cb.y)) * P.side);
            const float offz = (float)((double)((J.a.kmin2 + ca.z) - (J.b.kmin2 + cb.z)) * P.side);
            float ax[R], ay[R], az[R];
#pragma unroll
            for (int r = 0; r < R; ++r) {
                // slots without a point sit far away: their s^2 overflows to
                // +inf and never passes the candidate test
                ax[r] = ay[r] = az[r] = 1e30f;
                if (!EXACT && ai[r] != 0x7fffffff) {
                    const float4 p = J.a.pos[ai[r]];
                    ax[r] = p.x + offx;
                    ay[r] = p.y + offy;
                    az[r] = p.z + offz;
                }
            }
            const int ntiles = (sg.b_len + TBK - 1) / TBK;
            for (int t = 0; t < ntiles; ++t) {
                const int tstart = t * TBK;
                const int tlen = min(TBK, sg.b_len - tstart);
                if (!dev::mbar_wait_bounded(&bar[tcount % NB], (tcount / NB) & 1u, kWaitLimit) || P.force_timeout) {
                    atomicCAS(P.err, 0, kErrTimeout);  // device timeout: results are discarded by the host
                }
                const int jbase = sg.b_start + tstart;
                const int nsteps = (tlen + Pn - 1) / Pn;
                // Candidates that pass the (guard-widened) range test are
                // pushed into the warp's queue with a ballot; each time 32 are
                // queued the whole warp bins them (no divergent binning).
                int qn = 0;  // queued entries of this warp (warp-uniform)
                if (EXACT) {
                    const double4 *s_xyz = (const double4 *)(tile_base + (tcount % NB) * tile_stride);
                    for (int m = 0; m < nsteps; ++m) {
                        const int jj = grp + m * Pn;
                        const bool jv = thr_on && jj < tlen;
                        const double4 pb = s_xyz[min(jj, tlen - 1)];
                        const int jg = jbase + jj;
                        float d0[R], d1[R], d2[R];
                        bool hit[R];
#pragma unroll
                        for (int r = 0; r < R; ++r) {
                            if (MODE == MODE_ANGULAR) {
                                // tiles hold unit vectors: the binned value itself
                                d0[r] = __double2float_rn(omct_exact(dax[r], day[r], daz[r], pb.x, pb.y, pb.z));
                                d1[r] = d2[r] = 0.0f;
                                hit[r] = jv && (d0[r] >= s_t1[0]) && (d0[r] < s_t1[P.n1]) && (!self || jg > ai[r]);
                            } else {
                                d0[r] = __double2float_rn(__dsub_rn(dax[r], pb.x));
                                d1[r] = __double2float_rn(__dsub_rn(day[r], pb.y));
                                d2[r] = __double2float_rn(__dsub_rn(daz[r], pb.z));
                                const float s2 = __fadd_rn(
                                    __fadd_rn(__fmul_rn(d0[r], d0[r]), __fmul_rn(d1[r], d1[r])), __fmul_rn(d2[r], d2[r]));
                                hit[r] = jv && (s2 < P.max_r_sq) && (s2 > P.min_r_sq) && (!self || jg > ai[r]);
                            }
                        }
                        constexpr int QPX = qpush_exact(MODE);
#pragma unroll
                        for (int r0 = 0; r0 < R; r0 += QPX) {
                            // at most 31 + 32 * QPX entries: within the queue
#pragma unroll
                            for (int r = r0; r < r0 + QPX; ++r) {
                                const unsigned bal = __ballot_sync(0xffffffffu, hit[r]);
#ifdef TPCF_DEVICE_CHECKS
                                if (!dcheck(P.err, DC_QUEUE, qn + __popc(bal), 0, QCAP)) continue;
#endif
                                if (hit[r])
                                    s_q[qn + __popc(bal & lt_mask)] =
                                        make_float4(d0[r], d1[r], d2[r], __int_as_float(apack[r] | jj));
                                qn += __popc(bal);
                            }
                            while (qn >= 32) {
                                __syncwarp();
                                const float4 e = s_q[qn - 32 + lane];
                                const int pk = __float_as_int(e.w);
                                bin_exact<MODE, UNITW, WK>(P, J, EA, S, e.x, e.y, e.z, it.a_start + (pk >> kTileShift),
                                                           jbase + (pk & kTileMask), pk >> kTileShift, pk & kTileMask,
                                                           it.a_region, rb,
                                                           cnt);
                                __syncwarp();
                                qn -= 32;
                            }
                        }
                    }
                    if (qn > 0) {
                        __syncwarp();
                        if (lane < qn) {
                            const float4 e = s_q[lane];
                            const int pk = __float_as_int(e.w);
                            bin_exact<MODE, UNITW, WK>(P, J, EA, S, e.x, e.y, e.z, it.a_start + (pk >> kTileShift),
                                                       jbase + (pk & kTileMask), pk >> kTileShift, pk & kTileMask,
                                                       it.a_region, rb, cnt);
                        }
                        __syncwarp();
                    }
                } else {
                    const unsigned char *tile = tile_base + (tcount % NB) * tile_stride;
                    const float4 *s_pos = (const float4 *)tile;
                    const float4 *s_aux = (const float4 *)(tile + (size_t)TBK * 16);
                    int ns = 0;  // parked entries of this warp (warp-uniform)
                    // every lane of the warp calls park: a deferred pair's
                    // packed indices go to the side queue
                    auto park = [&](bool dfr, const float4 &e) {
                        const unsigned bd = __ballot_sync(0xffffffffu, dfr);
#ifdef TPCF_DEVICE_CHECKS
                        if (!dcheck(P.err, DC_SIDE_QUEUE, ns + __popc(bd), 0, kSlowCap)) return;
#endif
                        if (bd) {
                            if (dfr) s_slow[ns + __popc(bd & lt_mask)] = __float_as_int(e.w);
                            ns += __popc(bd);
                        }
                    };
                    // second pass over a parked pair: its separation again,
                    // from the A point (global) in this segment's frame and
                    // the B point of the tile, by the candidate loop's own
                    // operations, so bit for bit the value it was queued with
                    auto resolve = [&](int pk) {
                        const int ka = pk >> kTileShift, jl = pk & kTileMask;
                        const float4 pa = J.a.pos[it.a_start + ka];
                        const float4 pb = s_pos[jl];
                        const float ax0 = pa.x + offx, ay0 = pa.y + offy, az0 = pa.z + offz;
                        const float4 e = make_float4(ax0 - pb.x, ay0 - pb.y, az0 - pb.z, __int_as_float(pk));
                        bin_fast<MODE, UNITW, WK, true>(P, J, PA, EA, S, s_pos, s_aux, s_achunk, e, it.a_start, jbase,
                                                        it.a_region, rb, cnt);
                    };
                    // Candidates: (dx, dy, dz) of the pair in the segment's cell
                    // frame; those inside the guard-widened range are pushed
                    // into the warp's queue with a ballot, and each time 32 are
                    // queued the whole warp bins them (pi, weight, tables) at
                    // full occupancy.  Self segments (auto counts) keep j > i.
                    auto run = [&](auto self_c, auto one_c) {
                        constexpr bool SELF = decltype(self_c)::value;
                        constexpr bool ONE = decltype(one_c)::value;  // one group: B point m at step m
                        for (int m = 0; m < nsteps; ++m) {
                            const int jj = ONE ? m : grp + m * Pn;
                            const float4 pb = s_pos[ONE ? jj : min(jj, tlen - 1)];
                            const bool jv = ONE || jj < tlen;
                            const int jg = jbase + jj;
                            float dx[R], dy[R], dz[R];
                            bool hit[R];
#pragma unroll
                            for (int r = 0; r < R; ++r) {
                                dx[r] = ax[r] - pb.x;
                                dy[r] = ay[r] - pb.y;
                                dz[r] = az[r] - pb.z;
                                const float s2 = fmaf(dz[r], dz[r], fmaf(dy[r], dy[r], dx[r] * dx[r]));
                                hit[r] = jv && s2 < P.s2_test;
                                if (SELF) hit[r] = hit[r] && jg > ai[r];
                            }
#pragma unroll
                            for (int r0 = 0; r0 < R; r0 += QPF) {
#pragma unroll
                                for (int r = r0; r < r0 + QPF; ++r) {
                                    const unsigned bal = __ballot_sync(0xffffffffu, hit[r]);
#ifdef TPCF_DEVICE_CHECKS
                                    if (!dcheck(P.err, DC_QUEUE, qn + __popc(bal), 0, QCAP)) continue;
#endif
                                    if (hit[r])
                                        s_q[qn + __popc(bal & lt_mask)] =
                                            make_float4(dx[r], dy[r], dz[r], __int_as_float(apack[r] | jj));
                                    qn += __popc(bal);
                                }
                                while (qn >= 32) {
                                    __syncwarp();
                                    const float4 e = s_q[qn - 32 + lane];
                                    park(bin_fast<MODE, UNITW, WK, false>(P, J, PA, EA, S, s_pos, s_aux, s_achunk, e,
                                                                          it.a_start, jbase, it.a_region, rb, cnt),
                                         e);
                                    if (ns >= 32) {
                                        __syncwarp();
                                        resolve(s_slow[ns - 32 + lane]);
                                        ns -= 32;
                                    }
                                    __syncwarp();
                                    qn -= 32;
                                }
                            }
                        }
                    };
                    if (Pn == 1) {
                        if (self) run(std::true_type{}, std::true_type{});
                        else run(std::false_type{}, std::true_type{});
                    } else {
                        if (self) run(std::true_type{}, std::false_type{});
                        else run(std::false_type{}, std::false_type{});
                    }
                    // drain: the queued and parked entries refer to this
                    // tile's positions
                    if (qn > 0) {
                        __syncwarp();
                        bool dfr = false;
                        float4 e = make_float4(0.f, 0.f, 0.f, 0.f);
                        if (lane < qn) {
                            e = s_q[lane];
                            dfr = bin_fast<MODE, UNITW, WK, false>(P, J, PA, EA, S, s_pos, s_aux, s_achunk, e,
                                                                   it.a_start, jbase, it.a_region, rb, cnt);
                        }
                        park(dfr, e);
                        __syncwarp();
                    }
                    while (ns > 0) {
                        __syncwarp();
                        if (lane < ns) resolve(s_slow[ns > 32 ? ns - 32 + lane : lane]);
                        ns = ns > 32 ? ns - 32 : 0;
                    }
                    __syncwarp();
                }
                // This warp is done with the buffer: the last warp to finish it
                // refills it with the tile NB ahead (the arrivals of one tile
                // all precede those of the next tile in the same buffer, whose
                // data comes only after them).
                __syncwarp();
                if (lane == 0) {
                    __threadfence_block();
                    const unsigned done = atomicAdd(&s_done[tcount % NB], 1u);
                    if (done % NWARP == NWARP - 1) {
                        __threadfence_block();
                        int psi = si, pt = t;
                        bool more = true;
                        for (int b = 0; b < NB && more; ++b) more = tile_next(psi, pt);
                        if (more) issue_at(tcount + NB, psi, pt);
                    }
                }
                if constexpr (ADJ) {
                    // this tile's B gradients to their points
                    __syncthreads();
                    const int jb0 = sg.b_start + tstart;
                    for (int t2 = tid; t2 < tlen; t2 += NT) {
                        const long long q = (long long)(((unsigned long long)S.gb_hi[t2] << 32) | S.gb_lo[t2]);
                        if (q != 0) atomicAdd(&P.grad_b[J.b.idx[jb0 + t2]], (double)q * P.adj_inv);
                        S.gb_lo[t2] = S.gb_hi[t2] = 0u;
                    }
                    __syncthreads();
                }
                ++tcount;
            }
            // ---- jackknife: a region's pairs (JKHists::add_pair,
            // src/hist.cpp:246-260) go to its row once per run of equal
            // regions, and into the item's A-side total
            if (JK) {
                const bool last = (si + 1 == it.seg_end) || ((P.segs[si + 1].meta & 0xffff) != rb);
                if (last) {
                    __syncthreads();  // every warp's pairs of this region are in the histogram
                    for (int b = tid; b < P.nb; b += NT) {
                        const unsigned long long v = ((unsigned long long)s_hi[b] << 32) | s_lo[b];
                        if (!v) continue;
                        add64_owned(s_alo, s_ahi, b, v);
                        if (rb != it.a_region) dev::acc_add_global(P.g_sub, ((size_t)J.out * P.n_jk + rb) * P.nb + b, v);
                        s_lo[b] = 0;
                        s_hi[b] = 0;
                    }
                    ++n_flush;
                    __syncthreads();
                }
            }
        }
        // ---- jackknife: the item's total goes to the full histogram and to
        // the A region's row
        if (JK) {
            for (int b = tid; b < P.nb; b += NT) {
                const unsigned long long v = ((unsigned long long)s_ahi[b] << 32) | s_alo[b];
                if (!v) continue;
                dev::acc_add_global(P.g_full, (size_t)J.out * P.nb + b, v);
                dev::acc_add_global(P.g_sub, ((size_t)J.out * P.n_jk + it.a_region) * P.nb + b, v);
                s_alo[b] = 0;
                s_ahi[b] = 0;
            }
            __syncthreads();
        }
        // ---- adjoint: the A chunk's gradients to their points
        if constexpr (ADJ) {
            for (int k = tid; k < it.a_len; k += NT) {
                const long long q = (long long)(((unsigned long long)S.ga_hi[k] << 32) | S.ga_lo[k]);
                if (q != 0) atomicAdd(&P.grad_a[J.a.idx[it.a_start + k]], (double)q * P.adj_inv);
                S.ga_lo[k] = S.ga_hi[k] = 0u;
            }
            __syncthreads();
        }
    }

    // ---- a copy can still be in flight only after a wait gave up (the
    // results are discarded then): give the last copy into each buffer a
    // bounded wait before the CTA's shared memory is released
    if (tid == 0) {
        for (unsigned b = 0; b < (unsigned)NB && b < tcount; ++b) {
            const unsigned t_last = (tcount - 1) - ((tcount - 1 - b) % NB);  // last tile staged in buffer b
            dev::mbar_wait_bounded(&bar[b], (t_last / NB) & 1u, kWaitLimit);
        }
    }

    // ---- merge the privatised histogram
    __syncthreads();
    if (!JK && !ADJ) {
        for (int b = tid; b < P.nb; b += NT) {
            const unsigned long long v = ((unsigned long long)s_hi[b] << 32) | s_lo[b];
            if (v) dev::acc_add_global(P.g_full, b, v);
        }
    }
    // ---- counters
    unsigned long long v0 = tot_in + cnt.in_range, v1 = tot_guard + cnt.guard;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        v0 += __shfl_down_sync(0xffffffffu, v0, o);
        v1 += __shfl_down_sync(0xffffffffu, v1, o);
    }
    if ((tid & 31) == 0) {
        atomicAdd(&P.counters[1], v0);
        atomicAdd(&P.counters[2], v1);
    }
    if (tid == 0) {
        atomicAdd(&P.counters[0], n_cand);
        atomicAdd(&P.counters[3], n_flush);
    }
}

typedef void (*KernelFn)(const KParams);

template <int MODE, int WK>
KernelFn pick_kernel(bool unitw, bool jk, bool exact, int cfg = 0) {
    if constexpr (WK == W_ADJ) {  // no regions, per-point weights
        return exact ? pair_count_kernel<MODE, false, false, true, WK> : pair_count_kernel<MODE, false, false, false, WK>;
    } else {
        if constexpr (WK == W_PLAIN) {
            // the alternative configuration (plain-weight FP32+guard kernels)
            if (cfg == 1 && !exact) {
                if (unitw)
                    return jk ? pair_count_kernel<MODE, true, true, false, WK, 1>
                              : pair_count_kernel<MODE, true, false, false, WK, 1>;
                return jk ? pair_count_kernel<MODE, false, true, false, WK, 1>
                          : pair_count_kernel<MODE, false, false, false, WK, 1>;
            }
            if (unitw) {
                if (exact)
                    return jk ? pair_count_kernel<MODE, true, true, true, WK>
                              : pair_count_kernel<MODE, true, false, true, WK>;
                return jk ? pair_count_kernel<MODE, true, true, false, WK>
                          : pair_count_kernel<MODE, true, false, false, WK>;
            }
        }
        if (exact)
            return jk ? pair_count_kernel<MODE, false, true, true, WK> : pair_count_kernel<MODE, false, false, true, WK>;
        return jk ? pair_count_kernel<MODE, false, true, false, WK> : pair_count_kernel<MODE, false, false, false, WK>;
    }
}

template <int MODE>
KernelFn pick_3d(int wk, bool unitw, bool jk, bool exact, int cfg) {
    switch (wk) {
    case W_INVP_DD: return pick_kernel<MODE, W_INVP_DD>(unitw, jk, exact);
    case W_INVP_DR: return pick_kernel<MODE, W_INVP_DR>(unitw, jk, exact);
    case W_ADJ: return pick_kernel<MODE, W_ADJ>(unitw, jk, exact);
    default: return pick_kernel<MODE, W_PLAIN>(unitw, jk, exact, cfg);
    }
}

// Kernel for a mode, weight kind (W_PLAIN, W_INVP_DD, W_INVP_DR for 3-D;
// W_PLAIN, W_ANG_INVP for angular), unit weights, jackknife and precision.
KernelFn pick(int mode, int wk, bool unitw, bool jk, bool exact, int cfg = 0) {
    switch (mode) {
    case MODE_MONOPOLE: return pick_3d<MODE_MONOPOLE>(wk, unitw, jk, exact, cfg);
    case MODE_SIGMA_PI: return pick_3d<MODE_SIGMA_PI>(wk, unitw, jk, exact, cfg);
    case MODE_S_MU: return pick_3d<MODE_S_MU>(wk, unitw, jk, exact, cfg);
    default:
        return wk == W_ANG_INVP ? pick_kernel<MODE_ANGULAR, W_ANG_INVP>(unitw, jk, exact)
                                : pick_kernel<MODE_ANGULAR, W_PLAIN>(unitw, jk, exact, cfg);
    }
}

inline float f_from_bits(uint32_t u) {
    float f;
    std::memcpy(&f, &u, 4);
    return f;
}
inline uint32_t bits_of(float f) {
    uint32_t u;
    std::memcpy(&u, &f, 4);
    return u;
}

// Category of a value: bin index, or -1 when the pair is dropped.
struct Category {
    const std::vector<float> *t;
    int n;
    bool range;  // also apply the s^2 range test (min, max)
    float rmin, rmax;
    int operator()(double x) const {
        const float xf = (float)x;
        if (range && !(xf < rmax && xf > rmin)) return -1;
        int c = 0;
        for (int k = 0; k <= n; ++k)
            if ((*t)[k] <= xf) c = k + 1;
        const int b = c - 1;
        return (b >= 0 && b < n) ? b : -1;
    }
};

// Table entry for values in [v0, v1]: the category when every value within
// g of the interval shares it, else ambiguous.
unsigned char lut_entry(const Category &cat, const std::vector<double> &edges, double v0, double v1, double g,
                        bool edge_code = false) {
    const double lo = v0 - g, hi = v1 + g;
    int n_in = 0;
    double e_in = 0;
    for (double e : edges)
        if (e > lo && e <= hi && (n_in == 0 || e != e_in)) {
            ++n_in;
            e_in = e;
        }
    if (n_in == 0) {
        const int c = cat(0.5 * (v0 + v1));
        if (c != cat(lo) || c != cat(hi)) return LUT_AMB;
        return c < 0 ? LUT_INV : (unsigned char)c;
    }
    if (edge_code && n_in == 1) {
        // one threshold inside: bin k below it, k + 1 above
        const int k = cat(lo);
        if (k >= 0 && k + 1 < cat.n && cat(hi) == k + 1 && (double)(*cat.t)[k + 1] == e_in &&
            k < kLutEdgeMaxBins)
            return (unsigned char)(LUT_EDGE + k);
    }
    return LUT_AMB;
}

}  // namespace


#define TPCF_TRY(expr)                                                                        \
    do {                                                                                      \
        cudaError_t _e = (expr);                                                              \
        if (_e != cudaSuccess) {                                                              \
            err->status = (_e == cudaErrorMemoryAllocation) ? 2 : 3;                          \
            err->msg = std::string("CUDA error in pair count: ") + cudaGetErrorString(_e);    \
            return err->status;                                                               \
        }                                                                                     \
    } while (0)

// Error bounds of the FP32 path against the reference sequence.  delta bounds
// |dx_fast - dx_ref| per axis for cells of side `side` with offsets up to m
// cells: the cell-relative coordinates, the cell offset, the shifted A
// coordinate and the final difference each round once in float (relative
// 2^-24), and the reference's own float rounding of the difference adds one
// more.  The other bounds follow by first-order propagation through s^2, pi,
// sigma^2 = s^2 - pi^2 and mu = |pi| / s, each doubled for safety.
struct Guards {
    float g_s2, g_pi, g_a, c1_mu, c2_mu, g_mu0;
    float g_ang = 0;  // angular counts: bound on |chord^2 / 2 - (1 - cos(theta))_ref|
};

Guards compute_guards(double side, int m, double rb) {
    const double u = std::ldexp(1.0, -24);
    const double delta = 1.25 * u * ((2.0 * m + 3.0) * side + 2.0 * rb);
    Guards g;
    const double gs2 = 2.0 * (2.0 * std::sqrt(3.0) * delta * rb + 3.0 * delta * delta + 8.0 * u * rb * rb);
    const double gpi = 6.0 * delta + 50.0 * u * rb;
    const double ga = gs2 + 2.0 * rb * gpi + 0.5 * gpi * gpi + 6.0 * u * rb * rb;
    g.g_s2 = (float)gs2;
    g.g_pi = (float)gpi;
    g.g_a = (float)ga;
    g.c1_mu = (float)(gpi + 2.0 * std::sqrt(3.0) * delta);
    g.c2_mu = (float)(3.0 * delta * delta);
    g.g_mu0 = (float)(28.0 * u);
    return g;
}

// Host-built binning tables for one binning and one set of guards.
struct Luts {
    std::vector<unsigned char> l1, l2;
    bool edge1 = false, edge2 = false;  // edge-coded tables (LUT_EDGE)
    unsigned base1 = 0, shift1 = 23 - 8;
    int n1 = LUT1_N;  // buckets of table 1 in use
    float scale2 = 0;
    float s2_lut_min = 0;
    bool direct2 = false;  // axis 2 binned directly (direct_bin) instead of by table 2
    float inv2 = 0, k2 = 0;
};

// Direct binning of a linear axis 2 from 0 (mu, |pi|): the kernel bins
// y = value * c with the reference's own float c = 1 / step, so threshold k
// sits at t2[k] c, within dev of k (exact in double: a product of two
// floats).  y is within 2^-24 y of value * c, the value within its guard gx
// of the reference's; so a y farther than dev + gx c + 2^-24 y_max from its
// nearest integer lies in the reference's bin floor(y).  k2 is that bound (gx
// c added per pair for mu), each term at least doubled.  False when the axis
// needs table 2.
bool direct2_params(const Binning &bin, const Guards &g, float *inv2, float *k2_out) {
    if (bin.mode != MODE_SIGMA_PI && bin.mode != MODE_S_MU) return false;
    const double xmax2 = bin.mode == MODE_S_MU ? 1.25 : 1.25 * std::sqrt((double)bin.max_r_sq);
    const double c = (double)bin.ax2.inv_step;
    bool ok = !bin.ax2.log_binning && bin.ax2.min == 0.0f && bin.vs2 == ValueSpace::Direct && c > 0 &&
              std::isfinite(c);
    double dev = 0;
    for (int k = 0; ok && k <= bin.nb2; ++k) {
        ok = std::isfinite(bin.t2[k]);
        if (ok) dev = std::max(dev, std::fabs((double)bin.t2[k] * c - k));
    }
    const double ymax = xmax2 * c;
    const double k2 = 2.0 * dev + std::ldexp(ymax, -22) + (bin.mode == MODE_SIGMA_PI ? 2.0 * g.g_pi * c : 0.0);
    if (!(ok && dev < 1e-3 && k2 < 0.05 && ymax < 1e6)) return false;
    *inv2 = (float)c;
    *k2_out = (float)k2;
    return true;
}

Luts build_luts(const Binning &bin, const Guards &g) {
    Luts L;
    L.l1.assign(LUT1_N, LUT_AMB);
    float inv2 = 0, k2 = 0;
    const bool d2 = direct2_params(bin, g, &inv2, &k2);
    const bool table2 = (bin.mode == MODE_SIGMA_PI || bin.mode == MODE_S_MU) && !d2;
    L.n1 = table2 ? LUT1_N_T2 : LUT1_N;
    L.l2.assign(LUT2_N, LUT_AMB);
    // Table 1 over the float bits of s^2 (monopole, s-mu; the range test is
    // folded in), of sigma^2 (sigma-pi) or of 1 - cos(theta) (angular).
    const bool s_axis = bin.mode == MODE_MONOPOLE || bin.mode == MODE_S_MU;
    Category c1{&bin.t1, bin.nb1, s_axis, bin.min_r_sq, bin.max_r_sq};
    std::vector<double> e1(bin.t1.begin(), bin.t1.end());
    if (s_axis) {
        e1.push_back(bin.min_r_sq);
        e1.push_back(std::nextafter(bin.min_r_sq, INFINITY));
        e1.push_back(bin.max_r_sq);
    }
    const double xmax1 = std::max((double)bin.max_r_sq, 1e-30) * 2.0;
    const int ehi = (int)std::ceil(std::log2(xmax1)) + 1;
    const int bits1 = (bin.mode == MODE_SIGMA_PI && !bin.ax1.log_binning && !table2) ? 9 : 8;
    const int elo = ehi - (L.n1 >> bits1);
    const uint32_t sh = 23 - bits1;
    L.shift1 = sh;
    L.base1 = bits_of(std::ldexp(1.0f, elo)) >> sh;
    const double g1 = s_axis ? g.g_s2 : (bin.mode == MODE_ANGULAR ? g.g_ang : g.g_a);
    L.edge1 = bin.nb1 <= kLutEdgeMaxBins;
    for (int i = 1; i < L.n1 - 1; ++i) {
        const double v0 = f_from_bits((L.base1 + i) << sh);
        const double v1 = f_from_bits((L.base1 + i + 1) << sh);
        L.l1[i] = lut_entry(c1, e1, v0, v1, g1, L.edge1);
    }
    // Bucket 0 holds everything below the table (ambiguous); the last bucket
    // holds everything above it.
    {
        const double v0 = f_from_bits((L.base1 + L.n1 - 1) << sh);
        if (s_axis && v0 - g1 > bin.max_r_sq) L.l1[L.n1 - 1] = LUT_INV;
        if (!s_axis && std::isfinite(bin.t1[bin.nb1]) && v0 - g1 > bin.t1[bin.nb1]) L.l1[L.n1 - 1] = LUT_INV;
    }
    if (bin.mode == MODE_SIGMA_PI || bin.mode == MODE_S_MU) {
        // Table 2, linear buckets: mu on [0, 1.25) or |pi| on [0, 1.25 rmax).
        const double xmax2 = bin.mode == MODE_S_MU ? 1.25 : 1.25 * std::sqrt((double)bin.max_r_sq);
        L.scale2 = (float)(LUT2_N / xmax2);
        Category c2{&bin.t2, bin.nb2, false, 0, 0};
        std::vector<double> e2(bin.t2.begin(), bin.t2.end());
        double g2;
        if (bin.mode == MODE_S_MU) {
            // The mu guard grows as 1/s; the table holds for s^2 >= s2_lut_min.
            const double gt = 0.5 / L.scale2;
            const double a = gt - g.g_mu0;
            const double s = (g.c1_mu + std::sqrt((double)g.c1_mu * g.c1_mu + 4.0 * a * g.c2_mu)) / (2.0 * a);
            L.s2_lut_min = (float)(s * s * 1.0001);
            g2 = gt;
        } else {
            g2 = g.g_pi;
        }
        const double w = 1.0 / L.scale2;
        L.edge2 = bin.nb2 <= kLutEdgeMaxBins;
        for (int i = 0; i < LUT2_N - 1; ++i) {
            const double v0 = i * w, v1 = (i + 1) * w;
            const double slack = 4.0 * std::ldexp(1.0, -23) * v1;  // bucket-edge rounding of (int)(x * scale)
            L.l2[i] = lut_entry(c2, e2, v0, v1, g2 + slack, L.edge2);
        }
        const double vlast = (LUT2_N - 1) * w;
        if (c2(vlast - g2) < 0 && vlast - g2 > bin.t2[bin.nb2]) L.l2[LUT2_N - 1] = LUT_INV;
        if (d2) {
            L.direct2 = true;
            L.inv2 = inv2;
            L.k2 = k2;
            L.s2_lut_min = 0.0f;  // the per-pair guard of mu holds at every s
        }
    }
    return L;
}

namespace {

// Largest number of pairs one flush of a shared-memory histogram can hold:
// a work item's A points times the B points of all its segments.
long long max_item_pairs(const std::vector<WorkItem> &items, const std::vector<Segment> &segs) {
    long long pmax = 1;
#pragma omp parallel for schedule(static) reduction(max : pmax)
    for (long long q = 0; q < (long long)items.size(); ++q) {
        const WorkItem &w = items[q];
        long long bl = 0;
        for (int k = w.seg_begin; k < w.seg_end; ++k) bl += segs[k].b_len;
        pmax = std::max(pmax, (long long)w.a_len * bl);
    }
    return pmax;
}

// Fixed-point shift S: a pair weight w is added as round(w * 2^S) to 64-bit
// shared-memory sums and 128-bit global sums.  S keeps the largest flush
// (pmax pairs of weight at most wmax) below 2^62; every float weight of at
// least 2^(23-S) is then represented exactly, and smaller ones to 2^-(S+1).
// The plain-weight kernels stage each A weight times 2^S, so S also keeps
// wa_max 2^S (wa_max: the largest weight of either catalogue) far below the
// float range.
int fixed_point_shift(double wmax, long long pmax, double wa_max = 0) {
    const double lg = std::log2(std::max(wmax * (1.0 + 1e-6), 1e-30)) + std::log2((double)std::max(pmax, 1LL));
    int S = (int)std::floor(62.0 - lg);
    if (wa_max > 0) S = std::min(S, (int)std::floor(120.0 - std::log2(wa_max)));
    return std::max(-100, std::min(S, 100));
}

// A 128-bit two's-complement fixed-point sum (low word, high word) as a
// double, rounded once, times inv = 2^-S.
double fixed_to_double(const unsigned long long *p, double inv) {
    const unsigned __int128 u = ((unsigned __int128)p[1] << 64) | (unsigned __int128)p[0];
    return (double)(__int128)u * inv;
}

// Everything a count needs before device buffers exist: grids, work list,
// kernel choice, fixed-point scale, guards, tables, and the kernel
// parameters other than buffer addresses.
struct CountPlan {
    const Binning *bin = nullptr;
    const UpTable *up = nullptr;
    bool is_auto = false, jk = false, unitw = false, angular = false, adj = false;
    int nb = 0, n_jk = 1, wk = W_PLAIN;
    int n_a = 0, n_b = 0;  // catalogue sizes (adjoint outputs)
    const double *adj_G_host = nullptr;
    double *grad_a_host = nullptr, *grad_b_host = nullptr;
    double adj_scale = 1.0, adj_inv = 1.0;
    double inv = 1.0;  // 2^-S
    int scale_exp = 0;  // S
    long long *raw_out = nullptr;  // partial sums of a shard (kPartialWords per slot)
    std::vector<WorkItem> items;
    std::vector<Segment> segs;
    std::vector<JobK> jobs;  // one for a single count
    SmemLayout L;
    Luts luts;
    KParams P;
    KernelFn fn = nullptr;
    int m = 0;              // cells per maximum separation
    int cfg = 0;            // kernel configuration
    bool cfg_tunable = false;  // plain-weight FP32+guard count: both configurations exist
    double dens_a = 0, dens_b = 0;  // points per cell of side rb (the autotuner's density class)
    size_t n_flags() const { return wk == W_PLAIN ? 0 : (size_t)(1 + n_jk) * nb; }
    size_t n_up() const { return up ? up->thr.size() : 0; }
};

// Device addresses of the per-count buffers.
struct CountBuffers {
    WorkItem *items = nullptr;
    Segment *segs = nullptr;
    unsigned long long *full = nullptr, *sub = nullptr, *cnt = nullptr;
    int *head = nullptr, *err = nullptr;
    float *t1 = nullptr, *t2 = nullptr, *up_thr = nullptr;
    unsigned char *l1 = nullptr, *l2 = nullptr;
    unsigned *flags = nullptr;
    double *up_bins = nullptr, *up_centre = nullptr;
    double *adj_G = nullptr, *grad_a = nullptr, *grad_b = nullptr;
    JobK *jobs = nullptr;
};

// Device view of one catalogue's grid.
void fill_grid(GridK &k, const Grid &gr, const Catalog &c) {
    k.pos = gr.pos.p;
    k.aux = gr.aux.p;
    k.idx = gr.idx.p;
    k.xyz_s = gr.xyz_s.p;
    k.unit_s = gr.unit_s.p;
    k.coord = gr.cell_coord.p;
    k.kmin0 = gr.kmin[0];
    k.kmin1 = gr.kmin[1];
    k.kmin2 = gr.kmin[2];
    k.n_pts = gr.n;
    k.n_cells = gr.ncell;
    k.xyz = c.xyz.p;
    k.unit = c.unit.p;
}

// Kernel parameters that depend on the binning, guards and tables only (not
// on the catalogues or the work list).
void fill_params(CountPlan &C, const Binning *bin, const Guards &g, double side, double tn, float wscale,
                 int n_runs) {
    KParams &P = C.P;
    std::memset(&P, 0, sizeof(P));
    P.n_items = (int)C.items.size();
    P.n_segs = (int)C.segs.size();
    P.n_jobs = 1;
    P.side = side;
    P.n1 = bin->nb1;
    P.n2 = (bin->mode == MODE_SIGMA_PI || bin->mode == MODE_S_MU) ? bin->nb2 : 0;
    P.nb = C.nb;
    P.min_r_sq = bin->min_r_sq;
    P.max_r_sq = bin->max_r_sq;
    P.g_s2 = g.g_s2;
    P.g_pi = g.g_pi;
    P.g_a = g.g_a;
    P.c1_mu = g.c1_mu;
    P.c2_mu = g.c2_mu;
    P.g_mu0 = g.g_mu0;
    P.g_ang = g.g_ang;
    P.s2_lut_min = C.luts.s2_lut_min;
    if (C.angular) {
        // candidate test on the squared chord: v = chord^2 / 2 < T[n] + g_ang
        P.lo_cut = -1.0f;
        P.hi_cut = (float)(2.0 * (tn + g.g_ang) * (1.0 + 1e-6));
    } else {
        P.lo_cut = bin->min_r_sq - g.g_s2;
        P.hi_cut = bin->max_r_sq + g.g_s2;
    }
    // One compare: |s^2 - mid| < half, widened to cover the float rounding of
    // mid, half and the subtraction.
    P.cut_mid = (float)(0.5 * ((double)P.lo_cut + (double)P.hi_cut));
    P.cut_half = (float)(0.5 * ((double)P.hi_cut - (double)P.lo_cut) * (1.0 + 1e-5) +
                         1e-6 * std::fabs((double)P.cut_mid));
    // The FP32 candidate test keeps the upper side only: s^2 < h, h the
    // smallest float with fl(h - cut_mid) >= cut_half (rounding is monotone,
    // so s^2 < h exactly when fl(s^2 - cut_mid) < cut_half).  Pairs below
    // lo_cut (a minimum separation above 0) then reach the binning step,
    // whose tables and range test drop them.
    {
        volatile float h = (float)((double)P.cut_mid + (double)P.cut_half);
        while (!((float)(h - P.cut_mid) >= P.cut_half)) h = std::nextafter((float)h, INFINITY);
        for (;;) {
            const float lower = std::nextafter((float)h, -INFINITY);
            if (!((float)(lower - P.cut_mid) >= P.cut_half)) break;
            h = lower;
        }
        P.s2_test = h;
    }
    P.lut1_base = C.luts.base1;
    P.lut1_shift = C.luts.shift1;
    P.lut1_n = C.luts.n1;
    P.lut_edge1 = C.luts.edge1 ? 1 : 0;
    P.lut_edge2 = C.luts.edge2 ? 1 : 0;
    P.lut2_scale = C.luts.scale2;
    P.direct2 = C.luts.direct2 ? 1 : 0;
    P.inv2 = C.luts.inv2;
    P.k2 = C.luts.k2;
    // the mu guard scaled to bins, rounded up
    const double up = 1.0 + std::ldexp(1.0, -20);
    P.c1y = (float)((double)g.c1_mu * C.luts.inv2 * up);
    P.c2y = (float)((double)g.c2_mu * C.luts.inv2 * up);
    P.g0y = (float)(((double)g.g_mu0 * C.luts.inv2 + C.luts.k2) * up);
    P.n_jk = C.n_jk;
    P.wscale = wscale;
    P.n_runs_f = (float)n_runs;
    P.n_runs_d = (double)n_runs;
    P.los_mid = bin->los_midpoint ? 1 : 0;
    P.force_timeout = debug_force_tile_timeout().load() ? 1 : 0;
    if (C.up) {
        P.n_up = C.up->ax.n_bins;
        P.up_min = (double)C.up->ax.min;
        P.up_max = (double)C.up->ax.max;
    }
}

int plan_count(Ctx *ctx, const CountRequest &req, bool build, CountPlan &C, Error *err, bool grids_only = false) {
    const Binning *bin = req.bin;
    Catalog *A = const_cast<Catalog *>(req.a);
    Catalog *B = const_cast<Catalog *>(req.b ? req.b : req.a);
    C.bin = bin;
    C.up = req.up;
    C.is_auto = (req.b == nullptr);
    C.angular = bin->mode == MODE_ANGULAR;
    C.nb = bin->nb;
    C.n_jk = bin->n_jk;
    C.jk = C.n_jk > 1;
    C.adj = req.adj_G != nullptr;
    C.adj_G_host = req.adj_G;
    C.grad_a_host = req.grad_a;
    C.grad_b_host = req.grad_b;
    C.n_a = (int)A->n_all;
    C.n_b = (int)B->n_all;
    const int wt = req.weighting;
    // Weight kind, the weight each grid point carries, and the points
    // counted: 3-D counts use the d_comov partition (GalaxyBoxes); angular
    // counts use every point unless inverse-p weights ask for a redshift
    // (GalaxyPixels' require_redshift, src/correlators_invpweight.cpp:990-1028).
    if (C.angular) C.wk = wt == WEIGHTS_INVP_DD ? W_ANG_INVP : W_PLAIN;
    else C.wk = wt == WEIGHTS_INVP_DD ? W_INVP_DD : (wt == WEIGHTS_INVP_DR ? W_INVP_DR : W_PLAIN);
    const bool input_w = C.angular ? wt != WEIGHTS_INVP_DR : wt == WEIGHTS_INVP_DD;
    const bool subset = C.angular ? wt != WEIGHTS_PLAIN : true;
    auto wmax_of = [&](const Catalog *c) { return (double)(input_w ? c->iw_max : c->w_max); };
    auto unit_of = [&](const Catalog *c) { return input_w ? c->iw_unit : c->unit_weights; };
    C.unitw = C.wk == W_PLAIN && unit_of(A) && unit_of(B);
    if (C.adj) {
        if (C.angular || wt != WEIGHTS_PLAIN) {
            err->status = 6;
            err->msg = "the adjoint is defined for plain-weight 3-D counts";
            return err->status;
        }
        C.wk = W_ADJ;
        C.jk = false;  // dL/dw of the full histogram; regions play no part
        C.unitw = false;
    }

    // Per-axis bound on the separation of every counted pair: the maximum
    // separation (3-D), or the chord of the largest binned 1 - cos(theta),
    // widened by the double rounding of the reference's value and by how far
    // the unit vectors are from unit length (angular).
    double rb = bin->rmax_bound;
    double norm_dev = 0, tn = 2.0;
    if (C.angular) {
        if (std::isfinite(bin->t1[bin->nb1])) tn = std::max((double)bin->t1[bin->nb1], 0.0);
        norm_dev = std::max(A->norm_dev, B->norm_dev);
        rb = std::sqrt(2.0 * tn + 4e-15 + 2.0 * norm_dev) * (1.0 + 1e-6) + 1e-12;
    }
    auto per_cell = [&](const Catalog *X, int k) {
        const double *lo = C.angular ? (subset ? X->ulo_kept : X->ulo_all) : X->lo_kept;
        const double *hi = C.angular ? (subset ? X->uhi_kept : X->uhi_all) : X->hi_kept;
        const double n = subset ? (double)X->n_kept : (double)X->n_all;
        double vol = 1;
        for (int d = 0; d < 3; ++d) vol *= std::max(hi[d] - lo[d], rb);
        const double c = rb / k;
        return n * c * c * c / vol;
    };
    C.dens_a = per_cell(A, 1);
    C.dens_b = per_cell(B, 1);
    C.cfg_tunable = C.wk == W_PLAIN && !req.exact_fp64 && !C.adj;
    C.cfg = C.cfg_tunable ? (req.kernel_cfg >= 0 ? req.kernel_cfg : std::max(ctx->kernel_cfg, 0)) : 0;
    int m = req.refinement > 0 ? req.refinement : ctx->refinement;
    if (m <= 0) {
        // Automatic: refine to side rb/2 when cells of that size would still
        // hold a few hundred points on average in the denser catalogue (the
        // B points a cell's stencil visits set the candidate count; measured
        // on the survey benchmark, a cross count of sparse data against dense
        // randoms runs ~10 % faster at side rb/2 than at rb).  The FP64
        // path, whose candidate test costs several times the FP32 one, goes
        // to side rb/3 once the A catalogue holds ~50 points per such cell
        // (measured on the survey benchmark: 3-8 % faster on each count that
        // meets it; the FP32 path gains under 1 % there and keeps rb/2).
        m = std::max(per_cell(A, 2), per_cell(B, 2)) >= 256 ? 2 : 1;
        if (req.exact_fp64 && per_cell(A, 3) >= 50) m = 3;
    }
    C.m = m;
    const double side = rb / m * (1.0 + 1e-9);
    GridSpec gs;
    gs.side = side;
    gs.subset_kept = subset;
    gs.angular = C.angular;
    gs.input_w = input_w;
    Grid *ga = nullptr, *gb = nullptr;
    if (build) {
        if (build_grid(ctx, A, gs, req.exact_fp64, &ga, err)) return err->status;
        if (C.is_auto) gb = ga;
        else if (build_grid(ctx, B, gs, req.exact_fp64, &gb, err)) return err->status;
    } else {
        ga = find_grid(A, gs, req.exact_fp64);
        gb = C.is_auto ? ga : find_grid(B, gs, req.exact_fp64);
        if (!ga || !gb) {
            err->status = 1;
            err->msg = std::string("no cell grid cached on catalogue ") + (!ga ? "a" : "b") +
                       " for this binning, weighting, refinement and precision: the allocation-free count does "
                       "not build grids; count the same catalogues once with tpcf_count first";
            return err->status;
        }
    }
    if (grids_only) return 0;
    build_work_items(*ga, *gb, C.is_auto, m, side, rb, C.items, C.segs);

    if (C.adj) {
        // Fixed point of the gradient sums: an A point's sum takes one term
        // G[bin] w_b per B point of its item, a B point's tile sum one term
        // G[bin] w_a per A point of the chunk; the larger bound of the two
        // gets 2^62, so no 64-bit sum can overflow, and a term is resolved to
        // 2^-S (about 1e-15 of max|G| max w times the item's B points).
        double gmax = 0.0;
        for (int b = 0; b < C.nb; ++b) {
            if (!std::isfinite(C.adj_G_host[b])) {
                err->status = 1;
                err->msg = "dL/d(full histogram) must be finite";
                return err->status;
            }
            gmax = std::max(gmax, std::fabs(C.adj_G_host[b]));
        }
        long long nb_max = 1;
        for (const WorkItem &w : C.items) {
            long long bl = 0;
            for (int k = w.seg_begin; k < w.seg_end; ++k) bl += C.segs[k].b_len;
            nb_max = std::max(nb_max, bl);
        }
        const double bound = gmax * std::max((double)B->w_max * (double)nb_max, (double)A->w_max * (double)TA);
        const int S = bound > 0 ? std::max(-1000, std::min(1000, (int)std::floor(62.0 - std::log2(bound)))) : 0;
        C.adj_scale = std::ldexp(1.0, S);
        C.adj_inv = std::ldexp(1.0, -S);
    }
    float wscale = 1.0f;
    if (!C.unitw && !C.adj) {
        double wmax = wmax_of(A) * wmax_of(B);
        const double up_max = C.up ? 4.0 * C.up->abs_max : 0.0;  // interpolation stays within 4x the bins
        // the popcount-ratio numerator: n_runs, or a dither popcount (at most 64 per mask word)
        const double num = std::max(req.dither ? 64.0 * A->n_mask : (double)req.n_runs, 1.0);
        if (C.wk == W_INVP_DD) wmax *= up_max * num;
        else if (C.wk == W_INVP_DR) wmax *= up_max;
        else if (C.wk == W_ANG_INVP) wmax *= num;
        const int S = fixed_point_shift(wmax, max_item_pairs(C.items, C.segs), std::max(wmax_of(A), wmax_of(B)));
        wscale = std::ldexp(1.0f, S);
        C.inv = std::ldexp(1.0, -S);
        C.scale_exp = S;
    }
    if (req.n_shards > 1) {
        // This shard's items, dealt round-robin from the largest down; the
        // scale above came from the whole list, so every shard adds in the
        // same fixed point.
        std::vector<WorkItem> mine;
        mine.reserve(C.items.size() / req.n_shards + 1);
        for (size_t k = (size_t)req.shard; k < C.items.size(); k += (size_t)req.n_shards) mine.push_back(C.items[k]);
        C.items.swap(mine);
    }
    C.raw_out = req.raw_out;
    C.L = smem_layout(C.nb, bin->nb1, bin->nb2, req.exact_fp64, C.jk, C.adj, C.cfg);
    if (C.L.total + 1024 > ctx->smem_optin) {
        err->status = 6;
        err->msg = "histogram does not fit in shared memory";
        return err->status;
    }
    Guards g = compute_guards(side, m, rb);
    if (C.angular) g.g_ang = (float)((0.5 * g.g_s2 + 2.0 * norm_dev + 2e-15) * (1.0 + 1e-6));
    C.luts = build_luts(*bin, g);
    // without table 2 (axis 2 binned directly) the kernel's layout is smaller
    C.L = smem_layout(C.nb, bin->nb1, bin->nb2, req.exact_fp64, C.jk, C.adj, C.cfg,
                      (bin->mode == MODE_SIGMA_PI || bin->mode == MODE_S_MU) && !C.luts.direct2);

    fill_params(C, bin, g, side, tn, wscale, req.n_runs);
    KParams &P = C.P;
    JobK job;
    std::memset(&job, 0, sizeof(job));
    fill_grid(job.a, *ga, *A);
    fill_grid(job.b, *gb, *B);
    job.out = 0;
    C.jobs.assign(1, job);
    P.a_masks = A->masks.p;
    P.b_masks = B->masks.p;
    P.n_mask = A->n_mask;
    if (req.dither && (C.wk == W_INVP_DD || C.wk == W_ANG_INVP)) {
        P.dither = 1;
        P.a_dmasks = A->dmasks.p;
        P.b_dmasks = B->dmasks.p;
    }
    // widest mask load every row start allows (row stride n_mask words)
    auto aligned = [&](uintptr_t a) {
        const uintptr_t q = (uintptr_t)P.a_masks | (uintptr_t)P.b_masks |
                            (P.dither ? ((uintptr_t)P.a_dmasks | (uintptr_t)P.b_dmasks) : 0);
        return (q & (a - 1)) == 0;
    };
    P.mask_vec = (P.n_mask % 4 == 0 && aligned(32)) ? 4 : ((P.n_mask % 2 == 0 && aligned(16)) ? 2 : 1);
    C.fn = pick(bin->mode, C.wk, C.unitw, C.jk, req.exact_fp64, C.cfg);
    return 0;
}

// Host side of one count in flight: where its uploads are staged and where
// its results land.  With `stage` set (pinned memory, a count of
// count_many), every copy is asynchronous and the host can plan the next
// count while this one runs; otherwise the plan's vectors are uploaded
// directly and the results land in `own` (pageable).
struct HostIO {
    unsigned char *stage = nullptr;  // pinned: uploads, then results
    size_t stage_cap = 0;
    std::vector<unsigned long long> own;
    unsigned long long *hf = nullptr, *hs = nullptr, *hc = nullptr;
    int *herr = nullptr;
    unsigned *hflags = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr, done = nullptr;
    ~HostIO() {
        if (e0) cudaEventDestroy(e0);
        if (e1) cudaEventDestroy(e1);
        if (done) cudaEventDestroy(done);
    }
};

// Bytes of pinned staging a count needs (uploads and results).
size_t stage_bytes(const CountPlan &C) {
    auto up16 = [](size_t x) { return (x + 15) / 16 * 16; };
    const Binning *bin = C.bin;
    size_t t = 0;
    t += up16(sizeof(WorkItem) * C.items.size()) + up16(sizeof(Segment) * C.segs.size());
    t += up16(sizeof(JobK) * C.jobs.size()) + up16(sizeof(float) * bin->t1.size()) + up16(sizeof(float) * bin->t2.size());
    t += up16(LUT1_N) + up16(LUT2_N);
    t += 3 * up16(sizeof(double) * C.n_up());
    if (C.adj) t += up16(sizeof(double) * C.nb);
    t += up16(sizeof(unsigned long long) * 2 * C.nb) + up16(sizeof(unsigned long long) * 2 * (size_t)C.nb * C.n_jk);
    t += up16(sizeof(unsigned long long) * 4) + 16 + up16(sizeof(unsigned) * C.n_flags());
    return t;
}

// Upload the tables and the work list, clear the accumulators, launch, and
// queue the read-back of the results; timed: events around the kernel.
int launch_count(Ctx *ctx, CountPlan &C, const CountBuffers &D, HostIO &io, Error *err, bool timed) {
    const Binning *bin = C.bin;
    const int nb = C.nb, n_jk = C.n_jk;
    cudaStream_t stm = ctx->stream;
    size_t off = 0;
    // host source of an upload: the plan's own memory, or its copy in the
    // pinned stage
    auto src = [&](const void *h, size_t bytes) -> const void * {
        if (!io.stage) return h;
        unsigned char *d = io.stage + off;
        if (bytes) std::memcpy(d, h, bytes);
        off += (bytes + 15) / 16 * 16;
        return d;
    };
    auto h2d = [&](void *dst, const void *h, size_t bytes) -> cudaError_t {
        const void *s2 = src(h, bytes);
        return bytes ? cudaMemcpyAsync(dst, s2, bytes, cudaMemcpyHostToDevice, stm) : cudaSuccess;
    };
#ifdef TPCF_DEVICE_CHECKS
    if (debug_corrupt_work_list().exchange(0) == 1 && !C.segs.empty())
        C.segs[0].meta = (C.segs[0].meta & ~0xffff) | ((C.n_jk + 3) & 0xffff);
#endif
    if (!C.items.empty()) {
        TPCF_TRY(h2d(D.items, C.items.data(), sizeof(WorkItem) * C.items.size()));
        TPCF_TRY(h2d(D.segs, C.segs.data(), sizeof(Segment) * C.segs.size()));
    }
    TPCF_TRY(h2d(D.jobs, C.jobs.data(), sizeof(JobK) * C.jobs.size()));
    TPCF_TRY(h2d(D.t1, bin->t1.data(), sizeof(float) * bin->t1.size()));
    if (!bin->t2.empty()) TPCF_TRY(h2d(D.t2, bin->t2.data(), sizeof(float) * bin->t2.size()));
    TPCF_TRY(h2d(D.l1, C.luts.l1.data(), LUT1_N));
    TPCF_TRY(h2d(D.l2, C.luts.l2.data(), LUT2_N));
    if (C.up) {
        const size_t k = C.n_up();
        TPCF_TRY(h2d(D.up_thr, C.up->thr.data(), sizeof(float) * k));
        TPCF_TRY(h2d(D.up_bins, C.up->bins.data(), sizeof(double) * k));
        TPCF_TRY(h2d(D.up_centre, C.up->centre.data(), sizeof(double) * k));
    }
    // What the kernel accumulates into starts at zero on every call.
    TPCF_TRY(cudaMemsetAsync(D.full, 0, sizeof(unsigned long long) * 2 * nb, stm));
    TPCF_TRY(cudaMemsetAsync(D.sub, 0, sizeof(unsigned long long) * 2 * (size_t)nb * n_jk, stm));
    TPCF_TRY(cudaMemsetAsync(D.cnt, 0, sizeof(unsigned long long) * 4, stm));
    TPCF_TRY(cudaMemsetAsync(D.head, 0, sizeof(int), stm));
    TPCF_TRY(cudaMemsetAsync(D.err, 0, sizeof(int) * kErrWords, stm));
    if (C.n_flags()) TPCF_TRY(cudaMemsetAsync(D.flags, 0, sizeof(unsigned) * C.n_flags(), stm));
    if (C.adj) {
        TPCF_TRY(h2d(D.adj_G, C.adj_G_host, sizeof(double) * nb));
        TPCF_TRY(cudaMemsetAsync(D.grad_a, 0, sizeof(double) * std::max(C.n_a, 1), stm));
        if (!C.is_auto) TPCF_TRY(cudaMemsetAsync(D.grad_b, 0, sizeof(double) * std::max(C.n_b, 1), stm));
    }

    KParams P = C.P;
    P.n_segs = (int)C.segs.size();
    P.n_jobs = (int)C.jobs.size();
    P.jobs = D.jobs;
    P.job0 = C.jobs[0];
    P.items = D.items;
    P.segs = D.segs;
    P.head = D.head;
    P.t1g = D.t1;
    P.t2g = D.t2;
    P.lut1g = D.l1;
    P.lut2g = D.l2;
    P.g_full = D.full;
    P.g_sub = D.sub;
    P.counters = D.cnt;
    P.err = D.err;
    P.flags = D.flags;
    P.up_thr = D.up_thr;
    P.up_bins = D.up_bins;
    P.up_centre = D.up_centre;
    P.adj_G = D.adj_G;
    P.adj_scale = C.adj_scale;
    P.adj_inv = C.adj_inv;
    P.grad_a = D.grad_a;
    P.grad_b = C.is_auto ? D.grad_a : D.grad_b;

    TPCF_TRY(cudaFuncSetAttribute((const void *)C.fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)C.L.total));
    int per_sm = 1;
    TPCF_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, C.fn, NT, C.L.total));
    per_sm = std::max(per_sm, 1);
    if (timed) {
        TPCF_TRY(cudaEventCreate(&io.e0));
        TPCF_TRY(cudaEventCreate(&io.e1));
        TPCF_TRY(cudaEventRecord(io.e0, stm));
    }
    if (!C.items.empty()) {
        const int grid = (int)std::min<long long>((long long)ctx->num_sms * per_sm, (long long)C.items.size());
        C.fn<<<grid, NT, C.L.total, stm>>>(P);
        ++ctx->launches;
        TPCF_TRY(cudaGetLastError());
    }
    if (timed) TPCF_TRY(cudaEventRecord(io.e1, stm));
    // results: into the pinned stage after the uploads, or into `own`
    const size_t n_hf = 2 * (size_t)nb, n_hs = 2 * (size_t)nb * n_jk, n_fl = C.n_flags();
    unsigned char *r = nullptr;
    if (io.stage) {
        r = io.stage + off;
    } else {
        io.own.assign(n_hf + n_hs + 4 + 2 + (n_fl + 1) / 2, 0ull);
        r = reinterpret_cast<unsigned char *>(io.own.data());
    }
    io.hf = reinterpret_cast<unsigned long long *>(r);
    io.hs = io.hf + n_hf;
    io.hc = io.hs + n_hs;
    io.herr = reinterpret_cast<int *>(io.hc + 4);   // kErrWords ints
    io.hflags = reinterpret_cast<unsigned *>(io.hc + 6);
    TPCF_TRY(cudaMemcpyAsync(io.hf, D.full, sizeof(unsigned long long) * n_hf, cudaMemcpyDeviceToHost, stm));
    TPCF_TRY(cudaMemcpyAsync(io.hs, D.sub, sizeof(unsigned long long) * n_hs, cudaMemcpyDeviceToHost, stm));
    TPCF_TRY(cudaMemcpyAsync(io.hc, D.cnt, sizeof(unsigned long long) * 4, cudaMemcpyDeviceToHost, stm));
    TPCF_TRY(cudaMemcpyAsync(io.herr, D.err, sizeof(int) * kErrWords, cudaMemcpyDeviceToHost, stm));
    if (n_fl) TPCF_TRY(cudaMemcpyAsync(io.hflags, D.flags, sizeof(unsigned) * n_fl, cudaMemcpyDeviceToHost, stm));
    TPCF_TRY(cudaEventCreateWithFlags(&io.done, cudaEventDisableTiming));
    TPCF_TRY(cudaEventRecord(io.done, stm));
    return 0;
}

// The status and message of a count whose device error record is set.
int device_error(const int *e, Error *err) {
    if (e[0] == kErrCheck) {
        static const char *names[] = {"?", "bin index", "work item's job", "work item's segment range",
                                      "A chunk length", "A chunk's points", "A cell", "A region",
                                      "segment's B points", "B cell", "segment's region", "warp queue fill",
                                      "side queue fill"};
        const int id = e[1] >= 1 && e[1] <= DC_SIDE_QUEUE ? e[1] : 0;
        err->status = 7;
        err->msg = std::string("device bounds check failed: ") + names[id] + " " + std::to_string(e[2]) +
                   " outside its range (limit " + std::to_string(e[3]) + "); results discarded";
        return err->status;
    }
    err->status = 4;
    err->msg = "device wait exceeded its iteration limit; results discarded";
    return err->status;
}

// Wait for a launched count and convert its fixed-point sums (or hand back
// the shard's partial sums, or the adjoint's gradients).
int finish_count(Ctx *ctx, CountPlan &C, const CountBuffers &D, HostIO &io, double *full_out, double *region_out,
                 Stats *st, Error *err, bool timed) {
    (void)ctx;
    const int nb = C.nb, n_jk = C.n_jk;
    TPCF_TRY(cudaEventSynchronize(io.done));
    float ms = 0;
    if (timed) cudaEventElapsedTime(&ms, io.e0, io.e1);
    const unsigned long long *hf = io.hf, *hs = io.hs, *hc = io.hc;
    const bool has_flags = C.n_flags() > 0;
    const unsigned *hflags = io.hflags;
    if (*io.herr) return device_error(io.herr, err);
    if (C.adj) {
        TPCF_TRY(cudaMemcpy(C.grad_a_host, D.grad_a, sizeof(double) * C.n_a, cudaMemcpyDeviceToHost));
        if (!C.is_auto && C.grad_b_host)
            TPCF_TRY(cudaMemcpy(C.grad_b_host, D.grad_b, sizeof(double) * C.n_b, cudaMemcpyDeviceToHost));
        if (st) {
            st->candidates += hc[0];
            st->in_range += hc[1];
            st->guard += hc[2];
            st->items += C.items.size();
            st->ms_kernel += ms;
        }
        return 0;
    }
    if (C.raw_out) {
        // Partial sums of a shard: limbs of the 128-bit sums and the
        // non-finite markers as counts, slot by slot (full, then regions).
        const size_t slots = (size_t)(1 + n_jk) * nb;
        auto put = [&](size_t slot, const unsigned long long *w, unsigned f) {
            long long *o = C.raw_out + slot * kPartialWords;
            o[0] = (long long)(w[0] & 0xffffffffull);
            o[1] = (long long)(w[0] >> 32);
            o[2] = (long long)(w[1] & 0xffffffffull);
            o[3] = (long long)(w[1] >> 32);
            o[4] = (f & 1u) ? 1 : 0;
            o[5] = (f & 2u) ? 1 : 0;
            o[6] = (f & 4u) ? 1 : 0;
        };
        for (size_t slot = 0; slot < slots; ++slot) {
            const bool full = slot < (size_t)nb;
            const size_t b = full ? slot : (C.jk ? slot - nb : (slot - nb) % nb);
            const unsigned long long *w = (full || !C.jk) ? &hf[2 * b] : &hs[2 * b];
            const unsigned f = has_flags ? hflags[(full || !C.jk) ? b : nb + b] : 0u;
            put(slot, w, f);
        }
        if (st) {
            st->candidates += hc[0];
            st->in_range += hc[1];
            st->guard += hc[2];
            st->overflow += hc[3];
            st->items += C.items.size();
            st->ms_kernel += ms;
        }
        return 0;
    }
    // A bin that met a non-finite pair weight holds what double
    // accumulation would: NaN, or an infinity of one sign.  The NaN is the
    // one x86 arithmetic generates for 0/0 and inf - inf (sign bit set),
    // which the reference's up-weights carry into its sums and which its
    // ASCII outputs print as "-nan".
    auto flagged = [](unsigned f, double v) {
        if ((f & 1u) || ((f & 2u) && (f & 4u))) return std::copysign(std::numeric_limits<double>::quiet_NaN(), -1.0);
        if (f & 2u) return std::numeric_limits<double>::infinity();
        if (f & 4u) return -std::numeric_limits<double>::infinity();
        return v;
    };
    for (int b = 0; b < nb; ++b) {
        full_out[b] = fixed_to_double(&hf[2 * (size_t)b], C.inv);
        if (has_flags) full_out[b] = flagged(hflags[b], full_out[b]);
    }
    if (region_out) {
        if (C.jk) {
            for (size_t k = 0; k < (size_t)nb * n_jk; ++k) {
                region_out[k] = fixed_to_double(&hs[2 * k], C.inv);
                if (has_flags) region_out[k] = flagged(hflags[nb + k], region_out[k]);
            }
        } else {
            for (int b = 0; b < nb; ++b) region_out[b] = full_out[b];
        }
    }
    if (st) {
        st->candidates += hc[0];
        st->in_range += hc[1];
        st->guard += hc[2];
        st->overflow += hc[3];
        st->items += C.items.size();
        st->ms_kernel += ms;
    }
    return 0;
}

// One count from upload to results, synchronously, staging through the
// C++ heap.
int execute(Ctx *ctx, CountPlan &C, const CountBuffers &D, double *full_out, double *region_out, Stats *st,
            Error *err, bool timed) {
    HostIO io;
    if (launch_count(ctx, C, D, io, err, timed)) {
        if (!err->status) err->status = 3;
        return err->status;
    }
    return finish_count(ctx, C, D, io, full_out, region_out, st, err, timed);
}

}  // namespace

void partial_to_double(const long long *partial, size_t slots, int scale_exp, double *out) {
    const double inv = std::ldexp(1.0, -scale_exp);
    for (size_t s = 0; s < slots; ++s) {
        const long long *q = partial + s * kPartialWords;
        // sum of limbs * 2^(32 k), wrapped to 128 bits like the device sums
        unsigned __int128 u = 0;
        for (int k = 3; k >= 0; --k) u = (u << 32) + (unsigned __int128)(__int128)q[k];
        const unsigned long long w[2] = {(unsigned long long)u, (unsigned long long)(u >> 64)};
        double v = fixed_to_double(w, inv);
        const bool nan = q[4] > 0 || (q[5] > 0 && q[6] > 0);
        if (nan) v = std::copysign(std::numeric_limits<double>::quiet_NaN(), -1.0);
        else if (q[5] > 0) v = std::numeric_limits<double>::infinity();
        else if (q[6] > 0) v = -std::numeric_limits<double>::infinity();
        out[s] = v;
    }
}

namespace {

// The device scratch of one count, from the context's pool.
struct CountScratch {
    ScratchBuf<WorkItem> items;
    ScratchBuf<Segment> segs;
    ScratchBuf<unsigned long long> full, sub, cnt;
    ScratchBuf<int> head, err;
    ScratchBuf<float> t1, t2, up_thr;
    ScratchBuf<unsigned char> l1, l2;
    ScratchBuf<unsigned> flags;
    ScratchBuf<double> up_bins, up_centre;
    ScratchBuf<JobK> jobs;
    ScratchBuf<double> adj_G, grad_a, grad_b;
    CountBuffers D;
};

int alloc_scratch(Ctx *ctx, const CountPlan &C, CountScratch &S, Error *err) {
    const Binning *bin = C.bin;
    const Ctx &X = *ctx;
    TPCF_TRY(S.items.alloc(X, C.items.size()));
    TPCF_TRY(S.segs.alloc(X, C.segs.size()));
    TPCF_TRY(S.full.alloc(X, 2 * (size_t)C.nb));
    TPCF_TRY(S.sub.alloc(X, 2 * (size_t)C.nb * C.n_jk));
    TPCF_TRY(S.cnt.alloc(X, 4));
    TPCF_TRY(S.head.alloc(X, 1));
    TPCF_TRY(S.err.alloc(X, kErrWords));
    TPCF_TRY(S.t1.alloc(X, bin->t1.size()));
    TPCF_TRY(S.t2.alloc(X, std::max<size_t>(bin->t2.size(), 1)));
    TPCF_TRY(S.l1.alloc(X, LUT1_N));
    TPCF_TRY(S.l2.alloc(X, LUT2_N));
    if (C.n_flags()) TPCF_TRY(S.flags.alloc(X, C.n_flags()));
    if (C.up) {
        TPCF_TRY(S.up_thr.alloc(X, C.n_up()));
        TPCF_TRY(S.up_bins.alloc(X, C.n_up()));
        TPCF_TRY(S.up_centre.alloc(X, C.n_up()));
    }
    TPCF_TRY(S.jobs.alloc(X, C.jobs.size()));
    if (C.adj) {
        TPCF_TRY(S.adj_G.alloc(X, C.nb));
        TPCF_TRY(S.grad_a.alloc(X, std::max(C.n_a, 1)));
        if (!C.is_auto) TPCF_TRY(S.grad_b.alloc(X, std::max(C.n_b, 1)));
    }
    CountBuffers &D = S.D;
    D.jobs = S.jobs.p;
    D.adj_G = S.adj_G.p;
    D.grad_a = S.grad_a.p;
    D.grad_b = S.grad_b.p;
    D.items = S.items.p;
    D.segs = S.segs.p;
    D.full = S.full.p;
    D.sub = S.sub.p;
    D.cnt = S.cnt.p;
    D.head = S.head.p;
    D.err = S.err.p;
    D.t1 = S.t1.p;
    D.t2 = S.t2.p;
    D.l1 = S.l1.p;
    D.l2 = S.l2.p;
    D.flags = C.n_flags() ? S.flags.p : nullptr;
    D.up_thr = S.up_thr.p;
    D.up_bins = S.up_bins.p;
    D.up_centre = S.up_centre.p;
    return 0;
}

// A pinned staging slot of at least `bytes`; the slot's previous count has
// finished when this is called.
int pinned_slot(Ctx *ctx, int k, size_t bytes, unsigned char **out, size_t *cap, Error *err) {
    if (ctx->pinned_cap[k] < bytes) {
        if (ctx->pinned[k]) cudaFreeHost(ctx->pinned[k]);
        ctx->pinned[k] = nullptr;
        ctx->pinned_cap[k] = 0;
        const size_t want = bytes + bytes / 2 + 4096;
        TPCF_TRY(cudaHostAlloc((void **)&ctx->pinned[k], want, cudaHostAllocDefault));
        ctx->pinned_cap[k] = want;
    }
    *out = ctx->pinned[k];
    *cap = ctx->pinned_cap[k];
    return 0;
}

// ---- autotuning of counts (Ctx::autotune)
//
// A count class -- mode, regions, unit or plain weights, precision, weight
// kind, auto or cross, number of bins, and the two catalogues' points per
// cell of side r_max to within a factor of two -- gets the refinement (1-3
// cells per r_max) and kernel configuration whose timed probe counted the
// most in-range pairs per second.  A probe runs one candidate on a strided
// sample of its own work list (every k-th item, at least 32 per SM, so the
// ramp-down of the last wave weighs little); its histograms are discarded.
// Every candidate gives the same histograms: any complete cell scheme visits
// the same pairs, and the configurations differ only in staging.  The
// choice is kept in the context; sharded counts are not tuned (every rank
// must plan the same work list).
std::string tune_key(const CountPlan &C, const CountRequest &req) {
    auto lg = [](double v) { return (int)std::floor(std::log2(std::max(v, 1e-9))); };
    char b[160];
    std::snprintf(b, sizeof b, "mode %d, regions %d, unit weights %d, fp64 %d, weight kind %d, auto %d, bins %d, "
                  "density 2^%d / 2^%d", C.bin->mode, C.jk ? 1 : 0, C.unitw ? 1 : 0, req.exact_fp64 ? 1 : 0, C.wk,
                  C.is_auto ? 1 : 0, C.nb, lg(C.dens_a), lg(C.dens_b));
    return b;
}

// A cross count whose two catalogues may play either role: plain weights or
// inverse-p DR weights (the weight product and the angular up-weight of
// 1 - cos(theta) are symmetric in the two points, and DR reads no masks);
// not an adjoint, whose gradients are per catalogue.
bool swappable(const CountRequest &req) {
    return req.b != nullptr && req.b != req.a && !req.adj_G &&
           (req.weighting == WEIGHTS_PLAIN || req.weighting == WEIGHTS_INVP_DR);
}

// The request with its catalogues in the order it asks for (swap = 1: b's
// points in registers, a's streamed in tiles).
void apply_order(const Ctx *ctx, CountRequest &req) {
    const int s = req.swap >= 0 ? req.swap : std::max(ctx->swap, 0);
    req.swap = s;
    if (s == 1 && swappable(req)) std::swap(req.a, req.b);
}

int tune_probe(Ctx *ctx, const CountRequest &req, int m, int cfg, int swap, double *rate, Error *err) {
    CountRequest r = req;
    r.refinement = m;
    r.kernel_cfg = cfg;
    r.swap = swap;
    apply_order(ctx, r);
    CountPlan C;
    if (plan_count(ctx, r, true, C, err)) return err->status;
    const size_t want = std::max<size_t>((size_t)32 * ctx->num_sms, C.items.size() / 16);
    if (C.items.size() > want) {
        const size_t stride = C.items.size() / want;
        std::vector<WorkItem> sample;
        sample.reserve(C.items.size() / stride + 1);
        for (size_t k = 0; k < C.items.size(); k += stride) sample.push_back(C.items[k]);
        C.items.swap(sample);
        C.P.n_items = (int)C.items.size();
    }
    CountScratch S;
    if (alloc_scratch(ctx, C, S, err)) return err->status;
    std::vector<double> full(C.nb), reg((size_t)C.nb * std::max(C.n_jk, 1));
    Stats st;
    if (execute(ctx, C, S.D, full.data(), reg.data(), &st, err, true)) return err->status;
    *rate = st.ms_kernel > 0 ? (double)st.in_range / (st.ms_kernel * 1e-3) : 0.0;
    return 0;
}

// The tuned refinement and kernel configuration into `req` (probing the
// count's class the first time it is met).  Leaves `req` as it is when
// autotuning is off or the caller fixed either choice.
int autotune(Ctx *ctx, CountRequest &req, Error *err) {
    if (!ctx->autotune || req.n_shards > 1 || req.refinement > 0 || ctx->refinement > 0 ||
        req.kernel_cfg >= 0 || ctx->kernel_cfg >= 0 || req.swap >= 0 || ctx->swap >= 0)
        return 0;
    CountPlan C0;
    if (plan_count(ctx, req, true, C0, err, true)) return err->status;
    const std::string key = tune_key(C0, req);
    auto it = ctx->tuned.find(key);
    if (it == ctx->tuned.end()) {
        Ctx::Tuned t;
        t.rate.assign(12, 0.0);
        double best = -1.0;
        for (int swap = 0; swap < (swappable(req) ? 2 : 1); ++swap)
            for (int cfg = 0; cfg < (C0.cfg_tunable ? 2 : 1); ++cfg)
                for (int m = 1; m <= 3; ++m) {
                    double r = 0.0;
                    if (tune_probe(ctx, req, m, cfg, swap, &r, err)) return err->status;
                    t.rate[(size_t)(m - 1) + 3 * (size_t)cfg + 6 * (size_t)swap] = r;
                    if (r > best) {
                        best = r;
                        t.m = m;
                        t.cfg = cfg;
                        t.swap = swap;
                    }
                }
        if (trace_enabled()) {
            std::fprintf(stderr, "[tpcf trace] autotune %s: pairs/s", key.c_str());
            for (double r : t.rate) std::fprintf(stderr, " %.3g", r);
            std::fprintf(stderr, " -> refinement %d, configuration %d, order %d\n", t.m, t.cfg, t.swap);
        }
        it = ctx->tuned.emplace(key, t).first;
    }
    req.refinement = it->second.m;
    req.kernel_cfg = it->second.cfg;
    req.swap = it->second.swap;
    return 0;
}

}  // namespace

int run_count(Ctx *ctx, const CountRequest &req_in, double *full_out, double *region_out, Stats *st, Error *err) {
    CountRequest req = req_in;
    if (autotune(ctx, req, err)) return err->status;
    apply_order(ctx, req);
    CountPlan C;
    if (plan_count(ctx, req, true, C, err)) return err->status;
    if (req.scale_exp_out) *req.scale_exp_out = C.scale_exp;
    CountScratch S;
    if (alloc_scratch(ctx, C, S, err)) return err->status;
    return execute(ctx, C, S.D, full_out, region_out, st, err, true);
}

int run_count_many(Ctx *ctx, const std::vector<CountRequest> &reqs_in, const std::vector<CountOut> &outs,
                   Error *err) {
    std::vector<CountRequest> reqs(reqs_in);
    for (CountRequest &r : reqs) {
        if (autotune(ctx, r, err)) return err->status;
        apply_order(ctx, r);
    }
    // TPCF_TRACE=1: one stderr line per count with its host planning time
    // and where its kernel ran on the device, in ms from the call's start
    // (diagnostics of the pipelining; the counts are unchanged)
    const bool trace = trace_enabled();
    using clk = std::chrono::steady_clock;
    const auto h0 = clk::now();
    auto host_ms = [&](clk::time_point a) { return std::chrono::duration<double, std::milli>(clk::now() - a).count(); };
    struct EventGuard {
        cudaEvent_t e = nullptr;
        ~EventGuard() {
            if (e) cudaEventDestroy(e);
        }
    } start;
    if (trace) {
        TPCF_TRY(cudaEventCreate(&start.e));
        TPCF_TRY(cudaEventRecord(start.e, ctx->stream));
    }
    const cudaEvent_t ev0 = start.e;
    // every grid first: a grid build reads its cell tables back, which would
    // otherwise wait for the count kernel ahead of it on the stream
    for (const CountRequest &req : reqs) {
        CountPlan C;
        if (plan_count(ctx, req, true, C, err, true)) return err->status;
    }
    if (trace) std::fprintf(stderr, "[tpcf trace] %zu counts: grids built at %.1f ms (host)\n", reqs.size(), host_ms(h0));
    struct Flight {
        CountPlan C;
        CountScratch S;
        HostIO io;
        const CountOut *out = nullptr;
        size_t index = 0;
        double plan_ms = 0;
    };
    std::unique_ptr<Flight> prev;
    auto finish = [&](std::unique_ptr<Flight> &f) -> int {
        if (!f) return 0;
        const int rc = finish_count(ctx, f->C, f->S.D, f->io, f->out->full, f->out->region, f->out->st, err, true);
        if (trace && !rc) {
            float k0 = 0, k1 = 0;
            cudaEventElapsedTime(&k0, ev0, f->io.e0);
            cudaEventElapsedTime(&k1, ev0, f->io.e1);
            std::fprintf(stderr, "[tpcf trace] count %zu: %zu items, %zu segments, plan %.1f ms (host); "
                         "kernel %.1f-%.1f ms (device); finished at %.1f ms (host)\n", f->index, f->C.items.size(),
                         f->C.segs.size(), f->plan_ms, k0, k1, host_ms(h0));
        }
        f.reset();
        return rc;
    };
    for (size_t i = 0; i < reqs.size(); ++i) {
        std::unique_ptr<Flight> f(new Flight());
        f->out = &outs[i];
        f->index = i;
        // planned on the host while the previous count runs
        const auto hp = clk::now();
        int rc = plan_count(ctx, reqs[i], true, f->C, err);
        f->plan_ms = host_ms(hp);
        if (!rc) rc = alloc_scratch(ctx, f->C, f->S, err);
        if (!rc) rc = pinned_slot(ctx, (int)(i & 1), stage_bytes(f->C), &f->io.stage, &f->io.stage_cap, err);
        if (!rc) rc = launch_count(ctx, f->C, f->S.D, f->io, err, true);
        if (rc) {
            cudaStreamSynchronize(ctx->stream);
            return err->status ? err->status : 3;
        }
        // the previous count's results, while this one runs
        rc = finish(prev);
        if (rc) {
            cudaStreamSynchronize(ctx->stream);
            return rc;
        }
        prev = std::move(f);
    }
    return finish(prev);
}

// ---------------------------------------------------------------------------
// Batched counts.

namespace {

int plan_batch(Ctx *ctx, const std::vector<BatchJobSpec> &jobs, const Binning *bin, bool exact, int m, CountPlan &C,
               Error *err) {
    if (bin->mode == MODE_ANGULAR) {
        err->status = 6;
        err->msg = "batched counts are 3-D counts";
        return err->status;
    }
    C.bin = bin;
    C.nb = bin->nb;
    C.n_jk = bin->n_jk;
    C.jk = true;  // per-item flushes to each job's own histograms
    C.wk = W_PLAIN;
    bool unitw = true;
    double wmax = 0, wa_max = 0;
    for (const BatchJobSpec &j : jobs) {
        const Catalog *A = j.a, *B = j.b ? j.b : j.a;
        unitw = unitw && A->unit_weights && B->unit_weights;
        wmax = std::max(wmax, (double)A->w_max * (double)B->w_max);
        wa_max = std::max(wa_max, (double)std::max(A->w_max, B->w_max));
    }
    C.unitw = unitw;
    const double rb = bin->rmax_bound;
    const double side = rb / m * (1.0 + 1e-9);
    GridSpec gs;
    gs.side = side;
    std::vector<long long> cost;
    for (size_t j = 0; j < jobs.size(); ++j) {
        Catalog *A = const_cast<Catalog *>(jobs[j].a);
        Catalog *B = const_cast<Catalog *>(jobs[j].b ? jobs[j].b : jobs[j].a);
        const bool is_auto = jobs[j].b == nullptr;
        Grid *ga = nullptr, *gb = nullptr;
        if (build_grid(ctx, A, gs, exact, &ga, err)) return err->status;
        if (is_auto) gb = ga;
        else if (build_grid(ctx, B, gs, exact, &gb, err)) return err->status;
        JobK jk;
        std::memset(&jk, 0, sizeof(jk));
        fill_grid(jk.a, *ga, *A);
        fill_grid(jk.b, *gb, *B);
        jk.out = (int)j;
        C.jobs.push_back(jk);
        if (A->n_kept == 0 || B->n_kept == 0) continue;
        std::vector<WorkItem> it;
        std::vector<Segment> sg;
        build_work_items(*ga, *gb, is_auto, m, side, rb, it, sg);
        const int off = (int)C.segs.size();
        for (WorkItem w : it) {
            long long bl = 0;
            for (int k = w.seg_begin; k < w.seg_end; ++k) bl += sg[k].b_len;
            w.seg_begin += off;
            w.seg_end += off;
            w.job = (int)j;
            C.items.push_back(w);
            cost.push_back((long long)w.a_len * bl);
        }
        C.segs.insert(C.segs.end(), sg.begin(), sg.end());
    }
    // one order over every job's items: larger first by power-of-two cost
    // class (a balanced end of the queue), each job's items in cell order
    // inside a class (neighbouring cells in flight together share their B
    // tiles in L2)
    auto cls = [](long long c) { return c > 0 ? 63 - __builtin_clzll((unsigned long long)c) : -1; };
    std::vector<int> order(C.items.size());
    for (size_t k = 0; k < order.size(); ++k) order[k] = (int)k;
    std::stable_sort(order.begin(), order.end(), [&](int x, int y) { return cls(cost[x]) > cls(cost[y]); });
    std::vector<WorkItem> sorted(C.items.size());
    for (size_t k = 0; k < order.size(); ++k) sorted[k] = C.items[order[k]];
    C.items.swap(sorted);

    float wscale = 1.0f;
    if (!unitw) {
        const int S = fixed_point_shift(wmax, max_item_pairs(C.items, C.segs), wa_max);
        wscale = std::ldexp(1.0f, S);
        C.inv = std::ldexp(1.0, -S);
    }
    C.L = smem_layout(C.nb, bin->nb1, bin->nb2, exact, true);
    if (C.L.total + 1024 > ctx->smem_optin) {
        err->status = 6;
        err->msg = "histogram does not fit in shared memory";
        return err->status;
    }
    const Guards g = compute_guards(side, m, rb);
    C.luts = build_luts(*bin, g);
    C.L = smem_layout(C.nb, bin->nb1, bin->nb2, exact, true, false, 0,
                      (bin->mode == MODE_SIGMA_PI || bin->mode == MODE_S_MU) && !C.luts.direct2);
    fill_params(C, bin, g, side, 2.0, wscale, 0);
    C.P.job0 = C.jobs[0];
    C.fn = pick(bin->mode, W_PLAIN, unitw, true, exact);
    return 0;
}

}  // namespace

struct Batch {
    Ctx *ctx = nullptr;
    CountPlan C;
    int m = 0, grid = 0;
    int order = 0;  // 1: the DR jobs count the shared catalogue's points against each mock's
    size_t n_out = 0;
    DevBuf<WorkItem> items;
    DevBuf<Segment> segs;
    DevBuf<JobK> jobs;
    DevBuf<unsigned long long> full, sub, cnt;
    DevBuf<int> head, err;
    DevBuf<float> t1, t2;
    DevBuf<unsigned char> l1, l2;
    unsigned long long *h_full = nullptr, *h_sub = nullptr, *h_cnt = nullptr;  // pinned
    int *h_err = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    ~Batch() {
        if (exec) cudaGraphExecDestroy(exec);
        if (graph) cudaGraphDestroy(graph);
        if (h_full) cudaFreeHost(h_full);
        if (h_sub) cudaFreeHost(h_sub);
        if (h_cnt) cudaFreeHost(h_cnt);
        if (h_err) cudaFreeHost(h_err);
    }
};

namespace {

// Plan, allocate and upload a batch for one refinement, then capture its
// run (clears, the launch, the read-backs) as a CUDA graph.
// sample: keep every k-th work item only (at least 32 per SM), for the
// autotuner's timed probes.
int batch_build(Ctx *ctx, const std::vector<BatchJobSpec> &jobs, const Binning *bin, bool exact, int m,
                std::unique_ptr<Batch> &out, Error *err, bool sample = false) {
    std::unique_ptr<Batch> B(new Batch());
    B->ctx = ctx;
    B->m = m;
    CountPlan &C = B->C;
    if (plan_batch(ctx, jobs, bin, exact, m, C, err)) return err->status;
    if (sample) {
        const size_t want = std::max<size_t>((size_t)32 * ctx->num_sms, C.items.size() / 16);
        if (C.items.size() > want) {
            const size_t stride = C.items.size() / want;
            std::vector<WorkItem> kept;
            for (size_t k = 0; k < C.items.size(); k += stride) kept.push_back(C.items[k]);
            C.items.swap(kept);
            C.P.n_items = (int)C.items.size();
        }
    }
    B->n_out = C.jobs.size();
    const size_t nb = C.nb, nj = C.n_jk;
    cudaStream_t stm = ctx->stream;
    TPCF_TRY(B->items.alloc(C.items.size()));
    TPCF_TRY(B->segs.alloc(C.segs.size()));
    TPCF_TRY(B->jobs.alloc(C.jobs.size()));
    TPCF_TRY(B->full.alloc(2 * nb * B->n_out));
    TPCF_TRY(B->sub.alloc(2 * nb * nj * B->n_out));
    TPCF_TRY(B->cnt.alloc(4));
    TPCF_TRY(B->head.alloc(1));
    TPCF_TRY(B->err.alloc(kErrWords));
    TPCF_TRY(B->t1.alloc(bin->t1.size()));
    TPCF_TRY(B->t2.alloc(std::max<size_t>(bin->t2.size(), 1)));
    TPCF_TRY(B->l1.alloc(LUT1_N));
    TPCF_TRY(B->l2.alloc(LUT2_N));
    TPCF_TRY(cudaMallocHost((void **)&B->h_full, sizeof(unsigned long long) * 2 * nb * B->n_out));
    TPCF_TRY(cudaMallocHost((void **)&B->h_sub, sizeof(unsigned long long) * 2 * nb * nj * B->n_out));
    TPCF_TRY(cudaMallocHost((void **)&B->h_cnt, sizeof(unsigned long long) * 4));
    TPCF_TRY(cudaMallocHost((void **)&B->h_err, sizeof(int) * kErrWords));
    if (!C.items.empty()) {
        TPCF_TRY(cudaMemcpyAsync(B->items.p, C.items.data(), sizeof(WorkItem) * C.items.size(),
                                 cudaMemcpyHostToDevice, stm));
        TPCF_TRY(cudaMemcpyAsync(B->segs.p, C.segs.data(), sizeof(Segment) * C.segs.size(), cudaMemcpyHostToDevice,
                                 stm));
    }
    TPCF_TRY(cudaMemcpyAsync(B->jobs.p, C.jobs.data(), sizeof(JobK) * C.jobs.size(), cudaMemcpyHostToDevice, stm));
    TPCF_TRY(cudaMemcpyAsync(B->t1.p, bin->t1.data(), sizeof(float) * bin->t1.size(), cudaMemcpyHostToDevice, stm));
    if (!bin->t2.empty())
        TPCF_TRY(cudaMemcpyAsync(B->t2.p, bin->t2.data(), sizeof(float) * bin->t2.size(), cudaMemcpyHostToDevice, stm));
    TPCF_TRY(cudaMemcpyAsync(B->l1.p, C.luts.l1.data(), LUT1_N, cudaMemcpyHostToDevice, stm));
    TPCF_TRY(cudaMemcpyAsync(B->l2.p, C.luts.l2.data(), LUT2_N, cudaMemcpyHostToDevice, stm));
    TPCF_TRY(cudaStreamSynchronize(stm));

    KParams P = C.P;
    P.n_segs = (int)C.segs.size();
    P.n_jobs = (int)C.jobs.size();
    P.jobs = B->jobs.p;
    P.items = B->items.p;
    P.segs = B->segs.p;
    P.head = B->head.p;
    P.t1g = B->t1.p;
    P.t2g = B->t2.p;
    P.lut1g = B->l1.p;
    P.lut2g = B->l2.p;
    P.g_full = B->full.p;
    P.g_sub = B->sub.p;
    P.counters = B->cnt.p;
    P.err = B->err.p;
    TPCF_TRY(cudaFuncSetAttribute((const void *)C.fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)C.L.total));
    int per_sm = 1;
    TPCF_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, C.fn, NT, C.L.total));
    per_sm = std::max(per_sm, 1);
    B->grid = (int)std::min<long long>((long long)ctx->num_sms * per_sm, std::max<long long>(C.items.size(), 1));

    TPCF_TRY(cudaStreamBeginCapture(stm, cudaStreamCaptureModeThreadLocal));
    cudaMemsetAsync(B->full.p, 0, sizeof(unsigned long long) * 2 * nb * B->n_out, stm);
    cudaMemsetAsync(B->sub.p, 0, sizeof(unsigned long long) * 2 * nb * nj * B->n_out, stm);
    cudaMemsetAsync(B->cnt.p, 0, sizeof(unsigned long long) * 4, stm);
    cudaMemsetAsync(B->head.p, 0, sizeof(int), stm);
    cudaMemsetAsync(B->err.p, 0, sizeof(int) * kErrWords, stm);
    if (!C.items.empty()) C.fn<<<B->grid, NT, C.L.total, stm>>>(P);
    cudaMemcpyAsync(B->h_full, B->full.p, sizeof(unsigned long long) * 2 * nb * B->n_out, cudaMemcpyDeviceToHost, stm);
    cudaMemcpyAsync(B->h_sub, B->sub.p, sizeof(unsigned long long) * 2 * nb * nj * B->n_out, cudaMemcpyDeviceToHost,
                    stm);
    cudaMemcpyAsync(B->h_cnt, B->cnt.p, sizeof(unsigned long long) * 4, cudaMemcpyDeviceToHost, stm);
    cudaMemcpyAsync(B->h_err, B->err.p, sizeof(int) * kErrWords, cudaMemcpyDeviceToHost, stm);
    TPCF_TRY(cudaStreamEndCapture(stm, &B->graph));
    TPCF_TRY(cudaGraphInstantiate(&B->exec, B->graph, 0));
    out = std::move(B);
    return 0;
}

}  // namespace

int batch_run(Batch *B, double *full_out, double *region_out, Stats *st, Error *err) {
    Ctx *ctx = B->ctx;
    const CountPlan &C = B->C;
    cudaStream_t stm = ctx->stream;
    cudaEvent_t e0, e1;
    TPCF_TRY(cudaEventCreate(&e0));
    TPCF_TRY(cudaEventCreate(&e1));
    TPCF_TRY(cudaEventRecord(e0, stm));
    TPCF_TRY(cudaGraphLaunch(B->exec, stm));
    TPCF_TRY(cudaEventRecord(e1, stm));
    TPCF_TRY(cudaStreamSynchronize(stm));
    float ms = 0;
    cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (!C.items.empty()) ++ctx->launches;
    if (*B->h_err) return device_error(B->h_err, err);
    const size_t nb = C.nb, nj = C.n_jk;
    for (size_t k = 0; k < nb * B->n_out; ++k) full_out[k] = fixed_to_double(&B->h_full[2 * k], C.inv);
    if (region_out)
        for (size_t k = 0; k < nb * nj * B->n_out; ++k) region_out[k] = fixed_to_double(&B->h_sub[2 * k], C.inv);
    if (st) {
        st->candidates += B->h_cnt[0];
        st->in_range += B->h_cnt[1];
        st->guard += B->h_cnt[2];
        st->overflow += B->h_cnt[3];
        st->items += C.items.size();
        st->ms_kernel += ms;
    }
    return 0;
}

int batch_create(Ctx *ctx, const std::vector<BatchJobSpec> &jobs, const Binning *bin, bool exact_fp64, int refinement,
                 Batch **out, Error *err) {
    *out = nullptr;
    if (jobs.empty()) {
        err->status = 1;
        err->msg = "empty batch";
        return err->status;
    }
    if (refinement < 0) {
        // autotune: every (refinement 1-3, order) candidate planned on a
        // strided sample of its work items and timed once; the one that
        // counted the most in-range pairs per second is built in full.  Order
        // 1 swaps the catalogues of the DR jobs (the shared catalogue's points
        // in registers, the mock's streamed); the histograms are the same.
        bool any_cross = false;
        for (const BatchJobSpec &j : jobs) any_cross = any_cross || (j.b && j.b != j.a);
        std::vector<BatchJobSpec> swapped(jobs);
        for (BatchJobSpec &j : swapped)
            if (j.b && j.b != j.a) std::swap(j.a, j.b);
        int best_m = 0, best_order = 0;
        double best_rate = -1.0;
        for (int order = 0; order < (any_cross ? 2 : 1); ++order)
            for (int m = 1; m <= 3; ++m) {
                std::unique_ptr<Batch> b;
                if (batch_build(ctx, order ? swapped : jobs, bin, exact_fp64, m, b, err, true)) {
                    if (err->status == 6) continue;  // e.g. a grid too fine for this refinement
                    return err->status;
                }
                std::vector<double> f(b->C.nb * b->n_out);
                Stats st;
                if (batch_run(b.get(), f.data(), nullptr, &st, err)) return err->status;
                const double rate = st.ms_kernel > 0 ? (double)st.in_range / st.ms_kernel : 0.0;
                if (rate > best_rate) {
                    best_rate = rate;
                    best_m = m;
                    best_order = order;
                }
            }
        if (best_m == 0) {
            err->status = 6;
            err->msg = "no refinement could be planned";
            return err->status;
        }
        std::unique_ptr<Batch> b;
        if (batch_build(ctx, best_order ? swapped : jobs, bin, exact_fp64, best_m, b, err)) return err->status;
        b->order = best_order;
        *out = b.release();
        return 0;
    }
    std::vector<int> choices;
    if (refinement > 0) {
        choices.push_back(refinement);
    } else {
        // as run_count: from the largest catalogue's mean density
        const Catalog *big = jobs[0].a;
        for (const BatchJobSpec &j : jobs) {
            if (j.a->n_kept > big->n_kept) big = j.a;
            if (j.b && j.b->n_kept > big->n_kept) big = j.b;
        }
        const double rb = bin->rmax_bound;
        double vol = 1;
        for (int k = 0; k < 3; ++k) vol *= std::max(big->hi_kept[k] - big->lo_kept[k], rb);
        choices.push_back(big->n_kept * (rb / 2) * (rb / 2) * (rb / 2) / vol >= 256 ? 2 : 1);
    }
    std::unique_ptr<Batch> best;
    double best_ms = 0;
    for (int m : choices) {
        std::unique_ptr<Batch> b;
        if (batch_build(ctx, jobs, bin, exact_fp64, m, b, err)) {
            if (choices.size() > 1 && err->status == 6) continue;  // e.g. a grid too fine for this refinement
            return err->status;
        }
        if (choices.size() > 1) {
            // autotune: time one replay of each candidate refinement
            std::vector<double> f(b->C.nb * b->n_out);
            Stats st;
            if (batch_run(b.get(), f.data(), nullptr, &st, err)) return err->status;
            if (!best || st.ms_kernel < best_ms) {
                best_ms = st.ms_kernel;
                best = std::move(b);
            }
        } else {
            best = std::move(b);
        }
    }
    if (!best) {
        err->status = 6;
        err->msg = "no refinement could be planned";
        return err->status;
    }
    *out = best.release();
    return 0;
}

int batch_refinement(const Batch *b) { return b->m; }
int batch_order(const Batch *b) { return b->order; }
int batch_jobs(const Batch *b) { return (int)b->n_out; }
void batch_destroy(Batch *b) { delete b; }

// ---------------------------------------------------------------------------
// Counting without device allocation.
//
// Some callers cannot call cudaMalloc while they count: applications whose
// memory manager has reserved the device's memory for its own pool (a
// framework's caching allocator, a serving process sized to the whole card),
// where a foreign allocation fails or fragments that pool, and latency-bound
// loops that cannot take the device-wide synchronisation cudaFree implies.
// For them every scratch buffer of run_count — the work list, the segment
// list, the fixed-point histograms, the counters, the work-queue head, the
// error flag, the threshold, lookup and up-weight tables — is carved from the
// one static array below, of kStaticScratchBytes (32 MiB).  Each device that
// loads the library holds that array until the process exits.
//
// The array is shared by every call on a device and keeps the contents of
// the last call; each call clears the histograms, counters, queue head, error
// flag and non-finite flags before its launch.  Two calls whose work
// overlaps on the GPU (two contexts on one device, on different streams,
// from different host threads) race on it.  Calls from one thread do not
// overlap: each waits for its results before it returns.
static __device__ __align__(256) unsigned char g_count_scratch[kStaticScratchBytes];

namespace {

constexpr int kMaxScratchDevices = 64;
std::mutex g_scratch_mutex;
void *g_scratch_addr[kMaxScratchDevices];

// Device address of g_count_scratch on `device`, which must be current.  In
// host code g_count_scratch only names the symbol; its address on a device
// comes from cudaGetSymbolAddress, looked up on the first call per device
// and remembered.
int scratch_address(int device, void **out, Error *err) {
    int cur = -1;
    cudaError_t e = cudaGetDevice(&cur);
    if (e != cudaSuccess || cur != device || device < 0 || device >= kMaxScratchDevices) {
        err->status = 3;
        err->msg = "static scratch: device " + std::to_string(device) + " is not current or out of range";
        return err->status;
    }
    std::lock_guard<std::mutex> lock(g_scratch_mutex);
    if (!g_scratch_addr[device]) {
        void *p = nullptr;
        e = cudaGetSymbolAddress(&p, g_count_scratch);
        if (e != cudaSuccess || !p) {
            err->status = 3;
            err->msg = std::string("static scratch: cudaGetSymbolAddress failed: ") + cudaGetErrorString(e);
            return err->status;
        }
        g_scratch_addr[device] = p;
    }
    *out = g_scratch_addr[device];
    return 0;
}

// Byte offsets of the buffers inside the static array, each 256-aligned.
struct ScratchPlan {
    size_t total = 0;
    size_t take(size_t bytes) {
        const size_t off = total;
        total += (std::max<size_t>(bytes, 1) + 255) & ~size_t(255);
        return off;
    }
};

}  // namespace

int run_count_static(Ctx *ctx, const CountRequest &req, double *full_out, double *region_out, Stats *st,
                     Error *err) {
    const Binning *bin = req.bin;
    if (req.adj_G) {
        err->status = 6;
        err->msg = "the allocation-free count has no adjoint";
        return err->status;
    }
    const int nb = bin->nb, n_jk = bin->n_jk;
    // The histogram and table part of the scratch is known before the work
    // list is built; refuse an oversized binning before anything else.
    ScratchPlan sp;
    const size_t o_full = sp.take(sizeof(unsigned long long) * 2 * nb);
    const size_t o_sub = sp.take(sizeof(unsigned long long) * 2 * (size_t)nb * n_jk);
    const size_t o_cnt = sp.take(sizeof(unsigned long long) * 4);
    const size_t o_head = sp.take(sizeof(int));
    const size_t o_err = sp.take(sizeof(int) * kErrWords);
    const size_t o_t1 = sp.take(sizeof(float) * bin->t1.size());
    const size_t o_t2 = sp.take(sizeof(float) * std::max<size_t>(bin->t2.size(), 1));
    const size_t o_l1 = sp.take(LUT1_N);
    const size_t o_l2 = sp.take(LUT2_N);
    const size_t n_up = req.up ? req.up->thr.size() : 0;
    const size_t o_up_thr = sp.take(sizeof(float) * n_up);
    const size_t o_up_bins = sp.take(sizeof(double) * n_up);
    const size_t o_up_centre = sp.take(sizeof(double) * n_up);
    const size_t o_jobs = sp.take(sizeof(JobK));
    auto too_big = [&](size_t n_items, size_t n_segs) {
        err->status = 6;
        err->msg = "count needs " + std::to_string(sp.total) + " bytes of scratch (" + std::to_string(nb) +
                   " bins x " + std::to_string(n_jk) + " regions, " + std::to_string(n_items) + " work items, " +
                   std::to_string(n_segs) + " segments); the static scratch holds " +
                   std::to_string(kStaticScratchBytes) + " bytes: use tpcf_count";
        return err->status;
    };
    if (sp.total > kStaticScratchBytes) return too_big(0, 0);

    CountPlan C;
    if (plan_count(ctx, req, false, C, err)) return err->status;
    // non-finite flags: exactly what the kernel and finish_count use (none
    // for plain weights, and none for an angular count of inverse-p DR
    // weights, whose plan has plain pair weights)
    const size_t n_flags = C.n_flags();
    const size_t o_flags = sp.take(sizeof(unsigned) * n_flags);
    const size_t o_items = sp.take(sizeof(WorkItem) * C.items.size());
    const size_t o_segs = sp.take(sizeof(Segment) * C.segs.size());
    if (sp.total > kStaticScratchBytes) return too_big(C.items.size(), C.segs.size());

    void *base = nullptr;
    if (scratch_address(ctx->device, &base, err)) return err->status;
    unsigned char *p = static_cast<unsigned char *>(base);
    CountBuffers D;
    D.items = reinterpret_cast<WorkItem *>(p + o_items);
    D.segs = reinterpret_cast<Segment *>(p + o_segs);
    D.full = reinterpret_cast<unsigned long long *>(p + o_full);
    D.sub = reinterpret_cast<unsigned long long *>(p + o_sub);
    D.cnt = reinterpret_cast<unsigned long long *>(p + o_cnt);
    D.head = reinterpret_cast<int *>(p + o_head);
    D.err = reinterpret_cast<int *>(p + o_err);
    D.t1 = reinterpret_cast<float *>(p + o_t1);
    D.t2 = reinterpret_cast<float *>(p + o_t2);
    D.l1 = p + o_l1;
    D.l2 = p + o_l2;
    D.flags = n_flags ? reinterpret_cast<unsigned *>(p + o_flags) : nullptr;
    D.up_thr = reinterpret_cast<float *>(p + o_up_thr);
    D.up_bins = reinterpret_cast<double *>(p + o_up_bins);
    D.up_centre = reinterpret_cast<double *>(p + o_up_centre);
    D.jobs = reinterpret_cast<JobK *>(p + o_jobs);
    return execute(ctx, C, D, full_out, region_out, st, err, false);
}

}  // namespace tpcf
