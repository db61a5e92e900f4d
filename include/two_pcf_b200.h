/*
 * two_pcf_b200 — C ABI of the B200 grid-binned pair-counting engine.
 *
 * This is the drop-in boundary for the hot path of lstothert/two_pcf: the
 * reference's GalaxyBoxes + auto_/cross_pair_count_* + JKHists machinery
 * (src/boxes.h:16-39, src/correlators.h:7-31, src/hist.h:21-107,
 * src/correlators_invpweight.h:14-42).  Plain pointers and sizes only; every
 * call returns a status (0 = TPCF_OK) and no exception crosses it.  Host
 * buffers passed in are borrowed for the duration of the call.
 *
 * Threading: one tpcf_ctx per host thread; calls on one context are
 * serialised on its CUDA stream.
 */
#ifndef TWO_PCF_B200_H
#define TWO_PCF_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define TPCF_ABI_VERSION 1

typedef enum {
    TPCF_OK = 0,
    TPCF_E_INVALID_ARG = 1,     /* bad pointer, size, NaN coordinate, region index out of range */
    TPCF_E_OOM = 2,             /* device allocation failed */
    TPCF_E_CUDA = 3,            /* any other CUDA runtime error */
    TPCF_E_DEVICE_TIMEOUT = 4,  /* a bounded device wait gave up; results discarded */
    TPCF_E_OVERFLOW = 5,        /* a fixed-point histogram bin would overflow */
    TPCF_E_UNSUPPORTED = 6,     /* configuration outside the engine's limits */
    TPCF_E_DEVICE_CHECK = 7     /* a device bounds check failed (checked build only); results discarded */
} tpcf_status;

typedef enum {
    TPCF_MONOPOLE = 0, /* Hist on s                        (src/correlators.cpp:127-153) */
    TPCF_SIGMA_PI = 1, /* Hist2D on (sigma, |pi|)          (src/correlators.cpp:280-307) */
    TPCF_S_MU = 2,     /* Hist2D on (s, mu), mu in [0, 1]  (src/correlators.cpp:432-459) */
    TPCF_ANGULAR = 3   /* Hist on 1 - cos(theta)           (src/correlators_invpweight.cpp:985-1033);
                          ax1 = (0, 1 - cos(theta_max), theta_log_base, theta_n_bins) */
} tpcf_mode;

typedef enum {
    TPCF_FP32_GUARD = 0, /* FP32 from cell-relative coordinates, exact re-check near every edge */
    TPCF_FP64 = 1        /* every candidate evaluated with the reference's exact float/double sequence */
} tpcf_precision;

typedef struct tpcf_ctx tpcf_ctx;
typedef struct tpcf_catalog tpcf_catalog;
typedef struct tpcf_binning tpcf_binning;

/* One histogram axis with the parameter-file meaning (src/io.h:42-66):
 * log binning when log_base > 1.02 (src/hist.cpp:25). */
typedef struct {
    double min;
    double max;
    double log_base;
    int32_t n_bins;
} tpcf_axis_spec;

typedef struct {
    uint64_t candidates;       /* pair evaluations enumerated */
    uint64_t in_range;         /* pairs passing the reference range test (auto pairs once) */
    uint64_t guard_evals;      /* pairs re-evaluated with the exact sequence */
    uint64_t overflow_updates; /* jackknife updates that bypassed shared memory */
    uint64_t work_items;
    double ms_kernel;          /* device time of the counting kernels */
    double ms_total;           /* host wall time of the call */
} tpcf_stats;

int tpcf_abi_version(void);
const char *tpcf_status_string(int status);

/* Context on one CUDA device.  Replaces the OpenMP set-up of src/main.cpp:29-35. */
int tpcf_create(int device, tpcf_ctx **out);
int tpcf_destroy(tpcf_ctx *ctx);
const char *tpcf_last_error(const tpcf_ctx *ctx);
/* Run on a caller-owned cudaStream_t (NULL: the context's own stream). */
int tpcf_set_stream(tpcf_ctx *ctx, void *cuda_stream);
/* Cells per maximum separation (1..3; 0 = automatic). */
int tpcf_set_refinement(tpcf_ctx *ctx, int cells_per_rmax);
/* Autotuning of counts (no counterpart in the reference, whose cell side is
 * always the maximum separation, src/boxes.cpp:56-59).  on != 0: the first
 * count of each class (mode, regions, weights, precision, bins, auto or
 * cross, and the catalogues' points per cell of side r_max to within a
 * factor of two) probes cells of 1, 2 and 3 per maximum separation, for the
 * plain-weight FP32+guard kernels both kernel configurations, and for cross
 * counts with plain or inverse-p DR weights both orders (the adjoint tunes
 * its refinement only), each on a strided sample of its
 * work items, and keeps the one that counted the most in-range pairs per
 * second for every later count of the class in this context.  Counts do not
 * depend on the choice, nor do weighted sums whose pair weights all lie
 * within a factor 2^15 of the largest (the fixed-point resolution of smaller
 * ones, 2^-(S+1) in the notes of tpcf_count, follows the chosen plan).  A
 * fixed refinement, kernel configuration or order (here or per call) turns
 * the tuning off; sharded counts are never tuned. */
int tpcf_set_autotune(tpcf_ctx *ctx, int on);
/* Order of cross counts with plain or inverse-p DR weights: 0 counts a's points against b's (a's
 * points held in registers, b's streamed through shared memory), 1 the
 * reverse, -1 automatic (the autotuner's choice when it runs, else 0).  Same
 * results either way: each pair adds to the full histogram and to the rows of
 * both its regions, the pair weight is a commutative float product, and
 * swapping the points negates the separation exactly. */
int tpcf_set_cross_order(tpcf_ctx *ctx, int order);
/* Kernel configuration of the plain-weight FP32+guard kernels: 0 the default
 * per kind (jackknife kernels: three tile buffers of 256 points, ballots of
 * four A slots between queue checks; kernels without regions: two buffers,
 * two slots), 1 the alternative (jackknife: two buffers of 512 points, two
 * slots; without regions: three buffers, four slots), -1 automatic (the
 * autotuner's choice when it runs, else 0).  Same results either way. */
int tpcf_set_kernel_config(tpcf_ctx *ctx, int cfg);
/* The autotuner's choices so far as JSON text: a list of {"class", "refinement",
 * "kernel_config", "order", "pairs_per_s": [m = 1, 2, 3 with configuration 0,
 * then with configuration 1, first in order 0, then in order 1; 0 where not
 * probed]}.  Writes at most len bytes including
 * the terminating NUL; returns the length the full text needs (without the
 * NUL), or a negative status. */
int64_t tpcf_autotune_describe(const tpcf_ctx *ctx, char *buf, int64_t len);
int tpcf_synchronize(tpcf_ctx *ctx);

/* A catalogue resident on the device: the Galaxy fields of src/galaxy.h:16-35.
 *   xyz[3n]         comoving position (Galaxy::x)
 *   x_norm[3n]      unit vector (Galaxy::x_norm); NULL: x / |x| as the
 *                   cartesian reader computes it (src/io.cpp:393-399)
 *   d_comov[n]      NULL: |x|.  Points with d_comov < 0 are dropped by the
 *                   reference's partition loop (src/boxes.cpp:15-26), which is
 *                   reproduced exactly, including the points it drops early.
 *   weight[n]       Galaxy::weight (float); NULL: 1.0
 *   input_weight[n] Galaxy::input_weight (inverse-p build); NULL: weight
 *   jk_region[n]    in [0, n_jk_regions); NULL: 0
 *   bitmask[n * n_mask_ints]  Galaxy::bitmask, object-major; NULL: none
 * Replaces GalaxyBoxes(...) (src/boxes.h:30); the caller's arrays are not
 * permuted. */
int tpcf_catalog_create(tpcf_ctx *ctx, int64_t n, const double *xyz, const double *x_norm, const double *d_comov,
                        const float *weight, const float *input_weight, const int32_t *jk_region,
                        int32_t n_jk_regions, const int64_t *bitmask, int32_t n_mask_ints, tpcf_catalog **out);
/* Device arrays go back to the memory pool in the order of the legacy stream
 * (a catalogue may outlive its context and the context's stream). */
int tpcf_catalog_destroy(tpcf_catalog *cat);
/* Points kept by the d_comov partition (GalaxyBoxes::n_gals). */
int64_t tpcf_catalog_n_used(const tpcf_catalog *cat);
/* Drop the cell grids cached on the catalogue; the next count rebuilds them.
 * While the catalogue's context lives, their memory is released in the order
 * of the context's stream, which must still be valid (tpcf_set_stream). */
int tpcf_catalog_release_cache(tpcf_catalog *cat);

/* Histogram definition.  ax2 is the pi axis for TPCF_SIGMA_PI and supplies
 * only n_bins (mu bins on [0, 1]) for TPCF_S_MU; it is ignored otherwise.
 * Replaces Hist / Hist2D construction (src/hist.cpp:15-36, :64, :393).
 * Host-only: ctx may be NULL (errors are then reported by status alone). */
int tpcf_binning_create(tpcf_ctx *ctx, int mode, const tpcf_axis_spec *ax1, const tpcf_axis_spec *ax2,
                        int32_t n_jk_regions, tpcf_binning **out);
int tpcf_binning_destroy(tpcf_binning *bin);
int tpcf_binning_total_bins(const tpcf_binning *bin);
/* Threshold table of one axis (axis 1 or 2): T[0..n] with bin = #{T <= x} - 1.
 * Writes min(cap, n + 1) floats; returns n + 1, or a negative status. */
int tpcf_binning_thresholds(const tpcf_binning *bin, int axis, float *out, int cap);

/* Raw pair count.  b == NULL: auto count of a (each unordered pair once).
 *   full_out[nb]            sum of pair weights per bin
 *   region_out[n_jk * nb]   per region r: sum over pairs with either end in r
 *                           (JKHists::add_pair, src/hist.cpp:246-260), before
 *                           invert_jk_hists; may be NULL
 * Neither is doubled for auto counts.
 * Unit-weight counts are exact integers.  Weighted sums add each float pair
 * weight in fixed point (64-bit in shared memory, 128-bit in global memory)
 * with resolution 2^-(S+1), S = floor(62 - log2(wmax * P)), wmax a bound on
 * the pair weights and P the pairs of the largest work item (about 2^24):
 * every float pair weight of at least 2^(23-S), about wmax * 2^-15, is added
 * exactly, smaller ones to 2^-(S+1). */
int tpcf_count(tpcf_ctx *ctx, const tpcf_catalog *a, const tpcf_catalog *b, const tpcf_binning *bin,
               int precision, double *full_out, double *region_out, tpcf_stats *stats);

/* Pair weighting of tpcf_count_weighted (the reference's _USE_INV_WEIGHTS
 * build, src/correlators_invpweight.cpp). */
typedef enum {
    /* 3-D: weight1 * weight2 over the points kept by the d_comov partition.
     * Angular: input_weight1 * input_weight2 over every point
     * (auto/cross_pair_count_angular, :860-982). */
    TPCF_WEIGHTS_PLAIN = 0,
    /* Inverse-p DD: input_weight1 * input_weight2 * n_bitwise_runs / popc,
     * popc = number of bits set in mask1 & mask2 (1 when none), times the
     * angular up-weight in 3-D (auto_pair_count_*_invpweights, :14-709;
     * auto_pair_count_angular_invpweights, :713-818).  Angular counts use the
     * points with d_comov >= 0 (GalaxyPixels' require_redshift). */
    TPCF_WEIGHTS_INVP_DD = 1,
    /* Inverse-p DR: 3-D weight1 * weight2 * angular up-weight
     * (cross_pair_count_*_invpweights); angular weight1 * weight2 over points
     * with d_comov >= 0 (cross_pair_count_angular_invpweights). */
    TPCF_WEIGHTS_INVP_DR = 2,
    /* TPCF_WEIGHTS_INVP_DD of the build with _USE_DITHER_WEIGHTS
     * (src/correlators_invpweight.cpp:62-71, :749-757): n_bitwise_runs is
     * replaced per pair by the popcount of dither_mask1 & dither_mask2 (1 when
     * none).  Both catalogues need dither masks (tpcf_catalog_set_dither_masks). */
    TPCF_WEIGHTS_INVP_DD_DITHER = 3
} tpcf_weighting;

typedef struct {
    int32_t weighting;       /* tpcf_weighting */
    int32_t n_bitwise_runs;  /* Params::n_bitwise_runs */
    /* 3-D inverse-p counts only: the angular up-weight is JKHists::interp
     * (src/hist.cpp:369-391) of up_numerator / up_denominator bin by bin
     * (divide_by_hist, :224-231) on theta_axis = (0, 1 - cos(theta_max),
     * theta_log_base, theta_n_bins): the angular DD and DD-inverse-p full
     * histograms for DD counts, DR and DR-inverse-p for DR counts, as the
     * angular stage wrote them (calc_angular_upweight, :985-1033). */
    tpcf_axis_spec theta_axis;
    const double *up_numerator;
    const double *up_denominator;
} tpcf_weight_spec;

/* tpcf_count with a pair weighting (spec NULL: TPCF_WEIGHTS_PLAIN).  Angular
 * binnings (TPCF_ANGULAR) count (float)(1 - cos(theta)) of the unit vectors
 * with no separation cut.  TPCF_WEIGHTS_INVP_DD needs bitmasks of the same
 * width on both catalogues.  A pair whose up-weight is not finite (an empty
 * angular bin makes 0/0) turns its bins into NaN or an infinity, as the
 * reference's double sums do. */
int tpcf_count_weighted(tpcf_ctx *ctx, const tpcf_catalog *a, const tpcf_catalog *b, const tpcf_binning *bin,
                        const tpcf_weight_spec *spec, int precision, double *full_out, double *region_out,
                        tpcf_stats *stats);
/* The same with the reference's output convention (inverted jackknife
 * histograms, x2 for auto counts): what the *_invpweights and *_angular
 * counting functions leave in their JKHists. */
int tpcf_pair_count_weighted(tpcf_ctx *ctx, const tpcf_catalog *a, const tpcf_catalog *b, const tpcf_binning *bin,
                             const tpcf_weight_spec *spec, int precision, double *full_hist, double *sub_hist,
                             tpcf_stats *stats);
/* Adjoint of a plain-weight 3-D count (no counterpart in the reference; the
 * weight gradient of a loss on DD/DR/RR and xi).  dL_dfull[nb] is the
 * derivative of the loss with respect to the raw full histogram of
 * tpcf_count (unordered pairs, before x2).  Every counted pair (i, j) in bin
 * k adds w_j * dL_dfull[k] to dL_dw_a[i] and w_i * dL_dfull[k] to dL_dw_b[j]
 * (auto counts: both to dL_dw_a).  Outputs are indexed by catalogue index
 * (n points each; points dropped by the d_comov partition get 0).  Terms
 * are summed in 64-bit fixed point per work item (resolution about 1e-15 of
 * max|dL_dfull| * max weight times the item's points), the item sums in
 * double.  dL_dfull must be finite (else TPCF_E_INVALID_ARG).  Bin membership
 * is the forward count's, decided by the same kernels; no pair is stored
 * between the two passes. */
int tpcf_count_backward(tpcf_ctx *ctx, const tpcf_catalog *a, const tpcf_catalog *b, const tpcf_binning *bin,
                        int precision, const double *dL_dfull, double *dL_dw_a, double *dL_dw_b,
                        tpcf_stats *stats);
/* Replace a catalogue's weights (n floats, Galaxy::weight) in place: the
 * device copy and every cached cell grid.  Positions and grids are kept. */
int tpcf_catalog_set_weights(tpcf_catalog *cat, const float *weight);

/* Galaxy::dither_mask of the _USE_DITHER_WEIGHTS build (src/galaxy.h:28-30):
 * n * n_mask_ints int64 words, object-major, the width of the catalogue's
 * bitmasks. */
int tpcf_catalog_set_dither_masks(tpcf_catalog *cat, const int64_t *dither_mask);

/* Line of sight of pi in TPCF_SIGMA_PI and TPCF_S_MU binnings.
 * TPCF_LOS_ANGULAR (default): pi = (x1 - x2) . (x_norm1 + x_norm2) / 2, the
 * reference's default build (_ANGULAR_PI_DEFN, src/correlators.cpp:166-170).
 * TPCF_LOS_MIDPOINT: pi = (x1 - x2) . (x1 + x2) / |x1 + x2|, its build
 * without that flag (:172-182); counted with the exact sequence for every
 * candidate in either precision. */
typedef enum { TPCF_LOS_ANGULAR = 0, TPCF_LOS_MIDPOINT = 1 } tpcf_line_of_sight;
int tpcf_binning_set_line_of_sight(tpcf_binning *bin, int line_of_sight);

/* The inverse-p build's reading of the bitwise weights
 * (read_data_hdf5, src/io.cpp:519-586), on arrays: input_weight = weight;
 * total = popcount of the object's n_mask_ints mask words (1 when 0); where
 * total != n_bitwise_runs, weight *= n_bitwise_runs / total in double
 * (with dither_mask, not NULL: weight *= popcount(dither) / total).
 * weight[n] is updated in place; input_weight[n] receives the old values. */
int tpcf_iip_weights(int64_t n, int32_t n_mask_ints, const int64_t *bitmask, const int64_t *dither_mask,
                     int32_t n_bitwise_runs, float *weight, float *input_weight);

/* Batched counts (no single counterpart in the reference, whose driver counts
 * one catalogue at a time): DD of each mock and/or DR of each mock against a
 * shared random catalogue, as ONE persistent launch over the work items of
 * every pair.  The plan (cell grids, work list, tables, device buffers) is
 * built once by tpcf_batch_create and every tpcf_batch_run replays it as a
 * CUDA graph (clears, the launch, the read-backs).
 *   what: TPCF_BATCH_DD | TPCF_BATCH_DR; outputs are ordered mock by mock,
 *         DD then DR, each as tpcf_count returns it (raw, not doubled).
 *   refinement: cells per maximum separation 1..3, 0 automatic, or
 *         TPCF_BATCH_AUTOTUNE: each of 1, 2, 3, and for DR jobs each order
 *         (the mock's points against the randoms', or the reverse), is
 *         planned on a strided sample of its work items and timed once; the
 *         one that counted the most in-range pairs per second is built in
 *         full (tpcf_batch_refinement and tpcf_batch_order report it).  The
 *         histograms do not depend on the choice.
 * The catalogues must outlive the batch, keep their weights, and keep their
 * cached grids (no tpcf_catalog_release_cache) while it exists. */
typedef struct tpcf_batch tpcf_batch;
#define TPCF_BATCH_DD 1
#define TPCF_BATCH_DR 2
#define TPCF_BATCH_AUTOTUNE (-1)
int tpcf_batch_create(tpcf_ctx *ctx, const tpcf_catalog *const *mocks, int32_t n_mocks, const tpcf_catalog *randoms,
                      const tpcf_binning *bin, int precision, int32_t what, int32_t refinement, tpcf_batch **out);
/* full_out[n_outputs * nb]; region_out[n_outputs * n_jk * nb] or NULL. */
int tpcf_batch_run(tpcf_batch *batch, double *full_out, double *region_out, tpcf_stats *stats);
int tpcf_batch_n_outputs(const tpcf_batch *batch);
int tpcf_batch_refinement(const tpcf_batch *batch);
/* 1 when the batch counts its DR jobs the randoms' points against each mock's. */
int tpcf_batch_order(const tpcf_batch *batch);
int tpcf_batch_destroy(tpcf_batch *batch);

/* Host-side evaluation of the up-weight of a 3-D inverse-p spec at values of
 * 1 - cos(theta), with the tables and arithmetic the kernels use; replaces
 * JKHists::interp after divide_by_hist (src/hist.cpp:224-231, :369-391). */
int tpcf_upweight_eval(const tpcf_weight_spec *spec, const double *values, int64_t n, double *out);

/* tpcf_count without device allocation.  No counterpart in the reference.
 *
 * For callers that cannot call cudaMalloc while they count: applications
 * whose memory manager has reserved the device's memory for its own pool,
 * where a foreign allocation fails or fragments it, and latency-bound loops
 * that cannot take the device-wide synchronisation cudaFree implies.  Same
 * arguments, results and errors as tpcf_count; the caller passes the
 * catalogues, the binning and the output arrays as before.
 *
 * - Scratch: every device buffer the count needs (work list, segment list,
 *   fixed-point histograms, counters, tables) lives in one static device
 *   array of 32 MiB (33554432 bytes) that each device loading the library
 *   holds until the process exits.  A count that needs more (many work items,
 *   or bins x jackknife regions above ~2M) is refused with
 *   TPCF_E_UNSUPPORTED and a message giving the size; tpcf_count handles it.
 * - Set-up: the first call on a device looks up the array's device address
 *   (cudaGetSymbolAddress) with that device current; make that first call
 *   before any stream capture.
 * - Cell grids: the call builds none.  The catalogues must already hold the
 *   grid for this binning, refinement and precision, which an earlier
 *   tpcf_count (or tpcf_auto/cross_pair_count) of the same catalogues caches;
 *   otherwise TPCF_E_INVALID_ARG.  tpcf_catalog_release_cache drops them.
 * - Sharing: every call on a device uses the same array, which keeps the
 *   last call's contents; each call clears what it accumulates into.  Calls
 *   whose work overlaps on the GPU (contexts on different streams of one
 *   device, driven from several host threads) race on the array.  Calls from
 *   one thread never overlap: each returns after its results are read back.
 * - stats->ms_kernel is not measured (0); host staging buffers use the C++
 *   heap. */
int tpcf_count_noalloc(tpcf_ctx *ctx, const tpcf_catalog *a, const tpcf_catalog *b, const tpcf_binning *bin,
                       int precision, double *full_out, double *region_out, tpcf_stats *stats);

/* Several counts in one call (no counterpart in the reference, whose driver
 * runs DD, DR and RR one after another): the results are those of one
 * tpcf_count_weighted per job, in order (reference_form: those of
 * tpcf_pair_count_weighted — inverted regions, auto counts doubled).  Every
 * cell grid is built first; then each count's host work (work list, tables,
 * staging through pinned memory) runs while the previous count's kernel is
 * on the device, so the host work leaves the critical path.  stats->ms_total
 * is the wall time of the whole call. */
typedef struct {
    const tpcf_catalog *a;
    const tpcf_catalog *b;          /* NULL: auto count of a */
    const tpcf_binning *bin;
    const tpcf_weight_spec *spec;   /* NULL: TPCF_WEIGHTS_PLAIN */
    int32_t precision;
    int32_t reference_form;
    double *full_out;               /* nb */
    double *region_out;             /* n_jk * nb, or NULL (required with reference_form) */
    tpcf_stats *stats;              /* or NULL */
} tpcf_count_job;
int tpcf_count_many(tpcf_ctx *ctx, const tpcf_count_job *jobs, int32_t n_jobs);

/* One shard of a count split across processes or GPUs (strong scaling; no
 * counterpart in the reference, whose counts run on one node's threads).
 * Every shard plans the same work list (it depends only on the catalogues,
 * the binning and the refinement) and runs the items k with
 * k % n_shards == shard, dealt from the largest down.  It returns its partial
 * sums instead of doubles: per histogram slot (the nb full bins, then the
 * n_jk * nb region bins of tpcf_count's region_out) TPCF_PARTIAL_WORDS int64:
 * the slot's 128-bit two's-complement fixed-point sum as four 32-bit limbs,
 * least significant first, then the numbers of NaN, +inf and -inf pair
 * weights met.  Adding the partial arrays of all shards word by word (for
 * example an all-reduce SUM over int64) cannot overflow for up to 2^31
 * shards, and tpcf_shard_combine turns the sum into exactly the doubles one
 * tpcf_count would return, weighted sums included.  *scale_exp receives the
 * fixed-point exponent, the same on every shard.
 *   partial[(1 + n_jk) * nb * TPCF_PARTIAL_WORDS] */
#define TPCF_PARTIAL_WORDS 7
int tpcf_count_shard(tpcf_ctx *ctx, const tpcf_catalog *a, const tpcf_catalog *b, const tpcf_binning *bin,
                     const tpcf_weight_spec *spec, int precision, int32_t shard, int32_t n_shards, int64_t *partial,
                     int32_t *scale_exp, tpcf_stats *stats);
/* Summed partials to full_out[nb] and region_out[n_jk * nb] (may be NULL), as
 * tpcf_count returns them.  Host-only. */
int tpcf_shard_combine(const tpcf_binning *bin, const int64_t *partial, int32_t scale_exp, double *full_out,
                       double *region_out);

/* The reference's counting entry points with its output convention: the
 * histograms after invert_jk_hists() and, for auto counts, multiply_hists(2.0)
 * — what auto_pair_count_{monopole,sigma_pi,s_mu}(const GalaxyBoxes*, JKHists*)
 * and cross_pair_count_*(a, b, hist) leave in hist (src/correlators.cpp:11-430). */
int tpcf_auto_pair_count(tpcf_ctx *ctx, const tpcf_catalog *cat, const tpcf_binning *bin, int precision,
                         double *full_hist, double *sub_hist, tpcf_stats *stats);
int tpcf_cross_pair_count(tpcf_ctx *ctx, const tpcf_catalog *a, const tpcf_catalog *b, const tpcf_binning *bin,
                          int precision, double *full_hist, double *sub_hist, tpcf_stats *stats);

/* JKHists::normalise (src/hist.cpp:290-367) over the kept points of the
 * catalogue(s), in place on arrays of nb and n_jk * nb doubles. */
int tpcf_normalise_auto(const tpcf_catalog *cat, int32_t nb, double *full_hist, double *sub_hist);
int tpcf_normalise_cross(const tpcf_catalog *a, const tpcf_catalog *b, int32_t nb, double *full_hist,
                         double *sub_hist);

/* ls_estimator (src/io.cpp:643-651). */
double tpcf_ls_estimator(double dd, double dr, double rr);

/* Diagnostics (no counterpart in the reference): kernels launched by this
 * context so far, and the device's FP32 FMA rate (TFLOP/s) and returning
 * 32-bit shared-memory atomic rate (per second) measured with short probe
 * kernels — the two pipes that bound the pair-count kernels. */
uint64_t tpcf_kernel_launches(const tpcf_ctx *ctx);
int tpcf_measure_peaks(tpcf_ctx *ctx, double *fp32_tflops, double *smem_atomics_per_s);

/* Self-test of the device give-up path (no counterpart in the reference): one
 * kernel runs the pair kernels' bounded wait on a shared-memory barrier.  With
 * arrive != 0 the barrier is completed first and the call returns TPCF_OK;
 * with arrive == 0 nothing ever completes it, the wait gives up after `limit`
 * tries and the call returns TPCF_E_DEVICE_TIMEOUT, leaving the context
 * usable.  limit == 0: TPCF_E_INVALID_ARG. */
int tpcf_wait_selftest(tpcf_ctx *ctx, int32_t arrive, uint32_t limit);

/* Fault injection for the allocation error paths (no counterpart in the
 * reference; process-wide, for tests): after `after` more successful device
 * allocations of catalogues, cell grids and per-call scratch, every further
 * one fails as out of memory until this is called with after < 0.  The
 * failing call returns an error status and releases what it had allocated. */
int tpcf_debug_fail_allocations(int64_t after);

/* Give-up path of the count kernels themselves (no counterpart in the
 * reference; process-wide, for tests): with on != 0, counts planned after
 * this call take the branch of a tile wait that gave up (the device-timeout
 * flag is raised, the CTAs stop taking work items and the call returns
 * TPCF_E_DEVICE_TIMEOUT with its results discarded), after each wait has
 * still seen its copy complete, so no copy is left in flight.  on == 0
 * restores normal counts. */
int tpcf_debug_force_tile_timeout(int32_t on);

/* Device bounds checks (no counterpart in the reference).  The checked build
 * of this library (TPCF_DEVICE_CHECKS=1 python two_pcf_b200/build.py, written
 * to two_pcf_b200/lib/checked/) tests, in every count kernel, every index a
 * work item and its segments carry (segment range, A chunk, cells, regions,
 * B runs, job), every bin index and every queue fill against its bounds
 * before use; the first failure stops the count, which returns
 * TPCF_E_DEVICE_CHECK naming the check, the value and the limit, and no
 * access leaves its buffer.  tpcf_device_checks() is 1 in that build, 0 in
 * the release build.  tpcf_debug_corrupt_work_list(1), checked build only
 * (process-wide, for tests): the next count's first segment gets a region
 * past the histogram rows after planning, on the host; the release build
 * returns TPCF_E_UNSUPPORTED. */
int tpcf_device_checks(void);
int tpcf_debug_corrupt_work_list(int what);

/* ---------------------------------------------------------------------------
 * The command-line flow around the counts (src/main.cpp:11-84): parameter
 * file, redshift -> comoving distance, catalogue reader, result writers.
 * Host-only; these calls need no device.  A failed call leaves its message in
 * tpcf_host_last_error() of the calling thread.
 * ------------------------------------------------------------------------- */
typedef struct tpcf_params tpcf_params;
typedef struct tpcf_cosmology tpcf_cosmology;
typedef struct tpcf_host_catalog tpcf_host_catalog;

const char *tpcf_host_last_error(void);

/* Params(file) (src/io.cpp:16-237): a line that does not start with '#' and
 * holds '=' is cut at its first '#' and split at its first '=', and every
 * space is removed from key and value.  Numbers convert as std::stoi /
 * std::stod do; a value they would reject fails the call
 * (TPCF_E_INVALID_ARG).  Keys the file does not set read as 0 / "" (the
 * reference leaves them uninitialised); n_jk_regions <= 1 reads as 1. */
int tpcf_params_load(const char *path, tpcf_params **out);
int tpcf_params_parse(const char *text, tpcf_params **out);
int tpcf_params_destroy(tpcf_params *params);
/* Fields by their parameter-file key.  get_int also reads the boolean keys
 * (0/1).  get_string copies at most cap bytes including the terminator and
 * returns the string's length, or a negative status. */
int tpcf_params_get_double(const tpcf_params *params, const char *key, double *out);
int tpcf_params_get_int(const tpcf_params *params, const char *key, int32_t *out);
int tpcf_params_get_string(const tpcf_params *params, const char *key, char *out, int32_t cap);

/* Cosmology(omega_m, h, z_min, z_max, z_save_step, z_oversample) and
 * comov_dist (src/cosmology.cpp:11-100, src/dataset.cpp:110-126); the
 * reference's program uses z_save_step = 1e-4, z_oversample = 100
 * (src/main.cpp:40).  Outside [z_min, z_max'] comov_dist returns z_min or
 * z_max' (the table's last z), as the reference does. */
int tpcf_cosmology_create(double omega_m, double h, double z_min, double z_max, double z_save_step,
                          int32_t z_oversample, tpcf_cosmology **out);
int tpcf_cosmology_destroy(tpcf_cosmology *cosmo);
int tpcf_cosmology_comov_dist(const tpcf_cosmology *cosmo, const double *z, int64_t n, double *out);

/* Galaxy::set (src/galaxy.cpp:8-27) over n points: x_norm from ra/dec in
 * degrees, xyz = d_comov * x_norm, or 0 where d_comov < 0. */
int tpcf_galaxy_set(int64_t n, const double *ra_deg, const double *dec_deg, const double *d_comov, double *xyz,
                    double *x_norm);
/* The cartesian reader's transform (src/io.cpp:393-399): d_comov = |x|,
 * x_norm = x / d_comov. */
int tpcf_cartesian_set(int64_t n, const double *xyz, double *d_comov, double *x_norm);

typedef enum { TPCF_CARTESIAN = 0, TPCF_EQUATORIAL = 1 } tpcf_coord_system;

/* read_data_ascii (src/io.cpp:240-414), parsed in parallel.  Data lines are
 * the non-empty lines not starting with '#'; fields are split at ',' if the
 * line holds one, else at tabs if it holds one, else at spaces, empty pieces
 * skipped.  Columns: x y z or ra dec z, then the weight if use_weights, then
 * the jackknife region if n_jk_regions > 1.  A missing or unparsable field
 * fails the call with its line number (the reference aborts or loops
 * forever there).  cosmo is required for TPCF_EQUATORIAL. */
int tpcf_read_ascii(const char *path, int coord_system, int use_weights, int32_t n_jk_regions,
                    const tpcf_cosmology *cosmo, tpcf_host_catalog **out);
int64_t tpcf_host_catalog_size(const tpcf_host_catalog *cat);
/* Borrowed views, valid until the catalogue is destroyed: xyz[3n], x_norm[3n],
 * d_comov[n], weight[n], jk_region[n] — the arguments tpcf_catalog_create takes. */
int tpcf_host_catalog_arrays(const tpcf_host_catalog *cat, const double **xyz, const double **x_norm,
                             const double **d_comov, const float **weight, const int32_t **jk_region);
int tpcf_host_catalog_destroy(tpcf_host_catalog *cat);

/* generate_sub_filename (src/io.cpp:628-641): the region number goes before
 * the last '.' of the name.  Returns the length, or a negative status. */
int tpcf_sub_filename(const char *filename, int64_t sub, char *out, int32_t cap);

/* output_xi_1D / output_xi_2D with output type "ascii" (src/io.cpp:724-756,
 * :832-853): writes filename with the full histograms and, when the region
 * arrays are given, one file per jackknife region named by
 * tpcf_sub_filename.  Columns as the reference writes them (bin index(es),
 * centre(s), width(s), Landy-Szalay xi, DD, DR, RR; numbers as std::ostream
 * prints a double by default).  dd/dr/rr are normalised histograms of
 * tpcf_binning_total_bins(bin) values, the *_sub arrays n_jk * nb values.
 * TPCF_ANGULAR binnings are refused (the reference writes those as HDF5). */
int tpcf_write_xi_ascii(const char *filename, const tpcf_binning *bin, const double *dd, const double *dr,
                        const double *rr, const double *dd_sub, const double *dr_sub, const double *rr_sub);

/* The reference's program (src/main.cpp:11-84, plain build) on a parameter
 * file: read both catalogues, then for each of plot_monopole, plot_sigma_pi,
 * plot_s_mu count DD, DR and RR on the device, normalise and write the ASCII
 * outputs (auto_correlate_*, src/correlators.cpp:127-459).  HDF5 catalogues
 * and outputs are refused with TPCF_E_UNSUPPORTED (this build has no HDF5
 * library).  log: 0 quiet, 1 one line per step on stderr. */
int tpcf_run_param_file(const char *path, int device, int precision, int log);

/* tpcf_run_param_file with a run report (no counterpart in the reference,
 * which prints only its ASCII outputs).  summary_path non-NULL: a JSON
 * summary is written there, also when the run fails (its status and error):
 * catalogue sizes read and kept, wall time, and per mode and count the
 * in-range pairs, candidates, guard re-evaluations, kernel time and pairs/s.
 * check_fp64 != 0 (with precision TPCF_FP32_GUARD): every count runs again on
 * the plain FP64 path and the summary gives, per output (DD, DR, RR raw and
 * normalised; xi; full histogram and every region's slice), the largest
 * relative and absolute difference from the FP64 result and whether they
 * agree bit for bit.  The ASCII outputs are those of the run's own
 * precision. */
int tpcf_run_param_file_report(const char *path, int device, int precision, int log, int check_fp64,
                               const char *summary_path);

/* The inverse-p program after its catalogues are read (src/main.cpp:51-60):
 * the angular stage of calc_angular_upweight
 * (src/correlators_invpweight.cpp:985-1033) — angular DD (every point,
 * input-weight products), DD with inverse-p weights, DR, DR with inverse-p
 * weights on Hist(0, 1 - cos(theta_max), theta_n_bins, theta_log_base) —
 * then, for each plot_* flag, auto_correlate_*_invpweights
 * (:210-237, :445-474, :682-711): DD with inverse-p weights and the
 * DD / DD-inverse-p up-weight, DR with the DR / DR-inverse-p up-weight, plain
 * RR, normalised and written as ASCII where the parameters name the files.
 * The angular histograms stay in memory instead of going through HDF5 files,
 * so the calculate_angular_* flags and file names are not used: all four are
 * always computed.  data and randoms carry bitmasks (and input weights, e.g.
 * from tpcf_iip_weights); dither = 1 is the _USE_DITHER_WEIGHTS build (both
 * need dither masks).  angular_out: NULL or 4 * (1 + n_jk) * theta_n_bins
 * doubles receiving DD, DD-inverse-p, DR, DR-inverse-p, each as its full
 * histogram then its n_jk region rows, in the reference's convention. */
int tpcf_run_invp(tpcf_ctx *ctx, const tpcf_params *params, const tpcf_catalog *data, const tpcf_catalog *randoms,
                  int precision, int dither, double *angular_out, int log);

#ifdef __cplusplus
}
#endif

#endif /* TWO_PCF_B200_H */
