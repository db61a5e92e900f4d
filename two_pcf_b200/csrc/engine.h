// Internal engine objects behind the C ABI (include/two_pcf_b200.h).
#pragma once
#include <cuda_runtime.h>

#include <atomic>
#include <cstdint>
#include <cstdlib>
#include <map>
#include <memory>
#include <string>
#include <vector>

#include "axis.h"
#include "tpcf_common.h"

namespace tpcf {

// Device buffer with RAII ownership.
template <typename T>
struct DevBuf {
    T *p = nullptr;
    size_t n = 0;
    DevBuf() = default;
    DevBuf(const DevBuf &) = delete;
    DevBuf &operator=(const DevBuf &) = delete;
    ~DevBuf() { release(); }
    void release() {
        if (p) cudaFree(p);
        p = nullptr;
        n = 0;
    }
    cudaError_t alloc(size_t count) {
        release();
        if (count == 0) count = 1;
        cudaError_t e = cudaMalloc((void **)&p, count * sizeof(T));
        if (e == cudaSuccess) n = count;
        else p = nullptr;
        return e;
    }
};

// Injected allocation failure (tpcf_debug_fail_allocations): while the
// budget is >= 0, each device allocation of the engine's pool-backed buffers
// takes one from it and fails once it is exhausted.  -1: off.
inline std::atomic<long long> &alloc_fail_budget() {
    static std::atomic<long long> budget{-1};
    return budget;
}
// Checked build only (tpcf_debug_corrupt_work_list): 1 = give the next
// count's first segment a region past the histogram rows, on the host after
// planning, so the device bounds checks have something to find.
inline std::atomic<int> &debug_corrupt_work_list() {
    static std::atomic<int> v{0};
    return v;
}

// Forced tile timeout of the count kernels (tpcf_debug_force_tile_timeout):
// every wait for a staged tile still waits for its copy, then raises the
// device-timeout flag as a wait that gave up does.
inline std::atomic<int> &debug_force_tile_timeout() {
    static std::atomic<int> v{0};
    return v;
}

inline bool alloc_injected_failure() {
    auto &b = alloc_fail_budget();
    long long v = b.load(std::memory_order_relaxed);
    while (v >= 0) {
        if (v == 0) return true;
        if (b.compare_exchange_weak(v, v - 1, std::memory_order_relaxed)) return false;
    }
    return false;
}

// TPCF_TRACE set (and not "0"): count_many and the grid builds print their
// timelines on stderr.
inline bool trace_enabled() {
    const char *e = std::getenv("TPCF_TRACE");
    return e && e[0] && e[0] != '0';
}

struct Error {
    int status;
    std::string msg;
};

// A context's stream-ordered memory pool, shared by the context and by every
// catalogue and grid array allocated from it: the pool is destroyed when the
// last of them goes, so an array that outlives its context (a catalogue
// destroyed after tpcf_destroy) frees into a pool that still exists.
struct PoolRef {
    cudaMemPool_t pool = nullptr;
    PoolRef() = default;
    PoolRef(const PoolRef &) = delete;
    PoolRef &operator=(const PoolRef &) = delete;
    ~PoolRef() {
        if (pool) cudaMemPoolDestroy(pool);  // returns at once; reclaimed once pending frees complete
    }
};

struct Ctx {
    int device = 0;
    int num_sms = 148;
    size_t smem_optin = 0;
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    std::string last_error;
    int refinement = 0;  // 0 = automatic
    int kernel_cfg = -1;  // -1 = automatic (the autotuner's choice when it runs, else 0)
    int swap = -1;        // order of plain-weight cross counts (CountRequest::swap); -1 = automatic
    // autotuning of counts: the (refinement, kernel configuration) chosen per
    // count class by timed probes, kept for the context's lifetime
    bool autotune = false;
    struct Tuned {
        int m = 0, cfg = 0, swap = 0;
        // in-range pairs/s of each candidate probed, index (m - 1) + 3 cfg + 6 swap; 0 = not probed
        std::vector<double> rate;
    };
    std::map<std::string, Tuned> tuned;
    unsigned long long launches = 0;  // kernels launched by this context
    cudaMemPool_t pool = nullptr;     // stream-ordered pool for the scratch of each call (owned by pool_ref)
    std::shared_ptr<PoolRef> pool_ref;
    // pinned staging of the counts in flight in count_many (two slots, grown
    // on demand, freed with the context)
    unsigned char *pinned[2] = {nullptr, nullptr};
    size_t pinned_cap[2] = {0, 0};
    // lives exactly as long as the context: catalogues hold a weak reference
    // and release on the context's stream only while it lives
    std::shared_ptr<int> alive = std::make_shared<int>(0);
};

// Device scratch of one call, from the context's stream-ordered memory pool:
// allocation and release are queued on the context's stream and released
// memory stays in the pool for the next call, so a count neither
// synchronises the device nor hands memory back to the driver (a cudaFree of
// a large work list has been measured taking most of a second).  Only for
// buffers that do not outlive the call.
template <typename T>
struct ScratchBuf {
    T *p = nullptr;
    size_t n = 0;
    cudaStream_t s = nullptr;
    ScratchBuf() = default;
    ScratchBuf(const ScratchBuf &) = delete;
    ScratchBuf &operator=(const ScratchBuf &) = delete;
    ~ScratchBuf() { release(); }
    void release() {
        if (p) cudaFreeAsync(p, s);
        p = nullptr;
        n = 0;
    }
    cudaError_t alloc(const Ctx &ctx, size_t count) {
        release();
        if (count == 0) count = 1;
        s = ctx.stream;
        if (alloc_injected_failure()) return cudaErrorMemoryAllocation;
        cudaError_t e = ctx.pool ? cudaMallocFromPoolAsync((void **)&p, count * sizeof(T), ctx.pool, s)
                                 : cudaMallocAsync((void **)&p, count * sizeof(T), s);
        if (e == cudaSuccess) n = count;
        else p = nullptr;
        return e;
    }
};


// Device memory from a context's pool that outlives the call that made it
// (the cell grids cached on a catalogue): allocated in the context's stream
// order, and released on the legacy stream when its owner goes.  Every
// engine call returns with its stream drained, so nothing still reads the
// memory by then; the release neither synchronises the device nor unmaps
// memory, and it stays valid after the context (and its pool) is destroyed.
template <typename T>
struct PoolBuf {
    T *p = nullptr;
    size_t n = 0;
    int device = 0;
    std::shared_ptr<PoolRef> pool_ref;  // the pool p came from, kept until p is freed
    PoolBuf() = default;
    PoolBuf(const PoolBuf &) = delete;
    PoolBuf &operator=(const PoolBuf &) = delete;
    ~PoolBuf() { release(); }
    void release() { release_on(0); }
    // Release in the order of stream `s` (the legacy stream when 0): a
    // context that is still alive releases on its own stream, so that its
    // next allocations reuse the memory in stream order.
    void release_on(cudaStream_t s) {
        if (p) {
            int cur = device;
            cudaGetDevice(&cur);
            if (cur != device) cudaSetDevice(device);
            cudaFreeAsync(p, s);
            if (cur != device) cudaSetDevice(cur);
        }
        p = nullptr;
        n = 0;
        pool_ref.reset();  // after the free is queued: the last reference destroys the pool
    }
    cudaError_t alloc(const Ctx &ctx, size_t count) {
        release();
        if (count == 0) count = 1;
        device = ctx.device;
        if (alloc_injected_failure()) return cudaErrorMemoryAllocation;
        cudaError_t e = ctx.pool ? cudaMallocFromPoolAsync((void **)&p, count * sizeof(T), ctx.pool, ctx.stream)
                                 : cudaMallocAsync((void **)&p, count * sizeof(T), ctx.stream);
        if (e == cudaSuccess) {
            n = count;
            pool_ref = ctx.pool_ref;
        } else {
            p = nullptr;
        }
        return e;
    }
};

// The points of one catalogue sorted into cubic cells of side `side` on the
// lattice x = k * side (k integer), with points inside a cell ordered by
// jackknife region.  Replaces GalaxyBoxes (src/boxes.cpp:10-163).
struct Grid {
    double side = 0;
    bool angular = false;  // cells over the unit vectors instead of the positions
    bool input_w = false;  // the weight slot holds input_weight instead of weight
    int kmin[3] = {0, 0, 0};
    int dim[3] = {1, 1, 1};
    bool morton = false;  // dense cell id = Morton code of the local cell coords
    int ncell = 0;        // size of the dense cell table
    int n = 0;            // points in the grid
    bool subset_kept = true;
    PoolBuf<float4> pos;   // (x - kx*side, y - ky*side, z - kz*side, weight), float
    PoolBuf<float4> aux;   // (x_norm / 2 as float, weight): the pi step reads both with one load
    PoolBuf<int> idx;      // original catalogue index
    PoolBuf<double4> xyz_s;   // sorted double coordinates (exact path, FP64 path)
    PoolBuf<double4> unit_s;  // sorted double unit vectors
    PoolBuf<int> cell_start;  // ncell + 1
    PoolBuf<int3> cell_coord; // local coords of each dense cell id (for offsets)
    PoolBuf<int> region_start;  // ncell + 1, CSR of distinct jk regions per cell
    PoolBuf<int> regions;       // region of each run
    PoolBuf<int> run_start;     // first point of each run
    std::vector<int> h_cell_start;  // host copies for the work-list build
    std::vector<int> h_region_start;
    std::vector<int> h_regions;
    std::vector<int> h_run_start;
    bool has_fp64 = false;
    void release_on(cudaStream_t s) {
        pos.release_on(s);
        aux.release_on(s);
        idx.release_on(s);
        xyz_s.release_on(s);
        unit_s.release_on(s);
        cell_start.release_on(s);
        cell_coord.release_on(s);
        region_start.release_on(s);
        regions.release_on(s);
        run_start.release_on(s);
    }
};

struct Catalog {
    Ctx *ctx = nullptr;
    std::weak_ptr<int> ctx_alive;  // expired once the context is destroyed
    int64_t n_all = 0;
    int n_kept = 0;
    int n_mask = 0;
    int n_jk = 1;
    bool unit_weights = true;  // every weight == 1.0f
    float w_min = 1, w_max = 1, iw_min = 1, iw_max = 1;
    double lo_kept[3], hi_kept[3], lo_all[3], hi_all[3];
    double ulo_kept[3], uhi_kept[3], ulo_all[3], uhi_all[3];  // bounding boxes of the unit vectors
    double norm_dev = 0;          // max | x_norm . x_norm - 1 |
    bool iw_unit = true;          // every input weight == 1.0f
    PoolBuf<double> xyz, unit;
    PoolBuf<float> w, iw;
    PoolBuf<int> jk;
    PoolBuf<long long> masks;
    PoolBuf<long long> dmasks;    // dither masks (Galaxy::dither_mask), n_mask per point, or empty
    PoolBuf<int> kept;            // indices kept by the d_comov partition
    std::vector<float> h_w;       // host copies used by normalisation
    std::vector<int> h_jk;
    std::vector<int> h_kept;
    std::map<std::string, std::unique_ptr<Grid>> grids;  // cached by geometry
    // Drop the cached grids: on the context's stream while the context lives
    // (its next grid builds reuse the memory in stream order), else on the
    // legacy stream.
    void release_grids() {
        const cudaStream_t s = ctx_alive.expired() ? (cudaStream_t)0 : ctx->stream;
        for (auto &kv : grids) kv.second->release_on(s);
        grids.clear();
    }
};

struct Binning {
    int mode = 0;
    int n_jk = 1;
    AxisParams ax1, ax2;
    int nb1 = 0, nb2 = 1, nb = 0;
    float min_r_sq = 0, max_r_sq = 0;  // float range test of the reference
    double rmax_bound = 0;             // every in-range pair is closer than this on each axis
    std::vector<float> t1, t2;         // threshold tables (see axis.h)
    // Line of sight for pi: false = x_norm1 + x_norm2 (_ANGULAR_PI_DEFN,
    // src/correlators.cpp:166-170), true = x1 + x2 (:172-182).
    bool los_midpoint = false;
    ValueSpace vs1 = ValueSpace::Direct, vs2 = ValueSpace::Direct;
};

struct Stats {
    unsigned long long candidates = 0, in_range = 0, guard = 0, overflow = 0, items = 0;
    double ms_kernel = 0, ms_total = 0;
};


// grid.cu
// Which grid of a catalogue: cell side, the point subset (the d_comov
// partition or every point), the coordinates it is built on and the weight
// it carries.
struct GridSpec {
    double side = 0;
    bool subset_kept = true;
    bool angular = false;
    bool input_w = false;
};
int build_grid(Ctx *ctx, Catalog *cat, const GridSpec &spec, bool want_fp64, Grid **out, Error *err);
// The grid build_grid would return when it is already cached, else nullptr;
// never allocates.
Grid *find_grid(Catalog *cat, const GridSpec &spec, bool want_fp64);
// After the catalogue's weight array changed on the device: rewrite the
// weight slot of every cached grid that carries it.
int reweight_grids(Ctx *ctx, Catalog *cat, Error *err);

// pair_count.cu
// Angular up-weight of the 3-D inverse-p counts: JKHists::interp
// (src/hist.cpp:369-391) of the ratio of two angular histograms.
struct UpTable {
    AxisParams ax;
    std::vector<double> bins;    // n + 1: the ratio per bin, plus a spare copy of the last
    std::vector<double> centre;  // n + 1: Axis::bin_centre(b), host libm exp
    std::vector<float> thr;      // n + 1: interpolation-interval thresholds (see make_up_table)
    double abs_max = 0;          // largest finite |ratio|
};
// Builds the table from numerator and denominator histograms
// (JKHists::divide_by_hist, src/hist.cpp:224-231).
UpTable make_up_table(const AxisParams &ax, const double *num, const double *den);
// The interpolation exactly as the kernels evaluate it.
double up_eval(const UpTable &t, double v);

// Pair weighting of a count (reference build and function in brackets).
enum Weighting {
    WEIGHTS_PLAIN = 0,    // w1 * w2 [3-D]; input_weight products [angular DD / DR]
    WEIGHTS_INVP_DD = 1,  // inverse-p popcount weights [*_invpweights DD]
    WEIGHTS_INVP_DR = 2,  // angular DR up-weight [3-D DR]; w1 * w2 [angular DR inverse-p]
};

struct CountRequest {
    const Catalog *a = nullptr;
    const Catalog *b = nullptr;  // nullptr: auto count of a
    const Binning *bin = nullptr;
    bool exact_fp64 = false;     // plain FP64 path for every candidate
    int weighting = WEIGHTS_PLAIN;
    const UpTable *up = nullptr; // 3-D inverse-p counts
    int n_runs = 0;              // Params::n_bitwise_runs
    bool dither = false;         // _USE_DITHER_WEIGHTS: popc(dither masks) in place of n_runs
    // one shard of a count split across processes: the work items k with
    // k % n_shards == shard; with raw_out set, the fixed-point sums are
    // returned as limbs (kPartialWords per slot) instead of doubles
    int shard = 0, n_shards = 1;
    long long *raw_out = nullptr;
    int *scale_exp_out = nullptr;
    int refinement = 0;
    // kernel configuration of the plain-weight FP32+guard kernels (0 or 1;
    // -1: the context's setting, else the autotuner's choice, else 0)
    int kernel_cfg = -1;
    // order of a plain-weight cross count: 1 counts b's points against a's
    // (b in registers, a streamed in tiles), 0 a's against b's; -1 the
    // context's setting, else the autotuner's choice, else 0.  The histograms
    // are the same either way: each pair adds once to the full histogram and
    // to the rows of both its regions, the pair weight is a commutative float
    // product, and swapping the points negates the separation exactly.
    int swap = -1;
    // adjoint of a plain-weight 3-D count: with adj_G = dL/d(raw full
    // histogram) set, the count writes per-point dL/dw into grad_a (n_all of
    // a) and grad_b (n_all of b; unused for auto counts) instead of histograms
    const double *adj_G = nullptr;
    double *grad_a = nullptr, *grad_b = nullptr;
};
int run_count(Ctx *ctx, const CountRequest &req, double *full_out, double *region_out, Stats *st, Error *err);
// Several counts, results identical to run_count on each in order: every
// grid is built first, then each count's host planning (work list, tables)
// runs while the previous count's kernel is on the device.
struct CountOut {
    double *full = nullptr, *region = nullptr;
    Stats *st = nullptr;
};
int run_count_many(Ctx *ctx, const std::vector<CountRequest> &reqs, const std::vector<CountOut> &outs, Error *err);
// run_count without device allocation: every scratch buffer is carved from
// one static device array of kStaticScratchBytes, and the catalogues' cell
// grids must already be cached.
constexpr size_t kStaticScratchBytes = size_t(32) << 20;
// Words per histogram slot of a shard's partial sums: the 128-bit
// two's-complement fixed-point sum as four 32-bit limbs (least significant
// first), then the numbers of NaN, +inf and -inf pair weights met.
constexpr int kPartialWords = 7;
// Partial sums (already added over shards) to the doubles of a count.
void partial_to_double(const long long *partial, size_t slots, int scale_exp, double *out);
int run_count_static(Ctx *ctx, const CountRequest &req, double *full_out, double *region_out, Stats *st,
                     Error *err);

// pair_count.cu: batched counts — the work items of many catalogue pairs in
// one persistent launch, planned once and replayed as a CUDA graph.
struct Batch;
struct BatchJobSpec {
    const Catalog *a = nullptr;
    const Catalog *b = nullptr;  // nullptr: auto count of a
};
// refinement: cells per maximum separation (1..3), 0 automatic, -1 timed
// choice among 1, 2 and 3.
int batch_create(Ctx *ctx, const std::vector<BatchJobSpec> &jobs, const Binning *bin, bool exact_fp64, int refinement,
                 Batch **out, Error *err);
// full_out[n_jobs * nb], region_out[n_jobs * n_jk * nb] (may be null): raw
// sums as tpcf_count returns them, job after job.
int batch_run(Batch *b, double *full_out, double *region_out, Stats *st, Error *err);
int batch_refinement(const Batch *b);
int batch_order(const Batch *b);
int batch_jobs(const Batch *b);
void batch_destroy(Batch *b);

// worklist.cpp: the work items of one (A, B) count with cells of `side`
// (m cells per maximum separation rb), longest first.
void build_work_items(const Grid &ga, const Grid &gb, bool is_auto, int m, double side, double rb,
                      std::vector<WorkItem> &items, std::vector<Segment> &segs);

// diag.cu
int measure_peaks(Ctx *ctx, double *fp32_tflops, double *smem_atomics_per_s, Error *err);
int wait_selftest(Ctx *ctx, int arrive, unsigned limit, int *device_status, Error *err);

}  // namespace tpcf
