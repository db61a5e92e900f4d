// C ABI of the engine (include/two_pcf_b200.h).  Validation happens here,
// on the host, before anything is launched.
#include "../../include/two_pcf_b200.h"

#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <memory>
#include <new>
#include <string>
#include <vector>

#include "capi_types.h"

namespace {

int fail(tpcf_ctx *ctx, int status, const std::string &msg) {
    if (ctx) ctx->c.last_error = msg;
    return status;
}

int cuda_fail(tpcf_ctx *ctx, cudaError_t e, const char *where) {
    int st = (e == cudaErrorMemoryAllocation) ? TPCF_E_OOM : TPCF_E_CUDA;
    return fail(ctx, st, std::string(where) + ": " + cudaGetErrorString(e));
}

// The d_comov < 0 partition of GalaxyBoxes (src/boxes.cpp:15-26), applied to
// an index permutation; returns the number of points the reference keeps.
// The loop condition makes it stop before every point has been examined when
// points are dropped, so some good points at the end are dropped too.
int partition_kept(const double *dcom, int n, std::vector<int> &perm) {
    perm.resize(n);
    for (int i = 0; i < n; ++i) perm[i] = i;
    if (!dcom) return n;
    int n_gals = 0;
    for (int ii = 0; ii < n - ii + n_gals; ++ii) {
        if (dcom[perm[n_gals]] < 0.0) {
            std::swap(perm[n_gals], perm[n - 1 - ii + n_gals]);
        } else {
            ++n_gals;
        }
    }
    return n_gals;
}

}  // namespace

extern "C" {

int tpcf_abi_version(void) { return TPCF_ABI_VERSION; }

const char *tpcf_status_string(int status) {
    switch (status) {
    case TPCF_OK: return "ok";
    case TPCF_E_INVALID_ARG: return "invalid argument";
    case TPCF_E_OOM: return "out of device memory";
    case TPCF_E_CUDA: return "CUDA error";
    case TPCF_E_DEVICE_TIMEOUT: return "device wait timed out";
    case TPCF_E_OVERFLOW: return "histogram overflow";
    case TPCF_E_UNSUPPORTED: return "unsupported configuration";
    case TPCF_E_DEVICE_CHECK: return "device bounds check failed";
    default: return "unknown status";
    }
}

int tpcf_create(int device, tpcf_ctx **out) {
    if (!out) return TPCF_E_INVALID_ARG;
    *out = nullptr;
    int ndev = 0;
    cudaError_t e = cudaGetDeviceCount(&ndev);
    if (e != cudaSuccess || ndev == 0) return TPCF_E_CUDA;
    if (device < 0 || device >= ndev) return TPCF_E_INVALID_ARG;
    tpcf_ctx *ctx = new (std::nothrow) tpcf_ctx();
    if (!ctx) return TPCF_E_OOM;
    ctx->c.device = device;
    e = cudaSetDevice(device);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&ctx->c.num_sms, cudaDevAttrMultiProcessorCount, device);
    int optin = 0;
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, device);
    ctx->c.smem_optin = (size_t)optin;
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&ctx->c.stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) {
        // The context's own pool for per-call scratch: memory a call releases
        // stays reserved for the next call (the pool is destroyed with the
        // context), so counts never wait on the driver to map or unmap memory.
        cudaMemPoolProps props;
        std::memset(&props, 0, sizeof(props));
        props.allocType = cudaMemAllocationTypePinned;
        props.location.type = cudaMemLocationTypeDevice;
        props.location.id = device;
        e = cudaMemPoolCreate(&ctx->c.pool, &props);
        if (e == cudaSuccess) {
            ctx->c.pool_ref = std::make_shared<tpcf::PoolRef>();
            ctx->c.pool_ref->pool = ctx->c.pool;
            uint64_t keep = UINT64_MAX;
            e = cudaMemPoolSetAttribute(ctx->c.pool, cudaMemPoolAttrReleaseThreshold, &keep);
        }
    }
    if (e != cudaSuccess) {
        if (ctx->c.pool && !ctx->c.pool_ref) cudaMemPoolDestroy(ctx->c.pool);
        ctx->c.pool_ref.reset();
        if (ctx->c.stream) cudaStreamDestroy(ctx->c.stream);
        delete ctx;
        return TPCF_E_CUDA;
    }
    ctx->c.own_stream = true;
    *out = ctx;
    return TPCF_OK;
}

int tpcf_destroy(tpcf_ctx *ctx) {
    if (!ctx) return TPCF_E_INVALID_ARG;
    cudaSetDevice(ctx->c.device);
    if (ctx->c.stream) cudaStreamSynchronize(ctx->c.stream);
    for (unsigned char *p : ctx->c.pinned)
        if (p) cudaFreeHost(p);
    // the pool goes with the last array allocated from it (PoolRef): arrays of
    // catalogues that outlive the context still free into it
    ctx->c.pool_ref.reset();
    if (ctx->c.own_stream && ctx->c.stream) cudaStreamDestroy(ctx->c.stream);
    delete ctx;
    return TPCF_OK;
}

const char *tpcf_last_error(const tpcf_ctx *ctx) { return ctx ? ctx->c.last_error.c_str() : "no context"; }

int tpcf_set_stream(tpcf_ctx *ctx, void *stream) {
    if (!ctx) return TPCF_E_INVALID_ARG;
    if (ctx->c.own_stream && ctx->c.stream) cudaStreamDestroy(ctx->c.stream);
    ctx->c.own_stream = false;
    ctx->c.stream = (cudaStream_t)stream;
    if (!stream) {
        cudaError_t e = cudaStreamCreateWithFlags(&ctx->c.stream, cudaStreamNonBlocking);
        if (e != cudaSuccess) return cuda_fail(ctx, e, "stream");
        ctx->c.own_stream = true;
    }
    return TPCF_OK;
}

int tpcf_set_refinement(tpcf_ctx *ctx, int m) {
    if (!ctx || m < 0 || m > 3) return TPCF_E_INVALID_ARG;
    ctx->c.refinement = m;
    return TPCF_OK;
}

int tpcf_set_autotune(tpcf_ctx *ctx, int on) {
    if (!ctx) return TPCF_E_INVALID_ARG;
    ctx->c.autotune = on != 0;
    return TPCF_OK;
}

int tpcf_set_cross_order(tpcf_ctx *ctx, int order) {
    if (!ctx || order < -1 || order > 1) return TPCF_E_INVALID_ARG;
    ctx->c.swap = order;
    return TPCF_OK;
}

int tpcf_set_kernel_config(tpcf_ctx *ctx, int cfg) {
    if (!ctx || cfg < -1 || cfg > 1) return TPCF_E_INVALID_ARG;
    ctx->c.kernel_cfg = cfg;
    return TPCF_OK;
}

int64_t tpcf_autotune_describe(const tpcf_ctx *ctx, char *buf, int64_t len) {
    if (!ctx || len < 0 || (len > 0 && !buf)) return -TPCF_E_INVALID_ARG;
    std::string j = "[";
    bool first = true;
    for (const auto &kv : ctx->c.tuned) {
        j += first ? "" : ", ";
        first = false;
        j += "{\"class\": \"" + kv.first + "\", \"refinement\": " + std::to_string(kv.second.m) +
             ", \"kernel_config\": " + std::to_string(kv.second.cfg) +
             ", \"order\": " + std::to_string(kv.second.swap) + ", \"pairs_per_s\": [";
        for (size_t k = 0; k < kv.second.rate.size(); ++k) {
            char b[32];
            std::snprintf(b, sizeof b, "%s%.6g", k ? ", " : "", kv.second.rate[k]);
            j += b;
        }
        j += "]}";
    }
    j += "]";
    if (len > 0) {
        const size_t n = std::min<size_t>(j.size(), (size_t)len - 1);
        std::memcpy(buf, j.data(), n);
        buf[n] = '\0';
    }
    return (int64_t)j.size();
}

int tpcf_synchronize(tpcf_ctx *ctx) {
    if (!ctx) return TPCF_E_INVALID_ARG;
    cudaError_t e = cudaStreamSynchronize(ctx->c.stream);
    return e == cudaSuccess ? TPCF_OK : cuda_fail(ctx, e, "synchronize");
}

int tpcf_catalog_create(tpcf_ctx *ctx, int64_t n, const double *xyz, const double *x_norm, const double *d_comov,
                        const float *weight, const float *input_weight, const int32_t *jk_region,
                        int32_t n_jk_regions, const int64_t *bitmask, int32_t n_mask_ints, tpcf_catalog **out) {
    if (!ctx || !out) return TPCF_E_INVALID_ARG;
    *out = nullptr;
    if (n < 0 || n > 0x7fffffff - 1) return fail(ctx, TPCF_E_INVALID_ARG, "catalogue size out of range");
    if (n > 0 && !xyz) return fail(ctx, TPCF_E_INVALID_ARG, "xyz is NULL");
    if (n_jk_regions < 1 || n_jk_regions > tpcf::kMaxRegions)
        return fail(ctx, TPCF_E_INVALID_ARG, "n_jk_regions must be in [1, 4096]");
    if (n_mask_ints < 0 || n_mask_ints > tpcf::kMaxMaskInts || (n_mask_ints > 0 && !bitmask && n > 0))
        return fail(ctx, TPCF_E_INVALID_ARG, "bad bitmask arguments");
    cudaError_t e = cudaSetDevice(ctx->c.device);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "set device");

    const int N = (int)n;
    std::unique_ptr<tpcf_catalog> cat(new (std::nothrow) tpcf_catalog());
    if (!cat) return TPCF_E_OOM;
    tpcf::Catalog &c = cat->c;
    c.ctx = &ctx->c;
    c.ctx_alive = ctx->c.alive;
    c.n_all = n;
    c.n_jk = n_jk_regions;
    c.n_mask = bitmask ? n_mask_ints : 0;

    // Host checks and bounds, in parallel over the points.  Each check
    // reports its lowest failing index, in the order the checks are listed.
    std::vector<double> unit;
    int64_t bad = N;
#pragma omp parallel for schedule(static) reduction(min : bad)
    for (int i = 0; i < N; ++i)
        for (int m = 0; m < 3; ++m)
            if (!std::isfinite(xyz[3 * (size_t)i + m])) bad = std::min<int64_t>(bad, i);
    if (bad < N) return fail(ctx, TPCF_E_INVALID_ARG, "non-finite coordinate at index " + std::to_string(bad));
    if (!x_norm) {
        // src/io.cpp:393-399: d_comov = sqrt(x.x), x_norm = x / d_comov.
        unit.resize(3 * (size_t)N);
#pragma omp parallel for schedule(static)
        for (int i = 0; i < N; ++i) {
            const double *p = xyz + 3 * (size_t)i;
            double d = std::sqrt(p[0] * p[0] + p[1] * p[1] + p[2] * p[2]);
            for (int m = 0; m < 3; ++m) unit[3 * (size_t)i + m] = p[m] / d;
        }
        x_norm = unit.data();
    }
    c.h_jk.assign(N, 0);
    if (jk_region) {
#pragma omp parallel for schedule(static) reduction(min : bad)
        for (int i = 0; i < N; ++i) {
            if (jk_region[i] < 0 || jk_region[i] >= n_jk_regions) bad = std::min<int64_t>(bad, i);
            c.h_jk[i] = jk_region[i];
        }
        if (bad < N) return fail(ctx, TPCF_E_INVALID_ARG, "jk_region out of range at index " + std::to_string(bad));
    }
    c.h_w.assign(N, 1.0f);
    c.unit_weights = true;
    c.w_max = 0;
    c.w_min = 0;
    if (weight) {
        bool unitw = true;
#pragma omp parallel for schedule(static) reduction(min : bad) reduction(&& : unitw)
        for (int i = 0; i < N; ++i) {
            if (!std::isfinite(weight[i])) bad = std::min<int64_t>(bad, i);
            c.h_w[i] = weight[i];
            unitw = unitw && weight[i] == 1.0f;
        }
        if (bad < N) return fail(ctx, TPCF_E_INVALID_ARG, "non-finite weight");
        c.unit_weights = unitw;
    }
    c.n_kept = partition_kept(d_comov, N, c.h_kept);
    std::vector<char> is_kept(N, 0);
    for (int k = 0; k < c.n_kept; ++k) is_kept[c.h_kept[k]] = 1;
    // Bounding boxes of the positions and of the unit vectors (all points and
    // the kept ones), the largest |weight| and the largest deviation of
    // |x_norm|^2 from 1 (a term of the angular error bound).
    double lo_all[3] = {1e300, 1e300, 1e300}, hi_all[3] = {-1e300, -1e300, -1e300};
    double lo_kept[3] = {1e300, 1e300, 1e300}, hi_kept[3] = {-1e300, -1e300, -1e300};
    double ulo_all[3] = {1e300, 1e300, 1e300}, uhi_all[3] = {-1e300, -1e300, -1e300};
    double ulo_kept[3] = {1e300, 1e300, 1e300}, uhi_kept[3] = {-1e300, -1e300, -1e300};
    float w_max = 0;
    double norm_dev = 0;
#pragma omp parallel for schedule(static) reduction(min : bad, lo_all[:3], lo_kept[:3], ulo_all[:3], ulo_kept[:3]) \
    reduction(max : hi_all[:3], hi_kept[:3], uhi_all[:3], uhi_kept[:3], w_max, norm_dev)
    for (int i = 0; i < N; ++i) {
        w_max = std::max(w_max, std::fabs(c.h_w[i]));
        const double *u = x_norm + 3 * (size_t)i;
        for (int m = 0; m < 3; ++m) {
            const double v = xyz[3 * (size_t)i + m];
            lo_all[m] = std::min(lo_all[m], v);
            hi_all[m] = std::max(hi_all[m], v);
            if (!std::isfinite(u[m])) bad = std::min<int64_t>(bad, i);
            ulo_all[m] = std::min(ulo_all[m], u[m]);
            uhi_all[m] = std::max(uhi_all[m], u[m]);
            if (is_kept[i]) {
                lo_kept[m] = std::min(lo_kept[m], v);
                hi_kept[m] = std::max(hi_kept[m], v);
                ulo_kept[m] = std::min(ulo_kept[m], u[m]);
                uhi_kept[m] = std::max(uhi_kept[m], u[m]);
            }
        }
        norm_dev = std::max(norm_dev, std::fabs(u[0] * u[0] + u[1] * u[1] + u[2] * u[2] - 1.0));
    }
    if (bad < N) return fail(ctx, TPCF_E_INVALID_ARG, "non-finite x_norm at index " + std::to_string(bad));
    for (int m = 0; m < 3; ++m) {
        c.lo_all[m] = lo_all[m];
        c.hi_all[m] = hi_all[m];
        c.lo_kept[m] = lo_kept[m];
        c.hi_kept[m] = hi_kept[m];
        c.ulo_all[m] = ulo_all[m];
        c.uhi_all[m] = uhi_all[m];
        c.ulo_kept[m] = ulo_kept[m];
        c.uhi_kept[m] = uhi_kept[m];
    }
    c.w_max = w_max;
    c.norm_dev = norm_dev;
    c.iw_max = c.w_max;
    c.iw_unit = c.unit_weights;
    if (input_weight) {
        float iw_max = 0;
        bool iw_unit = true;
#pragma omp parallel for schedule(static) reduction(min : bad) reduction(max : iw_max) reduction(&& : iw_unit)
        for (int i = 0; i < N; ++i) {
            if (!std::isfinite(input_weight[i])) bad = std::min<int64_t>(bad, i);
            iw_max = std::max(iw_max, std::fabs(input_weight[i]));
            iw_unit = iw_unit && input_weight[i] == 1.0f;
        }
        if (bad < N) return fail(ctx, TPCF_E_INVALID_ARG, "non-finite input_weight");
        c.iw_max = iw_max;
        c.iw_unit = iw_unit;
    }

    cudaStream_t st = ctx->c.stream;
#define CAT_TRY(expr)                                            \
    do {                                                         \
        cudaError_t _e = (expr);                                 \
        if (_e != cudaSuccess) return cuda_fail(ctx, _e, "catalogue upload"); \
    } while (0)
    CAT_TRY(c.xyz.alloc(ctx->c, 3 * (size_t)N));
    CAT_TRY(c.unit.alloc(ctx->c, 3 * (size_t)N));
    CAT_TRY(c.w.alloc(ctx->c, N));
    CAT_TRY(c.jk.alloc(ctx->c, N));
    CAT_TRY(c.kept.alloc(ctx->c, c.n_kept));
    if (N > 0) {
        CAT_TRY(cudaMemcpyAsync(c.xyz.p, xyz, sizeof(double) * 3 * N, cudaMemcpyHostToDevice, st));
        CAT_TRY(cudaMemcpyAsync(c.unit.p, x_norm, sizeof(double) * 3 * N, cudaMemcpyHostToDevice, st));
        CAT_TRY(cudaMemcpyAsync(c.w.p, c.h_w.data(), sizeof(float) * N, cudaMemcpyHostToDevice, st));
        CAT_TRY(cudaMemcpyAsync(c.jk.p, c.h_jk.data(), sizeof(int) * N, cudaMemcpyHostToDevice, st));
    }
    if (c.n_kept > 0)
        CAT_TRY(cudaMemcpyAsync(c.kept.p, c.h_kept.data(), sizeof(int) * c.n_kept, cudaMemcpyHostToDevice, st));
    if (input_weight) {
        CAT_TRY(c.iw.alloc(ctx->c, N));
        if (N > 0) CAT_TRY(cudaMemcpyAsync(c.iw.p, input_weight, sizeof(float) * N, cudaMemcpyHostToDevice, st));
    }
    if (c.n_mask > 0) {
        CAT_TRY(c.masks.alloc(ctx->c, (size_t)N * c.n_mask));
        if (N > 0)
            CAT_TRY(cudaMemcpyAsync(c.masks.p, bitmask, sizeof(long long) * (size_t)N * c.n_mask,
                                    cudaMemcpyHostToDevice, st));
    }
    CAT_TRY(cudaStreamSynchronize(st));
#undef CAT_TRY
    *out = cat.release();
    return TPCF_OK;
}

int tpcf_catalog_destroy(tpcf_catalog *cat) {
    if (!cat) return TPCF_E_INVALID_ARG;
    delete cat;  // arrays released on the legacy stream (valid whatever became of the context's stream)
    return TPCF_OK;
}

int64_t tpcf_catalog_n_used(const tpcf_catalog *cat) { return cat ? cat->c.n_kept : -1; }

int tpcf_catalog_release_cache(tpcf_catalog *cat) {
    if (!cat) return TPCF_E_INVALID_ARG;
    cat->c.release_grids();
    return TPCF_OK;
}

int tpcf_binning_create(tpcf_ctx *ctx, int mode, const tpcf_axis_spec *ax1, const tpcf_axis_spec *ax2,
                        int32_t n_jk_regions, tpcf_binning **out) {
    if (!out || !ax1) return TPCF_E_INVALID_ARG;
    *out = nullptr;
    if (mode < TPCF_MONOPOLE || mode > TPCF_ANGULAR) return fail(ctx, TPCF_E_INVALID_ARG, "bad mode");
    if ((mode == TPCF_SIGMA_PI || mode == TPCF_S_MU) && !ax2) return fail(ctx, TPCF_E_INVALID_ARG, "ax2 required");
    if (n_jk_regions < 1 || n_jk_regions > tpcf::kMaxRegions) return fail(ctx, TPCF_E_INVALID_ARG, "bad n_jk");
    auto bad_axis = [](const tpcf_axis_spec *a) {
        return a->n_bins < 1 || a->n_bins > tpcf::kMaxBins1D || !std::isfinite(a->min) || !std::isfinite(a->max) ||
               !(a->max > a->min);
    };
    if (bad_axis(ax1)) return fail(ctx, TPCF_E_INVALID_ARG, "bad axis 1");
    std::unique_ptr<tpcf_binning> b(new (std::nothrow) tpcf_binning());
    if (!b) return TPCF_E_OOM;
    tpcf::Binning &B = b->b;
    B.mode = mode;
    B.n_jk = n_jk_regions;
    B.ax1 = tpcf::make_axis(ax1->min, ax1->max, ax1->n_bins, ax1->log_base);
    B.nb1 = ax1->n_bins;
    B.nb2 = 1;
    using tpcf::ValueSpace;
    if (mode == TPCF_MONOPOLE) {
        // src/correlators.cpp:13-14
        B.max_r_sq = B.ax1.max * B.ax1.max;
        B.min_r_sq = B.ax1.min * B.ax1.min;
        B.vs1 = ValueSpace::Sqrt;
    } else if (mode == TPCF_SIGMA_PI) {
        if (bad_axis(ax2)) return fail(ctx, TPCF_E_INVALID_ARG, "bad axis 2");
        B.ax2 = tpcf::make_axis(ax2->min, ax2->max, ax2->n_bins, ax2->log_base);
        B.nb2 = ax2->n_bins;
        // src/correlators.cpp:192-195
        B.max_r_sq = B.ax1.max * B.ax1.max + B.ax2.max * B.ax2.max;
        B.min_r_sq = B.ax1.min * B.ax1.min;
        if (B.ax1.min > B.ax2.min) B.min_r_sq = B.ax2.min * B.ax2.min;
        B.vs1 = ValueSpace::Sqrt;  // sigma = sqrtf(s^2 - pi^2)
        B.vs2 = ValueSpace::Direct;
    } else if (mode == TPCF_S_MU) {
        if (ax2->n_bins < 1 || ax2->n_bins > tpcf::kMaxBins1D) return fail(ctx, TPCF_E_INVALID_ARG, "bad mu bins");
        // src/correlators.cpp:436-437: Hist2D(s..., 0.0, 1.0, mu_n_bins, 0)
        B.ax2 = tpcf::make_axis(0.0, 1.0, ax2->n_bins, 0.0);
        B.nb2 = ax2->n_bins;
        B.max_r_sq = B.ax1.max * B.ax1.max;
        B.min_r_sq = B.ax1.min * B.ax1.min;
        B.vs1 = ValueSpace::Sqrt;
        B.vs2 = ValueSpace::Direct;
    } else {
        B.vs1 = ValueSpace::Direct;  // binned on (float)(1 - cos theta)
        B.max_r_sq = B.ax1.max;
        B.min_r_sq = 0;
    }
    B.nb = B.nb1 * B.nb2;
    if (B.nb > tpcf::kMaxBinsTotal) return fail(ctx, TPCF_E_UNSUPPORTED, "more than 8192 bins");
    // Threshold domains: the values a binned pair can present.  s^2 and
    // sigma^2 = s^2 - pi^2 lie in [0, max_r_sq); |pi| <= s (up to rounding);
    // mu = |pi| / s lies in [0, ~1]; 1 - cos(theta) in [-2, 2] (tiny negative
    // values occur and land in bin 0 in the reference).
    const float sq = B.max_r_sq;
    const float rmax_f = (float)(std::sqrt((double)sq) * 1.01 + 1.0);
    if (mode == TPCF_ANGULAR) {
        B.t1 = tpcf::build_thresholds(B.ax1, B.vs1, -2.0f, 2.0f);
    } else {
        B.t1 = tpcf::build_thresholds(B.ax1, B.vs1, 0.0f, sq);
    }
    if (mode == TPCF_SIGMA_PI) B.t2 = tpcf::build_thresholds(B.ax2, B.vs2, 0.0f, rmax_f);
    else if (mode == TPCF_S_MU) B.t2 = tpcf::build_thresholds(B.ax2, B.vs2, 0.0f, 2.0f);
    else B.t2.assign(1, 0.0f);
    // Every in-range pair has |x1_m - x2_m| below sqrt(max_r_sq) up to a few
    // float roundings.
    B.rmax_bound = std::sqrt((double)B.max_r_sq) * (1.0 + 1e-6) + 1e-30;
    *out = b.release();
    return TPCF_OK;
}

int tpcf_binning_destroy(tpcf_binning *bin) {
    if (!bin) return TPCF_E_INVALID_ARG;
    delete bin;
    return TPCF_OK;
}

int tpcf_binning_total_bins(const tpcf_binning *bin) { return bin ? bin->b.nb : -TPCF_E_INVALID_ARG; }

int tpcf_binning_thresholds(const tpcf_binning *bin, int axis, float *out, int cap) {
    if (!bin || (axis != 1 && axis != 2) || (cap > 0 && !out)) return -TPCF_E_INVALID_ARG;
    const std::vector<float> &t = axis == 1 ? bin->b.t1 : bin->b.t2;
    for (int k = 0; k < (int)t.size() && k < cap; ++k) out[k] = t[k];
    return (int)t.size();
}

}  // extern "C"

namespace {

// Validates a weight spec and builds the request's up-weight table.
int prepare_weights(tpcf_ctx *ctx, const tpcf_catalog *a, const tpcf_catalog *b, const tpcf_binning *bin,
                    const tpcf_weight_spec *spec, tpcf::CountRequest &req, tpcf::UpTable &up) {
    req.weighting = spec ? spec->weighting : TPCF_WEIGHTS_PLAIN;
    if (req.weighting < TPCF_WEIGHTS_PLAIN || req.weighting > TPCF_WEIGHTS_INVP_DD_DITHER)
        return fail(ctx, TPCF_E_INVALID_ARG, "bad weighting");
    if (req.weighting == TPCF_WEIGHTS_PLAIN) return TPCF_OK;
    if (req.weighting == TPCF_WEIGHTS_INVP_DD_DITHER) {
        req.weighting = TPCF_WEIGHTS_INVP_DD;
        req.dither = true;
    }
    req.n_runs = spec->n_bitwise_runs;
    if (req.weighting == TPCF_WEIGHTS_INVP_DD) {
        const tpcf::Catalog &ca = a->c, &cb = b ? b->c : a->c;
        if (ca.n_mask < 1 || ca.n_mask != cb.n_mask)
            return fail(ctx, TPCF_E_INVALID_ARG, "inverse-p DD weights need bitmasks of one width on both catalogues");
        if (req.dither && (!ca.dmasks.p || !cb.dmasks.p))
            return fail(ctx, TPCF_E_INVALID_ARG, "dither weights need dither masks on both catalogues");
    }
    if (bin->b.mode != TPCF_ANGULAR) {
        const tpcf_axis_spec &t = spec->theta_axis;
        if (!spec->up_numerator || !spec->up_denominator || t.n_bins < 1 || t.n_bins > tpcf::kMaxBins1D ||
            !std::isfinite(t.min) || !std::isfinite(t.max) || !(t.max > t.min))
            return fail(ctx, TPCF_E_INVALID_ARG, "3-D inverse-p counts need the angular up-weight histograms and axis");
        up = tpcf::make_up_table(tpcf::make_axis(t.min, t.max, t.n_bins, t.log_base), spec->up_numerator,
                                 spec->up_denominator);
        req.up = &up;
    }
    return TPCF_OK;
}

struct ShardArgs {
    int shard = 0, n_shards = 1;
    int64_t *partial = nullptr;
    int32_t *scale_exp = nullptr;
};

int count_impl(tpcf_ctx *ctx, const tpcf_catalog *a, const tpcf_catalog *b, const tpcf_binning *bin,
               const tpcf_weight_spec *spec, int precision, double *full_out, double *region_out, tpcf_stats *stats,
               bool noalloc, const ShardArgs &sh = ShardArgs()) {
    if (!ctx || !a || !bin || (!full_out && !sh.partial)) return TPCF_E_INVALID_ARG;
    if (precision != TPCF_FP32_GUARD && precision != TPCF_FP64) return fail(ctx, TPCF_E_INVALID_ARG, "bad precision");
    if (a->c.n_jk != bin->b.n_jk || (b && b->c.n_jk != bin->b.n_jk))
        return fail(ctx, TPCF_E_INVALID_ARG, "catalogue and binning disagree on n_jk_regions");
    tpcf::CountRequest req;
    tpcf::UpTable up;
    int rc = prepare_weights(ctx, a, b, bin, spec, req, up);
    if (rc) return rc;
    cudaError_t e = cudaSetDevice(ctx->c.device);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "set device");
    auto t0 = std::chrono::steady_clock::now();
    req.a = &a->c;
    req.b = b ? &b->c : nullptr;
    req.bin = &bin->b;
    req.exact_fp64 = precision == TPCF_FP64 || bin->b.los_midpoint;
    const int nb = bin->b.nb;
    // Points a count uses: every point for plain angular counts, the d_comov
    // partition otherwise.
    const bool all_points = bin->b.mode == TPCF_ANGULAR && req.weighting == TPCF_WEIGHTS_PLAIN;
    auto used = [&](const tpcf_catalog *c) { return all_points ? c->c.n_all : (int64_t)c->c.n_kept; };
    if (used(a) == 0 || (b && used(b) == 0)) {
        if (full_out) std::memset(full_out, 0, sizeof(double) * nb);
        if (region_out) std::memset(region_out, 0, sizeof(double) * nb * bin->b.n_jk);
        if (sh.partial)
            std::memset(sh.partial, 0, sizeof(int64_t) * (size_t)(1 + bin->b.n_jk) * nb * tpcf::kPartialWords);
        if (sh.scale_exp) *sh.scale_exp = 0;
        if (stats) std::memset(stats, 0, sizeof(*stats));
        return TPCF_OK;
    }
    req.shard = sh.shard;
    req.n_shards = sh.n_shards;
    req.raw_out = reinterpret_cast<long long *>(sh.partial);
    req.scale_exp_out = reinterpret_cast<int *>(sh.scale_exp);
    tpcf::Stats st;
    tpcf::Error err{0, ""};
    rc = noalloc ? tpcf::run_count_static(&ctx->c, req, full_out, region_out, &st, &err)
                 : tpcf::run_count(&ctx->c, req, full_out, region_out, &st, &err);
    if (rc) return fail(ctx, rc, err.msg);
    if (stats) {
        stats->candidates = st.candidates;
        stats->in_range = st.in_range;
        stats->guard_evals = st.guard;
        stats->overflow_updates = st.overflow;
        stats->work_items = st.items;
        stats->ms_kernel = st.ms_kernel;
        stats->ms_total = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    }
    return TPCF_OK;
}

int reference_form(tpcf_ctx *ctx, const tpcf_catalog *a, const tpcf_catalog *b, const tpcf_binning *bin,
                   const tpcf_weight_spec *spec, int precision, double *full, double *sub, tpcf_stats *stats) {
    if (!sub) return fail(ctx, TPCF_E_INVALID_ARG, "sub_hist is NULL");
    int rc = count_impl(ctx, a, b, bin, spec, precision, full, sub, stats, false);
    if (rc) return rc;
    const int nb = bin->b.nb, nj = bin->b.n_jk;
    // invert_jk_hists (src/hist.cpp:270-277, :464-471)
    for (int r = 0; r < nj; ++r)
        for (int k = 0; k < nb; ++k) sub[(size_t)r * nb + k] = full[k] - sub[(size_t)r * nb + k];
    if (!b) {
        // multiply_hists(2.0) (src/hist.cpp:279-288, :473-482)
        for (int k = 0; k < nb; ++k) full[k] *= 2.0;
        for (size_t k = 0; k < (size_t)nb * nj; ++k) sub[k] *= 2.0;
    }
    return TPCF_OK;
}

}  // namespace

extern "C" {

int tpcf_count(tpcf_ctx *ctx, const tpcf_catalog *a, const tpcf_catalog *b, const tpcf_binning *bin,
               int precision, double *full_out, double *region_out, tpcf_stats *stats) {
    return count_impl(ctx, a, b, bin, nullptr, precision, full_out, region_out, stats, false);
}

int tpcf_count_many(tpcf_ctx *ctx, const tpcf_count_job *jobs, int32_t n_jobs) {
    if (!ctx || n_jobs < 0 || (n_jobs > 0 && !jobs)) return TPCF_E_INVALID_ARG;
    std::vector<tpcf::CountRequest> reqs;
    std::vector<tpcf::CountOut> outs;
    std::vector<tpcf::UpTable> ups(n_jobs);
    std::vector<tpcf::Stats> sts(n_jobs);
    std::vector<int> run;  // jobs that reach the device
    for (int k = 0; k < n_jobs; ++k) {
        const tpcf_count_job &J = jobs[k];
        if (!J.a || !J.bin || !J.full_out) return fail(ctx, TPCF_E_INVALID_ARG, "job " + std::to_string(k) + ": NULL argument");
        if (J.reference_form && !J.region_out)
            return fail(ctx, TPCF_E_INVALID_ARG, "job " + std::to_string(k) + ": reference_form needs region_out");
        if (J.precision != TPCF_FP32_GUARD && J.precision != TPCF_FP64)
            return fail(ctx, TPCF_E_INVALID_ARG, "job " + std::to_string(k) + ": bad precision");
        if (J.a->c.n_jk != J.bin->b.n_jk || (J.b && J.b->c.n_jk != J.bin->b.n_jk))
            return fail(ctx, TPCF_E_INVALID_ARG, "job " + std::to_string(k) + ": catalogue and binning disagree on n_jk_regions");
        tpcf::CountRequest req;
        int rc = prepare_weights(ctx, J.a, J.b, J.bin, J.spec, req, ups[k]);
        if (rc) return rc;
        req.a = &J.a->c;
        req.b = J.b ? &J.b->c : nullptr;
        req.bin = &J.bin->b;
        req.exact_fp64 = J.precision == TPCF_FP64 || J.bin->b.los_midpoint;
        const int nb = J.bin->b.nb;
        const bool all_points = J.bin->b.mode == TPCF_ANGULAR && req.weighting == TPCF_WEIGHTS_PLAIN;
        auto used = [&](const tpcf_catalog *c) { return all_points ? c->c.n_all : (int64_t)c->c.n_kept; };
        if (used(J.a) == 0 || (J.b && used(J.b) == 0)) {
            std::memset(J.full_out, 0, sizeof(double) * nb);
            if (J.region_out) std::memset(J.region_out, 0, sizeof(double) * nb * J.bin->b.n_jk);
            if (J.stats) std::memset(J.stats, 0, sizeof(*J.stats));
            continue;
        }
        if (req.up) req.up = &ups[k];
        reqs.push_back(req);
        tpcf::CountOut o;
        o.full = J.full_out;
        o.region = J.region_out;
        o.st = &sts[k];
        outs.push_back(o);
        run.push_back(k);
    }
    cudaError_t e = cudaSetDevice(ctx->c.device);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "set device");
    auto t0 = std::chrono::steady_clock::now();
    tpcf::Error err{0, ""};
    if (!reqs.empty() && tpcf::run_count_many(&ctx->c, reqs, outs, &err)) return fail(ctx, err.status, err.msg);
    const double ms_total = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    for (int k : run) {
        const tpcf_count_job &J = jobs[k];
        if (J.stats) {
            const tpcf::Stats &st = sts[k];
            J.stats->candidates = st.candidates;
            J.stats->in_range = st.in_range;
            J.stats->guard_evals = st.guard;
            J.stats->overflow_updates = st.overflow;
            J.stats->work_items = st.items;
            J.stats->ms_kernel = st.ms_kernel;
            J.stats->ms_total = ms_total;
        }
        if (J.reference_form) {
            const int nb = J.bin->b.nb, nj = J.bin->b.n_jk;
            for (int r = 0; r < nj; ++r)
                for (int q = 0; q < nb; ++q) J.region_out[(size_t)r * nb + q] = J.full_out[q] - J.region_out[(size_t)r * nb + q];
            if (!J.b) {
                for (int q = 0; q < nb; ++q) J.full_out[q] *= 2.0;
                for (size_t q = 0; q < (size_t)nb * nj; ++q) J.region_out[q] *= 2.0;
            }
        }
    }
    return TPCF_OK;
}

int tpcf_count_shard(tpcf_ctx *ctx, const tpcf_catalog *a, const tpcf_catalog *b, const tpcf_binning *bin,
                     const tpcf_weight_spec *spec, int precision, int32_t shard, int32_t n_shards, int64_t *partial,
                     int32_t *scale_exp, tpcf_stats *stats) {
    if (!ctx || !partial || !scale_exp) return TPCF_E_INVALID_ARG;
    if (n_shards < 1 || shard < 0 || shard >= n_shards) return fail(ctx, TPCF_E_INVALID_ARG, "bad shard index");
    ShardArgs sh;
    sh.shard = shard;
    sh.n_shards = n_shards;
    sh.partial = partial;
    sh.scale_exp = scale_exp;
    return count_impl(ctx, a, b, bin, spec, precision, nullptr, nullptr, stats, false, sh);
}

int tpcf_shard_combine(const tpcf_binning *bin, const int64_t *partial, int32_t scale_exp, double *full_out,
                       double *region_out) {
    if (!bin || !partial || !full_out || scale_exp < -100 || scale_exp > 100) return TPCF_E_INVALID_ARG;
    const int nb = bin->b.nb, nj = bin->b.n_jk;
    std::vector<double> v((size_t)(1 + nj) * nb);
    tpcf::partial_to_double(reinterpret_cast<const long long *>(partial), v.size(), scale_exp, v.data());
    std::copy(v.begin(), v.begin() + nb, full_out);
    if (region_out) std::copy(v.begin() + nb, v.end(), region_out);
    return TPCF_OK;
}

int tpcf_count_noalloc(tpcf_ctx *ctx, const tpcf_catalog *a, const tpcf_catalog *b, const tpcf_binning *bin,
                       int precision, double *full_out, double *region_out, tpcf_stats *stats) {
    return count_impl(ctx, a, b, bin, nullptr, precision, full_out, region_out, stats, true);
}

int tpcf_count_weighted(tpcf_ctx *ctx, const tpcf_catalog *a, const tpcf_catalog *b, const tpcf_binning *bin,
                        const tpcf_weight_spec *spec, int precision, double *full_out, double *region_out,
                        tpcf_stats *stats) {
    return count_impl(ctx, a, b, bin, spec, precision, full_out, region_out, stats, false);
}

int tpcf_pair_count_weighted(tpcf_ctx *ctx, const tpcf_catalog *a, const tpcf_catalog *b, const tpcf_binning *bin,
                             const tpcf_weight_spec *spec, int precision, double *full_hist, double *sub_hist,
                             tpcf_stats *stats) {
    return reference_form(ctx, a, b, bin, spec, precision, full_hist, sub_hist, stats);
}

int tpcf_count_backward(tpcf_ctx *ctx, const tpcf_catalog *a, const tpcf_catalog *b, const tpcf_binning *bin,
                        int precision, const double *dL_dfull, double *dL_dw_a, double *dL_dw_b, tpcf_stats *stats) {
    if (!ctx || !a || !bin || !dL_dfull || !dL_dw_a || (b && !dL_dw_b)) return TPCF_E_INVALID_ARG;
    if (precision != TPCF_FP32_GUARD && precision != TPCF_FP64) return fail(ctx, TPCF_E_INVALID_ARG, "bad precision");
    if (bin->b.mode == TPCF_ANGULAR) return fail(ctx, TPCF_E_UNSUPPORTED, "the adjoint is defined for 3-D counts");
    if (a->c.n_jk != bin->b.n_jk || (b && b->c.n_jk != bin->b.n_jk))
        return fail(ctx, TPCF_E_INVALID_ARG, "catalogue and binning disagree on n_jk_regions");
    cudaError_t e = cudaSetDevice(ctx->c.device);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "set device");
    auto t0 = std::chrono::steady_clock::now();
    std::memset(dL_dw_a, 0, sizeof(double) * a->c.n_all);
    if (b) std::memset(dL_dw_b, 0, sizeof(double) * b->c.n_all);
    if (stats) std::memset(stats, 0, sizeof(*stats));
    if (a->c.n_kept == 0 || (b && b->c.n_kept == 0)) return TPCF_OK;
    tpcf::CountRequest req;
    req.a = &a->c;
    req.b = b ? &b->c : nullptr;
    req.bin = &bin->b;
    req.exact_fp64 = precision == TPCF_FP64 || bin->b.los_midpoint;
    req.adj_G = dL_dfull;
    req.grad_a = dL_dw_a;
    req.grad_b = dL_dw_b;
    tpcf::Stats st;
    tpcf::Error err{0, ""};
    int rc = tpcf::run_count(&ctx->c, req, nullptr, nullptr, &st, &err);
    if (rc) return fail(ctx, rc, err.msg);
    if (stats) {
        stats->candidates = st.candidates;
        stats->in_range = st.in_range;
        stats->guard_evals = st.guard;
        stats->work_items = st.items;
        stats->ms_kernel = st.ms_kernel;
        stats->ms_total = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    }
    return TPCF_OK;
}

int tpcf_catalog_set_weights(tpcf_catalog *cat, const float *weight) {
    if (!cat || !weight) return TPCF_E_INVALID_ARG;
    tpcf::Catalog &c = cat->c;
    tpcf::Ctx *ctx = c.ctx;
    const int N = (int)c.n_all;
    bool unit = true;
    float wmax = 0;
    for (int i = 0; i < N; ++i) {
        if (!std::isfinite(weight[i])) return TPCF_E_INVALID_ARG;
        if (weight[i] != 1.0f) unit = false;
        wmax = std::max(wmax, std::fabs(weight[i]));
    }
    cudaError_t e = cudaSetDevice(ctx->device);
    if (e == cudaSuccess && N > 0)
        e = cudaMemcpyAsync(c.w.p, weight, sizeof(float) * N, cudaMemcpyHostToDevice, ctx->stream);
    if (e != cudaSuccess) {
        ctx->last_error = std::string("set weights: ") + cudaGetErrorString(e);
        return TPCF_E_CUDA;
    }
    std::copy(weight, weight + N, c.h_w.begin());
    c.unit_weights = unit;
    c.w_max = wmax;
    if (!c.iw.p) {  // input weights default to the weights
        c.iw_max = wmax;
        c.iw_unit = unit;
    }
    tpcf::Error err{0, ""};
    if (tpcf::reweight_grids(ctx, &c, &err)) {
        ctx->last_error = err.msg;
        return err.status;
    }
    e = cudaStreamSynchronize(ctx->stream);
    if (e != cudaSuccess) {
        ctx->last_error = std::string("set weights: ") + cudaGetErrorString(e);
        return TPCF_E_CUDA;
    }
    return TPCF_OK;
}

int tpcf_catalog_set_dither_masks(tpcf_catalog *cat, const int64_t *dither_mask) {
    if (!cat || !dither_mask) return TPCF_E_INVALID_ARG;
    tpcf::Catalog &c = cat->c;
    tpcf::Ctx *ctx = c.ctx;
    if (c.n_mask < 1) {
        ctx->last_error = "dither masks need the catalogue's bitmasks (their width sets the dither masks' width)";
        return TPCF_E_INVALID_ARG;
    }
    const size_t words = (size_t)c.n_all * c.n_mask;
    cudaError_t e = cudaSetDevice(ctx->device);
    if (e == cudaSuccess) e = c.dmasks.alloc(*ctx, words);
    if (e == cudaSuccess && words > 0)
        e = cudaMemcpyAsync(c.dmasks.p, dither_mask, sizeof(long long) * words, cudaMemcpyHostToDevice, ctx->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    if (e != cudaSuccess) {
        c.dmasks.release();
        ctx->last_error = std::string("dither masks: ") + cudaGetErrorString(e);
        return e == cudaErrorMemoryAllocation ? TPCF_E_OOM : TPCF_E_CUDA;
    }
    return TPCF_OK;
}

int tpcf_binning_set_line_of_sight(tpcf_binning *bin, int line_of_sight) {
    if (!bin || (line_of_sight != TPCF_LOS_ANGULAR && line_of_sight != TPCF_LOS_MIDPOINT)) return TPCF_E_INVALID_ARG;
    bin->b.los_midpoint = line_of_sight == TPCF_LOS_MIDPOINT;
    return TPCF_OK;
}

int tpcf_iip_weights(int64_t n, int32_t n_mask_ints, const int64_t *bitmask, const int64_t *dither_mask,
                     int32_t n_bitwise_runs, float *weight, float *input_weight) {
    if (n < 0 || n_mask_ints < 1 || (n > 0 && (!bitmask || !weight || !input_weight))) return TPCF_E_INVALID_ARG;
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; ++i) {
        int total = 0, dtotal = 0;
        for (int k = 0; k < n_mask_ints; ++k) {
            total += __builtin_popcountll((unsigned long long)bitmask[(size_t)i * n_mask_ints + k]);
            if (dither_mask) dtotal += __builtin_popcountll((unsigned long long)dither_mask[(size_t)i * n_mask_ints + k]);
        }
        input_weight[i] = weight[i];
        if (total == 0) total = 1;
        if (total != n_bitwise_runs) {
            const double ratio = dither_mask ? (double)dtotal / (double)total : (double)n_bitwise_runs / (double)total;
            weight[i] = (float)((double)weight[i] * ratio);
        }
    }
    return TPCF_OK;
}

int tpcf_batch_create(tpcf_ctx *ctx, const tpcf_catalog *const *mocks, int32_t n_mocks, const tpcf_catalog *randoms,
                      const tpcf_binning *bin, int precision, int32_t what, int32_t refinement, tpcf_batch **out) {
    if (!ctx || !mocks || n_mocks < 1 || !bin || !out) return TPCF_E_INVALID_ARG;
    *out = nullptr;
    if (precision != TPCF_FP32_GUARD && precision != TPCF_FP64) return fail(ctx, TPCF_E_INVALID_ARG, "bad precision");
    if ((what & ~(TPCF_BATCH_DD | TPCF_BATCH_DR)) || !what) return fail(ctx, TPCF_E_INVALID_ARG, "bad batch outputs");
    if ((what & TPCF_BATCH_DR) && !randoms) return fail(ctx, TPCF_E_INVALID_ARG, "DR needs the random catalogue");
    if (refinement < -1 || refinement > 3) return fail(ctx, TPCF_E_INVALID_ARG, "bad refinement");
    if (bin->b.mode == TPCF_ANGULAR) return fail(ctx, TPCF_E_UNSUPPORTED, "batched counts are 3-D counts");
    std::vector<tpcf::BatchJobSpec> jobs;
    for (int i = 0; i < n_mocks; ++i) {
        if (!mocks[i] || mocks[i]->c.n_jk != bin->b.n_jk)
            return fail(ctx, TPCF_E_INVALID_ARG, "mock " + std::to_string(i) + " missing or with other n_jk_regions");
        if (what & TPCF_BATCH_DD) jobs.push_back({&mocks[i]->c, nullptr});
        if (what & TPCF_BATCH_DR) jobs.push_back({&mocks[i]->c, &randoms->c});
    }
    if (randoms && randoms->c.n_jk != bin->b.n_jk)
        return fail(ctx, TPCF_E_INVALID_ARG, "randoms and binning disagree on n_jk_regions");
    cudaError_t e = cudaSetDevice(ctx->c.device);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "set device");
    std::unique_ptr<tpcf_batch> B(new (std::nothrow) tpcf_batch());
    if (!B) return TPCF_E_OOM;
    B->ctx = ctx;
    tpcf::Error err{0, ""};
    if (tpcf::batch_create(&ctx->c, jobs, &bin->b, precision == TPCF_FP64 || bin->b.los_midpoint, refinement, &B->b, &err))
        return fail(ctx, err.status, err.msg);
    *out = B.release();
    return TPCF_OK;
}

int tpcf_batch_run(tpcf_batch *batch, double *full_out, double *region_out, tpcf_stats *stats) {
    if (!batch || !full_out) return TPCF_E_INVALID_ARG;
    tpcf_ctx *ctx = batch->ctx;
    cudaError_t e = cudaSetDevice(ctx->c.device);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "set device");
    auto t0 = std::chrono::steady_clock::now();
    tpcf::Stats st;
    tpcf::Error err{0, ""};
    if (tpcf::batch_run(batch->b, full_out, region_out, &st, &err)) return fail(ctx, err.status, err.msg);
    if (stats) {
        stats->candidates = st.candidates;
        stats->in_range = st.in_range;
        stats->guard_evals = st.guard;
        stats->overflow_updates = st.overflow;
        stats->work_items = st.items;
        stats->ms_kernel = st.ms_kernel;
        stats->ms_total = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    }
    return TPCF_OK;
}

int tpcf_batch_n_outputs(const tpcf_batch *batch) { return batch ? tpcf::batch_jobs(batch->b) : -TPCF_E_INVALID_ARG; }
int tpcf_batch_order(const tpcf_batch *batch) { return batch ? tpcf::batch_order(batch->b) : -TPCF_E_INVALID_ARG; }
int tpcf_batch_refinement(const tpcf_batch *batch) {
    return batch ? tpcf::batch_refinement(batch->b) : -TPCF_E_INVALID_ARG;
}
int tpcf_batch_destroy(tpcf_batch *batch) {
    if (!batch) return TPCF_E_INVALID_ARG;
    cudaSetDevice(batch->ctx->c.device);
    delete batch;
    return TPCF_OK;
}

int tpcf_upweight_eval(const tpcf_weight_spec *spec, const double *values, int64_t n, double *out) {
    if (!spec || !spec->up_numerator || !spec->up_denominator || n < 0 || (n > 0 && (!values || !out)))
        return TPCF_E_INVALID_ARG;
    const tpcf_axis_spec &t = spec->theta_axis;
    if (t.n_bins < 1 || t.n_bins > tpcf::kMaxBins1D || !(t.max > t.min)) return TPCF_E_INVALID_ARG;
    const tpcf::UpTable up =
        tpcf::make_up_table(tpcf::make_axis(t.min, t.max, t.n_bins, t.log_base), spec->up_numerator,
                            spec->up_denominator);
    for (int64_t i = 0; i < n; ++i) out[i] = tpcf::up_eval(up, values[i]);
    return TPCF_OK;
}

int tpcf_auto_pair_count(tpcf_ctx *ctx, const tpcf_catalog *cat, const tpcf_binning *bin, int precision,
                         double *full_hist, double *sub_hist, tpcf_stats *stats) {
    return reference_form(ctx, cat, nullptr, bin, nullptr, precision, full_hist, sub_hist, stats);
}

int tpcf_cross_pair_count(tpcf_ctx *ctx, const tpcf_catalog *a, const tpcf_catalog *b, const tpcf_binning *bin,
                          int precision, double *full_hist, double *sub_hist, tpcf_stats *stats) {
    if (!b) return TPCF_E_INVALID_ARG;
    return reference_form(ctx, a, b, bin, nullptr, precision, full_hist, sub_hist, stats);
}

int tpcf_normalise_auto(const tpcf_catalog *cat, int32_t nb, double *full, double *sub) {
    if (!cat || !full || !sub || nb < 1) return TPCF_E_INVALID_ARG;
    const tpcf::Catalog &c = cat->c;
    const int nj = c.n_jk;
    const int n = c.n_kept;
    // src/hist.cpp:290-321
    double sw = 0.0;
    std::vector<double> swj(nj, 0.0);
    std::vector<int> nj_cnt(nj, 0);
    for (int k = 0; k < n; ++k) {
        const int i = c.h_kept[k];
        sw += c.h_w[i];
        swj[c.h_jk[i]] += c.h_w[i];
        ++nj_cnt[c.h_jk[i]];
    }
    for (int r = 0; r < nj; ++r) swj[r] = sw - swj[r];
    sw = sw * sw * (1.0 - 1.0 / (double)n);
    for (int r = 0; r < nj; ++r) swj[r] = swj[r] * swj[r] * (1.0 - 1.0 / nj_cnt[r]);
    for (int k = 0; k < nb; ++k) full[k] /= sw;
    for (int r = 0; r < nj; ++r)
        for (int k = 0; k < nb; ++k) sub[(size_t)r * nb + k] /= swj[r];
    return TPCF_OK;
}

int tpcf_normalise_cross(const tpcf_catalog *a, const tpcf_catalog *b, int32_t nb, double *full, double *sub) {
    if (!a || !b || !full || !sub || nb < 1 || a->c.n_jk != b->c.n_jk) return TPCF_E_INVALID_ARG;
    const int nj = a->c.n_jk;
    // src/hist.cpp:323-367
    auto sums = [nj](const tpcf::Catalog &c, double &s, std::vector<double> &sj) {
        s = 0.0;
        sj.assign(nj, 0.0);
        for (int k = 0; k < c.n_kept; ++k) {
            const int i = c.h_kept[k];
            s += c.h_w[i];
            sj[c.h_jk[i]] += c.h_w[i];
        }
        for (int r = 0; r < nj; ++r) sj[r] = s - sj[r];
    };
    double s1, s2;
    std::vector<double> j1, j2;
    sums(a->c, s1, j1);
    sums(b->c, s2, j2);
    s1 *= s2;
    for (int r = 0; r < nj; ++r) j1[r] *= j2[r];
    for (int k = 0; k < nb; ++k) full[k] /= s1;
    for (int r = 0; r < nj; ++r)
        for (int k = 0; k < nb; ++k) sub[(size_t)r * nb + k] /= j1[r];
    return TPCF_OK;
}

double tpcf_ls_estimator(double dd, double dr, double rr) {
    if (rr == 0) return 0;
    return dd / rr - 2.0 * dr / rr + 1.0;
}

uint64_t tpcf_kernel_launches(const tpcf_ctx *ctx) { return ctx ? ctx->c.launches : 0; }

int tpcf_measure_peaks(tpcf_ctx *ctx, double *fp32_tflops, double *smem_atomics_per_s) {
    if (!ctx || !fp32_tflops || !smem_atomics_per_s) return TPCF_E_INVALID_ARG;
    cudaError_t e = cudaSetDevice(ctx->c.device);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "set device");
    tpcf::Error err{0, ""};
    int rc = tpcf::measure_peaks(&ctx->c, fp32_tflops, smem_atomics_per_s, &err);
    if (rc) return fail(ctx, rc, err.msg);
    ctx->c.launches += 5;
    return TPCF_OK;
}

int tpcf_debug_fail_allocations(int64_t after) {
    tpcf::alloc_fail_budget().store(after < 0 ? -1 : (long long)after);
    return TPCF_OK;
}

int tpcf_debug_force_tile_timeout(int32_t on) {
    tpcf::debug_force_tile_timeout().store(on ? 1 : 0);
    return TPCF_OK;
}

int tpcf_debug_corrupt_work_list(int what) {
#ifdef TPCF_DEVICE_CHECKS
    if (what != 0 && what != 1) return TPCF_E_INVALID_ARG;
    tpcf::debug_corrupt_work_list().store(what);
    return TPCF_OK;
#else
    (void)what;
    return TPCF_E_UNSUPPORTED;  // the release build has no device checks to catch it
#endif
}

int tpcf_device_checks(void) {
#ifdef TPCF_DEVICE_CHECKS
    return 1;
#else
    return 0;
#endif
}

int tpcf_wait_selftest(tpcf_ctx *ctx, int32_t arrive, uint32_t limit) {
    if (!ctx || limit == 0) return TPCF_E_INVALID_ARG;
    cudaError_t e = cudaSetDevice(ctx->c.device);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "set device");
    tpcf::Error err{0, ""};
    int status = -1;
    int rc = tpcf::wait_selftest(&ctx->c, arrive ? 1 : 0, limit, &status, &err);
    if (rc) return fail(ctx, rc, err.msg);
    ++ctx->c.launches;
    if (status == 4) return fail(ctx, TPCF_E_DEVICE_TIMEOUT, "device wait exceeded its iteration limit (self-test)");
    if (status != 0) return fail(ctx, TPCF_E_CUDA, "self-test kernel reported no status");
    return TPCF_OK;
}

}  // extern "C"
