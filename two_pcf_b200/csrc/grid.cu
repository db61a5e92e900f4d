// K1: device counting sort of a catalogue into lattice cells — the
// replacement for GalaxyBoxes (src/boxes.cpp:10-163) and
// adj_id_to_box_index (src/boxes.cpp:191-206).
//
// Points are bucketed by (cell, jackknife region), buckets are scanned, and
// every point is scattered into structure-of-arrays tiles: float4
// (cell-relative position, weight) and float4 (unit vector, weight).  Cells
// are numbered in Morton order of their lattice coordinates when the padded
// cube stays small, so that neighbouring cells are close in memory.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>

#include "engine.h"

namespace tpcf {

namespace {

constexpr int kScanThreads = 512;
constexpr int kScanItems = 8;
constexpr int kScanTile = kScanThreads * kScanItems;

__device__ __forceinline__ int warp_incl_scan(int v) {
    const unsigned lane = threadIdx.x & 31;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        int t = __shfl_up_sync(0xffffffffu, v, o);
        if (lane >= (unsigned)o) v += t;
    }
    return v;
}

// Exclusive scan of one tile of kScanTile ints per block; the tile total
// goes to block_sums.
__global__ void __launch_bounds__(kScanThreads) scan_tile_kernel(const int *__restrict__ in, int *__restrict__ out,
                                                                 int *__restrict__ block_sums, long long n) {
    __shared__ int warp_tot[kScanThreads / 32];
    const long long base = (long long)blockIdx.x * kScanTile + (long long)threadIdx.x * kScanItems;
    int v[kScanItems];
    int run = 0;
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) {
        long long i = base + k;
        int x = (i < n) ? in[i] : 0;
        v[k] = run;
        run += x;
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    int incl = warp_incl_scan(run);
    if (lane == 31) warp_tot[warp] = incl;
    __syncthreads();
    if (warp == 0) {
        int t = (lane < kScanThreads / 32) ? warp_tot[lane] : 0;
        int s = warp_incl_scan(t);
        if (lane < kScanThreads / 32) warp_tot[lane] = s - t;
        if (lane == kScanThreads / 32 - 1 && block_sums) block_sums[blockIdx.x] = s;
    }
    __syncthreads();
    int offset = warp_tot[warp] + incl - run;
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) {
        long long i = base + k;
        if (i < n) out[i] = offset + v[k];
    }
}

__global__ void scan_add_kernel(int *__restrict__ out, const int *__restrict__ offsets, long long n) {
    long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] += offsets[i / kScanTile];
}

// Exclusive scan of n ints (in may equal out).  Totals must fit in int.
// The tile sums come from `pool` (the context's pool, which keeps released
// memory): the device's default pool hands its memory back to the driver at
// every synchronisation, and mapping it again was measured stalling a grid
// build for up to 0.9 s.
cudaError_t exclusive_scan(const int *in, int *out, long long n, cudaStream_t st, unsigned long long *launches,
                           cudaMemPool_t pool) {
    if (n <= 0) return cudaSuccess;
    long long tiles = (n + kScanTile - 1) / kScanTile;
    if (tiles == 1) {
        scan_tile_kernel<<<1, kScanThreads, 0, st>>>(in, out, nullptr, n);
        ++*launches;
        return cudaGetLastError();
    }
    int *sums = nullptr;
    cudaError_t e = pool ? cudaMallocFromPoolAsync((void **)&sums, sizeof(int) * tiles, pool, st)
                         : cudaMallocAsync((void **)&sums, sizeof(int) * tiles, st);
    if (e != cudaSuccess) return e;
    scan_tile_kernel<<<(unsigned)tiles, kScanThreads, 0, st>>>(in, out, sums, n);
    ++*launches;
    e = exclusive_scan(sums, sums, tiles, st, launches, pool);
    if (e == cudaSuccess) {
        scan_add_kernel<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(out, sums, n);
        ++*launches;
        e = cudaGetLastError();
    }
    cudaFreeAsync(sums, st);
    return e;
}

__host__ __device__ __forceinline__ unsigned spread3(unsigned v) {
    v &= 0x3ffu;
    v = (v | (v << 16)) & 0x030000FFu;
    v = (v | (v << 8)) & 0x0300F00Fu;
    v = (v | (v << 4)) & 0x030C30C3u;
    v = (v | (v << 2)) & 0x09249249u;
    return v;
}

__host__ __device__ __forceinline__ unsigned compact3(unsigned v) {
    v &= 0x09249249u;
    v = (v | (v >> 2)) & 0x030C30C3u;
    v = (v | (v >> 4)) & 0x0300F00Fu;
    v = (v | (v >> 8)) & 0x030000FFu;
    v = (v | (v >> 16)) & 0x3ffu;
    return v;
}

struct GeomDev {
    double side;
    int kmin0, kmin1, kmin2;
    int dim0, dim1, dim2;
    int morton;
    int n_jk;
};

__device__ __forceinline__ int dense_id(const GeomDev &g, int cx, int cy, int cz) {
    if (g.morton) return (int)(spread3(cx) | (spread3(cy) << 1) | (spread3(cz) << 2));
    return (cx * g.dim1 + cy) * g.dim2 + cz;
}

__device__ __forceinline__ int cell_of(const GeomDev &g, double x, int kmin, int dim) {
    // Same formula as the host bounding box: floor(x / side).
    int c = (int)floor(x / g.side) - kmin;
    return c < 0 ? 0 : (c >= dim ? dim - 1 : c);
}

__global__ void assign_kernel(GeomDev g, const double *__restrict__ xyz, const int *__restrict__ jk,
                              const int *__restrict__ subset, int n, int *__restrict__ bucket,
                              int *__restrict__ counts) {
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    int i = subset ? subset[t] : t;
    double x = xyz[3 * (size_t)i], y = xyz[3 * (size_t)i + 1], z = xyz[3 * (size_t)i + 2];
    int cx = cell_of(g, x, g.kmin0, g.dim0), cy = cell_of(g, y, g.kmin1, g.dim1), cz = cell_of(g, z, g.kmin2, g.dim2);
    int r = jk ? jk[i] : 0;
    int b = dense_id(g, cx, cy, cz) * g.n_jk + r;
    bucket[t] = b;
    atomicAdd(&counts[b], 1);
}

__global__ void scatter_kernel(GeomDev g, const double *__restrict__ xyz, const double *__restrict__ unit,
                               const float *__restrict__ w, const int *__restrict__ jk,
                               const int *__restrict__ subset, int n, const int *__restrict__ bucket,
                               const int *__restrict__ start, int *__restrict__ fill, float4 *__restrict__ pos,
                               float4 *__restrict__ aux, int *__restrict__ idx, double4 *__restrict__ xyz_s,
                               double4 *__restrict__ unit_s) {
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    int i = subset ? subset[t] : t;
    int b = bucket[t];
    int dst = start[b] + atomicAdd(&fill[b], 1);
    double x = xyz[3 * (size_t)i], y = xyz[3 * (size_t)i + 1], z = xyz[3 * (size_t)i + 2];
    int cx = cell_of(g, x, g.kmin0, g.dim0), cy = cell_of(g, y, g.kmin1, g.dim1), cz = cell_of(g, z, g.kmin2, g.dim2);
    double ox = (double)(g.kmin0 + cx) * g.side, oy = (double)(g.kmin1 + cy) * g.side,
           oz = (double)(g.kmin2 + cz) * g.side;
    double nx = unit[3 * (size_t)i], ny = unit[3 * (size_t)i + 1], nz = unit[3 * (size_t)i + 2];
    float wi = w ? w[i] : 1.0f;
    pos[dst] = make_float4(__double2float_rn(x - ox), __double2float_rn(y - oy), __double2float_rn(z - oz), wi);
    const int r = jk ? jk[i] : 0;
    aux[dst] = make_float4(__double2float_rn(0.5 * nx), __double2float_rn(0.5 * ny), __double2float_rn(0.5 * nz), wi);
    idx[dst] = i;
    if (xyz_s) {
        xyz_s[dst] = make_double4(x, y, z, (double)wi);
        unit_s[dst] = make_double4(nx, ny, nz, (double)r);
    }
}

// Per dense cell: point range, local coordinates and the number of distinct
// regions present.
__global__ void cells_kernel(GeomDev g, int ncell, int npts, const int *__restrict__ bstart,
                             int *__restrict__ cell_start, int3 *__restrict__ coord, int *__restrict__ nreg) {
    int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c > ncell) return;
    if (c == ncell) {
        cell_start[c] = npts;
        return;
    }
    cell_start[c] = bstart[(size_t)c * g.n_jk];
    int cx, cy, cz;
    if (g.morton) {
        cx = (int)compact3((unsigned)c);
        cy = (int)compact3((unsigned)c >> 1);
        cz = (int)compact3((unsigned)c >> 2);
        if (cx >= g.dim0 || cy >= g.dim1 || cz >= g.dim2) cx = cy = cz = -1;
    } else {
        cx = c / (g.dim1 * g.dim2);
        cy = (c / g.dim2) % g.dim1;
        cz = c % g.dim2;
    }
    coord[c] = make_int3(cx, cy, cz);
    int k = 0;
    for (int r = 0; r < g.n_jk; ++r) {
        size_t b = (size_t)c * g.n_jk + r;
        k += (bstart[b + 1] > bstart[b]) ? 1 : 0;
    }
    nreg[c] = k;
}

// Runs of one region inside one cell, in sorted order: region id and first
// point of each run (CSR by cell).
__global__ void regions_kernel(GeomDev g, int ncell, const int *__restrict__ bstart, const int *__restrict__ rstart,
                               int *__restrict__ regions, int *__restrict__ run_start) {
    int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= ncell) return;
    int k = rstart[c];
    for (int r = 0; r < g.n_jk; ++r) {
        size_t b = (size_t)c * g.n_jk + r;
        if (bstart[b + 1] > bstart[b]) {
            regions[k] = r;
            run_start[k] = bstart[b];
            ++k;
        }
    }
}

// New weights for the points of a cached grid: pos.w (and xyz_s.w) from the
// catalogue's weight array through the grid's index.
__global__ void reweight_kernel(int n, const int *__restrict__ idx, const float *__restrict__ w,
                                float4 *__restrict__ pos, float4 *__restrict__ aux, double4 *__restrict__ xyz_s) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    const float wi = w[idx[k]];
    pos[k].w = wi;
    aux[k].w = wi;
    if (xyz_s) xyz_s[k].w = (double)wi;
}

}  // namespace

#define TPCF_CUDA_TRY(expr)                                                              \
    do {                                                                                 \
        cudaError_t _e = (expr);                                                         \
        if (_e != cudaSuccess) {                                                         \
            err->status = (_e == cudaErrorMemoryAllocation) ? 2 : 3;                     \
            err->msg = std::string("CUDA error in grid build: ") + cudaGetErrorString(_e); \
            return err->status;                                                          \
        }                                                                                \
    } while (0)

namespace {
std::string grid_key(const GridSpec &spec) {
    char key[128];
    snprintf(key, sizeof(key), "%a|%d|%d|%d", spec.side, spec.subset_kept ? 1 : 0, spec.angular ? 1 : 0,
             spec.input_w ? 1 : 0);
    return key;
}
}  // namespace

Grid *find_grid(Catalog *cat, const GridSpec &spec, bool want_fp64) {
    auto it = cat->grids.find(grid_key(spec));
    if (it == cat->grids.end() || (want_fp64 && !it->second->has_fp64)) return nullptr;
    return it->second.get();
}

int build_grid(Ctx *ctx, Catalog *cat, const GridSpec &spec, bool want_fp64, Grid **out, Error *err) {
    const std::string key = grid_key(spec);
    auto it = cat->grids.find(key);
    if (it != cat->grids.end() && (!want_fp64 || it->second->has_fp64)) {
        *out = it->second.get();
        return 0;
    }
    const double side = spec.side;
    const bool subset_kept = spec.subset_kept;
    cudaStream_t st = ctx->stream;
    // TPCF_TRACE=1: host time of the build's phases on stderr (diagnostics)
    const bool trace = trace_enabled();
    using clk = std::chrono::steady_clock;
    const auto t0 = clk::now();
    auto ms_since = [&](clk::time_point a) { return std::chrono::duration<double, std::milli>(clk::now() - a).count(); };
    double t_alloc = 0, t_launch = 0, t_sync1 = 0;
    std::unique_ptr<Grid> g(new Grid());
    g->side = side;
    g->subset_kept = subset_kept;
    g->angular = spec.angular;
    g->input_w = spec.input_w;
    const double *lo = spec.angular ? (subset_kept ? cat->ulo_kept : cat->ulo_all)
                                    : (subset_kept ? cat->lo_kept : cat->lo_all);
    const double *hi = spec.angular ? (subset_kept ? cat->uhi_kept : cat->uhi_all)
                                    : (subset_kept ? cat->hi_kept : cat->hi_all);
    // Coordinates the cells are built on, and the weight each point carries.
    const double *coords = spec.angular ? cat->unit.p : cat->xyz.p;
    const float *wsrc = nullptr;
    if (spec.input_w) wsrc = cat->iw.p ? cat->iw.p : (cat->unit_weights ? nullptr : cat->w.p);
    else wsrc = cat->unit_weights ? nullptr : cat->w.p;
    int n = subset_kept ? cat->n_kept : (int)cat->n_all;
    g->n = n;
    int maxdim = 1;
    long long dense = 1;
    for (int m = 0; m < 3; ++m) {
        if (n > 0) {
            g->kmin[m] = (int)std::floor(lo[m] / side);
            int kmax = (int)std::floor(hi[m] / side);
            g->dim[m] = kmax - g->kmin[m] + 1;
        } else {
            g->kmin[m] = 0;
            g->dim[m] = 1;
        }
        maxdim = std::max(maxdim, g->dim[m]);
        dense *= g->dim[m];
    }
    int p2 = 1;
    while (p2 < maxdim) p2 <<= 1;
    long long mcube = (long long)p2 * p2 * p2;
    g->morton = (p2 <= 1024) && (mcube <= 4 * dense || mcube <= (1 << 15));
    long long ncell = g->morton ? mcube : dense;
    if (ncell * (long long)cat->n_jk > (1LL << 28) || ncell > (1LL << 27)) {
        err->status = 6;
        err->msg = "grid too fine for the catalogue extent (more than 2^28 cell-region buckets); "
                   "use a coarser refinement";
        return err->status;
    }
    g->ncell = (int)ncell;
    GeomDev gd{side, g->kmin[0], g->kmin[1], g->kmin[2], g->dim[0], g->dim[1], g->dim[2], g->morton ? 1 : 0,
               cat->n_jk};

    long long nbucket = ncell * cat->n_jk;
    ScratchBuf<int> bucket, counts;
    TPCF_CUDA_TRY(bucket.alloc(*ctx, n));
    TPCF_CUDA_TRY(counts.alloc(*ctx, nbucket + 1));
    TPCF_CUDA_TRY(g->pos.alloc(*ctx, n));
    TPCF_CUDA_TRY(g->aux.alloc(*ctx, n));
    TPCF_CUDA_TRY(g->idx.alloc(*ctx, n));
    if (want_fp64) {
        TPCF_CUDA_TRY(g->xyz_s.alloc(*ctx, n));
        TPCF_CUDA_TRY(g->unit_s.alloc(*ctx, n));
        g->has_fp64 = true;
    }
    TPCF_CUDA_TRY(g->cell_start.alloc(*ctx, ncell + 1));
    TPCF_CUDA_TRY(g->cell_coord.alloc(*ctx, ncell));
    TPCF_CUDA_TRY(g->region_start.alloc(*ctx, ncell + 1));
    if (trace) t_alloc = ms_since(t0);
    TPCF_CUDA_TRY(cudaMemsetAsync(counts.p, 0, sizeof(int) * (nbucket + 1), st));
    const int *subset = subset_kept ? cat->kept.p : nullptr;
    const int *jk = cat->n_jk > 1 ? cat->jk.p : nullptr;
    if (n > 0) {
        assign_kernel<<<(n + 255) / 256, 256, 0, st>>>(gd, coords, jk, subset, n, bucket.p, counts.p);
        ++ctx->launches;
        TPCF_CUDA_TRY(cudaGetLastError());
    }
    // counts -> bucket starts (exclusive); the extra element becomes n.
    TPCF_CUDA_TRY(exclusive_scan(counts.p, counts.p, nbucket + 1, st, &ctx->launches, ctx->pool));
    ScratchBuf<int> fill;
    TPCF_CUDA_TRY(fill.alloc(*ctx, nbucket));
    TPCF_CUDA_TRY(cudaMemsetAsync(fill.p, 0, sizeof(int) * nbucket, st));
    if (n > 0) {
        scatter_kernel<<<(n + 255) / 256, 256, 0, st>>>(gd, coords, cat->unit.p, wsrc,
                                                        jk, subset, n, bucket.p, counts.p, fill.p, g->pos.p,
                                                        g->aux.p, g->idx.p, want_fp64 ? g->xyz_s.p : nullptr,
                                                        want_fp64 ? g->unit_s.p : nullptr);
        ++ctx->launches;
        TPCF_CUDA_TRY(cudaGetLastError());
    }
    ScratchBuf<int> nreg;
    TPCF_CUDA_TRY(nreg.alloc(*ctx, ncell + 1));
    TPCF_CUDA_TRY(cudaMemsetAsync(nreg.p, 0, sizeof(int) * (ncell + 1), st));
    cells_kernel<<<(unsigned)((ncell + 1 + 255) / 256), 256, 0, st>>>(gd, (int)ncell, n, counts.p, g->cell_start.p,
                                                                     g->cell_coord.p, nreg.p);
    ++ctx->launches;
    TPCF_CUDA_TRY(cudaGetLastError());
    TPCF_CUDA_TRY(exclusive_scan(nreg.p, g->region_start.p, ncell + 1, st, &ctx->launches, ctx->pool));
    g->h_region_start.resize(ncell + 1);
    TPCF_CUDA_TRY(cudaMemcpyAsync(g->h_region_start.data(), g->region_start.p, sizeof(int) * (ncell + 1),
                                  cudaMemcpyDeviceToHost, st));
    g->h_cell_start.resize(ncell + 1);
    TPCF_CUDA_TRY(cudaMemcpyAsync(g->h_cell_start.data(), g->cell_start.p, sizeof(int) * (ncell + 1),
                                  cudaMemcpyDeviceToHost, st));
    if (trace) t_launch = ms_since(t0);
    TPCF_CUDA_TRY(cudaStreamSynchronize(st));
    if (trace) t_sync1 = ms_since(t0);
    int nregions = g->h_region_start[ncell];
    TPCF_CUDA_TRY(g->regions.alloc(*ctx, nregions));
    TPCF_CUDA_TRY(g->run_start.alloc(*ctx, nregions));
    regions_kernel<<<(unsigned)((ncell + 255) / 256), 256, 0, st>>>(gd, (int)ncell, counts.p, g->region_start.p,
                                                                   g->regions.p, g->run_start.p);
    ++ctx->launches;
    TPCF_CUDA_TRY(cudaGetLastError());
    g->h_regions.resize(nregions);
    g->h_run_start.resize(nregions);
    if (nregions > 0) {
        TPCF_CUDA_TRY(cudaMemcpyAsync(g->h_regions.data(), g->regions.p, sizeof(int) * nregions,
                                      cudaMemcpyDeviceToHost, st));
        TPCF_CUDA_TRY(cudaMemcpyAsync(g->h_run_start.data(), g->run_start.p, sizeof(int) * nregions,
                                      cudaMemcpyDeviceToHost, st));
    }
    TPCF_CUDA_TRY(cudaStreamSynchronize(st));
    if (trace)
        std::fprintf(stderr, "[tpcf trace] grid of %d points, %d cells: allocated %.1f, launched %.1f, first sync %.1f, "
                     "done %.1f ms (host)\n", n, (int)ncell, t_alloc, t_launch, t_sync1, ms_since(t0));
    *out = g.get();
    cat->grids[key] = std::move(g);
    return 0;
}

int reweight_grids(Ctx *ctx, Catalog *cat, Error *err) {
    for (auto &kv : cat->grids) {
        Grid *g = kv.second.get();
        if (g->input_w && cat->iw.p) continue;  // carries input weights, which did not change
        if (g->n == 0) continue;
        reweight_kernel<<<(g->n + 255) / 256, 256, 0, ctx->stream>>>(g->n, g->idx.p, cat->w.p, g->pos.p, g->aux.p,
                                                                     g->has_fp64 ? g->xyz_s.p : nullptr);
        ++ctx->launches;
        TPCF_CUDA_TRY(cudaGetLastError());
    }
    return 0;
}

}  // namespace tpcf
