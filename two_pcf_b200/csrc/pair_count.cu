// K2 (FP32 + guard) and K7 (plain FP64) 3-D pair counting: the replacement
// for auto_/cross_pair_count_{monopole,sigma_pi,s_mu}
// (src/correlators.cpp:11-125, :156-278, :309-430).
//
// One persistent CTA per SM pulls work items (a chunk of cell A against all
// of cell B) from a device queue.  Each thread holds R points of A in
// registers; B is streamed through shared memory in tiles by one-dimensional
// bulk copies (cp.async.bulk, completion on an mbarrier, double buffered).
// Separations are evaluated in FP32 from cell-relative coordinates; a pair
// whose FP32 value lies within the proven error bound of the range limits or
// of a bin threshold is re-evaluated with the reference's exact float/double
// operation sequence (exact_pair below).  Pairs are binned into privatised
// shared-memory histograms — one slice for the full histogram and a set of
// slots for jackknife regions, assigned per work item — holding 64-bit fixed
// point sums, and merged into global 64-bit integers.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "engine.h"
#include "pair_kernels.cuh"

namespace tpcf {
namespace {

constexpr int NT = 256;        // threads per CTA
constexpr int R = 4;           // A points per thread
constexpr int TA = NT * R;     // A chunk
constexpr int TB = 256;        // B points per staged tile
constexpr int kMaxSlots = 32;  // jackknife slots per CTA
constexpr uint32_t kWaitLimit = 1u << 22;

struct GridK {
    const float4 *pos;
    const float4 *aux;
    const int *idx;
    const double4 *xyz_s;
    const double4 *unit_s;
    const int3 *coord;
    const int *rstart;
    const int *regions;
    int kmin0, kmin1, kmin2;
    const double *xyz;   // original catalogue arrays (exact path)
    const double *unit;
};

struct KParams {
    GridK a, b;
    const WorkItem *items;
    int n_items;
    int *head;
    double side;
    int n1, n2, nb;
    float min_r_sq, max_r_sq, lo_cut, hi_cut;
    float g_s2, g_pi, g_a, c1_mu, c2_mu, g_mu0;
    const float *t1g, *t2g;
    int ax1_log, ax2_log;
    float ax1_min, ax1_inv_step, ax1_ilb, ax1_ils;
    float ax2_min, ax2_inv_step, ax2_ilb, ax2_ils;
    unsigned long long *g_full, *g_sub;
    int n_jk, ns;
    float wscale;
    unsigned long long *counters;  // candidates, in_range, guard, overflow
    int *err;
};

struct Misc {
    int item;
    int stop;
    int n_evict;
    int slot_region[kMaxSlots];
    int slot_stamp[kMaxSlots];
    int evict_slot[kMaxSlots];
    int evict_region[kMaxSlots];
};

struct SmemLayout {
    size_t lo, hi, t1, t2, slotmap, misc, tile0, tile1, bar, total;
};

__host__ __device__ inline size_t tile_bytes(bool exact) { return (size_t)TB * (exact ? 64 : 32); }

__host__ __device__ inline SmemLayout smem_layout(int nb, int ns, int n1, int n2, int n_jk_map, bool exact) {
    SmemLayout L;
    size_t o = 0;
    L.lo = o;
    o += 4 * (size_t)(ns + 1) * nb;
    L.hi = o;
    o += 4 * (size_t)(ns + 1) * nb;
    L.t1 = o;
    o += 4 * (size_t)(n1 + 1);
    L.t2 = o;
    o += 4 * (size_t)(n2 + 1);
    o = (o + 3) / 4 * 4;
    L.slotmap = o;
    o += 2 * (size_t)n_jk_map;
    o = (o + 15) / 16 * 16;
    L.misc = o;
    o += sizeof(Misc);
    o = (o + 127) / 128 * 128;
    L.tile0 = o;
    o += tile_bytes(exact);
    L.tile1 = o;
    o += tile_bytes(exact);
    o = (o + 7) / 8 * 8;
    L.bar = o;
    o += 16;
    L.total = o;
    return L;
}

// Exact evaluation of one pair with the reference's operation sequence
// (src/correlators.cpp:33-40 separation and range test; :166-170 pi with
// _ANGULAR_PI_DEFN; :185 sigma; :338-340 s and mu; src/hist.cpp:484-502
// binning), bins looked up in the threshold tables.  Returns the flat bin or
// -1; *in_range receives the range-test result.
// Parameters of the exact evaluation, passed by value so that the
// non-inlined guard path needs no copy of the kernel parameter block.
struct ExactArgs {
    const double *a_xyz, *a_unit, *b_xyz, *b_unit;
    float min_r_sq, max_r_sq;
    int n1, n2;
};

template <int MODE>
__device__ __forceinline__ int exact_bin(const ExactArgs &E, const float *t1, const float *t2, float d0, float d1,
                                         float d2, double n1x, double n1y, double n1z, double n2x, double n2y,
                                         double n2z, bool *in_range) {
    float s2 = __fadd_rn(__fadd_rn(__fmul_rn(d0, d0), __fmul_rn(d1, d1)), __fmul_rn(d2, d2));
    *in_range = (s2 < E.max_r_sq) && (s2 > E.min_r_sq);
    if (!*in_range) return -1;
    if (MODE == MODE_MONOPOLE) {
        int b = dev::locate_exact(t1, E.n1, s2);
        return (b >= 0 && b < E.n1) ? b : -1;
    }
    float pi = __double2float_rn(__dmul_rn((double)d0, __dadd_rn(n1x, n2x)));
    pi = __double2float_rn(__dadd_rn((double)pi, __dmul_rn((double)d1, __dadd_rn(n1y, n2y))));
    pi = __double2float_rn(__dadd_rn((double)pi, __dmul_rn((double)d2, __dadd_rn(n1z, n2z))));
    pi = __double2float_rn(__dmul_rn((double)pi, 0.5));
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
template <int MODE>
__device__ __noinline__ int exact_pair(const ExactArgs E, const float *t1, const float *t2, int ia, int jb,
                                       bool *in_range) {
    const double *x1 = E.a_xyz + 3 * (size_t)ia, *x2 = E.b_xyz + 3 * (size_t)jb;
    float d0 = __double2float_rn(__dsub_rn(x1[0], x2[0]));
    float d1 = __double2float_rn(__dsub_rn(x1[1], x2[1]));
    float d2 = __double2float_rn(__dsub_rn(x1[2], x2[2]));
    double n1x = 0, n1y = 0, n1z = 0, n2x = 0, n2y = 0, n2z = 0;
    if (MODE != MODE_MONOPOLE) {
        const double *u1 = E.a_unit + 3 * (size_t)ia, *u2 = E.b_unit + 3 * (size_t)jb;
        n1x = u1[0];
        n1y = u1[1];
        n1z = u1[2];
        n2x = u2[0];
        n2y = u2[1];
        n2z = u2[2];
    }
    return exact_bin<MODE>(E, t1, t2, d0, d1, d2, n1x, n1y, n1z, n2x, n2y, n2z, in_range);
}

template <int MODE, bool UNITW, bool JK, bool EXACT>
__global__ void __launch_bounds__(NT, 1) pair_count_kernel(const KParams P) {
    extern __shared__ __align__(128) unsigned char smem[];
    constexpr bool kNeedAux = (MODE != MODE_MONOPOLE) || JK;
    const SmemLayout L = smem_layout(P.nb, P.ns, P.n1, P.n2, JK ? P.n_jk : 0, EXACT);
    uint32_t *s_lo = (uint32_t *)(smem + L.lo);
    uint32_t *s_hi = (uint32_t *)(smem + L.hi);
    float *s_t1 = (float *)(smem + L.t1);
    float *s_t2 = (float *)(smem + L.t2);
    short *s_slot = (short *)(smem + L.slotmap);
    Misc *s_misc = (Misc *)(smem + L.misc);
    unsigned char *tiles[2] = {smem + L.tile0, smem + L.tile1};
    uint64_t *bar = (uint64_t *)(smem + L.bar);
    const int tid = threadIdx.x;
    const int nslices = P.ns + 1;  // slice P.ns is the full histogram
    const int full_base = P.ns * P.nb;

    for (int i = tid; i < nslices * P.nb; i += NT) {
        s_lo[i] = 0;
        s_hi[i] = 0;
    }
    for (int i = tid; i <= P.n1; i += NT) s_t1[i] = P.t1g[i];
    for (int i = tid; i <= P.n2; i += NT) s_t2[i] = P.t2g[i];
    if (JK)
        for (int i = tid; i < P.n_jk; i += NT) s_slot[i] = -1;
    if (tid == 0) {
        for (int s = 0; s < kMaxSlots; ++s) {
            s_misc->slot_region[s] = -1;
            s_misc->slot_stamp[s] = -1;
        }
        s_misc->stop = 0;
        dev::mbar_init(&bar[0], 1);
        dev::mbar_init(&bar[1], 1);
        dev::mbar_init_fence();
    }
    __syncthreads();

    const ExactArgs EA{P.a.xyz, P.a.unit, P.b.xyz, P.b.unit, P.min_r_sq, P.max_r_sq, P.n1, P.n2};
    const dev::AxisK ax1{s_t1, P.n1, P.ax1_log, P.ax1_min, P.ax1_inv_step, P.ax1_ilb, P.ax1_ils};
    const dev::AxisK ax2{s_t2, P.n2, P.ax2_log, P.ax2_min, P.ax2_inv_step, P.ax2_ilb, P.ax2_ils};

    unsigned long long n_in = 0, n_guard = 0, n_over = 0, n_cand = 0;
    unsigned tcount = 0;  // tiles staged so far by this CTA (selects buffer and phase)
    int stamp = 0;

    for (;;) {
        if (tid == 0) {
            int item = atomicAdd(P.head, 1);
            if (*(volatile int *)P.err != 0) item = P.n_items;
            s_misc->item = item;
        }
        __syncthreads();
        const int item = s_misc->item;
        if (item >= P.n_items) break;
        const WorkItem it = P.items[item];
        ++stamp;
        if (tid == 0) {
            long long al = it.a_len, bl = it.b_len;
            n_cand += it.self ? (unsigned long long)(al * bl - al * (al + 1) / 2) : (unsigned long long)(al * bl);
        }

        // ---- jackknife slot assignment for the regions of cells A and B
        if (JK) {
            if (tid == 0) {
                s_misc->n_evict = 0;
                const int *la = P.a.regions + P.a.rstart[it.a_cell];
                const int na = P.a.rstart[it.a_cell + 1] - P.a.rstart[it.a_cell];
                const int *lb = P.b.regions + P.b.rstart[it.b_cell];
                const int nbr = P.b.rstart[it.b_cell + 1] - P.b.rstart[it.b_cell];
                // pass 1: regions that already hold a slot keep it
                for (int pass = 0; pass < 2; ++pass) {
                    for (int k = 0; k < na + nbr; ++k) {
                        const int r = k < na ? la[k] : lb[k - na];
                        const int s = s_slot[r];
                        if (pass == 0) {
                            if (s >= 0) s_misc->slot_stamp[s] = stamp;
                            continue;
                        }
                        if (s >= 0) continue;
                        int pick = -1;
                        for (int q = 0; q < P.ns; ++q)
                            if (s_misc->slot_region[q] < 0) {
                                pick = q;
                                break;
                            }
                        if (pick < 0)
                            for (int q = 0; q < P.ns; ++q)
                                if (s_misc->slot_stamp[q] != stamp) {
                                    pick = q;
                                    break;
                                }
                        if (pick < 0) continue;  // no slot left: this region goes to global memory
                        const int old = s_misc->slot_region[pick];
                        if (old >= 0) {
                            const int e = s_misc->n_evict++;
                            s_misc->evict_slot[e] = pick;
                            s_misc->evict_region[e] = old;
                            s_slot[old] = -1;
                        }
                        s_misc->slot_region[pick] = r;
                        s_misc->slot_stamp[pick] = stamp;
                        s_slot[r] = (short)pick;
                    }
                }
            }
            __syncthreads();
            const int ne = s_misc->n_evict;
            for (int e = 0; e < ne; ++e) {
                const int s = s_misc->evict_slot[e], r = s_misc->evict_region[e];
                for (int b = tid; b < P.nb; b += NT) {
                    const int i = s * P.nb + b;
                    const unsigned long long v = ((unsigned long long)s_hi[i] << 32) | s_lo[i];
                    if (v) {
                        atomicAdd(&P.g_sub[(size_t)r * P.nb + b], v);
                        s_lo[i] = 0;
                        s_hi[i] = 0;
                    }
                }
            }
            if (ne) __syncthreads();
        }

        // ---- A points into registers, shifted into B's cell frame
        const int3 ca = P.a.coord[it.a_cell], cb = P.b.coord[it.b_cell];
        const double offx = (double)((P.a.kmin0 + ca.x) - (P.b.kmin0 + cb.x)) * P.side;
        const double offy = (double)((P.a.kmin1 + ca.y) - (P.b.kmin1 + cb.y)) * P.side;
        const double offz = (double)((P.a.kmin2 + ca.z) - (P.b.kmin2 + cb.z)) * P.side;
        float ax[R], ay[R], az[R], aw[R], anx[R], any_[R], anz[R];
        int ai[R], ajk[R], aslot[R];
        double dax[R], day[R], daz[R];
        (void)dax; (void)day; (void)daz;
#pragma unroll
        for (int r = 0; r < R; ++r) {
            const int k = tid + r * NT;
            const bool valid = k < it.a_len;
            const int gi = it.a_start + k;
            ai[r] = valid ? gi : 0x7fffffff;
            ax[r] = ay[r] = az[r] = 1e30f;
            aw[r] = 0.0f;
            anx[r] = any_[r] = anz[r] = 0.0f;
            ajk[r] = 0;
            aslot[r] = -1;
            if (EXACT) {
                dax[r] = day[r] = daz[r] = 1e300;
                if (valid) {
                    const double4 p = P.a.xyz_s[gi];
                    dax[r] = p.x;
                    day[r] = p.y;
                    daz[r] = p.z;
                    aw[r] = (float)p.w;
                    if (JK) ajk[r] = (int)P.a.unit_s[gi].w;
                }
            } else if (valid) {
                const float4 p = P.a.pos[gi];
                ax[r] = p.x + (float)offx;
                ay[r] = p.y + (float)offy;
                az[r] = p.z + (float)offz;
                aw[r] = p.w;
                if (kNeedAux) {
                    const float4 q = P.a.aux[gi];
                    anx[r] = q.x;
                    any_[r] = q.y;
                    anz[r] = q.z;
                    ajk[r] = __float_as_int(q.w);
                }
            }
            if (JK && valid) aslot[r] = s_slot[ajk[r]];
        }

        // ---- stream B through shared memory
        const int ntiles = (it.b_len + TB - 1) / TB;
        auto issue = [&](unsigned tc, int start, int len) {
            unsigned char *dst = tiles[tc & 1];
            dev::fence_proxy_async();
            if (EXACT) {
                const uint32_t by = (uint32_t)len * 32u;
                dev::mbar_expect_tx(&bar[tc & 1], (MODE != MODE_MONOPOLE || JK) ? 2 * by : by);
                dev::bulk_g2s(dst, P.b.xyz_s + start, by, &bar[tc & 1]);
                if (MODE != MODE_MONOPOLE || JK) dev::bulk_g2s(dst + (size_t)TB * 32, P.b.unit_s + start, by, &bar[tc & 1]);
            } else {
                const uint32_t by = (uint32_t)len * 16u;
                dev::mbar_expect_tx(&bar[tc & 1], kNeedAux ? 2 * by : by);
                dev::bulk_g2s(dst, P.b.pos + start, by, &bar[tc & 1]);
                if (kNeedAux) dev::bulk_g2s(dst + (size_t)TB * 16, P.b.aux + start, by, &bar[tc & 1]);
            }
        };
        if (tid == 0 && ntiles > 0) issue(tcount, it.b_start, min(TB, it.b_len));

        for (int t = 0; t < ntiles; ++t) {
            const int tstart = t * TB;
            const int tlen = min(TB, it.b_len - tstart);
            if (tid == 0 && t + 1 < ntiles)
                issue(tcount + 1, it.b_start + tstart + TB, min(TB, it.b_len - tstart - TB));
            if (!dev::mbar_wait_bounded(&bar[tcount & 1], (tcount >> 1) & 1u, kWaitLimit)) {
                atomicExch(P.err, 4);  // device timeout: results are discarded by the host
            }
            const int jbase = it.b_start + tstart;
            if (EXACT) {
                const double4 *s_xyz = (const double4 *)tiles[tcount & 1];
                const double4 *s_unit = (const double4 *)(tiles[tcount & 1] + (size_t)TB * 32);
                for (int jj = 0; jj < tlen; ++jj) {
                    const double4 pb = s_xyz[jj];
                    const int jg = jbase + jj;
#pragma unroll
                    for (int r = 0; r < R; ++r) {
                        const float d0 = __double2float_rn(__dsub_rn(dax[r], pb.x));
                        const float d1 = __double2float_rn(__dsub_rn(day[r], pb.y));
                        const float d2 = __double2float_rn(__dsub_rn(daz[r], pb.z));
                        const float s2 = __fadd_rn(__fadd_rn(__fmul_rn(d0, d0), __fmul_rn(d1, d1)), __fmul_rn(d2, d2));
                        bool hit = (s2 < P.max_r_sq) && (s2 > P.min_r_sq);
                        if (it.self) hit = hit && (jg > ai[r]);
                        if (hit) {
                            ++n_in;
                            int bin;
                            double4 ub = make_double4(0, 0, 0, 0);
                            if (MODE != MODE_MONOPOLE || JK) ub = s_unit[jj];
                            if (MODE == MODE_MONOPOLE) {
                                bin = dev::locate_exact(s_t1, P.n1, s2);
                                if (bin >= P.n1) bin = -1;
                            } else {
                                const double4 ua = P.a.unit_s[ai[r]];
                                bool inr;
                                bin = exact_bin<MODE>(EA, s_t1, s_t2, d0, d1, d2, ua.x, ua.y, ua.z, ub.x, ub.y, ub.z,
                                                      &inr);
                            }
                            if (bin >= 0) {
                                const float w = UNITW ? 1.0f : __fmul_rn(aw[r], (float)pb.w);
                                const long long q = UNITW ? 1LL : __float2ll_rn(__fmul_rn(w, P.wscale));
                                dev::acc_add(s_lo, s_hi, full_base + bin, q);
                                if (JK) {
                                    const int ja = ajk[r], jb = (int)ub.w;
                                    const int sa = aslot[r];
                                    if (sa >= 0) dev::acc_add(s_lo, s_hi, sa * P.nb + bin, q);
                                    else { dev::acc_add_global(P.g_sub, (size_t)ja * P.nb + bin, q); ++n_over; }
                                    if (jb != ja) {
                                        const int sb = s_slot[jb];
                                        if (sb >= 0) dev::acc_add(s_lo, s_hi, sb * P.nb + bin, q);
                                        else { dev::acc_add_global(P.g_sub, (size_t)jb * P.nb + bin, q); ++n_over; }
                                    }
                                }
                            }
                        }
                    }
                }
            } else {
                const float4 *s_pos = (const float4 *)tiles[tcount & 1];
                const float4 *s_aux = (const float4 *)(tiles[tcount & 1] + (size_t)TB * 16);
                for (int jj = 0; jj < tlen; ++jj) {
                    const float4 pb = s_pos[jj];
                    const int jg = jbase + jj;
#pragma unroll
                    for (int r = 0; r < R; ++r) {
                        const float dx = ax[r] - pb.x, dy = ay[r] - pb.y, dz = az[r] - pb.z;
                        const float s2 = fmaf(dz, dz, fmaf(dy, dy, dx * dx));
                        bool hit = (s2 < P.hi_cut) && (s2 > P.lo_cut);
                        if (it.self) hit = hit && (jg > ai[r]);
                        if (!hit) continue;
                        float4 ab = make_float4(0.f, 0.f, 0.f, 0.f);
                        if (kNeedAux) ab = s_aux[jj];
                        bool ex = (fabsf(s2 - P.max_r_sq) <= P.g_s2) || (fabsf(s2 - P.min_r_sq) <= P.g_s2);
                        bool inr = false;
                        int bin = -1;
                        if (!ex) {
                            inr = (s2 < P.max_r_sq) && (s2 > P.min_r_sq);
                            if (inr) {
                                const float inv_s = rsqrtf(s2);
                                if (MODE == MODE_MONOPOLE) {
                                    const int b1 = dev::locate(ax1, s2, dev::approx_bin(ax1, s2 * inv_s));
                                    ex = dev::near_edge(ax1, s2, b1, P.g_s2);
                                    bin = (b1 >= 0 && b1 < P.n1) ? b1 : -1;
                                } else {
                                    const float pi = 0.5f * fmaf(dz, anz[r] + ab.z,
                                                                 fmaf(dy, any_[r] + ab.y, dx * (anx[r] + ab.x)));
                                    if (MODE == MODE_S_MU) {
                                        const int b1 = dev::locate(ax1, s2, dev::approx_bin(ax1, s2 * inv_s));
                                        const float mu = fabsf(pi) * inv_s;
                                        const int b2 = dev::locate(ax2, mu, dev::approx_bin(ax2, mu));
                                        const float gmu = fmaf(P.c2_mu * inv_s, inv_s, fmaf(P.c1_mu, inv_s, P.g_mu0));
                                        ex = dev::near_edge(ax1, s2, b1, P.g_s2) || dev::near_edge(ax2, mu, b2, gmu);
                                        bin = (b1 >= 0 && b1 < P.n1 && b2 >= 0 && b2 < P.n2) ? b1 * P.n2 + b2 : -1;
                                    } else {
                                        const float a = fmaf(-pi, pi, s2);
                                        const float api = fabsf(pi);
                                        const int b2 = dev::locate(ax2, api, dev::approx_bin(ax2, api));
                                        ex = dev::near_edge(ax2, api, b2, P.g_pi);
                                        int b1 = -1;
                                        if (a <= P.g_a) {
                                            ex = ex || (a >= -P.g_a);  // near zero: sqrt of a value of unknown sign
                                        } else {
                                            b1 = dev::locate(ax1, a, dev::approx_bin(ax1, a * rsqrtf(a)));
                                            ex = ex || dev::near_edge(ax1, a, b1, P.g_a);
                                        }
                                        bin = (b1 >= 0 && b1 < P.n1 && b2 >= 0 && b2 < P.n2) ? b1 * P.n2 + b2 : -1;
                                    }
                                }
                            }
                        }
                        if (ex) {
                            ++n_guard;
                            bin = exact_pair<MODE>(EA, s_t1, s_t2, P.a.idx[ai[r]], P.b.idx[jg], &inr);
                        }
                        if (inr) ++n_in;
                        if (bin < 0) continue;
                        const float w = UNITW ? 1.0f : __fmul_rn(aw[r], pb.w);
                        const long long q = UNITW ? 1LL : __float2ll_rn(__fmul_rn(w, P.wscale));
                        dev::acc_add(s_lo, s_hi, full_base + bin, q);
                        if (JK) {
                            const int ja = ajk[r], jb = __float_as_int(ab.w);
                            const int sa = aslot[r];
                            if (sa >= 0) dev::acc_add(s_lo, s_hi, sa * P.nb + bin, q);
                            else { dev::acc_add_global(P.g_sub, (size_t)ja * P.nb + bin, q); ++n_over; }
                            if (jb != ja) {
                                const int sb = s_slot[jb];
                                if (sb >= 0) dev::acc_add(s_lo, s_hi, sb * P.nb + bin, q);
                                else { dev::acc_add_global(P.g_sub, (size_t)jb * P.nb + bin, q); ++n_over; }
                            }
                        }
                    }
                }
            }
            __syncthreads();  // everyone is done with this buffer before it is refilled
            ++tcount;
        }
    }

    // ---- merge the privatised histograms
    __syncthreads();
    for (int i = tid; i < nslices * P.nb; i += NT) {
        const unsigned long long v = ((unsigned long long)s_hi[i] << 32) | s_lo[i];
        if (!v) continue;
        const int slice = i / P.nb, b = i - slice * P.nb;
        if (slice == P.ns) atomicAdd(&P.g_full[b], v);
        else {
            const int r = s_misc->slot_region[slice];
            if (r >= 0) atomicAdd(&P.g_sub[(size_t)r * P.nb + b], v);
        }
    }
    // ---- counters
    __shared__ unsigned long long red[3][NT / 32];
    unsigned long long v0 = n_in, v1 = n_guard, v2 = n_over;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        v0 += __shfl_down_sync(0xffffffffu, v0, o);
        v1 += __shfl_down_sync(0xffffffffu, v1, o);
        v2 += __shfl_down_sync(0xffffffffu, v2, o);
    }
    if ((tid & 31) == 0) {
        red[0][tid >> 5] = v0;
        red[1][tid >> 5] = v1;
        red[2][tid >> 5] = v2;
    }
    __syncthreads();
    if (tid == 0) {
        unsigned long long s0 = 0, s1 = 0, s2 = 0;
        for (int w = 0; w < NT / 32; ++w) {
            s0 += red[0][w];
            s1 += red[1][w];
            s2 += red[2][w];
        }
        atomicAdd(&P.counters[0], n_cand);
        atomicAdd(&P.counters[1], s0);
        atomicAdd(&P.counters[2], s1);
        atomicAdd(&P.counters[3], s2);
    }
}

typedef void (*KernelFn)(const KParams);

template <int MODE>
KernelFn pick_kernel(bool unitw, bool jk, bool exact) {
    if (exact) {
        if (unitw) return jk ? pair_count_kernel<MODE, true, true, true> : pair_count_kernel<MODE, true, false, true>;
        return jk ? pair_count_kernel<MODE, false, true, true> : pair_count_kernel<MODE, false, false, true>;
    }
    if (unitw) return jk ? pair_count_kernel<MODE, true, true, false> : pair_count_kernel<MODE, true, false, false>;
    return jk ? pair_count_kernel<MODE, false, true, false> : pair_count_kernel<MODE, false, false, false>;
}

KernelFn pick(int mode, bool unitw, bool jk, bool exact) {
    switch (mode) {
    case MODE_MONOPOLE: return pick_kernel<MODE_MONOPOLE>(unitw, jk, exact);
    case MODE_SIGMA_PI: return pick_kernel<MODE_SIGMA_PI>(unitw, jk, exact);
    default: return pick_kernel<MODE_S_MU>(unitw, jk, exact);
    }
}

void decode_cell(const Grid &g, int id, int c[3]) {
    if (g.morton) {
        unsigned v = (unsigned)id;
        for (int m = 0; m < 3; ++m) {
            unsigned x = (v >> m) & 0x09249249u;
            x = (x | (x >> 2)) & 0x030C30C3u;
            x = (x | (x >> 4)) & 0x0300F00Fu;
            x = (x | (x >> 8)) & 0x030000FFu;
            x = (x | (x >> 16)) & 0x3ffu;
            c[m] = (int)x;
        }
    } else {
        c[0] = id / (g.dim[1] * g.dim[2]);
        c[1] = (id / g.dim[2]) % g.dim[1];
        c[2] = id % g.dim[2];
    }
}

int encode_cell(const Grid &g, const int c[3]) {
    for (int m = 0; m < 3; ++m)
        if (c[m] < 0 || c[m] >= g.dim[m]) return -1;
    if (g.morton) {
        unsigned id = 0;
        for (int m = 0; m < 3; ++m) {
            unsigned x = (unsigned)c[m] & 0x3ffu;
            x = (x | (x << 16)) & 0x030000FFu;
            x = (x | (x << 8)) & 0x0300F00Fu;
            x = (x | (x << 4)) & 0x030C30C3u;
            x = (x | (x << 2)) & 0x09249249u;
            id |= x << m;
        }
        return (int)id;
    }
    return (c[0] * g.dim[1] + c[1]) * g.dim[2] + c[2];
}

}  // namespace

// Work list: every (chunk of A cell, B cell) pair whose cell boxes are closer
// than the maximum separation.  For an auto count a cell pair is visited
// once (B after A in cell order) and a cell with itself keeps only j > i.
void build_work_items(const Grid &ga, const Grid &gb, bool is_auto, int m, double side, double rb,
                      std::vector<WorkItem> &items) {
    std::vector<int> offs;
    for (int ox = -m; ox <= m; ++ox)
        for (int oy = -m; oy <= m; ++oy)
            for (int oz = -m; oz <= m; ++oz) {
                double g2 = 0;
                for (int o : {ox, oy, oz}) {
                    double gap = std::max(std::abs(o) - 1, 0) * side * (1.0 - 1e-12);
                    g2 += gap * gap;
                }
                if (g2 < rb * rb) {
                    offs.push_back(ox);
                    offs.push_back(oy);
                    offs.push_back(oz);
                }
            }
    items.clear();
    for (int ca = 0; ca < ga.ncell; ++ca) {
        const int a0 = ga.h_cell_start[ca], a1 = ga.h_cell_start[ca + 1];
        if (a1 == a0) continue;
        int c[3];
        decode_cell(ga, ca, c);
        for (size_t k = 0; k < offs.size(); k += 3) {
            int cbv[3];
            for (int mm = 0; mm < 3; ++mm) cbv[mm] = ga.kmin[mm] + c[mm] + offs[k + mm] - gb.kmin[mm];
            const int cb = encode_cell(gb, cbv);
            if (cb < 0) continue;
            const int b0 = gb.h_cell_start[cb], b1 = gb.h_cell_start[cb + 1];
            if (b1 == b0) continue;
            if (is_auto && cb < ca) continue;
            const bool self = is_auto && cb == ca;
            for (int s = a0; s < a1; s += TA) {
                WorkItem w;
                w.a_start = s;
                w.a_len = std::min(TA, a1 - s);
                w.a_cell = ca;
                w.b_cell = cb;
                w.self = self ? 1 : 0;
                w.a_cell_start = a0;
                if (self) {
                    // j > i: B starts at this chunk; later chunks' points follow.
                    w.b_start = s;
                    w.b_len = b1 - s;
                } else {
                    w.b_start = b0;
                    w.b_len = b1 - b0;
                }
                items.push_back(w);
            }
        }
    }
    std::stable_sort(items.begin(), items.end(), [](const WorkItem &x, const WorkItem &y) {
        return (long long)x.a_len * x.b_len > (long long)y.a_len * y.b_len;
    });
}

#define TPCF_TRY(expr)                                                                        \
    do {                                                                                      \
        cudaError_t _e = (expr);                                                              \
        if (_e != cudaSuccess) {                                                              \
            err->status = (_e == cudaErrorMemoryAllocation) ? 2 : 3;                          \
            err->msg = std::string("CUDA error in pair count: ") + cudaGetErrorString(_e);    \
            return err->status;                                                               \
        }                                                                                     \
    } while (0)

// Error bounds of the FP32 path against the reference sequence (see the
// derivation in the design notes): delta bounds |dx_fast - dx_ref| per axis.
struct Guards {
    float g_s2, g_pi, g_a, c1_mu, c2_mu, g_mu0;
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

int run_count(Ctx *ctx, const CountRequest &req, double *full_out, double *region_out, Stats *st, Error *err) {
    const Binning *bin = req.bin;
    Catalog *A = const_cast<Catalog *>(req.a);
    Catalog *B = const_cast<Catalog *>(req.b ? req.b : req.a);
    const bool is_auto = (req.b == nullptr);
    const int nb = bin->nb;
    const int n_jk = bin->n_jk;
    const bool jk = n_jk > 1;
    const double rb = bin->rmax_bound;

    int m = req.refinement > 0 ? req.refinement : ctx->refinement;
    if (m <= 0) {
        // Automatic: refine to side rb/2 when cells of that size would still
        // hold a few hundred points on average.
        double vol = 1;
        for (int k = 0; k < 3; ++k) vol *= std::max(A->hi_kept[k] - A->lo_kept[k], rb);
        const double per_cell = A->n_kept * (rb / 2) * (rb / 2) * (rb / 2) / vol;
        m = per_cell >= 256 ? 2 : 1;
    }
    const double side = rb / m * (1.0 + 1e-9);

    Grid *ga = nullptr, *gb = nullptr;
    if (build_grid(ctx, A, side, true, req.exact_fp64, &ga, err)) return err->status;
    if (is_auto) gb = ga;
    else if (build_grid(ctx, B, side, true, req.exact_fp64, &gb, err)) return err->status;

    std::vector<WorkItem> items;
    build_work_items(*ga, *gb, is_auto, m, side, rb, items);

    // Fixed-point scale: the largest pair weight stays below 2^31.
    bool unitw = A->unit_weights && B->unit_weights;
    float wscale = 1.0f;
    if (!unitw) {
        const double wmax = (double)A->w_max * (double)B->w_max * (1.0 + 1e-6);
        const double wmin_abs = 0;
        (void)wmin_abs;
        int S = (int)std::floor(30.0 - std::log2(std::max(wmax, 1e-30)));
        S = std::min(S, 100);
        wscale = (float)std::ldexp(1.0, S);
        if (!std::isfinite(wscale)) wscale = std::ldexp(1.0f, 100);
    }

    // Shared-memory budget: as many jackknife slots as fit.
    const SmemLayout l0 = smem_layout(nb, 0, bin->nb1, bin->nb2, jk ? n_jk : 0, req.exact_fp64);
    const size_t budget = ctx->smem_optin > 2048 ? ctx->smem_optin - 2048 : 0;  // static shared memory headroom
    if (l0.total > budget) {
        err->status = 6;
        err->msg = "histogram does not fit in shared memory";
        return err->status;
    }
    int ns = 0;
    if (jk) {
        const size_t per_slot = 8 * (size_t)nb;
        ns = (int)std::min<size_t>((budget - l0.total) / per_slot, kMaxSlots);
    }
    const SmemLayout L = smem_layout(nb, ns, bin->nb1, bin->nb2, jk ? n_jk : 0, req.exact_fp64);

    DevBuf<WorkItem> d_items;
    DevBuf<unsigned long long> d_full, d_sub, d_cnt;
    DevBuf<int> d_head, d_err;
    DevBuf<float> d_t1, d_t2;
    cudaStream_t stm = ctx->stream;
    TPCF_TRY(d_items.alloc(items.size()));
    TPCF_TRY(d_full.alloc(nb));
    TPCF_TRY(d_sub.alloc((size_t)nb * n_jk));
    TPCF_TRY(d_cnt.alloc(4));
    TPCF_TRY(d_head.alloc(1));
    TPCF_TRY(d_err.alloc(1));
    TPCF_TRY(d_t1.alloc(bin->t1.size()));
    TPCF_TRY(d_t2.alloc(std::max<size_t>(bin->t2.size(), 1)));
    if (!items.empty())
        TPCF_TRY(cudaMemcpyAsync(d_items.p, items.data(), sizeof(WorkItem) * items.size(), cudaMemcpyHostToDevice, stm));
    TPCF_TRY(cudaMemcpyAsync(d_t1.p, bin->t1.data(), sizeof(float) * bin->t1.size(), cudaMemcpyHostToDevice, stm));
    if (!bin->t2.empty())
        TPCF_TRY(cudaMemcpyAsync(d_t2.p, bin->t2.data(), sizeof(float) * bin->t2.size(), cudaMemcpyHostToDevice, stm));
    TPCF_TRY(cudaMemsetAsync(d_full.p, 0, sizeof(unsigned long long) * nb, stm));
    TPCF_TRY(cudaMemsetAsync(d_sub.p, 0, sizeof(unsigned long long) * nb * n_jk, stm));
    TPCF_TRY(cudaMemsetAsync(d_cnt.p, 0, sizeof(unsigned long long) * 4, stm));
    TPCF_TRY(cudaMemsetAsync(d_head.p, 0, sizeof(int), stm));
    TPCF_TRY(cudaMemsetAsync(d_err.p, 0, sizeof(int), stm));

    KParams P;
    std::memset(&P, 0, sizeof(P));
    auto fill = [&](GridK &k, const Grid &g, const Catalog &c) {
        k.pos = g.pos.p;
        k.aux = g.aux.p;
        k.idx = g.idx.p;
        k.xyz_s = g.xyz_s.p;
        k.unit_s = g.unit_s.p;
        k.coord = g.cell_coord.p;
        k.rstart = g.region_start.p;
        k.regions = g.regions.p;
        k.kmin0 = g.kmin[0];
        k.kmin1 = g.kmin[1];
        k.kmin2 = g.kmin[2];
        k.xyz = c.xyz.p;
        k.unit = c.unit.p;
    };
    fill(P.a, *ga, *A);
    fill(P.b, *gb, *B);
    P.items = d_items.p;
    P.n_items = (int)items.size();
    P.head = d_head.p;
    P.side = side;
    P.n1 = bin->nb1;
    P.n2 = bin->mode == MODE_MONOPOLE ? 0 : bin->nb2;
    P.nb = nb;
    P.min_r_sq = bin->min_r_sq;
    P.max_r_sq = bin->max_r_sq;
    const Guards g = compute_guards(side, m, rb);
    P.g_s2 = g.g_s2;
    P.g_pi = g.g_pi;
    P.g_a = g.g_a;
    P.c1_mu = g.c1_mu;
    P.c2_mu = g.c2_mu;
    P.g_mu0 = g.g_mu0;
    P.lo_cut = bin->min_r_sq - g.g_s2;
    P.hi_cut = bin->max_r_sq + g.g_s2;
    P.t1g = d_t1.p;
    P.t2g = d_t2.p;
    P.ax1_log = bin->ax1.log_binning;
    P.ax1_min = bin->ax1.min;
    P.ax1_inv_step = bin->ax1.inv_step;
    P.ax1_ilb = bin->ax1.inv_log_of_base;
    P.ax1_ils = bin->ax1.inv_log_step;
    P.ax2_log = bin->ax2.log_binning;
    P.ax2_min = bin->ax2.min;
    P.ax2_inv_step = bin->ax2.inv_step;
    P.ax2_ilb = bin->ax2.inv_log_of_base;
    P.ax2_ils = bin->ax2.inv_log_step;
    P.g_full = d_full.p;
    P.g_sub = d_sub.p;
    P.n_jk = n_jk;
    P.ns = ns;
    P.wscale = wscale;
    P.counters = d_cnt.p;
    P.err = d_err.p;

    KernelFn fn = pick(bin->mode, unitw, jk, req.exact_fp64);
    TPCF_TRY(cudaFuncSetAttribute((const void *)fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)L.total));
    cudaEvent_t e0, e1;
    TPCF_TRY(cudaEventCreate(&e0));
    TPCF_TRY(cudaEventCreate(&e1));
    TPCF_TRY(cudaEventRecord(e0, stm));
    if (!items.empty()) {
        const int grid = std::min<int>(ctx->num_sms, (int)items.size());
        fn<<<grid, NT, L.total, stm>>>(P);
        TPCF_TRY(cudaGetLastError());
    }
    TPCF_TRY(cudaEventRecord(e1, stm));
    std::vector<unsigned long long> hf(nb), hs((size_t)nb * n_jk), hc(4);
    int herr = 0;
    TPCF_TRY(cudaMemcpyAsync(hf.data(), d_full.p, sizeof(unsigned long long) * nb, cudaMemcpyDeviceToHost, stm));
    TPCF_TRY(cudaMemcpyAsync(hs.data(), d_sub.p, sizeof(unsigned long long) * hs.size(), cudaMemcpyDeviceToHost, stm));
    TPCF_TRY(cudaMemcpyAsync(hc.data(), d_cnt.p, sizeof(unsigned long long) * 4, cudaMemcpyDeviceToHost, stm));
    TPCF_TRY(cudaMemcpyAsync(&herr, d_err.p, sizeof(int), cudaMemcpyDeviceToHost, stm));
    TPCF_TRY(cudaStreamSynchronize(stm));
    float ms = 0;
    cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (herr) {
        err->status = 4;
        err->msg = "device wait exceeded its iteration limit; results discarded";
        return err->status;
    }
    const double inv = unitw ? 1.0 : 1.0 / (double)wscale;
    for (int b = 0; b < nb; ++b) full_out[b] = (double)(long long)hf[b] * inv;
    if (region_out) {
        if (jk)
            for (size_t k = 0; k < hs.size(); ++k) region_out[k] = (double)(long long)hs[k] * inv;
        else
            for (int b = 0; b < nb; ++b) region_out[b] = full_out[b];
    }
    if (st) {
        st->candidates += hc[0];
        st->in_range += hc[1];
        st->guard += hc[2];
        st->overflow += hc[3];
        st->items += items.size();
        st->ms_kernel += ms;
    }
    return 0;
}

}  // namespace tpcf
