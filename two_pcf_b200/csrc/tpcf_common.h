// Shared host/device definitions of the pair-counting engine.
#pragma once
#include <cstdint>

#ifdef __CUDACC__
#define TPCF_HD __host__ __device__
#else
#define TPCF_HD
#endif

namespace tpcf {

enum Mode { MODE_MONOPOLE = 0, MODE_SIGMA_PI = 1, MODE_S_MU = 2, MODE_ANGULAR = 3 };

// How a pair's weight is formed (src/correlators.cpp:40 for PLAIN;
// src/correlators_invpweight.cpp:51-77 for INVP_DD, :184-189 for INVP_DR,
// :743-764 / :853 / :901 / :968 for the angular kinds).
enum WeightKind {
    W_UNIT = 0,       // every weight is 1.0: integer counts
    W_PLAIN = 1,      // w1 * w2 (float product)
    W_INVP_DD = 2,    // iw1 * iw2 * (float)(interp(1-cos) * n_runs / popc)
    W_INVP_DR = 3,    // (float)((w1 * w2) * interp(1-cos))
    W_ANG_INPUT = 4,  // iw1 * iw2 (angular DD/DR: input weights)
    W_ANG_INVP = 5,   // iw1 * iw2 * (n_runs / popc)  (angular DD inverse-p)
    W_ADJ = 6,        // adjoint of a w1 * w2 count: per-point dL/dw instead of a histogram
};

// Histogram bins are decided by comparing a float value with a float
// threshold table: bin(v) = #{k : T[k] <= v} - 1, valid when 0 <= bin < n.
// The tables come from the host (axis.cpp), which evaluates the reference's
// own Axis::bin_num on the host's libm.
constexpr int kMaxBins1D = 256;      // per axis
constexpr int kMaxBinsTotal = 8192;  // per histogram
constexpr int kMaxMaskInts = 32;     // 64-bit masks per object for inverse-p weights
constexpr int kMaxRegions = 4096;    // jackknife regions
constexpr int kChunkA = 1024;        // A points per work item (256 threads x 4)
constexpr long long kItemMaxB = 16384;  // B points per work item (load balance)

// One unit of device work: a chunk of one (cell, jackknife region) run of
// catalogue A against a list of runs of catalogue B (its segments) from the
// neighbouring cells, sorted by region.  All A points of an item share one
// region and all points of a segment share one region, so each segment's
// pair histogram is added once to the row of its region and the item's total
// once to the full histogram and to the row of the A region.
struct WorkItem {
    int a_start;    // first point of the A chunk (sorted order, grid A)
    int a_len;
    int a_cell;     // dense cell index in grid A
    int a_region;   // jackknife region of every A point of the item
    int seg_begin;  // segments [seg_begin, seg_end) in the segment array
    int seg_end;
    int job;     // which (catalogue A, catalogue B, output) of a batched launch
    int pad;
};

struct Segment {
    int b_start;  // first point of the B run (sorted order, grid B)
    int b_len;
    int b_cell;   // dense cell index in grid B
    int meta;     // region of the run | (1 << 16) when it is the A run itself (auto count: only j > i)
};

}  // namespace tpcf
