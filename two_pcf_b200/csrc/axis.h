// Host replica of the reference's histogram axis and the float threshold
// tables that the CUDA kernels bin with.
#pragma once
#include <vector>

namespace tpcf {

// Field-for-field replica of Axis (src/hist.h:5-19, src/hist.cpp:15-36).
struct AxisParams {
    int n_bins = 0;
    bool log_binning = false;
    float min = 0, minus_min = 0, max = 0, step = 0, inv_step = 0, base = 0, inv_log_of_base = 0, inv_log_step = 0;
};

// Axis(float min, float max, int n, float base): the arguments are the
// parameter-file doubles narrowed to float at the call, as in the reference.
AxisParams make_axis(double min, double max, int n_bins, double log_base);

// Axis::bin_num (src/hist.cpp:46-53), evaluated with the host's libm.
float axis_bin_num(const AxisParams &ax, float value);

// (int) of a float as x86-64 cvttss2si does it: truncation toward zero,
// INT_MIN for NaN and out-of-range values.
int to_bin(float f);

// Axis::value_from_bin / bin_centre / bin_width (src/hist.cpp:38-62).
double axis_value_from_bin(const AxisParams &ax, double b);
double axis_bin_centre(const AxisParams &ax, int b);
double axis_bin_width(const AxisParams &ax, int b);

// Which float the reference bins on, as a function of the value the kernel
// has at hand: the value itself, or sqrtf of it (s from s^2, sigma from
// s^2 - pi^2).
enum class ValueSpace { Direct, Sqrt };

// Threshold table T[0..n] over the domain [lo, hi] of values the kernels can
// meet: T[k] is the smallest float x in [lo, hi] with
// to_bin(bin_num(f(x))) >= k, or +inf when there is none.  For every float x
// in the domain: bin = #{k : T[k] <= x} - 1, and the pair is binned when
// 0 <= bin < n.  Requires bin_num(f(x)) to be non-decreasing on the domain
// (outside it the reference's float-to-int conversion wraps to INT_MIN), which
// check_monotone() verifies.
std::vector<float> build_thresholds(const AxisParams &ax, ValueSpace vs, float lo, float hi);

// The reference's bin for a non-negative float x (with the value space
// applied), used by the exact path on the host and by the tests.
int reference_bin(const AxisParams &ax, ValueSpace vs, float x);

// Returns false if bin_num(f(x)) decreases anywhere on a dense sample of
// [0, hi] (every float in the neighbourhood of each threshold plus a strided
// sweep).
bool check_monotone(const AxisParams &ax, ValueSpace vs, float lo, float hi);

}  // namespace tpcf
