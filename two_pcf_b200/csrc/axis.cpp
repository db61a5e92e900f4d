// Host replica of the reference Axis and the threshold tables used for
// binning on the GPU.  Compiled with -ffp-contract=off so every float and
// double operation rounds once, as in the reference's x86-64 build.
#include "axis.h"

#include "engine.h"

#include <cmath>
#include <cstdint>
#include <cstring>
#include <algorithm>
#include <limits>

namespace tpcf {

AxisParams make_axis(double input_min_d, double input_max_d, int n_bins, double log_base_d) {
    // src/hist.cpp:15-36.  The constructor parameters are float.
    const float input_min = (float)input_min_d, input_max = (float)input_max_d, log_base = (float)log_base_d;
    AxisParams ax;
    ax.min = input_min;
    ax.minus_min = -input_min;
    ax.max = input_max;
    ax.n_bins = n_bins;
    ax.step = (ax.max - ax.min) / (float)n_bins;
    ax.inv_step = (float)(1.0 / (double)ax.step);
    ax.base = log_base;
    if ((double)ax.base > 1.02) {
        // log(float) is logf; pow(float, int) promotes both to double.
        ax.inv_log_of_base = (float)(1.0 / (double)::logf(log_base));
        ax.inv_log_step = (float)((std::pow((double)log_base, (double)n_bins) - 1) / (double)(input_max - input_min));
        ax.log_binning = true;
    } else {
        ax.inv_log_of_base = 0.0f;
        ax.inv_log_step = 0.0f;
        ax.log_binning = false;
    }
    return ax;
}

float axis_bin_num(const AxisParams &ax, float value) {
    if (ax.log_binning) return ax.inv_log_of_base * ::log1pf(ax.inv_log_step * (value - ax.min));
    return (value + ax.minus_min) * ax.inv_step;
}

int to_bin(float f) {
    if (!(f > -2147483648.0f && f < 2147483648.0f)) return INT32_MIN;
    return (int)f;
}

double axis_value_from_bin(const AxisParams &ax, double b) {
    if (ax.log_binning) return (std::exp(b / ax.inv_log_of_base) - 1.0) / ax.inv_log_step + ax.min;
    return ax.min + b * ax.step;
}

double axis_bin_centre(const AxisParams &ax, int b) {
    return (axis_value_from_bin(ax, b + 1.0) + axis_value_from_bin(ax, b)) / 2.0;
}

double axis_bin_width(const AxisParams &ax, int b) {
    return axis_value_from_bin(ax, b + 1.0) - axis_value_from_bin(ax, b);
}

namespace {

inline float from_bits(uint32_t u) {
    float f;
    std::memcpy(&f, &u, 4);
    return f;
}

inline uint32_t to_bits(float f) {
    uint32_t u;
    std::memcpy(&u, &f, 4);
    return u;
}

inline float apply_space(ValueSpace vs, float x) { return vs == ValueSpace::Sqrt ? ::sqrtf(x) : x; }

}  // namespace

int reference_bin(const AxisParams &ax, ValueSpace vs, float x) {
    return to_bin(axis_bin_num(ax, apply_space(vs, x)));
}

namespace {
// Order-preserving map of floats to unsigned keys (negative floats below
// positive ones, -0 just below +0).
inline uint32_t key_of(float f) {
    uint32_t u = to_bits(f);
    return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
inline float float_of(uint32_t k) { return from_bits((k & 0x80000000u) ? (k & 0x7fffffffu) : ~k); }
}  // namespace

std::vector<float> build_thresholds(const AxisParams &ax, ValueSpace vs, float lo, float hi) {
    std::vector<float> t(ax.n_bins + 1);
    const uint32_t klo = key_of(lo), khi = key_of(hi);
    for (int k = 0; k <= ax.n_bins; ++k) {
        if (reference_bin(ax, vs, lo) >= k) {
            t[k] = lo;
            continue;
        }
        if (reference_bin(ax, vs, hi) < k) {
            t[k] = std::numeric_limits<float>::infinity();
            continue;
        }
        uint32_t a = klo, b = khi;  // P(a) false, P(b) true
        while (b - a > 1) {
            const uint32_t mid = a + (b - a) / 2;
            if (reference_bin(ax, vs, float_of(mid)) >= k) b = mid;
            else a = mid;
        }
        t[k] = float_of(b);
    }
    return t;
}

bool check_monotone(const AxisParams &ax, ValueSpace vs, float lo, float hi) {
    const uint32_t klo = key_of(lo), khi = key_of(hi);
    std::vector<float> t = build_thresholds(ax, vs, lo, hi);
    // Every float within 4096 ulps of each finite threshold.
    for (float tk : t) {
        if (!std::isfinite(tk)) continue;
        const uint32_t kb = key_of(tk);
        const uint32_t a = kb - klo > 4096 ? kb - 4096 : klo;
        const uint32_t b = khi - kb > 4096 ? kb + 4096 : khi;
        int prev = reference_bin(ax, vs, float_of(a));
        for (uint32_t u = a + 1; u <= b; ++u) {
            const int cur = reference_bin(ax, vs, float_of(u));
            if (cur < prev) return false;
            prev = cur;
        }
    }
    // Strided sweep of the domain.
    int prev = reference_bin(ax, vs, lo);
    for (uint64_t u = klo; u <= khi; u += 97) {
        const int cur = reference_bin(ax, vs, float_of((uint32_t)u));
        if (cur < prev) return false;
        prev = cur;
    }
    return true;
}

namespace {

// Interval of JKHists::interp (src/hist.cpp:369-391) for a float argument x
// in [min, max]: bin_num = (float)(Axis::bin_num(x) - 0.5); -1 when it is
// negative, n when it exceeds n - 1, else (int)bin_num.
int up_category(const AxisParams &ax, float x) {
    const float bn = (float)((double)axis_bin_num(ax, x) - 0.5);
    if (bn < 0) return -1;
    if (bn > ax.n_bins - 1) return ax.n_bins;
    return (int)bn;
}

}  // namespace

UpTable make_up_table(const AxisParams &ax, const double *num, const double *den) {
    UpTable t;
    t.ax = ax;
    const int n = ax.n_bins;
    t.bins.resize(n + 1);
    t.centre.resize(n + 1);
    for (int b = 0; b < n; ++b) t.bins[b] = num[b] / den[b];
    // The reference reads bins[n] when (int)bin_num == n - 1 exactly (one
    // past its array); the table repeats the last bin there.
    t.bins[n] = t.bins[n - 1];
    for (int b = 0; b <= n; ++b) t.centre[b] = axis_bin_centre(ax, b);
    t.abs_max = 0;
    for (int b = 0; b < n; ++b)
        if (std::isfinite(t.bins[b])) t.abs_max = std::max(t.abs_max, std::fabs(t.bins[b]));
    // Thresholds: thr[k] = smallest float x in [min, max] with category >= k,
    // +inf when none; the category of x is #{k : thr[k] <= x} - 1.  The
    // category is non-decreasing in x because bin_num is (check_monotone).
    t.thr.assign(n + 1, std::numeric_limits<float>::infinity());
    const float lo = ax.min, hi = ax.max;
    const uint32_t klo = key_of(lo), khi = key_of(hi);
    for (int k = 0; k <= n; ++k) {
        if (up_category(ax, lo) >= k) {
            t.thr[k] = lo;
            continue;
        }
        if (up_category(ax, hi) < k) continue;
        uint32_t a = klo, b = khi;
        while (b - a > 1) {
            const uint32_t mid = a + (b - a) / 2;
            if (up_category(ax, float_of(mid)) >= k) b = mid;
            else a = mid;
        }
        t.thr[k] = float_of(b);
    }
    return t;
}

double up_eval(const UpTable &t, double v) {
    const int n = t.ax.n_bins;
    if (v < (double)t.ax.min) return t.bins[0];
    if (v > (double)t.ax.max) return t.bins[n - 1];
    const float x = (float)v;
    int c = -1;
    for (int k = 0; k <= n; ++k)
        if (t.thr[k] <= x) c = k;
    if (c < 0) return t.bins[0];
    if (c >= n) return t.bins[n - 1];
    return t.bins[c] + (t.bins[c + 1] - t.bins[c]) * (v - t.centre[c]) / (t.centre[c + 1] - t.centre[c]);
}

}  // namespace tpcf
