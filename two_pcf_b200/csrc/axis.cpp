// Host replica of the reference Axis and the threshold tables used for
// binning on the GPU.  Compiled with -ffp-contract=off so every float and
// double operation rounds once, as in the reference's x86-64 build.
#include "axis.h"

#include <cmath>
#include <cstdint>
#include <cstring>
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

}  // namespace tpcf
