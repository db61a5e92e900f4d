// The reference's program on a parameter file (src/main.cpp:11-84, plain
// build), with the pair counts on the device: tpcf_run_param_file.
#include <chrono>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#ifdef _OPENMP
#include <omp.h>
#endif

#include "capi_types.h"
#include "ingest.h"

namespace {

struct Log {
    int level;
    std::chrono::steady_clock::time_point t0 = std::chrono::steady_clock::now();
    void operator()(const char *fmt, ...) const {
        if (!level) return;
        double s = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        std::fprintf(stderr, "[two_pcf %8.3f s] ", s);
        va_list ap;
        va_start(ap, fmt);
        std::vfprintf(stderr, fmt, ap);
        va_end(ap);
        std::fputc('\n', stderr);
    }
};

struct Err {
    int status = TPCF_OK;
    std::string msg;
    bool set(int st, const std::string &m) {
        status = st;
        msg = m;
        return false;
    }
};

// A double for the JSON run summary: non-finite values as null.
std::string jnum(double v) {
    if (!std::isfinite(v)) return "null";
    char b[40];
    std::snprintf(b, sizeof b, "%.17g", v);
    return b;
}

std::string jstr(const std::string &v) {
    std::string o = "\"";
    for (char ch : v) {
        if (ch == '"' || ch == '\\') o += '\\';
        if ((unsigned char)ch < 0x20) {
            char b[8];
            std::snprintf(b, sizeof b, "\\u%04x", (unsigned)ch);
            o += b;
            continue;
        }
        o += ch;
    }
    return o + "\"";
}

// Largest difference of one output against the same output of the FP64
// path, over every bin of the full histogram and of every region's slice:
// relative |a - b| / |b| (bins where b is zero and a is not count as an
// infinite relative error), absolute |a - b|, and whether every value agrees
// bit for bit.  A NaN on both sides agrees; a non-finite value on one side
// only is counted as a mismatch.
struct ErrStat {
    double max_rel = 0.0, max_abs = 0.0;
    long long values = 0, nonfinite_mismatch = 0;
    bool identical = true;
    void add(const double *a, const double *b, size_t n) {
        for (size_t i = 0; i < n; ++i) {
            ++values;
            if (std::memcmp(&a[i], &b[i], sizeof(double)) != 0) identical = false;
            if (std::isnan(a[i]) && std::isnan(b[i])) continue;
            if (a[i] == b[i]) continue;
            if (!std::isfinite(a[i]) || !std::isfinite(b[i])) {
                ++nonfinite_mismatch;
                continue;
            }
            const double d = std::fabs(a[i] - b[i]);
            max_abs = std::max(max_abs, d);
            max_rel = std::max(max_rel, b[i] != 0.0 ? d / std::fabs(b[i]) : INFINITY);
        }
    }
    std::string json() const {
        return "{\"max_rel_err\": " + (std::isinf(max_rel) ? std::string("\"inf\"") : jnum(max_rel)) +
               ", \"max_abs_err\": " + jnum(max_abs) + ", \"values\": " + std::to_string(values) +
               ", \"nonfinite_mismatch\": " + std::to_string(nonfinite_mismatch) +
               ", \"bit_identical\": " + (identical ? "true" : "false") + "}";
    }
};

// What tpcf_run_param_file_report collects for its JSON run summary.
struct Report {
    bool check_fp64 = false;
    std::vector<std::string> modes;  // one JSON object per correlated mode
    double kernel_ms = 0.0, pairs = 0.0;
    long long n_data_read = 0, n_rand_read = 0, n_data_kept = 0, n_rand_kept = 0;
};

struct CtxDel {
    void operator()(tpcf_ctx *c) const { tpcf_destroy(c); }
};
struct CatDel {
    void operator()(tpcf_catalog *c) const { tpcf_catalog_destroy(c); }
};
struct BinDel {
    void operator()(tpcf_binning *b) const { tpcf_binning_destroy(b); }
};
using CtxPtr = std::unique_ptr<tpcf_ctx, CtxDel>;
using CatPtr = std::unique_ptr<tpcf_catalog, CatDel>;
using BinPtr = std::unique_ptr<tpcf_binning, BinDel>;

// read_file (src/io.cpp:597-626) for the file types this build reads.
bool read_catalogue(const tpcf::Params &p, const std::string &name, const std::string &type,
                    const tpcf::CosmologyTable *cosmo, tpcf::HostCatalogue &out, Err &e) {
    if (type == "hdf5")
        return e.set(TPCF_E_UNSUPPORTED, name + ": HDF5 catalogues need the HDF5 library, which this build lacks");
    if (type != "ascii") return e.set(TPCF_E_INVALID_ARG, "unknown file type '" + type + "' for " + name);
    tpcf::Coords c;
    if (p.coord_system == "cartesian") c = tpcf::Coords::Cartesian;
    else if (p.coord_system == "equatorial") c = tpcf::Coords::Equatorial;
    else return e.set(TPCF_E_INVALID_ARG, "unknown coord_system '" + p.coord_system + "'");
    std::string err;
    if (!tpcf::read_ascii(name, c, p.use_weights, p.n_jk_regions, cosmo, out, err))
        return e.set(TPCF_E_INVALID_ARG, err);
    return true;
}

bool upload(tpcf_ctx *ctx, const tpcf::HostCatalogue &h, int n_jk, CatPtr &out, Err &e) {
    tpcf_catalog *c = nullptr;
    int rc = tpcf_catalog_create(ctx, h.size(), h.xyz.data(), h.x_norm.data(), h.d_comov.data(), h.weight.data(),
                                 nullptr, n_jk > 1 ? h.jk_region.data() : nullptr, n_jk, nullptr, 0, &c);
    if (rc) return e.set(rc, std::string("catalogue upload: ") + tpcf_last_error(ctx));
    out.reset(c);
    return true;
}

// One auto_correlate_* (src/correlators.cpp:127-153, :280-307, :432-459), or
// with weight specs auto_correlate_*_invpweights
// (src/correlators_invpweight.cpp:210-237, :445-474, :682-711): DD, DR, RR in
// the reference's convention (jackknife-inverted, auto counts doubled), each
// normalised, then the ASCII outputs.  RR is always a plain count.
//
// With a report, the mode's counts go into the run summary; with
// report->check_fp64 the same three counts run again on the plain FP64 path
// and each output (raw DD, DR, RR; normalised DD, DR, RR; xi; full histogram
// and every region's slice) is compared with its FP64 counterpart.
bool correlate(tpcf_ctx *ctx, const char *what, int mode, const tpcf_axis_spec &a1, const tpcf_axis_spec *a2,
               int n_jk, const tpcf_catalog *data, const tpcf_catalog *rand, int precision,
               const std::string &filename, const std::string &output_type, const tpcf_weight_spec *dd_spec,
               const tpcf_weight_spec *dr_spec, const Log &log, Err &e, Report *report) {
    if (output_type == "hdf5")
        return e.set(TPCF_E_UNSUPPORTED, std::string(what) + ": HDF5 output needs the HDF5 library, which this build lacks");
    if (output_type != "ascii")
        return e.set(TPCF_E_INVALID_ARG, std::string(what) + ": unknown output type '" + output_type + "'");
    tpcf_binning *b = nullptr;
    int rc = tpcf_binning_create(ctx, mode, &a1, a2, n_jk, &b);
    if (rc) return e.set(rc, std::string(what) + " binning: " + tpcf_last_error(ctx));
    BinPtr bin(b);
    const int nb = tpcf_binning_total_bins(b);
    std::vector<double> full[3], sub[3];
    for (int k = 0; k < 3; ++k) {
        full[k].assign(nb, 0.0);
        sub[k].assign((size_t)n_jk * nb, 0.0);
    }
    tpcf_stats st[3];
    // DD, DR and RR in one call: each count's host planning overlaps the
    // previous count's kernel
    log("%s: DD, DR, RR", what);
    const tpcf_catalog *ja[3] = {data, data, rand}, *jb[3] = {nullptr, rand, nullptr};
    const tpcf_weight_spec *js[3] = {dd_spec, dr_spec, nullptr};
    // DD, DR, RR on one path, in the reference's convention, then normalised
    auto count3 = [&](int prec, std::vector<double> *f, std::vector<double> *r, tpcf_stats *s,
                      std::vector<double> *raw_f, std::vector<double> *raw_r) -> int {
        tpcf_count_job jobs[3];
        for (int k = 0; k < 3; ++k) {
            jobs[k].a = ja[k];
            jobs[k].b = jb[k];
            jobs[k].bin = b;
            jobs[k].spec = js[k];
            jobs[k].precision = prec;
            jobs[k].reference_form = 1;
            jobs[k].full_out = f[k].data();
            jobs[k].region_out = r[k].data();
            jobs[k].stats = &s[k];
        }
        int c = tpcf_count_many(ctx, jobs, 3);
        if (!c && raw_f)
            for (int k = 0; k < 3; ++k) {
                raw_f[k] = f[k];
                raw_r[k] = r[k];
            }
        if (!c) c = tpcf_normalise_auto(data, nb, f[0].data(), r[0].data());
        if (!c) c = tpcf_normalise_cross(data, rand, nb, f[1].data(), r[1].data());
        if (!c) c = tpcf_normalise_auto(rand, nb, f[2].data(), r[2].data());
        return c;
    };
    const bool check = report && report->check_fp64 && precision != TPCF_FP64;
    std::vector<double> raw_full[3], raw_sub[3];
    rc = count3(precision, full, sub, st, check ? raw_full : nullptr, check ? raw_sub : nullptr);
    if (rc) return e.set(rc, std::string(what) + ": " + tpcf_last_error(ctx));
    log("%s: %.3e + %.3e + %.3e pairs in range, kernels %.1f + %.1f + %.1f ms", what, (double)st[0].in_range,
        (double)st[1].in_range, (double)st[2].in_range, st[0].ms_kernel, st[1].ms_kernel, st[2].ms_kernel);
    rc = tpcf_write_xi_ascii(filename.c_str(), b, full[0].data(), full[1].data(), full[2].data(), sub[0].data(),
                             sub[1].data(), sub[2].data());
    if (rc) return e.set(rc, std::string(what) + ": " + tpcf_host_last_error());
    log("%s: wrote %s and %d region files", what, filename.c_str(), n_jk);
    if (!report) return true;

    const char *lab[3] = {"DD", "DR", "RR"};
    std::string j = "{\"mode\": " + jstr(what) + ", \"bins\": " + std::to_string(nb) +
                    ", \"n_jk_regions\": " + std::to_string(n_jk) + ", \"output\": " + jstr(filename) +
                    ", \"counts\": {";
    for (int k = 0; k < 3; ++k) {
        const double sec = st[k].ms_kernel * 1e-3;
        j += std::string(k ? ", " : "") + "\"" + lab[k] + "\": {\"in_range_pairs\": " +
             std::to_string(st[k].in_range) + ", \"candidates\": " + std::to_string(st[k].candidates) +
             ", \"guard_evals\": " + std::to_string(st[k].guard_evals) + ", \"kernel_ms\": " +
             jnum(st[k].ms_kernel) + ", \"pairs_per_s\": " + jnum(sec > 0 ? st[k].in_range / sec : NAN) + "}";
        report->kernel_ms += st[k].ms_kernel;
        report->pairs += (double)st[k].in_range;
    }
    j += "}";
    if (check) {
        // the FP64 path on the same counts
        std::vector<double> f64[3], s64[3], rf64[3], rs64[3];
        for (int k = 0; k < 3; ++k) {
            f64[k].assign(nb, 0.0);
            s64[k].assign((size_t)n_jk * nb, 0.0);
        }
        tpcf_stats st64[3];
        log("%s: DD, DR, RR on the FP64 path for the check", what);
        rc = count3(TPCF_FP64, f64, s64, st64, rf64, rs64);
        if (rc) return e.set(rc, std::string(what) + " (FP64 check): " + tpcf_last_error(ctx));
        j += ", \"fp64_check\": {";
        for (int k = 0; k < 3; ++k) {
            ErrStat raw, norm;
            raw.add(raw_full[k].data(), rf64[k].data(), nb);
            raw.add(raw_sub[k].data(), rs64[k].data(), raw_sub[k].size());
            norm.add(full[k].data(), f64[k].data(), nb);
            norm.add(sub[k].data(), s64[k].data(), sub[k].size());
            j += std::string(k ? ", " : "") + "\"" + lab[k] + "\": " + norm.json() + ", \"" + lab[k] +
                 "_raw\": " + raw.json();
        }
        // xi of the full sample and of every region's slice
        auto xi_of = [&](const std::vector<double> *f, const std::vector<double> *r) {
            std::vector<double> x((size_t)(1 + n_jk) * nb);
            for (int i = 0; i < nb; ++i) x[i] = tpcf_ls_estimator(f[0][i], f[1][i], f[2][i]);
            for (size_t i = 0; i < r[0].size(); ++i) x[nb + i] = tpcf_ls_estimator(r[0][i], r[1][i], r[2][i]);
            return x;
        };
        const std::vector<double> x32 = xi_of(full, sub), x64 = xi_of(f64, s64);
        ErrStat xe;
        xe.add(x32.data(), x64.data(), x32.size());
        double k64 = 0.0;
        for (int k = 0; k < 3; ++k) k64 += st64[k].ms_kernel;
        j += ", \"xi\": " + xe.json() + ", \"fp64_kernel_ms\": " + jnum(k64) + "}";
        log("%s: against the FP64 path, xi max relative error %.3g (bit identical: %s)", what, xe.max_rel,
            xe.identical ? "yes" : "no");
    }
    report->modes.push_back(j + "}");
    return true;
}

// The plot_monopole / plot_sigma_pi / plot_s_mu sequence of main
// (src/main.cpp:53-70) with the given DD and DR weightings.
bool correlate_modes(tpcf_ctx *c, const tpcf::Params &p, const tpcf_catalog *data, const tpcf_catalog *rand,
                     int precision, const tpcf_weight_spec *dd, const tpcf_weight_spec *dr, const Log &log, Err &e,
                     Report *report = nullptr) {
    if (p.plot_monopole) {
        tpcf_axis_spec a{p.monopole_min, p.monopole_max, p.monopole_log_base, p.monopole_n_bins};
        if (!correlate(c, "monopole", TPCF_MONOPOLE, a, nullptr, p.n_jk_regions, data, rand, precision,
                       p.monopole_filename, p.monopole_output_type, dd, dr, log, e, report))
            return false;
    }
    if (p.plot_sigma_pi) {
        tpcf_axis_spec a{p.sigma_min, p.sigma_max, p.sigma_log_base, p.sigma_n_bins};
        tpcf_axis_spec b{p.pi_min, p.pi_max, p.pi_log_base, p.pi_n_bins};
        if (!correlate(c, "sigma-pi", TPCF_SIGMA_PI, a, &b, p.n_jk_regions, data, rand, precision,
                       p.sigma_pi_filename, p.sigma_pi_output_type, dd, dr, log, e, report))
            return false;
    }
    if (p.plot_s_mu) {
        tpcf_axis_spec a{p.s_min, p.s_max, p.s_log_base, p.s_n_bins};
        tpcf_axis_spec b{0.0, 1.0, 0.0, p.mu_n_bins};
        if (!correlate(c, "s-mu", TPCF_S_MU, a, &b, p.n_jk_regions, data, rand, precision, p.s_mu_filename,
                       p.s_mu_output_type, dd, dr, log, e, report))
            return false;
    }
    return true;
}

// The inverse-p program after reading (src/main.cpp:51-60).  The angular
// stage of calc_angular_upweight (src/correlators_invpweight.cpp:985-1033)
// runs on the device and its four histograms stay in memory: the 3-D stage
// takes DD / DD-inverse-p and DR / DR-inverse-p as the up-weight ratios that
// the reference reads back from its HDF5 files (read_hdf5_hist +
// divide_by_hist, :20-24).
bool run_invp(tpcf_ctx *c, const tpcf::Params &p, const tpcf_catalog *data, const tpcf_catalog *rand,
              int precision, bool dither, double *angular_out, const Log &log, Err &e) {
    const int nt = p.theta_n_bins, n_jk = p.n_jk_regions;
    // Hist(0.0, 1.0 - cos(theta_max), theta_n_bins, theta_log_base) (:990-991)
    const tpcf_axis_spec th{0.0, 1.0 - std::cos(p.theta_max), p.theta_log_base, nt};
    tpcf_binning *b = nullptr;
    int rc = tpcf_binning_create(c, TPCF_ANGULAR, &th, nullptr, n_jk, &b);
    if (rc) return e.set(rc, std::string("angular binning: ") + tpcf_last_error(c));
    BinPtr bin(b);
    // kind 0 DD (plain, every point), 1 DD inverse-p, 2 DR, 3 DR inverse-p
    std::vector<double> ang[4];
    const char *names[4] = {"angular DD", "angular DD inverse-p", "angular DR", "angular DR inverse-p"};
    for (int k = 0; k < 4; ++k) {
        ang[k].assign((size_t)(1 + n_jk) * nt, 0.0);
        tpcf_weight_spec ws{};
        ws.weighting = k == 1 ? (dither ? TPCF_WEIGHTS_INVP_DD_DITHER : TPCF_WEIGHTS_INVP_DD)
                     : k == 3 ? TPCF_WEIGHTS_INVP_DR : TPCF_WEIGHTS_PLAIN;
        ws.n_bitwise_runs = p.n_bitwise_runs;
        tpcf_stats st;
        rc = tpcf_pair_count_weighted(c, data, k < 2 ? nullptr : rand, b, &ws, precision, ang[k].data(),
                                      ang[k].data() + nt, &st);
        if (rc) return e.set(rc, std::string(names[k]) + ": " + tpcf_last_error(c));
        log("%s: %.3e pairs binned, kernel %.1f ms", names[k], (double)st.in_range, st.ms_kernel);
        if (angular_out) std::copy(ang[k].begin(), ang[k].end(), angular_out + (size_t)k * (1 + n_jk) * nt);
    }
    tpcf_weight_spec dd{}, dr{};
    dd.weighting = dither ? TPCF_WEIGHTS_INVP_DD_DITHER : TPCF_WEIGHTS_INVP_DD;
    dd.n_bitwise_runs = p.n_bitwise_runs;
    dd.theta_axis = th;
    dd.up_numerator = ang[0].data();
    dd.up_denominator = ang[1].data();
    dr.weighting = TPCF_WEIGHTS_INVP_DR;
    dr.n_bitwise_runs = p.n_bitwise_runs;
    dr.theta_axis = th;
    dr.up_numerator = ang[2].data();
    dr.up_denominator = ang[3].data();
    return correlate_modes(c, p, data, rand, precision, &dd, &dr, log, e);
}

bool run(const char *path, int device, int precision, const Log &log, Err &e, Report *report) {
    tpcf::Params p;
    std::string err;
    if (!tpcf::load_params(path, p, err)) return e.set(TPCF_E_INVALID_ARG, err);
#ifdef _OPENMP
    if (p.n_threads > 0) omp_set_num_threads(p.n_threads);
#endif
    std::unique_ptr<tpcf::CosmologyTable> cosmo;
    if (p.coord_system == "equatorial") {
        cosmo.reset(new tpcf::CosmologyTable());
        if (!tpcf::make_cosmology(p.omega_m, p.h, p.z_min, p.z_max, 0.0001, 100, *cosmo, err))
            return e.set(TPCF_E_INVALID_ARG, err);
    }
    tpcf::HostCatalogue hd, hr;
    if (!read_catalogue(p, p.data_filename, p.data_file_type, cosmo.get(), hd, e)) return false;
    log("read %lld data points from %s", (long long)hd.size(), p.data_filename.c_str());
    if (!read_catalogue(p, p.random_filename, p.random_file_type, cosmo.get(), hr, e)) return false;
    log("read %lld random points from %s", (long long)hr.size(), p.random_filename.c_str());
    if (report) {
        report->n_data_read = (long long)hd.size();
        report->n_rand_read = (long long)hr.size();
    }

    // Each auto_correlate_* re-partitions the catalogues that the previous
    // one's GalaxyBoxes left permuted in place; with points at d_comov < 0 the
    // partition's early stop can then keep a different set, which is not
    // reproduced here.
    const int n_modes = (int)p.plot_monopole + (int)p.plot_sigma_pi + (int)p.plot_s_mu;
    auto has_negative = [](const tpcf::HostCatalogue &h) {
        for (double d : h.d_comov)
            if (d < 0.0) return true;
        return false;
    };
    if (n_modes > 1 && (has_negative(hd) || has_negative(hr)))
        return e.set(TPCF_E_UNSUPPORTED,
                     "catalogue points with d_comov < 0 and more than one of plot_monopole / plot_sigma_pi / "
                     "plot_s_mu: run the modes one per parameter file");

    tpcf_ctx *c = nullptr;
    int rc = tpcf_create(device, &c);
    if (rc) return e.set(rc, "device context: " + std::string(c ? tpcf_last_error(c) : tpcf_status_string(rc)));
    CtxPtr ctx(c);
    CatPtr data, rand;
    if (!upload(c, hd, p.n_jk_regions, data, e) || !upload(c, hr, p.n_jk_regions, rand, e)) return false;
    log("catalogues on device %d: %lld + %lld points kept", device, (long long)tpcf_catalog_n_used(data.get()),
        (long long)tpcf_catalog_n_used(rand.get()));

    if (report) {
        report->n_data_kept = (long long)tpcf_catalog_n_used(data.get());
        report->n_rand_kept = (long long)tpcf_catalog_n_used(rand.get());
    }
    return correlate_modes(c, p, data.get(), rand.get(), precision, nullptr, nullptr, log, e, report);
}

// The JSON run summary of tpcf_run_param_file_report.
bool write_summary(const char *summary_path, const char *path, int device, int precision, const Report &r,
                   double wall_s, const Err &e) {
    std::string j = "{\"parameter_file\": " + jstr(path) + ", \"device\": " + std::to_string(device) +
                    ", \"precision\": " + jstr(precision == TPCF_FP64 ? "fp64" : "fp32_guard") +
                    ", \"status\": " + std::to_string(e.status) + ", \"error\": " +
                    (e.status ? jstr(e.msg) : std::string("null")) + ", \"wall_s\": " + jnum(wall_s) +
                    ", \"catalogues\": {\"data\": {\"read\": " + std::to_string(r.n_data_read) +
                    ", \"kept\": " + std::to_string(r.n_data_kept) + "}, \"randoms\": {\"read\": " +
                    std::to_string(r.n_rand_read) + ", \"kept\": " + std::to_string(r.n_rand_kept) +
                    "}}, \"kernel_ms\": " + jnum(r.kernel_ms) + ", \"in_range_pairs\": " + jnum(r.pairs) +
                    ", \"pairs_per_s\": " + jnum(r.kernel_ms > 0 ? r.pairs / (r.kernel_ms * 1e-3) : NAN) +
                    ", \"fp64_check\": " + (r.check_fp64 ? "true" : "false") + ", \"modes\": [";
    for (size_t k = 0; k < r.modes.size(); ++k) j += (k ? ", " : "") + r.modes[k];
    j += "]}\n";
    FILE *f = std::fopen(summary_path, "w");
    if (!f) return false;
    const bool ok = std::fwrite(j.data(), 1, j.size(), f) == j.size();
    return std::fclose(f) == 0 && ok;
}

}  // namespace

extern "C" int tpcf_run_param_file_report(const char *path, int device, int precision, int log_level,
                                          int check_fp64, const char *summary_path) {
    if (!path) {
        tpcf::set_host_error("NULL parameter file path");
        return TPCF_E_INVALID_ARG;
    }
    if (precision != TPCF_FP32_GUARD && precision != TPCF_FP64) {
        tpcf::set_host_error("bad precision");
        return TPCF_E_INVALID_ARG;
    }
    Log log{log_level};
    Err e;
    Report report;
    report.check_fp64 = check_fp64 != 0;
    const bool want = summary_path || check_fp64;
    const auto t0 = std::chrono::steady_clock::now();
    bool ok = false;
    try {
        ok = run(path, device, precision, log, e, want ? &report : nullptr);
    } catch (const std::bad_alloc &) {
        e.status = TPCF_E_OOM;
        e.msg = "out of host memory";
    }
    if (!ok && !e.status) e.status = TPCF_E_INVALID_ARG;
    if (summary_path) {
        const double wall = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        if (!write_summary(summary_path, path, device, precision, report, wall, e) && ok) {
            e.set(TPCF_E_INVALID_ARG, std::string("cannot write the run summary ") + summary_path);
            ok = false;
        }
    }
    if (ok) return TPCF_OK;
    tpcf::set_host_error(e.msg);
    return e.status;
}

extern "C" int tpcf_run_param_file(const char *path, int device, int precision, int log_level) {
    return tpcf_run_param_file_report(path, device, precision, log_level, 0, nullptr);
}

extern "C" int tpcf_run_invp(tpcf_ctx *ctx, const tpcf_params *params, const tpcf_catalog *data,
                             const tpcf_catalog *randoms, int precision, int dither, double *angular_out,
                             int log_level) {
    if (!ctx || !params || !data || !randoms) {
        tpcf::set_host_error("NULL argument");
        return TPCF_E_INVALID_ARG;
    }
    if (precision != TPCF_FP32_GUARD && precision != TPCF_FP64) {
        tpcf::set_host_error("bad precision");
        return TPCF_E_INVALID_ARG;
    }
    const tpcf::Params &p = params->p;
    if (p.theta_n_bins < 1 || !(p.theta_max > 0)) {
        tpcf::set_host_error("theta_max and theta_n_bins must be set for the inverse-p flow");
        return TPCF_E_INVALID_ARG;
    }
    Log log{log_level};
    Err e;
    try {
        if (run_invp(ctx, p, data, randoms, precision, dither != 0, angular_out, log, e)) return TPCF_OK;
    } catch (const std::bad_alloc &) {
        e.status = TPCF_E_OOM;
        e.msg = "out of host memory";
    }
    tpcf::set_host_error(e.msg);
    return e.status ? e.status : TPCF_E_INVALID_ARG;
}
