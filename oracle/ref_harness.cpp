// TEST INFRASTRUCTURE ONLY — in-process harness around the reference's own
// sources.  oracle/build_ref.sh compiles this file together with the
// unmodified reference translation units (src/*.cpp, src/healpix/*.cpp) into
// oracle/_ref/libtwopcf_ref_{plain,invp}.so.  Tests, the golden-fixture
// generator and the CPU baseline leg of bench.py call these entry points to
// run the reference algorithm on in-memory catalogues; the product never
// links or loads this library.
//
// Every entry point builds GalaxyCatalogue objects exactly as the reference
// readers would (src/io.cpp:337-405 for cartesian input), constructs the
// reference's GalaxyBoxes / GalaxyPixels and histogram classes, and calls the
// reference's counting functions.  Outputs are the histograms as the
// reference leaves them after invert_jk_hists() and (auto counts)
// multiply_hists(2.0), i.e. before normalise().
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <iostream>
#include <sstream>
#include <string>
#include <unistd.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#include "boxes.h"
#include "correlators.h"
#include "cosmology.h"
#include "galaxy.h"
#include "hist.h"
#include "io.h"
#ifdef _USE_INV_WEIGHTS
#include "correlators_invpweight.h"
#include "hdf5.h"
#endif

namespace {

// The reference narrates every step on std::cout; silence it while a harness
// call runs so that test output stays readable.
struct NullBuf : std::streambuf {
    int overflow(int c) override { return c; }
};

struct Quiet {
    NullBuf nb;
    std::streambuf *old;
    Quiet() : old(std::cout.rdbuf(&nb)) {}
    ~Quiet() { std::cout.rdbuf(old); }
};

void set_threads(int n_threads) {
#ifdef _OPENMP
    if (n_threads <= 0) n_threads = omp_get_max_threads();
    omp_set_num_threads(n_threads);
#else
    (void)n_threads;
#endif
}

// Galaxy fields as the cartesian reader fills them (src/io.cpp:358-399):
// x from the file, d_comov = |x| (or as given), x_norm = x / d_comov (or as
// given), weight (1.0 when absent), jk_region (0 when absent).
void fill_cat(GalaxyCatalogue *cat, const double *xyz, const double *unit, const double *dcom,
              const float *w, const int *jk) {
    for (int i = 0; i < cat->n_gals; ++i) {
        Galaxy &g = cat->gals[i];
        for (int m = 0; m < 3; ++m) g.x[m] = xyz[3 * i + m];
        g.d_comov = dcom ? dcom[i] : std::sqrt(g.x[0] * g.x[0] + g.x[1] * g.x[1] + g.x[2] * g.x[2]);
        for (int m = 0; m < 3; ++m) g.x_norm[m] = unit ? unit[3 * i + m] : g.x[m] / g.d_comov;
        g.weight = w ? w[i] : 1.0f;
        g.jk_region = jk ? jk[i] : 0;
    }
}

std::string write_temp_params(const char *text) {
    char path[] = "/tmp/tpcf_ref_params_XXXXXX";
    int fd = mkstemp(path);
    if (fd < 0) return "";
    size_t len = std::strlen(text);
    if (write(fd, text, len) != (ssize_t)len) { close(fd); return ""; }
    close(fd);
    return path;
}

// Dither masks (the _USE_DITHER_WEIGHTS build) of the first and second
// catalogue of the next calls, object-major; set by ref_invp_set_dither.
const long long *g_dither[2] = {nullptr, nullptr};

}  // namespace

extern "C" {

struct RefAxisFields {
    int n_bins;
    int log_binning;
    float min, minus_min, max, step, inv_step, base, inv_log_of_base, inv_log_step;
};

// Axis fields exactly as src/hist.cpp:15-36 sets them.  Parameters arrive as
// double because the reference's Params stores them as double (src/io.h:42-66)
// and converts at the Hist/Axis constructor call.
void ref_axis_fields(double min, double max, int n_bins, double base, RefAxisFields *out) {
    Axis ax(min, max, n_bins, base);
    out->n_bins = ax.n_bins;
    out->log_binning = ax.log_binning ? 1 : 0;
    out->min = ax.min;
    out->minus_min = ax.minus_min;
    out->max = ax.max;
    out->step = ax.step;
    out->inv_step = ax.inv_step;
    out->base = ax.base;
    out->inv_log_of_base = ax.inv_log_of_base;
    out->inv_log_step = ax.inv_log_step;
}

// Axis::bin_num (src/hist.cpp:46-53) over an array of float values.
void ref_axis_bin_num(double min, double max, int n_bins, double base, const float *v, long long n,
                      float *out) {
    Axis ax(min, max, n_bins, base);
    for (long long i = 0; i < n; ++i) out[i] = ax.bin_num(v[i]);
}

// Axis::bin_centre / bin_width (src/hist.cpp:38-44).
void ref_axis_centres(double min, double max, int n_bins, double base, double *centre, double *width) {
    Axis ax(min, max, n_bins, base);
    for (int i = 0; i < n_bins; ++i) {
        centre[i] = ax.bin_centre(i);
        width[i] = ax.bin_width(i);
    }
}

double ref_ls_estimator(double dd, double dr, double rr) { return ls_estimator(dd, dr, rr); }

// Cosmology(omega_m, h, z_min, z_max, 1e-4, 100) as built in src/main.cpp:40,
// then comov_dist(z) (src/cosmology.cpp:98-100).
void ref_comov_dist(double omega_m, double h, double z_min, double z_max, const double *z, long long n,
                    double *out) {
    Quiet q;
    Cosmology cosmo(omega_m, h, z_min, z_max, 0.0001, 100);
    for (long long i = 0; i < n; ++i) out[i] = cosmo.comov_dist(z[i]);
}

// Galaxy::set (src/galaxy.cpp:8-27).
void ref_galaxy_set(const double *ra, const double *dec, const double *dcom, long long n, double *x,
                    double *x_norm) {
    for (long long i = 0; i < n; ++i) {
        Galaxy g;
        g.d_comov = dcom[i];
        g.set(ra[i], dec[i]);
        for (int m = 0; m < 3; ++m) {
            x[3 * i + m] = g.x[m];
            x_norm[3 * i + m] = g.x_norm[m];
        }
    }
}

// Params(file) (src/io.cpp:16-237) on the given text; returns the numeric
// fields in a fixed order (see tests/test_ingest_cpu.py) — doubles first,
// then ints.
int ref_params_parse(const char *text, double *dbl, int *ints) {
    std::string path = write_temp_params(text);
    if (path.empty()) return -1;
    Quiet q;
    Params p(path);
    std::remove(path.c_str());
    double d[] = {p.omega_m, p.h, p.z_min, p.z_max, p.monopole_log_base, p.monopole_min, p.monopole_max,
                  p.sigma_log_base, p.sigma_min, p.sigma_max, p.pi_log_base, p.pi_min, p.pi_max,
                  p.s_log_base, p.s_min, p.s_max, p.theta_max, p.theta_log_base};
    int k[] = {p.use_weights, p.n_threads, p.n_jk_regions, p.plot_monopole, p.monopole_n_bins,
               p.plot_sigma_pi, p.sigma_n_bins, p.pi_n_bins, p.plot_s_mu, p.s_n_bins, p.mu_n_bins,
               p.calculate_angular_dd, p.calculate_angular_dd_invpweights, p.calculate_angular_dr,
               p.calculate_angular_dr_invpweights, p.theta_n_bins, p.healpix_order, p.n_bitwise_runs};
    std::memcpy(dbl, d, sizeof(d));
    std::memcpy(ints, k, sizeof(k));
    return 0;
}

// read_file(path, "ascii", cosmo, params) (src/io.cpp:597-626) with the
// Params of the given text (coord_system, use_weights, n_jk_regions and the
// cosmology as src/main.cpp:39-45 sets them up).  Returns the number of
// points; the outputs are written only when cap >= that number.
long long ref_read_ascii(const char *param_text, const char *path, long long cap, double *x_out,
                         double *xnorm_out, double *dcom_out, float *weight_out, int *jk_out) {
    std::string ppath = write_temp_params(param_text);
    if (ppath.empty()) return -1;
    Quiet q;
    Params p(ppath);
    std::remove(ppath.c_str());
    Cosmology *cosmo = NULL;
    if (p.coord_system == "equatorial") cosmo = new Cosmology(p.omega_m, p.h, p.z_min, p.z_max, 0.0001, 100);
    GalaxyCatalogue *cat = read_file(path, "ascii", cosmo, p);
    delete cosmo;
    long long n = cat ? cat->n_gals : -1;
    if (cat && cap >= n) {
        for (long long i = 0; i < n; ++i) {
            const Galaxy &g = cat->gals[i];
            for (int m = 0; m < 3; ++m) { x_out[3 * i + m] = g.x[m]; xnorm_out[3 * i + m] = g.x_norm[m]; }
            dcom_out[i] = g.d_comov;
            weight_out[i] = g.weight;
            jk_out[i] = g.jk_region;
        }
    }
    delete cat;
    return n;
}

// output_xi_1D (mode 0) / output_xi_2D (mode 1 sigma-pi, 2 s-mu) with file
// type "ascii" (src/io.cpp:724-756, :832-853) on histograms given as arrays;
// axp = {min1, max1, base1, min2, max2, base2} as the Params doubles, the
// histograms built as the auto_correlate_* drivers build them
// (src/correlators.cpp:131, :284-285, :436-437).
int ref_write_xi(const char *filename, int mode, const double *axp, int nb1, int nb2, int n_jk, const double *dd,
                 const double *dr, const double *rr, const double *dd_sub, const double *dr_sub,
                 const double *rr_sub) {
    Quiet q;
    const double *src[3][2] = {{dd, dd_sub}, {dr, dr_sub}, {rr, rr_sub}};
    if (mode == 0) {
        Hist tmp(axp[0], axp[1], nb1, axp[2]);
        JKHists h0(n_jk, tmp), h1(n_jk, tmp), h2(n_jk, tmp);
        JKHists *h[3] = {&h0, &h1, &h2};
        for (int k = 0; k < 3; ++k) {
            std::memcpy(h[k]->full_hist.bins, src[k][0], sizeof(double) * nb1);
            std::memcpy(h[k]->sub_hist, src[k][1], sizeof(double) * nb1 * n_jk);
        }
        output_xi_1D(filename, "ascii", &h0, &h1, &h2, NULL, NULL);
    } else {
        Hist2D tmp = (mode == 1) ? Hist2D(axp[0], axp[1], nb1, axp[2], axp[3], axp[4], nb2, axp[5])
                                 : Hist2D(axp[0], axp[1], nb1, axp[2], 0.0, 1.0, nb2, 0);
        JKHists2D h0(n_jk, tmp), h1(n_jk, tmp), h2(n_jk, tmp);
        JKHists2D *h[3] = {&h0, &h1, &h2};
        const int nb = nb1 * nb2;
        for (int k = 0; k < 3; ++k) {
            std::memcpy(h[k]->full_hist.bins, src[k][0], sizeof(double) * nb);
            std::memcpy(h[k]->sub_hist, src[k][1], sizeof(double) * nb * n_jk);
        }
        output_xi_2D(filename, "ascii", mode == 1 ? "sigma" : "s", mode == 1 ? "pi" : "mu", &h0, &h1, &h2, NULL,
                     NULL);
    }
    return 0;
}

// Normalise a histogram pair set as JKHists::normalise does
// (src/hist.cpp:290-367; the 2-D versions at :512-589 are the same loops over
// total_bins).  full/sub are updated in place.  is_auto selects the
// one-catalogue form.  n1/n2 are the "n_gals" arguments (the boxes' counts).
void ref_normalise(int is_auto, const float *w1, const int *jk1, int n1, const float *w2, const int *jk2,
                   int n2, int n_jk, int nb, double *full, double *sub) {
    Hist tmp(0.0f, 1.0f, nb, 0.0f);
    JKHists h(n_jk, tmp);
    std::memcpy(h.full_hist.bins, full, sizeof(double) * nb);
    std::memcpy(h.sub_hist, sub, sizeof(double) * nb * n_jk);
    GalaxyCatalogue c1(n1, n_jk), c2(is_auto ? 1 : n2, n_jk);
    for (int i = 0; i < n1; ++i) { c1.gals[i].weight = w1[i]; c1.gals[i].jk_region = jk1 ? jk1[i] : 0; }
    if (is_auto) {
        h.normalise(&c1, n1);
    } else {
        for (int i = 0; i < n2; ++i) { c2.gals[i].weight = w2[i]; c2.gals[i].jk_region = jk2 ? jk2[i] : 0; }
        h.normalise(&c1, n1, &c2, n2);
    }
    std::memcpy(full, h.full_hist.bins, sizeof(double) * nb);
    std::memcpy(sub, h.sub_hist, sizeof(double) * nb * n_jk);
}

#ifndef _USE_INV_WEIGHTS
// One 3-D pair count through the reference: mode 0 = monopole
// (src/correlators.cpp:11-125), 1 = sigma-pi (:156-278), 2 = s-mu (:309-430).
// axp = {min1, max1, base1, min2, max2, base2} as the Params doubles.
// The boxes are built as the auto_correlate_* drivers build them
// (src/correlators.cpp:137-138, :291-292, :443-444): each catalogue's boxes
// take the other catalogue into the bounding box.  For an auto count the
// second catalogue, if given, only widens the bounding box.
// n_used[0..1] receive the boxes' n_gals (points with d_comov >= 0 after the
// reference's partition loop, src/boxes.cpp:15-26).
int ref_count_3d(int mode, int is_auto, const double *xyz1, const double *unit1, const double *dcom1,
                 const float *w1, const int *jk1, int n1, const double *xyz2, const double *unit2,
                 const double *dcom2, const float *w2, const int *jk2, int n2, int n_jk, const double *axp,
                 int nb1, int nb2, int n_threads, double *full_out, double *sub_out, int *n_used) {
    Quiet q;
    set_threads(n_threads);
    GalaxyCatalogue c1(n1, n_jk);
    fill_cat(&c1, xyz1, unit1, dcom1, w1, jk1);
    GalaxyCatalogue c2(n2 > 0 ? n2 : 1, n_jk);
    c2.n_gals = n2;
    if (n2 > 0) fill_cat(&c2, xyz2, unit2, dcom2, w2, jk2);

    double rmax;
    if (mode == 0) rmax = axp[1];
    else if (mode == 1) rmax = std::sqrt(axp[1] * axp[1] + axp[4] * axp[4]);
    else rmax = axp[1];

    GalaxyBoxes b1(c1.gals, n1, c2.gals, n2, rmax);
    n_used[0] = b1.n_gals;
    int nb = 0;
    if (mode == 0) {
        Hist tmp(axp[0], axp[1], nb1, axp[2]);
        JKHists h(n_jk, tmp);
        nb = nb1;
        if (is_auto) {
            auto_pair_count_monopole(&b1, &h);
            n_used[1] = 0;
        } else {
            GalaxyBoxes b2(c2.gals, n2, c1.gals, n1, rmax);
            n_used[1] = b2.n_gals;
            cross_pair_count_monopole(&b1, &b2, &h);
        }
        std::memcpy(full_out, h.full_hist.bins, sizeof(double) * nb);
        std::memcpy(sub_out, h.sub_hist, sizeof(double) * nb * n_jk);
    } else {
        Hist2D tmp = (mode == 1) ? Hist2D(axp[0], axp[1], nb1, axp[2], axp[3], axp[4], nb2, axp[5])
                                 : Hist2D(axp[0], axp[1], nb1, axp[2], 0.0, 1.0, nb2, 0);
        JKHists2D h(n_jk, tmp);
        nb = nb1 * nb2;
        if (is_auto) {
            if (mode == 1) auto_pair_count_sigma_pi(&b1, &h);
            else auto_pair_count_s_mu(&b1, &h);
            n_used[1] = 0;
        } else {
            GalaxyBoxes b2(c2.gals, n2, c1.gals, n1, rmax);
            n_used[1] = b2.n_gals;
            if (mode == 1) cross_pair_count_sigma_pi(&b1, &b2, &h);
            else cross_pair_count_s_mu(&b1, &b2, &h);
        }
        std::memcpy(full_out, h.full_hist.bins, sizeof(double) * nb);
        std::memcpy(sub_out, h.sub_hist, sizeof(double) * nb * n_jk);
    }
    if (is_auto) c2.n_gals = 0;
    return 0;
}
#endif  // !_USE_INV_WEIGHTS

#ifdef _USE_INV_WEIGHTS
int ref_n_mask_ints(void) { return _N_MASK_INTS; }

// Catalogue ingest through the reference's own HDF5 reader
// (src/io.cpp:418-593): the given columns are placed in an in-memory "file"
// under the dataset names of the params text, then read_file(..., "hdf5", ...)
// runs, including the bitwise-weight IIP rescaling (src/io.cpp:521-586).
// masks is dataset-major: masks[m * n + i] is BITWEIGHT<m> of object i.
// Outputs are the resulting Galaxy fields.
int ref_invp_read(const char *param_text, const double *c1, const double *c2, const double *c3,
                  const double *w, const int *jk, const long long *masks, int n, double *x_out,
                  double *xnorm_out, double *dcom_out, float *weight_out, float *input_weight_out,
                  int *jk_out, long long *mask_out) {
    std::string path = write_temp_params(param_text);
    if (path.empty()) return -1;
    Quiet q;
    Params p(path);
    std::remove(path.c_str());
    const char *fname = "__harness_input__.hdf5";
    hid_t f = H5Fcreate(fname, H5F_ACC_TRUNC, H5P_DEFAULT, H5P_DEFAULT);
    hsize_t dims = (hsize_t)n;
    auto put = [&](const std::string &name, hid_t type, const void *buf) {
        hid_t s = H5Screate_simple(1, &dims, NULL);
        hid_t d = H5Dcreate2(f, name.c_str(), type, s, H5P_DEFAULT, H5P_DEFAULT, H5P_DEFAULT);
        H5Dwrite(d, type, H5S_ALL, H5S_ALL, H5P_DEFAULT, buf);
        H5Dclose(d);
        H5Sclose(s);
    };
    put(p.ra_x_dataset_name, H5T_NATIVE_DOUBLE, c1);
    put(p.dec_y_dataset_name, H5T_NATIVE_DOUBLE, c2);
    put(p.z_z_dataset_name, H5T_NATIVE_DOUBLE, c3);
    if (w) put(p.weight_dataset_name, H5T_NATIVE_DOUBLE, w);
    if (jk) put(p.jk_dataset_name, H5T_NATIVE_INT, jk);
    std::vector<long> tmp(n);
    for (int m = 0; m < _N_MASK_INTS; ++m) {
        for (int i = 0; i < n; ++i) tmp[i] = (long)masks[(size_t)m * n + i];
        std::stringstream ss;
        ss << p.bitwise_weight_dataset_name << m;
        put(ss.str(), H5T_NATIVE_LONG, tmp.data());
    }
#ifdef _USE_DITHER_WEIGHTS
    // dither masks from ref_invp_set_dither (first catalogue), object-major
    for (int m = 0; m < _N_MASK_INTS; ++m) {
        for (int i = 0; i < n; ++i) tmp[i] = g_dither[0] ? (long)g_dither[0][(size_t)i * _N_MASK_INTS + m] : -1L;
        std::stringstream ss;
        ss << p.dither_weight_dataset_name << m;
        put(ss.str(), H5T_NATIVE_LONG, tmp.data());
    }
#endif
    H5Fclose(f);
    Cosmology *cosmo = NULL;
    if (p.coord_system == "equatorial") cosmo = new Cosmology(p.omega_m, p.h, p.z_min, p.z_max, 0.0001, 100);
    GalaxyCatalogue *cat = read_file(fname, "hdf5", cosmo, p);
    delete cosmo;
    for (int i = 0; i < n; ++i) {
        const Galaxy &g = cat->gals[i];
        for (int m = 0; m < 3; ++m) { x_out[3 * i + m] = g.x[m]; xnorm_out[3 * i + m] = g.x_norm[m]; }
        dcom_out[i] = g.d_comov;
        weight_out[i] = g.weight;
        input_weight_out[i] = g.input_weight;
        jk_out[i] = g.jk_region;
        for (int m = 0; m < _N_MASK_INTS; ++m) mask_out[(size_t)i * _N_MASK_INTS + m] = g.bitmask[m];
    }
    delete cat;
    return 0;
}

namespace {
void fill_cat_invp(GalaxyCatalogue *cat, const double *xyz, const double *unit, const double *dcom,
                   const float *w, const float *iw, const int *jk, const long long *masks, int which) {
    fill_cat(cat, xyz, unit, dcom, w, jk);
    for (int i = 0; i < cat->n_gals; ++i) {
        cat->gals[i].input_weight = iw ? iw[i] : cat->gals[i].weight;
        for (int m = 0; m < _N_MASK_INTS; ++m) cat->gals[i].bitmask[m] = masks ? masks[(size_t)i * _N_MASK_INTS + m] : -1LL;
#ifdef _USE_DITHER_WEIGHTS
        const long long *d = g_dither[which];
        for (int m = 0; m < _N_MASK_INTS; ++m) cat->gals[i].dither_mask[m] = d ? d[(size_t)i * _N_MASK_INTS + m] : -1LL;
#else
        (void)which;
#endif
    }
}
}  // namespace

int ref_has_dither(void) {
#ifdef _USE_DITHER_WEIGHTS
    return 1;
#else
    return 0;
#endif
}

void ref_invp_set_dither(const long long *d1, const long long *d2) {
    g_dither[0] = d1;
    g_dither[1] = d2;
}

// Angular stage (src/correlators_invpweight.cpp:713-982 via the stages of
// calc_angular_upweight, :985-1033).  kind: 0 = angular DD
// (auto_pair_count_angular, pixels built with require_redshift = 0), 1 = DD
// with inverse-p weights (require_redshift = 1), 2 = DR
// (cross_pair_count_angular), 3 = DR with inverse-p weights.  The histogram
// axis is Hist(0, 1 - cos(theta_max), theta_n_bins, theta_log_base) from the
// params text.
int ref_invp_angular(const char *param_text, int kind, const double *xyz1, const double *unit1,
                     const double *dcom1, const float *w1, const float *iw1, const int *jk1,
                     const long long *m1, int n1, const double *xyz2, const double *unit2,
                     const double *dcom2, const float *w2, const float *iw2, const int *jk2,
                     const long long *m2, int n2, int n_threads, double *full_out, double *sub_out) {
    std::string path = write_temp_params(param_text);
    if (path.empty()) return -1;
    Quiet q;
    set_threads(n_threads);
    Params p(path);
    std::remove(path.c_str());
    GalaxyCatalogue c1(n1, p.n_jk_regions);
    fill_cat_invp(&c1, xyz1, unit1, dcom1, w1, iw1, jk1, m1, 0);
    Hist tmp(0.0, 1.0 - cos(p.theta_max), p.theta_n_bins, p.theta_log_base);
    JKHists h(p.n_jk_regions, tmp);
    bool req = (kind == 1 || kind == 3);
    GalaxyPixels px1(c1.gals, n1, p.healpix_order, p.theta_max, req);
    if (kind == 0) auto_pair_count_angular(&px1, &h);
    else if (kind == 1) auto_pair_count_angular_invpweights(&px1, &h, p);
    else {
        GalaxyCatalogue c2(n2, p.n_jk_regions);
        fill_cat_invp(&c2, xyz2, unit2, dcom2, w2, iw2, jk2, m2, 1);
        GalaxyPixels px2(c2.gals, n2, p.healpix_order, p.theta_max, req);
        if (kind == 2) cross_pair_count_angular(&px1, &px2, &h);
        else cross_pair_count_angular_invpweights(&px1, &px2, &h);
    }
    int nb = h.full_hist.ax.n_bins;
    std::memcpy(full_out, h.full_hist.bins, sizeof(double) * nb);
    std::memcpy(sub_out, h.sub_hist, sizeof(double) * nb * p.n_jk_regions);
    return 0;
}

// Store an angular histogram under a file name with JKHists::output_hdf5
// (src/hist.cpp:180-220), so the 3-D inverse-p counts read it back through
// read_hdf5_hist (src/hist.cpp:115-178) exactly as in a reference run.
int ref_invp_store_angular(const char *param_text, const char *fname, const double *full, const double *sub) {
    std::string path = write_temp_params(param_text);
    if (path.empty()) return -1;
    Quiet q;
    Params p(path);
    std::remove(path.c_str());
    Hist tmp(0.0, 1.0 - cos(p.theta_max), p.theta_n_bins, p.theta_log_base);
    JKHists h(p.n_jk_regions, tmp);
    int nb = h.full_hist.ax.n_bins;
    std::memcpy(h.full_hist.bins, full, sizeof(double) * nb);
    std::memcpy(h.sub_hist, sub, sizeof(double) * nb * p.n_jk_regions);
    h.output_hdf5(fname);
    return 0;
}

// The angular up-weight as the 3-D stage forms it: read the parent and the
// inverse-p histograms, divide (src/hist.cpp:224-231), and evaluate
// JKHists::interp (src/hist.cpp:369-391) at the given 1 - cos(theta) values.
int ref_invp_interp(const char *num_file, const char *den_file, const double *v, long long n, double *out) {
    Quiet q;
    JKHists *num = nullptr, *den = nullptr;
    read_hdf5_hist(num_file, &num);
    read_hdf5_hist(den_file, &den);
    if (!num || !den) return -1;
    num->divide_by_hist(*den);
    for (long long i = 0; i < n; ++i) out[i] = num->interp(v[i]);
    delete num;
    delete den;
    return 0;
}

// 3-D counts of the inverse-p build (src/correlators_invpweight.cpp:14-709).
// mode 0/1/2 = monopole / sigma-pi / s-mu.  is_auto: 1 = DD with inverse-p
// weights, 0 = DR with the angular DR up-weight, 2 = plain auto count (RR,
// which the reference runs with the unweighted counter, :232, :469, :706).
// The angular histograms must have been stored under the params' file names.
int ref_invp_count_3d(const char *param_text, int mode, int is_auto, const double *xyz1, const double *unit1,
                      const double *dcom1, const float *w1, const float *iw1, const int *jk1,
                      const long long *m1, int n1, const double *xyz2, const double *unit2,
                      const double *dcom2, const float *w2, const float *iw2, const int *jk2,
                      const long long *m2, int n2, int n_threads, double *full_out, double *sub_out) {
    std::string path = write_temp_params(param_text);
    if (path.empty()) return -1;
    Quiet q;
    set_threads(n_threads);
    Params p(path);
    std::remove(path.c_str());
    int n_jk = p.n_jk_regions;
    GalaxyCatalogue c1(n1, n_jk);
    fill_cat_invp(&c1, xyz1, unit1, dcom1, w1, iw1, jk1, m1, 0);
    GalaxyCatalogue c2(n2 > 0 ? n2 : 1, n_jk);
    c2.n_gals = n2;
    if (n2 > 0) fill_cat_invp(&c2, xyz2, unit2, dcom2, w2, iw2, jk2, m2, 1);
    double rmax = mode == 0 ? p.monopole_max
                : mode == 1 ? std::sqrt(p.sigma_max * p.sigma_max + p.pi_max * p.pi_max) : p.s_max;
    GalaxyBoxes b1(c1.gals, n1, c2.gals, n2, rmax);
    int nb;
    if (mode == 0) {
        Hist tmp(p.monopole_min, p.monopole_max, p.monopole_n_bins, p.monopole_log_base);
        JKHists h(n_jk, tmp);
        nb = h.full_hist.ax.n_bins;
        if (is_auto == 1) auto_pair_count_monopole_invpweights(&b1, &h, p);
        else if (is_auto == 2) auto_pair_count_monopole(&b1, &h);
        else {
            GalaxyBoxes b2(c2.gals, n2, c1.gals, n1, rmax);
            cross_pair_count_monopole_invpweights(&b1, &b2, &h, p);
        }
        std::memcpy(full_out, h.full_hist.bins, sizeof(double) * nb);
        std::memcpy(sub_out, h.sub_hist, sizeof(double) * nb * n_jk);
    } else {
        Hist2D tmp = (mode == 1) ? Hist2D(p.sigma_min, p.sigma_max, p.sigma_n_bins, p.sigma_log_base, p.pi_min,
                                          p.pi_max, p.pi_n_bins, p.pi_log_base)
                                 : Hist2D(p.s_min, p.s_max, p.s_n_bins, p.s_log_base, 0.0, 1.0, p.mu_n_bins, 0);
        JKHists2D h(n_jk, tmp);
        nb = h.full_hist.total_bins;
        if (is_auto == 1) {
            if (mode == 1) auto_pair_count_sigma_pi_invpweights(&b1, &h, p);
            else auto_pair_count_s_mu_invpweights(&b1, &h, p);
        } else if (is_auto == 2) {
            if (mode == 1) auto_pair_count_sigma_pi(&b1, &h);
            else auto_pair_count_s_mu(&b1, &h);
        } else {
            GalaxyBoxes b2(c2.gals, n2, c1.gals, n1, rmax);
            if (mode == 1) cross_pair_count_sigma_pi_invpweights(&b1, &b2, &h, p);
            else cross_pair_count_s_mu_invpweights(&b1, &b2, &h, p);
        }
        std::memcpy(full_out, h.full_hist.bins, sizeof(double) * nb);
        std::memcpy(sub_out, h.sub_hist, sizeof(double) * nb * n_jk);
    }
    c2.n_gals = n2 > 0 ? n2 : 1;
    return 0;
}

// The inverse-p program after its catalogues are read (src/main.cpp:51-60):
// calc_angular_upweight (src/correlators_invpweight.cpp:985-1033), whose
// angular histograms go through the HDF5 stand-in under the params' file
// names, then auto_correlate_{monopole,sigma_pi,s_mu}_invpweights as the
// plot_* flags select, each writing its outputs (type "ascii") where the
// params name them.  Catalogue 1 is the data, catalogue 2 the randoms.
int ref_invp_correlate(const char *param_text, const double *xyz1, const double *unit1, const double *dcom1,
                       const float *w1, const float *iw1, const int *jk1, const long long *m1, int n1,
                       const double *xyz2, const double *unit2, const double *dcom2, const float *w2,
                       const float *iw2, const int *jk2, const long long *m2, int n2, int n_threads) {
    std::string path = write_temp_params(param_text);
    if (path.empty()) return -1;
    Quiet q;
    set_threads(n_threads);
    Params p(path);
    std::remove(path.c_str());
    GalaxyCatalogue data(n1, p.n_jk_regions), randoms(n2, p.n_jk_regions);
    fill_cat_invp(&data, xyz1, unit1, dcom1, w1, iw1, jk1, m1, 0);
    fill_cat_invp(&randoms, xyz2, unit2, dcom2, w2, iw2, jk2, m2, 1);
    calc_angular_upweight(&data, &randoms, p);
    if (p.plot_monopole) auto_correlate_monopole_invpweights(&data, &randoms, p);
    if (p.plot_sigma_pi) auto_correlate_sigma_pi_invpweights(&data, &randoms, p);
    if (p.plot_s_mu) auto_correlate_s_mu_invpweights(&data, &randoms, p);
    return 0;
}

void ref_h5_reset(void) { h5stub_reset(); }
#endif  // _USE_INV_WEIGHTS

}  // extern "C"
