// C ABI of the host-side command-line flow (include/two_pcf_b200.h, second
// part): parameter file, cosmology, coordinate transforms, ASCII reader and
// writers, and the whole program on a parameter file.
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <memory>
#include <new>
#include <string>
#include <vector>

#ifdef _OPENMP
#include <omp.h>
#endif

#include "capi_types.h"
#include "ingest.h"

namespace {

thread_local std::string g_host_error;

int host_fail(int status, const std::string &msg) {
    g_host_error = msg;
    return status;
}

int copy_out(const std::string &s, char *out, int32_t cap) {
    if (cap < 0 || (cap > 0 && !out)) return -TPCF_E_INVALID_ARG;
    if (cap > 0) {
        size_t k = std::min<size_t>(s.size(), (size_t)cap - 1);
        std::memcpy(out, s.data(), k);
        out[k] = '\0';
    }
    return (int)s.size();
}

}  // namespace

void tpcf::set_host_error(const std::string &msg) { g_host_error = msg; }

extern "C" {

const char *tpcf_host_last_error(void) { return g_host_error.c_str(); }

int tpcf_params_load(const char *path, tpcf_params **out) {
    if (!path || !out) return host_fail(TPCF_E_INVALID_ARG, "NULL argument");
    *out = nullptr;
    std::unique_ptr<tpcf_params> p(new (std::nothrow) tpcf_params());
    if (!p) return TPCF_E_OOM;
    std::string err;
    if (!tpcf::load_params(path, p->p, err)) return host_fail(TPCF_E_INVALID_ARG, err);
    *out = p.release();
    return TPCF_OK;
}

int tpcf_params_parse(const char *text, tpcf_params **out) {
    if (!text || !out) return host_fail(TPCF_E_INVALID_ARG, "NULL argument");
    *out = nullptr;
    std::unique_ptr<tpcf_params> p(new (std::nothrow) tpcf_params());
    if (!p) return TPCF_E_OOM;
    std::string err;
    if (!tpcf::parse_params(text, p->p, err)) return host_fail(TPCF_E_INVALID_ARG, err);
    *out = p.release();
    return TPCF_OK;
}

int tpcf_params_destroy(tpcf_params *params) {
    delete params;
    return TPCF_OK;
}

int tpcf_params_get_double(const tpcf_params *params, const char *key, double *out) {
    if (!params || !key || !out) return host_fail(TPCF_E_INVALID_ARG, "NULL argument");
    if (!tpcf::params_get_double(params->p, key, *out))
        return host_fail(TPCF_E_INVALID_ARG, std::string("no floating-point key ") + key);
    return TPCF_OK;
}

int tpcf_params_get_int(const tpcf_params *params, const char *key, int32_t *out) {
    if (!params || !key || !out) return host_fail(TPCF_E_INVALID_ARG, "NULL argument");
    int v = 0;
    if (!tpcf::params_get_int(params->p, key, v))
        return host_fail(TPCF_E_INVALID_ARG, std::string("no integer key ") + key);
    *out = v;
    return TPCF_OK;
}

int tpcf_params_get_string(const tpcf_params *params, const char *key, char *out, int32_t cap) {
    if (!params || !key) return -host_fail(TPCF_E_INVALID_ARG, "NULL argument");
    std::string v;
    if (!tpcf::params_get_string(params->p, key, v))
        return -host_fail(TPCF_E_INVALID_ARG, std::string("no string key ") + key);
    return copy_out(v, out, cap);
}

int tpcf_cosmology_create(double omega_m, double h, double z_min, double z_max, double z_save_step,
                          int32_t z_oversample, tpcf_cosmology **out) {
    if (!out) return host_fail(TPCF_E_INVALID_ARG, "NULL argument");
    *out = nullptr;
    std::unique_ptr<tpcf_cosmology> c(new (std::nothrow) tpcf_cosmology());
    if (!c) return TPCF_E_OOM;
    std::string err;
    if (!tpcf::make_cosmology(omega_m, h, z_min, z_max, z_save_step, z_oversample, c->t, err))
        return host_fail(TPCF_E_INVALID_ARG, err);
    *out = c.release();
    return TPCF_OK;
}

int tpcf_cosmology_destroy(tpcf_cosmology *cosmo) {
    delete cosmo;
    return TPCF_OK;
}

int tpcf_cosmology_comov_dist(const tpcf_cosmology *cosmo, const double *z, int64_t n, double *out) {
    if (!cosmo || n < 0 || (n > 0 && (!z || !out))) return host_fail(TPCF_E_INVALID_ARG, "bad argument");
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; ++i) out[i] = tpcf::comov_dist(cosmo->t, z[i]);
    return TPCF_OK;
}

int tpcf_galaxy_set(int64_t n, const double *ra_deg, const double *dec_deg, const double *d_comov, double *xyz,
                    double *x_norm) {
    if (n < 0 || (n > 0 && (!ra_deg || !dec_deg || !d_comov || !xyz || !x_norm)))
        return host_fail(TPCF_E_INVALID_ARG, "bad argument");
    tpcf::galaxy_set(n, ra_deg, dec_deg, d_comov, xyz, x_norm);
    return TPCF_OK;
}

int tpcf_cartesian_set(int64_t n, const double *xyz, double *d_comov, double *x_norm) {
    if (n < 0 || (n > 0 && (!xyz || !d_comov || !x_norm))) return host_fail(TPCF_E_INVALID_ARG, "bad argument");
    tpcf::cartesian_set(n, xyz, d_comov, x_norm);
    return TPCF_OK;
}

int tpcf_read_ascii(const char *path, int coord_system, int use_weights, int32_t n_jk_regions,
                    const tpcf_cosmology *cosmo, tpcf_host_catalog **out) {
    if (!path || !out) return host_fail(TPCF_E_INVALID_ARG, "NULL argument");
    *out = nullptr;
    if (coord_system != TPCF_CARTESIAN && coord_system != TPCF_EQUATORIAL)
        return host_fail(TPCF_E_INVALID_ARG, "coord_system must be TPCF_CARTESIAN or TPCF_EQUATORIAL");
    if (coord_system == TPCF_EQUATORIAL && !cosmo)
        return host_fail(TPCF_E_INVALID_ARG, "equatorial input needs a cosmology");
    std::unique_ptr<tpcf_host_catalog> c(new (std::nothrow) tpcf_host_catalog());
    if (!c) return TPCF_E_OOM;
    std::string err;
    try {
        if (!tpcf::read_ascii(path, coord_system == TPCF_EQUATORIAL ? tpcf::Coords::Equatorial : tpcf::Coords::Cartesian,
                              use_weights != 0, n_jk_regions, cosmo ? &cosmo->t : nullptr, c->c, err))
            return host_fail(TPCF_E_INVALID_ARG, err);
    } catch (const std::bad_alloc &) {
        return host_fail(TPCF_E_OOM, "out of host memory reading " + std::string(path));
    }
    *out = c.release();
    return TPCF_OK;
}

int64_t tpcf_host_catalog_size(const tpcf_host_catalog *cat) { return cat ? cat->c.size() : -TPCF_E_INVALID_ARG; }

int tpcf_host_catalog_arrays(const tpcf_host_catalog *cat, const double **xyz, const double **x_norm,
                             const double **d_comov, const float **weight, const int32_t **jk_region) {
    if (!cat) return host_fail(TPCF_E_INVALID_ARG, "NULL catalogue");
    if (xyz) *xyz = cat->c.xyz.data();
    if (x_norm) *x_norm = cat->c.x_norm.data();
    if (d_comov) *d_comov = cat->c.d_comov.data();
    if (weight) *weight = cat->c.weight.data();
    if (jk_region) *jk_region = cat->c.jk_region.data();
    return TPCF_OK;
}

int tpcf_host_catalog_destroy(tpcf_host_catalog *cat) {
    delete cat;
    return TPCF_OK;
}

int tpcf_sub_filename(const char *filename, int64_t sub, char *out, int32_t cap) {
    if (!filename) return -host_fail(TPCF_E_INVALID_ARG, "NULL argument");
    std::string r, err;
    if (!tpcf::sub_filename(filename, (long long)sub, r, err)) return -host_fail(TPCF_E_INVALID_ARG, err);
    return copy_out(r, out, cap);
}

int tpcf_write_xi_ascii(const char *filename, const tpcf_binning *bin, const double *dd, const double *dr,
                        const double *rr, const double *dd_sub, const double *dr_sub, const double *rr_sub) {
    if (!filename || !bin || !dd || !dr || !rr) return host_fail(TPCF_E_INVALID_ARG, "NULL argument");
    const tpcf::Binning &B = bin->b;
    if (B.mode == TPCF_ANGULAR) return host_fail(TPCF_E_UNSUPPORTED, "angular histograms have no ASCII output");
    const bool with_sub = dd_sub || dr_sub || rr_sub;
    if (with_sub && !(dd_sub && dr_sub && rr_sub))
        return host_fail(TPCF_E_INVALID_ARG, "give all three region arrays or none");
    const tpcf::AxisParams *ax2 = B.mode == TPCF_MONOPOLE ? nullptr : &B.ax2;
    std::string err;
    if (!tpcf::write_xi_ascii_single(filename, B.ax1, ax2, dd, dr, rr, err)) return host_fail(TPCF_E_INVALID_ARG, err);
    if (with_sub) {
        for (int r = 0; r < B.n_jk; ++r) {
            std::string name;
            if (!tpcf::sub_filename(filename, r, name, err)) return host_fail(TPCF_E_INVALID_ARG, err);
            const size_t off = (size_t)r * B.nb;
            if (!tpcf::write_xi_ascii_single(name, B.ax1, ax2, dd_sub + off, dr_sub + off, rr_sub + off, err))
                return host_fail(TPCF_E_INVALID_ARG, err);
        }
    }
    return TPCF_OK;
}

}  // extern "C"
