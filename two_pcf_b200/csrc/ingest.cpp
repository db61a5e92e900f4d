// Parameter file, cosmology table, coordinate transforms, ASCII catalogue
// reader and ASCII result writers: the host work around the pair counts in the
// reference's command-line program (src/main.cpp:11-84).
#include "ingest.h"

#include <cerrno>
#include <climits>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>

#ifdef _OPENMP
#include <omp.h>
#endif

namespace tpcf {

namespace {

// std::stod / std::stof / std::stoi as libstdc++ defines them: strtod /
// strtof / strtol(…, 10) on the string, an error if nothing was converted or
// errno says ERANGE (stoi also when the long does not fit an int).  Trailing
// characters are ignored, leading white space is skipped.
bool sto_d(const char *s, double &out) {
    char *end;
    int saved = errno;
    errno = 0;
    double v = std::strtod(s, &end);
    bool ok = end != s && errno != ERANGE;
    errno = saved;
    if (ok) out = v;
    return ok;
}

bool sto_f(const char *s, float &out) {
    char *end;
    int saved = errno;
    errno = 0;
    float v = std::strtof(s, &end);
    bool ok = end != s && errno != ERANGE;
    errno = saved;
    if (ok) out = v;
    return ok;
}

bool sto_i(const char *s, int &out) {
    char *end;
    int saved = errno;
    errno = 0;
    long v = std::strtol(s, &end, 10);
    bool ok = end != s && errno != ERANGE && v >= INT_MIN && v <= INT_MAX;
    errno = saved;
    if (ok) out = (int)v;
    return ok;
}

std::string without_spaces(const std::string &s) {
    std::string r;
    r.reserve(s.size());
    for (char c : s)
        if (c != ' ') r.push_back(c);
    return r;
}

bool read_file_text(const std::string &path, std::string &out) {
    FILE *f = std::fopen(path.c_str(), "rb");
    if (!f) return false;
    out.clear();
    char buf[1 << 16];
    size_t got;
    while ((got = std::fread(buf, 1, sizeof(buf), f)) > 0) out.append(buf, got);
    bool ok = !std::ferror(f);
    std::fclose(f);
    return ok;
}

enum class Kind { Str, Bool, Int, Dbl };

// One parameter-file key and the Params member it sets.
struct KeyRef {
    const char *key;
    Kind kind;
    std::string Params::*s;
    bool Params::*b;
    int Params::*i;
    double Params::*d;
};

constexpr KeyRef S(const char *k, std::string Params::*m) { return {k, Kind::Str, m, nullptr, nullptr, nullptr}; }
constexpr KeyRef B(const char *k, bool Params::*m) { return {k, Kind::Bool, nullptr, m, nullptr, nullptr}; }
constexpr KeyRef I(const char *k, int Params::*m) { return {k, Kind::Int, nullptr, nullptr, m, nullptr}; }
constexpr KeyRef D(const char *k, double Params::*m) { return {k, Kind::Dbl, nullptr, nullptr, nullptr, m}; }

// The keys of src/io.cpp:40-218.
#define TPCF_KEY(F, name) F(#name, &Params::name)
const KeyRef kKeys[] = {
    TPCF_KEY(S, data_filename),
    TPCF_KEY(S, data_file_type),
    TPCF_KEY(S, random_filename),
    TPCF_KEY(S, random_file_type),
    TPCF_KEY(S, coord_system),
    TPCF_KEY(S, ra_x_dataset_name),
    TPCF_KEY(S, dec_y_dataset_name),
    TPCF_KEY(S, z_z_dataset_name),
    TPCF_KEY(S, weight_dataset_name),
    TPCF_KEY(S, jk_dataset_name),
    TPCF_KEY(B, use_weights),
    TPCF_KEY(I, n_threads),
    TPCF_KEY(I, n_jk_regions),
    TPCF_KEY(D, omega_m),
    TPCF_KEY(D, h),
    TPCF_KEY(D, z_min),
    TPCF_KEY(D, z_max),
    TPCF_KEY(B, plot_monopole),
    TPCF_KEY(S, monopole_filename),
    TPCF_KEY(S, monopole_output_type),
    TPCF_KEY(D, monopole_log_base),
    TPCF_KEY(D, monopole_min),
    TPCF_KEY(D, monopole_max),
    TPCF_KEY(I, monopole_n_bins),
    TPCF_KEY(B, plot_sigma_pi),
    TPCF_KEY(S, sigma_pi_filename),
    TPCF_KEY(S, sigma_pi_output_type),
    TPCF_KEY(D, sigma_log_base),
    TPCF_KEY(D, sigma_min),
    TPCF_KEY(D, sigma_max),
    TPCF_KEY(I, sigma_n_bins),
    TPCF_KEY(D, pi_log_base),
    TPCF_KEY(D, pi_min),
    TPCF_KEY(D, pi_max),
    TPCF_KEY(I, pi_n_bins),
    TPCF_KEY(B, plot_s_mu),
    TPCF_KEY(S, s_mu_filename),
    TPCF_KEY(S, s_mu_output_type),
    TPCF_KEY(D, s_log_base),
    TPCF_KEY(D, s_min),
    TPCF_KEY(D, s_max),
    TPCF_KEY(I, s_n_bins),
    TPCF_KEY(I, mu_n_bins),
    TPCF_KEY(B, calculate_angular_dd),
    TPCF_KEY(S, angular_dd_filename),
    TPCF_KEY(B, calculate_angular_dd_invpweights),
    TPCF_KEY(S, angular_dd_invpweights_filename),
    TPCF_KEY(B, calculate_angular_dr),
    TPCF_KEY(S, angular_dr_filename),
    TPCF_KEY(B, calculate_angular_dr_invpweights),
    TPCF_KEY(S, angular_dr_invpweights_filename),
    TPCF_KEY(D, theta_max),
    TPCF_KEY(I, theta_n_bins),
    TPCF_KEY(D, theta_log_base),
    TPCF_KEY(I, healpix_order),
    TPCF_KEY(S, bitwise_weight_dataset_name),
    TPCF_KEY(S, dither_weight_dataset_name),
    TPCF_KEY(I, n_bitwise_runs),
};
#undef TPCF_KEY

const KeyRef *find_key(const std::string &key) {
    for (const KeyRef &k : kKeys)
        if (key == k.key) return &k;
    return nullptr;
}

}  // namespace

// Params::Params (src/io.cpp:16-237).  A line is a setting when it does not
// start with '#' and contains '='; it is cut at its first '#', split at the
// first '=' into key and value, and every ' ' is removed from both (tabs and
// carriage returns stay).  n_jk_regions <= 1 becomes 1.
bool parse_params(const std::string &text, Params &p, std::string &err) {
    p = Params();
    size_t pos = 0;
    int lineno = 0;
    while (pos < text.size()) {
        size_t nl = text.find('\n', pos);
        std::string line = text.substr(pos, nl == std::string::npos ? std::string::npos : nl - pos);
        pos = nl == std::string::npos ? text.size() : nl + 1;
        ++lineno;
        if (line.empty() || line[0] == '#' || line.find('=') == std::string::npos) continue;
        line = line.substr(0, line.find('#'));
        size_t eq = line.find('=');
        std::string key = without_spaces(line.substr(0, eq));
        std::string value = eq == std::string::npos ? std::string() : without_spaces(line.substr(eq + 1));
        const KeyRef *k = find_key(key);
        if (!k) {
            p.unknown_keys.push_back(key);
            continue;
        }
        bool ok = true;
        switch (k->kind) {
        case Kind::Str:
            p.*(k->s) = value;
            break;
        case Kind::Bool: {
            int v = 0;
            ok = sto_i(value.c_str(), v);
            if (ok) p.*(k->b) = v != 0;
            break;
        }
        case Kind::Int: {
            int v = 0;
            ok = sto_i(value.c_str(), v);
            if (ok) p.*(k->i) = v;
            break;
        }
        case Kind::Dbl: {
            double v = 0;
            ok = sto_d(value.c_str(), v);
            if (ok) p.*(k->d) = v;
            break;
        }
        }
        if (!ok) {
            err = "parameter line " + std::to_string(lineno) + ": cannot convert '" + value + "' for key " + key;
            return false;
        }
    }
    if (p.n_jk_regions <= 1) p.n_jk_regions = 1;
    return true;
}

bool load_params(const std::string &path, Params &out, std::string &err) {
    std::string text;
    if (!read_file_text(path, text)) {
        err = "cannot read parameter file " + path;
        return false;
    }
    return parse_params(text, out, err);
}

bool params_get_double(const Params &p, const std::string &key, double &out) {
    const KeyRef *k = find_key(key);
    if (!k || k->kind != Kind::Dbl) return false;
    out = p.*(k->d);
    return true;
}

bool params_get_int(const Params &p, const std::string &key, int &out) {
    const KeyRef *k = find_key(key);
    if (!k) return false;
    if (k->kind == Kind::Int) out = p.*(k->i);
    else if (k->kind == Kind::Bool) out = p.*(k->b) ? 1 : 0;
    else return false;
    return true;
}

bool params_get_string(const Params &p, const std::string &key, std::string &out) {
    const KeyRef *k = find_key(key);
    if (!k || k->kind != Kind::Str) return false;
    out = p.*(k->s);
    return true;
}

namespace {

// 1 / E(z) of a flat universe, as Cosmology::codist_integrand
// (src/cosmology.cpp:7-9) evaluates it: ((a * x) * x) * x + b.
inline double inv_e(double a, double b, double one_plus_z) {
    return 1.0 / std::sqrt(a * one_plus_z * one_plus_z * one_plus_z + b);
}

}  // namespace

// The trapezoid table of src/cosmology.cpp:11-71 (comoving distance only; the
// inverted tables and luminosity distances are not used on this path).  The
// sum first runs from z = 0 up to z_min in steps of z_save_step / z_oversample
// — with the integrand's arguments swapped in its second term, as the
// reference has it (:40-44) — and is then pulled back to z_min; with
// z_min = 0 that correction cancels the first step exactly.
bool make_cosmology(double omega_m, double h, double z_min, double z_max, double z_save_step, int z_oversample,
                    CosmologyTable &c, std::string &err) {
    if (!(z_save_step > 0) || z_oversample < 1 || !std::isfinite(z_min) || !std::isfinite(z_max)) {
        err = "bad cosmology table parameters";
        return false;
    }
    double nb_d = ((z_max - z_min) / z_save_step) + 1;
    if (!(nb_d >= 1) || nb_d > 1e8) {
        err = "cosmology table: z_max must be at least z_min and the table at most 1e8 entries";
        return false;
    }
    const int numbins = (int)nb_d;
    c = CosmologyTable();
    c.omega_m = omega_m;
    c.omega_l = 1.0 - omega_m;
    c.h = h;
    c.z_min = z_min;
    c.z_max = z_max;
    c.x_step = z_save_step;
    c.x_0 = z_min;
    c.x_n = c.x_0 + (numbins - 1) * c.x_step;
    c.codist.assign(numbins, 0.0);

    const double om = c.omega_m, ol = c.omega_l;
    const double hubble_dist = 299792.458 / (h * 100.0);
    const double fine = z_save_step / (double)z_oversample;
    double z = 0.0, cur = 0.0, prev = 0.0;
    while (z <= z_min) {
        prev = cur;
        cur += inv_e(om, ol, 1.0 + z) + inv_e(ol, om, 1.0 + z + fine);
        z += fine;
    }
    cur -= ((z - z_min) / fine) * (cur - prev);
    z = z_min;
    for (int i = 0; i < numbins; ++i) {
        c.codist[i] = 0.5 * fine * hubble_dist * cur;
        for (int j = 0; j < z_oversample; ++j) {
            cur += inv_e(om, ol, 1.0 + z) + inv_e(om, ol, 1.0 + z + fine);
            z += fine;
        }
    }
    return true;
}

// DatasetFixedXY::lin_interp (src/dataset.cpp:110-126): outside the table it
// returns the table's z bounds x_0 / x_n themselves, not distances.  The index
// can reach the last entry when z sits within rounding of x_n, where the
// reference reads one past its array; here the last interval is used.
double comov_dist(const CosmologyTable &c, double z) {
    if (z <= c.x_0) return c.x_0;
    if (z >= c.x_n) return c.x_n;
    int li = (int)((z - c.x_0) / c.x_step);
    const int last = (int)c.codist.size() - 1;
    if (li >= last) li = last - 1;
    const double *y = c.codist.data();
    return y[li] + ((z - (c.x_0 + li * c.x_step)) / c.x_step) * (y[li + 1] - y[li]);
}

void galaxy_set(int64_t n, const double *ra, const double *dec, const double *d_comov, double *xyz,
                double *x_norm) {
    const double deg_to_rad = M_PI / 180.0;
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; ++i) {
        const double cd = std::cos(deg_to_rad * dec[i]);
        double u[3];
        u[0] = cd * std::cos(deg_to_rad * ra[i]);
        u[1] = cd * std::sin(deg_to_rad * ra[i]);
        u[2] = std::sin(deg_to_rad * dec[i]);
        const double d = d_comov[i];
        for (int m = 0; m < 3; ++m) {
            x_norm[3 * i + m] = u[m];
            xyz[3 * i + m] = d >= 0.0 ? d * u[m] : 0.0;
        }
    }
}

void cartesian_set(int64_t n, const double *xyz, double *d_comov, double *x_norm) {
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; ++i) {
        const double *x = xyz + 3 * i;
        const double d = std::sqrt(x[0] * x[0] + x[1] * x[1] + x[2] * x[2]);
        d_comov[i] = d;
        for (int m = 0; m < 3; ++m) x_norm[3 * i + m] = x[m] / d;
    }
}

namespace {

// Field splitting of src/io.cpp:276-322: the separator is ',' if the line
// holds one, else '\t' if it holds one, else ' '.  Each field is the next
// non-empty piece between separators (std::getline skipped over empty
// pieces), with every ' ' removed.  Running out of pieces is an error (the
// reference loops forever there).
struct FieldCursor {
    const char *p, *end;
    char sep;
    bool done = false;

    FieldCursor(const char *b, const char *e) : p(b), end(e) {
        sep = ' ';
        if (std::memchr(b, '\t', e - b)) sep = '\t';
        if (std::memchr(b, ',', e - b)) sep = ',';
    }

    // Copies the next field (spaces removed) into buf; false when none is left.
    bool next(std::string &buf) {
        while (!done) {
            const char *q = static_cast<const char *>(std::memchr(p, sep, end - p));
            const char *stop = q ? q : end;
            if (!q && p == end) {
                done = true;
                break;
            }
            const char *b = p;
            if (q) p = q + 1;
            else {
                p = end;
                done = true;
            }
            if (stop == b) continue;  // empty piece
            buf.clear();
            for (const char *c = b; c < stop; ++c)
                if (*c != ' ') buf.push_back(*c);
            return true;
        }
        return false;
    }
};

}  // namespace

// read_data_ascii (src/io.cpp:240-414).  A data line is any line that is not
// empty and does not start with '#'.  Columns: x y z (cartesian) or ra dec z
// (equatorial), then the weight when use_weights (std::stof), then the
// jackknife region when n_jk_regions > 1 (std::stoi); further columns are
// ignored.  Cartesian: d_comov = |x|, x_norm = x / d_comov.  Equatorial:
// d_comov = comov_dist(z), then Galaxy::set(ra, dec).
bool read_ascii(const std::string &path, Coords coords, bool use_weights, int n_jk_regions,
                const CosmologyTable *cosmo, HostCatalogue &out, std::string &err) {
    if (coords == Coords::Equatorial && !cosmo) {
        err = "equatorial input needs a cosmology";
        return false;
    }
    std::string text;
    if (!read_file_text(path, text)) {
        err = "cannot read catalogue file " + path;
        return false;
    }
    // Line boundaries of the data lines.
    std::vector<int64_t> starts, ends, linenos;
    {
        const char *base = text.data();
        const size_t len = text.size();
        size_t pos = 0;
        int64_t lineno = 0;
        while (pos < len) {
            const char *nl = static_cast<const char *>(std::memchr(base + pos, '\n', len - pos));
            size_t e = nl ? (size_t)(nl - base) : len;
            ++lineno;
            if (e > pos && base[pos] != '#') {
                starts.push_back((int64_t)pos);
                ends.push_back((int64_t)e);
                linenos.push_back(lineno);
            }
            pos = e + 1;
        }
    }
    const int64_t n = (int64_t)starts.size();
    out = HostCatalogue();
    out.xyz.assign(3 * n, 0.0);
    out.x_norm.assign(3 * n, 0.0);
    out.d_comov.assign(n, 0.0);
    out.weight.assign(n, 1.0f);
    out.jk_region.assign(n, 0);
    std::vector<double> ra, dec;
    if (coords == Coords::Equatorial) {
        ra.assign(n, 0.0);
        dec.assign(n, 0.0);
    }
    static const char *const kCol[2][3] = {{"x", "y", "z"}, {"ra", "dec", "z"}};
    const int ci = coords == Coords::Equatorial ? 1 : 0;
    int64_t bad = INT64_MAX;  // first failing data line
    std::string bad_msg;
#pragma omp parallel
    {
        std::string buf;
        int64_t my_bad = INT64_MAX;
        std::string my_msg;
#pragma omp for schedule(dynamic, 4096)
        for (int64_t i = 0; i < n; ++i) {
            if (i > my_bad) continue;
            FieldCursor fc(text.data() + starts[i], text.data() + ends[i]);
            const char *what = nullptr;
            const char *col = nullptr;
            double v[3];
            for (int m = 0; m < 3 && !what; ++m) {
                col = kCol[ci][m];
                if (!fc.next(buf)) what = "missing column";
                else if (!sto_d(buf.c_str(), v[m])) what = "bad number in column";
            }
            float w = 1.0f;
            if (!what && use_weights) {
                col = "weight";
                if (!fc.next(buf)) what = "missing column";
                else if (!sto_f(buf.c_str(), w)) what = "bad number in column";
            }
            int jk = 0;
            if (!what && n_jk_regions > 1) {
                col = "jk_region";
                if (!fc.next(buf)) what = "missing column";
                else if (!sto_i(buf.c_str(), jk)) what = "bad integer in column";
            }
            if (!what && coords == Coords::Equatorial && std::isnan(v[2])) {
                col = "z";
                what = "NaN in column";
            }
            if (what) {
                if (i < my_bad) {
                    my_bad = i;
                    my_msg = std::string(what) + " '" + col + "'";
                }
                continue;
            }
            out.weight[i] = w;
            out.jk_region[i] = jk;
            if (coords == Coords::Cartesian) {
                for (int m = 0; m < 3; ++m) out.xyz[3 * i + m] = v[m];
            } else {
                ra[i] = v[0];
                dec[i] = v[1];
                out.d_comov[i] = comov_dist(*cosmo, v[2]);
            }
        }
#pragma omp critical
        {
            if (my_bad < bad) {
                bad = my_bad;
                bad_msg = my_msg;
            }
        }
    }
    if (bad != INT64_MAX) {
        err = path + " line " + std::to_string(linenos[bad]) + ": " + bad_msg;
        return false;
    }
    if (coords == Coords::Cartesian) cartesian_set(n, out.xyz.data(), out.d_comov.data(), out.x_norm.data());
    else galaxy_set(n, ra.data(), dec.data(), out.d_comov.data(), out.xyz.data(), out.x_norm.data());
    return true;
}

// generate_sub_filename (src/io.cpp:628-641): the number goes before the last
// '.' of the whole path (which may be a directory's).  The reference throws
// when there is no '.'.
bool sub_filename(const std::string &filename, long long sub, std::string &out, std::string &err) {
    size_t dot = filename.find_last_of('.');
    if (dot == std::string::npos) {
        err = "output file name '" + filename + "' has no '.' to put the region number before";
        return false;
    }
    out = filename.substr(0, dot) + std::to_string(sub) + filename.substr(dot);
    return true;
}

namespace {

// std::ostream << double with the default flags and precision: printf's
// "%.6g" in the C locale.
void put_double(std::string &s, double v) {
    char b[64];
    int k = std::snprintf(b, sizeof(b), "%.*g", 6, v);
    s.append(b, k);
}

void put_int(std::string &s, int v) {
    char b[16];
    int k = std::snprintf(b, sizeof(b), "%d", v);
    s.append(b, k);
}

double ls(double dd, double dr, double rr) { return rr == 0 ? 0 : dd / rr - 2.0 * dr / rr + 1.0; }

}  // namespace

bool write_xi_ascii_single(const std::string &filename, const AxisParams &ax1, const AxisParams *ax2,
                           const double *dd, const double *dr, const double *rr, std::string &err) {
    std::string s;
    const int n1 = ax1.n_bins, n2 = ax2 ? ax2->n_bins : 1;
    s.reserve((size_t)n1 * n2 * 96);
    for (int i = 0; i < n1; ++i) {
        for (int j = 0; j < n2; ++j) {
            const int b = i * n2 + j;
            put_int(s, i);
            s += '\t';
            if (ax2) {
                put_int(s, j);
                s += '\t';
                put_double(s, axis_bin_centre(ax1, i));
                s += '\t';
                put_double(s, axis_bin_centre(*ax2, j));
                s += '\t';
                put_double(s, axis_bin_width(ax1, i));
                s += '\t';
                put_double(s, axis_bin_width(*ax2, j));
            } else {
                put_double(s, axis_bin_centre(ax1, i));
                s += '\t';
                put_double(s, axis_bin_width(ax1, i));
            }
            s += '\t';
            put_double(s, ls(dd[b], dr[b], rr[b]));
            s += '\t';
            put_double(s, dd[b]);
            s += '\t';
            put_double(s, dr[b]);
            s += '\t';
            put_double(s, rr[b]);
            s += '\n';
        }
    }
    FILE *f = std::fopen(filename.c_str(), "wb");
    if (!f) {
        err = "cannot open " + filename + " for writing";
        return false;
    }
    bool ok = std::fwrite(s.data(), 1, s.size(), f) == s.size();
    ok = (std::fclose(f) == 0) && ok;
    if (!ok) err = "write to " + filename + " failed";
    return ok;
}

}  // namespace tpcf
