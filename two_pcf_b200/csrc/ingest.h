// Host side of the reference's command-line flow: the parameter file, the
// redshift -> comoving distance table, the catalogue readers and the ASCII
// result writers (src/io.cpp, src/cosmology.cpp, src/dataset.cpp,
// src/galaxy.cpp).  Everything here is plain host C++ compiled with
// -ffp-contract=off, so each double/float operation rounds once as in the
// reference's x86-64 build and the outputs match it bit for bit.
#pragma once
#include <cstdint>
#include <string>
#include <vector>

#include "axis.h"

namespace tpcf {

// Every key the reference's Params constructor recognises (src/io.h:10-83,
// src/io.cpp:16-237).  Fields the file does not set keep these defaults (the
// reference leaves them uninitialised).
struct Params {
    std::string data_filename, data_file_type, random_filename, random_file_type, coord_system;
    std::string ra_x_dataset_name, dec_y_dataset_name, z_z_dataset_name, weight_dataset_name, jk_dataset_name;
    bool use_weights = false;
    int n_threads = 0;
    int n_jk_regions = 1;
    double omega_m = 0, h = 0, z_min = 0, z_max = 0;

    bool plot_monopole = false;
    std::string monopole_filename, monopole_output_type;
    double monopole_log_base = 0, monopole_min = 0, monopole_max = 0;
    int monopole_n_bins = 0;

    bool plot_sigma_pi = false;
    std::string sigma_pi_filename, sigma_pi_output_type;
    double sigma_log_base = 0, sigma_min = 0, sigma_max = 0;
    int sigma_n_bins = 0;
    double pi_log_base = 0, pi_min = 0, pi_max = 0;
    int pi_n_bins = 0;

    bool plot_s_mu = false;
    std::string s_mu_filename, s_mu_output_type;
    double s_log_base = 0, s_min = 0, s_max = 0;
    int s_n_bins = 0, mu_n_bins = 0;

    bool calculate_angular_dd = false, calculate_angular_dd_invpweights = false;
    bool calculate_angular_dr = false, calculate_angular_dr_invpweights = false;
    std::string angular_dd_filename, angular_dd_invpweights_filename, angular_dr_filename,
        angular_dr_invpweights_filename;
    double theta_max = 0;
    int theta_n_bins = 0;
    double theta_log_base = 0;
    int healpix_order = 0;
    std::string bitwise_weight_dataset_name, dither_weight_dataset_name;
    int n_bitwise_runs = 0;

    // Keys seen but not recognised, in file order (the reference prints
    // "KEY NOT FOUND" for each and carries on).
    std::vector<std::string> unknown_keys;
};

// Parses parameter-file text with the reference's line rules.  Returns false
// with a message where the reference's std::stoi / std::stod would throw.
bool parse_params(const std::string &text, Params &out, std::string &err);
bool load_params(const std::string &path, Params &out, std::string &err);

// Numeric and string fields by key name (the parameter-file spelling).
bool params_get_double(const Params &p, const std::string &key, double &out);
bool params_get_int(const Params &p, const std::string &key, int &out);
bool params_get_string(const Params &p, const std::string &key, std::string &out);

// The z -> comoving distance table of Cosmology (src/cosmology.cpp:11-71)
// and its lookup DatasetFixedXY::lin_interp (src/dataset.cpp:99-126).
struct CosmologyTable {
    double omega_m = 0, omega_l = 0, h = 0, z_min = 0, z_max = 0;
    double x_step = 0, x_0 = 0, x_n = 0;  // the table's z grid
    std::vector<double> codist;           // comoving distance at z_min + i * x_step
};
bool make_cosmology(double omega_m, double h, double z_min, double z_max, double z_save_step, int z_oversample,
                    CosmologyTable &out, std::string &err);
double comov_dist(const CosmologyTable &c, double z);

// Galaxy::set (src/galaxy.cpp:8-27) and the cartesian reader's transform
// (src/io.cpp:393-399), over arrays, in parallel.
void galaxy_set(int64_t n, const double *ra, const double *dec, const double *d_comov, double *xyz,
                double *x_norm);
void cartesian_set(int64_t n, const double *xyz, double *d_comov, double *x_norm);

// A catalogue as the reference's readers leave it in GalaxyCatalogue, as
// structure-of-arrays.
struct HostCatalogue {
    std::vector<double> xyz, x_norm, d_comov;  // 3n, 3n, n
    std::vector<float> weight;                 // n
    std::vector<int32_t> jk_region;            // n
    int64_t size() const { return (int64_t)d_comov.size(); }
};

enum class Coords { Cartesian, Equatorial };

// read_data_ascii (src/io.cpp:240-414), parsing lines in parallel.
bool read_ascii(const std::string &path, Coords coords, bool use_weights, int n_jk_regions,
                const CosmologyTable *cosmo, HostCatalogue &out, std::string &err);

// generate_sub_filename (src/io.cpp:628-641).
bool sub_filename(const std::string &filename, long long sub, std::string &out, std::string &err);

// output_single_xi_1D_ascii / output_single_xi_2D_ascii (src/io.cpp:724-740,
// :832-853): one file of bins, centres, widths, xi and the three counts.
// ax2 == nullptr selects the 1-D layout.
bool write_xi_ascii_single(const std::string &filename, const AxisParams &ax1, const AxisParams *ax2,
                           const double *dd, const double *dr, const double *rr, std::string &err);

// The message tpcf_host_last_error() returns on this thread.
void set_host_error(const std::string &msg);

}  // namespace tpcf
