// two_pcf — command-line program taking the reference's parameter file
// (src/main.cpp:11-84):
//   two_pcf <parameter file> [--fp64] [--device N] [--quiet] [--summary FILE] [--check-fp64]
// The pair counts run on the GPU; the outputs are the reference's ASCII files.
// --summary writes a JSON run summary (pairs/s, times, counts per mode);
// --check-fp64 also counts on the plain FP64 path and puts every output's
// largest difference from it in the summary (and the log).
#include <cstdio>
#include <cstdlib>
#include <cstring>

#include "../../include/two_pcf_b200.h"

int main(int argc, char **argv) {
    const char *path = nullptr;
    const char *summary = nullptr;
    int device = 0, precision = TPCF_FP32_GUARD, log = 1, check = 0;
    for (int i = 1; i < argc; ++i) {
        if (!std::strcmp(argv[i], "--fp64")) precision = TPCF_FP64;
        else if (!std::strcmp(argv[i], "--check-fp64")) check = 1;
        else if (!std::strcmp(argv[i], "--summary") && i + 1 < argc) summary = argv[++i];
        else if (!std::strcmp(argv[i], "--quiet")) log = 0;
        else if (!std::strcmp(argv[i], "--device") && i + 1 < argc) device = std::atoi(argv[++i]);
        else if (!path && argv[i][0] != '-') path = argv[i];
        else {
            path = nullptr;
            break;
        }
    }
    if (!path) {
        std::fprintf(stderr,
                     "usage: %s <parameter file> [--fp64] [--device N] [--quiet] [--summary FILE] [--check-fp64]\n",
                     argv[0]);
        return 1;
    }
    int rc = tpcf_run_param_file_report(path, device, precision, log, check, summary);
    if (rc) {
        std::fprintf(stderr, "two_pcf: %s: %s\n", tpcf_status_string(rc), tpcf_host_last_error());
        return 2;
    }
    return 0;
}
