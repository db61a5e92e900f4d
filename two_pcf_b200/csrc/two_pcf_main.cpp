// two_pcf — command-line program taking the reference's parameter file
// (src/main.cpp:11-84): `two_pcf <parameter file> [--fp64] [--device N] [--quiet]`.
// The pair counts run on the GPU; the outputs are the reference's ASCII files.
#include <cstdio>
#include <cstdlib>
#include <cstring>

#include "../../include/two_pcf_b200.h"

int main(int argc, char **argv) {
    const char *path = nullptr;
    int device = 0, precision = TPCF_FP32_GUARD, log = 1;
    for (int i = 1; i < argc; ++i) {
        if (!std::strcmp(argv[i], "--fp64")) precision = TPCF_FP64;
        else if (!std::strcmp(argv[i], "--quiet")) log = 0;
        else if (!std::strcmp(argv[i], "--device") && i + 1 < argc) device = std::atoi(argv[++i]);
        else if (!path && argv[i][0] != '-') path = argv[i];
        else {
            path = nullptr;
            break;
        }
    }
    if (!path) {
        std::fprintf(stderr, "usage: %s <parameter file> [--fp64] [--device N] [--quiet]\n", argv[0]);
        return 1;
    }
    int rc = tpcf_run_param_file(path, device, precision, log);
    if (rc) {
        std::fprintf(stderr, "two_pcf: %s: %s\n", tpcf_status_string(rc), tpcf_host_last_error());
        return 2;
    }
    return 0;
}
