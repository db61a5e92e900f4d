// The opaque handle types of include/two_pcf_b200.h, shared by the C ABI
// translation units.
#pragma once
#include "../../include/two_pcf_b200.h"
#include "engine.h"
#include "ingest.h"

struct tpcf_ctx {
    tpcf::Ctx c;
};
struct tpcf_catalog {
    tpcf::Catalog c;
};
struct tpcf_binning {
    tpcf::Binning b;
};
struct tpcf_batch {
    tpcf_ctx *ctx = nullptr;
    tpcf::Batch *b = nullptr;
    ~tpcf_batch() {
        if (b) tpcf::batch_destroy(b);
    }
};
struct tpcf_params {
    tpcf::Params p;
};
struct tpcf_cosmology {
    tpcf::CosmologyTable t;
};
struct tpcf_host_catalog {
    tpcf::HostCatalogue c;
};
