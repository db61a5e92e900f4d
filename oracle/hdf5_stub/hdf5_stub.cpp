// TEST INFRASTRUCTURE ONLY — in-memory implementation of the HDF5 subset
// declared in hdf5.h.  Used solely when the reference sources are compiled as
// the parity oracle with _HAVE_HDF5; the product never links it.
#include "hdf5.h"

#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

const hid_t H5T_NATIVE_DOUBLE = 1;
const hid_t H5T_NATIVE_FLOAT = 2;
const hid_t H5T_NATIVE_INT = 3;
const hid_t H5T_NATIVE_LONG = 4;
const hid_t H5T_C_S1 = 5;

namespace {

struct Blob {
    hid_t type;                // one of the base type ids above
    std::vector<double> dvals; // numeric payload, converted through double
    std::vector<long long> lvals;  // exact payload for 64-bit integers
    std::string svalue;
    Blob() : type(0) {}
};

struct Group {
    std::map<std::string, std::shared_ptr<Group>> groups;
    std::map<std::string, Blob> datasets;
    std::map<std::string, Blob> attrs;
};

enum Kind { K_FILE, K_GROUP, K_DSET, K_ATTR, K_SPACE, K_TYPE };

struct Handle {
    Kind kind;
    std::shared_ptr<Group> group;  // file root or group (for K_FILE/K_GROUP), owner for K_DSET/K_ATTR
    std::string name;              // dataset / attribute name
    hid_t type;                    // base type for K_TYPE
    long long npoints;             // for K_SPACE
    Handle() : kind(K_FILE), type(0), npoints(1) {}
    Handle(Kind k, std::shared_ptr<Group> g, const std::string &n) : kind(k), group(g), name(n), type(0), npoints(1) {}
};

std::mutex g_mu;
std::map<std::string, std::shared_ptr<Group>> g_files;
std::map<hid_t, Handle> g_handles;
hid_t g_next = 100;

hid_t new_handle(const Handle &h) {
    hid_t id = g_next++;
    g_handles[id] = h;
    return id;
}

Handle *get(hid_t id) {
    auto it = g_handles.find(id);
    return it == g_handles.end() ? nullptr : &it->second;
}

hid_t base_type(hid_t t) {
    if (t >= 1 && t <= 5) return t;
    Handle *h = get(t);
    return (h && h->kind == K_TYPE) ? h->type : 0;
}

void store(Blob &b, hid_t mem_type, const void *buf, long long n) {
    hid_t t = base_type(mem_type);
    if (b.type == 0) b.type = t;
    b.dvals.assign(n, 0.0);
    b.lvals.assign(n, 0);
    for (long long i = 0; i < n; ++i) {
        switch (t) {
        case 1: b.dvals[i] = ((const double *)buf)[i]; break;
        case 2: b.dvals[i] = ((const float *)buf)[i]; break;
        case 3: b.lvals[i] = ((const int *)buf)[i]; b.dvals[i] = (double)b.lvals[i]; break;
        case 4: b.lvals[i] = ((const long *)buf)[i]; b.dvals[i] = (double)b.lvals[i]; break;
        case 5: b.svalue = std::string((const char *)buf); break;
        }
    }
    // Values are kept with the precision of the declared (file) type.
    if (b.type == 2)
        for (auto &v : b.dvals) v = (double)(float)v;
}

void load(const Blob &b, hid_t mem_type, void *buf) {
    hid_t t = base_type(mem_type);
    long long n = (long long)b.dvals.size();
    bool integral = (b.type == 3 || b.type == 4);
    for (long long i = 0; i < n; ++i) {
        switch (t) {
        case 1: ((double *)buf)[i] = b.dvals[i]; break;
        case 2: ((float *)buf)[i] = (float)b.dvals[i]; break;
        case 3: ((int *)buf)[i] = integral ? (int)b.lvals[i] : (int)b.dvals[i]; break;
        case 4: ((long *)buf)[i] = integral ? (long)b.lvals[i] : (long)b.dvals[i]; break;
        }
    }
    if (t == 5) std::strcpy((char *)buf, b.svalue.c_str());
}

}  // namespace

hid_t H5Fopen(const char *name, unsigned, hid_t) {
    std::lock_guard<std::mutex> lk(g_mu);
    auto it = g_files.find(name);
    if (it == g_files.end()) return -1;
    return new_handle(Handle(K_FILE, it->second, name));
}

hid_t H5Fcreate(const char *name, unsigned, hid_t, hid_t) {
    std::lock_guard<std::mutex> lk(g_mu);
    auto root = std::make_shared<Group>();
    g_files[name] = root;  // H5F_ACC_TRUNC semantics
    return new_handle(Handle(K_FILE, root, name));
}

herr_t H5Fclose(hid_t f) { std::lock_guard<std::mutex> lk(g_mu); g_handles.erase(f); return 0; }

hid_t H5Gopen(hid_t loc, const char *name, hid_t) {
    std::lock_guard<std::mutex> lk(g_mu);
    Handle *h = get(loc);
    if (!h) return -1;
    auto it = h->group->groups.find(name);
    if (it == h->group->groups.end()) return -1;
    return new_handle(Handle(K_GROUP, it->second, name));
}

hid_t H5Gcreate2(hid_t loc, const char *name, hid_t, hid_t, hid_t) {
    std::lock_guard<std::mutex> lk(g_mu);
    Handle *h = get(loc);
    if (!h) return -1;
    auto g = std::make_shared<Group>();
    h->group->groups[name] = g;
    return new_handle(Handle(K_GROUP, g, name));
}

herr_t H5Gclose(hid_t g) { std::lock_guard<std::mutex> lk(g_mu); g_handles.erase(g); return 0; }

hid_t H5Dopen2(hid_t loc, const char *name, hid_t) {
    std::lock_guard<std::mutex> lk(g_mu);
    Handle *h = get(loc);
    if (!h || !h->group->datasets.count(name)) return -1;
    return new_handle(Handle(K_DSET, h->group, name));
}

hid_t H5Dcreate2(hid_t loc, const char *name, hid_t type, hid_t space, hid_t, hid_t, hid_t) {
    std::lock_guard<std::mutex> lk(g_mu);
    Handle *h = get(loc);
    Handle *s = get(space);
    if (!h) return -1;
    Blob b;
    b.type = base_type(type);
    b.dvals.assign(s ? s->npoints : 1, 0.0);
    h->group->datasets[name] = b;
    return new_handle(Handle(K_DSET, h->group, name));
}

herr_t H5Dread(hid_t dset, hid_t mem_type, hid_t, hid_t, hid_t, void *buf) {
    std::lock_guard<std::mutex> lk(g_mu);
    Handle *h = get(dset);
    if (!h) return -1;
    load(h->group->datasets[h->name], mem_type, buf);
    return 0;
}

herr_t H5Dwrite(hid_t dset, hid_t mem_type, hid_t, hid_t, hid_t, const void *buf) {
    std::lock_guard<std::mutex> lk(g_mu);
    Handle *h = get(dset);
    if (!h) return -1;
    Blob &b = h->group->datasets[h->name];
    store(b, mem_type, buf, (long long)b.dvals.size());
    return 0;
}

hid_t H5Dget_space(hid_t dset) {
    std::lock_guard<std::mutex> lk(g_mu);
    Handle *h = get(dset);
    if (!h) return -1;
    Handle s(K_SPACE, nullptr, "");
    s.npoints = (long long)h->group->datasets[h->name].dvals.size();
    return new_handle(s);
}

herr_t H5Dclose(hid_t d) { std::lock_guard<std::mutex> lk(g_mu); g_handles.erase(d); return 0; }

hid_t H5Screate(H5S_class_t) {
    std::lock_guard<std::mutex> lk(g_mu);
    Handle s(K_SPACE, nullptr, "");
    s.npoints = 1;
    return new_handle(s);
}

hid_t H5Screate_simple(int rank, const hsize_t *dims, const hsize_t *) {
    std::lock_guard<std::mutex> lk(g_mu);
    Handle s(K_SPACE, nullptr, "");
    s.npoints = 1;
    for (int i = 0; i < rank; ++i) s.npoints *= (long long)dims[i];
    return new_handle(s);
}

hssize_t H5Sget_simple_extent_npoints(hid_t space) {
    std::lock_guard<std::mutex> lk(g_mu);
    Handle *h = get(space);
    return h ? h->npoints : -1;
}

herr_t H5Sclose(hid_t s) { std::lock_guard<std::mutex> lk(g_mu); g_handles.erase(s); return 0; }

hid_t H5Aopen(hid_t obj, const char *name, hid_t) {
    std::lock_guard<std::mutex> lk(g_mu);
    Handle *h = get(obj);
    if (!h || !h->group->attrs.count(name)) return -1;
    return new_handle(Handle(K_ATTR, h->group, name));
}

hid_t H5Acreate2(hid_t loc, const char *name, hid_t type, hid_t, hid_t, hid_t) {
    std::lock_guard<std::mutex> lk(g_mu);
    Handle *h = get(loc);
    if (!h) return -1;
    Blob b;
    b.type = base_type(type);
    b.dvals.assign(1, 0.0);
    h->group->attrs[name] = b;
    return new_handle(Handle(K_ATTR, h->group, name));
}

herr_t H5Aread(hid_t attr, hid_t mem_type, void *buf) {
    std::lock_guard<std::mutex> lk(g_mu);
    Handle *h = get(attr);
    if (!h) return -1;
    load(h->group->attrs[h->name], mem_type, buf);
    return 0;
}

herr_t H5Awrite(hid_t attr, hid_t mem_type, const void *buf) {
    std::lock_guard<std::mutex> lk(g_mu);
    Handle *h = get(attr);
    if (!h) return -1;
    store(h->group->attrs[h->name], mem_type, buf, 1);
    return 0;
}

herr_t H5Aclose(hid_t a) { std::lock_guard<std::mutex> lk(g_mu); g_handles.erase(a); return 0; }

hid_t H5Tcopy(hid_t type) {
    std::lock_guard<std::mutex> lk(g_mu);
    Handle t(K_TYPE, nullptr, "");
    t.type = base_type(type);
    return new_handle(t);
}

herr_t H5Tset_order(hid_t, H5T_order_t) { return 0; }

void h5stub_reset(void) {
    std::lock_guard<std::mutex> lk(g_mu);
    g_files.clear();
    g_handles.clear();
}
