// Entry points with the reference's own argument lists:
//   fast_sum              fast_sum_module.f90:291-332
//   proxy_source_compute  mom6_fast_sum_module.f90:33-74
//   pc_compute            mom6_fast_sum_module.f90:153-174
//   pp_compute            mom6_fast_sum_module.f90:177-192
// The reference recomputes everything on every call.  Here each call hashes
// its set-up arguments (coordinates, areas, the flattened cube_panel array,
// the interaction list, the degree) and reuses a device grid built earlier for
// the same contents, so a caller that changes any of them gets a new grid and
// never a stale one.  Only the per-call data (SSH, proxy weights) is copied per
// call.
#include <algorithm>
#include <cstdint>
#include <cstring>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/salgpu.h"
#include "sal_internal.hpp"

namespace sal {
int set_error(int code, const std::string &msg);  // capi.cpp
}

using namespace sal;

struct sal_tree : Tree {};

namespace {

// ------------------------------------------------------------------ content hash
inline uint64_t rotl(uint64_t x, int r) { return (x << r) | (x >> (64 - r)); }
inline uint64_t fmix(uint64_t h) {
    h ^= h >> 33;
    h *= 0xff51afd7ed558ccdULL;
    h ^= h >> 33;
    h *= 0xc4ceb9fe1a85ec53ULL;
    h ^= h >> 33;
    return h;
}

// 64-bit hash of a byte range: blocks of 1 MiB hashed in parallel, their
// hashes combined in block order (the result does not depend on the thread
// count).  Inside a block, four independent lanes take 8 bytes each per step,
// so the multiply chains overlap.
uint64_t hash_bytes(const void *p, size_t n) {
    constexpr size_t kBlock = 1 << 20;
    const unsigned char *b = static_cast<const unsigned char *>(p);
    const int64_t nb = (int64_t)((n + kBlock - 1) / kBlock);
    std::vector<uint64_t> hb((size_t)std::max<int64_t>(nb, 1), 0);
#pragma omp parallel for schedule(static) if (nb > 4)
    for (int64_t k = 0; k < nb; ++k) {
        const size_t lo = (size_t)k * kBlock, hi = std::min(n, lo + kBlock);
        uint64_t h[4];
        for (int l = 0; l < 4; ++l) h[l] = 0x9E3779B97F4A7C15ULL * (uint64_t)(4 * k + l + 1);
        size_t i = lo;
        for (; i + 32 <= hi; i += 32) {
            uint64_t w[4];
            std::memcpy(w, b + i, 32);
            for (int l = 0; l < 4; ++l) h[l] = rotl(h[l] ^ (w[l] * 0x87c37b91114253d5ULL), 31) * 0x4cf5ad432745937fULL;
        }
        for (; i + 8 <= hi; i += 8) {
            uint64_t w;
            std::memcpy(&w, b + i, 8);
            h[0] = rotl(h[0] ^ (w * 0x87c37b91114253d5ULL), 31) * 0x4cf5ad432745937fULL;
        }
        uint64_t t = 0;
        for (size_t j = 0; i < hi; ++i, ++j) t |= (uint64_t)b[i] << (8 * j);
        hb[(size_t)k] = fmix(fmix(h[0] ^ rotl(h[1], 17)) ^ fmix(h[2] ^ rotl(h[3], 29)) ^ t ^ (uint64_t)(hi - lo));
    }
    uint64_t h = (uint64_t)n;
    for (uint64_t v : hb) h = fmix(h ^ v) + 0x2545F4914F6CDD1DULL;
    return h;
}

struct Key {
    uint64_t h = 0xcbf29ce484222325ULL;
    void add_bytes(const void *p, size_t n) { h = fmix(h ^ hash_bytes(p, n)) ^ rotl(h, 17); }
    void add(int64_t v) { h = fmix(h ^ (uint64_t)v * 0x9E3779B97F4A7C15ULL) ^ rotl(h, 23); }
};

// The flattened cube_panel array of sal_tree_import.
struct Panels {
    int32_t np;
    const int32_t *ints9;
    const double *dbl7;
    const int64_t *pt_off;
    const int32_t *pt_idx;   // may be null
    void hash_into(Key &k) const {
        k.add(np);
        k.add_bytes(ints9, (size_t)np * 9 * sizeof(int32_t));
        k.add_bytes(dbl7, (size_t)np * 7 * sizeof(double));
        k.add_bytes(pt_off, (size_t)(np + 1) * sizeof(int64_t));
        k.add(pt_idx != nullptr);
        if (pt_idx) k.add_bytes(pt_idx, (size_t)pt_off[np] * sizeof(int32_t));
    }
};

int check_panels(const Panels &P) {
    if (!P.ints9 || !P.dbl7 || !P.pt_off) return set_error(SAL_EINVAL, "null panel arrays");
    if (P.np < 6) return set_error(SAL_EINVAL, "a cubed-sphere tree has at least 6 panels");
    return SAL_OK;
}

// The caller's tree as a sal_tree.  With points_inside (pt_idx) it is
// imported; without, it is rebuilt from the coordinates with a cluster
// threshold read off the panel counts (leaves hold fewer points than the
// threshold, refined panels at least as many: tree_module.f90:130) and must
// then equal the caller's panels field for field.
int make_tree(const Panels &P, int32_t n, const double *xs, const double *ys, const double *zs, sal_tree **out) {
    *out = nullptr;
    std::string err;
    if (P.pt_idx) {
        Tree *t = tree_import(P.np, P.ints9, P.dbl7, P.pt_off, P.pt_idx, n, xs, ys, zs, &err);
        if (!t) return set_error(SAL_EINVAL, err);
        sal_tree *s = new sal_tree();
        static_cast<Tree &>(*s) = std::move(*t);
        delete t;
        *out = s;
        return SAL_OK;
    }
    int64_t max_leaf = 0, min_inner = INT64_MAX;
    for (int32_t k = 0; k < P.np; ++k) {
        const int64_t c = P.pt_off[k + 1] - P.pt_off[k];
        if (P.ints9[9 * k + 1]) max_leaf = std::max(max_leaf, c);
        else min_inner = std::min(min_inner, c);
    }
    const int64_t thresh = std::max<int64_t>(2, max_leaf + 1);
    if (thresh > min_inner || thresh > INT32_MAX)
        return set_error(SAL_ETREE, "the panel counts fit no cluster threshold; pass points_inside");
    Tree *t = tree_build(xs, ys, zs, n, (int32_t)thresh);
    std::unique_ptr<Tree> own(t);
    bool same = (int32_t)t->p.size() == P.np;
    for (int32_t k = 0; same && k < P.np; ++k) {
        const Panel &q = t->p[k];
        const int32_t I[9] = {q.level, q.is_leaf, q.id, q.parent, q.child[0], q.child[1], q.child[2], q.child[3], q.face};
        const double D[7] = {q.min_xi, q.mid_xi, q.max_xi, q.min_eta, q.mid_eta, q.max_eta, q.radius};
        same = std::memcmp(I, P.ints9 + 9 * (size_t)k, sizeof(I)) == 0 &&
               std::memcmp(D, P.dbl7 + 7 * (size_t)k, sizeof(D)) == 0 &&
               q.count() == P.pt_off[k + 1] - P.pt_off[k];
    }
    if (!same)
        return set_error(SAL_ETREE, "the panels differ from the tree of these coordinates; pass points_inside");
    sal_tree *s = new sal_tree();
    static_cast<Tree &>(*s) = std::move(*t);
    *out = s;
    return SAL_OK;
}

// ------------------------------------------------------------------ grid caches
struct Entry {
    uint64_t key;
    sal_grid *grid;
    uint64_t used;
};

struct Cache {
    std::vector<Entry> v;
    static constexpr size_t kCap = 4;   // grids kept per entry point, least recently used dropped
};

std::mutex g_mu;                          // guards the caches and the settings
Cache g_fast, g_up, g_pc, g_pp;
uint64_t g_tick = 0;
int32_t g_form = SAL_FORM_REF;
int32_t g_mom6_mode = SAL_MODE_STT_REF_COMPAT;

sal_grid *lookup(Cache &c, uint64_t key) {
    for (auto &e : c.v)
        if (e.key == key) {
            e.used = ++g_tick;
            return e.grid;
        }
    return nullptr;
}

void insert(Cache &c, uint64_t key, sal_grid *g) {
    if (c.v.size() >= Cache::kCap) {
        auto it = std::min_element(c.v.begin(), c.v.end(), [](const Entry &a, const Entry &b) { return a.used < b.used; });
        sal_grid_destroy(it->grid);
        c.v.erase(it);
    }
    c.v.push_back({key, g, ++g_tick});
}

int current_device(int *dev) {
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) return set_error(SAL_ENODEV, "no CUDA device is available");
    if (cudaGetDevice(dev) != cudaSuccess) return set_error(SAL_ENODEV, "no current CUDA device");
    return SAL_OK;
}

// Builds a grid from the caller's panels and points (a tree made for it and
// dropped once the grid holds its own flattened copy).
int build_grid(const Panels &P, int32_t n, const double *xs, const double *ys, const double *zs, const double *areas,
               sal_grid_desc d, sal_grid **out) {
    sal_tree *t = nullptr;
    int rc = make_tree(P, n, xs, ys, zs, &t);
    if (rc) return rc;
    std::unique_ptr<sal_tree> own(t);
    d.point_count = n;
    d.xs = xs;
    d.ys = ys;
    d.zs = zs;
    d.areas = areas;
    rc = current_device(&d.device);
    if (rc) return rc;
    return sal_grid_create(t, &d, out);
}

}  // namespace

extern "C" int sal_dropin_config(int32_t form, int32_t mom6_mode) {
    if (form != SAL_FORM_REF && form != SAL_FORM_ACCURATE)
        return set_error(SAL_EINVAL, "fast_sum runs SAL_FORM_REF or SAL_FORM_ACCURATE");
    if (mom6_mode != SAL_MODE_STT_REF_COMPAT && mom6_mode != SAL_MODE_STT_CORRECT)
        return set_error(SAL_EINVAL, "mom6_mode is SAL_MODE_STT_REF_COMPAT or SAL_MODE_STT_CORRECT");
    std::lock_guard<std::mutex> lk(g_mu);
    if (mom6_mode != g_mom6_mode) {
        // weights already built in the other orientation must not be reused
        for (auto &e : g_up.v) sal_grid_destroy(e.grid);
        g_up.v.clear();
    }
    g_form = form;
    g_mom6_mode = mom6_mode;
    return SAL_OK;
}

extern "C" int sal_dropin_release(void) {
    std::lock_guard<std::mutex> lk(g_mu);
    for (Cache *c : {&g_fast, &g_up, &g_pc, &g_pp}) {
        for (auto &e : c->v) sal_grid_destroy(e.grid);
        c->v.clear();
    }
    return SAL_OK;
}

extern "C" int sal_fast_sum(double *sal_longrad, double *sal_latgrad, const int32_t *interaction_list,
                            int64_t list_count, int32_t npanels, const int32_t *ints9, const double *dbl7,
                            const int64_t *pt_off, const int32_t *pt_idx, const double *xs, const double *ys,
                            const double *zs, const double *area, const double *ssh, int32_t point_count,
                            int32_t interp_degree, int32_t rank, int32_t process_count) {
    if (!sal_longrad || !sal_latgrad || !xs || !ys || !zs || !area || !ssh || (list_count > 0 && !interaction_list))
        return set_error(SAL_EINVAL, "null argument");
    if (point_count < 0 || list_count < 0) return set_error(SAL_EINVAL, "negative size");
    if (process_count < 1 || rank < 0 || rank >= process_count) return set_error(SAL_EINVAL, "rank out of range");
    const Panels P{npanels, ints9, dbl7, pt_off, pt_idx};
    int rc = check_panels(P);
    if (rc) return rc;
    Key k;
    P.hash_into(k);
    for (const double *a : {xs, ys, zs, area}) k.add_bytes(a, (size_t)point_count * sizeof(double));
    k.add_bytes(interaction_list, (size_t)list_count * 3 * sizeof(int32_t));
    k.add(point_count);
    k.add(interp_degree);
    k.add(rank);
    k.add(process_count);
    std::lock_guard<std::mutex> lk(g_mu);
    sal_grid *g = lookup(g_fast, k.h);
    if (!g) {
        // the MPI split MOD(i, P) == rank of fast_sum_module.f90:304, i 1-based
        std::vector<int32_t> mine;
        mine.reserve((size_t)(list_count / process_count + 1) * 3);
        for (int64_t i = 1; i <= list_count; ++i)
            if (i % process_count == rank) mine.insert(mine.end(), interaction_list + 3 * (i - 1), interaction_list + 3 * i);
        sal_grid_desc d{};
        d.interp_degree = interp_degree;
        d.mode = SAL_MODE_DTT;
        d.list = mine.data();
        d.list_count = (int64_t)mine.size() / 3;
        d.max_fields = 1;
        rc = build_grid(P, point_count, xs, ys, zs, area, d, &g);
        if (rc) return rc;
        insert(g_fast, k.h, g);
    }
    return sal_fast_sum_host(g, ssh, sal_longrad, sal_latgrad, g_form);
}

extern "C" int sal_mom6_proxy_source_compute(double *proxy_source_weights, int32_t npanels, const int32_t *ints9,
                                             const double *dbl7, const int64_t *pt_off, const int32_t *pt_idx,
                                             const int32_t *points_panels, int32_t nlev, const double *xs,
                                             const double *ys, const double *zs, const double *sshs,
                                             const double *areas, int32_t interp_degree, int32_t point_count) {
    if (!proxy_source_weights || !points_panels || !xs || !ys || !zs || !sshs || !areas)
        return set_error(SAL_EINVAL, "null argument");
    if (point_count < 0 || nlev < 1) return set_error(SAL_EINVAL, "bad sizes");
    const Panels P{npanels, ints9, dbl7, pt_off, pt_idx};
    int rc = check_panels(P);
    if (rc) return rc;
    Key k;
    P.hash_into(k);
    for (const double *a : {xs, ys, zs, areas}) k.add_bytes(a, (size_t)point_count * sizeof(double));
    k.add_bytes(points_panels, (size_t)point_count * (size_t)nlev * sizeof(int32_t));
    k.add(point_count);
    k.add(nlev);
    k.add(interp_degree);
    std::lock_guard<std::mutex> lk(g_mu);
    k.add(g_mom6_mode);
    sal_grid *g = lookup(g_up, k.h);
    if (!g) {
        sal_grid_desc d{};
        d.interp_degree = interp_degree;
        d.mode = g_mom6_mode;
        d.max_fields = 1;
        sal_tree *t = nullptr;
        rc = make_tree(P, point_count, xs, ys, zs, &t);
        if (rc) return rc;
        std::unique_ptr<sal_tree> own(t);
        // the weights are summed over each point's panels as points_panels
        // lists them (mom6_fast_sum_module.f90:52-72); the grid sums over the
        // tree's own panel ranges, so the two must agree
        if (nlev < t->max_level() + 1) return set_error(SAL_EINVAL, "points_panels has fewer levels than the tree");
        std::vector<int32_t> mine((size_t)point_count * (size_t)nlev, -1);
        if (assign_points_to_panels(*t, xs, ys, zs, point_count, mine.data(), nlev) != 0 ||
            std::memcmp(mine.data(), points_panels, mine.size() * sizeof(int32_t)) != 0)
            return set_error(SAL_EINVAL, "points_panels does not match the panels (tree_module.f90:249-273)");
        d.point_count = point_count;
        d.xs = xs;
        d.ys = ys;
        d.zs = zs;
        d.areas = areas;
        rc = current_device(&d.device);
        if (rc) return rc;
        rc = sal_grid_create(t, &d, &g);
        if (rc) return rc;
        insert(g_up, k.h, g);
    }
    return sal_proxy_source_compute_host(g, sshs, proxy_source_weights);
}

extern "C" int sal_mom6_pc_compute(double *sal_longrad, double *sal_latgrad, const int32_t *pc_interaction_list,
                                   int64_t pc_count, int32_t npanels, const int32_t *ints9, const double *dbl7,
                                   const int64_t *pt_off, const int32_t *pt_idx, const double *xs, const double *ys,
                                   const double *zs, int32_t point_count, int32_t interp_degree,
                                   const double *proxy_weights) {
    if (!sal_longrad || !sal_latgrad || !xs || !ys || !zs || !proxy_weights || (pc_count > 0 && !pc_interaction_list))
        return set_error(SAL_EINVAL, "null argument");
    if (point_count < 0 || pc_count < 0) return set_error(SAL_EINVAL, "negative size");
    const Panels P{npanels, ints9, dbl7, pt_off, pt_idx};
    int rc = check_panels(P);
    if (rc) return rc;
    Key k;
    P.hash_into(k);
    for (const double *a : {xs, ys, zs}) k.add_bytes(a, (size_t)point_count * sizeof(double));
    k.add_bytes(pc_interaction_list, (size_t)pc_count * 2 * sizeof(int32_t));
    k.add(point_count);
    k.add(interp_degree);
    std::lock_guard<std::mutex> lk(g_mu);
    sal_grid *g = lookup(g_pc, k.h);
    if (!g) {
        // pc_compute reads no areas: the grid's point weights are never used
        const std::vector<double> zero((size_t)point_count, 0.0);
        sal_grid_desc d{};
        d.interp_degree = interp_degree;
        d.mode = SAL_MODE_STT_REF_COMPAT;
        d.pc_list = pc_interaction_list;
        d.pc_count = pc_count;
        d.max_fields = 1;
        rc = build_grid(P, point_count, xs, ys, zs, zero.data(), d, &g);
        if (rc) return rc;
        insert(g_pc, k.h, g);
    }
    return sal_pc_compute_host(g, proxy_weights, sal_longrad, sal_latgrad);
}

extern "C" int sal_mom6_pp_compute(double *sal_longrad, double *sal_latgrad, const int32_t *pp_interaction_list,
                                   int64_t pp_count, int32_t npanels, const int32_t *ints9, const double *dbl7,
                                   const int64_t *pt_off, const int32_t *pt_idx, const double *xs, const double *ys,
                                   const double *zs, const double *areas, const double *sshs, const double *e_xs,
                                   const double *e_ys, const double *e_zs, const double *e_areas, const double *e_sshs,
                                   int32_t extra_count, int32_t own_points) {
    (void)e_xs; (void)e_ys; (void)e_zs; (void)e_areas; (void)e_sshs;
    if (!sal_longrad || !sal_latgrad || !xs || !ys || !zs || !areas || !sshs || (pp_count > 0 && !pp_interaction_list))
        return set_error(SAL_EINVAL, "null argument");
    if (own_points < 0 || pp_count < 0) return set_error(SAL_EINVAL, "negative size");
    if (extra_count != 0)
        return set_error(SAL_EINVAL, "halo points of other MPI ranks (e_xs ...) are not supported: the GPU path "
                                     "solves the whole grid on one rank");
    const Panels P{npanels, ints9, dbl7, pt_off, pt_idx};
    int rc = check_panels(P);
    if (rc) return rc;
    Key k;
    P.hash_into(k);
    for (const double *a : {xs, ys, zs, areas}) k.add_bytes(a, (size_t)own_points * sizeof(double));
    k.add_bytes(pp_interaction_list, (size_t)pp_count * 2 * sizeof(int32_t));
    k.add(own_points);
    std::lock_guard<std::mutex> lk(g_mu);
    sal_grid *g = lookup(g_pp, k.h);
    if (!g) {
        sal_grid_desc d{};
        d.interp_degree = 1;   // pp_compute has no proxies
        d.mode = SAL_MODE_STT_REF_COMPAT;
        d.pp_list = pp_interaction_list;
        d.pp_count = pp_count;
        d.max_fields = 1;
        rc = build_grid(P, own_points, xs, ys, zs, areas, d, &g);
        if (rc) return rc;
        insert(g_pp, k.h, g);
    }
    return sal_pp_compute_host(g, sshs, sal_longrad, sal_latgrad);
}
