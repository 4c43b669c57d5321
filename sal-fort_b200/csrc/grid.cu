// Device-resident grids and the solve entry points of the C ABI.
#include <cuda_runtime.h>

#include <chrono>
#include <cmath>
#include <algorithm>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/salgpu.h"
#include "kernels.cuh"
#include "mixed.cuh"
#include "sal_internal.hpp"

namespace sal {
int set_error(int code, const std::string &msg);  // capi.cpp
}

using namespace sal;

namespace {

template <class T>
struct DBuf {
    T *p = nullptr;
    size_t n = 0;
};

struct GridImpl {
    int dev = 0;
    Plan plan;
    Tree tree;                        // kept to re-cut the tcgen05 plan (sal_grid_tune)
    cudaStream_t stream = nullptr;
    int64_t bytes = 0;
    double setup_seconds = 0;
    int nsrc = 0, ntgt = 0, rec_stride = 0, nup = 0, nproxy_units = 0;
    // device arrays
    double4 *xyz = nullptr;       // pool order x, y, z (w unused)
    double *area = nullptr;
    double2 *xieta = nullptr;
    int32_t *perm = nullptr;
    double4 *pool = nullptr;      // n points + nsrc*P proxies
    Group *leaf_groups = nullptr;
    Item *leaf_items = nullptr;
    uint32_t *masks = nullptr;
    Group *proxy_groups = nullptr;
    Item *proxy_items = nullptr;
    int32_t *proxy_unit_beg = nullptr;
    double4 *tgt_proxy = nullptr;
    double *records = nullptr;
    double4 *proxy_partial = nullptr;
    UpUnit *up_units = nullptr;
    int32_t *up_unit_beg = nullptr;
    double *src_nodes = nullptr;
    double *up_partial = nullptr;
    int *err = nullptr;
    int *h_flag = nullptr;            // pinned host copy of *err
    // batched mixed-precision form (allocated on its first solve)
    int FT = 0;                       // fields per block: 32 or 64
    int max_fields = 1;
    float *wF = nullptr, *phiF = nullptr, *mix_up_partial = nullptr, *mix_proxy_partial = nullptr;
    MixGroup *mix_leaf_groups = nullptr, *mix_proxy_groups = nullptr, *mix_up_groups = nullptr;
    MixGroup *tc_leaf_groups = nullptr;
    TcItem *tc_items = nullptr;
    MixGroup *tc_proxy_groups = nullptr;
    TcItem *tc_proxy_items = nullptr;
    MixGroup *tc_up_groups = nullptr;
    TcItem *tc_up_items = nullptr;
    int32_t *tc_up_unit_beg = nullptr;
    float *tc_up_partial = nullptr;
    float *basis = nullptr;           // upward pass: per-point BLI factors per basis k-step
    int32_t *bsrc = nullptr;
    float *bstore = nullptr;          // split weight store of the tcgen05 leaf pass
    void *bstore16 = nullptr;         // FP16 leaf pass: its FP16 hi/lo weight store (one spare unit at the end)
    float *tscale = nullptr, *tinv = nullptr;   // FP16 leaf pass: per target, its kernel values' scale
    unsigned *fmax = nullptr;         // FP16 leaf pass: the block's field maxima (source weights, potentials)
    unsigned char *ktile = nullptr;   // FP16 leaf pass with sal_tune.tile_store: its kernel tiles
    int64_t *ktile_off = nullptr;     // per leaf group, the byte offset of its tiles
    bool tile_recorded = false;       // a solve has been launched that records the tiles
    float4 *sloc = nullptr;
    float *sxyz = nullptr;
    int32_t *iperm = nullptr;         // caller index -> pool position
    double2 *selfk = nullptr;
    int nsm = 0;
    Item *mix_leaf_items = nullptr, *mix_proxy_items = nullptr;
    double *tgt_nodes = nullptr;
    // tcgen05 plan (tree passes, its own proxy units)
    int32_t *m2m_tasks = nullptr, *l2l_tasks = nullptr, *tc_proxy_unit_beg = nullptr;
    double *tc_up_nodes = nullptr, *tc_down_nodes = nullptr, *tc_transfer = nullptr;
    int64_t mix_bytes = 0;
    std::vector<std::pair<void **, size_t>> mix_allocs;   // the batched form's buffers (release_mixed frees them)
    // staging for the *_host entry points
    double *h_ssh = nullptr, *h_ox = nullptr, *h_oy = nullptr;  // device
    double *hb_ssh = nullptr, *hb_ox = nullptr, *hb_oy = nullptr;  // device, batched
    int hb_fields = 0;
    // pipelined host solves: two device staging slots, copy streams of their own
    struct HostSlot {
        double *ssh = nullptr, *ox = nullptr, *oy = nullptr;
        int64_t fields = 0;
        cudaEvent_t in = nullptr, solved = nullptr, out = nullptr;
        bool used = false;
    } hslot[2];
    int hnext = 0;
    cudaStream_t s_in = nullptr, s_out = nullptr;
    // CUDA graphs of batched solves, one per call shape (sal_grid_set_graphs)
    struct GraphShape {
        const double *ssh;
        int32_t nf;
        int64_t ld_ssh;
        double *ox, *oy;
        int64_t ld_out;
        bool operator==(const GraphShape &o) const {
            return ssh == o.ssh && nf == o.nf && ld_ssh == o.ld_ssh && ox == o.ox && oy == o.oy && ld_out == o.ld_out;
        }
    };
    struct GraphEntry {
        GraphShape shape;
        cudaGraphExec_t exec;
    };
    bool use_graphs = false;
    std::vector<GraphEntry> graphs;
    std::vector<GraphShape> seen;     // shapes solved once: captured on their second solve
    std::mutex graph_mu;              // guards use_graphs, graphs and seen
    double *h_w = nullptr;                                        // device, P*npanels
    uint32_t inject_polls = 0;        // sal_grid_inject_timeout: applies to the next FP64 solve
    std::vector<void *> allocs;
    std::mutex mu;
    // optional per-pass timers: events recorded on the launching stream
    bool timing = false;
    cudaEvent_t ev[8] = {};
    double phase_ms[4] = {0, 0, 0, 0};   // prep+upward, proxy, leaf, total
    int64_t phase_solves = 0;
};

}  // namespace

struct sal_grid {
    GridImpl g;
};
struct sal_tree : sal::Tree {};

#define CK(call)                                                                                  \
    do {                                                                                          \
        cudaError_t e_ = (call);                                                                  \
        if (e_ != cudaSuccess)                                                                    \
            return set_error(SAL_ECUDA, std::string(#call) + ": " + cudaGetErrorString(e_));     \
    } while (0)

template <class T>
static int dalloc(GridImpl &g, T **p, size_t count) {
    *p = nullptr;
    if (count == 0) return SAL_OK;
    cudaError_t e = cudaMalloc((void **)p, count * sizeof(T));
    if (e != cudaSuccess) {
        *p = nullptr;
        return set_error(e == cudaErrorMemoryAllocation ? SAL_ENOMEM : SAL_ECUDA,
                         std::string("cudaMalloc: ") + cudaGetErrorString(e));
    }
    g.allocs.push_back(*p);
    g.bytes += (int64_t)(count * sizeof(T));
    return SAL_OK;
}

// Frees a buffer dalloc made for this grid and stops counting it.  The caller
// has made sure no device work still reads or writes it.
template <class T>
static void dfree(GridImpl &g, T **p, size_t count) {
    if (!*p) return;
    for (size_t i = 0; i < g.allocs.size(); ++i)
        if (g.allocs[i] == (void *)*p) {
            g.allocs.erase(g.allocs.begin() + (std::ptrdiff_t)i);
            g.bytes -= (int64_t)(count * sizeof(T));
            break;
        }
    cudaFree(*p);
    *p = nullptr;
}

template <class T>
static int dupload(GridImpl &g, T **p, const T *src, size_t count) {
    int rc = dalloc(g, p, count);
    if (rc) return rc;
    if (count) CK(cudaMemcpy(*p, src, count * sizeof(T), cudaMemcpyHostToDevice));
    return SAL_OK;
}

// dalloc / dupload of a batched-form buffer, recorded for release_mixed.
template <class T>
static int malloc_mix(GridImpl &g, T **p, size_t count) {
    int rc = dalloc(g, p, count);
    if (!rc && *p) g.mix_allocs.push_back({(void **)p, count * sizeof(T)});
    return rc;
}
template <class T>
static int upload_mix(GridImpl &g, T **p, const std::vector<T> &v) {
    int rc = malloc_mix(g, p, v.size());
    if (rc || v.empty()) return rc;
    CK(cudaMemcpy(*p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice));
    return SAL_OK;
}

// Frees every batched-form buffer once the grid's stream is idle; the next
// batched solve allocates them again for the current tcgen05 plan.
static int release_mixed(GridImpl &g) {
    CK(cudaStreamSynchronize(g.stream));
    for (auto &e : g.mix_allocs) {
        void *ptr = *e.first;
        for (size_t i = 0; i < g.allocs.size(); ++i)
            if (g.allocs[i] == ptr) {
                g.allocs.erase(g.allocs.begin() + (std::ptrdiff_t)i);
                break;
            }
        cudaFree(ptr);
        g.bytes -= (int64_t)e.second;
        *e.first = nullptr;
    }
    g.mix_allocs.clear();
    g.FT = 0;
    g.mix_bytes = 0;
    g.tile_recorded = false;
    // captured graphs name the freed buffers
    std::lock_guard<std::mutex> lk(g.graph_mu);
    for (auto &e : g.graphs) cudaGraphExecDestroy(e.exec);
    g.graphs.clear();
    g.seen.clear();
    return SAL_OK;
}

static void grid_free(GridImpl &g) {
    if (g.dev >= 0) cudaSetDevice(g.dev);
    for (auto &e : g.ev)
        if (e) cudaEventDestroy(e);
    for (auto &h : g.hslot)
        for (cudaEvent_t e : {h.in, h.solved, h.out})
            if (e) cudaEventDestroy(e);
    for (auto &e : g.graphs) cudaGraphExecDestroy(e.exec);
    g.graphs.clear();
    if (g.s_in) cudaStreamDestroy(g.s_in);
    if (g.s_out) cudaStreamDestroy(g.s_out);
    for (void *p : g.allocs) cudaFree(p);
    g.allocs.clear();
    if (g.stream) cudaStreamDestroy(g.stream);
    g.stream = nullptr;
    if (g.h_flag) cudaFreeHost(g.h_flag);
    g.h_flag = nullptr;
}

static int require_device(int dev) {
    int count = 0;
    cudaError_t e = cudaGetDeviceCount(&count);
    if (e != cudaSuccess || count == 0) return set_error(SAL_ENODEV, "no CUDA device is available");
    if (dev < 0 || dev >= count) return set_error(SAL_EINVAL, "device ordinal out of range");
    CK(cudaSetDevice(dev));
    return SAL_OK;
}

extern "C" int sal_grid_create(const sal_tree *t_, const sal_grid_desc *d, sal_grid **out) {
    if (!t_ || !d || !out) return set_error(SAL_EINVAL, "null argument");
    *out = nullptr;
    const Tree &t = *static_cast<const Tree *>(t_);
    if (d->point_count != t.n) return set_error(SAL_EINVAL, "point_count differs from the tree's");
    if (!d->xs || !d->ys || !d->zs || !d->areas) return set_error(SAL_EINVAL, "null point arrays");
    if (d->mode < SAL_MODE_DTT || d->mode > SAL_MODE_STT_CORRECT) return set_error(SAL_EINVAL, "unknown mode");
    if (d->mode == SAL_MODE_DTT && d->list_count > 0 && !d->list) return set_error(SAL_EINVAL, "null list");
    if (d->mode != SAL_MODE_DTT && ((d->pc_count > 0 && !d->pc_list) || (d->pp_count > 0 && !d->pp_list)))
        return set_error(SAL_EINVAL, "null STT list");
    int rc = require_device(d->device);
    if (rc) return rc;
    auto t0 = std::chrono::steady_clock::now();
    sal_grid *G = new sal_grid();
    GridImpl &g = G->g;
    g.dev = d->device;
    g.max_fields = d->max_fields;
    if (d->mode == SAL_MODE_DTT) g.tree = t;
    std::string err;
    if (!plan_build(t, d->interp_degree, d->mode, d->list, d->list_count, d->pc_list, d->pc_count, d->pp_list,
                    d->pp_count, &g.plan, &err)) {
        delete G;
        return set_error(SAL_EINVAL, err);
    }
    // grids made for 32-field blocks get the mma.sync groups now, so their
    // stats count them; others build them if a tune switches to 32 fields
    if (d->mode == SAL_MODE_DTT && d->max_fields <= 32) plan_build_mix(t, &g.plan);
    Plan &pl = g.plan;
    const int n = pl.n, P = pl.P, nd = pl.d + 1;
    g.nsrc = (int)pl.src_slot_panel.size();
    g.ntgt = (int)pl.tgt_slot_panel.size();
    g.rec_stride = 4 * P + 2 * nd;
    g.rec_stride = (g.rec_stride + 3) & ~3;  // records start on 32-byte boundaries
    g.nup = (int)pl.up_units.size();
    g.nproxy_units = (int)pl.proxy_groups.size();
    if (cudaStreamCreateWithFlags(&g.stream, cudaStreamNonBlocking) != cudaSuccess) {
        delete G;
        return set_error(SAL_ECUDA, "cudaStreamCreate failed");
    }
#define TRY(x)                 \
    do {                       \
        int rc_ = (x);         \
        if (rc_) {             \
            grid_free(g);      \
            delete G;          \
            return rc_;        \
        }                      \
    } while (0)
    {
        std::vector<double4> xyz(n);
        std::vector<double> area(n);
        std::vector<double2> xe(n);
        for (int p = 0; p < n; ++p) {
            int i = pl.perm[p];
            xyz[p] = make_double4(d->xs[i], d->ys[i], d->zs[i], 0.0);
            area[p] = d->areas[i];
            xe[p] = make_double2(pl.pxi[p], pl.peta[p]);
        }
        TRY(dupload(g, &g.xyz, xyz.data(), (size_t)n));
        TRY(dupload(g, &g.area, area.data(), (size_t)n));
        TRY(dupload(g, &g.xieta, xe.data(), (size_t)n));
        TRY(dupload(g, &g.perm, pl.perm.data(), (size_t)n));
        std::vector<double4> pool((size_t)n + (size_t)g.nsrc * P);
        for (int p = 0; p < n; ++p) pool[p] = xyz[p];
        for (size_t q = 0; q < (size_t)g.nsrc * P; ++q)
            pool[n + q] = make_double4(pl.src_proxy_xyz[3 * q], pl.src_proxy_xyz[3 * q + 1], pl.src_proxy_xyz[3 * q + 2], 0.0);
        TRY(dupload(g, &g.pool, pool.data(), pool.size()));
        std::vector<double4> tp((size_t)g.ntgt * P);
        for (size_t q = 0; q < tp.size(); ++q)
            tp[q] = make_double4(pl.tgt_proxy_xyz[3 * q], pl.tgt_proxy_xyz[3 * q + 1], pl.tgt_proxy_xyz[3 * q + 2], 0.0);
        TRY(dupload(g, &g.tgt_proxy, tp.data(), tp.size()));
        std::vector<double> rec((size_t)g.ntgt * g.rec_stride, 0.0);
        for (int s = 0; s < g.ntgt; ++s)
            for (int i = 0; i < 2 * nd; ++i) rec[(size_t)s * g.rec_stride + 4 * P + i] = pl.tgt_nodes[(size_t)s * 2 * nd + i];
        TRY(dupload(g, &g.records, rec.data(), rec.size()));
    }
    TRY(dupload(g, &g.leaf_groups, pl.leaf_groups.data(), pl.leaf_groups.size()));
    TRY(dupload(g, &g.leaf_items, pl.leaf_items.data(), pl.leaf_items.size()));
    TRY(dupload(g, &g.masks, pl.masks.data(), pl.masks.size()));
    TRY(dupload(g, &g.proxy_groups, pl.proxy_groups.data(), pl.proxy_groups.size()));
    TRY(dupload(g, &g.proxy_items, pl.proxy_items.data(), pl.proxy_items.size()));
    TRY(dupload(g, &g.proxy_unit_beg, pl.proxy_unit_beg.data(), pl.proxy_unit_beg.size()));
    TRY(dalloc(g, &g.proxy_partial, (size_t)g.nproxy_units * P));
    TRY(dupload(g, &g.up_units, pl.up_units.data(), pl.up_units.size()));
    TRY(dupload(g, &g.up_unit_beg, pl.up_unit_beg.data(), pl.up_unit_beg.size()));
    TRY(dupload(g, &g.src_nodes, pl.src_nodes.data(), pl.src_nodes.size()));
    TRY(dupload(g, &g.tgt_nodes, pl.tgt_nodes.data(), pl.tgt_nodes.size()));
    TRY(dalloc(g, &g.up_partial, (size_t)g.nup * P));
    TRY(dalloc(g, &g.err, 1));
    CK(cudaMemset(g.err, 0, sizeof(int)));
    if (cudaMallocHost((void **)&g.h_flag, sizeof(int)) != cudaSuccess) {
        grid_free(g);
        delete G;
        return set_error(SAL_ENOMEM, "cudaMallocHost failed");
    }
    CK(cudaDeviceSynchronize());
    // host copies no longer needed on the device side
    pl.px.clear(); pl.py.clear(); pl.pz.clear(); pl.parea.clear();
    g.setup_seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    *out = G;
    return SAL_OK;
#undef TRY
}

extern "C" int sal_grid_destroy(sal_grid *G) {
    if (!G) return SAL_OK;
    grid_free(G->g);
    delete G;
    return SAL_OK;
}

// Device bytes ensure_mixed allocates for blocks of FT fields (the same
// buffers, counted without allocating).
static int64_t mixed_bytes_needed(const GridImpl &g, int FT) {
    const Plan &pl = g.plan;
    const bool tc = FT == 64 && !pl.tc_items.empty();
    const int64_t P = pl.P, n = pl.n;
    const int64_t nw = tc ? pl.n_wslots : g.nsrc, ndn = tc ? pl.n_dslots : g.ntgt;
    const int64_t nunits_p = std::max<int64_t>(g.nproxy_units, pl.tc_nproxy_units);
    auto vb = [](const auto &v) { return (int64_t)(v.size() * sizeof(v[0])); };
    int64_t b = 4 * (int64_t)FT * ((n + nw * P) + ndn * 3 * P + (int64_t)g.nup * P + nunits_p * 3 * P) + 4 * n;
    if (!tc) {
        b += vb(pl.mix_leaf_groups) + vb(pl.mix_leaf_items) + vb(pl.mix_proxy_groups) + vb(pl.mix_proxy_items) +
             vb(pl.mix_up_groups);
    } else {
        b += vb(pl.tc_leaf_groups) + vb(pl.tc_items) + vb(pl.tc_proxy_groups) + vb(pl.tc_proxy_items) +
             vb(pl.tc_proxy_unit_beg) + vb(pl.tc_up_groups) + vb(pl.tc_up_items) + vb(pl.tc_up_unit_beg) +
             vb(pl.tc_up_nodes) + vb(pl.tc_down_nodes) + vb(pl.m2m_tasks) + vb(pl.l2l_tasks) + vb(pl.tc_transfer);
        const int64_t nbk = (int64_t)pl.tc_bas.size() / 3, nunits = pl.tc_up_unit_beg.empty() ? 0 : pl.tc_up_unit_beg.back();
        b += 4 * nunits * P * FT + 4 * nbk * 16 * (pl.d + 1) + vb(pl.bsrc) + 4 * (int64_t)pl.bsrc.size() * 2 * FT +
             (int64_t)sizeof(float4) * (n + (int64_t)g.nsrc * P) + (int64_t)sizeof(double2) * n +
             4 * pl.tc_src_ksteps * 24;
        if (pl.tc_opt.f16) b += ((int64_t)pl.bsrc.size() / 8 + 1) * 2048 + 128 * 4 + 2 * 4 * n;
        if (pl.tc_opt.f16 && pl.tc_opt.tile_store) b += pl.tc_tile_off.back() + vb(pl.tc_tile_off);
    }
    return b;
}

// Kernel launches of one batched block of FT fields (solve_mixed_block's
// sequence for the current plan).
static int64_t batched_launches(const GridImpl &g, int FT) {
    const Plan &pl = g.plan;
    const bool tc = FT == 64 && !pl.tc_items.empty();
    if (!tc) return 1 + (pl.mix_up_groups.empty() ? 0 : 2) + (pl.mix_proxy_groups.empty() ? 0 : 2) + 1;
    const bool tree = pl.tc_opt.tree_passes != 0;
    auto levels = [](const std::vector<int32_t> &beg) {
        int64_t k = 0;
        for (size_t l = 0; l + 1 < beg.size(); ++l) k += beg[l + 1] > beg[l];
        return k;
    };
    int64_t k = 2;                                                         // prep, store (points)
    if (!pl.tc_up_groups.empty()) k += tree ? 1 : 2;                       // upward (+ finalize)
    if (tree) k += levels(pl.m2m_level_beg);
    k += 1;                                                                // store (proxies)
    if (!pl.tc_proxy_groups.empty()) k += 2 + (tree ? levels(pl.l2l_level_beg) : 0);   // proxy, finalize, l2l
    k += pl.tc_opt.f16 ? 3 : 1;                                            // leaf store: maxima + FP16, or TF32
    return k + 1;                                                          // leaf pass
}

extern "C" int sal_grid_stats_get(const sal_grid *G, sal_grid_stats *s) {
    if (!G || !s) return set_error(SAL_EINVAL, "null argument");
    const GridImpl &g = G->g;
    const Plan &pl = g.plan;
    std::memset(s, 0, sizeof(*s));
    s->point_count = pl.n;
    s->npanels = pl.npanels;
    s->nleaves = pl.nleaves;
    s->degree = pl.d;
    s->mode = pl.mode;
    s->list_count = (int64_t)pl.leaf_items.size();
    s->pairs_pp = pl.pairs[0];
    s->pairs_pc = pl.pairs[1];
    s->pairs_cp = pl.pairs[2];
    s->pairs_cc = pl.pairs[3];
    s->macs_up = pl.macs_up;
    s->macs_down = pl.macs_down;
    s->device_bytes = g.bytes;
    s->setup_seconds = g.setup_seconds;
    s->macs_up_batched = pl.tc_items.empty() ? pl.macs_up : pl.tc_macs_up;
    s->macs_down_batched = pl.tc_items.empty() ? pl.macs_down : pl.tc_macs_down;
    s->mixed_bytes = g.FT ? g.mix_bytes : mixed_bytes_needed(g, g.max_fields <= 32 ? 32 : 64);
    s->launches_batched = batched_launches(g, g.FT ? g.FT : (g.max_fields <= 32 ? 32 : 64));
    s->tile_store_bytes = pl.tc_tile_off.empty() ? 0 : pl.tc_tile_off.back();
    return SAL_OK;
}

// One FP64 solve of one field: ssh (caller order, device) -> outputs (caller order, device).
static void solve_fp64(GridImpl &g, const double *ssh, double *ox, double *oy, int form, int kinds, bool do_up,
                       cudaStream_t st) {
    const Plan &pl = g.plan;
    const int n = pl.n, P = pl.P;
    if (g.timing) cudaEventRecord(g.ev[0], st);
    dev::launch_prep(g.xyz, g.area, ssh, g.perm, n, g.pool, st);
    if (do_up && g.nup > 0) {
        dev::UpArgs u{g.pool, g.xieta, g.up_units, g.src_nodes, pl.d, P, g.up_partial};
        dev::launch_upward(u, g.nup, st);
        dev::launch_upward_finalize(g.up_unit_beg, g.up_partial, g.nsrc, pl.d, pl.mode == SAL_MODE_STT_REF_COMPAT ? 1 : 0,
                                    g.pool + n, st);
    }
    if (g.timing) cudaEventRecord(g.ev[1], st);
    if (g.nproxy_units > 0) {
        dev::EvalArgs a{};
        a.pool = g.pool;
        a.groups = g.proxy_groups;
        a.items = g.proxy_items;
        a.masks = g.masks;
        a.tgt = g.tgt_proxy;
        a.xieta = g.xieta;
        a.records = g.records;
        a.rec_stride = g.rec_stride;
        a.d = pl.d;
        a.P = P;
        a.kinds = 3;
        a.perm = g.perm;
        a.partial = g.proxy_partial;
        a.err = g.err;
        dev::launch_eval(1, form, a, g.nproxy_units, st);
        dev::launch_proxy_finalize(g.proxy_unit_beg, g.proxy_partial, g.ntgt, P, g.rec_stride, g.records, st);
    }
    if (g.timing) cudaEventRecord(g.ev[2], st);
    dev::EvalArgs a{};
    a.pool = g.pool;
    a.groups = g.leaf_groups;
    a.items = g.leaf_items;
    a.masks = g.masks;
    a.tgt = g.pool;
    a.xieta = g.xieta;
    a.records = g.records;
    a.rec_stride = g.rec_stride;
    a.d = pl.d;
    a.P = P;
    a.kinds = kinds;
    a.perm = g.perm;
    a.out_x = ox;
    a.out_y = oy;
    a.err = g.err;
    if (g.inject_polls) {
        a.polls = g.inject_polls;
        a.skip_last = 1;
        g.inject_polls = 0;
    }
    dev::launch_eval(0, form, a, (int)pl.leaf_groups.size(), st);
    if (g.timing) {
        cudaEventRecord(g.ev[3], st);
        cudaEventSynchronize(g.ev[3]);
        float t01 = 0, t12 = 0, t23 = 0;
        cudaEventElapsedTime(&t01, g.ev[0], g.ev[1]);
        cudaEventElapsedTime(&t12, g.ev[1], g.ev[2]);
        cudaEventElapsedTime(&t23, g.ev[2], g.ev[3]);
        g.phase_ms[0] += t01;
        g.phase_ms[1] += t12;
        g.phase_ms[2] += t23;
        g.phase_ms[3] += t01 + t12 + t23;
        g.phase_solves += 1;
    }
}

static mix::TcArgs leaf_args(GridImpl &g, double *ox, double *oy, int64_t ld_out, int f0, int nf);

// Device buffers of the batched form, sized for blocks of FT fields.
static int ensure_mixed(GridImpl &g, int FT) {
    if (g.FT == FT) return SAL_OK;
    if (g.FT != 0) return set_error(SAL_EINVAL, "a grid's batched buffers are sized for one field block width");
    const bool tc = FT == 64 && !g.plan.tc_items.empty();
    if (!tc && !g.plan.mix_built && g.plan.mode == SAL_MODE_DTT) plan_build_mix(g.tree, &g.plan);
    const Plan &pl = g.plan;
    const size_t P = (size_t)pl.P, n = (size_t)pl.n;
    const int64_t before = g.bytes;
    // proxy-weight rows: source slots (and, in the tree passes, the other
    // panels below them); potential rows: target slots (and the panels below)
    const size_t nw = tc ? (size_t)pl.n_wslots : (size_t)g.nsrc, ndn = tc ? (size_t)pl.n_dslots : (size_t)g.ntgt;
    const size_t nunits_p = std::max((size_t)g.nproxy_units, (size_t)pl.tc_nproxy_units);
    int rc = SAL_OK;
    if (!rc) rc = malloc_mix(g, &g.wF, (n + nw * P) * FT);
    if (!rc) rc = malloc_mix(g, &g.phiF, ndn * 3 * P * FT);
    if (!rc) rc = malloc_mix(g, &g.mix_up_partial, (size_t)g.nup * P * FT);
    if (!rc) rc = malloc_mix(g, &g.mix_proxy_partial, nunits_p * 3 * P * FT);
    if (!rc) {
        std::vector<int32_t> ip(n);
        for (size_t p = 0; p < n; ++p) ip[(size_t)pl.perm[p]] = (int32_t)p;
        rc = upload_mix(g, &g.iperm, ip);
    }
    if (!rc && !tc) {
        // mma.sync passes
        rc = upload_mix(g, &g.mix_leaf_groups, pl.mix_leaf_groups);
        if (!rc) rc = upload_mix(g, &g.mix_leaf_items, pl.mix_leaf_items);
        if (!rc) rc = upload_mix(g, &g.mix_proxy_groups, pl.mix_proxy_groups);
        if (!rc) rc = upload_mix(g, &g.mix_proxy_items, pl.mix_proxy_items);
        if (!rc) rc = upload_mix(g, &g.mix_up_groups, pl.mix_up_groups);
    }
    if (!rc && tc) {
        // tcgen05 passes: items, split weight store, per-row source
        // coordinates, the per-point self pairs and the tree transfers
        rc = upload_mix(g, &g.tc_leaf_groups, pl.tc_leaf_groups);
        if (!rc) rc = upload_mix(g, &g.tc_items, pl.tc_items);
        if (!rc) rc = upload_mix(g, &g.tc_proxy_groups, pl.tc_proxy_groups);
        if (!rc) rc = upload_mix(g, &g.tc_proxy_items, pl.tc_proxy_items);
        if (!rc) rc = upload_mix(g, &g.tc_proxy_unit_beg, pl.tc_proxy_unit_beg);
        if (!rc) rc = upload_mix(g, &g.tc_up_groups, pl.tc_up_groups);
        if (!rc) rc = upload_mix(g, &g.tc_up_items, pl.tc_up_items);
        if (!rc) rc = upload_mix(g, &g.tc_up_unit_beg, pl.tc_up_unit_beg);
        if (!rc) rc = upload_mix(g, &g.tc_up_nodes, pl.tc_up_nodes);
        if (!rc) rc = upload_mix(g, &g.tc_down_nodes, pl.tc_down_nodes);
        if (!rc) rc = upload_mix(g, &g.m2m_tasks, pl.m2m_tasks);
        if (!rc) rc = upload_mix(g, &g.l2l_tasks, pl.l2l_tasks);
        if (!rc) rc = upload_mix(g, &g.tc_transfer, pl.tc_transfer);
        const int64_t nbk = (int64_t)pl.tc_bas.size() / 3,
                      nunits = pl.tc_up_unit_beg.empty() ? 0 : pl.tc_up_unit_beg.back();
        if (!rc) rc = malloc_mix(g, &g.tc_up_partial, (size_t)nunits * P * FT);
        if (!rc) rc = malloc_mix(g, &g.basis, (size_t)nbk * 16 * (pl.d + 1));
        if (!rc && nbk > 0) {
            // the basis store, once per plan
            int32_t *bas = nullptr;
            CK(cudaMalloc((void **)&bas, pl.tc_bas.size() * sizeof(int32_t)));
            cudaError_t e = cudaMemcpy(bas, pl.tc_bas.data(), pl.tc_bas.size() * sizeof(int32_t), cudaMemcpyHostToDevice);
            if (e == cudaSuccess) {
                mix::launch_basis_store(bas, nbk, g.xieta, g.tc_up_nodes, pl.d + 1, g.basis, g.stream);
                e = cudaStreamSynchronize(g.stream);
            }
            cudaFree(bas);
            if (e != cudaSuccess) return set_error(SAL_ECUDA, std::string("basis store: ") + cudaGetErrorString(e));
        }
        if (!rc) rc = upload_mix(g, &g.bsrc, pl.bsrc);
        if (!rc) rc = malloc_mix(g, &g.bstore, pl.bsrc.size() * 2 * (size_t)FT);
        if (!rc) rc = malloc_mix(g, &g.sloc, n + (size_t)g.nsrc * P);
        if (!rc) rc = malloc_mix(g, &g.selfk, n);
        if (!rc) rc = malloc_mix(g, &g.sxyz, (size_t)pl.tc_src_ksteps * 24);
        if (!rc) {
            const size_t nr = pl.sloc_ranges.size() / 2;
            std::vector<int2> ranges(nr);
            std::vector<double4> centres(nr);
            for (size_t i = 0; i < nr; ++i) {
                ranges[i] = make_int2(pl.sloc_ranges[2 * i], pl.sloc_ranges[2 * i + 1]);
                centres[i] = make_double4(pl.sloc_centres[3 * i], pl.sloc_centres[3 * i + 1], pl.sloc_centres[3 * i + 2], 0.0);
            }
            int2 *dr = nullptr;
            double4 *dc = nullptr;
            CK(cudaMalloc((void **)&dr, ranges.size() * sizeof(int2)));
            cudaError_t e = cudaMalloc((void **)&dc, centres.size() * sizeof(double4));
            if (e == cudaSuccess) e = cudaMemcpy(dr, ranges.data(), ranges.size() * sizeof(int2), cudaMemcpyHostToDevice);
            if (e == cudaSuccess) e = cudaMemcpy(dc, centres.data(), centres.size() * sizeof(double4), cudaMemcpyHostToDevice);
            if (e == cudaSuccess) {
                mix::launch_source_local(g.pool, dr, dc, (int)ranges.size(), g.sloc, g.stream);
                mix::launch_self_pair(g.pool, (int)n, g.selfk, g.stream);
                mix::launch_source_ksteps(g.bsrc, pl.tc_src_ksteps, g.sloc, g.sxyz, g.stream);
                e = cudaStreamSynchronize(g.stream);
            }
            cudaFree(dr);
            if (dc) cudaFree(dc);
            if (e != cudaSuccess) return set_error(SAL_ECUDA, std::string("batched set-up: ") + cudaGetErrorString(e));
        }
        if (!rc && pl.tc_opt.f16) {
            // FP16 leaf pass: its weight store (zeroed: the spare unit past the
            // last item must hold finite values), field maxima, and the
            // per-target scales of the kernel values, once per plan
            const size_t units = pl.bsrc.size() / 8 + 1;
            rc = malloc_mix(g, reinterpret_cast<unsigned char **>(&g.bstore16), units * 2048);
            if (!rc) rc = malloc_mix(g, &g.fmax, (size_t)128);
            if (!rc) rc = malloc_mix(g, &g.tscale, n);
            if (!rc) rc = malloc_mix(g, &g.tinv, n);
            if (!rc) {
                // zeros in every row no pass writes, so the per-field maxima can
                // read the weight and potential rows whole
                CK(cudaMemsetAsync(g.wF, 0, (n + (size_t)pl.n_wslots * P) * FT * sizeof(float), g.stream));
                CK(cudaMemsetAsync(g.phiF, 0, (size_t)pl.n_dslots * 3 * P * FT * sizeof(float), g.stream));
                CK(cudaMemsetAsync(g.bstore16, 0, units * 2048, g.stream));
                mix::TcArgs t = leaf_args(g, nullptr, nullptr, 0, 0, 0);
                mix::launch_target_scales(t, g.tscale, g.tinv, g.stream);
                CK(cudaStreamSynchronize(g.stream));
                CK(cudaGetLastError());
            }
            // the kernel-tile store, written by the next leaf pass
            if (!rc && pl.tc_opt.tile_store) {
                rc = upload_mix(g, &g.ktile_off, pl.tc_tile_off);
                if (!rc) rc = malloc_mix(g, &g.ktile, (size_t)pl.tc_tile_off.back());
                g.tile_recorded = false;
            }
        }
        if (!rc) CK(cudaDeviceGetAttribute(&g.nsm, cudaDevAttrMultiProcessorCount, g.dev));
    }
    if (rc) {
        release_mixed(g);
        return rc;
    }
    g.FT = FT;
    g.mix_bytes = g.bytes - before;
    return SAL_OK;
}

// Arguments of the tcgen05 leaf pass of one 64-field block.
static mix::TcArgs leaf_args(GridImpl &g, double *ox, double *oy, int64_t ld_out, int f0, int nf) {
    const Plan &pl = g.plan;
    mix::TcArgs t{};
    t.groups = g.tc_leaf_groups;
    t.ngroups = (int)pl.tc_leaf_groups.size();
    t.items = g.tc_items;
    t.sxyz = g.sxyz;
    t.bstore = g.bstore;
    t.tgt = g.pool;
    t.xieta = g.xieta;
    t.tgt_nodes = g.tc_down_nodes;
    t.selfk = g.selfk;
    t.wF = g.wF;
    t.perm = g.perm;
    t.d = pl.d;
    t.P = pl.P;
    t.out_x = ox;
    t.out_y = oy;
    t.ld_out = ld_out;
    t.f0 = f0;
    t.nf = nf;
    if (g.bstore16) {
        t.bstore16 = g.bstore16;
        t.tscale = g.tscale;
        t.tinv = g.tinv;
        t.fmax = g.fmax;
        t.ktile = g.ktile;
        t.ktile_off = g.ktile_off;
        t.tile_every = g.plan.tc_opt.tile_store > 1 ? g.plan.tc_opt.tile_store : 1;
    }
    return t;
}

// One block of up to FT fields in the batched form: per-field weights, upward
// pass, proxy potentials, leaf pass.  With joint != NULL (tcgen05 blocks) the
// leaf pass is not launched: its arguments go to *joint.
static void solve_mixed_block(GridImpl &g, const double *ssh, int64_t ld_ssh, int f0, int nf, double *ox, double *oy,
                              int64_t ld_out, cudaStream_t st, mix::TcArgs *joint = nullptr) {
    const Plan &pl = g.plan;
    const int n = pl.n, P = pl.P, FT = g.FT;
    const bool timed = g.timing && !joint;   // a joint solve's leaf pass is not this grid's alone
    if (timed) cudaEventRecord(g.ev[0], st);
    mix::launch_prep_mix(g.area, ssh, ld_ssh, g.iperm, n, f0, nf, FT, g.wF, st);
    mix::MixArgs a{};
    a.pool = g.pool;
    a.wF = g.wF;
    a.phiF = g.phiF;
    a.xieta = g.xieta;
    a.d = pl.d;
    a.P = P;
    a.perm = g.perm;
    a.area = g.area;
    a.ssh = ssh;
    a.ld_ssh = ld_ssh;
    a.out_x = ox;
    a.out_y = oy;
    a.ld_out = ld_out;
    a.f0 = f0;
    a.nf = nf;
    const bool tree = g.bstore && pl.tc_opt.tree_passes;
    const int cg = pl.tc_opt.cta_groups;
    if (g.bstore) {
        // 64-field blocks, tcgen05: the points' rows of the split weight store,
        // then the upward pass; then the proxies' rows
        mix::launch_split_store(g.bsrc, 0, pl.tc_pt_ksteps, g.wF, g.phiF, g.bstore, st);
        if (!pl.tc_up_groups.empty()) {
            mix::TcArgs u{};
            u.groups = g.tc_up_groups;
            u.ngroups = (int)pl.tc_up_groups.size();
            u.items = g.tc_up_items;
            u.bstore = g.bstore;
            u.basis = g.basis;
            u.d = pl.d;
            u.P = P;
            // tree passes: every unit is one leaf, written straight to its
            // proxy-weight rows; direct passes: unit partials, summed per slot
            u.partial = tree ? g.wF + (size_t)n * FT : g.tc_up_partial;
            mix::launch_tc_upward(u, g.nsm, cg, g.err, st);
            if (!tree)
                mix::launch_finalize_mix(g.tc_up_unit_beg, g.tc_up_partial, g.nsrc, P, FT, g.wF + (size_t)n * FT, st);
        }
        if (tree)
            for (size_t l = 0; l + 1 < pl.m2m_level_beg.size(); ++l)
                mix::launch_m2m(g.m2m_tasks + 6 * (size_t)pl.m2m_level_beg[l], pl.m2m_level_beg[l + 1] - pl.m2m_level_beg[l],
                                g.tc_transfer, pl.d + 1, g.wF + (size_t)n * FT, st);
        mix::launch_split_store(g.bsrc, pl.tc_pt_ksteps, pl.tc_src_ksteps, g.wF, g.phiF, g.bstore, st);
    } else if (!pl.mix_up_groups.empty()) {
        mix::MixArgs u = a;
        u.groups = g.mix_up_groups;
        u.tgt_nodes = g.src_nodes;
        u.partial = g.mix_up_partial;
        mix::launch_mix(2, FT, u, (int)pl.mix_up_groups.size(), st);
        mix::launch_finalize_mix(g.up_unit_beg, g.mix_up_partial, g.nsrc, P, FT, g.wF + (size_t)n * FT, st);
    }
    if (timed) cudaEventRecord(g.ev[1], st);
    // 64-field blocks: the proxy pass on tcgen05
    if (g.bstore && !pl.tc_proxy_groups.empty()) {
        mix::TcArgs p{};
        p.groups = g.tc_proxy_groups;
        p.ngroups = (int)pl.tc_proxy_groups.size();
        p.items = g.tc_proxy_items;
        p.sxyz = g.sxyz;
        p.bstore = g.bstore;
        p.tgt = g.tgt_proxy;
        p.d = pl.d;
        p.P = P;
        p.partial = g.mix_proxy_partial;
        mix::launch_tc_proxy(p, g.nsm, cg, g.err, st);
        mix::launch_finalize_mix(g.tc_proxy_unit_beg, g.mix_proxy_partial, g.ntgt, 3 * P, FT, g.phiF, st);
        if (tree)
            for (size_t l = 0; l + 1 < pl.l2l_level_beg.size(); ++l)
                mix::launch_l2l(g.l2l_tasks + 4 * (size_t)pl.l2l_level_beg[l], pl.l2l_level_beg[l + 1] - pl.l2l_level_beg[l],
                                g.tc_transfer, pl.d + 1, g.phiF, st);
    } else if (!pl.mix_proxy_groups.empty()) {
        mix::MixArgs q = a;
        q.groups = g.mix_proxy_groups;
        q.items = g.mix_proxy_items;
        q.tgt = g.tgt_proxy;
        q.partial = g.mix_proxy_partial;
        mix::launch_mix(1, FT, q, (int)pl.mix_proxy_groups.size(), st);
        mix::launch_finalize_mix(g.proxy_unit_beg, g.mix_proxy_partial, g.ntgt, 3 * P, FT, g.phiF, st);
    }
    if (timed) cudaEventRecord(g.ev[2], st);
    // the leaf pass's weight rows: TF32 (the potential rows: the points' and
    // proxies' rows are in place), or FP16 (every row, scaled per field)
    auto leaf_store = [&]() {
        if (g.bstore16) {
            const size_t nw = (size_t)n + (size_t)pl.n_wslots * P, np = (size_t)pl.n_dslots * 3 * P;
            cudaMemsetAsync(g.fmax, 0, 128 * sizeof(unsigned), st);
            mix::launch_field_max(g.wF, (int64_t)nw, g.phiF, (int64_t)np, g.fmax, st);
            mix::launch_split_store16(g.bsrc, (int64_t)pl.bsrc.size() / 8, g.wF, g.phiF, g.fmax, g.bstore16, st);
        } else {
            mix::launch_split_store(g.bsrc, pl.tc_src_ksteps, (int64_t)pl.bsrc.size() / 8, g.wF, g.phiF, g.bstore, st);
        }
    };
    if (joint) {
        // the caller runs the leaf pass, jointly with other grids'
        leaf_store();
        *joint = leaf_args(g, ox, oy, ld_out, f0, nf);
        return;
    }
    a.items = g.mix_leaf_items;
    a.tgt = g.pool;
    a.tgt_nodes = g.tgt_nodes;
    if (g.bstore) {
        // 64-field blocks: the leaf pass's weight rows, then the tcgen05 leaf pass
        leaf_store();
        // with a kernel-tile store: the first leaf pass records the tiles, the
        // later ones (stream-ordered after it) replay them: all of them (2), or
        // one item in tile_store beside the producers' (3)
        const int tiles = g.ktile ? (!g.tile_recorded ? 1 : pl.tc_opt.tile_store > 1 ? 3 : 2) : 0;
        mix::launch_tc_leaf(leaf_args(g, ox, oy, ld_out, f0, nf), g.nsm, cg, g.err, st, tiles);
        if (tiles == 1) g.tile_recorded = true;
    } else {
        a.groups = g.mix_leaf_groups;
        mix::launch_mix(0, FT, a, (int)pl.mix_leaf_groups.size(), st);
    }
    if (timed) {
        cudaEventRecord(g.ev[3], st);
        cudaEventSynchronize(g.ev[3]);
        float t01 = 0, t12 = 0, t23 = 0;
        cudaEventElapsedTime(&t01, g.ev[0], g.ev[1]);
        cudaEventElapsedTime(&t12, g.ev[1], g.ev[2]);
        cudaEventElapsedTime(&t23, g.ev[2], g.ev[3]);
        g.phase_ms[0] += t01;
        g.phase_ms[1] += t12;
        g.phase_ms[2] += t23;
        g.phase_ms[3] += t01 + t12 + t23;
        g.phase_solves += 1;
    }
}

constexpr size_t kMaxGraphs = 128;

// Captures the batched solve of one call shape into a graph (nothing runs).
// The capture stream takes the caller stream's priority, which the graph's
// kernels keep.  Every allocation and kernel attribute the solve needs exists
// already: the same shape has just run.  Called with graph_mu held.
static int capture_mixed(GridImpl &g, const GridImpl::GraphShape &k, cudaStream_t caller) {
    // a graph replays its launches as captured: the tile store's recording
    // pass must not be one of them
    if (g.ktile && !g.tile_recorded) return SAL_OK;
    int prio = 0;
    CK(cudaStreamGetPriority(caller, &prio));
    cudaStream_t cs = nullptr;
    CK(cudaStreamCreateWithPriority(&cs, cudaStreamNonBlocking, prio));
    cudaGraph_t graph = nullptr;
    cudaError_t e = cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal);
    if (e == cudaSuccess) {
        for (int f0 = 0; f0 < k.nf; f0 += g.FT) solve_mixed_block(g, k.ssh, k.ld_ssh, f0, k.nf, k.ox, k.oy, k.ld_out, cs);
        e = cudaStreamEndCapture(cs, &graph);
    }
    cudaGraphExec_t exec = nullptr;
    if (e == cudaSuccess) e = cudaGraphInstantiate(&exec, graph, 0);
    if (graph) cudaGraphDestroy(graph);
    cudaStreamDestroy(cs);
    if (e != cudaSuccess) return set_error(SAL_ECUDA, std::string("graph capture: ") + cudaGetErrorString(e));
    if (g.graphs.size() >= kMaxGraphs) {
        cudaGraphExecDestroy(g.graphs.front().exec);
        g.graphs.erase(g.graphs.begin());
    }
    g.graphs.push_back({k, exec});
    return SAL_OK;
}

extern "C" int sal_solve_joint(sal_grid *const *grids, int32_t ngrids, const double *const *ssh,
                               const int32_t *nfields, const int64_t *ld_ssh, double *const *out_x,
                               double *const *out_y, const int64_t *ld_out, void *stream) {
    if (!grids || !ssh || !nfields || !ld_ssh || !out_x || !out_y || !ld_out) return set_error(SAL_EINVAL, "null argument");
    if (ngrids < 1 || ngrids > mix::kMaxJoint)
        return set_error(SAL_EINVAL, "ngrids must be in 1.." + std::to_string(mix::kMaxJoint));
    cudaStream_t st = (cudaStream_t)stream;
    mix::TcArgs args[mix::kMaxJoint];
    for (int k = 0; k < ngrids; ++k) {
        if (!grids[k] || !ssh[k] || !out_x[k] || !out_y[k]) return set_error(SAL_EINVAL, "null argument");
        for (int j = 0; j < k; ++j)
            if (grids[j] == grids[k]) return set_error(SAL_EINVAL, "a grid appears twice in a joint solve");
        GridImpl &g = grids[k]->g;
        if (g.plan.mode != SAL_MODE_DTT) return set_error(SAL_EINVAL, "the batched form needs a SAL_MODE_DTT grid");
        if (nfields[k] < 1 || nfields[k] > 64) return set_error(SAL_EINVAL, "a joint solve takes 1..64 fields per grid");
        if (nfields[k] > 1 && (ld_ssh[k] < g.plan.n || ld_out[k] < g.plan.n))
            return set_error(SAL_EINVAL, "leading dimension < point_count");
        if (g.dev != grids[0]->g.dev || g.plan.d != grids[0]->g.plan.d)
            return set_error(SAL_EINVAL, "the grids of a joint solve share one device and one degree");
        if (g.max_fields <= 32 || g.plan.tc_items.empty())
            return set_error(SAL_EINVAL, "a joint solve needs grids with 64-field blocks (max_fields > 32)");
        if (g.plan.tc_opt.f16 != grids[0]->g.plan.tc_opt.f16)
            return set_error(SAL_EINVAL, "the grids of a joint solve share one leaf-pass precision (sal_tune.f16)");
    }
    CK(cudaSetDevice(grids[0]->g.dev));
    for (int k = 0; k < ngrids; ++k) {
        GridImpl &g = grids[k]->g;
        int rc = ensure_mixed(g, 64);
        if (rc) return rc;
        solve_mixed_block(g, ssh[k], ld_ssh[k], 0, nfields[k], out_x[k], out_y[k], ld_out[k], st, &args[k]);
    }
    GridImpl &g0 = grids[0]->g;
    mix::launch_tc_leaf_joint(args, ngrids, g0.nsm, g0.plan.tc_opt.cta_groups, g0.err, st);
    CK(cudaGetLastError());
    return SAL_OK;
}

extern "C" int sal_grid_set_graphs(sal_grid *G, int32_t enable) {
    if (!G) return set_error(SAL_EINVAL, "null argument");
    GridImpl &g = G->g;
    std::lock_guard<std::mutex> lk(g.graph_mu);
    CK(cudaSetDevice(g.dev));
    if (!enable) {
        for (auto &e : g.graphs) cudaGraphExecDestroy(e.exec);
        g.graphs.clear();
        g.seen.clear();
    }
    g.use_graphs = enable != 0;
    return SAL_OK;
}

extern "C" int sal_solve(sal_grid *G, const double *ssh, int32_t nf, int64_t ld_ssh, double *ox, double *oy,
                         int64_t ld_out, int32_t form, void *stream) {
    if (!G || !ssh || !ox || !oy) return set_error(SAL_EINVAL, "null argument");
    GridImpl &g = G->g;
    if (nf < 1) return set_error(SAL_EINVAL, "nfields must be >= 1");
    if (nf > 1 && (ld_ssh < g.plan.n || ld_out < g.plan.n)) return set_error(SAL_EINVAL, "leading dimension < point_count");
    if (form != SAL_FORM_REF && form != SAL_FORM_ACCURATE && form != SAL_FORM_MIXED)
        return set_error(SAL_EINVAL, "unsupported form");
    CK(cudaSetDevice(g.dev));
    cudaStream_t st = (cudaStream_t)stream;  // NULL: the CUDA default stream
    if (form == SAL_FORM_MIXED) {
        if (g.plan.mode != SAL_MODE_DTT) return set_error(SAL_EINVAL, "the batched form needs a SAL_MODE_DTT grid");
        const int FT = g.FT ? g.FT : (g.max_fields <= 32 ? 32 : 64);
        int rc = ensure_mixed(g, FT);
        if (rc) return rc;
        const GridImpl::GraphShape shape{ssh, nf, ld_ssh, ox, oy, ld_out};
        bool graph = false;
        {
            // the lock keeps sal_grid_set_graphs from destroying a graph
            // between its lookup and its launch
            std::lock_guard<std::mutex> lk(g.graph_mu);
            graph = g.use_graphs && st != nullptr && !g.timing;
            if (graph)
                for (const auto &e : g.graphs)
                    if (e.shape == shape) {
                        CK(cudaGraphLaunch(e.exec, st));
                        return SAL_OK;
                    }
        }
        for (int f0 = 0; f0 < nf; f0 += FT) solve_mixed_block(g, ssh, ld_ssh, f0, nf, ox, oy, ld_out, st);
        CK(cudaGetLastError());
        if (!graph) return SAL_OK;
        // a shape is captured on its second solve, so callers that pass fresh
        // buffers every call do not pay a capture per call
        std::lock_guard<std::mutex> lk(g.graph_mu);
        if (!g.use_graphs) return SAL_OK;
        for (size_t i = 0; i < g.seen.size(); ++i)
            if (g.seen[i] == shape) {
                g.seen.erase(g.seen.begin() + (std::ptrdiff_t)i);
                return capture_mixed(g, shape, st);
            }
        if (g.seen.size() >= kMaxGraphs) g.seen.erase(g.seen.begin());
        g.seen.push_back(shape);
        return SAL_OK;
    }
    for (int f = 0; f < nf; ++f)
        solve_fp64(g, ssh + (size_t)f * ld_ssh, ox + (size_t)f * ld_out, oy + (size_t)f * ld_out,
                   g.plan.mode == SAL_MODE_DTT ? form : SAL_FORM_REF, 7, true, st);
    CK(cudaGetLastError());
    return SAL_OK;
}

// ------------------------------------------------------------------ tuning of the batched form
static sal_tune tune_of(const GridImpl &g) {
    const TcOptions &o = g.plan.tc_opt;
    sal_tune t{};
    t.chain_ksteps = o.chain_ksteps;
    t.tree_passes = o.tree_passes;
    t.up_chunk = o.up_chunk;
    t.proxy_unit_kpairs = o.proxy_unit_kpairs;
    t.cta_groups = o.cta_groups;
    t.field_block = g.FT ? g.FT : (g.max_fields <= 32 ? 32 : 64);
    t.f16 = o.f16;
    t.tile_store = o.tile_store;
    return t;
}

static int apply_tune(GridImpl &g, const sal_tune &t) {
    if (t.field_block != 32 && t.field_block != 64) return set_error(SAL_EINVAL, "field_block must be 32 or 64");
    TcOptions o;
    o.chain_ksteps = t.chain_ksteps;
    o.tree_passes = t.tree_passes ? 1 : 0;
    o.up_chunk = t.up_chunk;
    o.proxy_unit_kpairs = t.proxy_unit_kpairs;
    o.cta_groups = t.cta_groups;
    o.f16 = t.f16 ? 1 : 0;
    if (t.tile_store < 0) return set_error(SAL_EINVAL, "tile_store must be >= 0");
    o.tile_store = t.tile_store;
    const TcOptions &c = g.plan.tc_opt;
    const bool same_plan = o.chain_ksteps == c.chain_ksteps && o.tree_passes == c.tree_passes &&
                           o.up_chunk == c.up_chunk && o.proxy_unit_kpairs == c.proxy_unit_kpairs &&
                           o.f16 == c.f16;
    const int cur_block = g.FT ? g.FT : (g.max_fields <= 32 ? 32 : 64);
    if (same_plan && t.field_block == cur_block) {
        if (o.cta_groups < 1) return set_error(SAL_EINVAL, "tcgen05 options must be positive");
        // the tile store is allocated with the batched buffers: switching it
        // frees them (the next solve allocates them again)
        if (o.tile_store != c.tile_store) {
            int rc = release_mixed(g);
            if (rc) return rc;
            plan_tile_offsets(&g.plan, o.tile_store > 1 ? o.tile_store : 1);
        }
        g.plan.tc_opt.cta_groups = o.cta_groups;
        g.plan.tc_opt.tile_store = o.tile_store;
        return SAL_OK;
    }
    int rc = release_mixed(g);
    if (rc) return rc;
    g.max_fields = t.field_block;
    if (!same_plan) {
        std::string err;
        if (!plan_build_tc(g.tree, &g.plan, o, &err)) return set_error(SAL_EINVAL, err);
    } else {
        g.plan.tc_opt.cta_groups = o.cta_groups;
        g.plan.tc_opt.tile_store = o.tile_store;
        plan_tile_offsets(&g.plan, o.tile_store > 1 ? o.tile_store : 1);
    }
    if (t.field_block == 32 && !g.plan.mix_built) plan_build_mix(g.tree, &g.plan);
    return SAL_OK;
}

extern "C" int sal_grid_tune_get(const sal_grid *G, sal_tune *t) {
    if (!G || !t) return set_error(SAL_EINVAL, "null argument");
    if (G->g.plan.mode != SAL_MODE_DTT) return set_error(SAL_EINVAL, "the batched form needs a SAL_MODE_DTT grid");
    *t = tune_of(G->g);
    return SAL_OK;
}

extern "C" int sal_grid_tune_set(sal_grid *G, const sal_tune *t) {
    if (!G || !t) return set_error(SAL_EINVAL, "null argument");
    GridImpl &g = G->g;
    if (g.plan.mode != SAL_MODE_DTT) return set_error(SAL_EINVAL, "the batched form needs a SAL_MODE_DTT grid");
    CK(cudaSetDevice(g.dev));
    return apply_tune(g, *t);
}

static int finish(GridImpl &g, cudaStream_t st);

extern "C" int sal_grid_autotune(sal_grid *G, const double *ssh, int32_t nf, int64_t ld, int32_t ntargets,
                                 double max_rel_err, sal_tune *best, double *ms_best, double *ms_start) {
    if (!G || !ssh || !best) return set_error(SAL_EINVAL, "null argument");
    GridImpl &g = G->g;
    const Plan &pl = g.plan;
    const int64_t n = pl.n;
    if (pl.mode != SAL_MODE_DTT) return set_error(SAL_EINVAL, "the batched form needs a SAL_MODE_DTT grid");
    if (nf < 1 || nf > 64) return set_error(SAL_EINVAL, "nfields must be in 1..64");
    if (nf > 1 && ld < n) return set_error(SAL_EINVAL, "leading dimension < point_count");
    if (ntargets < 1 || ntargets > n || ntargets > (1 << 20)) return set_error(SAL_EINVAL, "ntargets out of range");
    if (!(max_rel_err > 0)) return set_error(SAL_EINVAL, "max_rel_err must be positive");
    CK(cudaSetDevice(g.dev));
    cudaStream_t st = g.stream;
    // scratch: outputs, the pool-order sources of field 0, the FP64 direct
    // sum at the targets, an L2 flush buffer
    const int nt = ntargets;
    const int nch = dev::direct_chunks((int)n);
    const size_t flush_bytes = 256u << 20;
    double *out = nullptr, *src = nullptr, *ref = nullptr, *dscr = nullptr;
    double4 *pool = nullptr;
    int32_t *tg = nullptr;
    void *flush = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    std::vector<int32_t> tpos(nt), tidx(nt);
    std::vector<double> rx(nt), ry(nt), ox(n), oy(n);
    auto cleanup = [&]() {
        for (void *p : {(void *)out, (void *)src, (void *)ref, (void *)dscr, (void *)pool, (void *)tg, flush})
            if (p) cudaFree(p);
        if (e0) cudaEventDestroy(e0);
        if (e1) cudaEventDestroy(e1);
    };
#define TCK(call)                                                                                 \
    do {                                                                                          \
        cudaError_t e_ = (call);                                                                  \
        if (e_ != cudaSuccess) {                                                                  \
            cleanup();                                                                            \
            return set_error(SAL_ECUDA, std::string(#call) + ": " + cudaGetErrorString(e_));     \
        }                                                                                         \
    } while (0)
    TCK(cudaMalloc((void **)&out, 2 * (size_t)n * nf * sizeof(double)));
    TCK(cudaMalloc((void **)&src, 4 * (size_t)n * sizeof(double)));
    TCK(cudaMalloc((void **)&ref, 2 * (size_t)nt * sizeof(double)));
    TCK(cudaMalloc((void **)&dscr, (size_t)nch * nt * 2 * sizeof(double)));
    TCK(cudaMalloc((void **)&pool, (size_t)n * sizeof(double4)));
    TCK(cudaMalloc((void **)&tg, (size_t)nt * sizeof(int32_t)));
    TCK(cudaMalloc(&flush, flush_bytes));
    TCK(cudaEventCreate(&e0));
    TCK(cudaEventCreate(&e1));
    // evenly spaced caller indices; the direct sum runs over pool-order sources
    std::vector<int32_t> iperm(n);
    for (int64_t p = 0; p < n; ++p) iperm[pl.perm[p]] = (int32_t)p;
    for (int k = 0; k < nt; ++k) {
        tidx[k] = (int32_t)(((int64_t)k * n) / nt);
        tpos[k] = iperm[tidx[k]];
    }
    TCK(cudaMemcpy(tg, tpos.data(), nt * sizeof(int32_t), cudaMemcpyHostToDevice));
    dev::launch_prep(g.xyz, g.area, ssh, g.perm, (int)n, pool, st);
    for (int c = 0; c < 4; ++c)
        TCK(cudaMemcpy2DAsync(src + (size_t)c * n, sizeof(double), (const double *)pool + c, sizeof(double4), sizeof(double),
                              (size_t)n, cudaMemcpyDeviceToDevice, st));
    dev::launch_direct(src, src + n, src + 2 * n, src + 3 * n, (int)n, tg, nt, ref, ref + nt, dscr, nch, st);
    TCK(cudaMemcpyAsync(rx.data(), ref, nt * sizeof(double), cudaMemcpyDeviceToHost, st));
    TCK(cudaMemcpyAsync(ry.data(), ref + nt, nt * sizeof(double), cudaMemcpyDeviceToHost, st));
    TCK(cudaStreamSynchronize(st));
    double den = 0;
    for (int k = 0; k < nt; ++k) den += rx[k] * rx[k] + ry[k] * ry[k];
    double *oxd = out, *oyd = out + (size_t)n * nf;
    // time and check one setting: -1 if it failed to run
    auto evaluate = [&](const sal_tune &t, double *ms, double *err) -> int {
        int rc = apply_tune(g, t);
        if (rc) return rc;
        rc = sal_solve(G, ssh, nf, ld, oxd, oyd, n, SAL_FORM_MIXED, st);
        if (rc) return rc;
        rc = finish(g, st);
        if (rc) return rc;
        cudaMemcpy(ox.data(), oxd, (size_t)n * sizeof(double), cudaMemcpyDeviceToHost);
        cudaMemcpy(oy.data(), oyd, (size_t)n * sizeof(double), cudaMemcpyDeviceToHost);
        double num = 0;
        for (int k = 0; k < nt; ++k) {
            const double dx = ox[tidx[k]] - rx[k], dy = oy[tidx[k]] - ry[k];
            num += dx * dx + dy * dy;
        }
        *err = den > 0 ? std::sqrt(num / den) : std::sqrt(num);
        double tmin = 1e30;
        for (int r = 0; r < 3; ++r) {
            cudaMemsetAsync(flush, r & 0xff, flush_bytes, st);
            cudaEventRecord(e0, st);
            rc = sal_solve(G, ssh, nf, ld, oxd, oyd, n, SAL_FORM_MIXED, st);
            if (rc) return rc;
            cudaEventRecord(e1, st);
            cudaEventSynchronize(e1);
            float t_ms = 0;
            cudaEventElapsedTime(&t_ms, e0, e1);
            tmin = std::min(tmin, (double)t_ms);
        }
        *ms = tmin;
        return finish(g, st);
    };
    sal_tune cur = tune_of(g), top = cur;
    double top_ms = 0, top_err = 0;
    int rc = evaluate(cur, &top_ms, &top_err);
    if (rc) { cleanup(); return rc; }
    const double start_ms = top_ms;
    const bool start_ok = top_err <= max_rel_err;
    if (!start_ok) top_ms = 1e30;   // any passing setting beats a failing start
    // coordinate descent: each choice's candidates with the others held at
    // the best so far; the leaf pass's choices (chain length, operand
    // precision, groups per CTA) interact, so they are swept again at the end
    struct Axis { int32_t sal_tune::*field; std::vector<int32_t> values; };
    const std::vector<Axis> axes = {
        {&sal_tune::tree_passes, {1, 0}},
        {&sal_tune::chain_ksteps, {8, 16, 32, 64}},
        {&sal_tune::f16, {0, 1}},
        {&sal_tune::cta_groups, {1, 2, 4}},
        {&sal_tune::proxy_unit_kpairs, {324, 648, 1296}},
        {&sal_tune::up_chunk, {2048, 4096, 8192}},
        {&sal_tune::field_block, {64, 32}},
        {&sal_tune::chain_ksteps, {32, 64}},
        {&sal_tune::f16, {0, 1}},
        {&sal_tune::cta_groups, {1, 2, 4}},
    };
    for (const Axis &ax : axes) {
        if (ax.field == &sal_tune::up_chunk && top.tree_passes) continue;   // only the direct upward pass uses it
        for (int32_t v : ax.values) {
            if (top.*(ax.field) == v) continue;
            sal_tune t = top;
            t.*(ax.field) = v;
            double ms = 0, err = 0;
            rc = evaluate(t, &ms, &err);
            if (rc) { cleanup(); return rc; }
            if (err <= max_rel_err && ms < top_ms) { top = t; top_ms = ms; top_err = err; }
        }
    }
    if (top_ms >= 1e30) {
        apply_tune(g, cur);
        cleanup();
        return set_error(SAL_EINVAL, "no setting meets max_rel_err");
    }
    rc = apply_tune(g, top);
    cleanup();
    if (rc) return rc;
    *best = top;
    if (ms_best) *ms_best = top_ms;
    if (ms_start) *ms_start = start_ms;
    return SAL_OK;
#undef TCK
}

// Synchronises the grid's work on `stream` and reports a kernel time-out.
// The flag travels on that stream (no default-stream copy), so a grid's
// synchronisation never waits on other streams' work.
static int finish(GridImpl &g, cudaStream_t st) {
    CK(cudaMemcpyAsync(g.h_flag, g.err, sizeof(int), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    const int flag = *g.h_flag;
    if (flag) {
        g.tile_recorded = false;   // a recording pass may have given up: record again
        cudaMemsetAsync(g.err, 0, sizeof(int), st);
        cudaStreamSynchronize(st);
        return set_error(SAL_ETIMEOUT, "a staging wait timed out on the device");
    }
    return SAL_OK;
}

extern "C" int sal_grid_timing(sal_grid *G, int32_t enable, double *phase_ms, int64_t *solves) {
    if (!G) return set_error(SAL_EINVAL, "null argument");
    GridImpl &g = G->g;
    CK(cudaSetDevice(g.dev));
    if (phase_ms)
        for (int i = 0; i < 4; ++i) phase_ms[i] = g.phase_ms[i];
    if (solves) *solves = g.phase_solves;
    if (enable >= 0) {
        if (enable && !g.ev[0])
            for (auto &e : g.ev) CK(cudaEventCreate(&e));
        g.timing = enable != 0;
        for (double &v : g.phase_ms) v = 0;
        g.phase_solves = 0;
    }
    return SAL_OK;
}

extern "C" int sal_grid_inject_timeout(sal_grid *G, int32_t polls) {
    if (!G) return set_error(SAL_EINVAL, "null argument");
    if (polls < 0) return set_error(SAL_EINVAL, "polls must be >= 0");
    G->g.inject_polls = (uint32_t)polls;
    return SAL_OK;
}

extern "C" int sal_grid_sync(sal_grid *G, void *stream) {
    if (!G) return set_error(SAL_EINVAL, "null argument");
    CK(cudaSetDevice(G->g.dev));
    return finish(G->g, stream ? (cudaStream_t)stream : G->g.stream);
}

static int ensure_host_staging(GridImpl &g) {
    if (g.h_ssh) return SAL_OK;
    const size_t n = (size_t)g.plan.n;
    int rc = dalloc(g, &g.h_ssh, n);
    if (!rc) rc = dalloc(g, &g.h_ox, n);
    if (!rc) rc = dalloc(g, &g.h_oy, n);
    if (!rc) rc = dalloc(g, &g.h_w, (size_t)g.plan.P * std::max(1, g.nsrc));
    return rc;
}

// Adds device results into the caller's intent(inout) host arrays.
static int add_back(GridImpl &g, double *hx, double *hy) {
    const size_t n = (size_t)g.plan.n;
    std::vector<double> tx(n), ty(n);
    CK(cudaMemcpyAsync(tx.data(), g.h_ox, n * 8, cudaMemcpyDeviceToHost, g.stream));
    CK(cudaMemcpyAsync(ty.data(), g.h_oy, n * 8, cudaMemcpyDeviceToHost, g.stream));
    int rc = finish(g, g.stream);
    if (rc) return rc;
    for (size_t i = 0; i < n; ++i) {
        hx[i] += tx[i];
        hy[i] += ty[i];
    }
    return SAL_OK;
}

extern "C" int sal_solve_host(sal_grid *G, const double *ssh, int32_t nf, int64_t ld_ssh, double *ox, double *oy,
                              int64_t ld_out, int32_t form) {
    if (!G || !ssh || !ox || !oy) return set_error(SAL_EINVAL, "null argument");
    GridImpl &g = G->g;
    const int64_t n = g.plan.n;
    if (nf < 1) return set_error(SAL_EINVAL, "nfields must be >= 1");
    if (nf > 1 && (ld_ssh < n || ld_out < n)) return set_error(SAL_EINVAL, "leading dimension < point_count");
    std::lock_guard<std::mutex> lk(g.mu);
    CK(cudaSetDevice(g.dev));
    if (g.hb_fields < nf) {
        // the old staging is too small: release it (after the grid's stream
        // has finished with it) before taking a larger one
        CK(cudaStreamSynchronize(g.stream));
        const size_t old = (size_t)n * g.hb_fields;
        dfree(g, &g.hb_ssh, old);
        dfree(g, &g.hb_ox, old);
        dfree(g, &g.hb_oy, old);
        g.hb_fields = 0;
        int rc = dalloc(g, &g.hb_ssh, (size_t)n * nf);
        if (!rc) rc = dalloc(g, &g.hb_ox, (size_t)n * nf);
        if (!rc) rc = dalloc(g, &g.hb_oy, (size_t)n * nf);
        if (rc) return rc;
        g.hb_fields = nf;
    }
    for (int f = 0; f < nf; ++f)
        CK(cudaMemcpyAsync(g.hb_ssh + (size_t)f * n, ssh + (size_t)f * ld_ssh, (size_t)n * 8, cudaMemcpyHostToDevice,
                           g.stream));
    int rc = sal_solve(G, g.hb_ssh, nf, n, g.hb_ox, g.hb_oy, n, form, g.stream);
    if (rc) return rc;
    for (int f = 0; f < nf; ++f) {
        CK(cudaMemcpyAsync(ox + (size_t)f * ld_out, g.hb_ox + (size_t)f * n, (size_t)n * 8, cudaMemcpyDeviceToHost,
                           g.stream));
        CK(cudaMemcpyAsync(oy + (size_t)f * ld_out, g.hb_oy + (size_t)f * n, (size_t)n * 8, cudaMemcpyDeviceToHost,
                           g.stream));
    }
    return finish(g, g.stream);
}

// Slot k's buffers are reused two calls later: its copy in waits for the solve
// that read its fields, and its solve waits for the copy out of its results.
extern "C" int sal_solve_host_async(sal_grid *G, const double *ssh, int32_t nf, int64_t ld_ssh, double *ox, double *oy,
                                    int64_t ld_out, int32_t form) {
    if (!G || !ssh || !ox || !oy) return set_error(SAL_EINVAL, "null argument");
    GridImpl &g = G->g;
    const int64_t n = g.plan.n;
    if (nf < 1) return set_error(SAL_EINVAL, "nfields must be >= 1");
    if (nf > 1 && (ld_ssh < n || ld_out < n)) return set_error(SAL_EINVAL, "leading dimension < point_count");
    std::lock_guard<std::mutex> lk(g.mu);
    CK(cudaSetDevice(g.dev));
    if (!g.s_in) {
        CK(cudaStreamCreateWithFlags(&g.s_in, cudaStreamNonBlocking));
        CK(cudaStreamCreateWithFlags(&g.s_out, cudaStreamNonBlocking));
        for (auto &h : g.hslot)
            for (cudaEvent_t *e : {&h.in, &h.solved, &h.out}) CK(cudaEventCreateWithFlags(e, cudaEventDisableTiming));
    }
    GridImpl::HostSlot &h = g.hslot[g.hnext];
    g.hnext ^= 1;
    if (h.fields < nf) {
        // the slot's last copy out has read its results, which follow its
        // solve: after that nothing uses the old buffers
        if (h.used) CK(cudaEventSynchronize(h.out));
        const size_t old = (size_t)n * (size_t)h.fields;
        dfree(g, &h.ssh, old);
        dfree(g, &h.ox, old);
        dfree(g, &h.oy, old);
        h.fields = 0;
        int rc = dalloc(g, &h.ssh, (size_t)n * nf);
        if (!rc) rc = dalloc(g, &h.ox, (size_t)n * nf);
        if (!rc) rc = dalloc(g, &h.oy, (size_t)n * nf);
        if (rc) return rc;
        h.fields = nf;
    }
    if (h.used) CK(cudaStreamWaitEvent(g.s_in, h.solved, 0));
    for (int f = 0; f < nf; ++f)
        CK(cudaMemcpyAsync(h.ssh + (size_t)f * n, ssh + (size_t)f * ld_ssh, (size_t)n * 8, cudaMemcpyHostToDevice,
                           g.s_in));
    CK(cudaEventRecord(h.in, g.s_in));
    CK(cudaStreamWaitEvent(g.stream, h.in, 0));
    if (h.used) CK(cudaStreamWaitEvent(g.stream, h.out, 0));
    int rc = sal_solve(G, h.ssh, nf, n, h.ox, h.oy, n, form, g.stream);
    if (rc) return rc;
    CK(cudaEventRecord(h.solved, g.stream));
    CK(cudaStreamWaitEvent(g.s_out, h.solved, 0));
    for (int f = 0; f < nf; ++f) {
        CK(cudaMemcpyAsync(ox + (size_t)f * ld_out, h.ox + (size_t)f * n, (size_t)n * 8, cudaMemcpyDeviceToHost,
                           g.s_out));
        CK(cudaMemcpyAsync(oy + (size_t)f * ld_out, h.oy + (size_t)f * n, (size_t)n * 8, cudaMemcpyDeviceToHost,
                           g.s_out));
    }
    CK(cudaEventRecord(h.out, g.s_out));
    h.used = true;
    return SAL_OK;
}

extern "C" int sal_solve_host_wait(sal_grid *G) {
    if (!G) return set_error(SAL_EINVAL, "null argument");
    GridImpl &g = G->g;
    std::lock_guard<std::mutex> lk(g.mu);
    CK(cudaSetDevice(g.dev));
    if (g.s_out) CK(cudaStreamSynchronize(g.s_out));
    return finish(g, g.stream);
}

extern "C" int sal_fast_sum_host(sal_grid *G, const double *ssh, double *lon, double *lat, int32_t form) {
    if (!G || !ssh || !lon || !lat) return set_error(SAL_EINVAL, "null argument");
    GridImpl &g = G->g;
    if (g.plan.mode != SAL_MODE_DTT) return set_error(SAL_EINVAL, "fast_sum needs a SAL_MODE_DTT grid");
    if (form != SAL_FORM_REF && form != SAL_FORM_ACCURATE) return set_error(SAL_EINVAL, "unsupported form");
    std::lock_guard<std::mutex> lk(g.mu);
    CK(cudaSetDevice(g.dev));
    int rc = ensure_host_staging(g);
    if (rc) return rc;
    CK(cudaMemcpyAsync(g.h_ssh, ssh, (size_t)g.plan.n * 8, cudaMemcpyHostToDevice, g.stream));
    solve_fp64(g, g.h_ssh, g.h_ox, g.h_oy, form, 7, true, g.stream);
    CK(cudaGetLastError());
    return add_back(g, lon, lat);
}

extern "C" int sal_proxy_source_compute_host(sal_grid *G, const double *sshs, double *weights) {
    if (!G || !sshs || !weights) return set_error(SAL_EINVAL, "null argument");
    GridImpl &g = G->g;
    if (g.plan.mode == SAL_MODE_DTT) return set_error(SAL_EINVAL, "proxy_source_compute needs an STT grid");
    std::lock_guard<std::mutex> lk(g.mu);
    CK(cudaSetDevice(g.dev));
    int rc = ensure_host_staging(g);
    if (rc) return rc;
    const Plan &pl = g.plan;
    const int n = pl.n, P = pl.P;
    CK(cudaMemcpyAsync(g.h_ssh, sshs, (size_t)n * 8, cudaMemcpyHostToDevice, g.stream));
    dev::launch_prep(g.xyz, g.area, g.h_ssh, g.perm, n, g.pool, g.stream);
    dev::UpArgs u{g.pool, g.xieta, g.up_units, g.src_nodes, pl.d, P, g.up_partial};
    dev::launch_upward(u, g.nup, g.stream);
    dev::launch_upward_finalize(g.up_unit_beg, g.up_partial, g.nsrc, pl.d, pl.mode == SAL_MODE_STT_REF_COMPAT ? 1 : 0,
                                g.pool + n, g.stream);
    const size_t cnt = (size_t)P * g.nsrc;
    dev::launch_extract_w(g.pool + n, (int)cnt, g.h_w, g.stream);
    std::vector<double> w(cnt);
    CK(cudaMemcpyAsync(w.data(), g.h_w, cnt * 8, cudaMemcpyDeviceToHost, g.stream));
    rc = finish(g, g.stream);
    if (rc) return rc;
    for (size_t i = 0; i < cnt; ++i) weights[i] += w[i];
    return SAL_OK;
}

extern "C" int sal_pc_compute_host(sal_grid *G, const double *weights, double *sx, double *sy) {
    if (!G || !weights || !sx || !sy) return set_error(SAL_EINVAL, "null argument");
    GridImpl &g = G->g;
    if (g.plan.mode == SAL_MODE_DTT) return set_error(SAL_EINVAL, "pc_compute needs an STT grid");
    std::lock_guard<std::mutex> lk(g.mu);
    CK(cudaSetDevice(g.dev));
    int rc = ensure_host_staging(g);
    if (rc) return rc;
    const size_t cnt = (size_t)g.plan.P * g.nsrc;
    CK(cudaMemcpyAsync(g.h_w, weights, cnt * 8, cudaMemcpyHostToDevice, g.stream));
    dev::launch_insert_w(g.h_w, (int)cnt, g.pool + g.plan.n, g.stream);
    // PC items only: point weights are not read, so no prep is needed
    dev::EvalArgs a{};
    a.pool = g.pool; a.groups = g.leaf_groups; a.items = g.leaf_items; a.masks = g.masks; a.tgt = g.pool;
    a.xieta = g.xieta; a.records = g.records; a.rec_stride = g.rec_stride; a.d = g.plan.d; a.P = g.plan.P;
    a.kinds = 2; a.perm = g.perm; a.out_x = g.h_ox; a.out_y = g.h_oy; a.err = g.err;
    dev::launch_eval(0, SAL_FORM_REF, a, (int)g.plan.leaf_groups.size(), g.stream);
    CK(cudaGetLastError());
    return add_back(g, sx, sy);
}

extern "C" int sal_pp_compute_host(sal_grid *G, const double *sshs, double *sx, double *sy) {
    if (!G || !sshs || !sx || !sy) return set_error(SAL_EINVAL, "null argument");
    GridImpl &g = G->g;
    if (g.plan.mode == SAL_MODE_DTT) return set_error(SAL_EINVAL, "pp_compute needs an STT grid");
    std::lock_guard<std::mutex> lk(g.mu);
    CK(cudaSetDevice(g.dev));
    int rc = ensure_host_staging(g);
    if (rc) return rc;
    CK(cudaMemcpyAsync(g.h_ssh, sshs, (size_t)g.plan.n * 8, cudaMemcpyHostToDevice, g.stream));
    dev::launch_prep(g.xyz, g.area, g.h_ssh, g.perm, g.plan.n, g.pool, g.stream);
    dev::EvalArgs a{};
    a.pool = g.pool; a.groups = g.leaf_groups; a.items = g.leaf_items; a.masks = g.masks; a.tgt = g.pool;
    a.xieta = g.xieta; a.records = g.records; a.rec_stride = g.rec_stride; a.d = g.plan.d; a.P = g.plan.P;
    a.kinds = 1; a.perm = g.perm; a.out_x = g.h_ox; a.out_y = g.h_oy; a.err = g.err;
    dev::launch_eval(0, SAL_FORM_REF, a, (int)g.plan.leaf_groups.size(), g.stream);
    CK(cudaGetLastError());
    return add_back(g, sx, sy);
}

// Scratch of the direct sum: per-device lazily grown buffer.
static std::mutex g_direct_mu;
static double *g_direct_scratch[64] = {nullptr};
static size_t g_direct_cap[64] = {0};

extern "C" int sal_direct_sum(const double *xs, const double *ys, const double *zs, const double *w, int32_t n,
                              const int32_t *targets, int32_t nt, double *ox, double *oy, void *stream) {
    if (!xs || !ys || !zs || !w || !targets || !ox || !oy) return set_error(SAL_EINVAL, "null argument");
    if (n < 0 || nt < 0) return set_error(SAL_EINVAL, "negative size");
    int dev = 0;
    CK(cudaGetDevice(&dev));
    if (dev >= 64) return set_error(SAL_EINVAL, "device ordinal >= 64");
    const int nch = dev::direct_chunks(n);
    const size_t need = (size_t)nch * (size_t)nt * 2;
    std::lock_guard<std::mutex> lk(g_direct_mu);
    if (g_direct_cap[dev] < need) {
        if (g_direct_scratch[dev]) cudaFree(g_direct_scratch[dev]);
        g_direct_scratch[dev] = nullptr;
        g_direct_cap[dev] = 0;
        if (cudaMalloc((void **)&g_direct_scratch[dev], need * 8) != cudaSuccess)
            return set_error(SAL_ENOMEM, "direct-sum scratch allocation failed");
        g_direct_cap[dev] = need;
    }
    dev::launch_direct(xs, ys, zs, w, n, targets, nt, ox, oy, g_direct_scratch[dev], nch, (cudaStream_t)stream);
    CK(cudaGetLastError());
    return SAL_OK;
}
