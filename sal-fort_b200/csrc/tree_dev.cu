// Device build of the cubed-sphere quadtree and of the dual-tree interaction
// list (tree_module.f90:59-246 and 277-398), for fast admission of new grids.
//
// The results have the host build's layout and order:
//  - panels in the reference's BFS order.  The host refines panel i before
//    panel i+1 and appends its four children, so the panels of one level are
//    contiguous and their children follow in parent order.  Here one level is
//    refined per step: a scan over the level's split flags gives each split
//    panel its children's first index.
//  - every panel a contiguous range of one permutation, its points in
//    increasing point index (the host's stable 4-way partitions).  Here the
//    points are stably sorted by their leaf's first position.
//  - the list in the reference's FIFO order.  The queue of panel pairs is
//    processed in generations (the 36 root pairs, then their refinements in
//    queue order, ...): FIFO processing finishes one generation before the
//    next, and stable scans keep each generation's order.
//
// Every floating-point decision is the host build's, bit for bit:
//  - the per-point (xi, eta) and the panels' radii and MAC centres come from
//    the host's glibc atan, tan and acos (tree.cpp, on every host thread;
//    they are a small part of the build), so the device compares exactly the
//    host's values against midpoints formed by the same operations (this
//    file is built with -fmad=false);
//  - the MAC's arc distance is CUDA's acos on the device.  A pair whose ratio
//    lies within 1e-12 of theta is decided again on the host (dtt_decide),
//    so an ulp of difference between the two acos cannot flip it.
// Grids with points exactly on panel midlines (a lon-lat grid has whole
// columns there) therefore give the host's tree and list.
#include <cuda_runtime.h>

#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>

#include <cmath>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/salgpu.h"
#include "sal_internal.hpp"

namespace sal {
int set_error(int code, const std::string &msg);

namespace {

constexpr int kMaxLevel = 40;  // as the host build: identical points would refine forever
constexpr int kThreads = 256;

struct DPanel {
    double mn_xi, md_xi, mx_xi, mn_eta, md_eta, mx_eta;
    int64_t begin;
    int32_t count, level, parent, child0, face, split;
};

inline int blocks_for(int64_t n) { return (int)((n + kThreads - 1) / kThreads); }

__device__ double dev_clamp_acos(double v) {
    v = v > -1.0 ? v : -1.0;
    v = v < 1.0 ? v : 1.0;
    return acos(v);
}

// Per point: its face's root panel, counted.
__global__ void roots_kernel(const int8_t *__restrict__ face, int32_t n, int32_t *__restrict__ panel, DPanel *P) {
    int32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int f = face[i];
    panel[i] = f - 1;
    atomicAdd(&P[f - 1].count, 1);
}

// tree_module.f90:80: a leaf with at least thresh points is refined.
__global__ void split_flags_kernel(DPanel *P, int32_t lo, int32_t hi, int32_t thresh, int32_t *flag) {
    int32_t k = lo + blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= hi) return;
    int s = P[k].count >= thresh && P[k].level < kMaxLevel;
    P[k].split = s;
    flag[k - lo] = s;
}

// The four children of every split panel of [lo, hi): SW, SE, NE, NW, each
// bounded by the parent's min/mid/max (tree_module.f90:92-177).
__global__ void children_kernel(DPanel *P, int32_t lo, int32_t hi, const int32_t *__restrict__ rank) {
    int32_t k = lo + blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= hi || !P[k].split) return;
    const DPanel par = P[k];
    int32_t c0 = hi + 4 * rank[k - lo];
    P[k].child0 = c0;
    const double bx[4][2] = {{par.mn_xi, par.md_xi}, {par.md_xi, par.mx_xi}, {par.md_xi, par.mx_xi}, {par.mn_xi, par.md_xi}};
    const double be[4][2] = {{par.mn_eta, par.md_eta}, {par.mn_eta, par.md_eta}, {par.md_eta, par.mx_eta}, {par.md_eta, par.mx_eta}};
    for (int j = 0; j < 4; ++j) {
        DPanel c{};
        c.mn_xi = bx[j][0]; c.mx_xi = bx[j][1]; c.md_xi = 0.5 * (bx[j][0] + bx[j][1]);
        c.mn_eta = be[j][0]; c.mx_eta = be[j][1]; c.md_eta = 0.5 * (be[j][0] + be[j][1]);
        c.level = par.level + 1; c.parent = k; c.child0 = -1; c.face = par.face;
        P[c0 + j] = c;
    }
}

// Every point of a panel refined this step moves to the child that holds it
// (tree_module.f90:179-205: xi < mid_xi, eta < mid_eta).
__global__ void move_points_kernel(const double *__restrict__ xi, const double *__restrict__ eta,
                                   int32_t *__restrict__ panel, int32_t n, DPanel *P, int32_t lo, int32_t hi) {
    int32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    int32_t k = panel[i];
    if (k < lo || k >= hi || !P[k].split) return;
    double mdx = P[k].md_xi, mde = P[k].md_eta;
    double a = xi[i], b = eta[i];
    int w = (a < mdx) ? ((b < mde) ? 0 : 3) : ((b < mde) ? 1 : 2);
    int32_t c = P[k].child0 + w;
    panel[i] = c;
    atomicAdd(&P[c].count, 1);
}

// First positions: the roots in face order, children in order inside their
// parent's range.
__global__ void root_begin_kernel(DPanel *P) {
    if (threadIdx.x || blockIdx.x) return;
    int64_t b = 0;
    for (int f = 0; f < 6; ++f) { P[f].begin = b; b += P[f].count; }
}

__global__ void child_begin_kernel(DPanel *P, int32_t lo, int32_t hi) {
    int32_t k = lo + blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= hi || !P[k].split) return;
    int64_t b = P[k].begin;
    for (int j = 0; j < 4; ++j) { P[P[k].child0 + j].begin = b; b += P[P[k].child0 + j].count; }
}

__global__ void sort_keys_kernel(const int32_t *__restrict__ panel, const DPanel *__restrict__ P, int32_t n,
                                 uint32_t *__restrict__ key, int32_t *__restrict__ idx) {
    int32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    key[i] = (uint32_t)P[panel[i]].begin;
    idx[i] = i;
}

// ------------------------------------------------------------ dual traversal
struct DttPanel {
    double radius, cx, cy, cz;
    int32_t count, leaf, child[4];  // children: 1-based panel ids
};

// Decision for one queued pair (tree_module.f90:300-392), as dtt_decide:
//   0 empty panel, 1..4 list entry of type code-1, 5 refine the source,
//   6 refine the target.  packed: (4 if refined) << 32 | (1 if listed).
// A MAC ratio within kMacTie of theta is left to the host (code kUndecided,
// index appended to amb; amb_cap bounds the list, *namb counts them all).
constexpr uint8_t kUndecided = 255;
constexpr double kMacTie = 1e-12;

__device__ __forceinline__ unsigned long long dtt_packed(uint8_t c) {
    return (c >= 5 && c <= 6 ? (4ull << 32) : 0ull) | (c >= 1 && c <= 4 ? 1ull : 0ull);
}

__global__ void dtt_classify_kernel(const int2 *__restrict__ q, int64_t m, const DttPanel *__restrict__ P,
                                    double theta, int32_t thresh, uint8_t *__restrict__ code,
                                    unsigned long long *__restrict__ packed, int64_t *__restrict__ amb,
                                    int64_t amb_cap, unsigned long long *__restrict__ namb) {
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m) return;
    const int2 pr = q[i];
    const DttPanel T = P[pr.x - 1], S = P[pr.y - 1];
    int64_t ct = T.count, cs = S.count;
    uint8_t c = 0;
    if (ct > 0 && cs > 0) {
        double dist = dev_clamp_acos(T.cx * S.cx + T.cy * S.cy + T.cz * S.cz);
        double sep = (T.radius + S.radius) / dist;
        if (dist > 0 && fabs(sep - theta) <= kMacTie * theta) {
            c = kUndecided;
            const unsigned long long k = atomicAdd(namb, 1ull);
            if ((int64_t)k < amb_cap) amb[k] = i;
        } else if (dist > 0 && sep < theta) {
            c = (uint8_t)(1 + (ct > thresh ? 2 : 0) + (cs > thresh ? 1 : 0));
        } else if ((ct < thresh && cs < thresh) || (T.leaf && S.leaf)) {
            c = 1;
        } else {
            bool refine_source = T.leaf ? true : (S.leaf ? false : !(ct >= cs));
            c = refine_source ? 5 : 6;
        }
    }
    code[i] = c;
    packed[i] = dtt_packed(c);
}

__global__ void dtt_gather_kernel(const int2 *__restrict__ q, const int64_t *__restrict__ amb, int64_t na,
                                  int2 *__restrict__ out) {
    int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (k < na) out[k] = q[amb[k]];
}

// The host's decisions for the undecided pairs.
__global__ void dtt_patch_kernel(const int64_t *__restrict__ amb, const uint8_t *__restrict__ decided, int64_t na,
                                 uint8_t *__restrict__ code, unsigned long long *__restrict__ packed) {
    int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= na) return;
    const int64_t i = amb[k];
    code[i] = decided[k];
    packed[i] = dtt_packed(decided[k]);
}

__global__ void dtt_scatter_kernel(const int2 *__restrict__ q, int64_t m, const DttPanel *__restrict__ P,
                                   const uint8_t *__restrict__ code, const unsigned long long *__restrict__ excl,
                                   int32_t *__restrict__ list, int64_t list_base, int2 *__restrict__ next) {
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m) return;
    const uint8_t c = code[i];
    if (c == 0) return;
    const int2 pr = q[i];
    const unsigned long long e = excl[i];
    if (c <= 4) {
        int32_t *o = list + 3 * (list_base + (int64_t)(e & 0xffffffffull));
        o[0] = pr.x; o[1] = pr.y; o[2] = c - 1;
    } else {
        int2 *o = next + (e >> 32);
        const DttPanel &R = c == 5 ? P[pr.y - 1] : P[pr.x - 1];
        for (int j = 0; j < 4; ++j) o[j] = c == 5 ? make_int2(pr.x, R.child[j]) : make_int2(R.child[j], pr.y);
    }
}

// ------------------------------------------------------------ host plumbing
// Stream-ordered scratch from a memory pool of the library's own per device,
// which keeps up to kPoolKeep bytes between builds: cudaMalloc and cudaFree
// (which synchronises the device) would cost more than building a small grid.
constexpr uint64_t kPoolKeep = 1ull << 30;
constexpr int kMaxDevices = 64;
std::mutex g_pool_mu;
cudaMemPool_t g_pool[kMaxDevices] = {};

cudaError_t pool_of(int dev, cudaMemPool_t *out) {
    std::lock_guard<std::mutex> lk(g_pool_mu);
    if (dev < 0 || dev >= kMaxDevices) return cudaErrorInvalidDevice;
    if (!g_pool[dev]) {
        cudaMemPoolProps props{};
        props.allocType = cudaMemAllocationTypePinned;
        props.location.type = cudaMemLocationTypeDevice;
        props.location.id = dev;
        cudaMemPool_t p = nullptr;
        cudaError_t e = cudaMemPoolCreate(&p, &props);
        if (e != cudaSuccess) return e;
        uint64_t keep = kPoolKeep;
        e = cudaMemPoolSetAttribute(p, cudaMemPoolAttrReleaseThreshold, &keep);
        if (e != cudaSuccess) {
            cudaMemPoolDestroy(p);
            return e;
        }
        g_pool[dev] = p;
    }
    *out = g_pool[dev];
    return cudaSuccess;
}

// Device buffers of one build, freed in stream order on every exit path.
struct Scratch {
    cudaStream_t st = nullptr;
    cudaMemPool_t pool = nullptr;
    std::vector<void *> ptrs;
    ~Scratch() {
        for (void *p : ptrs)
            if (p) cudaFreeAsync(p, st);
    }
    template <class T>
    cudaError_t get(T **p, size_t count) {
        *p = nullptr;
        if (count == 0) count = 1;
        cudaError_t e = cudaMallocFromPoolAsync((void **)p, count * sizeof(T), pool, st);
        if (e == cudaSuccess) ptrs.push_back(*p);
        return e;
    }
    void drop(void *p) {
        for (auto &q : ptrs)
            if (q == p) { cudaFreeAsync(q, st); q = nullptr; }
    }
};

struct DeviceGuard {
    int prev = -1;
    cudaStream_t st = nullptr;
    ~DeviceGuard() {
        if (st) cudaStreamDestroy(st);
        if (prev >= 0) cudaSetDevice(prev);
    }
};

int cuda_fail(cudaError_t e, const char *what) {
    return set_error(e == cudaErrorMemoryAllocation ? SAL_ENOMEM : SAL_ECUDA,
                     std::string(what) + ": " + cudaGetErrorString(e));
}

#define DCK(call)                                       \
    do {                                                \
        cudaError_t e_ = (call);                        \
        if (e_ != cudaSuccess) return cuda_fail(e_, #call); \
    } while (0)

int enter_device(int device, DeviceGuard *g, Scratch *S) {
    DCK(cudaGetDevice(&g->prev));
    DCK(cudaSetDevice(device));
    DCK(cudaStreamCreateWithFlags(&g->st, cudaStreamNonBlocking));
    DCK(pool_of(device, &S->pool));
    S->st = g->st;
    return SAL_OK;
}

// Makes *p hold at least `need` elements (contents not kept).  The old
// buffer is freed in stream order, after the kernels queued before.
template <class T>
int ensure(Scratch &S, T **p, int64_t *cap, int64_t need, cudaStream_t st) {
    (void)st;
    if (need <= *cap && *p) return SAL_OK;
    int64_t nc = std::max<int64_t>(std::max<int64_t>(need, 1), 2 * *cap);
    if (*p) S.drop(*p);
    DCK(S.get(p, (size_t)nc));
    *cap = nc;
    return SAL_OK;
}

// The same, keeping the first `used` elements.
template <class T>
int grow_keep(Scratch &S, T **p, int64_t *cap, int64_t used, int64_t need, cudaStream_t st) {
    if (need <= *cap) return SAL_OK;
    int64_t nc = std::max<int64_t>(need, 2 * *cap);
    T *np = nullptr;
    DCK(S.get(&np, (size_t)nc));
    if (used > 0) DCK(cudaMemcpyAsync(np, *p, (size_t)used * sizeof(T), cudaMemcpyDeviceToDevice, st));
    S.drop(*p);
    *p = np;
    *cap = nc;
    return SAL_OK;
}


}  // namespace

// tree_traverse (tree_module.f90:59-246) with the refinement on the device;
// the result is the host Tree the rest of the setup consumes.
int tree_build_device(const double *xs, const double *ys, const double *zs, int32_t n, int32_t thresh, int device,
                      Tree **out) {
    *out = nullptr;
    DeviceGuard dg;
    Scratch S;
    if (int rc = enter_device(device, &dg, &S)) return rc;
    cudaStream_t st = dg.st;
    std::unique_ptr<Tree> own(new Tree());
    Tree *t = own.get();
    t->n = n;
    // faces and (xi, eta) with the host's libm, on every host thread
    tree_set_points(t, xs, ys, zs);
    double *dxi = nullptr, *deta = nullptr;
    int8_t *dface = nullptr;
    int32_t *dpanel = nullptr, *didx = nullptr, *didx2 = nullptr;
    uint32_t *dkey = nullptr, *dkey2 = nullptr;
    DCK(S.get(&dxi, n)); DCK(S.get(&deta, n)); DCK(S.get(&dface, n)); DCK(S.get(&dpanel, n));
    if (n > 0) {
        DCK(cudaMemcpyAsync(dxi, t->xi.data(), (size_t)n * 8, cudaMemcpyHostToDevice, st));
        DCK(cudaMemcpyAsync(deta, t->eta.data(), (size_t)n * 8, cudaMemcpyHostToDevice, st));
        DCK(cudaMemcpyAsync(dface, t->face.data(), (size_t)n, cudaMemcpyHostToDevice, st));
    }

    // the six face roots, bounded by +-pi/4 as tree_module.f90:65-78
    const double pi = 4.0 * std::atan(1.0);
    std::vector<DPanel> roots(6);
    for (int f = 0; f < 6; ++f) {
        DPanel &q = roots[f];
        q = DPanel{};
        q.mn_xi = -pi / 4.0; q.md_xi = 0.0; q.mx_xi = pi / 4.0;
        q.mn_eta = -pi / 4.0; q.md_eta = 0.0; q.mx_eta = pi / 4.0;
        q.face = f + 1; q.parent = -1; q.child0 = -1;
    }
    int64_t cap = 6 + 8 * ((int64_t)n / std::max(1, thresh) + 8);
    DPanel *P = nullptr;
    DCK(S.get(&P, (size_t)cap));
    DCK(cudaMemcpyAsync(P, roots.data(), 6 * sizeof(DPanel), cudaMemcpyHostToDevice, st));
    if (n > 0) roots_kernel<<<blocks_for(n), kThreads, 0, st>>>(dface, n, dpanel, P);
    DCK(cudaGetLastError());

    // level by level: split flags, their scan, the children, the points
    std::vector<std::pair<int32_t, int32_t>> levels;
    int32_t lo = 0, hi = 6;
    int32_t *flag = nullptr, *rank = nullptr;
    int64_t flag_cap = 0, rank_cap = 0;
    char *tmp = nullptr;
    int64_t tmp_bytes = 0;
    int32_t total_h[2] = {0, 0};
    while (hi > lo) {
        const int32_t m = hi - lo;
        if (int rc = ensure(S, &flag, &flag_cap, m, st)) return rc;
        if (int rc = ensure(S, &rank, &rank_cap, m, st)) return rc;
        split_flags_kernel<<<blocks_for(m), kThreads, 0, st>>>(P, lo, hi, thresh, flag);
        DCK(cudaGetLastError());
        size_t need = 0;
        DCK(cub::DeviceScan::ExclusiveSum(nullptr, need, flag, rank, m, st));
        if (int rc = ensure(S, &tmp, &tmp_bytes, (int64_t)need, st)) return rc;
        DCK(cub::DeviceScan::ExclusiveSum(tmp, need, flag, rank, m, st));
        DCK(cudaMemcpyAsync(total_h, rank + (m - 1), sizeof(int32_t), cudaMemcpyDeviceToHost, st));
        DCK(cudaMemcpyAsync(total_h + 1, flag + (m - 1), sizeof(int32_t), cudaMemcpyDeviceToHost, st));
        DCK(cudaStreamSynchronize(st));
        levels.push_back({lo, hi});
        const int64_t splits = (int64_t)total_h[0] + total_h[1];
        if (splits == 0) break;
        if ((int64_t)hi + 4 * splits > INT32_MAX) return set_error(SAL_ENOMEM, "tree_traverse: too many panels");
        if (int rc = grow_keep(S, &P, &cap, hi, hi + 4 * splits, st)) return rc;
        children_kernel<<<blocks_for(m), kThreads, 0, st>>>(P, lo, hi, rank);
        DCK(cudaGetLastError());
        if (n > 0) move_points_kernel<<<blocks_for(n), kThreads, 0, st>>>(dxi, deta, dpanel, n, P, lo, hi);
        DCK(cudaGetLastError());
        lo = hi;
        hi = hi + (int32_t)(4 * splits);
    }
    const int32_t np = hi;

    // first positions, top-down, then the points stably sorted by their leaf's
    root_begin_kernel<<<1, 1, 0, st>>>(P);
    for (auto [a, b] : levels) child_begin_kernel<<<blocks_for(b - a), kThreads, 0, st>>>(P, a, b);
    DCK(cudaGetLastError());
    t->order.resize(n);
    if (n > 0) {
        DCK(S.get(&dkey, n)); DCK(S.get(&dkey2, n)); DCK(S.get(&didx, n)); DCK(S.get(&didx2, n));
        sort_keys_kernel<<<blocks_for(n), kThreads, 0, st>>>(dpanel, P, n, dkey, didx);
        DCK(cudaGetLastError());
        int bits = 1;
        while (bits < 32 && ((int64_t)1 << bits) <= (int64_t)n) ++bits;
        size_t need = 0;
        DCK(cub::DeviceRadixSort::SortPairs(nullptr, need, dkey, dkey2, didx, didx2, n, 0, bits, st));
        if (int rc = ensure(S, &tmp, &tmp_bytes, (int64_t)need, st)) return rc;
        DCK(cub::DeviceRadixSort::SortPairs(tmp, need, dkey, dkey2, didx, didx2, n, 0, bits, st));
        DCK(cudaMemcpyAsync(t->order.data(), didx2, (size_t)n * 4, cudaMemcpyDeviceToHost, st));
    }
    std::vector<DPanel> hp(np);
    DCK(cudaMemcpyAsync(hp.data(), P, (size_t)np * sizeof(DPanel), cudaMemcpyDeviceToHost, st));
    DCK(cudaStreamSynchronize(st));
    t->p.resize(np);
    for (int32_t k = 0; k < np; ++k) {
        const DPanel &d = hp[k];
        Panel &q = t->p[k];
        q.level = d.level; q.is_leaf = d.split ? 0 : 1; q.id = k + 1;
        q.parent = d.parent < 0 ? -1 : d.parent + 1;
        for (int j = 0; j < 4; ++j) q.child[j] = d.split ? d.child0 + j + 1 : -1;
        q.face = d.face;
        q.min_xi = d.mn_xi; q.mid_xi = d.md_xi; q.max_xi = d.mx_xi;
        q.min_eta = d.mn_eta; q.mid_eta = d.md_eta; q.max_eta = d.mx_eta;
        q.begin = d.begin; q.end = d.begin + d.count;
    }
    // radii and MAC centres with the host's libm
    tree_finish_panels(t);
    *out = own.release();
    return SAL_OK;
}

// dual_tree_traversal (tree_module.f90:277-398) on the device, over a host
// tree (its radii and MAC centres as they are).
int dual_tree_traversal_device(const Tree &t, double theta, int32_t thresh, int device, std::vector<int32_t> *L) {
    L->clear();
    DeviceGuard dg;
    Scratch S;
    if (int rc = enter_device(device, &dg, &S)) return rc;
    cudaStream_t st = dg.st;
    const int32_t np = (int32_t)t.p.size();
    std::vector<DttPanel> hp(np);
    for (int32_t k = 0; k < np; ++k) {
        const Panel &q = t.p[k];
        DttPanel &d = hp[k];
        d.radius = q.radius; d.cx = t.cx[k]; d.cy = t.cy[k]; d.cz = t.cz[k];
        d.count = (int32_t)q.count(); d.leaf = q.is_leaf;
        for (int j = 0; j < 4; ++j) d.child[j] = q.child[j];
    }
    DttPanel *P = nullptr;
    DCK(S.get(&P, np));
    DCK(cudaMemcpyAsync(P, hp.data(), (size_t)np * sizeof(DttPanel), cudaMemcpyHostToDevice, st));

    std::vector<int2> seed;
    for (int i = 1; i <= 6; ++i)
        for (int j = 1; j <= 6; ++j) seed.push_back(make_int2(i, j));
    // q: this generation's pairs; next: the next generation's; code, packed,
    // excl: per pair of this generation; list: the entries so far; amb: the
    // pairs left to the host
    int64_t cap_q = 0, cap_next = 0, cap_code = 0, cap_packed = 0, cap_excl = 0, cap_l = 0, cap_amb = 0;
    int64_t cap_dec = 0, m = 36, listed = 0;
    int2 *q = nullptr, *next = nullptr;
    int32_t *list = nullptr;
    uint8_t *code = nullptr, *dec = nullptr;
    unsigned long long *packed = nullptr, *excl = nullptr, *namb = nullptr;
    int64_t *amb = nullptr;
    char *tmp = nullptr;
    int64_t tmp_bytes = 0;
    if (int rc = ensure(S, &q, &cap_q, 1 << 14, st)) return rc;
    if (int rc = ensure(S, &list, &cap_l, 3 << 16, st)) return rc;
    if (int rc = ensure(S, &amb, &cap_amb, 1 << 12, st)) return rc;
    DCK(S.get(&namb, 1));
    DCK(cudaMemcpyAsync(q, seed.data(), 36 * sizeof(int2), cudaMemcpyHostToDevice, st));
    unsigned long long tot_h[3] = {0, 0, 0};
    std::vector<int2> pairs_h;
    std::vector<uint8_t> dec_h;
    int2 *amb_pairs = nullptr;
    int64_t cap_amb_pairs = 0;
    while (m > 0) {
        if (int rc = ensure(S, &code, &cap_code, m, st)) return rc;
        if (int rc = ensure(S, &packed, &cap_packed, m, st)) return rc;
        if (int rc = ensure(S, &excl, &cap_excl, m, st)) return rc;
        int64_t na = 0;
        for (;;) {
            DCK(cudaMemsetAsync(namb, 0, sizeof(unsigned long long), st));
            dtt_classify_kernel<<<blocks_for(m), kThreads, 0, st>>>(q, m, P, theta, thresh, code, packed, amb, cap_amb,
                                                                    namb);
            DCK(cudaGetLastError());
            DCK(cudaMemcpyAsync(tot_h + 2, namb, 8, cudaMemcpyDeviceToHost, st));
            DCK(cudaStreamSynchronize(st));
            na = (int64_t)tot_h[2];
            if (na <= cap_amb) break;
            if (int rc = ensure(S, &amb, &cap_amb, na, st)) return rc;   // too many to record: again, with room
        }
        if (na > 0) {
            // the host decides the pairs whose MAC ratio is within kMacTie of theta
            pairs_h.resize(na);
            dec_h.resize(na);
            if (int rc = ensure(S, &amb_pairs, &cap_amb_pairs, na, st)) return rc;
            dtt_gather_kernel<<<blocks_for(na), kThreads, 0, st>>>(q, amb, na, amb_pairs);
            DCK(cudaGetLastError());
            DCK(cudaMemcpyAsync(pairs_h.data(), amb_pairs, (size_t)na * sizeof(int2), cudaMemcpyDeviceToHost, st));
            DCK(cudaStreamSynchronize(st));
            for (int64_t k = 0; k < na; ++k)
                dec_h[k] = (uint8_t)dtt_decide(t, pairs_h[k].x, pairs_h[k].y, theta, thresh);
            if (int rc = ensure(S, &dec, &cap_dec, na, st)) return rc;
            DCK(cudaMemcpyAsync(dec, dec_h.data(), (size_t)na, cudaMemcpyHostToDevice, st));
            dtt_patch_kernel<<<blocks_for(na), kThreads, 0, st>>>(amb, dec, na, code, packed);
            DCK(cudaGetLastError());
        }
        size_t need = 0;
        DCK(cub::DeviceScan::ExclusiveSum(nullptr, need, packed, excl, m, st));
        if (int rc = ensure(S, &tmp, &tmp_bytes, (int64_t)need, st)) return rc;
        DCK(cub::DeviceScan::ExclusiveSum(tmp, need, packed, excl, m, st));
        DCK(cudaMemcpyAsync(tot_h, excl + (m - 1), 8, cudaMemcpyDeviceToHost, st));
        DCK(cudaMemcpyAsync(tot_h + 1, packed + (m - 1), 8, cudaMemcpyDeviceToHost, st));
        DCK(cudaStreamSynchronize(st));
        const unsigned long long tot = tot_h[0] + tot_h[1];
        const int64_t emits = (int64_t)(tot & 0xffffffffull), refined = (int64_t)(tot >> 32);
        if (int rc = grow_keep(S, &list, &cap_l, 3 * listed, 3 * (listed + emits), st)) return rc;
        if (int rc = ensure(S, &next, &cap_next, refined, st)) return rc;
        dtt_scatter_kernel<<<blocks_for(m), kThreads, 0, st>>>(q, m, P, code, excl, list, listed, next);
        DCK(cudaGetLastError());
        listed += emits;
        std::swap(q, next);
        std::swap(cap_q, cap_next);
        m = refined;
    }
    L->resize((size_t)(3 * listed));
    if (listed > 0)
        DCK(cudaMemcpyAsync(L->data(), list, (size_t)(3 * listed) * 4, cudaMemcpyDeviceToHost, st));
    DCK(cudaStreamSynchronize(st));
    return SAL_OK;
}

}  // namespace sal
