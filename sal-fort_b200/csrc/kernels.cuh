// Device kernels of the FP64 SAL-gradient treecode (sm_100a).
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#include "sal_internal.hpp"

namespace sal {
namespace dev {

// fast_sum_module.f90:14,23-25: literal constants folded in double precision,
// exactly as gfortran folds (1.0_8-6.21196_8) and (2.7_8+6.0_8).
constexpr double kCons = -2.343256857908601e-9;
constexpr double kC1 = 1.0 - 6.21196;
constexpr double kC2 = 2.7 + 6.0;
constexpr int kThreads = 256;
constexpr int kErrTimeout = 1;

// ----------------------------------------------------------------- PTX helpers
__device__ __forceinline__ uint32_t smem_u32(const void *p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void fence_mbar_init() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void fence_proxy_async() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}
// Bulk (non-tensor) TMA copy global -> this CTA's shared memory, completing
// on an mbarrier.  No multicast.  Both addresses 16-byte aligned, bytes a
// multiple of 16.
__device__ __forceinline__ void bulk_g2s(void *dst, const void *src, uint32_t bytes, uint64_t *bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
            smem_u32(dst)),
        "l"(src), "r"(bytes), "r"(smem_u32(bar))
        : "memory");
}
// The same with an L2 cache policy (createpolicy): a stream read once can
// leave L2 to data that is read again.
__device__ __forceinline__ void bulk_g2s_hint(void *dst, const void *src, uint32_t bytes, uint64_t *bar,
                                              uint64_t policy) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes.L2::cache_hint [%0], [%1], %2, [%3], %4;" ::"r"(
            smem_u32(dst)),
        "l"(src), "r"(bytes), "r"(smem_u32(bar)), "l"(policy)
        : "memory");
}
__device__ __forceinline__ uint64_t l2_evict_first() {
    uint64_t p;
    asm volatile("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(p));
    return p;
}
__device__ __forceinline__ uint64_t l2_evict_last() {
    uint64_t p;
    asm volatile("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(p));
    return p;
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}
// Bounded wait: gives up after `polls` polls and raises the grid's error
// flag, so a copy that never lands cannot hang the GPU.
constexpr uint32_t kDefaultPolls = 1u << 24;
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t *bar, uint32_t parity, int *err,
                                                  uint32_t polls = kDefaultPolls) {
    for (uint32_t it = 0; it < polls; ++it)
        if (mbar_try_wait(bar, parity)) return true;
    atomicExch(err, kErrTimeout);
    return false;
}

// ----------------------------------------------------------------- kernels of the SAL gradient
// Target-only terms of sal_grad_gfunc (fast_sum_module.f90:19,26-27), hoisted.
struct Tgt {
    double x, y, z, omx32, inv_mp2;
    bool live;  // outside the pole guard
};

__device__ __forceinline__ void tgt_init(Tgt &t, double x, double y, double z) {
    t.x = x; t.y = y; t.z = z;
    double x32 = __dmul_rn(z, z);
    t.omx32 = __dsub_rn(1.0, x32);
    t.inv_mp2 = __ddiv_rn(1.0, __dsqrt_rn(t.omx32));
    t.live = (fabs(__dsub_rn(z, 1.0)) > 1e-15) && (fabs(__dadd_rn(z, 1.0)) > 1e-15);
}

// sal_grad_gfunc (fast_sum_module.f90:9-31) for a live target, operation for
// operation with IEEE division and square root and without contraction, so the
// singular self pair s == t rounds exactly as the reference's does.  The
// division by sqrt(1-tz^2) is a multiply by its hoisted reciprocal.  Used by
// the direct sum, the accuracy judge.
__device__ __forceinline__ void gref_exact(const Tgt &t, double sx, double sy, double sz, double &gx, double &gy) {
    double gxy = __dadd_rn(__dmul_rn(t.x, sx), __dmul_rn(t.y, sy));
    double g = __dadd_rn(gxy, __dmul_rn(t.z, sz));
    g = fmax(fmin(g, 1.0), -1.0);
    double mp = __dsub_rn(2.0, __dmul_rn(2.0, g));
    double sqp = __dsqrt_rn(mp);
    double p1 = __ddiv_rn(kC1, __dadd_rn(__dmul_rn(sqp, mp), 1e-16));
    double p2 = __ddiv_rn(__dmul_rn(kC2, __dadd_rn(__dmul_rn(2.0, g), sqp)),
                          __dadd_rn(__dmul_rn(2.0, __dsub_rn(__dmul_rn(g, g), 1.0)), 1e-16));
    double val = __dmul_rn(__dadd_rn(p1, p2), kCons);
    double ny = __dsub_rn(__dmul_rn(sz, t.omx32), __dmul_rn(t.z, gxy));
    double nx = __dsub_rn(__dmul_rn(t.x, sy), __dmul_rn(t.y, sx));
    gy = __dmul_rn(__dmul_rn(ny, t.inv_mp2), val);
    gx = __dmul_rn(__dmul_rn(nx, t.inv_mp2), val);
}

// Reciprocal and square root for the treecode's inner loops: an FP32
// hardware approximation refined by Newton-Raphson iterations in FP64
// (reciprocal: r <- r + r(1 - x r), twice; square root: one step of the
// inverse-square-root iteration y <- y(3 - x y^2)/2, then one Heron step
// s <- s + y(x - s^2)/2), accurate to about one ulp.  Valid for
// 1e-37 < |x| < 1e37 (fast_rcp) and x == 0 or 1e-37 < x < 1e37 (fast_sqrt),
// the ranges their callers produce.
__device__ __forceinline__ double fast_rcp(double x) {
    float xf = __double2float_rn(x), rf;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(rf) : "f"(xf));
    double r = (double)rf;
    double e = fma(-x, r, 1.0);
    r = fma(r, e, r);
    e = fma(-x, r, 1.0);
    return fma(r, e, r);
}
__device__ __forceinline__ double fast_sqrt(double x) {
    float xf = __double2float_rn(x), yf;
    asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(yf) : "f"(xf));
    double y = (double)yf;
    double h = 0.5 * x;
    y = y * fma(-h * y, y, 1.5);
    double s = x * y;
    s = fma(fma(-s, s, x), 0.5 * y, s);
    return x > 0.0 ? s : 0.0;
}

// The reference kernel as the treecode evaluates it: g, mp = 2 - 2g, the two
// denominators and the two numerators in the reference's exact operation
// order (these carry the cancellations that make the self pair pure rounding
// noise), p1 + p2 over one common denominator, and the target factor
// 1/sqrt(1 - tz^2) left to the caller (applied once per target).  Adds the
// un-normalised (nx, ny) * val * w into (ax, ay).
__device__ __forceinline__ void gref_fast(const Tgt &t, double sx, double sy, double sz, double w, double &ax,
                                          double &ay) {
    double gxy = __dadd_rn(__dmul_rn(t.x, sx), __dmul_rn(t.y, sy));
    double g = __dadd_rn(gxy, __dmul_rn(t.z, sz));
    g = fmax(fmin(g, 1.0), -1.0);
    double g2 = __dmul_rn(2.0, g);
    double mp = __dsub_rn(2.0, g2);
    double sqp = fast_sqrt(mp);
    double d1 = __dadd_rn(__dmul_rn(sqp, mp), 1e-16);
    double n2 = __dmul_rn(kC2, __dadd_rn(g2, sqp));
    double d2 = __dadd_rn(__dmul_rn(2.0, __dsub_rn(__dmul_rn(g, g), 1.0)), 1e-16);
    double val = fma(kC1, d2, n2 * d1) * fast_rcp(d1 * d2) * (kCons * w);
    double ny = __dsub_rn(__dmul_rn(sz, t.omx32), __dmul_rn(t.z, gxy));
    double nx = __dsub_rn(__dmul_rn(t.x, sy), __dmul_rn(t.y, sx));
    ax = fma(nx, val, ax);
    ay = fma(ny, val, ay);
}

// The scalar val of the kernel with its removable antipodal singularity
// cancelled analytically (q = |t - s|):  2g + q = (2 - q)(1 + q) and
// 2(g^2 - 1) = -q^2 (2 - q)(2 + q)/2, so p2 = -2 * 8.7 * (1 + q) / (q^2 (2 + q)).
// mp = q^2 comes from coordinate differences, not from 2 - 2 t.s.
__device__ __forceinline__ double vstable(double mp) {
    double q = fast_sqrt(mp);
    double d1 = q * mp + 1e-16;
    double d2 = mp * (2.0 + q) + 1e-16;
    double num = kC1 * d2 - 2.0 * kC2 * (1.0 + q) * d1;
    return kCons * num * fast_rcp(d1 * d2);
}

// bli_coeffs, bli_module.f90:6-26 (0-based index i0 of degree d).
__device__ __forceinline__ double bli_coeff(int i0, int d) {
    if (d == 0) return 1.0;
    double s = (i0 & 1) ? -1.0 : 1.0;
    if (i0 == 0) return 0.5;
    if (i0 == d) return 0.5 * s;
    return s;
}

// One dimension of interp_vals_bli, bli_module.f90:67-105: the exact-node
// test, then the second barycentric form normalised by its denominator.
__device__ __forceinline__ void bli_basis(double x, const double *nodes, int n, double *f) {
    bool found = false;
    for (int i = 0; i < n; ++i) {
        f[i] = 0.0;
        if (fabs(__dsub_rn(x, nodes[i])) < 1e-16) { found = true; f[i] = 1.0; }
    }
    if (!found) {
        double denom = 0.0;
        for (int i = 0; i < n; ++i) {
            double v = __ddiv_rn(bli_coeff(i, n - 1), __dsub_rn(x, nodes[i]));
            f[i] = v;
            denom = __dadd_rn(denom, v);
        }
        for (int i = 0; i < n; ++i) f[i] = __ddiv_rn(f[i], denom);
    }
}

// ----------------------------------------------------------------- argument blocks
struct EvalArgs {
    const double4 *pool;     // sources: points then source proxies, (x, y, z, w)
    const Group *groups;
    const Item *items;
    const uint32_t *masks;
    const double4 *tgt;      // targets: the pool (leaf groups) or target proxies (proxy groups)
    const double2 *xieta;    // per pool position (leaf groups)
    const double *records;   // DOWN records, rec_stride doubles each
    int rec_stride, d, P;
    int kinds;               // bit k set: evaluate items of kind k (0 PP, 1 PC, 2 DOWN)
    const int32_t *perm;     // pool position -> caller index
    double *out_x, *out_y;   // leaf groups: caller order, overwritten
    double4 *partial;        // proxy groups: P outputs per unit
    int *err;
    uint32_t polls;          // poll limit of every staging wait (0: kDefaultPolls)
    int skip_last;           // fault injection: the last item's copy of every group is not issued
};

struct UpArgs {
    const double4 *pool;
    const double2 *xieta;
    const UpUnit *units;
    const double *nodes;     // per source slot 2(d+1) nodes
    int d, P;
    double *partial;         // P per unit
};

// launches (implemented in kernels.cu)
void launch_prep(const double4 *xyz, const double *area, const double *ssh, const int32_t *perm, int n, double4 *pool,
                 cudaStream_t st);
void launch_upward(const UpArgs &a, int nunits, cudaStream_t st);
void launch_upward_finalize(const int32_t *unit_beg, const double *partial, int nslots, int d, int transposed,
                            double4 *pool_proxy, cudaStream_t st);
void launch_eval(int tgt_kind, int form, const EvalArgs &a, int ngroups, cudaStream_t st);
void launch_proxy_finalize(const int32_t *unit_beg, const double4 *partial, int nslots, int P, int rec_stride,
                           double *records, cudaStream_t st);
void launch_direct(const double *xs, const double *ys, const double *zs, const double *w, int n,
                   const int32_t *targets, int nt, double *out_x, double *out_y, double *scratch, int nchunks,
                   cudaStream_t st);
int direct_chunks(int n);
void launch_extract_w(const double4 *pool_proxy, int count, double *out, cudaStream_t st);
void launch_insert_w(const double *w, int count, double4 *pool_proxy, cudaStream_t st);

}  // namespace dev
}  // namespace sal
