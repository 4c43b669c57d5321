// Launch interface of the batched mixed-precision kernels (mixed.cu).
#pragma once
#include <atomic>
#include <cstdint>
#include <cuda_runtime.h>

#include "sal_internal.hpp"

namespace sal {
namespace mix {

// Raises a kernel's dynamic shared memory limit once per device.  Setting a
// function attribute while that kernel runs on another stream can stall the
// host, so a launch path must not repeat it.
inline void smem_attr_once(const void *fn, int bytes, std::atomic<unsigned long long> &done) {
    int dev = 0;
    cudaGetDevice(&dev);
    const unsigned long long bit = 1ull << (dev & 63);
    if (done.load(std::memory_order_acquire) & bit) return;
    cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
    done.fetch_or(bit, std::memory_order_acq_rel);
}

struct MixArgs {
    const double4 *pool;      // FP64 source coordinates (points, then source proxies)
    const float *wF;          // per-field source rows: (n + nsrc*P) x FT
    const float *phiF;        // per-field Cartesian potentials: ntgt x 3P x FT
    const MixGroup *groups;
    const Item *items;
    const double4 *tgt;       // target coordinates: pool (leaf) or target proxies (proxy pass)
    const double2 *xieta;     // per pool position
    const double *tgt_nodes;  // 2(d+1) Chebyshev nodes per slot (target slots; source slots for the upward pass)
    int d, P;
    const int32_t *perm;      // leaf epilogue: pool position -> caller index
    const double *area;       // per pool position
    const double *ssh;        // caller's fields (column f at ssh + f*ld_ssh)
    int64_t ld_ssh;
    double *out_x, *out_y;    // caller's outputs (column f at + f*ld_out)
    int64_t ld_out;
    float *partial;           // proxy / upward: per-unit partial sums
    int f0, nf;               // first field of this block, total fields
};

void launch_mix(int kind, int FT, const MixArgs &a, int ngroups, cudaStream_t st);
void launch_prep_mix(const double *area, const double *ssh, int64_t ld, const int32_t *iperm, int n, int f0, int nf,
                     int FT, float *wF, cudaStream_t st);
void launch_finalize_mix(const int32_t *unit_beg, const float *partial, int nslots, int rows_per_slot, int FT,
                         float *dst, cudaStream_t st);
size_t mix_smem_bytes();
// tcgen05 leaf pass (64-field blocks), tc_leaf.cu
struct TcArgs {
    const MixGroup *groups;   // leaf groups of <= 128 targets, pool order
    int ngroups;
    const TcItem *items;
    const float *sxyz;        // per source k-step of the split store: x[8], y[8], z[8] relative to the panel centre
    const float *bstore;      // split weight store: 1024 floats per k-step of 8 rows
    const double4 *tgt;       // pool (targets are its first n rows)
    const double2 *xieta;     // per pool position
    const double *tgt_nodes;  // 2(d+1) Chebyshev nodes per target slot
    const double2 *selfk;     // per pool position: self pair / kernel constant
    const float *wF;          // per pool row: 64 field weights (carry the kernel constant)
    const int32_t *perm;      // pool position -> caller index
    int d, P;
    double *out_x, *out_y;    // caller's outputs (column f at + f*ld_out)
    int64_t ld_out;
    int f0, nf;
    float *partial;           // proxy / upward pass: per-unit rows (P x components x 64 fields)
    const float *basis;       // upward pass: BLI factors per basis k-step
    // FP16 leaf pass (bstore16 non-null): the FP16 hi/lo weight store (2 KB
    // per unit of 8 rows), per target its kernel-value scale and inverse, and
    // the block's field maxima (as float bits): 64 of source weights, then 64
    // of potentials
    const void *bstore16;
    const float *tscale, *tinv;
    const unsigned *fmax;
    // FP16 leaf pass with a kernel-tile store: the store, per group the byte
    // offset of its tiles (ngroups + 1 entries), and which items it holds:
    // items every-1, 2 every-1, ... of each group (all with every = 1)
    unsigned char *ktile;
    const int64_t *ktile_off;
    int tile_every;
};
// cta_groups: groups one CTA walks at most (the grid has every SM busy
// otherwise)
// Arguments of a leaf pass over several grids in one launch (same degree).
constexpr int kMaxJoint = 8;
struct TcJoint {
    TcArgs g[kMaxJoint];
    int32_t beg[kMaxJoint + 1];   // first joint group of each grid; beg[ngrids] = all groups
    int32_t ngrids;
};
// tiles (FP16 leaf pass with a.ktile set): 0 computes the kernel tiles,
// 1 computes them and records the stored items' in a.ktile, 2 replays them
// all from a.ktile, 3 replays the stored items' and computes the others
void launch_tc_leaf(const TcArgs &a, int nsm, int cta_groups, int *err, cudaStream_t st, int tiles = 0);
void launch_tc_leaf_joint(const TcArgs *grids, int ngrids, int nsm, int cta_groups, int *err, cudaStream_t st);
void launch_tc_proxy(const TcArgs &a, int nsm, int cta_groups, int *err, cudaStream_t st);
void launch_tc_upward(const TcArgs &a, int nsm, int cta_groups, int *err, cudaStream_t st);
void launch_basis_store(const int32_t *bas, int64_t nbk, const double2 *xieta, const double *src_nodes, int n,
                        float *basis, cudaStream_t st);
size_t tc_smem_bytes();
void launch_split_store(const int32_t *bsrc, int64_t k0, int64_t k1, const float *wF, const float *phiF,
                        float *bstore, cudaStream_t st);
// FP16 leaf pass: per field the largest |value| of the source weight rows
// (wF, nw rows) and of the potential rows (phiF, np rows) into fmax[f] and
// fmax[64 + f] (float bits; fmax zeroed first; rows no pass writes must hold
// zeros); the FP16 hi/lo store of units [0, nunits) with those scales; per
// target the scale of its kernel values (once per plan).
void launch_field_max(const float *wF, int64_t nw, const float *phiF, int64_t np, unsigned *fmax, cudaStream_t st);
void launch_split_store16(const int32_t *bsrc, int64_t nunits, const float *wF, const float *phiF,
                          const unsigned *fmax, void *bstore16, cudaStream_t st);
void launch_target_scales(const TcArgs &a, float *tscale, float *tinv, cudaStream_t st);
void launch_source_local(const double4 *pool, const int2 *ranges, const double4 *centres, int nranges, float4 *sloc,
                         cudaStream_t st);
void launch_self_pair(const double4 *pool, int n, double2 *selfk, cudaStream_t st);
void launch_source_ksteps(const int32_t *bsrc, int64_t nks, const float4 *sloc, float *sxyz, cudaStream_t st);
// tree transfers (transfer.cu): one launch per tree level; H holds the two
// n x n half-interval transfer matrices
void launch_m2m(const int32_t *tasks, int ntasks, const double *H, int n, float *w, cudaStream_t st);
void launch_l2l(const int32_t *tasks, int ntasks, const double *H, int n, float *phi, cudaStream_t st);

}  // namespace mix
}  // namespace sal
