// Leaf pass of the batched form on the 5th-generation tensor cores (tcgen05).
//
// One CTA = one leaf group of up to 128 targets (the MMA's M) x 64 fields.
// Warps 0-7 produce: thread t < 256 owns target row r = t % 128 and half
// h = t / 128 of every 8-column k-step.  Warp 8 only issues the MMAs, so no
// producer warp diverges around the issue (a lane blocked in an mbarrier wait
// would otherwise hold up the lane that must issue).  Per item (<= 64
// sources, or <= 64 Cartesian rows of a DOWN interpolation) the CTA
//   1. waits for the item's per-field rows (cp.async), folds the previous
//      item's accumulator into the running sum (both in tensor memory), and
//      rewrites the rows as TF32 hi / lo B tiles in the canonical no-swizzle
//      K-major layout;
//   2. for each k-step, every producer thread forms its 4 kernel-tile entries
//      in FP32 (east and north components, hi and lo parts) into one of two
//      shared A slots; the MMA warp issues the six tcgen05.mma of the k-step
//      (hi*hi + hi*lo + lo*hi for each component) into the item accumulator
//      and commits them to the slot's "empty" barrier.
// The item accumulator starts from zero at every item and is added to the
// running sum with round-to-nearest FP32 adds: the tensor cores accumulate
// with truncation, so chaining all k-steps of a target in one accumulator
// biases the result toward zero.
// Tensor memory (256 columns): item accumulator [east 64 | north 64] at
// columns 0..127, running sum at 128..255.  Shared memory ~102 KB, so at most
// two CTAs share an SM and their 2 x 256 columns fit the 512 the SM has.
#include <cuda_runtime.h>

#include "kernels.cuh"
#include "mixed.cuh"

namespace sal {
namespace mix {

using dev::smem_u32;

namespace {

constexpr int kThreads = 288;    // 8 producer warps + 1 MMA warp
constexpr int kProducers = 256;
constexpr int kRows = kTcRows;   // 128
constexpr int kF = 64;           // fields per CTA (the MMA's N per component)
constexpr int kK = kMixStage;    // 64 K rows per item
constexpr int kTmemCols = 256;
constexpr float kC1F = (float)dev::kC1;
constexpr float kTwoC2F = (float)(2.0 * dev::kC2);

// instruction descriptor: D F32, A/B TF32, both K-major, N = 64, M = 128
constexpr uint32_t kIdesc = (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(kF >> 3) << 17) |
                            ((uint32_t)(kRows >> 4) << 24);

struct TcSmem {
    float4 A[2][4][kRows * 2];          // 2 slots x {east hi, east lo, north hi, north lo} x 128 rows x 8 tf32
    float4 B[kK / 8][2][kF * 2];        // per k-step: {hi, lo} x 64 fields x 8 tf32 (canonical K-major)
    float Bp[kK * kF];                  // rows as copied (cp.async), XOR-swizzled 16-byte chunks
    double4 raw[kK];
    float4 loc[kK];
    float fx[kRows][kMaxDegree + 1];    // BLI bases of the row targets in the current DOWN panel
    float fe[kRows][kMaxDegree + 1];
    int kmap[3 * (kMaxDegree + 1) * (kMaxDegree + 1) + 8];
    uint64_t full[2], empty[2], item_done;
    uint32_t tmem_base;
    int down_slot;
    int abort;
};

__device__ __forceinline__ float val32(float mp) {
    float r, u;
    asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(mp));
    const float q = mp * r;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(u) : "f"(2.f + q));
    const float inner = fmaf(kC1F, r, fmaf(kTwoC2F, u, -kTwoC2F));
    const float v = inner * r * r;
    return mp > 0.f ? v : 0.f;
}

__device__ __forceinline__ uint32_t to_tf32(float x) {
    uint32_t r;
    asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
    return r;
}
__device__ __forceinline__ void split(float x, float &hi, float &lo) {
    const uint32_t h = to_tf32(x);
    hi = __uint_as_float(h);
    lo = __uint_as_float(to_tf32(x - hi));
}

__device__ __forceinline__ void cp16(void *dst, const void *src) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(smem_u32(dst)), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_wait0() { asm volatile("cp.async.wait_group 0;" ::: "memory"); }

__device__ __forceinline__ void mbar_arrive(uint64_t *bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}
// Bounded wait on an mbarrier phase; on time-out raises the error flag and
// the CTA-wide abort flag (later waits then return at once).
__device__ __forceinline__ void wait_bounded(uint64_t *bar, uint32_t parity, volatile int *abort, int *err) {
    if (*abort) return;
    for (uint32_t it = 0; it < (1u << 24); ++it)
        if (dev::mbar_try_wait(bar, parity)) return;
    *abort = 1;
    atomicExch(err, dev::kErrTimeout);
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// Shared-memory matrix descriptor, canonical K-major layout without swizzle:
// 8-row x 16-byte core matrices, LBO = 128 B between the two K halves of an
// 8-row group, SBO = 256 B between 8-row groups; version 1 (bits 46-47).
__device__ __forceinline__ uint64_t smem_desc(const void *p) {
    const uint64_t addr = smem_u32(p);
    return ((addr >> 4) & 0x3FFFull) | ((uint64_t)(128 >> 4) << 16) | ((uint64_t)(256 >> 4) << 32) |
           (1ull << 46);
}

__device__ __forceinline__ void mma_tf32(uint32_t d_tmem, uint64_t a, uint64_t b, uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(d_tmem),
        "l"(a), "l"(b), "r"(kIdesc), "r"(accumulate)
        : "memory");
}
__device__ __forceinline__ void mma_commit(uint64_t *bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
                 : "memory");
}

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float (&v)[16]) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
        "%15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
#pragma unroll
    for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}
__device__ __forceinline__ void tmem_st16(uint32_t taddr, const float (&v)[16]) {
    asm volatile(
        "tcgen05.st.sync.aligned.32x32b.x16.b32 [%0], {%1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, "
        "%14, %15, %16};" ::"r"(taddr),
        "r"(__float_as_uint(v[0])), "r"(__float_as_uint(v[1])), "r"(__float_as_uint(v[2])),
        "r"(__float_as_uint(v[3])), "r"(__float_as_uint(v[4])), "r"(__float_as_uint(v[5])),
        "r"(__float_as_uint(v[6])), "r"(__float_as_uint(v[7])), "r"(__float_as_uint(v[8])),
        "r"(__float_as_uint(v[9])), "r"(__float_as_uint(v[10])), "r"(__float_as_uint(v[11])),
        "r"(__float_as_uint(v[12])), "r"(__float_as_uint(v[13])), "r"(__float_as_uint(v[14])),
        "r"(__float_as_uint(v[15]))
        : "memory");
}
__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }
__device__ __forceinline__ void tmem_wait_st() { asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory"); }

// Byte offset of element (row, k) of a canonical K-major tile (k < 8).
__device__ __forceinline__ int canon(int row, int k) {
    return (row >> 3) * 256 + (k >> 2) * 128 + (row & 7) * 16 + (k & 3) * 4;
}

}  // namespace

__global__ void __launch_bounds__(kThreads, 2) tc_leaf_kernel(MixArgs a, int *err) {
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    TcSmem &sm = *reinterpret_cast<TcSmem *>(smem_raw);
    const MixGroup G = a.groups[blockIdx.x];
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const bool producer = tid < kProducers;
    const int row = tid & (kRows - 1), half = (tid >> 7) & 1;
    const int n = a.d + 1, P = a.P;
    volatile int *abort = &sm.abort;

    // ------------------------------------------------------------ set-up
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                         smem_u32(&sm.tmem_base)),
                     "r"(kTmemCols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    if (tid == 0) {
        dev::mbar_init(&sm.full[0], kProducers);
        dev::mbar_init(&sm.full[1], kProducers);
        dev::mbar_init(&sm.empty[0], 1);
        dev::mbar_init(&sm.empty[1], 1);
        dev::mbar_init(&sm.item_done, 1);
        dev::fence_mbar_init();
        sm.down_slot = -1;
        sm.abort = 0;
    }
    for (int k = tid; k < 3 * P + 8; k += kThreads) {
        const int kk = k < 3 * P ? k : 0;
        const int p = kk / 3;
        sm.kmap[k] = (p % n) | ((p / n) << 8) | ((kk % 3) << 16);
    }
    // the row's target: coordinates relative to the leaf centre and its
    // east / north unit vectors scaled by nothing (the reference's 1/sqrt(1-z^2)
    // is part of the unit vectors' normalisation)
    const bool rvalid = producer && row < G.nt;
    float tl0 = 0.f, tl1 = 0.f, tl2 = 0.f, el0 = 0.f, el1 = 0.f, ep0 = 0.f, ep1 = 0.f, ep2 = 0.f;
    if (rvalid) {
        const double4 c = a.tgt[G.tgt + row];
        tl0 = (float)(c.x - G.cx);
        tl1 = (float)(c.y - G.cy);
        tl2 = (float)(c.z - G.cz);
        if ((fabs(c.z - 1.0) > 1e-15) && (fabs(c.z + 1.0) > 1e-15)) {
            const double omz = 1.0 - c.z * c.z, inv = 1.0 / sqrt(omz);
            el0 = (float)(-c.y * inv);
            el1 = (float)(c.x * inv);
            ep0 = (float)(-c.z * c.x * inv);
            ep1 = (float)(-c.z * c.y * inv);
            ep2 = (float)(omz * inv);
        }
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = sm.tmem_base;
    const uint32_t lane_base = (uint32_t)(32 * (warp & 3)) << 16;   // this warp's TMEM lane quarter
    const uint32_t run_col = 128 + 64 * half;                      // running sum: east (half 0) / north (half 1)
    const uint32_t item_col = 64 * half;
    if (producer) {
        float z[16];
#pragma unroll
        for (int i = 0; i < 16; ++i) z[i] = 0.f;
#pragma unroll
        for (int c = 0; c < 4; ++c) tmem_st16(tmem + lane_base + run_col + 16 * c, z);
        tmem_wait_st();
    }

    const int ni = G.ie - G.ib;
    auto prefetch = [&](int k) {
        const Item it = a.items[G.ib + k];
        const float *src = it.kind == 2 ? a.phiF + ((size_t)it.off * 3 * P + it.mask) * kF
                                        : a.wF + (size_t)it.off * kF;
        if (it.kind != 2)
            for (int i = tid; i < it.cnt * 2; i += kThreads)
                cp16(reinterpret_cast<char *>(&sm.raw[i >> 1]) + 16 * (i & 1),
                     reinterpret_cast<const char *>(a.pool + it.off + (i >> 1)) + 16 * (i & 1));
        constexpr int CH = kF / 4;
        for (int i = tid; i < it.cnt * CH; i += kThreads) {
            const int r = i / CH, c = i % CH;
            cp16(&sm.Bp[r * kF + ((c ^ ((r & 3) << 1)) << 2)], src + (size_t)r * kF + c * 4);
        }
    };
    auto flush = [&]() {
        // running sum += item accumulator (this warp's 32 lanes x 64 columns)
#pragma unroll
        for (int c = 0; c < 4; ++c) {
            float x[16], y[16];
            tmem_ld16(tmem + lane_base + item_col + 16 * c, x);
            tmem_ld16(tmem + lane_base + run_col + 16 * c, y);
            tmem_wait_ld();
#pragma unroll
            for (int i = 0; i < 16; ++i) y[i] += x[i];
            tmem_st16(tmem + lane_base + run_col + 16 * c, y);
        }
        tmem_wait_st();
    };

    if (ni > 0) prefetch(0);
    cp_commit();
    uint32_t gk = 0;   // k-steps issued so far by this CTA
    for (int k = 0; k < ni; ++k) {
        cp_wait0();
        __syncthreads();
        const Item it = a.items[G.ib + k];
        const int cnt = it.cnt, ks = (cnt + 7) >> 3, kend = ks * 8;
        if (k > 0 && producer) {
            wait_bounded(&sm.item_done, (uint32_t)((k - 1) & 1), abort, err);
            tc_fence_after();
            flush();
        }
        // ------------------------------------------------ item preparation
        if (it.kind != 2) {
            if (tid < cnt) {
                const double4 s = sm.raw[tid];
                sm.loc[tid] = make_float4((float)(s.x - G.cx), (float)(s.y - G.cy), (float)(s.z - G.cz), 0.f);
            } else if (tid < kend) {
                sm.loc[tid] = make_float4(4.f, 4.f, 4.f, 0.f);   // padding column: finite entries, zero weights
            }
        } else if (sm.down_slot != it.off && tid < kRows) {   // producers of half 0
            float *fxr = sm.fx[tid], *fer = sm.fe[tid];
            if (tid < G.nt) {
                const double2 e = a.xieta[G.tgt + tid];
                const double *nodes = a.tgt_nodes + (size_t)it.off * 2 * n;
                double f[kMaxDegree + 1];
                dev::bli_basis(e.x, nodes, n, f);
                for (int i = 0; i < n; ++i) fxr[i] = (float)f[i];
                dev::bli_basis(e.y, nodes + n, n, f);
                for (int i = 0; i < n; ++i) fer[i] = (float)f[i];
            } else {
                for (int i = 0; i < n; ++i) fxr[i] = fer[i] = 0.f;
            }
        }
        // B rows -> TF32 hi / lo tiles, canonical K-major (rows = fields, K = sources)
        for (int e = tid; e < kend * kF; e += kThreads) {
            const int f = e & (kF - 1), kr = e >> 6;
            const float v = kr < cnt ? sm.Bp[kr * kF + ((((f >> 2) ^ ((kr & 3) << 1))) << 2) + (f & 3)] : 0.f;
            float hi, lo;
            split(v, hi, lo);
            const int off = canon(f, kr & 7);
            reinterpret_cast<float *>(sm.B[kr >> 3][0])[off >> 2] = hi;
            reinterpret_cast<float *>(sm.B[kr >> 3][1])[off >> 2] = lo;
        }
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        tc_fence_before();
        __syncthreads();
        tc_fence_after();
        if (tid == 0 && it.kind == 2) sm.down_slot = it.off;
        if (k + 1 < ni) prefetch(k + 1);
        cp_commit();
        // ------------------------------------------------ k-steps
        for (int s = 0; s < ks; ++s, ++gk) {
            const uint32_t slot = gk & 1, use = gk >> 1;
            if (!producer) {
                // the MMA warp: wait for the slot, issue the k-step's six MMAs
                wait_bounded(&sm.full[slot], use & 1, abort, err);
                tc_fence_after();
                if (lane == 0) {
                    if (!*abort) {
                        const uint64_t bh = smem_desc(sm.B[s][0]), bl = smem_desc(sm.B[s][1]);
#pragma unroll
                        for (int comp = 0; comp < 2; ++comp) {
                            const uint32_t d = tmem + 64 * comp;
                            const uint64_t ah = smem_desc(sm.A[slot][2 * comp]);
                            const uint64_t al = smem_desc(sm.A[slot][2 * comp + 1]);
                            mma_tf32(d, ah, bh, s > 0 ? 1u : 0u);
                            mma_tf32(d, ah, bl, 1u);
                            mma_tf32(d, al, bh, 1u);
                        }
                    }
                    mma_commit(&sm.empty[slot]);
                    if (s == ks - 1) mma_commit(&sm.item_done);
                }
                __syncwarp();
                continue;
            }
            if (use > 0) wait_bounded(&sm.empty[slot], (use - 1) & 1, abort, err);
            float ve[4], vn[4];
#pragma unroll
            for (int c = 0; c < 4; ++c) {
                const int col = s * 8 + half * 4 + c;
                if (it.kind == 2) {
                    const int m = sm.kmap[it.mask + col];
                    const float b = (col < cnt) ? sm.fx[row][m & 255] * sm.fe[row][(m >> 8) & 255] : 0.f;
                    const int j = m >> 16;
                    const float e = j == 0 ? el0 : el1;           // east z-component is 0
                    const float np = j == 0 ? ep0 : (j == 1 ? ep1 : ep2);
                    ve[c] = j == 2 ? 0.f : b * e;
                    vn[c] = b * np;
                } else {
                    const float4 q = sm.loc[col];
                    const float dx = q.x - tl0, dy = q.y - tl1, dz = q.z - tl2;
                    const float v = val32(dx * dx + dy * dy + dz * dz);
                    ve[c] = v * (el0 * dx + el1 * dy);
                    vn[c] = v * (ep0 * dx + ep1 * dy + ep2 * dz);
                }
            }
            float4 eh, elo, nh, nlo;
            split(ve[0], eh.x, elo.x);
            split(ve[1], eh.y, elo.y);
            split(ve[2], eh.z, elo.z);
            split(ve[3], eh.w, elo.w);
            split(vn[0], nh.x, nlo.x);
            split(vn[1], nh.y, nlo.y);
            split(vn[2], nh.z, nlo.z);
            split(vn[3], nh.w, nlo.w);
            const int ofs = canon(row, half * 4) >> 4;   // float4 index
            sm.A[slot][0][ofs] = eh;
            sm.A[slot][1][ofs] = elo;
            sm.A[slot][2][ofs] = nh;
            sm.A[slot][3][ofs] = nlo;
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            mbar_arrive(&sm.full[slot]);
        }
    }
    cp_wait0();
    // ------------------------------------------------ epilogue
    if (ni > 0 && producer) {
        wait_bounded(&sm.item_done, (uint32_t)((ni - 1) & 1), abort, err);
        tc_fence_after();
        flush();
    }
    if (producer) {
        // every thread takes part in the warp-wide tensor-memory loads; rows
        // beyond the group's targets discard what they read
        const bool write = rvalid && !*abort;
        int idx = 0;
        double self = 0.0, ar = 0.0;
        double *out = half == 0 ? a.out_x : a.out_y;
        if (write) {
            const int pos = G.tgt + row;
            idx = a.perm[pos];
            const double4 c = a.tgt[pos];
            dev::Tgt T;
            dev::tgt_init(T, c.x, c.y, c.z);
            double sx = 0.0, sy = 0.0;
            if (T.live) dev::gref_exact(T, c.x, c.y, c.z, sx, sy);   // the self pair, in FP64
            self = half == 0 ? sx : sy;
            ar = a.area[pos];
        }
#pragma unroll
        for (int cc = 0; cc < 4; ++cc) {
            float y[16];
            tmem_ld16(tmem + lane_base + run_col + 16 * cc, y);
            tmem_wait_ld();
            if (write) {
#pragma unroll
                for (int i = 0; i < 16; ++i) {
                    const int f = a.f0 + 16 * cc + i;
                    if (f < a.nf) {
                        const double w = ar * a.ssh[(size_t)f * a.ld_ssh + idx];
                        out[(size_t)f * a.ld_out + idx] = (double)y[i] + self * w;
                    }
                }
            }
        }
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 0) {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTmemCols) : "memory");
    }
}

size_t tc_smem_bytes() { return sizeof(TcSmem) + 1024; }

void launch_tc_leaf(const MixArgs &a, int ngroups, int *err, cudaStream_t st) {
    if (ngroups <= 0) return;
    const size_t smem = tc_smem_bytes();
    cudaFuncSetAttribute(tc_leaf_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    tc_leaf_kernel<<<ngroups, kThreads, smem, st>>>(a, err);
}

}  // namespace mix
}  // namespace sal
