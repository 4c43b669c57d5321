// Batched mixed-precision form of the DTT treecode: many SSH fields per solve.
//
// Each pass is a chain of small GEMMs C[rows x F] += A[rows x K] * B[K x F]
// whose A operand is generated on the fly and whose B operand is the per-field
// data of K sources:
//   leaf   : rows = targets of a leaf (<= 64 per CTA); A = the kernel tile
//            val(t,s) * (e(t) . (s - t)) on the target's east and north unit
//            vectors (2 components), or, for DOWN items, the BLI basis of the
//            target panel times those unit vectors (K = 3P Cartesian rows);
//            B = w = area * ssh of the sources (PP), proxy weights W (PC), or
//            Cartesian proxy potentials (DOWN).
//   proxy  : rows = Chebyshev proxies of a target panel; A = val(x,s) (s - x)
//            (3 Cartesian components); B as for the leaf pass.
//   upward : rows = proxies of a source panel; A = BLI basis at the panel's
//            points; B = w.
// The kernel tile is formed in FP32 from coordinates relative to the group's
// panel centre (small differences, no 1 - cos cancellation), with the
// antipode-stable val.  Products run on the tensor cores as TF32 with split
// hi + lo operands (hi*hi + hi*lo + lo*hi, about 21 significant bits) and FP32
// accumulation; the singular self pair is added in FP64 with the reference's
// exact operation order (fast_sum_module.f90:19-29), as the FP64 direct sum
// does.
#include <cuda_runtime.h>

#include "kernels.cuh"
#include "mixed.cuh"

namespace sal {
namespace mix {

using dev::smem_u32;

constexpr int kThr = 128;          // 4 warps, one 16-row tile each
constexpr int kS = kMixStage;      // K rows staged per item
constexpr float kC1F = (float)dev::kC1;
constexpr float kTwoC2F = (float)(2.0 * dev::kC2);

__device__ __forceinline__ uint32_t to_tf32(float x) {
    uint32_t r;
    asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
    return r;
}
__device__ __forceinline__ void split_tf32(float x, uint32_t &hi, uint32_t &lo) {
    hi = to_tf32(x);
    lo = to_tf32(x - __uint_as_float(hi));
}
// D = A * B + D, m16n8k8, TF32 inputs, FP32 accumulate (warp-wide).
__device__ __forceinline__ void mma8(float (&c)[4], const uint32_t (&a)[4], uint32_t b0, uint32_t b1) {
    asm volatile(
        "mma.sync.aligned.m16n8k8.row.col.f32.tf32.tf32.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
        "{%0,%1,%2,%3};\n"
        : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}
__device__ __forceinline__ void cp16(void *dst, const void *src) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(smem_u32(dst)), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_wait1() { asm volatile("cp.async.wait_group 1;" ::: "memory"); }
__device__ __forceinline__ void cp_wait0() { asm volatile("cp.async.wait_group 0;" ::: "memory"); }

// Word offset of B(k, f) in a staged tile: 16-byte chunks of row k are
// XOR-swizzled by (k & 3) << 1, so the fragment loads of one k-step (rows
// t4 and t4 + 4, columns n*8 + g) hit 32 distinct banks.  Needs FT >= 32.
template <int FT>
__device__ __forceinline__ int bofs(int k, int f) {
    return k * FT + ((((f >> 2) ^ ((k & 3) << 1))) << 2) + (f & 3);
}

// val / kCons of the kernel in FP32 from the chord length squared mp = |s - t|^2
// (the antipode-stable form of dev::vstable without its 1e-16 terms, which
// only matter at s == t):  with r = 1/q and u = 1/(2 + q),
//   kC1/q^3 - 2 kC2 (1 + q)/(q^2 (2 + q)) = r^2 (kC1 r - 2 kC2 (1 - u)).
// mp == 0 (the self pair, added separately in FP64) gives 0.  The constant
// kCons is folded into the per-field weights instead.
__device__ __forceinline__ float val32(float mp) {
    float r, u;
    asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(mp));
    const float q = mp * r;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(u) : "f"(2.f + q));
    const float inner = fmaf(kC1F, r, fmaf(kTwoC2F, u, -kTwoC2F));
    const float v = inner * r * r;
    return mp > 0.f ? v : 0.f;
}

struct Smem {
    // B tiles as copied, double-buffered: kS rows x FT floats each (sized for FT = 64)
    float B[2][kS * 64];
    // the current item's B tile split into TF32 hi/lo, in mma fragment order:
    // [k-step][n-tile][lane] = (b0 hi, b1 hi, b0 lo, b1 lo)
    float4 Bf[(kS / 8) * 8 * 32];
    double4 raw[2][kS];              // staged FP64 source coordinates
    float4 loc[kS];                  // sources relative to the group's centre (FP32)
    float fx[kMixRows][kMaxDegree + 1];  // BLI bases: of targets (leaf DOWN) or sources (upward)
    float fe[kMixRows][kMaxDegree + 1];
    int kmap[3 * (kMaxDegree + 1) * (kMaxDegree + 1)];
    int down_slot;
};

// KIND 0: leaf pass; 1: proxy pass; 2: upward pass.  NT: 8-column tiles of F.
template <int KIND, int NT>
__global__ void __launch_bounds__(kThr) mix_kernel(MixArgs a) {
    constexpr int NC = KIND == 0 ? 2 : (KIND == 1 ? 3 : 1);
    constexpr int FT = NT * 8;
    extern __shared__ __align__(128) unsigned char smem_raw[];
    Smem &sm = *reinterpret_cast<Smem *>(smem_raw);
    const MixGroup G = a.groups[blockIdx.x];
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31, g = lane >> 2, t4 = lane & 3;
    const int n = a.d + 1, P = a.P;
    const bool warp_live = warp * 16 < G.nt;

    // ---------------------------------------------------------- per-row target data
    float tl[2][3] = {{0, 0, 0}, {0, 0, 0}};          // target, local coordinates
    float el[2][3] = {{0, 0, 0}, {0, 0, 0}};          // east unit vector / sqrt(1-z^2) factor included
    float ep[2][3] = {{0, 0, 0}, {0, 0, 0}};          // north unit vector
    bool rv[2];
    int rk[2][2] = {{0, 0}, {0, 0}};                  // upward: (xi index, eta index) of the row's proxy
#pragma unroll
    for (int rr = 0; rr < 2; ++rr) {
        const int row = warp * 16 + g + 8 * rr;
        rv[rr] = row < G.nt;
        if (!rv[rr]) continue;
        if (KIND == 2) {
            const int p = G.row0 + row;
            rk[rr][0] = p % n;
            rk[rr][1] = p / n;
            continue;
        }
        const double4 c = KIND == 0 ? a.tgt[G.tgt + row] : a.tgt[(size_t)G.tgt * P + G.row0 + row];
        tl[rr][0] = (float)(c.x - G.cx);
        tl[rr][1] = (float)(c.y - G.cy);
        tl[rr][2] = (float)(c.z - G.cz);
        if (KIND == 0) {
            const bool live = (fabs(c.z - 1.0) > 1e-15) && (fabs(c.z + 1.0) > 1e-15);
            if (live) {
                const double omz = 1.0 - c.z * c.z, inv = 1.0 / sqrt(omz);
                el[rr][0] = (float)(-c.y * inv);
                el[rr][1] = (float)(c.x * inv);
                ep[rr][0] = (float)(-c.z * c.x * inv);
                ep[rr][1] = (float)(-c.z * c.y * inv);
                ep[rr][2] = (float)(omz * inv);
            }
        }
    }
    if (KIND == 0) {
        for (int k = tid; k < 3 * P; k += kThr) {
            const int p = k / 3;
            sm.kmap[k] = (p % n) | ((p / n) << 8) | ((k % 3) << 16);
        }
        if (tid == 0) sm.down_slot = -1;
    }

    float acc[NC][NT][4];
#pragma unroll
    for (int c = 0; c < NC; ++c)
#pragma unroll
        for (int j = 0; j < NT; ++j)
#pragma unroll
            for (int e = 0; e < 4; ++e) acc[c][j][e] = 0.f;

    // ---------------------------------------------------------- staging
    const int nitems = KIND == 2 ? (G.ie - G.ib + kS - 1) / kS : G.ie - G.ib;
    auto item_of = [&](int k, int &off, int &cnt, int &kind, int &r0) {
        if (KIND == 2) {
            off = G.ib + k * kS;
            cnt = min(kS, G.ie - off);
            kind = 0;
            r0 = 0;
        } else {
            const Item it = a.items[G.ib + k];
            off = it.off;
            cnt = it.cnt;
            kind = it.kind;
            r0 = it.mask;
        }
    };
    auto prefetch = [&](int k) {
        int off, cnt, kind, r0;
        item_of(k, off, cnt, kind, r0);
        const int buf = k & 1;
        const float *src;
        if (kind == 2) {
            src = a.phiF + ((size_t)off * 3 * P + r0) * FT;
        } else {
            src = a.wF + (size_t)off * FT;
            if (KIND != 2)
                for (int i = tid; i < cnt * 2; i += kThr)
                    cp16(reinterpret_cast<char *>(&sm.raw[buf][i >> 1]) + 16 * (i & 1),
                         reinterpret_cast<const char *>(a.pool + off + (i >> 1)) + 16 * (i & 1));
        }
        constexpr int CH = FT / 4;
        for (int i = tid; i < cnt * CH; i += kThr) {
            const int r = i / CH, c = i % CH;
            cp16(&sm.B[buf][r * FT + ((c ^ ((r & 3) << 1)) << 2)], src + (size_t)r * FT + c * 4);
        }
        const int kend = (cnt + 7) & ~7;
        for (int i = cnt * FT + tid; i < kend * FT; i += kThr) sm.B[buf][i] = 0.f;
    };

    if (nitems > 0) prefetch(0);
    cp_commit();
    for (int k = 0; k < nitems; ++k) {
        if (k + 1 < nitems) prefetch(k + 1);
        cp_commit();
        cp_wait1();
        __syncthreads();
        int off, cnt, kind, r0;
        item_of(k, off, cnt, kind, r0);
        const int buf = k & 1;
        // ------------------------------------------------------ item preparation
        if (KIND != 2 && kind != 2) {
            if (tid < cnt) {
                const double4 s = sm.raw[buf][tid];
                sm.loc[tid] = make_float4((float)(s.x - G.cx), (float)(s.y - G.cy), (float)(s.z - G.cz), 0.f);
            } else if (tid < ((cnt + 7) & ~7)) {
                sm.loc[tid] = make_float4(4.f, 4.f, 4.f, 0.f);   // padding: finite tile entry, zero weight row
            }
        } else if (KIND == 0 && kind == 2) {
            if (sm.down_slot != off) {
                // BLI bases of the leaf's targets in this target panel (bli_module.f90:50-113)
                if (tid < G.nt) {
                    const double2 e = a.xieta[G.tgt + tid];
                    const double *nodes = a.tgt_nodes + (size_t)off * 2 * n;
                    double f[kMaxDegree + 1];
                    dev::bli_basis(e.x, nodes, n, f);
                    for (int i = 0; i < n; ++i) sm.fx[tid][i] = (float)f[i];
                    dev::bli_basis(e.y, nodes + n, n, f);
                    for (int i = 0; i < n; ++i) sm.fe[tid][i] = (float)f[i];
                }
            }
        } else if (KIND == 2) {
            // BLI bases of the unit's points in the source panel
            const double *nodes = a.tgt_nodes + (size_t)G.tgt * 2 * n;
            double f[kMaxDegree + 1];
            if (tid < cnt) {
                dev::bli_basis(a.xieta[off + tid].x, nodes, n, f);
                for (int i = 0; i < n; ++i) sm.fx[tid][i] = (float)f[i];
            } else if (tid >= kS && tid - kS < cnt) {
                dev::bli_basis(a.xieta[off + tid - kS].y, nodes + n, n, f);
                for (int i = 0; i < n; ++i) sm.fe[tid - kS][i] = (float)f[i];
            }
        }
        {
            // split the staged B tile once for the whole CTA, in fragment order
            const float *Bt = sm.B[buf];
            const int nout = ((cnt + 7) >> 3) * NT * 32;
            for (int o = tid; o < nout; o += kThr) {
                const int ln = o & 31, j = (o >> 5) % NT, kk = (o >> 5) / NT;
                const int kr = kk * 8 + (ln & 3), col = j * 8 + (ln >> 2);
                uint32_t h0, l0, h1, l1;
                split_tf32(Bt[bofs<FT>(kr, col)], h0, l0);
                split_tf32(Bt[bofs<FT>(kr + 4, col)], h1, l1);
                sm.Bf[o] = make_float4(__uint_as_float(h0), __uint_as_float(h1), __uint_as_float(l0),
                                       __uint_as_float(l1));
            }
        }
        __syncthreads();
        if (KIND == 0 && kind == 2 && tid == 0) sm.down_slot = off;
        // ------------------------------------------------------ tensor-core tiles
        // The tensor cores accumulate without round-to-nearest, so each item
        // (at most 8 k-steps) gets fresh accumulators that are then added to the
        // running sums with IEEE FP32 adds; chaining hundreds of k-steps in one
        // accumulator would bias the result toward zero.
        if (warp_live) {
            float ai[NC][NT][4];
#pragma unroll
            for (int c = 0; c < NC; ++c)
#pragma unroll
                for (int j = 0; j < NT; ++j)
#pragma unroll
                    for (int e = 0; e < 4; ++e) ai[c][j][e] = 0.f;
            const int ksteps = (cnt + 7) >> 3;
            for (int kk = 0; kk < ksteps; ++kk) {
                float av[NC][4];
#pragma unroll
                for (int cc = 0; cc < 2; ++cc) {
                    const int col = kk * 8 + t4 + 4 * cc;
                    const bool cvalid = col < cnt;
#pragma unroll
                    for (int rr = 0; rr < 2; ++rr) {
                        const int idx = rr + 2 * cc;   // a0 (g, t4), a1 (g+8, t4), a2 (g, t4+4), a3 (g+8, t4+4)
                        const bool on = cvalid && rv[rr];
                        if (KIND == 2) {
                            const int row = warp * 16 + g + 8 * rr;
                            (void)row;
                            av[0][idx] = on ? sm.fx[col][rk[rr][0]] * sm.fe[col][rk[rr][1]] : 0.f;
                        } else if (KIND == 0 && kind == 2) {
                            const int m = sm.kmap[r0 + (on ? col : 0)];
                            const int row = warp * 16 + g + 8 * rr;
                            const float b = on ? sm.fx[row][m & 255] * sm.fe[row][(m >> 8) & 255] : 0.f;
                            const int j = m >> 16;
                            av[0][idx] = b * el[rr][j];
                            av[1][idx] = b * ep[rr][j];
                        } else {
                            // padded rows carry zero frames (leaf) and padded columns
                            // a far dummy point with zero weight, so no masks are needed
                            const float4 s = sm.loc[col];
                            const float dx = s.x - tl[rr][0], dy = s.y - tl[rr][1], dz = s.z - tl[rr][2];
                            const float v = val32(dx * dx + dy * dy + dz * dz);
                            if (KIND == 0) {
                                av[0][idx] = v * (el[rr][0] * dx + el[rr][1] * dy + el[rr][2] * dz);
                                av[1][idx] = v * (ep[rr][0] * dx + ep[rr][1] * dy + ep[rr][2] * dz);
                            } else {
                                av[0][idx] = v * dx;
                                av[1][idx] = v * dy;
                                av[2][idx] = v * dz;
                            }
                        }
                    }
                }
                uint32_t ah[NC][4], al[NC][4];
#pragma unroll
                for (int c = 0; c < NC; ++c)
#pragma unroll
                    for (int e = 0; e < 4; ++e) split_tf32(av[c][e], ah[c][e], al[c][e]);
#pragma unroll
                for (int j = 0; j < NT; ++j) {
                    const float4 bf = sm.Bf[(kk * NT + j) * 32 + lane];
                    const uint32_t bh0 = __float_as_uint(bf.x), bh1 = __float_as_uint(bf.y);
                    const uint32_t bl0 = __float_as_uint(bf.z), bl1 = __float_as_uint(bf.w);
#pragma unroll
                    for (int c = 0; c < NC; ++c) {
                        mma8(ai[c][j], ah[c], bh0, bh1);
                        mma8(ai[c][j], ah[c], bl0, bl1);
                        mma8(ai[c][j], al[c], bh0, bh1);
                    }
                }
            }
#pragma unroll
            for (int c = 0; c < NC; ++c)
#pragma unroll
                for (int j = 0; j < NT; ++j)
#pragma unroll
                    for (int e = 0; e < 4; ++e) acc[c][j][e] += ai[c][j][e];
        }
        __syncthreads();
    }
    cp_wait0();

    // ---------------------------------------------------------- epilogue
    if (!warp_live) return;
#pragma unroll
    for (int rr = 0; rr < 2; ++rr) {
        if (!rv[rr]) continue;
        const int row = warp * 16 + g + 8 * rr;
        if (KIND == 0) {
            const int pos = G.tgt + row;
            const int idx = a.perm[pos];
            const double4 c = a.tgt[pos];
            dev::Tgt T;
            dev::tgt_init(T, c.x, c.y, c.z);
            double sx = 0.0, sy = 0.0;
            if (T.live) dev::gref_exact(T, c.x, c.y, c.z, sx, sy);   // the self pair, in FP64
            const double ar = a.area[pos];
#pragma unroll
            for (int j = 0; j < NT; ++j)
#pragma unroll
                for (int h = 0; h < 2; ++h) {
                    const int f = a.f0 + j * 8 + 2 * t4 + h;
                    if (f >= a.nf) continue;
                    const double w = ar * a.ssh[(size_t)f * a.ld_ssh + idx];
                    a.out_x[(size_t)f * a.ld_out + idx] = (double)acc[0][j][2 * rr + h] + sx * w;
                    a.out_y[(size_t)f * a.ld_out + idx] = (double)acc[1][j][2 * rr + h] + sy * w;
                }
        } else {
            const int p = G.row0 + row;
#pragma unroll
            for (int j = 0; j < NT; ++j)
#pragma unroll
                for (int h = 0; h < 2; ++h) {
                    const int f = j * 8 + 2 * t4 + h;
#pragma unroll
                    for (int c = 0; c < NC; ++c)
                        a.partial[(((size_t)G.out * P + p) * NC + c) * FT + f] = acc[c][j][2 * rr + h];
                }
        }
    }
}

// Per-field FP32 weights of the points in pool order: wF[pos][f] =
// kCons * area[pos] * ssh[f0 + f][caller index], zero for fields past nf.
// One block transposes a tile of 32 consecutive caller indices x FT fields
// through shared memory, so the reads of ssh (caller order, field-major) and
// the writes of wF (pool order, field-minor) are both whole rows.
__global__ void prep_mix_kernel(const double *__restrict__ area, const double *__restrict__ ssh, int64_t ld,
                                const int32_t *__restrict__ iperm, int n, int f0, int nf, int FT,
                                float *__restrict__ wF) {
    __shared__ float tile[32][64 + 1];
    __shared__ int pos_s[32];
    const int idx0 = blockIdx.x * 32, lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int idx = idx0 + lane;
    const bool live = idx < n;
    const int pos = live ? iperm[idx] : 0;
    const double scale = live ? dev::kCons * area[pos] : 0.0;
    if (warp == 0) pos_s[lane] = live ? pos : -1;
    for (int f = warp; f < FT; f += blockDim.x >> 5) {
        const int ff = f0 + f;
        tile[lane][f] = (live && ff < nf) ? (float)(scale * ssh[(size_t)ff * ld + idx]) : 0.f;
    }
    __syncthreads();
    for (int r = warp; r < 32; r += blockDim.x >> 5) {
        const int p = pos_s[r];
        if (p < 0) continue;
        for (int f = lane; f < FT; f += 32) wF[(size_t)p * FT + f] = tile[r][f];
    }
}

// Sums unit partials (unit order, FP64) into FP32 rows: rows_per_slot rows of
// FT floats per slot, written at dst + (slot * rows_per_slot + row) * FT.
__global__ void finalize_mix_kernel(const int32_t *__restrict__ unit_beg, const float *__restrict__ partial,
                                    int nslots, int rows_per_slot, int FT, float *__restrict__ dst) {
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const long long per = (long long)rows_per_slot * FT;
    if (t >= (long long)nslots * per) return;
    const int s = (int)(t / per);
    const long long rf = t % per;
    double acc = 0.0;
    for (int u = unit_beg[s]; u < unit_beg[s + 1]; ++u) acc += (double)partial[(size_t)u * per + rf];
    dst[(size_t)s * per + rf] = (float)acc;
}

template <int KIND, int NT>
static void launch_kind(const MixArgs &a, int ngroups, cudaStream_t st) {
    const size_t smem = sizeof(Smem);
    static std::atomic<unsigned long long> done{0};
    smem_attr_once((const void *)mix_kernel<KIND, NT>, (int)smem, done);
    mix_kernel<KIND, NT><<<ngroups, kThr, smem, st>>>(a);
}

void launch_mix(int kind, int FT, const MixArgs &a, int ngroups, cudaStream_t st) {
    if (ngroups <= 0) return;
    if (FT == 64) {
        if (kind == 0) launch_kind<0, 8>(a, ngroups, st);
        else if (kind == 1) launch_kind<1, 8>(a, ngroups, st);
        else launch_kind<2, 8>(a, ngroups, st);
    } else {
        if (kind == 0) launch_kind<0, 4>(a, ngroups, st);
        else if (kind == 1) launch_kind<1, 4>(a, ngroups, st);
        else launch_kind<2, 4>(a, ngroups, st);
    }
}

void launch_prep_mix(const double *area, const double *ssh, int64_t ld, const int32_t *iperm, int n, int f0, int nf,
                     int FT, float *wF, cudaStream_t st) {
    if (n <= 0) return;
    prep_mix_kernel<<<(n + 31) / 32, 256, 0, st>>>(area, ssh, ld, iperm, n, f0, nf, FT, wF);
}

void launch_finalize_mix(const int32_t *unit_beg, const float *partial, int nslots, int rows_per_slot, int FT,
                         float *dst, cudaStream_t st) {
    const long long tot = (long long)nslots * rows_per_slot * FT;
    if (tot <= 0) return;
    finalize_mix_kernel<<<(unsigned)((tot + 255) / 256), 256, 0, st>>>(unit_beg, partial, nslots, rows_per_slot, FT,
                                                                       dst);
}

size_t mix_smem_bytes() { return sizeof(Smem); }

}  // namespace mix
}  // namespace sal
