// Leaf pass (MODE 0) and proxy pass (MODE 1) of the batched form on the
// 5th-generation tensor cores (tcgen05).  The proxy pass is the same machine
// with the Chebyshev proxies of a target slot as targets (at most 85 per
// group), three Cartesian components val (s - x) instead of the projected
// east / north ones (3 x 85 columns fill N = 256), no self pairs, no DOWN
// items, and the group's end written to its unit's partial rows.  The leaf
// pass is described below.
//
// One CTA per SM at a time, each walking leaf groups of up to 128 targets
// in pool order with a stride of the grid size.  A group's work is a list of
// items (<= 64 sources, or <= 64 Cartesian rows of a DOWN interpolation), cut
// into stages of 32 K columns (four k-steps of 8).  The contraction is
//     D[field part, target component] += W[field part, k] * T[k, target component]
// with M = 128 weight rows (64 fields, TF32 hi and lo parts, ordered so that
// field f's hi row 32(f/16) + f%16 and lo row +16 share a warp) and N = 256
// kernel-tile columns (east of the 128 targets, then north).  One tcgen05.mma
// costs the same whatever its N, so N = 256 keeps the tensor cores at full
// width: per k-step two MMAs, W * T_hi and W * T_lo, give all four hi/lo
// cross products.
// Warp roles:
//   warps 0-7   producers.  A task is one k-step of a 32-target row block:
//               8 kernel-tile entries per component and row in FP32, split
//               into TF32 hi + lo, stored to shared memory in the canonical
//               K-major layout (the MMA's B operand).  A stage's tasks are
//               dealt so that small groups use every warp (see the producer
//               branch).  The self pair enters as the tile's diagonal entry:
//               the reference kernel's FP64 value at distance zero (rounding
//               noise).  The sources' FP32 coordinates (per k-step x[8] y[8]
//               z[8]) come from shared memory, copied there by the loader.
//   warp 8      issues the MMAs.
//   warp 9      loads, per stage, the weight tiles (pre-split TF32 hi / lo,
//               written once per solve by split_store_kernel) and the
//               sources' coordinates (leaf and proxy passes) or BLI factors
//               (upward pass), with bulk copies into a 4-deep ring, and
//               prefetches the next item's tiles into L2.
//   warps 10-13 fold finished accumulator chains into the running sums and
//               write the outputs (warp w: tensor memory lanes 32(w%4)..+31).
// FP16 leaf pass (sal_tune.f16): the same machine with kind::f16 MMAs, 16
// sources per MMA.  A stage is 64 sources (eight units of 8, the split
// store's granularity; an odd unit count is completed with a zero unit);
// kernel tiles and weight tiles are FP16 hi + lo (11 + 11 bits, as TF32 hi +
// lo), in the same shared-memory bytes, so each stage carries twice the
// sources for the same MMA count and stores.  FP16's range needs scales:
// every target's kernel values are multiplied by a power of two that takes
// its largest one (computed once per plan) to at most 2^12, every field's
// source weights and its potentials by powers of two of their own (per
// solve), and the fold divides them out of each chain; DOWN items (O(1)
// interpolation weights against potentials) form chains of their own.
// Kernel-tile store (sal_tune.tile_store, FP16 leaf pass): the kernel tiles
// depend on the grid alone.  A recording launch (TS 1) computes them and also
// writes them to device memory; a replaying launch (TS 2) has the loader copy
// each stage's tiles and weights into two shared-memory byte rings, and the
// idle producer warps fold beside the fold warps; a partial replay (TS 3)
// has producer warp 0 copy the stored items' tiles into the ring slot while
// the producers compute the others.  All three give the computing launch's
// results bit for bit.
// The tensor cores accumulate with truncation, so one chain over all of a
// target's sources would bias the result toward zero: a chain ends after about
// 32 k-steps (plan flag kTcFlush) and is folded into the group's running sums
// with round-to-nearest FP32 adds.  The running sums live in tensor memory
// (columns 256-511, the accumulator's row layout) next to the accumulator
// (columns 0-255); shared memory holds only the operand rings.  The next chain
// starts once the fold warps have read the accumulator; the two-stage
// kernel-tile ring lets the producers run on meanwhile.
#include <cuda_fp16.h>
#include <algorithm>
#include <cuda_runtime.h>

#include "kernels.cuh"
#include "mixed.cuh"

namespace sal {
namespace mix {

using dev::smem_u32;

namespace {

constexpr int kProdWarps = 8;
constexpr int kProducers = kProdWarps * 32;
constexpr int kMmaWarp = kProdWarps;
constexpr int kLoadWarp = kProdWarps + 1;
constexpr int kFoldWarps = 4;                     // one per tensor memory lane quarter
constexpr int kThreads = (kProdWarps + 2 + kFoldWarps) * 32;   // 448
constexpr int kF = 64;                            // fields
constexpr int kStageK = 32;                       // K columns per stage (four k-steps of 8)
constexpr int kStageKs = kStageK / 8;             // k-steps per stage
constexpr int kKStages = 2;                       // kernel-tile ring
constexpr int kWStages = 4;                       // weight / upward-factor ring
constexpr int kAuxFloats = kStageKs * 16 * (kMaxDegree + 1);   // upward factors of a stage's k-steps
constexpr int kTileFloats = 2048;                 // kernel tile of one k-step: 256 rows x 8, one of hi / lo
constexpr int kWStepFloats = 1024;                // weight tile of one k-step: 128 rows x 8
constexpr int kTmemCols = 512;
constexpr int kKmap = 3 * (kMaxDegree + 1) * (kMaxDegree + 1) + 64;
constexpr uint32_t kWaitPolls = 1u << 22;
constexpr float kC1F = (float)dev::kC1;
constexpr float kTwoC2F = (float)(2.0 * dev::kC2);

static_assert(kTcChunk % kStageK == 0, "items are whole stages");

// instruction descriptor: D F32, A/B TF32, both K-major, N = 256, M = 128
constexpr uint32_t kIdesc = (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(256 >> 3) << 17) |
                            ((uint32_t)(128 >> 4) << 24);
// the same for kind::f16 with A/B FP16 (format 0), 16 sources per MMA
constexpr uint32_t kIdescF16 = (1u << 4) | ((uint32_t)(256 >> 3) << 17) | ((uint32_t)(128 >> 4) << 24);
// FP16 leaf pass: a stage is 64 sources, eight units of 8 (a unit is one
// TF32 k-step: the split store's granularity); a unit of the FP16 weight store
// is 128 rows x 8 halves, 8-row groups 128 B apart (2 KB)
constexpr int kStageKF16 = 64;
constexpr int kW16UnitBytes = 2048;
// FP16 operands are scaled by powers of two to at most 2^12 (FP16 max 65504)
constexpr int kF16TopExp = 12;
static_assert(kStageKF16 == kTcChunk, "an FP16 stage is one item: the tile store's layout");

// Replay of the kernel-tile store: the stages' kernel tiles and weight tiles
// go into two byte rings (a stage takes its own size, so the small groups'
// stages do not hold whole 64 KB slots), with up to kRStages stages in
// flight.  A stage's tiles are packed: per MMA step and hi / lo, the group's
// east rows then its north rows (rows rounded up to 16); an MMA reads 256
// rows from a tile's start, the rows past the group's are columns no fold
// reads.
constexpr int kRStages = 8;
constexpr int kTRingBytes = 180 * 1024;
constexpr int kWRingBytes = 44 * 1024;

// Shared memory of one CTA.  Computing launches: a kKStages-deep ring of
// 64 KB kernel-tile stages, a kWStages-deep weight ring and the producers'
// buffers (source coordinates / upward factors per weight stage, DOWN bases,
// the DOWN row map).  Replay: the two byte rings and the offsets of the
// stages in flight.
template <int TS>
struct TcSmem {
    static constexpr bool kReplay = TS == 2;
    static constexpr int KS = kReplay ? kRStages : kKStages;   // kernel-tile stage slots
    static constexpr int WS = kReplay ? 1 : kWStages;          // weight stage slots
    static constexpr size_t kKtBytes = kReplay ? (size_t)kTRingBytes : (size_t)kKStages * kStageKs * 2 * kTileFloats * 4;
    static constexpr size_t kWtBytes = kReplay ? (size_t)kWRingBytes : (size_t)kWStages * kStageKs * kWStepFloats * 4;
    unsigned char ring[kKtBytes + kWtBytes];
    float aux[kReplay ? 1 : kWStages][kReplay ? 4 : kAuxFloats];   // per stage: BLI factors F[n][8] G[n][8] per k-step
    float fx[kReplay ? 1 : kTcRows][kMaxDegree + 1];              // per target row: BLI bases in the current DOWN slot
    float fe[kReplay ? 1 : kTcRows][kMaxDegree + 1];
    int kmap[kReplay ? 1 : kKmap];
    uint32_t toff[KS], tlen[KS], woff[KS], wlen[KS];             // replay: each stage slot's ranges in the rings
    uint64_t kfull[KS], kempty[KS], wfull[WS], wempty[WS], accfull, accfree, fin;
    uint32_t tmem_base;
    int abort;
    // computing launches: kernel tile (stage slot, k-step, hi / lo), weight stage jb
    __device__ __forceinline__ float *Kt(uint32_t slot, int s, int h) {
        return reinterpret_cast<float *>(ring + (((size_t)slot * kStageKs + s) * 2 + h) * kTileFloats * 4);
    }
    __device__ __forceinline__ float *Wt(uint32_t jb) {
        return reinterpret_cast<float *>(ring + kKtBytes + (size_t)jb * kStageKs * kWStepFloats * 4);
    }
};
template <int TS> constexpr size_t tc_smem_need() { return sizeof(TcSmem<TS>) + 1024; }


// Packed FP32x2 arithmetic (two kernel-tile columns per instruction).
__device__ __forceinline__ float2 sub2(float2 a, float2 b) {
    unsigned long long r;
    asm("sub.rn.f32x2 %0, %1, %2;"
        : "=l"(r)
        : "l"(*reinterpret_cast<unsigned long long *>(&a)), "l"(*reinterpret_cast<unsigned long long *>(&b)));
    return *reinterpret_cast<float2 *>(&r);
}
__device__ __forceinline__ float2 f2(float x) { return make_float2(x, x); }
__device__ __forceinline__ float rsqrt_approx(float x) {
    float r;
    asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}
__device__ __forceinline__ float rcp_approx(float x) {
    float r;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}

__device__ __forceinline__ float tf32_hi(float x) {
    uint32_t r;
    asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
    return __uint_as_float(r);
}

// Hint: fetch a global range into L2 ahead of its bulk copy (16-byte
// aligned, a multiple of 16 bytes).
__device__ __forceinline__ void prefetch_l2(const void *p, uint32_t bytes) {
    asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(p), "r"(bytes) : "memory");
}

__device__ __forceinline__ void mbar_arrive(uint64_t *bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}
// Bounded wait on an mbarrier phase; on time-out raises the error flag and
// the CTA-wide abort flag (later waits then give up after one poll).  A phase
// that has already completed costs one poll and no read of the flag: every
// shared-memory round trip is on the producers' critical path.
__device__ __forceinline__ void wait_bounded(uint64_t *bar, uint32_t parity, volatile int *abort, int *err) {
    if (dev::mbar_try_wait(bar, parity)) return;
    for (uint32_t it = 0; it < kWaitPolls; ++it) {
        if (*abort) return;
        if (dev::mbar_try_wait(bar, parity)) return;
    }
    *abort = 1;
    atomicExch(err, dev::kErrTimeout);
}
// Bounded wait that ignores the abort flag (drains copies and MMAs in flight
// before the CTA exits).
__device__ __forceinline__ void wait_drain(uint64_t *bar, uint32_t parity, int *err) {
    for (uint32_t it = 0; it < kWaitPolls; ++it)
        if (dev::mbar_try_wait(bar, parity)) return;
    atomicExch(err, dev::kErrTimeout);
}

// Named barrier 1 over the producer warps.
__device__ __forceinline__ void producers_sync() { asm volatile("bar.sync 1, %0;" ::"r"(kProducers) : "memory"); }

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

// D[tmem] (+)= A[smem] * B[smem]
__device__ __forceinline__ void mma_ss(uint32_t d_tmem, uint64_t a, uint64_t b, uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(d_tmem),
        "l"(a), "l"(b), "r"(kIdesc), "r"(accumulate)
        : "memory");
}
// D[tmem] (+)= A[smem] * B[smem], FP16 operands, 16 sources
__device__ __forceinline__ void mma_ss_f16(uint32_t d_tmem, uint64_t a, uint64_t b, uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(d_tmem),
        "l"(a), "l"(b), "r"(kIdescF16), "r"(accumulate)
        : "memory");
}
// Descriptor of an FP16 weight tile of two store units (16 sources): K core
// matrices one unit (2 KB) apart, 8-row groups 128 B apart.
__device__ __forceinline__ uint64_t smem_desc_w16(const void *p) {
    const uint64_t addr = smem_u32(p);
    return ((addr >> 4) & 0x3FFFull) | ((uint64_t)(kW16UnitBytes >> 4) << 16) | ((uint64_t)(128 >> 4) << 32) |
           (1ull << 46);
}
// FP16 hi + lo of two values, packed as half2 words: hi = round(v), lo =
// round(v - hi).  (Rounding hi with cvt.rna.tf32 first, then converting both
// halves, measured 4.6 % slower in the leaf pass.)
__device__ __forceinline__ void split_f16x2(float a, float b, uint32_t &hi, uint32_t &lo) {
    const __half2 h = __floats2half2_rn(a, b);
    const float2 back = __half22float2(h);
    const __half2 l = __floats2half2_rn(a - back.x, b - back.y);
    hi = *reinterpret_cast<const uint32_t *>(&h);
    lo = *reinterpret_cast<const uint32_t *>(&l);
}
// The power of two that takes a magnitude m to at most 2^kF16TopExp (1 for
// m = 0), and its inverse.
__host__ __device__ inline float f16_scale(float m) {
    if (!(m > 0.f)) return 1.f;
    int e;
    frexpf(m, &e);   // m < 2^e
    e = kF16TopExp - e;
    e = e < -120 ? -120 : (e > 120 ? 120 : e);
    return ldexpf(1.f, e);
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
__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }
__device__ __forceinline__ void tmem_st16(uint32_t taddr, const float (&v)[16]) {
    asm volatile(
        "tcgen05.st.sync.aligned.32x32b.x16.b32 [%0], {%1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
        "%15, %16};" ::"r"(taddr),
        "r"(__float_as_uint(v[0])), "r"(__float_as_uint(v[1])), "r"(__float_as_uint(v[2])), "r"(__float_as_uint(v[3])),
        "r"(__float_as_uint(v[4])), "r"(__float_as_uint(v[5])), "r"(__float_as_uint(v[6])), "r"(__float_as_uint(v[7])),
        "r"(__float_as_uint(v[8])), "r"(__float_as_uint(v[9])), "r"(__float_as_uint(v[10])),
        "r"(__float_as_uint(v[11])), "r"(__float_as_uint(v[12])), "r"(__float_as_uint(v[13])),
        "r"(__float_as_uint(v[14])), "r"(__float_as_uint(v[15]))
        : "memory");
}
__device__ __forceinline__ void tmem_wait_st() { asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory"); }

// BLI basis (FP64, stored as FP32) of one coordinate of a target over one
// axis's Chebyshev nodes.  Out of line: its local array stays out of the
// stage loop's registers.
__device__ __noinline__ void down_basis(double x, const double *nodes, int n, float *out) {
    double f[kMaxDegree + 1];
    dev::bli_basis(x, nodes, n, f);
    for (int i = 0; i < n; ++i) out[i] = (float)f[i];
}

// Byte offset of element (row, k) of a canonical K-major tile without
// swizzle (8-row x 16-byte core matrices, K halves 128 B apart, 8-row groups
// 256 B apart), k < 8.
__host__ __device__ constexpr int canon(int row, int k) {
    return (row >> 3) * 256 + (k >> 2) * 128 + (row & 7) * 16 + (k & 3) * 4;
}
// Weight-tile row of field f's hi (part 0) or lo (part 1) TF32 part: the two
// rows of a field sit in one 32-lane quarter of the accumulator, 16 apart.
__host__ __device__ constexpr int wrow(int f, int part) { return 32 * (f >> 4) + 16 * part + (f & 15); }

}  // namespace

// Writes one finished 16-column chunk x (this lane's accumulator row, the
// running sum already added) to its destination at a group's end.  Lanes
// 0-15 hold fields' hi rows, lanes 16-31 the same fields' lo rows; per
// column pair, lanes 0-15 write the even column and lanes 16-31 the odd one,
// so hi + lo of a field meet in one lane.
template <int MODE>
__device__ __forceinline__ void emit_chunk(const float (&x)[16], int c0, int f, int odd, int nt, int idk, double *out,
                                           bool wr, float *part, int half) {
#pragma unroll
    for (int m = 0; m < 8; ++m) {
        const float lo_even = __shfl_down_sync(0xffffffffu, x[2 * m], 16);
        const float hi_odd = __shfl_up_sync(0xffffffffu, x[2 * m + 1], 16);
        const int j = c0 + 2 * m + odd;   // column
        if (MODE == 0) {
            const int t = j >= half ? j - half : j;
            const int ti = __shfl_sync(0xffffffffu, idk, t & 31);
            const double v = odd ? (double)hi_odd + (double)x[2 * m + 1] : (double)x[2 * m] + (double)lo_even;
            if (wr && t < nt) out[ti] = v;
        } else {
            const float v = odd ? hi_odd + x[2 * m + 1] : x[2 * m] + lo_even;
            if (MODE == 2) {
                // upward rows: column j is proxy row0 + j; the unit's partial
                // holds one row of 64 fields per proxy
                if (wr && j < nt) part[(size_t)j * kF + f] = v;
            } else {
                // proxy rows: column j = 85c + r is component c of proxy r; the
                // unit's partial holds (proxy, component) rows of 64 fields
                const int c = j / kTcProxyRows, r = j - c * kTcProxyRows;
                if (wr && c < 3 && r < nt) part[((size_t)r * 3 + c) * kF + f] = v;
            }
        }
    }
}

// Folds a finished accumulator chain into the running sums (warp-collective;
// this warp's lane quarter q: fields 16q..16q+15, hi rows in lanes 0-15 and
// lo rows in lanes 16-31).  The running sums live in tensor memory next to
// the accumulator (columns 256-511, same row layout): running sum (+)= chain
// with round-to-nearest FP32 adds (the group's first chain stores).  At a
// group's end only the chunks that hold targets are folded, and emit_sums
// writes them out after the accumulator has been handed back to the MMA
// warp, so the next group's first chain overlaps the output writes.
// MODE 0 (leaf): columns half c + t are component c (east, north) of target
// t (half = 128, or the group's rows rounded up to 16 for the packed tiles of
// a replayed kernel-tile store).  MODE 1 (proxy): columns 85c + r are
// Cartesian component c of proxy r.  MODE 2 (upward): columns j < 128 are
// proxies row0 + j.
//
// FP16 leaf pass (scaled, the same in every lane): the chain's operands were
// scaled by powers of two, the weight rows of field f by 1 / fsc and (kernel
// chains) the kernel tile's column of target t by tscale[tgt + t] (DOWN
// chains: unscaled columns).  The running sums are kept in the columns'
// scaled domain: a kernel chain adds chain x fsc, a DOWN chain chain x fsc x
// tscale, and emit_sums multiplies by tinv = 1 / tscale.  Powers of two
// commute with rounding, so this gives the unscaled sums' bits while kernel
// chains (all but one or a few per group) need no per-column factors.
// Several warps of one lane quarter can share a fold: warp part_i of nparts
// takes the chunk pairs (2p, 2p + 1) with p % nparts == part_i, and emits
// the same chunks.

// Chunks of 16 columns a fold covers: per component, at a group's end only
// those that hold targets; a pair (2p, 2p + 1) at a time.
template <int MODE>
__device__ __forceinline__ int fold_per(bool end, int nt, int half) {
    return (MODE != 1 && end) ? (nt + 15) / 16 : (MODE == 0 ? half / 16 : 8);
}

template <int MODE>
__device__ __noinline__ void fold_chain(uint32_t td, int lane, bool end, bool first, int tgt, int nt, bool scaled,
                                        float fsc, bool down, const float *__restrict__ tscale, int half, int part_i,
                                        int nparts) {
    // per target slot 32k + lane: its scale (DOWN chains)
    float csd[4] = {1.f, 1.f, 1.f, 1.f};
    if (MODE == 0 && scaled && down)
#pragma unroll
        for (int k = 0; k < 4; ++k) csd[k] = 32 * k + lane < nt ? tscale[tgt + 32 * k + lane] : 1.f;
    // the chain into the running sums' domain, on a 16-column chunk starting at column c
    auto unscale = [&](float (&x)[16], int c) {
        if (!scaled) return;
#pragma unroll
        for (int m = 0; m < 16; ++m) x[m] *= fsc;
        if (down) {
            const int b = c >= half ? c - half : c, k = b >> 5;
            const float src = k == 0 ? csd[0] : k == 1 ? csd[1] : k == 2 ? csd[2] : csd[3];
#pragma unroll
            for (int m = 0; m < 16; ++m) x[m] *= __shfl_sync(0xffffffffu, src, (b & 31) + m);
        }
    };
    const int per = fold_per<MODE>(end, nt, half);
    const int nchunk = MODE == 2 ? per : 2 * per;   // upward: one component, columns 0..127
    auto col = [&](int i) { return (i / per) * half + (i % per) * 16; };
    // two chunks' loads in flight per wait: the MMA warp waits for this fold
    float x0[16], x1[16], r0[16], r1[16];
#pragma unroll 1
    for (int i = 2 * part_i; i < nchunk; i += 2 * nparts) {
        const bool two = i + 1 < nchunk;   // a group's end in the upward pass can leave one
        const int c0 = col(i), c1 = col(two ? i + 1 : i);
        tmem_ld16(td + c0, x0);
        tmem_ld16(td + c1, x1);
        if (!first) {
            tmem_ld16(td + 256 + c0, r0);
            tmem_ld16(td + 256 + c1, r1);
        }
        tmem_wait_ld();
        unscale(x0, c0);
        unscale(x1, c1);
        if (!first) {
#pragma unroll
            for (int m = 0; m < 16; ++m) {
                x0[m] += r0[m];
                x1[m] += r1[m];
            }
        }
        tmem_st16(td + 256 + c0, x0);
        if (two) tmem_st16(td + 256 + c1, x1);
    }
    tmem_wait_st();
}

// A group's end: its running sums (this warp's chunks of fold_chain) to the
// destinations, hi + lo added in FP64: MODE 0 the caller's outputs, MODE 1 /
// 2 the unit's partial rows `part`.
template <int MODE>
__device__ __noinline__ void emit_sums(uint32_t td, int q, int lane, int tgt, int nt, const int32_t *__restrict__ perm,
                                       double *out_x, double *out_y, int64_t ld_out, int f0, int nf, bool skip,
                                       float *part, bool scaled, const float *__restrict__ tinv, int half, int part_i,
                                       int nparts) {
    const int f = 16 * q + (lane & 15), odd = lane >> 4;
    float cse[4] = {1.f, 1.f, 1.f, 1.f};   // per target slot 32k + lane: its scale's inverse
    if (MODE == 0 && scaled)
#pragma unroll
        for (int k = 0; k < 4; ++k) cse[k] = 32 * k + lane < nt ? tinv[tgt + 32 * k + lane] : 1.f;
    int idx[4] = {0, 0, 0, 0};   // caller index of target slot 32k + lane
    if (MODE == 0)
#pragma unroll
        for (int k = 0; k < 4; ++k) idx[k] = 32 * k + lane < nt ? perm[tgt + 32 * k + lane] : 0;
    const bool wr = (MODE != 0 || f0 + f < nf) && !skip;
    double *ox = MODE == 0 ? out_x + (size_t)(f0 + f) * ld_out : nullptr;
    double *oy = MODE == 0 ? out_y + (size_t)(f0 + f) * ld_out : nullptr;
    const int per = fold_per<MODE>(true, nt, half);
    const int nchunk = MODE == 2 ? per : 2 * per;
    auto col = [&](int i) { return (i / per) * half + (i % per) * 16; };
    float x[16];
#pragma unroll 1
    for (int i = 2 * part_i; i < nchunk; i += 2 * nparts)
#pragma unroll 1
        for (int h = i; h < i + 2 && h < nchunk; ++h) {
            const int c = col(h);
            tmem_ld16(td + 256 + c, x);
            tmem_wait_ld();
            const int b = c >= half ? c - half : c, k = b >> 5;
            if (MODE == 0 && scaled) {
                // out of the columns' scaled domain
                const float src = k == 0 ? cse[0] : k == 1 ? cse[1] : k == 2 ? cse[2] : cse[3];
#pragma unroll
                for (int m = 0; m < 16; ++m) x[m] *= __shfl_sync(0xffffffffu, src, (b & 31) + m);
            }
            const int idk = k == 0 ? idx[0] : k == 1 ? idx[1] : k == 2 ? idx[2] : idx[3];
            emit_chunk<MODE>(x, c, f, odd, nt, idk, c < half ? ox : oy, wr, part, half);
        }
}

// Outputs of target t of a leaf group without sources: its self pair alone.
__device__ __noinline__ void self_only(const TcArgs &a, const MixGroup &G, int t) {
    const int pos = G.tgt + t, idx = a.perm[pos];
    const double2 sk = a.selfk[pos];
    for (int f = 0; f < kF && a.f0 + f < a.nf; ++f) {
        const double w = (double)a.wF[(size_t)pos * kF + f];
        a.out_x[(size_t)(a.f0 + f) * a.ld_out + idx] = sk.x * w;
        a.out_y[(size_t)(a.f0 + f) * a.ld_out + idx] = sk.y * w;
    }
}

// A warp's window on a group's item records, 32 at a time: lane i holds
// record k0 + i, and the next 32 are loaded one batch ahead, so a warp that
// walks items faster than a global load returns (the MMA, loader and fold
// warps) does not wait on one load per item.  k must be warp-uniform and
// non-decreasing.
struct ItemWindow {
    const TcItem *items;
    int k0, ie;
    TcItem cur, nxt;
    __device__ __forceinline__ void start(const TcItem *it, int ib, int e, int lane) {
        items = it;
        k0 = ib;
        ie = e;
        cur = ib + lane < e ? it[ib + lane] : TcItem{};
        nxt = ib + 32 + lane < e ? it[ib + 32 + lane] : TcItem{};
    }
    __device__ __forceinline__ void seek(int k, int lane) {
        while (k >= k0 + 32) {
            cur = nxt;
            k0 += 32;
            nxt = k0 + 32 + lane < ie ? items[k0 + 32 + lane] : TcItem{};
        }
    }
    __device__ __forceinline__ TcItem get(int k, int lane) {
        seek(k, lane);
        const int l = k - k0;
        TcItem r;
        r.off = __shfl_sync(0xffffffffu, cur.off, l);
        r.cnt = __shfl_sync(0xffffffffu, cur.cnt, l);
        r.kb = __shfl_sync(0xffffffffu, cur.kb, l);
        r.kind = __shfl_sync(0xffffffffu, cur.kind, l);
        r.dx = __shfl_sync(0xffffffffu, cur.dx, l);
        r.dy = __shfl_sync(0xffffffffu, cur.dy, l);
        r.dz = __shfl_sync(0xffffffffu, cur.dz, l);
        r.row0 = __shfl_sync(0xffffffffu, cur.row0, l);
        return r;
    }
    __device__ __forceinline__ int kind(int k, int lane) {
        seek(k, lane);
        return __shfl_sync(0xffffffffu, cur.kind, k - k0);
    }
};

// JOINT: one launch over the groups of several grids (of one degree): group
// gi belongs to the grid k with J.beg[k] <= gi < J.beg[k + 1] and carries
// that grid's arguments.  Otherwise J.g[0] is the only grid.
// TS (FP16 leaf pass, one grid): 0 the producers compute the kernel tiles;
// 1 they compute them and also record them in the grid's kernel-tile store;
// 2 the loader copies them from the store into the kernel-tile ring and the
// producers only write the outputs of groups without sources.
template <int MODE, bool JOINT, bool F16, int TS = 0>
__global__ void __launch_bounds__(kThreads, 1) tc_leaf_kernel(const __grid_constant__ TcJoint J, int *err) {
    static_assert(!F16 || MODE == 0, "FP16 operands in the leaf pass only");
    static_assert(TS == 0 || (MODE == 0 && F16 && !JOINT), "kernel-tile store: FP16 leaf pass of one grid");
    constexpr int SK = F16 ? kStageKF16 : kStageK;   // sources per stage
    constexpr int SU = SK / 8;                        // store units (8 sources) per stage
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    constexpr int KS = TcSmem<TS>::KS, WS = TcSmem<TS>::WS;
    TcSmem<TS> &sm = *reinterpret_cast<TcSmem<TS> *>(smem_raw);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int n = J.g[0].d + 1, P = J.g[0].P;
    const int total = JOINT ? J.beg[J.ngrids] : J.g[0].ngroups;
    // the grid of joint group gi
    auto grid_of = [&](int gi) -> int {
        int k = 0;
        if (JOINT)
            while (k + 1 < J.ngrids && gi >= J.beg[k + 1]) ++k;
        return k;
    };
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
        for (int j = 0; j < KS; ++j) {
            // replay: the loader's arrival and its copies' bytes fill a stage
            dev::mbar_init(&sm.kfull[j], TS == 2 ? 1 : kProdWarps);
            dev::mbar_init(&sm.kempty[j], 1);
        }
        for (int j = 0; j < WS; ++j) {
            dev::mbar_init(&sm.wfull[j], 1);
            dev::mbar_init(&sm.wempty[j], 1);
        }
        dev::mbar_init(&sm.accfull, 1);
        // replay: the idle producer warps fold too, three warps per lane quarter
        dev::mbar_init(&sm.accfree, TS == 2 ? kFoldWarps + kProdWarps : kFoldWarps);
        dev::mbar_init(&sm.fin, 1);
        dev::fence_mbar_init();
        sm.abort = 0;
    }
    for (int k = tid; TS != 2 && k < kKmap; k += kThreads) {
        const int kk = k < 3 * P ? k : 0;
        const int p = kk / 3;
        sm.kmap[k] = (p % n) | ((p / n) << 8) | ((kk % 3) << 16);
    }
    if (TS == 2) {
        // replay copies only a group's rows: the ring's other rows hold
        // zeros or an earlier group's finite values (columns no output reads)
        uint4 *z = reinterpret_cast<uint4 *>(sm.ring);
        for (int i = tid; i < (int)(sizeof(sm.ring) / sizeof(uint4)); i += kThreads) z[i] = make_uint4(0u, 0u, 0u, 0u);
        dev::fence_proxy_async();
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = sm.tmem_base;
    uint32_t st = 0;   // stages this CTA has gone through

    if (TS != 2 && warp < kProdWarps) {
        // ============================================================ producers
        // A stage's tasks are (row block of 32 targets, unit) pairs, one
        // 8-source unit of 32 rows each (a TF32 stage has 4 units, an FP16
        // stage 8).  A stage costs the latency of the busiest warp's tasks,
        // so the tasks of small groups (one or two row blocks: the second
        // tile of a leaf with more than 128 points) are spread over all warps:
        //   3-4 row blocks: warp w takes row block w % 4, units w / 4 + 2i
        //   2 row blocks:   warp w takes row block w % 2, units w / 2 + 4i
        //   1 row block:    warp w takes unit w (TF32: warps 4-7 only arrive)
        // The source coordinates of a stage's k-steps (x[8] y[8] z[8] each,
        // relative to their panel's centre) arrive in shared memory with the
        // stage's weights: the loader warp copies them up to WS stages
        // ahead, so no global-memory latency sits in a producer task.

        for (int gi = blockIdx.x; gi < total; gi += gridDim.x) {
            const int gk = grid_of(gi);
            const TcArgs &a = J.g[gk];
            const MixGroup G = a.groups[gi - J.beg[gk]];
            const int ni = G.ie - G.ib;
            const int rb = (G.nt + 31) >> 5;
            const int wb = rb >= 3 ? (warp & 3) : rb == 2 ? (warp & 1) : 0;            // row block
            const int kfirst = rb >= 3 ? (warp >> 2) : rb == 2 ? (warp >> 1) : warp;    // first k-step
            const int kstride = rb >= 3 ? 2 : rb == 2 ? 4 : 8;
            const int row = 32 * wb + lane;
            const bool active = 32 * wb < G.nt, rvalid = row < G.nt;
            // canonical offsets (floats) of this thread's rows in a kernel tile:
            // leaf east / north at rows t, 128 + t; proxy x / y / z at 85c + r
            const int oe = canon(row, 0) >> 2;
            const int on = canon(MODE == 0 ? kTcRows + row : kTcProxyRows + row, 0) >> 2;
            const int oz = canon(MODE == 0 ? 0 : 2 * kTcProxyRows + row, 0) >> 2;
            const bool row_in_tile = MODE != 1 || row < kTcProxyRows;   // proxy components hold 85 rows
            // FP16 tiles: byte offset of the row's first K core matrix (8-row
            // groups 256 B apart, the two K halves 128 B apart)
            const int oe16 = (row >> 3) * 256 + (row & 7) * 16, on16 = oe16 + (kTcRows / 8) * 256;
            // the row's target relative to the leaf centre and its east /
            // north unit vectors (zero at the poles, as the reference's guard)
            float tl0 = 0.f, tl1 = 0.f, tl2 = 0.f, el0 = 0.f, el1 = 0.f, ep0 = 0.f, ep1 = 0.f, ep2 = 0.f;
            // FP16 leaf pass: this row's power-of-two scale of kernel values
            const float tsc = (F16 && rvalid) ? a.tscale[G.tgt + row] : 1.f;
            // upward: this row's proxy p = row0 + row = up_i + up_j n
            const int up_p = MODE == 2 ? G.row0 + (rvalid ? row : 0) : 0;
            const int up_i = up_p % n, up_j = up_p / n;
            if (MODE != 2 && rvalid) {
                // leaf: the pool point; proxy: proxy row0 + row of target slot G.tgt
                const double4 c = MODE == 0 ? a.tgt[G.tgt + row] : a.tgt[(size_t)G.tgt * P + G.row0 + row];
                tl0 = (float)(c.x - G.cx);
                tl1 = (float)(c.y - G.cy);
                tl2 = (float)(c.z - G.cz);
                if (MODE == 0 && (fabs(c.z - 1.0) > 1e-15) && (fabs(c.z + 1.0) > 1e-15)) {
                    const double omz = 1.0 - c.z * c.z, inv = 1.0 / sqrt(omz);
                    el0 = (float)(-c.y * inv);
                    el1 = (float)(c.x * inv);
                    ep0 = (float)(-c.z * c.x * inv);
                    ep1 = (float)(-c.z * c.y * inv);
                    ep2 = (float)(omz * inv);
                }
            }
            if (ni == 0) {
                // no sources: the self pair alone (thread t: target t)
                if (MODE == 0 && tid < G.nt && !*abort) self_only(a, G, tid);
                continue;
            }
            // the kernel values' projections; FP16: with the row's scale in them
            const float2 el0v = f2(el0 * tsc), el1v = f2(el1 * tsc), ep0v = f2(ep0 * tsc), ep1v = f2(ep1 * tsc),
                         ep2v = f2(ep2 * tsc);
            int cur_slot = -1;
            // the self pair (FP64 value / kernel constant, the weight carries the constant)
            const int my_pos = G.tgt + row;
            float self_e = 0.f, self_n = 0.f;
            if (MODE == 0 && rvalid) {
                const double2 sk = a.selfk[my_pos];
                self_e = (float)sk.x * tsc;
                self_n = (float)sk.y * tsc;
            }
            // record: the group's tiles in the store, stage after stage; per
            // MMA step four chunks (hi, lo x east, north) of the group's rows
            // rounded up to 16, each the bytes of the ring's rows
            const int nr16 = (G.nt + 15) & ~15;
            const size_t cb = (size_t)nr16 * 32;
            unsigned char *gtile = (TS == 1 || TS == 3) ? a.ktile + a.ktile_off[gi - J.beg[gk]] : nullptr;
            // item records are read one item ahead, so their latency hides
            // behind the current item's stages
            TcItem nxt = a.items[G.ib];
            for (int k = 0; k < ni; ++k) {
                const TcItem it = nxt;
                if (k + 1 < ni) nxt = a.items[G.ib + k + 1];
                const int kind = it.kind & 3;
                const int nst = (it.cnt + SK - 1) / SK;
                // an item the kernel-tile store holds (one in tile_every)
                const bool stored = (TS == 1 || TS == 3) && k % a.tile_every == a.tile_every - 1;
                if (TS == 3 && stored) {
                    // replay: warp 0 copies the stage's chunks (MMA step q / 4, hi / lo,
                    // east / north) into the ring slot once the MMAs that last read it
                    // are done; its arrival carries the bytes
                    const uint32_t slot = st % KS, kpar = ((st / KS) - 1) & 1;
                    const int nq = 4 * (((min(SK, it.cnt) + 7) / 8 + 1) / 2);
                    if (st >= (uint32_t)KS) wait_bounded(&sm.kempty[slot], kpar, abort, err);
                    if (warp == 0) {
                        if (lane == 0) dev::mbar_expect_tx(&sm.kfull[slot], (uint32_t)(nq * cb));
                        __syncwarp();
                        if (lane < nq && !*abort)
                            dev::bulk_g2s_hint(reinterpret_cast<unsigned char *>(sm.Kt(slot, lane >> 2, (lane >> 1) & 1)) +
                                                   (lane & 1) * (kTcRows / 8) * 256,
                                               gtile + (size_t)lane * cb, (uint32_t)cb, &sm.kfull[slot], dev::l2_evict_first());
                    } else if (lane == 0) {
                        mbar_arrive(&sm.kfull[slot]);
                    }
                    __syncwarp();
                    gtile += (size_t)nq * cb;
                    ++st;
                    continue;
                }
                if (MODE == 0 && kind == 2 && it.off != cur_slot) {
                    // BLI bases of every target row in the new slot: thread
                    // t < 128 the xi basis of target t, thread 128 + t its
                    // eta basis
                    cur_slot = it.off;
                    producers_sync();
                    const int brow = tid & (kTcRows - 1);
                    if (brow < G.nt) {
                        const double2 e = a.xieta[G.tgt + brow];
                        const double *nodes = a.tgt_nodes + (size_t)it.off * 2 * n;
                        if (tid < kTcRows) down_basis(e.x, nodes, n, sm.fx[brow]);
                        else down_basis(e.y, nodes + n, n, sm.fe[brow]);
                    }
                    producers_sync();
                }
                const float2 tx2 = f2(tl0 - it.dx), ty2 = f2(tl1 - it.dy), tz2 = f2(tl2 - it.dz);
                // only the item whose sources are the group's own points holds
                // self pairs (one test per item, the same for every thread)
                const bool self_item = MODE == 0 && kind == 0 && it.off < G.tgt + G.nt && G.tgt < it.off + it.cnt;
                for (int j = 0; j < nst; ++j, ++st) {
                    const uint32_t slot = st % KS, kpar = ((st / KS) - 1) & 1;
                    const int nks = (min(SK, it.cnt - SK * j) + 7) >> 3;   // k-steps of this stage
                    // the MMAs that last read this slot must be done before
                    // the first store into it
                    bool slot_free = st < (uint32_t)KS;
                    // the stage's upward factors (MODE 2) or source
                    // coordinates (point and proxy sources) are in aux
                    if ((MODE == 2 || kind != 2) && active && kfirst < nks)
                        wait_bounded(&sm.wfull[st % WS], (st / WS) & 1, abort, err);
                    const float4 *crd = reinterpret_cast<const float4 *>(sm.aux[st % WS]);
                    // one task: the kernel-tile values of k-step kk for this
                    // lane's row (east / north, or the three Cartesian
                    // components in the proxy pass)
                    auto values = [&](int kk, float (&ve)[8], float (&vn)[8], float (&vz)[8]) {
                            if (MODE == 2) {
                                // upward: the BLI basis of proxy (i, j) at the 8 points,
                                // F_i(xi) G_j(eta) from the per-point factors
                                const float *Fb = sm.aux[st % WS] + 16 * n * kk;
                                const float4 f0 = *reinterpret_cast<const float4 *>(Fb + 8 * up_i);
                                const float4 f1 = *reinterpret_cast<const float4 *>(Fb + 8 * up_i + 4);
                                const float4 g0 = *reinterpret_cast<const float4 *>(Fb + 8 * n + 8 * up_j);
                                const float4 g1 = *reinterpret_cast<const float4 *>(Fb + 8 * n + 8 * up_j + 4);
                                ve[0] = f0.x * g0.x; ve[1] = f0.y * g0.y; ve[2] = f0.z * g0.z; ve[3] = f0.w * g0.w;
                                ve[4] = f1.x * g1.x; ve[5] = f1.y * g1.y; ve[6] = f1.z * g1.z; ve[7] = f1.w * g1.w;
#pragma unroll
                                for (int c = 0; c < 8; ++c) vn[c] = 0.f;
                            } else if (MODE == 0 && kind == 2) {
                                // DOWN: BLI basis of the target x its unit vector's
                                // component of the Cartesian row
                                const int *km0 = sm.kmap + it.row0 + SK * j + 8 * kk;
                                const float *fxr = sm.fx[row], *fer = sm.fe[row];
#pragma unroll
                                for (int c = 0; c < 8; ++c) {
                                    const int km = km0[c];
                                    const float b = fxr[km & 255] * fer[(km >> 8) & 255];
                                    const int comp = km >> 16;
                                    ve[c] = comp == 2 ? 0.f : b * (comp == 0 ? el0 : el1);
                                    vn[c] = b * (comp == 0 ? ep0 : (comp == 1 ? ep1 : ep2));
                                }
                            } else {
                                // PP / PC: kernel value x projected displacement,
                                // two columns per packed instruction
                                // this k-step's x[8] y[8] z[8] (same address in every
                                // lane: shared-memory broadcasts)
                                float4 pre[6];
#pragma unroll
                                for (int i = 0; i < 6; ++i) pre[i] = crd[6 * kk + i];
#pragma unroll
                                for (int c2 = 0; c2 < 4; ++c2) {
                                    // pre[0..1] = x[8], pre[2..3] = y[8], pre[4..5] = z[8]
                                    const float4 X = pre[c2 >> 1], Y = pre[2 + (c2 >> 1)], Z = pre[4 + (c2 >> 1)];
                                    const float2 dx = sub2((c2 & 1) ? make_float2(X.z, X.w) : make_float2(X.x, X.y), tx2);
                                    const float2 dy = sub2((c2 & 1) ? make_float2(Y.z, Y.w) : make_float2(Y.x, Y.y), ty2);
                                    const float2 dz = sub2((c2 & 1) ? make_float2(Z.z, Z.w) : make_float2(Z.x, Z.y), tz2);
                                    // + 1e-20: mp = 0 only for a source on the target itself (or
                                    // a repeated point), and the floor keeps the value finite;
                                    // chords of neighbours (mp >= 1e-12) do not see it
                                    const float2 mp = __ffma2_rn(dz, dz, __ffma2_rn(dy, dy, __ffma2_rn(dx, dx, f2(1e-20f))));
                                    const float2 r = make_float2(rsqrt_approx(mp.x), rsqrt_approx(mp.y));
                                    const float2 w = __fadd2_rn(__fmul2_rn(mp, r), f2(2.f));
                                    const float2 u = make_float2(rcp_approx(w.x), rcp_approx(w.y));
                                    const float2 inner = __ffma2_rn(f2(kC1F), r, __ffma2_rn(f2(kTwoC2F), u, f2(-kTwoC2F)));
                                    const float2 v = __fmul2_rn(inner, __fmul2_rn(r, r));
                                    if (MODE == 0) {
                                        const float2 pe = __ffma2_rn(el1v, dy, __fmul2_rn(el0v, dx));
                                        const float2 pn = __ffma2_rn(ep2v, dz, __ffma2_rn(ep1v, dy, __fmul2_rn(ep0v, dx)));
                                        const float2 e2 = __fmul2_rn(v, pe), n2 = __fmul2_rn(v, pn);
                                        ve[2 * c2] = e2.x;
                                        ve[2 * c2 + 1] = e2.y;
                                        vn[2 * c2] = n2.x;
                                        vn[2 * c2 + 1] = n2.y;
                                    } else {
                                        // proxy targets: the Cartesian vector val (s - x)
                                        const float2 x2 = __fmul2_rn(v, dx), y2 = __fmul2_rn(v, dy), z2 = __fmul2_rn(v, dz);
                                        ve[2 * c2] = x2.x;
                                        ve[2 * c2 + 1] = x2.y;
                                        vn[2 * c2] = y2.x;
                                        vn[2 * c2 + 1] = y2.y;
                                        vz[2 * c2] = z2.x;
                                        vz[2 * c2 + 1] = z2.y;
                                    }
                                }
                                // the target itself among these 8 sources: the self pair
                                if (self_item) {
                                    const int cs = my_pos - (it.off + SK * j + 8 * kk);
                                    if ((unsigned)cs < 8u) {
#pragma unroll
                                        for (int c = 0; c < 8; ++c)
                                            if (c == cs) { ve[c] = self_e; vn[c] = self_n; }
                                    }
                                }
                            }
                    };
                    // its TF32 hi + lo split, stored into the kernel tile
                    auto store = [&](int kk, const float (&ve)[8], const float (&vn)[8], const float (&vz)[8]) {
                            if constexpr (F16) {
                                // FP16 hi + lo: unit kk is K half kk & 1 of MMA step kk / 2,
                                // the row's 8 values one 16-byte core-matrix row
                                char *th = reinterpret_cast<char *>(sm.Kt(slot, kk >> 1, 0));
                                char *tlo = reinterpret_cast<char *>(sm.Kt(slot, kk >> 1, 1));
                                const int hb = 128 * (kk & 1);
                                uint4 eh, el, nh, nl;
                                split_f16x2(ve[0], ve[1], eh.x, el.x);
                                split_f16x2(ve[2], ve[3], eh.y, el.y);
                                split_f16x2(ve[4], ve[5], eh.z, el.z);
                                split_f16x2(ve[6], ve[7], eh.w, el.w);
                                split_f16x2(vn[0], vn[1], nh.x, nl.x);
                                split_f16x2(vn[2], vn[3], nh.y, nl.y);
                                split_f16x2(vn[4], vn[5], nh.z, nl.z);
                                split_f16x2(vn[6], vn[7], nh.w, nl.w);
                                *reinterpret_cast<uint4 *>(th + oe16 + hb) = eh;
                                *reinterpret_cast<uint4 *>(tlo + oe16 + hb) = el;
                                *reinterpret_cast<uint4 *>(th + on16 + hb) = nh;
                                *reinterpret_cast<uint4 *>(tlo + on16 + hb) = nl;
                                if (TS == 1 && stored && row < nr16) {
                                    unsigned char *g = gtile + (size_t)(kk >> 1) * 4 * cb + oe16 + hb;
                                    *reinterpret_cast<uint4 *>(g) = eh;
                                    *reinterpret_cast<uint4 *>(g + cb) = nh;
                                    *reinterpret_cast<uint4 *>(g + 2 * cb) = el;
                                    *reinterpret_cast<uint4 *>(g + 3 * cb) = nl;
                                }
                                return;
                            }
                            // TF32 hi + lo (the tensor cores read lo's top 11 bits)
                            float *th = sm.Kt(slot, kk, 0), *tlo = sm.Kt(slot, kk, 1);
#pragma unroll
                            for (int hh = 0; hh < 2; ++hh) {
                                const float4 eh = make_float4(tf32_hi(ve[4 * hh]), tf32_hi(ve[4 * hh + 1]),
                                                              tf32_hi(ve[4 * hh + 2]), tf32_hi(ve[4 * hh + 3]));
                                const float4 nh = make_float4(tf32_hi(vn[4 * hh]), tf32_hi(vn[4 * hh + 1]),
                                                              tf32_hi(vn[4 * hh + 2]), tf32_hi(vn[4 * hh + 3]));
                                const float2 el01 = sub2(make_float2(ve[4 * hh], ve[4 * hh + 1]), make_float2(eh.x, eh.y));
                                const float2 el23 = sub2(make_float2(ve[4 * hh + 2], ve[4 * hh + 3]), make_float2(eh.z, eh.w));
                                const float2 nl01 = sub2(make_float2(vn[4 * hh], vn[4 * hh + 1]), make_float2(nh.x, nh.y));
                                const float2 nl23 = sub2(make_float2(vn[4 * hh + 2], vn[4 * hh + 3]), make_float2(nh.z, nh.w));
                                if (row_in_tile) {
                                    *reinterpret_cast<float4 *>(th + oe + 32 * hh) = eh;
                                    *reinterpret_cast<float4 *>(tlo + oe + 32 * hh) = make_float4(el01.x, el01.y, el23.x, el23.y);
                                    if (MODE != 2) {
                                        *reinterpret_cast<float4 *>(th + on + 32 * hh) = nh;
                                        *reinterpret_cast<float4 *>(tlo + on + 32 * hh) = make_float4(nl01.x, nl01.y, nl23.x, nl23.y);
                                    }
                                }
                                if (MODE == 1) {
                                    const float4 zh = make_float4(tf32_hi(vz[4 * hh]), tf32_hi(vz[4 * hh + 1]),
                                                                  tf32_hi(vz[4 * hh + 2]), tf32_hi(vz[4 * hh + 3]));
                                    const float2 zl01 = sub2(make_float2(vz[4 * hh], vz[4 * hh + 1]), make_float2(zh.x, zh.y));
                                    const float2 zl23 = sub2(make_float2(vz[4 * hh + 2], vz[4 * hh + 3]), make_float2(zh.z, zh.w));
                                    if (row_in_tile) {
                                        *reinterpret_cast<float4 *>(th + oz + 32 * hh) = zh;
                                        *reinterpret_cast<float4 *>(tlo + oz + 32 * hh) = make_float4(zl01.x, zl01.y, zl23.x, zl23.y);
                                    }
                                }
                            }
                    };
                    // FP16: an odd last unit's partner in its 16-source MMA
                    // step is written as zeros
                    const int nut = F16 ? ((nks + 1) & ~1) : nks;
                    auto compute = [&](int k, float (&ve)[8], float (&vn)[8], float (&vz)[8]) {
                        if (!F16 || k < nks) {
                            values(k, ve, vn, vz);   // FP16: kernel values come scaled
                        } else {
#pragma unroll
                            for (int c = 0; c < 8; ++c) ve[c] = vn[c] = vz[c] = 0.f;
                        }
                    };
                    // The proxy pass takes two tasks at a time (their values are
                    // independent, so the second's arithmetic fills the first's
                    // latencies; measured 5 % on that pass).  The leaf pass gains
                    // nothing from it and keeps its registers.
                    constexpr int kPair = MODE == 1 ? 2 : 1;
#pragma unroll 1
                    for (int kk = kfirst; active && kk < nut; kk += kPair * kstride) {
                        float ve[8], vn[8], vz[8], ve2[8], vn2[8], vz2[8];
                        const int k2 = kk + kstride;
                        const bool two = kPair == 2 && k2 < nut;
                        compute(kk, ve, vn, vz);
                        if (kPair == 2) compute(two ? k2 : kk, ve2, vn2, vz2);
                        if (!slot_free) {
                            wait_bounded(&sm.kempty[slot], kpar, abort, err);
                            slot_free = true;
                        }
                        store(kk, ve, vn, vz);
                        if (two) store(k2, ve2, vn2, vz2);
                    }
                    if (!slot_free) {
                        // warps that wrote nothing: their arrival must still
                        // not run a ring phase ahead of the MMAs
                        wait_bounded(&sm.kempty[slot], kpar, abort, err);
                    } else {
                        dev::fence_proxy_async();
                    }
                    __syncwarp();
                    if (lane == 0) mbar_arrive(&sm.kfull[slot]);
                    if (TS == 1 && stored) gtile += (size_t)4 * ((nks + 1) >> 1) * cb;
                }
            }
        }
    } else if (warp == kMmaWarp) {
        // ============================================================ MMA issue
        uint32_t cc = 0;           // chains started
        bool chain_open = false;
        for (int gi = blockIdx.x; gi < total; gi += gridDim.x) {
            const int gk = grid_of(gi);
            const TcArgs &a = J.g[gk];
            const MixGroup G = a.groups[gi - J.beg[gk]];
            ItemWindow w;
            w.start(a.items, G.ib, G.ie, lane);
            // replay: bytes of one packed tile (east rows, then north rows)
            const uint32_t ptile = 2u * (uint32_t)((G.nt + 15) & ~15) * 32u;
            for (int k = G.ib; k < G.ie; ++k) {
                const TcItem it = w.get(k, lane);
                const int nst = (it.cnt + SK - 1) / SK;
                for (int j = 0; j < nst; ++j, ++st) {
                    const uint32_t slot = st % KS, jb = st % WS;
                    // replay: the stage's one barrier covers its weight and kernel tiles
                    if (TS != 2) wait_bounded(&sm.wfull[jb], (st / WS) & 1, abort, err);
                    wait_bounded(&sm.kfull[slot], (st / KS) & 1, abort, err);
                    // a new chain overwrites the accumulator, whose last chain
                    // (cc - 1) the fold warps must have read
                    if (!chain_open && cc >= 1) wait_bounded(&sm.accfree, (cc - 1) & 1, abort, err);
                    tc_fence_after();
                    if (lane == 0) {
                        if (!*abort) {
                            const int nks = (min(SK, it.cnt - SK * j) + 7) >> 3;
                            if constexpr (TS == 2) {
                                // packed tiles of MMA step s: hi at (2s) ptile, lo at (2s + 1) ptile
                                const unsigned char *tb = sm.ring + sm.toff[slot];
                                const unsigned char *wb = sm.ring + TcSmem<TS>::kKtBytes + sm.woff[slot];
                                for (int s = 0; 2 * s < nks; ++s) {
                                    const uint64_t aw = smem_desc_w16(wb + s * 2 * kW16UnitBytes);
                                    const uint64_t bh = smem_desc(tb + 2 * s * ptile), bl = smem_desc(tb + (2 * s + 1) * ptile);
                                    mma_ss_f16(tmem, aw, bh, (chain_open || s > 0) ? 1u : 0u);
                                    mma_ss_f16(tmem, aw, bl, 1u);
                                }
                            } else if constexpr (F16) {
                                // 16 sources per MMA: weight units 2s and 2s + 1
                                for (int s = 0; 2 * s < nks; ++s) {
                                    const uint64_t aw = smem_desc_w16(sm.Wt(jb) + s * (2 * kW16UnitBytes / 4));
                                    const uint64_t bh = smem_desc(sm.Kt(slot, s, 0)), bl = smem_desc(sm.Kt(slot, s, 1));
                                    mma_ss_f16(tmem, aw, bh, (chain_open || s > 0) ? 1u : 0u);
                                    mma_ss_f16(tmem, aw, bl, 1u);
                                }
                            } else {
                                for (int s = 0; s < nks; ++s) {
                                    const uint64_t aw = smem_desc(sm.Wt(jb) + s * kWStepFloats);
                                    const uint64_t bh = smem_desc(sm.Kt(slot, s, 0)), bl = smem_desc(sm.Kt(slot, s, 1));
                                    mma_ss(tmem, aw, bh, (chain_open || s > 0) ? 1u : 0u);
                                    mma_ss(tmem, aw, bl, 1u);
                                }
                            }
                        }
                        mma_commit(&sm.kempty[slot]);
                        if (TS != 2) mma_commit(&sm.wempty[jb]);
                    }
                    chain_open = true;
                    __syncwarp();
                }
                if (it.kind & kTcFlush) {
                    if (lane == 0) mma_commit(&sm.accfull);
                    __syncwarp();
                    chain_open = false;
                    ++cc;
                }
            }
        }
        // every MMA issued by this CTA completes before tensor memory is freed
        if (lane == 0) {
            mma_commit(&sm.fin);
            wait_drain(&sm.fin, 0, err);
        }
        __syncwarp();
    } else if (warp == kLoadWarp) {
        // ============================================================ loads
        // replay: ring heads, the oldest stage still in flight
        uint32_t thead = 0, whead = 0, oldest = 0;
        for (int gi = blockIdx.x; gi < total; gi += gridDim.x) {
            const int gk = grid_of(gi);
            const TcArgs &a = J.g[gk];
            const MixGroup G = a.groups[gi - J.beg[gk]];
            ItemWindow w;
            w.start(a.items, G.ib, G.ie, lane);
            // replay: the group's recorded tiles, stage after stage (per MMA
            // step, hi then lo, each the group's east rows then its north
            // rows, rounded up to 16 rows of 32 bytes)
            const unsigned char *tsrc = TS == 2 ? a.ktile + a.ktile_off[gi - J.beg[gk]] : nullptr;
            const uint32_t cb = (uint32_t)((G.nt + 15) & ~15) * 32u;
            for (int k = G.ib; k < G.ie; ++k) {
                const TcItem it = w.get(k, lane);
                if (k + 1 < G.ie) {
                    const TcItem nxt = w.get(k + 1, lane);
                    // the next item's weight tiles (and source coordinates)
                    // into L2 while this item's stages run
                    if (lane == 0 && MODE != 2) {
                        const uint32_t nks = (uint32_t)(nxt.cnt + 7) >> 3;
                        if (F16)
                            prefetch_l2(static_cast<const char *>(a.bstore16) + (size_t)nxt.kb * kW16UnitBytes,
                                        ((nks + 1) & ~1u) * kW16UnitBytes);
                        else
                            prefetch_l2(a.bstore + (size_t)nxt.kb * kWStepFloats, nks * kWStepFloats * 4u);
                        if (TS != 2 && (nxt.kind & 3) != 2) prefetch_l2(a.sxyz + (size_t)nxt.kb * 24, nks * 96u);
                    }
                }
                const int nst = (it.cnt + SK - 1) / SK;
                for (int j = 0; j < nst; ++j, ++st) {
                    const int nks = (min(SK, it.cnt - SK * j) + 7) >> 3;
                    if constexpr (TS == 2) {
                        // the stage's kernel tiles and weight tiles, each one
                        // bulk copy into its ring (from the start of a ring
                        // when they do not fit before its end), once the stage
                        // slot and both ranges are free: stages retire in order
                        const uint32_t nsteps = (uint32_t)(nks + 1) >> 1;
                        const uint32_t sb = nsteps * 4u * cb, wb = nsteps * 2u * kW16UnitBytes;
                        const uint32_t tpos = thead + sb > (uint32_t)kTRingBytes ? 0u : thead;
                        const uint32_t wpos = whead + wb > (uint32_t)kWRingBytes ? 0u : whead;
                        while (oldest < st) {
                            bool clash = st - oldest >= (uint32_t)KS;
                            for (uint32_t x = oldest; !clash && x < st; ++x) {
                                const uint32_t xs = x % KS;
                                const uint32_t t0 = sm.toff[xs], t1 = t0 + sm.tlen[xs];
                                const uint32_t w0 = sm.woff[xs], w1 = w0 + sm.wlen[xs];
                                clash = (tpos < t1 && t0 < tpos + sb) || (wpos < w1 && w0 < wpos + wb);
                            }
                            if (!clash) break;
                            wait_bounded(&sm.kempty[oldest % KS], (oldest / KS) & 1, abort, err);
                            ++oldest;
                        }
                        const uint32_t slot = st % KS;
                        if (lane == 0) {
                            sm.toff[slot] = tpos;
                            sm.tlen[slot] = sb;
                            sm.woff[slot] = wpos;
                            sm.wlen[slot] = wb;
                            // the offsets are written before the arrival the MMA warp waits on
                            dev::mbar_expect_tx(&sm.kfull[slot], sb + wb);
                            if (!*abort) {
                                // the tiles are read once per solve: they leave L2 first, to
                                // the weight tiles, which other groups read again
                                dev::bulk_g2s_hint(sm.ring + tpos, tsrc, sb, &sm.kfull[slot], dev::l2_evict_first());
                                dev::bulk_g2s_hint(sm.ring + TcSmem<TS>::kKtBytes + wpos,
                                                   static_cast<const char *>(a.bstore16) + (size_t)(it.kb + SU * j) * kW16UnitBytes,
                                                   wb, &sm.kfull[slot], dev::l2_evict_last());
                            }
                        }
                        __syncwarp();
                        tsrc += sb;
                        thead = tpos + sb;
                        whead = wpos + wb;
                    } else {
                        const uint32_t jb = st % WS, ub = st / WS;
                        if (ub > 0) wait_bounded(&sm.wempty[jb], (ub - 1) & 1, abort, err);
                        if (lane == 0) {
                            // FP16: whole 16-source MMA steps (the store has a spare unit at its end)
                            const uint32_t wbytes = F16 ? (uint32_t)((nks + 1) & ~1) * kW16UnitBytes
                                                        : (uint32_t)nks * kWStepFloats * 4;
                            // with the weights: the stage's BLI factors (upward) or
                            // its point / proxy sources' coordinates (24 floats per
                            // k-step; DOWN rows need none)
                            const uint32_t lbytes = MODE == 2 ? (uint32_t)nks * 64 * n
                                                    : (it.kind & 3) != 2 ? (uint32_t)nks * 96u : 0u;
                            dev::mbar_expect_tx(&sm.wfull[jb], wbytes + lbytes);
                            if (!*abort) {
                                if (lbytes)
                                    dev::bulk_g2s(sm.aux[jb],
                                                  MODE == 2 ? (const void *)(a.basis + (size_t)(it.row0 + SU * j) * 16 * n)
                                                            : (const void *)(a.sxyz + (size_t)(it.kb + SU * j) * 24),
                                                  lbytes, &sm.wfull[jb]);
                                const void *wsrc =
                                    F16 ? static_cast<const void *>(static_cast<const char *>(a.bstore16) +
                                                                    (size_t)(it.kb + SU * j) * kW16UnitBytes)
                                        : static_cast<const void *>(a.bstore + (size_t)(it.kb + SU * j) * kWStepFloats);
                                dev::bulk_g2s(sm.Wt(jb), wsrc, wbytes, &sm.wfull[jb]);
                            }
                        }
                        __syncwarp();
                    }
                }
            }
        }
        // no bulk copy may still be landing when the CTA exits
        if (TS == 2 && lane == 0)
            for (uint32_t x = oldest; x < st; ++x) wait_drain(&sm.kfull[x % KS], (x / KS) & 1, err);
        if (TS != 2 && lane == 0)
            for (uint32_t j = 0; j < (uint32_t)WS && j < st; ++j) {
                const uint32_t uses = (st - 1 - j) / WS + 1;
                wait_drain(&sm.wfull[j], (uses - 1) & 1, err);
            }
        __syncwarp();
    }
    else {
        // ============================================================ folds
        // (replay: warps 0-7 and 10-13, fold part 0, 1 or 2 of their lane
        // quarter warp % 4; otherwise warps 10-13)
        const int q = warp & 3;
        const uint32_t tq = tmem + ((uint32_t)(32 * q) << 16);
        const int part_i = TS == 2 ? (warp < 4 ? 0 : warp < kProdWarps ? 1 : 2) : 0, nparts = TS == 2 ? 3 : 1;
        uint32_t cc = 0;   // chains folded
        for (int gi = blockIdx.x; gi < total; gi += gridDim.x) {
            const int gk = grid_of(gi);
            const TcArgs &a = J.g[gk];
            const MixGroup G = a.groups[gi - J.beg[gk]];
            if (TS == 2 && G.ib == G.ie) {
                // a group without sources: the self pairs, by warps 0-7
                if (tid < G.nt && !*abort) self_only(a, G, tid);
                continue;
            }
            bool first = true;
            const int half = TS == 2 ? (G.nt + 15) & ~15 : 128;   // columns per component
            ItemWindow w;
            w.start(a.items, G.ib, G.ie, lane);
            for (int k = G.ib; k < G.ie; ++k) {
                const int kind = w.kind(k, lane);
                if (!(kind & kTcFlush)) continue;
                wait_bounded(&sm.accfull, cc & 1, abort, err);
                tc_fence_after();
                // FP16: the chain's weight rows are the fields' source weights
                // (scaled per field) against scaled kernel columns, or their
                // potentials (scaled per field) against unscaled DOWN columns
                const bool down_chain = (kind & 3) == 2;
                const float fsc = F16 ? 1.f / f16_scale(__uint_as_float(a.fmax[(down_chain ? kF : 0) + 16 * q + (lane & 15)]))
                                      : 1.f;
                const bool end = k == G.ie - 1;
                fold_chain<MODE>(tq, lane, end, first, G.tgt, G.nt, F16, fsc, down_chain, a.tscale, half, part_i,
                                 nparts);
                tc_fence_before();
                __syncwarp();
                if (lane == 0) mbar_arrive(&sm.accfree);
                // the next group's first chain may run into the accumulator meanwhile
                if (end)
                    emit_sums<MODE>(tq, q, lane, G.tgt, G.nt, a.perm, a.out_x, a.out_y, a.ld_out, a.f0, a.nf,
                                    *abort != 0,
                                    MODE == 1   ? a.partial + ((size_t)G.out * P + G.row0) * 3 * kF
                                    : MODE == 2 ? a.partial + ((size_t)G.out * P + G.row0) * kF
                                                : nullptr,
                                    F16, a.tinv, half, part_i, nparts);
                first = false;
                ++cc;
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

// Split weight store (k-steps [k0, k1) of it, with bsrc and bstore offset
// by the caller): per k-step of 8 store rows, the 64-field rows as one
// 128-row TF32 tile (field f's hi part at row wrow(f, 0), lo part at
// wrow(f, 1)) in the canonical no-swizzle K-major layout.  One thread per
// (k-step, field).
__global__ void split_store_kernel(const int32_t *__restrict__ bsrc, int64_t nk, const float *__restrict__ wF,
                                   const float *__restrict__ phiF, float *__restrict__ bstore) {
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= nk * kF) return;
    const int64_t ks = t / kF;
    const int f = (int)(t % kF);
    float hi[8], lo[8];
#pragma unroll
    for (int r = 0; r < 8; ++r) {
        const int32_t s = bsrc[ks * 8 + r];
        const float v = s >= 0 ? wF[(size_t)s * kF + f] : (s <= -2 ? phiF[(size_t)(-2 - s) * kF + f] : 0.f);
        hi[r] = tf32_hi(v);
        lo[r] = tf32_hi(v - hi[r]);
    }
    float *base = bstore + ks * kWStepFloats;
    const int oh = canon(wrow(f, 0), 0) >> 2, ol = canon(wrow(f, 1), 0) >> 2;
    *reinterpret_cast<float4 *>(base + oh) = make_float4(hi[0], hi[1], hi[2], hi[3]);
    *reinterpret_cast<float4 *>(base + oh + 32) = make_float4(hi[4], hi[5], hi[6], hi[7]);
    *reinterpret_cast<float4 *>(base + ol) = make_float4(lo[0], lo[1], lo[2], lo[3]);
    *reinterpret_cast<float4 *>(base + ol + 32) = make_float4(lo[4], lo[5], lo[6], lo[7]);
}

// FP16 leaf pass: per field the largest |value| of nrows rows of 64 fields
// (one float4 of 4 fields per thread and row, contiguous reads), merged into
// out[f] as float bits with atomicMax (non-negative floats order as their
// bits).
__global__ void field_max_kernel(const float4 *__restrict__ x, int64_t nrows, unsigned *__restrict__ out) {
    __shared__ float part[16][kF];
    const int c4 = threadIdx.x & 15;
    float m0 = 0.f, m1 = 0.f, m2 = 0.f, m3 = 0.f;
    for (int64_t r = (int64_t)blockIdx.x * 16 + (threadIdx.x >> 4); r < nrows; r += (int64_t)gridDim.x * 16) {
        const float4 v = x[r * 16 + c4];
        m0 = fmaxf(m0, fabsf(v.x));
        m1 = fmaxf(m1, fabsf(v.y));
        m2 = fmaxf(m2, fabsf(v.z));
        m3 = fmaxf(m3, fabsf(v.w));
    }
    part[threadIdx.x >> 4][4 * c4] = m0;
    part[threadIdx.x >> 4][4 * c4 + 1] = m1;
    part[threadIdx.x >> 4][4 * c4 + 2] = m2;
    part[threadIdx.x >> 4][4 * c4 + 3] = m3;
    __syncthreads();
    if (threadIdx.x < kF) {
        float m = 0.f;
        for (int i = 0; i < 16; ++i) m = fmaxf(m, part[i][threadIdx.x]);
        atomicMax(out + threadIdx.x, __float_as_uint(m));
    }
}

// FP16 hi/lo weight store: per unit of 8 store rows, the 64-field rows as
// one 128-row FP16 tile (field f's hi part at row wrow(f, 0), lo at
// wrow(f, 1); row m at byte (m / 8) 128 + (m % 8) 16, 8 halves), source
// weights scaled by their field's power of two, potentials by theirs.  One
// thread per (unit, 4 fields): float4 row loads, 64-byte row-group stores.
__global__ void split_store16_kernel(const int32_t *__restrict__ bsrc, int64_t nu, const float *__restrict__ wF,
                                     const float *__restrict__ phiF, const unsigned *__restrict__ fmax,
                                     unsigned char *__restrict__ out) {
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= nu * (kF / 4)) return;
    const int64_t u = t / (kF / 4);
    const int f0 = 4 * (int)(t % (kF / 4));
    float sw[4], sp[4];
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        sw[i] = f16_scale(__uint_as_float(fmax[f0 + i]));
        sp[i] = f16_scale(__uint_as_float(fmax[kF + f0 + i]));
    }
    float v[4][8];   // [field][row]
#pragma unroll
    for (int r = 0; r < 8; ++r) {
        const int32_t s = bsrc[u * 8 + r];
        float4 x = make_float4(0.f, 0.f, 0.f, 0.f);
        const float *sc = sw;
        if (s >= 0) {
            x = *reinterpret_cast<const float4 *>(wF + (size_t)s * kF + f0);
        } else if (s <= -2) {
            x = *reinterpret_cast<const float4 *>(phiF + (size_t)(-2 - s) * kF + f0);
            sc = sp;
        }
        v[0][r] = x.x * sc[0];
        v[1][r] = x.y * sc[1];
        v[2][r] = x.z * sc[2];
        v[3][r] = x.w * sc[3];
    }
    unsigned char *base = out + u * kW16UnitBytes;
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        uint4 hi, lo;
        split_f16x2(v[i][0], v[i][1], hi.x, lo.x);
        split_f16x2(v[i][2], v[i][3], hi.y, lo.y);
        split_f16x2(v[i][4], v[i][5], hi.z, lo.z);
        split_f16x2(v[i][6], v[i][7], hi.w, lo.w);
        const int mh = wrow(f0 + i, 0), ml = wrow(f0 + i, 1);
        *reinterpret_cast<uint4 *>(base + (mh >> 3) * 128 + (mh & 7) * 16) = hi;
        *reinterpret_cast<uint4 *>(base + (ml >> 3) * 128 + (ml & 7) * 16) = lo;
    }
}

// FP16 leaf pass: per target the power of two that takes its largest kernel
// value (east or north, over its PP and PC sources, with the leaf pass's own
// FP32 arithmetic, and its self pair) to at most 2^12, and the inverse.  One
// block per leaf group, thread t its target t.  Once per plan.
__global__ void target_scales_kernel(const TcArgs a, float *__restrict__ tscale, float *__restrict__ tinv) {
    const MixGroup G = a.groups[blockIdx.x];
    const int row = threadIdx.x;
    if (row >= G.nt) return;
    const double4 c = a.tgt[G.tgt + row];
    const float tl0 = (float)(c.x - G.cx), tl1 = (float)(c.y - G.cy), tl2 = (float)(c.z - G.cz);
    float el0 = 0.f, el1 = 0.f, ep0 = 0.f, ep1 = 0.f, ep2 = 0.f;
    if ((fabs(c.z - 1.0) > 1e-15) && (fabs(c.z + 1.0) > 1e-15)) {
        const double omz = 1.0 - c.z * c.z, inv = 1.0 / sqrt(omz);
        el0 = (float)(-c.y * inv);
        el1 = (float)(c.x * inv);
        ep0 = (float)(-c.z * c.x * inv);
        ep1 = (float)(-c.z * c.y * inv);
        ep2 = (float)(omz * inv);
    }
    const double2 sk = a.selfk[G.tgt + row];
    float m = fmaxf(fabsf((float)sk.x), fabsf((float)sk.y));
    for (int k = G.ib; k < G.ie; ++k) {
        const TcItem it = a.items[k];
        if ((it.kind & 3) == 2) continue;
        const float tx = tl0 - it.dx, ty = tl1 - it.dy, tz = tl2 - it.dz;
        for (int i = 0; i < it.cnt; ++i) {
            const float *u = a.sxyz + (size_t)(it.kb + (i >> 3)) * 24;
            const float dx = u[i & 7] - tx, dy = u[8 + (i & 7)] - ty, dz = u[16 + (i & 7)] - tz;
            const float mp = fmaxf(dz * dz + (dy * dy + dx * dx), 1e-20f);
            const float r = rsqrt_approx(mp);
            const float uu = rcp_approx(mp * r + 2.f);
            const float v = (kC1F * r + (kTwoC2F * uu - kTwoC2F)) * (r * r);
            const float pe = el0 * dx + el1 * dy, pn = ep0 * dx + ep1 * dy + ep2 * dz;
            m = fmaxf(m, fmaxf(fabsf(v * pe), fabsf(v * pn)));
        }
    }
    const float sc = f16_scale(m);
    tscale[G.tgt + row] = sc;
    tinv[G.tgt + row] = 1.f / sc;
}

// Per pool row, the FP32 coordinates relative to the centre of the row's own
// panel (a leaf for points, the slot panel for proxies).  One block per range.
__global__ void source_local_kernel(const double4 *__restrict__ pool, const int2 *__restrict__ ranges,
                                    const double4 *__restrict__ centres, float4 *__restrict__ sloc) {
    const int2 r = ranges[blockIdx.x];
    const double4 c = centres[blockIdx.x];
    for (int p = r.x + threadIdx.x; p < r.y; p += blockDim.x) {
        const double4 s = pool[p];
        sloc[p] = make_float4((float)(s.x - c.x), (float)(s.y - c.y), (float)(s.z - c.z), 0.f);
    }
}

// Source coordinates per k-step of the split store: x[8], y[8], z[8] of its
// rows (a far dummy point for padding rows, which carry zero weights).
__global__ void source_ksteps_kernel(const int32_t *__restrict__ bsrc, int64_t nks, const float4 *__restrict__ sloc,
                                     float *__restrict__ sxyz) {
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= nks * 8) return;
    const int64_t ks = t >> 3;
    const int i = (int)(t & 7);
    const int32_t r = bsrc[t];
    const float4 p = r >= 0 ? sloc[r] : make_float4(4.f, 4.f, 4.f, 0.f);
    sxyz[ks * 24 + i] = p.x;
    sxyz[ks * 24 + 8 + i] = p.y;
    sxyz[ks * 24 + 16 + i] = p.z;
}

// Basis store of the upward pass: per k-step b of an upward item (slot s,
// pool rows first..first+cnt-1), the FP64 BLI factors of its 8 points over the
// slot panel's nodes, rounded to FP32: F[i][8] (xi nodes) then G[j][8] (eta
// nodes); zero for padding rows.  One thread per (k-step, point).
__global__ void basis_store_kernel(const int32_t *__restrict__ bas, int64_t nbk, const double2 *__restrict__ xieta,
                                   const double *__restrict__ src_nodes, int n, float *__restrict__ basis) {
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= nbk * 8) return;
    const int64_t b = t >> 3;
    const int i = (int)(t & 7);
    const int s = bas[3 * b], first = bas[3 * b + 1], cnt = bas[3 * b + 2];
    float *F = basis + b * 16 * n, *G = F + 8 * n;
    if (i >= cnt) {
        for (int k = 0; k < n; ++k) F[8 * k + i] = G[8 * k + i] = 0.f;
        return;
    }
    const double2 e = xieta[first + i];
    const double *nodes = src_nodes + (size_t)s * 2 * n;
    double f[kMaxDegree + 1];
    dev::bli_basis(e.x, nodes, n, f);
    for (int k = 0; k < n; ++k) F[8 * k + i] = (float)f[k];
    dev::bli_basis(e.y, nodes + n, n, f);
    for (int k = 0; k < n; ++k) G[8 * k + i] = (float)f[k];
}

// Per pool point, the self pair of sal_grad_gfunc (fast_sum_module.f90:9-31)
// in FP64 divided by the kernel constant: the leaf epilogue multiplies it by
// the point's FP32 weight row, which carries the constant.
__global__ void self_pair_kernel(const double4 *__restrict__ pool, int n, double2 *__restrict__ selfk) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= n) return;
    const double4 c = pool[p];
    dev::Tgt T;
    dev::tgt_init(T, c.x, c.y, c.z);
    double sx = 0.0, sy = 0.0;
    if (T.live) dev::gref_exact(T, c.x, c.y, c.z, sx, sy);
    selfk[p] = make_double2(sx / dev::kCons, sy / dev::kCons);
}

static_assert(tc_smem_need<0>() <= 227 * 1024 && tc_smem_need<2>() <= 227 * 1024,
              "the leaf kernel's shared memory fits one SM");

// Dynamic shared memory of a launch: above half of the SM's, so one CTA per
// SM, which owns all 512 tensor memory columns.
template <int TS>
static size_t tc_smem_launch() {
    return tc_smem_need<TS>() > 120 * 1024 ? tc_smem_need<TS>() : 120 * 1024;
}
size_t tc_smem_bytes() { return tc_smem_launch<0>(); }

template <int MODE, bool JOINT, bool F16 = false, int TS = 0>
static void launch_tc(const TcJoint &J, int nsm, int cta_groups, int *err, cudaStream_t st) {
    const int total = J.beg[J.ngrids];
    if (total <= 0) return;
    const size_t smem = tc_smem_launch<TS>();
    static std::atomic<unsigned long long> done{0};
    smem_attr_once((const void *)tc_leaf_kernel<MODE, JOINT, F16, TS>, (int)smem, done);
    // every SM busy, but no CTA longer than cta_groups groups: with short
    // CTAs, kernels of other streams (higher-priority grids) get SMs as CTAs
    // retire
    const int per = cta_groups > 0 ? cta_groups : 1;
    int grid = (total + per - 1) / per;
    if (grid < nsm) grid = total < nsm ? total : nsm;
    tc_leaf_kernel<MODE, JOINT, F16, TS><<<grid, kThreads, smem, st>>>(J, err);
}

template <int MODE, bool F16 = false, int TS = 0>
static void launch_tc(const TcArgs &a, int nsm, int cta_groups, int *err, cudaStream_t st) {
    TcJoint J{};
    J.g[0] = a;
    J.ngrids = 1;
    J.beg[0] = 0;
    J.beg[1] = a.ngroups;
    launch_tc<MODE, false, F16, TS>(J, nsm, cta_groups, err, st);
}

void launch_tc_leaf_joint(const TcArgs *grids, int ngrids, int nsm, int cta_groups, int *err, cudaStream_t st) {
    TcJoint J{};
    J.ngrids = ngrids;
    J.beg[0] = 0;
    for (int k = 0; k < ngrids; ++k) {
        J.g[k] = grids[k];
        J.beg[k + 1] = J.beg[k] + grids[k].ngroups;
    }
    // the caller checks that all grids use one operand precision
    if (grids[0].bstore16)
        launch_tc<0, true, true>(J, nsm, cta_groups, err, st);
    else
        launch_tc<0, true, false>(J, nsm, cta_groups, err, st);
}

void launch_tc_leaf(const TcArgs &a, int nsm, int cg, int *err, cudaStream_t st, int tiles) {
    if (a.bstore16 && a.ktile && tiles == 1)
        launch_tc<0, true, 1>(a, nsm, cg, err, st);
    else if (a.bstore16 && a.ktile && tiles == 2)
        launch_tc<0, true, 2>(a, nsm, cg, err, st);
    else if (a.bstore16 && a.ktile && tiles == 3)
        launch_tc<0, true, 3>(a, nsm, cg, err, st);
    else if (a.bstore16)
        launch_tc<0, true>(a, nsm, cg, err, st);
    else
        launch_tc<0, false>(a, nsm, cg, err, st);
}
void launch_tc_proxy(const TcArgs &a, int nsm, int cg, int *err, cudaStream_t st) { launch_tc<1>(a, nsm, cg, err, st); }
void launch_tc_upward(const TcArgs &a, int nsm, int cg, int *err, cudaStream_t st) { launch_tc<2>(a, nsm, cg, err, st); }

void launch_split_store(const int32_t *bsrc, int64_t k0, int64_t k1, const float *wF, const float *phiF,
                        float *bstore, cudaStream_t st) {
    const int64_t nk = k1 - k0;
    if (nk <= 0) return;
    const int64_t threads = nk * kF;
    split_store_kernel<<<(unsigned)((threads + 255) / 256), 256, 0, st>>>(bsrc + k0 * 8, nk, wF, phiF,
                                                                          bstore + k0 * kWStepFloats);
}

void launch_field_max(const float *wF, int64_t nw, const float *phiF, int64_t np, unsigned *fmax, cudaStream_t st) {
    if (nw > 0)
        field_max_kernel<<<(unsigned)std::min<int64_t>((nw + 15) / 16, 148 * 16), 256, 0, st>>>(
            reinterpret_cast<const float4 *>(wF), nw, fmax);
    if (np > 0)
        field_max_kernel<<<(unsigned)std::min<int64_t>((np + 15) / 16, 148 * 16), 256, 0, st>>>(
            reinterpret_cast<const float4 *>(phiF), np, fmax + kF);
}

void launch_split_store16(const int32_t *bsrc, int64_t nunits, const float *wF, const float *phiF,
                          const unsigned *fmax, void *bstore16, cudaStream_t st) {
    if (nunits <= 0) return;
    const int64_t threads = nunits * (kF / 4);
    split_store16_kernel<<<(unsigned)((threads + 255) / 256), 256, 0, st>>>(bsrc, nunits, wF, phiF, fmax,
                                                                            static_cast<unsigned char *>(bstore16));
}

void launch_target_scales(const TcArgs &a, float *tscale, float *tinv, cudaStream_t st) {
    if (a.ngroups > 0) target_scales_kernel<<<a.ngroups, kTcRows, 0, st>>>(a, tscale, tinv);
}

void launch_source_local(const double4 *pool, const int2 *ranges, const double4 *centres, int nranges, float4 *sloc,
                         cudaStream_t st) {
    if (nranges > 0) source_local_kernel<<<nranges, 128, 0, st>>>(pool, ranges, centres, sloc);
}

void launch_source_ksteps(const int32_t *bsrc, int64_t nks, const float4 *sloc, float *sxyz, cudaStream_t st) {
    if (nks > 0) source_ksteps_kernel<<<(unsigned)((nks * 8 + 255) / 256), 256, 0, st>>>(bsrc, nks, sloc, sxyz);
}

void launch_basis_store(const int32_t *bas, int64_t nbk, const double2 *xieta, const double *src_nodes, int n,
                        float *basis, cudaStream_t st) {
    if (nbk > 0)
        basis_store_kernel<<<(unsigned)((nbk * 8 + 255) / 256), 256, 0, st>>>(bas, nbk, xieta, src_nodes, n, basis);
}

void launch_self_pair(const double4 *pool, int n, double2 *selfk, cudaStream_t st) {
    if (n > 0) self_pair_kernel<<<(n + 255) / 256, 256, 0, st>>>(pool, n, selfk);
}

}  // namespace mix
}  // namespace sal
