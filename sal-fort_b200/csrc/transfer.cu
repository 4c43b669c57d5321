// Tree transfers of the batched form (64 fields per block).
//
// The proxies of a panel are its N x N Chebyshev nodes (N = d + 1), proxy
// p = i + l N at (xi_i, eta_l).  A parent's degree-d barycentric Lagrange
// basis (bli_module.f90:50-113) restricted to a child is a degree-d
// polynomial in each coordinate, so the child's nodes reproduce it exactly:
//     L^p_j(x) = sum_i L^p_j(xc_i) L^c_i(x).
// Children halve their parent's interval in each coordinate, and the bases
// are invariant under affine maps of the interval, so the matrices
// H_h[j][i] = L^p_j(xc_i) are the same two (lower half h = 0, upper h = 1) for
// every panel.  With A = H of the child's xi half and B = H of its eta half:
//   child-to-parent (upward):  W_p(j, k) += sum_i A[j][i] sum_l B[k][l] W_c(i, l)
//     -- the parent's proxy weights sum_s L^p_j(xi_s) L^p_k(eta_s) w_s from
//     its children's, without revisiting the points;
//   parent-to-child (downward): Phi_c(i, l) (+)= sum_j A[j][i] sum_k B[k][l] Phi_p(j, k)
//     -- the parent's potential interpolant evaluated at the child's nodes,
//     so the child's interpolant reproduces it.
// Both are exact in exact arithmetic.  Each is two 1-D transfers (2 N^3
// multiply-adds per field instead of N^4), in FP32 like the rows they read
// and write (a transfer rounds at the 1e-7 level; FP64 sums made the solve
// 0.35 ms slower at 2.3M cells x 64 fields and were no more accurate against
// the direct sum).  One CTA of 64 N threads per task: thread
// (f = t % 64, r = t / 64) keeps row r of the tile for field f in registers,
// so every shared-memory value it loads feeds N multiply-adds, and the loops
// are unrolled over the compile-time N.
#include <cuda_runtime.h>

#include "kernels.cuh"
#include "mixed.cuh"

namespace sal {
namespace mix {

namespace {
constexpr int kF = 64;

template <int N>
constexpr size_t transfer_smem() {
    // both matrices and two float tiles
    return (2 * N * N + 2 * (size_t)N * N * kF) * sizeof(float);
}
}  // namespace

// Child-to-parent transfer of one tree level.  tasks: 6 per parent (parent
// slot, 4 child slots or -1, the children's halves: bits 2c (xi) and 2c + 1
// (eta) for child c).  H: the two N x N transfer matrices.  w: the weight
// rows of the slots, N^2 rows of 64 fields per slot.
template <int N>
__global__ void __launch_bounds__(64 * N) m2m_kernel(const int32_t *__restrict__ tasks, const double *__restrict__ H,
                                                     float *__restrict__ w) {
    constexpr int P = N * N;
    extern __shared__ __align__(16) float smf[];
    float *Hs = smf, *T = Hs + 2 * P, *Wc = T + (size_t)P * kF;
    const int32_t *tk = tasks + 6 * (size_t)blockIdx.x;
    const int tid = threadIdx.x, f = tid & (kF - 1), r = tid >> 6;
    for (int e = tid; e < 2 * P; e += 64 * N) Hs[e] = (float)H[e];
    float acc[N];   // W_p(j, r), j = 0 .. N-1
#pragma unroll
    for (int j = 0; j < N; ++j) acc[j] = 0.f;
    const int code = tk[5];
    for (int c = 0; c < 4; ++c) {
        const int child = tk[1 + c];
        if (child < 0) continue;
        const float *A = Hs + ((code >> (2 * c)) & 1) * P, *B = Hs + ((code >> (2 * c + 1)) & 1) * P;
        __syncthreads();   // the previous child's tiles are consumed
        const float *src = w + (size_t)child * P * kF;
        for (int e = tid; e < P * kF; e += 64 * N) Wc[e] = src[e];
        __syncthreads();
        // T(r, k) = sum_l B[k][l] W_c(r, l)
        {
            float wv[N];
#pragma unroll
            for (int l = 0; l < N; ++l) wv[l] = Wc[(r + l * N) * kF + f];
#pragma unroll
            for (int k = 0; k < N; ++k) {
                float s = 0.f;
#pragma unroll
                for (int l = 0; l < N; ++l) s = fmaf(B[k * N + l], wv[l], s);
                T[(r + k * N) * kF + f] = s;
            }
        }
        __syncthreads();
        // W_p(j, r) += sum_i A[j][i] T(i, r)
        {
            float tv[N];
#pragma unroll
            for (int i = 0; i < N; ++i) tv[i] = T[(i + r * N) * kF + f];
#pragma unroll
            for (int j = 0; j < N; ++j) {
                float s = 0.f;
#pragma unroll
                for (int i = 0; i < N; ++i) s = fmaf(A[j * N + i], tv[i], s);
                acc[j] += s;
            }
        }
    }
    float *dst = w + (size_t)tk[0] * P * kF;
#pragma unroll
    for (int j = 0; j < N; ++j) dst[(j + r * N) * kF + f] = acc[j];
}

// Parent-to-child transfer of one tree level.  tasks: 4 per child (child
// slot, parent slot, own: 1 adds to the child's own potentials, 0 replaces
// them, the child's halves: bit 0 xi, bit 1 eta).  phi: per slot 3 N^2 rows
// (proxy p, Cartesian component c at row 3p + c) of 64 fields.
template <int N>
__global__ void __launch_bounds__(64 * N) l2l_kernel(const int32_t *__restrict__ tasks, const double *__restrict__ H,
                                                     float *__restrict__ phi) {
    constexpr int P = N * N;
    extern __shared__ __align__(16) float smf[];
    float *Hs = smf, *T = Hs + 2 * P, *Pp = T + (size_t)P * kF;
    const int32_t *tk = tasks + 4 * (size_t)blockIdx.x;
    const int child = tk[0], parent = tk[1], own = tk[2], code = tk[3];
    const int tid = threadIdx.x, f = tid & (kF - 1), r = tid >> 6;
    for (int e = tid; e < 2 * P; e += 64 * N) Hs[e] = (float)H[e];
    const float *A = Hs + (code & 1) * P, *B = Hs + ((code >> 1) & 1) * P;
    const float *src = phi + (size_t)parent * 3 * P * kF;
    float *dst = phi + (size_t)child * 3 * P * kF;
    for (int c = 0; c < 3; ++c) {
        __syncthreads();
        for (int e = tid; e < P * kF; e += 64 * N) Pp[e] = src[((size_t)3 * (e / kF) + c) * kF + (e % kF)];
        __syncthreads();
        // T(r, l) = sum_k B[k][l] Phi_p(r, k)
        {
            float pv[N];
#pragma unroll
            for (int k = 0; k < N; ++k) pv[k] = Pp[(r + k * N) * kF + f];
#pragma unroll
            for (int l = 0; l < N; ++l) {
                float s = 0.f;
#pragma unroll
                for (int k = 0; k < N; ++k) s = fmaf(B[k * N + l], pv[k], s);
                T[(r + l * N) * kF + f] = s;
            }
        }
        __syncthreads();
        // Phi_c(i, r) (+)= sum_j A[j][i] T(j, r)
        {
            float tv[N];
#pragma unroll
            for (int j = 0; j < N; ++j) tv[j] = T[(j + r * N) * kF + f];
#pragma unroll
            for (int i = 0; i < N; ++i) {
                float s = 0.f;
#pragma unroll
                for (int j = 0; j < N; ++j) s = fmaf(A[j * N + i], tv[j], s);
                float *out = dst + ((size_t)3 * (i + r * N) + c) * kF + f;
                *out = own ? *out + s : s;
            }
        }
    }
}

template <int N>
static void launch_m2m_n(const int32_t *tasks, int ntasks, const double *H, float *w, cudaStream_t st) {
    static std::atomic<unsigned long long> done{0};
    smem_attr_once((const void *)m2m_kernel<N>, (int)transfer_smem<N>(), done);
    m2m_kernel<N><<<ntasks, 64 * N, transfer_smem<N>(), st>>>(tasks, H, w);
}

template <int N>
static void launch_l2l_n(const int32_t *tasks, int ntasks, const double *H, float *phi, cudaStream_t st) {
    static std::atomic<unsigned long long> done{0};
    smem_attr_once((const void *)l2l_kernel<N>, (int)transfer_smem<N>(), done);
    l2l_kernel<N><<<ntasks, 64 * N, transfer_smem<N>(), st>>>(tasks, H, phi);
}

// N = d + 1 from 2 to kMaxTreeDegree + 1 (the plan turns the tree passes off
// above that)
#define SAL_TRANSFER_DISPATCH(fn, n, ...)                       \
    switch (n) {                                                \
        case 2: fn<2>(__VA_ARGS__); break;                      \
        case 3: fn<3>(__VA_ARGS__); break;                      \
        case 4: fn<4>(__VA_ARGS__); break;                      \
        case 5: fn<5>(__VA_ARGS__); break;                      \
        case 6: fn<6>(__VA_ARGS__); break;                      \
        case 7: fn<7>(__VA_ARGS__); break;                      \
        case 8: fn<8>(__VA_ARGS__); break;                      \
        case 9: fn<9>(__VA_ARGS__); break;                      \
        case 10: fn<10>(__VA_ARGS__); break;                    \
        case 11: fn<11>(__VA_ARGS__); break;                    \
        default: break;                                         \
    }
static_assert(kMaxTreeDegree + 1 == 11, "the dispatch covers N = 2 .. kMaxTreeDegree + 1");

void launch_m2m(const int32_t *tasks, int ntasks, const double *H, int n, float *w, cudaStream_t st) {
    if (ntasks <= 0) return;
    SAL_TRANSFER_DISPATCH(launch_m2m_n, n, tasks, ntasks, H, w, st)
}

void launch_l2l(const int32_t *tasks, int ntasks, const double *H, int n, float *phi, cudaStream_t st) {
    if (ntasks <= 0) return;
    SAL_TRANSFER_DISPATCH(launch_l2l_n, n, tasks, ntasks, H, phi, st)
}

}  // namespace mix
}  // namespace sal
