// Tree transfers of the batched form (64 fields per block).
//
// The proxies of a panel are its (d+1) x (d+1) Chebyshev nodes, proxy
// p = i + l (d+1) at (xi_i, eta_l).  A parent's degree-d barycentric
// Lagrange basis (bli_module.f90:50-113) restricted to a child is a degree-d
// polynomial in each coordinate, so the child's nodes reproduce it exactly:
//     L^p_j(x) = sum_i L^p_j(xc_i) L^c_i(x).
// With A[j][i] = L^p_j(xc_i) (xi) and B[k][l] = L^p_k(ec_l) (eta):
//   child-to-parent (upward):  W_p(j, k) += sum_i A[j][i] sum_l B[k][l] W_c(i, l)
//     -- the parent's proxy weights sum_s L^p_j(xi_s) L^p_k(eta_s) w_s from
//     its children's, without revisiting the points;
//   parent-to-child (downward): Phi_c(i, l) (+)= sum_j A[j][i] sum_k B[k][l] Phi_p(j, k)
//     -- the parent's potential interpolant evaluated at the child's nodes,
//     so the child's interpolant reproduces it.
// Both are exact in exact arithmetic.  Each is applied as two 1-D transfers
// (2 (d+1)^3 multiply-adds per field instead of (d+1)^4), summed in FP64 and
// stored in FP32 like the rows they read.  One CTA per task, 256 threads:
// thread t works on field t % 64 and every fourth (row, column) of the tile.
#include <cuda_runtime.h>

#include "kernels.cuh"
#include "mixed.cuh"

namespace sal {
namespace mix {

namespace {

constexpr int kF = 64;
constexpr int kThr = 256;

// A[j n + i] = L^p_j(xc_i) and B[k n + l] = L^p_k(ec_l): threads 0..n-1 form
// the xi matrix, n..2n-1 the eta matrix (FP64, the library's BLI basis).
__device__ void transfer_matrices(const double *pnodes, const double *cnodes, int n, double *A, double *B) {
    const int t = threadIdx.x;
    double f[kMaxDegree + 1];
    if (t < n) {
        dev::bli_basis(cnodes[t], pnodes, n, f);
        for (int j = 0; j < n; ++j) A[j * n + t] = f[j];
    } else if (t < 2 * n) {
        const int l = t - n;
        dev::bli_basis(cnodes[n + l], pnodes + n, n, f);
        for (int k = 0; k < n; ++k) B[k * n + l] = f[k];
    }
}

}  // namespace

// Child-to-parent transfer of one tree level.  tasks: 5 per parent (parent
// slot, 4 child slots, -1 for none).  w: the weight rows of the slots, P rows
// of 64 fields per slot.  Dynamic shared memory: m2m_smem_bytes(n).
__global__ void __launch_bounds__(kThr) m2m_kernel(const int32_t *__restrict__ tasks, const double *__restrict__ nodes,
                                                   int n, float *__restrict__ w) {
    extern __shared__ __align__(16) double sm[];
    const int P = n * n;
    double *A = sm, *B = A + kMaxTreeP, *T = B + kMaxTreeP, *Wp = T + (size_t)kMaxTreeP * kF;
    float *Wc = reinterpret_cast<float *>(Wp + (size_t)kMaxTreeP * kF);
    const int32_t *tk = tasks + 5 * (size_t)blockIdx.x;
    const int parent = tk[0];
    const int tid = threadIdx.x, f = tid & (kF - 1), q = tid >> 6;
    for (int o = q; o < P; o += kThr / kF) Wp[o * kF + f] = 0.0;
    for (int c = 0; c < 4; ++c) {
        const int child = tk[1 + c];
        if (child < 0) continue;
        __syncthreads();   // the previous child's tiles are consumed
        transfer_matrices(nodes + (size_t)parent * 2 * n, nodes + (size_t)child * 2 * n, n, A, B);
        const float *src = w + (size_t)child * P * kF;
        for (int e = tid; e < P * kF; e += kThr) Wc[e] = src[e];
        __syncthreads();
        // T(i, k) = sum_l B[k][l] W_c(i, l)
        for (int o = q; o < P; o += kThr / kF) {
            const int i = o % n, k = o / n;
            double s = 0.0;
            for (int l = 0; l < n; ++l) s += B[k * n + l] * (double)Wc[(i + l * n) * kF + f];
            T[o * kF + f] = s;
        }
        __syncthreads();
        // W_p(j, k) += sum_i A[j][i] T(i, k)
        for (int o = q; o < P; o += kThr / kF) {
            const int j = o % n, k = o / n;
            double s = 0.0;
            for (int i = 0; i < n; ++i) s += A[j * n + i] * T[(i + k * n) * kF + f];
            Wp[o * kF + f] += s;
        }
    }
    __syncthreads();
    float *dst = w + (size_t)parent * P * kF;
    for (int o = q; o < P; o += kThr / kF) dst[o * kF + f] = (float)Wp[o * kF + f];
}

// Parent-to-child transfer of one tree level.  tasks: 3 per child (child
// slot, parent slot, own: 1 adds to the child's own potentials, 0 replaces
// them).  phi: per slot 3P rows (proxy p, Cartesian component c at row
// 3p + c) of 64 fields.  Dynamic shared memory: l2l_smem_bytes(n).
__global__ void __launch_bounds__(kThr) l2l_kernel(const int32_t *__restrict__ tasks, const double *__restrict__ nodes,
                                                   int n, float *__restrict__ phi) {
    extern __shared__ __align__(16) double sm[];
    const int P = n * n;
    double *A = sm, *B = A + kMaxTreeP, *T = B + kMaxTreeP;
    float *Pp = reinterpret_cast<float *>(T + (size_t)kMaxTreeP * kF);
    const int32_t *tk = tasks + 3 * (size_t)blockIdx.x;
    const int child = tk[0], parent = tk[1], own = tk[2];
    const int tid = threadIdx.x, f = tid & (kF - 1), q = tid >> 6;
    transfer_matrices(nodes + (size_t)parent * 2 * n, nodes + (size_t)child * 2 * n, n, A, B);
    const float *src = phi + (size_t)parent * 3 * P * kF;
    float *dst = phi + (size_t)child * 3 * P * kF;
    for (int c = 0; c < 3; ++c) {
        __syncthreads();
        for (int e = tid; e < P * kF; e += kThr) {
            const int p = e / kF;
            Pp[e] = src[((size_t)3 * p + c) * kF + (e % kF)];
        }
        __syncthreads();
        // T(j, l) = sum_k B[k][l] Phi_p(j, k)
        for (int o = q; o < P; o += kThr / kF) {
            const int j = o % n, l = o / n;
            double s = 0.0;
            for (int k = 0; k < n; ++k) s += B[k * n + l] * (double)Pp[(j + k * n) * kF + f];
            T[o * kF + f] = s;
        }
        __syncthreads();
        // Phi_c(i, l) (+)= sum_j A[j][i] T(j, l)
        for (int o = q; o < P; o += kThr / kF) {
            const int i = o % n, l = o / n;
            double s = 0.0;
            for (int j = 0; j < n; ++j) s += A[j * n + i] * T[(j + l * n) * kF + f];
            float *out = dst + ((size_t)3 * o + c) * kF + f;
            *out = own ? (float)((double)*out + s) : (float)s;
        }
    }
}

size_t m2m_smem_bytes() {
    return (2 * (size_t)kMaxTreeP + 2 * (size_t)kMaxTreeP * kF) * sizeof(double) + (size_t)kMaxTreeP * kF * sizeof(float);
}
size_t l2l_smem_bytes() {
    return (2 * (size_t)kMaxTreeP + (size_t)kMaxTreeP * kF) * sizeof(double) + (size_t)kMaxTreeP * kF * sizeof(float);
}

void launch_m2m(const int32_t *tasks, int ntasks, const double *nodes, int n, float *w, cudaStream_t st) {
    if (ntasks <= 0) return;
    static std::atomic<unsigned long long> done{0};
    smem_attr_once((const void *)m2m_kernel, (int)m2m_smem_bytes(), done);
    m2m_kernel<<<ntasks, kThr, m2m_smem_bytes(), st>>>(tasks, nodes, n, w);
}

void launch_l2l(const int32_t *tasks, int ntasks, const double *nodes, int n, float *phi, cudaStream_t st) {
    if (ntasks <= 0) return;
    static std::atomic<unsigned long long> done{0};
    smem_attr_once((const void *)l2l_kernel, (int)l2l_smem_bytes(), done);
    l2l_kernel<<<ntasks, kThr, l2l_smem_bytes(), st>>>(tasks, nodes, n, phi);
}

}  // namespace mix
}  // namespace sal
