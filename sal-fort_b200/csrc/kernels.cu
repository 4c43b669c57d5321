// FP64 kernels of the SAL-gradient treecode for sm_100a.
//
// All passes are compute-bound on the FP64 pipe: every staged source tile is
// reused by every target of its group (up to 256), so HBM traffic per pair is
// a few bytes against ~60 FP64 operations.
#include <cuda_runtime.h>

#include "kernels.cuh"

namespace sal {
namespace dev {

// ------------------------------------------------------------------ prep
// Per-solve source weights w = area * ssh in pool order (the factor
// area(j)*ssh(j) of fast_sum_module.f90:69-70).
__global__ void prep_kernel(const double4 *__restrict__ xyz, const double *__restrict__ area,
                            const double *__restrict__ ssh, const int32_t *__restrict__ perm, int n,
                            double4 *__restrict__ pool) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double4 p = xyz[i];
    p.w = area[i] * ssh[perm[i]];
    pool[i] = p;
}

void launch_prep(const double4 *xyz, const double *area, const double *ssh, const int32_t *perm, int n, double4 *pool,
                 cudaStream_t st) {
    if (n <= 0) return;
    prep_kernel<<<(n + 255) / 256, 256, 0, st>>>(xyz, area, ssh, perm, n, pool);
}

// ------------------------------------------------------------------ upward pass
// Proxy weights of one (source slot, chunk) unit: W[j + k n] = sum over the
// chunk's points of xi_basis_j * eta_basis_k * w (fast_sum_module.f90:99-111).
// Threads 0..127 form the xi bases of 128 points, threads 128..255 the eta
// bases times w; then P accumulators (3 thread groups for d = 8) reduce the
// tile.
__global__ void __launch_bounds__(kThreads) upward_kernel(UpArgs a) {
    __shared__ double fx[128][kMaxDegree + 1];
    __shared__ double fe[128][kMaxDegree + 1];
    __shared__ double nod[2 * (kMaxDegree + 1)];
    __shared__ double red[kThreads];
    const UpUnit u = a.units[blockIdx.x];
    const int tid = threadIdx.x, n = a.d + 1, P = a.P;
    if (tid < 2 * n) nod[tid] = a.nodes[(size_t)u.slot * 2 * n + tid];
    __syncthreads();
    const int nsub = kThreads / P;
    const int grp = tid / P, pidx = tid % P, j = pidx % n, k = pidx / n;
    double W = 0.0;
    double f[kMaxDegree + 1];
    for (int b = u.beg; b < u.end; b += 128) {
        const int m = min(128, u.end - b);
        if (tid < m) {
            bli_basis(a.xieta[b + tid].x, nod, n, f);
            for (int i = 0; i < n; ++i) fx[tid][i] = f[i];
        } else if (tid >= 128 && tid - 128 < m) {
            const int s = tid - 128;
            bli_basis(a.xieta[b + s].y, nod + n, n, f);
            const double w = a.pool[b + s].w;
            for (int i = 0; i < n; ++i) fe[s][i] = f[i] * w;
        }
        __syncthreads();
        if (grp < nsub)
            for (int s = grp; s < m; s += nsub) W += fx[s][j] * fe[s][k];
        __syncthreads();
    }
    red[tid] = W;
    __syncthreads();
    if (grp == 0) {
        double acc = 0.0;
        for (int g = 0; g < nsub; ++g) acc += red[g * P + pidx];
        a.partial[(size_t)blockIdx.x * P + pidx] = acc;
    }
}

void launch_upward(const UpArgs &a, int nunits, cudaStream_t st) {
    if (nunits <= 0) return;
    upward_kernel<<<nunits, kThreads, 0, st>>>(a);
}

// Sums each slot's unit partials in unit order into the w of its pool
// proxies.  transposed != 0 stores W[k + j n] at proxy j + k n, the layout
// mom6_fast_sum_module.f90:63-70 produces.
__global__ void upward_finalize_kernel(const int32_t *__restrict__ unit_beg, const double *__restrict__ partial,
                                       int nslots, int d, int transposed, double4 *__restrict__ pool_proxy) {
    const int n = d + 1, P = n * n;
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (long long)nslots * P) return;
    const int s = (int)(t / P), p = (int)(t % P);
    const int j = p % n, k = p / n;
    const int src = transposed ? (k + j * n) : p;
    double acc = 0.0;
    for (int u = unit_beg[s]; u < unit_beg[s + 1]; ++u) acc += partial[(size_t)u * P + src];
    pool_proxy[(size_t)s * P + p].w = acc;
}

void launch_upward_finalize(const int32_t *unit_beg, const double *partial, int nslots, int d, int transposed,
                            double4 *pool_proxy, cudaStream_t st) {
    long long tot = (long long)nslots * (d + 1) * (d + 1);
    if (tot <= 0) return;
    upward_finalize_kernel<<<(unsigned)((tot + 255) / 256), 256, 0, st>>>(unit_beg, partial, nslots, d, transposed,
                                                                          pool_proxy);
}

// ------------------------------------------------------------------ targets x staged sources
// One CTA per group (a leaf, or a unit of a target slot's proxies).  Its item
// list is walked in order; each item's sources (a pool range, or a DOWN record)
// are brought into shared memory by one bulk copy, double-buffered, and every
// target of the group consumes them.  Targets are spread over the 256 threads
// as ti = tid % ntp with nsplit = 256 / ntp source splits that are summed in
// a fixed order at the end, so results are deterministic.
//   TGT 0: leaf targets (pool points), items PP / PC / DOWN, writes outputs.
//   TGT 1: proxy targets, items CP (points) / CC (proxies), writes partials.
//   FORM 0: reference kernel everywhere (2 components in each target's frame).
//   FORM 1: proxy targets accumulate the Cartesian sum val*(s-x)*w with the
//           antipode-stable val; DOWN interpolates it and projects on the
//           leaf target's frame.
template <int TGT, int FORM>
__global__ void __launch_bounds__(kThreads) eval_kernel(EvalArgs a) {
    __shared__ __align__(128) double4 buf[2][kMaxStage];
    __shared__ __align__(8) uint64_t bar[2];
    __shared__ double red[3][kThreads];
    __shared__ int tout;
    const Group G = a.groups[blockIdx.x];
    const int tid = threadIdx.x;
    const int nt = G.nt;
    const int ntp = (nt + 31) & ~31;
    const int nsplit = max(1, kThreads / ntp);
    const int ti = tid % ntp, sp = tid / ntp;
    const bool active = (ti < nt) && (sp < nsplit);
    Tgt T;
    double txi = 0.0, teta = 0.0;
    if (active) {
        const double4 c = (TGT == 0) ? a.tgt[G.tgt + ti] : a.tgt[(size_t)G.tgt * a.P + ti];
        tgt_init(T, c.x, c.y, c.z);
        if (TGT == 0) {
            const double2 e = a.xieta[G.tgt + ti];
            txi = e.x;
            teta = e.y;
        }
    } else {
        tgt_init(T, 0.0, 0.0, 0.5);
        T.live = false;
    }
    double ax = 0.0, ay = 0.0, az = 0.0;  // PP/PC sums, before the target factor (proxy targets in FORM 1: Cartesian)
    double ux = 0.0, uy = 0.0, uz = 0.0;  // DOWN sums (FORM 0: east/north; FORM 1: Cartesian)
    if (tid == 0) {
        mbar_init(&bar[0], 1);
        mbar_init(&bar[1], 1);
        fence_mbar_init();
        tout = 0;
    }
    __syncthreads();
    const int ni = G.ie - G.ib;
    const uint32_t polls = a.polls ? a.polls : kDefaultPolls;
    auto issue = [&](int k) {
        // fault injection (tests of the time-out path): the group's last copy
        // is never issued, so its wait runs out with no copy in flight
        if (a.skip_last && k == ni - 1) return;
        const Item it = a.items[G.ib + k];
        const void *src;
        uint32_t bytes;
        if (it.kind == 2) {
            src = a.records + (size_t)it.off * a.rec_stride;
            bytes = (uint32_t)a.rec_stride * 8u;
        } else {
            src = a.pool + it.off;
            bytes = (uint32_t)it.cnt * 32u;
        }
        uint64_t *b = &bar[k & 1];
        fence_proxy_async();
        mbar_expect_tx(b, bytes);
        bulk_g2s(buf[k & 1], src, bytes, b);
    };
    if (tid == 0 && ni > 0) issue(0);
    const int n = a.d + 1;
    for (int k = 0; k < ni; ++k) {
        if (tid == 0 && k + 1 < ni) issue(k + 1);
        const Item it = a.items[G.ib + k];
        if (!mbar_wait_bounded(&bar[k & 1], (uint32_t)((k >> 1) & 1), a.err, polls)) tout = 1;
        const double4 *S = buf[k & 1];
        if (it.kind == 2) {
            if (TGT == 0 && active && sp == 0 && ((a.kinds >> 2) & 1)) {
                // interp_vals_bli + the loops of fast_sum_module.f90:186-199
                const double *R = reinterpret_cast<const double *>(S);
                const double *nodes = R + 4 * a.P;
                double fx[kMaxDegree + 1], fe[kMaxDegree + 1];
                bli_basis(txi, nodes, n, fx);
                bli_basis(teta, nodes + n, n, fe);
                for (int kk = 0; kk < n; ++kk)
                    for (int jj = 0; jj < n; ++jj) {
                        const double bv = fx[jj] * fe[kk];
                        const double4 ph = S[jj + kk * n];
                        if (FORM == 0) {
                            ux += bv * ph.x;
                            uy += bv * ph.y;
                        } else {
                            ux += bv * ph.x;
                            uy += bv * ph.y;
                            uz += bv * ph.z;
                        }
                    }
            }
        } else if ((a.kinds >> it.kind) & 1) {
            bool on = active && (T.live || (TGT == 1 && FORM == 1));
            if (on && it.mask >= 0) on = (a.masks[it.mask + (ti >> 5)] >> (ti & 31)) & 1u;
            if (on) {
                if (TGT == 1 && FORM == 1) {
                    for (int s = sp; s < it.cnt; s += nsplit) {
                        const double4 q = S[s];
                        const double dx = q.x - T.x, dy = q.y - T.y, dz = q.z - T.z;
                        const double v = vstable(dx * dx + dy * dy + dz * dz) * q.w;
                        ax += v * dx;
                        ay += v * dy;
                        az += v * dz;
                    }
                } else {
                    for (int s = sp; s < it.cnt; s += nsplit) {
                        const double4 q = S[s];
                        gref_fast(T, q.x, q.y, q.z, q.w, ax, ay);
                    }
                }
            }
        }
        __syncthreads();
    }
    if (!(TGT == 1 && FORM == 1)) {
        // the target factor 1/sqrt(1 - tz^2) of every pair sum (zero outside the pole guard)
        ax *= T.live ? T.inv_mp2 : 0.0;
        ay *= T.live ? T.inv_mp2 : 0.0;
    }
    if (TGT == 0 && FORM == 0) {
        ax += ux;
        ay += uy;
    }
    if (TGT == 0 && FORM == 1 && active && sp == 0 && T.live) {
        // project the interpolated Cartesian sum on the target's east/north frame
        ax += (T.x * uy - T.y * ux) * T.inv_mp2;
        ay += (uz * T.omx32 - T.z * (T.x * ux + T.y * uy)) * T.inv_mp2;
    }
    red[0][tid] = ax;
    red[1][tid] = ay;
    red[2][tid] = az;
    __syncthreads();
    if (active && sp == 0) {
        double rx = 0.0, ry = 0.0, rz = 0.0;
        for (int s = 0; s < nsplit; ++s) {
            rx += red[0][s * ntp + ti];
            ry += red[1][s * ntp + ti];
            rz += red[2][s * ntp + ti];
        }
        if (TGT == 0) {
            const int idx = a.perm[G.tgt + ti];
            a.out_x[idx] = rx;
            a.out_y[idx] = ry;
        } else {
            a.partial[(size_t)G.out * a.P + ti] = make_double4(rx, ry, rz, 0.0);
        }
    }
    if (tout && tid == 0) {
        // a copy timed out: give any copy still in flight a last bounded wait
        for (int k = max(0, ni - 2); k < ni; ++k) mbar_wait_bounded(&bar[k & 1], (uint32_t)((k >> 1) & 1), a.err, polls);
    }
}

void launch_eval(int tgt_kind, int form, const EvalArgs &a, int ngroups, cudaStream_t st) {
    if (ngroups <= 0) return;
    if (tgt_kind == 0 && form == 0) eval_kernel<0, 0><<<ngroups, kThreads, 0, st>>>(a);
    else if (tgt_kind == 0) eval_kernel<0, 1><<<ngroups, kThreads, 0, st>>>(a);
    else if (form == 0) eval_kernel<1, 0><<<ngroups, kThreads, 0, st>>>(a);
    else eval_kernel<1, 1><<<ngroups, kThreads, 0, st>>>(a);
}

// Sums each target slot's unit partials in unit order into its record.
__global__ void proxy_finalize_kernel(const int32_t *__restrict__ unit_beg, const double4 *__restrict__ partial,
                                      int nslots, int P, int rec_stride, double *__restrict__ records) {
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (long long)nslots * P) return;
    const int s = (int)(t / P), p = (int)(t % P);
    double x = 0.0, y = 0.0, z = 0.0;
    for (int u = unit_beg[s]; u < unit_beg[s + 1]; ++u) {
        const double4 v = partial[(size_t)u * P + p];
        x += v.x;
        y += v.y;
        z += v.z;
    }
    double4 *rec = reinterpret_cast<double4 *>(records + (size_t)s * rec_stride);
    rec[p] = make_double4(x, y, z, 0.0);
}

void launch_proxy_finalize(const int32_t *unit_beg, const double4 *partial, int nslots, int P, int rec_stride,
                           double *records, cudaStream_t st) {
    long long tot = (long long)nslots * P;
    if (tot <= 0) return;
    proxy_finalize_kernel<<<(unsigned)((tot + 255) / 256), 256, 0, st>>>(unit_beg, partial, nslots, P, rec_stride,
                                                                         records);
}

// ------------------------------------------------------------------ direct sum
// FP64 direct O(N^2) sum at sampled targets with the reference kernel, sources
// split into chunks (blockIdx.y) whose partial sums are added in chunk order.
constexpr int kDirectTile = 128;
__global__ void __launch_bounds__(kDirectTile) direct_kernel(const double *__restrict__ xs, const double *__restrict__ ys,
                                                             const double *__restrict__ zs, const double *__restrict__ w,
                                                             int n, const int32_t *__restrict__ targets, int nt,
                                                             int chunk, double *__restrict__ partial) {
    __shared__ double4 S[kDirectTile];
    const int k = blockIdx.x * kDirectTile + threadIdx.x;
    const int s0 = blockIdx.y * chunk, s1 = min(n, s0 + chunk);
    Tgt T;
    if (k < nt) {
        const int ti = targets[k];
        tgt_init(T, xs[ti], ys[ti], zs[ti]);
    } else {
        tgt_init(T, 0.0, 0.0, 0.5);
        T.live = false;
    }
    double ax = 0.0, ay = 0.0;
    for (int b = s0; b < s1; b += kDirectTile) {
        const int m = min(kDirectTile, s1 - b);
        if (threadIdx.x < m) {
            const int s = b + threadIdx.x;
            S[threadIdx.x] = make_double4(xs[s], ys[s], zs[s], w[s]);
        }
        __syncthreads();
        if (T.live)
            for (int s = 0; s < m; ++s) {
                double gx, gy;
                gref_exact(T, S[s].x, S[s].y, S[s].z, gx, gy);
                ax += gx * S[s].w;
                ay += gy * S[s].w;
            }
        __syncthreads();
    }
    if (k < nt) {
        partial[((size_t)blockIdx.y * nt + k) * 2] = ax;
        partial[((size_t)blockIdx.y * nt + k) * 2 + 1] = ay;
    }
}

__global__ void direct_reduce_kernel(const double *__restrict__ partial, int nt, int nchunks, double *__restrict__ ox,
                                     double *__restrict__ oy) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= nt) return;
    double x = 0.0, y = 0.0;
    for (int c = 0; c < nchunks; ++c) {
        x += partial[((size_t)c * nt + k) * 2];
        y += partial[((size_t)c * nt + k) * 2 + 1];
    }
    ox[k] = x;
    oy[k] = y;
}

int direct_chunks(int n) { return max(1, min(64, (n + 32767) / 32768)); }

void launch_direct(const double *xs, const double *ys, const double *zs, const double *w, int n,
                   const int32_t *targets, int nt, double *out_x, double *out_y, double *scratch, int nchunks,
                   cudaStream_t st) {
    if (nt <= 0) return;
    const int chunk = (n + nchunks - 1) / nchunks;
    dim3 grid((nt + kDirectTile - 1) / kDirectTile, nchunks);
    direct_kernel<<<grid, kDirectTile, 0, st>>>(xs, ys, zs, w, n, targets, nt, chunk, scratch);
    direct_reduce_kernel<<<(nt + 255) / 256, 256, 0, st>>>(scratch, nt, nchunks, out_x, out_y);
}

// ------------------------------------------------------------------ proxy weight transfer
__global__ void extract_w_kernel(const double4 *__restrict__ pp, int count, double *__restrict__ out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < count) out[i] = pp[i].w;
}
__global__ void insert_w_kernel(const double *__restrict__ w, int count, double4 *__restrict__ pp) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < count) pp[i].w = w[i];
}
void launch_extract_w(const double4 *pool_proxy, int count, double *out, cudaStream_t st) {
    if (count > 0) extract_w_kernel<<<(count + 255) / 256, 256, 0, st>>>(pool_proxy, count, out);
}
void launch_insert_w(const double *w, int count, double4 *pool_proxy, cudaStream_t st) {
    if (count > 0) insert_w_kernel<<<(count + 255) / 256, 256, 0, st>>>(w, count, pool_proxy);
}

}  // namespace dev
}  // namespace sal
