// Antenna gain calibration (param_code/code_fft_1core/src/CPU/
// gains_calibration_run.c): one Gauss-Newton step of the gains through the
// pseudo-inverse of the normal matrix.
//
//   update_gain_calibration_actor      :20-54, 62-252  normal equations: A (2R x 2R) and Q (2R)
//   execute_calibration_SVD_actor      :254-298        A = U S V^T (LAPACK gesvd, "All")
//   calculate_SUQ_product_actor        :439-455        SUQ_i = (U^T Q)_i / S_i, 0 when |S_i| <= 1e-6
//   calculate_delta_update_gains_actor :457-476        g_r += ((V SUQ)_2r, (V SUQ)_2r+1)
//
// The normal equations, the SUQ product and the gain update are bit-exact
// with the reference's float build: every product and sum is rounded where C
// rounds it (no fused multiply-add), the per-baseline terms are formed in
// float and widened to double for the accumulation into the float arrays
// (:97-249), and every array element receives its terms in the reference's
// order (one warp owns two rows of A and two entries of Q and walks the
// baselines in index order).  The SVD is this file's own one-sided Jacobi
// method (Hestenes) in FP64 on the device, not LAPACK's bidiagonalisation,
// so U and V agree with gesvd's up to the sign of each singular pair (and a
// rotation inside degenerate subspaces); S is sorted in decreasing order as
// gesvd returns it.
#include <cuda/atomic>

#include <algorithm>
#include <cmath>

#include "internal.cuh"

namespace sdp {
namespace {

__device__ __forceinline__ float2 cmul_f(float2 a, float2 b)  // complex_multiply_CPU (:487-490)
{
    return make_float2(__fsub_rn(__fmul_rn(a.x, b.x), __fmul_rn(a.y, b.y)),
                       __fadd_rn(__fmul_rn(a.x, b.y), __fmul_rn(a.y, b.x)));
}

// p.x q.x + p.y q.y in float, as the reference's double aValue / qValue
// initialisers evaluate it (float operands), then widened
__device__ __forceinline__ double dot_f(float2 p, float2 q)
{
    return (double)__fadd_rn(__fmul_rn(p.x, q.x), __fmul_rn(p.y, q.y));
}

// A_array[i] += aValue with a float array and a double term (:99-249)
__device__ __forceinline__ void acc_f(float *a, double v) { *a = __double2float_rn(__dadd_rn((double)*a, v)); }

// Warp w owns receiver a = w: rows 2a, 2a + 1 of A and Q[2a], Q[2a + 1].
// The lanes read 32 baselines at a time; the matching ones (either receiver
// a) are applied one after the other in index order by the whole warp's
// lane 0, and within a baseline in the reference's statement order.
__global__ void k_normal_equations(int nbl, int nrx, const float2 *__restrict__ measured,
                                   const float2 *__restrict__ predicted, const float2 *__restrict__ gains,
                                   const int2 *__restrict__ pairs, float *__restrict__ A, float *__restrict__ Q,
                                   int *__restrict__ flags)
{
    const int lane = threadIdx.x & 31;
    const int a = (int)((blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5);
    if (a >= nrx) return;
    const long long ncol = 2LL * nrx;
    float *row0 = A + (2LL * a) * ncol, *row1 = row0 + ncol;
    for (int base = 0; base < nbl; base += 32) {
        const int k = base + lane;
        int2 rp = make_int2(-1, -1);
        if (k < nbl) rp = pairs[k];
        const bool bad = k < nbl && (rp.x < 0 || rp.x >= nrx || rp.y < 0 || rp.y >= nrx);
        if (bad && a == 0) atomicOr(flags, 1);
        unsigned m = __ballot_sync(0xffffffffu, !bad && k < nbl && (rp.x == a || rp.y == a));
        if (lane != 0) continue;
        while (m) {
            const int j = __ffs(m) - 1;
            m &= m - 1;
            const int b = base + j;
            const int2 ab = pairs[b];
            const int x = ab.x, y = ab.y;
            // :77-90
            const float2 vm = measured[b], vp = predicted[b];
            const float2 ga = gains[x], gy = gains[y];
            const float2 gbc = make_float2(gy.x, -gy.y);
            const float2 model = cmul_f(vp, cmul_f(ga, gbc));
            const float2 res = make_float2(__fsub_rn(vm.x, model.x), __fsub_rn(vm.y, model.y));
            const float2 ra = cmul_f(vp, gbc);
            const float2 ia = make_float2(-ra.y, ra.x);   // flip_for_i_CPU (:492-495)
            const float2 rb = cmul_f(vp, ga);
            const float2 ib = make_float2(rb.y, -rb.x);   // flip_for_neg_i_CPU (:497-500)
            const long long cx = 2LL * x, cy = 2LL * y;
            // Q (:92-104), then A (:107-249), each in statement order
            if (x == a) {
                acc_f(Q + 2 * a, dot_f(ra, res));
                acc_f(Q + 2 * a + 1, dot_f(ia, res));
            }
            if (y == a) {
                acc_f(Q + 2 * a, dot_f(rb, res));
                acc_f(Q + 2 * a + 1, dot_f(ib, res));
            }
            if (x == a) {
                acc_f(row0 + cx, dot_f(ra, ra));
                acc_f(row0 + cx + 1, dot_f(ra, ia));
                acc_f(row0 + cy, dot_f(ra, rb));
                acc_f(row0 + cy + 1, dot_f(ra, ib));
                acc_f(row1 + cx, dot_f(ia, ra));
                acc_f(row1 + cx + 1, dot_f(ia, ia));
                acc_f(row1 + cy, dot_f(ia, rb));
                acc_f(row1 + cy + 1, dot_f(ia, ib));
            }
            if (y == a) {
                acc_f(row0 + cx, dot_f(rb, ra));
                acc_f(row0 + cx + 1, dot_f(rb, ia));
                acc_f(row0 + cy, dot_f(rb, rb));
                acc_f(row0 + cy + 1, dot_f(rb, ib));
                acc_f(row1 + cx, dot_f(ib, ra));
                acc_f(row1 + cx + 1, dot_f(ib, ia));
                acc_f(row1 + cy, dot_f(ib, rb));
                acc_f(row1 + cy + 1, dot_f(ib, ib));
            }
        }
    }
}

// SUQ_i = (sum_k Q_k U[i n + k]) * sinv_i, the sum in float in k order
// (:439-455); U in LAPACK's column-major layout, so U[i n + k] = U(k, i).
__global__ void k_suq(int n, const float *__restrict__ S, const float *__restrict__ U, const float *__restrict__ Q,
                      float *__restrict__ SUQ)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float s = S[i];
    const float sinv = (fabs((double)fabsf(s)) > 1e-6) ? __double2float_rn(__ddiv_rn(1.0, (double)s)) : 0.f;
    float product = 0.f;
    const float *u = U + (long long)i * n;
    for (int k = 0; k < n; ++k) product = __fadd_rn(product, __fmul_rn(Q[k], u[k]));
    SUQ[i] = __fmul_rn(product, sinv);
}

// g_r += (sum_i SUQ_i VT[2r n + i], sum_i SUQ_i VT[(2r + 1) n + i]) (:457-476);
// VT column-major, so VT[c n + i] = VT(i, c) = V(c, i).
__global__ void k_gain_update(int n, int nrx, const float *__restrict__ SUQ, const float *__restrict__ VT,
                              const float2 *__restrict__ gin, float2 *__restrict__ gout)
{
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= nrx) return;
    const float *v0 = VT + (2LL * r) * n, *v1 = v0 + n;
    float top = 0.f, bottom = 0.f;
    for (int i = 0; i < n; ++i) {
        top = __fadd_rn(top, __fmul_rn(SUQ[i], v0[i]));
        bottom = __fadd_rn(bottom, __fmul_rn(SUQ[i], v1[i]));
    }
    const float2 g = gin[r];
    gout[r] = make_float2(__fadd_rn(g.x, top), __fadd_rn(g.y, bottom));
}

// ---------------------------------------------------------------------------
// One-sided Jacobi SVD of a square n x n matrix (FP64).  W starts as A and V
// as the identity; a sweep visits every column pair once, in n - 1 steps of
// n / 2 disjoint pairs (a round-robin schedule over n rounded up to even;
// pairs with the padding column are skipped; W and V are read around L1,
// since other CTAs rewrite their columns between steps).  A pair (p, q) with
// |w_p . w_q| > tol sqrt(|w_p|^2 |w_q|^2) is rotated so that the two
// columns become orthogonal (the same rotation applied to V).  At
// convergence W = U S: sigma_j = |w_j|, u_j = w_j / sigma_j.  One CTA per
// pair slot (all resident, cooperative launch); steps are separated by a
// bounded grid barrier (on timeout the kernel records an error and returns).
// ---------------------------------------------------------------------------
struct JacobiBar {
    unsigned count;
    unsigned gen;
    int err;
    int sweeps;  // sweeps run (the last one found every pair orthogonal)
    unsigned long long rotations[2];  // rotations of the current / previous sweep
};

constexpr int kJacobiThreads = 256;
constexpr int kJacobiRows = 8;  // rows per thread: n <= 2048
constexpr long long kJacobiSpins = 1LL << 23;
constexpr int kJacobiMaxSweeps = 60;

// Grid barrier: an arrival counter and a generation word; the last CTA to
// arrive resets the counter and advances the generation (release), the others
// poll the generation (acquire).  Bounded: after `spins` polls, or once
// another CTA gave up, a CTA records the error and returns false.  (Measured
// alternatives, one 512 x 512 SVD: a two-level counter tree, the same time;
// every CTA polling all CTAs' flags, as the persistent CLEAN kernel does,
// 1.6x slower with 256 CTAs.)
__device__ bool jacobi_barrier(JacobiBar *bar, unsigned nblocks, long long spin_limit = kJacobiSpins)
{
    __shared__ int s_ok;
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) {
        cuda::atomic_ref<unsigned, cuda::thread_scope_device> gen(bar->gen), cnt(bar->count);
        cuda::atomic_ref<int, cuda::thread_scope_device> err(bar->err);
        const unsigned g = gen.load(cuda::memory_order_acquire);
        int ok = 1;
        if (cnt.fetch_add(1u, cuda::memory_order_acq_rel) == nblocks - 1) {
            cnt.store(0u, cuda::memory_order_relaxed);
            gen.store(g + 1u, cuda::memory_order_release);
        } else {
            long long spins = 0;
            while (gen.load(cuda::memory_order_acquire) == g) {
                if (err.load(cuda::memory_order_relaxed) != 0 || ++spins > spin_limit) {
                    err.store(1, cuda::memory_order_relaxed);
                    ok = 0;
                    break;
                }
                __nanosleep(32);
            }
        }
        s_ok = ok && err.load(cuda::memory_order_relaxed) == 0;
    }
    __syncthreads();
    return s_ok != 0;
}

__device__ __forceinline__ double block_sum3(double &a, double &b, double &c)
{
    __shared__ double sa[kJacobiThreads / 32], sb[kJacobiThreads / 32], sc[kJacobiThreads / 32];
    for (int o = 16; o > 0; o >>= 1) {
        a += __shfl_xor_sync(0xffffffffu, a, o);
        b += __shfl_xor_sync(0xffffffffu, b, o);
        c += __shfl_xor_sync(0xffffffffu, c, o);
    }
    const int w = threadIdx.x >> 5;
    if ((threadIdx.x & 31) == 0) {
        sa[w] = a;
        sb[w] = b;
        sc[w] = c;
    }
    __syncthreads();
    double x = 0, y = 0, z = 0;
    for (int k = 0; k < kJacobiThreads / 32; ++k) {
        x += sa[k];
        y += sb[k];
        z += sc[k];
    }
    __syncthreads();
    a = x;
    b = y;
    c = z;
    return 0;
}

// round-robin pair i of step t over m (even) columns: column 0 fixed, the
// others rotate
__device__ __forceinline__ void rr_pair(int i, int t, int m, int &p, int &q)
{
    const int r = m - 1;
    if (i == 0) {
        p = 0;
        q = 1 + t % r;
    } else {
        p = 1 + (t + i) % r;
        q = 1 + (t - i + r) % r;
    }
}

__global__ void __launch_bounds__(kJacobiThreads) k_jacobi_svd(int n, const float *__restrict__ A, double *W,
                                                               double *V, double *sigma, JacobiBar *bar,
                                                               float *__restrict__ S, float *__restrict__ U,
                                                               float *__restrict__ VT, double tol)
{
    const unsigned nb = gridDim.x;
    const long long nn = (long long)n * n;
    for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < nn; k += (long long)nb * blockDim.x) {
        W[k] = (double)A[k];
        V[k] = (k % (n + 1) == 0) ? 1.0 : 0.0;
    }
    if (!jacobi_barrier(bar, nb)) return;
    const int m = n + (n & 1);
    const int npairs = m / 2;
    __shared__ int s_rot;
    for (int sweep = 0; sweep < kJacobiMaxSweeps; ++sweep) {
        unsigned long long rot = 0;
        for (int t = 0; t < m - 1; ++t) {
            for (int i = blockIdx.x; i < npairs; i += nb) {
                int p, q;
                rr_pair(i, t, m, p, q);
                if (p >= n || q >= n) continue;
                double *wp = W + (long long)p * n, *wq = W + (long long)q * n;
                double x[kJacobiRows], y[kJacobiRows];
                double alpha = 0, beta = 0, gamma = 0;
#pragma unroll
                for (int k = 0; k < kJacobiRows; ++k) {
                    const int r = threadIdx.x + k * kJacobiThreads;
                    x[k] = r < n ? __ldcg(wp + r) : 0.0;
                    y[k] = r < n ? __ldcg(wq + r) : 0.0;
                    alpha = fma(x[k], x[k], alpha);
                    beta = fma(y[k], y[k], beta);
                    gamma = fma(x[k], y[k], gamma);
                }
                block_sum3(alpha, beta, gamma);
                if (!(gamma != 0.0 && fabs(gamma) > tol * sqrt(alpha * beta))) continue;
                const double zeta = (beta - alpha) / (2.0 * gamma);
                const double tt = (zeta >= 0 ? 1.0 : -1.0) / (fabs(zeta) + sqrt(1.0 + zeta * zeta));
                const double c = 1.0 / sqrt(1.0 + tt * tt), s = c * tt;
                double *vp = V + (long long)p * n, *vq = V + (long long)q * n;
#pragma unroll
                for (int k = 0; k < kJacobiRows; ++k) {
                    const int r = threadIdx.x + k * kJacobiThreads;
                    if (r < n) {
                        wp[r] = c * x[k] - s * y[k];
                        wq[r] = s * x[k] + c * y[k];
                        const double u = __ldcg(vp + r), v = __ldcg(vq + r);
                        vp[r] = c * u - s * v;
                        vq[r] = s * u + c * v;
                    }
                }
                ++rot;
            }
            if (!jacobi_barrier(bar, nb)) return;
        }
        // agree on convergence: every CTA adds its count, one barrier, all read
        if (threadIdx.x == 0 && rot) atomicAdd(&bar->rotations[sweep & 1], rot);
        if (!jacobi_barrier(bar, nb)) return;
        if (threadIdx.x == 0) {
            cuda::atomic_ref<unsigned long long, cuda::thread_scope_device> cur(bar->rotations[sweep & 1]);
            s_rot = cur.load(cuda::memory_order_acquire) != 0;
        }
        __syncthreads();
        const int again = s_rot;
        // the other slot is reset for the next sweep (nobody reads it before
        // the next barrier)
        if (blockIdx.x == 0 && threadIdx.x == 0) bar->rotations[(sweep + 1) & 1] = 0;
        if (!jacobi_barrier(bar, nb)) return;
        if (blockIdx.x == 0 && threadIdx.x == 0) bar->sweeps = sweep + 1;
        if (!again) break;
    }
    // singular values, then ranks (decreasing; ties by index), then outputs
    for (int j = blockIdx.x; j < n; j += nb) {
        const double *w = W + (long long)j * n;
        double a = 0, b = 0, c = 0;
        for (int r = threadIdx.x; r < n; r += blockDim.x) {
            const double x = __ldcg(w + r);
            a = fma(x, x, a);
        }
        block_sum3(a, b, c);
        if (threadIdx.x == 0) sigma[j] = sqrt(a);
    }
    if (!jacobi_barrier(bar, nb)) return;
    for (int j = blockIdx.x; j < n; j += nb) {
        const double sj = __ldcg(sigma + j);
        __shared__ int s_rank;
        if (threadIdx.x == 0) s_rank = 0;
        __syncthreads();
        int cntr = 0;
        for (int k = threadIdx.x; k < n; k += blockDim.x) {
            const double sk = __ldcg(sigma + k);
            cntr += (sk > sj || (sk == sj && k < j)) ? 1 : 0;
        }
        atomicAdd(&s_rank, cntr);
        __syncthreads();
        const int rk = s_rank;
        const double inv = sj > 0.0 ? 1.0 / sj : 0.0;
        const double *w = W + (long long)j * n, *v = V + (long long)j * n;
        for (int r = threadIdx.x; r < n; r += blockDim.x) {
            U[(long long)rk * n + r] = (float)(__ldcg(w + r) * inv);  // column rk of U
            VT[(long long)r * n + rk] = (float)__ldcg(v + r);         // row rk of V^T
        }
        if (threadIdx.x == 0) S[rk] = (float)sj;
        __syncthreads();
    }
}

// Bounded-wait self test of the grid barrier: the barrier is told to expect
// one CTA more than the launch has, so every CTA's wait runs out after
// spin_limit polls and the error flag is set; nothing faults and the kernel
// ends.
__global__ void k_jacobi_barrier_probe(JacobiBar *bar, long long spin_limit)
{
    jacobi_barrier(bar, gridDim.x + 1, spin_limit);
}

}  // namespace

// [JacobiBar | W | V | sigma]
constexpr size_t kJacobiHead = 256;

size_t jacobi_workspace_bytes(int n)
{
    return kJacobiHead + sizeof(double) * (2 * (size_t)n * n + (size_t)n);
}

}  // namespace sdp

using namespace sdp;

SDP_EXPORT int sdp_gaincal_normal_equations(int num_baselines, int num_receivers, const sdp_float2 *measured,
                                            const sdp_float2 *predicted, const sdp_float2 *gains,
                                            const sdp_int2 *receiver_pairs, float *A, float *Q, int *flags_dev,
                                            void *stream)
{
    SDP_CHECK_ARG(num_baselines >= 0 && num_receivers >= 1, "bad sizes");
    SDP_CHECK_ARG(A && Q && flags_dev && (num_baselines == 0 || (measured && predicted && gains && receiver_pairs)),
                  "NULL argument");
    cudaStream_t st = as_stream(stream);
    const size_t nc = 2 * (size_t)num_receivers;
    SDP_CUDA_TRY(cudaMemsetAsync(Q, 0, sizeof(float) * nc, st));  // :36-37
    SDP_CUDA_TRY(cudaMemsetAsync(A, 0, sizeof(float) * nc * nc, st));
    if (num_baselines == 0) return SDP_OK;
    const long long threads = 32LL * num_receivers;
    k_normal_equations<<<(unsigned)((threads + 255) / 256), 256, 0, st>>>(
        num_baselines, num_receivers, reinterpret_cast<const float2 *>(measured),
        reinterpret_cast<const float2 *>(predicted), reinterpret_cast<const float2 *>(gains),
        reinterpret_cast<const int2 *>(receiver_pairs), A, Q, flags_dev);
    SDP_LAUNCH_CHECK();
    return SDP_OK;
}

SDP_EXPORT int sdp_svd_workspace_bytes(int n, size_t *bytes)
{
    SDP_CHECK_ARG(n >= 1 && bytes, "bad argument");
    *bytes = jacobi_workspace_bytes(n);
    return SDP_OK;
}

SDP_EXPORT int sdp_svd(int n, const float *A, float *S, float *U, float *VT, void *workspace, size_t ws_bytes,
                       void *stream)
{
    SDP_CHECK_ARG(n >= 1 && A && S && U && VT && workspace, "bad argument");
    if (ws_bytes < jacobi_workspace_bytes(n))
        return set_error(SDP_ERR_RANGE, "svd workspace %zu B < %zu B", ws_bytes, jacobi_workspace_bytes(n));
    cudaStream_t st = as_stream(stream);
    char *w = static_cast<char *>(workspace);
    JacobiBar *bar = reinterpret_cast<JacobiBar *>(w);
    double *W = reinterpret_cast<double *>(w + kJacobiHead);
    double *V = W + (size_t)n * n;
    double *sigma = V + (size_t)n * n;
    SDP_CHECK_ARG(n <= kJacobiRows * kJacobiThreads, "svd: n = %d above %d", n, kJacobiRows * kJacobiThreads);
    SDP_CUDA_TRY(cudaMemsetAsync(bar, 0, kJacobiHead, st));
    int dev = 0, per_sm = 0;
    SDP_CUDA_TRY(cudaGetDevice(&dev));
    SDP_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_jacobi_svd, kJacobiThreads, 0));
    if (per_sm < 1) return set_error(SDP_ERR_CUDA, "svd kernel does not fit on an SM");
    const int npairs = (n + (n & 1)) / 2;
    const int nb = std::max(1, std::min(npairs, per_sm * num_sms()));
    int nv = n;
    const float *a = A;
    // a pair counts as orthogonal below n x the FP64 epsilon (relative)
    double tol = std::max(1e-15, (double)n * 2.220446049250313e-16);
    void *args[] = {&nv, (void *)&a, &W, &V, &sigma, &bar, &S, &U, &VT, &tol};
    SDP_CUDA_TRY(cudaLaunchCooperativeKernel((const void *)k_jacobi_svd, dim3(nb), dim3(kJacobiThreads), args, 0, st));
    return SDP_OK;
}

// Status of the last sdp_svd on this workspace: SDP_ERR_TIMEOUT when a
// barrier wait gave up; sweeps (may be NULL) receives the sweeps it ran.
SDP_EXPORT int sdp_svd_check(const void *workspace, int *sweeps, void *stream)
{
    SDP_CHECK_ARG(workspace, "NULL argument");
    cudaStream_t st = as_stream(stream);
    JacobiBar b;
    SDP_CUDA_TRY(cudaMemcpyAsync(&b, workspace, sizeof(JacobiBar), cudaMemcpyDeviceToHost, st));
    SDP_CUDA_TRY(cudaStreamSynchronize(st));
    if (sweeps) *sweeps = b.sweeps;
    return b.err ? set_error(SDP_ERR_TIMEOUT, "svd: a grid barrier wait gave up") : SDP_OK;
}

SDP_EXPORT int sdp_selftest_svd_barrier(int nblocks, long long spin_limit, int *status)
{
    SDP_CHECK_ARG(status != nullptr && nblocks >= 1 && nblocks <= 64 && spin_limit >= 1, "bad argument");
    *status = SDP_OK;
    JacobiBar *bar = nullptr;
    SDP_CUDA_TRY(cudaMalloc(&bar, sizeof(JacobiBar)));
    int err = 0;
    cudaError_t e = cudaMemset(bar, 0, sizeof(JacobiBar));
    if (e == cudaSuccess) {
        k_jacobi_barrier_probe<<<nblocks, 32>>>(bar, spin_limit);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaDeviceSynchronize();
    if (e == cudaSuccess) e = cudaMemcpy(&err, &bar->err, sizeof(int), cudaMemcpyDeviceToHost);
    cudaFree(bar);
    if (e != cudaSuccess) return cuda_error(e, "svd barrier self test");
    *status = err ? SDP_ERR_TIMEOUT : SDP_OK;
    return SDP_OK;
}

SDP_EXPORT int sdp_gaincal_suq(int n, const float *S, const float *U, const float *Q, float *SUQ, void *stream)
{
    SDP_CHECK_ARG(n >= 1 && S && U && Q && SUQ, "bad argument");
    k_suq<<<(n + 127) / 128, 128, 0, as_stream(stream)>>>(n, S, U, Q, SUQ);
    SDP_LAUNCH_CHECK();
    return SDP_OK;
}

SDP_EXPORT int sdp_gaincal_update(int n, int num_receivers, const float *SUQ, const float *VT,
                                  const sdp_float2 *gains_in, sdp_float2 *gains_out, void *stream)
{
    SDP_CHECK_ARG(n >= 1 && num_receivers >= 1 && 2 * num_receivers <= n, "bad sizes");
    SDP_CHECK_ARG(SUQ && VT && gains_in && gains_out, "NULL argument");
    k_gain_update<<<(num_receivers + 127) / 128, 128, 0, as_stream(stream)>>>(
        n, num_receivers, SUQ, VT, reinterpret_cast<const float2 *>(gains_in), reinterpret_cast<float2 *>(gains_out));
    SDP_LAUNCH_CHECK();
    return SDP_OK;
}

// ---------------------------------------------------------------------------
// Actors (host buffers; gains_calibration_run.h:25-35)
// ---------------------------------------------------------------------------
namespace {

int stage_buffers(ThreadCtx **ctx, size_t bytes, char **d)
{
    SDP_TRY(thread_ctx(ctx));
    void *p = nullptr;
    SDP_TRY(ctx_buffer(*ctx, kSlotRestore + 0, bytes, &p));
    *d = static_cast<char *>(p);
    return SDP_OK;
}

size_t al(size_t b) { return (b + 255) / 256 * 256; }

int do_update(int NBL, int NRX, const sdp_float2 *measured, const sdp_float2 *vis, const sdp_float2 *gains,
              const sdp_int2 *pairs, float *A, float *Q)
{
    SDP_CHECK_ARG(NBL >= 0 && NRX >= 1 && A && Q && (NBL == 0 || (measured && vis && gains && pairs)),
                  "bad argument");
    const size_t nc = 2 * (size_t)NRX;
    const size_t bm = al(sizeof(float2) * std::max(NBL, 1)), bg = al(sizeof(float2) * NRX),
                 bp = al(sizeof(int2) * std::max(NBL, 1)), ba = al(sizeof(float) * nc * nc), bq = al(sizeof(float) * nc);
    ThreadCtx *ctx = nullptr;
    char *d = nullptr;
    SDP_TRY(stage_buffers(&ctx, 2 * bm + bg + bp + ba + bq + 256, &d));
    cudaStream_t st = ctx->stream;
    float2 *dm = reinterpret_cast<float2 *>(d), *dv = reinterpret_cast<float2 *>(d + bm);
    float2 *dg = reinterpret_cast<float2 *>(d + 2 * bm);
    int2 *dp = reinterpret_cast<int2 *>(d + 2 * bm + bg);
    float *dA = reinterpret_cast<float *>(d + 2 * bm + bg + bp), *dQ = reinterpret_cast<float *>(d + 2 * bm + bg + bp + ba);
    int *df = reinterpret_cast<int *>(d + 2 * bm + bg + bp + ba + bq);
    if (NBL > 0) {
        SDP_CUDA_TRY(cudaMemcpyAsync(dm, measured, sizeof(float2) * NBL, cudaMemcpyHostToDevice, st));
        SDP_CUDA_TRY(cudaMemcpyAsync(dv, vis, sizeof(float2) * NBL, cudaMemcpyHostToDevice, st));
        SDP_CUDA_TRY(cudaMemcpyAsync(dp, pairs, sizeof(int2) * NBL, cudaMemcpyHostToDevice, st));
    }
    SDP_CUDA_TRY(cudaMemcpyAsync(dg, gains, sizeof(float2) * NRX, cudaMemcpyHostToDevice, st));
    SDP_CUDA_TRY(cudaMemsetAsync(df, 0, sizeof(int), st));
    SDP_TRY(sdp_gaincal_normal_equations(NBL, NRX, reinterpret_cast<sdp_float2 *>(dm), reinterpret_cast<sdp_float2 *>(dv),
                                         reinterpret_cast<sdp_float2 *>(dg), reinterpret_cast<sdp_int2 *>(dp), dA, dQ,
                                         df, st));
    int flags = 0;
    SDP_CUDA_TRY(cudaMemcpyAsync(A, dA, sizeof(float) * nc * nc, cudaMemcpyDeviceToHost, st));
    SDP_CUDA_TRY(cudaMemcpyAsync(Q, dQ, sizeof(float) * nc, cudaMemcpyDeviceToHost, st));
    SDP_CUDA_TRY(cudaMemcpyAsync(&flags, df, sizeof(int), cudaMemcpyDeviceToHost, st));
    SDP_CUDA_TRY(cudaStreamSynchronize(st));
    if (flags) return set_error(SDP_ERR_DATA, "a receiver pair indexes outside the %d gains", NRX);
    return SDP_OK;
}

int do_svd(int NCOLS, int NROWS, const float *A, float *S, float *U, float *V)
{
    SDP_CHECK_ARG(NCOLS >= 1 && NROWS >= 1 && A && S && U && V, "bad argument");
    if (NCOLS != NROWS)
        return set_error(SDP_ERR_INVALID, "the SVD actor takes square matrices (%d x %d); the calibration's is", NROWS,
                         NCOLS);
    const int n = NCOLS;
    const size_t nn = (size_t)n * n, bm = al(sizeof(float) * nn), bs = al(sizeof(float) * n);
    const size_t bw = al(jacobi_workspace_bytes(n));
    ThreadCtx *ctx = nullptr;
    char *d = nullptr;
    SDP_TRY(stage_buffers(&ctx, 3 * bm + bs + bw, &d));
    cudaStream_t st = ctx->stream;
    float *dA = reinterpret_cast<float *>(d), *dU = reinterpret_cast<float *>(d + bm);
    float *dV = reinterpret_cast<float *>(d + 2 * bm), *dS = reinterpret_cast<float *>(d + 3 * bm);
    void *ws = d + 3 * bm + bs;
    SDP_CUDA_TRY(cudaMemcpyAsync(dA, A, sizeof(float) * nn, cudaMemcpyHostToDevice, st));
    SDP_TRY(sdp_svd(n, dA, dS, dU, dV, ws, bw, st));
    SDP_TRY(sdp_svd_check(ws, nullptr, st));
    SDP_CUDA_TRY(cudaMemcpyAsync(S, dS, sizeof(float) * n, cudaMemcpyDeviceToHost, st));
    SDP_CUDA_TRY(cudaMemcpyAsync(U, dU, sizeof(float) * nn, cudaMemcpyDeviceToHost, st));
    SDP_CUDA_TRY(cudaMemcpyAsync(V, dV, sizeof(float) * nn, cudaMemcpyDeviceToHost, st));
    SDP_CUDA_TRY(cudaStreamSynchronize(st));
    return SDP_OK;
}

int do_suq(int NCOLS, const float *S, const float *U, const float *Q, float *SUQ)
{
    SDP_CHECK_ARG(NCOLS >= 1 && S && U && Q && SUQ, "bad argument");
    const int n = NCOLS;
    const size_t nn = (size_t)n * n, bm = al(sizeof(float) * nn), bs = al(sizeof(float) * n);
    ThreadCtx *ctx = nullptr;
    char *d = nullptr;
    SDP_TRY(stage_buffers(&ctx, bm + 3 * bs, &d));
    cudaStream_t st = ctx->stream;
    float *dU = reinterpret_cast<float *>(d), *dS = reinterpret_cast<float *>(d + bm);
    float *dQ = reinterpret_cast<float *>(d + bm + bs), *dR = reinterpret_cast<float *>(d + bm + 2 * bs);
    SDP_CUDA_TRY(cudaMemcpyAsync(dU, U, sizeof(float) * nn, cudaMemcpyHostToDevice, st));
    SDP_CUDA_TRY(cudaMemcpyAsync(dS, S, sizeof(float) * n, cudaMemcpyHostToDevice, st));
    SDP_CUDA_TRY(cudaMemcpyAsync(dQ, Q, sizeof(float) * n, cudaMemcpyHostToDevice, st));
    SDP_TRY(sdp_gaincal_suq(n, dS, dU, dQ, dR, st));
    SDP_CUDA_TRY(cudaMemcpyAsync(SUQ, dR, sizeof(float) * n, cudaMemcpyDeviceToHost, st));
    SDP_CUDA_TRY(cudaStreamSynchronize(st));
    return SDP_OK;
}

int do_delta(int NCOLS, int NRX, const float *SUQ, const float *V, const sdp_float2 *gin, sdp_float2 *gout)
{
    SDP_CHECK_ARG(NCOLS >= 1 && NRX >= 1 && 2 * NRX <= NCOLS && SUQ && V && gin && gout, "bad argument");
    const int n = NCOLS;
    const size_t nn = (size_t)n * n, bm = al(sizeof(float) * nn), bs = al(sizeof(float) * n),
                 bg = al(sizeof(float2) * NRX);
    ThreadCtx *ctx = nullptr;
    char *d = nullptr;
    SDP_TRY(stage_buffers(&ctx, bm + bs + 2 * bg, &d));
    cudaStream_t st = ctx->stream;
    float *dV = reinterpret_cast<float *>(d), *dR = reinterpret_cast<float *>(d + bm);
    sdp_float2 *dgi = reinterpret_cast<sdp_float2 *>(d + bm + bs), *dgo = reinterpret_cast<sdp_float2 *>(d + bm + bs + bg);
    SDP_CUDA_TRY(cudaMemcpyAsync(dV, V, sizeof(float) * nn, cudaMemcpyHostToDevice, st));
    SDP_CUDA_TRY(cudaMemcpyAsync(dR, SUQ, sizeof(float) * n, cudaMemcpyHostToDevice, st));
    SDP_CUDA_TRY(cudaMemcpyAsync(dgi, gin, sizeof(float2) * NRX, cudaMemcpyHostToDevice, st));
    SDP_TRY(sdp_gaincal_update(n, NRX, dR, dV, dgi, dgo, st));
    SDP_CUDA_TRY(cudaMemcpyAsync(gout, dgo, sizeof(float2) * NRX, cudaMemcpyDeviceToHost, st));
    SDP_CUDA_TRY(cudaStreamSynchronize(st));
    return SDP_OK;
}

}  // namespace

SDP_EXPORT void update_gain_calibration_actor(int NUM_BASELINES, int NUM_RECEIVERS, int NUM_VISIBILITIES,
                                              int *loop_cycle_token, sdp_float2 *measured_vis,
                                              sdp_float2 *visibilities, sdp_float2 *gains,
                                              sdp_int2 *receiver_pairs, sdp_config *config, float *A_array,
                                              float *Q_array)
{
    (void)NUM_VISIBILITIES;
    (void)loop_cycle_token;
    (void)config;
    if (do_update(NUM_BASELINES, NUM_RECEIVERS, measured_vis, visibilities, gains, receiver_pairs, A_array,
                  Q_array) != SDP_OK)
        actor_fail("update_gain_calibration_actor");
}

SDP_EXPORT void execute_calibration_SVD_actor(int NUM_COLS, int NUM_ROWS, float *A_array, float *S_array,
                                              float *U_array, float *V_array)
{
    if (do_svd(NUM_COLS, NUM_ROWS, A_array, S_array, U_array, V_array) != SDP_OK)
        actor_fail("execute_calibration_SVD_actor");
}

SDP_EXPORT void calculate_SUQ_product_actor(int NUM_COLS, int NUM_ROWS, float *S_array, float *U_array,
                                            float *Q_array, sdp_config *config, float *SUQ_array)
{
    (void)NUM_ROWS;
    (void)config;
    if (do_suq(NUM_COLS, S_array, U_array, Q_array, SUQ_array) != SDP_OK) actor_fail("calculate_SUQ_product_actor");
}

SDP_EXPORT void calculate_delta_update_gains_actor(int NUM_COLS, int NUM_RECEIVERS, float *SUQ_array,
                                                   float *V_array, sdp_config *config, sdp_float2 *gains_in,
                                                   sdp_float2 *gains_out)
{
    (void)config;
    if (do_delta(NUM_COLS, NUM_RECEIVERS, SUQ_array, V_array, gains_in, gains_out) != SDP_OK)
        actor_fail("calculate_delta_update_gains_actor");
}
