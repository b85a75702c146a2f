// Inputs the reference reads from files but never generates: W-projection
// kernel tables and the dirty PSF.
//
// W-projection kernels (Cornwell, Golap & Bhatnagar 2008).  The image-plane
// kernel of plane p is the taper times the w screen, taper(l) taper(m)
// exp(-i pi w_p (l^2 + m^2)) with the paraxial approximation; both factors
// are separable, so the uv-plane kernel is the outer product of one 1-D
// kernel with itself.  The taper is the prolate spheroidal the pipeline's
// taper correction divides by (top.c:412-451), sampled at M points across the
// field of view L: l_j = (j - M/2) L / M, taper_j = prolate(|2 l_j / L|).  The
// 1-D kernel, oversampled OS times, is the Fourier transform of that screen
// zero-padded to M*OS points, taken at uv offsets s / OS cells:
//   k(s) = sum_j taper_j exp(-i pi w l_j^2) exp(-2 pi i s (j - M/2) / (M OS))
// for s = 0 .. (hs+1) OS - 1 (the quarter-plane layout of the reference's
// tables: index |dv| OS, |du| OS, top.c:256-261).  Plane p has w_p = p^2
// max_w / (P-1)^2, the centre of the plane index round(sqrt(|w| w_scale)).
// Every plane is divided by the sum of the w = 0 kernel over its taps at
// whole-cell offsets (-hs0 .. hs0), so the w = 0 kernel sums to 1.  The
// degridding tables are the complex conjugates.  The sums run in double on
// the GPU (M terms per sample); the tables are rounded to float.
//
// Dirty PSF: unit visibilities gridded with a plan, transformed and
// taper-corrected exactly as a major cycle images them, then normalised by
// the maximum as psf_host_set_up does with the PSF it reads (top.c:481-509).
#include <cmath>

#include <algorithm>
#include <vector>

#include "internal.cuh"

namespace sdp {

// 1-D kernel samples k_p(s) (double complex), one block per (s, plane).
__global__ void k_wkernel_1d(int M, int OS, double fov, double max_w, int P, const int *__restrict__ n1,
                             double2 *__restrict__ out, int stride)
{
    const int s = blockIdx.x, p = blockIdx.y;
    if (s >= n1[p]) return;
    const double w = P > 1 ? (double)p * p * max_w / ((double)(P - 1) * (P - 1)) : 0.0;
    double re = 0.0, im = 0.0;
    for (int j = threadIdx.x; j < M; j += blockDim.x) {
        const double l = (double)(j - M / 2) * (fov / M);
        const double t = prolate_schwab(fabs(2.0 * l / fov));
        // phase in turns: -(w l^2 / 2) - s (j - M/2) / (M OS)
        const double turns = -0.5 * w * l * l - (double)s * (double)(j - M / 2) / ((double)M * OS);
        double sn, cs;
        sincospi(2.0 * turns, &sn, &cs);
        re += t * cs;
        im += t * sn;
    }
    __shared__ double sre[256], sim[256];
    sre[threadIdx.x] = re;
    sim[threadIdx.x] = im;
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
        if ((int)threadIdx.x < o) {
            sre[threadIdx.x] += sre[threadIdx.x + o];
            sim[threadIdx.x] += sim[threadIdx.x + o];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) out[(size_t)p * stride + s] = make_double2(sre[0], sim[0]);
}

// Normalisation: Re sum over t in [-hs0, hs0] of the w = 0 kernel at uv
// offset t cells, k_0(t OS) (k_0(-s) is the sum with the opposite sign of s).
__global__ void k_wkernel_norm(int M, int OS, double fov, int hs0, double *norm)
{
    double acc = 0.0;
    for (int t = -hs0; t <= hs0; ++t) {
        double re = 0.0;
        for (int j = threadIdx.x; j < M; j += blockDim.x) {
            const double l = (double)(j - M / 2) * (fov / M);
            const double tap = prolate_schwab(fabs(2.0 * l / fov));
            re += tap * cospi(-2.0 * (double)t * OS * (double)(j - M / 2) / ((double)M * OS));
        }
        acc += re;
    }
    __shared__ double s[256];
    s[threadIdx.x] = acc;
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
        if ((int)threadIdx.x < o) s[threadIdx.x] += s[threadIdx.x + o];
        __syncthreads();
    }
    if (threadIdx.x == 0) *norm = s[0];
}

// Quarter-plane tables: sample (a, b) of plane p = k(a) k(b) / norm^2.
__global__ void k_wkernel_outer(int P, const int *__restrict__ n1, const int *__restrict__ off,
                                const double2 *__restrict__ k1, int stride, const double *__restrict__ norm,
                                float2 *__restrict__ gk, float2 *__restrict__ dk)
{
    const int p = blockIdx.y;
    const int n = n1[p];
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n * n) return;
    const int a = i / n, b = i % n;
    const double nn = *norm;
    const double2 x = k1[(size_t)p * stride + a], y = k1[(size_t)p * stride + b];
    const double re = (x.x * y.x - x.y * y.y) / (nn * nn);
    const double im = (x.x * y.y + x.y * y.x) / (nn * nn);
    const size_t o = (size_t)off[p] + i;
    gk[o] = make_float2((float)re, (float)im);
    if (dk) dk[o] = make_float2((float)re, (float)-im);
}

__global__ void k_fill_unit(int n, float2 *v)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) v[i] = make_float2(1.f, 0.f);
}

// max over the image (one block, then every pixel divided by it in double,
// rounded to float: psf[i] /= *psf_max_value, top.c:506-509)
__global__ void k_max_reduce(size_t n, const float *__restrict__ x, double *out)
{
    __shared__ float s[1024];
    float m = 0.f;  // psf_max_value starts at 0 (the reference's caller passes 0)
    for (size_t i = threadIdx.x; i < n; i += blockDim.x) m = fmaxf(m, x[i]);
    s[threadIdx.x] = m;
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
        if ((int)threadIdx.x < o) s[threadIdx.x] = fmaxf(s[threadIdx.x], s[threadIdx.x + o]);
        __syncthreads();
    }
    if (threadIdx.x == 0) *out = (double)s[0];
}

__global__ void k_normalise(size_t n, float *x, const double *mx)
{
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) x[i] = (float)((double)x[i] / *mx);
}

// Sum of x^2 over n floats in FP64 (one block; deterministic order): each
// thread keeps four accumulators over 16-byte loads (memory-level
// parallelism for a single SM), then a fixed tree.
__global__ void __launch_bounds__(1024) k_sum_sq(size_t n, const float *__restrict__ x, double *out)
{
    __shared__ double s[1024];
    double a0 = 0.0, a1 = 0.0, a2 = 0.0, a3 = 0.0;
    size_t head = 0;
    if ((reinterpret_cast<uintptr_t>(x) & 15) == 0) {
        const size_t n4 = n / 4;
        const float4 *x4 = reinterpret_cast<const float4 *>(x);
        size_t i = threadIdx.x;
        for (; i + 3 * blockDim.x < n4; i += 4 * blockDim.x) {
            const float4 p = __ldg(x4 + i), q = __ldg(x4 + i + blockDim.x);
            const float4 r = __ldg(x4 + i + 2 * blockDim.x), t = __ldg(x4 + i + 3 * blockDim.x);
            a0 = fma((double)p.x, (double)p.x, fma((double)p.y, (double)p.y, a0));
            a1 = fma((double)p.z, (double)p.z, fma((double)p.w, (double)p.w, a1));
            a2 = fma((double)q.x, (double)q.x, fma((double)q.y, (double)q.y, a2));
            a3 = fma((double)q.z, (double)q.z, fma((double)q.w, (double)q.w, a3));
            a0 = fma((double)r.x, (double)r.x, fma((double)r.y, (double)r.y, a0));
            a1 = fma((double)r.z, (double)r.z, fma((double)r.w, (double)r.w, a1));
            a2 = fma((double)t.x, (double)t.x, fma((double)t.y, (double)t.y, a2));
            a3 = fma((double)t.z, (double)t.z, fma((double)t.w, (double)t.w, a3));
        }
        for (; i < n4; i += blockDim.x) {
            const float4 p = __ldg(x4 + i);
            a0 = fma((double)p.x, (double)p.x, fma((double)p.y, (double)p.y, a0));
            a1 = fma((double)p.z, (double)p.z, fma((double)p.w, (double)p.w, a1));
        }
        head = n4 * 4;
    }
    for (size_t i = head + threadIdx.x; i < n; i += blockDim.x) a0 = fma((double)x[i], (double)x[i], a0);
    s[threadIdx.x] = (a0 + a1) + (a2 + a3);
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
        if ((int)threadIdx.x < o) s[threadIdx.x] += s[threadIdx.x + o];
        __syncthreads();
    }
    if (threadIdx.x == 0) *out = sqrt(s[0] / (double)(n ? n : 1));
}

}  // namespace sdp

using namespace sdp;

SDP_EXPORT int sdp_image_rms(int grid_size, const float *image, double *rms_dev, void *stream)
{
    SDP_CHECK_ARG(grid_size >= 1 && image && rms_dev, "bad argument");
    k_sum_sq<<<1, 1024, 0, as_stream(stream)>>>((size_t)grid_size * grid_size, image, rms_dev);
    SDP_LAUNCH_CHECK();
    return SDP_OK;
}

SDP_EXPORT int sdp_wkernels_generate_sizes(int num_planes, const int *half_supports, int oversampling,
                                           int *total_samples)
{
    SDP_CHECK_ARG(num_planes >= 1 && half_supports && oversampling >= 1 && total_samples, "bad argument");
    long long t = 0;
    for (int p = 0; p < num_planes; ++p) {
        SDP_CHECK_ARG(half_supports[p] >= 0, "negative half support at plane %d", p);
        const long long n = (long long)(half_supports[p] + 1) * oversampling;
        t += n * n;
    }
    SDP_CHECK_ARG(t < (1LL << 31), "kernel tables too large");
    *total_samples = (int)t;
    return SDP_OK;
}

SDP_EXPORT int sdp_wkernels_generate(int num_planes, const int *half_supports, int oversampling, double max_w,
                                     double fov_rad, int image_samples, sdp_float2 *grid_kernels,
                                     sdp_float2 *degrid_kernels, sdp_int2 *supports, void *scratch,
                                     size_t scratch_bytes, void *stream)
{
    SDP_CHECK_ARG(num_planes >= 1 && half_supports && oversampling >= 1 && grid_kernels && supports && scratch,
                  "bad argument");
    SDP_CHECK_ARG(image_samples >= 2 && image_samples % 2 == 0, "image_samples %d: an even count >= 2 required",
                  image_samples);
    SDP_CHECK_ARG(fov_rad > 0.0 && max_w >= 0.0, "fov %g / max_w %g", fov_rad, max_w);
    int total = 0;
    SDP_TRY(sdp_wkernels_generate_sizes(num_planes, half_supports, oversampling, &total));
    int nmax = 0;
    std::vector<int> n1((size_t)num_planes), off((size_t)num_planes);
    std::vector<sdp_int2> sup((size_t)num_planes);
    int o = 0;
    for (int p = 0; p < num_planes; ++p) {
        n1[(size_t)p] = (half_supports[p] + 1) * oversampling;
        nmax = std::max(nmax, n1[(size_t)p]);
        off[(size_t)p] = o;
        sup[(size_t)p] = sdp_int2{half_supports[p], o};
        o += n1[(size_t)p] * n1[(size_t)p];
    }
    const size_t need = 64 + sizeof(int) * 2 * (size_t)num_planes + 64 + sizeof(double2) * (size_t)num_planes * nmax;
    if (scratch_bytes < need) return set_error(SDP_ERR_RANGE, "kernel generation scratch %zu B < %zu B", scratch_bytes, need);
    cudaStream_t st = as_stream(stream);
    char *w = static_cast<char *>(scratch);
    double *norm = reinterpret_cast<double *>(w);
    int *d_n1 = reinterpret_cast<int *>(w + 64);
    int *d_off = d_n1 + num_planes;
    double2 *k1 = reinterpret_cast<double2 *>(w + 64 + ((sizeof(int) * 2 * (size_t)num_planes + 63) / 64) * 64);
    SDP_CUDA_TRY(cudaMemcpyAsync(d_n1, n1.data(), sizeof(int) * num_planes, cudaMemcpyHostToDevice, st));
    SDP_CUDA_TRY(cudaMemcpyAsync(d_off, off.data(), sizeof(int) * num_planes, cudaMemcpyHostToDevice, st));
    SDP_CUDA_TRY(cudaMemcpyAsync(supports, sup.data(), sizeof(sdp_int2) * num_planes, cudaMemcpyDefault, st));
    k_wkernel_1d<<<dim3(nmax, num_planes), 256, 0, st>>>(image_samples, oversampling, fov_rad, max_w, num_planes, d_n1,
                                                         k1, nmax);
    k_wkernel_norm<<<1, 256, 0, st>>>(image_samples, oversampling, fov_rad, half_supports[0], norm);
    k_wkernel_outer<<<dim3((nmax * nmax + 255) / 256, num_planes), 256, 0, st>>>(
        num_planes, d_n1, d_off, k1, nmax, norm, reinterpret_cast<float2 *>(grid_kernels),
        reinterpret_cast<float2 *>(degrid_kernels));
    SDP_LAUNCH_CHECK();
    SDP_CUDA_TRY(cudaStreamSynchronize(st));  // the host arrays above are released on return
    return SDP_OK;
}

SDP_EXPORT size_t sdp_wkernels_generate_scratch_bytes(int num_planes, const int *half_supports, int oversampling)
{
    int nmax = 0;
    for (int p = 0; p < num_planes; ++p) nmax = std::max(nmax, (half_supports[p] + 1) * oversampling);
    return 64 + sizeof(int) * 2 * (size_t)num_planes + 64 + sizeof(double2) * (size_t)num_planes * nmax;
}

SDP_EXPORT int sdp_psf_generate(sdp_visplan *plan, const float *prolate_ext, sdp_float2 *unit_vis_scratch,
                                sdp_float2 *grid_scratch, sdp_float2 *work, float *psf, double *psf_max_dev,
                                void *stream)
{
    SDP_CHECK_ARG(plan && prolate_ext && grid_scratch && work && psf && psf_max_dev && (unit_vis_scratch || plan->n == 0),
                  "NULL argument");
    cudaStream_t st = as_stream(stream);
    const int G = plan->geom.grid_size;
    const size_t G2 = (size_t)G * G;
    if (plan->n > 0) {
        k_fill_unit<<<(plan->n + 255) / 256, 256, 0, st>>>(plan->n, reinterpret_cast<float2 *>(unit_vis_scratch));
        SDP_LAUNCH_CHECK();
    }
    SDP_TRY(sdp_visplan_grid(plan, unit_vis_scratch, grid_scratch, 0, st));
    SDP_TRY(sdp_grid_to_image(G, grid_scratch, prolate_ext, work, psf, st));
    k_max_reduce<<<1, 1024, 0, st>>>(G2, psf, psf_max_dev);
    k_normalise<<<(unsigned)((G2 + 255) / 256), 256, 0, st>>>(G2, psf, psf_max_dev);
    SDP_LAUNCH_CHECK();
    return SDP_OK;
}
