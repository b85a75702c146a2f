// Device kernels of the learned major cycle (no counterpart in the
// reference): the network's input planes from a residual image, the choice
// of the proposed components (the largest positive values of the network's
// output), the exact line search of a proposal against the residual, and the
// synthetic skies (points and circular Gaussians) that the training pairs
// are made from, with their visibilities.
//
// Image convention (the one the DFT predict, the gridder and Hogbom share,
// deconvolution_run.c:300-306): pixel (x, y) of a G x G image is the
// direction l = (x - G/2) * cell, m = (y - G/2) * cell.
#include <cmath>

#include "common.cuh"

namespace sdp {
namespace {

constexpr int kThreads = 256;
constexpr int kHistBins = 2048;

inline int blocks_for(long long n)
{
    long long b = (n + kThreads - 1) / kThreads;
    const long long cap = (long long)num_sms() * 16;
    return (int)(b < 1 ? 1 : (b > cap ? cap : b));
}

// Non-negative float max via the ordered integer view (valid for x >= 0).
__device__ __forceinline__ void atomic_max_nonneg(float *addr, float x)
{
    atomicMax(reinterpret_cast<int *>(addr), __float_as_int(x));
}

__global__ void k_absmax(long long n, const float *__restrict__ x, float *__restrict__ out)
{
    float m = 0.f;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x)
        m = fmaxf(m, fabsf(x[i]));
    for (int off = 16; off; off >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, off));
    if ((threadIdx.x & 31) == 0) atomic_max_nonneg(out, m);
}

// planes[0] = r / s, planes[1] = sign(r) sqrt(|r| / s), planes[2] = psf,
// s = max |r| (1 when the residual is zero).
__global__ void k_planes(long long n, const float *__restrict__ r, const float *__restrict__ psf,
                         const float *__restrict__ smax, float *__restrict__ planes)
{
    const float s = smax[0] > 0.f ? smax[0] : 1.f;
    const float inv = 1.f / s;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x) {
        const float v = r[i] * inv;
        planes[i] = v;
        planes[n + i] = copysignf(sqrtf(fabsf(v)), v);
        planes[2 * n + i] = psf[i];
    }
}

// The same planes for the centred window of side W of a G x G residual and
// PSF (offset o = (G - W) / 2 in both axes); s is still the whole image's
// max |r|.
__global__ void k_planes_window(int G, int W, const float *__restrict__ r, const float *__restrict__ psf,
                                const float *__restrict__ smax, float *__restrict__ planes)
{
    const float s = smax[0] > 0.f ? smax[0] : 1.f;
    const float inv = 1.f / s;
    const long long n = (long long)W * W;
    const int o = (G - W) / 2;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x) {
        const int y = (int)(i / W), x = (int)(i - (long long)y * W);
        const long long src = (long long)(y + o) * G + (x + o);
        const float v = r[src] * inv;
        planes[i] = v;
        planes[n + i] = copysignf(sqrtf(fabsf(v)), v);
        planes[2 * n + i] = psf[src];
    }
}

// Largest value (signed = 0: of the positive values; 1: of |x|).
__device__ __forceinline__ float sel_key(float v, int signed_values) { return signed_values ? fabsf(v) : v; }

__global__ void k_pos_max(long long n, const float *__restrict__ x, int signed_values, float *__restrict__ out)
{
    float m = 0.f;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x)
        m = fmaxf(m, sel_key(x[i], signed_values));  // fmaxf drops NaN
    for (int off = 16; off; off >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, off));
    if ((threadIdx.x & 31) == 0) atomic_max_nonneg(out, m);
}

struct SelectWs {
    float vmax;       // largest positive value
    float thr;        // chosen threshold
    int count;        // candidates written (capped at max_count by the reader)
    int pad;
    int hist[kHistBins];
};

// Histogram of the keys in [lo, vmax], lo = rel * vmax, in linear bins.
__global__ void k_hist(long long n, const float *__restrict__ x, int signed_values, float rel, SelectWs *ws)
{
    const float vmax = ws->vmax;
    if (!(vmax > 0.f)) return;
    const float lo = rel * vmax;
    const float scale = (float)kHistBins / fmaxf(vmax - lo, 1e-30f);
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x) {
        const float v = sel_key(x[i], signed_values);
        if (!(v >= lo) || !(v > 0.f)) continue;
        int b = (int)((v - lo) * scale);
        b = b < 0 ? 0 : (b >= kHistBins ? kHistBins - 1 : b);
        atomicAdd(&ws->hist[b], 1);
    }
}

// Lowest bin edge whose bins above hold at most max_count values (at least
// the top bin).
__global__ void k_threshold(float rel, int max_count, SelectWs *ws)
{
    const float vmax = ws->vmax;
    if (!(vmax > 0.f)) {
        ws->thr = INFINITY;
        return;
    }
    const float lo = rel * vmax;
    const float width = (vmax - lo) / (float)kHistBins;
    long long acc = 0;
    int b = kHistBins - 1;
    for (; b >= 0; --b) {
        if (acc + ws->hist[b] > max_count && b < kHistBins - 1) break;
        acc += ws->hist[b];
    }
    // bins b + 1 .. top are kept
    ws->thr = (b < 0) ? lo : lo + width * (float)(b + 1);
    if (ws->thr <= 0.f) ws->thr = 1e-30f;
}

__global__ void k_compact(int G, double cell, const float *__restrict__ x, int signed_values,
                          const float *__restrict__ sval, int max_count, SelectWs *ws, float4 *__restrict__ comps,
                          float *__restrict__ delta)
{
    const float thr = ws->thr;
    const float s = sval ? sval[0] : 1.f;
    const long long n = (long long)G * G;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x) {
        const float v = x[i];
        if (!(sel_key(v, signed_values) >= thr)) continue;
        const int slot = atomicAdd(&ws->count, 1);
        if (slot >= max_count) continue;
        const int yy = (int)(i / G), xx = (int)(i - (long long)yy * G);
        const float f = v * s;
        comps[slot] = make_float4((float)((xx - G / 2) * cell), (float)((yy - G / 2) * cell), f, 0.f);
        if (delta) delta[i] = f;
    }
}

__global__ void k_clamp_count(int max_count, SelectWs *ws, int *count_out)
{
    const int c = ws->count;
    count_out[0] = c < max_count ? c : max_count;
}

// FP64 <a, b> and <b, b>.
__global__ void __launch_bounds__(kThreads) k_dots(long long n, const float *__restrict__ a,
                                                  const float *__restrict__ b, double *__restrict__ out)
{
    __shared__ double s_ab[kThreads / 32], s_bb[kThreads / 32];
    double ab = 0.0, bb = 0.0;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x) {
        const double x = a[i], y = b[i];
        ab += x * y;
        bb += y * y;
    }
    for (int off = 16; off; off >>= 1) {
        ab += __shfl_xor_sync(0xffffffffu, ab, off);
        bb += __shfl_xor_sync(0xffffffffu, bb, off);
    }
    if ((threadIdx.x & 31) == 0) {
        s_ab[threadIdx.x >> 5] = ab;
        s_bb[threadIdx.x >> 5] = bb;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double x = 0.0, y = 0.0;
        for (int k = 0; k < kThreads / 32; ++k) {
            x += s_ab[k];
            y += s_bb[k];
        }
        atomicAdd(out, x);
        atomicAdd(out + 1, y);
    }
}

__device__ __forceinline__ float ratio_alpha(const double *dots, double alpha_max)
{
    const double ab = dots[0], bb = dots[1];
    double a = (bb > 0.0) ? ab / bb : 0.0;
    a = a < 0.0 ? 0.0 : (a > alpha_max ? alpha_max : a);
    return (float)a;
}

// y += sign alpha x, alpha = clamp(<a,b>/<b,b>, 0, alpha_max) from dots.
__global__ void k_axpy_ratio(long long n, const double *__restrict__ dots, double alpha_max, float sign,
                             const float *__restrict__ x, float *__restrict__ y, float *__restrict__ alpha_out)
{
    const float a = ratio_alpha(dots, alpha_max);
    if (alpha_out && blockIdx.x == 0 && threadIdx.x == 0) alpha_out[0] = a;
    const float sa = sign * a;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x)
        y[i] = fmaf(sa, x[i], y[i]);
}

__global__ void k_scale(long long n, float *__restrict__ x, float f)
{
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x)
        x[i] *= f;
}

// One block per component: points (sigma == 0) add their flux to the
// nearest pixel; circular Gaussians add flux / (2 pi s^2) exp(-r^2 / (2 s^2))
// (s in pixels) over +-4 s around their centre.
__global__ void k_render(int G, double cell, int num, const float4 *__restrict__ comps, float *__restrict__ image)
{
    const float4 c = comps[blockIdx.x];
    const double xc = (double)c.x / cell + G / 2, yc = (double)c.y / cell + G / 2;
    if (c.w <= 0.f) {
        if (threadIdx.x == 0) {
            const long long xi = llrint(xc), yi = llrint(yc);
            if (xi >= 0 && xi < G && yi >= 0 && yi < G) atomicAdd(image + yi * G + xi, c.z);
        }
        return;
    }
    const double s = (double)c.w / cell;
    const int R = (int)fmin(ceil(4.0 * s), (double)G);
    const int side = 2 * R + 1;
    const double norm = (double)c.z / (2.0 * M_PI * s * s);
    const long long x0 = llrint(xc), y0 = llrint(yc);
    for (int k = threadIdx.x; k < side * side; k += blockDim.x) {
        const long long xx = x0 - R + k % side, yy = y0 - R + k / side;
        if (xx < 0 || xx >= G || yy < 0 || yy >= G) continue;
        const double dx = xx - xc, dy = yy - yc;
        atomicAdd(image + yy * G + xx, (float)(norm * exp(-(dx * dx + dy * dy) / (2.0 * s * s))));
    }
}

// Zeroes the pixels within `border` of the edge of a G x G image (only the
// border band is visited: 4 strips of border x G).
__global__ void k_zero_border(int G, int border, float *__restrict__ image)
{
    const long long strip = (long long)border * G;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < 4 * strip;
         i += (long long)gridDim.x * blockDim.x) {
        const int which = (int)(i / strip);
        const long long k = i - which * strip;
        const int a = (int)(k / G), b = (int)(k - (long long)a * G);  // a: 0..border-1, b: 0..G-1
        long long px;
        if (which == 0) px = (long long)a * G + b;                    // top rows
        else if (which == 1) px = (long long)(G - 1 - a) * G + b;     // bottom rows
        else if (which == 2) px = (long long)b * G + a;               // left columns
        else px = (long long)b * G + (G - 1 - a);                     // right columns
        image[px] = 0.f;
    }
}

}  // namespace
}  // namespace sdp

using namespace sdp;

SDP_EXPORT int sdp_zero_border(int grid_size, int border, float *image, void *stream)
{
    SDP_CHECK_ARG(grid_size > 0 && border >= 0, "invalid size");
    SDP_CHECK_ARG(image, "NULL argument");
    if (border == 0) return SDP_OK;
    if (2 * border >= grid_size) {
        SDP_CUDA_TRY(cudaMemsetAsync(image, 0, sizeof(float) * (size_t)grid_size * grid_size, as_stream(stream)));
        return SDP_OK;
    }
    const long long n = 4LL * border * grid_size;
    k_zero_border<<<blocks_for(n), kThreads, 0, as_stream(stream)>>>(grid_size, border, image);
    SDP_LAUNCH_CHECK();
    return SDP_OK;
}

SDP_EXPORT int sdp_unet_input_planes(int grid_size, const float *residual, const float *psf, float *planes,
                                     float *scale_dev, void *stream)
{
    SDP_CHECK_ARG(grid_size > 0, "grid_size must be positive");
    SDP_CHECK_ARG(residual && psf && planes && scale_dev, "NULL argument");
    cudaStream_t st = as_stream(stream);
    const long long n = (long long)grid_size * grid_size;
    SDP_CUDA_TRY(cudaMemsetAsync(scale_dev, 0, sizeof(float), st));
    k_absmax<<<blocks_for(n), kThreads, 0, st>>>(n, residual, scale_dev);
    SDP_LAUNCH_CHECK();
    k_planes<<<blocks_for(n), kThreads, 0, st>>>(n, residual, psf, scale_dev, planes);
    SDP_LAUNCH_CHECK();
    return SDP_OK;
}

SDP_EXPORT int sdp_unet_input_planes_window(int grid_size, int window, const float *residual, const float *psf,
                                            float *planes, float *scale_dev, void *stream)
{
    SDP_CHECK_ARG(grid_size > 0 && window > 0 && window <= grid_size && (grid_size - window) % 2 == 0,
                  "window %d must be positive, at most grid_size %d and of the same parity", window, grid_size);
    SDP_CHECK_ARG(residual && psf && planes && scale_dev, "NULL argument");
    cudaStream_t st = as_stream(stream);
    const long long n = (long long)grid_size * grid_size, nw = (long long)window * window;
    SDP_CUDA_TRY(cudaMemsetAsync(scale_dev, 0, sizeof(float), st));
    k_absmax<<<blocks_for(n), kThreads, 0, st>>>(n, residual, scale_dev);
    SDP_LAUNCH_CHECK();
    k_planes_window<<<blocks_for(nw), kThreads, 0, st>>>(grid_size, window, residual, psf, scale_dev, planes);
    SDP_LAUNCH_CHECK();
    return SDP_OK;
}

SDP_EXPORT int sdp_select_workspace_bytes(size_t *bytes)
{
    SDP_CHECK_ARG(bytes, "NULL argument");
    *bytes = sizeof(SelectWs);
    return SDP_OK;
}

SDP_EXPORT int sdp_select_components(int grid_size, double cell_size, const float *proposal, const float *scale_dev,
                                     int signed_values, float rel_threshold, int max_count, sdp_float4 *components,
                                     int *count_dev, float *delta_image, void *workspace, void *stream)
{
    SDP_CHECK_ARG(grid_size > 0 && max_count >= 0, "invalid size");
    SDP_CHECK_ARG(rel_threshold >= 0.f && rel_threshold < 1.f, "rel_threshold must be in [0, 1)");
    SDP_CHECK_ARG(proposal && components && count_dev && workspace, "NULL argument");
    cudaStream_t st = as_stream(stream);
    const long long n = (long long)grid_size * grid_size;
    SelectWs *ws = static_cast<SelectWs *>(workspace);
    SDP_CUDA_TRY(cudaMemsetAsync(ws, 0, sizeof(SelectWs), st));
    if (delta_image) SDP_CUDA_TRY(cudaMemsetAsync(delta_image, 0, n * sizeof(float), st));
    const int sv = signed_values ? 1 : 0;
    k_pos_max<<<blocks_for(n), kThreads, 0, st>>>(n, proposal, sv, &ws->vmax);
    SDP_LAUNCH_CHECK();
    k_hist<<<blocks_for(n), kThreads, 0, st>>>(n, proposal, sv, rel_threshold, ws);
    SDP_LAUNCH_CHECK();
    k_threshold<<<1, 1, 0, st>>>(rel_threshold, max_count, ws);
    SDP_LAUNCH_CHECK();
    k_compact<<<blocks_for(n), kThreads, 0, st>>>(grid_size, cell_size, proposal, sv, scale_dev, max_count, ws,
                                                  reinterpret_cast<float4 *>(components), delta_image);
    SDP_LAUNCH_CHECK();
    k_clamp_count<<<1, 1, 0, st>>>(max_count, ws, count_dev);
    SDP_LAUNCH_CHECK();
    return SDP_OK;
}

SDP_EXPORT int sdp_dots(long long n, const float *a, const float *b, double *dots_dev, void *stream)
{
    SDP_CHECK_ARG(n >= 0, "negative size");
    SDP_CHECK_ARG(a && b && dots_dev, "NULL argument");
    cudaStream_t st = as_stream(stream);
    SDP_CUDA_TRY(cudaMemsetAsync(dots_dev, 0, 2 * sizeof(double), st));
    if (n == 0) return SDP_OK;
    k_dots<<<blocks_for(n), kThreads, 0, st>>>(n, a, b, dots_dev);
    SDP_LAUNCH_CHECK();
    return SDP_OK;
}

SDP_EXPORT int sdp_axpy_ratio(long long n, const double *dots_dev, double alpha_max, float sign, const float *x,
                              float *y, float *alpha_dev, void *stream)
{
    SDP_CHECK_ARG(n >= 0 && alpha_max >= 0.0, "invalid argument");
    SDP_CHECK_ARG(dots_dev && x && y, "NULL argument");
    k_axpy_ratio<<<blocks_for(n > 0 ? n : 1), kThreads, 0, as_stream(stream)>>>(n, dots_dev, alpha_max, sign, x,
                                                                                 y, alpha_dev);
    SDP_LAUNCH_CHECK();
    return SDP_OK;
}

SDP_EXPORT int sdp_scale(long long n, float *x, float factor, void *stream)
{
    SDP_CHECK_ARG(n >= 0 && x, "invalid argument");
    if (n == 0) return SDP_OK;
    k_scale<<<blocks_for(n), kThreads, 0, as_stream(stream)>>>(n, x, factor);
    SDP_LAUNCH_CHECK();
    return SDP_OK;
}

SDP_EXPORT int sdp_sky_render(int grid_size, double cell_size, int num, const sdp_float4 *components, float *image,
                              void *stream)
{
    SDP_CHECK_ARG(grid_size > 0 && num >= 0 && cell_size > 0.0, "invalid size");
    SDP_CHECK_ARG(image && (components || num == 0), "NULL argument");
    if (num == 0) return SDP_OK;
    k_render<<<num, kThreads, 0, as_stream(stream)>>>(grid_size, cell_size, num,
                                                     reinterpret_cast<const float4 *>(components), image);
    SDP_LAUNCH_CHECK();
    return SDP_OK;
}
