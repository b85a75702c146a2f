// DFT predict (dft_run.c:3-48, approximation branch :219-230):
//   V_i = sum_s I_s / (1 - r_s^2/2) * exp(-2 pi i (u l + v m - w r_s^2/2)),
//   r_s^2 = l^2 + m^2.
//
// Precision: the phase argument in cycles, t = u l + v m - w r^2/2, is formed
// in FP64 and reduced exactly to f = t - round(t) in [-1/2, 1/2]; sin/cos of
// 2 pi f are taken in FP32 with the hardware approximation (__sincosf, whose
// absolute error on [-pi, pi] is below 4e-7), and the per-source amplitude
// I / (1 - r^2/2) is formed in FP64 and rounded once.  Sums run in FP32
// (3.4e-7 rel-RMS against FP64 for 200 sources; sincospif gave 2.6e-7 at
// twice the time).
// The reference's float build evaluates the whole argument in float, whose
// error grows with |u l| (about |t| * 6e-8 rad per term); this path stays
// near FP32 rounding of the final sum for any baseline length.
//
// Sources are staged through shared memory in tiles; one thread owns one
// visibility and walks the tile.
#include "common.cuh"

namespace sdp {

constexpr int kDftThreads = 256;
constexpr int kDftTile = 512;

struct SrcTerm {
    double l, m, half_r2;
    float amp;
    float pad;
};

__global__ void __launch_bounds__(kDftThreads) k_dft(int n, int ns, const float3 *__restrict__ src,
                                                    const float3 *__restrict__ uvw, float2 *__restrict__ vis)
{
    __shared__ SrcTerm tile[kDftTile];
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    double u = 0, v = 0, w = 0;
    if (i < n) {
        const float3 c = uvw[i];
        u = c.x;
        v = c.y;
        w = c.z;
    }
    float sx = 0.f, sy = 0.f;
    for (int base = 0; base < ns; base += kDftTile) {
        const int cnt = min(kDftTile, ns - base);
        __syncthreads();
        for (int k = threadIdx.x; k < cnt; k += blockDim.x) {
            const float3 s = src[base + k];
            const double l = s.x, m = s.y;
            const double h = 0.5 * (l * l + m * m);
            SrcTerm t;
            t.l = l;
            t.m = m;
            t.half_r2 = h;
            t.amp = (float)((double)s.z / (1.0 - h));
            t.pad = 0.f;
            tile[k] = t;
        }
        __syncthreads();
        if (i < n) {
            for (int k = 0; k < cnt; ++k) {
                const SrcTerm t = tile[k];
                const double cyc = fma(u, t.l, fma(v, t.m, -w * t.half_r2));
                // cyc - nearest integer, exactly in double (adding and
                // subtracting 1.5 * 2^52 rounds to the nearest integer)
                const double kRound = 6755399441055744.0;
                const float f = (float)__dsub_rn(cyc, __dsub_rn(__dadd_rn(cyc, kRound), kRound));
                float s, c;
                __sincosf(6.28318530717958647692f * f, &s, &c);
                sx = fmaf(c, t.amp, sx);
                sy = fmaf(-s, t.amp, sy);
            }
        }
    }
    if (i < n) vis[i] = make_float2(sx, sy);
}

// Points and circular Gaussians (training skies of the learned major cycle;
// no counterpart in the reference): source s = (l, m, I, sigma) with sigma
// the Gaussian's standard deviation in direction cosines (0: a point).  The
// visibility of a circular Gaussian is the point term times
// exp(-2 pi^2 sigma^2 (u^2 + v^2)); the phase is formed and reduced as in
// k_dft.
struct SrcTermG {
    double l, m, half_r2;
    float amp;
    float g;  // 2 pi^2 sigma^2
};

__global__ void __launch_bounds__(kDftThreads) k_dft_gauss(int n, int ns, const float4 *__restrict__ src,
                                                          const float3 *__restrict__ uvw, float2 *__restrict__ vis)
{
    __shared__ SrcTermG tile[kDftTile];
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    double u = 0, v = 0, w = 0;
    if (i < n) {
        const float3 c = uvw[i];
        u = c.x;
        v = c.y;
        w = c.z;
    }
    const float q = (float)(u * u + v * v);
    float sx = 0.f, sy = 0.f;
    for (int base = 0; base < ns; base += kDftTile) {
        const int cnt = min(kDftTile, ns - base);
        __syncthreads();
        for (int k = threadIdx.x; k < cnt; k += blockDim.x) {
            const float4 s = src[base + k];
            const double l = s.x, m = s.y;
            const double h = 0.5 * (l * l + m * m);
            SrcTermG t;
            t.l = l;
            t.m = m;
            t.half_r2 = h;
            t.amp = (float)((double)s.z / (1.0 - h));
            t.g = (float)(2.0 * 9.869604401089358 * (double)s.w * (double)s.w);
            tile[k] = t;
        }
        __syncthreads();
        if (i < n) {
            for (int k = 0; k < cnt; ++k) {
                const SrcTermG t = tile[k];
                const double cyc = fma(u, t.l, fma(v, t.m, -w * t.half_r2));
                const double kRound = 6755399441055744.0;
                const float f = (float)__dsub_rn(cyc, __dsub_rn(__dadd_rn(cyc, kRound), kRound));
                float s, c;
                __sincosf(6.28318530717958647692f * f, &s, &c);
                const float a = t.g > 0.f ? t.amp * __expf(-t.g * q) : t.amp;
                sx = fmaf(c, a, sx);
                sy = fmaf(-s, a, sy);
            }
        }
    }
    if (i < n) vis[i] = make_float2(sx, sy);
}

// Components on the image's pixel grid (CLEAN components and network
// proposals; no counterpart in the reference, whose dft_actor takes any
// (l, m)): component k at pixel offset (X, Y) from the centre, l = X cell,
// m = Y cell.  The phase u l + v m - w (l^2 + m^2)/2 = U X + V Y - W R2 with
// U = u cell, V = v cell, W = w cell^2 / 2 (formed in FP64 per visibility)
// and R2 = X^2 + Y^2 is reduced modulo one cycle exactly in fixed point:
// frac(U) and frac(V) as 32-bit fractions (integer products wrap modulo 2^32,
// i.e. modulo one cycle; error <= |X| 2^-33 cycles) and W as a 44-bit
// fraction multiplied by R2 in 64 bits (error <= R2 2^-45 cycles).  The
// reduced phase (23 bits) becomes a float in [-1/2, 1/2) cycles by its bit
// pattern, so the only special-function work per term is the sine and the
// cosine (__sincosf on [-pi, pi)).
struct PixTerm {
    int x, y;
    unsigned r2;
    float amp;
};

constexpr int kPixTile = 1024;

__global__ void __launch_bounds__(kDftThreads) k_dft_pixels(int n, int ns, const float *__restrict__ comps, int stride,
                                                           double cell, const float3 *__restrict__ uvw,
                                                           float2 *__restrict__ vis, int accumulate)
{
    __shared__ PixTerm tile[kPixTile];
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    unsigned ufx = 0, vfx = 0;
    unsigned long long wfx = 0;
    bool wneg = false;
    if (i < n) {
        const float3 c = uvw[i];
        const double U = (double)c.x * cell, V = (double)c.y * cell;
        const double W = (double)c.z * cell * cell * 0.5;
        ufx = (unsigned)(long long)llrint((U - floor(U)) * 4294967296.0);
        vfx = (unsigned)(long long)llrint((V - floor(V)) * 4294967296.0);
        wneg = W < 0.0;
        wfx = (unsigned long long)llrint(fabs(W) * 17592186044416.0);  // 2^44
    }
    float sx = 0.f, sy = 0.f;
    const double inv_cell = 1.0 / cell;
    for (int base = 0; base < ns; base += kPixTile) {
        const int cnt = min(kPixTile, ns - base);
        __syncthreads();
        for (int k = threadIdx.x; k < cnt; k += blockDim.x) {
            const float *s = comps + (size_t)(base + k) * stride;
            PixTerm t;
            t.x = (int)llrint((double)s[0] * inv_cell);
            t.y = (int)llrint((double)s[1] * inv_cell);
            t.r2 = (unsigned)(t.x * t.x + t.y * t.y);
            const double h = 0.5 * (double)t.r2 * cell * cell;
            t.amp = (float)((double)s[2] / (1.0 - h));
            tile[k] = t;
        }
        __syncthreads();
        if (i < n) {
            // |W| 2^44 below 2^32 (|W| < 2^-12, the usual case): one 32 x 32 -> 64-bit product
            const bool w32 = (wfx >> 32) == 0ull;
            const unsigned wlo = (unsigned)wfx;
            for (int k = 0; k < cnt; ++k) {
                const PixTerm t = tile[k];
                // w term: frac(W R2) in units of 2^-32 cycles
                const unsigned long long wp =
                    w32 ? (unsigned long long)wlo * (unsigned long long)t.r2 : wfx * (unsigned long long)t.r2;
                unsigned wq = (unsigned)(wp >> 12);
                if (wneg) wq = 0u - wq;
                // phase U X + V Y - W R2 modulo 1, as a 32-bit fraction
                const unsigned p = ufx * (unsigned)t.x + vfx * (unsigned)t.y - wq;
                // [-1/2, 1/2) cycles from the top 23 bits (rounded): 1.5 + f as a float
                const float f = __uint_as_float(0x3F800000u | ((p + 0x80000100u) >> 9)) - 1.5f;
                float sn, cs;
                __sincosf(6.28318530717958647692f * f, &sn, &cs);
                sx = fmaf(cs, t.amp, sx);
                sy = fmaf(-sn, t.amp, sy);
            }
        }
    }
    if (i < n) {
        if (accumulate) {
            const float2 o = vis[i];
            vis[i] = make_float2(o.x + sx, o.y + sy);
        } else {
            vis[i] = make_float2(sx, sy);
        }
    }
}

}  // namespace sdp

using namespace sdp;

SDP_EXPORT int sdp_dft_pixels(int num_vis, int num_components, const float *components, int stride, double cell_size,
                              const sdp_float3 *uvw, sdp_float2 *vis, int accumulate, void *stream)
{
    SDP_CHECK_ARG(num_vis >= 0 && num_components >= 0, "negative size");
    SDP_CHECK_ARG(stride >= 3, "stride must be >= 3 floats (l, m, flux, ...)");
    SDP_CHECK_ARG(cell_size > 0.0, "cell_size must be positive");
    if (num_vis == 0) return SDP_OK;
    SDP_CHECK_ARG(uvw && vis && (components || num_components == 0), "NULL argument");
    k_dft_pixels<<<(num_vis + kDftThreads - 1) / kDftThreads, kDftThreads, 0, as_stream(stream)>>>(
        num_vis, num_components, components, stride, cell_size, reinterpret_cast<const float3 *>(uvw),
        reinterpret_cast<float2 *>(vis), accumulate ? 1 : 0);
    SDP_LAUNCH_CHECK();
    return SDP_OK;
}

SDP_EXPORT int sdp_dft_gauss(int num_vis, int num_sources, const sdp_float4 *sources, const sdp_float3 *uvw,
                             sdp_float2 *vis, void *stream)
{
    SDP_CHECK_ARG(num_vis >= 0 && num_sources >= 0, "negative size");
    if (num_vis == 0) return SDP_OK;
    SDP_CHECK_ARG(uvw && vis && (sources || num_sources == 0), "NULL argument");
    k_dft_gauss<<<(num_vis + kDftThreads - 1) / kDftThreads, kDftThreads, 0, as_stream(stream)>>>(
        num_vis, num_sources, reinterpret_cast<const float4 *>(sources), reinterpret_cast<const float3 *>(uvw),
        reinterpret_cast<float2 *>(vis));
    SDP_LAUNCH_CHECK();
    return SDP_OK;
}

SDP_EXPORT int sdp_dft(int num_vis, int num_sources, const sdp_float3 *sources, const sdp_float3 *uvw,
                       sdp_float2 *vis, void *stream)
{
    SDP_CHECK_ARG(num_vis >= 0 && num_sources >= 0, "negative size");
    if (num_vis == 0) return SDP_OK;
    SDP_CHECK_ARG(uvw && vis && (sources || num_sources == 0), "NULL argument");
    k_dft<<<(num_vis + kDftThreads - 1) / kDftThreads, kDftThreads, 0, as_stream(stream)>>>(
        num_vis, num_sources, reinterpret_cast<const float3 *>(sources), reinterpret_cast<const float3 *>(uvw),
        reinterpret_cast<float2 *>(vis));
    SDP_LAUNCH_CHECK();
    return SDP_OK;
}
