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

}  // namespace sdp

using namespace sdp;

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
