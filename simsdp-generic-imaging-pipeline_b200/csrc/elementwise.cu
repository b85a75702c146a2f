// Element-wise device kernels of the imaging cycle.  These are HBM-bound;
// each is a grid-stride loop over 16-byte (two-complex) or 8-byte items with
// a grid sized to a multiple of the SM count.
#include <algorithm>

#include "internal.cuh"

namespace sdp {

static inline int ew_grid(size_t n, int threads = 256)
{
    size_t blocks = (n + threads - 1) / threads;
    size_t cap = (size_t)num_sms() * 16;
    return (int)std::max<size_t>(1, std::min(blocks, cap));
}

#define GRID_STRIDE(i, n)                                                         \
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < (size_t)(n); \
         i += (size_t)gridDim.x * blockDim.x)

// degridgrid.c:194-200: nearest grid cell (out-of-grid positions read 0).
__global__ void k_degrid_nearest(int G, double uv_scale, int n, const float3 *__restrict__ uvw,
                                 const float2 *__restrict__ grid, float2 *__restrict__ out)
{
    const int gc = G / 2;
    GRID_STRIDE(i, n)
    {
        float3 c = uvw[i];
        int x = ref_nearest(ref_grid_pos(c.x, uv_scale), gc);
        int y = ref_nearest(ref_grid_pos(c.y, uv_scale), gc);
        long long gi = (long long)x + (long long)y * G;
        out[i] = (gi >= 0 && gi < (long long)G * G) ? grid[gi] : make_float2(0.f, 0.f);
    }
}

// degridgrid.c:24-25, 52-54 (simplification off): snap to the 1/OS fine grid.
__global__ void k_correct_to_finegrid(int G, int OS, double uv_scale, int n, const float3 *__restrict__ uvw,
                                      float3 *__restrict__ out)
{
    const double half = (double)(G / 2);
    GRID_STRIDE(i, n)
    {
        float3 c = uvw[i];
        double tx = __dadd_rn(__dmul_rn(__dadd_rn(__dmul_rn((double)c.x, uv_scale), half), (double)OS), 0.5);
        double ty = __dadd_rn(__dmul_rn(__dadd_rn(__dmul_rn((double)c.y, uv_scale), half), (double)OS), 0.5);
        long long fx = __double2ll_rz(tx), fy = __double2ll_rz(ty);
        float3 o;
        o.x = __double2float_rn(__ddiv_rn(__dsub_rn(__ddiv_rn((double)fx, (double)OS), half), uv_scale));
        o.y = __double2float_rn(__ddiv_rn(__dsub_rn(__ddiv_rn((double)fy, (double)OS), half), uv_scale));
        o.z = c.z;
        out[i] = o;
    }
}

__global__ void k_sub2(int n, const float2 *__restrict__ a, const float2 *__restrict__ b, float2 *__restrict__ o)
{
    GRID_STRIDE(i, n)
    {
        float2 x = a[i], y = b[i];
        o[i] = make_float2(__fsub_rn(x.x, y.x), __fsub_rn(x.y, y.y));
    }
}

__global__ void k_add2(int n, const float2 *__restrict__ a, const float2 *__restrict__ b, float2 *__restrict__ o)
{
    GRID_STRIDE(i, n)
    {
        float2 x = a[i], y = b[i];
        o[i] = make_float2(__fadd_rn(x.x, y.x), __fadd_rn(x.y, y.y));
    }
}

__global__ void k_sub1(size_t n, const float *__restrict__ a, const float *__restrict__ b, float *__restrict__ o)
{
    GRID_STRIDE(i, n) o[i] = __fsub_rn(a[i], b[i]);
}

// splitmerge.c:14-24: sum of SLICES grids, in slice order from 0.
__global__ void k_merge(size_t g2, int slices, const float2 *__restrict__ grids, float2 *__restrict__ out)
{
    GRID_STRIDE(i, g2)
    {
        float2 s = make_float2(0.f, 0.f);
        for (int j = 0; j < slices; ++j) {
            float2 t = grids[(size_t)j * g2 + i];
            s.x = __fadd_rn(s.x, t.x);
            s.y = __fadd_rn(s.y, t.y);
        }
        out[i] = s;
    }
}

// fft_run.c:5-20, 86-121: checkerboard sign (-1)^(row+col).
__global__ void k_shift_c2c(int G, const float2 *__restrict__ in, float2 *__restrict__ out)
{
    size_t g2 = (size_t)G * G;
    GRID_STRIDE(i, g2)
    {
        int r = (int)(i / G), c = (int)(i % G);
        float a = ((r + c) & 1) ? -1.f : 1.f;
        float2 x = in[i];
        out[i] = make_float2(x.x * a, x.y * a);
    }
}

__global__ void k_shift_c2r(int G, const float2 *__restrict__ in, float *__restrict__ out)
{
    size_t g2 = (size_t)G * G;
    GRID_STRIDE(i, g2)
    {
        int r = (int)(i / G), c = (int)(i % G);
        float a = ((r + c) & 1) ? -1.f : 1.f;
        out[i] = in[i].x * a;
    }
}

__global__ void k_shift_r2c(int G, const float *__restrict__ in, float2 *__restrict__ out)
{
    size_t g2 = (size_t)G * G;
    GRID_STRIDE(i, g2)
    {
        int r = (int)(i / G), c = (int)(i % G);
        float a = ((r + c) & 1) ? -1.f : 1.f;
        out[i] = make_float2(in[i] * a, 0.f);
    }
}

// convolution_correction_run.c:4-35.  prolate_ext[G/2] is 0 (see header).
__device__ __forceinline__ float taper_divide(float v, int r, int c, int G, const float *__restrict__ p)
{
    const int half = G / 2;
    const int dc = abs(c - half), dr = abs(r - half);
    float taper = __fmul_rn(p[dc], p[dr]);
    if (dc == 1229 || dr == 1229) taper = 0.f;
    return ((double)fabsf(taper) > 1E-10) ? __fdiv_rn(v, taper) : 0.f;
}

__global__ void k_conv_correction(int G, const float *__restrict__ in, const float *__restrict__ p,
                                  float *__restrict__ out)
{
    size_t g2 = (size_t)G * G;
    GRID_STRIDE(i, g2)
    {
        int r = (int)(i / G), c = (int)(i % G);
        out[i] = taper_divide(in[i], r, c, G, p);
    }
}


__global__ void k_prolate(int G, float *__restrict__ out)
{
    const int half = G / 2;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i <= half; i += gridDim.x * blockDim.x)
        out[i] = (i < half) ? __double2float_rn(prolate_schwab(__ddiv_rn((double)i, (double)half))) : 0.f;
}

}  // namespace sdp

using namespace sdp;

SDP_EXPORT int sdp_degrid_nearest(int grid_size, double uv_scale, int n, const sdp_float3 *uvw,
                                  const sdp_float2 *grid, sdp_float2 *out, void *stream)
{
    SDP_CHECK_ARG(n >= 0 && grid_size >= 2, "bad sizes");
    if (n == 0) return SDP_OK;
    SDP_CHECK_ARG(uvw && grid && out, "NULL argument");
    k_degrid_nearest<<<ew_grid(n), 256, 0, as_stream(stream)>>>(grid_size, uv_scale, n,
                                                               reinterpret_cast<const float3 *>(uvw),
                                                               reinterpret_cast<const float2 *>(grid),
                                                               reinterpret_cast<float2 *>(out));
    SDP_LAUNCH_CHECK();
    return SDP_OK;
}

SDP_EXPORT int sdp_correct_to_finegrid(int grid_size, int oversampling, double uv_scale, int n,
                                       const sdp_float3 *uvw, sdp_float3 *out, void *stream)
{
    SDP_CHECK_ARG(n >= 0 && grid_size >= 2 && oversampling >= 1, "bad sizes");
    if (n == 0) return SDP_OK;
    SDP_CHECK_ARG(uvw && out, "NULL argument");
    k_correct_to_finegrid<<<ew_grid(n), 256, 0, as_stream(stream)>>>(grid_size, oversampling, uv_scale, n,
                                                                    reinterpret_cast<const float3 *>(uvw),
                                                                    reinterpret_cast<float3 *>(out));
    SDP_LAUNCH_CHECK();
    return SDP_OK;
}

SDP_EXPORT int sdp_subtract_vis(int n, const sdp_float2 *a, const sdp_float2 *b, sdp_float2 *o, void *stream)
{
    SDP_CHECK_ARG(n >= 0, "bad size");
    if (n == 0) return SDP_OK;
    SDP_CHECK_ARG(a && b && o, "NULL argument");
    k_sub2<<<ew_grid(n), 256, 0, as_stream(stream)>>>(n, reinterpret_cast<const float2 *>(a),
                                                     reinterpret_cast<const float2 *>(b),
                                                     reinterpret_cast<float2 *>(o));
    SDP_LAUNCH_CHECK();
    return SDP_OK;
}

SDP_EXPORT int sdp_add_vis(int n, const sdp_float2 *a, const sdp_float2 *b, sdp_float2 *o, void *stream)
{
    SDP_CHECK_ARG(n >= 0, "bad size");
    if (n == 0) return SDP_OK;
    SDP_CHECK_ARG(a && b && o, "NULL argument");
    k_add2<<<ew_grid(n), 256, 0, as_stream(stream)>>>(n, reinterpret_cast<const float2 *>(a),
                                                     reinterpret_cast<const float2 *>(b),
                                                     reinterpret_cast<float2 *>(o));
    SDP_LAUNCH_CHECK();
    return SDP_OK;
}

SDP_EXPORT int sdp_subtract_image(int G, const float *a, const float *b, float *o, void *stream)
{
    SDP_CHECK_ARG(G >= 1 && a && b && o, "bad argument");
    size_t n = (size_t)G * G;
    k_sub1<<<ew_grid(n), 256, 0, as_stream(stream)>>>(n, a, b, o);
    SDP_LAUNCH_CHECK();
    return SDP_OK;
}

SDP_EXPORT int sdp_merge_grids(int G, int slices, const sdp_float2 *grids, sdp_float2 *out, void *stream)
{
    SDP_CHECK_ARG(G >= 1 && slices >= 0 && grids && out, "bad argument");
    size_t n = (size_t)G * G;
    k_merge<<<ew_grid(n), 256, 0, as_stream(stream)>>>(n, slices, reinterpret_cast<const float2 *>(grids),
                                                      reinterpret_cast<float2 *>(out));
    SDP_LAUNCH_CHECK();
    return SDP_OK;
}

SDP_EXPORT int sdp_fft_shift_c2c(int G, const sdp_float2 *in, sdp_float2 *out, void *stream)
{
    SDP_CHECK_ARG(G >= 1 && in && out, "bad argument");
    k_shift_c2c<<<ew_grid((size_t)G * G), 256, 0, as_stream(stream)>>>(G, reinterpret_cast<const float2 *>(in),
                                                                      reinterpret_cast<float2 *>(out));
    SDP_LAUNCH_CHECK();
    return SDP_OK;
}

SDP_EXPORT int sdp_fft_shift_c2r(int G, const sdp_float2 *in, float *out, void *stream)
{
    SDP_CHECK_ARG(G >= 1 && in && out, "bad argument");
    k_shift_c2r<<<ew_grid((size_t)G * G), 256, 0, as_stream(stream)>>>(G, reinterpret_cast<const float2 *>(in), out);
    SDP_LAUNCH_CHECK();
    return SDP_OK;
}

SDP_EXPORT int sdp_fft_shift_r2c(int G, const float *in, sdp_float2 *out, void *stream)
{
    SDP_CHECK_ARG(G >= 1 && in && out, "bad argument");
    k_shift_r2c<<<ew_grid((size_t)G * G), 256, 0, as_stream(stream)>>>(G, in, reinterpret_cast<float2 *>(out));
    SDP_LAUNCH_CHECK();
    return SDP_OK;
}

SDP_EXPORT int sdp_conv_correction(int G, const float *in, const float *prolate_ext, float *out, void *stream)
{
    SDP_CHECK_ARG(G >= 2 && G % 2 == 0 && in && prolate_ext && out, "bad argument");
    k_conv_correction<<<ew_grid((size_t)G * G), 256, 0, as_stream(stream)>>>(G, in, prolate_ext, out);
    SDP_LAUNCH_CHECK();
    return SDP_OK;
}

SDP_EXPORT int sdp_prolate_table(int G, float *prolate_ext, void *stream)
{
    SDP_CHECK_ARG(G >= 2 && G % 2 == 0 && prolate_ext, "bad argument");
    k_prolate<<<ew_grid((size_t)G / 2 + 1), 256, 0, as_stream(stream)>>>(G, prolate_ext);
    SDP_LAUNCH_CHECK();
    return SDP_OK;
}
