/*
 * ORACLE — test infrastructure only (see sdp_oracle.h).  CPU restatement of
 * the reference's imaging actors, written to keep the reference's C type
 * promotions: with REAL = float, expressions mixing REAL with the double
 * fields of the reference's Config (uv_scale, w_scale, loop_gain, ...) are
 * evaluated in double and rounded where the reference assigns to REAL.
 * Built with -ffp-contract=off so no multiply-add is fused.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include "sdp_oracle.h"
#include "fft_ref.h"

#ifdef ORACLE_DOUBLE
#define R_SQRT sqrt
#define R_ABS fabs
#define R_ROUND round
#define R_CEIL ceil
#define R_FLOOR floor
#define R_SIN sin
#define R_COS cos
#define R_PI ((double)3.1415926535897931)
#else
#define R_SQRT sqrtf
#define R_ABS fabsf
#define R_ROUND roundf
#define R_CEIL ceilf
#define R_FLOOR floorf
#define R_SIN sinf
#define R_COS cosf
#define R_PI ((float)3.141592654)
#endif

#define R_MIN(a, b) (((a) < (b)) ? (a) : (b))
#define R_MAX(a, b) (((a) > (b)) ? (a) : (b))

typedef struct { REAL x, y; } R2;
typedef struct { REAL x, y, z; } R3;
typedef struct { int x, y; } I2;

int or_real_size(void) { return (int)sizeof(REAL); }

/* degridgrid.c:5-8 */
static R2 cmul(R2 a, R2 b)
{
    R2 r;
    r.x = a.x * b.x - a.y * b.y;
    r.y = a.y * b.x + a.x * b.y;
    return r;
}

/* degridgrid.c:12-65, simplification off (the hash-map merge of :33-49 is not
 * taken by any generated schedule). */
void or_correct_to_finegrid(int n, int grid_size, int os, const REAL *uvw_, const REAL *vis_, double uv_scale,
                            REAL *out_vis_, REAL *out_uvw_, int *num_out)
{
    const R3 *uvw = (const R3 *)uvw_;
    const R2 *vis = (const R2 *)vis_;
    R2 *out_vis = (R2 *)out_vis_;
    R3 *out_uvw = (R3 *)out_uvw_;
    memset(out_vis, 0, sizeof(R2) * (size_t)n);
    *num_out = 0;
    for (int i = 0; i < n; ++i) {
        /* :24-25: the sum is formed in double and truncated to an integer */
        long long fx = (long long)((uvw[i].x * uv_scale + grid_size / 2) * os + 0.5f);
        long long fy = (long long)((uvw[i].y * uv_scale + grid_size / 2) * os + 0.5f);
        out_vis[*num_out] = vis[i];
        /* :52-54 */
        out_uvw[*num_out].x = ((double)fx / os - grid_size / 2) / uv_scale;
        out_uvw[*num_out].y = ((double)fy / os - grid_size / 2) / uv_scale;
        out_uvw[*num_out].z = uvw[i].z;
        *num_out = *num_out + 1;
    }
}

/* degridgrid.c:69-125 */
void or_std_gridding(int grid_size, int os, int n, const REAL *kernels_, const int *supports_, const REAL *uvw_,
                     const REAL *vis_, double uv_scale, double w_scale, REAL *grid_)
{
    const R2 *kernels = (const R2 *)kernels_;
    const I2 *supports = (const I2 *)supports_;
    const R3 *uvw = (const R3 *)uvw_;
    const R2 *vis = (const R2 *)vis_;
    R2 *grid = (R2 *)grid_;
    memset(grid, 0, sizeof(R2) * (size_t)grid_size * grid_size);
    int grid_center = grid_size / 2;
    for (int i = 0; i < n; ++i) {
        int w_idx = (int)(R_SQRT(R_ABS(uvw[i].z * w_scale)) + 0.5);                 /* :84 */
        R2 pos;
        pos.x = uvw[i].x * uv_scale;                                                  /* :85 */
        pos.y = uvw[i].y * uv_scale;
        int hs = supports[w_idx].x;
        REAL conjugate = (uvw[i].z < 0.0) ? -1.0 : 1.0;                               /* :89 */
        int w_offset = supports[w_idx].y;
        for (int v = R_CEIL(pos.y - hs); v < R_CEIL(pos.y + hs); ++v) {               /* :93 */
            if (v < -grid_center || v >= grid_center) continue;
            int ky = abs((int)R_ROUND((v - pos.y) * os));                              /* :101 */
            for (int u = R_CEIL(pos.x - hs); u < R_CEIL(pos.x + hs); ++u) {
                if (u < -grid_center || u >= grid_center) continue;
                int kx = abs((int)R_ROUND((u - pos.x) * os));
                int k_idx = w_offset + ky * (hs + 1) * os + kx;                        /* :112 */
                R2 ks = kernels[k_idx];
                ks.y *= conjugate;
                int g = (v + grid_center) * grid_size + (u + grid_center);
                R2 prod = cmul(vis[i], ks);
                grid[g].x += prod.x;
                grid[g].y += prod.y;
            }
        }
    }
}

/* degridgrid.c:127-202 */
void or_std_degridding(int grid_size, int os, int n, const REAL *kernels_, const int *supports_, const REAL *grid_,
                       const REAL *uvw_, double uv_scale, double w_scale, REAL *out_, int nearest)
{
    const R2 *kernels = (const R2 *)kernels_;
    const I2 *supports = (const I2 *)supports_;
    const R2 *grid = (const R2 *)grid_;
    const R3 *uvw = (const R3 *)uvw_;
    R2 *out = (R2 *)out_;
    memset(out, 0, sizeof(R2) * (size_t)n);
    int grid_center = grid_size / 2;
    for (int i = 0; i < n; ++i) {
        int w_idx = (int)(R_SQRT(R_ABS(uvw[i].z * w_scale)) + 0.5);
        int hs = supports[w_idx].x;
        int w_offset = supports[w_idx].y;
        R2 pos;
        pos.x = uvw[i].x * uv_scale;
        pos.y = uvw[i].y * uv_scale;
        REAL conjugate = (uvw[i].z < 0.0) ? -1.0 : 1.0;
        float comm_norm = 0.f;                                                        /* :145 float in both builds */
        if (!nearest) {
            for (int v = R_CEIL(pos.y - hs); v < R_CEIL(pos.y + hs); ++v) {
                int cv = v;                                                           /* :149-155 mirror at edges */
                if (v < -grid_center) cv = (-grid_center - v) - grid_center;
                else if (v >= grid_center) cv = (grid_center - v) + grid_center;
                int ky = abs((int)R_ROUND((cv - pos.y) * os));
                for (int u = R_CEIL(pos.x - hs); u < R_CEIL(pos.x + hs); ++u) {
                    int cu = u;
                    if (u < -grid_center) cu = (-grid_center - u) - grid_center;
                    else if (u >= grid_center) cu = (grid_center - u) + grid_center;
                    int kx = abs((int)R_ROUND((cu - pos.x) * os));
                    int k_idx = w_offset + ky * (hs + 1) * os + kx;
                    R2 ks;
                    if (kx < (hs + 1) * os && ky < (hs + 1) * os) {
                        ks = kernels[k_idx];
                    } else {
                        /* a mirrored tap can land just past the quarter-plane row
                         * (|du| = hs + 1); the reference then reads a neighbouring
                         * sample.  Defined here as a zero sample. */
                        ks.x = 0;
                        ks.y = 0;
                    }
                    ks.y *= conjugate;
                    /* The mirror of :153-154/:167-168 sends v = G/2 to row G, one past
                     * the grid (an out-of-bounds read in the reference).  Such a tap
                     * reads 0 here; its kernel weight still enters comm_norm. */
                    R2 gv;
                    if (cv + grid_center < grid_size && cu + grid_center < grid_size) {
                        gv = grid[(cv + grid_center) * grid_size + (cu + grid_center)];
                    } else {
                        gv.x = 0;
                        gv.y = 0;
                    }
                    R2 prod = cmul(gv, ks);
                    comm_norm += ks.x * ks.x + ks.y * ks.y;                          /* :181 */
                    out[i].x += prod.x;
                    out[i].y += prod.y;
                }
            }
            comm_norm = sqrt(comm_norm);                                              /* :188 */
            /* :190-191, including the reference's use of .x in the .y fallback */
            out[i].x = comm_norm < 1e-5f ? out[i].x / 1e-5f : out[i].x / comm_norm;
            out[i].y = comm_norm < 1e-5f ? out[i].x / 1e-5f : out[i].y / comm_norm;
        } else {
            /* :194-200 */
            int x = (int)(pos.x + (REAL)grid_center + 0.5);
            int y = (int)(pos.y + (REAL)grid_center + 0.5);
            long long idx = (long long)x + (long long)y * grid_size;
            if (idx >= 0 && idx < (long long)grid_size * grid_size) {
                out[i].x = grid[idx].x;
                out[i].y = grid[idx].y;
            } else {
                /* out of the grid: undefined in the reference; defined as 0 here */
                out[i].x = 0;
                out[i].y = 0;
            }
        }
    }
}

/* degridgrid.c:204-326.  The kernel-weighted degrid of :231-263 is discarded
 * by the reference (its value is replaced at :278-285 and comm_norm is unused),
 * so it is not recomputed here. */
void or_g2g_degridgrid(int grid_size, int os, int n, const REAL *gkernels_, const int *gsupports_,
                       const REAL *dkernels_, const int *dsupports_, const REAL *in_grid_, const REAL *uvw_,
                       double uv_scale, REAL *out_grid_)
{
    const R2 *gkernels = (const R2 *)gkernels_;
    const I2 *gsupports = (const I2 *)gsupports_;
    const R2 *in_grid = (const R2 *)in_grid_;
    const R3 *uvw = (const R3 *)uvw_;
    R2 *out_grid = (R2 *)out_grid_;
    (void)dkernels_;
    (void)dsupports_;
    memset(out_grid, 0, sizeof(R2) * (size_t)grid_size * grid_size);
    int grid_center = grid_size / 2;
    for (int i = 0; i < n; ++i) {
        int w_idx = 0;                                                                /* :215 */
        R2 pos;
        pos.x = uvw[i].x * uv_scale;
        pos.y = uvw[i].y * uv_scale;
        REAL conjugate = (uvw[i].z < 0.0) ? -1.0 : 1.0;
        R2 dv;
        int x = (int)(pos.x + (REAL)grid_center + 0.5);                              /* :273-276 */
        int y = (int)(pos.y + (REAL)grid_center + 0.5);
        long long idx = (long long)x + (long long)y * grid_size;
        if (idx >= 0 && idx < (long long)grid_size * grid_size) {                    /* :278 (lower bound) */
            dv = in_grid[idx];
        } else {
            dv.x = 0;
            dv.y = 0;
        }
        int hs = gsupports[w_idx].x;                                                  /* :292-324 */
        int w_offset = gsupports[w_idx].y;
        for (int v = R_CEIL(pos.y - hs); v < R_CEIL(pos.y + hs); ++v) {
            if (v < -grid_center || v >= grid_center) continue;
            int ky = abs((int)R_ROUND((v - pos.y) * os));
            for (int u = R_CEIL(pos.x - hs); u < R_CEIL(pos.x + hs); ++u) {
                if (u < -grid_center || u >= grid_center) continue;
                int kx = abs((int)R_ROUND((u - pos.x) * os));
                int k_idx = w_offset + ky * (hs + 1) * os + kx;
                R2 ks = gkernels[k_idx];
                ks.y *= conjugate;
                int g = (v + grid_center) * grid_size + (u + grid_center);
                R2 prod = cmul(dv, ks);
                out_grid[g].x += prod.x;
                out_grid[g].y += prod.y;
            }
        }
    }
}

/* gridding_run.c:55-137 */
void or_gridding_cpu(REAL *grid_, const REAL *kernels_, const int *supports_, const REAL *uvw_, const REAL *vis_,
                     int n, int os, int grid_size, double uv_scale, double w_scale)
{
    R2 *grid = (R2 *)grid_;
    const R2 *kernels = (const R2 *)kernels_;
    const I2 *supports = (const I2 *)supports_;
    const R3 *uvw = (const R3 *)uvw_;
    const R2 *vis = (const R2 *)vis_;
    for (int i = 0; i < n; ++i) {
        const int plane = (int)R_ROUND(R_SQRT(R_ABS(uvw[i].z * w_scale)));         /* :67 */
        R2 gc;
        gc.x = (REAL)(uvw[i].x * uv_scale);                                           /* :70-73 */
        gc.y = (REAL)(uvw[i].y * uv_scale);
        const int half_grid = grid_size / 2;
        const int hs = supports[plane].x;
        REAL conjugate = (uvw[i].z < 0.0) ? -1.0 : 1.0;
        R2 snapped;
        snapped.x = R_ROUND(gc.x * os) / os;                                          /* :79-82 */
        snapped.y = R_ROUND(gc.y * os) / os;
        R2 mn, mx;
        mn.x = R_CEIL(snapped.x - hs);                                                /* :84-92 */
        mn.y = R_CEIL(snapped.y - hs);
        mx.x = R_FLOOR(snapped.x + hs);
        mx.y = R_FLOOR(snapped.y + hs);
        int w_offset = supports[plane].y;
        for (int gv = mn.y; gv <= mx.y; ++gv) {                                       /* :104 */
            if (gv < -half_grid || gv >= half_grid) continue;
            int ky = abs((int)R_ROUND((gv - snapped.y) * os));
            for (int gu = mn.x; gu <= mx.x; ++gu) {
                if (gu < -half_grid || gu >= half_grid) continue;
                int kx = abs((int)R_ROUND((gu - snapped.x) * os));
                int k = w_offset + ky * (hs + 1) * os + kx;
                R2 ks;
                ks.x = kernels[k].x;
                ks.y = kernels[k].y * conjugate;
                int g = (gv + half_grid) * grid_size + (gu + half_grid);
                R2 c = cmul(vis[i], ks);                                              /* gridding_run.c:148-151 */
                grid[g].x += c.x;
                grid[g].y += c.y;
            }
        }
    }
}

/* gains_apply_run.c:273-297 (keepold is always false) */
void or_subtract_vis(int n, const REAL *measured, const REAL *predicted, REAL *delta)
{
    for (int i = 0; i < 2 * n; ++i) delta[i] = measured[i] - predicted[i];
}

/* degridgrid.c:328-335 */
void or_subtract_image(int grid_size, const REAL *a, const REAL *b, REAL *out)
{
    for (long long i = 0; i < (long long)grid_size * grid_size; ++i) out[i] = a[i] - b[i];
}

/* fft_run.c:5-20: checkerboard sign (-1)^(row+col) */
void or_fft_shift_c2c(int grid_size, const REAL *in, REAL *out)
{
    for (int r = 0; r < grid_size; ++r)
        for (int c = 0; c < grid_size; ++c) {
            int a = 1 - 2 * ((r + c) & 1);
            long long i = (long long)r * grid_size + c;
            out[2 * i] = in[2 * i] * a;
            out[2 * i + 1] = in[2 * i + 1] * a;
        }
}

/* fft_run.c:86-102 */
void or_fft_shift_c2r(int grid_size, const REAL *in, REAL *out)
{
    for (int r = 0; r < grid_size; ++r)
        for (int c = 0; c < grid_size; ++c) {
            int a = 1 - 2 * ((r + c) & 1);
            long long i = (long long)r * grid_size + c;
            out[i] = in[2 * i] * a;
        }
}

/* fft_run.c:104-121 */
void or_fft_shift_r2c(int grid_size, const REAL *in, REAL *out)
{
    for (int r = 0; r < grid_size; ++r)
        for (int c = 0; c < grid_size; ++c) {
            int a = 1 - 2 * ((r + c) & 1);
            long long i = (long long)r * grid_size + c;
            out[2 * i] = in[i] * a;
            out[2 * i + 1] = 0;
        }
}

/* fft_run.c:23-83 */
void or_fft2d(int grid_size, const REAL *in, REAL *out, int sign)
{
#ifdef ORACLE_DOUBLE
    oracle_fft2d_c128(grid_size, grid_size, in, out, sign);
#else
    oracle_fft2d_c64(grid_size, grid_size, in, out, sign);
#endif
}

/* top.c:412-451: Schwab's rational approximation of the zero-order prolate
 * spheroidal wave function (Schwab 1984), two intervals split at nu = 0.75. */
double or_prolate_spheroidal(double nu)
{
    static const double p[] = {0.08203343, -0.3644705, 0.627866, -0.5335581, 0.2312756,
                               0.004028559, -0.03697768, 0.1021332, -0.1201436, 0.06412774};
    static const double q[] = {1.0, 0.8212018, 0.2078043, 1.0, 0.9599102, 0.2918724};
    int part;
    double nuend;
    if (nu >= 0.0 && nu < 0.75) {
        part = 0;
        nuend = 0.75;
    } else if (nu >= 0.75 && nu < 1.0) {
        part = 1;
        nuend = 1.0;
    } else {
        return 0.0;
    }
    double delta = nu * nu - nuend * nuend;
    double top = p[part * 5], bottom = q[part * 3];
    for (int i = 1; i < 5; i++) top += p[part * 5 + i] * pow(delta, i);
    for (int i = 1; i < 3; i++) bottom += q[part * 3 + i] * pow(delta, i);
    return (bottom == 0.0) ? 0.0 : top / bottom;
}

/* top.c:399-408 */
void or_create_1D_half_prolate(REAL *prolate, int grid_size)
{
    int half = grid_size / 2;
    for (int i = 0; i < half; ++i) prolate[i] = (REAL)or_prolate_spheroidal((double)i / (double)half);
}

/* convolution_correction_run.c:4-35 */
void or_conv_correction(int grid_size, const REAL *in, const REAL *prolate, REAL *out)
{
    const int half = grid_size / 2;
    for (int r = 0; r < grid_size; ++r)
        for (int c = 0; c < grid_size; ++c) {
            long long i = (long long)r * grid_size + c;
            REAL taper = prolate[abs(c - half)] * prolate[abs(r - half)];
            if (abs(c - half) == 1229 || abs(r - half) == 1229) taper = 0.0;
            out[i] = (R_ABS(taper) > (1E-10)) ? in[i] / taper : 0.0;
        }
}

/* dft_run.c:3-48 (approximation branch :219-221) */
void or_dft(int n, int num_sources, const REAL *sources_, const REAL *uvw_, REAL *vis_)
{
    const R3 *sources = (const R3 *)sources_;
    const R3 *uvw = (const R3 *)uvw_;
    R2 *vis = (R2 *)vis_;
    for (int i = 0; i < n; ++i) {
        const REAL two_pi = R_PI + R_PI;
        const R3 v = uvw[i];
        R2 sum;
        sum.x = 0.0;
        sum.y = 0.0;
        for (int s = 0; s < num_sources; ++s) {
            R3 src = sources[s];
            REAL term = 0.5 * ((src.x * src.x) + (src.y * src.y));
            REAL w_correction = -term;
            REAL image_correction = 1.0 - term;
            REAL src_correction = src.z / image_correction;
            REAL theta = (v.x * src.x + v.y * src.y + v.z * w_correction) * two_pi;
            REAL s_ = R_SIN(theta);
            REAL c_ = R_COS(theta);
            sum.x += c_ * src_correction;
            sum.y += -s_ * src_correction;
        }
        vis[i] = sum;
    }
}

/* preesm_pipelines/simsdp_fft_imaging_pipeline/Code/src/CPU/deconvolution_run.c:197-311 */
void or_hogbom_clean(int grid_size, int num_minor_cycles, int max_sources, const REAL *residual, const REAL *psf,
                     double loop_gain, double noise_factor, double weak_source_percent, double psf_max_value,
                     double cell_size, const REAL *current_model, int *num_sources_out, REAL *sources_out_,
                     REAL *output_model, REAL *residual_out)
{
    const long long g2 = (long long)grid_size * grid_size;
    R3 *sources_out = (R3 *)sources_out_;
    REAL *r = residual_out;
    memcpy(r, residual, sizeof(REAL) * (size_t)g2);
    memcpy(output_model, current_model, sizeof(REAL) * (size_t)g2);
    *num_sources_out = 0;
    const double WEAK = weak_source_percent, GAIN = loop_gain, NOISE = noise_factor;
    (void)max_sources;
    for (int it = 0; it < num_minor_cycles; ++it) {
        REAL curr_max = 0.f;                                                          /* :218-233 */
        I2 max_pos = {0, 0};
        REAL curr_average = 0.f;
        for (int y = 0; y < grid_size; ++y)
            for (int x = 0; x < grid_size; ++x) {
                int idx = y * grid_size + x;
                REAL val = R_ABS(r[idx]);
                curr_average = idx == 0 ? val : curr_average + (val - curr_average) / idx;
                if (val > curr_max) {
                    curr_max = fabs(r[idx]);
                    max_pos.x = x;
                    max_pos.y = y;
                }
            }
        int max_idx = max_pos.y * grid_size + max_pos.x;
        int extracting_noise = R_ABS(curr_max) < NOISE * curr_average * GAIN;         /* :238-242 */
        int weak_source = *num_sources_out > 0 && R_ABS(curr_max) < (R_ABS(sources_out[0].z) * WEAK);
        if (extracting_noise || weak_source) break;
        I2 psf_center = {grid_size / 2, grid_size / 2};
        float max_val = r[max_idx] / psf_max_value;                                   /* :247 */
        sources_out[*num_sources_out].x = max_pos.x;
        sources_out[*num_sources_out].y = max_pos.y;
        sources_out[*num_sources_out].z = max_val * GAIN;
        *num_sources_out = *num_sources_out + 1;
        output_model[max_idx] += max_val * GAIN;                                      /* :256 */
        I2 s0 = {R_MIN(max_pos.x, grid_size / 2), R_MIN(max_pos.y, grid_size / 2)};   /* :263-264 */
        I2 e0 = {R_MIN(grid_size - max_pos.x, grid_size / 2), R_MIN(grid_size - max_pos.y, grid_size / 2)};
        for (int y = max_pos.y - s0.y; y < max_pos.y + e0.y; ++y)
            for (int x = max_pos.x - s0.x; x < max_pos.x + e0.x; ++x) {
                int image_idx = y * grid_size + x;
                /* :269: PSF mirrored in x; column index grid_size wraps to the next row */
                int psf_idx = (y - max_pos.y + psf_center.y) * grid_size + (grid_size - (x - max_pos.x + psf_center.x));
                r[image_idx] -= GAIN * max_val * psf[psf_idx] * psf_max_value;
            }
    }
    if (*num_sources_out > 0)                                                         /* :297-306 */
        for (int k = 0; k < *num_sources_out; k++) {
            sources_out[k].x = (sources_out[k].x - grid_size / 2) * cell_size;
            sources_out[k].y = (sources_out[k].y - grid_size / 2) * cell_size;
        }
}

/* splitmerge.c:14-24 */
void or_merge_grids(int grid_size, int slices, const REAL *grids, REAL *out)
{
    long long g2 = (long long)grid_size * grid_size;
    for (long long i = 0; i < g2; ++i) {
        REAL cx = 0, cy = 0;
        for (int j = 0; j < slices; ++j) {
            cx += grids[2 * (j * g2 + i)];
            cy += grids[2 * (j * g2 + i) + 1];
        }
        out[2 * i] = cx;
        out[2 * i + 1] = cy;
    }
}

/* splitmerge.c:50-56 */
void or_split_uvgrid(int grid_size, int slices, const REAL *in, REAL *out)
{
    long long g2 = (long long)grid_size * grid_size;
    for (int j = 0; j < slices; ++j) memcpy(out + 2 * j * g2, in, sizeof(REAL) * 2 * (size_t)g2);
}

/* top.c:453-515 (the file read of :466-491 replaced by an array argument) */
double or_psf_crop_normalise(int grid_size, int psf_grid_size, const REAL *full_psf, REAL *psf)
{
    double psf_max = 0.0;
    long long full2 = (long long)psf_grid_size * psf_grid_size;
    for (long long i = 0; i < full2; ++i)
        if ((double)full_psf[i] > psf_max) psf_max = (REAL)full_psf[i];
    memset(psf, 0, sizeof(REAL) * (size_t)grid_size * grid_size);
    int smaller = R_MIN(psf_grid_size, grid_size);
    int psf_off = R_MAX(0, (psf_grid_size - grid_size) / 2);
    int grid_off = R_MAX(0, (grid_size - psf_grid_size) / 2);
    for (int y = 0; y < smaller; ++y)
        for (int x = 0; x < smaller; ++x)
            psf[(long long)(y + grid_off) * grid_size + (x + grid_off)] =
                full_psf[(long long)(y + psf_off) * psf_grid_size + (x + psf_off)];
    for (long long i = 0; i < (long long)grid_size * grid_size; ++i) psf[i] /= psf_max;
    return psf_max;
}

/* top.c:523-526 */
static float gaussian2d(float x, float y, float xs, float ys)
{
    return exp(-(x * x) / (2 * xs * xs) - (y * y) / (2 * ys * ys)) / (2 * R_PI * xs * ys);
}

/* top.c:530-595 */
void or_clean_psf(int grid_size, double psf_max_value, const REAL *dirty_psf, REAL *clean_psf, int *halfdims)
{
    int center_box[4] = {grid_size / 2};
    const int dir[4][2] = {{1, 0}, {0, 1}, {-1, 0}, {0, -1}};
    int half_extent = grid_size / 2;
    I2 center = {grid_size / 2 + 1, grid_size / 2 + 1};
    for (int i = 0; i < 4; ++i) {
        int prev_sign = -1;
        for (int j = 1; j < half_extent; ++j) {
            int cx = center.x + dir[i][0] * j, cy = center.y + dir[i][1] * j;
            int lx = center.x + dir[i][0] * (j - 1), ly = center.y + dir[i][1] * (j - 1);
            float deriv = dirty_psf[cx + cy * grid_size] - dirty_psf[lx + ly * grid_size];
            int sign = deriv >= 0.f ? 1 : -1;
            if (sign != prev_sign) {
                center_box[i] = j;
                break;
            }
        }
    }
    int hd = R_MAX(R_MAX(R_MAX(center_box[0], center_box[1]), center_box[2]), center_box[3]);
    halfdims[0] = halfdims[1] = hd;
    memset(clean_psf, 0, sizeof(REAL) * (size_t)grid_size * grid_size);
    float psf_max_val = psf_max_value;
    float xs = hd / 2.f, ys = hd / 2.f;
    float sum = 0.f;
    for (int y = -hd; y < hd; ++y)
        for (int x = -hd; x < hd; ++x) {
            int idx = center.x + x + (center.y + y) * grid_size;
            clean_psf[idx] = gaussian2d(x, y, xs, ys);
            clean_psf[idx] *= clean_psf[idx];
            sum += clean_psf[idx];
        }
    for (int y = -hd; y < hd; ++y)
        for (int x = -hd; x < hd; ++x) {
            int idx = center.x + x + (center.y + y) * grid_size;
            clean_psf[idx] = clean_psf[idx] / sum * psf_max_val;
        }
}
