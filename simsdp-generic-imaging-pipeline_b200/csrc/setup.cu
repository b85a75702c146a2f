// Setup math of the reference (src/top.c): the prolate spheroidal used by the
// taper correction, and the Gaussian clean beam fitted to the dirty PSF.
#include <cmath>
#include <cstring>

#include "internal.cuh"

namespace sdp {

// top.c:412-451, Schwab's two-interval rational approximation (host copy of
// the device evaluation in elementwise.cu).
double prolate_host(double nu)
{
    static const double p[10] = {0.08203343, -0.3644705, 0.627866, -0.5335581, 0.2312756,
                                 0.004028559, -0.03697768, 0.1021332, -0.1201436, 0.06412774};
    static const double q[6] = {1.0, 0.8212018, 0.2078043, 1.0, 0.9599102, 0.2918724};
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
    const double d = nu * nu - nuend * nuend;
    double top = p[part * 5], bot = q[part * 3];
    for (int i = 1; i < 5; i++) top += p[part * 5 + i] * pow(d, i);
    for (int i = 1; i < 3; i++) bot += q[part * 3 + i] * pow(d, i);
    return (bot == 0.0) ? 0.0 : top / bot;
}

// top.c:530-595 in one thread: the box edges are found by walking out from
// (G/2+1, G/2+1) until the first non-negative derivative (the reference
// never updates prev_sign, so that is its rule), the clean beam is a squared
// Gaussian of sigma = halfdim / 2 normalised to sum psf_max.  The loops are
// sequential to keep the reference's float summation order.
__global__ void k_clean_psf(int G, float psf_max_val, const float *__restrict__ dirty, float *__restrict__ clean,
                            int *__restrict__ halfdims)
{
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    int box[4] = {G / 2, 0, 0, 0};
    const int dir[4][2] = {{1, 0}, {0, 1}, {-1, 0}, {0, -1}};
    const int half = G / 2;
    const int cx = G / 2 + 1, cy = G / 2 + 1;
    for (int i = 0; i < 4; ++i) {
        for (int j = 1; j < half; ++j) {
            const int x1 = cx + dir[i][0] * j, y1 = cy + dir[i][1] * j;
            const int x0 = cx + dir[i][0] * (j - 1), y0 = cy + dir[i][1] * (j - 1);
            // flat indices as in the reference (x = G wraps to the next row);
            // a flat index outside the image ends the walk
            const long long f1 = x1 + (long long)y1 * G, f0 = x0 + (long long)y0 * G;
            if (f1 < 0 || f1 >= (long long)G * G || f0 < 0 || f0 >= (long long)G * G) break;
            const float deriv = __fsub_rn(dirty[f1], dirty[f0]);
            if (deriv >= 0.f) {
                box[i] = j;
                break;
            }
        }
    }
    const int hd = max(max(max(box[0], box[1]), box[2]), box[3]);
    halfdims[0] = hd;
    halfdims[1] = hd;
    const float xs = hd / 2.f, ys = hd / 2.f;
    const float pi_f = 3.141592654f;
    float sum = 0.f;
    for (int y = -hd; y < hd; ++y)
        for (int x = -hd; x < hd; ++x) {
            const long long idx = (long long)cx + x + (long long)(cy + y) * G;
            if (idx < 0 || idx >= (long long)G * G) continue;
            const float fx = (float)x, fy = (float)y;
            const float ex = __fsub_rn(__fdiv_rn(-__fmul_rn(fx, fx), __fmul_rn(__fmul_rn(2.f, xs), xs)),
                                       __fdiv_rn(__fmul_rn(fy, fy), __fmul_rn(__fmul_rn(2.f, ys), ys)));
            const float den = __fmul_rn(__fmul_rn(__fmul_rn(2.f, pi_f), xs), ys);
            float g = __double2float_rn(__ddiv_rn(exp((double)ex), (double)den));
            g = __fmul_rn(g, g);
            clean[idx] = g;
            sum = __fadd_rn(sum, g);
        }
    for (int y = -hd; y < hd; ++y)
        for (int x = -hd; x < hd; ++x) {
            const long long idx = (long long)cx + x + (long long)(cy + y) * G;
            if (idx < 0 || idx >= (long long)G * G) continue;
            clean[idx] = __fmul_rn(__fdiv_rn(clean[idx], sum), psf_max_val);
        }
}

}  // namespace sdp

using namespace sdp;

SDP_EXPORT int sdp_clean_psf(int G, double psf_max_value, const float *dirty_psf, float *clean_psf,
                             int *halfdims_dev, void *stream)
{
    SDP_CHECK_ARG(G >= 4 && dirty_psf && clean_psf && halfdims_dev, "bad argument");
    cudaStream_t st = as_stream(stream);
    SDP_CUDA_TRY(cudaMemsetAsync(clean_psf, 0, sizeof(float) * (size_t)G * G, st));
    k_clean_psf<<<1, 32, 0, st>>>(G, (float)psf_max_value, dirty_psf, clean_psf, halfdims_dev);
    SDP_LAUNCH_CHECK();
    return SDP_OK;
}

SDP_EXPORT void clean_psf_host_set_up(int GRID_SIZE, int GAUSSIAN_CLEAN_PSF, sdp_config *config, float *dirty_psf,
                                      float *clean_psf, sdp_int2 *partial_psf_halfdims)
{
    (void)GAUSSIAN_CLEAN_PSF;
    int status = SDP_OK;
    do {
        if (!config || !dirty_psf || !clean_psf || !partial_psf_halfdims || GRID_SIZE < 4) {
            status = set_error(SDP_ERR_INVALID, "bad argument");
            break;
        }
        ThreadCtx *ctx = nullptr;
        if ((status = thread_ctx(&ctx)) != SDP_OK) break;
        const size_t G2 = (size_t)GRID_SIZE * GRID_SIZE;
        void *dd = nullptr, *dc = nullptr, *dh = nullptr;
        if ((status = ctx_buffer(ctx, 0, sizeof(float) * G2, &dd)) != SDP_OK) break;
        if ((status = ctx_buffer(ctx, 1, sizeof(float) * G2, &dc)) != SDP_OK) break;
        if ((status = ctx_buffer(ctx, 2, sizeof(int) * 2, &dh)) != SDP_OK) break;
        cudaError_t e = cudaMemcpyAsync(dd, dirty_psf, sizeof(float) * G2, cudaMemcpyHostToDevice, ctx->stream);
        if (e != cudaSuccess) {
            status = cuda_error(e, "clean_psf upload");
            break;
        }
        if ((status = sdp_clean_psf(GRID_SIZE, config->psf_max_value, (const float *)dd, (float *)dc, (int *)dh,
                                    ctx->stream)) != SDP_OK)
            break;
        e = cudaMemcpyAsync(clean_psf, dc, sizeof(float) * G2, cudaMemcpyDeviceToHost, ctx->stream);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(partial_psf_halfdims, dh, sizeof(int) * 2, cudaMemcpyDeviceToHost, ctx->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
        if (e != cudaSuccess) status = cuda_error(e, "clean_psf download");
    } while (0);
    if (status != SDP_OK) actor_fail("clean_psf_host_set_up");
}
