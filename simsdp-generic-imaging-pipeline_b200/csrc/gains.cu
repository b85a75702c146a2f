// Antenna gains applied to visibilities (param_code/code_fft_1core/src/CPU/
// gains_apply_run.c, and the set-up of top.c:71-136):
//
//   reciprocal_transform_actor  :4-18    g' = conj(g) / |g|^2, per receiver
//   apply_gains_actor           :20-69   v' = m * g'_a * conj(g'_b) [- v_in]
//   subtract_from_measurements  :71-97   v' = m * g'_a * conj(g'_b) - v_in
//   apply_gains_only            :99-120  v' = m (the product is discarded, :117)
//   gains_host_set_up           top.c:71-116 (unit gains, or the gains file)
//   calculate_receiver_pairs    top.c:118-136
//
// Visibility i belongs to baseline i % NUM_BASELINES (time-major order) whose
// receivers are receiver_pairs[baseline].  One thread per visibility; every
// product and sum is rounded as the reference's float build rounds it (no
// fused multiply-add), so the outputs are bit-exact.
#include <cstdio>
#include <cstring>

#include <algorithm>
#include <string>
#include <vector>

#include "internal.cuh"

namespace sdp {

__device__ __forceinline__ float2 cmul_ref(float2 a, float2 b)  // complex_multiply_apply (:148-151)
{
    return make_float2(__fsub_rn(__fmul_rn(a.x, b.x), __fmul_rn(a.y, b.y)),
                       __fadd_rn(__fmul_rn(a.x, b.y), __fmul_rn(a.y, b.x)));
}

__global__ void k_reciprocal(int n, const float2 *__restrict__ in, float2 *__restrict__ out)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float2 z = in[i];
    const float d = __fadd_rn(__fmul_rn(z.x, z.x), __fmul_rn(z.y, z.y));
    out[i] = make_float2(__fdiv_rn(z.x, d), -__fdiv_rn(z.y, d));
}

// subtract != 0: m * g_a * conj(g_b) - v_in; else m * g_a * conj(g_b).
__global__ void k_apply_gains(int n, int nbl, int nrx, const float2 *__restrict__ measured,
                              const float2 *__restrict__ vin, const float2 *__restrict__ gains,
                              const int2 *__restrict__ pairs, int subtract, float2 *__restrict__ out,
                              int *__restrict__ flags)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int2 rp = pairs[i % nbl];
    if (rp.x < 0 || rp.x >= nrx || rp.y < 0 || rp.y >= nrx) {  // the reference would read outside gains[]
        atomicOr(flags, 1);
        out[i] = make_float2(0.f, 0.f);
        return;
    }
    const float2 ga = gains[rp.x], gb = gains[rp.y];
    const float2 prod = cmul_ref(ga, make_float2(gb.x, -gb.y));
    const float2 mg = cmul_ref(measured[i], prod);
    out[i] = subtract ? make_float2(__fsub_rn(mg.x, vin[i].x), __fsub_rn(mg.y, vin[i].y)) : mg;
}

}  // namespace sdp

using namespace sdp;

SDP_EXPORT int sdp_gains_reciprocal(int num_receivers, const sdp_float2 *gains_in, sdp_float2 *gains_out, void *stream)
{
    SDP_CHECK_ARG(num_receivers >= 0 && (num_receivers == 0 || (gains_in && gains_out)), "bad argument");
    if (num_receivers == 0) return SDP_OK;
    k_reciprocal<<<(num_receivers + 255) / 256, 256, 0, as_stream(stream)>>>(
        num_receivers, reinterpret_cast<const float2 *>(gains_in), reinterpret_cast<float2 *>(gains_out));
    SDP_LAUNCH_CHECK();
    return SDP_OK;
}

SDP_EXPORT int sdp_apply_gains(int num_vis, int num_baselines, int num_receivers, const sdp_float2 *measured,
                               const sdp_float2 *vis_in, const sdp_float2 *gains, const sdp_int2 *receiver_pairs,
                               int subtract, sdp_float2 *vis_out, int *flags_dev, void *stream)
{
    SDP_CHECK_ARG(num_vis >= 0 && num_baselines >= 1 && num_receivers >= 1, "bad sizes");
    if (num_vis == 0) return SDP_OK;
    SDP_CHECK_ARG(measured && gains && receiver_pairs && vis_out && flags_dev && (!subtract || vis_in),
                  "NULL argument");
    k_apply_gains<<<(num_vis + 255) / 256, 256, 0, as_stream(stream)>>>(
        num_vis, num_baselines, num_receivers, reinterpret_cast<const float2 *>(measured),
        reinterpret_cast<const float2 *>(vis_in), reinterpret_cast<const float2 *>(gains),
        reinterpret_cast<const int2 *>(receiver_pairs), subtract, reinterpret_cast<float2 *>(vis_out), flags_dev);
    SDP_LAUNCH_CHECK();
    return SDP_OK;
}

// ---------------------------------------------------------------------------
// Actors (host buffers)
// ---------------------------------------------------------------------------
namespace {

int gains_actor(int NRX, int NBL, int NV, const sdp_float2 *measured, const sdp_float2 *vin, const sdp_float2 *gains,
                const sdp_int2 *pairs, int subtract, sdp_float2 *out)
{
    SDP_CHECK_ARG(NV >= 0 && NBL >= 1 && NRX >= 1 && measured && gains && pairs && out && (!subtract || vin),
                  "bad argument");
    ThreadCtx *ctx = nullptr;
    SDP_TRY(thread_ctx(&ctx));
    cudaStream_t st = ctx->stream;
    const size_t nv = (size_t)std::max(NV, 1);
    void *dm = nullptr, *dv = nullptr, *dg = nullptr, *dp = nullptr, *dout = nullptr, *df = nullptr;
    SDP_TRY(ctx_buffer(ctx, kSlotRestore + 0, sizeof(float2) * nv, &dm));
    SDP_TRY(ctx_buffer(ctx, kSlotRestore + 1, sizeof(float2) * nv, &dv));
    SDP_TRY(ctx_buffer(ctx, kSlotRestore + 2, sizeof(float2) * nv, &dout));
    SDP_TRY(ctx_buffer(ctx, kSlotRestore + 3, sizeof(float2) * NRX + sizeof(int2) * NBL + 256, &dg));
    dp = static_cast<char *>(dg) + ((sizeof(float2) * NRX + 15) / 16) * 16;
    df = static_cast<char *>(dp) + ((sizeof(int2) * NBL + 15) / 16) * 16;
    SDP_CUDA_TRY(cudaMemcpyAsync(dm, measured, sizeof(float2) * NV, cudaMemcpyHostToDevice, st));
    if (subtract) SDP_CUDA_TRY(cudaMemcpyAsync(dv, vin, sizeof(float2) * NV, cudaMemcpyHostToDevice, st));
    SDP_CUDA_TRY(cudaMemcpyAsync(dg, gains, sizeof(float2) * NRX, cudaMemcpyHostToDevice, st));
    SDP_CUDA_TRY(cudaMemcpyAsync(dp, pairs, sizeof(int2) * NBL, cudaMemcpyHostToDevice, st));
    SDP_CUDA_TRY(cudaMemsetAsync(df, 0, sizeof(int), st));
    SDP_TRY(sdp_apply_gains(NV, NBL, NRX, static_cast<sdp_float2 *>(dm), static_cast<sdp_float2 *>(dv),
                            static_cast<sdp_float2 *>(dg), static_cast<sdp_int2 *>(dp), subtract,
                            static_cast<sdp_float2 *>(dout), static_cast<int *>(df), st));
    int flags = 0;
    SDP_CUDA_TRY(cudaMemcpyAsync(out, dout, sizeof(float2) * NV, cudaMemcpyDeviceToHost, st));
    SDP_CUDA_TRY(cudaMemcpyAsync(&flags, df, sizeof(int), cudaMemcpyDeviceToHost, st));
    SDP_CUDA_TRY(cudaStreamSynchronize(st));
    if (flags) return set_error(SDP_ERR_DATA, "a receiver pair indexes outside the %d gains", NRX);
    return SDP_OK;
}

}  // namespace

SDP_EXPORT void reciprocal_transform_actor(int NUM_RECEIVERS, sdp_float2 *gains_in, sdp_config *config,
                                           sdp_float2 *gains_out)
{
    (void)config;
    int status = SDP_OK;
    do {
        if (NUM_RECEIVERS < 0 || (NUM_RECEIVERS > 0 && (!gains_in || !gains_out))) {
            status = set_error(SDP_ERR_INVALID, "bad argument");
            break;
        }
        if (NUM_RECEIVERS == 0) break;
        ThreadCtx *ctx = nullptr;
        if ((status = thread_ctx(&ctx)) != SDP_OK) break;
        void *d = nullptr;
        if ((status = ctx_buffer(ctx, kSlotRestore + 3, sizeof(float2) * 2 * NUM_RECEIVERS, &d)) != SDP_OK) break;
        float2 *din = static_cast<float2 *>(d), *dout = din + NUM_RECEIVERS;
        cudaStream_t st = ctx->stream;
        cudaError_t e = cudaMemcpyAsync(din, gains_in, sizeof(float2) * NUM_RECEIVERS, cudaMemcpyHostToDevice, st);
        if (e != cudaSuccess) {
            status = cuda_error(e, "upload");
            break;
        }
        if ((status = sdp_gains_reciprocal(NUM_RECEIVERS, reinterpret_cast<sdp_float2 *>(din),
                                           reinterpret_cast<sdp_float2 *>(dout), st)) != SDP_OK)
            break;
        e = cudaMemcpyAsync(gains_out, dout, sizeof(float2) * NUM_RECEIVERS, cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        if (e != cudaSuccess) status = cuda_error(e, "download");
    } while (0);
    if (status != SDP_OK) actor_fail("reciprocal_transform_actor");
}

SDP_EXPORT void apply_gains_actor(int CALIBRATION, int NUM_RECEIVERS, int NUM_BASELINES, int NUM_VISIBILITIES,
                                  sdp_float2 *measured_vis, sdp_float2 *visibilities_in, sdp_float2 *gains,
                                  sdp_int2 *receiver_pairs, sdp_config *config, sdp_float2 *visibilities_out)
{
    (void)config;
    // :34-48 (not calibrating: subtract the prediction) / :52-63 (calibrating)
    if (gains_actor(NUM_RECEIVERS, NUM_BASELINES, NUM_VISIBILITIES, measured_vis, visibilities_in, gains,
                    receiver_pairs, CALIBRATION ? 0 : 1, visibilities_out) != SDP_OK)
        actor_fail("apply_gains_actor");
}

SDP_EXPORT void subtract_from_measurements(int NUM_RECEIVERS, int NUM_BASELINES, int NUM_VISIBILITIES,
                                           sdp_float2 *measured_vis, sdp_float2 *visibilities_in, sdp_float2 *gains,
                                           sdp_int2 *receiver_pairs, sdp_config *config, sdp_float2 *visibilities_out)
{
    (void)config;
    if (gains_actor(NUM_RECEIVERS, NUM_BASELINES, NUM_VISIBILITIES, measured_vis, visibilities_in, gains,
                    receiver_pairs, 1, visibilities_out) != SDP_OK)
        actor_fail("subtract_from_measurements");
}

SDP_EXPORT void apply_gains_only(int NUM_RECEIVERS, int NUM_BASELINES, int NUM_VISIBILITIES, sdp_float2 *measured_vis,
                                 sdp_float2 *gains, sdp_int2 *receiver_pairs, sdp_config *config,
                                 sdp_float2 *visibilities_out)
{
    (void)NUM_RECEIVERS;
    (void)NUM_BASELINES;
    (void)gains;
    (void)receiver_pairs;
    (void)config;
    // the reference computes the gain product and then stores the measured
    // visibility unchanged (:117): a copy
    if (NUM_VISIBILITIES > 0) memmove(visibilities_out, measured_vis, sizeof(sdp_float2) * (size_t)NUM_VISIBILITIES);
}

SDP_EXPORT void calculate_receiver_pairs(int NUM_BASELINES, int NUM_RECEIVERS, sdp_int2 *receiver_pairs)
{
    int a = 0, b = 1;  // top.c:118-136
    for (int i = 0; i < NUM_BASELINES; ++i) {
        receiver_pairs[i].x = a;
        receiver_pairs[i].y = b;
        if (++b >= NUM_RECEIVERS) {
            ++a;
            b = a + 1;
        }
    }
}

SDP_EXPORT void gains_host_set_up(int NUM_RECEIVERS, int NUM_BASELINES, sdp_config *config, sdp_float2 *gains,
                                  sdp_int2 *receiver_pairs)
{
    if (config->use_default_gains) {  // top.c:73-79
        for (int i = 0; i < NUM_RECEIVERS; ++i) gains[i] = sdp_float2{1.0f, 0.0f};
    } else {  // top.c:80-103: "%lf %lf " per receiver
        FILE *f = config->default_gains_file ? fopen(config->default_gains_file, "r") : nullptr;
        if (!f) {
            set_error(SDP_ERR_IO, "unable to open the gains file %s",
                      config->default_gains_file ? config->default_gains_file : "(null)");
            actor_fail("gains_host_set_up");
            return;
        }
        double re = 0.0, im = 0.0;
        for (int i = 0; i < NUM_RECEIVERS; ++i) {
            if (fscanf(f, "%lf %lf ", &re, &im) < 0) {
            }  // a short file repeats the last values, as the reference's does
            gains[i] = sdp_float2{(float)re, (float)im};
        }
        fclose(f);
    }
    calculate_receiver_pairs(NUM_BASELINES, NUM_RECEIVERS, receiver_pairs);
}
