// Device-resident major cycle of the FFT imaging pipeline
// (param_code/code_fft_1core/generated/Core0.c, delta_k / psi_k):
//
//   model image --inverse taper (identity, convolution_correction_run.c:61)
//               --shift r2c, forward FFT, shift c2c--> model grid          (sdp_image_to_grid)
//   model grid  --degrid, subtract from measured, grid--> residual grid      (sdp_visplan_cycle)
//   residual grid --shift c2c, inverse FFT, shift c2r, taper--> residual     (sdp_grid_to_image)
//   residual, PSF --Hogbom CLEAN--> components, model += components          (sdp_hogbom)
//
// Everything stays in HBM between cycles; the only host traffic is what the
// caller asks for.  With use_graph the cycle is captured once as a CUDA graph
// on the caller's stream and replayed; if capture is refused the cycle runs
// as direct launches.
#include <cstdio>
#include <cstring>

#include "internal.cuh"

struct sdp_pipeline {
    sdp_pipeline_config cfg;
    sdp_visplan *plan = nullptr;
    float *model_image = nullptr;
    float *residual_image = nullptr;
    float *clean_scratch = nullptr;  // residual copy consumed by CLEAN
    float *psf = nullptr;
    float *prolate = nullptr;
    sdp_float2 *model_grid = nullptr;
    sdp_float2 *residual_grid = nullptr;
    sdp_float2 *work = nullptr;
    sdp_float3 *sources = nullptr;
    int *num_sources = nullptr;
    void *clean_ws = nullptr;
    size_t clean_ws_bytes = 0;
    void *arena = nullptr;
    cudaGraphExec_t graph = nullptr;
    cudaStream_t stream = nullptr;   // the pipeline's own stream (capture and replay)
    cudaEvent_t ev_in = nullptr, ev_out = nullptr;
    int graph_failed = 0;
    int in_capture = 0;
    int capture_persistent = 1;  // capture CLEAN as the cooperative kernel (first attempt)
    int cycles_run = 0;
    char graph_error[256] = {0};
};

namespace sdp {

static size_t al(size_t x) { return (x + 255) / 256 * 256; }

static int run_cycle(sdp_pipeline *p, cudaStream_t st)
{
    const sdp_pipeline_config &c = p->cfg;
    const int G = c.grid_size;
    const size_t G2 = (size_t)G * G;
    SDP_TRY(sdp_image_to_grid(G, p->model_image, p->work, p->model_grid, st));
    SDP_TRY(sdp_visplan_cycle(p->plan, p->model_grid, c.degrid_mode, nullptr, nullptr, p->residual_grid, st));
    SDP_TRY(sdp_grid_to_image(G, p->residual_grid, p->prolate, p->work, p->residual_image, st));
    if (c.num_minor_cycles > 0) {
        SDP_CUDA_TRY(cudaMemcpyAsync(p->clean_scratch, p->residual_image, sizeof(float) * G2,
                                     cudaMemcpyDeviceToDevice, st));
        sdp_clean_params cp{G, c.num_minor_cycles, c.max_sources, c.loop_gain, c.noise_factor,
                            c.weak_source_percent, c.psf_max_value, c.cell_size};
        // the persistent cooperative kernel, or one launch per minor cycle
        // when a capture of the cooperative launch was refused
        SDP_TRY(hogbom_launch(&cp, p->clean_scratch, p->psf, p->model_image, p->sources, p->num_sources,
                              p->clean_ws, p->clean_ws_bytes, !p->in_capture || p->capture_persistent, st));
    }
    return SDP_OK;
}

}  // namespace sdp

using namespace sdp;

SDP_EXPORT int sdp_pipeline_create(sdp_pipeline **out, const sdp_pipeline_config *cfg, const sdp_wkernels *gk,
                                   const sdp_wkernels *dk, int num_vis, const sdp_float3 *uvw,
                                   const sdp_float2 *measured, const float *psf, void *stream)
{
    SDP_CHECK_ARG(out && cfg && gk && psf && (num_vis == 0 || (uvw && measured)), "NULL argument");
    *out = nullptr;
    SDP_TRY(check_fft_size(cfg->grid_size));
    SDP_CHECK_ARG(cfg->degrid_mode == SDP_DEGRID_NEAREST || cfg->degrid_mode == SDP_DEGRID_CONV,
                  "degrid mode %d unknown", cfg->degrid_mode);
    SDP_CHECK_ARG(cfg->num_minor_cycles >= 0 && cfg->max_sources >= 0, "bad CLEAN sizes");
    SDP_CHECK_ARG(cfg->num_minor_cycles == 0 || cfg->psf_max_value != 0.0, "psf_max_value is 0");
    if (dk == nullptr) dk = gk;
    cudaStream_t st = as_stream(stream);
    const int G = cfg->grid_size;
    const size_t G2 = (size_t)G * G;
    sdp_pipeline *p = new sdp_pipeline();
    p->cfg = *cfg;
    int status = SDP_OK;
    do {
        size_t wsb = 0;
        if ((status = sdp_hogbom_workspace_bytes(G, &wsb)) != SDP_OK) break;
        p->clean_ws_bytes = wsb;
        const size_t nsrc = (size_t)std::max(1, cfg->max_sources);
        size_t o = 0;
        const size_t o_model = o;
        o = al(o + sizeof(float) * G2);
        const size_t o_res = o;
        o = al(o + sizeof(float) * G2);
        const size_t o_scr = o;
        o = al(o + sizeof(float) * G2);
        const size_t o_psf = o;
        o = al(o + sizeof(float) * G2);
        const size_t o_pro = o;
        o = al(o + sizeof(float) * (G2 > 0 ? (size_t)G / 2 + 1 : 1));
        const size_t o_mg = o;
        o = al(o + sizeof(sdp_float2) * G2);
        const size_t o_rg = o;
        o = al(o + sizeof(sdp_float2) * G2);
        const size_t o_work = o;
        o = al(o + sizeof(sdp_float2) * G2);
        const size_t o_src = o;
        o = al(o + sizeof(sdp_float3) * nsrc);
        const size_t o_cnt = o;
        o = al(o + sizeof(int));
        const size_t o_ws = o;
        o = al(o + wsb);
        cudaError_t e = cudaMalloc(&p->arena, o);
        if (e != cudaSuccess) {
            status = cuda_error(e, "cudaMalloc(pipeline)");
            break;
        }
        char *a = static_cast<char *>(p->arena);
        p->model_image = reinterpret_cast<float *>(a + o_model);
        p->residual_image = reinterpret_cast<float *>(a + o_res);
        p->clean_scratch = reinterpret_cast<float *>(a + o_scr);
        p->psf = reinterpret_cast<float *>(a + o_psf);
        p->prolate = reinterpret_cast<float *>(a + o_pro);
        p->model_grid = reinterpret_cast<sdp_float2 *>(a + o_mg);
        p->residual_grid = reinterpret_cast<sdp_float2 *>(a + o_rg);
        p->work = reinterpret_cast<sdp_float2 *>(a + o_work);
        p->sources = reinterpret_cast<sdp_float3 *>(a + o_src);
        p->num_sources = reinterpret_cast<int *>(a + o_cnt);
        p->clean_ws = a + o_ws;
        if ((e = cudaMemsetAsync(p->model_image, 0, sizeof(float) * G2, st)) != cudaSuccess ||
            (e = cudaMemsetAsync(p->num_sources, 0, sizeof(int), st)) != cudaSuccess ||
            (e = cudaMemcpyAsync(p->psf, psf, sizeof(float) * G2, cudaMemcpyDefault, st)) != cudaSuccess) {
            status = cuda_error(e, "pipeline set-up copy");
            break;
        }
        if ((status = sdp_prolate_table(G, p->prolate, st)) != SDP_OK) break;
        sdp_geometry geom{G, cfg->oversampling, cfg->uv_scale, cfg->w_scale};
        int mode = SDP_GRID_STD | SDP_PLAN_SNAP;
        if (cfg->coord_mode == SDP_COORD_F64) mode |= SDP_PLAN_COORD_F64;
        if (!cfg->snap) mode &= ~SDP_PLAN_SNAP;
        if ((status = sdp_visplan_create(&p->plan, &geom, gk, dk, num_vis, uvw, mode, stream)) != SDP_OK) break;
        if ((status = sdp_visplan_set_measured(p->plan, measured, stream)) != SDP_OK) break;
        // warm the FFT twiddle tables and check the plan's data flags before any capture
        if ((status = sdp_visplan_check(p->plan, stream)) != SDP_OK) break;
        if ((status = sdp_image_to_grid(G, p->model_image, p->work, p->model_grid, st)) != SDP_OK) break;
        e = cudaStreamSynchronize(st);
        if (e != cudaSuccess) status = cuda_error(e, "pipeline set-up");
    } while (0);
    if (status == SDP_OK) {
        cudaError_t e = cudaStreamCreateWithFlags(&p->stream, cudaStreamNonBlocking);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&p->ev_in, cudaEventDisableTiming);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&p->ev_out, cudaEventDisableTiming);
        if (e != cudaSuccess) status = cuda_error(e, "pipeline stream");
    }
    if (status != SDP_OK) {
        if (p->plan) sdp_visplan_destroy(p->plan);
        if (p->arena) cudaFree(p->arena);
        if (p->ev_in) cudaEventDestroy(p->ev_in);
        if (p->ev_out) cudaEventDestroy(p->ev_out);
        if (p->stream) cudaStreamDestroy(p->stream);
        delete p;
        return status;
    }
    *out = p;
    return SDP_OK;
}

SDP_EXPORT int sdp_pipeline_major_cycle(sdp_pipeline *p, void *stream)
{
    SDP_CHECK_ARG(p, "pipeline is NULL");
    // the cycle runs on the pipeline's own stream (the caller's may be the
    // legacy default stream, which cannot be captured), ordered after the
    // caller's earlier work and before its later work by two events
    cudaStream_t caller = as_stream(stream);
    cudaStream_t st = p->stream;
    SDP_CUDA_TRY(cudaEventRecord(p->ev_in, caller));
    SDP_CUDA_TRY(cudaStreamWaitEvent(st, p->ev_in, 0));
    // first with CLEAN as the cooperative kernel, then with one launch per
    // minor cycle, then eagerly
    for (int attempt = 0; attempt < 2 && p->cfg.use_graph && !p->graph_failed && !p->graph; ++attempt) {
        p->capture_persistent = attempt == 0;
        cudaGraph_t g = nullptr;
        cudaError_t e = cudaStreamBeginCapture(st, cudaStreamCaptureModeRelaxed);
        int status = SDP_OK;
        const char *where = "cudaStreamBeginCapture";
        if (e == cudaSuccess) {
            p->in_capture = 1;
            status = run_cycle(p, st);
            p->in_capture = 0;
            where = status != SDP_OK ? sdp_last_error() : "cudaStreamEndCapture";
            cudaError_t e2 = cudaStreamEndCapture(st, &g);
            if (status == SDP_OK) e = e2;
        }
        if (e == cudaSuccess && status == SDP_OK) {
            where = "cudaGraphInstantiate";
            e = cudaGraphInstantiate(&p->graph, g, 0);
        }
        if (g) cudaGraphDestroy(g);
        if (e != cudaSuccess || status != SDP_OK || !p->graph) {
            snprintf(p->graph_error, sizeof(p->graph_error), "%s: %s", where,
                     e != cudaSuccess ? cudaGetErrorString(e) : "launch failed during capture");
            cudaGetLastError();
            sdp_clear_error();
            p->graph = nullptr;
            // (the message of a refused first attempt stays readable through
            // sdp_pipeline_graph_error when the second succeeds)
            if (attempt == 0) continue;
            // capture refused (or a launch inside it failed): run eagerly from now on
            p->graph_failed = 1;
        }
    }
    if (p->graph) {
        SDP_CUDA_TRY(cudaGraphLaunch(p->graph, st));
    } else {
        SDP_TRY(run_cycle(p, st));
    }
    SDP_CUDA_TRY(cudaEventRecord(p->ev_out, st));
    SDP_CUDA_TRY(cudaStreamWaitEvent(caller, p->ev_out, 0));
    p->cycles_run += 1;
    return SDP_OK;
}

SDP_EXPORT int sdp_pipeline_outputs(sdp_pipeline *p, float **residual_image, float **model_image,
                                    sdp_float3 **sources, int **num_sources)
{
    SDP_CHECK_ARG(p, "pipeline is NULL");
    if (residual_image) *residual_image = p->residual_image;
    if (model_image) *model_image = p->model_image;
    if (sources) *sources = p->sources;
    if (num_sources) *num_sources = p->num_sources;
    return SDP_OK;
}

SDP_EXPORT int sdp_pipeline_copy_outputs(sdp_pipeline *p, float *residual_image, float *model_image,
                                         sdp_float3 *sources, int *num_sources, void *stream)
{
    SDP_CHECK_ARG(p, "pipeline is NULL");
    cudaStream_t st = as_stream(stream);
    const size_t G2 = (size_t)p->cfg.grid_size * p->cfg.grid_size;
    if (residual_image)
        SDP_CUDA_TRY(cudaMemcpyAsync(residual_image, p->residual_image, sizeof(float) * G2, cudaMemcpyDefault, st));
    if (model_image)
        SDP_CUDA_TRY(cudaMemcpyAsync(model_image, p->model_image, sizeof(float) * G2, cudaMemcpyDefault, st));
    if (sources && p->cfg.max_sources > 0)
        SDP_CUDA_TRY(cudaMemcpyAsync(sources, p->sources, sizeof(sdp_float3) * (size_t)p->cfg.max_sources,
                                     cudaMemcpyDefault, st));
    if (num_sources) SDP_CUDA_TRY(cudaMemcpyAsync(num_sources, p->num_sources, sizeof(int), cudaMemcpyDefault, st));
    SDP_CUDA_TRY(cudaStreamSynchronize(st));
    return SDP_OK;
}

SDP_EXPORT int sdp_pipeline_graph_active(const sdp_pipeline *p) { return (p && p->graph) ? 1 : 0; }

SDP_EXPORT const char *sdp_pipeline_graph_error(const sdp_pipeline *p) { return p ? p->graph_error : ""; }

SDP_EXPORT int sdp_pipeline_visplan(sdp_pipeline *p, sdp_visplan **plan)
{
    SDP_CHECK_ARG(p && plan, "NULL argument");
    *plan = p->plan;
    return SDP_OK;
}

SDP_EXPORT int sdp_pipeline_destroy(sdp_pipeline *p)
{
    if (!p) return SDP_OK;
    if (p->stream) cudaStreamSynchronize(p->stream);
    if (p->graph) cudaGraphExecDestroy(p->graph);
    if (p->ev_in) cudaEventDestroy(p->ev_in);
    if (p->ev_out) cudaEventDestroy(p->ev_out);
    if (p->stream) cudaStreamDestroy(p->stream);
    if (p->plan) sdp_visplan_destroy(p->plan);
    if (p->arena) SDP_CUDA_TRY(cudaFree(p->arena));
    delete p;
    return SDP_OK;
}
