// Restoring the model with the clean beam, and the image writers
// (param_code/code_fft_1core/src/major_loop_iter.c):
//   conv2D                        :8-46   result = model (*) clean PSF window
//   save_image_to_file            :168-199
//   save_extracted_sources_actor  :201-224
//   save_output                   :253-278
//
// conv2D visits every model pixel >= 1e-5 in row-major order and adds
// model * psf[(c - fy) G + (c - fx)], c = G/2 + 1, for each offset (fy, fx)
// in [-hy, hy) x [-hx, hx) that lands inside the image.  On the GPU each
// output pixel gathers instead: the model pixels that contribute to it lie in
// rows (y - hy, y + hy], so a compacted per-row list of the contributing
// pixels (in column order) is built first and every output pixel walks it in
// row-major order, adding with the same float products and the same order of
// additions as the reference (no FMA contraction).  The result is bit-exact.
//
// The writers format "%f, " per pixel and a newline per row, as the
// reference's fprintf loop does, but format blocks of rows on all host
// threads (snprintf, so the digits are libc's) and write them in order.
#include <cstdio>
#include <cstring>

#include <algorithm>
#include <string>
#include <thread>
#include <vector>

#include "internal.cuh"

namespace sdp {

constexpr int kRestoreThreads = 256;

__device__ __forceinline__ bool contributes(float v) { return !((double)v < 1e-5); }  // :19, in double (NaN contributes)

// Count of contributing pixels per row (one block per row).
__global__ void k_row_count_exact(int G, const float *__restrict__ model, int *__restrict__ cnt)
{
    __shared__ int s[32];
    const int y = blockIdx.x;
    int c = 0;
    for (int x = threadIdx.x; x < G; x += blockDim.x) c += contributes(model[(size_t)y * G + x]) ? 1 : 0;
    for (int o = 16; o > 0; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
    if ((threadIdx.x & 31) == 0) s[threadIdx.x >> 5] = c;
    __syncthreads();
    if (threadIdx.x < 32) {
        c = threadIdx.x < (blockDim.x >> 5) ? s[threadIdx.x] : 0;
        for (int o = 16; o > 0; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
        if (threadIdx.x == 0) cnt[y] = c;
    }
}

// Exclusive scan of the G row counts into off[0..G] (one block).
__global__ void k_row_scan(int G, const int *__restrict__ cnt, int *__restrict__ off)
{
    __shared__ int s[1024];
    const int per = (G + blockDim.x - 1) / blockDim.x;
    const int b = threadIdx.x * per;
    int sum = 0;
    for (int i = 0; i < per; ++i)
        if (b + i < G) sum += cnt[b + i];
    s[threadIdx.x] = sum;
    __syncthreads();
    for (int o = 1; o < (int)blockDim.x; o <<= 1) {
        const int v = threadIdx.x >= (unsigned)o ? s[threadIdx.x - o] : 0;
        __syncthreads();
        s[threadIdx.x] += v;
        __syncthreads();
    }
    int run = s[threadIdx.x] - sum;
    for (int i = 0; i < per; ++i)
        if (b + i < G) {
            off[b + i] = run;
            run += cnt[b + i];
        }
    if (threadIdx.x == blockDim.x - 1) off[G] = s[threadIdx.x];
}

// Contributing pixels of row y, in column order: (x, value) at off[y]...
// (one warp per row, a ballot per 32 columns).
__global__ void k_row_fill(int G, const float *__restrict__ model, const int *__restrict__ off, int2 *__restrict__ list)
{
    const int y = blockIdx.x * (blockDim.x / 32) + (threadIdx.x >> 5);
    const int lane = threadIdx.x & 31;
    if (y >= G) return;
    int pos = off[y];
    for (int x0 = 0; x0 < G; x0 += 32) {
        const int x = x0 + lane;
        const float v = x < G ? model[(size_t)y * G + x] : 0.f;
        const bool c = x < G && contributes(v);
        const unsigned m = __ballot_sync(0xffffffffu, c);
        if (c) list[pos + __popc(m & ((1u << lane) - 1u))] = make_int2(x, __float_as_int(v));
        pos += __popc(m);
    }
}

// One thread per output pixel: sum over contributing model pixels q with
// (y - qy, x - qx) in [-hy, hy) x [-hx, hx), in row-major order of q.
__global__ void __launch_bounds__(kRestoreThreads) k_restore(int G, int hx, int hy, const int *__restrict__ off,
                                                             const int2 *__restrict__ list,
                                                             const float *__restrict__ psf, float *__restrict__ out)
{
    const long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= (long long)G * G) return;
    const int y = (int)(p / G), x = (int)(p % G);
    const int c = G / 2 + 1;
    const long long g2 = (long long)G * G;
    float acc = 0.f;
    const int qy0 = max(0, y - hy + 1), qy1 = min(G - 1, y + hy);
    for (int qy = qy0; qy <= qy1; ++qy) {
        const int fy = y - qy;
        const int b = off[qy], e = off[qy + 1];
        for (int k = b; k < e; ++k) {
            const int2 q = __ldg(&list[k]);
            const int fx = x - q.x;
            if (fx >= hx) continue;   // q left of the window
            if (fx < -hx) break;      // the rest of the row is right of it
            const long long fi = (long long)(c - fy) * G + (c - fx);
            const float f = (fi >= 0 && fi < g2) ? __ldg(&psf[fi]) : 0.f;
            acc = __fadd_rn(acc, __fmul_rn(__int_as_float(q.y), f));
        }
    }
    out[p] = acc;
}

size_t restore_workspace_bytes(int G)
{
    const size_t rows = ((sizeof(int) * (2 * (size_t)G + 1) + 255) / 256) * 256;
    return rows + sizeof(int2) * (size_t)G * G;
}

}  // namespace sdp

using namespace sdp;

SDP_EXPORT int sdp_restore_workspace_bytes(int grid_size, size_t *bytes)
{
    SDP_CHECK_ARG(grid_size >= 1 && bytes, "bad argument");
    *bytes = restore_workspace_bytes(grid_size);
    return SDP_OK;
}

SDP_EXPORT int sdp_restore(int grid_size, const float *model, const float *clean_psf, int half_x, int half_y,
                           float *result, void *workspace, size_t workspace_bytes, void *stream)
{
    const int G = grid_size;
    SDP_CHECK_ARG(G >= 1 && model && clean_psf && result && workspace, "bad argument");
    SDP_CHECK_ARG(half_x >= 0 && half_y >= 0, "negative half dimensions (%d, %d)", half_x, half_y);
    SDP_CHECK_ARG(model != result, "model and result must not alias");
    if (workspace_bytes < restore_workspace_bytes(G))
        return set_error(SDP_ERR_RANGE, "restore workspace %zu B < %zu B", workspace_bytes, restore_workspace_bytes(G));
    cudaStream_t st = as_stream(stream);
    char *w = static_cast<char *>(workspace);
    int *cnt = reinterpret_cast<int *>(w);
    int *off = cnt + G;
    int2 *list = reinterpret_cast<int2 *>(w + ((sizeof(int) * (2 * (size_t)G + 1) + 255) / 256) * 256);
    k_row_count_exact<<<G, 256, 0, st>>>(G, model, cnt);
    k_row_scan<<<1, 1024, 0, st>>>(G, cnt, off);
    k_row_fill<<<(G + 7) / 8, 256, 0, st>>>(G, model, off, list);
    const long long n = (long long)G * G;
    k_restore<<<(unsigned)((n + kRestoreThreads - 1) / kRestoreThreads), kRestoreThreads, 0, st>>>(
        G, half_x, half_y, off, list, clean_psf, result);
    SDP_LAUNCH_CHECK();
    return SDP_OK;
}

// ---------------------------------------------------------------------------
// Host side: the reference's conv2D and writers
// ---------------------------------------------------------------------------
namespace {

int restore_host(int G, const float *model, const float *psf, sdp_int2 half, float *out)
{
    ThreadCtx *ctx = nullptr;
    SDP_TRY(thread_ctx(&ctx));
    const size_t G2 = (size_t)G * G;
    void *dm = nullptr, *dp = nullptr, *dr = nullptr, *ws = nullptr;
    SDP_TRY(ctx_buffer(ctx, kSlotRestore + 0, sizeof(float) * G2, &dm));
    SDP_TRY(ctx_buffer(ctx, kSlotRestore + 1, sizeof(float) * G2, &dp));
    SDP_TRY(ctx_buffer(ctx, kSlotRestore + 2, sizeof(float) * G2, &dr));
    SDP_TRY(ctx_buffer(ctx, kSlotRestore + 3, restore_workspace_bytes(G), &ws));
    cudaStream_t st = ctx->stream;
    SDP_CUDA_TRY(cudaMemcpyAsync(dm, model, sizeof(float) * G2, cudaMemcpyHostToDevice, st));
    SDP_CUDA_TRY(cudaMemcpyAsync(dp, psf, sizeof(float) * G2, cudaMemcpyHostToDevice, st));
    SDP_TRY(sdp_restore(G, static_cast<float *>(dm), static_cast<float *>(dp), half.x, half.y,
                        static_cast<float *>(dr), ws, restore_workspace_bytes(G), st));
    SDP_CUDA_TRY(cudaMemcpyAsync(out, dr, sizeof(float) * G2, cudaMemcpyDeviceToHost, st));
    SDP_CUDA_TRY(cudaStreamSynchronize(st));
    return SDP_OK;
}

// fprintf(f, "%f, ", pixel) per pixel and "\n" per row (:185-196), rows
// formatted on all host threads and written in order.
void write_image(const sdp_config *config, const float *image, const char *file_name, int start_x, int start_y,
                 int range_x, int range_y, int cycle)
{
    char path[256];
    snprintf(path, 255, "%scycle_%d_%s", config->output_path ? config->output_path : "", cycle,
             file_name ? file_name : "");
    printf("UPDATE >>> Attempting to save image to %s... \n\n", path);
    FILE *f = fopen(path, "w");
    if (!f) {
        printf(">>> ERROR: Unable to save image to file %s, check file/folder structure exists...\n\n", path);
        return;
    }
    const int rows = range_y;
    unsigned nt = std::max(1u, std::min(32u, std::thread::hardware_concurrency()));
    if ((long long)range_x * range_y < 65536) nt = 1;
    const int block = 64;  // rows per formatting task
    for (int r0 = 0; r0 < rows; r0 += block * (int)nt) {
        std::vector<std::string> out(nt);
        auto work = [&](unsigned t) {
            const int b = r0 + (int)t * block, e = std::min(rows, b + block);
            std::string &s = out[t];
            char tmp[64];
            for (int row = start_y + b; row < start_y + e; ++row) {
                for (int col = start_x; col < start_x + range_x; ++col) {
                    const int n = snprintf(tmp, sizeof(tmp), "%f, ", (double)image[(size_t)row * range_x + col]);
                    s.append(tmp, (size_t)n);
                }
                s.push_back('\n');
            }
        };
        std::vector<std::thread> th;
        for (unsigned t = 1; t < nt; ++t) th.emplace_back(work, t);
        work(0);
        for (auto &x : th) x.join();
        for (auto &s : out) fwrite(s.data(), 1, s.size(), f);
    }
    fclose(f);
}

}  // namespace

SDP_EXPORT void conv2D(float *image, float *filter, float *result, int IMAGE_DIM, sdp_int2 filter_half_dims)
{
    if (!image || !filter || !result || IMAGE_DIM < 1) {
        set_error(SDP_ERR_INVALID, "bad argument");
        actor_fail("conv2D");
        return;
    }
    if (restore_host(IMAGE_DIM, image, filter, filter_half_dims, result) != SDP_OK) actor_fail("conv2D");
}

SDP_EXPORT void save_image_to_file(sdp_config *config, float *image, const char *file_name, int start_x, int start_y,
                                   int range_x, int range_y, int cycle)
{
    write_image(config, image, file_name, start_x, start_y, range_x, range_y, cycle);
}

SDP_EXPORT void save_output(int GRID_SIZE, float *residual, float *model, float *clean_psf, sdp_int2 *clean_psf_halfdims,
                            float *psf, sdp_config *config, int *cycle)
{
    const int G = GRID_SIZE;
    write_image(config, residual, config->residual_image_output, 0, 0, G, G, *cycle);
    write_image(config, psf, config->psf_image_output, 0, 0, G, G, *cycle);
    write_image(config, clean_psf, config->clean_psf_image_output, 0, 0, G, G, *cycle);
    write_image(config, model, config->model_image_output, 0, 0, G, G, *cycle);
    std::vector<float> final_image((size_t)G * G);
    if (restore_host(G, model, clean_psf, *clean_psf_halfdims, final_image.data()) != SDP_OK) {
        actor_fail("save_output");
        return;
    }
    write_image(config, final_image.data(), config->final_image_output, 0, 0, G, G, *cycle);
}

SDP_EXPORT void save_extracted_sources_actor(int GRID_SIZE, int SAVE_EXTRACTED_SOURCES, int NUM_MAX_SOURCES,
                                             int *num_sources, sdp_float3 *sources, int *cycle_count,
                                             sdp_config *config, float *image_in, float *clean_psf,
                                             sdp_int2 *clean_psf_halfdims, float *image_out)
{
    (void)SAVE_EXTRACTED_SOURCES;
    (void)NUM_MAX_SOURCES;
    const int G = GRID_SIZE;
    memcpy(image_out, image_in, sizeof(float) * (size_t)G * G);
    const float cell = (float)config->cell_size;
    for (int i = 0; i < *num_sources; ++i) {  // :209-215
        const int row = (int)roundf(sources[i].y / cell + (float)(G / 2));
        const int col = (int)roundf(sources[i].x / cell + (float)(G / 2));
        image_out[col + row * G] += sources[i].z;
    }
    std::vector<float> conv((size_t)G * G);
    if (restore_host(G, image_out, clean_psf, *clean_psf_halfdims, conv.data()) != SDP_OK) {
        actor_fail("save_extracted_sources_actor");
        return;
    }
    write_image(config, conv.data(), config->model_sources_output, 0, 0, G, G, *cycle_count);
}
