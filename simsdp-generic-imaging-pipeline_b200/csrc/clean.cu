// Hogbom CLEAN on the device, with the semantics of the live reference
// (preesm_pipelines/simsdp_fft_imaging_pipeline/Code/src/CPU/deconvolution_run.c:197-311):
//
//   per minor cycle: argmax |r| in row-major order (first index wins ties)
//   and the mean of |r| over indices >= 1 (the reference's running mean,
//   :226, divides by idx, which drops index 0); stop when
//   |max| < noise_factor * mean * gain or |max| < weak% * |first component|;
//   max_val = (float)(r[max] / psf_max); component (x, y, max_val * gain);
//   model[max] += max_val * gain; and r -= gain * max_val * psf * psf_max over
//   the window clipped to +-G/2, with the PSF mirrored in x and column index G
//   wrapping to the next row (:263-271).  psf[G*G] (one past the end, read
//   when the wrap hits the last row) is taken as 0.
//
// The products are evaluated in double in the reference's order and rounded
// to float where it assigns, so with the same residual the components and
// the model match the reference bit for bit; the mean is an FP64 sum instead
// of the reference's float recurrence, which only matters when |max| sits
// within rounding of the noise threshold.
//
// One minor cycle is two launches: k_clean_step applies the previous
// component's PSF subtraction and reduces (max, index, sum) per block in the
// same pass over the image; k_clean_select (one block) finishes the
// reduction, applies the stopping rule and records the component.  After a
// stop every later launch returns at once, so a fixed number of launches can
// be captured in a CUDA graph.
#include <algorithm>

#include "common.cuh"

namespace sdp {

struct CleanState {
    int stop;
    int count;
    int pending;   // a component whose PSF has not been subtracted yet
    int mx, my;
    float val;     // max_val of the pending component
    float first_z; // flux of the first component (the weak-source test, :239)
    int pad;
};

struct CleanWs {
    CleanState *st;
    float *pmax;
    int *pidx;
    double *psum;
    int nblocks;
};

constexpr int kCleanThreads = 256;

static int clean_blocks() { return num_sms() * 4; }

static void clean_layout(int nb, size_t *off, size_t *total)
{
    size_t o = 0;
    off[0] = o; o += 64;                                   // state
    off[1] = o; o += ((sizeof(double) * nb + 255) / 256) * 256;
    off[2] = o; o += ((sizeof(float) * nb + 255) / 256) * 256;
    off[3] = o; o += ((sizeof(int) * nb + 255) / 256) * 256;
    *total = o;
}

__device__ __forceinline__ void better(float &v, int &i, float v2, int i2)
{
    if (v2 > v || (v2 == v && i2 < i)) {
        v = v2;
        i = i2;
    }
}

// Subtract the pending component from r[i] (reference :266-272).
__device__ __forceinline__ void subtract_component(float *__restrict__ r, const float *__restrict__ psf, int G,
                                                   size_t i, const CleanState &s, double gain, double psf_max)
{
    const int y = (int)(i / G), x = (int)(i % G);
    const int half = G / 2;
    const int sx = min(s.mx, half), sy = min(s.my, half);
    const int ex = min(G - s.mx, half), ey = min(G - s.my, half);
    if (x < s.mx - sx || x >= s.mx + ex || y < s.my - sy || y >= s.my + ey) return;
    const long long pi = (long long)(y - s.my + half) * G + (G - (x - s.mx + half));
    const float pv = (pi < (long long)G * G) ? psf[pi] : 0.f;
    const double t = __dmul_rn(__dmul_rn(__dmul_rn(gain, (double)s.val), (double)pv), psf_max);
    r[i] = __double2float_rn(__dsub_rn((double)r[i], t));
}

__global__ void __launch_bounds__(kCleanThreads) k_clean_step(int G, float *__restrict__ r,
                                                             const float *__restrict__ psf, double gain,
                                                             double psf_max, CleanWs ws, int reduce)
{
    const CleanState s = *ws.st;
    if (s.stop && !s.pending) return;
    const size_t n = (size_t)G * G;
    float bv = -1.f;
    int bi = 0x7fffffff;
    double sum = 0.0;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        if (s.pending) subtract_component(r, psf, G, i, s, gain, psf_max);
        if (reduce) {
            const float a = fabsf(r[i]);
            better(bv, bi, a, (int)i);
            if (i >= 1) sum += (double)a;
        }
    }
    if (!reduce) return;
    __shared__ float sv[32];
    __shared__ int si[32];
    __shared__ double ss[32];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        float v2 = __shfl_xor_sync(0xffffffffu, bv, o);
        int i2 = __shfl_xor_sync(0xffffffffu, bi, o);
        better(bv, bi, v2, i2);
        sum += __shfl_xor_sync(0xffffffffu, sum, o);
    }
    if (lane == 0) {
        sv[wid] = bv;
        si[wid] = bi;
        ss[wid] = sum;
    }
    __syncthreads();
    if (wid == 0) {
        const int nw = blockDim.x / 32;
        bv = (lane < nw) ? sv[lane] : -1.f;
        bi = (lane < nw) ? si[lane] : 0x7fffffff;
        sum = (lane < nw) ? ss[lane] : 0.0;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            float v2 = __shfl_xor_sync(0xffffffffu, bv, o);
            int i2 = __shfl_xor_sync(0xffffffffu, bi, o);
            better(bv, bi, v2, i2);
            sum += __shfl_xor_sync(0xffffffffu, sum, o);
        }
        if (lane == 0) {
            ws.pmax[blockIdx.x] = bv;
            ws.pidx[blockIdx.x] = bi;
            ws.psum[blockIdx.x] = sum;
        }
    }
}

__global__ void k_clean_select(int G, int max_records, const float *__restrict__ r,
                               float *__restrict__ model, float3 *__restrict__ src, double gain, double noise,
                               double weak, double psf_max, CleanWs ws)
{
    CleanState *st = ws.st;
    if (st->stop) {
        if (threadIdx.x == 0) st->pending = 0;
        return;
    }
    float bv = -1.f;
    int bi = 0x7fffffff;
    double sum = 0.0;
    for (int b = threadIdx.x; b < ws.nblocks; b += blockDim.x) {
        better(bv, bi, ws.pmax[b], ws.pidx[b]);
        sum += ws.psum[b];
    }
    __shared__ float sv[32];
    __shared__ int si[32];
    __shared__ double ss[32];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        float v2 = __shfl_xor_sync(0xffffffffu, bv, o);
        int i2 = __shfl_xor_sync(0xffffffffu, bi, o);
        better(bv, bi, v2, i2);
        sum += __shfl_xor_sync(0xffffffffu, sum, o);
    }
    if (lane == 0) {
        sv[wid] = bv;
        si[wid] = bi;
        ss[wid] = sum;
    }
    __syncthreads();
    if (threadIdx.x != 0) return;
    const int nw = blockDim.x / 32;
    for (int w = 1; w < nw; ++w) {
        better(sv[0], si[0], sv[w], si[w]);
        ss[0] += ss[w];
    }
    float curr_max = sv[0];
    int idx = si[0];
    if (curr_max <= 0.f) {  // all zero (or empty): the reference keeps index 0
        curr_max = 0.f;
        idx = 0;
    }
    const long long n = (long long)G * G;
    const float avg = (n > 1) ? (float)(ss[0] / (double)(n - 1)) : 0.f;
    const bool extracting_noise = (double)fabsf(curr_max) < noise * (double)avg * gain;       // :238
    const bool weak_source = st->count > 0 && (double)fabsf(curr_max) < (double)fabsf(st->first_z) * weak;  // :239
    if (extracting_noise || weak_source) {
        st->stop = 1;
        st->pending = 0;
        return;
    }
    const float max_val = __double2float_rn(__ddiv_rn((double)r[idx], psf_max));          // :247
    const int mx = idx % G, my = idx / G;
    const float z = __double2float_rn(__dmul_rn((double)max_val, gain));
    if (st->count == 0) st->first_z = z;
    // the reference writes past MAX_SOURCES when NUM_MINOR_CYCLES exceeds it;
    // here cleaning continues and only the first max_records are stored
    if (st->count < max_records) src[st->count] = make_float3((float)mx, (float)my, z);
    st->count += 1;
    model[idx] = __double2float_rn(__dadd_rn((double)model[idx], __dmul_rn((double)max_val, gain)));  // :256
    st->pending = 1;
    st->mx = mx;
    st->my = my;
    st->val = max_val;
}

// :297-306: pixel coordinates to (x - G/2) * cell_size.
__global__ void k_clean_finish(int G, double cell, int max_records, float3 *__restrict__ src, CleanWs ws,
                               int *__restrict__ count_out)
{
    const int n = min(ws.st->count, max_records);
    for (int k = threadIdx.x; k < n; k += blockDim.x) {
        float3 s = src[k];
        s.x = __double2float_rn(__dmul_rn((double)__fsub_rn(s.x, (float)(G / 2)), cell));
        s.y = __double2float_rn(__dmul_rn((double)__fsub_rn(s.y, (float)(G / 2)), cell));
        src[k] = s;
    }
    if (threadIdx.x == 0 && count_out) *count_out = n;
}

}  // namespace sdp

using namespace sdp;

SDP_EXPORT int sdp_hogbom_workspace_bytes(int G, size_t *bytes)
{
    SDP_CHECK_ARG(bytes != nullptr && G >= 2, "bad argument");
    size_t off[4];
    clean_layout(clean_blocks(), off, bytes);
    return SDP_OK;
}

SDP_EXPORT int sdp_hogbom(const sdp_clean_params *p, float *residual, const float *psf, float *model,
                          sdp_float3 *sources, int *num_sources_dev, void *workspace, size_t ws_bytes, void *stream)
{
    SDP_CHECK_ARG(p && residual && psf && model && workspace, "NULL argument");
    SDP_CHECK_ARG(p->grid_size >= 2, "grid_size %d", p->grid_size);
    SDP_CHECK_ARG(p->num_minor_cycles >= 0, "num_minor_cycles %d", p->num_minor_cycles);
    SDP_CHECK_ARG(p->num_minor_cycles == 0 || sources, "sources is NULL");
    SDP_CHECK_ARG(p->psf_max_value != 0.0, "psf_max_value is 0");
    const int G = p->grid_size;
    const int nb = clean_blocks();
    size_t off[4], need;
    clean_layout(nb, off, &need);
    if (ws_bytes < need) return set_error(SDP_ERR_RANGE, "hogbom workspace %zu B < %zu B", ws_bytes, need);
    char *w = static_cast<char *>(workspace);
    CleanWs ws;
    ws.st = reinterpret_cast<CleanState *>(w + off[0]);
    ws.psum = reinterpret_cast<double *>(w + off[1]);
    ws.pmax = reinterpret_cast<float *>(w + off[2]);
    ws.pidx = reinterpret_cast<int *>(w + off[3]);
    ws.nblocks = nb;
    cudaStream_t st = as_stream(stream);
    SDP_CUDA_TRY(cudaMemsetAsync(ws.st, 0, sizeof(CleanState), st));
    // the stored component list is bounded by the caller's buffer (MAX_SOURCES)
    const int cap = std::max(0, std::min(p->num_minor_cycles, p->max_sources));
    float3 *src = reinterpret_cast<float3 *>(sources);
    for (int it = 0; it < p->num_minor_cycles; ++it) {
        k_clean_step<<<nb, kCleanThreads, 0, st>>>(G, residual, psf, p->loop_gain, p->psf_max_value, ws, 1);
        k_clean_select<<<1, 1024, 0, st>>>(G, cap, residual, model, src, p->loop_gain, p->noise_factor,
                                          p->weak_source_percent, p->psf_max_value, ws);
    }
    // subtract the last component so residual_inout is the final residual
    k_clean_step<<<nb, kCleanThreads, 0, st>>>(G, residual, psf, p->loop_gain, p->psf_max_value, ws, 0);
    k_clean_finish<<<1, 256, 0, st>>>(G, p->cell_size, cap, src, ws, num_sources_dev);
    SDP_LAUNCH_CHECK();
    return SDP_OK;
}

// ---------------------------------------------------------------------------
// Hogbom CLEAN without any device allocation.
//
// For callers that cannot call cudaMalloc: a dataflow runtime that, like the
// reference's PREESM schedule (one static arena, generated/Core0.c:19), fixes
// all of its memory before the schedule starts and must not take an
// allocator call (which can block and synchronise the device) in the middle
// of it, or a host program whose device memory is owned by another allocator.
// The caller still passes the residual, PSF, model and source buffers; the
// minor-cycle state and the per-block partial results live in the fixed
// array below, one per GPU, kept until the process exits.
// ---------------------------------------------------------------------------
#include <mutex>

namespace sdp {

constexpr int kNoAllocMaxGrid = 4096;  // grid_size limit of sdp_hogbom_noalloc
constexpr size_t kNoAllocStateBytes = 256;
// state + one (double sum, float max, int index) partial per image row
constexpr size_t kNoAllocScratchBytes = kNoAllocStateBytes + 16 * (size_t)kNoAllocMaxGrid;  // 65,792 B

static_assert(sizeof(CleanState) <= kNoAllocStateBytes, "CLEAN state must fit its slot");

static __device__ __align__(256) unsigned char g_clean_scratch[kNoAllocScratchBytes];

static std::mutex g_clean_scratch_mutex;
static void *g_clean_scratch_addr[128];

// Device address of g_clean_scratch on the current device, looked up once per
// device (the host-side name of the array is not a device address).
static int clean_scratch_address(void **out)
{
    int dev = 0;
    SDP_CUDA_TRY(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 128) return set_error(SDP_ERR_RANGE, "device ordinal %d beyond 127", dev);
    std::lock_guard<std::mutex> lock(g_clean_scratch_mutex);
    if (g_clean_scratch_addr[dev] == nullptr) {
        void *p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_clean_scratch);
        if (e != cudaSuccess) return cuda_error(e, "cudaGetSymbolAddress(g_clean_scratch)");
        g_clean_scratch_addr[dev] = p;
    }
    *out = g_clean_scratch_addr[dev];
    return SDP_OK;
}

}  // namespace sdp

SDP_EXPORT int sdp_hogbom_noalloc(const sdp_clean_params *p, float *residual, const float *psf, float *model,
                                  sdp_float3 *sources, int *num_sources_dev, void *stream)
{
    SDP_CHECK_ARG(p && residual && psf && model, "NULL argument");
    SDP_CHECK_ARG(p->grid_size >= 2, "grid_size %d", p->grid_size);
    if (p->grid_size > kNoAllocMaxGrid)
        return set_error(SDP_ERR_RANGE,
                         "sdp_hogbom_noalloc: grid_size %d exceeds its fixed scratch limit of %d; use sdp_hogbom",
                         p->grid_size, kNoAllocMaxGrid);
    SDP_CHECK_ARG(p->num_minor_cycles >= 0, "num_minor_cycles %d", p->num_minor_cycles);
    SDP_CHECK_ARG(p->num_minor_cycles == 0 || sources, "sources is NULL");
    SDP_CHECK_ARG(p->psf_max_value != 0.0, "psf_max_value is 0");
    const int G = p->grid_size;
    void *base = nullptr;
    SDP_TRY(clean_scratch_address(&base));  // first call on a device: symbol lookup
    char *w = static_cast<char *>(base);
    const int nb = G;  // one partial per block, G blocks
    CleanWs ws;
    ws.st = reinterpret_cast<CleanState *>(w);
    ws.psum = reinterpret_cast<double *>(w + kNoAllocStateBytes);
    ws.pmax = reinterpret_cast<float *>(w + kNoAllocStateBytes + 8 * (size_t)nb);
    ws.pidx = reinterpret_cast<int *>(w + kNoAllocStateBytes + 12 * (size_t)nb);
    ws.nblocks = nb;
    cudaStream_t st = as_stream(stream);
    // every call starts from a cleared state (the array keeps the last call's contents)
    SDP_CUDA_TRY(cudaMemsetAsync(ws.st, 0, sizeof(CleanState), st));
    const int cap = std::max(0, std::min(p->num_minor_cycles, p->max_sources));
    float3 *src = reinterpret_cast<float3 *>(sources);
    for (int it = 0; it < p->num_minor_cycles; ++it) {
        k_clean_step<<<nb, kCleanThreads, 0, st>>>(G, residual, psf, p->loop_gain, p->psf_max_value, ws, 1);
        k_clean_select<<<1, 1024, 0, st>>>(G, cap, residual, model, src, p->loop_gain, p->noise_factor,
                                          p->weak_source_percent, p->psf_max_value, ws);
    }
    k_clean_step<<<nb, kCleanThreads, 0, st>>>(G, residual, psf, p->loop_gain, p->psf_max_value, ws, 0);
    k_clean_finish<<<1, 256, 0, st>>>(G, p->cell_size, cap, src, ws, num_sources_dev);
    SDP_LAUNCH_CHECK();
    return SDP_OK;
}
