// Shared definitions for libsdp_b200: status handling, the per-thread
// context used by the actor drop-ins, and the index arithmetic that decides
// which grid cells a visibility touches.
//
// The index helpers reproduce the reference's C expressions operation by
// operation with explicitly rounded intrinsics (no fused multiply-add), so
// the set of taps, kernel samples and nearest cells chosen on the GPU is
// bit-identical to the reference's float build (PRECISION = float,
// param_code/code_fft_1core/include/common.h:62-71).  Config's uv_scale and
// w_scale are doubles, so the reference evaluates u * uv_scale in double and
// rounds to float when storing grid_pos (degridgrid.c:85).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>
#include <stddef.h>

#include "../../include/sdp_b200.h"

#define SDP_EXPORT extern "C" __attribute__((visibility("default")))

namespace sdp {

// ----------------------------------------------------------------------------
// Errors
// ----------------------------------------------------------------------------
int set_error(int status, const char *fmt, ...);  // records, returns status
int cuda_error(cudaError_t err, const char *what);  // maps a CUDA error
void actor_fail(const char *actor);                  // abort policy for actors

#define SDP_CUDA_TRY(expr)                                          \
    do {                                                            \
        cudaError_t _e = (expr);                                    \
        if (_e != cudaSuccess) return ::sdp::cuda_error(_e, #expr); \
    } while (0)

#define SDP_TRY(expr)                   \
    do {                                \
        int _s = (expr);                \
        if (_s != SDP_OK) return _s;    \
    } while (0)

#define SDP_CHECK_ARG(cond, ...)                                         \
    do {                                                                 \
        if (!(cond)) return ::sdp::set_error(SDP_ERR_INVALID, __VA_ARGS__); \
    } while (0)

inline cudaStream_t as_stream(void *s) { return reinterpret_cast<cudaStream_t>(s); }

// Launch check after a kernel launch.
#define SDP_LAUNCH_CHECK() SDP_CUDA_TRY(cudaGetLastError())

// ----------------------------------------------------------------------------
// Per-thread context for the actor layer: one non-blocking stream and a set
// of grow-only device buffers, so concurrent actor calls from several host
// threads (the reference's 6-thread schedule, code_g2g_6c) never share state.
// ----------------------------------------------------------------------------
struct DevBuf {
    void *ptr = nullptr;
    size_t bytes = 0;
};

struct ThreadCtx {
    cudaStream_t stream = nullptr;
    cudaStream_t side = nullptr;  // second stream: uploads that overlap work on `stream`
    cudaEvent_t ev[4] = {};       // ordering between the two (timing disabled)
    int device = -1;
    DevBuf bufs[24];
    ~ThreadCtx();
};

// Buffer slots 0 .. kSlotRestore-1 belong to the actor layer (actors.cu),
// kSlotRestore .. +3 to the restore / writer actors (restore.cu).
constexpr int kSlotRestore = 20;

int thread_ctx(ThreadCtx **out);
// Returns a device buffer of at least `bytes` for slot `slot` of this thread.
int ctx_buffer(ThreadCtx *ctx, int slot, size_t bytes, void **out);

int num_sms();

// ----------------------------------------------------------------------------
// Reference-exact index arithmetic (device and host)
// ----------------------------------------------------------------------------
#ifdef __CUDACC__
// grid_pos = (float)(u * uv_scale)                         degridgrid.c:85
__device__ __forceinline__ float ref_grid_pos(float u, double uv_scale)
{
    return __double2float_rn(__dmul_rn((double)u, uv_scale));
}

// w_idx = (int)(sqrtf(fabsf((float)(z * w_scale))) + 0.5)   degridgrid.c:84
__device__ __forceinline__ int ref_widx_std(float z, double w_scale)
{
    float a = fabsf(__double2float_rn(__dmul_rn((double)z, w_scale)));
    return __double2int_rz(__dadd_rn((double)__fsqrt_rn(a), 0.5));
}

// plane_index = (int)roundf(sqrtf(fabsf((float)(z * w_scale))))   gridding_run.c:67
__device__ __forceinline__ int ref_widx_round(float z, double w_scale)
{
    float a = fabsf(__double2float_rn(__dmul_rn((double)z, w_scale)));
    return (int)roundf(__fsqrt_rn(a));
}

// abs((int)roundf(((float)g - p) * os))                     degridgrid.c:101,110
__device__ __forceinline__ int ref_kidx(int g, float p, float os)
{
    return abs((int)roundf(__fmul_rn(__fsub_rn((float)g, p), os)));
}

// (int)((double)(p + (float)gc) + 0.5)                      degridgrid.c:194-195
__device__ __forceinline__ int ref_nearest(float p, int gc)
{
    return __double2int_rz(__dadd_rn((double)__fadd_rn(p, (float)gc), 0.5));
}

// roundf(p * os) / os                                       gridding_run.c:79-82
__device__ __forceinline__ float ref_snap(float p, int os)
{
    return __fdiv_rn(roundf(__fmul_rn(p, (float)os)), (float)os);
}

// The same expressions in the reference's double build (PRECISION = double,
// common.h:78-83, 114-134): every intermediate stays in double.
__device__ __forceinline__ double ref_grid_pos(double u, double uv_scale) { return __dmul_rn(u, uv_scale); }

__device__ __forceinline__ int ref_widx_std(double z, double w_scale)
{
    return __double2int_rz(__dadd_rn(__dsqrt_rn(fabs(__dmul_rn(z, w_scale))), 0.5));
}

__device__ __forceinline__ int ref_widx_round(double z, double w_scale)
{
    return (int)round(__dsqrt_rn(fabs(__dmul_rn(z, w_scale))));
}

__device__ __forceinline__ int ref_kidx(int g, double p, double os)
{
    return abs((int)round(__dmul_rn(__dsub_rn((double)g, p), os)));
}

__device__ __forceinline__ int ref_nearest(double p, int gc)
{
    return __double2int_rz(__dadd_rn(__dadd_rn(p, (double)gc), 0.5));
}

__device__ __forceinline__ double ref_snap(double p, int os)
{
    return __ddiv_rn(round(__dmul_rn(p, (double)os)), (double)os);
}

// correct_to_finegrid in PRECISION T (degridgrid.c:24-25, 52-54): the
// snapped coordinate as the build stores it.
template <typename T>
__device__ __forceinline__ T ref_finegrid(float u, int G, int os, double uv_scale)
{
    const double half = (double)(G / 2);
    const double t = __dadd_rn(__dmul_rn(__dadd_rn(__dmul_rn((double)u, uv_scale), half), (double)os), 0.5);
    const long long f = __double2ll_rz(t);
    return (T)__ddiv_rn(__dsub_rn(__ddiv_rn((double)f, (double)os), half), uv_scale);
}
#endif

}  // namespace sdp
