// Status reporting and the per-thread context of the actor layer.
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>

#include "common.cuh"

namespace sdp {

namespace {
thread_local int t_status = SDP_OK;
thread_local char t_message[512] = {0};
int g_abort_on_error = -1;  // -1: read SDP_ABORT_ON_ERROR on first use

bool abort_on_error()
{
    if (g_abort_on_error < 0) {
        const char *e = getenv("SDP_ABORT_ON_ERROR");
        g_abort_on_error = (e && e[0] == '1') ? 1 : 0;
    }
    return g_abort_on_error == 1;
}

thread_local ThreadCtx t_ctx;
}  // namespace

int set_error(int status, const char *fmt, ...)
{
    t_status = status;
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(t_message, sizeof(t_message), fmt, ap);
    va_end(ap);
    return status;
}

int cuda_error(cudaError_t err, const char *what)
{
    int status = (err == cudaErrorMemoryAllocation) ? SDP_ERR_NOMEM : SDP_ERR_CUDA;
    return set_error(status, "%s: %s (%s)", what, cudaGetErrorName(err), cudaGetErrorString(err));
}

void actor_fail(const char *actor)
{
    if (abort_on_error()) {
        fprintf(stderr, "ERROR >>> %s: %s\n", actor, t_message);
        exit(EXIT_FAILURE);
    }
}

ThreadCtx::~ThreadCtx()
{
    // Buffers are released while the runtime is still alive (thread exit);
    // at process exit the driver reclaims them.
    for (auto &b : bufs)
        if (b.ptr) cudaFree(b.ptr);
    for (auto &e : ev)
        if (e) cudaEventDestroy(e);
    if (side) cudaStreamDestroy(side);
    if (stream) cudaStreamDestroy(stream);
}

int thread_ctx(ThreadCtx **out)
{
    ThreadCtx *c = &t_ctx;
    int dev = 0;
    SDP_CUDA_TRY(cudaGetDevice(&dev));
    if (c->stream == nullptr || c->device != dev) {
        if (c->stream) {
            for (auto &b : c->bufs) {
                if (b.ptr) cudaFree(b.ptr);
                b.ptr = nullptr;
                b.bytes = 0;
            }
            for (auto &e : c->ev) {
                if (e) cudaEventDestroy(e);
                e = nullptr;
            }
            if (c->side) cudaStreamDestroy(c->side);
            cudaStreamDestroy(c->stream);
            c->stream = nullptr;
            c->side = nullptr;
        }
        SDP_CUDA_TRY(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking));
        SDP_CUDA_TRY(cudaStreamCreateWithFlags(&c->side, cudaStreamNonBlocking));
        for (auto &e : c->ev) SDP_CUDA_TRY(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
        c->device = dev;
    }
    *out = c;
    return SDP_OK;
}

int ctx_buffer(ThreadCtx *ctx, int slot, size_t bytes, void **out)
{
    if (slot < 0 || slot >= (int)(sizeof(ctx->bufs) / sizeof(ctx->bufs[0])))
        return set_error(SDP_ERR_INVALID, "internal: buffer slot %d out of range", slot);
    DevBuf &b = ctx->bufs[slot];
    if (bytes == 0) bytes = 16;
    if (b.bytes < bytes) {
        if (b.ptr) {
            // the previous contents may still be in use by queued work
            SDP_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
            SDP_CUDA_TRY(cudaStreamSynchronize(ctx->side));
            SDP_CUDA_TRY(cudaFree(b.ptr));
            b.ptr = nullptr;
            b.bytes = 0;
        }
        size_t grown = bytes + bytes / 4;
        SDP_CUDA_TRY(cudaMalloc(&b.ptr, grown));
        b.bytes = grown;
    }
    *out = b.ptr;
    return SDP_OK;
}

int num_sms()
{
    static int cached[64] = {0};
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return 148;
    if (dev < 0 || dev >= 64) return 148;
    if (cached[dev] == 0) {
        int n = 0;
        if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || n <= 0) n = 148;
        cached[dev] = n;
    }
    return cached[dev];
}

}  // namespace sdp

SDP_EXPORT int sdp_last_status(void) { return sdp::t_status; }
SDP_EXPORT const char *sdp_last_error(void) { return sdp::t_message; }
SDP_EXPORT void sdp_clear_error(void)
{
    sdp::t_status = SDP_OK;
    sdp::t_message[0] = 0;
}
SDP_EXPORT void sdp_set_abort_on_error(int on) { sdp::g_abort_on_error = on ? 1 : 0; }
SDP_EXPORT int sdp_version(void) { return 10; }
