// On-chip ceilings measured on the device the library runs on, used as the
// denominators of roofline fractions for the kernels that HBM does not bound:
// the Hogbom pass reads the PSF from L2 and applies the reference's double
// precision update; the visibility kernels are bound by FP32 issue and
// shared memory.  Each measurement is one kernel launched `reps` times after
// a warm-up launch, timed with CUDA events on the caller's stream.

#include "common.cuh"

namespace sdp {
namespace {

constexpr int kPeakThreads = 512;
constexpr int kPeakBlocksPerSm = 4;  // 2048 threads per SM
constexpr int kChains = 8;           // independent dependency chains per thread

// 16-byte loads that skip L1 (ld.global.cg), grid-stride over a buffer that
// fits in L2, `passes` times.
__global__ void __launch_bounds__(kPeakThreads) k_peak_l2(const uint4 *__restrict__ buf, long long n16, int passes,
                                                          unsigned *sink)
{
    unsigned acc = 0;
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (int p = 0; p < passes; ++p)
        for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n16; i += stride) {
            const uint4 v = __ldcg(buf + i);
            acc ^= v.x ^ v.y ^ v.z ^ v.w;
        }
    if (acc == 0x9e3779b9u) atomicAdd(sink, 1u);  // keeps the loads; practically never taken
}

// 16-byte shared-memory loads, conflict-free (consecutive threads, consecutive
// 16-byte words), `iters` sweeps over a 32 KB array.
__global__ void __launch_bounds__(kPeakThreads) k_peak_smem(int iters, unsigned seed, unsigned *sink)
{
    __shared__ uint4 s[2048];
    for (int k = threadIdx.x; k < 2048; k += blockDim.x) s[k] = make_uint4(seed + k, k, seed ^ k, 3u * k);
    __syncthreads();
    unsigned acc = 0;
    for (int it = 0; it < iters; ++it) {
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const uint4 v = s[(threadIdx.x + j * kPeakThreads + it) & 2047];
            acc ^= v.x ^ v.y ^ v.z ^ v.w;
        }
    }
    if (acc == 0x9e3779b9u) atomicAdd(sink, 1u);
}

// Scalar FFMA: kChains independent chains per thread.
__global__ void __launch_bounds__(kPeakThreads) k_peak_ffma(int iters, float a, float b, float *sink)
{
    float x[kChains];
#pragma unroll
    for (int j = 0; j < kChains; ++j) x[j] = (float)(threadIdx.x + j);
    for (int it = 0; it < iters; ++it) {
#pragma unroll
        for (int u = 0; u < 4; ++u)
#pragma unroll
            for (int j = 0; j < kChains; ++j) x[j] = __fmaf_rn(x[j], a, b);
    }
    float s = 0.f;
#pragma unroll
    for (int j = 0; j < kChains; ++j) s += x[j];
    if (s == 1234.5f) sink[0] = s;
}

// Packed FFMA2 (two FP32 lanes per instruction).
__global__ void __launch_bounds__(kPeakThreads) k_peak_ffma2(int iters, float a, float b, float *sink)
{
    float2 x[kChains];
    const float2 a2 = make_float2(a, a), b2 = make_float2(b, b);
#pragma unroll
    for (int j = 0; j < kChains; ++j) x[j] = make_float2((float)(threadIdx.x + j), (float)(threadIdx.x - j));
    for (int it = 0; it < iters; ++it) {
#pragma unroll
        for (int u = 0; u < 4; ++u)
#pragma unroll
            for (int j = 0; j < kChains; ++j) x[j] = __ffma2_rn(x[j], a2, b2);
    }
    float s = 0.f;
#pragma unroll
    for (int j = 0; j < kChains; ++j) s += x[j].x + x[j].y;
    if (s == 1234.5f) sink[0] = s;
}

// The Hogbom residual update r <- float(double(r) - (scale * double(p)) * psf_max)
// (deconvolution_run.c:271 evaluated in the reference's types), kChains
// independent pixels per thread; each update's PSF sample is another chain's
// previous value so nothing is loop-invariant.
__global__ void __launch_bounds__(kPeakThreads) k_peak_update(int iters, double scale, double psf_max, float *sink)
{
    float r[kChains];
#pragma unroll
    for (int j = 0; j < kChains; ++j) r[j] = 1.0f + 1e-3f * (float)(threadIdx.x + j);
    for (int it = 0; it < iters; ++it) {
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            float p[kChains];
#pragma unroll
            for (int j = 0; j < kChains; ++j) p[j] = r[(j + 1) % kChains];
#pragma unroll
            for (int j = 0; j < kChains; ++j)
                r[j] = __double2float_rn(__dsub_rn((double)r[j], __dmul_rn(__dmul_rn(scale, (double)p[j]), psf_max)));
        }
    }
    float s = 0.f;
#pragma unroll
    for (int j = 0; j < kChains; ++j) s += r[j];
    if (s == 1234.5f) sink[0] = s;
}

}  // namespace
}  // namespace sdp

using namespace sdp;

SDP_EXPORT int sdp_peak_measure(int kind, void *scratch, size_t scratch_bytes, int reps, double *rate, void *stream)
{
    SDP_CHECK_ARG(rate, "NULL argument");
    SDP_CHECK_ARG(reps >= 1, "reps must be >= 1");
    SDP_CHECK_ARG(kind >= SDP_PEAK_L2_READ && kind <= SDP_PEAK_HOGBOM_UPDATE, "unknown peak kind %d", kind);
    SDP_CHECK_ARG(scratch && scratch_bytes >= 4096 && ((uintptr_t)scratch & 15u) == 0,
                  "scratch must be a 16-byte aligned device buffer of at least 4096 bytes");
    cudaStream_t st = as_stream(stream);
    const int grid = num_sms() * kPeakBlocksPerSm;
    const double threads = (double)grid * kPeakThreads;
    // the first 16 bytes are the sink; the L2 buffer follows
    unsigned *usink = static_cast<unsigned *>(scratch);
    float *fsink = static_cast<float *>(scratch);
    const uint4 *buf = static_cast<const uint4 *>(scratch) + 1;
    const long long n16 = (long long)(scratch_bytes / 16) - 1;
    const int l2_passes = 8, smem_iters = 4096, fma_iters = 8192, upd_iters = 1024;
    double work = 0.0;  // units per launch
    auto launch = [&]() {
        switch (kind) {
        case SDP_PEAK_L2_READ:
            k_peak_l2<<<grid, kPeakThreads, 0, st>>>(buf, n16, l2_passes, usink);
            work = 16.0 * (double)n16 * l2_passes;
            break;
        case SDP_PEAK_SMEM_READ:
            k_peak_smem<<<grid, kPeakThreads, 0, st>>>(smem_iters, 7u, usink);
            work = threads * smem_iters * 4.0 * 16.0;
            break;
        case SDP_PEAK_FP32_FMA:
            k_peak_ffma<<<grid, kPeakThreads, 0, st>>>(fma_iters, 0.999f, 1e-3f, fsink);
            work = threads * fma_iters * 4.0 * kChains * 2.0;
            break;
        case SDP_PEAK_FP32X2_FMA:
            k_peak_ffma2<<<grid, kPeakThreads, 0, st>>>(fma_iters, 0.999f, 1e-3f, fsink);
            work = threads * fma_iters * 4.0 * kChains * 4.0;
            break;
        default:
            k_peak_update<<<grid, kPeakThreads, 0, st>>>(upd_iters, 1e-3, 0.5, fsink);
            work = threads * upd_iters * 4.0 * kChains;
            break;
        }
    };
    cudaEvent_t e0, e1;
    SDP_CUDA_TRY(cudaEventCreate(&e0));
    if (cudaEventCreate(&e1) != cudaSuccess) {
        cudaEventDestroy(e0);
        return cuda_error(cudaErrorMemoryAllocation, "cudaEventCreate");
    }
    launch();  // warm-up (also brings the L2 buffer on chip)
    cudaEventRecord(e0, st);
    for (int i = 0; i < reps; ++i) launch();
    cudaEventRecord(e1, st);
    cudaError_t err = cudaGetLastError();
    if (err == cudaSuccess) err = cudaEventSynchronize(e1);
    float ms = 0.f;
    if (err == cudaSuccess) err = cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    SDP_CUDA_TRY(err);
    *rate = ms > 0.f ? work * reps / (ms * 1e-3) : 0.0;
    return SDP_OK;
}
