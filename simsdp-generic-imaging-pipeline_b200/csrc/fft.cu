// 2-D complex FFT (FFTW convention: sign -1 forward, +1 inverse,
// unnormalised; fft_run.c:23-83) and the fused imaging transforms of the
// FFT pipeline.
//
// A transform is a row pass and a column pass.  Each CTA loads whole lines
// (L rows, or C adjacent columns so global loads stay in 32-byte sectors) into
// shared memory in bit-reversed order and runs an in-place decimation-in-time
// FFT whose stages are taken two at a time (radix-2^2: one 4-point butterfly
// per pair of radix-2 stages, one barrier per pair), finishing with a single
// radix-2 stage when log2 N is odd.  Twiddles come from a per-size table of
// exp(-2 pi i k / N), k < N/2, built in double on the device.
//
// The checkerboard fftshift (fft_run.c:14, 96, 114) is applied while loading
// the first pass and while storing the second, and the taper correction
// (convolution_correction_run.c:4-35) is applied in the second pass's store,
// so grid -> image and image -> grid each cost two HBM round trips.
#include <algorithm>
#include <mutex>
#include <unordered_map>

#include "common.cuh"

namespace sdp {

enum { LOAD_PLAIN = 0, LOAD_CHECKER = 1, LOAD_REAL_CHECKER = 2 };
enum { STORE_PLAIN = 0, STORE_CHECKER = 1, STORE_REAL_CHECKER_TAPER = 2 };

constexpr int kFftThreads = 256;
constexpr int kFftSmemElems = 8192;  // complex elements per CTA (64 KB)

__global__ void k_twiddles(int N, float2 *tw)
{
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < N / 2; k += gridDim.x * blockDim.x) {
        double s, c;
        sincospi(__ddiv_rn(2.0 * (double)k, (double)N), &s, &c);
        tw[k] = make_float2((float)c, (float)(-s));
    }
}

__device__ __forceinline__ float2 cmulf(float2 a, float2 b)
{
    return make_float2(fmaf(a.x, b.x, -a.y * b.y), fmaf(a.x, b.y, a.y * b.x));
}

__device__ __forceinline__ float checker(int r, int c) { return ((r + c) & 1) ? -1.f : 1.f; }

// In-place FFT of `lines` lines of length N (power of two) held in smem in
// bit-reversed order.  inverse: conjugated twiddles.
__device__ __forceinline__ void smem_fft(float2 *s, int N, int log2n, int lines, const float2 *__restrict__ tw,
                                         bool inverse)
{
    const int quarter = N >> 2;
    const float tsign = inverse ? -1.f : 1.f;  // multiplies the imaginary part of tw
    int m = 1;
    int stages = log2n;
    for (; stages >= 2; stages -= 2, m <<= 2) {
        const int total = lines * quarter;
        const int sh1 = log2n - 1 - __ffs(m) + 1;  // N / (2m) = 1 << (log2n - 1 - log2 m)
        for (int q = threadIdx.x; q < total; q += blockDim.x) {
            const int l = q / quarter;
            const int qq = q - l * quarter;
            const int j = qq & (m - 1);
            const int g = qq / m;
            float2 *base = s + (size_t)l * N + g * 4 * m + j;
            float2 w1 = tw[j << sh1];
            float2 w2 = tw[j << (sh1 - 1)];
            w1.y *= tsign;
            w2.y *= tsign;
            const float2 a = base[0], b = base[m], c = base[2 * m], d = base[3 * m];
            const float2 b1 = cmulf(b, w1), d1 = cmulf(d, w1);
            const float2 ap = make_float2(a.x + b1.x, a.y + b1.y);
            const float2 bp = make_float2(a.x - b1.x, a.y - b1.y);
            const float2 cp = make_float2(c.x + d1.x, c.y + d1.y);
            const float2 dp = make_float2(c.x - d1.x, c.y - d1.y);
            const float2 c2 = cmulf(cp, w2);
            float2 d2 = cmulf(dp, w2);
            // times W_4^1 = -i (forward) or +i (inverse)
            d2 = inverse ? make_float2(-d2.y, d2.x) : make_float2(d2.y, -d2.x);
            base[0] = make_float2(ap.x + c2.x, ap.y + c2.y);
            base[2 * m] = make_float2(ap.x - c2.x, ap.y - c2.y);
            base[m] = make_float2(bp.x + d2.x, bp.y + d2.y);
            base[3 * m] = make_float2(bp.x - d2.x, bp.y - d2.y);
        }
        __syncthreads();
    }
    if (stages == 1) {  // final radix-2 stage, len = N
        const int half = N >> 1;
        const int total = lines * half;
        for (int q = threadIdx.x; q < total; q += blockDim.x) {
            const int l = q / half;
            const int j = q - l * half;
            float2 *base = s + (size_t)l * N + j;
            float2 w = tw[j];
            w.y *= tsign;
            const float2 a = base[0];
            const float2 t = cmulf(base[half], w);
            base[0] = make_float2(a.x + t.x, a.y + t.y);
            base[half] = make_float2(a.x - t.x, a.y - t.y);
        }
        __syncthreads();
    }
}

// One pass over all lines of a G x G array.  ROWS: lines are rows.
template <bool ROWS, int LOAD, int STORE>
__global__ void __launch_bounds__(kFftThreads) k_fft_pass(int G, int log2n, int lines_per_cta,
                                                         const void *__restrict__ in_, void *__restrict__ out_,
                                                         const float2 *__restrict__ tw, bool inverse,
                                                         const float *__restrict__ prolate)
{
    extern __shared__ float2 s[];
    const int N = G;
    const int L = lines_per_cta;
    const int first = blockIdx.x * L;
    const int total = L * N;
    // load (bit-reversed position within each line)
    for (int t = threadIdx.x; t < total; t += blockDim.x) {
        int l, i;
        if (ROWS) {
            l = t / N;
            i = t - l * N;
        } else {
            i = t / L;
            l = t - i * L;
        }
        const int r = ROWS ? first + l : i;
        const int c = ROWS ? i : first + l;
        const size_t gi = (size_t)r * G + c;
        float2 v;
        if (LOAD == LOAD_REAL_CHECKER) {
            v = make_float2(static_cast<const float *>(in_)[gi] * checker(r, c), 0.f);
        } else {
            v = static_cast<const float2 *>(in_)[gi];
            if (LOAD == LOAD_CHECKER) {
                const float a = checker(r, c);
                v.x *= a;
                v.y *= a;
            }
        }
        s[(size_t)l * N + (__brev((unsigned)i) >> (32 - log2n))] = v;
    }
    __syncthreads();
    smem_fft(s, N, log2n, L, tw, inverse);
    for (int t = threadIdx.x; t < total; t += blockDim.x) {
        int l, i;
        if (ROWS) {
            l = t / N;
            i = t - l * N;
        } else {
            i = t / L;
            l = t - i * L;
        }
        const int r = ROWS ? first + l : i;
        const int c = ROWS ? i : first + l;
        const size_t gi = (size_t)r * G + c;
        float2 v = s[(size_t)l * N + i];
        if (STORE == STORE_REAL_CHECKER_TAPER) {
            const float x = v.x * checker(r, c);
            const int half = G / 2;
            const int dc = abs(c - half), dr = abs(r - half);
            float taper = __fmul_rn(prolate[dc], prolate[dr]);
            if (dc == 1229 || dr == 1229) taper = 0.f;
            static_cast<float *>(out_)[gi] = ((double)fabsf(taper) > 1E-10) ? __fdiv_rn(x, taper) : 0.f;
        } else {
            if (STORE == STORE_CHECKER) {
                const float a = checker(r, c);
                v.x *= a;
                v.y *= a;
            }
            static_cast<float2 *>(out_)[gi] = v;
        }
    }
}

struct TwKey {
    int dev, n;
    bool operator==(const TwKey &o) const { return dev == o.dev && n == o.n; }
};
struct TwHash {
    size_t operator()(const TwKey &k) const { return (size_t)k.dev * 1000003u + (size_t)k.n; }
};

static std::mutex g_tw_mutex;
static std::unordered_map<TwKey, float2 *, TwHash> g_tw;

// Twiddle table for size N on the current device (allocated once, kept).
int fft_twiddles(int N, cudaStream_t st, const float2 **out)
{
    int dev = 0;
    SDP_CUDA_TRY(cudaGetDevice(&dev));
    std::lock_guard<std::mutex> lock(g_tw_mutex);
    auto it = g_tw.find({dev, N});
    if (it != g_tw.end()) {
        *out = it->second;
        return SDP_OK;
    }
    float2 *p = nullptr;
    SDP_CUDA_TRY(cudaMalloc(&p, sizeof(float2) * (size_t)std::max(1, N / 2)));
    k_twiddles<<<std::max(1, std::min(1024, N / 2 / 256 + 1)), 256, 0, st>>>(N, p);
    SDP_LAUNCH_CHECK();
    SDP_CUDA_TRY(cudaStreamSynchronize(st));
    g_tw[{dev, N}] = p;
    *out = p;
    return SDP_OK;
}

static int ilog2(int n)
{
    int l = 0;
    while ((1 << l) < n) ++l;
    return l;
}

int check_fft_size(int G)
{
    if (G < 16 || G > 16384 || (G & (G - 1)) != 0)
        return set_error(SDP_ERR_RANGE, "FFT size %d must be a power of two in [16, 16384]", G);
    return SDP_OK;
}

template <bool ROWS, int LOAD, int STORE>
static int launch_pass(int G, const void *in, void *out, const float2 *tw, bool inverse, const float *prolate,
                       cudaStream_t st)
{
    const int L = std::max(1, kFftSmemElems / G);
    const int lines = std::min(L, G);
    const size_t smem = sizeof(float2) * (size_t)lines * G;
    auto fn = k_fft_pass<ROWS, LOAD, STORE>;
    if (smem > 48 * 1024) SDP_CUDA_TRY(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    fn<<<G / lines, kFftThreads, smem, st>>>(G, ilog2(G), lines, in, out, tw, inverse, prolate);
    SDP_LAUNCH_CHECK();
    return SDP_OK;
}

}  // namespace sdp

using namespace sdp;

SDP_EXPORT int sdp_fft2d(int G, const sdp_float2 *in, sdp_float2 *out, int sign, void *stream)
{
    SDP_TRY(check_fft_size(G));
    SDP_CHECK_ARG(in && out, "NULL argument");
    SDP_CHECK_ARG(sign == -1 || sign == 1, "sign %d must be -1 or +1", sign);
    cudaStream_t st = as_stream(stream);
    const float2 *tw = nullptr;
    SDP_TRY(fft_twiddles(G, st, &tw));
    const bool inv = (sign == 1);
    SDP_TRY((launch_pass<true, LOAD_PLAIN, STORE_PLAIN>(G, in, out, tw, inv, nullptr, st)));
    SDP_TRY((launch_pass<false, LOAD_PLAIN, STORE_PLAIN>(G, out, out, tw, inv, nullptr, st)));
    return SDP_OK;
}

SDP_EXPORT int sdp_grid_to_image(int G, const sdp_float2 *grid, const float *prolate_ext, sdp_float2 *work,
                                 float *image, void *stream)
{
    SDP_TRY(check_fft_size(G));
    SDP_CHECK_ARG(grid && prolate_ext && work && image, "NULL argument");
    cudaStream_t st = as_stream(stream);
    const float2 *tw = nullptr;
    SDP_TRY(fft_twiddles(G, st, &tw));
    SDP_TRY((launch_pass<true, LOAD_CHECKER, STORE_PLAIN>(G, grid, work, tw, true, nullptr, st)));
    SDP_TRY((launch_pass<false, LOAD_PLAIN, STORE_REAL_CHECKER_TAPER>(G, work, image, tw, true, prolate_ext, st)));
    return SDP_OK;
}

SDP_EXPORT int sdp_image_to_grid(int G, const float *image, sdp_float2 *work, sdp_float2 *grid, void *stream)
{
    SDP_TRY(check_fft_size(G));
    SDP_CHECK_ARG(image && work && grid, "NULL argument");
    cudaStream_t st = as_stream(stream);
    const float2 *tw = nullptr;
    SDP_TRY(fft_twiddles(G, st, &tw));
    SDP_TRY((launch_pass<true, LOAD_REAL_CHECKER, STORE_PLAIN>(G, image, work, tw, false, nullptr, st)));
    SDP_TRY((launch_pass<false, LOAD_PLAIN, STORE_CHECKER>(G, work, grid, tw, false, nullptr, st)));
    return SDP_OK;
}
