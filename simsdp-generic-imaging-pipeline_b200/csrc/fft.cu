// 2-D complex FFT (FFTW convention: sign -1 forward, +1 inverse,
// unnormalised; fft_run.c:23-83) and the fused imaging transforms of the
// FFT pipeline.
//
// A transform is a row pass and a column pass.  Each CTA owns whole lines
// (L rows, or C adjacent columns so that global loads stay in full 32-byte
// sectors) and runs a Stockham autosort FFT: N = R1 R2 ... with radices 16
// (then 8, 4 or 2 for the remainder), one stage per radix.  In a stage each
// thread takes R elements at stride N/R, multiplies element t by the twiddle
// W_{Ns R}^{t k} (k = butterfly index mod the span Ns done so far), does an
// R-point DFT in registers (16 = 4 x 4, 8 = 2 x 4) and writes the outputs
// to their sorted places; shared memory is touched once per stage, and the
// first stage reads, the last stage writes global memory directly.
// Twiddles come from a per-size table of exp(-2 pi i k / N), built in double.
//
// The checkerboard fftshift (fft_run.c:14, 96, 114) is applied while the
// first pass loads and while the second pass stores, and the taper
// correction (convolution_correction_run.c:4-35) in the second pass's
// store, so grid -> image and image -> grid each cost two HBM round trips.
#include <algorithm>
#include <mutex>
#include <unordered_map>

#include "common.cuh"

namespace sdp {

enum { LOAD_PLAIN = 0, LOAD_CHECKER = 1, LOAD_REAL_CHECKER = 2 };
enum { STORE_PLAIN = 0, STORE_CHECKER = 1, STORE_REAL_CHECKER_TAPER = 2 };

constexpr int kFftSmemElems = 8192;  // complex elements per CTA (64 KB)
__global__ void k_twiddles(int N, float2 *tw)
{
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < N; k += gridDim.x * blockDim.x) {
        double s, c;
        sincospi(__ddiv_rn(2.0 * (double)k, (double)N), &s, &c);
        tw[k] = make_float2((float)c, (float)(-s));
    }
}

__device__ __forceinline__ float2 cadd(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ float2 csub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ float2 cmulf(float2 a, float2 b)
{
    return make_float2(fmaf(a.x, b.x, -a.y * b.y), fmaf(a.x, b.y, a.y * b.x));
}
// times -i (forward, sg = 1) or +i (inverse, sg = -1)
__device__ __forceinline__ float2 rot90(float2 a, float sg) { return make_float2(sg * a.y, -sg * a.x); }

__device__ __forceinline__ void dft2(float2 &a, float2 &b)
{
    const float2 t = a;
    a = cadd(t, b);
    b = csub(t, b);
}

__device__ __forceinline__ void dft4(float2 &a0, float2 &a1, float2 &a2, float2 &a3, float sg)
{
    const float2 t0 = cadd(a0, a2), t1 = csub(a0, a2);
    const float2 t2 = cadd(a1, a3), t3 = rot90(csub(a1, a3), sg);
    a0 = cadd(t0, t2);
    a2 = csub(t0, t2);
    a1 = cadd(t1, t3);
    a3 = csub(t1, t3);
}

// exp(-sg 2 pi i j / 16) for j = 0..15 written as constants of cos/sin(pi j / 8)
__device__ __forceinline__ float2 w16(int j, float sg)
{
    const float c1 = 0.92387953251128674f, s1 = 0.38268343236508978f, h = 0.70710678118654752f;
    float2 w;
    switch (j & 15) {
    case 0: w = make_float2(1.f, 0.f); break;
    case 1: w = make_float2(c1, -s1); break;
    case 2: w = make_float2(h, -h); break;
    case 3: w = make_float2(s1, -c1); break;
    case 4: w = make_float2(0.f, -1.f); break;
    case 5: w = make_float2(-s1, -c1); break;
    case 6: w = make_float2(-h, -h); break;
    case 7: w = make_float2(-c1, -s1); break;
    case 8: w = make_float2(-1.f, 0.f); break;
    case 9: w = make_float2(-c1, s1); break;
    case 10: w = make_float2(-h, h); break;
    case 11: w = make_float2(-s1, c1); break;
    case 12: w = make_float2(0.f, 1.f); break;
    case 13: w = make_float2(s1, c1); break;
    case 14: w = make_float2(h, h); break;
    default: w = make_float2(c1, s1); break;
    }
    w.y *= sg;
    return w;
}

// In-register R-point DFT (natural order in and out); sg = 1 forward, -1 inverse.
template <int R>
__device__ __forceinline__ void dft_r(float2 (&a)[R], float sg)
{
    if (R == 2) {
        dft2(a[0], a[1]);
    } else if (R == 4) {
        dft4(a[0], a[1], a[2], a[3], sg);
    } else if (R == 8) {
        // n = m + 2 l (m < 2, l < 4); k = k1 + 4 k2
        dft4(a[0], a[2], a[4], a[6], sg);
        dft4(a[1], a[3], a[5], a[7], sg);
        // twiddle W8^{k1} on the odd half, then 2-point DFTs
#pragma unroll
        for (int k1 = 0; k1 < 4; ++k1) {
            float2 o = a[2 * k1 + 1];
            if (k1) o = cmulf(o, w16(2 * k1, sg));
            const float2 e = a[2 * k1];
            a[2 * k1] = cadd(e, o);
            a[2 * k1 + 1] = csub(e, o);
        }
        // X[k1] is in a[2 k1], X[k1 + 4] in a[2 k1 + 1]
        const float2 x0 = a[0], x4 = a[1], x1 = a[2], x5 = a[3], x2 = a[4], x6 = a[5], x3 = a[6], x7 = a[7];
        a[0] = x0; a[1] = x1; a[2] = x2; a[3] = x3; a[4] = x4; a[5] = x5; a[6] = x6; a[7] = x7;
    } else if (R == 16) {
        // n = m + 4 l; inner DFT4 over l for each m, twiddle W16^{m k1}, outer DFT4 over m
#pragma unroll
        for (int m = 0; m < 4; ++m) dft4(a[m], a[m + 4], a[m + 8], a[m + 12], sg);
#pragma unroll
        for (int m = 1; m < 4; ++m)
#pragma unroll
            for (int k1 = 1; k1 < 4; ++k1) a[m + 4 * k1] = cmulf(a[m + 4 * k1], w16(m * k1, sg));
#pragma unroll
        for (int k1 = 0; k1 < 4; ++k1) dft4(a[4 * k1], a[4 * k1 + 1], a[4 * k1 + 2], a[4 * k1 + 3], sg);
        // a[4 k1 + k2] holds X[k1 + 4 k2]: transpose the 4 x 4 index
        float2 t[16];
#pragma unroll
        for (int k1 = 0; k1 < 4; ++k1)
#pragma unroll
            for (int k2 = 0; k2 < 4; ++k2) t[k1 + 4 * k2] = a[4 * k1 + k2];
#pragma unroll
        for (int i = 0; i < 16; ++i) a[i] = t[i];
    }
}

__device__ __forceinline__ float checker(int r, int c) { return ((r + c) & 1) ? -1.f : 1.f; }

// Element addressing of a pass: line l (row or column index within the
// CTA's block), position i along the line.
template <bool ROWS>
struct Lines {
    int G, first, L;
    __device__ __forceinline__ int row(int l, int i) const { return ROWS ? first + l : i; }
    __device__ __forceinline__ int col(int l, int i) const { return ROWS ? i : first + l; }
    // shared memory: rows line-major, columns element-major (lines
    // interleaved), with one padding element after every 16: the first
    // radix-16 stage writes at a stride of 16 elements (128 bytes), which
    // without the padding puts a warp's stores on one bank pair
    __device__ __forceinline__ int sidx(int l, int i, int N) const
    {
        const int k = ROWS ? l * N + i : i * L + l;
        return k + (k >> 4);
    }
};

template <bool ROWS>
__device__ __forceinline__ float2 load_elem(const void *__restrict__ in, const Lines<ROWS> &ln, int l, int i, int LOAD)
{
    const int r = ln.row(l, i), c = ln.col(l, i);
    const size_t gi = (size_t)r * ln.G + c;
    if (LOAD == LOAD_REAL_CHECKER) return make_float2(__ldg(static_cast<const float *>(in) + gi) * checker(r, c), 0.f);
    float2 v = __ldg(static_cast<const float2 *>(in) + gi);
    if (LOAD == LOAD_CHECKER) {
        const float a = checker(r, c);
        v.x *= a;
        v.y *= a;
    }
    return v;
}

template <bool ROWS>
__device__ __forceinline__ void store_elem(void *__restrict__ out, const Lines<ROWS> &ln, int l, int i, float2 v,
                                           const float *__restrict__ prolate, int STORE)
{
    const int r = ln.row(l, i), c = ln.col(l, i);
    const size_t gi = (size_t)r * ln.G + c;
    if (STORE == STORE_REAL_CHECKER_TAPER) {
        const float x = v.x * checker(r, c);
        const int half = ln.G / 2;
        const int dc = abs(c - half), dr = abs(r - half);
        float taper = __fmul_rn(prolate[dc], prolate[dr]);
        if (dc == 1229 || dr == 1229) taper = 0.f;
        static_cast<float *>(out)[gi] = ((double)fabsf(taper) > 1E-10) ? __fdiv_rn(x, taper) : 0.f;
    } else {
        if (STORE == STORE_CHECKER) {
            const float a = checker(r, c);
            v.x *= a;
            v.y *= a;
        }
        static_cast<float2 *>(out)[gi] = v;
    }
}

constexpr int kElemsPerThread = 32;  // complex values a thread holds per stage

struct FftArgs {
    int L;                  // lines per CTA
    const void *in;
    void *out;
    const float2 *tw;       // exp(-2 pi i k / N), k < N
    const float *prolate;   // taper table (STORE_REAL_CHECKER_TAPER)
    float sg;               // 1 forward, -1 inverse
    int load_op, store_op;
};

// One Stockham stage of radix R over all L lines of the CTA.  Every thread
// first reads all of its butterflies (32 values) into registers; a barrier
// separates those reads from the writes, so one shared buffer serves in
// place.  FIRST: inputs from global memory; LAST: outputs to global memory.
template <int R, int N, bool ROWS, bool FIRST, bool LAST>
__device__ __forceinline__ void stage(float2 *__restrict__ s, const Lines<ROWS> &ln, int Ns, const FftArgs &A)
{
    constexpr int NB = kElemsPerThread / R;
    constexpr int per_line = N / R;
    const int total = ln.L * per_line;
    const int tw_step = N / (Ns * R);
    float2 a[NB][R];
    int jj[NB], ll[NB];
#pragma unroll
    for (int q = 0; q < NB; ++q) {
        const int b = threadIdx.x + q * blockDim.x;
        int l = 0, j = 0;
        if (b < total) {
            if (ROWS) {
                l = b / per_line;
                j = b - l * per_line;
            } else {
                j = b / ln.L;
                l = b - j * ln.L;
            }
#pragma unroll
            for (int t = 0; t < R; ++t) {
                const int i = j + t * per_line;
                a[q][t] = FIRST ? load_elem<ROWS>(A.in, ln, l, i, A.load_op) : s[ln.sidx(l, i, N)];
            }
        }
        jj[q] = j;
        ll[q] = l;
    }
    if (!FIRST && !LAST) __syncthreads();  // reads of this stage complete before in-place writes
#pragma unroll
    for (int q = 0; q < NB; ++q) {
        const int b = threadIdx.x + q * blockDim.x;
        if (b < total) {
            const int j = jj[q], l = ll[q];
            const int k = j & (Ns - 1);
            if (!FIRST) {
#pragma unroll
                for (int t = 1; t < R; ++t) {
                    float2 w = __ldg(&A.tw[(t * k * tw_step) & (N - 1)]);
                    w.y *= A.sg;
                    a[q][t] = cmulf(a[q][t], w);
                }
            }
            dft_r<R>(a[q], A.sg);
            const int base = (j - k) * R + k;
#pragma unroll
            for (int t = 0; t < R; ++t) {
                const int i = base + t * Ns;
                if (LAST) {
                    store_elem<ROWS>(A.out, ln, l, i, a[q][t], A.prolate, A.store_op);
                } else {
                    s[ln.sidx(l, i, N)] = a[q][t];
                }
            }
        }
    }
    if (!LAST) __syncthreads();  // writes visible to the next stage
}

// Radix-16 stages, then one radix-2^(log2 N mod 4) stage, unrolled at
// compile time.
template <int LOG2N, int ST, bool ROWS>
__device__ __forceinline__ void run_stages(float2 *s, const Lines<ROWS> &ln, int Ns, const FftArgs &A)
{
    constexpr int NS16 = LOG2N / 4, REM = LOG2N % 4;
    constexpr int NST = NS16 + (REM ? 1 : 0);
    if constexpr (ST < NST) {
        constexpr int R = (ST < NS16) ? 16 : (1 << REM);
        stage<R, (1 << LOG2N), ROWS, ST == 0, ST == NST - 1>(s, ln, Ns, A);
        run_stages<LOG2N, ST + 1, ROWS>(s, ln, Ns * R, A);
    }
}

// One pass over all lines of a G x G array (ROWS: lines are rows).
template <bool ROWS, int LOG2N>
__global__ void __launch_bounds__(512) k_fft_pass(FftArgs A)
{
    extern __shared__ float2 s[];
    Lines<ROWS> ln{1 << LOG2N, (int)blockIdx.x * A.L, A.L};
    run_stages<LOG2N, 0, ROWS>(s, ln, 1, A);
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

// Twiddle table exp(-2 pi i k / N), k < N, for size N on the current device
// (allocated on first use, kept).
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
    SDP_CUDA_TRY(cudaMalloc(&p, sizeof(float2) * (size_t)N));
    k_twiddles<<<std::max(1, std::min(1024, N / 256 + 1)), 256, 0, st>>>(N, p);
    SDP_LAUNCH_CHECK();
    SDP_CUDA_TRY(cudaStreamSynchronize(st));
    g_tw[{dev, N}] = p;
    *out = p;
    return SDP_OK;
}

int check_fft_size(int G)
{
    if (G < 16 || G > 16384 || (G & (G - 1)) != 0)
        return set_error(SDP_ERR_RANGE, "FFT size %d must be a power of two in [16, 16384]", G);
    return SDP_OK;
}

template <bool ROWS, int LOG2N>
static int launch_pass_n(const FftArgs &A, int G, size_t smem, int threads, cudaStream_t st)
{
    auto fn = k_fft_pass<ROWS, LOG2N>;
    if (smem > 48 * 1024) SDP_CUDA_TRY(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    fn<<<G / A.L, threads, smem, st>>>(A);
    SDP_LAUNCH_CHECK();
    return SDP_OK;
}

template <bool ROWS>
static int launch_pass(int G, const void *in, void *out, const float2 *tw, bool inverse, const float *prolate,
                       int load_op, int store_op, cudaStream_t st)
{
    // L lines of G elements per CTA (64 KB of shared memory, 128 KB for G = 16384), 32 elements per thread
    const int elems = std::max(G, kFftSmemElems);
    FftArgs A;
    A.L = std::min(G, elems / G);
    A.in = in;
    A.out = out;
    A.tw = tw;
    A.prolate = prolate;
    A.sg = inverse ? -1.f : 1.f;
    A.load_op = load_op;
    A.store_op = store_op;
    const int threads = std::max(32, (A.L * G) / kElemsPerThread);
    const size_t smem = sizeof(float2) * ((size_t)A.L * G + (size_t)A.L * G / 16);  // + the padding (sidx)
    switch (G) {
    case 16: return launch_pass_n<ROWS, 4>(A, G, smem, threads, st);
    case 32: return launch_pass_n<ROWS, 5>(A, G, smem, threads, st);
    case 64: return launch_pass_n<ROWS, 6>(A, G, smem, threads, st);
    case 128: return launch_pass_n<ROWS, 7>(A, G, smem, threads, st);
    case 256: return launch_pass_n<ROWS, 8>(A, G, smem, threads, st);
    case 512: return launch_pass_n<ROWS, 9>(A, G, smem, threads, st);
    case 1024: return launch_pass_n<ROWS, 10>(A, G, smem, threads, st);
    case 2048: return launch_pass_n<ROWS, 11>(A, G, smem, threads, st);
    case 4096: return launch_pass_n<ROWS, 12>(A, G, smem, threads, st);
    case 8192: return launch_pass_n<ROWS, 13>(A, G, smem, threads, st);
    case 16384: return launch_pass_n<ROWS, 14>(A, G, smem, threads, st);
    default: return set_error(SDP_ERR_RANGE, "FFT size %d unsupported", G);
    }
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
    SDP_TRY(launch_pass<true>(G, in, out, tw, inv, nullptr, LOAD_PLAIN, STORE_PLAIN, st));
    SDP_TRY(launch_pass<false>(G, out, out, tw, inv, nullptr, LOAD_PLAIN, STORE_PLAIN, st));
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
    SDP_TRY(launch_pass<true>(G, grid, work, tw, true, nullptr, LOAD_CHECKER, STORE_PLAIN, st));
    SDP_TRY(launch_pass<false>(G, work, image, tw, true, prolate_ext, LOAD_PLAIN, STORE_REAL_CHECKER_TAPER, st));
    return SDP_OK;
}

SDP_EXPORT int sdp_image_to_grid(int G, const float *image, sdp_float2 *work, sdp_float2 *grid, void *stream)
{
    SDP_TRY(check_fft_size(G));
    SDP_CHECK_ARG(image && work && grid, "NULL argument");
    cudaStream_t st = as_stream(stream);
    const float2 *tw = nullptr;
    SDP_TRY(fft_twiddles(G, st, &tw));
    SDP_TRY(launch_pass<true>(G, image, work, tw, false, nullptr, LOAD_REAL_CHECKER, STORE_PLAIN, st));
    SDP_TRY(launch_pass<false>(G, work, grid, tw, false, nullptr, LOAD_PLAIN, STORE_CHECKER, st));
    return SDP_OK;
}
