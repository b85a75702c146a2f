// 2-D complex FFT on the tensor cores in BF16 with split hi/lo compensated
// products accumulated in FP32 (the precision path of the imaging FFT; the
// FFTW-convention transform of fft_run.c:23-83, unnormalised, sign -1
// forward, +1 inverse).  No counterpart in the reference, which calls FFTW.
//
// A line of N = 256 r points (r = 4, 8 or 16: N = 1024, 2048, 4096) is
// decomposed N = 16 x 16 x r (Cooley-Tukey, decimation in time):
//   A: for each q < 16 r: Y[k1][q] = sum_n1 x[n1 16 r + q] W16^(n1 k1),
//      times the twiddle W_N^(q k1);
//   B: for each (k1, q2 < r): Z[k1][k2][q2] = sum_q1 Y[k1][q1 r + q2] W16^(q1 k2),
//      times W_(16 r)^(q2 k2);
//   C: X[k1 + 16 k2 + 256 k3] = sum_q2 Z[k1][k2][q2] W_r^(q2 k3),
// with W_L = exp(sign 2 pi i / L).  Each stage is a product of the real
// block matrix [[C, -sS], [sS, C]] of the L-point DFT (L = 16, or r padded
// to 16) with the stage's inputs, 8 columns per mma.sync m16n8k16.  Both
// operands are split into BF16 hi + lo (hi = bf16(v), lo = bf16(v - hi))
// and the product is A_hi B_hi + A_hi B_lo + A_lo B_hi in FP32, so the
// representation error per stage is ~2^-17 and the omitted A_lo B_lo term
// ~2^-18 of the operands; twiddles are FP32 (from the FP64-built table).
//
// The 2-D transform is a row pass that writes its output transposed, twice:
// pass 1 transforms the rows of `in` into the columns of `work`, pass 2 the
// rows of `work` (the original columns) back into `out` in the original
// orientation.  A CTA holds 4 lines (2 at N = 4096) in shared memory,
// every stage in place (index padding p + p / 64 against bank conflicts);
// its 8 warps, 2 (4) per line, split each stage's 8-column groups.
#include <cuda_bf16.h>

#include "common.cuh"

namespace sdp {
int fft_twiddles(int N, cudaStream_t st, const float2 **out);

namespace {

constexpr int kTcThreads = 256;
// lines per CTA: 4 (N <= 2048) or 2 (N = 4096), one padded buffer each
// (the transposed store writes 32 / 16-byte pieces)
__host__ __device__ constexpr int tc_lines(int r) { return r == 16 ? 2 : 4; }

__device__ __forceinline__ int pad(int p) { return p + (p >> 6); }

__device__ __forceinline__ void mma_bf16(float (&d)[4], const uint32_t (&a)[4], uint32_t b0, uint32_t b1)
{
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
        "{%0,%1,%2,%3};\n"
        : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

__device__ __forceinline__ uint32_t pack2(__nv_bfloat16 lo_col, __nv_bfloat16 hi_col)
{
    __nv_bfloat162 v;
    v.x = lo_col;
    v.y = hi_col;
    return *reinterpret_cast<uint32_t *>(&v);
}

// hi / lo BF16 pair of two floats (column order kept)
__device__ __forceinline__ void split2(float a, float b, uint32_t &hi, uint32_t &lo)
{
    const __nv_bfloat16 ah = __float2bfloat16_rn(a), bh = __float2bfloat16_rn(b);
    hi = pack2(ah, bh);
    lo = pack2(__float2bfloat16_rn(a - __bfloat162float(ah)), __float2bfloat16_rn(b - __bfloat162float(bh)));
}

// Element of the real block matrix of the L-point DFT, output (k, re/im),
// input (n, re/im); FP32 (about 1e-7, far below the BF16 hi + lo split).
__device__ float dft_block(int L, int sign, int k, int kim, int n, int nim)
{
    float sn, c;
    sincospif(2.0f * (float)((k * n) % L) / (float)L, &sn, &c);
    if (kim == nim) return c;
    return kim ? sign * sn : -sign * sn;
}

// A fragments (hi, lo) of a 16 x 16 block of the real DFT matrix.  big: the
// 32 x 32 matrix of the 16-point DFT (rows/cols 0-15 real, 16-31 imaginary;
// m-tile mt, k-tile kt); else the r-point matrix padded to 16 x 16 (rows /
// cols 0..r-1 real, 8..8+r-1 imaginary).
__device__ void a_frag(int L, int sign, bool big, int mt, int kt, uint32_t (&hi)[4], uint32_t (&lo)[4])
{
    const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
    for (int reg = 0; reg < 4; ++reg) {
        const int row = g + 8 * (reg & 1), col = 2 * t + 8 * (reg >> 1);
        __nv_bfloat16 h[2], l[2];
        for (int e = 0; e < 2; ++e) {
            const int rr = 16 * mt + row, cc = 16 * kt + col + e;
            float v = 0.f;
            if (big) {
                v = dft_block(L, sign, rr & 15, rr >> 4, cc & 15, cc >> 4);
            } else {
                const int k = rr & 7, n = cc & 7;
                if (k < L && n < L) v = dft_block(L, sign, k, rr >> 3, n, cc >> 3);
            }
            h[e] = __float2bfloat16_rn(v);
            l[e] = __float2bfloat16_rn(v - __bfloat162float(h[e]));
        }
        hi[reg] = pack2(h[0], h[1]);
        lo[reg] = pack2(l[0], l[1]);
    }
}

struct Frag16 {
    uint32_t hi[2][2][4], lo[2][2][4];
};

// One 8-column group of a 16-point stage on a line: column c of the group
// reads its inputs x[pin(c, n)], n < 16, and writes output k (< 16) times
// the twiddle tw(c, k) to y[pout(c, k)].
template <class PIn, class POut, class Tw>
__device__ __forceinline__ void stage16(const Frag16 &F, float2 *x, float2 *y, int c0, PIn pin, POut pout, Tw tw)
{
    const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
    const int c = c0 + g;
    const float2 v0 = x[pad(pin(c, 2 * t))], v1 = x[pad(pin(c, 2 * t + 1))];
    const float2 v2 = x[pad(pin(c, 2 * t + 8))], v3 = x[pad(pin(c, 2 * t + 9))];
    uint32_t reh[2], rel[2], imh[2], iml[2];
    split2(v0.x, v1.x, reh[0], rel[0]);
    split2(v2.x, v3.x, reh[1], rel[1]);
    split2(v0.y, v1.y, imh[0], iml[0]);
    split2(v2.y, v3.y, imh[1], iml[1]);
    float d[2][4];
#pragma unroll
    for (int mt = 0; mt < 2; ++mt) {
#pragma unroll
        for (int e = 0; e < 4; ++e) d[mt][e] = 0.f;
        // k-tile 0: real parts of the inputs, k-tile 1: imaginary parts
        mma_bf16(d[mt], F.hi[mt][0], reh[0], reh[1]);
        mma_bf16(d[mt], F.hi[mt][0], rel[0], rel[1]);
        mma_bf16(d[mt], F.lo[mt][0], reh[0], reh[1]);
        mma_bf16(d[mt], F.hi[mt][1], imh[0], imh[1]);
        mma_bf16(d[mt], F.hi[mt][1], iml[0], iml[1]);
        mma_bf16(d[mt], F.lo[mt][1], imh[0], imh[1]);
    }
    __syncwarp();  // every lane has read the group before any writes it
#pragma unroll
    for (int e = 0; e < 4; ++e) {
        const int k = g + 8 * (e >> 1), cc = c0 + 2 * t + (e & 1);
        const float2 w = tw(cc, k);
        const float re = d[0][e], im = d[1][e];
        y[pad(pout(cc, k))] = make_float2(fmaf(re, w.x, -im * w.y), fmaf(re, w.y, im * w.x));
    }
}

// One 8-column group of an r-point stage (r = 4 or 8, padded to 16 x 16;
// input n at rows n (real) and 8 + n (imaginary)), no twiddle.
template <int R, class PIn, class POut>
__device__ __forceinline__ void stage_small(const uint32_t (&ahi)[4], const uint32_t (&alo)[4], const float2 *x,
                                            float2 *y, int c0, PIn pin, POut pout)  // y may alias x
{
    const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
    const int c = c0 + g;
    float2 v0 = make_float2(0.f, 0.f), v1 = v0;
    if (2 * t < R) {
        v0 = x[pad(pin(c, 2 * t))];
        v1 = x[pad(pin(c, 2 * t + 1))];
    }
    uint32_t bh0, bl0, bh1, bl1;
    split2(v0.x, v1.x, bh0, bl0);  // rows 2t, 2t + 1: real parts
    split2(v0.y, v1.y, bh1, bl1);  // rows 8 + 2t, 9 + 2t: imaginary parts
    float d[4] = {0.f, 0.f, 0.f, 0.f};
    mma_bf16(d, ahi, bh0, bh1);
    mma_bf16(d, ahi, bl0, bl1);
    mma_bf16(d, alo, bh0, bh1);
    __syncwarp();  // every lane has read the group before any writes it
    // rows g (< R): real part of output g; rows 8 + g: imaginary part
    if (g < R) {
        y[pad(pout(c0 + 2 * t, g))] = make_float2(d[0], d[2]);
        y[pad(pout(c0 + 2 * t + 1, g))] = make_float2(d[1], d[3]);
    }
}

template <int R>
__global__ void __launch_bounds__(kTcThreads) k_fft_tc_pass(int G, const float2 *__restrict__ in,
                                                           float2 *__restrict__ out, const float2 *__restrict__ twt,
                                                           int sign)
{
    constexpr int N = 256 * R, M1 = 16 * R;
    constexpr int P = N + N / 64;  // padded line
    constexpr int LINES = tc_lines(R), WPL = (kTcThreads / 32) / LINES;  // warps per line
    extern __shared__ __align__(16) float2 sm[];
    float2 *xs = sm;                      // LINES padded lines, every stage in place
    const int warp = threadIdx.x >> 5;
    const int line = warp / WPL, half = warp % WPL;
    const int row0 = blockIdx.x * LINES;

    Frag16 F;
#pragma unroll
    for (int mt = 0; mt < 2; ++mt)
#pragma unroll
        for (int kt = 0; kt < 2; ++kt) a_frag(16, sign, true, mt, kt, F.hi[mt][kt], F.lo[mt][kt]);
    uint32_t rhi[4], rlo[4];
    if (R < 16) a_frag(R, sign, false, 0, 0, rhi, rlo);

    // load LINES lines
    for (int i = threadIdx.x; i < LINES * N / 2; i += kTcThreads) {
        const int l = i / (N / 2), n = 2 * (i - l * (N / 2));
        const float4 v = __ldg(reinterpret_cast<const float4 *>(in + (size_t)(row0 + l) * G + n));
        xs[l * P + pad(n)] = make_float2(v.x, v.y);
        xs[l * P + pad(n + 1)] = make_float2(v.z, v.w);
    }
    __syncthreads();
    float2 *x = xs + line * P;
    // twiddle W_N^j (table exp(-2 pi i j / N); conjugate for the inverse)
    auto twN = [&](int j) {
        const float2 w = __ldg(twt + j);
        return make_float2(w.x, sign < 0 ? w.y : -w.y);
    };
    // stage A: columns q < M1, input n1 at n1 M1 + q, output k1 at k1 M1 + q, twiddle W_N^(q k1)
    for (int grp = half; grp < M1 / 8; grp += WPL)
        stage16(F, x, x, grp * 8, [](int q, int n) { return n * M1 + q; }, [](int q, int k) { return k * M1 + q; },
                [&](int q, int k) { return twN(q * k); });
    __syncthreads();
    // stage B: columns j = k1 r + q2 (16 r of them), input q1 at k1 M1 + q1 r + q2,
    // output k2 at k1 M1 + k2 r + q2, twiddle W_M1^(q2 k2) = W_N^(16 q2 k2)
    for (int grp = half; grp < (16 * R) / 8; grp += WPL)
        stage16(F, x, x, grp * 8, [](int j, int n) { return (j / R) * M1 + n * R + (j % R); },
                [](int j, int k) { return (j / R) * M1 + k * R + (j % R); },
                [&](int j, int k) { return twN(16 * (j % R) * k); });
    __syncthreads();
    // stage C: columns (k1, k2) = j, j = 16 k1 + k2, input q2 at k1 M1 + k2 r + q2,
    // output k3 in place at k1 M1 + k2 r + k3 (natural index k1 + 16 k2 + 256 k3)
    for (int grp = half; grp < 256 / 8; grp += WPL) {
        auto pin = [](int j, int n) { return (j >> 4) * M1 + (j & 15) * R + n; };
        if constexpr (R == 16) {
            stage16(F, x, x, grp * 8, pin, pin, [](int, int) { return make_float2(1.f, 0.f); });
        } else {
            stage_small<R>(rhi, rlo, x, x, grp * 8, pin, pin);
        }
    }
    __syncthreads();
    // transposed store: out[k][row0 + l], k = k1 + 16 k2 + 256 k3 at k1 M1 + k2 r + k3
    for (int i = threadIdx.x; i < LINES * N; i += kTcThreads) {
        const int k = i / LINES, l = i - k * LINES;
        const int pos = (k & 15) * M1 + ((k >> 4) & 15) * R + (k >> 8);
        out[(size_t)k * G + row0 + l] = xs[l * P + pad(pos)];
    }
}

template <int R>
int launch_tc_pass(int G, const float2 *in, float2 *out, const float2 *tw, int sign, cudaStream_t st)
{
    constexpr int N = 256 * R;
    const size_t smem = sizeof(float2) * tc_lines(R) * (N + N / 64);
    auto fn = k_fft_tc_pass<R>;
    SDP_CUDA_TRY(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    fn<<<G / tc_lines(R), kTcThreads, smem, st>>>(G, in, out, tw, sign);
    SDP_LAUNCH_CHECK();
    return SDP_OK;
}

}  // namespace
}  // namespace sdp

using namespace sdp;

SDP_EXPORT int sdp_fft2d_tc(int G, const sdp_float2 *in, sdp_float2 *out, int sign, sdp_float2 *work, void *stream)
{
    SDP_CHECK_ARG(G == 1024 || G == 2048 || G == 4096, "tensor-core FFT size %d: 1024, 2048 or 4096", G);
    SDP_CHECK_ARG(sign == -1 || sign == 1, "sign must be -1 or +1");
    SDP_CHECK_ARG(in && out && work, "NULL argument");
    SDP_CHECK_ARG(work != in && work != out, "work must not alias in or out");
    cudaStream_t st = as_stream(stream);
    const float2 *tw = nullptr;
    SDP_TRY(fft_twiddles(G, st, &tw));
    const float2 *src = reinterpret_cast<const float2 *>(in);
    float2 *w = reinterpret_cast<float2 *>(work), *dst = reinterpret_cast<float2 *>(out);
    switch (G) {
    case 1024:
        SDP_TRY(launch_tc_pass<4>(G, src, w, tw, sign, st));
        SDP_TRY(launch_tc_pass<4>(G, w, dst, tw, sign, st));
        break;
    case 2048:
        SDP_TRY(launch_tc_pass<8>(G, src, w, tw, sign, st));
        SDP_TRY(launch_tc_pass<8>(G, w, dst, tw, sign, st));
        break;
    default:
        SDP_TRY(launch_tc_pass<16>(G, src, w, tw, sign, st));
        SDP_TRY(launch_tc_pass<16>(G, w, dst, tw, sign, st));
        break;
    }
    return SDP_OK;
}
