// U-Net that proposes CLEAN components from a residual image: BF16
// tensor-core convolutions with FP32 accumulation (forward, data gradient,
// weight gradient), the pooling / upsampling / output-head kernels around
// them, the blurred squared-error loss and the Adam optimiser.
//
// No counterpart in the reference (its deconvolution is Hogbom only,
// deconvolution_run.c:197-311); the network proposes components that the
// major cycle verifies, with Hogbom as the fallback.
//
// Network (levels 0..3, c_l = base * 2^l channels, level l at H/2^l x W/2^l):
//   e0a = relu(conv(x)),            e0 = relu(conv(e0a))
//   e1a = relu(conv(pool(e0))),     e1 = relu(conv(e1a))
//   e2a = relu(conv(pool(e1))),     e2 = relu(conv(e2a))
//   e3a = relu(conv(pool(e2))),     e3 = relu(conv(e3a))
//   d2a = relu(conv([e2, up(e3)])), d2 = relu(conv(d2a))
//   d1a = relu(conv([e1, up(d2)])), d1 = relu(conv(d1a))
//   d0a = relu(conv([e0, up(d1)])), d0 = relu(conv(d0a))
//   out = head(d0)   (1x1 convolution to one channel, FP32 output)
// conv = 3x3, zero padding; pool = 2x2 mean; up = nearest (2x2 repeat);
// [a, b] = channel concatenation.  The concatenation and the upsampling are
// never materialised: the convolution's loader reads channels below c_a
// from a and the rest from b at (y/2, x/2).
//
// Layouts: activations and their gradients are BF16, NHWC (channels
// innermost; every channel count is a multiple of 32, the network input is
// padded to 32 channels).  Weights: FP32 master copy [tap][cout][cin]
// (tap = 3 * (dy + 1) + (dx + 1)) followed by the FP32 bias; the BF16 copy
// in the same order feeds the forward pass and a transposed, tap-flipped
// copy [8 - tap][cin][cout] the data gradient.
//
// Tensor-core path: mma.sync m16n8k16 BF16 -> FP32, operands loaded from
// shared memory with ldmatrix (conflict-free: every 8-channel group is a
// 16-byte row of its own plane), tiles staged by cp.async with zero fill
// outside the image, double buffered.
#include <cuda.h>
#include <cuda_bf16.h>
#include <cudaTypedefs.h>

#include <cmath>
#include <cstring>

#include "common.cuh"

namespace sdp {
namespace unet {

typedef __nv_bfloat16 bf16;

constexpr int kTH = 8, kTW = 16;              // output tile: 8 rows x 16 columns
constexpr int kHH = kTH + 2, kHW = kTW + 2;   // input halo of the tile
constexpr int kHalo = kHH * kHW;              // 180 pixels
constexpr int kInPad = 32;                    // network input channels padded to 32
constexpr int kLayers = 14;                   // 3x3 convolutions
constexpr int kLevels = 4;

__device__ __forceinline__ uint32_t smem_u32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void cp_async16(uint32_t dst, const void *src, int bytes)
{
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(dst), "l"(src), "r"(bytes));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N>
__device__ __forceinline__ void cp_async_wait()
{
    asm volatile("cp.async.wait_group %0;\n" ::"n"(N));
}

__device__ __forceinline__ void ldsm4(uint32_t (&r)[4], uint32_t addr)
{
    asm volatile("ldmatrix.sync.aligned.m8n8.x4.shared.b16 {%0,%1,%2,%3}, [%4];\n"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3])
                 : "r"(addr));
}
__device__ __forceinline__ void ldsm4t(uint32_t (&r)[4], uint32_t addr)
{
    asm volatile("ldmatrix.sync.aligned.m8n8.x4.trans.shared.b16 {%0,%1,%2,%3}, [%4];\n"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3])
                 : "r"(addr));
}
// D += A (16x16, row) * B (16x8, col), BF16 inputs, FP32 accumulators
__device__ __forceinline__ void mma16816(float (&d)[4], const uint32_t (&a)[4], uint32_t b0, uint32_t b1)
{
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
        "{%0,%1,%2,%3};\n"
        : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

// 8 BF16 channels = one 16-byte vector
union V8 {
    uint4 u;
    __nv_bfloat162 h[4];
};

__device__ __forceinline__ void unpack8(const uint4 &u, float (&f)[8])
{
    V8 v;
    v.u = u;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        f[2 * k] = __low2float(v.h[k]);
        f[2 * k + 1] = __high2float(v.h[k]);
    }
}
__device__ __forceinline__ uint4 pack8(const float (&f)[8])
{
    V8 v;
#pragma unroll
    for (int k = 0; k < 4; ++k) v.h[k] = __floats2bfloat162_rn(f[2 * k], f[2 * k + 1]);
    return v.u;
}

// Source of one 8-channel group of the (virtual) convolution input at image
// pixel (yy, xx) of image img: channels [c, c + 8) of [a, up(b)].
struct VIn {
    const bf16 *a;
    const bf16 *b;
    int ca, cb, h, w;
    __device__ __forceinline__ const bf16 *at(int img, int yy, int xx, int c) const
    {
        if (c < ca) return a + (((size_t)img * h + yy) * w + xx) * ca + c;
        return b + (((size_t)img * (h >> 1) + (yy >> 1)) * (w >> 1) + (xx >> 1)) * cb + (c - ca);
    }
};

// ----------------------------------------------------------------------------
// 3x3 convolution, implicit GEMM: out[p][o] = sum_tap sum_i in[p + off(tap)][i]
// * wk[tap][o][i] (+ bias, relu, mask).  One CTA: an 8 x 16 pixel tile and
// BN output channels; warp w owns tile rows 2w, 2w + 1 (two m16 tiles) and
// all BN channels.  K runs over 16-channel chunks, each chunk over 9 taps.
// Used for the forward pass (wk = W) and the data gradient (wk = flipped
// transpose, no bias; mask = the forward activation whose relu gates it).
// ----------------------------------------------------------------------------
struct ConvArgs {
    VIn in;
    const bf16 *wk;      // [9][cout][cin]
    const float *bias;   // [cout] or null
    const bf16 *mask;    // [n][h][w][cout] or null: out = 0 where mask <= 0
    bf16 *out;           // [n][h][w][cout]
    int cout, relu;
    int tiles_x, tiles_y;
};

template <int BN>
struct ConvSmem {
    static constexpr int kHaloBytes = 2 * kHalo * 16;
    static constexpr int kWBytes = 9 * 2 * BN * 16;
    static constexpr int kStage = kHaloBytes + kWBytes;
    static constexpr int kBytes = 2 * kStage;
};

template <int BN>
__global__ void __launch_bounds__(128) k_conv3x3(ConvArgs p)
{
    extern __shared__ __align__(128) unsigned char smem[];
    using SM = ConvSmem<BN>;
    const int cin = p.in.ca + p.in.cb;
    const int nchunks = cin >> 4;
    int t = blockIdx.x;
    const int tx = t % p.tiles_x;
    t /= p.tiles_x;
    const int ty = t % p.tiles_y;
    const int img = t / p.tiles_y;
    const int y0 = ty * kTH, x0 = tx * kTW;
    const int co0 = blockIdx.y * BN;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int H = p.in.h, W = p.in.w;

    auto load_chunk = [&](int k, int s) {
        unsigned char *base = smem + s * SM::kStage;
        const uint32_t hs = smem_u32(base), ws = smem_u32(base + SM::kHaloBytes);
        const int c0 = k << 4;
        for (int i = tid; i < 2 * kHalo; i += 128) {
            const int half = i >= kHalo;
            const int hidx = i - half * kHalo;
            const int yy = y0 - 1 + hidx / kHW, xx = x0 - 1 + hidx % kHW;
            const bool inside = yy >= 0 && yy < H && xx >= 0 && xx < W;
            const bf16 *src = inside ? p.in.at(img, yy, xx, c0 + 8 * half) : p.in.a;
            cp_async16(hs + i * 16, src, inside ? 16 : 0);
        }
        for (int i = tid; i < 9 * 2 * BN; i += 128) {
            const int co = i % BN, th = i / BN;  // th = 2 * tap + half
            const bf16 *src = p.wk + ((size_t)(th >> 1) * p.cout + co0 + co) * cin + c0 + 8 * (th & 1);
            cp_async16(ws + i * 16, src, 16);
        }
    };

    float acc[2][BN / 8][4];
#pragma unroll
    for (int a = 0; a < 2; ++a)
#pragma unroll
        for (int b = 0; b < BN / 8; ++b)
#pragma unroll
            for (int c = 0; c < 4; ++c) acc[a][b][c] = 0.f;

    load_chunk(0, 0);
    cp_async_commit();
    const int q = lane >> 3, i8 = lane & 7;
    for (int k = 0; k < nchunks; ++k) {
        if (k + 1 < nchunks) load_chunk(k + 1, (k + 1) & 1);
        cp_async_commit();
        cp_async_wait<1>();
        __syncthreads();
        const unsigned char *base = smem + (k & 1) * SM::kStage;
        const uint32_t hs = smem_u32(base), ws = smem_u32(base + SM::kHaloBytes);
#pragma unroll 1
        for (int tap = 0; tap < 9; ++tap) {
            const int dy = tap / 3, dx = tap - 3 * (tap / 3);
            uint32_t af[2][4];
#pragma unroll
            for (int mt = 0; mt < 2; ++mt) {
                // matrix q: pixels (q & 1) * 8 + 0..7 of tile row r, channel half q >> 1
                const int r = warp * 2 + mt;
                const int hidx = (r + dy) * kHW + (q & 1) * 8 + i8 + dx;
                ldsm4(af[mt], hs + ((q >> 1) * kHalo + hidx) * 16);
            }
#pragma unroll
            for (int j = 0; j < BN / 8; j += 2) {
                // matrix q: output channels of n-tile j + (q >> 1), channel half q & 1
                uint32_t bfr[4];
                const int co = (j + (q >> 1)) * 8 + i8;
                ldsm4(bfr, ws + ((tap * 2 + (q & 1)) * BN + co) * 16);
#pragma unroll
                for (int mt = 0; mt < 2; ++mt) {
                    mma16816(acc[mt][j], af[mt], bfr[0], bfr[1]);
                    mma16816(acc[mt][j + 1], af[mt], bfr[2], bfr[3]);
                }
            }
        }
        __syncthreads();
    }

    const int g = lane >> 2, tq = lane & 3;
#pragma unroll
    for (int mt = 0; mt < 2; ++mt) {
        const int y = y0 + warp * 2 + mt;
#pragma unroll
        for (int hr = 0; hr < 2; ++hr) {
            const int x = x0 + g + hr * 8;
            if (y >= H || x >= W) continue;
            const size_t pix = ((size_t)img * H + y) * W + x;
#pragma unroll
            for (int j = 0; j < BN / 8; ++j) {
                const int co = co0 + j * 8 + tq * 2;
                float v0 = acc[mt][j][hr * 2], v1 = acc[mt][j][hr * 2 + 1];
                if (p.bias) {
                    v0 += p.bias[co];
                    v1 += p.bias[co + 1];
                }
                if (p.relu) {
                    v0 = v0 > 0.f ? v0 : 0.f;
                    v1 = v1 > 0.f ? v1 : 0.f;
                }
                if (p.mask) {
                    const __nv_bfloat162 m = *reinterpret_cast<const __nv_bfloat162 *>(p.mask + pix * p.cout + co);
                    if (!(__low2float(m) > 0.f)) v0 = 0.f;
                    if (!(__high2float(m) > 0.f)) v1 = 0.f;
                }
                *reinterpret_cast<__nv_bfloat162 *>(p.out + pix * p.cout + co) = __floats2bfloat162_rn(v0, v1);
            }
        }
    }
}

// ----------------------------------------------------------------------------
// The same convolution on the 5th-generation tensor cores (tcgen05), as a
// persistent warp-specialised kernel.  Tile = R consecutive image rows
// (R = 1, 2, 4 or 8; each a 128-pixel segment, M = 128 per row) x nt output
// channels (nt <= 256, a multiple of 32), R accumulators in tensor memory.
// K = 9 taps x Cin, walked as (chunk of KC = 32 channels, column tap dx)
// pairs; one pair = one pipeline stage:
//   A: the (R + 2) x 128 input pixels the three row taps of dx read (rows
//      y0 - 1 .. y0 + R, columns x0 + dx - 1 ..), KC channels each, by one
//      4-D TMA box {KC, 128, R + 2, 1} (reads outside the image return zero);
//      row tap dy of output row r is box row r + dy;
//   B: the pair's 3 x nt x KC weights (dy = 0, 1, 2), pre-arranged in global
//      memory as the shared-memory image, by one bulk copy;
// both in the K-major canonical layout with the 64-byte swizzle, which the
// TMA writes and the MMA reads (rows of 32 channels; 8-row atoms of 512
// bytes; K advanced 16 channels = 32 bytes inside the row; the descriptor
// helper also knows the 128-byte form for 64-channel rows).  A stage is
// 3 x R x KC / 16 tcgen05.mma (M128 x nt
// x K16, BF16 -> FP32 in tensor memory); each row's A starts on an atom.
// Packed row taps (nt = 32, where an N = 32 MMA would leave most of the
// tensor core idle: any N <= 128 costs about the same time per K16 step):
// one MMA per box row i and K16 step takes the three dy weight blocks as one
// N = 96 operand (they are contiguous in the staged B), and writes them to
// three consecutive 32-column accumulator blocks.  Output row r lives at
// columns 32 (R + 1 - r), so block dy of box row i (output row i - dy) is at
// 32 (R + 1 - i) + 32 dy for every dy: the MMAs of rows i and i + 1 overlap
// by two blocks and accumulate into the same rows.  One set is 32 (R + 4)
// columns (two blocks above and below the R real rows take contributions
// that belong to neighbouring tiles and are discarded); every MMA
// accumulates, so the epilogue stores zeros to the set after reading it.
// (R + 2) x KC / 16 MMAs per stage instead of 3 R KC / 16.
//   warp 0 (one thread): loads, through an S-stage ring (full/empty
//     mbarriers, transaction counts);
//   warp 1: MMAs, issued by lane 0 while the whole warp walks the loop (the
//     descriptors stay warp-uniform); commits free a stage (empty) and, after
//     a tile's last stage, hand its accumulator to the epilogue;
//   warps 2-9: epilogue, tcgen05.ld of the accumulator (warp w reads lanes
//     32 (w % 4) .., the two warps of a quarter alternate over the 32-column
//     slices), bias, relu or the gradient mask, BF16 stores; then free the
//     accumulator.  Two accumulators in tensor memory let the
//     epilogue of one tile overlap the MMAs of the next.
// Every wait is bounded: on timeout the CTA records the error and each role
// leaves its loop (its later waits are bounded too); before the tensor memory
// is released the CTA waits, again bounded, for the copies and MMAs it had
// already issued (the drain at the end of the kernel).
// ----------------------------------------------------------------------------
constexpr int kTcM = 128;                       // pixels per tile
constexpr int kTcMaxStages = 16;
constexpr int kTcSmemBudget = 200 * 1024;       // stages; +1 KB for the 1024-byte alignment
constexpr long long kTcSpins = 1LL << 20;       // bounded mbarrier polls
constexpr int kTcEpiWarps = 8;                  // two epilogue warps per tensor-memory lane quarter
constexpr int kTcThreads = 32 * (2 + kTcEpiWarps);

inline int tc_kc(int) { return 32; }  // 32-channel chunks (64-byte swizzle) for every layer
__host__ __device__ constexpr int tc_row_bytes(int kc) { return kTcM * kc * 2; }
// sa: shared A (the column taps read one buffer of 18 slabs; see below)
__host__ __device__ constexpr int tc_slab_bytes(int kc, int rows) { return (rows + 2) * 8 * kc * 2; }
__host__ __device__ constexpr int tc_a_bytes(int kc, int rows, int sa = 0)
{
    return sa ? 18 * tc_slab_bytes(kc, rows) : (rows + 2) * tc_row_bytes(kc);
}
__host__ __device__ constexpr int tc_b_bytes(int nt, int kc, int sa = 0) { return (sa ? 9 : 3) * nt * kc * 2; }
__host__ __device__ constexpr int tc_stage_bytes(int nt, int kc, int rows, int sa = 0)
{
    return (tc_a_bytes(kc, rows, sa) + tc_b_bytes(nt, kc, sa) + 1023) & ~1023;
}
inline int tc_stages(int nt, int kc, int rows, int sa = 0)
{
    int s = kTcSmemBudget / tc_stage_bytes(nt, kc, rows, sa);
    return s > kTcMaxStages ? kTcMaxStages : s;
}
__host__ __device__ constexpr uint32_t tc_ncols(int nt) { return nt <= 32 ? 32u : (nt <= 64 ? 64u : (nt <= 128 ? 128u : 256u)); }

struct TcArgs {
    int n, h, w;         // image batch and size (input = output)
    int cin, cout, nt;   // nt: output channels per slice (blockIdx.y)
    int kc, nchunks;     // channels per chunk (32 or 64), cin / kc
    int rows;            // image rows per tile (R)
    int tiles_x, tiles_y, ntiles; // tiles per slice
    int stages;
    const bf16 *wtc;     // [slice][chunk][tap] blocks of nt x kc, swizzled as in shared memory
    const float *bias;   // [cout] or null
    const bf16 *mask;    // [n][h][w][cout] or null
    bf16 *out;           // [n][h][w][cout]
    int relu;
    int *err;            // set to 1 when a bounded wait gave up
    long long spins;     // polls of a bounded mbarrier wait (loads, MMAs, the drain)
    long long epi_spins; // polls of the epilogue's wait for an accumulator
    int pack;            // packed row taps (nt = 32)
    int sa;              // shared A: one stage per chunk, pixels in slab order
    // 1x1 head fused into the epilogue (nt = cout = 32: a thread holds all of a pixel's channels):
    // head_out[p] = (sum_c bf16(out[p][c]) bf16(head_w[c]) + head_b[0]) * head_scale[image];
    // head_only: the BF16 output itself is not stored
    const float *head_w, *head_b, *head_scale;
    float *head_out;
    int head_only;
};

__host__ __device__ constexpr uint32_t tc_acc_cols(int pack, int rows, int nt)
{
    return pack ? 32u * (uint32_t)(rows + 4) : (uint32_t)rows * tc_ncols(nt);
}
__host__ __device__ constexpr uint32_t tc_tmem_cols(uint32_t need)
{
    return need <= 32u ? 32u : need <= 64u ? 64u : need <= 128u ? 128u : need <= 256u ? 256u : 512u;
}

// K-major operand descriptor with the 64-byte swizzle (layout 4) and a
// given stride between 8-row groups (the shared-A slabs).
__device__ __forceinline__ uint64_t umma_desc_sw64_sbo(uint32_t saddr, uint32_t sbo)
{
    uint64_t d = (uint64_t)((saddr >> 4) & 0x3FFFu);
    d |= (uint64_t)1 << 16;
    d |= (uint64_t)((sbo >> 4) & 0x3FFFu) << 32;
    d |= (uint64_t)1 << 46;
    d |= (uint64_t)4 << 61;
    return d;
}

// K-major operand descriptor with the 128-byte (layout 2) or 64-byte
// (layout 4) swizzle: SBO = one 8-row atom, LBO unused (1).
__device__ __forceinline__ uint64_t umma_desc_sw(uint32_t saddr, int kc)
{
    const uint32_t sbo = (uint32_t)(8 * kc * 2);
    uint64_t d = (uint64_t)((saddr >> 4) & 0x3FFFu);
    d |= (uint64_t)1 << 16;
    d |= (uint64_t)((sbo >> 4) & 0x3FFFu) << 32;
    d |= (uint64_t)1 << 46;  // descriptor version of sm_100
    d |= (uint64_t)(kc == 64 ? 2 : 4) << 61;
    return d;
}

// Zeros 32 consecutive tensor-memory columns of the warp's 32 lanes.
__device__ __forceinline__ void tmem_zero32(uint32_t taddr)
{
    const uint32_t z = 0u;
    asm volatile(
        "tcgen05.st.sync.aligned.32x32b.x32.b32 [%0], {%1,%1,%1,%1,%1,%1,%1,%1,%1,%1,%1,%1,%1,%1,%1,%1,"
        "%1,%1,%1,%1,%1,%1,%1,%1,%1,%1,%1,%1,%1,%1,%1,%1};" ::"r"(taddr),
        "r"(z)
        : "memory");
}

__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity, long long limit = kTcSpins)
{
    for (long long i = 0; i < limit; ++i) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred P1;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2;\n\t"
            "selp.b32 %0, 1, 0, P1;\n\t}"
            : "=r"(done)
            : "r"(bar), "r"(parity)
            : "memory");
        if (done) return true;
    }
    return false;
}

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count));
}

__device__ __forceinline__ void mbar_arrive(uint32_t bar)
{
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}

__global__ void __launch_bounds__(kTcThreads, 1) k_conv3x3_tc(const __grid_constant__ CUtensorMap tin,
                                                           const __grid_constant__ CUtensorMap tslab,
                                                           const __grid_constant__ CUtensorMap thalo, TcArgs p)
{
    extern __shared__ __align__(128) unsigned char smem[];
    __shared__ __align__(8) uint64_t s_full[kTcMaxStages], s_empty[kTcMaxStages], s_tfull[2], s_tempty[2], s_drain;
    __shared__ uint32_t s_tmem;
    __shared__ int s_fail, s_issued, s_consumed;
    __shared__ float s_bias[256];
    __shared__ float s_hw[32];
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int nt = p.nt, S = p.stages, kc = p.kc, R = p.rows;
    for (int i = tid; i < nt; i += blockDim.x) s_bias[i] = p.bias ? p.bias[blockIdx.y * nt + i] : 0.f;
    if (p.head_out)
        for (int i = tid; i < nt; i += blockDim.x) s_hw[i] = __bfloat162float(__float2bfloat16_rn(p.head_w[i]));
    const int slice = blockIdx.y;
    const uint32_t ncols = tc_ncols(nt);
    const int pack = p.pack;
    const uint32_t acc_cols = tc_acc_cols(pack, R, nt);  // one accumulator set
    const uint32_t tmem_cols = tc_tmem_cols(2 * acc_cols);
    const int sa = p.sa;
    const int stage_bytes = tc_stage_bytes(nt, kc, R, sa);
    // stages start on 1024-byte boundaries (the swizzle atoms)
    const uint32_t sbase = (smem_u32(smem) + 1023u) & ~1023u;
    const int per_tile = sa ? p.nchunks : 3 * p.nchunks;

    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&s_tmem)),
                     "r"(tmem_cols));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::);
    }
    if (tid == 32) {
        for (int i = 0; i < S; ++i) {
            mbar_init(smem_u32(&s_full[i]), 1);
            mbar_init(smem_u32(&s_empty[i]), 1);
        }
        for (int i = 0; i < 2; ++i) {
            mbar_init(smem_u32(&s_tfull[i]), 1);
            mbar_init(smem_u32(&s_tempty[i]), kTcEpiWarps);
        }
        mbar_init(smem_u32(&s_drain), 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        s_fail = 0;
        s_issued = 0;
        s_consumed = 0;
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = s_tmem;
    const int first = blockIdx.x, step = gridDim.x;
    volatile int *fail = &s_fail;  // read afresh in every loop condition
    if (pack) {
        // packed row taps: every MMA accumulates, so both sets start at zero
        if (warp >= 2) {
            const uint32_t lanes = (uint32_t)((warp & 3) * 32) << 16;
            for (uint32_t c = 32u * (uint32_t)((warp - 2) >> 2); c < 2 * acc_cols; c += 64u)
                tmem_zero32(tmem + lanes + c);
            asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory");
        }
        asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
        __syncthreads();
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    }

    if (warp == 0) {
        if (lane == 0) {
            // ---------------- loads ----------------
            const uint32_t a_bytes = (uint32_t)tc_a_bytes(kc, R, sa), b_bytes = (uint32_t)tc_b_bytes(nt, kc, sa);
            const uint32_t slab = (uint32_t)tc_slab_bytes(kc, R);
            int s = 0;
            uint32_t phase = 0;
            bool first_lap = true;
            int issued = 0;  // stage loads issued (their sequence numbers are 0 .. issued - 1)
            for (int t = first; t < p.ntiles && !*fail; t += step) {
                const int tx = t % p.tiles_x, trow = t / p.tiles_x;
                const int img = trow / p.tiles_y, y = (trow - img * p.tiles_y) * R;
                for (int k = 0; k < per_tile; ++k) {
                    const int chunk = k / 3, dx = k - 3 * chunk;
                    if (!first_lap && !mbar_wait(smem_u32(&s_empty[s]), phase ^ 1u, p.spins)) {
                        *fail = 1;
                        break;
                    }
                    const uint32_t st = sbase + (uint32_t)(s * stage_bytes);
                    const uint32_t bar = smem_u32(&s_full[s]);
                    mbar_expect_tx(bar, a_bytes + b_bytes);
                    const bf16 *wsrc;
                    if (sa) {
                        // slabs 1..16: pixel groups k = 0..15 (x = x0 + 16 j + k), then
                        // slab 0 (k = -1: the left neighbours) and slab 17 (k = 16)
                        const int c0 = kc * k, j0 = tx * (kTcM / 16);
                        asm volatile(
                            "cp.async.bulk.tensor.5d.shared::cluster.global.tile.mbarrier::complete_tx::bytes "
                            "[%0], [%1, {%2, %3, %4, %5, %6}], [%7];" ::"r"(st + slab),
                            "l"(reinterpret_cast<uint64_t>(&tslab)), "r"(c0), "r"(j0), "r"(y - 1), "r"(0), "r"(img),
                            "r"(bar)
                            : "memory");
                        asm volatile(
                            "cp.async.bulk.tensor.5d.shared::cluster.global.tile.mbarrier::complete_tx::bytes "
                            "[%0], [%1, {%2, %3, %4, %5, %6}], [%7];" ::"r"(st),
                            "l"(reinterpret_cast<uint64_t>(&thalo)), "r"(c0), "r"(j0 - 1), "r"(y - 1), "r"(15),
                            "r"(img), "r"(bar)
                            : "memory");
                        asm volatile(
                            "cp.async.bulk.tensor.5d.shared::cluster.global.tile.mbarrier::complete_tx::bytes "
                            "[%0], [%1, {%2, %3, %4, %5, %6}], [%7];" ::"r"(st + 17u * slab),
                            "l"(reinterpret_cast<uint64_t>(&thalo)), "r"(c0), "r"(j0 + 1), "r"(y - 1), "r"(0),
                            "r"(img), "r"(bar)
                            : "memory");
                        wsrc = p.wtc + ((size_t)slice * p.nchunks + k) * (size_t)(9 * nt * kc);
                    } else {
                        asm volatile(
                            "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes "
                            "[%0], [%1, {%2, %3, %4, %5}], [%6];" ::"r"(st),
                            "l"(reinterpret_cast<uint64_t>(&tin)), "r"(kc * chunk), "r"(tx * kTcM + dx - 1),
                            "r"(y - 1), "r"(img), "r"(bar)
                            : "memory");
                        wsrc = p.wtc + (((size_t)slice * p.nchunks + chunk) * 3 + dx) * (size_t)(3 * nt * kc);
                    }
                    asm volatile(
                        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                            st + a_bytes),
                        "l"(wsrc), "r"(b_bytes), "r"(bar)
                        : "memory");
                    ++issued;
                    if (++s == S) {
                        s = 0;
                        phase ^= 1u;
                        first_lap = false;
                    }
                }
            }
            s_issued = issued;
        }
    } else if (warp == 1) {
        // ---------------- MMAs ----------------
        // The whole warp walks the loop, so the descriptors are warp-uniform
        // values; lane 0 issues.  Descriptors advance by adding (bytes >> 4)
        // to the start-address field (shared addresses stay below 2^18).
        const uint32_t idesc = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(nt >> 3) << 17) |
                               ((uint32_t)(kTcM >> 4) << 24);
        const uint32_t idesc_pack = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(96 >> 3) << 17) |
                                    ((uint32_t)(kTcM >> 4) << 24);
        const uint64_t desc0 = umma_desc_sw(sbase, kc);
        const uint32_t slab = (uint32_t)tc_slab_bytes(kc, R);
        const uint64_t sdesc0 = umma_desc_sw64_sbo(sbase, slab);  // shared A: 8-row groups one slab apart
        const uint32_t slab16 = slab >> 4;
        const uint32_t a16 = (uint32_t)tc_a_bytes(kc, R, sa) >> 4, row16 = (uint32_t)tc_row_bytes(kc) >> 4;
        const uint32_t tap16 = (uint32_t)(nt * kc * 2) >> 4, stage16 = (uint32_t)stage_bytes >> 4;
        const uint32_t leader = lane == 0 ? 1u : 0u;
        int s = 0;
        uint32_t phase = 0;
        int j = 0;
        int consumed = 0;  // stage loads waited for (their MMAs issued and committed)
        for (int t = first; t < p.ntiles && !*fail; t += step, ++j) {
            const int acc = j & 1, use = j >> 1;
            if (use > 0 &&
                !__all_sync(0xffffffffu, mbar_wait(smem_u32(&s_tempty[acc]), (uint32_t)((use - 1) & 1), p.spins))) {
                if (leader) *fail = 1;
                break;
            }
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            const uint32_t d = tmem + (uint32_t)acc * acc_cols;
            bool ok = true;
            for (int k = 0; k < per_tile; ++k) {
                if (!__all_sync(0xffffffffu, mbar_wait(smem_u32(&s_full[s]), phase, p.spins))) {
                    ok = false;
                    break;
                }
                ++consumed;
                asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                const uint64_t ad0 = desc0 + (uint64_t)((uint32_t)s * stage16);
                const uint64_t bd0 = ad0 + a16;
                // shared A: the stage is a whole chunk; column tap dx reads the
                // 16 slabs from slab dx on (one slab = one pixel column shift)
                const int ndx = sa ? 3 : 1;
                const uint32_t arow16 = sa ? (uint32_t)(8 * kc * 2) >> 4 : row16;  // next image row
#pragma unroll 1
                for (int dxi = 0; dxi < ndx; ++dxi) {
                    const uint64_t aB = sa ? sdesc0 + (uint32_t)s * stage16 + (uint32_t)dxi * slab16 : ad0;
                    const uint64_t bB = bd0 + (uint32_t)dxi * 3u * tap16;
                    if (pack) {
                        // box row i, all three row taps: N = 96 at columns 32 (R + 1 - i)
#pragma unroll 1
                        for (int i = 0; i < R + 2; ++i)
#pragma unroll
                            for (int kk = 0; kk < 2; ++kk) {
                                const uint64_t ad = aB + (uint32_t)i * arow16 + (uint32_t)(2 * kk);
                                const uint64_t bd = bB + (uint32_t)(2 * kk);
                                asm volatile(
                                    "{\n\t.reg .pred p, e;\n\t"
                                    "setp.ne.b32 e, %5, 0;\n\t"
                                    "setp.ne.b32 p, %4, 0;\n\t"
                                    "@e tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}"
                                    :
                                    : "r"(d + 32u * (uint32_t)(R + 1 - i)), "l"(ad), "l"(bd), "r"(idesc_pack),
                                      "r"(1u), "r"(leader));
                            }
                    }
#pragma unroll 1
                    for (int dy = 0; dy < 3 && !pack; ++dy)
#pragma unroll
                        for (int kk = 0; kk < 2; ++kk) {  // kc = 32: two K16 steps
                            const uint64_t bd = bB + (uint32_t)dy * tap16 + (uint32_t)(2 * kk);
                            const uint32_t accum = (k > 0 || dxi > 0 || dy > 0 || kk > 0) ? 1u : 0u;
                            for (int r = 0; r < R; ++r) {
                                const uint64_t ad = aB + (uint32_t)(r + dy) * arow16 + (uint32_t)(2 * kk);
                                asm volatile(
                                    "{\n\t.reg .pred p, e;\n\t"
                                    "setp.ne.b32 e, %5, 0;\n\t"
                                    "setp.ne.b32 p, %4, 0;\n\t"
                                    "@e tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}"
                                    :
                                    : "r"(d + (uint32_t)r * ncols), "l"(ad), "l"(bd), "r"(idesc), "r"(accum),
                                      "r"(leader));
                            }
                        }
                }
                if (leader)
                    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                                     smem_u32(&s_empty[s]))
                                 : "memory");
                __syncwarp();
                if (++s == S) {
                    s = 0;
                    phase ^= 1u;
                }
            }
            if (!ok) {
                if (leader) *fail = 1;
                break;
            }
            if (leader)
                asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                                 smem_u32(&s_tfull[acc]))
                             : "memory");
            __syncwarp();
        }
        if (leader) s_consumed = consumed;
    } else {
        // ---------------- epilogue (warps 2..9) ----------------
        const int q = warp & 3;           // tensor-memory lane quarter this warp may read
        const int half = (warp - 2) >> 2; // the two warps of a quarter take alternate slices
        const int per_row = nt / 32, nslices = R * per_row;
        uint32_t ra[32], rb[32];
        auto tld = [&](uint32_t (&r)[32], uint32_t taddr) {
            asm volatile(
                "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
                "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
                : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
                  "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]),
                  "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]),
                  "=r"(r[22]), "=r"(r[23]), "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]),
                  "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
                : "r"(taddr));
        };
        // waits for every outstanding tcgen05.ld; the registers pass through
        // it so no use of them is scheduled before the wait
        auto twait = [&](uint32_t (&r)[32]) {
            asm volatile("tcgen05.wait::ld.sync.aligned;"
                         : "+r"(r[0]), "+r"(r[1]), "+r"(r[2]), "+r"(r[3]), "+r"(r[4]), "+r"(r[5]), "+r"(r[6]),
                           "+r"(r[7]), "+r"(r[8]), "+r"(r[9]), "+r"(r[10]), "+r"(r[11]), "+r"(r[12]), "+r"(r[13]),
                           "+r"(r[14]), "+r"(r[15]), "+r"(r[16]), "+r"(r[17]), "+r"(r[18]), "+r"(r[19]),
                           "+r"(r[20]), "+r"(r[21]), "+r"(r[22]), "+r"(r[23]), "+r"(r[24]), "+r"(r[25]),
                           "+r"(r[26]), "+r"(r[27]), "+r"(r[28]), "+r"(r[29]), "+r"(r[30]), "+r"(r[31])
                         :
                         : "memory");
        };
        int j = 0;
        for (int t = first; t < p.ntiles; t += step, ++j) {
            const int acc = j & 1, use = j >> 1;
            if (__any_sync(0xffffffffu, *fail != 0)) break;
            bool ok = mbar_wait(smem_u32(&s_tfull[acc]), (uint32_t)(use & 1), p.epi_spins);
            ok = __all_sync(0xffffffffu, ok);
            if (!ok) {
                if (lane == 0) *fail = 1;
                break;
            }
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            const int tx = t % p.tiles_x, trow = t / p.tiles_x;
            const int img = trow / p.tiles_y, y0 = (trow - img * p.tiles_y) * R;
            // shared A keeps the tile's pixels in slab order: accumulator lane
            // m = 32 q + lane holds pixel 16 (m % 8) + m / 8 of the tile
            const int x = sa ? tx * kTcM + 16 * (lane & 7) + 4 * q + (lane >> 3) : tx * kTcM + q * 32 + lane;
            const int cbase = slice * nt;
            const uint32_t tbase = tmem + (uint32_t)acc * acc_cols + ((uint32_t)(q * 32) << 16);
            // slice i: row i / per_row, columns 32 (i % per_row) ..
            auto taddr = [&](int i) {
                return pack ? tbase + 32u * (uint32_t)(R + 1 - i)
                            : tbase + (uint32_t)(i / per_row) * ncols + (uint32_t)(32 * (i % per_row));
            };
            auto process = [&](const uint32_t (&r)[32], int i) {
                const int rr = i / per_row, c = 32 * (i % per_row);
                const int y = y0 + rr;
                if (!(x < p.w && y < p.h)) return;
                const size_t pix = ((size_t)img * p.h + y) * p.w + x;
                const int cg = cbase + c;
                float hs = 0.f;  // fused head: channels in order (one 32-channel slice per pixel)
#pragma unroll
                for (int gi = 0; gi < 4; ++gi) {
                    float v[8];
#pragma unroll
                    for (int e = 0; e < 8; ++e) {
                        float f = __uint_as_float(r[8 * gi + e]);
                        if (p.bias) f += s_bias[c + 8 * gi + e];
                        if (p.relu) f = f > 0.f ? f : 0.f;
                        v[e] = f;
                    }
                    if (p.mask) {
                        float m[8];
                        unpack8(*reinterpret_cast<const uint4 *>(p.mask + pix * p.cout + cg + 8 * gi), m);
#pragma unroll
                        for (int e = 0; e < 8; ++e)
                            if (!(m[e] > 0.f)) v[e] = 0.f;
                    }
                    const uint4 pk = pack8(v);
                    if (!p.head_only) *reinterpret_cast<uint4 *>(p.out + pix * p.cout + cg + 8 * gi) = pk;
                    if (p.head_out) {
                        float vb[8];
                        unpack8(pk, vb);  // the BF16 values the head reads
#pragma unroll
                        for (int e = 0; e < 8; ++e) hs = fmaf(vb[e], s_hw[c + 8 * gi + e], hs);
                    }
                }
                if (p.head_out) {
                    hs += p.head_b[0];
                    if (p.head_scale) hs *= p.head_scale[img];
                    p.head_out[pix] = hs;
                }
            };
            // slices half, half + 2, ...; two register sets: the next slice's
            // load overlaps this slice's stores
            if (half < nslices) tld(ra, taddr(half));
            for (int i = half; i < nslices; i += 4) {
                twait(ra);
                if (i + 2 < nslices) tld(rb, taddr(i + 2));
                process(ra, i);
                if (i + 2 < nslices) {
                    twait(rb);
                    if (i + 4 < nslices) tld(ra, taddr(i + 4));
                    process(rb, i + 2);
                }
            }
            if (pack) {
                for (uint32_t c = 32u * (uint32_t)half; c < acc_cols; c += 64u) tmem_zero32(tbase + c);
                asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory");
            }
            asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
            __syncwarp();
            if (lane == 0) mbar_arrive(smem_u32(&s_tempty[acc]));
        }
    }
    __syncthreads();
    if (*fail) {
        // A wait gave up and the roles left their loops early: before the
        // tensor memory and the stages are released, let every copy and MMA
        // already issued finish.  Loads issued but never waited for have the
        // sequence numbers consumed .. issued - 1 (at most S of them, each in
        // its own stage, so the stage barrier's current phase is that load's);
        // one more commit arrives when every MMA issued so far has completed.
        // These waits are bounded too.
        if (tid == 0)
            for (int k = s_consumed; k < s_issued; ++k)
                if (!mbar_wait(smem_u32(&s_full[k % S]), (uint32_t)((k / S) & 1), p.spins)) break;
        if (warp == 1) {
            if (lane == 0) {
                asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                                 smem_u32(&s_drain))
                             : "memory");
                mbar_wait(smem_u32(&s_drain), 0u, p.spins);
            }
            __syncwarp();
        }
        __syncthreads();
        if (tid == 0 && p.err) atomicExch(p.err, 1);
    }
    if (warp == 0) {
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(tmem_cols));
    }
}

// Weights in the tensor-core kernel's staging order: one block of nt x kc
// per (slice, chunk, dx, dy), row co = output channel, kc input channels, the
// 16-byte groups of row co stored at group ^ swizzle(co) (128-byte swizzle:
// co & 7; 64-byte swizzle: (co >> 1) & 3), i.e. the shared-memory image.
__global__ void k_weights_tc(int cout, int cin, int nt, int kc, const bf16 *__restrict__ wk, bf16 *__restrict__ wtc)
{
    const long long total = 9LL * cout * cin;
    const int nch = cin / kc;
    for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < total;
         k += (long long)gridDim.x * blockDim.x) {
        // source index: tap, output channel, input channel
        const int ci = (int)(k % cin);
        const long long r = k / cin;
        const int co_all = (int)(r % cout);
        const int tap = (int)(r / cout);
        const int slice = co_all / nt, co = co_all - slice * nt;
        const int chunk = ci / kc, cl = ci - chunk * kc;
        const int grp = cl >> 3;
        const int swz = kc == 64 ? (co & 7) : ((co >> 1) & 3);
        const int dy = tap / 3, dx = tap - 3 * dy;
        const size_t block = ((((size_t)slice * nch + chunk) * 3 + dx) * 3 + dy) * (size_t)(nt * kc);
        wtc[block + (size_t)co * kc + (size_t)(((grp ^ swz) << 3) + (cl & 7))] = wk[k];
    }
}

// out[p] = [a[p], b[p / 2]] (nearest upsampling of b, then concatenation).
__global__ void k_concat_up(int n, int h, int w, int ca, int cb, const bf16 *__restrict__ a,
                            const bf16 *__restrict__ b, bf16 *__restrict__ out)
{
    const int ct = ca + cb, g8 = ct >> 3;
    const long long total = (long long)n * h * w * g8;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
         i += (long long)gridDim.x * blockDim.x) {
        const int g = (int)(i % g8);
        const long long pix = i / g8;
        const int x = (int)(pix % w), y = (int)((pix / w) % h);
        const long long img = pix / ((long long)w * h);
        const int c = 8 * g;
        const uint4 v = c < ca ? *reinterpret_cast<const uint4 *>(a + pix * ca + c)
                               : *reinterpret_cast<const uint4 *>(
                                     b + ((img * (h >> 1) + (y >> 1)) * (w >> 1) + (x >> 1)) * cb + (c - ca));
        *reinterpret_cast<uint4 *>(out + pix * ct + c) = v;
    }
}

// ----------------------------------------------------------------------------
// Weight gradient: dw[tap][o][i] += sum_p dz[p][o] * in[p + off(tap)][i].
// One CTA: 32 output x 32 input channels, all 9 taps (warp = tap), over a
// strided set of pixel tiles; per tile and tile row one k16 step of
// m = output channel, n = input channel, k = pixel.  Partial sums are added
// to the FP32 gradient with atomics once per CTA.
// ----------------------------------------------------------------------------
struct WgradArgs {
    const bf16 *dz;  // [n][h][w][cout]
    int cout;
    VIn in;
    float *dw;       // [9][cout][cin]
    int n, tiles_x, tiles_y, ntiles;
};

constexpr int kWgDz = 4 * (kTH * kTW) * 16;  // dz tile: 4 planes x 128 pixels
constexpr int kWgX = 4 * kHalo * 16;         // input halo: 4 planes x 180 pixels
constexpr int kWgStage = kWgDz + kWgX;
constexpr int kWgBytes = 2 * kWgStage;

__global__ void __launch_bounds__(288) k_wgrad3x3(WgradArgs p)
{
    extern __shared__ __align__(128) unsigned char smem[];
    const int co0 = blockIdx.x * 32, ci0 = blockIdx.y * 32;
    const int cin = p.in.ca + p.in.cb;
    const int tid = threadIdx.x, lane = tid & 31, tap = tid >> 5;
    const int dy = tap / 3, dx = tap - 3 * (tap / 3);
    const int H = p.in.h, W = p.in.w;

    auto load_tile = [&](int t, int s) {
        const int tx = t % p.tiles_x;
        const int ty = (t / p.tiles_x) % p.tiles_y;
        const int img = t / (p.tiles_x * p.tiles_y);
        const int y0 = ty * kTH, x0 = tx * kTW;
        unsigned char *base = smem + s * kWgStage;
        const uint32_t ds = smem_u32(base), xs = smem_u32(base + kWgDz);
        for (int i = tid; i < 4 * kTH * kTW; i += 288) {
            const int pl = i >> 7, px = i & 127;
            const int yy = y0 + (px >> 4), xx = x0 + (px & 15);
            const bool inside = yy < H && xx < W;
            const bf16 *src = inside ? p.dz + (((size_t)img * H + yy) * W + xx) * p.cout + co0 + 8 * pl : p.dz;
            cp_async16(ds + i * 16, src, inside ? 16 : 0);
        }
        for (int i = tid; i < 4 * kHalo; i += 288) {
            const int pl = i / kHalo, hidx = i - pl * kHalo;
            const int yy = y0 - 1 + hidx / kHW, xx = x0 - 1 + hidx % kHW;
            const bool inside = yy >= 0 && yy < H && xx >= 0 && xx < W;
            const bf16 *src = inside ? p.in.at(img, yy, xx, ci0 + 8 * pl) : p.in.a;
            cp_async16(xs + i * 16, src, inside ? 16 : 0);
        }
    };

    float acc[2][4][4];
#pragma unroll
    for (int a = 0; a < 2; ++a)
#pragma unroll
        for (int b = 0; b < 4; ++b)
#pragma unroll
            for (int c = 0; c < 4; ++c) acc[a][b][c] = 0.f;

    int t = blockIdx.z;
    if (t < p.ntiles) {
        load_tile(t, 0);
        cp_async_commit();
        const int q = lane >> 3, i8 = lane & 7;
        for (int s = 0; t < p.ntiles; t += gridDim.z, s ^= 1) {
            if (t + (int)gridDim.z < p.ntiles) load_tile(t + gridDim.z, s ^ 1);
            cp_async_commit();
            cp_async_wait<1>();
            __syncthreads();
            const unsigned char *base = smem + s * kWgStage;
            const uint32_t ds = smem_u32(base), xs = smem_u32(base + kWgDz);
#pragma unroll 1
            for (int r = 0; r < kTH; ++r) {
                uint32_t af[2][4];
#pragma unroll
                for (int mt = 0; mt < 2; ++mt) {
                    // transposed: matrix q = (channel half q & 1, pixel half q >> 1)
                    const int pl = 2 * mt + (q & 1);
                    const int px = r * kTW + (q >> 1) * 8 + i8;
                    ldsm4t(af[mt], ds + (pl * (kTH * kTW) + px) * 16);
                }
#pragma unroll
                for (int j = 0; j < 4; j += 2) {
                    // transposed: matrix q = (pixel half q & 1, input plane j + (q >> 1))
                    uint32_t bfr[4];
                    const int pl = j + (q >> 1);
                    const int hidx = (r + dy) * kHW + (q & 1) * 8 + i8 + dx;
                    ldsm4t(bfr, xs + (pl * kHalo + hidx) * 16);
#pragma unroll
                    for (int mt = 0; mt < 2; ++mt) {
                        mma16816(acc[mt][j], af[mt], bfr[0], bfr[1]);
                        mma16816(acc[mt][j + 1], af[mt], bfr[2], bfr[3]);
                    }
                }
            }
            __syncthreads();
        }
    }
    const int g = lane >> 2, tq = lane & 3;
#pragma unroll
    for (int mt = 0; mt < 2; ++mt)
#pragma unroll
        for (int j = 0; j < 4; ++j)
#pragma unroll
            for (int e = 0; e < 4; ++e) {
                const int co = co0 + mt * 16 + g + (e >> 1) * 8;
                const int ci = ci0 + j * 8 + tq * 2 + (e & 1);
                atomicAdd(p.dw + ((size_t)tap * p.cout + co) * cin + ci, acc[mt][j][e]);
            }
}

// db[c] += sum_p dz[p][c]; c divides 256 (32 .. 256 channels).
__global__ void __launch_bounds__(256) k_bias_grad(const bf16 *__restrict__ dz, long long npix, int c,
                                                  float *__restrict__ db)
{
    const int rows = 256 / c;
    const int ch = threadIdx.x % c, r0 = threadIdx.x / c;
    float s = 0.f;
    for (long long p = (long long)blockIdx.x * rows + r0; p < npix; p += (long long)gridDim.x * rows)
        s += __bfloat162float(dz[p * c + ch]);
    atomicAdd(db + ch, s);
}

// ----------------------------------------------------------------------------
// Element-wise kernels (8 channels = one 16-byte vector per thread)
// ----------------------------------------------------------------------------
// x[n][y][x][0..31] = in[n][c][y][x] / scale[n] (c < cin), 0 above.  Only
// the 8-channel groups that hold input channels are written: the groups
// above are the zeros the arena was cleared to, and nothing else writes x.
__global__ void k_pack_input(int n, int cin, int h, int w, const float *__restrict__ in,
                             const float *__restrict__ scale, bf16 *__restrict__ x)
{
    const long long npix = (long long)n * h * w;
    const int groups = (cin + 7) / 8;
    for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < npix;
         p += (long long)gridDim.x * blockDim.x) {
        const long long img = p / ((long long)h * w), yx = p - img * h * w;
        const float inv = scale ? 1.0f / scale[img] : 1.0f;
        uint4 *dst = reinterpret_cast<uint4 *>(x + p * kInPad);
        for (int k = 0; k < groups; ++k) {
            float g[8];
#pragma unroll
            for (int e = 0; e < 8; ++e) {
                const int c = 8 * k + e;
                g[e] = c < cin ? in[(img * cin + c) * h * w + yx] * inv : 0.f;
            }
            dst[k] = pack8(g);
        }
    }
}

// out[n][y][x][c] = mean of in over the 2x2 block (h, w of the input).
__global__ void k_pool2(int n, int h, int w, int c, const bf16 *__restrict__ in, bf16 *__restrict__ out)
{
    const int h2 = h >> 1, w2 = w >> 1, cg = c >> 3;
    const long long total = (long long)n * h2 * w2 * cg;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
         i += (long long)gridDim.x * blockDim.x) {
        const int g = (int)(i % cg);
        const long long pix = i / cg;
        const int x = (int)(pix % w2), y = (int)((pix / w2) % h2);
        const long long img = pix / ((long long)w2 * h2);
        float s[8] = {0, 0, 0, 0, 0, 0, 0, 0};
#pragma unroll
        for (int d = 0; d < 4; ++d) {
            const long long q = (img * h + 2 * y + (d >> 1)) * w + 2 * x + (d & 1);
            float f[8];
            unpack8(*reinterpret_cast<const uint4 *>(in + q * c + 8 * g), f);
#pragma unroll
            for (int e = 0; e < 8; ++e) s[e] += f[e];
        }
#pragma unroll
        for (int e = 0; e < 8; ++e) s[e] *= 0.25f;
        *reinterpret_cast<uint4 *>(out + pix * c + 8 * g) = pack8(s);
    }
}

// de[p][c] = (dp[p/2][c] / 4 + dcat[p][c]) * (e[p][c] > 0): the gradient of
// an encoder output e used by the pool below it and by the decoder's
// concatenation (first c of its ctot channels).
__global__ void k_pool_bwd_add(int n, int h, int w, int c, const bf16 *__restrict__ dp, const bf16 *__restrict__ dcat,
                               int ctot, const bf16 *__restrict__ e, bf16 *__restrict__ de)
{
    const int cg = c >> 3, w2 = w >> 1, h2 = h >> 1;
    const long long total = (long long)n * h * w * cg;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
         i += (long long)gridDim.x * blockDim.x) {
        const int g = (int)(i % cg);
        const long long pix = i / cg;
        const int x = (int)(pix % w), y = (int)((pix / w) % h);
        const long long img = pix / ((long long)w * h);
        float a[8], b[8], m[8];
        unpack8(*reinterpret_cast<const uint4 *>(dp + ((img * h2 + (y >> 1)) * w2 + (x >> 1)) * c + 8 * g), a);
        unpack8(*reinterpret_cast<const uint4 *>(dcat + pix * ctot + 8 * g), b);
        unpack8(*reinterpret_cast<const uint4 *>(e + pix * c + 8 * g), m);
        float o[8];
#pragma unroll
        for (int k = 0; k < 8; ++k) o[k] = (m[k] > 0.f) ? (a[k] * 0.25f + b[k]) : 0.f;
        *reinterpret_cast<uint4 *>(de + pix * c + 8 * g) = pack8(o);
    }
}

// dlow[q][c] = sum over the 2x2 block of dcat[p][coff + c], times
// (ylow[q][c] > 0); h, w of the full-resolution dcat.
__global__ void k_up_bwd(int n, int h, int w, int ctot, int coff, int c, const bf16 *__restrict__ dcat,
                         const bf16 *__restrict__ ylow, bf16 *__restrict__ dlow)
{
    const int h2 = h >> 1, w2 = w >> 1, cg = c >> 3;
    const long long total = (long long)n * h2 * w2 * cg;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
         i += (long long)gridDim.x * blockDim.x) {
        const int g = (int)(i % cg);
        const long long pix = i / cg;
        const int x = (int)(pix % w2), y = (int)((pix / w2) % h2);
        const long long img = pix / ((long long)w2 * h2);
        float s[8] = {0, 0, 0, 0, 0, 0, 0, 0};
#pragma unroll
        for (int d = 0; d < 4; ++d) {
            const long long q = (img * h + 2 * y + (d >> 1)) * w + 2 * x + (d & 1);
            float f[8];
            unpack8(*reinterpret_cast<const uint4 *>(dcat + q * ctot + coff + 8 * g), f);
#pragma unroll
            for (int e = 0; e < 8; ++e) s[e] += f[e];
        }
        float m[8];
        unpack8(*reinterpret_cast<const uint4 *>(ylow + pix * c + 8 * g), m);
#pragma unroll
        for (int e = 0; e < 8; ++e) s[e] = (m[e] > 0.f) ? s[e] : 0.f;
        *reinterpret_cast<uint4 *>(dlow + pix * c + 8 * g) = pack8(s);
    }
}

// out[p] = sum_c d0[p][c] * bf16(hw[c]) + hb, times scale[img] when given.
__global__ void k_head_fwd(long long npix, long long pix_per_img, int c, const bf16 *__restrict__ d0,
                           const float *__restrict__ hw, const float *__restrict__ hb,
                           const float *__restrict__ scale, float *__restrict__ out)
{
    for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < npix;
         p += (long long)gridDim.x * blockDim.x) {
        float s = 0.f;
        for (int g = 0; g < c / 8; ++g) {
            float f[8];
            unpack8(*reinterpret_cast<const uint4 *>(d0 + p * c + 8 * g), f);
#pragma unroll
            for (int e = 0; e < 8; ++e) s += f[e] * __bfloat162float(__float2bfloat16_rn(hw[8 * g + e]));
        }
        s += hb[0];
        if (scale) s *= scale[p / pix_per_img];
        out[p] = s;
    }
}

// dd0[p][c] = go[p] * bf16(hw[c]) * (d0[p][c] > 0); dhw[c] += sum_p go[p] d0[p][c];
// dhb += sum_p go[p].  c <= 64.
__global__ void __launch_bounds__(256) k_head_bwd(long long npix, int c, const bf16 *__restrict__ d0,
                                                 const float *__restrict__ hw, const float *__restrict__ go,
                                                 bf16 *__restrict__ dd0, float *__restrict__ dhw,
                                                 float *__restrict__ dhb)
{
    __shared__ float s_dw[65];
    for (int i = threadIdx.x; i < 65; i += blockDim.x) s_dw[i] = 0.f;
    __syncthreads();
    float part[64];
    for (int k = 0; k < 64; ++k) part[k] = 0.f;
    float pb = 0.f;
    for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < npix;
         p += (long long)gridDim.x * blockDim.x) {
        const float g = go[p];
        pb += g;
        for (int gi = 0; gi < c / 8; ++gi) {
            float f[8], o[8];
            unpack8(*reinterpret_cast<const uint4 *>(d0 + p * c + 8 * gi), f);
#pragma unroll
            for (int e = 0; e < 8; ++e) {
                const float wv = __bfloat162float(__float2bfloat16_rn(hw[8 * gi + e]));
                o[e] = (f[e] > 0.f) ? g * wv : 0.f;
                part[8 * gi + e] += g * f[e];
            }
            *reinterpret_cast<uint4 *>(dd0 + p * c + 8 * gi) = pack8(o);
        }
    }
    for (int k = 0; k < c; ++k) {
        float v = part[k];
        for (int off = 16; off; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
        if ((threadIdx.x & 31) == 0) atomicAdd(&s_dw[k], v);
    }
    for (int off = 16; off; off >>= 1) pb += __shfl_xor_sync(0xffffffffu, pb, off);
    if ((threadIdx.x & 31) == 0) atomicAdd(&s_dw[64], pb);
    __syncthreads();
    for (int k = threadIdx.x; k < c; k += blockDim.x) atomicAdd(dhw + k, s_dw[k]);
    if (threadIdx.x == 0) atomicAdd(dhb, s_dw[64]);
}

// BF16 copies of one layer's FP32 weights: w[tap][o][i] and the data-gradient
// form wt[8 - tap][i][o].
__global__ void k_layer_weights(int cout, int cin, const float *__restrict__ master, bf16 *__restrict__ w,
                                bf16 *__restrict__ wt)
{
    const int total = 9 * cout * cin;
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < total; k += gridDim.x * blockDim.x) {
        const int ci = k % cin, co = (k / cin) % cout, tap = k / (cin * cout);
        const bf16 v = __float2bfloat16_rn(master[k]);
        w[k] = v;
        wt[((size_t)(8 - tap) * cin + ci) * cout + co] = v;
    }
}

// Adam (Kingma & Ba 2015) on the FP32 master weights; c1 = 1 - beta1^t,
// c2 = 1 - beta2^t.
__global__ void k_adam(long long n, float *__restrict__ w, const float *__restrict__ g, float *__restrict__ m,
                       float *__restrict__ v, float lr, float b1, float b2, float eps, float c1, float c2)
{
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x) {
        const float gi = g[i];
        const float mi = b1 * m[i] + (1.f - b1) * gi;
        const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
        m[i] = mi;
        v[i] = vi;
        w[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
    }
}

// ----------------------------------------------------------------------------
// Loss: L = mean over pixels of (g * (pred - target))^2 with g the 3x3
// binomial kernel (1 2 1)^T (1 2 1) / 16, zero padding per image, so a
// component one pixel off costs little; grad = 2/npix * g * (g * (pred - target)).
// ----------------------------------------------------------------------------
__device__ __forceinline__ float binom3(const float *a, int h, int w, int y, int x)
{
    float s = 0.f;
#pragma unroll
    for (int dy = -1; dy <= 1; ++dy) {
        const int yy = y + dy;
        if (yy < 0 || yy >= h) continue;
#pragma unroll
        for (int dx = -1; dx <= 1; ++dx) {
            const int xx = x + dx;
            if (xx < 0 || xx >= w) continue;
            s += a[(size_t)yy * w + xx] * (float)((2 - (dy < 0 ? -dy : dy)) * (2 - (dx < 0 ? -dx : dx)));
        }
    }
    return s * (1.f / 16.f);
}

__global__ void k_diff(long long n, const float *__restrict__ a, const float *__restrict__ b, float *__restrict__ d)
{
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x)
        d[i] = a[i] - b[i];
}

__global__ void __launch_bounds__(256) k_blur_sq(int n, int h, int w, const float *__restrict__ d,
                                                float *__restrict__ bd, double *__restrict__ loss_sum)
{
    __shared__ double s_part[8];
    const long long total = (long long)n * h * w;
    double acc = 0.0;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
         i += (long long)gridDim.x * blockDim.x) {
        const long long img = i / ((long long)h * w);
        const int yx = (int)(i - img * h * w);
        const float v = binom3(d + img * h * w, h, w, yx / w, yx % w);
        bd[i] = v;
        acc += (double)v * v;
    }
    for (int off = 16; off; off >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, off);
    if ((threadIdx.x & 31) == 0) s_part[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        double s = 0.0;
        for (int k = 0; k < (int)(blockDim.x >> 5); ++k) s += s_part[k];
        atomicAdd(loss_sum, s);
    }
}

__global__ void k_blur_grad(int n, int h, int w, const float *__restrict__ bd, float scale, float *__restrict__ grad)
{
    const long long total = (long long)n * h * w;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
         i += (long long)gridDim.x * blockDim.x) {
        const long long img = i / ((long long)h * w);
        const int yx = (int)(i - img * h * w);
        grad[i] = scale * binom3(bd + img * h * w, h, w, yx / w, yx % w);
    }
}

__global__ void k_scale_loss(double *loss_sum, double inv_n) { loss_sum[0] *= inv_n; }

inline int grid_for(long long n, int threads = 256)
{
    long long b = (n + threads - 1) / threads;
    const long long cap = (long long)num_sms() * 16;
    return (int)(b < 1 ? 1 : (b > cap ? cap : b));
}

}  // namespace unet
}  // namespace sdp

// ============================================================================
// Host object
// ============================================================================
using namespace sdp;
using namespace sdp::unet;

namespace {
struct Layer {
    int cin, cout;
    size_t woff, boff;  // into the FP32 parameter vector
    bf16 *w = nullptr, *wt = nullptr;
    bf16 *wtc = nullptr, *wttc = nullptr;  // the two in the tensor-core kernel's staging order
};
struct Act {  // one activation tensor (and its gradient scratch)
    bf16 *p = nullptr;
    int level = 0, c = 0;
};
}  // namespace

struct sdp_unet {
    int base = 32, in_ch = 1, max_n = 1, max_h = 8, max_w = 8, training = 0;
    Layer layer[kLayers];
    size_t nparams = 0, head_off = 0;
    float *master = nullptr, *grad = nullptr, *adam_m = nullptr, *adam_v = nullptr;
    bf16 *wbuf = nullptr;  // BF16 weights (forward and transposed) of all layers
    long long step = 0;
    // forward activations
    bf16 *x = nullptr;
    bf16 *e[kLevels][2] = {};  // e[l][0] = e_l a, e[l][1] = e_l
    bf16 *pool[kLevels] = {};  // pool[l] = pool(e_{l-1}), l >= 1
    bf16 *d[kLevels - 1][2] = {};
    // gradient scratch (training)
    bf16 *gz[kLevels][2] = {};
    bf16 *dcat[kLevels - 1] = {};
    bf16 *cat[kLevels - 1] = {};  // [e_l, up(low)] materialised for the tensor-core path
    // shape of the last forward pass
    int n = 0, h = 0, w = 0;
    bool have_forward = false;
    int tensor_path = 1;    // 1: tcgen05 convolutions, 0: mma.sync
    int *err = nullptr;     // device flag: a bounded wait gave up
    long long epi_spins = 0;  // epilogue wait limit of the tensor-core kernel (0: the default)
    void *arena = nullptr;
};

namespace {

int ch(const sdp_unet *u, int l) { return u->base << l; }

size_t pix(const sdp_unet *u, int l) { return (size_t)u->max_n * (u->max_h >> l) * (u->max_w >> l); }

// Layer table in parameter order: e0a e0 e1a e1 e2a e2 e3a e3 d2a d2 d1a d1 d0a d0.
void layer_shapes(sdp_unet *u)
{
    int k = 0;
    for (int l = 0; l < kLevels; ++l) {
        u->layer[k].cin = l == 0 ? kInPad : ch(u, l - 1);
        u->layer[k++].cout = ch(u, l);
        u->layer[k].cin = ch(u, l);
        u->layer[k++].cout = ch(u, l);
    }
    for (int l = kLevels - 2; l >= 0; --l) {
        u->layer[k].cin = ch(u, l) + ch(u, l + 1);
        u->layer[k++].cout = ch(u, l);
        u->layer[k].cin = ch(u, l);
        u->layer[k++].cout = ch(u, l);
    }
    size_t off = 0;
    for (auto &L : u->layer) {
        L.woff = off;
        off += (size_t)9 * L.cin * L.cout;
        L.boff = off;
        off += L.cout;
    }
    u->head_off = off;
    u->nparams = off + ch(u, 0) + 1;
}

int enc_layer(int l, int second) { return 2 * l + second; }
int dec_layer(int l, int second) { return 8 + 2 * (kLevels - 2 - l) + second; }

size_t tiles(int n, int h, int w) { return (size_t)n * ((h + kTH - 1) / kTH) * ((w + kTW - 1) / kTW); }

// Output-channel slices of a tensor-core convolution: nt = cout / slices <= 256,
// a multiple of 32.
int tc_slices(int cout)
{
    int ny = (cout + 255) / 256;
    while (cout % ny != 0 || (cout / ny) % 32 != 0) ++ny;
    return ny;
}

PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder()
{
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    if (!fn) {
        void *f = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &f, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(f);
    }
    return fn;
}

// The 1x1 head fused into a convolution's epilogue (see TcArgs).
struct HeadFuse {
    const float *w = nullptr, *b = nullptr, *scale = nullptr;
    float *out = nullptr;
    int only = 0;
};

int conv_tc(const bf16 *in, int cin, int h, int w, int n, const bf16 *wtc, const float *bias, const bf16 *mask,
            bf16 *out, int cout, int relu, int *err, long long epi_spins, cudaStream_t st,
            const HeadFuse *head = nullptr)
{
    SDP_CHECK_ARG(cin % 32 == 0 && cout % 32 == 0, "tensor-core convolution: channels %d -> %d", cin, cout);
    auto enc = tensor_map_encoder();
    if (!enc) return set_error(SDP_ERR_CUDA, "cuTensorMapEncodeTiled unavailable");
    const int ny = tc_slices(cout);
    const int nt = cout / ny;
    const int tiles_x = (w + kTcM - 1) / kTcM;
    // rows per tile: as many as tensor memory holds (two sets of R
    // accumulators) while the tiles still cover the SMs and at least three
    // stages fit in shared memory
    const int kc = tc_kc(cin);
    const int pack = nt == 32 ? 1 : 0;
    auto choose_rows = [&](int sa, int min_stages) {
        int rr = 8;
        while (rr > 1 && (2u * tc_acc_cols(pack, rr, nt) > 512u || tc_stages(nt, kc, rr, sa) < min_stages ||
                          (long long)n * ((h + rr - 1) / rr) * tiles_x * ny < num_sms()))
            rr >>= 1;
        return rr;
    };
    const cuuint64_t dims[4] = {(cuuint64_t)cin, (cuuint64_t)w, (cuuint64_t)h, (cuuint64_t)n};
    const cuuint64_t strides[3] = {(cuuint64_t)cin * 2, (cuuint64_t)w * cin * 2, (cuuint64_t)h * w * cin * 2};
    const cuuint32_t estr[5] = {1, 1, 1, 1, 1};
    // Shared A (one load of each chunk serves the three column taps): the
    // tile's 128 pixels x0 + 16 j + k (j < 8, k < 16) are staged as slabs
    // k = -1 .. 16 of 8 pixels (rows of KC channels), slab-major, so a shift
    // of one pixel is one slab (8 rows, one 512-byte swizzle atom) and the
    // MMA of column tap dx starts at slab dx.  Two 5-D tensor maps view the
    // image as {C, j (16 pixels apart), y, k (1 pixel apart), n}: slabs 0..15
    // of one tile in one box, the two neighbour slabs (k = 15 of the group to
    // the left, k = 0 of the group to the right) in boxes of one slab; reads
    // outside the image (j or y out of range) return zero.  Needs W % 16 == 0
    // and nt <= 64 (the chunk's nine weight blocks share the stage).
    int sa = (w % 16 == 0 && nt <= 64) ? 1 : 0;
    int R = sa ? choose_rows(1, 2) : choose_rows(0, 3);
    CUtensorMap tmap, tslab, thalo;
    if (sa) {
        const cuuint64_t d5[5] = {(cuuint64_t)cin, (cuuint64_t)(w / 16), (cuuint64_t)h, 16, (cuuint64_t)n};
        const cuuint64_t s5[4] = {(cuuint64_t)cin * 2 * 16, (cuuint64_t)w * cin * 2, (cuuint64_t)cin * 2,
                                  (cuuint64_t)h * w * cin * 2};
        const cuuint32_t bslab[5] = {(cuuint32_t)kc, 8, (cuuint32_t)(R + 2), 16, 1};
        const cuuint32_t bhalo[5] = {(cuuint32_t)kc, 8, (cuuint32_t)(R + 2), 1, 1};
        const CUresult r1 = enc(&tslab, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 5, const_cast<bf16 *>(in), d5, s5, bslab,
                                estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_64B,
                                CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
        const CUresult r2 = enc(&thalo, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 5, const_cast<bf16 *>(in), d5, s5, bhalo,
                                estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_64B,
                                CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
        if (r1 != CUDA_SUCCESS || r2 != CUDA_SUCCESS) {  // the driver refused the view: one box per column tap
            sa = 0;
            R = choose_rows(0, 3);
        }
    }
    SDP_CHECK_ARG(tc_stages(nt, kc, R, sa) >= 2, "tensor-core convolution: %d output channels do not fit", nt);
    {
        const cuuint32_t box[4] = {(cuuint32_t)kc, (cuuint32_t)kTcM, (cuuint32_t)(R + 2), 1};
        const CUresult r = enc(&tmap, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 4, const_cast<bf16 *>(in), dims, strides, box,
                               estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_64B,
                               CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
        if (r != CUDA_SUCCESS) return set_error(SDP_ERR_CUDA, "cuTensorMapEncodeTiled failed (%d)", (int)r);
    }
    if (!sa) tslab = thalo = tmap;  // unused
    TcArgs a;
    a.n = n;
    a.h = h;
    a.w = w;
    a.cin = cin;
    a.cout = cout;
    a.nt = nt;
    a.kc = kc;
    a.nchunks = cin / kc;
    a.rows = R;
    a.tiles_x = tiles_x;
    a.tiles_y = (h + R - 1) / R;
    a.ntiles = n * a.tiles_y * tiles_x;
    a.stages = tc_stages(nt, kc, R, sa);
    a.wtc = wtc;
    a.bias = bias;
    a.mask = mask;
    a.out = out;
    a.relu = relu;
    a.err = err;
    a.spins = kTcSpins;
    a.epi_spins = epi_spins > 0 ? epi_spins : kTcSpins;
    a.pack = pack;
    a.sa = sa;
    a.head_w = head ? head->w : nullptr;
    a.head_b = head ? head->b : nullptr;
    a.head_scale = head ? head->scale : nullptr;
    a.head_out = head ? head->out : nullptr;
    a.head_only = head ? head->only : 0;
    SDP_CHECK_ARG(!head || (ny == 1 && nt == 32), "head fusion needs 32 output channels");
    int per_slice = num_sms() / ny;
    if (per_slice < 1) per_slice = 1;
    if (per_slice > a.ntiles) per_slice = a.ntiles;
    const size_t smem = (size_t)a.stages * tc_stage_bytes(nt, kc, R, sa) + 1024;
    k_conv3x3_tc<<<dim3((unsigned)per_slice, ny), kTcThreads, smem, st>>>(tmap, tslab, thalo, a);
    SDP_LAUNCH_CHECK();
    return SDP_OK;
}

// wk: [9][cout][cin] for the mma.sync kernel; wtc: the same weights in the
// tensor-core staging order (the tensor-core path reads a plain input, in.cb == 0).
int conv(const sdp_unet *u, VIn in, const bf16 *wk, const bf16 *wtc, const float *bias, const bf16 *mask, bf16 *out,
         int cout, int relu, int n, cudaStream_t st, const HeadFuse *head = nullptr)
{
    if (u->tensor_path) {
        SDP_CHECK_ARG(in.cb == 0, "tensor-core convolution reads a materialised input");
        return conv_tc(in.a, in.ca, in.h, in.w, n, wtc, bias, mask, out, cout, relu, u->err, u->epi_spins, st, head);
    }
    SDP_CHECK_ARG(!head, "the head is fused on the tensor-core path only");
    ConvArgs a;
    a.in = in;
    a.wk = wk;
    a.bias = bias;
    a.mask = mask;
    a.out = out;
    a.cout = cout;
    a.relu = relu;
    a.tiles_x = (in.w + kTW - 1) / kTW;
    a.tiles_y = (in.h + kTH - 1) / kTH;
    const size_t nt = tiles(n, in.h, in.w);
    if (cout % 64 == 0 && nt * (cout / 64) >= (size_t)2 * num_sms()) {
        k_conv3x3<64><<<dim3((unsigned)nt, cout / 64), 128, ConvSmem<64>::kBytes, st>>>(a);
    } else {
        k_conv3x3<32><<<dim3((unsigned)nt, cout / 32), 128, ConvSmem<32>::kBytes, st>>>(a);
    }
    SDP_LAUNCH_CHECK();
    return SDP_OK;
}

int wgrad(const bf16 *dz, int cout, VIn in, float *dw, float *db, int n, cudaStream_t st)
{
    WgradArgs a;
    a.dz = dz;
    a.cout = cout;
    a.in = in;
    a.dw = dw;
    a.n = n;
    a.tiles_x = (in.w + kTW - 1) / kTW;
    a.tiles_y = (in.h + kTH - 1) / kTH;
    a.ntiles = (int)tiles(n, in.h, in.w);
    const int cin = in.ca + in.cb;
    const int blocks_xy = (cout / 32) * (cin / 32);
    int z = (4 * num_sms() + blocks_xy - 1) / blocks_xy;
    if (z > a.ntiles) z = a.ntiles;
    if (z < 1) z = 1;
    k_wgrad3x3<<<dim3(cout / 32, cin / 32, z), 288, kWgBytes, st>>>(a);
    SDP_LAUNCH_CHECK();
    const long long np = (long long)n * in.h * in.w;
    k_bias_grad<<<grid_for(np / (256 / cout) + 1), 256, 0, st>>>(dz, np, cout, db);
    SDP_LAUNCH_CHECK();
    return SDP_OK;
}

VIn vin(const bf16 *a, int ca, const bf16 *b, int cb, int h, int w)
{
    VIn v;
    v.a = a;
    v.b = b;
    v.ca = ca;
    v.cb = cb;
    v.h = h;
    v.w = w;
    return v;
}

int set_attrs()
{
    static bool done = false;
    if (done) return SDP_OK;
    SDP_CUDA_TRY(cudaFuncSetAttribute(k_conv3x3<32>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      ConvSmem<32>::kBytes));
    SDP_CUDA_TRY(cudaFuncSetAttribute(k_conv3x3<64>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      ConvSmem<64>::kBytes));
    SDP_CUDA_TRY(cudaFuncSetAttribute(k_wgrad3x3, cudaFuncAttributeMaxDynamicSharedMemorySize, kWgBytes));
    SDP_CUDA_TRY(cudaFuncSetAttribute(k_conv3x3_tc, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      kTcSmemBudget + 1024));
    done = true;
    return SDP_OK;
}

int refresh_weights(sdp_unet *u, cudaStream_t st)
{
    for (auto &L : u->layer) {
        const int total = 9 * L.cin * L.cout;
        k_layer_weights<<<grid_for(total), 256, 0, st>>>(L.cout, L.cin, u->master + L.woff, L.w, L.wt);
        SDP_LAUNCH_CHECK();
        k_weights_tc<<<grid_for(total), 256, 0, st>>>(L.cout, L.cin, L.cout / tc_slices(L.cout), tc_kc(L.cin), L.w,
                                                      L.wtc);
        SDP_LAUNCH_CHECK();
        k_weights_tc<<<grid_for(total), 256, 0, st>>>(L.cin, L.cout, L.cin / tc_slices(L.cin), tc_kc(L.cout), L.wt,
                                                      L.wttc);
        SDP_LAUNCH_CHECK();
    }
    return SDP_OK;
}

}  // namespace

SDP_EXPORT int sdp_unet_create(sdp_unet **out, int base_channels, int in_channels, int max_batch, int max_height,
                               int max_width, int training)
{
    SDP_CHECK_ARG(out, "NULL handle");
    *out = nullptr;
    SDP_CHECK_ARG(base_channels == 32, "base_channels must be 32");
    SDP_CHECK_ARG(in_channels >= 1 && in_channels <= kInPad, "in_channels must be 1..%d", kInPad);
    SDP_CHECK_ARG(max_batch >= 1 && max_height >= 8 && max_width >= 8, "sizes must be positive, images >= 8 x 8");
    SDP_CHECK_ARG(max_height % 8 == 0 && max_width % 8 == 0, "image sides must be multiples of 8");
    SDP_CHECK_ARG((long long)max_batch * max_height * max_width <= (1LL << 31) / 2,
                  "batch x height x width too large");
    SDP_TRY(set_attrs());
    sdp_unet *u = new sdp_unet();
    u->base = base_channels;
    u->in_ch = in_channels;
    u->max_n = max_batch;
    u->max_h = max_height;
    u->max_w = max_width;
    u->training = training ? 1 : 0;
    layer_shapes(u);

    // one arena: FP32 parameters (+ gradient and Adam moments when training),
    // BF16 weights, activations and gradient scratch
    size_t bytes = 0;
    auto take = [&](size_t b) {
        const size_t at = bytes;
        bytes += (b + 255) & ~(size_t)255;
        return at;
    };
    const size_t o_err = take(sizeof(int));
    const size_t o_master = take(u->nparams * 4);
    const size_t o_grad = u->training ? take(u->nparams * 4) : 0;
    const size_t o_m = u->training ? take(u->nparams * 4) : 0;
    const size_t o_v = u->training ? take(u->nparams * 4) : 0;
    size_t o_w[kLayers], o_wt[kLayers], o_wtc[kLayers], o_wttc[kLayers];
    for (int k = 0; k < kLayers; ++k) {
        const size_t wb = (size_t)9 * u->layer[k].cin * u->layer[k].cout * 2;
        o_w[k] = take(wb);
        o_wt[k] = take(wb);
        o_wtc[k] = take(wb);
        o_wttc[k] = take(wb);
    }
    const size_t o_x = take(pix(u, 0) * kInPad * 2);
    size_t o_e[kLevels][2], o_pool[kLevels] = {}, o_d[kLevels - 1][2], o_gz[kLevels][2] = {}, o_dcat[kLevels - 1] = {};
    for (int l = 0; l < kLevels; ++l) {
        o_e[l][0] = take(pix(u, l) * ch(u, l) * 2);
        o_e[l][1] = take(pix(u, l) * ch(u, l) * 2);
        if (l > 0) o_pool[l] = take(pix(u, l) * ch(u, l - 1) * 2);
    }
    size_t o_cat[kLevels - 1];
    for (int l = 0; l < kLevels - 1; ++l) {
        o_d[l][0] = take(pix(u, l) * ch(u, l) * 2);
        o_d[l][1] = take(pix(u, l) * ch(u, l) * 2);
        o_cat[l] = take(pix(u, l) * (ch(u, l) + ch(u, l + 1)) * 2);
    }
    if (u->training) {
        for (int l = 0; l < kLevels; ++l) {
            o_gz[l][0] = take(pix(u, l) * ch(u, l) * 2);
            o_gz[l][1] = take(pix(u, l) * ch(u, l) * 2);
        }
        for (int l = 0; l < kLevels - 1; ++l) o_dcat[l] = take(pix(u, l) * (ch(u, l) + ch(u, l + 1)) * 2);
    }
    void *arena = nullptr;
    cudaError_t e = cudaMalloc(&arena, bytes);
    if (e != cudaSuccess) {
        delete u;
        return cuda_error(e, "cudaMalloc(unet arena)");
    }
    u->arena = arena;
    char *A = static_cast<char *>(arena);
    u->err = reinterpret_cast<int *>(A + o_err);
    u->master = reinterpret_cast<float *>(A + o_master);
    if (u->training) {
        u->grad = reinterpret_cast<float *>(A + o_grad);
        u->adam_m = reinterpret_cast<float *>(A + o_m);
        u->adam_v = reinterpret_cast<float *>(A + o_v);
    }
    for (int k = 0; k < kLayers; ++k) {
        u->layer[k].w = reinterpret_cast<bf16 *>(A + o_w[k]);
        u->layer[k].wt = reinterpret_cast<bf16 *>(A + o_wt[k]);
        u->layer[k].wtc = reinterpret_cast<bf16 *>(A + o_wtc[k]);
        u->layer[k].wttc = reinterpret_cast<bf16 *>(A + o_wttc[k]);
    }
    u->x = reinterpret_cast<bf16 *>(A + o_x);
    for (int l = 0; l < kLevels; ++l) {
        u->e[l][0] = reinterpret_cast<bf16 *>(A + o_e[l][0]);
        u->e[l][1] = reinterpret_cast<bf16 *>(A + o_e[l][1]);
        if (l > 0) u->pool[l] = reinterpret_cast<bf16 *>(A + o_pool[l]);
        if (u->training) {
            u->gz[l][0] = reinterpret_cast<bf16 *>(A + o_gz[l][0]);
            u->gz[l][1] = reinterpret_cast<bf16 *>(A + o_gz[l][1]);
        }
    }
    for (int l = 0; l < kLevels - 1; ++l) {
        u->d[l][0] = reinterpret_cast<bf16 *>(A + o_d[l][0]);
        u->d[l][1] = reinterpret_cast<bf16 *>(A + o_d[l][1]);
        u->cat[l] = reinterpret_cast<bf16 *>(A + o_cat[l]);
        if (u->training) u->dcat[l] = reinterpret_cast<bf16 *>(A + o_dcat[l]);
    }
    e = cudaMemset(arena, 0, bytes);
    if (e != cudaSuccess) {
        cudaFree(arena);
        delete u;
        return cuda_error(e, "cudaMemset(unet arena)");
    }
    *out = u;
    return SDP_OK;
}

SDP_EXPORT int sdp_unet_destroy(sdp_unet *u)
{
    if (!u) return SDP_OK;
    cudaDeviceSynchronize();
    if (u->arena) cudaFree(u->arena);
    delete u;
    return SDP_OK;
}

SDP_EXPORT int sdp_unet_set_tensor_path(sdp_unet *u, int tcgen05)
{
    SDP_CHECK_ARG(u, "NULL handle");
    u->tensor_path = tcgen05 ? 1 : 0;
    return SDP_OK;
}

SDP_EXPORT int sdp_unet_set_wait_limit(sdp_unet *u, long long epilogue_polls)
{
    SDP_CHECK_ARG(u, "NULL handle");
    SDP_CHECK_ARG(epilogue_polls >= 0, "epilogue_polls %lld is negative", epilogue_polls);
    u->epi_spins = epilogue_polls;
    return SDP_OK;
}

SDP_EXPORT int sdp_unet_check(sdp_unet *u, void *stream)
{
    SDP_CHECK_ARG(u, "NULL handle");
    int h = 0;
    SDP_CUDA_TRY(cudaMemcpyAsync(&h, u->err, sizeof(int), cudaMemcpyDeviceToHost, as_stream(stream)));
    SDP_CUDA_TRY(cudaStreamSynchronize(as_stream(stream)));
    if (h) {
        SDP_CUDA_TRY(cudaMemsetAsync(u->err, 0, sizeof(int), as_stream(stream)));
        return set_error(SDP_ERR_TIMEOUT, "a tensor-core convolution gave up waiting for its MMAs");
    }
    return SDP_OK;
}

SDP_EXPORT int sdp_unet_num_params(const sdp_unet *u, size_t *count)
{
    SDP_CHECK_ARG(u && count, "NULL argument");
    *count = u->nparams;
    return SDP_OK;
}

SDP_EXPORT int sdp_unet_layer(const sdp_unet *u, int layer, int *in_channels, int *out_channels,
                              size_t *weight_offset, size_t *bias_offset)
{
    SDP_CHECK_ARG(u, "NULL handle");
    SDP_CHECK_ARG(layer >= 0 && layer <= kLayers, "layer must be 0..%d (%d = output head)", kLayers, kLayers);
    if (layer == kLayers) {
        if (in_channels) *in_channels = ch(u, 0);
        if (out_channels) *out_channels = 1;
        if (weight_offset) *weight_offset = u->head_off;
        if (bias_offset) *bias_offset = u->head_off + ch(u, 0);
        return SDP_OK;
    }
    const Layer &L = u->layer[layer];
    if (in_channels) *in_channels = L.cin;
    if (out_channels) *out_channels = L.cout;
    if (weight_offset) *weight_offset = L.woff;
    if (bias_offset) *bias_offset = L.boff;
    return SDP_OK;
}

SDP_EXPORT int sdp_unet_set_params(sdp_unet *u, const float *params, void *stream)
{
    SDP_CHECK_ARG(u && params, "NULL argument");
    cudaStream_t st = as_stream(stream);
    SDP_CUDA_TRY(cudaMemcpyAsync(u->master, params, u->nparams * 4, cudaMemcpyDefault, st));
    SDP_TRY(refresh_weights(u, st));
    if (u->training) {
        SDP_CUDA_TRY(cudaMemsetAsync(u->adam_m, 0, u->nparams * 4, st));
        SDP_CUDA_TRY(cudaMemsetAsync(u->adam_v, 0, u->nparams * 4, st));
        u->step = 0;
    }
    return SDP_OK;
}

SDP_EXPORT int sdp_unet_get_params(const sdp_unet *u, float *params, void *stream)
{
    SDP_CHECK_ARG(u && params, "NULL argument");
    SDP_CUDA_TRY(cudaMemcpyAsync(params, u->master, u->nparams * 4, cudaMemcpyDefault, as_stream(stream)));
    return SDP_OK;
}

SDP_EXPORT int sdp_unet_get_grads(const sdp_unet *u, float *grads, void *stream)
{
    SDP_CHECK_ARG(u && grads, "NULL argument");
    if (!u->training) return set_error(SDP_ERR_INVALID, "network created without training buffers");
    SDP_CUDA_TRY(cudaMemcpyAsync(grads, u->grad, u->nparams * 4, cudaMemcpyDefault, as_stream(stream)));
    return SDP_OK;
}

SDP_EXPORT int sdp_unet_zero_grads(sdp_unet *u, void *stream)
{
    SDP_CHECK_ARG(u, "NULL handle");
    if (!u->training) return set_error(SDP_ERR_INVALID, "network created without training buffers");
    SDP_CUDA_TRY(cudaMemsetAsync(u->grad, 0, u->nparams * 4, as_stream(stream)));
    return SDP_OK;
}

SDP_EXPORT int sdp_unet_forward(sdp_unet *u, int n, int h, int w, const float *input, const float *scale,
                                float *output, void *stream)
{
    SDP_CHECK_ARG(u && input && output, "NULL argument");
    SDP_CHECK_ARG(n >= 1 && n <= u->max_n && h >= 8 && h <= u->max_h && w >= 8 && w <= u->max_w,
                  "batch %d x %d x %d outside the network's capacity %d x %d x %d", n, h, w, u->max_n, u->max_h,
                  u->max_w);
    SDP_CHECK_ARG(h % 8 == 0 && w % 8 == 0, "image sides must be multiples of 8");
    cudaStream_t st = as_stream(stream);
    const long long np = (long long)n * h * w;
    k_pack_input<<<grid_for(np), 256, 0, st>>>(n, u->in_ch, h, w, input, scale, u->x);
    SDP_LAUNCH_CHECK();
    const float *P = u->master;
    // encoder
    for (int l = 0; l < kLevels; ++l) {
        const int hl = h >> l, wl = w >> l, c = ch(u, l);
        const bf16 *src = l == 0 ? u->x : u->pool[l];
        const int cs = l == 0 ? kInPad : ch(u, l - 1);
        if (l > 0) {
            const int cp = ch(u, l - 1);
            k_pool2<<<grid_for((long long)n * hl * wl * (cp / 8)), 256, 0, st>>>(n, h >> (l - 1), w >> (l - 1), cp,
                                                                              u->e[l - 1][1], u->pool[l]);
            SDP_LAUNCH_CHECK();
        }
        const Layer &La = u->layer[enc_layer(l, 0)], &Lb = u->layer[enc_layer(l, 1)];
        SDP_TRY(conv(u, vin(src, cs, nullptr, 0, hl, wl), La.w, La.wtc, P + La.boff, nullptr, u->e[l][0], c, 1, n,
                     st));
        SDP_TRY(conv(u, vin(u->e[l][0], c, nullptr, 0, hl, wl), Lb.w, Lb.wtc, P + Lb.boff, nullptr, u->e[l][1], c,
                     1, n,
                     st));
    }
    // decoder
    for (int l = kLevels - 2; l >= 0; --l) {
        const int hl = h >> l, wl = w >> l, c = ch(u, l), c1 = ch(u, l + 1);
        const bf16 *low = (l == kLevels - 2) ? u->e[l + 1][1] : u->d[l + 1][1];
        const Layer &La = u->layer[dec_layer(l, 0)], &Lb = u->layer[dec_layer(l, 1)];
        VIn cat_in = vin(u->e[l][1], c, low, c1, hl, wl);
        if (u->tensor_path) {
            k_concat_up<<<grid_for((long long)n * hl * wl * ((c + c1) / 8)), 256, 0, st>>>(n, hl, wl, c, c1,
                                                                                           u->e[l][1], low, u->cat[l]);
            SDP_LAUNCH_CHECK();
            cat_in = vin(u->cat[l], c + c1, nullptr, 0, hl, wl);
        }
        SDP_TRY(conv(u, cat_in, La.w, La.wtc, P + La.boff, nullptr, u->d[l][0], c, 1, n, st));
        // the top level's last convolution also computes the 1x1 head in its
        // epilogue on the tensor-core path (and, without training buffers,
        // does not store its activations: nothing reads them)
        HeadFuse hf;
        const bool fuse = u->tensor_path && l == 0 && ch(u, 0) == 32;
        if (fuse) {
            hf.w = P + u->head_off;
            hf.b = P + u->head_off + ch(u, 0);
            hf.scale = scale;
            hf.out = output;
            hf.only = u->training ? 0 : 1;
        }
        SDP_TRY(conv(u, vin(u->d[l][0], c, nullptr, 0, hl, wl), Lb.w, Lb.wtc, P + Lb.boff, nullptr, u->d[l][1], c,
                     1, n, st, fuse ? &hf : nullptr));
    }
    if (!(u->tensor_path && ch(u, 0) == 32)) {
        k_head_fwd<<<grid_for(np), 256, 0, st>>>(np, (long long)h * w, ch(u, 0), u->d[0][1], P + u->head_off,
                                                 P + u->head_off + ch(u, 0), scale, output);
        SDP_LAUNCH_CHECK();
    }
    u->n = n;
    u->h = h;
    u->w = w;
    u->have_forward = true;
    return SDP_OK;
}

SDP_EXPORT int sdp_unet_backward(sdp_unet *u, const float *grad_output, void *stream)
{
    SDP_CHECK_ARG(u && grad_output, "NULL argument");
    if (!u->training) return set_error(SDP_ERR_INVALID, "network created without training buffers");
    if (!u->have_forward) return set_error(SDP_ERR_INVALID, "backward before forward");
    cudaStream_t st = as_stream(stream);
    const int n = u->n, h = u->h, w = u->w;
    const long long np = (long long)n * h * w;
    float *G = u->grad;
    const int c0 = ch(u, 0);
    // head: dZ(d0) -> gz[0][0]
    k_head_bwd<<<grid_for(np), 256, 0, st>>>(np, c0, u->d[0][1], u->master + u->head_off, grad_output, u->gz[0][0],
                                             G + u->head_off, G + u->head_off + c0);
    SDP_LAUNCH_CHECK();
    // decoder, top (level 0) down to level kLevels - 2; gz[l][0] holds dZ of d_l on entry
    for (int l = 0; l <= kLevels - 2; ++l) {
        const int hl = h >> l, wl = w >> l, c = ch(u, l), c1 = ch(u, l + 1);
        const Layer &La = u->layer[dec_layer(l, 0)], &Lb = u->layer[dec_layer(l, 1)];
        // second conv: d_l = conv(d_l a)
        SDP_TRY(wgrad(u->gz[l][0], c, vin(u->d[l][0], c, nullptr, 0, hl, wl), G + Lb.woff, G + Lb.boff, n, st));
        SDP_TRY(conv(u, vin(u->gz[l][0], c, nullptr, 0, hl, wl), Lb.wt, Lb.wttc, nullptr, u->d[l][0], u->gz[l][1],
                     c, 0, n,
                     st));
        // first conv: d_l a = conv([e_l, up(low)])
        const bf16 *low = (l == kLevels - 2) ? u->e[l + 1][1] : u->d[l + 1][1];
        SDP_TRY(wgrad(u->gz[l][1], c, vin(u->e[l][1], c, low, c1, hl, wl), G + La.woff, G + La.boff, n, st));
        SDP_TRY(conv(u, vin(u->gz[l][1], c, nullptr, 0, hl, wl), La.wt, La.wttc, nullptr, nullptr, u->dcat[l],
                     c + c1, 0, n,
                     st));
        // up-sampled part -> dZ of the lower tensor (d_{l+1} or e_3)
        k_up_bwd<<<grid_for((long long)n * (hl / 2) * (wl / 2) * (c1 / 8)), 256, 0, st>>>(
            n, hl, wl, c + c1, c, c1, u->dcat[l], low, u->gz[l + 1][0]);
        SDP_LAUNCH_CHECK();
    }
    // encoder, bottom (level kLevels - 1) up to level 0; gz[l][0] holds dZ of e_l on entry
    for (int l = kLevels - 1; l >= 0; --l) {
        const int hl = h >> l, wl = w >> l, c = ch(u, l);
        const Layer &La = u->layer[enc_layer(l, 0)], &Lb = u->layer[enc_layer(l, 1)];
        SDP_TRY(wgrad(u->gz[l][0], c, vin(u->e[l][0], c, nullptr, 0, hl, wl), G + Lb.woff, G + Lb.boff, n, st));
        SDP_TRY(conv(u, vin(u->gz[l][0], c, nullptr, 0, hl, wl), Lb.wt, Lb.wttc, nullptr, u->e[l][0], u->gz[l][1],
                     c, 0, n,
                     st));
        const bf16 *src = l == 0 ? u->x : u->pool[l];
        const int cs = l == 0 ? kInPad : ch(u, l - 1);
        SDP_TRY(wgrad(u->gz[l][1], c, vin(src, cs, nullptr, 0, hl, wl), G + La.woff, G + La.boff, n, st));
        if (l == 0) break;
        // data gradient of the pooled input (cs channels at level l), into gz[l][0]
        SDP_TRY(conv(u, vin(u->gz[l][1], c, nullptr, 0, hl, wl), La.wt, La.wttc, nullptr, nullptr, u->gz[l][0],
                     cs, 0, n,
                     st));
        // dZ(e_{l-1}) = (pool backward + concatenation part) * relu'
        const int hu = h >> (l - 1), wu = w >> (l - 1);
        k_pool_bwd_add<<<grid_for((long long)n * hu * wu * (cs / 8)), 256, 0, st>>>(
            n, hu, wu, cs, u->gz[l][0], u->dcat[l - 1], cs + c, u->e[l - 1][1], u->gz[l - 1][0]);
        SDP_LAUNCH_CHECK();
    }
    return SDP_OK;
}

SDP_EXPORT int sdp_unet_adam_step(sdp_unet *u, float lr, float beta1, float beta2, float eps, void *stream)
{
    SDP_CHECK_ARG(u, "NULL handle");
    if (!u->training) return set_error(SDP_ERR_INVALID, "network created without training buffers");
    SDP_CHECK_ARG(lr >= 0.f && beta1 >= 0.f && beta1 < 1.f && beta2 >= 0.f && beta2 < 1.f && eps > 0.f,
                  "invalid Adam hyper-parameters");
    cudaStream_t st = as_stream(stream);
    u->step += 1;
    const float c1 = (float)(1.0 - std::pow((double)beta1, (double)u->step));
    const float c2 = (float)(1.0 - std::pow((double)beta2, (double)u->step));
    k_adam<<<grid_for((long long)u->nparams), 256, 0, st>>>((long long)u->nparams, u->master, u->grad, u->adam_m,
                                                           u->adam_v, lr, beta1, beta2, eps, c1, c2);
    SDP_LAUNCH_CHECK();
    return refresh_weights(u, st);
}

SDP_EXPORT int sdp_blur_mse(int n, int h, int w, const float *pred, const float *target, float *diff_scratch,
                            float *grad, double *loss, void *stream)
{
    SDP_CHECK_ARG(n >= 1 && h >= 1 && w >= 1, "empty images");
    SDP_CHECK_ARG(pred && target && diff_scratch && loss, "NULL argument");
    cudaStream_t st = as_stream(stream);
    const long long np = (long long)n * h * w;
    // diff_scratch holds 2 * np floats: the difference, then its blur
    float *d = diff_scratch, *bd = diff_scratch + np;
    k_diff<<<grid_for(np), 256, 0, st>>>(np, pred, target, d);
    SDP_LAUNCH_CHECK();
    SDP_CUDA_TRY(cudaMemsetAsync(loss, 0, sizeof(double), st));
    k_blur_sq<<<grid_for(np), 256, 0, st>>>(n, h, w, d, bd, loss);
    SDP_LAUNCH_CHECK();
    k_scale_loss<<<1, 1, 0, st>>>(loss, 1.0 / (double)np);
    SDP_LAUNCH_CHECK();
    if (grad) {
        k_blur_grad<<<grid_for(np), 256, 0, st>>>(n, h, w, bd, (float)(2.0 / (double)np), grad);
        SDP_LAUNCH_CHECK();
    }
    return SDP_OK;
}
