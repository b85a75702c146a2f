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
// One minor cycle is one launch (k_clean_cycle): every block applies the
// previous component's PSF subtraction to its rows and reduces (max, index,
// sum) in the same pass over the image; the last block to finish (a
// completion counter) applies the stopping rule and records the component.
// After a stop every later launch returns at once, so a fixed number of
// launches can be captured in a CUDA graph.
#include <cuda/atomic>

#include <algorithm>

#include "internal.cuh"

namespace sdp {

struct CleanState {
    int stop;
    int count;
    int pending;   // a component whose PSF has not been subtracted yet
    int mx, my;
    float val;     // max_val of the pending component
    float first_z; // flux of the first component (the weak-source test, :239)
    unsigned done; // blocks finished in the current minor cycle
};

struct CleanWs {
    CleanState *st;
    float *pmax;
    int *pidx;
    double *psum;
    int nblocks;
};


static int clean_blocks() { return num_sms() * 8; }

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


// Block-wide (max |r|, first index) and sum reduction; result in thread 0.
__device__ __forceinline__ void block_reduce(float &bv, int &bi, double &sum)
{
    __shared__ float sv[32];
    __shared__ int si[32];
    __shared__ double ss[32];
    const int tid = threadIdx.x;
    const int lane = tid & 31, wid = tid >> 5;
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
    }
}

// Stopping rule and component bookkeeping of one minor cycle (:235-256).
__device__ void select_component(int G, int max_records, float curr_max, int idx, double sum,
                                 const float *__restrict__ r, float *__restrict__ model, float3 *__restrict__ src,
                                 double gain, double noise, double weak, double psf_max, CleanState *st)
{
    if (curr_max <= 0.f) {  // all zero (or empty): the reference keeps index 0
        curr_max = 0.f;
        idx = 0;
    }
    const long long n = (long long)G * G;
    const float avg = (n > 1) ? (float)(sum / (double)(n - 1)) : 0.f;
    const bool extracting_noise = (double)fabsf(curr_max) < noise * (double)avg * gain;       // :238
    const bool weak_source = st->count > 0 && (double)fabsf(curr_max) < (double)fabsf(st->first_z) * weak;  // :239
    if (extracting_noise || weak_source) {
        st->stop = 1;
        st->pending = 0;
        return;
    }
    const float max_val = __double2float_rn(__ddiv_rn((double)__ldcg(&r[idx]), psf_max));  // :247
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

// The reference's residual update of one pixel (deconvolution_run.c:271 in
// its types: float residual, double gain x max_val, float PSF, double
// psf_max_value).
__device__ __forceinline__ float hogbom_update(float w, float p, double scale, double psf_max)
{
    return __double2float_rn(__dsub_rn((double)w, __dmul_rn(__dmul_rn(scale, (double)p), psf_max)));
}

// Subtraction of the pending component at pixel (y, x) (:266-272).
__device__ __forceinline__ float clean_pixel(float v, int x, bool row_in, int x0, int x1, long long pbase,
                                             long long g2, const float *__restrict__ psf, double scale,
                                             double psf_max)
{
    if (row_in && x >= x0 && x < x1) {
        const long long pi = pbase - x;  // mirrored in x; index G*G reads 0
        const float pv = (pi < g2) ? __ldg(&psf[pi]) : 0.f;
        v = hogbom_update(v, pv, scale, psf_max);
    }
    return v;
}

constexpr int kCleanThreads = 256;
constexpr int kCleanUnroll = 4;  // independent 4-pixel chunks in flight per thread

// One minor cycle in one launch: every block subtracts the pending
// component's PSF (:263-272, PSF mirrored in x, column G wrapping to the
// next row, psf[G*G] read as 0) from its share of the image, 4 pixels per
// vector load and several loads in flight per thread, and reduces max |r|,
// its first index and the sum of |r| over indices >= 1; the last block to
// finish reduces the block results and applies the stopping rule
// (select = 1).  select = 0 only applies the pending subtraction.
__global__ void __launch_bounds__(kCleanThreads) k_clean_cycle(int G, float *__restrict__ r,
                                                              const float *__restrict__ psf,
                                                              float *__restrict__ model, float3 *__restrict__ src,
                                                              int max_records, double gain, double noise,
                                                              double weak, double psf_max, CleanWs ws, int select)
{
    const CleanState s = *ws.st;
    if (s.stop && !s.pending) return;
    const int half = G / 2;
    const int x0 = s.mx - min(s.mx, half), x1 = s.mx + min(G - s.mx, half);
    const int y0 = s.my - min(s.my, half), y1 = s.my + min(G - s.my, half);
    const long long g2 = (long long)G * G;
    const double scale = __dmul_rn(gain, (double)s.val);
    const bool pending = s.pending != 0;
    float bv = -1.f;
    int bi = 0x7fffffff;
    double sum = 0.0;
    const unsigned ug = (unsigned)G;
    if ((G & 3) == 0) {
        // 4-pixel chunks (a chunk never crosses a row when G % 4 == 0)
        const unsigned nchunks = (unsigned)(g2 >> 2);
        const unsigned stride = gridDim.x * kCleanThreads;
        for (unsigned c0 = blockIdx.x * kCleanThreads + threadIdx.x; c0 < nchunks; c0 += stride * kCleanUnroll) {
            float4 v[kCleanUnroll];
#pragma unroll
            for (int u = 0; u < kCleanUnroll; ++u) {
                const unsigned c = c0 + u * stride;
                v[u] = (c < nchunks) ? reinterpret_cast<const float4 *>(r)[c] : make_float4(0.f, 0.f, 0.f, 0.f);
            }
#pragma unroll
            for (int u = 0; u < kCleanUnroll; ++u) {
                const unsigned c = c0 + u * stride;
                if (c >= nchunks) continue;
                const unsigned i0 = c << 2;
                const int y = (int)(i0 / ug), x = (int)(i0 - (unsigned)y * ug);
                if (pending && y >= y0 && y < y1 && x + 3 >= x0 && x < x1) {
                    const long long pbase = (long long)(y - s.my + half) * G + (G + s.mx - half);
                    v[u].x = clean_pixel(v[u].x, x, true, x0, x1, pbase, g2, psf, scale, psf_max);
                    v[u].y = clean_pixel(v[u].y, x + 1, true, x0, x1, pbase, g2, psf, scale, psf_max);
                    v[u].z = clean_pixel(v[u].z, x + 2, true, x0, x1, pbase, g2, psf, scale, psf_max);
                    v[u].w = clean_pixel(v[u].w, x + 3, true, x0, x1, pbase, g2, psf, scale, psf_max);
                    reinterpret_cast<float4 *>(r)[c] = v[u];
                }
                if (select) {
                    const int i = (int)i0;
                    better(bv, bi, fabsf(v[u].x), i);
                    better(bv, bi, fabsf(v[u].y), i + 1);
                    better(bv, bi, fabsf(v[u].z), i + 2);
                    better(bv, bi, fabsf(v[u].w), i + 3);
                    sum += (double)(i >= 1 ? fabsf(v[u].x) : 0.f) + (double)fabsf(v[u].y) + (double)fabsf(v[u].z) +
                           (double)fabsf(v[u].w);
                }
            }
        }
    } else {
        for (unsigned i = blockIdx.x * kCleanThreads + threadIdx.x; i < (unsigned)g2; i += gridDim.x * kCleanThreads) {
            const int y = (int)(i / ug), x = (int)(i - (unsigned)y * ug);
            float v = r[i];
            if (pending && y >= y0 && y < y1 && x >= x0 && x < x1) {
                const long long pbase = (long long)(y - s.my + half) * G + (G + s.mx - half);
                v = clean_pixel(v, x, true, x0, x1, pbase, g2, psf, scale, psf_max);
                r[i] = v;
            }
            if (select) {
                better(bv, bi, fabsf(v), (int)i);
                if (i >= 1) sum += (double)fabsf(v);
            }
        }
    }
    if (!select) return;
    block_reduce(bv, bi, sum);
    __shared__ bool is_last;
    const int tid = threadIdx.x;
    if (tid == 0) {
        ws.pmax[blockIdx.x] = bv;
        ws.pidx[blockIdx.x] = bi;
        ws.psum[blockIdx.x] = sum;
        __threadfence();
        const unsigned ticket = atomicAdd(&ws.st->done, 1u);
        is_last = (ticket == gridDim.x - 1);
    }
    __syncthreads();
    if (!is_last) return;
    // last block: reduce the per-block results (read past L1) and select
    __threadfence();
    bv = -1.f;
    bi = 0x7fffffff;
    sum = 0.0;
    for (int b = tid; b < (int)gridDim.x; b += kCleanThreads) {
        better(bv, bi, __ldcg(&ws.pmax[b]), __ldcg(&ws.pidx[b]));
        sum += __ldcg(&ws.psum[b]);
    }
    block_reduce(bv, bi, sum);
    if (tid == 0) {
        CleanState *st = ws.st;
        st->done = 0;
        select_component(G, max_records, bv, bi, sum, r, model, src, gain, noise, weak, psf_max, st);
    }
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

// ---------------------------------------------------------------------------
// Persistent variant: the residual stays in shared memory for all minor
// cycles.  Used when the image fits on chip (G^2 floats over all SMs, at
// most kPersistSlice floats per SM, i.e. G <= 2752 on 148 SMs).
//
// One CTA per SM (cooperative launch, so all CTAs are resident), each owning
// a contiguous slice of pixels.  A minor cycle: apply the pending component
// to the slice, reduce (max |r|, first index, signed value, sum |r|) per
// block and publish it with a release-stored flag (results double-buffered
// by cycle parity).  Warp 0 of every block then waits for all blocks' flags
// (acquire loads, no shared counter), reduces the results in the same order
// and takes the same decision, so the blocks stay in step without a second
// barrier.  Block 0 records the component and adds it to the model while
// the next minor cycle runs.  Waits are bounded: after kBarrierSpins polls a
// block sets an error flag, every block stops at its next wait, and the host
// reads SDP_ERR_TIMEOUT.
// ---------------------------------------------------------------------------
// One block's result of a minor cycle: two 64-bit words that each carry the
// minor cycle's tag ((minor cycle + 1) mod 512), so a reader that sees the
// tag in both has both values from one round of loads (no flag, no second
// round trip).  Each word is written and read whole (8-byte relaxed atomics).
//   a: bits 0-22 the first pixel of the slice's max |r| (kNoPixel: empty
//      slice), bits 23-31 the tag, bits 32-63 r there (float bits)
//   b: the sum of |r| over the slice (double; block 0 leaves out pixel 0,
//      which the reference's running mean skips) with its 9 low mantissa
//      bits replaced by the tag
struct PPart {
    unsigned long long a;
    unsigned long long b;
};
constexpr unsigned kTagMask = 511u;
constexpr int kPixelBits = 23;                       // G <= 2752 for the on-chip path: G^2 < 2^23
constexpr unsigned kNoPixel = (1u << kPixelBits) - 1u;

__device__ __forceinline__ unsigned part_tag(int minor) { return (unsigned)(minor + 1) & kTagMask; }

// SUM = false: only word a is written and read (the noise test cannot stop
// the loop, see k_clean_persistent).
template <bool SUM>
__device__ __forceinline__ void part_store(PPart *p, unsigned tag, float val, int idx, double sum)
{
    const unsigned lo = ((unsigned)idx & kNoPixel) | (tag << kPixelBits);
    const unsigned long long a = ((unsigned long long)__float_as_uint(val) << 32) | lo;
    cuda::atomic_ref<unsigned long long, cuda::thread_scope_device>(p->a).store(a, cuda::memory_order_relaxed);
    if constexpr (SUM) {
        const unsigned long long b =
            ((unsigned long long)__double_as_longlong(sum) & ~(unsigned long long)kTagMask) | tag;
        cuda::atomic_ref<unsigned long long, cuda::thread_scope_device>(p->b).store(b, cuda::memory_order_relaxed);
    }
}

// Order key of a candidate (max |r| v >= 0, or v < 0 for none): larger v,
// larger key; none is 0.  Non-negative floats order as their bit patterns.
__device__ __forceinline__ unsigned cand_key(float v) { return v < 0.f ? 0u : __float_as_uint(v) + 1u; }
__device__ __forceinline__ float key_value(unsigned k) { return k == 0u ? -1.f : __uint_as_float(k - 1u); }

// Warp-wide best candidate: the largest key, on ties the smallest pixel
// index (every lane gets the result).
__device__ __forceinline__ void warp_best(unsigned &key, unsigned &idx)
{
    const unsigned kmax = __reduce_max_sync(0xffffffffu, key);
    idx = __reduce_min_sync(0xffffffffu, key == kmax ? idx : 0xffffffffu);
    key = kmax;
}

struct CleanBar {
    int err;
    int pad[15];
};

constexpr int kPersistThreads = 1024;
constexpr int kPersistSlice = 51200;           // floats of residual per block (200 KB)
constexpr int kBatch = 8;                      // pixels per thread whose PSF loads are in flight together
constexpr long long kBarrierSpins = 4000000;   // polling rounds of ~32 ns sleep + an L2 read: one to two seconds


// Waits (one warp) until the results of blocks 0..nb-1 in buf carry `tag`,
// then folds lane l's blocks l, l + 32, ... into (bv, bi, bs, sum) in block
// order.  Each polling round issues all of a lane's loads at once (a round
// costs one L2 round trip).  Bounded: after spin_limit rounds, or once
// another block has timed out, it sets bar->err and returns false.
// nb <= 32 * kWaitPerLane.  Not inlined: its registers stay out of the
// pixel pass of the kernel that calls it.
constexpr int kWaitPerLane = 5;  // 160 blocks: one per SM of a 148-SM part

struct PBest {
    float bv;    // max |r| (-1: none)
    int bi;      // its first pixel
    float bs;    // r there
    int ok;      // 0: the wait gave up
    double sum;  // sum of |r| (SUM)
};

template <bool SUM>
__device__ __noinline__ PBest wait_results(PPart *buf, int nb, unsigned tag, CleanBar *bar, long long spin_limit)
{
    cuda::atomic_ref<int, cuda::thread_scope_device> err(bar->err);
    const int lane = (int)(threadIdx.x & 31);
    unsigned long long a[kWaitPerLane], b[kWaitPerLane];
    int fail = 0;
    for (long long spins = 0;;) {
        bool ready = true;
#pragma unroll
        for (int j = 0; j < kWaitPerLane; ++j) {
            const int k = lane + 32 * j;
            if (k < nb) {
                a[j] = cuda::atomic_ref<unsigned long long, cuda::thread_scope_device>(buf[k].a).load(
                    cuda::memory_order_relaxed);
                ready &= (((unsigned)a[j] >> kPixelBits) & kTagMask) == tag;
                if constexpr (SUM) {
                    b[j] = cuda::atomic_ref<unsigned long long, cuda::thread_scope_device>(buf[k].b).load(
                        cuda::memory_order_relaxed);
                    ready &= ((unsigned)b[j] & kTagMask) == tag;
                }
            }
        }
        if (ready) break;
        if (err.load(cuda::memory_order_relaxed) != 0 || ++spins > spin_limit) {
            err.store(1, cuda::memory_order_relaxed);
            fail = 1;
            break;
        }
        __nanosleep(32);
    }
    // this lane's blocks in block order, then the warp
    unsigned key = 0u, idx = 0xffffffffu;
    float val = 0.f;
    double sum = 0.0;
    if (!fail) {
#pragma unroll
        for (int j = 0; j < kWaitPerLane; ++j)
            if (lane + 32 * j < nb) {
                const unsigned pix = (unsigned)a[j] & kNoPixel;
                const float v = __uint_as_float((unsigned)(a[j] >> 32));
                const unsigned k = pix == kNoPixel ? 0u : cand_key(fabsf(v));
                if (k > key || (k == key && k != 0u && pix < idx)) {
                    key = k;
                    idx = pix;
                    val = v;
                }
                if constexpr (SUM) sum += __longlong_as_double((long long)(b[j] & ~(unsigned long long)kTagMask));
            }
    }
    const unsigned key0 = key, idx0 = idx;
    warp_best(key, idx);
    const unsigned win = __ballot_sync(0xffffffffu, key0 == key && idx0 == idx);
    val = __shfl_sync(0xffffffffu, val, win ? __ffs(win) - 1 : 0);
    if constexpr (SUM) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) sum += __shfl_xor_sync(0xffffffffu, sum, o);
    }
    PBest r;
    r.bv = key_value(key);
    r.bi = (int)idx;
    r.bs = val;
    r.sum = sum;
    r.ok = !__any_sync(0xffffffffu, fail);
    return r;
}

// Block-wide best candidate (bv, bi) and, with SUM, the sum; the result is
// in warp 0 (all lanes).
template <bool SUM>
__device__ __forceinline__ void block_best(float &bv, int &bi, double &sum)
{
    __shared__ unsigned s_key[32], s_idx[32];
    __shared__ double s_sum[32];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    unsigned key = cand_key(bv), idx = (unsigned)bi;
    warp_best(key, idx);
    if constexpr (SUM) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) sum += __shfl_xor_sync(0xffffffffu, sum, o);
    }
    if (lane == 0) {
        s_key[wid] = key;
        s_idx[wid] = idx;
        if constexpr (SUM) s_sum[wid] = sum;
    }
    __syncthreads();
    if (wid == 0) {
        const int nw = blockDim.x / 32;
        key = lane < nw ? s_key[lane] : 0u;
        idx = lane < nw ? s_idx[lane] : 0xffffffffu;
        warp_best(key, idx);
        bv = key_value(key);
        bi = (int)idx;
        if constexpr (SUM) {
            sum = lane < nw ? s_sum[lane] : 0.0;
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) sum += __shfl_xor_sync(0xffffffffu, sum, o);
        }
    }
    // no barrier here: only warp 0 goes on with the result, and the next
    // call's writes to the arrays above come after the caller's next barrier
}

__device__ __forceinline__ void cp_async4(float *dst_smem, const float *src)
{
    const unsigned d = (unsigned)__cvta_generic_to_shared(dst_smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(d), "l"(src) : "memory");
}

// Pass variants of the persistent kernel (one per instantiation, chosen by
// the host):
//   kPassStage  the PSF samples of a minor cycle are first copied into a
//               second shared-memory slice with asynchronous copies (all of
//               a thread's copies in flight at once, one wait), then read
//               from there; small slices (at most two pixels per thread,
//               G <= ~550 on 148 SMs)
//   kPassScalar one pixel per thread and step, eight PSF loads in flight
//   kPassQuad   four adjacent pixels per thread and step (G and the slice
//               length multiples of 4)
enum : int { kPassStage = 0, kPassScalar = 1, kPassQuad = 2 };

template <int MODE, bool SUM>
__global__ void __launch_bounds__(kPersistThreads, 1) k_clean_persistent(
    int G, float *__restrict__ r, const float *__restrict__ psf, float *__restrict__ model,
    float3 *__restrict__ src, int *__restrict__ count_out, int max_records, int num_minor, double gain,
    double noise, double weak, double psf_max, double cell, PPart *__restrict__ parts, CleanBar *bar, int P,
    long long spin_limit)
{
    extern __shared__ __align__(16) float sr[];
    __shared__ int s_pending, s_mx, s_my, s_stop, s_fail;
    __shared__ float s_val;
    const int tid = threadIdx.x;
    const int nb = (int)gridDim.x;
    const int g2 = G * G;  // the persistent path holds G <= 2752 images
    const int p0 = blockIdx.x * P;
    const int n = max(0, min(p0 + P, g2) - p0);
    for (int k = tid; k < n; k += kPersistThreads) sr[k] = r[p0 + k];
    if (tid == 0) {
        s_pending = 0;
        s_stop = 0;
        s_fail = 0;
        s_mx = 0;
        s_my = 0;
        s_val = 0.f;
    }
    __syncthreads();
    int count = 0;
    float first_z = 0.f;
    int model_idx = -1;  // block 0, thread 0: component not yet added to the model
    double model_add = 0.0;
    const int half = G / 2;
    const int step_y = kPersistThreads / G, step_x = kPersistThreads - (kPersistThreads / G) * G;
    // quads: G and the slice start are multiples of 4, so a quad never
    // crosses a row
    constexpr bool STAGE = MODE == kPassStage;
    const int step_y4 = 4 * kPersistThreads / G, step_x4 = 4 * kPersistThreads - step_y4 * G;
    for (int it = 0; it <= num_minor; ++it) {
        const bool apply_only = (it == num_minor);
        const int pending = s_pending, mx = s_mx, my = s_my;
        const double scale = __dmul_rn(gain, (double)s_val);
        const int x0 = mx - min(mx, half), wx = min(mx, half) + min(G - mx, half);
        const int y0 = my - min(my, half), wy = min(my, half) + min(G - my, half);
        // PSF sample of pixel (y, x): psf[(y - my + G/2) G + (G - (x - mx + G/2))]
        // (x-mirrored; column G runs into the next PSF row, and past the
        // last row reads as 0), i.e. psf[y G - x + pofs]
        const int pofs = (half - my) * G + G + mx - half;
        float bv = -1.f, bs = 0.f;
        int bi = 0x7fffffff;
        // pixel k = tid + m * 1024 of the slice, (y, x) advanced
        // incrementally; kBatch pixels at a time, their PSF loads issued
        // together so the L2 latency is paid once per batch
        int y = (p0 + tid) / G, x = (p0 + tid) - y * G;
        float rsum = 0.f;
        if constexpr (STAGE) {
            float *ps = sr + P;
            const int ys = y, xs = x;
            for (int k = tid; k < n; k += kPersistThreads) {
                const bool in = pending && (unsigned)(y - y0) < (unsigned)wy && (unsigned)(x - x0) < (unsigned)wx;
                const int pi = y * G - x + pofs;
                if (in && pi < g2) {
                    cp_async4(ps + k, psf + pi);
                } else {
                    ps[k] = 0.f;
                }
                x += step_x;
                y += step_y;
                if (x >= G) {
                    x -= G;
                    y += 1;
                }
            }
            asm volatile("cp.async.commit_group;\n\tcp.async.wait_group 0;" ::: "memory");
            y = ys;
            x = xs;
            for (int k = tid; k < n; k += kPersistThreads) {
                float wv = sr[k];
                if (pending && (unsigned)(y - y0) < (unsigned)wy && (unsigned)(x - x0) < (unsigned)wx) {
                    wv = hogbom_update(wv, ps[k], scale, psf_max);
                    sr[k] = wv;
                }
                const float a = fabsf(wv);
                if (a > bv) {  // pixels visited in increasing index: the first maximum wins
                    bv = a;
                    bi = y * G + x;
                    bs = wv;
                }
                if constexpr (SUM) rsum += a;
                x += step_x;
                y += step_y;
                if (x >= G) {
                    x -= G;
                    y += 1;
                }
            }
        }
        if constexpr (MODE == kPassQuad) {
            // four adjacent pixels of one row per thread and step (one
            // 16-byte shared access; window rows and PSF offsets once per
            // quad): quad q = tid + m * 1024 is pixels p0 + 4 q .. + 3, two
            // quads' PSF loads in flight together
            // the argmax keeps the first quad holding the thread's max |r|
            // (bq); its first pixel with that |r| is read back afterwards
            float4 *sr4 = reinterpret_cast<float4 *>(sr);
            const int nq = n >> 2;
            int qy = (p0 + 4 * tid) / G, qx = (p0 + 4 * tid) - qy * G;
            int bq = 0;
            for (int qb = tid; qb < nq; qb += 2 * kPersistThreads) {
                float4 w4[2];
                float pv[2][4];
                bool in[2][4];
#pragma unroll
                for (int u = 0; u < 2; ++u) {
                    const int q = qb + u * kPersistThreads;
                    const bool live = q < nq;
                    w4[u] = live ? sr4[q] : make_float4(0.f, 0.f, 0.f, 0.f);
                    const bool iny = live && pending && (unsigned)(qy - y0) < (unsigned)wy;
                    const int ux = qx - x0;
                    const int pi = qy * G - qx + pofs;  // PSF index of the quad's pixel 0; pixel j: pi - j
#pragma unroll
                    for (int j = 0; j < 4; ++j) {
                        in[u][j] = iny && (unsigned)(ux + j) < (unsigned)wx && pi - j < g2;
                        pv[u][j] = in[u][j] ? __ldg(&psf[pi - j]) : 0.f;
                    }
                    qx += step_x4;
                    qy += step_y4;
                    if (qx >= G) {
                        qx -= G;
                        qy += 1;
                    }
                }
#pragma unroll
                for (int u = 0; u < 2; ++u) {
                    const int q = qb + u * kPersistThreads;
                    float wv[4] = {w4[u].x, w4[u].y, w4[u].z, w4[u].w};
#pragma unroll
                    for (int j = 0; j < 4; ++j)
                        if (in[u][j])
                            wv[j] = hogbom_update(wv[j], pv[u][j], scale, psf_max);
                    if (in[u][0] || in[u][1] || in[u][2] || in[u][3])
                        sr4[q] = make_float4(wv[0], wv[1], wv[2], wv[3]);
                    const float a0 = fabsf(wv[0]), a1 = fabsf(wv[1]), a2 = fabsf(wv[2]), a3 = fabsf(wv[3]);
                    const float qm = fmaxf(fmaxf(a0, a1), fmaxf(a2, a3));
                    if (q < nq && qm > bv) {  // quads visited in increasing index: the first maximum wins
                        bv = qm;
                        bq = q;
                    }
                    if constexpr (SUM) {
                        rsum += a0;  // 0 for the padding past the slice
                        rsum += a1;
                        rsum += a2;
                        rsum += a3;
                    }
                }
            }
            if (bv >= 0.f) {  // the first pixel of the best quad with |r| = bv
                const float4 wq = sr4[bq];
                int j = 3;
                if (fabsf(wq.z) == bv) j = 2;
                if (fabsf(wq.y) == bv) j = 1;
                if (fabsf(wq.x) == bv) j = 0;
                bi = p0 + 4 * bq + j;
            }
        }
        for (int kb = tid; MODE == kPassScalar && kb < n; kb += kBatch * kPersistThreads) {
            float w[kBatch], pv[kBatch];
            int ii[kBatch];
            bool in[kBatch];
#pragma unroll
            for (int u = 0; u < kBatch; ++u) {
                const int k = kb + u * kPersistThreads;
                const bool live = k < n;
                ii[u] = y * G + x;
                w[u] = live ? sr[k] : 0.f;
                in[u] = live && pending && (unsigned)(y - y0) < (unsigned)wy && (unsigned)(x - x0) < (unsigned)wx;
                const int pi = ii[u] - 2 * x + pofs;
                pv[u] = (in[u] && pi < g2) ? __ldg(&psf[pi]) : 0.f;
                x += step_x;
                y += step_y;
                if (x >= G) {
                    x -= G;
                    y += 1;
                }
            }
#pragma unroll
            for (int u = 0; u < kBatch; ++u) {
                float wv = w[u];
                if (in[u]) {
                    wv = hogbom_update(wv, pv[u], scale, psf_max);
                    sr[kb + u * kPersistThreads] = wv;
                }
                const float a = fabsf(wv);
                if (a > bv) {  // pixels visited in increasing index: the first maximum wins
                    bv = a;
                    bi = ii[u];
                    bs = wv;
                }
                if constexpr (SUM) rsum += a;  // 0 for the padding past the slice
            }
        }
        if (apply_only) break;
        double sum = (double)rsum;
        block_best<SUM>(bv, bi, sum);
        PPart *buf = parts + (size_t)(it & 1) * nb;
        const unsigned tag = part_tag(it);
        if (tid == 0) {
            // block 0 leaves out pixel 0 (the reference's running mean skips it)
            if (SUM && blockIdx.x == 0 && n > 0) sum = __dsub_rn(sum, (double)fabsf(sr[0]));
            part_store<SUM>(buf + blockIdx.x, tag, bv < 0.f ? 0.f : sr[bi - p0], bv < 0.f ? (int)kNoPixel : bi, sum);
            // block 0 adds the previous component to the model here, off the
            // critical path (model updates keep the reference's order)
            if (model_idx >= 0) {
                model[model_idx] = __double2float_rn(__dadd_rn((double)model[model_idx], model_add));
                model_idx = -1;
            }
        }
        // warp 0 of every block waits for every block's result of this
        // minor cycle, reduces them in the same order and takes the same
        // decision
        if (tid < 32) {
            const PBest w = wait_results<SUM>(buf, nb, tag, bar, spin_limit);
            const int fail = w.ok ? 0 : 1;
            bv = w.bv;
            bi = w.bi;
            bs = w.bs;
            sum = w.sum;
            if (tid == 0) {
                if (fail) {
                    s_fail = 1;
                    s_stop = 1;
                    s_pending = 0;
                } else {
                    float curr_max = bv;
                    int idx = bi;
                    float sval = bs;
                    if (curr_max <= 0.f) {  // all zero (or empty): the reference keeps index 0
                        curr_max = 0.f;
                        idx = 0;
                        sval = 0.f;
                    }
                    // :238; without SUM (noise x gain < 0.5) it cannot hold: the mean of
                    // |r| is at most the max
                    const float avg = (SUM && g2 > 1) ? (float)(sum / (double)(g2 - 1)) : 0.f;
                    const bool extracting_noise = SUM && (double)fabsf(curr_max) < noise * (double)avg * gain;
                    const bool weak_source =
                        count > 0 && (double)fabsf(curr_max) < (double)fabsf(first_z) * weak;  // :239
                    if (extracting_noise || weak_source) {
                        s_stop = 1;
                        s_pending = 0;
                    } else {
                        const float max_val = __double2float_rn(__ddiv_rn((double)sval, psf_max));  // :247
                        const float z = __double2float_rn(__dmul_rn((double)max_val, gain));
                        if (count == 0) first_z = z;
                        if (blockIdx.x == 0) {
                            if (count < max_records) src[count] = make_float3((float)(idx % G), (float)(idx / G), z);
                            model_idx = idx;  // :256, added after the next publish
                            model_add = __dmul_rn((double)max_val, gain);
                        }
                        count += 1;
                        s_pending = 1;
                        s_mx = idx % G;
                        s_my = idx / G;
                        s_val = max_val;
                    }
                }
            }
        }
        __syncthreads();
        if (s_stop) break;
    }
    __syncthreads();
    for (int k = tid; k < n; k += kPersistThreads) r[p0 + k] = sr[k];
    if (model_idx >= 0) model[model_idx] = __double2float_rn(__dadd_rn((double)model[model_idx], model_add));
    if (blockIdx.x == 0 && tid == 0) {
        const int nrec = min(count, max_records);
        for (int k = 0; k < nrec; ++k) {  // :297-306
            float3 q = src[k];
            q.x = __double2float_rn(__dmul_rn((double)__fsub_rn(q.x, (float)(G / 2)), cell));
            q.y = __double2float_rn(__dmul_rn((double)__fsub_rn(q.y, (float)(G / 2)), cell));
            src[k] = q;
        }
        if (count_out) *count_out = s_fail ? -1 : nrec;
    }
}

// Bounded-wait self test: every block publishes its result and waits for
// one more block than there are.  Each gives up after spin_limit polls and
// the kernel ends with the error flag set (the host reads SDP_ERR_TIMEOUT).
__global__ void k_wait_timeout_probe(PPart *parts, CleanBar *bar, long long spin_limit)
{
    if (threadIdx.x == 0) part_store<true>(parts + blockIdx.x, part_tag(0), 1.f, (int)blockIdx.x, 1.0);
    if (threadIdx.x < 32) wait_results<true>(parts, (int)gridDim.x + 1, part_tag(0), bar, spin_limit);
}

static void persist_layout(int nb, size_t base, size_t *bar_off, size_t *parts_off, size_t *total)
{
    *bar_off = base;
    *parts_off = base + 64;
    *total = *parts_off + sizeof(PPart) * 2 * (size_t)nb;
}

static int persistent_fits(int G, int *nb_out)
{
    const int nb = num_sms();
    const long long P = (((long long)G * G + nb - 1) / nb + 3) / 4 * 4;
    *nb_out = nb;
    return P <= kPersistSlice;
}

}  // namespace sdp

using namespace sdp;

SDP_EXPORT int sdp_hogbom_workspace_bytes(int G, size_t *bytes)
{
    SDP_CHECK_ARG(bytes != nullptr && G >= 2, "bad argument");
    size_t off[4], base, bar, parts, total;
    clean_layout(clean_blocks(), off, &base);
    persist_layout(num_sms(), base, &bar, &parts, &total);
    *bytes = total;
    return SDP_OK;
}

SDP_EXPORT int sdp_hogbom(const sdp_clean_params *p, float *residual, const float *psf, float *model,
                          sdp_float3 *sources, int *num_sources_dev, void *workspace, size_t ws_bytes, void *stream)
{
    return hogbom_launch(p, residual, psf, model, sources, num_sources_dev, workspace, ws_bytes, true,
                         as_stream(stream));
}

int sdp::hogbom_launch(const sdp_clean_params *p, float *residual, const float *psf, float *model,
                       sdp_float3 *sources, int *num_sources_dev, void *workspace, size_t ws_bytes,
                       bool allow_persistent, cudaStream_t st)
{
    SDP_CHECK_ARG(p && residual && psf && model && workspace, "NULL argument");
    SDP_CHECK_ARG(p->grid_size >= 2, "grid_size %d", p->grid_size);
    SDP_CHECK_ARG(p->num_minor_cycles >= 0, "num_minor_cycles %d", p->num_minor_cycles);
    SDP_CHECK_ARG(p->num_minor_cycles == 0 || sources, "sources is NULL");
    SDP_CHECK_ARG(p->psf_max_value != 0.0, "psf_max_value is 0");
    const int G = p->grid_size;
    size_t need = 0;
    SDP_TRY(sdp_hogbom_workspace_bytes(G, &need));
    if (ws_bytes < need) return set_error(SDP_ERR_RANGE, "hogbom workspace %zu B < %zu B", ws_bytes, need);
    char *w = static_cast<char *>(workspace);
    // the stored component list is bounded by the caller's buffer (MAX_SOURCES)
    const int cap = std::max(0, std::min(p->num_minor_cycles, p->max_sources));
    float3 *src = reinterpret_cast<float3 *>(sources);

    int pnb = 0;
    if (allow_persistent && persistent_fits(G, &pnb) && pnb <= 32 * kWaitPerLane) {
        size_t off[4], base, bar_off, parts_off, total;
        clean_layout(clean_blocks(), off, &base);
        persist_layout(pnb, base, &bar_off, &parts_off, &total);
        CleanBar *bar = reinterpret_cast<CleanBar *>(w + bar_off);
        PPart *parts = reinterpret_cast<PPart *>(w + parts_off);
        const int P = (int)((((long long)G * G + pnb - 1) / pnb + 3) / 4 * 4);
        int dev = 0, optin = 0;
        SDP_CUDA_TRY(cudaGetDevice(&dev));
        SDP_CUDA_TRY(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
        // staging pays when a thread has few pixels (measured: 512^2 gains
        // 13 %, 1024^2 and 2048^2 lose 5-10 % to the extra pass)
        const bool stage = P <= 2 * kPersistThreads &&
                           2 * sizeof(float) * (size_t)P + 2048 <= (size_t)optin;  // 2 KB: the static arrays
        const size_t smem = sizeof(float) * (size_t)P * (stage ? 2 : 1);
        const bool quad = (G & 3) == 0 && (P & 3) == 0;
        // the noise test (|max| < noise x mean |r| x gain) cannot stop the
        // loop when noise x gain < 0.5, since the mean of |r| is at most its
        // max: the kernel then skips the sum of |r|
        const bool sum = !(p->noise_factor * p->loop_gain < 0.5);
        auto fn = stage  ? (sum ? k_clean_persistent<kPassStage, true> : k_clean_persistent<kPassStage, false>)
                  : quad ? (sum ? k_clean_persistent<kPassQuad, true> : k_clean_persistent<kPassQuad, false>)
                         : (sum ? k_clean_persistent<kPassScalar, true> : k_clean_persistent<kPassScalar, false>);
        SDP_CUDA_TRY(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        int per_sm = 0;
        SDP_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, kPersistThreads, smem));
        if (per_sm >= 1) {
            SDP_CUDA_TRY(cudaMemsetAsync(bar, 0, sizeof(CleanBar), st));
            SDP_CUDA_TRY(cudaMemsetAsync(parts, 0, sizeof(PPart) * 2 * (size_t)pnb, st));
            int Gv = G, nminor = p->num_minor_cycles, maxr = cap;
            double gain = p->loop_gain, noise = p->noise_factor, weak = p->weak_source_percent,
                   pmax = p->psf_max_value, cell = p->cell_size;
            int *cnt = num_sources_dev;
            int Pv = P;
            long long spins = kBarrierSpins;
            void *args[] = {&Gv, &residual, (void *)&psf, &model, &src, &cnt, &maxr, &nminor, &gain, &noise,
                            &weak, &pmax, &cell, &parts, &bar, &Pv, &spins};
            SDP_CUDA_TRY(cudaLaunchCooperativeKernel((const void *)fn, dim3(pnb), dim3(kPersistThreads), args, smem,
                                                     st));
            return SDP_OK;
        }
    }

    // general path: one launch per minor cycle
    const int nb = std::max(1, std::min((int)(((long long)G * G / 4 + kCleanThreads - 1) / kCleanThreads),
                                        clean_blocks()));
    size_t off[4], base;
    clean_layout(nb, off, &base);
    CleanWs ws;
    ws.st = reinterpret_cast<CleanState *>(w + off[0]);
    ws.psum = reinterpret_cast<double *>(w + off[1]);
    ws.pmax = reinterpret_cast<float *>(w + off[2]);
    ws.pidx = reinterpret_cast<int *>(w + off[3]);
    ws.nblocks = nb;
    SDP_CUDA_TRY(cudaMemsetAsync(ws.st, 0, sizeof(CleanState), st));
    const dim3 block(kCleanThreads);
    for (int it = 0; it < p->num_minor_cycles; ++it)
        k_clean_cycle<<<nb, block, 0, st>>>(G, residual, psf, model, src, cap, p->loop_gain, p->noise_factor,
                                            p->weak_source_percent, p->psf_max_value, ws, 1);
    // subtract the last component so residual_inout is the final residual
    k_clean_cycle<<<nb, block, 0, st>>>(G, residual, psf, model, src, cap, p->loop_gain, p->noise_factor,
                                        p->weak_source_percent, p->psf_max_value, ws, 0);
    k_clean_finish<<<1, 256, 0, st>>>(G, p->cell_size, cap, src, ws, num_sources_dev);
    SDP_LAUNCH_CHECK();
    return SDP_OK;
}

SDP_EXPORT int sdp_selftest_bounded_wait(int nblocks, long long spin_limit, int *status)
{
    SDP_CHECK_ARG(status != nullptr && nblocks >= 1 && nblocks <= 64 && spin_limit >= 1, "bad argument");
    *status = SDP_OK;
    // one allocation: the error flag, then nblocks + 1 result slots
    const size_t bytes = 64 + sizeof(PPart) * ((size_t)nblocks + 1);
    char *mem = nullptr;
    SDP_CUDA_TRY(cudaMalloc(&mem, bytes));
    CleanBar *bar = reinterpret_cast<CleanBar *>(mem);
    PPart *parts = reinterpret_cast<PPart *>(mem + 64);
    int err = 0;
    cudaError_t e = cudaMemset(mem, 0, bytes);
    if (e == cudaSuccess) {
        k_wait_timeout_probe<<<nblocks, 32>>>(parts, bar, spin_limit);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaDeviceSynchronize();
    if (e == cudaSuccess) e = cudaMemcpy(&err, &bar->err, sizeof(int), cudaMemcpyDeviceToHost);
    cudaFree(mem);
    if (e != cudaSuccess) return cuda_error(e, "bounded-wait self test");
    *status = err ? SDP_ERR_TIMEOUT : SDP_OK;
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
#include <cuda.h>

#include <mutex>

namespace sdp {

constexpr int kNoAllocMaxGrid = 4096;  // grid_size limit of sdp_hogbom_noalloc
constexpr size_t kNoAllocStateBytes = 256;
// state + one (double sum, float max, int index) partial per image row
constexpr size_t kNoAllocScratchBytes = kNoAllocStateBytes + 16 * (size_t)kNoAllocMaxGrid;  // 65,792 B

static_assert(sizeof(CleanState) <= kNoAllocStateBytes, "CLEAN state must fit its slot");

static __device__ __align__(256) unsigned char g_clean_scratch[kNoAllocScratchBytes];

// The array's device address belongs to the context the module was loaded
// into.  It is cached per device together with that context's unique id
// (cuCtxGetId), so a context made again after cudaDeviceReset (or after the
// primary context was released) gets a fresh lookup instead of the old,
// dangling address.
struct ScratchSlot {
    unsigned long long ctx_id = 0;
    void *addr = nullptr;
};
static std::mutex g_clean_scratch_mutex;
static ScratchSlot g_clean_scratch_slot[128];

typedef CUresult (*CtxGetCurrentFn)(CUcontext *);
typedef CUresult (*CtxGetIdFn)(CUcontext, unsigned long long *);

// Unique id of the current context; *id = 0 when no context is current yet
// (a thread whose first runtime call this is).
static int current_context_id(unsigned long long *id)
{
    *id = 0;
    static CtxGetCurrentFn get_current = nullptr;
    static CtxGetIdFn get_id = nullptr;
    if (!get_current || !get_id) {
        void *f1 = nullptr, *f2 = nullptr;
        cudaDriverEntryPointQueryResult q1, q2;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f1, cudaEnableDefault, &q1) != cudaSuccess ||
            q1 != cudaDriverEntryPointSuccess ||
            cudaGetDriverEntryPoint("cuCtxGetId", &f2, cudaEnableDefault, &q2) != cudaSuccess ||
            q2 != cudaDriverEntryPointSuccess)
            return set_error(SDP_ERR_CUDA, "cuCtxGetCurrent / cuCtxGetId unavailable");
        get_current = reinterpret_cast<CtxGetCurrentFn>(f1);
        get_id = reinterpret_cast<CtxGetIdFn>(f2);
    }
    CUcontext ctx = nullptr;
    if (get_current(&ctx) != CUDA_SUCCESS) return set_error(SDP_ERR_CUDA, "cuCtxGetCurrent failed");
    if (ctx == nullptr) return SDP_OK;
    if (get_id(ctx, id) != CUDA_SUCCESS) return set_error(SDP_ERR_CUDA, "cuCtxGetId failed");
    return SDP_OK;
}

// Device address of g_clean_scratch in the current device's context, looked
// up on the first call in each context (the host-side name of the array is
// not a device address).
static int clean_scratch_address(void **out)
{
    int dev = 0;
    SDP_CUDA_TRY(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 128) return set_error(SDP_ERR_RANGE, "device ordinal %d beyond 127", dev);
    std::lock_guard<std::mutex> lock(g_clean_scratch_mutex);
    unsigned long long id = 0;
    SDP_TRY(current_context_id(&id));
    ScratchSlot &s = g_clean_scratch_slot[dev];
    if (id == 0 || s.addr == nullptr || s.ctx_id != id) {
        // the lookup also makes the device's primary context current when
        // this thread had none; the id is read again afterwards
        void *p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_clean_scratch);
        if (e != cudaSuccess) return cuda_error(e, "cudaGetSymbolAddress(g_clean_scratch)");
        SDP_TRY(current_context_id(&id));
        if (id == 0) return set_error(SDP_ERR_CUDA, "no current CUDA context after the symbol lookup");
        s.addr = p;
        s.ctx_id = id;
    }
    *out = s.addr;
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
    // blocks: at most one per 1024 pixels, hence <= G / 4 <= kNoAllocMaxGrid partials
    const int nb = std::max(1, std::min((int)(((long long)G * G / 4 + kCleanThreads - 1) / kCleanThreads),
                                        std::min(clean_blocks(), G)));
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
    const dim3 block(kCleanThreads);
    for (int it = 0; it < p->num_minor_cycles; ++it)
        k_clean_cycle<<<nb, block, 0, st>>>(G, residual, psf, model, src, cap, p->loop_gain, p->noise_factor,
                                            p->weak_source_percent, p->psf_max_value, ws, 1);
    k_clean_cycle<<<nb, block, 0, st>>>(G, residual, psf, model, src, cap, p->loop_gain, p->noise_factor,
                                        p->weak_source_percent, p->psf_max_value, ws, 0);
    k_clean_finish<<<1, 256, 0, st>>>(G, p->cell_size, cap, src, ws, num_sources_dev);
    SDP_LAUNCH_CHECK();
    return SDP_OK;
}
