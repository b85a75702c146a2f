// Visibility-side kernels: binning by uv tile, W-projection gridding and
// degridding, and the fused degrid -> subtract -> grid pass of a major cycle.
//
// Reference behaviour (param_code/code_fft_1core/src/CPU/degridgrid.c):
//   std_gridding   :69-125   taps [ceil(p-hs), ceil(p+hs)), kernel sample
//                            kernels[off + |round((v-p_y)OS)|(hs+1)OS + |round((u-p_x)OS)|],
//                            imaginary part negated for w < 0, taps outside
//                            [-G/2, G/2) skipped.
//   std_degridding :127-202  same taps with the edges mirrored, normalised by
//                            sqrt(sum |k|^2), then replaced by the nearest cell.
//   g2g_degridgrid :204-326  nearest cell, regridded with the w = 0 kernel.
//   gridding_CPU (gridding_run.c:55-137): snapped p, taps [ceil(p-hs), floor(p+hs)].
//
// B200 design.  A plan bins the visibilities once per uvw set: a counting
// sort by (uv tile of the tap-box origin, w-plane) gives the bins, a radix
// sort orders each tile's visibilities by (origin, plane), and each tile's
// list is cut into work items; persistent CTAs pull items from an atomic
// queue.  The warp-per-visibility kernels (k_vis_fast*, half supports up to
// 4) stage an item's records in shared memory with bulk copies, give every
// warp a private subgrid (plain read-modify-writes; lane (r, c) owns tap
// column c, rows r and r + 4) and flush the warps' sum with one vector
// atomic per touched cell; batches of four half-support-4 visibilities read
// one 16-byte quad record each (table bases, origin, normalisation index)
// and reuse model reads and subgrid updates along runs of one origin.  The
// group kernels (k_tiles*, several visibilities per warp on one shared
// subgrid) serve the other plans: snapped coordinates, g2g, nearest-cell
// cycles and half supports above 4.
#include <cstdio>
#include <cstring>

#include <algorithm>
#include <vector>

#include <cub/device/device_radix_sort.cuh>

#include "internal.cuh"

namespace sdp {

// Order of the visibilities inside a uv tile: by w-plane, then by tap-box
// origin (0), or by origin, then by plane (1, the default: longer runs of
// one origin, which the warp-per-visibility kernels exploit).
#ifndef SDP_SORT_CELL_MAJOR
#define SDP_SORT_CELL_MAJOR 1
#endif

constexpr int kTile = 16;    // default uv tile side
constexpr int kChunk = 512;   // default visibilities per work item
constexpr int kMaxHalfSupport = 15;

enum : int {
    OP_GRID = 0,         // grid vis (original order) into grid
    OP_DEGRID = 1,       // convolutional degrid into predicted
    OP_CYCLE_CONV = 2,   // degrid (conv) -> subtract -> grid
    OP_CYCLE_NEAR = 3,   // degrid (nearest) -> subtract -> grid
    OP_G2G = 4           // nearest sample of in_grid regridded (w = 0 plane)
};

// Device-side error flags (OR-ed together).
enum : int { FLAG_PLANE = 1, FLAG_SUPPORT = 2, FLAG_BOX = 4, FLAG_STAGE = 8 };

struct PlanDev {
    int G, gc, OS, nk_g, nk_d, ntx, nty, W, S, tile;
    int phase_major, os_mask, os_shift;
    double uv_scale, w_scale;
    const float2 *gk;   // gridding kernels (phase-major copy when phase_major)
    const int2 *gs;     // gridding supports (hs used; offsets superseded by gpoff)
    const int *gpoff;   // gridding plane offsets into gk
    const float2 *dk;   // degridding kernels
    const int2 *ds;     // degridding supports
    const int *dpoff;   // degridding plane offsets into dk
    const void *rec;    // plan order, Rec<float> or Rec<double>
    const int4 *items;  // (tile, begin, end, -)
    const int *n_items;
    int *item_counter;
    int *flags;
    const int *kdiff;  // bit 0: degridding set != gridding set; bit 1: != its conjugate
    int pitch;          // row pitch (float2) of the shared tiles of the warp-per-visibility kernels
    int chunk;          // visibilities per work item (at most)
    const uint4 *geo;   // packed tap-box geometry in plan order (see fast_geometry)
    const int *perm;    // plan position -> original visibility index
    const float *dinv;  // degridding normalisation of each fast-path tap box (nullptr: none), see k_dinv
    const uint4 *gbase; // quad records of the fast visibilities in plan order (k_gather_plan; nullptr: none)
};

// ----------------------------------------------------------------------------
// Generic exclusive scan (int), out has n + 1 entries (out[n] = total).
// ----------------------------------------------------------------------------
constexpr int kScanThreads = 1024;
constexpr int kScanPer = 4;
constexpr int kScanBlock = kScanThreads * kScanPer;

__global__ void k_scan_blocks(const int *in, int *out, int *block_sums, int n)
{
    __shared__ int warp_sums[32];
    int base = blockIdx.x * kScanBlock + threadIdx.x * kScanPer;
    int v[kScanPer];
    int local = 0;
#pragma unroll
    for (int k = 0; k < kScanPer; ++k) {
        int i = base + k;
        v[k] = (i < n) ? in[i] : 0;
        local += v[k];
    }
    int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    int incl = local;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        int t = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += t;
    }
    if (lane == 31) warp_sums[wid] = incl;
    __syncthreads();
    if (wid == 0) {
        int s = (lane < (kScanThreads / 32)) ? warp_sums[lane] : 0;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            int t = __shfl_up_sync(0xffffffffu, s, o);
            if (lane >= o) s += t;
        }
        warp_sums[lane] = s;  // inclusive over warps
    }
    __syncthreads();
    int excl = incl - local + (wid > 0 ? warp_sums[wid - 1] : 0);
#pragma unroll
    for (int k = 0; k < kScanPer; ++k) {
        int i = base + k;
        if (i < n) out[i] = excl;
        excl += v[k];
    }
    if (threadIdx.x == kScanThreads - 1) block_sums[blockIdx.x] = warp_sums[(kScanThreads / 32) - 1];
}

__global__ void k_scan_sums(int *block_sums, int nb, int *total_out)
{
    // one block; sequential over chunks of blockDim
    __shared__ int carry;
    __shared__ int warp_sums[32];
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    for (int start = 0; start < nb; start += blockDim.x) {
        int i = start + threadIdx.x;
        int v = (i < nb) ? block_sums[i] : 0;
        int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
        int incl = v;
        for (int o = 1; o < 32; o <<= 1) {
            int t = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += t;
        }
        if (lane == 31) warp_sums[wid] = incl;
        __syncthreads();
        if (wid == 0) {
            int s = (lane < (int)(blockDim.x / 32)) ? warp_sums[lane] : 0;
            for (int o = 1; o < 32; o <<= 1) {
                int t = __shfl_up_sync(0xffffffffu, s, o);
                if (lane >= o) s += t;
            }
            warp_sums[lane] = s;
        }
        __syncthreads();
        int excl = carry + incl - v + (wid > 0 ? warp_sums[wid - 1] : 0);
        if (i < nb) block_sums[i] = excl;
        __syncthreads();
        if (threadIdx.x == 0) carry += warp_sums[(blockDim.x / 32) - 1];
        __syncthreads();
    }
    if (threadIdx.x == 0) *total_out = carry;
}

__global__ void k_scan_add(int *out, const int *block_sums, int n, const int *total, int *out_last)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] += block_sums[i / kScanBlock];
    if (i == 0) *out_last = *total;
}

// scratch: ceil(n / kScanBlock) + 1 ints
static int exclusive_scan(const int *in, int *out, int n, int *scratch, cudaStream_t st)
{
    int nb = (n + kScanBlock - 1) / kScanBlock;
    if (nb < 1) nb = 1;
    k_scan_blocks<<<nb, kScanThreads, 0, st>>>(in, out, scratch, n);
    k_scan_sums<<<1, 1024, 0, st>>>(scratch, nb, scratch + nb);
    k_scan_add<<<(n + 255) / 256 + 1, 256, 0, st>>>(out, scratch, n, scratch + nb, out + n);
    SDP_LAUNCH_CHECK();
    return SDP_OK;
}

// ----------------------------------------------------------------------------
// Arithmetic of the two reference builds (correctly rounded, no contraction)
// ----------------------------------------------------------------------------
__device__ __forceinline__ float tadd(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ double tadd(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ float tsub(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ double tsub(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ float tceil(float a) { return ceilf(a); }
__device__ __forceinline__ double tceil(double a) { return ceil(a); }
__device__ __forceinline__ float tfloor(float a) { return floorf(a); }
__device__ __forceinline__ double tfloor(double a) { return floor(a); }

// ----------------------------------------------------------------------------
// Binning
// ----------------------------------------------------------------------------
__device__ __forceinline__ int floor_div(int a, int b) { return (a >= 0) ? a / b : -((-a + b - 1) / b); }

// Computes the record of each visibility and its bin key.  snap applies
// correct_to_finegrid (degridgrid.c:24-25, 52-54) in precision T first.
// Kernel index of tap i (0 .. 2 hs - 1) of a box whose first tap lies
// hs - d below the visibility (0 < d <= 1): the taps below the visibility
// (i < hs) read |round(OS (i - hs + d'))| = OS (hs - i) - ko + h, the others
// OS (i - hs) + ko, with ko the index of tap hs and h in {0, 1} (h = 1 when
// the sub-sample offset is exactly half a sample: round() goes away from zero
// on both sides).  k_bin checks this form against the reference's expression
// for every tap of a visibility before it marks the visibility for the fast
// path.
__host__ __device__ __forceinline__ int fast_kidx(int i, int hs, int os, int ko, int h)
{
    return i < hs ? os * (hs - i) - ko + h : os * (i - hs) + ko;
}

// Offsets of kernel sample (ky, kx) within a plane of half support A - 1, in
// the plan's table layout (phase-major for power-of-two OS, see kcol / krow
// below: pm = 1), as the plan build computes them.
__device__ __forceinline__ int geo_kcol(int kx, int A, int pm, int OS, int shift)
{
    return pm ? ((kx & (OS - 1)) * A * A + (kx >> shift)) : kx;
}
__device__ __forceinline__ int geo_krow(int ky, int A, int pm, int OS, int shift)
{
    return pm ? ((ky & (OS - 1)) * OS * A * A + (ky >> shift) * A) : ky * A * OS;
}

// Packed tap-box geometry of a visibility for the warp-per-visibility kernels
// (16 bytes):
//   x: box origin in the tile as a cell of the kernels' shared tiles
//      (row * pitch + column, bits 0-15), w-plane (16-31);
//   y: CN (0-15), CP (16-31): table offsets of the columns; tap column i < hs
//      sits at CN - i * SC, column i >= hs at CP + (i - hs) * SC;
//   z: RN (0-15), RP (16-31): the same for the rows with step RS;
//   w: hs (0-3), kernel conjugated (4: w < 0), fast path (5), first of a
//      batch of four half-support-4 fast visibilities (6, k_batch_flags), index of the
//      tap box's degridding normalisation in the plan's dinv table (7-31:
//      (plane NC + row configuration) NC + column configuration, NC =
//      2 (OS + 1); a configuration is 2 ko + h of fast_kidx).
// SC = 1, RS = hs + 1 in the phase-major layout (SC = OS, RS = (hs + 1) OS^2
// in the reference layout, where row ky starts at ky (hs + 1) OS): below the
// visibility the kernel index falls by OS per tap (the phase stays, the
// block index falls by one), above it rises by OS.
// Fast path: std_gridding plan, both kernel sets with the same half support
// 1 <= hs <= 4, a 2 hs x 2 hs box inside the grid, and every tap's kernel
// index equal to fast_kidx (the reference's float subtraction (g - p) is
// exact for all but the tiniest |p|; those, and every other visibility, take
// the general path that evaluates degridgrid.c's expressions tap by tap).
template <typename T>
__device__ __forceinline__ uint4 fast_geometry(const Rec<T> &r, int plane, int hs, int hsd, int G, int OS, int tile,
                                               int tx, int ty, int pm, int shift, int nc, int pitch)
{
    uint4 g = make_uint4((uint32_t)plane << 16, 0u, 0u, (r.meta < 0) ? (1u << 4) : 0u);
    if (hs != hsd || hs < 1 || hs > 4) return g;
    const T fos = (T)OS;
    const T lox = tceil(tsub(r.px, (T)hs)), loy = tceil(tsub(r.py, (T)hs));
    const int ncols = (int)(tceil(tadd(r.px, (T)hs)) - lox);
    const int nrows = (int)(tceil(tadd(r.py, (T)hs)) - loy);
    const int n = 2 * hs;
    const int ix0 = (int)lox + G / 2, iy0 = (int)loy + G / 2;
    if (ncols != n || nrows != n || ix0 < 0 || iy0 < 0 || ix0 + n > G || iy0 + n > G) return g;
    const int tx0 = ix0 - tx * tile, ty0 = iy0 - ty * tile;
    if (tx0 < 0 || ty0 < 0 || tx0 >= tile || ty0 >= tile || tx0 > 255 || ty0 > 255) return g;
    const int kox = ref_kidx((int)lox + hs, r.px, fos), koy = ref_kidx((int)loy + hs, r.py, fos);
    const int kx0 = ref_kidx((int)lox, r.px, fos), ky0 = ref_kidx((int)loy, r.py, fos);
    const int hx = kx0 + kox - OS * hs, hy = ky0 + koy - OS * hs;
    if ((hx != 0 && hx != 1) || (hy != 0 && hy != 1)) return g;
    for (int i = 0; i < n; ++i) {
        if (ref_kidx((int)lox + i, r.px, fos) != fast_kidx(i, hs, OS, kox, hx)) return g;
        if (ref_kidx((int)loy + i, r.py, fos) != fast_kidx(i, hs, OS, koy, hy)) return g;
    }
    const int A = hs + 1;
    const int cn = geo_kcol(kx0, A, pm, OS, shift), cp = geo_kcol(kox, A, pm, OS, shift);
    const int rn = geo_krow(ky0, A, pm, OS, shift), rp = geo_krow(koy, A, pm, OS, shift);
    if (cn > 65535 || cp > 65535 || rn > 65535 || rp > 65535) return g;
    if (ty0 * pitch + tx0 > 65535) return g;
    g.x |= (uint32_t)(ty0 * pitch + tx0);
    g.y = (uint32_t)cn | ((uint32_t)cp << 16);
    g.z = (uint32_t)rn | ((uint32_t)rp << 16);
    g.w |= (uint32_t)hs | (1u << 5);
    if (nc) g.w |= (uint32_t)((plane * nc + 2 * koy + hy) * nc + 2 * kox + hx) << 7;
    return g;
}

template <typename T>
__global__ void k_bin(const float3 *__restrict__ uvw, int n, int mode, int snap, int G, int OS, double uv_scale,
                      double w_scale, const int2 *__restrict__ sup, const int2 *__restrict__ dsup, int nk, int nkd,
                      long long ntot_g, long long ntot_d, int hs_max, int ntx, int nty, int tile,
                      Rec<T> *__restrict__ rec_tmp, uint4 *__restrict__ geo_tmp, int pm, int os_shift,
                      int nc, int pitch, int cbits, int pbits, unsigned long long *__restrict__ skeys,
                      int *__restrict__ svals,
                      int *__restrict__ counts, int *__restrict__ flags)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float3 c = uvw[i];
    Rec<T> r;
    if (snap) {
        const T fu = ref_finegrid<T>(c.x, G, OS, uv_scale), fv = ref_finegrid<T>(c.y, G, OS, uv_scale);
        r.px = ref_grid_pos(fu, uv_scale);
        r.py = ref_grid_pos(fv, uv_scale);
    } else {
        r.px = ref_grid_pos((T)c.x, uv_scale);
        r.py = ref_grid_pos((T)c.y, uv_scale);
    }
    const T cz = (T)c.z;
    int plane;
    if (mode == SDP_GRID_SNAPPED) {
        plane = ref_widx_round(cz, w_scale);
        r.px = ref_snap(r.px, OS);
        r.py = ref_snap(r.py, OS);
    } else if (mode == kPlanG2G) {  // g2g: plane forced to 0 (degridgrid.c:215)
        plane = 0;
    } else {
        plane = ref_widx_std(cz, w_scale);
    }
    r.meta = plane | ((c.z < 0.0f) ? (int)0x80000000u : 0);
    r.idx = i;
    unsigned long long skey = ~0ull;  // unbinned: sorts after every binned visibility
    uint4 geo = make_uint4(0u, 0u, 0u, 0u);
    if (plane < 0 || plane >= nk || plane >= nkd) {
        atomicOr(flags, FLAG_PLANE);
    } else {
        const int2 sg = sup[plane], sd = dsup[plane];
        const int hs = sg.x, hsd = sd.x;
        // the plane's quarter table must lie inside the kernel array
        const long long eg = (long long)sg.y + (long long)(hs + 1) * OS * (hs + 1) * OS;
        const long long ed = (long long)sd.y + (long long)(hsd + 1) * OS * (hsd + 1) * OS;
        if (hs < 0 || hs > hs_max || hsd < 0 || hsd > hs_max || sg.y < 0 || sd.y < 0 || eg > ntot_g ||
            ed > ntot_d) {
            atomicOr(flags, FLAG_SUPPORT);
        } else {
            int lox = (int)tceil(tsub(r.px, (T)hs)) + G / 2;
            int loy = (int)tceil(tsub(r.py, (T)hs)) + G / 2;
            int tx = min(max(floor_div(lox, tile), 0), ntx - 1);
            int ty = min(max(floor_div(loy, tile), 0), nty - 1);
            const int key = (ty * ntx + tx) * nk + plane;
            atomicAdd(&counts[key], 1);
            // sort key: the (tile, plane) bin, then the tap-box origin in the
            // tile, so that visibilities of one origin are adjacent
            const int cx = min(max(lox - tx * tile, 0), tile - 1), cy = min(max(loy - ty * tile, 0), tile - 1);
            const unsigned long long cell = (unsigned long long)(cy * tile + cx);
#if SDP_SORT_CELL_MAJOR
            skey = ((((unsigned long long)(ty * ntx + tx) << cbits) | cell) << pbits) | (unsigned long long)plane;
#else
            skey = ((unsigned long long)key << cbits) | cell;
#endif
            if (mode == SDP_GRID_STD) geo = fast_geometry<T>(r, plane, hs, hsd, G, OS, tile, tx, ty, pm, os_shift, nc, pitch);
        }
    }
    rec_tmp[i] = r;
    geo_tmp[i] = geo;
    skeys[i] = skey;
    svals[i] = i;
}

// Plan order from the sorted visibility indices (perm): binned visibilities
// occupy positions [0, offsets[nbins]), the rest are marked -1.
// With gbase, also the quad record of each fast visibility of half support
// 4, all that the four-visibility path reads of it:
//   x: box origin as a cell of the shared tiles (bits 0-15), first of a
//      flagged batch of four (16, k_batch_flags);
//   y, z: table offsets of its tap quadrants (columns below, rows below) and
//      (columns below, rows above) in the degridding table, the conjugated
//      copy for w < 0 (plane offset + CN + RN, + CN + RP);
//   w: CP - CN (bits 0-12, signed: the columns-above quadrants lie that far
//      from the columns-below ones), its normalisation entry (13-31).
template <typename T>
__global__ void k_gather_plan(const Rec<T> *__restrict__ rec_tmp, const uint4 *__restrict__ geo_tmp, int n,
                              const int *__restrict__ n_binned, int *__restrict__ perm, Rec<T> *__restrict__ rec,
                              uint4 *__restrict__ geo, uint4 *__restrict__ gbase, const int *__restrict__ dpoff,
                              int conj_off)
{
    int pos = blockIdx.x * blockDim.x + threadIdx.x;
    if (pos >= n) return;
    if (pos >= *n_binned) {
        perm[pos] = -1;
        return;
    }
    const int i = perm[pos];
    rec[pos] = rec_tmp[i];
    const uint4 g = geo_tmp[i];
    geo[pos] = g;
    if (gbase) {
        uint4 q = make_uint4(0u, 0u, 0u, 0u);
        if ((g.w & 0x2fu) == 0x24u) {
            const int o = dpoff[g.x >> 16] + ((g.w & (1u << 4)) ? conj_off : 0);
            const int cn = (int)(g.y & 0xffffu), cp = (int)(g.y >> 16);
            const int rn = (int)(g.z & 0xffffu), rp = (int)(g.z >> 16);
            q = make_uint4(g.x & 0xffffu, (uint32_t)(o + cn + rn), (uint32_t)(o + cn + rp),
                           ((uint32_t)(cp - cn) & 0x1fffu) | ((g.w >> 7) << 13));
        }
        gbase[pos] = q;
    }
}

__global__ void k_item_counts(const int *__restrict__ offsets, int ntiles, int nk, int chunk,
                              int *__restrict__ item_counts)
{
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= ntiles) return;
    int b = offsets[t * nk], e = offsets[(t + 1) * nk];
    item_counts[t] = (e - b + chunk - 1) / chunk;
}

__global__ void k_item_fill(const int *__restrict__ offsets, const int *__restrict__ item_offsets, int ntiles,
                            int nk, int chunk, int4 *__restrict__ items)
{
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= ntiles) return;
    int b = offsets[t * nk], e = offsets[(t + 1) * nk];
    int o = item_offsets[t];
    for (int s = b; s < e; s += chunk) items[o++] = make_int4(t, s, min(e, s + chunk), 0);
}

// Marks (bit 6 of w) the first visibility of every batch of four, counted
// from its work item's start, whose four visibilities all take the fast path
// with half support 4: the warp-per-visibility kernels run such a batch
// branch-free.  One thread per work item.
__global__ void k_batch_flags(const int4 *__restrict__ items, const int *__restrict__ n_items, int cap,
                              uint4 *__restrict__ geo, uint4 *__restrict__ quad)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= cap || k >= *n_items) return;
    const int4 it = items[k];
    for (int b = it.y; b + 3 < it.z; b += 4) {
        bool all = true;
#pragma unroll
        for (int j = 0; j < 4; ++j) all = all && (geo[b + j].w & 0x2fu) == 0x24u;
        if (all) {
            geo[b].w |= 1u << 6;
            if (quad) quad[b].x |= 1u << 16;
        }
    }
}

// ----------------------------------------------------------------------------
// Tile kernels
// ----------------------------------------------------------------------------
__device__ __forceinline__ void cmac(float2 &acc, float2 a, float2 b)
{
    acc.x = fmaf(a.x, b.x, fmaf(-a.y, b.y, acc.x));
    acc.y = fmaf(a.y, b.x, fmaf(a.x, b.y, acc.y));
}

// Mirror of degridgrid.c:149-169 (in grid-centred coordinates).
__device__ __forceinline__ int mirror(int v, int gc)
{
    if (v < -gc) return (-gc - v) - gc;
    if (v >= gc) return (gc - v) + gc;
    return v;
}

// Kernel-table address of sample (ky, kx) of a plane.  The plan re-lays the
// tables out phase-major (k_relayout): with A = hs + 1 and OS a power of
// two, sample (ky, kx) is stored at
//   poff + ((ky % OS) * OS + kx % OS) * A^2 + (ky / OS) * A + kx / OS,
// so the taps of one visibility (a fixed sub-sample phase per axis, or its
// mirror) read a few short contiguous runs instead of one 32-byte sector per
// tap.  For other OS the plan keeps the reference layout ky * A * OS + kx.
__device__ __forceinline__ int kcol(const PlanDev &P, int A, int kx)
{
    return P.phase_major ? ((kx & P.os_mask) * A * A + (kx >> P.os_shift)) : kx;
}

__device__ __forceinline__ int krow(const PlanDev &P, int A, int ky)
{
    return P.phase_major ? ((ky & P.os_mask) * P.OS * A * A + (ky >> P.os_shift) * A) : ky * A * P.OS;
}

constexpr int kThreads = 256;  // 8 warps per CTA of the tile kernels

// One CTA per work item (persistent, items pulled from an atomic queue).
// LG lanes serve one visibility, so a warp works on 32 / LG visibilities at
// once.  Shared memory holds the input-grid tile (degridding, nearest cell)
// and the output subgrid as separate real / imaginary planes, both
// (32 + 2 hs_max)^2.
//
// Fast path (a visibility whose tap box lies inside the grid and the tile,
// with at most LG taps per axis and one support for both directions): lane
// c of the group owns tap column c and also computes the kernel-row offset
// and subgrid row of tap row c; a tap-row loop then broadcasts the row
// information with one shuffle per row, so each tap costs a kernel load, a
// shared load or two shared atomics and the multiply-adds.  Every other
// visibility (grid edges, where the reference mirrors or skips taps, 2 hs + 1
// taps, differing supports) takes the general path, which evaluates the
// reference's index arithmetic tap by tap.
// One work item of the tile kernels (the whole CTA): stage the input-grid
// tile, walk the item's visibilities, flush the subgrid.  `planes` holds the
// plan's per-plane constants; `share` / `share_sign` say whether the
// gridding samples can be taken from the degridding samples.
template <typename T, int GMODE, int OP, int LG>
__device__ __forceinline__ void tile_item(const PlanDev &P, const int4 it, float *smem_f, const int4 *planes,
                                          bool share, float share_sign, const float2 *__restrict__ vis_in,
                                          const float2 *__restrict__ in_grid, float2 *__restrict__ out_grid,
                                          float2 *__restrict__ pred_out, float2 *__restrict__ delta_out,
                                          const float2 *__restrict__ measured)
{
    constexpr bool kGrids = (OP != OP_DEGRID);
    constexpr bool kConv = (OP == OP_DEGRID || OP == OP_CYCLE_CONV);
    constexpr bool kStageIn = (OP != OP_GRID);
    constexpr int VPW = 32 / LG;
    constexpr bool kShareable = (OP == OP_CYCLE_CONV) && LG == 8;
    const int S = P.S, SS = S * S;
    float2 *mtile = reinterpret_cast<float2 *>(smem_f);
    float *sub_re = smem_f + (kStageIn ? 2 * SS : 0);
    float *sub_im = sub_re + SS;
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    const int grp = lane / LG;
    const int cl = lane % LG;
    const T fos = (T)P.OS;
    const Rec<T> *__restrict__ recs = static_cast<const Rec<T> *>(P.rec);
    float2 ksr[kShareable ? LG : 1];
    const int ox = (it.x % P.ntx) * P.tile;  // tile origin in grid cells
    const int oy = (it.x / P.ntx) * P.tile;
    if (kGrids)
        for (int k = threadIdx.x; k < 2 * SS; k += kThreads) sub_re[k] = 0.f;
    if (kStageIn)
        for (int k = threadIdx.x; k < SS; k += kThreads) {
            const int gy = oy + k / S, gx = ox + k % S;
            mtile[k] = (gx < P.G && gy < P.G) ? __ldg(&in_grid[(size_t)gy * P.G + gx]) : make_float2(0.f, 0.f);
        }
    __syncthreads();

    for (int base = it.y + warp * VPW; base < it.z; base += (kThreads / 32) * VPW) {
        const int r = base + grp;
        const bool valid = r < it.z;
        Rec<T> rec;
        if (valid) {
            rec = recs[r];
        } else {
            rec.px = (T)0;
            rec.py = (T)0;
            rec.meta = 0;
            rec.idx = 0;
        }
        const int plane = rec.meta & 0xffff;
        const float conj = (rec.meta < 0) ? -1.f : 1.f;

        // ---------------- tap geometry and the fast-path test ----------------
        const int4 pl = planes[plane];
        const int hs_d = kConv ? pl.x : 0;
        const int hs_g = kGrids ? pl.z : 0;
        const int hs = kGrids ? hs_g : hs_d;
        const T lox = tceil(tsub(rec.px, (T)hs));
        const T loy = tceil(tsub(rec.py, (T)hs));
        int ncols, nrows;
        if (GMODE == SDP_GRID_SNAPPED) {  // gridding_run.c:84-112: inclusive floor bound
            ncols = (int)(tfloor(tadd(rec.px, (T)hs)) - lox) + 1;
            nrows = (int)(tfloor(tadd(rec.py, (T)hs)) - loy) + 1;
        } else {  // degridgrid.c:93, 103
            ncols = (int)(tceil(tadd(rec.px, (T)hs)) - lox);
            nrows = (int)(tceil(tadd(rec.py, (T)hs)) - loy);
        }
        const int ix0 = (int)lox + P.gc, iy0 = (int)loy + P.gc;  // grid index of the first tap
        const int tx0 = ix0 - ox, ty0 = iy0 - oy;                // ... and in the tile
        const bool fast = valid && (!(kConv && kGrids) || hs_d == hs_g) && ncols <= LG && nrows <= LG &&
                          ix0 >= 0 && iy0 >= 0 && ix0 + ncols <= P.G && iy0 + nrows <= P.G && tx0 >= 0 &&
                          ty0 >= 0 && tx0 + ncols <= S && ty0 + nrows <= S;
        const unsigned fmask = __ballot_sync(0xffffffffu, fast);
        int colp_d = 0, colp_g = 0, lx = 0, rowpack = 0;
        bool colok = false;
        if (fast) {
            const int A = hs + 1;
            colok = cl < ncols;
            const int kc = kcol(P, A, ref_kidx((int)lox + cl, rec.px, fos));
            if (kConv) colp_d = pl.y + kc;
            if (kGrids) colp_g = pl.w + kc;
            lx = tx0 + cl;
            // row cl of the box: kernel-row offset and tile row (8 bits: S <= 256), packed
            rowpack = (krow(P, A, ref_kidx((int)loy + cl, rec.py, fos)) << 8) | (ty0 + cl);
        }

        // ---------------- degrid (prediction) ----------------
        float2 value = make_float2(0.f, 0.f);
        if (kConv) {
            // sum gv * Re(k) and gv * Im(k) separately; the conjugation of
            // k for w < 0 (degridgrid.c:143, 175) is applied after the sum
            float2 a1 = make_float2(0.f, 0.f), a2 = make_float2(0.f, 0.f);
            float nrm = 0.f;
            if (fast) {
#pragma unroll
                for (int rr = 0; rr < LG; ++rr) {
                    const int pk = __shfl_sync(fmask, rowpack, grp * LG + rr);
                    if (rr < nrows && colok) {
                        const float2 ks = __ldg(&P.dk[colp_d + (pk >> 8)]);
                        if constexpr (kShareable) ksr[rr] = ks;
                        const float2 gv = mtile[(pk & 255) * S + lx];
                        a1.x = fmaf(gv.x, ks.x, a1.x);
                        a1.y = fmaf(gv.y, ks.x, a1.y);
                        a2.x = fmaf(gv.x, ks.y, a2.x);
                        a2.y = fmaf(gv.y, ks.y, a2.y);
                        nrm = fmaf(ks.x, ks.x, fmaf(ks.y, ks.y, nrm));
                    }
                }
            } else if (valid) {
                // general path: degridgrid.c:147-186 tap by tap, edges mirrored
                const int A = hs_d + 1, stride = A * P.OS;
                const T dlox = tceil(tsub(rec.px, (T)hs_d));
                const T dloy = tceil(tsub(rec.py, (T)hs_d));
                const int dnc = (int)(tceil(tadd(rec.px, (T)hs_d)) - dlox);
                const int dnr = (int)(tceil(tadd(rec.py, (T)hs_d)) - dloy);
                const int off = pl.y;
                for (int c = cl; c < dnc; c += LG) {
                    const int cu = mirror((int)dlox + c, P.gc);
                    const int kx = ref_kidx(cu, rec.px, fos);
                    const bool kx_ok = kx < stride;
                    const int colp = off + kcol(P, A, kx);
                    const int gx = cu + P.gc;
                    const int tx = gx - ox;
                    for (int rr = 0; rr < dnr; ++rr) {
                        const int cv = mirror((int)dloy + rr, P.gc);
                        const int ky = ref_kidx(cv, rec.py, fos);
                        float2 ks = make_float2(0.f, 0.f);
                        if (kx_ok && ky < stride) ks = __ldg(&P.dk[colp + krow(P, A, ky)]);
                        const int gy = cv + P.gc;
                        const int ty = gy - oy;
                        float2 gv;
                        if ((unsigned)tx < (unsigned)S && (unsigned)ty < (unsigned)S) {
                            gv = mtile[ty * S + tx];
                        } else if (gx >= 0 && gy >= 0 && gx < P.G && gy < P.G) {
                            gv = __ldg(&in_grid[(size_t)gy * P.G + gx]);
                        } else {
                            gv = make_float2(0.f, 0.f);
                        }
                        a1.x = fmaf(gv.x, ks.x, a1.x);
                        a1.y = fmaf(gv.y, ks.x, a1.y);
                        a2.x = fmaf(gv.x, ks.y, a2.x);
                        a2.y = fmaf(gv.y, ks.y, a2.y);
                        nrm = fmaf(ks.x, ks.x, fmaf(ks.y, ks.y, nrm));
                    }
                }
            }
#pragma unroll
            for (int o = LG / 2; o > 0; o >>= 1) {
                a1.x += __shfl_xor_sync(0xffffffffu, a1.x, o);
                a1.y += __shfl_xor_sync(0xffffffffu, a1.y, o);
                a2.x += __shfl_xor_sync(0xffffffffu, a2.x, o);
                a2.y += __shfl_xor_sync(0xffffffffu, a2.y, o);
                nrm += __shfl_xor_sync(0xffffffffu, nrm, o);
            }
            // gv * (kr + i conj ki) summed; then degridgrid.c:188-191
            // (the .y fallback uses the new .x)
            const float sx = fmaf(-conj, a2.y, a1.x);
            const float sy = fmaf(conj, a2.x, a1.y);
            // (one correctly rounded reciprocal instead of two divides: the
            // sum's order already differs from the reference's)
            const float cn = __fsqrt_rn(nrm);
            const bool tiny = cn < 1e-5f;
            const float inv = tiny ? 1e5f : __frcp_rn(cn);
            const float nx = sx * inv;
            const float ny = tiny ? nx * inv : sy * inv;
            value = make_float2(nx, ny);
        } else if (OP == OP_CYCLE_NEAR || OP == OP_G2G) {
            // degridgrid.c:194-200 / :273-285
            const int x = ref_nearest(rec.px, P.gc), y = ref_nearest(rec.py, P.gc);
            const int tx = x - ox, ty = y - oy;
            if ((unsigned)tx < (unsigned)S && (unsigned)ty < (unsigned)S && x < P.G && y < P.G) {
                value = mtile[ty * S + tx];
            } else {
                const long long gi = (long long)x + (long long)y * P.G;
                if (gi >= 0 && gi < (long long)P.G * P.G) value = __ldg(&in_grid[gi]);
            }
        }

        float2 gval = make_float2(0.f, 0.f);
        if (OP == OP_GRID) {
            if (valid) gval = __ldg(&vis_in[rec.idx]);
        } else if (OP == OP_G2G) {
            gval = value;
        } else if (OP == OP_CYCLE_CONV || OP == OP_CYCLE_NEAR) {
            if (valid) {
                const float2 m = measured[r];
                gval = make_float2(__fsub_rn(m.x, value.x), __fsub_rn(m.y, value.y));
                if (cl == 0) {
                    if (pred_out) pred_out[rec.idx] = value;
                    if (delta_out) delta_out[rec.idx] = gval;
                }
            }
        } else {  // OP_DEGRID
            if (valid && cl == 0) pred_out[rec.idx] = value;
        }

        // ---------------- grid ----------------
        if (kGrids) {
            // vis * (kr + i conj ki): re = vr kr - (conj vi) ki, im = vi kr + (conj vr) ki
            const float ca = conj * gval.y, cb = conj * gval.x;
            if (fast) {
#pragma unroll
                for (int rr = 0; rr < LG; ++rr) {
                    const int pk = __shfl_sync(fmask, rowpack, grp * LG + rr);
                    if (rr < nrows && colok) {
                        float2 ks;
                        if constexpr (kShareable) {
                            ks = share ? make_float2(ksr[rr].x, share_sign * ksr[rr].y)
                                       : __ldg(&P.gk[colp_g + (pk >> 8)]);
                        } else {
                            ks = __ldg(&P.gk[colp_g + (pk >> 8)]);
                        }
                        const int cell = (pk & 255) * S + lx;
                        atomicAdd(sub_re + cell, fmaf(-ca, ks.y, gval.x * ks.x));
                        atomicAdd(sub_im + cell, fmaf(cb, ks.y, gval.y * ks.x));
                    }
                }
            } else if (valid) {
                // general path: degridgrid.c:93-122 / gridding_run.c:104-132 tap by tap
                const int A = hs_g + 1, stride = A * P.OS;
                const int off = pl.w;
                for (int c = cl; c < ncols; c += LG) {
                    const int u = (int)lox + c;
                    const int gx = u + P.gc;
                    if (gx < 0 || gx >= P.G) continue;
                    const int tx = gx - ox;
                    const int kx = ref_kidx(u, rec.px, fos);
                    if (kx >= stride || (unsigned)tx >= (unsigned)S) {  // cannot happen for a valid plan
                        atomicOr(P.flags, FLAG_BOX);
                        continue;
                    }
                    const int colp = off + kcol(P, A, kx);
                    for (int rr = 0; rr < nrows; ++rr) {
                        const int v = (int)loy + rr;
                        const int gy = v + P.gc;
                        if (gy < 0 || gy >= P.G) continue;
                        const int ty = gy - oy;
                        const int ky = ref_kidx(v, rec.py, fos);
                        if (ky >= stride || (unsigned)ty >= (unsigned)S) {
                            atomicOr(P.flags, FLAG_BOX);
                            continue;
                        }
                        const float2 ks = __ldg(&P.gk[colp + krow(P, A, ky)]);
                        const int cell = ty * S + tx;
                        atomicAdd(sub_re + cell, fmaf(-ca, ks.y, gval.x * ks.x));
                        atomicAdd(sub_im + cell, fmaf(cb, ks.y, gval.y * ks.x));
                    }
                }
            }
        }
    }
    if (kGrids) {
        __syncthreads();
        // flush: one vector atomic per touched cell of the subgrid
        for (int k = threadIdx.x; k < SS; k += kThreads) {
            const float2 v = make_float2(sub_re[k], sub_im[k]);
            if (v.x != 0.f || v.y != 0.f) {
                const int gy = oy + k / S, gx = ox + k % S;
                if (gx < P.G && gy < P.G) atomicAdd(&out_grid[(size_t)gy * P.G + gx], v);
            }
        }
    }
    __syncthreads();
}

// Per-plane constants {hs_d, degrid offset, hs_g, grid offset} of a plan
// into shared memory (the whole CTA).
template <int OP>
__device__ __forceinline__ void load_planes(const PlanDev &P, int4 *planes)
{
    constexpr bool kGrids = (OP != OP_DEGRID);
    constexpr bool kConv = (OP == OP_DEGRID || OP == OP_CYCLE_CONV);
    for (int k = threadIdx.x; k < P.nk_g; k += kThreads)
        planes[k] = make_int4(kConv && k < P.nk_d ? P.ds[k].x : 0, kConv && k < P.nk_d ? P.dpoff[k] : 0,
                              kGrids ? P.gs[k].x : 0, kGrids ? P.gpoff[k] : 0);
}

template <typename T, int GMODE, int OP, int LG>
__global__ void __launch_bounds__(kThreads, 4) k_tiles(PlanDev P, const float2 *__restrict__ vis_in,
                                                   const float2 *__restrict__ in_grid,
                                                   float2 *__restrict__ out_grid, float2 *__restrict__ pred_out,
                                                   float2 *__restrict__ delta_out,
                                                   const float2 *__restrict__ measured)
{
    extern __shared__ float smem_f[];
    constexpr bool kGrids = (OP != OP_DEGRID);
    constexpr bool kStageIn = (OP != OP_GRID);
    const int SS = P.S * P.S;
    int4 *planes = reinterpret_cast<int4 *>(smem_f + (kStageIn ? 2 * SS : 0) + (kGrids ? 2 * SS : 0));
    load_planes<OP>(P, planes);
    __shared__ int s_item;
    // When the degridding set equals the gridding set or its conjugate (bit
    // for bit, checked at plan build), the fast path of a cycle reads each
    // kernel sample once and keeps it in registers for the gridding pass.
    const int kdiff = (OP == OP_CYCLE_CONV && LG == 8) ? *P.kdiff : 3;
    const bool share = (kdiff & 1) == 0 || (kdiff & 2) == 0;
    const float share_sign = (kdiff & 1) == 0 ? 1.f : -1.f;
    for (;;) {
        if (threadIdx.x == 0) s_item = atomicAdd(P.item_counter, 1);
        __syncthreads();
        const int item = s_item;
        if (item >= *P.n_items) break;
        tile_item<T, GMODE, OP, LG>(P, P.items[item], smem_f, planes, share, share_sign, vis_in, in_grid, out_grid,
                                    pred_out, delta_out, measured);
    }
}

// Several plans (one per frequency channel) in one persistent launch over a
// shared (channel, tile) work queue: item.w is the channel.  A CTA copies a
// channel's plan description and per-plane constants to shared memory when
// its next item belongs to another channel (items are channel-major, so that
// is rare).
struct BatchIO {
    const float2 *in_grid;   // model grid of the channel
    float2 *out_grid;        // residual grid of the channel
    const float2 *measured;  // measured visibilities in plan order
    float2 *pred_out;
    float2 *delta_out;
};

template <typename T, int GMODE, int OP, int LG>
__global__ void __launch_bounds__(kThreads, 4) k_tiles_batch(const PlanDev *__restrict__ plans,
                                                         const BatchIO *__restrict__ io,
                                                         const int4 *__restrict__ items, int n_items,
                                                         int *item_counter, int smem_stride)
{
    extern __shared__ float smem_f[];
    __shared__ PlanDev sP;
    __shared__ BatchIO sIO;
    __shared__ int s_item, s_share;
    int4 *planes = reinterpret_cast<int4 *>(smem_f + smem_stride);
    int cur = -1;
    for (;;) {
        if (threadIdx.x == 0) s_item = atomicAdd(item_counter, 1);
        __syncthreads();
        const int item = s_item;
        if (item >= n_items) break;
        const int4 it = items[item];
        if (it.w != cur) {
            if (threadIdx.x == 0) {
                sP = plans[it.w];
                sIO = io[it.w];
                s_share = (OP == OP_CYCLE_CONV && LG == 8) ? *sP.kdiff : 3;
            }
            __syncthreads();
            load_planes<OP>(sP, planes);
            __syncthreads();
            cur = it.w;
        }
        const int kdiff = s_share;
        tile_item<T, GMODE, OP, LG>(sP, it, smem_f, planes, (kdiff & 1) == 0 || (kdiff & 2) == 0,
                                    (kdiff & 1) == 0 ? 1.f : -1.f, nullptr, sIO.in_grid, sIO.out_grid,
                                    sIO.pred_out, sIO.delta_out, sIO.measured);
    }
}

// ----------------------------------------------------------------------------
// Warp-per-visibility tile kernels (std_gridding plans, 1 <= hs <= 4)
// ----------------------------------------------------------------------------
// The group kernels above serve four visibilities per warp instruction and so
// must update the CTA's subgrid with shared-memory atomics (on sm_100 a float
// atomicAdd to shared memory is a compare-and-swap loop) and pay four-way
// bank conflicts on every access.  Here a warp serves one visibility at a
// time: lane (r, c) = (lane / 8, lane % 8) owns tap column c and tap rows r and
// r + 4 of the 2 hs x 2 hs box, so one warp access covers four box rows of
// eight cells (two conflict-free wavefronts with the row pitch = 8 mod 16),
// and each warp accumulates into its own private subgrid with plain loads and
// stores (the cells of one visibility are distinct; __syncwarp orders
// consecutive visibilities).  The subgrids are summed and flushed with one
// vector atomic per touched cell when the work item ends.  The tap geometry
// comes precomputed from the plan (fast_geometry), so a visibility costs an
// 8-byte load and a few integer operations per lane before its taps.
// Degridding sums are reduced for four visibilities at once (a transposed
// butterfly: 30 shuffles for 4 x 5 values).
constexpr int kFastVB = 4;  // visibilities per warp batch

// Lane's share of the five degridding sums of one general-path visibility
// (degridgrid.c:147-186 tap by tap, edges mirrored; the whole warp strides
// over the taps).
struct Sums5 {
    float v[5];
};

template <typename T>
__device__ __forceinline__ Sums5 slow_degrid(const PlanDev &P, const Rec<T> rec, int hs_d, int doff,
                                          const float2 *mtile, int ox, int oy, const float2 *__restrict__ in_grid)
{
    Sums5 acc = {{0.f, 0.f, 0.f, 0.f, 0.f}};
    const int lane = threadIdx.x & 31;
    const T fos = (T)P.OS;
    const int A = hs_d + 1, stride = A * P.OS;
    const T dlox = tceil(tsub(rec.px, (T)hs_d));
    const T dloy = tceil(tsub(rec.py, (T)hs_d));
    const int dnc = (int)(tceil(tadd(rec.px, (T)hs_d)) - dlox);
    const int dnr = (int)(tceil(tadd(rec.py, (T)hs_d)) - dloy);
    const int S = P.S;
    for (int t = lane; t < dnc * dnr; t += 32) {
        const int cc = t % dnc, rr = t / dnc;
        const int cu = mirror((int)dlox + cc, P.gc);
        const int kx = ref_kidx(cu, rec.px, fos);
        const int cv = mirror((int)dloy + rr, P.gc);
        const int ky = ref_kidx(cv, rec.py, fos);
        float2 ks = make_float2(0.f, 0.f);
        if (kx < stride && ky < stride) ks = __ldg(&P.dk[doff + kcol(P, A, kx) + krow(P, A, ky)]);
        const int gx = cu + P.gc, gy = cv + P.gc;
        const int tx = gx - ox, ty = gy - oy;
        float2 gv;
        if ((unsigned)tx < (unsigned)S && (unsigned)ty < (unsigned)S) {
            gv = mtile[ty * P.pitch + tx];
        } else if (gx >= 0 && gy >= 0 && gx < P.G && gy < P.G) {
            gv = __ldg(&in_grid[(size_t)gy * P.G + gx]);
        } else {
            gv = make_float2(0.f, 0.f);
        }
        acc.v[0] = fmaf(gv.x, ks.x, acc.v[0]);
        acc.v[1] = fmaf(gv.y, ks.x, acc.v[1]);
        acc.v[2] = fmaf(gv.x, ks.y, acc.v[2]);
        acc.v[3] = fmaf(gv.y, ks.y, acc.v[3]);
        acc.v[4] = fmaf(ks.x, ks.x, fmaf(ks.y, ks.y, acc.v[4]));
    }
    return acc;
}

// General-path gridding of one visibility into the warp's private subgrid
// (degridgrid.c:93-122 tap by tap; taps outside the grid skipped).  The taps
// of one visibility are distinct cells, so plain read-modify-writes suffice.
template <typename T>
__device__ __forceinline__ void slow_grid(const PlanDev &P, const Rec<T> rec, int hs_g, int goff, float2 *sub, int ox,
                                       int oy, float2 gval, float conj)
{
    const int lane = threadIdx.x & 31;
    const T fos = (T)P.OS;
    const int A = hs_g + 1, stride = A * P.OS;
    const T lox = tceil(tsub(rec.px, (T)hs_g));
    const T loy = tceil(tsub(rec.py, (T)hs_g));
    const int ncols = (int)(tceil(tadd(rec.px, (T)hs_g)) - lox);
    const int nrows = (int)(tceil(tadd(rec.py, (T)hs_g)) - loy);
    const float ca = conj * gval.y, cb = conj * gval.x;
    const int S = P.S;
    for (int t = lane; t < ncols * nrows; t += 32) {
        const int c = t % ncols, rr = t / ncols;
        const int u = (int)lox + c, v = (int)loy + rr;
        const int gx = u + P.gc, gy = v + P.gc;
        if (gx < 0 || gx >= P.G || gy < 0 || gy >= P.G) continue;
        const int tx = gx - ox, ty = gy - oy;
        const int kx = ref_kidx(u, rec.px, fos), ky = ref_kidx(v, rec.py, fos);
        if (kx >= stride || ky >= stride || (unsigned)tx >= (unsigned)S || (unsigned)ty >= (unsigned)S) {
            atomicOr(P.flags, FLAG_BOX);  // cannot happen for a valid plan
            continue;
        }
        const float2 ks = __ldg(&P.gk[goff + kcol(P, A, kx) + krow(P, A, ky)]);
        float2 *cell = sub + ty * P.pitch + tx;
        float2 a = *cell;
        a.x += fmaf(-ca, ks.y, gval.x * ks.x);
        a.y += fmaf(cb, ks.y, gval.y * ks.x);
        *cell = a;
    }
}

// g[j] for a runtime j < 4 without indexing the register array (which would
// move it to local memory).
__device__ __forceinline__ uint4 pick4(const uint4 (&g)[kFastVB], int j)
{
    return j == 0 ? g[0] : j == 1 ? g[1] : j == 2 ? g[2] : g[3];
}

// This lane's two taps (column c, rows r and r + 4) of a fast-path
// visibility: table offsets relative to the plane, the subgrid cell of tap
// (r, c), and which of the two taps lie in the 2 hs x 2 hs box (bits 0, 1).
__device__ __forceinline__ void fast_taps(const uint4 g, int c, int r, int lanecell, int pitch, int pm, int OS,
                                          int &off0, int &off1, int &ce, unsigned &aj)
{
    const int hs = (int)(g.w & 15u), A = hs + 1, n = 2 * hs;
    const int cn = (int)(g.y & 0xffffu), cp = (int)(g.y >> 16);
    const int rn = (int)(g.z & 0xffffu), rp = (int)(g.z >> 16);
    ce = (int)(g.x & 0xffffu) + lanecell;
    const int sc = pm ? 1 : OS, rs = pm ? A : A * OS * OS;
    const int colp = (c < hs) ? cn - c * sc : cp + (c - hs) * sc;
    const int r1 = r + 4;
    off0 = colp + ((r < hs) ? rn - r * rs : rp + (r - hs) * rs);
    off1 = colp + ((r1 < hs) ? rn - r1 * rs : rp + (r1 - hs) * rs);
    aj = ((c < n && r < n) ? 1u : 0u) | ((c < n && r1 < n) ? 2u : 0u);
}

// Reduces v[j][q] (j < 4 visibilities, q < 5 sums) over the warp; lanes
// 8 j .. 8 j + 7 end with visibility j's five totals in out[0..4].
__device__ __forceinline__ void reduce4x5(const float (&v)[kFastVB][5], float (&out)[5])
{
    const int lane = threadIdx.x & 31;
    const bool b4 = (lane & 16) != 0, b3 = (lane & 8) != 0;
    float w[2][5];
#pragma unroll
    for (int jj = 0; jj < 2; ++jj)
#pragma unroll
        for (int q = 0; q < 5; ++q) {
            const float keep = b4 ? v[2 + jj][q] : v[jj][q];
            const float send = b4 ? v[jj][q] : v[2 + jj][q];
            w[jj][q] = keep + __shfl_xor_sync(0xffffffffu, send, 16);
        }
#pragma unroll
    for (int q = 0; q < 5; ++q) {
        const float keep = b3 ? w[1][q] : w[0][q];
        const float send = b3 ? w[0][q] : w[1][q];
        out[q] = keep + __shfl_xor_sync(0xffffffffu, send, 8);
    }
#pragma unroll
    for (int o = 4; o > 0; o >>= 1)
#pragma unroll
        for (int q = 0; q < 5; ++q) out[q] += __shfl_xor_sync(0xffffffffu, out[q], o);
}

// Reduces v[j][q] (j < 4 visibilities, q < 2 sums) over the warp; lanes
// 8 j .. 8 j + 7 end with visibility j's two totals in s0, s1.
__device__ __forceinline__ void reduce4x2(const float (&v)[kFastVB][2], float &s0, float &s1)
{
    const int lane = threadIdx.x & 31;
    const bool b4 = (lane & 16) != 0, b3 = (lane & 8) != 0, b2 = (lane & 4) != 0;
    float w[2][2];
#pragma unroll
    for (int jj = 0; jj < 2; ++jj)
#pragma unroll
        for (int q = 0; q < 2; ++q) {
            const float keep = b4 ? v[2 + jj][q] : v[jj][q];
            const float send = b4 ? v[jj][q] : v[2 + jj][q];
            w[jj][q] = keep + __shfl_xor_sync(0xffffffffu, send, 16);
        }
    float u[2];
#pragma unroll
    for (int q = 0; q < 2; ++q) {
        const float keep = b3 ? w[1][q] : w[0][q];
        const float send = b3 ? w[0][q] : w[1][q];
        u[q] = keep + __shfl_xor_sync(0xffffffffu, send, 8);
    }
    // lanes 8 j + 4 q .. 8 j + 4 q + 3: sum q of visibility j
    float t = (b2 ? u[1] : u[0]) + __shfl_xor_sync(0xffffffffu, b2 ? u[0] : u[1], 4);
    t += __shfl_xor_sync(0xffffffffu, t, 2);
    t += __shfl_xor_sync(0xffffffffu, t, 1);
    const float o = __shfl_xor_sync(0xffffffffu, t, 4);
    s0 = b2 ? o : t;
    s1 = b2 ? t : o;
}

// Bulk (TMA) staging of a work item's records: one thread arms an mbarrier
// with the byte count and issues cp.async.bulk copies of the item's 16-byte
// geometry records and measured values into shared memory; the wait is
// bounded.  Addresses are 16-byte aligned: the geometry records are 16 bytes
// each, and the measured values (8 bytes) are copied from the even index at
// or below the item's first to the even index at or above its end (the
// plan's measured array is padded to 256 bytes, so the one value past the
// last item stays inside it).
constexpr long long kStageSpins = 1LL << 22;  // bounded mbarrier polls (well over a second)

__device__ __forceinline__ void stage_arm(uint32_t bar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}

__device__ __forceinline__ void stage_copy(uint32_t dst, const void *src, uint32_t bytes, uint32_t bar)
{
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst),
                 "l"(src), "r"(bytes), "r"(bar)
                 : "memory");
}

__device__ __forceinline__ bool stage_wait(uint32_t bar, uint32_t parity)
{
    for (long long i = 0; i < kStageSpins; ++i) {
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

// Per-CTA staging state: the item's records in shared memory and the
// mbarrier's phase.
struct ItemStage {
    uint4 *geo;         // chunk records
    uint4 *gb;          // chunk quad records (plans with gbase)
    float2 *meas;       // chunk + 2 values (from the even index at or below the item's first)
    uint64_t *bar;
    uint32_t phase;     // parity of the next completion
    int *fail;          // shared flag: a staging wait gave up
};

// One work item of the warp-per-visibility kernels (the whole CTA).
// OP is OP_GRID, OP_DEGRID or OP_CYCLE_CONV.  smem: the model tile (OP !=
// OP_GRID) and NW private subgrids (OP != OP_DEGRID), S rows of P.pitch cells.
// kShared: the launch holds only plans whose two kernel sets are equal or
// conjugate (the batched kernel checks this at creation), so the quad path
// needs no test of share.
template <typename T, int OP, int NW, bool kShared = false>
__device__ __forceinline__ bool fast_item(const PlanDev &Pin, const int4 it, ItemStage &stg, float2 *mtile,
                                          float2 *subs,
                                          float *wscr_all, const int4 *planes, bool share, float share_sign,
                                          const float2 *__restrict__ vis_in, const float2 *__restrict__ in_grid,
                                          float2 *__restrict__ out_grid, float2 *__restrict__ pred_out,
                                          float2 *__restrict__ delta_out, const float2 *__restrict__ measured)
{
    constexpr bool kGrids = (OP != OP_DEGRID);
    constexpr bool kConv = (OP != OP_GRID);
    const PlanDev &P = Pin;
    const int S = P.S, pitch = P.pitch, OS = P.OS;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int c = lane & 7, r = lane >> 3;
    const int ox = (it.x % P.ntx) * P.tile, oy = (it.x / P.ntx) * P.tile;
    float2 *sub = subs + (size_t)warp * S * pitch;
    float *wscr = wscr_all + warp * (kFastVB * 5);  // general-path sums of this warp's batch
    const Rec<T> *__restrict__ recs = static_cast<const Rec<T> *>(P.rec);
    // the item's records and measured values, copied into shared memory while
    // the model tile is staged
    const int m0 = it.y & ~1;
    const uint32_t bar = (uint32_t)__cvta_generic_to_shared(stg.bar);
    if (threadIdx.x == 0) {
        // the previous item's records were read through the generic proxy
        // (the CTA synchronised since): order those reads before the bulk
        // copies overwrite them
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        const uint32_t gbytes = (uint32_t)(it.z - it.y) * 16u;
        const uint32_t mbytes = (OP == OP_CYCLE_CONV) ? (uint32_t)(((it.z + 1) & ~1) - m0) * 8u : 0u;
        const uint32_t bbytes = (P.gbase && (kGrids ? (kShared || share) : true)) ? gbytes : 0u;
        stage_arm(bar, gbytes + bbytes + mbytes);
        stage_copy((uint32_t)__cvta_generic_to_shared(stg.geo), P.geo + it.y, gbytes, bar);
        if (bbytes) stage_copy((uint32_t)__cvta_generic_to_shared(stg.gb), P.gbase + it.y, bbytes, bar);
        if (OP == OP_CYCLE_CONV) stage_copy((uint32_t)__cvta_generic_to_shared(stg.meas), measured + m0, mbytes, bar);
    }
    if (kConv) {
        for (int k = threadIdx.x; k < S * S; k += 32 * NW) {
            const int y = k / S, x = k - y * S;
            const int gy = oy + y, gx = ox + x;
            mtile[y * pitch + x] =
                (gx < P.G && gy < P.G) ? __ldg(&in_grid[(size_t)gy * P.G + gx]) : make_float2(0.f, 0.f);
        }
    } else {
        // the item's input visibilities in plan order (gathered through the
        // permutation once per item, all loads of the CTA in flight together)
        for (int k = threadIdx.x; k < it.z - it.y; k += 32 * NW) stg.meas[k] = __ldg(&vis_in[P.perm[it.y + k]]);
    }
    if (threadIdx.x == 0) {
        if (!stage_wait(bar, stg.phase)) {
            // record the failure, then give the copies in flight one more
            // bounded wait before the CTA stops
            atomicOr(P.flags, FLAG_STAGE);
            stage_wait(bar, stg.phase);
            *stg.fail = 1;
        }
    }
    stg.phase ^= 1u;
    __syncthreads();
    if (*stg.fail) return false;
    const uint4 *sgeo = stg.geo - it.y;   // indexed by plan position
    const float2 *smeas = stg.meas - m0;
    const float2 *svis = stg.meas - it.y;  // OP_GRID: the item's input visibilities in plan order
    // four-visibility path (half support 4, and for the passes that grid, a
    // gridding set equal to the degridding set or its conjugate): a batch
    // reads only the quad records (k_gather_plan); lane (r, c) takes its two taps (rows r below
    // the visibility, r + 4 above) from the columns-below quadrants, or for
    // c >= 4 from the columns-above ones CP - CN further on; the lane's
    // offsets within the quadrants fold into its table pointers
    const bool quad = P.gbase != nullptr && (kGrids ? (kShared || share) : true);  // the gridding half reuses the samples
    const uint4 *squad = stg.gb - it.y;  // indexed by plan position
    const int cqm = (c < 4) ? 0 : -1;
    const int cofs4 = (c < 4) ? -c : c - 4;
    const float2 *dk_l0 = reinterpret_cast<const float2 *>(reinterpret_cast<uintptr_t>(P.dk) +
                                                           (intptr_t)(cofs4 - 5 * r) * (intptr_t)sizeof(float2));
    const float2 *dk_l1 = reinterpret_cast<const float2 *>(reinterpret_cast<uintptr_t>(P.dk) +
                                                           (intptr_t)(cofs4 + 5 * r) * (intptr_t)sizeof(float2));

    const int lanecell = r * pitch + c;
    const int pm = P.phase_major;
    // half support 4: column c < 4 of a box reads CN - c, the others CP + c - 4
    // (byte_perm picks the 16-bit field of the geometry word)
    const unsigned csel = (c < 4) ? 0x4410u : 0x4432u;
    const int cofs = cofs4;
    for (int b = it.y + warp * kFastVB; b < it.z; b += NW * kFastVB) {
        const int nv = min(kFastVB, it.z - b);  // visibilities in this batch (warp-uniform)
        const bool all4q = quad && nv == kFastVB && (squad[b].x & (1u << 16)) != 0u;
        uint4 g[kFastVB];
#pragma unroll
        for (int j = 0; j < kFastVB; ++j)
            g[j] = (j < nv && !all4q) ? sgeo[b + j] : make_uint4(0u, 0u, 0u, 0u);
        float2 meas_r = make_float2(0.f, 0.f);  // lanes 8 j ..: visibility j's measured value
        if (OP == OP_CYCLE_CONV && r < nv) meas_r = smeas[b + r];
        // A batch of four fast-path visibilities of half support 4 in the
        // phase-major layout (nearly every batch): straight-line code, every
        // tap of the 8 x 8 box active (rows r below the visibility at RN - 5 r,
        // rows r + 4 above it at RP + 5 r; columns c < 4 at CN - c, the others
        // at CP + c - 4), packed FP32x2 arithmetic.
        // (the plan marks the first visibility of such a batch, k_batch_flags;
        // plans without quad records take the grid-only form from the
        // geometry records)
        const bool all4 = all4q || (!kConv && !quad && nv == kFastVB && pm && (g[0].w & (1u << 6)));
        if (all4) {
            uint4 qr[kFastVB];
#pragma unroll
            for (int j = 0; j < kFastVB; ++j) qr[j] = all4q ? squad[b + j] : make_uint4(0u, 0u, 0u, 0u);
            float2 q0[kFastVB], q1[kFastVB];
            int ce4[kFastVB];
            bool fresh[kFastVB];  // visibility j starts a run of one tap-box origin
            float2 gv4 = make_float2(0.f, 0.f);
            float ie = 0.f;  // lanes 8 j ..: visibility j's normalisation entry, loaded ahead of its use
            if (kConv) ie = __ldg(&P.dinv[squad[b + r].w >> 13]);
            if (kConv) {
                // per visibility the lane's share of the real and imaginary
                // parts of sum m k; the samples come from the plan's
                // conjugated copy for w < 0 (degridgrid.c:176-183), the
                // normalisation from its table
                float acc[kFastVB][2];
                float2 m0 = make_float2(0.f, 0.f), m1 = m0;
#pragma unroll
                for (int j = 0; j < kFastVB; ++j) {
                    const int dc = ((int)(qr[j].w << 19) >> 19) & cqm;
                    q0[j] = __ldg(dk_l0 + ((int)qr[j].y + dc));
                    q1[j] = __ldg(dk_l1 + ((int)qr[j].z + dc));
                    const int ce = (int)(qr[j].x & 0xffffu) + lanecell;
                    ce4[j] = ce;
                    // the plan orders a tile's visibilities by tap-box origin:
                    // a visibility with its predecessor's origin reads the same
                    // model cells
                    fresh[j] = (j == 0) || ce != ce4[j > 0 ? j - 1 : 0];
                    if (fresh[j]) {
                        m0 = mtile[ce];
                        m1 = mtile[ce + 4 * pitch];
                    }
                    // a1 = (sum m.x kr, sum m.y kr), a2 = (sum m.x ki, sum m.y ki)
                    const float2 a1 = __ffma2_rn(m1, make_float2(q1[j].x, q1[j].x),
                                                 __fmul2_rn(m0, make_float2(q0[j].x, q0[j].x)));
                    const float2 a2 = __ffma2_rn(m1, make_float2(q1[j].y, q1[j].y),
                                                 __fmul2_rn(m0, make_float2(q0[j].y, q0[j].y)));
                    acc[j][0] = a1.x - a2.y;
                    acc[j][1] = a1.y + a2.x;
                }
                float sx, sy;
                reduce4x2(acc, sx, sy);
                // normalisation (degridgrid.c:188-191; a negative entry marks
                // sqrt(sum |k|^2) < 1e-5)
                const bool tiny = ie < 0.f;
                const float inv = fabsf(ie);
                const float nx = sx * inv;
                const float ny = tiny ? nx * inv : sy * inv;
                const float2 value = make_float2(nx, ny);
                const int i = b + r;
                if (OP == OP_CYCLE_CONV) {
                    gv4 = make_float2(__fsub_rn(meas_r.x, value.x), __fsub_rn(meas_r.y, value.y));
                    if (c == 0 && (pred_out || delta_out)) {
                        const int o = P.perm[i];
                        if (pred_out) pred_out[o] = value;
                        if (delta_out) delta_out[o] = gv4;
                    }
                } else if (c == 0) {
                    pred_out[P.perm[i]] = value;
                }
            }
            if (kGrids) {
                // the batch's four residuals to every lane: lane 8 j stores
                // visibility j's, each lane reads all four (two 16-byte loads)
                float4 gvp[2];
                if (kConv) {
                    if (c == 0) reinterpret_cast<float2 *>(wscr)[r] = gv4;
                    __syncwarp();
                    gvp[0] = reinterpret_cast<const float4 *>(wscr)[0];
                    gvp[1] = reinterpret_cast<const float4 *>(wscr)[1];
                }
                // a run of visibilities with one tap-box origin accumulates in
                // registers: one read and one write of the lane's two cells per
                // run, in the same order of operations as cell by cell
                float2 s0 = make_float2(0.f, 0.f), s1 = s0;
                int run_ce = 0;
#pragma unroll
                for (int j = 0; j < kFastVB; ++j) {
                    const uint4 gj = g[j];
                    float2 gv;
                    if (kConv) {
                        const float4 p2 = gvp[j >> 1];
                        gv = (j & 1) ? make_float2(p2.z, p2.w) : make_float2(p2.x, p2.y);
                    } else {
                        gv = svis[b + j];
                    }
                    float2 t0, t1;
                    int ce;
                    float2 nc;
                    if (all4q) {
                        // the degridding samples (conjugated for w < 0) with the
                        // gridding set's sign of the imaginary part:
                        // vis * (kr + i ks ki) = (vr kr - ks vi ki, vi kr + ks vr ki)
                        if (kConv) {
                            t0 = q0[j];
                            t1 = q1[j];
                            ce = ce4[j];
                        } else {
                            const int dc = ((int)(qr[j].w << 19) >> 19) & cqm;
                            t0 = __ldg(dk_l0 + ((int)qr[j].y + dc));
                            t1 = __ldg(dk_l1 + ((int)qr[j].z + dc));
                            ce = (int)(qr[j].x & 0xffffu) + lanecell;
                        }
                        nc = make_float2(-share_sign * gv.y, share_sign * gv.x);
                    } else {
                        const int colp = (int)__byte_perm(gj.y, 0u, csel) + cofs;
                        const float2 *kp = P.gk + planes[gj.x >> 16].w + colp;
                        t0 = __ldg(kp + (int)(gj.z & 0xffffu) - 5 * r);
                        t1 = __ldg(kp + (int)(gj.z >> 16) + 5 * r);
                        ce = (int)(gj.x & 0xffffu) + lanecell;
                        // vis * (kr + i conj ki): re = vr kr - (conj vi) ki, im = vi kr + (conj vr) ki
                        const float conj = (gj.w & (1u << 4)) ? -1.f : 1.f;
                        nc = make_float2(-conj * gv.y, conj * gv.x);
                    }
                    const uint32_t xprev = all4q ? qr[j > 0 ? j - 1 : 0].x : g[j > 0 ? j - 1 : 0].x;
                    const uint32_t xcur = all4q ? qr[j].x : gj.x;
                    if (kConv ? fresh[j] : (j == 0 || ((xcur ^ xprev) & 0xffffu) != 0u)) {
                        if (j > 0) {
                            sub[run_ce] = s0;
                            sub[run_ce + 4 * pitch] = s1;
                            __syncwarp();
                        }
                        run_ce = ce;
                        s0 = sub[ce];
                        s1 = sub[ce + 4 * pitch];
                    }
                    s0 = __ffma2_rn(nc, make_float2(t0.y, t0.y), __ffma2_rn(gv, make_float2(t0.x, t0.x), s0));
                    s1 = __ffma2_rn(nc, make_float2(t1.y, t1.y), __ffma2_rn(gv, make_float2(t1.x, t1.x), s1));
                }
                sub[run_ce] = s0;
                sub[run_ce + 4 * pitch] = s1;
                __syncwarp();
            }
            continue;
        }
        // per visibility: this lane's two taps (kernel samples and cell)
        float2 k0[kFastVB], k1[kFastVB];
        int cell[kFastVB];
        unsigned act = 0;  // bit 2j: tap (r, c) active, bit 2j+1: tap (r + 4, c) active
        unsigned slow = 0;  // bit j: visibility j takes the general path (warp-uniform)
#pragma unroll
        for (int j = 0; j < kFastVB; ++j)
            if (j < nv && !(g[j].w & (1u << 5))) slow |= 1u << j;
        float2 gval = make_float2(0.f, 0.f);  // lanes 8 j ..: visibility j's residual (CONV) / value (GRID)
        if (kConv) {
            if (slow) {
                // general-path visibilities of the batch: their sums, reduced
                // over the warp, go to shared memory (lane 0 adds them below)
                for (int j = 0; j < nv; ++j) {
                    if (!((slow >> j) & 1u)) continue;
                    const int4 pl = planes[pick4(g, j).x >> 16];
                    Sums5 t = slow_degrid<T>(P, recs[b + j], pl.x, pl.y, mtile, ox, oy, in_grid);
#pragma unroll
                    for (int o = 16; o > 0; o >>= 1)
#pragma unroll
                        for (int q = 0; q < 5; ++q) t.v[q] += __shfl_xor_sync(0xffffffffu, t.v[q], o);
                    if (lane == 0)
#pragma unroll
                        for (int q = 0; q < 5; ++q) wscr[j * 5 + q] = t.v[q];
                }
                __syncwarp();
            }
            float acc[kFastVB][5];
#pragma unroll
            for (int j = 0; j < kFastVB; ++j) {
#pragma unroll
                for (int q = 0; q < 5; ++q) acc[j][q] = 0.f;
                k0[j] = k1[j] = make_float2(0.f, 0.f);
                cell[j] = 0;
                if (j >= nv) continue;
                if (g[j].w & (1u << 5)) {
                    const int doff = planes[g[j].x >> 16].y;
                    int off0, off1, ce;
                    unsigned aj;
                    fast_taps(g[j], c, r, lanecell, pitch, pm, OS, off0, off1, ce, aj);
                    cell[j] = ce;
                    act |= aj << (2 * j);
                    float2 m0 = make_float2(0.f, 0.f), m1 = make_float2(0.f, 0.f);
                    if (aj & 1u) {
                        k0[j] = __ldg(&P.dk[doff + off0]);
                        m0 = mtile[ce];
                    }
                    if (aj & 2u) {
                        k1[j] = __ldg(&P.dk[doff + off1]);
                        m1 = mtile[ce + 4 * pitch];
                    }
                    acc[j][0] = fmaf(m0.x, k0[j].x, m1.x * k1[j].x);
                    acc[j][1] = fmaf(m0.y, k0[j].x, m1.y * k1[j].x);
                    acc[j][2] = fmaf(m0.x, k0[j].y, m1.x * k1[j].y);
                    acc[j][3] = fmaf(m0.y, k0[j].y, m1.y * k1[j].y);
                    acc[j][4] = fmaf(k0[j].x, k0[j].x, fmaf(k0[j].y, k0[j].y, fmaf(k1[j].x, k1[j].x, k1[j].y * k1[j].y)));
                } else if (lane == 0) {
#pragma unroll
                    for (int q = 0; q < 5; ++q) acc[j][q] = wscr[j * 5 + q];
                }
            }
            float tot[5];
            reduce4x5(acc, tot);
            // lanes 8 j .. 8 j + 7: visibility j (degridgrid.c:188-191; the
            // conjugation of k for w < 0 applied after the sum)
            const int j = r;
            const float conj = (pick4(g, j).w & (1u << 4)) ? -1.f : 1.f;
            const float sx = fmaf(-conj, tot[3], tot[0]);
            const float sy = fmaf(conj, tot[2], tot[1]);
            const float cn = __fsqrt_rn(tot[4]);
            const bool tiny = cn < 1e-5f;
            const float inv = tiny ? 1e5f : __frcp_rn(cn);
            const float nx = sx * inv;
            const float ny = tiny ? nx * inv : sy * inv;
            const float2 value = make_float2(nx, ny);
            if (j < nv) {
                const int i = b + j;
                if (OP == OP_CYCLE_CONV) {
                    const float2 m = meas_r;
                    gval = make_float2(__fsub_rn(m.x, value.x), __fsub_rn(m.y, value.y));
                    if (c == 0 && (pred_out || delta_out)) {
                        const int o = P.perm[i];
                        if (pred_out) pred_out[o] = value;
                        if (delta_out) delta_out[o] = gval;
                    }
                } else if (c == 0) {
                    pred_out[P.perm[i]] = value;
                }
            }
        }

        if (kGrids) {
#pragma unroll
            for (int j = 0; j < kFastVB; ++j) {
                if (j >= nv) break;
                if (!(g[j].w & (1u << 5))) continue;  // general path below
                float2 gv;
                if (kConv) {
                    gv.x = __shfl_sync(0xffffffffu, gval.x, 8 * j);
                    gv.y = __shfl_sync(0xffffffffu, gval.y, 8 * j);
                } else {
                    gv = svis[b + j];
                }
                const float conj = (g[j].w & (1u << 4)) ? -1.f : 1.f;
                float2 q0, q1;
                int ce;
                unsigned aj;
                float ksign;  // sign of the imaginary part of the gridding sample
                if (kConv && share) {
                    q0 = k0[j];
                    q1 = k1[j];
                    ce = cell[j];
                    aj = (act >> (2 * j)) & 3u;
                    ksign = share_sign;
                } else {
                    const int goff = planes[g[j].x >> 16].w;
                    int off0, off1;
                    fast_taps(g[j], c, r, lanecell, pitch, pm, OS, off0, off1, ce, aj);
                    q0 = (aj & 1u) ? __ldg(&P.gk[goff + off0]) : make_float2(0.f, 0.f);
                    q1 = (aj & 2u) ? __ldg(&P.gk[goff + off1]) : make_float2(0.f, 0.f);
                    ksign = 1.f;
                }
                // vis * (kr + i conj ki): re = vr kr - (conj vi) ki, im = vi kr + (conj vr) ki,
                // with ki = ksign * (the stored imaginary part)
                const float nca = -conj * ksign * gv.y, ncb = conj * ksign * gv.x;
                if (aj & 1u) {
                    float2 a = sub[ce];
                    a.x = fmaf(nca, q0.y, fmaf(gv.x, q0.x, a.x));
                    a.y = fmaf(ncb, q0.y, fmaf(gv.y, q0.x, a.y));
                    sub[ce] = a;
                }
                if (aj & 2u) {
                    float2 a = sub[ce + 4 * pitch];
                    a.x = fmaf(nca, q1.y, fmaf(gv.x, q1.x, a.x));
                    a.y = fmaf(ncb, q1.y, fmaf(gv.y, q1.x, a.y));
                    sub[ce + 4 * pitch] = a;
                }
                __syncwarp();
            }
            if (slow) {
                for (int j = 0; j < nv; ++j) {
                    if (!((slow >> j) & 1u)) continue;
                    float2 gv;
                    if (kConv) {
                        gv.x = __shfl_sync(0xffffffffu, gval.x, 8 * j);
                        gv.y = __shfl_sync(0xffffffffu, gval.y, 8 * j);
                    } else {
                        gv = svis[b + j];
                    }
                    const uint4 gj = pick4(g, j);
                    const int4 pl = planes[gj.x >> 16];
                    slow_grid<T>(P, recs[b + j], pl.z, pl.w, sub, ox, oy, gv, (gj.w & (1u << 4)) ? -1.f : 1.f);
                    __syncwarp();
                }
            }
        }
    }
    if (kGrids) {
        __syncthreads();
        // flush: the warps' subgrids summed, one vector atomic per touched cell
        for (int k = threadIdx.x; k < S * S; k += 32 * NW) {
            const int y = k / S, x = k - y * S;
            const int o = y * pitch + x;
            float2 v = make_float2(0.f, 0.f);
#pragma unroll
            for (int w = 0; w < NW; ++w) {
                const float2 t = subs[(size_t)w * S * pitch + o];
                v.x += t.x;
                v.y += t.y;
                subs[(size_t)w * S * pitch + o] = make_float2(0.f, 0.f);
            }
            if (v.x != 0.f || v.y != 0.f) {
                const int gy = oy + y, gx = ox + x;
                if (gx < P.G && gy < P.G) atomicAdd(&out_grid[(size_t)gy * P.G + gx], v);
            }
        }
    }
    __syncthreads();
    return true;
}

// Shared-memory layout of the warp-per-visibility kernels: the staged
// records of one work item (chunk 16-byte geometry records, chunk 16-byte
// quad records, chunk + 2 measured values), per-plane constants (nk int4),
// then the model tile and the NW subgrids.
// Shared memory of a block on sm_100 (opt-in limit) and an upper bound on
// the static arrays of the tile kernels (at most 896 B): the dynamic part
// must fit in what is left, and needs the opt-in attribute once the two
// together pass 48 KB.
constexpr size_t kSmemOptin = 227 * 1024;
constexpr size_t kStaticSmem = 1024;

__host__ __device__ __forceinline__ size_t fast_stage_bytes(int chunk)
{
    // geometry, quad records, measured values; the plane table after it is int4
    return (32 * (size_t)chunk + 8 * ((size_t)chunk + 2) + 15) / 16 * 16;
}
__host__ __device__ __forceinline__ size_t fast_smem_bytes(int op, int nw, int S, int pitch, int nk, int chunk)
{
    const size_t tilef2 = (size_t)S * pitch;
    return fast_stage_bytes(chunk) + 16 * (size_t)nk +
           8 * tilef2 * ((op != OP_GRID ? 1 : 0) + (op != OP_DEGRID ? nw : 0));
}

template <typename T, int OP, int NW>
__global__ void __launch_bounds__(32 * NW, 20 / NW) k_vis_fast(PlanDev P, const float2 *__restrict__ vis_in,
                                                      const float2 *__restrict__ in_grid,
                                                      float2 *__restrict__ out_grid, float2 *__restrict__ pred_out,
                                                      float2 *__restrict__ delta_out,
                                                      const float2 *__restrict__ measured)
{
    extern __shared__ __align__(16) unsigned char smem_fast[];
    const size_t stage_b = fast_stage_bytes(P.chunk);
    int4 *planes = reinterpret_cast<int4 *>(smem_fast + stage_b);
    float2 *mtile = reinterpret_cast<float2 *>(smem_fast + stage_b + 16 * (size_t)P.nk_g);
    float2 *subs = mtile + (OP != OP_GRID ? (size_t)P.S * P.pitch : 0);
    __shared__ __align__(16) float s_wscr[NW * kFastVB * 5];
    __shared__ int s_item, s_fail;
    __shared__ __align__(8) uint64_t s_bar;
    ItemStage stg{reinterpret_cast<uint4 *>(smem_fast), reinterpret_cast<uint4 *>(smem_fast + 16 * (size_t)P.chunk),
                  reinterpret_cast<float2 *>(smem_fast + 32 * (size_t)P.chunk), &s_bar, 0u, &s_fail};
    if (threadIdx.x == 0) {
        s_fail = 0;
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"((uint32_t)__cvta_generic_to_shared(&s_bar)));
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    for (int k = threadIdx.x; k < P.nk_g; k += 32 * NW)
        planes[k] = make_int4(OP != OP_GRID && k < P.nk_d ? P.ds[k].x : 0,
                              OP != OP_GRID && k < P.nk_d ? P.dpoff[k] : 0, OP != OP_DEGRID ? P.gs[k].x : 0,
                              OP != OP_DEGRID ? P.gpoff[k] : 0);
    if (OP != OP_DEGRID)
        for (size_t k = threadIdx.x; k < (size_t)NW * P.S * P.pitch; k += 32 * NW) subs[k] = make_float2(0.f, 0.f);
    const int kdiff = (OP == OP_CYCLE_CONV || OP == OP_GRID) ? *P.kdiff : 3;
    const bool share = (kdiff & 1) == 0 || (kdiff & 2) == 0;
    const float share_sign = (kdiff & 1) == 0 ? 1.f : -1.f;
    __syncthreads();
    for (;;) {
        if (threadIdx.x == 0) s_item = atomicAdd(P.item_counter, 1);
        __syncthreads();
        const int item = s_item;
        if (item >= *P.n_items) break;
        if (!fast_item<T, OP, NW>(P, P.items[item], stg, mtile, subs, s_wscr, planes, share, share_sign, vis_in,
                                  in_grid, out_grid, pred_out, delta_out, measured))
            break;
    }
}

// The fused pass of several plans (one per frequency channel) in one
// persistent launch over the (channel, tile) queue; smem sized for the
// largest channel (S_max rows of pitch_max, nk_max planes).
template <typename T, int NW>
__global__ void __launch_bounds__(32 * NW, 20 / NW) k_vis_fast_batch(const PlanDev *__restrict__ plans,
                                                            const BatchIO *__restrict__ io,
                                                            const int4 *__restrict__ items, int n_items,
                                                            int *item_counter, int nk_max, int tile_f2,
                                                            int chunk_max)
{
    extern __shared__ __align__(16) unsigned char smem_fast[];
    const size_t stage_b = fast_stage_bytes(chunk_max);
    int4 *planes = reinterpret_cast<int4 *>(smem_fast + stage_b);
    float2 *mtile = reinterpret_cast<float2 *>(smem_fast + stage_b + 16 * (size_t)nk_max);
    float2 *subs = mtile + tile_f2;
    __shared__ PlanDev sP;
    __shared__ BatchIO sIO;
    __shared__ int s_item, s_share, s_fail;
    __shared__ __align__(16) float s_wscr[NW * kFastVB * 5];
    __shared__ __align__(8) uint64_t s_bar;
    ItemStage stg{reinterpret_cast<uint4 *>(smem_fast), reinterpret_cast<uint4 *>(smem_fast + 16 * (size_t)chunk_max),
                  reinterpret_cast<float2 *>(smem_fast + 32 * (size_t)chunk_max), &s_bar, 0u, &s_fail};
    if (threadIdx.x == 0) {
        s_fail = 0;
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"((uint32_t)__cvta_generic_to_shared(&s_bar)));
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    for (size_t k = threadIdx.x; k < (size_t)NW * tile_f2; k += 32 * NW) subs[k] = make_float2(0.f, 0.f);
    int cur = -1;
    for (;;) {
        if (threadIdx.x == 0) s_item = atomicAdd(item_counter, 1);
        __syncthreads();
        const int item = s_item;
        if (item >= n_items) break;
        const int4 it = items[item];
        if (it.w != cur) {
            if (threadIdx.x == 0) {
                sP = plans[it.w];
                sIO = io[it.w];
                s_share = *sP.kdiff;
            }
            __syncthreads();
            for (int k = threadIdx.x; k < sP.nk_g; k += 32 * NW)
                planes[k] = make_int4(k < sP.nk_d ? sP.ds[k].x : 0, k < sP.nk_d ? sP.dpoff[k] : 0, sP.gs[k].x,
                                      sP.gpoff[k]);
            __syncthreads();
            cur = it.w;
        }
        const int kdiff = s_share;
        if (!fast_item<T, OP_CYCLE_CONV, NW, true>(sP, it, stg, mtile, subs, s_wscr, planes,
                                             (kdiff & 1) == 0 || (kdiff & 2) == 0, (kdiff & 1) == 0 ? 1.f : -1.f,
                                             nullptr, sIO.in_grid, sIO.out_grid, sIO.pred_out, sIO.delta_out,
                                             sIO.measured))
            break;
    }
}

// Degridding normalisation of every fast-path tap box (degridgrid.c:145-191)
// of a phase-major degridding set: entry (plane NC + cy) NC + cx, with
// c = 2 ko + h per axis (fast_kidx), holds 1 / sqrt(sum of |k|^2 over the
// 2 hs x 2 hs taps), summed row by row and column by column as the reference
// does; -1e5 when sqrt(sum) < 1e-5 (the reference then divides by 1e-5 and
// takes the imaginary part from the real one).  Planes outside the fast
// path's half supports (1..4) get 0.
__global__ void k_dinv(const float2 *__restrict__ dk2, const int *__restrict__ dpoff, const int2 *__restrict__ ds,
                       int nk, int OS, int shift, int nc, float *__restrict__ dinv)
{
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= nk * nc * nc) return;
    const int plane = e / (nc * nc), cy = (e / nc) % nc, cx = e % nc;
    const int hs = ds[plane].x;
    float v = 0.f;
    if (hs >= 1 && hs <= 4) {
        const int A = hs + 1;
        const int kox = cx >> 1, hx = cx & 1, koy = cy >> 1, hy = cy & 1;
        const float2 *k = dk2 + dpoff[plane];
        float norm = 0.f;
        for (int i = 0; i < 2 * hs; ++i) {
            const int ky = fast_kidx(i, hs, OS, koy, hy);
            for (int j = 0; j < 2 * hs; ++j) {
                const int kx = fast_kidx(j, hs, OS, kox, hx);
                const float2 t = k[geo_kcol(kx, A, 1, OS, shift) + geo_krow(ky, A, 1, OS, shift)];
                norm = __fadd_rn(norm, __fadd_rn(__fmul_rn(t.x, t.x), __fmul_rn(t.y, t.y)));
            }
        }
        const float cn = __fsqrt_rn(norm);
        v = cn < 1e-5f ? -1e5f : __frcp_rn(cn);
    }
    dinv[e] = v;
}

// dst = conj(src), n samples.
__global__ void k_conj_copy(const float2 *__restrict__ src, long long n, float2 *__restrict__ dst)
{
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const float2 v = src[i];
        dst[i] = make_float2(v.x, -v.y);
    }
}

// Phase-major copy of a kernel set (see kcol / krow).  One thread per output
// sample; plane p of the source starts at supports[p].y, of the copy at
// poff[p] (planes packed back to back).
__global__ void k_relayout(const float2 *__restrict__ src, long long src_total, const int2 *__restrict__ sup,
                           const int *__restrict__ poff, int nk, int OS, int os_shift, int max_per_plane,
                           float2 *__restrict__ dst)
{
    const int p = blockIdx.y;
    if (p >= nk) return;
    const int hs = sup[p].x;
    if (hs < 0) return;
    const int A = hs + 1, stride = A * OS;
    // planes wider than the plan's maximum are never addressed (binning flags them)
    const int n = stride * stride;
    if (n > max_per_plane) return;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const int ky = i / stride, kx = i % stride;
        const long long si = (long long)sup[p].y + i;
        const float2 v = (sup[p].y >= 0 && si < src_total) ? src[si] : make_float2(0.f, 0.f);
        const int di = ((ky & (OS - 1)) * OS + (kx & (OS - 1))) * A * A + (ky >> os_shift) * A + (kx >> os_shift);
        dst[poff[p] + di] = v;
    }
}

// Packed plane offsets of the copy (one thread; nk is small).  A plane wider
// than hs_max takes no room: binning never lets a visibility use it.
__global__ void k_plane_offsets(const int2 *__restrict__ sup, int nk, int OS, int hs_max, int *__restrict__ poff)
{
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    int o = 0;
    for (int p = 0; p < nk; ++p) {
        poff[p] = o;
        const int hs = sup[p].x;
        if (hs >= 0 && hs <= hs_max) o += (hs + 1) * OS * (hs + 1) * OS;
    }
}

// Sets bit 0 of *diff when some sample of the degridding set differs from
// the gridding set, bit 1 when some sample differs from the gridding set's
// conjugate (equal supports required; `related` = 0 sets both).  The tile
// kernel reads each sample once for both passes when a bit is clear.
__global__ void k_kernels_differ(const int2 *__restrict__ gs, const int2 *__restrict__ ds,
                                 const int *__restrict__ gpoff, const int *__restrict__ dpoff,
                                 const float2 *__restrict__ gk, const float2 *__restrict__ dk, int related, int nk,
                                 int OS, int max_per_plane, int *diff)
{
    const int p = blockIdx.y;
    if (!related) {
        if (threadIdx.x == 0 && blockIdx.x == 0) atomicOr(diff, 3);
        return;
    }
    if (p >= nk) return;
    const int hs = gs[p].x;
    if (ds[p].x != hs) {
        if (threadIdx.x == 0 && blockIdx.x == 0) atomicOr(diff, 3);
        return;
    }
    if (hs < 0) return;
    const int n = (hs + 1) * OS * (hs + 1) * OS;
    if (n > max_per_plane) return;
    int d = 0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const float2 a = gk[gpoff[p] + i], b = dk[dpoff[p] + i];
        const bool re = __float_as_uint(a.x) == __float_as_uint(b.x);
        if (!re || __float_as_uint(a.y) != __float_as_uint(b.y)) d |= 1;
        if (!re || (__float_as_uint(a.y) ^ 0x80000000u) != __float_as_uint(b.y)) d |= 2;
    }
    if (d) atomicOr(diff, d);
}

// Identity offsets (reference layout kept): poff[p] = supports[p].y.
__global__ void k_plane_offsets_identity(const int2 *__restrict__ sup, int nk, int *__restrict__ poff)
{
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < nk; p += gridDim.x * blockDim.x) poff[p] = sup[p].y;
}

__global__ void k_gather_sorted(const float2 *__restrict__ src, const int *__restrict__ perm, int n,
                                float2 *__restrict__ dst)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int j = perm[i];  // -1 past the binned records (visibilities flagged out of the tables)
    dst[i] = (j >= 0 && j < n) ? src[j] : make_float2(0.f, 0.f);
}

__global__ void k_fill_zero2(float2 *p, size_t n)
{
    size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    size_t stride = (size_t)gridDim.x * blockDim.x;
    for (; i < n; i += stride) p[i] = make_float2(0.f, 0.f);
}

}  // namespace sdp

namespace sdp {

static size_t align_up(size_t x, size_t a) { return (x + a - 1) / a * a; }

static PlanDev plan_dev(const sdp_visplan *p)
{
    PlanDev d;
    d.G = p->geom.grid_size;
    d.gc = d.G / 2;
    d.OS = p->geom.oversampling;
    d.nk_g = p->gk.num_kernels;
    d.nk_d = p->dk.num_kernels;
    d.ntx = p->ntx;
    d.tile = p->tile;
    d.nty = p->nty;
    d.W = p->W;
    d.S = p->S;
    d.uv_scale = p->geom.uv_scale;
    d.w_scale = p->geom.w_scale;
    d.phase_major = p->phase_major;
    d.os_mask = p->geom.oversampling - 1;
    d.os_shift = 0;
    while ((1 << d.os_shift) < p->geom.oversampling) ++d.os_shift;
    d.gk = p->phase_major ? p->gk2 : reinterpret_cast<const float2 *>(p->gk.kernels);
    d.gs = reinterpret_cast<const int2 *>(p->gk.supports);
    d.gpoff = p->gpoff;
    d.dk = p->phase_major ? p->dk2 : reinterpret_cast<const float2 *>(p->dk.kernels);
    d.ds = reinterpret_cast<const int2 *>(p->dk.supports);
    d.dpoff = p->dpoff;
    d.kdiff = p->kshare;
    d.rec = p->rec;
    d.items = p->items;
    d.n_items = p->n_items;
    d.item_counter = p->item_counter;
    d.flags = p->flags;
    d.pitch = p->pitch;
    d.chunk = p->chunk;
    d.geo = p->geo;
    d.perm = p->perm;
    d.dinv = p->dinv;
    d.gbase = p->gbase;
    return d;
}

static int check_geometry(const sdp_geometry *g)
{
    SDP_CHECK_ARG(g != nullptr, "geometry is NULL");
    SDP_CHECK_ARG(g->grid_size >= 8 && g->grid_size % 2 == 0, "grid_size %d must be even and >= 8", g->grid_size);
    if (g->grid_size > 32768) return set_error(SDP_ERR_RANGE, "grid_size %d exceeds 32768", g->grid_size);
    SDP_CHECK_ARG(g->oversampling >= 1 && g->oversampling <= 64, "oversampling %d out of [1, 64]", g->oversampling);
    return SDP_OK;
}

static int check_kernels(const sdp_wkernels *k, const char *what)
{
    SDP_CHECK_ARG(k != nullptr && k->kernels != nullptr && k->supports != nullptr, "%s kernels are NULL", what);
    SDP_CHECK_ARG(k->num_kernels >= 1 && k->num_kernels <= 65535, "%s: num_kernels %d", what, k->num_kernels);
    if (k->max_half_support < 0 || k->max_half_support > kMaxHalfSupport)
        return set_error(SDP_ERR_RANGE, "%s: max half support %d outside [0, %d]", what, k->max_half_support,
                         kMaxHalfSupport);
    return SDP_OK;
}

// Bits of the plan's sort key (k_bin): cbits for the tap-box origin in the
// tile, pbits for the plane (cell-major order only), end_bit in all.  The
// bin field is one bit wider than the largest bin needs, so the all-ones key
// of an unbinned visibility sorts after every binned one.
static int bit_length(unsigned long long x)
{
    int b = 0;
    while (b < 64 && (x >> b) != 0ull) ++b;
    return b;
}

static void plan_sort_bits(const sdp_visplan *p, int *cbits, int *pbits, int *end_bit)
{
    *cbits = bit_length((unsigned long long)p->tile * p->tile - 1);
#if SDP_SORT_CELL_MAJOR
    *pbits = bit_length((unsigned long long)p->nk - 1);
    *end_bit = bit_length((unsigned long long)p->ntiles) + *cbits + *pbits;
#else
    *pbits = 0;
    *end_bit = bit_length((unsigned long long)p->nbins) + *cbits;
#endif
}

// Temporary storage of the radix sort of the plan build (the keys and
// values ping-pong between arena regions that are free at that point).
static size_t plan_sort_temp_bytes(const sdp_visplan *p)
{
    if (p->n <= 0) return 0;
    int cbits, pbits, end_bit;
    plan_sort_bits(p, &cbits, &pbits, &end_bit);
    cub::DoubleBuffer<unsigned long long> k(nullptr, nullptr);
    cub::DoubleBuffer<int> v(nullptr, nullptr);
    size_t bytes = 0;
    if (cub::DeviceRadixSort::SortPairs(nullptr, bytes, k, v, p->n, 0, end_bit) != cudaSuccess) {
        (void)cudaGetLastError();
        // no device to ask: a bound well above what the sort needs (its
        // per-tile histograms and look-back state)
        bytes = ((size_t)64 << 20) + (size_t)p->n;
    }
    return bytes;
}

// Entries of the degridding normalisation table (0: not built).  The fast
// path's packed geometry has 26 bits for the entry index.
// Samples of one plane's phase-major copy (the largest half support).
static size_t plan_per_plane(const sdp_visplan *p)
{
    return (size_t)(p->hs_max + 1) * p->geom.oversampling * (p->hs_max + 1) * p->geom.oversampling;
}

// Entries of the degridding normalisation table, 0 when the four-visibility
// path is not available (it needs the phase-major layout, a table index
// that fits the geometry's 25 bits, and table bases, the conjugated copy
// included, that fit an int; the quad record holds the entry index in 19
// bits).
static size_t plan_dinv_entries(const sdp_visplan *p)
{
    if (!p->phase_major || p->dinv_nc <= 0) return 0;
    const size_t e = (size_t)p->dk.num_kernels * p->dinv_nc * p->dinv_nc;
    if (2 * plan_per_plane(p) * (size_t)p->dk.num_kernels >= ((size_t)1 << 31)) return 0;
    return e < ((size_t)1 << 19) ? e : 0;
}

// Arena layout of a plan (offsets in bytes).
static void plan_layout(const sdp_visplan *p, size_t *off, size_t *total)
{
    const int n = p->n;
    size_t o = 0;
    const size_t nb_scan = (size_t)((std::max(p->nbins, p->ntiles) + kScanBlock - 1) / kScanBlock + 2);
    const size_t rb = visplan_record_bytes(p);
    off[0] = o; o = align_up(o + rb * (size_t)std::max(n, 1), 256);                       // rec
    off[1] = o; o = align_up(o + rb * (size_t)std::max(n, 1), 256);                       // rec_tmp
    off[2] = o; o = align_up(o + sizeof(int) * (size_t)std::max(n, 1), 256);              // perm
    off[3] = o; o = align_up(o + sizeof(int) * (size_t)std::max(n, 1), 256);              // sort values
    off[4] = o; o = align_up(o + sizeof(int) * ((size_t)p->nbins + 1), 256);              // counts / fill
    off[5] = o; o = align_up(o + sizeof(int) * ((size_t)p->nbins + 1), 256);              // offsets
    off[6] = o; o = align_up(o + sizeof(int) * ((size_t)p->ntiles + 1), 256);             // item counts
    off[7] = o; o = align_up(o + sizeof(int) * ((size_t)p->ntiles + 1), 256);             // item offsets
    off[8] = o; o = align_up(o + sizeof(int4) * ((size_t)n / p->chunk + p->ntiles + 1), 256);// items
    off[9] = o; o = align_up(o + sizeof(int) * nb_scan, 256);                             // scan scratch
    off[10] = o; o = align_up(o + sizeof(int) * 4, 256);                                  // scalars
    off[11] = o; o = align_up(o + sizeof(float2) * (size_t)std::max(n, 1), 256);          // measured
    off[12] = o; o = align_up(o + sizeof(int) * (size_t)p->gk.num_kernels, 256);          // gpoff
    off[13] = o; o = align_up(o + sizeof(int) * (size_t)p->dk.num_kernels, 256);          // dpoff
    const size_t per = (size_t)(p->hs_max + 1) * p->geom.oversampling * (p->hs_max + 1) * p->geom.oversampling;
    off[14] = o; o = align_up(o + (p->phase_major ? sizeof(float2) * per * p->gk.num_kernels : 0), 256);  // gk2
    // dk2: the phase-major degridding set, then (four-visibility path) its
    // conjugate at dk_conj_off = per * num_kernels
    off[15] = o; o = align_up(o + (p->phase_major ? sizeof(float2) * per * p->dk.num_kernels : 0) *
                                      (plan_dinv_entries(p) ? 2 : 1), 256);
    off[16] = o; o = align_up(o + sizeof(uint4) * (size_t)std::max(n, 1), 256);          // geo
    off[17] = o; o = align_up(o + sizeof(uint4) * (size_t)std::max(n, 1), 256);          // geo_tmp
    off[18] = o; o = align_up(o + plan_sort_temp_bytes(p), 256);                           // sort temp
    off[19] = o; o = align_up(o + sizeof(float) * plan_dinv_entries(p), 256);              // dinv
    off[20] = o; o = align_up(o + (plan_dinv_entries(p) ? sizeof(uint4) * (size_t)std::max(n, 1) : 0), 256);  // gbase
    *total = o;
}

size_t visplan_record_bytes(const sdp_visplan *p)
{
    return p->coord_f64 ? sizeof(Rec<double>) : sizeof(Rec<float>);
}

int visplan_setup(sdp_visplan *p, const sdp_geometry *geom, const sdp_wkernels *gk, const sdp_wkernels *dk, int n,
                  int mode_flags)
{
    const int mode = mode_flags & 0xff;
    SDP_CHECK_ARG((mode_flags & ~(0xff | SDP_PLAN_COORD_F64 | SDP_PLAN_SNAP)) == 0, "unknown plan flags 0x%x",
                  mode_flags);
    p->coord_f64 = (mode_flags & SDP_PLAN_COORD_F64) ? 1 : 0;
    p->snap = (mode_flags & SDP_PLAN_SNAP) ? 1 : 0;
    SDP_TRY(check_geometry(geom));
    SDP_TRY(check_kernels(gk, "gridding"));
    if (dk == nullptr) dk = gk;
    SDP_TRY(check_kernels(dk, "degridding"));
    SDP_CHECK_ARG(n >= 0, "num_vis %d is negative", n);
    SDP_CHECK_ARG(mode == SDP_GRID_STD || mode == SDP_GRID_SNAPPED || mode == kPlanG2G, "grid_mode %d unknown", mode);
    p->geom = *geom;
    p->gk = *gk;
    p->dk = *dk;
    p->mode = mode;
    p->n = n;
    const int G = geom->grid_size;
    p->ntx = (G + p->tile - 1) / p->tile;
    p->nty = p->ntx;
    p->ntiles = p->ntx * p->nty;
    p->nk = gk->num_kernels;
    p->nbins = p->ntiles * p->nk;
    p->hs_max = std::max(gk->max_half_support, dk->max_half_support);
    p->W = 2 * p->hs_max + 1;
    p->S = p->tile + 2 * p->hs_max;
    // rows of 8-byte cells whose starts are 16 banks apart: the four rows a
    // warp touches in one access fall into two conflict-free bank halves
    p->pitch = p->S + ((8 - p->S % 16) + 16) % 16;
    const int os = geom->oversampling;
    p->phase_major = (os & (os - 1)) == 0 ? 1 : 0;
    p->dinv_nc = 2 * (os + 1);
    return SDP_OK;
}

size_t visplan_arena_bytes(const sdp_visplan *p)
{
    size_t off[21], total;
    plan_layout(p, off, &total);
    return total;
}

// (Re)builds the plan's kernel-table copies and the sharing flag from
// p->gk / p->dk (the binning does not depend on the table contents, only on
// the supports, so a plan can be reused with other tables of the same
// supports after this).
int visplan_kernels(sdp_visplan *p, cudaStream_t st)
{
    SDP_CUDA_TRY(cudaMemsetAsync(p->kshare, 0, sizeof(int), st));
    // kernel tables: phase-major copies (or the caller's tables as they are)
    {
        const int os = p->geom.oversampling;
        int os_shift = 0;
        while ((1 << os_shift) < os) ++os_shift;
        const int per = (p->hs_max + 1) * os * (p->hs_max + 1) * os;
        const sdp_wkernels *sets[2] = {&p->gk, &p->dk};
        int *poffs[2] = {p->gpoff, p->dpoff};
        float2 *dsts[2] = {p->gk2, p->dk2};
        for (int t = 0; t < 2; ++t) {
            const int2 *sup = reinterpret_cast<const int2 *>(sets[t]->supports);
            const int nk = sets[t]->num_kernels;
            if (p->phase_major) {
                k_plane_offsets<<<1, 32, 0, st>>>(sup, nk, os, p->hs_max, poffs[t]);
                dim3 grid((per + 255) / 256, nk);
                k_relayout<<<grid, 256, 0, st>>>(reinterpret_cast<const float2 *>(sets[t]->kernels),
                                                 (long long)sets[t]->total_samples, sup, poffs[t], nk, os, os_shift,
                                                 per, dsts[t]);
            } else {
                k_plane_offsets_identity<<<(nk + 255) / 256, 256, 0, st>>>(sup, nk, poffs[t]);
            }
            SDP_LAUNCH_CHECK();
        }
        // is the degridding set the gridding set, or its conjugate, bit for bit?
        const int related = p->phase_major && p->gk.num_kernels == p->dk.num_kernels;
        const int nk = related ? p->gk.num_kernels : 1;
        k_kernels_differ<<<dim3((per + 255) / 256, nk), 256, 0, st>>>(
            reinterpret_cast<const int2 *>(p->gk.supports), reinterpret_cast<const int2 *>(p->dk.supports), p->gpoff,
            p->dpoff, p->gk2, p->dk2, related, nk, os, per, p->kshare);
        SDP_LAUNCH_CHECK();
        if (p->dinv) {
            // conjugated copy of the degridding set: a w < 0 visibility's taps
            // read it, so the four-visibility path needs no sign per sample
            const long long nconj = (long long)p->dk_conj_off;
            k_conj_copy<<<(int)std::min<long long>((nconj + 255) / 256, 148 * 16), 256, 0, st>>>(
                p->dk2, nconj, p->dk2 + nconj);
            SDP_LAUNCH_CHECK();
            const int ne = (int)plan_dinv_entries(p);
            k_dinv<<<(ne + 255) / 256, 256, 0, st>>>(p->dk2, p->dpoff, reinterpret_cast<const int2 *>(p->dk.supports),
                                                     p->dk.num_kernels, os, os_shift, p->dinv_nc, p->dinv);
            SDP_LAUNCH_CHECK();
        }
    }

    return SDP_OK;
}

int visplan_build(sdp_visplan *p, void *arena, const float3 *uvw, cudaStream_t st)
{
    size_t off[21], total;
    plan_layout(p, off, &total);
    char *a = static_cast<char *>(arena);
    p->arena = arena;
    p->rec = a + off[0];
    void *rec_tmp = a + off[1];
    p->perm = reinterpret_cast<int *>(a + off[2]);
    int *svals = reinterpret_cast<int *>(a + off[3]);
    int *counts = reinterpret_cast<int *>(a + off[4]);
    int *offsets = reinterpret_cast<int *>(a + off[5]);
    int *item_counts = reinterpret_cast<int *>(a + off[6]);
    int *item_offsets = reinterpret_cast<int *>(a + off[7]);
    p->items = reinterpret_cast<int4 *>(a + off[8]);
    int *scan_scratch = reinterpret_cast<int *>(a + off[9]);
    int *scalars = reinterpret_cast<int *>(a + off[10]);
    p->n_items = scalars;
    p->item_counter = scalars + 1;
    p->flags = scalars + 2;
    p->kshare = scalars + 3;
    p->measured = reinterpret_cast<float2 *>(a + off[11]);
    p->gpoff = reinterpret_cast<int *>(a + off[12]);
    p->dpoff = reinterpret_cast<int *>(a + off[13]);
    p->gk2 = reinterpret_cast<float2 *>(a + off[14]);
    p->dk2 = reinterpret_cast<float2 *>(a + off[15]);
    p->geo = reinterpret_cast<uint4 *>(a + off[16]);
    uint4 *geo_tmp = reinterpret_cast<uint4 *>(a + off[17]);
    void *sort_temp = a + off[18];
    p->dinv = plan_dinv_entries(p) ? reinterpret_cast<float *>(a + off[19]) : nullptr;
    p->gbase = p->dinv ? reinterpret_cast<uint4 *>(a + off[20]) : nullptr;
    p->dk_conj_off = p->dinv ? (int)(plan_per_plane(p) * (size_t)p->dk.num_kernels) : 0;
    // sort keys: both buffers in the geo region (16 bytes per visibility),
    // written by the gather only after the sort
    unsigned long long *skeys0 = reinterpret_cast<unsigned long long *>(p->geo);
    unsigned long long *skeys1 = skeys0 + std::max(p->n, 1);
    int cbits, pbits, end_bit;
    plan_sort_bits(p, &cbits, &pbits, &end_bit);
    int os_shift = 0;
    while ((1 << os_shift) < p->geom.oversampling) ++os_shift;
    const int n = p->n;

    SDP_CUDA_TRY(cudaMemsetAsync(scalars, 0, sizeof(int) * 4, st));
    SDP_TRY(visplan_kernels(p, st));
    SDP_CUDA_TRY(cudaMemsetAsync(counts, 0, sizeof(int) * ((size_t)p->nbins + 1), st));
    if (n > 0) {
        const int2 *gs = reinterpret_cast<const int2 *>(p->gk.supports);
        const int2 *ds = reinterpret_cast<const int2 *>(p->dk.supports);
        if (p->coord_f64) {
            k_bin<double><<<(n + 255) / 256, 256, 0, st>>>(
                uvw, n, p->mode, p->snap, p->geom.grid_size, p->geom.oversampling, p->geom.uv_scale, p->geom.w_scale,
                gs, ds, p->gk.num_kernels, p->dk.num_kernels, (long long)p->gk.total_samples,
                (long long)p->dk.total_samples, p->hs_max, p->ntx, p->nty, p->tile, static_cast<Rec<double> *>(rec_tmp),
                geo_tmp, p->phase_major, os_shift, p->dinv ? p->dinv_nc : 0, p->pitch, cbits, pbits, skeys0, svals, counts,
                p->flags);
        } else {
            k_bin<float><<<(n + 255) / 256, 256, 0, st>>>(
                uvw, n, p->mode, p->snap, p->geom.grid_size, p->geom.oversampling, p->geom.uv_scale, p->geom.w_scale,
                gs, ds, p->gk.num_kernels, p->dk.num_kernels, (long long)p->gk.total_samples,
                (long long)p->dk.total_samples, p->hs_max, p->ntx, p->nty, p->tile, static_cast<Rec<float> *>(rec_tmp),
                geo_tmp, p->phase_major, os_shift, p->dinv ? p->dinv_nc : 0, p->pitch, cbits, pbits, skeys0, svals, counts,
                p->flags);
        }
        SDP_LAUNCH_CHECK();
    }
    SDP_TRY(exclusive_scan(counts, offsets, p->nbins, scan_scratch, st));
    if (n > 0) {
        // visibilities in (tile, plane, tap-box origin) order: a stable radix
        // sort of the keys with the original indices (the result lands in
        // perm); then records and geometry gathered into plan order
        cub::DoubleBuffer<unsigned long long> dk(skeys0, skeys1);
        cub::DoubleBuffer<int> dv(svals, p->perm);
        size_t temp_bytes = total - off[18];
        SDP_CUDA_TRY(cub::DeviceRadixSort::SortPairs(sort_temp, temp_bytes, dk, dv, n, 0, end_bit, st));
        if (dv.Current() != p->perm)
            SDP_CUDA_TRY(cudaMemcpyAsync(p->perm, dv.Current(), sizeof(int) * (size_t)n, cudaMemcpyDeviceToDevice, st));
        const int *n_binned = offsets + p->nbins;
        if (p->coord_f64)
            k_gather_plan<double><<<(n + 255) / 256, 256, 0, st>>>(static_cast<const Rec<double> *>(rec_tmp), geo_tmp,
                                                                   n, n_binned, p->perm,
                                                                   static_cast<Rec<double> *>(p->rec), p->geo,
                                                                   p->gbase, p->dpoff, p->dk_conj_off);
        else
            k_gather_plan<float><<<(n + 255) / 256, 256, 0, st>>>(static_cast<const Rec<float> *>(rec_tmp), geo_tmp,
                                                                  n, n_binned, p->perm,
                                                                  static_cast<Rec<float> *>(p->rec), p->geo,
                                                                  p->gbase, p->dpoff, p->dk_conj_off);
        SDP_LAUNCH_CHECK();
    }
    k_item_counts<<<(p->ntiles + 255) / 256, 256, 0, st>>>(offsets, p->ntiles, p->nk, p->chunk, item_counts);
    SDP_LAUNCH_CHECK();
    SDP_TRY(exclusive_scan(item_counts, item_offsets, p->ntiles, scan_scratch, st));
    k_item_fill<<<(p->ntiles + 255) / 256, 256, 0, st>>>(offsets, item_offsets, p->ntiles, p->nk, p->chunk,
                                                          p->items);
    SDP_LAUNCH_CHECK();
    SDP_CUDA_TRY(cudaMemcpyAsync(p->n_items, item_offsets + p->ntiles, sizeof(int), cudaMemcpyDeviceToDevice, st));
    if (n > 0) {
        const int cap = n / p->chunk + p->ntiles + 1;  // the items region's capacity
        k_batch_flags<<<(cap + 255) / 256, 256, 0, st>>>(p->items, p->n_items, cap, p->geo, p->gbase);
        SDP_LAUNCH_CHECK();
    }
    return SDP_OK;
}

int visplan_check_flags(sdp_visplan *p, cudaStream_t st)
{
    int flags = 0;
    SDP_CUDA_TRY(cudaMemcpyAsync(&flags, p->flags, sizeof(int), cudaMemcpyDeviceToHost, st));
    SDP_CUDA_TRY(cudaStreamSynchronize(st));
    if (flags) {
        SDP_CUDA_TRY(cudaMemsetAsync(p->flags, 0, sizeof(int), st));
        return set_error(SDP_ERR_DATA, "visibility data outside the kernel tables (flags 0x%x:%s%s%s%s)", flags,
                         (flags & FLAG_PLANE) ? " w-plane index beyond NUM_KERNELS;" : "",
                         (flags & FLAG_SUPPORT) ? " support beyond the declared maximum or table;" : "",
                         (flags & FLAG_BOX) ? " tap box wider than 2*hs+1;" : "",
                         (flags & FLAG_STAGE) ? " a work item's records did not arrive in shared memory;" : "");
    }
    return SDP_OK;
}

}  // namespace sdp

using namespace sdp;

SDP_EXPORT int sdp_visplan_create(sdp_visplan **out, const sdp_geometry *geom, const sdp_wkernels *gk,
                                  const sdp_wkernels *dk, int num_vis, const sdp_float3 *uvw, int grid_mode,
                                  void *stream)
{
    SDP_CHECK_ARG(out != nullptr, "plan output pointer is NULL");
    *out = nullptr;
    SDP_CHECK_ARG(num_vis == 0 || uvw != nullptr, "uvw is NULL");
    sdp_visplan *p = new sdp_visplan();
    int status = visplan_setup(p, geom, gk, dk, num_vis, grid_mode);
    if (status != SDP_OK) {
        delete p;
        return status;
    }
    void *arena = nullptr;
    cudaError_t e = cudaMalloc(&arena, visplan_arena_bytes(p));
    if (e != cudaSuccess) {
        delete p;
        return cuda_error(e, "cudaMalloc(visibility plan)");
    }
    p->owns_arena = true;
    status = visplan_build(p, arena, reinterpret_cast<const float3 *>(uvw), as_stream(stream));
    if (status != SDP_OK) {
        cudaFree(arena);
        delete p;
        return status;
    }
    *out = p;
    return SDP_OK;
}

SDP_EXPORT int sdp_visplan_create_opt(sdp_visplan **out, const sdp_geometry *geom, const sdp_wkernels *gk,
                                      const sdp_wkernels *dk, int num_vis, const sdp_float3 *uvw, int grid_mode,
                                      const sdp_plan_options *opt, void *stream)
{
    SDP_CHECK_ARG(out != nullptr, "plan output pointer is NULL");
    *out = nullptr;
    SDP_CHECK_ARG(num_vis == 0 || uvw != nullptr, "uvw is NULL");
    const int tile = (opt && opt->tile) ? opt->tile : kTile;
    const int chunk = (opt && opt->chunk) ? opt->chunk : kChunk;
    const int lanes = opt ? opt->lanes : 0;
    const int warps = opt ? opt->warps : 0;
    SDP_CHECK_ARG(tile >= 8 && tile <= 128 && tile % 8 == 0, "tile %d: a multiple of 8 in 8..128", tile);
    SDP_CHECK_ARG(chunk >= 64 && chunk <= (1 << 16), "chunk %d: 64..65536 visibilities", chunk);
    SDP_CHECK_ARG(lanes == 0 || lanes == 8 || lanes == 16 || lanes == 32, "lanes %d: 0, 8, 16 or 32", lanes);
    SDP_CHECK_ARG(warps == 0 || warps == 4 || warps == 8, "warps %d: 0, 4 or 8", warps);
    sdp_visplan *p = new sdp_visplan();
    p->tile = tile;
    p->chunk = chunk;
    p->lanes = lanes;
    p->warps = warps;
    int status = visplan_setup(p, geom, gk, dk, num_vis, grid_mode);
    if (status == SDP_OK && lanes != 0 && 2 * p->hs_max > lanes)
        status = set_error(SDP_ERR_INVALID, "lanes %d below the %d tap columns of the support", lanes,
                           2 * p->hs_max);
    if (status != SDP_OK) {
        delete p;
        return status;
    }
    void *arena = nullptr;
    cudaError_t e = cudaMalloc(&arena, visplan_arena_bytes(p));
    if (e != cudaSuccess) {
        delete p;
        return cuda_error(e, "cudaMalloc(visibility plan)");
    }
    p->owns_arena = true;
    status = visplan_build(p, arena, reinterpret_cast<const float3 *>(uvw), as_stream(stream));
    if (status != SDP_OK) {
        cudaFree(arena);
        delete p;
        return status;
    }
    *out = p;
    return SDP_OK;
}

SDP_EXPORT int sdp_visplan_options(const sdp_visplan *p, sdp_plan_options *opt)
{
    SDP_CHECK_ARG(p && opt, "NULL argument");
    opt->tile = p->tile;
    opt->chunk = p->chunk;
    opt->lanes = p->lanes;
    opt->warps = p->warps;
    return SDP_OK;
}

SDP_EXPORT int sdp_visplan_autotune(const sdp_geometry *geom, const sdp_wkernels *gk, const sdp_wkernels *dk,
                                    int num_vis, const sdp_float3 *uvw, int grid_mode, const sdp_float2 *measured,
                                    const sdp_float2 *model_grid, sdp_float2 *residual_grid, int degrid_mode,
                                    int reps, sdp_plan_options *best, float *best_ms, int *candidates,
                                    void *stream)
{
    SDP_CHECK_ARG(best && best_ms && measured && model_grid && residual_grid, "NULL argument");
    SDP_CHECK_ARG(reps >= 1 && reps <= 100, "reps %d: 1..100", reps);
    cudaStream_t st = as_stream(stream);
    // candidates: the warp-per-visibility kernel (lanes 0) over tile sides,
    // work-item sizes and warps per CTA, and two shapes of the group kernels
    struct Cand {
        int tile, chunk, lanes, warps;
    };
    std::vector<Cand> cands;
    for (int ti : {8, 16, 24, 32})
        for (int ch : {256, 512, 1024})
            for (int nw : {4, 8}) cands.push_back({ti, ch, 0, nw});
    cands.push_back({32, 512, 8, 0});
    cands.push_back({32, 1024, 16, 0});
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    SDP_CUDA_TRY(cudaEventCreate(&e0));
    cudaError_t ce = cudaEventCreate(&e1);
    if (ce != cudaSuccess) {
        cudaEventDestroy(e0);
        return cuda_error(ce, "cudaEventCreate");
    }
    float best_t = 0.f;
    int tried = 0;
    bool have = false;
    int status = SDP_OK;
    for (const Cand &cd : cands) {
                if (status != SDP_OK) break;
                sdp_plan_options o{cd.tile, cd.chunk, cd.lanes, cd.warps};
                sdp_visplan *p = nullptr;
                // candidates the device cannot hold (shared memory, lanes) are skipped
                if (sdp_visplan_create_opt(&p, geom, gk, dk, num_vis, uvw, grid_mode, &o, stream) != SDP_OK) continue;
                int s = sdp_visplan_set_measured(p, measured, stream);
                if (s == SDP_OK)
                    s = sdp_visplan_cycle(p, model_grid, degrid_mode, nullptr, nullptr, residual_grid, stream);  // warm
                float ms = 0.f;
                if (s == SDP_OK) {
                    cudaEventRecord(e0, st);
                    for (int r = 0; r < reps && s == SDP_OK; ++r)
                        s = sdp_visplan_cycle(p, model_grid, degrid_mode, nullptr, nullptr, residual_grid, stream);
                    cudaEventRecord(e1, st);
                    if (cudaEventSynchronize(e1) != cudaSuccess || cudaEventElapsedTime(&ms, e0, e1) != cudaSuccess)
                        s = SDP_ERR_CUDA;
                }
                if (s == SDP_OK) s = visplan_check_flags(p, st);
                sdp_visplan_destroy(p);
                if (s == SDP_ERR_RANGE) continue;  // the tile kernel does not fit this configuration
                if (s != SDP_OK) {
                    status = s;  // a failing pass is an error, not a slow candidate
                    break;
                }
                ms /= (float)reps;
                ++tried;
                if (!have || ms < best_t) {
                    have = true;
                    best_t = ms;
                    *best = o;
                }
            }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (status != SDP_OK) return status;
    if (!have) return set_error(SDP_ERR_RANGE, "no plan configuration fits this device");
    sdp_clear_error();
    *best_ms = best_t;
    if (candidates) *candidates = tried;
    return SDP_OK;
}

SDP_EXPORT int sdp_visplan_destroy(sdp_visplan *p)
{
    if (!p) return SDP_OK;
    if (p->arena && p->owns_arena) SDP_CUDA_TRY(cudaFree(p->arena));
    delete p;
    return SDP_OK;
}

SDP_EXPORT int sdp_visplan_num_work_items(const sdp_visplan *p, int *count)
{
    SDP_CHECK_ARG(p && count, "NULL argument");
    SDP_CUDA_TRY(cudaMemcpy(count, p->n_items, sizeof(int), cudaMemcpyDeviceToHost));
    return SDP_OK;
}

// Reads and clears the device error flags of a plan (blocking).
SDP_EXPORT int sdp_visplan_check(sdp_visplan *p, void *stream)
{
    SDP_CHECK_ARG(p, "plan is NULL");
    return visplan_check_flags(p, as_stream(stream));
}

SDP_EXPORT int sdp_visplan_set_measured(sdp_visplan *p, const sdp_float2 *measured, void *stream)
{
    SDP_CHECK_ARG(p && (measured || p->n == 0), "NULL argument");
    if (p->n == 0) return SDP_OK;
    k_gather_sorted<<<(p->n + 255) / 256, 256, 0, as_stream(stream)>>>(reinterpret_cast<const float2 *>(measured),
                                                                      p->perm, p->n, p->measured);
    SDP_LAUNCH_CHECK();
    return SDP_OK;
}

namespace sdp {

template <typename T, int LG>
static int launch_tiles_lg(sdp_visplan *p, int op, const float2 *vis_in, const float2 *in_grid, float2 *out_grid,
                           float2 *pred, float2 *delta, cudaStream_t st)
{
    PlanDev d = plan_dev(p);
    const size_t SS = (size_t)p->S * p->S;
    const size_t smem = sizeof(float2) * SS * ((op != OP_GRID ? 1 : 0) + (op != OP_DEGRID ? 1 : 0)) +
                        sizeof(int4) * (size_t)p->gk.num_kernels;
    void (*fn)(PlanDev, const float2 *, const float2 *, float2 *, float2 *, float2 *, const float2 *) = nullptr;
    const bool snapped = (p->mode == SDP_GRID_SNAPPED);
    switch (op) {
    case OP_GRID: fn = snapped ? k_tiles<T, SDP_GRID_SNAPPED, OP_GRID, LG> : k_tiles<T, SDP_GRID_STD, OP_GRID, LG>; break;
    case OP_DEGRID: fn = k_tiles<T, SDP_GRID_STD, OP_DEGRID, LG>; break;
    case OP_CYCLE_CONV: fn = k_tiles<T, SDP_GRID_STD, OP_CYCLE_CONV, LG>; break;
    case OP_CYCLE_NEAR: fn = k_tiles<T, SDP_GRID_STD, OP_CYCLE_NEAR, LG>; break;
    case OP_G2G: fn = k_tiles<T, SDP_GRID_STD, OP_G2G, LG>; break;
    default: return set_error(SDP_ERR_INVALID, "internal: op %d", op);
    }
    if (smem + kStaticSmem > 48 * 1024) SDP_CUDA_TRY(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    int per_sm = 0;
    SDP_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, kThreads, smem));
    if (per_sm < 1) return set_error(SDP_ERR_RANGE, "tile kernel does not fit (%zu B shared memory)", smem);
    SDP_CUDA_TRY(cudaMemsetAsync(p->item_counter, 0, sizeof(int), st));
    fn<<<per_sm * num_sms(), kThreads, smem, st>>>(d, vis_in, in_grid, out_grid, pred, delta, p->measured);
    SDP_LAUNCH_CHECK();
    return SDP_OK;
}

// The warp-per-visibility kernels serve std_gridding plans with half
// supports 1..4 (boxes of at most 8 x 8 taps) unless the plan asks for the
// group kernels (lanes != 0).
static bool fast_eligible(const sdp_visplan *p)
{
    return p->mode == SDP_GRID_STD && p->lanes == 0 && p->hs_max >= 1 && p->hs_max <= 4 &&
           fast_smem_bytes(OP_CYCLE_CONV, 4, p->S, p->pitch, p->gk.num_kernels, p->chunk) + kStaticSmem <= kSmemOptin;
}

template <typename T, int OP, int NW>
static int launch_fast_nw(sdp_visplan *p, const float2 *vis_in, const float2 *in_grid, float2 *out_grid,
                          float2 *pred, float2 *delta, cudaStream_t st, int *resident_warps)
{
    const size_t smem = fast_smem_bytes(OP, NW, p->S, p->pitch, p->gk.num_kernels, p->chunk);
    void (*fn)(PlanDev, const float2 *, const float2 *, float2 *, float2 *, float2 *, const float2 *) =
        k_vis_fast<T, OP, NW>;
    if (smem + kStaticSmem > kSmemOptin) {
        if (resident_warps) {
            *resident_warps = 0;
            return SDP_OK;
        }
        return set_error(SDP_ERR_RANGE, "tile kernel does not fit (%zu B shared memory)", smem);
    }
    if (smem + kStaticSmem > 48 * 1024) SDP_CUDA_TRY(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    int per_sm = 0;
    SDP_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, 32 * NW, smem));
    if (resident_warps) {  // query only
        *resident_warps = per_sm * NW;
        return SDP_OK;
    }
    if (per_sm < 1) return set_error(SDP_ERR_RANGE, "tile kernel does not fit (%zu B shared memory)", smem);
    PlanDev d = plan_dev(p);
    SDP_CUDA_TRY(cudaMemsetAsync(p->item_counter, 0, sizeof(int), st));
    fn<<<per_sm * num_sms(), 32 * NW, smem, st>>>(d, vis_in, in_grid, out_grid, pred, delta, p->measured);
    SDP_LAUNCH_CHECK();
    return SDP_OK;
}

template <typename T, int OP>
static int launch_fast_op(sdp_visplan *p, const float2 *vis_in, const float2 *in_grid, float2 *out_grid,
                          float2 *pred, float2 *delta, cudaStream_t st)
{
    int nw = p->warps;
    if (nw == 0) {  // the shape that keeps more warps resident (8 on a tie)
        int w4 = 0, w8 = 0;
        SDP_TRY((launch_fast_nw<T, OP, 4>(p, vis_in, in_grid, out_grid, pred, delta, st, &w4)));
        SDP_TRY((launch_fast_nw<T, OP, 8>(p, vis_in, in_grid, out_grid, pred, delta, st, &w8)));
        nw = (w4 > w8) ? 4 : 8;
    }
    if (nw == 4) return launch_fast_nw<T, OP, 4>(p, vis_in, in_grid, out_grid, pred, delta, st, nullptr);
    return launch_fast_nw<T, OP, 8>(p, vis_in, in_grid, out_grid, pred, delta, st, nullptr);
}

template <typename T>
static int launch_fast(sdp_visplan *p, int op, const float2 *vis_in, const float2 *in_grid, float2 *out_grid,
                       float2 *pred, float2 *delta, cudaStream_t st)
{
    switch (op) {
    case OP_GRID: return launch_fast_op<T, OP_GRID>(p, vis_in, in_grid, out_grid, pred, delta, st);
    case OP_DEGRID: return launch_fast_op<T, OP_DEGRID>(p, vis_in, in_grid, out_grid, pred, delta, st);
    case OP_CYCLE_CONV: return launch_fast_op<T, OP_CYCLE_CONV>(p, vis_in, in_grid, out_grid, pred, delta, st);
    default: return set_error(SDP_ERR_INVALID, "internal: op %d", op);
    }
}

static int launch_tiles(sdp_visplan *p, int op, const float2 *vis_in, const float2 *in_grid, float2 *out_grid,
                        float2 *pred, float2 *delta, cudaStream_t st)
{
    if (fast_eligible(p) && (op == OP_GRID || op == OP_DEGRID || op == OP_CYCLE_CONV)) {
        if (p->coord_f64) return launch_fast<double>(p, op, vis_in, in_grid, out_grid, pred, delta, st);
        return launch_fast<float>(p, op, vis_in, in_grid, out_grid, pred, delta, st);
    }
    // lanes per visibility: the tap columns (2 hs + 1 at most) in at most two
    // passes; a plan may ask for more lanes than its support needs
    if (p->lanes == 16 && 2 * p->hs_max <= 16) {
        if (p->coord_f64) return launch_tiles_lg<double, 16>(p, op, vis_in, in_grid, out_grid, pred, delta, st);
        return launch_tiles_lg<float, 16>(p, op, vis_in, in_grid, out_grid, pred, delta, st);
    }
    if (p->lanes == 32) {
        if (p->coord_f64) return launch_tiles_lg<double, 32>(p, op, vis_in, in_grid, out_grid, pred, delta, st);
        return launch_tiles_lg<float, 32>(p, op, vis_in, in_grid, out_grid, pred, delta, st);
    }
    if (p->coord_f64) {
        if (2 * p->hs_max <= 8) return launch_tiles_lg<double, 8>(p, op, vis_in, in_grid, out_grid, pred, delta, st);
        if (2 * p->hs_max <= 16) return launch_tiles_lg<double, 16>(p, op, vis_in, in_grid, out_grid, pred, delta, st);
        return launch_tiles_lg<double, 32>(p, op, vis_in, in_grid, out_grid, pred, delta, st);
    }
    if (2 * p->hs_max <= 8) return launch_tiles_lg<float, 8>(p, op, vis_in, in_grid, out_grid, pred, delta, st);
    if (2 * p->hs_max <= 16) return launch_tiles_lg<float, 16>(p, op, vis_in, in_grid, out_grid, pred, delta, st);
    return launch_tiles_lg<float, 32>(p, op, vis_in, in_grid, out_grid, pred, delta, st);
}

}  // namespace sdp

SDP_EXPORT int sdp_visplan_grid(sdp_visplan *p, const sdp_float2 *vis, sdp_float2 *grid, int accumulate, void *stream)
{
    SDP_CHECK_ARG(p && grid && (vis || p->n == 0), "NULL argument");
    SDP_CHECK_ARG(p->mode != kPlanG2G, "plan was built for g2g; use sdp_visplan_g2g");
    cudaStream_t st = as_stream(stream);
    const size_t G2 = (size_t)p->geom.grid_size * p->geom.grid_size;
    if (!accumulate) SDP_CUDA_TRY(cudaMemsetAsync(grid, 0, sizeof(float2) * G2, st));
    if (p->n == 0) return SDP_OK;
    return launch_tiles(p, OP_GRID, reinterpret_cast<const float2 *>(vis), nullptr, reinterpret_cast<float2 *>(grid),
                        nullptr, nullptr, st);
}

SDP_EXPORT int sdp_visplan_degrid(sdp_visplan *p, const sdp_float2 *model_grid, sdp_float2 *predicted, int mode,
                                  void *stream)
{
    SDP_CHECK_ARG(p && model_grid && (predicted || p->n == 0), "NULL argument");
    cudaStream_t st = as_stream(stream);
    if (p->n == 0) return SDP_OK;
    if (mode == SDP_DEGRID_NEAREST) {
        return set_error(SDP_ERR_INVALID, "nearest degridding needs no plan: use sdp_degrid_nearest");
    }
    SDP_CHECK_ARG(mode == SDP_DEGRID_CONV, "degrid mode %d unknown", mode);
    // visibilities dropped by binning (invalid plane) keep 0
    SDP_CUDA_TRY(cudaMemsetAsync(predicted, 0, sizeof(float2) * (size_t)p->n, st));
    return launch_tiles(p, OP_DEGRID, nullptr, reinterpret_cast<const float2 *>(model_grid), nullptr,
                        reinterpret_cast<float2 *>(predicted), nullptr, st);
}

SDP_EXPORT int sdp_visplan_cycle(sdp_visplan *p, const sdp_float2 *model_grid, int degrid_mode,
                                 sdp_float2 *predicted, sdp_float2 *delta, sdp_float2 *residual_grid, void *stream)
{
    SDP_CHECK_ARG(p && model_grid && residual_grid, "NULL argument");
    SDP_CHECK_ARG(p->mode == SDP_GRID_STD, "the major-cycle pass needs a std_gridding plan");
    SDP_CHECK_ARG(degrid_mode == SDP_DEGRID_NEAREST || degrid_mode == SDP_DEGRID_CONV, "degrid mode %d unknown",
                  degrid_mode);
    cudaStream_t st = as_stream(stream);
    const size_t G2 = (size_t)p->geom.grid_size * p->geom.grid_size;
    SDP_CUDA_TRY(cudaMemsetAsync(residual_grid, 0, sizeof(float2) * G2, st));
    if (p->n == 0) return SDP_OK;
    return launch_tiles(p, degrid_mode == SDP_DEGRID_CONV ? OP_CYCLE_CONV : OP_CYCLE_NEAR, nullptr,
                        reinterpret_cast<const float2 *>(model_grid), reinterpret_cast<float2 *>(residual_grid),
                        reinterpret_cast<float2 *>(predicted), reinterpret_cast<float2 *>(delta), st);
}

SDP_EXPORT int sdp_visplan_g2g(sdp_visplan *p, const sdp_float2 *in_grid, sdp_float2 *out_grid, void *stream)
{
    SDP_CHECK_ARG(p && in_grid && out_grid, "NULL argument");
    SDP_CHECK_ARG(p->mode == kPlanG2G, "plan was not built for g2g");
    cudaStream_t st = as_stream(stream);
    const size_t G2 = (size_t)p->geom.grid_size * p->geom.grid_size;
    SDP_CUDA_TRY(cudaMemsetAsync(out_grid, 0, sizeof(float2) * G2, st));
    if (p->n == 0) return SDP_OK;
    return launch_tiles(p, OP_G2G, nullptr, reinterpret_cast<const float2 *>(in_grid),
                        reinterpret_cast<float2 *>(out_grid), nullptr, nullptr, st);
}

// ----------------------------------------------------------------------------
// Batches of plans (frequency channels) in one launch
// ----------------------------------------------------------------------------
struct sdp_visbatch {
    int n = 0;
    bool f64 = false;
    bool fast = true;  // every plan takes the warp-per-visibility kernel
    int warps = 0;
    int hs_max = 0, S_max = 0, nk_max = 0, n_items = 0;
    size_t tile_f2 = 0;  // largest S x pitch of the plans
    int chunk_max = 0;   // largest work item of the plans
    std::vector<sdp_visplan *> plans;
    std::vector<sdp::BatchIO> io;
    sdp::PlanDev *d_plans = nullptr;
    sdp::BatchIO *d_io = nullptr;
    int4 *d_items = nullptr;
    int *d_counter = nullptr;
    bool io_set = false;
};

namespace sdp {

template <typename T, int LG>
static int launch_batch_lg(sdp_visbatch *b, int op, cudaStream_t st)
{
    const size_t SS = (size_t)b->S_max * b->S_max;
    const int stride = (int)(4 * SS);  // floats: model tile (2 SS) + subgrid (2 SS) of the widest channel
    const size_t smem = sizeof(float) * (size_t)stride + sizeof(int4) * (size_t)b->nk_max;
    void (*fn)(const PlanDev *, const BatchIO *, const int4 *, int, int *, int) =
        op == OP_CYCLE_CONV ? k_tiles_batch<T, SDP_GRID_STD, OP_CYCLE_CONV, LG>
                            : k_tiles_batch<T, SDP_GRID_STD, OP_CYCLE_NEAR, LG>;
    if (smem + kStaticSmem > 48 * 1024) SDP_CUDA_TRY(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    int per_sm = 0;
    SDP_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, kThreads, smem));
    if (per_sm < 1) return set_error(SDP_ERR_RANGE, "batched tile kernel does not fit (%zu B shared memory)", smem);
    SDP_CUDA_TRY(cudaMemsetAsync(b->d_counter, 0, sizeof(int), st));
    fn<<<per_sm * num_sms(), kThreads, smem, st>>>(b->d_plans, b->d_io, b->d_items, b->n_items, b->d_counter,
                                                   stride);
    SDP_LAUNCH_CHECK();
    return SDP_OK;
}

template <typename T, int NW>
static int launch_batch_fast_nw(sdp_visbatch *b, cudaStream_t st, int *resident_warps)
{
    const size_t smem = fast_stage_bytes(b->chunk_max) + 16 * (size_t)b->nk_max + 8 * b->tile_f2 * (1 + NW);
    void (*fn)(const PlanDev *, const BatchIO *, const int4 *, int, int *, int, int, int) = k_vis_fast_batch<T, NW>;
    if (smem + kStaticSmem > kSmemOptin) {
        if (resident_warps) {
            *resident_warps = 0;
            return SDP_OK;
        }
        return set_error(SDP_ERR_RANGE, "batched tile kernel does not fit (%zu B shared memory)", smem);
    }
    if (smem + kStaticSmem > 48 * 1024) SDP_CUDA_TRY(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    int per_sm = 0;
    SDP_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, 32 * NW, smem));
    if (resident_warps) {
        *resident_warps = per_sm * NW;
        return SDP_OK;
    }
    if (per_sm < 1) return set_error(SDP_ERR_RANGE, "batched tile kernel does not fit (%zu B shared memory)", smem);
    SDP_CUDA_TRY(cudaMemsetAsync(b->d_counter, 0, sizeof(int), st));
    fn<<<per_sm * num_sms(), 32 * NW, smem, st>>>(b->d_plans, b->d_io, b->d_items, b->n_items, b->d_counter,
                                                  b->nk_max, (int)b->tile_f2, b->chunk_max);
    SDP_LAUNCH_CHECK();
    return SDP_OK;
}

template <typename T>
static int launch_batch_fast(sdp_visbatch *b, cudaStream_t st)
{
    int nw = b->warps;
    if (nw == 0) {
        int w4 = 0, w8 = 0;
        SDP_TRY((launch_batch_fast_nw<T, 4>(b, st, &w4)));
        SDP_TRY((launch_batch_fast_nw<T, 8>(b, st, &w8)));
        nw = (w4 > w8) ? 4 : 8;
    }
    if (nw == 4) return launch_batch_fast_nw<T, 4>(b, st, nullptr);
    return launch_batch_fast_nw<T, 8>(b, st, nullptr);
}

}  // namespace sdp

static void visbatch_free(sdp_visbatch *b)
{
    if (!b) return;
    cudaFree(b->d_plans);
    cudaFree(b->d_io);
    cudaFree(b->d_items);
    cudaFree(b->d_counter);
    delete b;
}

SDP_EXPORT int sdp_visbatch_create(sdp_visbatch **out, sdp_visplan *const *plans, int num_plans, void *stream)
{
    SDP_CHECK_ARG(out && plans && num_plans >= 1, "bad argument");
    *out = nullptr;
    cudaStream_t st = as_stream(stream);
    sdp_visbatch *b = new sdp_visbatch();
    b->n = num_plans;
    b->f64 = plans[0] && plans[0]->coord_f64;
    std::vector<PlanDev> devs;
    std::vector<int4> items;
    for (int c = 0; c < num_plans; ++c) {
        sdp_visplan *p = plans[c];
        if (!p || p->mode != SDP_GRID_STD || p->coord_f64 != b->f64) {
            visbatch_free(b);
            return set_error(SDP_ERR_INVALID, "plan %d: a batch holds std_gridding plans of one coordinate mode", c);
        }
        b->plans.push_back(p);
        devs.push_back(plan_dev(p));
        b->hs_max = std::max(b->hs_max, p->hs_max);
        b->S_max = std::max(b->S_max, p->S);
        b->tile_f2 = std::max(b->tile_f2, (size_t)p->S * p->pitch);
        b->chunk_max = std::max(b->chunk_max, p->chunk);
        b->fast = b->fast && fast_eligible(p);
        if (b->fast && p->gbase) {
            // the batched warp-per-visibility kernel assumes each plan's two
            // kernel sets are equal or conjugate (kShared in fast_item)
            int kdiff = 3;
            cudaError_t e = cudaMemcpyAsync(&kdiff, p->kshare, sizeof(int), cudaMemcpyDeviceToHost, st);
            if (e == cudaSuccess) e = cudaStreamSynchronize(st);
            if (e != cudaSuccess) {
                visbatch_free(b);
                return cuda_error(e, "reading a plan's kernel-set relation");
            }
            if ((kdiff & 1) && (kdiff & 2)) b->fast = false;
        }
        if (c == 0) b->warps = p->warps;
        b->nk_max = std::max(b->nk_max, p->gk.num_kernels);
        int ni = 0;
        cudaError_t e = cudaMemcpyAsync(&ni, p->n_items, sizeof(int), cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        if (e != cudaSuccess) {
            visbatch_free(b);
            return cuda_error(e, "reading a plan's work-item count");
        }
        std::vector<int4> pi((size_t)ni);
        if (ni > 0) {
            e = cudaMemcpy(pi.data(), p->items, sizeof(int4) * (size_t)ni, cudaMemcpyDeviceToHost);
            if (e != cudaSuccess) {
                visbatch_free(b);
                return cuda_error(e, "reading a plan's work items");
            }
        }
        for (int4 it : pi) items.push_back(make_int4(it.x, it.y, it.z, c));
    }
    // the batched kernel holds the largest channel's tiles and work item
    if (b->fast && fast_stage_bytes(b->chunk_max) + 16 * (size_t)b->nk_max + 8 * b->tile_f2 * (1 + 4) + kStaticSmem >
                       kSmemOptin)
        b->fast = false;
    b->n_items = (int)items.size();
    b->io.resize((size_t)num_plans);
    cudaError_t e = cudaMalloc(&b->d_plans, sizeof(PlanDev) * devs.size());
    if (e == cudaSuccess) e = cudaMalloc(&b->d_io, sizeof(BatchIO) * (size_t)num_plans);
    if (e == cudaSuccess) e = cudaMalloc(&b->d_items, sizeof(int4) * std::max<size_t>(items.size(), 1));
    if (e == cudaSuccess) e = cudaMalloc(&b->d_counter, sizeof(int));
    if (e == cudaSuccess) e = cudaMemcpy(b->d_plans, devs.data(), sizeof(PlanDev) * devs.size(), cudaMemcpyHostToDevice);
    if (e == cudaSuccess && !items.empty())
        e = cudaMemcpy(b->d_items, items.data(), sizeof(int4) * items.size(), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) {
        visbatch_free(b);
        return cuda_error(e, "visibility batch set-up");
    }
    *out = b;
    return SDP_OK;
}

SDP_EXPORT int sdp_visbatch_set_grids(sdp_visbatch *b, const sdp_float2 *const *model_grids,
                                      sdp_float2 *const *residual_grids, void *stream)
{
    SDP_CHECK_ARG(b && model_grids && residual_grids, "NULL argument");
    for (int c = 0; c < b->n; ++c) {
        SDP_CHECK_ARG(model_grids[c] && residual_grids[c], "channel %d: NULL grid", c);
        b->io[(size_t)c] = BatchIO{reinterpret_cast<const float2 *>(model_grids[c]),
                                   reinterpret_cast<float2 *>(residual_grids[c]), b->plans[(size_t)c]->measured,
                                   nullptr, nullptr};
    }
    cudaStream_t st = as_stream(stream);
    SDP_CUDA_TRY(cudaMemcpyAsync(b->d_io, b->io.data(), sizeof(BatchIO) * (size_t)b->n, cudaMemcpyHostToDevice, st));
    SDP_CUDA_TRY(cudaStreamSynchronize(st));  // the host array may change after return
    b->io_set = true;
    return SDP_OK;
}

SDP_EXPORT int sdp_visbatch_cycle(sdp_visbatch *b, int degrid_mode, void *stream)
{
    SDP_CHECK_ARG(b, "batch is NULL");
    SDP_CHECK_ARG(b->io_set, "sdp_visbatch_set_grids was not called");
    SDP_CHECK_ARG(degrid_mode == SDP_DEGRID_NEAREST || degrid_mode == SDP_DEGRID_CONV, "degrid mode %d unknown",
                  degrid_mode);
    cudaStream_t st = as_stream(stream);
    for (int c = 0; c < b->n; ++c) {
        const size_t G2 = (size_t)b->plans[(size_t)c]->geom.grid_size * b->plans[(size_t)c]->geom.grid_size;
        SDP_CUDA_TRY(cudaMemsetAsync(b->io[(size_t)c].out_grid, 0, sizeof(float2) * G2, st));
    }
    if (b->n_items == 0) return SDP_OK;
    const int op = degrid_mode == SDP_DEGRID_CONV ? OP_CYCLE_CONV : OP_CYCLE_NEAR;
    if (op == OP_CYCLE_CONV && b->fast) return b->f64 ? launch_batch_fast<double>(b, st) : launch_batch_fast<float>(b, st);
    const int taps = 2 * b->hs_max;
    if (b->f64) {
        if (taps <= 8) return launch_batch_lg<double, 8>(b, op, st);
        if (taps <= 16) return launch_batch_lg<double, 16>(b, op, st);
        return launch_batch_lg<double, 32>(b, op, st);
    }
    if (taps <= 8) return launch_batch_lg<float, 8>(b, op, st);
    if (taps <= 16) return launch_batch_lg<float, 16>(b, op, st);
    return launch_batch_lg<float, 32>(b, op, st);
}

SDP_EXPORT int sdp_visbatch_num_work_items(const sdp_visbatch *b, int *count)
{
    SDP_CHECK_ARG(b && count, "NULL argument");
    *count = b->n_items;
    return SDP_OK;
}

SDP_EXPORT int sdp_visbatch_destroy(sdp_visbatch *b)
{
    visbatch_free(b);
    return SDP_OK;
}
