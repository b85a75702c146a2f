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
// B200 design.  Visibilities are binned once per uvw set by the 32 x 32 uv
// tile holding the origin of their tap box, then by w-plane, with a
// counting sort.  Each tile's list is cut into work items of at most
// kChunk visibilities; persistent CTAs pull items from an atomic queue.  A
// CTA keeps one (32 + 2 hs_max)^2 complex subgrid per warp in shared memory,
// so a warp updates its subgrid with plain loads and stores (the lanes of a
// warp always touch distinct cells of one visibility), and flushes the sum of
// its warps' subgrids to HBM with one vector atomic per touched cell.  A
// visibility's tap box is mapped onto lanes as (column = lane % W, row phase =
// lane / W), W = 2 hs_max + 1, so a lane computes its column's kernel index
// once per visibility and walks rows.
#include <cstdio>
#include <cstring>

#include <algorithm>

#include "internal.cuh"

namespace sdp {

constexpr int kTile = 32;
constexpr int kChunk = 1024;
constexpr int kWarps = 4;          // warps per CTA of the tile kernels
constexpr int kMaxHalfSupport = 15;

enum : int {
    OP_GRID = 0,         // grid vis (original order) into grid
    OP_DEGRID = 1,       // convolutional degrid into predicted
    OP_CYCLE_CONV = 2,   // degrid (conv) -> subtract -> grid
    OP_CYCLE_NEAR = 3,   // degrid (nearest) -> subtract -> grid
    OP_G2G = 4           // nearest sample of in_grid regridded (w = 0 plane)
};

// Device-side error flags (OR-ed together).
enum : int { FLAG_PLANE = 1, FLAG_SUPPORT = 2, FLAG_BOX = 4 };

struct PlanDev {
    int G, gc, OS, nk_g, nk_d, ntx, nty, W, S;
    double uv_scale, w_scale;
    const float2 *gk;  // gridding kernels
    const int2 *gs;    // gridding supports
    const float2 *dk;  // degridding kernels
    const int2 *ds;    // degridding supports
    const VisRec *rec; // plan order
    const int4 *items; // (tile, begin, end, -)
    const int *n_items;
    int *item_counter;
    int *flags;
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
// Binning
// ----------------------------------------------------------------------------
__device__ __forceinline__ int floor_div(int a, int b) { return (a >= 0) ? a / b : -((-a + b - 1) / b); }

// Computes the record of each visibility and its bin key.
__global__ void k_bin(const float3 *__restrict__ uvw, int n, int mode, int G, int OS, double uv_scale,
                      double w_scale, const int2 *__restrict__ sup, const int2 *__restrict__ dsup, int nk, int nkd,
                      long long ntot_g, long long ntot_d, int hs_max, int ntx, int nty, VisRec *__restrict__ rec_tmp,
                      int *__restrict__ keys, int *__restrict__ counts, int *__restrict__ flags)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float3 c = uvw[i];
    VisRec r;
    r.px = ref_grid_pos(c.x, uv_scale);
    r.py = ref_grid_pos(c.y, uv_scale);
    int plane;
    if (mode == SDP_GRID_SNAPPED) {
        plane = ref_widx_round(c.z, w_scale);
        r.px = ref_snap(r.px, OS);
        r.py = ref_snap(r.py, OS);
    } else if (mode == kPlanG2G) {  // g2g: plane forced to 0 (degridgrid.c:215)
        plane = 0;
    } else {
        plane = ref_widx_std(c.z, w_scale);
    }
    r.meta = plane | ((c.z < 0.0f) ? (int)0x80000000u : 0);
    r.idx = i;
    int key = -1;
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
            int lox = (int)ceilf(__fsub_rn(r.px, (float)hs)) + G / 2;
            int loy = (int)ceilf(__fsub_rn(r.py, (float)hs)) + G / 2;
            int tx = min(max(floor_div(lox, kTile), 0), ntx - 1);
            int ty = min(max(floor_div(loy, kTile), 0), nty - 1);
            key = (ty * ntx + tx) * nk + plane;
            atomicAdd(&counts[key], 1);
        }
    }
    rec_tmp[i] = r;
    keys[i] = key;
}

__global__ void k_scatter(const VisRec *__restrict__ rec_tmp, const int *__restrict__ keys, int n,
                          const int *__restrict__ offsets, int *__restrict__ fill, VisRec *__restrict__ rec,
                          int *__restrict__ perm)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    int key = keys[i];
    if (key < 0) return;
    int pos = offsets[key] + atomicAdd(&fill[key], 1);
    rec[pos] = rec_tmp[i];
    perm[pos] = i;
}

__global__ void k_item_counts(const int *__restrict__ offsets, int ntiles, int nk, int *__restrict__ item_counts)
{
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= ntiles) return;
    int b = offsets[t * nk], e = offsets[(t + 1) * nk];
    item_counts[t] = (e - b + kChunk - 1) / kChunk;
}

__global__ void k_item_fill(const int *__restrict__ offsets, const int *__restrict__ item_offsets, int ntiles,
                            int nk, int4 *__restrict__ items)
{
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= ntiles) return;
    int b = offsets[t * nk], e = offsets[(t + 1) * nk];
    int o = item_offsets[t];
    for (int s = b; s < e; s += kChunk) items[o++] = make_int4(t, s, min(e, s + kChunk), 0);
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

template <int GMODE, int OP>
__global__ void __launch_bounds__(kWarps * 32) k_tiles(PlanDev P, const float2 *__restrict__ vis_in,
                                                      const float2 *__restrict__ in_grid,
                                                      float2 *__restrict__ out_grid, float2 *__restrict__ pred_out,
                                                      float2 *__restrict__ delta_out,
                                                      const float2 *__restrict__ measured)
{
    extern __shared__ float2 smem[];
    constexpr bool kGrids = (OP != OP_DEGRID);
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    const int W = P.W, S = P.S, SS = S * S;
    float2 *sub = smem + (size_t)warp * SS;
    // lane -> (column, row phase) of the W x W tap box
    const int R = 32 / W;  // rows handled in parallel
    const int col = lane % W;
    const int row0 = lane / W;
    const bool lane_active = row0 < R;
    const float fos = (float)P.OS;
    __shared__ int s_item;

    for (;;) {
        if (threadIdx.x == 0) s_item = atomicAdd(P.item_counter, 1);
        __syncthreads();
        const int item = s_item;
        if (item >= *P.n_items) break;
        const int4 it = P.items[item];
        const int tile = it.x;
        const int ox = (tile % P.ntx) * kTile;  // subgrid origin in grid cells
        const int oy = (tile / P.ntx) * kTile;
        if (kGrids) {
            for (int k = lane; k < SS; k += 32) sub[k] = make_float2(0.f, 0.f);
            __syncwarp();
        }
        // contiguous slice of the item per warp (keeps w-plane runs together)
        const int len = it.z - it.y;
        const int per = (len + kWarps - 1) / kWarps;
        const int b = it.y + warp * per;
        const int e = min(it.z, b + per);
        for (int r = b; r < e; ++r) {
            const VisRec rec = P.rec[r];
            const int plane = rec.meta & 0xffff;
            const float conj = (rec.meta < 0) ? -1.f : 1.f;

            // ---------------- degrid (prediction) ----------------
            float2 value = make_float2(0.f, 0.f);
            if (OP == OP_DEGRID || OP == OP_CYCLE_CONV) {
                const int2 sp = P.ds[plane];
                const int hs = sp.x;
                const int stride = (hs + 1) * P.OS;
                const float lox = ceilf(__fsub_rn(rec.px, (float)hs));
                const float hix = ceilf(__fadd_rn(rec.px, (float)hs));
                const float loy = ceilf(__fsub_rn(rec.py, (float)hs));
                const float hiy = ceilf(__fadd_rn(rec.py, (float)hs));
                float2 acc = make_float2(0.f, 0.f);
                float nrm = 0.f;
                const int u = (int)lox + col;
                if (lane_active && (float)u < hix) {
                    const int cu = mirror(u, P.gc);
                    const int kx = ref_kidx(cu, rec.px, fos);
                    for (int rr = row0; rr < W; rr += R) {
                        const int v = (int)loy + rr;
                        if (!((float)v < hiy)) break;
                        const int cv = mirror(v, P.gc);
                        const int ky = ref_kidx(cv, rec.py, fos);
                        float2 ks = make_float2(0.f, 0.f);
                        if (kx < stride && ky < stride) ks = __ldg(&P.dk[sp.y + ky * stride + kx]);
                        ks.y *= conj;
                        float2 gv = make_float2(0.f, 0.f);
                        const int gx = cu + P.gc, gy = cv + P.gc;
                        if (gx >= 0 && gy >= 0 && gx < P.G && gy < P.G) gv = __ldg(&in_grid[(size_t)gy * P.G + gx]);
                        cmac(acc, gv, ks);
                        nrm = fmaf(ks.x, ks.x, fmaf(ks.y, ks.y, nrm));
                    }
                }
#pragma unroll
                for (int o = 16; o > 0; o >>= 1) {
                    acc.x += __shfl_xor_sync(0xffffffffu, acc.x, o);
                    acc.y += __shfl_xor_sync(0xffffffffu, acc.y, o);
                    nrm += __shfl_xor_sync(0xffffffffu, nrm, o);
                }
                // degridgrid.c:188-191 (the .y fallback uses the new .x)
                const float cn = __fsqrt_rn(nrm);
                const float nx = (cn < 1e-5f) ? __fdiv_rn(acc.x, 1e-5f) : __fdiv_rn(acc.x, cn);
                const float ny = (cn < 1e-5f) ? __fdiv_rn(nx, 1e-5f) : __fdiv_rn(acc.y, cn);
                value = make_float2(nx, ny);
            } else if (OP == OP_CYCLE_NEAR || OP == OP_G2G) {
                // degridgrid.c:194-200 / :273-285
                const int x = ref_nearest(rec.px, P.gc), y = ref_nearest(rec.py, P.gc);
                const long long gi = (long long)x + (long long)y * P.G;
                if (gi >= 0 && gi < (long long)P.G * P.G) value = __ldg(&in_grid[gi]);
            }

            float2 gval;
            if (OP == OP_GRID) {
                gval = __ldg(&vis_in[rec.idx]);
            } else if (OP == OP_G2G) {
                gval = value;
            } else if (OP == OP_CYCLE_CONV || OP == OP_CYCLE_NEAR) {
                const float2 m = measured[r];
                gval = make_float2(__fsub_rn(m.x, value.x), __fsub_rn(m.y, value.y));
                if (lane == 0) {
                    if (pred_out) pred_out[rec.idx] = value;
                    if (delta_out) delta_out[rec.idx] = gval;
                }
            } else {  // OP_DEGRID
                if (lane == 0) pred_out[rec.idx] = value;
            }

            // ---------------- grid ----------------
            if (kGrids) {
                const int2 sp = P.gs[plane];
                const int hs = sp.x;
                const int stride = (hs + 1) * P.OS;
                const float lox = ceilf(__fsub_rn(rec.px, (float)hs));
                const float loy = ceilf(__fsub_rn(rec.py, (float)hs));
                float hix, hiy;
                if (GMODE == SDP_GRID_SNAPPED) {  // inclusive floor bound
                    hix = floorf(__fadd_rn(rec.px, (float)hs)) + 0.5f;
                    hiy = floorf(__fadd_rn(rec.py, (float)hs)) + 0.5f;
                } else {
                    hix = ceilf(__fadd_rn(rec.px, (float)hs));
                    hiy = ceilf(__fadd_rn(rec.py, (float)hs));
                }
                const int u = (int)lox + col;
                const int gx = u + P.gc;
                if (lane_active && (float)u < hix && gx >= 0 && gx < P.G) {
                    const int kx = ref_kidx(u, rec.px, fos);
                    const int lx = gx - ox;
                    for (int rr = row0; rr < W; rr += R) {
                        const int v = (int)loy + rr;
                        if (!((float)v < hiy)) break;
                        const int gy = v + P.gc;
                        if (gy < 0 || gy >= P.G) continue;
                        const int ky = ref_kidx(v, rec.py, fos);
                        float2 ks = __ldg(&P.gk[sp.y + ky * stride + kx]);
                        ks.y *= conj;
                        float2 &cell = sub[(gy - oy) * S + lx];
                        float2 acc = cell;
                        cmac(acc, gval, ks);
                        cell = acc;
                    }
                }
                if (lane == 0) {
                    // a box wider than W would lose taps: flag it
                    if ((float)((int)lox + W) < hix || (float)((int)loy + W) < hiy) atomicOr(P.flags, FLAG_BOX);
                }
                __syncwarp();
            }
        }
        if (kGrids) {
            __syncthreads();
            // flush: sum the warps' subgrids, one vector atomic per touched cell
            for (int k = threadIdx.x; k < SS; k += blockDim.x) {
                float2 s = smem[k];
#pragma unroll
                for (int w = 1; w < kWarps; ++w) {
                    float2 t = smem[(size_t)w * SS + k];
                    s.x += t.x;
                    s.y += t.y;
                }
                if (s.x != 0.f || s.y != 0.f) {
                    const int gy = oy + k / S, gx = ox + k % S;
                    if (gx < P.G && gy < P.G) atomicAdd(&out_grid[(size_t)gy * P.G + gx], s);
                }
            }
        }
        __syncthreads();
    }
}

__global__ void k_gather_sorted(const float2 *__restrict__ src, const int *__restrict__ perm, int n,
                                float2 *__restrict__ dst)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) dst[i] = src[perm[i]];
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
    d.nty = p->nty;
    d.W = p->W;
    d.S = p->S;
    d.uv_scale = p->geom.uv_scale;
    d.w_scale = p->geom.w_scale;
    d.gk = reinterpret_cast<const float2 *>(p->gk.kernels);
    d.gs = reinterpret_cast<const int2 *>(p->gk.supports);
    d.dk = reinterpret_cast<const float2 *>(p->dk.kernels);
    d.ds = reinterpret_cast<const int2 *>(p->dk.supports);
    d.rec = p->rec;
    d.items = p->items;
    d.n_items = p->n_items;
    d.item_counter = p->item_counter;
    d.flags = p->flags;
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

// Arena layout of a plan (offsets in bytes).
static void plan_layout(const sdp_visplan *p, size_t *off, size_t *total)
{
    const int n = p->n;
    size_t o = 0;
    const size_t nb_scan = (size_t)((std::max(p->nbins, p->ntiles) + kScanBlock - 1) / kScanBlock + 2);
    off[0] = o; o = align_up(o + sizeof(VisRec) * (size_t)std::max(n, 1), 256);           // rec
    off[1] = o; o = align_up(o + sizeof(VisRec) * (size_t)std::max(n, 1), 256);           // rec_tmp
    off[2] = o; o = align_up(o + sizeof(int) * (size_t)std::max(n, 1), 256);              // perm
    off[3] = o; o = align_up(o + sizeof(int) * (size_t)std::max(n, 1), 256);              // keys
    off[4] = o; o = align_up(o + sizeof(int) * ((size_t)p->nbins + 1), 256);              // counts / fill
    off[5] = o; o = align_up(o + sizeof(int) * ((size_t)p->nbins + 1), 256);              // offsets
    off[6] = o; o = align_up(o + sizeof(int) * ((size_t)p->ntiles + 1), 256);             // item counts
    off[7] = o; o = align_up(o + sizeof(int) * ((size_t)p->ntiles + 1), 256);             // item offsets
    off[8] = o; o = align_up(o + sizeof(int4) * ((size_t)n / kChunk + p->ntiles + 1), 256);// items
    off[9] = o; o = align_up(o + sizeof(int) * nb_scan, 256);                             // scan scratch
    off[10] = o; o = align_up(o + sizeof(int) * 4, 256);                                  // scalars
    off[11] = o; o = align_up(o + sizeof(float2) * (size_t)std::max(n, 1), 256);          // measured
    *total = o;
}

int visplan_setup(sdp_visplan *p, const sdp_geometry *geom, const sdp_wkernels *gk, const sdp_wkernels *dk, int n,
                  int mode)
{
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
    p->ntx = (G + kTile - 1) / kTile;
    p->nty = p->ntx;
    p->ntiles = p->ntx * p->nty;
    p->nk = gk->num_kernels;
    p->nbins = p->ntiles * p->nk;
    p->hs_max = std::max(gk->max_half_support, dk->max_half_support);
    p->W = 2 * p->hs_max + 1;
    p->S = kTile + 2 * p->hs_max;
    return SDP_OK;
}

size_t visplan_arena_bytes(const sdp_visplan *p)
{
    size_t off[12], total;
    plan_layout(p, off, &total);
    return total;
}

int visplan_build(sdp_visplan *p, void *arena, const float3 *uvw, cudaStream_t st)
{
    size_t off[12], total;
    plan_layout(p, off, &total);
    char *a = static_cast<char *>(arena);
    p->arena = arena;
    p->rec = reinterpret_cast<VisRec *>(a + off[0]);
    VisRec *rec_tmp = reinterpret_cast<VisRec *>(a + off[1]);
    p->perm = reinterpret_cast<int *>(a + off[2]);
    int *keys = reinterpret_cast<int *>(a + off[3]);
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
    p->measured = reinterpret_cast<float2 *>(a + off[11]);
    const int n = p->n;

    SDP_CUDA_TRY(cudaMemsetAsync(counts, 0, sizeof(int) * ((size_t)p->nbins + 1), st));
    SDP_CUDA_TRY(cudaMemsetAsync(scalars, 0, sizeof(int) * 4, st));
    if (n > 0) {
        k_bin<<<(n + 255) / 256, 256, 0, st>>>(uvw, n, p->mode, p->geom.grid_size, p->geom.oversampling,
                                               p->geom.uv_scale, p->geom.w_scale,
                                               reinterpret_cast<const int2 *>(p->gk.supports),
                                               reinterpret_cast<const int2 *>(p->dk.supports), p->gk.num_kernels,
                                               p->dk.num_kernels, (long long)p->gk.total_samples,
                                               (long long)p->dk.total_samples, p->hs_max, p->ntx, p->nty, rec_tmp,
                                               keys, counts, p->flags);
        SDP_LAUNCH_CHECK();
    }
    SDP_TRY(exclusive_scan(counts, offsets, p->nbins, scan_scratch, st));
    SDP_CUDA_TRY(cudaMemsetAsync(counts, 0, sizeof(int) * ((size_t)p->nbins + 1), st));
    if (n > 0) {
        k_scatter<<<(n + 255) / 256, 256, 0, st>>>(rec_tmp, keys, n, offsets, counts, p->rec, p->perm);
        SDP_LAUNCH_CHECK();
    }
    k_item_counts<<<(p->ntiles + 255) / 256, 256, 0, st>>>(offsets, p->ntiles, p->nk, item_counts);
    SDP_LAUNCH_CHECK();
    SDP_TRY(exclusive_scan(item_counts, item_offsets, p->ntiles, scan_scratch, st));
    k_item_fill<<<(p->ntiles + 255) / 256, 256, 0, st>>>(offsets, item_offsets, p->ntiles, p->nk, p->items);
    SDP_LAUNCH_CHECK();
    SDP_CUDA_TRY(cudaMemcpyAsync(p->n_items, item_offsets + p->ntiles, sizeof(int), cudaMemcpyDeviceToDevice, st));
    return SDP_OK;
}

int visplan_check_flags(sdp_visplan *p, cudaStream_t st)
{
    int flags = 0;
    SDP_CUDA_TRY(cudaMemcpyAsync(&flags, p->flags, sizeof(int), cudaMemcpyDeviceToHost, st));
    SDP_CUDA_TRY(cudaStreamSynchronize(st));
    if (flags) {
        SDP_CUDA_TRY(cudaMemsetAsync(p->flags, 0, sizeof(int), st));
        return set_error(SDP_ERR_DATA, "visibility data outside the kernel tables (flags 0x%x:%s%s%s)", flags,
                         (flags & FLAG_PLANE) ? " w-plane index beyond NUM_KERNELS;" : "",
                         (flags & FLAG_SUPPORT) ? " support beyond the declared maximum or table;" : "",
                         (flags & FLAG_BOX) ? " tap box wider than 2*hs+1;" : "");
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

static int launch_tiles(sdp_visplan *p, int op, const float2 *vis_in, const float2 *in_grid, float2 *out_grid,
                        float2 *pred, float2 *delta, cudaStream_t st)
{
    PlanDev d = plan_dev(p);
    const size_t smem = (op == OP_DEGRID) ? 0 : sizeof(float2) * (size_t)kWarps * p->S * p->S;
    SDP_CUDA_TRY(cudaMemsetAsync(p->item_counter, 0, sizeof(int), st));
    void (*fn)(PlanDev, const float2 *, const float2 *, float2 *, float2 *, float2 *, const float2 *) = nullptr;
    const bool snapped = (p->mode == SDP_GRID_SNAPPED);
    switch (op) {
    case OP_GRID: fn = snapped ? k_tiles<SDP_GRID_SNAPPED, OP_GRID> : k_tiles<SDP_GRID_STD, OP_GRID>; break;
    case OP_DEGRID: fn = k_tiles<SDP_GRID_STD, OP_DEGRID>; break;
    case OP_CYCLE_CONV: fn = k_tiles<SDP_GRID_STD, OP_CYCLE_CONV>; break;
    case OP_CYCLE_NEAR: fn = k_tiles<SDP_GRID_STD, OP_CYCLE_NEAR>; break;
    case OP_G2G: fn = k_tiles<SDP_GRID_STD, OP_G2G>; break;
    default: return set_error(SDP_ERR_INVALID, "internal: op %d", op);
    }
    if (smem > 48 * 1024) SDP_CUDA_TRY(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    int per_sm = 0;
    SDP_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, kWarps * 32, smem));
    if (per_sm < 1) return set_error(SDP_ERR_RANGE, "tile kernel does not fit (%zu B shared memory)", smem);
    const int grid = per_sm * num_sms();
    fn<<<grid, kWarps * 32, smem, st>>>(d, vis_in, in_grid, out_grid, pred, delta, p->measured);
    SDP_LAUNCH_CHECK();
    return SDP_OK;
}

}  // namespace sdp

SDP_EXPORT int sdp_visplan_grid(sdp_visplan *p, const sdp_float2 *vis, sdp_float2 *grid, int accumulate, void *stream)
{
    SDP_CHECK_ARG(p && grid && (vis || p->n == 0), "NULL argument");
    SDP_CHECK_ARG(p->mode != 2, "plan was built for g2g; use sdp_visplan_g2g");
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
    SDP_CHECK_ARG(p->mode == 2, "plan was not built for g2g");
    cudaStream_t st = as_stream(stream);
    const size_t G2 = (size_t)p->geom.grid_size * p->geom.grid_size;
    SDP_CUDA_TRY(cudaMemsetAsync(out_grid, 0, sizeof(float2) * G2, st));
    if (p->n == 0) return SDP_OK;
    return launch_tiles(p, OP_G2G, nullptr, reinterpret_cast<const float2 *>(in_grid),
                        reinterpret_cast<float2 *>(out_grid), nullptr, nullptr, st);
}
