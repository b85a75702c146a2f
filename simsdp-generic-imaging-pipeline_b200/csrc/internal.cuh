// Internal interfaces shared between the compilation units of libsdp_b200.
#pragma once

#include "common.cuh"

namespace sdp {

// Visibility record in plan order.  T is the PRECISION of the reference
// build whose index arithmetic the plan reproduces: float (the default
// build) or double (the FP64 build).
template <typename T>
struct Rec {
    T px, py;  // grid coordinates (reference rounding; snapped in SNAPPED mode)
    int meta;  // bits 0-15 plane, bit 31 conjugate (w < 0)
    int idx;   // original visibility index
};
static_assert(sizeof(Rec<float>) == 16, "float record is one 16-byte load");
static_assert(sizeof(Rec<double>) == 24, "double record is 24 bytes");

// Plan modes: the low byte is SDP_GRID_STD / SDP_GRID_SNAPPED / SDP_GRID_G2G,
// flags SDP_PLAN_COORD_F64 and SDP_PLAN_SNAP above it.
constexpr int kPlanG2G = 2;

}  // namespace sdp

struct sdp_visplan {
    sdp_geometry geom;
    sdp_wkernels gk, dk;
    int mode;
    int n;
    int ntx, nty, nk, nbins, ntiles, hs_max, W, S;
    int tile = 16;                // uv tile side (grid cells)
    int chunk = 512;              // visibilities per work item (at most)
    int lanes = 0;                // lanes per visibility of the group kernels (0: warp-per-visibility kernel)
    int warps = 4;                // warps per CTA of the warp-per-visibility kernel (0: by occupancy)
    int pitch = 0;                // row pitch (float2) of the shared tiles: >= S, = 8 mod 16
    uint4 *geo = nullptr;         // plan order: packed tap-box geometry (fast path), see fast_geometry
    void *rec = nullptr;          // Rec<float> or Rec<double>
    int coord_f64 = 0;            // index arithmetic of the double build
    int snap = 0;                 // correct_to_finegrid applied to the uvw at plan build
    int *perm = nullptr;
    int4 *items = nullptr;
    int *n_items = nullptr;       // device scalar
    int *item_counter = nullptr;  // device scalar
    int *flags = nullptr;         // device scalar
    int *kshare = nullptr;        // device scalar: bit 0 set = degridding set differs from gridding set, bit 1 = differs from its conjugate
    float2 *measured = nullptr;   // plan order
    int phase_major = 0;          // kernel tables copied phase-major (OS a power of two)
    int *gpoff = nullptr;         // plane offsets into the gridding table in use
    int *dpoff = nullptr;         // plane offsets into the degridding table in use
    float2 *gk2 = nullptr;        // phase-major gridding kernels
    float2 *dk2 = nullptr;        // phase-major degridding kernels
    float *dinv = nullptr;        // 1 / sqrt(sum |k|^2) of each fast-path tap box of the degridding set (nullptr: none)
    int dinv_nc = 0;              // tap-box configurations per axis of dinv, 2 (OS + 1)
    uint4 *gbase = nullptr;       // plan order: quad records of the half-support-4 fast visibilities (nullptr: none)
    int dk_conj_off = 0;          // offset of the conjugated copy of the phase-major degridding set in dk2
    void *arena = nullptr;
    bool owns_arena = true;
};

namespace sdp {

// Fills the host-side fields of a plan (no device work).
int visplan_setup(sdp_visplan *p, const sdp_geometry *geom, const sdp_wkernels *gk, const sdp_wkernels *dk, int n,
                  int mode);
// Device bytes a plan needs.
size_t visplan_arena_bytes(const sdp_visplan *p);
// Bins the visibilities into the arena (which must hold visplan_arena_bytes).
int visplan_build(sdp_visplan *p, void *arena, const float3 *uvw, cudaStream_t st);
size_t visplan_record_bytes(const sdp_visplan *p);
// Rebuilds the kernel-table copies of a built plan from p->gk / p->dk (same
// supports as at build time).
int visplan_kernels(sdp_visplan *p, cudaStream_t st);
// Reads and clears the device error flags (blocking on st).
int visplan_check_flags(sdp_visplan *p, cudaStream_t st);

// FFT helpers.
int check_fft_size(int G);

// Host-side Schwab prolate spheroidal (same evaluation as the device table).
double prolate_host(double nu);

// sdp_hogbom with a choice of the persistent on-chip kernel (when it fits)
// or one launch per minor cycle.
int hogbom_launch(const sdp_clean_params *p, float *residual, const float *psf, float *model, sdp_float3 *sources,
                  int *num_sources_dev, void *workspace, size_t ws_bytes, bool allow_persistent, cudaStream_t st);

#ifdef __CUDACC__
// top.c:399-451: Schwab's rational approximation of the prolate spheroidal,
// evaluated in double with the reference's two-interval split at nu = 0.75.
__device__ __forceinline__ double prolate_schwab(double nu)
{
    const double p[10] = {0.08203343, -0.3644705, 0.627866, -0.5335581, 0.2312756,
                          0.004028559, -0.03697768, 0.1021332, -0.1201436, 0.06412774};
    const double q[6] = {1.0, 0.8212018, 0.2078043, 1.0, 0.9599102, 0.2918724};
    int part;
    double nuend;
    if (nu >= 0.0 && nu < 0.75) {
        part = 0;
        nuend = 0.75;
    } else if (nu >= 0.75 && nu < 1.0) {
        part = 1;
        nuend = 1.0;
    } else {
        return 0.0;
    }
    const double d = nu * nu - nuend * nuend;
    // powers formed by repeated multiplication (pow(delta, i) for small
    // integer i is exact to the last bit on glibc only up to rounding; the
    // table is checked against the reference to 1 ulp)
    double top = p[part * 5], bot = q[part * 3], dp = 1.0;
    for (int i = 1; i < 5; ++i) {
        dp = __dmul_rn(dp, d);
        top = __dadd_rn(top, __dmul_rn(p[part * 5 + i], dp));
    }
    dp = 1.0;
    for (int i = 1; i < 3; ++i) {
        dp = __dmul_rn(dp, d);
        bot = __dadd_rn(bot, __dmul_rn(q[part * 3 + i], dp));
    }
    return (bot == 0.0) ? 0.0 : __ddiv_rn(top, bot);
}
#endif

}  // namespace sdp
