// Internal interfaces shared between the compilation units of libsdp_b200.
#pragma once

#include "common.cuh"

namespace sdp {

struct VisRec {
    float px, py;  // grid coordinates (reference rounding; snapped in SNAPPED mode)
    int meta;      // bits 0-15 plane, bit 31 conjugate (w < 0)
    int idx;       // original visibility index
};
static_assert(sizeof(VisRec) == 16, "record is one 16-byte load");

// Plan modes beyond the public SDP_GRID_STD / SDP_GRID_SNAPPED.
constexpr int kPlanG2G = 2;

}  // namespace sdp

struct sdp_visplan {
    sdp_geometry geom;
    sdp_wkernels gk, dk;
    int mode;
    int n;
    int ntx, nty, nk, nbins, ntiles, hs_max, W, S;
    sdp::VisRec *rec = nullptr;
    int *perm = nullptr;
    int4 *items = nullptr;
    int *n_items = nullptr;       // device scalar
    int *item_counter = nullptr;  // device scalar
    int *flags = nullptr;         // device scalar
    float2 *measured = nullptr;   // plan order
    int phase_major = 0;          // kernel tables copied phase-major (OS a power of two)
    int *gpoff = nullptr;         // plane offsets into the gridding table in use
    int *dpoff = nullptr;         // plane offsets into the degridding table in use
    float2 *gk2 = nullptr;        // phase-major gridding kernels
    float2 *dk2 = nullptr;        // phase-major degridding kernels
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
// Reads and clears the device error flags (blocking on st).
int visplan_check_flags(sdp_visplan *p, cudaStream_t st);

// FFT helpers.
int check_fft_size(int G);

// Host-side Schwab prolate spheroidal (same evaluation as the device table).
double prolate_host(double nu);

}  // namespace sdp
