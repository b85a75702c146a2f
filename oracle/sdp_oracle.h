/*
 * ORACLE — test infrastructure only.  Only tests/, __graft_entry__.smoke() and
 * bench.py's cpu_baseline leg may load this code, and only as the checker.
 *
 * CPU restatement of the reference's imaging actors (param_code/code_fft_1core
 * and the live Hogbom in preesm_pipelines/simsdp_fft_imaging_pipeline), built
 * twice from one source: liboracle_f32.so (PRECISION = float, the reference's
 * default, common.h:62-71) and liboracle_f64.so (PRECISION = double, the FP64
 * oracle, common.h:78-83).  Each function cites the reference lines it
 * follows and keeps the reference's C type promotions, so that the f32 build
 * matches the compiled reference bit for bit wherever the reference is
 * sequential.  Parity is pinned by tests/test_oracle_pins.py against the
 * reference itself compiled from its own sources (oracle/_ref) and against
 * the golden fixtures in tests/golden/.
 *
 * Every pointer is a plain host array.  REAL is float or double by build;
 * 2-vectors and 3-vectors are arrays of REAL with 2 or 3 entries per item.
 */
#ifndef SDP_ORACLE_H
#define SDP_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

#ifdef ORACLE_DOUBLE
typedef double REAL;
#else
typedef float REAL;
#endif

int or_real_size(void);

/* degridgrid.c:12-65 with PERFORM_SIMPLIFICATION = 0 (the generated schedules'
 * setting, code_fft_1core/generated/Core0.c:3101). */
void or_correct_to_finegrid(int n, int grid_size, int os, const REAL *uvw, const REAL *vis, double uv_scale,
                            REAL *out_vis, REAL *out_uvw, int *num_out);

/* degridgrid.c:69-125 (BYPASS = 0 path). */
void or_std_gridding(int grid_size, int os, int n, const REAL *kernels, const int *supports, const REAL *uvw,
                     const REAL *vis, double uv_scale, double w_scale, REAL *grid);

/* degridgrid.c:127-202.  nearest = 1 keeps the reference's override by the
 * nearest grid cell (:193-200); nearest = 0 returns the normalised kernel
 * convolution computed at :147-191 (the value the reference discards). */
void or_std_degridding(int grid_size, int os, int n, const REAL *kernels, const int *supports, const REAL *grid,
                       const REAL *uvw, double uv_scale, double w_scale, REAL *out_vis, int nearest);

/* degridgrid.c:204-326 (w_idx forced to 0 at :215). */
void or_g2g_degridgrid(int grid_size, int os, int n, const REAL *gkernels, const int *gsupports,
                       const REAL *dkernels, const int *dsupports, const REAL *in_grid, const REAL *uvw,
                       double uv_scale, REAL *out_grid);

/* gridding_run.c:55-137 (gridding_CPU); gridding_actor passes os = 16 (:43). */
void or_gridding_cpu(REAL *grid, const REAL *kernels, const int *supports, const REAL *uvw, const REAL *vis,
                     int n, int os, int grid_size, double uv_scale, double w_scale);

/* gains_apply_run.c:273-297 and degridgrid.c:328-335. */
void or_subtract_vis(int n, const REAL *measured, const REAL *predicted, REAL *delta);
void or_subtract_image(int grid_size, const REAL *a, const REAL *b, REAL *out);

/* fft_run.c:5-20, 86-102, 104-121. */
void or_fft_shift_c2c(int grid_size, const REAL *in, REAL *out);
void or_fft_shift_c2r(int grid_size, const REAL *in, REAL *out);
void or_fft_shift_r2c(int grid_size, const REAL *in, REAL *out);
/* fft_run.c:23-83: FFTW semantics, sign -1 forward / +1 inverse, unnormalised. */
void or_fft2d(int grid_size, const REAL *in, REAL *out, int sign);

/* top.c:399-451 */
double or_prolate_spheroidal(double nu);
void or_create_1D_half_prolate(REAL *prolate, int grid_size);
/* convolution_correction_run.c:4-35.  prolate must hold grid_size/2 + 1
 * entries: the reference reads prolate[grid_size/2] (one past its G/2-entry
 * array, top.c:401-407); this restatement defines that entry as the
 * spheroidal at nu = 1, which is 0 (top.c:437-438). */
void or_conv_correction(int grid_size, const REAL *in, const REAL *prolate, REAL *out);

/* dft_run.c:3-48.  sources: (l, m, intensity) triples. */
void or_dft(int n, int num_sources, const REAL *sources, const REAL *uvw, REAL *vis);

/* Live Hogbom, preesm_pipelines/simsdp_fft_imaging_pipeline/Code/src/CPU/deconvolution_run.c:197-311.
 * psf must hold grid_size^2 + 1 entries (the reference can read psf[G*G],
 * one past the end, at :269; this restatement defines that entry as 0). */
void or_hogbom_clean(int grid_size, int num_minor_cycles, int max_sources, const REAL *residual, const REAL *psf,
                     double loop_gain, double noise_factor, double weak_source_percent, double psf_max_value,
                     double cell_size, const REAL *current_model, int *num_sources_out, REAL *sources_out,
                     REAL *output_model, REAL *residual_out);

/* splitmerge.c:14-24, 50-56. */
void or_merge_grids(int grid_size, int slices, const REAL *grids, REAL *out);
void or_split_uvgrid(int grid_size, int slices, const REAL *in, REAL *out);

/* top.c:453-515 without the file read: crop the centre of a full PSF and
 * normalise by the full PSF's maximum; returns that maximum. */
double or_psf_crop_normalise(int grid_size, int psf_grid_size, const REAL *full_psf, REAL *psf);

/* top.c:530-595 */
void or_clean_psf(int grid_size, double psf_max_value, const REAL *dirty_psf, REAL *clean_psf, int *halfdims);

#ifdef __cplusplus
}
#endif
#endif
