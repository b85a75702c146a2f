/*
 * sdp_b200 — B200 (sm_100a) imaging major/minor cycle behind the reference's
 * PREESM actor C ABI.
 *
 * Two layers are exported by libsdp_b200.so:
 *
 *  1. Actor drop-ins.  Same symbol names and argument lists as the reference
 *     actors in param_code/code_*_1core/include/*.h compiled with
 *     SINGLE_PRECISION = 1 (PRECISION = float, common.h:62-71), so the
 *     generated PREESM schedule (generated/Core0.c) links against this
 *     library unchanged.  Every pointer is a HOST pointer, as in the
 *     reference; each call stages its inputs to the GPU, runs the CUDA path
 *     and copies its outputs back before returning.  They return void like
 *     the reference; failures are reported through sdp_last_status() /
 *     sdp_last_error() and, when sdp_set_abort_on_error(1) is set (or
 *     SDP_ABORT_ON_ERROR=1 in the environment), by printing the error and
 *     calling exit(EXIT_FAILURE) as the reference's setup actors do
 *     (src/top.c:85-89).
 *
 *  2. Device-resident layer (sdp_*).  Device pointers, an explicit CUDA
 *     stream passed as void*, and an int status (SDP_OK = 0).  The actor
 *     drop-ins are thin staging wrappers over these calls.
 *
 * There is no CPU fallback: without a usable CUDA device every call fails
 * with SDP_ERR_CUDA.
 */
#ifndef SDP_B200_H
#define SDP_B200_H

#include <stddef.h>

#ifdef __cplusplus
#include <cstdbool>
extern "C" {
#else
#include <stdbool.h>
#endif

/* ---------------------------------------------------------------------------
 * ABI types — layout-identical to the reference's C structs
 * (common.h:137-168 int2 / float2 / float3, and Config common.h:187-265,
 * sizeof 360 on x86-64).
 * ------------------------------------------------------------------------- */
typedef struct { int x, y; } sdp_int2;
typedef struct { float x, y; } sdp_float2;
typedef struct { float x, y, z; } sdp_float3;
typedef struct { float x, y, z, w; } sdp_float4;

typedef struct sdp_config {
    bool retain_device_mem;
    int num_major_cycles;
    int num_recievers;
    int num_baselines;
    int grid_size;
    double cell_size;
    const char *output_path;
    const char *dirty_image_output;
    int gpu_max_threads_per_block;
    int gpu_max_threads_per_block_dimension;
    bool right_ascension;
    bool save_dirty_image;
    bool save_residual_image;
    bool save_extracted_sources;
    bool save_predicted_visibilities;
    bool save_estimated_gains;
    bool perform_system_test;
    const char *system_test_image;
    const char *system_test_sources;
    const char *system_test_visibilities;
    const char *system_test_gains;
    const char *default_gains_file;
    const char *output_gains_file;
    bool perform_gain_calibration;
    bool use_default_gains;
    int max_calibration_cycles;
    int number_cal_major_cycles;
    bool force_weight_to_one;
    double frequency_hz;
    int oversampling;
    double uv_scale;
    int num_visibilities;
    int num_kernels;
    int total_kernel_samples;
    double max_w;
    double w_scale;
    const char *kernel_real_file;
    const char *kernel_imag_file;
    const char *kernel_support_file;
    const char *degridding_kernel_real_file;
    const char *degridding_kernel_imag_file;
    const char *degridding_kernel_support_file;
    const char *visibility_source_file;
    unsigned int number_minor_cycles_cal;
    unsigned int number_minor_cycles_img;
    double loop_gain;
    double weak_source_percent_gc;
    double weak_source_percent_img;
    double noise_factor;
    double psf_max_value;
    const char *model_sources_output;
    const char *residual_image_output;
    const char *psf_input_file;
    const char *psf_image_output;
    const char *clean_psf_image_output;
    const char *model_image_output;
    const char *final_image_output;
    int num_sources;
    const char *predicted_vis_output;
} sdp_config;

/* ---------------------------------------------------------------------------
 * Status and error reporting
 * ------------------------------------------------------------------------- */
enum {
    SDP_OK = 0,
    SDP_ERR_INVALID = 1,  /* NULL pointer, negative or inconsistent size  */
    SDP_ERR_RANGE = 2,    /* size beyond a documented limit                */
    SDP_ERR_CUDA = 3,     /* CUDA runtime error or no usable device         */
    SDP_ERR_NOMEM = 4,    /* device allocation failed                        */
    SDP_ERR_TIMEOUT = 5,  /* a bounded device-side wait gave up             */
    SDP_ERR_DATA = 6,     /* input data outside the grid / kernel tables     */
    SDP_ERR_IO = 7        /* an input file could not be opened or read      */
};

int sdp_last_status(void);           /* status of the calling thread's last failing call */
const char *sdp_last_error(void);    /* message for it ("" when none)                     */
void sdp_clear_error(void);
void sdp_set_abort_on_error(int on); /* 1: print and exit(EXIT_FAILURE) on error         */
int sdp_version(void);               /* 100 * major + minor                               */

/* Degridding mode of the std_degridding drop-in (process wide).
 * SDP_DEGRID_NEAREST (default) reproduces the reference exactly: the value
 * is the nearest grid cell (degridgrid.c:193-200).  SDP_DEGRID_CONV returns
 * the normalised kernel convolution the reference computes and then
 * discards (degridgrid.c:147-191). */
enum { SDP_DEGRID_NEAREST = 0, SDP_DEGRID_CONV = 1 };
int sdp_set_degrid_mode(int mode);
int sdp_get_degrid_mode(void);

/* ---------------------------------------------------------------------------
 * Layer 1: actor drop-ins (host pointers, reference signatures)
 * ------------------------------------------------------------------------- */

/* degridgrid.h:10-11 — snap uvw to the 1/OS fine grid (simplification must be 0). */
void correct_to_finegrid(int NUM_VISIBILITIES, int GRID_SIZE, int OVERSAMPLING_FACTOR, int PERFORM_SIMPLIFICATION,
                         sdp_float3 *vis_uvw_coords, sdp_float2 *input_visibilities, sdp_config *config,
                         sdp_float2 *output_visibilities, sdp_float3 *output_finegrid_vis_coords,
                         int *num_output_visibilities);

/* degridgrid.h:13-14 — w-projection gridding. */
void std_gridding(int GRID_SIZE, int NUM_VISIBILITIES, int NUM_KERNELS, int TOTAL_KERNEL_SAMPLES,
                  int OVERSAMPLING_FACTOR, int BYPASS, int *maj_iter, int *num_corrected_visibilities,
                  sdp_float2 *kernels, sdp_int2 *kernel_supports, sdp_float3 *corrected_vis_uvw_coords,
                  sdp_float2 *visibilities, sdp_config *config, sdp_float2 *prev_grid, sdp_float2 *output_grid);

/* degridgrid.h:16-18 — degridding (mode per sdp_set_degrid_mode). */
void std_degridding(int GRID_SIZE, int NUM_VISIBILITIES, int NUM_KERNELS, int TOTAL_KERNEL_SAMPLES,
                    int OVERSAMPLING_FACTOR, sdp_float2 *kernels, sdp_int2 *kernel_supports, sdp_float2 *input_grid,
                    sdp_float3 *corrected_vis_uvw_coords, int *num_corrected_visibilities, sdp_config *config,
                    sdp_float2 *output_visibilities);

/* degridgrid.h:20-23 — grid-to-grid: nearest-cell sample, regrid with the w = 0 kernel. */
void g2g_degridgrid(int GRID_SIZE, int NUM_VISIBILITIES, int NUM_GRIDDING_KERNELS, int NUM_DEGRIDDING_KERNELS,
                    int TOTAL_GRIDDING_KERNEL_SAMPLES, int TOTAL_DEGRIDDING_KERNEL_SAMPLES, int OVERSAMPLING_FACTOR,
                    sdp_float2 *gridding_kernels, sdp_int2 *gridding_kernel_supports, sdp_float2 *degridding_kernels,
                    sdp_int2 *degridding_kernel_supports, sdp_float2 *input_grid,
                    sdp_float3 *corrected_vis_uvw_coords, int *num_corrected_visibilities, sdp_config *config,
                    sdp_float2 *output_grid);

/* degridgrid.h:25 */
void subtract_image_space(int GRID_SIZE, float *measurements, float *estimate, float *result);
/* degridgrid.h:27 (a sink: does nothing, as in the reference) */
void degridding_kernel_sink(int NUM_DEGRIDDING_KERNELS, int TOTAL_DEGRIDDING_KERNEL_SAMPLES, sdp_int2 *supports,
                            sdp_float2 *kernels);

/* gridding_run.h:12-13 — DFT-pipeline gridder (snapped coordinates, inclusive taps, OS = 16). */
void gridding_actor(int GRID_SIZE, int NUM_VISIBILITIES, int NUM_KERNELS, int TOTAL_KERNEL_SAMPLES,
                    sdp_float2 *kernels, sdp_int2 *kernel_supports, sdp_float3 *vis_uvw_coords,
                    sdp_float2 *visibilities, sdp_config *config, sdp_float2 *uv_grid);
/* gridding_run.h:15-17 — the gridder behind gridding_actor; accumulates into grid. */
void gridding_CPU(sdp_float2 *grid, const sdp_float2 *kernel, const sdp_int2 *supports, const sdp_float3 *vis_uvw,
                  const sdp_float2 *vis, const int num_vis, const int oversampling, const int grid_size,
                  const double uv_scale, const double w_scale);
/* gridding_run.h:21 */
void add_visibilities(int NUM_VISIBILITIES, sdp_float2 *v1, sdp_float2 *v2, sdp_float2 *output);

/* fft_run.h:13-21 */
void fft_shift_complex_to_complex_actor(int GRID_SIZE, sdp_float2 *uv_grid_in, sdp_config *config,
                                        sdp_float2 *uv_grid_out);
void CUFFT_EXECUTE_FORWARD_C2C_actor(int GRID_SIZE, sdp_float2 *uv_grid_in, sdp_float2 *uv_grid_out);
void CUFFT_EXECUTE_INVERSE_C2C_actor(int GRID_SIZE, sdp_float2 *uv_grid_in, sdp_float2 *uv_grid_out);
void fft_shift_complex_to_real_actor(int GRID_SIZE, sdp_float2 *uv_grid, sdp_config *config, float *dirty_image);
void fft_shift_real_to_complex_actor(int GRID_SIZE, float *image, sdp_config *config, sdp_float2 *fourier);

/* convolution_correction_run.h:11-12.  prolate holds GRID_SIZE/2 entries;
 * the reference also reads prolate[GRID_SIZE/2] (one past the end); here that
 * entry is taken as the spheroidal at nu = 1, which is 0. */
void execute_convolution_correction_actor(int GRID_SIZE, float *dirty_image_in, float *prolate, sdp_config *config,
                                          float *dirty_image_out);
void execute_inv_convolution_correction_actor(int GRID_SIZE, float *dirty_image_in, float *prolate,
                                              sdp_config *config, float *dirty_image_out);

/* dft_run.h:15-16 */
void dft_actor(int NUM_VISIBILITIES, int NUM_MAX_SOURCES, sdp_float3 *sources, sdp_float3 *vis_uvw_coords,
               int *num_sources, sdp_config *config, sdp_float2 *visibilities);

/* deconvolution_run.h:14-15 — the live Hogbom CLEAN of
 * preesm_pipelines/simsdp_fft_imaging_pipeline/Code/src/CPU/deconvolution_run.c:197-311
 * (the param_code copy has its body commented out). */
void hogbom_clean(int GRID_SIZE, int NUM_MINOR_CYCLES, int MAX_SOURCES, float *residual, float *psf,
                  sdp_int2 *partial_psf_halfdims, sdp_config *config, float *current_model, int *num_sources_out,
                  sdp_float3 *sources_out, float *output_model);

/* splitmerge.h:15-21 */
void split_visibilities(sdp_config *config, int NUM_VISIBILITIES, int SLICES, sdp_float2 *measured_visibilities,
                        sdp_float3 *vis_coords, sdp_float2 *visibilities, sdp_float3 *out_vis_coords,
                        sdp_config *output_configs, sdp_config *output_config);
void merge_gridded_visibilities(int GRID_SIZE, int SLICES, sdp_float2 *grids, sdp_float2 *output_grid);
void merge_configs(sdp_config *in_configs, sdp_config *out_config);
void split_fftdegrid_visibilities(int NUM_VISIBILITIES, int SLICES, int GRID_SIZE, sdp_config *config,
                                  sdp_float3 *vis_coords, sdp_float2 *measured_visibilities, int *num_corrected_vis,
                                  int *maj_iter, sdp_float2 *output_visibilities, sdp_float3 *out_vis_coords,
                                  sdp_config *output_configs, int *num_vis, int *maj_iter_out);
void split_uvgrid(int GRID_SIZE, int SLICES, sdp_float2 *input_grid, sdp_float2 *output_grid);

/* gains_apply_run.h:14, 19, 23, 28 and top.h:19, 22 — gains (gains_apply_run.c:4-120,
 * top.c:71-136): conj(g)/|g|^2 per receiver, and measured * g_a * conj(g_b)
 * (minus the prediction) per visibility, baseline = index % NUM_BASELINES;
 * bit-exact with the float build.  apply_gains_only stores the measured
 * visibilities unchanged, as the reference does (:117).  A receiver pair
 * outside [0, NUM_RECEIVERS) sets SDP_ERR_DATA (the reference reads past
 * gains[]). */
void reciprocal_transform_actor(int NUM_RECEIVERS, sdp_float2 *gains_in, sdp_config *config, sdp_float2 *gains_out);
void apply_gains_actor(int CALIBRATION, int NUM_RECEIVERS, int NUM_BASELINES, int NUM_VISIBILITIES,
                       sdp_float2 *measured_vis, sdp_float2 *visibilities_in, sdp_float2 *gains,
                       sdp_int2 *receiver_pairs, sdp_config *config, sdp_float2 *visibilities_out);
void subtract_from_measurements(int NUM_RECEIVERS, int NUM_BASELINES, int NUM_VISIBILITIES, sdp_float2 *measured_vis,
                                sdp_float2 *visibilities_in, sdp_float2 *gains, sdp_int2 *receiver_pairs,
                                sdp_config *config, sdp_float2 *visibilities_out);
void apply_gains_only(int NUM_RECEIVERS, int NUM_BASELINES, int NUM_VISIBILITIES, sdp_float2 *measured_vis,
                      sdp_float2 *gains, sdp_int2 *receiver_pairs, sdp_config *config, sdp_float2 *visibilities_out);
void gains_host_set_up(int NUM_RECEIVERS, int NUM_BASELINES, sdp_config *config, sdp_float2 *gains,
                       sdp_int2 *receiver_pairs);
void calculate_receiver_pairs(int NUM_BASELINES, int NUM_RECEIVERS, sdp_int2 *receiver_pairs);

/* gains_calibration_run.h:25-35 — gain calibration (gains_calibration_run.c):
 * the normal equations A (2R x 2R, row-major) and Q (2R) of one Gauss-Newton
 * step from measured and predicted visibilities per baseline (:20-252), the
 * SVD A = U S V^T (:254-298; LAPACK's column-major U and V^T, S decreasing),
 * SUQ = S^-1 U^T Q with |S| <= 1e-6 dropped (:439-455), and gains += V SUQ
 * (:457-476).  The first, third and fourth are bit-exact with the float
 * build.  The SVD is a one-sided Jacobi method in FP64 (singular vectors
 * agree with LAPACK's up to sign); it takes square matrices (the
 * calibration's) and leaves A_array unchanged. */
void update_gain_calibration_actor(int NUM_BASELINES, int NUM_RECEIVERS, int NUM_VISIBILITIES, int *loop_cycle_token,
                                   sdp_float2 *measured_vis, sdp_float2 *visibilities, sdp_float2 *gains,
                                   sdp_int2 *receiver_pairs, sdp_config *config, float *A_array, float *Q_array);
void execute_calibration_SVD_actor(int NUM_COLS, int NUM_ROWS, float *A_array, float *S_array, float *U_array,
                                   float *V_array);
void calculate_SUQ_product_actor(int NUM_COLS, int NUM_ROWS, float *S_array, float *U_array, float *Q_array,
                                 sdp_config *config, float *SUQ_array);
void calculate_delta_update_gains_actor(int NUM_COLS, int NUM_RECEIVERS, float *SUQ_array, float *V_array,
                                        sdp_config *config, sdp_float2 *gains_in, sdp_float2 *gains_out);

/* gains_apply_run.h:31 */
void subtract_from_measurements_finegrid(int NUM_VISIBILITIES, sdp_float2 *gridded_measured_vis,
                                         sdp_float2 *input_vis, int *num_finegrid_vis, sdp_float2 *delta_vis);

/* top.h:24, 26, 28, 37 — file-reading setup actors (top.c:139-380, 453-510):
 * the same files, values and float roundings as the reference, parsed by
 * several host threads instead of one fscanf per number.  Host code only.
 * A file that cannot be opened sets SDP_ERR_IO (the reference exits). */
void visibility_host_set_up(int NUM_VISIBILITIES, sdp_config *config, sdp_float3 *vis_uvw_coords,
                            sdp_float2 *measured_vis);
void kernel_host_set_up(int NUM_KERNELS, int TOTAL_KERNEL_SAMPLES, sdp_config *config, sdp_int2 *kernel_supports,
                        sdp_float2 *kernels);
void degridding_kernel_host_set_up(int NUM_KERNELS, int TOTAL_KERNEL_SAMPLES, sdp_config *config,
                                   sdp_int2 *degridding_kernel_supports, sdp_float2 *degridding_kernels);
void psf_host_set_up(int GRID_SIZE, int PSF_GRID_SIZE, sdp_config *config, float *psf, double *psf_max_value);

/* major_loop_iter.h:22, 27-30 and major_loop_iter.c:8 — restoring and
 * writing (major_loop_iter.c:8-46, 168-278): conv2D runs on the GPU with the
 * reference's products and order of additions (bit-exact); the writers
 * format "%f, " as the reference does, on all host threads.  The reference
 * prints an MD5 of every image it saves; these writers do not. */
void conv2D(float *image, float *filter, float *result, int IMAGE_DIM, sdp_int2 filter_half_dims);
void save_image_to_file(sdp_config *config, float *image, const char *file_name, int start_x, int start_y,
                        int range_x, int range_y, int cycle);
void save_output(int GRID_SIZE, float *residual, float *model, float *clean_psf, sdp_int2 *clean_psf_halfdims,
                 float *psf, sdp_config *config, int *cycle);
void save_extracted_sources_actor(int GRID_SIZE, int SAVE_EXTRACTED_SOURCES, int NUM_MAX_SOURCES, int *num_sources,
                                  sdp_float3 *sources, int *cycle_count, sdp_config *config, float *image_in,
                                  float *clean_psf, sdp_int2 *clean_psf_halfdims, float *image_out);

/* top.h:17, 31-41, 43-45 — setup math. */
void config_struct_set_up(int GRID_SIZE, int NUM_KERNELS, sdp_config *config);
void correction_set_up(int GRID_SIZE, float *prolate);
void create_1D_half_prolate(float *prolate, int grid_size);
double prolate_spheroidal(double nu);
void config_struct_set_up_sequel(sdp_config *config_in, double *psf_max_value, sdp_config *config_out);
void clean_psf_host_set_up(int GRID_SIZE, int GAUSSIAN_CLEAN_PSF, sdp_config *config, float *dirty_psf,
                           float *clean_psf, sdp_int2 *partial_psf_halfdims);
void model_set_up(int GRID_SIZE, sdp_config *config, float *initial_image);
void sources_set_up(int MAX_SOURCES, int *num_sources, sdp_float3 *sources);

/* ---------------------------------------------------------------------------
 * Layer 2: device-resident API (device pointers, stream as void*, int status)
 * ------------------------------------------------------------------------- */

/* Geometry shared by gridding and degridding (Config fields uv_scale,
 * w_scale, oversampling and GRID_SIZE). */
typedef struct sdp_geometry {
    int grid_size;     /* even, 8 <= grid_size <= 32768            */
    int oversampling;  /* 1 <= oversampling <= 64                   */
    double uv_scale;
    double w_scale;
} sdp_geometry;

/* One W-projection kernel set: planes concatenated, supports[p] = (half
 * support, sample offset) as kernel_host_set_up builds them (top.c:256-261). */
typedef struct sdp_wkernels {
    const sdp_float2 *kernels;   /* device */
    const sdp_int2 *supports;    /* device */
    int num_kernels;             /* planes */
    int total_samples;           /* entries of kernels                          */
    int max_half_support;        /* max over planes of supports[p].x (host value) */
} sdp_wkernels;

/* Gridding semantics (low byte of grid_mode). */
enum {
    SDP_GRID_STD = 0,         /* std_gridding: taps [ceil(p-hs), ceil(p+hs))                 */
    SDP_GRID_SNAPPED = 1      /* gridding_CPU: snapped p, taps [ceil(p-hs), floor(p+hs)]      */
};
/* Plan flags, OR-ed into grid_mode.
 * SDP_PLAN_COORD_F64: grid coordinates, tap boxes, kernel indices and nearest
 *   cells follow the reference's double build (PRECISION = double) instead
 *   of its float build; the kernel products stay FP32.  Use it to match the
 *   FP64 oracle: the float build's ceil/round decisions differ from the
 *   double build's for coordinates within an ulp of an integer.
 * SDP_PLAN_SNAP: apply correct_to_finegrid (degridgrid.c:24-25, 52-54) to
 *   the raw uvw at plan build, in the plan's coordinate precision, so the
 *   snapped coordinates are never rounded to float in between. */
enum { SDP_PLAN_COORD_F64 = 0x100, SDP_PLAN_SNAP = 0x200 };

/* Visibility set binned by uv tile (and w-plane) once, reused by every
 * gridding / degridding pass of a major cycle. */
typedef struct sdp_visplan sdp_visplan;

int sdp_visplan_create(sdp_visplan **plan, const sdp_geometry *geom, const sdp_wkernels *grid_kernels,
                       const sdp_wkernels *degrid_kernels, int num_vis, const sdp_float3 *uvw, int grid_mode,
                       void *stream);
int sdp_visplan_destroy(sdp_visplan *plan);
/* Plan shape (no counterpart in the reference): uv tile side (a multiple of
 * 8 in 8..128, default 16), visibilities per work item (64..65536, default
 * 512), lanes per visibility (0: std_gridding plans with half supports up
 * to 4 take the warp-per-visibility kernel, one warp per visibility and a
 * private subgrid per warp, other plans the fewest lanes their support needs;
 * 8 / 16 / 32: the group kernels with that many lanes per visibility, several
 * visibilities per warp on one shared subgrid), warps per CTA of the
 * warp-per-visibility kernel (0: by occupancy, or 4 / 8).  Zero fields take
 * the defaults.  sdp_visplan_create and the actors use tile 16, 512
 * visibilities per item, 4 warps.  Results are the same for every shape up
 * to the order of the floating-point sums. */
typedef struct sdp_plan_options {
    int tile;
    int chunk;
    int lanes;
    int warps;
} sdp_plan_options;
int sdp_visplan_create_opt(sdp_visplan **plan, const sdp_geometry *geom, const sdp_wkernels *grid_kernels,
                           const sdp_wkernels *degrid_kernels, int num_vis, const sdp_float3 *uvw, int grid_mode,
                           const sdp_plan_options *options, void *stream);
int sdp_visplan_options(const sdp_visplan *plan, sdp_plan_options *options);
/* Autotuner: builds a plan for each candidate shape (warp-per-visibility
 * kernel: tiles 8 / 16 / 24 / 32, work items of 256 / 512 / 1024
 * visibilities, 4 or 8 warps per CTA; group kernels: tile 32 with 8 and 16
 * lanes per visibility), times reps fused major-cycle passes (sdp_visplan_cycle on model_grid,
 * residual_grid as scratch) with CUDA events on the stream, and returns the
 * fastest shape, its time per pass (ms) and the number of shapes timed.
 * Blocking; allocates and frees one plan at a time. */
int sdp_visplan_autotune(const sdp_geometry *geom, const sdp_wkernels *grid_kernels,
                         const sdp_wkernels *degrid_kernels, int num_vis, const sdp_float3 *uvw, int grid_mode,
                         const sdp_float2 *measured, const sdp_float2 *model_grid, sdp_float2 *residual_grid,
                         int degrid_mode, int reps, sdp_plan_options *best, float *best_ms, int *candidates,
                         void *stream);
int sdp_visplan_num_work_items(const sdp_visplan *plan, int *count); /* blocking read */
/* Measured visibilities (original order) copied into plan order. */
int sdp_visplan_set_measured(sdp_visplan *plan, const sdp_float2 *measured, void *stream);
/* grid: output_grid (G^2, zeroed first unless accumulate) += vis (original order) convolved. */
int sdp_visplan_grid(sdp_visplan *plan, const sdp_float2 *vis, sdp_float2 *grid, int accumulate, void *stream);
/* degrid with mode SDP_DEGRID_*; predicted written in original order. */
int sdp_visplan_degrid(sdp_visplan *plan, const sdp_float2 *model_grid, sdp_float2 *predicted, int mode,
                       void *stream);
/* Fused visibility pass of one FFT-pipeline major cycle:
 * predicted = degrid(model_grid); delta = measured - predicted;
 * residual_grid = grid(delta).  predicted/delta may be NULL (not stored). */
int sdp_visplan_cycle(sdp_visplan *plan, const sdp_float2 *model_grid, int degrid_mode, sdp_float2 *predicted,
                      sdp_float2 *delta, sdp_float2 *residual_grid, void *stream);

/* Several frequency channels' fused passes in one persistent launch over a
 * shared (channel, uv-tile) work queue (the reference runs channels as
 * separate pipelines: read_ms/joint_nnode_ms/main.c:118-145 distributes them
 * over MPI ranks).  Each plan is one channel's std_gridding plan with its
 * measured visibilities set; all plans use one coordinate mode and stay
 * owned by the caller (they must outlive the batch).  set_grids takes host
 * arrays of device pointers (one model and one residual grid per channel);
 * cycle zeroes every residual grid and runs the pass of sdp_visplan_cycle
 * for all channels at once. */
typedef struct sdp_visbatch sdp_visbatch;
int sdp_visbatch_create(sdp_visbatch **batch, sdp_visplan *const *plans, int num_plans, void *stream);
int sdp_visbatch_set_grids(sdp_visbatch *batch, const sdp_float2 *const *model_grids,
                           sdp_float2 *const *residual_grids, void *stream);
int sdp_visbatch_cycle(sdp_visbatch *batch, int degrid_mode, void *stream);
int sdp_visbatch_num_work_items(const sdp_visbatch *batch, int *count);
int sdp_visbatch_destroy(sdp_visbatch *batch);
/* g2g_degridgrid on a plan built with grid_mode SDP_GRID_G2G:
 * out_grid = regrid(nearest_cell(in_grid)) with the plane-0 gridding kernel. */
enum { SDP_GRID_G2G = 2 };
int sdp_visplan_g2g(sdp_visplan *plan, const sdp_float2 *in_grid, sdp_float2 *out_grid, void *stream);
/* Reads and clears the plan's device-side data flags (blocking): returns
 * SDP_ERR_DATA when a visibility addressed a w-plane beyond the kernel
 * tables or a support wider than declared. */
int sdp_visplan_check(sdp_visplan *plan, void *stream);

/* Element-wise and setup kernels (device pointers). */
int sdp_degrid_nearest(int grid_size, double uv_scale, int num_vis, const sdp_float3 *uvw, const sdp_float2 *grid,
                       sdp_float2 *out, void *stream);
int sdp_correct_to_finegrid(int grid_size, int oversampling, double uv_scale, int num_vis, const sdp_float3 *uvw,
                            sdp_float3 *out_uvw, void *stream);
int sdp_subtract_vis(int num_vis, const sdp_float2 *measured, const sdp_float2 *predicted, sdp_float2 *delta,
                     void *stream);
int sdp_add_vis(int num_vis, const sdp_float2 *a, const sdp_float2 *b, sdp_float2 *out, void *stream);
int sdp_subtract_image(int grid_size, const float *a, const float *b, float *out, void *stream);
int sdp_merge_grids(int grid_size, int slices, const sdp_float2 *grids, sdp_float2 *out, void *stream);
int sdp_fft_shift_c2c(int grid_size, const sdp_float2 *in, sdp_float2 *out, void *stream);
int sdp_fft_shift_c2r(int grid_size, const sdp_float2 *in, float *out, void *stream);
int sdp_fft_shift_r2c(int grid_size, const float *in, sdp_float2 *out, void *stream);
int sdp_conv_correction(int grid_size, const float *in, const float *prolate_ext, float *out, void *stream);
int sdp_prolate_table(int grid_size, float *prolate_ext, void *stream); /* G/2 + 1 entries, last = 0 */
/* top.c:530-595: Gaussian clean beam from the dirty PSF; halfdims_dev: 2 ints. */
int sdp_clean_psf(int grid_size, double psf_max_value, const float *dirty_psf, float *clean_psf, int *halfdims_dev,
                  void *stream);

/* The model image convolved with the clean PSF window (conv2D,
 * major_loop_iter.c:8-46), bit-exact with the reference: model pixels >= 1e-5
 * contribute model * psf[(G/2+1 - fy) G + (G/2+1 - fx)] for (fy, fx) in
 * [-half_y, half_y) x [-half_x, half_x) inside the image.  Device pointers;
 * workspace of sdp_restore_workspace_bytes(grid_size). */
int sdp_restore_workspace_bytes(int grid_size, size_t *bytes);
int sdp_restore(int grid_size, const float *model, const float *clean_psf, int half_x, int half_y, float *result,
                void *workspace, size_t workspace_bytes, void *stream);

/* Gains on the device: reciprocal per receiver; per visibility
 * out = measured * g[pair.x] * conj(g[pair.y]) (- vis_in when subtract),
 * pair = receiver_pairs[i % num_baselines].  flags_dev (device int, cleared
 * by the caller) gets 1 when a pair indexes outside the gains. */
int sdp_gains_reciprocal(int num_receivers, const sdp_float2 *gains_in, sdp_float2 *gains_out, void *stream);
int sdp_apply_gains(int num_vis, int num_baselines, int num_receivers, const sdp_float2 *measured,
                    const sdp_float2 *vis_in, const sdp_float2 *gains, const sdp_int2 *receiver_pairs, int subtract,
                    sdp_float2 *vis_out, int *flags_dev, void *stream);

/* Gain calibration on the device (the actors above, device pointers).
 * flags_dev (device int, cleared by the caller) gets 1 when a receiver pair
 * indexes outside the gains.  sdp_svd: square n x n A (column-major, n <= 2048), S (n),
 * U and VT (n x n, column-major); workspace of sdp_svd_workspace_bytes(n);
 * one cooperative launch whose grid barriers are bounded (sdp_svd_check
 * reports SDP_ERR_TIMEOUT when one gave up, and the sweeps run). */
int sdp_gaincal_normal_equations(int num_baselines, int num_receivers, const sdp_float2 *measured,
                                 const sdp_float2 *predicted, const sdp_float2 *gains, const sdp_int2 *receiver_pairs,
                                 float *A, float *Q, int *flags_dev, void *stream);
int sdp_svd_workspace_bytes(int n, size_t *bytes);
int sdp_svd(int n, const float *A, float *S, float *U, float *VT, void *workspace, size_t workspace_bytes,
            void *stream);
int sdp_svd_check(const void *workspace, int *sweeps, void *stream);
int sdp_gaincal_suq(int n, const float *S, const float *U, const float *Q, float *SUQ, void *stream);
int sdp_gaincal_update(int n, int num_receivers, const float *SUQ, const float *VT, const sdp_float2 *gains_in,
                       sdp_float2 *gains_out, void *stream);

/* Inputs the reference reads from files and never generates (no counterpart
 * in its code; its kernel files follow the layout of top.c:256-312):
 * W-projection kernel tables for num_planes planes of the given half
 * supports, oversampling, maximum |w| and field of view (separable
 * prolate-tapered w screen, image_samples points across the field), written
 * in the reference's quarter-plane layout with supports[p] = (hs, offset);
 * degrid_kernels (may be NULL) receives the conjugates.  Device tables;
 * supports may be host or device memory; scratch of
 * sdp_wkernels_generate_scratch_bytes.  Synchronises the stream. */
int sdp_wkernels_generate_sizes(int num_planes, const int *half_supports, int oversampling, int *total_samples);
size_t sdp_wkernels_generate_scratch_bytes(int num_planes, const int *half_supports, int oversampling);
int sdp_wkernels_generate(int num_planes, const int *half_supports, int oversampling, double max_w, double fov_rad,
                          int image_samples, sdp_float2 *grid_kernels, sdp_float2 *degrid_kernels,
                          sdp_int2 *supports, void *scratch, size_t scratch_bytes, void *stream);
/* The dirty PSF of a std_gridding plan: unit visibilities gridded, shifted,
 * inverse-transformed, taper-corrected (as a major cycle images), then
 * divided by its maximum, which lands in *psf_max_dev (device double), as
 * psf_host_set_up normalises the PSF it reads (top.c:481-509).  Scratch:
 * num_vis complex, two G^2 complex. */
int sdp_psf_generate(sdp_visplan *plan, const float *prolate_ext, sdp_float2 *unit_vis_scratch,
                     sdp_float2 *grid_scratch, sdp_float2 *work, float *psf, double *psf_max_dev, void *stream);

/* RMS of an image, summed in FP64 in a fixed order (the residual level that
 * decides major-cycle convergence).  *rms_dev is a device double. */
int sdp_image_rms(int grid_size, const float *image, double *rms_dev, void *stream);

/* 2-D complex FFT, FFTW sign convention (-1 forward, +1 inverse), unnormalised.
 * Power-of-two grid_size from 16 to 16384; in may equal out. */
int sdp_fft2d(int grid_size, const sdp_float2 *in, sdp_float2 *out, int sign, void *stream);
/* The same transform on the tensor cores (no counterpart in the reference):
 * BF16 split hi/lo DFT-matrix products (radix 16, 16, r) accumulated in
 * FP32, G = 1024, 2048 or 4096; about 3e-5 relative RMS against FP64 (the
 * FP32 transform above: about 1e-7).  work: G^2 elements, distinct from in
 * and out. */
int sdp_fft2d_tc(int grid_size, const sdp_float2 *in, sdp_float2 *out, int sign, sdp_float2 *work, void *stream);
/* Fused imaging transforms of the FFT pipeline:
 * image = taper_correct(shift_c2r(iFFT(shift_c2c(grid))))  and
 * grid  = shift_c2c(FFT(shift_r2c(image))).  work: G^2 complex scratch. */
int sdp_grid_to_image(int grid_size, const sdp_float2 *grid, const float *prolate_ext, sdp_float2 *work,
                      float *image, void *stream);
int sdp_image_to_grid(int grid_size, const float *image, sdp_float2 *work, sdp_float2 *grid, void *stream);

/* DFT predict: sources (l, m, I); phase argument in FP64 (north-star
 * precision), sin/cos in FP32 (hardware approximation) after exact range
 * reduction to one turn. */
int sdp_dft(int num_vis, int num_sources, const sdp_float3 *sources, const sdp_float3 *uvw, sdp_float2 *vis,
            void *stream);

/* Hogbom CLEAN on the device, reference semantics.  psf holds G^2 entries.
 * On return (after the stream completes) *num_sources_dev holds the count. */
typedef struct sdp_clean_params {
    int grid_size;
    int num_minor_cycles;
    int max_sources;
    double loop_gain;
    double noise_factor;
    double weak_source_percent;
    double psf_max_value;
    double cell_size;
} sdp_clean_params;
/* Workspace for sdp_hogbom.  For grid_size up to about 2750 (G^2 floats
 * spread over the SMs' shared memory) the CLEAN runs as one persistent
 * cooperative kernel with the residual held on chip and one bounded grid
 * barrier per minor cycle; if a barrier wait gives up (about one second),
 * *num_sources_dev is set to -1.  Larger images use one launch per minor
 * cycle. */
int sdp_hogbom_workspace_bytes(int grid_size, size_t *bytes);
int sdp_hogbom(const sdp_clean_params *p, float *residual_inout, const float *psf, float *model_inout,
               sdp_float3 *sources, int *num_sources_dev, void *workspace, size_t workspace_bytes, void *stream);
/* No counterpart in the reference.  sdp_hogbom for callers that cannot
 * allocate device memory (a runtime that fixes all its memory before it
 * starts, as the PREESM schedule does with its static arena, and must not
 * call an allocator, which can block, while it runs; or a program whose
 * device memory belongs to another allocator).  Same arguments and results
 * as sdp_hogbom, without the workspace: the minor-cycle state and per-block
 * partials live in one fixed 65,792-byte device array per GPU (held until
 * the process exits), so grid_size is limited to 4096 (larger sizes return
 * SDP_ERR_RANGE).  It calls no cudaMalloc/cudaFree.  The first call on a
 * device looks up the array's device address (cudaGetSymbolAddress); make
 * that first call before any stream capture.  The address is cached with
 * the id of the context it was found in, so after cudaDeviceReset (or any
 * re-creation of the device's context) the next call looks it up again:
 * make that call, too, outside stream capture.  Every call clears the state
 * it needs; calls that overlap on the GPU share the array and race, so
 * serialise them (one stream, or events). */
int sdp_hogbom_noalloc(const sdp_clean_params *p, float *residual_inout, const float *psf, float *model_inout,
                       sdp_float3 *sources, int *num_sources_dev, void *stream);

/* ---------------------------------------------------------------------------
 * Binary input files (no counterpart in the reference, which reads text:
 * top.c:139-222 visibilities, :224-380 kernel tables, :453-510 the PSF).
 * A 64-byte header ("SDPBIN1", kind, count, aux, two payload sections on
 * 4096-byte boundaries) followed by the raw little-endian arrays:
 *   kind 1 visibilities: uvw float[n][3], vis float[n][2]; aux bit 0 = the
 *          uvw are already snapped by correct_to_finegrid;
 *   kind 2 kernel set: supports int[planes][2] (half support, offset), then
 *          samples float[total][2]; count = total, aux = planes;
 *   kind 3 image: float[rows][cols]; count = rows, aux = cols.
 * The sdp_bin_load_* calls read the file with several host threads into a
 * ring of pinned staging buffers and copy each filled buffer to the device
 * asynchronously on `stream` while the next one is read; they return after
 * the last copy has completed.  Errors: SDP_ERR_IO (open/read/write),
 * SDP_ERR_DATA (not such a file, wrong kind, truncated), SDP_ERR_RANGE
 * (larger than the caller's buffers).
 * ------------------------------------------------------------------------- */
int sdp_bin_info(const char *path, int *kind, long long *count, long long *aux);
int sdp_bin_write_vis(const char *path, long long num_vis, const sdp_float3 *uvw, const sdp_float2 *vis, int snapped);
int sdp_bin_write_kernels(const char *path, int num_planes, long long total_samples, const sdp_int2 *supports,
                          const sdp_float2 *samples);
int sdp_bin_write_image(const char *path, int rows, int cols, const float *image);
int sdp_bin_read_vis_host(const char *path, long long max_vis, sdp_float3 *uvw, sdp_float2 *vis, long long *num_vis,
                          int *snapped);
int sdp_bin_load_vis(const char *path, long long max_vis, sdp_float3 *uvw_dev, sdp_float2 *vis_dev,
                     long long *num_vis, int *snapped, void *stream);
int sdp_bin_load_kernels(const char *path, int max_planes, long long max_samples, sdp_int2 *supports_dev,
                         sdp_float2 *samples_dev, int *num_planes, long long *total_samples, void *stream);
int sdp_bin_load_image(const char *path, int max_rows, int max_cols, float *image_dev, int *rows, int *cols,
                       void *stream);

/* ---------------------------------------------------------------------------
 * Device-resident major cycle of the FFT imaging pipeline
 * (code_fft_1core/generated/Core0.c, delta_k / psi_k):
 *   model image -> [shift, FFT, shift] -> model grid -> [degrid, subtract
 *   from measured, grid] -> residual grid -> [shift, iFFT, shift, taper]
 *   -> residual image -> [Hogbom] -> components, model image += components.
 * The model image starts at zero; each call of sdp_pipeline_major_cycle runs
 * one cycle on the stream (captured once as a CUDA graph when use_graph).
 * ------------------------------------------------------------------------- */
enum { SDP_COORD_F32 = 0, SDP_COORD_F64 = 1 };

typedef struct sdp_pipeline_config {
    int grid_size;            /* power of two, 16..16384                                  */
    int oversampling;
    double uv_scale, w_scale, cell_size;
    int num_minor_cycles, max_sources;
    double loop_gain, noise_factor, weak_source_percent, psf_max_value;
    int degrid_mode;          /* SDP_DEGRID_NEAREST (reference) or SDP_DEGRID_CONV        */
    int coord_mode;           /* SDP_COORD_F32 (float build) or SDP_COORD_F64 (double build) */
    int snap;                 /* 1: the uvw given are raw and are snapped to the fine grid */
    int use_graph;            /* 1: capture the cycle as a CUDA graph                      */
} sdp_pipeline_config;

typedef struct sdp_pipeline sdp_pipeline;
/* uvw and measured (N each) are device pointers; psf (G^2, normalised to
 * peak 1) may be host or device memory.  All three are copied.  The kernel
 * tables are copied when the oversampling is a power of two; otherwise the
 * pipeline reads the caller's tables, which must outlive it. */
int sdp_pipeline_create(sdp_pipeline **p, const sdp_pipeline_config *cfg, const sdp_wkernels *grid_kernels,
                        const sdp_wkernels *degrid_kernels, int num_vis, const sdp_float3 *uvw,
                        const sdp_float2 *measured, const float *psf, void *stream);
int sdp_pipeline_major_cycle(sdp_pipeline *p, void *stream);
/* Device pointers owned by the pipeline: the last cycle's residual image,
 * the model image, the last cycle's components (x, y in radians, flux) and
 * their count. */
int sdp_pipeline_outputs(sdp_pipeline *p, float **residual_image, float **model_image, sdp_float3 **sources,
                         int **num_sources);
/* Copies the outputs (host or device destinations, any may be NULL;
 * sources: max_sources entries) and synchronises the stream. */
int sdp_pipeline_copy_outputs(sdp_pipeline *p, float *residual_image, float *model_image, sdp_float3 *sources,
                              int *num_sources, void *stream);
int sdp_pipeline_graph_active(const sdp_pipeline *p);
/* Why the graph capture was refused ("" when it was not). */
const char *sdp_pipeline_graph_error(const sdp_pipeline *p);
int sdp_pipeline_visplan(sdp_pipeline *p, sdp_visplan **plan);
int sdp_pipeline_destroy(sdp_pipeline *p);

/* ---------------------------------------------------------------------------
 * Learned CLEAN proposals (no counterpart in the reference, whose only
 * deconvolution is Hogbom, deconvolution_run.c:197-311).  A 4-level U-Net
 * (base 32 channels, 3x3 convolutions, 2x2 mean pooling, nearest
 * upsampling, skip concatenations, one-channel 1x1 output head) maps the
 * residual image and the PSF to a sky map; its largest values become a batch
 * of components, which the caller verifies through an exact major cycle and
 * rejects in favour of Hogbom when the residual RMS does not fall.
 * BF16 weights and activations, FP32 accumulation, FP32 master weights,
 * forward and backward passes and Adam on the device.
 * ------------------------------------------------------------------------- */
typedef struct sdp_unet sdp_unet;
/* Images up to max_batch x max_height x max_width (sides multiples of 8);
 * in_channels 1..32; base_channels 32; training = 0 allocates no gradient
 * or optimiser buffers.  Parameters start at zero (see sdp_unet_set_params). */
int sdp_unet_create(sdp_unet **net, int base_channels, int in_channels, int max_batch, int max_height,
                    int max_width, int training);
int sdp_unet_destroy(sdp_unet *net);
/* Flat FP32 parameter vector: for each 3x3 layer (0..13: e0a e0 e1a e1 e2a
 * e2 e3a e3 d2a d2 d1a d1 d0a d0) the weights [9][out][in] (tap = 3 (dy+1) +
 * (dx+1); layer 0's input is padded to 32 channels) then the bias [out];
 * then the head (layer 14): weights [base], bias [1]. */
int sdp_unet_num_params(const sdp_unet *net, size_t *count);
int sdp_unet_layer(const sdp_unet *net, int layer, int *in_channels, int *out_channels, size_t *weight_offset,
                   size_t *bias_offset);
/* Host or device pointers (cudaMemcpyDefault); set resets the Adam state. */
int sdp_unet_set_params(sdp_unet *net, const float *params, void *stream);
int sdp_unet_get_params(const sdp_unet *net, float *params, void *stream);
int sdp_unet_get_grads(const sdp_unet *net, float *grads, void *stream);
int sdp_unet_zero_grads(sdp_unet *net, void *stream);
/* input [batch][in_channels][height][width] FP32 (device); scale (device,
 * [batch], or NULL): every input channel is divided and the output
 * multiplied by it; output [batch][height][width] FP32 (device).  Keeps the
 * activations for sdp_unet_backward. */
int sdp_unet_forward(sdp_unet *net, int batch, int height, int width, const float *input, const float *scale,
                     float *output, void *stream);
/* Adds d(loss)/d(params) for d(loss)/d(output) = grad_output (the last
 * forward's shape; scale NULL) to the gradient vector. */
int sdp_unet_backward(sdp_unet *net, const float *grad_output, void *stream);
/* Convolution engine: 1 (default) tcgen05 tensor cores with the accumulator
 * in tensor memory (TMA-fed, warp-specialised); 0 the mma.sync kernel (kept
 * for comparison). */
int sdp_unet_set_tensor_path(sdp_unet *net, int tcgen05);
/* Blocking: SDP_ERR_TIMEOUT when a tensor-core convolution gave up a bounded
 * wait since the last check (its outputs are then incomplete), else SDP_OK. */
int sdp_unet_check(sdp_unet *net, void *stream);
/* No counterpart in the reference: the failure path of the tensor-core
 * convolution.  Sets how many times its epilogue polls for a finished
 * accumulator before it gives up (0: the default, about a second).  A tiny
 * limit makes the wait run out on purpose: the kernel then drains the copies
 * and MMAs it had issued, returns, and sdp_unet_check reports
 * SDP_ERR_TIMEOUT; the outputs of that pass are incomplete. */
int sdp_unet_set_wait_limit(sdp_unet *net, long long epilogue_polls);
/* One Adam step on the master weights (bias-corrected moments). */
int sdp_unet_adam_step(sdp_unet *net, float lr, float beta1, float beta2, float eps, void *stream);
/* loss = mean over pixels of (b * (pred - target))^2, b the 3x3 binomial
 * blur (zero padding per image); grad (may be NULL) = d(loss)/d(pred);
 * diff_scratch holds 2 x batch x height x width floats; loss a device double. */
int sdp_blur_mse(int batch, int height, int width, const float *pred, const float *target, float *diff_scratch,
                 float *grad, double *loss, void *stream);
/* The network's input planes from a residual image (all device, G^2 each):
 * r / s, sign(r) sqrt(|r| / s), psf, with s = max |r| written to scale_dev. */
int sdp_unet_input_planes(int grid_size, const float *residual, const float *psf, float *planes, float *scale_dev,
                          void *stream);
/* The same planes for the centred window x 0 .. window-1 of the image,
 * offset (grid_size - window) / 2 in both axes (planes are window^2 each; s
 * is the whole image's max |r|).  A network run on the window gives the
 * full-image run's output wherever its receptive field stays inside the
 * window; with the offset a multiple of 16 its pooling levels line up. */
int sdp_unet_input_planes_window(int grid_size, int window, const float *residual, const float *psf, float *planes,
                                 float *scale_dev, void *stream);
/* Components from a proposal image: the largest values (signed_values = 0:
 * positive values; 1: largest |value|, either sign) at or above
 * rel_threshold x the maximum, at most max_count of them (whole histogram
 * bins from the top), as (l, m, value x scale, 0) with l = (x - G/2) cell,
 * m = (y - G/2) cell; *count_dev receives their number; delta_image (may be
 * NULL) receives them as an image.  workspace: sdp_select_workspace_bytes. */
int sdp_select_workspace_bytes(size_t *bytes);
int sdp_select_components(int grid_size, double cell_size, const float *proposal, const float *scale_dev,
                          int signed_values, float rel_threshold, int max_count, sdp_float4 *components,
                          int *count_dev, float *delta_image, void *workspace, void *stream);
/* dots_dev[0] = <a, b>, dots_dev[1] = <b, b>, summed in FP64. */
int sdp_dots(long long n, const float *a, const float *b, double *dots_dev, void *stream);
/* y += sign x alpha x with alpha = clamp(dots[0] / dots[1], 0, alpha_max)
 * (the least-squares step of a proposal); alpha_dev (may be NULL) receives
 * alpha. */
int sdp_axpy_ratio(long long n, const double *dots_dev, double alpha_max, float sign, const float *x, float *y,
                   float *alpha_dev, void *stream);
int sdp_scale(long long n, float *x, float factor, void *stream);
/* Zeroes the pixels within `border` of the edges of a G x G image (the
 * proposal window of the learned cycle: the outer band of the image carries
 * the taper correction's amplified imaging errors, not sources). */
int sdp_zero_border(int grid_size, int border, float *image, void *stream);
/* Adds components (l, m, flux, sigma) to a G x G image: points (sigma = 0)
 * at the nearest pixel, circular Gaussians of standard deviation sigma
 * (direction cosines) sampled over +-4 sigma. */
int sdp_sky_render(int grid_size, double cell_size, int num, const sdp_float4 *components, float *image,
                   void *stream);
/* DFT predict of components on the pixel grid (CLEAN components, network
 * proposals): component k = (l, m, flux, ...) at components + k * stride
 * floats, l and m multiples of cell_size (rounded to the nearest pixel
 * offset); the sdp_dft formula with the phase reduced modulo one cycle in
 * fixed point (error below 1e-6 rad for offsets up to 2048 pixels).
 * accumulate = 1 adds to vis. */
int sdp_dft_pixels(int num_vis, int num_components, const float *components, int stride, double cell_size,
                   const sdp_float3 *uvw, sdp_float2 *vis, int accumulate, void *stream);
/* DFT predict of points and circular Gaussians (l, m, flux, sigma): the
 * sdp_dft term times exp(-2 pi^2 sigma^2 (u^2 + v^2)). */
int sdp_dft_gauss(int num_vis, int num_sources, const sdp_float4 *sources, const sdp_float3 *uvw, sdp_float2 *vis,
                  void *stream);

/* Failure-detection self test (no counterpart in the reference): launches
 * nblocks (1..64) blocks that each publish a result and wait, with the wait
 * the persistent CLEAN kernel uses, for one result more than there are
 * blocks.  Each wait gives up after spin_limit polls (a ~32 ns sleep and an
 * L2 read each), so the kernel ends; *status receives SDP_ERR_TIMEOUT when
 * the bounded wait reported the timeout (the expected result), SDP_OK
 * otherwise. */
int sdp_selftest_bounded_wait(int nblocks, long long spin_limit, int *status);
/* The same for the SVD's grid barrier (sdp_svd): a barrier expecting one CTA
 * more than launched; *status = SDP_ERR_TIMEOUT when its waits ran out. */
int sdp_selftest_svd_barrier(int nblocks, long long spin_limit, int *status);

/* Measured on-chip ceilings (no counterpart in the reference): the
 * denominators of the roofline fractions of kernels that HBM does not bound.
 *   SDP_PEAK_L2_READ        bytes/s of 16-byte L1-bypassing loads from the
 *                           L2-resident part of scratch (pass 32 MB or so)
 *   SDP_PEAK_SMEM_READ      bytes/s of conflict-free 16-byte shared loads
 *   SDP_PEAK_FP32_FMA       FLOP/s of scalar FP32 fused multiply-adds
 *   SDP_PEAK_FP32X2_FMA     FLOP/s of packed two-lane FP32 multiply-adds
 *   SDP_PEAK_HOGBOM_UPDATE  pixel updates/s of the Hogbom residual update
 *                           float(double(r) - (scale * double(psf)) * psf_max)
 * scratch: a 16-byte aligned device buffer of at least 4096 bytes; reps
 * timed launches after one warm-up launch on `stream` (blocking). */
enum {
    SDP_PEAK_L2_READ = 0,
    SDP_PEAK_SMEM_READ = 1,
    SDP_PEAK_FP32_FMA = 2,
    SDP_PEAK_FP32X2_FMA = 3,
    SDP_PEAK_HOGBOM_UPDATE = 4
};
int sdp_peak_measure(int kind, void *scratch, size_t scratch_bytes, int reps, double *rate, void *stream);

#ifdef __cplusplus
}
#endif
#endif
