/*
 * mbir_b200.h -- C ABI of the sm_100a MBIR hot path.
 *
 * Plain pointers and sizes only: every array argument is a DEVICE pointer
 * (CUDA global memory of the current device) unless stated otherwise, and
 * every entry point enqueues work on the CUDA stream passed as `stream`
 * (a cudaStream_t; NULL means the legacy default stream).  Nothing here
 * allocates device memory: callers pass output buffers and, where a
 * function needs scratch space, a workspace whose size the matching
 * *_workspace_size() function reports.
 *
 * Error behaviour: every function returns MBIR_OK (0) or a nonzero code and
 * records a message readable with mbir_last_error() (thread-local).  Invalid
 * arguments are rejected on the host before any launch.
 *
 * Sinogram layouts:
 *   MBIR_LAYOUT_VRC  (views, detector rows, channels) -- the reference's
 *                    public sinogram layout, channel contiguous.
 *   MBIR_LAYOUT_VCR  (views, channels, detector rows) -- channel-major, row
 *                    contiguous: the resident layout of the VCD state, in
 *                    which the projectors' row walks are unit-stride.
 *
 * Reference interfaces replaced (mbirtorch v0.0.2, file:line):
 *   mbir_forward_project  <- _parallel_forward_view_batch
 *                            (parallel_beam.py:56-73) and
 *                            _cone_forward_view_batch (cone_beam.py:161-234),
 *                            the bodies bound by _view_batch_bodies
 *                            (parallel_beam.py:234-276, cone_beam.py:354-395)
 *                            and driven by Projectors.
 *                            sparse_forward_project_view_range
 *                            (projectors.py:518-588)
 *   mbir_forward_project_binned <- the same bodies for whole cylinders, through
 *                            channel-sorted bins (forward_project,
 *                            tomography_model.py:1877-1909)
 *   mbir_back_project     <- _parallel_back_view_batch (parallel_beam.py:76-94)
 *                            and _cone_back_view_batch (cone_beam.py:237-299),
 *                            driven by sparse_back_project_view_range
 *                            (projectors.py:590-646); coeff_power 2 is
 *                            compute_hessian_diagonal
 *                            (tomography_model.py:1951-2032)
 *   mbir_vcd_subset_update <- the callable returned by
 *                            create_vcd_subset_updater
 *                            (tomography_model.py:2434-2660), with the qGGMRF
 *                            prior of qggmrf.py:77-183 and the cone DC
 *                            damping of cone_beam.py:45-55, 479-496
 *   mbir_vcd_partition_pass <- vcd_partition_iterator
 *                            (tomography_model.py:2662-2697)
 *   mbir_iteration_stats  <- _vcd_iteration_stats / get_forward_model_loss
 *                            (tomography_model.py:2325-2393)
 *   mbir_error_init       <- _initial_error_state (tomography_model.py:1666-1712)
 *   mbir_sino_convert     <- the host->device placement of the sinogram,
 *                            _shard_sinogram (tomography_model.py:1490-1512),
 *                            plus the storage-precision conversion
 */
#ifndef MBIR_B200_H
#define MBIR_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define MBIR_OK 0
#define MBIR_ERR_INVALID 1     /* bad argument (caught on the host) */
#define MBIR_ERR_CUDA 2        /* a CUDA call failed */
#define MBIR_ERR_WORKSPACE 3   /* workspace too small */

#define MBIR_PARALLEL 0
#define MBIR_CONE 1

#define MBIR_LAYOUT_VRC 0
#define MBIR_LAYOUT_VCR 1

#define MBIR_F32 0
#define MBIR_BF16 1
#define MBIR_F16 2

/* Largest tap radius (psf_radius, bp_psf_radius) the kernels unroll. */
#define MBIR_MAX_TAP_RADIUS 3

/* Geometry of one model: the scalars of the reference's _view_batch_args
 * (parallel_beam.py:278-291, cone_beam.py:397-414).  Parallel beam reads
 * only the channel and in-plane voxel fields and psf_radius; its detector
 * row count must equal num_slices. */
typedef struct mbir_geometry {
    int32_t geometry;              /* MBIR_PARALLEL or MBIR_CONE */
    int32_t num_views;             /* views in view_params */
    int32_t num_det_rows;
    int32_t num_det_channels;
    int32_t num_recon_rows;
    int32_t num_recon_cols;
    int32_t num_slices;            /* full slice count (the z anchor) */
    int32_t psf_radius;            /* channel taps; cone back row taps */
    int32_t bp_psf_radius;         /* cone forward slice taps */
    int32_t use_curved_detector;
    float delta_det_channel;
    float delta_det_row;
    float det_channel_offset;
    float det_row_offset;
    float delta_voxel;
    float delta_voxel_row;
    float delta_voxel_slice;
    float recon_slice_offset;
    float magnification;
    float source_detector_dist;    /* +inf allowed (parallel-ray limit) */
} mbir_geometry;

/* Regularization and line-search scalars of one reconstruction
 * (create_vcd_subset_updater, tomography_model.py:2472-2482). */
typedef struct mbir_vcd_params {
    float fm_constant;   /* 1 / sigma_y^2 */
    float sigma_x;
    float p;
    float q;
    float T;
    float b[6];          /* neighbour weights: row+1, row-1, col+1, col-1,
                            slice+1, slice-1 (get_b_from_nbr_wts) */
    float max_alpha;
    int32_t positivity;  /* clip so that recon + alpha * delta >= 0 */
    int32_t storage;     /* MBIR_F32 / MBIR_BF16 / MBIR_F16 for the error
                            sinogram, the weights and the delta sinogram */
    /* Proximal-map prior (prox_map, tomography_model.py:3251-3373, with the
     * gradient of qggmrf.py:186-206 and the scalar Hessian of
     * tomography_model.py:2530-2537).  prox_input == NULL selects the
     * qGGMRF prior and the two fields below are ignored; otherwise the
     * prior's gradient is prox_constant * (x - prox_input) and its Hessian
     * prox_constant. */
    float prox_constant;          /* 1 / sigma_prox^2, > 0 */
    int32_t reserved;             /* zero */
    const float *prox_input;      /* (N*N, S) f32 device array, like flat_recon */
} mbir_vcd_params;

/* Version of this ABI (major * 10000 + minor * 100 + patch). */
int32_t mbir_abi_version(void);

/* Message of the last failed call on this thread ("" if none). */
const char *mbir_last_error(void);

/* Number of kernel launches this library has issued in this process (a
 * diagnostic counter; no counterpart in the reference, which launches
 * through Triton). */
unsigned long long mbir_launch_count(void);

/* Per-kernel timing (diagnostic; no counterpart in the reference).  While
 * enabled, every kernel launch of this library is bracketed by two CUDA
 * events recorded on the launch's own stream.  mbir_timing_enable returns
 * the previous setting.  mbir_timing_collect waits for the recorded
 * events, writes up to max_entries kernel names ('\n'-separated, into the
 * HOST buffer names), their summed milliseconds and launch counts (HOST
 * arrays), clears the record and returns the number of entries. */
int32_t mbir_timing_enable(int32_t on);
int32_t mbir_timing_collect(char *names, int32_t names_bytes, double *total_ms,
                            int64_t *counts, int32_t max_entries);

/* Forward projection of voxel cylinders onto views
 * [view_start, view_start + view_count):
 *   values         (num_pixels, band_len) f32, slice axis contiguous; a band
 *                  of global slices [slice_start, slice_start + band_len)
 *   pixel_indices  (num_pixels) int64 into the flattened recon grid
 *   view_params    (num_views, 2) f32: angle, helical z shift (parallel
 *                  reads the angle only)
 *   sino_out       (view_count, R, C) or (view_count, C, R) f32 per
 *                  out_layout, OVERWRITTEN (parallel: R == band_len).
 * Deterministic: no atomics, fixed summation order. */
int32_t mbir_forward_project(const mbir_geometry *geom, const float *view_params,
                             int32_t view_start, int32_t view_count,
                             const float *values, int64_t num_pixels,
                             int32_t band_len, int32_t slice_start,
                             const int64_t *pixel_indices, float *sino_out,
                             int32_t out_layout, void *stream);

/* Forward projection of whole cylinders read straight from a flat
 * (N*N, num_slices) f32 volume at the rows pixel_indices[p] (no gathered
 * copy); otherwise as mbir_forward_project with slice_start 0 and
 * band_len num_slices.  Replaces the gather + sparse_forward_project of
 * forward_project (tomography_model.py:1877-1909). */
int32_t mbir_forward_project_volume(const mbir_geometry *geom, const float *view_params,
                                    int32_t view_start, int32_t view_count,
                                    const float *flat_volume, const int64_t *pixel_indices,
                                    int64_t num_pixels, float *sino_out, int32_t out_layout,
                                    void *stream);

/* Forward projection of whole cylinders through channel-sorted bins: per
 * chunk of views, every (view, pixel) record is formed once and sorted by
 * centre channel, and each (view, 16-channel block) CTA walks only the
 * pixels that reach it (the scanning forward above tests every pixel in
 * every block).  Same operator as mbir_forward_project_volume (values_by_pixel
 * 1: values is the flat (N*N, num_slices) volume read at rows
 * pixel_indices[p]) or mbir_forward_project with slice_start 0 and band_len
 * num_slices (values_by_pixel 0: values is (num_pixels, num_slices)); the
 * sums run in another fixed order, so results agree with those to FP32
 * rounding.  Covers the geometries with psf radius 1 and at most 1024
 * detector rows (MBIR_ERR_INVALID otherwise).  The workspace (256-byte
 * aligned) holds the bins of as many views as fit; a larger one means fewer
 * chunks.  Replaces _parallel_forward_view_batch / _cone_forward_view_batch
 * (parallel_beam.py:56-73, cone_beam.py:161-234) for whole volumes. */
int32_t mbir_forward_project_binned(const mbir_geometry *geom, const float *view_params,
                                    int32_t view_start, int32_t view_count,
                                    const float *values, int32_t values_by_pixel,
                                    const int64_t *pixel_indices, int64_t num_pixels,
                                    float *sino_out, int32_t out_layout, void *workspace,
                                    size_t workspace_bytes, void *stream);

/* Workspace bytes for mbir_forward_project_binned: the bins of
 * min(view_count, views whose records fit 1 GiB) views, at least one; 0 when
 * the geometry is not covered. */
size_t mbir_forward_project_binned_workspace_size(const mbir_geometry *geom,
                                                  int32_t view_count, int64_t num_pixels);

/* Workspace bytes mbir_back_project needs for this call shape. */
size_t mbir_back_project_workspace_size(const mbir_geometry *geom,
                                        int32_t view_count, int64_t num_pixels,
                                        int32_t band_len);

/* Back projection (adjoint) of views [view_start, view_start + view_count):
 *   sino        (view_count, ...) f32 in sino_layout
 *   out         (num_pixels, band_len) f32, OVERWRITTEN with the sum over the
 *               views; coeff_power 1 or 2 (2 squares every weight: the
 *               Hessian diagonal).
 * Deterministic: view chunks reduce in a fixed order. */
int32_t mbir_back_project(const mbir_geometry *geom, const float *view_params,
                          int32_t view_start, int32_t view_count,
                          const float *sino, int32_t sino_layout,
                          const int64_t *pixel_indices, int64_t num_pixels,
                          int32_t coeff_power, int32_t slice_start,
                          int32_t band_len, float *out, void *workspace,
                          size_t workspace_bytes, void *stream);

/* mbir_back_project for callers that cannot allocate device memory (no
 * counterpart in the reference, whose bodies allocate through torch).
 * An application whose device memory belongs to another allocator -- a
 * framework's caching pool, a pipeline with a fixed memory budget -- cannot
 * hand this library a fresh workspace, and a cudaMalloc of our own would
 * bypass that owner.  This variant allocates nothing: its scratch is a
 * file-scope device array of 32 MiB that every GPU loading the library
 * holds until the process exits.  It holds the channel-major copy of a
 * (views, rows, channels) input (such an input above 32 MiB is rejected
 * with MBIR_ERR_WORKSPACE; pass the channel-major layout instead) and the
 * view-chunk partial sums, whose count shrinks to fit.  The first call on
 * each device looks up the array's device address (cudaGetSymbolAddress,
 * with that device current), so make the first call on a device before any
 * stream capture.  All calls share the array: calls that overlap on the GPU
 * race on it.  Arguments and results are those of mbir_back_project. */
int32_t mbir_back_project_noalloc(const mbir_geometry *geom, const float *view_params,
                                  int32_t view_start, int32_t view_count,
                                  const float *sino, int32_t sino_layout,
                                  const int64_t *pixel_indices, int64_t num_pixels,
                                  int32_t coeff_power, int32_t slice_start,
                                  int32_t band_len, float *out, void *stream);

/* Layout / precision conversion of a whole sinogram between the public f32
 * VRC form and the resident VCR form in `dtype` with a per-view scale:
 * stored = value / scale[v].  direction 0: f32 VRC -> dtype VCR (computing
 * scale[v] when compute_scale != 0: 1 for f32/bf16, max|value_v| / 256 for
 * f16); direction 1: dtype VCR -> f32 VRC (reading scale). */
int32_t mbir_sino_convert(int32_t direction, int32_t views, int32_t rows,
                          int32_t channels, const void *src, void *dst,
                          int32_t dtype, float *scale, int32_t compute_scale,
                          void *stream);

/* Initial error state: error = y - alpha * Ax with
 * alpha = <w Ax, y> / <w Ax, Ax> when scale_to_data != 0 and the
 * denominator is positive, else 1 (FP64 reductions).  y and ax are f32 VRC;
 * weights may be NULL (unit weights).  error_out (same layout) may alias y.
 * alpha_out is a device f64 scalar. */
int32_t mbir_error_init(int64_t count, const float *y, const float *ax,
                        const float *weights, int32_t scale_to_data,
                        float *error_out, double *alpha_out, void *workspace,
                        size_t workspace_bytes, void *stream);
size_t mbir_error_init_workspace_size(int64_t count);

/* Workspace bytes for mbir_vcd_subset_update / mbir_vcd_partition_pass with
 * subsets of at most max_subset_pixels pixels. */
size_t mbir_vcd_workspace_size(const mbir_geometry *geom,
                               int64_t max_subset_pixels,
                               const mbir_vcd_params *params);

/* One VCD subset update, in place (recon and error sinogram):
 *   flat_recon   (N*N, S) f32
 *   error_sino   (V, C, R) in params->storage, stored / err_scale[v]
 *   weights      same layout and dtype, / w_scale[v]; NULL = unit weights
 *   fm_hessian   (N*N, S) f32 Hessian diagonal of the data term
 *   dc_profile   (S) f32 slice damping s_k, or NULL (no damping)
 *   accum        device f64 accumulators, 2 + S entries, ADDED to:
 *                [0] += ell1 of the update, [1] += alpha, [2 + k] += per-
 *                slice sum of squared updates.
 *   alpha_out    device f32 scalar receiving this subset's alpha (or NULL). */
int32_t mbir_vcd_subset_update(const mbir_geometry *geom,
                               const float *view_params,
                               const mbir_vcd_params *params, float *flat_recon,
                               void *error_sino, const float *err_scale,
                               const void *weights, const float *w_scale,
                               const float *fm_hessian, const float *dc_profile,
                               const int64_t *pixel_indices, int64_t num_pixels,
                               double *accum, float *alpha_out, void *workspace,
                               size_t workspace_bytes, void *stream);

/* One VCD iteration over a partition: the subsets of `partition`
 * (num_subsets, subset_pixels) int64 are updated in the order given by the
 * HOST array `order` (num_subsets entries), each exactly as
 * mbir_vcd_subset_update.  accum as above (summed over the subsets). */
int32_t mbir_vcd_partition_pass(const mbir_geometry *geom,
                                const float *view_params,
                                const mbir_vcd_params *params, float *flat_recon,
                                void *error_sino, const float *err_scale,
                                const void *weights, const float *w_scale,
                                const float *fm_hessian, const float *dc_profile,
                                const int64_t *partition, int32_t num_subsets,
                                int64_t subset_pixels, const int32_t *order,
                                double *accum, void *workspace,
                                size_t workspace_bytes, void *stream);

/* Up to MBIR_MAX_BATCH reconstructions that share a geometry, stepped
 * together (no counterpart in the reference, which reconstructs one job at
 * a time; the serving layer's cross-job batching): each subset index i
 * updates subset order[j][i] of job j, exactly as mbir_vcd_partition_pass
 * would for that job alone, but each kernel of the subset step is launched
 * once for all jobs (job index on grid z).  The arguments are HOST arrays
 * of num_jobs entries -- params and the per-job device pointers -- plus
 * order, a HOST (num_jobs, num_subsets) int32 array.  The jobs must agree
 * in storage, positivity, prior kind and weighting; their regularization
 * scalars may differ.  Each job has its own workspace (workspace_bytes
 * each) and its own accumulators.  Geometries that the binned subset path
 * does not cover step their jobs one after another. */
#define MBIR_MAX_BATCH 16
int32_t mbir_vcd_partition_pass_batched(
    int32_t num_jobs, const mbir_geometry *geom, const float *view_params,
    const mbir_vcd_params *params, float *const *flat_recon, void *const *error_sino,
    const float *const *err_scale, const void *const *weights, const float *const *w_scale,
    const float *const *fm_hessian, const float *dc_profile, const int64_t *const *partition,
    int32_t num_subsets, int64_t subset_pixels, const int32_t *order, double *const *accum,
    void *const *workspace, size_t workspace_bytes, void *stream);

/* Workspace bytes for mbir_denoise_pass with subsets of subset_pixels
 * pixels of an image with num_slices slices. */
size_t mbir_denoise_workspace_size(int32_t num_slices, int64_t subset_pixels);

/* One QGGMRF-denoiser iteration (QGGMRFDenoiser.denoise's inner loop and
 * vcd_subset_denoiser, denoising.py:35-83 and :390-425): the identity
 * forward model, so the residual image plays the error sinogram.  The
 * subsets of `partition` (num_subsets, subset_pixels) int64 are updated in
 * their stored order (the denoiser never reshuffles).
 *   flat_image, flat_error   (num_rows * num_cols, num_slices) f32, updated
 *                            in place (error = noisy image - image)
 *   params                   fm_constant = 1 / sigma_noise^2, the qGGMRF
 *                            scalars and max_alpha; storage, positivity and
 *                            the proximal fields are ignored
 *   accum                    device f64 [2], ADDED to: sum |alpha delta|,
 *                            sum alpha over the subsets */
int32_t mbir_denoise_pass(int32_t num_rows, int32_t num_cols, int32_t num_slices,
                          const mbir_vcd_params *params, float *flat_image,
                          float *flat_error, const int64_t *partition,
                          int32_t num_subsets, int64_t subset_pixels, double *accum,
                          void *workspace, size_t workspace_bytes, void *stream);

/* Re-form the resident error sinogram from the measured one:
 * error = (y - A x) / err_scale[v] in `storage`, with y the FP32 sinogram
 * in the (V, C, R) layout and x the flat (N*N, S) recon at pixel_indices.
 * Part of the storage-precision layer (no counterpart in the reference,
 * whose error sinogram is FP32 and updated in place only): it bounds the
 * drift that in-place 16-bit updates accumulate.  With a workspace of
 * mbir_forward_project_binned_workspace_size(geom, num_views, num_pixels)
 * bytes (256-byte aligned; any size holding one view's bins) A x is formed
 * through the channel-sorted bins; with none (NULL), by the scanning
 * forward. */
int32_t mbir_vcd_refresh_error(const mbir_geometry *geom, const float *view_params,
                               const float *flat_recon, const int64_t *pixel_indices,
                               int64_t num_pixels, const float *y_vcr, void *error_sino,
                               const float *err_scale, int32_t storage, void *workspace,
                               size_t workspace_bytes, void *stream);

/* Per-iteration statistics in FP64 (device out[4]):
 *   out[0] = sum(w e^2)  (sum(e^2) without weights)
 *   out[1] = sum(w)      (count without weights)
 *   out[2] = sum(e^2)
 *   out[3] = sum(|x|) over flat_recon (recon_count entries). */
int32_t mbir_iteration_stats(int32_t views, int32_t rows, int32_t channels,
                             const void *error_sino, const float *err_scale,
                             const void *weights, const float *w_scale,
                             int32_t storage, const float *flat_recon,
                             int64_t recon_count, double *out, void *workspace,
                             size_t workspace_bytes, void *stream);
size_t mbir_iteration_stats_workspace_size(void);

#ifdef __cplusplus
}
#endif

#endif /* MBIR_B200_H */
