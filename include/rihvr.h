/*
 * rihvr.h - C ABI of the B200 reconstruction core.
 *
 * Drop-in boundary for RIHVR's sparse inverse reconstruction path
 * (FASTA/FISTA with L1 + TV regularisation over a Rayleigh-Sommerfeld model).
 * Every entry point names the reference interface it replaces; paths are
 * relative to the RIHVR source tree (src/core/...).
 *
 * Conventions
 *  - Status codes: 0 on success; 1..12 are the reference's umnholo::HoloError
 *    values (src/core/umnholo.h:132-146); 20+ are runtime conditions.  No C++
 *    exception crosses this boundary.
 *  - Complex arrays are interleaved float pairs (re, im), row-major,
 *    volumes ordered [plane][row][column].
 *  - `is_device` != 0 means the pointer is CUDA device memory borrowed for the
 *    duration of the call; otherwise it is host memory.
 *  - A context owns all device memory it allocates and runs on its own CUDA
 *    stream; calls on one context are not re-entrant.
 */
#ifndef RIHVR_H
#define RIHVR_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

enum rihvr_status {
  RIHVR_OK = 0,
  /* umnholo::HoloError (src/core/umnholo.h:132-146) */
  RIHVR_ERR_UNKNOWN_TYPE = 1,
  RIHVR_ERR_BAD_FILENAME = 2,
  RIHVR_ERR_MISSING_DATA = 3,
  RIHVR_ERR_INVALID_STATE = 4,
  RIHVR_ERR_OUT_OF_MEMORY = 5,
  RIHVR_ERR_UNKNOWN_MODE = 6,
  RIHVR_ERR_INVALID_ARGUMENT = 7,
  RIHVR_ERR_UNKNOWN_ERROR = 8,
  RIHVR_ERR_INVALID_FILE = 9,
  RIHVR_ERR_INVALID_DATA = 10,
  RIHVR_ERR_CRITICAL_ASSUMPTION = 11,
  RIHVR_ERR_INFINITE_LOOP = 12,
  /* runtime conditions (the reference throws CUDA_ERROR_UNKNOWN, umnholo.h:14-34) */
  RIHVR_ERR_CUDA = 20,
  RIHVR_ERR_NO_DEVICE = 21,
  RIHVR_ERR_UNSUPPORTED_SIZE = 22
};

/* Reconstruction modes: umnholo::CompressiveHoloMode (src/core/compressive_holo.h:20-29). */
enum rihvr_mode {
  RIHVR_MODE_FASTA_L1 = 5,
  RIHVR_MODE_FASTA_FUSED_LASSO = 6,    /* L1 + 3-D TV */
  RIHVR_MODE_FASTA_FUSED_LASSO_2D = 7  /* L1 + per-plane 2-D TV (the CLI default) */
};

/* Storage of the three iterate volumes; arithmetic is FP32 in every case.
 * FP16 keeps the objective within 1e-2 of the FP64 solution (2.6e-4 at the
 * 1024 x 1024 x 1000 workload).  BF16 does not (2.3e-2 there: its 8-bit
 * mantissa adds rounding noise to every stored iterate, and the objective gap
 * grows with its square), so rihvr_create accepts BF16 only with
 * faithful = 0, where no agreement with the reference is claimed. */
enum rihvr_storage { RIHVR_STORE_F32 = 0, RIHVR_STORE_BF16 = 1, RIHVR_STORE_F16 = 2 };

/* Solver parameters.  The first block mirrors umnholo::Parameters
 * (src/core/holo_ui.h:83-145), kept in float like the reference; the second
 * block selects build options that have no reference counterpart. */
typedef struct rihvr_params {
  float start_plane;             /* 3001  z0 */
  float plane_stepsize;          /* 3002  dz */
  int num_planes;                /* 3003  Nz */
  float wavelength;              /* 3004  lambda (same length unit as dx and z) */
  float resolution;              /* 3005  dx, pixel pitch */
  int zero_padding;              /* 3010  pixels added on every side */
  int num_inverse_iterations;    /* 6001  FISTA iterations */
  float regularization_param;    /* 6002  L1 (sparsity) weight */
  float regularization_TV_param; /* 6004  TV weight; 0 selects the L1-only prox */
  int num_tv_iterations;         /* 6005  Chambolle iterations per prox (0..20) */
  int mode;                      /* rihvr_mode, default 7 */
  int storage;                   /* rihvr_storage of the volumes, default FP32 */
  int faithful;                  /* 1 (default): reference arithmetic - separable
                                    complex shrink and the restart statistic as the
                                    reference sums it; 0: complex-modulus shrink
                                    and the plain restart dot product */
  int max_backtracks;            /* 2 in the reference (sparse_compressive_holo.cu:423) */
  double initial_step;           /* <= 0: 1/num_planes as the reference (:247) */
  int record_objective;          /* 1: objective terms at every iteration */
  int autotune;                  /* 1: rihvr_set_hologram tunes launch shapes once (rihvr_autotune) */
} rihvr_params;

/* Per-iteration record (what inverseReconstruct prints, :561-565, plus terms). */
typedef struct rihvr_iter_record {
  double f_prox;       /* objective at the accepted prox output */
  double f_resid_prox; /* 0.5 ||A p - b||^2 */
  double lim;          /* line-search limit (calcLineSearchLimit, :4307-4390) */
  double ratio;        /* backtracking ratio of the accepted step (:402-403) */
  double t;            /* step size used */
  double beta;         /* momentum factor (alpha0 - 1) / alpha1 */
  double f_x;          /* objective at the momentum point ("new f", :548) */
  double f_resid_x;    /* 0.5 ||A x - b||^2 at the momentum point */
  double l1_x, tv_x;   /* regulariser norms at the momentum point */
  double restart_sum;  /* restart statistic (fistaRestart, :4434-4482) */
  int backtracks;
  int restarted;
} rihvr_iter_record;

/* File-level fields of the .param format the CLI needs (holo_ui.h:83-145). */
typedef struct rihvr_file_params {
  char image_filename[4096];       /* 2001, or 2002 + 2003 */
  char image_path[4096];           /* 2002 */
  char image_formatted_name[4096]; /* 2003 */
  char output_path[4096];          /* 2004 */
  char background_filename[4096];  /* 2005 */
  int remove_background;           /* set by 2005 */
  int image_count;                 /* 1001 */
  int start_image;                 /* 1002 */
  int roi_x, roi_y, roi_size;      /* 3006, 3007, 3009 */
  int roi_rect_x, roi_rect_y, roi_rect_w, roi_rect_h; /* 3011-3014 */
  int output_planes;               /* 7001 */
  int output_steps;                /* 7005 */
  int segment_min_area;            /* 5009 */
  double segment_min_intensity;    /* 5010 */
  int segment_close_size;          /* 5011 */
  int background_start;            /* 1003 (-1: unset) */
  int background_end;              /* 1004 (-1: unset) */
  int use_median_background;       /* 7006 */
} rihvr_file_params;

typedef struct rihvr_ctx rihvr_ctx;

/* HoloUi::HoloUi defaults (src/core/holo_ui.cpp:10-62) plus mode 7, FP32,
 * faithful arithmetic, 2 backtracks, reference step. */
int rihvr_params_default(rihvr_params* params);

/* HoloUi::readFile (src/core/holo_ui.cpp:171-486): "name code value" lines,
 * '%' or '#' comments.  `files` may be NULL. */
int rihvr_read_param_file(const char* path, rihvr_params* params, rihvr_file_params* files);

/* Plane positions as the reference computes them in float
 * (holo_ui.cpp:478-483): z_i = start_plane + i * plane_stepsize. */
int rihvr_plane_list(const rihvr_params* params, double* z_out);

/* SparseCompressiveHolo::SparseCompressiveHolo(Hologram)
 * (src/core/sparse_compressive_holo.cu:58-135).  width x height is the padded
 * hologram size.  Each side is even, 16..4096, with prime factors 2, 3, 5 and 7
 * only (the reference needs multiples of 16); square planes of side 32, 48, 64,
 * 128, 256, 384, 512, 640, 768, 1024 or 2304 take the fastest FFT passes. */
int rihvr_create(const rihvr_params* params, int width, int height, rihvr_ctx** out);

/* SparseCompressiveHolo::destroy (:137-146). */
void rihvr_destroy(rihvr_ctx* ctx);

/* Testing hook, no counterpart in the reference: once n more device or pinned
 * host allocations of rihvr_create have succeeded, the next one fails as if
 * memory were exhausted (RIHVR_ERR_OUT_OF_MEMORY), so that a test can walk
 * every cleanup path of rihvr_create without exhausting a GPU.  n < 0 (the
 * default) turns the injection off.  Process-wide; returns the previous
 * setting. */
int rihvr_debug_fail_allocations_after(int n);

/* The measured hologram b (the preprocessed, padded Hologram passed to the
 * constructor and to inverseReconstruct): real, height x width floats.  Also
 * resets the iterate to x = 0.  A hologram holding NaN or infinite samples is
 * refused with RIHVR_ERR_INVALID_DATA and the context is left unchanged (the
 * reference only prints a warning per bad sample, check_isnan_mdata,
 * sparse_compressive_holo.cu:9-35, and goes on to a solve full of NaNs). */
int rihvr_set_hologram(rihvr_ctx* ctx, const float* b, int is_device);

/* The driver's preprocessing (main_sparse_inverse.cu:106-124, as
 * rihvr_preprocess) on the GPU, straight into the context's hologram: the raw
 * width x height camera frame travels as stored, `bits` per sample (8:
 * uint8, 16: uint16, 32: floats holding 8/16-bit sample values), and so does
 * `background` (same type and size; used when files->remove_background).  The
 * crop comes from `files` (NULL: whole frame, no background) and the padding
 * from the context's zero_padding; cropped size + 2 * padding must equal the
 * context's width and height.  The result equals rihvr_preprocess's bit for
 * bit.  RIHVR_ERR_INVALID_DATA for a frame of zero mean or float samples that
 * are not integers in [0, 65535]; the context then keeps its state. */
int rihvr_set_hologram_frame(rihvr_ctx* ctx, const void* frame, int bits, int width, int height,
                             const void* background, const rihvr_file_params* files, int is_device);
/* The context's hologram b (height x width floats), as set. */
int rihvr_get_hologram(rihvr_ctx* ctx, float* out, int is_device);

/* Background generation (src/core/main_create_background.cu), on the GPU.
 * `frames`: count frames of width x height samples, `bits` as for
 * rihvr_set_hologram_frame, one after another, host or device memory
 * (is_device, which also applies to the outputs).  Backgrounds are floats on
 * the samples' scale (0-255 for 8-bit frames).
 * rihvr_background_mean: HoloSequence::useBackgroundSubtraction
 * (holo_sequence.cu:309-447): background = (sum of the frames in order, FP32)
 * * fl(1/count); stats (may be NULL) = alpha, beta, minimum, average as
 * background_stats.txt lists them: alpha = mean of the frames' means of
 * frame - background minus 5 times the mean of their standard deviations,
 * beta = 255 / (10 * mean standard deviation), minimum = 0, average = mean of
 * the background.  The caller picks the frames (the reference's selection is
 * in the create-background program). */
int rihvr_background_mean(const void* frames, int bits, int width, int height, int count, int is_device,
                          float* background, double* stats);
/* median_background_calc (main_create_background.cu:103-193): count >= 5
 * frames in, count - 2 backgrounds out (background_0000 .. of the frames'
 * numbering), each the per-pixel median of the five frames the reference's
 * five-frame stack holds at that point (rihvr_background_median5_frames
 * lists them, 5 per background). */
int rihvr_background_median5(const void* frames, int bits, int width, int height, int count, int is_device,
                             float* backgrounds);
int rihvr_background_median5_frames(int count, int* frame_indices);

/* SparseCompressiveHolo::inverseReconstruct(Hologram, mode) (:173-633): runs
 * num_inverse_iterations from x = 0.  final_objective (may be NULL) receives
 * the objective at the final momentum point. */
int rihvr_reconstruct(rihvr_ctx* ctx, double* final_objective);

/* Several frames at once: the replacement for the reference's frame loop,
 * which runs sparse-inverse-recon once per hologram
 * (src/QTGUI/rihvr.cpp:2414-2905, reconstructioncompute.cpp:117-142).  Frame i
 * does rihvr_set_hologram(ctxs[i], holograms[i], is_device) and
 * rihvr_reconstruct(ctxs[i], &final_objectives[i]).  Every context runs on its
 * own host thread and CUDA stream, so the frames' kernels and host decisions
 * overlap on the GPU (batch mode 0, the default).  In batch mode 1
 * (rihvr_set_batch_mode), frames that share a device and iteration count run
 * the iterations after the first as ONE graph launch per iteration for all
 * frames: each frame's iteration (its attempts, backtracking test and
 * momentum step, decided on the device) is a branch of the same graph.  In
 * batch mode 2, frames that share a device run all their iterations after the
 * first as ONE graph launch (up to 256 iterations a frame per launch): each
 * frame is a branch that loops on the device at its own pace, with its own
 * iteration count; the graph of the last mode-2 call is kept, and a call on
 * the same contexts (none re-tuned or destroyed since) launches it without
 * capturing again.  Either way the results are those of the sequential calls,
 * bit for bit.  The
 * contexts must be distinct and may differ in size and parameters.
 * final_objectives and statuses (n entries each) may be NULL; statuses[i]
 * receives frame i's status.  Returns the first nonzero status in frame order. */
int rihvr_reconstruct_batch(rihvr_ctx* const* ctxs, int n, const float* const* holograms, int is_device,
                            double* final_objectives, int* statuses);

/* Process-wide batch mode: 0 = one host thread and stream per frame
 * (default), 1 = one graph launch per iteration for all frames, 2 = one graph
 * launch for the whole solves of all frames.  Modes 1 and 2 pay a graph build
 * per call; mode 1 also keeps the frames in step at every iteration.  Returns
 * RIHVR_ERR_INVALID_ARGUMENT for other values. */
int rihvr_set_batch_mode(int mode);

/* 1 when the last rihvr_reconstruct_batch call on this host thread ran its
 * frames as one graph launch per iteration, 2 when it ran their whole solves
 * as one graph launch, else 0. */
int rihvr_batch_last_combined(void);

/* Launch-shape autotuner (no reference counterpart).  Times the candidate
 * shapes of the passes that have a free parameter on this context's own
 * buffers - the column passes' algorithms for evenly spaced planes
 * (transfer function by recurrence or Horner's scheme, or evaluated at every
 * plane) and their z-chunks, runs per plane of the
 * streaming TV prox and streaming versus tiled TV prox - and keeps the
 * fastest.  Results are cached per process for
 * the plane size, plane count, TV iterations, mode, storage and objective
 * recording, so later contexts of the same shape reuse them.  Safe between
 * iterations (only scratch buffers are written).  Tuned shapes may change the
 * order of the FP32 partial sums, hence the last bits of the sums; with
 * autotune off the shapes are fixed.  best_ms (may be NULL) receives the sum
 * of the chosen passes' times in milliseconds. */
int rihvr_autotune(rihvr_ctx* ctx, double* best_ms);

/* The launch shapes in use: z-chunks of the adjoint and forward column passes,
 * runs per plane of the streaming TV prox and the TV kernel (1 tiled,
 * 2 streaming in 2-warp blocks, 3 streaming in 4-warp blocks, 4 streaming in
 * one launch where 6-10 TV iterations would take two); 0 means the built-in
 * choice.  adj_recurrence receives the
 * adjoint column pass's variant for evenly spaced planes (square planes of side
 * 32 to 2304 except 640): 0 transfer function evaluated at every
 * plane, 1 advanced by a recurrence with the inter-stage twiddles regenerated
 * each plane, 2 the recurrence with the twiddles kept in registers (these two
 * up to side 1024, except 384 and 768), 3 the recurrence with the twiddles
 * read from a per-block shared table.  fwd_horner receives the forward column
 * pass's variant: 1 when it sums over evenly spaced planes by Horner's scheme
 * (square planes of side 32 to 512 and 1024) with its input strip
 * double-buffered, 2 for the same sum with the strip staged in the exchange
 * buffer and a shared twiddle table (also sides 384, 768 and 2304), 3 for
 * that form with the strip loaded by TMA, else 0.  Any pointer may be NULL. */
int rihvr_tuning(const rihvr_ctx* ctx, int* adj_chunks, int* fwd_chunks, int* tv_runs, int* tv_kernel,
                 int* adj_recurrence, int* fwd_horner);

/* Restart from x = 0 without changing the hologram. */
int rihvr_reset(rihvr_ctx* ctx);

/* Z-slab sharding of one hologram (no counterpart in the reference, whose
 * volume lives on one GPU).  A slab context holds planes
 * [z_first, z_first + z_count) of the params' plane list; params, sizes and
 * step rules are those of the whole volume (the first step is still
 * 1 / num_planes).  Modes 5 and 7 only: their prox is separable by plane,
 * which 3-D TV (mode 6) is not.  Give every slab the same hologram
 * (rihvr_set_hologram), then run rihvr_slab_iterate; each slab returns its
 * own planes (rihvr_get_volume, rihvr_get_plane with z counted from
 * z_first) and the whole solve's iteration log (rihvr_get_iterations).
 * Calls that need every plane (rihvr_iterate, rihvr_reconstruct and its batch
 * form, rihvr_objective, rihvr_set_initial_volume, rihvr_warm_start,
 * rihvr_initial_estimate, rihvr_lipschitz, rihvr_segment) return
 * RIHVR_ERR_INVALID_STATE on a slab that holds fewer than num_planes planes;
 * rihvr_forward on one returns its planes' contribution to the hologram. */
int rihvr_create_slab(const rihvr_params* params, int width, int height, int z_first, int z_count,
                      rihvr_ctx** out);

/* The planes a context holds (0 and num_planes for rihvr_create's). */
int rihvr_slab_range(const rihvr_ctx* ctx, int* z_first, int* z_count);

enum rihvr_dtype { RIHVR_DTYPE_F32 = 0, RIHVR_DTYPE_F64 = 1 };

/* Sum over the processes that hold the other slabs of the solve (one slab a
 * process, e.g. one process per GPU).  sum(user, data, count, dtype,
 * on_device) must replace the count values at data by their sum over all
 * processes, identical bit for bit in every process (an NCCL or MPI
 * all-reduce is), and return 0 when done; data is device memory of the
 * slab's device when on_device is 1, host memory when 0.  With host_staged
 * set, the partial spectrum is passed through pinned host memory too, for
 * process groups that reduce host buffers only. */
typedef struct rihvr_slab_reducer {
  int (*sum)(void* user, void* data, long long count, int dtype, int on_device);
  void* user;
  int host_staged;
} rihvr_slab_reducer;

/* `iterations` FISTA iterations (inverseReconstruct's loop, :299-611) of one
 * hologram whose planes are split over slab contexts.  Without a reducer the
 * n contexts (1..16, on one device or several with peer access, which is
 * enabled here) must tile the plane list in order; the partial spectra are
 * summed on every slab's device by peer reads, in slab order.  With a reducer,
 * n is 1 and the other slabs belong to other processes, which call this
 * function at the same time with the same iteration count.  Each attempt
 * exchanges one H x W complex FP32 plane (the partial spectrum) and 8 FP64
 * sums; the backtracking, restart and momentum decisions are made on the sums
 * and agree in every slab.  The objective and iterates equal those of one
 * context over all planes up to the order of the FP32 spectrum and FP64
 * sums; a single slab holding every plane reproduces rihvr_iterate bit for
 * bit. */
int rihvr_slab_iterate(rihvr_ctx* const* ctxs, int n, int iterations, const rihvr_slab_reducer* reducer);

/* Checkpoint and resume (no counterpart in the reference, whose voxel CSV,
 * SparseVolume::saveData at sparse_volume.cu:518-682, keeps intensities only
 * and cannot restart a solve).  rihvr_save_state writes, between iterations,
 * everything the next iteration reads: the hologram, the hologram-space
 * momentum buffers, the last two prox outputs in the storage type, the step,
 * momentum and restart scalars and the iteration log.  rihvr_load_state
 * restores them into a context created with the same sizes, plane range
 * (z-slabs), storage, mode and iteration parameters (else
 * RIHVR_ERR_INVALID_FILE, context unchanged);
 * further rihvr_iterate calls then continue the solve bit for bit as if it
 * had not stopped (with the same launch shapes: both contexts untuned, or
 * tuned alike).  The file takes about 2 x Nz x H x W x storage size bytes. */
int rihvr_save_state(rihvr_ctx* ctx, const char* path);
int rihvr_load_state(rihvr_ctx* ctx, const char* path);

/* Restart from a given volume instead of x = 0 (a warm start; the reference
 * always starts from 0, sparse_compressive_holo.cu:273): x0 is num_planes x
 * height x width complex interleaved (host or device), stored in the
 * context's storage type.  The momentum restarts (P_{k-1} = P_k = x0, beta =
 * 0), the estimated hologram, residual and step size are those of x0, and the
 * iteration log is cleared.  Typical sources: the previous frame of a time
 * series, or a network's estimate. */
int rihvr_set_initial_volume(rihvr_ctx* ctx, const float* x0, int is_device);

/* Continue the current solve by n iterations (the loop body :299-611). */
int rihvr_iterate(rihvr_ctx* ctx, int n);

/* Same, timed on the device with CUDA events around the n iterations. */
int rihvr_iterate_timed(rihvr_ctx* ctx, int n, float* device_ms);

/* Number of iterations run since the last reset. */
int rihvr_iteration_count(const rihvr_ctx* ctx);

/* calcObjectiveFunction (:2838-2899) at the current momentum point:
 * f and its three terms (0.5||r||^2, sum|x|, TV(x)). */
int rihvr_objective(rihvr_ctx* ctx, double* f, double* terms3);

/* Iteration log since the last reset. */
int rihvr_get_iterations(const rihvr_ctx* ctx, rihvr_iter_record* out, int max_records, int* n_out);

/* SparseCompressiveHolo::getPlane (:1197-1202): plane z of the current
 * momentum point x1, complex interleaved height x width. */
int rihvr_get_plane(rihvr_ctx* ctx, int z, float* out, int is_device);

/* The whole momentum point volume, complex interleaved Nz x height x width. */
int rihvr_get_volume(rihvr_ctx* ctx, float* out, int is_device);

/* The momentum point volume without a copy out: *dev_ptr receives a device
 * pointer to it (complex interleaved FP32, Nz x height x width, on the
 * context's device), *dtype 0 (FP32 complex).  The volume is materialised in
 * the context's intermediate buffer and the call synchronises the context's
 * stream, so the pointer may be read on any stream once it returns; it stays
 * valid until the next call on the context and must not be written or freed.
 * For GPU consumers of the volume (segmentation, export) in the caller's own
 * kernels.  (rihvr_get_volume_ptr of the replacement interface in the
 * reference's hot-path survey; the reference returns planes only,
 * getPlane, sparse_compressive_holo.h:92.) */
int rihvr_get_volume_ptr(rihvr_ctx* ctx, const void** dev_ptr, int* dtype);

/* Estimated hologram A x (estimate_final.tif, :621-622) and residual
 * A x - b (residual_final.tif, :623-624), height x width floats. */
int rihvr_get_estimate(rihvr_ctx* ctx, float* out, int is_device);
int rihvr_get_residual(rihvr_ctx* ctx, float* out, int is_device);

/* Fraction of non-zero voxels of the current momentum point
 * (SparseVolume::getSparsity, as printed per iteration at :561-565). */
int rihvr_sparsity(rihvr_ctx* ctx, double* fraction);

/* backPropagateInitial + calcInitialResidual (:2079-2133, :2725-2771): the
 * hologram estimated from t A^H b with t = 1/num_planes, written by the
 * reference as estimate_initial.tif.  Leaves the solve reset to x = 0. */
int rihvr_initial_estimate(rihvr_ctx* ctx, float* estimate_out, int is_device);

/* Lipschitz constant of the data term's gradient, L = largest eigenvalue of
 * A^H A, by an FP64 power iteration on the device: x_0 has seeded uniform
 * entries in [-1, 1) (splitmix64 of seed * 0x100000001B3 + 2 i and + 2 i + 1
 * for the real and imaginary parts of element i), each step forms A x_k and
 * A^H A x_k with the solver's own operators, the norms are reduced in FP64,
 * and *L_out receives the last Rayleigh quotient ||A x_k||^2 / ||x_k||^2
 * (history, if not NULL, all `iterations` of them; they rise towards L).
 * For this operator L = num_planes (reached by volumes constant over x, y and
 * z), which is why the reference fixes the step at 1 / num_planes.  The
 * reference's estimateLipschitz (sparse_compressive_holo.cu:2205-2464, called
 * at :226-246) is a one-step estimate from two random volumes whose result
 * the solve then discards (:247); as there, the value is reported and not
 * used.  Needs a hologram; leaves the solve reset to x = 0. */
int rihvr_lipschitz(rihvr_ctx* ctx, int iterations, unsigned long long seed, double* L_out, double* history);

/* Operator entry points. */
/* backPropagate (:1935-2077): d = Re(IFFT(sum_z H'_z FFT(x_z))), x complex
 * interleaved Nz x height x width, d height x width floats. */
int rihvr_forward(rihvr_ctx* ctx, const float* volume, float* holo_out, int is_device);
/* SparseGradient::reconstruct + getPlane for every plane
 * (src/core/sparse_gradient.cu:47-165): g_z = IFFT(conj(H'_z) FFT(r)). */
int rihvr_adjoint(rihvr_ctx* ctx, const float* residual, float* volume_out, int is_device);
/* One prox step, denoise() (:2969-2994): p = prox(x - t A^H r, t) for the
 * configured mode.  sums3 (may be NULL) receives the line-search terms
 * sum (p - x).g, sum |p - x|^2 and the restart statistic against y0 = x. */
int rihvr_prox_step(rihvr_ctx* ctx, const float* x, const float* residual, double t, float* p_out,
                    double* sums3, int is_device);

/* Image I/O and preprocessing of the hologram frame (the OpenCV parts of
 * Hologram on the reconstruction path).
 * rihvr_read_image: Hologram::read (hologram.cu:139-199) - 8/16-bit grayscale
 * or RGB TIFF (uncompressed, PackBits, LZW, horizontal predictor), 8/16-bit
 * grayscale or 8-bit RGB PNG, or binary PGM; values as stored.  Call with
 * pixels == NULL to get the size, then with a width*height buffer and the same
 * width/height. */
int rihvr_read_image(const char* path, float* pixels, int* width, int* height, int* bits);
/* cv::imwrite of an 8-bit grayscale image: baseline uncompressed TIFF. */
int rihvr_write_tiff8(const char* path, const unsigned char* pixels, int width, int height);
/* cv::imwrite of an 8-bit grayscale image as PNG (the backgrounds'
 * format, main_create_background.cu:154, 249). */
int rihvr_write_png8(const char* path, const unsigned char* pixels, int width, int height);
/* The preprocessing of main_sparse_inverse.cu:106-124: /255 (hologram.cu:
 * 401-439); I/mean - 1 (:332-358) or, when files->remove_background, (I - B) /
 * max(sqrt(B), 0.1) (:1365-1432); crop to files' ROI (:768-887); zero padding
 * (:889-945).  `files` may be NULL (whole frame, no background).  Size query
 * and call protocol as rihvr_read_image. */
int rihvr_preprocess(const float* holo, int width, int height, const float* background,
                     const rihvr_file_params* files, int zero_padding, float* out, int* out_width, int* out_height);
/* Message of the last failed image call on this thread. */
const char* rihvr_io_error(void);

/* Particle segmentation of a reconstructed volume: the reference's separate
 * segmentation program (src/core/main_segmentation.cu:37-138,
 * sparse_segmentation.cu, object_cloud.cu, blob3d.cu), run on the dense
 * volume without the voxel-file round trip. */
typedef struct rihvr_segment_params {
  double min_intensity; /* 5010 segment_min_intensity: voxels with q > min_intensity * max q / 256 are on */
  int close_size;       /* 5011 segment_close_size: radius of the closing ball (<= 0: none, at most 15) */
  int min_area;         /* 5009 segment_min_area: objects with fewer voxels are dropped */
  int faithful;         /* 1: the reference's in-plane neighbours (linear offsets, continuing on the
                           next row past a row's end, :493-511); 0: the geometric 26-neighbourhood */
} rihvr_segment_params;

/* One object, as ObjectCloud::writeCentroids reports it (object_cloud.cu:408-470). */
typedef struct rihvr_object {
  float x, y, z;          /* centroid (pixels, pixels, planes), Blob3d::getCentroid */
  float wx, wy, wz;       /* intensity-weighted centroid, Blob3d::getWeightedCentroid */
  int num_voxels;
  float max_value;        /* largest voxel intensity */
  float mean_value;       /* mean voxel intensity */
  int xmin, xmax, ymin, ymax, zmin, zmax; /* bounding box, Blob3d::getBounds */
} rihvr_object;

typedef struct rihvr_segment_info {
  double max_intensity;     /* largest q (SparseVolume::calcMaxIntensity, sparse_volume.cu:482-516) */
  double threshold;         /* min_intensity * max_intensity / 256 */
  long long closed_voxels;  /* voxels on after the closing */
  long long labelled_objects; /* components before the size filter */
  int strel_size;           /* voxels in the closing ball */
  long long kernel_launches;
} rihvr_segment_info;

/* HoloUi defaults (holo_ui.cpp:44-46): min_intensity 1, close_size 3,
 * min_area 2; faithful 1. */
int rihvr_segment_params_default(rihvr_segment_params* sp);
/* Segment the context's current volume.  Each voxel's value is
 * q = fl(fl(sqrt(I))^2) with I = fl(re^2 + im^2), what the reference computes
 * from the voxel after writing I to its voxel file and loading (sqrt(I), 0)
 * back (sparse_volume.cu:550, 645-650); the file's seven significant digits
 * are not applied.  Objects come in the reference's order (first appearance
 * by linear index, then the size filter's swaps).  At most max_objects are
 * written; *num_objects receives the count, and a count above max_objects
 * returns RIHVR_ERR_INVALID_ARGUMENT.  info may be NULL.  Device memory:
 * three bit-packed volumes and two 32-bit counts a 32-voxel word (about half a
 * byte a voxel) plus lists over the voxels that are on after the closing and
 * over the objects; the context keeps them for the next call and
 * rihvr_destroy frees them. */
int rihvr_segment(rihvr_ctx* ctx, const rihvr_segment_params* sp, rihvr_object* objects, int max_objects,
                  int* num_objects, rihvr_segment_info* info);
/* The same on a stack of voxel intensities I (num_planes x height x width
 * floats, the values a voxel file holds; zero where the file has no voxel),
 * on the device or the host.  Runs on the legacy default stream; its device
 * buffers are allocated and freed within the call. */
int rihvr_segment_intensity(const float* intensity, int width, int height, int num_planes, int is_device,
                            const rihvr_segment_params* sp, rihvr_object* objects, int max_objects,
                            int* num_objects, rihvr_segment_info* info);
/* ObjectCloud::writeCentroids (object_cloud.cu:408-470): centroids_XXXX.csv
 * (weighted 0, verbose 0), centroids_weighted_XXXX.csv (weighted 1) and
 * centroids_verbose_XXXX.csv (verbose 1). */
int rihvr_write_centroids(const char* filename, const rihvr_object* objects, int n, int weighted, int verbose);

/* Allocation-free adjoint.  No counterpart in the reference: for callers that
 * cannot allocate device memory - plugin hosts that hand out all device memory
 * from their own pool and forbid other allocations, real-time loops that
 * cannot take an allocation's latency and implicit synchronisation.  Computes what rihvr_adjoint
 * computes (g_z = IFFT(conj(H'_z) FFT(r)) for every plane) without a context:
 * `residual` (height x width floats) and `volume_out` (Nz x height x width
 * complex interleaved) are device memory owned by the caller; `stream` is a
 * cudaStream_t (NULL = legacy default stream); the call is asynchronous on it.
 * Scratch lives in one fixed 24 MiB + 32 KiB device array that every GPU
 * loading the library holds until exit: planes must be square with a supported
 * side of at most 1024 and num_planes at most 4096, otherwise
 * RIHVR_ERR_UNSUPPORTED_SIZE is returned.  Every call looks the array's device
 * address up in the current context; the first call on a device (or in a new
 * context) may also load the library's module there, so make that first call
 * before any stream capture.  Calls share the array and race if they overlap
 * on the GPU; serialise them. */
int rihvr_adjoint_noalloc(const rihvr_params* params, int width, int height, const float* residual,
                          float* volume_out, void* stream);

/* Learned warm start.  No counterpart in the reference: its reconstruction
 * always starts from x = 0 (sparse_compressive_holo.cu:273), which stays the
 * fallback and the reference.  A 3-D U-Net (3 levels, 16/32/64 channels, BF16
 * tensor-core convolutions with FP32 accumulation, FP32 master weights) maps
 * the back-propagated volume xbp = t A^H b (t the initial step) to an initial
 * iterate x0 = g * alpha * xbp, g a per-voxel gain in (0, 1).  Volumes are
 * depth x height x width complex interleaved device arrays; each side a
 * multiple of 4.  Calls run on the legacy default stream and return when done. */
typedef struct rihvr_unet rihvr_unet;
int rihvr_unet_create(int depth, int height, int width, unsigned long long seed, rihvr_unet** out);
void rihvr_unet_destroy(rihvr_unet* net);
long long rihvr_unet_param_count(const rihvr_unet* net);
/* all parameters as FP32 (convolution weights [cout][27][cin] and biases per
 * layer, then the head's 16 weights, its bias and alpha) */
int rihvr_unet_get_params(rihvr_unet* net, float* out);
int rihvr_unet_set_params(rihvr_unet* net, const float* in);
int rihvr_unet_predict(rihvr_unet* net, const float* xbp, float* x0);
/* loss sum |x0 - x*|^2 / sum |x*|^2 against a solution x* and its gradient
 * (host array of rihvr_unet_param_count floats; may be NULL) */
int rihvr_unet_gradients(rihvr_unet* net, const float* xbp, const float* xstar, float* grad_out, double* loss);
/* one Adam step (beta 0.9 / 0.999) on that loss */
int rihvr_unet_train_step(rihvr_unet* net, const float* xbp, const float* xstar, float lr, double* loss);
long long rihvr_unet_launch_count(const rihvr_unet* net);
/* Activation precision rihvr_unet_predict (and rihvr_warm_start) use at the
 * network's size: 16 when every level's width is a multiple of 128 (widths
 * that are multiples of 512) - BF16 activations between tcgen05
 * convolutions fed by TMA, the head fused into the last one - else 32 (FP32
 * activations, the training path).  RIHVR_UNET_MMA=sync forces 32. */
int rihvr_unet_activation_bits(rihvr_unet* net);
/* xbp = t A^H b of the context's hologram (t its initial step); leaves the
 * solve reset to x = 0. */
int rihvr_backpropagate(rihvr_ctx* ctx, float* xbp_out, int is_device);
/* Start the solve from the network's x0 for the context's hologram (as
 * rihvr_set_initial_volume does); the network's volume must be the context's
 * num_planes x height x width. */
int rihvr_warm_start(rihvr_ctx* ctx, rihvr_unet* net);

/* Device time per kernel class of the iterations run with profiling on
 * (names "adj_col", "adj_row", "prox", "fwd_row", "fwd_col", "plane").
 * Enabling records a pair of CUDA events around each launch. */
int rihvr_set_profiling(rihvr_ctx* ctx, int enable);
int rihvr_kernel_times(rihvr_ctx* ctx, const char** names, double* total_ms, int* launches, int max, int* n_out);

/* The context's CUDA stream (a cudaStream_t), for callers that order their own
 * work or timing events against it. */
void* rihvr_get_stream(rihvr_ctx* ctx);

/* Number of kernels the context has launched since it was created. */
long long rihvr_launch_count(const rihvr_ctx* ctx);

/* Bytes of device memory the context holds. */
size_t rihvr_device_bytes(const rihvr_ctx* ctx);

const char* rihvr_status_string(int status);
const char* rihvr_last_error(void);

#ifdef __cplusplus
}
#endif

#endif /* RIHVR_H */
