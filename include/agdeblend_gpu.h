/*
 * Extension API of the B200 implementation (not in the reference).
 *
 * The reference keeps all state inside one agd_deblend call.  These entry
 * points expose the same planning and operators on a persistent problem
 * handle so that callers (tests, benchmarks, batch drivers) can apply the
 * operator A = mute . blend . wavelet . FK and its adjoint, or run the solver,
 * without re-planning.  Every function returns 0 on success and 1 on failure
 * with a message on stderr, like the reference.
 *
 * Layouts at this boundary are the reference's:
 *   model   every window's [n_time_windows][padded space...][padded_time/2+1]
 *           complex (interleaved re, im), windows in the reference's order
 *           (allocate_model_fk, reference src/model.c:1160-1185);
 *   record  every (channel, interval) segment of the blend configuration,
 *           channel-major (allocate_blended, reference src/blend.c:796-829).
 */
#ifndef AGD_GPU_H
#define AGD_GPU_H

#include "agdeblend.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct agd_gpu_problem agd_gpu_problem;

/* Validates and plans a problem (the arguments of agd_deblend up to the
 * wavelets) and uploads its tables to the current device.  Replaces the
 * set-up half of agd_deblend: check_deblend_inputs + set_model +
 * get_stepsize (reference src/agdeblend.c:548-576). */
int agd_gpu_problem_create(int n_patches, int const *volumes, int const *n_dims,
                           int const *const *window_shapes, int const *const *coords,
                           int const *const *shapes, long int const *const *shottimes,
                           int const *const *channels,
                           enum AGDTraceType const *const *trace_types,
                           int const *wavelet_lengths, int const *const *wavelet_idxs,
                           AGD_TYPE const *const *wavelets, agd_gpu_problem **problem);

void agd_gpu_problem_destroy(agd_gpu_problem *problem);

/* info (23 values): [0] windows, [1] model complex elements, [2] record
 * samples, [3] window traces (all windows), [4] record segments, [5] mute
 * spans, [6] device bytes held, [7] blend contributions per forward,
 * [8] 1 if the shape-specialised kernels serve every window, 2 if they
 * serve some, 0 if none, [9] 1 if the prime-factor wavelet kernel serves
 * the problem, [10] and [11] the space-kernel candidates picked by the
 * set-up timing for the forward and adjoint of the first window class (-1
 * without shape-specialised kernels), [12] and [13] that class's number of
 * candidates, [14] kernels launched per iteration, [15] window classes on
 * the shape-specialised kernels, [16] windows on them, [17] and [18] the
 * time-kernel candidates picked for the first time group (-1 without
 * one), [19] its number of candidates, [20] the wavelet-kernel candidate
 * picked (-1 without the prime-factor kernel), [21] their number, [22]
 * windows with one space axis on the line-DFT kernels (lengths without a
 * shape-specialised kernel, up to 128). */
int agd_gpu_problem_info(agd_gpu_problem const *problem, long int *info);

/* Kernel families serving the first window class and time group, as a
 * profiler lists them: "space_fwd=... space_adj=... time_fwd=... time_adj=...
 * wavelet=..." (no reference counterpart: it names this library's
 * kernels).  Returns 1 if buf (len bytes) is too short. */
int agd_gpu_problem_kernels(agd_gpu_problem const *problem, char *buf, int len);

/* Step size 0.5 / max blend fold (reference get_stepsize, src/model.c:1230-1312). */
int agd_gpu_stepsize(agd_gpu_problem *problem, AGD_TYPE *stepsize);

/* record = A model (reference model_forward, src/model.c:1067-1114). */
int agd_gpu_forward(agd_gpu_problem *problem, AGD_TYPE const *model, AGD_TYPE *record);

/* model = A^H record (reference model_adjoint_update with step -1 on a zero
 * model, src/model.c:1116-1157). */
int agd_gpu_adjoint(agd_gpu_problem *problem, AGD_TYPE const *record, AGD_TYPE *model);

/* record = mute(mean-blend(data)) (reference blend_input, src/blend.c:1294-1335). */
int agd_gpu_blend_input(agd_gpu_problem *problem, AGD_TYPE const *const *data,
                        AGD_TYPE *record);

/* data = sum over windows of W F model (reference set_output,
 * src/model.c:1425-1515). */
int agd_gpu_set_output(agd_gpu_problem *problem, AGD_TYPE const *model,
                       AGD_TYPE *const *data);

/* The solver of agd_deblend on a planned problem: data is the blended input
 * and receives the deblended output (reference src/agdeblend.c:578-633). */
int agd_gpu_solve(agd_gpu_problem *problem, AGD_TYPE initial_factor, int n_its,
                  int print_freq, AGD_TYPE *const *data);

/* Checkpoint / resume (no counterpart in the reference, which keeps the
 * solver state inside agd_deblend): runs iterations [it_begin, it_end) of
 * the n_its-iteration schedule of agd_gpu_solve.  it_begin = 0 starts from
 * the initial step; it_begin > 0 starts from model_in, the model after
 * iteration it_begin - 1 (layout as agd_gpu_forward).  model_out (may be
 * NULL) receives the model after iteration it_end - 1, and `data` the
 * output of that model.  The thresholds are recomputed from the data, so
 * stopping after iteration k and resuming from model_out with it_begin = k
 * + 1 gives agd_gpu_solve's result. */
int agd_gpu_solve_range(agd_gpu_problem *problem, AGD_TYPE initial_factor, int n_its,
                        int it_begin, int it_end, int print_freq, AGD_TYPE const *model_in,
                        AGD_TYPE *model_out, AGD_TYPE *const *data);

/* Benchmark hook: loads `data`, runs the set-up step, then `warmup` untimed
 * and `steps` timed ISTA iterations with every input resident on the device,
 * each iteration a replay of one captured CUDA graph (as agd_gpu_solve runs
 * them).  Timing uses CUDA events on the library's stream.  timing[0] = total ms of
 * the timed iterations, timing[1] = ms of the forward half, timing[2] = ms of
 * the adjoint half (separately timed pass), timing[3] = iterations timed. */
int agd_gpu_time_iterations(agd_gpu_problem *problem, AGD_TYPE const *const *data,
                            AGD_TYPE initial_factor, int n_its, int warmup, int steps,
                            double *timing);

/* Benchmark hook: one ISTA iteration on the current device state with CUDA
 * events between its launch groups (call after agd_gpu_time_iterations).
 * ms[0] forward space passes (all windows), [1] time c2r + overlap-add,
 * [2] wavelet forward, [3] blend gather + residual, [4] adjoint time axis
 * (with its record gather and wavelet), [5] adjoint space passes with the
 * update; [6] = [0], [10] = [5], [14] = 1 (ms has 16 entries). */
int agd_gpu_profile_iteration(agd_gpu_problem *problem, AGD_TYPE lamb, double *ms);

/* Host planning only (no device use): writes the plan's size summary
 * (info layout as agd_gpu_problem_info, [6] and [7] zero) and, when the
 * arrays are non-NULL, per window `win` (32 ints each: patch, D, T, F, Lt,
 * Pt, h, n_fk, C, n_traces, L[4], P[4], use_taper[10]), per window trace
 * `blend` (3 longs each: record start or -1, trace start, samples). */
int agd_plan_export(int n_patches, int const *volumes, int const *n_dims,
                    int const *const *window_shapes, int const *const *coords,
                    int const *const *shapes, long int const *const *shottimes,
                    int const *const *channels, enum AGDTraceType const *const *trace_types,
                    int const *wavelet_lengths, int const *const *wavelet_idxs,
                    AGD_TYPE const *const *wavelets, long int *info, int *win,
                    long int *blend);

/* Independent problems solved together (no counterpart in the reference,
 * whose agd_deblend solves one problem per call).  Each argument is an
 * array over the n_problems problems of the corresponding agd_deblend
 * argument (n_patches[q] patches for problem q; the three wavelet arrays may
 * be NULL, or hold NULL for problems without wavelets).  initial_factor and
 * n_its are shared.  Every problem keeps its own step size, initial
 * threshold and threshold schedule, so data[q] ends as agd_deblend would
 * leave it for problem q alone; all problems run in the same kernel
 * launches, one captured CUDA graph per iteration.  No residual printing. */
int agd_deblend_batch(int n_problems, int const *n_patches, int const *const *volumes,
                      int const *const *n_dims, int const *const *const *window_shapes,
                      int const *const *const *coords, int const *const *const *shapes,
                      long int const *const *const *shottimes, int const *const *const *channels,
                      enum AGDTraceType const *const *const *trace_types,
                      int const *const *wavelet_lengths, int const *const *const *wavelet_idxs,
                      AGD_TYPE const *const *const *wavelets, AGD_TYPE initial_factor,
                      int n_its, AGD_TYPE *const *const *data);

/* The persistent handle of a batch (arguments as agd_deblend_batch up to
 * the wavelets).  The handle's patches are all problems' patches in
 * problem order: agd_gpu_solve, agd_gpu_blend_input, agd_gpu_set_output and
 * agd_gpu_time_iterations take data for all of them; the model and record
 * of agd_gpu_forward / agd_gpu_adjoint are the problems' models and records
 * one after another. */
int agd_gpu_batch_create(int n_problems, int const *n_patches, int const *const *volumes,
                         int const *const *n_dims, int const *const *const *window_shapes,
                         int const *const *const *coords, int const *const *const *shapes,
                         long int const *const *const *shottimes,
                         int const *const *const *channels,
                         enum AGDTraceType const *const *const *trace_types,
                         int const *const *wavelet_lengths, int const *const *const *wavelet_idxs,
                         AGD_TYPE const *const *const *wavelets, agd_gpu_problem **problem);

/* Step size of every problem of the handle (one value for a single
 * problem). */
int agd_gpu_problem_steps(agd_gpu_problem const *problem, AGD_TYPE *steps);

/* The library keeps the large device arrays of finished problems (at most
 * half the device memory) for the next problem on the same device, since a
 * fresh allocation of gigabytes costs more than a solve; this returns them
 * to the device.  AGD_GPU_CACHE=0 in the environment disables the cache. */
void agd_gpu_release_cache(void);

/* agd_blend for callers that cannot allocate device memory (hosts whose own
 * pool owns all device memory, real-time callers that must not wait on or
 * fail in the allocator).  No counterpart in the reference: it is an
 * addition of this library.  Same arguments and results as agd_blend, except
 * that the data are device pointers - data_dev holds all input patches one
 * after another ([n_traces][n_times] each), data_out_dev receives all output
 * patches the same way - and `stream` (a cudaStream_t, NULL for the default
 * stream) orders the work.  It allocates nothing: every intermediate lives
 * in a fixed 16 MiB device array built into the library; larger problems are
 * rejected with an error (use agd_blend).  The first call on a device looks
 * up that array's device address and keeps it for the life of the process,
 * so make it before any stream capture, and do not reset the device between
 * calls.  Calls overlapping on one device race on the shared array.  Each
 * call copies its tables from temporary host memory and waits on `stream`
 * until its own work has finished before it returns (it blocks). */
int agd_blend_device_noalloc(int n_patches, int const *n_traces, int const *n_times,
                             long int const *const *shottimes, int const *const *channels,
                             enum AGDTraceType const *const *trace_types,
                             AGD_TYPE const *data_dev, enum AGDBlendMode blend_mode,
                             int taper_length, int n_patches_out, int const *n_traces_out,
                             int const *n_times_out, long int const *const *shottimes_out,
                             int const *const *channels_out,
                             enum AGDTraceType const *const *trace_types_out,
                             AGD_TYPE *data_out_dev, void *stream);

/* Precision of the space axes of the FK operator (no counterpart in the
 * reference, whose FFTs are FFTW's in AGD_TYPE; src/fk.c:307-452).
 * 0 (default): FP32 FFT kernels.  1: split-BF16 tensor-core contractions -
 * the space DFT of every window whose three space axes have padded length 20
 * and window length 16 (windows (16, 16, 16, nt)) runs as hi + lo BF16
 * products with FP32 accumulation on the tcgen05 tensor cores (about 16
 * significant bits per operand); the time axis, the wavelet, the blend and
 * the ISTA update stay FP32.  Mode 1 needs the float library.  tc_windows
 * (may be NULL) receives the number of windows the tensor-core kernels
 * serve.  Applies to later operator, solver and timing calls on the
 * handle. */
int agd_gpu_problem_set_precision(agd_gpu_problem *problem, int precision,
                                  long int *tc_windows);

/* ---------------------------------------------------------------------------
 * Learned warm start (no counterpart in the reference, whose solver starts
 * every solve from a zero model, src/model.c:1160-1185).
 * ------------------------------------------------------------------------- */

/* C = alpha A B^T + beta C on the tcgen05 tensor cores: A (M x K) and B
 * (N x K) row-major BF16 device arrays (16-byte aligned, K, lda, ldb
 * multiples of 8), C row-major FP32, FP32 accumulation.  `stream` is a
 * cudaStream_t (NULL: default stream); returns after the product is done. */
int agd_nn_gemm_bf16(const void *A, const void *B, float *C, int M, int N, int K, int lda,
                     int ldb, int ldc, float alpha, float beta, void *stream);

/* The network's 3 x 3 convolution (padding 1, no bias) on the tensor cores:
 * y[n][h][w][cout] (FP32) = sum over (ky, kx, ci) of
 * x[n][h + ky - 1][w + kx - 1][ci] * weights[cout][ky][kx][ci], x and weights
 * BF16 device arrays (NHWC, cin a multiple of 8, 16-byte aligned), FP32
 * accumulation.  Layers with cin a multiple of 32 and w a multiple of 128
 * whose weights fit shared memory in at most two groups of output channels
 * run on the halo-tile kernel, the others on the implicit GEMM.  Returns
 * after it is done. */
int agd_nn_conv3x3_bf16(const void *x, int n, int h, int w, int cin, const void *weights,
                        int cout, float *y, void *stream);

/* Warm start (no counterpart in the reference, whose solver starts from a
 * zero model, src/model.c:1160-1185, and whose threshold schedule starts at
 * the largest coefficient of the first adjoint, src/agdeblend.c:526-589).
 * `estimate` is an estimate of the deblended data (patch layout as `data`).
 * agd_gpu_warm_model writes the model x0 whose FK (and wavelet) operator
 * reproduces the estimate on the live traces' samples (layout as
 * agd_gpu_forward).  agd_gpu_solve_warm runs agd_gpu_solve's initial step
 * and threshold schedule from the blended input `data`, replaces the model
 * by the warm model of `estimate`, and runs iterations [it_begin, n_its) of
 * that schedule (1 <= it_begin <= n_its): the thresholds start at the
 * schedule's level for iteration it_begin instead of the largest
 * coefficient.  `data` receives the deblended output. */
int agd_gpu_warm_model(agd_gpu_problem *problem, AGD_TYPE const *const *estimate,
                       AGD_TYPE *model);
int agd_gpu_solve_warm(agd_gpu_problem *problem, AGD_TYPE initial_factor, int n_its,
                       int it_begin, int print_freq, AGD_TYPE const *const *estimate,
                       AGD_TYPE *const *data);

typedef struct agd_nn agd_nn;

/* agd_gpu_solve_warm with the network's estimate: `data` (blended input,
 * receives the output) is cut on the device into 2-D images - every line of
 * a patch along a source axis (a space axis along which the shot times
 * change: receiver gathers) x the time samples - each normalised by its
 * RMS, run through `net` and scaled back; the estimate is the mean of the
 * estimates from the lines along every source axis.  A network with 3
 * input channels instead gets the lines along the slowest source axis (the
 * largest shot-time step), each with its two neighbouring lines along the
 * next faster source axis as channels 1 and 2 (clamped at the patch edge;
 * the line itself where the patch has one source axis).  Float library
 * only. */
int agd_gpu_solve_learned(agd_gpu_problem *problem, agd_nn *net, AGD_TYPE initial_factor,
                          int n_its, int it_begin, int print_freq, AGD_TYPE *const *data);

/* The warm-start network: a 4-level 2-D convolutional encoder-decoder on
 * images of n x h x w samples (traces x time; h, w multiples of 8), base
 * channels c (32: 1,162,945 parameters with one input channel), output =
 * input channel 0 + a learned correction.  Convolutions run as BF16
 * tensor-core GEMMs with FP32 accumulation, forward and backward; FP32
 * master parameters, Adam.  Arrays are host memory, row-major float: inputs
 * [n][h][w][in_channels], outputs and targets [n][h][w].  Parameter layout:
 * per layer (encoder, bottleneck, decoder order) the weights
 * [cout][3][3][cin] then the biases [cout].  agd_nn_create: one input
 * channel; agd_nn_create_channels: 1 to 8. */
int agd_nn_create(int base_channels, unsigned seed, agd_nn **net);
int agd_nn_create_channels(int base_channels, int in_channels, unsigned seed, agd_nn **net);
int agd_nn_input_channels(const agd_nn *net);
void agd_nn_destroy(agd_nn *net);
long agd_nn_param_count(const agd_nn *net);
int agd_nn_get_params(const agd_nn *net, float *params);
int agd_nn_set_params(agd_nn *net, const float *params);
/* output = network(input) */
int agd_nn_forward(agd_nn *net, const float *input, int n, int h, int w, float *output);
/* mean squared error of network(input) against target, and its gradient
 * with respect to the parameters (grad may be NULL) */
int agd_nn_loss_grad(agd_nn *net, const float *input, const float *target, int n, int h, int w,
                     double *loss, float *grad);
/* Adam (learning rate lr) over shuffled batches of the n_samples pairs
 * (inputs, targets), `epochs` passes; epoch_loss (may be NULL) receives the
 * mean loss of each pass. */
int agd_nn_train(agd_nn *net, const float *inputs, const float *targets, long n_samples, int h,
                 int w, int batch, int epochs, float lr, unsigned seed, double *epoch_loss);

#ifdef __cplusplus
}
#endif

#endif
