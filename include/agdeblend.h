/*
 * AGDeblend C API, served by the B200 implementation.
 *
 * Drop-in declarations for the two functions of the reference's public
 * header (include/agdeblend.h:22-44 of the reference).  Argument order,
 * types, enum values and the AGD_TYPE switch are unchanged so that existing
 * callers (the cffi Python wrapper, Julia ccall, the Fortran C shim, C/C++
 * programs) link against libagdeblend.so / libagdeblend_double.so without
 * edits.  The MPI variants (AGD_MPI) are not provided: this library runs one
 * problem on one GPU.
 */
#ifndef AGD_H
#define AGD_H

#ifdef __cplusplus
extern "C" {
#endif

/* Trace categories (reference include/agdeblend.h:8) */
enum AGDTraceType { AGDLive, AGDBad, AGDMissing };
/* Blend modes for agd_blend (reference include/agdeblend.h:9) */
enum AGDBlendMode { AGDBlendSum, AGDBlendMean, AGDBlendOverwrite };

#ifdef AGD_DOUBLE
#define AGD_TYPE double
#else
#define AGD_TYPE float
#endif

/* Tunables with the reference's values (reference include/agdeblend.h:17-20) */
#define AGD_PAD_FRACTION ((AGD_TYPE)0.25)
#define AGD_TARGET_LAMB ((AGD_TYPE)0.001) /* 1e-3 */
#define AGD_MAX_N_COORDS 4

/*
 * Deblend `data` in place by ISTA with a decaying threshold, n_its
 * iterations.  Replaces agd_deblend (reference include/agdeblend.h:22-32;
 * src/agdeblend.c:511-649).  Returns 0 on success, 1 on failure with a
 * message on stderr.  The iteration runs on the current CUDA device.
 */
int agd_deblend(int n_patches, int const *volumes, int const *n_dims,
                int const *const *window_shapes, int const *const *coords,
                int const *const *shapes, long int const *const *shottimes,
                int const *const *channels,
                enum AGDTraceType const *const *trace_types,
                int const *wavelet_lengths, int const *const *wavelet_idxs,
                AGD_TYPE const *const *wavelets, AGD_TYPE const initial_factor,
                int n_its, int print_freq, AGD_TYPE *const *data);

/*
 * Blend traces into continuous records (sum, mean or overwrite), mute bad
 * traces, and extract output traces.  Replaces agd_blend (reference
 * include/agdeblend.h:33-44; src/agdeblend.c:800-938).
 */
int agd_blend(int n_patches, int const *n_traces, int const *n_times,
              long int const *const *shottimes, int const *const *channels,
              enum AGDTraceType const *const *trace_types,
              AGD_TYPE *const *data, enum AGDBlendMode blend_mode,
              int taper_length, int n_patches_out, int const *n_traces_out,
              int const *n_times_out, long int const *const *shottimes_out,
              int const *const *channels_out,
              enum AGDTraceType const *const *trace_types_out,
              AGD_TYPE *const *data_out);

#ifdef __cplusplus
}
#endif

#endif
