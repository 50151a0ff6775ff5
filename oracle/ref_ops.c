/*
 * Test infrastructure only.  Operator-level access to the reference's own,
 * unchanged sources: this file #includes the reference's src/agdeblend.c (the
 * reference's tests do the same, src/test.cpp:24-28) so that its static
 * planning and operator functions can be called on chosen inputs.  It is
 * compiled only by oracle/Makefile into oracle/_ref/ and only when the
 * reference tree is present; nothing in the product links it.
 *
 * Layouts exchanged with callers:
 *   model:   windows in the reference's window order, each window
 *            [n_time_windows][padded space dims...][padded_time/2+1] complex
 *            (interleaved re, im) exactly as allocate_model_fk lays it out
 *            (src/model.c:1160-1185).
 *   blended: every (channel, interval) segment of the blend config
 *            concatenated in channel-major, interval-minor order
 *            (src/blend.c:796-829).
 */
#include "agdeblend.c"

struct RefOps {
  struct Model model;
  AGD_FFTW_COMPLEX **model_fk;
  AGD_TYPE ***blended;
  AGD_TYPE stepsize;
  int n_patches;
  int const *volumes;
  int const *n_dims;
  int const *const *shapes;
  long int const *const *shottimes;
  int const *const *channels;
  enum AGDTraceType const *const *trace_types;
};

static size_t window_model_size(struct Model const *const m, int const w) {
  struct FKWindowConfig const *const c =
      m->fk_configs.window_configs + m->windows[w].fk_config_idx;
  return (size_t)c->n_time_windows * (size_t)c->n_elements_padded_window_fk;
}

void refops_destroy(struct RefOps *const h) {
  if (h == NULL) return;
  free_blended(&(h->model.blend_config), &(h->blended));
  free_model_fk(h->model.n_windows, &(h->model_fk));
  free_model(&(h->model));
  free(h);
}

struct RefOps *refops_create(
    int n_patches, int const *volumes, int const *n_dims,
    int const *const *window_shapes, int const *const *coords,
    int const *const *shapes, long int const *const *shottimes,
    int const *const *channels, enum AGDTraceType const *const *trace_types,
    int const *wavelet_lengths, int const *const *wavelet_idxs,
    AGD_TYPE const *const *wavelets) {
  struct RefOps *h = (struct RefOps *)calloc(1, sizeof(struct RefOps));
  if (h == NULL) return NULL;
  h->n_patches = n_patches;
  h->volumes = volumes;
  h->n_dims = n_dims;
  h->shapes = shapes;
  h->shottimes = shottimes;
  h->channels = channels;
  h->trace_types = trace_types;
  if (set_model(n_patches, volumes, n_dims, window_shapes, coords, shapes,
                shottimes, channels, trace_types, wavelet_lengths,
                wavelet_idxs, wavelets, &(h->model)))
    goto err;
  if (allocate_model_fk(&(h->model), &(h->model_fk))) goto err;
  if (allocate_blended(&(h->model.blend_config), &(h->blended))) goto err;
  h->stepsize = get_stepsize(&(h->model), h->blended);
  return h;
err:
  refops_destroy(h);
  return NULL;
}

int refops_n_windows(struct RefOps const *const h) { return h->model.n_windows; }

double refops_stepsize(struct RefOps const *const h) { return (double)h->stepsize; }

long refops_model_size(struct RefOps const *const h) {
  long total = 0;
  int w;
  for (w = 0; w < h->model.n_windows; w++)
    total += (long)window_model_size(&(h->model), w);
  return total;
}

/* Per-window description: out must hold 64 ints.
 * [0] n_dims (space + time), [1] n_time_windows, [2] patch_idx,
 * [3] n_traces, [4] n_times (data portion), [5] n_times_output_capacity,
 * [8 + d] window_shape[d], [16 + d] padded_window_shape[d],
 * [24 + 2d], [25 + 2d] use_taper, [40 + d] window coords (space dims). */
void refops_window_info(struct RefOps const *const h, int const w,
                        int *const out) {
  struct ModelWindow const *const win = h->model.windows + w;
  struct FKWindowConfig const *const c =
      h->model.fk_configs.window_configs + win->fk_config_idx;
  int d;
  memset(out, 0, 64 * sizeof(int));
  out[0] = c->n_dims;
  out[1] = c->n_time_windows;
  out[2] = win->space_window.patch_idx;
  out[3] = c->n_traces;
  out[4] = c->n_times;
  out[5] = c->n_times_output_capacity;
  for (d = 0; d < c->n_dims; d++) {
    out[8 + d] = c->window_shape[d];
    out[16 + d] = c->padded_window_shape[d];
    out[24 + 2 * d] = c->use_taper[2 * d];
    out[25 + 2 * d] = c->use_taper[2 * d + 1];
  }
  for (d = 0; d < c->n_dims - 1; d++) out[40 + d] = win->space_window.coords[d];
}

/* Segment lengths of the blended record; returns the number of segments. */
int refops_blended_layout(struct RefOps const *const h, long *const lengths) {
  struct BlendConfig const *const b = &(h->model.blend_config);
  int n = 0;
  int ch;
  for (ch = 0; ch < b->n_channels; ch++) {
    int iv;
    for (iv = 0; iv < b->channels_intervals[ch].n_intervals; iv++) {
      struct Interval const *const it = b->channels_intervals[ch].intervals + iv;
      if (lengths != NULL) lengths[n] = it->stop - it->start;
      n++;
    }
  }
  return n;
}

static void flatten_blended(struct RefOps const *const h,
                            AGD_TYPE *const flat) {
  struct BlendConfig const *const b = &(h->model.blend_config);
  size_t off = 0;
  int ch;
  for (ch = 0; ch < b->n_channels; ch++) {
    int iv;
    for (iv = 0; iv < b->channels_intervals[ch].n_intervals; iv++) {
      struct Interval const *const it = b->channels_intervals[ch].intervals + iv;
      size_t const n = (size_t)(it->stop - it->start);
      memcpy(flat + off, h->blended[ch][iv], n * sizeof(AGD_TYPE));
      off += n;
    }
  }
}

static void unflatten_blended(struct RefOps const *const h,
                              AGD_TYPE const *const flat) {
  struct BlendConfig const *const b = &(h->model.blend_config);
  size_t off = 0;
  int ch;
  for (ch = 0; ch < b->n_channels; ch++) {
    int iv;
    for (iv = 0; iv < b->channels_intervals[ch].n_intervals; iv++) {
      struct Interval const *const it = b->channels_intervals[ch].intervals + iv;
      size_t const n = (size_t)(it->stop - it->start);
      memcpy(h->blended[ch][iv], flat + off, n * sizeof(AGD_TYPE));
      off += n;
    }
  }
}

static void load_model(struct RefOps const *const h, AGD_TYPE const *const in) {
  size_t off = 0;
  int w;
  for (w = 0; w < h->model.n_windows; w++) {
    size_t const n = window_model_size(&(h->model), w);
    memcpy(h->model_fk[w], in + 2 * off, 2 * n * sizeof(AGD_TYPE));
    off += n;
  }
}

static void store_model(struct RefOps const *const h, AGD_TYPE *const out) {
  size_t off = 0;
  int w;
  for (w = 0; w < h->model.n_windows; w++) {
    size_t const n = window_model_size(&(h->model), w);
    memcpy(out + 2 * off, h->model_fk[w], 2 * n * sizeof(AGD_TYPE));
    off += n;
  }
}

/* blended_out = mute(B W F x)   (model_forward, src/model.c:1067-1114) */
void refops_forward(struct RefOps *const h, AGD_TYPE const *const model_in,
                    AGD_TYPE *const blended_out) {
  load_model(h, model_in);
  model_forward((AGD_FFTW_COMPLEX const *const *)h->model_fk, &(h->model),
                h->blended);
  flatten_blended(h, blended_out);
}

/* model_out = F^H W^H B^H blended_in   (model_adjoint_update with stepsize -1
 * applied to a zero model, src/model.c:1116-1157) */
void refops_adjoint(struct RefOps *const h, AGD_TYPE const *const blended_in,
                    AGD_TYPE *const model_out) {
  int w;
  for (w = 0; w < h->model.n_windows; w++)
    memset(h->model_fk[w], 0,
           window_model_size(&(h->model), w) * sizeof(AGD_FFTW_COMPLEX));
  unflatten_blended(h, blended_in);
  model_adjoint_update((AGD_TYPE const *const *const *)h->blended, &(h->model),
                       -AGD_ONE, h->model_fk);
  store_model(h, model_out);
}

/* x <- x - stepsize * A^H r, with the model given and returned */
void refops_adjoint_update(struct RefOps *const h,
                           AGD_TYPE const *const blended_in,
                           AGD_TYPE const stepsize, AGD_TYPE *const model_io) {
  load_model(h, model_io);
  unflatten_blended(h, blended_in);
  model_adjoint_update((AGD_TYPE const *const *const *)h->blended, &(h->model),
                       stepsize, h->model_fk);
  store_model(h, model_io);
}

/* d = mute(mean-blend(data)) as used for the recorded data
 * (blend_input, src/blend.c:1294-1335) */
int refops_blend_input(struct RefOps *const h, int const *const *const shapes,
                       AGD_TYPE const *const *const data,
                       AGD_TYPE *const blended_out) {
  AGD_TYPE ***blended = NULL;
  struct BlendConfig const *const b = &(h->model.blend_config);
  size_t off = 0;
  int ch;
  if (blend_input(data, h->n_patches, h->volumes, h->n_dims, shapes,
                  h->shottimes, h->channels, h->trace_types,
                  &(h->model.blend_config), &blended))
    return 1;
  for (ch = 0; ch < b->n_channels; ch++) {
    int iv;
    for (iv = 0; iv < b->channels_intervals[ch].n_intervals; iv++) {
      struct Interval const *const it = b->channels_intervals[ch].intervals + iv;
      size_t const n = (size_t)(it->stop - it->start);
      memcpy(blended_out + off, blended[ch][iv], n * sizeof(AGD_TYPE));
      off += n;
    }
  }
  free_blended(&(h->model.blend_config), &blended);
  return 0;
}

/* data = window sum of W F x  (set_output, src/model.c:1425-1515) */
void refops_set_output(struct RefOps *const h, AGD_TYPE const *const model_in,
                       AGD_TYPE *const *const data) {
  load_model(h, model_in);
  set_output((AGD_FFTW_COMPLEX const *const *)h->model_fk, h->n_patches,
             h->volumes, h->n_dims, h->shapes, &(h->model), data);
}

/* lambda_0 = sqrt(max |x|^2)  (get_initial_lamb, src/model.c:1202-1227) */
double refops_initial_lamb(struct RefOps *const h,
                           AGD_TYPE const *const model_in) {
  load_model(h, model_in);
  return (double)get_initial_lamb(&(h->model),
                                  (AGD_FFTW_COMPLEX const *const *)h->model_fk);
}

/* complex soft threshold (shrink_threshold, src/model.c:1392-1423) */
void refops_threshold(struct RefOps *const h, AGD_TYPE *const model_io,
                      AGD_TYPE const lamb) {
  load_model(h, model_io);
  shrink_threshold(&(h->model), lamb, h->model_fk);
  store_model(h, model_io);
}

/* residual norm (get_residual_norm, src/model.c:1343-1384) */
double refops_residual_norm(struct RefOps *const h,
                            AGD_TYPE const *const blended_in) {
  unflatten_blended(h, blended_in);
  return (double)get_residual_norm(&(h->model.blend_config),
                                   (AGD_TYPE const *const *const *)h->blended);
}

int refops_type_size(void) { return (int)sizeof(AGD_TYPE); }
