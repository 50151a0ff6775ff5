/*
 * Test infrastructure only (the oracle's FFT).  Implements the subset of the
 * FFTW3 API declared in fftw3.h from the definition of the discrete Fourier
 * transform:
 *   forward:  X[k] = sum_t x[t] exp(-2 pi i k t / n)
 *   backward: x[t] = sum_k X[k] exp(+2 pi i k t / n)       (no 1/n)
 * Complex transforms use a mixed-radix Stockham autosort FFT (radices 4, 2,
 * 3, 5, then any remaining prime by a direct small DFT).  Even-length real
 * transforms use the standard half-length complex packing (real and odd
 * samples as one complex sequence, then a split step); odd lengths go through
 * a full-length complex transform.  Multi-dimensional transforms run the real
 * transform along the last dimension and complex transforms along the others
 * (row-column).
 *
 * Compiled twice: with -DAGD_SHIM_FLOAT it defines the fftwf_* symbols in
 * single precision, otherwise the fftw_* symbols in double precision.
 * Twiddle factors are computed in double precision and rounded once.
 * Plans are read-only during execution, so one plan may be executed
 * concurrently from several threads on different arrays (the reference does
 * this under OpenMP, src/model.c:1073-1101); scratch space is thread-local.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include "fftw3.h"

#ifdef AGD_SHIM_FLOAT
typedef float R;
typedef fftwf_complex CPX;
typedef fftwf_plan PLANPTR;
#define PFX(name) fftwf_##name
#define PLAN_STRUCT agd_shim_plan_f
#else
typedef double R;
typedef fftw_complex CPX;
typedef fftw_plan PLANPTR;
#define PFX(name) fftw_##name
#define PLAN_STRUCT agd_shim_plan_d
#endif

#define SHIM_PI 3.14159265358979323846
#define MAX_RANK 8
#define MAX_FACTORS 40

typedef struct {
  R re;
  R im;
} cpx;

/* Complex FFT of one length, forward and backward share the tables. */
typedef struct {
  int n;
  int n_factors;
  int factors[MAX_FACTORS];
  cpx *tw; /* tw[k] = exp(-2 pi i k / n), k < n */
} cfft;

enum { KIND_R2C = 0, KIND_C2R = 1 };

struct PLAN_STRUCT {
  int kind;
  int rank;
  int n[MAX_RANK];
  int howmany;
  int idist;
  int odist;
  void *in;
  void *out;
  long n_real;   /* product of n */
  long n_cplx;   /* product of n[0..rank-2] * (n[rank-1]/2+1) */
  cfft dim[MAX_RANK]; /* complex FFT per leading dimension */
  cfft last;          /* complex FFT along the last dimension (n/2 or n) */
  cpx *split_tw;      /* exp(-2 pi i k / n_last), k <= n_last/2 (even n) */
};

static int cfft_init(cfft *const p, int const n) {
  int m = n;
  int k;
  p->n = n;
  p->n_factors = 0;
  while (m % 4 == 0) {
    p->factors[p->n_factors++] = 4;
    m /= 4;
  }
  while (m % 2 == 0) {
    p->factors[p->n_factors++] = 2;
    m /= 2;
  }
  while (m % 3 == 0) {
    p->factors[p->n_factors++] = 3;
    m /= 3;
  }
  while (m % 5 == 0) {
    p->factors[p->n_factors++] = 5;
    m /= 5;
  }
  {
    int q = 7;
    while (m > 1) {
      while (m % q == 0) {
        if (p->n_factors >= MAX_FACTORS) return 1;
        p->factors[p->n_factors++] = q;
        m /= q;
      }
      q += 2;
    }
  }
  p->tw = (cpx *)malloc((size_t)(n > 0 ? n : 1) * sizeof(cpx));
  if (p->tw == NULL) return 1;
  for (k = 0; k < n; k++) {
    double const a = -2.0 * SHIM_PI * (double)k / (double)n;
    p->tw[k].re = (R)cos(a);
    p->tw[k].im = (R)sin(a);
  }
  return 0;
}

static void cfft_free(cfft *const p) {
  free(p->tw);
  p->tw = NULL;
}

/* Thread-local scratch, grown on demand. */
static _Thread_local cpx *tl_buf[3];
static _Thread_local size_t tl_cap[3];

static cpx *scratch(int const which, size_t const n) {
  if (tl_cap[which] < n) {
    free(tl_buf[which]);
    tl_buf[which] = (cpx *)malloc(n * sizeof(cpx));
    tl_cap[which] = tl_buf[which] != NULL ? n : 0;
  }
  return tl_buf[which];
}

static inline cpx cmul(cpx const a, cpx const b) {
  cpx r;
  r.re = a.re * b.re - a.im * b.im;
  r.im = a.re * b.im + a.im * b.re;
  return r;
}

static inline cpx twid(cfft const *const p, long const idx, int const inverse) {
  cpx w = p->tw[idx % p->n];
  if (inverse) w.im = -w.im;
  return w;
}

/* One Stockham pass of radix R over a contiguous sequence. */
static void stockham_pass(cfft const *const p, int const radix, int const ns,
                          cpx const *const a, cpx *const b,
                          int const inverse) {
  int const n = p->n;
  int const m = n / radix;
  long const tw_step = n / (ns * radix);
  int j;
  for (j = 0; j < m; j++) {
    int const k = j % ns;
    int const base = (j / ns) * ns * radix + k;
    cpx v[64];
    int r;
    if (radix > 64) break; /* guarded by cfft_pass_generic */
    v[0] = a[j];
    for (r = 1; r < radix; r++) {
      v[r] = cmul(a[j + r * m], twid(p, (long)r * k * tw_step, inverse));
    }
    if (radix == 2) {
      b[base] = (cpx){v[0].re + v[1].re, v[0].im + v[1].im};
      b[base + ns] = (cpx){v[0].re - v[1].re, v[0].im - v[1].im};
    } else if (radix == 4) {
      /* X0 = a+b+c+d, X1 = a - s i b - c + s i d, ... with s = -1 forward */
      cpx const s02 = {v[0].re + v[2].re, v[0].im + v[2].im};
      cpx const d02 = {v[0].re - v[2].re, v[0].im - v[2].im};
      cpx const s13 = {v[1].re + v[3].re, v[1].im + v[3].im};
      cpx const d13 = {v[1].re - v[3].re, v[1].im - v[3].im};
      /* rot = -i * d13 (forward) or +i * d13 (inverse) */
      cpx const rot = inverse ? (cpx){-d13.im, d13.re} : (cpx){d13.im, -d13.re};
      b[base] = (cpx){s02.re + s13.re, s02.im + s13.im};
      b[base + ns] = (cpx){d02.re + rot.re, d02.im + rot.im};
      b[base + 2 * ns] = (cpx){s02.re - s13.re, s02.im - s13.im};
      b[base + 3 * ns] = (cpx){d02.re - rot.re, d02.im - rot.im};
    } else {
      long const step = n / radix;
      int q;
      for (q = 0; q < radix; q++) {
        cpx acc = v[0];
        for (r = 1; r < radix; r++) {
          cpx const t = cmul(v[r], twid(p, (long)r * q * step, inverse));
          acc.re += t.re;
          acc.im += t.im;
        }
        b[base + q * ns] = acc;
      }
    }
  }
}

/* Direct DFT for a radix too large for the pass buffer. */
static void direct_dft(cfft const *const p, cpx const *const a, cpx *const b,
                       int const inverse) {
  int const n = p->n;
  int q;
  for (q = 0; q < n; q++) {
    double re = 0.0;
    double im = 0.0;
    int t;
    for (t = 0; t < n; t++) {
      cpx const w = twid(p, (long)q * t, inverse);
      re += (double)a[t].re * w.re - (double)a[t].im * w.im;
      im += (double)a[t].re * w.im + (double)a[t].im * w.re;
    }
    b[q].re = (R)re;
    b[q].im = (R)im;
  }
}

/* Transform one contiguous sequence in place (uses scratch slot 2). */
static void cfft_exec(cfft const *const p, cpx *const data, int const inverse) {
  int const n = p->n;
  cpx *a = data;
  cpx *b;
  int ns = 1;
  int f;
  if (n <= 1) return;
  b = scratch(2, (size_t)n);
  for (f = 0; f < p->n_factors; f++) {
    int const radix = p->factors[f];
    if (radix > 64) {
      if (p->n_factors != 1) {
        /* large prime factor mixed with others: fall back to a direct DFT */
        if (a != data) memcpy(data, a, (size_t)n * sizeof(cpx));
        direct_dft(p, data, b, inverse);
        memcpy(data, b, (size_t)n * sizeof(cpx));
        return;
      }
      direct_dft(p, a, b, inverse);
    } else {
      stockham_pass(p, radix, ns, a, b, inverse);
    }
    {
      cpx *const t = a;
      a = b;
      b = t;
    }
    ns *= radix;
  }
  if (a != data) memcpy(data, a, (size_t)n * sizeof(cpx));
}

/* Complex FFT along dimension `d` of a C-ordered complex array. */
static void cfft_along(cfft const *const p, cpx *const arr, long const outer,
                       long const inner, int const inverse) {
  int const n = p->n;
  cpx *const line = scratch(1, (size_t)n);
  long o;
  long i;
  int t;
  if (n <= 1) return;
  for (o = 0; o < outer; o++) {
    cpx *const block = arr + o * (long)n * inner;
    for (i = 0; i < inner; i++) {
      for (t = 0; t < n; t++) line[t] = block[(long)t * inner + i];
      cfft_exec(p, line, inverse);
      for (t = 0; t < n; t++) block[(long)t * inner + i] = line[t];
    }
  }
}

/* Real to half-complex along one line of length n (out has n/2+1 bins). */
static void r2c_line(struct PLAN_STRUCT const *const p, R const *const x,
                     cpx *const out) {
  int const n = p->n[p->rank - 1];
  if (n % 2 == 0 && n >= 2) {
    int const h = n / 2;
    cpx *const z = scratch(0, (size_t)h);
    int k;
    for (k = 0; k < h; k++) {
      z[k].re = x[2 * k];
      z[k].im = x[2 * k + 1];
    }
    cfft_exec(&p->last, z, 0);
    for (k = 0; k <= h; k++) {
      cpx const zk = z[k % h];
      cpx const zc = {z[(h - k) % h].re, -z[(h - k) % h].im};
      cpx const e = {(R)0.5 * (zk.re + zc.re), (R)0.5 * (zk.im + zc.im)};
      /* o = (zk - zc) / (2i) */
      cpx const o = {(R)0.5 * (zk.im - zc.im), -(R)0.5 * (zk.re - zc.re)};
      cpx const wo = cmul(p->split_tw[k], o);
      out[k].re = e.re + wo.re;
      out[k].im = e.im + wo.im;
    }
  } else {
    cpx *const z = scratch(0, (size_t)n);
    int k;
    for (k = 0; k < n; k++) {
      z[k].re = x[k];
      z[k].im = (R)0;
    }
    cfft_exec(&p->last, z, 0);
    for (k = 0; k <= n / 2; k++) out[k] = z[k];
  }
}

/* Half-complex (n/2+1 bins) to real along one line of length n. */
static void c2r_line(struct PLAN_STRUCT const *const p, cpx const *const in,
                     R *const x) {
  int const n = p->n[p->rank - 1];
  if (n % 2 == 0 && n >= 2) {
    int const h = n / 2;
    cpx *const z = scratch(0, (size_t)h);
    int k;
    for (k = 0; k < h; k++) {
      cpx a = in[k];
      cpx b = in[h - k];
      if (k == 0) {
        a.im = (R)0;
        b.im = (R)0;
      }
      {
        cpx const bc = {b.re, -b.im};
        cpx const e = {a.re + bc.re, a.im + bc.im};
        cpx const d = {a.re - bc.re, a.im - bc.im};
        cpx const w = {p->split_tw[k].re, -p->split_tw[k].im};
        cpx const o = cmul(d, w);
        z[k].re = e.re - o.im;
        z[k].im = e.im + o.re;
      }
    }
    cfft_exec(&p->last, z, 1);
    for (k = 0; k < h; k++) {
      x[2 * k] = z[k].re;
      x[2 * k + 1] = z[k].im;
    }
  } else {
    cpx *const z = scratch(0, (size_t)n);
    int k;
    for (k = 0; k < n; k++) {
      if (k <= n / 2) {
        z[k] = in[k];
      } else {
        z[k].re = in[n - k].re;
        z[k].im = -in[n - k].im;
      }
    }
    z[0].im = (R)0;
    cfft_exec(&p->last, z, 1);
    for (k = 0; k < n; k++) x[k] = z[k].re;
  }
}

static PLANPTR make_plan(int const kind, int const rank, const int *const n,
                         int const howmany, void *const in,
                         const int *const inembed, int const istride,
                         int const idist, void *const out,
                         const int *const onembed, int const ostride,
                         int const odist) {
  struct PLAN_STRUCT *p;
  int d;
  int nl;
  if (rank < 1 || rank > MAX_RANK || howmany < 0) return NULL;
  if (inembed != NULL || onembed != NULL || istride != 1 || ostride != 1)
    return NULL;
  p = (struct PLAN_STRUCT *)calloc(1, sizeof(*p));
  if (p == NULL) return NULL;
  p->kind = kind;
  p->rank = rank;
  p->howmany = howmany;
  p->idist = idist;
  p->odist = odist;
  p->in = in;
  p->out = out;
  p->n_real = 1;
  p->n_cplx = 1;
  for (d = 0; d < rank; d++) {
    if (n[d] < 1) {
      free(p);
      return NULL;
    }
    p->n[d] = n[d];
    p->n_real *= n[d];
    p->n_cplx *= (d == rank - 1) ? (n[d] / 2 + 1) : n[d];
  }
  for (d = 0; d < rank - 1; d++) {
    if (cfft_init(&p->dim[d], n[d])) goto err;
  }
  nl = n[rank - 1];
  if (nl % 2 == 0 && nl >= 2) {
    int k;
    if (cfft_init(&p->last, nl / 2)) goto err;
    p->split_tw = (cpx *)malloc((size_t)(nl / 2 + 1) * sizeof(cpx));
    if (p->split_tw == NULL) goto err;
    for (k = 0; k <= nl / 2; k++) {
      double const a = -2.0 * SHIM_PI * (double)k / (double)nl;
      p->split_tw[k].re = (R)cos(a);
      p->split_tw[k].im = (R)sin(a);
    }
  } else {
    if (cfft_init(&p->last, nl)) goto err;
  }
  return (PLANPTR)p;
err:
  for (d = 0; d < MAX_RANK; d++) cfft_free(&p->dim[d]);
  cfft_free(&p->last);
  free(p->split_tw);
  free(p);
  return NULL;
}

static void exec_r2c(struct PLAN_STRUCT const *const p, R const *const in,
                     cpx *const out) {
  int const nl = p->n[p->rank - 1];
  int const fl = nl / 2 + 1;
  long const rows = p->n_real / nl;
  int b;
  for (b = 0; b < p->howmany; b++) {
    R const *const x = in + (long)b * p->idist;
    cpx *const y = out + (long)b * p->odist;
    long r;
    int d;
    for (r = 0; r < rows; r++) r2c_line(p, x + r * nl, y + r * fl);
    for (d = p->rank - 2; d >= 0; d--) {
      long outer = 1;
      long inner = fl;
      int e;
      for (e = 0; e < d; e++) outer *= p->n[e];
      for (e = d + 1; e < p->rank - 1; e++) inner *= p->n[e];
      cfft_along(&p->dim[d], y, outer, inner, 0);
    }
  }
}

static void exec_c2r(struct PLAN_STRUCT const *const p, cpx const *const in,
                     R *const out) {
  int const nl = p->n[p->rank - 1];
  int const fl = nl / 2 + 1;
  long const rows = p->n_real / nl;
  int b;
  /* The input is left unmodified: work on a copy. */
  cpx *work = (cpx *)malloc((size_t)(p->n_cplx > 0 ? p->n_cplx : 1) *
                            sizeof(cpx));
  if (work == NULL) return;
  for (b = 0; b < p->howmany; b++) {
    cpx const *const y = in + (long)b * p->idist;
    R *const x = out + (long)b * p->odist;
    long r;
    int d;
    memcpy(work, y, (size_t)p->n_cplx * sizeof(cpx));
    for (d = 0; d < p->rank - 1; d++) {
      long outer = 1;
      long inner = fl;
      int e;
      for (e = 0; e < d; e++) outer *= p->n[e];
      for (e = d + 1; e < p->rank - 1; e++) inner *= p->n[e];
      cfft_along(&p->dim[d], work, outer, inner, 1);
    }
    for (r = 0; r < rows; r++) c2r_line(p, work + r * fl, x + r * nl);
  }
  free(work);
}

PLANPTR PFX(plan_many_dft_r2c)(int rank, const int *n, int howmany, R *in,
                               const int *inembed, int istride, int idist,
                               CPX *out, const int *onembed, int ostride,
                               int odist, unsigned flags) {
  (void)flags;
  return make_plan(KIND_R2C, rank, n, howmany, in, inembed, istride, idist,
                   out, onembed, ostride, odist);
}

PLANPTR PFX(plan_many_dft_c2r)(int rank, const int *n, int howmany, CPX *in,
                               const int *inembed, int istride, int idist,
                               R *out, const int *onembed, int ostride,
                               int odist, unsigned flags) {
  (void)flags;
  return make_plan(KIND_C2R, rank, n, howmany, in, inembed, istride, idist,
                   out, onembed, ostride, odist);
}

PLANPTR PFX(plan_dft_r2c_1d)(int n, R *in, CPX *out, unsigned flags) {
  return PFX(plan_many_dft_r2c)(1, &n, 1, in, NULL, 1, n, out, NULL, 1,
                                n / 2 + 1, flags);
}

PLANPTR PFX(plan_dft_c2r_1d)(int n, CPX *in, R *out, unsigned flags) {
  return PFX(plan_many_dft_c2r)(1, &n, 1, in, NULL, 1, n / 2 + 1, out, NULL, 1,
                                n, flags);
}

void PFX(execute_dft_r2c)(const PLANPTR plan, R *in, CPX *out) {
  struct PLAN_STRUCT const *const p = (struct PLAN_STRUCT const *)plan;
  if (p == NULL || p->kind != KIND_R2C) return;
  exec_r2c(p, in, (cpx *)out);
}

void PFX(execute_dft_c2r)(const PLANPTR plan, CPX *in, R *out) {
  struct PLAN_STRUCT const *const p = (struct PLAN_STRUCT const *)plan;
  if (p == NULL || p->kind != KIND_C2R) return;
  exec_c2r(p, (cpx const *)in, out);
}

void PFX(execute)(const PLANPTR plan) {
  struct PLAN_STRUCT const *const p = (struct PLAN_STRUCT const *)plan;
  if (p == NULL) return;
  if (p->kind == KIND_R2C) {
    exec_r2c(p, (R const *)p->in, (cpx *)p->out);
  } else {
    exec_c2r(p, (cpx const *)p->in, (R *)p->out);
  }
}

void PFX(destroy_plan)(PLANPTR plan) {
  struct PLAN_STRUCT *const p = (struct PLAN_STRUCT *)plan;
  int d;
  if (p == NULL) return;
  for (d = 0; d < MAX_RANK; d++) cfft_free(&p->dim[d]);
  cfft_free(&p->last);
  free(p->split_tw);
  free(p);
}

void *PFX(malloc)(size_t n) { return malloc(n > 0 ? n : 1); }

void PFX(free)(void *p) { free(p); }

CPX *PFX(alloc_complex)(size_t n) {
  return (CPX *)malloc((n > 0 ? n : 1) * sizeof(CPX));
}

R *PFX(alloc_real)(size_t n) { return (R *)malloc((n > 0 ? n : 1) * sizeof(R)); }
