/*
 * kmm_cpu.c - FP64 CPU restatement of the KMM RK3 time step, in C with OpenMP.
 *
 * TEST INFRASTRUCTURE ONLY.  This is the oracle's compiled twin: the same algorithm as
 * oracle/kmm.py (each routine cites the reference routine it restates), fast enough to run the
 * long trajectories of the parity tests at the benchmark's grid and to serve as the timed CPU
 * baseline.  The product library never links, loads or calls it; only tests/, the smoke check
 * and bench.py's CPU legs do.  Parity against the reference binary is unpinned (the reference
 * cannot be built here: no gfortran, MPI, FFTW, GSL or HDF5), exactly as for oracle/kmm.py,
 * which this file is checked against.
 *
 * Layouts (C order, the Fortran shapes reversed; complex = interleaved re, im doubles):
 *   U   [10][nz][nxh][ny]   = Fortran U(ny, nxh, nz, 10)          (wavespace.f90:29)
 *   RK  [3][nz][nxh][ny]    = Fortran RK_STORE(ny, nxh, nz, 3)
 *   bands (2bw+1, ny) Fortran column-major: entry r (1-based) of column j at [(j-1)(2bw+1)+r-1]
 * Wavenumbers: kx = 0..nxh-1; kz = 0..nz/2, -nz/2+1..-1 (set_waveno, module_ppdfftw.f90:347-384).
 *
 * One substep (time_march, time_march.f90:36-128), per wall-normal plane y in parallel:
 *   y_to_x + ppdfftw_dft_z_inverse (module_ppdfftw.f90:830-861): pad in kz, backward c2c in z;
 *   dft_x_realspace (dft_x_realspace.f90:68-213): pad in kx, c2r in x, products, CFL maximum,
 *     r2c in x, truncate;
 *   x_to_y + ppdfftw_dft_z_forward (module_ppdfftw.f90:794-823): forward c2c in z, truncate,
 *     zero the kz Nyquist row; rescale_data (rescale_data.f90:10-39).
 * then per (kx, kz) mode in parallel: wavespace (wavespace.f90:22-113) = hvhg, solve_g,
 * solve_v_f (with the opposition-control wall values), solve_u_w, solve_t; and wave00 for (0,0).
 * FFTW's unnormalised conventions are restated with a self-sorting mixed-radix (2, 3, 4, 5)
 * Stockham FFT written here.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

typedef struct {
  double re, im;
} cx;

static inline cx C(double re, double im) { cx z = {re, im}; return z; }
static inline cx cadd(cx a, cx b) { return C(a.re + b.re, a.im + b.im); }
static inline cx csub(cx a, cx b) { return C(a.re - b.re, a.im - b.im); }
static inline cx cmul(cx a, cx b) { return C(a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re); }
static inline cx cscale(double s, cx a) { return C(s * a.re, s * a.im); }
static inline cx cimul(double s, cx a) { return C(-s * a.im, s * a.re); } /* (i s) a */
static inline cx cdiv(cx a, cx b) {
  const double d = b.re * b.re + b.im * b.im;
  return C((a.re * b.re + a.im * b.im) / d, (a.im * b.re - a.re * b.im) / d);
}

/* ------------------------------------------------------------------------------------------ */
/* FFT: self-sorting Stockham, decimation in frequency.  A length-n stage with radix r and     */
/* m = n / r maps element (q + s (p + j m)) to (q + s (r p + k)) with the twiddle W_n^{p k};   */
/* the next stage runs on length m with stride r s.  Lines are batched along the fastest axis: */
/* element i of line l sits at x[i * B + l].                                                    */
/* ------------------------------------------------------------------------------------------ */
typedef struct {
  int n, nf;
  int f[24];
  cx *tw[24]; /* per stage: tw[st][p * r + k] = W_n^{p k}, n the stage's length */
} fftplan;

static int plan_init(fftplan *P, int n) {
  P->n = n;
  P->nf = 0;
  int m = n;
  while (m % 4 == 0) { P->f[P->nf++] = 4; m /= 4; }
  while (m % 2 == 0) { P->f[P->nf++] = 2; m /= 2; }
  while (m % 3 == 0) { P->f[P->nf++] = 3; m /= 3; }
  while (m % 5 == 0) { P->f[P->nf++] = 5; m /= 5; }
  if (m != 1) return -1;
  int len = n;
  for (int st = 0; st < P->nf; ++st) {
    const int r = P->f[st], mm = len / r;
    P->tw[st] = (cx *)malloc(sizeof(cx) * (size_t)len);
    for (int p = 0; p < mm; ++p)
      for (int k = 0; k < r; ++k) {
        const long t = ((long)p * k) % len;
        const long double a = -2.0L * 3.141592653589793238462643383279502884L * (long double)t / (long double)len;
        P->tw[st][p * r + k] = C((double)cosl(a), (double)sinl(a));
      }
    len = mm;
  }
  return 0;
}

static void plan_free(fftplan *P) {
  for (int st = 0; st < P->nf; ++st) free(P->tw[st]);
}

/* twiddle w (forward) or its conjugate (backward) times t */
static inline cx twmul(cx t, cx w, int sign) {
  return sign < 0 ? cmul(t, w) : C(t.re * w.re + t.im * w.im, t.im * w.re - t.re * w.im);
}

/* One Stockham stage of radix R over B batched lines (R fixed so the loops unroll). */
#define STAGE_BODY(R, ...)                                                                     \
  for (int p = 0; p < m; ++p) {                                                                \
    const cx *w = tw + p * R;                                                                  \
    for (int q = 0; q < s; ++q) {                                                              \
      const cx *src = a + (size_t)(q + s * p) * B;                                             \
      cx *dst = b + (size_t)(q + s * R * p) * B;                                               \
      const size_t is = (size_t)s * m * B, os = (size_t)s * B;                                 \
      for (int l = 0; l < B; ++l) {                                                            \
        cx v[R], t[R];                                                                         \
        for (int j = 0; j < R; ++j) v[j] = src[j * is + l];                                    \
        __VA_ARGS__;                                                                           \
        dst[l] = t[0];                                                                         \
        for (int k = 1; k < R; ++k) dst[k * os + l] = twmul(t[k], w[k], sign);                 \
      }                                                                                        \
    }                                                                                          \
  }

static void stage2(const cx *a, cx *b, const cx *tw, int m, int s, int B, int sign) {
  STAGE_BODY(2, { t[0] = cadd(v[0], v[1]); t[1] = csub(v[0], v[1]); })
}

static void stage4(const cx *a, cx *b, const cx *tw, int m, int s, int B, int sign) {
  STAGE_BODY(4, {
    const cx s02 = cadd(v[0], v[2]), d02 = csub(v[0], v[2]);
    const cx s13 = cadd(v[1], v[3]), d13 = csub(v[1], v[3]);
    const cx jd = cimul((double)sign, d13); /* forward: -i d13 */
    t[0] = cadd(s02, s13);
    t[2] = csub(s02, s13);
    t[1] = cadd(d02, jd);
    t[3] = csub(d02, jd);
  })
}

static void stage3(const cx *a, cx *b, const cx *tw, int m, int s, int B, int sign) {
  const double c = -0.5, sn = (double)sign * 0.86602540378443864676372317075294;
  STAGE_BODY(3, {
    const cx sum = cadd(v[1], v[2]), dif = csub(v[1], v[2]);
    const cx base = C(v[0].re + c * sum.re, v[0].im + c * sum.im);
    const cx rot = cimul(sn, dif);
    t[0] = cadd(v[0], sum);
    t[1] = cadd(base, rot);
    t[2] = csub(base, rot);
  })
}

static void stage5(const cx *a, cx *b, const cx *tw, int m, int s, int B, int sign) {
  const double c1 = 0.30901699437494742410229341718282, c2 = -0.80901699437494742410229341718282;
  const double s1 = (double)sign * 0.95105651629515357211643933337938;
  const double s2 = (double)sign * 0.58778525229247312916870595463907;
  STAGE_BODY(5, {
    const cx p1 = cadd(v[1], v[4]), m1 = csub(v[1], v[4]);
    const cx p2 = cadd(v[2], v[3]), m2 = csub(v[2], v[3]);
    const cx b1 = C(v[0].re + c1 * p1.re + c2 * p2.re, v[0].im + c1 * p1.im + c2 * p2.im);
    const cx b2 = C(v[0].re + c2 * p1.re + c1 * p2.re, v[0].im + c2 * p1.im + c1 * p2.im);
    const cx r1 = cadd(cimul(s1, m1), cimul(s2, m2));
    const cx r2 = csub(cimul(s2, m1), cimul(s1, m2));
    t[0] = cadd(v[0], cadd(p1, p2));
    t[1] = cadd(b1, r1);
    t[4] = csub(b1, r1);
    t[2] = cadd(b2, r2);
    t[3] = csub(b2, r2);
  })
}
#undef STAGE_BODY

/* Unnormalised transform of B lines in place: sign -1 forward (e^{-i}, FFTW_FORWARD), +1
 * backward (e^{+i}, FFTW_BACKWARD).  work holds n * B complex. */
static void fft_batch(const fftplan *P, cx *x, cx *work, int B, int sign) {
  const int N = P->n;
  int n = N, s = 1;
  cx *a = x, *b = work;
  for (int st = 0; st < P->nf; ++st) {
    const int r = P->f[st], m = n / r;
    switch (r) {
      case 4: stage4(a, b, P->tw[st], m, s, B, sign); break;
      case 2: stage2(a, b, P->tw[st], m, s, B, sign); break;
      case 3: stage3(a, b, P->tw[st], m, s, B, sign); break;
      default: stage5(a, b, P->tw[st], m, s, B, sign); break;
    }
    n = m;
    s *= r;
    cx *tmp = a;
    a = b;
    b = tmp;
  }
  if (a != x) memcpy(x, a, sizeof(cx) * (size_t)N * B);
}

/* ------------------------------------------------------------------------------------------ */
/* LABS packed-band routines (module_labs.f90), in the reference's loop orders.                 */
/* ------------------------------------------------------------------------------------------ */
#define A_(r, c) A[((c)-1) * ld + (r)-1]
/* The per-mode chain is inlined into one function per band width (solve_mode_bw), so bw is a
 * compile-time constant in every loop below. */
#define KO_INLINE static inline __attribute__((always_inline))

/* fixed_bandec (module_labs.f90:3487-3636): in-place Crout LU, no pivoting; L keeps the
 * pivots, U is unit upper. */
KO_INLINE void labs_lu(double *A, int bw, int n) {
  const int ld = 2 * bw + 1, m = bw + 1;
  for (int i = 1; i <= bw; ++i) { /* upper region */
    const double dummy = 1.0 / A_(m, i);
    for (int j = 1; j <= bw + 1 - i; ++j) {
      double acc = A_(m + j, i);
      for (int k = 1; k <= i - 1; ++k) acc -= A_(m - k, i) * A_(m + j + k, i - k);
      A_(m + j, i) = dummy * acc;
    }
    for (int j = bw + 2 - i; j <= bw; ++j) {
      double acc = A_(m + j, i);
      for (int k = 1; k <= bw - j; ++k) acc -= A_(m - k, i) * A_(m + j + k, i - k);
      for (int k = bw - j + 1; k <= i - 1; ++k) acc -= A_(m - k, i) * A_(m + bw - i - j + 1, i - k);
      A_(m + j, i) = dummy * acc;
    }
    for (int j = i; j <= bw; ++j) {
      double acc = A_(m - j, i);
      for (int k = 1; k <= i - 1; ++k) acc -= A_(m - k, i) * A_(m - j, i - k);
      A_(m - j, i) = dummy * acc;
    }
    for (int j = 1; j <= bw + 1 - i; ++j) {
      double acc = A_(m + 1 - j, i + j);
      for (int k = 1; k <= i; ++k) acc -= A_(m + 1 - j - k, i + j) * A_(m + k, i + 1 - k);
      A_(m + 1 - j, i + j) = acc;
    }
    for (int j = bw + 2 - i; j <= bw; ++j) {
      double acc = A_(m + 1 - j, i + j);
      for (int k = 1; k <= bw + 1 - j; ++k) acc -= A_(m + 1 - j - k, i + j) * A_(m + k, i + 1 - k);
      A_(m + 1 - j, i + j) = acc;
    }
  }
  for (int i = m; i <= 2 * bw; ++i) { /* subupper region */
    const double dummy = 1.0 / A_(m, i);
    for (int j = 1; j <= 2 * bw + 1 - i; ++j) {
      double acc = A_(m + j, i);
      for (int k = 1; k <= bw - j; ++k) acc -= A_(m - k, i) * A_(m + j + k, i - k);
      for (int k = bw - j + 1; k <= bw; ++k) acc -= A_(m - k, i) * A_(2 * m - i - j, i - k);
      A_(m + j, i) = dummy * acc;
    }
    for (int j = 2 * bw + 2 - i; j <= bw; ++j) {
      double acc = A_(m + j, i);
      for (int k = 1; k <= bw - j; ++k) acc -= A_(m - k, i) * A_(m + j + k, i - k);
      A_(m + j, i) = dummy * acc;
    }
    for (int j = 1; j <= bw; ++j) {
      double acc = A_(m - j + 1, i + j);
      for (int k = 1; k <= bw + 1 - j; ++k) acc -= A_(m - j + 1 - k, i + j) * A_(m + k, i - k + 1);
      A_(m - j + 1, i + j) = acc;
    }
  }
  for (int i = 2 * bw + 1; i <= n - 2 * bw - 1; ++i) { /* centre region */
    const double dummy = 1.0 / A_(m, i);
    for (int j = 1; j <= bw; ++j) {
      double acc = A_(m + j, i);
      for (int k = 1; k <= bw - j; ++k) acc -= A_(m - k, i) * A_(m + j + k, i - k);
      A_(m + j, i) = dummy * acc;
    }
    for (int j = 1; j <= bw; ++j) {
      double acc = A_(m - j + 1, i + j);
      for (int k = 1; k <= bw - j + 1; ++k) acc -= A_(m + 1 - j - k, i + j) * A_(m + k, i + 1 - k);
      A_(m - j + 1, i + j) = acc;
    }
  }
  for (int i = n - 2 * bw; i <= n - bw - 1; ++i) { /* sublower region */
    const double dummy = 1.0 / A_(m, i);
    for (int j = 1; j <= bw; ++j) {
      double acc = A_(m + j, i);
      for (int k = 1; k <= bw - j; ++k) acc -= A_(m - k, i) * A_(m + j + k, i - k);
      A_(m + j, i) = dummy * acc;
    }
    for (int j = 1; j <= n - bw - i; ++j) {
      double acc = A_(m - j + 1, i + j);
      for (int k = 1; k <= bw - j + 1; ++k) acc -= A_(m + 1 - j - k, i + j) * A_(m + k, i + 1 - k);
      A_(m - j + 1, i + j) = acc;
    }
    for (int j = n - bw - i + 1; j <= bw + 1; ++j) {
      double acc = A_(m - j + 1, i + j);
      for (int k = 1; k <= bw + 1 - j; ++k) acc -= A_(m + 1 - j - k, i + j) * A_(m + k, i + 1 - k);
      for (int k = bw + 2 - j; k <= i - n + 2 * bw + 1; ++k)
        acc -= A_(m + n - bw - 1 + k - i, i + j) * A_(m + k, i + 1 - k);
      A_(m - j + 1, i + j) = acc;
    }
    for (int j = bw + 2; j <= n - i; ++j) {
      double acc = A_(m + n - bw - 1 - i, i + j);
      for (int k = 1; k <= i - n + 2 * bw + 1; ++k) acc -= A_(m + n - bw - 1 - i + k, i + j) * A_(m + k, i + 1 - k);
      A_(m + n - bw - 1 - i, i + j) = acc;
    }
  }
  for (int i = n - bw; i <= n - 1; ++i) { /* lower region */
    const double dummy = 1.0 / A_(m, i);
    for (int j = 1; j <= n - i; ++j) {
      double acc = A_(m + j, i);
      for (int k = 1; k <= bw - j; ++k) acc -= A_(m - k, i) * A_(m + j + k, i - k);
      A_(m + j, i) = dummy * acc;
    }
    for (int j = 1; j <= n - i; ++j) {
      double acc = A_(m - j + 1, i + j);
      for (int k = 1; k <= bw + 1 - j; ++k) acc -= A_(m + 1 - j - k, i + j) * A_(m + k, i + 1 - k);
      for (int k = bw + 2 - j; k <= bw; ++k) acc -= A_(m + n - bw - 1 - i + k, i + j) * A_(m + k, i + 1 - k);
      A_(m - j + 1, i + j) = acc;
    }
  }
}

/* fixed_banbks (module_labs.f90:4252-4318): solve in place with the factored band (complex). */
KO_INLINE void labs_bs(const double *A, int bw, int n, cx *b) {
  const int ld = 2 * bw + 1, m = bw + 1;
  for (int i = 1; i <= bw; ++i) {
    cx acc = b[i - 1];
    for (int j = 1; j <= i - 1; ++j) acc = csub(acc, cscale(A_(m - i + j, i), b[j - 1]));
    b[i - 1] = C(acc.re / A_(m, i), acc.im / A_(m, i));
  }
  for (int i = bw + 1; i <= n - bw; ++i) {
    cx acc = b[i - 1];
    for (int j = 1; j <= bw; ++j) acc = csub(acc, cscale(A_(m - bw - 1 + j, i), b[i - bw - 2 + j]));
    b[i - 1] = C(acc.re / A_(m, i), acc.im / A_(m, i));
  }
  for (int i = 1; i <= bw; ++i) {
    const int r = n - bw + i;
    cx acc = b[r - 1];
    for (int j = 1; j <= i; ++j) acc = csub(acc, cscale(A_(m + bw + 1 - j, r), b[n - 2 * bw - 2 + j]));
    for (int j = i + 1; j <= i + bw; ++j) acc = csub(acc, cscale(A_(m - bw + j - i - 1, r), b[n - 2 * bw - 2 + j]));
    b[r - 1] = C(acc.re / A_(m, r), acc.im / A_(m, r));
  }
  for (int i = 1; i <= bw - 1; ++i) {
    cx acc = b[n - i - 1];
    for (int j = 1; j <= i; ++j) acc = csub(acc, cscale(A_(m + j, n - i), b[n - i + j - 1]));
    b[n - i - 1] = acc;
  }
  for (int i = n - bw; i >= bw + 1; --i) {
    cx acc = b[i - 1];
    for (int j = 1; j <= bw; ++j) acc = csub(acc, cscale(A_(m + j, i), b[i + j - 1]));
    b[i - 1] = acc;
  }
  for (int i = 1; i <= bw; ++i) {
    const int r = bw + 1 - i;
    cx acc = b[r - 1];
    for (int j = 1; j <= bw; ++j) acc = csub(acc, cscale(A_(m + j, r), b[r + j - 1]));
    for (int j = bw + 1; j <= bw + i; ++j) acc = csub(acc, cscale(A_(m + i - j, r), b[r + j - 1]));
    b[r - 1] = acc;
  }
}

/* LABS_mat_mul_bw (module_labs.f90:4687-4722): out = A x. */
KO_INLINE void labs_mm(const double *A, int bw, int n, const cx *x, cx *out) {
  const int ld = 2 * bw + 1;
  for (int j = 1; j <= bw; ++j) {
    cx acc = C(0.0, 0.0);
    for (int i = 1 - j; i <= bw; ++i) acc = cadd(acc, cscale(A_(bw + 1 + i, j), x[j + i - 1]));
    for (int i = 1; i <= bw + 1 - j; ++i) acc = cadd(acc, cscale(A_(bw + 2 - j - i, j), x[j + bw + i - 1]));
    out[j - 1] = acc;
  }
  for (int j = bw + 1; j <= n - bw; ++j) {
    cx acc = C(0.0, 0.0);
    for (int i = -bw; i <= bw; ++i) acc = cadd(acc, cscale(A_(bw + 1 + i, j), x[j + i - 1]));
    out[j - 1] = acc;
  }
  for (int j = n - bw + 1; j <= n; ++j) {
    cx acc = C(0.0, 0.0);
    for (int i = -bw; i <= n - j; ++i) acc = cadd(acc, cscale(A_(bw + 1 + i, j), x[j + i - 1]));
    for (int i = 1; i <= j - n + bw; ++i) acc = cadd(acc, cscale(A_(n + bw + 1 - j + i, j), x[j - bw - i - 1]));
    out[j - 1] = acc;
  }
}
#undef A_

/* ------------------------------------------------------------------------------------------ */
/* Problem description                                                                         */
/* ------------------------------------------------------------------------------------------ */
typedef struct kmm_oracle_params {
  int32_t nx, ny, nz, bw;
  double lmfx, lmfz;
  double nu, pr;
  double bulk_u, bulk_w, bulk_t, u_gal;
  double cflx;       /* CFL / pi (read_input_file.f90:107) */
  double dt_factor;
  double dxr, dzr;   /* nx / Lx, nz / Lz (read_input_file.f90:105-106) */
  int32_t fixed_dt;  /* 1: dt held */
  int32_t nthreads;  /* 0: OpenMP default */
  double control_amp;
} kmm_oracle_params;

/* Operators: D0, D1, D2, D0_LU bands, integration weights, 1/dy (module_ppdfftw.f90:573-583),
 * control weights w_lo, w_hi (v(+-y_d) = w . v), per-mode gains [nz][nxh] (NULL = 1). */
typedef struct kmm_oracle_ops {
  const double *d0, *d1, *d2, *d0lu;
  const double *integ, *dyr, *wlo, *whi;
  const double *gains;
} kmm_oracle_ops;

typedef struct kmm_oracle_scalars {
  double dt, velmax;
  double phi_dpdx[4], phi_dtdx[4];
  double wall_shear_stress, wall_theta_stress;
} kmm_oracle_scalars;

/* module_runge_kutta.f90:33-48 */
static const double RK_ALPHA[3] = {29.0 / 96.0, -3.0 / 40.0, 1.0 / 6.0};
static const double RK_BETA[3] = {37.0 / 160.0, 5.0 / 24.0, 1.0 / 6.0};
static const double RK_GAMMA[3] = {8.0 / 15.0, 5.0 / 12.0, 3.0 / 4.0};
static const double RK_ZETA[3] = {0.0, -17.0 / 60.0, -5.0 / 12.0};

/* ------------------------------------------------------------------------------------------ */
/* Transforms of one wall-normal plane                                                          */
/* ------------------------------------------------------------------------------------------ */
typedef struct {
  fftplan pz, px;
  int nx, nz, nxh, nx32, nz32, nh;
} tplans;

/* The nine product planes, in the order of U's product slots after x_to_y
 * (dft_x_realspace.f90:109-123; 0-based slots 0-4, 6-9): uu - vv, uv, ww - vv, vw, uw, u theta,
 * v theta, w theta, and v itself (vold, slot 9). */

/* One plane: in = state planes [4][nz][nxh] (u, v, w, theta), out = product planes [9][nz][nxh]
 * (product slot order), rescaled.  Returns the plane's velocity maximum (substep 1). */
static double plane_step(const tplans *T, const cx *in, cx *out, double dxr, double dyr_y, double dzr,
                         int want_vel, double rescale, cx *zb, cx *xb, cx *xb2, cx *pw, cx *work) {
  const int nz = T->nz, nxh = T->nxh, nx32 = T->nx32, nz32 = T->nz32, nh = T->nh;
  const size_t zplane = (size_t)nz32 * nxh;
  /* y_to_x + ppdfftw_dft_z_inverse: pad in kz, backward c2c along z (batched over kx) */
  for (int f = 0; f < 4; ++f) {
    cx *z = zb + f * zplane;
    const cx *src = in + (size_t)f * nz * nxh;
    memset(z, 0, sizeof(cx) * zplane);
    for (int k = 0; k < nh; ++k) memcpy(z + (size_t)k * nxh, src + (size_t)k * nxh, sizeof(cx) * nxh);
    for (int k = nh + 1; k < nz; ++k) memcpy(z + (size_t)(k + nh) * nxh, src + (size_t)k * nxh, sizeof(cx) * nxh);
    fft_batch(&T->pz, z, work, nxh, +1);
  }
  /* dft_x_realspace: c2r along x of (u + i v) and (w + i theta) per z, batched over z.
   * xb[x][z]: Hermitian extension of a plus i times that of b; FFTW's c2r drops Im of DC. */
  for (int pr = 0; pr < 2; ++pr) {
    const cx *A = zb + (2 * pr) * zplane, *B = zb + (2 * pr + 1) * zplane;
    cx *X = pr == 0 ? xb : xb2;
    memset(X, 0, sizeof(cx) * (size_t)nx32 * nz32);
    for (int z = 0; z < nz32; ++z) {
      const cx *a = A + (size_t)z * nxh, *b = B + (size_t)z * nxh;
      X[z] = C(a[0].re, b[0].re);
      for (int k = 1; k < nxh; ++k) {
        /* bin k: a_k + i b_k; bin N - k: conj(a_k) + i conj(b_k) */
        X[(size_t)k * nz32 + z] = C(a[k].re - b[k].im, a[k].im + b[k].re);
        X[(size_t)(nx32 - k) * nz32 + z] = C(a[k].re + b[k].im, -a[k].im + b[k].re);
      }
    }
    fft_batch(&T->px, X, work, nz32, +1);
  }
  /* products, CFL maximum (dft_x_realspace.f90:109-127) */
  double vmax = 0.0;
  const size_t np = (size_t)nx32 * nz32;
  /* the nine products, paired into five complex lines for the r2c: (f0,f1) (f2,f3) (f4,f6) (f7,f8) (f9, 0) */
  for (int pi = 0; pi < 5; ++pi) {
    cx *Pp = pw;
    for (size_t i = 0; i < np; ++i) {
      const double u = xb[i].re, v = xb[i].im, w = xb2[i].re, t = xb2[i].im;
      const double bv2 = v * v;
      double pa, pb;
      switch (pi) {
        case 0: pa = u * u - bv2; pb = u * v; break;
        case 1: pa = w * w - bv2; pb = v * w; break;
        case 2: pa = u * w; pb = u * t; break;
        case 3: pa = v * t; pb = w * t; break;
        default: pa = v; pb = 0.0; break;
      }
      Pp[i] = C(pa, pb);
      if (pi == 0 && want_vel) {
        const double vel = fabs(u) * dxr + fabs(v) * dyr_y + fabs(w) * dzr;
        if (vel > vmax) vmax = vel;
      }
    }
    fft_batch(&T->px, Pp, work, nz32, -1);
    /* unpack the two real transforms and keep kx < nxh, into the z-scratch of product q
     * (one [z][kx] plane each, behind the x buffer in pw) */
    for (int half = 0; half < 2; ++half) {
      const int q = 2 * pi + half;
      if (q >= 9) break;
      cx *dst = pw + np + (size_t)q * zplane;
      for (int z = 0; z < nz32; ++z) {
        for (int k = 0; k < nxh; ++k) {
          const cx c = Pp[(size_t)k * nz32 + z];
          const cx cm = Pp[(size_t)((nx32 - k) % nx32) * nz32 + z];
          /* A_k = (C_k + conj C_{N-k}) / 2, B_k = (C_k - conj C_{N-k}) / (2 i) */
          cx v;
          if (half == 0) v = C(0.5 * (c.re + cm.re), 0.5 * (c.im - cm.im));
          else v = C(0.5 * (c.im + cm.im), -0.5 * (c.re - cm.re));
          dst[(size_t)z * nxh + k] = v;
        }
      }
    }
  }
  /* x_to_y + ppdfftw_dft_z_forward: forward c2c along z, keep 1..nh, zero the kz Nyquist,
   * U(j - nh) = buf(j) for j = 2nh+2..nz32; rescale_data */
  for (int q = 0; q < 9; ++q) {
    cx *z = pw + np + (size_t)q * zplane;
    fft_batch(&T->pz, z, work, nxh, -1);
    cx *dst = out + (size_t)q * nz * nxh;
    for (int k = 0; k < nz; ++k) {
      if (k == nh) {
        memset(dst + (size_t)k * nxh, 0, sizeof(cx) * nxh);
        continue;
      }
      const cx *src = z + (size_t)(k < nh ? k : k + nh) * nxh;
      for (int x = 0; x < nxh; ++x) dst[(size_t)k * nxh + x] = cscale(rescale, src[x]);
    }
  }
  return vmax;
}

/* ------------------------------------------------------------------------------------------ */
/* Per-mode solves                                                                              */
/* ------------------------------------------------------------------------------------------ */
typedef struct {
  const kmm_oracle_params *p;
  const kmm_oracle_ops *o;
  int n, bw, ld;
} ctx;

/* a D0 - b D2 with the Dirichlet first/last rows (solve_g.f90:45-67) */
KO_INLINE void helmholtz_band(const ctx *c, double a, double b, double *A) {
  const int ld = c->ld, n = c->n, bw = c->bw;
  for (int j = 0; j < n; ++j)
    for (int r = 0; r < ld; ++r) A[j * ld + r] = a * c->o->d0[j * ld + r] - b * c->o->d2[j * ld + r];
  for (int col = 0; col < 2; ++col) {
    const int j = col == 0 ? 0 : n - 1;
    const double diag = a * c->o->d0[j * ld + bw] - b * c->o->d2[j * ld + bw];
    for (int r = 0; r < ld; ++r) A[j * ld + r] = 0.0;
    A[j * ld + bw] = diag;
  }
}

KO_INLINE double visc_of(double dt, double coef, double nu, double pr, int is_t) {
  const double v = dt * coef * nu;
  return is_t ? v / pr : v;
}

/* solve_g.f90:28-201 (is_t = 0) / solve_t.f90:28-201 (is_t = 1): u holds h on entry and the
 * new field on exit; store is updated; Dbuf receives the factored operator. */
KO_INLINE void solve_scalar_helmholtz(const ctx *c, cx *u, cx *store, double kx, double kz, int is_t, int s,
                                   double dt, double *Dbuf, cx *buf1, cx *buf2, cx *tmp) {
  const int n = c->n, bw = c->bw;
  const double nu = c->p->nu, pr = c->p->pr;
  const double k2 = kx * kx + kz * kz;
  const double beta = visc_of(dt, RK_BETA[s - 1], nu, pr, is_t);
  double dummy = 1.0 + beta * k2;
  helmholtz_band(c, dummy, beta, Dbuf);
  labs_lu(Dbuf, bw, n);
  if (s == 1) {
    const double alpha = visc_of(dt, RK_ALPHA[s - 1], nu, pr, is_t);
    const double gamma = dt * RK_GAMMA[s - 1];
    dummy = 1.0 - alpha * k2;
    for (int i = 0; i < n; ++i) buf1[i] = cadd(cscale(dummy, store[i]), cscale(gamma, u[i]));
    memcpy(tmp, store, sizeof(cx) * n);
    labs_bs(c->o->d0lu, bw, n, tmp);
    labs_mm(c->o->d2, bw, n, tmp, buf2);
    for (int i = 0; i < n; ++i) buf1[i] = cadd(buf1[i], cscale(alpha, buf2[i]));
  } else {
    const double gamma = dt * RK_GAMMA[s - 1];
    for (int i = 0; i < n; ++i) buf1[i] = cadd(store[i], cscale(gamma, u[i]));
  }
  buf1[0] = C(0.0, 0.0);
  buf1[n - 1] = C(0.0, 0.0);
  if (s != 3) {
    const double zeta = dt * RK_ZETA[s];
    for (int i = 0; i < n; ++i) store[i] = cscale(zeta, u[i]);
  }
  labs_bs(Dbuf, bw, n, buf1);
  labs_mm(c->o->d0, bw, n, buf1, u);
  labs_mm(c->o->d2, bw, n, buf1, buf2);
  if (s != 3) {
    const double alpha = visc_of(dt, RK_ALPHA[s], nu, pr, is_t);
    dummy = 1.0 - alpha * k2;
    for (int i = 0; i < n; ++i) store[i] = cadd(cadd(store[i], cscale(dummy, u[i])), cscale(alpha, buf2[i]));
  } else {
    memcpy(store, u, sizeof(cx) * n);
  }
}

/* solve_v_f.f90:38-375: hv (in) -> v, dv; store_phi updated.  vwall (2 values) or NULL. */
KO_INLINE void solve_v_f(const ctx *c, const cx *hv_in, cx *store_phi, const double *Dg, double kx, double kz, int s,
                      double dt, const cx *vwall, cx *v, cx *dv, double *Dv, cx *w) {
  const int n = c->n, bw = c->bw, ld = c->ld;
  const double nu = c->p->nu;
  const double k2 = kx * kx + kz * kz;
  cx *buf1 = w, *buf2 = w + n, *buf3 = w + 2 * n, *hv = w + 3 * n, *tmp = w + 4 * n, *hv2 = w + 5 * n;
  /* part 1 */
  if (s == 1) {
    const double alpha = dt * RK_ALPHA[s - 1] * nu, gamma = dt * RK_GAMMA[s - 1];
    const double dummy = 1.0 - alpha * k2;
    for (int i = 0; i < n; ++i) buf1[i] = cadd(cscale(dummy, store_phi[i]), cscale(gamma, hv_in[i]));
    memcpy(tmp, store_phi, sizeof(cx) * n);
    labs_bs(c->o->d0lu, bw, n, tmp);
    labs_mm(c->o->d2, bw, n, tmp, buf2);
    for (int i = 0; i < n; ++i) buf1[i] = cadd(buf1[i], cscale(alpha, buf2[i]));
  } else {
    const double gamma = dt * RK_GAMMA[s - 1];
    for (int i = 0; i < n; ++i) buf1[i] = cadd(store_phi[i], cscale(gamma, hv_in[i]));
  }
  buf1[0] = C(0.0, 0.0);
  buf1[n - 1] = C(0.0, 0.0);
  /* part 2 */
  if (s != 3) {
    const double zeta = dt * RK_ZETA[s];
    for (int i = 0; i < n; ++i) store_phi[i] = cscale(zeta, hv_in[i]);
  }
  /* part 3 */
  for (int i = 0; i < n; ++i) buf2[i] = C(0.0, 0.0);
  buf2[0] = C(Dg[bw], Dg[bw]);
  labs_bs(Dg, bw, n, buf1);
  labs_bs(Dg, bw, n, buf2);
  labs_mm(c->o->d0, bw, n, buf1, hv);
  labs_mm(c->o->d0, bw, n, buf2, buf3);
  labs_mm(c->o->d2, bw, n, buf1, dv);
  /* part 4 */
  if (s != 3) {
    const double alpha = dt * nu * RK_ALPHA[s];
    const double dummy = 1.0 - alpha * k2;
    for (int i = 0; i < n; ++i) store_phi[i] = cadd(cadd(store_phi[i], cscale(dummy, hv[i])), cscale(alpha, dv[i]));
  } else {
    memcpy(store_phi, hv, sizeof(cx) * n);
  }
  /* part 5: (D2 - k2 D0) with D0 Dirichlet rows */
  for (int j = 0; j < n; ++j)
    for (int r = 0; r < ld; ++r) Dv[j * ld + r] = (-k2) * c->o->d0[j * ld + r] + c->o->d2[j * ld + r];
  for (int col = 0; col < 2; ++col) {
    const int j = col == 0 ? 0 : n - 1;
    for (int r = 0; r < ld; ++r) Dv[j * ld + r] = 0.0;
    Dv[j * ld + bw] = c->o->d0[j * ld + bw];
  }
  labs_lu(Dv, bw, n);
  /* part 6 */
  if (vwall) {
    hv[0] = vwall[0];
    hv[n - 1] = vwall[1];
  } else {
    hv[0] = C(0.0, 0.0);
    hv[n - 1] = C(0.0, 0.0);
  }
  labs_bs(Dv, bw, n, hv);
  memcpy(buf1, buf3, sizeof(cx) * n);
  buf1[0] = C(0.0, 0.0);
  buf1[n - 1] = C(0.0, 0.0);
  labs_bs(Dv, bw, n, buf1);
  labs_mm(c->o->d0, bw, n, hv, v);
  labs_mm(c->o->d1, bw, n, hv, dv);
  labs_mm(c->o->d1, bw, n, buf1, hv2);
  const cx den = csub(cmul(hv2[0], hv2[0]), cmul(hv2[n - 1], hv2[n - 1]));
  const cx C1 = cdiv(csub(cmul(hv2[n - 1], dv[n - 1]), cmul(hv2[0], dv[0])), den);
  const cx C2 = cdiv(csub(cmul(hv2[0], dv[n - 1]), cmul(hv2[n - 1], dv[0])), den);
  for (int i = 0; i < n; ++i) tmp[i] = csub(cadd(dv[i], cmul(C1, hv2[i])), cmul(C2, hv2[n - 1 - i]));
  memcpy(dv, tmp, sizeof(cx) * n);
  /* part 7 */
  labs_mm(c->o->d2, bw, n, buf2, hv);
  if (s != 3) {
    const double alpha = dt * nu * RK_ALPHA[s];
    const double dummy = 1.0 - alpha * k2;
    for (int i = 0; i < n; ++i) {
      cx a = store_phi[i];
      a = cadd(a, cscale(dummy, cmul(C1, buf3[i])));
      a = cadd(a, cscale(dummy, cmul(C2, buf3[n - 1 - i])));
      a = cadd(a, cscale(alpha, cmul(C1, hv[i])));
      a = cadd(a, cscale(alpha, cmul(C2, hv[n - 1 - i])));
      store_phi[i] = a;
    }
  } else {
    for (int i = 0; i < n; ++i) store_phi[i] = cadd(cadd(store_phi[i], cmul(C1, buf3[i])), cmul(C2, buf3[n - 1 - i]));
  }
  /* part 8 */
  labs_mm(c->o->d0, bw, n, buf1, hv);
  for (int i = 0; i < n; ++i) v[i] = cadd(cadd(v[i], cmul(C1, hv[i])), cmul(C2, hv[n - 1 - i]));
}

/* hvhg.f90:28-163 on lines u1..u5, u7..u9 (slots 0-4, 6-8): returns hg (in u1), hv (in u5),
 * ht (in u7). */
KO_INLINE void hvhg(const ctx *c, cx *u1, cx *u2, cx *u3, cx *u4, cx *u5, cx *u7, cx *u8, cx *u9, double kx, double kz,
                 cx *t1, cx *t2) {
  const int n = c->n, bw = c->bw;
  const double kz2 = kz * kz, kx2 = kx * kx, kxkz = kx * kz;
  const double ikx3 = kx * kx * kx, ikxkz2 = kx * (kz * kz), ikx2kz = (kx * kx) * kz, ikz3 = kz * kz * kz;
  for (int i = 0; i < n; ++i) {
    const cx d = u1[i];
    u1[i] = cadd(cscale(kxkz, csub(u1[i], u3[i])), cscale(kz2 - kx2, u5[i]));
    u3[i] = csub(csub(cscale(-kx2, d), cscale(2.0 * kxkz, u5[i])), cscale(kz2, u3[i]));
  }
  labs_bs(c->o->d0lu, bw, n, u3);
  labs_mm(c->o->d1, bw, n, u3, u5);
  for (int i = 0; i < n; ++i) u5[i] = cadd(cadd(u5[i], cimul(ikx3 + ikxkz2, u2[i])), cimul(ikx2kz + ikz3, u4[i]));
  for (int i = 0; i < n; ++i) {
    const cx a = csub(cimul(kx, u4[i]), cimul(kz, u2[i]));
    const cx b = cadd(cimul(kz, u4[i]), cimul(kx, u2[i]));
    u3[i] = a;
    u4[i] = b;
  }
  labs_bs(c->o->d0lu, bw, n, u3);
  labs_mm(c->o->d1, bw, n, u3, u2);
  labs_bs(c->o->d0lu, bw, n, u4);
  labs_mm(c->o->d2, bw, n, u4, u3);
  for (int i = 0; i < n; ++i) {
    u5[i] = cadd(u5[i], u3[i]);
    u1[i] = cadd(u1[i], u2[i]);
    u7[i] = cadd(cimul(kx, u7[i]), cimul(kz, u9[i]));
  }
  labs_bs(c->o->d0lu, bw, n, u8);
  labs_mm(c->o->d1, bw, n, u8, u9);
  for (int i = 0; i < n; ++i) u7[i] = C(-(u7[i].re + u9[i].re), -(u7[i].im + u9[i].im));
  (void)t1;
  (void)t2;
}

/* wave00.f90:41-685 for one mean line (U: line 0, W: line 1, Theta: line 2). */
static void mean_line(const ctx *c, int line, cx *store, const cx *flux, int s, double dt, cx *prof, double *phi_out,
                      double *wall_out, double *A, cx *w) {
  const int n = c->n, bw = c->bw, ld = c->ld;
  const kmm_oracle_params *p = c->p;
  const double visc = line == 2 ? p->nu / p->pr : p->nu;
  const double gal = line == 0 ? p->u_gal : 0.0;
  const double bulk = line == 0 ? p->bulk_u : line == 1 ? p->bulk_w : p->bulk_t;
  cx *buf1 = w, *cc = w + n, *b = w + 2 * n, *d = w + 3 * n, *st = w + 4 * n;
  /* lhs: D0 - beta D2 with Dirichlet rows */
  const double beta = dt * RK_BETA[s - 1] * visc;
  for (int j = 0; j < n; ++j)
    for (int r = 0; r < ld; ++r) A[j * ld + r] = c->o->d0[j * ld + r] - beta * c->o->d2[j * ld + r];
  for (int col = 0; col < 2; ++col) {
    const int j = col == 0 ? 0 : n - 1;
    for (int r = 0; r < ld; ++r) A[j * ld + r] = 0.0;
    A[j * ld + bw] = c->o->d0[j * ld + bw] - beta * c->o->d2[j * ld + bw];
  }
  labs_lu(A, bw, n);
  for (int i = 0; i < n; ++i) buf1[i] = C(0.0, 0.0);
  memcpy(b, flux, sizeof(cx) * n);
  labs_bs(c->o->d0lu, bw, n, b);
  labs_mm(c->o->d1, bw, n, b, d);
  const double gamma = dt * RK_GAMMA[s - 1];
  if (s == 1) {
    memcpy(cc, store, sizeof(cx) * n);
    labs_bs(c->o->d0lu, bw, n, cc);
    labs_mm(c->o->d2, bw, n, cc, buf1);
    const double alpha = dt * RK_ALPHA[s - 1] * visc;
    for (int i = 1; i < n; ++i) buf1[i] = csub(cadd(store[i], cscale(alpha, buf1[i])), cscale(gamma, d[i]));
  } else {
    for (int i = 1; i < n; ++i) buf1[i] = csub(store[i], cscale(gamma, d[i]));
  }
  buf1[0] = C(0.0, 0.0);
  for (int i = 1; i < n - 1; ++i) buf1[i] = C(buf1[i].re + gal, 1.0);
  buf1[n - 1] = C(0.0, 0.0);
  labs_bs(A, bw, n, buf1);
  cx integral = C(0.0, 0.0);
  for (int i = 0; i < n; ++i) integral = cadd(integral, cscale(c->o->integ[i], buf1[i]));
  double phi = (bulk - 0.5 * integral.re) / (0.5 * integral.im); /* calculate_phi, wave00.f90:704-714 */
  if (line == 1) phi = 0.0;                                       /* wave00.f90:396 */
  for (int i = 0; i < n; ++i) buf1[i] = C(buf1[i].re + phi * buf1[i].im, 0.0);
  if (wall_out && s == 3) {
    const double *D1 = c->o->d1;
    *wall_out = D1[0 * ld + bw] * buf1[0].re + D1[0 * ld + bw + 1] * buf1[1].re -
                D1[(n - 1) * ld + bw - 1] * buf1[n - 2].re - D1[(n - 1) * ld + bw] * buf1[n - 1].re;
  }
  labs_mm(c->o->d0, bw, n, buf1, prof);
  if (line == 0)
    for (int i = 0; i < n; ++i) prof[i].re -= p->u_gal;
  if (s != 3) {
    labs_mm(c->o->d2, bw, n, buf1, st);
    const double alpha = dt * RK_ALPHA[s] * visc, zeta = dt * RK_ZETA[s];
    for (int i = 0; i < n; ++i) store[i] = csub(cadd(cscale(alpha, st[i]), prof[i]), cscale(zeta, d[i]));
  } else {
    memcpy(store, prof, sizeof(cx) * n);
  }
  *phi_out = phi;
}

/* The solves of one (kx, kz) mode other than (0,0) (wavespace.f90:43-109): hvhg, solve_g, the
 * opposition-control wall values, solve_v_f, solve_u_w, solve_t. */
typedef struct {
  cx *U, *RK;
  const cx *P9;
  size_t plane, field;
  int s;
  double dt;
} mode_io;

KO_INLINE void solve_mode(const ctx *c, const mode_io *io, int64_t m, cx *L, double *Dg, double *Dt, double *Dv) {
  const kmm_oracle_params *p = c->p;
  const kmm_oracle_ops *o = c->o;
  const int nxh = p->nx / 2, nz = p->nz, ny = p->ny, s = io->s;
  const double dt = io->dt;
  const int kzi = (int)(m / nxh), kxi = (int)(m % nxh);
  const int kzint = kzi <= nz / 2 ? kzi : kzi - nz;
  const double kx = kxi * (1.0 / p->lmfx), kz = kzint * (1.0 / p->lmfz);
  cx *u[9];
  for (int q = 0; q < 9; ++q) {
    u[q] = L + (size_t)q * ny;
    for (int y = 0; y < ny; ++y) u[q][y] = io->P9[(size_t)q * io->field + (size_t)y * io->plane + m];
  }
  cx *sg = io->RK + 0 * io->field + (size_t)m * ny, *sp = io->RK + 1 * io->field + (size_t)m * ny, *st = io->RK + 2 * io->field + (size_t)m * ny;
  cx *b1 = L + 9 * ny, *b2 = L + 10 * ny, *tmp = L + 11 * ny, *v = L + 12 * ny, *dv = L + 13 * ny, *w6 = L + 14 * ny;
  /* product lines: u[0]=f1 u[1]=f2 u[2]=f3 u[3]=f4 u[4]=f5 u[5]=f7 u[6]=f8 u[7]=f9 u[8]=vold */
  hvhg(c, u[0], u[1], u[2], u[3], u[4], u[5], u[6], u[7], kx, kz, b1, b2);
  cx *g = u[0], *hv = u[4], *th = u[5];
  solve_scalar_helmholtz(c, g, sg, kx, kz, 0, s, dt, Dg, b1, b2, tmp);
  cx vw[2];
  const cx *vwall = NULL;
  if (p->control_amp != 0.0) {
    const double gm = o->gains ? o->gains[m] : 1.0;
    cx lo = C(0.0, 0.0), hi = C(0.0, 0.0);
    for (int y = 0; y < ny; ++y) {
      lo = cadd(lo, cscale(o->wlo[y], u[8][y]));
      hi = cadd(hi, cscale(o->whi[y], u[8][y]));
    }
    vw[0] = cscale(p->control_amp * gm, lo);
    vw[1] = cscale(p->control_amp * gm, hi);
    vwall = vw;
  }
  solve_v_f(c, hv, sp, Dg, kx, kz, s, dt, vwall, v, dv, Dv, w6);
  /* solve_u_w.f90:18-42 */
  const double k2 = kx * kx + kz * kz;
  const double kxx = kx / k2, kzz = kz / k2;
  cx *Uu = io->U + 0 * io->field + (size_t)m * ny, *Uv = io->U + 1 * io->field + (size_t)m * ny;
  cx *Uw = io->U + 2 * io->field + (size_t)m * ny, *Ut = io->U + 6 * io->field + (size_t)m * ny;
  for (int y = 0; y < ny; ++y) {
    const cx dxg = cimul(kxx, g[y]), dzg = cimul(kzz, g[y]);
    const cx dxf = cimul(kxx, dv[y]), dzf = cimul(kzz, dv[y]);
    Uu[y] = csub(dxf, dzg);
    Uw[y] = cadd(dxg, dzf);
    Uv[y] = v[y];
  }
  solve_scalar_helmholtz(c, th, st, kx, kz, 1, s, dt, Dt, b1, b2, tmp);
  memcpy(Ut, th, sizeof(cx) * ny);
}

#define SOLVE_MODE_BW(BW)                                                                        \
  static void solve_mode_bw##BW(const ctx *c0, const mode_io *io, int64_t m, cx *L, double *D) { \
    ctx c = *c0;                                                                                 \
    c.bw = BW;                                                                                   \
    c.ld = 2 * BW + 1;                                                                           \
    solve_mode(&c, io, m, L, D, D + c.ld * c.n, D + 2 * c.ld * c.n);                             \
  }
SOLVE_MODE_BW(2)
SOLVE_MODE_BW(3)
SOLVE_MODE_BW(4)
SOLVE_MODE_BW(5)
SOLVE_MODE_BW(6)
SOLVE_MODE_BW(7)
#undef SOLVE_MODE_BW

static void solve_mode_any(const ctx *c, const mode_io *io, int64_t m, cx *L, double *D) {
  solve_mode(c, io, m, L, D, D + c->ld * c->n, D + 2 * c->ld * c->n);
}

typedef void (*solve_mode_t)(const ctx *, const mode_io *, int64_t, cx *, double *);

static solve_mode_t solve_mode_for(int bw) {
  switch (bw) {
    case 2: return solve_mode_bw2;
    case 3: return solve_mode_bw3;
    case 4: return solve_mode_bw4;
    case 5: return solve_mode_bw5;
    case 6: return solve_mode_bw6;
    case 7: return solve_mode_bw7;
    default: return solve_mode_any;
  }
}

/* ------------------------------------------------------------------------------------------ */
/* Substep                                                                                      */
/* ------------------------------------------------------------------------------------------ */
typedef struct {
  tplans T;
  cx *S4;  /* [4][ny][nz][nxh] state planes */
  cx *P9;  /* [9][ny][nz][nxh] product planes */
  int nthreads;
  cx **zb, **xb, **xb2, **pw, **work;
} engine;

static int engine_init(engine *E, const kmm_oracle_params *p) {
  memset(E, 0, sizeof(*E));
  const int nxh = p->nx / 2, nz = p->nz, ny = p->ny;
  E->T.nx = p->nx;
  E->T.nz = nz;
  E->T.nxh = nxh;
  E->T.nx32 = p->nx * 3 / 2;
  E->T.nz32 = nz * 3 / 2;
  E->T.nh = nz / 2;
  if (plan_init(&E->T.pz, E->T.nz32) || plan_init(&E->T.px, E->T.nx32)) return -1;
  const size_t plane = (size_t)nz * nxh;
  E->S4 = (cx *)malloc(sizeof(cx) * 4 * plane * ny);
  E->P9 = (cx *)malloc(sizeof(cx) * 9 * plane * ny);
#ifdef _OPENMP
  E->nthreads = p->nthreads > 0 ? p->nthreads : omp_get_max_threads();
#else
  E->nthreads = 1;
#endif
  const int nt = E->nthreads;
  E->zb = (cx **)calloc(nt, sizeof(cx *));
  E->xb = (cx **)calloc(nt, sizeof(cx *));
  E->xb2 = (cx **)calloc(nt, sizeof(cx *));
  E->pw = (cx **)calloc(nt, sizeof(cx *));
  E->work = (cx **)calloc(nt, sizeof(cx *));
  const size_t zplane = (size_t)E->T.nz32 * nxh, xplane = (size_t)E->T.nx32 * E->T.nz32;
  for (int t = 0; t < nt; ++t) {
    E->zb[t] = (cx *)malloc(sizeof(cx) * 4 * zplane);
    E->xb[t] = (cx *)malloc(sizeof(cx) * xplane);
    E->xb2[t] = (cx *)malloc(sizeof(cx) * xplane);
    E->pw[t] = (cx *)malloc(sizeof(cx) * (xplane + 9 * zplane));
    E->work[t] = (cx *)malloc(sizeof(cx) * (xplane > zplane ? xplane : zplane));
  }
  return 0;
}

static void engine_free(engine *E) {
  for (int t = 0; t < E->nthreads; ++t) {
    free(E->zb[t]);
    free(E->xb[t]);
    free(E->xb2[t]);
    free(E->pw[t]);
    free(E->work[t]);
  }
  free(E->zb);
  free(E->xb);
  free(E->xb2);
  free(E->pw);
  free(E->work);
  free(E->S4);
  free(E->P9);
  plan_free(&E->T.pz);
  plan_free(&E->T.px);
}

static int thread_id(void) {
#ifdef _OPENMP
  return omp_get_thread_num();
#else
  return 0;
#endif
}

static int substep(engine *E, const kmm_oracle_params *p, const kmm_oracle_ops *o, cx *U, cx *RK, int s,
                   double *dt_io, kmm_oracle_scalars *sc) {
  const int nxh = p->nx / 2, nz = p->nz, ny = p->ny, bw = p->bw;
  const int64_t nmodes = (int64_t)nxh * nz;
  const size_t plane = (size_t)nmodes, field = (size_t)nmodes * ny;
  const int state_slots[4] = {0, 1, 2, 6};
  const int nt = E->nthreads;
  const double rescale = 1.0 / ((double)E->T.nx32 * E->T.nz32);
  /* reference layout [f][mode][y] -> planes [f][y][mode] */
#pragma omp parallel for num_threads(nt) schedule(static)
  for (int64_t m = 0; m < nmodes; ++m)
    for (int f = 0; f < 4; ++f) {
      const cx *src = U + (size_t)state_slots[f] * field + (size_t)m * ny;
      for (int y = 0; y < ny; ++y) E->S4[(size_t)f * field + (size_t)y * plane + m] = src[y];
    }
  double vmax = 0.0;
#pragma omp parallel for num_threads(nt) schedule(dynamic, 1) reduction(max : vmax)
  for (int y = 0; y < ny; ++y) {
    const int t = thread_id();
    cx *inp = (cx *)malloc(sizeof(cx) * 4 * plane);
    cx *outp = (cx *)malloc(sizeof(cx) * 9 * plane);
    for (int f = 0; f < 4; ++f) memcpy(inp + f * plane, E->S4 + (size_t)f * field + (size_t)y * plane, sizeof(cx) * plane);
    const double v = plane_step(&E->T, inp, outp, p->dxr, o->dyr[y], p->dzr, s == 1, rescale, E->zb[t], E->xb[t],
                                E->xb2[t], E->pw[t], E->work[t]);
    for (int q = 0; q < 9; ++q) memcpy(E->P9 + (size_t)q * field + (size_t)y * plane, outp + q * plane, sizeof(cx) * plane);
    free(inp);
    free(outp);
    if (v > vmax) vmax = v;
  }
  double dt = *dt_io;
  if (s == 1) {
    sc->velmax = vmax;
    if (!p->fixed_dt) dt = p->dt_factor * dt + (1.0 - p->dt_factor) * p->cflx / vmax; /* dft_x_realspace.f90:490-493 */
    if (!(dt > 1e-14 && dt <= 1e5)) return 3;                                         /* :494-497 */
  }
  const ctx c = {p, o, ny, bw, 2 * bw + 1};
  const int ld = 2 * bw + 1;
  const mode_io io = {U, RK, E->P9, plane, field, s, dt};
  const solve_mode_t solve_mode_fn = solve_mode_for(bw);
  /* per (kx, kz) mode, (0,0) excluded: wavespace.f90:43-109 */
#pragma omp parallel num_threads(nt)
  {
    cx *L = (cx *)malloc(sizeof(cx) * (size_t)ny * 24);
    double *Dg = (double *)malloc(sizeof(double) * ld * ny * 3);
#pragma omp for schedule(dynamic, 16)
    for (int64_t m = 1; m < nmodes; ++m) {
      solve_mode_fn(&c, &io, m, L, Dg);
    }
    free(L);
    free(Dg);
  }
  /* (0,0): wave00 */
  {
    cx *L = (cx *)malloc(sizeof(cx) * (size_t)ny * 10);
    double *A = (double *)malloc(sizeof(double) * ld * ny);
    cx *flux = L, *prof = L + ny, *w = L + 2 * ny;
    const int pslot[3] = {1, 3, 6}; /* uv, vw, v theta among the nine product planes */
    const int uslot[3] = {0, 2, 6};
    double phi[3] = {0, 0, 0}, wall[3] = {0, 0, 0};
    for (int line = 0; line < 3; ++line) {
      for (int y = 0; y < ny; ++y) flux[y] = E->P9[(size_t)pslot[line] * field + (size_t)y * plane + 0];
      cx *store = RK + (size_t)line * field;
      mean_line(&c, line, store, flux, s, dt, prof, &phi[line], &wall[line], A, w);
      memcpy(U + (size_t)uslot[line] * field, prof, sizeof(cx) * ny);
    }
    for (int y = 0; y < ny; ++y) U[1 * field + y] = C(0.0, 0.0);
    sc->phi_dpdx[s - 1] = phi[0];
    sc->phi_dtdx[s - 1] = phi[2];
    if (s == 3) {
      sc->wall_shear_stress = 0.5 * p->nu * wall[0];
      sc->wall_theta_stress = 0.5 * p->nu / p->pr * wall[2];
    }
    free(L);
    free(A);
  }
  sc->dt = dt;
  *dt_io = dt;
  return 0;
}

/* nsteps RK3 steps (main.f90:134-193 without I/O).  U (10 fields) and RK are updated in place;
 * fields 1, 2, 3, 7 hold u, v, w, theta on return, the other slots are scratch.  *dt is the
 * time step in and the last one out.  scalars (may be NULL) receives one record per step.
 * Returns 0, or 3 when dt leaves (1e-14, 1e5] (the reference's abort). */
int kmm_oracle_rk3(const kmm_oracle_params *p, const kmm_oracle_ops *o, double *U, double *RK, double *dt,
                   int nsteps, kmm_oracle_scalars *scalars) {
  engine E;
  if (engine_init(&E, p)) return 1;
  int rc = 0;
  for (int n = 0; n < nsteps && !rc; ++n) {
    kmm_oracle_scalars sc;
    memset(&sc, 0, sizeof(sc));
    for (int s = 1; s <= 3 && !rc; ++s) rc = substep(&E, p, o, (cx *)U, (cx *)RK, s, dt, &sc);
    sc.phi_dpdx[3] = (sc.phi_dpdx[0] + sc.phi_dpdx[1] + sc.phi_dpdx[2]) / *dt; /* main.f90:147-148 */
    sc.phi_dtdx[3] = (sc.phi_dtdx[0] + sc.phi_dtdx[1] + sc.phi_dtdx[2]) / *dt;
    if (scalars) scalars[n] = sc;
  }
  engine_free(&E);
  return rc;
}

/* One substep (time_march) for the step-by-step checks. */
int kmm_oracle_substep(const kmm_oracle_params *p, const kmm_oracle_ops *o, double *U, double *RK, double *dt,
                       int s, kmm_oracle_scalars *sc) {
  engine E;
  if (s < 1 || s > 3 || engine_init(&E, p)) return 1;
  kmm_oracle_scalars tmp;
  memset(&tmp, 0, sizeof(tmp));
  const int rc = substep(&E, p, o, (cx *)U, (cx *)RK, s, dt, sc ? sc : &tmp);
  engine_free(&E);
  return rc;
}

/* set_initial_data_uvw (initial_step.f90:139-179): the RK stores from u, v, w, theta.  For the
 * (0,0) mode the stores are U, W and Theta; otherwise g = i kz u - i kx w, phi = D2 D0^{-1} v -
 * k^2 v and the theta store = theta. */
int kmm_oracle_set_initial_data_uvw(const kmm_oracle_params *p, const kmm_oracle_ops *o, const double *Ud,
                                    double *RKd) {
  const int nxh = p->nx / 2, nz = p->nz, ny = p->ny, bw = p->bw;
  const int64_t nmodes = (int64_t)nxh * nz;
  const size_t field = (size_t)nmodes * ny;
  const cx *U = (const cx *)Ud;
  cx *RK = (cx *)RKd;
#ifdef _OPENMP
  const int nt = p->nthreads > 0 ? p->nthreads : omp_get_max_threads();
#endif
#pragma omp parallel num_threads(nt)
  {
    cx *c = (cx *)malloc(sizeof(cx) * 2 * (size_t)ny), *d2 = c + ny;
#pragma omp for schedule(static)
    for (int64_t m = 0; m < nmodes; ++m) {
      const int kzi = (int)(m / nxh), kxi = (int)(m % nxh);
      const int kzint = kzi <= nz / 2 ? kzi : kzi - nz;
      const cx *u = U + (size_t)m * ny, *v = U + field + (size_t)m * ny, *w = U + 2 * field + (size_t)m * ny;
      const cx *t = U + 6 * field + (size_t)m * ny;
      cx *r0 = RK + (size_t)m * ny, *r1 = RK + field + (size_t)m * ny, *r2 = RK + 2 * field + (size_t)m * ny;
      if (m == 0) {
        memcpy(r0, u, sizeof(cx) * ny);
        memcpy(r1, w, sizeof(cx) * ny);
        memcpy(r2, t, sizeof(cx) * ny);
        continue;
      }
      const double kxr = kxi * (1.0 / p->lmfx), kzr = kzint * (1.0 / p->lmfz);
      memcpy(c, v, sizeof(cx) * ny);
      labs_bs(o->d0lu, bw, ny, c);
      labs_mm(o->d2, bw, ny, c, d2);
      const double k2 = kxr * kxr + kzr * kzr;
      for (int y = 0; y < ny; ++y) {
        r1[y] = csub(d2[y], cscale(k2, v[y]));
        r0[y] = csub(cimul(kzr, u[y]), cimul(kxr, w[y]));
        r2[y] = t[y];
      }
    }
    free(c);
  }
  return 0;
}

int kmm_oracle_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}
