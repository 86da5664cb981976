/* sfnl_cpu_fft.c -- TEST INFRASTRUCTURE: the timed CPU baseline of the GPU library.
 *
 * A C restatement of the reference's FFTW path of the dealiased products
 * (SOURCES/POST_PROCESSING/fft_parallel.F90: FFT_PAR_CROSS_PROD_DCL :147-328,
 * FFT_PAR_DOT_PROD_DCL :330-500, FFT_PAR_PROD_DCL :502-665) with all modes of
 * a point on one process, as the reference has them after its first
 * MPI_ALLTOALL (:217):
 *   pack c_0 = a_0, c_n = (a_n - i b_n)/2, zero-padded (:223-241),
 *   c2r of length N, unnormalised, sign +1 (:254-267),
 *   the pointwise product (:270-274, :449-451, :617),
 *   r2c, sign -1 (:278-284), scale 1/N (:288),
 *   a_n = 2 Re, b_n = -2 Im (n >= 1), a_0 = Re, b_0 = 0, truncated to m (:295-299).
 * The real transforms are O(N log N): a real sequence of even length N is
 * transformed through a complex FFT of length N/2, the way FFTW's r2c/c2r
 * treat even lengths; an odd N runs as a complex FFT of length N.  The complex
 * FFT is a Stockham autosort (radices 4, 2, 3, 5 and a generic odd radix,
 * per-pass twiddle tables) applied to 8 points at once: the data of a block of
 * 8 points is held point-fastest, which is the layout of one 64-byte line of a
 * coefficient row, and every butterfly runs as 8-wide vector arithmetic.
 * Blocks are spread over POSIX threads standing for the reference's ranks (no
 * all-to-all cost), each thread a contiguous range of blocks.
 *
 * It is never linked into the product: only bench.py's CPU-baseline legs and
 * the tests load it.
 */
#include <math.h>
#include <pthread.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <unistd.h>

#define VB 8 /* points per block = vector width of the transforms */

typedef struct {
  double re[VB], im[VB];
} vcpx; /* 8 complex numbers, one per point of the block */

/* One Stockham pass: radix R, Ns = product of the radices before it. */
typedef struct {
  int R, Ns;
  double *wr, *wi; /* [Ns][R]: exp(-2 pi i (j mod Ns) r / (Ns R)) */
} pass_t;

typedef struct {
  int n, np_;
  pass_t pass[32];
  double *rr, *ri; /* generic radix: exp(-2 pi i t / R), t < R, per pass (shared when R repeats) */
} cplan;

static int cplan_init(cplan *p, int n) {
  int fac[32], nf = 0, r = n;
  while (r % 4 == 0) { fac[nf++] = 4; r /= 4; }
  while (r % 2 == 0) { fac[nf++] = 2; r /= 2; }
  for (int q = 3; r > 1;) {
    if (r % q == 0) {
      fac[nf++] = q;
      r /= q;
    } else {
      q += 2;
      if (q * q > r) q = r;
    }
  }
  p->n = n;
  p->np_ = nf;
  const long double pi = acosl(-1.0L);
  int Ns = 1;
  for (int f = 0; f < nf; ++f) {
    pass_t *ps = &p->pass[f];
    ps->R = fac[f];
    ps->Ns = Ns;
    ps->wr = (double *)malloc(sizeof(double) * (size_t)Ns * fac[f]);
    ps->wi = (double *)malloc(sizeof(double) * (size_t)Ns * fac[f]);
    if (!ps->wr || !ps->wi) return -1;
    for (int j = 0; j < Ns; ++j)
      for (int t = 0; t < fac[f]; ++t) {
        const long double x = -2.0L * pi * (long double)(j * t) / (long double)(Ns * fac[f]);
        ps->wr[j * fac[f] + t] = (double)cosl(x);
        ps->wi[j * fac[f] + t] = (double)sinl(x);
      }
    Ns *= fac[f];
  }
  return 0;
}
static void cplan_free(cplan *p) {
  for (int f = 0; f < p->np_; ++f) {
    free(p->pass[f].wr);
    free(p->pass[f].wi);
  }
}

/* Small DFTs in place on v[0..R) (8 points each), sign -1 (inv = 0) or +1 (inv = 1). */
static inline void dft2(vcpx *v) {
  for (int b = 0; b < VB; ++b) {
    const double ar = v[0].re[b], ai = v[0].im[b], br = v[1].re[b], bi = v[1].im[b];
    v[0].re[b] = ar + br;
    v[0].im[b] = ai + bi;
    v[1].re[b] = ar - br;
    v[1].im[b] = ai - bi;
  }
}
static inline void dft4(vcpx *v, int inv) {
  const double sg = inv ? 1.0 : -1.0; /* X1 = (x0 - x2) + sg i (x1 - x3) */
  for (int b = 0; b < VB; ++b) {
    const double s02r = v[0].re[b] + v[2].re[b], s02i = v[0].im[b] + v[2].im[b];
    const double d02r = v[0].re[b] - v[2].re[b], d02i = v[0].im[b] - v[2].im[b];
    const double s13r = v[1].re[b] + v[3].re[b], s13i = v[1].im[b] + v[3].im[b];
    const double d13r = v[1].re[b] - v[3].re[b], d13i = v[1].im[b] - v[3].im[b];
    v[0].re[b] = s02r + s13r;
    v[0].im[b] = s02i + s13i;
    v[2].re[b] = s02r - s13r;
    v[2].im[b] = s02i - s13i;
    v[1].re[b] = d02r - sg * d13i;
    v[1].im[b] = d02i + sg * d13r;
    v[3].re[b] = d02r + sg * d13i;
    v[3].im[b] = d02i - sg * d13r;
  }
}
static inline void dft3(vcpx *v, int inv) {
  const double c = -0.5, s = (inv ? 1.0 : -1.0) * 0.86602540378443864676; /* sin(2 pi / 3) */
  for (int b = 0; b < VB; ++b) {
    const double tr = v[1].re[b] + v[2].re[b], ti = v[1].im[b] + v[2].im[b];
    const double ur = v[1].re[b] - v[2].re[b], ui = v[1].im[b] - v[2].im[b];
    const double mr = v[0].re[b] + c * tr, mi = v[0].im[b] + c * ti;
    v[0].re[b] += tr;
    v[0].im[b] += ti;
    v[1].re[b] = mr - s * ui;
    v[1].im[b] = mi + s * ur;
    v[2].re[b] = mr + s * ui;
    v[2].im[b] = mi - s * ur;
  }
}
static void dftR(vcpx *v, int R, int inv, vcpx *tmp) {
  const long double pi = acosl(-1.0L);
  for (int q = 0; q < R; ++q)
    for (int b = 0; b < VB; ++b) tmp[q].re[b] = tmp[q].im[b] = 0.0;
  for (int t = 0; t < R; ++t)
    for (int q = 0; q < R; ++q) {
      const long double x = (inv ? 2.0L : -2.0L) * pi * (long double)((t * q) % R) / (long double)R;
      const double wr = (double)cosl(x), wi = (double)sinl(x);
      for (int b = 0; b < VB; ++b) {
        tmp[q].re[b] += v[t].re[b] * wr - v[t].im[b] * wi;
        tmp[q].im[b] += v[t].re[b] * wi + v[t].im[b] * wr;
      }
    }
  for (int q = 0; q < R; ++q) v[q] = tmp[q];
}

/* Complex FFT of 8 sequences at once: x[0..n) -> y (both [n] of vcpx); x is overwritten. */
__attribute__((target_clones("arch=x86-64-v3", "default")))
static void vfft(const cplan *p, vcpx *x, vcpx *y, int inv, vcpx *scratch) {
  const int n = p->n;
  vcpx *src = x, *dst = y;
  vcpx v[64];
  for (int f = 0; f < p->np_; ++f) {
    const pass_t *ps = &p->pass[f];
    const int R = ps->R, Ns = ps->Ns, nr = n / R;
    vcpx *vv = R <= 64 ? v : scratch;
    vcpx *tmp = scratch + (R <= 64 ? 0 : R);
    for (int j = 0; j < nr; ++j) {
      const int jm = j % Ns;
      const double *wr = ps->wr + (size_t)jm * R, *wi = ps->wi + (size_t)jm * R;
      for (int r = 0; r < R; ++r) {
        const vcpx *a = &src[j + r * nr];
        const double c = wr[r], sn = inv ? -wi[r] : wi[r];
        for (int b = 0; b < VB; ++b) {
          vv[r].re[b] = a->re[b] * c - a->im[b] * sn;
          vv[r].im[b] = a->re[b] * sn + a->im[b] * c;
        }
      }
      if (R == 4)
        dft4(vv, inv);
      else if (R == 2)
        dft2(vv);
      else if (R == 3)
        dft3(vv, inv);
      else
        dftR(vv, R, inv, tmp);
      const int idxD = (j / Ns) * Ns * R + jm;
      for (int r = 0; r < R; ++r) dst[idxD + r * Ns] = vv[r];
    }
    vcpx *t = src;
    src = dst;
    dst = t;
  }
  if (src != y) memcpy(y, src, sizeof(vcpx) * (size_t)n);
}

/* Real transforms of length N (8 sequences at once) through a complex FFT of length N/2 (even N)
 * or N (odd N). */
typedef struct {
  int N, even, h;
  cplan c;
  double *wr, *wi; /* exp(-2 pi i k / N), k <= N/2 */
} rplan;

static int rplan_init(rplan *r, int N) {
  r->N = N;
  r->even = (N % 2 == 0);
  r->h = r->even ? N / 2 : N;
  if (cplan_init(&r->c, r->h)) return -1;
  r->wr = (double *)malloc(sizeof(double) * (size_t)(N / 2 + 1));
  r->wi = (double *)malloc(sizeof(double) * (size_t)(N / 2 + 1));
  if (!r->wr || !r->wi) return -1;
  const long double pi = acosl(-1.0L);
  for (int k = 0; k <= N / 2; ++k) {
    const long double x = -2.0L * pi * (long double)k / (long double)N;
    r->wr[k] = (double)cosl(x);
    r->wi[k] = (double)sinl(x);
  }
  return 0;
}
static void rplan_free(rplan *r) {
  cplan_free(&r->c);
  free(r->wr);
  free(r->wi);
}

/* x[j][b] = sum_{n<N} X_n e^{+2 pi i n j / N}, X Hermitian given by X[0..N/2];
 * work: 2h + scratch vcpx. */
__attribute__((target_clones("arch=x86-64-v3", "default")))
static void c2r(const rplan *r, const vcpx *X, double *x, vcpx *work) {
  const int N = r->N, h = r->h;
  vcpx *Z = work, *z = work + h, *scr = work + 2 * h;
  if (r->even) {
    for (int k = 0; k < h; ++k) {
      const vcpx *A = &X[k], *Bc = &X[h - k];
      const double wr = r->wr[k], wi = -r->wi[k]; /* e^{+2 pi i k / N} */
      for (int b = 0; b < VB; ++b) {
        const double ar = A->re[b], ai = A->im[b], br = Bc->re[b], bi = -Bc->im[b];
        const double dr0 = ar - br, di0 = ai - bi;
        const double dr = wr * dr0 - wi * di0, di = wr * di0 + wi * dr0;
        Z[k].re[b] = ar + br - di;
        Z[k].im[b] = ai + bi + dr;
      }
    }
    vfft(&r->c, Z, z, 1, scr);
    for (int j = 0; j < h; ++j)
      for (int b = 0; b < VB; ++b) {
        x[(size_t)(2 * j) * VB + b] = z[j].re[b];
        x[(size_t)(2 * j + 1) * VB + b] = z[j].im[b];
      }
  } else {
    Z[0] = X[0];
    for (int k = 1; k <= N / 2; ++k) {
      Z[k] = X[k];
      for (int b = 0; b < VB; ++b) {
        Z[N - k].re[b] = X[k].re[b];
        Z[N - k].im[b] = -X[k].im[b];
      }
    }
    vfft(&r->c, Z, z, 1, scr);
    for (int j = 0; j < N; ++j)
      for (int b = 0; b < VB; ++b) x[(size_t)j * VB + b] = z[j].re[b];
  }
}

/* X_k = sum_j x_j e^{-2 pi i k j / N} for k <= N/2 (8 sequences); work: 2h + scratch vcpx. */
__attribute__((target_clones("arch=x86-64-v3", "default")))
static void r2c(const rplan *r, const double *x, vcpx *X, vcpx *work) {
  const int N = r->N, h = r->h;
  vcpx *z = work, *Z = work + h, *scr = work + 2 * h;
  if (r->even) {
    for (int j = 0; j < h; ++j)
      for (int b = 0; b < VB; ++b) {
        z[j].re[b] = x[(size_t)(2 * j) * VB + b];
        z[j].im[b] = x[(size_t)(2 * j + 1) * VB + b];
      }
    vfft(&r->c, z, Z, 0, scr);
    for (int k = 0; k <= h; ++k) {
      const vcpx *A = &Z[k % h], *Bc = &Z[(h - k) % h];
      const double wr = r->wr[k], wi = r->wi[k];
      for (int b = 0; b < VB; ++b) {
        const double ar = A->re[b], ai = A->im[b], br = Bc->re[b], bi = -Bc->im[b];
        const double er = ar + br, ei = ai + bi, orr = ar - br, oi = ai - bi; /* 2E, 2iO */
        const double pr = oi, pi_ = -orr;                                     /* 2O */
        X[k].re[b] = 0.5 * (er + wr * pr - wi * pi_);
        X[k].im[b] = 0.5 * (ei + wr * pi_ + wi * pr);
      }
    }
  } else {
    for (int j = 0; j < N; ++j)
      for (int b = 0; b < VB; ++b) {
        z[j].re[b] = x[(size_t)j * VB + b];
        z[j].im[b] = 0.0;
      }
    vfft(&r->c, z, Z, 0, scr);
    for (int k = 0; k <= N / 2; ++k) X[k] = Z[k];
  }
}

enum { CPU_CROSS = 0, CPU_DOT = 1, CPU_PROD = 2 };

/* Per-thread state of one block of VB points. */
typedef struct {
  const rplan *rp;
  int m, N;
  int64_t np;
  vcpx *X, *work; /* (N/2 + 1); 2h + scratch */
  double *grid;   /* [7 fields][N][VB] */
} ctx_t;

/* Synthesis of scalar field `comp` of V (nsl slots) for the block at p0 (nb <= VB points) into g[N][VB]. */
static void synth_field(ctx_t *c, const double *V, int nsl, int comp, int64_t p0, int nb, double *g) {
  const int m = c->m, H = c->N / 2;
  memset(c->X, 0, sizeof(vcpx) * (size_t)(H + 1));
  for (int n = 0; n < m && n <= H; ++n) {
    const double *a = V + p0 + c->np * (2 * comp + (int64_t)nsl * n);
    const double *s = V + p0 + c->np * (2 * comp + 1 + (int64_t)nsl * n);
    for (int b = 0; b < nb; ++b) {
      c->X[n].re[b] = n == 0 ? a[b] : 0.5 * a[b];
      c->X[n].im[b] = n == 0 ? 0.0 : -0.5 * s[b];
    }
  }
  c2r(c->rp, c->X, g, c->work);
}

/* Analysis of g[N][VB] into scalar field `comp` of out (nsl slots) for the block at p0. */
static void analyse_field(ctx_t *c, const double *g, double *out, int nsl, int comp, int64_t p0, int nb) {
  const int m = c->m;
  const double invN = 1.0 / (double)c->N, twoN = 2.0 * invN;
  r2c(c->rp, g, c->X, c->work);
  for (int n = 0; n < m; ++n) {
    double *a = out + p0 + c->np * (2 * comp + (int64_t)nsl * n);
    double *s = out + p0 + c->np * (2 * comp + 1 + (int64_t)nsl * n);
    const int live = n <= c->N / 2;
    for (int b = 0; b < nb; ++b) {
      a[b] = live ? (n == 0 ? invN : twoN) * c->X[n].re[b] : 0.0;
      s[b] = (live && n > 0) ? -twoN * c->X[n].im[b] : 0.0;
    }
  }
}

typedef struct {
  const rplan *rp;
  int nprog, m, N;
  const int *op;
  const double *const *A, *const *B;
  double *const *out;
  int64_t np, b0, b1; /* block range of this thread */
  int err;
} job_t;

static void *run_blocks(void *arg) {
  job_t *J = (job_t *)arg;
  const int N = J->N;
  ctx_t c;
  c.rp = J->rp;
  c.m = J->m;
  c.N = N;
  c.np = J->np;
  c.X = (vcpx *)calloc((size_t)(N / 2 + 1), sizeof(vcpx));
  c.work = (vcpx *)calloc((size_t)(2 * J->rp->h + 2 * N + 128), sizeof(vcpx));
  c.grid = (double *)calloc((size_t)7 * VB * N, sizeof(double));
  if (!c.X || !c.work || !c.grid) {
    J->err = -2;
  } else {
    for (int64_t ib = J->b0; ib < J->b1; ++ib) {
      const int64_t p0 = ib * VB;
      const int nb = (int)((J->np - p0) < VB ? (J->np - p0) : VB);
      for (int q = 0; q < J->nprog; ++q) {
        const int op = J->op[q], nsl = op == CPU_PROD ? 2 : 6, nf = nsl / 2;
        double *g1 = c.grid, *g2 = c.grid + (size_t)3 * VB * N, *go = c.grid + (size_t)6 * VB * N;
        for (int k = 0; k < nf; ++k) {
          synth_field(&c, J->A[q], nsl, k, p0, nb, g1 + (size_t)k * VB * N);
          synth_field(&c, J->B[q], nsl, k, p0, nb, g2 + (size_t)k * VB * N);
        }
        const size_t F = (size_t)VB * N;
        if (op == CPU_CROSS) {
          for (int k = 0; k < 3; ++k) {
            const int k1 = (k + 1) % 3, k2 = (k + 2) % 3;
            for (size_t i = 0; i < (size_t)VB * N; ++i)
              go[i] = g1[k1 * F + i] * g2[k2 * F + i] - g1[k2 * F + i] * g2[k1 * F + i];
            analyse_field(&c, go, J->out[q], 6, k, p0, nb);
          }
        } else if (op == CPU_DOT) {
          for (size_t i = 0; i < (size_t)VB * N; ++i)
            go[i] = g1[i] * g2[i] + g1[F + i] * g2[F + i] + g1[2 * F + i] * g2[2 * F + i];
          analyse_field(&c, go, J->out[q], 2, 0, p0, nb);
        } else {
          for (size_t i = 0; i < (size_t)VB * N; ++i) go[i] = g1[i] * g2[i];
          analyse_field(&c, go, J->out[q], 2, 0, p0, nb);
        }
      }
    }
  }
  free(c.X);
  free(c.work);
  free(c.grid);
  return NULL;
}

/* Runs `nprog` products over the same points.  Program q: op[q] on inputs (A[q], B[q]) into out[q]. */
static int run_programs(int nprog, const int *op, const double *const *A, const double *const *B, double *const *out,
                        int64_t np, int m, int N, int nthreads) {
  if (np <= 0) return 0;
  if (m < 1 || N < 2 * m - 1) return -1;
  rplan rp;
  if (rplan_init(&rp, N)) return -2;
  const int64_t nblk = (np + VB - 1) / VB;
  int nt = nthreads > 0 ? nthreads : (int)sysconf(_SC_NPROCESSORS_ONLN);
  if (nt < 1) nt = 1;
  if (nt > 1024) nt = 1024;
  if (nt > nblk) nt = (int)nblk;
  job_t *jobs = (job_t *)calloc((size_t)nt, sizeof(job_t));
  pthread_t *th = (pthread_t *)calloc((size_t)nt, sizeof(pthread_t));
  int err = (!jobs || !th) ? -2 : 0;
  for (int t = 0; t < nt && !err; ++t) {
    job_t J = {&rp, nprog, m, N, op, A, B, out, np, nblk * t / nt, nblk * (t + 1) / nt, 0};
    jobs[t] = J;
  }
  int started = 0;
  for (int t = 1; t < nt && !err; ++t, ++started)
    if (pthread_create(&th[t], NULL, run_blocks, &jobs[t])) {
      err = -3;
      break;
    }
  if (!err) run_blocks(&jobs[0]);
  for (int t = 1; t <= started; ++t) pthread_join(th[t], NULL);
  for (int t = 0; t < nt && !err; ++t)
    if (jobs[t].err) err = jobs[t].err;
  free(jobs);
  free(th);
  rplan_free(&rp);
  return err;
}

/* FFT_PAR_CROSS_PROD_DCL / _DOT_ / _PROD_DCL (op 0/1/2) on (np, nslot, m) Fortran arrays, grid N. */
int sfnl_cpu_product(int op, const double *V1, const double *V2, double *out, int64_t np, int m, int N, int nthreads) {
  if (op < 0 || op > 2) return -1;
  const double *A[1] = {V1}, *B[1] = {V2};
  double *O[1] = {out};
  return run_programs(1, &op, A, B, O, np, m, N, nthreads);
}

/* The MHD bundle: u x w, u x b, j x b (6 slots) and u . gradT (2 slots), point block by point block. */
int sfnl_cpu_mhd_bundle(const double *u, const double *w, const double *b, const double *j, const double *gT,
                        double *uxw, double *uxb, double *jxb, double *ugT, int64_t np, int m, int N, int nthreads) {
  const int op[4] = {CPU_CROSS, CPU_CROSS, CPU_CROSS, CPU_DOT};
  const double *A[4] = {u, u, j, u}, *B[4] = {w, b, b, gT};
  double *O[4] = {uxw, uxb, jxb, ugT};
  return run_programs(4, op, A, B, O, np, m, N, nthreads);
}

/* Host threads used when nthreads <= 0 (the CPU baseline reports it as its core count). */
int sfnl_cpu_threads(void) { return (int)sysconf(_SC_NPROCESSORS_ONLN); }
