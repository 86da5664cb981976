/*
 * sfnl_oracle.c -- CPU oracle for the dealiased pseudo-spectral products.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker: the parity tests,
 * __graft_entry__.smoke() and the CPU-baseline leg of bench.py call it to
 * check the CUDA path.  The product library (sfemans_b200/csrc) never links,
 * loads or calls it.
 *
 * It restates, step by step and in long double arithmetic, the three SFEMaNS
 * routines of SOURCES/POST_PROCESSING/fft_parallel.F90:
 *
 *   FFT_PAR_CROSS_PROD_DCL  fft_parallel.F90:147-328
 *   FFT_PAR_DOT_PROD_DCL    fft_parallel.F90:330-500
 *   FFT_PAR_PROD_DCL        fft_parallel.F90:502-665
 *   FFT_PAR_DIV_DCL         fft_parallel.F90:667-830
 *   FFT_SCALAR_VECT_DCL     fft_parallel.F90:1021-1220  (pb = 1 product, pb = 2 quotient)
 *   FFT_TENSOR_DCL          fft_parallel.F90:1543-1796  (with and without opt_tension)
 *   FFT_PAR_REAL            fft_parallel.F90:28-145     (synthesis only)
 *   FFT_MAX_VEL_DCL         fft_parallel.F90:1426-1541  (synthesis, |v|, maximum)
 *
 * and the Navier-Stokes caller that builds the operands of the cross product at the Gauss points:
 *
 *   smb_cross_prod_gauss_sft_par  SOURCES/SIMULATION/subroutine_ns_with_velocity.F90:512-629
 *
 * including the nb_procs / bloc_size bookkeeping: each emulated rank owns
 * m_max_c contiguous Fourier modes, packs a mode-major dist_field with dummy
 * points set to 1.d100 (:205-211), the MPI_ALLTOALL is emulated by block
 * copies between per-rank buffers (:217, :306), and the unpack drops the
 * dummy points (:311-324).  The FFTW calls are replaced by the definitions
 * FFTW documents for them (unnormalised c2r with sign +1, r2c with sign -1,
 * imaginary parts of the DC and Nyquist inputs of c2r ignored), evaluated as
 * O(N^2) sums with exactly reduced angles (j*k mod N) in long double.
 *
 * FFTW itself (the arithmetic dependency of the reference, unpinned in
 * LIBS/CMakeLists.txt:24) is not present; the DFT definitions above are the
 * published semantics of dfftw_plan_many_dft_c2r / _r2c.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "sfnl_oracle.h"

typedef long double ld;

/* Fortran column-major index helpers. */
#define IDX3(a, b, c, n1, n2) ((size_t)(a) + (size_t)(n1) * ((size_t)(b) + (size_t)(n2) * (size_t)(c)))

static ld two_pi_l(void) { return 2.0L * acosl(-1.0L); }

/* Trig tables cos(2*pi*r/N), sin(2*pi*r/N), r = 0..N-1, long double. */
static int make_tables(int N, ld **ct, ld **st) {
  *ct = (ld *)malloc(sizeof(ld) * (size_t)N);
  *st = (ld *)malloc(sizeof(ld) * (size_t)N);
  if (!*ct || !*st) return -1;
  const ld tp = two_pi_l();
  for (int r = 0; r < N; ++r) {
    ld a = tp * (ld)r / (ld)N;
    (*ct)[r] = cosl(a);
    (*st)[r] = sinl(a);
  }
  return 0;
}

/*
 * c2r of length N from a half-complex array X[0..nx-1] (entries beyond nx
 * are zero).  FFTW c2r: out_j = sum_{k=0}^{N-1} X_k e^{+2 pi i jk/N} with
 * X_{N-k} = conj(X_k); Im X_0 and (N even) Im X_{N/2} are ignored.
 */
static void c2r_ld(int N, int nx, const ld *xr, const ld *xi, ld *out, const ld *ct, const ld *st) {
  for (int j = 0; j < N; ++j) {
    ld s = xr[0];
    for (int k = 1; k < nx && 2 * k <= N; ++k) {
      int r = (int)(((int64_t)j * k) % N);
      ld w = (2 * k == N) ? 1.0L : 2.0L;
      if (2 * k == N)
        s += w * xr[k] * ct[r];
      else
        s += w * (xr[k] * ct[r] - xi[k] * st[r]);
    }
    out[j] = s;
  }
}

/* r2c: Y_k = sum_j x_j e^{-2 pi i jk/N}, k = 0..ny-1. */
static void r2c_ld(int N, int ny, const ld *x, ld *yr, ld *yi, const ld *ct, const ld *st) {
  for (int k = 0; k < ny; ++k) {
    ld sr = 0.0L, si = 0.0L;
    for (int j = 0; j < N; ++j) {
      int r = (int)(((int64_t)j * k) % N);
      sr += x[j] * ct[r];
      si -= x[j] * st[r];
    }
    yr[k] = sr;
    yi[k] = si;
  }
}

/* Pointwise maps of fft_parallel.F90:270-274 (cross), :449-451 (dot), :617 (prod), :786 (div),
 * :1150-1157 (scalar x vector, vector / scalar), :1676-1706 (tensor, tension). ru is (N, nf)
 * column-major: ru[j + N*f]; prod is (N, nout). Tensor outputs are ordered o = 3*k + l. */
static void pointwise(int op, int N, const ld *ru, ld *prod) {
  for (int j = 0; j < N; ++j) {
    const ld *r = ru + j;
#define RU(f) r[(size_t)N * (f)]
#define PR(o) prod[j + (size_t)N * (o)]
    if (op == ORC_CROSS) {
      PR(0) = RU(1) * RU(5) - RU(2) * RU(4);
      PR(1) = RU(2) * RU(3) - RU(0) * RU(5);
      PR(2) = RU(0) * RU(4) - RU(1) * RU(3);
    } else if (op == ORC_DOT) {
      PR(0) = RU(0) * RU(3) + RU(1) * RU(4) + RU(2) * RU(5);
    } else if (op == ORC_PROD) {
      PR(0) = RU(0) * RU(1);
    } else if (op == ORC_DIV) {
      PR(0) = RU(0) / RU(1);
    } else if (op == ORC_SVECT) {
      for (int k = 0; k < 3; ++k) PR(k) = RU(3) * RU(k);
    } else if (op == ORC_SVDIV) {
      for (int k = 0; k < 3; ++k) PR(k) = RU(k) / RU(3);
    } else if (op == ORC_TENSOR) {
      for (int k = 0; k < 3; ++k)
        for (int l = 0; l < 3; ++l) PR(3 * k + l) = RU(k) * RU(3 + l);
    } else { /* ORC_TENSION */
      const ld nrm = sqrtl(RU(3) * RU(3) + RU(4) * RU(4) + RU(5) * RU(5));
      for (int k = 0; k < 3; ++k)
        for (int l = 0; l < 3; ++l) PR(3 * k + l) = RU(k) * RU(3 + l) / (nrm + 1.0e-14L) - (k == l ? nrm : 0.0L);
    }
#undef RU
#undef PR
  }
}

static int op_nout(int op) {
  return (op == ORC_CROSS || op == ORC_SVECT || op == ORC_SVDIV) ? 3 : (op == ORC_TENSOR || op == ORC_TENSION) ? 9 : 1;
}

int orc_fft_par_dcl(int op, const double *V1, const double *V2, double *Vout, int np, int nb_field,
                    int m_max_c, int nb_procs, int bloc_size, int m_max_pad) {
  return orc_fft_par_dcl_n(op, V1, V2, Vout, np, nb_field, m_max_c, nb_procs, bloc_size, m_max_pad,
                           2 * m_max_pad - 1);
}

int orc_fft_par_dcl_n(int op, const double *V1, const double *V2, double *Vout, int np, int nb_field,
                      int m_max_c, int nb_procs, int bloc_size, int m_max_pad, int N) {
  if (op != ORC_CROSS && op != ORC_DOT && op != ORC_PROD && op != ORC_DIV) return -1;
  if (op == ORC_PROD || op == ORC_DIV) nb_field = 2; /* c_in is (np,2,m_max_c), fft_parallel.F90:510 */
  return orc_apply_n(op, V1, nb_field, V2, nb_field, Vout, np, m_max_c, nb_procs, bloc_size, m_max_pad, N);
}

int orc_apply_n(int op, const double *V1, int nsl1, const double *V2, int nsl2, double *Vout, int np,
                int m_max_c, int nb_procs, int bloc_size, int m_max_pad, int N) {
  if (op < ORC_CROSS || op > ORC_TENSION) return -1;
  /* fft_parallel.F90:188-191, :370-373, :560-563, :1068-1071, :1590-1593 */
  if ((nsl1 % 2) != 0 || (nsl2 % 2) != 0 || m_max_c <= 0) return -1;
  /* the product is only formed for these slot counts (:270, :449, :1130, :1676) */
  if ((op == ORC_CROSS || op == ORC_DOT || op == ORC_TENSOR || op == ORC_TENSION) && (nsl1 != 6 || nsl2 != 6)) return -1;
  if ((op == ORC_SVECT || op == ORC_SVDIV) && (nsl1 != 6 || nsl2 != 2)) return -1;
  if ((op == ORC_PROD || op == ORC_DIV) && (nsl1 != 2 || nsl2 != 2)) return -1;
  if (nb_procs < 1 || bloc_size < 1 || np < 0) return -1;
  const int m_max = m_max_c * nb_procs;
  const int np_tot = nb_procs * bloc_size;
  if (np > np_tot) return -2;        /* dist_field would overflow (:204-208) */
  if (m_max_pad < m_max) return -3;  /* cu(shiftl+1:shiftl+m_max_c) beyond m_max_pad (:229) */
  if (N < 1) return -3;
  const int nx = N / 2 + 1 < m_max_pad ? N / 2 + 1 : m_max_pad; /* half-complex entries used by c2r */
  if (m_max > N / 2 + 1) return -3;

  const int nfc = (nsl1 + nsl2) / 2;                    /* complex fields in cu (both inputs) */
  const int nout = op_nout(op);                         /* complex output fields */
  const int tensor = (op == ORC_TENSOR || op == ORC_TENSION);
  const int nslot_out = tensor ? 6 : 2 * nout;          /* V_out slots (tensor: V_out(3, np, 6, m)) */
  const int dslots = nsl1 + nsl2;                       /* dist_field second dimension */

  ld *ct = NULL, *st = NULL;
  if (make_tables(N, &ct, &st)) return -4;

  /* Per-rank buffers: dist_field(m_max_c, dslots, np_tot), combined_field same. */
  const size_t dsz = (size_t)m_max_c * dslots * np_tot;
  double **dist = (double **)calloc((size_t)nb_procs, sizeof(double *));
  double **comb = (double **)calloc((size_t)nb_procs, sizeof(double *));
  /* combined_prod_cu(nout, bloc_size, m_max) complex, per rank; dist_prod_cu same. */
  const size_t psz = (size_t)nout * bloc_size * m_max;
  ld **cpr = (ld **)calloc((size_t)nb_procs, sizeof(ld *)), **cpi = (ld **)calloc((size_t)nb_procs, sizeof(ld *));
  ld **dpr = (ld **)calloc((size_t)nb_procs, sizeof(ld *)), **dpi = (ld **)calloc((size_t)nb_procs, sizeof(ld *));
  int rc = 0;
  for (int r = 0; r < nb_procs; ++r) {
    dist[r] = (double *)malloc(sizeof(double) * (dsz ? dsz : 1));
    comb[r] = (double *)malloc(sizeof(double) * (dsz ? dsz : 1));
    cpr[r] = (ld *)calloc(psz ? psz : 1, sizeof(ld));
    cpi[r] = (ld *)calloc(psz ? psz : 1, sizeof(ld));
    dpr[r] = (ld *)calloc(psz ? psz : 1, sizeof(ld));
    dpi[r] = (ld *)calloc(psz ? psz : 1, sizeof(ld));
    if (!dist[r] || !comb[r] || !cpr[r] || !cpi[r] || !dpr[r] || !dpi[r]) rc = -4;
  }
  ld *cur = (ld *)malloc(sizeof(ld) * (size_t)m_max_pad * nfc);
  ld *cui = (ld *)malloc(sizeof(ld) * (size_t)m_max_pad * nfc);
  ld *ru = (ld *)malloc(sizeof(ld) * (size_t)N * nfc);
  ld *pru = (ld *)malloc(sizeof(ld) * (size_t)N * nout);
  ld *pcr = (ld *)malloc(sizeof(ld) * (size_t)m_max_pad * nout);
  ld *pci = (ld *)malloc(sizeof(ld) * (size_t)m_max_pad * nout);
  if (!cur || !cui || !ru || !pru || !pcr || !pci) rc = -4;
  if (rc) goto done;

  /* (1) TRANSPOSE pack on every rank, dummy points = 1.d100 (:205-211). */
  for (int r = 0; r < nb_procs; ++r) {
    for (size_t t = 0; t < dsz; ++t) dist[r][t] = 1.0e100;
    for (int i = 0; i < m_max_c; ++i) {
      const int g = r * m_max_c + i; /* global mode of local mode i (initialization.F90:823-835) */
      for (int p = 0; p < np; ++p) {
        for (int s = 0; s < nsl1; ++s) dist[r][IDX3(i, s, p, m_max_c, dslots)] = V1[IDX3(p, s, g, np, nsl1)];
        for (int s = 0; s < nsl2; ++s) dist[r][IDX3(i, nsl1 + s, p, m_max_c, dslots)] = V2[IDX3(p, s, g, np, nsl2)];
      }
    }
  }
  /* (2) MPI_ALLTOALL: block q of rank r's send buffer lands in block r of rank q (:217). */
  for (int r = 0; r < nb_procs; ++r)
    for (int q = 0; q < nb_procs; ++q) {
      const size_t blk = (size_t)m_max_c * dslots * bloc_size;
      memcpy(comb[q] + (size_t)r * blk, dist[r] + (size_t)q * blk, sizeof(double) * blk);
    }

  /* (3)-(8) per rank: pack, c2r, product, r2c, scale, 2*CONJG. */
  for (int q = 0; q < nb_procs; ++q) {
    for (int n = 0; n < bloc_size; ++n) {
      for (size_t t = 0; t < (size_t)m_max_pad * nfc; ++t) cur[t] = cui[t] = 0.0L; /* cu = 0 (:222) */
      for (int nb = 0; nb < nb_procs; ++nb) {
        const int shiftc = nb * bloc_size, shiftl = nb * m_max_c, jindex = n + shiftc;
        for (int nf = 0; nf < nfc; ++nf)
          for (int i = 0; i < m_max_c; ++i) {
            /* c_n = (a_n - i b_n)/2 (:234-235) */
            cur[(shiftl + i) + m_max_pad * nf] = 0.5L * (ld)comb[q][IDX3(i, 2 * nf, jindex, m_max_c, dslots)];
            cui[(shiftl + i) + m_max_pad * nf] = -0.5L * (ld)comb[q][IDX3(i, 2 * nf + 1, jindex, m_max_c, dslots)];
          }
      }
      for (int nf = 0; nf < nfc; ++nf) { /* cu(1,:,:) = 2*REAL(cu(1,:,:)) (:241) */
        cur[m_max_pad * nf] = 2.0L * cur[m_max_pad * nf];
        cui[m_max_pad * nf] = 0.0L;
      }
      for (int nf = 0; nf < nfc; ++nf)
        c2r_ld(N, nx, cur + (size_t)m_max_pad * nf, cui + (size_t)m_max_pad * nf, ru + (size_t)N * nf, ct, st);
      pointwise(op, N, ru, pru);
      const ld invN = 1.0L / (ld)N; /* (:288) */
      for (size_t t = 0; t < (size_t)m_max_pad * nout; ++t) pcr[t] = pci[t] = 0.0L;
      for (int o = 0; o < nout; ++o) {
        r2c_ld(N, m_max_pad < N / 2 + 1 ? m_max_pad : N / 2 + 1, pru + (size_t)N * o, pcr + (size_t)m_max_pad * o,
               pci + (size_t)m_max_pad * o, ct, st);
        for (int k = 0; k < m_max_pad; ++k) {
          pcr[k + m_max_pad * o] *= invN;
          pci[k + m_max_pad * o] *= invN;
        }
      }
      /* combined_prod_cu(:,n,1) = prod_cu(1); (:,n,k) = 2*CONJG(prod_cu(k)) for k>=2 (:295-299) */
      for (int o = 0; o < nout; ++o)
        for (int k = 0; k < m_max; ++k) {
          const ld re = pcr[k + m_max_pad * o], im = pci[k + m_max_pad * o];
          const size_t at = IDX3(o, n, k, nout, bloc_size);
          cpr[q][at] = (k == 0) ? re : 2.0L * re;
          cpi[q][at] = (k == 0) ? im : -2.0L * im;
        }
    }
  }
  /* (9) MPI_ALLTOALL back: block r (modes r*m_max_c..) of rank q goes to block q of rank r (:306). */
  for (int q = 0; q < nb_procs; ++q)
    for (int r = 0; r < nb_procs; ++r) {
      const size_t blk = (size_t)nout * bloc_size * m_max_c;
      memcpy(dpr[r] + (size_t)q * blk, cpr[q] + (size_t)r * blk, sizeof(ld) * blk);
      memcpy(dpi[r] + (size_t)q * blk, cpi[q] + (size_t)r * blk, sizeof(ld) * blk);
    }
  /* (10) unpack into v_out(n+shiftc, 2*i_field-1:2*i_field, i), dropping dummy points (:311-324). */
  for (int r = 0; r < nb_procs; ++r)
    for (int i = 0; i < m_max_c; ++i)
      for (int nb = 0; nb < nb_procs; ++nb) {
        const int shiftc = nb * bloc_size, shiftl = nb * m_max_c;
        for (int n = 0; n < bloc_size; ++n) {
          if (n + shiftc >= np) continue;
          for (int o = 0; o < nout; ++o) {
            const size_t at = IDX3(o, n, shiftl + i, nout, bloc_size);
            const int g = r * m_max_c + i;
            if (tensor) { /* v_out(k, n+shiftc, 2l-1:2l, i) (:1786-1787) */
              const int k = o / 3, l = o % 3;
              Vout[k + 3 * IDX3(n + shiftc, 2 * l, g, np, 6)] = (double)dpr[r][at];
              Vout[k + 3 * IDX3(n + shiftc, 2 * l + 1, g, np, 6)] = (double)dpi[r][at];
            } else {
              Vout[IDX3(n + shiftc, 2 * o, g, np, nslot_out)] = (double)dpr[r][at];
              Vout[IDX3(n + shiftc, 2 * o + 1, g, np, nslot_out)] = (double)dpi[r][at];
            }
          }
        }
      }

done:
  for (int r = 0; r < nb_procs; ++r) {
    free(dist[r]); free(comb[r]); free(cpr[r]); free(cpi[r]); free(dpr[r]); free(dpi[r]);
  }
  free(dist); free(comb); free(cpr); free(cpi); free(dpr); free(dpi);
  free(cur); free(cui); free(ru); free(pru); free(pcr); free(pci);
  free(ct); free(st);
  return rc;
}

/* Shared by the two synthesis-only routines: every emulated rank packs dist_field(m_max_c, nsl,
 * np_tot) (dummy points set to `dummy`), the MPI_ALLTOALL is emulated, and rank q synthesises its
 * bloc_size points: ru_q(N, nsl/2, bloc_size) = c2r of the half-complex pack of every field
 * (fft_parallel.F90:88-131, :1474-1519).  `visit(ctx, q, n, ru)` receives ru (N, nsl/2) of point n of
 * rank q. */
typedef void (*synth_visit)(void *ctx, int q, int n, const ld *ru, int N, int nfc);

static int synth_ranks(const double *V1, int nsl, int np, int m_max_c, int nb_procs, int bloc_size, int m_max_pad,
                       double dummy, synth_visit visit, void *ctx) {
  const int np_tot = nb_procs * bloc_size, N = 2 * m_max_pad - 1, nfc = nsl / 2;
  const int m_max = m_max_c * nb_procs;
  if (m_max_pad < m_max) return -3;
  if (np > np_tot) return -2; /* dist_field(:,:,np_tot) would overflow */
  ld *ct = NULL, *st = NULL;
  if (make_tables(N, &ct, &st)) return -4;
  const size_t dsz = (size_t)m_max_c * nsl * np_tot, blk = (size_t)m_max_c * nsl * bloc_size;
  double *dist = (double *)malloc(sizeof(double) * (dsz ? dsz : 1) * (size_t)nb_procs);
  double *comb = (double *)malloc(sizeof(double) * (dsz ? dsz : 1) * (size_t)nb_procs);
  ld *cur = (ld *)malloc(sizeof(ld) * (size_t)m_max_pad * nfc), *cui = (ld *)malloc(sizeof(ld) * (size_t)m_max_pad * nfc);
  ld *ru = (ld *)malloc(sizeof(ld) * (size_t)N * nfc);
  int rc = (!dist || !comb || !cur || !cui || !ru) ? -4 : 0;
  if (!rc) {
    for (int r = 0; r < nb_procs; ++r) { /* TRANSPOSE pack, dummy points */
      double *d = dist + (size_t)r * dsz;
      for (size_t t = 0; t < dsz; ++t) d[t] = dummy;
      for (int i = 0; i < m_max_c; ++i)
        for (int p = 0; p < np; ++p)
          for (int s2 = 0; s2 < nsl; ++s2) d[IDX3(i, s2, p, m_max_c, nsl)] = V1[IDX3(p, s2, r * m_max_c + i, np, nsl)];
    }
    for (int r = 0; r < nb_procs; ++r) /* MPI_ALLTOALL */
      for (int q = 0; q < nb_procs; ++q)
        memcpy(comb + (size_t)q * dsz + (size_t)r * blk, dist + (size_t)r * dsz + (size_t)q * blk, sizeof(double) * blk);
    for (int q = 0; q < nb_procs; ++q)
      for (int n = 0; n < bloc_size; ++n) {
        for (size_t t = 0; t < (size_t)m_max_pad * nfc; ++t) cur[t] = cui[t] = 0.0L;
        for (int nb = 0; nb < nb_procs; ++nb) {
          const int shiftc = nb * bloc_size, shiftl = nb * m_max_c, jindex = n + shiftc;
          for (int nf = 0; nf < nfc; ++nf)
            for (int i = 0; i < m_max_c; ++i) {
              cur[(shiftl + i) + m_max_pad * nf] = 0.5L * (ld)comb[(size_t)q * dsz + IDX3(i, 2 * nf, jindex, m_max_c, nsl)];
              cui[(shiftl + i) + m_max_pad * nf] = -0.5L * (ld)comb[(size_t)q * dsz + IDX3(i, 2 * nf + 1, jindex, m_max_c, nsl)];
            }
        }
        for (int nf = 0; nf < nfc; ++nf) {
          cur[m_max_pad * nf] *= 2.0L;
          cui[m_max_pad * nf] = 0.0L;
        }
        for (int nf = 0; nf < nfc; ++nf)
          c2r_ld(N, m_max_pad, cur + (size_t)m_max_pad * nf, cui + (size_t)m_max_pad * nf, ru + (size_t)N * nf, ct, st);
        visit(ctx, q, n, ru, N, nfc);
      }
  }
  free(dist); free(comb); free(cur); free(cui); free(ru); free(ct); free(st);
  return rc;
}

int orc_fft_par_real_planes(int m_max, int opt_nb_plane) {
  /* m_max_pad = (opt_nb_plane+1)/2 if opt_nb_plane > 2*m_max-1, else m_max (fft_parallel.F90:71-79) */
  const int m_max_pad = (opt_nb_plane > 2 * m_max - 1) ? (opt_nb_plane + 1) / 2 : m_max;
  return 2 * m_max_pad - 1;
}

struct real_ctx { double *Vout; int bloc_size, N; };
static void real_visit(void *c, int q, int n, const ld *ru, int N, int nfc) {
  struct real_ctx *x = (struct real_ctx *)c;
  const int p = q * x->bloc_size + n; /* rank q holds points q*bloc_size .. */
  for (int f = 0; f < nfc; ++f)
    for (int j = 0; j < N; ++j) x->Vout[IDX3(j, f, p, N, nfc)] = (double)ru[(size_t)N * f + j];
}

int orc_fft_par_real(const double *V1, int nsl, int np, int m_max_c, int nb_procs, int opt_nb_plane, double *Vout) {
  if ((nsl % 2) != 0 || m_max_c <= 0 || nb_procs < 1 || np < 0) return -1; /* :59-61 */
  if (np % nb_procs) return -2;                                              /* :65-71 */
  const int m_max = m_max_c * nb_procs, N = orc_fft_par_real_planes(m_max, opt_nb_plane);
  struct real_ctx c = {Vout, np / nb_procs, N};
  return synth_ranks(V1, nsl, np, m_max_c, nb_procs, np / nb_procs, (N + 1) / 2, 0.0, real_visit, &c);
}

struct maxv_ctx { ld vmax; int nsl; };
static void maxv_visit(void *c, int q, int n, const ld *ru, int N, int nfc) {
  struct maxv_ctx *x = (struct maxv_ctx *)c;
  (void)q; (void)n; (void)nfc;
  for (int j = 0; j < N; ++j) {
    /* |v| of the first vector for nb_field == 6, |first field| otherwise (:1528-1532) */
    const ld v = (x->nsl == 6) ? sqrtl(ru[j] * ru[j] + ru[N + j] * ru[N + j] + ru[2 * N + j] * ru[2 * N + j])
                               : sqrtl(ru[j] * ru[j]);
    if (v > x->vmax) x->vmax = v;
  }
}

int orc_fft_max_vel(const double *V1, int nsl, int np, int m_max_c, int nb_procs, int bloc_size, int m_max_pad,
                    double *vmax) {
  if ((nsl % 2) != 0 || m_max_c <= 0 || nb_procs < 1 || bloc_size < 1 || np < 0) return -1; /* :1457-1460 */
  struct maxv_ctx c = {0.0L, nsl};
  /* dummy points are 0 (:1478): their |v| = 0 never exceeds the maximum of the others */
  const int rc = synth_ranks(V1, nsl, np, m_max_c, nb_procs, bloc_size, m_max_pad, 0.0, maxv_visit, &c);
  *vmax = (double)c.vmax; /* MAXVAL per rank, then MPI_ALLREDUCE MAX (:1533-1535) */
  return rc;
}

/* smb_cross_prod_gauss_sft_par (subroutine_ns_with_velocity.F90:512-629), one Fourier rank holding
 * the nmod modes list_mode[0..nmod): for every mode i, element m and Gauss point l (Gauss index
 * (m l_G + l), :563-574) the velocity W = sum_n V(jj(n,m)) ww(n,l), the rotation Om likewise from
 * omega (NULL: no precession, Om = 0, :615-617), the radius ray = sum_n rr(1,jj(n,m)) ww(n,l) (:573)
 * and the curl in cylindrical coordinates of Fourier mode `mode` (:592-607); RotV += 2 Om (:620);
 * then FFT_PAR_CROSS_PROD_DCL(RotV, W) with m_max_pad = 3*nmod/2 (:624-626).  jj is 1-based
 * (n_w, me); ww (n_w, l_G); dw (2, n_w, l_G, me); rr (2, np_nodes); V, omega (np_nodes, 6, nmod);
 * Vout (l_G*me, 6, nmod), or NULL to skip the product.  RotV and W (l_G*me, 6, nmod) may be returned
 * (NULL: not wanted). */
int orc_cross_gauss(const double *V, const int *jj, const double *ww, const double *dw, const double *rr,
                    const int *list_mode, const double *omega, int np_nodes, int me, int n_w, int l_G, int nmod,
                    double *Vout, double *RotV_out, double *W_out) {
  if (np_nodes < 1 || me < 0 || n_w < 1 || l_G < 1 || nmod < 1) return -1;
  const int ng = l_G * me;
  double *RotV = (double *)calloc((size_t)ng * 6 * nmod + 1, sizeof(double));
  double *W = (double *)calloc((size_t)ng * 6 * nmod + 1, sizeof(double));
  if (!RotV || !W) { free(RotV); free(W); return -4; }
  for (int m = 0; m < me; ++m)
    for (int n = 0; n < n_w; ++n)
      if (jj[n + (size_t)n_w * m] < 1 || jj[n + (size_t)n_w * m] > np_nodes) { free(RotV); free(W); return -2; }
  for (int i = 0; i < nmod; ++i) {
    const double mode = (double)list_mode[i];
    for (int m = 0; m < me; ++m)
      for (int l = 0; l < l_G; ++l) {
        const size_t idx = (size_t)m * l_G + l;
        const double *dwl = dw + (size_t)2 * n_w * (l + (size_t)l_G * m); /* dw_loc = dw(:,:,l,m) */
        double ray = 0.0, w[6] = {0, 0, 0, 0, 0, 0}, om[6] = {0, 0, 0, 0, 0, 0};
        double d1[6] = {0, 0, 0, 0, 0, 0}, d2[6] = {0, 0, 0, 0, 0, 0}; /* SUM(Vs(:,k)*dw_loc(1|2,:)) */
        for (int n = 0; n < n_w; ++n) {
          const int node = jj[n + (size_t)n_w * m] - 1;
          const double wv = ww[n + (size_t)n_w * l];
          ray += rr[2 * (size_t)node] * wv;
          for (int k = 0; k < 6; ++k) {
            const double vs = V[IDX3(node, k, i, np_nodes, 6)];
            w[k] += vs * wv;
            d1[k] += vs * dwl[2 * n];
            d2[k] += vs * dwl[2 * n + 1];
            if (omega) om[k] += omega[IDX3(node, k, i, np_nodes, 6)] * wv;
          }
        }
        double *R = RotV + idx, *Wo = W + idx;
#define AT(a, k) a[(size_t)ng * ((k) + 6 * (size_t)i)]
        for (int k = 0; k < 6; ++k) AT(Wo, k) = w[k];
        AT(R, 0) = mode / ray * w[5] - d2[2];
        AT(R, 3) = d2[1] - d1[5];
        AT(R, 4) = 1 / ray * w[2] + d1[2] - mode / ray * w[1];
        AT(R, 1) = -mode / ray * w[4] - d2[3];
        AT(R, 2) = d2[0] - d1[4];
        AT(R, 5) = 1 / ray * w[3] + d1[3] + mode / ray * w[0];
        for (int k = 0; k < 6; ++k) AT(R, k) = AT(R, k) + 2.0 * om[k];
#undef AT
      }
  }
  const int pad = 3 * nmod / 2 < nmod ? nmod : 3 * nmod / 2;
  int rc = Vout ? orc_apply_n(ORC_CROSS, RotV, 6, W, 6, Vout, ng, nmod, 1, ng + 1, pad, 2 * pad - 1) : 0;
  if (RotV_out) memcpy(RotV_out, RotV, sizeof(double) * (size_t)ng * 6 * nmod);
  if (W_out) memcpy(W_out, W, sizeof(double) * (size_t)ng * 6 * nmod);
  free(RotV);
  free(W);
  return rc;
}

/* smb_CurlH_cross_B_gauss_sft_par (subroutine_ns_with_m.F90:788-883): W = B and RotV = curl H at the
 * Gauss points (loop :812-869, the same curl formulas as the Navier-Stokes caller, no precession), then
 * FFT_PAR_CROSS_PROD_DCL(RotV, W) with m_max_pad = 3*nmod/2 (:876-878). */
int orc_curlh_cross_b_gauss(const double *H, const double *B, const int *jj, const double *ww, const double *dw,
                            const double *rr, const int *list_mode, int np_nodes, int me, int n_w, int l_G, int nmod,
                            double *Vout, double *RotV_out, double *W_out) {
  if (np_nodes < 1 || me < 0 || n_w < 1 || l_G < 1 || nmod < 1) return -1;
  const int ng = l_G * me;
  double *RotV = (double *)calloc((size_t)ng * 6 * nmod + 1, sizeof(double));
  double *W = (double *)calloc((size_t)ng * 6 * nmod + 1, sizeof(double));
  if (!RotV || !W) { free(RotV); free(W); return -4; }
  for (int m = 0; m < me; ++m)
    for (int n = 0; n < n_w; ++n)
      if (jj[n + (size_t)n_w * m] < 1 || jj[n + (size_t)n_w * m] > np_nodes) { free(RotV); free(W); return -2; }
  for (int i = 0; i < nmod; ++i) {
    const double mode = (double)list_mode[i];
    for (int m = 0; m < me; ++m)
      for (int l = 0; l < l_G; ++l) {
        const size_t idx = (size_t)m * l_G + l;
        const double *dwl = dw + (size_t)2 * n_w * (l + (size_t)l_G * m);
        double ray = 0.0, v[6] = {0, 0, 0, 0, 0, 0}, w[6] = {0, 0, 0, 0, 0, 0};
        double d1[6] = {0, 0, 0, 0, 0, 0}, d2[6] = {0, 0, 0, 0, 0, 0};
        for (int n = 0; n < n_w; ++n) {
          const int node = jj[n + (size_t)n_w * m] - 1;
          const double wv = ww[n + (size_t)n_w * l];
          ray += rr[2 * (size_t)node] * wv;
          for (int k = 0; k < 6; ++k) {
            const double vs = H[IDX3(node, k, i, np_nodes, 6)];
            v[k] += vs * wv;
            d1[k] += vs * dwl[2 * n];
            d2[k] += vs * dwl[2 * n + 1];
            w[k] += B[IDX3(node, k, i, np_nodes, 6)] * wv;
          }
        }
        double *R = RotV + idx, *Wo = W + idx;
#define AT(a, k) a[(size_t)ng * ((k) + 6 * (size_t)i)]
        for (int k = 0; k < 6; ++k) AT(Wo, k) = w[k];
        AT(R, 0) = mode / ray * v[5] - d2[2];
        AT(R, 3) = d2[1] - d1[5];
        AT(R, 4) = 1 / ray * v[2] + d1[2] - mode / ray * v[1];
        AT(R, 1) = -mode / ray * v[4] - d2[3];
        AT(R, 2) = d2[0] - d1[4];
        AT(R, 5) = 1 / ray * v[3] + d1[3] + mode / ray * v[0];
#undef AT
      }
  }
  const int pad = 3 * nmod / 2 < nmod ? nmod : 3 * nmod / 2;
  int rc = Vout ? orc_apply_n(ORC_CROSS, RotV, 6, W, 6, Vout, ng, nmod, 1, ng + 1, pad, 2 * pad - 1) : 0;
  if (RotV_out) memcpy(RotV_out, RotV, sizeof(double) * (size_t)ng * 6 * nmod);
  if (W_out) memcpy(W_out, W, sizeof(double) * (size_t)ng * 6 * nmod);
  free(RotV);
  free(W);
  return rc;
}

/* smb_ugradc_gauss_fft_par (subroutine_level_set.F90:434-534; subroutine_temperature_with_T.F90:247-350
 * with heat != NULL; smb_ugradc_gauss_fft_par_conc, subroutine_concentration.F90:243-341): W = u,
 * Gradc = grad c, Div = div u and Cgauss = c at the Gauss points (:469-514), Gradc and Cgauss times
 * heat(m); c_out = FFT_PAR_DOT_PROD_DCL(Gradc, W) [+ FFT_PAR_PROD_DCL(Div, Cgauss) when conservative,
 * the two results added as the reference does].  V (np_nodes, 6, nmod), C (np_nodes, 2, nmod), heat (me)
 * or NULL, Vout (l_G*me, 2, nmod); the operand outputs (l_G*me, 6 | 6 | 2 | 2, nmod) may be NULL. */
int orc_ugradc_gauss(const double *V, const double *C, const double *heat, int conservative, const int *jj,
                     const double *ww, const double *dw, const double *rr, const int *list_mode, int np_nodes, int me,
                     int n_w, int l_G, int nmod, double *Vout, double *Gradc_out, double *W_out, double *Div_out,
                     double *Cg_out) {
  if (np_nodes < 1 || me < 0 || n_w < 1 || l_G < 1 || nmod < 1) return -1;
  const int ng = l_G * me;
  const size_t n6 = (size_t)ng * 6 * nmod, n2 = (size_t)ng * 2 * nmod;
  double *G = (double *)calloc(n6 + 1, sizeof(double)), *W = (double *)calloc(n6 + 1, sizeof(double));
  double *D = (double *)calloc(n2 + 1, sizeof(double)), *Cg = (double *)calloc(n2 + 1, sizeof(double));
  double *T = (double *)calloc(n2 + 1, sizeof(double));
  if (!G || !W || !D || !Cg || !T) { free(G); free(W); free(D); free(Cg); free(T); return -4; }
  int rc = 0;
  for (int m = 0; m < me && !rc; ++m)
    for (int n = 0; n < n_w; ++n)
      if (jj[n + (size_t)n_w * m] < 1 || jj[n + (size_t)n_w * m] > np_nodes) rc = -2;
  for (int i = 0; i < nmod && !rc; ++i) {
    const double mode = (double)list_mode[i];
    for (int m = 0; m < me; ++m)
      for (int l = 0; l < l_G; ++l) {
        const size_t idx = (size_t)m * l_G + l;
        const double *dwl = dw + (size_t)2 * n_w * (l + (size_t)l_G * m);
        double ray = 0.0, w[6] = {0, 0, 0, 0, 0, 0}, d1[6] = {0, 0, 0, 0, 0, 0}, d2[6] = {0, 0, 0, 0, 0, 0};
        double cw[2] = {0, 0}, c1[2] = {0, 0}, c2[2] = {0, 0};
        for (int n = 0; n < n_w; ++n) {
          const int node = jj[n + (size_t)n_w * m] - 1;
          const double wv = ww[n + (size_t)n_w * l];
          ray += rr[2 * (size_t)node] * wv;
          for (int k = 0; k < 6; ++k) {
            const double vs = V[IDX3(node, k, i, np_nodes, 6)];
            w[k] += vs * wv;
            d1[k] += vs * dwl[2 * n];
            d2[k] += vs * dwl[2 * n + 1];
          }
          for (int k = 0; k < 2; ++k) {
            const double cs = C[IDX3(node, k, i, np_nodes, 2)];
            cw[k] += cs * wv;
            c1[k] += cs * dwl[2 * n];
            c2[k] += cs * dwl[2 * n + 1];
          }
        }
        const double hc = heat ? heat[m] : 1.0;
#define AT6(a, k) a[idx + (size_t)ng * ((k) + 6 * (size_t)i)]
#define AT2(a, k) a[idx + (size_t)ng * ((k) + 2 * (size_t)i)]
        for (int k = 0; k < 6; ++k) AT6(W, k) = w[k];
        AT2(D, 0) = d1[0] + w[0] / ray + (mode / ray) * w[3] + d2[4];
        AT2(D, 1) = d1[1] + w[1] / ray - (mode / ray) * w[2] + d2[5];
        AT6(G, 0) = c1[0];
        AT6(G, 1) = c1[1];
        AT6(G, 2) = mode / ray * cw[1];
        AT6(G, 3) = -mode / ray * cw[0];
        AT6(G, 4) = c2[0];
        AT6(G, 5) = c2[1];
        AT2(Cg, 0) = cw[0];
        AT2(Cg, 1) = cw[1];
        if (heat) {
          for (int k = 0; k < 6; ++k) AT6(G, k) = hc * AT6(G, k);
          AT2(Cg, 0) = hc * AT2(Cg, 0);
          AT2(Cg, 1) = hc * AT2(Cg, 1);
        }
#undef AT6
#undef AT2
      }
  }
  const int pad = 3 * nmod / 2 < nmod ? nmod : 3 * nmod / 2;
  if (!rc && Vout) {
    rc = orc_apply_n(ORC_DOT, G, 6, W, 6, Vout, ng, nmod, 1, ng + 1, pad, 2 * pad - 1);
    if (!rc && conservative) {
      rc = orc_apply_n(ORC_PROD, D, 2, Cg, 2, T, ng, nmod, 1, ng + 1, pad, 2 * pad - 1);
      for (size_t t = 0; t < n2; ++t) Vout[t] += T[t];
    }
  }
  if (Gradc_out) memcpy(Gradc_out, G, sizeof(double) * n6);
  if (W_out) memcpy(W_out, W, sizeof(double) * n6);
  if (Div_out) memcpy(Div_out, D, sizeof(double) * n2);
  if (Cg_out) memcpy(Cg_out, Cg, sizeof(double) * n2);
  free(G); free(W); free(D); free(Cg); free(T);
  return rc;
}
