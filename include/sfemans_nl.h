/*
 * sfemans_nl.h -- C-ABI of the B200 pseudo-spectral nonlinear-term library.
 *
 * Replaces the dealiased products of SFEMaNS's MODULE fft_parallele
 * (SOURCES/POST_PROCESSING/fft_parallel.F90, PUBLIC list :8-17):
 *   FFT_PAR_CROSS_PROD_DCL  :147-328   V_out = V1 x V2
 *   FFT_PAR_DOT_PROD_DCL    :330-500   c_out = V1 . V2
 *   FFT_PAR_PROD_DCL        :502-665   c_out = c1 * c2
 * and the same-pattern siblings with another pointwise map:
 *   FFT_PAR_DIV_DCL         :667-830   c_out = c1 / c2
 *   FFT_SCALAR_VECT_DCL     :1021-1220 V_out = s V (pb = 1) or V / s (pb = 2)
 *   FFT_TENSOR_DCL          :1543-1796 V_out(k, :, 2l-1:2l, :) = V1_k V2_l, or with
 *                                      opt_tension V1_k V2_l / (|V2| + 1e-14) - |V2| delta_kl
 * and the synthesis-only routines:
 *   FFT_PAR_REAL            :28-145    V_out(N, nb_field/2, np) = values on the grid
 *   FFT_MAX_VEL_DCL         :1426-1541 V_out = max over points and angles of |V1|
 *
 * Array layout: every coefficient array is the Fortran array V(np, nslot, m)
 * in column-major order, point index fastest: element (p, s, n) is at
 * V[p + np*(s + nslot*n)].  Slot 2k (0-based) holds the cosine coefficient
 * and slot 2k+1 the sine coefficient of component k (r, theta, z for
 * 3-vectors).  Input sine-of-mode-0 entries are ignored; output ones are 0.
 * Batched arrays append a last dimension: V(np, nslot, m, k_batch).
 *
 * Semantics: out = T[ (S a) op (S b) ] where S evaluates the Fourier series
 * f(theta) = a_0 + sum_{n<m} a_n cos(n theta) + b_n sin(n theta) on a grid of
 * N equispaced angles and T is the DFT analysis truncated to n < m
 * (a_0 = (1/N) sum f, a_n = (2/N) sum f cos, b_n = (2/N) sum f sin).
 * With m_max_pad >= ceil((3m-1)/2), which every SFEMaNS caller uses
 * (m_max_pad = 3*m_max/2, subroutine_ns_with_velocity.F90:626), the result
 * is the exact truncated product and does not depend on N.
 *
 * Return value of every entry point: SFNL_OK (0) or a negative SFNL_ERR_*
 * code; sfnl_last_error() gives a one-line message for the calling thread.
 * The reference prints 'BUG in FFT_PAR_...' and STOPs (fft_parallel.F90:188-191);
 * the Fortran shim (sfemans_b200/fortran/fft_parallele_gpu.F90) turns a
 * non-zero status into the same STOP.
 *
 * Threading: entry points are thread-safe; work is enqueued on the stream
 * passed in (NULL = the legacy default stream) and the device-pointer entry
 * points return without synchronising.  The *_host entry points take host
 * arrays, copy them in and out, and return after the result is on the host.
 */
#ifndef SFEMANS_NL_H
#define SFEMANS_NL_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef void *sfnl_stream_t; /* a cudaStream_t */

enum {
  SFNL_OK = 0,
  SFNL_ERR_ARG = -1,         /* null pointer, np < 0, m < 1, k_batch < 1, odd nb_field ... */
  SFNL_ERR_SHAPE = -2,       /* nb_field/nslot not what the product needs, np > nb_procs*bloc_size */
  SFNL_ERR_ALIAS = -3,       /* m_max_pad < m_max, or (fast/split forms) grid too short to dealias */
  SFNL_ERR_UNSUPPORTED = -4, /* size beyond this library's limits, nb_procs != 1 on one GPU */
  SFNL_ERR_CUDA = -5,        /* a CUDA runtime call or kernel launch failed */
  SFNL_ERR_NONFINITE = -6,   /* (check mode) a NaN/Inf was found in the output */
  SFNL_ERR_ALLOC = -7,       /* device or pinned host allocation failed */
  SFNL_ERR_TIMEOUT = -8      /* a split-form kernel gave up a bounded wait on its tensor-core
                                operations, or the FAST MHD bundle on its bulk copies; the outputs of
                                that call are incomplete (reported by the next split-form or FAST
                                MHD bundle call, which share one status word, or at the end of a
                                host-array call) */
};

/* Algorithm of the all-FP64 forms. */
enum {
  SFNL_ALGO_AUTO = 0, /* FAST when the grid dealiases, GRID otherwise */
  SFNL_ALGO_GRID = 1, /* dense DFT on the caller's grid N (reproduces aliasing of short pads) */
  SFNL_ALGO_FAST = 2  /* factored transforms on an internal alias-free grid */
};

/* Products by op code (sfnl_product_f64, sfnl_product_split, sfnl_product_f64_host).
 * Layouts: a, b as listed; out (np, nslot, m) except the tensor layout (3, np, 6, m)
 * of fft_parallel.F90:1552, whose element (k, p, s, n) is at out[k + 3*(p + np*(s + 6*n))]. */
enum {
  SFNL_OP_CROSS = 0,       /* a, b (np, 6, m) -> (np, 6, m)   a x b         (:271-273) */
  SFNL_OP_DOT = 1,         /* a, b (np, 6, m) -> (np, 2, m)   a . b         (:450) */
  SFNL_OP_PROD = 2,        /* a, b (np, 2, m) -> (np, 2, m)   a b           (:617) */
  SFNL_OP_DIV = 3,         /* a, b (np, 2, m) -> (np, 2, m)   a / b         (:786) */
  SFNL_OP_SCALAR_VECT = 4, /* a (np, 6, m), b (np, 2, m) -> (np, 6, m)   b a  (:1150-1153, pb = 1) */
  SFNL_OP_VECT_SCALAR = 5, /* a (np, 6, m), b (np, 2, m) -> (np, 6, m)   a / b (:1154-1157, pb = 2) */
  SFNL_OP_TENSOR = 6,      /* a, b (np, 6, m) -> (3, np, 6, m)   a_k b_l    (:1676-1687) */
  SFNL_OP_TENSION = 7      /* a, b (np, 6, m) -> (3, np, 6, m)   a_k b_l / (|b| + 1e-14) - |b| delta_kl (:1689-1703) */
};
/* The quotients (3, 5) and the tension tensor (7) are not products of two
 * band-limited series: their result depends on the grid, so they run on the
 * caller's grid N = 2*m_max_pad-1 (GRID form) only; FAST and split forms
 * return SFNL_ERR_UNSUPPORTED for them. */

/* Split-precision forms (tensor cores, FP32 accumulation, FP64 recombination). */
enum {
  SFNL_SPLIT_BF16X2 = 2, /* 2 bf16 slices, 3 slice products ("hi/lo") */
  SFNL_SPLIT_BF16X3 = 3  /* 3 bf16 slices, 6 slice products */
};

/* ---------------------------------------------------------------------------
 * FP64 forms, device pointers.
 *   np        number of points (Gauss points or nodes), >= 0
 *   m_max     number of Fourier modes held per point (all modes: one GPU)
 *   m_max_pad zero-padding length; the grid has N = 2*m_max_pad-1 angles
 *             (fft_parallel.F90:183); must be >= m_max
 * ------------------------------------------------------------------------- */

/* FFT_PAR_CROSS_PROD_DCL (fft_parallel.F90:147-328): v1, v2, out are (np, 6, m_max). */
int sfnl_cross_f64(const double *v1, const double *v2, double *out, int64_t np, int m_max, int m_max_pad,
                   sfnl_stream_t stream);
/* FFT_PAR_DOT_PROD_DCL (fft_parallel.F90:330-500): v1, v2 (np, 6, m_max) -> out (np, 2, m_max). */
int sfnl_dot_f64(const double *v1, const double *v2, double *out, int64_t np, int m_max, int m_max_pad,
                 sfnl_stream_t stream);
/* FFT_PAR_PROD_DCL (fft_parallel.F90:502-665): c1, c2, out are (np, 2, m_max). */
int sfnl_prod_f64(const double *c1, const double *c2, double *out, int64_t np, int m_max, int m_max_pad,
                  sfnl_stream_t stream);

/* Any product by op code (SFNL_OP_*) with an explicit algorithm and grid length.
 * n_theta = 0 selects N = 2*m_max_pad-1. */
int sfnl_product_f64(int op, const double *a, const double *b, double *out, int64_t np, int m_max,
                     int m_max_pad, int n_theta, int algo, sfnl_stream_t stream);

/* FFT_PAR_DIV_DCL (fft_parallel.F90:667-830): c1, c2, out are (np, 2, m_max); out = T[S c1 / S c2]. */
int sfnl_div_f64(const double *c1, const double *c2, double *out, int64_t np, int m_max, int m_max_pad,
                 sfnl_stream_t stream);
/* FFT_SCALAR_VECT_DCL (fft_parallel.F90:1021-1220): v, out (np, 6, m_max), s (np, 2, m_max);
 * pb = 1: out = T[S s * S v]; pb = 2: out = T[S v / S s]; other pb: SFNL_ERR_ARG. */
int sfnl_scalar_vect_f64(const double *v, const double *s, double *out, int64_t np, int m_max, int m_max_pad, int pb,
                         sfnl_stream_t stream);
/* FFT_TENSOR_DCL (fft_parallel.F90:1543-1796): v1, v2 (np, 6, m_max) -> out (3, np, 6, m_max);
 * tension != 0 selects the opt_tension form. */
int sfnl_tensor_f64(const double *v1, const double *v2, double *out, int64_t np, int m_max, int m_max_pad,
                    int tension, sfnl_stream_t stream);

/* FFT_PAR_REAL (fft_parallel.F90:28-145): v (np, nslot, m_max) -> out (n_theta, nslot/2, np), the
 * value of every field (slot pair) at theta_j = 2 pi j / n_theta, angle fastest.  The reference grid is
 * n_theta = sfnl_fft_par_real_planes(m_max, opt_nb_plane); n_theta < 2*m_max-1 is SFNL_ERR_ALIAS. */
int sfnl_real_f64(const double *v, double *out, int64_t np, int nslot, int m_max, int n_theta, sfnl_stream_t stream);
/* FFT_MAX_VEL_DCL (fft_parallel.F90:1426-1541): *vmax (one double in device memory, written on `stream`)
 * = the maximum over the points and the 2*m_max_pad-1 angles of |v|: the first 3-vector's length when
 * nslot == 6, |first field| otherwise (:1527-1532).  A NaN in the field propagates to the result. */
int sfnl_max_vel_f64(const double *v, double *vmax, int64_t np, int nslot, int m_max, int m_max_pad,
                     sfnl_stream_t stream);

/* The MHD nonlinear bundle in one launch, each term with the semantics of
 * the reference routine that computes it today:
 *   uxw   = u x w     (FFT_PAR_CROSS_PROD_DCL, subroutine_ns_with_velocity.F90:627 passes (RotV, W))
 *   uxb   = u x b     (update_maxwell_with_B.F90:555)
 *   jxb   = j x b     (subroutine_ns_with_velocity.F90:719, J = curl H)
 *   ugradt= u . gradt (FFT_PAR_DOT_PROD_DCL, subroutine_temperature_with_T.F90:341)
 * u, w, b, j, gradt, uxw, uxb, jxb: (np, 6, m_max); ugradt: (np, 2, m_max). */
int sfnl_bundle_mhd_f64(const double *u, const double *w, const double *b, const double *j, const double *gradt,
                        double *uxw, double *uxb, double *jxb, double *ugradt, int64_t np, int m_max,
                        int m_max_pad, int algo, sfnl_stream_t stream);

/* ---------------------------------------------------------------------------
 * The Navier-Stokes caller of the cross product, smb_cross_prod_gauss_sft_par
 * (SOURCES/SIMULATION/subroutine_ns_with_velocity.F90:512-629): from the nodal
 * velocity it builds, at every Gauss point and for every mode, the velocity W, the
 * curl RotV in cylindrical coordinates (mode list_mode[i]) and, with precession, the
 * rotation Om, and returns out = (RotV + 2 Om) x W (FFT_PAR_CROSS_PROD_DCL).
 *   v, omega   (np_nodes, 6, nmod) nodal coefficients; omega NULL: no precession
 *   jj         (n_w, me) int, 1-based node numbers of each element (mesh%jj); numbers
 *              outside 1..np_nodes are clamped on the device (the host entry rejects them)
 *   ww         (n_w, l_G) basis values at the Gauss points (mesh%gauss%ww)
 *   dw         (2, n_w, l_G, me) basis (d/dr, d/dz) on each element (mesh%gauss%dw)
 *   rr         (2, np_nodes) node coordinates (r, z) (mesh%rr)
 *   list_mode  (nmod) int, the Fourier mode numbers
 *   out        (l_G*me, 6, nmod), Gauss points element by element
 *   m_max_pad  <= 0: 3*nmod/2, the caller's choice (:625)
 *   work       device buffer of 12*l_G*me*nmod doubles for RotV and W, or NULL: a buffer
 *              owned by the library (one per device, grown with cudaMalloc when too small;
 *              calls that overlap on the GPU then share it and race).  For nmod <= 96 RotV
 *              and W are built inside the product kernel (the third-fold kernel at nmod = 64 on
 *              P2 elements, the general FAST kernel otherwise) and work holds node-major copies
 *              of the nodal fields instead (6*np_nodes*nmod doubles per field, v and omega),
 *              when they fit in it; larger nmod write RotV and W to work and read them back
 * ------------------------------------------------------------------------- */
int sfnl_cross_gauss_f64(const double *v, const int *jj, const double *ww, const double *dw, const double *rr,
                         const int *list_mode, const double *omega, double *out, int np_nodes, int me, int n_w,
                         int l_G, int nmod, int m_max_pad, double *work, sfnl_stream_t stream);
/* The same on host arrays (k_d = SIZE(mesh%rr,1) must be 2; nb_procs must be 1), for the Fortran shim. */
int sfnl_smb_cross_prod_gauss(const double *V_in, const int *jj, const double *ww, const double *dw, const double *rr,
                              int k_d, const int *list_mode, const double *omega, double *V_out, int np_nodes, int me,
                              int n_w, int l_G, int nmod, int nb_procs);

/* The Lorentz-force caller, smb_CurlH_cross_B_gauss_sft_par (SOURCES/SIMULATION/
 * subroutine_ns_with_m.F90:788-883): out = (curl h) x b at the Gauss points from two
 * nodal fields h (the magnetic field H) and b (the induction B), both (np_nodes, 6, nmod);
 * no precession term.  Mesh arrays, list_mode, out and m_max_pad as above; work: 12*l_G*me*nmod
 * doubles or NULL. */
int sfnl_curlh_cross_b_gauss_f64(const double *h, const double *b, const int *jj, const double *ww, const double *dw,
                                 const double *rr, const int *list_mode, double *out, int np_nodes, int me, int n_w,
                                 int l_G, int nmod, int m_max_pad, double *work, sfnl_stream_t stream);
/* The same on host arrays (V_in = H, W_in = B; k_d must be 2, nb_procs 1). */
int sfnl_smb_curlh_cross_b_gauss(const double *V_in, const double *W_in, const int *jj, const double *ww,
                                 const double *dw, const double *rr, int k_d, const int *list_mode, double *V_out,
                                 int np_nodes, int me, int n_w, int l_G, int nmod, int nb_procs);

/* The scalar-advection callers, smb_ugradc_gauss_fft_par of the level set
 * (SOURCES/SIMULATION/subroutine_level_set.F90:434-534: conservative = 0, heat = NULL), of the
 * temperature (subroutine_temperature_with_T.F90:247-350: conservative = 1, heat = the
 * volumetric heat capacity of each element) and smb_ugradc_gauss_fft_par_conc of the
 * concentration (subroutine_concentration.F90:243-341: conservative = 1, heat = NULL):
 *   out (l_G*me, 2, nmod) = (heat grad c) . u  [+ div u (heat c) when conservative]
 * with FFT_PAR_DOT_PROD_DCL (+ FFT_PAR_PROD_DCL, the two analyses added, computed here as one
 * program analysed once).
 *   v     (np_nodes, 6, nmod) nodal velocity;  c (np_nodes, 2, nmod) nodal scalar
 *   heat  (me) per-element factor of grad c and c, or NULL (factor 1)
 *   work  16*l_G*me*nmod doubles (12 when conservative == 0) or NULL.  For nmod <= 96 the
 *         operands are built inside the product kernel and work holds node-major copies of
 *         v and c (8*np_nodes*nmod doubles) instead, when they fit in it. */
int sfnl_ugradc_gauss_f64(const double *v, const double *c, const double *heat, int conservative, const int *jj,
                          const double *ww, const double *dw, const double *rr, const int *list_mode, double *out,
                          int np_nodes, int me, int n_w, int l_G, int nmod, int m_max_pad, double *work,
                          sfnl_stream_t stream);
/* The same on host arrays (k_d must be 2, nb_procs 1). */
int sfnl_smb_ugradc_gauss(const double *V_in, const double *c_in, const double *heat_capa, int conservative,
                          const int *jj, const double *ww, const double *dw, const double *rr, int k_d,
                          const int *list_mode, double *c_out, int np_nodes, int me, int n_w, int l_G, int nmod,
                          int nb_procs);

/* The Gauss-point operands alone (the loops before the FFT call in the three callers above), for
 * callers that run the product themselves, e.g. over a mode-distributed communicator with
 * sfemans_b200.parallel.  Device arrays; every output (l_G*me, nslot, nmod) Fortran:
 *   SFNL_GAUSS_NS       v (+ omega, may be NULL)  o0 = RotV + 2 Om, o1 = W           (6 slots each)
 *   SFNL_GAUSS_LORENTZ  v = H, v2 = B            o0 = curl H, o1 = B at the points  (6 slots each)
 *   SFNL_GAUSS_ADVECT   v = u, v2 = c, heat      o0 = heat grad c, o1 = W (6 slots); conservative: o2 =
 *                       div u, o3 = heat c (2 slots each), else o2, o3 ignored.  */
enum { SFNL_GAUSS_NS = 0, SFNL_GAUSS_LORENTZ = 1, SFNL_GAUSS_ADVECT = 2 };
int sfnl_gauss_operands_f64(int kind, const double *v, const double *v2, const double *omega, const double *heat,
                            int conservative, const int *jj, const double *ww, const double *dw, const double *rr,
                            const int *list_mode, double *o0, double *o1, double *o2, double *o3, int np_nodes,
                            int me, int n_w, int l_G, int nmod, sfnl_stream_t stream);

/* ---------------------------------------------------------------------------
 * Linearised cross product N(u, w) = u x w about a base state (u, w).
 * New capability: the reference's LightKrylov operator binds rmatvec to the
 * forward map (LIGHTKRYLOV_OBJECTS/exponential_propagator.F90:61-62).
 *   JVP  tan (np, 12, m, k): slots 0-5 = du, 6-11 = dw;  out (np, 6, m, k) = du x w + u x dw
 *   VJP  cot (np, 6, m, k) -> out (np, 12, m, k) = J^T cot, the transpose for the
 *        plain Euclidean inner product of the coefficient arrays, so that
 *        <J v, c> = <v, J^T c> exactly in exact arithmetic.
 * u, w: (np, 6, m) shared by all k_batch tangents.  Beyond m = 96 (the
 * two-kernel form) the base state is synthesised once per point chunk and the
 * tangents in one launch per chunk; the grid-value workspace then grows to
 * hold every tangent of a chunk of at least 4096 points, up to 8 GiB or a
 * quarter of the free device memory (kept until sfnl_finalize).
 * ------------------------------------------------------------------------- */
int sfnl_cross_jvp_f64(const double *u, const double *w, const double *tan, double *out, int64_t np, int m_max,
                       int m_max_pad, int k_batch, sfnl_stream_t stream);
int sfnl_cross_vjp_f64(const double *u, const double *w, const double *cot, double *out, int64_t np, int m_max,
                       int m_max_pad, int k_batch, sfnl_stream_t stream);

/* Linearised pair (u x w, u x b) about (u, w, b), sharing u:
 *   JVP  tan (np, 18, m, k) = (du, dw, db) -> out (np, 12, m, k) = (du x w + u x dw, du x b + u x db)
 *   VJP  cot (np, 12, m, k) -> out (np, 18, m, k). */
int sfnl_mhd_jvp_f64(const double *u, const double *w, const double *b, const double *tan, double *out, int64_t np,
                     int m_max, int m_max_pad, int k_batch, sfnl_stream_t stream);
int sfnl_mhd_vjp_f64(const double *u, const double *w, const double *b, const double *cot, double *out, int64_t np,
                     int m_max, int m_max_pad, int k_batch, sfnl_stream_t stream);

/* The four linearised programs on HOST arrays (same layouts and meaning; the
 * points are copied through the device in chunks, as by the *_host entries).
 * For operators applied from host code, e.g. a LightKrylov linear operator
 * (sfemans_b200/fortran/nl_linop.F90) whose matvec is the JVP and whose
 * rmatvec is the VJP. */
int sfnl_cross_jvp_host(const double *u, const double *w, const double *tan, double *out, int64_t np, int m_max,
                        int m_max_pad, int k_batch);
int sfnl_cross_vjp_host(const double *u, const double *w, const double *cot, double *out, int64_t np, int m_max,
                        int m_max_pad, int k_batch);
int sfnl_mhd_jvp_host(const double *u, const double *w, const double *b, const double *tan, double *out, int64_t np,
                      int m_max, int m_max_pad, int k_batch);
int sfnl_mhd_vjp_host(const double *u, const double *w, const double *b, const double *cot, double *out, int64_t np,
                      int m_max, int m_max_pad, int k_batch);

/* ---------------------------------------------------------------------------
 * Split-precision forms: operands split into bf16 slices with a per-point
 * power-of-two scale, DFT contractions on the tcgen05 tensor cores with FP32
 * accumulation in TMEM, FP64 recombination, pointwise product and final
 * truncation.  split = SFNL_SPLIT_BF16X2 or SFNL_SPLIT_BF16X3.
 * ------------------------------------------------------------------------- */
int sfnl_product_split(int op, const double *a, const double *b, double *out, int64_t np, int m_max, int m_max_pad,
                       int split, sfnl_stream_t stream);
int sfnl_bundle_mhd_split(const double *u, const double *w, const double *b, const double *j, const double *gradt,
                          double *uxw, double *uxb, double *jxb, double *ugradt, int64_t np, int m_max,
                          int m_max_pad, int split, sfnl_stream_t stream);
int sfnl_mhd_jvp_split(const double *u, const double *w, const double *b, const double *tan, double *out,
                       int64_t np, int m_max, int m_max_pad, int k_batch, int split, sfnl_stream_t stream);
int sfnl_mhd_vjp_split(const double *u, const double *w, const double *b, const double *cot, double *out,
                       int64_t np, int m_max, int m_max_pad, int k_batch, int split, sfnl_stream_t stream);

/* ---------------------------------------------------------------------------
 * Reference-signature entry points on HOST arrays, for the ISO_C_BINDING
 * shim.  Arguments are those of fft_parallel.F90:147 / :330 / :502:
 *   np, nb_field, m_max_c = SIZE(V1_in,1..3); nb_procs, bloc_size, m_max_pad as
 *   passed by the caller; temps (may be NULL) = the optional REAL(8) temps(3):
 *   zeroed (fft_parallel.F90:179), then temps[0] += device seconds of the
 *   host<->device copies (where the reference counts its MPI_ALLTOALLs),
 *   temps[1] += device seconds of the kernels (its FFTs and product), temps[2]
 *   stays 0 (no repacking); sums over point chunks that overlap on streams.
 * One GPU holds all modes, so nb_procs must be 1 (SFNL_ERR_UNSUPPORTED
 * otherwise); bloc_size is checked (np <= nb_procs*bloc_size, the reference's
 * buffer bound) and otherwise unused: there are no dummy points.
 * ------------------------------------------------------------------------- */
int sfnl_fft_par_cross_prod_dcl(const double *V1_in, const double *V2_in, double *V_out, int np, int nb_field,
                                int m_max_c, int nb_procs, int bloc_size, int m_max_pad, double *temps);
int sfnl_fft_par_dot_prod_dcl(const double *V1_in, const double *V2_in, double *c_out, int np, int nb_field,
                              int m_max_c, int nb_procs, int bloc_size, int m_max_pad, double *temps);
int sfnl_fft_par_prod_dcl(const double *c1_in, const double *c2_in, double *c_out, int np, int m_max_c,
                          int nb_procs, int bloc_size, int m_max_pad, double *temps);
/* fft_parallel.F90:667 (FFT_PAR_DIV_DCL): arguments as sfnl_fft_par_prod_dcl. */
int sfnl_fft_par_div_dcl(const double *c1_in, const double *c2_in, double *c_out, int np, int m_max_c,
                         int nb_procs, int bloc_size, int m_max_pad, double *temps);
/* fft_parallel.F90:1021 (FFT_SCALAR_VECT_DCL): nb_field1 = SIZE(V1_in,2) must be 6 and
 * nb_field2 = SIZE(V2_in,2) 2 (SFNL_ERR_SHAPE, the reference's error_petsc at :1163);
 * pb outside {1, 2}: SFNL_ERR_ARG (:1160). */
int sfnl_fft_scalar_vect_dcl(const double *V1_in, const double *V2_in, double *V_out, int pb, int np, int nb_field1,
                             int nb_field2, int m_max_c, int nb_procs, int bloc_size, int m_max_pad, double *temps);
/* fft_parallel.F90:1543 (FFT_TENSOR_DCL): V_out (3, np, 6, m_max_c).  opt_tension < 0: argument
 * absent (plain tensor); > 0: present and .TRUE. (tension form); 0: present and .FALSE., which the
 * reference rejects (error_petsc at :1705): SFNL_ERR_ARG.  nb_field != 6: SFNL_ERR_SHAPE. */
int sfnl_fft_tensor_dcl(const double *V1_in, const double *V2_in, double *V_out, int np, int nb_field, int m_max_c,
                        int nb_procs, int bloc_size, int m_max_pad, int opt_tension, double *temps);

/* fft_parallel.F90:71-80: the grid length of FFT_PAR_REAL, 2*m_max_pad-1 with m_max_pad =
 * (opt_nb_plane+1)/2 when opt_nb_plane > 2*m_max-1, else m_max (opt_nb_plane <= 0: argument absent). */
int sfnl_fft_par_real_planes(int m_max, int opt_nb_plane);
/* fft_parallel.F90:28 (FFT_PAR_REAL): V_out, allocated by the caller, holds
 * N * (nb_field/2) * np doubles, N = sfnl_fft_par_real_planes(m_max_c, opt_nb_plane): with one rank
 * every point is local (the reference's bloc_size = np/nb_procs).  nb_procs must be 1. */
int sfnl_fft_par_real(const double *V1_in, double *V_out, int np, int nb_field, int m_max_c, int nb_procs,
                      int opt_nb_plane);
/* fft_parallel.F90:1426 (FFT_MAX_VEL_DCL): *V_out (host) = the maximum of |V1_in| on the
 * 2*m_max_pad-1 angles; the per-point maxima come back from the GPU and are reduced on the host. */
int sfnl_fft_max_vel_dcl(const double *V1_in, double *V_out, int np, int nb_field, int m_max_c, int nb_procs,
                         int bloc_size, int m_max_pad);

/* Host-array variants of the device entry points (copy in, compute, copy out). */
int sfnl_product_f64_host(int op, const double *a, const double *b, double *out, int64_t np, int m_max,
                          int m_max_pad, int algo);
int sfnl_bundle_mhd_host(const double *u, const double *w, const double *b, const double *j, const double *gradt,
                         double *uxw, double *uxb, double *jxb, double *ugradt, int64_t np, int m_max,
                         int m_max_pad, int form /* 0 = FP64, 2/3 = split */);

/* ---------------------------------------------------------------------------
 * No-allocation variant.  No counterpart in the reference.
 * The FAST FP64 cross product (same arguments and result as sfnl_cross_f64 on
 * a dealiasing pad) for callers that must not allocate device memory: codes
 * whose GPU memory is owned by their own pool or by another framework, and
 * callers that cannot afford cudaMalloc's implicit device synchronisation in
 * their time loop.  Its DFT tables live in a fixed array inside the library
 * (144 KiB of static device memory on every GPU that loads the library, held
 * until the process exits), so m_max is limited to 64 (SFNL_ERR_UNSUPPORTED
 * above).  The first call on a device, and any call whose m_max differs from
 * the previous call's, looks up that array and rewrites it on `stream`; make
 * that first call before any stream capture.  All calls share the array:
 * calls that overlap on the GPU (different streams) race on it when their
 * m_max differs or while a rewrite is in flight.
 * ------------------------------------------------------------------------- */
int sfnl_cross_f64_noalloc(const double *v1, const double *v2, double *out, int64_t np, int m_max, int m_max_pad,
                           sfnl_stream_t stream);

/* ---------------------------------------------------------------------------
 * Fourier-mode-distributed callers, nb_procs > 1 (replace the body of the
 * reference routines of fft_parallel.F90:147 / :330 / :502 / :667 / :1021 /
 * :1543 between and around its two MPI_ALLTOALLs, :205-217 and :306-324).
 * Every rank holds m_max_c modes of np points; block q = points
 * [q*bloc_size, (q+1)*bloc_size).  The caller keeps its MPI:
 *   pack_modes(V1) -> send1, pack_modes(V2) -> send2   (per peer q: block q of my modes)
 *   MPI_ALLTOALL(send1 -> recv1), MPI_ALLTOALL(send2 -> recv2)
 *   fft_par_block(op, recv1, recv2 -> back)            (my block, all modes, on the GPU)
 *   MPI_ALLTOALL(back -> got)
 *   unpack_modes(got) -> V_out                          (my modes of all points)
 * Buffers hold nb_procs peers of bloc_size*nslot*m_max_c*ew doubles, ordered
 * [peer][mode][slot][point][e]; ew = 3 only for the output of the tensor
 * products (V_out(3, np, 6, m)), else 1.  op: SFNL_OP_*; its slot counts are
 * those of sfnl_product_f64.  temps as in the reference-signature entries.
 * ------------------------------------------------------------------------- */
int sfnl_fft_par_pack_modes(const double *V, double *send, int np, int nslot, int m_max_c, int nb_procs, int bloc_size,
                            int ew);
int sfnl_fft_par_block(int op, const double *recv1, const double *recv2, double *back, int bloc_size, int m_max_c,
                       int nb_procs, int m_max_pad, double *temps);
int sfnl_fft_par_unpack_modes(const double *got, double *V_out, int np, int nslot, int m_max_c, int nb_procs,
                              int bloc_size, int ew);

/* ---------------------------------------------------------------------------
 * Library state.
 * ------------------------------------------------------------------------- */
const char *sfnl_last_error(void); /* message of the last failing call on this thread */
const char *sfnl_version(void);
int sfnl_set_check_finite(int on); /* 1: scan outputs for NaN/Inf after each call (synchronises) */
/* Releases cached device tables, workspaces and staging buffers, and forgets the
 * per-device set-up of sfnl_cross_f64_noalloc.  Call it before cudaDeviceReset or
 * any other teardown of a device's primary context while the library stays
 * loaded: cached device addresses do not survive the context. */
int sfnl_finalize(void);
/* Diagnostic (no counterpart in the reference): FP64 throughput of the current
 * device in TFLOP/s for mma.sync.m8n8k4.f64 and for FP64 FMAs, each measured
 * alone with CUDA events (long register-only chains, every SM busy, best of
 * five launches): the compute roofline of the all-FP64 forms. */
int sfnl_probe_fp64_tflops(double *dmma_tflops, double *dfma_tflops);
/* Kernel of the FAST MHD bundle at m_max = 64 (sfnl_bundle_mhd_f64 and the
 * host entry), process-wide: SFNL_BUNDLE_RESIDUE (default) splits the
 * 192-angle grid into its three residue classes (64-angle grids, half the
 * FP64 tensor-core work); SFNL_BUNDLE_THIRD_FOLD runs the single 192-angle
 * transform.  Both give the same truncated products (to rounding).  Returns
 * the previous kind, or SFNL_ERR_ARG for another value. */
enum { SFNL_BUNDLE_RESIDUE = 0, SFNL_BUNDLE_THIRD_FOLD = 1 };
int sfnl_set_bundle_kernel(int kind);
/* Host-side fault injection for tests of the error path: marks the split-form
 * status word as a kernel does when a bounded wait on its tensor-core
 * operations gives up (no GPU work is involved).  The next split-form call
 * returns SFNL_ERR_TIMEOUT and clears the word, as after a real timeout. */
int sfnl_test_inject_timeout(void);
/* Test hook: bounds the two workspaces of the large-m FAST form (grid values; the residues' coefficients and
 * sums) to `bytes` so that small calls run many point chunks and batch groups, the path very large calls
 * take; 0 restores the production bounds.  Process-wide.  bytes < 0: SFNL_ERR_ARG. */
int sfnl_test_large_workspace_cap(int64_t bytes);
/* Test hook: the number of residue classes (3, 6 or 12) into which the large-m FAST form splits its
 * 3m-angle grid, where the split gives whole quadrant-tile pairs (3m/R a multiple of 64, at most 512), else
 * the whole grid; 0 restores the automatic choice (from m = 256: 6 where it fits, else 3; the whole grid
 * below m = 256).  Every choice gives the same products to rounding.  Process-wide.  Other values:
 * SFNL_ERR_ARG. */
int sfnl_test_large_residues(int R);
/* Device-timed seconds of the last host-array call of this thread (the *_host,
 * sfnl_fft_* and sfnl_smb_* entries): [0] host<->device copies, [1] kernels,
 * [2] 0 (nothing is repacked).  Each is a sum over the call's point chunks; the
 * chunks run on several streams, so [0] + [1] may exceed the call's wall time.
 * The same two sums are added to temps(1) and temps(2) where a temps argument
 * is passed. */
int sfnl_last_host_timing(double *seconds3);

#ifdef __cplusplus
}
#endif
#endif /* SFEMANS_NL_H */
