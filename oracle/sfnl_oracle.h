/* sfnl_oracle.h -- CPU oracle (test infrastructure only; see sfnl_oracle.c). */
#ifndef SFNL_ORACLE_H
#define SFNL_ORACLE_H
#include <stdint.h>
#ifdef __cplusplus
extern "C" {
#endif

enum { ORC_CROSS = 0, ORC_DOT = 1, ORC_PROD = 2, ORC_DIV = 3, ORC_SVECT = 4, ORC_SVDIV = 5, ORC_TENSOR = 6, ORC_TENSION = 7 };

/* Restatement of FFT_PAR_{CROSS_PROD,DOT_PROD,PROD}_DCL (fft_parallel.F90:147-665).
 * V1, V2: global arrays (np, nb_field, m_max_c*nb_procs), Fortran order; rank r
 * owns modes [r*m_max_c, (r+1)*m_max_c).  Vout: (np, 6 | 2, m_max_c*nb_procs).
 * Returns 0, or <0 for arguments the reference rejects or cannot handle. */
int orc_fft_par_dcl(int op, const double *V1, const double *V2, double *Vout, int np, int nb_field,
                    int m_max_c, int nb_procs, int bloc_size, int m_max_pad);
/* Same with an explicit grid length N (the reference uses N = 2*m_max_pad-1). */
int orc_fft_par_dcl_n(int op, const double *V1, const double *V2, double *Vout, int np, int nb_field,
                      int m_max_c, int nb_procs, int bloc_size, int m_max_pad, int N);

/* Any of the routines on inputs with nsl1 / nsl2 slots (scalar x vector: 6 and 2). Tensor outputs are
 * V_out(3, np, 6, m_max) (fft_parallel.F90:1552); the others V_out(np, 2*nout, m_max). */
int orc_apply_n(int op, const double *V1, int nsl1, const double *V2, int nsl2, double *Vout, int np,
                int m_max_c, int nb_procs, int bloc_size, int m_max_pad, int N);

/* FFT_PAR_REAL (fft_parallel.F90:28-145): values of every field at the N angles 2*pi*j/N, N =
 * orc_fft_par_real_planes(m_max, opt_nb_plane) (opt_nb_plane <= 0: absent).  Vout(N, nsl/2, np): the
 * ranks' V_out(N, nsl/2, np/nb_procs) one after the other (rank r holds points r*np/nb_procs ..). */
int orc_fft_par_real_planes(int m_max, int opt_nb_plane);
int orc_fft_par_real(const double *V1, int nsl, int np, int m_max_c, int nb_procs, int opt_nb_plane, double *Vout);
/* FFT_MAX_VEL_DCL (fft_parallel.F90:1426-1541): the maximum over points and the N = 2*m_max_pad-1
 * angles of |V1| (first 3-vector for nsl == 6, |first field| otherwise). */
int orc_fft_max_vel(const double *V1, int nsl, int np, int m_max_c, int nb_procs, int bloc_size, int m_max_pad,
                    double *vmax);
/* smb_cross_prod_gauss_sft_par (subroutine_ns_with_velocity.F90:512-629): W, RotV (+2 Om) at the Gauss
 * points of a P-k mesh from nodal V, then RotV x W.  jj 1-based (n_w, me); ww (n_w, l_G); dw (2, n_w,
 * l_G, me); rr (2, np_nodes); V, omega (np_nodes, 6, nmod), omega may be NULL; Vout (l_G*me, 6, nmod);
 * RotV_out / W_out (same shape) may be NULL. */
int orc_cross_gauss(const double *V, const int *jj, const double *ww, const double *dw, const double *rr,
                    const int *list_mode, const double *omega, int np_nodes, int me, int n_w, int l_G, int nmod,
                    double *Vout, double *RotV_out, double *W_out);
/* smb_CurlH_cross_B_gauss_sft_par (subroutine_ns_with_m.F90:788-883): (curl H) x B at the Gauss points
 * from nodal H, B (np_nodes, 6, nmod); outputs as orc_cross_gauss. */
int orc_curlh_cross_b_gauss(const double *H, const double *B, const int *jj, const double *ww, const double *dw,
                            const double *rr, const int *list_mode, int np_nodes, int me, int n_w, int l_G, int nmod,
                            double *Vout, double *RotV_out, double *W_out);
/* smb_ugradc_gauss_fft_par (subroutine_level_set.F90:434-534, subroutine_temperature_with_T.F90:247-350)
 * and smb_ugradc_gauss_fft_par_conc (subroutine_concentration.F90:243-341): (heat grad c) . u
 * [+ div u (heat c) when conservative]; V (np_nodes, 6, nmod), C (np_nodes, 2, nmod), heat (me) or NULL;
 * Vout (l_G*me, 2, nmod); operand outputs Gradc, W (l_G*me, 6, nmod), Div, Cg (l_G*me, 2, nmod) or NULL. */
int orc_ugradc_gauss(const double *V, const double *C, const double *heat, int conservative, const int *jj,
                     const double *ww, const double *dw, const double *rr, const int *list_mode, int np_nodes, int me,
                     int n_w, int l_G, int nmod, double *Vout, double *Gradc_out, double *W_out, double *Div_out,
                     double *Cg_out);

#ifdef __cplusplus
}
#endif
#endif
