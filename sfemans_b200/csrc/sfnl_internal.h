// sfnl_internal.h -- shared host-side helpers of the library (not installed).
#pragma once
#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>
#include <vector>

#include "../../include/sfemans_nl.h"

namespace sfnl {

struct ProgArgs;

// Records the message for sfnl_last_error() on this thread and returns code.
int set_error(int code, const char *msg);
// Checks cudaGetLastError() after a launch; records "<what>: <cuda error>".
int check_launch(const char *what);
// Number of SMs of the current device (cached per device).
int num_sms();

// Kernel families.
int launch_grid(const ProgArgs &a, cudaStream_t st);   // sfnl_grid.cu
int launch_fast(const ProgArgs &a, cudaStream_t st);   // sfnl_fast.cu
int launch_bundle_r3(const ProgArgs &a, cudaStream_t st);  // sfnl_r3.cu: the MHD bundle at m = 64
void r3_release_tables();                               // sfnl_r3.cu
int bundle_kernel();                                    // sfnl_capi.cu: SFNL_BUNDLE_* in use
bool fast_supported(int op, int m, int N_int);          // sfnl_fast.cu
int fast_grid_length(int m);                            // sfnl_fast.cu
void fast_release_tables();                             // sfnl_fast.cu
void large_release_workspaces();                        // sfnl_large.cu: the grid-value workspaces
void large_test_workspace_cap(size_t bytes);            // sfnl_large.cu: tests' workspace bound (0: none)
void large_test_residues(int R);                        // sfnl_large.cu: tests' residue classes (0: automatic)
int launch_split(const ProgArgs &a, int split, cudaStream_t st);  // sfnl_split.cu
void split_release_tables();                            // sfnl_split.cu
int split_take_status();     // 1 if a split kernel gave up a bounded wait since the last call; clears it
int split_inject_timeout();  // sets that status from the host (tests of the error path)
int wait_status_word(int **dev);  // that status word's device address (kernels with bounded waits set it)
// Synthesis only (sfnl_synth.cu): out (N, nslot/2, np); vmax a zeroed device double that receives the
// maximum of |v|; pmax (np) the maximum of |v| of each point.
int launch_real(const double *v, double *out, int64_t np, int nslot, int m, int N, cudaStream_t st);
int launch_max_vel(const double *v, double *vmax, int64_t np, int nslot, int m, int N, cudaStream_t st);
int launch_point_max_vel(const double *v, double *pmax, int64_t np, int nslot, int m, int N, cudaStream_t st);

// Operands of the Gauss-point callers (sfnl_gauss.cu): device arrays of the mesh (jj 1-based (n_w, me),
// ww (n_w, l_G), dw (2, n_w, l_G, me), rr (2, np_nodes)), the nodal vector field v (np_nodes, 6, nmod),
// the precession rotation omega (same shape, GK_NS, may be null), the second nodal field v2 (GK_LORENTZ:
// B (np_nodes, 6, nmod); GK_ADVECT: the scalar c (np_nodes, 2, nmod)), the heat capacity of each element
// heat (me, GK_ADVECT, may be null) and the modes list_mode (nmod).
enum { GK_NS = 0, GK_LORENTZ = 1, GK_ADVECT = 2 };
struct GaussArgs {
  const double *v, *omega, *ww, *dw, *rr;
  const int *jj, *list_mode;
  int np_nodes, me, n_w, l_G, nmod;
  const double *v2, *heat;
};
// Outputs, each (l_G*me, nslot, nmod): GK_NS o0 = RotV + 2 Om, o1 = W (6 slots); GK_LORENTZ o0 = curl v,
// o1 = v2 (6 slots); GK_ADVECT o0 = Gradc, o1 = W (6 slots), o2 = Div, o3 = Cgauss (2 slots; both
// null: no conservative term).
int launch_gauss_eval(const GaussArgs &a, int kind, double *o0, double *o1, double *o2, double *o3, cudaStream_t st);
// Node-major copy of a nodal field (sfnl_gauss.cu): vt (np_nodes, nslot, m) with vt[node*nslot*m + k*m + i] =
// v[node + np_nodes*(k + nslot i)].
int launch_nodal_transpose(const double *v, double *vt, int np_nodes, int m, cudaStream_t st, int nslot = 6);
// The curl callers (GK_NS, GK_LORENTZ) in one kernel with the FAST cross product (sfnl_fast.cu): the
// operands are built in the product kernel's staging from node-major nodal fields (ga.v, ga.v2,
// ga.omega as written by launch_nodal_transpose); out (l_G*me, 6, m).  m = 64 and P2 elements (n_w = 6) only.
bool gauss_cross_fused_supported(int m, int n_w);
int launch_gauss_cross_fused(const GaussArgs &ga, int kind, double *out, int64_t ng, int m, cudaStream_t st);
// The advection callers (GK_ADVECT) the same way: ga.v the node-major velocity (np_nodes, 6, m), ga.v2 the
// node-major scalar (np_nodes, 2, m), ga.heat per element or null; out (l_G*me, 2, m).  m = 64, n_w = 6.
int launch_gauss_advect_fused(const GaussArgs &ga, bool conservative, double *out, int64_t ng, int m,
                              cudaStream_t st);
// Every caller at the other m that the fused FAST kernels serve (any n_w): the operands staged from the
// node-major nodal fields (stride m) by the general FAST kernel.  out: (l_G*me, 6, m) for the curl
// callers, (l_G*me, 2, m) for the advection callers.
bool gauss_general_fused_supported(int kind, bool conservative, int m);
int launch_gauss_general_fused(const GaussArgs &ga, int kind, bool conservative, double *out, int64_t ng, int m,
                               cudaStream_t st);

// Elementary programs: cross (6 -> 3), dot (6 -> 1), product (2 -> 1),
// scalar x vector (4 -> 3) and tensor (6 -> 9).  Every bilinear program of
// sfnl_ops.cuh is a sequence of them on one stream (the bundle is four, a
// linearised cross product two or four, accumulating where a term adds to an
// earlier one).
enum { EK_CROSS = 0, EK_DOT = 1, EK_PROD = 2, EK_SVECT = 3, EK_TENSOR = 4,
       EK_ADVECT = 5,    // g . w + d c (8 -> 1): the fused conservative advection callers only
       EK_CROSS2 = 6 };  // a x b + c x d (12 -> 3): the linearised cross product, in two passes
struct Elem {
  int ek;
  int in[12];    // field indices into ProgArgs.in
  int out[9];    // indices into ProgArgs.out
  unsigned adj;  // bit f: operand f is a cotangent (synthesised with the analysis weights)
  int acc;       // 1: add to the output instead of overwriting it
};
// fuse: which sums of two cross products a x b + c x d run as one EK_CROSS2 program of the generic FAST kernel
// instead of two launches (kFuseJvp: the JVPs; kFuseVjpSum: w x c1 + b x c2 of the MHD VJP)
enum { kFuseJvp = 1, kFuseVjpSum = 2 };
int decompose_program(int op, std::vector<Elem> &seq, int fuse = 0);  // sfnl_fast.cu
bool split_supported(int op, int m);                    // sfnl_split.cu

}  // namespace sfnl
