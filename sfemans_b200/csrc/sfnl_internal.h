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
bool fast_supported(int op, int m, int N_int);          // sfnl_fast.cu
int fast_grid_length(int m);                            // sfnl_fast.cu
void fast_release_tables();                             // sfnl_fast.cu
int launch_split(const ProgArgs &a, int split, cudaStream_t st);  // sfnl_split.cu
void split_release_tables();                            // sfnl_split.cu
// Synthesis only (sfnl_synth.cu): out (N, nslot/2, np); vmax a zeroed device double that receives the
// maximum of |v|; pmax (np) the maximum of |v| of each point.
int launch_real(const double *v, double *out, int64_t np, int nslot, int m, int N, cudaStream_t st);
int launch_max_vel(const double *v, double *vmax, int64_t np, int nslot, int m, int N, cudaStream_t st);
int launch_point_max_vel(const double *v, double *pmax, int64_t np, int nslot, int m, int N, cudaStream_t st);

// Operands of the Navier-Stokes cross product at the Gauss points (sfnl_gauss.cu): device arrays of
// the mesh (jj 1-based (n_w, me), ww (n_w, l_G), dw (2, n_w, l_G, me), rr (2, np_nodes)), the nodal
// velocity v and rotation omega (np_nodes, 6, nmod; omega may be null) and the modes list_mode (nmod).
struct GaussArgs {
  const double *v, *omega, *ww, *dw, *rr;
  const int *jj, *list_mode;
  int np_nodes, me, n_w, l_G, nmod;
};
// rotv, w: (l_G*me, 6, nmod) outputs (RotV + 2 Om, W).
int launch_gauss_eval(const GaussArgs &a, double *rotv, double *w, cudaStream_t st);

// Elementary programs: cross (6 -> 3), dot (6 -> 1), product (2 -> 1),
// scalar x vector (4 -> 3) and tensor (6 -> 9).  Every bilinear program of
// sfnl_ops.cuh is a sequence of them on one stream (the bundle is four, a
// linearised cross product two or four, accumulating where a term adds to an
// earlier one).
enum { EK_CROSS = 0, EK_DOT = 1, EK_PROD = 2, EK_SVECT = 3, EK_TENSOR = 4 };
struct Elem {
  int ek;
  int in[6];     // field indices into ProgArgs.in
  int out[9];    // indices into ProgArgs.out
  unsigned adj;  // bit f: operand f is a cotangent (synthesised with the analysis weights)
  int acc;       // 1: add to the output instead of overwriting it
};
int decompose_program(int op, std::vector<Elem> &seq);   // sfnl_fast.cu
bool split_supported(int op, int m);                    // sfnl_split.cu

}  // namespace sfnl
