// sfnl_gauss.cu -- the operands of the Navier-Stokes cross product at the Gauss points.
//
// SOURCES/SIMULATION/subroutine_ns_with_velocity.F90:512-629 (smb_cross_prod_gauss_sft_par) builds,
// for every local Fourier mode, element and Gauss point of the velocity mesh, the velocity W, the
// precession rotation Om and the curl RotV of the mode in cylindrical coordinates from the nodal
// coefficients, and passes (RotV + 2 Om, W) to FFT_PAR_CROSS_PROD_DCL.  This kernel does the first
// part on the GPU: one thread per (Gauss point, mode), the element's nodes gathered through jj; the
// outputs are the (l_G*me, 6, nmod) Fortran arrays the FAST cross product then reads.
#include <cuda_runtime.h>

#include "sfnl_internal.h"

namespace sfnl {

namespace {

constexpr int kMaxNw = 10;  // nodes per element (P2 triangles: 6)

__global__ void __launch_bounds__(256) gauss_eval_kernel(GaussArgs a, double *rotv, double *w) {
  const int64_t ng = (int64_t)a.l_G * a.me, total = ng * a.nmod;
  for (int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; idx < total; idx += (int64_t)gridDim.x * blockDim.x) {
    const int64_t p = idx % ng;
    const int i = (int)(idx / ng);
    const int m = (int)(p / a.l_G), l = (int)(p % a.l_G);
    const double mode = (double)a.list_mode[i];
    const double *dwl = a.dw + (size_t)2 * a.n_w * (l + (size_t)a.l_G * m);  // dw_loc = dw(:,:,l,m)
    double ray = 0.0, wv[6] = {0, 0, 0, 0, 0, 0}, om[6] = {0, 0, 0, 0, 0, 0};
    double d1[6] = {0, 0, 0, 0, 0, 0}, d2[6] = {0, 0, 0, 0, 0, 0};  // sum Vs(:,k) dw_loc(1|2,:)
    for (int n = 0; n < a.n_w; ++n) {
      int node = a.jj[n + (size_t)a.n_w * m] - 1;  // 1-based node numbers
      node = node < 0 ? 0 : node >= a.np_nodes ? a.np_nodes - 1 : node;  // no access outside V
      const double wt = a.ww[n + (size_t)a.n_w * l], g1 = dwl[2 * n], g2 = dwl[2 * n + 1];
      ray = fma(a.rr[2 * (size_t)node], wt, ray);
      const double *vn = a.v + node + (size_t)a.np_nodes * 6 * i;
#pragma unroll
      for (int k = 0; k < 6; ++k) {
        const double vs = vn[(size_t)a.np_nodes * k];
        wv[k] = fma(vs, wt, wv[k]);
        d1[k] = fma(vs, g1, d1[k]);
        d2[k] = fma(vs, g2, d2[k]);
      }
      if (a.omega) {
        const double *on = a.omega + node + (size_t)a.np_nodes * 6 * i;
#pragma unroll
        for (int k = 0; k < 6; ++k) om[k] = fma(on[(size_t)a.np_nodes * k], wt, om[k]);
      }
    }
    const double mr = mode / ray, ir = 1.0 / ray;
    double r[6];
    r[0] = mr * wv[5] - d2[2];               // cos, r:     mode/ray W6 - d/dz W3
    r[3] = d2[1] - d1[5];                    // sin, theta: d/dz W2 - d/dr W6
    r[4] = ir * wv[2] + d1[2] - mr * wv[1];  // cos, z:     W3/ray + d/dr W3 - mode/ray W2
    r[1] = -mr * wv[4] - d2[3];              // sin, r
    r[2] = d2[0] - d1[4];                    // cos, theta
    r[5] = ir * wv[3] + d1[3] + mr * wv[0];  // sin, z
#pragma unroll
    for (int k = 0; k < 6; ++k) {
      const size_t at = (size_t)p + (size_t)ng * (k + 6 * (size_t)i);
      rotv[at] = r[k] + 2.0 * om[k];
      w[at] = wv[k];
    }
  }
}

}  // namespace

int launch_gauss_eval(const GaussArgs &a, double *rotv, double *w, cudaStream_t st) {
  if (a.n_w < 1 || a.n_w > kMaxNw) return set_error(SFNL_ERR_UNSUPPORTED, "nodes per element outside 1..10");
  const int64_t total = (int64_t)a.l_G * a.me * a.nmod;
  if (total == 0) return SFNL_OK;
  int64_t blocks = (total + 255) / 256;
  const int64_t cap = (int64_t)num_sms() * 32;
  if (blocks > cap) blocks = cap;
  gauss_eval_kernel<<<(unsigned)blocks, 256, 0, st>>>(a, rotv, w);
  return check_launch("Gauss-point operands");
}

}  // namespace sfnl
