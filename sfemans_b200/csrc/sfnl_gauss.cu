// sfnl_gauss.cu -- the operands of the Gauss-point callers of the dealiased products.
//
// Each caller builds, for every local Fourier mode, element and Gauss point of its mesh, cylindrical
// (r, theta, z) quantities of the mode from the nodal coefficients (the element's nodes gathered through
// jj, values with ww, (d/dr, d/dz) with dw) and passes them to one of the products of fft_parallel.F90:
//   GK_NS      smb_cross_prod_gauss_sft_par (SOURCES/SIMULATION/subroutine_ns_with_velocity.F90:512-629):
//              RotV = curl u + 2 Om (precession rotation) and W = u, for (RotV, W) -> cross product;
//   GK_LORENTZ smb_CurlH_cross_B_gauss_sft_par (subroutine_ns_with_m.F90:788-883): RotV = curl H
//              and W = B (two nodal fields), for the cross product;
//   GK_ADVECT  smb_ugradc_gauss_fft_par (subroutine_level_set.F90:434-534, and the temperature and
//              concentration versions subroutine_temperature_with_T.F90:247-350,
//              subroutine_concentration.F90:243-341): Gradc = grad c, W = u, and for the conservative
//              form Div = div u and Cgauss = c (Gradc and Cgauss times the element's heat capacity
//              in the temperature version), for Gradc . W (+ Div Cgauss).
// One thread per (Gauss point, mode); the outputs are the (l_G*me, nslot, nmod) Fortran arrays the
// FAST products then read.
#include <cuda_runtime.h>

#include "sfnl_gauss.cuh"
#include "sfnl_internal.h"

namespace sfnl {

namespace {

constexpr int kMaxNw = 10;  // nodes per element (P2 triangles: 6)

template <int KIND>
__global__ void __launch_bounds__(256) gauss_eval_kernel(GaussArgs a, double *o0, double *o1, double *o2, double *o3) {
  const int64_t ng = (int64_t)a.l_G * a.me, total = ng * a.nmod;
  for (int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; idx < total; idx += (int64_t)gridDim.x * blockDim.x) {
    const int64_t p = idx % ng;
    const int i = (int)(idx / ng);
    if constexpr (KIND == GK_NS || KIND == GK_LORENTZ) {
      double r[6], w[6];
      gauss_curl_point<KIND>(a, p, i, r, w);
#pragma unroll
      for (int k = 0; k < 6; ++k) {
        const size_t at = (size_t)p + (size_t)ng * (k + 6 * (size_t)i);
        o0[at] = r[k];
        o1[at] = w[k];
      }
    } else {
      const int m = (int)(p / a.l_G), l = (int)(p % a.l_G);
      const double mode = (double)a.list_mode[i];
      const double *dwl = a.dw + (size_t)2 * a.n_w * (l + (size_t)a.l_G * m);  // dw_loc = dw(:,:,l,m)
      double ray = 0.0, wv[6] = {0, 0, 0, 0, 0, 0}, d1[6] = {0, 0, 0, 0, 0, 0}, d2[6] = {0, 0, 0, 0, 0, 0};
      double cw[2] = {0, 0}, c1[2] = {0, 0}, c2[2] = {0, 0};  // the scalar: values, d/dr, d/dz
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
        const double *cn = a.v2 + node + (size_t)a.np_nodes * 2 * i;
#pragma unroll
        for (int k = 0; k < 2; ++k) {
          const double cs = cn[(size_t)a.np_nodes * k];
          cw[k] = fma(cs, wt, cw[k]);
          c1[k] = fma(cs, g1, c1[k]);
          c2[k] = fma(cs, g2, c2[k]);
        }
      }
      const double mr = mode / ray;
      const double hc = a.heat ? a.heat[m] : 1.0;  // heat_capa_in(m), temperature version
      const double gc[6] = {c1[0], c1[1], mr * cw[1], -mr * cw[0], c2[0], c2[1]};
#pragma unroll
      for (int k = 0; k < 6; ++k) {
        const size_t at = (size_t)p + (size_t)ng * (k + 6 * (size_t)i);
        o0[at] = a.heat ? hc * gc[k] : gc[k];
        o1[at] = wv[k];
      }
      if (o2) {  // the conservative term c div u
        const size_t at = (size_t)p + (size_t)ng * 2 * (size_t)i;
        o2[at] = d1[0] + wv[0] / ray + mr * wv[3] + d2[4];
        o2[at + ng] = d1[1] + wv[1] / ray - mr * wv[2] + d2[5];
        o3[at] = a.heat ? hc * cw[0] : cw[0];
        o3[at + ng] = a.heat ? hc * cw[1] : cw[1];
      }
    }
  }
}

// vt[node][k][i] = v[node + np_nodes*(k + nslot i)]: 32 modes x 32 nodes per CTA through shared memory, both
// sides coalesced.
__global__ void __launch_bounds__(256) nodal_transpose_kernel(const double *__restrict__ v, double *__restrict__ vt,
                                                              int np_nodes, int m, int nslot) {
  __shared__ double t[32][33];
  const int64_t node0 = (int64_t)blockIdx.x * 32;
  const int k = blockIdx.y, i0 = blockIdx.z * 32;
  const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;  // 8 rows of 32
  for (int r = ty; r < 32; r += 8) {
    const int i = i0 + r;
    const int64_t node = node0 + tx;
    if (i < m && node < np_nodes) t[r][tx] = v[node + (int64_t)np_nodes * (k + nslot * (int64_t)i)];
  }
  __syncthreads();
  for (int r = ty; r < 32; r += 8) {
    const int64_t node = node0 + r;
    const int i = i0 + tx;
    if (i < m && node < np_nodes) vt[node * nslot * m + (int64_t)k * m + i] = t[tx][r];
  }
}

}  // namespace

int launch_nodal_transpose(const double *v, double *vt, int np_nodes, int m, cudaStream_t st, int nslot) {
  if (np_nodes == 0) return SFNL_OK;
  dim3 grid((unsigned)((np_nodes + 31) / 32), (unsigned)nslot, (unsigned)((m + 31) / 32));
  nodal_transpose_kernel<<<grid, 256, 0, st>>>(v, vt, np_nodes, m, nslot);
  return check_launch("nodal transpose");
}

int launch_gauss_eval(const GaussArgs &a, int kind, double *o0, double *o1, double *o2, double *o3, cudaStream_t st) {
  if (a.n_w < 1 || a.n_w > kMaxNw) return set_error(SFNL_ERR_UNSUPPORTED, "nodes per element outside 1..10");
  const int64_t total = (int64_t)a.l_G * a.me * a.nmod;
  if (total == 0) return SFNL_OK;
  int64_t blocks = (total + 255) / 256;
  const int64_t cap = (int64_t)num_sms() * 32;
  if (blocks > cap) blocks = cap;
  switch (kind) {
    case GK_NS: gauss_eval_kernel<GK_NS><<<(unsigned)blocks, 256, 0, st>>>(a, o0, o1, o2, o3); break;
    case GK_LORENTZ: gauss_eval_kernel<GK_LORENTZ><<<(unsigned)blocks, 256, 0, st>>>(a, o0, o1, o2, o3); break;
    case GK_ADVECT: gauss_eval_kernel<GK_ADVECT><<<(unsigned)blocks, 256, 0, st>>>(a, o0, o1, o2, o3); break;
    default: return set_error(SFNL_ERR_ARG, "unknown Gauss-point caller");
  }
  return check_launch("Gauss-point operands");
}

}  // namespace sfnl
