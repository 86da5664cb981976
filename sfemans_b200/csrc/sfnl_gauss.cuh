// sfnl_gauss.cuh -- the Gauss-point operands of one (Gauss point, mode), shared by the operand kernel
// (sfnl_gauss.cu) and the fused Gauss-point products (sfnl_fast.cu).
#pragma once
#include <cuda_runtime.h>

#include "sfnl_internal.h"

namespace sfnl {

// Gauss point p (element p / l_G, quadrature point p % l_G) and mode index i: rot = curl v in
// cylindrical coordinates for the mode number list_mode[i] (subroutine_ns_with_velocity.F90:592-607,
// subroutine_ns_with_m.F90:851-867), plus 2 omega for GK_NS when omega is given; w = v (GK_NS) or v2
// (GK_LORENTZ) at the point.  Slots: 0/1 cos/sin of r, 2/3 of theta, 4/5 of z.
// The curl of the mode from the sums over the element's nodes (subroutine_ns_with_velocity.F90:592-607):
// wv = sum V ww, d1 / d2 = sum V d/dr / d/dz, om = sum omega ww, w2 = sum v2 ww.
template <int KIND>
__device__ __forceinline__ void curl_from_sums(double mode, double ray, const double (&wv)[6], const double (&d1)[6],
                                               const double (&d2)[6], const double (&om)[6], const double (&w2)[6],
                                               double (&rot)[6], double (&w)[6]) {
  const double mr = mode / ray, ir = 1.0 / ray;
  rot[0] = mr * wv[5] - d2[2];               // cos, r:     mode/ray W6 - d/dz W3
  rot[3] = d2[1] - d1[5];                    // sin, theta: d/dz W2 - d/dr W6
  rot[4] = ir * wv[2] + d1[2] - mr * wv[1];  // cos, z:     W3/ray + d/dr W3 - mode/ray W2
  rot[1] = -mr * wv[4] - d2[3];              // sin, r
  rot[2] = d2[0] - d1[4];                    // cos, theta
  rot[5] = ir * wv[3] + d1[3] + mr * wv[0];  // sin, z
#pragma unroll
  for (int k = 0; k < 6; ++k) {
    if (KIND == GK_NS) rot[k] += 2.0 * om[k];
    w[k] = KIND == GK_NS ? wv[k] : w2[k];
  }
}

// TM = 0: the nodal fields in the callers' layout (np_nodes, 6, nmod), value (node, k, i) at
// node + np_nodes*(k + 6 i); TM = nmod > 0: node-major copies (nodal_transpose), value at
// node*6*TM + k*TM + i, so that the lanes of a warp taking consecutive modes of one point read
// consecutive addresses.
template <int KIND, int TM = 0>
__device__ __forceinline__ size_t nodal_at(const GaussArgs &a, int node, int k, int i) {
  return TM ? (size_t)node * 6 * TM + (size_t)k * TM + i : node + (size_t)a.np_nodes * (k + 6 * (size_t)i);
}

template <int KIND, int TM = 0>
__device__ __forceinline__ void gauss_curl_point(const GaussArgs &a, int64_t p, int i, double (&rot)[6],
                                                 double (&w)[6]) {
  static_assert(KIND == GK_NS || KIND == GK_LORENTZ, "curl-type callers only");
  const int m = (int)(p / a.l_G), l = (int)(p % a.l_G);
  const double mode = (double)a.list_mode[i];
  const double *dwl = a.dw + (size_t)2 * a.n_w * (l + (size_t)a.l_G * m);  // dw_loc = dw(:,:,l,m)
  double ray = 0.0, wv[6] = {0, 0, 0, 0, 0, 0}, om[6] = {0, 0, 0, 0, 0, 0}, w2[6] = {0, 0, 0, 0, 0, 0};
  double d1[6] = {0, 0, 0, 0, 0, 0}, d2[6] = {0, 0, 0, 0, 0, 0};  // sum Vs(:,k) dw_loc(1|2,:)
  for (int n = 0; n < a.n_w; ++n) {
    int node = a.jj[n + (size_t)a.n_w * m] - 1;  // 1-based node numbers
    node = node < 0 ? 0 : node >= a.np_nodes ? a.np_nodes - 1 : node;  // no access outside V
    const double wt = a.ww[n + (size_t)a.n_w * l], g1 = dwl[2 * n], g2 = dwl[2 * n + 1];
    ray = fma(a.rr[2 * (size_t)node], wt, ray);
#pragma unroll
    for (int k = 0; k < 6; ++k) {
      const double vs = a.v[nodal_at<KIND, TM>(a, node, k, i)];
      wv[k] = fma(vs, wt, wv[k]);
      d1[k] = fma(vs, g1, d1[k]);
      d2[k] = fma(vs, g2, d2[k]);
    }
    if (KIND == GK_NS && a.omega) {
#pragma unroll
      for (int k = 0; k < 6; ++k) om[k] = fma(a.omega[nodal_at<KIND, TM>(a, node, k, i)], wt, om[k]);
    }
    if (KIND == GK_LORENTZ) {
#pragma unroll
      for (int k = 0; k < 6; ++k) w2[k] = fma(a.v2[nodal_at<KIND, TM>(a, node, k, i)], wt, w2[k]);
    }
  }
  curl_from_sums<KIND>(mode, ray, wv, d1, d2, om, w2, rot, w);
}

// The same for the n_w = NW nodes of the point already gathered (node numbers, basis values and
// derivatives at the point, radius): every load of the nodal fields is independent.
template <int KIND, int TM, int NW>
__device__ __forceinline__ void gauss_curl_gathered(const GaussArgs &a, const int *node, const double *wt,
                                                    const double *g1, const double *g2, double ray, int i,
                                                    double (&rot)[6], double (&w)[6]) {
  const double mode = (double)a.list_mode[i];
  double wv[6] = {0, 0, 0, 0, 0, 0}, om[6] = {0, 0, 0, 0, 0, 0}, w2[6] = {0, 0, 0, 0, 0, 0};
  double d1[6] = {0, 0, 0, 0, 0, 0}, d2[6] = {0, 0, 0, 0, 0, 0};
#pragma unroll
  for (int n = 0; n < NW; ++n) {
#pragma unroll
    for (int k = 0; k < 6; ++k) {
      const double vs = a.v[nodal_at<KIND, TM>(a, node[n], k, i)];
      wv[k] = fma(vs, wt[n], wv[k]);
      d1[k] = fma(vs, g1[n], d1[k]);
      d2[k] = fma(vs, g2[n], d2[k]);
    }
    if (KIND == GK_NS && a.omega) {
#pragma unroll
      for (int k = 0; k < 6; ++k) om[k] = fma(a.omega[nodal_at<KIND, TM>(a, node[n], k, i)], wt[n], om[k]);
    }
    if (KIND == GK_LORENTZ) {
#pragma unroll
      for (int k = 0; k < 6; ++k) w2[k] = fma(a.v2[nodal_at<KIND, TM>(a, node[n], k, i)], wt[n], w2[k]);
    }
  }
  curl_from_sums<KIND>(mode, ray, wv, d1, d2, om, w2, rot, w);
}

// The operands of one (Gauss point p, mode index i) from node-major nodal fields with a run-time mode
// stride tm (launch_nodal_transpose: value (node, k, i) at node*ns*tm + k*tm + i, ns = 6 for a.v, a.omega
// and the Lorentz field a.v2, 2 for the advection scalar a.v2).  f[field][cos, sin]:
//   GK_NS, GK_LORENTZ: fields 0-2 = RotV (r, theta, z), 3-5 = W;
//   GK_ADVECT: 0-2 = heat grad c, 3-5 = u, 6 = div u, 7 = heat c (subroutine_temperature_with_T.F90:300-331).
template <int KIND>
__device__ __forceinline__ void gauss_operands_nm(const GaussArgs &a, int64_t p, int i, int tm, double (&f)[8][2]) {
  const int me = (int)(p / a.l_G), l = (int)(p % a.l_G);
  const double mode = (double)a.list_mode[i];
  const double *dwl = a.dw + (size_t)2 * a.n_w * (l + (size_t)a.l_G * me);
  double ray = 0.0, wv[6] = {0, 0, 0, 0, 0, 0}, d1[6] = {0, 0, 0, 0, 0, 0}, d2[6] = {0, 0, 0, 0, 0, 0};
  double om[6] = {0, 0, 0, 0, 0, 0}, w2[6] = {0, 0, 0, 0, 0, 0};
  double cw[2] = {0, 0}, c1[2] = {0, 0}, c2[2] = {0, 0};
  for (int n = 0; n < a.n_w; ++n) {
    int node = a.jj[n + (size_t)a.n_w * me] - 1;  // 1-based node numbers
    node = node < 0 ? 0 : node >= a.np_nodes ? a.np_nodes - 1 : node;  // no access outside the fields
    const double wt = a.ww[n + (size_t)a.n_w * l], g1 = dwl[2 * n], g2 = dwl[2 * n + 1];
    ray = fma(a.rr[2 * (size_t)node], wt, ray);
    const double *vn = a.v + (size_t)node * 6 * tm + i;
#pragma unroll
    for (int k = 0; k < 6; ++k) {
      const double vs = vn[(size_t)k * tm];
      wv[k] = fma(vs, wt, wv[k]);
      d1[k] = fma(vs, g1, d1[k]);
      d2[k] = fma(vs, g2, d2[k]);
    }
    if (KIND == GK_NS && a.omega) {
      const double *on = a.omega + (size_t)node * 6 * tm + i;
#pragma unroll
      for (int k = 0; k < 6; ++k) om[k] = fma(on[(size_t)k * tm], wt, om[k]);
    }
    if (KIND == GK_LORENTZ) {
      const double *bn = a.v2 + (size_t)node * 6 * tm + i;
#pragma unroll
      for (int k = 0; k < 6; ++k) w2[k] = fma(bn[(size_t)k * tm], wt, w2[k]);
    }
    if (KIND == GK_ADVECT) {
      const double *cn = a.v2 + (size_t)node * 2 * tm + i;
#pragma unroll
      for (int k = 0; k < 2; ++k) {
        const double cs = cn[(size_t)k * tm];
        cw[k] = fma(cs, wt, cw[k]);
        c1[k] = fma(cs, g1, c1[k]);
        c2[k] = fma(cs, g2, c2[k]);
      }
    }
  }
  if constexpr (KIND == GK_ADVECT) {
    const double mr = mode / ray, hc = a.heat ? a.heat[me] : 1.0;
    f[0][0] = hc * c1[0];
    f[0][1] = hc * c1[1];
    f[1][0] = hc * (mr * cw[1]);
    f[1][1] = hc * (-mr * cw[0]);
    f[2][0] = hc * c2[0];
    f[2][1] = hc * c2[1];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      f[3 + k][0] = wv[2 * k];
      f[3 + k][1] = wv[2 * k + 1];
    }
    f[6][0] = d1[0] + wv[0] / ray + mr * wv[3] + d2[4];
    f[6][1] = d1[1] + wv[1] / ray - mr * wv[2] + d2[5];
    f[7][0] = hc * cw[0];
    f[7][1] = hc * cw[1];
  } else {
    double rot[6], w[6];
    curl_from_sums<KIND>(mode, ray, wv, d1, d2, om, w2, rot, w);
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      f[k][0] = rot[2 * k];
      f[k][1] = rot[2 * k + 1];
      f[3 + k][0] = w[2 * k];
      f[3 + k][1] = w[2 * k + 1];
    }
    f[6][0] = f[6][1] = f[7][0] = f[7][1] = 0.0;
  }
}

}  // namespace sfnl
