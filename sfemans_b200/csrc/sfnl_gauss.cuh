// sfnl_gauss.cuh -- the curl-type Gauss-point operands of one (Gauss point, mode), shared by the
// operand kernel (sfnl_gauss.cu) and the fused Gauss-point cross product (sfnl_fast.cu).
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

}  // namespace sfnl
