// sfnl_ops.cuh -- pointwise "programs" applied on the azimuthal grid.
//
// Every entry point of the library is one program: NI scalar input fields
// are synthesised on the grid, the program maps their values at each angle
// to NO scalar output values, and the outputs are analysed back to cos/sin
// coefficients.  A scalar field is one (cos, sin) slot pair of a Fortran
// array V(np, nslot, m).
//
// The pointwise maps restate fft_parallel.F90:270-274 (cross: components
// (r,theta,z) = slot pairs (1,2),(3,4),(5,6); out_r = v1_t v2_z - v1_z v2_t,
// ...), :449-451 (dot), :617 (scalar product), :786 (quotient), :1150-1157
// (scalar x vector, vector / scalar) and :1676-1706 (tensor u_k v_l, and the
// tension form u_k v_l / (|v| + 1e-14) - |v| delta_kl), plus the
// linearisations and transposes used by the JVP/VJP entry points and the
// advection term of the scalar equations (grad c . u + c div u,
// SOURCES/SIMULATION/subroutine_temperature_with_T.F90:339-342: a dot product
// and a product whose analyses the reference adds).
#pragma once
#include <cstdint>

namespace sfnl {

enum Op : int {
  OP_CROSS = 0,     // [v1(3), v2(3)]                 -> [v1 x v2]
  OP_DOT = 1,       // [v1(3), v2(3)]                 -> [v1 . v2]
  OP_PROD = 2,      // [c1, c2]                       -> [c1 c2]
  OP_BUNDLE = 3,    // [u, w, b, j, gT] (15)          -> [u x w, u x b, j x b, u . gT] (10)
  OP_CROSS_JVP = 4, // [u, w, du, dw] (12)            -> [du x w + u x dw] (3)
  OP_CROSS_VJP = 5, // [u, w, c] (9), c adjoint input -> [w x c, c x u] (6), adjoint outputs
  OP_MHD_JVP = 6,   // [u, w, b, du, dw, db] (18)     -> [du x w + u x dw, du x b + u x db] (6)
  OP_MHD_VJP = 7,   // [u, w, b, c1, c2] (15)         -> [w x c1 + b x c2, c1 x u, c2 x u] (9)
  OP_DIV = 8,       // [c1, c2]                       -> [c1 / c2]
  OP_SVECT = 9,     // [v(3), s]                      -> [s v] (3)
  OP_SVDIV = 10,    // [v(3), s]                      -> [v / s] (3)
  OP_TENSOR = 11,   // [u(3), v(3)]                   -> [u_k v_l] (9, o = 3k + l)
  OP_TENSION = 12,  // [u(3), v(3)]                   -> [u_k v_l / (|v| + 1e-14) - |v| delta_kl] (9)
  OP_ADVECT = 13,   // [g(3), w(3), d, c] (8)         -> [g . w + d c] (advection of a scalar, conservative form)
  OP_COUNT = 14
};

constexpr int kMaxIn = 18;
constexpr int kMaxOut = 10;

__host__ __device__ constexpr int op_nin(int op) {
  return op == OP_CROSS ? 6 : op == OP_DOT ? 6 : op == OP_PROD ? 2 : op == OP_BUNDLE ? 15
       : op == OP_CROSS_JVP ? 12 : op == OP_CROSS_VJP ? 9 : op == OP_MHD_JVP ? 18 : op == OP_MHD_VJP ? 15
       : op == OP_DIV ? 2 : op == OP_SVECT || op == OP_SVDIV ? 4 : op == OP_ADVECT ? 8 : 6;
}
__host__ __device__ constexpr int op_nout(int op) {
  return op == OP_CROSS ? 3 : op == OP_DOT ? 1 : op == OP_PROD ? 1 : op == OP_BUNDLE ? 10
       : op == OP_CROSS_JVP ? 3 : op == OP_CROSS_VJP ? 6 : op == OP_MHD_JVP ? 6 : op == OP_MHD_VJP ? 9
       : op == OP_DIV ? 1 : op == OP_SVECT || op == OP_SVDIV ? 3 : op == OP_ADVECT ? 1 : 9;
}
// Programs whose result is the exact truncated product on any alias-free grid
// (bilinear in the synthesised fields); the quotients and the tension tensor
// depend on the grid and are evaluated on the caller's grid only.
__host__ __device__ constexpr bool op_bilinear(int op) {
  return op != OP_DIV && op != OP_SVDIV && op != OP_TENSION;
}
// Adjoint fields: inputs that are cotangents are synthesised with the analysis
// weights D = (1/N, 2/N, 2/N, ...) (the transpose of the analysis), and the
// outputs of a VJP are analysed without D (the transpose of the synthesis).
__host__ __device__ constexpr bool op_adjoint_in(int op, int f) {
  return (op == OP_CROSS_VJP && f >= 6) || (op == OP_MHD_VJP && f >= 9);
}
__host__ __device__ constexpr bool op_adjoint_out(int op) { return op == OP_CROSS_VJP || op == OP_MHD_VJP; }

template <typename T>
__device__ __forceinline__ void cross3(const T *a, const T *b, T *o) {
  o[0] = a[1] * b[2] - a[2] * b[1];
  o[1] = a[2] * b[0] - a[0] * b[2];
  o[2] = a[0] * b[1] - a[1] * b[0];
}
template <typename T>
__device__ __forceinline__ void cross3_acc(const T *a, const T *b, T *o) {
  o[0] += a[1] * b[2] - a[2] * b[1];
  o[1] += a[2] * b[0] - a[0] * b[2];
  o[2] += a[0] * b[1] - a[1] * b[0];
}

// y[0..NO) = program(x[0..NI)) at one angle.
template <int OP, typename T>
__device__ __forceinline__ void apply_op(const T *x, T *y) {
  if constexpr (OP == OP_CROSS) {
    cross3(x, x + 3, y);
  } else if constexpr (OP == OP_DOT) {
    y[0] = x[0] * x[3] + x[1] * x[4] + x[2] * x[5];
  } else if constexpr (OP == OP_PROD) {
    y[0] = x[0] * x[1];
  } else if constexpr (OP == OP_BUNDLE) {
    cross3(x, x + 3, y);           // u x w
    cross3(x, x + 6, y + 3);       // u x b
    cross3(x + 9, x + 6, y + 6);   // j x b
    y[9] = x[0] * x[12] + x[1] * x[13] + x[2] * x[14];  // u . gradT
  } else if constexpr (OP == OP_CROSS_JVP) {
    cross3(x + 6, x + 3, y);       // du x w
    cross3_acc(x, x + 9, y);       // + u x dw
  } else if constexpr (OP == OP_CROSS_VJP) {
    cross3(x + 3, x + 6, y);       // w x c     (d/d du)
    cross3(x + 6, x, y + 3);       // c x u     (d/d dw)
  } else if constexpr (OP == OP_MHD_JVP) {
    cross3(x + 9, x + 3, y);       // du x w
    cross3_acc(x, x + 12, y);      // + u x dw
    cross3(x + 9, x + 6, y + 3);   // du x b
    cross3_acc(x, x + 15, y + 3);  // + u x db
  } else if constexpr (OP == OP_MHD_VJP) {
    cross3(x + 3, x + 9, y);       // w x c1
    cross3_acc(x + 6, x + 12, y);  // + b x c2   (d/d du)
    cross3(x + 9, x, y + 3);       // c1 x u     (d/d dw)
    cross3(x + 12, x, y + 6);      // c2 x u     (d/d db)
  } else if constexpr (OP == OP_DIV) {
    y[0] = x[0] / x[1];
  } else if constexpr (OP == OP_SVECT) {
#pragma unroll
    for (int k = 0; k < 3; ++k) y[k] = x[3] * x[k];
  } else if constexpr (OP == OP_SVDIV) {
#pragma unroll
    for (int k = 0; k < 3; ++k) y[k] = x[k] / x[3];
  } else if constexpr (OP == OP_TENSOR) {
#pragma unroll
    for (int k = 0; k < 3; ++k)
#pragma unroll
      for (int l = 0; l < 3; ++l) y[3 * k + l] = x[k] * x[3 + l];
  } else if constexpr (OP == OP_ADVECT) {
    y[0] = x[0] * x[3] + x[1] * x[4] + x[2] * x[5] + x[6] * x[7];
  } else if constexpr (OP == OP_TENSION) {
    const T nrm = sqrt(x[3] * x[3] + x[4] * x[4] + x[5] * x[5]);
    const T den = nrm + T(1.0e-14);
#pragma unroll
    for (int k = 0; k < 3; ++k)
#pragma unroll
      for (int l = 0; l < 3; ++l) y[3 * k + l] = x[k] * x[3 + l] / den - (k == l ? nrm : T(0));
  }
}

// Description of one launch: where each scalar field lives.
// Field f of input i: cos coefficient of mode n for point p (batch entry b) at
//   in[f] + b*in_bs[f] + p + n*in_ldm[f]; the sine is np elements further.
// Output field o: at out[o] + b*out_bs[o] + p*out_ps + n*out_ldm[o], the sine
// out_ps*np elements further (out_ps = 3 for the tensor layout V(3, np, 6, m)
// of fft_parallel.F90:1552, 1 otherwise).
struct ProgArgs {
  const double *in[kMaxIn];
  double *out[kMaxOut];
  int64_t in_ldm[kMaxIn];
  int64_t out_ldm[kMaxOut];
  int64_t in_bs[kMaxIn];
  int64_t out_bs[kMaxOut];
  int64_t out_ps;
  int64_t np;
  int m;      // modes
  int N;      // grid length used by the kernel
  int batch;  // k_batch (grid.y)
  int op;
};

}  // namespace sfnl
