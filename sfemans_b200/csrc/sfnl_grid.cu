// sfnl_grid.cu -- all-FP64 products on the caller's grid (SFNL_ALGO_GRID).
//
// Dense DFT on the grid the reference uses, N = 2*m_max_pad-1
// (fft_parallel.F90:183): synthesis f(theta_j) = a_0 + sum_n a_n cos(n theta_j)
// + b_n sin(n theta_j) (the c2r of :261-267 applied to the half-complex pack
// of :223-241), the pointwise program, then analysis a_n = (c_n/N) sum_j g_j
// cos(n theta_j), b_n = (2/N) sum_j g_j sin(n theta_j), n < m (the r2c, 1/N,
// 2*CONJG and truncation of :278-299).  Angles come from an exact table
// cos/sin(2 pi r / N) indexed by (n*j mod N), so the arithmetic is the same
// for every N, odd or even, dealiasing or not: with a pad too short to
// dealias it reproduces the reference's aliased result.
//
// Parallel decomposition: one warp per point.  The point's coefficients are
// staged in shared memory (read by all lanes as broadcasts), lanes own grid
// angles during synthesis and modes during analysis.  This form is the
// parity anchor, the fallback for any (m, N), and the only form of the
// programs that depend on the grid (the quotients and the tension tensor);
// the fast and split forms carry the throughput of the products.
#include <cuda_runtime.h>

#include "sfnl_internal.h"
#include "sfnl_ops.cuh"

namespace sfnl {

namespace {

constexpr int kGridThreads = 128;

template <int OP>
__global__ void __launch_bounds__(kGridThreads) grid_kernel(const ProgArgs a, int warps_per_cta, int per_warp) {
  constexpr int NI = op_nin(OP), NO = op_nout(OP);
  extern __shared__ __align__(16) double smem[];
  const int N = a.N, m = a.m;
  double2 *tab = reinterpret_cast<double2 *>(smem);
  const int tab_doubles = 2 * N;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  double *X = smem + tab_doubles + (size_t)warp * per_warp;  // NI x 2m
  double *G = X + NI * 2 * m;                                  // NO x N

  for (int r = threadIdx.x; r < N; r += blockDim.x) {
    double s, c;
    sincospi(2.0 * (double)r / (double)N, &s, &c);
    tab[r] = make_double2(c, s);
  }
  __syncthreads();
  if (warp >= warps_per_cta) return;

  const int b = blockIdx.y;
  const double invN = 1.0 / (double)N, twoN = 2.0 / (double)N;
  for (int64_t p = (int64_t)blockIdx.x * warps_per_cta + warp; p < a.np; p += (int64_t)gridDim.x * warps_per_cta) {
    // 1. stage the point's coefficients: X[f][k], k < m cos, k >= m sin.
    for (int idx = lane; idx < NI * 2 * m; idx += 32) {
      const int f = idx / (2 * m), k = idx - f * 2 * m;
      const int n = k < m ? k : k - m;
      double v = 0.0;
      if (k != m) {  // the sine of mode 0 is ignored (fft_parallel.F90:241)
        const double *src = a.in[f] + (int64_t)b * a.in_bs[f] + p + (int64_t)n * a.in_ldm[f] + (k >= m ? a.np : 0);
        v = __ldg(src);
      }
      if (op_adjoint_in(OP, f)) v *= (n == 0 ? invN : twoN);
      X[idx] = v;
    }
    __syncwarp();
    // 2. synthesis + program at the lane's angles.
    for (int j = lane; j < N; j += 32) {
      double x[NI];
#pragma unroll
      for (int f = 0; f < NI; ++f) x[f] = 0.0;
      int r = 0;  // n*j mod N
      for (int n = 0; n < m; ++n) {
        const double2 cs = tab[r];
#pragma unroll
        for (int f = 0; f < NI; ++f) x[f] = fma(X[f * 2 * m + n], cs.x, fma(X[f * 2 * m + m + n], cs.y, x[f]));
        r += j;
        if (r >= N) r -= N;
      }
      double y[NO];
      apply_op<OP>(x, y);
#pragma unroll
      for (int o = 0; o < NO; ++o) G[o * N + j] = y[o];
    }
    __syncwarp();
    // 3. analysis of the lane's modes, truncated to n < m.
    for (int n = lane; n < m; n += 32) {
      double ya[NO], yb[NO];
#pragma unroll
      for (int o = 0; o < NO; ++o) ya[o] = yb[o] = 0.0;
      int r = 0;  // n*j mod N
      for (int j = 0; j < N; ++j) {
        const double2 cs = tab[r];
#pragma unroll
        for (int o = 0; o < NO; ++o) {
          const double g = G[o * N + j];
          ya[o] = fma(g, cs.x, ya[o]);
          yb[o] = fma(g, cs.y, yb[o]);
        }
        r += n;
        if (r >= N) r -= N;
      }
      const double sc = op_adjoint_out(OP) ? 1.0 : (n == 0 ? invN : twoN);
#pragma unroll
      for (int o = 0; o < NO; ++o) {
        double *dst = a.out[o] + (int64_t)b * a.out_bs[o] + p * a.out_ps + (int64_t)n * a.out_ldm[o];
        dst[0] = ya[o] * sc;
        dst[a.np * a.out_ps] = (n == 0) ? 0.0 : yb[o] * sc;
      }
    }
    __syncwarp();
  }
}

template <int OP>
int launch_grid_op(const ProgArgs &a, cudaStream_t st) {
  constexpr int NI = op_nin(OP), NO = op_nout(OP);
  const int per_warp = NI * 2 * a.m + NO * a.N;  // doubles
  const size_t tab_bytes = sizeof(double) * 2 * (size_t)a.N;
  const size_t budget = 200 * 1024;
  if (tab_bytes + sizeof(double) * (size_t)per_warp > budget) return set_error(SFNL_ERR_UNSUPPORTED, "grid form: m or N too large for shared memory");
  int warps = (int)((budget - tab_bytes) / (sizeof(double) * (size_t)per_warp));
  if (warps > kGridThreads / 32) warps = kGridThreads / 32;
  const size_t smem = tab_bytes + sizeof(double) * (size_t)per_warp * warps;
  auto kern = grid_kernel<OP>;
  if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess)
    return set_error(SFNL_ERR_CUDA, "cudaFuncSetAttribute failed (grid form)");
  int64_t blocks = (a.np + warps - 1) / warps;
  const int64_t cap = (int64_t)num_sms() * 16;
  if (blocks > cap) blocks = cap;
  if (blocks < 1) blocks = 1;
  dim3 grid((unsigned)blocks, (unsigned)a.batch);
  kern<<<grid, kGridThreads, smem, st>>>(a, warps, per_warp);
  return check_launch("grid form");
}

}  // namespace

int launch_grid(const ProgArgs &a, cudaStream_t st) {
  if (a.np == 0) return SFNL_OK;
  switch (a.op) {
    case OP_CROSS: return launch_grid_op<OP_CROSS>(a, st);
    case OP_DOT: return launch_grid_op<OP_DOT>(a, st);
    case OP_PROD: return launch_grid_op<OP_PROD>(a, st);
    case OP_BUNDLE: return launch_grid_op<OP_BUNDLE>(a, st);
    case OP_CROSS_JVP: return launch_grid_op<OP_CROSS_JVP>(a, st);
    case OP_CROSS_VJP: return launch_grid_op<OP_CROSS_VJP>(a, st);
    case OP_MHD_JVP: return launch_grid_op<OP_MHD_JVP>(a, st);
    case OP_MHD_VJP: return launch_grid_op<OP_MHD_VJP>(a, st);
    case OP_DIV: return launch_grid_op<OP_DIV>(a, st);
    case OP_SVECT: return launch_grid_op<OP_SVECT>(a, st);
    case OP_SVDIV: return launch_grid_op<OP_SVDIV>(a, st);
    case OP_TENSOR: return launch_grid_op<OP_TENSOR>(a, st);
    case OP_TENSION: return launch_grid_op<OP_TENSION>(a, st);
    case OP_ADVECT: return launch_grid_op<OP_ADVECT>(a, st);
  }
  return set_error(SFNL_ERR_ARG, "unknown program");
}

}  // namespace sfnl
