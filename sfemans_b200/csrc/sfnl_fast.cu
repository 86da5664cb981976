// sfnl_fast.cu -- all-FP64 products on an internal alias-free grid (SFNL_ALGO_FAST).
//
// When the caller's pad dealiases (2*m_max_pad-1 >= 3*m_max-2, which every
// SFEMaNS caller satisfies with m_max_pad = 3*m_max/2), the reference's result
// is the exact truncated product (fft_parallel.F90:147-665 with N = 2*m_pad-1)
// and does not depend on the grid.  This form evaluates it on a grid chosen
// for the hardware: N = 4Q angles theta_j = pi(2j+1)/N, Q a multiple of 8
// with 4Q >= 3m-2.
//
// Transforms.  The two symmetry levels of a real Fourier series on that grid
// are folded out exactly (the first two radix-2 stages of a real FFT, which
// need no twiddles): with CE/CO the cosine sums over even/odd modes and SE/SO
// the sine sums, evaluated at the Q angles of the first quadrant,
//   f(t)      = CE+CO+SE+SO      f(pi-t)  = CE-CO-SE+SO
//   f(pi+t)   = CE-CO+SE-SO      f(2pi-t) = CE+CO-SE-SO,
// and the analysis folds the products g1..g4 at those four angles into
//   PE = g1+g2+g3+g4 (even cos)  PO = g1-g2-g3+g4 (odd cos)
//   QE = g1-g2+g3-g4 (even sin)  QO = g1+g2-g3-g4 (odd sin).
// What remains are eight small dense contractions per field (K = m/2 modes x
// Q angles each way), a quarter of the dense DFT, run on the FP64 tensor cores
// (mma.sync m8n8k4 f64).  The product and both folds happen in registers on
// the accumulator fragments: lane (g, q) of a warp holds point g and angles
// 2q, 2q+1 of an 8-angle tile for every field and class, so the product needs
// no data exchange, and the analysis takes each k-step's A fragment straight
// from the element the same lane produced (the angle order inside a k-step is
// chosen to make that true).
//
// Parallel decomposition: one CTA per 8-point tile; warp w owns quarter-angle
// tiles t = w, w+NW, ... in the synthesis (the CTA's warps read the tile's
// coefficients together, so L1 serves all but the first read), the folded
// products go through shared memory in fragment order, then warp w owns output
// mode tiles in the analysis.  Elementary programs are cross (6 -> 3), dot
// (6 -> 1), product (2 -> 1), scalar x vector (4 -> 3, FFT_SCALAR_VECT_DCL
// pb = 1), tensor (6 -> 9, FFT_TENSOR_DCL) and the sum of two cross products
// (12 -> 3, the JVP du x w + u x dw: two synthesis passes, one analysis); the
// bundle (away from m = 64) and the transposed programs are sequences of
// elementary launches on one stream.
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <map>
#include <mutex>
#include <type_traits>
#include <vector>

#include "sfnl_fold.cuh"
#include "sfnl_gauss.cuh"
#include "sfnl_internal.h"
#include "sfnl_ops.cuh"

namespace sfnl {

namespace {



std::mutex g_tab_mu;
std::map<std::pair<int, int>, Tables> g_tabs;  // (device, m) -> tables

}  // namespace

// Device copies of a synthesis and an analysis table (none kept on failure).
static int upload_tables(const std::vector<double> &syn, const std::vector<double> &ana, Tables *T) {
  T->syn = T->ana = nullptr;
  if (cudaMalloc(&T->syn, syn.size() * sizeof(double)) != cudaSuccess ||
      cudaMalloc(&T->ana, ana.size() * sizeof(double)) != cudaSuccess) {
    cudaGetLastError();
    cudaFree(T->syn);
    T->syn = nullptr;
    return set_error(SFNL_ERR_ALLOC, "cudaMalloc of the DFT tables failed");
  }
  if (cudaMemcpy(T->syn, syn.data(), syn.size() * sizeof(double), cudaMemcpyHostToDevice) != cudaSuccess ||
      cudaMemcpy(T->ana, ana.data(), ana.size() * sizeof(double), cudaMemcpyHostToDevice) != cudaSuccess) {
    cudaFree(T->syn);
    cudaFree(T->ana);
    T->syn = T->ana = nullptr;
    return set_error(SFNL_ERR_CUDA, "upload of the DFT tables failed");
  }
  return SFNL_OK;
}

int get_tables(const Geo &g, Tables *out) {
  int dev = 0;
  cudaGetDevice(&dev);
  std::lock_guard<std::mutex> lk(g_tab_mu);
  auto it = g_tabs.find({dev, g.m});
  if (it != g_tabs.end()) {
    *out = it->second;
    return SFNL_OK;
  }
  const long double pi = acosl(-1.0L);
  auto ang = [&](int j) { return pi * (long double)(2 * j + 1) / (long double)g.N; };
  std::vector<double> syn((size_t)g.KS_tot * g.NT * 32, 0.0);
  for (int c = 0; c < 4; ++c)
    for (int s = 0; s < g.KS[c]; ++s)
      for (int t = 0; t < g.NT; ++t)
        for (int l = 0; l < 32; ++l) {
          const int k = 4 * s + (l & 3), j = 8 * t + (l >> 2);
          double v = 0.0;
          if (k < g.ke[c]) {
            const int n = class_mode(c, k);
            const long double x = (long double)n * ang(j);
            v = (double)(c < 2 ? cosl(x) : sinl(x));
          }
          syn[(((size_t)(g.ks_off[c] + s)) * g.NT + t) * 32 + l] = v;
        }
  std::vector<double> ana((size_t)2 * g.NU_tot * g.NT * 2 * 32, 0.0);
  for (int var = 0; var < 2; ++var)
    for (int c = 0; c < 4; ++c)
      for (int u = 0; u < g.NU[c]; ++u)
        for (int t = 0; t < g.NT; ++t)
          for (int e = 0; e < 2; ++e)
            for (int l = 0; l < 32; ++l) {
              const int j = 8 * t + 2 * (l & 3) + e;  // angle of k-value (l & 3) in k-step (t, e)
              const int kk = 8 * u + (l >> 2);         // output column inside the class
              double v = 0.0;
              if (kk < g.ke[c]) {
                const int n = class_mode(c, kk);
                const long double x = (long double)n * ang(j);
                const long double w = var == 1 ? 1.0L : (n == 0 ? 1.0L : 2.0L) / (long double)g.N;
                v = (double)(w * (c < 2 ? cosl(x) : sinl(x)));
              }
              ana[((((size_t)var * g.NU_tot + g.nu_off[c] + u) * g.NT + t) * 2 + e) * 32 + l] = v;
            }
  Tables T;
  if (int rc = upload_tables(syn, ana, &T)) return rc;
  g_tabs[{dev, g.m}] = T;
  *out = T;
  return SFNL_OK;
}

namespace {

constexpr bool third_fold(int M) { return M == 64 && tf_NT(M) % 2 == 0; }

// Tables of the third fold for m (a Geo with make_geo(m).N): synthesis B fragments
// [KS_tot][NT][32] (lane (g, q): mode tf_mode(gr, 4s + q), angle 8t + g) and analysis B fragments
// [2 variants][sum of NU * TE][32] (lane (g, q): mode tf_mode(gr, 8u + g), angle 8t + 2q + e; variant 0
// carries the analysis weights, variant 1 not).
std::mutex g_tftab_mu;
std::map<std::pair<int, int>, Tables> g_tftabs;  // (device, m) -> tables

}  // namespace

int get_tf_tables(const Geo &g, Tables *out) {
  int dev = 0;
  cudaGetDevice(&dev);
  std::lock_guard<std::mutex> lk(g_tftab_mu);
  auto it = g_tftabs.find({dev, g.m});
  if (it != g_tftabs.end()) {
    *out = it->second;
    return SFNL_OK;
  }
  const long double pi = acosl(-1.0L);
  auto ang = [&](int j) { return pi * (long double)(2 * j + 1) / (long double)g.N; };
  int ks_tot = 0, asteps = 0;
  for (int gr = 0; gr < 6; ++gr) {
    ks_tot += tf_KS(g.m, gr);
    asteps += tf_NU(g.m, gr) * tf_TE(g.m, gr);
  }
  std::vector<double> syn((size_t)ks_tot * g.NT * 32, 0.0);
  for (int gr = 0; gr < 6; ++gr)
    for (int s = 0; s < tf_KS(g.m, gr); ++s)
      for (int t = 0; t < g.NT; ++t)
        for (int l = 0; l < 32; ++l) {
          const int k = 4 * s + (l & 3), j = 8 * t + (l >> 2);
          double v = 0.0;
          if (k < tf_ke(g.m, gr)) {
            const long double x = (long double)tf_mode(gr, k) * ang(j);
            v = (double)(gr < 3 ? cosl(x) : sinl(x));
          }
          syn[(((size_t)(tf_koff(g.m, gr) + s)) * g.NT + t) * 32 + l] = v;
        }
  std::vector<double> ana((size_t)2 * asteps * 32, 0.0);
  for (int var = 0; var < 2; ++var)
    for (int gr = 0; gr < 6; ++gr)
      for (int u = 0; u < tf_NU(g.m, gr); ++u)
        for (int te = 0; te < tf_TE(g.m, gr); ++te)
          for (int l = 0; l < 32; ++l) {
            const int j = 8 * (te >> 1) + 2 * (l & 3) + (te & 1);
            const int kk = 8 * u + (l >> 2);
            double v = 0.0;
            if (kk < tf_ke(g.m, gr)) {
              const int n = tf_mode(gr, kk);
              const long double x = (long double)n * ang(j);
              const long double w = var == 1 ? 1.0L : (n == 0 ? 1.0L : 2.0L) / (long double)g.N;
              v = (double)(w * (gr < 3 ? cosl(x) : sinl(x)));
            }
            ana[(((size_t)var * asteps + tf_aoff(g.m, gr) + u * tf_TE(g.m, gr) + te) * 32) + l] = v;
          }
  Tables T;
  if (int rc = upload_tables(syn, ana, &T)) return rc;
  g_tftabs[{dev, g.m}] = T;
  *out = T;
  return SFNL_OK;
}

namespace {

// ---------------------------------------------------------------------------
// kernel
// ---------------------------------------------------------------------------
struct FastArgs {
  const double *in[12];
  double *out[9];
  int64_t in_ldm[12], out_ldm[9], in_bs[12], out_bs[9];
  int64_t out_ps;   // point stride of the outputs (3 in the tensor layout), sine at out_ps*np
  int64_t np;
  int m, N, NT;
  int ks_off[4], KS[4], nu_off[4], NU[4], ke[4];
  int NU_tot;
  int KT;           // staged coefficient rows per field (4 * total synthesis k-steps)
  unsigned adj_in;  // bit f: input field f is a cotangent (synthesise with D)
  int adj_out;      // 1: analyse without D (transpose of the synthesis)
  int accumulate;   // 1: out += result
  int vec16;        // 1: every input row starts 16-byte aligned (bases aligned, np even): 16-byte copies
  int allow_tf;     // 1: the third-fold kernel may be used (it allocates its own cached tables)
  const double *syn, *ana;
  GaussArgs ga;     // the Gauss-point staging of fast_kernel<..., GK >= 0>: node-major nodal fields (stride m)
};


template <int EK>
struct EKDef;
template <>
struct EKDef<EK_CROSS> {
  static constexpr int NI = 6, NO = 3;
  __device__ static void op(const double *x, double *y) { cross3(x, x + 3, y); }
};
template <>
struct EKDef<EK_DOT> {
  static constexpr int NI = 6, NO = 1;
  __device__ static void op(const double *x, double *y) { y[0] = x[0] * x[3] + x[1] * x[4] + x[2] * x[5]; }
};
template <>
struct EKDef<EK_PROD> {
  static constexpr int NI = 2, NO = 1;
  __device__ static void op(const double *x, double *y) { y[0] = x[0] * x[1]; }
};
template <>
struct EKDef<EK_SVECT> {
  static constexpr int NI = 4, NO = 3;
  __device__ static void op(const double *x, double *y) {
#pragma unroll
    for (int k = 0; k < 3; ++k) y[k] = x[3] * x[k];
  }
};
template <>
struct EKDef<EK_ADVECT> {  // [heat grad c 0-2, u 3-5, div u 6, heat c 7] -> grad c . u + div u c
  static constexpr int NI = 8, NO = 1;
  __device__ static void op(const double *x, double *y) {
    y[0] = fma(x[6], x[7], x[0] * x[3] + x[1] * x[4] + x[2] * x[5]);
  }
};
template <>
struct EKDef<EK_CROSS2> {  // fields [a, b, c, d] -> a x b + c x d, one pair (6 fields) per pass
  static constexpr int NI = 12, NO = 3;
  __device__ static void op(const double *x, double *y) { cross3(x, x + 3, y); }
};
template <>
struct EKDef<EK_TENSOR> {
  static constexpr int NI = 6, NO = 9;
  __device__ static void op(const double *x, double *y) {
#pragma unroll
    for (int k = 0; k < 3; ++k)
#pragma unroll
      for (int l = 0; l < 3; ++l) y[3 * k + l] = x[k] * x[3 + l];
  }
};
__host__ __device__ constexpr int ek_nin(int ek) {
  return ek == EK_PROD ? 2 : ek == EK_SVECT ? 4 : ek == EK_ADVECT ? 8 : ek == EK_CROSS2 ? 12 : 6;
}
// Synthesis passes of a program: EK_CROSS2 synthesises its two operand pairs one after the other through the
// accumulators of one pair and adds the second pair's products to the first's pre-folded ones.
__host__ __device__ constexpr int ek_passes(int ek) { return ek == EK_CROSS2 ? 2 : 1; }
__host__ __device__ constexpr int ek_nout(int ek) {
  return ek == EK_CROSS || ek == EK_SVECT || ek == EK_CROSS2 ? 3 : ek == EK_TENSOR ? 9 : 1;
}
// Shared memory of one CTA: folded products [NO][4][NT][2][32] and staged coefficients [NI][KT][8].
// With NT <= 8 angle tiles every warp (pair, with the class split) owns one tile and the products
// (and the exchange) overlay the coefficients.
// The class split (two warps per angle tile, one per class pair) halves the accumulators of a warp
// and doubles the warps per SM; it pays for the six-field programs at m >= 64, where the accumulator
// registers limit residency, and costs shared memory and a barrier elsewhere (measured on B200).
constexpr bool class_split(int ek, int M) { return (ek == EK_CROSS || ek == EK_DOT) && (M == 64 || M == 0); }
// With several passes the products (written after a barrier that ends pass 0's synthesis, added to in the
// later passes) may overlay only pass 0's coefficients.
__host__ __device__ constexpr bool fast_overlay(int ek, int NT, int KT) {
  return NT <= 8 && (ek_passes(ek) == 1 ||
                     (size_t)ek_nout(ek) * 4 * NT * 2 * 32 <= (size_t)ek_nin(ek) / ek_passes(ek) * KT * 8);
}
inline size_t fast_smem_bytes(int ek, int NT, int KT, bool cs) {
  const int nwt = NT < 8 ? NT : 8;
  const size_t prod = (size_t)ek_nout(ek) * 4 * NT * 2 * 32, coef = (size_t)ek_nin(ek) * KT * 8;
  const size_t xch = cs ? (size_t)nwt * ek_nin(ek) * 128 : 0;
  return sizeof(double) * (fast_overlay(ek, NT, KT) ? (prod + xch > coef ? prod + xch : coef) : prod + xch + coef);
}


// Geometry of make_geo as constant expressions (the kernels specialise on m).
__host__ __device__ constexpr int cg_qmin(int m) { return (3 * m - 2 + 3) / 4 < 1 ? 1 : (3 * m - 2 + 3) / 4; }
__host__ __device__ constexpr int cg_NT(int m) { return (cg_qmin(m) + 7) / 8; }
__host__ __device__ constexpr int cg_ke(int m, int c) { return (c & 1) ? m / 2 : (m + 1) / 2; }
__host__ __device__ constexpr int cg_KS(int m, int c) { return (cg_ke(m, c) + 3) / 4; }
__host__ __device__ constexpr int cg_NU(int m, int c) { return (cg_ke(m, c) + 7) / 8; }
__host__ __device__ constexpr int cg_ksoff(int m, int c) { return c == 0 ? 0 : cg_ksoff(m, c - 1) + cg_KS(m, c - 1); }
__host__ __device__ constexpr int cg_nuoff(int m, int c) { return c == 0 ? 0 : cg_nuoff(m, c - 1) + cg_NU(m, c - 1); }


// EK: elementary program; M: modes when specialised (0: any m, geometry at run time);
// ADJ: 0 plain, 1 first operand (fields 0-2) a cotangent, 2 second operand (fields 3-5) a cotangent.
// Launch bounds (measured on B200): the class-split cross product at m = 64 runs best at 3 CTAs of 12
// warps per SM (56 registers); the tensor program wants registers (no residency target); the others
// keep the compiler's default register target.
constexpr int fast_max_threads(int M, bool cs) { return cs ? (M == 64 ? 384 : 512) : 256; }
constexpr int fast_min_blocks(int ek, int M, bool cs) { return (cs && M == 64 && ek == EK_CROSS) ? 3 : ek == EK_TENSOR ? 1 : 0; }

// GK >= 0 (a Gauss-point caller, GK_*): the operands are built in the staging from the node-major nodal
// fields of a.ga instead of read from a.in (one batch entry).
template <int EK, int M, int ADJ, bool CS, int GK = -1>
__global__ void __launch_bounds__(fast_max_threads(M, CS),
                                  GK >= 0 && fast_min_blocks(EK, M, CS) > 2 ? 2 : fast_min_blocks(EK, M, CS))
    fast_kernel(const FastArgs a) {
  constexpr bool CT = M > 0;
  constexpr int NI = EKDef<EK>::NI, NO = EKDef<EK>::NO;
  // Shared memory: folded products ps [NO][4][NT][2][32], with the class split (CS) the exchange
  // between the two warps of an angle tile xc [NW/2][2][NI][2][32], and the staged coefficients
  // xs [NI][KT/4][4][8].  When every warp (pair) owns at most one angle tile, ps and xc overlay xs
  // (written after a barrier that ends the synthesis), which leaves L1 room for the DFT tables.
  extern __shared__ double smem[];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, NW = blockDim.x >> 5;
  const int g = lane >> 2, q = lane & 3;
  const int64_t p0 = (int64_t)blockIdx.x * 8, p = p0 + g;
  const bool valid = p < a.np;
  const int b = blockIdx.y;
  const int NT = CT ? cg_NT(M) : a.NT;
  int KS[4], KOFF[4], KE[4], NU[4], NOFF[4];
#pragma unroll
  for (int c = 0; c < 4; ++c) {
    KS[c] = CT ? cg_KS(M, c) : a.KS[c];
    KOFF[c] = CT ? cg_ksoff(M, c) : a.ks_off[c];
    KE[c] = CT ? cg_ke(M, c) : a.ke[c];
    NU[c] = CT ? cg_NU(M, c) : a.NU[c];
    NOFF[c] = CT ? cg_nuoff(M, c) : a.nu_off[c];
  }
  const int KS_tot = KS[0] + KS[1] + KS[2] + KS[3], KT = 4 * KS_tot;
  const int NU_tot = NU[0] + NU[1] + NU[2] + NU[3];
  int ks_max = KS[0];
#pragma unroll
  for (int c = 1; c < 4; ++c) ks_max = KS[c] > ks_max ? KS[c] : ks_max;
  const double invN = 1.0 / (4.0 * 8.0 * NT), twoN = 2.0 * invN;

  // ---- stage the tile's coefficients ----
  // Global row r = 4*ks + q of field f (class c, mode index k = r - 4*KOFF[c]) holds 8 points; it
  // lands at xs[(f*KS_tot + ks)*32 + a_frag_slot(q, point)], so that lane (g, q) of a warp reads the
  // A fragment of k-step ks from one 256-byte block without bank conflicts.  Four
  // consecutive threads copy one row (two points each, one 16-byte copy when the row is 16-byte
  // aligned), so a warp instruction moves 8 whole 64-byte rows.
  const int NWT = CS ? NW >> 1 : NW;  // angle tiles per pass (two warps per tile with the class split)
  constexpr int NPASS = ek_passes(EK), NIP = NI / NPASS;  // synthesis passes, fields per pass
  static_assert(NPASS == 1 || (!CS && GK < 0), "passes: the four-class kernel on staged fields only");
  const bool overlay = NT <= NWT && fast_overlay(EK, NT, KT);
  const size_t prod_d = (size_t)NO * 4 * NT * 2 * 32, xch_d = CS ? (size_t)NWT * NI * 128 : 0;
  double *ps = smem, *xc = smem + prod_d;
  double *xs = overlay ? smem : smem + prod_d + xch_d;
  if constexpr (GK >= 0) {
    // the operands of the tile's 8 Gauss points and every mode, from the nodal fields: mode i's cosine
    // row is 4*KOFF[i & 1] + (i >> 1), its sine row 4*KOFF[2 + (i & 1)] + (i >> 1); other rows stay 0
    for (int t = threadIdx.x; t < NI * KS_tot * 32; t += blockDim.x) xs[t] = 0.0;
    __syncthreads();
    const int m = CT ? M : a.m;
    for (int it = threadIdx.x; it < 8 * m; it += blockDim.x) {
      const int i = it % m, gp = it / m;  // a warp takes consecutive modes of one point
      if (p0 + gp >= a.np) continue;
      double f[8][2];
      gauss_operands_nm<GK>(a.ga, p0 + gp, i, m, f);
      const int c = i & 1, k = i >> 1;
      const int rc = 4 * sel4(KOFF, c) + k, rs = 4 * sel4(KOFF, 2 + c) + k;
      const int oc = (rc >> 2) * 32 + a_frag_slot(rc & 3, gp), os = (rs >> 2) * 32 + a_frag_slot(rs & 3, gp);
#pragma unroll
      for (int fi = 0; fi < NI; ++fi) {
        xs[(size_t)fi * KS_tot * 32 + oc] = f[fi][0];
        if (i != 0) xs[(size_t)fi * KS_tot * 32 + os] = f[fi][1];  // the sine of mode 0 is ignored
      }
    }
  } else {
    const int pc = 2 * (threadIdx.x & 3), rstep = blockDim.x >> 2;
    const bool v16 = a.vec16 && p0 + 8 <= a.np;
    const bool pv0 = p0 + pc < a.np, pv1 = p0 + pc + 1 < a.np;
    if constexpr (M != 0) {
      // rows outermost: the row's class, mode and sine offset are decoded once for the NI fields
      for (int r = threadIdx.x >> 2; r < KT; r += rstep) {
        const int c = (r >= 4 * KOFF[1]) + (r >= 4 * KOFF[2]) + (r >= 4 * KOFF[3]);
        const int k = r - 4 * sel4(KOFF, c), n = class_mode(c, k);
        double *dst0 = xs + (size_t)(r >> 2) * 32 + a_frag_slot(r & 3, pc);
        const bool live = k < sel4(KE, c) && !(c == 2 && n == 0);  // the sine of mode 0 is ignored
        const int64_t off = p0 + pc + (c >= 2 ? a.np : 0);
#pragma unroll
        for (int f = 0; f < NI; ++f) {
          double *dst = dst0 + (size_t)f * KS_tot * 32;
          const double *src = a.in[f] + (int64_t)b * a.in_bs[f] + off + (int64_t)n * a.in_ldm[f];
          if (live && v16) {
            cp_async16(dst, src);
          } else {
            if (live && pv0) cp_async8(dst, src); else dst[0] = 0.0;
            if (live && pv1) cp_async8(dst + 1, src + 1); else dst[1] = 0.0;
          }
        }
      }
    } else {  // run-time geometry: fields outermost (measured faster there)
#pragma unroll
      for (int f = 0; f < NI; ++f) {
        const double *base = a.in[f] + (int64_t)b * a.in_bs[f] + p0 + pc;
        const int64_t ldm = a.in_ldm[f];
        double *xf = xs + (size_t)f * KS_tot * 32;
        for (int r = threadIdx.x >> 2; r < KT; r += rstep) {
          const int c = (r >= 4 * KOFF[1]) + (r >= 4 * KOFF[2]) + (r >= 4 * KOFF[3]);
          const int k = r - 4 * sel4(KOFF, c), n = class_mode(c, k);
          double *dst = xf + (size_t)(r >> 2) * 32 + a_frag_slot(r & 3, pc);
          const bool live = k < sel4(KE, c) && !(c == 2 && n == 0);  // the sine of mode 0 is ignored
          const double *src = base + (int64_t)n * ldm + (c >= 2 ? a.np : 0);
          if (live && v16) {
            cp_async16(dst, src);
          } else {
            if (live && pv0) cp_async8(dst, src); else dst[0] = 0.0;
            if (live && pv1) cp_async8(dst + 1, src + 1); else dst[1] = 0.0;
          }
        }
      }
    }
  }
  cp_async_wait_all();
  __syncthreads();

  if constexpr (CS) {
    // ---- synthesis, fold, program, analysis pre-fold ----
    // The two warps of angle tile t split the classes: warp half 0 accumulates the cosine classes
    // (CE, CO), half 1 the sine classes (SE, SO), 2*NI accumulator chains each.  They then swap half of
    // their folded sums (A = CE+CO, B = CE-CO against C = SE+SO, D = SO-SE) through shared memory, and
    // half e evaluates the program and the analysis pre-fold for the angles of k-step parity e.
    const int wp = warp >> 1, half = warp & 1;
    for (int t0 = 0; t0 < NT; t0 += NWT) {  // one pass when ps and xc overlay the coefficients
      const int t = t0 + wp;
      double acc[NI][2][2];
#pragma unroll
      for (int f = 0; f < NI; ++f)
#pragma unroll
        for (int cc = 0; cc < 2; ++cc) acc[f][cc][0] = acc[f][cc][1] = 0.0;
      auto synth = [&](auto cb_tag) {
        constexpr int CB = decltype(cb_tag)::value;  // first class of this warp's pair
        const double *syn_t = a.syn + (size_t)t * 32 + lane;
        const double *xs_l = xs + a_frag_slot(lane & 3, lane >> 2);
#pragma unroll
        for (int s = 0; s < ks_max; ++s) {
#pragma unroll
          for (int cc = 0; cc < 2; ++cc) {
            const int c = CB + cc;
            if (s >= KS[c]) continue;
            const double bv = __ldg(syn_t + (size_t)(KOFF[c] + s) * NT * 32);
            const double *xa = xs_l + (size_t)(KOFF[c] + s) * 32;
            double av[NI];
#pragma unroll
            for (int f = 0; f < NI; ++f) av[f] = xa[(size_t)f * KS_tot * 32];
            if constexpr (ADJ != 0) {
              const double wn = (s == 0 && q == 0 && (c & 1) == 0) ? invN : twoN;  // n == 0 only there
#pragma unroll
              for (int f = 0; f < NI; ++f)
                if ((ADJ == 1 && f < 3) || (ADJ == 2 && f >= 3)) av[f] *= wn;
            }
#pragma unroll
            for (int f = 0; f < NI; ++f) dmma(acc[f][cc], av[f], bv);
          }
        }
      };
      if (t < NT) {
        if (half == 0)
          synth(std::integral_constant<int, 0>{});
        else
          synth(std::integral_constant<int, 2>{});
      }
      if (overlay) __syncthreads();  // every warp has read its last coefficient
      // sums and differences of the pair's classes at parity e: (A, B) for half 0, (C, D) for half 1
      auto pair_sums = [&](int f, int e, double &X, double &Y) {
        const double lo = e ? acc[f][0][1] : acc[f][0][0], hi = e ? acc[f][1][1] : acc[f][1][0];
        X = lo + hi;
        Y = half ? hi - lo : lo - hi;
      };
      double *xw = xc + (size_t)wp * 2 * NI * 64 + lane;  // [writer half][f][X, Y][32]
      if (t < NT) {
#pragma unroll
        for (int f = 0; f < NI; ++f) {
          double X, Y;
          pair_sums(f, 1 - half, X, Y);  // the parity the partner finishes
          xw[((half * NI + f) * 2 + 0) * 32] = X;
          xw[((half * NI + f) * 2 + 1) * 32] = Y;
        }
      }
      __syncthreads();
      if (t < NT) {
        const int e = half;
        double v[4][NI];
#pragma unroll
        for (int f = 0; f < NI; ++f) {
          double X, Y;
          pair_sums(f, e, X, Y);
          const double Xp = xw[(((1 - half) * NI + f) * 2 + 0) * 32], Yp = xw[(((1 - half) * NI + f) * 2 + 1) * 32];
          const double A = half ? Xp : X, B = half ? Yp : Y, C = half ? X : Xp, D = half ? Y : Yp;
          v[0][f] = A + C;  // theta
          v[1][f] = B + D;  // pi - theta
          v[2][f] = B - D;  // pi + theta
          v[3][f] = A - C;  // 2 pi - theta
        }
        double gq[4][NO];
#pragma unroll
        for (int r = 0; r < 4; ++r) EKDef<EK>::op(v[r], gq[r]);
#pragma unroll
        for (int o = 0; o < NO; ++o) {
          const double s14 = gq[0][o] + gq[3][o], d14 = gq[0][o] - gq[3][o];
          const double s23 = gq[1][o] + gq[2][o], d32 = gq[2][o] - gq[1][o];
          double *dst = ps + ((size_t)((o * 4) * NT + t) * 2 + e) * 32 + lane;
          const size_t cstride = (size_t)NT * 2 * 32;
          dst[0] = s14 + s23;            // PE
          dst[cstride] = s14 - s23;      // PO
          dst[2 * cstride] = d14 + d32;  // QE
          dst[3 * cstride] = d14 - d32;  // QO
        }
      }
      if (!overlay) __syncthreads();  // xc is rewritten by the next pass
    }
    __syncthreads();

  } else {
    // ---- synthesis, fold, program, analysis pre-fold ----
    for (int t0 = 0; t0 < NT; t0 += NW) {  // one pass when the products overlay the coefficients
      const int t = t0 + warp;
      // NPASS > 1: the operand pairs one after the other, fields NIP*pass .. NIP*pass+NIP-1; the products
      // overlay only pass 0's coefficients, and the later passes add theirs to the pre-folded ones
#pragma unroll 1
      for (int pass = 0; pass < NPASS; ++pass) {
      double acc[NIP][4][2];
#pragma unroll
      for (int f = 0; f < NIP; ++f)
#pragma unroll
        for (int c = 0; c < 4; ++c) acc[f][c][0] = acc[f][c][1] = 0.0;
      if (t < NT) {
      // k-steps outermost, the four classes inside: 4*NIP independent accumulator chains per step
      const double *syn_t = a.syn + (size_t)t * 32 + lane;
      const double *xs_l = xs + (size_t)pass * NIP * KS_tot * 32 + a_frag_slot(lane & 3, lane >> 2);
#pragma unroll
      for (int s = 0; s < ks_max; ++s) {
#pragma unroll
        for (int c = 0; c < 4; ++c) {
          if (s >= KS[c]) continue;
          const double bv = __ldg(syn_t + (size_t)(KOFF[c] + s) * NT * 32);
          const double *xa = xs_l + (size_t)(KOFF[c] + s) * 32;
          double av[NIP];
#pragma unroll
          for (int f = 0; f < NIP; ++f) av[f] = xa[(size_t)f * KS_tot * 32];
          if constexpr (ADJ != 0) {
            const double wn = (s == 0 && q == 0 && (c & 1) == 0) ? invN : twoN;  // n == 0 only there
            // ADJ 1 / 2: the first / second operand (of every pass)
#pragma unroll
            for (int f = 0; f < NIP; ++f)
              if ((ADJ == 1 && f < 3) || (ADJ == 2 && f >= 3)) av[f] *= wn;
          }
#pragma unroll
          for (int f = 0; f < NIP; ++f) dmma(acc[f][c], av[f], bv);
        }
      }
      }
      if (overlay && pass == 0) __syncthreads();  // every warp has read pass 0's last coefficient
      if (t < NT) {
#pragma unroll
      for (int e = 0; e < 2; ++e) {
        double v[4][NIP];
#pragma unroll
        for (int f = 0; f < NIP; ++f) {
          const double A = acc[f][0][e] + acc[f][1][e], B = acc[f][0][e] - acc[f][1][e];
          const double C = acc[f][2][e] + acc[f][3][e], D = acc[f][3][e] - acc[f][2][e];
          v[0][f] = A + C;  // theta
          v[1][f] = B + D;  // pi - theta
          v[2][f] = B - D;  // pi + theta
          v[3][f] = A - C;  // 2 pi - theta
        }
        double gq[4][NO];
#pragma unroll
        for (int r = 0; r < 4; ++r) EKDef<EK>::op(v[r], gq[r]);
#pragma unroll
        for (int o = 0; o < NO; ++o) {
          const double s14 = gq[0][o] + gq[3][o], d14 = gq[0][o] - gq[3][o];
          const double s23 = gq[1][o] + gq[2][o], d32 = gq[2][o] - gq[1][o];
          double *dst = ps + ((size_t)((o * 4) * NT + t) * 2 + e) * 32 + lane;
          const size_t cstride = (size_t)NT * 2 * 32;
          const double pe = s14 + s23, po = s14 - s23, qe = d14 + d32, qo = d14 - d32;
          if (pass == 0) {
            dst[0] = pe;
            dst[cstride] = po;
            dst[2 * cstride] = qe;
            dst[3 * cstride] = qo;
          } else {  // the same lane wrote these in pass 0
            dst[0] += pe;
            dst[cstride] += po;
            dst[2 * cstride] += qe;
            dst[3 * cstride] += qo;
          }
        }
      }
      }
      }
    }
    __syncthreads();

  }

  // ---- analysis: output tiles (class c, tile u) ----
  const double *anav = a.ana + (size_t)(a.adj_out ? 1 : 0) * NU_tot * NT * 2 * 32 + lane;
  for (int cu = warp; cu < NU_tot; cu += NW) {
    const int c = (cu >= NOFF[1]) + (cu >= NOFF[2]) + (cu >= NOFF[3]);
    const int u = cu - sel4(NOFF, c), kec = sel4(KE, c);
    // PC partial sums per output over alternating k-steps: NO*PC independent accumulator chains
    constexpr int PC = NO >= 6 ? 1 : NO >= 3 ? 2 : 4;
    double y[NO][2], yp[PC][NO][2];
#pragma unroll
    for (int i = 0; i < PC; ++i)
#pragma unroll
      for (int o = 0; o < NO; ++o) yp[i][o][0] = yp[i][o][1] = 0.0;
    const double *bt = anav + (size_t)cu * NT * 2 * 32;
    const double *pa = ps + (size_t)c * NT * 2 * 32 + lane;
#pragma unroll
    for (int te = 0; te < 2 * NT; ++te) {
      const double bv = __ldg(bt + (size_t)te * 32);
#pragma unroll
      for (int o = 0; o < NO; ++o) dmma(yp[te % PC][o], pa[((size_t)o * 4 * NT * 2 + te) * 32], bv);
    }
#pragma unroll
    for (int o = 0; o < NO; ++o)
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        y[o][h] = yp[0][o][h];
#pragma unroll
        for (int i = 1; i < PC; ++i) y[o][h] += yp[i][o][h];
      }
    if (!valid) continue;
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const int kk = 8 * u + 2 * q + h;
      if (kk >= kec) continue;
      const int n = class_mode(c, kk);
#pragma unroll
      for (int o = 0; o < NO; ++o) {
        double *dst = a.out[o] + (int64_t)b * a.out_bs[o] + p * a.out_ps + (int64_t)n * a.out_ldm[o] +
                      (c >= 2 ? a.np * a.out_ps : 0);
        const double v = (c == 2 && n == 0) ? 0.0 : y[o][h];
        if (a.accumulate)
          *dst += v;
        else
          *dst = v;
      }
    }
  }
}

// ---------------------------------------------------------------------------
// third-fold building blocks (class split, one angle tile per warp pair, M with tf_NT(M) even)
// ---------------------------------------------------------------------------
// Warp w of a CTA: angle tile tau = w / 2, half h = w % 2 (0: cosine classes, 1: sine classes).  It
// accumulates the odd class of half h on tile tau and one part of the even class of half h on tile
// min(tau, NT-1-tau): E0 (n = 0 mod 4) for the first half of the tiles, E2 (n = 2 mod 4) for the second.
template <int M>
struct TfGeo {
  static constexpr int NT = tf_NT(M), NH = NT / 2, KS_tot = tf_koff(M, 6), KT = 4 * KS_tot;
  static constexpr int NU_tot = tf_nuoff(M, 6), ASTEPS = tf_aoff(M, 6);
};
template <int NG>
struct FieldSet {  // NG scalar fields: cos of mode n, point p at p[f][p + n*ldm[f]], sine np further
  const double *p[NG];
  int64_t ldm[NG];
};

// Stages the NG fields of the 8-point tile at p0 into xs [NG][KS_tot][4][8] (rows in group order:
// CE0, CE2, CO, SE0, SE2, SO) with cp.async and commits one group.  Four consecutive threads copy one
// row (two points each, one 16-byte copy when the row is 16-byte aligned).
template <int M, int NG>
__device__ __forceinline__ void tf_stage(double *xs, const FieldSet<NG> &fs, int64_t p0, int64_t np, bool vec16) {
  constexpr int KS_tot = TfGeo<M>::KS_tot, KT = TfGeo<M>::KT;
  const int pc = 2 * (threadIdx.x & 3), rstep = blockDim.x >> 2;
  const bool v16 = vec16 && p0 + 8 <= np;
  const bool pv0 = p0 + pc < np, pv1 = p0 + pc + 1 < np;
  // rows outermost: the row's group, mode and sine offset are decoded once for the NG fields
  for (int r = threadIdx.x >> 2; r < KT; r += rstep) {
    const int gr = (r >= 4 * tf_koff(M, 1)) + (r >= 4 * tf_koff(M, 2)) + (r >= 4 * tf_koff(M, 3)) +
                   (r >= 4 * tf_koff(M, 4)) + (r >= 4 * tf_koff(M, 5));
    const int kg = gr == 0 ? 0 : gr == 1 ? tf_koff(M, 1) : gr == 2 ? tf_koff(M, 2) : gr == 3 ? tf_koff(M, 3)
                 : gr == 4 ? tf_koff(M, 4) : tf_koff(M, 5);
    const int keg = gr % 3 == 0 ? tf_ke(M, 0) : gr % 3 == 1 ? tf_ke(M, 1) : tf_ke(M, 2);
    const int k = r - 4 * kg, n = tf_mode(gr, k);
    double *dst0 = xs + (size_t)(r >> 2) * 32 + a_frag_slot(r & 3, pc);
    const bool live = k < keg && !(gr == 3 && k == 0);  // the sine of mode 0 is ignored
    const int64_t off = p0 + pc + (gr >= 3 ? np : 0);
#pragma unroll
    for (int f = 0; f < NG; ++f) {
      double *dst = dst0 + (size_t)f * KS_tot * 32;
      const double *src = fs.p[f] + off + (int64_t)n * fs.ldm[f];
      if (live && v16) {
        cp_async16(dst, src);
      } else {
        if (live && pv0) cp_async8(dst, src); else dst[0] = 0.0;
        if (live && pv1) cp_async8(dst + 1, src + 1); else dst[1] = 0.0;
      }
    }
  }
  cp_async_commit();
}

// Synthesis of NG staged fields: the warp's even part and odd class.  ADJ: bit f set = field f is a
// cotangent (synthesised with the analysis weights).
template <int M, int NG, unsigned ADJ>
__device__ __forceinline__ void tf_synth(const double *xs, const double *syn, double (&acc_e)[NG][2],
                                         double (&acc_o)[NG][2]) {
  constexpr int NT = TfGeo<M>::NT, NH = TfGeo<M>::NH, KS_tot = TfGeo<M>::KS_tot;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, q = lane & 3;
  const int tau = warp >> 1, half = warp & 1;
  const bool first = tau < NH;
  const int te_tile = first ? tau : NT - 1 - tau;
  const double invN = 1.0 / (4.0 * 8.0 * NT), twoN = 2.0 * invN;
#pragma unroll
  for (int f = 0; f < NG; ++f) acc_e[f][0] = acc_e[f][1] = acc_o[f][0] = acc_o[f][1] = 0.0;
  const int ge = 3 * half + (first ? 0 : 1);
  const int koff_e = ge == 0 ? tf_koff(M, 0) : ge == 1 ? tf_koff(M, 1) : ge == 3 ? tf_koff(M, 3) : tf_koff(M, 4);
  const int ks_e = (ge % 3 == 0) ? tf_KS(M, 0) : tf_KS(M, 1);
  const int koff_o = half ? tf_koff(M, 5) : tf_koff(M, 2);
  const double *xs_l = xs + a_frag_slot(lane & 3, lane >> 2);
  const double *syn_e = syn + (size_t)te_tile * 32 + lane, *syn_o = syn + (size_t)tau * 32 + lane;
  constexpr int KSE = tf_KS(M, 0) > tf_KS(M, 1) ? tf_KS(M, 0) : tf_KS(M, 1);
  // the next k-step's B fragment is loaded while the current one feeds the DMMAs (the table is read from L2)
  double bnext = __ldg(syn_e + (size_t)koff_e * NT * 32);
#pragma unroll
  for (int s = 0; s < KSE; ++s) {
    if (s >= ks_e) break;
    const double bv = bnext;
    bnext = s + 1 < ks_e ? __ldg(syn_e + (size_t)(koff_e + s + 1) * NT * 32) : __ldg(syn_o + (size_t)koff_o * NT * 32);
    const double *xa = xs_l + (size_t)(koff_e + s) * 32;
    double av[NG];
#pragma unroll
    for (int f = 0; f < NG; ++f) av[f] = xa[(size_t)f * KS_tot * 32];
    if constexpr (ADJ != 0) {
      const double wn = (s == 0 && q == 0 && ge % 3 == 0) ? invN : twoN;  // n == 0 only there
#pragma unroll
      for (int f = 0; f < NG; ++f)
        if ((ADJ >> f) & 1u) av[f] *= wn;
    }
#pragma unroll
    for (int f = 0; f < NG; ++f) dmma(acc_e[f], av[f], bv);
  }
#pragma unroll
  for (int s = 0; s < tf_KS(M, 2); ++s) {
    const double bv = bnext;
    if (s + 1 < tf_KS(M, 2)) bnext = __ldg(syn_o + (size_t)(koff_o + s + 1) * NT * 32);
    const double *xa = xs_l + (size_t)(koff_o + s) * 32;
    double av[NG];
#pragma unroll
    for (int f = 0; f < NG; ++f) av[f] = xa[(size_t)f * KS_tot * 32];
    if constexpr (ADJ != 0) {
#pragma unroll
      for (int f = 0; f < NG; ++f)
        if ((ADJ >> f) & 1u) av[f] *= twoN;
    }
#pragma unroll
    for (int f = 0; f < NG; ++f) dmma(acc_o[f], av[f], bv);
  }
}

// Both exchanges of the CTA's warps (fold_exchange with the CTA barrier; call with every thread, after a
// barrier that ends the reads of whatever xc overlays).  xc holds 2 * NT * NG * 64 doubles.
template <int M, int NG>
__device__ __forceinline__ void tf_fold(const double (&acc_e)[NG][2], const double (&acc_o)[NG][2], double *xc,
                                        double (&v)[4][NG]) {
  const int warp = threadIdx.x >> 5;
  fold_exchange<TfGeo<M>::NT, NG>(acc_e, acc_o, xc, warp >> 1, warp & 1, CtaSync{}, v);
}

// Analysis pre-fold of NO program outputs gq[quadrant][o] at the warp's angles (tile tau, parity half)
// into ps slots slot0 .. slot0+NO-1 ([slot][class][NT][2][32]).
template <int M, int NO>
__device__ __forceinline__ void tf_prefold(const double (&gq)[4][NO], double *ps, int slot0) {
  const int warp = threadIdx.x >> 5;
  prefold_store<TfGeo<M>::NT, NO>(gq, ps, slot0, warp >> 1, warp & 1);
}

template <int NO>
struct OutSet {  // NO output fields: cos of mode n, point p at p[o][p*ps + n*ldm[o]], sine np*ps further
  double *p[NO];
  int64_t ldm[NO];
};

// Analysis of ps slots 0..NO-1 into the outputs (every warp, output tiles cu = warp, warp + NW, ...): the
// even output groups over the first half of the tiles with P(t) +- P(mirror).  ana: the analysis table
// variant (weights or not); accumulate: add to the outputs.
template <int M, int NO>
__device__ __forceinline__ void tf_analysis(const double *ps, const double *ana, const OutSet<NO> &os, int64_t p0,
                                            int64_t np, int64_t out_ps, bool accumulate) {
  constexpr int NT = TfGeo<M>::NT, NU_tot = TfGeo<M>::NU_tot;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, NW = blockDim.x >> 5;
  const int q = lane & 3;
  const int64_t p = p0 + (lane >> 2);
  const bool valid = p < np;
  const double *anav = ana + lane;
  // Output tiles of the odd groups cost 2*NT k-steps, those of the even groups NT (mirror-folded): the
  // odd tiles go one per warp and the even ones two per remaining warp (M = 64, 12 warps: 8 + 4 x 2, every
  // warp 12 k-steps), else round robin.
  constexpr int NU0 = tf_NU(M, 0), NU1 = tf_NU(M, 1), NU3 = tf_NU(M, 3), NU4 = tf_NU(M, 4);
  constexpr int n_odd = tf_NU(M, 2) + tf_NU(M, 5), n_even = NU_tot - n_odd;
  const bool balanced = n_odd < NW;
  const int nwe = NW - n_odd;
  for (int j = 0;; ++j) {
    int cu;
    if (balanced) {
      if (warp < n_odd) {
        if (j > 0) break;
        cu = warp < tf_NU(M, 2) ? tf_nuoff(M, 2) + warp : tf_nuoff(M, 5) + warp - tf_NU(M, 2);
      } else {
        const int k = warp - n_odd + j * nwe;
        if (k >= n_even) break;
        cu = k < NU0 ? k : k < NU0 + NU1 ? tf_nuoff(M, 1) + k - NU0
           : k < NU0 + NU1 + NU3 ? tf_nuoff(M, 3) + k - NU0 - NU1 : tf_nuoff(M, 4) + k - NU0 - NU1 - NU3;
      }
    } else {
      cu = warp + j * NW;
      if (cu >= NU_tot) break;
    }
    (void)NU4;
    const int gr = (cu >= tf_nuoff(M, 1)) + (cu >= tf_nuoff(M, 2)) + (cu >= tf_nuoff(M, 3)) +
                   (cu >= tf_nuoff(M, 4)) + (cu >= tf_nuoff(M, 5));
    const int nuo = gr == 0 ? 0 : gr == 1 ? tf_nuoff(M, 1) : gr == 2 ? tf_nuoff(M, 2) : gr == 3 ? tf_nuoff(M, 3)
                  : gr == 4 ? tf_nuoff(M, 4) : tf_nuoff(M, 5);
    const int aof = gr == 0 ? 0 : gr == 1 ? tf_aoff(M, 1) : gr == 2 ? tf_aoff(M, 2) : gr == 3 ? tf_aoff(M, 3)
                  : gr == 4 ? tf_aoff(M, 4) : tf_aoff(M, 5);
    const bool odd = gr % 3 == 2;
    const int u = cu - nuo, TE = odd ? 2 * NT : NT, c = gr < 3 ? (odd ? 1 : 0) : (odd ? 3 : 2);
    const int keg = gr % 3 == 0 ? tf_ke(M, 0) : gr % 3 == 1 ? tf_ke(M, 1) : tf_ke(M, 2);
    // mirror sign of the even groups: PE0 +, PE2 -, QE0 -, QE2 +
    const double sg = (gr == 0 || gr == 4) ? 1.0 : -1.0;
    constexpr int PC = NO >= 6 ? 1 : NO >= 3 ? 2 : 4;
    double yp[PC][NO][2];
#pragma unroll
    for (int i = 0; i < PC; ++i)
#pragma unroll
      for (int o = 0; o < NO; ++o) yp[i][o][0] = yp[i][o][1] = 0.0;
    const double *bt = anav + (size_t)(aof + u * TE) * 32;
    const double *pa = ps + (size_t)c * NT * 2 * 32;
    double bnext = __ldg(bt);  // the next k-step's B fragment is loaded while the current one is used
#pragma unroll
    for (int te = 0; te < 2 * NT; ++te) {
      if (te >= TE) break;
      const double bv = bnext;
      if (te + 1 < TE) bnext = __ldg(bt + (size_t)(te + 1) * 32);
      const int t = te >> 1, e = te & 1;
#pragma unroll
      for (int o = 0; o < NO; ++o) {
        const double *po = pa + (size_t)o * 4 * NT * 2 * 32;
        double av = po[(t * 2 + e) * 32 + lane];
        if (!odd) av += sg * po[((NT - 1 - t) * 2 + 1 - e) * 32 + (lane ^ 3)];
        dmma(yp[te % PC][o], av, bv);
      }
    }
    double y[NO][2];
#pragma unroll
    for (int o = 0; o < NO; ++o)
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        y[o][h] = yp[0][o][h];
#pragma unroll
        for (int i = 1; i < PC; ++i) y[o][h] += yp[i][o][h];
      }
    if (!valid) continue;
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const int kk = 8 * u + 2 * q + h;
      if (kk >= keg) continue;
      const int n = tf_mode(gr, kk);
#pragma unroll
      for (int o = 0; o < NO; ++o) {
        double *dst = os.p[o] + p * out_ps + (int64_t)n * os.ldm[o] + (gr >= 3 ? np * out_ps : 0);
        const double v = (gr >= 3 && n == 0) ? 0.0 : y[o][h];
        if (accumulate)
          *dst += v;
        else
          *dst = v;
      }
    }
  }
}

// The FAST kernel with the third fold (one elementary program, class split, NT even: M = 64).
template <int EK, int M, int ADJ>
__global__ void __launch_bounds__(384, EK == EK_CROSS ? 3 : 0) fast_tf_kernel(const FastArgs a) {
  static_assert(third_fold(M), "third fold needs the specialised geometry");
  constexpr int NI = EKDef<EK>::NI, NO = EKDef<EK>::NO, NT = TfGeo<M>::NT;
  constexpr unsigned ADJMASK = ADJ == 1 ? 0x07u : ADJ == 2 ? 0x38u : 0u;
  extern __shared__ double smem[];
  const int b = blockIdx.y;
  const int64_t p0 = (int64_t)blockIdx.x * 8;
  constexpr size_t prod_d = (size_t)NO * 4 * NT * 2 * 32;
  double *ps = smem, *xc = smem + prod_d, *xs = smem;  // ps and xc overlay xs after the synthesis
  FieldSet<NI> fs;
#pragma unroll
  for (int f = 0; f < NI; ++f) {
    fs.p[f] = a.in[f] + (int64_t)b * a.in_bs[f];
    fs.ldm[f] = a.in_ldm[f];
  }
  tf_stage<M, NI>(xs, fs, p0, a.np, a.vec16);
  cp_async_wait_0();
  __syncthreads();
  double acc_e[NI][2], acc_o[NI][2];
  tf_synth<M, NI, ADJMASK>(xs, a.syn, acc_e, acc_o);
  __syncthreads();  // every warp has read its last coefficient: xc and ps may overwrite xs
  double v[4][NI];
  tf_fold<M, NI>(acc_e, acc_o, xc, v);
  double gq[4][NO];
#pragma unroll
  for (int r = 0; r < 4; ++r) EKDef<EK>::op(v[r], gq[r]);
  tf_prefold<M, NO>(gq, ps, 0);
  __syncthreads();
  OutSet<NO> os;
#pragma unroll
  for (int o = 0; o < NO; ++o) {
    os.p[o] = a.out[o] + (int64_t)b * a.out_bs[o];
    os.ldm[o] = a.out_ldm[o];
  }
  tf_analysis<M, NO>(ps, a.ana + (size_t)(a.adj_out ? 1 : 0) * TfGeo<M>::ASTEPS * 32, os, p0, a.np, a.out_ps,
                     a.accumulate != 0);
}

// The Gauss-point cross products with their operands built in the staging (third fold, M = 64):
// Navier-Stokes (curl u + 2 Om) x u (GK_NS) and Lorentz force (curl H) x B (GK_LORENTZ).  The tile's
// 8 Gauss points get the curl and values of every mode straight from the nodal fields (node-major
// copies: the element's nodes gathered through jj, the lanes of a warp reading 32 consecutive modes of
// one node) into the coefficient layout, so the (l_G*me, 6, m) operand arrays never go through HBM.
template <int M, int KIND>
__global__ void __launch_bounds__(384, 2) gauss_tf_cross_kernel(const FastArgs a, const GaussArgs ga) {
  static_assert(third_fold(M), "third fold needs the specialised geometry");
  constexpr int NI = 6, NO = 3, NT = TfGeo<M>::NT, KS_tot = TfGeo<M>::KS_tot;
  constexpr size_t fstride = (size_t)KS_tot * 32;
  extern __shared__ double smem[];
  const int64_t p0 = (int64_t)blockIdx.x * 8;
  constexpr size_t prod_d = (size_t)NO * 4 * NT * 2 * 32;
  double *ps = smem, *xc = smem + prod_d, *xs = smem;  // ps and xc overlay xs after the synthesis
  constexpr int NW = 6;  // P2 elements
  __shared__ int s_node[8][NW];
  __shared__ double s_wt[8][NW], s_g1[8][NW], s_g2[8][NW], s_ray[8];
  for (int t = threadIdx.x; t < NI * (int)fstride; t += blockDim.x) xs[t] = 0.0;  // padding rows, sine of mode 0
  if (threadIdx.x < 8 * NW) {  // the points' nodes, basis values and derivatives (mesh%jj, ww, dw)
    const int g = threadIdx.x / NW, n = threadIdx.x % NW;
    const int64_t p = p0 + g < a.np ? p0 + g : a.np - 1;
    const int me = (int)(p / ga.l_G), l = (int)(p % ga.l_G);
    int node = ga.jj[n + (size_t)NW * me] - 1;
    node = node < 0 ? 0 : node >= ga.np_nodes ? ga.np_nodes - 1 : node;  // no access outside the fields
    s_node[g][n] = node;
    s_wt[g][n] = ga.ww[n + (size_t)NW * l];
    const double *dwl = ga.dw + (size_t)2 * NW * (l + (size_t)ga.l_G * me);
    s_g1[g][n] = dwl[2 * n];
    s_g2[g][n] = dwl[2 * n + 1];
  }
  __syncthreads();
  if (threadIdx.x < 8) {  // radius of the point: sum rr(1, nodes) ww
    double ray = 0.0;
#pragma unroll
    for (int n = 0; n < NW; ++n) ray = fma(ga.rr[2 * (size_t)s_node[threadIdx.x][n]], s_wt[threadIdx.x][n], ray);
    s_ray[threadIdx.x] = ray;
  }
  __syncthreads();
  for (int it = threadIdx.x; it < 8 * M; it += blockDim.x) {
    const int i = it % M, g = it / M;  // mode index, point of the tile: a warp reads 32 modes of a node
    if (p0 + g >= a.np) continue;
    double rot[6], w[6];
    gauss_curl_gathered<KIND, M, NW>(ga, s_node[g], s_wt[g], s_g1[g], s_g2[g], s_ray[g], i, rot, w);
    // rows of mode i: cosine group CE0 (i = 0 mod 4), CE2 (i = 2 mod 4) or CO (odd), sine group 3 further
    const int gc = (i & 1) ? 2 : (i & 3) == 0 ? 0 : 1, k = (i & 1) ? i >> 1 : i >> 2;
    const int rc = 4 * tf_koff(M, gc) + k, rs = 4 * tf_koff(M, gc + 3) + k;
    const int oc = (rc >> 2) * 32 + a_frag_slot(rc & 3, g), os = (rs >> 2) * 32 + a_frag_slot(rs & 3, g);
#pragma unroll
    for (int f = 0; f < 3; ++f) {
      xs[f * fstride + oc] = rot[2 * f];
      xs[(3 + f) * fstride + oc] = w[2 * f];
      if (i != 0) {  // the sine of mode 0 is ignored
        xs[f * fstride + os] = rot[2 * f + 1];
        xs[(3 + f) * fstride + os] = w[2 * f + 1];
      }
    }
  }
  __syncthreads();
  double acc_e[NI][2], acc_o[NI][2];
  tf_synth<M, NI, 0u>(xs, a.syn, acc_e, acc_o);
  __syncthreads();  // every warp has read its last coefficient: xc and ps may overwrite xs
  double v[4][NI];
  tf_fold<M, NI>(acc_e, acc_o, xc, v);
  double gq[4][NO];
#pragma unroll
  for (int r = 0; r < 4; ++r) EKDef<EK_CROSS>::op(v[r], gq[r]);
  tf_prefold<M, NO>(gq, ps, 0);
  __syncthreads();
  OutSet<NO> os;
#pragma unroll
  for (int o = 0; o < NO; ++o) {
    os.p[o] = a.out[o];
    os.ldm[o] = a.out_ldm[o];
  }
  tf_analysis<M, NO>(ps, a.ana, os, p0, a.np, a.out_ps, false);
}

// The advection callers with their operands built in the staging (third fold, M = 64, P2 elements):
// smb_ugradc_gauss_fft_par (subroutine_level_set.F90:434-534) and the temperature and concentration
// versions (subroutine_temperature_with_T.F90:247-350, subroutine_concentration.F90:243-341).  Fields 0-2:
// Gradc = heat grad c, 3-5: W = u, and for the conservative form 6: Div = div u, 7: Cgauss = heat c; the
// program Gradc . W (+ Div Cgauss) is evaluated on the grid and analysed once.  ga.v is the node-major
// velocity (np_nodes, 6, nmod), ga.v2 the node-major scalar (np_nodes, 2, nmod), ga.heat the element's heat
// capacity or null.
template <int M, bool CONS>
__global__ void __launch_bounds__(384, 2) gauss_tf_advect_kernel(const FastArgs a, const GaussArgs ga) {
  static_assert(third_fold(M), "third fold needs the specialised geometry");
  constexpr int NI = CONS ? 8 : 6, NT = TfGeo<M>::NT, KS_tot = TfGeo<M>::KS_tot;
  constexpr size_t fstride = (size_t)KS_tot * 32;
  extern __shared__ double smem[];
  const int64_t p0 = (int64_t)blockIdx.x * 8;
  constexpr size_t prod_d = (size_t)1 * 4 * NT * 2 * 32;
  double *ps = smem, *xc = smem + prod_d, *xs = smem;  // ps and xc overlay xs after the synthesis
  constexpr int NW = 6;  // P2 elements
  __shared__ int s_node[8][NW];
  __shared__ double s_wt[8][NW], s_g1[8][NW], s_g2[8][NW], s_ray[8], s_heat[8];
  for (int t = threadIdx.x; t < NI * (int)fstride; t += blockDim.x) xs[t] = 0.0;  // padding rows, sine of mode 0
  if (threadIdx.x < 8 * NW) {  // the points' nodes, basis values and derivatives (mesh%jj, ww, dw)
    const int g = threadIdx.x / NW, n = threadIdx.x % NW;
    const int64_t p = p0 + g < a.np ? p0 + g : a.np - 1;
    const int me = (int)(p / ga.l_G), l = (int)(p % ga.l_G);
    int node = ga.jj[n + (size_t)NW * me] - 1;
    node = node < 0 ? 0 : node >= ga.np_nodes ? ga.np_nodes - 1 : node;  // no access outside the fields
    s_node[g][n] = node;
    s_wt[g][n] = ga.ww[n + (size_t)NW * l];
    const double *dwl = ga.dw + (size_t)2 * NW * (l + (size_t)ga.l_G * me);
    s_g1[g][n] = dwl[2 * n];
    s_g2[g][n] = dwl[2 * n + 1];
    if (n == 0) s_heat[g] = ga.heat ? ga.heat[me] : 1.0;  // heat_capa_in(m), temperature version
  }
  __syncthreads();
  if (threadIdx.x < 8) {  // radius of the point: sum rr(1, nodes) ww
    double ray = 0.0;
#pragma unroll
    for (int n = 0; n < NW; ++n) ray = fma(ga.rr[2 * (size_t)s_node[threadIdx.x][n]], s_wt[threadIdx.x][n], ray);
    s_ray[threadIdx.x] = ray;
  }
  __syncthreads();
  for (int it = threadIdx.x; it < 8 * M; it += blockDim.x) {
    const int i = it % M, g = it / M;  // mode index, point of the tile: a warp reads 32 modes of a node
    if (p0 + g >= a.np) continue;
    double wv[6] = {0, 0, 0, 0, 0, 0}, d1[6] = {0, 0, 0, 0, 0, 0}, d2[6] = {0, 0, 0, 0, 0, 0};
    double cw[2] = {0, 0}, c1[2] = {0, 0}, c2[2] = {0, 0};
#pragma unroll
    for (int n = 0; n < NW; ++n) {
      const double wt = s_wt[g][n], g1 = s_g1[g][n], g2 = s_g2[g][n];
      const double *vn = ga.v + (size_t)s_node[g][n] * 6 * M + i;
#pragma unroll
      for (int k = 0; k < 6; ++k) {
        const double vs = vn[(size_t)k * M];
        wv[k] = fma(vs, wt, wv[k]);
        d1[k] = fma(vs, g1, d1[k]);
        d2[k] = fma(vs, g2, d2[k]);
      }
      const double *cn = ga.v2 + (size_t)s_node[g][n] * 2 * M + i;
#pragma unroll
      for (int k = 0; k < 2; ++k) {
        const double cs = cn[(size_t)k * M];
        cw[k] = fma(cs, wt, cw[k]);
        c1[k] = fma(cs, g1, c1[k]);
        c2[k] = fma(cs, g2, c2[k]);
      }
    }
    // the cylindrical gradient of the scalar's mode and the divergence of the velocity's mode
    // (subroutine_temperature_with_T.F90:300-331, subroutine_level_set.F90:470-500)
    const double ray = s_ray[g], hc = s_heat[g], mr = (double)ga.list_mode[i] / ray;
    double f[NI][2];
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
    if constexpr (CONS) {
      f[6][0] = d1[0] + wv[0] / ray + mr * wv[3] + d2[4];
      f[6][1] = d1[1] + wv[1] / ray - mr * wv[2] + d2[5];
      f[7][0] = hc * cw[0];
      f[7][1] = hc * cw[1];
    }
    // rows of mode i: cosine group CE0 (i = 0 mod 4), CE2 (i = 2 mod 4) or CO (odd), sine group 3 further
    const int gc = (i & 1) ? 2 : (i & 3) == 0 ? 0 : 1, k = (i & 1) ? i >> 1 : i >> 2;
    const int rc = 4 * tf_koff(M, gc) + k, rs = 4 * tf_koff(M, gc + 3) + k;
    const int oc = (rc >> 2) * 32 + a_frag_slot(rc & 3, g), os = (rs >> 2) * 32 + a_frag_slot(rs & 3, g);
#pragma unroll
    for (int fi = 0; fi < NI; ++fi) {
      xs[fi * fstride + oc] = f[fi][0];
      if (i != 0) xs[fi * fstride + os] = f[fi][1];  // the sine of mode 0 is ignored
    }
  }
  __syncthreads();
  double acc_e[NI][2], acc_o[NI][2];
  tf_synth<M, NI, 0u>(xs, a.syn, acc_e, acc_o);
  __syncthreads();  // every warp has read its last coefficient: xc and ps may overwrite xs
  double v[4][NI];
  tf_fold<M, NI>(acc_e, acc_o, xc, v);
  double gq[4][1];
#pragma unroll
  for (int r = 0; r < 4; ++r) {
    gq[r][0] = v[r][0] * v[r][3] + v[r][1] * v[r][4] + v[r][2] * v[r][5];
    if constexpr (CONS) gq[r][0] = fma(v[r][6], v[r][7], gq[r][0]);
  }
  tf_prefold<M, 1>(gq, ps, 0);
  __syncthreads();
  OutSet<1> os1;
  os1.p[0] = a.out[0];
  os1.ldm[0] = a.out_ldm[0];
  tf_analysis<M, 1>(ps, a.ana, os1, p0, a.np, 1, false);
}

// The MHD bundle (u x w, u x b, j x b, u . gradT) in one launch with the third fold (M = 64): the five
// vector operands are staged and synthesised one at a time (u, w, gradT, b, j), so u and b are
// transformed once instead of three and two times (15 field transforms instead of 24); u's and b's
// quadrant values stay in registers while their partners are synthesised.  Each operand's copies are
// issued during the previous operand's exchanges; the outputs are analysed in three rounds (u x w;
// u x b with u . gradT; j x b) through a four-output product buffer.
struct BundleArgs {
  const double *in[15];  // u 0-2, w 3-5, b 6-8, j 9-11, gradT 12-14
  double *out[10];       // u x w 0-2, u x b 3-5, j x b 6-8, u . gradT 9
  int64_t in_ldm[15], out_ldm[10];
  int64_t np;
  int vec16;
  const double *syn, *ana;
};

template <int M>
__global__ void __launch_bounds__(384, 2) fast_bundle_tf_kernel(const BundleArgs a) {
  static_assert(third_fold(M), "third fold needs the specialised geometry");
  constexpr int NT = TfGeo<M>::NT, KS_tot = TfGeo<M>::KS_tot;
  extern __shared__ double smem[];
  double *xs = smem;                                  // one operand: 3 x KS_tot x 32
  double *xc = xs + (size_t)3 * KS_tot * 32;          // exchanges: 2 x NT x 3 x 64
  double *ps = xc + (size_t)2 * NT * 3 * 64;          // products: 4 slots x 4 x NT x 2 x 32
  const int64_t p0 = (int64_t)blockIdx.x * 8;
  auto fields = [&](int first) {
    FieldSet<3> fs;
#pragma unroll
    for (int f = 0; f < 3; ++f) {
      fs.p[f] = a.in[first + f];
      fs.ldm[f] = a.in_ldm[first + f];
    }
    return fs;
  };
  auto outs3 = [&](int first) {
    OutSet<3> os;
#pragma unroll
    for (int o = 0; o < 3; ++o) {
      os.p[o] = a.out[first + o];
      os.ldm[o] = a.out_ldm[first + o];
    }
    return os;
  };
  // one operand: wait for its copies, synthesise, issue the next operand's copies, fold
  auto operand = [&](int next_first, double (&v)[4][3]) {
    cp_async_wait_0();
    __syncthreads();
    double acc_e[3][2], acc_o[3][2];
    tf_synth<M, 3, 0u>(xs, a.syn, acc_e, acc_o);
    __syncthreads();  // xs is read
    if (next_first >= 0) tf_stage<M, 3>(xs, fields(next_first), p0, a.np, a.vec16 != 0);
    tf_fold<M, 3>(acc_e, acc_o, xc, v);
  };
  double vu[4][3], vb[4][3], vx[4][3];
  tf_stage<M, 3>(xs, fields(0), p0, a.np, a.vec16 != 0);  // u
  operand(3, vu);                                        // u; next w
  operand(12, vx);                                       // w; next gradT
  {
    double gq[4][3];
#pragma unroll
    for (int r = 0; r < 4; ++r) cross3(vu[r], vx[r], gq[r]);
    tf_prefold<M, 3>(gq, ps, 0);
  }
  __syncthreads();
  tf_analysis<M, 3>(ps, a.ana, outs3(0), p0, a.np, 1, false);  // u x w
  operand(6, vx);                                              // gradT; next b
  {
    double gq[4][1];
#pragma unroll
    for (int r = 0; r < 4; ++r) gq[r][0] = vu[r][0] * vx[r][0] + vu[r][1] * vx[r][1] + vu[r][2] * vx[r][2];
    __syncthreads();  // the u x w analysis has read ps
    tf_prefold<M, 1>(gq, ps, 3);
  }
  operand(9, vb);  // b; next j
  {
    double gq[4][3];
#pragma unroll
    for (int r = 0; r < 4; ++r) cross3(vu[r], vb[r], gq[r]);
    tf_prefold<M, 3>(gq, ps, 0);
  }
  __syncthreads();
  {
    OutSet<4> os;
#pragma unroll
    for (int o = 0; o < 3; ++o) {
      os.p[o] = a.out[3 + o];
      os.ldm[o] = a.out_ldm[3 + o];
    }
    os.p[3] = a.out[9];
    os.ldm[3] = a.out_ldm[9];
    tf_analysis<M, 4>(ps, a.ana, os, p0, a.np, 1, false);  // u x b, u . gradT
  }
  operand(-1, vx);  // j
  {
    double gq[4][3];
#pragma unroll
    for (int r = 0; r < 4; ++r) cross3(vx[r], vb[r], gq[r]);
    __syncthreads();  // the previous analysis has read ps
    tf_prefold<M, 3>(gq, ps, 0);
  }
  __syncthreads();
  tf_analysis<M, 3>(ps, a.ana, outs3(6), p0, a.np, 1, false);  // j x b
}

template <int EK, int M, int ADJ>
int launch_ek_m(FastArgs &fa, int batch, cudaStream_t st) {
  constexpr int NI = EKDef<EK>::NI, NO = EKDef<EK>::NO;
  static_assert(ek_nin(EK) == NI && ek_nout(EK) == NO, "elementary program table");
  constexpr bool CS = class_split(EK, M);
  fa.KT = 4 * (fa.KS[0] + fa.KS[1] + fa.KS[2] + fa.KS[3]);
  const size_t smem = fast_smem_bytes(EK, fa.NT, fa.KT, CS);
  if (smem > 200 * 1024) return set_error(SFNL_ERR_UNSUPPORTED, "FAST form: m too large for shared memory");
  const int tiles_per_pass = fa.NT < 8 ? fa.NT : 8;
  const int nw = CS ? 2 * tiles_per_pass : (tiles_per_pass < 2 ? 2 : tiles_per_pass);
  auto kern = fast_kernel<EK, M, ADJ, CS>;
  if constexpr (CS && third_fold(M)) {
    if (fa.allow_tf) {  // the third-fold kernel (same shared memory and warps, its own tables)
      Tables T;
      if (int rc = get_tf_tables(make_geo(fa.m), &T)) return rc;
      fa.syn = T.syn;
      fa.ana = T.ana;
      kern = fast_tf_kernel<EK, M, ADJ>;
    }
  }
  if (smem > 48 * 1024 && cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess)
    return set_error(SFNL_ERR_CUDA, "cudaFuncSetAttribute failed (fast form)");
  const int64_t tiles = (fa.np + 7) / 8;
  if (tiles > 0x7fffffff) return set_error(SFNL_ERR_UNSUPPORTED, "np too large");
  dim3 grid((unsigned)tiles, (unsigned)batch);
  kern<<<grid, nw * 32, smem, st>>>(fa);
  return check_launch("fast form");
}

template <int EK, int ADJ>
int launch_ek_adj(FastArgs &fa, int batch, cudaStream_t st) {
  switch (fa.m) {
    case 16: return launch_ek_m<EK, 16, ADJ>(fa, batch, st);
    case 32: return launch_ek_m<EK, 32, ADJ>(fa, batch, st);
    case 64: return launch_ek_m<EK, 64, ADJ>(fa, batch, st);
    default: return launch_ek_m<EK, 0, ADJ>(fa, batch, st);
  }
}

template <int EK>
int launch_ek(FastArgs &fa, int batch, cudaStream_t st) {
  if constexpr (ek_passes(EK) == 2) {  // the cotangents' fields among the 12 staged ones (pass 0: 0-5, pass 1: 6-11)
    if (fa.adj_in == 0u) return launch_ek_adj<EK, 0>(fa, batch, st);
    if (fa.adj_in == 0xE38u) return launch_ek_adj<EK, 2>(fa, batch, st);  // second operand of both passes
    return set_error(SFNL_ERR_ARG, "FAST form: unsupported cotangent operands");
  } else if constexpr (EK == EK_CROSS) {
    if (fa.adj_in == 0x07u) return launch_ek_adj<EK, 1>(fa, batch, st);
    if (fa.adj_in == 0x38u) return launch_ek_adj<EK, 2>(fa, batch, st);
    if (fa.adj_in != 0u) return set_error(SFNL_ERR_ARG, "FAST form: unsupported cotangent operand");
  } else {
    if (fa.adj_in != 0u) return set_error(SFNL_ERR_ARG, "FAST form: unsupported cotangent operand");
  }
  return launch_ek_adj<EK, 0>(fa, batch, st);
}

}  // namespace

namespace {
// 16-byte copies of whole rows need every row start 16-byte aligned: field bases, the sine offset np,
// the mode stride and the batch stride all multiples of two doubles.
int rows_aligned16(const FastArgs &fa, int ni) {
  if (fa.np & 1) return 0;
  for (int i = 0; i < ni; ++i)
    if ((reinterpret_cast<uintptr_t>(fa.in[i]) & 15) || (fa.in_ldm[i] & 1) || (fa.in_bs[i] & 1)) return 0;
  return 1;
}
}  // namespace

int decompose_program(int op, std::vector<Elem> &seq, int fuse) {
  seq.clear();
  auto add = [&](int ek, std::initializer_list<int> in, std::initializer_list<int> out, unsigned adj, int acc) {
    Elem e{};
    e.ek = ek;
    int i = 0;
    for (int v : in) e.in[i++] = v;
    i = 0;
    for (int v : out) e.out[i++] = v;
    e.adj = adj;
    e.acc = acc;
    seq.push_back(e);
  };
  const unsigned A1 = 0x38u, A0 = 0x07u;  // cotangent as second / first operand
  switch (op) {
    case OP_CROSS: add(EK_CROSS, {0, 1, 2, 3, 4, 5}, {0, 1, 2}, 0, 0); break;
    case OP_DOT: add(EK_DOT, {0, 1, 2, 3, 4, 5}, {0}, 0, 0); break;
    case OP_PROD: add(EK_PROD, {0, 1}, {0}, 0, 0); break;
    case OP_SVECT: add(EK_SVECT, {0, 1, 2, 3}, {0, 1, 2}, 0, 0); break;
    case OP_TENSOR: add(EK_TENSOR, {0, 1, 2, 3, 4, 5}, {0, 1, 2, 3, 4, 5, 6, 7, 8}, 0, 0); break;
    case OP_BUNDLE:
      add(EK_CROSS, {0, 1, 2, 3, 4, 5}, {0, 1, 2}, 0, 0);     // u x w
      add(EK_CROSS, {0, 1, 2, 6, 7, 8}, {3, 4, 5}, 0, 0);     // u x b
      add(EK_CROSS, {9, 10, 11, 6, 7, 8}, {6, 7, 8}, 0, 0);   // j x b
      add(EK_DOT, {0, 1, 2, 12, 13, 14}, {9}, 0, 0);          // u . gradT
      break;
    case OP_ADVECT:  // [g, w, d, c]
      add(EK_DOT, {0, 1, 2, 3, 4, 5}, {0}, 0, 0);            // g . w
      add(EK_PROD, {6, 7}, {0}, 0, 1);                       // + d c
      break;
    case OP_CROSS_JVP:  // [u, w, du, dw]
      if (fuse & kFuseJvp) {
        add(EK_CROSS2, {6, 7, 8, 3, 4, 5, 0, 1, 2, 9, 10, 11}, {0, 1, 2}, 0, 0);  // du x w + u x dw
        break;
      }
      add(EK_CROSS, {6, 7, 8, 3, 4, 5}, {0, 1, 2}, 0, 0);     // du x w
      add(EK_CROSS, {0, 1, 2, 9, 10, 11}, {0, 1, 2}, 0, 1);   // + u x dw
      break;
    case OP_CROSS_VJP:  // [u, w, c]
      add(EK_CROSS, {3, 4, 5, 6, 7, 8}, {0, 1, 2}, A1, 0);    // w x c
      add(EK_CROSS, {6, 7, 8, 0, 1, 2}, {3, 4, 5}, A0, 0);    // c x u
      break;
    case OP_MHD_JVP:  // [u, w, b, du, dw, db]
      if (fuse & kFuseJvp) {
        add(EK_CROSS2, {9, 10, 11, 3, 4, 5, 0, 1, 2, 12, 13, 14}, {0, 1, 2}, 0, 0);  // du x w + u x dw
        add(EK_CROSS2, {9, 10, 11, 6, 7, 8, 0, 1, 2, 15, 16, 17}, {3, 4, 5}, 0, 0);  // du x b + u x db
        break;
      }
      add(EK_CROSS, {9, 10, 11, 3, 4, 5}, {0, 1, 2}, 0, 0);   // du x w
      add(EK_CROSS, {0, 1, 2, 12, 13, 14}, {0, 1, 2}, 0, 1);  // + u x dw
      add(EK_CROSS, {9, 10, 11, 6, 7, 8}, {3, 4, 5}, 0, 0);   // du x b
      add(EK_CROSS, {0, 1, 2, 15, 16, 17}, {3, 4, 5}, 0, 1);  // + u x db
      break;
    case OP_MHD_VJP:  // [u, w, b, c1, c2]
      if (fuse & kFuseVjpSum) {
        add(EK_CROSS2, {3, 4, 5, 9, 10, 11, 6, 7, 8, 12, 13, 14}, {0, 1, 2}, 0xE38u, 0);  // w x c1 + b x c2
      } else {
        add(EK_CROSS, {3, 4, 5, 9, 10, 11}, {0, 1, 2}, A1, 0);  // w x c1
        add(EK_CROSS, {6, 7, 8, 12, 13, 14}, {0, 1, 2}, A1, 1); // + b x c2
      }
      add(EK_CROSS, {9, 10, 11, 0, 1, 2}, {3, 4, 5}, A0, 0);  // c1 x u
      add(EK_CROSS, {12, 13, 14, 0, 1, 2}, {6, 7, 8}, A0, 0); // c2 x u
      break;
    default: return set_error(SFNL_ERR_ARG, "unknown program");
  }
  return SFNL_OK;
}

bool fast_fused_fits(int op, int m) {
  const Geo g = make_geo(m);
  return fast_smem_bytes(op == OP_TENSOR ? EK_TENSOR : EK_CROSS, g.NT, 4 * g.KS_tot, true) <= 200 * 1024;
}

int fast_grid_length(int m) { return make_geo(m).N; }

bool gauss_cross_fused_supported(int m, int n_w) { return third_fold(64) && m == 64 && n_w == 6; }

namespace {
template <int EK, int GK, int M>
int launch_gauss_general_m(FastArgs &fa, int64_t ng, cudaStream_t st) {
  constexpr bool CS = class_split(EK, M);
  fa.KT = 4 * (fa.KS[0] + fa.KS[1] + fa.KS[2] + fa.KS[3]);
  const size_t smem = fast_smem_bytes(EK, fa.NT, fa.KT, CS);
  if (smem > 200 * 1024) return set_error(SFNL_ERR_UNSUPPORTED, "fused Gauss-point product: m too large");
  const int tiles_per_pass = fa.NT < 8 ? fa.NT : 8;
  const int nw = CS ? 2 * tiles_per_pass : (tiles_per_pass < 2 ? 2 : tiles_per_pass);
  auto kern = fast_kernel<EK, M, 0, CS, GK>;
  if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess)
    return set_error(SFNL_ERR_CUDA, "cudaFuncSetAttribute failed (fused Gauss-point product)");
  const int64_t tiles = (ng + 7) / 8;
  if (tiles > 0x7fffffff) return set_error(SFNL_ERR_UNSUPPORTED, "np too large");
  kern<<<(unsigned)tiles, nw * 32, smem, st>>>(fa);
  return check_launch("fused Gauss-point product");
}
// the geometries the plain products specialise (m = 16, 32, 64), else run-time geometry
template <int EK, int GK>
int launch_gauss_general(FastArgs &fa, int64_t ng, cudaStream_t st) {
  switch (fa.m) {
    case 16: return launch_gauss_general_m<EK, GK, 16>(fa, ng, st);
    case 32: return launch_gauss_general_m<EK, GK, 32>(fa, ng, st);
    case 64: return launch_gauss_general_m<EK, GK, 64>(fa, ng, st);
    default: return launch_gauss_general_m<EK, GK, 0>(fa, ng, st);
  }
}
constexpr int gauss_ek(int kind, bool conservative) {
  return kind == GK_ADVECT ? (conservative ? EK_ADVECT : EK_DOT) : EK_CROSS;
}
}  // namespace

bool gauss_general_fused_supported(int kind, bool conservative, int m) {
  if (m < 1 || m > 96 || kind < GK_NS || kind > GK_ADVECT) return false;
  const int ek = gauss_ek(kind, conservative);
  const Geo g = make_geo(m);
  return fast_smem_bytes(ek, g.NT, 4 * g.KS_tot, class_split(ek, 0)) <= 200 * 1024;
}

int launch_gauss_general_fused(const GaussArgs &ga, int kind, bool conservative, double *out, int64_t ng, int m,
                               cudaStream_t st) {
  if (!gauss_general_fused_supported(kind, conservative, m))
    return set_error(SFNL_ERR_UNSUPPORTED, "fused Gauss-point product: not built for this size");
  if (ng == 0) return SFNL_OK;
  const Geo g = make_geo(m);
  Tables T;
  if (int rc = get_tables(g, &T)) return rc;
  FastArgs fa;
  std::memset(&fa, 0, sizeof(fa));
  const int nout = kind == GK_ADVECT ? 1 : 3, nsl = kind == GK_ADVECT ? 2 : 6;
  for (int o = 0; o < nout; ++o) {
    fa.out[o] = out + (int64_t)2 * o * ng;  // V_out(l_G*me, nsl, m): component o in slots 2o, 2o+1
    fa.out_ldm[o] = (int64_t)nsl * ng;
  }
  fa.out_ps = 1;
  fa.np = ng;
  fa.m = g.m;
  fa.N = g.N;
  fa.NT = g.NT;
  for (int c = 0; c < 4; ++c) {
    fa.ks_off[c] = g.ks_off[c];
    fa.KS[c] = g.KS[c];
    fa.nu_off[c] = g.nu_off[c];
    fa.NU[c] = g.NU[c];
    fa.ke[c] = g.ke[c];
  }
  fa.NU_tot = g.NU_tot;
  fa.syn = T.syn;
  fa.ana = T.ana;  // variant 0: with the analysis weights
  fa.ga = ga;
  switch (kind) {
    case GK_NS: return launch_gauss_general<EK_CROSS, GK_NS>(fa, ng, st);
    case GK_LORENTZ: return launch_gauss_general<EK_CROSS, GK_LORENTZ>(fa, ng, st);
    default:
      return conservative ? launch_gauss_general<EK_ADVECT, GK_ADVECT>(fa, ng, st)
                          : launch_gauss_general<EK_DOT, GK_ADVECT>(fa, ng, st);
  }
}

int launch_gauss_advect_fused(const GaussArgs &ga, bool conservative, double *out, int64_t ng, int m,
                              cudaStream_t st) {
  constexpr int M = 64;
  if (m != M) return set_error(SFNL_ERR_UNSUPPORTED, "fused Gauss-point advection: m = 64 only");
  if (ng == 0) return SFNL_OK;
  const Geo g = make_geo(M);
  Tables T;
  if (int rc = get_tf_tables(g, &T)) return rc;
  FastArgs fa;
  std::memset(&fa, 0, sizeof(fa));
  fa.out[0] = out;  // c_out(l_G*me, 2, m)
  fa.out_ldm[0] = 2 * ng;
  fa.out_ps = 1;
  fa.np = ng;
  fa.m = M;
  fa.N = g.N;
  fa.NT = g.NT;
  fa.syn = T.syn;
  fa.ana = T.ana;  // variant 0: with the analysis weights
  const int ni = conservative ? 8 : 6;
  const size_t xs = sizeof(double) * (size_t)ni * g.KS_tot * 32;
  const size_t ovl = sizeof(double) * ((size_t)4 * g.NT * 2 * 32 + (size_t)2 * g.NT * ni * 64);
  const size_t smem = xs > ovl ? xs : ovl;
  auto kern = conservative ? gauss_tf_advect_kernel<M, true> : gauss_tf_advect_kernel<M, false>;
  // opt in whatever the size: the kernel's static shared memory counts against the 48 KB default too
  if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess)
    return set_error(SFNL_ERR_CUDA, "cudaFuncSetAttribute failed (fused Gauss-point advection)");
  const int64_t tiles = (ng + 7) / 8;
  kern<<<(unsigned)tiles, 384, smem, st>>>(fa, ga);
  return check_launch("fused Gauss-point advection");
}

int launch_gauss_cross_fused(const GaussArgs &ga, int kind, double *out, int64_t ng, int m, cudaStream_t st) {
  constexpr int M = 64;
  if (m != M) return set_error(SFNL_ERR_UNSUPPORTED, "fused Gauss-point cross product: m = 64 only");
  if (ng == 0) return SFNL_OK;
  const Geo g = make_geo(M);
  Tables T;
  if (int rc = get_tf_tables(g, &T)) return rc;
  FastArgs fa;
  std::memset(&fa, 0, sizeof(fa));
  for (int o = 0; o < 3; ++o) {
    fa.out[o] = out + (int64_t)2 * o * ng;  // V_out(l_G*me, 6, m): component o in slots 2o, 2o+1
    fa.out_ldm[o] = 6 * ng;
  }
  fa.out_ps = 1;
  fa.np = ng;
  fa.m = M;
  fa.N = g.N;
  fa.NT = g.NT;
  fa.syn = T.syn;
  fa.ana = T.ana;  // variant 0: with the analysis weights
  const size_t smem = fast_smem_bytes(EK_CROSS, g.NT, 4 * g.KS_tot, true);
  auto kern = kind == GK_NS ? gauss_tf_cross_kernel<M, GK_NS> : gauss_tf_cross_kernel<M, GK_LORENTZ>;
  if (kind != GK_NS && kind != GK_LORENTZ) return set_error(SFNL_ERR_ARG, "fused Gauss-point cross product: curl callers only");
  if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess)  // static smem too
    return set_error(SFNL_ERR_CUDA, "cudaFuncSetAttribute failed (fused Gauss-point cross product)");
  const int64_t tiles = (ng + 7) / 8;
  kern<<<(unsigned)tiles, 384, smem, st>>>(fa, ga);
  return check_launch("fused Gauss-point cross product");
}

bool fast_supported(int op, int m, int N) {
  if (m < 1 || m > 512 || !op_bilinear(op)) return false;
  const Geo g = make_geo(m);
  // fused kernels when the largest elementary program fits; else the two-kernel form (up to 48 angle tiles
  // and 128 output tiles: m <= 512)
  return g.N == N;
}

namespace {
// The MHD bundle in one third-fold launch (m = 64, one batch entry, plain layouts).
int launch_bundle_tf(const ProgArgs &a, cudaStream_t st) {
  constexpr int M = 64;
  BundleArgs ba;
  std::memset(&ba, 0, sizeof(ba));
  int v16 = (a.np & 1) ? 0 : 1;
  for (int f = 0; f < 15; ++f) {
    ba.in[f] = a.in[f];
    ba.in_ldm[f] = a.in_ldm[f];
    if ((reinterpret_cast<uintptr_t>(a.in[f]) & 15) || (a.in_ldm[f] & 1)) v16 = 0;
  }
  for (int o = 0; o < 10; ++o) {
    ba.out[o] = a.out[o];
    ba.out_ldm[o] = a.out_ldm[o];
  }
  ba.np = a.np;
  ba.vec16 = v16;
  Tables T;
  if (int rc = get_tf_tables(make_geo(M), &T)) return rc;
  ba.syn = T.syn;
  ba.ana = T.ana;  // variant 0: with the analysis weights
  constexpr int NT = TfGeo<M>::NT, KS_tot = TfGeo<M>::KS_tot;
  const size_t smem = sizeof(double) * ((size_t)3 * KS_tot * 32 + (size_t)2 * NT * 3 * 64 + (size_t)4 * 4 * NT * 2 * 32);
  auto kern = fast_bundle_tf_kernel<M>;
  if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess)
    return set_error(SFNL_ERR_CUDA, "cudaFuncSetAttribute failed (fast bundle)");
  const int64_t tiles = (a.np + 7) / 8;
  if (tiles > 0x7fffffff) return set_error(SFNL_ERR_UNSUPPORTED, "np too large");
  kern<<<(unsigned)tiles, 2 * NT * 32, smem, st>>>(ba);
  return check_launch("fast form (bundle)");
}
}  // namespace

int launch_fast(const ProgArgs &a, cudaStream_t st) {
  if (a.np == 0) return SFNL_OK;
  const Geo g = make_geo(a.m);
  if (g.N != a.N) return set_error(SFNL_ERR_ARG, "FAST form: unexpected grid length");
  if (a.op == OP_BUNDLE && a.m == 64 && a.batch == 1 && a.out_ps == 1)
    return bundle_kernel() == SFNL_BUNDLE_THIRD_FOLD ? launch_bundle_tf(a, st) : launch_bundle_r3(a, st);
  Tables T;
  int rc = get_tables(g, &T);
  if (rc) return rc;
  if (!fast_fused_fits(a.op, a.m)) return launch_fast_large(a, g, T, st);
  std::vector<Elem> seq;
  // the linearised cross products as one two-pass program each (the output written once, one analysis):
  // 1.7x faster than two launches at m = 32 (700k points, one tangent: 3.26 -> 1.92 ms) and 1.25x at
  // m = 64, where the two launches ran on the third-fold kernel (200k points, 4 tangents: 8.40 -> 6.70 ms);
  // where their products cannot overlay their coefficients (more than 8 angle tiles, m > 85) the two
  // launches stay.  The MHD VJP's w x c1 + b x c2 likewise (m = 32, 200k points, 4 tangents: 6.51 -> 5.09 ms)
  // but at m = 64, where its two launches on the third-fold kernel are a little faster (7.74 against
  // 7.98 ms); the other transposed products (two cross products into different outputs) gained nothing from
  // one launch of two passes (m = 32: 2.41 -> 2.69 ms).
  const bool fuse_ok = fast_overlay(EK_CROSS2, g.NT, 4 * g.KS_tot);
  rc = decompose_program(a.op, seq, fuse_ok ? kFuseJvp | (a.m != 64 ? kFuseVjpSum : 0) : 0);
  if (rc) return rc;
  const bool adj_out = op_adjoint_out(a.op);
  for (const Elem &e : seq) {
    FastArgs fa;
    std::memset(&fa, 0, sizeof(fa));
    const int ni = ek_nin(e.ek), no = ek_nout(e.ek);
    fa.out_ps = a.out_ps;
    for (int i = 0; i < ni; ++i) {
      fa.in[i] = a.in[e.in[i]];
      fa.in_ldm[i] = a.in_ldm[e.in[i]];
      fa.in_bs[i] = a.in_bs[e.in[i]];
    }
    for (int o = 0; o < no; ++o) {
      fa.out[o] = a.out[e.out[o]];
      fa.out_ldm[o] = a.out_ldm[e.out[o]];
      fa.out_bs[o] = a.out_bs[e.out[o]];
    }
    fa.np = a.np;
    fa.m = g.m;
    fa.N = g.N;
    fa.NT = g.NT;
    for (int c = 0; c < 4; ++c) {
      fa.ks_off[c] = g.ks_off[c];
      fa.KS[c] = g.KS[c];
      fa.nu_off[c] = g.nu_off[c];
      fa.NU[c] = g.NU[c];
      fa.ke[c] = g.ke[c];
    }
    fa.NU_tot = g.NU_tot;
    fa.adj_in = e.adj;
    fa.adj_out = adj_out ? 1 : 0;
    fa.accumulate = e.acc;
    fa.vec16 = rows_aligned16(fa, ni);
    fa.allow_tf = 1;
    fa.syn = T.syn;
    fa.ana = T.ana;
    int r = e.ek == EK_CROSS  ? launch_ek<EK_CROSS>(fa, a.batch, st)
          : e.ek == EK_CROSS2 ? launch_ek<EK_CROSS2>(fa, a.batch, st)
          : e.ek == EK_DOT    ? launch_ek<EK_DOT>(fa, a.batch, st)
          : e.ek == EK_PROD   ? launch_ek<EK_PROD>(fa, a.batch, st)
          : e.ek == EK_SVECT  ? launch_ek<EK_SVECT>(fa, a.batch, st)
                              : launch_ek<EK_TENSOR>(fa, a.batch, st);
    if (r) return r;
  }
  return SFNL_OK;
}

// ---------------------------------------------------------------------------
// sfnl_cross_f64_noalloc: the FAST cross product for callers that cannot
// allocate device memory.  Its DFT tables live in the static device array
// below (one copy per device that loads the library, kept until exit) and are
// written on the device by build_tables_kernel, so the entry point calls no
// cudaMalloc, cudaFree or other allocating routine.
// ---------------------------------------------------------------------------
constexpr int kNoAllocMaxM = 64;
constexpr int kNoAllocDoubles = 18432;  // synthesis + both analysis variants at m = 64 (144 KiB)
static __device__ __align__(256) double g_noalloc_tab[kNoAllocDoubles];

namespace {
std::mutex g_na_mu;
double *g_na_ptr[64];  // device address of g_noalloc_tab, per device (set up on first use)
int g_na_m[64];        // m_max whose tables the array holds, per device (0: none)

// Writes the folded-transform tables of make_geo(m) (same entries as get_tables,
// angles reduced exactly as n(2j+1) mod 2N before sincospi).
__global__ void build_tables_kernel(double *syn, double *ana, FastArgs g) {
  int ks_tot = 0;
  for (int c = 0; c < 4; ++c) ks_tot += g.KS[c];
  const int64_t n_syn = (int64_t)ks_tot * g.NT * 32, n_ana = (int64_t)2 * g.NU_tot * g.NT * 64;
  for (int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; idx < n_syn + n_ana;
       idx += (int64_t)gridDim.x * blockDim.x) {
    int c = 0, k, j, n, var = 0;
    bool live;
    if (idx < n_syn) {
      const int l = (int)(idx % 32), r = (int)(idx / 32), t = r % g.NT, ks = r / g.NT;
      while (c < 3 && ks >= g.ks_off[c + 1]) ++c;
      k = 4 * (ks - g.ks_off[c]) + (l & 3);
      j = 8 * t + (l >> 2);
      live = k < g.ke[c];
    } else {
      int64_t r = idx - n_syn;
      const int l = (int)(r % 32);
      r /= 32;
      const int e = (int)(r % 2);
      r /= 2;
      const int t = (int)(r % g.NT);
      r /= g.NT;
      const int cu = (int)(r % g.NU_tot);
      var = (int)(r / g.NU_tot);
      while (c < 3 && cu >= g.nu_off[c + 1]) ++c;
      j = 8 * t + 2 * (l & 3) + e;
      k = 8 * (cu - g.nu_off[c]) + (l >> 2);
      live = k < g.ke[c];
    }
    double v = 0.0;
    if (live) {
      n = 2 * k + (c & 1);
      const long long rr = ((long long)n * (2 * j + 1)) % (2LL * g.N);
      double sv, cv;
      sincospi((double)rr / (double)g.N, &sv, &cv);
      v = c < 2 ? cv : sv;
      if (idx >= n_syn && var == 0) v *= (n == 0 ? 1.0 : 2.0) / (double)g.N;
    }
    if (idx < n_syn)
      syn[idx] = v;
    else
      ana[idx - n_syn] = v;
  }
}
}  // namespace

void fast_release_tables() {
  r3_release_tables();
  std::lock_guard<std::mutex> lk(g_tab_mu);
  int prev = 0;
  cudaGetDevice(&prev);
  for (auto &kv : g_tabs) {
    cudaSetDevice(kv.first.first);
    cudaFree(kv.second.syn);
    cudaFree(kv.second.ana);
  }
  g_tabs.clear();
  {
    std::lock_guard<std::mutex> lk2(g_tftab_mu);
    for (auto &kv : g_tftabs) {
      cudaSetDevice(kv.first.first);
      cudaFree(kv.second.syn);
      cudaFree(kv.second.ana);
    }
    g_tftabs.clear();
  }
  cudaSetDevice(prev);
  {
    // The no-allocation entry's cached array addresses and table state belong to the current
    // contexts; after a device reset they would be stale, so the next call sets them up again.
    std::lock_guard<std::mutex> lk3(g_na_mu);
    for (int d = 0; d < 64; ++d) {
      g_na_ptr[d] = nullptr;
      g_na_m[d] = 0;
    }
  }
}

}  // namespace sfnl

extern "C" int sfnl_cross_f64_noalloc(const double *v1, const double *v2, double *out, int64_t np, int m_max,
                                      int m_max_pad, sfnl_stream_t stream) {
  using namespace sfnl;
  if (np < 0 || m_max < 1) return set_error(SFNL_ERR_ARG, "sfnl_cross_f64_noalloc: np < 0 or m_max < 1");
  if (m_max_pad < m_max) return set_error(SFNL_ERR_ALIAS, "sfnl_cross_f64_noalloc: m_max_pad < m_max");
  if (2 * m_max_pad - 1 < 3 * m_max - 2)
    return set_error(SFNL_ERR_ALIAS, "sfnl_cross_f64_noalloc: needs a dealiasing pad (2*m_max_pad-1 >= 3*m_max-2)");
  if (m_max > kNoAllocMaxM)
    return set_error(SFNL_ERR_UNSUPPORTED, "sfnl_cross_f64_noalloc: m_max > 64 does not fit its static table");
  if (np == 0) return SFNL_OK;
  if (!v1 || !v2 || !out) return set_error(SFNL_ERR_ARG, "sfnl_cross_f64_noalloc: null array");
  const Geo g = make_geo(m_max);
  const int n_syn = g.KS_tot * g.NT * 32, n_ana = 2 * g.NU_tot * g.NT * 64;
  if (n_syn + n_ana > kNoAllocDoubles) return set_error(SFNL_ERR_UNSUPPORTED, "sfnl_cross_f64_noalloc: table overflow");
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  FastArgs fa;
  std::memset(&fa, 0, sizeof(fa));
  fa.out_ps = 1;
  for (int k = 0; k < 3; ++k) {
    fa.in[k] = v1 + (int64_t)2 * k * np;
    fa.in[3 + k] = v2 + (int64_t)2 * k * np;
    fa.out[k] = out + (int64_t)2 * k * np;
  }
  for (int f = 0; f < 6; ++f) fa.in_ldm[f] = 6 * np;
  for (int o = 0; o < 3; ++o) fa.out_ldm[o] = 6 * np;
  fa.np = np;
  fa.m = g.m;
  fa.N = g.N;
  fa.NT = g.NT;
  for (int c = 0; c < 4; ++c) {
    fa.ks_off[c] = g.ks_off[c];
    fa.KS[c] = g.KS[c];
    fa.nu_off[c] = g.nu_off[c];
    fa.NU[c] = g.NU[c];
    fa.ke[c] = g.ke[c];
  }
  fa.NU_tot = g.NU_tot;
  fa.vec16 = rows_aligned16(fa, 6);
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64)
    return set_error(SFNL_ERR_CUDA, "sfnl_cross_f64_noalloc: no current device");
  {
    std::lock_guard<std::mutex> lk(g_na_mu);
    if (!g_na_ptr[dev]) {
      void *p = nullptr;
      const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_tab);
      if (e != cudaSuccess || !p) return set_error(SFNL_ERR_CUDA, "sfnl_cross_f64_noalloc: cudaGetSymbolAddress failed");
      g_na_ptr[dev] = static_cast<double *>(p);
      g_na_m[dev] = 0;
    }
    fa.syn = g_na_ptr[dev];
    fa.ana = g_na_ptr[dev] + n_syn;
    if (g_na_m[dev] != m_max) {
      build_tables_kernel<<<64, 256, 0, st>>>(g_na_ptr[dev], g_na_ptr[dev] + n_syn, fa);
      const int rc = check_launch("sfnl_cross_f64_noalloc table set-up");
      if (rc) return rc;
      g_na_m[dev] = m_max;
    }
  }
  return launch_ek<EK_CROSS>(fa, 1, st);
}
