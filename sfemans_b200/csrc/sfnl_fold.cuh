// sfnl_fold.cuh -- geometry, DFT tables and device helpers shared by the FAST
// form's kernels (sfnl_fast.cu: one fused kernel per 8-point tile; sfnl_large.cu:
// synthesis and program+analysis as two kernels for large m).
#pragma once
#include <cuda_runtime.h>

#include <cstdint>

#include "sfnl_ops.cuh"

namespace sfnl {

// ---------------------------------------------------------------------------
// geometry of the folded transforms
// ---------------------------------------------------------------------------
struct Geo {
  int m, Q, N;   // modes, quarter angles, grid length
  int NT;        // quarter-angle tiles of 8
  int ke[4];     // modes per class (0 cos-even, 1 cos-odd, 2 sin-even, 3 sin-odd)
  int KS[4];     // synthesis k-steps per class (modes padded to 4)
  int NU[4];     // analysis output tiles per class (modes padded to 8)
  int ks_off[4]; // prefix offsets
  int nu_off[4];
  int KS_tot, NU_tot;
};

inline Geo make_geo(int m) {
  Geo g;
  g.m = m;
  int qmin = (3 * m - 2 + 3) / 4;
  if (qmin < 1) qmin = 1;
  // Q a multiple of 8 (angle tiles of 8); beyond m = 96 a multiple of 16, so that the tiles pair with their
  // mirrors and the third fold applies (a few more angles, a quarter fewer DMMAs)
  const int qa = m > 96 ? 16 : 8;
  g.Q = ((qmin + qa - 1) / qa) * qa;
  g.N = 4 * g.Q;
  g.NT = g.Q / 8;
  const int ev = (m + 1) / 2, od = m / 2;
  const int cnt[4] = {ev, od, ev, od};
  g.KS_tot = g.NU_tot = 0;
  for (int c = 0; c < 4; ++c) {
    g.ke[c] = cnt[c];
    g.KS[c] = (cnt[c] + 3) / 4;
    g.NU[c] = (cnt[c] + 7) / 8;
    g.ks_off[c] = g.KS_tot;
    g.nu_off[c] = g.NU_tot;
    g.KS_tot += g.KS[c];
    g.NU_tot += g.NU[c];
  }
  return g;
}

__host__ __device__ inline int class_mode(int c, int k) { return 2 * k + (c & 1); }

// Device tables for one m: synthesis B fragments and two analysis variants.
struct Tables {
  double *syn = nullptr;   // [KS_tot][NT][32]
  double *ana = nullptr;   // [2 variants][NU_tot][NT][2][32]
};
// Cached per (device, m); built on first use (sfnl_fast.cu).
int get_tables(const Geo &g, Tables *out);

__device__ __forceinline__ void dmma(double (&d)[2], double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
               : "+d"(d[0]), "+d"(d[1])
               : "d"(a), "d"(b));
}

__device__ __forceinline__ void cp_async8(void *smem_dst, const void *gsrc) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"((uint32_t)__cvta_generic_to_shared(smem_dst)),
               "l"(gsrc)
               : "memory");
}
__device__ __forceinline__ void cp_async16(void *smem_dst, const void *gsrc) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"((uint32_t)__cvta_generic_to_shared(smem_dst)),
               "l"(gsrc)
               : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() {
  asm volatile("cp.async.commit_group;\n\tcp.async.wait_group 0;" ::: "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_0() { asm volatile("cp.async.wait_group 0;" ::: "memory"); }

// ---------------------------------------------------------------------------
// third fold: the mirror symmetry theta -> pi/2 - theta of the quadrant grid
// ---------------------------------------------------------------------------
// On theta_j = pi(2j+1)/(4Q) the quadrant is its own mirror: theta_{Q-1-j} = pi/2 - theta_j.  For even
// n, cos(n(pi/2 - x)) = (-1)^(n/2) cos(nx) and sin(n(pi/2 - x)) = -(-1)^(n/2) sin(nx).  So an even class
// split into its n = 0 mod 4 and n = 2 mod 4 parts (E0, E2) gives both mirror angles from one of them:
// CE(x) = E0 + E2, CE(pi/2 - x) = E0 - E2 and SE(x) = S0 + S2, SE(pi/2 - x) = S2 - S0, each part having
// half the modes; and the analysis of an even class contracts P(x) +- P(pi/2 - x) over half the quadrant
// for each part.  The odd classes gain nothing (their mirror is the other trigonometric function).
// With NT even, angle tile t and its mirror NT-1-t form a pair: local angle a of one is local angle 7-a
// of the other, i.e. lane (g, 3-q) (lane ^ 3) and the other k-step parity e.  A quarter of the DMMAs of
// both transforms goes.
//
// Row and output groups: 0 CE0, 1 CE2, 2 CO, 3 SE0, 4 SE2, 5 SO (cosine coefficients for 0-2, sine 3-5).
__host__ __device__ constexpr int tf_ke(int m, int gr) {
  return (gr % 3 == 0) ? (m + 3) / 4 : (gr % 3 == 1) ? (m + 1) / 4 : m / 2;
}
__host__ __device__ constexpr int tf_mode(int gr, int k) { return gr % 3 == 0 ? 4 * k : gr % 3 == 1 ? 4 * k + 2 : 2 * k + 1; }
__host__ __device__ constexpr int tf_KS(int m, int gr) { return (tf_ke(m, gr) + 3) / 4; }
__host__ __device__ constexpr int tf_koff(int m, int gr) { return gr == 0 ? 0 : tf_koff(m, gr - 1) + tf_KS(m, gr - 1); }
__host__ __device__ constexpr int tf_NU(int m, int gr) { return (tf_ke(m, gr) + 7) / 8; }
__host__ __device__ constexpr int tf_nuoff(int m, int gr) { return gr == 0 ? 0 : tf_nuoff(m, gr - 1) + tf_NU(m, gr - 1); }
// quadrant angle tiles and analysis k-steps of an output group (half the quadrant for the even groups)
__host__ __device__ constexpr int tf_NT(int m) {  // make_geo(m).NT
  return m > 96 ? 2 * (((3 * m - 2 + 3) / 4 + 15) / 16) : ((3 * m - 2 + 3) / 4 + 7) / 8;
}
__host__ __device__ constexpr int tf_TE(int m, int gr) { return gr % 3 == 2 ? 2 * tf_NT(m) : tf_NT(m); }
// first analysis k-step (units of 32 doubles) of group gr in the analysis table
__host__ __device__ constexpr int tf_aoff(int m, int gr) {
  return gr == 0 ? 0 : tf_aoff(m, gr - 1) + tf_NU(m, gr - 1) * tf_TE(m, gr - 1);
}
// the third fold needs an even number of angle tiles; it is built for the specialised m = 64 kernels
// Tables of the third fold for m (a Geo with make_geo(m).N; sfnl_fast.cu): synthesis B fragments
// [KS_tot][NT][32] (lane (g, q): mode tf_mode(gr, 4s + q), angle 8t + g) and analysis B fragments
// [2 variants][tf_aoff(m, 6)][32] (lane (g, q): mode tf_mode(gr, 8u + g), angle 8t + 2q + e; variant 0
// with the analysis weights).  Cached per (device, m).
int get_tf_tables(const Geo &g, Tables *out);

// Barriers of the exchanges: the whole CTA, or one of three groups of 4 warps on its own named barrier.
struct CtaSync {
  __device__ __forceinline__ void operator()() const { __syncthreads(); }
};
struct GroupSync {  // groups 0, 1, 2 of 4 warps on barriers 1, 2, 3 (immediate ids: the kernel reserves 4)
  int group;
  __device__ __forceinline__ void operator()() const {
    if (group == 0)
      asm volatile("bar.sync 1, 128;" ::: "memory");
    else if (group == 1)
      asm volatile("bar.sync 2, 128;" ::: "memory");
    else
      asm volatile("bar.sync 3, 128;" ::: "memory");
  }
};

// Both exchanges of the third fold inside a group of 2*NT warps, warp (tau, half) holding the even part and
// odd class of half `half` (0 cosine, 1 sine) on angle tile tau (tf_synth).  X1 assembles the even class on
// the warp's own tile from the two parts (a first-half tile adds its partner's part at the same lane; a
// second-half tile takes both parts at the mirror lane (lane ^ 3) and parity 1 - e: CE = E0 - E2,
// SE = S2 - S0); X2 swaps half of the folded sums (A = CE+CO, B = CE-CO against C = SE+SO, D = SO-SE) with
// the other half, so that half e ends with the four quadrant values v[r][f] of its angles of parity e.
// xc (the group's own) holds 2 * NT * NG * 64 doubles; call after a barrier of the group that ends the
// reads of whatever xc overlays.  Returns after the X2 reads.
template <int NT, int NG, typename Sync>
__device__ __forceinline__ void fold_exchange(const double (&acc_e)[NG][2], const double (&acc_o)[NG][2], double *xc,
                                              int tau, int half, Sync sync, double (&v)[4][NG]) {
  constexpr int NH = NT / 2;
  const int lane = threadIdx.x & 31;
  const bool first = tau < NH;
  double acc[NG][2][2];  // [f][even, odd class][e]
  {
    double *x1 = xc + (size_t)((tau * 2 + half) * NG) * 64 + lane;
#pragma unroll
    for (int f = 0; f < NG; ++f) {
      x1[(f * 2 + 0) * 32] = acc_e[f][0];
      x1[(f * 2 + 1) * 32] = acc_e[f][1];
    }
    sync();
    const double *own = xc + (size_t)((tau * 2 + half) * NG) * 64;
    const double *mate = xc + (size_t)(((NT - 1 - tau) * 2 + half) * NG) * 64;
#pragma unroll
    for (int f = 0; f < NG; ++f)
#pragma unroll
      for (int e = 0; e < 2; ++e) {
        double ev;
        if (first) {
          ev = acc_e[f][e] + mate[(f * 2 + e) * 32 + lane];
        } else {
          const double p0m = mate[(f * 2 + 1 - e) * 32 + (lane ^ 3)];  // E0 / S0 at the mirror angle
          const double p2m = own[(f * 2 + 1 - e) * 32 + (lane ^ 3)];   // E2 / S2 at the mirror angle
          ev = half ? p2m - p0m : p0m - p2m;
        }
        acc[f][0][e] = ev;
        acc[f][1][e] = acc_o[f][e];
      }
    sync();  // X1 is read: X2 reuses xc
  }
  auto pair_sums = [&](int f, int e, double &X, double &Y) {
    const double lo = e ? acc[f][0][1] : acc[f][0][0], hi = e ? acc[f][1][1] : acc[f][1][0];
    X = lo + hi;
    Y = half ? hi - lo : lo - hi;
  };
  double *xw = xc + (size_t)tau * 2 * NG * 64 + lane;  // [writer half][f][X, Y][32]
#pragma unroll
  for (int f = 0; f < NG; ++f) {
    double X, Y;
    pair_sums(f, 1 - half, X, Y);
    xw[((half * NG + f) * 2 + 0) * 32] = X;
    xw[((half * NG + f) * 2 + 1) * 32] = Y;
  }
  sync();
  const int e = half;
#pragma unroll
  for (int f = 0; f < NG; ++f) {
    double X, Y;
    pair_sums(f, e, X, Y);
    const double Xp = xw[(((1 - half) * NG + f) * 2 + 0) * 32], Yp = xw[(((1 - half) * NG + f) * 2 + 1) * 32];
    const double A = half ? Xp : X, B = half ? Yp : Y, C = half ? X : Xp, D = half ? Y : Yp;
    v[0][f] = A + C;  // theta
    v[1][f] = B + D;  // pi - theta
    v[2][f] = B - D;  // pi + theta
    v[3][f] = A - C;  // 2 pi - theta
  }
}

// Analysis pre-fold of NO program outputs gq[quadrant][o] at angle tile t, parity e of the lane into ps
// slots slot0 .. slot0+NO-1 ([slot][class PE, PO, QE, QO][NT][2][32]).
template <int NT, int NO>
__device__ __forceinline__ void prefold_store(const double (&gq)[4][NO], double *ps, int slot0, int t, int e) {
  const int lane = threadIdx.x & 31;
#pragma unroll
  for (int o = 0; o < NO; ++o) {
    const double s14 = gq[0][o] + gq[3][o], d14 = gq[0][o] - gq[3][o];
    const double s23 = gq[1][o] + gq[2][o], d32 = gq[2][o] - gq[1][o];
    double *dst = ps + ((size_t)(((slot0 + o) * 4) * NT + t) * 2 + e) * 32 + lane;
    const size_t cstride = (size_t)NT * 2 * 32;
    dst[0] = s14 + s23;            // PE
    dst[cstride] = s14 - s23;      // PO
    dst[2 * cstride] = d14 + d32;  // QE
    dst[3 * cstride] = d14 - d32;  // QO
  }
}

// Slot of (k-value kq, point p) in a 32-double A-fragment block [4 k][8 points].  A lane (g, q) of
// m8n8k4 reads (q, g); a 64-bit shared load is served per half-warp, and with the plain order q*8 + g
// the lanes q and q + 2 of a half-warp hit the same banks (two wavefronts per half-warp).  Flipping
// bit 2 of the point for q >= 2 spreads a half-warp over all 32 banks and keeps point pairs (2h, 2h+1)
// adjacent, so 16-byte stores of two points stay possible.
__host__ __device__ __forceinline__ int a_frag_slot(int kq, int p) { return kq * 8 + (p ^ ((kq & 2) << 1)); }

// Element c of a 4-array without dynamic indexing (keeps the arrays in registers).
__device__ __forceinline__ int sel4(const int (&v)[4], int c) { return c == 0 ? v[0] : c == 1 ? v[1] : c == 2 ? v[2] : v[3]; }

// The fused kernels hold an 8-point tile's coefficients and folded products in shared memory; beyond
// that (m ~ 100 for six fields) the two-kernel form runs (sfnl_large.cu).
bool fast_fused_fits(int op, int m);
int launch_fast_large(const ProgArgs &a, const Geo &g, const Tables &T, cudaStream_t st);

}  // namespace sfnl
