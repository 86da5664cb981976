// sfnl_large.cu -- the FAST form's folded transforms for large m (SFNL_ALGO_FAST,
// m up to 512), as two kernels that meet at the grid values.
//
// Same grid, folds and DFT tables as the fused kernels of sfnl_fast.cu (the
// exact truncated product of fft_parallel.F90:147-665 evaluated on an
// alias-free grid N = 4Q); only the split of the work differs.
#include <cuda_runtime.h>

#include <cstring>
#include <map>
#include <atomic>
#include <mutex>
#include <tuple>

#include "sfnl_fold.cuh"
#include "sfnl_internal.h"
#include "sfnl_ops.cuh"

namespace sfnl {

namespace {
// ---------------------------------------------------------------------------
// large m: the same folded transforms in two kernels, program by program
// ---------------------------------------------------------------------------
// Beyond m ~ 100 one CTA cannot hold an 8-point tile's coefficients of six fields and its folded
// products at once (at m = 256: 196 KB and 147 KB), so the transforms are split at the grid values:
//   large_syn_kernel  one CTA per (four 8-point tiles, field): stages the field's 2m coefficient rows,
//                     runs the four class contractions on every angle tile (each B fragment of the
//                     table shared by the four point tiles), folds to the four quadrants and writes
//                     the grid values in fragment order, G[field][tile][t][quadrant][e][32];
//   large_prod_kernel one CTA per 8-point tile and group of up to three outputs: for chunks of LCT angle
//                     tiles it reads the program's grid values (each lane its own fragment elements),
//                     evaluates the whole program (sfnl_ops.cuh) and the analysis pre-fold of the group's
//                     outputs into shared memory, and every warp adds the chunk's k-steps to the
//                     accumulators of its output tiles; the outputs are written at the end.
// The whole program is evaluated on the grid, so a linearised product du x w + u x dw is analysed once,
// and the fields shared by all tangents of a batch (the base state) are transformed once per point chunk.
// With an even number of quadrant angle tiles (every m > 96: the quadrant is a multiple of 16 angles)
// large_syn_tf_kernel and large_prod_tf_kernel do the same with the third fold (mirror tile pairs),
// a quarter fewer DMMAs.
// G lives in a per-(device, stream) workspace; the points are processed in chunks that bound it.
constexpr int kLargeSynMaxWarps = 12, kLargeProdWarps = 16, kLCT = 4, kLargeGroup = 3;
constexpr int kLargeTfPairs = 4;  // mirror pairs per chunk of the third-fold program kernel (16 warps: 8 tiles x 2)
constexpr size_t kLargeSynSmem = 200 * 1024;  // staged coefficients of one synthesis CTA

struct LargeArgs {
  const double *in[kMaxIn];
  double *out[kMaxOut];
  int64_t in_ldm[kMaxIn], out_ldm[kMaxOut], in_bs[kMaxIn], out_bs[kMaxOut];
  int64_t gslot[kMaxIn];  // G offset of each field (units of tiles * NT * 256 doubles)
  int syn_f[kMaxIn];      // large_syn_kernel: the fields this launch synthesises (blockIdx.y indexes it)
  int64_t npts;     // points of this chunk (fields are offset to its first point)
  int64_t in_sin;   // sine offset of the inputs (the arrays' np)
  int64_t out_sin;  // sine offset of the outputs (np * point stride)
  int64_t out_ps;   // point stride of the outputs
  int NT, NU_tot, KS_tot;
  int ks_off[4], KS[4], nu_off[4], ke[4];
  unsigned adj_in;  // bit f: field f is a cotangent
  int adj_out, vec16, batch_entry;  // batch entry of blockIdx.z == 0 (synthesis) / blockIdx.y == 0 (program)
  int nown;                          // workspace slots per batch entry (the batched fields)
  int nbl;                           // batch entries per launch (gridDim.z of the synthesis, gridDim.y of the program)
  const double *syn, *ana;
  double *G;
  int64_t tiles;
  // third fold (NT even): groups 0 CE0, 1 CE2, 2 CO, 3 SE0, 4 SE2, 5 SO
  int tkoff[7], tks[6], tnuoff[7], tnu[6], taoff[7], tke[3];
  int asteps;  // k-steps of one analysis-table variant
  int nyq;     // residue pass: the sine row and output of mode 0 carry the residue grid's Nyquist mode
};

// PT 8-point tiles of one field per CTA: each B fragment of the DFT table (read from L2) feeds PT
// DMMAs.  With one tile per CTA the whole table (786 KB at m = 256) streams from L2 for every 8 points
// of every field, and L2 bandwidth, not the FP64 pipe, sets the time.  Warps take the angle tiles in turn.
template <int PT>
__global__ void __launch_bounds__(kLargeSynMaxWarps * 32) large_syn_kernel(const LargeArgs a) {
  extern __shared__ double xs[];  // [PT][KS_tot][4][8] of one field, points swizzled (a_frag_slot)
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  const int f = a.syn_f[blockIdx.y];
  const int64_t tile0 = (int64_t)blockIdx.x * PT, p0 = tile0 * 8;
  const int NT = a.NT, KT = 4 * a.KS_tot;
  const size_t pts = (size_t)a.KS_tot * 32;  // point-tile stride in xs
  const int bz = blockIdx.z;  // entries a.batch_entry + bz (batched fields only; 0 for the shared ones)
  const double *in_f = a.in[f] + (int64_t)(a.batch_entry + bz) * a.in_bs[f];
  const int64_t gslot_f = a.gslot[f] + (a.in_bs[f] ? (int64_t)bz * a.nown : 0);
  const int64_t ldm = a.in_ldm[f];
  int KS[4], KOFF[4], KE[4];
#pragma unroll
  for (int c = 0; c < 4; ++c) {
    KS[c] = a.KS[c];
    KOFF[c] = a.ks_off[c];
    KE[c] = a.ke[c];
  }
  {  // stage: 4*PT threads per row, two points each (16-byte copies when aligned)
    constexpr int tpr = 4 * PT;
    const int pc = 2 * (threadIdx.x % tpr), rstep = blockDim.x / tpr;
    const bool v16 = a.vec16 && p0 + pc + 2 <= a.npts;
    const bool pv0 = p0 + pc < a.npts, pv1 = p0 + pc + 1 < a.npts;
    const double *base = in_f + p0 + pc;
    double *dst0 = xs + (size_t)(pc >> 3) * pts;
    for (int r = threadIdx.x / tpr; r < KT; r += rstep) {
      const int c = (r >= 4 * KOFF[1]) + (r >= 4 * KOFF[2]) + (r >= 4 * KOFF[3]);
      const int k = r - 4 * sel4(KOFF, c), n = class_mode(c, k);
      double *dst = dst0 + (size_t)(r >> 2) * 32 + a_frag_slot(r & 3, pc & 7);
      const bool live = k < sel4(KE, c) && !(c == 2 && n == 0);  // the sine of mode 0 is ignored
      const double *src = base + (int64_t)n * ldm + (c >= 2 ? a.in_sin : 0);
      if (live && v16) {
        cp_async16(dst, src);
      } else {
        if (live && pv0) cp_async8(dst, src); else dst[0] = 0.0;
        if (live && pv1) cp_async8(dst + 1, src + 1); else dst[1] = 0.0;
      }
    }
  }
  cp_async_wait_all();
  __syncthreads();
  if ((a.adj_in >> f) & 1u) {  // a cotangent: synthesised with the analysis weights 1/N (n = 0), 2/N
    const double invN = 1.0 / (4.0 * 8.0 * NT), twoN = 2.0 * invN;
    for (size_t i = threadIdx.x; i < PT * pts; i += blockDim.x) {
      const int ks = (int)((i % pts) >> 5);
      const bool n0 = (ks == KOFF[0] || ks == KOFF[2]) && ((i >> 3) & 3) == 0;  // k = 0 of an even class
      xs[i] *= n0 ? invN : twoN;
    }
    __syncthreads();
  }
  const double *xs_l = xs + a_frag_slot(lane & 3, lane >> 2);
  int ks_max = KS[0];
#pragma unroll
  for (int c = 1; c < 4; ++c) ks_max = KS[c] > ks_max ? KS[c] : ks_max;
  const size_t bstride = (size_t)NT * 32;
  for (int t = warp; t < NT; t += nw) {
    double acc[PT][4][2];
#pragma unroll
    for (int pt = 0; pt < PT; ++pt)
#pragma unroll
      for (int c = 0; c < 4; ++c) acc[pt][c][0] = acc[pt][c][1] = 0.0;
    const double *bt = a.syn + (size_t)t * 32 + lane;
    // B fragments of k-step s + 1 are loaded while those of s feed the DMMAs (the table is read from L2)
    double bn[4];
#pragma unroll
    for (int c = 0; c < 4; ++c) bn[c] = KS[c] > 0 ? __ldg(bt + (size_t)KOFF[c] * bstride) : 0.0;
    for (int s = 0; s < ks_max; ++s) {
      double bc[4];
#pragma unroll
      for (int c = 0; c < 4; ++c) {
        bc[c] = bn[c];
        if (s + 1 < sel4(KS, c)) bn[c] = __ldg(bt + (size_t)(sel4(KOFF, c) + s + 1) * bstride);
      }
#pragma unroll
      for (int c = 0; c < 4; ++c) {
        if (s >= sel4(KS, c)) continue;
        const size_t ks = (size_t)(sel4(KOFF, c) + s);
#pragma unroll
        for (int pt = 0; pt < PT; ++pt) dmma(acc[pt][c], xs_l[pt * pts + ks * 32], bc[c]);
      }
    }
#pragma unroll
    for (int pt = 0; pt < PT; ++pt) {
      const int64_t tile = tile0 + pt;
      if (tile >= a.tiles) break;
      double *gp0 = a.G + ((gslot_f * a.tiles + tile) * NT + t) * 256 + lane;
#pragma unroll
      for (int e = 0; e < 2; ++e) {
        const double A = acc[pt][0][e] + acc[pt][1][e], B = acc[pt][0][e] - acc[pt][1][e];
        const double C = acc[pt][2][e] + acc[pt][3][e], D = acc[pt][3][e] - acc[pt][2][e];
        double *gp = gp0 + e * 32;
        gp[0 * 64] = A + C;  // theta
        gp[1 * 64] = B + D;  // pi - theta
        gp[2 * 64] = B - D;  // pi + theta
        gp[3 * 64] = A - C;  // 2 pi - theta
      }
    }
  }
}

// The synthesis with the third fold (NT even): the quadrant grid is its own mirror (theta -> pi/2 - theta
// maps tile t to NT-1-t, local angle a to 7-a: lane (g, q) to (g, 3-q), parity e to 1-e), and for even n
// cos(n(pi/2 - x)) = (-1)^(n/2) cos(nx), sin(n(pi/2 - x)) = -(-1)^(n/2) sin(nx).  So a warp takes a pair
// (t, NT-1-t): the even classes split into n = 0 and n = 2 (mod 4) parts are contracted on tile t only
// (CE = E0 + E2 there, E0 - E2 at the mirror tile; SE = S0 + S2, S2 - S0), the odd classes on both tiles.
// A quarter of the DMMAs goes.  Staged rows in group order CE0, CE2, CO, SE0, SE2, SO.
template <int PT>
__global__ void __launch_bounds__(kLargeSynMaxWarps * 32, 1) large_syn_tf_kernel(const LargeArgs a) {
  extern __shared__ double xs[];  // [PT][KS_tot][4][8], points swizzled (a_frag_slot)
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  const int f = a.syn_f[blockIdx.y];
  const int64_t tile0 = (int64_t)blockIdx.x * PT, p0 = tile0 * 8;
  const int NT = a.NT, NH = NT >> 1, KS_tot = a.tkoff[6], KT = 4 * KS_tot;
  const size_t pts = (size_t)KS_tot * 32;
  const int bz = blockIdx.z;  // entries a.batch_entry + bz (batched fields only; 0 for the shared ones)
  const double *in_f = a.in[f] + (int64_t)(a.batch_entry + bz) * a.in_bs[f];
  const int64_t gslot_f = a.gslot[f] + (a.in_bs[f] ? (int64_t)bz * a.nown : 0);
  const int64_t ldm = a.in_ldm[f];
  {  // stage: 4*PT threads per row, two points each
    constexpr int tpr = 4 * PT;
    const int pc = 2 * (threadIdx.x % tpr), rstep = blockDim.x / tpr;
    const bool v16 = a.vec16 && p0 + pc + 2 <= a.npts;
    const bool pv0 = p0 + pc < a.npts, pv1 = p0 + pc + 1 < a.npts;
    const double *base = in_f + p0 + pc;
    double *dst0 = xs + (size_t)(pc >> 3) * pts;
    for (int r = threadIdx.x / tpr; r < KT; r += rstep) {
      const int ks = r >> 2;
      const int gr = (ks >= a.tkoff[1]) + (ks >= a.tkoff[2]) + (ks >= a.tkoff[3]) + (ks >= a.tkoff[4]) + (ks >= a.tkoff[5]);
      const int kg = gr == 0 ? 0 : gr == 1 ? a.tkoff[1] : gr == 2 ? a.tkoff[2] : gr == 3 ? a.tkoff[3]
                   : gr == 4 ? a.tkoff[4] : a.tkoff[5];
      const int keg = gr % 3 == 0 ? a.tke[0] : gr % 3 == 1 ? a.tke[1] : a.tke[2];
      const int k = r - 4 * kg, n = tf_mode(gr, k);
      double *dst = dst0 + (size_t)ks * 32 + a_frag_slot(r & 3, pc & 7);
      const bool live = k < keg && (a.nyq || !(gr == 3 && k == 0));  // the sine of mode 0 is ignored
      const double *src = base + (int64_t)n * ldm + (gr >= 3 ? a.in_sin : 0);
      if (live && v16) {
        cp_async16(dst, src);
      } else {
        if (live && pv0) cp_async8(dst, src); else dst[0] = 0.0;
        if (live && pv1) cp_async8(dst + 1, src + 1); else dst[1] = 0.0;
      }
    }
  }
  cp_async_wait_all();
  __syncthreads();
  if ((a.adj_in >> f) & 1u) {  // a cotangent: synthesised with the analysis weights 1/N (n = 0), 2/N
    const double invN = 1.0 / (4.0 * 8.0 * NT), twoN = 2.0 * invN;
    for (size_t i = threadIdx.x; i < PT * pts; i += blockDim.x) {
      const int ks = (int)((i % pts) >> 5);
      const bool n0 = (ks == 0 || ks == a.tkoff[3]) && ((i >> 3) & 3) == 0;  // k = 0 of CE0 / SE0
      xs[i] *= n0 ? invN : twoN;
    }
    __syncthreads();
  }
  const double *xs_l = xs + a_frag_slot(lane & 3, lane >> 2);
  const size_t bstride = (size_t)NT * 32;
  const int ks0 = a.tks[0], ks1 = a.tks[1], ks2 = a.tks[2];
  const int ko0 = a.tkoff[0], ko1 = a.tkoff[1], ko2 = a.tkoff[2], ko3 = a.tkoff[3], ko4 = a.tkoff[4], ko5 = a.tkoff[5];
  for (int tau = warp; tau < NH; tau += nw) {
    const int tm = NT - 1 - tau;
    // even parts on tile tau: E0 (CE0), E2 (CE2), S0 (SE0), S2 (SE2)
    double ev[4][PT][2];
#pragma unroll
    for (int j = 0; j < 4; ++j)
#pragma unroll
      for (int pt = 0; pt < PT; ++pt) ev[j][pt][0] = ev[j][pt][1] = 0.0;
    {
      const double *bt = a.syn + (size_t)tau * 32 + lane;
      const int kse = ks0 > ks1 ? ks0 : ks1;
      for (int s = 0; s < kse; ++s) {
#pragma unroll
        for (int j = 0; j < 4; ++j) {
          const int kso = j == 0 ? ko0 : j == 1 ? ko1 : j == 2 ? ko3 : ko4;
          if (s >= ((j & 1) ? ks1 : ks0)) continue;
          const size_t ks = (size_t)(kso + s);
          const double bv = __ldg(bt + ks * bstride);
#pragma unroll
          for (int pt = 0; pt < PT; ++pt) dmma(ev[j][pt], xs_l[pt * pts + ks * 32], bv);
        }
      }
    }
    // the even classes on both tiles: own lane on tau, mirror lane (lane ^ 3) and parity 1 - e on tm
    double ce[2][PT][2], se[2][PT][2];
#pragma unroll
    for (int pt = 0; pt < PT; ++pt)
#pragma unroll
      for (int e = 0; e < 2; ++e) {
        ce[0][pt][e] = ev[0][pt][e] + ev[1][pt][e];
        se[0][pt][e] = ev[2][pt][e] + ev[3][pt][e];
        const double e0 = __shfl_xor_sync(0xffffffffu, ev[0][pt][1 - e], 3);
        const double e2 = __shfl_xor_sync(0xffffffffu, ev[1][pt][1 - e], 3);
        const double s0 = __shfl_xor_sync(0xffffffffu, ev[2][pt][1 - e], 3);
        const double s2 = __shfl_xor_sync(0xffffffffu, ev[3][pt][1 - e], 3);
        ce[1][pt][e] = e0 - e2;
        se[1][pt][e] = s2 - s0;
      }
#pragma unroll
    for (int side = 0; side < 2; ++side) {
      const int t = side ? tm : tau;
      double od[2][PT][2];  // CO, SO
#pragma unroll
      for (int j = 0; j < 2; ++j)
#pragma unroll
        for (int pt = 0; pt < PT; ++pt) od[j][pt][0] = od[j][pt][1] = 0.0;
      const double *bt = a.syn + (size_t)t * 32 + lane;
      for (int s = 0; s < ks2; ++s) {
#pragma unroll
        for (int j = 0; j < 2; ++j) {
          const size_t ks = (size_t)((j ? ko5 : ko2) + s);
          const double bv = __ldg(bt + ks * bstride);
#pragma unroll
          for (int pt = 0; pt < PT; ++pt) dmma(od[j][pt], xs_l[pt * pts + ks * 32], bv);
        }
      }
#pragma unroll
      for (int pt = 0; pt < PT; ++pt) {
        const int64_t tile = tile0 + pt;
        if (tile >= a.tiles) break;
        double *gp0 = a.G + ((gslot_f * a.tiles + tile) * NT + t) * 256 + lane;
#pragma unroll
        for (int e = 0; e < 2; ++e) {
          const double CE = ce[side][pt][e], SE = se[side][pt][e], CO = od[0][pt][e], SO = od[1][pt][e];
          const double A = CE + CO, B = CE - CO, C = SE + SO, D = SO - SE;
          double *gp = gp0 + e * 32;
          gp[0 * 64] = A + C;  // theta
          gp[1 * 64] = B + D;  // pi - theta
          gp[2 * 64] = B - D;  // pi + theta
          gp[3 * 64] = A - C;  // 2 pi - theta
        }
      }
    }
  }
}

// Program and analysis with the third fold: chunks of two angle-tile pairs (t, t+1 and their mirrors); the
// odd output groups contract all four tiles, the even ones P(t) +- P(mirror) over the first-half tiles
// (signs PE0 +, PE2 -, QE0 -, QE2 +).  With up to two output tiles per warp (m <= 256 on the grid's residue
// classes, m <= 192 without them) the kernel is held to 64 registers, two CTAs per SM: a spill of about
// 136 bytes buys twice the resident warps, 4-11 % faster on a B200 from m = 128 to 256; with more tiles per
// warp the accumulators spill too much and one CTA per SM was as fast or faster (m = 384, 512).
template <int OP, int O0, int CPW>
__global__ void __launch_bounds__(kLargeProdWarps * 32, CPW <= 2 ? 2 : 1) large_prod_tf_kernel(const LargeArgs a) {
  constexpr int NI = op_nin(OP), NO = op_nout(OP);
  constexpr int NOG = NO - O0 < kLargeGroup ? NO - O0 : kLargeGroup;
  constexpr int KP = kLargeTfPairs, LT = 2 * KP;  // pairs per chunk, local tiles
  extern __shared__ double pc_s[];  // [NOG][4 classes][LT local tiles][2][32]
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, q = lane & 3;
  const int by = blockIdx.y, b = a.batch_entry + by;  // batch entry of this CTA
  const int64_t tile = blockIdx.x, p = tile * 8 + (lane >> 2);
  const int NT = a.NT, NH = NT >> 1;
  double y[CPW][NOG][2];
#pragma unroll
  for (int j = 0; j < CPW; ++j)
#pragma unroll
    for (int o = 0; o < NOG; ++o) y[j][o][0] = y[j][o][1] = 0.0;
  const int64_t fstride = a.tiles * NT * 256;
  const double *Gl = a.G + tile * NT * 256 + lane;
  const double *anav = a.ana + (size_t)(a.adj_out ? 1 : 0) * a.asteps * 32 + lane;
  const int NU_tot = a.tnuoff[6];
  const size_t cst = (size_t)LT * 2 * 32;  // class stride in pc_s
  for (int c0 = 0; c0 < NH; c0 += KP) {
    const int npr = NH - c0 < KP ? NH - c0 : KP;  // pairs in this chunk
    // local tiles 0 .. KP-1: c0 + lt; KP .. 2KP-1: their mirrors NT-1-(c0 + lt - KP)
    if (warp < 4 * npr) {
      const int li = warp >> 1, e = warp & 1;
      const int lt = li < npr ? li : KP + li - npr;
      const int t = lt < KP ? c0 + lt : NT - 1 - (c0 + lt - KP);
      double gq[4][NOG];
#pragma unroll
      for (int r = 0; r < 4; ++r) {
        double x[NI], yy[NO];
#pragma unroll
        for (int f = 0; f < NI; ++f)
          x[f] = Gl[(a.gslot[f] + (a.in_bs[f] ? (int64_t)by * a.nown : 0)) * fstride + (size_t)t * 256 + r * 64 + e * 32];
        apply_op<OP>(x, yy);
#pragma unroll
        for (int o = 0; o < NOG; ++o) gq[r][o] = yy[O0 + o];
      }
#pragma unroll
      for (int o = 0; o < NOG; ++o) {
        const double s14 = gq[0][o] + gq[3][o], d14 = gq[0][o] - gq[3][o];
        const double s23 = gq[1][o] + gq[2][o], d32 = gq[2][o] - gq[1][o];
        double *dst = pc_s + ((size_t)(o * 4) * LT + lt) * 64 + e * 32 + lane;
        dst[0] = s14 + s23;        // PE
        dst[cst] = s14 - s23;      // PO
        dst[2 * cst] = d14 + d32;  // QE
        dst[3 * cst] = d14 - d32;  // QO
      }
    }
    __syncthreads();
#pragma unroll
    for (int j = 0; j < CPW; ++j) {
      const int cu = warp + kLargeProdWarps * j;
      if (cu >= NU_tot) continue;
      const int gr = (cu >= a.tnuoff[1]) + (cu >= a.tnuoff[2]) + (cu >= a.tnuoff[3]) + (cu >= a.tnuoff[4]) +
                     (cu >= a.tnuoff[5]);
      const int nuo = gr == 0 ? 0 : gr == 1 ? a.tnuoff[1] : gr == 2 ? a.tnuoff[2] : gr == 3 ? a.tnuoff[3]
                    : gr == 4 ? a.tnuoff[4] : a.tnuoff[5];
      const int aof = gr == 0 ? 0 : gr == 1 ? a.taoff[1] : gr == 2 ? a.taoff[2] : gr == 3 ? a.taoff[3]
                    : gr == 4 ? a.taoff[4] : a.taoff[5];
      const bool odd = gr % 3 == 2;
      const int u = cu - nuo, TE = odd ? 2 * NT : NT, c = gr < 3 ? (odd ? 1 : 0) : (odd ? 3 : 2);
      const double sg = (gr == 0 || gr == 4) ? 1.0 : -1.0;
      const double *bt = anav + (size_t)(aof + u * TE) * 32;
      const double *pa = pc_s + (size_t)c * cst + lane;
      if (odd) {
        for (int li = 0; li < 2 * npr; ++li) {
          const int lt = li < npr ? li : KP + li - npr;
          const int t = lt < KP ? c0 + lt : NT - 1 - (c0 + lt - KP);
#pragma unroll
          for (int e = 0; e < 2; ++e) {
            const double bv = __ldg(bt + (size_t)(2 * t + e) * 32);
#pragma unroll
            for (int o = 0; o < NOG; ++o) dmma(y[j][o], pa[(size_t)o * 4 * cst + (size_t)(lt * 2 + e) * 32], bv);
          }
        }
      } else {
        const int lx = (lane ^ 3) - lane;  // mirror lane offset
        for (int lt = 0; lt < npr; ++lt) {
#pragma unroll
          for (int e = 0; e < 2; ++e) {
            const double bv = __ldg(bt + (size_t)(2 * (c0 + lt) + e) * 32);
#pragma unroll
            for (int o = 0; o < NOG; ++o) {
              const double *po = pa + (size_t)o * 4 * cst;
              const double av = po[(size_t)(lt * 2 + e) * 32] + sg * po[(size_t)((KP + lt) * 2 + 1 - e) * 32 + lx];
              dmma(y[j][o], av, bv);
            }
          }
        }
      }
    }
    __syncthreads();
  }
  if (p >= a.npts) return;
#pragma unroll
  for (int j = 0; j < CPW; ++j) {
    const int cu = warp + kLargeProdWarps * j;
    if (cu >= NU_tot) continue;
    const int gr = (cu >= a.tnuoff[1]) + (cu >= a.tnuoff[2]) + (cu >= a.tnuoff[3]) + (cu >= a.tnuoff[4]) +
                   (cu >= a.tnuoff[5]);
    const int nuo = gr == 0 ? 0 : gr == 1 ? a.tnuoff[1] : gr == 2 ? a.tnuoff[2] : gr == 3 ? a.tnuoff[3]
                  : gr == 4 ? a.tnuoff[4] : a.tnuoff[5];
    const int keg = gr % 3 == 0 ? a.tke[0] : gr % 3 == 1 ? a.tke[1] : a.tke[2];
    const int u = cu - nuo;
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const int kk = 8 * u + 2 * q + h;
      if (kk >= keg) continue;
      const int n = tf_mode(gr, kk);
#pragma unroll
      for (int o = 0; o < NOG; ++o) {
        const int og = O0 + o;
        double *dst = a.out[og] + (int64_t)b * a.out_bs[og] + p * a.out_ps + (int64_t)n * a.out_ldm[og] +
                      (gr >= 3 ? a.out_sin : 0);
        *dst = (gr >= 3 && n == 0 && !a.nyq) ? 0.0 : y[j][o][h];
      }
    }
  }
}

// Outputs O0 .. O0+NOG-1 of program OP for batch entry a.batch_entry (the output group is a template
// parameter so that the program's values stay in registers).
template <int OP, int O0, int CPW>
__global__ void __launch_bounds__(kLargeProdWarps * 32) large_prod_kernel(const LargeArgs a) {
  constexpr int NI = op_nin(OP), NO = op_nout(OP);
  constexpr int NOG = NO - O0 < kLargeGroup ? NO - O0 : kLargeGroup;
  extern __shared__ double pc_s[];  // [NOG][4][LCT][2][32]
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, q = lane & 3;
  const int by = blockIdx.y, b = a.batch_entry + by;  // batch entry of this CTA
  const int64_t tile = blockIdx.x, p = tile * 8 + (lane >> 2);
  const int NT = a.NT;
  double y[CPW][NOG][2];
#pragma unroll
  for (int j = 0; j < CPW; ++j)
#pragma unroll
    for (int o = 0; o < NOG; ++o) y[j][o][0] = y[j][o][1] = 0.0;
  const int64_t fstride = a.tiles * NT * 256;
  const double *Gl = a.G + tile * NT * 256 + lane;
  const double *anav = a.ana + (size_t)(a.adj_out ? 1 : 0) * a.NU_tot * NT * 2 * 32 + lane;
  const size_t cst = (size_t)kLCT * 2 * 32;  // class stride in pc_s
  for (int t0 = 0; t0 < NT; t0 += kLCT) {
    const int ct = NT - t0 < kLCT ? NT - t0 : kLCT;
    // the program and the analysis pre-fold of the group at (tile t0 + tt, parity e) = warp
    if (warp < 2 * ct) {
      const int tt = warp >> 1, e = warp & 1, t = t0 + tt;
      double gq[4][NOG];
#pragma unroll
      for (int r = 0; r < 4; ++r) {
        double x[NI], yy[NO];
#pragma unroll
        for (int f = 0; f < NI; ++f)
          x[f] = Gl[(a.gslot[f] + (a.in_bs[f] ? (int64_t)by * a.nown : 0)) * fstride + (size_t)t * 256 + r * 64 + e * 32];
        apply_op<OP>(x, yy);
#pragma unroll
        for (int o = 0; o < NOG; ++o) gq[r][o] = yy[O0 + o];
      }
#pragma unroll
      for (int o = 0; o < NOG; ++o) {
        const double s14 = gq[0][o] + gq[3][o], d14 = gq[0][o] - gq[3][o];
        const double s23 = gq[1][o] + gq[2][o], d32 = gq[2][o] - gq[1][o];
        double *dst = pc_s + ((size_t)(o * 4) * kLCT + tt) * 64 + e * 32 + lane;
        dst[0] = s14 + s23;        // PE
        dst[cst] = s14 - s23;      // PO
        dst[2 * cst] = d14 + d32;  // QE
        dst[3 * cst] = d14 - d32;  // QO
      }
    }
    __syncthreads();
#pragma unroll
    for (int j = 0; j < CPW; ++j) {
      const int cu = warp + kLargeProdWarps * j;
      if (cu >= a.NU_tot) continue;
      const int c = (cu >= a.nu_off[1]) + (cu >= a.nu_off[2]) + (cu >= a.nu_off[3]);
      const double *bt = anav + ((size_t)cu * NT + t0) * 2 * 32;
      const double *pa = pc_s + (size_t)c * cst + lane;
      for (int te = 0; te < 2 * ct; ++te) {
        const double bv = __ldg(bt + (size_t)te * 32);
#pragma unroll
        for (int o = 0; o < NOG; ++o) dmma(y[j][o], pa[(size_t)o * 4 * cst + (size_t)te * 32], bv);
      }
    }
    __syncthreads();
  }
  if (p >= a.npts) return;
#pragma unroll
  for (int j = 0; j < CPW; ++j) {
    const int cu = warp + kLargeProdWarps * j;
    if (cu >= a.NU_tot) continue;
    const int c = (cu >= a.nu_off[1]) + (cu >= a.nu_off[2]) + (cu >= a.nu_off[3]);
    const int u = cu - (c == 0 ? 0 : c == 1 ? a.nu_off[1] : c == 2 ? a.nu_off[2] : a.nu_off[3]);
    const int kec = c == 0 ? a.ke[0] : c == 1 ? a.ke[1] : c == 2 ? a.ke[2] : a.ke[3];
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const int kk = 8 * u + 2 * q + h;
      if (kk >= kec) continue;
      const int n = class_mode(c, kk);
#pragma unroll
      for (int o = 0; o < NOG; ++o) {
        const int og = O0 + o;
        double *dst = a.out[og] + (int64_t)b * a.out_bs[og] + p * a.out_ps + (int64_t)n * a.out_ldm[og] +
                      (c >= 2 ? a.out_sin : 0);
        *dst = (c == 2 && n == 0) ? 0.0 : y[j][o][h];
      }
    }
  }
}

// workspaces, one per (device, stream, use): calls on different streams do not share them.  Use 0: the
// grid values; 1: the residue coefficients and sums of launch_large_res.
std::mutex g_lws_mu;
std::map<std::tuple<int, cudaStream_t, int>, std::pair<double *, size_t>> g_lws;

int large_workspace(cudaStream_t st, size_t bytes, double **out, int use = 0) {
  int dev = 0;
  cudaGetDevice(&dev);
  std::lock_guard<std::mutex> lk(g_lws_mu);
  auto &w = g_lws[{dev, st, use}];
  if (w.second < bytes) {
    if (w.first) {
      cudaStreamSynchronize(st);  // the previous call on this stream may still read it
      cudaFree(w.first);
    }
    w.first = nullptr;
    w.second = 0;
    if (cudaMalloc(&w.first, bytes) != cudaSuccess) {
      cudaGetLastError();
      return set_error(SFNL_ERR_ALLOC, "cudaMalloc of the large-m workspace failed");
    }
    w.second = bytes;
  }
  *out = w.first;
  return SFNL_OK;
}

template <int OP, int O0, int CPW>
int launch_large_prod(const LargeArgs &la, bool tf, cudaStream_t st) {
  constexpr int NO = op_nout(OP), NOG = NO - O0 < kLargeGroup ? NO - O0 : kLargeGroup;
  const size_t smem = sizeof(double) * (size_t)NOG * 4 * (tf ? 2 * kLargeTfPairs : kLCT) * 2 * 32;
  auto kern = tf ? large_prod_tf_kernel<OP, O0, CPW> : large_prod_kernel<OP, O0, CPW>;
  if (smem > 48 * 1024 && cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess)
    return set_error(SFNL_ERR_CUDA, "cudaFuncSetAttribute failed (large-m program and analysis)");
  kern<<<dim3((unsigned)la.tiles, (unsigned)la.nbl), kLargeProdWarps * 32, smem, st>>>(la);
  return check_launch("large-m program and analysis");
}

// Output group G (outputs 3G .. 3G+2) of program OP.
template <int OP, int G>
int launch_large_group(const LargeArgs &la, bool tf, cudaStream_t st) {
  constexpr int O0 = kLargeGroup * G;
  if constexpr (O0 >= op_nout(OP)) {
    return SFNL_OK;
  } else {
    const int nu = tf ? la.tnuoff[6] : la.NU_tot;
    switch ((nu + kLargeProdWarps - 1) / kLargeProdWarps) {
      case 1: return launch_large_prod<OP, O0, 1>(la, tf, st);
      case 2: return launch_large_prod<OP, O0, 2>(la, tf, st);
      case 3: return launch_large_prod<OP, O0, 3>(la, tf, st);
      case 4: return launch_large_prod<OP, O0, 4>(la, tf, st);
      case 5: return launch_large_prod<OP, O0, 5>(la, tf, st);
      case 6: return launch_large_prod<OP, O0, 6>(la, tf, st);
      case 7: return launch_large_prod<OP, O0, 7>(la, tf, st);
      case 8: return launch_large_prod<OP, O0, 8>(la, tf, st);
    }
    return set_error(SFNL_ERR_UNSUPPORTED, "large-m FAST form: too many output tiles");
  }
}

template <int OP>
int launch_large_prod_all(const LargeArgs &la, bool tf, cudaStream_t st) {
  static_assert(op_nout(OP) <= 4 * kLargeGroup, "output groups");
  if (int rc = launch_large_group<OP, 0>(la, tf, st)) return rc;
  if (int rc = launch_large_group<OP, 1>(la, tf, st)) return rc;
  if (int rc = launch_large_group<OP, 2>(la, tf, st)) return rc;
  return launch_large_group<OP, 3>(la, tf, st);
}

int launch_large_prod_op(int op, const LargeArgs &la, bool tf, cudaStream_t st) {
  switch (op) {
    case OP_CROSS: return launch_large_prod_all<OP_CROSS>(la, tf, st);
    case OP_DOT: return launch_large_prod_all<OP_DOT>(la, tf, st);
    case OP_PROD: return launch_large_prod_all<OP_PROD>(la, tf, st);
    case OP_BUNDLE: return launch_large_prod_all<OP_BUNDLE>(la, tf, st);
    case OP_CROSS_JVP: return launch_large_prod_all<OP_CROSS_JVP>(la, tf, st);
    case OP_CROSS_VJP: return launch_large_prod_all<OP_CROSS_VJP>(la, tf, st);
    case OP_MHD_JVP: return launch_large_prod_all<OP_MHD_JVP>(la, tf, st);
    case OP_MHD_VJP: return launch_large_prod_all<OP_MHD_VJP>(la, tf, st);
    case OP_SVECT: return launch_large_prod_all<OP_SVECT>(la, tf, st);
    case OP_TENSOR: return launch_large_prod_all<OP_TENSOR>(la, tf, st);
    case OP_ADVECT: return launch_large_prod_all<OP_ADVECT>(la, tf, st);
  }
  return set_error(SFNL_ERR_ARG, "large-m FAST form: program not bilinear");
}

// nbz: batch entries (blockIdx.z) of the launch, 1 for the batch-invariant fields.
int launch_large_syn(const LargeArgs &la, int nfields, int nbz, bool tf, cudaStream_t st) {
  if (nfields == 0) return SFNL_OK;
  // angle tiles (pairs of mirror tiles with the third fold) spread evenly over at most kLargeSynMaxWarps warps
  const int units = tf ? la.NT / 2 : la.NT;
  const int rounds = (units + kLargeSynMaxWarps - 1) / kLargeSynMaxWarps, nw = (units + rounds - 1) / rounds;
  const size_t tile_bytes = sizeof(double) * (size_t)(tf ? la.tkoff[6] : la.KS_tot) * 32;
  auto go = [&](auto kern, int pt) {
    const size_t smem = tile_bytes * pt;
    if (smem > 48 * 1024 && cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess)
      return set_error(SFNL_ERR_CUDA, "cudaFuncSetAttribute failed (large-m synthesis)");
    const int64_t blocks = (la.tiles + pt - 1) / pt;
    kern<<<dim3((unsigned)blocks, (unsigned)nfields, (unsigned)nbz), nw * 32, smem, st>>>(la);
    return check_launch("large-m synthesis");
  };
  if (tf) {
    // two point tiles per CTA: at 118 registers and 2 x 16-32 KB of staged rows, four CTAs share an SM; four
    // tiles per CTA (each B fragment feeding four DMMAs) left three 4-warp CTAs per SM (168 registers) and
    // were 10-30 % slower (m = 128 to 512)
    if (2 * tile_bytes <= kLargeSynSmem) return go(large_syn_tf_kernel<2>, 2);
  } else {
    if (4 * tile_bytes <= kLargeSynSmem) return go(large_syn_kernel<4>, 4);
    if (2 * tile_bytes <= kLargeSynSmem) return go(large_syn_kernel<2>, 2);
  }
  return set_error(SFNL_ERR_UNSUPPORTED, "large-m FAST form: m too large");
}

constexpr size_t kLargeWorkspaceBytes = size_t(1) << 30;  // grid values of one point chunk
// Tests only (sfnl_test_large_workspace_cap): a bound on both workspaces far below the production ones, so
// that small calls run many point chunks and batch groups; 0: none.
std::atomic<size_t> g_test_cap{0};
// Batched programs (tangents): the workspace may grow to this, or to a quarter of the free device memory,
// so that one launch serves every batch entry of a point chunk of at least kLargeMinChunk points.
constexpr size_t kLargeBatchWorkspaceBytes = size_t(8) << 30;
constexpr int64_t kLargeMinChunk = 4096;

}  // namespace

void large_res_release_tables();

void large_release_workspaces() {
  std::lock_guard<std::mutex> lk(g_lws_mu);
  int prev = 0;
  cudaGetDevice(&prev);
  for (auto &kv : g_lws)
    if (kv.second.first) {
      cudaSetDevice(std::get<0>(kv.first));
      cudaFree(kv.second.first);  // waits for the work still reading it
    }
  g_lws.clear();
  cudaSetDevice(prev);
  large_res_release_tables();
}

namespace {

struct LargePlan {
  int N, NT;                 // grid length and quadrant angle tiles of the pass
  int mt;                    // modes of its third-fold row and output groups
  double *syn, *ana;         // its tables
};

// The two-kernel form: per point chunk, the batch-invariant fields (base state) once, then the batch
// entries in groups of kb: one synthesis launch for the group's own fields (blockIdx.z = entry) and one
// launch per group of three outputs (blockIdx.y = entry).  The grid-value workspace holds the shared
// fields and kb entries' own fields of one point chunk: kb = the whole batch when a chunk of at least
// kLargeMinChunk points fits the batched workspace bound, else as many entries as such a chunk allows.
// rp: a residue pass (launch_large_res): the residue grid's geometry and tables, the Nyquist mode in the
// sine row of mode 0, no analysis weights and no cotangent weights (both applied outside).
int run_large(const ProgArgs &a, const Geo &g, const Tables &T, const LargePlan *rp, cudaStream_t st) {
  const int ni = op_nin(a.op), no = op_nout(a.op);
  int nshared = 0, nown = 0;  // batch-invariant fields take the first G slots, the batched ones the next
  int64_t gslot[kMaxIn];
  for (int f = 0; f < ni; ++f) gslot[f] = a.in_bs[f] == 0 ? nshared++ : -1;
  for (int f = 0; f < ni; ++f)
    if (gslot[f] < 0) gslot[f] = nshared + nown++;
  const size_t field_bytes = sizeof(double) * (size_t)(rp ? rp->N : g.N);  // one field's grid values per point
  size_t cap = kLargeWorkspaceBytes;
  int kb = 1;
  if (a.batch > 1 && nown > 0) {
    size_t free_b = 0, total_b = 0;
    if (cudaMemGetInfo(&free_b, &total_b) != cudaSuccess) {
      cudaGetLastError();
      free_b = 0;
    }
    size_t bcap = kLargeBatchWorkspaceBytes < free_b / 4 ? kLargeBatchWorkspaceBytes : free_b / 4;
    if (bcap < cap) bcap = cap;
    const size_t per_entry = field_bytes * nown * (size_t)kLargeMinChunk;
    const size_t shared_b = field_bytes * nshared * (size_t)kLargeMinChunk;
    const int64_t fit = bcap > shared_b ? (int64_t)((bcap - shared_b) / per_entry) : 0;
    kb = (int)(fit < 1 ? 1 : fit > a.batch ? a.batch : fit);
    cap = bcap;
  }
  if (const size_t tc = g_test_cap.load()) {
    cap = tc;
    if (a.batch > 1 && nown > 0) {
      const int64_t fit = (int64_t)(tc / (field_bytes * (size_t)(nshared + nown) * 32));
      kb = (int)(fit < 1 ? 1 : fit > a.batch ? a.batch : fit);
    }
  }
  const size_t per_point = field_bytes * (size_t)(nshared + (int64_t)kb * nown);
  int64_t chunk = (int64_t)(cap / per_point);
  chunk = (chunk / 32) * 32;
  if (chunk < 32) chunk = 32;
  if (chunk > a.np) chunk = ((a.np + 7) / 8) * 8;
  double *G = nullptr;
  if (int rc = large_workspace(st, per_point * (size_t)chunk, &G)) return rc;
  // the third fold needs mirror pairs of angle tiles
  const int NT = rp ? rp->NT : g.NT, mt = rp ? rp->mt : g.m;
  const bool tf = NT % 2 == 0;
  Tables TT = T;
  if (rp) {
    TT.syn = rp->syn;
    TT.ana = rp->ana;
  } else if (tf) {
    if (int rc = get_tf_tables(g, &TT)) return rc;
  }
  const bool adj_out = rp ? true : op_adjoint_out(a.op);
  unsigned adj = 0;
  for (int f = 0; f < ni && !rp; ++f)
    if (op_adjoint_in(a.op, f)) adj |= 1u << f;
  for (int64_t c0 = 0; c0 < a.np; c0 += chunk) {
    LargeArgs la;
    std::memset(&la, 0, sizeof(la));
    la.npts = a.np - c0 < chunk ? a.np - c0 : chunk;
    la.tiles = (la.npts + 7) / 8;
    la.in_sin = a.np;
    la.out_ps = a.out_ps;
    la.out_sin = a.np * a.out_ps;
    la.nown = nown;
    int v16 = (a.np & 1) ? 0 : 1;
    for (int f = 0; f < ni; ++f) {
      la.in[f] = a.in[f] + c0;
      la.in_ldm[f] = a.in_ldm[f];
      la.in_bs[f] = a.in_bs[f];
      la.gslot[f] = gslot[f];
      if ((reinterpret_cast<uintptr_t>(la.in[f]) & 15) || (la.in_ldm[f] & 1) || (la.in_bs[f] & 1)) v16 = 0;
    }
    for (int o = 0; o < no; ++o) {
      la.out[o] = a.out[o] + c0 * a.out_ps;
      la.out_ldm[o] = a.out_ldm[o];
      la.out_bs[o] = a.out_bs[o];
    }
    la.NT = NT;
    la.NU_tot = g.NU_tot;
    la.KS_tot = g.KS_tot;
    for (int c = 0; c < 4; ++c) {
      la.ks_off[c] = g.ks_off[c];
      la.KS[c] = g.KS[c];
      la.nu_off[c] = g.nu_off[c];
      la.ke[c] = g.ke[c];
    }
    la.adj_in = adj;
    la.adj_out = adj_out ? 1 : 0;
    la.vec16 = v16;
    la.syn = TT.syn;
    la.ana = TT.ana;
    la.G = G;
    // third-fold row and output groups of mt modes; the analysis k-steps of a group over NT angle tiles
    la.taoff[0] = 0;
    for (int gr = 0; gr < 7; ++gr) {
      la.tkoff[gr] = tf_koff(mt, gr);
      la.tnuoff[gr] = tf_nuoff(mt, gr);
      if (gr > 0) la.taoff[gr] = la.taoff[gr - 1] + tf_NU(mt, gr - 1) * ((gr - 1) % 3 == 2 ? 2 * NT : NT);
    }
    for (int gr = 0; gr < 6; ++gr) {
      la.tks[gr] = tf_KS(mt, gr);
      la.tnu[gr] = tf_NU(mt, gr);
    }
    for (int gr = 0; gr < 3; ++gr) la.tke[gr] = tf_ke(mt, gr);
    la.asteps = la.taoff[6];
    la.nyq = rp ? 1 : 0;
    // the batch-invariant fields, once per chunk
    int k = 0;
    for (int f = 0; f < ni; ++f)
      if (a.in_bs[f] == 0) la.syn_f[k++] = f;
    la.batch_entry = 0;
    la.nbl = 1;
    if (int rc = launch_large_syn(la, k, 1, tf, st)) return rc;
    for (int b0 = 0; b0 < a.batch; b0 += kb) {
      la.batch_entry = b0;
      la.nbl = a.batch - b0 < kb ? a.batch - b0 : kb;
      k = 0;
      for (int f = 0; f < ni; ++f)
        if (a.in_bs[f] != 0) la.syn_f[k++] = f;
      if (int rc = launch_large_syn(la, k, la.nbl, tf, st)) return rc;
      if (int rc = launch_large_prod_op(a.op, la, tf, st)) return rc;
    }
  }
  return SFNL_OK;
}

// ---------------------------------------------------------------------------
// the grid's residue classes (m >= 256)
// ---------------------------------------------------------------------------
// On theta_j = pi(2j+1)/N with N = 3m, j = R i + r (r < R, R dividing N) gives theta_j = phi_i + d_r with
// phi_i = pi(2i+1)/M the offset grid of M = N/R angles and d_r = pi(2r + 1 - R)/N.  A field
// Re sum_n z_n e^{i n theta} (z_n = a_n - i b_n, n < m) is on residue r the series of y_n = z_n e^{i n d_r}
// on phi, where e^{i M phi_i} = -1: mode n = qM + k (k < M) is mode k with the sign (-1)^q, so that
// Y_k = sum_q (-1)^q y_{qM+k}, and the modes k and M - k fold into alpha_k - i beta_k = Y_k - conj(Y_{M-k})
// (k = 1 .. M/2 - 1), alpha_0 = Re Y_0, with mode M/2 alone as a sine (cos(M/2 phi_i) = 0):
// beta_{M/2} = -Im Y_{M/2}.  Each residue is a transform of M real coefficients to M angles, third-folded
// like the whole grid: 1/R of the DMMAs of each of R transforms instead of one on N angles, i.e. 3/R of
// the work at the same m.  With C^r_k, S^r_k the residue's cosine and sine sums of a product,
// sum_j p_j e^{-i n theta_j} = sum_r e^{-i n d_r} P^r_n with P^r_k = C^r_k - i S^r_k (k <= M/2),
// P^r_{M-k} = -conj(P^r_k), P^r_{qM+k} = (-1)^q P^r_k and P^r_{M/2} = -i S^r_{M/2}.  The residue passes run
// the two kernels above on the M-angle grid (mode M/2's sine in the sine row of mode 0), between a kernel
// that forms the residues' coefficients and one that adds their shares to the outputs.  Both move N doubles
// per field and point whatever R is, so more residues cost only their twiddles (R complex products per
// mode).  At m = 128 the passes over the coefficients and sums cost more than the DMMAs saved (cross
// product at 100k points 2.65 -> 2.93 ms with R = 3); from m = 256 on the residues win.
constexpr int kMaxResidues = 12;
std::atomic<int> g_test_residues{0};  // tests: force R (0: the choice below)

bool residues_fit(int m, int N, int R) {
  if (N != 3 * m || R < 3 || R > kMaxResidues || N % R) return false;
  const int M = N / R;
  return M >= 64 && M % 64 == 0 && M <= 512;  // an even number of quadrant tiles (third fold), kernels' range
}

// Residue classes of the two-kernel form for m modes on the N-angle grid; 0: the whole grid.  Six where
// they fit, else three: on a B200, R = 6 against 3 took the cross product at m = 256 (350k points) from
// 18.7 to 16.9 ms, at m = 384 (100k points) from 11.4 to 7.9 ms and at m = 512 (60k points) from 10.1 to
// 6.8 ms, the 16-tangent MHD JVP at m = 256 (50k points) from 87.0 to 80.3 ms; residue grids of 64 angles
// (R = 12 at m = 256) were slower than both.
int large_residues(int m, int N) {
  if (const int R = g_test_residues.load()) return residues_fit(m, N, R) ? R : 0;
  if (m < 256 || m > 512) return 0;
  return residues_fit(m, N, 6) ? 6 : residues_fit(m, N, 3) ? 3 : 0;
}

struct ResTab {
  double *base = nullptr;  // syn, ana (two equal variants, no weights), tw [R][m][2]
  double *syn = nullptr, *ana = nullptr;
  const double *tw = nullptr;
};
std::mutex g_res_mu;
std::map<std::tuple<int, int, int>, ResTab> g_res;  // (device, m, R) -> tables

__host__ __device__ constexpr int res_mode(int gr, int k, int mh) { return (gr == 3 && k == 0) ? mh : tf_mode(gr, k); }

// Third-fold tables of the residue grid (M angles, quadrant tiles NT = M/32, row and output groups of M/2
// modes with mode M/2 as the sine of group 3's k = 0), laid out like get_tf_tables', and the twiddles
// cos, sin of n d_r for n < m, r < R.
int get_residue_tables(int m, int N, int R, ResTab *out) {
  int dev = 0;
  cudaGetDevice(&dev);
  std::lock_guard<std::mutex> lk(g_res_mu);
  auto it = g_res.find({dev, m, R});
  if (it != g_res.end()) {
    *out = it->second;
    return SFNL_OK;
  }
  const int M = N / R, mh = M / 2, NT = M / 32;
  const long double pi = acosl(-1.0L);
  auto phi = [&](int j) { return pi * (long double)(2 * j + 1) / (long double)M; };
  const int ks_tot = tf_koff(mh, 6);
  int asteps = 0, aoff[7];
  for (int gr = 0; gr < 6; ++gr) {
    aoff[gr] = asteps;
    asteps += tf_NU(mh, gr) * (gr % 3 == 2 ? 2 * NT : NT);
  }
  aoff[6] = asteps;
  const size_t nsyn = (size_t)ks_tot * NT * 32, nana = (size_t)2 * asteps * 32;
  std::vector<double> h(nsyn + nana + 2 * (size_t)R * m, 0.0);
  for (int gr = 0; gr < 6; ++gr)
    for (int s = 0; s < tf_KS(mh, gr); ++s)
      for (int t = 0; t < NT; ++t)
        for (int l = 0; l < 32; ++l) {
          const int k = 4 * s + (l & 3);
          if (k >= tf_ke(mh, gr)) continue;
          const long double x = (long double)res_mode(gr, k, mh) * phi(8 * t + (l >> 2));
          h[((size_t)(tf_koff(mh, gr) + s) * NT + t) * 32 + l] = (double)(gr < 3 ? cosl(x) : sinl(x));
        }
  for (int var = 0; var < 2; ++var)
    for (int gr = 0; gr < 6; ++gr) {
      const int TE = gr % 3 == 2 ? 2 * NT : NT;
      for (int u = 0; u < tf_NU(mh, gr); ++u)
        for (int te = 0; te < TE; ++te)
          for (int l = 0; l < 32; ++l) {
            const int kk = 8 * u + (l >> 2);
            if (kk >= tf_ke(mh, gr)) continue;
            const long double x = (long double)res_mode(gr, kk, mh) * phi(8 * (te >> 1) + 2 * (l & 3) + (te & 1));
            h[nsyn + ((size_t)var * asteps + aoff[gr] + u * TE + te) * 32 + l] = (double)(gr < 3 ? cosl(x) : sinl(x));
          }
    }
  for (int r = 0; r < R; ++r)
    for (int n = 0; n < m; ++n) {
      const long double x = pi * (long double)n * (long double)(2 * r + 1 - R) / (long double)N;
      h[nsyn + nana + 2 * ((size_t)r * m + n)] = (double)cosl(x);
      h[nsyn + nana + 2 * ((size_t)r * m + n) + 1] = (double)sinl(x);
    }
  ResTab T;
  if (cudaMalloc(&T.base, h.size() * sizeof(double)) != cudaSuccess) {
    cudaGetLastError();
    return set_error(SFNL_ERR_ALLOC, "cudaMalloc of the residue-grid tables failed");
  }
  if (cudaMemcpy(T.base, h.data(), h.size() * sizeof(double), cudaMemcpyHostToDevice) != cudaSuccess) {
    cudaFree(T.base);
    return set_error(SFNL_ERR_CUDA, "upload of the residue-grid tables failed");
  }
  T.syn = T.base;
  T.ana = T.base + nsyn;
  T.tw = T.base + nsyn + nana;
  g_res[{dev, m, R}] = T;
  *out = T;
  return SFNL_OK;
}

// The R residues of one input field (batch entry blockIdx.z) at the chunk's points: thread (point, k),
// k < M/2, gathers Y_k and Y_{M-k} of each residue from the modes qM + k and qM + M - k (k = 0: Y_0 and
// Y_{M/2} from qM and qM + M/2) and writes alpha_k, beta_k (k = 0: alpha_0 and beta_{M/2}) into
// y + r * ystride, each (npc, 2, M/2): cosine k at 2k npc, sine k at (2k + 1) npc, the sine row 0 holding
// beta_{M/2}.  Cotangents (adj) take the analysis weights 1/N (n = 0), 2/N first.  The residues pair as
// d_{R-1-r} = -d_r (and d = 0 for the middle one of an odd R), so one twiddle serves two residues.
template <int R>
__global__ void large_res_coef_kernel(const double *x, int64_t ldm, int64_t xsin, int64_t xbs, double *y,
                                      int64_t ystride, int64_t npc, int m, int adj, double invN, const double *tw) {
  constexpr int RP = R / 2;  // residue pairs
  const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= npc) return;
  const int k = blockIdx.y, M = 3 * m / R, mh = M >> 1;
  const double *xp = x + (int64_t)blockIdx.z * xbs + p;
  double *yp = y + (int64_t)blockIdx.z * M * npc + p;
  double yr[2][R], yi[2][R];  // Y_k (side 0) and Y_{M-k} (side 1; k = 0: Y_{M/2}) of each residue
#pragma unroll
  for (int side = 0; side < 2; ++side)
#pragma unroll
    for (int r = 0; r < R; ++r) yr[side][r] = yi[side][r] = 0.0;
  const int khi = k == 0 ? mh : M - k;
#pragma unroll
  for (int q = 0; q < R / 3; ++q) {  // m = (R/3) M: every qM + k and qM + M - k is a mode
    const double sg = (q & 1) ? -1.0 : 1.0;
#pragma unroll
    for (int side = 0; side < 2; ++side) {
      const int n = q * M + (side ? khi : k);
      const double wn = (adj ? (n == 0 ? invN : 2.0 * invN) : 1.0) * sg;
      const double a = xp[(int64_t)n * ldm] * wn, b = xp[(int64_t)n * ldm + xsin] * wn;
      // y_n = (a - i b)(c +- i s): residue r (+s) and R-1-r (-s)
#pragma unroll
      for (int r = 0; r < RP; ++r) {
        const double2 cs = __ldg(reinterpret_cast<const double2 *>(tw) + (size_t)r * m + n);
        const double ac = a * cs.x, bs = b * cs.y, as = a * cs.y, bc = b * cs.x;
        yr[side][r] += ac + bs;
        yi[side][r] += as - bc;
        yr[side][R - 1 - r] += ac - bs;
        yi[side][R - 1 - r] -= as + bc;
      }
      if (R & 1) {
        yr[side][RP] += a;
        yi[side][RP] -= b;
      }
    }
  }
  const int64_t ic = (int64_t)(2 * k) * npc, is = (int64_t)(2 * k + 1) * npc;
#pragma unroll
  for (int r = 0; r < R; ++r) {
    double *yo = yp + (int64_t)r * ystride;
    if (k == 0) {
      yo[ic] = yr[0][r];   // alpha_0 = Re Y_0
      yo[is] = -yi[1][r];  // beta_{M/2} = -Im Y_{M/2}
    } else {
      yo[ic] = yr[0][r] - yr[1][r];     // Re (Y_k - conj Y_{M-k})
      yo[is] = -(yi[0][r] + yi[1][r]);  // -Im (Y_k - conj Y_{M-k})
    }
  }
}

// One output (batch entry blockIdx.z) from the R residues' sums S + r * rstride, each (npc, 2, M/2) with
// the sine row 0 holding S_{M/2}: thread (point, k), k < M/2, writes the modes qM + k and qM + M - k
// (k = 0: qM and qM + M/2) below m.  w = 2/N (or 1 without analysis weights), w0 = 1/N (or 1).  Paired
// residues share their twiddle as in large_res_coef_kernel.
template <int R>
__global__ void large_res_out_kernel(const double *S, int64_t rstride, double *out, int64_t ldm, int64_t osin,
                                     int64_t ops, int64_t obs, int64_t npc, int m, double w, double w0,
                                     const double *tw) {
  constexpr int RP = R / 2;
  const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= npc) return;
  const int k = blockIdx.y, M = 3 * m / R, mh = M >> 1;
  const double *sp = S + (int64_t)blockIdx.z * M * npc + p;
  double *op = out + (int64_t)blockIdx.z * obs + p * ops;
  const int64_t ic = (int64_t)(2 * k) * npc, is = (int64_t)(2 * k + 1) * npc;
  // P^r_k = C - i S; the mirror P^r_{M-k} = -conj(P^r_k) = -C - i S; k = 0: P^r_0 = C, P^r_{M/2} = -i S
  double C[R], Sv[R];
#pragma unroll
  for (int r = 0; r < R; ++r) {
    C[r] = sp[(int64_t)r * rstride + ic];
    Sv[r] = sp[(int64_t)r * rstride + is];
  }
  const int khi = k == 0 ? mh : M - k;
#pragma unroll
  for (int q = 0; q < R / 3; ++q) {
    const double sg = (q & 1) ? -1.0 : 1.0;
#pragma unroll
    for (int side = 0; side < 2; ++side) {
      const int n = q * M + (side ? khi : k);
      // P^r_n = x_r + i y_r
      auto px = [&](int r) { return k == 0 ? (side ? 0.0 : C[r]) : (side ? -C[r] : C[r]); };
      auto py = [&](int r) { return k == 0 ? (side ? -Sv[r] : 0.0) : -Sv[r]; };
      // c_n = sum_r e^{-i n d_r} P^r_n; a pair (r, R-1-r) with e^{-i n d} = c -+ i s gives
      // c (x + x') + s (y - y') + i (c (y + y') - s (x - x'))
      double re = 0.0, im = 0.0;
#pragma unroll
      for (int r = 0; r < RP; ++r) {
        const double2 cs = __ldg(reinterpret_cast<const double2 *>(tw) + (size_t)r * m + n);
        const double x0 = px(r), y0 = py(r), x1 = px(R - 1 - r), y1 = py(R - 1 - r);
        re += fma(cs.x, x0 + x1, cs.y * (y0 - y1));
        im += fma(cs.x, y0 + y1, -cs.y * (x0 - x1));
      }
      if (R & 1) {
        re += px(RP);
        im += py(RP);
      }
      const double wn = (n == 0 ? w0 : w) * sg;
      op[(int64_t)n * ldm] = wn * re;
      op[(int64_t)n * ldm + osin] = n == 0 ? 0.0 : -wn * im;
    }
  }
}

template <int R>
void launch_res_coef(dim3 grid, int threads, cudaStream_t st, const double *x, int64_t ldm, int64_t xsin,
                     int64_t xbs, double *y, int64_t ystride, int64_t npc, int m, int adj, double invN,
                     const double *tw) {
  large_res_coef_kernel<R><<<grid, threads, 0, st>>>(x, ldm, xsin, xbs, y, ystride, npc, m, adj, invN, tw);
}
template <int R>
void launch_res_out(dim3 grid, int threads, cudaStream_t st, const double *S, int64_t rstride, double *out, int64_t ldm,
                    int64_t osin, int64_t ops, int64_t obs, int64_t npc, int m, double w, double w0, const double *tw) {
  large_res_out_kernel<R><<<grid, threads, 0, st>>>(S, rstride, out, ldm, osin, ops, obs, npc, m, w, w0, tw);
}

// The two-kernel form on the residue grids: per point chunk, the R residues' coefficients of every input
// field in one pass (N/R doubles per point, field instance and residue), the residue passes of the program
// (run_large; sums into N/R doubles per point, output instance and residue), and the outputs from the R
// residues' sums in one pass.
int launch_large_res(const ProgArgs &a, const Geo &g, int R, cudaStream_t st) {
  const int m = a.m, N = g.N, M = N / R, mh = M / 2, ni = op_nin(a.op), no = op_nout(a.op);
  ResTab T;
  if (int rc = get_residue_tables(m, N, R, &T)) return rc;
  const LargePlan rp{M, M / 32, mh, T.syn, T.ana};
  int64_t inst_in = 0;
  for (int f = 0; f < ni; ++f) inst_in += a.in_bs[f] ? a.batch : 1;
  const int64_t inst_out = (int64_t)no * a.batch;
  const size_t per_point = sizeof(double) * (size_t)N * (size_t)(inst_in + inst_out);
  size_t free_b = 0, total_b = 0;
  if (cudaMemGetInfo(&free_b, &total_b) != cudaSuccess) {
    cudaGetLastError();
    free_b = 0;
  }
  size_t cap = free_b / 4;
  if (cap > (size_t(32) << 30)) cap = size_t(32) << 30;
  if (cap < (size_t(1) << 30)) cap = size_t(1) << 30;
  if (const size_t tc = g_test_cap.load()) cap = tc;
  int64_t chunk = (int64_t)(cap / per_point);
  chunk = (chunk / 32) * 32;
  if (chunk < 32) chunk = 32;
  if (chunk > a.np) chunk = ((a.np + 7) / 8) * 8;
  double *W = nullptr;
  if (int rc = large_workspace(st, per_point * (size_t)chunk, &W, 1)) return rc;
  const bool adj_out = op_adjoint_out(a.op);
  const double invN = 1.0 / N, w = adj_out ? 1.0 : 2.0 * invN, w0 = adj_out ? 1.0 : invN;
  constexpr int kThreads = 256;
  auto coef = R == 3 ? launch_res_coef<3> : R == 6 ? launch_res_coef<6> : launch_res_coef<12>;
  auto outk = R == 3 ? launch_res_out<3> : R == 6 ? launch_res_out<6> : launch_res_out<12>;
  for (int64_t c0 = 0; c0 < a.np; c0 += chunk) {
    const int64_t npc = a.np - c0 < chunk ? a.np - c0 : chunk;
    const unsigned bx = (unsigned)((npc + kThreads - 1) / kThreads);
    // residue r's arrays: inputs at W + r * rin, outputs at W + R rin + r * rout
    const int64_t rin = inst_in * M * npc, rout = inst_out * M * npc;
    ProgArgs ar = a;
    ar.np = npc;
    ar.out_ps = 1;
    int64_t off = 0;
    for (int f = 0; f < ni; ++f) {
      const int nb = a.in_bs[f] ? a.batch : 1;
      coef(dim3(bx, (unsigned)mh, (unsigned)nb), kThreads, st, a.in[f] + c0, a.in_ldm[f], a.np, a.in_bs[f], W + off, rin,
           npc, m, op_adjoint_in(a.op, f) ? 1 : 0, invN, T.tw);
      ar.in[f] = W + off;
      ar.in_ldm[f] = 2 * npc;
      ar.in_bs[f] = a.in_bs[f] ? (int64_t)M * npc : 0;
      off += (int64_t)nb * M * npc;
    }
    if (int rc = check_launch("large-m residue coefficients")) return rc;
    off = R * rin;
    for (int o = 0; o < no; ++o) {
      ar.out[o] = W + off;
      ar.out_ldm[o] = 2 * npc;
      ar.out_bs[o] = (int64_t)M * npc;
      off += (int64_t)a.batch * M * npc;
    }
    for (int r = 0; r < R; ++r) {
      ProgArgs rr = ar;
      for (int f = 0; f < ni; ++f) rr.in[f] = ar.in[f] + r * rin;
      for (int o = 0; o < no; ++o) rr.out[o] = ar.out[o] + r * rout;
      if (int rc = run_large(rr, g, Tables{}, &rp, st)) return rc;
    }
    for (int o = 0; o < no; ++o)
      outk(dim3(bx, (unsigned)mh, (unsigned)a.batch), kThreads, st, ar.out[o], rout, a.out[o] + c0 * a.out_ps,
           a.out_ldm[o], a.np * a.out_ps, a.out_ps, a.out_bs[o], npc, m, w, w0, T.tw);
    if (int rc = check_launch("large-m residue outputs")) return rc;
  }
  return SFNL_OK;
}

}  // namespace

void large_test_workspace_cap(size_t bytes) { g_test_cap.store(bytes); }

void large_test_residues(int R) { g_test_residues.store(R); }

void large_res_release_tables() {
  std::lock_guard<std::mutex> lk(g_res_mu);
  int prev = 0;
  cudaGetDevice(&prev);
  for (auto &kv : g_res) {
    cudaSetDevice(std::get<0>(kv.first));
    cudaFree(kv.second.base);
  }
  g_res.clear();
  cudaSetDevice(prev);
}

// The two-kernel form: on the grid's residue classes when the grid is 3m angles and m >= 256 (R of them:
// 3/R of the DMMAs of the whole grid, launch_large_res), else on the whole grid.
int launch_fast_large(const ProgArgs &a, const Geo &g, const Tables &T, cudaStream_t st) {
  if (const int R = large_residues(a.m, g.N)) return launch_large_res(a, g, R, st);
  return run_large(a, g, T, nullptr, st);
}

}  // namespace sfnl
