// sfnl_r3.cu -- the FAST MHD bundle at m = 64 on the 192-angle grid split into the three residue classes
// of the angle index (one radix-3 decimation-in-time step), each residue an offset 64-angle grid folded
// three times as in the 192-angle kernels.
//
// Grid theta_j = pi(2j+1)/192.  With j = 3i + r (r = 0, 1, 2; i < 64), theta_j = phi_i + d_r where
// phi_i = pi(2i+1)/64 is the offset 64-angle grid and d_r = 2 pi (r-1)/192.  A field with coefficients
// (a_n, b_n), n < 64, is x(theta) = Re sum_n z_n e^{i n theta} with z_n = a_n - i b_n, so on residue r
//   x(phi_i + d_r) = Re sum_n y_n e^{i n phi_i},   y_n = z_n e^{i n d_r},
// and because e^{i (64-k) phi_i} = -e^{-i k phi_i} the modes k and 64 - k meet in one coefficient:
//   x = sum_k alpha_k cos(k phi) + beta_k sin(k phi),   alpha_k - i beta_k = y_k - conj(y_{64-k})
// for k = 1..31, alpha_0 = a_0, and mode 32 alone with cos(32 phi_i) = 0: beta_32 = -Im y_32.  Each
// residue is a transform of 64 real coefficients (cosines 0..31, sines 1..32) to 64 angles: with the
// three folds, 24 DMMAs per field and 8-point tile, against 144 for the 192-angle transform of the 64
// modes, i.e. half the DMMAs for the three residues; the twiddles cost about 14 FP64 operations per
// (point, field, mode pair).  The analysis runs backwards: for a product p,
//   P^r_k = sum_i p(phi_i + d_r) e^{-i k phi_i} = C^r_k - i S^r_k   (C: k = 0..31, S: k = 1..32),
// P^r_{64-k} = -conj(P^r_k), and sum_j p_j e^{-i n theta_j} = P^1_n + w^n P^0_n + w^{-n} P^2_n with
// w = e^{2 pi i/192}; the output coefficients are (2/192, or 1/192 for n = 0) times its real part and
// minus its imaginary part, the grid being alias-free for the product of two fields of 64 modes
// (fft_parallel.F90:147-328 on its own grid gives the same truncated product).
//
// CTA: 8-point tiles one after the other (kR3TilesPerCta of them), 12 warps = 3 residue groups of 4 warps
// (tile tau of the 16-angle quadrant, half 0 cosine / 1 sine classes).  A group's synthesis, exchanges, products and analysis touch only its
// own shared memory and synchronise on its own named barrier; the CTA meets only where the twiddles mix
// the residues (after the coefficients arrive, and before the outputs are combined).  The DFT tables
// of a residue transform are 14 KB (L1-resident) instead of the 86 KB that streamed from L2.
#include <cuda.h>  // CUtensorMap (the encoder is reached through the runtime's driver entry point)
#include <cudaTypedefs.h>
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <map>
#include <mutex>
#include <type_traits>
#include <vector>

#include "sfnl_fold.cuh"
#include "sfnl_internal.h"
#include "sfnl_ops.cuh"

namespace sfnl {

namespace {

constexpr int kR3NT = 2;                   // angle tiles of 8 in the 16-angle quadrant of a residue grid
constexpr int kR3KS = 16;                  // synthesis k-steps of a field (64 coefficients)
constexpr int kR3RS = 3 * kR3KS * 32;      // doubles per residue: 3 fields' A fragments
constexpr int kR3PS = 4 * 4 * kR3NT * 64;  // doubles per residue: 4 product slots x 4 classes x 16 angles x 8
constexpr int kR3TilesPerCta = 4;          // tiles walked by one CTA (see fast_bundle_r3_kernel)
constexpr int kR3Smem = (3 * 128 * 8 + 3 * kR3RS + 3 * kR3PS + 128 + 2) * (int)sizeof(double);  // 109 KB
constexpr int kR3StageBytes = 3 * 128 * 8 * (int)sizeof(double);  // one operand's three staged fields

// Row groups of a residue transform: 0 CE0 (cos 4k), 1 CE2 (cos 4k+2), 2 CO (cos 2k+1), 3 SE0 (sin 4k+4,
// mode 32 included), 4 SE2 (sin 4k+2), 5 SO (sin 2k+1).  The third fold needs the even groups split by
// n mod 4, which mode 32 (n = 0 mod 4) follows like the others.
__host__ __device__ constexpr int r3_ke(int gr) { return gr % 3 == 2 ? 16 : 8; }
__host__ __device__ constexpr int r3_KS(int gr) { return r3_ke(gr) / 4; }
__host__ __device__ constexpr int r3_koff(int gr) { return gr == 0 ? 0 : r3_koff(gr - 1) + r3_KS(gr - 1); }
__host__ __device__ constexpr int r3_mode(int gr, int k) {
  return gr == 3 ? 4 * k + 4 : gr % 3 == 0 ? 4 * k : gr % 3 == 1 ? 4 * k + 2 : 2 * k + 1;
}
// analysis: one output tile of 8 modes per even group (k-steps over half the quadrant with the mirror),
// two per odd group (k-steps over the whole quadrant)
__host__ __device__ constexpr int r3_NU(int gr) { return gr % 3 == 2 ? 2 : 1; }
__host__ __device__ constexpr int r3_TE(int gr) { return gr % 3 == 2 ? 2 * kR3NT : kR3NT; }
__host__ __device__ constexpr int r3_aoff(int gr) {
  return gr == 0 ? 0 : r3_aoff(gr - 1) + r3_NU(gr - 1) * r3_TE(gr - 1);
}
static_assert(r3_koff(6) == kR3KS && r3_aoff(6) == 24, "residue transform geometry");

// Row (4 * k-step + k-value) of cosine mode k (0..31) and of sine mode k (1..32) in a field's A fragments.
__device__ __forceinline__ int r3_cos_row(int k) {
  return (k & 1) ? 4 * r3_koff(2) + (k >> 1) : (k & 2) ? 4 * r3_koff(1) + (k >> 2) : (k >> 2);
}
__device__ __forceinline__ int r3_sin_row(int k) {
  return (k & 1) ? 4 * r3_koff(5) + (k >> 1) : (k & 2) ? 4 * r3_koff(4) + (k >> 2) : 4 * r3_koff(3) + (k >> 2) - 1;
}

// Shared-memory orders chosen so that every warp access below is conflict-free (each quarter-warp's eight
// 16-byte accesses, or each half-warp's sixteen 8-byte ones, on distinct banks): the staged row of mode n
// (r3_stage / the bulk tensor copies, r3_precombine) and the row and point swizzle of slot s of the
// analysed sums (cos mode k at slot k, sine mode k at 32 + k % 32; r3_analysis writes them, r3_combine
// reads them).  The staged row moves bit 2 of the mode to the bottom, (n >> 3, n & 3, (n >> 2) & 1), an
// order a five-dimensional tensor map copies directly (one dimension per group of mode bits), so that the
// 64-byte rows that one quarter-warp of r3_precombine reads (modes k = 4i and 4i + 4, 4i + 2 and 4i + 6, or
// odd modes paired with bit 1 of their task flipped) sit on opposite halves of the banks.
__host__ __device__ __forceinline__ int r3_trow(int n) { return ((n >> 3) << 3) | ((n & 3) << 1) | ((n >> 2) & 1); }
__device__ __forceinline__ int r3_rpos(int s, int p) { return (s ^ (((s >> 2) ^ (s >> 4)) & 1)) * 8 + (p ^ (((s >> 3) & 1) << 2)); }

struct R3Tables {
  double *base = nullptr;  // syn [16 k-steps][2 tiles][32], ana [24 k-steps][32], tw [64][2]
  const double *syn() const { return base; }
  const double *ana() const { return base + kR3KS * kR3NT * 32; }
  const double *tw() const { return base + kR3KS * kR3NT * 32 + 24 * 32; }
};
constexpr size_t kR3TabDoubles = (size_t)kR3KS * kR3NT * 32 + 24 * 32 + 128;

std::mutex g_r3_mu;
std::map<int, R3Tables> g_r3_tabs;  // device -> tables

// Synthesis B fragments: lane (g, q) of k-step s of group gr on tile t holds mode r3_mode(gr, 4s + q) at
// angle phi_{8t + g}.  Analysis B fragments (no weights): lane (g, q) of k-step te of output tile u holds
// mode r3_mode(gr, 8u + g) at angle phi_{8 (te / 2) + 2q + te % 2}.  Twiddles: cos, sin of 2 pi n / 192.
int get_r3_tables(R3Tables *out) {
  int dev = 0;
  cudaGetDevice(&dev);
  std::lock_guard<std::mutex> lk(g_r3_mu);
  auto it = g_r3_tabs.find(dev);
  if (it != g_r3_tabs.end()) {
    *out = it->second;
    return SFNL_OK;
  }
  const long double pi = acosl(-1.0L), dphi = pi / 64.0L;  // phi_j = (2j + 1) dphi
  std::vector<double> h(kR3TabDoubles, 0.0);
  for (int gr = 0; gr < 6; ++gr)
    for (int s = 0; s < r3_KS(gr); ++s)
      for (int t = 0; t < kR3NT; ++t)
        for (int l = 0; l < 32; ++l) {
          const long double x = (long double)r3_mode(gr, 4 * s + (l & 3)) * (2 * (8 * t + (l >> 2)) + 1) * dphi;
          h[((size_t)(r3_koff(gr) + s) * kR3NT + t) * 32 + l] = (double)(gr < 3 ? cosl(x) : sinl(x));
        }
  double *ana = h.data() + kR3KS * kR3NT * 32;
  for (int gr = 0; gr < 6; ++gr)
    for (int u = 0; u < r3_NU(gr); ++u)
      for (int te = 0; te < r3_TE(gr); ++te)
        for (int l = 0; l < 32; ++l) {
          const int j = 8 * (te >> 1) + 2 * (l & 3) + (te & 1);
          const long double x = (long double)r3_mode(gr, 8 * u + (l >> 2)) * (2 * j + 1) * dphi;
          ana[((size_t)r3_aoff(gr) + u * r3_TE(gr) + te) * 32 + l] = (double)(gr < 3 ? cosl(x) : sinl(x));
        }
  double *tw = ana + 24 * 32;
  for (int n = 0; n < 64; ++n) {
    tw[2 * n] = (double)cosl(2.0L * pi * n / 192.0L);
    tw[2 * n + 1] = (double)sinl(2.0L * pi * n / 192.0L);
  }
  R3Tables T;
  if (cudaMalloc(&T.base, h.size() * sizeof(double)) != cudaSuccess) {
    cudaGetLastError();
    return set_error(SFNL_ERR_ALLOC, "cudaMalloc of the residue-split DFT tables failed");
  }
  if (cudaMemcpy(T.base, h.data(), h.size() * sizeof(double), cudaMemcpyHostToDevice) != cudaSuccess) {
    cudaFree(T.base);
    return set_error(SFNL_ERR_CUDA, "upload of the residue-split DFT tables failed");
  }
  g_r3_tabs[dev] = T;
  *out = T;
  return SFNL_OK;
}

struct R3Fields {  // three fields: cos of mode n, point p at p[f][p + n*ldm[f]], sine np further
  const double *p[3];
  int64_t ldm[3];
};

// Bulk tensor copies of the staged fields: one tensor map per input field over (point, bit 2 of the mode,
// mode & 3, mode >> 3, cos/sin) with the box (8, 2, 4, 8, 2) lands an 8-point tile in xr's row order
// (r3_trow) in one copy; a single thread issues an operand's three copies on the stage barrier, whose
// transaction count is the 24 KB they write (points past np arrive as zeros).  No multicast: each CTA
// fetches its own tile.
__device__ __forceinline__ uint32_t r3_smem_addr(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void r3_bar_init(uint64_t *bar) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(r3_smem_addr(bar)) : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// Issued by one thread after a CTA barrier that ends every read of xr.
__device__ __forceinline__ void r3_bulk_stage(double *xr, const CUtensorMap *const (&maps)[3], int64_t p0,
                                              uint64_t *bar) {
  const uint32_t b = r3_smem_addr(bar);
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");  // the generic reads of xr before the copies
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(b), "r"(kR3StageBytes) : "memory");
  const int x = (int)p0;
#pragma unroll
  for (int f = 0; f < 3; ++f)
    asm volatile(
        "cp.async.bulk.tensor.5d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %3, %3, %3}], [%4];"
        ::"r"(r3_smem_addr(xr + (size_t)f * 128 * 8)), "l"(reinterpret_cast<uint64_t>(maps[f])), "r"(x), "r"(0), "r"(b)
        : "memory");
}

// Bounded wait for phase `parity` of the stage barrier; false if it gave up (the copies never landed).
__device__ __forceinline__ bool r3_bar_wait(uint64_t *bar, uint32_t parity) {
  const uint32_t b = r3_smem_addr(bar);
  for (int it = 0; it < (1 << 22); ++it) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(done)
        : "r"(b), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
}

// Stages the three fields of the 8-point tile at p0 into xr [3][128 rows: cos, then sin, of mode n at row
// r3_trow(n)][8 points] with cp.async and commits one group (the sine of mode 0 is not read: zero); the
// form for inputs that the bulk tensor copies cannot take (odd np, unaligned bases or odd mode strides).
// 384 threads: thread t copies 16 bytes (points pc, pc + 1) of modes rb, rb + 32 (cosines and sines) of
// field t / 128, so that four consecutive threads move one whole 64-byte row and every address derives
// from two bases by constant offsets; rb swaps bits 0 and 2 of (t % 128) / 4, so that a quarter-warp's two
// rows sit on opposite bank halves.
__device__ __forceinline__ void r3_stage(double *xr, const R3Fields &fs, int64_t p0, int64_t np, bool vec16) {
  const int t = threadIdx.x, f = t >> 7, pc = 2 * (t & 3), j = (t & 127) >> 2;
  const int rb = (j & ~5) | ((j & 1) << 2) | ((j >> 2) & 1);
  const double *base = f == 0 ? fs.p[0] : f == 1 ? fs.p[1] : fs.p[2];
  const int64_t ldm = f == 0 ? fs.ldm[0] : f == 1 ? fs.ldm[1] : fs.ldm[2];
  const double *src = base + p0 + pc + (int64_t)rb * ldm;        // cosine row rb; rb + 32 at 32 ldm, sines np on
  double *dst = xr + ((size_t)f * 128 + r3_trow(rb)) * 8 + pc;  // r3_trow(rb + 32) = r3_trow(rb) + 32
  const bool v16 = vec16 && p0 + 8 <= np, pv0 = p0 + pc < np, pv1 = p0 + pc + 1 < np;
  // a rolled loop: the four copies' addresses at once would cost registers the synthesis needs
#pragma unroll 1
  for (int i = 0; i < 4; ++i) {
    const double *s_i = src + ((i & 1) ? 32 * ldm : 0) + ((i & 2) ? np : 0);
    double *d_i = dst + (i & 1) * 256 + (i & 2) * 256;
    const bool live = !(i == 2 && rb == 0);  // the sine of mode 0
    if (live && v16) {
      cp_async16(d_i, s_i);
    } else {
      if (live && pv0) cp_async8(d_i, s_i); else d_i[0] = 0.0;
      if (live && pv1) cp_async8(d_i + 1, s_i + 1); else d_i[1] = 0.0;
    }
  }
  cp_async_commit();
}

// The residues' coefficients of the three staged fields: thread t forms alpha^r_k, beta^r_k of the three
// residues at two adjacent points from modes k and 64 - k (k = 0 also does mode 32) and writes them into
// xs [r][f][16][32]; its task (field, cosine row rc, point pair) makes a warp the 4 rows of 2 A-fragment
// blocks.  tws: cos, sin of 2 pi n / 192 in shared memory.
__device__ __forceinline__ void r3_precombine(const double *xr, double *xs, const double *tws) {
  const int t = threadIdx.x;
  // task rc: even modes (rc < 16) in order, odd ones with bit 1 flipped on odd slots, so that the two tasks
  // of a quarter-warp differ in the parity of rc (their A-fragment stores) and in bit 2 of their modes
  // (their staged rows)
  const int p = 2 * (t & 3), j = (t >> 2) & 31, f = t >> 7;
  const int rc = j < 16 ? j : 16 + ((j - 16) ^ ((j & 1) << 1));
  const int k = rc < 8 ? 4 * rc : rc < 16 ? 4 * (rc - 8) + 2 : 2 * (rc - 16) + 1;  // cosine mode of row rc
  const double *x = xr + (size_t)f * 128 * 8 + p;
  auto cosv = [&](int n) { return *reinterpret_cast<const double2 *>(x + r3_trow(n) * 8); };
  auto sinv = [&](int n) { return *reinterpret_cast<const double2 *>(x + (64 + r3_trow(n)) * 8); };
  double2 al[3], be[3];
  int rs;
  if (k == 0) {
    const double2 a0 = cosv(0), a32 = cosv(32), b32 = sinv(32);
    const double2 cs = *reinterpret_cast<const double2 *>(tws + 64);  // d_r = -+ 2 pi/192: 32 d_r = -+ pi/3
    al[0] = al[1] = al[2] = a0;
    be[1] = b32;
    be[0] = make_double2(fma(a32.x, cs.y, b32.x * cs.x), fma(a32.y, cs.y, b32.y * cs.x));
    be[2] = make_double2(fma(-a32.x, cs.y, b32.x * cs.x), fma(-a32.y, cs.y, b32.y * cs.x));
    rs = r3_sin_row(32);
  } else {
    const int k2 = 64 - k;
    const double2 a = cosv(k), b = sinv(k), a2 = cosv(k2), b2 = sinv(k2);
    const double2 cs = *reinterpret_cast<const double2 *>(tws + 2 * k), cs2 = *reinterpret_cast<const double2 *>(tws + 2 * k2);
    // X = a c - a' c', Y = b s - b' s', Z = b c + b' c', W = a s + a' s' at each of the two points
    const double2 X = make_double2(fma(a.x, cs.x, -a2.x * cs2.x), fma(a.y, cs.x, -a2.y * cs2.x));
    const double2 Y = make_double2(fma(b.x, cs.y, -b2.x * cs2.y), fma(b.y, cs.y, -b2.y * cs2.y));
    const double2 Z = make_double2(fma(b.x, cs.x, b2.x * cs2.x), fma(b.y, cs.x, b2.y * cs2.x));
    const double2 W = make_double2(fma(a.x, cs.y, a2.x * cs2.y), fma(a.y, cs.y, a2.y * cs2.y));
    al[1] = make_double2(a.x - a2.x, a.y - a2.y);  // r = 1: d = 0
    be[1] = make_double2(b.x + b2.x, b.y + b2.y);
    al[0] = make_double2(X.x - Y.x, X.y - Y.y);    // r = 0: e^{-i n 2 pi/192}
    be[0] = make_double2(Z.x + W.x, Z.y + W.y);
    al[2] = make_double2(X.x + Y.x, X.y + Y.y);    // r = 2: e^{+i n 2 pi/192}
    be[2] = make_double2(Z.x - W.x, Z.y - W.y);
    rs = r3_sin_row(k);
  }
  double *d = xs + (size_t)f * kR3KS * 32;
  const int oc = (rc >> 2) * 32 + a_frag_slot(rc & 3, p), os = (rs >> 2) * 32 + a_frag_slot(rs & 3, p);
#pragma unroll
  for (int r = 0; r < 3; ++r) {
    *reinterpret_cast<double2 *>(d + (size_t)r * kR3RS + oc) = al[r];
    *reinterpret_cast<double2 *>(d + (size_t)r * kR3RS + os) = be[r];
  }
}

// Synthesis of the group's residue for the three fields: warp (tau, half) accumulates the odd class of
// half `half` on tile tau and the even part E0 (tau 0) or E2 (tau 1) on tile 0 (fold_exchange assembles
// both tiles of the even class from them).
__device__ __forceinline__ void r3_synth(const double *xs_r, const double *syn, int tau, int half,
                                         double (&acc_e)[3][2], double (&acc_o)[3][2]) {
  const int lane = threadIdx.x & 31;
  const int ke = r3_koff(3 * half + tau), ko = r3_koff(3 * half + 2);
  // k-step s < 2: even part on tile 0; s >= 2: odd class on tile tau.  The next k-step's B fragment is
  // loaded while the current one feeds the DMMAs.
  auto bfrag = [&](int s) {
    return __ldg(syn + (s < 2 ? (size_t)(ke + s) * kR3NT : (size_t)(ko + s - 2) * kR3NT + tau) * 32 + lane);
  };
#pragma unroll
  for (int f = 0; f < 3; ++f) acc_e[f][0] = acc_e[f][1] = acc_o[f][0] = acc_o[f][1] = 0.0;
  const double *xa = xs_r + a_frag_slot(lane & 3, lane >> 2);
  double bnext = bfrag(0);
#pragma unroll
  for (int s = 0; s < 6; ++s) {
    const double bv = bnext;
    if (s + 1 < 6) bnext = bfrag(s + 1);
    const int ks = s < 2 ? ke + s : ko + s - 2;
#pragma unroll
    for (int f = 0; f < 3; ++f) {
      if (s < 2)
        dmma(acc_e[f], xa[((size_t)f * kR3KS + ks) * 32], bv);
      else
        dmma(acc_o[f], xa[((size_t)f * kR3KS + ks) * 32], bv);
    }
  }
}

// Analysis of the group's NO product slots (ps_r [slot][class][2][2][32]): warp wg takes one odd output
// tile (CO 0-7, CO 8-15, SO 0-7, SO 8-15 for wg = 0..3) and one even one (CE0, CE2, SE0, SE2) and writes
// the sums of outputs 0-2 into R_lo [o][64 slots x 8 points] (r3_rpos) and those of output 3 into R_hi
// (over the product slots, after a barrier of the group).
template <int NO, typename Sync>
__device__ __forceinline__ void r3_analysis(const double *ps_r, const double *ana, int wg, double *R_lo, double *R_hi,
                                            Sync sync) {
  static_assert(NO <= 4, "at most four product slots");
  const int lane = threadIdx.x & 31, g = lane >> 2, q = lane & 3;
  const int go = wg < 2 ? 2 : 5, uo = wg & 1;
  const int ge = wg < 2 ? wg : wg + 1;
  const int co = go == 2 ? 1 : 3, ce = ge < 3 ? 0 : 2;  // classes PO / QO and PE / QE
  const double sg = (ge == 0 || ge == 4) ? 1.0 : -1.0;   // mirror sign: PE0 +, PE2 -, QE0 -, QE2 +
  double yo[NO][2], ye[NO][2];
#pragma unroll
  for (int o = 0; o < NO; ++o) yo[o][0] = yo[o][1] = ye[o][0] = ye[o][1] = 0.0;
  const double *bo = ana + ((size_t)r3_aoff(go) + uo * r3_TE(go)) * 32 + lane;
  const double *be = ana + (size_t)r3_aoff(ge) * 32 + lane;
#pragma unroll
  for (int te = 0; te < 2 * kR3NT; ++te) {
    const double bv = __ldg(bo + (size_t)te * 32);
    const int t = te >> 1, e = te & 1;
#pragma unroll
    for (int o = 0; o < NO; ++o) dmma(yo[o], ps_r[((((size_t)o * 4 + co) * kR3NT + t) * 2 + e) * 32 + lane], bv);
  }
#pragma unroll
  for (int te = 0; te < kR3NT; ++te) {
    const double bv = __ldg(be + (size_t)te * 32);
    const int t = te >> 1, e = te & 1;
#pragma unroll
    for (int o = 0; o < NO; ++o) {
      const double *pc = ps_r + ((size_t)o * 4 + ce) * kR3NT * 2 * 32;
      const double av = pc[(t * 2 + e) * 32 + lane] + sg * pc[((kR3NT - 1 - t) * 2 + 1 - e) * 32 + (lane ^ 3)];
      dmma(ye[o], av, bv);
    }
  }
#pragma unroll
  for (int h = 0; h < 2; ++h) {
    const int no = r3_mode(go, 8 * uo + 2 * q + h), ne = r3_mode(ge, 2 * q + h);
    const int po = r3_rpos(go < 3 ? no : 32 + (no & 31), g), pe = r3_rpos(ge < 3 ? ne : 32 + (ne & 31), g);
#pragma unroll
    for (int o = 0; o < (NO < 3 ? NO : 3); ++o) {
      R_lo[(size_t)o * 512 + po] = yo[o][h];
      R_lo[(size_t)o * 512 + pe] = ye[o][h];
    }
  }
  if constexpr (NO == 4) {
    sync();  // the group has read its product slots: the fourth output's sums overlay them
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const int no = r3_mode(go, 8 * uo + 2 * q + h), ne = r3_mode(ge, 2 * q + h);
      R_hi[r3_rpos(go < 3 ? no : 32 + (no & 31), g)] = yo[3][h];
      R_hi[r3_rpos(ge < 3 ? ne : 32 + (ne & 31), g)] = ye[3][h];
    }
  }
}

struct R3Outs {
  double *p[3];
  int64_t ldm[3];
};

// The output coefficients from the three residues' sums (R: residue r at R + r * rstride): thread t < 128 NO
// writes modes k and 64 - k (k = 0 also mode 32) of output t / 128 at two adjacent points, with 16-byte
// stores when v16 (output bases 16-byte aligned, even mode stride and np).
template <int NO>
__device__ __forceinline__ void r3_combine(const double *R, int rstride, const double *tws, const R3Outs &os, int64_t p0,
                                           int64_t np, bool v16) {
  const int t = threadIdx.x;
  if (t >= NO * 128) return;
  const int p = 2 * (t & 3), k = (t >> 2) & 31, o = t >> 7;
  const int64_t pp = p0 + p;
  if (pp >= np) return;
  const bool two = pp + 1 < np;
  const double w = 2.0 / 192.0;
  const double *Ro = R + (size_t)o * 512;
  auto rv = [&](int r, int slot) { return *reinterpret_cast<const double2 *>(Ro + (size_t)r * rstride + r3_rpos(slot, p)); };
  double *dst = (o == 0 ? os.p[0] : o == 1 ? os.p[1] : os.p[2]) + pp;
  const int64_t ldm = o == 0 ? os.ldm[0] : o == 1 ? os.ldm[1] : os.ldm[2];
  auto put = [&](int64_t off, double v0, double v1) {
    if (v16 && two) {
      *reinterpret_cast<double2 *>(dst + off) = make_double2(v0, v1);
    } else {
      dst[off] = v0;
      if (two) dst[off + 1] = v1;
    }
  };
  if (k == 0) {
    const double2 S0 = rv(0, 32), S1 = rv(1, 32), S2 = rv(2, 32);  // sine of mode 32
    const double2 C0 = rv(0, 0), C1 = rv(1, 0), C2 = rv(2, 0);
    const double2 cs = *reinterpret_cast<const double2 *>(tws + 64);
    put(0, (C0.x + C1.x + C2.x) * (1.0 / 192.0), (C0.y + C1.y + C2.y) * (1.0 / 192.0));
    put(np, 0.0, 0.0);
    put(32 * ldm, w * (cs.y * (S0.x - S2.x)), w * (cs.y * (S0.y - S2.y)));
    put(32 * ldm + np, w * fma(cs.x, S0.x + S2.x, S1.x), w * fma(cs.x, S0.y + S2.y, S1.y));
  } else {
    const double2 C0 = rv(0, k), C1 = rv(1, k), C2 = rv(2, k);
    const double2 S0 = rv(0, 32 + k), S1 = rv(1, 32 + k), S2 = rv(2, 32 + k);
    const int k2 = 64 - k;
    const double2 cs = *reinterpret_cast<const double2 *>(tws + 2 * k), cs2 = *reinterpret_cast<const double2 *>(tws + 2 * k2);
    double A[2], B[2], A2[2], B2[2];
    auto one = [&](double c0, double c1, double c2, double s0, double s1, double s2, int h) {
      const double CS = c0 + c2, CD = c0 - c2, SS = s0 + s2, SD = s0 - s2;
      A[h] = w * fma(cs.y, SD, fma(cs.x, CS, c1));
      B[h] = w * fma(-cs.y, CD, fma(cs.x, SS, s1));
      A2[h] = w * fma(cs2.y, SD, fma(-cs2.x, CS, -c1));
      B2[h] = w * fma(cs2.y, CD, fma(cs2.x, SS, s1));
    };
    one(C0.x, C1.x, C2.x, S0.x, S1.x, S2.x, 0);
    one(C0.y, C1.y, C2.y, S0.y, S1.y, S2.y, 1);
    put(k * ldm, A[0], A[1]);
    put(k * ldm + np, B[0], B[1]);
    put(k2 * ldm, A2[0], A2[1]);
    put(k2 * ldm + np, B2[0], B2[1]);
  }
}

struct R3BundleArgs {
  CUtensorMap tm[15];    // bulk-copy maps of the inputs (the kTma kernel)
  const double *in[15];  // u 0-2, w 3-5, b 6-8, j 9-11, gradT 12-14
  double *out[10];       // u x w 0-2, u x b 3-5, j x b 6-8, u . gradT 9
  int64_t in_ldm[15], out_ldm[10];
  int64_t np;
  int vec16;     // inputs: bases 16-byte aligned, even mode strides and np
  int vec16out;  // outputs: the same
  const double *syn, *ana, *tw;
  int *status;  // the mapped wait-status word (set if a bounded wait on the bulk copies gave up)
};

// The MHD bundle (u x w, u x b, j x b, u . gradT) on the residue grids, one CTA per 8-point tile (CTAs that
// start as others end keep the two CTAs of an SM out of step, so that one's DMMA phases overlap the
// other's shared-memory phases; persistent CTAs walking the tiles ran in step and were 9 % slower): the
// five vector operands are staged and transformed one after the other (u, w, gradT, b, j; each one's
// copies issued as soon as the previous one's coefficients are combined), u's and b's grid values stay in
// registers while their partners are transformed, and the products are analysed in three rounds (u x w
// with u . gradT; u x b; j x b).  kTma: the operands arrive by bulk tensor copies (r3_bulk_stage) on the
// stage barrier, else by every thread's cp.async (r3_stage).
template <bool kTma>
__global__ void __launch_bounds__(384, 2) fast_bundle_r3_kernel(const __grid_constant__ R3BundleArgs a) {
  extern __shared__ __align__(128) double smem[];
  double *xr = smem;                  // staged coefficients of one operand
  double *xs = xr + 3 * 128 * 8;      // per residue: A fragments, then the exchanges, then the analysed sums
  double *ps = xs + 3 * kR3RS;        // per residue: folded products (then the fourth output's sums)
  double *tws = ps + 3 * kR3PS;       // twiddles cos, sin of 2 pi n / 192
  uint64_t *sbar = reinterpret_cast<uint64_t *>(tws + 128);  // stage barrier (kTma)
  if (threadIdx.x < 128) tws[threadIdx.x] = __ldg(a.tw + threadIdx.x);
  if constexpr (kTma) {
    if (threadIdx.x == 0) r3_bar_init(sbar);
    __syncthreads();
  }
  uint32_t phase = 0;     // parity of the stage barrier's next phase
  bool gave_up = false;   // a bounded wait on the copies ran out
  const int warp = threadIdx.x >> 5, r = warp >> 2, wg = warp & 3, tau = wg >> 1, half = wg & 1;
  double *xs_r = xs + (size_t)r * kR3RS, *ps_r = ps + (size_t)r * kR3PS;
  const GroupSync gsync{r};
  const bool v16o = a.vec16out != 0;
  auto fields = [&](int first) {
    R3Fields fs;
#pragma unroll
    for (int f = 0; f < 3; ++f) {
      fs.p[f] = a.in[first + f];
      fs.ldm[f] = a.in_ldm[first + f];
    }
    return fs;
  };
  auto outs = [&](int first, int n) {
    R3Outs os;
#pragma unroll
    for (int o = 0; o < 3; ++o) {
      os.p[o] = a.out[first + (o < n ? o : 0)];
      os.ldm[o] = a.out_ldm[first + (o < n ? o : 0)];
    }
    return os;
  };
  // the copies of the operand whose fields start at a.in[NEXT] for the tile at p0
  auto stage = [&](auto tag, int64_t p0) {
    constexpr int NEXT = decltype(tag)::value;
    if constexpr (kTma) {
      if (threadIdx.x == 0) {
        const CUtensorMap *const mp[3] = {&a.tm[NEXT], &a.tm[NEXT + 1], &a.tm[NEXT + 2]};
        r3_bulk_stage(xr, mp, p0, sbar);
      }
    } else {
      r3_stage(xr, fields(NEXT), p0, a.np, a.vec16 != 0);
    }
  };
  // one operand: wait for its copies, form the residues' coefficients, issue the copies of the operand whose
  // fields start at a.in[NEXT] (a compile-time index, so that the kernel parameters are read at fixed offsets)
  // at point next_p0 when stage_next, synthesise the group's residue, fold
  auto operand = [&](auto next_tag, bool stage_next, int64_t next_p0, double (&v)[4][3]) {
    if constexpr (kTma) {
      if (!r3_bar_wait(sbar, phase)) gave_up = true;
      phase ^= 1;
    } else {
      cp_async_wait_0();
    }
    __syncthreads();  // the copies have landed; the previous round's sums are read
    r3_precombine(xr, xs, tws);
    __syncthreads();  // xs complete, xr read
    if (stage_next) stage(next_tag, next_p0);
    double acc_e[3][2], acc_o[3][2];
    r3_synth(xs_r, a.syn, tau, half, acc_e, acc_o);
    gsync();  // the group has read its A fragments: the exchanges overlay them
    fold_exchange<kR3NT, 3>(acc_e, acc_o, xs_r, tau, half, gsync, v);
  };
  const int64_t ntiles = (a.np + 7) / 8;
  int64_t tile = blockIdx.x;
  if (tile < ntiles) stage(std::integral_constant<int, 0>{}, tile * 8);  // u of the first tile
  for (; tile < ntiles; tile += gridDim.x) {
    const int64_t p0 = tile * 8;
    const bool more = tile + gridDim.x < ntiles;
    double vu[4][3], vb[4][3], vx[4][3];
    operand(std::integral_constant<int, 3>{}, true, p0, vu);    // u; next w
    operand(std::integral_constant<int, 12>{}, true, p0, vx);   // w; next gradT
    {
      double gq[4][3];
#pragma unroll
      for (int q = 0; q < 4; ++q) cross3(vu[q], vx[q], gq[q]);
      prefold_store<kR3NT, 3>(gq, ps_r, 0, tau, half);
    }
    operand(std::integral_constant<int, 6>{}, true, p0, vx);  // gradT; next b
    {
      double gq[4][1];
#pragma unroll
      for (int q = 0; q < 4; ++q) gq[q][0] = vu[q][0] * vx[q][0] + vu[q][1] * vx[q][1] + vu[q][2] * vx[q][2];
      prefold_store<kR3NT, 1>(gq, ps_r, 3, tau, half);
      gsync();
      r3_analysis<4>(ps_r, a.ana, wg, xs_r, ps_r, gsync);
      __syncthreads();
      r3_combine<3>(xs, kR3RS, tws, outs(0, 3), p0, a.np, v16o);  // u x w
      r3_combine<1>(ps, kR3PS, tws, outs(9, 1), p0, a.np, v16o);  // u . gradT
    }
    operand(std::integral_constant<int, 9>{}, true, p0, vb);  // b; next j
    {
      double gq[4][3];
#pragma unroll
      for (int q = 0; q < 4; ++q) cross3(vu[q], vb[q], gq[q]);
      prefold_store<kR3NT, 3>(gq, ps_r, 0, tau, half);
      gsync();
      r3_analysis<3>(ps_r, a.ana, wg, xs_r, ps_r, gsync);
      __syncthreads();
      r3_combine<3>(xs, kR3RS, tws, outs(3, 3), p0, a.np, v16o);  // u x b
    }
    operand(std::integral_constant<int, 0>{}, more, p0 + 8 * (int64_t)gridDim.x, vx);  // j; next the next tile's u
    {
      double gq[4][3];
#pragma unroll
      for (int q = 0; q < 4; ++q) cross3(vx[q], vb[q], gq[q]);
      prefold_store<kR3NT, 3>(gq, ps_r, 0, tau, half);
      gsync();
      r3_analysis<3>(ps_r, a.ana, wg, xs_r, ps_r, gsync);
      __syncthreads();
      r3_combine<3>(xs, kR3RS, tws, outs(6, 3), p0, a.np, v16o);  // j x b
    }
  }
  if (kTma && gave_up) {
    // the call's outputs are incomplete: say so, and give a copy still in flight one more bounded wait
    // before the CTA's shared memory is released
    if (a.status) {
      *reinterpret_cast<volatile int *>(a.status) = 1;
      __threadfence_system();
    }
    r3_bar_wait(sbar, phase ^ 1);
  }
}

}  // namespace

// cuTensorMapEncodeTiled through the runtime (the library links no driver library); null if absent.
static PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
  static std::once_flag once;
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  std::call_once(once, [] {
    void *p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &p, 12000, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    else
      cudaGetLastError();
  });
  return fn;
}

// The bulk-copy map of one input field (cos of mode n, point p at base[p + n ldm], sine np further): dims
// (point, bit 2 of n, n & 3, n >> 3, cos/sin), box (8, 2, 4, 8, 2).  Needs a 16-byte aligned base and even
// ldm and np (strides in multiples of 16 bytes), which the caller has checked.
static bool encode_field_map(PFN_cuTensorMapEncodeTiled_v12000 enc, CUtensorMap *map, const double *base, int64_t ldm,
                      int64_t np) {
  const cuuint64_t dims[5] = {(cuuint64_t)np, 2, 4, 8, 2};
  const cuuint64_t strides[4] = {(cuuint64_t)(4 * ldm * 8), (cuuint64_t)(ldm * 8), (cuuint64_t)(8 * ldm * 8),
                                 (cuuint64_t)(np * 8)};
  const cuuint32_t box[5] = {8, 2, 4, 8, 2}, estr[5] = {1, 1, 1, 1, 1};
  return enc(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 5, const_cast<double *>(base), dims, strides, box, estr,
             CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_NONE,
             CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

int launch_bundle_r3(const ProgArgs &a, cudaStream_t st) {
  R3BundleArgs ba;
  std::memset(&ba, 0, sizeof(ba));
  int v16 = (a.np & 1) ? 0 : 1;
  for (int f = 0; f < 15; ++f) {
    ba.in[f] = a.in[f];
    ba.in_ldm[f] = a.in_ldm[f];
    if ((reinterpret_cast<uintptr_t>(a.in[f]) & 15) || (a.in_ldm[f] & 1)) v16 = 0;
  }
  int v16o = (a.np & 1) ? 0 : 1;
  for (int o = 0; o < 10; ++o) {
    ba.out[o] = a.out[o];
    ba.out_ldm[o] = a.out_ldm[o];
    if ((reinterpret_cast<uintptr_t>(a.out[o]) & 15) || (a.out_ldm[o] & 1)) v16o = 0;
  }
  ba.np = a.np;
  ba.vec16 = v16;
  ba.vec16out = v16o;
  R3Tables T;
  if (int rc = get_r3_tables(&T)) return rc;
  ba.syn = T.syn();
  ba.ana = T.ana();
  ba.tw = T.tw();
  // bulk tensor copies where every field's strides allow them (tile coordinates are 32-bit)
  bool tma = v16 && a.np < ((int64_t)1 << 31);
  PFN_cuTensorMapEncodeTiled_v12000 enc = tma ? tensor_map_encoder() : nullptr;
  for (int f = 0; f < 15 && tma; ++f) tma = enc && encode_field_map(enc, &ba.tm[f], a.in[f], a.in_ldm[f], a.np);
  if (tma)
    if (int rc = wait_status_word(&ba.status)) return rc;
  auto kern = tma ? fast_bundle_r3_kernel<true> : fast_bundle_r3_kernel<false>;
  if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, kR3Smem) != cudaSuccess)
    return set_error(SFNL_ERR_CUDA, "cudaFuncSetAttribute failed (residue-split bundle)");
  const int64_t tiles = (a.np + 7) / 8, ctas = (tiles + kR3TilesPerCta - 1) / kR3TilesPerCta;
  if (ctas > 0x7fffffff) return set_error(SFNL_ERR_UNSUPPORTED, "np too large");
  kern<<<(unsigned)ctas, 384, kR3Smem, st>>>(ba);
  return check_launch("fast form (residue-split bundle)");
}

void r3_release_tables() {
  std::lock_guard<std::mutex> lk(g_r3_mu);
  int prev = 0;
  cudaGetDevice(&prev);
  for (auto &kv : g_r3_tabs) {
    cudaSetDevice(kv.first);
    cudaFree(kv.second.base);
  }
  g_r3_tabs.clear();
  cudaSetDevice(prev);
}

}  // namespace sfnl
