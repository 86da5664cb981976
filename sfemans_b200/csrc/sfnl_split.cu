// sfnl_split.cu -- split-precision products on the tcgen05 tensor cores.
//
// Same mathematics as the FAST form (sfnl_fast.cu): the exact truncated
// product of fft_parallel.F90:147-665, :1021-1220 (pb = 1) and :1543-1796
// (without opt_tension) evaluated on an internal alias-free
// grid, N = 4Q angles theta_j = pi(2j+1)/N with Q a multiple of 16, the two
// real-FFT symmetry levels folded out so that each field needs four small
// class contractions (cos/sin x even/odd modes) each way.  Here those
// contractions run on the 5th-generation tensor cores in bf16 with FP32
// accumulation in tensor memory, and FP64 is used for the recombination of
// the partial products, the folds, the pointwise program and the final
// truncation.
//
// Slicing.  Every row of an operand (one field of one point for one class,
// or one folded product row of one 16-angle chunk) is cut into 3 bf16
// fixed-point slices relative to a power-of-two bound 2^E of the row:
//   h = RN(x / 2^(E-8)) 2^(E-8),  m = RN((x-h) / 2^(E-17)) 2^(E-17),
//   l = RN((x-h-m) / 2^(E-26)) 2^(E-26),
// each slice an integer of at most 8 significant bits times a power of two,
// so exactly representable in bf16; the DFT tables are sliced the same way
// with E = 0.  Products of first slices are integers in one unit per row and
// their sums stay below 2^24 units for K <= 256, so the synthesis accumulates
// hi x hi in its own TMEM accumulator exactly and the five correction
// products (hi.mid, mid.hi, hi.lo, mid.mid, lo.hi) in a second one; the
// analysis (whose rounding matters less) uses one accumulator with the
// corrections issued before hi x hi.  With 2 slices (3 products) the form
// is the plain "bf16 hi/lo" split.
//
// Tile.  One launch runs a whole program (the MHD bundle: 15 fields in, 10
// out).  The 128 MMA rows are (field slot, point) pairs: 16 slots x 8 points
// for programs with more than 8 input fields, 8 x 16 for the cross and dot
// products, 4 x 32 for the scalar and scalar x vector products (the tensor
// product of FFT_TENSOR_DCL runs as three scalar x vector programs).  A row's TMEM accumulators hold its
// field's four classes at all Q angles (8Q fp32 columns, 384 at m=64).  After
// the synthesis each row is folded to the 4Q physical angles in FP64 and the
// rows of one point meet in shared memory, 16 quarter-angles at a time; each
// output of the pointwise program is a sum of at most four signed products of
// two fields (a constant term table per program), evaluated by one thread per
// (output, point, half-chunk).  The folded products, sliced, are the A operand
// of the analysis, whose rows are (output, point) pairs; each 16-angle chunk is
// analysed into a fresh accumulator and added in FP64 to the output, which the
// same thread updates chunk after chunk (the lines stay in L2).
//
// One CTA of 8 warps, persistent over tiles; two threads per row.  Thread 0
// issues the MMAs; completion is signalled through an mbarrier whose waits
// are bounded (a timeout sets a status word and abandons the tile instead of
// spinning forever).
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <map>
#include <mutex>
#include <vector>

#include "sfnl_internal.h"
#include "sfnl_ops.cuh"

namespace sfnl {

namespace {

constexpr int kW = 8;            // bits of the first slice (integers up to 2^8)
constexpr int kKeMax = 32;       // modes per class held in registers (m <= 64)

// Status word of the split kernels: a pinned host word mapped into the device address space, set to 1
// by a CTA whose bounded wait on its tensor-core operations gave up.  The host reads it without a copy
// or a synchronisation (split_take_status); it is shared by every device and stream of the process.
std::mutex g_status_mu;
int *g_status_host = nullptr;  // pinned, mapped
int *g_status_dev = nullptr;   // its device address

// ---------------------------------------------------------------------------
// geometry
// ---------------------------------------------------------------------------
struct SGeo {
  int m, Q, N, NC, pts;
  int ke[4], Ks[4], No[4];      // modes per class, K padded to 16, output cols padded to 16
  int Ks_tot, No_tot;
  int tmem_cols, tmem_alloc;
  // shared-memory byte offsets (relative to the dynamic smem base)
  int off_asyn[4][3], off_bsyn[4][3], off_bana[4][3], off_x, off_aana[4][3], off_bar, smem_bytes;
  int ana_col[4];
};

int pow2_at_least(int v) {
  int p = 32;
  while (p < v) p <<= 1;
  return p;
}

bool make_sgeo(int m, int pts, int nin, SGeo *out) {
  SGeo g;
  std::memset(&g, 0, sizeof(g));
  g.m = m;
  g.pts = pts;
  const int qmin = (3 * m - 2 + 3) / 4;
  g.Q = ((qmin + 15) / 16) * 16;
  if (g.Q < 16) g.Q = 16;
  g.N = 4 * g.Q;
  g.NC = g.Q / 16;
  const int ev = (m + 1) / 2, od = m / 2;
  const int cnt[4] = {ev, od, ev, od};
  for (int c = 0; c < 4; ++c) {
    g.ke[c] = cnt[c];
    g.Ks[c] = ((cnt[c] + 15) / 16) * 16;
    if (g.Ks[c] == 0) g.Ks[c] = 16;  // keep every class present (zero rows) to simplify indexing
    g.No[c] = g.Ks[c];
    g.Ks_tot += g.Ks[c];
    g.No_tot += g.No[c];
  }
  if (ev > kKeMax) return false;
  g.tmem_cols = 8 * g.Q + g.No_tot;
  if (g.tmem_cols > 512) return false;
  g.tmem_alloc = pow2_at_least(g.tmem_cols);
  int acc = 0;
  for (int c = 0; c < 4; ++c) {
    g.ana_col[c] = 8 * g.Q + acc;
    acc += g.No[c];
  }
  // Region 1: synthesis A operands, later overlaid by the exchange buffer and the analysis A operands.
  int asyn = 0;
  for (int c = 0; c < 4; ++c)
    for (int i = 0; i < 3; ++i) {
      g.off_asyn[c][i] = asyn;
      asyn += 128 * g.Ks[c] * 2;
    }
  const int xbytes = nin * 64 * pts * 8;
  int r1b = xbytes;
  for (int c = 0; c < 4; ++c)
    for (int i = 0; i < 3; ++i) {
      g.off_aana[c][i] = r1b;
      r1b += 128 * 16 * 2;
    }
  g.off_x = 0;
  int r1 = asyn > r1b ? asyn : r1b;
  r1 = (r1 + 127) & ~127;
  int off = r1;
  for (int c = 0; c < 4; ++c)
    for (int j = 0; j < 3; ++j) {
      g.off_bsyn[c][j] = off;
      off += g.Q * g.Ks[c] * 2;
    }
  for (int c = 0; c < 4; ++c)
    for (int j = 0; j < 3; ++j) {
      g.off_bana[c][j] = off;
      off += g.No[c] * g.Q * 2;
    }
  off = (off + 15) & ~15;
  g.off_bar = off;
  off += 16;
  g.smem_bytes = off;
  if (g.smem_bytes > 227 * 1024) return false;
  *out = g;
  return true;
}

// Canonical K-major, no-swizzle offset of element (row, k) in a tile whose rows have K elements.
inline size_t kmajor_off(int row, int k, int K) {
  return (size_t)(row / 8) * (16 * K) + (size_t)(k / 8) * 128 + (size_t)(row % 8) * 16 + (size_t)(k % 8) * 2;
}

// Host-side fixed-point slices of a value with |x| <= 2^E.
void slice3_host(double x, int E, double s[3]) {
  double unit = std::ldexp(1.0, E - kW);
  double r = x;
  for (int i = 0; i < 3; ++i) {
    const double q = std::nearbyint(r / unit) * unit;
    s[i] = q;
    r -= q;
    unit = std::ldexp(unit, -(kW + 1));
  }
}

uint16_t to_bf16_bits(double v) {
  const float f = (float)v;  // exact: at most 8 significant bits
  uint32_t u;
  std::memcpy(&u, &f, 4);
  return (uint16_t)(u >> 16);  // exact truncation: low 16 bits are zero
}

struct STables {
  void *bsyn = nullptr;  // all synthesis B tiles, contiguous in smem order
  void *bana = nullptr;
  size_t bsyn_bytes = 0, bana_bytes = 0;
};
std::mutex g_stab_mu;
std::map<std::pair<int, int>, STables> g_stabs;  // (device, m)

int get_stables(const SGeo &g, STables *out) {
  int dev = 0;
  cudaGetDevice(&dev);
  std::lock_guard<std::mutex> lk(g_stab_mu);
  auto it = g_stabs.find({dev, g.m});
  if (it != g_stabs.end()) {
    *out = it->second;
    return SFNL_OK;
  }
  const long double pi = acosl(-1.0L);
  auto ang = [&](int j) { return pi * (long double)(2 * j + 1) / (long double)g.N; };
  // synthesis: per class c, slice j: Q rows (angles) x Ks[c] (modes)
  size_t bs = 0, ba = 0;
  for (int c = 0; c < 4; ++c) {
    bs += (size_t)3 * g.Q * g.Ks[c] * 2;
    ba += (size_t)3 * g.No[c] * g.Q * 2;
  }
  std::vector<uint16_t> hs(bs / 2, 0), ha(ba / 2, 0);
  size_t base = 0;
  for (int c = 0; c < 4; ++c) {
    for (int jj = 0; jj < g.Q; ++jj)
      for (int k = 0; k < g.ke[c]; ++k) {
        const int n = 2 * k + (c & 1);
        const long double x = (long double)n * ang(jj);
        const double v = (double)(c < 2 ? cosl(x) : sinl(x));
        double s[3];
        slice3_host(v, 0, s);
        for (int sl = 0; sl < 3; ++sl)
          hs[(base + (size_t)sl * g.Q * g.Ks[c] * 2 + kmajor_off(jj, k, g.Ks[c])) / 2] = to_bf16_bits(s[sl]);
      }
    base += (size_t)3 * g.Q * g.Ks[c] * 2;
  }
  base = 0;
  for (int c = 0; c < 4; ++c) {
    for (int kk = 0; kk < g.ke[c]; ++kk)
      for (int jj = 0; jj < g.Q; ++jj) {
        const int n = 2 * kk + (c & 1);
        const long double x = (long double)n * ang(jj);
        const double v = (double)(c < 2 ? cosl(x) : sinl(x));
        double s[3];
        slice3_host(v, 0, s);
        for (int sl = 0; sl < 3; ++sl)
          ha[(base + (size_t)sl * g.No[c] * g.Q * 2 + kmajor_off(kk, jj, g.Q)) / 2] = to_bf16_bits(s[sl]);
      }
    base += (size_t)3 * g.No[c] * g.Q * 2;
  }
  STables T;
  T.bsyn_bytes = bs;
  T.bana_bytes = ba;
  if (cudaMalloc(&T.bsyn, bs) != cudaSuccess || cudaMalloc(&T.bana, ba) != cudaSuccess) {
    cudaGetLastError();
    return set_error(SFNL_ERR_ALLOC, "cudaMalloc of the split DFT tables failed");
  }
  if (cudaMemcpy(T.bsyn, hs.data(), bs, cudaMemcpyHostToDevice) != cudaSuccess ||
      cudaMemcpy(T.bana, ha.data(), ba, cudaMemcpyHostToDevice) != cudaSuccess)
    return set_error(SFNL_ERR_CUDA, "upload of the split DFT tables failed");
  g_stabs[{dev, g.m}] = T;
  *out = T;
  return SFNL_OK;
}

// ---------------------------------------------------------------------------
// device helpers (inline PTX for tcgen05 / mbarrier)
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint32_t smem_u32(const void *p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ uint64_t make_sdesc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  uint64_t d = 0;
  d |= (uint64_t)((saddr >> 4) & 0x3FFF);
  d |= (uint64_t)((lbo >> 4) & 0x3FFF) << 16;
  d |= (uint64_t)((sbo >> 4) & 0x3FFF) << 32;
  d |= (uint64_t)1 << 46;  // descriptor version for sm_100
  // base offset 0, lbo mode 0, layout type 0 (no swizzle)
  return d;
}

// kind::f16 instruction descriptor: bf16 x bf16 -> f32, both K-major, M = 128.
__device__ __forceinline__ uint32_t make_idesc(int N) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(128 >> 4) << 24);
}

__device__ __forceinline__ void umma_bf16(uint32_t d_tmem, uint64_t a, uint64_t b, uint32_t idesc, uint32_t acc) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(d_tmem),
      "l"(a), "l"(b), "r"(idesc), "r"(acc));
}

__device__ __forceinline__ void umma_commit(uint32_t mbar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(mbar) : "memory");
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

__device__ __forceinline__ void mbar_init(uint32_t mbar, int count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(mbar), "r"(count) : "memory");
}

// Bounded wait for the given phase parity; returns false on timeout.
__device__ __forceinline__ bool mbar_wait(uint32_t mbar, uint32_t parity) {
  for (int it = 0; it < (1 << 22); ++it) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(done)
        : "r"(mbar), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
}

// Marks the call as failed in the mapped status word (visible to the host without a copy).
__device__ __forceinline__ void report_timeout(int *status) {
  if (status) {
    *reinterpret_cast<volatile int *>(status) = 1;
    __threadfence_system();
  }
}

__device__ __forceinline__ void tmem_ld8(uint32_t taddr, float (&v)[8]) {
  uint32_t r[8];
  asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
               : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7])
               : "r"(taddr));
#pragma unroll
  for (int i = 0; i < 8; ++i) v[i] = __uint_as_float(r[i]);
}
__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

// 2^e as a double (e clamped to the normal range).
__device__ __forceinline__ double pow2(int e) {
  e = e < -1022 ? -1022 : (e > 1023 ? 1023 : e);
  return __longlong_as_double((long long)(e + 1023) << 52);
}

__device__ __forceinline__ int row_exponent(double mx) {
  int e = 0;
  frexp(mx, &e);  // mx = f 2^e, f in [0.5, 1) -> mx < 2^e
  return e;
}

// 2^e as a float (e in the normal range).
__device__ __forceinline__ float pow2f(int e) { return __int_as_float((e + 127) << 23); }

// Per-row slicing factors for the bound 2^E: the first slice is cut in FP64, the remainder
// (|r| <= 2^(E-9)) is rounded once to FP32 (error <= 2^(E-33), far below the last slice's
// 2^(E-27)) and cut into the second and third slices in FP32; every step multiplies by an
// exact power of two, so the slices are exact integers (<= 2^8) times powers of two.
struct SliceScale {
  double i0, u0;
  float i1, u1, i2, u2;
};
__device__ __forceinline__ SliceScale slice_scale(int E) {
  E = E < -100 ? -100 : (E > 100 ? 100 : E);  // keep the FP32 factors normal
  SliceScale s;
  s.i0 = pow2(kW - E);
  s.u0 = pow2(E - kW);
  s.i1 = pow2f(2 * kW + 1 - E);
  s.u1 = pow2f(E - 2 * kW - 1);
  s.i2 = pow2f(3 * kW + 2 - E);
  s.u2 = pow2f(E - 3 * kW - 2);
  return s;
}
__device__ __forceinline__ void slice3f(double x, const SliceScale &s, float &h, float &m, float &l) {
  const double hd = rint(x * s.i0) * s.u0;
  const float r = (float)(x - hd);
  m = rintf(r * s.i1) * s.u1;
  l = rintf((r - m) * s.i2) * s.u2;
  h = (float)hd;
}
__device__ __forceinline__ uint32_t pack_bf16(float lo, float hi) {
  const __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
  return *reinterpret_cast<const uint32_t *>(&v);
}

// ---------------------------------------------------------------------------
// programs: each output is a sum of at most 4 signed products x[a]*x[b]
// ---------------------------------------------------------------------------
enum { PR_BUNDLE = 0, PR_CROSS, PR_DOT, PR_PROD, PR_CJVP, PR_CVJP, PR_MVJP, PR_SVECT, PR_COUNT };

struct STerm {
  signed char a, b, s;
};
#define T2(a0, b0, a1, b1) {{a0, b0, 1}, {a1, b1, -1}, {0, 0, 0}, {0, 0, 0}}
#define T4(a0, b0, a1, b1, a2, b2, a3, b3) {{a0, b0, 1}, {a1, b1, -1}, {a2, b2, 1}, {a3, b3, -1}}
constexpr STerm kTerms[PR_COUNT][10][4] = {
    // bundle [u 0-2, w 3-5, b 6-8, j 9-11, gradT 12-14] -> [u x w, u x b, j x b, u . gradT]
    {T2(1, 5, 2, 4), T2(2, 3, 0, 5), T2(0, 4, 1, 3), T2(1, 8, 2, 7), T2(2, 6, 0, 8), T2(0, 7, 1, 6),
     T2(10, 8, 11, 7), T2(11, 6, 9, 8), T2(9, 7, 10, 6), {{0, 12, 1}, {1, 13, 1}, {2, 14, 1}, {0, 0, 0}}},
    // cross [v1 0-2, v2 3-5] -> v1 x v2
    {T2(1, 5, 2, 4), T2(2, 3, 0, 5), T2(0, 4, 1, 3)},
    // dot -> v1 . v2
    {{{0, 3, 1}, {1, 4, 1}, {2, 5, 1}, {0, 0, 0}}},
    // scalar product
    {{{0, 1, 1}, {0, 0, 0}, {0, 0, 0}, {0, 0, 0}}},
    // linearised cross [u 0-2, w 3-5, du 6-8, dw 9-11] -> du x w + u x dw
    {T4(7, 5, 8, 4, 1, 11, 2, 10), T4(8, 3, 6, 5, 2, 9, 0, 11), T4(6, 4, 7, 3, 0, 10, 1, 9)},
    // its transpose [u 0-2, w 3-5, c 6-8] -> [w x c, c x u]
    {T2(4, 8, 5, 7), T2(5, 6, 3, 8), T2(3, 7, 4, 6), T2(7, 2, 8, 1), T2(8, 0, 6, 2), T2(6, 1, 7, 0)},
    // transpose of (du x w + u x dw, du x b + u x db): [u, w, b, c1 9-11, c2 12-14] -> [w x c1 + b x c2, c1 x u, c2 x u]
    {T4(4, 11, 5, 10, 7, 14, 8, 13), T4(5, 9, 3, 11, 8, 12, 6, 14), T4(3, 10, 4, 9, 6, 13, 7, 12),
     T2(10, 2, 11, 1), T2(11, 0, 9, 2), T2(9, 1, 10, 0), T2(13, 2, 14, 1), T2(14, 0, 12, 2), T2(12, 1, 13, 0)},
    // scalar x vector [v 0-2, s 3] -> s v (fft_parallel.F90:1150-1153); the tensor u_k v_l is three of
    // these, [v, u_k] -> u_k v (:1676-1687)
    {{{0, 3, 1}, {0, 0, 0}, {0, 0, 0}, {0, 0, 0}},
     {{1, 3, 1}, {0, 0, 0}, {0, 0, 0}, {0, 0, 0}},
     {{2, 3, 1}, {0, 0, 0}, {0, 0, 0}, {0, 0, 0}}},
};
#undef T2
#undef T4
__constant__ STerm c_terms[PR_COUNT][10][4];  // filled from kTerms at first use (see upload_terms)

__host__ __device__ constexpr int pr_nin(int pr) {
  return pr == PR_BUNDLE ? 15 : pr == PR_CROSS ? 6 : pr == PR_DOT ? 6 : pr == PR_PROD ? 2 : pr == PR_CJVP ? 12
       : pr == PR_CVJP ? 9 : pr == PR_MVJP ? 15 : 4;
}
__host__ __device__ constexpr int pr_nout(int pr) {
  return pr == PR_BUNDLE ? 10 : pr == PR_CROSS ? 3 : pr == PR_DOT ? 1 : pr == PR_PROD ? 1 : pr == PR_CJVP ? 3
       : pr == PR_CVJP ? 6 : pr == PR_MVJP ? 9 : 3;
}
__host__ __device__ constexpr int pr_slots(int pr) { return pr_nin(pr) > 8 ? 16 : pr_nin(pr) > 4 ? 8 : 4; }
__host__ __device__ constexpr int pr_pts(int pr) { return 128 / pr_slots(pr); }
// cotangent inputs (synthesised with the analysis weights) and transposed outputs (analysed without them)
__host__ __device__ constexpr unsigned pr_adj_in(int pr) { return pr == PR_CVJP ? 0x1C0u : pr == PR_MVJP ? 0x7E00u : 0u; }
__host__ __device__ constexpr bool pr_adj_out(int pr) { return pr == PR_CVJP || pr == PR_MVJP; }

struct SplitArgs {
  const double *in[16];
  double *out[10];
  int64_t in_ldm[16], out_ldm[10], in_bs[16], out_bs[10];
  int64_t out_ps;  // point stride of the outputs (3 in the tensor layout), sine at out_ps*np
  int64_t np;
  int nsl;
  SGeo g;
  const void *bsyn, *bana;
  int bsyn_bytes, bana_bytes;
  int *status;  // the mapped status word
};

constexpr int kThreads = 256;

// Compile-time geometry of make_sgeo for a given m (0: read it from the arguments).
__host__ __device__ constexpr int sg_qmin(int m) { return (3 * m - 2 + 3) / 4; }
__host__ __device__ constexpr int sg_Q(int m) { return ((sg_qmin(m) + 15) / 16) * 16 < 16 ? 16 : ((sg_qmin(m) + 15) / 16) * 16; }
__host__ __device__ constexpr int sg_ke(int m, int c) { return (c & 1) ? m / 2 : (m + 1) / 2; }
__host__ __device__ constexpr int sg_Ks(int m, int c) { return ((sg_ke(m, c) + 15) / 16) * 16 < 16 ? 16 : ((sg_ke(m, c) + 15) / 16) * 16; }
__host__ __device__ constexpr int sg_anacol(int m, int c) { return c == 0 ? 8 * sg_Q(m) : sg_anacol(m, c - 1) + sg_Ks(m, c - 1); }

// Product phase for one output O of program PR (warp-uniform): lane = point p + PTS*jg, each lane owns
// J consecutive quarter-angles of the 16-angle chunk.  Evaluates the output at the 4 quadrant angles,
// folds the products into the analysis classes, finds each class row's bound over the chunk (shuffles
// across the lanes of the same point), slices and writes the analysis A operand row O*PTS + p.
// Product phase for one output o (warp-uniform): lane = point p + PTS*jg, each lane owns J consecutive
// quarter-angles of the 16-angle chunk.  The output's (at most 4) terms s*x[a]*x[b] are read once from
// constant memory into registers as shared-memory offsets.  Evaluates the output at the 4 quadrant
// angles, folds the products into the analysis classes, finds each class row's bound over the chunk
// (shuffles across the lanes of the same point), slices and writes the analysis A operand row o*PTS + p.
template <int PR>
__device__ __forceinline__ void product_rows(int o, const double *X, unsigned char *sm, const SGeo &g, int lane) {
  constexpr int PTS = pr_pts(PR), JG = 32 / PTS, J = 16 / JG;
  const int p = lane % PTS, jg = lane / PTS;
  const double *xa[4], *xb[4];
  double sg[4];
#pragma unroll
  for (int u = 0; u < 4; ++u) {
    const STerm tm = c_terms[PR][o][u];
    xa[u] = X + (size_t)tm.a * 64 * PTS + (size_t)jg * J * PTS + p;
    xb[u] = X + (size_t)tm.b * 64 * PTS + (size_t)jg * J * PTS + p;
    sg[u] = (double)tm.s;  // 0 for an unused term
  }
  double P[4][J];
  double mx[4] = {0.0, 0.0, 0.0, 0.0};
#pragma unroll
  for (int jj = 0; jj < J; ++jj) {
    double gq[4];
#pragma unroll
    for (int r = 0; r < 4; ++r) {
      const int off = (r * 16 + jj) * PTS;
      double acc = 0.0;
#pragma unroll
      for (int u = 0; u < 4; ++u)
        if (sg[u] != 0.0) acc = fma(sg[u] * xa[u][off], xb[u][off], acc);  // warp-uniform branch
      gq[r] = acc;
    }
    const double s14 = gq[0] + gq[3], d14 = gq[0] - gq[3], s23 = gq[1] + gq[2], d32 = gq[2] - gq[1];
    P[0][jj] = s14 + s23;
    P[1][jj] = s14 - s23;
    P[2][jj] = d14 + d32;
    P[3][jj] = d14 - d32;
#pragma unroll
    for (int c = 0; c < 4; ++c) mx[c] = fmax(mx[c], fabs(P[c][jj]));
  }
#pragma unroll
  for (int c = 0; c < 4; ++c)
#pragma unroll
    for (int sh = PTS; sh < 32; sh <<= 1) mx[c] = fmax(mx[c], __shfl_xor_sync(0xffffffffu, mx[c], sh));
  const int ro = o * PTS + p, k0 = jg * J;
#pragma unroll
  for (int c = 0; c < 4; ++c) {
    const SliceScale sc = slice_scale(row_exponent(mx[c]));
    uint32_t w[3][J / 2];
#pragma unroll
    for (int q = 0; q < J / 2; ++q) {
      float h0, m0, l0, h1, m1, l1;
      slice3f(P[c][2 * q], sc, h0, m0, l0);
      slice3f(P[c][2 * q + 1], sc, h1, m1, l1);
      w[0][q] = pack_bf16(h0, h1);
      w[1][q] = pack_bf16(m0, m1);
      w[2][q] = pack_bf16(l0, l1);
    }
#pragma unroll
    for (int i = 0; i < 3; ++i) {
      unsigned char *rowp = sm + g.off_aana[c][i] + (size_t)(ro / 8) * 256 + (size_t)(ro % 8) * 16;
#pragma unroll
      for (int q0 = 0; q0 < J / 2; q0 += 4) {
        const int k = k0 + 2 * q0;  // first of the (up to) 8 k-values of this store
        unsigned char *dst = rowp + (size_t)(k / 8) * 128 + (size_t)(k % 8) * 2;
        if constexpr (J / 2 >= 4)
          *reinterpret_cast<uint4 *>(dst) = make_uint4(w[i][q0], w[i][q0 + 1], w[i][q0 + 2], w[i][q0 + 3]);
        else
          *reinterpret_cast<uint2 *>(dst) = make_uint2(w[i][0], w[i][1]);
      }
    }
  }
}

template <int PR, int M>
__global__ void __launch_bounds__(kThreads, 1) split_kernel(const SplitArgs a) {
  constexpr int NI = pr_nin(PR), NO = pr_nout(PR), PTS = pr_pts(PR);
  constexpr unsigned ADJ = pr_adj_in(PR);
  constexpr bool CT = M > 0;
  constexpr int KE_MAX = CT ? (M + 1) / 2 : kKeMax;
  extern __shared__ __align__(128) unsigned char sm[];
  __shared__ uint32_t s_tmem;
  const SGeo &g = a.g;
  const int t = threadIdx.x, warp = t >> 5, lane = t & 31;
  const int row = t & 127, half = t >> 7;  // TMEM lane = row (warp w reads lanes 32*(w%4)..)
  const uint32_t mbar = smem_u32(sm + g.off_bar);
  const int Q = CT ? sg_Q(M) : g.Q, NC = Q / 16;
  int KE[4], KS[4], ACOL[4];
#pragma unroll
  for (int c = 0; c < 4; ++c) {
    KE[c] = CT ? sg_ke(M, c) : g.ke[c];
    KS[c] = CT ? sg_Ks(M, c) : g.Ks[c];
    ACOL[c] = CT ? sg_anacol(M, c) : g.ana_col[c];
  }

  // ---- setup: TMEM, mbarrier, DFT tables ----
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&s_tmem)),
                 "r"(g.tmem_alloc));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  if (t == 0) mbar_init(mbar, 1);
  {
    const uint4 *src = reinterpret_cast<const uint4 *>(a.bsyn);
    uint4 *dst = reinterpret_cast<uint4 *>(sm + g.off_bsyn[0][0]);
    for (int i = t; i < a.bsyn_bytes / 16; i += kThreads) dst[i] = src[i];
    const uint4 *src2 = reinterpret_cast<const uint4 *>(a.bana);
    uint4 *dst2 = reinterpret_cast<uint4 *>(sm + g.off_bana[0][0]);
    for (int i = t; i < a.bana_bytes / 16; i += kThreads) dst2[i] = src2[i];
  }
  fence_async_smem();
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = s_tmem;
  const uint32_t lane_base = (uint32_t)((warp & 3) * 32) << 16;
  uint32_t phase = 0;
  bool ok = true;

  const int64_t ntiles = (a.np + PTS - 1) / PTS;
  const double invN = 1.0 / (4.0 * Q), twoN = 2.0 * invN;
  const int npairs = a.nsl == 3 ? 6 : 3;
  double *X = reinterpret_cast<double *>(sm + g.off_x);  // [f][quadrant][16][PTS], point fastest

  // Reads the analysis of one chunk and adds it (weighted) to the outputs: row = (o, p), half = class pair.
  auto flush_chunk = [&](int64_t tile, int chk) {
    const int o = row / PTS, p = row % PTS;
    const int64_t gp = tile * PTS + p;
    const bool live = row < NO * PTS && gp < a.np;
#pragma unroll
    for (int cc = 0; cc < 2; ++cc) {
      const int c = 2 * half + cc;  // classes 0,1 (cos) or 2,3 (sin)
      const int kec = half ? KE[2 + cc] : KE[cc], ksc = half ? KS[2 + cc] : KS[cc];
      const int acol = half ? ACOL[2 + cc] : ACOL[cc];
      for (int k0 = 0; k0 < ksc; k0 += 8) {
        float v[8];
        tmem_ld8(tmem + lane_base + (uint32_t)(acol + k0), v);
        tmem_wait_ld();
        if (!live) continue;
        double *dst = a.out[o] + gp * a.out_ps + (half ? a.np * a.out_ps : 0);
        const int64_t ldm = a.out_ldm[o];
#pragma unroll
        for (int e = 0; e < 8; ++e) {
          const int kk = k0 + e;
          if (kk >= kec) break;
          const int n = 2 * kk + cc;
          const double sc = pr_adj_out(PR) ? 1.0 : (n == 0 ? invN : twoN);
          const double val = (half && n == 0) ? 0.0 : (double)v[e] * sc;
          double *q = dst + (int64_t)n * ldm;
          *q = (chk == 0 ? 0.0 : *q) + val;
        }
      }
      (void)c;
    }
  };

  for (int64_t tile = blockIdx.x; tile < ntiles && ok; tile += gridDim.x) {
    // ---- 1. load + slice the input rows: row = field slot f, point p; half = class pair ----
    {
      const int f = row / PTS, p = row % PTS;
      const int64_t gp = tile * PTS + p;
      const bool valid = f < NI && gp < a.np;
      const double *src = valid ? a.in[f] + gp : nullptr;
      const int64_t ldm = valid ? a.in_ldm[f] : 0;
      const bool cot = f < NI && ((ADJ >> f) & 1u);
#pragma unroll
      for (int cc = 0; cc < 2; ++cc) {
        const int c = 2 * half + cc;
        const int kec = half ? KE[2 + cc] : KE[cc], ksc = half ? KS[2 + cc] : KS[cc];
        double x[KE_MAX];
        double mx = 0.0;
#pragma unroll
        for (int k = 0; k < KE_MAX; ++k) {
          const int n = 2 * k + cc;
          double v = 0.0;
          if (valid && k < kec && !(half && n == 0)) {
            v = __ldg(src + (int64_t)n * ldm + (half ? a.np : 0));
            if (cot) v *= (n == 0 ? invN : twoN);
          }
          x[k] = v;
          mx = fmax(mx, fabs(v));
        }
        const SliceScale sc = slice_scale(row_exponent(mx));
#pragma unroll
        for (int kg = 0; kg < (KE_MAX + 7) / 8 + 1; ++kg) {
          if (kg * 8 >= ksc) break;
          uint32_t w[3][4];
#pragma unroll
          for (int q = 0; q < 4; ++q) {
            float hv[2], mv[2], lv[2];
#pragma unroll
            for (int e = 0; e < 2; ++e) {
              const int k = kg * 8 + 2 * q + e;
              slice3f(k < KE_MAX ? x[k < KE_MAX ? k : 0] : 0.0, sc, hv[e], mv[e], lv[e]);
            }
            w[0][q] = pack_bf16(hv[0], hv[1]);
            w[1][q] = pack_bf16(mv[0], mv[1]);
            w[2][q] = pack_bf16(lv[0], lv[1]);
          }
          const size_t off = (size_t)(row / 8) * (16 * ksc) + (size_t)kg * 128 + (size_t)(row % 8) * 16;
#pragma unroll
          for (int i = 0; i < 3; ++i)
            *reinterpret_cast<uint4 *>(sm + g.off_asyn[c][i] + off) = make_uint4(w[i][0], w[i][1], w[i][2], w[i][3]);
        }
      }
    }
    fence_async_smem();
    tc_fence_before();
    __syncthreads();

    // ---- 2. synthesis MMAs: D0 (hi x hi) and D1 (corrections) per class ----
    if (t == 0) {
      tc_fence_after();
      const uint32_t idesc = make_idesc(Q);
      for (int c = 0; c < 4; ++c) {
        const uint32_t sbo = 16 * KS[c];
        for (int s = 0; s < KS[c] / 16; ++s)
          for (int pr = 0; pr < npairs; ++pr) {
            const int i = pr == 0 ? 0 : pr == 1 ? 0 : pr == 2 ? 1 : pr == 3 ? 0 : pr == 4 ? 1 : 2;
            const int j = pr == 0 ? 0 : pr == 1 ? 1 : pr == 2 ? 0 : pr == 3 ? 2 : pr == 4 ? 1 : 0;
            const int accn = (i + j == 0) ? 0 : 1;
            const uint32_t dcol = tmem + (uint32_t)((c * 2 + accn) * Q);
            const uint64_t ad = make_sdesc(smem_u32(sm + g.off_asyn[c][i]) + 256 * s, 128, sbo);
            const uint64_t bd = make_sdesc(smem_u32(sm + g.off_bsyn[c][j]) + 256 * s, 128, sbo);
            const uint32_t en = (s > 0 || (accn == 1 && pr > 1)) ? 1u : 0u;
            umma_bf16(dcol, ad, bd, idesc, en);
          }
      }
      umma_commit(mbar);
    }
    __syncwarp();
    // Every thread waits (bounded) and the CTA agrees on the outcome before any barrier or loop
    // condition depends on it; on a timeout the phase stays, so the final drain waits for it again.
    if (!__syncthreads_and(mbar_wait(mbar, phase))) {
      ok = false;
      if (t == 0) report_timeout(a.status);
    } else {
      phase ^= 1;
    }
    tc_fence_after();

    for (int ch = 0; ch < NC && ok; ++ch) {
      // ---- 3a. read out, recombine in FP64, fold to the 4 quadrant angles (half = 8 quarter-angles) ----
      {
        const int f = row / PTS, p = row % PTS;
        float d[4][2][8];
#pragma unroll
        for (int c = 0; c < 4; ++c)
#pragma unroll
          for (int ac = 0; ac < 2; ++ac)
            tmem_ld8(tmem + lane_base + (uint32_t)((c * 2 + ac) * Q + ch * 16 + half * 8), d[c][ac]);
        tmem_wait_ld();
        if (f < NI) {
          double *xr = X + (size_t)f * 64 * PTS + (size_t)half * 8 * PTS + p;
#pragma unroll
          for (int jj = 0; jj < 8; ++jj) {
            const double CE = (double)d[0][0][jj] + (double)d[0][1][jj];
            const double CO = (double)d[1][0][jj] + (double)d[1][1][jj];
            const double SE = (double)d[2][0][jj] + (double)d[2][1][jj];
            const double SO = (double)d[3][0][jj] + (double)d[3][1][jj];
            const double A = CE + CO, B = CE - CO, C = SE + SO, D = SO - SE;
            xr[(0 * 16 + jj) * PTS] = A + C;  // theta
            xr[(1 * 16 + jj) * PTS] = B + D;  // pi - theta
            xr[(2 * 16 + jj) * PTS] = B - D;  // pi + theta
            xr[(3 * 16 + jj) * PTS] = A - C;  // 2 pi - theta
          }
        }
      }
      tc_fence_before();
      __syncthreads();
      // The previous chunk's analysis must be complete before its A operand is rewritten.
      if (ch > 0) {
        if (!__syncthreads_and(mbar_wait(mbar, phase))) {
          ok = false;
          if (t == 0) report_timeout(a.status);
          break;
        }
        phase ^= 1;
        tc_fence_after();
        flush_chunk(tile, ch - 1);
      }
      // ---- 3b. program, analysis pre-fold, slicing: one output per warp ----
      for (int o = warp; o < NO; o += kThreads / 32) product_rows<PR>(o, X, sm, g, lane);
      fence_async_smem();
      tc_fence_before();
      __syncthreads();
      // ---- 3c. analysis MMAs for this chunk, fresh accumulator (corrections first, then hi x hi) ----
      if (t == 0 && ok) {
        tc_fence_after();
        for (int c = 0; c < 4; ++c) {
          const uint32_t idesc = make_idesc(KS[c]);
          const uint32_t dcol = tmem + (uint32_t)ACOL[c];
          for (int pr = 0; pr < npairs; ++pr) {
            int i, j;
            if (a.nsl == 3) {
              i = pr == 0 ? 0 : pr == 1 ? 1 : pr == 2 ? 0 : pr == 3 ? 1 : pr == 4 ? 2 : 0;
              j = pr == 0 ? 1 : pr == 1 ? 0 : pr == 2 ? 2 : pr == 3 ? 1 : pr == 4 ? 0 : 0;
            } else {
              i = pr == 1 ? 1 : 0;
              j = pr == 0 ? 1 : 0;
            }
            const uint64_t ad = make_sdesc(smem_u32(sm + g.off_aana[c][i]), 128, 256);
            const uint64_t bd = make_sdesc(smem_u32(sm + g.off_bana[c][j]) + 256 * ch, 128, 16 * Q);
            umma_bf16(dcol, ad, bd, idesc, pr > 0 ? 1u : 0u);
          }
        }
        umma_commit(mbar);
      }
      __syncwarp();
    }
    // ---- 4. the last chunk into the outputs ----
    if (ok) {
      if (!__syncthreads_and(mbar_wait(mbar, phase))) {
        ok = false;
        if (t == 0) report_timeout(a.status);
      } else {
        phase ^= 1;
      }
    }
    tc_fence_after();
    if (ok) flush_chunk(tile, NC - 1);
    tc_fence_before();
    __syncthreads();
  }
  __syncthreads();
  // After a timeout the last commit's phase is still pending: wait for it once more (bounded) so that
  // no tensor-core operation still writes the columns being freed; the status word already reports
  // the call as failed either way.
  if (!ok) {
    const bool drained = mbar_wait(mbar, phase);
    __syncthreads();
    (void)drained;
  }
  if (warp == 0) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(g.tmem_alloc));
  }
}

template <int PR, int M>
int launch_split_pr(SplitArgs &sa, int batch, const ProgArgs &pa, const int *in_map, const int *out_map,
                    cudaStream_t st) {
  constexpr int NI = pr_nin(PR), NO = pr_nout(PR), PTS = pr_pts(PR);
  auto kern = split_kernel<PR, M>;
  if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, sa.g.smem_bytes) != cudaSuccess)
    return set_error(SFNL_ERR_CUDA, "cudaFuncSetAttribute failed (split form)");
  const int64_t ntiles = (sa.np + PTS - 1) / PTS;
  int per_sm_tmem = 512 / sa.g.tmem_alloc;
  int per_sm_smem = (int)((228 * 1024) / (sa.g.smem_bytes + 1024));
  int per_sm = per_sm_tmem < per_sm_smem ? per_sm_tmem : per_sm_smem;
  if (per_sm < 1) per_sm = 1;
  int64_t grid = (int64_t)num_sms() * per_sm;
  if (grid > ntiles) grid = ntiles;
  if (grid < 1) grid = 1;
  for (int b = 0; b < batch; ++b) {
    for (int i = 0; i < NI; ++i) {
      sa.in[i] = pa.in[in_map[i]] + (int64_t)b * pa.in_bs[in_map[i]];
      sa.in_ldm[i] = pa.in_ldm[in_map[i]];
    }
    for (int o = 0; o < NO; ++o) {
      sa.out[o] = pa.out[out_map[o]] + (int64_t)b * pa.out_bs[out_map[o]];
      sa.out_ldm[o] = pa.out_ldm[out_map[o]];
    }
    kern<<<(unsigned)grid, kThreads, sa.g.smem_bytes, st>>>(sa);
    int rc = check_launch("split form");
    if (rc) return rc;
  }
  return SFNL_OK;
}

// Copies the term table into constant memory once per device.
int upload_terms() {
  static std::mutex mu;
  static bool done[64] = {false};
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return set_error(SFNL_ERR_CUDA, "no current device");
  std::lock_guard<std::mutex> lk(mu);
  if (!done[dev]) {
    if (cudaMemcpyToSymbol(c_terms, kTerms, sizeof(kTerms)) != cudaSuccess)
      return set_error(SFNL_ERR_CUDA, "upload of the program term table failed");
    done[dev] = true;
  }
  return SFNL_OK;
}

// The mapped status word, allocated on first use (pinned host memory, portable to every device).
int status_word(int **dev) {
  std::lock_guard<std::mutex> lk(g_status_mu);
  if (!g_status_host) {
    int *h = nullptr;
    if (cudaHostAlloc(reinterpret_cast<void **>(&h), sizeof(int), cudaHostAllocMapped | cudaHostAllocPortable) !=
        cudaSuccess) {
      cudaGetLastError();
      return set_error(SFNL_ERR_ALLOC, "pinned allocation of the split-form status word failed");
    }
    *h = 0;
    int *d = nullptr;
    if (cudaHostGetDevicePointer(reinterpret_cast<void **>(&d), h, 0) != cudaSuccess) {
      cudaGetLastError();
      cudaFreeHost(h);
      return set_error(SFNL_ERR_CUDA, "the split-form status word cannot be mapped");
    }
    g_status_host = h;
    g_status_dev = d;
  }
  *dev = g_status_dev;
  return SFNL_OK;
}

template <int PR>
int run_split_program(const ProgArgs &pa, int split, const int *in_map, const int *out_map, cudaStream_t st) {
  if (int rc = upload_terms()) return rc;
  SplitArgs sa;
  std::memset(&sa, 0, sizeof(sa));
  if (int rc = status_word(&sa.status)) return rc;
  if (!make_sgeo(pa.m, pr_pts(PR), pr_nin(PR), &sa.g)) return set_error(SFNL_ERR_UNSUPPORTED, "split form: m too large");
  STables T;
  int rc = get_stables(sa.g, &T);
  if (rc) return rc;
  sa.np = pa.np;
  sa.out_ps = pa.out_ps;
  sa.nsl = split;
  sa.bsyn = T.bsyn;
  sa.bana = T.bana;
  sa.bsyn_bytes = (int)T.bsyn_bytes;
  sa.bana_bytes = (int)T.bana_bytes;
  if (sa.g.off_bsyn[0][0] + sa.bsyn_bytes != sa.g.off_bana[0][0] || sa.g.off_bana[0][0] + sa.bana_bytes > sa.g.off_bar)
    return set_error(SFNL_ERR_UNSUPPORTED, "split form: table layout mismatch");
  switch (pa.m) {
    case 16: return launch_split_pr<PR, 16>(sa, pa.batch, pa, in_map, out_map, st);
    case 32: return launch_split_pr<PR, 32>(sa, pa.batch, pa, in_map, out_map, st);
    case 64: return launch_split_pr<PR, 64>(sa, pa.batch, pa, in_map, out_map, st);
    default: return launch_split_pr<PR, 0>(sa, pa.batch, pa, in_map, out_map, st);
  }
}

}  // namespace

bool split_supported(int op, int m) {
  if (m < 1 || m > 64 || !op_bilinear(op) || op == OP_ADVECT) return false;
  SGeo g;
  return make_sgeo(m, 8, 16, &g) && make_sgeo(m, 16, 8, &g) && make_sgeo(m, 32, 4, &g);
}

int launch_split(const ProgArgs &a, int split, cudaStream_t st) {
  if (a.np == 0) return SFNL_OK;
  static const int id[16] = {0, 1, 2, 3, 4, 5, 6, 7, 8, 9, 10, 11, 12, 13, 14, 15};
  switch (a.op) {
    case OP_BUNDLE: return run_split_program<PR_BUNDLE>(a, split, id, id, st);
    case OP_CROSS: return run_split_program<PR_CROSS>(a, split, id, id, st);
    case OP_DOT: return run_split_program<PR_DOT>(a, split, id, id, st);
    case OP_PROD: return run_split_program<PR_PROD>(a, split, id, id, st);
    case OP_CROSS_JVP: return run_split_program<PR_CJVP>(a, split, id, id, st);
    case OP_CROSS_VJP: return run_split_program<PR_CVJP>(a, split, id, id, st);
    case OP_MHD_VJP: return run_split_program<PR_MVJP>(a, split, id, id, st);
    case OP_SVECT: return run_split_program<PR_SVECT>(a, split, id, id, st);
    case OP_TENSOR: {  // [u, v] -> u_k v_l: one scalar x vector program per k, outputs 3k..3k+2
      for (int k = 0; k < 3; ++k) {
        const int in_k[4] = {3, 4, 5, k}, out_k[3] = {3 * k, 3 * k + 1, 3 * k + 2};
        if (int rc = run_split_program<PR_SVECT>(a, split, in_k, out_k, st)) return rc;
      }
      return SFNL_OK;
    }
    case OP_MHD_JVP: {  // [u, w, b, du, dw, db] -> two linearised cross products with disjoint outputs
      static const int in1[12] = {0, 1, 2, 3, 4, 5, 9, 10, 11, 12, 13, 14}, out1[3] = {0, 1, 2};
      static const int in2[12] = {0, 1, 2, 6, 7, 8, 9, 10, 11, 15, 16, 17}, out2[3] = {3, 4, 5};
      int rc = run_split_program<PR_CJVP>(a, split, in1, out1, st);
      if (rc) return rc;
      return run_split_program<PR_CJVP>(a, split, in2, out2, st);
    }
  }
  return set_error(SFNL_ERR_ARG, "unknown program");
}

int split_take_status() {
  std::lock_guard<std::mutex> lk(g_status_mu);
  if (!g_status_host) return 0;
  return __atomic_exchange_n(reinterpret_cast<volatile int *>(g_status_host), 0, __ATOMIC_SEQ_CST);
}

int wait_status_word(int **dev) { return status_word(dev); }

int split_inject_timeout() {
  int *d = nullptr;
  if (int rc = status_word(&d)) return rc;
  std::lock_guard<std::mutex> lk(g_status_mu);
  __atomic_store_n(reinterpret_cast<volatile int *>(g_status_host), 1, __ATOMIC_SEQ_CST);
  return SFNL_OK;
}

void split_release_tables() {
  std::lock_guard<std::mutex> lk(g_stab_mu);
  int prev = 0;
  cudaGetDevice(&prev);
  for (auto &kv : g_stabs) {
    cudaSetDevice(kv.first.first);
    cudaFree(kv.second.bsyn);
    cudaFree(kv.second.bana);
  }
  g_stabs.clear();
  cudaSetDevice(prev);
}

}  // namespace sfnl
