// sfnl_split.cu -- split-precision products on the tcgen05 tensor cores.
//
// Same mathematics as the FAST form (sfnl_fast.cu): the exact truncated
// product of fft_parallel.F90:147-665 evaluated on an internal alias-free
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
// Tile.  The 128 MMA rows are (field slot, point) pairs: 8 slots x 16 points
// for cross/dot (6 fields), 4 slots x 32 points for the scalar product.  A
// row's TMEM accumulators hold its field's four classes at all Q angles
// (8Q fp32 columns, 384 at m=64).  After the synthesis each thread folds its
// row to the 4Q physical angles in FP64 and the rows of one point meet in
// shared memory, 16 quarter-angles at a time, where the pointwise program
// runs; its folded products, sliced, are the A operand of the analysis,
// whose 128 rows are (output, point) pairs and which accumulates over the
// angle chunks in TMEM.
//
// One CTA of 4 warps per SM (or two when they fit), persistent over tiles.
// Thread 0 issues the MMAs; completion is signalled through an mbarrier
// whose waits are bounded (a timeout sets a status word and abandons the
// tile instead of spinning forever).
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
constexpr int kThreads = 128;

__device__ int g_split_status;   // 0 ok; 1 an mbarrier wait timed out

// ---------------------------------------------------------------------------
// geometry
// ---------------------------------------------------------------------------
struct SGeo {
  int m, Q, N, NC;
  int ke[4], Ks[4], No[4];      // modes per class, K padded to 16, output cols padded to 16
  int Ks_tot, No_tot;
  int tmem_cols, tmem_alloc;
  // shared-memory byte offsets (relative to the dynamic smem base)
  int off_asyn[4][3], off_bsyn[4][3], off_bana[4][3], off_x, off_aana[4][3], off_sum, off_bar, smem_bytes;
  int rs;  // analysis rows in use (outputs x points)
  int ana_col[4];
};

int pow2_at_least(int v) {
  int p = 32;
  while (p < v) p <<= 1;
  return p;
}

bool make_sgeo(int m, int nslots, int nin, int nout, SGeo *out) {
  SGeo g;
  std::memset(&g, 0, sizeof(g));
  g.m = m;
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
  const int pts = 128 / nslots;
  int asyn = 0;
  for (int c = 0; c < 4; ++c)
    for (int i = 0; i < 3; ++i) {
      g.off_asyn[c][i] = asyn;
      asyn += 128 * g.Ks[c] * 2;
    }
  const int xbytes = pts * nin * 64 * 8;
  int r1b = xbytes;
  for (int c = 0; c < 4; ++c)
    for (int i = 0; i < 3; ++i) {
      g.off_aana[c][i] = r1b;
      r1b += 128 * 16 * 2;
    }
  g.rs = nout * pts;
  g.off_sum = r1b;
  r1b += g.rs * g.No_tot * 8;
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

__device__ __forceinline__ void tmem_ld8(uint32_t taddr, float (&v)[8]) {
  uint32_t r[8];
  asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
               : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7])
               : "r"(taddr));
#pragma unroll
  for (int i = 0; i < 8; ++i) v[i] = __uint_as_float(r[i]);
}
__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

__device__ __forceinline__ uint32_t bf16_bits(double v) {
  return (uint32_t)__bfloat16_as_ushort(__float2bfloat16_rn((float)v));
}

// 2^e as a double (e clamped to the normal range).
__device__ __forceinline__ double pow2(int e) {
  e = e < -1022 ? -1022 : (e > 1023 ? 1023 : e);
  return __longlong_as_double((long long)(e + 1023) << 52);
}

// Slices of x relative to the row bound 2^E (E from frexp of the row max).
// Every step multiplies by an exact power of two, so h, mi, lo are exact.
__device__ __forceinline__ void slice3(double x, int E, double &h, double &mi, double &lo) {
  const double u0 = pow2(E - kW), i0 = pow2(kW - E);
  const double u1 = pow2(E - 2 * kW - 1), i1 = pow2(2 * kW + 1 - E);
  const double u2 = pow2(E - 3 * kW - 2), i2 = pow2(3 * kW + 2 - E);
  h = rint(x * i0) * u0;
  double r = x - h;
  mi = rint(r * i1) * u1;
  r -= mi;
  lo = rint(r * i2) * u2;
}

__device__ __forceinline__ int row_exponent(double mx) {
  int e = 0;
  frexp(mx, &e);  // mx = f 2^e, f in [0.5, 1) -> mx < 2^e
  return e;
}

struct SplitArgs {
  const double *in[6];
  double *out[3];
  int64_t in_ldm[6], out_ldm[3], in_bs[6], out_bs[3];
  int64_t np;
  int batch;
  unsigned adj_in;
  int adj_out, accumulate, nsl;
  SGeo g;
  const void *bsyn, *bana;
  int bsyn_bytes, bana_bytes;
};

template <int EK>
struct SDef;
template <>
struct SDef<EK_CROSS> {
  static constexpr int NI = 6, NO = 3, SLOTS = 8;
  __device__ static void op(const double *x, double *y) { cross3(x, x + 3, y); }
};
template <>
struct SDef<EK_DOT> {
  static constexpr int NI = 6, NO = 1, SLOTS = 8;
  __device__ static void op(const double *x, double *y) { y[0] = x[0] * x[3] + x[1] * x[4] + x[2] * x[5]; }
};
template <>
struct SDef<EK_PROD> {
  static constexpr int NI = 2, NO = 1, SLOTS = 4;
  __device__ static void op(const double *x, double *y) { y[0] = x[0] * x[1]; }
};

template <int EK>
__global__ void __launch_bounds__(kThreads, 1) split_kernel(const SplitArgs a) {
  constexpr int NI = SDef<EK>::NI, NO = SDef<EK>::NO, SLOTS = SDef<EK>::SLOTS, PTS = 128 / SLOTS;
  extern __shared__ __align__(128) unsigned char sm[];
  __shared__ uint32_t s_tmem;
  const SGeo &g = a.g;
  const int t = threadIdx.x, warp = t >> 5;
  const uint32_t mbar = smem_u32(sm + g.off_bar);

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
    const int n16 = a.bsyn_bytes / 16;
    for (int i = t; i < n16; i += kThreads) dst[i] = src[i];
    const uint4 *src2 = reinterpret_cast<const uint4 *>(a.bana);
    uint4 *dst2 = reinterpret_cast<uint4 *>(sm + g.off_bana[0][0]);
    const int n16b = a.bana_bytes / 16;
    for (int i = t; i < n16b; i += kThreads) dst2[i] = src2[i];
  }
  fence_async_smem();
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = s_tmem;
  const uint32_t lane_base = (uint32_t)(warp * 32) << 16;
  uint32_t phase = 0;
  bool ok = true;

  const int b = blockIdx.y;
  const int64_t ntiles = (a.np + PTS - 1) / PTS;
  const double invN = 1.0 / g.N, twoN = 2.0 / g.N;
  const int npairs = a.nsl == 3 ? 6 : 3;

  for (int64_t tile = blockIdx.x; tile < ntiles && ok; tile += gridDim.x) {
    // ---- 1. load + slice the input rows (row t = field slot f, point p) ----
    {
      const int f = t / PTS, p = t % PTS;
      const int64_t gp = tile * PTS + p;
      const bool valid = f < NI && gp < a.np;
      const double *src = valid ? a.in[f] + (int64_t)b * a.in_bs[f] + gp : nullptr;
      const double dsc = (f < NI && (a.adj_in >> f) & 1u) ? 1.0 : 0.0;  // 1: cotangent row
#pragma unroll 1
      for (int c = 0; c < 4; ++c) {
        double x[kKeMax];
        double mx = 0.0;
#pragma unroll
        for (int k = 0; k < kKeMax; ++k) {
          x[k] = 0.0;
          const int n = 2 * k + (c & 1);
          if (valid && k < g.ke[c] && !(c == 2 && n == 0)) {
            double v = __ldg(src + (int64_t)n * a.in_ldm[f] + (c >= 2 ? a.np : 0));
            if (dsc != 0.0) v *= (n == 0 ? invN : twoN);
            x[k] = v;
            mx = fmax(mx, fabs(v));
          }
        }
        const int E = row_exponent(mx);
        const int K = g.Ks[c];
#pragma unroll
        for (int kg = 0; kg < kKeMax / 8; ++kg) {
          if (kg * 8 >= K) break;
          uint32_t w[3][4];
#pragma unroll
          for (int q = 0; q < 4; ++q) {
            double s0[2], s1[2], s2[2];
#pragma unroll
            for (int e = 0; e < 2; ++e) {
              if (mx > 0.0)
                slice3(x[kg * 8 + 2 * q + e], E, s0[e], s1[e], s2[e]);
              else
                s0[e] = s1[e] = s2[e] = 0.0;
            }
            w[0][q] = bf16_bits(s0[0]) | (bf16_bits(s0[1]) << 16);
            w[1][q] = bf16_bits(s1[0]) | (bf16_bits(s1[1]) << 16);
            w[2][q] = bf16_bits(s2[0]) | (bf16_bits(s2[1]) << 16);
          }
          const size_t off = (size_t)(t / 8) * (16 * K) + (size_t)kg * 128 + (size_t)(t % 8) * 16;
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
      const uint32_t idesc = make_idesc(g.Q);
      static const int pi_[6] = {0, 0, 1, 0, 1, 2}, pj_[6] = {0, 1, 0, 2, 1, 0};
      for (int c = 0; c < 4; ++c) {
        const uint32_t sbo = 16 * g.Ks[c];
        for (int s = 0; s < g.Ks[c] / 16; ++s)
          for (int pr = 0; pr < npairs; ++pr) {
            const int i = pi_[pr], j = pj_[pr];
            const int accn = (i + j == 0) ? 0 : 1;
            const uint32_t dcol = tmem + (uint32_t)((c * 2 + accn) * g.Q);
            const uint64_t ad = make_sdesc(smem_u32(sm + g.off_asyn[c][i]) + 256 * s, 128, sbo);
            const uint64_t bd = make_sdesc(smem_u32(sm + g.off_bsyn[c][j]) + 256 * s, 128, sbo);
            const uint32_t en = (s > 0 || (accn == 1 && pr > 1)) ? 1u : 0u;
            umma_bf16(dcol, ad, bd, idesc, en);
          }
      }
      umma_commit(mbar);
    }
    __syncwarp();
    if (!mbar_wait(mbar, phase)) {
      ok = false;
      g_split_status = 1;
    }
    phase ^= 1;
    tc_fence_after();

    double *X = reinterpret_cast<double *>(sm + g.off_x);  // [f][quadrant][16][p], point fastest
    double *sums = reinterpret_cast<double *>(sm + g.off_sum);  // [analysis column][row]
    // Adds the analysis of one chunk (TMEM, fp32) to the FP64 sums of the thread's row.
    auto add_chunk = [&](int chk) {
#pragma unroll 1
      for (int col = 0; col < g.No_tot; col += 8) {
        float v[8];
        tmem_ld8(tmem + lane_base + (uint32_t)(8 * g.Q + col), v);
        tmem_wait_ld();
        if (t < g.rs) {
#pragma unroll
          for (int e = 0; e < 8; ++e) {
            double *sp = sums + (size_t)(col + e) * g.rs + t;
            *sp = (chk == 0 ? 0.0 : *sp) + (double)v[e];
          }
        }
      }
    };
    for (int ch = 0; ch < g.NC && ok; ++ch) {
      // ---- 3a. read out, recombine in FP64, fold to the 4 quadrant angles ----
      {
        const int f = t / PTS, p = t % PTS;
#pragma unroll 1
        for (int h = 0; h < 2; ++h) {
          float d[4][2][8];
#pragma unroll
          for (int c = 0; c < 4; ++c)
#pragma unroll
            for (int ac = 0; ac < 2; ++ac)
              tmem_ld8(tmem + lane_base + (uint32_t)((c * 2 + ac) * g.Q + ch * 16 + h * 8), d[c][ac]);
          tmem_wait_ld();
          if (f < NI) {
            double *xr = X + (size_t)f * 64 * PTS + p;
#pragma unroll
            for (int jj = 0; jj < 8; ++jj) {
              const double CE = (double)d[0][0][jj] + (double)d[0][1][jj];
              const double CO = (double)d[1][0][jj] + (double)d[1][1][jj];
              const double SE = (double)d[2][0][jj] + (double)d[2][1][jj];
              const double SO = (double)d[3][0][jj] + (double)d[3][1][jj];
              const double A = CE + CO, B = CE - CO, C = SE + SO, D = SO - SE;
              const int j = h * 8 + jj;
              xr[(0 * 16 + j) * PTS] = A + C;  // theta
              xr[(1 * 16 + j) * PTS] = B + D;  // pi - theta
              xr[(2 * 16 + j) * PTS] = B - D;  // pi + theta
              xr[(3 * 16 + j) * PTS] = A - C;  // 2 pi - theta
            }
          }
        }
      }
      tc_fence_before();
      __syncthreads();
      // The previous chunk's analysis must be complete: fold it into the FP64 sums.
      if (ch > 0) {
        if (!mbar_wait(mbar, phase)) {
          ok = false;
          g_split_status = 1;
        }
        phase ^= 1;
        tc_fence_after();
        add_chunk(ch - 1);
      }
      // ---- 3b. pointwise program, analysis pre-fold, slicing (row t = output o, point p) ----
      if (t < NO * PTS) {
        const int o = t / PTS, p = t % PTS;
        double P[4][16];
#pragma unroll
        for (int j = 0; j < 16; ++j) {
          double gq[4];
#pragma unroll
          for (int r = 0; r < 4; ++r) {
            double xv[NI], yv[NO];
#pragma unroll
            for (int f = 0; f < NI; ++f) xv[f] = X[((size_t)(f * 4 + r) * 16 + j) * PTS + p];
            SDef<EK>::op(xv, yv);
            gq[r] = yv[0];
#pragma unroll
            for (int oo = 1; oo < NO; ++oo)
              if (oo == o) gq[r] = yv[oo];
          }
          const double s14 = gq[0] + gq[3], d14 = gq[0] - gq[3], s23 = gq[1] + gq[2], d32 = gq[2] - gq[1];
          P[0][j] = s14 + s23;
          P[1][j] = s14 - s23;
          P[2][j] = d14 + d32;
          P[3][j] = d14 - d32;
        }
#pragma unroll
        for (int c = 0; c < 4; ++c) {
          double mx = 0.0;
#pragma unroll
          for (int j = 0; j < 16; ++j) mx = fmax(mx, fabs(P[c][j]));
          const int E = row_exponent(mx);
#pragma unroll
          for (int kg = 0; kg < 2; ++kg) {
            uint32_t w[3][4];
#pragma unroll
            for (int q = 0; q < 4; ++q) {
              double s0[2], s1[2], s2[2];
#pragma unroll
              for (int e = 0; e < 2; ++e) {
                if (mx > 0.0)
                  slice3(P[c][kg * 8 + 2 * q + e], E, s0[e], s1[e], s2[e]);
                else
                  s0[e] = s1[e] = s2[e] = 0.0;
              }
              w[0][q] = bf16_bits(s0[0]) | (bf16_bits(s0[1]) << 16);
              w[1][q] = bf16_bits(s1[0]) | (bf16_bits(s1[1]) << 16);
              w[2][q] = bf16_bits(s2[0]) | (bf16_bits(s2[1]) << 16);
            }
            const size_t off = (size_t)(t / 8) * 256 + (size_t)kg * 128 + (size_t)(t % 8) * 16;
#pragma unroll
            for (int i = 0; i < 3; ++i)
              *reinterpret_cast<uint4 *>(sm + g.off_aana[c][i] + off) = make_uint4(w[i][0], w[i][1], w[i][2], w[i][3]);
          }
        }
      }
      fence_async_smem();
      tc_fence_before();
      __syncthreads();
      // ---- 3c. analysis MMAs for this chunk (corrections first, then hi x hi) ----
      if (t == 0 && ok) {
        tc_fence_after();
        static const int qi_[6] = {0, 1, 0, 1, 2, 0}, qj_[6] = {1, 0, 2, 1, 0, 0};
        static const int ri_[3] = {0, 1, 0}, rj_[3] = {1, 0, 0};
        for (int c = 0; c < 4; ++c) {
          const uint32_t idesc = make_idesc(g.No[c]);
          const uint32_t dcol = tmem + (uint32_t)g.ana_col[c];
          for (int pr = 0; pr < npairs; ++pr) {
            const int i = a.nsl == 3 ? qi_[pr] : ri_[pr], j = a.nsl == 3 ? qj_[pr] : rj_[pr];
            const uint64_t ad = make_sdesc(smem_u32(sm + g.off_aana[c][i]), 128, 256);
            const uint64_t bd = make_sdesc(smem_u32(sm + g.off_bana[c][j]) + 256 * ch, 128, 16 * g.Q);
            const uint32_t en = pr > 0 ? 1u : 0u;  // each chunk starts a fresh accumulator
            umma_bf16(dcol, ad, bd, idesc, en);
          }
        }
        umma_commit(mbar);
      }
      __syncwarp();
    }
    // ---- 4. last chunk into the sums, then the store: row t = (output o, point p) ----
    if (ok) {
      if (!mbar_wait(mbar, phase)) {
        ok = false;
        g_split_status = 1;
      }
      phase ^= 1;
    }
    tc_fence_after();
    if (ok) add_chunk(g.NC - 1);
    __syncthreads();
    if (ok) {
      // rows t = o*PTS + p; a warp covers 32 consecutive rows -> consecutive points of one output
      for (int idx = t; idx < g.rs * g.No_tot; idx += kThreads) {
        const int row = idx % g.rs, col = idx / g.rs;
        const int o = row / PTS, p = row % PTS;
        int c = 0;
        while (c < 3 && col >= g.ana_col[c + 1] - 8 * g.Q) ++c;
        const int kk = col - (g.ana_col[c] - 8 * g.Q);
        const int64_t gp = tile * PTS + p;
        if (kk >= g.ke[c] || gp >= a.np) continue;
        const int n = 2 * kk + (c & 1);
        const double sc = a.adj_out ? 1.0 : (n == 0 ? invN : twoN);
        const double val = (c == 2 && n == 0) ? 0.0 : sums[idx] * sc;
        double *q = a.out[o] + (int64_t)b * a.out_bs[o] + gp + (int64_t)n * a.out_ldm[o] + (c >= 2 ? a.np : 0);
        if (a.accumulate)
          *q += val;
        else
          *q = val;
      }
    }
    tc_fence_before();
    __syncthreads();
  }
  __syncthreads();
  if (warp == 0) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(g.tmem_alloc));
  }
}

template <int EK>
int launch_split_ek(SplitArgs &sa, cudaStream_t st) {
  constexpr int SLOTS = SDef<EK>::SLOTS, PTS = 128 / SLOTS;
  auto kern = split_kernel<EK>;
  if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, sa.g.smem_bytes) != cudaSuccess)
    return set_error(SFNL_ERR_CUDA, "cudaFuncSetAttribute failed (split form)");
  const int64_t ntiles = (sa.np + PTS - 1) / PTS;
  // Keep the per-SM TMEM demand within its 512 columns: at most 512/alloc CTAs per SM,
  // also bounded by shared memory.
  int per_sm_tmem = 512 / sa.g.tmem_alloc;
  int per_sm_smem = (int)((228 * 1024) / (sa.g.smem_bytes + 1024));
  int per_sm = per_sm_tmem < per_sm_smem ? per_sm_tmem : per_sm_smem;
  if (per_sm < 1) per_sm = 1;
  int64_t grid = (int64_t)num_sms() * per_sm;
  if (grid > ntiles) grid = ntiles;
  if (grid < 1) grid = 1;
  dim3 gdim((unsigned)grid, (unsigned)sa.batch);
  kern<<<gdim, kThreads, sa.g.smem_bytes, st>>>(sa);
  return check_launch("split form");
}

}  // namespace

bool split_supported(int op, int m) {
  (void)op;
  if (m < 1 || m > 64) return false;
  SGeo g;
  return make_sgeo(m, 8, 6, 3, &g) && make_sgeo(m, 8, 6, 1, &g) && make_sgeo(m, 4, 2, 1, &g);
}

int launch_split(const ProgArgs &a, int split, cudaStream_t st) {
  if (a.np == 0) return SFNL_OK;
  std::vector<Elem> seq;
  int rc = decompose_program(a.op, seq);
  if (rc) return rc;
  const bool adj_out = op_adjoint_out(a.op);
  for (const Elem &e : seq) {
    const int nslots = e.ek == EK_PROD ? 4 : 8, nin = e.ek == EK_PROD ? 2 : 6, nout = e.ek == EK_CROSS ? 3 : 1;
    SplitArgs sa;
    std::memset(&sa, 0, sizeof(sa));
    if (!make_sgeo(a.m, nslots, nin, nout, &sa.g)) return set_error(SFNL_ERR_UNSUPPORTED, "split form: m too large");
    STables T;
    rc = get_stables(sa.g, &T);
    if (rc) return rc;
    const int no = e.ek == EK_CROSS ? 3 : 1;
    for (int i = 0; i < nin; ++i) {
      sa.in[i] = a.in[e.in[i]];
      sa.in_ldm[i] = a.in_ldm[e.in[i]];
      sa.in_bs[i] = a.in_bs[e.in[i]];
    }
    for (int o = 0; o < no; ++o) {
      sa.out[o] = a.out[e.out[o]];
      sa.out_ldm[o] = a.out_ldm[e.out[o]];
      sa.out_bs[o] = a.out_bs[e.out[o]];
    }
    sa.np = a.np;
    sa.batch = a.batch;
    sa.adj_in = e.adj;
    sa.adj_out = adj_out ? 1 : 0;
    sa.accumulate = e.acc;
    sa.nsl = split;
    sa.bsyn = T.bsyn;
    sa.bana = T.bana;
    sa.bsyn_bytes = (int)T.bsyn_bytes;
    sa.bana_bytes = (int)T.bana_bytes;
    if (sa.g.off_bsyn[0][0] + sa.bsyn_bytes != sa.g.off_bana[0][0] || sa.g.off_bana[0][0] + sa.bana_bytes > sa.g.off_bar)
      return set_error(SFNL_ERR_UNSUPPORTED, "split form: table layout mismatch");
    rc = e.ek == EK_CROSS ? launch_split_ek<EK_CROSS>(sa, st)
       : e.ek == EK_DOT   ? launch_split_ek<EK_DOT>(sa, st)
                          : launch_split_ek<EK_PROD>(sa, st);
    if (rc) return rc;
  }
  return SFNL_OK;
}

int split_status_and_clear() {
  int h = 0, z = 0;
  if (cudaMemcpyFromSymbol(&h, g_split_status, sizeof(int)) != cudaSuccess) return -1;
  cudaMemcpyToSymbol(g_split_status, &z, sizeof(int));
  return h;
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
