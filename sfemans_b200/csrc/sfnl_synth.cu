// sfnl_synth.cu -- synthesis-only routines on the caller's grid.
//
//   FFT_PAR_REAL     (fft_parallel.F90:28-145)     values of every field at theta_j = 2 pi j / N
//   FFT_MAX_VEL_DCL  (fft_parallel.F90:1426-1541)  max over points and angles of |v|
//
// Both evaluate f(theta) = a_0 + sum_{n<m} a_n cos(n theta) + b_n sin(n theta) (the c2r of the
// half-complex pack of :88-112, :1497-1511, whose sine of mode 0 is ignored) on the N = 2*m_max_pad-1
// angles of the reference grid.  The mirror symmetry of that grid, theta_{N-j} = 2 pi - theta_j, is
// folded out: with C_j the cosine part and S_j the sine part at angle j, f_j = C_j + S_j and
// f_{N-j} = C_j - S_j, so each warp evaluates (N+1)/2 angles.
//
// Parallel decomposition: one warp per point (as the GRID form).  The point's coefficients are staged
// in shared memory and read as broadcasts; lanes own angles, with an exact cos/sin table of
// 2 pi r / N indexed by n*j mod N.  FFT_PAR_REAL writes the angles of one field contiguously
// (V_out(N, nf, np), angle fastest); FFT_MAX_VEL_DCL reduces |v| (the first 3-vector when there are
// six slots, |first field| otherwise, :1527-1532) to one maximum per point (host entry: the points'
// maxima are reduced on the host) or per launch with an integer atomic max on the bit patterns
// (device entry: non-negative doubles order like their bits, and a NaN wins, as it propagates).
#include <cuda_runtime.h>

#include "sfnl_internal.h"

namespace sfnl {

namespace {

constexpr int kSynthThreads = 128;

// MODE 0: grid values to out (N, nslot/2, np); 1: maximum of |v| into *vmax (atomic); 2: maximum of
// |v| of each point to out[p].
template <int MODE>
__global__ void __launch_bounds__(kSynthThreads) synth_kernel(const double *v, double *out, unsigned long long *vmax,
                                                              int64_t np, int nslot, int m, int N, int warps_per_cta) {
  constexpr bool MAXV = MODE != 0;
  extern __shared__ __align__(16) double smem[];
  const int nf = nslot / 2;
  double2 *tab = reinterpret_cast<double2 *>(smem);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  double *X = smem + 2 * N + (size_t)warp * nslot * m;  // X[f][0..m) cos, X[f][m..2m) sin
  for (int r = threadIdx.x; r < N; r += blockDim.x) {
    double s, c;
    sincospi(2.0 * (double)r / (double)N, &s, &c);
    tab[r] = make_double2(c, s);
  }
  __syncthreads();
  if (warp >= warps_per_cta) return;
  const int nh = (N + 1) / 2;  // angles 0..nh-1 and their mirrors N-j
  double vm = 0.0;
  for (int64_t p = (int64_t)blockIdx.x * warps_per_cta + warp; p < np; p += (int64_t)gridDim.x * warps_per_cta) {
    for (int idx = lane; idx < nslot * m; idx += 32) {
      const int f = idx / (2 * m), k = idx - f * 2 * m;
      const int n = k < m ? k : k - m;
      // cos of mode n of field f is slot 2f, sine slot 2f+1; the sine of mode 0 is ignored
      X[idx] = (k == m) ? 0.0 : __ldg(v + p + (int64_t)np * ((k < m ? 2 * f : 2 * f + 1) + (int64_t)nslot * n));
    }
    __syncwarp();
    const int nfe = MAXV ? (nslot == 6 ? 3 : 1) : nf;  // fields that matter
    for (int j = lane; j < nh; j += 32) {
      double fp[3] = {0.0, 0.0, 0.0}, fm[3] = {0.0, 0.0, 0.0};
      for (int f = 0; f < nfe; ++f) {
        const double *xc = X + (size_t)f * 2 * m, *xs = xc + m;
        double C = 0.0, S = 0.0;
        int r = 0;  // n*j mod N
        for (int n = 0; n < m; ++n) {
          const double2 cs = tab[r];
          C = fma(xc[n], cs.x, C);
          S = fma(xs[n], cs.y, S);
          r += j;
          if (r >= N) r -= N;
        }
        if constexpr (MAXV) {
          fp[f] = C + S;
          fm[f] = C - S;
        } else {
          double *o = out + (size_t)N * (f + (int64_t)nf * p);
          o[j] = C + S;
          if (j > 0) o[N - j] = C - S;
        }
      }
      if constexpr (MAXV) {
        const double a = sqrt(fp[0] * fp[0] + fp[1] * fp[1] + fp[2] * fp[2]);
        const double bm = sqrt(fm[0] * fm[0] + fm[1] * fm[1] + fm[2] * fm[2]);
        vm = fmax(vm, a);
        if (j > 0) vm = fmax(vm, bm);
      }
    }
    if constexpr (MODE == 2) {
      for (int off = 16; off > 0; off >>= 1) vm = fmax(vm, __shfl_xor_sync(0xffffffffu, vm, off));
      if (lane == 0) out[p] = vm;
      vm = 0.0;
    }
    __syncwarp();
  }
  if constexpr (MODE == 1) {
    for (int off = 16; off > 0; off >>= 1) vm = fmax(vm, __shfl_xor_sync(0xffffffffu, vm, off));
    if (lane == 0) atomicMax(vmax, (unsigned long long)__double_as_longlong(vm));
  }
}

template <int MODE>
int launch_synth(const double *v, double *out, double *vmax, int64_t np, int nslot, int m, int N, cudaStream_t st) {
  const size_t tab_bytes = sizeof(double) * 2 * (size_t)N, per_warp = sizeof(double) * (size_t)nslot * m;
  const size_t budget = 200 * 1024;
  if (tab_bytes + per_warp > budget) return set_error(SFNL_ERR_UNSUPPORTED, "synthesis: m or N too large for shared memory");
  int warps = (int)((budget - tab_bytes) / per_warp);
  if (warps > kSynthThreads / 32) warps = kSynthThreads / 32;
  const size_t smem = tab_bytes + per_warp * warps;
  auto kern = synth_kernel<MODE>;
  if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess)
    return set_error(SFNL_ERR_CUDA, "cudaFuncSetAttribute failed (synthesis)");
  int64_t blocks = (np + warps - 1) / warps;
  const int64_t cap = (int64_t)num_sms() * 16;
  if (blocks > cap) blocks = cap;
  if (blocks < 1) blocks = 1;
  kern<<<(unsigned)blocks, kSynthThreads, smem, st>>>(v, out, reinterpret_cast<unsigned long long *>(vmax), np, nslot,
                                                      m, N, warps);
  return check_launch("synthesis");
}

}  // namespace

int launch_real(const double *v, double *out, int64_t np, int nslot, int m, int N, cudaStream_t st) {
  if (np == 0) return SFNL_OK;
  return launch_synth<0>(v, out, nullptr, np, nslot, m, N, st);
}

// vmax: device double, not reset here (the caller zeroes it first)
int launch_max_vel(const double *v, double *vmax, int64_t np, int nslot, int m, int N, cudaStream_t st) {
  if (np == 0) return SFNL_OK;
  return launch_synth<1>(v, nullptr, vmax, np, nslot, m, N, st);
}

int launch_point_max_vel(const double *v, double *pmax, int64_t np, int nslot, int m, int N, cudaStream_t st) {
  if (np == 0) return SFNL_OK;
  return launch_synth<2>(v, pmax, nullptr, np, nslot, m, N, st);
}

}  // namespace sfnl
