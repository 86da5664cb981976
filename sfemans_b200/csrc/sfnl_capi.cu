// sfnl_capi.cu -- the extern "C" boundary (include/sfemans_nl.h).
//
// Validates arguments the way the reference does (fft_parallel.F90:184-191:
// nb_field even, m_max_c > 0; the buffers of :163-171 bound np by
// nb_procs*bloc_size and the padded modes by m_max_pad), describes each call
// as a program over scalar fields (sfnl_ops.cuh) and dispatches it to one of
// the kernel families:
//   GRID  sfnl_grid.cu   dense FP64 DFT on the caller's grid (any N)
//   FAST  sfnl_fast.cu   FP64 factored transforms on an internal alias-free grid
//   SPLIT sfnl_split.cu  bf16-sliced tcgen05 contractions, FP64 recombination
#include <cuda_runtime.h>

#include <atomic>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/sfemans_nl.h"
#include "sfnl_internal.h"
#include "sfnl_ops.cuh"

namespace sfnl {

namespace {
thread_local std::string g_err = "no error";
thread_local double g_host_timing[3] = {0, 0, 0};
int g_check_finite = 0;
std::atomic<int> g_bundle_kernel{SFNL_BUNDLE_RESIDUE};

struct DevState {
  int sms = 0;
  int *d_flag = nullptr;
  char *work = nullptr;
  size_t work_bytes = 0;
  char *gwork = nullptr;  // Gauss-point operands (device entry without a caller workspace, host entry)
  size_t gwork_bytes = 0;
  std::mutex mu;       // workspaces (held for a whole host call)
  std::mutex flag_mu;  // the finite-check flag (taken inside host calls too)
};

// Grows the per-device Gauss-point buffer to `bytes` (caller holds s->mu).
int grow_gwork(DevState *s, size_t bytes) {
  if (bytes <= s->gwork_bytes) return SFNL_OK;
  if (s->gwork) cudaFree(s->gwork);
  s->gwork = nullptr;
  s->gwork_bytes = 0;
  if (cudaMalloc(&s->gwork, bytes) != cudaSuccess) {
    cudaGetLastError();
    return set_error(SFNL_ERR_ALLOC, "cudaMalloc of the Gauss-point workspace failed");
  }
  s->gwork_bytes = bytes;
  return SFNL_OK;
}
constexpr int kMaxDev = 64;
DevState g_dev[kMaxDev];
std::mutex g_dev_mu;

DevState *dev_state() {
  int d = 0;
  if (cudaGetDevice(&d) != cudaSuccess || d < 0 || d >= kMaxDev) return nullptr;
  return &g_dev[d];
}
}  // namespace

int set_error(int code, const char *msg) {
  g_err = msg;
  return code;
}

int check_launch(const char *what) {
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    g_err = std::string(what) + ": " + cudaGetErrorString(e);
    return SFNL_ERR_CUDA;
  }
  return SFNL_OK;
}

int num_sms() {
  DevState *s = dev_state();
  if (!s) return 148;
  std::lock_guard<std::mutex> lk(g_dev_mu);
  if (s->sms == 0) {
    int d = 0, v = 0;
    cudaGetDevice(&d);
    cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, d);
    s->sms = v > 0 ? v : 148;
  }
  return s->sms;
}

namespace {

__global__ void finite_scan(const double *p, int64_t n, int *flag) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    if (!isfinite(p[i])) {
      *flag = 1;
      return;
    }
}

int scan_outputs(const ProgArgs &a, cudaStream_t st) {
  DevState *s = dev_state();
  if (!s) return set_error(SFNL_ERR_CUDA, "no current device");
  std::lock_guard<std::mutex> lk(s->flag_mu);
  if (!s->d_flag && cudaMalloc(&s->d_flag, sizeof(int)) != cudaSuccess)
    return set_error(SFNL_ERR_ALLOC, "cudaMalloc of the finite-check flag failed");
  if (cudaMemsetAsync(s->d_flag, 0, sizeof(int), st) != cudaSuccess) return set_error(SFNL_ERR_CUDA, "memset failed");
  const int no = op_nout(a.op);
  for (int o = 0; o < no; ++o) {
    // Each output field is a strided set of (cos,sin) rows; scan the span each row covers
    // (with a point stride of 3 the span also holds the other two tensor rows, all outputs).
    for (int b = 0; b < a.batch; ++b)
      for (int n = 0; n < a.m; ++n) {
        const double *row = a.out[o] + (int64_t)b * a.out_bs[o] + (int64_t)n * a.out_ldm[o];
        finite_scan<<<32, 256, 0, st>>>(row, (2 * a.np - 1) * a.out_ps + 1, s->d_flag);
      }
  }
  int h = 0;
  if (cudaMemcpyAsync(&h, s->d_flag, sizeof(int), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
      cudaStreamSynchronize(st) != cudaSuccess)
    return set_error(SFNL_ERR_CUDA, "finite check failed");
  return h ? set_error(SFNL_ERR_NONFINITE, "non-finite value in the output") : SFNL_OK;
}

// ---------------------------------------------------------------------------
// argument checks shared by all forms
// ---------------------------------------------------------------------------
int check_common(int64_t np, int m, int pad, int n_theta, int k_batch, int *N_out) {
  if (np < 0) return set_error(SFNL_ERR_ARG, "np < 0");
  if (m < 1) return set_error(SFNL_ERR_ARG, "m_max < 1 (the reference stops on m_max_c==0)");
  if (k_batch < 1 || k_batch > 65535) return set_error(SFNL_ERR_ARG, "k_batch outside [1, 65535]");
  if (pad < m) return set_error(SFNL_ERR_ALIAS, "m_max_pad < m_max: the padded spectrum cannot hold the modes");
  if (m > 4096 || pad > (1 << 20)) return set_error(SFNL_ERR_UNSUPPORTED, "m_max or m_max_pad beyond this library's limits");
  const int N = n_theta > 0 ? n_theta : 2 * pad - 1;
  if (m > N / 2 + 1) return set_error(SFNL_ERR_ALIAS, "grid shorter than 2*m_max-1 angles");
  *N_out = N;
  return SFNL_OK;
}

bool dealiased(int m, int N) { return N >= 3 * m - 2; }

// Field of a Fortran array V(np, nslot, m[, k]): component k -> slots 2k, 2k+1.
void set_in(ProgArgs &a, int f, const double *base, int64_t np, int nslot, int comp, int m, bool batched) {
  a.in[f] = base + (int64_t)2 * comp * np;
  a.in_ldm[f] = np * nslot;
  a.in_bs[f] = batched ? np * nslot * (int64_t)m : 0;
}
void set_out(ProgArgs &a, int o, double *base, int64_t np, int nslot, int comp, int m, bool batched) {
  a.out[o] = base + (int64_t)2 * comp * np;
  a.out_ldm[o] = np * nslot;
  a.out_bs[o] = batched ? np * nslot * (int64_t)m : 0;
}

ProgArgs make_args(int op, int64_t np, int m, int N, int batch) {
  ProgArgs a;
  std::memset(&a, 0, sizeof(a));
  a.op = op;
  a.np = np;
  a.m = m;
  a.N = N;
  a.batch = batch;
  a.out_ps = 1;
  return a;
}

int timeout_error();

int run_fp64(ProgArgs a, int algo, int N_caller, cudaStream_t st) {
  const bool alias_free = dealiased(a.m, N_caller);
  if (algo == SFNL_ALGO_AUTO)
    algo = (alias_free && op_bilinear(a.op) && fast_supported(a.op, a.m, fast_grid_length(a.m))) ? SFNL_ALGO_FAST
                                                                                                 : SFNL_ALGO_GRID;
  int rc;
  if (algo == SFNL_ALGO_GRID) {
    a.N = N_caller;
    rc = launch_grid(a, st);
  } else if (algo == SFNL_ALGO_FAST) {
    if (!op_bilinear(a.op))
      return set_error(SFNL_ERR_UNSUPPORTED, "FAST form: quotients and the tension tensor depend on the grid (use GRID)");
    if (!alias_free) return set_error(SFNL_ERR_ALIAS, "FAST form needs a dealiasing pad (2*m_max_pad-1 >= 3*m_max-2)");
    a.N = fast_grid_length(a.m);
    if (!fast_supported(a.op, a.m, a.N)) return set_error(SFNL_ERR_UNSUPPORTED, "FAST form not built for this size");
    // the MHD bundle's bounded waits report through the same word as the split kernels' (see run_split)
    if (a.op == OP_BUNDLE && split_take_status()) return timeout_error();
    rc = launch_fast(a, st);
  } else {
    return set_error(SFNL_ERR_ARG, "unknown algo");
  }
  if (rc == SFNL_OK && g_check_finite) rc = scan_outputs(a, st);
  if (rc == SFNL_OK && g_check_finite && a.op == OP_BUNDLE && split_take_status()) rc = timeout_error();
  return rc;
}

int timeout_error() {
  return set_error(SFNL_ERR_TIMEOUT,
                   "a kernel gave up a bounded wait (a split-form kernel on its tensor-core operations, or the FAST "
                   "MHD bundle on its bulk copies): the outputs of that call are incomplete");
}

int run_split(ProgArgs a, int split, int N_caller, cudaStream_t st) {
  if (split != SFNL_SPLIT_BF16X2 && split != SFNL_SPLIT_BF16X3) return set_error(SFNL_ERR_ARG, "split must be 2 or 3");
  if (!op_bilinear(a.op))
    return set_error(SFNL_ERR_UNSUPPORTED, "split forms: quotients and the tension tensor depend on the grid (use GRID)");
  if (!dealiased(a.m, N_caller)) return set_error(SFNL_ERR_ALIAS, "split forms need a dealiasing pad (2*m_max_pad-1 >= 3*m_max-2)");
  if (!split_supported(a.op, a.m)) return set_error(SFNL_ERR_UNSUPPORTED, "split form not built for this program/size");
  // The split kernels report a bounded wait that gave up through a mapped status word; the device entry
  // points do not synchronise, so a failure of an earlier call surfaces at the next split call (or after
  // the synchronisation of a host-array call or of the finite-check mode).
  if (split_take_status()) return timeout_error();
  int rc = launch_split(a, split, st);
  if (rc == SFNL_OK && g_check_finite) rc = scan_outputs(a, st);
  if (rc == SFNL_OK && g_check_finite && split_take_status()) rc = timeout_error();
  return rc;
}

// The products of fft_parallel.F90 by library op code (SFNL_OP_*): internal program, slots of the
// first and second input, and output slots (6 with tensor_out: the layout V(3, np, 6, m)).
struct ProductKind {
  int op, nsl_a, nsl_b, nsl_out;
  bool tensor_out;
};
constexpr ProductKind kProducts[8] = {
    {OP_CROSS, 6, 6, 6, false},  {OP_DOT, 6, 6, 2, false},   {OP_PROD, 2, 2, 2, false},
    {OP_DIV, 2, 2, 2, false},    {OP_SVECT, 6, 2, 6, false}, {OP_SVDIV, 6, 2, 6, false},
    {OP_TENSOR, 6, 6, 6, true},  {OP_TENSION, 6, 6, 6, true}};
constexpr int kNumProducts = 8;

int build_product(int op, const double *x, const double *y, double *out, int64_t np, int m, int N, ProgArgs *pa) {
  if (op < 0 || op >= kNumProducts) return set_error(SFNL_ERR_ARG, "op must be one of SFNL_OP_* (0..7)");
  if (np > 0 && (!x || !y || !out)) return set_error(SFNL_ERR_ARG, "null array");
  const ProductKind &pk = kProducts[op];
  ProgArgs a = make_args(pk.op, np, m, N, 1);
  const int na = pk.nsl_a / 2, nb = pk.nsl_b / 2;
  for (int k = 0; k < na; ++k) set_in(a, k, x, np, pk.nsl_a, k, m, false);
  for (int k = 0; k < nb; ++k) set_in(a, na + k, y, np, pk.nsl_b, k, m, false);
  if (pk.tensor_out) {
    // V_out(k, p, 2l-1:2l, n) holds the coefficients of u_k v_l (fft_parallel.F90:1786-1787).
    for (int k = 0; k < 3; ++k)
      for (int l = 0; l < 3; ++l) {
        const int o = 3 * k + l;
        a.out[o] = out + k + (int64_t)3 * 2 * l * np;
        a.out_ldm[o] = (int64_t)3 * 6 * np;
        a.out_bs[o] = 0;
      }
    a.out_ps = 3;
  } else {
    for (int o = 0; o < op_nout(pk.op); ++o) set_out(a, o, out, np, pk.nsl_out, o, m, false);
  }
  *pa = a;
  return SFNL_OK;
}

int build_bundle(const double *u, const double *w, const double *b, const double *j, const double *gt, double *uxw,
                 double *uxb, double *jxb, double *ugt, int64_t np, int m, int N, ProgArgs *pa) {
  if (np > 0 && (!u || !w || !b || !j || !gt || !uxw || !uxb || !jxb || !ugt)) return set_error(SFNL_ERR_ARG, "null array");
  ProgArgs a = make_args(OP_BUNDLE, np, m, N, 1);
  const double *ins[5] = {u, w, b, j, gt};
  for (int v = 0; v < 5; ++v)
    for (int k = 0; k < 3; ++k) set_in(a, 3 * v + k, ins[v], np, 6, k, m, false);
  double *outs[3] = {uxw, uxb, jxb};
  for (int v = 0; v < 3; ++v)
    for (int k = 0; k < 3; ++k) set_out(a, 3 * v + k, outs[v], np, 6, k, m, false);
  set_out(a, 9, ugt, np, 2, 0, m, false);
  *pa = a;
  return SFNL_OK;
}

// Linearised programs.  kind: 0 cross JVP, 1 cross VJP, 2 mhd JVP, 3 mhd VJP.
int build_linear(int kind, const double *u, const double *w, const double *b, const double *x, double *out, int64_t np,
                 int m, int N, int kb, ProgArgs *pa) {
  if (np > 0 && (!u || !w || !x || !out || (kind >= 2 && !b))) return set_error(SFNL_ERR_ARG, "null array");
  static const int ops[4] = {OP_CROSS_JVP, OP_CROSS_VJP, OP_MHD_JVP, OP_MHD_VJP};
  ProgArgs a = make_args(ops[kind], np, m, N, kb);
  const int nbase = kind >= 2 ? 3 : 2;
  const double *base[3] = {u, w, b};
  for (int v = 0; v < nbase; ++v)
    for (int k = 0; k < 3; ++k) set_in(a, 3 * v + k, base[v], np, 6, k, m, false);
  // batched input x: JVP tangents (6*nbase slots) or VJP cotangents (6*(nbase-1) slots)
  const int nx = (kind == 0) ? 12 : (kind == 1) ? 6 : (kind == 2) ? 18 : 12;
  const int ny = (kind == 0) ? 6 : (kind == 1) ? 12 : (kind == 2) ? 12 : 18;
  for (int k = 0; k < nx / 2; ++k) set_in(a, 3 * nbase + k, x, np, nx, k, m, true);
  for (int k = 0; k < ny / 2; ++k) set_out(a, k, out, np, ny, k, m, true);
  *pa = a;
  return SFNL_OK;
}

cudaStream_t as_stream(sfnl_stream_t s) { return reinterpret_cast<cudaStream_t>(s); }

// ---------------------------------------------------------------------------
// host-array plumbing: chunked copy/compute pipeline
//
// Every program is independent per point, so a host call streams the points
// through the GPU in chunks: chunk i is copied in (one cudaMemcpy2DAsync per
// array: a chunk of points is one strided segment per (slot, mode) row), its
// kernels run, and its result is copied out, on stream i % 3.  With pinned
// host memory the host-to-device copies, the kernels and the device-to-host
// copies of consecutive chunks overlap (two copy engines, full-duplex PCIe).
// Device memory: 3 chunk slots of a grow-only per-device workspace.
// ---------------------------------------------------------------------------
struct HostBuf {
  const void *src;  // host input (copied in) or nullptr
  void *dst;        // host output (copied out) or nullptr
  int nslot;        // slots of the Fortran array (np, nslot, m), or (ew, np, nslot, m)
  double *dev;      // device buffer of the current chunk, same layout with np_chunk points
  int ew = 1;       // leading extent (3 for the tensor layout V(3, np, 6, m))
  int mrows = 0;    // > 0: the array has nslot * mrows rows of points instead of nslot * m
};
size_t buf_rows(const HostBuf &b, int m) { return (size_t)b.nslot * (b.mrows > 0 ? b.mrows : m); }

constexpr int kPipe = 4;
constexpr size_t kChunkBytes = size_t(512) << 20;  // target bytes per chunk (inputs + outputs)

// Device-timed intervals of a host call: each interval is a pair of CUDA events on the stream that
// runs it, tagged 0 (host<->device copies) or 1 (kernels).  sum() adds the durations per tag after
// the streams have been synchronised.  The reference's temps(1) is the MPI_ALLTOALL time, temps(2)
// the FFTs and the product and temps(3) the repacking (fft_parallel.F90:203-290); here the copies
// stand where the all-to-alls stood, and nothing is repacked.
struct Intervals {
  std::vector<cudaEvent_t> ev;  // begin, end, begin, end, ...
  std::vector<int> tag;
  bool ok = true;
  int begin(cudaStream_t st) {
    cudaEvent_t a = nullptr, b = nullptr;
    if (cudaEventCreate(&a) != cudaSuccess || cudaEventCreate(&b) != cudaSuccess) {
      cudaGetLastError();
      if (a) cudaEventDestroy(a);
      ok = false;
      return -1;
    }
    ev.push_back(a);
    ev.push_back(b);
    tag.push_back(0);
    if (cudaEventRecord(a, st) != cudaSuccess) ok = false;
    return (int)tag.size() - 1;
  }
  void end(int i, cudaStream_t st, int t) {
    if (i < 0) return;
    tag[i] = t;
    if (cudaEventRecord(ev[2 * i + 1], st) != cudaSuccess) ok = false;
  }
  // Adds the seconds of each tag to s[0] (copies) and s[1] (kernels); false if any event failed.
  bool sum(double *s) {
    if (!ok) return false;
    for (size_t i = 0; i < tag.size(); ++i) {
      float ms = 0.f;
      if (cudaEventElapsedTime(&ms, ev[2 * i], ev[2 * i + 1]) != cudaSuccess) {
        cudaGetLastError();
        return false;
      }
      s[tag[i]] += 1e-3 * ms;
    }
    return true;
  }
  ~Intervals() {
    for (cudaEvent_t e : ev) cudaEventDestroy(e);
  }
};

// Publishes the copy and kernel seconds of a host call: to the thread's sfnl_last_host_timing record
// and, when given, to the reference's temps(3) (zeroed on entry by the callers, then added to).
void report_timing(Intervals &iv, double *temps) {
  double s[2] = {0.0, 0.0};
  if (!iv.sum(s)) s[0] = s[1] = 0.0;
  g_host_timing[0] = s[0];
  g_host_timing[1] = s[1];
  g_host_timing[2] = 0.0;
  if (temps) {
    temps[0] += s[0];
    temps[1] += s[1];
  }
}

struct PipeState {
  cudaStream_t st[kPipe] = {nullptr, nullptr, nullptr, nullptr};
};
PipeState g_pipe[kMaxDev];

using ChunkRun = int (*)(std::vector<HostBuf> &, int64_t np_chunk, void *, cudaStream_t);

int with_device_buffers(std::vector<HostBuf> &bufs, int64_t np, int m, ChunkRun run, void *ctx, double *temps) {
  int d = 0;
  if (cudaGetDevice(&d) != cudaSuccess || d < 0 || d >= kMaxDev) return set_error(SFNL_ERR_CUDA, "no current CUDA device");
  DevState *s = &g_dev[d];
  std::lock_guard<std::mutex> lk(s->mu);
  PipeState &ps = g_pipe[d];
  for (int i = 0; i < kPipe; ++i)
    if (!ps.st[i] && cudaStreamCreateWithFlags(&ps.st[i], cudaStreamNonBlocking) != cudaSuccess)
      return set_error(SFNL_ERR_CUDA, "cudaStreamCreate failed");
  size_t per_point = 0;
  for (auto &b : bufs) per_point += sizeof(double) * (size_t)b.ew * buf_rows(b, m);
  int64_t cp = (int64_t)(kChunkBytes / (per_point ? per_point : 1));
  cp = (cp / 128) * 128;
  if (cp < 128) cp = 128;
  if (cp > np) cp = np;
  const int64_t nchunks = (np + cp - 1) / cp;
  const int slots = nchunks < kPipe ? (int)nchunks : kPipe;
  size_t slot_bytes = 0;
  for (auto &b : bufs) slot_bytes += (sizeof(double) * (size_t)b.ew * buf_rows(b, m) * cp + 255) & ~size_t(255);
  const size_t total = slot_bytes * slots;
  if (total > s->work_bytes) {
    if (s->work) cudaFree(s->work);
    s->work = nullptr;
    s->work_bytes = 0;
    if (cudaMalloc(&s->work, total) != cudaSuccess) {
      cudaGetLastError();
      return set_error(SFNL_ERR_ALLOC, "cudaMalloc of the host-call workspace failed");
    }
    s->work_bytes = total;
  }
  Intervals iv;
  int rc = SFNL_OK;
  for (int64_t c = 0; c < nchunks && rc == SFNL_OK; ++c) {
    const int slot = (int)(c % slots);
    cudaStream_t st = ps.st[slot];
    const int64_t p0 = c * cp, n = (p0 + cp <= np) ? cp : np - p0;
    size_t off = slot_bytes * slot;
    int ic = iv.begin(st);
    for (auto &b : bufs) {
      b.dev = reinterpret_cast<double *>(s->work + off);
      off += (sizeof(double) * (size_t)b.ew * buf_rows(b, m) * cp + 255) & ~size_t(255);
      const size_t w = sizeof(double) * b.ew;  // bytes per point in a row
      if (b.src && cudaMemcpy2DAsync(b.dev, w * n, static_cast<const double *>(b.src) + b.ew * p0, w * np, w * n,
                                     buf_rows(b, m), cudaMemcpyHostToDevice, st) != cudaSuccess)
        rc = set_error(SFNL_ERR_CUDA, "host-to-device copy failed");
    }
    iv.end(ic, st, 0);
    const int ik = iv.begin(st);
    if (rc == SFNL_OK) rc = run(bufs, n, ctx, st);
    iv.end(ik, st, 1);
    ic = iv.begin(st);
    for (auto &b : bufs) {
      const size_t w = sizeof(double) * b.ew;
      if (rc == SFNL_OK && b.dst &&
          cudaMemcpy2DAsync(static_cast<double *>(b.dst) + b.ew * p0, w * np, b.dev, w * n, w * n,
                            buf_rows(b, m), cudaMemcpyDeviceToHost, st) != cudaSuccess)
        rc = set_error(SFNL_ERR_CUDA, "device-to-host copy failed");
    }
    iv.end(ic, st, 0);
  }
  for (int i = 0; i < slots; ++i)
    if (cudaStreamSynchronize(ps.st[i]) != cudaSuccess && rc == SFNL_OK)
      rc = set_error(SFNL_ERR_CUDA, "host call failed on the device");
  if (rc != SFNL_OK) return rc;
  if (split_take_status()) return timeout_error();
  // Sums over the chunks: a chunk's copies overlap other chunks' kernels on the other streams, so
  // temps(1) + temps(2) may exceed the wall time of the call.
  report_timing(iv, temps);
  return SFNL_OK;
}

struct ProdCtx {
  int op, m, pad, n_theta, algo;
  int64_t np;
};

int run_prod_dev(std::vector<HostBuf> &b, int64_t np_chunk, void *vctx, cudaStream_t st) {
  auto *c = static_cast<ProdCtx *>(vctx);
  ProgArgs a;
  int N = 0;
  int rc = check_common(np_chunk, c->m, c->pad, c->n_theta, 1, &N);
  if (rc) return rc;
  rc = build_product(c->op, b[0].dev, b[1].dev, b[2].dev, np_chunk, c->m, N, &a);
  if (rc) return rc;
  return run_fp64(a, c->algo, N, st);
}

int host_product(int op, const double *x, const double *y, double *out, int64_t np, int m, int pad, int n_theta,
                 int algo, double *temps) {
  if (temps) temps[0] = temps[1] = temps[2] = 0.0;
  int N = 0;
  int rc = check_common(np, m, pad, n_theta, 1, &N);
  if (rc) return rc;
  if (op < 0 || op >= kNumProducts) return set_error(SFNL_ERR_ARG, "op must be one of SFNL_OP_* (0..7)");
  if (np == 0) return SFNL_OK;
  if (!x || !y || !out) return set_error(SFNL_ERR_ARG, "null array");
  const ProductKind &pk = kProducts[op];
  std::vector<HostBuf> bufs = {{x, nullptr, pk.nsl_a, nullptr},
                               {y, nullptr, pk.nsl_b, nullptr},
                               {nullptr, out, pk.nsl_out, nullptr, pk.tensor_out ? 3 : 1}};
  ProdCtx c{op, m, pad, n_theta, algo, np};
  return with_device_buffers(bufs, np, m, run_prod_dev, &c, temps);
}

int check_fortran_args(int np, int nb_field, int m_max_c, int nb_procs, int bloc_size, bool need6) {
  if (np < 0 || m_max_c <= 0 || (nb_field % 2) != 0)
    return set_error(SFNL_ERR_ARG, "BUG in FFT_PAR_*: MOD(nb_field,2)/=0 .OR. m_max_c==0");
  if (need6 && nb_field != 6) return set_error(SFNL_ERR_SHAPE, "the cross/dot products need nb_field == 6");
  if (nb_procs != 1) return set_error(SFNL_ERR_UNSUPPORTED, "one GPU holds all modes: nb_procs must be 1");
  if (bloc_size < 1 || (int64_t)np > (int64_t)nb_procs * bloc_size)
    return set_error(SFNL_ERR_SHAPE, "np > nb_procs*bloc_size");
  return SFNL_OK;
}

// Synthesis-only routines (sfnl_synth.cu) on host arrays: grid values, or per-point maxima of |v|
// reduced on the host.
struct SynthCtx {
  int nslot, m, N;
  bool maxv;
};

int run_synth_dev(std::vector<HostBuf> &b, int64_t np_chunk, void *vctx, cudaStream_t st) {
  auto *c = static_cast<SynthCtx *>(vctx);
  return c->maxv ? launch_point_max_vel(b[0].dev, b[1].dev, np_chunk, c->nslot, c->m, c->N, st)
                 : launch_real(b[0].dev, b[1].dev, np_chunk, c->nslot, c->m, c->N, st);
}

int check_synth(int64_t np, int nslot, int m, const char *what) {
  if (np < 0 || m < 1 || nslot < 2 || (nslot % 2) != 0) {
    std::string msg = std::string("Bug in ") + what + ": MOD(nb_field,2)/=0 .OR. m_max_c==0";
    return set_error(SFNL_ERR_ARG, msg.c_str());
  }
  if (m > 4096) return set_error(SFNL_ERR_UNSUPPORTED, "m_max beyond this library's limits");
  return SFNL_OK;
}

struct BundleCtx {
  int64_t np;
  int m, pad, algo, form;
};

int run_bundle_dev(std::vector<HostBuf> &b, int64_t np_chunk, void *vctx, cudaStream_t st);

}  // namespace
int bundle_kernel() { return g_bundle_kernel.load(); }

}  // namespace sfnl

using namespace sfnl;

extern "C" {

const char *sfnl_last_error(void) { return g_err.c_str(); }
const char *sfnl_version(void) { return "sfemans_nl 0.1 (sm_100a)"; }
int sfnl_set_check_finite(int on) {
  g_check_finite = on ? 1 : 0;
  return SFNL_OK;
}
int sfnl_test_inject_timeout(void) { return split_inject_timeout(); }
int sfnl_test_large_workspace_cap(int64_t bytes) {
  if (bytes < 0) return set_error(SFNL_ERR_ARG, "workspace bound must be >= 0");
  large_test_workspace_cap((size_t)bytes);
  return SFNL_OK;
}
int sfnl_test_large_residues(int R) {
  if (R != 0 && R != 3 && R != 6 && R != 12) return set_error(SFNL_ERR_ARG, "residue classes: 0, 3, 6 or 12");
  large_test_residues(R);
  return SFNL_OK;
}
int sfnl_set_bundle_kernel(int kind) {
  if (kind != SFNL_BUNDLE_RESIDUE && kind != SFNL_BUNDLE_THIRD_FOLD)
    return set_error(SFNL_ERR_ARG, "bundle kernel: SFNL_BUNDLE_RESIDUE or SFNL_BUNDLE_THIRD_FOLD");
  return g_bundle_kernel.exchange(kind);
}
int sfnl_last_host_timing(double *s3) {
  if (!s3) return set_error(SFNL_ERR_ARG, "null pointer");
  for (int i = 0; i < 3; ++i) s3[i] = g_host_timing[i];
  return SFNL_OK;
}

int sfnl_finalize(void) {
  fast_release_tables();
  large_release_workspaces();
  split_release_tables();
  for (int d = 0; d < kMaxDev; ++d) {
    DevState &s = g_dev[d];
    std::lock_guard<std::mutex> lk(s.mu);
    if (!s.work && !s.d_flag && !s.gwork) continue;
    int prev = 0;
    cudaGetDevice(&prev);
    cudaSetDevice(d);
    if (s.work) cudaFree(s.work);
    if (s.d_flag) cudaFree(s.d_flag);
    if (s.gwork) cudaFree(s.gwork);
    s.gwork = nullptr;
    s.gwork_bytes = 0;
    for (int i = 0; i < kPipe; ++i)
      if (g_pipe[d].st[i]) {
        cudaStreamDestroy(g_pipe[d].st[i]);
        g_pipe[d].st[i] = nullptr;
      }
    s.work = nullptr;
    s.d_flag = nullptr;
    s.work_bytes = 0;
    cudaSetDevice(prev);
  }
  return SFNL_OK;
}

int sfnl_product_f64(int op, const double *a, const double *b, double *out, int64_t np, int m_max, int m_max_pad,
                     int n_theta, int algo, sfnl_stream_t stream) {
  int N = 0;
  int rc = check_common(np, m_max, m_max_pad, n_theta, 1, &N);
  if (rc) return rc;
  ProgArgs pa;
  rc = build_product(op, a, b, out, np, m_max, N, &pa);
  if (rc) return rc;
  if (np == 0) return SFNL_OK;
  return run_fp64(pa, algo, N, as_stream(stream));
}

int sfnl_cross_f64(const double *v1, const double *v2, double *out, int64_t np, int m_max, int m_max_pad,
                   sfnl_stream_t stream) {
  return sfnl_product_f64(OP_CROSS, v1, v2, out, np, m_max, m_max_pad, 0, SFNL_ALGO_AUTO, stream);
}
int sfnl_dot_f64(const double *v1, const double *v2, double *out, int64_t np, int m_max, int m_max_pad,
                 sfnl_stream_t stream) {
  return sfnl_product_f64(OP_DOT, v1, v2, out, np, m_max, m_max_pad, 0, SFNL_ALGO_AUTO, stream);
}
int sfnl_prod_f64(const double *c1, const double *c2, double *out, int64_t np, int m_max, int m_max_pad,
                  sfnl_stream_t stream) {
  return sfnl_product_f64(OP_PROD, c1, c2, out, np, m_max, m_max_pad, 0, SFNL_ALGO_AUTO, stream);
}

int sfnl_bundle_mhd_f64(const double *u, const double *w, const double *b, const double *j, const double *gradt,
                        double *uxw, double *uxb, double *jxb, double *ugradt, int64_t np, int m_max, int m_max_pad,
                        int algo, sfnl_stream_t stream) {
  int N = 0;
  int rc = check_common(np, m_max, m_max_pad, 0, 1, &N);
  if (rc) return rc;
  ProgArgs pa;
  rc = build_bundle(u, w, b, j, gradt, uxw, uxb, jxb, ugradt, np, m_max, N, &pa);
  if (rc) return rc;
  if (np == 0) return SFNL_OK;
  return run_fp64(pa, algo, N, as_stream(stream));
}

static int linear_f64(int kind, const double *u, const double *w, const double *b, const double *x, double *out,
                      int64_t np, int m, int pad, int kb, sfnl_stream_t stream) {
  int N = 0;
  int rc = check_common(np, m, pad, 0, kb, &N);
  if (rc) return rc;
  ProgArgs pa;
  rc = build_linear(kind, u, w, b, x, out, np, m, N, kb, &pa);
  if (rc) return rc;
  if (np == 0) return SFNL_OK;
  return run_fp64(pa, SFNL_ALGO_AUTO, N, as_stream(stream));
}

int sfnl_cross_jvp_f64(const double *u, const double *w, const double *tan, double *out, int64_t np, int m_max,
                       int m_max_pad, int k_batch, sfnl_stream_t stream) {
  return linear_f64(0, u, w, nullptr, tan, out, np, m_max, m_max_pad, k_batch, stream);
}
int sfnl_cross_vjp_f64(const double *u, const double *w, const double *cot, double *out, int64_t np, int m_max,
                       int m_max_pad, int k_batch, sfnl_stream_t stream) {
  return linear_f64(1, u, w, nullptr, cot, out, np, m_max, m_max_pad, k_batch, stream);
}
int sfnl_mhd_jvp_f64(const double *u, const double *w, const double *b, const double *tan, double *out, int64_t np,
                     int m_max, int m_max_pad, int k_batch, sfnl_stream_t stream) {
  return linear_f64(2, u, w, b, tan, out, np, m_max, m_max_pad, k_batch, stream);
}
int sfnl_mhd_vjp_f64(const double *u, const double *w, const double *b, const double *cot, double *out, int64_t np,
                     int m_max, int m_max_pad, int k_batch, sfnl_stream_t stream) {
  return linear_f64(3, u, w, b, cot, out, np, m_max, m_max_pad, k_batch, stream);
}

}  // extern "C"

namespace sfnl {
namespace {
struct LinCtx {
  int kind, m, pad, kb;
};
// One point chunk of a linearised program on the device copies of the host arrays.
int run_linear_dev(std::vector<HostBuf> &b, int64_t np_chunk, void *vctx, cudaStream_t st) {
  auto *c = static_cast<LinCtx *>(vctx);
  const bool mhd = c->kind >= 2;
  return linear_f64(c->kind, b[0].dev, b[1].dev, mhd ? b[2].dev : nullptr, b[mhd ? 3 : 2].dev, b[mhd ? 4 : 3].dev,
                    np_chunk, c->m, c->pad, c->kb, reinterpret_cast<sfnl_stream_t>(st));
}
// The linearised programs on host arrays (point chunks through the pipelined copies of the host entries).
int linear_host(int kind, const double *u, const double *w, const double *b, const double *x, double *out, int64_t np,
                int m, int pad, int kb) {
  int N = 0;
  int rc = check_common(np, m, pad, 0, kb, &N);
  if (rc) return rc;
  if (np == 0) return SFNL_OK;
  if (!u || !w || !x || !out || (kind >= 2 && !b)) return set_error(SFNL_ERR_ARG, "null array");
  static const int xs[4] = {12, 6, 18, 12}, os[4] = {6, 12, 12, 18};
  std::vector<HostBuf> bufs = {{u, nullptr, 6, nullptr}, {w, nullptr, 6, nullptr}};
  if (kind >= 2) bufs.push_back({b, nullptr, 6, nullptr});
  bufs.push_back({x, nullptr, xs[kind], nullptr, 1, m * kb});
  bufs.push_back({nullptr, out, os[kind], nullptr, 1, m * kb});
  LinCtx c{kind, m, pad, kb};
  return with_device_buffers(bufs, np, m, run_linear_dev, &c, nullptr);
}
}  // namespace
}  // namespace sfnl

extern "C" {

int sfnl_cross_jvp_host(const double *u, const double *w, const double *tan, double *out, int64_t np, int m_max,
                        int m_max_pad, int k_batch) {
  return linear_host(0, u, w, nullptr, tan, out, np, m_max, m_max_pad, k_batch);
}
int sfnl_cross_vjp_host(const double *u, const double *w, const double *cot, double *out, int64_t np, int m_max,
                        int m_max_pad, int k_batch) {
  return linear_host(1, u, w, nullptr, cot, out, np, m_max, m_max_pad, k_batch);
}
int sfnl_mhd_jvp_host(const double *u, const double *w, const double *b, const double *tan, double *out, int64_t np,
                      int m_max, int m_max_pad, int k_batch) {
  return linear_host(2, u, w, b, tan, out, np, m_max, m_max_pad, k_batch);
}
int sfnl_mhd_vjp_host(const double *u, const double *w, const double *b, const double *cot, double *out, int64_t np,
                      int m_max, int m_max_pad, int k_batch) {
  return linear_host(3, u, w, b, cot, out, np, m_max, m_max_pad, k_batch);
}

int sfnl_product_split(int op, const double *a, const double *b, double *out, int64_t np, int m_max, int m_max_pad,
                       int split, sfnl_stream_t stream) {
  int N = 0;
  int rc = check_common(np, m_max, m_max_pad, 0, 1, &N);
  if (rc) return rc;
  ProgArgs pa;
  rc = build_product(op, a, b, out, np, m_max, N, &pa);
  if (rc) return rc;
  if (np == 0) return SFNL_OK;
  return run_split(pa, split, N, as_stream(stream));
}

int sfnl_bundle_mhd_split(const double *u, const double *w, const double *b, const double *j, const double *gradt,
                          double *uxw, double *uxb, double *jxb, double *ugradt, int64_t np, int m_max, int m_max_pad,
                          int split, sfnl_stream_t stream) {
  int N = 0;
  int rc = check_common(np, m_max, m_max_pad, 0, 1, &N);
  if (rc) return rc;
  ProgArgs pa;
  rc = build_bundle(u, w, b, j, gradt, uxw, uxb, jxb, ugradt, np, m_max, N, &pa);
  if (rc) return rc;
  if (np == 0) return SFNL_OK;
  return run_split(pa, split, N, as_stream(stream));
}

static int linear_split(int kind, const double *u, const double *w, const double *b, const double *x, double *out,
                        int64_t np, int m, int pad, int kb, int split, sfnl_stream_t stream) {
  int N = 0;
  int rc = check_common(np, m, pad, 0, kb, &N);
  if (rc) return rc;
  ProgArgs pa;
  rc = build_linear(kind, u, w, b, x, out, np, m, N, kb, &pa);
  if (rc) return rc;
  if (np == 0) return SFNL_OK;
  return run_split(pa, split, N, as_stream(stream));
}

int sfnl_mhd_jvp_split(const double *u, const double *w, const double *b, const double *tan, double *out, int64_t np,
                       int m_max, int m_max_pad, int k_batch, int split, sfnl_stream_t stream) {
  return linear_split(2, u, w, b, tan, out, np, m_max, m_max_pad, k_batch, split, stream);
}
int sfnl_mhd_vjp_split(const double *u, const double *w, const double *b, const double *cot, double *out, int64_t np,
                       int m_max, int m_max_pad, int k_batch, int split, sfnl_stream_t stream) {
  return linear_split(3, u, w, b, cot, out, np, m_max, m_max_pad, k_batch, split, stream);
}

int sfnl_fft_par_cross_prod_dcl(const double *V1_in, const double *V2_in, double *V_out, int np, int nb_field,
                                int m_max_c, int nb_procs, int bloc_size, int m_max_pad, double *temps) {
  int rc = check_fortran_args(np, nb_field, m_max_c, nb_procs, bloc_size, true);
  if (rc) return rc;
  return host_product(OP_CROSS, V1_in, V2_in, V_out, np, m_max_c * nb_procs, m_max_pad, 0, SFNL_ALGO_AUTO, temps);
}
int sfnl_fft_par_dot_prod_dcl(const double *V1_in, const double *V2_in, double *c_out, int np, int nb_field,
                              int m_max_c, int nb_procs, int bloc_size, int m_max_pad, double *temps) {
  int rc = check_fortran_args(np, nb_field, m_max_c, nb_procs, bloc_size, true);
  if (rc) return rc;
  return host_product(OP_DOT, V1_in, V2_in, c_out, np, m_max_c * nb_procs, m_max_pad, 0, SFNL_ALGO_AUTO, temps);
}
int sfnl_fft_par_prod_dcl(const double *c1_in, const double *c2_in, double *c_out, int np, int m_max_c, int nb_procs,
                          int bloc_size, int m_max_pad, double *temps) {
  int rc = check_fortran_args(np, 2, m_max_c, nb_procs, bloc_size, false);
  if (rc) return rc;
  return host_product(OP_PROD, c1_in, c2_in, c_out, np, m_max_c * nb_procs, m_max_pad, 0, SFNL_ALGO_AUTO, temps);
}

int sfnl_fft_par_div_dcl(const double *c1_in, const double *c2_in, double *c_out, int np, int m_max_c, int nb_procs,
                         int bloc_size, int m_max_pad, double *temps) {
  int rc = check_fortran_args(np, 2, m_max_c, nb_procs, bloc_size, false);
  if (rc) return rc;
  return host_product(SFNL_OP_DIV, c1_in, c2_in, c_out, np, m_max_c * nb_procs, m_max_pad, 0, SFNL_ALGO_AUTO, temps);
}

int sfnl_fft_scalar_vect_dcl(const double *V1_in, const double *V2_in, double *V_out, int pb, int np, int nb_field1,
                             int nb_field2, int m_max_c, int nb_procs, int bloc_size, int m_max_pad, double *temps) {
  int rc = check_fortran_args(np, nb_field1, m_max_c, nb_procs, bloc_size, false);
  if (rc) return rc;
  if (nb_field2 % 2 != 0) return set_error(SFNL_ERR_ARG, "BUG in FFT_SCALAR_VECT_DCL: MOD(nb_field2,2)/=0");
  if (nb_field1 != 6 || nb_field2 != 2)
    return set_error(SFNL_ERR_SHAPE, "error in dimension of INPUT variables while calling FFT_SCALAR_VECT_DCL");
  if (pb != 1 && pb != 2) return set_error(SFNL_ERR_ARG, "error in problem type while calling FFT_SCALAR_VECT_DCL");
  return host_product(pb == 1 ? SFNL_OP_SCALAR_VECT : SFNL_OP_VECT_SCALAR, V1_in, V2_in, V_out, np,
                      m_max_c * nb_procs, m_max_pad, 0, SFNL_ALGO_AUTO, temps);
}

int sfnl_fft_tensor_dcl(const double *V1_in, const double *V2_in, double *V_out, int np, int nb_field, int m_max_c,
                        int nb_procs, int bloc_size, int m_max_pad, int opt_tension, double *temps) {
  int rc = check_fortran_args(np, nb_field, m_max_c, nb_procs, bloc_size, false);
  if (rc) return rc;
  if (nb_field != 6) return set_error(SFNL_ERR_SHAPE, "FFT_TENSOR_DCL forms the tensor only for nb_field == 6");
  if (opt_tension == 0) return set_error(SFNL_ERR_ARG, "BUG in FFT_TENSOR_DCL : opt_tension should be true if used");
  return host_product(opt_tension > 0 ? SFNL_OP_TENSION : SFNL_OP_TENSOR, V1_in, V2_in, V_out, np, m_max_c * nb_procs,
                      m_max_pad, 0, SFNL_ALGO_AUTO, temps);
}

// ---------------------------------------------------------------------------
// Fourier-mode-distributed callers (nb_procs > 1).  The reference splits the modes over the ranks of its
// Fourier communicator and exchanges them twice per call (fft_parallel.F90:205-217 and :306-324): each
// rank sends every peer q the points of q's block [q*bloc_size, (q+1)*bloc_size) of its own m_max_c
// modes, computes the product on its block with all m_max = nb_procs*m_max_c modes, and sends the modes
// of peer q back.  The exchanges stay with the caller's MPI (the Fortran shim calls MPI_ALLTOALL); these
// entries lay the buffers out and run the block's product on the GPU.  Buffer layout, per peer:
// [mode i < m_max_c][slot s < nslot][point n < bloc_size][e < ew] (ew = 3 for the tensor's V(3, np, 6, m)),
// bloc_size*nslot*m_max_c*ew doubles per peer; points beyond np are zero.
// ---------------------------------------------------------------------------
int sfnl_fft_par_pack_modes(const double *V, double *send, int np, int nslot, int m_max_c, int nb_procs, int bloc_size,
                            int ew) {
  if (np < 0 || nslot < 1 || m_max_c < 1 || nb_procs < 1 || bloc_size < 1 || (ew != 1 && ew != 3))
    return set_error(SFNL_ERR_ARG, "sfnl_fft_par_pack_modes: bad sizes");
  if ((int64_t)np > (int64_t)nb_procs * bloc_size) return set_error(SFNL_ERR_SHAPE, "np > nb_procs*bloc_size");
  if ((np > 0 && !V) || !send) return set_error(SFNL_ERR_ARG, "null array");
  for (int q = 0; q < nb_procs; ++q)
    for (int i = 0; i < m_max_c; ++i)
      for (int sl = 0; sl < nslot; ++sl) {
        double *dst = send + (((size_t)q * m_max_c + i) * nslot + sl) * (size_t)bloc_size * ew;
        for (int n = 0; n < bloc_size; ++n) {
          const int64_t gp = (int64_t)q * bloc_size + n;
          for (int e = 0; e < ew; ++e)
            dst[(size_t)n * ew + e] = gp < np ? V[e + ew * (gp + (int64_t)np * (sl + (int64_t)nslot * i))] : 0.0;
        }
      }
  return SFNL_OK;
}

int sfnl_fft_par_unpack_modes(const double *got, double *V_out, int np, int nslot, int m_max_c, int nb_procs,
                              int bloc_size, int ew) {
  if (np < 0 || nslot < 1 || m_max_c < 1 || nb_procs < 1 || bloc_size < 1 || (ew != 1 && ew != 3))
    return set_error(SFNL_ERR_ARG, "sfnl_fft_par_unpack_modes: bad sizes");
  if ((int64_t)np > (int64_t)nb_procs * bloc_size) return set_error(SFNL_ERR_SHAPE, "np > nb_procs*bloc_size");
  if (!got || (np > 0 && !V_out)) return set_error(SFNL_ERR_ARG, "null array");
  for (int q = 0; q < nb_procs; ++q)
    for (int i = 0; i < m_max_c; ++i)
      for (int sl = 0; sl < nslot; ++sl) {
        const double *src = got + (((size_t)q * m_max_c + i) * nslot + sl) * (size_t)bloc_size * ew;
        for (int n = 0; n < bloc_size; ++n) {
          const int64_t gp = (int64_t)q * bloc_size + n;
          if (gp >= np) break;  // dummy points are dropped (fft_parallel.F90:317)
          for (int e = 0; e < ew; ++e) V_out[e + ew * (gp + (int64_t)np * (sl + (int64_t)nslot * i))] = src[(size_t)n * ew + e];
        }
      }
  return SFNL_OK;
}

int sfnl_fft_par_block(int op, const double *recv1, const double *recv2, double *back, int bloc_size, int m_max_c,
                       int nb_procs, int m_max_pad, double *temps) {
  if (temps) temps[0] = temps[1] = temps[2] = 0.0;
  if (op < 0 || op >= kNumProducts) return set_error(SFNL_ERR_ARG, "op must be one of SFNL_OP_* (0..7)");
  if (bloc_size < 1 || m_max_c < 1 || nb_procs < 1) return set_error(SFNL_ERR_ARG, "sfnl_fft_par_block: bad sizes");
  if (!recv1 || !recv2 || !back) return set_error(SFNL_ERR_ARG, "null array");
  const ProductKind &pk = kProducts[op];
  const int m = m_max_c * nb_procs, ew = pk.tensor_out ? 3 : 1;
  const size_t b1 = (size_t)bloc_size * pk.nsl_a * m, b2 = (size_t)bloc_size * pk.nsl_b * m;
  const size_t bo = (size_t)bloc_size * pk.nsl_out * m * ew;
  std::vector<double> x(b1), y(b2), z(bo);
  // gathered block (bloc_size, nslot, m_max): global mode r*m_max_c + i from peer r (:223-231)
  auto gather = [&](const double *recv, int nsl, double *blk) {
    for (int r = 0; r < nb_procs; ++r)
      for (int i = 0; i < m_max_c; ++i)
        for (int sl = 0; sl < nsl; ++sl)
          std::memcpy(blk + (size_t)bloc_size * (sl + (size_t)nsl * (r * m_max_c + i)),
                      recv + (((size_t)r * m_max_c + i) * nsl + sl) * bloc_size, sizeof(double) * bloc_size);
  };
  gather(recv1, pk.nsl_a, x.data());
  gather(recv2, pk.nsl_b, y.data());
  int rc = host_product(op, x.data(), y.data(), z.data(), bloc_size, m, m_max_pad, 0, SFNL_ALGO_AUTO, temps);
  if (rc) return rc;
  // modes of peer q back to q (:306-324)
  for (int q = 0; q < nb_procs; ++q)
    for (int i = 0; i < m_max_c; ++i)
      for (int sl = 0; sl < pk.nsl_out; ++sl)
        std::memcpy(back + (((size_t)q * m_max_c + i) * pk.nsl_out + sl) * bloc_size * ew,
                    z.data() + (size_t)ew * bloc_size * (sl + (size_t)pk.nsl_out * (q * m_max_c + i)),
                    sizeof(double) * bloc_size * ew);
  return SFNL_OK;
}

int sfnl_scalar_vect_f64(const double *v, const double *s, double *out, int64_t np, int m_max, int m_max_pad, int pb,
                         sfnl_stream_t stream) {
  if (pb != 1 && pb != 2) return set_error(SFNL_ERR_ARG, "error in problem type while calling FFT_SCALAR_VECT_DCL");
  return sfnl_product_f64(pb == 1 ? SFNL_OP_SCALAR_VECT : SFNL_OP_VECT_SCALAR, v, s, out, np, m_max, m_max_pad, 0,
                          SFNL_ALGO_AUTO, stream);
}
int sfnl_tensor_f64(const double *v1, const double *v2, double *out, int64_t np, int m_max, int m_max_pad, int tension,
                    sfnl_stream_t stream) {
  return sfnl_product_f64(tension ? SFNL_OP_TENSION : SFNL_OP_TENSOR, v1, v2, out, np, m_max, m_max_pad, 0,
                          SFNL_ALGO_AUTO, stream);
}
int sfnl_div_f64(const double *c1, const double *c2, double *out, int64_t np, int m_max, int m_max_pad,
                 sfnl_stream_t stream) {
  return sfnl_product_f64(SFNL_OP_DIV, c1, c2, out, np, m_max, m_max_pad, 0, SFNL_ALGO_AUTO, stream);
}

int sfnl_fft_par_real_planes(int m_max, int opt_nb_plane) {
  if (m_max < 1) return set_error(SFNL_ERR_ARG, "m_max < 1");
  const int m_max_pad = opt_nb_plane > 2 * m_max - 1 ? (opt_nb_plane + 1) / 2 : m_max;
  return 2 * m_max_pad - 1;
}

int sfnl_real_f64(const double *v, double *out, int64_t np, int nslot, int m_max, int n_theta, sfnl_stream_t stream) {
  int rc = check_synth(np, nslot, m_max, "FFT_PAR_REAL");
  if (rc) return rc;
  if (n_theta < 2 * m_max - 1) return set_error(SFNL_ERR_ALIAS, "n_theta < 2*m_max-1: the grid cannot hold the modes");
  if (n_theta > (1 << 21)) return set_error(SFNL_ERR_UNSUPPORTED, "n_theta beyond this library's limits");
  if (np == 0) return SFNL_OK;
  if (!v || !out) return set_error(SFNL_ERR_ARG, "null array");
  return launch_real(v, out, np, nslot, m_max, n_theta, as_stream(stream));
}

int sfnl_max_vel_f64(const double *v, double *vmax, int64_t np, int nslot, int m_max, int m_max_pad,
                     sfnl_stream_t stream) {
  int rc = check_synth(np, nslot, m_max, "FFT_MAX_VEL_DCL");
  if (rc) return rc;
  if (m_max_pad < m_max) return set_error(SFNL_ERR_ALIAS, "m_max_pad < m_max: the padded spectrum cannot hold the modes");
  if (m_max_pad > (1 << 20)) return set_error(SFNL_ERR_UNSUPPORTED, "m_max_pad beyond this library's limits");
  if (!vmax || (np > 0 && !v)) return set_error(SFNL_ERR_ARG, "null array");
  cudaStream_t st = as_stream(stream);
  if (cudaMemsetAsync(vmax, 0, sizeof(double), st) != cudaSuccess) return set_error(SFNL_ERR_CUDA, "memset of the result failed");
  return launch_max_vel(v, vmax, np, nslot, m_max, 2 * m_max_pad - 1, st);
}

int sfnl_fft_par_real(const double *V1_in, double *V_out, int np, int nb_field, int m_max_c, int nb_procs,
                      int opt_nb_plane) {
  int rc = check_synth(np, nb_field, m_max_c, "FFT_PAR_REAL");
  if (rc) return rc;
  if (nb_procs != 1) return set_error(SFNL_ERR_UNSUPPORTED, "one GPU holds all modes: nb_procs must be 1");
  const int N = sfnl_fft_par_real_planes(m_max_c, opt_nb_plane);
  if (np == 0) return SFNL_OK;
  if (!V1_in || !V_out) return set_error(SFNL_ERR_ARG, "null array");
  std::vector<HostBuf> bufs = {{V1_in, nullptr, nb_field, nullptr}, {nullptr, V_out, 1, nullptr, N * (nb_field / 2), 1}};
  SynthCtx c{nb_field, m_max_c, N, false};
  return with_device_buffers(bufs, np, m_max_c, run_synth_dev, &c, nullptr);
}

int sfnl_fft_max_vel_dcl(const double *V1_in, double *V_out, int np, int nb_field, int m_max_c, int nb_procs,
                         int bloc_size, int m_max_pad) {
  int rc = check_synth(np, nb_field, m_max_c, "FFT_MAX_VEL_DCL");
  if (rc) return rc;
  if (nb_procs != 1) return set_error(SFNL_ERR_UNSUPPORTED, "one GPU holds all modes: nb_procs must be 1");
  if (bloc_size < 1 || (int64_t)np > (int64_t)nb_procs * bloc_size) return set_error(SFNL_ERR_SHAPE, "np > nb_procs*bloc_size");
  if (m_max_pad < m_max_c) return set_error(SFNL_ERR_ALIAS, "m_max_pad < m_max: the padded spectrum cannot hold the modes");
  if (!V_out) return set_error(SFNL_ERR_ARG, "null result");
  *V_out = 0.0;
  if (np == 0) return SFNL_OK;
  if (!V1_in) return set_error(SFNL_ERR_ARG, "null array");
  std::vector<double> pmax((size_t)np);
  std::vector<HostBuf> bufs = {{V1_in, nullptr, nb_field, nullptr}, {nullptr, pmax.data(), 1, nullptr, 1, 1}};
  SynthCtx c{nb_field, m_max_c, 2 * m_max_pad - 1, true};
  rc = with_device_buffers(bufs, np, m_max_c, run_synth_dev, &c, nullptr);
  if (rc) return rc;
  double best = 0.0;
  for (double x : pmax)
    if (!(x <= best)) best = x;  // a NaN propagates, as in the device entry
  *V_out = best;
  return SFNL_OK;
}

static int check_gauss(int np_nodes, int me, int n_w, int l_G, int nmod) {
  if (np_nodes < 1 || me < 0 || n_w < 1 || l_G < 1 || nmod < 1)
    return set_error(SFNL_ERR_ARG, "np_nodes, n_w, l_G and the number of modes must be >= 1, me >= 0");
  if (n_w > 10) return set_error(SFNL_ERR_UNSUPPORTED, "more than 10 nodes per element");
  if ((int64_t)l_G * me > ((int64_t)1 << 31)) return set_error(SFNL_ERR_UNSUPPORTED, "too many Gauss points");
  return SFNL_OK;
}

// Doubles of the Gauss-point operands of one caller.
static size_t gauss_operand_doubles(int kind, int conservative, int64_t ng, int nmod) {
  const size_t o6 = (size_t)ng * 6 * nmod, o2 = (size_t)ng * 2 * nmod;
  return 2 * o6 + (kind == sfnl::GK_ADVECT && conservative ? 2 * o2 : 0);
}

// A Gauss-point caller on device arrays: the operands into `work` (or the library's per-device buffer,
// held for the whole call), then the product on the FAST form.
static int gauss_product(int kind, const double *v, const double *v2, const double *omega, const double *heat,
                         int conservative, const int *jj, const double *ww, const double *dw, const double *rr,
                         const int *list_mode, double *out, int np_nodes, int me, int n_w, int l_G, int nmod,
                         int m_max_pad, double *work, sfnl_stream_t stream) {
  int rc = check_gauss(np_nodes, me, n_w, l_G, nmod);
  if (rc) return rc;
  const int pad = m_max_pad > 0 ? m_max_pad : (3 * nmod / 2 < nmod ? nmod : 3 * nmod / 2);
  const int64_t ng = (int64_t)l_G * me;
  int N = 0;
  if ((rc = check_common(ng, nmod, pad, 0, 1, &N))) return rc;
  if (ng == 0) return SFNL_OK;
  if (!v || !jj || !ww || !dw || !rr || !list_mode || !out || (kind != GK_NS && !v2))
    return set_error(SFNL_ERR_ARG, "null array");
  cudaStream_t st = as_stream(stream);
  // The curl callers at m = 64: node-major copies of the nodal fields (NF x np_nodes x 6 x nmod doubles),
  // then one kernel that builds the operands in the product's staging.  A caller's work buffer
  // (12*l_G*me*nmod doubles) holds the copies when NF*np_nodes <= 2*l_G*me (P2 meshes: about 4 me <= 14 me).
  // The advection callers likewise: node-major copies of the velocity and of the scalar (8 x np_nodes x nmod
  // doubles, within a caller's 12*l_G*me*nmod work buffer when 8*np_nodes <= 12*l_G*me).
  const int nf = 1 + (kind == GK_LORENTZ || (kind == GK_NS && omega) ? 1 : 0);
  const size_t nodal = (size_t)np_nodes * 6 * nmod;
  const size_t fused_doubles = kind == GK_ADVECT ? (size_t)np_nodes * 8 * nmod : nf * nodal;
  // m = 64 on P2 elements: the third-fold kernels; other m up to 96 (any element): the general FAST kernel
  const bool fused_tf = gauss_cross_fused_supported(nmod, n_w);
  const bool fused_gen = !fused_tf && gauss_general_fused_supported(kind, conservative != 0, nmod);
  const bool fused = (fused_tf || fused_gen) && dealiased(nmod, N) &&
                     (!work || fused_doubles <= gauss_operand_doubles(kind, conservative, ng, nmod));
  std::unique_lock<std::mutex> lk;
  double *wk = work;
  if (!wk) {
    DevState *s = dev_state();
    if (!s) return set_error(SFNL_ERR_CUDA, "no current device");
    lk = std::unique_lock<std::mutex>(s->mu);
    const size_t need = fused ? fused_doubles : gauss_operand_doubles(kind, conservative, ng, nmod);
    if ((rc = grow_gwork(s, need * sizeof(double)))) return rc;
    wk = reinterpret_cast<double *>(s->gwork);
  }
  if (fused && kind == GK_ADVECT) {
    double *vt = wk, *ct = wk + nodal;
    if ((rc = launch_nodal_transpose(v, vt, np_nodes, nmod, st))) return rc;
    if ((rc = launch_nodal_transpose(v2, ct, np_nodes, nmod, st, 2))) return rc;
    GaussArgs ga{vt, nullptr, ww, dw, rr, jj, list_mode, np_nodes, me, n_w, l_G, nmod, ct, heat};
    if ((rc = fused_gen ? launch_gauss_general_fused(ga, GK_ADVECT, conservative != 0, out, ng, nmod, st)
                        : launch_gauss_advect_fused(ga, conservative != 0, out, ng, nmod, st)))
      return rc;
    if (g_check_finite) {
      ProgArgs pa;
      if ((rc = build_product(OP_PROD, out, out, out, ng, nmod, N, &pa))) return rc;
      rc = scan_outputs(pa, st);
    }
    return rc;
  }
  if (fused) {
    double *vt = wk, *xt = wk + nodal;
    if ((rc = launch_nodal_transpose(v, vt, np_nodes, nmod, st))) return rc;
    const double *v2t = nullptr, *omt = nullptr;
    if (kind == GK_LORENTZ) {
      if ((rc = launch_nodal_transpose(v2, xt, np_nodes, nmod, st))) return rc;
      v2t = xt;
    } else if (omega) {
      if ((rc = launch_nodal_transpose(omega, xt, np_nodes, nmod, st))) return rc;
      omt = xt;
    }
    GaussArgs ga{vt, omt, ww, dw, rr, jj, list_mode, np_nodes, me, n_w, l_G, nmod, v2t, nullptr};
    if ((rc = fused_gen ? launch_gauss_general_fused(ga, kind, false, out, ng, nmod, st)
                        : launch_gauss_cross_fused(ga, kind, out, ng, nmod, st)))
      return rc;
    if (g_check_finite) {
      ProgArgs pa;
      if ((rc = build_product(OP_CROSS, out, out, out, ng, nmod, N, &pa))) return rc;
      rc = scan_outputs(pa, st);
    }
    return rc;
  }
  const size_t o6 = (size_t)ng * 6 * nmod, o2 = (size_t)ng * 2 * nmod;
  double *g0 = wk, *g1 = wk + o6;
  double *g2 = kind == GK_ADVECT && conservative ? wk + 2 * o6 : nullptr, *g3 = g2 ? g2 + o2 : nullptr;
  GaussArgs ga{v, kind == GK_NS ? omega : nullptr, ww, dw, rr, jj, list_mode, np_nodes, me, n_w, l_G, nmod,
               v2, kind == GK_ADVECT ? heat : nullptr};
  if ((rc = launch_gauss_eval(ga, kind, g0, g1, g2, g3, st))) return rc;
  ProgArgs pa;
  if (kind != GK_ADVECT) {
    if ((rc = build_product(OP_CROSS, g0, g1, out, ng, nmod, N, &pa))) return rc;  // RotV x W
  } else if (!conservative) {
    if ((rc = build_product(OP_DOT, g0, g1, out, ng, nmod, N, &pa))) return rc;    // Gradc . W
  } else {  // Gradc . W + Div Cgauss, analysed once
    pa = make_args(OP_ADVECT, ng, nmod, N, 1);
    for (int k = 0; k < 3; ++k) {
      set_in(pa, k, g0, ng, 6, k, nmod, false);
      set_in(pa, 3 + k, g1, ng, 6, k, nmod, false);
    }
    set_in(pa, 6, g2, ng, 2, 0, nmod, false);
    set_in(pa, 7, g3, ng, 2, 0, nmod, false);
    set_out(pa, 0, out, ng, 2, 0, nmod, false);
  }
  return run_fp64(pa, SFNL_ALGO_AUTO, N, st);
}

// A Gauss-point caller on host arrays (the reference signatures): every array copied to the device,
// the device caller, the result copied back.
static int host_gauss(int kind, const double *V_in, const double *V2_in, int nslot2, const double *omega,
                      const double *heat, int conservative, const int *jj, const double *ww, const double *dw,
                      const double *rr, int k_d, const int *list_mode, double *V_out, int nslot_out, int np_nodes,
                      int me, int n_w, int l_G, int nmod, int nb_procs) {
  int rc = check_gauss(np_nodes, me, n_w, l_G, nmod);
  if (rc) return rc;
  if (k_d != 2) return set_error(SFNL_ERR_UNSUPPORTED, "meridian meshes only (k_d == 2)");
  if (nb_procs != 1) return set_error(SFNL_ERR_UNSUPPORTED, "one GPU holds all modes: nb_procs must be 1");
  if (!V_in || !jj || !ww || !dw || !rr || !list_mode || !V_out || (nslot2 && !V2_in))
    return set_error(SFNL_ERR_ARG, "null array");
  for (int64_t t = 0; t < (int64_t)n_w * me; ++t)
    if (jj[t] < 1 || jj[t] > np_nodes) return set_error(SFNL_ERR_ARG, "jj holds a node number outside 1..np_nodes");
  const int64_t ng = (int64_t)l_G * me;
  const size_t nv = (size_t)np_nodes * 6 * nmod, nv2 = (size_t)np_nodes * nslot2 * nmod;
  const size_t nout = (size_t)ng * nslot_out * nmod, nwork = gauss_operand_doubles(kind, conservative, ng, nmod);
  const size_t nww = (size_t)n_w * l_G, ndw = (size_t)2 * n_w * l_G * me, nrr = (size_t)2 * np_nodes;
  auto al = [](size_t b) { return (b + 255) & ~size_t(255); };
  const size_t bytes = al(8 * nv) * (omega ? 2 : 1) + al(8 * nv2) + al(8 * (size_t)me) + al(8 * nout) +
                       al(8 * nwork) + al(8 * nww) + al(8 * ndw) + al(8 * nrr) + al(4 * (size_t)n_w * me) +
                       al(4 * (size_t)nmod);
  DevState *s = dev_state();
  if (!s) return set_error(SFNL_ERR_CUDA, "no current device");
  std::lock_guard<std::mutex> lk(s->mu);
  if ((rc = grow_gwork(s, bytes))) return rc;
  char *q = s->gwork;
  auto take = [&](size_t b) { char *r = q; q += al(b); return r; };
  double *d_v = (double *)take(8 * nv), *d_om = omega ? (double *)take(8 * nv) : nullptr;
  double *d_v2 = nslot2 ? (double *)take(8 * nv2) : nullptr, *d_heat = heat ? (double *)take(8 * (size_t)me) : nullptr;
  double *d_out = (double *)take(8 * nout), *d_work = (double *)take(8 * nwork);
  double *d_ww = (double *)take(8 * nww), *d_dw = (double *)take(8 * ndw), *d_rr = (double *)take(8 * nrr);
  int *d_jj = (int *)take(4 * (size_t)n_w * me), *d_lm = (int *)take(4 * (size_t)nmod);
  cudaStream_t st = nullptr;
  Intervals iv;
  const int ic = iv.begin(st);
  bool ok = cudaMemcpyAsync(d_v, V_in, 8 * nv, cudaMemcpyHostToDevice, st) == cudaSuccess &&
            (!omega || cudaMemcpyAsync(d_om, omega, 8 * nv, cudaMemcpyHostToDevice, st) == cudaSuccess) &&
            (!nslot2 || cudaMemcpyAsync(d_v2, V2_in, 8 * nv2, cudaMemcpyHostToDevice, st) == cudaSuccess) &&
            (!heat || cudaMemcpyAsync(d_heat, heat, 8 * (size_t)me, cudaMemcpyHostToDevice, st) == cudaSuccess) &&
            cudaMemcpyAsync(d_ww, ww, 8 * nww, cudaMemcpyHostToDevice, st) == cudaSuccess &&
            cudaMemcpyAsync(d_dw, dw, 8 * ndw, cudaMemcpyHostToDevice, st) == cudaSuccess &&
            cudaMemcpyAsync(d_rr, rr, 8 * nrr, cudaMemcpyHostToDevice, st) == cudaSuccess &&
            cudaMemcpyAsync(d_jj, jj, 4 * (size_t)n_w * me, cudaMemcpyHostToDevice, st) == cudaSuccess &&
            cudaMemcpyAsync(d_lm, list_mode, 4 * (size_t)nmod, cudaMemcpyHostToDevice, st) == cudaSuccess;
  if (!ok) return set_error(SFNL_ERR_CUDA, "host-to-device copy failed");
  iv.end(ic, st, 0);
  const int ik = iv.begin(st);
  rc = gauss_product(kind, d_v, d_v2, d_om, d_heat, conservative, d_jj, d_ww, d_dw, d_rr, d_lm, d_out, np_nodes, me,
                     n_w, l_G, nmod, 0, d_work, reinterpret_cast<sfnl_stream_t>(st));
  if (rc) return rc;
  iv.end(ik, st, 1);
  const int io = iv.begin(st);
  if (cudaMemcpyAsync(V_out, d_out, 8 * nout, cudaMemcpyDeviceToHost, st) != cudaSuccess)
    return set_error(SFNL_ERR_CUDA, "device-to-host copy failed");
  iv.end(io, st, 0);
  if (cudaStreamSynchronize(st) != cudaSuccess) return set_error(SFNL_ERR_CUDA, "device-to-host copy failed");
  report_timing(iv, nullptr);
  return SFNL_OK;
}

int sfnl_cross_gauss_f64(const double *v, const int *jj, const double *ww, const double *dw, const double *rr,
                         const int *list_mode, const double *omega, double *out, int np_nodes, int me, int n_w,
                         int l_G, int nmod, int m_max_pad, double *work, sfnl_stream_t stream) {
  return gauss_product(GK_NS, v, nullptr, omega, nullptr, 0, jj, ww, dw, rr, list_mode, out, np_nodes, me, n_w, l_G,
                       nmod, m_max_pad, work, stream);
}

int sfnl_smb_cross_prod_gauss(const double *V_in, const int *jj, const double *ww, const double *dw, const double *rr,
                              int k_d, const int *list_mode, const double *omega, double *V_out, int np_nodes, int me,
                              int n_w, int l_G, int nmod, int nb_procs) {
  return host_gauss(GK_NS, V_in, nullptr, 0, omega, nullptr, 0, jj, ww, dw, rr, k_d, list_mode, V_out, 6, np_nodes,
                    me, n_w, l_G, nmod, nb_procs);
}

int sfnl_curlh_cross_b_gauss_f64(const double *h, const double *b, const int *jj, const double *ww, const double *dw,
                                 const double *rr, const int *list_mode, double *out, int np_nodes, int me, int n_w,
                                 int l_G, int nmod, int m_max_pad, double *work, sfnl_stream_t stream) {
  return gauss_product(GK_LORENTZ, h, b, nullptr, nullptr, 0, jj, ww, dw, rr, list_mode, out, np_nodes, me, n_w, l_G,
                       nmod, m_max_pad, work, stream);
}

int sfnl_smb_curlh_cross_b_gauss(const double *V_in, const double *W_in, const int *jj, const double *ww,
                                 const double *dw, const double *rr, int k_d, const int *list_mode, double *V_out,
                                 int np_nodes, int me, int n_w, int l_G, int nmod, int nb_procs) {
  return host_gauss(GK_LORENTZ, V_in, W_in, 6, nullptr, nullptr, 0, jj, ww, dw, rr, k_d, list_mode, V_out, 6,
                    np_nodes, me, n_w, l_G, nmod, nb_procs);
}

int sfnl_gauss_operands_f64(int kind, const double *v, const double *v2, const double *omega, const double *heat,
                            int conservative, const int *jj, const double *ww, const double *dw, const double *rr,
                            const int *list_mode, double *o0, double *o1, double *o2, double *o3, int np_nodes,
                            int me, int n_w, int l_G, int nmod, sfnl_stream_t stream) {
  static_assert(SFNL_GAUSS_NS == GK_NS && SFNL_GAUSS_LORENTZ == GK_LORENTZ && SFNL_GAUSS_ADVECT == GK_ADVECT,
                "caller kinds");
  if (kind < SFNL_GAUSS_NS || kind > SFNL_GAUSS_ADVECT) return set_error(SFNL_ERR_ARG, "kind must be SFNL_GAUSS_*");
  if (conservative != 0 && conservative != 1) return set_error(SFNL_ERR_ARG, "conservative must be 0 or 1");
  int rc = check_gauss(np_nodes, me, n_w, l_G, nmod);
  if (rc) return rc;
  if ((int64_t)l_G * me == 0) return SFNL_OK;
  const bool cons = kind == GK_ADVECT && conservative;
  if (!v || !jj || !ww || !dw || !rr || !list_mode || !o0 || !o1 || (kind != GK_NS && !v2) || (cons && (!o2 || !o3)))
    return set_error(SFNL_ERR_ARG, "null array");
  GaussArgs ga{v, kind == GK_NS ? omega : nullptr, ww, dw, rr, jj, list_mode, np_nodes, me, n_w, l_G, nmod, v2,
               kind == GK_ADVECT ? heat : nullptr};
  return launch_gauss_eval(ga, kind, o0, o1, cons ? o2 : nullptr, cons ? o3 : nullptr, as_stream(stream));
}

int sfnl_ugradc_gauss_f64(const double *v, const double *c, const double *heat, int conservative, const int *jj,
                          const double *ww, const double *dw, const double *rr, const int *list_mode, double *out,
                          int np_nodes, int me, int n_w, int l_G, int nmod, int m_max_pad, double *work,
                          sfnl_stream_t stream) {
  if (conservative != 0 && conservative != 1) return set_error(SFNL_ERR_ARG, "conservative must be 0 or 1");
  return gauss_product(GK_ADVECT, v, c, nullptr, heat, conservative, jj, ww, dw, rr, list_mode, out, np_nodes, me,
                       n_w, l_G, nmod, m_max_pad, work, stream);
}

int sfnl_smb_ugradc_gauss(const double *V_in, const double *c_in, const double *heat_capa, int conservative,
                          const int *jj, const double *ww, const double *dw, const double *rr, int k_d,
                          const int *list_mode, double *c_out, int np_nodes, int me, int n_w, int l_G, int nmod,
                          int nb_procs) {
  if (conservative != 0 && conservative != 1) return set_error(SFNL_ERR_ARG, "conservative must be 0 or 1");
  return host_gauss(GK_ADVECT, V_in, c_in, 2, nullptr, heat_capa, conservative, jj, ww, dw, rr, k_d, list_mode,
                    c_out, 2, np_nodes, me, n_w, l_G, nmod, nb_procs);
}

int sfnl_product_f64_host(int op, const double *a, const double *b, double *out, int64_t np, int m_max, int m_max_pad,
                          int algo) {
  return host_product(op, a, b, out, np, m_max, m_max_pad, 0, algo, nullptr);
}

int sfnl_bundle_mhd_host(const double *u, const double *w, const double *b, const double *j, const double *gradt,
                         double *uxw, double *uxb, double *jxb, double *ugradt, int64_t np, int m_max, int m_max_pad,
                         int form) {
  int N = 0;
  int rc = check_common(np, m_max, m_max_pad, 0, 1, &N);
  if (rc) return rc;
  if (form != 0 && form != SFNL_SPLIT_BF16X2 && form != SFNL_SPLIT_BF16X3) return set_error(SFNL_ERR_ARG, "form must be 0, 2 or 3");
  if (np == 0) return SFNL_OK;
  if (!u || !w || !b || !j || !gradt || !uxw || !uxb || !jxb || !ugradt) return set_error(SFNL_ERR_ARG, "null array");
  std::vector<HostBuf> bufs = {{u, nullptr, 6, nullptr},   {w, nullptr, 6, nullptr},     {b, nullptr, 6, nullptr},
                               {j, nullptr, 6, nullptr},   {gradt, nullptr, 6, nullptr}, {nullptr, uxw, 6, nullptr},
                               {nullptr, uxb, 6, nullptr}, {nullptr, jxb, 6, nullptr},   {nullptr, ugradt, 2, nullptr}};
  BundleCtx c{np, m_max, m_max_pad, SFNL_ALGO_AUTO, form};
  return with_device_buffers(bufs, np, m_max, run_bundle_dev, &c, nullptr);
}

}  // extern "C"

namespace sfnl {
namespace {
int run_bundle_dev(std::vector<HostBuf> &b, int64_t np_chunk, void *vctx, cudaStream_t st) {
  auto *c = static_cast<BundleCtx *>(vctx);
  if (c->form == 0)
    return sfnl_bundle_mhd_f64(b[0].dev, b[1].dev, b[2].dev, b[3].dev, b[4].dev, b[5].dev, b[6].dev, b[7].dev,
                               b[8].dev, np_chunk, c->m, c->pad, c->algo, st);
  return sfnl_bundle_mhd_split(b[0].dev, b[1].dev, b[2].dev, b[3].dev, b[4].dev, b[5].dev, b[6].dev, b[7].dev,
                               b[8].dev, np_chunk, c->m, c->pad, c->form, st);
}
}  // namespace
}  // namespace sfnl
