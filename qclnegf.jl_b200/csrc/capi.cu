// C-ABI entry points (declared in include/qclb200.h).
#include <stdarg.h>
#include <string.h>

#include <algorithm>
#include <mutex>
#include <string>
#include <vector>

#include "kernels.cuh"

namespace qcl {

static thread_local char g_last_error[512] = "";

void set_last_error(const char* fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_last_error, sizeof(g_last_error), fmt, ap);
  va_end(ap);
}

static thread_local int g_singular_pivot = 0;

int singular_status(const char* what, int where) {
  const int block = (int)(where / kSingularPivotSpan), k = (int)(where % kSingularPivotSpan);
  g_singular_pivot = k;
  set_last_error("%s: singular block (linear block index %d, SingularException(%d))", what, block, k);
  return QCL_SINGULAR;
}

int cuda_status(cudaError_t e, const char* where) {
  set_last_error("CUDA error %s (%s) at %s", cudaGetErrorName(e), cudaGetErrorString(e), where);
  if (e == cudaErrorMemoryAllocation) return QCL_NOMEM;
  return QCL_CUDA;
}

// ---------------------------------------------------------------------------
// Small RAII device buffer for the host-buffer entry points.
// ---------------------------------------------------------------------------
struct DevBuf {
  void* p = nullptr;
  size_t bytes = 0;
  ~DevBuf() {
    if (p) cudaFree(p);
  }
  int alloc(size_t n) {
    bytes = n;
    if (n == 0) return QCL_OK;
    cudaError_t e = cudaMalloc(&p, n);
    if (e != cudaSuccess) return cuda_status(e, "cudaMalloc");
    return QCL_OK;
  }
  int upload(const void* host, size_t n) {
    int s = alloc(n);
    if (s) return s;
    if (host && n) {
      cudaError_t e = cudaMemcpy(p, host, n, cudaMemcpyHostToDevice);
      if (e != cudaSuccess) return cuda_status(e, "cudaMemcpy H2D");
    }
    return QCL_OK;
  }
  int download(void* host) const {
    if (host && bytes) {
      cudaError_t e = cudaMemcpy(host, p, bytes, cudaMemcpyDeviceToHost);
      if (e != cudaSuccess) return cuda_status(e, "cudaMemcpy D2H");
    }
    return QCL_OK;
  }
};

static size_t cbytes(int precision) { return precision == QCL_C128 ? 16 : 8; }

static int check_precision(int precision) {
  if (precision != QCL_C128 && precision != QCL_C64 && precision != QCL_MIXED) {
    set_last_error("unknown precision %d", precision);
    return QCL_ARG;
  }
  return QCL_OK;
}

static int read_status(const int* dstatus, const char* what) {
  int h[2] = {0, 0};
  cudaError_t e = cudaMemcpy(h, dstatus, sizeof(h), cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) return cuda_status(e, what);
  if (h[0] == QCL_SINGULAR) return singular_status(what, h[1]);
  if (h[0] != 0) {
    set_last_error("%s: device status %d at %d", what, h[0], h[1]);
    return h[0];
  }
  return QCL_OK;
}

// Device workspace of the host-buffer entry points: grows to the largest
// problem seen and is reused across calls, so a call allocates nothing once
// warm.  Calls are serialised by a mutex (one workspace per process).
struct Grow {
  void* p = nullptr;
  size_t cap = 0;
  int ensure(size_t n) {
    if (n <= cap && p) return QCL_OK;
    if (p) cudaFree(p);
    p = nullptr;
    cap = 0;
    cudaError_t e = cudaMalloc(&p, n > 0 ? n : 16);
    if (e != cudaSuccess) return cuda_status(e, "cudaMalloc (workspace)");
    cap = n;
    return QCL_OK;
  }
};

struct Pipeline {
  cudaStream_t st[3] = {nullptr, nullptr, nullptr};
  Grow eps, h, in[3], out[3], scale, trL, trG, status, wE, sum, gam;
  int init() {
    for (auto& s : st)
      if (!s) {
        cudaError_t e = cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking);
        if (e != cudaSuccess) return cuda_status(e, "cudaStreamCreate");
      }
    return QCL_OK;
  }
};
static std::mutex g_pipe_mutex;
static Pipeline& pipeline() {
  static Pipeline p;
  return p;
}

static HilbertTables& shared_hilbert_tables() {
  static HilbertTables t;
  return t;
}
static std::mutex g_hilbert_mutex;

struct ScbaCtx;
int scba_create(const qcl_scba_problem* p, const qcl_mechanism* mechs, ScbaCtx** out);
void scba_destroy(ScbaCtx* c);
int scba_seed(ScbaCtx* c, double* mu_out);
int scba_step(ScbaCtx* c, qcl_scba_row* row);
int scba_populations(ScbaCtx* c, double* out);
int scba_download(ScbaCtx* c, int which, void* host);
int scba_upload(ScbaCtx* c, int which, const void* host);
int scba_set_graph(ScbaCtx* c, int enable);
int scba_green_state(ScbaCtx* c, void* A, double* kappa, double* scale);
int scba_witness(ScbaCtx* c, double* out12);
int scba_retarget(ScbaCtx* c, double Ep, double N_LO, double kBT, const void* h, const double* q);
int scba_estimate_memory(const qcl_scba_problem* p, const qcl_mechanism* mechs, size_t out[6]);
int scba_promote(ScbaCtx* c);
int scba_tangent_init(ScbaCtx* c);
int scba_tangent_set(ScbaCtx* c, int which, const void* host);
int scba_tangent_step(ScbaCtx* c, double* out);
int scba_download_candidate(ScbaCtx* c, int which, void* host);
int scba_set_norm_branch(ScbaCtx* c, int branch);
int scba_norm_branch(ScbaCtx* c, int* out);
struct Sweep;
int sweep_create(int n, const qcl_scba_problem* problems, const qcl_mechanism* const* mechanisms, size_t budget,
                 Sweep** out);
int sweep_run(Sweep* sw, int max_iter, double tol, qcl_scba_row* last, int* iters, double* stats);
void sweep_destroy(Sweep* sw);
int scba_set_telemetry(ScbaCtx* c, int enable);
int scba_phase_times(ScbaCtx* c, double* ms, double* init_ms);
int scba_mixer_info(ScbaCtx* c, qcl_anderson_info* out);
int scba_density_matrix(ScbaCtx* c, void* out);

static int shift_plan_dev(int NE, const double* eps, double delta, DevBuf& l, DevBuf& r, DevBuf& th, DevBuf& v,
                          ShiftPlanDev* out) {
  std::vector<int> hl(NE), hr(NE);
  std::vector<double> ht(NE);
  std::vector<unsigned char> hv(NE);
  int s = build_shift_plan_host(NE, eps, delta, hl.data(), hr.data(), ht.data(), hv.data());
  if (s) return s;
  if ((s = l.upload(hl.data(), NE * sizeof(int)))) return s;
  if ((s = r.upload(hr.data(), NE * sizeof(int)))) return s;
  if ((s = th.upload(ht.data(), NE * sizeof(double)))) return s;
  if ((s = v.upload(hv.data(), NE))) return s;
  out->left = (const int*)l.p;
  out->right = (const int*)r.p;
  out->theta = (const double*)th.p;
  out->valid = (const unsigned char*)v.p;
  return QCL_OK;
}

int launch_convert(int precision, size_t n, const void* in_c128, void* out, cudaStream_t st);

// upload a complex128 host array converted to the field precision
static int upload_converted(int precision, const void* host, size_t n, DevBuf& dst) {
  DevBuf tmp;
  int s;
  if ((s = tmp.upload(host, n * 16))) return s;
  if ((s = dst.alloc(n * cbytes(precision)))) return s;
  return launch_convert(precision, n, tmp.p, dst.p, 0);
}

}  // namespace qcl

using namespace qcl;

extern "C" {

int qcl_version(void) { return 100; }
const char* qcl_last_error(void) { return g_last_error; }
int qcl_last_singular_pivot(void) { return g_singular_pivot; }
int qcl_max_basis(void) { return 48; }

int qcl_dev_dyson_keldysh(void* stream, int precision, int NE, int Nk, int Nb, const double* eps, double eta,
                          const void* h, const void* sigR, const void* sigL, const void* sigG, void* GR, void* GL,
                          void* GG, double* scale, void* traceL, void* traceG, int* status) {
  if (int s = check_precision(precision)) return s;
  return launch_dyson_keldysh(precision, NE, Nk, Nb, eps, eta, h, sigR, sigL, sigG, GR, GL, GG, scale, traceL,
                              traceG, status, (cudaStream_t)stream);
}

int qcl_dyson_keldysh(int precision, int NE, int Nk, int Nb, const double* eps, double eta, const void* h,
                      const void* sigR, const void* sigL, const void* sigG, void* GR, void* GL, void* GG,
                      double* scale, void* traceL, void* traceG) {
  if (int s = check_precision(precision)) return s;
  if (NE <= 0 || Nk <= 0 || Nb <= 0) {
    set_last_error("non-positive dimension (%d,%d,%d)", NE, Nk, Nb);
    return QCL_DIM;
  }
  if (!eps || !h || !sigR) {
    set_last_error("eps, h and sigR are required");
    return QCL_ARG;
  }
  if (padded_size(Nb) == 0) {
    set_last_error("basis size N_b=%d exceeds the supported maximum 48", Nb);
    return QCL_UNSUPPORTED;
  }
  std::lock_guard<std::mutex> lock(g_pipe_mutex);
  Pipeline& P = pipeline();
  int s;
  if ((s = P.init())) return s;
  const size_t es = cbytes(precision);
  const size_t nf = field_elems(NE, Nk, Nb) * es;
  const size_t nb = (size_t)NE * Nk;
  const void* hin[3] = {sigR, sigL, sigG};
  void* hout[3] = {GR, sigL ? GL : nullptr, sigG ? GG : nullptr};
  if ((s = P.eps.ensure(NE * sizeof(double)))) return s;
  if ((s = P.h.ensure((size_t)Nk * Nb * Nb * 16))) return s;
  for (int i = 0; i < 3; ++i) {
    if (hin[i] && (s = P.in[i].ensure(nf))) return s;
    if (hout[i] && (s = P.out[i].ensure(nf))) return s;
  }
  if (scale && (s = P.scale.ensure(nb * sizeof(double)))) return s;
  if (traceL && sigL && (s = P.trL.ensure(nb * 16))) return s;
  if (traceG && sigG && (s = P.trG.ensure(nb * 16))) return s;
  if ((s = P.status.ensure(2 * sizeof(int)))) return s;
  // on the pipeline's own (non-blocking) streams: legacy-stream copies and
  // memsets would not be ordered before the slab kernels
  QCL_CUDA_CHECK(cudaMemcpyAsync(P.eps.p, eps, NE * sizeof(double), cudaMemcpyHostToDevice, P.st[0]));
  QCL_CUDA_CHECK(cudaMemcpyAsync(P.h.p, h, (size_t)Nk * Nb * Nb * 16, cudaMemcpyHostToDevice, P.st[0]));
  QCL_CUDA_CHECK(cudaMemsetAsync(P.status.p, 0, 2 * sizeof(int), P.st[0]));
  QCL_CUDA_CHECK(cudaStreamSynchronize(P.st[0]));
  // momentum slabs of ~64 MiB per field, round-robin over three streams so
  // that the upload of one slab, the kernel of the previous one and the
  // download of the one before overlap
  const size_t slab_bytes = (size_t)NE * Nb * Nb * es;
  int ms = (int)std::max<size_t>(1, (64u << 20) / std::max<size_t>(slab_bytes, 1));
  ms = std::min(ms, Nk);
  const size_t pitch = (size_t)NE * Nk * es;
  int k = 0;
  for (int m0 = 0; m0 < Nk; m0 += ms, ++k) {
    const int cnt = std::min(ms, Nk - m0);
    cudaStream_t st = P.st[k % 3];
    const size_t off = (size_t)NE * m0 * es, width = (size_t)NE * cnt * es;
    for (int i = 0; i < 3; ++i)
      if (hin[i])
        QCL_CUDA_CHECK(cudaMemcpy2DAsync((char*)P.in[i].p + off, pitch, (const char*)hin[i] + off, pitch, width,
                                         (size_t)Nb * Nb, cudaMemcpyHostToDevice, st));
    s = launch_dyson_keldysh(precision, NE, Nk, Nb, (const double*)P.eps.p, eta, P.h.p, P.in[0].p,
                             sigL ? P.in[1].p : nullptr, sigG ? P.in[2].p : nullptr, GR ? P.out[0].p : nullptr,
                             hout[1] ? P.out[1].p : nullptr, hout[2] ? P.out[2].p : nullptr,
                             scale ? (double*)P.scale.p : nullptr, (traceL && sigL) ? P.trL.p : nullptr,
                             (traceG && sigG) ? P.trG.p : nullptr, (int*)P.status.p, st, m0, cnt);
    if (s) return s;
    for (int i = 0; i < 3; ++i)
      if (hout[i])
        QCL_CUDA_CHECK(cudaMemcpy2DAsync((char*)hout[i] + off, pitch, (const char*)P.out[i].p + off, pitch, width,
                                         (size_t)Nb * Nb, cudaMemcpyDeviceToHost, st));
    const size_t boff = (size_t)NE * m0, bcnt = (size_t)NE * cnt;
    if (scale)
      QCL_CUDA_CHECK(cudaMemcpyAsync(scale + boff, (double*)P.scale.p + boff, bcnt * sizeof(double),
                                     cudaMemcpyDeviceToHost, st));
    if (traceL && sigL)
      QCL_CUDA_CHECK(cudaMemcpyAsync((char*)traceL + boff * 16, (char*)P.trL.p + boff * 16, bcnt * 16,
                                     cudaMemcpyDeviceToHost, st));
    if (traceG && sigG)
      QCL_CUDA_CHECK(cudaMemcpyAsync((char*)traceG + boff * 16, (char*)P.trG.p + boff * 16, bcnt * 16,
                                     cudaMemcpyDeviceToHost, st));
  }
  for (int i = 0; i < 3; ++i) QCL_CUDA_CHECK(cudaStreamSynchronize(P.st[i]));
  return read_status((int*)P.status.p, "dyson_keldysh");
}

int qcl_dev_weighted_trace(void* stream, int NE, int Nk, const void* trace, const double* wE, const double* wk,
                           double* out) {
  static double* partial = nullptr;
  if (!partial) QCL_CUDA_CHECK(cudaMalloc(&partial, 296 * 2 * sizeof(double)));
  return launch_weighted_trace(NE, Nk, trace, wE, wk, partial, out, (cudaStream_t)stream);
}

int qcl_dev_paired_coefficients(void* stream, const double* trL, const double* trG, int gs, double target,
                                double* coeffs, int* status) {
  return launch_paired_coefficients(trL, trG, gs, target, coeffs, status, (cudaStream_t)stream);
}

int qcl_dev_normalize_pair(void* stream, int precision, size_t n, void* GL, void* GG, const double* coeffs) {
  if (int s = check_precision(precision)) return s;
  return launch_normalize_pair(precision, n, GL, GG, coeffs, (cudaStream_t)stream);
}

static int hilbert_host(int precision, int NE, size_t ncols, const double* eps, const double* wE, const void* Gam,
                        const void* SL, const void* SG, void* out_lam, void* out_SR, void* out_gam,
                        double* roundoff) {
  if (int s = check_precision(precision)) return s;
  if (!eps || !wE) {
    set_last_error("eps and wE are required");
    return QCL_ARG;
  }
  double de;
  if (int s = check_uniform_grid(NE, eps, &de)) return s;
  std::lock_guard<std::mutex> lock(g_pipe_mutex);
  std::lock_guard<std::mutex> lock2(g_hilbert_mutex);
  HilbertTables& t = shared_hilbert_tables();
  Pipeline& P = pipeline();
  int s;
  if ((s = P.init())) return s;
  if ((s = prepare_hilbert_tables(t, NE, de, precision))) return s;
  const int sp = precision == QCL_MIXED ? QCL_C64 : precision;
  const size_t es = cbytes(sp);
  const size_t nf = (size_t)NE * ncols * es;
  const bool verify = roundoff != nullptr;
  if ((s = P.wE.ensure(NE * sizeof(double)))) return s;
  if (Gam && (s = P.in[0].ensure(nf))) return s;
  if (SL && (s = P.in[1].ensure(nf))) return s;
  if (SG && (s = P.in[2].ensure(nf))) return s;
  if ((s = P.out[0].ensure(nf))) return s;
  if (out_gam && (s = P.gam.ensure(nf))) return s;
  if (verify && (s = ensure_partial(t, (long long)ncols))) return s;
  if ((s = P.sum.ensure(2 * sizeof(double)))) return s;
  QCL_CUDA_CHECK(cudaMemcpyAsync(P.wE.p, wE, NE * sizeof(double), cudaMemcpyHostToDevice, P.st[0]));
  QCL_CUDA_CHECK(cudaStreamSynchronize(P.st[0]));
  // column slabs of ~64 MiB, three streams
  size_t cs = std::max<size_t>(1, (64u << 20) / ((size_t)NE * es));
  cs = std::min(cs, ncols);
  int k = 0;
  for (size_t c0 = 0; c0 < ncols; c0 += cs, ++k) {
    const size_t cnt = std::min(cs, ncols - c0);
    cudaStream_t st = P.st[k % 3];
    const size_t off = c0 * NE * es, bytes = cnt * NE * es;
    if (Gam) QCL_CUDA_CHECK(cudaMemcpyAsync((char*)P.in[0].p + off, (const char*)Gam + off, bytes, cudaMemcpyHostToDevice, st));
    if (SL) QCL_CUDA_CHECK(cudaMemcpyAsync((char*)P.in[1].p + off, (const char*)SL + off, bytes, cudaMemcpyHostToDevice, st));
    if (SG) QCL_CUDA_CHECK(cudaMemcpyAsync((char*)P.in[2].p + off, (const char*)SG + off, bytes, cudaMemcpyHostToDevice, st));
    s = launch_hilbert(t, sp, (long long)cnt, (const double*)P.wE.p, Gam ? (char*)P.in[0].p + off : nullptr,
                       SL ? (char*)P.in[1].p + off : nullptr, SG ? (char*)P.in[2].p + off : nullptr,
                       out_lam ? (char*)P.out[0].p + off : nullptr, out_SR ? (char*)P.out[0].p + off : nullptr,
                       out_gam ? (char*)P.gam.p + off : nullptr, verify, st, (long long)c0);
    if (s) return s;
    QCL_CUDA_CHECK(cudaMemcpyAsync((char*)(out_lam ? out_lam : out_SR) + off, (char*)P.out[0].p + off, bytes,
                                   cudaMemcpyDeviceToHost, st));
    if (out_gam) QCL_CUDA_CHECK(cudaMemcpyAsync((char*)out_gam + off, (char*)P.gam.p + off, bytes, cudaMemcpyDeviceToHost, st));
  }
  for (int i = 0; i < 3; ++i) QCL_CUDA_CHECK(cudaStreamSynchronize(P.st[i]));
  if (verify) {
    if ((s = launch_combine(t.partial, (int)ncols, 2, (double*)P.sum.p, 0))) return s;
    double h2[2];
    QCL_CUDA_CHECK(cudaMemcpy(h2, P.sum.p, sizeof(h2), cudaMemcpyDeviceToHost));
    *roundoff = isfinite(h2[0]) && isfinite(h2[1]) ? sqrt(h2[0]) / (sqrt(h2[1]) + 1e-14) : INFINITY;
  }
  return QCL_OK;
}

int qcl_dev_fft_hilbert_transform(void* stream, int precision, int NE, size_t ncols, double de, const double* wE,
                                  const void* Gam, void* Lam, double* roundoff_sums) {
  if (int s = check_precision(precision)) return s;
  if (NE < 2 || !(de > 0)) {
    set_last_error("fft_hilbert: need N_E >= 2 and a positive spacing");
    return QCL_ARG;
  }
  std::lock_guard<std::mutex> lock(g_hilbert_mutex);
  HilbertTables& t = shared_hilbert_tables();
  int s;
  if ((s = prepare_hilbert_tables(t, NE, de, precision))) return s;
  const int sp = precision == QCL_MIXED ? QCL_C64 : precision;
  const bool verify = roundoff_sums != nullptr;
  if ((s = launch_hilbert(t, sp, (long long)ncols, wE, Gam, nullptr, nullptr, Lam, nullptr, nullptr, verify,
                          (cudaStream_t)stream)))
    return s;
  if (verify) return launch_combine(t.partial, (int)ncols, 2, roundoff_sums, (cudaStream_t)stream);
  return QCL_OK;
}

int qcl_fft_hilbert_transform(int precision, int NE, size_t ncols, const double* eps, const double* wE,
                              const void* Gam, void* Lam, double* roundoff) {
  if (!Gam || !Lam) {
    set_last_error("Gam and Lam are required");
    return QCL_ARG;
  }
  return hilbert_host(precision, NE, ncols, eps, wE, Gam, nullptr, nullptr, Lam, nullptr, nullptr, roundoff);
}

int qcl_apply_energy_shift(int precision, int NE, size_t ncols, const double* eps, double delta, const void* X,
                           void* Y) {
  if (int s = check_precision(precision)) return s;
  if (!eps || !X || !Y) {
    set_last_error("eps, X and Y are required");
    return QCL_ARG;
  }
  if (X == Y) {
    set_last_error("in-place aliasing is not supported");  // production_cache.jl:308-309
    return QCL_ARG;
  }
  const int sp = precision == QCL_MIXED ? QCL_C64 : precision;
  DevBuf l, r, th, v, dX, dY;
  ShiftPlanDev plan;
  int s;
  if ((s = shift_plan_dev(NE, eps, delta, l, r, th, v, &plan))) return s;
  const size_t nb = (size_t)NE * ncols * cbytes(sp);
  if ((s = dX.upload(X, nb))) return s;
  if ((s = dY.alloc(nb))) return s;
  if ((s = launch_shift(sp, NE, (long long)ncols, plan, dX.p, dY.p, 0))) return s;
  QCL_CUDA_CHECK(cudaDeviceSynchronize());
  return dY.download(Y);
}

int qcl_static_contraction(int precision, const qcl_mechanism* op, int NE, int Nk, int Nb, const double* wk,
                           double alpha, double beta, const void* G, void* S) {
  if (int s = check_precision(precision)) return s;
  if (!op || !wk || !G || !S) {
    set_last_error("operator, wk, G and S are required");
    return QCL_ARG;
  }
  const int sp = precision == QCL_MIXED ? QCL_C64 : precision;
  const size_t N2 = (size_t)Nb * Nb;
  DevBuf blk, mat, le, ri, ra, dwk, dG, dS, work;
  KernelOpDev k;
  k.kind = op->kind;
  k.J = op->J;
  int s;
  if (op->kind == QCL_KERNEL_MOMENTUM_INDEPENDENT) {
    if ((s = upload_converted(sp, op->block, N2 * N2, blk))) return s;
    k.block = blk.p;
  } else if (op->kind == QCL_KERNEL_DENSE) {
    const size_t nc = (size_t)Nk * N2;
    if ((s = upload_converted(sp, op->matrix, nc * nc, mat))) return s;
    k.matrix = mat.p;
  } else if (op->kind == QCL_KERNEL_IFR) {
    if (op->J < 1) {
      set_last_error("IFR operator needs J >= 1");
      return QCL_ARG;
    }
    if ((s = upload_converted(sp, op->left, N2 * op->J, le))) return s;
    if ((s = upload_converted(sp, op->right, N2 * op->J, ri))) return s;
    if ((s = upload_converted(sp, op->radial, (size_t)Nk * Nk, ra))) return s;
    k.left = le.p;
    k.right = ri.p;
    k.radial = ra.p;
  } else if (op->kind == QCL_KERNEL_LOW_RANK) {
    if (op->J < 1) {
      set_last_error("low-rank operator needs rank J >= 1");
      return QCL_ARG;
    }
    const size_t nc = (size_t)Nk * N2;
    if ((s = upload_converted(sp, op->left, nc * op->J, le))) return s;
    if ((s = upload_converted(sp, op->right, nc * op->J, ri))) return s;
    k.left = le.p;
    k.right = ri.p;
  } else if (op->kind == QCL_KERNEL_SEPARABLE_SUM) {
    if (op->J < 1) {
      set_last_error("separable-sum operator needs J >= 1 terms");
      return QCL_ARG;
    }
    if ((s = upload_converted(sp, op->radial, (size_t)Nk * Nk * op->J, ra))) return s;
    if ((s = upload_converted(sp, op->block, N2 * N2 * op->J, blk))) return s;
    k.radial = ra.p;
    k.block = blk.p;
  } else {
    set_last_error("unknown kernel kind %d", op->kind);
    return QCL_ARG;
  }
  const size_t nb = field_elems(NE, Nk, Nb) * cbytes(sp);
  if ((s = dwk.upload(wk, Nk * sizeof(double)))) return s;
  DevBuf st;
  if ((s = st.upload(nullptr, 2 * sizeof(int)))) return s;
  QCL_CUDA_CHECK(cudaMemset(st.p, 0, 2 * sizeof(int)));
  void* bop = nullptr;
  struct TcFree {
    void** a;
    ~TcFree() { cudaFree(*a); }
  } tc_free{&bop};
  if (op->kind == QCL_KERNEL_DENSE && sp == QCL_C64) {  // complex64: tensor-core operand
    if ((s = tc_build_operator(Nk * (int)N2, Nk, mat.p, (const double*)dwk.p, &bop, 0))) return s;
    k.tc_bop = bop;
    k.status = (int*)st.p;
  }
  std::vector<void*> chunk_ops, stage1_ops;  // separable sum, complex64: tensor-core operands per term chunk
  struct ChunkFree {
    std::vector<void*>* v;
    ~ChunkFree() {
      for (void* q : *v) cudaFree(q);
    }
  } chunk_free{&chunk_ops}, stage1_free{&stage1_ops};
  if (op->kind == QCL_KERNEL_SEPARABLE_SUM && sp == QCL_C64) {
    if ((s = sep_build_tc_operands(Nk, Nb, op->J, ra.p, blk.p, (const double*)dwk.p, chunk_ops, stage1_ops, 0)))
      return s;
    k.tc_chunks = chunk_ops.data();
    k.tc_stage1 = stage1_ops.data();
    k.status = (int*)st.p;
  }
  if ((s = dG.upload(G, nb))) return s;
  if ((s = dS.upload(beta != 0.0 ? S : nullptr, nb))) return s;
  if ((s = work.alloc(contraction_work_elems(k, NE, Nk, Nb) * cbytes(sp)))) return s;
  if ((s = launch_contraction(sp, k, NE, Nk, Nb, (const double*)dwk.p, dG.p, dS.p, alpha * op->q, beta, work.p, 0)))
    return s;
  QCL_CUDA_CHECK(cudaDeviceSynchronize());
  int hst[2] = {0, 0};
  QCL_CUDA_CHECK(cudaMemcpy(hst, st.p, sizeof(hst), cudaMemcpyDeviceToHost));
  if (hst[0]) {
    set_last_error("static contraction: device wait gave up (status %d at tile %d)", hst[0], hst[1]);
    return hst[0];
  }
  return dS.download(S);
}

int qcl_embedding_component(int precision, int NE, int Nk, int Nb, const double* eps, double delta, const void* T,
                            const void* G, void* S) {
  if (int s = check_precision(precision)) return s;
  if (!eps || !T || !G || !S) {
    set_last_error("eps, T, G and S are required");
    return QCL_ARG;
  }
  if (padded_size(Nb) == 0) {
    set_last_error("basis size N_b=%d exceeds the supported maximum 48", Nb);
    return QCL_UNSUPPORTED;
  }
  const int sp = precision == QCL_MIXED ? QCL_C64 : precision;
  DevBuf l, r, th, v, dT, dG, dS;
  ShiftPlanDev plan;
  int s;
  if ((s = shift_plan_dev(NE, eps, delta, l, r, th, v, &plan))) return s;
  const size_t nb = field_elems(NE, Nk, Nb) * cbytes(sp);
  if ((s = dT.upload(T, (size_t)Nb * Nb * 16))) return s;
  if ((s = dG.upload(G, nb))) return s;
  if ((s = dS.alloc(nb))) return s;
  SandwichJob job;
  job.X[0] = dG.p;
  job.S[0] = dS.p;
  job.T = dT.p;
  job.plan = plan;
  if ((s = launch_sandwich(sp, NE, Nk, Nb, &job, 1, 0))) return s;
  QCL_CUDA_CHECK(cudaDeviceSynchronize());
  return dS.download(S);
}

static void witness_from_doubles(const double* v, qcl_psd_witness* w) {
  w->matrix_kind = (int)v[0];
  w->energy_index = (int)v[1];
  w->momentum_index = (int)v[2];
  w->minimum_eigenvalue = v[3];
  w->block_norm = v[4];
  w->floor = v[5];
  w->ratio = v[6];
  w->absolute_defect = v[7];
  w->relative_defect = v[8];
  w->backward_error = v[9];
  w->hermiticity_defect = v[10];
  w->construction_scale = v[11];
}

static int residual_suite_host(int precision, int NE, int Nk, int Nb, const double* eps, const void* h,
                               const void* GR, const void* GL, const void* GG, const void* SR, const void* SL,
                               const void* SG, const void* SLc, double* out, qcl_psd_witness* witness) {
  if (int s = check_precision(precision)) return s;
  if (!eps || !h || !GR || !GL || !GG || !SR || !SL || !SG || !SLc || !out) {
    set_last_error("all residual-suite arrays are required");
    return QCL_ARG;
  }
  if (padded_size(Nb) == 0) {
    set_last_error("basis size N_b=%d exceeds the supported maximum 48", Nb);
    return QCL_UNSUPPORTED;
  }
  const int sp = precision == QCL_MIXED ? QCL_C64 : precision;
  const size_t nb = field_elems(NE, Nk, Nb) * cbytes(sp);
  DevBuf de, dh, d[7], work, o;
  const void* host[7] = {GR, GL, GG, SR, SL, SG, SLc};
  int s;
  if ((s = de.upload(eps, NE * sizeof(double)))) return s;
  if ((s = dh.upload(h, (size_t)Nk * Nb * Nb * 16))) return s;
  for (int i = 0; i < 7; ++i)
    if ((s = d[i].upload(host[i], nb))) return s;
  if ((s = work.alloc(residual_work_doubles(NE, Nk) * sizeof(double)))) return s;
  if ((s = o.alloc(5 * sizeof(double)))) return s;
  if ((s = launch_residual_suite(sp, NE, Nk, Nb, (const double*)de.p, dh.p, d[0].p, d[1].p, d[2].p, d[3].p, d[4].p,
                                 d[5].p, d[6].p, (double*)work.p, (double*)o.p, 0)))
    return s;
  DevBuf wpart, wout;
  if (witness) {
    if ((s = wpart.alloc(residual_witness_partial_doubles() * sizeof(double)))) return s;
    if ((s = wout.alloc(12 * sizeof(double)))) return s;
    if ((s = launch_residual_witness(sp, NE, Nk, Nb, d[0].p, d[1].p, d[2].p, d[4].p, d[5].p, (const double*)work.p,
                                     (double*)wpart.p, (double*)wout.p, 0)))
      return s;
  }
  QCL_CUDA_CHECK(cudaDeviceSynchronize());
  if ((s = o.download(out))) return s;
  if (witness) {
    double v[12];
    if ((s = wout.download(v))) return s;
    witness_from_doubles(v, witness);
  }
  return QCL_OK;
}

int qcl_residual_suite(int precision, int NE, int Nk, int Nb, const double* eps, const void* h, const void* GR,
                       const void* GL, const void* GG, const void* SR, const void* SL, const void* SG,
                       const void* SLc, double* out) {
  return residual_suite_host(precision, NE, Nk, Nb, eps, h, GR, GL, GG, SR, SL, SG, SLc, out, nullptr);
}

int qcl_residual_suite_witness(int precision, int NE, int Nk, int Nb, const double* eps, const void* h,
                               const void* GR, const void* GL, const void* GG, const void* SR, const void* SL,
                               const void* SG, const void* SLc, double* out, qcl_psd_witness* witness) {
  if (!witness) {
    set_last_error("residual_suite_witness: witness output is required");
    return QCL_ARG;
  }
  return residual_suite_host(precision, NE, Nk, Nb, eps, h, GR, GL, GG, SR, SL, SG, SLc, out, witness);
}

int qcl_hermitian_eigvals(int n, size_t count, const void* H, double* vals) {
  if (n < 1 || !H || !vals) {
    set_last_error("hermitian_eigvals: n >= 1 and arrays are required");
    return QCL_ARG;
  }
  DevBuf dH, dv;
  int s;
  if ((s = dH.upload(H, (size_t)n * n * count * 16))) return s;
  if ((s = dv.alloc((size_t)n * count * sizeof(double)))) return s;
  if ((s = launch_eigvals(n, (long long)count, dH.p, (double*)dv.p, 0))) return s;
  QCL_CUDA_CHECK(cudaDeviceSynchronize());
  return dv.download(vals);
}

int qcl_selfenergy_residual(int precision, size_t n, const void* old_, const void* new_, double* out) {
  if (int s = check_precision(precision)) return s;
  const int sp = precision == QCL_MIXED ? QCL_C64 : precision;
  DevBuf a, b, part, o;
  int s;
  if ((s = a.upload(old_, n * cbytes(sp)))) return s;
  if ((s = b.upload(new_, n * cbytes(sp)))) return s;
  if ((s = part.alloc(kReduceCtas * 2 * sizeof(double)))) return s;
  if ((s = o.alloc(2 * sizeof(double)))) return s;
  if ((s = launch_residual_mix(sp, n, a.p, b.p, 0.0, (double*)part.p, (double*)o.p, 0))) return s;
  QCL_CUDA_CHECK(cudaDeviceSynchronize());
  double h2[2];
  if ((s = o.download(h2))) return s;
  *out = (isfinite(h2[0]) && isfinite(h2[1])) ? sqrt(h2[0]) / (sqrt(h2[1]) + 1e-14) : INFINITY;
  return QCL_OK;
}

int qcl_current_populations(int precision, int NE, int Nk, int Nb, const double* wE, const double* wk, int gs,
                            double target, const void* SG, const void* SL, const void* GL, const void* GG,
                            double* out) {
  if (int s = check_precision(precision)) return s;
  const int sp = precision == QCL_MIXED ? QCL_C64 : precision;
  const size_t nb = field_elems(NE, Nk, Nb) * cbytes(sp);
  DevBuf dwE, dwk, a, b, c, d, part, o;
  int s;
  if ((s = dwE.upload(wE, NE * sizeof(double)))) return s;
  if ((s = dwk.upload(wk, Nk * sizeof(double)))) return s;
  if ((s = a.upload(SG, nb))) return s;
  if ((s = b.upload(SL, nb))) return s;
  if ((s = c.upload(GL, nb))) return s;
  if ((s = d.upload(GG, nb))) return s;
  if ((s = part.alloc(observables_partial_doubles(Nb) * sizeof(double)))) return s;
  if ((s = o.alloc((2 + Nb) * sizeof(double)))) return s;
  if ((s = launch_observables(sp, NE, Nk, Nb, (const double*)dwE.p, (const double*)dwk.p, a.p, b.p, c.p, d.p, gs,
                              target, (double*)part.p, (double*)o.p, 0)))
    return s;
  QCL_CUDA_CHECK(cudaDeviceSynchronize());
  return o.download(out);
}

int qcl_scba_create(const qcl_scba_problem* problem, const qcl_mechanism* mechanisms, qcl_scba** out) {
  if (!out) {
    set_last_error("out is required");
    return QCL_ARG;
  }
  ScbaCtx* c = nullptr;
  int s = scba_create(problem, mechanisms, &c);
  *out = (qcl_scba*)c;
  return s;
}
void qcl_scba_destroy(qcl_scba* ctx) { scba_destroy((ScbaCtx*)ctx); }
int qcl_scba_seed(qcl_scba* ctx, double* mu) { return ctx ? scba_seed((ScbaCtx*)ctx, mu) : QCL_ARG; }
int qcl_scba_step(qcl_scba* ctx, qcl_scba_row* row) {
  if (!ctx || !row) {
    set_last_error("ctx and row are required");
    return QCL_ARG;
  }
  return scba_step((ScbaCtx*)ctx, row);
}
int qcl_scba_run(qcl_scba* ctx, int max_iter, double tol_sigma, qcl_scba_row* history, int* n_done) {
  if (!ctx || !history || max_iter < 0) {
    set_last_error("ctx and history are required");
    return QCL_ARG;
  }
  int n = 0, s = QCL_OK;
  for (; n < max_iter; ++n) {
    s = scba_step((ScbaCtx*)ctx, &history[n]);
    if (s) break;
    if (history[n].status != QCL_OK || history[n].r_Sigma <= tol_sigma) {
      ++n;
      break;
    }
  }
  if (n_done) *n_done = n;
  return s;
}
int qcl_scba_populations(qcl_scba* ctx, double* out) { return scba_populations((ScbaCtx*)ctx, out); }
int qcl_scba_download(qcl_scba* ctx, int which, void* host) { return scba_download((ScbaCtx*)ctx, which, host); }
int qcl_scba_upload(qcl_scba* ctx, int which, const void* host) { return scba_upload((ScbaCtx*)ctx, which, host); }
int qcl_scba_use_graph(qcl_scba* ctx, int enable) { return scba_set_graph((ScbaCtx*)ctx, enable); }
int qcl_scba_green_state(qcl_scba* ctx, void* A, double* kappa, double* scale) {
  if (!ctx) {
    set_last_error("ctx is required");
    return QCL_ARG;
  }
  return scba_green_state((ScbaCtx*)ctx, A, kappa, scale);
}

int qcl_scba_retarget(qcl_scba* ctx, double Ep, double N_LO, double kBT, const void* h, const double* q) {
  if (!ctx) {
    set_last_error("ctx is required");
    return QCL_ARG;
  }
  return scba_retarget((ScbaCtx*)ctx, Ep, N_LO, kBT, h, q);
}

int qcl_scba_estimate_memory(const qcl_scba_problem* problem, const qcl_mechanism* mechanisms,
                             qcl_memory_estimate* out) {
  if (!problem || !out || (problem->nmech > 0 && !mechanisms)) {
    set_last_error("problem, mechanisms and out are required");
    return QCL_ARG;
  }
  size_t v[6];
  int s = scba_estimate_memory(problem, mechanisms, v);
  if (s) return s;
  out->fields = v[0];
  out->operators = v[1];
  out->workspace = v[2];
  out->anderson = v[3];
  out->resident = v[4];
  out->peak = v[5];
  return QCL_OK;
}

int qcl_scba_use_telemetry(qcl_scba* ctx, int enable) {
  if (!ctx) {
    set_last_error("ctx is required");
    return QCL_ARG;
  }
  return scba_set_telemetry((ScbaCtx*)ctx, enable);
}

int qcl_scba_phase_times(qcl_scba* ctx, double* ms, double* initialization_ms) {
  if (!ctx) {
    set_last_error("ctx is required");
    return QCL_ARG;
  }
  return scba_phase_times((ScbaCtx*)ctx, ms, initialization_ms);
}

int qcl_sweep_create(int npoints, const qcl_scba_problem* problems, const qcl_mechanism* const* mechanisms,
                     size_t memory_budget_bytes, qcl_sweep** out) {
  if (!out) {
    set_last_error("out is required");
    return QCL_ARG;
  }
  return sweep_create(npoints, problems, mechanisms, memory_budget_bytes, (Sweep**)out);
}

int qcl_sweep_run(qcl_sweep* sweep, int max_iter, double tol_sigma, qcl_scba_row* last_rows, int* iterations,
                  double* stats) {
  if (!sweep || !last_rows || !iterations || max_iter < 1) {
    set_last_error("sweep, last_rows, iterations and max_iter >= 1 are required");
    return QCL_ARG;
  }
  return sweep_run((Sweep*)sweep, max_iter, tol_sigma, last_rows, iterations, stats);
}

void qcl_sweep_destroy(qcl_sweep* sweep) { sweep_destroy((Sweep*)sweep); }

int qcl_scba_tangent_init(qcl_scba* ctx) {
  if (!ctx) {
    set_last_error("ctx is required");
    return QCL_ARG;
  }
  return scba_tangent_init((ScbaCtx*)ctx);
}

int qcl_scba_tangent_set(qcl_scba* ctx, int which, const void* host) {
  if (!ctx) {
    set_last_error("ctx is required");
    return QCL_ARG;
  }
  return scba_tangent_set((ScbaCtx*)ctx, which, host);
}

int qcl_scba_tangent_step(qcl_scba* ctx, double* out) {
  if (!ctx || !out) {
    set_last_error("ctx and out are required");
    return QCL_ARG;
  }
  return scba_tangent_step((ScbaCtx*)ctx, out);
}

int qcl_scba_download_candidate(qcl_scba* ctx, int which, void* host) {
  if (!ctx || !host) {
    set_last_error("ctx and host are required");
    return QCL_ARG;
  }
  return scba_download_candidate((ScbaCtx*)ctx, which, host);
}

int qcl_scba_set_normalization_branch(qcl_scba* ctx, int branch) {
  if (!ctx) {
    set_last_error("ctx is required");
    return QCL_ARG;
  }
  return scba_set_norm_branch((ScbaCtx*)ctx, branch);
}

int qcl_scba_normalization_branch(qcl_scba* ctx, int* branch) {
  if (!ctx || !branch) {
    set_last_error("ctx and branch are required");
    return QCL_ARG;
  }
  return scba_norm_branch((ScbaCtx*)ctx, branch);
}

int qcl_debug_set_wait_limit(long long rounds) { return tc_set_wait_limit(rounds); }

int qcl_scba_promote(qcl_scba* ctx) {
  if (!ctx) {
    set_last_error("ctx is required");
    return QCL_ARG;
  }
  return scba_promote((ScbaCtx*)ctx);
}

int qcl_anderson_guard(int precision, int NE, int Nk, int Nb, int nfam, const void* const* fields,
                       long long* first_failure, int* code) {
  if (int s = check_precision(precision)) return s;
  if (NE <= 0 || Nk <= 0 || Nb <= 0 || nfam < 1 || nfam > kMaxMixFields / 3) {
    set_last_error("anderson_guard: bad dimensions (%d,%d,%d) or family count %d", NE, Nk, Nb, nfam);
    return QCL_DIM;
  }
  if (!fields || !first_failure || !code) {
    set_last_error("anderson_guard: fields and outputs are required");
    return QCL_ARG;
  }
  const int sp = precision == QCL_MIXED ? QCL_C64 : precision;
  const size_t nb = field_elems(NE, Nk, Nb) * cbytes(sp);
  std::vector<DevBuf> d(3 * nfam);
  void* ptr[kMaxMixFields];
  int s;
  for (int i = 0; i < 3 * nfam; ++i) {
    if (!fields[i]) {
      set_last_error("anderson_guard: field %d is NULL", i);
      return QCL_ARG;
    }
    if ((s = d[i].upload(fields[i], nb))) return s;
    ptr[i] = d[i].p;
  }
  DevBuf meta;
  if ((s = meta.alloc(sizeof(AndersonMeta)))) return s;
  if ((s = launch_anderson_reset((AndersonMeta*)meta.p, 0))) return s;
  if ((s = launch_anderson_guard(sp, NE, Nk, Nb, ptr, nfam, (AndersonMeta*)meta.p, 0, 0.0, 0))) return s;
  QCL_CUDA_CHECK(cudaDeviceSynchronize());
  AndersonMeta h;
  QCL_CUDA_CHECK(cudaMemcpy(&h, meta.p, sizeof(h), cudaMemcpyDeviceToHost));
  const bool failed = h.guard_key != ~0ull;
  *first_failure = failed ? (long long)(h.guard_key >> 3) : 0;
  *code = failed ? (int)(h.guard_key & 7ull) : 0;
  return QCL_OK;
}

int qcl_scba_density_matrix(qcl_scba* ctx, void* rho) {
  if (!ctx || !rho) {
    set_last_error("ctx and rho are required");
    return QCL_ARG;
  }
  return scba_density_matrix((ScbaCtx*)ctx, rho);
}

int qcl_density_matrix(int precision, int NE, int Nk, int Nb, const double* wE, const double* wk, const void* GL,
                       void* rho) {
  if (int s = check_precision(precision)) return s;
  if (NE <= 0 || Nk <= 0 || Nb <= 0) {
    set_last_error("density_matrix: non-positive dimension (%d,%d,%d)", NE, Nk, Nb);
    return QCL_DIM;
  }
  if (!wE || !wk || !GL || !rho) {
    set_last_error("density_matrix: wE, wk, GL and rho are required");
    return QCL_ARG;
  }
  const int sp = precision == QCL_MIXED ? QCL_C64 : precision;
  DevBuf dwE, dwk, dG, dr;
  int s;
  if ((s = dwE.upload(wE, NE * sizeof(double)))) return s;
  if ((s = dwk.upload(wk, Nk * sizeof(double)))) return s;
  if ((s = dG.upload(GL, field_elems(NE, Nk, Nb) * cbytes(sp)))) return s;
  if ((s = dr.alloc(2 * (size_t)Nb * Nb * sizeof(double)))) return s;
  if ((s = launch_density_matrix(sp, NE, Nk, Nb, dG.p, (const double*)dwE.p, (const double*)dwk.p, (double*)dr.p,
                                 0)))
    return s;
  QCL_CUDA_CHECK(cudaDeviceSynchronize());
  return dr.download(rho);
}

static int check_assembly(int form, int Nk, int Nb, int T) {
  if (form != QCL_ASSEMBLE_RANK1 && form != QCL_ASSEMBLE_TABLE) {
    set_last_error("kernel assembly: unknown form %d", form);
    return QCL_ARG;
  }
  if (Nk <= 0 || Nb <= 0 || T <= 0) {
    set_last_error("kernel assembly: non-positive dimension (Nk=%d, Nb=%d, T=%d)", Nk, Nb, T);
    return QCL_DIM;
  }
  return QCL_OK;
}

int qcl_dev_assemble_kernel(void* stream, int form, int Nk, int Nb, int T, const double* W, const void* X,
                            void* matrix, double* work) {
  if (int s = check_assembly(form, Nk, Nb, T)) return s;
  if (!W || !X || !matrix || !work) {
    set_last_error("kernel assembly: W, X, matrix and work are required");
    return QCL_ARG;
  }
  return launch_assemble_kernel(form, Nk, Nb, T, W, X, matrix, work, (cudaStream_t)stream);
}

int qcl_assemble_kernel(int form, int Nk, int Nb, int T, const double* W, const void* X, void* matrix, double* qK) {
  if (int s = check_assembly(form, Nk, Nb, T)) return s;
  if (!W || !X || !matrix || !qK) {
    set_last_error("kernel assembly: W, X, matrix and qK are required");
    return QCL_ARG;
  }
  const size_t N2 = (size_t)Nb * Nb, Nc = (size_t)Nk * N2;
  const size_t xelems = form == QCL_ASSEMBLE_RANK1 ? (size_t)T * N2 : (size_t)T * N2 * N2;
  DevBuf dW, dX, dM, work;
  int s;
  if ((s = dW.upload(W, (size_t)Nk * Nk * T * sizeof(double)))) return s;
  if ((s = dX.upload(X, xelems * 16))) return s;
  if ((s = dM.alloc(Nc * Nc * 16))) return s;
  if ((s = work.alloc(assemble_work_doubles() * sizeof(double)))) return s;
  if ((s = launch_assemble_kernel(form, Nk, Nb, T, (const double*)dW.p, dX.p, dM.p, (double*)work.p, 0))) return s;
  QCL_CUDA_CHECK(cudaDeviceSynchronize());
  QCL_CUDA_CHECK(cudaMemcpy(qK, (double*)work.p + assemble_work_doubles() - 1, sizeof(double), cudaMemcpyDeviceToHost));
  return dM.download(matrix);
}

int qcl_scba_mixer_info(qcl_scba* ctx, qcl_anderson_info* info) {
  if (!ctx || !info) {
    set_last_error("ctx and info are required");
    return QCL_ARG;
  }
  return scba_mixer_info((ScbaCtx*)ctx, info);
}

int qcl_scba_witness(qcl_scba* ctx, qcl_psd_witness* witness) {
  if (!ctx || !witness) {
    set_last_error("ctx and witness are required");
    return QCL_ARG;
  }
  double v[12];
  if (int s = scba_witness((ScbaCtx*)ctx, v)) return s;
  witness_from_doubles(v, witness);
  return QCL_OK;
}

int qcl_condition_number(int precision, int NE, int Nk, int Nb, const double* eps, double eta, const void* h,
                         const void* SR, const void* GR, double* kappa, double* scale) {
  if (int s = check_precision(precision)) return s;
  if (NE <= 0 || Nk <= 0 || Nb <= 0) {
    set_last_error("condition_number: non-positive dimension (%d,%d,%d)", NE, Nk, Nb);
    return QCL_DIM;
  }
  if (!eps || !h || !GR || (!kappa && !scale)) {
    set_last_error("condition_number: eps, h, GR and at least one of kappa / scale are required");
    return QCL_ARG;
  }
  if (!isfinite(eta)) {
    set_last_error("condition_number: eta must be finite");
    return QCL_ARG;
  }
  const int sp = precision == QCL_MIXED ? QCL_C64 : precision;
  const size_t nf = field_elems(NE, Nk, Nb) * cbytes(sp), nb = (size_t)NE * Nk * sizeof(double);
  DevBuf de, dh, dS, dG, dk, ds;
  int s;
  if ((s = de.upload(eps, NE * sizeof(double)))) return s;
  if ((s = dh.upload(h, (size_t)Nk * Nb * Nb * 16))) return s;
  if (SR && (s = dS.upload(SR, nf))) return s;
  if ((s = dG.upload(GR, nf))) return s;
  if (kappa && (s = dk.alloc(nb))) return s;
  if (scale && (s = ds.alloc(nb))) return s;
  if ((s = launch_condition(sp, NE, Nk, Nb, (const double*)de.p, eta, dh.p, SR ? dS.p : nullptr, dG.p,
                            (double*)dk.p, (double*)ds.p, 0)))
    return s;
  QCL_CUDA_CHECK(cudaDeviceSynchronize());
  if (kappa && (s = dk.download(kappa))) return s;
  if (scale && (s = ds.download(scale))) return s;
  return QCL_OK;
}

int qcl_spectral_function(int precision, int NE, int Nk, int Nb, const void* GR, void* A) {
  if (int s = check_precision(precision)) return s;
  if (NE <= 0 || Nk <= 0 || Nb <= 0) {
    set_last_error("spectral_function: non-positive dimension (%d,%d,%d)", NE, Nk, Nb);
    return QCL_DIM;
  }
  if (!GR || !A || GR == A) {
    set_last_error("spectral_function: distinct GR and A are required");
    return QCL_ARG;
  }
  const int sp = precision == QCL_MIXED ? QCL_C64 : precision;
  const size_t nf = field_elems(NE, Nk, Nb) * cbytes(sp);
  DevBuf dG, dA;
  int s;
  if ((s = dG.upload(GR, nf))) return s;
  if ((s = dA.alloc(nf))) return s;
  if ((s = launch_spectral(sp, NE, Nk, Nb, dG.p, dA.p, 0))) return s;
  QCL_CUDA_CHECK(cudaDeviceSynchronize());
  return dA.download(A);
}

int qcl_retarded_self_energy(int precision, int NE, size_t ncols, const double* eps, const double* wE,
                             const void* SL, const void* SG, void* SR, void* Gam, double* roundoff) {
  if (!SL || !SG || !SR) {
    set_last_error("SL, SG and SR are required");
    return QCL_ARG;
  }
  return hilbert_host(precision, NE, ncols, eps, wE, nullptr, SL, SG, nullptr, SR, Gam, roundoff);
}

}  // extern "C"
