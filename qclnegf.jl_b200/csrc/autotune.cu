// Project autotuner: picks the CTA shape of the Dyson + Keldysh kernel (the
// number of (E, k) blocks per CTA, which sets the threads, shared memory and
// register budget per CTA) for one basis class and precision by timing every
// compiled candidate on a synthetic batch with CUDA events, and records the
// fastest for every later launch in the process (dyson_bpc).  The reference
// exposes the analogous knobs as hints set by hand (ProductionOptions.
// energy_chunk / worker_count, numerics/optimized/production_contracts.jl:
// 143-165); here they are measured on the device.
#include <vector>

#include "kernels.cuh"

namespace qcl {

// Deterministic pseudo-random values in [0, 1) from an index and a seed.
__device__ __forceinline__ double tune_hash(unsigned long long i, unsigned seed) {
  unsigned long long x = (i + 1) * 0x9E3779B97F4A7C15ull ^ ((unsigned long long)seed << 32);
  x ^= x >> 31;
  x *= 0xBF58476D1CE4E5B9ull;
  x ^= x >> 29;
  return (double)(x >> 11) * (1.0 / 9007199254740992.0);
}

// The value ranges of the operator batch: h with diagonal levels in [0, 2.5]
// plus an in-plane shift and couplings ~0.02; Sigma^R = -i (0.02 .. 0.05) on
// the diagonal plus 0.01 noise; Sigma^< = i 0.005 .. 0.015 on the diagonal.
template <typename R>
__global__ void tune_fill_kernel(int NE, int Nk, int N, Cx<double>* h, Cx<R>* SR, Cx<R>* SL) {
  const size_t nf = (size_t)NE * Nk * N * N, blk = (size_t)NE * Nk;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < nf; i += (size_t)gridDim.x * blockDim.x) {
    const int a = (int)((i / blk) % N), b = (int)(i / (blk * N));
    const double u = tune_hash(i, 1), v = tune_hash(i, 2);
    double sr = 0.01 * (u - 0.5), si = 0.01 * (v - 0.5), li = 0;
    if (a == b) {
      si = -(0.02 + 0.03 * u);
      li = 0.01 * (0.5 + v);
    }
    SR[i] = cx<R>((R)sr, (R)si);
    SL[i] = cx<R>((R)0, (R)li);
    if (i < (size_t)Nk * N * N) {  // h[m + Nk (a + N b)]
      const int m = (int)(i % Nk), ha = (int)((i / Nk) % N), hb = (int)(i / ((size_t)Nk * N));
      h[i] = ha == hb ? cx<double>(2.5 * (double)ha / N + 0.1 * m, 0.0) : cx<double>(0.02 * (tune_hash(i, 3) - 0.5), 0.0);
    }
  }
}

// Times every blocks-per-CTA candidate for (precision, N) on an NE x Nk
// batch (2 warm-up and 5 timed launches each); records and returns the
// fastest.  ms[i] is the mean device time per launch of candidate i.
int autotune_dyson(int precision, int N, int NE, int Nk, int* best, int* ncand, int* cands, float* ms) {
  const int NP = padded_size(N);
  if (NP == 0) {
    set_last_error("autotune: basis size %d exceeds the supported maximum 48", N);
    return QCL_UNSUPPORTED;
  }
  if (NE < 1 || Nk < 1) {
    set_last_error("autotune: non-positive batch (%d, %d)", NE, Nk);
    return QCL_DIM;
  }
  const int n = dyson_bpc_candidates(NP, cands);
  *ncand = n;
  const size_t esz = precision == QCL_C128 ? 16 : 8;
  const size_t nf = (size_t)NE * Nk * N * N;
  struct Bufs {
    void* p[7] = {};
    cudaStream_t st = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    ~Bufs() {
      if (st) cudaStreamSynchronize(st);
      for (void* q : p) cudaFree(q);
      if (e0) cudaEventDestroy(e0);
      if (e1) cudaEventDestroy(e1);
      if (st) cudaStreamDestroy(st);
    }
  } b;
  QCL_CUDA_CHECK(cudaStreamCreateWithFlags(&b.st, cudaStreamNonBlocking));
  QCL_CUDA_CHECK(cudaEventCreate(&b.e0));
  QCL_CUDA_CHECK(cudaEventCreate(&b.e1));
  QCL_CUDA_CHECK(cudaMalloc(&b.p[0], (size_t)NE * sizeof(double)));  // eps
  QCL_CUDA_CHECK(cudaMalloc(&b.p[1], (size_t)Nk * N * N * 16));      // h
  for (int i = 2; i < 6; ++i) QCL_CUDA_CHECK(cudaMalloc(&b.p[i], nf * esz));  // SR, SL, GR, GL
  QCL_CUDA_CHECK(cudaMalloc(&b.p[6], 2 * sizeof(int)));              // status
  {
    std::vector<double> eps(NE);
    for (int e = 0; e < NE; ++e) eps[e] = -1.0 + 4.0 * e / (NE > 1 ? NE - 1 : 1);
    QCL_CUDA_CHECK(cudaMemcpyAsync(b.p[0], eps.data(), NE * sizeof(double), cudaMemcpyHostToDevice, b.st));
    QCL_CUDA_CHECK(cudaStreamSynchronize(b.st));  // eps is a temporary
  }
  QCL_CUDA_CHECK(cudaMemsetAsync(b.p[6], 0, 2 * sizeof(int), b.st));
  if (precision == QCL_C128)
    tune_fill_kernel<double><<<148 * 8, 256, 0, b.st>>>(NE, Nk, N, (Cx<double>*)b.p[1], (Cx<double>*)b.p[2],
                                                        (Cx<double>*)b.p[3]);
  else
    tune_fill_kernel<float><<<148 * 8, 256, 0, b.st>>>(NE, Nk, N, (Cx<double>*)b.p[1], (Cx<float>*)b.p[2],
                                                       (Cx<float>*)b.p[3]);
  QCL_LAUNCH_CHECK("tune_fill_kernel");
  int bi = -1;
  for (int i = 0; i < n; ++i) {
    auto launch = [&]() {
      return launch_dyson_keldysh_bpc(precision, NE, Nk, N, (const double*)b.p[0], 0.0, b.p[1], b.p[2], b.p[3],
                                      nullptr, b.p[4], b.p[5], nullptr, nullptr, nullptr, nullptr, (int*)b.p[6], b.st,
                                      0, -1, cands[i]);
    };
    int s;
    for (int w = 0; w < 2; ++w)
      if ((s = launch())) return s;
    constexpr int reps = 5;
    QCL_CUDA_CHECK(cudaEventRecord(b.e0, b.st));
    for (int r = 0; r < reps; ++r)
      if ((s = launch())) return s;
    QCL_CUDA_CHECK(cudaEventRecord(b.e1, b.st));
    QCL_CUDA_CHECK(cudaEventSynchronize(b.e1));
    float t = 0;
    QCL_CUDA_CHECK(cudaEventElapsedTime(&t, b.e0, b.e1));
    ms[i] = t / reps;
    if (bi < 0 || ms[i] < ms[bi]) bi = i;
  }
  int hst[2] = {0, 0};
  QCL_CUDA_CHECK(cudaMemcpy(hst, b.p[6], sizeof(hst), cudaMemcpyDeviceToHost));
  if (hst[0]) {
    set_last_error("autotune: the synthetic batch failed (status %d)", hst[0]);
    return hst[0];
  }
  *best = cands[bi];
  dyson_set_bpc(precision, NP, cands[bi]);
  return QCL_OK;
}

}  // namespace qcl

using namespace qcl;

extern "C" int qcl_autotune(int precision, int Nb, int NE, int Nk, qcl_tune_result* out) {
  if (precision != QCL_C128 && precision != QCL_C64 && precision != QCL_MIXED) {
    set_last_error("unknown precision %d", precision);
    return QCL_ARG;
  }
  if (!out) {
    set_last_error("autotune: out is required");
    return QCL_ARG;
  }
  qcl_tune_result r{};
  int s = autotune_dyson(precision, Nb, NE, Nk, &r.dyson_bpc, &r.candidates, r.bpc, r.ms);
  if (s) return s;
  r.default_bpc = dyson_default_bpc(precision, padded_size(Nb));
  *out = r;
  return QCL_OK;
}

extern "C" int qcl_autotune_reset(void) {
  for (int p : {QCL_C128, QCL_C64, QCL_MIXED})
    for (int np : {8, 16, 24, 32, 48}) dyson_set_bpc(p, np, 0);
  return QCL_OK;
}

extern "C" int qcl_tuned_dyson_bpc(int precision, int Nb) {
  const int np = padded_size(Nb);
  return np ? dyson_bpc(precision, np) : 0;
}
