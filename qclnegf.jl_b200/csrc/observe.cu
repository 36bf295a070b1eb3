// Current and population reductions (FP64, fixed-order).
//
// Current (_production_boundary_flux_bar, numerics/optimized/production_
// iteration.jl:174-201; oracle _boundary_flux_complex, physics/observables.jl:
// 176-214):
//   Jbar = Re[ g_s/(2 pi) sum_{e,m} wE_e wk_m sum_{a,b}
//              (S>_{em,ab} G<_{em,ba} - S<_{em,ab} G>_{em,ba}) ]
// Populations (_production_state_populations, production_iteration.jl:
// 204-215):  p_a = Re[-i g_s/(2 pi) sum_{e,m} wE wk G<_{em,aa}] / target.
//
// The reference accumulates the current in (|eps|, eps) order to limit
// cancellation; here every term is accumulated in FP64 by a fixed two-level
// tree (per-thread strided sums, fixed CTA partials combined in CTA order),
// which is deterministic and whose rounding is of the same order.
#include "kernels.cuh"

namespace qcl {

constexpr int OBS_CTAS = 296, OBS_THREADS = 256;

__device__ __forceinline__ double wsum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

template <int K> __device__ __forceinline__ void cta_sum(double (&v)[K], double* out) {
  __shared__ double red[K][OBS_THREADS / 32];
#pragma unroll
  for (int k = 0; k < K; ++k) v[k] = wsum(v[k]);
  if ((threadIdx.x & 31) == 0)
#pragma unroll
    for (int k = 0; k < K; ++k) red[k][threadIdx.x >> 5] = v[k];
  __syncthreads();
  if (threadIdx.x == 0)
#pragma unroll
    for (int k = 0; k < K; ++k) {
      double s = 0;
      for (int w = 0; w < OBS_THREADS / 32; ++w) s += red[k][w];
      out[k] = s;
    }
}

template <typename R>
__global__ void current_partial_kernel(int NE, int Nk, int N, const double* __restrict__ wE,
                                       const double* __restrict__ wk, const Cx<R>* __restrict__ SG,
                                       const Cx<R>* __restrict__ SL, const Cx<R>* __restrict__ GL,
                                       const Cx<R>* __restrict__ GG, double* partial) {
  const long long n = (long long)NE * Nk * N * N;
  const long long blocks = (long long)NE * Nk;
  double v[2] = {0, 0};
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const long long em = i % blocks, ab = i / blocks;
    const int e = (int)(em % NE), m = (int)(em / NE);
    const int a = (int)(ab % N), b = (int)(ab / N);
    const long long it = em + blocks * ((long long)b + (long long)N * a);  // (e, m, b, a)
    const Cx<R> sg = SG[i], sl = SL[i], gl = GL[it], gg = GG[it];
    const double w = wE[e] * wk[m];
    const double re = ((double)sg.x * gl.x - (double)sg.y * gl.y) - ((double)sl.x * gg.x - (double)sl.y * gg.y);
    const double im = ((double)sg.x * gl.y + (double)sg.y * gl.x) - ((double)sl.x * gg.y + (double)sl.y * gg.x);
    v[0] += w * re;
    v[1] += w * im;
  }
  cta_sum<2>(v, partial + 2 * blockIdx.x);
}

template <typename R>
__global__ void population_partial_kernel(int NE, int Nk, int N, const double* __restrict__ wE,
                                          const double* __restrict__ wk, const Cx<R>* __restrict__ GL,
                                          double* partial) {
  const int a = blockIdx.y;
  const long long blocks = (long long)NE * Nk;
  const size_t off = (size_t)blocks * ((size_t)a + (size_t)N * a);
  double v[2] = {0, 0};
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < blocks;
       i += (long long)gridDim.x * blockDim.x) {
    const int e = (int)(i % NE), m = (int)(i / NE);
    const Cx<R> g = GL[off + i];
    const double w = wE[e] * wk[m];
    v[0] += w * g.x;
    v[1] += w * g.y;
  }
  cta_sum<2>(v, partial + 2 * ((size_t)a * gridDim.x + blockIdx.x));
}

// Combines partials into the final scalars:
//   out[0] = Jbar, out[1] = Im of the complex flux (diagnostic),
//   out[2 + a] = p_a.
// One CTA per quantity (current, then each population), fixed-order sums.
__global__ void observables_combine_kernel(int N, int ncta, const double* cur, const double* pop, int gs, double target,
                                           double* out) {
  const int q = blockIdx.x;  // 0: current, 1 + a: population a
  const double* src = q == 0 ? cur : pop + 2 * (size_t)(q - 1) * ncta;
  double re = 0, im = 0;
  for (int c = threadIdx.x; c < ncta; c += blockDim.x) {
    re += src[2 * c];
    im += src[2 * c + 1];
  }
  __shared__ double red[2][32];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    re += __shfl_xor_sync(0xffffffffu, re, o);
    im += __shfl_xor_sync(0xffffffffu, im, o);
  }
  if ((threadIdx.x & 31) == 0) {
    red[0][threadIdx.x >> 5] = re;
    red[1][threadIdx.x >> 5] = im;
  }
  __syncthreads();
  if (threadIdx.x != 0) return;
  re = 0;
  im = 0;
  for (int w = 0; w < (int)(blockDim.x >> 5); ++w) {
    re += red[0][w];
    im += red[1][w];
  }
  const double pre = gs / (2.0 * M_PI);
  if (q == 0) {
    out[0] = pre * re;
    out[1] = pre * im;
  } else {
    // -i pre (re + i im) = pre (im - i re): real part = pre * im
    out[1 + q] = pre * im / target;
  }
}

size_t observables_partial_doubles(int N) { return 2 * (size_t)OBS_CTAS * (1 + N); }

// SG, SL: the plus-embedding family (Sigma+^>, Sigma+^<); GL, GG: the state.
int launch_observables(int precision, int NE, int Nk, int N, const double* wE, const double* wk, const void* SG,
                       const void* SL, const void* GL, const void* GG, int gs, double target, double* partial,
                       double* out, cudaStream_t st) {
  double* cur = partial;
  double* pop = partial + 2 * OBS_CTAS;
  if (precision == QCL_C128) {
    current_partial_kernel<double><<<OBS_CTAS, OBS_THREADS, 0, st>>>(NE, Nk, N, wE, wk, (const Cx<double>*)SG,
                                                                     (const Cx<double>*)SL, (const Cx<double>*)GL,
                                                                     (const Cx<double>*)GG, cur);
    population_partial_kernel<double><<<dim3(OBS_CTAS, N), OBS_THREADS, 0, st>>>(NE, Nk, N, wE, wk,
                                                                                 (const Cx<double>*)GL, pop);
  } else {
    current_partial_kernel<float><<<OBS_CTAS, OBS_THREADS, 0, st>>>(NE, Nk, N, wE, wk, (const Cx<float>*)SG,
                                                                    (const Cx<float>*)SL, (const Cx<float>*)GL,
                                                                    (const Cx<float>*)GG, cur);
    population_partial_kernel<float><<<dim3(OBS_CTAS, N), OBS_THREADS, 0, st>>>(NE, Nk, N, wE, wk,
                                                                                (const Cx<float>*)GL, pop);
  }
  observables_combine_kernel<<<1 + N, 128, 0, st>>>(N, OBS_CTAS, cur, pop, gs, target, out);
  QCL_LAUNCH_CHECK("observables");
  return QCL_OK;
}

}  // namespace qcl
