// Seed-state kernels and the embedding-total residual.
#include <math.h>

#include "kernels.cuh"

namespace qcl {

static unsigned gcap(long long n, int t) {
  long long g = (n + t - 1) / t;
  return (unsigned)(g < 148 * 16 ? (g > 0 ? g : 1) : 148 * 16);
}

// q_e = g_s/(2 pi) wE_e sum_m wk_m tr A_em, A = i(GR - GR^H)
// (_seed_number_weights_production, numerics/optimized/seed.jl:28-66).
template <typename R>
__global__ void seed_weights_kernel(int NE, int Nk, int N, const Cx<R>* __restrict__ GR, const double* __restrict__ wE,
                                    const double* __restrict__ wk, int gs, double* q) {
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < NE; e += gridDim.x * blockDim.x) {
    double msum = 0;
    for (int m = 0; m < Nk; ++m) {
      double trA = 0;
      for (int a = 0; a < N; ++a) {
        const Cx<R> z = GR[(size_t)e + (size_t)NE * ((size_t)m + (size_t)Nk * ((size_t)a + (size_t)N * a))];
        trA += -2.0 * (double)z.y;  // real(i (z - conj z)) = -2 Im z
      }
      msum += wk[m] * trA;
    }
    q[e] = gs / (2.0 * M_PI) * wE[e] * msum;
  }
}

int launch_seed_weights(int precision, int NE, int Nk, int N, const void* GR, const double* wE, const double* wk,
                        int gs, double* q, cudaStream_t st) {
  if (precision == QCL_C128)
    seed_weights_kernel<double><<<gcap(NE, 128), 128, 0, st>>>(NE, Nk, N, (const Cx<double>*)GR, wE, wk, gs, q);
  else
    seed_weights_kernel<float><<<gcap(NE, 128), 128, 0, st>>>(NE, Nk, N, (const Cx<float>*)GR, wE, wk, gs, q);
  QCL_LAUNCH_CHECK("seed_weights");
  return QCL_OK;
}

// G< = -f(eps_e) (GR - GR^H)  (_seed_lesser_production!, seed.jl:99-128),
// G> = GR - GR^H + G<        (greater_green, numerics/reference/greens.jl:84-93).
template <typename R>
__global__ void seed_green_kernel(int NE, int Nk, int N, const Cx<R>* __restrict__ GR, const double* __restrict__ f,
                                  Cx<R>* __restrict__ GL, Cx<R>* __restrict__ GG) {
  const long long blocks = (long long)NE * Nk, n = blocks * N * N;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const long long em = i % blocks, ab = i / blocks;
    const int e = (int)(em % NE);
    const int a = (int)(ab % N), b = (int)(ab / N);
    const Cx<R> g = GR[i], gt = GR[em + blocks * ((long long)b + (long long)N * a)];
    const double dx = (double)g.x - gt.x, dy = (double)g.y + gt.y;  // GR - GR^H
    const double fe = f[e];
    const double lx = -fe * dx, ly = -fe * dy;
    GL[i] = cx<R>((R)lx, (R)ly);
    GG[i] = cx<R>((R)(dx + lx), (R)(dy + ly));
  }
}

int launch_seed_green(int precision, int NE, int Nk, int N, const void* GR, const double* f, void* GL, void* GG,
                      cudaStream_t st) {
  const long long n = (long long)NE * Nk * N * N;
  if (precision == QCL_C128)
    seed_green_kernel<double><<<gcap(n, 256), 256, 0, st>>>(NE, Nk, N, (const Cx<double>*)GR, f, (Cx<double>*)GL,
                                                           (Cx<double>*)GG);
  else
    seed_green_kernel<float><<<gcap(n, 256), 256, 0, st>>>(NE, Nk, N, (const Cx<float>*)GR, f, (Cx<float>*)GL,
                                                          (Cx<float>*)GG);
  QCL_LAUNCH_CHECK("seed_green");
  return QCL_OK;
}

// Residual of a sum of two families against the sum of their candidates
// (the embedding total = plus + minus, _selfenergy_residual(embedding,
// candidate_embedding), numerics/reference/scba.jl:236):
//   partial <- (|(n1 + n2) - (o1 + o2)|^2, |n1 + n2|^2) per CTA.
template <typename R>
__global__ void residual_pair_kernel(size_t n, const Cx<R>* __restrict__ o1, const Cx<R>* __restrict__ o2,
                                     const Cx<R>* __restrict__ n1, const Cx<R>* __restrict__ n2, double* partial) {
  double d2 = 0, s2 = 0;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const double nx = (double)n1[i].x + n2[i].x, ny = (double)n1[i].y + n2[i].y;
    const double dx = nx - ((double)o1[i].x + o2[i].x), dy = ny - ((double)o1[i].y + o2[i].y);
    const double a = dx * dx + dy * dy, b = nx * nx + ny * ny;
    if (isfinite(a) && isfinite(b)) {
      d2 += a;
      s2 += b;
    } else {
      d2 = INFINITY;
    }
  }
  __shared__ double red[2][8];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    d2 += __shfl_xor_sync(0xffffffffu, d2, o);
    s2 += __shfl_xor_sync(0xffffffffu, s2, o);
  }
  if ((threadIdx.x & 31) == 0) {
    red[0][threadIdx.x >> 5] = d2;
    red[1][threadIdx.x >> 5] = s2;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double a = 0, b = 0;
    for (int w = 0; w < 8; ++w) {
      a += red[0][w];
      b += red[1][w];
    }
    partial[2 * blockIdx.x] = a;
    partial[2 * blockIdx.x + 1] = b;
  }
}

int launch_residual_pair(int precision, size_t n, const void* o1, const void* o2, const void* n1, const void* n2,
                         double* partial, double* out2, cudaStream_t st) {
  if (precision == QCL_C128)
    residual_pair_kernel<double><<<kReduceCtas, 256, 0, st>>>(n, (const Cx<double>*)o1, (const Cx<double>*)o2,
                                                              (const Cx<double>*)n1, (const Cx<double>*)n2, partial);
  else
    residual_pair_kernel<float><<<kReduceCtas, 256, 0, st>>>(n, (const Cx<float>*)o1, (const Cx<float>*)o2,
                                                             (const Cx<float>*)n1, (const Cx<float>*)n2, partial);
  QCL_LAUNCH_CHECK("residual_pair");
  return launch_combine(partial, kReduceCtas, 2, out2, st);
}

// Precision conversion of a host complex128 array into a device array of the
// field precision (kernel operators, Hamiltonians of the mixed path).
template <typename R> __global__ void convert_kernel(size_t n, const Cx<double>* __restrict__ in, Cx<R>* __restrict__ out) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    out[i] = cvt<R>(in[i]);
}

int launch_convert(int precision, size_t n, const void* in_c128, void* out, cudaStream_t st) {
  if (precision == QCL_C128) {
    QCL_CUDA_CHECK(cudaMemcpyAsync(out, in_c128, n * 16, cudaMemcpyDeviceToDevice, st));
    return QCL_OK;
  }
  convert_kernel<float><<<gcap((long long)n, 256), 256, 0, st>>>(n, (const Cx<double>*)in_c128, (Cx<float>*)out);
  QCL_LAUNCH_CHECK("convert");
  return QCL_OK;
}

// complex64 -> complex128 (exact): the FP64 refinement of a mixed-precision
// state.
__global__ void promote_kernel(size_t n, const Cx<float>* __restrict__ in, Cx<double>* __restrict__ out) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const Cx<float> v = in[i];
    out[i] = cx<double>((double)v.x, (double)v.y);
  }
}

// X <- (X - X^H) / 2 per (e, m) block of a complex128 field, in place: one
// thread per unordered pair (a <= b).
__global__ void antihermitian_kernel(int NE, int Nk, int N, Cx<double>* X) {
  const long long blocks = (long long)NE * Nk, pairs = (long long)N * (N + 1) / 2;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < blocks * pairs;
       i += (long long)gridDim.x * blockDim.x) {
    const long long blk = i % blocks;
    int q = (int)(i / blocks), b = 0;
    while (q >= N - b) {  // pair index -> (a, b), a >= b
      q -= N - b;
      ++b;
    }
    const int a = b + q;
    Cx<double>* pab = X + blk + blocks * ((long long)a + (long long)N * b);
    Cx<double>* pba = X + blk + blocks * ((long long)b + (long long)N * a);
    const Cx<double> u = *pab, v = *pba;
    // (X - X^H)_ab / 2 = (u - conj v) / 2, and (X - X^H)_ba = -conj of it
    const Cx<double> w = cx<double>(0.5 * (u.x - v.x), 0.5 * (u.y + v.y));
    *pab = w;
    *pba = cx<double>(-w.x, w.y);
  }
}

int launch_antihermitian_part(int NE, int Nk, int N, void* X, cudaStream_t st) {
  const long long n = (long long)NE * Nk * N * (N + 1) / 2;
  antihermitian_kernel<<<gcap(n, 256), 256, 0, st>>>(NE, Nk, N, (Cx<double>*)X);
  QCL_LAUNCH_CHECK("antihermitian");
  return QCL_OK;
}

int launch_promote(size_t n, const void* in_c64, void* out_c128, cudaStream_t st) {
  promote_kernel<<<gcap((long long)n, 256), 256, 0, st>>>(n, (const Cx<float>*)in_c64, (Cx<double>*)out_c128);
  QCL_LAUNCH_CHECK("promote");
  return QCL_OK;
}

}  // namespace qcl
