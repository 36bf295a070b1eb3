// Reductions and element-wise field updates.
//
// Deterministic FP64 reductions: a fixed grid of REDUCE_CTAS CTAs, each
// summing a fixed strided subset in a fixed order, then one CTA combining the
// partials in CTA order.  Results therefore do not depend on scheduling, the
// GPU analogue of the reference's canonical-order sums (_canonical_sum,
// numerics/optimized/residuals.jl:493-503).
#include <math.h>

#include "kernels.cuh"

namespace qcl {

constexpr int REDUCE_CTAS = 296;  // 2 x 148 SMs
constexpr int REDUCE_THREADS = 256;

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}
__device__ __forceinline__ double warp_max(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}

// Block sum of K values per thread, result valid in thread 0.
template <int K> __device__ __forceinline__ void block_sum(double (&v)[K]) {
  __shared__ double red[K][REDUCE_THREADS / 32];
#pragma unroll
  for (int k = 0; k < K; ++k) v[k] = warp_sum(v[k]);
  if ((threadIdx.x & 31) == 0)
#pragma unroll
    for (int k = 0; k < K; ++k) red[k][threadIdx.x >> 5] = v[k];
  __syncthreads();
  if (threadIdx.x == 0) {
#pragma unroll
    for (int k = 0; k < K; ++k) {
      double s = 0;
      for (int w = 0; w < REDUCE_THREADS / 32; ++w) s += red[k][w];
      v[k] = s;
    }
  }
  __syncthreads();
}

// ---------------------------------------------------------------------------
// sum_{e,m} wE_e wk_m tr_em (complex) -> partial[cta] (2 doubles)
// ---------------------------------------------------------------------------
__global__ void weighted_trace_partial(int NE, int Nk, const Cx<double>* __restrict__ tr, const double* wE,
                                       const double* wk, double* partial) {
  const long long n = (long long)NE * Nk;
  double v[2] = {0, 0};
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const int e = (int)(i % NE), m = (int)(i / NE);
    const double w = wE[e] * wk[m];
    v[0] += w * tr[i].x;
    v[1] += w * tr[i].y;
  }
  block_sum<2>(v);
  if (threadIdx.x == 0) {
    partial[2 * blockIdx.x] = v[0];
    partial[2 * blockIdx.x + 1] = v[1];
  }
}

// Combine `count` partials of K doubles each (fixed order) into out[K].
template <int K> __global__ void combine_partials(const double* partial, int count, double* out) {
  double v[K];
#pragma unroll
  for (int k = 0; k < K; ++k) v[k] = 0;
  for (int i = threadIdx.x; i < count; i += blockDim.x)
#pragma unroll
    for (int k = 0; k < K; ++k) v[k] += partial[(size_t)K * i + k];
  block_sum<K>(v);
  if (threadIdx.x == 0)
#pragma unroll
    for (int k = 0; k < K; ++k) out[k] = v[k];
}

int launch_weighted_trace(int NE, int Nk, const void* tr, const double* wE, const double* wk, double* partial,
                          double* out, cudaStream_t st) {
  weighted_trace_partial<<<REDUCE_CTAS, REDUCE_THREADS, 0, st>>>(NE, Nk, (const Cx<double>*)tr, wE, wk,
                                                                  partial);
  combine_partials<2><<<1, REDUCE_THREADS, 0, st>>>(partial, REDUCE_CTAS, out);
  QCL_LAUNCH_CHECK("weighted_trace");
  return QCL_OK;
}

// ---------------------------------------------------------------------------
// Paired number coefficients (numerics/reference/greens.jl:155-185) from the
// weighted traces trL, trG (each (re, im) of sum wE wk tr G):
//   N = Re[-i gs/(2pi) trL] = gs/(2pi) Im trL,  H = -Re[-i gs/(2pi) trG]
// coeffs = (a, c, lambda, N, H); status gets QCL_DOMAIN / QCL_ARG.
// The realness check of number_functional (greens.jl:100-110) is applied to
// both functionals.  scalar != 0 is the occupation_normalization =
// :scalar_lesser comparator (production_state.jl:54-61): only N and lambda
// are checked (the reference never forms H there), a = 1, c = 0.
// ---------------------------------------------------------------------------
// branch: 0 = the reference's choice (scale G< when number >= target, else
// move G> weight into it); 1 or 2 forces the first or the second form (its
// formula continued across the switch), for a derivative whose explicit part
// must stay on the branch of the fixed point.
__global__ void paired_coefficients_kernel(const double* trL, const double* trG, int gs, double target,
                                           double limit, double* coeffs, int* status, int scalar, int branch) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  const double pre = gs / (2.0 * M_PI);
  // -i * pre * (x + i y) = pre * (y - i x)
  const double Nre = pre * trL[1], Nim = -pre * trL[0];
  const double Gre = pre * trG[1], Gim = -pre * trG[0];
  double number = Nre, holes = -Gre;
  coeffs[3] = number;
  coeffs[4] = holes;
  int code = 0;
  if (!(fabs(Nim) <= limit * fmax(fabs(Nre), 1.0)) ||
      (!scalar && !(fabs(Gim) <= limit * fmax(fabs(Gre), 1.0))))
    code = QCL_DOMAIN;
  double a = 1, c = 0, lam = number / target;
  if (scalar) {
    if (!code && !(isfinite(lam) && lam > 0)) code = QCL_DOMAIN;
    if (code && status) record_status(status, code, -1);
    coeffs[0] = 1.0;
    coeffs[1] = 0.0;
    coeffs[2] = lam;
    return;
  }
  if (!code) {
    if (!(isfinite(target) && target > 0)) code = QCL_ARG;
    else if (!(isfinite(lam) && lam > 0)) code = QCL_DOMAIN;
    else if (!(isfinite(number) && number > 0)) code = QCL_DOMAIN;
    else if (!(isfinite(holes) && holes >= 0)) code = QCL_DOMAIN;
    else if (!(target <= number + holes)) code = QCL_DOMAIN;
  }
  if (!code) {
    if (branch == 1 || (branch == 0 && number >= target)) {
      a = target / number;
      c = 0.0;
    } else {
      a = 1.0;
      c = (target - number) / holes;
    }
  } else {
    a = 1.0;
    c = 0.0;
    if (status) record_status(status, code, -1);
  }
  coeffs[0] = a;
  coeffs[1] = c;
  coeffs[2] = lam;
}

// realness_limit: _NUMBER_FUNCTIONAL_REALNESS_LIMIT = 1e-10 (domain/
// numerical_invariants.jl:5) for complex128 fields; complex64 fields carry
// ~1e-7 relative rounding in every diagonal element, so their limit is 1e-5.
int launch_paired_coefficients(const double* trL, const double* trG, int gs, double target, double* coeffs,
                               int* status, cudaStream_t st, double realness_limit, int scalar, int branch) {
  paired_coefficients_kernel<<<1, 32, 0, st>>>(trL, trG, gs, target, realness_limit, coeffs, status, scalar,
                                               branch);
  QCL_LAUNCH_CHECK("paired_coefficients");
  return QCL_OK;
}

// G< <- a G< - c G>,  G> <- (1-c) G> - (1-a) G<   (production_state.jl:62-70)
template <typename R>
__global__ void normalize_pair_kernel(size_t n, Cx<R>* __restrict__ GL, Cx<R>* __restrict__ GG,
                                      const double* __restrict__ coeffs) {
  const R a = (R)coeffs[0], c = (R)coeffs[1];
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const Cx<R> l = GL[i], g = GG[i];
    GL[i] = cx<R>(a * l.x - c * g.x, a * l.y - c * g.y);
    GG[i] = cx<R>((1 - c) * g.x - (1 - a) * l.x, (1 - c) * g.y - (1 - a) * l.y);
  }
}

// occupation_normalization = :scalar_lesser (production_state.jl:54-61 with
// the greater component of _green_state_production, production_operators.jl:
// 1405-1409): G< <- G< / lambda, G> <- (G^R - G^R^H) + G<.
template <typename R>
__global__ void scalar_lesser_kernel(int NE, int Nk, int N, const Cx<R>* __restrict__ GR, Cx<R>* __restrict__ GL,
                                     Cx<R>* __restrict__ GG, const double* __restrict__ coeffs) {
  const double lam = coeffs[2];
  const long long blocks = (long long)NE * Nk, n = blocks * N * N;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const long long em = i % blocks, ab = i / blocks;
    const int a = (int)(ab % N), b = (int)(ab / N);
    const Cx<R> l = GL[i], g = GR[i], gt = GR[em + blocks * ((long long)b + (long long)N * a)];
    const double lx = (double)l.x / lam, ly = (double)l.y / lam;
    GL[i] = cx<R>((R)lx, (R)ly);
    GG[i] = cx<R>((R)(((double)g.x - (double)gt.x) + lx), (R)(((double)g.y + (double)gt.y) + ly));
  }
}

static unsigned grid_for(size_t n, int threads) {
  size_t g = (n + threads - 1) / threads;
  const size_t cap = 148 * 16;
  return (unsigned)(g < cap ? (g > 0 ? g : 1) : cap);
}

int launch_normalize_pair(int precision, size_t n, void* GL, void* GG, const double* coeffs, cudaStream_t st) {
  if (precision == QCL_C128)
    normalize_pair_kernel<double><<<grid_for(n, 256), 256, 0, st>>>(n, (Cx<double>*)GL, (Cx<double>*)GG, coeffs);
  else
    normalize_pair_kernel<float><<<grid_for(n, 256), 256, 0, st>>>(n, (Cx<float>*)GL, (Cx<float>*)GG, coeffs);
  QCL_LAUNCH_CHECK("normalize_pair");
  return QCL_OK;
}

int launch_scalar_lesser(int precision, int NE, int Nk, int N, const void* GR, void* GL, void* GG,
                         const double* coeffs, cudaStream_t st) {
  const size_t n = (size_t)NE * Nk * N * N;
  if (precision == QCL_C128)
    scalar_lesser_kernel<double><<<grid_for(n, 256), 256, 0, st>>>(NE, Nk, N, (const Cx<double>*)GR, (Cx<double>*)GL,
                                                                    (Cx<double>*)GG, coeffs);
  else
    scalar_lesser_kernel<float><<<grid_for(n, 256), 256, 0, st>>>(NE, Nk, N, (const Cx<float>*)GR, (Cx<float>*)GL,
                                                                   (Cx<float>*)GG, coeffs);
  QCL_LAUNCH_CHECK("scalar_lesser");
  return QCL_OK;
}

// ---------------------------------------------------------------------------
// Integrated coherence matrix rho_ab = sum_{m,e} wE_e wk_m G<_{e,m,a,b}
// (the `integrated` array of _electron_density_bar, physics/observables.jl:
// 1-22): one CTA per (a, b), whose N_E N_k entries are contiguous in the
// E-fastest layout; fixed-order sum.
// ---------------------------------------------------------------------------
template <typename R>
__global__ void __launch_bounds__(REDUCE_THREADS)
    density_matrix_kernel(int NE, int Nk, const Cx<R>* __restrict__ GL, const double* __restrict__ wE,
                          const double* __restrict__ wk, double* out) {
  const long long blocks = (long long)NE * Nk;
  const Cx<R>* g = GL + (size_t)blockIdx.x * blocks;
  double v[2] = {0, 0};
  for (long long i = threadIdx.x; i < blocks; i += blockDim.x) {
    const double w = wE[i % NE] * wk[i / NE];
    const Cx<R> z = g[i];
    v[0] += w * (double)z.x;
    v[1] += w * (double)z.y;
  }
  block_sum<2>(v);
  if (threadIdx.x == 0) {
    out[2 * blockIdx.x] = v[0];
    out[2 * blockIdx.x + 1] = v[1];
  }
}

int launch_density_matrix(int precision, int NE, int Nk, int N, const void* GL, const double* wE, const double* wk,
                          double* out, cudaStream_t st) {
  if (precision == QCL_C128)
    density_matrix_kernel<double><<<N * N, REDUCE_THREADS, 0, st>>>(NE, Nk, (const Cx<double>*)GL, wE, wk, out);
  else
    density_matrix_kernel<float><<<N * N, REDUCE_THREADS, 0, st>>>(NE, Nk, (const Cx<float>*)GL, wE, wk, out);
  QCL_LAUNCH_CHECK("density_matrix");
  return QCL_OK;
}

// ---------------------------------------------------------------------------
// Sum of up to 8 fields (component-wise totals, _total_family_production,
// production_operators.jl:1447-1473): out = sum_j src[j].
// ---------------------------------------------------------------------------
template <typename R> struct SumArgs {
  const Cx<R>* src[8];
  int count;
  Cx<R>* out;
  size_t n;
};

template <typename R> __global__ void sum_fields_kernel(SumArgs<R> p) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < p.n; i += (size_t)gridDim.x * blockDim.x) {
    Cx<R> v = p.src[0][i];
    for (int j = 1; j < p.count; ++j) v = v + p.src[j][i];
    p.out[i] = v;
  }
}
// complex64 with 16-byte aligned fields and even n: two elements per 16-byte
// access (the same per-element sums)
__global__ void sum_fields_pair_kernel(SumArgs<float> p) {
  const size_t n2 = p.n / 2;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n2; i += (size_t)gridDim.x * blockDim.x) {
    float4 v = reinterpret_cast<const float4*>(p.src[0])[i];
    for (int j = 1; j < p.count; ++j) {
      const float4 w = reinterpret_cast<const float4*>(p.src[j])[i];
      v.x += w.x;
      v.y += w.y;
      v.z += w.z;
      v.w += w.w;
    }
    reinterpret_cast<float4*>(p.out)[i] = v;
  }
}
static bool aligned16(const void* q) { return ((uintptr_t)q & 15u) == 0; }

int launch_sum_fields(int precision, size_t n, const void* const* src, int count, void* out, cudaStream_t st) {
  if (count < 1 || count > 8) {
    set_last_error("sum_fields: 1..8 inputs supported, got %d", count);
    return QCL_ARG;
  }
  if (precision == QCL_C128) {
    SumArgs<double> a;
    for (int j = 0; j < count; ++j) a.src[j] = (const Cx<double>*)src[j];
    a.count = count;
    a.out = (Cx<double>*)out;
    a.n = n;
    sum_fields_kernel<double><<<grid_for(n, 256), 256, 0, st>>>(a);
  } else {
    SumArgs<float> a;
    bool pairs = n % 2 == 0 && aligned16(out);
    for (int j = 0; j < count; ++j) {
      a.src[j] = (const Cx<float>*)src[j];
      pairs = pairs && aligned16(src[j]);
    }
    a.count = count;
    a.out = (Cx<float>*)out;
    a.n = n;
    if (pairs) sum_fields_pair_kernel<<<grid_for(n / 2, 256), 256, 0, st>>>(a);
    else sum_fields_kernel<float><<<grid_for(n, 256), 256, 0, st>>>(a);
  }
  QCL_LAUNCH_CHECK("sum_fields");
  return QCL_OK;
}

// ---------------------------------------------------------------------------
// Fused self-energy residual + linear mixing for one component:
//   partial <- (|new - old|^2, |new|^2) per CTA, non-finite -> +inf
//   mixed   <- (1 - alpha) old + alpha new        (written over `new_`)
// r_Sigma = sqrt(sum d^2) / (sqrt(sum n^2) + 1e-14)
// (production_selfenergy_residual, numerics/optimized/residuals.jl:802-865;
// _mix_family_production!, production_operators.jl:1475-1490).
// With alpha <= 0 no mixing happens (residual only).
// ---------------------------------------------------------------------------
template <typename R>
__global__ void residual_mix_kernel(size_t n, const Cx<R>* __restrict__ old, Cx<R>* __restrict__ new_, double alpha,
                                    double* partial) {
  double v[2] = {0, 0};
  const R al = (R)alpha, be = (R)(1.0 - alpha);
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const Cx<R> o = old[i], c = new_[i];
    const double dx = (double)c.x - o.x, dy = (double)c.y - o.y;
    const double d2 = dx * dx + dy * dy, n2 = (double)c.x * c.x + (double)c.y * c.y;
    if (isfinite(d2) && isfinite(n2) && isfinite((double)o.x) && isfinite((double)o.y)) {
      v[0] += d2;
      v[1] += n2;
    } else {
      v[0] = INFINITY;
    }
    if (alpha > 0) new_[i] = cx<R>(be * o.x + al * c.x, be * o.y + al * c.y);
  }
  block_sum<2>(v);
  if (threadIdx.x == 0) {
    partial[2 * blockIdx.x] = v[0];
    partial[2 * blockIdx.x + 1] = v[1];
  }
}

int launch_residual_mix(int precision, size_t n, const void* old, void* new_, double alpha, double* partial,
                        double* out2, cudaStream_t st) {
  if (precision == QCL_C128)
    residual_mix_kernel<double><<<REDUCE_CTAS, REDUCE_THREADS, 0, st>>>(n, (const Cx<double>*)old,
                                                                        (Cx<double>*)new_, alpha, partial);
  else
    residual_mix_kernel<float><<<REDUCE_CTAS, REDUCE_THREADS, 0, st>>>(n, (const Cx<float>*)old, (Cx<float>*)new_,
                                                                       alpha, partial);
  combine_partials<2><<<1, REDUCE_THREADS, 0, st>>>(partial, REDUCE_CTAS, out2);
  QCL_LAUNCH_CHECK("residual_mix");
  return QCL_OK;
}

// All state/candidate field pairs of an iteration in one launch: blockIdx.y
// selects the field, MIX_CTAS CTAs per field write (|new - old|^2, |new|^2)
// partials and mix new <- (1 - alpha) old + alpha new in place.
constexpr int MIX_CTAS = 64;
template <typename R> struct MixFields {
  const Cx<R>* old[kMaxMixFields];
  Cx<R>* cand[kMaxMixFields];
};

template <typename R>
__global__ void __launch_bounds__(REDUCE_THREADS) residual_mix_multi_kernel(size_t n, MixFields<R> f, double alpha,
                                                                            double* partial) {
  const Cx<R>* __restrict__ old = f.old[blockIdx.y];
  Cx<R>* __restrict__ new_ = f.cand[blockIdx.y];
  double v[2] = {0, 0};
  const R al = (R)alpha, be = (R)(1.0 - alpha);
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const Cx<R> o = old[i], c = new_[i];
    const double dx = (double)c.x - o.x, dy = (double)c.y - o.y;
    const double d2 = dx * dx + dy * dy, n2 = (double)c.x * c.x + (double)c.y * c.y;
    if (isfinite(d2) && isfinite(n2) && isfinite((double)o.x) && isfinite((double)o.y)) {
      v[0] += d2;
      v[1] += n2;
    } else {
      v[0] = INFINITY;
    }
    if (alpha > 0) new_[i] = cx<R>(be * o.x + al * c.x, be * o.y + al * c.y);
  }
  block_sum<2>(v);
  if (threadIdx.x == 0) {
    double* pp = partial + 2 * ((size_t)blockIdx.y * gridDim.x + blockIdx.x);
    pp[0] = v[0];
    pp[1] = v[1];
  }
}

// complex64 with 16-byte aligned fields and even n: two elements per 16-byte
// access, each with the arithmetic of residual_mix_multi_kernel.
__global__ void __launch_bounds__(REDUCE_THREADS) residual_mix_multi_pair_kernel(size_t n, MixFields<float> f,
                                                                                double alpha, double* partial) {
  const float4* __restrict__ old = reinterpret_cast<const float4*>(f.old[blockIdx.y]);
  float4* __restrict__ new_ = reinterpret_cast<float4*>(f.cand[blockIdx.y]);
  double v[2] = {0, 0};
  const float al = (float)alpha, be = (float)(1.0 - alpha);
  const size_t n2 = n / 2;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n2; i += (size_t)gridDim.x * blockDim.x) {
    const float4 o4 = old[i], c4 = new_[i];
    const Cx<float> os[2] = {cx<float>(o4.x, o4.y), cx<float>(o4.z, o4.w)};
    const Cx<float> cs[2] = {cx<float>(c4.x, c4.y), cx<float>(c4.z, c4.w)};
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const Cx<float> o = os[h], c = cs[h];
      const double dx = (double)c.x - o.x, dy = (double)c.y - o.y;
      const double d2 = dx * dx + dy * dy, n2v = (double)c.x * c.x + (double)c.y * c.y;
      if (isfinite(d2) && isfinite(n2v) && isfinite((double)o.x) && isfinite((double)o.y)) {
        v[0] += d2;
        v[1] += n2v;
      } else {
        v[0] = INFINITY;
      }
    }
    if (alpha > 0)
      new_[i] = make_float4(be * os[0].x + al * cs[0].x, be * os[0].y + al * cs[0].y, be * os[1].x + al * cs[1].x,
                            be * os[1].y + al * cs[1].y);
  }
  block_sum<2>(v);
  if (threadIdx.x == 0) {
    double* pp = partial + 2 * ((size_t)blockIdx.y * gridDim.x + blockIdx.x);
    pp[0] = v[0];
    pp[1] = v[1];
  }
}

// One CTA per segment: out[2 s + k] = sum_c partial[s][c][k], fixed order.
__global__ void combine_segments_kernel(const double* partial, int count, double* out) {
  const double* seg = partial + 2 * (size_t)blockIdx.x * count;
  double v[2] = {0, 0};
  for (int i = threadIdx.x; i < count; i += blockDim.x) {
    v[0] += seg[2 * i];
    v[1] += seg[2 * i + 1];
  }
  block_sum<2>(v);
  if (threadIdx.x == 0) {
    out[2 * blockIdx.x] = v[0];
    out[2 * blockIdx.x + 1] = v[1];
  }
}

size_t residual_mix_multi_partial_doubles(int nf) { return 2 * (size_t)MIX_CTAS * nf; }

int launch_residual_mix_multi(int precision, size_t n, const void* const* old, void* const* cand, int nf,
                              double alpha, double* partial, double* out, cudaStream_t st) {
  if (nf <= 0) return QCL_OK;
  if (nf > kMaxMixFields) {
    set_last_error("residual_mix: %d fields exceed %d", nf, kMaxMixFields);
    return QCL_ARG;
  }
  const dim3 grid(MIX_CTAS, nf);
  if (precision == QCL_C128) {
    MixFields<double> f{};
    for (int i = 0; i < nf; ++i) {
      f.old[i] = (const Cx<double>*)old[i];
      f.cand[i] = (Cx<double>*)cand[i];
    }
    residual_mix_multi_kernel<double><<<grid, REDUCE_THREADS, 0, st>>>(n, f, alpha, partial);
  } else {
    MixFields<float> f{};
    bool pairs = n % 2 == 0;
    for (int i = 0; i < nf; ++i) {
      f.old[i] = (const Cx<float>*)old[i];
      f.cand[i] = (Cx<float>*)cand[i];
      pairs = pairs && aligned16(old[i]) && aligned16(cand[i]);
    }
    if (pairs) residual_mix_multi_pair_kernel<<<grid, REDUCE_THREADS, 0, st>>>(n, f, alpha, partial);
    else residual_mix_multi_kernel<float><<<grid, REDUCE_THREADS, 0, st>>>(n, f, alpha, partial);
  }
  combine_segments_kernel<<<nf, REDUCE_THREADS, 0, st>>>(partial, MIX_CTAS, out);
  QCL_LAUNCH_CHECK("residual_mix_multi");
  return QCL_OK;
}

int launch_combine(const double* partial, int count, int K, double* out, cudaStream_t st) {
  switch (K) {
    case 1: combine_partials<1><<<1, REDUCE_THREADS, 0, st>>>(partial, count, out); break;
    case 2: combine_partials<2><<<1, REDUCE_THREADS, 0, st>>>(partial, count, out); break;
    case 4: combine_partials<4><<<1, REDUCE_THREADS, 0, st>>>(partial, count, out); break;
    default: set_last_error("combine: K=%d unsupported", K); return QCL_ARG;
  }
  QCL_LAUNCH_CHECK("combine_partials");
  return QCL_OK;
}

// out = a x + b y (complex fields; used for pairwise embedding totals)
template <typename R>
__global__ void axpby_kernel(size_t n, double a, const Cx<R>* x, double b, const Cx<R>* y, Cx<R>* out) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const Cx<R> u = x[i], v = y[i];
    out[i] = cx<R>((R)(a * u.x + b * v.x), (R)(a * u.y + b * v.y));
  }
}

int launch_axpby(int precision, size_t n, double a, const void* x, double b, const void* y, void* out,
                 cudaStream_t st) {
  if (precision == QCL_C128)
    axpby_kernel<double><<<grid_for(n, 256), 256, 0, st>>>(n, a, (const Cx<double>*)x, b, (const Cx<double>*)y,
                                                           (Cx<double>*)out);
  else
    axpby_kernel<float><<<grid_for(n, 256), 256, 0, st>>>(n, a, (const Cx<float>*)x, b, (const Cx<float>*)y,
                                                          (Cx<float>*)out);
  QCL_LAUNCH_CHECK("axpby");
  return QCL_OK;
}

}  // namespace qcl
