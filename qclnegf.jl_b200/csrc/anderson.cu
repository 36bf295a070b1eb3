// Anderson mixing of the SCBA self-energy families, device-resident.
//
// Reference: _anderson_mix! and its helpers (numerics/optimized/
// production_mixing.jl:120-317), called on the ordered families
// [mechanisms..., plus, minus] (production_solver.jl:798-818):
//   append:   R = candidate - state; the history keeps (state, R) for the last
//             `depth` steps and the Gram matrix G_ij = Re <R_i, R_j> summed
//             over every family and component (_anderson_inner, :129-138);
//             the history is cleared first when <R, R> exceeds the previous
//             entry's by more than (1 + 64 eps) (_anderson_append!, :189-222);
//   solve:    (G + reg s I) / s, s = max(max_i |G_ii|, eps), by a symmetric
//             eigen-decomposition; eigenvalues below max(reg, sqrt eps) are
//             dropped; c = V diag(1/lambda) V^T 1 normalised to sum 1
//             (_anderson_coefficients, :155-180); a failed solve or
//             sum |c| > 10 falls back to the newest entry alone (:240-250);
//   mix:      state = sum_j c_j (x_j + alpha damping R_j)       (:252-264);
//   guard:    every block of every family must stay causal and
//             Keldysh-consistent (_anderson_block_failure!, :48-96); if not,
//             the linear step x_last + alpha damping R_last replaces the
//             mixed state and the history is cleared; a linear step that
//             also fails is a DomainError (:266-282).
// The mixer state lives in device memory (AndersonMeta), so every decision
// is taken by a kernel and an iteration stays a plain stream-ordered (and
// graph-capturable) launch sequence.  Reductions run on a fixed grid and are
// combined in a fixed order.
#include <float.h>
#include <math.h>

#include "kernels.cuh"

namespace qcl {

constexpr int AND_CTAS = 64;       // CTAs per field in the append pass
constexpr int AND_THREADS = 256;
constexpr int AND_K = kAndersonMaxDepth + 2;  // per-CTA partials: num, den, dots[0..depth-1] (last = <R,R>)
constexpr int MD = kAndersonMaxDepth;
constexpr unsigned long long kNoFailure = ~0ull;

template <int K> __device__ __forceinline__ void and_block_sum(double (&v)[K]) {
  __shared__ double red[K][AND_THREADS / 32];
#pragma unroll
  for (int k = 0; k < K; ++k) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v[k] += __shfl_xor_sync(0xffffffffu, v[k], o);
  }
  if ((threadIdx.x & 31) == 0)
#pragma unroll
    for (int k = 0; k < K; ++k) red[k][threadIdx.x >> 5] = v[k];
  __syncthreads();
  if (threadIdx.x == 0)
#pragma unroll
    for (int k = 0; k < K; ++k) {
      double s = 0;
      for (int w = 0; w < AND_THREADS / 32; ++w) s += red[k][w];
      v[k] = s;
    }
  __syncthreads();
}

size_t anderson_partial_doubles(int nf) { return (size_t)AND_K * AND_CTAS * nf; }

__global__ void anderson_reset_kernel(AndersonMeta* m) {
  m->count = 0;
  m->head = 0;
  m->slot = 0;
  m->reason = 0;
  m->fallback = 0;
  m->accepted = 0;
  m->used = 0;
  m->guard_code = 0;
  m->guard_key = kNoFailure;
  m->guard_first = 0;
  m->prior = -1.0;
  m->l1 = 0.0;
}

int launch_anderson_reset(AndersonMeta* m, cudaStream_t st) {
  anderson_reset_kernel<<<1, 1, 0, st>>>(m);
  QCL_LAUNCH_CHECK("anderson_reset");
  return QCL_OK;
}

// Prior residual norm, eviction of the oldest entry, slot of the new one.
__global__ void anderson_plan_kernel(AndersonMeta* m, int depth) {
  const int c = m->count;
  m->prior = c > 0 ? m->gram[(c - 1) * MD + (c - 1)] : -1.0;
  if (c >= depth) {  // evict before the new entry is written (production_mixing.jl:192-197)
    m->head = (m->head + 1) % depth;
    for (int i = 0; i < c - 1; ++i)
      for (int j = 0; j < c - 1; ++j) m->gram[i * MD + j] = m->gram[(i + 1) * MD + (j + 1)];
    m->count = c - 1;
  }
  m->slot = (m->head + m->count) % depth;
  m->reason = 0;
  m->fallback = 0;
  m->accepted = 0;
  m->guard_code = 0;
  m->guard_key = kNoFailure;
  m->guard_first = 0;
}

int launch_anderson_plan(AndersonMeta* m, int depth, cudaStream_t st) {
  anderson_plan_kernel<<<1, 1, 0, st>>>(m, depth);
  QCL_LAUNCH_CHECK("anderson_plan");
  return QCL_OK;
}

template <typename R> struct AndFields {
  const Cx<R>* state[kMaxMixFields];
  const Cx<R>* cand[kMaxMixFields];
};

// Field blockIdx.y: saves x and R = c - x into the new slot and accumulates
// |c - x|^2, |c|^2 (the family residual r_Sigma) and Re <R_j, R> for the
// current history entries j plus <R, R>.
template <typename R>
__global__ void __launch_bounds__(AND_THREADS)
    anderson_append_kernel(size_t n, AndFields<R> f, int nf, Cx<R>* __restrict__ Xh, Cx<R>* __restrict__ Rh,
                           int depth, const AndersonMeta* __restrict__ m, double* partial) {
  const int fld = blockIdx.y;
  const Cx<R>* __restrict__ st = f.state[fld];
  const Cx<R>* __restrict__ cd = f.cand[fld];
  const int count = m->count, head = m->head, slot = m->slot;
  Cx<R>* xs = Xh + ((size_t)slot * nf + fld) * n;
  Cx<R>* rs = Rh + ((size_t)slot * nf + fld) * n;
  const Cx<R>* hist[MD];
  for (int j = 0; j < MD; ++j)
    hist[j] = j < count ? Rh + ((size_t)((head + j) % depth) * nf + fld) * n : nullptr;
  double v[AND_K];
#pragma unroll
  for (int k = 0; k < AND_K; ++k) v[k] = 0;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const Cx<R> x = st[i], c = cd[i];
    const double rx = (double)c.x - (double)x.x, ry = (double)c.y - (double)x.y;
    const double d2 = rx * rx + ry * ry, n2 = (double)c.x * c.x + (double)c.y * c.y;
    if (isfinite(d2) && isfinite(n2) && isfinite((double)x.x) && isfinite((double)x.y)) {
      v[0] += d2;
      v[1] += n2;
    } else {
      v[0] = INFINITY;
    }
    xs[i] = x;
    const Cx<R> r = cx<R>((R)rx, (R)ry);
    rs[i] = r;
#pragma unroll
    for (int j = 0; j < MD; ++j)
      if (j < count) {
        const Cx<R> q = hist[j][i];
        v[2 + j] += (double)q.x * (double)r.x + (double)q.y * (double)r.y;
      }
    // <R, R> at index count (in storage precision, as the history holds it)
    const double sr = (double)r.x * (double)r.x + (double)r.y * (double)r.y;
#pragma unroll
    for (int j = 0; j < MD; ++j)
      if (j == count) v[2 + j] += sr;
  }
  and_block_sum<AND_K>(v);
  if (threadIdx.x == 0) {
    double* pp = partial + (size_t)AND_K * ((size_t)fld * gridDim.x + blockIdx.x);
#pragma unroll
    for (int k = 0; k < AND_K; ++k) pp[k] = v[k];
  }
}

// Blocks 0..nf-1: (num, den) of field b -> fam_out[2b..]; block nf: the
// Anderson inner products over every field -> m->dots.  Fixed order.
__global__ void __launch_bounds__(AND_THREADS)
    anderson_combine_kernel(const double* partial, int nf, double* fam_out, AndersonMeta* m) {
  if ((int)blockIdx.x < nf) {
    const double* seg = partial + (size_t)AND_K * AND_CTAS * blockIdx.x;
    double v[2] = {0, 0};
    for (int c = threadIdx.x; c < AND_CTAS; c += blockDim.x) {
      v[0] += seg[AND_K * c];
      v[1] += seg[AND_K * c + 1];
    }
    and_block_sum<2>(v);
    if (threadIdx.x == 0) {
      fam_out[2 * blockIdx.x] = v[0];
      fam_out[2 * blockIdx.x + 1] = v[1];
    }
    return;
  }
  double v[MD];
#pragma unroll
  for (int k = 0; k < MD; ++k) v[k] = 0;
  for (int c = threadIdx.x; c < AND_CTAS * nf; c += blockDim.x)
#pragma unroll
    for (int k = 0; k < MD; ++k) v[k] += partial[(size_t)AND_K * c + 2 + k];
  and_block_sum<MD>(v);
  if (threadIdx.x == 0)
    for (int k = 0; k < MD; ++k) m->dots[k] = v[k];
}

int launch_anderson_append(int precision, size_t n, const void* const* state, const void* const* cand, int nf,
                           void* Xh, void* Rh, int depth, AndersonMeta* meta, double* partial, double* fam_out,
                           cudaStream_t st) {
  if (nf <= 0 || nf > kMaxMixFields || depth < 1 || depth > kAndersonMaxDepth) {
    set_last_error("anderson: %d fields / depth %d out of range", nf, depth);
    return QCL_ARG;
  }
  const dim3 grid(AND_CTAS, nf);
  if (precision == QCL_C128) {
    AndFields<double> f{};
    for (int i = 0; i < nf; ++i) {
      f.state[i] = (const Cx<double>*)state[i];
      f.cand[i] = (const Cx<double>*)cand[i];
    }
    anderson_append_kernel<double><<<grid, AND_THREADS, 0, st>>>(n, f, nf, (Cx<double>*)Xh, (Cx<double>*)Rh, depth,
                                                                 meta, partial);
  } else {
    AndFields<float> f{};
    for (int i = 0; i < nf; ++i) {
      f.state[i] = (const Cx<float>*)state[i];
      f.cand[i] = (const Cx<float>*)cand[i];
    }
    anderson_append_kernel<float><<<grid, AND_THREADS, 0, st>>>(n, f, nf, (Cx<float>*)Xh, (Cx<float>*)Rh, depth,
                                                                meta, partial);
  }
  anderson_combine_kernel<<<nf + 1, AND_THREADS, 0, st>>>(partial, nf, fam_out, meta);
  QCL_LAUNCH_CHECK("anderson_append");
  return QCL_OK;
}

// Eigen-decomposition of the symmetric n x n matrix A (row-major, stride MD,
// destroyed) by cyclic Jacobi rotations (Golub & Van Loan, Matrix
// Computations, sec. 8.5): w gets the eigenvalues, V (stride MD) the
// eigenvectors in its columns.
__device__ void sym_jacobi(int n, double* A, double* V, double* w) {
  for (int i = 0; i < n; ++i)
    for (int j = 0; j < n; ++j) V[i * MD + j] = i == j ? 1.0 : 0.0;
  for (int sweep = 0; sweep < 64; ++sweep) {
    double off = 0, tot = 0;
    for (int i = 0; i < n; ++i)
      for (int j = 0; j < n; ++j) {
        const double a = A[i * MD + j] * A[i * MD + j];
        tot += a;
        if (i != j) off += a;
      }
    if (!(off > 1e-34 * tot)) break;  // also ends on NaN
    for (int p = 0; p < n - 1; ++p)
      for (int q = p + 1; q < n; ++q) {
        const double apq = A[p * MD + q];
        if (apq == 0.0) continue;
        const double theta = (A[q * MD + q] - A[p * MD + p]) / (2.0 * apq);
        const double t = (theta >= 0 ? 1.0 : -1.0) / (fabs(theta) + sqrt(theta * theta + 1.0));
        const double c = 1.0 / sqrt(t * t + 1.0), s = t * c;
        for (int k = 0; k < n; ++k) {  // columns p, q
          const double akp = A[k * MD + p], akq = A[k * MD + q];
          A[k * MD + p] = c * akp - s * akq;
          A[k * MD + q] = s * akp + c * akq;
        }
        for (int k = 0; k < n; ++k) {  // rows p, q
          const double apk = A[p * MD + k], aqk = A[q * MD + k];
          A[p * MD + k] = c * apk - s * aqk;
          A[q * MD + k] = s * apk + c * aqk;
        }
        for (int k = 0; k < n; ++k) {
          const double vkp = V[k * MD + p], vkq = V[k * MD + q];
          V[k * MD + p] = c * vkp - s * vkq;
          V[k * MD + q] = s * vkp + c * vkq;
        }
      }
  }
  for (int i = 0; i < n; ++i) w[i] = A[i * MD + i];
}

// Append the Gram row (or reset), then the coefficients.
__global__ void anderson_coefficients_kernel(AndersonMeta* m, int depth, double reg) {
  const double eps = DBL_EPSILON;
  int c = m->count;
  const double rn = m->dots[c];
  if (m->prior >= 0 && rn > (1 + 64 * eps) * fmax(m->prior, DBL_MIN)) {  // residual increase: restart
    m->head = m->slot;
    c = 0;
    m->reason = 1;
  } else {
    for (int i = 0; i < c; ++i) m->gram[i * MD + c] = m->gram[c * MD + i] = m->dots[i];
  }
  m->gram[c * MD + c] = rn;
  const int count = c + 1;
  m->count = count;
  m->used = count;
  double coef[MD];
  bool ok = true;
  if (count == 1) {
    coef[0] = 1.0;
  } else {
    double A[MD * MD], V[MD * MD], w[MD];
    double scale = eps;
    for (int i = 0; i < count; ++i) scale = fmax(scale, fabs(m->gram[i * MD + i]));
    for (int i = 0; i < count; ++i)
      for (int j = 0; j < count; ++j)
        A[i * MD + j] = (m->gram[i * MD + j] + (i == j ? reg * scale : 0.0)) / scale;
    sym_jacobi(count, A, V, w);
    const double cutoff = fmax(reg, sqrt(eps));
    double wt[MD];
    for (int i = 0; i < count; ++i) {
      double proj = 0;
      for (int k = 0; k < count; ++k) proj += V[k * MD + i];
      wt[i] = w[i] > cutoff ? proj / w[i] : 0.0;
    }
    double denom = 0;
    for (int k = 0; k < count; ++k) {
      double v = 0;
      for (int i = 0; i < count; ++i) v += V[k * MD + i] * wt[i];
      coef[k] = v;
      denom += v;
    }
    if (!(isfinite(denom) && fabs(denom) > eps)) ok = false;
    for (int k = 0; k < count && ok; ++k) {
      coef[k] /= denom;
      if (!isfinite(coef[k])) ok = false;
    }
    if (!ok) m->reason = 2;  // coefficient_solve
  }
  double l1 = 0;
  bool finite = ok;
  for (int k = 0; k < count && ok; ++k) {
    l1 += fabs(coef[k]);
    finite = finite && isfinite(coef[k]);
  }
  if (!ok || l1 > 10 || !finite) {
    if (ok) m->reason = 3;  // coefficient_bound
    for (int k = 0; k < count; ++k) coef[k] = k == count - 1 ? 1.0 : 0.0;
    l1 = 1.0;
  }
  int nonzero = 0;
  for (int k = 0; k < count; ++k) {
    m->coef[k] = coef[k];
    nonzero += coef[k] != 0.0;
  }
  m->l1 = l1;
  m->accepted = nonzero > 1;
}

int launch_anderson_coefficients(AndersonMeta* m, int depth, double regularization, cudaStream_t st) {
  anderson_coefficients_kernel<<<1, 1, 0, st>>>(m, depth, regularization);
  QCL_LAUNCH_CHECK("anderson_coefficients");
  return QCL_OK;
}

template <typename R> struct AndOut {
  Cx<R>* out[kMaxMixFields];
};

// out_f = sum_j c_j (x_j + d R_j) over the used history (fallback: the newest
// entry with c = 1, run only after a failed guard).
template <typename R>
__global__ void __launch_bounds__(AND_THREADS)
    anderson_mix_kernel(size_t n, AndOut<R> o, int nf, const Cx<R>* __restrict__ Xh, const Cx<R>* __restrict__ Rh,
                        int depth, const AndersonMeta* __restrict__ m, double damping, int fallback) {
  if (fallback && !m->fallback) return;
  const int fld = blockIdx.y;
  const int used = fallback ? 1 : m->used;
  const Cx<R>* xs[MD];
  const Cx<R>* rs[MD];
  double c[MD];
  for (int j = 0; j < MD; ++j) {
    const int slot = fallback ? m->slot : (m->head + j) % depth;
    xs[j] = Xh + ((size_t)slot * nf + fld) * n;
    rs[j] = Rh + ((size_t)slot * nf + fld) * n;
    c[j] = fallback ? 1.0 : (j < used ? m->coef[j] : 0.0);
  }
  Cx<R>* out = o.out[fld];
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    double vx = 0, vy = 0;
#pragma unroll
    for (int j = 0; j < MD; ++j)
      if (j < used) {
        const Cx<R> x = xs[j][i], r = rs[j][i];
        vx += c[j] * ((double)x.x + damping * (double)r.x);
        vy += c[j] * ((double)x.y + damping * (double)r.y);
      }
    out[i] = cx<R>((R)vx, (R)vy);
  }
}

int launch_anderson_mix(int precision, size_t n, void* const* out, int nf, const void* Xh, const void* Rh, int depth,
                        const AndersonMeta* m, double damping, int fallback, cudaStream_t st) {
  const dim3 grid(AND_CTAS * 4, nf);
  if (precision == QCL_C128) {
    AndOut<double> o{};
    for (int i = 0; i < nf; ++i) o.out[i] = (Cx<double>*)out[i];
    anderson_mix_kernel<double><<<grid, AND_THREADS, 0, st>>>(n, o, nf, (const Cx<double>*)Xh,
                                                              (const Cx<double>*)Rh, depth, m, damping, fallback);
  } else {
    AndOut<float> o{};
    for (int i = 0; i < nf; ++i) o.out[i] = (Cx<float>*)out[i];
    anderson_mix_kernel<float><<<grid, AND_THREADS, 0, st>>>(n, o, nf, (const Cx<float>*)Xh, (const Cx<float>*)Rh,
                                                             depth, m, damping, fallback);
  }
  QCL_LAUNCH_CHECK("anderson_mix");
  return QCL_OK;
}

// After guard pass 0: a failure switches to the linear fallback and clears the
// history (_anderson_clear!).  After pass 1: a failing fallback is the
// reference's DomainError.
__global__ void anderson_after_guard_kernel(AndersonMeta* m, int pass, int* status) {
  if (pass == 0) {
    if (m->guard_key != kNoFailure) {
      m->guard_first = m->guard_key >> 3;
      m->guard_code = (int)(m->guard_key & 7ull);
      m->fallback = 1;
      m->accepted = 0;
      m->reason = 4;  // causality_guard
      m->count = 0;
      m->head = 0;
    }
    m->guard_key = kNoFailure;
  } else if (m->fallback && m->guard_key != kNoFailure) {
    record_status(status, QCL_DOMAIN, (long long)(m->guard_key >> 3) - 1);
  }
}

int launch_anderson_after_guard(AndersonMeta* m, int pass, int* status, cudaStream_t st) {
  anderson_after_guard_kernel<<<1, 1, 0, st>>>(m, pass, status);
  QCL_LAUNCH_CHECK("anderson_after_guard");
  return QCL_OK;
}

}  // namespace qcl
