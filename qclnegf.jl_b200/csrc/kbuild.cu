// Dense kernel operators assembled on the device from angular node weights.
//
// The reference builds each momentum-dependent kernel as an angular average
// over the in-plane angle grid phi_r = 2 pi (r - 1) / N_phi
// (_angular_average_kernel, numerics/reference/kernels.jl:5-19;
// _assemble_exact_parallel_kernel / _assemble_lookup_kernel,
// numerics/optimized/kernels.jl:303-341):
//   K[m,m',a,c,d,b] = (1/N_phi) sum_phi C(q(kappa_m, kappa_m', phi))[a,c,d,b].
// Both of its forms are linear in a set of node tensors X_t:
//   * exact LO phonon kernel (lo_phonon_kernel, kernels.jl:321-356):
//     C(q) = sum_h f_h(q) F_h[a,c] conj(F_h[b,d]), so W[(m,m'),h] is the
//     angular mean of f_h and X_h = F_h (x) conj(F_h) (rank one);
//   * tabulated kernels (_lookup_block, optimized/kernels.jl:205-217): C(q) is
//     the linear interpolation between the node tensors X_t = C(q_t), so
//     W[(m,m'),t] is the angular mean of the interpolation weights.
// So K(m,m') = sum_t W[(m,m'),t] X_t.  The host forms W (N_k^2 x T numbers);
// the device writes K straight into the production dense layout, rows
// (m,a,b), columns (m',c,d) (_production_kernel, production_cache.jl:402-405),
// then normalises by q^K = max |K| (build_kernels, kernels.jl:393-403).
// One CTA per output column (m',c,d): the column's node slices are staged in
// shared memory, threads walk the rows with m fastest (coalesced stores).
#include <math.h>

#include "kernels.cuh"

namespace qcl {

constexpr int KB_THREADS = 256;

// rank-one form: out[r + Nc j] = sum_t W[m + Nk m', t] F[t, a + Nb c] conj(F[t, b + Nb d])
__global__ void __launch_bounds__(KB_THREADS)
    assemble_rank1_kernel(int Nk, int Nb, int T, const double* __restrict__ W, const Cx<double>* __restrict__ F,
                          Cx<double>* __restrict__ out) {
  extern __shared__ __align__(16) unsigned char kb_raw[];
  const int N2 = Nb * Nb, Nc = Nk * N2;
  const int j = blockIdx.x;  // column (m', c, d)
  const int mp = j % Nk, c = (j / Nk) % Nb, d = j / (Nk * Nb);
  Cx<double>* Fc = reinterpret_cast<Cx<double>*>(kb_raw);  // [t][a] = F[t, a + Nb c]
  Cx<double>* Fd = Fc + (size_t)T * Nb;                    // [t][b] = conj F[t, b + Nb d]
  double* Wm = reinterpret_cast<double*>(Fd + (size_t)T * Nb);  // [t][m] = W[m + Nk m', t]
  for (int i = threadIdx.x; i < T * Nb; i += blockDim.x) {
    const int t = i / Nb, x = i % Nb;
    Fc[i] = F[t + (size_t)T * (x + Nb * c)];
    Fd[i] = conj(F[t + (size_t)T * (x + Nb * d)]);
  }
  for (int i = threadIdx.x; i < T * Nk; i += blockDim.x) {
    const int t = i / Nk, m = i % Nk;
    Wm[i] = W[(size_t)(m + Nk * mp) + (size_t)Nk * Nk * t];
  }
  __syncthreads();
  for (int r = threadIdx.x; r < Nc; r += blockDim.x) {
    const int m = r % Nk, a = (r / Nk) % Nb, b = r / (Nk * Nb);
    double sx = 0, sy = 0;
    for (int t = 0; t < T; ++t) {
      const Cx<double> p = Fc[t * Nb + a] * Fd[t * Nb + b];
      const double w = Wm[t * Nk + m];
      sx += w * p.x;
      sy += w * p.y;
    }
    out[(size_t)r + (size_t)Nc * j] = cx<double>(sx, sy);
  }
}

// table form: out[r + Nc j] = sum_t W[m + Nk m', t] X[t][(a + Nb c) + Nb^2 (b + Nb d)]
__global__ void __launch_bounds__(KB_THREADS)
    assemble_table_kernel(int Nk, int Nb, int T, const double* __restrict__ W, const Cx<double>* __restrict__ X,
                          Cx<double>* __restrict__ out) {
  extern __shared__ __align__(16) unsigned char kb_raw[];
  const int N2 = Nb * Nb, Nc = Nk * N2;
  const int j = blockIdx.x;
  const int mp = j % Nk, c = (j / Nk) % Nb, d = j / (Nk * Nb);
  double* Wm = reinterpret_cast<double*>(kb_raw);  // [t][m]
  for (int i = threadIdx.x; i < T * Nk; i += blockDim.x) {
    const int t = i / Nk, m = i % Nk;
    Wm[i] = W[(size_t)(m + Nk * mp) + (size_t)Nk * Nk * t];
  }
  __syncthreads();
  for (int r = threadIdx.x; r < Nc; r += blockDim.x) {
    const int m = r % Nk, a = (r / Nk) % Nb, b = r / (Nk * Nb);
    const size_t off = (size_t)(a + Nb * c) + (size_t)N2 * (b + Nb * d);
    double sx = 0, sy = 0;
    for (int t = 0; t < T; ++t) {
      const Cx<double> x = X[off + (size_t)N2 * N2 * t];
      const double w = Wm[t * Nk + m];
      sx += w * x.x;
      sy += w * x.y;
    }
    out[(size_t)r + (size_t)Nc * j] = cx<double>(sx, sy);
  }
}

// max |out| over n entries: per-CTA partials, then a fixed-order combine.
__global__ void __launch_bounds__(KB_THREADS) maxabs_partial_kernel(size_t n, const Cx<double>* x, double* partial) {
  double v = 0;
  bool bad = false;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const double a = hypot(x[i].x, x[i].y);
    bad |= !isfinite(a);
    v = fmax(v, a);
  }
  if (bad) v = INFINITY;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
  __shared__ double red[KB_THREADS / 32];
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
  __syncthreads();
  if (threadIdx.x == 0) {
    double s = 0;
    for (int w = 0; w < KB_THREADS / 32; ++w) s = fmax(s, red[w]);
    partial[blockIdx.x] = s;
  }
}

__global__ void scale_kernel(size_t n, const double* partial, int np, double* qK, Cx<double>* x) {
  __shared__ double q;
  if (threadIdx.x == 0) {
    double s = 0;
    for (int i = 0; i < np; ++i) s = fmax(s, partial[i]);
    q = s;
    if (blockIdx.x == 0) *qK = s;
  }
  __syncthreads();
  const double qq = q;
  if (!(qq > 0) || !isfinite(qq)) return;  // zero or non-finite kernel: left unnormalised, reported through qK
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    x[i] = cx<double>(x[i].x / qq, x[i].y / qq);
}

constexpr int KB_REDUCE_CTAS = 296;

size_t assemble_work_doubles() { return KB_REDUCE_CTAS + 1; }

int launch_assemble_kernel(int form, int Nk, int Nb, int T, const double* W, const void* X, void* out, double* work,
                           cudaStream_t st) {
  const int Nc = Nk * Nb * Nb;
  if (form == 0) {
    const size_t smem = 2 * (size_t)T * Nb * sizeof(Cx<double>) + (size_t)T * Nk * sizeof(double);
    if (smem > 220 * 1024) {
      set_last_error("kernel assembly: %d nodes x (2 N_b + N_k) exceed the shared-memory staging", T);
      return QCL_UNSUPPORTED;
    }
    QCL_CUDA_CHECK(cudaFuncSetAttribute(assemble_rank1_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    assemble_rank1_kernel<<<Nc, KB_THREADS, smem, st>>>(Nk, Nb, T, W, (const Cx<double>*)X, (Cx<double>*)out);
  } else {
    const size_t smem = (size_t)T * Nk * sizeof(double);
    if (smem > 220 * 1024) {
      set_last_error("kernel assembly: %d nodes x N_k exceed the shared-memory staging", T);
      return QCL_UNSUPPORTED;
    }
    QCL_CUDA_CHECK(cudaFuncSetAttribute(assemble_table_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    assemble_table_kernel<<<Nc, KB_THREADS, smem, st>>>(Nk, Nb, T, W, (const Cx<double>*)X, (Cx<double>*)out);
  }
  QCL_LAUNCH_CHECK("assemble_kernel");
  const size_t n = (size_t)Nc * Nc;
  maxabs_partial_kernel<<<KB_REDUCE_CTAS, KB_THREADS, 0, st>>>(n, (const Cx<double>*)out, work);
  scale_kernel<<<KB_REDUCE_CTAS, KB_THREADS, 0, st>>>(n, work, KB_REDUCE_CTAS, work + KB_REDUCE_CTAS,
                                                       (Cx<double>*)out);
  QCL_LAUNCH_CHECK("kernel normalisation");
  return QCL_OK;
}

}  // namespace qcl
