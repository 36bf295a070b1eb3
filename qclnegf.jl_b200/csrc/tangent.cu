// Implicit differentiation of the SCBA fixed point, tangent (forward) mode.
//
// At a fixed point Sigma* = Phi(Sigma*, p) of the SCBA map (the candidate
// families of solve_scba_production's iteration, production_solver.jl:
// 435-844), the derivative v = dSigma*/dp solves the linear fixed point
//     v = Phi_Sigma v + Phi_p,
// and dJ/dp = J_Sigma v + J_p.  This file holds the pieces of Phi_Sigma v
// that are not linear maps the forward path already has:
//   * the Dyson + Keldysh tangent per (E, k) block,
//       X   = dG^R = G (dSigma^R) G,
//       dL  = X S< G^H + G dS< G^H + G S< X^H    (S< the lesser total),
//       dG  = X S> G^H + G dS> G^H + G S> X^H,
//     as batched complex128 triple products on the FP64 tensor path;
//   * the tangent of the paired number normalisation (_paired_number_
//     coefficients / _normalize_keldysh_pair!, numerics/reference/greens.jl:
//     155-199): da, dc from the weighted traces of dL and dG, then
//       dG<_n = da L + a dL - dc G - c dG,  dG>_n = -dc G + (1-c) dG + da L - (1-a) dL,
//     with the raw L, G recovered from the normalised fields.
// The candidate maps (contractions, shifts, FFT Hilbert, embedding) and the
// mixing are linear and run through the forward kernels (scba.cu).
#include <algorithm>

#include "blockmat.cuh"
#include "kernels.cuh"

namespace qcl {

// out = alpha A B op(C) + beta out per block (op = identity or ^H), complex128;
// trace (may be null) receives tr(out) per block (E fastest).
template <int NP>
__global__ void __launch_bounds__(Tile<NP>::TT) block_triple_kernel(int NE, int Nk, int N, const Cx<double>* A,
                                                                    const Cx<double>* B, const Cx<double>* C, int adjC,
                                                                    double alpha, double beta, Cx<double>* out,
                                                                    Cx<double>* trace) {
  constexpr int TT = Tile<NP>::TT;
  constexpr size_t MSZ = (size_t)NP * NP;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  Cx<double>* bA = reinterpret_cast<Cx<double>*>(smem_raw);
  Cx<double>* bB = bA + MSZ;
  Cx<double>* bC = bB + MSZ;
  Cx<double>* bT = bC + MSZ;
  __shared__ double red[TT / 32 + 1];
  const int e = blockIdx.x, m = blockIdx.y, tt = threadIdx.x;
  for (int i = tt; i < (int)MSZ; i += TT) bA[i] = bB[i] = bC[i] = bT[i] = cx<double>(0, 0);
  __syncthreads();
  load_blocks<double, double, NP, 1>(A, bA, MSZ, e, m, NE, Nk, N);
  load_blocks<double, double, NP, 1>(B, bB, MSZ, e, m, NE, Nk, N);
  load_blocks<double, double, NP, 1>(C, bC, MSZ, e, m, NE, Nk, N);
  __syncthreads();
  team_matmul<double, double, NP>(bA, bB, bT, N, tt, false);  // T = A B
  __syncthreads();
  team_matmul<double, double, NP>(bT, bC, bA, N, tt, adjC != 0);  // A <- T op(C)
  __syncthreads();
  const size_t base = (size_t)e + (size_t)NE * m, cs = (size_t)NE * Nk;
  double tr = 0, ti = 0;
  for (int i = tt; i < N * N; i += TT) {
    const int a = i % N, b = i / N;
    const Cx<double> v = bA[sw<NP>(a, b)];
    Cx<double>* dst = out + base + cs * ((size_t)a + (size_t)N * b);
    Cx<double> r = cx<double>(alpha * v.x, alpha * v.y);
    if (beta != 0.0) {
      const Cx<double> o = *dst;
      r = cx<double>(r.x + beta * o.x, r.y + beta * o.y);
    }
    *dst = r;
    if (a == b) {
      tr += r.x;
      ti += r.y;
    }
  }
  if (trace) {
    tr = team_sum<TT>(tr, tt, red, 0);
    ti = team_sum<TT>(ti, tt, red, 0);
    if (tt == 0) trace[base] = cx<double>(tr, ti);
  }
}

int launch_block_triple(int NE, int Nk, int N, const void* A, const void* B, const void* C, int adjC, double alpha,
                        double beta, void* out, void* trace, cudaStream_t st) {
  const int NP = padded_size(N);
  dim3 grid(NE, Nk);
  switch (NP) {
#define QCL_TRIPLE(P)                                                                                              \
  case P: {                                                                                                        \
    constexpr size_t smem = 4 * (size_t)P * P * sizeof(Cx<double>);                                               \
    static bool configured = false;                                                                                \
    if (!configured) {                                                                                             \
      QCL_CUDA_CHECK(cudaFuncSetAttribute(block_triple_kernel<P>, cudaFuncAttributeMaxDynamicSharedMemorySize,     \
                                          (int)smem));                                                             \
      configured = true;                                                                                           \
    }                                                                                                              \
    block_triple_kernel<P><<<grid, Tile<P>::TT, smem, st>>>(NE, Nk, N, (const Cx<double>*)A, (const Cx<double>*)B, \
                                                           (const Cx<double>*)C, adjC, alpha, beta,                \
                                                           (Cx<double>*)out, (Cx<double>*)trace);                  \
    break;                                                                                                         \
  }
    QCL_TRIPLE(8)
    QCL_TRIPLE(16)
    QCL_TRIPLE(24)
    QCL_TRIPLE(32)
    QCL_TRIPLE(48)
#undef QCL_TRIPLE
    default:
      set_last_error("basis size N_b=%d exceeds the supported maximum 48", N);
      return QCL_UNSUPPORTED;
  }
  QCL_LAUNCH_CHECK("block_triple_kernel");
  return QCL_OK;
}

// da, dc of the paired coefficients from the weighted raw traces of the
// tangents: coeffs = (a, c, lambda, N, H) of the forward step; dtrL / dtrG =
// sum wE wk tr of dL, dG (complex); out = (da, dc).  N = pre Im trL,
// H = -pre Im trG (paired_coefficients_kernel), so dN = pre Im dtrL,
// dH = -pre Im dtrG; branch N >= target: a = target / N, c = 0; else a = 1,
// c = (target - N) / H.
__global__ void norm_tangent_coeffs_kernel(const double* coeffs, const double* dtrL, const double* dtrG, int gs,
                                           double target, int branch, double* out) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  const double pre = gs / (2.0 * M_PI);
  const double N = coeffs[3], H = coeffs[4];
  const double dN = pre * dtrL[1], dH = -pre * dtrG[1];
  double da = 0, dc = 0;
  if (branch == 1 || (branch == 0 && N >= target)) {  // the form of the forward step
    da = -target / (N * N) * dN;
  } else {
    dc = -dN / H - (target - N) / (H * H) * dH;
  }
  out[0] = da;
  out[1] = dc;
}

// In place on the raw tangents dL, dG: the normalised tangents, with the raw
// L, G recovered from the normalised Ln, Gn of the forward step:
//   L = ((1-c) Ln + c Gn) / (a - c),  G = ((1-a) Ln + a Gn) / (a - c).
__global__ void norm_tangent_apply_kernel(size_t n, const Cx<double>* __restrict__ Ln,
                                          const Cx<double>* __restrict__ Gn, const double* __restrict__ coeffs,
                                          const double* __restrict__ dcoef, Cx<double>* __restrict__ dL,
                                          Cx<double>* __restrict__ dG) {
  const double a = coeffs[0], c = coeffs[1], da = dcoef[0], dc = dcoef[1];
  const double inv = 1.0 / (a - c);
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const Cx<double> ln = Ln[i], gn = Gn[i], l = dL[i], g = dG[i];
    const double Lx = ((1 - c) * ln.x + c * gn.x) * inv, Ly = ((1 - c) * ln.y + c * gn.y) * inv;
    const double Gx = ((1 - a) * ln.x + a * gn.x) * inv, Gy = ((1 - a) * ln.y + a * gn.y) * inv;
    dL[i] = cx<double>(da * Lx + a * l.x - dc * Gx - c * g.x, da * Ly + a * l.y - dc * Gy - c * g.y);
    dG[i] = cx<double>(-dc * Gx + (1 - c) * g.x + da * Lx - (1 - a) * l.x,
                       -dc * Gy + (1 - c) * g.y + da * Ly - (1 - a) * l.y);
  }
}

int launch_norm_tangent(size_t n, const void* Ln, const void* Gn, const double* coeffs, const double* dtrL,
                        const double* dtrG, int gs, double target, int branch, double* dcoef, void* dL, void* dG,
                        cudaStream_t st) {
  norm_tangent_coeffs_kernel<<<1, 32, 0, st>>>(coeffs, dtrL, dtrG, gs, target, branch, dcoef);
  QCL_LAUNCH_CHECK("norm_tangent_coeffs_kernel");
  const long long g = std::min<long long>(((long long)n + 255) / 256, 148 * 16);
  norm_tangent_apply_kernel<<<(unsigned)g, 256, 0, st>>>(n, (const Cx<double>*)Ln, (const Cx<double>*)Gn, coeffs,
                                                        dcoef, (Cx<double>*)dL, (Cx<double>*)dG);
  QCL_LAUNCH_CHECK("norm_tangent_apply_kernel");
  return QCL_OK;
}

}  // namespace qcl
