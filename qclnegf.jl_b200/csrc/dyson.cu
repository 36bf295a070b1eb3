// Fused batched Dyson + Keldysh kernel.
//
// Per (E_e, k_m) block (production form: _retarded_green_production,
// numerics/optimized/production_operators.jl:1337-1385, and the sandwiches of
// _current_green_production, numerics/optimized/production_state.jl:23-48):
//   D  = (eps_e + i eta) I - h_m - SigmaR_em
//   s  = max_a sum_b |D_ab|                     (row-sum equilibration)
//   GR = inv(D / s) / s                         (partial pivoting by |Re|+|Im|)
//   G< = GR Sigma< GR^H,  G> = GR Sigma> GR^H   (raw Keldysh products)
//   tr G<, tr G>                                (for the paired number functional)
//
// B200 mapping.  A CTA owns BPC consecutive energies at one k, so that every
// global load/store of a field touches BPC*sizeof(complex) contiguous bytes
// per matrix element (the reference's E-fastest Julia layout).  Each block is
// worked by a "team" of TT threads: the inversion is a register-resident
// Gauss-Jordan elimination with implicit row pivoting (each thread owns a
// COLS-wide chunk of one row, so no row is ever moved), the products are
// shared-memory tiled matmuls with TRxTC register tiles per thread.  Shared
// memory rows are XOR-swizzled on the low three column bits so that column
// walks hit distinct banks.
#include "blockmat.cuh"

namespace qcl {

template <typename RS> struct DysonArgs {
  int NE, Nk, N, m0;  // blocks of momenta m0 .. m0 + gridDim.y - 1
  const double* eps;
  double eta;
  const Cx<double>* h;  // (Nk, N, N), FP64 always
  const Cx<RS>* sigR;
  const Cx<RS>* sigL;
  const Cx<RS>* sigG;   // may be null
  Cx<RS>* GR;           // may be null
  Cx<RS>* GL;           // may be null
  Cx<RS>* GG;           // may be null
  double* scale;        // (NE, Nk), may be null
  Cx<double>* traceL;   // (NE, Nk) raw tr G<, may be null
  Cx<double>* traceG;   // (NE, Nk) raw tr G>, may be null
  int* status;
  int mcount;
};

// Argmax key: the pivot magnitude's IEEE bits with the low 8 bits replaced
// by (255 - row).  Unsigned order = magnitude order with ties to the smaller
// row (the perturbation is below 2^-44 relative, far below the gap between
// distinct pivot candidates that matters for stability).
__device__ __forceinline__ unsigned long long pivot_key(double mag, int row) {
  return (((unsigned long long)__double_as_longlong(mag)) & ~0xffull) | (unsigned long long)(255 - row);
}
__device__ __forceinline__ unsigned long long warp_max_key(unsigned long long k) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    const unsigned long long q = __shfl_xor_sync(0xffffffffu, k, o);
    k = q > k ? q : k;
  }
  return k;
}

// RS: storage precision, RL: inversion precision, RM: product precision.
template <typename RS, typename RL, typename RM, int NP, int BPC>
__global__ void __launch_bounds__(BPC* Tile<NP>::TT) dyson_keldysh_kernel(DysonArgs<RS> p) {
  constexpr int CPR = Tile<NP>::CPR, TT = Tile<NP>::TT, COLS = NP / CPR;
  constexpr size_t MSZ = (size_t)NP * NP;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  Cx<RS>* bufA = reinterpret_cast<Cx<RS>*>(smem_raw);  // BPC matrices: staged Sigma / products
  Cx<RS>* bufG = bufA + BPC * MSZ;                    // BPC matrices: G^R
  Cx<RS>* bufT = bufG + BPC * MSZ;                    // BPC matrices: G^R Sigma
  TeamScratch<RL, NP, TT>* scr = reinterpret_cast<TeamScratch<RL, NP, TT>*>(bufT + BPC * MSZ);

  const int N = p.N, NE = p.NE, Nk = p.Nk;
  const int m = p.m0 + blockIdx.y;
  const int e0 = blockIdx.x * BPC;
  const int team = threadIdx.x / TT;
  const int tt = threadIdx.x % TT;
  const int e = e0 + team;
  const bool live = e < NE;
  Cx<RS>* A = bufA + team * MSZ;
  Cx<RS>* G = bufG + team * MSZ;
  Cx<RS>* T = bufT + team * MSZ;
  TeamScratch<RL, NP, TT>& S = scr[team];
  const Cx<RS>* first_sig = p.sigL ? p.sigL : p.sigG;
  const bool first_is_L = p.sigL != nullptr;

  // ---- stage SigmaR (all copies in flight at once) ---------------------------
  load_blocks_async<RS, NP, BPC>(p.sigR, bufA, MSZ, e0, m, NE, Nk, N);
  cp_async_wait_all();
  __syncthreads();

  // ---- D rows into registers, row-sum equilibration ---------------------------
  const int row = tt / CPR, chunk = tt % CPR;
  const bool has_row = row < NP;
  Cx<RL> w[COLS];
  const double eps_e = live ? p.eps[e] : 0.0;
  double rowsum = 0.0;
#pragma unroll
  for (int j = 0; j < COLS; ++j) {
    const int col = chunk * COLS + j;
    Cx<RL> d = cx<RL>(0, 0);
    if (has_row && row < N && col < N) {
      const Cx<double> hv = p.h[(size_t)m + (size_t)Nk * ((size_t)row + (size_t)N * col)];
      const Cx<RS> sv = A[sw<NP>(row, col)];
      double re = -hv.x - (double)sv.x, im = -hv.y - (double)sv.y;
      if (row == col) {
        re += eps_e;
        im += p.eta;
      }
      d = cx<RL>((RL)re, (RL)im);
      rowsum += sqrt(re * re + im * im);
    }
    w[j] = d;
  }
  __syncthreads();  // every team has read its SigmaR tile: bufA is free
  // prefetch the first Keldysh input while the inversion runs
  if (first_sig && (first_is_L ? p.GL : p.GG)) load_blocks_async<RS, NP, BPC>(first_sig, bufA, MSZ, e0, m, NE, Nk, N);

#pragma unroll
  for (int o = 1; o < CPR; o <<= 1) rowsum += __shfl_xor_sync(0xffffffffu, rowsum, o);
  const double s = team_max<TT>(rowsum, tt, S.red, team);
  const RL inv_s = (RL)(1.0 / s);
  const bool scale_ok = s > 0.0 && isfinite(s);
#pragma unroll
  for (int j = 0; j < COLS; ++j) {
    const int col = chunk * COLS + j;
    w[j] = inv_s * w[j];
    if (has_row && row >= N && col == row) w[j] = cx<RL>(1, 0);  // identity padding
  }

  // ---- register-resident Gauss-Jordan with implicit row pivoting -------------
  bool used = !has_row;
  bool singular = !scale_ok;
  int mystep = row;
  const int lane = threadIdx.x & 31;
  const int srclane = lane - chunk;  // first lane of this row's chunk group
  if (tt < NP && tt >= N) S.pivrow[tt] = tt;  // padded steps are identities
  // The step loop stays rolled (small code, no instruction-cache misses); the
  // pivot column is picked out of the register row with predicated selects.
#pragma unroll 1
  for (int k = 0; k < N; ++k) {
    const int kc = k / COLS, kj = k - kc * COLS;
    Cx<RL> wk = w[0];
#pragma unroll
    for (int j = 1; j < COLS; ++j)
      if (j == kj) wk = w[j];
    const bool cand = !used && chunk == kc;
    // speculative reciprocal of every candidate (off the argmax critical path)
    Cx<RL> rc = cx<RL>(0, 0);
    unsigned long long key = 0ull;
    if (cand) {
      key = pivot_key((double)cabs1(wk), row);
      rc = crecip_scaled(wk);
    }
    key = warp_max_key(key);
    if (TT > 32) {
      if (lane == 0) S.wkey[tt >> 5] = key;
      team_sync<TT>(team);
#pragma unroll
      for (int q = 0; q < TT / 32; ++q) {
        const unsigned long long o = S.wkey[q];
        key = o > key ? o : key;
      }
    }
    const int best = 255 - (int)(key & 0xffull);
    const bool zero = (key >> 8) == 0ull;
    if (zero) singular = true;
    if (tt == 0) S.pivrow[k] = best;
    // multiplier of this row and (for the pivot row) its reciprocal
    Cx<RL> f = wk;
    if (CPR > 1) {
      f.x = __shfl_sync(0xffffffffu, wk.x, srclane + kc);
      f.y = __shfl_sync(0xffffffffu, wk.y, srclane + kc);
      rc.x = __shfl_sync(0xffffffffu, rc.x, srclane + kc);
      rc.y = __shfl_sync(0xffffffffu, rc.y, srclane + kc);
    }
    Cx<RL>* rb = S.rowbuf[k & 1];
    const bool is_pivot = has_row && row == best;
    const Cx<RL> colk = is_pivot ? cx<RL>(1, 0) : cx<RL>(0, 0);
    if (chunk == kc) {
#pragma unroll
      for (int j = 0; j < COLS; ++j)
        if (j == kj) w[j] = colk;
    }
    if (is_pivot) {
      const Cx<RL> inv = zero ? cx<RL>(0, 0) : rc;
#pragma unroll
      for (int j = 0; j < COLS; ++j) {
        w[j] = w[j] * inv;
        rb[chunk * COLS + j] = w[j];
      }
      used = true;
      mystep = k;
    }
    team_sync<TT>(team);
    if (has_row && !is_pivot) {
#pragma unroll
      for (int j = 0; j < COLS; ++j) cfms(w[j], f, rb[chunk * COLS + j]);
    }
  }
  team_sync<TT>(team);
  if (singular && live && tt == 0) record_status(p.status, QCL_SINGULAR, (long long)e + (long long)NE * m);
  // inverse(D/s)[step][pivrow[k']] = w[k'];  GR = that / s
  if (has_row) {
#pragma unroll
    for (int j = 0; j < COLS; ++j) {
      const int kp = chunk * COLS + j;
      const int col = S.pivrow[kp];
      Cx<RL> g = inv_s * w[j];
      if (mystep >= N || col >= N) g = cx<RL>(0, 0);
      G[sw<NP>(mystep, col)] = cvt<RS>(g);
    }
  }
  if (tt == 0 && live && p.scale) p.scale[(size_t)e + (size_t)NE * m] = s;
  __syncthreads();
  if (p.GR) store_blocks<RS, RS, NP, BPC>(p.GR, bufG, MSZ, e0, m, NE, Nk, N);

  // ---- Keldysh products ------------------------------------------------------
  bool prefetched = first_sig && (first_is_L ? p.GL : p.GG);
  for (int which = 0; which < 2; ++which) {
    const Cx<RS>* sig = which == 0 ? p.sigL : p.sigG;
    Cx<RS>* out = which == 0 ? p.GL : p.GG;
    Cx<double>* tr = which == 0 ? p.traceL : p.traceG;
    if (sig == nullptr || out == nullptr) continue;  // uniform
    if (!prefetched) {
      __syncthreads();  // previous store out of bufA is complete
      load_blocks_async<RS, NP, BPC>(sig, bufA, MSZ, e0, m, NE, Nk, N);
    }
    prefetched = false;
    cp_async_wait_all();
    __syncthreads();
    team_matmul<RS, RM, NP>(G, A, T, N, tt, false);
    team_sync<TT>(team);
    team_matmul<RS, RM, NP>(T, G, A, N, tt, true);
    team_sync<TT>(team);
    if (tr) {
      double re = 0, im = 0;
      if (tt < N) {
        const Cx<RS> d = A[sw<NP>(tt, tt)];
        re = d.x;
        im = d.y;
      }
      re = team_sum<TT>(re, tt, S.red, team);
      im = team_sum<TT>(im, tt, S.red, team);
      if (tt == 0 && live) tr[(size_t)e + (size_t)NE * m] = cx<double>(re, im);
    }
    __syncthreads();
    store_blocks<RS, RS, NP, BPC>(out, bufA, MSZ, e0, m, NE, Nk, N);
  }
}

template <typename RS, typename RL, int NP, int TT, int BPC> constexpr size_t dyson_smem() {
  return 3 * (size_t)BPC * NP * NP * sizeof(Cx<RS>) + BPC * sizeof(TeamScratch<RL, NP, TT>);
}

template <typename RS, typename RL, typename RM, int NP, int BPC>
static int launch_dyson_t(const DysonArgs<RS>& a, cudaStream_t st) {
  constexpr int TT = Tile<NP>::TT;
  constexpr size_t smem = dyson_smem<RS, RL, NP, TT, BPC>();
  static bool configured = false;
  if (!configured) {
    QCL_CUDA_CHECK(cudaFuncSetAttribute(dyson_keldysh_kernel<RS, RL, RM, NP, BPC>,
                                        cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    configured = true;
  }
  dim3 grid((a.NE + BPC - 1) / BPC, a.mcount);
  dyson_keldysh_kernel<RS, RL, RM, NP, BPC><<<grid, BPC * TT, smem, st>>>(a);
  QCL_LAUNCH_CHECK("dyson_keldysh_kernel");
  return QCL_OK;
}

int padded_size(int N) {
  if (N <= 8) return 8;
  if (N <= 16) return 16;
  if (N <= 24) return 24;
  if (N <= 32) return 32;
  if (N <= 48) return 48;
  return 0;
}

template <typename RS, typename RL, typename RM>
static int launch_dyson_prec(const DysonArgs<RS>& a, cudaStream_t st) {
  constexpr bool wide = sizeof(RS) == 8;  // FP64 storage: half the blocks per CTA
  switch (padded_size(a.N)) {
    case 8: return launch_dyson_t<RS, RL, RM, 8, 16>(a, st);
    case 16: return launch_dyson_t<RS, RL, RM, 16, wide ? 4 : 8>(a, st);
    case 24: return launch_dyson_t<RS, RL, RM, 24, wide ? 2 : 4>(a, st);
    case 32: return launch_dyson_t<RS, RL, RM, 32, wide ? 1 : 2>(a, st);
    case 48: return launch_dyson_t<RS, RL, RM, 48, 1>(a, st);
    default:
      set_last_error("basis size N_b=%d exceeds the supported maximum 48", a.N);
      return QCL_UNSUPPORTED;
  }
}

int launch_dyson_keldysh(int precision, int NE, int Nk, int N, const double* eps, double eta, const void* h,
                         const void* sigR, const void* sigL, const void* sigG, void* GR, void* GL, void* GG,
                         double* scale, void* traceL, void* traceG, int* status, cudaStream_t st, int m0,
                         int mcount) {
  if (mcount < 0) mcount = Nk - m0;
  if (m0 < 0 || mcount <= 0 || m0 + mcount > Nk) {
    set_last_error("dyson_keldysh: momentum slab [%d, %d) outside [0, %d)", m0, m0 + mcount, Nk);
    return QCL_DIM;
  }
  if (NE <= 0 || Nk <= 0 || N <= 0) {
    set_last_error("dyson_keldysh: non-positive dimension (%d,%d,%d)", NE, Nk, N);
    return QCL_DIM;
  }
  if (precision == QCL_C128) {
    DysonArgs<double> a{NE, Nk, N, m0, eps, eta, (const Cx<double>*)h, (const Cx<double>*)sigR,
                        (const Cx<double>*)sigL, (const Cx<double>*)sigG, (Cx<double>*)GR, (Cx<double>*)GL,
                        (Cx<double>*)GG, scale, (Cx<double>*)traceL, (Cx<double>*)traceG, status, mcount};
    return launch_dyson_prec<double, double, double>(a, st);
  }
  DysonArgs<float> a{NE, Nk, N, m0, eps, eta, (const Cx<double>*)h, (const Cx<float>*)sigR,
                     (const Cx<float>*)sigL, (const Cx<float>*)sigG, (Cx<float>*)GR, (Cx<float>*)GL,
                     (Cx<float>*)GG, scale, (Cx<double>*)traceL, (Cx<double>*)traceG, status, mcount};
  if (precision == QCL_MIXED) return launch_dyson_prec<float, double, float>(a, st);
  if (precision == QCL_C64) return launch_dyson_prec<float, float, float>(a, st);
  set_last_error("unknown precision %d", precision);
  return QCL_ARG;
}

}  // namespace qcl
