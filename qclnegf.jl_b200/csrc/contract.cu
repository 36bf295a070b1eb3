// Energy shifts and the static self-energy contractions.
//
// Shift: apply_energy_shift! (numerics/optimized/production_cache.jl:300-325)
//   Y[e] = valid[e] ? ((l == r || th == 0) ? X[l] : (1-th) X[l] + th X[r]) : 0
// Contractions (production_static_contraction, production_operators.jl:
// 402-658), S = beta S + alpha q K[wk G]:
//   momentum independent: X[e,(c,d)] = sum_m' wk G[e,m',c,d]; Y = B X;
//                         S[e,m,(a,b)] broadcast over m;
//   dense:                S[e,(m,a,b)] = sum_(m',c,d) M wk[m'] G[e,(m',c,d)];
//   separable IFR:        S = left * (radial * (wk .* (right * G)));
//   low rank:             S = left * (right_adjoint * (wk .* G));
//   separable sum:        S[e,m,(a,b)] = sum_i sum_(c,d) block_i[(a,b),(c,d)]
//                                        sum_m' radial_i[m,m'] wk[m'] G[e,m',c,d].
// Every stage is one call of a tiled complex GEMM whose operand and output
// index maps are strided views of the E-fastest fields: the energy axis is the
// GEMM's M dimension, so all A loads and C stores are coalesced along E.
#include "kernels.cuh"

namespace qcl {

// ---------------------------------------------------------------------------
template <typename R>
__global__ void shift_kernel(int NE, long long ncols, const int* __restrict__ left, const int* __restrict__ right,
                             const double* __restrict__ theta, const unsigned char* __restrict__ valid,
                             const Cx<R>* __restrict__ X, Cx<R>* __restrict__ Y) {
  const long long n = (long long)NE * ncols;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const int e = (int)(i % NE);
    const long long base = i - e;
    Cx<R> v = cx<R>(0, 0);
    if (valid[e]) {
      const int l = left[e], r = right[e];
      const double th = theta[e];
      if (l == r || th == 0.0) {
        v = X[base + l];
      } else {
        const Cx<R> a = X[base + l], b = X[base + r];
        v = cx<R>((R)((1 - th) * a.x + th * b.x), (R)((1 - th) * a.y + th * b.y));
      }
    }
    Y[i] = v;
  }
}

static unsigned grid_cap(long long n, int threads) {
  long long g = (n + threads - 1) / threads;
  const long long cap = 148 * 16;
  return (unsigned)(g < cap ? (g > 0 ? g : 1) : cap);
}

int launch_shift(int precision, int NE, long long ncols, const ShiftPlanDev& plan, const void* X, void* Y,
                 cudaStream_t st) {
  const long long n = (long long)NE * ncols;
  if (precision == QCL_C128)
    shift_kernel<double><<<grid_cap(n, 256), 256, 0, st>>>(NE, ncols, plan.left, plan.right, plan.theta, plan.valid,
                                                          (const Cx<double>*)X, (Cx<double>*)Y);
  else
    shift_kernel<float><<<grid_cap(n, 256), 256, 0, st>>>(NE, ncols, plan.left, plan.right, plan.theta, plan.valid,
                                                         (const Cx<float>*)X, (Cx<float>*)Y);
  QCL_LAUNCH_CHECK("shift_kernel");
  return QCL_OK;
}

// Y = a X(eps + d1) + b X(eps + d2): two shifts of the same field combined in
// one pass (the linear combination the thermal-LO self-energy contracts,
// production_operators.jl:1107-1163, formed before the contraction).
template <typename R>
__global__ void shift_pair_kernel(int NE, long long ncols, ShiftPlanDev p1, ShiftPlanDev p2, double a, double b,
                                  const Cx<R>* __restrict__ X, Cx<R>* __restrict__ Y) {
  const long long n = (long long)NE * ncols;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const int e = (int)(i % NE);
    const long long base = i - e;
    double vx = 0, vy = 0;
#pragma unroll
    for (int s = 0; s < 2; ++s) {
      const ShiftPlanDev& pl = s == 0 ? p1 : p2;
      const double c = s == 0 ? a : b;
      if (!pl.valid[e]) continue;
      const int l = pl.left[e], r = pl.right[e];
      const double th = pl.theta[e];
      double ux, uy;
      if (l == r || th == 0.0) {
        const Cx<R> q = X[base + l];
        ux = q.x;
        uy = q.y;
      } else {
        const Cx<R> ql = X[base + l], qr = X[base + r];
        ux = (1 - th) * ql.x + th * qr.x;
        uy = (1 - th) * ql.y + th * qr.y;
      }
      vx += c * ux;
      vy += c * uy;
    }
    Y[i] = cx<R>((R)vx, (R)vy);
  }
}

int launch_shift_pair(int precision, int NE, long long ncols, const ShiftPlanDev& p1, const ShiftPlanDev& p2, double a,
                      double b, const void* X, void* Y, cudaStream_t st) {
  const long long n = (long long)NE * ncols;
  if (precision == QCL_C128)
    shift_pair_kernel<double><<<grid_cap(n, 256), 256, 0, st>>>(NE, ncols, p1, p2, a, b, (const Cx<double>*)X,
                                                               (Cx<double>*)Y);
  else
    shift_pair_kernel<float><<<grid_cap(n, 256), 256, 0, st>>>(NE, ncols, p1, p2, a, b, (const Cx<float>*)X,
                                                              (Cx<float>*)Y);
  QCL_LAUNCH_CHECK("shift_pair_kernel");
  return QCL_OK;
}

// build_shift_plan (production_cache.jl:258-290), 0-based, on the host.
int build_shift_plan_host(int NE, const double* eps, double delta, int* left, int* right, double* theta,
                          unsigned char* valid) {
  if (NE < 2 || !isfinite(delta)) {
    set_last_error("shift plan: at least two nodes and a finite displacement are required");
    return QCL_ARG;
  }
  for (int e = 1; e < NE; ++e)
    if (!(eps[e] > eps[e - 1]) || !isfinite(eps[e])) {
      set_last_error("energy nodes must be finite and strictly increasing");
      return QCL_ARG;
    }
  int j = 0;
  for (int e = 0; e < NE; ++e) {
    const double target = eps[e] + delta;
    left[e] = right[e] = 0;
    theta[e] = 0.0;
    valid[e] = 0;
    if (target < eps[0] || target > eps[NE - 1]) continue;
    if (target == eps[NE - 1]) {
      left[e] = right[e] = NE - 1;
      valid[e] = 1;
      continue;
    }
    while (j < NE - 2 && eps[j + 1] <= target) ++j;
    left[e] = j;
    right[e] = j + 1;
    theta[e] = (target - eps[j]) / (eps[j + 1] - eps[j]);
    valid[e] = 1;
  }
  return QCL_OK;
}

// ---------------------------------------------------------------------------
// Momentum reduction: X[e + NE q] = sum_m' wk[m'] G[e + NE (m' + Nk q)]
// ---------------------------------------------------------------------------
template <typename R>
__global__ void momentum_sum_kernel(int NE, int Nk, int NQ, const double* __restrict__ wk,
                                    const Cx<R>* __restrict__ G, Cx<R>* __restrict__ X) {
  const long long n = (long long)NE * NQ;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const int e = (int)(i % NE);
    const long long q = i / NE;
    double sx = 0, sy = 0;
    for (int mp = 0; mp < Nk; ++mp) {
      const Cx<R> g = G[(size_t)e + (size_t)NE * ((size_t)mp + (size_t)Nk * q)];
      sx += wk[mp] * (double)g.x;
      sy += wk[mp] * (double)g.y;
    }
    X[i] = cx<R>((R)sx, (R)sy);
  }
}

// ---------------------------------------------------------------------------
// Tiled complex GEMM over strided views:
//   C[e, j] (bcast copies) = alpha * sum_k A[e,k] w(k,b) B[j,k] + beta * C
//   A[e,k] = A[e + lda k + a_b b],  B[j,k] = B[j ldb_j + k ldb_k + b_b b],
//   C[e,j] = C[e + ldc j + c_b b + bcast_stride r], r < bcast.
// ---------------------------------------------------------------------------
template <typename R> struct GemmArgs {
  int M, Nout, K, batch;
  const Cx<R>* A;
  long long lda, a_b;
  const double* wk;  // optional weight wk[k % wk_mod]
  int wk_mod;
  const double* wb;  // optional weight wb[b]
  const Cx<R>* B;
  long long ldb_j, ldb_k, b_b;
  Cx<R>* C;
  long long ldc, c_b;
  int bcast;
  long long bcast_stride;
  double alpha, beta;
};

constexpr int GK = 16;

// Output tile GE x GJ per CTA of GT threads: a 16 x (GT / 16) thread grid,
// each thread GE/16 x GJ/(GT/16) outputs.  Two shapes: 64 x 32 (256 threads)
// and, when that gives fewer than two CTAs per SM, 32 x 16 (128 threads) --
// the same per-output arithmetic and summation order, more CTAs in flight.
template <typename R, int GE, int GJ, int GT> __global__ void __launch_bounds__(GT) gemm_kernel(GemmArgs<R> p) {
  constexpr int TJ = GT / 16, NI = GE / 16, NU = GJ / TJ;
  static_assert(GE % 16 == 0 && GJ % TJ == 0, "tile shape");
  __shared__ Cx<R> As[GK][GE];
  __shared__ Cx<R> Bs[GK][GJ];
  const int b = blockIdx.z;
  const int e0 = blockIdx.x * GE, j0 = blockIdx.y * GJ;
  const int te = threadIdx.x % 16, tj = threadIdx.x / 16;
  const double wbb = p.wb ? p.wb[b] : 1.0;
  Cx<R> acc[NI][NU];
#pragma unroll
  for (int i = 0; i < NI; ++i)
#pragma unroll
    for (int u = 0; u < NU; ++u) acc[i][u] = cx<R>(0, 0);
  for (int k0 = 0; k0 < p.K; k0 += GK) {
    for (int idx = threadIdx.x; idx < GE * GK; idx += GT) {
      const int el = idx % GE, kl = idx / GE;
      const int e = e0 + el, k = k0 + kl;
      Cx<R> v = cx<R>(0, 0);
      if (e < p.M && k < p.K) {
        v = p.A[(size_t)e + (size_t)p.lda * k + (size_t)p.a_b * b];
        double w = wbb;
        if (p.wk) w *= p.wk[k % p.wk_mod];
        if (w != 1.0) v = cx<R>((R)(w * v.x), (R)(w * v.y));
      }
      As[kl][el] = v;
    }
    for (int idx = threadIdx.x; idx < GJ * GK; idx += GT) {
      const int jl = idx % GJ, kl = idx / GJ;
      const int j = j0 + jl, k = k0 + kl;
      Bs[kl][jl] = (j < p.Nout && k < p.K) ? p.B[(size_t)p.ldb_j * j + (size_t)p.ldb_k * k + (size_t)p.b_b * b]
                                           : cx<R>(0, 0);
    }
    __syncthreads();
#pragma unroll
    for (int kl = 0; kl < GK; ++kl) {
      Cx<R> a[NI], bb[NU];
#pragma unroll
      for (int i = 0; i < NI; ++i) a[i] = As[kl][te + 16 * i];
#pragma unroll
      for (int u = 0; u < NU; ++u) bb[u] = Bs[kl][tj + TJ * u];
#pragma unroll
      for (int i = 0; i < NI; ++i)
#pragma unroll
        for (int u = 0; u < NU; ++u) cfma(acc[i][u], a[i], bb[u]);
    }
    __syncthreads();
  }
#pragma unroll
  for (int i = 0; i < NI; ++i) {
    const int e = e0 + te + 16 * i;
    if (e >= p.M) continue;
#pragma unroll
    for (int u = 0; u < NU; ++u) {
      const int j = j0 + tj + TJ * u;
      if (j >= p.Nout) continue;
      const double vx = p.alpha * (double)acc[i][u].x, vy = p.alpha * (double)acc[i][u].y;
      for (int r = 0; r < p.bcast; ++r) {
        const size_t idx = (size_t)e + (size_t)p.ldc * j + (size_t)p.c_b * b + (size_t)p.bcast_stride * r;
        if (p.beta == 0.0) {
          p.C[idx] = cx<R>((R)vx, (R)vy);
        } else {
          const Cx<R> o = p.C[idx];
          p.C[idx] = cx<R>((R)(p.beta * o.x + vx), (R)(p.beta * o.y + vy));
        }
      }
    }
  }
}

template <typename R> static int launch_gemm(const GemmArgs<R>& a, cudaStream_t st) {
  if (a.M <= 0 || a.Nout <= 0 || a.batch <= 0) return QCL_OK;
  const long long big = (long long)((a.M + 63) / 64) * ((a.Nout + 31) / 32) * a.batch;
  if (big >= 2 * 148) {
    dim3 grid((a.M + 63) / 64, (a.Nout + 31) / 32, a.batch);
    gemm_kernel<R, 64, 32, 256><<<grid, 256, 0, st>>>(a);
  } else {
    dim3 grid((a.M + 31) / 32, (a.Nout + 15) / 16, a.batch);
    gemm_kernel<R, 32, 16, 128><<<grid, 128, 0, st>>>(a);
  }
  QCL_LAUNCH_CHECK("gemm_kernel");
  return QCL_OK;
}

// ---------------------------------------------------------------------------
// Dense complex128 contraction on the FP64 tensor path (mma.sync m8n8k4 f64):
//   C[e, j] = alpha sum_k A[e + lda k] w[k % wmod] B[j + ldb k] + beta C[e + ldc j].
// CTA: 8 warps, 128 (e) x 32 (j) outputs; warp (wm, wn) owns rows 32 wm ..
// + 31 and columns 16 wn .. + 15 as 4 x 2 tiles of 8 x 8, each accumulated as
// four real products (Re C += Ar Br - Ai Bi, Im C += Ar Bi + Ai Br).  K
// advances by 16 through two cp.async stages; shared rows are padded to a
// stride of 2 (mod 8) 16-byte units so the fragment loads of a quarter warp
// hit 8 distinct bank groups.  Fragment layouts (m8n8k4, f64): A lane l holds
// (l / 4, l % 4), B holds (l % 4, l / 4), C holds (l / 4, 2 (l % 4) + i).
// ---------------------------------------------------------------------------
constexpr int DM_BM = 128, DM_BN = 32, DM_BK = 16, DM_THREADS = 256;
constexpr int DM_APAD = DM_BM + 2, DM_BPAD = DM_BN + 2;
constexpr size_t DM_SMEM = (2 * DM_BK * DM_APAD + 2 * DM_BK * DM_BPAD) * sizeof(Cx<double>) + 2 * DM_BK * sizeof(double);

struct DmArgs {
  int M, N, K;
  const Cx<double>* A;
  long long lda;
  const double* w;
  int wmod;
  const Cx<double>* B;
  long long ldb;
  Cx<double>* C;
  long long ldc;
  double alpha, beta;
  // tile order: 0 = row tiles fastest (the CTAs in flight share B tiles),
  // 1 = column tiles fastest (they share A tiles: an A larger than L2 is
  // read once); set by launch_dmma_dense
  int cols_fastest;
};

__device__ __forceinline__ void dm_cp16(Cx<double>* dst, const Cx<double>* src, bool valid) {
  const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(d), "l"(src), "r"(valid ? 16 : 0) : "memory");
}
__device__ __forceinline__ void dmma(double (&c)[2], double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};"
               : "+d"(c[0]), "+d"(c[1])
               : "d"(a), "d"(b));
}

__global__ void __launch_bounds__(DM_THREADS, 2) dmma_dense_kernel(DmArgs p) {
  extern __shared__ __align__(16) unsigned char dm_raw[];
  Cx<double>* As = reinterpret_cast<Cx<double>*>(dm_raw);   // [2][DM_BK][DM_APAD]
  Cx<double>* Bs = As + 2 * DM_BK * DM_APAD;                 // [2][DM_BK][DM_BPAD]
  double* ws = reinterpret_cast<double*>(Bs + 2 * DM_BK * DM_BPAD);  // [2][DM_BK]
  const int m0 = (p.cols_fastest ? blockIdx.y : blockIdx.x) * DM_BM;
  const int n0 = (p.cols_fastest ? blockIdx.x : blockIdx.y) * DM_BN;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int wm = warp & 3, wn = warp >> 2;
  const int lr = lane >> 2, lc = lane & 3;
  double cr[4][2][2], ci[4][2][2];
#pragma unroll
  for (int t = 0; t < 4; ++t)
#pragma unroll
    for (int u = 0; u < 2; ++u) cr[t][u][0] = cr[t][u][1] = ci[t][u][0] = ci[t][u][1] = 0.0;

  const int nkb = (p.K + DM_BK - 1) / DM_BK;
  auto load = [&](int kb, int s) {
    const int k0 = kb * DM_BK;
    Cx<double>* as = As + s * DM_BK * DM_APAD;
    Cx<double>* bs = Bs + s * DM_BK * DM_BPAD;
#pragma unroll
    for (int i = threadIdx.x; i < DM_BK * DM_BM; i += DM_THREADS) {
      const int kk = i / DM_BM, el = i % DM_BM;
      const int k = k0 + kk, e = m0 + el;
      const bool ok = k < p.K && e < p.M;
      dm_cp16(as + kk * DM_APAD + el, ok ? p.A + (size_t)e + (size_t)p.lda * k : p.A, ok);
    }
#pragma unroll
    for (int i = threadIdx.x; i < DM_BK * DM_BN; i += DM_THREADS) {
      const int kk = i / DM_BN, jl = i % DM_BN;
      const int k = k0 + kk, j = n0 + jl;
      const bool ok = k < p.K && j < p.N;
      dm_cp16(bs + kk * DM_BPAD + jl, ok ? p.B + (size_t)j + (size_t)p.ldb * k : p.B, ok);
    }
    if (threadIdx.x < DM_BK) {
      const int k = k0 + threadIdx.x;
      ws[s * DM_BK + threadIdx.x] = (k < p.K && p.w) ? p.w[k % p.wmod] : 1.0;
    }
    asm volatile("cp.async.commit_group;" ::: "memory");
  };

  load(0, 0);
  for (int kb = 0; kb < nkb; ++kb) {
    const int s = kb & 1;
    if (kb + 1 < nkb) {
      load(kb + 1, s ^ 1);  // stage s^1 was released by the barrier at the end of iteration kb-1
      asm volatile("cp.async.wait_group 1;" ::: "memory");
    } else {
      asm volatile("cp.async.wait_group 0;" ::: "memory");
    }
    __syncthreads();
    const Cx<double>* as = As + s * DM_BK * DM_APAD;
    const Cx<double>* bs = Bs + s * DM_BK * DM_BPAD;
#pragma unroll
    for (int c = 0; c < DM_BK / 4; ++c) {
      const int kk = 4 * c + lc;
      const double w = ws[s * DM_BK + kk];
      double ar[4], ai[4], nai[4], br[2], bi[2];
#pragma unroll
      for (int t = 0; t < 4; ++t) {
        const Cx<double> a = as[kk * DM_APAD + wm * 32 + t * 8 + lr];
        ar[t] = a.x * w;
        ai[t] = a.y * w;
        nai[t] = -ai[t];
      }
#pragma unroll
      for (int u = 0; u < 2; ++u) {
        const Cx<double> b = bs[kk * DM_BPAD + wn * 16 + u * 8 + lr];
        br[u] = b.x;
        bi[u] = b.y;
      }
#pragma unroll
      for (int t = 0; t < 4; ++t)
#pragma unroll
        for (int u = 0; u < 2; ++u) {
          dmma(cr[t][u], ar[t], br[u]);
          dmma(cr[t][u], nai[t], bi[u]);
          dmma(ci[t][u], ar[t], bi[u]);
          dmma(ci[t][u], ai[t], br[u]);
        }
    }
    __syncthreads();  // every warp is done with stage s before it is refilled
  }
#pragma unroll
  for (int t = 0; t < 4; ++t) {
    const int e = m0 + wm * 32 + t * 8 + lr;
    if (e >= p.M) continue;
#pragma unroll
    for (int u = 0; u < 2; ++u)
#pragma unroll
      for (int i = 0; i < 2; ++i) {
        const int j = n0 + wn * 16 + u * 8 + 2 * lc + i;
        if (j >= p.N) continue;
        Cx<double>* dst = p.C + (size_t)e + (size_t)p.ldc * j;
        const double vr = p.alpha * cr[t][u][i], vi = p.alpha * ci[t][u][i];
        if (p.beta == 0.0) {
          *dst = cx<double>(vr, vi);
        } else {
          const Cx<double> o = *dst;
          *dst = cx<double>(p.beta * o.x + vr, p.beta * o.y + vi);
        }
      }
  }
}

static int launch_dmma_dense(const DmArgs& args, cudaStream_t st) {
  static bool configured = false;
  if (!configured) {
    QCL_CUDA_CHECK(cudaFuncSetAttribute(dmma_dense_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)DM_SMEM));
    configured = true;
  }
  DmArgs a = args;
  const int mt = (a.M + DM_BM - 1) / DM_BM, nt = (a.N + DM_BN - 1) / DM_BN;
  // the larger operand is read once: an A larger than B and than L2 streams
  // with the column tiles fastest
  a.cols_fastest = a.M > a.N && (size_t)a.M * a.K * sizeof(Cx<double>) > ((size_t)96 << 20) && mt <= 65535;
  const dim3 grid = a.cols_fastest ? dim3(nt, mt) : dim3(mt, nt);
  dmma_dense_kernel<<<grid, DM_THREADS, DM_SMEM, st>>>(a);
  QCL_LAUNCH_CHECK("dmma_dense_kernel");
  return QCL_OK;
}

// ---------------------------------------------------------------------------
// Contraction dispatch
// ---------------------------------------------------------------------------
template <typename R>
static int contraction_t(const KernelOpDev& op, int NE, int Nk, int N, const double* wk, const void* Gv, void* Sv,
                         double alpha_q, double beta, void* work, cudaStream_t st) {
  const Cx<R>* G = (const Cx<R>*)Gv;
  Cx<R>* S = (Cx<R>*)Sv;
  const int N2 = N * N;
  const long long NEl = NE;
  if (op.kind == QCL_KERNEL_MOMENTUM_INDEPENDENT) {
    Cx<R>* X = (Cx<R>*)work;  // NE * N2
    const long long n = NEl * N2;
    momentum_sum_kernel<R><<<grid_cap(n, 256), 256, 0, st>>>(NE, Nk, N2, wk, G, X);
    QCL_LAUNCH_CHECK("momentum_sum_kernel");
    GemmArgs<R> g{};
    g.M = NE; g.Nout = N2; g.K = N2; g.batch = 1;
    g.A = X; g.lda = NEl; g.a_b = 0;
    g.B = (const Cx<R>*)op.block; g.ldb_j = 1; g.ldb_k = N2; g.b_b = 0;
    g.C = S; g.ldc = NEl * Nk; g.c_b = 0; g.bcast = Nk; g.bcast_stride = NEl;
    g.alpha = alpha_q; g.beta = beta;
    return launch_gemm<R>(g, st);
  }
  if (op.kind == QCL_KERNEL_DENSE) {
    const int Nc = Nk * N2;
    if (sizeof(R) == 4 && op.tc_bop)  // complex64 fields: tensor cores (scaled FP16 hi/lo)
      return launch_tc_dense_contraction(NE, Nc, op.tc_bop, Gv, Sv, alpha_q, beta, (float*)work, op.status, st);
    if (sizeof(R) == 8) {  // complex128: FP64 tensor path (DMMA)
      DmArgs d{NE, Nc, Nc, (const Cx<double>*)Gv, NEl, wk, Nk, (const Cx<double>*)op.matrix, Nc, (Cx<double>*)Sv, NEl,
               alpha_q, beta};
      return launch_dmma_dense(d, st);
    }
    GemmArgs<R> g{};
    g.M = NE; g.Nout = Nc; g.K = Nc; g.batch = 1;
    g.A = G; g.lda = NEl; g.wk = wk; g.wk_mod = Nk;
    g.B = (const Cx<R>*)op.matrix; g.ldb_j = 1; g.ldb_k = Nc;
    g.C = S; g.ldc = NEl; g.bcast = 1;
    g.alpha = alpha_q; g.beta = beta;
    return launch_gemm<R>(g, st);
  }
  if (op.kind == QCL_KERNEL_IFR) {
    const int J = op.J;
    Cx<R>* T = (Cx<R>*)work;                  // T[e + NE (j + J m')]
    Cx<R>* F = T + (size_t)NE * J * Nk;       // F[e + NE (j + J m)]
    int s;
    GemmArgs<R> g{};
    // stage 1, batch m': T = wk[m'] right * G_m'
    g.M = NE; g.Nout = J; g.K = N2; g.batch = Nk;
    g.A = G; g.lda = NEl * Nk; g.a_b = NEl; g.wb = wk;
    g.B = (const Cx<R>*)op.right; g.ldb_j = 1; g.ldb_k = J; g.b_b = 0;
    g.C = T; g.ldc = NEl; g.c_b = NEl * J; g.bcast = 1;
    g.alpha = 1.0; g.beta = 0.0;
    if ((s = launch_gemm<R>(g, st))) return s;
    // stage 2, batch j: F[., j, m] = sum_m' radial[m, m'] T[., j, m']
    GemmArgs<R> h{};
    h.M = NE; h.Nout = Nk; h.K = Nk; h.batch = J;
    h.A = T; h.lda = NEl * J; h.a_b = NEl;
    h.B = (const Cx<R>*)op.radial; h.ldb_j = 1; h.ldb_k = Nk; h.b_b = 0;
    h.C = F; h.ldc = NEl * J; h.c_b = NEl; h.bcast = 1;
    h.alpha = 1.0; h.beta = 0.0;
    if ((s = launch_gemm<R>(h, st))) return s;
    // stage 3, batch m: S[., m, p] = alpha q sum_j left[p, j] F[., j, m] + beta S
    GemmArgs<R> f{};
    f.M = NE; f.Nout = N2; f.K = J; f.batch = Nk;
    f.A = F; f.lda = NEl; f.a_b = NEl * J;
    f.B = (const Cx<R>*)op.left; f.ldb_j = 1; f.ldb_k = N2; f.b_b = 0;
    f.C = S; f.ldc = NEl * Nk; f.c_b = NEl; f.bcast = 1;
    f.alpha = alpha_q; f.beta = beta;
    return launch_gemm<R>(f, st);
  }
  if (op.kind == QCL_KERNEL_LOW_RANK) {
    // LowRankProductionKernel (production_operators.jl:597-658):
    //   T[e, r] = sum_q right_adjoint[r, q] wk[q % Nk] G[e, q]      (NE x rank)
    //   S[e, q] = alpha q^K sum_r left[q, r] T[e, r] + beta S[e, q]
    const int Nc = Nk * N2, r = op.J;
    Cx<R>* T = (Cx<R>*)work;
    int s;
    if (sizeof(R) == 8) {
      DmArgs d1{NE, r, Nc, (const Cx<double>*)Gv, NEl, wk, Nk, (const Cx<double>*)op.right, r, (Cx<double>*)work,
                NEl, 1.0, 0.0};
      if ((s = launch_dmma_dense(d1, st))) return s;
      DmArgs d2{NE, Nc, r, (const Cx<double>*)work, NEl, nullptr, 1, (const Cx<double>*)op.left, Nc,
                (Cx<double>*)Sv, NEl, alpha_q, beta};
      return launch_dmma_dense(d2, st);
    }
    GemmArgs<R> g{};
    g.M = NE; g.Nout = r; g.K = Nc; g.batch = 1;
    g.A = G; g.lda = NEl; g.wk = wk; g.wk_mod = Nk;
    g.B = (const Cx<R>*)op.right; g.ldb_j = 1; g.ldb_k = r;
    g.C = T; g.ldc = NEl; g.bcast = 1;
    g.alpha = 1.0; g.beta = 0.0;
    if ((s = launch_gemm<R>(g, st))) return s;
    GemmArgs<R> f{};
    f.M = NE; f.Nout = Nc; f.K = r; f.batch = 1;
    f.A = T; f.lda = NEl;
    f.B = (const Cx<R>*)op.left; f.ldb_j = 1; f.ldb_k = Nc;
    f.C = S; f.ldc = NEl; f.bcast = 1;
    f.alpha = alpha_q; f.beta = beta;
    return launch_gemm<R>(f, st);
  }
  if (op.kind == QCL_KERNEL_SEPARABLE_SUM) {
    // K(m,m') = sum_i radial_i(m,m') block_i: a Kronecker sum of J terms (the
    // exact LO form sum_h R_h(m,m') F_h (x) conj F_h of lo_phonon_kernel,
    // numerics/reference/kernels.jl:321-356, and the tabulated kernels of
    // numerics/optimized/kernels.jl:303-320, compressed on the host).  Per
    // chunk of up to kSepChunk terms:
    //   stage 1 (term i, batch (c,d)):  Z_i[e + NE m + NE Nk (c,d)] =
    //            sum_m' radial_i[m + Nk m'] wk[m'] G[e + NE m' + NE Nk (c,d)]
    //   stage 2 (one GEMM over the chunk, K = (c,d,i)):
    //            S[(e,m), (a,b)] = alpha q sum_k Z[(e,m), k] block[(a,b), k] + beta S
    // The rows of stage 2 are the (e, m) pairs, contiguous in the E-fastest
    // layout, so S and Z are plain column-major (NE Nk) x N^2 matrices.
    const int J = op.J;
    const long long Mr = NEl * Nk;                // stage-2 rows
    const size_t zfield = (size_t)Mr * N2;        // one intermediate field
    Cx<R>* Z = (Cx<R>*)work;
    const int jmax = J < kSepChunk ? J : kSepChunk;  // terms per chunk
    float* awork = (float*)((char*)work + (size_t)jmax * zfield * sizeof(Cx<R>));
    // complex64 with tensor-core stage-1 operands: G split once for all chunks,
    // rows (e, (c,d)), K = m', behind the stage-2 work area
    float* gwork = awork + tc_a_work_floats2((int)Mr, jmax * N2);
    int s;
    if (sizeof(R) == 4 && op.tc_stage1 && (s = tc_split_rows(NE * N2, Nk, Gv, NEl, NEl * Nk, gwork, st))) return s;
    for (int c = 0, i0 = 0; i0 < J; ++c, i0 += kSepChunk) {
      const int jc = min(kSepChunk, J - i0);
      if (sizeof(R) == 4 && op.tc_stage1) {
        // stage 1 on the tensor cores: rows (e, (c,d)), columns (m, i), K = m';
        // the output index (e, m, (c,d), i) is the chunk's intermediate layout
        if ((s = launch_tc_presplit(NE * N2, Nk * jc, Nk, op.tc_stage1[c], gwork, Z, NEl, Nk, N2, 1.0, 0.0,
                                    op.status, st)))
          return s;
      } else
      for (int i = i0; i < i0 + jc; ++i) {
        GemmArgs<R> g{};
        g.M = NE; g.Nout = Nk; g.K = Nk; g.batch = N2;
        g.A = G; g.lda = NEl; g.a_b = Mr; g.wk = wk; g.wk_mod = Nk;
        g.B = (const Cx<R>*)op.radial + (size_t)Nk * Nk * i; g.ldb_j = 1; g.ldb_k = Nk; g.b_b = 0;
        g.C = Z + zfield * (i - i0); g.ldc = NEl; g.c_b = Mr; g.bcast = 1;
        g.alpha = 1.0; g.beta = 0.0;
        if ((s = launch_gemm<R>(g, st))) return s;
      }
      const double bc = c == 0 ? beta : 1.0;
      const Cx<R>* blk = (const Cx<R>*)op.block + (size_t)N2 * N2 * i0;
      if (sizeof(R) == 8) {
        DmArgs d{(int)Mr, N2, jc * N2, (const Cx<double>*)Z, Mr, nullptr, 1, (const Cx<double>*)blk, N2,
                 (Cx<double>*)Sv, Mr, alpha_q, bc};
        if ((s = launch_dmma_dense(d, st))) return s;
      } else if (op.tc_chunks) {
        if ((s = launch_tc_contraction2((int)Mr, N2, jc * N2, op.tc_chunks[c], Z, Sv, alpha_q, bc, awork, op.status,
                                        st)))
          return s;
      } else {
        GemmArgs<R> f{};
        f.M = (int)Mr; f.Nout = N2; f.K = jc * N2; f.batch = 1;
        f.A = Z; f.lda = Mr;
        f.B = blk; f.ldb_j = 1; f.ldb_k = N2;
        f.C = S; f.ldc = Mr; f.bcast = 1;
        f.alpha = alpha_q; f.beta = bc;
        if ((s = launch_gemm<R>(f, st))) return s;
      }
    }
    return QCL_OK;
  }
  set_last_error("unknown kernel operator kind %d", op.kind);
  return QCL_ARG;
}

// Stage-1 operand of a chunk of separable-sum terms [i0, i0 + jc):
// Mop[(m + Nk i') + Nk jc m'] = radial[m + Nk m' + Nk^2 (i0 + i')] (complex64).
__global__ void sep_radial_gather_kernel(int Nk, int i0, int jc, const Cx<float>* __restrict__ radial,
                                         Cx<float>* __restrict__ out) {
  const long long n = (long long)Nk * jc * Nk;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
    const int m = (int)(t % Nk), ip = (int)((t / Nk) % jc), mp = (int)(t / ((long long)Nk * jc));
    out[t] = radial[(size_t)m + (size_t)Nk * mp + (size_t)Nk * Nk * (i0 + ip)];
  }
}

// Tensor-core operands of a complex64 separable sum: per chunk of kSepChunk
// terms the stage-2 operand (the stacked blocks, N^2 x jc N^2) and the
// stage-1 operand (the radial factors with the momentum weights, Nk jc x Nk).
int sep_build_tc_operands(int Nk, int N, int J, const void* radial_c64, const void* block_c64, const double* wk,
                          std::vector<void*>& stage2, std::vector<void*>& stage1, cudaStream_t st) {
  const int N2 = N * N;
  void* tmp = nullptr;
  QCL_CUDA_CHECK(cudaMalloc(&tmp, (size_t)Nk * Nk * kSepChunk * sizeof(Cx<float>)));
  int s = QCL_OK;
  for (int i0 = 0; i0 < J && !s; i0 += kSepChunk) {
    const int jc = J - i0 < kSepChunk ? J - i0 : kSepChunk;
    void* b = nullptr;
    s = tc_build_operator2(N2, jc * N2, 1, (const Cx<float>*)block_c64 + (size_t)N2 * N2 * i0, nullptr, &b, st);
    if (b) stage2.push_back(b);
    if (s) break;
    sep_radial_gather_kernel<<<grid_cap((long long)Nk * jc * Nk, 256), 256, 0, st>>>(
        Nk, i0, jc, (const Cx<float>*)radial_c64, (Cx<float>*)tmp);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
      s = cuda_status(e, "sep_radial_gather_kernel");
      break;
    }
    b = nullptr;
    s = tc_build_operator2(Nk * jc, Nk, Nk, tmp, wk, &b, st);
    if (b) stage1.push_back(b);
    cudaStreamSynchronize(st);  // tmp is reused by the next chunk
  }
  cudaStreamSynchronize(st);
  cudaFree(tmp);
  return s;
}

size_t contraction_work_elems(const KernelOpDev& op, int NE, int Nk, int N) {
  if (op.kind == QCL_KERNEL_MOMENTUM_INDEPENDENT) return (size_t)NE * N * N;
  if (op.kind == QCL_KERNEL_DENSE && op.tc_bop) return (tc_a_work_floats(NE, Nk * N * N) + 1) / 2;  // complex64 units
  if (op.kind == QCL_KERNEL_IFR) return 2 * (size_t)NE * op.J * Nk;
  if (op.kind == QCL_KERNEL_LOW_RANK) return (size_t)NE * op.J;
  if (op.kind == QCL_KERNEL_SEPARABLE_SUM) {
    // kSepChunk intermediate fields (field precision), then for complex64
    // tensor-core chunks the stage-2 A operand (floats) in complex64 units
    const int jmax = op.J < kSepChunk ? op.J : kSepChunk;
    const size_t zf = (size_t)jmax * NE * Nk * N * N;
    if (op.tc_chunks)
      return zf + (tc_a_work_floats2(NE * Nk, jmax * N * N) + (op.tc_stage1 ? tc_a_work_floats2(NE * N * N, Nk) : 0) +
                   1) / 2;
    return zf;
  }
  return 0;
}

int launch_contraction(int precision, const KernelOpDev& op, int NE, int Nk, int N, const double* wk, const void* G,
                       void* S, double alpha_q, double beta, void* work, cudaStream_t st) {
  if (precision == QCL_C128) return contraction_t<double>(op, NE, Nk, N, wk, G, S, alpha_q, beta, work, st);
  return contraction_t<float>(op, NE, Nk, N, wk, G, S, alpha_q, beta, work, st);
}

}  // namespace qcl
