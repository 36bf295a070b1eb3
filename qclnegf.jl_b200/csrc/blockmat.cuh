// Block-matrix building blocks shared by the per-(E,k) kernels: swizzled
// shared-memory N x N tiles, team barriers and reductions, team-tiled complex
// matmuls, and coalesced copies between E-fastest fields and the tiles.
#pragma once
#include "kernels.cuh"

namespace qcl {

template <int NP> __device__ __forceinline__ int sw(int r, int c) { return r * NP + (c ^ (r & 7)); }

// Static tiling per padded block size NP.
template <int NP> struct Tile;
template <> struct Tile<8> { static constexpr int CPR = 4, TT = 32, TR = 1, TC = 2; };
template <> struct Tile<16> { static constexpr int CPR = 2, TT = 32, TR = 2, TC = 4; };
template <> struct Tile<24> { static constexpr int CPR = 1, TT = 32, TR = 3, TC = 6; };
template <> struct Tile<32> { static constexpr int CPR = 2, TT = 64, TR = 4, TC = 4; };
template <> struct Tile<48> { static constexpr int CPR = 2, TT = 96, TR = 4, TC = 6; };

// Team barrier: a warp sync for one-warp teams, a named barrier otherwise.
template <int TT> __device__ __forceinline__ void team_sync(int team) {
  if (TT == 32) {
    __syncwarp();
  } else {
    asm volatile("bar.sync %0, %1;" ::"r"(team + 1), "n"(TT) : "memory");
  }
}

// Team-wide sum of a double (fixed tree order -> deterministic).
template <int TT>
__device__ __forceinline__ double team_sum(double v, int tt, double* scratch /* TT/32 */, int team) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  if (TT == 32) return v;
  team_sync<TT>(team);
  if ((tt & 31) == 0) scratch[tt >> 5] = v;
  team_sync<TT>(team);
  double s = 0;
#pragma unroll
  for (int w = 0; w < TT / 32; ++w) s += scratch[w];
  return s;
}

template <int TT>
__device__ __forceinline__ double team_max(double v, int tt, double* scratch, int team) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
  if (TT == 32) return v;
  team_sync<TT>(team);
  if ((tt & 31) == 0) scratch[tt >> 5] = v;
  team_sync<TT>(team);
  double s = scratch[0];
#pragma unroll
  for (int w = 1; w < TT / 32; ++w) s = fmax(s, scratch[w]);
  return s;
}

// Per-team shared scratch besides the three matrices.
template <typename RL, int NP, int TT> struct TeamScratch {
  Cx<RL> rowbuf[2][NP];
  int pivrow[NP];
  double red[TT / 32 > 0 ? TT / 32 : 1];
  // multi-warp argmax exchange
  unsigned long long wkey[TT / 32 > 0 ? TT / 32 : 1];
};

// Warp argmax of (mag, row), ties broken towards the smaller row index.
__device__ __forceinline__ void warp_argmax(double& mag, int& row) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    double om = __shfl_xor_sync(0xffffffffu, mag, o);
    int orow = __shfl_xor_sync(0xffffffffu, row, o);
    if (om > mag || (om == mag && orow < row)) {
      mag = om;
      row = orow;
    }
  }
}

// Register tile of a team matmul: thread tt owns rows rg*TR + t and columns
// cg*TC + u of the NP x NP product.
template <typename RM, int NP> struct MatTile {
  static constexpr int TR = Tile<NP>::TR, TC = Tile<NP>::TC, RG = NP / TR;
  Cx<RM> v[TR][TC];
};

// acc = A * B (adjB = false) or A * B^H (adjB = true) over the N x N active
// part of NP x NP swizzled shared matrices; RM is the arithmetic precision.
template <typename RS, typename RM, int NP>
__device__ __forceinline__ void team_matmul_regs(const Cx<RS>* A, const Cx<RS>* B, MatTile<RM, NP>& acc, int N,
                                                 int tt, bool adjB) {
  // thread (rg, cg) owns rows rg + RG t and columns cg + CG u: the rows a warp
  // reads together differ in their low three bits, so the swizzled column walk
  // of A (and of B^H) is free of bank conflicts
  constexpr int TR = Tile<NP>::TR, TC = Tile<NP>::TC, RG = NP / TR, CG = NP / TC;
  const int rg = tt % RG, cg = tt / RG;
#pragma unroll
  for (int t = 0; t < TR; ++t)
#pragma unroll
    for (int u = 0; u < TC; ++u) acc.v[t][u] = cx<RM>(0, 0);
  for (int l = 0; l < N; ++l) {
    Cx<RM> a[TR], b[TC];
#pragma unroll
    for (int t = 0; t < TR; ++t) a[t] = cvt<RM>(A[sw<NP>(rg + RG * t, l)]);
#pragma unroll
    for (int u = 0; u < TC; ++u) {
      const int j = cg + CG * u;
      b[u] = adjB ? conj(cvt<RM>(B[sw<NP>(j, l)])) : cvt<RM>(B[sw<NP>(l, j)]);
    }
#pragma unroll
    for (int t = 0; t < TR; ++t)
#pragma unroll
      for (int u = 0; u < TC; ++u) cfma(acc.v[t][u], a[t], b[u]);
  }
}

template <typename RS, typename RM, int NP>
__device__ __forceinline__ void team_store_regs(Cx<RS>* C, const MatTile<RM, NP>& acc, int tt) {
  constexpr int TR = Tile<NP>::TR, TC = Tile<NP>::TC, RG = NP / TR, CG = NP / TC;
  const int rg = tt % RG, cg = tt / RG;
#pragma unroll
  for (int t = 0; t < TR; ++t)
#pragma unroll
    for (int u = 0; u < TC; ++u) C[sw<NP>(rg + RG * t, cg + CG * u)] = cvt<RS>(acc.v[t][u]);
}


// ---------------------------------------------------------------------------
// FP64 tensor-core (DMMA, mma.sync m8n8k4 f64) version of the team matmul for
// complex128 tiles.  The NP x NP product is cut into (NP/8)^2 tiles of 8 x 8;
// warp w of the team owns tile rows w, w + NW, ...  Each complex product is
// four real DMMAs (Re C += Ar Br - Ai Bi, Im C += Ar Bi + Ai Br), and K
// advances by 4 with entries past N read as zero.  Fragment layouts (PTX
// m8n8k4 .f64): A lane l holds (l/4, l%4), B holds (l%4, l/4), C holds
// (l/4, 2 (l%4) + i).  One DMMA issue does the 256 FMAs of 8 DFMA issues
// per lane.
// ---------------------------------------------------------------------------
__device__ __forceinline__ void dmma_f64(double (&c)[2], double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};"
               : "+d"(c[0]), "+d"(c[1])
               : "d"(a), "d"(b));
}

template <int NP, int TT> struct DmmaTile {
  static constexpr int NT = NP / 8, NW = TT / 32, RPW = (NT + NW - 1) / NW;
  double re[RPW][NT][2], im[RPW][NT][2];
};

template <int NP, int TT>
__device__ __forceinline__ void team_matmul_dmma(const Cx<double>* A, const Cx<double>* B, DmmaTile<NP, TT>& acc,
                                                 int N, int tt, bool adjB) {
  constexpr int NT = DmmaTile<NP, TT>::NT, NW = DmmaTile<NP, TT>::NW, RPW = DmmaTile<NP, TT>::RPW;
  const int warp = tt >> 5, lane = tt & 31, lr = lane >> 2, lc = lane & 3;
#pragma unroll
  for (int r = 0; r < RPW; ++r)
#pragma unroll
    for (int j = 0; j < NT; ++j) acc.re[r][j][0] = acc.re[r][j][1] = acc.im[r][j][0] = acc.im[r][j][1] = 0.0;
  for (int k0 = 0; k0 < N; k0 += 4) {
    const int k = k0 + lc;
    const bool kin = k < N;
    double ar[RPW], ai[RPW], nai[RPW], br[NT], bi[NT];
#pragma unroll
    for (int r = 0; r < RPW; ++r) {
      const bool rin = warp + r * NW < NT;  // warp-uniform
      const Cx<double> a = kin && rin ? A[sw<NP>((warp + r * NW) * 8 + lr, k)] : cx<double>(0, 0);
      ar[r] = a.x;
      ai[r] = a.y;
      nai[r] = -a.y;
    }
#pragma unroll
    for (int j = 0; j < NT; ++j) {
      Cx<double> b = cx<double>(0, 0);
      if (kin) b = adjB ? conj(B[sw<NP>(j * 8 + lr, k)]) : B[sw<NP>(k, j * 8 + lr)];
      br[j] = b.x;
      bi[j] = b.y;
    }
#pragma unroll
    for (int r = 0; r < RPW; ++r)
#pragma unroll
      for (int j = 0; j < NT; ++j) {
        if (RPW * NW != NT && warp + r * NW >= NT) continue;  // warp-uniform: no tile row here
        dmma_f64(acc.re[r][j], ar[r], br[j]);
        dmma_f64(acc.re[r][j], nai[r], bi[j]);
        dmma_f64(acc.im[r][j], ar[r], bi[j]);
        dmma_f64(acc.im[r][j], ai[r], br[j]);
      }
  }
}

// The same product with three real DMMAs per complex tile product (the 3M
// form): T1 = Ar Br, T2 = Ai Bi, T3 = (Ar + Ai)(Br + Bi), then Re C = T1 - T2
// and Im C = T3 - T1 - T2.  A quarter fewer tensor-core issues; the error
// stays within the norm-wise bound of the four-product form (a few eps times
// (|Ar| + |Ai|)(|Br| + |Bi|) per term).  Used by the Keldysh products of the
// Dyson kernel.
template <int NP, int TT>
__device__ __forceinline__ void team_matmul_dmma3(const Cx<double>* A, const Cx<double>* B, DmmaTile<NP, TT>& acc,
                                                  int N, int tt, bool adjB) {
  constexpr int NT = DmmaTile<NP, TT>::NT, NW = DmmaTile<NP, TT>::NW, RPW = DmmaTile<NP, TT>::RPW;
  const int warp = tt >> 5, lane = tt & 31, lr = lane >> 2, lc = lane & 3;
  double t3[RPW][NT][2];
#pragma unroll
  for (int r = 0; r < RPW; ++r)
#pragma unroll
    for (int j = 0; j < NT; ++j)
#pragma unroll
      for (int i = 0; i < 2; ++i) acc.re[r][j][i] = acc.im[r][j][i] = t3[r][j][i] = 0.0;  // re: T1, im: T2
  for (int k0 = 0; k0 < N; k0 += 4) {
    const int k = k0 + lc;
    const bool kin = k < N;
    double ar[RPW], ai[RPW], as[RPW], br[NT], bi[NT], bs[NT];
#pragma unroll
    for (int r = 0; r < RPW; ++r) {
      const bool rin = warp + r * NW < NT;  // warp-uniform
      const Cx<double> a = kin && rin ? A[sw<NP>((warp + r * NW) * 8 + lr, k)] : cx<double>(0, 0);
      ar[r] = a.x;
      ai[r] = a.y;
      as[r] = a.x + a.y;
    }
#pragma unroll
    for (int j = 0; j < NT; ++j) {
      Cx<double> b = cx<double>(0, 0);
      if (kin) b = adjB ? conj(B[sw<NP>(j * 8 + lr, k)]) : B[sw<NP>(k, j * 8 + lr)];
      br[j] = b.x;
      bi[j] = b.y;
      bs[j] = b.x + b.y;
    }
#pragma unroll
    for (int r = 0; r < RPW; ++r)
#pragma unroll
      for (int j = 0; j < NT; ++j) {
        if (RPW * NW != NT && warp + r * NW >= NT) continue;  // warp-uniform: no tile row here
        dmma_f64(acc.re[r][j], ar[r], br[j]);
        dmma_f64(acc.im[r][j], ai[r], bi[j]);
        dmma_f64(t3[r][j], as[r], bs[j]);
      }
  }
#pragma unroll
  for (int r = 0; r < RPW; ++r)
#pragma unroll
    for (int j = 0; j < NT; ++j)
#pragma unroll
      for (int i = 0; i < 2; ++i) {
        const double t1 = acc.re[r][j][i], t2 = acc.im[r][j][i];
        acc.re[r][j][i] = t1 - t2;
        acc.im[r][j][i] = (t3[r][j][i] - t1) - t2;
      }
}

template <int NP, int TT>
__device__ __forceinline__ void team_store_dmma(Cx<double>* C, const DmmaTile<NP, TT>& acc, int tt) {
  constexpr int NT = DmmaTile<NP, TT>::NT, NW = DmmaTile<NP, TT>::NW, RPW = DmmaTile<NP, TT>::RPW;
  const int warp = tt >> 5, lane = tt & 31, lr = lane >> 2, lc = lane & 3;
#pragma unroll
  for (int r = 0; r < RPW; ++r) {
    if (RPW * NW != NT && warp + r * NW >= NT) continue;
#pragma unroll
    for (int j = 0; j < NT; ++j)
#pragma unroll
      for (int i = 0; i < 2; ++i)
        C[sw<NP>((warp + r * NW) * 8 + lr, j * 8 + 2 * lc + i)] = cx<double>(acc.re[r][j][i], acc.im[r][j][i]);
  }
}

// C = A * B (adjB = false) or C = A * B^H (adjB = true); C distinct from A, B.
// complex128 tiles go through the FP64 tensor path (DMMA).
template <typename RS, typename RM, int NP>
__device__ __forceinline__ void team_matmul(const Cx<RS>* A, const Cx<RS>* B, Cx<RS>* C, int N, int tt,
                                            bool adjB) {
  if constexpr (sizeof(RS) == 8 && sizeof(RM) == 8) {
    DmmaTile<NP, Tile<NP>::TT> acc;
    team_matmul_dmma<NP, Tile<NP>::TT>((const Cx<double>*)A, (const Cx<double>*)B, acc, N, tt, adjB);
    team_store_dmma<NP, Tile<NP>::TT>((Cx<double>*)C, acc, tt);
  } else {
    MatTile<RM, NP> acc;
    team_matmul_regs<RS, RM, NP>(A, B, acc, N, tt, adjB);
    team_store_regs<RS, RM, NP>(C, acc, tt);
  }
}

// Cooperative, coalesced copy of BPC consecutive-energy blocks between a
// global field (E fastest) and the per-block shared matrices.
template <typename RG_, typename RS, int NP, int BPC>
__device__ __forceinline__ void load_blocks(const Cx<RG_>* __restrict__ X, Cx<RS>* bufs, size_t stride_buf,
                                            int e0, int m, int NE, int Nk, int N) {
  const int total = BPC * NP * N;  // rows padded to NP: compile-time index split
  const size_t base = (size_t)e0 + (size_t)NE * m, cstride = (size_t)NE * Nk;
  for (int i = threadIdx.x; i < total; i += blockDim.x) {
    const int eloc = i % BPC, el = i / BPC;
    const int a = el % NP, b = el / NP;
    if (a >= N) continue;
    const int e = e0 + eloc;
    Cx<RS> v = cx<RS>(0, 0);
    if (e < NE) v = cvt<RS>(X[base + eloc + cstride * ((size_t)a + (size_t)N * b)]);
    bufs[eloc * stride_buf + sw<NP>(a, b)] = v;
  }
}

// Asynchronous variant (cp.async, zero fill past N_E): issues every copy of the
// tile without waiting, so the whole tile is in flight at once; the caller
// commits, waits and synchronises.  Storage and shared precision must match.
template <typename R> __device__ __forceinline__ void cp_async_elem(Cx<R>* smem, const Cx<R>* gmem, bool valid) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  const int n = valid ? (int)sizeof(Cx<R>) : 0;
  if (sizeof(Cx<R>) == 16)
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(s), "l"(gmem), "r"(n) : "memory");
  else
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;" ::"r"(s), "l"(gmem), "r"(n) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;" ::: "memory"); }

template <typename R, int NP, int BPC>
__device__ __forceinline__ void load_blocks_async(const Cx<R>* __restrict__ X, Cx<R>* bufs, size_t stride_buf, int e0,
                                                  int m, int NE, int Nk, int N) {
  const int total = BPC * NP * N;
  const size_t base = (size_t)e0 + (size_t)NE * m, cstride = (size_t)NE * Nk;
  for (int i = threadIdx.x; i < total; i += blockDim.x) {
    const int eloc = i % BPC, el = i / BPC;
    const int a = el % NP, b = el / NP;
    if (a >= N) continue;
    const bool ok = e0 + eloc < NE;
    const Cx<R>* src = X + (ok ? base + eloc + cstride * ((size_t)a + (size_t)N * b) : 0);
    cp_async_elem<R>(bufs + eloc * stride_buf + sw<NP>(a, b), src, ok);
  }
  cp_async_commit();
}

template <typename RG_, typename RS, int NP, int BPC>
__device__ __forceinline__ void store_blocks(Cx<RG_>* __restrict__ X, const Cx<RS>* bufs, size_t stride_buf,
                                             int e0, int m, int NE, int Nk, int N) {
  const int total = BPC * NP * N;
  const size_t base = (size_t)e0 + (size_t)NE * m, cstride = (size_t)NE * Nk;
  for (int i = threadIdx.x; i < total; i += blockDim.x) {
    const int eloc = i % BPC, el = i / BPC;
    const int a = el % NP, b = el / NP;
    if (a >= N || e0 + eloc >= NE) continue;
    X[base + eloc + cstride * ((size_t)a + (size_t)N * b)] = cvt<RG_>(bufs[eloc * stride_buf + sw<NP>(a, b)]);
  }
}


}  // namespace qcl
