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
#include <mutex>

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

// Argmax key of a pivot candidate: the high 32 bits of its magnitude (IEEE
// order = unsigned order for non-negative values) with the low 6 bits replaced
// by (63 - row), so that one unsigned warp max (redux.sync) finds the largest
// candidate, ties and near-ties (below 2^-14 relative, for double; 2^-17 for
// float) going to the smaller row.  Any candidate within that margin of the
// maximum is as good a partial pivot.  Key 0 = no candidate.
__device__ __forceinline__ unsigned pivot_key(double mag, int row) {
  return ((unsigned)__double2hiint(mag) & ~63u) | (unsigned)(63 - row);
}
__device__ __forceinline__ unsigned pivot_key(float mag, int row) {
  return (__float_as_uint(mag) & ~63u) | (unsigned)(63 - row);
}
__device__ __forceinline__ bool pivot_key_zero(unsigned key) { return (key >> 6) == 0u; }

// Shared-memory store under a predicate, without a branch.
__device__ __forceinline__ void st_shared_if(Cx<double>* ptr, Cx<double> v, bool pred) {
  const unsigned a = (unsigned)__cvta_generic_to_shared(ptr);
  asm volatile(
      "{\n .reg .pred q;\n setp.ne.u32 q, %3, 0;\n @q st.shared.v2.f64 [%0], {%1, %2};\n}" ::"r"(a),
      "d"(v.x), "d"(v.y), "r"((unsigned)pred)
      : "memory");
}
__device__ __forceinline__ void st_shared_if(Cx<float>* ptr, Cx<float> v, bool pred) {
  const unsigned a = (unsigned)__cvta_generic_to_shared(ptr);
  asm volatile(
      "{\n .reg .pred q;\n setp.ne.u32 q, %3, 0;\n @q st.shared.v2.f32 [%0], {%1, %2};\n}" ::"r"(a),
      "f"(v.x), "f"(v.y), "r"((unsigned)pred)
      : "memory");
}

// Per-team scratch of the Dyson kernel (the pivot-row exchange buffer lives in
// the team's G^R tile, which is unused until the elimination ends).
template <int TT> struct DysonScratch {
  int pivrow[48];
  double red[TT / 32];
  unsigned wkey[2 * (TT / 32)];
};

// Steps of the elimination unrolled per group (static register indices); the
// row chunk is rotated by the group width between groups.  Wider groups save
// the rotation moves, narrower ones keep the loop in the instruction cache.
#ifndef QCL_GJ_GROUP
#define QCL_GJ_GROUP 4
#endif
template <int NP> struct GjUnroll {
  static constexpr int COLS = NP / Tile<NP>::CPR;
  static constexpr int U = COLS % QCL_GJ_GROUP == 0 ? QCL_GJ_GROUP : COLS;
};

template <typename RS, typename RL, int NP, int TT, int BPC> constexpr size_t dyson_smem() {
  static_assert(2 * (NP + 1) * sizeof(Cx<RL>) <= NP * NP * sizeof(Cx<RS>), "pivot rows fit the G tile");
  return 2 * (size_t)BPC * NP * NP * sizeof(Cx<RS>) + BPC * sizeof(DysonScratch<TT>);
}

// CTAs per SM that the shared memory allows (228 KB per SM, 1 KB reserved per
// CTA), as the register budget's occupancy target -- but never below 128
// registers per thread, where the elimination rows would spill (160 for the
// two-dimensional elimination with FP64 entries at N_b <= 24).
template <typename RS, typename RL, int NP, int BPC> constexpr int dyson_min_ctas() {
  constexpr size_t per = dyson_smem<RS, RL, NP, Tile<NP>::TT, BPC>() + 1024;
  constexpr int by_smem = (int)((228 * 1024) / per);
  constexpr int floor_regs = NP == 24 && sizeof(RL) == 8 ? 160 : 128;
  constexpr int by_regs = 65536 / (BPC * Tile<NP>::TT * floor_regs);
  constexpr int n = by_smem < by_regs ? by_smem : by_regs;
  return n < 1 ? 1 : n;
}

// D build, equilibration and Gauss-Jordan of one N_b <= 24 block on a 32-lane
// team with two-dimensional ownership: lane (rg, cg) = (lane / 4, lane % 4)
// holds rows rg, rg + 8, rg + 16 and columns 6 cg .. 6 cg + 5 (18 entries), so
// all 32 lanes update where one row per lane leaves 8 idle.  The arithmetic
// per entry is that of the row-per-lane form (same pivot keys, deferred
// scaling, speculative reciprocal); only the row sums of the equilibration
// are added in a different order.  Step k: the 8 lanes holding column k
// offer their best unused row, one warp max picks the pivot row p; those
// lanes publish column k (the multipliers) and turn it into e_p; the 4 lanes
// holding row p publish it; every lane then updates its 18 entries.  Writes
// G (inverse columns in pivot order) into the team's G tile and the scale.
template <typename RS, typename RL, int BPC>
__device__ __forceinline__ void dyson_gj_2d24(const DysonArgs<RS>& p, Cx<RS>* X, Cx<RS>* G, DysonScratch<32>& S,
                                              Cx<RS>* bufX, int team, int tt, int e, int e0, int m, bool live,
                                              const Cx<RS>* first_sig, bool first_is_L) {
  constexpr int NP = 24, RW = 3, CW = 6;
  const int N = p.N, NE = p.NE, Nk = p.Nk;
  const int rg = tt >> 2, cg = tt & 3;
  Cx<RL> w[RW][CW];
  const double eps_e = live ? p.eps[e] : 0.0;
  double rmax = 0.0;
#pragma unroll
  for (int i = 0; i < RW; ++i) {
    const int row = rg + 8 * i;
    double rsum = 0.0;
#pragma unroll
    for (int c = 0; c < CW; ++c) {
      const int col = CW * cg + c;
      Cx<RL> d = cx<RL>(0, 0);
      if (row < N && col < N) {
        const Cx<double> hv = p.h[(size_t)m + (size_t)Nk * ((size_t)row + (size_t)N * col)];
        const Cx<RS> sv = X[sw<NP>(row, col)];
        double re = -hv.x - (double)sv.x, im = -hv.y - (double)sv.y;
        if (row == col) {
          re += eps_e;
          im += p.eta;
        }
        d = cx<RL>((RL)re, (RL)im);
        rsum += sqrt(re * re + im * im);
      }
      w[i][c] = d;
    }
    rsum += __shfl_xor_sync(0xffffffffu, rsum, 1);  // the row's four column groups
    rsum += __shfl_xor_sync(0xffffffffu, rsum, 2);
    rmax = fmax(rmax, rsum);
  }
  __syncthreads();  // every team has read its SigmaR tile: bufX is free
  // prefetch the first Keldysh input while the inversion runs
  if (first_sig && (first_is_L ? p.GL : p.GG)) load_blocks_async<RS, NP, BPC>(first_sig, bufX, NP * NP, e0, m, NE, Nk, N);
  const double s = team_max<32>(rmax, tt, S.red, team);
  const RL inv_s = (RL)(1.0 / s);
  const bool scale_ok = s > 0.0 && isfinite(s);
#pragma unroll
  for (int i = 0; i < RW; ++i)
#pragma unroll
    for (int c = 0; c < CW; ++c) {
      const int row = rg + 8 * i, col = CW * cg + c;
      w[i][c] = inv_s * w[i][c];
      if (row >= N && col == row) w[i][c] = cx<RL>(1, 0);  // identity padding
    }

  // rows rg + 8 i; bit i of `used` set once the row has been a pivot.  The G
  // tile holds, until the elimination ends, two step buffers (pivot row,
  // multipliers, spare slot), then each row's pivot reciprocal and step.
  unsigned used = 0u;
  bool singular = !scale_ok;
  int zstep = -1;
  Cx<RL>* rb0 = reinterpret_cast<Cx<RL>*>(G);
  Cx<RL>* rcrow = rb0 + 2 * (2 * NP + 1);
  int* stepof = reinterpret_cast<int*>(rcrow + NP);
  static_assert((2 * (2 * NP + 1) + NP) * sizeof(Cx<RL>) + NP * sizeof(int) <= NP * NP * sizeof(Cx<RS>),
                "elimination scratch fits the G tile");
#pragma unroll 1
  for (int kc = 0; kc < NP / CW; ++kc) {
    const bool own = cg == kc;
#pragma unroll
    for (int u = 0; u < CW; ++u) {
      const int k = kc * CW + u;
      // this lane's best unused row in column k (keys as the row-per-lane form;
      // non-zero keys are distinct, so the winner is found by equality)
      unsigned kk[RW];
#pragma unroll
      for (int i = 0; i < RW; ++i)
        kk[i] = own && !((used >> i) & 1u) ? pivot_key(cabs1(w[i][u]), rg + 8 * i) : 0u;
      const unsigned mykey = max(kk[0], max(kk[1], kk[2]));
      Cx<RL> cv = mykey == kk[1] ? w[1][u] : w[0][u];
      cv = mykey == kk[2] ? w[2][u] : cv;
      const Cx<RL> rc = crecip_pivot(cv);  // speculative, off the argmax path
      const unsigned key = __reduce_max_sync(0xffffffffu, mykey);
      const int best = 63 - (int)(key & 63u);
      const bool zero = pivot_key_zero(key);
      const bool plane = own && mykey == key;  // the lane holding the pivot
      singular |= zero;
      if (zero && zstep < 0) zstep = k;
      if (tt == 0) S.pivrow[k] = best;
      Cx<RL>* rb = rb0 + (k & 1) * (2 * NP + 1);
      // column k: the multipliers, then e_best in place
#pragma unroll
      for (int i = 0; i < RW; ++i) {
        st_shared_if(rb + NP + rg + 8 * i, w[i][u], own);
        if (own) w[i][u] = rg + 8 * i == best ? cx<RL>(1, 0) : cx<RL>(0, 0);
      }
      // row best: slot best / 8 of the four lanes with rg = best % 8
      const bool prow = rg == (best & 7);
#pragma unroll
      for (int i = 0; i < RW; ++i)
#pragma unroll
        for (int c = 0; c < CW; ++c) st_shared_if(rb + CW * cg + c, w[i][c], prow && (best >> 3) == i);
      // the pivot row's own multiplier is zero; its step and reciprocal are kept
      st_shared_if(rb + NP + best, cx<RL>(0, 0), plane);
      st_shared_if(rcrow + best, zero ? cx<RL>(0, 0) : rc, plane);
      if (plane) stepof[best] = k;
      Cx<RL> rp;
      const int src = ((best & 7) << 2) | kc;
      rp.x = __shfl_sync(0xffffffffu, rc.x, src);
      rp.y = __shfl_sync(0xffffffffu, rc.y, src);
      team_sync<32>(team);
      if (zero) rp = cx<RL>(0, 0);
      used |= prow ? 1u << (best >> 3) : 0u;
      Cx<RL> pv[CW];
#pragma unroll
      for (int c = 0; c < CW; ++c) pv[c] = rb[CW * cg + c];
#pragma unroll
      for (int i = 0; i < RW; ++i) {
        const Cx<RL> fp = rb[NP + rg + 8 * i] * rp;
#pragma unroll
        for (int c = 0; c < CW; ++c) cfms(w[i][c], fp, pv[c]);
      }
    }
  }
  team_sync<32>(team);
  int mystep[RW];
  Cx<RL> myrc[RW];
#pragma unroll
  for (int i = 0; i < RW; ++i) {
    mystep[i] = stepof[rg + 8 * i];
    myrc[i] = rcrow[rg + 8 * i];
  }
  team_sync<32>(team);  // the scratch is read before G overwrites it
  if (singular && live && tt == 0)
    record_status(p.status, QCL_SINGULAR,
                  ((long long)e + (long long)NE * m) * kSingularPivotSpan + (scale_ok ? zstep + 1 : 0));
  // inverse(D/s)[step][pivrow[k']] = w[k'] / pivot(step);  GR = that / s
#pragma unroll
  for (int i = 0; i < RW; ++i) {
    const Cx<RL> rs = inv_s * myrc[i];
#pragma unroll
    for (int c = 0; c < CW; ++c) {
      const int col = S.pivrow[CW * cg + c];
      Cx<RL> g = rs * w[i][c];
      if (mystep[i] >= N || col >= N) g = cx<RL>(0, 0);
      G[sw<NP>(mystep[i], col)] = cvt<RS>(g);
    }
  }
  if (tt == 0 && live && p.scale) p.scale[(size_t)e + (size_t)NE * m] = s;
}

// RS: storage precision, RL: inversion precision, RM: product precision.
template <typename RS, typename RL, typename RM, int NP, int BPC>
__global__ void __launch_bounds__(BPC* Tile<NP>::TT, (dyson_min_ctas<RS, RL, NP, BPC>()))
    dyson_keldysh_kernel(DysonArgs<RS> p) {
  constexpr int CPR = Tile<NP>::CPR, TT = Tile<NP>::TT, COLS = NP / CPR;
  constexpr int U = GjUnroll<NP>::U, GROUPS = COLS / U;
  static_assert(COLS % U == 0, "group width must divide the row chunk");
  constexpr size_t MSZ = (size_t)NP * NP;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  Cx<RS>* bufX = reinterpret_cast<Cx<RS>*>(smem_raw);  // BPC tiles: Sigma^R, then Sigma^<,> and products
  Cx<RS>* bufG = bufX + BPC * MSZ;                    // BPC tiles: pivot rows, then G^R
  DysonScratch<TT>* scr = reinterpret_cast<DysonScratch<TT>*>(bufG + BPC * MSZ);

  const int N = p.N, NE = p.NE, Nk = p.Nk;
  const int m = p.m0 + blockIdx.y;
  const int e0 = blockIdx.x * BPC;
  const int team = threadIdx.x / TT;
  const int tt = threadIdx.x % TT;
  const int e = e0 + team;
  const bool live = e < NE;
  Cx<RS>* X = bufX + team * MSZ;
  Cx<RS>* G = bufG + team * MSZ;
  Cx<RL>* rowbuf = reinterpret_cast<Cx<RL>*>(G);  // 2 x (NP + 1): row chunks + pivot reciprocal
  DysonScratch<TT>& S = scr[team];
  const Cx<RS>* first_sig = p.sigL ? p.sigL : p.sigG;
  const bool first_is_L = p.sigL != nullptr;

  // ---- stage SigmaR (all copies in flight at once) ---------------------------
  load_blocks_async<RS, NP, BPC>(p.sigR, bufX, MSZ, e0, m, NE, Nk, N);
  cp_async_wait_all();
  __syncthreads();

  // two-dimensional ownership at N_b <= 24 (one row per lane leaves 8 of 32 lanes idle)
  if constexpr (NP == 24) {
    dyson_gj_2d24<RS, RL, BPC>(p, X, G, S, bufX, team, tt, e, e0, m, live, first_sig, first_is_L);
  } else {
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
        const Cx<RS> sv = X[sw<NP>(row, col)];
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
    __syncthreads();  // every team has read its SigmaR tile: bufX is free
    // prefetch the first Keldysh input while the inversion runs
    if (first_sig && (first_is_L ? p.GL : p.GG)) load_blocks_async<RS, NP, BPC>(first_sig, bufX, MSZ, e0, m, NE, Nk, N);

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

    // ---- register-resident Gauss-Jordan, implicit pivoting, deferred scaling ----
    // Step k picks the pivot row p among the unused rows (largest |Re|+|Im| in
    // column k), every other row i does  w_i[k] = 0;  w_i -= (w_i[k] / w_p[k]) w_p
    // with w_p[k] replaced by 1, and row p is left unscaled (its column-k entry
    // becomes 1).  A row that was pivot at step k is then 1 / w_p[k] times the
    // row of the standard in-place inverse, and it stays that multiple under the
    // later (linear) updates, so the division by the pivot is applied once per
    // row at the end instead of to the whole pivot row at every step.
    bool used = !has_row;
    bool singular = !scale_ok;
    int zstep = -1;  // first step without a non-zero pivot (the k of SingularException(k) is zstep + 1)
    int mystep = row;
    Cx<RL> myrc = cx<RL>(1, 0);
    const int lane = threadIdx.x & 31;
    const int srclane = lane - chunk;  // first lane of this row's chunk group
  #pragma unroll 1
    for (int kc = 0; kc < CPR; ++kc) {
  #pragma unroll 1
      for (int grp = 0; grp < GROUPS; ++grp) {
  #pragma unroll
        for (int u = 0; u < U; ++u) {
          // Steps k >= N (padding) pick the identity rows and change nothing.
          const int k = kc * COLS + grp * U + u;
          const Cx<RL> wk = w[u];  // column k in the lanes of chunk kc (rotated chunk)
          const bool cand = !used && chunk == kc;
          const Cx<RL> rc = crecip_pivot(wk);  // speculative, off the argmax path
          unsigned key = cand ? pivot_key(cabs1(wk), row) : 0u;
          key = __reduce_max_sync(0xffffffffu, key);
          if (TT > 32) {
            if (lane == 0) S.wkey[(k & 1) * (TT / 32) + (tt >> 5)] = key;
            team_sync<TT>(team);
  #pragma unroll
            for (int q = 0; q < TT / 32; ++q) key = max(key, S.wkey[(k & 1) * (TT / 32) + q]);
          }
          const int best = 63 - (int)(key & 63u);
          const bool zero = pivot_key_zero(key);
          singular |= zero;
          if (zero && zstep < 0) zstep = k;
          if (tt == 0) S.pivrow[k] = best;
          Cx<RL> f = wk;
          if (CPR > 1) {
            f.x = __shfl_sync(0xffffffffu, wk.x, srclane + kc);
            f.y = __shfl_sync(0xffffffffu, wk.y, srclane + kc);
          }
          const bool is_pivot = row == best;
          if (chunk == kc) w[u] = is_pivot ? cx<RL>(1, 0) : cx<RL>(0, 0);
          Cx<RL>* rb = rowbuf + (k & 1) * (NP + 1);
  #pragma unroll
          for (int j = 0; j < COLS; ++j) st_shared_if(rb + chunk * COLS + j, w[j], is_pivot);
          Cx<RL> rp;
          if (TT == 32) {
            const int plane = (best * CPR + kc) & 31;
            rp.x = __shfl_sync(0xffffffffu, rc.x, plane);
            rp.y = __shfl_sync(0xffffffffu, rc.y, plane);
            team_sync<TT>(team);
          } else {
            st_shared_if(rb + NP, rc, is_pivot && chunk == kc);
            team_sync<TT>(team);
            rp = rb[NP];
          }
          if (zero) rp = cx<RL>(0, 0);
          used |= is_pivot;
          mystep = is_pivot ? k : mystep;
          myrc = is_pivot ? rp : myrc;
          const Cx<RL> fp = is_pivot ? cx<RL>(0, 0) : f * rp;
  #pragma unroll
          for (int j = 0; j < COLS; ++j) cfms(w[j], fp, rb[chunk * COLS + j]);
        }
        if (GROUPS > 1) {  // rotate the chunk so that the next group is at w[0..U)
          Cx<RL> t[U];
  #pragma unroll
          for (int j = 0; j < U; ++j) t[j] = w[j];
  #pragma unroll
          for (int j = 0; j < COLS - U; ++j) w[j] = w[j + U];
  #pragma unroll
          for (int j = 0; j < U; ++j) w[COLS - U + j] = t[j];
        }
      }
    }
    team_sync<TT>(team);
    // where = block * 64 + k: k = 0 for a zero or non-finite row-sum scale, else the 1-based first zero
    // pivot (LAPACK getrf's info), as SingularException(k) in production_operators.jl:39, 94, 1372
    if (singular && live && tt == 0)
      record_status(p.status, QCL_SINGULAR,
                    ((long long)e + (long long)NE * m) * kSingularPivotSpan + (scale_ok ? zstep + 1 : 0));
    // inverse(D/s)[step][pivrow[k']] = w[k'] / pivot(step);  GR = that / s
    if (has_row) {
      const Cx<RL> rs = inv_s * myrc;
  #pragma unroll
      for (int j = 0; j < COLS; ++j) {
        const int kp = chunk * COLS + j;
        const int col = S.pivrow[kp];
        Cx<RL> g = rs * w[j];
        if (mystep >= N || col >= N) g = cx<RL>(0, 0);
        G[sw<NP>(mystep, col)] = cvt<RS>(g);
      }
    }
    if (tt == 0 && live && p.scale) p.scale[(size_t)e + (size_t)NE * m] = s;
  }
  __syncthreads();
  if (p.GR) store_blocks<RS, RS, NP, BPC>(p.GR, bufG, MSZ, e0, m, NE, Nk, N);

  // ---- Keldysh products: X = G (X G^H), product tiles in registers ----------
  bool prefetched = first_sig && (first_is_L ? p.GL : p.GG);
  for (int which = 0; which < 2; ++which) {
    const Cx<RS>* sig = which == 0 ? p.sigL : p.sigG;
    Cx<RS>* out = which == 0 ? p.GL : p.GG;
    Cx<double>* tr = which == 0 ? p.traceL : p.traceG;
    if (sig == nullptr || out == nullptr) continue;  // uniform
    if (!prefetched) {
      __syncthreads();  // previous store out of bufX is complete
      load_blocks_async<RS, NP, BPC>(sig, bufX, MSZ, e0, m, NE, Nk, N);
    }
    prefetched = false;
    cp_async_wait_all();
    __syncthreads();
    // complex128: the products on the FP64 tensor path (DMMA): 3.3x fewer
    // issued instructions for the products; measured 4.07 -> 4.00 ms at
    // N_b = 24 and 32.6 -> 29.3 ms at N_b = 48 on the operator batch.
    if constexpr (sizeof(RS) == 8 && sizeof(RM) == 8) {
      // three real DMMAs per complex tile product up to N_b = 32; at 48 the
      // third accumulator set spills
      DmmaTile<NP, TT> acc;
      if constexpr (NP <= 32) {
        team_matmul_dmma3<NP, TT>(G, X, acc, N, tt, false);  // T = G Sigma
      } else {
        team_matmul_dmma<NP, TT>(G, X, acc, N, tt, false);
      }
      team_sync<TT>(team);
      team_store_dmma<NP, TT>(X, acc, tt);
      team_sync<TT>(team);
      if constexpr (NP <= 32) {
        team_matmul_dmma3<NP, TT>(X, G, acc, N, tt, true);  // T G^H
      } else {
        team_matmul_dmma<NP, TT>(X, G, acc, N, tt, true);
      }
      team_sync<TT>(team);
      team_store_dmma<NP, TT>(X, acc, tt);
      team_sync<TT>(team);
    } else {
      MatTile<RM, NP> acc;
      team_matmul_regs<RS, RM, NP>(G, X, acc, N, tt, false);  // T = G Sigma
      team_sync<TT>(team);
      team_store_regs<RS, RM, NP>(X, acc, tt);
      team_sync<TT>(team);
      team_matmul_regs<RS, RM, NP>(X, G, acc, N, tt, true);  // T G^H
      team_sync<TT>(team);
      team_store_regs<RS, RM, NP>(X, acc, tt);
      team_sync<TT>(team);
    }
    if (tr) {
      double re = 0, im = 0;
      if (tt < N) {
        const Cx<RS> d = X[sw<NP>(tt, tt)];
        re = d.x;
        im = d.y;
      }
      re = team_sum<TT>(re, tt, S.red, team);
      im = team_sum<TT>(im, tt, S.red, team);
      if (tt == 0 && live) tr[(size_t)e + (size_t)NE * m] = cx<double>(re, im);
    }
    __syncthreads();
    store_blocks<RS, RS, NP, BPC>(out, bufX, MSZ, e0, m, NE, Nk, N);
  }
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

// ---------------------------------------------------------------------------
// CTA shape: blocks per CTA (BPC).  Each padded size has a few compiled
// candidates (the search space of the autotuner, autotune_dyson in
// autotune.cu); the default is the measured choice of the operator batch,
// and a tuned choice per (precision, padded size) replaces it once the
// autotuner has run.
// ---------------------------------------------------------------------------
static int np_index(int NP) { return NP == 8 ? 0 : NP == 16 ? 1 : NP == 24 ? 2 : NP == 32 ? 3 : NP == 48 ? 4 : -1; }
static int prec_index(int precision) { return precision == QCL_C128 ? 0 : precision == QCL_MIXED ? 1 : 2; }
static int g_tuned_bpc[3][5] = {};  // 0: not tuned
static std::mutex g_tune_mutex;

int dyson_bpc_candidates(int NP, int* out) {
  static const int c8[] = {8, 16, 32}, c16[] = {2, 4, 8}, c24[] = {1, 2, 4}, c32[] = {1, 2}, c48[] = {1, 2};
  const int* c = nullptr;
  int n = 0;
  switch (NP) {
    case 8: c = c8; n = 3; break;
    case 16: c = c16; n = 3; break;
    case 24: c = c24; n = 3; break;
    case 32: c = c32; n = 2; break;
    case 48: c = c48; n = 2; break;
    default: return 0;
  }
  for (int i = 0; i < n; ++i) out[i] = c[i];
  return n;
}

int dyson_default_bpc(int precision, int NP) {
  const bool wide = precision == QCL_C128;  // FP64 storage: half the blocks per CTA
  switch (NP) {
    case 8: return 16;
    case 16: return wide ? 4 : 8;
    case 24: return 4;  // complex128: 3.80 ms against 4.09 ms with 2 on the 4096 x 32 batch
    case 32: return wide ? 1 : 2;
    case 48: return 1;
    default: return 0;
  }
}

int dyson_bpc(int precision, int NP) {
  std::lock_guard<std::mutex> lock(g_tune_mutex);
  const int i = np_index(NP);
  if (i < 0) return 0;
  const int t = g_tuned_bpc[prec_index(precision)][i];
  return t ? t : dyson_default_bpc(precision, NP);
}

void dyson_set_bpc(int precision, int NP, int bpc) {
  std::lock_guard<std::mutex> lock(g_tune_mutex);
  const int i = np_index(NP);
  if (i >= 0) g_tuned_bpc[prec_index(precision)][i] = bpc;
}

template <typename RS, typename RL, typename RM, int NP>
static int launch_dyson_np(const DysonArgs<RS>& a, int bpc, cudaStream_t st) {
  if constexpr (NP == 8) {
    if (bpc == 8) return launch_dyson_t<RS, RL, RM, 8, 8>(a, st);
    if (bpc == 32) return launch_dyson_t<RS, RL, RM, 8, 32>(a, st);
    return launch_dyson_t<RS, RL, RM, 8, 16>(a, st);
  } else if constexpr (NP == 16) {
    if (bpc == 2) return launch_dyson_t<RS, RL, RM, 16, 2>(a, st);
    if (bpc == 8) return launch_dyson_t<RS, RL, RM, 16, 8>(a, st);
    return launch_dyson_t<RS, RL, RM, 16, 4>(a, st);
  } else if constexpr (NP == 24) {
    if (bpc == 1) return launch_dyson_t<RS, RL, RM, 24, 1>(a, st);
    if (bpc == 4) return launch_dyson_t<RS, RL, RM, 24, 4>(a, st);
    return launch_dyson_t<RS, RL, RM, 24, 2>(a, st);
  } else if constexpr (NP == 32) {
    if (bpc == 2) return launch_dyson_t<RS, RL, RM, 32, 2>(a, st);
    return launch_dyson_t<RS, RL, RM, 32, 1>(a, st);
  } else {
    if (bpc == 2) return launch_dyson_t<RS, RL, RM, 48, 2>(a, st);
    return launch_dyson_t<RS, RL, RM, 48, 1>(a, st);
  }
}

template <typename RS, typename RL, typename RM>
static int launch_dyson_prec(const DysonArgs<RS>& a, int precision, int bpc_override, cudaStream_t st) {
  const int NP = padded_size(a.N);
  const int bpc = bpc_override > 0 ? bpc_override : dyson_bpc(precision, NP);
  switch (NP) {
    case 8: return launch_dyson_np<RS, RL, RM, 8>(a, bpc, st);
    case 16: return launch_dyson_np<RS, RL, RM, 16>(a, bpc, st);
    case 24: return launch_dyson_np<RS, RL, RM, 24>(a, bpc, st);
    case 32: return launch_dyson_np<RS, RL, RM, 32>(a, bpc, st);
    case 48: return launch_dyson_np<RS, RL, RM, 48>(a, bpc, st);
    default:
      set_last_error("basis size N_b=%d exceeds the supported maximum 48", a.N);
      return QCL_UNSUPPORTED;
  }
}

int launch_dyson_keldysh(int precision, int NE, int Nk, int N, const double* eps, double eta, const void* h,
                         const void* sigR, const void* sigL, const void* sigG, void* GR, void* GL, void* GG,
                         double* scale, void* traceL, void* traceG, int* status, cudaStream_t st, int m0,
                         int mcount) {
  return launch_dyson_keldysh_bpc(precision, NE, Nk, N, eps, eta, h, sigR, sigL, sigG, GR, GL, GG, scale, traceL,
                                  traceG, status, st, m0, mcount, 0);
}

int launch_dyson_keldysh_bpc(int precision, int NE, int Nk, int N, const double* eps, double eta, const void* h,
                             const void* sigR, const void* sigL, const void* sigG, void* GR, void* GL, void* GG,
                             double* scale, void* traceL, void* traceG, int* status, cudaStream_t st, int m0,
                             int mcount, int bpc) {
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
    return launch_dyson_prec<double, double, double>(a, precision, bpc, st);
  }
  DysonArgs<float> a{NE, Nk, N, m0, eps, eta, (const Cx<double>*)h, (const Cx<float>*)sigR,
                     (const Cx<float>*)sigL, (const Cx<float>*)sigG, (Cx<float>*)GR, (Cx<float>*)GL,
                     (Cx<float>*)GG, scale, (Cx<double>*)traceL, (Cx<double>*)traceG, status, mcount};
  if (precision == QCL_MIXED) return launch_dyson_prec<float, double, float>(a, precision, bpc, st);
  if (precision == QCL_C64) return launch_dyson_prec<float, float, float>(a, precision, bpc, st);
  set_last_error("unknown precision %d", precision);
  return QCL_ARG;
}

}  // namespace qcl
