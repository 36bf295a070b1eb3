// Dense self-energy contraction on the 5th-generation tensor cores (complex64
// fields; the mixed and c64 precisions).
//
// Reference: _production_static_contraction! for a dense operator
// (numerics/optimized/production_operators.jl:402-465):
//   S[e,(m,a,b)] = beta S + alpha q sum_(m',c,d) M[(m,a,b),(m',c,d)] wk[m'] G[e,(m',c,d)].
//
// The complex product is one real GEMM.  With k = (m',c,d), j = (m,a,b) and
// interleaved real indices kk = 2k + {0: Re, 1: Im}, nn = 2j + {0, 1}:
//   A[e][kk]  = G[e,k] parts                       (M = N_E rows, K-contiguous)
//   B[nn][kk] = wk * [[Re M, -Im M], [Im M, Re M]]  (built once per operator)
//   S[e,j] = alpha q (C[e][2j] + i C[e][2j+1]) + beta S[e,j],  C = A B^T.
//
// Operands: FP16 pairs.  Each row of A is scaled by a power of two s_e so
// that its largest entry lies in [2^13, 2^14), B by one power of two s_B, and
// every value is split into x = hi + lo with hi = fp16(x), lo = fp16(x - hi)
// (11 + 11 significant bits, as TF32 hi/lo).  C accumulates A_hi B_hi +
// A_hi B_lo + A_lo B_hi in FP32 (relative error ~3 * 2^-22 per product; a
// value below 2^-28 of its row maximum keeps an absolute error under 2^-38
// of it) and the epilogue divides by s_e s_B (exact).  Against TF32 hi/lo the
// operands are half the bytes and the MMA rate is twice as high.
//
// Kernel: CTAs of 320 threads over 128 x BN output tiles (BN = 256 or 224),
// 1 CTA per SM: one tile per CTA, or, for a short K, persistent CTAs that
// walk several tiles so that one tile's epilogue overlaps the next tile's
// loads and MMAs.  K advances in blocks of 32 (one 64-byte swizzle row per
// operand row).  Warp 8 streams the blocks with TMA into a 4-stage ring of
// 64B-swizzled K-major tiles; warp 9 issues the 3 x 2 tcgen05.mma (M = 128,
// N = BN, K = 16, kind::f16) of a block into one of two tensor-memory
// accumulators (128 lanes x BN FP32 columns each).
//
// Accumulation: the tensor core's FP32 accumulation truncates (measured: a
// relative bias of about -0.17 ulp per accumulate).  So every second K block
// starts a fresh accumulator, and while the tensor core fills one buffer the
// 8 drain warps read the other (tcgen05.ld, warp w: lanes 32 (w % 4) .. + 31,
// columns BN/2 (w / 4) .. ) and add it to per-thread FP32 running sums with
// IEEE rounding; an mbarrier (256 arrivals) hands the buffer back.  Each
// truncated chain is then 12 MMAs long.
// Every wait is bounded: a wait that gives up records QCL_TIMEOUT, the CTA
// then waits (bounded) for its own MMAs, releases its tensor memory and ends.
#include <cuda.h>  // CUtensorMap (the encoder is reached through cudaGetDriverEntryPoint)
#include <cuda_fp16.h>

#include <algorithm>
#include <mutex>

#include "kernels.cuh"

namespace qcl {

constexpr int TC_BM = 128, TC_BN = 256, TC_BK = 32;  // TC_BN: the widest tile (operand padding); TC_BK fp16
constexpr int TC_STAGES = 4;      // operand stages: the producer runs up to 3 blocks ahead
constexpr int TC_ACC_KB = 2;      // K blocks per tensor-memory accumulation (12 MMAs)
constexpr int TC_DRAIN_WARPS = 8; // warps that read accumulators out and write the tile
constexpr int TC_THREADS = 32 * (TC_DRAIN_WARPS + 2);  // + producer warp + MMA warp
constexpr int TC_A_BYTES = TC_BM * TC_BK * 2;   // 8 KiB per A part
constexpr int TC_BAR_BYTES = 128;
constexpr uint32_t TC_TMEM_COLS = 512;  // two accumulators of up to 256 columns
// Per tile width BN (the N of one MMA): B part bytes, stage bytes, shared memory.
template <int BN> struct TcShape {
  static constexpr int B_BYTES = BN * TC_BK * 2;
  static constexpr int STAGE_BYTES = 2 * TC_A_BYTES + 2 * B_BYTES;
  static constexpr int SMEM_BYTES = TC_STAGES * STAGE_BYTES + 1024 + TC_BAR_BYTES;
  static constexpr int CH = BN / 2;                   // accumulator columns per drain warp
  static constexpr int LDW = CH % 32 == 0 ? 32 : 16;  // tensor-memory load width
};
constexpr long long TC_WAIT_LIMIT = 1ll << 22;  // try_wait rounds (~1 s) before a wait gives up
// Rounds of the main-loop waits (producer, MMA issuer, accumulator drain).  The
// waits after a failure (in-flight copies and MMAs) always use TC_WAIT_LIMIT.
// qcl_debug_set_wait_limit lowers it so that a test can take the timeout path.
__device__ long long g_tc_main_wait_limit = TC_WAIT_LIMIT;

// UMMA shared-memory descriptor, K-major, 64-byte swizzle (the layout TMA
// writes with CU_TENSOR_MAP_SWIZZLE_64B): start address (>> 4), leading byte
// offset 1 (unused for swizzled K-major), stride byte offset 512 B between
// 8-row groups (>> 4), descriptor version 1, swizzle mode 4 (64B).
__device__ __forceinline__ uint64_t umma_desc_k_sw64(uint32_t saddr) {
  return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)1 << 16) | ((uint64_t)32 << 32) | ((uint64_t)1 << 46) |
         ((uint64_t)4 << 61);
}
// Instruction descriptor (kind::f16): D f32, A/B f16, both K-major, N = BN, M = 128.
template <int BN> __device__ __forceinline__ constexpr uint32_t tc_idesc() {
  return (1u << 4) | (0u << 7) | (0u << 10) | ((uint32_t)(BN >> 3) << 17) | ((uint32_t)(TC_BM >> 4) << 24);
}

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint32_t bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}
// Bounded parity wait; returns false if it gave up.
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity, long long limit = TC_WAIT_LIMIT) {
  for (long long i = 0; i < limit; ++i) {
    uint32_t done;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
        : "=r"(done)
        : "r"(bar), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
}

// 2D tiled TMA load (no multicast) of the box at (x = K offset, y = row).
__device__ __forceinline__ void tma_load(uint32_t dst, const CUtensorMap* map, int x, int y, uint32_t bar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::
          "r"(dst),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(bar)
      : "memory");
}

__device__ __forceinline__ void tc_mma(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                       uint32_t accumulate) {
  asm volatile(
      "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
      " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n}" ::"r"(tmem_d),
      "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate), "r"(0), "r"(0), "r"(0), "r"(0)
      : "memory");
}
__device__ __forceinline__ void tc_commit(uint32_t bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar) : "memory");
}

// Reads 16 consecutive accumulator columns of this thread's lane.
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, uint32_t (&v)[16]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
      : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]), "=r"(v[8]),
        "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15])
      : "r"(taddr));
}
// Reads 32 consecutive accumulator columns of this thread's lane.
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, uint32_t (&v)[32]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
      "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
      : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]), "=r"(v[8]),
        "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15]), "=r"(v[16]),
        "=r"(v[17]), "=r"(v[18]), "=r"(v[19]), "=r"(v[20]), "=r"(v[21]), "=r"(v[22]), "=r"(v[23]), "=r"(v[24]),
        "=r"(v[25]), "=r"(v[26]), "=r"(v[27]), "=r"(v[28]), "=r"(v[29]), "=r"(v[30]), "=r"(v[31])
      : "r"(taddr));
}

struct TcMaps {  // TMA descriptors of the four operand parts (K-contiguous rows)
  CUtensorMap ahi, alo, bhi, blo;
};

struct TcArgs {
  int M;        // rows of C actually stored (N_E)
  int Ncols;    // real columns of C actually stored (2 Nc)
  int Kpad;     // padded real K (multiple of TC_BK)
  Cx<float>* S; // element (row e, complex column j) at the output index below
  int NE;
  double alpha, beta;
  const float* ainv;  // 1 / s_e per row of A
  const float* binv;  // 1 / s_B (device scalar)
  int* status;
  // output index (e mod oP) + oP (j mod oQ) + oP oQ (e / oP) + oP oQ oR (j / oQ);
  // oP = M and oQ larger than every j give the plain column-major e + M j
  long long oP, oQ, oR;
  // linear tile order: 0 = row tiles fastest (the CTAs in flight share B
  // tiles), 1 = column tiles fastest (they share A tiles, so an A larger than
  // L2 is read once)
  int cols_fastest;
  int mtiles;  // row tiles (M padded to TC_BM)
};

// The column part of the output index, walked j, j + 1, ... with j mod oQ and
// j / oQ carried instead of divided per element (the row part is one per thread).
struct TcColWalk {
  long long r, q, step_r, step_q, oQ;
  __device__ __forceinline__ TcColWalk(const TcArgs& p, long long j0)
      : r(j0 % p.oQ), q(j0 / p.oQ), step_r(p.oP), step_q(p.oP * p.oQ * p.oR), oQ(p.oQ) {}
  __device__ __forceinline__ long long offset() const { return step_r * r + step_q * q; }
  __device__ __forceinline__ void next() {
    if (++r == oQ) {
      r = 0;
      ++q;
    }
  }
};

// Warp roles: warps 0-7 read accumulators out (warp w: tensor-memory lanes
// 32 (w % 4) .. + 31, columns 128 (w / 4) .. + 127) into FP32 running sums and
// write the tile; warp 8 lane 0 streams the operand blocks with TMA; warp 9
// lane 0 issues the MMAs (warp 9 also owns the tensor-memory allocation).
// Hand-offs are mbarriers only: full[s] (TMA bytes), empty[s] (MMAs done
// reading stage s), acc_full[b] (accumulation in buffer b done), acc_empty[b]
// (256 readers done with buffer b).
// PERSIST: the CTA walks several tiles (short K); otherwise exactly one
// (blockIdx.x), and the tile loops fold away at compile time.
template <int BN, bool PERSIST>
__global__ void __launch_bounds__(TC_THREADS, 1) tc_gemm_kernel(const __grid_constant__ TcMaps maps, TcArgs p) {
  using S = TcShape<BN>;
  constexpr int TC_STAGE_BYTES = S::STAGE_BYTES, TC_B_BYTES = S::B_BYTES;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const uint32_t raw = smem_u32(smem_raw);
  const uint32_t base = (raw + 1023u) & ~1023u;  // 1024-byte aligned stages
  unsigned char* gbase = smem_raw + (base - raw);
  const uint32_t bars = base + TC_STAGES * TC_STAGE_BYTES;
  const uint32_t full = bars, empty = bars + 8 * TC_STAGES, acc_full = bars + 16 * TC_STAGES, acc_empty = acc_full + 16;
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(gbase + TC_STAGES * TC_STAGE_BYTES + 16 * TC_STAGES + 32);
  __shared__ volatile int s_fail;

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  // this CTA's tiles are blockIdx.x + i gridDim.x (i < ntile) in the linear
  // tile order (one tile when the grid covers them all; several when it is
  // persistent); its K blocks and accumulation groups are counted
  // across its tiles, so the ring stages, the two accumulators and their
  // barrier phases run on from one tile to the next, and the epilogue of a
  // tile overlaps the loads and MMAs of the next
  const int nkb = p.Kpad / TC_BK;  // K blocks per tile
  const int nch = (nkb + TC_ACC_KB - 1) / TC_ACC_KB;  // accumulation groups per tile
  const int ntiles_n = (p.Ncols + BN - 1) / BN;
  const long long tiles = (long long)p.mtiles * ntiles_n;
  const int ntile = !PERSIST ? 1 : blockIdx.x < tiles ? (int)((tiles - 1 - blockIdx.x) / gridDim.x + 1) : 0;
  const int mtiles = p.mtiles, cols_fastest = p.cols_fastest;
  const auto tile_origin = [mtiles, ntiles_n, cols_fastest](int i, int& m0, int& n0) {
    const int t = (int)blockIdx.x + i * (int)gridDim.x;  // tiles < 2^31
    m0 = (cols_fastest ? t / ntiles_n : t % mtiles) * TC_BM;
    n0 = (cols_fastest ? t % ntiles_n : t / mtiles) * BN;
  };
  const long long lim = g_tc_main_wait_limit;
  if (threadIdx.x == 0) {
    for (int i = 0; i < TC_STAGES; ++i) {
      mbar_init(full + 8 * i, 1);
      mbar_init(empty + 8 * i, 1);
    }
    for (int i = 0; i < 2; ++i) {
      mbar_init(acc_full + 8 * i, 1);
      mbar_init(acc_empty + 8 * i, 32 * TC_DRAIN_WARPS);
    }
    s_fail = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == TC_DRAIN_WARPS + 1) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                 "r"(TC_TMEM_COLS)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = *tmem_slot;
  int issued = 0;  // MMA warp: blocks whose MMAs were issued and committed
  int loaded = 0;  // producer: blocks whose TMA copies were issued

  if (warp == TC_DRAIN_WARPS) {
    // ---- producer ---------------------------------------------------------
    if (lane == 0) {
      for (int kb = 0; kb < ntile * nkb && !s_fail; ++kb) {  // kb: this CTA's K blocks over its tiles
        const int s = kb % TC_STAGES, kt = PERSIST ? kb % nkb : kb;
        int m0, n0;
        tile_origin(PERSIST ? kb / nkb : 0, m0, n0);
        if (kb >= TC_STAGES && !mbar_wait(empty + 8 * s, (uint32_t)((kb / TC_STAGES - 1) & 1), lim)) {
          s_fail = 1;
          break;
        }
        loaded = kb + 1;
        const uint32_t st = base + s * TC_STAGE_BYTES;
        mbar_expect_tx(full + 8 * s, TC_STAGE_BYTES);
        tma_load(st, &maps.ahi, kt * TC_BK, m0, full + 8 * s);
        tma_load(st + TC_A_BYTES, &maps.alo, kt * TC_BK, m0, full + 8 * s);
        tma_load(st + 2 * TC_A_BYTES, &maps.bhi, kt * TC_BK, n0, full + 8 * s);
        tma_load(st + 2 * TC_A_BYTES + TC_B_BYTES, &maps.blo, kt * TC_BK, n0, full + 8 * s);
      }
    }
  } else if (warp == TC_DRAIN_WARPS + 1) {
    // ---- MMA issue --------------------------------------------------------
    if (lane == 0) {
      for (int kb = 0; kb < ntile * nkb && !s_fail; ++kb) {
        // group ch counts this CTA's accumulation groups over its tiles
        const int kt = PERSIST ? kb % nkb : kb, s = kb % TC_STAGES;
        const int ch = (PERSIST ? (kb / nkb) * nch : 0) + kt / TC_ACC_KB, b = ch & 1;
        const bool first = kt % TC_ACC_KB == 0, last = (kt % TC_ACC_KB == TC_ACC_KB - 1) || kt == nkb - 1;
        if (!mbar_wait(full + 8 * s, (uint32_t)((kb / TC_STAGES) & 1), lim) ||
            (first && ch >= 2 && !mbar_wait(acc_empty + 8 * b, (uint32_t)(((ch - 2) >> 1) & 1), lim))) {
          s_fail = 1;
          break;
        }
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        const uint32_t st = base + s * TC_STAGE_BYTES;
        const uint32_t tAh = st, tAl = st + TC_A_BYTES, tBh = st + 2 * TC_A_BYTES, tBl = tBh + TC_B_BYTES;
        const uint32_t dacc = tmem + (uint32_t)(b * BN);
        constexpr uint32_t idesc = tc_idesc<BN>();
#pragma unroll
        for (int ks = 0; ks < TC_BK / 16; ++ks) {  // K = 16 fp16 = 32 bytes per MMA
          const uint32_t off = ks * 32;
          const uint64_t ah = umma_desc_k_sw64(tAh + off), al = umma_desc_k_sw64(tAl + off);
          const uint64_t bh = umma_desc_k_sw64(tBh + off), bl = umma_desc_k_sw64(tBl + off);
          tc_mma(dacc, ah, bh, idesc, (first && ks == 0) ? 0u : 1u);
          tc_mma(dacc, ah, bl, idesc, 1u);
          tc_mma(dacc, al, bh, idesc, 1u);
        }
        tc_commit(empty + 8 * s);
        if (last) tc_commit(acc_full + 8 * b);
        issued = kb + 1;
      }
      // the tensor memory is released below: let every issued MMA finish (bounded)
      if (issued > 0) {
        const int kl = issued - 1;
        mbar_wait(empty + 8 * (kl % TC_STAGES), (uint32_t)((kl / TC_STAGES) & 1));
      }
    }
  } else {
    // ---- accumulator read-out and epilogue --------------------------------
    constexpr int CH = S::CH, LDW = S::LDW;
    const uint32_t tlane = (uint32_t)((warp & 3) * 32) << 16;
    const int cbase = (warp >> 2) * CH;
    bool ok = true;
    for (int it = 0; it < ntile && ok; ++it) {
    int m0, n0;
    tile_origin(it, m0, n0);
    float sum[CH];
#pragma unroll
    for (int i = 0; i < CH; ++i) sum[i] = 0.0f;
    for (int cl = 0; cl < nch; ++cl) {
      const int ch = it * nch + cl, b = ch & 1;
      // warp-uniform decision: the tensor-memory loads below are .sync.aligned
      const bool stop = __any_sync(0xffffffffu, s_fail != 0);
      const bool got = __all_sync(0xffffffffu, !stop && mbar_wait(acc_full + 8 * b, (uint32_t)((ch >> 1) & 1), lim));
      if (!got) {
        ok = false;
        s_fail = 1;
        break;
      }
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      const uint32_t taddr = tmem + tlane + (uint32_t)(b * BN + cbase);
      // up to 64 columns in flight per wait (2 waits per buffer instead of CH / LDW)
      constexpr int NL = CH / LDW, GL = 64 / LDW;
#pragma unroll
      for (int c0 = 0; c0 < NL; c0 += GL) {
        uint32_t v[GL][LDW];
#pragma unroll
        for (int g = 0; g < GL; ++g) {
          if (c0 + g < NL) {
            if constexpr (LDW == 32) tmem_ld32(taddr + (c0 + g) * 32, v[g]);
            else tmem_ld16(taddr + (c0 + g) * 16, v[g]);
          }
        }
        asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
        for (int g = 0; g < GL; ++g) {
          if (c0 + g < NL) {
#pragma unroll
            for (int i = 0; i < LDW; ++i) sum[(c0 + g) * LDW + i] += __uint_as_float(v[g][i]);
          }
        }
      }
      asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
      mbar_arrive(acc_empty + 8 * b);
    }
    const int e = m0 + (warp & 3) * 32 + lane;
    if (ok && e < p.M) {
      // undo the operand scales (powers of two) and apply alpha in FP64, so that
      // no intermediate under- or overflows: one rounding to FP32, as before
      const double al = p.alpha * (double)p.ainv[e] * (double)__ldg(p.binv);
      const float be = (float)p.beta;
      Cx<float>* row = p.S + ((e % p.oP) + p.oP * p.oQ * (e / p.oP));
      TcColWalk col(p, (n0 + cbase) >> 1);  // n0 and cbase are even
#pragma unroll
      for (int q = 0; q < CH / 2; ++q, col.next()) {
        const int nn = n0 + cbase + 2 * q;
        if (nn >= p.Ncols) continue;
        Cx<float>* dst = row + col.offset();
        const float re = (float)(al * (double)sum[2 * q]), im = (float)(al * (double)sum[2 * q + 1]);
        if (p.beta == 0.0) {
          *dst = cx<float>(re, im);
        } else {
          const Cx<float> o = *dst;
          *dst = cx<float>(be * o.x + re, be * o.y + im);
        }
      }
    }
    }  // tiles
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (threadIdx.x == 0 && s_fail) record_status(p.status, QCL_TIMEOUT, (long long)blockIdx.x);
  if (warp == TC_DRAIN_WARPS + 1)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TC_TMEM_COLS) : "memory");
  // After a failure (s_fail is final past the barrier above) copies may still be
  // in flight into this CTA's shared memory: the producer waits (full limit) for
  // the last TC_STAGES loads, one per stage at its latest phase, before the CTA
  // ends (a phase the MMA warp already consumed has completed: its wait returns
  // at once).  Without a failure every load was consumed by an MMA.
  if (warp == TC_DRAIN_WARPS && lane == 0 && s_fail)
    for (int kl = loaded > TC_STAGES ? loaded - TC_STAGES : 0; kl < loaded; ++kl)
      mbar_wait(full + 8 * (kl % TC_STAGES), (uint32_t)((kl / TC_STAGES) & 1));
}

// ---------------------------------------------------------------------------
// Operand preparation
// ---------------------------------------------------------------------------
// Power-of-two scale that takes a largest magnitude mx into [2^13, 2^14)
// (1 for zero or non-finite mx; the exponent is clamped to keep the scale and
// its inverse normal FP32 numbers).
__device__ __forceinline__ float tc_scale_for(float mx) {
  if (!(mx > 0.0f) || !isfinite(mx)) return 1.0f;
  int ex;
  frexpf(mx, &ex);  // mx = f 2^ex, f in [0.5, 1)
  const int sh = min(max(14 - ex, -120), 120);
  return ldexpf(1.0f, sh);
}
// x = hi + lo in FP16 (x already scaled); x - hi is exact in FP32.
__device__ __forceinline__ void split_f16(float x, __half& hi, __half& lo) {
  hi = __float2half_rn(x);
  lo = __float2half_rn(x - __half2float(hi));
}

// Row maxima of A: max_kk |A[e][kk]| into rowmax[e] as FP32 bits (non-negative
// values order as unsigned integers; a non-finite entry gives +inf), which
// the caller zeroes first.  A CTA covers 32 rows x 256 values of k (coalesced
// along e); the atomic maximum is independent of the order.
// Rows of A address G at (e mod P) + P k + Bs (e / P): P = NE, Bs = 0 is the
// plain column-major matrix; P = N_E, Bs = N_E N_k reads a field with rows
// (e, (c,d)) and columns m' (the first stage of a separable-sum contraction).
__global__ void tc_row_max_kernel(int NE, int Nc, long long P, long long Bs, const Cx<float>* __restrict__ G,
                                  unsigned* __restrict__ rowmax) {
  __shared__ float red[8][32];
  const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;  // 32 x 8 threads
  const int e = blockIdx.x * 32 + tx;
  const int k0 = blockIdx.y * 256, k1 = min(Nc, k0 + 256);
  float mx = 0.0f;
  if (e < NE)
    for (int k = k0 + ty; k < k1; k += 8) {
      const Cx<float> g = G[(size_t)(e % P) + (size_t)P * k + (size_t)Bs * (size_t)(e / P)];
      const float a = fmaxf(fabsf(g.x), fabsf(g.y));
      mx = (isfinite(g.x) && isfinite(g.y)) ? fmaxf(mx, a) : INFINITY;
    }
  red[ty][tx] = mx;
  __syncthreads();
  if (ty == 0 && e < NE) {
    for (int q = 1; q < 8; ++q) mx = fmaxf(mx, red[q][tx]);
    atomicMax(rowmax + e, __float_as_uint(mx));
  }
}

// A[e][2k + c] = s_e * part c of G[e + NE k] for k < Nc (zero in the padding),
// split into fp16 hi / lo, s_e from the row maximum (rows past N_E: 1); the
// CTAs of the first K slice also write ainv[e] = 1 / s_e.  A CTA owns 32 rows
// and walks K in tiles of 64 complex columns (128 real), gridDim.y tiles
// apart: each complex value is read once (coalesced along e), the tile is
// transposed through shared memory, and each row's 128 values are written as
// half2 pairs (coalesced along K).
constexpr int TC_SPLIT_KK = 128;
__global__ void tc_split_a_kernel(int NE, int Nc, int Mpad, int Kpad, long long P, long long Bs,
                                  const Cx<float>* __restrict__ G,
                                  const unsigned* __restrict__ rowmax, __half* __restrict__ Ahi,
                                  __half* __restrict__ Alo, float* __restrict__ ainv) {
  __shared__ float tile[TC_SPLIT_KK][33];
  const int e0 = blockIdx.x * 32;
  const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;  // 32 x 8 threads
  const int er = e0 + tx;  // this thread's row in the read phase
  const bool rin = er < NE;
  const float sc = rin ? tc_scale_for(__uint_as_float(rowmax[er])) : 1.0f;
  if (blockIdx.y == 0 && ty == 0 && er < Mpad) ainv[er] = 1.0f / sc;
  const size_t rowbase = rin ? (size_t)(er % P) + (size_t)Bs * (size_t)(er / P) : 0;
  for (int kk0 = blockIdx.y * TC_SPLIT_KK; kk0 < Kpad; kk0 += gridDim.y * TC_SPLIT_KK) {
#pragma unroll
    for (int q = 0; q < TC_SPLIT_KK / 16; ++q) {
      const int kl = ty + 8 * q;  // complex column within the tile
      const int k = (kk0 >> 1) + kl;
      Cx<float> g = cx<float>(0.0f, 0.0f);
      if (rin && k < Nc) g = G[rowbase + (size_t)P * k];
      tile[2 * kl][tx] = g.x * sc;
      tile[2 * kl + 1][tx] = g.y * sc;
    }
    __syncthreads();
    for (int r = ty; r < 32; r += 8) {
      const int e = e0 + r;
      if (e >= Mpad) continue;  // warp-uniform
#pragma unroll
      for (int h = tx; h < TC_SPLIT_KK / 2; h += 32) {
        const int kk = kk0 + 2 * h;  // even, and Kpad is even
        if (kk >= Kpad) continue;
        __half h0, l0, h1, l1;
        split_f16(tile[2 * h][r], h0, l0);
        split_f16(tile[2 * h + 1][r], h1, l1);
        const size_t idx = (size_t)e * Kpad + kk;
        *reinterpret_cast<__half2*>(Ahi + idx) = __halves2half2(h0, h1);
        *reinterpret_cast<__half2*>(Alo + idx) = __halves2half2(l0, l1);
      }
    }
    __syncthreads();
  }
}

// max |B| into *mxbits (non-negative FP32 bits order as unsigned integers;
// a non-finite entry gives +inf).  Mop is column-major Nout x Kc; column k
// carries the weight wk[k % Nk] (no weight if wk is NULL).
__global__ void tc_b_maxabs_kernel(int Nout, int Kc, int Nk, const Cx<float>* __restrict__ Mop,
                                   const double* __restrict__ wk, unsigned* __restrict__ mxbits) {
  const long long n = (long long)Nout * Kc;
  float mx = 0.0f;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const Cx<float> m = Mop[i];
    const float w = wk ? fabsf((float)wk[(i / Nout) % Nk]) : 1.0f;
    const float a = fmaxf(fabsf(m.x), fabsf(m.y)) * w;
    mx = isfinite(a) ? fmaxf(mx, a) : INFINITY;
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) mx = fmaxf(mx, __shfl_xor_sync(0xffffffffu, mx, o));
  if ((threadIdx.x & 31) == 0) atomicMax(mxbits, __float_as_uint(mx));
}
// B[2j + c'][2k + c] from the complex operator M (column-major Nout x Kc,
// complex64) and the momentum weights wk[k % Nk] (1 if wk is NULL):
//   s_B [[Re, -Im], [Im, Re]] * w  (rows c' = 0 real part of the output, 1 imaginary),
// as fp16 hi / lo.  One CTA per 32 (j) x 16 (k) tile of M: M is read
// coalesced along j into shared memory, B written coalesced along its K axis
// (each M entry feeds a 2 x 2 block of B; the padding past Nout / Kc is zero).
__global__ void tc_build_b_kernel(int Nout, int Kc, int Nk, int Kpad, const Cx<float>* __restrict__ Mop,
                                  const double* __restrict__ wk, const unsigned* __restrict__ mxbits,
                                  __half* __restrict__ Bhi, __half* __restrict__ Blo, float* __restrict__ binv) {
  __shared__ Cx<float> tile[16][33];  // [k][j]
  const float sc = tc_scale_for(__uint_as_float(*mxbits));
  if (blockIdx.x == 0 && blockIdx.y == 0 && threadIdx.x == 0) *binv = 1.0f / sc;
  const int j0 = blockIdx.x * 32, k0 = blockIdx.y * 16;
  const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;  // 32 x 8 threads
  for (int r = ty; r < 16; r += 8) {
    const int j = j0 + tx, k = k0 + r;
    tile[r][tx] = (j < Nout && k < Kc) ? Mop[(size_t)j + (size_t)Nout * k] : cx<float>(0, 0);
  }
  __syncthreads();
  // 64 rows x 32 columns of B: thread column kk = 2 k0 + tx, rows in steps of 8
  const int kk = 2 * k0 + tx, kl = tx >> 1, c = tx & 1, k = k0 + kl;
  const float w = k < Kc ? (wk ? (float)wk[k % Nk] : 1.0f) : 0.0f;
  for (int rr = ty; rr < 64; rr += 8) {
    const int nn = 2 * j0 + rr, jl = rr >> 1, cp = rr & 1;
    const Cx<float> m = tile[kl][jl];
    const float val = (cp == c) ? m.x : (cp == 0 ? -m.y : m.y);
    const size_t i = (size_t)nn * Kpad + kk;
    split_f16(sc * (w * val), Bhi[i], Blo[i]);
  }
}

// Padded extents of a C[M x Nout] = A[M x Kc] B^T product (complex counts;
// real extents twice that), in whole tiles.
static void tc_dims2(int M, int Nout, int Kc, int* Mpad, int* Npad, int* Kpad) {
  *Mpad = (M + TC_BM - 1) / TC_BM * TC_BM;
  *Npad = (2 * Nout + TC_BN - 1) / TC_BN * TC_BN;
  *Kpad = (2 * Kc + TC_BK - 1) / TC_BK * TC_BK;
}
int tc_dims(int NE, int Nc, int* Mpad, int* Npad, int* Kpad) {
  tc_dims2(NE, Nc, Nc, Mpad, Npad, Kpad);
  return QCL_OK;
}

// A work area, in floats: fp16 hi and lo (Mpad x Kpad each), then the row
// maxima (FP32 bits) and the inverse row scales (Mpad each).
size_t tc_a_work_floats2(int M, int Kc) {
  int Mpad, Npad, Kpad;
  tc_dims2(M, 1, Kc, &Mpad, &Npad, &Kpad);
  return (size_t)Mpad * Kpad + 2 * (size_t)Mpad;
}
size_t tc_a_work_floats(int NE, int Nc) { return tc_a_work_floats2(NE, Nc); }

// Prepared operator: one allocation holding 1 / s_B (256 bytes reserved), the
// max-|B| word, then B_hi and B_lo (Npad x Kpad fp16 each).  *Bop receives it.
// Mop is column-major Nout x Kc (complex64); wk (may be NULL) weights column
// k by wk[k % Nk].
int tc_build_operator2(int Nout, int Kc, int Nk, const void* Mop_c64, const double* wk, void** Bop, cudaStream_t st) {
  int Mpad, Npad, Kpad;
  tc_dims2(1, Nout, Kc, &Mpad, &Npad, &Kpad);
  const size_t n = (size_t)Npad * Kpad;
  QCL_CUDA_CHECK(cudaMalloc(Bop, 256 + 2 * n * sizeof(__half)));
  char* b = (char*)*Bop;
  float* binv = (float*)b;
  unsigned* mxbits = (unsigned*)(b + 16);
  __half* Bhi = (__half*)(b + 256);
  QCL_CUDA_CHECK(cudaMemsetAsync(mxbits, 0, sizeof(unsigned), st));
  tc_b_maxabs_kernel<<<148 * 4, 256, 0, st>>>(Nout, Kc, Nk, (const Cx<float>*)Mop_c64, wk, mxbits);
  QCL_LAUNCH_CHECK("tc_b_maxabs_kernel");
  tc_build_b_kernel<<<dim3(Npad / 64, Kpad / 32), 256, 0, st>>>(Nout, Kc, Nk, Kpad, (const Cx<float>*)Mop_c64, wk,
                                                                 mxbits, Bhi, Bhi + n, binv);
  QCL_LAUNCH_CHECK("tc_build_b_kernel");
  return QCL_OK;
}
// Bytes of a prepared operand (tc_build_operator2).
size_t tc_operator_bytes(int Nout, int Kc) {
  int Mpad, Npad, Kpad;
  tc_dims2(1, Nout, Kc, &Mpad, &Npad, &Kpad);
  return 256 + 2 * (size_t)Npad * Kpad * sizeof(__half);
}
int tc_build_operator(int Nc, int Nk, const void* Mop_c64, const double* wk, void** Bop, cudaStream_t st) {
  return tc_build_operator2(Nc, Nc, Nk, Mop_c64, wk, Bop, st);
}

typedef CUresult (*TensorMapEncodeTiled)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                          const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                          CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

static TensorMapEncodeTiled tensor_map_encoder() {
  static TensorMapEncodeTiled fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void* f = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &f, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = (TensorMapEncodeTiled)f;
  });
  return fn;
}

// K-contiguous FP16 matrix [rows][Kpad] in boxes of TC_BK x box_rows, 64B swizzle.
static int make_operand_map(CUtensorMap* m, const __half* ptr, int rows, int Kpad, int box_rows) {
  TensorMapEncodeTiled enc = tensor_map_encoder();
  if (!enc) {
    set_last_error("cuTensorMapEncodeTiled is not available from the driver");
    return QCL_CUDA;
  }
  const cuuint64_t dims[2] = {(cuuint64_t)Kpad, (cuuint64_t)rows};
  const cuuint64_t strides[1] = {(cuuint64_t)Kpad * sizeof(__half)};
  const cuuint32_t box[2] = {(cuuint32_t)TC_BK, (cuuint32_t)box_rows};
  const cuuint32_t es[2] = {1, 1};
  const CUresult r = enc(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT16, 2, (void*)ptr, dims, strides, box, es,
                         CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_64B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                         CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) {
    set_last_error("cuTensorMapEncodeTiled failed (%d) for a %d x %d operand", (int)r, rows, Kpad);
    return QCL_CUDA;
  }
  return QCL_OK;
}

// Tile width for an output of Ncols real columns: of 256 and 224 the one
// whose tiles fill the most of their waves over the 148 SMs (one CTA per SM),
// weighted by the share of the last tile that is padding; ties go to the
// wider tile (fewer operand bytes per flop).  (192-wide tiles spill the drain
// registers.)
static int tc_pick_bn(int mtiles, int Ncols) {
  const int cand[2] = {256, 224};
  int best = 256;
  double best_eff = -1;
  for (int bn : cand) {
    const int nt = (Ncols + bn - 1) / bn;
    const long long tiles = (long long)mtiles * nt;
    const long long waves = (tiles + 147) / 148;
    const double eff = (double)tiles / (double)(waves * 148) * ((double)Ncols / ((double)nt * bn));
    if (eff > best_eff + 1e-9) {
      best_eff = eff;
      best = bn;
    }
  }
  return best;
}

template <int BN> static int launch_tc_t(const TcMaps& maps, const TcArgs& a, int mtiles, cudaStream_t st) {
  static bool configured = false;
  if (!configured) {
    QCL_CUDA_CHECK(cudaFuncSetAttribute(tc_gemm_kernel<BN, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        TcShape<BN>::SMEM_BYTES));
    QCL_CUDA_CHECK(cudaFuncSetAttribute(tc_gemm_kernel<BN, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        TcShape<BN>::SMEM_BYTES));
    configured = true;
  }
  TcArgs b = a;
  b.mtiles = mtiles;
  const long long tiles = (long long)mtiles * ((a.Ncols + BN - 1) / BN);
  int sms = 148;
  int dev = 0;
  if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  // Short K (a few blocks per tile, the momentum-mixing stage of a separable
  // sum): one persistent CTA per SM, so that a tile's epilogue overlaps the
  // next tile's loads and MMAs (1.41 -> 1.21 ms on the 524 288 x 1024 x 128
  // case).  Long K: one CTA per tile, which the hardware schedules as SMs
  // free up (the persistent form measured 10 % slower there: 5.23 -> 5.78 ms
  // on the 32 768 x 2048 x 16 384 case).
  const bool persistent = b.Kpad / TC_BK <= 8;
  const long long grid = persistent ? std::min<long long>(tiles, sms) : tiles;
  if (persistent)
    tc_gemm_kernel<BN, true><<<(unsigned)grid, TC_THREADS, TcShape<BN>::SMEM_BYTES, st>>>(maps, b);
  else
    tc_gemm_kernel<BN, false><<<(unsigned)grid, TC_THREADS, TcShape<BN>::SMEM_BYTES, st>>>(maps, b);
  QCL_LAUNCH_CHECK("tc_gemm_kernel");
  return QCL_OK;
}

// C = A B^T on the tensor cores for complex64 operands:
//   S[e + M j] = alpha sum_k A[e + M k] Bop[j, k] + beta S[e + M j],
// e < M, j < Nout, k < Kc; Bop prepared by tc_build_operator2(Nout, Kc, ...).
int launch_tc_contraction2(int M, int Nout, int Kc, const void* Bop, const void* A, void* S, double alpha,
                           double beta, float* awork, int* status, cudaStream_t st) {
  int s = tc_split_rows(M, Kc, A, M, 0, awork, st);
  if (s) return s;
  return launch_tc_presplit(M, Nout, Kc, Bop, awork, S, M, 1ll << 40, 0, alpha, beta, status, st);
}

// The FP16 hi / lo split of A (rows addressed as in tc_row_max_kernel) into
// awork: hi, lo (Mpad x Kpad each), row maxima, inverse row scales.
int tc_split_rows(int M, int Kc, const void* A, long long P, long long Bs, float* awork, cudaStream_t st) {
  int Mpad, Npad, Kpad;
  tc_dims2(M, 1, Kc, &Mpad, &Npad, &Kpad);
  __half* Ahi = (__half*)awork;
  __half* Alo = Ahi + (size_t)Mpad * Kpad;
  unsigned* rowmax = (unsigned*)(Alo + (size_t)Mpad * Kpad);
  float* ainv = (float*)(rowmax + Mpad);
  QCL_CUDA_CHECK(cudaMemsetAsync(rowmax, 0, (size_t)Mpad * sizeof(unsigned), st));
  tc_row_max_kernel<<<dim3(Mpad / 32, (Kc + 255) / 256), 256, 0, st>>>(M, Kc, P, Bs, (const Cx<float>*)A, rowmax);
  QCL_LAUNCH_CHECK("tc_row_max_kernel");
  dim3 sg((Mpad + 31) / 32, std::min((Kpad + TC_SPLIT_KK - 1) / TC_SPLIT_KK, 32));
  tc_split_a_kernel<<<sg, 256, 0, st>>>(M, Kc, Mpad, Kpad, P, Bs, (const Cx<float>*)A, rowmax, Ahi, Alo, ainv);
  QCL_LAUNCH_CHECK("tc_split_a_kernel");
  return QCL_OK;
}

// The product of an A already split into awork (tc_split_rows with the same
// M, Kc) and a prepared operand; the output index is (e mod oP) + oP (j mod oQ)
// + oP oQ (e / oP) + oP oQ oR (j / oQ) (see TcArgs).
int launch_tc_presplit(int M, int Nout, int Kc, const void* Bop, const float* awork, void* S, long long oP,
                       long long oQ, long long oR, double alpha, double beta, int* status, cudaStream_t st) {
  int Mpad, Npad, Kpad;
  tc_dims2(M, Nout, Kc, &Mpad, &Npad, &Kpad);
  const __half* Ahi = (const __half*)awork;
  const __half* Alo = Ahi + (size_t)Mpad * Kpad;
  const float* ainv = (const float*)((const unsigned*)(Alo + (size_t)Mpad * Kpad) + Mpad);
  const char* b = (const char*)Bop;
  const __half* Bhi = (const __half*)(b + 256);
  const __half* Blo = Bhi + (size_t)Npad * Kpad;
  const int mtiles = Mpad / TC_BM;
  const int bn = tc_pick_bn(mtiles, 2 * Nout);
  TcMaps maps;
  int s;
  if ((s = make_operand_map(&maps.ahi, Ahi, Mpad, Kpad, TC_BM))) return s;
  if ((s = make_operand_map(&maps.alo, Alo, Mpad, Kpad, TC_BM))) return s;
  // B rows past Npad (the last tile of a narrower width) read the zero fill
  if ((s = make_operand_map(&maps.bhi, Bhi, Npad, Kpad, bn))) return s;
  if ((s = make_operand_map(&maps.blo, Blo, Npad, Kpad, bn))) return s;
  // the larger operand is read once: A larger than B (and than L2) streams
  // with the column tiles fastest, else B does with the row tiles fastest
  const int cols_fastest = (size_t)Mpad > (size_t)Npad && (size_t)Mpad * Kpad * 4 > (size_t)(96u << 20);
  TcArgs a{M, 2 * Nout, Kpad, (Cx<float>*)S, M, alpha, beta, ainv, (const float*)b, status, oP, oQ, oR, cols_fastest};
  if (bn == 224) return launch_tc_t<224>(maps, a, mtiles, st);
  return launch_tc_t<256>(maps, a, mtiles, st);
}

// Sets the main-loop wait limit of the tensor-core kernels on the current
// device (rounds of mbarrier.try_wait; 0 makes every main-loop wait give up at
// once; a negative value restores the default).
int tc_set_wait_limit(long long rounds) {
  const long long v = rounds >= 0 ? rounds : TC_WAIT_LIMIT;
  QCL_CUDA_CHECK(cudaMemcpyToSymbol(g_tc_main_wait_limit, &v, sizeof(v)));
  return QCL_OK;
}

int launch_tc_dense_contraction(int NE, int Nc, const void* Bop, const void* G, void* S, double alpha, double beta,
                                float* awork, int* status, cudaStream_t st) {
  return launch_tc_contraction2(NE, Nc, Nc, Bop, G, S, alpha, beta, awork, status, st);
}

}  // namespace qcl
