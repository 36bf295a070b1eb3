// Zero-padded linear-convolution Hilbert transform, fused with the retarded
// self-energy assembly.
//
// Reference: _fft_hilbert_with_length / fft_hilbert_transform
// (numerics/optimized/production_operators.jl:735-809) and
// ProductionFFTHilbertPlan (numerics/optimized/fft_parallel.jl:27-291):
//   kernel[lag + NE - 1] = 1 / (2 pi lag de), 0 < |lag| < NE, zero elsewhere
//   buffer = wE .* Gam padded to L = nextpow2(2 NE - 1)
//   Lam_e = IFFT(FFT(buffer) .* FFT(kernel))[e + NE - 1]
// and _retarded_self_energy_fft_production (:842-884):
//   Gam = i (S> - S<),  SR = Lam - i Gam / 2.
//
// B200 mapping: one CTA per column (m, a, b).  The padded column lives in
// shared memory, the two FFTs are Stockham passes (radix 16 after a first
// pass of radix L / 16^P) with the butterflies in registers, the last forward
// pass, the spectrum product and the first inverse pass run as one register
// pass, the kernel spectrum is read from L2 (from shared memory in the
// half-length form, whose centred kernel has a real, odd spectrum: a quarter
// of the table), and the inputs are read once and
// the outputs written once (E is the contiguous axis, so every load/store is
// coalesced).  The complex128 L = 8192 transform runs as two half-length
// transforms (even / odd frequencies) in a 68 KiB buffer, so that two columns
// share an SM (hilbert_halves_kernel).
//
// Roundoff verification (fft_parallel.jl:279-290 runs a second transform at
// length 2L).  Because the input is zero beyond N_E <= L/2 + 1 and only
// outputs below L are used, the length-2L convolution splits exactly into the
// length-L convolution (even frequencies; its kernel spectrum folds to the
// length-L one) plus one twisted length-L convolution (odd frequencies):
//   y_2L[n] = (y_L[n] + W_2L^{-n} IFFT_L(FFT_L(x W_2L^n) .* K2L_odd)[n]) / 2.
// So verification costs two extra length-L FFTs instead of two length-2L
// ones, and the same per-column partial sums of |y_2L - y_L|^2 and |y_L|^2.

#include <math.h>

#include <algorithm>
#include <vector>

#include "kernels.cuh"

namespace qcl {

__device__ __forceinline__ int fpad(int p) { return p + (p >> 4); }

// Read-only (non-coherent cache) loads of the constant tables.
__device__ __forceinline__ Cx<double> ldg_cx(const Cx<double>* p) {
  const double2 v = __ldg(reinterpret_cast<const double2*>(p));
  return cx<double>(v.x, v.y);
}
__device__ __forceinline__ Cx<float> ldg_cx(const Cx<float>* p) {
  const float2 v = __ldg(reinterpret_cast<const float2*>(p));
  return cx<float>(v.x, v.y);
}

// W_16^t = exp(-2 pi i t / 16); multiply z by W_16^t (t compile-time).
template <typename R, int t> __device__ __forceinline__ Cx<R> w16mul(Cx<R> z) {
  constexpr int u = t & 15;
  if (u == 0) return z;
  if (u == 4) return cx<R>(z.y, -z.x);
  if (u == 8) return cx<R>(-z.x, -z.y);
  if (u == 12) return cx<R>(-z.y, z.x);
  const R c1 = (R)0.92387953251128674, s1 = (R)0.38268343236508978, c2 = (R)0.70710678118654752;
  R c, s;  // W = c - i s
  switch (u) {
    case 1: c = c1; s = s1; break;
    case 2: c = c2; s = c2; break;
    case 3: c = s1; s = c1; break;
    case 5: c = -s1; s = c1; break;
    case 6: c = -c2; s = c2; break;
    case 7: c = -c1; s = s1; break;
    case 9: c = -c1; s = -s1; break;
    case 10: c = -c2; s = -c2; break;
    case 11: c = -s1; s = -c1; break;
    case 13: c = s1; s = -c1; break;
    case 14: c = c2; s = -c2; break;
    default: c = c1; s = -s1; break;  // 15
  }
  return cx<R>(z.x * c + z.y * s, z.y * c - z.x * s);
}

// z * W_32^k = z * exp(-2 pi i k / 32), k in [0, 16) (a compile-time value
// once the caller's loop is unrolled): cos and sin of k pi / 16.
template <typename R> __device__ __forceinline__ Cx<R> w32mul(Cx<R> z, int k) {
  const R c1 = (R)0.98078528040323044913, s1 = (R)0.19509032201612826785;
  const R c2 = (R)0.92387953251128675613, s2 = (R)0.38268343236508977173;
  const R c3 = (R)0.83146961230254523708, s3 = (R)0.55557023301960222474;
  const R c4 = (R)0.70710678118654752440;
  R c, s;  // W = c - i s
  switch (k & 15) {
    case 0: return z;
    case 1: c = c1; s = s1; break;
    case 2: c = c2; s = s2; break;
    case 3: c = c3; s = s3; break;
    case 4: c = c4; s = c4; break;
    case 5: c = s3; s = c3; break;
    case 6: c = s2; s = c2; break;
    case 7: c = s1; s = c1; break;
    case 8: return cx<R>(z.y, -z.x);
    case 9: c = -s1; s = c1; break;
    case 10: c = -s2; s = c2; break;
    case 11: c = -s3; s = c3; break;
    case 12: c = -c4; s = c4; break;
    case 13: c = -c3; s = s3; break;
    case 14: c = -c2; s = s2; break;
    default: c = -c1; s = s1; break;  // 15
  }
  return cx<R>(z.x * c + z.y * s, z.y * c - z.x * s);
}

template <int P> __host__ __device__ constexpr int bitrev(int i) {
  int r = 0;
  for (int b = 1; b < P; b <<= 1) {
    r <<= 1;
    if (i & b) r |= 1;
  }
  return r;
}

// In-register forward DFT of size P in {2,4,8,16} (radix-2 DIF); output is
// left in bit-reversed order: X[i] = v[bitrev<P>(i)].
template <typename R, int P, int H> struct DifStage {
  __device__ __forceinline__ static void run(Cx<R> (&v)[P]) {
#pragma unroll
    for (int start = 0; start < P; start += 2 * H) {
#pragma unroll
      for (int k = 0; k < H; ++k) {
        Cx<R> a = v[start + k], b = v[start + k + H];
        v[start + k] = a + b;
        Cx<R> d = a - b;
        // W_{2H}^k = W_16^{k * 8 / H}
        switch ((k * 8 / H) & 15) {
          case 0: v[start + k + H] = d; break;
          case 1: v[start + k + H] = w16mul<R, 1>(d); break;
          case 2: v[start + k + H] = w16mul<R, 2>(d); break;
          case 3: v[start + k + H] = w16mul<R, 3>(d); break;
          case 4: v[start + k + H] = w16mul<R, 4>(d); break;
          case 5: v[start + k + H] = w16mul<R, 5>(d); break;
          case 6: v[start + k + H] = w16mul<R, 6>(d); break;
          default: v[start + k + H] = w16mul<R, 7>(d); break;
        }
      }
    }
    DifStage<R, P, H / 2>::run(v);
  }
};
template <typename R, int P> struct DifStage<R, P, 0> {
  __device__ __forceinline__ static void run(Cx<R> (&)[P]) {}
};

template <int L> struct FftPlan {
  static constexpr int T = (L / 16 >= 32) ? L / 16 : 32;
};

// Pass adaptors: a pass reads its inputs through In(i) and writes its outputs
// through Out(t, v), so that the first pass can read the field from global
// memory and the last pass can multiply by the kernel spectrum or write the
// result straight to global memory, without extra shared-memory sweeps.
template <typename R> struct SmemIn {
  static constexpr bool kShared = true;
  static constexpr bool kBatch = false;
  const Cx<R>* buf;
  __device__ __forceinline__ Cx<R> operator()(int i) const { return buf[fpad(i)]; }
};
template <typename R> struct SmemOut {
  static constexpr bool kBatch = false;
  Cx<R>* buf;
  __device__ __forceinline__ void operator()(int t, Cx<R> v) const { buf[fpad(t)] = v; }
};
// v * W_{2H}^k for compile-time k (H a power of two, 2H <= 16).
template <typename R, int H, int k> __device__ __forceinline__ Cx<R> w2h_mul(Cx<R> d) {
  switch ((k * 8 / H) & 15) {
    case 0: return d;
    case 1: return w16mul<R, 1>(d);
    case 2: return w16mul<R, 2>(d);
    case 3: return w16mul<R, 3>(d);
    case 4: return w16mul<R, 4>(d);
    case 5: return w16mul<R, 5>(d);
    case 6: return w16mul<R, 6>(d);
    default: return w16mul<R, 7>(d);
  }
}
template <typename R, int H, int K> struct ZeroHiStage {
  // first DIF stage when v[H..2H) are zero: v[k] stays, v[k + H] = v[k] W_{2H}^k
  __device__ __forceinline__ static void run(Cx<R>* v) {
    v[K - 1 + H] = w2h_mul<R, H, K - 1>(v[K - 1]);
    ZeroHiStage<R, H, K - 1>::run(v);
  }
};
template <typename R, int H> struct ZeroHiStage<R, H, 0> {
  __device__ __forceinline__ static void run(Cx<R>*) {}
};

// Twiddles of a pass (radix RADIX, stride NS): v[r] *= W_L^{k c r}, r = 1 ..
// RADIX-1, k = j mod NS, c = L / (NS RADIX).
// complex128: w_1 = W_L^{k c} from the length-L table and its powers by binary
// powering (products of at most four factors, so the twiddle error stays a
// few ulps).  complex64: every power read from the pass's own table seg[(r-1)
// NS + k] (correctly rounded, and contiguous in k so a warp's loads coalesce);
// a few FP32 ulps of twiddle error would otherwise be the largest term of the
// transform error (about twice the table form's).
template <typename R, int L, int RADIX, int NS>
__device__ __forceinline__ Cx<R> first_twiddle(int k, const Cx<R>* __restrict__ tw, const Cx<R>* __restrict__ seg) {
  if constexpr (sizeof(R) == 4) return ldg_cx(seg + k);
  return ldg_cx(tw + k * (L / (NS * RADIX)));
}
template <typename R, int L, int RADIX, int NS>
__device__ __forceinline__ void apply_twiddles(Cx<R>* v, Cx<R> w1, int k, const Cx<R>* __restrict__ seg) {
  if constexpr (sizeof(R) == 4) {
    v[1] = v[1] * w1;
#pragma unroll
    for (int r = 2; r < RADIX; ++r) v[r] = v[r] * ldg_cx(seg + (r - 1) * NS + k);
  } else {
    Cx<R> w[RADIX];
    w[1] = w1;
#pragma unroll
    for (int r = 2; r < RADIX; ++r) {
      const int hi = (r & (r - 1)) ? (r & (r - 1)) : r / 2;  // r = hi + lo, hi >= lo
      w[r] = w[hi] * w[r - hi];
    }
#pragma unroll
    for (int r = 1; r < RADIX; ++r) v[r] = v[r] * w[r];
  }
}

// One mixed-radix Stockham pass (natural-order output after all passes).
// ZHI: the inputs of slots r >= RADIX/2 are known to be zero (the padding).
// tw: W_L^t, t < L; seg: this pass's complex64 twiddle table (null otherwise).
template <typename R, int L, int RADIX, int NS, bool ZHI, typename In, typename Out>
__device__ __forceinline__ void stockham_pass(const In& in, const Out& out, const Cx<R>* __restrict__ tw,
                                              const Cx<R>* __restrict__ seg) {
  const int tid = threadIdx.x;
  constexpr int T = FftPlan<L>::T;
  constexpr int NB = L / RADIX;
  constexpr int Q = (NB + T - 1) / T;
  constexpr int RIN = ZHI ? RADIX / 2 : RADIX;
  static_assert(!ZHI || NS == 1, "pruned inputs only in the first pass");
  // One twiddle-table load per butterfly, issued first (read-only path) so
  // that its latency overlaps the shared-memory reads and the barrier.
  Cx<R> w1[Q];
  if (NS > 1) {
#pragma unroll
    for (int q = 0; q < Q; ++q) {
      const int j = tid + q * T;
      w1[q] = first_twiddle<R, L, RADIX, NS>(j < NB ? j % NS : 0, tw, seg);
    }
  }
  Cx<R> v[Q][RADIX];
#pragma unroll
  for (int q = 0; q < Q; ++q) {
    const int j = tid + q * T;
    if (j < NB) {
      if constexpr (In::kBatch) {
        in.template batch<NB, RIN, RADIX>(j, v[q]);
      } else {
#pragma unroll
        for (int r = 0; r < RIN; ++r) v[q][r] = in(j + r * NB);
      }
    }
  }
  if (In::kShared) __syncthreads();  // in place: every read before any write
#pragma unroll
  for (int q = 0; q < Q; ++q) {
    const int j = tid + q * T;
    if (j < NB) {
      const int k = j % NS;
      if (NS > 1) apply_twiddles<R, L, RADIX, NS>(v[q], w1[q], k, seg);
      if (ZHI) {
        ZeroHiStage<R, RADIX / 2, RADIX / 2>::run(v[q]);
        DifStage<R, RADIX, RADIX / 4>::run(v[q]);
      } else {
        DifStage<R, RADIX, RADIX / 2>::run(v[q]);
      }
      const int idxD = (j / NS) * NS * RADIX + k;
      if constexpr (Out::kBatch) {
        out.template batch<NS, RADIX>(idxD, v[q]);
      } else {
#pragma unroll
        for (int r = 0; r < RADIX; ++r) out(idxD + r * NS, v[q][bitrev<RADIX>(r)]);
      }
    }
  }
  __syncthreads();
}

// Pass plan of the length-L convolution: the forward transform is a first
// pass of radix S = L / 16^P (2 <= S <= 16) followed by P radix-16 passes,
// the inverse runs the same radices in reverse order.  The last forward pass
// (NS = L/16) and the first inverse pass (NS = 1) touch the same indices
// j + r L/16 in the same thread, so they run as one register-resident pass
// with the spectrum product between them (spectrum_pass).
constexpr int conv_passes(int L) {
  int p = 0;
  while (L > 16) {
    L /= 16;
    ++p;
  }
  return p;
}

// complex64 pass tables, in pass order: the forward radix-16 passes (NS = S
// 16^i, i < P; the last is the fused one), the inverse radix-16 passes (NS =
// 16^i, 1 <= i < P), the final radix-S pass (NS = L/S); a pass's table is
// (RADIX - 1) NS entries.  Offsets in entries:
constexpr int conv_fwd_seg(int L, int i) {  // S (16^i - 1)
  const int P = conv_passes(L);
  int off = 0, ns = L >> (4 * P);
  for (int t = 0; t < i; ++t, ns *= 16) off += 15 * ns;
  return off;
}
constexpr int conv_inv_seg(int L, int i) {  // (L - S) + 16^i - 16
  const int P = conv_passes(L);
  int off = L - (L >> (4 * P)), ns = 16;
  for (int t = 1; t < i; ++t, ns *= 16) off += 15 * ns;
  return off;
}
constexpr int conv_table_entries(int L) {  // 2L - S - 16
  return conv_inv_seg(L, conv_passes(L)) + ((L >> (4 * conv_passes(L))) - 1) * (L / (L >> (4 * conv_passes(L))));
}

template <typename R, int L, int NS, int COUNT> struct Radix16Passes {
  __device__ __forceinline__ static void run(Cx<R>* buf, const Cx<R>* tw, const Cx<R>* seg) {
    stockham_pass<R, L, 16, NS, false>(SmemIn<R>{buf}, SmemOut<R>{buf}, tw, seg);
    Radix16Passes<R, L, NS * 16, COUNT - 1>::run(buf, tw, seg ? seg + 15 * NS : nullptr);
  }
};
template <typename R, int L, int NS> struct Radix16Passes<R, L, NS, 0> {
  __device__ __forceinline__ static void run(Cx<R>*, const Cx<R>*, const Cx<R>*) {}
};

// Spectrum product of the spectrum pass, conj(v K[f]) at f = j + r L/16 (r a
// constant after unrolling).  SpecTable reads a full complex spectrum from
// global memory (L2).
template <typename R, int L> struct SpecTable {
  const Cx<R>* K;
  __device__ __forceinline__ void prepare() const {}
  __device__ __forceinline__ Cx<R> operator()(Cx<R> v, int j, int r) const {
    return conj(v * ldg_cx(K + j + r * (L / 16)));
  }
};

// Spectrum of the circularly centred kernel, k[lag mod L] (lag in (-N_E,
// N_E)).  The kernel is real and odd, so its spectrum is purely imaginary,
// K[f] = i S[f] with S real and S[L - f] = -S[f].  In the even / odd
// frequency halves of length LH = L/2, E[f] = S[2f] and O[f] = S[2f+1] obey
// E[LH - f] = -E[f] and O[LH - 1 - f] = -O[f], so the table holds E[0..LH/2]
// and O[0..LH/2): LH + 1 doubles (32 KB at L = 8192) instead of the L complex
// values (128 KB) of the offset kernel's spectrum.  It is staged in shared
// memory once per column (cp.async, waited for before the first spectrum
// product).  Centring moves the wanted outputs from [N_E - 1, 2 N_E - 2] to
// [0, N_E): the same linear convolution, since L >= 2 N_E - 1.
__device__ __forceinline__ void hil_cp_async16(void* smem, const void* gmem) {
  const unsigned a = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(a), "l"(gmem) : "memory");
}
__device__ __forceinline__ void hil_cp_async_wait() {
  asm volatile("cp.async.commit_group;\n\tcp.async.wait_group 0;" ::: "memory");
}
__host__ __device__ constexpr int sym_table_odd_offset(int LH) { return LH / 2 + 2; }  // E padded to a 16-byte multiple
__host__ __device__ constexpr int sym_table_doubles(int LH) { return sym_table_odd_offset(LH) + LH / 2; }
template <int LH, bool ODD> struct SpecSym {
  const double* S;  // shared memory, sym_table_doubles(LH) entries
  __device__ __forceinline__ void prepare() const { hil_cp_async_wait(); }
  __device__ __forceinline__ Cx<double> operator()(Cx<double> v, int j, int r) const {
    constexpr int NB = LH / 16;
    const int f = j + r * NB;
    double s;
    if (!ODD) {
      s = r < 8 ? S[f] : -S[LH - f];  // r >= 8: f >= LH/2
    } else {
      constexpr int o = sym_table_odd_offset(LH);
      s = r < 8 ? S[o + f] : -S[o + LH - 1 - f];
    }
    return cx<double>(-v.y * s, -v.x * s);  // conj(v i s)
  }
};

// Last radix-16 pass of the forward transform, times K and conjugated (so
// that the next forward transform computes the inverse one: IFFT(X) =
// conj(FFT(conj X)) / L), and the first radix-16 pass of that transform.
template <typename R, int L, typename Spec>
__device__ __forceinline__ void spectrum_pass(Cx<R>* buf, const Spec& spec, const Cx<R>* __restrict__ tw,
                                              const Cx<R>* __restrict__ seg) {
  constexpr int T = FftPlan<L>::T;
  constexpr int NB = L / 16;
  constexpr int Q = (NB + T - 1) / T;
  const int tid = threadIdx.x;
  Cx<R> w1[Q];
#pragma unroll
  for (int q = 0; q < Q; ++q) {
    const int j = tid + q * T;
    w1[q] = first_twiddle<R, L, 16, NB>(j < NB ? j : 0, tw, seg);  // NS = L/16: W_L^j
  }
  Cx<R> v[Q][16];
#pragma unroll
  for (int q = 0; q < Q; ++q) {
    const int j = tid + q * T;
    if (j < NB) {
#pragma unroll
      for (int r = 0; r < 16; ++r) v[q][r] = buf[fpad(j + r * NB)];
    }
  }
  spec.prepare();
  __syncthreads();
#pragma unroll
  for (int q = 0; q < Q; ++q) {
    const int j = tid + q * T;
    if (j < NB) {
      apply_twiddles<R, L, 16, NB>(v[q], w1[q], j, seg);
      DifStage<R, 16, 8>::run(v[q]);
      // forward output j + r NB is v[bitrev(r)]; it is input r of the next pass
      Cx<R> u[16];
#pragma unroll
      for (int r = 0; r < 16; ++r) u[r] = spec(v[q][bitrev<16>(r)], j, r);
      DifStage<R, 16, 8>::run(u);
#pragma unroll
      for (int r = 0; r < 16; ++r) buf[fpad(16 * j + r)] = u[bitrev<16>(r)];
    }
  }
  __syncthreads();
}

// Pulls this thread's kernel-spectrum entries of the spectrum pass (K[j + r
// L/16], r < 16) toward L1 ahead of use, without holding registers.  Used in
// complex64, where it took the N_E = 1024 transform from 0.297 to 0.248 ms
// (with verification); complex128 measured no gain.
template <typename R, int L> __device__ __forceinline__ void prefetch_spectrum(const Cx<R>* K) {
  constexpr int T = FftPlan<L>::T, NB = L / 16, Q = (NB + T - 1) / T;
#pragma unroll
  for (int q = 0; q < Q; ++q) {
    const int j = threadIdx.x + q * T;
    if (j < NB) {
#pragma unroll
      for (int r = 0; r < 16; ++r) asm volatile("prefetch.global.L1 [%0];" ::"l"(K + j + r * NB));
    }
  }
}

// conj(L * IFFT(FFT(x) .* K)) for a field read through `in` (ZHI: zero on
// [L/2, L)), written through `out`; `buf` holds the padded column, `twt` the
// complex64 pass tables (null for complex128).
template <typename R, int L, bool ZHI, typename In, typename Spec, typename Out>
__device__ __forceinline__ void convolve_run(const In& in, const Spec& spec, const Out& out, Cx<R>* buf,
                                             const Cx<R>* tw, const Cx<R>* twt) {
  static_assert(L >= 64 && L <= 16384, "unsupported FFT length");
  constexpr int P = conv_passes(L);
  constexpr int S = L >> (4 * P);
  static_assert(S >= 2 && S <= 16, "first-pass radix");
  static_assert(conv_table_entries(L) == 2 * L - S - 16, "pass-table layout");
  const bool t = twt != nullptr;
  stockham_pass<R, L, S, 1, ZHI>(in, SmemOut<R>{buf}, tw, nullptr);
  if constexpr (sizeof(R) == 4) prefetch_spectrum<R, L>(spec.K);
  Radix16Passes<R, L, S, P - 1>::run(buf, tw, t ? twt + conv_fwd_seg(L, 0) : nullptr);
  spectrum_pass<R, L>(buf, spec, tw, t ? twt + conv_fwd_seg(L, P - 1) : nullptr);
  Radix16Passes<R, L, 16, P - 1>::run(buf, tw, t ? twt + conv_inv_seg(L, 1) : nullptr);
  stockham_pass<R, L, S, L / S, false>(SmemIn<R>{buf}, out, tw, t ? twt + conv_inv_seg(L, P) : nullptr);
}

template <typename R> struct HilbertArgs {
  int NE;
  long long ncols;
  const double* wE;
  const Cx<R>* Gam;   // input Gam (if SL == null)
  const Cx<R>* SL;    // fused input: Gam = i (SG - SL)
  const Cx<R>* SG;
  Cx<R>* Lam;         // output Lam (if SR == null)
  Cx<R>* SR;          // fused output: SR = Lam - i Gam / 2
  Cx<R>* GamOut;      // optional copy of Gam
  const Cx<R>* khat;  // FFT_L(kernel), L entries
  const Cx<R>* kodd;  // FFT_2L(kernel)[2k+1], L entries (verification)
  const Cx<R>* tw;    // W_L^t, t < L
  const Cx<R>* twist; // W_2L^n, n < L
  double* partial;    // per column (|y2L - yL|^2, |yL|^2), or null
  double scale_out;   // 1 / L
  const Cx<R>* ksplit;  // [FFT_L(kernel)[2j], j < L/2 | FFT_L(kernel)[2j+1], j < L/2]
  const Cx<R>* twh;     // W_{L/2}^t, t < L/2
  const Cx<R>* twt;     // complex64 pass twiddle tables (null for complex128)
  const double* ksym;   // centred kernel's spectrum / i, symmetric halves (complex128, L = 8192)
};

template <typename R>
__device__ __forceinline__ Cx<R> gamma_at(const HilbertArgs<R>& p, size_t idx) {
  if (p.SL) {
    Cx<R> d = p.SG[idx] - p.SL[idx];
    return cx<R>(-d.y, d.x);  // i * d
  }
  return p.Gam[idx];
}

// x_e = wE_e Gam_e (times the twist W_2L^e for the odd-frequency half), zero
// for e >= N_E; optionally copies Gam out.
template <typename R> struct FieldIn {
  static constexpr bool kShared = false;
  static constexpr bool kBatch = true;
  const HilbertArgs<R>* p;
  size_t base;
  const Cx<R>* twist;  // per-sample phase W_2L^e, or null
  __device__ __forceinline__ Cx<R> operator()(int e) const {
    if (e >= p->NE) return cx<R>(0, 0);
    Cx<R> g = gamma_at(*p, base + e);
    if (twist) {
      g = g * ldg_cx(twist + e);
    } else if (p->GamOut) {
      p->GamOut[base + e] = g;
    }
    return (R)__ldg(p->wE + e) * g;
  }
  // The first pass's inputs e = j + r NB, r < RIN (NB = L / RADIX).  In
  // complex128 the twist W_2L^(j + r NB) = W_2L^j W_(2 RADIX)^r is one table
  // load and a constant per r instead of RIN table loads.
  template <int NB, int RIN, int RADIX> __device__ __forceinline__ void batch(int j, Cx<R>* v) const {
    if (sizeof(R) == 4 || !twist) {
#pragma unroll
      for (int r = 0; r < RIN; ++r) v[r] = (*this)(j + r * NB);
      return;
    }
    static_assert(RADIX <= 16 && 16 % RADIX == 0, "twist constants cover W_32");
    const Cx<R> w0 = ldg_cx(twist + j);
#pragma unroll
    for (int r = 0; r < RIN; ++r) {
      const int e = j + r * NB;
      if (e >= p->NE) {
        v[r] = cx<R>(0, 0);
        continue;
      }
      const Cx<R> g = w32mul(gamma_at(*p, base + e) * w0, r * (16 / RADIX));
      v[r] = (R)__ldg(p->wE + e) * g;
    }
  }
};
// Lam_e = conj(y[e + NE - 1]) / L straight to global memory (or the fused
// SR_e = Lam_e - i Gam_e / 2); outputs outside [NE - 1, 2 NE - 2] are dropped.
template <typename R> struct ResultOut {
  static constexpr bool kBatch = false;
  const HilbertArgs<R>* p;
  size_t base;
  __device__ __forceinline__ void operator()(int t, Cx<R> v) const {
    const int e = t - (p->NE - 1);
    if (e < 0 || e >= p->NE) return;
    const R sc = (R)p->scale_out;
    const Cx<R> lam = cx<R>(sc * v.x, -sc * v.y);
    if (p->SR) {
      const Cx<R> g = gamma_at(*p, base + e);
      p->SR[base + e] = cx<R>(lam.x + (R)0.5 * g.y, lam.y - (R)0.5 * g.x);
    } else {
      p->Lam[base + e] = lam;
    }
  }
};

// Registers are capped (128 per thread for complex128; 64 for complex64, 80
// with verification, which spills at 64) so that the register file holds as
// many CTAs as the shared memory does.
template <typename R, bool VERIFY> constexpr int hilbert_reg_cap() { return sizeof(R) == 8 ? 128 : (VERIFY ? 80 : 64); }
template <typename R, int T, bool VERIFY = false> constexpr int hilbert_min_blocks() {
  return 65536 / (hilbert_reg_cap<R, VERIFY>() * T) < 1 ? 1 : 65536 / (hilbert_reg_cap<R, VERIFY>() * T);
}
// Shared memory of the one-pass kernel: the padded column, plus (with
// verification) the length-L results y_L[e + NE - 1] kept for the comparison.
template <typename R, int L, bool VERIFY> constexpr size_t hilbert_smem_bytes() {
  return (size_t)(L + L / 16 + (VERIFY ? L / 2 : 0)) * sizeof(Cx<R>);
}

template <typename R, int L, bool VERIFY>
__global__ void __launch_bounds__(FftPlan<L>::T, (hilbert_min_blocks<R, FftPlan<L>::T, VERIFY>()))
    hilbert_kernel(HilbertArgs<R> p) {
  constexpr int T = FftPlan<L>::T;
  constexpr int PER = (L / 2 + T - 1) / T;  // outputs per thread (NE <= L/2)
  extern __shared__ __align__(16) unsigned char smem_raw[];
  Cx<R>* buf = reinterpret_cast<Cx<R>*>(smem_raw);
  const long long col = blockIdx.x + (long long)blockIdx.y * gridDim.x;
  if (col >= p.ncols) return;
  const int NE = p.NE;
  const size_t base = (size_t)col * NE;
  const SmemOut<R> so{buf};

  if constexpr (!VERIFY) {
    // results written from registers by the last pass
    convolve_run<R, L, true>(FieldIn<R>{&p, base, nullptr}, SpecTable<R, L>{p.khat}, ResultOut<R>{&p, base}, buf, p.tw, p.twt);
    return;
  }
  convolve_run<R, L, true>(FieldIn<R>{&p, base, nullptr}, SpecTable<R, L>{p.khat}, so, buf, p.tw, p.twt);
  // y_L of this thread's outputs, kept in shared memory (read back by the
  // same thread) instead of registers across the second transform
  Cx<R>* lam = buf + (L + L / 16);
  const R sc = (R)p.scale_out;
#pragma unroll
  for (int q = 0; q < PER; ++q) {
    const int e = threadIdx.x + q * T;
    if (e < NE) lam[e] = sc * conj(buf[fpad(e + NE - 1)]);
  }
  __syncthreads();
  // ---- odd-frequency half of the length-2L transform -------------------------
  convolve_run<R, L, true>(FieldIn<R>{&p, base, p.twist}, SpecTable<R, L>{p.kodd}, so, buf, p.tw, p.twt);
  double dsum = 0, lsum = 0;
#pragma unroll
  for (int q = 0; q < PER; ++q) {
    const int e = threadIdx.x + q * T;
    if (e < NE) {
      const int n = e + NE - 1;
      Cx<R> yo = sc * (conj(buf[fpad(n)]) * conj(p.twist[n]));
      const Cx<R> yl = lam[e];
      // y_2L - y_L = (y_L + yo)/2 - y_L = (yo - y_L)/2
      Cx<R> d = (R)0.5 * (yo - yl);
      dsum += (double)d.x * d.x + (double)d.y * d.y;
      lsum += (double)yl.x * yl.x + (double)yl.y * yl.y;
      if (p.SR) {
        Cx<R> g = gamma_at(p, base + e);
        p.SR[base + e] = cx<R>(yl.x + (R)0.5 * g.y, yl.y - (R)0.5 * g.x);
      } else {
        p.Lam[base + e] = yl;
      }
    }
  }
  // deterministic block reduction
  __shared__ double red[2][T / 32];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    dsum += __shfl_xor_sync(0xffffffffu, dsum, o);
    lsum += __shfl_xor_sync(0xffffffffu, lsum, o);
  }
  if ((threadIdx.x & 31) == 0) {
    red[0][threadIdx.x >> 5] = dsum;
    red[1][threadIdx.x >> 5] = lsum;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double a = 0, b = 0;
    for (int w = 0; w < T / 32; ++w) {
      a += red[0][w];
      b += red[1][w];
    }
    p.partial[2 * col] = a;
    p.partial[2 * col + 1] = b;
  }
}

// ---------------------------------------------------------------------------
// Even/odd frequency halves in sequence (no verification).
//
// The padded field is zero on [L/2, L), so its length-L spectrum splits into
//   X[2j]   = FFT_{L/2}(x)[j],   X[2j+1] = FFT_{L/2}(x W_L^n)[j].
// The kernel is the circularly centred one (SpecSym: K = i S, a real table of
// L/2 + 1 entries in shared memory), whose wanted outputs are y[0, N_E), all
// in the first half (N_E <= L/2).  With Y = X K the length-L inverse
// transform there is
//   y[n] = (ye[n] + W_L^{-n} yo[n]) / L,   0 <= n < L/2,
// ye, yo the unnormalised length-L/2 inverse transforms of Y[2j], Y[2j+1].
// One CTA transforms the even half, parks conj(ye) of the wanted outputs in
// the output array, then transforms the odd half and completes each output
// in the same thread that parked it.  The column buffer is L/2 long, so two
// columns share an SM where one length-L column filled it.  Arithmetic is
// that of the one-pass kernel, minus the zero-pruned radix-2 pass of the
// inverse transform.  The output must not alias the input (the field is read
// again for the odd half).
// ---------------------------------------------------------------------------
// Output slot of padded index t in [0, L/2): e = t for t < N_E, else -1.
template <int LH> __device__ __forceinline__ int half_slot(int t, int NE) { return t < NE ? t : -1; }
template <typename R, int LH> struct ParkOut {
  static constexpr bool kBatch = false;
  const HilbertArgs<R>* p;
  size_t base;
  __device__ __forceinline__ void operator()(int t, Cx<R> v) const {
    const int e = half_slot<LH>(t, p->NE);
    if (e < 0) return;
    (p->SR ? p->SR : p->Lam)[base + e] = v;
  }
};
template <typename R, int LH> struct CompleteOut {
  static constexpr bool kBatch = true;
  const HilbertArgs<R>* p;
  size_t base;
  // d = v W_L^t (L = 2 LH) completes the parked even-half value
  __device__ __forceinline__ void complete(int t, Cx<R> d) const {
    const int NE = p->NE;
    const int e = half_slot<LH>(t, NE);
    if (e < 0) return;
    Cx<R>* dst = p->SR ? p->SR : p->Lam;
    const Cx<R> a = dst[base + e];  // parked by this thread in the even half
    const Cx<R> y = a + d;
    const R sc = (R)p->scale_out;
    const Cx<R> lam = cx<R>(sc * y.x, -sc * y.y);
    if (p->SR) {
      const Cx<R> g = gamma_at(*p, base + e);
      p->SR[base + e] = cx<R>(lam.x + (R)0.5 * g.y, lam.y - (R)0.5 * g.x);
    } else {
      p->Lam[base + e] = lam;
    }
  }
  __device__ __forceinline__ void operator()(int t, Cx<R> v) const { complete(t, v * ldg_cx(p->tw + t)); }
  // The final pass's outputs t = t0 + r NS (t0 < NS = LH / RADIX): in
  // complex128 W_L^t = W_L^t0 W_(2 RADIX)^r, one table load per thread.
  template <int NS, int RADIX> __device__ __forceinline__ void batch(int t0, const Cx<R>* v) const {
    if constexpr (sizeof(R) == 4 || NS * RADIX != LH) {
#pragma unroll
      for (int r = 0; r < RADIX; ++r) (*this)(t0 + r * NS, v[bitrev<RADIX>(r)]);
    } else {
      static_assert(RADIX <= 16 && 16 % RADIX == 0, "phase constants cover W_32");
      const Cx<R> w0 = ldg_cx(p->tw + t0);
#pragma unroll
      for (int r = 0; r < RADIX; ++r) complete(t0 + r * NS, w32mul(v[bitrev<RADIX>(r)] * w0, r * (16 / RADIX)));
    }
  }
};

template <typename R, int LH>
__global__ void __launch_bounds__(FftPlan<LH>::T, (hilbert_min_blocks<R, FftPlan<LH>::T>()))
    hilbert_halves_kernel(HilbertArgs<R> p) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  Cx<R>* buf = reinterpret_cast<Cx<R>*>(smem_raw);
  static_assert(sizeof(R) == 8, "the centred half-length form is complex128 only");
  double* ksh = reinterpret_cast<double*>(buf + (LH + LH / 16));  // sym_table_doubles(LH) entries
  const long long col = blockIdx.x + (long long)blockIdx.y * gridDim.x;
  if (col >= p.ncols) return;
  // stage the spectrum table (waited for in the first spectrum pass)
  constexpr int CHUNKS = sym_table_doubles(LH) / 2;  // 16-byte copies
  static_assert(sym_table_doubles(LH) % 2 == 0, "16-byte table copies");
  for (int i = threadIdx.x; i < CHUNKS; i += FftPlan<LH>::T) hil_cp_async16(ksh + 2 * i, p.ksym + 2 * i);
  const size_t base = (size_t)col * p.NE;
  convolve_run<R, LH, false>(FieldIn<R>{&p, base, nullptr}, SpecSym<LH, false>{ksh}, ParkOut<R, LH>{&p, base}, buf,
                             p.twh, nullptr);
  convolve_run<R, LH, false>(FieldIn<R>{&p, base, p.tw}, SpecSym<LH, true>{ksh}, CompleteOut<R, LH>{&p, base}, buf,
                             p.twh, nullptr);
}

// ---------------------------------------------------------------------------
// Host side: per-(N_E, spacing) tables.
// ---------------------------------------------------------------------------
static void host_fft(std::vector<double>& re, std::vector<double>& im) {
  const size_t n = re.size();
  for (size_t i = 1, j = 0; i < n; ++i) {
    size_t bit = n >> 1;
    for (; j & bit; bit >>= 1) j ^= bit;
    j ^= bit;
    if (i < j) {
      std::swap(re[i], re[j]);
      std::swap(im[i], im[j]);
    }
  }
  for (size_t len = 2; len <= n; len <<= 1) {
    for (size_t k = 0; k < len / 2; ++k) {
      const double ang = -2.0 * M_PI * (double)k / (double)len;
      const double wr = cos(ang), wi = sin(ang);
      for (size_t i = 0; i < n; i += len) {
        const size_t a = i + k, b = i + k + len / 2;
        const double xr = re[b] * wr - im[b] * wi, xi = re[b] * wi + im[b] * wr;
        re[b] = re[a] - xr;
        im[b] = im[a] - xi;
        re[a] += xr;
        im[a] += xi;
      }
    }
  }
}

int next_pow2(int n) {
  int L = 1;
  while (L < n) L <<= 1;
  return L;
}

void free_hilbert_tables(HilbertTables& t) {
  cudaFree(t.khat);
  cudaFree(t.kodd);
  cudaFree(t.tw);
  cudaFree(t.twist);
  cudaFree(t.ksplit);
  cudaFree(t.twh);
  cudaFree(t.twt);
  cudaFree(t.ksym);
  cudaFree(t.partial);
  t = HilbertTables();
}

template <typename R> static int upload_cx(void** dst, const std::vector<double>& re, const std::vector<double>& im) {
  std::vector<Cx<R>> h(re.size());
  for (size_t i = 0; i < re.size(); ++i) h[i] = cx<R>((R)re[i], (R)im[i]);
  QCL_CUDA_CHECK(cudaMalloc(dst, h.size() * sizeof(Cx<R>)));
  QCL_CUDA_CHECK(cudaMemcpy(*dst, h.data(), h.size() * sizeof(Cx<R>), cudaMemcpyHostToDevice));
  // the tables are read by kernels on non-blocking streams, which are not
  // ordered after this legacy-stream copy: wait until it has landed
  QCL_CUDA_CHECK(cudaDeviceSynchronize());
  return QCL_OK;
}

int check_uniform_grid(int NE, const double* eps_host, double* de_out) {
  if (NE < 2) {
    set_last_error("at least two energy nodes are required");
    return QCL_ARG;
  }
  const double de = eps_host[1] - eps_host[0];
  if (!(de > 0)) {
    set_last_error("energy grid must be strictly increasing");
    return QCL_ARG;
  }
  double dev = 0, mx = fmax(fabs(de), 1.0);
  for (int e = 0; e < NE; ++e) mx = fmax(mx, fabs(eps_host[e]));
  for (int e = 1; e < NE; ++e) dev = fmax(dev, fabs((eps_host[e] - eps_host[e - 1]) - de));
  if (!(dev <= 256 * 2.220446049250313e-16 * mx)) {
    set_last_error("FFT Hilbert transform requires a uniform energy grid");
    return QCL_ARG;
  }
  *de_out = de;
  return QCL_OK;
}

// Builds (or reuses) the tables for (NE, de, precision).
int prepare_hilbert_tables(HilbertTables& t, int NE, double de, int precision) {
  const int L = next_pow2(2 * NE - 1);
  const int storage = precision == QCL_C128 ? QCL_C128 : QCL_C64;
  if (t.NE == NE && t.de == de && t.precision == storage && t.khat) return QCL_OK;
  free_hilbert_tables(t);
  const int maxL = storage == QCL_C128 ? 8192 : 16384;
  if (L < 64 || L > maxL) {
    set_last_error("FFT Hilbert length %d outside the supported range [64, %d]", L, maxL);
    return QCL_UNSUPPORTED;
  }
  // kernel spectra at L and 2L
  std::vector<double> kr(L, 0.0), ki(L, 0.0), kr2(2 * L, 0.0), ki2(2 * L, 0.0);
  for (int lag = -(NE - 1); lag <= NE - 1; ++lag) {
    if (lag == 0) continue;
    const double v = 1.0 / (2.0 * M_PI * lag * de);
    kr[lag + NE - 1] = v;
    kr2[lag + NE - 1] = v;
  }
  host_fft(kr, ki);
  host_fft(kr2, ki2);
  const int LH = L / 2;
  std::vector<double> kor(L), koi(L), twr(L), twi(L), tsr(L), tsi(L), ksr(L), ksi(L), thr(LH), thi(LH);
  for (int k = 0; k < L; ++k) {
    kor[k] = kr2[2 * k + 1];
    koi[k] = ki2[2 * k + 1];
    twr[k] = cos(2.0 * M_PI * k / L);
    twi[k] = -sin(2.0 * M_PI * k / L);
    tsr[k] = cos(M_PI * k / L);
    tsi[k] = -sin(M_PI * k / L);
    const int j = k >> 1, r = k & 1;  // even spectrum first, then odd
    ksr[r * LH + j] = kr[k];
    ksi[r * LH + j] = ki[k];
  }
  for (int k = 0; k < LH; ++k) {
    thr[k] = cos(2.0 * M_PI * k / LH);
    thi[k] = -sin(2.0 * M_PI * k / LH);
  }
  int st;
  if (storage == QCL_C128) {
    // centred kernel k[lag mod L]: its spectrum is i S, S real and odd
    // (S[L - f] = -S[f]); the table keeps S[2f], f <= L/4, padded to an even
    // count, then S[2f + 1], f < L/4 (the layout SpecSym reads)
    std::vector<double> cr(L, 0.0), ci(L, 0.0);
    for (int lag = 1; lag <= NE - 1; ++lag) {
      const double v = 1.0 / (2.0 * M_PI * lag * de);
      cr[lag] = v;
      cr[L - lag] = -v;
    }
    host_fft(cr, ci);
    const int odd0 = LH / 2 + 2;
    std::vector<double> sym(odd0 + LH / 2, 0.0);
    for (int f = 1; f <= LH / 2; ++f) {
      const int g = 2 * f;  // S[0] = S[L/2] = 0 exactly
      sym[f] = g == LH ? 0.0 : 0.5 * (ci[g] - ci[L - g]);
    }
    for (int f = 0; f < LH / 2; ++f) sym[odd0 + f] = 0.5 * (ci[2 * f + 1] - ci[L - 2 * f - 1]);
    QCL_CUDA_CHECK(cudaMalloc(&t.ksym, sym.size() * sizeof(double)));
    QCL_CUDA_CHECK(cudaMemcpy(t.ksym, sym.data(), sym.size() * sizeof(double), cudaMemcpyHostToDevice));
    QCL_CUDA_CHECK(cudaDeviceSynchronize());
    if ((st = upload_cx<double>(&t.khat, kr, ki))) return st;
    if ((st = upload_cx<double>(&t.kodd, kor, koi))) return st;
    if ((st = upload_cx<double>(&t.tw, twr, twi))) return st;
    if ((st = upload_cx<double>(&t.twist, tsr, tsi))) return st;
    if ((st = upload_cx<double>(&t.ksplit, ksr, ksi))) return st;
    if ((st = upload_cx<double>(&t.twh, thr, thi))) return st;
  } else {
    if ((st = upload_cx<float>(&t.khat, kr, ki))) return st;
    if ((st = upload_cx<float>(&t.kodd, kor, koi))) return st;
    if ((st = upload_cx<float>(&t.tw, twr, twi))) return st;
    if ((st = upload_cx<float>(&t.twist, tsr, tsi))) return st;
    if ((st = upload_cx<float>(&t.ksplit, ksr, ksi))) return st;
    if ((st = upload_cx<float>(&t.twh, thr, thi))) return st;
    // pass twiddle tables (the order and offsets of conv_fwd_seg / conv_inv_seg)
    int P = 0;
    for (int x = L; x > 16; x /= 16) ++P;
    const int S = L >> (4 * P);
    std::vector<double> pr, pi;
    auto seg = [&](int radix, int ns) {
      for (int r = 1; r < radix; ++r)
        for (int k = 0; k < ns; ++k) {
          const long long m = (long long)k * (L / (ns * radix)) * r;  // < L
          pr.push_back(cos(2.0 * M_PI * (double)m / L));
          pi.push_back(-sin(2.0 * M_PI * (double)m / L));
        }
    };
    for (int i = 0, ns = S; i < P; ++i, ns *= 16) seg(16, ns);
    for (int i = 1, ns = 16; i < P; ++i, ns *= 16) seg(16, ns);
    seg(S, L / S);
    if (pr.size() != (size_t)(2 * L - S - 16)) {
      set_last_error("internal: FFT pass-table size %zu for L = %d", pr.size(), L);
      return QCL_UNSUPPORTED;
    }
    if ((st = upload_cx<float>(&t.twt, pr, pi))) return st;
  }
  t.NE = NE;
  t.L = L;
  t.de = de;
  t.precision = storage;
  return QCL_OK;
}

int ensure_partial(HilbertTables& t, long long ncols) {
  if (t.partial_cols >= ncols) return QCL_OK;
  cudaFree(t.partial);
  t.partial = nullptr;
  QCL_CUDA_CHECK(cudaMalloc(&t.partial, (size_t)ncols * 2 * sizeof(double)));
  t.partial_cols = ncols;
  return QCL_OK;
}

template <typename R, int L, bool VERIFY> static int launch_hilbert_LV(const HilbertArgs<R>& a, cudaStream_t st) {
  constexpr int T = FftPlan<L>::T;
  constexpr size_t smem = hilbert_smem_bytes<R, L, VERIFY>();
  static bool configured = false;
  if (!configured) {
    QCL_CUDA_CHECK(cudaFuncSetAttribute(hilbert_kernel<R, L, VERIFY>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        (int)smem));
    configured = true;
  }
  const long long nc = a.ncols;
  dim3 grid((unsigned)(nc < 65535 ? nc : 65535), (unsigned)((nc + 65534) / 65535));
  hilbert_kernel<R, L, VERIFY><<<grid, T, smem, st>>>(a);
  QCL_LAUNCH_CHECK("hilbert_kernel");
  return QCL_OK;
}
template <typename R, int LH> static int launch_hilbert_halves(const HilbertArgs<R>& a, cudaStream_t st) {
  constexpr int T = FftPlan<LH>::T;
  constexpr size_t smem = (size_t)(LH + LH / 16) * sizeof(Cx<R>) + sym_table_doubles(LH) * sizeof(double);
  static_assert(2 * (smem + 1024) <= 228 * 1024, "two columns per SM");
  static bool configured = false;
  if (!configured) {
    QCL_CUDA_CHECK(cudaFuncSetAttribute(hilbert_halves_kernel<R, LH>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        (int)smem));
    configured = true;
  }
  const long long nc = a.ncols;
  dim3 grid((unsigned)(nc < 65535 ? nc : 65535), (unsigned)((nc + 65534) / 65535));
  hilbert_halves_kernel<R, LH><<<grid, T, smem, st>>>(a);
  QCL_LAUNCH_CHECK("hilbert_halves_kernel");
  return QCL_OK;
}

// The half-length form is used for the complex128 transform whose length-L
// column fills an SM's shared memory (L = 8192; at L = 4096 two columns
// already share an SM and the one-pass kernel is faster).
template <typename R, int L> constexpr bool kHilbertHalves = sizeof(R) == 8 && L == 8192;

template <typename R, int L> static int launch_hilbert_L(const HilbertArgs<R>& a, bool halves, cudaStream_t st) {
  if (a.partial) return launch_hilbert_LV<R, L, true>(a, st);
  if constexpr (kHilbertHalves<R, L>) {
    if (halves) return launch_hilbert_halves<R, L / 2>(a, st);
  }
  return launch_hilbert_LV<R, L, false>(a, st);
}

template <typename R> static int launch_hilbert_t(const HilbertArgs<R>& a, int L, bool halves, cudaStream_t st) {
  switch (L) {
    case 64: return launch_hilbert_L<R, 64>(a, halves, st);
    case 128: return launch_hilbert_L<R, 128>(a, halves, st);
    case 256: return launch_hilbert_L<R, 256>(a, halves, st);
    case 512: return launch_hilbert_L<R, 512>(a, halves, st);
    case 1024: return launch_hilbert_L<R, 1024>(a, halves, st);
    case 2048: return launch_hilbert_L<R, 2048>(a, halves, st);
    case 4096: return launch_hilbert_L<R, 4096>(a, halves, st);
    case 8192: return launch_hilbert_L<R, 8192>(a, halves, st);
    case 16384:
      if constexpr (sizeof(R) == 4) return launch_hilbert_L<R, 16384>(a, halves, st);
      [[fallthrough]];
    default:
      set_last_error("unsupported FFT length %d", L);
      return QCL_UNSUPPORTED;
  }
}

// Launch on device arrays.  Exactly one of (Gam) or (SL, SG) is the input and
// one of (Lam) or (SR) the output.  If verify, per-column partial sums land in
// t.partial (2 doubles per column).
int launch_hilbert(HilbertTables& t, int precision, long long ncols, const double* wE, const void* Gam,
                   const void* SL, const void* SG, void* Lam, void* SR, void* GamOut, bool verify,
                   cudaStream_t st, long long partial_offset) {
  if (verify) {
    int s = ensure_partial(t, ncols + partial_offset);
    if (s) return s;
  }
  if (ncols <= 0) return QCL_OK;
  // the half-length kernel reads the field twice: not used when the output
  // overlaps it ...
  const size_t bytes = (size_t)ncols * t.NE * (precision == QCL_C128 ? 16 : 8);
  const char* out = (const char*)(SR ? SR : Lam);
  auto overlaps = [&](const void* in) {
    const char* c = (const char*)in;
    return c && c < out + bytes && out < c + bytes;
  };
  // ... nor below two columns per SM, where the one-pass kernel's 2x wider
  // CTAs finish a column sooner
  int dev = 0, sms = 148;
  if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const bool halves = ncols >= 2LL * sms && !overlaps(Gam) && !overlaps(SL) && !overlaps(SG);
  if (precision == QCL_C128) {
    HilbertArgs<double> a{t.NE,
                          ncols,
                          wE,
                          (const Cx<double>*)Gam,
                          (const Cx<double>*)SL,
                          (const Cx<double>*)SG,
                          (Cx<double>*)Lam,
                          (Cx<double>*)SR,
                          (Cx<double>*)GamOut,
                          (const Cx<double>*)t.khat,
                          (const Cx<double>*)t.kodd,
                          (const Cx<double>*)t.tw,
                          (const Cx<double>*)t.twist,
                          verify ? t.partial + 2 * partial_offset : nullptr,
                          1.0 / t.L,
                          (const Cx<double>*)t.ksplit,
                          (const Cx<double>*)t.twh,
                          nullptr,
                          (const double*)t.ksym};
    return launch_hilbert_t<double>(a, t.L, halves, st);
  }
  HilbertArgs<float> a{t.NE,
                       ncols,
                       wE,
                       (const Cx<float>*)Gam,
                       (const Cx<float>*)SL,
                       (const Cx<float>*)SG,
                       (Cx<float>*)Lam,
                       (Cx<float>*)SR,
                       (Cx<float>*)GamOut,
                       (const Cx<float>*)t.khat,
                       (const Cx<float>*)t.kodd,
                       (const Cx<float>*)t.tw,
                       (const Cx<float>*)t.twist,
                       verify ? t.partial + 2 * partial_offset : nullptr,
                       1.0 / t.L,
                       (const Cx<float>*)t.ksplit,
                       (const Cx<float>*)t.twh,
                       (const Cx<float>*)t.twt,
                       nullptr};
  return launch_hilbert_t<float>(a, t.L, halves, st);
}

}  // namespace qcl
