// Neighbour-period embedding self-energies: shifted sandwiches.
//
// Reference: _embedding_component_production / _embedding_self_energy_
// production (numerics/optimized/production_operators.jl:886-941); oracle
// embedding_self_energy (numerics/reference/periodicity.jl:113-150):
//   Sigma+^x(E) = T+ G^x(E + E^p) T+^H,  Sigma-^x(E) = T- G^x(E - E^p) T-^H,
// x in {R, <, >}, with G(E +- E^p) the 2-point linear interpolation of the
// EnergyShiftPlan and zero outside the window.
//
// One kernel does all (sign, component) jobs: grid.z is the sign, the three
// components are processed in turn by the same CTA so T is staged in shared
// memory once.  The interpolation is fused into the coalesced block load.
#include "blockmat.cuh"

namespace qcl {

template <typename R> struct SandwichArgs {
  int NE, Nk, N, njobs;
  SandwichJob jobs[2];
};

template <typename R, int NP, int BPC>
__device__ __forceinline__ void load_shifted(const Cx<R>* __restrict__ X, const ShiftPlanDev& plan, Cx<R>* bufs,
                                             int e0, int m, int NE, int Nk, int N) {
  // blockDim.x is a multiple of BPC, so each thread serves one energy of the
  // CTA: its interpolation plan is read once; the padded tile index is split
  // at compile time (entries past N are left as they are, as before)
  const int eloc = threadIdx.x % BPC;
  const int e = e0 + eloc;
  const bool ok = e < NE && plan.valid[e];
  int l = 0, r = 0;
  double th = 0.0;
  if (ok) {
    l = plan.left[e];
    r = plan.right[e];
    th = plan.theta[e];
  }
  const bool two = l != r && th != 0.0;
  const size_t base = (size_t)NE * m, cstride = (size_t)NE * Nk;
  for (int i = threadIdx.x; i < BPC * NP * NP; i += blockDim.x) {
    const int el = i / BPC;
    const int a = el % NP, b = el / NP;
    if (a >= N || b >= N) continue;
    Cx<R> v = cx<R>(0, 0);
    if (ok) {
      const size_t col = base + cstride * ((size_t)a + (size_t)N * b);
      if (!two) {
        v = X[col + l];
      } else {
        const Cx<R> u = X[col + l], w = X[col + r];
        v = cx<R>((R)((1 - th) * u.x + th * w.x), (R)((1 - th) * u.y + th * w.y));
      }
    }
    bufs[(size_t)eloc * NP * NP + sw<NP>(a, b)] = v;
  }
}

template <typename R, int NP, int BPC>
__global__ void __launch_bounds__(BPC* Tile<NP>::TT) sandwich_kernel(SandwichArgs<R> p) {
  constexpr int TT = Tile<NP>::TT;
  constexpr size_t MSZ = (size_t)NP * NP;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  Cx<R>* Ts = reinterpret_cast<Cx<R>*>(smem_raw);
  Cx<R>* bufX = Ts + MSZ;
  Cx<R>* bufT = bufX + BPC * MSZ;
  const SandwichJob& job = p.jobs[blockIdx.z];
  const int N = p.N, NE = p.NE, Nk = p.Nk;
  const int m = blockIdx.y, e0 = blockIdx.x * BPC;
  const int team = threadIdx.x / TT, tt = threadIdx.x % TT;
  const Cx<double>* T = (const Cx<double>*)job.T;
  for (int i = threadIdx.x; i < NP * NP; i += blockDim.x) {
    const int a = i % NP, b = i / NP;
    Ts[sw<NP>(a, b)] = (a < N && b < N) ? cvt<R>(T[a + (size_t)N * b]) : cx<R>(0, 0);
  }
  Cx<R>* X = bufX + team * MSZ;
  Cx<R>* W = bufT + team * MSZ;
  for (int c = 0; c < 3; ++c) {
    if (job.X[c] == nullptr || job.S[c] == nullptr) continue;  // uniform
    __syncthreads();
    load_shifted<R, NP, BPC>((const Cx<R>*)job.X[c], job.plan, bufX, e0, m, NE, Nk, N);
    __syncthreads();
    team_matmul<R, R, NP>(Ts, X, W, N, tt, false);  // W = T X
    team_sync<TT>(team);
    team_matmul<R, R, NP>(W, Ts, X, N, tt, true);   // X = W T^H
    __syncthreads();
    store_blocks<R, R, NP, BPC>((Cx<R>*)job.S[c], bufX, MSZ, e0, m, NE, Nk, N);
  }
}

template <typename R, int NP, int BPC>
static int launch_sandwich_t(const SandwichArgs<R>& a, cudaStream_t st) {
  constexpr int TT = Tile<NP>::TT;
  constexpr size_t smem = (1 + 2 * (size_t)BPC) * NP * NP * sizeof(Cx<R>);
  static bool configured = false;
  if (!configured) {
    QCL_CUDA_CHECK(cudaFuncSetAttribute(sandwich_kernel<R, NP, BPC>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        (int)smem));
    configured = true;
  }
  dim3 grid((a.NE + BPC - 1) / BPC, a.Nk, a.njobs);
  sandwich_kernel<R, NP, BPC><<<grid, BPC * TT, smem, st>>>(a);
  QCL_LAUNCH_CHECK("sandwich_kernel");
  return QCL_OK;
}

template <typename R> static int launch_sandwich_p(const SandwichArgs<R>& a, cudaStream_t st) {
  constexpr bool wide = sizeof(R) == 8;
  switch (padded_size(a.N)) {
    case 8: return launch_sandwich_t<R, 8, 8>(a, st);
    case 16: return launch_sandwich_t<R, 16, wide ? 4 : 8>(a, st);
    case 24: return launch_sandwich_t<R, 24, wide ? 2 : 4>(a, st);
    case 32: return launch_sandwich_t<R, 32, wide ? 1 : 2>(a, st);
    case 48: return launch_sandwich_t<R, 48, 1>(a, st);
    default:
      set_last_error("basis size N_b=%d exceeds the supported maximum 48", a.N);
      return QCL_UNSUPPORTED;
  }
}

int launch_sandwich(int precision, int NE, int Nk, int N, const SandwichJob* jobs, int njobs, cudaStream_t st) {
  if (njobs < 1 || njobs > 2) {
    set_last_error("sandwich: 1 or 2 jobs per launch");
    return QCL_ARG;
  }
  if (precision == QCL_C128) {
    SandwichArgs<double> a;
    a.NE = NE; a.Nk = Nk; a.N = N; a.njobs = njobs;
    for (int j = 0; j < njobs; ++j) a.jobs[j] = jobs[j];
    return launch_sandwich_p<double>(a, st);
  }
  SandwichArgs<float> a;
  a.NE = NE; a.Nk = Nk; a.N = N; a.njobs = njobs;
  for (int j = 0; j < njobs; ++j) a.jobs[j] = jobs[j];
  return launch_sandwich_p<float>(a, st);
}

}  // namespace qcl
