// Optional scattering-model switches applied to each candidate family.
//
//   retarded_real_part = :drop   Sigma^R = -i Gamma / 2 with Gamma = i (Sigma^> - Sigma^<),
//                                i.e. Sigma^R = (Sigma^> - Sigma^<) / 2
//                                (_retarded_self_energy_selected, numerics/optimized/
//                                production_operators.jl:1174-1177);
//   self_energy_structure = :diagonal   off-diagonal (a != b) entries zeroed
//                                (_diagonalize_blocks!, :1208-1217);
//   transverse_momentum = :averaged     X[e,m,a,b] <- sum_m' wk[m'] X[e,m',a,b] / sum wk
//                                for every m (_average_transverse_momentum!, :1219-1238).
// All three are HBM-bound elementwise / strided-reduction sweeps.  The last
// two act per (e, a, b) column over the momenta, so one thread owns one
// (e, (a,b)) pair for all three components: reads along e are coalesced.
#include "kernels.cuh"

namespace qcl {

static unsigned model_grid(long long n, int t) {
  long long g = (n + t - 1) / t;
  return (unsigned)(g < 148 * 16 ? (g > 0 ? g : 1) : 148 * 16);
}

template <typename R>
__global__ void retarded_drop_kernel(long long n, const Cx<R>* __restrict__ SL, const Cx<R>* __restrict__ SG,
                                     Cx<R>* __restrict__ SR) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const Cx<R> l = SL[i], g = SG[i];
    SR[i] = cx<R>((R)(0.5 * ((double)g.x - (double)l.x)), (R)(0.5 * ((double)g.y - (double)l.y)));
  }
}

int launch_retarded_drop(int precision, size_t n, const void* SL, const void* SG, void* SR, cudaStream_t st) {
  if (precision == QCL_C128)
    retarded_drop_kernel<double><<<model_grid((long long)n, 256), 256, 0, st>>>(
        (long long)n, (const Cx<double>*)SL, (const Cx<double>*)SG, (Cx<double>*)SR);
  else
    retarded_drop_kernel<float><<<model_grid((long long)n, 256), 256, 0, st>>>(
        (long long)n, (const Cx<float>*)SL, (const Cx<float>*)SG, (Cx<float>*)SR);
  QCL_LAUNCH_CHECK("retarded_drop_kernel");
  return QCL_OK;
}

template <typename R> struct ModelFields {
  Cx<R>* x[3];
};

template <typename R>
__global__ void scattering_model_kernel(int NE, int Nk, int N, const double* __restrict__ wk, double norm,
                                        int diagonal, int averaged, ModelFields<R> f) {
  const long long cols = (long long)NE * N * N;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < cols;
       i += (long long)gridDim.x * blockDim.x) {
    const int e = (int)(i % NE);
    const long long p = i / NE;  // (a, b), a fastest
    const int a = (int)(p % N), b = (int)(p / N);
    const size_t base = (size_t)e + (size_t)NE * (size_t)Nk * (size_t)p;
    const bool zero = diagonal && a != b;
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      Cx<R>* X = f.x[c];
      if (zero) {
        for (int m = 0; m < Nk; ++m) X[base + (size_t)NE * m] = cx<R>(0, 0);
      } else if (averaged) {
        double sx = 0, sy = 0;
        for (int m = 0; m < Nk; ++m) {
          const Cx<R> v = X[base + (size_t)NE * m];
          sx += wk[m] * (double)v.x;
          sy += wk[m] * (double)v.y;
        }
        const Cx<R> v = cx<R>((R)(sx / norm), (R)(sy / norm));
        for (int m = 0; m < Nk; ++m) X[base + (size_t)NE * m] = v;
      }
    }
  }
}

int launch_scattering_model(int precision, int NE, int Nk, int N, const double* wk, double norm, int diagonal,
                            int averaged, void* const* fields, cudaStream_t st) {
  if (!diagonal && !averaged) return QCL_OK;
  const long long cols = (long long)NE * N * N;
  if (precision == QCL_C128) {
    ModelFields<double> f{{(Cx<double>*)fields[0], (Cx<double>*)fields[1], (Cx<double>*)fields[2]}};
    scattering_model_kernel<double><<<model_grid(cols, 256), 256, 0, st>>>(NE, Nk, N, wk, norm, diagonal,
                                                                          averaged, f);
  } else {
    ModelFields<float> f{{(Cx<float>*)fields[0], (Cx<float>*)fields[1], (Cx<float>*)fields[2]}};
    scattering_model_kernel<float><<<model_grid(cols, 256), 256, 0, st>>>(NE, Nk, N, wk, norm, diagonal,
                                                                         averaged, f);
  }
  QCL_LAUNCH_CHECK("scattering_model_kernel");
  return QCL_OK;
}

}  // namespace qcl
