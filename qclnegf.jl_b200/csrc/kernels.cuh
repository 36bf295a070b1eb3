// Internal launch interfaces shared by the translation units.
#pragma once
#include <vector>

#include "common.cuh"

namespace qcl {

int padded_size(int N);
int next_pow2(int n);

int launch_dyson_keldysh(int precision, int NE, int Nk, int N, const double* eps, double eta, const void* h,
                         const void* sigR, const void* sigL, const void* sigG, void* GR, void* GL, void* GG,
                         double* scale, void* traceL, void* traceG, int* status, cudaStream_t st, int m0 = 0,
                         int mcount = -1);

int launch_dyson_keldysh_bpc(int precision, int NE, int Nk, int N, const double* eps, double eta, const void* h,
                             const void* sigR, const void* sigL, const void* sigG, void* GR, void* GL, void* GG,
                             double* scale, void* traceL, void* traceG, int* status, cudaStream_t st, int m0,
                             int mcount, int bpc);
// Dyson CTA shapes (blocks per CTA): candidates, default, current (tuned or default), set
int dyson_bpc_candidates(int NP, int* out);
int dyson_default_bpc(int precision, int NP);
int dyson_bpc(int precision, int NP);
void dyson_set_bpc(int precision, int NP, int bpc);

int launch_weighted_trace(int NE, int Nk, const void* tr, const double* wE, const double* wk, double* partial,
                          double* out, cudaStream_t st);
int launch_paired_coefficients(const double* trL, const double* trG, int gs, double target, double* coeffs,
                               int* status, cudaStream_t st, double realness_limit = 1e-10, int scalar = 0,
                               int branch = 0);
int launch_density_matrix(int precision, int NE, int Nk, int N, const void* GL, const double* wE, const double* wk,
                          double* out, cudaStream_t st);
int launch_scalar_lesser(int precision, int NE, int Nk, int N, const void* GR, void* GL, void* GG,
                         const double* coeffs, cudaStream_t st);
int launch_normalize_pair(int precision, size_t n, void* GL, void* GG, const double* coeffs, cudaStream_t st);
// condition number / Dyson scale and the spectral function (residual.cu)
int launch_condition(int precision, int NE, int Nk, int N, const double* eps, double eta, const void* h,
                     const void* SR, const void* GR, double* kappa, double* scale, cudaStream_t st);
int launch_spectral(int precision, int NE, int Nk, int N, const void* GR, void* A, cudaStream_t st);
// positivity witness of a residual-suite run (residual.cu)
int launch_residual_witness(int precision, int NE, int Nk, int N, const void* GR, const void* GL, const void* GG,
                            const void* SL, const void* SG, const double* work, double* partial, double* out12,
                            cudaStream_t st);
size_t residual_witness_partial_doubles();
// Anderson mixing (anderson.cu; guard in residual.cu).  Device-resident mixer
// state, so that an iteration stays one stream-ordered launch sequence.
constexpr int kAndersonMaxDepth = 8;
struct AndersonMeta {
  int count;   // history entries; logical entry j is ring slot (head + j) % depth
  int head;
  int slot;    // ring slot of this step's entry
  int reason;  // 0 none, 1 residual_increase, 2 coefficient_solve, 3 coefficient_bound, 4 causality_guard
  int fallback;    // the guard rejected the accelerated state; linear fallback applied
  int accepted;    // accelerated state accepted with more than one non-zero coefficient
  int used;        // history entries the mix used
  int guard_code;  // code of the first failing block of the first guard pass (0 none)
  unsigned long long guard_key;   // (1-based first failing index << 3) | code of the current pass
  unsigned long long guard_first; // 1-based first failing index of the first pass (0 none)
  double prior;    // <R_last, R_last> before this step (< 0: empty history)
  double l1;       // sum |coefficients|
  double gram[kAndersonMaxDepth * kAndersonMaxDepth];
  double coef[kAndersonMaxDepth];
  double dots[kAndersonMaxDepth + 1];
};
size_t anderson_partial_doubles(int nf);
int launch_anderson_reset(AndersonMeta* m, cudaStream_t st);
int launch_anderson_plan(AndersonMeta* m, int depth, cudaStream_t st);
int launch_anderson_append(int precision, size_t n, const void* const* state, const void* const* cand, int nf,
                           void* Xh, void* Rh, int depth, AndersonMeta* meta, double* partial, double* fam_out,
                           cudaStream_t st);
int launch_anderson_coefficients(AndersonMeta* m, int depth, double regularization, cudaStream_t st);
int launch_anderson_mix(int precision, size_t n, void* const* out, int nf, const void* Xh, const void* Rh, int depth,
                        const AndersonMeta* m, double damping, int fallback, cudaStream_t st);
int launch_anderson_after_guard(AndersonMeta* m, int pass, int* status, cudaStream_t st);
int launch_anderson_guard(int precision, int NE, int Nk, int N, void* const* fields, int nfam, AndersonMeta* m,
                          int pass, double roundoff, cudaStream_t st);
// dense kernel operators from angular node weights (kbuild.cu)
size_t assemble_work_doubles();
int launch_assemble_kernel(int form, int Nk, int Nb, int T, const double* W, const void* X, void* out, double* work,
                           cudaStream_t st);
// scattering-model switches (model.cu)
int launch_retarded_drop(int precision, size_t n, const void* SL, const void* SG, void* SR, cudaStream_t st);
int launch_scattering_model(int precision, int NE, int Nk, int N, const double* wk, double norm, int diagonal,
                            int averaged, void* const* fields, cudaStream_t st);
int launch_sum_fields(int precision, size_t n, const void* const* src, int count, void* out, cudaStream_t st);
constexpr int kMaxMixFields = 32;
size_t residual_mix_multi_partial_doubles(int nf);
int launch_residual_mix_multi(int precision, size_t n, const void* const* old, void* const* cand, int nf,
                              double alpha, double* partial, double* out, cudaStream_t st);
int launch_residual_mix(int precision, size_t n, const void* old, void* new_, double alpha, double* partial,
                        double* out2, cudaStream_t st);
int launch_combine(const double* partial, int count, int K, double* out, cudaStream_t st);
int launch_axpby(int precision, size_t n, double a, const void* x, double b, const void* y, void* out,
                 cudaStream_t st);
constexpr int kReduceCtas = 296;

// Device view of an EnergyShiftPlan (0-based left/right).
struct ShiftPlanDev {
  const int* left = nullptr;
  const int* right = nullptr;
  const double* theta = nullptr;
  const unsigned char* valid = nullptr;
};
int build_shift_plan_host(int NE, const double* eps, double delta, int* left, int* right, double* theta,
                          unsigned char* valid);
int launch_shift(int precision, int NE, long long ncols, const ShiftPlanDev& plan, const void* X, void* Y,
                 cudaStream_t st);
int launch_shift_pair(int precision, int NE, long long ncols, const ShiftPlanDev& p1, const ShiftPlanDev& p2, double a,
                      double b, const void* X, void* Y, cudaStream_t st);

// Device view of a factorised kernel operator (arrays in the field precision).
struct KernelOpDev {
  int kind = 0;
  int J = 0;
  const void* block = nullptr;   // (N^2, N^2): rows (a,b), cols (c,d)
  const void* matrix = nullptr;  // (Nk N^2)^2: rows (m,a,b), cols (m',c,d)
  const void* left = nullptr;    // IFR (N^2, J); low rank (Nk N^2, rank)
  const void* right = nullptr;   // IFR (J, N^2); low rank right_adjoint (rank, Nk N^2)
  const void* radial = nullptr;  // IFR (Nk, Nk); separable sum (Nk, Nk, J)
  // dense operators, complex64 fields: tensor-core operand (scaled FP16 hi/lo
  // pair) prepared by tc_build_operator; when set, the contraction runs on tcgen05
  const void* tc_bop = nullptr;
  // separable sums, complex64 fields: one prepared operand per chunk of
  // kSepChunk terms (host array of device pointers)
  const void* const* tc_chunks = nullptr;
  const void* const* tc_stage1 = nullptr;  // separable sum: stage-1 operand per chunk (radial factors)
  int* status = nullptr;  // device status word for bounded-wait timeouts
};
// Terms of a separable-sum operator contracted per stage-2 GEMM: the
// intermediate of a chunk holds kSepChunk fields.
constexpr int kSepChunk = 8;
inline int sep_chunks(int J) { return (J + kSepChunk - 1) / kSepChunk; }
size_t contraction_work_elems(const KernelOpDev& op, int NE, int Nk, int N);
int sep_build_tc_operands(int Nk, int N, int J, const void* radial_c64, const void* block_c64, const double* wk,
                          std::vector<void*>& stage2, std::vector<void*>& stage1, cudaStream_t st);
// tensor-core dense contraction (tc_gemm.cu)
int tc_build_operator(int Nc, int Nk, const void* Mop_c64, const double* wk, void** Bop, cudaStream_t st);
int tc_build_operator2(int Nout, int Kc, int Nk, const void* Mop_c64, const double* wk, void** Bop, cudaStream_t st);
size_t tc_a_work_floats(int NE, int Nc);
size_t tc_a_work_floats2(int M, int Kc);
size_t tc_operator_bytes(int Nout, int Kc);
int tc_set_wait_limit(long long rounds);
int launch_tc_contraction2(int M, int Nout, int Kc, const void* Bop, const void* A, void* S, double alpha,
                           double beta, float* awork, int* status, cudaStream_t st);
int tc_split_rows(int M, int Kc, const void* A, long long P, long long Bs, float* awork, cudaStream_t st);
int launch_tc_presplit(int M, int Nout, int Kc, const void* Bop, const float* awork, void* S, long long oP,
                       long long oQ, long long oR, double alpha, double beta, int* status, cudaStream_t st);
int launch_tc_dense_contraction(int NE, int Nc, const void* Bop, const void* G, void* S, double alpha, double beta,
                                float* awork, int* status, cudaStream_t st);
int launch_contraction(int precision, const KernelOpDev& op, int NE, int Nk, int N, const double* wk, const void* G,
                       void* S, double alpha_q, double beta, void* work, cudaStream_t st);

// Shifted sandwiches  S_c(e,m) = T X_c(shift(e), m) T^H  for up to 3
// components and 2 signs (embedding self-energies).
struct SandwichJob {
  const void* X[3] = {nullptr, nullptr, nullptr};
  void* S[3] = {nullptr, nullptr, nullptr};
  const void* T = nullptr;  // complex128 N x N (column-major)
  ShiftPlanDev plan;
};
int launch_sandwich(int precision, int NE, int Nk, int N, const SandwichJob* jobs, int njobs, cudaStream_t st);

struct HilbertTables {
  int NE = 0, L = 0, precision = -1;
  double de = 0;
  void* khat = nullptr;
  void* kodd = nullptr;
  void* tw = nullptr;
  void* twist = nullptr;
  void* ksplit = nullptr;
  void* twh = nullptr;
  void* twt = nullptr;
  void* ksym = nullptr;  // complex128: the centred kernel's real spectrum halves
  double* partial = nullptr;
  long long partial_cols = 0;
};
void free_hilbert_tables(HilbertTables& t);
int check_uniform_grid(int NE, const double* eps_host, double* de_out);
int prepare_hilbert_tables(HilbertTables& t, int NE, double de, int precision);
int ensure_partial(HilbertTables& t, long long ncols);
int launch_hilbert(HilbertTables& t, int precision, long long ncols, const double* wE, const void* Gam,
                   const void* SL, const void* SG, void* Lam, void* SR, void* GamOut, bool verify,
                   cudaStream_t st, long long partial_offset = 0);

int launch_residual_suite(int precision, int NE, int Nk, int N, const double* eps, const void* h, const void* GR,
                          const void* GL, const void* GG, const void* SR, const void* SL, const void* SG,
                          const void* SLc, double* work, double* out5, cudaStream_t st);
size_t residual_work_doubles(int NE, int Nk);
enum { RES_PART_ALL = 0, RES_PART_MAIN = 1, RES_PART_RK = 2 };
int launch_residual_blocks(int precision, int part, int NE, int Nk, int N, const double* eps, const void* h,
                           const void* GR, const void* GL, const void* GG, const void* SR, const void* SL,
                           const void* SG, const void* SLc, double* work, cudaStream_t st);
int launch_residual_reduce(int NE, int Nk, double* work, double* out5, cudaStream_t st);
int launch_eigvals(int n, long long count, const void* A, double* vals, cudaStream_t st);
size_t observables_partial_doubles(int N);
int launch_observables(int precision, int NE, int Nk, int N, const double* wE, const double* wk, const void* SG,
                       const void* SL, const void* GL, const void* GG, int gs, double target, double* partial,
                       double* out, cudaStream_t st);
int launch_seed_weights(int precision, int NE, int Nk, int N, const void* GR, const double* wE, const double* wk,
                        int gs, double* q, cudaStream_t st);
int launch_seed_green(int precision, int NE, int Nk, int N, const void* GR, const double* f, void* GL, void* GG,
                      cudaStream_t st);
int launch_residual_pair(int precision, size_t n, const void* o1, const void* o2, const void* n1, const void* n2,
                         double* partial, double* out2, cudaStream_t st);
int launch_convert(int precision, size_t n, const void* in_c128, void* out, cudaStream_t st);
// tangent of the SCBA map (tangent.cu)
int launch_block_triple(int NE, int Nk, int N, const void* A, const void* B, const void* C, int adjC, double alpha,
                        double beta, void* out, void* trace, cudaStream_t st);
int launch_norm_tangent(size_t n, const void* Ln, const void* Gn, const double* coeffs, const double* dtrL,
                        const double* dtrG, int gs, double target, int branch, double* dcoef, void* dL, void* dG,
                        cudaStream_t st);
int launch_promote(size_t n, const void* in_c64, void* out_c128, cudaStream_t st);
int launch_antihermitian_part(int NE, int Nk, int N, void* X, cudaStream_t st);

}  // namespace qcl
