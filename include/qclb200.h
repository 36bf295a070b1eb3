/*
 * qclb200 -- C ABI of the B200 (sm_100a) SCBA hot path for QCLNEGF.jl.
 *
 * Every entry point returns an int status (QCL_OK on success); the message of
 * the last failure on the calling thread is available from qcl_last_error().
 * The Julia shim maps the codes to the reference's exceptions exactly as the
 * reference maps LAPACK's `info` (numerics/optimized/production_operators.jl:
 * 39-61): QCL_SINGULAR -> SingularException, QCL_DOMAIN -> DomainError,
 * QCL_DIM -> DimensionMismatch, QCL_ARG -> ArgumentError, QCL_NONFINITE ->
 * the :nonfinite_metrics status (numerics/optimized/production_solver.jl:
 * 624-656).
 *
 * Array convention (all entry points): the reference's Julia layout.  A field
 * is a column-major (N_E, N_k, N_b, N_b) array of complex numbers stored as
 * interleaved (re, im) pairs, energy fastest: element (e, m, a, b) (0-based)
 * is at e + N_E*(m + N_k*(a + N_b*b)).  h is (N_k, N_b, N_b) complex128.
 * Matrices are column-major.  `precision` selects the storage/arithmetic:
 *   QCL_C128  complex128 fields, FP64 arithmetic (the reference's precision);
 *   QCL_C64   complex64 fields, FP32 arithmetic;
 *   QCL_MIXED complex64 fields, FP64 Dyson inversion, FP32 products,
 *             FP64 reductions.
 * Host-buffer entry points (qcl_<name>) take host pointers, copy in, compute
 * and copy out; device entry points (qcl_dev_<name>) take device pointers and
 * a cudaStream_t (NULL = legacy default stream) and are asynchronous.
 */
#ifndef QCLB200_H
#define QCLB200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define QCL_OK 0
#define QCL_SINGULAR 1
#define QCL_DOMAIN 2
#define QCL_DIM 3
#define QCL_ARG 4
#define QCL_NONFINITE 5
#define QCL_TIMEOUT 6
#define QCL_CUDA 7
#define QCL_NOMEM 8
#define QCL_UNSUPPORTED 9

#define QCL_KERNEL_MOMENTUM_INDEPENDENT 0
#define QCL_KERNEL_DENSE 1
#define QCL_KERNEL_IFR 2
#define QCL_KERNEL_LOW_RANK 3
#define QCL_KERNEL_SEPARABLE_SUM 4

#define QCL_C128 0
#define QCL_C64 1
#define QCL_MIXED 2

/* Library version (major*10000 + minor*100 + patch). */
int qcl_version(void);
/* Message of the last failing call on this thread ("" if none). */
const char* qcl_last_error(void);
/* The k of the last QCL_SINGULAR failure on this thread: 0 for a block whose
 * row-sum scale is zero or non-finite, else the 1-based index of the first
 * zero pivot of the block's partial-pivoting elimination (LAPACK getrf's
 * info) -- the argument of the reference's SingularException(k)
 * (numerics/optimized/production_operators.jl:39, 94, 1372). */
int qcl_last_singular_pivot(void);
/* Largest supported basis size N_b. */
int qcl_max_basis(void);

/* ------------------------------------------------------------------------ */
/* Operator level                                                           */
/* ------------------------------------------------------------------------ */

/* Batched retarded Dyson solve and raw Keldysh products.
 * Replaces retarded_green (numerics/reference/greens.jl:18-42) /
 * _retarded_green_production (numerics/optimized/production_operators.jl:
 * 1337-1385) fused with keldysh_green (greens.jl:67-75) and the sandwiches of
 * _current_green_production (numerics/optimized/production_state.jl:23-48).
 * GR = inv(D/s)/s, D = (eps+i eta)I - h - sigR, s = max row sum |D|;
 * GL = GR sigL GR^H; GG = GR sigG GR^H.  sigL/sigG/GR/GL/GG/scale/traceL/
 * traceG may be NULL (the matching product or output is skipped).  scale is
 * (N_E, N_k) float64; traceL/traceG are (N_E, N_k) complex128 raw block
 * traces (unweighted).  A singular block returns QCL_SINGULAR. */
int qcl_dyson_keldysh(int precision, int NE, int Nk, int Nb, const double* eps, double eta, const void* h,
                      const void* sigR, const void* sigL, const void* sigG, void* GR, void* GL, void* GG,
                      double* scale, void* traceL, void* traceG);
int qcl_dev_dyson_keldysh(void* stream, int precision, int NE, int Nk, int Nb, const double* eps, double eta,
                          const void* h, const void* sigR, const void* sigL, const void* sigG, void* GR, void* GL,
                          void* GG, double* scale, void* traceL, void* traceG, int* status);

/* Weighted trace sum  sum_{e,m} wE_e wk_m tr_em  in FP64 with a fixed
 * reduction order; out = (re, im).  Replaces the sum of
 * _number_functional_production (production_operators.jl:1417-1445). */
int qcl_dev_weighted_trace(void* stream, int NE, int Nk, const void* trace, const double* wE, const double* wk,
                           double* out);

/* Paired number normalisation, in place on device fields:
 * GL <- a GL - c GG,  GG <- (1-c) GG - (1-a) GL  with (a, c, lambda) from
 * _paired_number_coefficients (numerics/reference/greens.jl:155-185) applied
 * as in production_state.jl:62-70.  coeffs = device double[3] (a, c, lambda)
 * produced by qcl_dev_paired_coefficients. */
int qcl_dev_paired_coefficients(void* stream, const double* trL, const double* trG, int gs, double target,
                                double* coeffs, int* status);
int qcl_dev_normalize_pair(void* stream, int precision, size_t n, void* GL, void* GG, const double* coeffs);

/* Zero-padded linear-convolution Hilbert transform of the columns of an
 * (N_E, ncols) complex array: Lam_e = sum_{e'!=e} wE_e' Gam_e' /
 * (2 pi (eps_e - eps_e')) on a uniform grid, through FFTs of length
 * L = nextpow2(2 N_E - 1).  Replaces fft_hilbert_transform /
 * production_fft_hilbert_transform (production_operators.jl:793-809,
 * numerics/optimized/fft_parallel.jl:266-291).  If roundoff != NULL the
 * transform is repeated at length 2L and ||Lam_2L - Lam_L||/(||Lam_L||+1e-14)
 * is returned there (fft_parallel.jl:279-290). */
int qcl_fft_hilbert_transform(int precision, int NE, size_t ncols, const double* eps, const double* wE,
                              const void* Gam, void* Lam, double* roundoff);

/* Device variant (asynchronous on `stream`): de is the uniform energy
 * spacing, wE a device array.  If roundoff_sums != NULL it receives (device,
 * 2 doubles) sum |Lam_2L - Lam_L|^2 and sum |Lam_L|^2.  Lam may be Gam (in
 * place). */
int qcl_dev_fft_hilbert_transform(void* stream, int precision, int NE, size_t ncols, double de, const double* wE,
                                  const void* Gam, void* Lam, double* roundoff_sums);

/* Retarded self-energy from the Keldysh components: Gam = i (SG - SL),
 * SR = H[Gam] - i Gam/2 (retarded_self_energy_fft / _retarded_self_energy_
 * fft_production, production_operators.jl:811-884).  Gam may be NULL. */
int qcl_retarded_self_energy(int precision, int NE, size_t ncols, const double* eps, const double* wE,
                             const void* SL, const void* SG, void* SR, void* Gam, double* roundoff);

/* Non-periodic two-point energy shift X(eps + delta) of the columns of an
 * (N_E, ncols) array, zero outside the window.  Replaces build_shift_plan +
 * apply_energy_shift! (numerics/optimized/production_cache.jl:258-325). */
int qcl_apply_energy_shift(int precision, int NE, size_t ncols, const double* eps, double delta, const void* X,
                           void* Y);

/* One factorised scattering-kernel operator (the AbstractProductionKernel
 * subtypes of numerics/optimized/production_contracts.jl:262-323, built by
 * production_cache.jl:387-448).  Arrays are complex128, column-major:
 *   QCL_KERNEL_MOMENTUM_INDEPENDENT  block  (N^2, N^2), rows (a,b), cols (c,d)
 *   QCL_KERNEL_DENSE                 matrix (Nk N^2)^2, rows (m,a,b), cols (m',c,d)
 *   QCL_KERNEL_IFR                   left (N^2, J), right (J, N^2), radial (Nk, Nk)
 *   QCL_KERNEL_LOW_RANK              left (Nk N^2, J), right = right_adjoint (J, Nk N^2),
 *                                    J = rank >= 1 (LowRankProductionKernel, built by
 *                                    _low_rank_production_kernel, production_cache.jl:348-385)
 *   QCL_KERNEL_SEPARABLE_SUM         radial (Nk, Nk, J), block (N^2, N^2, J) -- rows (a,b),
 *                                    cols (c,d) per term: K(m,m') = sum_i radial_i(m,m') block_i,
 *                                    J >= 1 terms.  The Kronecker-sum form of the
 *                                    momentum-dependent kernels: the exact LO kernel
 *                                    sum_h R_h(m,m') F_h (x) conj F_h (lo_phonon_kernel,
 *                                    numerics/reference/kernels.jl:321-356) and the tabulated
 *                                    kernels sum_t W_t(m,m') C(q_t) (numerics/optimized/
 *                                    kernels.jl:303-320) are such sums; a host-side
 *                                    compression keeps J small.  The SeparableIFR operator
 *                                    (production_operators.jl:467-533) is the J = 1 case.
 *                                    The contraction costs 8 J N_k N^4 N_E real flop per map
 *                                    against 8 N_k^2 N^4 N_E for the dense matrix, and the
 *                                    operator holds (N_k^2 + N^4) J entries instead of
 *                                    (N_k N^2)^2.
 * q is the kernel scale q^K; is_LO selects the phonon-shifted contraction in
 * the SCBA loop. */
typedef struct qcl_mechanism {
  int kind;
  int is_LO;
  int J;
  double q;
  const void* block;
  const void* matrix;
  const void* left;
  const void* right;
  const void* radial;
} qcl_mechanism;

/* S = beta S + alpha q K[wk G]: production_static_contraction /
 * _production_static_contraction! (production_operators.jl:402-722). */
int qcl_static_contraction(int precision, const qcl_mechanism* op, int NE, int Nk, int Nb, const double* wk,
                           double alpha, double beta, const void* G, void* S);

/* Shifted sandwich S(e) = T G(eps_e + delta) T^H for one field:
 * _embedding_component_production (production_operators.jl:886-922). */
int qcl_embedding_component(int precision, int NE, int Nk, int Nb, const double* eps, double delta, const void* T,
                            const void* G, void* S);

/* Fixed-point residual suite, out = (r_D, r_A, r_K, r_PSD, r_caus):
 * production_residual_suite (numerics/optimized/residuals.jl:537-770).
 * SR/SL/SG are the current totals, SLc the candidate total lesser. */
int qcl_residual_suite(int precision, int NE, int Nk, int Nb, const double* eps, const void* h, const void* GR,
                       const void* GL, const void* GG, const void* SR, const void* SL, const void* SG,
                       const void* SLc, double* out);

/* The condition_number and dyson_scale fields of GreenState
 * (domain/types.jl:733-740) for a Dyson solve: per block D = (eps + i eta) I
 * - h - SR, kappa = cond_2(D) = ||D||_2 ||D^-1||_2 (LAPACK cond via SVD in
 * retarded_green, numerics/reference/greens.jl:38, and
 * _retarded_green_production, production_operators.jl:1379) and the
 * row-sum scale s.  GR must be the Dyson output for the same inputs (it is
 * D^-1); SR may be NULL (zero); kappa / scale are (N_E, N_k) float64, either
 * may be NULL. */
int qcl_condition_number(int precision, int NE, int Nk, int Nb, const double* eps, double eta, const void* h,
                         const void* SR, const void* GR, double* kappa, double* scale);

/* A = i (GR - GR^H) per block: spectral_function (numerics/reference/
 * greens.jl:50-57), the A field written by _green_state_production
 * (production_operators.jl:1387-1415). */
int qcl_spectral_function(int precision, int NE, int Nk, int Nb, const void* GR, void* A);

/* Dense kernel operators assembled on the device from angular node weights.
 * The reference's momentum-dependent kernels are angular averages over
 * phi_r = 2 pi (r-1) / N_phi of a transfer-momentum kernel C(q) (the exact
 * LO phonon kernel, lo_phonon_kernel, numerics/reference/kernels.jl:321-356;
 * the tabulated lookup of numerics/optimized/kernels.jl:205-217, 303-320),
 * which makes K(m,m') = sum_t W[(m,m'),t] X_t for node weights W (host-formed
 * angular means, N_k^2 x T, column-major, (m,m') index m + N_k m') and node
 * tensors X_t:
 *   QCL_ASSEMBLE_RANK1: X_t = F_t (x) conj(F_t), X = F (T x N_b^2 complex128,
 *                       F[t + T (a + N_b c)]);
 *   QCL_ASSEMBLE_TABLE: X_t the (N_b^2 x N_b^2) pair covariance at table node t,
 *                       X[(a + N_b c) + N_b^2 (b + N_b d) + N_b^4 t].
 * Output: the production dense matrix (rows (m,a,b), columns (m',c,d);
 * _production_kernel, production_cache.jl:400-405) normalised by
 * qK = max |K| (build_kernels, kernels.jl:393-403); a zero or non-finite
 * kernel is left unnormalised and reported through qK. */
#define QCL_ASSEMBLE_RANK1 0
#define QCL_ASSEMBLE_TABLE 1
int qcl_assemble_kernel(int form, int Nk, int Nb, int T, const double* W, const void* X, void* matrix, double* qK);
/* Device-array variant on `stream`; work holds (296 + 1) doubles and receives
 * qK in its last entry. */
int qcl_dev_assemble_kernel(void* stream, int form, int Nk, int Nb, int T, const double* W, const void* X,
                            void* matrix, double* work);

/* Integrated coherences rho_ab = sum_{m,e} wE_e wk_m G<_{e,m,a,b} (Nb x Nb,
 * complex128, column-major): the `integrated` matrix of
 * _electron_density_bar (physics/observables.jl:1-22) from which the outer
 * Poisson loop forms n(z) = g_s/(2 pi) Re(-i chi(z) rho chi(z)^H)
 * (production_solver.jl:1043). */
int qcl_density_matrix(int precision, int NE, int Nk, int Nb, const double* wE, const double* wk, const void* GL,
                       void* rho);

/* Eigenvalues (unsorted) of `count` Hermitian n x n matrices stored back to
 * back (column-major complex128; the Hermitian part is used), n <= 48.
 * Replaces the per-block LAPACK zheev calls of the residual suite
 * (_production_hermitian_eigvals!, numerics/optimized/residuals.jl:311-353). */
int qcl_hermitian_eigvals(int n, size_t count, const void* H, double* vals);

/* The positivity witness of a residual-suite evaluation (_PositivityWitness,
 * numerics/reference/positivity_diagnostics.jl:41-91): over the blocks in the
 * reference's order (e slow, m fast) and the six matrices in kind order, the
 * first with the largest ratio (production_residual_suite, residuals.jl:
 * 662-726; _production_positivity_witness, :773-779).  matrix_kind: -1 none,
 * 0 spectral A, 1 occupied -iG<, 2 unoccupied iG>, 3 broadening Gamma,
 * 4 raw occupied -i G S< G^H, 5 raw unoccupied i G S> G^H; indices 0-based. */
typedef struct qcl_psd_witness {
  int matrix_kind;
  int energy_index;
  int momentum_index;
  double minimum_eigenvalue, block_norm, floor, ratio, absolute_defect, relative_defect, backward_error,
      hermiticity_defect, construction_scale;
} qcl_psd_witness;

/* qcl_residual_suite plus its positivity witness. */
int qcl_residual_suite_witness(int precision, int NE, int Nk, int Nb, const double* eps, const void* h,
                               const void* GR, const void* GL, const void* GG, const void* SR, const void* SL,
                               const void* SG, const void* SLc, double* out, qcl_psd_witness* witness);

/* Allocation-free residual suite on device arrays (no counterpart in the
 * reference).  For callers that cannot call cudaMalloc -- a host whose
 * device memory belongs to its own pool allocator, a fixed up-front device
 * budget, or a loop that must not risk the synchronisation of an allocation.
 * Same result as qcl_residual_suite (out: 5 doubles in device memory, written
 * asynchronously on `stream`); the per-block scratch is a fixed device array
 * of the library (about 18.9 MB per GPU, held until exit), so N_E * N_k must
 * not exceed 262144 (QCL_UNSUPPORTED otherwise).  Calls share that array:
 * calls that overlap on the GPU race.  The first call on a device looks up
 * the array's address on that device; make it before any stream capture.
 * After a device reset (cudaDeviceReset) that address is stale: do not call
 * the entry point again in that process. */
int qcl_dev_residual_suite_noalloc(void* stream, int precision, int NE, int Nk, int Nb, const double* eps,
                                   const void* h, const void* GR, const void* GL, const void* GG, const void* SR,
                                   const void* SL, const void* SG, const void* SLc, double* out);

/* out = ||new - old||_F / (||new||_F + 1e-14) for one component
 * (production_selfenergy_residual, residuals.jl:802-865). */
int qcl_selfenergy_residual(int precision, size_t n, const void* old_, const void* new_, double* out);

/* Boundary flux and populations: out[0] = Jbar (solver units,
 * _production_boundary_flux_bar, production_iteration.jl:174-201),
 * out[1] = imaginary part of the complex flux (diagnostic), out[2 + a] =
 * population p_a (_production_state_populations, :204-215).  SG/SL are the
 * plus-embedding family components. */
int qcl_current_populations(int precision, int NE, int Nk, int Nb, const double* wE, const double* wk, int gs,
                            double target, const void* SG, const void* SL, const void* GL, const void* GG,
                            double* out);

/* ------------------------------------------------------------------------ */
/* SCBA level: one device-resident production cache + state per context    */
/* ------------------------------------------------------------------------ */

/* The inputs solve_scba_production consumes at fixed Hartree potential
 * (numerics/optimized/production_solver.jl:21-846), in solver units
 * (domain/scaling.jl:10-110).  eps is uniform (FFT Hilbert); Tminus =
 * Tplus^H (numerics/reference/basis.jl:56-57). */
typedef struct qcl_scba_problem {
  int NE, Nk, Nb;
  const double* eps;
  const double* wE;
  const double* wk;
  const void* h;      /* (Nk, Nb, Nb) complex128 */
  const void* Tplus;  /* (Nb, Nb) complex128 */
  const void* Tminus; /* (Nb, Nb) complex128 */
  double Ep;          /* period energy drop F L_p */
  double hw_LO;       /* LO phonon energy */
  double N_LO;        /* thermal LO occupation */
  int gs;             /* spin degeneracy */
  double target;      /* sheet doping N_D in solver units */
  double eta_seed;    /* seed broadening */
  double kBT;         /* lattice temperature in solver units */
  double alpha;       /* linear mixing factor in (0, 1] */
  double J0;          /* current unit in A/m^2 */
  int precision;      /* QCL_C128 / QCL_C64 / QCL_MIXED */
  int verify_roundoff;/* repeat each Hilbert transform at 2L */
  int nmech;          /* number of mechanisms, in _SCATTERING_MECHANISM_ORDER */
  /* Model switches of AlgorithmOptions (algorithm_options.jl:19-39; checked
   * as in _check_algorithm_options, :42-93), applied to every scattering
   * candidate; 0 is the reference default.
   *   self_energy_structure 0 :full, 1 :diagonal -- off-diagonal entries
   *     zeroed (_diagonalize_blocks!, production_operators.jl:1208-1217);
   *   transverse_momentum 0 :resolved, 1 :averaged -- wk-weighted mean over
   *     k, sum(wk) > 0 required (_average_transverse_momentum!, :1219-1238);
   *   retarded_real_part 0 :kramers_kronig, 1 :drop -- Sigma^R = -i Gamma/2,
   *     no Hilbert transform (_retarded_self_energy_selected, :1174-1177);
   *   elastic_retarded 0 :hilbert, 1 :direct_green -- Sigma^R = K[G^R] for
   *     the elastic (non-LO) mechanisms unless the real part is dropped
   *     (_scattering_candidate_production, :1306-1311); a truncated low-rank
   *     operator is rejected with it, as the reference rejects the pair. */
  int self_energy_structure;
  int transverse_momentum;
  int retarded_real_part;
  int elastic_retarded;
  /* occupation_normalization 0 :paired_convex (_normalize_keldysh_pair!),
   * 1 :scalar_lesser -- G< / lambda and G> = G^R - G^A + G<
   * (production_state.jl:54-61). */
  int occupation_normalization;
  /* mixing 0 :linear (alpha), 1 :anderson -- bounded-history Anderson
   * acceleration with the exact causality guard and its linear fallback
   * (_anderson_mix!, numerics/optimized/production_mixing.jl:224-317); the
   * three parameters as in AlgorithmOptions (depth 1..8 here; the reference
   * defaults are 5, 1.0, 1e-12). */
  int mixing;
  int anderson_history_depth;
  double anderson_damping;
  double anderson_regularization;
  /* Execution budget of the memory preflight in bytes (ProductionOptions.
   * memory_budget_bytes, production_contracts.jl:143-165); 0 = the device's
   * free memory when the context is created.  qcl_scba_create refuses with
   * QCL_NOMEM, before any allocation, when the estimated peak exceeds it
   * (build_production_cache, numerics/optimized/production_cache.jl:764-770). */
  size_t memory_budget_bytes;
  /* 1: a QCL_C64 / QCL_MIXED context that reserves complex128 fields and
   * keeps complex128 operator copies, so that qcl_scba_promote can finish the
   * solve in FP64 (mixed-precision iterations, then FP64 refinement of the
   * fixed point); 0 otherwise. */
  int refinement;
} qcl_scba_problem;

/* Device-memory estimate of qcl_scba_create (bytes): the SCBA fields (state
 * and candidate families, G, totals, scratch fields), the operators (with the
 * tensor-core operands and refinement copies), the contraction / reduction /
 * FFT workspace, the Anderson history, their sum (resident) and the peak
 * during creation (resident plus the largest complex128 staging copy of an
 * operator array).  The role of _estimate_production_memory
 * (numerics/optimized/production_cache.jl:475-668) for this library's own
 * allocation plan. */
typedef struct qcl_memory_estimate {
  size_t fields, operators, workspace, anderson, resident, peak;
} qcl_memory_estimate;
int qcl_scba_estimate_memory(const qcl_scba_problem* problem, const qcl_mechanism* mechanisms,
                             qcl_memory_estimate* out);

/* Mixer diagnostics of the last step (the metrics _anderson_mix! reports,
 * production_mixing.jl:283-298).  reset_reason: 0 none, 1 residual_increase,
 * 2 coefficient_solve, 3 coefficient_bound, 4 causality_guard;
 * guard_first_failure: 1-based block index (family, e, m; m fastest) of the
 * first guard failure, 0 if none. */
typedef struct qcl_anderson_info {
  int history_depth;
  int reset_reason;
  int acceleration_accepted;
  int fallback;
  int guard_failure_code;
  long long guard_first_failure;
  double coefficients_l1;
} qcl_anderson_info;

/* One SCBAIteration row (domain/types.jl:908).  status: QCL_OK or
 * QCL_NONFINITE (the :nonfinite_metrics exit). */
typedef struct qcl_scba_row {
  int nu;
  int status;
  double r_D, r_A, r_K, r_Sigma, r_lambda, lambda, r_PSD, r_caus, r_roundoff;
  double r_J, r_pop, J, Jbar, number, holes, occupied_fraction, empty_fraction;
  /* SCBAIteration's target_charge, normalized_charge (the number functional
   * of the normalised G<) and lambda_change (NaN on the first row),
   * production_solver.jl:607-610; raw_charge is `number`. */
  double target_charge, normalized_charge, lambda_change;
} qcl_scba_row;

typedef struct qcl_scba qcl_scba;

/* Allocates the device state and uploads grids, h, T+-, shift plans and
 * kernel operators (build_production_cache, production_cache.jl:759-840).
 * The operator arrays of `mechanisms` may be host or device memory (e.g. a
 * dense operator from qcl_dev_assemble_kernel); they are copied. */
int qcl_scba_create(const qcl_scba_problem* problem, const qcl_mechanism* mechanisms, qcl_scba** out);
void qcl_scba_destroy(qcl_scba* ctx);
/* Equilibrium seed + initial candidates (_seed_green_production,
 * numerics/optimized/seed.jl:151-197); mu receives the seed chemical
 * potential. */
int qcl_scba_seed(qcl_scba* ctx, double* mu);
/* One SCBA iteration (production_solver.jl:435-844).  The linear mixing of
 * the iteration is committed when the next step starts, so a caller that
 * stops after reading `row` keeps the unmixed state, as the reference does on
 * a terminal decision. */
int qcl_scba_step(qcl_scba* ctx, qcl_scba_row* row);
/* Up to max_iter steps, stopping early once r_Sigma <= tol_sigma or on a
 * non-finite row; history receives n_done rows. */
int qcl_scba_run(qcl_scba* ctx, int max_iter, double tol_sigma, qcl_scba_row* history, int* n_done);
/* Populations p_a of the last step (N_b doubles). */
int qcl_scba_populations(qcl_scba* ctx, double* out);
/* Checkpoint / warm start.  which: 0, 1, 2 = GR, G<, G> of the last step;
 * 3 + 3 f + c = family f (0..nmech-1 mechanisms, nmech plus, nmech+1 minus),
 * component c (0 R, 1 <, 2 >) of the current state. */
int qcl_scba_download(qcl_scba* ctx, int which, void* host);
int qcl_scba_upload(qcl_scba* ctx, int which, const void* host);
/* A new operating point of a bias or temperature sweep on the same context
 * (retarget_problem + retarget_production_cache, composition/
 * operating_point.jl:25-170): the +-Ep shift plans are rebuilt for the new
 * period drop Ep, and the Hartree Hamiltonian h ((Nk, Nb, Nb) complex128),
 * the LO occupation N_LO, kBT and the kernel scales q (nmech doubles, e.g.
 * the acoustic q^K proportional to the lattice temperature) are replaced
 * where given (h, q may be NULL).  Kernel operators, grids and the state stay
 * resident: the next step continues from the last unmixed state (warm
 * start); the row history (r_J, r_pop, lambda_change, nu) restarts. */
int qcl_scba_retarget(qcl_scba* ctx, double Ep, double N_LO, double kBT, const void* h, const double* q);
/* The causality / Keldysh guard of a set of self-energy families
 * (_anderson_guard / _anderson_block_failure!, numerics/optimized/
 * production_mixing.jl:48-118): fields = nfam x (SigmaR, Sigma<, Sigma>).
 * first_failure = 1-based index of the first failing block over (family, e,
 * m), m fastest, 0 if all pass; code = the reference's failure code 1..5. */
int qcl_anderson_guard(int precision, int NE, int Nk, int Nb, int nfam, const void* const* fields,
                       long long* first_failure, int* code);
/* qcl_density_matrix of the last Dyson solve (seed or step) of a context. */
int qcl_scba_density_matrix(qcl_scba* ctx, void* rho);
/* Anderson mixer diagnostics of the last step (all zero for linear mixing). */
int qcl_scba_mixer_info(qcl_scba* ctx, qcl_anderson_info* info);
/* FP64 refinement: switches a context created with refinement = 1 from
 * QCL_C64 / QCL_MIXED to QCL_C128 for the steps that follow.  The current
 * state (with the last step's mixing committed) is converted exactly to
 * complex128 and the next step continues from it; operators switch to their
 * complex128 copies; the Anderson history restarts, and its causality guard
 * keeps budgets at the FP32 roundoff the converted state carries (at FP64
 * roundoff nearly every block of it would fail).  The scheme "FP32 bulk,
 * FP64 refinement of the fixed point": iterate in mixed precision
 * until r_Sigma reaches its FP32 floor, then converge in FP64 (no reference
 * counterpart: the reference has no reduced precision,
 * application/algorithm_registry.jl:226-240).  QCL_ARG if the context was
 * not created for refinement; a no-op on a QCL_C128 context. */
int qcl_scba_promote(qcl_scba* ctx);
/* Phase telemetry (the :phase_begin / :phase_end SolverEvents of
 * ProductionOptions.phase_timing, application/production_telemetry.jl:81-200,
 * emitted at production_solver.jl:438-590 and production_iteration.jl:1-65):
 * with telemetry on, CUDA events at the phase boundaries of every iteration
 * (event-record nodes inside a captured graph) give the device time of each
 * phase.  qcl_scba_phase_times writes the last step's times in milliseconds
 * for the QCL_PHASES phases in this order -- dyson, candidate_scattering,
 * candidate_embedding, candidate_assembly, residuals, observables, mixing --
 * and the last seed's :initialization time.  Phases run back to back on the
 * context's stream except that the G-only part of the residual suite runs on
 * a side stream during the candidate phases; "residuals" is the time from the
 * candidate total to the end of the reduction. */
#define QCL_PHASES 7
int qcl_scba_use_telemetry(qcl_scba* ctx, int enable);
int qcl_scba_phase_times(qcl_scba* ctx, double* ms, double* initialization_ms);
/* Replay each iteration as one captured CUDA graph (default off). */
int qcl_scba_use_graph(qcl_scba* ctx, int enable);
/* The derived GreenState fields of the last Dyson solve (seed or step) --
 * A (a field in the context's storage precision), condition_number and
 * dyson_scale ((N_E, N_k) float64) -- as _green_state_production returns
 * them (production_operators.jl:1387-1415).  Any output may be NULL. */
int qcl_scba_green_state(qcl_scba* ctx, void* A, double* kappa, double* scale);
/* The positivity witness of the last step's residual suite (the witness of
 * its SCBAIteration row, production_solver.jl:611-619), valid until the next
 * step or seed. */
int qcl_scba_witness(qcl_scba* ctx, qcl_psd_witness* witness);

/* Implicit differentiation of the converged SCBA (tangent mode; the
 * reference has no derivatives).  At the state of the last step -- a fixed
 * point Sigma_fp = Phi(Sigma_fp, p) once converged -- the derivative
 * v of Sigma_fp with respect to p solves v = Phi_Sigma v + Phi_p (the implicit-function
 * theorem), and dJ/dp = J_Sigma v + J_p.  qcl_scba_tangent_init allocates the
 * tangent fields (complex128 context, linear mixing, paired normalisation);
 * qcl_scba_tangent_set uploads a component of the source Phi_p (which as in
 * qcl_scba_download; host NULL zeroes it; which = -1 zeroes v);
 * qcl_scba_tangent_step does one damped step v <- (1 - alpha) v +
 * alpha (Phi_Sigma v + Phi_p) with Phi_Sigma v from the linearised Dyson,
 * Keldysh and normalisation steps and the (linear) candidate maps, and writes
 * out[0] = J_Sigma v (solver units, J = Jbar J0) and out[1] = the largest
 * relative change of a tangent field.  qcl_scba_download_candidate returns a
 * family field of the last step's mixed candidate (1 - alpha) Sigma +
 * alpha Phi(Sigma), from which a caller forms Phi_p by differences. */
int qcl_scba_tangent_init(qcl_scba* ctx);
int qcl_scba_tangent_set(qcl_scba* ctx, int which, const void* host);
int qcl_scba_tangent_step(qcl_scba* ctx, double* out);
int qcl_scba_download_candidate(qcl_scba* ctx, int which, void* host);
/* The form of the paired number normalisation (_paired_number_coefficients,
 * numerics/reference/greens.jl:155-199): the reference scales G< when the
 * raw number is at or above the target (form 1) and otherwise moves G>
 * weight into G< (form 2).  A particle-conserving fixed point sits on that
 * switch, so the explicit part Phi_p of a derivative must keep the fixed
 * point's form on both sides of p: qcl_scba_normalization_branch returns
 * the form the last step used (1 or 2) and
 * qcl_scba_set_normalization_branch forces one (0 restores the reference's
 * choice). */
int qcl_scba_set_normalization_branch(qcl_scba* ctx, int branch);
int qcl_scba_normalization_branch(qcl_scba* ctx, int* branch);

/* Batched sweep of independent operating points: a bias sweep, or points of
 * different structures (basis sizes, energy grids).  The reference solves
 * operating points one after another, re-using basis and kernels across
 * biases (retarget_problem + retarget_production_cache, composition/
 * operating_point.jl:25-170).  Here the points that fit the memory budget
 * together (each point's qcl_scba_estimate_memory peak; 0 = the device's
 * free memory) are resident at once, and one iteration of all resident
 * points is one CUDA graph launch whose child graphs (the points' captured
 * iterations) run concurrently.  A point leaves when r_Sigma <= tol_sigma, on
 * a failure or non-finite row, or after max_iter steps, and the next pending
 * point takes its memory.  qcl_sweep_create copies the problem and mechanism
 * structs (not the arrays they point to, which must stay valid until
 * qcl_sweep_run returns).  qcl_sweep_run fills, per point, its last row and
 * its iteration count; stats (may be NULL) receives 5 doubles: wall seconds,
 * total iterations, graph launches, largest number of resident points,
 * parent-graph builds. */
typedef struct qcl_sweep qcl_sweep;
int qcl_sweep_create(int npoints, const qcl_scba_problem* problems, const qcl_mechanism* const* mechanisms,
                     size_t memory_budget_bytes, qcl_sweep** out);
int qcl_sweep_run(qcl_sweep* sweep, int max_iter, double tol_sigma, qcl_scba_row* last_rows, int* iterations,
                  double* stats);
void qcl_sweep_destroy(qcl_sweep* sweep);

/* Autotuner (the reference sets the analogous execution knobs by hand:
 * ProductionOptions.energy_chunk / hilbert_columns / worker_count,
 * numerics/optimized/production_contracts.jl:143-165).  qcl_autotune times
 * every compiled CTA shape of the Dyson + Keldysh kernel -- the number of
 * (E, k) blocks per CTA, which sets threads, shared memory and registers per
 * CTA -- for one basis class (N_b padded to 8, 16, 24, 32 or 48) and
 * precision on a synthetic NE x Nk batch; every later Dyson launch of that
 * class in the process uses the fastest.  qcl_autotune_reset restores the
 * built-in choices; qcl_tuned_dyson_bpc reports the one in use. */
typedef struct qcl_tune_result {
  int dyson_bpc;   /* chosen blocks per CTA */
  int default_bpc; /* the built-in choice */
  int candidates;  /* number of candidates timed */
  int bpc[4];      /* the candidates */
  float ms[4];     /* mean device time per launch of each candidate */
} qcl_tune_result;
int qcl_autotune(int precision, int Nb, int NE, int Nk, qcl_tune_result* out);
int qcl_autotune_reset(void);
int qcl_tuned_dyson_bpc(int precision, int Nb);

/* Test hook (no counterpart in the reference): the number of polling rounds
 * after which a main-loop wait of the tensor-core contraction kernel gives up
 * on the current device (0: at once; negative: the default, about 1 s).  A
 * wait that gives up records QCL_TIMEOUT in the call's status; the kernel then
 * waits with the full limit for its copies and MMAs in flight, frees its
 * tensor memory and returns, so the context stays usable. */
int qcl_debug_set_wait_limit(long long rounds);

#ifdef __cplusplus
}
#endif

#endif /* QCLB200_H */
