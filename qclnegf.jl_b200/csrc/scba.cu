// Device-resident SCBA inner loop (the production cache + state + iteration).
//
// Reference: solve_scba_production (numerics/optimized/production_solver.jl:
// 21-846; loop body :435-844) and the educational solve_scba
// (numerics/reference/scba.jl:142-354).  One iteration nu:
//   1. total = plus + minus + sum_mech                (_total_family_production)
//   2. GR, G<, G> = Dyson + Keldysh(total); paired number normalisation
//                                                       (_current_green_production)
//   3. candidate scattering families (contractions, LO shifts, FFT Hilbert
//      with roundoff verification)                      (_scattering_candidate_production)
//   4. candidate embedding families (shifted sandwiches)
//   5. residual suite and r_Sigma                       (_production_fixed_point_measurement)
//   6. J, populations                                   (_production_observable_measurement)
//   7. mixing (linear), committed only if the caller continues
// Every field stays in HBM; each iteration reads back one small block of
// scalars (residuals, J, populations, lambda) to the host, which applies the
// reference's termination policy.  The whole launch sequence of an
// iteration can be captured once into a CUDA graph and replayed.
#include <math.h>
#include <string.h>

#include <algorithm>
#include <chrono>
#include <map>
#include <vector>

#include "kernels.cuh"

namespace qcl {

struct DevShift {
  int* left = nullptr;
  int* right = nullptr;
  double* theta = nullptr;
  unsigned char* valid = nullptr;
  ShiftPlanDev view() const { return ShiftPlanDev{left, right, theta, valid}; }
};

struct Mech {
  int kind = 0, is_LO = 0, J = 0;
  double q = 0;
  void* block = nullptr;
  void* matrix = nullptr;
  void* left = nullptr;
  void* right = nullptr;
  void* radial = nullptr;
  void* tc_bop = nullptr;  // dense operator prepared for the tensor cores (complex64 fields)
  // complex128 copies of the operator arrays (refinement contexts): swapped in by promote
  void *block64 = nullptr, *matrix64 = nullptr, *left64 = nullptr, *right64 = nullptr, *radial64 = nullptr;
  std::vector<void*> tc_chunks;  // separable sum: tensor-core operand per term chunk (complex64 fields)
  std::vector<void*> tc_stage1;  // separable sum: stage-1 operand per term chunk
  int* status = nullptr;
  KernelOpDev view() const {
    KernelOpDev k;
    k.tc_bop = tc_bop;
    k.tc_chunks = tc_chunks.empty() ? nullptr : tc_chunks.data();
    k.tc_stage1 = tc_stage1.size() == tc_chunks.size() && !tc_stage1.empty() ? tc_stage1.data() : nullptr;
    k.status = status;
    k.kind = kind;
    k.J = J;
    k.block = block;
    k.matrix = matrix;
    k.left = left;
    k.right = right;
    k.radial = radial;
    return k;
  }
};

// Device scalar block layout (doubles), downloaded once per iteration.
enum {
  SC_TRL = 0,      // 2: sum wE wk tr G<  (raw)
  SC_TRG = 2,      // 2: sum wE wk tr G>
  SC_COEF = 4,     // 5: a, c, lambda, N, H
  SC_RES = 9,      // 5: rD, rA, rK, rPSD, rcaus
  SC_EMB = 14,     // 6: embedding-total residual (num, den) x 3 components
  SC_OBS = 20,     // 2 + N: Jbar, Im, populations
  SC_FAM = 20 + 2 + 48,  // (M + 2) families x 3 components x (num, den)
  SC_ROUND = SC_FAM + 7 * 3 * 2,  // M x (num, den) Hilbert roundoff
  SC_TOTAL = SC_ROUND + 5 * 2
};

// Phases of an iteration, in the reference's names (production_solver.jl:438-590,
// production_iteration.jl:1-65): dyson, candidate_scattering, candidate_embedding,
// candidate_assembly, residuals, observables, mixing.
constexpr int kPhases = 7;

struct ScbaCtx {
  int NE, Nk, N, M, precision, gs, verify;
  int refinement = 0;  // FP64-sized state and complex128 operator copies for qcl_scba_promote
  // unit roundoff of the Anderson guard's budgets when above the storage
  // precision's (a promoted state keeps the FP32 rounding it was made with)
  double guard_roundoff = 0.0;
  int diagonal = 0, averaged = 0, drop_real = 0, direct_green = 0;  // scattering-model switches
  int scalar_lesser = 0;                                             // occupation_normalization
  int norm_branch = 0;  // paired normalisation form: 0 the reference's choice, 1 / 2 forced
  // Anderson mixing (mixing = :anderson): device history and mixer state
  int mixing = 0, and_depth = 5;
  double and_damping = 1.0, and_reg = 1e-12;
  void *Xh = nullptr, *Rh = nullptr;
  AndersonMeta* ameta = nullptr;
  AndersonMeta* ameta_h = nullptr;  // pinned copy, read after each step
  double* apartial = nullptr;
  double wk_sum = 0;
  double Ep, hw_LO, N_LO, target, eta_seed, kBT, alpha, J0;
  double de = 0;  // uniform energy spacing (FFT tables)
  size_t nfield, fbytes;  // elements per field, bytes per field at the active precision
  size_t fcap = 0;        // allocated bytes per field (complex128 size in refinement contexts)
  cudaStream_t st = nullptr;
  // grids and operators
  double *eps = nullptr, *wE = nullptr, *wk = nullptr;
  void *h = nullptr, *Tp = nullptr, *Tm = nullptr;
  std::vector<double> eps_h, wE_h;
  DevShift shift[4];  // +Ep, -Ep, +LO, -LO
  std::vector<Mech> mech;
  // fields: family f (0..M-1 mechanisms, M plus, M+1 minus), component c (R,<,>)
  std::vector<void*> state, cand;  // (M+2)*3 each
  void *GR = nullptr, *GL = nullptr, *GG = nullptr;
  void *tot[3] = {nullptr, nullptr, nullptr};
  void* candSL = nullptr;
  void* tmp = nullptr;
  void* cwork = nullptr;
  size_t cwork_bytes = 0;
  // reductions
  Cx<double>*trL = nullptr, *trG = nullptr;
  double* rpartial = nullptr;
  double* mpartial = nullptr;  // per-field partials of the fused residual + mixing
  double* reswork = nullptr;
  double* obspartial = nullptr;
  double* scal = nullptr;
  double* scal_h = nullptr;  // pinned
  int* status = nullptr;
  HilbertTables hil;
  // graph of one iteration (two parities: state/cand swap)
  cudaGraphExec_t graph[2] = {nullptr, nullptr};
  cudaGraph_t gtpl[2] = {nullptr, nullptr};  // the captured iterations (child graphs of a batched sweep)
  cudaStream_t st2 = nullptr;  // side stream of an iteration (forked from st, joined back)
  cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
  bool use_graph = false;
  // phase telemetry: device time between CUDA events at the phase boundaries of an
  // iteration (the :phase_begin / :phase_end events of production_telemetry.jl:81-200)
  bool telemetry = false;
  cudaEvent_t pev[kPhases + 1] = {};
  double phase_ms[kPhases] = {};
  double init_ms = 0;
  // tangent of the fixed point (qcl_scba_tangent_*): v and its update (families),
  // the source Phi_p (families), dG^{R,<,>}, the tangent totals, traces, scalars
  std::vector<void*> tv, tw, tsrc;
  void *tG[3] = {nullptr, nullptr, nullptr}, *ttot[3] = {nullptr, nullptr, nullptr};
  Cx<double>*ttrL = nullptr, *ttrG = nullptr;
  double* tscal = nullptr;  // dtrL (2), dtrG (2), dcoef (2), residual partial sums, J (2 x (2 + N))
  double* tscal_h = nullptr;
  int parity = 0;
  bool pending_commit = false;
  int nu = 0;
  double Jprev = NAN;
  double lam_prev = NAN;
  std::vector<double> pprev, pops;
  bool seeded = false;
  bool have_green = false;  // GR holds the Dyson solution of (eps + i green_eta, h, tot[0])
  bool have_residual = false;  // reswork holds the per-block residual outputs of the last step
  double green_eta = 0;
};

static void* field_of(const std::vector<void*>& v, int f, int c) { return v[3 * f + c]; }
int scba_step_launch(ScbaCtx* c, cudaGraph_t* child);
int scba_step_finish(ScbaCtx* c, qcl_scba_row* row);

static int dalloc(void** p, size_t bytes) {
  cudaError_t e = cudaMalloc(p, bytes > 0 ? bytes : 16);
  if (e != cudaSuccess) return cuda_status(e, "cudaMalloc (SCBA context)");
  return QCL_OK;
}
// Uploads go on the context's stream: the context's kernels run on a
// non-blocking stream, which a plain cudaMemcpy (legacy stream; from pageable
// memory it may return before the DMA has landed) would not order them after.
// The source may be host or device memory (unified addressing picks the
// direction), so operators assembled on the device need no host round trip.
template <typename T> static int dupload(T** p, const void* host, size_t bytes, cudaStream_t st) {
  int s = dalloc((void**)p, bytes);
  if (s) return s;
  QCL_CUDA_CHECK(cudaMemcpyAsync(*p, host, bytes, cudaMemcpyDefault, st));
  QCL_CUDA_CHECK(cudaStreamSynchronize(st));  // the host buffer may be a temporary
  return QCL_OK;
}

// Uploads an operator array in the context's precision; a refinement context
// of reduced precision also keeps the complex128 array (*keep64) for promote.
static int upload_op(ScbaCtx* c, void** dst, const void* host_c128, size_t n, void** keep64 = nullptr) {
  void* tmp = nullptr;
  int s = dupload(&tmp, host_c128, n * 16, c->st);
  if (s) return s;
  if (c->precision == QCL_C128) {
    *dst = tmp;
    return QCL_OK;
  }
  if ((s = dalloc(dst, n * 8))) {
    cudaFree(tmp);
    return s;
  }
  s = launch_convert(c->precision, n, tmp, *dst, c->st);
  cudaStreamSynchronize(c->st);
  if (c->refinement && keep64) *keep64 = tmp;
  else cudaFree(tmp);
  return s;
}

static int build_plan(ScbaCtx* c, DevShift& d, double delta) {
  std::vector<int> l(c->NE), r(c->NE);
  std::vector<double> th(c->NE);
  std::vector<unsigned char> v(c->NE);
  int s = build_shift_plan_host(c->NE, c->eps_h.data(), delta, l.data(), r.data(), th.data(), v.data());
  if (s) return s;
  if ((s = dupload(&d.left, l.data(), c->NE * sizeof(int), c->st))) return s;
  if ((s = dupload(&d.right, r.data(), c->NE * sizeof(int), c->st))) return s;
  if ((s = dupload(&d.theta, th.data(), c->NE * sizeof(double), c->st))) return s;
  return dupload(&d.valid, v.data(), c->NE, c->st);
}

// Rebuilds a shift plan into its existing device arrays.
static int refill_plan(ScbaCtx* c, DevShift& d, double delta) {
  std::vector<int> l(c->NE), r(c->NE);
  std::vector<double> th(c->NE);
  std::vector<unsigned char> v(c->NE);
  int s = build_shift_plan_host(c->NE, c->eps_h.data(), delta, l.data(), r.data(), th.data(), v.data());
  if (s) return s;
  QCL_CUDA_CHECK(cudaMemcpyAsync(d.left, l.data(), c->NE * sizeof(int), cudaMemcpyHostToDevice, c->st));
  QCL_CUDA_CHECK(cudaMemcpyAsync(d.right, r.data(), c->NE * sizeof(int), cudaMemcpyHostToDevice, c->st));
  QCL_CUDA_CHECK(cudaMemcpyAsync(d.theta, th.data(), c->NE * sizeof(double), cudaMemcpyHostToDevice, c->st));
  QCL_CUDA_CHECK(cudaMemcpyAsync(d.valid, v.data(), c->NE, cudaMemcpyHostToDevice, c->st));
  QCL_CUDA_CHECK(cudaStreamSynchronize(c->st));  // the host vectors are temporaries
  return QCL_OK;
}

void scba_destroy(ScbaCtx* c) {
  if (!c) return;
  if (c->st) cudaStreamSynchronize(c->st);
  for (int g = 0; g < 2; ++g)
    if (c->graph[g]) cudaGraphExecDestroy(c->graph[g]);
  for (int g = 0; g < 2; ++g)
    if (c->gtpl[g]) cudaGraphDestroy(c->gtpl[g]);
  cudaFree(c->eps);
  cudaFree(c->wE);
  cudaFree(c->wk);
  cudaFree(c->h);
  cudaFree(c->Tp);
  cudaFree(c->Tm);
  for (auto& d : c->shift) {
    cudaFree(d.left);
    cudaFree(d.right);
    cudaFree(d.theta);
    cudaFree(d.valid);
  }
  for (auto& m : c->mech) {
    cudaFree(m.block);
    cudaFree(m.matrix);
    cudaFree(m.left);
    cudaFree(m.right);
    cudaFree(m.radial);
    cudaFree(m.tc_bop);
    for (void* q : m.tc_chunks) cudaFree(q);
    for (void* q : m.tc_stage1) cudaFree(q);
    for (void* q : {m.block64, m.matrix64, m.left64, m.right64, m.radial64}) cudaFree(q);
  }
  for (void* p : c->state) cudaFree(p);
  for (void* p : c->cand) cudaFree(p);
  for (auto* v : {&c->tv, &c->tw, &c->tsrc})
    for (void* p : *v) cudaFree(p);
  for (int k = 0; k < 3; ++k) {
    cudaFree(c->tG[k]);
    cudaFree(c->ttot[k]);
  }
  cudaFree(c->ttrL);
  cudaFree(c->ttrG);
  cudaFree(c->tscal);
  if (c->tscal_h) cudaFreeHost(c->tscal_h);
  cudaFree(c->GR);
  cudaFree(c->GL);
  cudaFree(c->GG);
  for (auto p : c->tot) cudaFree(p);
  cudaFree(c->candSL);
  cudaFree(c->tmp);
  cudaFree(c->cwork);
  cudaFree(c->trL);
  cudaFree(c->trG);
  cudaFree(c->rpartial);
  cudaFree(c->mpartial);
  cudaFree(c->reswork);
  cudaFree(c->obspartial);
  cudaFree(c->scal);
  cudaFreeHost(c->scal_h);
  cudaFree(c->status);
  cudaFree(c->Xh);
  cudaFree(c->Rh);
  cudaFree(c->ameta);
  cudaFree(c->apartial);
  if (c->ameta_h) cudaFreeHost(c->ameta_h);
  free_hilbert_tables(c->hil);
  for (auto& e : c->pev)
    if (e) cudaEventDestroy(e);
  if (c->ev_fork) cudaEventDestroy(c->ev_fork);
  if (c->ev_join) cudaEventDestroy(c->ev_join);
  if (c->st2) cudaStreamDestroy(c->st2);
  if (c->st) cudaStreamDestroy(c->st);
  delete c;
}

// ---------------------------------------------------------------------------
// Memory preflight (the estimate and refusal of build_production_cache,
// numerics/optimized/production_cache.jl:475-668, 764-770): the device bytes
// scba_create allocates, computed before the first allocation.
// ---------------------------------------------------------------------------
struct MemPlan {
  size_t fields = 0, operators = 0, workspace = 0, anderson = 0, transient = 0;
  size_t resident() const { return fields + operators + workspace + anderson; }
  size_t peak() const { return resident() + transient; }
};

// Element counts of a mechanism's operator arrays (as uploaded).
static std::vector<size_t> op_arrays(const qcl_mechanism& q, int Nk, int N) {
  const size_t N2 = (size_t)N * N, nc = (size_t)Nk * N2, J = q.J > 0 ? (size_t)q.J : 0;
  switch (q.kind) {
    case QCL_KERNEL_MOMENTUM_INDEPENDENT: return {N2 * N2};
    case QCL_KERNEL_DENSE: return {nc * nc};
    case QCL_KERNEL_IFR: return {N2 * J, J * N2, (size_t)Nk * Nk};
    case QCL_KERNEL_LOW_RANK: return {nc * J, J * nc};
    case QCL_KERNEL_SEPARABLE_SUM: return {(size_t)Nk * Nk * J, N2 * N2 * J};
    default: return {};
  }
}

// Contraction scratch elements of a mechanism at one precision.
static size_t op_work_elems(const qcl_mechanism& q, int precision, int NE, int Nk, int N) {
  KernelOpDev k;
  k.kind = q.kind;
  k.J = q.J;
  static const void* dummy[1] = {nullptr};
  if (precision != QCL_C128) {  // the tensor-core operands exist
    if (q.kind == QCL_KERNEL_DENSE) k.tc_bop = dummy;
    if (q.kind == QCL_KERNEL_SEPARABLE_SUM) {
      k.tc_chunks = dummy;
      k.tc_stage1 = dummy;
    }
  }
  return contraction_work_elems(k, NE, Nk, N);
}

static int plan_memory(const qcl_scba_problem* p, const qcl_mechanism* mechs, MemPlan* mp) {
  *mp = MemPlan();
  if (!p || p->NE < 2 || p->Nk < 1 || p->Nb < 1 || p->nmech < 0 || p->nmech > 5) {
    set_last_error("memory estimate: invalid dimensions or mechanism count");
    return QCL_DIM;
  }
  const int NE = p->NE, Nk = p->Nk, N = p->Nb, M = p->nmech;
  const bool c128 = p->precision == QCL_C128;
  const size_t esz = c128 ? 16 : 8, nfield = field_elems(NE, Nk, N);
  const size_t fcap = nfield * (p->refinement ? 16 : esz);
  mp->fields = (size_t)(6 * (M + 2) + 8) * fcap;  // state + candidate families, G x 3, totals x 3, candSL, tmp
  size_t cwork = 0;
  for (int i = 0; i < M; ++i) {
    const qcl_mechanism& q = mechs[i];
    for (size_t n : op_arrays(q, Nk, N)) {
      mp->operators += n * esz;
      if (!c128 && p->refinement) mp->operators += n * 16;  // kept complex128 copy
      mp->transient = std::max(mp->transient, c128 ? (size_t)0 : n * 16);  // staging copy
    }
    const int N2 = N * N;
    if (!c128 && q.kind == QCL_KERNEL_DENSE) mp->operators += tc_operator_bytes(Nk * N2, Nk * N2);
    if (!c128 && q.kind == QCL_KERNEL_SEPARABLE_SUM)
      for (int i0 = 0; i0 < q.J; i0 += kSepChunk)
        mp->operators += tc_operator_bytes(N2, std::min(kSepChunk, q.J - i0) * N2) +
                         tc_operator_bytes(Nk * std::min(kSepChunk, q.J - i0), Nk);
    cwork = std::max(cwork, op_work_elems(q, p->precision, NE, Nk, N) * esz);
    if (p->refinement && !c128) cwork = std::max(cwork, op_work_elems(q, QCL_C128, NE, Nk, N) * 16);
  }
  const int L = next_pow2(2 * NE - 1);
  mp->workspace = cwork + 2 * (size_t)NE * Nk * 16 + (size_t)kReduceCtas * 2 * 8 +
                  residual_mix_multi_partial_doubles(3 * (M + 2)) * 8 + residual_work_doubles(NE, Nk) * 8 +
                  observables_partial_doubles(N) * 8 + 4096 /* scalars, status */ +
                  (size_t)16 * 16 * L /* FFT tables */ + (size_t)Nk * N * N * 2 * 8 /* per-column partials */;
  if (p->mixing)
    mp->anderson = 2 * (size_t)p->anderson_history_depth * 3 * (M + 2) * fcap +
                   anderson_partial_doubles(3 * (M + 2)) * 8 + sizeof(AndersonMeta);
  return QCL_OK;
}

int scba_estimate_memory(const qcl_scba_problem* p, const qcl_mechanism* mechs, size_t out[6]) {
  MemPlan mp;
  int s = plan_memory(p, mechs, &mp);
  if (s) return s;
  out[0] = mp.fields;
  out[1] = mp.operators;
  out[2] = mp.workspace;
  out[3] = mp.anderson;
  out[4] = mp.resident();
  out[5] = mp.peak();
  return QCL_OK;
}

int scba_create(const qcl_scba_problem* p, const qcl_mechanism* mechs, ScbaCtx** out) {
  *out = nullptr;
  if (!p || p->NE < 2 || p->Nk < 1 || p->Nb < 1) {
    set_last_error("scba_create: invalid dimensions");
    return QCL_DIM;
  }
  if (padded_size(p->Nb) == 0) {
    set_last_error("basis size N_b=%d exceeds the supported maximum 48", p->Nb);
    return QCL_UNSUPPORTED;
  }
  if (p->nmech < 0 || p->nmech > 5) {
    set_last_error("scba_create: 0..5 scattering mechanisms supported, got %d", p->nmech);
    return QCL_ARG;
  }
  if (!(p->alpha > 0 && p->alpha <= 1)) {
    set_last_error("mixing factor must lie in (0,1]");
    return QCL_ARG;
  }
  if (p->precision != QCL_C128 && p->precision != QCL_C64 && p->precision != QCL_MIXED) {
    set_last_error("unknown precision %d", p->precision);
    return QCL_ARG;
  }
  if (p->refinement && p->precision == QCL_C128) {
    set_last_error("refinement applies to a reduced-precision context (QCL_C64 or QCL_MIXED)");
    return QCL_ARG;
  }
  {
    // preflight: refuse before the first allocation (build_production_cache,
    // production_cache.jl:764-770)
    MemPlan mp;
    int s0 = plan_memory(p, mechs, &mp);
    if (s0) return s0;
    size_t budget = p->memory_budget_bytes;
    if (budget == 0) {
      size_t fr = 0, tot = 0;
      cudaError_t e = cudaMemGetInfo(&fr, &tot);
      if (e != cudaSuccess) return cuda_status(e, "cudaMemGetInfo");
      budget = fr;
    }
    if (mp.peak() > budget) {
      set_last_error("estimated peak device memory %zu bytes exceeds the execution budget %zu bytes (fields %zu, "
                     "operators %zu, workspace %zu, Anderson history %zu, staging %zu)",
                     mp.peak(), budget, mp.fields, mp.operators, mp.workspace, mp.anderson, mp.transient);
      return QCL_NOMEM;
    }
  }
  ScbaCtx* c = new ScbaCtx();
  c->refinement = p->refinement;
  c->NE = p->NE;
  c->Nk = p->Nk;
  c->N = p->Nb;
  c->M = p->nmech;
  c->precision = p->precision;
  c->gs = p->gs;
  c->verify = p->verify_roundoff;
  c->Ep = p->Ep;
  c->hw_LO = p->hw_LO;
  c->N_LO = p->N_LO;
  c->target = p->target;
  c->eta_seed = p->eta_seed;
  c->kBT = p->kBT;
  c->alpha = p->alpha;
  c->J0 = p->J0;
  c->diagonal = p->self_energy_structure;
  c->averaged = p->transverse_momentum;
  c->drop_real = p->retarded_real_part;
  c->direct_green = p->elastic_retarded;
  c->scalar_lesser = p->occupation_normalization;
  c->mixing = p->mixing;
  c->and_depth = p->anderson_history_depth;
  c->and_damping = p->anderson_damping;
  c->and_reg = p->anderson_regularization;
  c->nfield = field_elems(c->NE, c->Nk, c->N);
  c->fbytes = c->nfield * (c->precision == QCL_C128 ? 16 : 8);
  c->fcap = c->refinement ? c->nfield * 16 : c->fbytes;
  c->eps_h.assign(p->eps, p->eps + p->NE);
  c->wE_h.assign(p->wE, p->wE + p->NE);
  int s;
#define TRY(x)            \
  do {                    \
    if ((s = (x))) {      \
      scba_destroy(c);    \
      return s;           \
    }                     \
  } while (0)
  double de;
  TRY(check_uniform_grid(c->NE, p->eps, &de));
  c->de = de;
  // _check_algorithm_options (algorithm_options.jl:42-93) for the model switches
  for (int sw : {c->diagonal, c->averaged, c->drop_real, c->direct_green, c->scalar_lesser})
    if (sw != 0 && sw != 1)
      TRY((set_last_error("model switches (self_energy_structure, transverse_momentum, retarded_real_part, "
                          "elastic_retarded, occupation_normalization) must be 0 or 1"),
           QCL_ARG));
  if (c->mixing != 0 && c->mixing != 1) TRY((set_last_error("mixing must be 0 (:linear) or 1 (:anderson)"), QCL_ARG));
  if (c->mixing) {  // _check_algorithm_options (algorithm_options.jl:84-91)
    if (c->and_depth < 1) TRY((set_last_error("anderson_history_depth must be positive"), QCL_ARG));
    if (c->and_depth > kAndersonMaxDepth)
      TRY((set_last_error("anderson_history_depth %d exceeds the supported maximum %d", c->and_depth,
                          kAndersonMaxDepth),
           QCL_UNSUPPORTED));
    if (!(c->and_damping > 0 && c->and_damping <= 1)) TRY((set_last_error("anderson_damping must lie in (0,1]"), QCL_ARG));
    if (!(c->and_reg >= 0) || !isfinite(c->and_reg))
      TRY((set_last_error("anderson_regularization cannot be negative"), QCL_ARG));
  }
  for (int m = 0; m < c->Nk; ++m) c->wk_sum += p->wk[m];
  if (c->averaged && !(c->wk_sum > 0)) TRY((set_last_error("radial weights must have positive sum"), QCL_ARG));
  if (c->direct_green && !c->drop_real)
    for (int i = 0; i < c->M; ++i)
      if (mechs[i].kind == QCL_KERNEL_LOW_RANK && mechs[i].J < c->Nk * c->N * c->N)
        TRY((set_last_error("direct_green elastic retarded closure requires an untruncated kernel; a truncated "
                            "low-rank operator does not preserve adjoints and positivity"),
             QCL_ARG));
  {
    cudaError_t e = cudaStreamCreateWithFlags(&c->st, cudaStreamNonBlocking);
    if (e != cudaSuccess) TRY(cuda_status(e, "cudaStreamCreate"));
    // the residual suite's G-only part runs beside the candidate construction
    e = cudaStreamCreateWithFlags(&c->st2, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&c->ev_fork, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&c->ev_join, cudaEventDisableTiming);
    if (e != cudaSuccess) TRY(cuda_status(e, "cudaStreamCreate"));
  }
  TRY(dupload(&c->eps, p->eps, c->NE * sizeof(double), c->st));
  TRY(dupload(&c->wE, p->wE, c->NE * sizeof(double), c->st));
  TRY(dupload(&c->wk, p->wk, c->Nk * sizeof(double), c->st));
  TRY(dupload(&c->h, p->h, (size_t)c->Nk * c->N * c->N * 16, c->st));
  TRY(dupload(&c->Tp, p->Tplus, (size_t)c->N * c->N * 16, c->st));
  TRY(dupload(&c->Tm, p->Tminus, (size_t)c->N * c->N * 16, c->st));
  TRY(build_plan(c, c->shift[0], +c->Ep));
  TRY(build_plan(c, c->shift[1], -c->Ep));
  TRY(build_plan(c, c->shift[2], +c->hw_LO));
  TRY(build_plan(c, c->shift[3], -c->hw_LO));
  size_t cwork = 0;
  const int N2 = c->N * c->N;
  for (int i = 0; i < c->M; ++i) {
    const qcl_mechanism& q = mechs[i];
    Mech m;
    m.kind = q.kind;
    m.is_LO = q.is_LO;
    m.q = q.q;
    m.J = q.J;
    c->mech.push_back(m);
    Mech& d = c->mech.back();
    if (q.kind == QCL_KERNEL_MOMENTUM_INDEPENDENT) {
      TRY(upload_op(c, &d.block, q.block, (size_t)N2 * N2, &d.block64));
    } else if (q.kind == QCL_KERNEL_DENSE) {
      const size_t nc = (size_t)c->Nk * N2;
      TRY(upload_op(c, &d.matrix, q.matrix, nc * nc, &d.matrix64));
      if (c->precision != QCL_C128)
        TRY(tc_build_operator((int)nc, c->Nk, d.matrix, c->wk, &d.tc_bop, c->st));
    } else if (q.kind == QCL_KERNEL_IFR) {
      if (q.J < 1) TRY((set_last_error("IFR operator needs J >= 1"), QCL_ARG));
      TRY(upload_op(c, &d.left, q.left, (size_t)N2 * q.J, &d.left64));
      TRY(upload_op(c, &d.right, q.right, (size_t)q.J * N2, &d.right64));
      TRY(upload_op(c, &d.radial, q.radial, (size_t)c->Nk * c->Nk, &d.radial64));
    } else if (q.kind == QCL_KERNEL_LOW_RANK) {
      if (q.J < 1) TRY((set_last_error("low-rank operator needs rank J >= 1"), QCL_ARG));
      const size_t nc = (size_t)c->Nk * N2;
      TRY(upload_op(c, &d.left, q.left, nc * q.J, &d.left64));
      TRY(upload_op(c, &d.right, q.right, (size_t)q.J * nc, &d.right64));
    } else if (q.kind == QCL_KERNEL_SEPARABLE_SUM) {
      if (q.J < 1) TRY((set_last_error("separable-sum operator needs J >= 1 terms"), QCL_ARG));
      TRY(upload_op(c, &d.radial, q.radial, (size_t)c->Nk * c->Nk * q.J, &d.radial64));
      TRY(upload_op(c, &d.block, q.block, (size_t)N2 * N2 * q.J, &d.block64));
      if (c->precision != QCL_C128)
        TRY(sep_build_tc_operands(c->Nk, c->N, q.J, d.radial, d.block, c->wk, d.tc_chunks, d.tc_stage1, c->st));
    } else {
      TRY((set_last_error("unknown kernel kind %d", q.kind), QCL_ARG));
    }
    cwork = std::max(cwork, contraction_work_elems(d.view(), c->NE, c->Nk, c->N) * (c->precision == QCL_C128 ? 16 : 8));
    if (c->refinement) {  // the complex128 contraction after promote
      KernelOpDev k64;
      k64.kind = d.kind;
      k64.J = d.J;
      cwork = std::max(cwork, contraction_work_elems(k64, c->NE, c->Nk, c->N) * 16);
    }
  }
  const int F = c->M + 2;
  c->state.assign(3 * F, nullptr);
  c->cand.assign(3 * F, nullptr);
  for (int i = 0; i < 3 * F; ++i) {
    TRY(dalloc(&c->state[i], c->fcap));
    TRY(dalloc(&c->cand[i], c->fcap));
  }
  TRY(dalloc(&c->GR, c->fcap));
  TRY(dalloc(&c->GL, c->fcap));
  TRY(dalloc(&c->GG, c->fcap));
  for (auto& t : c->tot) TRY(dalloc(&t, c->fcap));
  TRY(dalloc(&c->candSL, c->fcap));
  TRY(dalloc(&c->tmp, c->fcap));
  TRY(dalloc(&c->cwork, cwork));
  c->cwork_bytes = cwork;
  TRY(dalloc((void**)&c->trL, (size_t)c->NE * c->Nk * 16));
  TRY(dalloc((void**)&c->trG, (size_t)c->NE * c->Nk * 16));
  TRY(dalloc((void**)&c->rpartial, kReduceCtas * 2 * sizeof(double)));
  TRY(dalloc((void**)&c->mpartial, residual_mix_multi_partial_doubles(3 * (c->M + 2)) * sizeof(double)));
  TRY(dalloc((void**)&c->reswork, residual_work_doubles(c->NE, c->Nk) * sizeof(double)));
  TRY(dalloc((void**)&c->obspartial, observables_partial_doubles(c->N) * sizeof(double)));
  TRY(dalloc((void**)&c->scal, SC_TOTAL * sizeof(double)));
  {
    cudaError_t e = cudaMallocHost((void**)&c->scal_h, SC_TOTAL * sizeof(double));
    if (e != cudaSuccess) TRY(cuda_status(e, "cudaMallocHost"));
  }
  TRY(dalloc((void**)&c->status, 2 * sizeof(int)));
  QCL_CUDA_CHECK(cudaMemsetAsync(c->status, 0, 2 * sizeof(int), c->st));
  for (auto& m : c->mech) m.status = c->status;
  QCL_CUDA_CHECK(cudaMemsetAsync(c->scal, 0, SC_TOTAL * sizeof(double), c->st));
  if (c->mixing) {
    const size_t nf = 3 * (size_t)(c->M + 2);
    TRY(dalloc(&c->Xh, (size_t)c->and_depth * nf * c->fcap));
    TRY(dalloc(&c->Rh, (size_t)c->and_depth * nf * c->fcap));
    TRY(dalloc((void**)&c->ameta, sizeof(AndersonMeta)));
    TRY(dalloc((void**)&c->apartial, anderson_partial_doubles((int)nf) * sizeof(double)));
    cudaError_t e = cudaMallocHost((void**)&c->ameta_h, sizeof(AndersonMeta));
    if (e != cudaSuccess) TRY(cuda_status(e, "cudaMallocHost"));
    memset(c->ameta_h, 0, sizeof(AndersonMeta));
    TRY(launch_anderson_reset(c->ameta, c->st));
  }
  TRY(prepare_hilbert_tables(c->hil, c->NE, de, c->precision));
  TRY(ensure_partial(c->hil, (long long)c->Nk * N2));
#undef TRY
  QCL_CUDA_CHECK(cudaStreamSynchronize(c->st));
  c->pops.assign(c->N, 0.0);
  *out = c;
  return QCL_OK;
}

// ---------------------------------------------------------------------------
// Candidate maps (stream-ordered launches; no host synchronisation)
// ---------------------------------------------------------------------------
static int scattering_candidates(ScbaCtx* c, const void* GR, const void* GL, const void* GG, std::vector<void*>& dst,
                                 bool verify) {
  int s;
  const int p = c->precision;
  // contractions run at storage precision (mixed: FP32 with FP64 k-sums)
  const int cp = p == QCL_MIXED ? QCL_C64 : p;
  const long long ncols = (long long)c->Nk * c->N * c->N;
  for (int i = 0; i < c->M; ++i) {
    const Mech& m = c->mech[i];
    const KernelOpDev op = m.view();
    void* SL = field_of(dst, i, 1);
    void* SG = field_of(dst, i, 2);
    if (m.is_LO) {
      // _production_lo_contraction, thermal branch (production_operators.jl:1045-1163):
      //   Sigma< = (N+1) K[G<(E+hw)] + N K[G<(E-hw)],  Sigma> = (N+1) K[G>(E-hw)] + N K[G>(E+hw)].
      // K is linear, so each is one contraction of the combined shifted field,
      // K[(N+1) G(E+-hw) + N G(E-+hw)]: two dense maps instead of four.
      const double n = c->N_LO;
      if ((s = launch_shift_pair(cp, c->NE, ncols, c->shift[2].view(), c->shift[3].view(), n + 1, n, GL, c->tmp,
                                 c->st)))
        return s;
      if ((s = launch_contraction(cp, op, c->NE, c->Nk, c->N, c->wk, c->tmp, SL, m.q, 0.0, c->cwork, c->st))) return s;
      if ((s = launch_shift_pair(cp, c->NE, ncols, c->shift[3].view(), c->shift[2].view(), n + 1, n, GG, c->tmp,
                                 c->st)))
        return s;
      if ((s = launch_contraction(cp, op, c->NE, c->Nk, c->N, c->wk, c->tmp, SG, m.q, 0.0, c->cwork, c->st))) return s;
    } else {
      if ((s = launch_contraction(cp, op, c->NE, c->Nk, c->N, c->wk, GL, SL, m.q, 0.0, c->cwork, c->st))) return s;
      if ((s = launch_contraction(cp, op, c->NE, c->Nk, c->N, c->wk, GG, SG, m.q, 0.0, c->cwork, c->st))) return s;
    }
    void* SR = field_of(dst, i, 0);
    if (c->drop_real) {
      // Sigma^R = -i Gamma / 2 (production_operators.jl:1174-1177); no roundoff estimate
      if ((s = launch_retarded_drop(cp, c->nfield, SL, SG, SR, c->st))) return s;
    } else if (c->direct_green && !m.is_LO) {
      // elastic closure Sigma^R = K[G^R] (production_operators.jl:1311-1316)
      if ((s = launch_contraction(cp, op, c->NE, c->Nk, c->N, c->wk, GR, SR, m.q, 0.0, c->cwork, c->st))) return s;
    } else {
      if ((s = launch_hilbert(c->hil, cp, ncols, c->wE, nullptr, SL, SG, nullptr, SR, nullptr, verify, c->st)))
        return s;
      if (verify && (s = launch_combine(c->hil.partial, (int)ncols, 2, c->scal + SC_ROUND + 2 * i, c->st))) return s;
    }
    // _apply_scattering_model! (production_operators.jl:1240-1256)
    void* fam[3] = {SR, SL, SG};
    if ((s = launch_scattering_model(cp, c->NE, c->Nk, c->N, c->wk, c->wk_sum, c->diagonal, c->averaged, fam, c->st)))
      return s;
  }
  return QCL_OK;
}

static int embedding_candidates(ScbaCtx* c, std::vector<void*>& dst, const void* GR = nullptr,
                                const void* GL = nullptr, const void* GG = nullptr) {
  const int cp = c->precision == QCL_MIXED ? QCL_C64 : c->precision;
  SandwichJob jobs[2];
  for (int sgn = 0; sgn < 2; ++sgn) {
    jobs[sgn].X[0] = GR ? GR : c->GR;
    jobs[sgn].X[1] = GL ? GL : c->GL;
    jobs[sgn].X[2] = GG ? GG : c->GG;
    for (int k = 0; k < 3; ++k) jobs[sgn].S[k] = field_of(dst, c->M + sgn, k);
    jobs[sgn].T = sgn == 0 ? c->Tp : c->Tm;
    jobs[sgn].plan = c->shift[sgn].view();
  }
  return launch_sandwich(cp, c->NE, c->Nk, c->N, jobs, 2, c->st);
}

static int totals(ScbaCtx* c, const std::vector<void*>& fam, void* const* out, int comps_mask) {
  const int F = c->M + 2;
  for (int k = 0; k < 3; ++k) {
    if (!(comps_mask & (1 << k))) continue;
    const void* src[8];
    for (int f = 0; f < F; ++f) src[f] = field_of(fam, f, k);
    int s = launch_sum_fields(c->precision == QCL_MIXED ? QCL_C64 : c->precision, c->nfield, src, F, out[k], c->st);
    if (s) return s;
  }
  return QCL_OK;
}

// The current Green state from the state families (_current_green_production).
static int current_green(ScbaCtx* c, const std::vector<void*>& fam) {
  int s;
  if ((s = totals(c, fam, c->tot, 7))) return s;
  if ((s = launch_dyson_keldysh(c->precision, c->NE, c->Nk, c->N, c->eps, 0.0, c->h, c->tot[0], c->tot[1], c->tot[2],
                                c->GR, c->GL, c->GG, nullptr, c->trL, c->trG, c->status, c->st)))
    return s;
  if ((s = launch_weighted_trace(c->NE, c->Nk, c->trL, c->wE, c->wk, c->rpartial, c->scal + SC_TRL, c->st))) return s;
  if ((s = launch_weighted_trace(c->NE, c->Nk, c->trG, c->wE, c->wk, c->rpartial, c->scal + SC_TRG, c->st))) return s;
  if ((s = launch_paired_coefficients(c->scal + SC_TRL, c->scal + SC_TRG, c->gs, c->target, c->scal + SC_COEF,
                                      c->status, c->st, c->precision == QCL_C128 ? 1e-10 : 1e-5, c->scalar_lesser,
                                      c->norm_branch)))
    return s;
  const int sp = c->precision == QCL_MIXED ? QCL_C64 : c->precision;
  if (c->scalar_lesser) return launch_scalar_lesser(sp, c->NE, c->Nk, c->N, c->GR, c->GL, c->GG, c->scal + SC_COEF, c->st);
  return launch_normalize_pair(sp, c->nfield, c->GL, c->GG, c->scal + SC_COEF, c->st);
}

// Everything of one iteration after the state is fixed; writes candidates into
// `cand`, mixed values into `cand` as well (speculatively) and all scalars.
// Marks the end of phase i - 1 / start of phase i (an event-record node when
// the iteration is captured into a graph).
static int phase_mark(ScbaCtx* c, int i) {
  if (!c->telemetry) return QCL_OK;
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  QCL_CUDA_CHECK(cudaStreamIsCapturing(c->st, &cs));
  if (cs == cudaStreamCaptureStatusActive)  // an event-record node of the captured iteration
    QCL_CUDA_CHECK(cudaEventRecordWithFlags(c->pev[i], c->st, cudaEventRecordExternal));
  else
    QCL_CUDA_CHECK(cudaEventRecord(c->pev[i], c->st));
  return QCL_OK;
}

static int iteration_body(ScbaCtx* c, std::vector<void*>& state, std::vector<void*>& cand) {
  int s;
  const int sp = c->precision == QCL_MIXED ? QCL_C64 : c->precision;
  if ((s = phase_mark(c, 0))) return s;
  if ((s = current_green(c, state))) return s;
  if ((s = phase_mark(c, 1))) return s;
  // Everything of the residual suite except r_K needs only G and the totals:
  // it runs on the side stream while the candidates are built; r_K follows the
  // candidate total lesser, and the fixed-order reduction waits for both (the
  // two parts write disjoint per-block slots).
  QCL_CUDA_CHECK(cudaEventRecord(c->ev_fork, c->st));
  QCL_CUDA_CHECK(cudaStreamWaitEvent(c->st2, c->ev_fork, 0));
  if ((s = launch_residual_blocks(c->precision, RES_PART_MAIN, c->NE, c->Nk, c->N, c->eps, c->h, c->GR, c->GL, c->GG,
                                  c->tot[0], c->tot[1], c->tot[2], nullptr, c->reswork, c->st2)))
    return s;
  QCL_CUDA_CHECK(cudaEventRecord(c->ev_join, c->st2));
  if ((s = scattering_candidates(c, c->GR, c->GL, c->GG, cand, c->verify != 0))) return s;
  if ((s = phase_mark(c, 2))) return s;
  if ((s = embedding_candidates(c, cand))) return s;
  if ((s = phase_mark(c, 3))) return s;
  // candidate total lesser for r_K
  {
    const void* src[8];
    const int F = c->M + 2;
    for (int f = 0; f < F; ++f) src[f] = field_of(cand, f, 1);
    if ((s = launch_sum_fields(sp, c->nfield, src, F, c->candSL, c->st))) return s;
  }
  if ((s = phase_mark(c, 4))) return s;
  if ((s = launch_residual_blocks(c->precision, RES_PART_RK, c->NE, c->Nk, c->N, c->eps, c->h, c->GR, c->GL, c->GG,
                                  c->tot[0], c->tot[1], c->tot[2], c->candSL, c->reswork, c->st)))
    return s;
  QCL_CUDA_CHECK(cudaStreamWaitEvent(c->st, c->ev_join, 0));
  if ((s = launch_residual_reduce(c->NE, c->Nk, c->reswork, c->scal + SC_RES, c->st))) return s;
  // embedding-total residual (before the plus/minus candidates are mixed over)
  for (int k = 0; k < 3; ++k)
    if ((s = launch_residual_pair(sp, c->nfield, field_of(state, c->M, k), field_of(state, c->M + 1, k),
                                  field_of(cand, c->M, k), field_of(cand, c->M + 1, k), c->rpartial,
                                  c->scal + SC_EMB + 2 * k, c->st)))
      return s;
  if ((s = phase_mark(c, 5))) return s;
  // J from the (unmixed) plus family and the state's G
  if ((s = launch_observables(sp, c->NE, c->Nk, c->N, c->wE, c->wk, field_of(state, c->M, 2), field_of(state, c->M, 1),
                              c->GL, c->GG, c->gs, c->target, c->obspartial, c->scal + SC_OBS, c->st)))
    return s;
  if ((s = phase_mark(c, 6))) return s;
  // per-family residual + speculative linear mixing into the candidate buffers
  const int F = c->M + 2;
  const void* olds[kMaxMixFields];
  void* cands[kMaxMixFields];
  for (int f = 0; f < F; ++f)
    for (int k = 0; k < 3; ++k) {
      olds[3 * f + k] = field_of(state, f, k);
      cands[3 * f + k] = field_of(cand, f, k);
    }
  if (c->mixing) {
    // Anderson mixing with the causality guard (production_mixing.jl:224-317)
    const int nf = 3 * F;
    if ((s = launch_anderson_plan(c->ameta, c->and_depth, c->st))) return s;
    if ((s = launch_anderson_append(sp, c->nfield, olds, (const void* const*)cands, nf, c->Xh, c->Rh, c->and_depth,
                                    c->ameta, c->apartial, c->scal + SC_FAM, c->st)))
      return s;
    if ((s = launch_anderson_coefficients(c->ameta, c->and_depth, c->and_reg, c->st))) return s;
    const double damping = c->alpha * c->and_damping;
    for (int pass = 0; pass < 2; ++pass) {  // pass 1 (linear fallback) runs only if pass 0's guard failed
      if ((s = launch_anderson_mix(sp, c->nfield, cands, nf, c->Xh, c->Rh, c->and_depth, c->ameta, damping, pass,
                                   c->st)))
        return s;
      if ((s = launch_anderson_guard(sp, c->NE, c->Nk, c->N, cands, F, c->ameta, pass, c->guard_roundoff,
                                     c->st)))
        return s;
      if ((s = launch_anderson_after_guard(c->ameta, pass, c->status, c->st))) return s;
    }
    QCL_CUDA_CHECK(cudaMemcpyAsync(c->ameta_h, c->ameta, sizeof(AndersonMeta), cudaMemcpyDeviceToHost, c->st));
  } else if ((s = launch_residual_mix_multi(sp, c->nfield, olds, cands, 3 * F, c->alpha, c->mpartial,
                                            c->scal + SC_FAM, c->st))) {
    return s;
  }
  if ((s = phase_mark(c, 7))) return s;
  QCL_CUDA_CHECK(cudaMemcpyAsync(c->scal_h, c->scal, SC_TOTAL * sizeof(double), cudaMemcpyDeviceToHost, c->st));
  return QCL_OK;
}

static double fermi(double e, double mu, double kBT) {
  const double x = (e - mu) / kBT;
  if (x > 40.0) return 0.0;   // _FERMI_EXPONENT_SATURATION
  if (x < -40.0) return 1.0;
  return 1.0 / (exp(x) + 1.0);
}

int scba_seed(ScbaCtx* c, double* mu_out) {
  int s;
  const int sp = c->precision == QCL_MIXED ? QCL_C64 : c->precision;
  if (c->telemetry) QCL_CUDA_CHECK(cudaEventRecord(c->pev[0], c->st));
  // Dyson with eta_seed and Sigma = 0 (cand fields used as scratch zeros)
  QCL_CUDA_CHECK(cudaMemsetAsync(c->tot[0], 0, c->fbytes, c->st));
  if ((s = launch_dyson_keldysh(c->precision, c->NE, c->Nk, c->N, c->eps, c->eta_seed, c->h, c->tot[0], nullptr,
                                nullptr, c->GR, nullptr, nullptr, nullptr, nullptr, nullptr, c->status, c->st)))
    return s;
  double* q_d = c->reswork;  // scratch
  if ((s = launch_seed_weights(sp, c->NE, c->Nk, c->N, c->GR, c->wE, c->wk, c->gs, q_d, c->st))) return s;
  std::vector<double> q(c->NE), f(c->NE);
  QCL_CUDA_CHECK(cudaMemcpyAsync(q.data(), q_d, c->NE * sizeof(double), cudaMemcpyDeviceToHost, c->st));
  QCL_CUDA_CHECK(cudaStreamSynchronize(c->st));
  int hst[2];
  QCL_CUDA_CHECK(cudaMemcpy(hst, c->status, sizeof(hst), cudaMemcpyDeviceToHost));
  if (hst[0] == QCL_SINGULAR) return singular_status("seed Dyson solve", hst[1]);
  if (hst[0]) {
    set_last_error("seed Dyson solve failed (status %d at block %d)", hst[0], hst[1]);
    return hst[0];
  }
  for (int e = 0; e < c->NE; ++e)
    if (!isfinite(q[e])) {
      set_last_error("seed spectral number weights must be finite");
      return QCL_DOMAIN;
    }
  auto number_at = [&](double mu) {
    double v = 0;
    for (int e = 0; e < c->NE; ++e) v += q[e] * fermi(c->eps_h[e], mu, c->kBT);
    return v - c->target;
  };
  double lo = c->eps_h.front() - 50 * c->kBT, hi = c->eps_h.back() + 50 * c->kBT;
  double flo = number_at(lo), fhi = number_at(hi);
  if (!(flo * fhi <= 0)) {
    set_last_error("seed chemical-potential root is not bracketed");
    return QCL_ARG;
  }
  // bisection to adjacent doubles (the role of Roots.jl Bisection, seed.jl:182)
  double mu;
  if (flo == 0) mu = lo;
  else if (fhi == 0) mu = hi;
  else {
    for (int it = 0; it < 2000; ++it) {
      const double mid = 0.5 * (lo + hi);
      if (mid == lo || mid == hi) break;
      const double fm = number_at(mid);
      if (fm == 0) {
        lo = hi = mid;
        break;
      }
      if ((fm < 0) == (flo < 0)) {
        lo = mid;
        flo = fm;
      } else {
        hi = mid;
      }
    }
    mu = fabs(number_at(lo)) <= fabs(number_at(hi)) ? lo : hi;
  }
  for (int e = 0; e < c->NE; ++e) f[e] = fermi(c->eps_h[e], mu, c->kBT);
  double* f_d = c->reswork + c->NE;
  QCL_CUDA_CHECK(cudaMemcpyAsync(f_d, f.data(), c->NE * sizeof(double), cudaMemcpyHostToDevice, c->st));
  if ((s = launch_seed_green(sp, c->NE, c->Nk, c->N, c->GR, f_d, c->GL, c->GG, c->st))) return s;
  // initial candidates (no roundoff verification), straight into the state
  if ((s = scattering_candidates(c, c->GR, c->GL, c->GG, c->state, false))) return s;
  if ((s = embedding_candidates(c, c->state))) return s;
  QCL_CUDA_CHECK(cudaStreamSynchronize(c->st));
  QCL_CUDA_CHECK(cudaMemcpy(hst, c->status, sizeof(hst), cudaMemcpyDeviceToHost));
  if (hst[0]) {
    set_last_error("seed candidate failed (status %d)", hst[0]);
    return hst[0];
  }
  if (mu_out) *mu_out = mu;
  if (c->telemetry) {  // :initialization (seed + initial candidates)
    QCL_CUDA_CHECK(cudaEventRecord(c->pev[1], c->st));
    QCL_CUDA_CHECK(cudaEventSynchronize(c->pev[1]));
    float ms = 0;
    QCL_CUDA_CHECK(cudaEventElapsedTime(&ms, c->pev[0], c->pev[1]));
    c->init_ms = ms;
  }
  c->seeded = true;
  c->have_green = true;
  c->green_eta = c->eta_seed;
  c->have_residual = false;  // the seed used the residual scratch
  if (c->mixing) {
    if ((s = launch_anderson_reset(c->ameta, c->st))) return s;
    QCL_CUDA_CHECK(cudaStreamSynchronize(c->st));
  }
  c->nu = 0;
  c->pending_commit = false;
  c->Jprev = NAN;
  c->lam_prev = NAN;
  c->pprev.clear();
  return QCL_OK;
}

// Drops the captured iteration graphs (they hold the context's current
// scalars, precision and telemetry marks).
static void drop_graphs(ScbaCtx* c) {
  for (int g = 0; g < 2; ++g) {
    if (c->graph[g]) cudaGraphExecDestroy(c->graph[g]);
    if (c->gtpl[g]) cudaGraphDestroy(c->gtpl[g]);
    c->graph[g] = nullptr;
    c->gtpl[g] = nullptr;
  }
}

// Enqueues one iteration.  With `child` non-null and a captured iteration
// available, the iteration is not launched: *child receives its graph, for
// the caller to launch as a node of a larger graph (a batched sweep);
// otherwise *child is null and the iteration is on the context's stream.
static int run_body(ScbaCtx* c, cudaGraph_t* child) {
  if (child) *child = nullptr;
  std::vector<void*>& st = c->parity == 0 ? c->state : c->cand;
  std::vector<void*>& cd = c->parity == 0 ? c->cand : c->state;
  // graphs are captured once every kernel has been launched (and configured) eagerly
  if (!c->use_graph || c->nu < 1) return iteration_body(c, st, cd);
  if (!c->graph[c->parity]) {
    cudaGraph_t g;
    QCL_CUDA_CHECK(cudaStreamBeginCapture(c->st, cudaStreamCaptureModeThreadLocal));
    int s = iteration_body(c, st, cd);
    cudaError_t e = cudaStreamEndCapture(c->st, &g);
    if (s) {
      if (e == cudaSuccess) cudaGraphDestroy(g);
      return s;
    }
    if (e != cudaSuccess) return cuda_status(e, "cudaStreamEndCapture");
    e = cudaGraphInstantiate(&c->graph[c->parity], g, 0);
    if (e != cudaSuccess) {
      cudaGraphDestroy(g);
      return cuda_status(e, "cudaGraphInstantiate");
    }
    c->gtpl[c->parity] = g;
  }
  if (child) {
    *child = c->gtpl[c->parity];
    return QCL_OK;
  }
  QCL_CUDA_CHECK(cudaGraphLaunch(c->graph[c->parity], c->st));
  return QCL_OK;
}

// One SCBA iteration.  Commits the previous iteration's mixing first.
int scba_step(ScbaCtx* c, qcl_scba_row* row) {
  int s = scba_step_launch(c, nullptr);
  if (s) return s;
  return scba_step_finish(c, row);
}

// First half of a step: commit, then enqueue the iteration (or hand its
// captured graph to the caller through `child`, see run_body).
int scba_step_launch(ScbaCtx* c, cudaGraph_t* child) {
  if (!c->seeded) {
    set_last_error("scba_step before scba_seed");
    return QCL_ARG;
  }
  if (c->pending_commit) {
    c->parity ^= 1;
    c->pending_commit = false;
  }
  return run_body(c, child);
}

// Second half of a step: once the iteration has run (on the context's stream
// or inside the caller's graph, whose stream the caller has synchronised),
// read its scalars into the row and apply the reference's status handling.
int scba_step_finish(ScbaCtx* c, qcl_scba_row* row) {
  int s;
  c->have_green = true;
  c->green_eta = 0.0;
  c->have_residual = true;
  QCL_CUDA_CHECK(cudaStreamSynchronize(c->st));
  if (c->telemetry)
    for (int i = 0; i < kPhases; ++i) {
      float ms = 0;
      QCL_CUDA_CHECK(cudaEventElapsedTime(&ms, c->pev[i], c->pev[i + 1]));
      c->phase_ms[i] = ms;
    }
  int hst[2];
  QCL_CUDA_CHECK(cudaMemcpy(hst, c->status, sizeof(hst), cudaMemcpyDeviceToHost));
  const double* h = c->scal_h;
  c->nu += 1;
  memset(row, 0, sizeof(*row));
  row->nu = c->nu;
  row->lambda = h[SC_COEF + 2];
  row->r_lambda = fabs(row->lambda - 1.0);
  row->number = h[SC_COEF + 3];
  row->holes = h[SC_COEF + 4];
  row->occupied_fraction = h[SC_COEF + 0];
  row->empty_fraction = h[SC_COEF + 1];
  row->target_charge = c->target;
  // number functional of the normalised G< (production_solver.jl:609): a N + c H
  // for the paired transfer (N(G>) = -H), N / lambda for the scalar comparator
  row->normalized_charge = c->scalar_lesser ? row->number / row->lambda
                                            : row->occupied_fraction * row->number +
                                                  row->empty_fraction * row->holes;
  row->lambda_change = isnan(c->lam_prev) ? NAN : row->lambda - c->lam_prev;
  row->r_D = h[SC_RES + 0];
  row->r_A = h[SC_RES + 1];
  row->r_K = h[SC_RES + 2];
  row->r_PSD = h[SC_RES + 3];
  row->r_caus = h[SC_RES + 4];
  double rS = 0;
  auto rel = [](double num, double den) {
    return (isfinite(num) && isfinite(den)) ? sqrt(num) / (sqrt(den) + 1e-14) : INFINITY;
  };
  for (int k = 0; k < 3; ++k) rS = fmax(rS, rel(h[SC_EMB + 2 * k], h[SC_EMB + 2 * k + 1]));
  for (int f = 0; f < c->M + 2; ++f)
    for (int k = 0; k < 3; ++k) {
      const double v = rel(h[SC_FAM + 2 * (3 * f + k)], h[SC_FAM + 2 * (3 * f + k) + 1]);
      rS = isfinite(v) ? fmax(rS, v) : INFINITY;
    }
  row->r_Sigma = rS;
  double rr = 0;
  if (c->verify)
    for (int i = 0; i < c->M; ++i) rr = fmax(rr, rel(h[SC_ROUND + 2 * i], h[SC_ROUND + 2 * i + 1]));
  row->r_roundoff = rr;
  row->Jbar = h[SC_OBS + 0];
  row->J = row->Jbar * c->J0;
  for (int a = 0; a < c->N; ++a) c->pops[a] = h[SC_OBS + 2 + a];
  row->r_J = isnan(c->Jprev) ? INFINITY : fabs(row->J - c->Jprev) / fmax(fmax(fabs(row->J), fabs(c->Jprev)), 1e-12);
  if (c->pprev.empty()) {
    row->r_pop = INFINITY;
  } else {
    double dn = 0, nn = 0;
    for (int a = 0; a < c->N; ++a) {
      dn += (c->pops[a] - c->pprev[a]) * (c->pops[a] - c->pprev[a]);
      nn += c->pops[a] * c->pops[a];
    }
    row->r_pop = sqrt(dn) / (sqrt(nn) + 1e-14);
  }
  row->status = hst[0];
  c->Jprev = row->J;
  c->lam_prev = row->lambda;
  c->pprev = c->pops;
  c->pending_commit = true;
  if (hst[0] == QCL_SINGULAR) {
    // a Dyson failure carries no partial state (production_solver.jl:447-469)
    c->pending_commit = false;
    return singular_status("SCBA Dyson solve", hst[1]);
  }
  if (hst[0] == QCL_DOMAIN) {
    c->pending_commit = false;
    if (c->mixing && c->ameta_h->fallback)
      set_last_error("convex Anderson fallback is not admissible; inspect raw self-energies (block %d)", hst[1]);
    else
      set_last_error("paired number normalisation rejected the raw occupation");
    return QCL_DOMAIN;
  }
  const double m[] = {row->r_D, row->r_A, row->r_K, row->r_Sigma, row->r_lambda, row->r_PSD, row->r_caus,
                      row->r_roundoff, row->J, row->lambda};
  for (double v : m)
    if (!isfinite(v)) {
      row->status = QCL_NONFINITE;
      c->pending_commit = false;
      return QCL_OK;  // reported as a row status (:nonfinite_metrics), not an error
    }
  return QCL_OK;
}

int scba_populations(ScbaCtx* c, double* out) {
  for (int a = 0; a < c->N; ++a) out[a] = c->pops[a];
  return QCL_OK;
}

// Copies a state field to host memory (checkpoint).  which: 0..2 = GR, G<, G>
// of the last iteration; 3 + 3 f + k = family f component k of the current
// (unmixed) state, f in [0, M) mechanisms, M plus, M + 1 minus.
int scba_download(ScbaCtx* c, int which, void* host) {
  const void* src = nullptr;
  if (which == 0) src = c->GR;
  else if (which == 1) src = c->GL;
  else if (which == 2) src = c->GG;
  else {
    const int idx = which - 3;
    if (idx < 0 || idx >= 3 * (c->M + 2)) {
      set_last_error("download: field index %d out of range", which);
      return QCL_ARG;
    }
    std::vector<void*>& st = c->parity == 0 ? c->state : c->cand;
    src = st[idx];
  }
  QCL_CUDA_CHECK(cudaStreamSynchronize(c->st));
  QCL_CUDA_CHECK(cudaMemcpy(host, src, c->fbytes, cudaMemcpyDeviceToHost));
  return QCL_OK;
}

// Replaces a state family component (warm start / resume, production_solver.jl:216-429).
int scba_upload(ScbaCtx* c, int which, const void* host) {
  const int idx = which - 3;
  if (idx < 0 || idx >= 3 * (c->M + 2)) {
    set_last_error("upload: field index %d out of range", which);
    return QCL_ARG;
  }
  if (c->pending_commit) {
    c->parity ^= 1;
    c->pending_commit = false;
  }
  std::vector<void*>& st = c->parity == 0 ? c->state : c->cand;
  if (c->mixing) {  // a replaced state starts a new Anderson history
    int s = launch_anderson_reset(c->ameta, c->st);
    if (s) return s;
  }
  QCL_CUDA_CHECK(cudaMemcpyAsync(st[idx], host, c->fbytes, cudaMemcpyHostToDevice, c->st));
  QCL_CUDA_CHECK(cudaStreamSynchronize(c->st));
  c->seeded = true;
  return QCL_OK;
}

// The derived GreenState fields of the last Dyson solve (seed or step):
// A = i (G^R - G^R^H), condition_number = cond_2(D), dyson_scale = s
// (_green_state_production, production_operators.jl:1387-1415, with the
// kappa / scale outputs of _retarded_green_production, :1337-1385).  Any
// output may be NULL; A is a field in the context's storage precision,
// kappa and scale are (N_E, N_k) float64.
int scba_green_state(ScbaCtx* c, void* A_host, double* kappa, double* scale) {
  if (!c->have_green) {
    set_last_error("green_state: no Green state yet (call seed or step first)");
    return QCL_ARG;
  }
  const int sp = c->precision == QCL_MIXED ? QCL_C64 : c->precision;
  const size_t nb = (size_t)c->NE * c->Nk * sizeof(double);
  struct Tmp {
    void* p[3] = {nullptr, nullptr, nullptr};
    ~Tmp() {
      for (void* q : p)
        if (q) cudaFree(q);
    }
  } t;
  int s;
  if (A_host && (s = dalloc(&t.p[0], c->fbytes))) return s;
  if (kappa && (s = dalloc(&t.p[1], nb))) return s;
  if (scale && (s = dalloc(&t.p[2], nb))) return s;
  if (A_host && (s = launch_spectral(sp, c->NE, c->Nk, c->N, c->GR, t.p[0], c->st))) return s;
  if ((kappa || scale) && (s = launch_condition(sp, c->NE, c->Nk, c->N, c->eps, c->green_eta, c->h, c->tot[0], c->GR,
                                                (double*)t.p[1], (double*)t.p[2], c->st)))
    return s;
  if (A_host) QCL_CUDA_CHECK(cudaMemcpyAsync(A_host, t.p[0], c->fbytes, cudaMemcpyDeviceToHost, c->st));
  if (kappa) QCL_CUDA_CHECK(cudaMemcpyAsync(kappa, t.p[1], nb, cudaMemcpyDeviceToHost, c->st));
  if (scale) QCL_CUDA_CHECK(cudaMemcpyAsync(scale, t.p[2], nb, cudaMemcpyDeviceToHost, c->st));
  QCL_CUDA_CHECK(cudaStreamSynchronize(c->st));
  return QCL_OK;
}

// Positivity witness of the last step's residual suite (SCBAIteration.witness,
// production_solver.jl:611-619): reduced on request from the per-block
// outputs the step left in the residual scratch.
int scba_witness(ScbaCtx* c, double* out12) {
  if (!c->have_residual) {
    set_last_error("witness: no residual evaluation yet (call step first)");
    return QCL_ARG;
  }
  const int sp = c->precision == QCL_MIXED ? QCL_C64 : c->precision;
  double* dev = nullptr;
  int s = dalloc((void**)&dev, (residual_witness_partial_doubles() + 12) * sizeof(double));
  if (s) return s;
  s = launch_residual_witness(sp, c->NE, c->Nk, c->N, c->GR, c->GL, c->GG, c->tot[1], c->tot[2], c->reswork, dev,
                              dev + residual_witness_partial_doubles(), c->st);
  if (!s) {
    cudaError_t e = cudaMemcpyAsync(out12, dev + residual_witness_partial_doubles(), 12 * sizeof(double),
                                    cudaMemcpyDeviceToHost, c->st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->st);
    if (e != cudaSuccess) s = cuda_status(e, "witness download");
  }
  cudaFree(dev);
  return s;
}

// A new operating point on the same cache (retarget_problem +
// retarget_production_cache, composition/operating_point.jl:25-170): the
// +-Ep shift plans are rebuilt for the new field, h (the new Hartree
// Hamiltonian), N_LO, kBT and the kernel scales q^K are replaced where given;
// the kernel operators, grids, LO plans and the state stay resident, so the
// next step continues from the last (unmixed) state as a warm start.  The
// per-run history (r_J, r_pop, lambda_change, iteration count) restarts, and
// captured iteration graphs are rebuilt (they hold the old scalars).
int scba_retarget(ScbaCtx* c, double Ep, double N_LO, double kBT, const void* h, const double* q) {
  if (!isfinite(Ep) || !isfinite(N_LO) || N_LO < 0 || !(kBT > 0) || !isfinite(kBT)) {
    set_last_error("retarget: Ep, N_LO >= 0 and kBT > 0 must be finite");
    return QCL_ARG;
  }
  if (q)
    for (int i = 0; i < c->M; ++i)
      if (!isfinite(q[i])) {
        set_last_error("retarget: kernel scale q[%d] is not finite", i);
        return QCL_ARG;
      }
  QCL_CUDA_CHECK(cudaStreamSynchronize(c->st));
  int s;
  if ((s = refill_plan(c, c->shift[0], +Ep))) return s;
  if ((s = refill_plan(c, c->shift[1], -Ep))) return s;
  if (h) {
    QCL_CUDA_CHECK(cudaMemcpyAsync(c->h, h, (size_t)c->Nk * c->N * c->N * 16, cudaMemcpyHostToDevice, c->st));
    QCL_CUDA_CHECK(cudaStreamSynchronize(c->st));
  }
  c->Ep = Ep;
  c->N_LO = N_LO;
  c->kBT = kBT;
  if (q)
    for (int i = 0; i < c->M; ++i) c->mech[i].q = q[i];
  drop_graphs(c);
  c->pending_commit = false;  // keep the unmixed state of the last step
  c->nu = 0;
  c->Jprev = NAN;
  c->lam_prev = NAN;
  c->pprev.clear();
  c->have_green = false;
  c->have_residual = false;
  if (c->mixing) {  // a new operating point starts a new Anderson history
    if ((s = launch_anderson_reset(c->ameta, c->st))) return s;
    QCL_CUDA_CHECK(cudaStreamSynchronize(c->st));
  }
  return QCL_OK;
}

// rho_ab = sum wE wk G<_ab of the last Dyson solve (the electron-density
// coherences the outer Poisson loop projects on the position grid,
// _electron_density_bar, physics/observables.jl:1-22).  out: N x N complex128.
int scba_density_matrix(ScbaCtx* c, void* out) {
  if (!c->have_green) {
    set_last_error("density_matrix: no Green state yet (call seed or step first)");
    return QCL_ARG;
  }
  const int sp = c->precision == QCL_MIXED ? QCL_C64 : c->precision;
  double* d = nullptr;
  int s = dalloc((void**)&d, 2 * (size_t)c->N * c->N * sizeof(double));
  if (s) return s;
  s = launch_density_matrix(sp, c->NE, c->Nk, c->N, c->GL, c->wE, c->wk, d, c->st);
  if (!s) {
    cudaError_t e = cudaMemcpyAsync(out, d, 2 * (size_t)c->N * c->N * sizeof(double), cudaMemcpyDeviceToHost, c->st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->st);
    if (e != cudaSuccess) s = cuda_status(e, "density_matrix download");
  }
  cudaFree(d);
  return s;
}

// Mixer diagnostics of the last step (the SolverMetric list of _anderson_mix!,
// production_mixing.jl:283-298).
int scba_mixer_info(ScbaCtx* c, qcl_anderson_info* out) {
  memset(out, 0, sizeof(*out));
  if (!c->mixing) return QCL_OK;
  const AndersonMeta& m = *c->ameta_h;
  out->history_depth = m.used;
  out->reset_reason = m.reason;
  out->coefficients_l1 = m.l1;
  out->acceleration_accepted = m.accepted;
  out->fallback = m.fallback;
  out->guard_first_failure = (long long)m.guard_first;
  out->guard_failure_code = m.guard_code;
  return QCL_OK;
}

int scba_set_graph(ScbaCtx* c, int enable) {
  c->use_graph = enable != 0;
  return QCL_OK;
}

// Phase telemetry on / off; captured graphs are rebuilt (they hold the marks or not).
int scba_set_telemetry(ScbaCtx* c, int enable) {
  QCL_CUDA_CHECK(cudaStreamSynchronize(c->st));
  if (enable && !c->pev[0])
    for (auto& e : c->pev) QCL_CUDA_CHECK(cudaEventCreate(&e));
  c->telemetry = enable != 0;
  drop_graphs(c);
  return QCL_OK;
}

int scba_phase_times(ScbaCtx* c, double* ms, double* init_ms) {
  if (!c->telemetry) {
    set_last_error("phase_times: telemetry is off");
    return QCL_ARG;
  }
  if (ms)
    for (int i = 0; i < kPhases; ++i) ms[i] = c->phase_ms[i];
  if (init_ms) *init_ms = c->init_ms;
  return QCL_OK;
}

// Switches a refinement context (QCL_MIXED or QCL_C64 storage) to complex128
// for the iterations that follow: the FP64 refinement of a reduced-precision
// fixed point.  The current state families (with the last step's mixing
// committed) are converted exactly to complex128, the operators switch to the
// complex128 copies kept at creation, the FFT tables are rebuilt and the
// captured graphs and the Anderson history are dropped.  The next step
// continues from the same state; the row history (r_J, r_pop) continues.
int scba_promote(ScbaCtx* c) {
  if (!c->refinement) {
    set_last_error("promote: the context was not created with refinement enabled");
    return QCL_ARG;
  }
  if (c->precision == QCL_C128) return QCL_OK;
  QCL_CUDA_CHECK(cudaStreamSynchronize(c->st));
  if (c->pending_commit) {
    c->parity ^= 1;
    c->pending_commit = false;
  }
  int s;
  std::vector<void*>& st = c->parity == 0 ? c->state : c->cand;
  for (size_t i = 0; i < st.size(); ++i) {  // state field -> tmp (complex128), then swap the buffers
    void*& f = st[i];
    if ((s = launch_promote(c->nfield, f, c->tmp, c->st))) return s;
    std::swap(f, c->tmp);
    // Sigma< and Sigma> are anti-Hermitian (i times Hermitian) per block; the
    // reduced-precision iterations computed the (a,b) and (b,a) entries apart,
    // so they are only anti-Hermitian to FP32 rounding, which the FP64 checks
    // of the iterations that follow (the realness of the number functional,
    // 1e-10) would reject.  The promoted state keeps their anti-Hermitian part.
    if (i % 3 != 0 && (s = launch_antihermitian_part(c->NE, c->Nk, c->N, f, c->st))) return s;
  }
  for (auto& m : c->mech) {
    auto swap_in = [](void*& cur, void*& keep) {
      if (keep) {
        cudaFree(cur);
        cur = keep;
        keep = nullptr;
      }
    };
    swap_in(m.block, m.block64);
    swap_in(m.matrix, m.matrix64);
    swap_in(m.left, m.left64);
    swap_in(m.right, m.right64);
    swap_in(m.radial, m.radial64);
    cudaFree(m.tc_bop);
    m.tc_bop = nullptr;
    for (void* q : m.tc_chunks) cudaFree(q);
    m.tc_chunks.clear();
    for (void* q : m.tc_stage1) cudaFree(q);
    m.tc_stage1.clear();
  }
  c->precision = QCL_C128;
  c->guard_roundoff = 1.1920928955078125e-07;  // the promoted state's FP32 rounding
  c->fbytes = c->nfield * 16;
  if ((s = prepare_hilbert_tables(c->hil, c->NE, c->de, QCL_C128))) return s;
  if ((s = ensure_partial(c->hil, (long long)c->Nk * c->N * c->N))) return s;
  drop_graphs(c);
  if (c->mixing && (s = launch_anderson_reset(c->ameta, c->st))) return s;
  c->have_green = false;
  c->have_residual = false;
  QCL_CUDA_CHECK(cudaStreamSynchronize(c->st));
  return QCL_OK;
}

int scba_precision(ScbaCtx* c) { return c->precision; }

cudaStream_t scba_stream(ScbaCtx* c) { return c->st; }

// ---------------------------------------------------------------------------
// Batched sweep of independent operating points (bias points of a sweep,
// structures of different sizes).  The reference solves operating points one
// after another, re-using basis and kernels (retarget_problem +
// retarget_production_cache, composition/operating_point.jl:25-170).  Here
// every point is a context; the points that fit the memory budget together
// (the preflight estimate of each) are resident at once, and one iteration of
// all of them is ONE graph launch: a parent graph whose child nodes are the
// points' captured iterations, which the GPU runs concurrently.  A point
// leaves when it converges (r_Sigma <= tol), fails, or reaches max_iter; the
// next pending point takes its memory.  The parent graph is rebuilt when the
// resident set changes and otherwise alternates between the two parities.
// ---------------------------------------------------------------------------
struct SweepPoint {
  qcl_scba_problem problem;
  std::vector<qcl_mechanism> mechs;
};

struct Sweep {
  std::vector<SweepPoint> points;
  size_t budget = 0;
  cudaStream_t st = nullptr;
};

void sweep_destroy(Sweep* sw) {
  if (!sw) return;
  if (sw->st) cudaStreamDestroy(sw->st);
  delete sw;
}

int sweep_create(int n, const qcl_scba_problem* problems, const qcl_mechanism* const* mechanisms, size_t budget,
                 Sweep** out) {
  *out = nullptr;
  if (n < 1 || !problems || !mechanisms) {
    set_last_error("sweep: at least one point with its problem and mechanisms is required");
    return QCL_ARG;
  }
  Sweep* sw = new Sweep();
  sw->budget = budget;
  for (int i = 0; i < n; ++i) {
    SweepPoint pt;
    pt.problem = problems[i];
    if (pt.problem.nmech > 0 && !mechanisms[i]) {
      sweep_destroy(sw);
      set_last_error("sweep: point %d has no mechanism array", i);
      return QCL_ARG;
    }
    pt.mechs.assign(mechanisms[i], mechanisms[i] + std::max(pt.problem.nmech, 0));
    MemPlan mp;
    int s = plan_memory(&pt.problem, pt.mechs.data(), &mp);
    if (s) {
      sweep_destroy(sw);
      return s;
    }
    sw->points.push_back(pt);
  }
  cudaError_t e = cudaStreamCreateWithFlags(&sw->st, cudaStreamNonBlocking);
  if (e != cudaSuccess) {
    sweep_destroy(sw);
    return cuda_status(e, "cudaStreamCreate (sweep)");
  }
  *out = sw;
  return QCL_OK;
}

// stats: [0] wall seconds, [1] total iterations, [2] parent-graph launches,
// [3] largest number of resident points, [4] parent-graph builds.
int sweep_run(Sweep* sw, int max_iter, double tol, qcl_scba_row* last, int* iters, double* stats) {
  const int n = (int)sw->points.size();
  size_t budget = sw->budget;
  if (budget == 0) {
    size_t fr = 0, tot = 0;
    QCL_CUDA_CHECK(cudaMemGetInfo(&fr, &tot));
    budget = fr;
  }
  struct Active {
    int idx;
    ScbaCtx* ctx;
    size_t bytes;
  };
  std::vector<Active> active;
  std::vector<size_t> peak(n);
  for (int i = 0; i < n; ++i) {
    MemPlan mp;
    plan_memory(&sw->points[i].problem, sw->points[i].mechs.data(), &mp);
    peak[i] = mp.peak();
    if (peak[i] > budget) {
      set_last_error("sweep: point %d alone needs %zu bytes, over the budget %zu", i, peak[i], budget);
      return QCL_NOMEM;
    }
    iters[i] = 0;
    memset(&last[i], 0, sizeof(qcl_scba_row));
  }
  auto t0 = std::chrono::steady_clock::now();
  double launches = 0, builds = 0, total_iters = 0, max_resident = 0;
  int next = 0;
  size_t used = 0;
  std::map<std::vector<std::pair<void*, int>>, cudaGraphExec_t> parents;
  auto clear_parents = [&]() {
    for (auto& kv : parents) cudaGraphExecDestroy(kv.second);
    parents.clear();
  };
  auto fail = [&](int s) {
    clear_parents();
    for (auto& a : active) scba_destroy(a.ctx);
    return s;
  };
  while (next < n || !active.empty()) {
    // admit pending points while they fit
    bool changed = false;
    while (next < n && used + peak[next] <= budget) {
      qcl_scba_problem p = sw->points[next].problem;
      p.memory_budget_bytes = budget - used;
      ScbaCtx* c = nullptr;
      int s = scba_create(&p, sw->points[next].mechs.data(), &c);
      if (s) return fail(s);
      c->use_graph = true;
      if ((s = scba_seed(c, nullptr))) {
        scba_destroy(c);
        return fail(s);
      }
      active.push_back({next, c, peak[next]});
      used += peak[next];
      ++next;
      changed = true;
    }
    if (changed) clear_parents();
    max_resident = std::max(max_resident, (double)active.size());
    // one iteration of every resident point
    std::vector<cudaGraph_t> kids;
    std::vector<std::pair<void*, int>> key;
    for (auto& a : active) {
      cudaGraph_t g = nullptr;
      int s = scba_step_launch(a.ctx, &g);
      if (s) return fail(s);
      if (g) {
        kids.push_back(g);
        key.push_back({(void*)a.ctx, a.ctx->parity});
      }
    }
    if (!kids.empty()) {
      auto it = parents.find(key);
      if (it == parents.end()) {
        cudaGraph_t parent;
        QCL_CUDA_CHECK(cudaGraphCreate(&parent, 0));
        for (cudaGraph_t g : kids) {
          cudaGraphNode_t node;
          cudaError_t e = cudaGraphAddChildGraphNode(&node, parent, nullptr, 0, g);
          if (e != cudaSuccess) {
            cudaGraphDestroy(parent);
            return fail(cuda_status(e, "cudaGraphAddChildGraphNode"));
          }
        }
        cudaGraphExec_t ex;
        cudaError_t e = cudaGraphInstantiate(&ex, parent, 0);
        cudaGraphDestroy(parent);
        if (e != cudaSuccess) return fail(cuda_status(e, "cudaGraphInstantiate (sweep)"));
        it = parents.emplace(key, ex).first;
        builds += 1;
      }
      cudaError_t e = cudaGraphLaunch(it->second, sw->st);
      if (e == cudaSuccess) e = cudaStreamSynchronize(sw->st);
      if (e != cudaSuccess) return fail(cuda_status(e, "sweep iteration"));
      launches += 1;
    }
    // rows; converged, failed or exhausted points leave
    std::vector<Active> keep;
    for (auto& a : active) {
      qcl_scba_row row;
      int s = scba_step_finish(a.ctx, &row);
      iters[a.idx] += 1;
      total_iters += 1;
      last[a.idx] = row;
      const bool done = s != QCL_OK || row.status != QCL_OK || row.r_Sigma <= tol || iters[a.idx] >= max_iter;
      if (s != QCL_OK) last[a.idx].status = s;
      if (done) {
        scba_destroy(a.ctx);
        used -= a.bytes;
        changed = true;
      } else {
        keep.push_back(a);
      }
    }
    active.swap(keep);
    if (changed) clear_parents();
  }
  clear_parents();
  if (stats) {
    stats[0] = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    stats[1] = total_iters;
    stats[2] = launches;
    stats[3] = max_resident;
    stats[4] = builds;
  }
  return QCL_OK;
}

// ---------------------------------------------------------------------------
// Tangent of the fixed point (implicit differentiation, forward mode).  At
// the state of the last step, v solves v = Phi_Sigma v + s for a source s
// (the explicit parameter derivative Phi_p, uploaded by the caller), by the
// damped iteration v <- (1 - alpha) v + alpha (Phi_Sigma v + s), the
// linearisation of the linear-mixing SCBA iteration itself.  Each tangent step
// also returns the tangent of the current density, J_Sigma v.  Requires a
// complex128 context with linear mixing and the paired normalisation.
// ---------------------------------------------------------------------------
enum { TS_DTRL = 0, TS_DTRG = 2, TS_DCOEF = 4, TS_FAM = 6 };
static size_t tangent_scal_doubles(const ScbaCtx* c) { return TS_FAM + 2 * 3 * (c->M + 2) + 2 * (2 + 48) + 8; }

int scba_tangent_init(ScbaCtx* c) {
  if (c->precision != QCL_C128 || c->mixing || c->scalar_lesser) {
    set_last_error("tangent: requires a complex128 context with linear mixing and the paired normalisation");
    return QCL_UNSUPPORTED;
  }
  if (!c->tv.empty()) return QCL_OK;
  const int nf = 3 * (c->M + 2);
  int s;
  for (auto* v : {&c->tv, &c->tw, &c->tsrc}) {
    v->assign(nf, nullptr);
    for (int i = 0; i < nf; ++i) {
      if ((s = dalloc(&(*v)[i], c->fbytes))) return s;
      QCL_CUDA_CHECK(cudaMemsetAsync((*v)[i], 0, c->fbytes, c->st));
    }
  }
  for (int k = 0; k < 3; ++k) {
    if ((s = dalloc(&c->tG[k], c->fbytes))) return s;
    if ((s = dalloc(&c->ttot[k], c->fbytes))) return s;
  }
  if ((s = dalloc((void**)&c->ttrL, (size_t)c->NE * c->Nk * 16))) return s;
  if ((s = dalloc((void**)&c->ttrG, (size_t)c->NE * c->Nk * 16))) return s;
  if ((s = dalloc((void**)&c->tscal, tangent_scal_doubles(c) * sizeof(double)))) return s;
  QCL_CUDA_CHECK(cudaMallocHost((void**)&c->tscal_h, tangent_scal_doubles(c) * sizeof(double)));
  QCL_CUDA_CHECK(cudaStreamSynchronize(c->st));
  return QCL_OK;
}

// which = 3 + 3 f + k (as qcl_scba_download): the source's family f component
// k; host == NULL zeroes it.  which = -1 zeroes the tangent v itself.
int scba_tangent_set(ScbaCtx* c, int which, const void* host) {
  if (c->tv.empty()) {
    set_last_error("tangent: call qcl_scba_tangent_init first");
    return QCL_ARG;
  }
  if (which == -1) {
    for (void* p : c->tv) QCL_CUDA_CHECK(cudaMemsetAsync(p, 0, c->fbytes, c->st));
    QCL_CUDA_CHECK(cudaStreamSynchronize(c->st));
    return QCL_OK;
  }
  const int idx = which - 3;
  if (idx < 0 || idx >= (int)c->tsrc.size()) {
    set_last_error("tangent: field index %d out of range", which);
    return QCL_ARG;
  }
  if (host) QCL_CUDA_CHECK(cudaMemcpyAsync(c->tsrc[idx], host, c->fbytes, cudaMemcpyHostToDevice, c->st));
  else QCL_CUDA_CHECK(cudaMemsetAsync(c->tsrc[idx], 0, c->fbytes, c->st));
  QCL_CUDA_CHECK(cudaStreamSynchronize(c->st));
  return QCL_OK;
}

// One tangent step at the state of the last SCBA step.  out[0] = J_Sigma v
// (solver units, before the step's update: the tangent of the step's J),
// out[1] = max over fields ||v_new - v|| / (||v_new|| + 1e-300).
int scba_tangent_step(ScbaCtx* c, double* out) {
  if (c->tv.empty() || !c->have_green) {
    set_last_error("tangent: needs qcl_scba_tangent_init and a completed SCBA step");
    return QCL_ARG;
  }
  int s;
  const int F = c->M + 2, nf = 3 * F, NE = c->NE, Nk = c->Nk, N = c->N;
  std::vector<void*>& st = c->parity == 0 ? c->state : c->cand;  // the linearisation point
  // tangent totals
  if ((s = totals(c, c->tv, c->ttot, 7))) return s;
  // Dyson + Keldysh tangent
  void *X = c->tG[0], *dL = c->tG[1], *dG = c->tG[2];
  if ((s = launch_block_triple(NE, Nk, N, c->GR, c->ttot[0], c->GR, 0, 1.0, 0.0, X, nullptr, c->st))) return s;
  const void* Sig[2] = {c->tot[1], c->tot[2]};
  void* dOut[2] = {dL, dG};
  Cx<double>* tr[2] = {c->ttrL, c->ttrG};
  for (int k = 0; k < 2; ++k) {
    if ((s = launch_block_triple(NE, Nk, N, X, Sig[k], c->GR, 1, 1.0, 0.0, dOut[k], nullptr, c->st))) return s;
    if ((s = launch_block_triple(NE, Nk, N, c->GR, c->ttot[1 + k], c->GR, 1, 1.0, 1.0, dOut[k], nullptr, c->st)))
      return s;
    if ((s = launch_block_triple(NE, Nk, N, c->GR, Sig[k], X, 1, 1.0, 1.0, dOut[k], tr[k], c->st))) return s;
  }
  if ((s = launch_weighted_trace(NE, Nk, c->ttrL, c->wE, c->wk, c->rpartial, c->tscal + TS_DTRL, c->st))) return s;
  if ((s = launch_weighted_trace(NE, Nk, c->ttrG, c->wE, c->wk, c->rpartial, c->tscal + TS_DTRG, c->st))) return s;
  if ((s = launch_norm_tangent(c->nfield, c->GL, c->GG, c->scal + SC_COEF, c->tscal + TS_DTRL, c->tscal + TS_DTRG,
                               c->gs, c->target, c->norm_branch, c->tscal + TS_DCOEF, dL, dG, c->st)))
    return s;
  // J tangent: J(v_plus, G) + J(Sigma_plus, dG)
  double* jout = c->tscal + TS_FAM + 2 * nf;
  if ((s = launch_observables(QCL_C128, NE, Nk, N, c->wE, c->wk, field_of(c->tv, c->M, 2), field_of(c->tv, c->M, 1),
                              c->GL, c->GG, c->gs, c->target, c->obspartial, jout, c->st)))
    return s;
  if ((s = launch_observables(QCL_C128, NE, Nk, N, c->wE, c->wk, field_of(st, c->M, 2), field_of(st, c->M, 1), dL, dG,
                              c->gs, c->target, c->obspartial, jout + 2 + N, c->st)))
    return s;
  // Phi_Sigma v: the linear candidate maps of the tangent Green's functions
  if ((s = scattering_candidates(c, X, dL, dG, c->tw, false))) return s;
  if ((s = embedding_candidates(c, c->tw, X, dL, dG))) return s;
  // w <- Phi_Sigma v + s, then the damped update into w with the residual norms
  const void* olds[kMaxMixFields];
  void* cands[kMaxMixFields];
  for (int i = 0; i < nf; ++i) {
    if ((s = launch_axpby(QCL_C128, c->nfield, 1.0, c->tw[i], 1.0, c->tsrc[i], c->tw[i], c->st))) return s;
    olds[i] = c->tv[i];
    cands[i] = c->tw[i];
  }
  if ((s = launch_residual_mix_multi(QCL_C128, c->nfield, olds, cands, nf, c->alpha, c->mpartial, c->tscal + TS_FAM,
                                     c->st)))
    return s;
  std::swap(c->tv, c->tw);
  QCL_CUDA_CHECK(cudaMemcpyAsync(c->tscal_h, c->tscal, tangent_scal_doubles(c) * sizeof(double),
                                 cudaMemcpyDeviceToHost, c->st));
  QCL_CUDA_CHECK(cudaStreamSynchronize(c->st));
  const double* h = c->tscal_h;
  double r = 0;
  for (int i = 0; i < nf; ++i) {
    const double num = h[TS_FAM + 2 * i], den = h[TS_FAM + 2 * i + 1];
    r = fmax(r, sqrt(num) / (sqrt(den) + 1e-300));
  }
  out[0] = h[TS_FAM + 2 * nf] + h[TS_FAM + 2 * nf + 2 + N];
  out[1] = r;
  return QCL_OK;
}

// The form of the paired normalisation (0: the reference's choice by the sign
// of number - target; 1 / 2: the first / second form forced, its formula
// continued across the switch).  Graphs capture the form, so they are rebuilt.
int scba_set_norm_branch(ScbaCtx* c, int branch) {
  if (branch < 0 || branch > 2) {
    set_last_error("normalisation branch %d: expected 0, 1 or 2", branch);
    return QCL_ARG;
  }
  if (c->norm_branch != branch) {
    QCL_CUDA_CHECK(cudaStreamSynchronize(c->st));
    c->norm_branch = branch;
    drop_graphs(c);
  }
  return QCL_OK;
}

// The form the last step used: 1 (scale G<) or 2 (move G> weight into G<).
int scba_norm_branch(ScbaCtx* c, int* out) {
  if (!c->have_green) {
    set_last_error("normalisation branch: no completed step");
    return QCL_ARG;
  }
  QCL_CUDA_CHECK(cudaStreamSynchronize(c->st));
  *out = c->norm_branch ? c->norm_branch : (c->scal_h[SC_COEF + 3] >= c->target ? 1 : 2);
  return QCL_OK;
}

// The last step's mixed candidate family field (the speculative linear mix
// (1 - alpha) Sigma + alpha Phi(Sigma) the next step would commit), for the
// caller's difference quotient Phi_p; which as qcl_scba_download.
int scba_download_candidate(ScbaCtx* c, int which, void* host) {
  const int idx = which - 3;
  if (!c->pending_commit || idx < 0 || idx >= 3 * (c->M + 2)) {
    set_last_error("download_candidate: no pending step or field index %d out of range", which);
    return QCL_ARG;
  }
  std::vector<void*>& cd = c->parity == 0 ? c->cand : c->state;
  QCL_CUDA_CHECK(cudaStreamSynchronize(c->st));
  QCL_CUDA_CHECK(cudaMemcpy(host, cd[idx], c->fbytes, cudaMemcpyDeviceToHost));
  return QCL_OK;
}

}  // namespace qcl
