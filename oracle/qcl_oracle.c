/*
 * CPU FP64 oracle for the SCBA hot path of QCLNEGF.jl.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is a plain-C restatement of the
 * reference's Julia operators.  Only the test suite, the smoke check and the
 * CPU-baseline leg of the benchmark load it, and only as the checker: nothing
 * in the CUDA product path calls it, links it or falls back to it.
 *
 * Layout: every field is a Julia column-major (N_E, N_k, N_b, N_b) array of
 * ComplexF64 (two interleaved doubles), energy fastest, so that element
 * (e, m, a, b) sits at e + NE*(m + Nk*(a + Nb*b)) (0-based here).  Small
 * dense N_b x N_b matrices are column-major as in Julia.
 *
 * Every function names the reference file:line it restates; paths are relative
 * to the QCLNEGF.jl project root.
 */
#include <complex.h>
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

typedef double complex dc;

#define ORC_OK 0
#define ORC_SINGULAR 1
#define ORC_DOMAIN 2
#define ORC_DIM 3
#define ORC_ARG 4

#define IX(e, m, a, b)                                                         \
  ((size_t)(e) + (size_t)NE * ((size_t)(m) +                                   \
                               (size_t)Nk * ((size_t)(a) + (size_t)Nb * (size_t)(b))))
#define MAT(A, i, j, n) ((A)[(size_t)(i) + (size_t)(n) * (size_t)(j)])

static double cabs1(dc z) { return fabs(creal(z)) + fabs(cimag(z)); }

/* a*b with the textbook formula (no inf/nan recovery of the C99 library
 * multiply): the operands here are finite. */
static inline dc cmul(dc a, dc b) {
  double ar = creal(a), ai = cimag(a), br = creal(b), bi = cimag(b);
  return CMPLX(ar * br - ai * bi, ar * bi + ai * br);
}

/* ------------------------------------------------------------------------ */
/* Small dense linear algebra                                                */
/* ------------------------------------------------------------------------ */

/* Partial-pivot LU (pivot by |Re|+|Im|, as LAPACK izamax / the reference's
 * small-block path production_operators.jl:84-139) followed by the explicit
 * inverse from solving A X = I column by column.  In place, column-major.
 * Returns 0, or k (1-based) for an exactly zero pivot (SingularException(k),
 * production_operators.jl:39,94). */
int orc_inverse(int n, dc *A, dc *work /* n*n */, int *piv /* n */) {
  for (int k = 0; k < n; ++k) {
    int p = k;
    double largest = cabs1(MAT(A, k, k, n));
    for (int i = k + 1; i < n; ++i) {
      double mag = cabs1(MAT(A, i, k, n));
      if (mag > largest) {
        largest = mag;
        p = i;
      }
    }
    if (MAT(A, p, k, n) == 0.0) return k + 1;
    piv[k] = p;
    if (p != k)
      for (int j = 0; j < n; ++j) {
        dc t = MAT(A, k, j, n);
        MAT(A, k, j, n) = MAT(A, p, j, n);
        MAT(A, p, j, n) = t;
      }
    for (int i = k + 1; i < n; ++i) MAT(A, i, k, n) /= MAT(A, k, k, n);
    for (int j = k + 1; j < n; ++j)
      for (int i = k + 1; i < n; ++i) MAT(A, i, j, n) -= cmul(MAT(A, i, k, n), MAT(A, k, j, n));
  }
  for (int col = 0; col < n; ++col) {
    dc *X = work + (size_t)col * n;
    for (int i = 0; i < n; ++i) X[i] = (i == col) ? 1.0 : 0.0;
    for (int k = 0; k < n; ++k) {
      int p = piv[k];
      dc t = X[k];
      X[k] = X[p];
      X[p] = t;
    }
    for (int i = 0; i < n; ++i) {
      dc v = X[i];
      for (int k = 0; k < i; ++k) v -= cmul(MAT(A, i, k, n), X[k]);
      X[i] = v;
    }
    for (int i = n - 1; i >= 0; --i) {
      dc v = X[i];
      for (int k = i + 1; k < n; ++k) v -= cmul(MAT(A, i, k, n), X[k]);
      X[i] = v / MAT(A, i, i, n);
    }
  }
  memcpy(A, work, sizeof(dc) * (size_t)n * n);
  return 0;
}

/* C = A * op(B), op = identity (adj=0) or adjoint (adj=1). n x n, col-major. */
static void matmul(int n, const dc *A, const dc *B, int adj, dc *C) {
  for (int j = 0; j < n; ++j) {
    for (int i = 0; i < n; ++i) MAT(C, i, j, n) = 0;
    for (int l = 0; l < n; ++l) {
      dc b = adj ? conj(MAT(B, j, l, n)) : MAT(B, l, j, n);
      double br = creal(b), bi = cimag(b);
      const double *a = (const double *)&MAT(A, 0, l, n);
      double *c = (double *)&MAT(C, 0, j, n);
      for (int i = 0; i < n; ++i) {
        c[2 * i] += a[2 * i] * br - a[2 * i + 1] * bi;
        c[2 * i + 1] += a[2 * i] * bi + a[2 * i + 1] * br;
      }
    }
  }
}

/* Eigenvalues of a Hermitian matrix by cyclic complex Jacobi rotations.  The
 * input H (col-major, n x n) is overwritten.  Stands in for LAPACK zheev
 * (residuals.jl:311-353); the tests pin it against numpy.linalg.eigvalsh. */
void orc_hermitian_eigvals(int n, dc *H, double *values) {
  for (int j = 0; j < n; ++j) {
    MAT(H, j, j, n) = creal(MAT(H, j, j, n));
    for (int i = j + 1; i < n; ++i) {
      dc avg = 0.5 * (MAT(H, i, j, n) + conj(MAT(H, j, i, n)));
      MAT(H, i, j, n) = avg;
      MAT(H, j, i, n) = conj(avg);
    }
  }
  for (int sweep = 0; sweep < 100; ++sweep) {
    double off = 0.0, diag = 0.0;
    for (int j = 0; j < n; ++j)
      for (int i = 0; i < n; ++i) {
        double v = creal(MAT(H, i, j, n) * conj(MAT(H, i, j, n)));
        if (i == j) diag += v; else off += v;
      }
    if (off <= 1e-34 * diag || off == 0.0) break;
    for (int p = 0; p < n - 1; ++p)
      for (int q = p + 1; q < n; ++q) {
        dc apq = MAT(H, p, q, n);
        double mag = cabs(apq);
        if (mag == 0.0) continue;
        dc phase = apq / mag; /* scale column q by conj(phase), row q by phase */
        for (int k = 0; k < n; ++k) {
          MAT(H, k, q, n) *= conj(phase);
          MAT(H, q, k, n) *= phase;
        }
        double app = creal(MAT(H, p, p, n)), aqq = creal(MAT(H, q, q, n));
        double theta = (aqq - app) / (2.0 * mag);
        double t = (theta >= 0 ? 1.0 : -1.0) / (fabs(theta) + sqrt(theta * theta + 1.0));
        double c = 1.0 / sqrt(t * t + 1.0), s = t * c;
        for (int k = 0; k < n; ++k) {
          if (k == p || k == q) continue;
          dc akp = MAT(H, k, p, n), akq = MAT(H, k, q, n);
          dc nkp = c * akp - s * akq, nkq = s * akp + c * akq;
          MAT(H, k, p, n) = nkp;
          MAT(H, p, k, n) = conj(nkp);
          MAT(H, k, q, n) = nkq;
          MAT(H, q, k, n) = conj(nkq);
        }
        MAT(H, p, p, n) = app - t * mag;
        MAT(H, q, q, n) = aqq + t * mag;
        MAT(H, p, q, n) = 0;
        MAT(H, q, p, n) = 0;
      }
  }
  for (int i = 0; i < n; ++i) values[i] = creal(MAT(H, i, i, n));
  /* ascending order, like LAPACK */
  for (int i = 1; i < n; ++i) {
    double v = values[i];
    int j = i - 1;
    while (j >= 0 && values[j] > v) {
      values[j + 1] = values[j];
      --j;
    }
    values[j + 1] = v;
  }
}

/* Largest singular value via eig(X^H X); for the spectral norms used by the
 * condition number and the causality residual (residuals.jl:355-409). */
static double spectral_norm(int n, const dc *X, dc *work, double *values) {
  for (int j = 0; j < n; ++j)
    for (int i = 0; i < n; ++i) {
      dc s = 0;
      for (int l = 0; l < n; ++l) s += conj(MAT(X, l, i, n)) * MAT(X, l, j, n);
      MAT(work, i, j, n) = s;
    }
  orc_hermitian_eigvals(n, work, values);
  double v = values[n - 1];
  return sqrt(v > 0 ? v : 0);
}

static double frob(int n, const dc *X) {
  double s = 0;
  for (size_t i = 0; i < (size_t)n * n; ++i) s += creal(X[i] * conj(X[i]));
  return sqrt(s);
}

static double norm1(int n, const dc *X) {
  double best = 0;
  for (int j = 0; j < n; ++j) {
    double s = 0;
    for (int i = 0; i < n; ++i) s += cabs(MAT(X, i, j, n));
    if (s > best) best = s;
  }
  return best;
}

/* ------------------------------------------------------------------------ */
/* Dyson / Keldysh / number functional                                       */
/* ------------------------------------------------------------------------ */

/* retarded_green (numerics/reference/greens.jl:18-42) and its production form
 * _retarded_green_production (numerics/optimized/production_operators.jl:
 * 1337-1385): D = (eps_e + i eta) I - h_m - SigmaR_em; s = max row sum of |D|;
 * G = inv(D/s)/s.  kappa1 = ||D||_1 ||D^-1||_1, kappa2 = cond_2(D) (may be
 * NULL).  Returns 0 or the 1-based singular pivot of the first failing block
 * (scale 0 reports pivot 0 as ORC_SINGULAR with *bad_block set). */
int orc_retarded_green(int NE, int Nk, int Nb, const double *eps, double eta,
                       const dc *h /* (Nk,Nb,Nb) */, const dc *sigR, dc *GR,
                       double *kappa1, double *kappa2, double *scale,
                       long *bad_block) {
  int status = 0;
  long first_bad = -1;
#pragma omp parallel
  {
    dc *D = malloc(sizeof(dc) * Nb * Nb);
    dc *A = malloc(sizeof(dc) * Nb * Nb);
    dc *W = malloc(sizeof(dc) * Nb * Nb);
    double *vals = malloc(sizeof(double) * Nb);
    int *piv = malloc(sizeof(int) * Nb);
#pragma omp for schedule(static)
    for (long linear = 0; linear < (long)NE * Nk; ++linear) {
      int e = (int)(linear % NE), m = (int)(linear / NE);
      for (int b = 0; b < Nb; ++b)
        for (int a = 0; a < Nb; ++a) {
          dc d = (a == b) ? (eps[e] + I * eta) : 0.0;
          d -= h[(size_t)m + (size_t)Nk * (a + (size_t)Nb * b)];
          d -= sigR ? sigR[IX(e, m, a, b)] : 0.0;
          MAT(D, a, b, Nb) = d;
        }
      double s = 0;
      for (int a = 0; a < Nb; ++a) {
        double row = 0;
        for (int b = 0; b < Nb; ++b) row += cabs(MAT(D, a, b, Nb));
        if (row > s) s = row;
      }
      int info = 0;
      if (!(s > 0)) info = -1;
      else {
        for (int i = 0; i < Nb * Nb; ++i) A[i] = D[i] / s;
        info = orc_inverse(Nb, A, W, piv);
      }
      if (info != 0) {
#pragma omp critical
        {
          if (first_bad < 0 || linear < first_bad) {
            first_bad = linear;
            status = info < 0 ? 0 : info;
          }
        }
        for (int b = 0; b < Nb; ++b)
          for (int a = 0; a < Nb; ++a) GR[IX(e, m, a, b)] = NAN;
        continue;
      }
      for (int b = 0; b < Nb; ++b)
        for (int a = 0; a < Nb; ++a) GR[IX(e, m, a, b)] = MAT(A, a, b, Nb) / s;
      if (scale) scale[linear] = s;
      if (kappa1) {
        double inv1 = norm1(Nb, A) / s;
        kappa1[linear] = norm1(Nb, D) * inv1;
      }
      if (kappa2) {
        /* cond_2(D) = ||D||_2 ||D^-1||_2 */
        double nd = spectral_norm(Nb, D, W, vals);
        for (int i = 0; i < Nb * Nb; ++i) D[i] = A[i] / s;
        double ni = spectral_norm(Nb, D, W, vals);
        kappa2[linear] = nd * ni;
      }
    }
    free(D); free(A); free(W); free(vals); free(piv);
  }
  if (bad_block) *bad_block = first_bad;
  if (first_bad >= 0) return status == 0 ? 1000000 : status;
  return 0;
}

/* keldysh_green (greens.jl:67-75), production sandwiches production_state.jl:
 * 23-48: out_em = G_em Sigma_em G_em^H. */
void orc_keldysh_green(int NE, int Nk, int Nb, const dc *GR, const dc *sig, dc *out) {
#pragma omp parallel
  {
    dc *G = malloc(sizeof(dc) * Nb * Nb), *S = malloc(sizeof(dc) * Nb * Nb);
    dc *T = malloc(sizeof(dc) * Nb * Nb), *R = malloc(sizeof(dc) * Nb * Nb);
#pragma omp for schedule(static)
    for (long linear = 0; linear < (long)NE * Nk; ++linear) {
      int e = (int)(linear % NE), m = (int)(linear / NE);
      for (int b = 0; b < Nb; ++b)
        for (int a = 0; a < Nb; ++a) {
          MAT(G, a, b, Nb) = GR[IX(e, m, a, b)];
          MAT(S, a, b, Nb) = sig[IX(e, m, a, b)];
        }
      matmul(Nb, G, S, 0, T);
      matmul(Nb, T, G, 1, R);
      for (int b = 0; b < Nb; ++b)
        for (int a = 0; a < Nb; ++a) out[IX(e, m, a, b)] = MAT(R, a, b, Nb);
    }
    free(G); free(S); free(T); free(R);
  }
}

/* greater_green (greens.jl:84-93): G> = GR - GR^H + G<. */
void orc_greater_green(int NE, int Nk, int Nb, const dc *GR, const dc *GL, dc *GG) {
  for (int b = 0; b < Nb; ++b)
    for (int a = 0; a < Nb; ++a)
      for (int m = 0; m < Nk; ++m)
        for (int e = 0; e < NE; ++e)
          GG[IX(e, m, a, b)] = GR[IX(e, m, a, b)] - conj(GR[IX(e, m, b, a)]) + GL[IX(e, m, a, b)];
}

/* spectral_function (greens.jl:50-57): A = i (GR - GR^H). */
void orc_spectral_function(int NE, int Nk, int Nb, const dc *GR, dc *A) {
  for (int b = 0; b < Nb; ++b)
    for (int a = 0; a < Nb; ++a)
      for (int m = 0; m < Nk; ++m)
        for (int e = 0; e < NE; ++e)
          A[IX(e, m, a, b)] = I * (GR[IX(e, m, a, b)] - conj(GR[IX(e, m, b, a)]));
}

/* Sum_{e,m} wE_e wk_m tr X_em in the reference's serial order (e outer, m
 * inner; number_functional greens.jl:100-110 and
 * _number_functional_production production_operators.jl:1417-1445). */
dc orc_weighted_trace(int NE, int Nk, int Nb, const dc *X, const double *wE, const double *wk) {
  dc value = 0;
  for (int e = 0; e < NE; ++e)
    for (int m = 0; m < Nk; ++m) {
      dc tr = 0;
      for (int a = 0; a < Nb; ++a) tr += X[IX(e, m, a, a)];
      value += wE[e] * wk[m] * tr;
    }
  return value;
}

/* number_functional (greens.jl:100-110): N = Re[-i g_s/(2pi) sum wE wk tr G<]
 * with the realness check (DomainError when |Im| > limit*max(|Re|,1)). */
int orc_number_functional(int NE, int Nk, int Nb, const dc *GL, const double *wE,
                          const double *wk, int gs, double realness_limit, double *out) {
  dc value = orc_weighted_trace(NE, Nk, Nb, GL, wE, wk) * (-I * gs / (2 * M_PI));
  *out = creal(value);
  if (!(fabs(cimag(value)) <= realness_limit * fmax(fabs(creal(value)), 1.0))) return ORC_DOMAIN;
  return ORC_OK;
}

/* _paired_number_coefficients (greens.jl:155-185). */
int orc_paired_coefficients(double number, double holes, double target, double *a,
                            double *c, double *lambda) {
  if (!(isfinite(target) && target > 0)) return ORC_ARG;
  if (!(isfinite(number) && number > 0)) return ORC_DOMAIN;
  if (!(isfinite(holes) && holes >= 0)) return ORC_DOMAIN;
  if (!(target <= number + holes)) return ORC_DOMAIN;
  *lambda = number / target;
  if (number >= target) {
    *a = target / number;
    *c = 0.0;
  } else {
    *a = 1.0;
    *c = (target - number) / holes;
  }
  return ORC_OK;
}

/* _normalize_keldysh_pair! (greens.jl:188-199) / production_state.jl:62-70. */
void orc_normalize_pair(size_t n, dc *GL, dc *GG, double a, double c) {
  for (size_t i = 0; i < n; ++i) {
    dc l = GL[i], g = GG[i];
    GL[i] = a * l - c * g;
    GG[i] = (1 - c) * g - (1 - a) * l;
  }
}

/* ------------------------------------------------------------------------ */
/* Energy shifts                                                             */
/* ------------------------------------------------------------------------ */

/* build_shift_plan (numerics/optimized/production_cache.jl:258-290), 0-based
 * left/right.  Equivalent to the dense build_shift_matrix
 * (numerics/reference/periodicity.jl:11-33). */
int orc_shift_plan(int NE, const double *eps, double delta, int *left, int *right,
                   double *theta, unsigned char *valid) {
  if (NE < 2 || !isfinite(delta)) return ORC_ARG;
  for (int e = 1; e < NE; ++e)
    if (!(eps[e] > eps[e - 1]) || !isfinite(eps[e])) return ORC_ARG;
  int j = 0;
  for (int e = 0; e < NE; ++e) {
    double target = eps[e] + delta;
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
  return ORC_OK;
}

/* apply_energy_shift! (production_cache.jl:300-325) on columns of length NE. */
void orc_apply_shift(int NE, size_t ncols, const int *left, const int *right,
                     const double *theta, const unsigned char *valid, const dc *X, dc *Y) {
  for (size_t col = 0; col < ncols; ++col) {
    const dc *x = X + col * NE;
    dc *y = Y + col * NE;
    for (int e = 0; e < NE; ++e) {
      if (!valid[e]) {
        y[e] = 0;
        continue;
      }
      int l = left[e], r = right[e];
      double t = theta[e];
      y[e] = (l == r || t == 0.0) ? x[l] : (1 - t) * x[l] + t * x[r];
    }
  }
}

/* Dense shift matrix row application, the educational form
 * (periodicity.jl:11-33, applied by apply_energy_shift periodicity.jl:85-94). */
void orc_shift_matrix(int NE, const double *eps, double delta, double *W /* NE x NE col-major */) {
  memset(W, 0, sizeof(double) * (size_t)NE * NE);
  for (int e = 0; e < NE; ++e) {
    double target = eps[e] + delta;
    if (target < eps[0] || target > eps[NE - 1]) continue;
    if (target == eps[NE - 1]) {
      W[e + (size_t)NE * (NE - 1)] = 1.0;
      continue;
    }
    /* searchsortedlast, clamped to [1, N-1] (1-based) */
    int j = 0;
    while (j + 1 < NE && eps[j + 1] <= target) ++j;
    if (j > NE - 2) j = NE - 2;
    double th = (target - eps[j]) / (eps[j + 1] - eps[j]);
    W[e + (size_t)NE * j] = 1 - th;
    W[e + (size_t)NE * (j + 1)] = th;
  }
}

/* ------------------------------------------------------------------------ */
/* Static contractions                                                       */
/* ------------------------------------------------------------------------ */

/* _static_contraction (numerics/reference/kernels.jl:416-435):
 * S[e,m,a,b] = q sum_{m',c,d} wk[m'] K[m,m',a,c,d,b] G[e,m',c,d].
 * K is (Nk,Nk,Nb,Nb,Nb,Nb) col-major. */
void orc_contraction_literal(int NE, int Nk, int Nb, const dc *K, const dc *G,
                             const double *wk, double q, dc *S) {
  size_t sk[6] = {1, (size_t)Nk, (size_t)Nk * Nk, (size_t)Nk * Nk * Nb,
                  (size_t)Nk * Nk * Nb * Nb, (size_t)Nk * Nk * Nb * Nb * Nb};
#pragma omp parallel for collapse(2) schedule(static)
  for (int e = 0; e < NE; ++e)
    for (int m = 0; m < Nk; ++m)
      for (int a = 0; a < Nb; ++a)
        for (int b = 0; b < Nb; ++b) {
          dc value = 0;
          for (int mp = 0; mp < Nk; ++mp)
            for (int c = 0; c < Nb; ++c)
              for (int d = 0; d < Nb; ++d)
                value += wk[mp] * K[m * sk[0] + mp * sk[1] + a * sk[2] + c * sk[3] + d * sk[4] + b * sk[5]] *
                         G[IX(e, mp, c, d)];
          S[IX(e, m, a, b)] = q * value;
        }
}

/* MomentumIndependentProductionKernel contraction
 * (production_operators.jl:535-595): X[(c,d),e] = sum_m' wk G[e,m',c,d];
 * Y = B X with B[(a,b),(c,d)] = K[1,1,a,c,d,b]; S = beta S + alpha q Y
 * broadcast over m.  `block` is B as an (N^2, N^2) column-major matrix, rows
 * (a,b) and columns (c,d), first index fastest (production_cache.jl:396-399). */
void orc_contraction_momentum_independent(int NE, int Nk, int Nb, const dc *block,
                                          const dc *G, const double *wk, double alpha_q,
                                          double beta, dc *S) {
  int N2 = Nb * Nb;
#pragma omp parallel
  {
    dc *X = malloc(sizeof(dc) * N2);
    dc *Y = malloc(sizeof(dc) * N2);
#pragma omp for schedule(static)
    for (int e = 0; e < NE; ++e) {
      for (int d = 0; d < Nb; ++d)
        for (int c = 0; c < Nb; ++c) {
          dc s = 0;
          for (int mp = 0; mp < Nk; ++mp) s += wk[mp] * G[IX(e, mp, c, d)];
          X[c + Nb * d] = s;
        }
      for (int b = 0; b < Nb; ++b)
        for (int a = 0; a < Nb; ++a) {
          dc s = 0;
          for (int d = 0; d < Nb; ++d)
            for (int c = 0; c < Nb; ++c)
              s += block[(a + (size_t)Nb * b) + (size_t)N2 * (c + (size_t)Nb * d)] * X[c + Nb * d];
          Y[a + Nb * b] = s;
        }
      for (int b = 0; b < Nb; ++b)
        for (int a = 0; a < Nb; ++a)
          for (int m = 0; m < Nk; ++m) {
            size_t ix = IX(e, m, a, b);
            S[ix] = (beta == 0.0 ? 0.0 : beta * S[ix]) + alpha_q * Y[a + Nb * b];
          }
    }
    free(X); free(Y);
  }
}

/* DenseProductionKernel contraction (production_operators.jl:402-465):
 * M has rows (m,a,b) and columns (m',c,d), first index fastest, size
 * (Nk Nb^2)^2, col-major.  S = beta S + alpha q M (wk .* G). */
void orc_contraction_dense(int NE, int Nk, int Nb, const dc *M, const dc *G,
                           const double *wk, double alpha_q, double beta, dc *S) {
  size_t Nc = (size_t)Nk * Nb * Nb;
#pragma omp parallel for schedule(static)
  for (int e = 0; e < NE; ++e)
    for (size_t row = 0; row < Nc; ++row) {
      dc s = 0;
      for (size_t col = 0; col < Nc; ++col) {
        int mp = (int)(col % Nk);
        s += M[row + Nc * col] * wk[mp] * G[e + (size_t)NE * col];
      }
      size_t ix = e + (size_t)NE * row;
      S[ix] = (beta == 0.0 ? 0.0 : beta * S[ix]) + alpha_q * s;
    }
}

/* LowRankProductionKernel contraction (production_operators.jl:597-658):
 * S[e,q] = beta S + alpha q sum_r left[q,r] sum_q' right_adjoint[r,q']
 *          wk[q' % Nk] G[e,q'], q = (m,a,b) with m fastest. */
void orc_contraction_low_rank(int NE, int Nk, int Nb, int rank, const dc *left /* Nc x rank */,
                              const dc *right /* rank x Nc */, const dc *G, const double *wk,
                              double alpha_q, double beta, dc *S) {
  size_t Nc = (size_t)Nk * Nb * Nb;
#pragma omp parallel
  {
    dc *T = malloc(sizeof(dc) * (rank > 0 ? rank : 1));
#pragma omp for schedule(static)
    for (int e = 0; e < NE; ++e) {
      for (int r = 0; r < rank; ++r) {
        dc s = 0;
        for (size_t q = 0; q < Nc; ++q) s += right[r + (size_t)rank * q] * wk[q % Nk] * G[e + (size_t)NE * q];
        T[r] = s;
      }
      for (size_t q = 0; q < Nc; ++q) {
        dc s = 0;
        for (int r = 0; r < rank; ++r) s += left[q + Nc * r] * T[r];
        size_t ix = e + (size_t)NE * q;
        S[ix] = (beta == 0.0 ? 0.0 : beta * S[ix]) + alpha_q * s;
      }
    }
    free(T);
  }
}

/* _SeparableIFRProductionKernel contraction (production_operators.jl:467-533):
 * S[e,m,(a,b)] = beta S + alpha q sum_j left[(a,b),j] sum_m' radial[m,m']
 *                wk[m'] sum_(c,d) right[j,(c,d)] G[e,m',c,d]. */
void orc_contraction_ifr(int NE, int Nk, int Nb, int J, const dc *left /* N2 x J */,
                         const dc *right /* J x N2 */, const dc *radial /* Nk x Nk */,
                         const dc *G, const double *wk, double alpha_q, double beta, dc *S) {
  int N2 = Nb * Nb;
#pragma omp parallel
  {
    dc *T = malloc(sizeof(dc) * J * Nk);
    dc *F = malloc(sizeof(dc) * J * Nk);
#pragma omp for schedule(static)
    for (int e = 0; e < NE; ++e) {
      for (int mp = 0; mp < Nk; ++mp)
        for (int j = 0; j < J; ++j) {
          dc s = 0;
          for (int p = 0; p < N2; ++p) s += right[j + (size_t)J * p] * G[e + (size_t)NE * (mp + (size_t)Nk * p)];
          T[j + J * mp] = wk[mp] * s;
        }
      for (int m = 0; m < Nk; ++m)
        for (int j = 0; j < J; ++j) {
          dc s = 0;
          for (int mp = 0; mp < Nk; ++mp) s += radial[m + (size_t)Nk * mp] * T[j + J * mp];
          F[j + J * m] = s;
        }
      for (int p = 0; p < N2; ++p)
        for (int m = 0; m < Nk; ++m) {
          dc s = 0;
          for (int j = 0; j < J; ++j) s += left[p + (size_t)N2 * j] * F[j + J * m];
          size_t ix = e + (size_t)NE * (m + (size_t)Nk * p);
          S[ix] = (beta == 0.0 ? 0.0 : beta * S[ix]) + alpha_q * s;
        }
    }
    free(T); free(F);
  }
}

/* ------------------------------------------------------------------------ */
/* Hilbert transform                                                         */
/* ------------------------------------------------------------------------ */

/* _direct_hilbert_ordered (numerics/reference/kernels.jl:457-481): the
 * principal-value sum over e' != e accumulated symmetrically by distance
 * (reverse=1 gives the opposite order used for the roundoff estimate). */
void orc_direct_hilbert(int NE, size_t ncols, const double *eps, const double *wE,
                        const dc *Gam, dc *Lam, int reverse) {
  int *order = malloc(sizeof(int) * (NE > 1 ? NE - 1 : 1));
  for (int e = 0; e < NE; ++e) {
    int count = 0;
    int span = (e > NE - 1 - e) ? e : NE - 1 - e;
    for (int d = 1; d <= span; ++d) {
      if (e - d >= 0) order[count++] = e - d;
      if (e + d <= NE - 1) order[count++] = e + d;
    }
    if (reverse)
      for (int i = 0; i < count / 2; ++i) {
        int t = order[i];
        order[i] = order[count - 1 - i];
        order[count - 1 - i] = t;
      }
    for (size_t col = 0; col < ncols; ++col) Lam[e + (size_t)NE * col] = 0;
    for (int i = 0; i < count; ++i) {
      int ep = order[i];
      double factor = wE[ep] / (2 * M_PI * (eps[e] - eps[ep]));
      for (size_t col = 0; col < ncols; ++col)
        Lam[e + (size_t)NE * col] += factor * Gam[ep + (size_t)NE * col];
    }
  }
  free(order);
}

/* In-place iterative radix-2 FFT; sign -1 forward, +1 inverse (unnormalised). */
static void fft_inplace_tw(int L, dc *x, int sign, const dc *tw /* exp(-2 pi i t / L), t < L/2 */) {
  for (int i = 1, j = 0; i < L; ++i) {
    int bit = L >> 1;
    for (; j & bit; bit >>= 1) j ^= bit;
    j ^= bit;
    if (i < j) {
      dc t = x[i];
      x[i] = x[j];
      x[j] = t;
    }
  }
  for (int len = 2; len <= L; len <<= 1) {
    int step = L / len;
    for (int i = 0; i < L; i += len)
      for (int k = 0; k < len / 2; ++k) {
        dc w = tw[k * step];
        if (sign > 0) w = conj(w);
        dc u = x[i + k], v = cmul(x[i + k + len / 2], w);
        x[i + k] = u + v;
        x[i + k + len / 2] = u - v;
      }
  }
}

static void fft_inplace(int L, dc *x, int sign) {
  for (int i = 1, j = 0; i < L; ++i) {
    int bit = L >> 1;
    for (; j & bit; bit >>= 1) j ^= bit;
    j ^= bit;
    if (i < j) {
      dc t = x[i];
      x[i] = x[j];
      x[j] = t;
    }
  }
  for (int len = 2; len <= L; len <<= 1) {
    double ang = sign * 2 * M_PI / len;
    for (int i = 0; i < L; i += len)
      for (int k = 0; k < len / 2; ++k) {
        dc w = cos(ang * k) + I * sin(ang * k);
        dc u = x[i + k], v = x[i + k + len / 2] * w;
        x[i + k] = u + v;
        x[i + k + len / 2] = u - v;
      }
  }
}

static int next_pow2(int n) {
  int L = 1;
  while (L < n) L <<= 1;
  return L;
}

/* The zero-padded linear-convolution Hilbert transform
 * (_fft_hilbert_with_length, numerics/optimized/production_operators.jl:735-781,
 * and ProductionFFTHilbertPlan, numerics/optimized/fft_parallel.jl:74-225):
 * kernel[lag + NE - 1] = 1/(2 pi lag de) for 0 < |lag| < NE, buffer = wE .* Gam
 * padded to L, output Lam_e = conv[e + NE - 1].  L = 0 picks nextpow2(2NE-1). */
int orc_fft_hilbert(int NE, size_t ncols, const double *eps, const double *wE,
                    const dc *Gam, dc *Lam, int L) {
  if (L == 0) L = next_pow2(2 * NE - 1);
  if (L < 2 * NE - 1 || NE < 2) return ORC_ARG;
  double de = eps[1] - eps[0];
  dc *kernel = calloc(L, sizeof(dc));
  for (int lag = -(NE - 1); lag <= NE - 1; ++lag)
    if (lag != 0) kernel[lag + NE - 1] = 1.0 / (2 * M_PI * lag * de);
  fft_inplace(L, kernel, -1);
  dc *tw = malloc(sizeof(dc) * (L / 2 + 1));
  for (int t = 0; t < L / 2; ++t) tw[t] = cos(2 * M_PI * t / L) - I * sin(2 * M_PI * t / L);
#pragma omp parallel
  {
    dc *buf = malloc(sizeof(dc) * L);
#pragma omp for schedule(static)
    for (long col = 0; col < (long)ncols; ++col) {
      for (int i = 0; i < L; ++i) buf[i] = 0;
      for (int e = 0; e < NE; ++e) buf[e] = wE[e] * Gam[e + (size_t)NE * col];
      fft_inplace_tw(L, buf, -1, tw);
      for (int i = 0; i < L; ++i) buf[i] = cmul(buf[i], kernel[i]);
      fft_inplace_tw(L, buf, +1, tw);
      for (int e = 0; e < NE; ++e) Lam[e + (size_t)NE * col] = buf[e + NE - 1] / L;
    }
    free(buf);
  }
  free(tw);
  free(kernel);
  return ORC_OK;
}

/* fft_hilbert_transform with return_roundoff (production_operators.jl:
 * 793-809): ||Lam(2L) - Lam(L)|| / (||Lam(L)|| + 1e-14). */
int orc_fft_hilbert_roundoff(int NE, size_t ncols, const double *eps, const double *wE,
                             const dc *Gam, dc *Lam, double *roundoff) {
  int L = next_pow2(2 * NE - 1);
  int st = orc_fft_hilbert(NE, ncols, eps, wE, Gam, Lam, L);
  if (st) return st;
  dc *second = malloc(sizeof(dc) * NE * ncols);
  orc_fft_hilbert(NE, ncols, eps, wE, Gam, second, 2 * L);
  double num = 0, den = 0;
  for (size_t i = 0; i < (size_t)NE * ncols; ++i) {
    dc d = second[i] - Lam[i];
    num += creal(d * conj(d));
    den += creal(Lam[i] * conj(Lam[i]));
  }
  *roundoff = sqrt(num) / (sqrt(den) + 1e-14);
  free(second);
  return ORC_OK;
}

/* retarded_self_energy(_fft) (kernels.jl:600-615, production_operators.jl:
 * 842-884): Gam = i (S> - S<), SR = H[Gam] - i Gam / 2.  method 0 = FFT,
 * 1 = direct PV.  roundoff may be NULL. */
int orc_retarded_self_energy(int NE, size_t ncols, const double *eps, const double *wE,
                             const dc *SL, const dc *SG, dc *SR, dc *Gam_out, int method,
                             double *roundoff) {
  size_t n = (size_t)NE * ncols;
  dc *Gam = malloc(sizeof(dc) * n);
  for (size_t i = 0; i < n; ++i) Gam[i] = I * (SG[i] - SL[i]);
  int st = ORC_OK;
  if (method == 0) {
    if (roundoff) st = orc_fft_hilbert_roundoff(NE, ncols, eps, wE, Gam, SR, roundoff);
    else st = orc_fft_hilbert(NE, ncols, eps, wE, Gam, SR, 0);
  } else {
    orc_direct_hilbert(NE, ncols, eps, wE, Gam, SR, 0);
    if (roundoff) {
      dc *rev = malloc(sizeof(dc) * n);
      orc_direct_hilbert(NE, ncols, eps, wE, Gam, rev, 1);
      double num = 0, den = 0;
      for (size_t i = 0; i < n; ++i) {
        dc d = SR[i] - rev[i];
        num += creal(d * conj(d));
        den += creal(SR[i] * conj(SR[i]));
      }
      *roundoff = sqrt(num) / (sqrt(den) + 1e-14);
      free(rev);
    }
  }
  for (size_t i = 0; i < n; ++i) SR[i] = SR[i] - 0.5 * I * Gam[i];
  if (Gam_out) memcpy(Gam_out, Gam, sizeof(dc) * n);
  free(Gam);
  return st;
}

/* ------------------------------------------------------------------------ */
/* Embedding                                                                 */
/* ------------------------------------------------------------------------ */

/* _embedding_component_production (production_operators.jl:886-922):
 * S_em = T G~_em T^H with G~ the shifted (interpolated) field; invalid rows
 * are zero.  Equals _embedding_component(T, apply_energy_shift(W, G))
 * (periodicity.jl:113-120). */
void orc_embedding_component(int NE, int Nk, int Nb, const dc *T, const dc *G,
                             const int *left, const int *right, const double *theta,
                             const unsigned char *valid, dc *S) {
#pragma omp parallel
  {
    dc *X = malloc(sizeof(dc) * Nb * Nb), *Tm = malloc(sizeof(dc) * Nb * Nb);
    dc *R = malloc(sizeof(dc) * Nb * Nb);
#pragma omp for schedule(static)
    for (long linear = 0; linear < (long)NE * Nk; ++linear) {
      int e = (int)(linear % NE), m = (int)(linear / NE);
      if (!valid[e]) {
        for (int b = 0; b < Nb; ++b)
          for (int a = 0; a < Nb; ++a) S[IX(e, m, a, b)] = 0;
        continue;
      }
      int l = left[e], r = right[e];
      double t = theta[e];
      for (int b = 0; b < Nb; ++b)
        for (int a = 0; a < Nb; ++a)
          MAT(X, a, b, Nb) = (l == r || t == 0.0) ? G[IX(l, m, a, b)]
                                                  : (1 - t) * G[IX(l, m, a, b)] + t * G[IX(r, m, a, b)];
      matmul(Nb, T, X, 0, Tm);
      matmul(Nb, Tm, T, 1, R);
      for (int b = 0; b < Nb; ++b)
        for (int a = 0; a < Nb; ++a) S[IX(e, m, a, b)] = MAT(R, a, b, Nb);
    }
    free(X); free(Tm); free(R);
  }
}

/* ------------------------------------------------------------------------ */
/* Observables                                                               */
/* ------------------------------------------------------------------------ */

/* _production_boundary_flux_bar (numerics/optimized/production_iteration.jl:
 * 174-201) = _boundary_flux_bar (physics/observables.jl:176-214):
 * Jbar = Re[g_s/(2pi) sum_{e in (|eps|,eps) order} sum_m wE wk
 *        tr(S> G< - S< G>)]. */
double orc_current(int NE, int Nk, int Nb, const double *eps, const double *wE,
                   const double *wk, int gs, const dc *SG, const dc *SL, const dc *GL,
                   const dc *GG) {
  int *order = malloc(sizeof(int) * NE);
  for (int e = 0; e < NE; ++e) order[e] = e;
  /* stable insertion sort by (|eps|, eps) */
  for (int i = 1; i < NE; ++i) {
    int v = order[i];
    int j = i - 1;
    while (j >= 0) {
      double ka = fabs(eps[order[j]]), kb = fabs(eps[v]);
      int greater = ka > kb || (ka == kb && eps[order[j]] > eps[v]);
      if (!greater) break;
      order[j + 1] = order[j];
      --j;
    }
    order[j + 1] = v;
  }
  dc value = 0;
  for (int i = 0; i < NE; ++i) {
    int e = order[i];
    for (int m = 0; m < Nk; ++m) {
      dc tr = 0;
      for (int a = 0; a < Nb; ++a) {
        dc out = 0, in = 0;
        for (int b = 0; b < Nb; ++b) {
          out += SG[IX(e, m, a, b)] * GL[IX(e, m, b, a)];
          in += SL[IX(e, m, a, b)] * GG[IX(e, m, b, a)];
        }
        tr += out - in;
      }
      value += wE[e] * wk[m] * tr;
    }
  }
  free(order);
  return creal(gs * value / (2 * M_PI));
}

/* _production_state_populations (production_iteration.jl:204-215):
 * p_a = Re[-i g_s/(2pi) sum wE wk G<_{em,aa}] / target. */
void orc_populations(int NE, int Nk, int Nb, const double *wE, const double *wk, int gs,
                     double target, const dc *GL, double *pop) {
  dc pre = -I * gs / (2 * M_PI);
  for (int a = 0; a < Nb; ++a) {
    dc s = 0;
    for (int e = 0; e < NE; ++e)
      for (int m = 0; m < Nk; ++m) s += pre * wE[e] * wk[m] * GL[IX(e, m, a, a)];
    pop[a] = creal(s) / target;
  }
}

/* _mix (kernels.jl:676-691), _mix_family_production! (production_operators.jl:
 * 1475-1490): X <- (1 - alpha) X + alpha Y. */
void orc_mix(size_t n, dc *X, const dc *Y, double alpha) {
  double beta = 1 - alpha;
  for (size_t i = 0; i < n; ++i) X[i] = beta * X[i] + alpha * Y[i];
}

/* norm(Y - X) / (norm(Y) + 1e-14) for one component (_selfenergy_residual,
 * validation.jl:78-86; production_selfenergy_residual residuals.jl:802-865). */
double orc_relative_change(size_t n, const dc *Xold, const dc *Ynew) {
  double num = 0, den = 0;
  for (size_t i = 0; i < n; ++i) {
    dc d = Ynew[i] - Xold[i];
    num += creal(d * conj(d));
    den += creal(Ynew[i] * conj(Ynew[i]));
  }
  if (!isfinite(num) || !isfinite(den)) return INFINITY;
  return sqrt(num) / (sqrt(den) + 1e-14);
}

/* ------------------------------------------------------------------------ */
/* Residual suite                                                            */
/* ------------------------------------------------------------------------ */

/* psd_error_budget (numerics/reference/positivity_diagnostics.jl:15-40) and
 * the witness ratio (:60-90): ratio = max(0, -lmin - 64 n eps max(|l|)) /
 * max(|l|). */
static double negative_part(int n, const dc *X, dc factor, dc *H, double *vals) {
  for (int j = 0; j < n; ++j)
    for (int i = 0; i < n; ++i) {
      dc v = factor * MAT(X, i, j, n);
      dc w = factor * MAT(X, j, i, n);
      if (!isfinite(creal(v)) || !isfinite(cimag(v))) return INFINITY;
      MAT(H, i, j, n) = 0.5 * (v + conj(w));
    }
  orc_hermitian_eigvals(n, H, vals);
  double lmin = vals[0], bn = 0;
  for (int i = 0; i < n; ++i) bn = fmax(bn, fabs(vals[i]));
  double budget = 64.0 * n * 2.220446049250313e-16 * fmax(bn, 1.0);
  double absolute = fmax(0.0, -lmin);
  return fmax(0.0, absolute - budget) / fmax(bn, 2.2250738585072014e-308);
}

/* One witness candidate (_positivity_witness, numerics/reference/
 * positivity_diagnostics.jl:61-91) for the Hermitian part of f X: w[0..8] =
 * minimum_eigenvalue, block_norm, floor, ratio, absolute_defect,
 * relative_defect, backward_error, hermiticity_defect, construction_scale.
 * Returns 0 when X is non-finite (no candidate). */
static int witness_candidate(int n, const dc *X, dc f, dc *H, double *vals, double *w) {
  double herm = 0;
  for (int j = 0; j < n; ++j)
    for (int i = 0; i < n; ++i) {
      dc v = f * MAT(X, i, j, n), u = f * MAT(X, j, i, n);
      if (!isfinite(creal(v)) || !isfinite(cimag(v))) return 0;
      MAT(H, i, j, n) = 0.5 * (v + conj(u));
      dc d = v - conj(u);
      herm += creal(d * conj(d));
    }
  orc_hermitian_eigvals(n, H, vals);
  double lmin = vals[0], bn = 0;
  for (int i = 0; i < n; ++i) bn = fmax(bn, fabs(vals[i]));
  double budget = 64.0 * n * 2.220446049250313e-16 * fmax(bn, 1.0);
  double absolute = fmax(0.0, -lmin), den = fmax(bn, 2.2250738585072014e-308);
  w[0] = lmin; w[1] = bn; w[2] = budget; w[3] = fmax(0.0, absolute - budget) / den;
  w[4] = absolute; w[5] = absolute / den; w[6] = budget; w[7] = sqrt(herm) / 2; w[8] = 1.0;
  return 1;
}

/* The positivity witness of production_residual_suite
 * (numerics/optimized/residuals.jl:662-726 collecting per chunk,
 * _production_positivity_witness :773-779 reducing): over the blocks in the
 * reference's order (e slow, m fast; residuals.jl:126-131) and the matrices
 * in the order spectral A, occupied -iG<, unoccupied iG>, broadening Gam,
 * raw occupied -i G S< G^H, raw unoccupied i G S> G^H (kinds 0..5), the
 * first candidate with the largest ratio.  A non-finite primary matrix
 * (kinds 0..3) is a candidate of ratio Inf with NaN eigen data
 * (_nonfinite_positivity_witness, positivity_diagnostics.jl:56-57); a
 * non-finite raw product is not a candidate.  ikem = {kind, e, m} 0-based
 * (kind -1: none), w as in witness_candidate.  Single-threaded. */
void orc_residual_witness(int NE, int Nk, int Nb, const dc *GR, const dc *GL, const dc *GG, const dc *SLt,
                          const dc *SGt, int *ikem, double *w) {
  int n = Nb;
  dc *G = malloc(sizeof(dc) * n * n), *X = malloc(sizeof(dc) * n * n), *H = malloc(sizeof(dc) * n * n);
  dc *T1 = malloc(sizeof(dc) * n * n), *T2 = malloc(sizeof(dc) * n * n);
  double *vals = malloc(sizeof(double) * n), cand[9];
  const double empty[9] = {0.0, 0.0, 0.0, -1.0, 0.0, 0.0, 0.0, 0.0, 1.0};
  const dc factors[6] = {1.0, -I, I, 1.0, -I, I};
  for (int k = 0; k < 9; ++k) w[k] = empty[k];
  ikem[0] = -1; ikem[1] = 0; ikem[2] = 0;
  for (int e = 0; e < NE; ++e)
    for (int m = 0; m < Nk; ++m) {
      for (int b = 0; b < n; ++b)
        for (int a = 0; a < n; ++a) MAT(G, a, b, n) = GR[IX(e, m, a, b)];
      for (int kind = 0; kind < 6; ++kind) {
        for (int b = 0; b < n; ++b)
          for (int a = 0; a < n; ++a) {
            size_t ix = IX(e, m, a, b);
            dc v = 0;
            if (kind == 0) v = I * (MAT(G, a, b, n) - conj(MAT(G, b, a, n)));
            else if (kind == 1) v = GL[ix];
            else if (kind == 2) v = GG[ix];
            else if (kind == 3) v = I * (SGt[ix] - SLt[ix]);
            else v = kind == 4 ? SLt[ix] : SGt[ix];
            MAT(X, a, b, n) = v;
          }
        if (kind >= 4) {
          matmul(n, G, X, 0, T1);
          matmul(n, T1, G, 1, T2);
          memcpy(X, T2, sizeof(dc) * n * n);
        }
        int ok = witness_candidate(n, X, factors[kind], H, vals, cand);
        if (!ok) {
          if (kind >= 4) continue;
          const double nf[9] = {NAN, INFINITY, 1e-14, INFINITY, NAN, NAN, 1e-14, 0.0, 1.0};
          memcpy(cand, nf, sizeof(nf));
        }
        if (cand[3] > w[3]) {
          memcpy(w, cand, sizeof(cand));
          ikem[0] = kind; ikem[1] = e; ikem[2] = m;
        }
      }
    }
  free(G); free(X); free(H); free(T1); free(T2); free(vals);
}

/* production_residual_suite (numerics/optimized/residuals.jl:537-770), with
 * the definitions of validation.jl:33-103.  out = {rD, rA, rK, rPSD, rcaus}.
 * A = i(GR - GR^H) is formed per block; Gam = i(SG_total - SL_total). */
void orc_residual_suite(int NE, int Nk, int Nb, const double *eps, const dc *h,
                        const dc *GR, const dc *GL, const dc *GG, const dc *SRt,
                        const dc *SLt, const dc *SGt, const dc *SLcand, double *out) {
  double rD = 0, rPSD = 0, rcaus = 0;
  double aNum = 0, aDen = 0, kNum = 0, kDen = 0;
  long blocks = (long)NE * Nk;
  double *part = calloc(4 * blocks, sizeof(double));
#pragma omp parallel reduction(max : rD, rPSD, rcaus)
  {
    int n = Nb;
    dc *D = malloc(sizeof(dc) * n * n), *G = malloc(sizeof(dc) * n * n);
    dc *X = malloc(sizeof(dc) * n * n), *Y = malloc(sizeof(dc) * n * n);
    dc *T1 = malloc(sizeof(dc) * n * n), *T2 = malloc(sizeof(dc) * n * n);
    dc *H = malloc(sizeof(dc) * n * n), *Gam = malloc(sizeof(dc) * n * n);
    dc *A = malloc(sizeof(dc) * n * n);
    double *vals = malloc(sizeof(double) * n);
#pragma omp for schedule(static)
    for (long linear = 0; linear < blocks; ++linear) {
      int e = (int)(linear % NE), m = (int)(linear / NE);
      for (int b = 0; b < n; ++b)
        for (int a = 0; a < n; ++a) {
          MAT(D, a, b, n) = ((a == b) ? eps[e] : 0.0) - h[(size_t)m + (size_t)Nk * (a + (size_t)n * b)] -
                            SRt[IX(e, m, a, b)];
          MAT(G, a, b, n) = GR[IX(e, m, a, b)];
          MAT(Gam, a, b, n) = I * (SGt[IX(e, m, a, b)] - SLt[IX(e, m, a, b)]);
        }
      for (int b = 0; b < n; ++b)
        for (int a = 0; a < n; ++a) MAT(A, a, b, n) = I * (MAT(G, a, b, n) - conj(MAT(G, b, a, n)));
      /* r_D */
      matmul(n, D, G, 0, T1);
      for (int i = 0; i < n; ++i) MAT(T1, i, i, n) -= 1;
      double v = frob(n, T1) / (frob(n, D) * frob(n, G) + sqrt((double)n));
      rD = fmax(rD, isfinite(v) ? v : INFINITY);
      /* r_A numerator/denominator */
      matmul(n, G, Gam, 0, T1);
      matmul(n, T1, G, 1, T2);
      double num = 0, den = 0;
      for (int i = 0; i < n * n; ++i) {
        dc d = A[i] - T2[i];
        num += creal(d * conj(d));
        den += creal(A[i] * conj(A[i]));
      }
      part[4 * linear + 0] = num;
      part[4 * linear + 1] = den;
      /* r_K against the candidate lesser self-energy */
      for (int b = 0; b < n; ++b)
        for (int a = 0; a < n; ++a) MAT(X, a, b, n) = SLcand[IX(e, m, a, b)];
      matmul(n, G, X, 0, T1);
      matmul(n, T1, G, 1, T2);
      num = den = 0;
      for (int b = 0; b < n; ++b)
        for (int a = 0; a < n; ++a) {
          dc gl = GL[IX(e, m, a, b)];
          dc d = gl - MAT(T2, a, b, n);
          num += creal(d * conj(d));
          den += creal(gl * conj(gl));
        }
      part[4 * linear + 2] = num;
      part[4 * linear + 3] = den;
      /* r_PSD: A, -iG<, iG>, Gam, -i G S< G^H, i G S> G^H */
      double p = negative_part(n, A, 1.0, H, vals);
      for (int b = 0; b < n; ++b)
        for (int a = 0; a < n; ++a) MAT(X, a, b, n) = GL[IX(e, m, a, b)];
      p = fmax(p, negative_part(n, X, -I, H, vals));
      for (int b = 0; b < n; ++b)
        for (int a = 0; a < n; ++a) MAT(X, a, b, n) = GG[IX(e, m, a, b)];
      p = fmax(p, negative_part(n, X, I, H, vals));
      p = fmax(p, negative_part(n, Gam, 1.0, H, vals));
      for (int b = 0; b < n; ++b)
        for (int a = 0; a < n; ++a) MAT(X, a, b, n) = SLt[IX(e, m, a, b)];
      matmul(n, G, X, 0, T1);
      matmul(n, T1, G, 1, T2);
      p = fmax(p, negative_part(n, T2, -I, H, vals));
      for (int b = 0; b < n; ++b)
        for (int a = 0; a < n; ++a) MAT(X, a, b, n) = SGt[IX(e, m, a, b)];
      matmul(n, G, X, 0, T1);
      matmul(n, T1, G, 1, T2);
      p = fmax(p, negative_part(n, T2, I, H, vals));
      rPSD = fmax(rPSD, p);
      /* r_caus: lambda_max(Im_H SR) / (||SR||_2 + 1e-14) */
      for (int b = 0; b < n; ++b)
        for (int a = 0; a < n; ++a) {
          dc sab = SRt[IX(e, m, a, b)], sba = SRt[IX(e, m, b, a)];
          MAT(H, a, b, n) = (sab - conj(sba)) / (2 * I);
          MAT(X, a, b, n) = sab;
        }
      orc_hermitian_eigvals(n, H, vals);
      double numc = fmax(0.0, vals[n - 1]);
      if (numc > 0) {
        double ns = spectral_norm(n, X, T1, vals);
        rcaus = fmax(rcaus, numc / (ns + 1e-14));
      }
    }
    free(D); free(G); free(X); free(Y); free(T1); free(T2); free(H); free(Gam); free(A); free(vals);
  }
  /* canonical (energy-major) order, like _canonical_sum (residuals.jl:493-503):
   * the reference linearises blocks with e slow, m fast. */
  for (int e = 0; e < NE; ++e)
    for (int m = 0; m < Nk; ++m) {
      long linear = e + (long)NE * m;
      aNum += part[4 * linear + 0];
      aDen += part[4 * linear + 1];
      kNum += part[4 * linear + 2];
      kDen += part[4 * linear + 3];
    }
  free(part);
  out[0] = rD;
  out[1] = sqrt(aNum) / (sqrt(aDen) + 1e-14);
  out[2] = sqrt(kNum) / (sqrt(kDen) + 1e-14);
  out[3] = rPSD;
  out[4] = rcaus;
}

/* ------------------------------------------------------------------------ */
/* Fused Dyson + Keldysh (the batch used by the operator-level benchmark)    */
/* ------------------------------------------------------------------------ */

/* _current_green_production up to the raw products
 * (numerics/optimized/production_state.jl:1-48): GR = Dyson(SR), GL = GR SL
 * GR^H and (if SG != NULL) GG = GR SG GR^H, in one pass over the blocks. */
int orc_dyson_keldysh(int NE, int Nk, int Nb, const double *eps, const dc *h,
                      const dc *SR, const dc *SL, const dc *SG, dc *GR, dc *GL, dc *GG,
                      double *scale) {
  long bad = -1;
  int st = orc_retarded_green(NE, Nk, Nb, eps, 0.0, h, SR, GR, NULL, NULL, scale, &bad);
  if (st) return st;
  orc_keldysh_green(NE, Nk, Nb, GR, SL, GL);
  if (SG) orc_keldysh_green(NE, Nk, Nb, GR, SG, GG);
  return ORC_OK;
}

/* Fermi function with the reference's saturation (numerics/reference/
 * scba.jl:1-6; the threshold _FERMI_EXPONENT_SATURATION is passed in). */
double orc_fermi(double x_energy, double mu, double kBT, double saturation) {
  double x = (x_energy - mu) / kBT;
  if (x > saturation) return 0.0;
  if (x < -saturation) return 1.0;
  return 1.0 / (exp(x) + 1.0);
}
