"""Kernel builders: dense scattering operators assembled on the device.

The reference's momentum-dependent kernels are angular averages of a
transfer-momentum kernel C(q) over the in-plane angle grid (grids.jl:44,
phi_r = 2 pi (r - 1) / N_phi; _angular_average_kernel,
numerics/reference/kernels.jl:5-19).  Both of its construction paths are
linear in node tensors, K(m, m') = sum_t W[(m, m'), t] X_t:

* the exact LO phonon kernel (lo_phonon_kernel, kernels.jl:321-356):
  C(q) = pre sum_h f_h(q) F_h[a,c] conj(F_h[b,d]) with
  f_h(q) = wqz_h L0 / (2 pi (q^2 + qz_h^2 + qs^2)); W is the angular mean of
  pre f_h and X_h = F_h (x) conj(F_h);
* tabulated kernels (_lookup_block / _assemble_lookup_kernel,
  numerics/optimized/kernels.jl:205-217, 303-320): C(q) interpolated linearly
  between node tensors C(q_t); W is the angular mean of the interpolation
  weights.

The host forms W (N_k^2 x T numbers, cheap); ``qcl_assemble_kernel`` writes
the (N_k N_b^2)^2 production matrix and its scale q^K = max|K|
(build_kernels, kernels.jl:393-403) on the GPU.
"""
from __future__ import annotations

import ctypes
import math

import numpy as np

from ._lib import check, lib
from .problem import Mechanism

RANK1, TABLE = 0, 1


def angle_grid(Nphi: int) -> np.ndarray:
    """phi_r = 2 pi (r - 1) / N_phi (grids.jl:44)."""
    return 2 * math.pi * np.arange(Nphi) / Nphi


def transfer_momenta(kappa, Nphi: int) -> np.ndarray:
    """q[m, m', r] = sqrt(max(k_m^2 + k_m'^2 - 2 k_m k_m' cos phi_r, 0))."""
    k = np.asarray(kappa, dtype=np.float64)
    phi = angle_grid(Nphi)
    q2 = k[:, None, None] ** 2 + k[None, :, None] ** 2 - 2 * k[:, None, None] * k[None, :, None] * np.cos(phi)
    return np.sqrt(np.maximum(q2, 0.0))


def lo_form_factors(chi, x, wx, qz) -> np.ndarray:
    """F[h, a, c] = sum_g wx_g conj(chi_ga) exp(i qz_h x_g) chi_gc
    (lo_phonon_kernel, kernels.jl:329-338)."""
    chi = np.asarray(chi, dtype=np.complex128)
    ph = np.exp(1j * np.outer(np.asarray(qz), np.asarray(x)))  # (Nq, Nz)
    return np.einsum("g,ga,hg,gc->hac", np.asarray(wx), np.conj(chi), ph, chi)


def lo_weights(kappa, Nphi: int, qz, wqz, qscreen: float, prefactor: float, L0: float = 1.0) -> np.ndarray:
    """W[(m, m'), h] = prefactor / N_phi sum_r wqz_h L0 / (2 pi (q^2 + qz_h^2 + qs^2)),
    column-major over (m + N_k m', h)."""
    q = transfer_momenta(kappa, Nphi)  # (Nk, Nk, Nphi)
    qz, wqz = np.asarray(qz, dtype=np.float64), np.asarray(wqz, dtype=np.float64)
    f = wqz[None, None, None, :] * L0 / (2 * math.pi * (q[..., None] ** 2 + qz ** 2 + qscreen ** 2))
    W = prefactor * f.mean(axis=2)  # (Nk, Nk, Nq)
    Nk = len(kappa)
    return np.asfortranarray(W.reshape((Nk * Nk, len(qz)), order="F"))


def lookup_weights(nodes, kappa, Nphi: int) -> np.ndarray:
    """W[(m, m'), t]: the angular mean of the linear-interpolation weights of
    _lookup_block (numerics/optimized/kernels.jl:205-217), clamped to the
    node interval within 64 eps (a query outside raises ValueError)."""
    nodes = np.asarray(nodes, dtype=np.float64)
    T = len(nodes)
    qlo, qhi = nodes[0], nodes[-1]
    tol = 64 * np.finfo(np.float64).eps * max(abs(qlo), abs(qhi), 1.0)
    q = transfer_momenta(kappa, Nphi)
    if np.any(q < qlo - tol) or np.any(q > qhi + tol):
        raise ValueError("lookup query lies outside the tabulated interval")
    Nk = len(kappa)
    W = np.zeros((Nk, Nk, T))
    for m in range(Nk):
        for mp in range(Nk):
            for qv in q[m, mp]:
                qc = min(max(qv, qlo), qhi)
                if qc == qhi:
                    W[m, mp, T - 1] += 1.0
                    continue
                j = int(np.clip(np.searchsorted(nodes, qc, side="right") - 1, 0, T - 2))
                th = (qc - nodes[j]) / (nodes[j + 1] - nodes[j])
                W[m, mp, j] += 1 - th
                W[m, mp, j + 1] += th
    W /= Nphi
    return np.asfortranarray(W.reshape((Nk * Nk, T), order="F"))


def impurity_pair_covariance(q, chi, x, wx, donor_weights, q_s, prefactor_scale: float) -> np.ndarray:
    """The screened ionised-donor covariance C(q)[(a,c),(b,d)] of
    _production_impurity_evaluator (numerics/optimized/kernels.jl:122-158):
    V[(a,c), D] = pre(q) sum_g wx_g conj(chi_ga) chi_gc exp(-q |x_g - x_D|),
    pre(q) = prefactor_scale / (q + q_s), C = V diag(w_D) V^H."""
    chi = np.asarray(chi, dtype=np.complex128)
    Nb = chi.shape[1]
    donors = np.nonzero(np.asarray(donor_weights))[0]
    if len(donors) == 0:
        raise ValueError("impurity kernel has no ionized donors")
    pair = (np.asarray(wx)[:, None, None] * np.conj(chi)[:, :, None] * chi[:, None, :]).reshape(
        (len(x), Nb * Nb), order="F")  # [g, a + Nb c]
    dist = np.abs(np.asarray(x)[:, None] - np.asarray(x)[donors][None, :])
    V = prefactor_scale / (q + q_s) * (pair.T @ np.exp(-q * dist))
    return (V * np.asarray(donor_weights)[donors][None, :]) @ np.conj(V).T


def assemble_operator(name: str, form: int, Nk: int, Nb: int, W: np.ndarray, X: np.ndarray) -> Mechanism:
    """Run the device assembly; returns the dense Mechanism (matrix = K / q^K,
    q = q^K).  Raises ValueError for a zero or non-finite kernel (the
    reference declares a zero kernel disabled, kernels.jl:395-401)."""
    W = np.asfortranarray(np.asarray(W, dtype=np.float64))
    T = W.shape[1]
    if W.shape[0] != Nk * Nk:
        raise ValueError("W must have N_k^2 rows")
    X = np.asfortranarray(np.asarray(X, dtype=np.complex128))
    Nc = Nk * Nb * Nb
    M = np.zeros((Nc, Nc), dtype=np.complex128, order="F")
    qK = ctypes.c_double()
    check(lib().qcl_assemble_kernel(form, Nk, Nb, T, ctypes.c_void_p(W.ctypes.data), ctypes.c_void_p(X.ctypes.data),
                                    ctypes.c_void_p(M.ctypes.data), ctypes.byref(qK)))
    if not (qK.value > 0 and math.isfinite(qK.value)):
        raise ValueError(f"kernel {name} has scale {qK.value}: zero or non-finite")
    return Mechanism(name, "dense", float(qK.value), matrix=M)


def assemble_operator_device(name: str, form: int, Nk: int, Nb: int, W: np.ndarray, X: np.ndarray) -> Mechanism:
    """As assemble_operator, with the dense matrix left in device memory (a
    torch CUDA tensor whose transpose view is the column-major operator), for
    operators too large to pass through the host; qcl_scba_create copies it
    device to device."""
    import torch

    W = np.asfortranarray(np.asarray(W, dtype=np.float64))
    T = W.shape[1]
    X = np.asfortranarray(np.asarray(X, dtype=np.complex128))
    Nc = Nk * Nb * Nb
    dev = torch.device("cuda")
    dW = torch.from_numpy(np.ravel(W, order="F")).to(dev)
    dX = torch.from_numpy(np.ravel(X, order="F")).to(dev)
    M = torch.empty((Nc, Nc), dtype=torch.complex128, device=dev)  # row j = column j of the operator
    work = torch.zeros(297, dtype=torch.float64, device=dev)
    stream = torch.cuda.current_stream().cuda_stream
    check(lib().qcl_dev_assemble_kernel(ctypes.c_void_p(stream), form, Nk, Nb, T, ctypes.c_void_p(dW.data_ptr()),
                                        ctypes.c_void_p(dX.data_ptr()), ctypes.c_void_p(M.data_ptr()),
                                        ctypes.c_void_p(work.data_ptr())))
    torch.cuda.synchronize()
    q = float(work[-1].item())
    if not (q > 0 and math.isfinite(q)):
        raise ValueError(f"kernel {name} has scale {q}: zero or non-finite")
    return Mechanism(name, "dense", q, matrix=M)


def lo_kernel_operator(chi, x, wx, qz, wqz, kappa, Nphi: int, qscreen: float, prefactor: float,
                       L0: float = 1.0) -> Mechanism:
    """The LO phonon Mechanism (exact angular form) built on the GPU."""
    F = lo_form_factors(chi, x, wx, qz)  # (Nq, Nb, Nb)
    Nq, Nb = F.shape[0], F.shape[1]
    W = lo_weights(kappa, Nphi, qz, wqz, qscreen, prefactor, L0)
    return assemble_operator("LO", RANK1, len(kappa), Nb, W, F.reshape((Nq, Nb * Nb), order="F"))


def table_kernel_operator(name: str, nodes, covariances, kappa, Nphi: int) -> Mechanism:
    """A tabulated Mechanism built on the GPU from node pair covariances
    C_t[(a,c),(b,d)] (T x N_b^2 x N_b^2)."""
    C = np.asarray(covariances, dtype=np.complex128)
    T, N2 = C.shape[0], C.shape[1]
    Nb = int(round(math.sqrt(N2)))
    X = np.transpose(C, (1, 2, 0))  # [(a,c), (b,d), t] column-major
    W = lookup_weights(nodes, kappa, Nphi)
    return assemble_operator(name, TABLE, len(kappa), Nb, W, X)


def impurity_pair_factors(q, chi, x, wx, donor_weights, q_s, prefactor_scale: float):
    """The factors of the screened ionised-donor covariance at one transfer
    momentum q: C(q) = V diag(w_D) V^H with V[(a,c), D] as in
    impurity_pair_covariance (_production_impurity_evaluator,
    numerics/optimized/kernels.jl:122-158).  Returns (V, w_D) over the doped
    cells only."""
    chi = np.asarray(chi, dtype=np.complex128)
    Nb = chi.shape[1]
    donors = np.nonzero(np.asarray(donor_weights))[0]
    if len(donors) == 0:
        raise ValueError("impurity kernel has no ionized donors")
    pair = (np.asarray(wx)[:, None, None] * np.conj(chi)[:, :, None] * chi[:, None, :]).reshape(
        (len(x), Nb * Nb), order="F")  # [g, a + Nb c]
    dist = np.abs(np.asarray(x)[:, None] - np.asarray(x)[donors][None, :])
    V = prefactor_scale / (q + q_s) * (pair.T @ np.exp(-q * dist))
    return V, np.asarray(donor_weights, dtype=np.float64)[donors]


def separable_sum_operator(name: str, W, V, d=None, rtol: float = 1e-15, max_terms: int = 0) -> Mechanism:
    """Kronecker-sum form K(m, m') = q sum_i radial_i(m, m') block_i of a
    kernel given by angular node weights and node tensors,

        K[m, m', a, c, d, b] = sum_t W[(m, m'), t] X_t[(a, c), (b, d)],
        X_t = V_t diag(d) V_t^H                       (pair layout),

    which covers both of the reference's momentum-dependent kernels: the
    exact LO kernel (lo_phonon_kernel, numerics/reference/kernels.jl:321-356:
    X_h = F_h (x) conj F_h, V_h = vec F_h, d = 1, W = lo_weights) and the
    tabulated kernels (_assemble_lookup_kernel, numerics/optimized/
    kernels.jl:303-320: X_t = C(q_t), W = lookup_weights; the impurity
    covariance C = V diag(w_D) V^H, impurity_pair_factors).

    W: (N_k^2, T) (row m + N_k m'); V: (T, N_b^2, D) with pair index
    a + N_b c; d: (D,) non-negative (default ones).

    The compression is exact up to the singular values it drops, which are
    all below `rtol` of the largest (in the norm of the N_k^2 x N_b^4
    unfolding of K):
      1. Q = orthonormal basis of the columns sqrt(d_j) V_t[:, j] (SVD);
         then X_t = Q Y_t Q^H with Y_t (k x k) -- no N_b^4-sized array;
      2. QR of the k^2 x T matrix of the vec(Y_t)^H: W Y = (W R^H) Q_Y^H;
      3. SVD of W R^H (N_k^2 x T) gives the terms.
    The smooth transfer-momentum dependence of these kernels makes J small
    (about 20-30 terms at rtol 1e-15 for the LO and impurity kernels of a
    32-state basis on a 64-point momentum grid) where the dense operator has
    (N_k N_b^2)^2 entries.  q is max_(m,m') sum_i |radial_i(m,m')| max|block_i|
    (an upper bound of max|K|; only the product q K enters the map).
    `max_terms` (0 = none) caps J; ValueError if the cap drops a term above
    rtol."""
    W = np.asarray(W)
    V = np.asarray(V, dtype=np.complex128)
    if V.ndim == 2:
        V = V[:, :, None]
    T, N2, D = V.shape
    n1 = W.shape[0]
    Nk, Nb = int(round(math.sqrt(n1))), int(round(math.sqrt(N2)))
    if Nk * Nk != n1 or Nb * Nb != N2 or W.shape[1] != T:
        raise ValueError("W must be (N_k^2, T) and V (T, N_b^2, D)")
    d = np.ones(D) if d is None else np.asarray(d, dtype=np.float64)
    if d.shape != (D,) or np.any(d < 0) or not np.all(np.isfinite(d)):
        raise ValueError("node weights d must be D finite non-negative numbers")
    A = (V * np.sqrt(d)[None, None, :]).transpose(1, 0, 2).reshape(N2, T * D)  # columns sqrt(d_j) V_t[:, j]
    U, sA, _ = np.linalg.svd(A, full_matrices=False)
    if not (sA.size and sA[0] > 0 and np.isfinite(sA[0])):
        raise ValueError(f"kernel {name} is zero or non-finite")
    k = int(np.count_nonzero(sA > sA[0] * 1e-17))
    Q = U[:, :k]
    Bt = np.ascontiguousarray((Q.conj().T @ A).reshape(k, T, D).transpose(1, 0, 2))  # (T, k, D): Q^H sqrt(d) V_t
    Y = Bt @ np.conj(np.transpose(Bt, (0, 2, 1)))  # Y_t = B_t B_t^H, (T, k, k)
    del Bt
    Yflat = np.transpose(Y, (0, 2, 1)).reshape(T, k * k)  # column-major vec of each Y_t
    del Y
    QY, RY = np.linalg.qr(np.conj(Yflat.T))  # Yflat = RY^H QY^H, QY orthonormal columns (k^2 x T)
    del Yflat
    P, Sig, Zh = np.linalg.svd(W @ np.conj(RY.T), full_matrices=False)  # K-unfolding = P Sig (Zh QY^H)
    if not (Sig.size and Sig[0] > 0 and np.isfinite(Sig[0])):
        raise ValueError(f"kernel {name} is zero or non-finite")
    R = int(np.count_nonzero(Sig > Sig[0] * rtol))
    if max_terms and R > max_terms:
        raise ValueError(f"{name}: {R} terms exceed max_terms={max_terms} at rtol={rtol}")
    rho = Zh[:R] @ np.conj(QY.T)  # (R, k^2): vec Y^(i)
    del QY
    radial = np.empty((Nk, Nk, R), dtype=np.complex128, order="F")
    block = np.empty((N2, N2, R), dtype=np.complex128, order="F")
    for i in range(R):
        Yi = rho[i].reshape((k, k), order="F")
        Pi = (Q @ Yi @ Q.conj().T).reshape((Nb, Nb, Nb, Nb), order="F")  # [a, c, b, d]
        blk = np.transpose(Pi, (0, 2, 1, 3)).reshape((N2, N2), order="F")  # rows a + Nb b, cols c + Nb d
        mx = float(np.max(np.abs(blk)))
        block[:, :, i] = blk / mx
        radial[:, :, i] = (P[:, i] * (Sig[i] * mx)).reshape((Nk, Nk), order="F")
    q = float(np.max(np.sum(np.abs(radial), axis=2)))
    if not (q > 0 and math.isfinite(q)):
        raise ValueError(f"kernel {name} has scale {q}: zero or non-finite")
    mech = Mechanism(name, "separable_sum", q, block=block, radial=np.asfortranarray(radial / q))
    mech.residual = float(Sig[R] / Sig[0]) if R < len(Sig) else 0.0
    return mech


def exact_node_kernel(W, V, d=None) -> np.ndarray:
    """The literal six-index K[m, m', a, c, d, b] = sum_t W[(m, m'), t]
    (V_t diag(d) V_t^H)[(a, c), (b, d)] on the host (small sizes; tests)."""
    W = np.asarray(W)
    V = np.asarray(V, dtype=np.complex128)
    if V.ndim == 2:
        V = V[:, :, None]
    T, N2, D = V.shape
    Nk, Nb = int(round(math.sqrt(W.shape[0]))), int(round(math.sqrt(N2)))
    d = np.ones(D) if d is None else np.asarray(d, dtype=np.float64)
    X = np.einsum("tpj,j,tqj->tpq", V, d, V.conj())  # [t, (a,c), (b,d)]
    K = np.tensordot(W, X, axes=(1, 0))  # [(m,m'), (a,c), (b,d)]
    K = K.reshape((Nk, Nk, Nb, Nb, Nb, Nb), order="F")  # [m, m', a, c, b, d]
    return np.asfortranarray(np.transpose(K, (0, 1, 2, 3, 5, 4)))
