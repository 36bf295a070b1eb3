"""Seeded synthetic inputs shared by the parity tests."""
import numpy as np


def approx_err(x, y):
    """Relative error in Julia's isapprox sense: norm(x-y)/max(norm(x), norm(y))."""
    x = np.asarray(x, dtype=np.complex128).ravel()
    y = np.asarray(y, dtype=np.complex128).ravel()
    den = max(np.linalg.norm(x), np.linalg.norm(y))
    return 0.0 if den == 0 else float(np.linalg.norm(x - y) / den)


def psd_blocks(rng, NE, Nk, N, scale):
    X = rng.standard_normal((NE, Nk, N, N)) + 1j * rng.standard_normal((NE, Nk, N, N))
    P = np.einsum("emab,emcb->emac", X, np.conj(X)) * (scale / N)
    return P


def dyson_inputs(seed, NE, Nk, N, broad=0.05):
    """h Hermitian per k; SigmaR = -i PSD + small Hermitian; SigmaL = i PSD;
    SigmaG = SigmaL + SigmaR - SigmaR^H (Keldysh-consistent)."""
    rng = np.random.default_rng(seed)
    h0 = np.diag(rng.uniform(0.0, 2.5, N)).astype(complex)
    c = 0.02 * (rng.standard_normal((N, N)) + 1j * rng.standard_normal((N, N)))
    h0 += np.triu(c, 1) + np.triu(c, 1).conj().T
    kin = np.linspace(0, 0.6, Nk)
    h = np.zeros((Nk, N, N), dtype=complex, order="F")
    for m in range(Nk):
        h[m] = h0 + kin[m] * np.eye(N)
    eps = np.linspace(-0.5, 3.0, NE)
    herm = 0.01 * (rng.standard_normal((NE, Nk, N, N)) + 1j * rng.standard_normal((NE, Nk, N, N)))
    herm = herm + np.conj(np.transpose(herm, (0, 1, 3, 2)))
    SR = -1j * psd_blocks(rng, NE, Nk, N, broad) + herm
    SL = 1j * psd_blocks(rng, NE, Nk, N, 0.5 * broad)
    SG = SL + SR - np.conj(np.transpose(SR, (0, 1, 3, 2)))
    f = lambda a: np.asfortranarray(a)
    return eps, h, f(SR), f(SL), f(SG)
