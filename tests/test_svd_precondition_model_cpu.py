"""The algebra of the block SVD's QR preconditioning (csrc/svd.cu), restated in
numpy with the same formulas and checked against numpy's SVD:

  * columns of W0 = op(A) (A, or A^H when m < n) ordered by decreasing norm (P);
  * blocked Householder QR, panels of NB columns: larfg reflections (beta =
    -sign(Re alpha) |x|, tau = (beta - alpha) / beta, v = x / (alpha - beta), none
    when the column below the diagonal is zero and alpha is real), T of the
    compact WY form (forward, columnwise), trailing tiles updated by
    I - Y T^H Y^H;
  * the same QR of R^H, the Jacobi's input R1^H (its SVD taken here from numpy);
  * the outputs W = Q [R1^H V2; 0] (the left factor times S) and V = P Q1 V2.

Checked: op(A) V = W, V unitary, the columns of W orthogonal with norms the
singular values of A, on real and complex, tall and wide, rank-deficient and
all-zero blocks, with the real (16) and complex (8) panel widths.
"""
import numpy as np
import pytest


def _qr_blocked(W0, NB):
    A = W0.copy()
    R, C = A.shape
    panels = []
    for k in range((C + NB - 1) // NB):
        r0, w = k * NB, min(NB, C - k * NB)
        P = A[r0:, r0:r0 + w].copy()
        taus = []
        for j in range(w):
            x = P[j:, j]
            alpha, s2 = x[0], float(np.sum(np.abs(x[1:]) ** 2))
            tau = 0.0
            if s2 > 0 or np.imag(alpha) != 0:
                beta = -np.copysign(np.sqrt(abs(alpha) ** 2 + s2), np.real(alpha))
                tau = (beta - np.real(alpha)) / beta - 1j * np.imag(alpha) / beta if np.iscomplexobj(A) \
                    else (beta - alpha) / beta
                x[1:] = x[1:] / (alpha - beta)
                x[0] = beta
            taus.append(tau)
            v = np.concatenate([[1.0], x[1:]])
            for l in range(j + 1, w):   # H_j^H on the panel's later columns
                P[j:, l] -= v * (np.conj(tau) * np.vdot(v, P[j:, l]))
        V = np.tril(P, -1)
        V[np.arange(w), np.arange(w)] = 1.0
        T = np.zeros((w, w), dtype=A.dtype)
        for j in range(w):
            T[j, j] = taus[j]
            if j:
                T[:j, j] = -taus[j] * (T[:j, :j] @ (V[:, :j].conj().T @ V[:, j]))
        A[r0:, r0:r0 + w] = P
        X = A[r0:, r0 + w:]
        A[r0:, r0 + w:] = X - V @ (T.conj().T @ (V.conj().T @ X))
        panels.append((V, T, r0))
    return A, panels


def _apply_q(panels, X):
    X = X.copy()
    for V, T, r0 in reversed(panels):
        X[r0:] = X[r0:] - V @ (T @ (V.conj().T @ X[r0:]))
    return X


def _preconditioned_svd(A, NB):
    m, n = A.shape
    opA = A.conj().T if m < n else A
    R_, C_ = opA.shape
    perm = np.argsort(-np.sum(np.abs(opA) ** 2, 0), kind="stable")
    Aq, Ts = _qr_blocked(opA[:, perm], NB)
    Aq2, Ts2 = _qr_blocked(np.triu(Aq[:C_]).conj().T.copy(), NB)
    Wj = np.triu(Aq2[:C_]).conj().T                 # R1^H, the Jacobi's input
    _, _, v2h = np.linalg.svd(Wj)
    V2 = v2h.conj().T
    W = _apply_q(Ts, np.concatenate([Wj @ V2, np.zeros((R_ - C_, C_), dtype=Wj.dtype)], 0))
    Vq = _apply_q(Ts2, V2)
    Vout = np.zeros_like(Vq)
    Vout[perm] = Vq
    return opA, W, Vout


@pytest.mark.parametrize("cplx", [False, True])
@pytest.mark.parametrize("m,n,rank", [(70, 50, 50), (40, 90, 40), (33, 33, 20), (20, 12, 5), (12, 20, 3), (6, 6, 0),
                                      (2, 2, 1), (1, 5, 1)])
def test_preconditioning_algebra(cplx, m, n, rank):
    rng = np.random.default_rng(m * 100 + n + rank)
    NB = 8 if cplx else 16

    def rnd(*s):
        return rng.standard_normal(s) + (1j * rng.standard_normal(s) if cplx else 0)

    A = rnd(m, rank) @ rnd(rank, n) if rank else np.zeros((m, n), dtype=complex if cplx else float)
    opA, W, V = _preconditioned_svd(A, NB)
    scale = max(1.0, np.abs(A).max())
    np.testing.assert_allclose(opA @ V, W, rtol=0, atol=1e-13 * scale * max(m, n))
    np.testing.assert_allclose(V.conj().T @ V, np.eye(V.shape[0]), rtol=0, atol=1e-13 * max(m, n))
    G = W.conj().T @ W
    off = G - np.diag(np.diag(G))
    assert np.abs(off).max() <= 1e-12 * scale ** 2 * max(m, n)
    s = np.sort(np.sqrt(np.abs(np.diag(G))))[::-1]
    ref = np.linalg.svd(A, compute_uv=False)
    np.testing.assert_allclose(s[:len(ref)], ref, rtol=0, atol=1e-12 * scale * max(m, n))
