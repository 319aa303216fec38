"""The Jacobi visit's algebra (csrc/svd.cu: jacobi_rotation, jacobi_pair_visit),
restated in numpy with the kernel's formulas and update order and checked on CPU:

  * the division-free rotation: d = b - a and g scaled by the power of two that
    brings max(|d|, 2 g) into [1, 2) (built from the exponent bits),
    r = sqrt(d^2 + 4 g^2), u = |d| + r, q = 1 / sqrt(2 r u); c = u q,
    s = 2 g q sgn(d), t g = 4 g r q^2 sgn(d) g;
  * one round of the circle method on the Gram matrix: every active pair's
    columns of G and Q rotated ([x y] <- [x y] J, J = [[c, s e^{i phi}],
    [-s e^{-i phi}, c]]), then its rows (G <- J^H G), the rotated 2 x 2 block set
    to a - t g, b + t g and 0; a pair rotates when |g|^2 > tol^2 a b.

Checked: c^2 + s^2 = 1 and the rotation zeroes the pair's Gram entry, at unit
scale and at 1e+-140 (norms to 1e+-292, where the unscaled squares of d and g
would overflow or underflow);
the exact diagonal values agree with J^H G J; inner sweeps to convergence give Q
unitary, W Q with orthogonal columns whose norms are the singular values of W.
"""
import numpy as np
import pytest


def _pow2_scale_of(m):
    e = (np.float64(m).view(np.uint64) >> np.uint64(52)) & np.uint64(0x7FF)
    return np.ldexp(1.0, 1023 - int(e))


def _rotation(a, b, g):
    d = b - a
    sc = _pow2_scale_of(max(abs(d), 2.0 * g))
    dn, gn = d * sc, g * sc
    x = dn * dn + 4.0 * gn * gn
    r = x / np.sqrt(x)
    u = abs(dn) + r
    q = 1.0 / np.sqrt(2.0 * r * u)
    sg = 1.0 if d >= 0.0 else -1.0
    return u * q, sg * (2.0 * gn * q), sg * (4.0 * gn * r * q * q) * g


def _pairs(N, rnd):
    out = []
    for w in range(N // 2):
        if w == 0:
            p, q = N - 1, rnd
        else:
            p = (rnd + w) % (N - 1)
            q = (rnd - w) % (N - 1)
        out.append((min(p, q), max(p, q)))
    return out


def _inner_sweep(G, Q, tol):
    """One cyclic sweep of the visit: rounds of disjoint pairs, all columns first,
    then all rows, then the exact 2 x 2 values.  Returns the number of rotations."""
    nc = G.shape[0]
    N = nc + (nc & 1)
    nrot = 0
    for rnd in range(N - 1):
        act = []
        for p, q in _pairs(N, rnd):
            if q >= nc:
                continue
            a, b, gpq = G[p, p].real, G[q, q].real, G[p, q]
            g2 = abs(gpq) ** 2
            if a * b > 0.0 and g2 > tol * tol * a * b:
                g = np.sqrt(g2)
                e = gpq / g
                c, s, tg = _rotation(a, b, g)
                act.append((p, q, c, s, e, a, b, tg))
        for p, q, c, s, e, *_ in act:
            for M in (G, Q):
                x, y = M[:, p].copy(), M[:, q].copy()
                M[:, p] = c * x - s * np.conj(e) * y
                M[:, q] = s * e * x + c * y
        for p, q, c, s, e, a, b, tg in act:
            x, y = G[p, :].copy(), G[q, :].copy()
            G[p, :] = c * x - s * e * y
            G[q, :] = s * np.conj(e) * x + c * y
            G[p, p], G[q, q], G[p, q], G[q, p] = a - tg, b + tg, 0.0, 0.0
        nrot += len(act)
    return nrot


@pytest.mark.parametrize("scale", [1.0, 1e-140, 1e140])
@pytest.mark.parametrize("cplx", [False, True])
def test_rotation_zeroes_the_pair(scale, cplx):
    rng = np.random.default_rng(7)
    for _ in range(200):
        w = rng.standard_normal((20, 2)) * scale
        if cplx:
            w = w + 1j * rng.standard_normal((20, 2)) * scale
        w[:, 1] *= 10.0 ** rng.uniform(-6, 6)
        a, b = np.vdot(w[:, 0], w[:, 0]).real, np.vdot(w[:, 1], w[:, 1]).real
        gpq = np.vdot(w[:, 0], w[:, 1])
        g = abs(gpq)
        e = gpq / g
        c, s, tg = _rotation(a, b, g)
        assert abs(c * c + s * s - 1.0) <= 1e-15
        w2 = np.stack([c * w[:, 0] - s * np.conj(e) * w[:, 1], s * e * w[:, 0] + c * w[:, 1]], 1)
        n0, n1 = np.linalg.norm(w2, axis=0)
        assert abs(np.vdot(w2[:, 0], w2[:, 1])) <= 1e-14 * n0 * n1 * 20
        # the exact values the kernel stores for the rotated diagonal
        assert abs((a - tg) - n0 * n0) <= 1e-13 * max(a, b)
        assert abs((b + tg) - n1 * n1) <= 1e-13 * max(a, b)


@pytest.mark.parametrize("cplx", [False, True])
@pytest.mark.parametrize("m,nc", [(40, 16), (40, 32), (12, 16), (100, 15), (3, 2), (50, 1)])
def test_gram_sweeps_diagonalise(cplx, m, nc):
    rng = np.random.default_rng(m * 31 + nc)
    W = rng.standard_normal((m, nc)) * 10.0 ** rng.uniform(-4, 4, nc)
    if cplx:
        W = W + 1j * rng.standard_normal((m, nc))
    G = W.conj().T @ W
    G = (np.triu(G) + np.triu(G, 1).conj().T)   # exactly Hermitian, as the kernel mirrors it
    Q = np.eye(nc, dtype=G.dtype)
    tol = np.sqrt(m) * np.finfo(float).eps
    for _ in range(30):
        if _inner_sweep(G, Q, tol) == 0:
            break
    else:
        raise AssertionError("no convergence")
    np.testing.assert_allclose(Q.conj().T @ Q, np.eye(nc), rtol=0, atol=1e-13 * nc)
    WQ = W @ Q
    n = np.linalg.norm(WQ, axis=0)
    off = WQ.conj().T @ WQ - np.diag(n * n)
    # relative orthogonality; the Gram form keeps the null columns of a
    # rank-deficient W (m < nc) only to an absolute 8 eps m nc |W|^2 (their entries
    # take the rounding of every rotation that touches them)
    floor = 8 * np.finfo(float).eps * m * nc * n.max() ** 2
    assert np.all(np.abs(off) <= 1e-12 * np.outer(n, n) * m + floor)
    ref = np.linalg.svd(W, compute_uv=False)
    np.testing.assert_allclose(np.sort(n)[::-1][:len(ref)], ref, rtol=1e-11, atol=np.sqrt(floor))
    # the tracked Gram diagonal: squared norms to the same absolute floor
    np.testing.assert_allclose(np.diag(G).real, n * n, rtol=1e-10, atol=floor)
