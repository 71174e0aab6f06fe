"""Why the FP32 preconditioner keeps the QGauss(p+1) operator: two cheaper fine-level operators
are too far from it spectrally.

For FE_Q(3) on a box (Dirichlet faces, M/dt + K with dt = 5e-4 and k = 1, the benchmark's
scales), the generalized eigenvalues of the assembled operators are computed densely on 4^3
cells (1331 interior DoFs):
  - GLL collocation (quadrature at the Gauss-Lobatto support points, a diagonal mass, 6 instead
    of 12 sum-factorisation sweeps): eig(A_gll^-1 A) in [0.18, 1.0], a condition number ~5.6;
  - low-order refined (Q1 on the sub-mesh through the GLL nodes, a 27-point stencil on the same
    DoFs): eig(A_lor^-1 A) in [0.42, 5.6] (consistent Q1 mass) or [0.10, 1.5] (lumped).
A multigrid V-cycle built on either would precondition the exact operator with that much worse
a bound than one built on the QGauss operator itself, which reaches 4-6 outer iterations per
benchmark step; either kernel would have to run several times faster to pay for the extra outer
iterations. Pure numpy (no oracle, no GPU)."""
import numpy as np
import pytest
from numpy.polynomial.legendre import Legendre, leggauss

scipy_linalg = pytest.importorskip("scipy.linalg")


def gll(n):
    P = Legendre.basis(n - 1)
    x = np.concatenate([[-1.0], np.sort(P.deriv().roots()), [1.0]])
    w = 2.0 / (n * (n - 1) * P(x) ** 2)
    return (x + 1) / 2, w / 2


def lagrange(nodes, x):
    n = len(nodes)
    V, D = np.zeros((len(x), n)), np.zeros((len(x), n))
    for i in range(n):
        others = [j for j in range(n) if j != i]
        den = np.prod([nodes[i] - nodes[j] for j in others])
        for q, xq in enumerate(x):
            V[q, i] = np.prod([xq - nodes[j] for j in others]) / den
            D[q, i] = sum(np.prod([xq - nodes[j] for j in others if j != m]) for m in others) / den
    return V, D


def tensor_operator(M1s, K1s, dt, k):
    M = np.kron(M1s[2], np.kron(M1s[1], M1s[0]))
    K = (np.kron(M1s[2], np.kron(M1s[1], K1s[0])) + np.kron(M1s[2], np.kron(K1s[1], M1s[0])) +
         np.kron(K1s[2], np.kron(M1s[1], M1s[0])))
    return M / dt + k * K


def assemble(p, m, dt, k, rule):
    n, N1, h = p + 1, p * m + 1, 1.0 / m
    nodes, _ = gll(n)
    if rule == "gauss":
        xg, wg = leggauss(n)
        xq, wq = (xg + 1) / 2, wg / 2
    else:
        xq, wq = gll(n)
    V, D = lagrange(nodes, xq)
    M1, K1 = V.T @ np.diag(wq) @ V * h, D.T @ np.diag(wq) @ D / h
    Ae = tensor_operator([M1] * 3, [K1] * 3, dt, k)
    A = np.zeros((N1 ** 3, N1 ** 3))
    for cz in range(m):
        for cy in range(m):
            for cx in range(m):
                idx = [(p * cx + i) + N1 * ((p * cy + j) + N1 * (p * cz + kk))
                       for kk in range(n) for j in range(n) for i in range(n)]
                A[np.ix_(idx, idx)] += Ae
    return interior(A, N1)


def assemble_lor(p, m, dt, k, lumped):
    n, N1, h = p + 1, p * m + 1, 1.0 / m
    nodes, _ = gll(n)
    coords = np.concatenate([c * h + nodes[:-1] * h for c in range(m)] + [[1.0]])
    xg, wg = leggauss(2)
    V, D = lagrange(np.array([0.0, 1.0]), (xg + 1) / 2)
    wq = wg / 2
    A = np.zeros((N1 ** 3, N1 ** 3))
    for iz in range(N1 - 1):
        for iy in range(N1 - 1):
            for ix in range(N1 - 1):
                hs = [coords[i + 1] - coords[i] for i in (ix, iy, iz)]
                Ms = [V.T @ np.diag(wq) @ V * s for s in hs]
                if lumped:
                    Ms = [np.diag(M.sum(1)) for M in Ms]
                Ks = [D.T @ np.diag(wq) @ D / s for s in hs]
                idx = [(ix + i) + N1 * ((iy + j) + N1 * (iz + kk))
                       for kk in range(2) for j in range(2) for i in range(2)]
                A[np.ix_(idx, idx)] += tensor_operator(Ms, Ks, dt, k)
    return interior(A, N1)


def interior(A, N1):
    keep = [i for i in range(N1 ** 3)
            if all(0 < c < N1 - 1 for c in (i % N1, (i // N1) % N1, i // N1 ** 2))]
    return A[np.ix_(keep, keep)]


def spectrum(A, B):
    ev = scipy_linalg.eigh(A, B, eigvals_only=True)
    return ev.min(), ev.max()


def test_gll_collocated_and_low_order_refined_operators_are_poor_substitutes():
    p, m, dt = 3, 4, 5e-4
    A = assemble(p, m, dt, 1.0, "gauss")
    lo, hi = spectrum(A, assemble(p, m, dt, 1.0, "gll"))
    assert 0.15 < lo < 0.2 and abs(hi - 1.0) < 1e-6  # [0.177, 1.000]
    assert hi / lo > 5.0
    for lumped in (False, True):
        lo, hi = spectrum(A, assemble_lor(p, m, dt, 1.0, lumped))
        assert hi / lo > 10.0  # [0.416, 5.563] consistent, [0.102, 1.527] lumped
    # sanity: the QGauss operator against itself
    lo, hi = spectrum(A, A)
    assert abs(lo - 1.0) < 1e-9 and abs(hi - 1.0) < 1e-9
