"""The matrices of the tensor-core Picard operator (host side, no GPU): the two shared-memory
layouts hold the same TF32-rounded entries, and G^T diag(f) G with them reproduces the oracle's
Picard cell operator (FE_Q(3), one cell, no constraints) to TF32 accuracy."""
import ctypes

import numpy as np

from meltpooldg_b200 import _lib
from oracle import oracle as O


def dense_matrices():
    lib = _lib.load()
    buf = np.zeros(2 * 16384, np.float32)
    assert lib.mpdg_picard_tc_matrices(buf.ctypes.data_as(ctypes.c_void_p)) == _lib.OK
    j, i = np.meshgrid(np.arange(256), np.arange(64), indexing="ij")
    gt = buf[(j // 8) * 512 + (i // 4) * 32 + (j % 8) * 4 + i % 4]       # G^T layout, (j, i)
    g = buf[16384 + (i // 8) * 2048 + (j // 4) * 32 + (i % 8) * 4 + j % 4]  # G layout, (j, i)
    return gt.astype(np.float64), g.astype(np.float64)


def test_both_layouts_hold_the_same_tf32_matrix():
    gt, g = dense_matrices()
    assert np.array_equal(gt, g)
    bits = gt.astype(np.float32).view(np.uint32)
    assert np.all(bits & 0x1FFF == 0)  # 10 mantissa bits
    # values rows (c = 3) interpolate: each row sums to 1; gradient rows of a constant vanish
    assert np.allclose(gt[192:].sum(axis=1), 1.0, atol=2e-3)
    assert np.abs(gt[:192].sum(axis=1)).max() < 2e-3 * np.abs(gt[:192]).max()


def test_cell_operator_matches_oracle_picard_form():
    gt, _ = dense_matrices()
    hi = (0.7, 0.4, 1.1)
    dt, k_l, k1, T0 = 5e-4, 1.0, 0.5, 0.8
    o = O.Oracle(3, (1, 1, 1), hi=hi, dirichlet_mask=0)
    o.set_material(O.material(O.LAW_LINEAR_K, k=k_l, k1=k1), dt)
    rng = np.random.default_rng(3)
    src = rng.uniform(-1, 1, o.n_dofs)
    Tl = np.full(o.n_dofs, T0)
    ref = o.vmult(src, Tl, Tl, form=2)  # lexicographic = the cell's DoF order on one cell
    w = np.polynomial.legendre.leggauss(4)[1] / 2
    wq = np.array([w[q & 3] * w[(q >> 2) & 3] * w[q >> 4] for q in range(64)])
    h = np.array(hi)
    det = h.prod()
    k = k_l + k1 * T0
    f = np.concatenate([k * wq * det / h[0] ** 2, k * wq * det / h[1] ** 2,
                        k * wq * det / h[2] ** 2, wq * det / dt])
    v = gt.T @ (f * (gt @ src))
    assert np.abs(v - ref).max() <= 2e-3 * np.abs(ref).max()
