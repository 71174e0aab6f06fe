"""The hanging-node mesh of the C ABI (mpdg_amr_*), built on the host without a GPU, against
the oracle's two-level mesh: DoF numbering, support points, Dirichlet mask, the per-cell
gathered DoFs and hanging codes the cell kernel reads."""
import numpy as np
import pytest

from meltpooldg_b200 import _lib as L
from meltpooldg_b200 import heat as H
from meltpooldg_b200.amr import AmrHeatOperator
from oracle import amr as A

REFINE = [(1, 1, 1), (2, 1, 1), (1, 2, 1), (1, 1, 2), (0, 0, 0)]


@pytest.mark.parametrize("p", [1, 2, 3, 4])
@pytest.mark.parametrize("refine", ["none", "some", "all"])
def test_host_description_matches_oracle(p, refine):
    cells = (4, 3, 3)
    ref = {"none": [], "some": REFINE, "all": np.ones((3, 3, 4), dtype=bool)}[refine]
    mesh = H.box_mesh(p, cells, hi=(2.0, 1.5, 1.0), dirichlet=("x-", "y+", "z-", "z+"))
    op = AmrHeatOperator(mesh, ref, device=None)
    o = A.TwoLevelBoxMesh(p, cells, refine=ref, hi=(2.0, 1.5, 1.0),
                          dirichlet=("x-", "y+", "z-", "z+"))
    assert op.n_dofs == o.n_dofs and op.n_cells == o.n_cells
    assert np.abs(op.support_points() - o.support_points()).max() < 1e-14
    assert np.array_equal(op.constraint_mask().astype(bool), o.mask)
    dofs, codes = op.cell_data()
    for c in range(o.n_cells):
        idx, _ = o.cell_map(c)
        assert np.array_equal(dofs[c], idx), c
        assert int(codes[c]) & 0x1FF == o.hanging_code(c), c
        assert bool(int(codes[c]) & 0x200) == (o.sizes[c] == 0.5)


def test_invalid_meshes_rejected_without_gpu():
    import ctypes
    lib = L.load()
    h = ctypes.c_void_p()
    ref = np.zeros(8, dtype=np.uint8)
    d = H.box_mesh(5, (2, 2, 2))
    assert lib.mpdg_amr_create(ctypes.byref(d), ref.ctypes.data_as(ctypes.c_void_p), -1,
                               ctypes.byref(h)) == L.ERR_INVALID_ARGUMENT
    d = H.box_mesh(2, (2, 2, 2), perturb=0.1)
    assert lib.mpdg_amr_create(ctypes.byref(d), ref.ctypes.data_as(ctypes.c_void_p), -1,
                               ctypes.byref(h)) == L.ERR_INVALID_ARGUMENT
    op = AmrHeatOperator(H.box_mesh(2, (2, 2, 2)), [(0, 0, 0)], device=None)
    with pytest.raises(H.ExcNotImplemented):
        op.set_material(H.material(law=L.LAW_LIQUID_SOLID), 1e-3)


def test_multilevel_host_description_matches_oracle():
    """Levels 0, 1 and 2 (2:1 balanced) on the host: DoFs, support points, mask, gathered DoFs
    and codes (bits 10-12 the level) equal the oracle's multi-level mesh; a level above the
    maximum or an unbalanced mesh is refused before any CUDA call, on a device too."""
    p = 2
    lev = np.zeros((5, 5, 5), dtype=np.int64)
    lev[1:4, 1:4, 1:4] = 1
    lev[2, 2, 2] = 2
    mesh = H.box_mesh(p, (5, 5, 5), dirichlet=("x-", "x+", "z-"))
    op = AmrHeatOperator(mesh, lev, device=None)
    o = A.MultiLevelBoxMesh(p, (5, 5, 5), lev, dirichlet=("x-", "x+", "z-"))
    assert op.n_dofs == o.n_dofs and op.n_cells == o.n_cells
    assert np.abs(op.support_points() - o.support_points()).max() < 1e-14
    assert np.array_equal(op.constraint_mask().astype(bool), o.mask)
    dofs, codes = op.cell_data()
    for c in range(o.n_cells):
        idx, _ = o.cell_map(c)
        assert np.array_equal(dofs[c], idx), c
        assert int(codes[c]) & 0x1FF == o.hanging_code(c), c
        assert (int(codes[c]) >> 10) & 7 == o.cell_level[c]
    too_deep = lev.copy()
    too_deep[2, 2, 2] = 7
    with pytest.raises(H.ExcInvalidArgument):
        AmrHeatOperator(mesh, too_deep, device=0)
    bad = lev.copy()
    bad[0, 0, 0] = 2
    with pytest.raises(H.ExcInvalidArgument):
        AmrHeatOperator(mesh, bad, device=None)
