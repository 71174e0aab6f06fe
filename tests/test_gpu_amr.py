"""The hanging-node cell kernel (mpdg_amr_vmult) against the oracle's two-level operator, and
against the structured GPU operator where no cell is refined."""
import numpy as np
import pytest
import torch

from meltpooldg_b200 import _lib as L
from meltpooldg_b200 import heat as H
from meltpooldg_b200.amr import AmrHeatOperator
from oracle import amr as A

pytestmark = pytest.mark.gpu

# cells with one, two and three hanging faces, a face and an edge, and hanging edges only
REFINE = [(1, 1, 1), (2, 1, 1), (1, 2, 1), (1, 1, 2), (0, 0, 0)]
BOX = dict(hi=(2.0, 1.5, 1.0), dirichlet=("x-", "y+", "z-", "z+"))


@pytest.mark.parametrize("p", [1, 2, 3, 4])
@pytest.mark.parametrize("law", ["constant", "linear_k"])
def test_vmult_with_hanging_nodes_matches_oracle(p, law):
    cells = (4, 3, 3)
    op = AmrHeatOperator(H.box_mesh(p, cells, **BOX), REFINE, device=0)
    o = A.TwoLevelBoxMesh(p, cells, refine=REFINE, **BOX)
    assert op.n_dofs == o.n_dofs and o.hanging.any()
    rng = np.random.default_rng(30 + p)
    src = rng.uniform(-1.0, 1.0, o.n_dofs)
    dt = 1e-2
    if law == "constant":
        op.set_material(H.material(rho=2.0, cp=1.5, k=0.7), dt)
        ref = o.vmult(src, rho_cp=3.0, dt=dt, k0=0.7)
        T = None
    else:
        op.set_material(H.material(law=L.LAW_LINEAR_K, k=1.0, k1=0.5), dt)
        Tn = rng.uniform(0.0, 1.0, o.n_dofs)
        ref = o.vmult(src, rho_cp=1.0, dt=dt, k0=1.0, k1=0.5, T_lin=Tn)
        T = torch.tensor(Tn, device="cuda")
    dst = torch.empty(o.n_dofs, dtype=torch.float64, device="cuda")
    op.vmult(dst, torch.tensor(src, device="cuda"), T)
    got = dst.cpu().numpy()
    assert np.abs(got - ref).max() <= 1e-12 * np.abs(ref).max()


def test_unrefined_mesh_matches_structured_operator():
    p, cells = 3, (5, 4, 3)
    mesh = H.box_mesh(p, cells, **BOX)
    amr = AmrHeatOperator(mesh, (), device=0)
    st = H.HeatDiffuseOperator(mesh)
    assert amr.n_dofs == st.n_dofs
    dt = 5e-3
    m = H.material(law=L.LAW_LINEAR_K, k=1.0, k1=0.5)
    amr.set_material(m, dt)
    st.set_material(m)
    st.reset_time_increment(dt)
    g = torch.Generator(device="cuda").manual_seed(4)
    T = torch.rand(st.n_dofs, dtype=torch.float64, device="cuda", generator=g)
    src = torch.rand(st.n_dofs, dtype=torch.float64, device="cuda", generator=g)
    st.set_linearization(T, T)
    a = torch.empty_like(src)
    b = torch.empty_like(src)
    amr.vmult(a, src, T)
    st.vmult(b, src)
    assert (a - b).abs().max().item() <= 1e-12 * b.abs().max().item()
