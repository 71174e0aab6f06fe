"""The allocation-free L2 norm (mpdg_heat_l2_norm_noalloc) through the C ABI.

Callers that cannot allocate device memory (code inside a foreign memory pool whose
accounting a raw allocation would break) use this entry point; it must agree with the ordinary mpdg_heat_l2_norm and
must not change the device's free memory. Two calls in a row check that the shared
static scratch is reset between calls. Collected last on purpose.
"""
import ctypes as C

import pytest
import torch

from meltpooldg_b200 import _lib as L
from meltpooldg_b200 import heat as H

pytestmark = pytest.mark.gpu


def test_l2_norm_noalloc_matches_existing_entry_point():
    lib = L.load()
    # deformed mesh: per-q geometry, and the library's own kernels have run once
    op = H.HeatDiffuseOperator(H.box_mesh(3, (12, 10, 8), perturb=0.2, seed=4))
    g = torch.Generator(device="cuda").manual_seed(7)
    vecs = [torch.rand(op.n_dofs, dtype=torch.float64, device="cuda", generator=g)
            for _ in range(2)]
    vecs[1] *= 1e3  # a different scale on the second call
    refs = [op.l2_norm(u) for u in vecs]
    out = torch.zeros(1, dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    free_before = torch.cuda.mem_get_info()[0]
    got = []
    for u in vecs:
        H.check(lib.mpdg_heat_l2_norm_noalloc(op.h, C.c_void_p(u.data_ptr()),
                                              C.c_void_p(out.data_ptr())))
        torch.cuda.synchronize()
        got.append(out.item())
    free_after = torch.cuda.mem_get_info()[0]
    for a, b in zip(got, refs):
        assert abs(a - b) <= 1e-13 * b, (a, b)
    assert free_after == free_before


def test_l2_norm_noalloc_rejects_null_arguments():
    lib = L.load()
    op = H.HeatDiffuseOperator(H.box_mesh(1, (2, 2, 2)))
    out = torch.zeros(1, dtype=torch.float64, device="cuda")
    assert lib.mpdg_heat_l2_norm_noalloc(op.h, None, C.c_void_p(out.data_ptr())) == \
        L.ERR_INVALID_ARGUMENT
