"""The reference-side adapter (include/mpdg_heat_dealii.hpp) compiles against MeltPoolDG's own
include/meltpooldg/core/operator_base.hpp, core/exceptions.hpp and
linear_algebra/preconditioner_jacobi.hpp (deal.II replaced by the declaration-only stand-ins of
tests/dealii_stub, since deal.II is not installed), derives from OperatorMatrixFree<3, double>
with the base's host VectorType, satisfies the reference's JacobiPreconditionerOperatorType
concept, and links against the library with every symbol resolved. Needs the MeltPoolDG source
tree (skipped without it); no GPU."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REFERENCE_INCLUDE = "/root/reference/include"
LIB = os.path.join(ROOT, "meltpooldg_b200", "libmpdg_heat.so")


@pytest.mark.skipif(not os.path.exists(os.path.join(REFERENCE_INCLUDE, "meltpooldg", "core",
                                                    "operator_base.hpp")),
                    reason="MeltPoolDG source tree not present")
@pytest.mark.skipif(shutil.which("g++") is None, reason="no C++ compiler")
def test_adapter_compiles_against_reference_headers_and_links(tmp_path):
    obj = tmp_path / "adapter_check.o"
    cmd = ["g++", "-std=c++20", "-fPIC", "-c", "-Wall", "-Wextra", "-Werror",
           "-I", os.path.join(ROOT, "tests", "dealii_stub"), "-I", REFERENCE_INCLUDE,
           "-I", os.path.join(ROOT, "include"),
           os.path.join(ROOT, "tests", "dealii_stub", "adapter_check.cpp"), "-o", str(obj)]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-4000:]
    if not os.path.exists(LIB):
        pytest.skip("library not built")
    so = tmp_path / "adapter_check.so"
    r = subprocess.run(["g++", "-shared", "-o", str(so), str(obj), "-Wl,--no-undefined",
                        "-L", os.path.dirname(LIB), "-l:libmpdg_heat.so"],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-4000:]
