"""The C++ adapters of integration/ (DevicePrecondition, DeviceSolver): what a
PrisPack maintainer adds next to BasePrecondition / BaseSolver
(include/Preconditioner/BasePreconditon.h:34-145, include/Solver/BaseSolver.h:16).

CPU: the adapters implement every pure-virtual member the reference declares,
and they compiled against the reference's own headers into
oracle/_ref/device_cg_driver (built with the reference checker by
`make -C oracle ref integration`).  GPU: that driver runs the reference's own
HOST::CG<double> with DevicePrecondition as its preconditioner, against the
same CG with the reference's IncompleteCholesky / AMSEDPrecondition."""
from __future__ import annotations

import json
import os
import re
import subprocess

import pytest

from oracle import ref

ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), ".."))
DRIVER = os.path.join(ROOT, "oracle", "_ref", "device_cg_driver")


def test_adapter_implements_every_pure_virtual_member():
    src = open(os.path.join(ROOT, "integration", "DevicePrecondition.hpp")).read()
    overloads = re.findall(r"void MInvSolve\(([^)]*)\) override", src)
    assert sorted(len(a.split(",")) for a in overloads) == [1, 2, 2, 4]
    assert "void setup() override" in src
    solver = open(os.path.join(ROOT, "integration", "DeviceSolver.hpp")).read()
    assert re.search(r"void solve\(const HOST::CSRMatrix<T>& matA, const HostVector<T>& b, HostVector<T>& x\) "
                     r"override", solver)


@pytest.mark.skipif(not ref.available(), reason="reference checker build absent")
def test_adapters_compiled_against_the_reference_headers():
    assert os.access(DRIVER, os.X_OK), "make -C oracle integration did not produce the driver"


def _driver_json(*grid):
    r = subprocess.run([DRIVER, *map(str, grid)], capture_output=True, text=True, timeout=600)
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
    assert lines, r.stdout[-2000:] + r.stderr[-2000:]
    out = json.loads(lines[-1])
    assert r.returncode == 0 and out.get("ok") == 1, out
    return out


@pytest.mark.gpu
@pytest.mark.skipif(not os.path.exists(DRIVER), reason="adapter driver not built")
def test_reference_cg_with_device_preconditioner():
    d = _driver_json(40, 40, 40)
    ic_ref, ic_dev, ic_sol = d["ic.reference"], d["ic.device"], d["ic.solver"]
    assert ic_ref["converged"] and ic_dev["converged"] and ic_sol["converged"]
    # the device factor is the reference's bit for bit; only the sweeps' summation order differs
    assert d["ic.mnnz"][0] == d["ic.mnnz"][1]
    assert abs(ic_dev["iters"] - ic_ref["iters"]) <= 1 and abs(ic_sol["iters"] - ic_ref["iters"]) <= 1
    assert ic_dev["diff"] <= 1e-10 and ic_sol["diff"] <= 1e-10
    assert ic_dev["true_rel_residual"] <= 1.5e-10 and ic_sol["true_rel_residual"] <= 1.5e-10
    # MInvSolve(in, out), MInvSolve(vec), MInvSolve(vec, offset), MInvSolve(in, off, out, off) agree
    assert max(d["overloads_max_diff"]) == 0.0
    # new values on the same pattern: the device refactorisation against a new reference setup
    rf_ref, rf_dev = d["refactor.reference"], d["refactor.device"]
    assert rf_ref["converged"] and rf_dev["converged"] and d["refactor.mnnz"][0] == d["refactor.mnnz"][1]
    assert abs(rf_dev["iters"] - rf_ref["iters"]) <= 1 and rf_dev["diff"] <= 1e-10
    am_ref, am_dev = d["amsed.reference"], d["amsed.device"]
    assert am_ref["converged"] and am_dev["converged"]
    assert abs(am_dev["iters"] - am_ref["iters"]) <= 1
    assert am_dev["diff"] <= 1e-9
