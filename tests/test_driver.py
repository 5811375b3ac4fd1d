"""The standalone C++ driver (dogpup_b200/driver/dgp_forward.cpp).

CPU: it builds, prints its usage, and rejects malformed case files before
touching the GPU.  GPU: on a case written from a DMesh it reproduces the
Python API's detector data (FP64 to 1e-12: 1e-10 relative; mixed: 1e-6).
"""
import json
import subprocess

import numpy as np
import pytest

from dogpup_b200 import build


@pytest.fixture(scope="module")
def driver():
    return str(build.build_driver())


def test_driver_usage_and_bad_case(driver, tmp_path):
    r = subprocess.run([driver], capture_output=True, text=True)
    assert r.returncode == 2 and "usage" in r.stderr
    bad = tmp_path / "bad.dgp"
    bad.write_bytes(b"NOTACASE" + bytes(64))
    r = subprocess.run([driver, str(bad), str(tmp_path / "o.bin")], capture_output=True, text=True)
    assert r.returncode == 1 and "not a DGPCASE1 file" in r.stderr
    short = tmp_path / "short.dgp"
    short.write_bytes(b"DGPCASE1" + np.array([10, 5, 1, 1, 1, 2], dtype="<i8").tobytes() + bytes(16) + bytes(8))
    r = subprocess.run([driver, str(short), str(tmp_path / "o.bin")], capture_output=True, text=True)
    assert r.returncode == 1 and "truncated" in r.stderr


@pytest.mark.gpu
@pytest.mark.parametrize("precision,tol,bound", [("fp64", 1e-12, 1e-10), ("mixed", 1e-10, 1e-6)])
def test_driver_matches_python_api(driver, tmp_path, precision, tol, bound):
    from dogpup_b200 import caseio, workloads
    w = workloads.small_fwd(ns=4, nd=5, nf=8)
    mesh = workloads.build_dmesh(w)
    _, data = mesh.flu_solve(precision="fp64", tol=1e-12)
    case = tmp_path / "case.dgp"
    out = tmp_path / "data.bin"
    caseio.write_case(case, caseio.case_arrays(mesh))
    r = subprocess.run([driver, str(case), str(out), "--precision", precision, "--tol", str(tol), "--repeat", "2"],
                       capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    info = json.loads(r.stdout.strip().splitlines()[-1])
    assert info["nodes"] == mesh.nn and info["max_rel_residual"] < tol and info["step_ms"] > 0
    d = caseio.read_data(out)
    d0 = data.cpu().numpy()
    assert np.abs(d - d0).max() <= bound * np.abs(d0).max()
