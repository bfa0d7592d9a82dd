"""The reg:: C++ facade (include/claire_b200.hpp): compiled here with g++
against the library; option parsing on the host, and a registration through
the facade equal to the Python binding's on the same inputs (GPU)."""
import json
import os
import shutil
import subprocess

import numpy as np
import pytest

from oracle import claire_ref as R

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIBDIR = os.path.join(ROOT, "claire_b200")


@pytest.fixture(scope="module")
def facade(tmp_path_factory):
    if not shutil.which("g++"):
        pytest.skip("g++ not available")
    import claire_b200  # noqa: F401  (the library is built)
    exe = str(tmp_path_factory.mktemp("facade") / "facade_main")
    cmd = ["g++", "-std=c++17", "-O2", "-Wall", "-Werror", os.path.join(ROOT, "tests", "cpp", "facade_main.cpp"),
           "-I", os.path.join(ROOT, "include"), "-L", LIBDIR, "-lclaire_b200", "-Wl,-rpath," + LIBDIR, "-o", exe]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return exe


def test_facade_parses_like_regopt(facade):
    r = subprocess.run([facade, "opts", "-nx", "64", "-nt", "8", "-regnorm", "h2", "-beta", "1e-3", "-maxit", "7",
                        "-opttol", "1e-2", "-distance", "ncc"], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    o = json.loads(r.stdout)
    assert o["nx"] == [64, 64, 64] and o["nt"] == 8 and o["beta"] == 1e-3 and o["maxit"] == 7
    assert o["opttol"] == 1e-2 and o["distance"] == 1 and o["bytes"] > 0
    bad = subprocess.run([facade, "opts", "-regnorm", "nonsense"], capture_output=True, text=True)
    assert bad.returncode != 0


@pytest.mark.gpu
@pytest.mark.parametrize("precond", ["invreg", "2level"])
def test_facade_registration_equals_python_binding(facade, tmp_path, cuda, precond):
    import claire_b200 as cb
    n, nt = 32, 4
    mR, mT, _ = R.synthetic_c1(n, np.float64, nt)
    mR = mR.astype(np.float32)
    mT = mT.astype(np.float32)
    mR.tofile(tmp_path / "mR.bin")
    mT.tofile(tmp_path / "mT.bin")
    args = ["-nx", str(n), "-nt", str(nt), "-regnorm", "h1s", "-beta", "1e-2", "-maxit", "10", "-opttol", "1e-2",
            "-precond", precond]
    r = subprocess.run([facade, "run", str(tmp_path)] + args, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr
    out = json.loads(r.stdout)
    v_cpp = np.fromfile(tmp_path / "v.bin", dtype=np.float32).reshape(3, n, n, n)
    pv_cpp = np.fromfile(tmp_path / "pv.bin", dtype=np.float32).reshape(3, n, n, n)
    with cb.CLAIREInterface(cb.RegOpt(args)) as ci:
        ci.set_images(mR, mT)
        ci.Run()
        v_py = np.asarray(ci.GetSolution())
        st = ci.stats()
        pv_py = ci.ApplyInvRegularizationOperator(v_py)
    assert np.array_equal(v_cpp, v_py)
    assert np.array_equal(pv_cpp, pv_py)  # reg::Preconditioner::MatVec
    assert out["gn"] == st["gn_iterations"] and out["pcg"] == st["pcg_iterations"]
    assert 0.0 < out["det_min"] <= 1.0 <= out["det_max"]
