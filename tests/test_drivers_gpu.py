"""The benchmark drivers and the reference-named runtime API on the GPU.

clspmv_run_method_f32 (behind the C++ spmv_<fmt> drivers) must run every
variant the reference sweeps, and each variant's one-SpMV check against
the host COO product must be within the FP32 bound; the Cocktail compat
calls (init_mat_kernels, do_spmv, cpy_*, evaluate) must reproduce the
reference's A^k x example (src/eval.cpp:19-72) from a C++ caller.
"""
import os
import subprocess
import sys

import numpy as np
import pytest

from clspmv_mic_b200 import _abi, drivers, tables
from clspmv_mic_b200 import formats as F
from oracle import oracle as O

from conftest import ROOT
from matrices import coo_of, cases
from test_compat_host import write_mtx

pytestmark = pytest.mark.gpu

METHODS = {
    "laplace33": ["csr_scalar", "csr_vector", "csr_merge", "coo", "dia", "bdia", "ell", "sell", "bell", "sbell", "bcsr"],
    "powerlaw3k": ["csr_scalar", "csr_vector", "csr_merge", "coo", "ell", "sell", "bell", "sbell", "bcsr"],
    "blocks300": ["bell", "sbell", "bcsr", "csr_merge", "coo"],
    "random_empty_rows": ["csr_vector", "coo", "sell", "sbell"],
}
N_VARIANTS = {"csr_scalar": 2, "csr_vector": 5, "csr_merge": 1, "coo": 1, "dia": 1, "bdia": 1, "ell": 1, "sell": 2,
              "bell": 8, "sbell": 8, "bcsr": 8}


def _scale(coo, x):
    csr = F.coo2csr(coo)
    _, sc = O.csr_f64(csr, x)
    return float(sc.max()) if sc.size else 1.0


@pytest.mark.parametrize("name,method", [(n, m) for n, ms in METHODS.items() for m in ms])
def test_run_method(name, method):
    coo = coo_of(name)
    r = drivers.run_method(coo, method, ntimes=5)
    assert len(r["variants"]) == N_VARIANTS[method]
    assert r["best"] >= 0 and r["best_gflops"] > 0
    w = coo.shape[1]
    x = (np.arange(w) % 1024).astype(np.float32) if method == "sbell" else np.ones(w, np.float32)
    bound = 1e-5 * _scale(coo, x) + 1e-6
    ran = 0
    for v in r["variants"]:
        if v["status"] != "ok":
            assert v["status"] in (_abi.STATUS[_abi.ERR_REFUSED], _abi.STATUS[_abi.ERR_UNSUPPORTED]), v
            continue
        ran += 1
        assert v["max_diff"] <= bound, (v, bound)
        assert v["ms"] > 0
    assert ran >= 1


def test_run_method_rejects_unsorted():
    coo = F.coo_matrix(4, 4, [2, 0], [1, 3], [1.0, 2.0])
    with pytest.raises(_abi.ClspmvError) as e:
        drivers.run_method(coo, "coo", 1)
    assert e.value.status == _abi.ERR_NOT_SORTED


def test_dia_refused_like_reference():
    # a scattered matrix fails coo2dia's padding rule: the driver reports the refusal
    r = drivers.run_method(coo_of("random_sparse"), "dia", 2)
    assert r["best"] == -1 and r["status"] == _abi.STATUS[_abi.ERR_REFUSED]


def test_bandwidth_test():
    b = drivers.bandwidth_test(64 << 20, 5)
    assert b["copy_gbs"] > 100 and 0 < b["launch_us"] < 1000


def test_cocktail_evaluate():
    from clspmv_mic_b200.cocktail import analyze
    coo = coo_of("blocks300")
    h, w = coo.shape
    vec = np.ones(w, np.float32)
    res = np.zeros(h, np.float32)
    coores = O.spmv_port(coo, vec)
    mat = analyze(coo, tables.ensure_default_tables())
    r = drivers.evaluate(mat, vec, res, coores, ntimes=20)
    assert r["ms"] > 0 and r["gflops"] > 0
    assert r["max_diff"] <= 1e-5 * _scale(coo, vec) + 1e-6


def test_cli_all(tmp_path):
    h, w, r, c, v = cases()["laplace33"]
    p = tmp_path / "lap.mtx"
    write_mtx(p, h, w, r, c, v)
    out = subprocess.run([sys.executable, "-m", "clspmv_mic_b200", "all", str(p), "7", "3"], capture_output=True,
                         text=True, cwd=ROOT, timeout=300)
    assert out.returncode == 0, out.stderr
    assert "Final BELL best time" in out.stdout and "Correctness Check" in out.stdout


@pytest.mark.parametrize("name", ["laplace33", "blocks300", "banded7"])
def test_cpp_cocktail_example(tmp_path, name):
    import shutil
    if shutil.which("g++") is None:
        pytest.skip("g++ not available")
    exe = tmp_path / "cocktail_example"
    libdir = _abi.LIB_PATH.parent
    cmd = ["g++", "-O2", "-std=c++17", "-I", str(ROOT / "include"), str(ROOT / "tests" / "compat" / "cocktail_example.cpp"),
           "-L", str(libdir), "-lclspmv_b200", f"-Wl,-rpath,{libdir}", "-o", str(exe)]
    res = subprocess.run(cmd, capture_output=True, text=True)
    assert res.returncode == 0, res.stderr
    h, w, r, c, v = cases()[name]
    p = tmp_path / f"{name}.mtx"
    write_mtx(p, h, w, r, c, v)
    env = dict(os.environ, CLSPMVPATH=str(tables.ensure_default_tables()))
    run = subprocess.run([str(exe), str(p), "4"], capture_output=True, text=True, env=env, timeout=300)
    assert run.returncode == 0, run.stdout[-3000:] + run.stderr[-2000:]
    assert "Cocktail gpu time" in run.stdout
