"""Benchmark drivers and Matrix Market input, mirroring clSpMV's callers.

    run_method(coo, "bell", ntimes)   spmv_bell() and the other spmv_<fmt>
                                      drivers (src/spmv_<fmt>.cpp)
    bandwidth_test(bytes, ntimes)     method 0 of spmv_all (src/mem_bandwidth.cpp)
    read_mmf(path)                    ReadMMF (src/fileio.cpp:10-109)
    evaluate(cocktail, vec, res, coores, ntimes)
                                      evaluate (src/spmv_cocktail.cpp:1431-1455)

All of them call libclspmv_b200.so; the timings are CUDA-event times of the
library's kernels on the current device.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from . import _abi
from ._abi import METHODS, check, lib
from .formats import HostMatrix


def _variant(v: _abi.BenchVariant, method: str) -> dict:
    d = dict(status=_abi.STATUS.get(v.status, v.status), ms=v.ms, gflops=v.gflops, distance=v.distance,
             max_diff=v.max_diff, max_diff_ratio=v.max_diff_ratio)
    if method in ("bell", "sbell", "bcsr"):
        d.update(bheight=v.param0, bwidth=v.param1)
    elif method == "sell":
        d.update(slice_height=v.param0)
    elif method == "csr_vector":
        d.update(lanes=v.param0)
    elif method == "csr_scalar":
        d.update(padding=v.param0)
    return d


def run_method(coo: HostMatrix, method: str, ntimes: int = 20, verbose: bool = False) -> dict:
    """Runs the spmv_<method> driver on a sorted COO matrix and returns every
    variant's time, GFLOP/s and check against the host COO product."""
    if method not in METHODS or method == "bandwidth":
        raise ValueError(f"unknown method {method!r}; one of {sorted(k for k in METHODS if k != 'bandwidth')}")
    r = _abi.BenchResult()
    status = lib().clspmv_run_method_f32(C.byref(coo.struct), METHODS[method], int(ntimes), int(verbose), C.byref(r))
    variants = [_variant(r.v[i], method) for i in range(r.nvariants)]
    if status not in (_abi.OK, _abi.ERR_REFUSED):
        check(status, f"spmv_{method}")
    return dict(method=method, status=_abi.STATUS.get(status, status), best=r.best, best_ms=r.best_ms,
                best_gflops=r.best_gflops, variants=variants)


def bandwidth_test(nbytes: int = 256 << 20, ntimes: int = 20, verbose: bool = False) -> dict:
    gbs, us = C.c_double(), C.c_double()
    check(lib().clspmv_bandwidth_test(int(nbytes), int(ntimes), int(verbose), C.byref(gbs), C.byref(us)),
          "bandwidth_test")
    return dict(copy_gbs=gbs.value, launch_us=us.value, bytes=int(nbytes))


def gather_test(x_len: int = 1 << 20, count: int = 1 << 24, ntimes: int = 20, verbose: bool = False) -> float:
    """Random gathers per second from an x of x_len floats (the bound of the
    scattered-column formats)."""
    g = C.c_double()
    check(lib().clspmv_gather_test(int(x_len), int(count), int(ntimes), int(verbose), C.byref(g)), "gather_test")
    return g.value


def read_mmf(path: str | os.PathLike) -> HostMatrix:
    """ReadMMF: a coordinate Matrix Market file as a row-sorted COO matrix."""
    out = _abi.Coo()
    status = lib().clspmv_read_mmf_f32(os.fsencode(path), C.byref(out))
    check(status, f"read_mmf({path})")
    return HostMatrix("coo", out, lib_owned=True)


def evaluate(cocktail, vec: np.ndarray, res: np.ndarray, coores: np.ndarray | None = None, ntimes: int = 1000,
             verbose: bool = False) -> dict:
    """evaluate(): upload a partitioned matrix, check one SpMV res + A*vec
    against `coores`, time `ntimes` SpMVs."""
    vec = np.ascontiguousarray(vec, dtype=np.float32)
    res = np.ascontiguousarray(res, dtype=np.float32)
    cr = None if coores is None else np.ascontiguousarray(coores, dtype=np.float32)
    ms, gf, md = C.c_double(), C.c_double(), C.c_double(float("nan"))
    check(lib().clspmv_cocktail_evaluate_f32(C.byref(cocktail.struct), vec.ctypes.data, res.ctypes.data,
                                             None if cr is None else cr.ctypes.data, int(ntimes), int(verbose),
                                             C.byref(ms), C.byref(gf), C.byref(md)), "evaluate")
    return dict(ms=ms.value, gflops=gf.value, max_diff=md.value)
