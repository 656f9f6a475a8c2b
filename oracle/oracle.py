"""ctypes access to the CPU oracle. TEST INFRASTRUCTURE ONLY.

* ``port()``: oracle/libclspmv_oracle.so, the plain-C restatement of the
  reference's serial SpMV (clspmv_oracle.c).
* ``ref()``:  oracle/_ref/libclspmv_ref.so, the reference's own templates
  compiled from its sources (None where that build is absent, e.g. on a
  machine without the reference checkout).

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use
this module.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from pathlib import Path

import numpy as np

from clspmv_mic_b200 import _abi
from clspmv_mic_b200.formats import HostMatrix

HERE = Path(__file__).resolve().parent
PORT_LIB = HERE / "libclspmv_oracle.so"
REF_LIB = HERE / "_ref" / "libclspmv_ref.so"
# the reference checkout the recipe compiles from (absent on machines that
# only run the prebuilt oracle/_ref library); CLSPMV_REFERENCE overrides it
REFERENCE_TREE = Path(os.environ.get("CLSPMV_REFERENCE", "/root/reference"))

_port = None
_ref = None
_ref_tried = False


def build(ref: bool = True) -> None:
    """make -C oracle [ref]; the ref target only where the reference tree exists."""
    subprocess.run(["make", "-s", "-C", str(HERE), "all"], check=True)
    if ref and (REFERENCE_TREE / "include" / "matrix_storage.h").exists():
        subprocess.run(["make", "-s", "-C", str(HERE), "ref", f"REF={REFERENCE_TREE}"], check=True)


def _sp(fmt):
    return C.POINTER(_abi.FORMATS[fmt][0])


def port():
    global _port
    if _port is None:
        if not PORT_LIB.exists():
            build(ref=False)
        L = C.CDLL(str(PORT_LIB))
        VP = C.c_void_p
        for fmt in ("coo", "csr", "ell", "sell", "sbell", "bell", "b4csr", "b4ell"):
            fn = getattr(L, f"orc_{fmt}_spmv_f32")
            fn.restype = None
            fn.argtypes = [_sp(fmt), VP, VP]
        for fmt in ("dia", "bdia", "bcsr"):
            fn = getattr(L, f"orc_{fmt}_spmv_f32")
            fn.restype = None
            fn.argtypes = [_sp(fmt), VP, VP, C.c_int]
        L.orc_csr_spmv_f64.restype = None
        L.orc_csr_spmv_f64.argtypes = [_sp("csr"), VP, VP, VP]
        _port = L
    return _port


def ref():
    """The compiled reference, or None when oracle/_ref was not built."""
    global _ref, _ref_tried
    if not _ref_tried:
        _ref_tried = True
        if REF_LIB.exists():
            L = C.CDLL(str(REF_LIB))
            VP, I, U = C.c_void_p, C.c_int, C.c_uint
            sig = {
                "ref_free": (None, [VP]),
                "ref_sort_coo": (I, [_sp("coo")]),
                "ref_if_sorted_coo": (I, [_sp("coo")]),
                "ref_coo2csr": (None, [_sp("coo"), _sp("csr")]),
                "ref_pad_csr": (None, [_sp("csr"), _sp("csr"), I]),
                "ref_coo2dia": (I, [_sp("coo"), _sp("dia"), I]),
                "ref_coo2bdia": (I, [_sp("coo"), _sp("bdia"), I]),
                "ref_coo2ell": (None, [_sp("coo"), _sp("ell"), I, I]),
                "ref_coo2sell": (None, [_sp("coo"), _sp("sell"), U]),
                "ref_coo2bcsr": (None, [_sp("coo"), _sp("bcsr"), U, U, I]),
                "ref_coo2b4csr": (I, [_sp("coo"), _sp("b4csr"), U, U, I]),
                "ref_coo2bell": (None, [_sp("coo"), _sp("bell"), U, U, I, I]),
                "ref_coo2b4ell": (I, [_sp("coo"), _sp("b4ell"), U, U, I, I]),
                "ref_coo2sbell": (I, [_sp("coo"), _sp("sbell"), U, U, U]),
                "ref_spmv_only": (None, [_sp("coo"), VP, VP]),
                "ref_read_mmf": (None, [C.c_char_p, _sp("coo")]),
                "ref_analyze_matrix": (None, [_sp("coo"), C.POINTER(_abi.Cocktail), C.c_char_p, C.c_float, I, I]),
            }
            for fmt in ("dia", "bdia", "ell", "bcsr", "bell"):
                sig[f"ref_{fmt}2coo"] = (None, [_sp(fmt), _sp("coo")])
            for fmt in ("coo", "csr", "dia", "bdia", "ell", "sell", "sbell", "bcsr", "bell"):
                sig[f"ref_{fmt}_spmv"] = (None, [_sp(fmt), VP, VP, I])
            for name, (res, args) in sig.items():
                fn = getattr(L, name)
                fn.restype = res
                fn.argtypes = args
            _ref = L
    return _ref


class RefMatrix(HostMatrix):
    """A struct filled by the compiled reference (arrays malloc'ed there)."""

    def __del__(self):
        L = ref()
        if L is not None and getattr(self, "_ref_owned", False):
            for field, _, _ in _abi.FORMATS[self.fmt][1]:
                p = getattr(self.struct, field)
                if p:
                    L.ref_free(p)
            self._ref_owned = False


def ref_convert(fmt: str, coo: HostMatrix, *args):
    """Runs the reference's coo2<fmt> on a private copy of `coo` (the
    reference sorts its input in place). Returns (ok, RefMatrix)."""
    L = ref()
    src = coo.copy()
    out = _abi.FORMATS[fmt][0]()
    rc = getattr(L, f"ref_coo2{fmt}")(C.byref(src.struct), C.byref(out), *args)
    ok = True if rc is None else bool(rc)
    m = RefMatrix(fmt, out)
    m._ref_owned = ok
    return ok, m


def _f32(a):
    return np.ascontiguousarray(a, dtype=np.float32)


def _x_padded(x):
    """x followed by 64 zeros. The reference's serial block products
    (bell_spmv, include/spmv_serial.h:251-279) read x up to a block's width
    past the last block column without a bound check, so every oracle call
    gets a buffer with zero padding; the logical length stays x.size."""
    x = _f32(x)
    xp = np.zeros(x.size + 64, dtype=np.float32)
    xp[:x.size] = x
    return xp, x.size


def spmv_port(m: HostMatrix, x: np.ndarray, y: np.ndarray | None = None, out_len: int | None = None) -> np.ndarray:
    """result += A x with the C restatement; returns the result array."""
    L = port()
    x, nx = _x_padded(x)
    n = out_len if out_len is not None else m.shape[0]
    res = np.zeros(n, dtype=np.float32) if y is None else _f32(y).copy()
    fn = getattr(L, f"orc_{m.fmt}_spmv_f32")
    if m.fmt in ("dia", "bdia", "bcsr"):
        fn(C.byref(m.struct), x.ctypes.data, res.ctypes.data, nx)
    else:
        fn(C.byref(m.struct), x.ctypes.data, res.ctypes.data)
    return res


def spmv_ref(m: HostMatrix, x: np.ndarray, y: np.ndarray | None = None, out_len: int | None = None) -> np.ndarray:
    """result += A x with the reference's own <fmt>_spmv."""
    L = ref()
    x, nx = _x_padded(x)
    n = out_len if out_len is not None else m.shape[0]
    res = np.zeros(n, dtype=np.float32) if y is None else _f32(y).copy()
    getattr(L, f"ref_{m.fmt}_spmv")(C.byref(m.struct), x.ctypes.data, res.ctypes.data, nx)
    return res


def csr_f64(csr: HostMatrix, x: np.ndarray):
    """FP64 row sums and the tolerance scale sum_j |a_ij x_j|."""
    L = port()
    x = _f32(x)
    h = csr.shape[0]
    y64 = np.zeros(h, dtype=np.float64)
    sc = np.zeros(h, dtype=np.float64)
    L.orc_csr_spmv_f64(C.byref(csr.struct), x.ctypes.data, y64.ctypes.data, sc.ctypes.data)
    return y64, sc
