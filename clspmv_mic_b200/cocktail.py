"""Cocktail partitioning (analyze_matrix) and the partitioned matrix.

analyze(coo, table_dir) runs the library's restatement of clSpMV's
analyze_matrix (src/analyze.cpp) through the C ABI and returns a
CocktailMatrix: the nine part slots of cocktail<int,int,float> as
HostMatrix views (None for unused parts) plus the chosen variants.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

from . import _abi
from ._abi import COCKTAIL_PARTS, check, lib
from .formats import HostMatrix


class CocktailMatrix:
    def __init__(self, struct: _abi.Cocktail, owner: str = "lib", releaser=None):
        self.struct = struct
        self._owner = owner
        self._releaser = releaser

    def __del__(self):
        if getattr(self, "_owner", None) == "lib":
            try:
                lib().clspmv_free_cocktail_f32(C.byref(self.struct))
            except Exception:
                pass
        elif getattr(self, "_releaser", None) is not None:
            try:
                self._releaser(self.struct)
            except Exception:
                pass
        self._owner = None
        self._releaser = None

    def uses(self, part: str) -> bool:
        return bool(getattr(self.struct, f"ifuse{part}"))

    def part(self, part: str):
        """HostMatrix view of one part (no copy), or None when unused."""
        if not self.uses(part):
            return None
        fmt = dict(COCKTAIL_PARTS)[part]
        return HostMatrix(fmt, getattr(self.struct, part))

    def parts(self) -> dict:
        return {p: self.part(p) for p, _ in COCKTAIL_PARTS if self.uses(p)}

    def with_flat_as_csr(self) -> "CocktailMatrix | None":
        """The same partition with its COO part stored as CSR instead (same
        nonzeros; the chunked CSR kernel reads 8 bytes per nonzero where COO
        reads 12), or None when there is no COO part or a CSR part exists
        already. The parts are shared with this matrix, which the result
        keeps alive."""
        if not self.uses("coo") or self.uses("csr"):
            return None
        from .formats import coo2csr
        csr = coo2csr(self.part("coo"))
        st = _abi.Cocktail.from_buffer_copy(self.struct)
        st.ifusecoo = False
        st.ifusecsr = True
        st.csr = _abi.Csr.from_buffer_copy(csr.struct)
        st.coo = _abi.Coo()
        out = CocktailMatrix(st, owner=None)
        out._base, out._csr = self, csr
        return out

    def with_part(self, part: str, host: HostMatrix) -> "CocktailMatrix":
        """The same partition with part `part` replaced by `host` (the same
        nonzeros in another layout of that slot's format, e.g. another block
        shape or slice height). Shares the other parts with this matrix,
        which the result keeps alive."""
        if not self.uses(part):
            raise ValueError(f"part {part} is not used")
        st = _abi.Cocktail.from_buffer_copy(self.struct)
        setattr(st, part, type(getattr(st, part)).from_buffer_copy(host.struct))
        out = CocktailMatrix(st, owner=None)
        out._base, out._part = self, host
        return out

    def to_device(self) -> "DeviceCocktail":
        return DeviceCocktail(self)

    def summary(self) -> dict:
        s = self.struct
        out = {"shape": (s.mat_height, s.mat_width), "nnz": s.mat_nnz}
        for p, _ in COCKTAIL_PARTS:
            if self.uses(p):
                m = self.part(p)
                out[p] = {"nnz": m.nnz, "meth": getattr(s, f"{p}_meth_num")}
        out["csr_group_num"] = s.csr_group_num
        out["coo_group_num"] = s.coo_group_num
        return out


def analyze(coo: HostMatrix, table_dir: str | os.PathLike | None = None, dia_priority_multiplier: float = 1.0,
            estimate_flat_partial: bool = True, estimate_flat_full: bool = False) -> CocktailMatrix:
    """analyze_matrix (src/analyze.cpp:3714-3900): tables from
    <table_dir>/benchmark/*.ben (default: $CLSPMVPATH, then the package's
    tables)."""
    if table_dir is None:
        table_dir = os.environ.get("CLSPMVPATH")
    if table_dir is None:
        from .tables import ensure_default_tables
        table_dir = ensure_default_tables()
    out = _abi.Cocktail()
    rc = lib().clspmv_analyze_matrix_f32(C.byref(coo.struct), C.byref(out), str(table_dir).encode(),
                                         dia_priority_multiplier, int(estimate_flat_partial), int(estimate_flat_full))
    m = CocktailMatrix(out, owner="lib" if rc == 0 else None)
    check(rc, "analyze_matrix")
    return m


class DeviceCocktail:
    """Device residency of a CocktailMatrix (clspmv_cocktail_upload_f32)."""

    def __init__(self, host: CocktailMatrix):
        self.handle = C.c_void_p()
        check(lib().clspmv_cocktail_upload_f32(C.byref(host.struct), C.byref(self.handle)), "cocktail_upload")
        self.shape = (host.struct.mat_height, host.struct.mat_width)
        self.nnz = host.struct.mat_nnz
        self.parts = [p for p, _ in COCKTAIL_PARTS if host.uses(p)]
        self.stored_bytes = sum(m.stored_bytes() for m in host.parts().values())

    SCHEDULES = {"auto": 0, "fused": 1, "per_part": 2}

    def set_schedule(self, schedule: str) -> None:
        """"auto" (= "per_part": one launch per part on forked streams) or
        "fused" (one persistent launch over all parts from an interleaved
        work list; refused where a part is not covered)."""
        check(lib().clspmv_cocktail_set_schedule(self.handle, self.SCHEDULES[schedule]), "cocktail_set_schedule")

    def set_csr_lanes(self, lanes: int) -> None:
        """CSR part's kernel: 0 nonzero chunks, or CSR-vector with `lanes`
        lanes per row (1..32, powers of two)."""
        check(lib().clspmv_cocktail_set_csr_lanes(self.handle, int(lanes)), "cocktail_set_csr_lanes")

    @property
    def sell_planned(self) -> bool:
        """The SELL part runs through a length plan (clspmv_cocktail_sell_planned)."""
        return lib().clspmv_cocktail_sell_planned(self.handle) == 1

    @property
    def fused_items(self) -> int:
        """Work-list entries of the fused schedule (0: the handle has none)."""
        return int(lib().clspmv_cocktail_fused_items(self.handle))

    def spmv(self, x, y, alpha: float = 1.0, beta: float = 1.0, stream=None) -> None:
        """y <- alpha * A x + beta * y, asynchronous on `stream`."""
        from .formats import _stream_handle
        check(lib().clspmv_cocktail_spmv_f32(self.handle, x.data_ptr(), y.data_ptr(), alpha, beta,
                                             _stream_handle(stream)), "cocktail_spmv")

    def iterate(self, x, y, iterations: int, alpha: float = 1.0, beta: float = 1.0, stream=None) -> None:
        """`iterations` steps of y <- alpha * A x + beta * y; x[:rows] <- y
        (the reference's A^k x loop, src/eval.cpp:19-72), asynchronous on
        `stream`, replayed from a cached CUDA graph (clspmv_cocktail_iterate_f32)."""
        from .formats import _stream_handle
        check(lib().clspmv_cocktail_iterate_f32(self.handle, x.data_ptr(), y.data_ptr(), alpha, beta, int(iterations),
                                                _stream_handle(stream)), "cocktail_iterate")

    def close(self):
        if self.handle:
            lib().clspmv_cocktail_free(self.handle)
            self.handle = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
