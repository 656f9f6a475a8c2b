"""Batches of SpMM jobs run as one persistent kernel launch.

    b = Batch(max_jobs=256)
    b.set([Job(matrix, X, Y), Job(matrix2, X2, Y2, packed=matrix2.pack("bf16")), ...])
    b.run()                    # one launch; capturable in a CUDA graph
    b.close()

Each Job is Y <- alpha * A * X + beta * Y with its own format, value type and
number of right-hand sides (X: width x k, Y: height x k, float32, unit column
stride). The reference has no batched path; one call of its drivers runs one
matrix (src/spmv_cocktail.cpp:1088-1132).
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass
from typing import Optional, Sequence

from . import _abi
from ._abi import check, lib
from .formats import DeviceMatrix, PackedValues, _stream_handle


@dataclass
class Job:
    matrix: DeviceMatrix
    X: object
    Y: object
    alpha: float = 1.0
    beta: float = 0.0
    packed: Optional[PackedValues] = None

    def to_c(self) -> _abi.SpmmJob:
        if self.matrix.fmt not in _abi.FORMAT_IDS or self.matrix.fmt == "coo":
            raise ValueError(f"format {self.matrix.fmt} cannot run in a batch")
        X, Y = self.X, self.Y
        if X.dim() != 2 or Y.dim() != 2 or X.stride(1) != 1 or Y.stride(1) != 1 or X.shape[1] != Y.shape[1]:
            raise ValueError("X and Y must be 2-D, unit column stride, same k")
        p = self.packed
        return _abi.SpmmJob(_abi.FORMAT_IDS[self.matrix.fmt], C.cast(C.byref(self.matrix.struct), C.c_void_p),
                            0 if p is None else _abi.VALUE_TYPES[p.value_type],
                            None if p is None else p.values.data_ptr(), None if p is None else p.row_scale.data_ptr(),
                            X.shape[1], X.data_ptr(), X.stride(0), Y.data_ptr(), Y.stride(0), self.alpha, self.beta)


class Batch:
    def __init__(self, max_jobs: int = 256):
        self._h = C.c_void_p()
        check(lib().clspmv_batch_create(int(max_jobs), C.byref(self._h)), "batch_create")
        self.max_jobs = max_jobs
        self.jobs: list[Job] = []

    def set(self, jobs: Sequence[Job], stream=None) -> None:
        arr = (_abi.SpmmJob * max(len(jobs), 1))(*[j.to_c() for j in jobs])
        bad = C.c_int(-1)
        rc = lib().clspmv_batch_set(self._h, arr, len(jobs), _stream_handle(stream), C.byref(bad))
        check(rc, f"batch_set (job {bad.value})")
        self.jobs = list(jobs)   # keeps the tensors alive while the batch may run

    def run(self, stream=None) -> None:
        check(lib().clspmv_batch_run(self._h, _stream_handle(stream)), "batch_run")

    def close(self) -> None:
        if self._h:
            lib().clspmv_batch_free(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
