"""Command line equivalents of clSpMV's programs.

    python -m clspmv_mic_b200 all <matrix.mtx> [method] [ntimes]
        spmv_all (src/spmv_all.cpp:156-256): method 0 measures copy
        bandwidth and launch overhead; 1 csr scalar, 2 csr vector, 3 bdia,
        4 dia, 5 ell, 6 coo, 7 bell, 8 bcsr, 9 sell, 10 sbell (as the
        reference); 11 csr merge-path (this library's CSR kernel).
    python -m clspmv_mic_b200 cocktail <matrix.mtx> [table_dir]
        spmv_cocktail (src/eval.cpp:100-131): read, print the matrix info,
        partition with the benchmark tables of table_dir (default
        $CLSPMVPATH, else the tables shipped with the package), evaluate.
    python -m clspmv_mic_b200 spmm <b4csr|b4ell|sbell|csr|coo> <k> [reps] [block_rows] [f32|bf16|f16|tc]
        Y = A X with k right-hand sides on the synthetic 4x4-block matrix
        (block_rows x 8 dense blocks, default 500,000) or, for csr / coo, the
        power-law matrix (2^20 rows): prints the mean time and GFLOP/s. "tc"
        runs b4csr on the tensor cores (FP32 values). The command the SpMM
        kernel profiles are taken with.
"""
from __future__ import annotations

import os
import sys

import numpy as np

from . import _abi
from .cocktail import analyze
from .drivers import bandwidth_test, evaluate, read_mmf, run_method
from .tables import ensure_default_tables

_BY_NUMBER = {v: k for k, v in _abi.METHODS.items()}


def _usage() -> int:
    print(__doc__)
    return 0


def main(argv: list[str]) -> int:
    if len(argv) < 2:
        return _usage()
    cmd, path = argv[0], argv[1]
    if cmd == "all":
        method = int(argv[2]) if len(argv) > 2 else 1
        ntimes = int(argv[3]) if len(argv) > 3 else 20
        if method == 0:
            for nbytes in [32 << (10 + k) for k in range(11)]:
                bandwidth_test(nbytes, 100, verbose=True)
            return 0
        if method not in _BY_NUMBER:
            return _usage()
        coo = read_mmf(path)
        run_method(coo, _BY_NUMBER[method], ntimes, verbose=True)
        return 0
    if cmd == "spmm":
        return _spmm(path, argv[2:])
    if cmd == "cocktail":
        coo = read_mmf(path)
        table_dir = argv[2] if len(argv) > 2 else os.environ.get("CLSPMVPATH") or str(ensure_default_tables())
        h, w = coo.shape
        print(f"\nMatInfo: Width {w} Height {h} NNZ {coo.nnz}")
        vec = np.ones(w, dtype=np.float32)
        res = np.zeros(h, dtype=np.float32)
        a = coo.arrays()
        coores = np.zeros(h, dtype=np.float32)
        np.add.at(coores, a["coo_row_id"], a["coo_data"] * vec[a["coo_col_id"]])
        mat = analyze(coo, table_dir)
        evaluate(mat, vec, res, coores, 1000, verbose=True)
        return 0
    return _usage()


def _spmm(fmt: str, rest: list[str]) -> int:
    import torch
    from . import formats as F
    from . import synth
    k = int(rest[0]) if rest else 32
    reps = int(rest[1]) if len(rest) > 1 else 20
    brows = int(rest[2]) if len(rest) > 2 else 500_000
    vt = rest[3] if len(rest) > 3 else "f32"
    if fmt in ("csr", "coo"):   # the power-law matrix (2^20 rows, Zipf 2.0, mean 16)
        coo = F.coo_matrix(*synth.powerlaw(1 << 20))
        host = F.coo2csr(coo) if fmt == "csr" else coo
    else:
        coo = F.coo_matrix(*synth.block_rows(brows, 8))
        host = {"b4csr": lambda: F.coo2b4csr(coo, 4, 4), "b4ell": lambda: F.coo2b4ell(coo, 4, 4),
                "sbell": lambda: F.coo2sbell(coo, 4, 4, 32)}[fmt]()
    m = F.DeviceMatrix(host)
    rows, cols = m.shape
    g = torch.Generator(device="cuda")
    g.manual_seed(5)
    X = torch.rand((cols, k), generator=g, device="cuda") * 2 - 1
    Y = torch.empty((rows, k), device="cuda")
    if vt == "tc":
        run = lambda: F.device_spmm_tc(m, X, Y, 1.0, 0.0)
    else:
        p = None if vt == "f32" else m.pack(vt)
        run = lambda: m.spmm(X, Y, 1.0, 0.0, packed=p)
    for _ in range(3):
        run()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(reps):
        run()
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / reps
    print(f"{fmt} k={k} {vt}: {ms:.4f} ms, {2.0 * m.nnz * k / (ms * 1e-3) / 1e9:.1f} GFLOP/s")
    if vt == "tc" and F.tensor_timeouts():
        print("tensor-core kernel: a bounded wait ran out")
        return 1
    return 0


if __name__ == "__main__":
    sys.exit(main(sys.argv[1:]))
