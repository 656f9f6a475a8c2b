"""Cocktail benchmark tables in the reference's `.ben` formats.

The Cocktail partitioner (analyze_matrix) interpolates per-format GFLOP/s
tables that the reference's bench_* programs write to
$CLSPMVPATH/benchmark/<fmt>.ben (src/bench_*.cpp). Formats, as read by
src/analyze.cpp:16-174:

    overhead.ben   groupnum threadnum microseconds
    bdia.ben       dimension width  g0 .. g4        (5 variants)
    dia.ben        dimension width  g0 .. g3        (rows aligned 1:1 with bdia.ben)
    sbell.ben      bh bw dimension blocknum  g0     (shapes: bw in {4,8} outer, bh in {1,2,4,8} inner)
    bell.ben       bh bw dimension blocknum  g0 g1
    bcsr.ben       bh bw dimension blocknum  g0
    sell.ben       dimension width  g0 g1           (slice 32, slice 128)
    ell.ben        dimension width  g0 g1
    csr.ben        dimension width groupnum  g0 g1  (the same group list for every (dim, width))
    coo.ben        dimension width groupnum  g0

model_tables() writes a deterministic bandwidth model of this library's
kernels on B200 (measured HBM copy bandwidth, launch overhead, x-gather
cost); `seed` perturbs the variant factors so tests can drive the
partitioner down different branches. measure_tables() fills the same files
from timings of the library's kernels on the device (regular synthetic
matrices of each format built on the device).
"""
from __future__ import annotations

import math
import os
from pathlib import Path

import numpy as np

DIMS = [1024 << k for k in range(12)]                       # 1024 .. 2,097,152 rows
DIA_WIDTHS = [1, 3, 5, 7, 9, 11, 13, 15, 19, 23, 27, 31, 35, 39, 43, 47, 51, 55, 59, 63]
FLAT_WIDTHS = [1, 2, 3, 4, 6, 8, 12, 16, 24, 32, 48, 64]
CSR_WIDTHS = [1, 2, 4, 8, 16, 32, 64]
GROUPS = [24, 48, 96, 192, 288]
BLOCKNUMS = [1, 2, 3, 4, 6, 8, 12, 16]
SHAPES = [(bh, bw) for bw in (4, 8) for bh in (1, 2, 4, 8)]   # analyze.cpp:545-560 order
OVH_GROUPS = [1 << k for k in range(17)]
OVH_THREADS = [64, 128, 256]
IMP = {"bdia": 5, "dia": 4, "sbell": 1, "bell": 2, "bcsr": 1, "sell": 2, "ell": 2, "csr": 2, "coo": 1}


def _gflops(flops, bytes_, bw, t0, gather=0.0):
    t = bytes_ / bw + t0 + gather
    return flops / t / 1e9


def model_tables(root: str | os.PathLike, seed: int = 0, hbm_gbs: float = 6000.0, launch_us: float = 4.0,
                 scale: dict | None = None, gather_per_s: float = 160e9) -> Path:
    """Writes <root>/benchmark/*.ben from the bandwidth model; returns root.
    `scale` multiplies whole formats' GFLOP/s (e.g. {"coo": 0.3}), which is
    how tests steer the partitioner into multi-format partitions."""
    rng = np.random.default_rng(seed)
    sc = {k: 1.0 for k in IMP}
    sc.update(scale or {})

    def f(n):   # per-variant factors, perturbed by the seed
        base = np.linspace(1.0, 0.9, n)
        return base * (1.0 + (rng.uniform(-0.08, 0.08, n) if seed else 0.0))

    bw = hbm_gbs * 1e9
    t0 = launch_us * 1e-6
    gather_s = 1.0 / gather_per_s   # seconds per random x gather (~160e9/s measured on B200 power-law runs)
    out = Path(root) / "benchmark"
    out.mkdir(parents=True, exist_ok=True)
    lines = {k: [] for k in ["overhead", "bdia", "dia", "sbell", "bell", "bcsr", "sell", "ell", "csr", "coo"]}

    for g in OVH_GROUPS:
        for th in OVH_THREADS:
            lines["overhead"].append(f"{g} {th} {launch_us + 0.0002 * g * th / 256:.6f}")

    fb, fd = f(5), f(4)
    for d in DIMS:
        for w in DIA_WIDTHS:
            by = d * (4.0 * w + 12.0)
            dia = [_gflops(2.0 * d * w, by, bw, t0) * fd[i] * sc["dia"] for i in range(4)]
            reuse = 0.88 + 0.025 * min(w, 8)          # BDIA pays off on wide bands
            bdia = [_gflops(2.0 * d * w, by, bw, t0) * fb[i] * reuse * sc["bdia"] for i in range(5)]
            lines["bdia"].append(f"{d} {w} " + " ".join(f"{v:.6f}" for v in bdia))
            lines["dia"].append(f"{d} {w} " + " ".join(f"{v:.6f}" for v in dia))

    shape_f = {name: {s: f(IMP[name]) * (1.0 + 0.02 * k) for k, s in enumerate(SHAPES)} for name in ("sbell", "bell", "bcsr")}
    for name in ("sbell", "bell", "bcsr"):
        for (bh, bwid) in SHAPES:
            for d in DIMS:
                for b in BLOCKNUMS:
                    nnz_row = b * bwid
                    by = d * (4.0 * nnz_row + 4.0 * b / bh + 12.0)
                    g = [_gflops(2.0 * d * nnz_row, by, bw, t0) * shape_f[name][(bh, bwid)][i] * sc[name]
                         for i in range(IMP[name])]
                    lines[name].append(f"{bh} {bwid} {d} {b} " + " ".join(f"{v:.6f}" for v in g))

    fs, fe = f(2), f(2)
    for d in DIMS:
        for w in FLAT_WIDTHS:
            by = d * (8.0 * w + 12.0)
            gat = d * w * gather_s
            sell = [_gflops(2.0 * d * w, by, bw, t0, gat) * fs[i] * sc["sell"] for i in range(2)]
            ell = [_gflops(2.0 * d * w, by, bw, t0, gat) * fe[i] * 0.97 * sc["ell"] for i in range(2)]
            lines["sell"].append(f"{d} {w} " + " ".join(f"{v:.6f}" for v in sell))
            lines["ell"].append(f"{d} {w} " + " ".join(f"{v:.6f}" for v in ell))

    fc, fo = f(2), f(1)
    for d in DIMS:
        for w in CSR_WIDTHS:
            gat = d * w * gather_s
            for g in GROUPS:
                occ = min(1.0, g / 192.0) ** 0.5
                csr = [_gflops(2.0 * d * w, d * (8.0 * w + 16.0), bw, t0, gat) * fc[i] * occ * sc["csr"] for i in range(2)]
                coo = [_gflops(2.0 * d * w, d * (12.0 * w + 12.0), bw, t0, gat) * fo[0] * occ * sc["coo"]]
                lines["csr"].append(f"{d} {w} {g} " + " ".join(f"{v:.6f}" for v in csr))
                lines["coo"].append(f"{d} {w} {g} " + " ".join(f"{v:.6f}" for v in coo))

    for name, ls in lines.items():
        (out / f"{name}.ben").write_text("\n".join(ls) + "\n")
    return Path(root)


# grids of the device-measured tables (the partitioner interpolates between
# grid points and clamps outside them, src/analyze.cpp:294-428)
M_DIMS = [16384, 131072, 1048576, 2097152]
M_BLOCK_DIMS = [16384, 131072, 1048576]
M_DIA_WIDTHS = [1, 3, 5, 7, 9, 15, 27, 31, 63]
M_FLAT_WIDTHS = [1, 2, 4, 8, 16, 32, 64]
M_BLOCKNUMS = [1, 2, 4, 8, 16]
M_GROUPS = [24, 192]


def _time_ms(run, reps: int = 10) -> float:
    import torch
    for _ in range(3):
        run()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(reps):
        run()
    e1.record()
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / reps


def measure_tables(root: str | os.PathLike, reps: int = 10, device="cuda") -> Path:
    """Writes <root>/benchmark/*.ben from timings of this library's kernels
    on the current device (what the reference's bench_* programs do with
    its OpenCL kernels, src/bench_dia.cpp:355-400 and the others): regular
    synthetic matrices of each format built on the device
    (device_build.py), y += A x timed with CUDA events, GFLOP/s =
    2 nnz / time. Every kernel-variant column of a table gets the value of
    this library's one kernel for that format, except SELL, whose two
    columns are slice heights 32 and 128."""
    import torch
    from . import device_build as D
    from .drivers import bandwidth_test
    out = Path(root) / "benchmark"
    out.mkdir(parents=True, exist_ok=True)
    lines = {k: [] for k in ["overhead", "bdia", "dia", "sbell", "bell", "bcsr", "sell", "ell", "csr", "coo"]}

    def gflops(m, nnz, **kw):
        x = torch.rand(m.shape[1], device=device)
        y = torch.zeros(m.shape[0], device=device)
        ms = _time_ms(lambda: m.spmv(x, y, 1.0, 1.0, **kw), reps)
        return 2.0 * nnz / (ms * 1e-3) / 1e9

    launch_us = bandwidth_test(1 << 20, 50)["launch_us"]
    for g in OVH_GROUPS:
        for th in OVH_THREADS:
            lines["overhead"].append(f"{g} {th} {launch_us:.6f}")
    for d in M_DIMS:
        for w in M_DIA_WIDTHS:
            dv = gflops(D.dia(d, w, device=device), d * w)
            bv = gflops(D.bdia(d, w, device=device), d * w)
            lines["dia"].append(f"{d} {w} " + " ".join(f"{dv:.6f}" for _ in range(IMP["dia"])))
            lines["bdia"].append(f"{d} {w} " + " ".join(f"{bv:.6f}" for _ in range(IMP["bdia"])))
            torch.cuda.empty_cache()
    for name, build in (("sbell", D.sbell), ("bell", D.b4ell), ("bcsr", D.b4csr)):
        for (bh, bw) in SHAPES:
            for d in M_BLOCK_DIMS:
                for b in M_BLOCKNUMS:
                    v = gflops(build(d, b, bh, bw, device=device), d * b * bw)
                    lines[name].append(f"{bh} {bw} {d} {b} " + " ".join(f"{v:.6f}" for _ in range(IMP[name])))
                torch.cuda.empty_cache()
    for d in M_DIMS:
        for w in M_FLAT_WIDTHS:
            s32 = gflops(D.sell(d, w, 32, device=device), d * w)
            s128 = gflops(D.sell(d, w, 128, device=device), d * w)
            ev = gflops(D.ell(d, w, device=device), d * w)
            lines["sell"].append(f"{d} {w} {s32:.6f} {s128:.6f}")
            lines["ell"].append(f"{d} {w} " + " ".join(f"{ev:.6f}" for _ in range(IMP["ell"])))
            cv = gflops(D.csr(d, w, device=device), d * w, variant="merge")
            ov = gflops(D.coo(d, w, device=device), d * w)
            for g in M_GROUPS:
                lines["csr"].append(f"{d} {w} {g} " + " ".join(f"{cv:.6f}" for _ in range(IMP["csr"])))
                lines["coo"].append(f"{d} {w} {g} {ov:.6f}")
            torch.cuda.empty_cache()
    for name, ls in lines.items():
        (out / f"{name}.ben").write_text("\n".join(ls) + "\n")
    return Path(root)


def default_table_root() -> Path:
    """Tables shipped with the package (written by model_tables at build
    time when absent)."""
    return Path(__file__).resolve().parent / "tables"


def ensure_default_tables() -> Path:
    root = default_table_root()
    if not (root / "benchmark" / "coo.ben").exists():
        model_tables(root)
    return root


if __name__ == "__main__":
    import sys
    print(model_tables(sys.argv[1] if len(sys.argv) > 1 else default_table_root()))
