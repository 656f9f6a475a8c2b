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
from timings of the library's kernels on the device.
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
