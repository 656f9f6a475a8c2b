"""Device-measured choice of a matrix's Cocktail partition.

The Cocktail partitioner (analyze_matrix, src/analyze.cpp:3714-3900) picks
formats from benchmark tables and its own cost estimates; some of those
estimates are blind to costs that dominate on a GPU (an SBELL slice as wide
as its widest block row, for instance, is estimated at the mean block
count). The reference exposes three knobs for such cases
(src/eval.cpp:83-95: the DIA priority multiplier, estimate_flat_partial,
estimate_flat_full). tune() runs the partitioner under each knob setting,
measures every distinct partition on the device with the Cocktail runtime,
keeps the fastest, and caches the winning setting per matrix signature, so
the next matrix with the same structure is partitioned once, without
measuring. Beyond the reference's knobs, each partition with a COO part is
also measured with that part stored as CSR ("flat_as": "csr"), since on this
GPU the chunked CSR kernel and the COO kernel reach the same gather rate and
CSR moves a third fewer bytes. The winning partition is then refined part
by part (refine_parts): the SELL part over slice heights and the block
parts over the eight block shapes, each candidate converted on the device
and timed alone, the fastest kept and cached with the knob.
"""
from __future__ import annotations

import hashlib
import json
import os
from dataclasses import dataclass, field
from pathlib import Path

import numpy as np

from . import formats as F
from .cocktail import CocktailMatrix, analyze
from .formats import HostMatrix

KNOBS = [
    {},                                   # the reference's defaults
    {"estimate_flat_partial": False},
    {"estimate_flat_full": True},
    {"dia_priority_multiplier": 2.0},
    {"dia_priority_multiplier": 2.0, "estimate_flat_partial": False},
    {"dia_priority_multiplier": 0.5},
    # diagonals held back and flat rows split off: on a stacked matrix whose
    # band spans a fraction of the rows, a DIA part pays for its whole
    # height, which the tables' square benchmark matrices do not show
    {"dia_priority_multiplier": 0.5, "estimate_flat_partial": False},
]


def signature(coo: HostMatrix) -> str:
    """Structural fingerprint: shape, nonzeros, and log2 histograms of the
    row lengths and of the distances |col - row| (matrices that share it
    get the same partition setting)."""
    a = coo.arrays()
    h, w = coo.shape
    r, c = a["coo_row_id"].astype(np.int64), a["coo_col_id"].astype(np.int64)
    lens = np.bincount(r, minlength=h) if r.size else np.zeros(h, np.int64)
    lh = np.bincount(np.log2(lens + 1).astype(np.int64), minlength=16)[:32]
    dh = np.bincount(np.log2(np.abs(c - r) + 1).astype(np.int64), minlength=32)[:40]
    frac = lambda v: np.round(v / max(1, v.sum()), 3).tolist()
    key = json.dumps([h, w, int(coo.nnz), frac(lh), frac(dh)])
    return hashlib.sha1(key.encode()).hexdigest()[:20]


def partition(coo: HostMatrix, table_dir, knob: dict) -> CocktailMatrix:
    """analyze_matrix under `knob` (its reference settings), then the flat
    part's storage choice ("flat_as")."""
    ref = {k: v for k, v in knob.items() if k != "flat_as"}
    m = analyze(coo, table_dir, **ref)
    if knob.get("flat_as") == "csr":
        alt = m.with_flat_as_csr()
        if alt is not None:
            return alt
    return m


# part -> candidate layouts of its nonzeros: (converter, arguments after the COO)
SELL_HEIGHTS = (8, 16, 32, 64, 128)
PART_LAYOUTS = {
    "sell": [("sell", (sh,)) for sh in SELL_HEIGHTS],
    "sbell": [("sbell", (bw, bh, 32)) for bh, bw in F.BLOCK_SHAPES],
    "bell": [("b4ell", (bw, bh)) for bh, bw in F.BLOCK_SHAPES],
    "bcsr": [("b4csr", (bw, bh)) for bh, bw in F.BLOCK_SHAPES],
}


def _layout_of(m: CocktailMatrix, part: str):
    st = getattr(m.struct, part)
    if part == "sell":
        return ("sell", (int(st.sell_slice_height),))
    if part == "sbell":
        return ("sbell", (int(st.sbell_bwidth), int(st.sbell_bheight), int(st.sbell_slice_height)))
    if part == "bell":
        return ("b4ell", (int(st.b4ell_bwidth), int(st.b4ell_bheight)))
    return ("b4csr", (int(st.b4csr_bwidth), int(st.b4csr_bheight)))


def _time_alone(dev, reps: int) -> float:
    import torch
    h, w = dev.shape
    x = torch.rand(w, device="cuda")
    y = torch.zeros(h, device="cuda")
    for _ in range(3):
        dev.spmv(x, y, 1.0, 1.0)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(reps):
        dev.spmv(x, y, 1.0, 1.0)
    e1.record()
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / reps


def apply_part_layouts(m: CocktailMatrix, layouts: dict) -> CocktailMatrix:
    """Re-stores the listed parts in the given layouts ({part: [converter,
    [args]]}), converting each part's nonzeros on the host."""
    for part, (conv, args) in layouts.items():
        if not m.uses(part) or _layout_of(m, part) == (conv, tuple(args)):
            continue
        coo = F.to_coo(m.part(part))
        m = m.with_part(part, getattr(F, f"coo2{conv}")(coo, *args))
    return m


def refine_parts(m: CocktailMatrix, reps: int = 10, report: list | None = None) -> dict:
    """Fastest layout of each refinable part, each candidate converted on the
    device from the part's nonzeros (clspmv_device_coo2<fmt>_f32) and timed
    alone; returns {part: [converter, [args]]} for the parts whose best
    layout differs from the partitioner's."""
    from . import _abi
    chosen = {}
    for part, cands in PART_LAYOUTS.items():
        if not m.uses(part):
            continue
        dcoo = F.DeviceMatrix(F.to_coo(m.part(part)))
        current = _layout_of(m, part)
        best, best_ms, tried = None, None, []
        for conv, args in cands:
            try:
                d = F.device_convert(dcoo, conv, *args)
            except _abi.ClspmvError:
                tried.append(dict(layout=[conv, list(args)], refused=True))
                continue
            ms = _time_alone(d, reps)
            del d
            tried.append(dict(layout=[conv, list(args)], ms=round(ms, 4)))
            if best_ms is None or ms < best_ms:
                best, best_ms = (conv, args), ms
        if report is not None:
            report.append(dict(part=part, partitioner=[current[0], list(current[1])], candidates=tried))
        if best is not None and best != current:
            chosen[part] = [best[0], list(best[1])]
        del dcoo
    return chosen


def _partition_key(m: CocktailMatrix):
    return tuple(sorted((k, v["nnz"]) for k, v in m.summary().items() if isinstance(v, dict) and "nnz" in v))


def apply_runtime(dev, runtime: dict) -> None:
    """Runtime settings of a tuned partition on its device handle: schedule
    ("per_part" / "fused") and the CSR part's lanes per row (0: chunks)."""
    if runtime.get("schedule", "per_part") != "per_part":
        dev.set_schedule(runtime["schedule"])
    if runtime.get("csr_lanes", 0):
        dev.set_csr_lanes(runtime["csr_lanes"])


def measure_ms(m: CocktailMatrix, reps: int = 10, runtime: dict | None = None) -> float:
    """Mean time of y += A x over `reps` runs of the Cocktail runtime."""
    import torch
    dev = m.to_device()
    if runtime:
        apply_runtime(dev, runtime)
    try:
        h, w = m.struct.mat_height, m.struct.mat_width
        x = torch.rand(w, device="cuda")
        y = torch.zeros(h, device="cuda")
        for _ in range(3):
            dev.spmv(x, y, 1.0, 1.0)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(reps):
            dev.spmv(x, y, 1.0, 1.0)
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / reps
    finally:
        dev.close()


CSR_LANES = (0, 1, 2, 4, 8, 16, 32)


def tune_runtime(m: CocktailMatrix, reps: int = 10, report: list | None = None) -> tuple:
    """The launch schedule (one launch per part, or the fused persistent
    launch when the partition has two or more parts it covers) and, with a
    CSR part, its threads per row (nonzero chunks, or CSR-vector with 1..32
    lanes per row), measured in that order. Returns (settings, ms)."""
    best = {"schedule": "per_part", "csr_lanes": 0}
    best_ms = measure_ms(m, reps, best)
    if report is not None:
        report.append(dict(runtime=dict(best), ms=round(best_ms, 4)))
    dev = m.to_device()
    fusable = dev.fused_items > 0
    dev.close()
    cands = [{"schedule": "fused", "csr_lanes": 0}] if fusable else []
    if m.uses("csr"):
        cands += [{"schedule": "per_part", "csr_lanes": t} for t in CSR_LANES if t]
    for rt in cands:
        if rt["csr_lanes"] and best["schedule"] == "fused":
            continue   # the fused launch runs the CSR part by chunks
        ms = measure_ms(m, reps, rt)
        if report is not None:
            report.append(dict(runtime=dict(rt), ms=round(ms, 4)))
        if ms < best_ms:
            best, best_ms = dict(rt), ms
    return best, best_ms


@dataclass
class TuneResult:
    matrix: CocktailMatrix
    knob: dict
    ms: float
    from_cache: bool = False
    report: list = field(default_factory=list)
    parts: dict = field(default_factory=dict)        # refined part layouts
    part_report: list = field(default_factory=list)
    ms_partition: float | None = None                 # before the part refinement
    runtime: dict = field(default_factory=dict)      # schedule and CSR lanes per row
    runtime_report: list = field(default_factory=list)

    def to_device(self):
        """The tuned partition on the device with its runtime settings."""
        dev = self.matrix.to_device()
        apply_runtime(dev, self.runtime)
        return dev


def default_cache() -> Path:
    return Path(os.environ.get("CLSPMV_TUNE_CACHE", Path.home() / ".cache" / "clspmv_b200" / "cocktail_tune.json"))


def tune(coo: HostMatrix, table_dir=None, cache: str | os.PathLike | None = None, reps: int = 10,
         knobs=KNOBS, use_cache: bool = True, refine: bool = True, runtime: bool = True) -> TuneResult:
    """Fastest measured partition of `coo` over the knob settings, its parts'
    layouts (refine) and its runtime settings: launch schedule and the CSR
    part's threads per row (runtime)."""
    cache = Path(cache) if cache is not None else default_cache()
    sig = signature(coo)
    entries = {}
    if cache.exists():
        try:
            entries = json.loads(cache.read_text())
        except (OSError, ValueError):
            entries = {}
    if use_cache and sig in entries:
        knob, parts = entries[sig]["knob"], entries[sig].get("parts", {})
        m = apply_part_layouts(partition(coo, table_dir, knob), parts)
        return TuneResult(m, knob, entries[sig]["ms"], from_cache=True, parts=parts,
                          runtime=entries[sig].get("runtime", {}))
    best, seen, report = None, {}, []
    for ref_knob in knobs:
        base = analyze(coo, table_dir, **ref_knob)
        alt = base.with_flat_as_csr()
        for knob, m in [(ref_knob, base)] + ([({**ref_knob, "flat_as": "csr"}, alt)] if alt is not None else []):
            key = _partition_key(m)
            if key in seen:
                report.append(dict(knob=knob, partition=dict(key), ms=seen[key], same_as_earlier=True))
                continue
            ms = measure_ms(m, reps)
            seen[key] = ms
            report.append(dict(knob=knob, partition=dict(key), ms=round(ms, 4)))
            if best is None or ms < best.ms:
                best = TuneResult(m, knob, ms)
    best.report = report
    best.ms_partition = best.ms
    if refine:
        layouts = refine_parts(best.matrix, reps, best.part_report)
        if layouts:
            m = apply_part_layouts(best.matrix, layouts)
            ms = measure_ms(m, reps)
            if ms < best.ms:
                best.matrix, best.ms, best.parts = m, ms, layouts
    if runtime:
        rt, ms = tune_runtime(best.matrix, reps, best.runtime_report)
        if ms < best.ms:
            best.ms = ms
        best.runtime = rt
    entries[sig] = {"knob": best.knob, "parts": best.parts, "runtime": best.runtime, "ms": best.ms,
                    "shape": list(coo.shape), "nnz": int(coo.nnz)}
    try:
        cache.parent.mkdir(parents=True, exist_ok=True)
        cache.write_text(json.dumps(entries, indent=1))
    except OSError:
        pass
    return best
