#!/usr/bin/env python
"""bench.py — per-format FP32 SpMV sweep on B200 (the reference's per-format
benchmark, src/spmv_all.cpp:196-250, on synthetic matrices of the named
shapes).

One step = one y += A x launch of each of the nine formats on its matrix,
with the format's best kernel (the reference's drivers likewise report the
best variant per format, e.g. src/spmv_csr_vector.cpp:649-656):

  stencil27   3D 27-point stencil 128^3 (2,097,152 rows, 55,742,968 nnz):  DIA, BDIA
  powerlaw    2^20 rows, Zipf(2.0) lengths on [1,10000] scaled to mean 16:  CSR (nonzero-chunk kernel),
              COO, ELL (ELL(K) + COO tail, K by the 1/3-of-rows rule), SELL-32 (read
              through its length plan: real entries only)
  blocks4x4   500,000 block rows x 8 dense 4x4 blocks (2,000,000 rows, 64M nnz):  BELL, SBELL, BCSR

The merge-path, CSR-vector and CSR-scalar kernels (the last two are the
reference's CSR drivers' mappings) and SELL read slot by slot, padding
included (the reference's SELL kernel's reads), are timed separately and
reported under "variants".

value = sum of useful flops (2 nnz per SpMV) / sum of kernel times, GFLOP/s.
Kernel times are CUDA events on the launching stream; every matrix is larger
than the 126 MB L2 and the formats run back to back, so no explicit flush.

After timing, every format's y is computed once more at full size and
compared per row with the reference's csr_spmv (|y - y_ref| <= 1e-5
sum|a x|, the check the reference prints after each variant's first launch,
src/util.cpp:93-131) and with the FP64 oracle ("parity" in the line).

Output: one JSON line per detail block ("detail": ...), then the headline
line last (compact, parsed by callers from the last line of stdout).

--impl reference: the reference's own serial csr_spmv (include/spmv_serial.h
:198-217, compiled from its sources into oracle/_ref; the C restatement in
oracle/ where that build is absent) on all host threads over row blocks, on
the same matrices; this arm never loads libclspmv_b200.so.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "SpMV GFLOP/s (per-format FP32 sweep)"
UNIT = "GFLOP/s"
FALLBACK_HBM_GBS = 6650.0
RTOL = 1e-5   # per-row bound: |y - y_ref| <= RTOL * sum_j |a_ij x_j|


def parse_args():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=200)
    p.add_argument("--warmup", type=int, default=5)
    p.add_argument("--impl", choices=["ours", "reference"], default="ours")
    p.add_argument("--small", action="store_true", help="scaled-down matrices (quick check)")
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--only", default="", help="comma list of format keys to run (debugging)")
    p.add_argument("--no-extras", action="store_true",
                   help="skip the several-right-hand-side, batched and serving measurements")
    p.add_argument("--serving-requests", type=int, default=4000)
    p.add_argument("--detail-file", default="",
                   help="also write every measurement (per format, variants, parity, extras) to this JSON file")
    return p.parse_args()


# ---------------------------------------------------------------------------
# Workload
# ---------------------------------------------------------------------------
def hyb_width(lengths: np.ndarray) -> int:
    """ELL width of the ELL+COO split: the largest K such that at least a
    third of the rows (and at least 4096) have K or more nonzeros."""
    need = max(4096, len(lengths) // 3)
    hist = np.bincount(lengths)
    at_least = np.cumsum(hist[::-1])[::-1]
    ks = np.nonzero(at_least >= need)[0]
    return int(max(1, ks.max())) if ks.size else 1


def split_hyb(coo_arrays, k):
    """Rows' first k entries -> ELL part, the rest -> COO tail (both sorted)."""
    h, w, r, c, v = coo_arrays
    start = np.searchsorted(r, r, side="left")
    pos = np.arange(r.size) - start
    head = pos < k
    return (h, w, r[head], c[head], v[head]), (h, w, r[~head], c[~head], v[~head])


VARIANT_KEYS = {"csr_merge", "csr_vector", "csr_scalar", "sell32_padded"}
FORMAT_KEYS = {"stencil27": ["dia", "bdia"],
               "powerlaw": ["csr_chunk", "csr_merge", "csr_vector", "csr_scalar", "coo", "ell", "ell_tail_coo", "sell32", "sell32_padded"],
               "blocks4x4": ["bell", "sbell", "bcsr"]}


def build_workload(small: bool, only=None):
    """Host matrices of the sweep; `only` restricts it to some format keys
    (and builds only the matrices they need)."""
    from clspmv_mic_b200 import formats as F

    want = set(only) if only else {k for ks in FORMAT_KEYS.values() for k in ks}
    if "ell" in want or "ell_tail_coo" in want:
        want |= {"ell", "ell_tail_coo"}
    mats = {name: arrs for name, arrs in sweep_matrices(small, [n for n in FORMAT_KEYS if want & set(FORMAT_KEYS[n])]).items()}
    items = []
    meta = {"ell_width": None}

    def add(key, mat, make, kw=None, part_of=None, conv=None):
        """conv = (source COO arrays, format, converter arguments): how the
        host matrix was converted, for the device-conversion comparison."""
        if key not in want:
            return
        t0 = time.perf_counter()
        host = make()
        host_s = time.perf_counter() - t0
        h, w = mats[mat][0], mats[mat][1]
        items.append(dict(key=key, matrix=mat, host=host, kw=kw or {}, rows=h, cols=w, nnz=int(host.nnz),
                          stored=host.stored_bytes(), part_of=part_of, conv=conv,
                          host_convert_s=host_s if conv else None))

    def once(make):
        box = []
        return lambda: box[0] if box else (box.append(make()) or box[0])

    if "stencil27" in mats:
        st = mats["stencil27"]
        coo = F.coo_matrix(*st)
        add("dia", "stencil27", lambda: F.coo2dia(coo), conv=(st, "dia", ()))
        add("bdia", "stencil27", lambda: F.coo2bdia(coo), conv=(st, "bdia", ()))
    if "powerlaw" in mats:
        pl = mats["powerlaw"]
        coo = F.coo_matrix(*pl)
        csr = once(lambda: F.coo2csr(coo))
        add("csr_chunk", "powerlaw", csr, {"variant": "chunk"}, conv=(pl, "csr", ()))
        add("csr_merge", "powerlaw", csr, {"variant": "merge"})
        add("csr_vector", "powerlaw", csr, {"variant": "vector"})
        add("csr_scalar", "powerlaw", csr, {"variant": "scalar"})
        add("coo", "powerlaw", lambda: coo)
        if "ell" in want:
            k = hyb_width(np.diff(csr().array("csr_row_ptr")))
            meta["ell_width"] = k
            ell_part, coo_tail = split_hyb(pl, k)
            add("ell", "powerlaw", lambda: F.coo2ell(F.coo_matrix(*ell_part), 32, k), part_of="ell",
                conv=(ell_part, "ell", (32, k)))
            add("ell_tail_coo", "powerlaw", lambda: F.coo_matrix(*coo_tail), part_of="ell")
        sell = once(lambda: F.coo2sell(coo, 32))
        # with its length plan (real entries only, tails' column ids compact), and every stored slot
        add("sell32", "powerlaw", sell, {"variant": "planned"}, conv=(pl, "sell", (32,)))
        add("sell32_padded", "powerlaw", sell)
    if "blocks4x4" in mats:
        bl = mats["blocks4x4"]
        coo = F.coo_matrix(*bl)
        add("bell", "blocks4x4", lambda: F.coo2b4ell(coo, 4, 4), conv=(bl, "b4ell", (4, 4)))
        add("sbell", "blocks4x4", lambda: F.coo2sbell(coo, 4, 4, 32), conv=(bl, "sbell", (4, 4, 32)))
        add("bcsr", "blocks4x4", lambda: F.coo2b4csr(coo, 4, 4), conv=(bl, "b4csr", (4, 4)))
    return mats, items, meta


def algorithmic_bytes(it) -> int:
    """Arrays the kernel must stream (values, indices, pointers, padding),
    plus x read once and y read and written once. SELL with its length plan
    reads, of each slice column, only the 128-byte lines holding real
    entries (B200 moves whole lines between DRAM and L2), the tails' column
    ids from the plan's compact copy, the plan's arrays and the slice
    pointers."""
    if it.get("needed") is not None:
        return int(it["needed"] + 4 * it["cols"] + 8 * it["rows"])
    return int(it["stored"] + 4 * it["cols"] + 8 * it["rows"])


def format_flops(it) -> int:
    return 2 * it["nnz"]


# ---------------------------------------------------------------------------
# Clocks
# ---------------------------------------------------------------------------
class ClockSampler:
    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index: int):
        self.dev = device_index
        self.proc = None
        self.path = Path(os.environ.get("TMPDIR", "/tmp")) / f"clspmv_clocks_{os.getpid()}.csv"

    def start(self):
        try:
            self.fh = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.dev}", f"--query-gpu={self.QUERY}",
                                          "--format=csv,noheader,nounits", "-lms", "50"],
                                         stdout=self.fh, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.fh.close()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.path.read_text().splitlines():
            f = [t.strip() for t in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax.append(float(f[2]))
            except ValueError:
                continue
            for n, val in zip(names, f[5:9]):
                if val.lower() == "active":
                    reasons.add(n)
        try:
            self.path.unlink()
        except OSError:
            pass
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def hbm_peak():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        try:
            return float(json.loads(p.read_text())["hbm_gbs"]), "measured"
        except Exception:
            pass
    return FALLBACK_HBM_GBS, "fallback"


def ncu_traffic():
    """Per-launch DRAM bytes from committed ncu summaries
    (profiles/ncu_traffic.txt: `<format key> <bytes per launch> ...`)."""
    out = {}
    p = ROOT / "profiles" / "ncu_traffic.txt"
    if p.exists():
        for line in p.read_text().splitlines():
            t = line.split()
            if len(t) >= 2 and not line.startswith("#"):
                try:
                    out[t[0]] = float(t[1])
                except ValueError:
                    pass
    return out


# ---------------------------------------------------------------------------
# CPU leg: the reference's serial csr_spmv, timed as the baseline and used
# as the checker of every format's y
# ---------------------------------------------------------------------------
def host_threads() -> int:
    return max(1, len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else (os.cpu_count() or 1))


def ref_csr(arrs):
    """Host CSR of a generated COO built by the reference's own coo2csr
    (include/matrix_storage.h:1268-1307, compiled into oracle/_ref); the C
    restatement's arrays where that build is absent. Touches nothing of
    libclspmv_b200.so."""
    from clspmv_mic_b200 import formats as F
    from oracle import oracle as O
    coo = F.coo_matrix(*arrs)
    if O.ref() is not None:
        ok, csr = O.ref_convert("csr", coo)
        assert ok
        return csr
    h, w, r, c, v = arrs
    rp = np.zeros(h + 1, np.int64)
    np.add.at(rp, r.astype(np.int64) + 1, 1)
    return F.from_arrays("csr", dict(width=w, height=h, nnz=r.size),
                         dict(csr_row_ptr=np.cumsum(rp).astype(np.int32), csr_col_id=c, csr_data=v))


def row_blocks(csr, parts: int):
    """(r0, r1, slab) row blocks of a host CSR matrix with about nnz / parts
    nonzeros each; each slab is a CSR view of rows [r0, r1) (its row
    pointer rebased, col_id / data sliced), for the host threads."""
    from clspmv_mic_b200 import formats as F
    rp, col, val = csr.array("csr_row_ptr"), csr.array("csr_col_id"), csr.array("csr_data")
    h, w = csr.shape
    cuts = [0] + [int(np.searchsorted(rp, csr.nnz * t / parts)) for t in range(1, parts)] + [h]
    out = []
    for t in range(parts):
        r0, r1 = cuts[t], max(cuts[t], cuts[t + 1])
        if r1 <= r0:
            continue
        lo, hi = int(rp[r0]), int(rp[r1])
        out.append((r0, r1, F.from_arrays("csr", dict(width=w, height=r1 - r0, nnz=hi - lo),
                                          dict(csr_row_ptr=(rp[r0:r1 + 1] - lo).astype(np.int32),
                                               csr_col_id=col[lo:hi], csr_data=val[lo:hi]))))
    return out


def csr_spmv_call():
    """(call(csr, x, y), kind): the reference's csr_spmv compiled from its
    sources, else the C restatement."""
    import ctypes as C
    from oracle import oracle as O
    if O.ref() is not None:
        return (lambda m, x, y: O.ref().ref_csr_spmv(C.byref(m.struct), x.ctypes.data, y.ctypes.data, x.size)), \
            "reference"
    return (lambda m, x, y: O.port().orc_csr_spmv_f32(C.byref(m.struct), x.ctypes.data, y.ctypes.data)), "port"


class Oracle:
    """y = A x of one matrix by the reference's csr_spmv (FP32, each row
    summed left to right as written) and by the FP64 oracle with the row
    scale sum_j |a_ij x_j|, each on all host threads over row blocks (rows
    are independent, so the blocks give the one-thread result bit for bit)."""

    def __init__(self, csr, x, pool, threads):
        import ctypes as C
        from oracle import oracle as O
        h = csr.shape[0]
        call, _ = csr_spmv_call()
        self.y32 = np.zeros(h, np.float32)
        self.y64 = np.zeros(h, np.float64)
        self.scale = np.zeros(h, np.float64)
        blocks = row_blocks(csr, threads)
        L = O.port()

        def one(b):
            r0, r1, slab = b
            call(slab, x, self.y32[r0:r1])
            L.orc_csr_spmv_f64(C.byref(slab.struct), x.ctypes.data, self.y64[r0:r1].ctypes.data,
                               self.scale[r0:r1].ctypes.data)
        list(pool.map(one, blocks))

    def check(self, y):
        """rows over the bound |y - y_ref| <= 1e-5 sum|a x|, and the largest
        |y - y64| / sum|a x|."""
        y = y.astype(np.float64)
        err = np.abs(y - self.y32.astype(np.float64))
        over = int(np.count_nonzero(err > RTOL * self.scale + 1e-30))
        with np.errstate(divide="ignore", invalid="ignore"):
            e64 = np.abs(y - self.y64) / np.where(self.scale > 0, self.scale, 1.0)
        return over, float(e64.max()) if e64.size else 0.0

    def ref_err64(self):
        with np.errstate(divide="ignore", invalid="ignore"):
            e = np.abs(self.y32.astype(np.float64) - self.y64) / np.where(self.scale > 0, self.scale, 1.0)
        return float(e.max()) if e.size else 0.0


def cpu_csr_seconds(csrs, xs, budget_s: float = 15.0):
    """Best-of-k one-thread csr_spmv per matrix (the reference's serial path
    as written). Returns (sum of best times, flops, kind, sample text)."""
    call, kind = csr_spmv_call()
    total_t, total_f, desc = 0.0, 0, []
    per = budget_s / len(csrs)
    for name, csr in csrs.items():
        x = xs[name]
        best, n, t_start = float("inf"), 0, time.perf_counter()
        while n < 3 or (time.perf_counter() - t_start < per and n < 50):
            y = np.zeros(csr.shape[0], np.float32)
            t0 = time.perf_counter()
            call(csr, x, y)
            best = min(best, time.perf_counter() - t0)
            n += 1
        total_t += best
        total_f += 2 * csr.nnz
        desc.append(f"{name} best of {n}")
    return total_t, total_f, kind, "csr_spmv on " + ", ".join(desc) + ", 1 thread"


def loaded_native_libs():
    """Shared objects of this repository mapped into the process (from
    /proc/self/maps): the reference arm must map oracle/ libraries only."""
    out = set()
    try:
        for line in Path("/proc/self/maps").read_text().splitlines():
            t = line.split()
            if len(t) >= 6 and t[-1].endswith(".so") and t[-1].startswith(str(ROOT)):
                out.add(os.path.relpath(t[-1], ROOT))
    except OSError:
        pass
    return sorted(out)


# ---------------------------------------------------------------------------
# Arms
# ---------------------------------------------------------------------------
def dist_init(args):
    """One process per GPU under torchrun (NCCL); gloo when CUDA is absent
    (the multi-process logic is tested that way on the CPU)."""
    import torch
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime
        import torch.distributed as dist
        if torch.cuda.is_available():
            torch.cuda.set_device(local)
            dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600),
                                    device_id=torch.device("cuda", local))
        else:
            dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=60))
    return world, rank, local


def max_over_ranks(value: float, device) -> float:
    """The slowest rank's time (replicas are timed on their own devices; the
    job's time is the maximum)."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_value(flops_per_replica_step: float, world: int, ms_per_step: float) -> float:
    """Whole-job GFLOP/s: every replica does the same step, the job takes the
    slowest replica's time."""
    return flops_per_replica_step * world / (ms_per_step * 1e-3) / 1e9


def sweep_matrices(small: bool, names=None):
    """The sweep's three matrices (row-sorted COO tuples from the numpy
    generators), or the named ones."""
    from clspmv_mic_b200 import synth
    gens = {
        "stencil27": (lambda: synth.stencil_27pt(32)) if small else (lambda: synth.stencil_27pt(128)),
        "powerlaw": (lambda: synth.powerlaw(1 << 15, maxlen=2000)) if small else (lambda: synth.powerlaw(1 << 20)),
        "blocks4x4": (lambda: synth.block_rows(8000, 8)) if small else (lambda: synth.block_rows(500_000, 8)),
    }
    return {n: g() for n, g in gens.items() if names is None or n in names}


WORKLOAD = ("nine-format FP32 sweep: stencil27 128^3 -> DIA,BDIA; powerlaw 2^20 Zipf(2.0) mean 16 -> "
            "CSR,COO,ELL(K)+COO tail,SELL-32; 4x4 blocks 500k x 8 -> BELL,SBELL,BCSR")


def run_reference(args):
    """The reference's serial csr_spmv (its own code, compiled from its
    sources into oracle/_ref) on every host thread: each thread runs it on a
    block of rows holding about nnz / threads nonzeros (ctypes releases the
    GIL during the call). Matrices come from the numpy generators and their
    CSR from the reference's coo2csr; libclspmv_b200.so is never loaded."""
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    from concurrent.futures import ThreadPoolExecutor

    from clspmv_mic_b200 import synth
    mats = sweep_matrices(args.small)
    call, kind = csr_spmv_call()
    threads = host_threads()
    prepared, keep = [], []
    for name, arrs in mats.items():
        csr = ref_csr(arrs)
        keep.append(csr)
        h, w = csr.shape
        x = synth.x_vector(arrs[1])
        y = np.zeros(h, np.float32)
        for r0, r1, slab in row_blocks(csr, threads):
            prepared.append((slab, x, y[r0:r1]))
    flops = sum(2 * c.nnz for c in keep)
    pool = ThreadPoolExecutor(threads)

    def step():
        for _, _, y in prepared:
            y.fill(0.0)
        list(pool.map(lambda t: call(*t), prepared))

    for _ in range(max(3, args.warmup)):
        step()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        step()
    dt = (time.perf_counter() - t0) / args.steps
    pool.shutdown()
    value = flops / dt / 1e9
    native = loaded_native_libs()
    if any("clspmv_mic_b200" in n for n in native):
        raise RuntimeError(f"the reference arm mapped this library: {native}")
    line = {
        "metric": METRIC, "value": round(value, 3), "unit": UNIT, "impl": "reference", "n_gpus": world,
        "steps": args.steps, "warmup": max(3, args.warmup), "ms_per_step": round(dt * 1e3, 4),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": "csr_spmv (the reference's serial CPU path) over stencil27 128^3, powerlaw 2^20, "
                               "blocks4x4 500k x 8" + (" (small)" if args.small else ""),
                   "parallelism": f"{threads} host threads, each running csr_spmv on a block of rows with "
                                  "nnz / threads nonzeros"},
        "cpu_baseline": {"value": round(value, 3), "unit": UNIT, "cores": threads, "kind": kind,
                         "sample": f"{args.steps} steps of csr_spmv over the three matrices"},
        "e2e": {"value": round(value, 3), "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "native_libs": native,
    }
    print(json.dumps(line), flush=True)
    return 0


def headline(*, value, world, steps, warmup, ms_per_step, small, roofline, e2e, launches, clocks, cpu_baseline,
             parity, fracs, ell_width, gather_peak):
    """The line the driver parses: compact (well under 2 KB), printed last."""
    return {
        "metric": METRIC, "value": round(value, 2), "unit": UNIT, "n_gpus": world, "steps": steps,
        "warmup": warmup, "ms_per_step": round(ms_per_step, 5), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded generators)",
        "config": {"workload": WORKLOAD + (" (SMALL)" if small else ""), "global_batch": 1,
                   "parallelism": f"replicas x{world}" if world > 1 else "1 GPU",
                   "l2": "no flush: every matrix > 126 MB L2", "ell_width": ell_width},
        "roofline": roofline,
        "e2e": e2e,
        "gpu_launches": int(launches),
        "clocks": {k: clocks.get(k) for k in ("sm_mhz", "sm_max_mhz", "reasons")},
        "cpu_baseline": cpu_baseline,
        "parity": parity,
        "format_frac": fracs,
        "gather_peak_g_per_s": gather_peak,
    }


def run_ours(args):
    import torch
    from concurrent.futures import ThreadPoolExecutor

    from clspmv_mic_b200 import formats as F
    from clspmv_mic_b200 import synth

    world, rank, local = dist_init(args)
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    mats, items, meta = build_workload(args.small, args.only.split(",") if args.only else None)

    stream = torch.cuda.Stream(device=dev)
    xs, ys = {}, {}
    for name, arrs in mats.items():
        xs[name] = torch.from_numpy(synth.x_vector(arrs[1])).to(dev)
    for it in items:
        it["dev"] = F.DeviceMatrix(it["host"], device=dev)
        ys[it["key"]] = torch.zeros(it["rows"], dtype=torch.float32, device=dev)
        if it["host"].fmt == "csr" and it["kw"].get("variant") == "merge":
            it["dev"].merge_plan(stream)
        if it["host"].fmt == "csr" and it["kw"].get("variant") == "chunk":
            it["dev"].chunk_plan(stream)
        if it["host"].fmt == "sell" and it["kw"].get("variant") == "planned":
            # the 128-byte lines holding real entries (a data line per tail
            # entry, the tails' column ids compact), the plan's arrays and
            # the slice pointers
            d = it["dev"]
            it["needed"] = d.sell_plan_line_bytes() + 4 * (it["host"].struct.sell_slice_num + 1)
        it.pop("host")
    torch.cuda.synchronize()

    variants = [it for it in items if it["key"] in VARIANT_KEYS]
    items = [it for it in items if it["key"] not in VARIANT_KEYS]
    if not items:   # --only named variants alone: they form the step
        items, variants = variants, []
    K = len(items)
    ev = [[torch.cuda.Event(enable_timing=True) for _ in range(K + 1)] for _ in range(args.steps)]

    def step(i=None):
        with torch.cuda.stream(stream):
            for j, it in enumerate(items):
                if i is not None:
                    ev[i][j].record(stream)
                it["dev"].spmv(xs[it["matrix"]], ys[it["key"]], 1.0, 1.0, stream=stream, **it["kw"])
            if i is not None:
                ev[i][K].record(stream)

    clocks = ClockSampler(local)
    clocks.start()          # sampling starts before the warm-up so it covers the timed region
    t_warm = time.perf_counter()
    warmup = max(3, args.warmup)
    for _ in range(warmup):
        step()
    torch.cuda.synchronize()
    while time.perf_counter() - t_warm < 0.5:   # keep the GPU busy while nvidia-smi spins up
        step()
        torch.cuda.synchronize()
    if world > 1:
        torch.distributed.barrier()
    launches0 = F.launch_count()
    t_all0 = torch.cuda.Event(enable_timing=True)
    t_all1 = torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    t_all0.record(stream)
    for i in range(args.steps):
        step(i)
    t_all1.record(stream)
    torch.cuda.synchronize()
    launches = F.launch_count() - launches0
    total_ms = t_all0.elapsed_time(t_all1)
    per_kernel_ms = np.array([[ev[i][j].elapsed_time(ev[i][j + 1]) for j in range(K)] for i in range(args.steps)])
    clk = clocks.stop()
    if world > 1:
        total_ms = max_over_ranks(total_ms, dev)
        torch.distributed.barrier()

    # e2e through the public API with host buffers: per kernel, pinned x
    # copied in and y read back, inside the timed region. The copies run on
    # their own streams (one per direction), so while one SpMV runs, the next
    # x is uploading and the previous y downloading: both copy engines and the
    # SMs work at once, as a caller issuing the step's SpMVs would arrange.
    h2d = d2h = 0
    hx = {name: torch.from_numpy(synth.x_vector(a[1])).pin_memory() for name, a in mats.items()}
    hy = {it["key"]: torch.zeros(it["rows"], dtype=torch.float32).pin_memory() for it in items}
    dx = {it["key"]: torch.empty(it["cols"], dtype=torch.float32, device=dev) for it in items}
    for it in items:
        h2d += 4 * it["cols"]
        d2h += 4 * it["rows"]
    up, down = torch.cuda.Stream(device=dev), torch.cuda.Stream(device=dev)
    x_in = {it["key"]: torch.cuda.Event() for it in items}      # x of this step is on the device
    done = {it["key"]: torch.cuda.Event() for it in items}      # the SpMV has run (x free, y ready)
    y_out = {it["key"]: torch.cuda.Event() for it in items}     # y has left for the host (y free)

    def e2e_step():
        for it in items:
            k = it["key"]
            up.wait_event(done[k])                  # the previous step's SpMV no longer reads dx
            with torch.cuda.stream(up):
                dx[k].copy_(hx[it["matrix"]], non_blocking=True)
            x_in[k].record(up)
            stream.wait_event(x_in[k])
            stream.wait_event(y_out[k])             # the previous step's y has been read
            it["dev"].spmv(dx[k], ys[k], 1.0, 1.0, stream=stream, **it["kw"])
            done[k].record(stream)
            down.wait_event(done[k])
            with torch.cuda.stream(down):
                hy[k].copy_(ys[k], non_blocking=True)
            y_out[k].record(down)

    for _ in range(3):
        e2e_step()
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    up.wait_stream(stream)
    down.wait_stream(stream)
    for _ in range(args.steps):
        e2e_step()
    stream.wait_stream(up)
    stream.wait_stream(down)
    e1.record(stream)
    torch.cuda.synchronize()
    e2e_ms = e0.elapsed_time(e1) / args.steps
    if world > 1:
        e2e_ms = max_over_ranks(e2e_ms, dev)
    del hx, hy, dx

    # the ELL part and its COO tail together carry the matrix's flops once
    flops_step = sum(format_flops(it) for it in items if it["part_of"] is None) + \
        sum(format_flops(it) for it in items if it["part_of"] == "ell")
    ms_per_step = total_ms / args.steps
    value = job_value(flops_step, world, ms_per_step)
    e2e_value = job_value(flops_step, world, e2e_ms)

    peak, peak_kind = hbm_peak()
    # the scattered-column formats are bound by random x gathers, not bytes:
    # measure that ceiling on the power-law matrix's x length
    gather_peak = None
    if "powerlaw" in mats:
        from clspmv_mic_b200.drivers import gather_test
        gather_peak = gather_test(int(mats["powerlaw"][1]), 1 << 24, 20)
    med = np.median(per_kernel_ms, axis=0)
    mean = per_kernel_ms.mean(axis=0)
    formats = {}
    for j, it in enumerate(items):
        ab = algorithmic_bytes(it)
        useful = 12 * it["nnz"] + 4 * it["cols"] + 8 * it["rows"]
        formats[it["key"]] = {
            "matrix": it["matrix"], "ms": round(float(med[j]), 5), "gflops": round(format_flops(it) / (med[j] * 1e-3) / 1e9, 2),
            "gbs": round(ab / (med[j] * 1e-3) / 1e9, 1), "frac": round(ab / (med[j] * 1e-3) / 1e9 / peak, 3),
            # COO-equivalent bytes (12 nnz + x + y) over the time: above 1 where the format moves fewer
            # bytes than COO would (no per-entry indices), far below where it streams padding
            "frac_coo_equiv": round(useful / (med[j] * 1e-3) / 1e9 / peak, 3),
            "alg_bytes": ab, "useful_bytes": useful, "nnz": it["nnz"], "rows": it["rows"],
        }
        if gather_peak and it["matrix"] == "powerlaw":
            g = it["nnz"] / (med[j] * 1e-3)
            formats[it["key"]].update(gathers_per_s=round(g / 1e9, 1), gather_frac=round(g / gather_peak, 3))
    # the CSR-vector / CSR-scalar / merge-path / planned-SELL variants, outside the timed step
    variant_stats = {}
    for it in variants:
        with torch.cuda.stream(stream):
            for _ in range(3):
                it["dev"].spmv(xs[it["matrix"]], ys[it["key"]], 1.0, 1.0, stream=stream, **it["kw"])
            v0 = torch.cuda.Event(enable_timing=True)
            v1 = torch.cuda.Event(enable_timing=True)
            reps = max(3, min(10, args.steps))
            v0.record(stream)
            for _ in range(reps):
                it["dev"].spmv(xs[it["matrix"]], ys[it["key"]], 1.0, 1.0, stream=stream, **it["kw"])
            v1.record(stream)
        torch.cuda.synchronize()
        ms = v0.elapsed_time(v1) / reps
        ab = algorithmic_bytes(it)
        if gather_peak and it["matrix"] == "powerlaw":
            g = it["nnz"] / (ms * 1e-3)
            gextra = {"gathers_per_s": round(g / 1e9, 1), "gather_frac": round(g / gather_peak, 3)}
        else:
            gextra = {}
        variant_stats[it["key"]] = {**gextra, "matrix": it["matrix"], "ms": round(ms, 5),
                                    "gflops": round(format_flops(it) / (ms * 1e-3) / 1e9, 2),
                                    "gbs": round(ab / (ms * 1e-3) / 1e9, 1), "frac": round(ab / (ms * 1e-3) / 1e9 / peak, 3)}
    dom = int(np.argmax(mean))
    dom_it = items[dom]
    ab = algorithmic_bytes(dom_it)
    achieved = ab / (mean[dom] * 1e-3) / 1e9
    useful_dom = 12 * dom_it["nnz"] + 4 * dom_it["cols"] + 8 * dom_it["rows"]
    fr = {k: v["frac"] for k, v in formats.items()}
    min_key = min(fr, key=fr.get)
    roofline = {"bound": "hbm", "kernel": dom_it["key"], "achieved": round(achieved, 1), "peak": peak,
                "peak_kind": peak_kind, "unit": "GB/s", "frac": round(achieved / peak, 3),
                "frac_useful": round(useful_dom / (mean[dom] * 1e-3) / 1e9 / peak, 3),
                "min_frac": fr[min_key], "min_frac_kernel": min_key,
                "traffic": ncu_traffic().get(dom_it["key"]), "alg_bytes_per_launch": ab,
                "share_of_step": round(float(mean[dom] / mean.sum()), 3)}
    e2e = {"value": round(e2e_value, 2), "unit": UNIT, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
           "ms_per_step": round(e2e_ms, 4)}

    # CPU leg (rank 0 at N=1): the reference's csr_spmv as the baseline,
    # and every format's y at full size against it and the FP64 oracle
    cpu_baseline = None
    parity = None
    detail = {"formats": formats, "variants": variant_stats}
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        csrs = {name: ref_csr(arrs) for name, arrs in mats.items()}
        xh = {name: synth.x_vector(arrs[1]) for name, arrs in mats.items()}
        t_cpu, f_cpu, kind, sample = cpu_csr_seconds(csrs, xh)
        cpu_baseline = {"value": round(f_cpu / t_cpu / 1e9, 3), "unit": UNIT, "cores": 1, "kind": kind,
                        "sample": sample}
        threads = host_threads()
        with ThreadPoolExecutor(threads) as pool:
            oracles = {name: Oracle(csrs[name], xh[name], pool, threads) for name in mats}
        parity, detail["parity"] = check_parity(items + variants, xs, oracles, stream)
        del csrs, oracles

    if not args.no_extras and not args.only:
        # every rank takes part (one all-gather per step)
        detail["sharded_akx"] = run_sharded_akx(world, dev)
        if rank == 0:
            print(json.dumps({"detail": "sharded_akx", **detail["sharded_akx"]}), flush=True)
        detail["sharded_serving"] = run_sharded_serving(world, rank, dev)
        if rank == 0:
            print(json.dumps({"detail": "sharded_serving", **detail["sharded_serving"]}), flush=True)
    if not args.no_extras and not args.only and world == 1:
        for name, fn in (("extras", lambda: run_extras(args, items, mats, peak)),
                         ("cocktail_c3", lambda: run_cocktail_c3(args, peak)),
                         ("iterate_c1", run_iterate_c1)):
            detail[name] = fn()
            if rank == 0:
                print(json.dumps({"detail": name, **detail[name]}), flush=True)
    line = headline(value=value, world=world, steps=args.steps, warmup=warmup, ms_per_step=ms_per_step,
                    small=args.small, roofline=roofline, e2e=e2e, launches=launches, clocks=clk,
                    cpu_baseline=cpu_baseline, parity=parity, fracs=fr, ell_width=meta["ell_width"],
                    gather_peak=None if gather_peak is None else round(gather_peak / 1e9, 1))
    if rank == 0:
        print(json.dumps({"detail": "formats", "formats": formats, "variants": variant_stats,
                          "parity": detail.get("parity"), "clocks": clk}), flush=True)
        if args.detail_file:
            Path(args.detail_file).parent.mkdir(parents=True, exist_ok=True)
            Path(args.detail_file).write_text(json.dumps({"headline": line, **detail}, indent=1))
        print(json.dumps(line), flush=True)
    if world > 1:
        torch.distributed.destroy_process_group()
    return 0


def check_parity(items, xs, oracles, stream):
    """Every format's y = A x at full size (beta = 0; the ELL part and its
    COO tail accumulate into one y) against the reference's csr_spmv within
    the per-row bound 1e-5 sum|a x|, and its error against the FP64 oracle.
    Returns (summary for the headline, per-format detail)."""
    import torch
    per = {}
    groups = {}
    for it in items:
        groups.setdefault(it["part_of"] or it["key"], []).append(it)
    for key, parts in groups.items():
        m = parts[0]["matrix"]
        y = torch.zeros(parts[0]["rows"], dtype=torch.float32, device=xs[m].device)
        with torch.cuda.stream(stream):
            for j, it in enumerate(parts):
                it["dev"].spmv(xs[m], y, 1.0, 0.0 if j == 0 else 1.0, stream=stream, **it["kw"])
        torch.cuda.synchronize()
        over, e64 = oracles[m].check(y.cpu().numpy())
        per[key] = {"matrix": m, "rows_over_bound": over, "max_err_fp64": e64}
    summary = {"checked": sorted(per), "rows_over_bound": int(sum(v["rows_over_bound"] for v in per.values())),
               "max_err_fp64": max((v["max_err_fp64"] for v in per.values()), default=0.0),
               "ref_err_fp64": max(o.ref_err64() for o in oracles.values()),
               "bound": "per row |y-y_ref| <= 1e-5 sum|a x|, full size"}
    summary["max_err_fp64"] = float(f"{summary['max_err_fp64']:.3g}")
    summary["ref_err_fp64"] = float(f"{summary['ref_err_fp64']:.3g}")
    return summary, per


def run_sharded_akx(world: int, dev, n: int = 128, steps: int = 40):
    """The reference's A^k x loop (src/eval.cpp:19-72) on the 27-point
    stencil 128^3 with its rows split evenly over the ranks: each rank builds
    its own rows only, and a step is the rank's SpMV (CSR by nonzero chunks)
    plus one all-gather of every rank's y block into x (NCCL over NVLink /
    NVSwitch; a device copy at one rank). Time per step: CUDA events around
    `steps` steps, the slowest rank's."""
    import torch
    import torch.distributed as dist
    from clspmv_mic_b200 import sharded as S
    from clspmv_mic_b200 import synth
    m = n ** 3
    s = S.ShardedCsr(None, device=dev, n=m, make_rows=lambda r0, r1: synth.stencil_27pt_rows(n, r0, r1))
    rng = np.random.default_rng(5)
    s.load(rng.uniform(-1, 1, m).astype(np.float32), np.zeros(m, np.float32))
    alpha = 1.0 / 32.0   # |row sums| <= 27: x stays bounded over the steps
    nnz = torch.tensor([s.nnz], dtype=torch.float64, device=dev)
    if world > 1:
        dist.all_reduce(nnz)
    s.iterate(3, alpha, 0.0)
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    s.iterate(steps, alpha, 0.0)
    e1.record()
    torch.cuda.synchronize()
    ms = max_over_ranks(e0.elapsed_time(e1) / steps, dev)
    total = float(nnz.item())
    finite = bool(torch.isfinite(s.x).all().item())
    return {"matrix": f"stencil27 {n}^3", "rows": m, "nnz": int(total), "world": world, "steps": steps,
            "ms_per_step": round(ms, 4), "gflops": round(2 * total / (ms * 1e-3) / 1e9, 1),
            "gather_bytes_per_step": 4 * s.block * world, "x_finite": finite,
            "note": "rows split evenly, each rank's slab built from its own rows; one all_gather_into_tensor per step"}


def run_sharded_serving(world: int, rank: int, dev, n_requests: int = 3000, rate: float = 30_000.0):
    """Serving across the node's GPUs as independent units: 16 matrices
    (banded, power-law, 4x4 blocks; 0.5-3M nonzeros) placed whole by
    serving.place over the ranks' equal budgets, one Poisson stream of
    requests (k uniform in [1, 8]) of which each rank serves those of its own
    matrices on its own GPU (serving.ShardedServer on that device), at the
    stream's arrival times. No data crosses between GPUs. Whole-job req/s =
    all requests over the slowest rank's span; p50 / p99 from rank 0."""
    import torch
    import torch.distributed as dist
    from clspmv_mic_b200 import serving as SV
    from clspmv_mic_b200 import workloads as W
    hosts = W.sharded_serving_hosts()
    budget = 16 << 30
    assign = SV.place({i: SV.resident_bytes(h) for i, (_, h) in enumerate(hosts)}, [budget] * world)
    owned = [i for i, r in assign.items() if r == rank]
    if world > 1:
        dist.barrier()
    res = W.serve_sharded(hosts, [dev], budget, n_requests=n_requests, rate=rate, owned=owned)
    span = torch.tensor([res.get("span_s", 0.0)], dtype=torch.float64, device=dev)
    count = torch.tensor([float(res["requests"])], dtype=torch.float64, device=dev)
    if world > 1:
        dist.all_reduce(span, op=dist.ReduceOp.MAX)
        dist.all_reduce(count)
    total = float(count.item())
    return {"ranks": world, "matrices": len(hosts), "requests": int(total), "offered_req_per_s": rate, "k": [1, 8],
            "req_per_s": round(total / float(span.item()), 1) if span.item() > 0 else None,
            "rank0": {k: res[k] for k in ("matrices", "requests", "served", "standalone", "allocator") if k in res},
            "note": "matrices placed whole (serving.place), each rank serves its own on its GPU; "
                    "req/s = all requests / slowest rank's span"}


def run_device_convert(items):
    """Each sweep matrix converted again on the device from its COO
    (clspmv_device_coo2<fmt>_f32, COO already resident) against the host
    converter that built it: seconds, and the converted arrays compared bit
    for bit with the uploaded host result."""
    import torch
    from clspmv_mic_b200 import formats as F
    res = {}
    coos = {}
    for it in items:
        if not it.get("conv"):
            continue
        src, fmt, cargs = it["conv"]
        key = id(src)
        if key not in coos:
            coos.clear()
            torch.cuda.empty_cache()
            coos[key] = F.DeviceMatrix(F.coo_matrix(*src))
        dcoo = coos[key]
        times = []
        for _ in range(2):   # the first call also warms the allocator and the sort's scratch sizes
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            m = F.device_convert(dcoo, fmt, *cargs)
            torch.cuda.synchronize()
            times.append(time.perf_counter() - t0)
            if len(times) < 2:
                del m
        ref = it["dev"].tensors
        equal = all(torch.equal(m.tensors[f].view(torch.int32), ref[f].view(torch.int32)) for f in m.tensors)
        dev_s = min(times)
        res[it["key"]] = {"format": fmt, "args": list(cargs), "nnz": int(dcoo.nnz), "host_s": round(it["host_convert_s"], 3),
                          "device_s": round(dev_s, 4), "speedup": round(it["host_convert_s"] / dev_s, 1),
                          "equal_to_host": bool(equal)}
        del m
    coos.clear()
    torch.cuda.empty_cache()
    return {"note": "host_s = the library's host converter (one core) that built the sweep's matrix; device_s = "
                    "clspmv_device_coo2<fmt>_f32 from a resident device COO incl. output allocation, best of 2; "
                    "equal_to_host = every array identical bit for bit", "results": res}


def run_extras(args, items, mats, peak):
    """Several right-hand sides with FP32 / BF16 / FP16 values on the sweep's
    matrices, 256 uneven matrices as one batched launch, and the serving
    loop against sequential launches (Poisson arrivals)."""
    import torch
    from clspmv_mic_b200 import formats as F
    from clspmv_mic_b200 import workloads as W
    out = {"device_convert": run_device_convert(items)}
    t0 = time.perf_counter()
    by_key = {it["key"]: it for it in items}
    csr64 = {}
    for name, arrs in mats.items():
        csr_dev = by_key["csr_chunk"]["dev"] if name == "powerlaw" else F.DeviceMatrix(F.coo2csr(F.coo_matrix(*arrs)))
        csr64[name] = W.fp64_of_csr(csr_dev)
        del csr_dev
    # single-vector SpMV with 16-bit values in each format's own kernel
    spmv16 = {}
    gen = torch.Generator(device="cuda")
    gen.manual_seed(11)
    for key in ("dia", "bdia", "csr_chunk", "coo", "sell32", "bell", "sbell", "bcsr"):
        if key not in by_key:
            continue
        it = by_key[key]
        m = it["dev"]
        x = torch.rand(it["cols"], generator=gen, device="cuda") * 2 - 1
        y = torch.zeros(it["rows"], device="cuda")
        for vt in ("bf16", "f16"):
            p = m.pack(vt)
            m.spmv(x, y, 1.0, 0.0, packed=p, **it["kw"])
            err = csr64[it["matrix"]].error(x[:, None], y[:, None])
            for _ in range(3):
                m.spmv(x, y, 1.0, 0.0, packed=p, **it["kw"])
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            for _ in range(20):
                m.spmv(x, y, 1.0, 0.0, packed=p, **it["kw"])
            e1.record()
            torch.cuda.synchronize()
            ms = e0.elapsed_time(e1) / 20
            res = {"ms": round(ms, 5), "gflops": round(2 * it["nnz"] / (ms * 1e-3) / 1e9, 1), "err_fp64": err}
            if it["kw"].get("variant") != "planned":   # SELL through its plan reads less than its stored bytes
                ab = W.matrix_bytes(m, vt) + 4 * it["cols"] + 8 * it["rows"]
                res.update(gbs=round(ab / (ms * 1e-3) / 1e9, 1), frac=round(ab / (ms * 1e-3) / 1e9 / peak, 3), alg_bytes=ab)
            spmv16[f"{key}/{vt}"] = res
            del p
    out["spmv16"] = {"note": "y = A x with values stored as BF16 / FP16 (per-row power-of-two scale, FP32 "
                             "accumulation) in each format's own kernel (SELL-32 through its plan, as in the sweep); "
                             "GB/s over the stored bytes at 2-byte values (none for the planned SELL, which reads less)",
                     "results": spmv16}
    entries = [(k, by_key[k]["dev"], csr64[by_key[k]["matrix"]]) for k in ("dia", "csr_chunk", "bcsr", "sbell")
               if k in by_key]
    out["spmm"] = {"note": "Y = A X, beta 0; GB/s over matrix bytes at the stored value width + k (4n + 4m); "
                           "err_fp64 = max |Y - Y64| / (|A| |X|); CUDA-core kernels",
                   "results": W.spmm_sweep(entries, hbm_gbs=peak)}
    if "bcsr" in by_key:
        out["spmm_tc"] = {"note": "b4csr 4x4 blocks (500k block rows x 8), Y = A X: tcgen05 kind::tf32 with a "
                                  "head/remainder split of A and X (FP32 accuracy) against the CUDA-core kernel",
                          "results": W.spmm_tc_sweep(by_key["bcsr"]["dev"], csr64[by_key["bcsr"]["matrix"]],
                                                     hbm_gbs=peak)}
    del csr64, entries
    torch.cuda.empty_cache()
    out["spmm"]["seconds"] = round(time.perf_counter() - t0, 1)

    t0 = time.perf_counter()
    mats256 = W.uneven_matrices(256, tuned=True, check=8)
    out["batched"] = {"config": "256 matrices, rows log-uniform [1k, 500k], 5-64 nnz/row, banded/blocked/random "
                                "(generated on the device), each stored in the fastest layout for its structure "
                                "(banded: DIA/ELL/CSR, blocked: SBELL/BCSR/BELL 4x4/CSR, random: CSR; converted on "
                                "the device); one persistent launch replayed from a CUDA graph vs one plain launch "
                                "per matrix; err_fp64 over every row of the first 8 matrices",
                      "nnz_total": int(sum(e[1].nnz for e in mats256)),
                      "layouts": W.layout_counts(mats256),
                      "results": W.batched(mats256)}
    del mats256
    torch.cuda.empty_cache()
    out["batched"]["seconds"] = round(time.perf_counter() - t0, 1)

    t0 = time.perf_counter()
    smats = W.serving_matrices(64, tuned=True)
    nnz = int(sum(m.nnz for m in smats))
    budget = 120 * 10 ** 9
    n = args.serving_requests
    out["serving"] = {"config": f"64 resident matrices (rows 10k-4M, 20M-200M nnz, {nnz} nnz in all), each in the "
                                f"fastest layout for its structure, 120 GB budget, Poisson arrivals, sequential = one "
                                f"plain launch + sync per request; long enough streams for tens of batches",
                      "layouts": W.layout_counts([(getattr(m, "structure", "?"), m) for m in smats]),
                      "mixed_k": W.serve(smats, budget, n, rate=20_000.0, k_lo=1, k_hi=32),
                      "k1": W.serve(smats, budget, 3 * n, rate=50_000.0, k_lo=1, k_hi=1),
                      "k1_bf16": W.serve(smats, budget, 3 * n, rate=50_000.0, k_lo=1, k_hi=1, value_type="bf16"),
                      # below the sequential capacity: latency without a queue
                      "mixed_k_light": W.serve(smats, budget, 300, rate=200.0, k_lo=1, k_hi=32)}
    del smats
    torch.cuda.empty_cache()
    out["serving"]["seconds"] = round(time.perf_counter() - t0, 1)
    return out


def run_iterate_c1(steps: int = 480):
    """The reference's A^k x loop (src/eval.cpp:19-72) on the 5-point
    Laplacian of a 256 x 256 grid through the Cocktail runtime, three ways:
    synchronised after every SpMV and every copy (the reference's do_spmv /
    cpy_vector_from_gpu each end in clFinish), stream ordered without host
    waits, and clspmv_cocktail_iterate_f32 (graph-replayed groups of 16
    steps). alpha = 1/8, beta = 0 keeps x bounded (eigenvalues of A/8 in [0, 1])."""
    import torch
    from clspmv_mic_b200 import cocktail as CK
    from clspmv_mic_b200 import formats as F
    from clspmv_mic_b200 import synth
    arrs = synth.laplacian_2d(256)
    coo = F.coo_matrix(*arrs)
    ck = CK.analyze(coo)
    dev = ck.to_device()
    n = coo.shape[0]
    x0 = torch.from_numpy(synth.x_vector(n)).cuda()
    alpha, beta = 0.125, 0.0

    def fresh():
        return x0.clone(), torch.zeros(n, device="cuda")

    x, y = fresh()
    dev.iterate(x, y, 32, alpha, beta)          # captures the graph
    for _ in range(4):
        dev.spmv(x, y, alpha, beta)
        x.copy_(y)
    torch.cuda.synchronize()

    x, y = fresh()
    t0 = time.perf_counter()
    for _ in range(steps):
        dev.spmv(x, y, alpha, beta)
        torch.cuda.synchronize()
        x.copy_(y)
        torch.cuda.synchronize()
    sync_us = (time.perf_counter() - t0) / steps * 1e6

    def timed(fn):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        fn()
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) * 1e3 / steps

    x, y = fresh()

    def loop():
        for _ in range(steps):
            dev.spmv(x, y, alpha, beta)
            x.copy_(y)
    loop_us = timed(loop)
    y_loop = y.clone()
    x, y = fresh()
    graph_us = timed(lambda: dev.iterate(x, y, steps, alpha, beta))
    diff = float((y - y_loop).abs().max() / (y_loop.abs().max() + 1e-30))
    flops = 2 * coo.nnz
    dev.close()
    return {"matrix": "5-point Laplacian 256 x 256", "rows": n, "nnz": int(coo.nnz), "parts": dev.parts,
            "steps": steps, "us_per_step": {"synchronised": round(sync_us, 2), "stream_ordered": round(loop_us, 2),
                                            "graph_iterate": round(graph_us, 2)},
            "gflops_graph": round(flops / (graph_us * 1e-6) / 1e9, 1),
            "speedup_vs_synchronised": round(sync_us / graph_us, 1),
            "max_rel_diff_graph_vs_loop": diff,
            "note": "x (256 KB) and A (3.7 MB) stay in L2: a step is launch-bound, which is what the graph removes"}


def run_cocktail_c3(args, peak):
    """The Cocktail matrix (4M rows: 7-diagonal band 1.5M rows, 4x4 blocks
    1.5M rows, power-law 1M rows): benchmark tables measured on this GPU,
    partitioned by analyze_matrix, the parts run concurrently by the
    Cocktail runtime."""
    import tempfile
    import torch
    from clspmv_mic_b200 import formats as F
    from clspmv_mic_b200 import synth
    from clspmv_mic_b200 import tables as T
    from clspmv_mic_b200 import workloads as W
    out = {}
    t0 = time.perf_counter()
    root = Path(tempfile.mkdtemp(prefix="clspmv_tables_"))
    T.measure_tables(root)
    out["tables_seconds"] = round(time.perf_counter() - t0, 1)
    t0 = time.perf_counter()
    arrs = synth.cocktail_mixed()
    coo = F.coo_matrix(*arrs)
    out["generate_seconds"] = round(time.perf_counter() - t0, 1)
    from clspmv_mic_b200.autotune import tune
    t0 = time.perf_counter()
    res = tune(coo, root, cache=root / "tune.json", use_cache=False)
    mat = res.matrix
    out["tune_seconds"] = round(time.perf_counter() - t0, 1)
    out["tuning"] = {"chosen_knob": res.knob, "candidates": res.report,
                     "part_layouts": res.parts, "ms_before_part_refinement": res.ms_partition,
                     "part_candidates": res.part_report,
                     "note": "each analyze_matrix knob setting of the reference (and the COO part as CSR), partition "
                             "measured with the Cocktail runtime; the first candidate is the reference's default; "
                             "then each SELL / block part re-stored in every slice height / block shape, timed alone, "
                             "the fastest kept when the whole partition gets faster"}
    out["partition"] = mat.summary()
    out["runtime"] = {"chosen": res.runtime, "candidates": res.runtime_report}
    dev = res.to_device()
    h, w = coo.shape
    x = torch.rand(w, device="cuda") * 2 - 1
    y = torch.zeros(h, device="cuda")
    dev.spmv(x, y, 1.0, 0.0)
    csr = F.DeviceMatrix(F.coo2csr(coo))
    band, block = 1_500_000, 1_500_000
    ref = W.Fp64Rows(csr, rows=1 << 15, starts=(0, band, band + block))
    out["err_fp64"] = ref.error(x[:, None], y[:, None])
    del csr, ref
    def timed(schedule, reps=20):
        dev.set_schedule(schedule)
        for _ in range(5):
            dev.spmv(x, y, 1.0, 1.0)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(reps):
            dev.spmv(x, y, 1.0, 1.0)
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / reps

    ms_fused = timed("fused") if dev.fused_items > 0 else None
    ms = timed(res.runtime.get("schedule", "auto"))
    stored = sum(p.stored_bytes() for p in mat.parts().values())
    ab = stored + 4 * w + 8 * h
    out.update(rows=h, nnz=int(coo.nnz), ms=round(ms, 4), gflops=round(2 * coo.nnz / (ms * 1e-3) / 1e9, 1),
               alg_bytes=int(ab), gbs=round(ab / (ms * 1e-3) / 1e9, 1), frac=round(ab / (ms * 1e-3) / 1e9 / peak, 3),
               fused_items=dev.fused_items, ms_fused=None if ms_fused is None else round(ms_fused, 4),
               note="alg bytes = every part's stored arrays + x once + y read and written once; ms = the runtime's "
                    "default schedule (one launch per part), ms_fused = one persistent launch over all parts "
                    "from an interleaved work list")
    dev.close()
    return out


def main():
    args = parse_args()
    if args.impl == "reference":
        return run_reference(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
