"""Measured workloads beyond the single-vector sweep: several right-hand
sides with FP32 / BF16 / FP16 values, batches of uneven matrices in one
persistent launch, and the serving loop against sequential launches.

Accuracy is measured against FP64 on the device: the products and the
per-entry scale sum_j |a_ij x_jc| are formed from the FP64 copy of the
matrix (torch sparse CSR, used here only as the checker), and the reported
error is max |Y - Y64| / scale.
"""
from __future__ import annotations

import gc
import math
import threading
import time

import numpy as np

from .batch import Batch, Job
from .formats import DeviceMatrix
from . import formats as F
from . import synth

VALUE_BYTES = {"f32": 4, "bf16": 2, "f16": 2}


def _events(torch):
    return torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)


class Fp64Rows:
    """Rows of a device CSR matrix kept for the FP64 accuracy check (row of
    each entry, column, FP64 value): the first `rows` rows, or `rows` rows
    from each start in `starts`."""

    def __init__(self, dev_csr: DeviceMatrix, rows: int = 1 << 16, starts=(0,)):
        import torch
        t = dev_csr.tensors
        h = dev_csr.shape[0]
        rp_all = t["csr_row_ptr"].long()
        ids, cols, vals = [], [], []
        sel = []
        for s0 in starts:
            s1 = min(h, s0 + rows)
            if s1 <= s0:
                continue
            rp = rp_all[s0: s1 + 1]
            a, b = int(rp[0].item()), int(rp[-1].item())
            local = torch.repeat_interleave(torch.arange(s1 - s0, device=rp.device), rp[1:] - rp[:-1])
            ids.append(local + len(torch.cat(sel)) if sel else local)
            sel.append(torch.arange(s0, s1, device=rp.device))
            cols.append(t["csr_col_id"][a:b].long())
            vals.append(t["csr_data"][a:b].double())
        self.sel = torch.cat(sel)
        self.rows = int(self.sel.numel())
        self.row_of = torch.cat(ids)
        self.col = torch.cat(cols)
        self.val = torch.cat(vals)

    def error(self, X, Y) -> float:
        """max over the kept rows of |Y - A X| / (|A| |X|), in FP64."""
        import torch
        Xd = X.double()
        k = Xd.shape[1]
        ref = torch.zeros((self.rows, k), dtype=torch.float64, device=Xd.device)
        scale = torch.zeros_like(ref)
        xr = Xd[self.col]
        ref.index_add_(0, self.row_of, self.val[:, None] * xr)
        scale.index_add_(0, self.row_of, (self.val[:, None] * xr).abs())
        err = (Y[self.sel].double() - ref).abs() / scale.clamp_min(1e-300)
        return float(err.max().item()) if err.numel() else 0.0


def fp64_of_csr(dev_csr: DeviceMatrix, rows: int | None = 1 << 16) -> Fp64Rows:
    """FP64 checker of the first `rows` rows (None: every row)."""
    return Fp64Rows(dev_csr, dev_csr.shape[0] if rows is None else rows)


def fp64_error(ref: Fp64Rows, X, Y, rows: int | None = None) -> float:
    return ref.error(X, Y)


def matrix_bytes(m: DeviceMatrix, value_type: str) -> int:
    """Stored bytes of the matrix as the kernel reads it: indices and
    pointers, values at their stored width, plus the row scales of 16-bit
    values."""
    import torch
    vals = {"csr": "csr_data", "dia": "dia_data", "bdia": "bdia_data", "ell": "ell_data", "sell": "sell_data",
            "b4csr": "b4csr_data", "b4ell": "b4ell_data", "sbell": "sbell_data", "coo": "coo_data"}[m.fmt]
    v = m.tensors[vals]
    rest = m.stored_bytes - v.numel() * 4
    extra = 4 * m.shape[0] if value_type != "f32" else 0
    return int(rest + v.numel() * VALUE_BYTES[value_type] + extra)


def spmm_sweep(entries, ks=(1, 4, 16, 32), value_types=("f32", "bf16", "f16"), reps: int = 10, hbm_gbs=None):
    """entries: (key, DeviceMatrix, FP64 sparse copy). Y = A X (beta 0) per
    k and value type; GFLOP/s = 2 nnz k / t, GB/s over matrix bytes + k (4n + 4m)."""
    import torch
    out = {}
    rng = torch.Generator(device="cuda")
    rng.manual_seed(5)
    for key, m, A64 in entries:
        rows, cols = m.shape
        nnz = int(m.nnz)
        packs = {vt: (None if vt == "f32" else m.pack(vt)) for vt in value_types}
        for k in ks:
            X = torch.rand((cols, k), generator=rng, device="cuda") * 2 - 1
            Y = torch.empty((rows, k), device="cuda")
            for vt in value_types:
                p = packs[vt]
                for _ in range(3):
                    m.spmm(X, Y, 1.0, 0.0, packed=p)
                e0, e1 = _events(torch)
                e0.record()
                for _ in range(reps):
                    m.spmm(X, Y, 1.0, 0.0, packed=p)
                e1.record()
                torch.cuda.synchronize()
                ms = e0.elapsed_time(e1) / reps
                ab = matrix_bytes(m, vt) + k * (4 * cols + 4 * rows)
                r = dict(ms=round(ms, 4), gflops=round(2.0 * nnz * k / (ms * 1e-3) / 1e9, 1),
                         gbs=round(ab / (ms * 1e-3) / 1e9, 1), err_fp64=fp64_error(A64, X, Y, rows=min(rows, 1 << 18)))
                if hbm_gbs:
                    r["frac"] = round(r["gbs"] / hbm_gbs, 3)
                out[f"{key}/k{k}/{vt}"] = r
            del X, Y
    return out


def spmm_tc_sweep(m, A64, ks=(16, 32, 64), reps: int = 10, hbm_gbs=None):
    """A b4csr matrix of 4 x 4 blocks times k right-hand sides (beta 0) on
    the tensor cores (tcgen05, TF32 head and remainder) and in the CUDA-core
    lane-group kernel, per k: time, GFLOP/s, GB/s over matrix bytes +
    k (4n + 4m), error against FP64."""
    import torch
    out = {}
    rows, cols = m.shape
    nnz = int(m.nnz)
    rng = torch.Generator(device="cuda")
    rng.manual_seed(6)
    for k in ks:
        X = torch.rand((cols, k), generator=rng, device="cuda") * 2 - 1
        Y = torch.empty((rows, k), device="cuda")
        runs = {"tensor_cores": lambda: F.device_spmm_tc(m, X, Y, 1.0, 0.0), "cuda_cores": lambda: m.spmm(X, Y, 1.0, 0.0)}
        for name, run in runs.items():
            for _ in range(3):
                run()
            e0, e1 = _events(torch)
            e0.record()
            for _ in range(reps):
                run()
            e1.record()
            torch.cuda.synchronize()
            ms = e0.elapsed_time(e1) / reps
            ab = matrix_bytes(m, "f32") + k * (4 * cols + 4 * rows)
            r = dict(ms=round(ms, 4), gflops=round(2.0 * nnz * k / (ms * 1e-3) / 1e9, 1),
                     gbs=round(ab / (ms * 1e-3) / 1e9, 1), err_fp64=fp64_error(A64, X, Y, rows=min(rows, 1 << 18)))
            if hbm_gbs:
                r["frac"] = round(r["gbs"] / hbm_gbs, 3)
            out[f"k{k}/{name}"] = r
        out[f"k{k}/tensor_speedup"] = round(out[f"k{k}/cuda_cores"]["ms"] / out[f"k{k}/tensor_cores"]["ms"], 3)
        del X, Y
    out["timeouts"] = F.tensor_timeouts()
    return out


# ---------------------------------------------------------------------------
# Batches of uneven matrices (one persistent launch, captured in a graph)
# ---------------------------------------------------------------------------
def device_coo_of_csr(m: DeviceMatrix) -> DeviceMatrix:
    """The entries of a device CSR matrix as a device COO (row ids expanded
    from row_ptr; column ids and values shared with the CSR)."""
    import torch
    t = m.tensors
    rp = t["csr_row_ptr"].long()
    rows = torch.repeat_interleave(torch.arange(m.shape[0], device=rp.device, dtype=torch.int32), rp[1:] - rp[:-1])
    return DeviceMatrix.from_device_arrays("coo", dict(width=m.shape[1], height=m.shape[0], nnz=m.nnz),
                                           dict(coo_row_id=rows, coo_col_id=t["csr_col_id"], coo_data=t["csr_data"]))


# candidate layouts per generated structure: (format, converter arguments); CSR is the generated matrix itself
LAYOUTS = {
    "banded": [("dia", ()), ("ell", ()), ("csr", None)],
    "blocked": [("sbell", (4, 4, 32)), ("b4csr", (4, 4)), ("b4ell", (4, 4)), ("csr", None)],
    "random": [("csr", None)],
}


def tuned_layout(m_csr: DeviceMatrix, structure: str, ks=(1, 16), reps: int = 3):
    """The fastest of the structure's candidate layouts (LAYOUTS), timed as
    one job of the shared batch launch at each k in `ks` (one and many right-
    hand sides) and ranked by the sum, each candidate converted on the device
    from the matrix's entries (clspmv_device_coo2<fmt>_f32; the same entries,
    so the same product). Returns (matrix, format, {format: ms summed})."""
    import torch
    from . import _abi
    from .formats import device_convert
    rows, cols = m_csr.shape
    coo = device_coo_of_csr(m_csr)
    XY = [(torch.rand((cols, k), device="cuda"), torch.zeros((rows, k), device="cuda")) for k in ks]
    b = Batch(1)
    best, best_fmt, best_ms, times = m_csr, "csr", None, {}
    try:
        for fmt, args in LAYOUTS[structure]:
            try:
                cand = m_csr if fmt == "csr" else device_convert(coo, fmt, *args)
            except _abi.ClspmvError:      # refused (DIA fill rule, block caps) or unsorted input
                times[fmt] = None
                continue
            ms = 0.0
            for X, Y in XY:
                b.set([Job(cand, X, Y, alpha=1.0, beta=1.0)])
                b.run()
                e0, e1 = _events(torch)
                e0.record()
                for _ in range(reps):
                    b.run()
                e1.record()
                torch.cuda.synchronize()
                ms += e0.elapsed_time(e1) / reps
            times[fmt] = round(ms, 4)
            if best_ms is None or ms < best_ms:
                best, best_fmt, best_ms = cand, fmt, ms
    finally:
        b.close()
    del coo, XY
    return best, best_fmt, times


def uneven_matrices(count: int = 256, rows_lo: int = 1000, rows_hi: int = 500_000, npr_lo: int = 5, npr_hi: int = 64,
                    seed: int = 1234, tuned: bool = False, check: int = 0):
    """Device matrices: rows log-uniform in [rows_lo, rows_hi], mean
    nonzeros per row uniform in [npr_lo, npr_hi], structure banded /
    blocked / random drawn per matrix. Returns (structure, matrix, checker)
    triples: the matrix as CSR, or (tuned) in the fastest layout for its
    structure (tuned_layout); checker = the FP64 checker of every row
    (Fp64Rows of the CSR) for the first `check` matrices, else None."""
    rng = np.random.default_rng(seed)
    mats = []
    for i in range(count):
        rows = int(math.exp(rng.uniform(math.log(rows_lo), math.log(rows_hi))))
        npr = int(rng.integers(npr_lo, npr_hi + 1))
        structure = ["banded", "blocked", "random"][int(rng.integers(3))]
        lo, hi = max(1, npr - npr // 4), npr + npr // 4
        csr = synth.device_csr(rows, rows, lo, hi, structure, seed=seed + i)
        ref = fp64_of_csr(csr, None) if i < check else None
        m = tuned_layout(csr, structure)[0] if tuned else csr
        mats.append((structure, m, ref))
    return mats


def layout_counts(mats) -> dict:
    """How many matrices of each structure ended in each format."""
    out = {}
    for entry in mats:
        key = f"{entry[0]}->{entry[1].fmt}"
        out[key] = out.get(key, 0) + 1
    return out


def batched(mats, ks=(1, 4, 16, 32), value_types=("f32", "bf16", "f16"), reps: int = 10, check: int = 8):
    """Per (value type, k): all matrices as ONE batch launch replayed from a
    CUDA graph, against the same jobs as one plain launch per matrix.
    `mats`: (structure, matrix[, checker]) entries; the error against FP64
    covers the entries that carry a checker (else the first `check` CSR
    matrices, every row)."""
    import torch
    out = {}
    nnz_total = sum(e[1].nnz for e in mats)
    refs = [e[2] if len(e) > 2 else None for e in mats]
    if not any(r is not None for r in refs):
        refs = [fp64_of_csr(e[1], None) if i < check and e[1].fmt == "csr" else None for i, e in enumerate(mats)]
    checked = [i for i, r in enumerate(refs) if r is not None]
    mats = [(e[0], e[1]) for e in mats]
    packs = {vt: [None if vt == "f32" else m.pack(vt) for _, m in mats] for vt in value_types}
    gen = torch.Generator(device="cuda")
    gen.manual_seed(7)
    s = torch.cuda.Stream()
    for k in ks:
        Xs = [torch.rand((m.shape[1], k), generator=gen, device="cuda") * 2 - 1 for _, m in mats]
        Ys = [torch.empty((m.shape[0], k), device="cuda") for _, m in mats]
        for vt in value_types:
            # Y += A X (beta 1): CSR jobs are cut by nonzeros; Y is zeroed before the checked run
            jobs = [Job(m, X, Y, 1.0, 1.0, packed=p) for (_, m), X, Y, p in zip(mats, Xs, Ys, packs[vt])]
            b = Batch(len(jobs))
            s.wait_stream(torch.cuda.current_stream())
            with torch.cuda.stream(s):
                b.set(jobs, s)
                for _ in range(3):
                    b.run(s)
                n0 = F.launch_count()
                b.run(s)
                launches = F.launch_count() - n0     # 1, or 2 with 4x4-block jobs (their own launch)
            torch.cuda.current_stream().wait_stream(s)
            torch.cuda.synchronize()
            g = torch.cuda.CUDAGraph()
            with torch.cuda.graph(g):
                b.run()
            g.replay()
            e0, e1 = _events(torch)
            e0.record()
            for _ in range(reps):
                g.replay()
            e1.record()
            torch.cuda.synchronize()
            t_batch = e0.elapsed_time(e1) / reps
            for Y in Ys:
                Y.zero_()
            g.replay()
            torch.cuda.synchronize()
            err = max((fp64_error(refs[i], Xs[i], Ys[i]) for i in checked), default=0.0)
            # the same jobs, one plain clspmv_spmm launch each
            for j in jobs:
                j.matrix.spmm(j.X, j.Y, 1.0, 0.0, packed=j.packed)
            e0.record()
            for _ in range(reps):
                for j in jobs:
                    j.matrix.spmm(j.X, j.Y, 1.0, 0.0, packed=j.packed)
            e1.record()
            torch.cuda.synchronize()
            t_seq = e0.elapsed_time(e1) / reps
            del g
            b.close()
            out[f"k{k}/{vt}"] = dict(ms=round(t_batch, 4), gflops=round(2.0 * nnz_total * k / (t_batch * 1e-3) / 1e9, 1),
                                     plain_ms=round(t_seq, 4), speedup=round(t_seq / t_batch, 2), err_fp64=err,
                                     launches=launches)
        del Xs, Ys
    return out


# ---------------------------------------------------------------------------
# Serving: Poisson arrivals against resident matrices
# ---------------------------------------------------------------------------
def serving_matrices(count: int = 64, rows_lo: int = 10_000, rows_hi: int = 4_000_000, nnz_lo: float = 20e6,
                     nnz_hi: float = 200e6, seed: int = 99, tuned: bool = False):
    """Device matrices for the serving stream (rows log-uniform, nonzeros
    log-uniform, structure banded / blocked / random), as CSR or (tuned)
    each in the fastest layout for its structure (tuned_layout)."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(count):
        rows = int(math.exp(rng.uniform(math.log(rows_lo), math.log(rows_hi))))
        nnz = math.exp(rng.uniform(math.log(nnz_lo), math.log(nnz_hi)))
        npr = max(1, int(round(nnz / rows)))
        npr = min(npr, rows)
        structure = ["banded", "blocked", "random"][int(rng.integers(3))]
        m = synth.device_csr(rows, rows, max(1, npr - npr // 8), npr + npr // 8, structure, seed=seed + i)
        if tuned:
            m = tuned_layout(m, structure)[0]
            m.structure = structure
        out.append(m)
    return out


def _alloc_counts(torch) -> dict:
    """The caching allocator's device allocations, frees and retries so far
    (a retry frees every cached block and synchronises the device)."""
    st = torch.cuda.memory_stats()
    return {"device_allocs": int(st.get("num_device_alloc", 0)), "device_frees": int(st.get("num_device_free", 0)),
            "retries": int(st.get("num_alloc_retries", 0))}


def _wait_until(t: float) -> None:
    """Sleep until perf_counter() reaches t. Sleeping (not spinning) leaves
    the interpreter lock to the serving loop's thread."""
    dt = t - time.perf_counter()
    if dt > 0:
        time.sleep(dt)


def sharded_serving_hosts(count: int = 16, seed: int = 21):
    """Host matrices for the multi-GPU serving leg: banded, power-law and
    4x4-block matrices of 0.5-3M nonzeros, as CSR."""
    from . import formats as Fm
    rng = np.random.default_rng(seed)
    out = []
    for i in range(count):
        kind = ("banded", "powerlaw", "blocked")[i % 3]
        if kind == "banded":
            arrs = synth.banded(int(rng.integers(100_000, 400_000)), 7, seed=seed + i)
        elif kind == "powerlaw":
            arrs = synth.powerlaw(int(rng.integers(50_000, 150_000)), mean=16.0, maxlen=2000, seed=seed + i)
        else:
            arrs = synth.block_rows(int(rng.integers(10_000, 40_000)), 8, seed=seed + i)
        out.append((kind, Fm.coo2csr(Fm.coo_matrix(*arrs))))
    return out


def serve_sharded(hosts, devices, budget_per_device: int, n_requests: int = 2000, rate: float = 20_000.0,
                  k_lo: int = 1, k_hi: int = 8, seed: int = 5, owned=None):
    """serving.ShardedServer over `devices`: the host matrices registered
    whole on the device with the most budget left, an open-loop Poisson
    stream of `n_requests` (k uniform in [k_lo, k_hi], matrix uniform over
    all `hosts`), each request routed to its matrix's device. With `owned`
    (indices into `hosts`), only those matrices are registered and only
    their requests are submitted, at the stream's arrival times: the share
    of one process of a node that serves a placement (serving.place) on its
    own GPU. Returns served req/s, p50 / p99, the time from the first
    submission to the last completion, and matrices / requests per device."""
    import torch
    from .serving import ShardedServer, latency_stats
    rng = np.random.default_rng(seed)
    pick_all = rng.integers(len(hosts), size=n_requests)
    ks_all = rng.integers(k_lo, k_hi + 1, size=n_requests)
    arrivals_all = np.cumsum(rng.exponential(1.0 / rate, size=n_requests))
    mine = set(range(len(hosts))) if owned is None else set(int(i) for i in owned)
    srv = ShardedServer(budget_per_device, devices=devices)
    for i in sorted(mine):
        if srv.register(f"m{i}", hosts[i][1]) is None:
            raise RuntimeError(f"matrix {i} fits no device")
    sel = [j for j in range(n_requests) if int(pick_all[j]) in mine]
    # one (width x k_hi) block of right-hand sides per matrix, on the matrix's device
    pools = {}
    for i in sorted(mine):
        d = srv.devices[srv.owner[f"m{i}"]]
        gen = torch.Generator(device=d)
        gen.manual_seed(seed + i)
        pools[i] = torch.rand((hosts[i][1].shape[1], k_hi), generator=gen, device=d)
    for d in srv.devices:
        torch.cuda.synchronize(d)
    futures = []

    def client():
        t_start = time.perf_counter()
        for j in sel:
            _wait_until(t_start + arrivals_all[j])
            futures.append(srv.submit(f"m{int(pick_all[j])}", pools[int(pick_all[j])][:, :int(ks_all[j])],
                                      keep_result=False))

    gc.collect()
    gc.freeze()
    torch.cuda.empty_cache()
    a0 = _alloc_counts(torch)
    try:
        with srv:
            for i in sorted(mine):   # warm every matrix's path once
                srv.submit(f"m{i}", pools[i][:, :1], keep_result=False).result(timeout=600)
            th = threading.Thread(target=client)
            th.start()
            th.join()
            for f in futures:
                f.result(timeout=600)
    finally:
        gc.unfreeze()
    a1 = _alloc_counts(torch)
    out = dict(devices=len(srv.devices), matrices=len(mine), requests=len(sel), offered_req_per_s=rate,
               k=[k_lo, k_hi],
               matrices_per_device=[sum(1 for i in mine if srv.owner[f"m{i}"] == j) for j in range(len(srv.devices))],
               requests_per_device=[sum(1 for j in sel if srv.owner[f"m{int(pick_all[j])}"] == d)
                                    for d in range(len(srv.devices))],
               standalone=sum(1 for s in srv.servers for r in s.mats.values() if r.standalone),
               allocator={k: a1[k] - a0[k] for k in a0})
    if futures:
        st = latency_stats(futures)
        reqs = [f.request for f in futures]
        out["span_s"] = max(r.t_done for r in reqs) - min(r.t_submit for r in reqs)
        out["served"] = dict(req_per_s=round(st["req_per_s"], 1), p50_ms=round(st["p50_ms"], 3),
                             p99_ms=round(st["p99_ms"], 3))
    return out


def serve(mats, budget_bytes: int, n_requests: int = 1000, rate: float = 20_000.0, k_lo: int = 1, k_hi: int = 32,
          value_type: str = "f32", seed: int = 3, slots: int = 2, max_requests: int = 4096):
    """Open-loop Poisson stream of `n_requests` at `rate` req/s, k uniform in
    [k_lo, k_hi], matrix uniform among the admitted ones. Returns the serving
    loop's and the sequential baseline's req/s and p50 / p99 latency."""
    import torch
    from .serving import SpmvServer, latency_stats
    rng = np.random.default_rng(seed)
    srv = SpmvServer(budget_bytes, slots=slots, max_requests=max_requests)
    names = []
    for i, m in enumerate(mats):
        p = None if value_type == "f32" else m.pack(value_type)
        if srv.register(f"m{i}", m, p):
            names.append(f"m{i}")
    admitted_bytes = srv.used
    pick = rng.integers(len(names), size=n_requests)
    ks = rng.integers(k_lo, k_hi + 1, size=n_requests)
    arrivals = np.cumsum(rng.exponential(1.0 / rate, size=n_requests))
    gen = torch.Generator(device="cuda")
    gen.manual_seed(seed)
    # one (width x k_hi) block of right-hand sides per matrix; a request uses its first k columns
    pools = {nm: torch.rand((srv.mats[nm].matrix.shape[1], k_hi), generator=gen, device="cuda") for nm in names}
    Xs = [pools[names[p]][:, :int(k)] for p, k in zip(pick, ks)]
    torch.cuda.synchronize()

    # sequential plain launches: one clspmv_spmm + synchronize per request, same arrival times
    lat_seq = []
    t0 = time.perf_counter()
    for i in range(n_requests):
        _wait_until(t0 + arrivals[i])
        res = srv.mats[names[pick[i]]]
        Y = torch.empty((res.matrix.shape[0], int(ks[i])), device="cuda")
        res.matrix.spmm(Xs[i], Y, 1.0, 0.0, packed=res.packed)
        torch.cuda.synchronize()
        lat_seq.append(time.perf_counter() - t0 - arrivals[i])
        del Y
    span_seq = time.perf_counter() - t0
    lat_seq = np.array(lat_seq) * 1e3

    # the serving loop, fed by a client thread on the same schedule; the
    # objects alive before the stream are moved out of the cyclic collector's
    # reach for its duration (a full collection over a large process can
    # stall the loop thread for a whole batch)
    futures = [None] * n_requests
    def client():
        t_start = time.perf_counter()
        for i in range(n_requests):
            _wait_until(t_start + arrivals[i])
            futures[i] = srv.submit(names[pick[i]], Xs[i], keep_result=False)

    gc.collect()
    gc.freeze()
    torch.cuda.empty_cache()   # blocks cached by earlier work go back; the stream's own allocations stay cached
    a0 = _alloc_counts(torch)
    try:
        with srv:
            # warm the loop's batches once
            srv.submit(names[pick[0]], Xs[0], keep_result=False).result(timeout=600)
            th = threading.Thread(target=client)
            th.start()
            th.join()
            for f in futures:
                f.result(timeout=600)
            batches = srv.batches_run
    finally:
        gc.unfreeze()
    a1 = _alloc_counts(torch)
    stats = latency_stats(futures)
    return dict(requests=n_requests, offered_req_per_s=rate, k=[k_lo, k_hi], value_type=value_type,
                matrices=len(names), resident_gb=round(admitted_bytes / 1e9, 2),
                served=dict(req_per_s=round(stats["req_per_s"], 1), p50_ms=round(stats["p50_ms"], 3),
                            p99_ms=round(stats["p99_ms"], 3), batches=batches - 1),
                sequential=dict(req_per_s=round(n_requests / span_seq, 1), p50_ms=round(float(np.percentile(lat_seq, 50)), 3),
                                p99_ms=round(float(np.percentile(lat_seq, 99)), 3)),
                speedup=round(stats["req_per_s"] / (n_requests / span_seq), 2),
                standalone=sum(1 for nm in names if srv.mats[nm].standalone),
                allocator={k: a1[k] - a0[k] for k in a0})
