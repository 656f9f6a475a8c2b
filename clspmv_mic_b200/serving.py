"""A serving loop for SpMV / SpMM requests against resident matrices.

Matrices are registered once and stay in HBM in their tuned format (FP32 or
packed 16-bit values) while their bytes fit the memory budget; registration
past the budget is refused (admission by memory). Requests are
Y = alpha * A * X with any k; a loop thread forms batches continuously:

* requests waiting when a slot frees up are grouped by matrix, and the X
  columns of one matrix's requests are placed side by side, so A is read
  once for all of them (up to 128 columns per job);
* the fused jobs of the batch run in ONE persistent launch
  (clspmv_batch_run); a request that is alone for its matrix runs in that
  format's own load-balanced kernel on the same stream, so a lightly loaded
  server answers as fast as a plain launch; registration times a fused
  product both ways for each matrix and sends that matrix's fused groups to
  its own kernel when that is faster (long rows split by nonzeros beat the
  shared launch's row walk; short rows the other way round);
* `slots` batches can be in flight at once on separate streams, so requests
  that arrive while a batch runs are admitted into the next slot and their
  work overlaps the running batch on the device.

Each request's result is the same whether it runs alone or in a mix, within
the FP32 bound: in a batch every row of Y is one group's sum over that row's
stored elements in storage order, whatever the other columns and jobs are;
alone, the same values may be summed in another order (CSR splits rows by
nonzeros, k = 1 uses the format's single-vector kernel)
(tests/test_serving_gpu.py).

ShardedServer runs one such server per GPU of a node, with every matrix
resident whole on one device and its requests routed there.

The reference has no serving path; its runtime runs one matrix per call and
waits for it (src/spmv_cocktail.cpp:1088-1132).
"""
from __future__ import annotations

import threading
import time
from collections import deque
from concurrent.futures import Future
from dataclasses import dataclass, field
from typing import Optional

from .batch import Batch, Job
from .formats import DeviceMatrix, PackedValues

MAX_COLUMNS = 128


@dataclass
class Resident:
    name: str
    matrix: DeviceMatrix
    packed: Optional[PackedValues]
    nbytes: int
    last_used: float = 0.0
    standalone: bool = False   # fused groups run the matrix's own SpMM kernel, not the shared launch


@dataclass
class Request:
    name: str
    X: object
    alpha: float
    future: Future
    t_submit: float
    stream: object = None         # the stream X was produced on (current at submission)
    t_done: float = 0.0
    nbytes: int = 0               # X and Y bytes the request holds on the device
    keep: bool = True             # False: the future resolves to None


@dataclass
class _Flight:
    event: object
    requests: list
    outputs: list = field(default_factory=list)


class SpmvServer:
    def __init__(self, budget_bytes: int, slots: int = 2, max_jobs: int = 256, max_requests: int = 1024,
                 max_batch_bytes: int = 8 << 30, device: str = "cuda", tune_k: int = 8):
        import torch
        self.torch = torch
        self.budget = int(budget_bytes)
        self.used = 0
        dev = torch.device(device)
        self.device = torch.device("cuda", torch.cuda.current_device()) if dev.index is None else dev
        self.max_requests = max_requests
        self.max_batch_bytes = int(max_batch_bytes)
        # width of the fused product timed at registration to choose, per
        # matrix, between the shared persistent launch and the matrix's own
        # SpMM kernel for its fused groups (0: always the shared launch)
        self.tune_k = int(tune_k)
        self.mats: dict[str, Resident] = {}
        self._pending: deque[Request] = deque()
        self._cv = threading.Condition()
        self._streams = [torch.cuda.Stream(device=device) for _ in range(slots)]
        self._batches = [Batch(max_jobs) for _ in range(slots)]
        self._flights: list[Optional[_Flight]] = [None] * slots
        self._stop = False
        self._thread: Optional[threading.Thread] = None
        self.batches_run = 0
        self.jobs_run = 0

    # -- residency ---------------------------------------------------------
    def register(self, name: str, matrix: DeviceMatrix, packed: Optional[PackedValues] = None) -> bool:
        """Keeps `matrix` resident for requests; False (nothing kept) when its
        bytes do not fit the remaining budget."""
        nbytes = int(matrix.stored_bytes) + (packed.nbytes if packed is not None else 0)
        with self._cv:
            if name in self.mats:
                raise KeyError(f"{name} is already registered")
            if self.used + nbytes > self.budget:
                return False
            self.mats[name] = Resident(name, matrix, packed, nbytes)
            self.used += nbytes
        if self.tune_k > 0:
            self.mats[name].standalone = self._standalone_faster(matrix, packed)
        return True

    def _standalone_faster(self, matrix: DeviceMatrix, packed: Optional[PackedValues], reps: int = 5) -> bool:
        """Times a fused product of `tune_k` columns both ways a group can
        run (one job of the shared persistent launch, or the matrix's own
        SpMM kernel) and tells whether the second is faster. Row-walked
        short rows favour the shared launch; long rows split by nonzeros
        favour the matrix's kernel."""
        torch = self.torch
        m, n = matrix.shape
        with torch.cuda.device(self.device):
            X = torch.rand((n, self.tune_k), device=self.device)
            Y = torch.zeros((m, self.tune_k), device=self.device)
            b = Batch(1)
            try:
                def shared():
                    b.set([Job(matrix, X, Y, alpha=1.0, beta=1.0, packed=packed)])
                    b.run()

                def own():
                    matrix.spmm(X, Y, 1.0, 0.0, packed=packed)

                times = []
                for fn in (shared, own):
                    fn()
                    torch.cuda.synchronize()
                    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                    e0.record()
                    for _ in range(reps):
                        fn()
                    e1.record()
                    torch.cuda.synchronize()
                    times.append(e0.elapsed_time(e1))
            finally:
                b.close()
            del X, Y
        return times[1] < 0.9 * times[0]   # a clear win only: the timings of a shared GPU are noisy

    def unregister(self, name: str) -> None:
        with self._cv:
            r = self.mats.pop(name)
            self.used -= r.nbytes

    # -- requests ----------------------------------------------------------
    def submit(self, name: str, X, alpha: float = 1.0, keep_result: bool = True) -> Future:
        """Y = alpha * A_name * X (X: CUDA float32, width x k or width, unit
        column stride); the future resolves to Y (height x k), or to None
        with keep_result=False (the request is only timed)."""
        torch = self.torch
        if name not in self.mats:
            raise KeyError(name)
        if X.dim() == 1:
            X = X.view(-1, 1)
        src = torch.cuda.current_stream(X.device)
        f: Future = Future()
        m, n = self.mats[name].matrix.shape
        req = Request(name, X, alpha, f, time.perf_counter(), stream=src,
                      nbytes=4 * X.shape[1] * (m + n), keep=keep_result)
        f.request = req     # submission / completion times for latency_stats
        with self._cv:
            self._pending.append(req)
            self._cv.notify()
        return f

    # -- loop --------------------------------------------------------------
    def start(self) -> "SpmvServer":
        self._thread = threading.Thread(target=self._loop, name="clspmv-serving", daemon=True)
        self._thread.start()
        return self

    def stop(self) -> None:
        with self._cv:
            self._stop = True
            self._cv.notify()
        if self._thread:
            self._thread.join()
        for b in self._batches:
            b.close()

    def __enter__(self):
        return self.start()

    def __exit__(self, *exc):
        self.stop()

    def _reap(self) -> bool:
        done_any = False
        for i, fl in enumerate(self._flights):
            if fl is not None and fl.event.query():
                now = time.perf_counter()
                for req, out in zip(fl.requests, fl.outputs):
                    req.t_done = now
                    req.future.set_result(out if req.keep else None)
                self._flights[i] = None
                done_any = True
        return done_any

    def _take(self) -> list:
        """Waiting requests, oldest first, up to max_requests and to
        max_batch_bytes of X and Y (always at least one)."""
        out, nbytes = [], 0
        with self._cv:
            while self._pending and len(out) < self.max_requests:
                r = self._pending[0]
                if out and nbytes + r.nbytes > self.max_batch_bytes:
                    break
                out.append(self._pending.popleft())
                nbytes += r.nbytes
        return out

    def _launch(self, slot: int, reqs: list) -> None:
        torch = self.torch
        st = self._streams[slot]
        groups: dict[str, list] = {}
        for r in reqs:
            groups.setdefault(r.name, []).append(r)
        jobs, order, outputs = [], [], []
        # one wait per source stream: an event recorded there now follows the
        # production of every X of this batch made on it (each was queued
        # before its submission), so no event is made per request
        sources = {}
        for r in reqs:
            sources[(r.stream.device, r.stream.cuda_stream)] = r.stream
        for src in sources.values():
            ev = torch.cuda.Event()
            ev.record(src)
            st.wait_event(ev)
        with torch.cuda.stream(st):
            for name, rs in groups.items():
                res = self.mats[name]
                res.last_used = time.perf_counter()
                m, n = res.matrix.shape
                # pack this matrix's requests into jobs of at most MAX_COLUMNS columns
                i = 0
                while i < len(rs):
                    part, cols = [], 0
                    while i < len(rs) and (not part or cols + rs[i].X.shape[1] <= MAX_COLUMNS):
                        part.append(rs[i])
                        cols += rs[i].X.shape[1]
                        i += 1
                    same_alpha = all(r.alpha == part[0].alpha for r in part)
                    if len(part) > 1:
                        # fused columns padded with zeros to a multiple of 4: the 16-byte row
                        # kernels (warp per long row, float4 gathers) need it
                        srcs = [r.X if same_alpha else r.X * r.alpha for r in part]
                        pad = -sum(x.shape[1] for x in srcs) % 4
                        if pad:
                            srcs.append(torch.zeros((srcs[0].shape[0], pad), dtype=torch.float32, device=srcs[0].device))
                        Xc = torch.cat(srcs, dim=1)
                    else:   # a lone request's X is used in place (any row stride)
                        Xc = part[0].X if part[0].X.stride(1) == 1 else part[0].X.contiguous()
                        if Xc.shape[1] % 4 and Xc.shape[1] > 32:
                            Xc = torch.nn.functional.pad(Xc, (0, 4 - Xc.shape[1] % 4))
                    alpha = part[0].alpha if same_alpha else 1.0
                    if len(part) == 1 or res.matrix.fmt == "coo" or res.standalone:
                        # a lone request, or a matrix whose own kernel is faster: on this slot's stream
                        Yc = torch.empty((m, Xc.shape[1]), dtype=torch.float32, device=Xc.device)
                        res.matrix.spmm(Xc, Yc, alpha, 0.0, packed=res.packed, stream=st)
                    else:
                        # Y += A X on a zeroed Y: CSR jobs with long rows are then split between warps
                        Yc = torch.zeros((m, Xc.shape[1]), dtype=torch.float32, device=Xc.device)
                        jobs.append(Job(res.matrix, Xc, Yc, alpha=alpha, beta=1.0, packed=res.packed))
                    off = 0
                    for r in part:
                        k = r.X.shape[1]
                        outputs.append(Yc[:, off:off + k])
                        order.append(r)
                        off += k
            if jobs:
                b = self._batches[slot]
                b.set(jobs, st)
                b.run(st)
            ev = torch.cuda.Event()
            ev.record(st)
        self._flights[slot] = _Flight(ev, order, outputs)
        self.batches_run += 1
        self.jobs_run += len(jobs)

    def _loop(self) -> None:
        try:
            self._serve()
        except BaseException as e:   # the loop died: fail every request it still holds
            with self._cv:
                pending = list(self._pending)
                self._pending.clear()
            for fl in self._flights:
                if fl is not None:
                    pending.extend(fl.requests)
            for r in pending:
                if not r.future.done():
                    r.future.set_exception(e)
            raise

    def _serve(self) -> None:
        torch = self.torch
        torch.cuda.set_device(self.device)
        while True:
            self._reap()
            free = [i for i, f in enumerate(self._flights) if f is None]
            with self._cv:
                if self._stop and not self._pending and len(free) == len(self._flights):
                    return
                has_work = bool(self._pending)
                if not has_work and len(free) == len(self._flights):
                    self._cv.wait(timeout=0.01)
                    continue
            if has_work and free:
                reqs = self._take()
                if reqs:
                    try:
                        self._launch(free[0], reqs)
                    except Exception as e:   # report the failure on every request of the batch
                        for r in reqs:
                            if not r.future.done():
                                r.future.set_exception(e)
                continue
            time.sleep(20e-6)


def latency_stats(requests: list) -> dict:
    """p50 / p99 / mean latency in ms and the request rate between the first
    submission and the last completion (Requests or the futures submit
    returned)."""
    import numpy as np
    requests = [getattr(r, "request", r) for r in requests]
    lat = np.array([r.t_done - r.t_submit for r in requests]) * 1e3
    span = max(r.t_done for r in requests) - min(r.t_submit for r in requests)
    return dict(requests=len(requests), p50_ms=float(np.percentile(lat, 50)), p99_ms=float(np.percentile(lat, 99)),
                mean_ms=float(lat.mean()), req_per_s=len(requests) / span if span > 0 else float("inf"))


# ---------------------------------------------------------------------------
# Several GPUs of one node: matrices placed whole, requests routed, no exchange
# ---------------------------------------------------------------------------
def resident_bytes(host, value_type: Optional[str] = None) -> int:
    """Device bytes a host matrix takes once registered: its arrays as
    uploaded, plus the 16-bit values (2 bytes per stored value) and per-row
    scales of the packed copy when `value_type` is "bf16" / "f16"."""
    nbytes = int(host.stored_bytes())
    if value_type is not None:
        values = sum(a.nbytes for k, a in host.arrays().items() if k.endswith("_data"))
        nbytes += values // 2 + 4 * int(host.shape[0])
    return nbytes


def place(sizes: dict, budgets: list) -> dict:
    """Whole matrices onto devices: largest first, each onto the device with
    the most budget left, if it fits there (longest-processing-time greedy,
    which keeps the most loaded device within one matrix of the best split).
    Returns name -> device index; names that fit on no device are left out."""
    free = [int(b) for b in budgets]
    out = {}
    for name, nbytes in sorted(sizes.items(), key=lambda kv: (-kv[1], str(kv[0]))):
        dev = max(range(len(free)), key=lambda i: (free[i], -i))
        if free[dev] >= nbytes:
            out[name] = dev
            free[dev] -= nbytes
    return out


def _upload(host, device, value_type: Optional[str]):
    import torch
    with torch.cuda.device(torch.device(device)):
        m = DeviceMatrix(host, device=device)
        return m, (m.pack(value_type) if value_type is not None else None)


class ShardedServer:
    """Serving on the GPUs of one node as independent units: each matrix is
    resident whole on one device, its requests go to that device's
    SpmvServer (own loop thread, streams and batches), and nothing crosses
    between devices except a request's X when the caller made it on another
    one. A matrix goes to the device with the most budget left that fits it,
    so devices fill evenly; registration past every device's budget is
    refused. With one device it is one SpmvServer.

    `make_server(device)` and `upload(host, device, value_type)` default to
    SpmvServer(budget_per_device, device=..., **server_kw) built on that
    device and to DeviceMatrix(host, device) (+ its packed copy)."""

    def __init__(self, budget_per_device: int, devices=None, make_server=None, upload=None, **server_kw):
        if devices is None:
            import torch
            devices = [f"cuda:{i}" for i in range(torch.cuda.device_count())]
        self.devices = list(devices)
        if not self.devices:
            raise ValueError("no devices to serve on")
        if make_server is None:
            def make_server(dev):
                import torch
                with torch.cuda.device(torch.device(dev)):   # the server's batches live on its device
                    return SpmvServer(budget_per_device, device=dev, **server_kw)
        self.servers = [make_server(d) for d in self.devices]
        self._upload = upload or _upload
        self.owner: dict = {}
        self._lock = threading.Lock()

    def free_bytes(self) -> list:
        return [s.budget - s.used for s in self.servers]

    def register(self, name: str, host, value_type: Optional[str] = None) -> Optional[int]:
        """Uploads `host` to the device with the most budget left and keeps it
        resident there; returns that device's index, or None (nothing kept)
        when it fits no device."""
        need = resident_bytes(host, value_type)
        with self._lock:
            if name in self.owner:
                raise KeyError(f"{name} is already registered")
            free = self.free_bytes()
            dev = max(range(len(free)), key=lambda i: (free[i], -i))
            if free[dev] < need:
                return None
            matrix, packed = self._upload(host, self.devices[dev], value_type)
            if not self.servers[dev].register(name, matrix, packed):
                return None
            self.owner[name] = dev
        return dev

    def unregister(self, name: str) -> None:
        with self._lock:
            dev = self.owner.pop(name)
        self.servers[dev].unregister(name)

    def submit(self, name: str, X, alpha: float = 1.0, keep_result: bool = True) -> Future:
        """Routes Y = alpha * A_name * X to the device holding A_name; the
        future resolves to Y on that device."""
        dev = self.owner.get(name)
        if dev is None:
            raise KeyError(name)
        server = self.servers[dev]
        device = getattr(server, "device", None)
        if device is not None and getattr(X, "device", device) != device:
            X = X.to(device)
        return server.submit(name, X, alpha, keep_result)

    def start(self) -> "ShardedServer":
        for s in self.servers:
            s.start()
        return self

    def stop(self) -> None:
        for s in self.servers:
            s.stop()

    def __enter__(self):
        return self.start()

    def __exit__(self, *exc):
        self.stop()
