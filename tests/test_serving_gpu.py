"""Batched persistent launches and the serving loop, against the oracle.

* one clspmv_batch_run over jobs of every batchable format, FP32 / BF16 /
  FP16 values and k from 1 to 64: every column of every job within the
  per-row bound of the oracle's csr_spmv (FP32 values: 1e-5 sum|a x|;
  BF16 / FP16 values against FP64: 2^-8 / 2^-10 sum|a x|), and equal to the
  same job run alone (clspmv_spmm) within twice the FP32 row bound;
* the batch launch replays correctly from a captured CUDA graph;
* the server admits matrices by memory budget, fuses requests, and every
  result meets the oracle's per-row bound and equals the same request run
  alone within twice the FP32 row bound (the stored values are the same;
  only the summation order may differ).
"""
import random
import threading

import numpy as np
import pytest

from clspmv_mic_b200 import _abi
from clspmv_mic_b200 import formats as F
from clspmv_mic_b200.batch import Batch, Job
from clspmv_mic_b200.serving import SpmvServer, latency_stats

from matrices import coo_of
from tests.gpu_util import RTOL, assert_columns_close, columns_reference

pytestmark = pytest.mark.gpu

MATS = [("laplace33", "csr", ()), ("laplace33", "dia", ()), ("stencil6", "bdia", ()), ("powerlaw3k", "ell", ()),
        ("powerlaw3k", "sell", (32,)), ("blocks_odd", "b4csr", (4, 4)), ("blocks300", "b4ell", (8, 2)),
        ("blocks300", "sbell", (4, 4)), ("random_empty_rows", "csr", ()), ("tall", "sell", (128,))]


def _device(name, fmt, args):
    coo = coo_of(name)
    return F.DeviceMatrix(getattr(F, f"coo2{fmt}")(coo, *args))


def _bound(dev_alone_y):
    return np.abs(dev_alone_y) + 1e-30


def _alone(dev, X, alpha, packed):
    import torch
    Y = torch.zeros((dev.shape[0], X.shape[1]), device="cuda")
    dev.spmm(X, Y, alpha, 0.0, packed=packed)
    return Y


@pytest.mark.parametrize("graph", [False, True])
def test_batch_matches_alone(graph):
    import torch
    rng = np.random.default_rng(4)
    jobs, alone, devs = [], [], []
    for i, (name, fmt, args) in enumerate(MATS * 2):
        dev = _device(name, fmt, args)
        devs.append(dev)
        vt = ["f32", "bf16", "f16"][i % 3]
        packed = None if vt == "f32" else dev.pack(vt)
        k = [1, 3, 4, 16, 36, 64, 2, 8][i % 8]
        X = torch.from_numpy(rng.uniform(-1, 1, (dev.shape[1], k)).astype(np.float32)).cuda()
        Y = torch.full((dev.shape[0], k), float("nan"), device="cuda")
        jobs.append(Job(dev, X, Y, alpha=1.5, beta=0.0, packed=packed))
        alone.append(_alone(dev, X, 1.5, packed))
    b = Batch(64)
    b.set(jobs)
    if graph:
        g = torch.cuda.CUDAGraph()
        s = torch.cuda.Stream()
        s.wait_stream(torch.cuda.current_stream())
        with torch.cuda.stream(s):
            b.run(s)          # warm-up outside capture
        torch.cuda.current_stream().wait_stream(s)
        for j in jobs:
            j.Y.fill_(float("nan"))
        with torch.cuda.graph(g):
            b.run()
        g.replay()
        g.replay()
    else:
        b.run()
    torch.cuda.synchronize()
    for i, (j, a, (name, fmt, _)) in enumerate(zip(jobs, alone, MATS * 2)):
        got, ref = j.Y.cpu().numpy(), a.cpu().numpy()
        assert np.all(np.isfinite(got)), (name, fmt)
        vt = ["f32", "bf16", "f16"][i % 3]
        cref = columns_reference(coo_of(name), j.X.cpu().numpy(), 1.5)
        assert_columns_close(got, cref, vt, f"batch {name} {fmt} {vt}")
        # the same stored values as alone; CSR splits rows by nonzeros and k = 1 runs the format's
        # own single-vector kernel, so the summation order (not the values) may differ
        assert np.all(np.abs(got.astype(np.float64) - ref) <= 2 * RTOL * cref[2] + 1e-30), (name, fmt, "alone")
    b.close()


def test_batch_block_jobs_same_bits_as_alone():
    """4x4-block jobs with 128-bit X rows run in the batch's block-row launch
    (k_batch_blocks), the others in the row launch: with the two kinds
    interleaved in the caller's list, every block job's Y equals the same
    product run alone (the same block-row code) bit for bit, and every job
    meets the oracle's per-row bound."""
    import torch
    rng = np.random.default_rng(11)
    specs = []
    for name in ("blocks300", "blocks_odd", "ragged_tail"):
        for fmt in ("b4csr", "b4ell", "sbell"):
            specs.append((name, fmt, (4, 4)))
        specs.append((name, "csr", ()))
    jobs, alone = [], []
    for i, (name, fmt, args) in enumerate(specs):
        dev = _device(name, fmt, args)
        vt = ["f32", "bf16"][i % 2]
        packed = None if vt == "f32" else dev.pack(vt)
        k = [4, 16, 32, 8][i % 4]
        X = torch.from_numpy(rng.uniform(-1, 1, (dev.shape[1], k)).astype(np.float32)).cuda()
        Y = torch.full((dev.shape[0], k), float("nan"), device="cuda")
        jobs.append(Job(dev, X, Y, alpha=0.5, beta=0.0, packed=packed))
        alone.append(_alone(dev, X, 0.5, packed))
    b = Batch(len(jobs))
    b.set(jobs)
    b.run()
    torch.cuda.synchronize()
    for i, (j, a, (name, fmt, _)) in enumerate(zip(jobs, alone, specs)):
        got = j.Y.cpu().numpy()
        vt = ["f32", "bf16"][i % 2]
        cref = columns_reference(coo_of(name), j.X.cpu().numpy(), 0.5)
        assert_columns_close(got, cref, vt, f"batch {name} {fmt} {vt}")
        if fmt != "csr":
            assert np.array_equal(got.view(np.uint32), a.cpu().numpy().view(np.uint32)), (name, fmt, vt)
    b.close()


def test_batch_rejects():
    import torch
    coo = coo_of("laplace16")
    dev = F.DeviceMatrix(coo)
    X = torch.zeros((coo.shape[1], 1), device="cuda")
    Y = torch.zeros((coo.shape[0], 1), device="cuda")
    b = Batch(4)
    with pytest.raises(ValueError):
        b.set([Job(dev, X, Y)])          # COO has no row starts to walk
    ok = _device("laplace16", "csr", ())
    with pytest.raises(_abi.ClspmvError):
        b.set([Job(ok, X, Y)] * 5)       # more jobs than the table holds
    b.close()


def test_server_budget_admission():
    devs = [_device(n, f, a) for n, f, a in MATS[:3]]
    budget = devs[0].stored_bytes + devs[1].stored_bytes
    srv = SpmvServer(budget)
    assert srv.register("a", devs[0]) and srv.register("b", devs[1])
    assert not srv.register("c", devs[2])
    srv.unregister("a")
    assert srv.register("c", devs[2]) or devs[2].stored_bytes > devs[0].stored_bytes
    srv.stop()


def test_server_mixed_requests_match_alone():
    import torch
    rng = np.random.default_rng(9)
    devs = {}
    for i, (name, fmt, args) in enumerate(MATS):
        dev = _device(name, fmt, args)
        packed = dev.pack("bf16") if i % 4 == 3 else None
        devs[f"m{i}"] = (dev, packed)
    names = {}
    with SpmvServer(1 << 34, slots=2) as srv:
        for i, (key, (dev, packed)) in enumerate(devs.items()):
            names[key] = (MATS[i][0], "bf16" if packed is not None else "f32")
            assert srv.register(key, dev, packed)
        reqs = []
        keys = list(devs)
        for i in range(300):
            key = keys[rng.integers(len(keys))]
            dev, packed = devs[key]
            k = int(rng.integers(1, 33))
            X = torch.from_numpy(rng.uniform(-1, 1, (dev.shape[1], k)).astype(np.float32)).cuda()
            reqs.append((key, X, srv.submit(key, X)))
        results = [(key, X, f.result(timeout=120)) for key, X, f in reqs]
        stats = latency_stats([f for _, _, f in reqs])
        assert srv.batches_run < len(reqs)        # requests were fused into batches
    for key, X, Y in results:
        dev, packed = devs[key]
        name, vt = names[key]
        alone = _alone(dev, X, 1.0, packed).cpu().numpy()
        got = Y.cpu().numpy()
        cref = columns_reference(coo_of(name), X.cpu().numpy(), 1.0)
        assert_columns_close(got, cref, vt, f"served {key} {dev.fmt} {vt}")
        # the same request alone: the same stored values, another summation order at most
        assert np.all(np.abs(got.astype(np.float64) - alone) <= 2 * RTOL * cref[2] + 1e-30), (key, dev.fmt, "alone")
    assert stats["p99_ms"] >= stats["p50_ms"] > 0


def test_batch_csr_accumulate_splits_rows():
    """CSR jobs with beta 1 and long rows are cut by nonzeros (rows shared
    between warps), others by rows: Y0 + alpha A X agrees with the
    single-matrix SpMM."""
    import torch
    rng = np.random.default_rng(21)
    jobs, expect = [], []
    from clspmv_mic_b200 import synth
    long_rows = F.coo_matrix(*synth.random_coo(500, 4000, 0.1, seed=8, empty_row_frac=0.1))   # ~400 per row
    for name in ["long_rows", "powerlaw3k", "long_rows", "laplace33"]:
        dev = F.DeviceMatrix(F.coo2csr(long_rows)) if name == "long_rows" else _device(name, "csr", ())
        for k, vt in [(1, "f32"), (6, "bf16"), (16, "f32"), (36, "f16")]:
            packed = None if vt == "f32" else dev.pack(vt)
            X = torch.from_numpy(rng.uniform(-1, 1, (dev.shape[1], k)).astype(np.float32)).cuda()
            Y0 = torch.from_numpy(rng.uniform(-1, 1, (dev.shape[0], k)).astype(np.float32)).cuda()
            ref = Y0.clone()
            dev.spmm(X, ref, 0.75, 1.0, packed=packed)
            jobs.append(Job(dev, X, Y0, alpha=0.75, beta=1.0, packed=packed))
            expect.append(ref)
    b = Batch(len(jobs))
    b.set(jobs)
    b.run()
    torch.cuda.synchronize()
    for j, ref in zip(jobs, expect):
        got, r = j.Y.cpu().numpy(), ref.cpu().numpy()
        assert np.max(np.abs(got - r)) <= 1e-5 * (np.abs(r).max() + 1.0), j.matrix.shape
    b.close()
