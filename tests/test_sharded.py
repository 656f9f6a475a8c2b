"""Row-sharded A^k x (clspmv_mic_b200/sharded.py).

On the CPU: the row split and the column renumbering, and the whole loop as
2 and 3 gloo ranks whose local SpMV is the oracle's csr_spmv (the
reference's serial routine) on each rank's slab, against the same loop on
one process with the unsharded matrix: rows are independent and each keeps
its column order, so x must match bit for bit. On one GPU: the device path
(world of one) against DeviceMatrix's own loop, bit for bit. More than one
GPU is not available to these tests."""
import os
import socket
import sys

import numpy as np
import pytest
import torch.multiprocessing as mp

from clspmv_mic_b200 import formats as F
from clspmv_mic_b200 import sharded as S

from conftest import ROOT


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_split_rows_balances_nonzeros():
    rng = np.random.default_rng(0)
    lens = rng.integers(0, 50, 1000)
    lens[500] = 5000                      # one heavy row
    rp = np.concatenate([[0], np.cumsum(lens)])
    for world in (1, 2, 3, 8):
        b = S.split_rows(rp, world)
        assert b[0][0] == 0 and b[-1][1] == 1000
        assert all(b[i][1] == b[i + 1][0] for i in range(world - 1))
        nnz = [rp[r1] - rp[r0] for r0, r1 in b]
        assert sum(nnz) == rp[-1]
        assert max(nnz) <= rp[-1] / world + lens.max()


def test_padded_columns_with_empty_ranks():
    bounds = [(0, 4), (4, 4), (4, 10)]     # rank 1 owns no rows
    block = 6
    col = np.arange(10)
    got = S.padded_columns(col, bounds, block)
    np.testing.assert_array_equal(got, [0, 1, 2, 3, 12, 13, 14, 15, 16, 17])


def _loop_reference(csr, x, y, k, alpha, beta):
    from oracle import oracle as O
    x, y = x.copy(), y.copy()
    for _ in range(k):
        ax = O.spmv_port(csr, x)
        y = (np.float32(alpha) * ax + np.float32(beta) * y).astype(np.float32)
        x = y.copy()
    return x


def _case(name):
    from tests.matrices import coo_of
    return F.coo2csr(coo_of(name))


def _vectors(n, seed=3):
    rng = np.random.default_rng(seed)
    return (rng.uniform(-1, 1, n).astype(np.float32) * np.float32(0.1),
            rng.standard_normal(n).astype(np.float32) * np.float32(0.1))


def _worker(rank, world, port, q, name, k, alpha, beta):
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    sys.path.insert(0, str(ROOT))
    import datetime
    import torch
    import torch.distributed as dist
    from oracle import oracle as O
    dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=60))
    try:
        csr = _case(name)
        holder = {}

        def local(x, y, a, b):
            ax = O.spmv_port(holder["s"].host, x.numpy())
            y.copy_(torch.from_numpy((np.float32(a) * ax + np.float32(b) * y.numpy()).astype(np.float32)))

        s = S.ShardedCsr(csr, device="cpu", local_spmv=local)
        holder["s"] = s
        x0, y0 = _vectors(csr.shape[0])
        s.load(x0, y0)
        s.iterate(k, alpha, beta)
        q.put((rank, s.global_x(), s.bounds))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world,name,k,alpha,beta", [(2, "powerlaw3k", 3, 0.5, 0.5), (3, "laplace33", 4, 0.25, 1.0),
                                                      (2, "random_empty_rows", 2, 1.0, 1.0)])
def test_gloo_ranks_match_one_process(world, name, k, alpha, beta):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q, name, k, alpha, beta)) for r in range(world)]
    for p in procs:
        p.start()
    out = sorted((q.get(timeout=180) for _ in procs), key=lambda t: t[0])
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    csr = _case(name)
    x0, y0 = _vectors(csr.shape[0])
    ref = _loop_reference(csr, x0, y0, k, alpha, beta)
    for rank, x, bounds in out:
        assert len(bounds) == world
        assert np.array_equal(x.view(np.uint32), ref.view(np.uint32)), rank


@pytest.mark.gpu
def test_device_world_of_one_matches_device_loop():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("needs a GPU")
    csr = _case("powerlaw3k")
    n = csr.shape[0]
    x0, y0 = _vectors(n)
    s = S.ShardedCsr(csr, device="cuda")
    s.load(x0, y0)
    s.iterate(5, 0.5, 0.5)
    dev = F.DeviceMatrix(csr)
    x = torch.from_numpy(x0).cuda()
    y = torch.from_numpy(y0).cuda()
    for _ in range(5):
        dev.spmv(x, y, 0.5, 0.5)
        x.copy_(y)
    torch.cuda.synchronize()
    got = s.global_x()
    want = x.cpu().numpy()
    # both run the chunked CSR kernel, whose cut rows add atomically: equal
    # within summation-order noise
    assert np.abs(got - want).max() <= 1e-5 * (np.abs(want).max() + 1e-30)


def _rows_worker(rank, world, port, q, n, k):
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    sys.path.insert(0, str(ROOT))
    import datetime
    import torch
    import torch.distributed as dist
    from clspmv_mic_b200 import synth
    from oracle import oracle as O
    dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=60))
    try:
        holder = {}

        def local(x, y, a, b):
            ax = O.spmv_port(holder["s"].host, x.numpy())
            y.copy_(torch.from_numpy((np.float32(a) * ax + np.float32(b) * y.numpy()).astype(np.float32)))

        # this rank generates its own rows only
        s = S.ShardedCsr(None, device="cpu", local_spmv=local, n=n ** 3,
                         make_rows=lambda r0, r1: synth.stencil_27pt_rows(n, r0, r1))
        holder["s"] = s
        x0, y0 = _vectors(n ** 3)
        s.load(x0, y0)
        s.iterate(k, 0.05, 0.5)
        q.put((rank, s.global_x(), s.bounds, s.host.nnz))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_gloo_ranks_from_own_rows_match_one_process(world):
    """Each rank builds its slab from its own rows of the 27-point stencil
    (no rank holds the whole matrix; rows split evenly): x after k steps
    equals the one-process loop on the whole matrix assembled from the same
    row generator, bit for bit."""
    from clspmv_mic_b200 import synth
    n, k = 9, 3
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rows_worker, args=(r, world, port, q, n, k)) for r in range(world)]
    for p in procs:
        p.start()
    out = sorted((q.get(timeout=180) for _ in procs), key=lambda t: t[0])
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    m = n ** 3
    bounds = S.split_rows_even(m, world)
    parts = [synth.stencil_27pt_rows(n, r0, r1) for r0, r1 in bounds]
    rp = np.concatenate([[0]] + [p[0][1:] + sum(int(q[0][-1]) for q in parts[:i]) for i, p in enumerate(parts)])
    csr = F.from_arrays("csr", dict(width=m, height=m, nnz=int(rp[-1])),
                        dict(csr_row_ptr=rp.astype(np.int32), csr_col_id=np.concatenate([p[1] for p in parts]),
                             csr_data=np.concatenate([p[2] for p in parts])))
    x0, y0 = _vectors(m)
    ref = _loop_reference(csr, x0, y0, k, 0.05, 0.5)
    assert sum(t[3] for t in out) == csr.nnz
    for rank, x, b, _ in out:
        assert b == bounds
        assert np.array_equal(x.view(np.uint32), ref.view(np.uint32)), rank
