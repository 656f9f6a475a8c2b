"""bench.py's multi-process path on the CPU (gloo, world size 2): ranks are
independent replicas, the job time is the slowest rank's, the whole-job
value counts every replica's work, and only rank 0 prints."""
import io
import os
import socket
import sys
from contextlib import redirect_stdout

import pytest
import torch.multiprocessing as mp

from conftest import ROOT


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, q):
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank), MASTER_ADDR="127.0.0.1",
                      MASTER_PORT=str(port))
    sys.path.insert(0, str(ROOT))
    import torch.distributed as dist
    import bench
    w, r, _ = bench.dist_init(None)
    slowest = bench.max_over_ranks(10.0 + 5.0 * rank, "cpu")
    value = bench.job_value(2e9, w, slowest)
    buf = io.StringIO()
    with redirect_stdout(buf):
        # the reference arm: ranks other than 0 leave at once, without output
        rc = bench.run_reference(type("A", (), {"small": True, "warmup": 0, "steps": 0})()) if r != 0 else 0
    dist.barrier()
    dist.destroy_process_group()
    q.put((r, w, slowest, value, rc, buf.getvalue()))


def test_two_ranks_gloo():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for r, w, slowest, value, rc, text in out:
        assert w == 2 and slowest == 15.0              # max over ranks
        assert value == pytest.approx(2e9 * 2 / 15e-3 / 1e9)
        assert rc == 0
        if r == 1:
            assert text == ""


@pytest.mark.parametrize("parts", [1, 3, 8])
def test_reference_arm_row_blocks_give_the_same_y(parts):
    """The reference arm runs csr_spmv on nnz-balanced row blocks in host
    threads; the blocks cover every row once and give y bit for bit."""
    import numpy as np
    sys.path.insert(0, str(ROOT))
    import bench
    from clspmv_mic_b200 import formats as F
    from oracle import oracle as O
    from tests.matrices import coo_of
    csr = F.coo2csr(coo_of("powerlaw3k"))
    x = np.random.default_rng(1).uniform(-1, 1, csr.shape[1]).astype(np.float32)
    fn = O.spmv_ref if O.ref() is not None else O.spmv_port
    full = fn(csr, x)
    y = np.zeros(csr.shape[0], np.float32)
    blocks = bench.row_blocks(csr, parts)
    assert blocks[0][0] == 0 and blocks[-1][1] == csr.shape[0]
    for (r0, r1, slab), nxt in zip(blocks, blocks[1:] + [(csr.shape[0], None, None)]):
        assert r1 == nxt[0]
        y[r0:r1] = fn(slab, x)
    assert np.array_equal(y.view(np.uint32), full.view(np.uint32))
