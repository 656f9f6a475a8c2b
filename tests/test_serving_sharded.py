"""Serving on several GPUs as independent units (clspmv_mic_b200/serving.py:
place, resident_bytes, ShardedServer), without a GPU: placement is plain
host arithmetic, and the router is driven with stand-in servers that record
what reaches them. Matrices are never split, every device stays within its
budget, and a request reaches exactly the server that holds its matrix."""
from concurrent.futures import Future

import numpy as np
import pytest

from clspmv_mic_b200 import formats as F
from clspmv_mic_b200 import serving as SV

from matrices import coo_of


class FakeServer:
    def __init__(self, device, budget):
        self.device = device
        self.budget = budget
        self.used = 0
        self.mats = {}
        self.requests = []
        self.running = False

    def register(self, name, matrix, packed):
        nbytes = matrix[2]
        if self.used + nbytes > self.budget:
            return False
        self.mats[name] = nbytes
        self.used += nbytes
        return True

    def unregister(self, name):
        self.used -= self.mats.pop(name)

    def submit(self, name, X, alpha, keep_result):
        f = Future()
        self.requests.append((name, X, alpha))
        f.set_result((self.device, name))
        return f

    def start(self):
        self.running = True

    def stop(self):
        self.running = False


def _router(budget, ndev=3):
    def upload(host, device, value_type):
        return (host, device, SV.resident_bytes(host, value_type)), None
    return SV.ShardedServer(budget, devices=[f"dev{i}" for i in range(ndev)],
                            make_server=lambda d: FakeServer(d, budget), upload=upload)


def test_place_fits_and_balances():
    rng = np.random.default_rng(0)
    sizes = {f"m{i}": int(s) for i, s in enumerate(rng.integers(1, 100, 64))}
    budgets = [1000, 1000, 1000, 1000]
    where = SV.place(sizes, budgets)
    assert set(where) == set(sizes)                      # everything fits (sum ~3200 of 4000)
    load = [0] * 4
    for name, dev in where.items():
        load[dev] += sizes[name]
    assert all(l <= b for l, b in zip(load, budgets))
    # longest-first greedy: the most loaded device is within one matrix of the mean
    assert max(load) <= sum(sizes.values()) / 4 + max(sizes.values())


def test_place_leaves_out_what_fits_nowhere():
    where = SV.place({"big": 150, "a": 60, "b": 60, "c": 30}, [100, 100])
    assert "big" not in where
    assert where["a"] != where["b"]                      # never two 60s on one 100
    assert sorted(where) == ["a", "b", "c"]
    assert SV.place({}, [10]) == {}


def test_resident_bytes_counts_packed_copy():
    csr = F.coo2csr(coo_of("powerlaw3k"))
    base = SV.resident_bytes(csr)
    assert base == csr.stored_bytes()
    assert SV.resident_bytes(csr, "bf16") == base + 2 * csr.nnz + 4 * csr.shape[0]


def test_router_spreads_refuses_and_routes():
    mats = {name: F.coo2csr(coo_of(name)) for name in ("powerlaw3k", "laplace33", "random_sparse", "banded7")}
    need = {n: SV.resident_bytes(h) for n, h in mats.items()}
    budget = max(need.values()) * 2
    r = _router(budget)
    got = {n: r.register(n, h) for n, h in mats.items()}
    assert all(d is not None for d in got.values())
    assert len(set(got.values())) == 3                  # four matrices over three devices: all used
    for s in r.servers:
        assert s.used <= s.budget
    with pytest.raises(KeyError):
        r.register("laplace33", mats["laplace33"])
    # a matrix larger than any device's free budget is refused and leaves nothing behind
    huge = F.coo2csr(coo_of("powerlaw3k"))
    small = _router(need["powerlaw3k"] - 1, ndev=2)
    assert small.register("too_big", huge) is None
    assert "too_big" not in small.owner and all(s.used == 0 for s in small.servers)
    # requests reach the owner's server only
    r.start()
    assert all(s.running for s in r.servers)
    for n in mats:
        dev, name = r.submit(n, X=None).result()
        assert (dev, name) == (f"dev{got[n]}", n)
    for i, s in enumerate(r.servers):
        assert sorted(q[0] for q in s.requests) == sorted(n for n in mats if got[n] == i)
    with pytest.raises(KeyError):
        r.submit("unknown", X=None)
    # unregistering returns the bytes to that device
    dev = got["powerlaw3k"]
    before = r.servers[dev].used
    r.unregister("powerlaw3k")
    assert r.servers[dev].used == before - need["powerlaw3k"]
    r.stop()
    assert not any(s.running for s in r.servers)


def test_router_fills_most_free_device_first():
    host = F.coo2csr(coo_of("laplace16"))
    n = SV.resident_bytes(host)
    r = _router(2 * n, ndev=2)
    order = [r.register(f"m{i}", host) for i in range(5)]
    assert order == [0, 1, 0, 1, None]                   # ties go to the lower index; the fifth fits nowhere
    assert [s.used for s in r.servers] == [2 * n, 2 * n]
