"""The bench's extra workloads on small sizes: several right-hand sides with
FP32 / BF16 / FP16 values, a batch of uneven matrices, the serving loop."""
import numpy as np
import pytest

from clspmv_mic_b200 import formats as F
from clspmv_mic_b200 import synth
from clspmv_mic_b200 import workloads as W

from matrices import coo_of

pytestmark = pytest.mark.gpu


def test_spmm_sweep_small():
    csr = F.DeviceMatrix(F.coo2csr(coo_of("powerlaw3k")))
    dia = F.DeviceMatrix(F.coo2dia(coo_of("laplace33")))
    ref_dia = W.fp64_of_csr(F.DeviceMatrix(F.coo2csr(coo_of("laplace33"))))
    out = W.spmm_sweep([("csr", csr, W.fp64_of_csr(csr)), ("dia", dia, ref_dia)], ks=(1, 16), reps=2)
    assert len(out) == 2 * 2 * 3
    for key, r in out.items():
        assert r["ms"] > 0
        bound = 1e-5 if key.endswith("f32") else (2.0 ** -8 if key.endswith("bf16") else 2.0 ** -10)
        assert r["err_fp64"] <= bound, (key, r)


def test_batched_small():
    mats = W.uneven_matrices(12, rows_lo=500, rows_hi=20_000, npr_lo=5, npr_hi=40)
    out = W.batched(mats, ks=(1, 8), reps=2, check=4)
    for key, r in out.items():
        bound = 1e-5 if key.endswith("f32") else (2.0 ** -8 if key.endswith("bf16") else 2.0 ** -10)
        assert r["err_fp64"] <= bound, (key, r)
        assert r["ms"] > 0 and r["plain_ms"] > 0


def test_batched_tuned_layouts():
    """The batch with each matrix in the fastest layout for its structure
    (DIA / ELL for banded, SBELL / BCSR / BELL 4x4 for blocked, converted on
    the device from the generated CSR): every checked matrix (all rows)
    within the FP64 bound, and the layouts come from the candidate lists."""
    mats = W.uneven_matrices(12, rows_lo=500, rows_hi=20_000, npr_lo=5, npr_hi=40, tuned=True, check=12)
    for structure, m, _ in mats:
        assert m.fmt in [f for f, _ in W.LAYOUTS[structure]], (structure, m.fmt)
    out = W.batched(mats, ks=(1, 8), reps=2)
    for key, r in out.items():
        bound = 1e-5 if key.endswith("f32") else (2.0 ** -8 if key.endswith("bf16") else 2.0 ** -10)
        assert r["err_fp64"] <= bound, (key, r)


def test_tuned_layout_is_the_same_matrix():
    """A banded and a blocked generated matrix converted to every candidate
    layout give the CSR's product (the generators emit sorted, distinct
    columns for these structures, so the conversion keeps every entry)."""
    import torch
    from clspmv_mic_b200 import synth
    for structure in ("banded", "blocked"):
        csr = synth.device_csr(3000, 3000, 8, 24, structure, seed=11)
        coo = W.device_coo_of_csr(csr)
        ref = W.fp64_of_csr(csr, None)              # every row, FP64, per-row scale sum|a x|
        x = torch.rand(3000, device="cuda") * 2 - 1
        converted = 0
        for fmt, args in W.LAYOUTS[structure]:
            try:
                m = csr if fmt == "csr" else F.device_convert(coo, fmt, *args)
            except __import__("clspmv_mic_b200")._abi.ClspmvError as e:
                assert e.status == __import__("clspmv_mic_b200")._abi.ERR_REFUSED, (structure, fmt)
                continue    # the DIA fill rule refuses bands shifted at the matrix edges
            converted += 1
            y = torch.full((3000,), float("nan"), device="cuda")
            m.spmv(x, y, 1.0, 0.0)
            torch.cuda.synchronize()
            assert ref.error(x[:, None], y[:, None]) <= 1e-5, (structure, fmt)
        assert converted >= 2, structure


def test_serve_small():
    mats = W.serving_matrices(4, rows_lo=2000, rows_hi=20_000, nnz_lo=2e5, nnz_hi=1e6)
    r = W.serve(mats, 1 << 34, n_requests=60, rate=5000.0, k_lo=1, k_hi=8)
    assert r["matrices"] == 4
    assert r["served"]["req_per_s"] > 0 and r["sequential"]["req_per_s"] > 0
    assert r["served"]["p99_ms"] >= r["served"]["p50_ms"]


def test_serve_sharded_shares_cover_the_stream():
    """The multi-GPU serving leg's split: each process serves the requests
    of the matrices placed on it; the shares of a 3-way placement, run one
    after another on this GPU, serve every request of the stream once."""
    from clspmv_mic_b200 import serving as SV
    hosts = W.sharded_serving_hosts(count=6)
    whole = W.serve_sharded(hosts, ["cuda:0"], 1 << 32, n_requests=150, rate=20_000.0)
    assert whole["requests"] == 150 and whole["matrices"] == 6 and whole["served"]["req_per_s"] > 0
    assign = SV.place({i: SV.resident_bytes(h) for i, (_, h) in enumerate(hosts)}, [1 << 32] * 3)
    assert sorted(assign) == list(range(6))
    total = 0
    for r in range(3):
        owned = [i for i, d in assign.items() if d == r]
        part = W.serve_sharded(hosts, ["cuda:0"], 1 << 32, n_requests=150, rate=20_000.0, owned=owned)
        assert part["matrices"] == len(owned)
        total += part["requests"]
    assert total == 150


def test_measure_tables_small(tmp_path, monkeypatch):
    """Device-measured .ben tables are readable by the partitioner and give
    positive rates for every grid point."""
    from clspmv_mic_b200 import tables as T
    from clspmv_mic_b200.cocktail import analyze
    monkeypatch.setattr(T, "M_DIMS", [4096, 65536])
    monkeypatch.setattr(T, "M_BLOCK_DIMS", [4096, 65536])
    monkeypatch.setattr(T, "M_DIA_WIDTHS", [1, 5, 27])
    monkeypatch.setattr(T, "M_FLAT_WIDTHS", [1, 8, 32])
    monkeypatch.setattr(T, "M_BLOCKNUMS", [1, 4])
    T.measure_tables(tmp_path, reps=2)
    for name in ["overhead", "bdia", "dia", "sbell", "bell", "bcsr", "sell", "ell", "csr", "coo"]:
        rows = [list(map(float, l.split())) for l in (tmp_path / "benchmark" / f"{name}.ben").read_text().splitlines()]
        assert rows and all(v > 0 for r in rows for v in r), name
    m = analyze(coo_of("blocks300"), tmp_path)
    assert sum(v["nnz"] for k, v in m.summary().items() if isinstance(v, dict) and "nnz" in v and k != "shape") > 0


def test_tune_measures_and_caches(tmp_path):
    from clspmv_mic_b200 import tables as T
    from clspmv_mic_b200.autotune import tune
    root = T.model_tables(tmp_path / "t", seed=3, scale={"coo": 0.3})
    coo = coo_of("powerlaw3k")
    cache = tmp_path / "tune.json"
    r = tune(coo, root, cache=cache, reps=2)
    assert not r.from_cache and r.ms > 0 and r.report and r.report[0]["knob"] == {}
    assert min(c["ms"] for c in r.report) == pytest.approx(r.ms_partition, abs=1e-4)
    assert r.ms <= r.ms_partition + 1e-9
    again = tune(coo, root, cache=cache)
    assert again.from_cache and again.knob == r.knob and again.parts == r.parts and again.runtime == r.runtime
    assert r.runtime.get("schedule") in ("per_part", "fused") and r.runtime_report
    import torch
    dev = again.to_device()
    x = torch.rand(coo.shape[1], device="cuda")
    y = torch.zeros(coo.shape[0], device="cuda")
    dev.spmv(x, y, 1.0, 0.0)
    torch.cuda.synchronize()
    csr = F.coo2csr(coo)
    y64, sc = __import__("oracle.oracle", fromlist=["x"]).csr_f64(csr, x.cpu().numpy())
    assert np.all(np.abs(y.cpu().numpy() - y64) <= 1e-5 * sc + 1e-30)
    dev.close()


def test_tune_refines_block_part(tmp_path):
    """A partition with a block part: every block shape is tried for it on
    the device, and the tuned (possibly re-shaped) matrix still gives y."""
    from clspmv_mic_b200 import tables as T
    from clspmv_mic_b200.autotune import tune
    import torch
    root = T.model_tables(tmp_path / "t", seed=5, scale={"bcsr": 0.2, "sbell": 2.0, "bell": 1.8})
    coo = F.coo_matrix(*__import__("clspmv_mic_b200.synth", fromlist=["x"]).block_rows(3000, 6, seed=2))
    r = tune(coo, root, cache=tmp_path / "tune.json", reps=3)
    block_parts = [p for p in ("sbell", "bell", "bcsr", "sell") if r.matrix.uses(p)]
    assert block_parts, r.matrix.summary()
    tried = {e["part"]: e for e in r.part_report}
    for p in block_parts:
        assert len(tried[p]["candidates"]) >= 5
    dev = r.matrix.to_device()
    x = torch.rand(coo.shape[1], device="cuda")
    y = torch.zeros(coo.shape[0], device="cuda")
    dev.spmv(x, y, 1.0, 0.0)
    torch.cuda.synchronize()
    csr = F.coo2csr(coo)
    y64, sc = __import__("oracle.oracle", fromlist=["x"]).csr_f64(csr, x.cpu().numpy())
    assert np.all(np.abs(y.cpu().numpy() - y64) <= 1e-5 * sc + 1e-30)
    dev.close()
    again = tune(coo, root, cache=tmp_path / "tune.json")
    assert again.from_cache and again.parts == r.parts
