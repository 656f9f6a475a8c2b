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


def test_serve_small():
    mats = W.serving_matrices(4, rows_lo=2000, rows_hi=20_000, nnz_lo=2e5, nnz_hi=1e6)
    r = W.serve(mats, 1 << 34, n_requests=60, rate=5000.0, k_lo=1, k_hi=8)
    assert r["matrices"] == 4
    assert r["served"]["req_per_s"] > 0 and r["sequential"]["req_per_s"] > 0
    assert r["served"]["p99_ms"] >= r["served"]["p50_ms"]
