"""GPU parity: every format kernel, through the C ABI, against the oracle's
csr_spmv (FP32, the reference's serial path) within the per-row bound
|y - y_ref| <= 1e-5 * sum_j |a_ij x_j|. y starts at 0 as in the reference's
drivers (initVectorZero, e.g. src/spmv_dia.cpp:374), plus alpha/beta cases."""
import numpy as np
import pytest

from clspmv_mic_b200 import _abi
from clspmv_mic_b200 import formats as F
from clspmv_mic_b200 import synth
from tests.gpu_util import assert_close, fp64_error, reference_y, run_device
from tests.matrices import cases, coo_of, rect_cases

pytestmark = pytest.mark.gpu

ALL = sorted(cases())
ALL_RECT = sorted({**cases(), **rect_cases()})


@pytest.fixture(scope="module", autouse=True)
def _cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


def _check(coo, host, what, alpha=1.0, beta=1.0, y0=None, **kw):
    x = synth.x_vector(coo.shape[1])
    h = coo.shape[0]
    y_init = np.zeros(h, np.float32) if y0 is None else y0
    y = run_device(host, x, y_init, alpha, beta, **kw)
    y_ref, y64, bound = reference_y(coo, x, y0, alpha, beta)
    assert_close(y, y_ref, bound, what)
    assert fp64_error(y, y64, bound) <= 1e-5
    return y


@pytest.mark.parametrize("name", ALL_RECT)
@pytest.mark.parametrize("variant", ["merge", "chunk", "vector", "scalar"])
def test_csr(name, variant):
    coo = coo_of(name)
    _check(coo, F.coo2csr(coo), f"csr-{variant}", variant=variant)


@pytest.mark.parametrize("name", ["powerlaw3k", "laplace33", "random_empty_rows", "tall"])
@pytest.mark.parametrize("tpr", [1, 2, 4, 8, 16, 32])
def test_csr_vector_lanes(name, tpr):
    coo = coo_of(name)
    _check(coo, F.coo2csr(coo), f"csr-vector-{tpr}", variant="vector", threads_per_row=tpr)


@pytest.mark.parametrize("name", ["powerlaw3k", "laplace33", "random_empty_rows"])
@pytest.mark.parametrize("align,variant", [(4, "scalar"), (16, "vector"), (4, "merge"), (4, "chunk")])
def test_csr_padded(name, align, variant):
    """pad_csr input (the reference's padded CSR drivers) takes the 128-bit path."""
    coo = coo_of(name)
    _check(coo, F.pad_csr(F.coo2csr(coo), align), f"padcsr{align}-{variant}", variant=variant)


@pytest.mark.parametrize("name", ALL_RECT)
def test_coo(name):
    coo = coo_of(name)
    _check(coo, coo, "coo")


@pytest.mark.parametrize("name", ALL)
def test_dia_bdia(name):
    coo = coo_of(name)
    for conv in (F.coo2dia, F.coo2bdia):
        try:
            host = conv(coo, 32)
        except _abi.ClspmvError as e:
            assert e.status == _abi.ERR_REFUSED
            continue
        _check(coo, host, conv.__name__)


@pytest.mark.parametrize("name", ALL_RECT)
def test_ell(name):
    coo = coo_of(name)
    _check(coo, F.coo2ell(coo), "ell")


@pytest.mark.parametrize("name", ALL_RECT)
@pytest.mark.parametrize("sh", [32, 128, 7])
def test_sell(name, sh):
    coo = coo_of(name)
    _check(coo, F.coo2sell(coo, sh), f"sell{sh}")


@pytest.mark.parametrize("name", ["laplace33", "blocks300", "blocks_odd", "random_empty_rows", "wide", "tall", "stencil6"])
@pytest.mark.parametrize("bh,bw", F.BLOCK_SHAPES)
def test_block_formats(name, bh, bw):
    coo = coo_of(name)
    _check(coo, F.coo2b4csr(coo, bw, bh), f"b4csr{bh}x{bw}")
    _check(coo, F.coo2b4ell(coo, bw, bh), f"b4ell{bh}x{bw}")
    _check(coo, F.coo2sbell(coo, bw, bh, 32), f"sbell{bh}x{bw}")


@pytest.mark.parametrize("alpha,beta", [(2.5, -0.5), (1.0, 0.0), (-1.0, 1.0), (0.5, 2.0)])
@pytest.mark.parametrize("fmt", ["csr-merge", "csr-chunk", "csr-vector", "csr-scalar", "coo", "dia", "bdia", "ell", "sell",
                                 "b4csr", "b4ell", "sbell"])
def test_alpha_beta(fmt, alpha, beta):
    coo = coo_of("powerlaw3k" if fmt in ("csr-merge", "csr-chunk", "coo", "ell", "sell") else "stencil9" if "dia" in fmt else
                 "blocks_odd" if fmt[:2] in ("b4", "sb") else "laplace33")
    y0 = np.random.default_rng(8).standard_normal(coo.shape[0]).astype(np.float32)
    kw = {}
    if fmt.startswith("csr"):
        host = F.coo2csr(coo)
        kw["variant"] = fmt.split("-")[1]
    elif fmt == "coo":
        host = coo
    elif fmt in ("b4csr", "b4ell"):
        host = getattr(F, f"coo2{fmt}")(coo, 4, 4)
    elif fmt == "sbell":
        host = F.coo2sbell(coo, 4, 4, 32)
    else:
        host = getattr(F, f"coo2{fmt}")(coo)
    _check(coo, host, f"{fmt} a={alpha} b={beta}", alpha, beta, y0, **kw)


def test_beta_zero_ignores_nan_y():
    """beta == 0 must not read y (BLAS convention)."""
    coo = coo_of("laplace16")
    x = synth.x_vector(coo.shape[1])
    y0 = np.full(coo.shape[0], np.nan, np.float32)
    for host, kw in ((F.coo2csr(coo), {"variant": "merge"}), (F.coo2csr(coo), {"variant": "vector"}),
                     (coo, {}), (F.coo2dia(coo), {}), (F.coo2ell(coo), {})):
        y = run_device(host, x, y0, 1.0, 0.0, **kw)
        assert np.isfinite(y).all(), host.fmt


def test_empty_matrix():
    import torch
    coo = F.coo_matrix(10, 10, [], [], [])
    x = np.ones(10, np.float32)
    y0 = np.arange(10, dtype=np.float32)
    for host, kw in ((F.coo2csr(coo), {"variant": "merge"}), (F.coo2csr(coo), {"variant": "scalar"}),
                     (coo, {}), (F.coo2ell(coo), {}), (F.coo2sell(coo, 32), {})):
        y = run_device(host, x, y0, 1.0, 1.0, **kw)
        assert np.array_equal(y, y0), host.fmt


def test_launch_counter_moves():
    before = F.launch_count()
    coo = coo_of("laplace16")
    run_device(F.coo2csr(coo), synth.x_vector(coo.shape[1]), np.zeros(coo.shape[0], np.float32), variant="merge")
    assert F.launch_count() >= before + 2   # plan + spmv


@pytest.mark.gpu
@pytest.mark.parametrize("sh", [4, 20, 32, 128])
@pytest.mark.parametrize("name", ["powerlaw3k", "random_empty_rows", "explicit_zeros", "one_entry"])
def test_sell_planned_matches_padded(name, sh):
    """SELL read only up to each row's last real entry (heads per thread,
    long tails per warp) equals the padded read and the oracle, with
    explicit zero values inside and at the end of rows and empty rows."""
    if name == "explicit_zeros":
        rng = np.random.default_rng(12)
        h = 301
        lens = rng.integers(0, 120, h)
        lens[::7] = 0
        rows = np.repeat(np.arange(h), lens)
        cols = np.concatenate([np.sort(rng.choice(900, l, replace=False)) for l in lens])
        vals = rng.standard_normal(rows.size).astype(np.float32)
        vals[::5] = 0.0
        coo = F.coo_matrix(h, 900, rows, cols, vals)
    else:
        coo = coo_of(name)
    m, n = coo.shape
    x = synth.x_vector(n, seed=4) * 1e3
    y0 = np.random.default_rng(1).uniform(-1, 1, m).astype(np.float32)
    for alpha, beta in [(1.0, 0.0), (0.5, -1.5)]:
        ref, _, bound = reference_y(coo, x, y0, alpha, beta)
        for variant in ("planned", "padded"):
            y = run_device(F.coo2sell(coo, sh), x, y0, alpha, beta, variant=variant)
            assert_close(y, ref, bound, f"sell{sh} {variant}")
    dev = F.DeviceMatrix(F.coo2sell(coo, sh))
    host = F.coo2sell(coo, sh)                   # kept alive while its array is read
    assert coo.nnz <= dev.sell_plan_entries() <= int(host.array("sell_slice_ptr")[-1])


@pytest.mark.parametrize("rows,lens", [
    (300, "empty_runs"),      # long runs of empty rows inside a chunk
    (5, "one_long"),          # one row spanning many chunks
    (4097, "ones"),           # a chunk spanning 256 rows
])
def test_csr_chunk_row_shapes(rows, lens):
    """The chunked CSR kernel recovers rows from row_ptr: rows that span
    many chunks, chunks that span hundreds of rows, and empty rows."""
    rng = np.random.default_rng(12)
    if lens == "empty_runs":
        ln = np.zeros(rows, int)
        ln[::37] = rng.integers(1, 700, ln[::37].size)
    elif lens == "one_long":
        ln = np.array([0, 3, 5000, 0, 1])
    else:
        ln = np.ones(rows, int)
    w = 6000
    r = np.repeat(np.arange(rows), ln)
    c = np.concatenate([np.sort(rng.choice(w, k, replace=False)) for k in ln if k > 0])
    v = rng.standard_normal(r.size).astype(np.float32)
    coo = F.coo_matrix(rows, w, r, c, v)
    for alpha, beta in [(1.0, 1.0), (0.5, 0.0)]:
        y0 = rng.standard_normal(rows).astype(np.float32)
        _check(coo, F.coo2csr(coo), f"csr-chunk {lens}", alpha, beta, y0, variant="chunk")
