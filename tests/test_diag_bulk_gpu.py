"""GPU parity of the bulk-copy DIA / BDIA kernels (clspmv_dia_bulk_spmv_f32,
clspmv_bdia_bulk_spmv_f32: diagonals staged in shared memory by
cp.async.bulk with an mbarrier ring) against the oracle's csr_spmv within the
per-row 1e-5 bound, on every test matrix the diagonal converters accept,
with alpha / beta, a partial last tile, more diagonals than one stage holds
(32) and more than the shared offset table holds, and no wait running out."""
import numpy as np
import pytest

from clspmv_mic_b200 import _abi
from clspmv_mic_b200 import formats as F
from clspmv_mic_b200 import synth
from tests.gpu_util import assert_close, fp64_error, reference_y, run_device
from tests.matrices import cases, coo_of

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def _cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


def _check(coo, host, what, alpha=1.0, beta=1.0, y0=None):
    x = synth.x_vector(coo.shape[1])
    h = coo.shape[0]
    y_init = np.zeros(h, np.float32) if y0 is None else y0
    y = run_device(host, x, y_init, alpha, beta, variant="bulk")
    y_ref, y64, bound = reference_y(coo, x, y0, alpha, beta)
    assert_close(y, y_ref, bound, what)
    assert fp64_error(y, y64, bound) <= 1e-5
    assert F.pipeline_timeouts() == 0


@pytest.mark.parametrize("name", sorted(cases()))
def test_bulk_dia_bdia(name):
    coo = coo_of(name)
    for conv in (F.coo2dia, F.coo2bdia):
        try:
            host = conv(coo, 32)
        except _abi.ClspmvError as e:
            assert e.status == _abi.ERR_REFUSED
            continue
        _check(coo, host, f"bulk {conv.__name__} {name}")


@pytest.mark.parametrize("alpha,beta", [(2.5, -0.5), (1.0, 0.0), (-1.0, 1.0), (0.5, 2.0)])
@pytest.mark.parametrize("fmt", ["dia", "bdia"])
def test_bulk_alpha_beta(fmt, alpha, beta):
    coo = coo_of("stencil9")
    y0 = np.random.default_rng(8).standard_normal(coo.shape[0]).astype(np.float32)
    _check(coo, getattr(F, f"coo2{fmt}")(coo), f"bulk {fmt} a={alpha} b={beta}", alpha, beta, y0)


@pytest.mark.parametrize("ndiag", [33, 70, 1100])
@pytest.mark.parametrize("fmt", ["dia", "bdia"])
def test_bulk_many_diagonals(fmt, ndiag):
    """Diagonals in several stages per tile (33, 70) and past the 1024
    offsets kept in shared memory (1100), over 2,000 rows (a partial last
    tile of 256)."""
    rng = np.random.default_rng(ndiag)
    n = 2000
    if fmt == "dia":   # offsets near the main diagonal (long diagonals: the converter accepts them)
        offs = np.sort(rng.choice(np.arange(-ndiag, ndiag + 1), ndiag, replace=False))
    else:   # bands of up to 40 consecutive offsets with gaps between them
        offs, o = [], -ndiag
        while len(offs) < ndiag:
            w = int(rng.integers(5, 41))
            offs.extend(range(o, o + w))
            o += w + int(rng.integers(1, 4))
        offs = np.array(offs[:ndiag])
    r = np.repeat(np.arange(n), offs.size)
    c = r + np.tile(offs, n)
    keep = (c >= 0) & (c < n)
    r, c = r[keep], c[keep]
    o = np.lexsort((c, r))
    coo = F.coo_matrix(n, n, r[o], c[o], rng.standard_normal(r.size).astype(np.float32))
    host = getattr(F, f"coo2{fmt}")(coo)
    y0 = rng.standard_normal(n).astype(np.float32)
    _check(coo, host, f"bulk {fmt} {offs.size} diagonals", 1.0, 0.5, y0)


def test_bulk_beta_zero_ignores_nan_y():
    coo = coo_of("laplace33")
    x = synth.x_vector(coo.shape[1])
    for host in (F.coo2dia(coo), F.coo2bdia(coo)):
        y = run_device(host, x, np.full(coo.shape[0], np.nan, np.float32), 1.0, 0.0, variant="bulk")
        assert np.isfinite(y).all(), host.fmt
