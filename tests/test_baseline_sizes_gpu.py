"""GPU parity at the benchmark sizes: every format's y = A x on the full
matrices of the benchmark configurations against the oracle's csr_spmv
(FP32, the reference's serial path), per row |y - y_ref| <= 1e-5 sum|a x|,
and against the FP64 oracle (the reference compares every variant's result
after its first launch, src/util.cpp:93-131).

  C1   5-point Laplacian 256 x 256 (65,536 rows, 326,656 nnz), values 4 / -1: every format
  C2a  27-point stencil 128^3 (2,097,152 rows, 55,742,968 nnz): DIA, BDIA, CSR, SELL-32
  C2b  power-law 2^20 rows, Zipf(2.0) lengths to 10,000: CSR (4 kernels), COO, ELL(K) + COO tail, SELL-32
  C2c  500,000 block rows x 8 dense 4x4 blocks (64M nnz): BELL, SBELL, BCSR, CSR
  C3   Cocktail matrix (4M rows: band, 4x4 blocks, power law): the partitioned SpMV

These are the large persistent grids, 10,000-long rows and 64M-entry block
matrices that the small parity tests do not reach."""
import numpy as np
import pytest

from clspmv_mic_b200 import formats as F
from clspmv_mic_b200 import synth
from oracle import oracle as O

pytestmark = pytest.mark.gpu

RTOL = 1e-5


@pytest.fixture(scope="module", autouse=True)
def _cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


class Case:
    """One matrix: COO, host CSR, x, and the oracle's y (FP32 csr_spmv),
    FP64 y and row scale."""

    def __init__(self, arrs):
        import torch
        self.arrs = arrs
        self.coo = F.coo_matrix(*arrs)
        self.csr = F.coo2csr(self.coo)
        self.x = synth.x_vector(arrs[1])
        self.y_ref = O.spmv_port(self.csr, self.x)
        self.y64, self.scale = O.csr_f64(self.csr, self.x)
        self.xd = torch.from_numpy(self.x).cuda()

    def check(self, y, what):
        y = y.astype(np.float64)
        err = np.abs(y - self.y_ref.astype(np.float64))
        bad = np.nonzero(err > RTOL * self.scale + 1e-30)[0]
        assert bad.size == 0, f"{what}: {bad.size} rows outside the 1e-5 bound, first {bad[:5]}"
        with np.errstate(divide="ignore", invalid="ignore"):
            e64 = np.abs(y - self.y64) / np.where(self.scale > 0, self.scale, 1.0)
        assert e64.max() <= RTOL, f"{what}: error against FP64 {e64.max():.3g}"

    def run(self, host, what, parts=(), **kw):
        """y = A x (beta 0) through the C ABI; `parts` are further
        (host, kw) matrices accumulated into the same y (beta 1)."""
        import torch
        y = torch.full((self.coo.shape[0],), 7.0, dtype=torch.float32, device="cuda")   # beta 0 never reads y
        dev = F.DeviceMatrix(host)
        dev.spmv(self.xd, y, 1.0, 0.0, **kw)
        del dev
        for h2, kw2 in parts:
            d2 = F.DeviceMatrix(h2)
            d2.spmv(self.xd, y, 1.0, 1.0, **kw2)
            del d2
        torch.cuda.synchronize()
        self.check(y.cpu().numpy(), what)


_CASES = {}


def case(name):
    if name not in _CASES:
        _CASES.clear()   # one full-size matrix on the host at a time
        gen = {"c1": lambda: synth.laplacian_2d(256), "c2a": lambda: synth.stencil_27pt(128),
               "c2b": lambda: synth.powerlaw(1 << 20), "c2c": lambda: synth.block_rows(500_000, 8)}[name]
        _CASES[name] = Case(gen())
    return _CASES[name]


C1_FORMATS = [("csr", {"variant": v}) for v in ("chunk", "merge", "vector", "scalar")] + \
    [("coo", {}), ("dia", {}), ("bdia", {}), ("ell", {}), ("sell32", {}), ("sell32", {"variant": "planned"}),
     ("b4csr", {}), ("b4ell", {}), ("sbell", {})]


def _convert(c, fmt):
    return {"csr": lambda: c.csr, "coo": lambda: c.coo, "dia": lambda: F.coo2dia(c.coo),
            "bdia": lambda: F.coo2bdia(c.coo), "ell": lambda: F.coo2ell(c.coo),
            "sell32": lambda: F.coo2sell(c.coo, 32), "b4csr": lambda: F.coo2b4csr(c.coo, 4, 4),
            "b4ell": lambda: F.coo2b4ell(c.coo, 4, 4), "sbell": lambda: F.coo2sbell(c.coo, 4, 4, 32)}[fmt]()


@pytest.mark.parametrize("fmt,kw", C1_FORMATS, ids=[f"{f}-{k.get('variant', '')}" for f, k in C1_FORMATS])
def test_c1_laplacian_256(fmt, kw):
    c = case("c1")
    c.run(_convert(c, fmt), f"C1 {fmt} {kw}", **kw)


@pytest.mark.parametrize("fmt,kw", [("dia", {}), ("bdia", {}), ("csr", {"variant": "chunk"}), ("sell32", {})])
def test_c2a_stencil27_128(fmt, kw):
    c = case("c2a")
    c.run(_convert(c, fmt), f"C2a {fmt}", **kw)


@pytest.mark.parametrize("fmt,kw", [("csr", {"variant": "chunk"}), ("csr", {"variant": "merge"}),
                                    ("csr", {"variant": "vector"}), ("csr", {"variant": "scalar"}), ("coo", {}),
                                    ("sell32", {}), ("sell32", {"variant": "planned"})])
def test_c2b_powerlaw(fmt, kw):
    c = case("c2b")
    c.run(_convert(c, fmt), f"C2b {fmt} {kw}", **kw)


def test_c2b_powerlaw_ell_with_coo_tail():
    """ELL(K) of every row's first K entries plus the rest as COO (a full
    ELL of 10,000-long rows overflows the reference's int slot count)."""
    import bench
    c = case("c2b")
    k = bench.hyb_width(np.diff(c.csr.array("csr_row_ptr")))
    head, tail = bench.split_hyb(c.arrs, k)
    c.run(F.coo2ell(F.coo_matrix(*head), 32, k), f"C2b ELL({k}) + COO tail",
          parts=[(F.coo_matrix(*tail), {})])


@pytest.mark.parametrize("fmt", ["b4ell", "sbell", "b4csr", "csr"])
def test_c2c_blocks4x4(fmt):
    c = case("c2c")
    c.run(_convert(c, fmt), f"C2c {fmt}")


def test_c3_cocktail_partitions():
    """The Cocktail matrix under the reference's default knobs (whole matrix
    in SBELL) and with estimate_flat_partial off (SBELL + COO, the partition
    the tuner picks on this matrix), through the Cocktail runtime."""
    import torch
    from clspmv_mic_b200 import cocktail as CK
    _CASES.clear()
    c = Case(synth.cocktail_mixed())
    for flat_partial in (True, False):
        ck = CK.analyze(c.coo, None, 1.0, flat_partial, False)
        dev = ck.to_device()
        y = torch.full((c.coo.shape[0],), 7.0, dtype=torch.float32, device="cuda")
        dev.spmv(c.xd, y, 1.0, 0.0)
        torch.cuda.synchronize()
        c.check(y.cpu().numpy(), f"C3 parts={dev.parts}")
        dev.close()
        del ck
