"""Converters on the device (clspmv_device_coo2<fmt>_f32) against the host
converters, which the converter tests pin to the reference's own templates:
every array byte for byte, every scalar, and the same status on the inputs
the host converters reject or refuse (unsorted COO, ids outside the matrix,
unsupported block shapes, the DIA padding rule, ELL / b4ell / BELL widths,
the MAX_MEM_OBJ caps), for the eight GPU formats and the generic BCSR / BELL
of any block shape. Plus the device sort against the host's stable sort."""
import ctypes as C

import numpy as np
import pytest

from clspmv_mic_b200 import _abi
from clspmv_mic_b200 import formats as F
from clspmv_mic_b200 import synth
from tests.matrices import cases, coo_of, rect_cases

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")

ALL = sorted(cases())
ALL_RECT = sorted({**cases(), **rect_cases()})
WIDE_OK = [n for n in ALL_RECT if n != "tall"]   # "tall" has entries below row aligned(width): DIA / BDIA reject it
BLOCK = [(4, 4), (8, 2), (4, 1), (8, 8)]          # (bwidth, bheight)

_HOST_DEFAULTS = {
    "csr": (0, ()), "dia": (0, (32,)), "bdia": (0, (32,)), "ell": (0, (32, 0)), "sell": (0, (32,)),
    "b4csr": (2, (32,)), "b4ell": (2, (32, 0)), "sbell": (2, (32,)),
    "bcsr": (2, (32,)), "bell": (2, (32, 0)),
}
GENERIC = [(4, 4), (1, 1), (3, 2), (2, 5), (8, 8), (7, 3)]     # (bwidth, bheight): any shape


@pytest.fixture(scope="module", autouse=True)
def _cuda():
    if not torch.cuda.is_available():
        pytest.skip("needs a GPU")


def host_raw(fmt, coo, *args):
    required, defaults = _HOST_DEFAULTS[fmt]
    full = tuple(args) + defaults[len(args) - required:]
    out = _abi.FORMATS[fmt][0]()
    status = getattr(F.lib(), f"clspmv_coo2{fmt}_f32")(C.byref(coo.struct), C.byref(out), *full)
    return status, F.HostMatrix(fmt, out, lib_owned=(status == _abi.OK))


def device_coo(coo):
    return F.DeviceMatrix(coo)


def assert_same(fmt, dev, host):
    got = F.HostMatrix(fmt, dev.struct).scalars()
    assert got == host.scalars(), fmt
    for field, _, _ in _abi.FORMATS[fmt][1]:
        a = dev.tensors[field].cpu().numpy()
        b = host.array(field)
        assert a.shape == b.shape, f"{fmt}.{field}: {a.shape} != {b.shape}"
        assert np.array_equal(a.view(np.uint32), b.view(np.uint32)), f"{fmt}.{field} differs"


def check_pair(fmt, coo, *args):
    st_h, host = host_raw(fmt, coo, *args)
    st_d, out = F.device_convert_raw(device_coo(coo), fmt, *args)
    assert st_d == st_h, (fmt, args, st_d, st_h)
    if st_h == _abi.OK:
        getattr(F.lib(), f"clspmv_device_free_{fmt}_f32")(C.byref(out))
        dev = F.device_convert(device_coo(coo), fmt, *args)
        assert_same(fmt, dev, host)
    return st_h


@pytest.mark.parametrize("name", ALL_RECT)
@pytest.mark.parametrize("fmt", ["csr", "ell", "sell"])
def test_flat_formats(name, fmt):
    assert check_pair(fmt, coo_of(name)) == _abi.OK


@pytest.mark.parametrize("name", ["powerlaw3k", "random_empty_rows", "ragged_tail", "tall", "one_entry"])
@pytest.mark.parametrize("sh", [1, 4, 7, 128])
def test_sell_slice_heights(name, sh):
    assert check_pair("sell", coo_of(name), sh) == _abi.OK


@pytest.mark.parametrize("name", WIDE_OK)
@pytest.mark.parametrize("fmt", ["dia", "bdia"])
def test_diagonal_formats(name, fmt):
    check_pair(fmt, coo_of(name))   # accepted or refused alike


@pytest.mark.parametrize("name", ["stencil6", "banded7", "laplace33"])
@pytest.mark.parametrize("align", [1, 8, 64])
def test_dia_alignments(name, align):
    assert check_pair("dia", coo_of(name), align) == _abi.OK
    assert check_pair("bdia", coo_of(name), align) == _abi.OK


def test_dia_refusal_keeps_count():
    coo = coo_of("random_sparse")
    st_h, host = host_raw("dia", coo)
    st_d, out = F.device_convert_raw(device_coo(coo), "dia")
    assert st_h == st_d == _abi.ERR_REFUSED
    assert (out.dia_num, out.dia_length, out.dia_length_aligned) == (
        host.struct.dia_num, host.struct.dia_length, host.struct.dia_length_aligned)


@pytest.mark.parametrize("name", ALL_RECT)
@pytest.mark.parametrize("fmt", ["b4csr", "b4ell", "sbell"])
@pytest.mark.parametrize("shape", BLOCK)
def test_block_formats(name, fmt, shape):
    bw, bh = shape
    check_pair(fmt, coo_of(name), bw, bh)


@pytest.mark.parametrize("name", ALL_RECT)
@pytest.mark.parametrize("fmt", ["bcsr", "bell"])
@pytest.mark.parametrize("shape", GENERIC)
def test_generic_block_formats(name, fmt, shape):
    """The generic BCSR / BELL of any block shape (the layouts only the
    serial bcsr_spmv / bell_spmv read) equal the host converters' arrays."""
    bw, bh = shape
    assert check_pair(fmt, coo_of(name), bw, bh) == _abi.OK


@pytest.mark.parametrize("fmt,args", [("bcsr", (3, 2, 1)), ("bcsr", (4, 4, 7)), ("bell", (3, 2, 1, 0)),
                                      ("bell", (4, 4, 32, 1)), ("bell", (4, 4, 32, 40)), ("bell", (5, 1, 5, 0)),
                                      ("bcsr", (0, 4)), ("bell", (4, 0)), ("bell", (4, 4, 32, -1))])
def test_generic_block_arguments(fmt, args):
    """Alignments, ellnum (too small: CLSPMV_ERR_ARG on both sides) and zero
    block dimensions (CLSPMV_ERR_ARG)."""
    check_pair(fmt, coo_of("powerlaw3k"), *args)


def test_generic_bell_too_few_slots_rejected():
    assert check_pair("bell", coo_of("blocks300"), 4, 4, 32, 1) == _abi.ERR_ARG


@pytest.mark.parametrize("fmt", ["bcsr", "bell"])
def test_generic_block_upload_roundtrip(fmt):
    """clspmv_upload_<fmt>_f32 of the host arrays holds what the device
    converter makes."""
    coo = coo_of("blocks_odd")
    host = getattr(F, f"coo2{fmt}")(coo, 3, 2)
    up = F.DeviceMatrix(host)
    dev = F.device_convert(device_coo(coo), fmt, 3, 2)
    for field, _, _ in _abi.FORMATS[fmt][1]:
        a, b = up.tensors[field].cpu().numpy(), dev.tensors[field].cpu().numpy()
        assert np.array_equal(a.view(np.uint32), b.view(np.uint32)), field
    with pytest.raises(ValueError):
        dev.spmv(torch.zeros(coo.shape[1], device="cuda"), torch.zeros(coo.shape[0], device="cuda"))


@pytest.mark.parametrize("sh", [1, 3, 32])
def test_sbell_slice_heights(sh):
    assert check_pair("sbell", coo_of("blocks_odd"), 4, 4, sh) == _abi.OK
    assert check_pair("sbell", coo_of("powerlaw3k"), 8, 2, sh) == _abi.OK


@pytest.mark.parametrize("fmt,args", [("ell", (32, 3)), ("ell", (32, 600)), ("ell", (7, 0)),
                                      ("b4ell", (4, 4, 32, 1)), ("b4ell", (4, 4, 32, 40)), ("b4ell", (8, 1, 5, 0))])
def test_width_arguments(fmt, args):
    check_pair(fmt, coo_of("powerlaw3k"), *args)


def test_block_cap_refusal():
    """More 8x8 blocks than MAX_MEM_OBJ / 256 B: b4csr, b4ell and sbell refuse."""
    h, w = 8 * 8300, 8 * 1100
    nb_row = 128                  # 8300 * 128 = 1,062,400 blocks > 2^28 / 256 = 1,048,576
    rng = np.random.default_rng(5)
    rows, cols = [], []
    for br in range(h // 8):
        bc = np.sort(rng.choice(w // 8, nb_row, replace=False))
        rows.append(np.full(nb_row, br * 8))
        cols.append(bc * 8)
    r, c = np.concatenate(rows), np.concatenate(cols)
    coo = F.coo_matrix(h, w, r, c, np.ones(r.size, np.float32))
    for fmt in ("b4csr", "b4ell", "sbell"):
        assert check_pair(fmt, coo, 8, 8) == _abi.ERR_REFUSED


def _with_duplicates(name, seed=0):
    h, w, r, c, v = {**cases(), **rect_cases()}[name]
    r, c, v = np.asarray(r), np.asarray(c), np.asarray(v, np.float32)
    rng = np.random.default_rng(seed)
    pick = rng.choice(r.size, size=max(1, r.size // 10), replace=False)
    r2, c2 = np.r_[r, r[pick]], np.r_[c, c[pick]]
    v2 = np.r_[v, (v[pick] + 100).astype(np.float32)]
    order = np.lexsort((c2, r2))          # stable: the originals first, then their repeats
    return h, w, r2, c2, v2, order


@pytest.mark.parametrize("fmt,args", [("csr", ()), ("ell", ()), ("sell", ()), ("dia", ()),
                                      ("b4csr", (4, 4)), ("b4ell", (8, 2)), ("sbell", (4, 2)),
                                      ("bcsr", (3, 2)), ("bell", (2, 3))])
def test_repeated_entries_keep_last(fmt, args):
    h, w, r, c, v, order = _with_duplicates("banded7" if fmt == "dia" else "blocks_odd")
    coo = F.coo_matrix(h, w, r[order], c[order], v[order])
    assert check_pair(fmt, coo, *args) == _abi.OK


@pytest.mark.parametrize("name", ["stencil6", "banded7", "random_empty_rows"])
def test_dia_unsorted_input(name):
    """DIA takes any COO order; a repeated (row, col) keeps its last value in COO order."""
    h, w, r, c, v, _ = _with_duplicates(name, seed=3)
    perm = np.random.default_rng(4).permutation(r.size)
    coo = F.coo_matrix(h, w, r[perm], c[perm], v[perm])
    check_pair("dia", coo)
    check_pair("bdia", coo)


@pytest.mark.parametrize("fmt,args", [("csr", ()), ("ell", ()), ("sell", ()), ("b4csr", (4, 4)),
                                      ("b4ell", (4, 4)), ("sbell", (4, 4)), ("bcsr", (3, 3)), ("bell", (4, 4))])
def test_unsorted_rejected(fmt, args):
    h, w, r, c, v = cases()["random_sparse"]
    perm = np.random.default_rng(1).permutation(len(r))
    coo = F.coo_matrix(h, w, np.asarray(r)[perm], np.asarray(c)[perm], np.asarray(v)[perm])
    assert check_pair(fmt, coo, *args) == _abi.ERR_NOT_SORTED


@pytest.mark.parametrize("fmt,args", [("csr", ()), ("dia", ()), ("sell", ()), ("b4csr", (4, 4)), ("bcsr", (2, 2)),
                                      ("bell", (2, 2))])
def test_out_of_range_rejected(fmt, args):
    coo = F.coo_matrix(10, 10, [0, 3, 10], [1, 2, 3], [1.0, 2.0, 3.0])
    assert check_pair(fmt, coo, *args) == _abi.ERR_ARG


@pytest.mark.parametrize("fmt,args", [("b4csr", (2, 4)), ("b4ell", (4, 3)), ("sbell", (16, 1))])
def test_block_shape_unsupported(fmt, args):
    assert check_pair(fmt, coo_of("blocks_odd"), *args) == _abi.ERR_UNSUPPORTED


def test_tall_dia_rejected():
    assert check_pair("dia", coo_of("tall")) == _abi.ERR_ARG


@pytest.mark.parametrize("fmt", ["dia", "bdia"])
@pytest.mark.parametrize("h,w,top", [(300, 100, 128), (300, 100, 140), (129, 97, 97), (64, 30, 32), (500, 37, 64),
                                     (500, 37, 65)])
def test_tall_dia_with_entries_above_the_aligned_width(fmt, h, w, top):
    """A taller-than-wide matrix (a 7-diagonal band in rows < top) converts
    exactly as on the host (and as by the reference) while every entry sits
    in a row below aligned(width, 32), and both reject it (CLSPMV_ERR_ARG)
    when an entry sits at or past it."""
    rng = np.random.default_rng(h * 7 + w)
    r = np.repeat(np.arange(min(top, h)), 7)
    c = r + np.tile(np.arange(-3, 4), min(top, h))
    keep = (c >= 0) & (c < w)
    r, c = list(r[keep]), list(c[keep])
    if top - 1 >= w:                      # one entry in the rows below the square part, at row top - 1
        r.append(top - 1)
        c.append(0)
    r, c = np.array(r), np.array(c)
    coo = F.coo_matrix(h, w, r, c, rng.standard_normal(r.size).astype(np.float32))
    aligned = (w + 31) // 32 * 32
    st = check_pair(fmt, coo)
    assert st == (_abi.ERR_ARG if r.max() >= aligned else _abi.OK), (st, r.max(), aligned)


def test_empty_matrix():
    coo = F.coo_matrix(37, 41, np.zeros(0, int), np.zeros(0, int), np.zeros(0, np.float32))
    for fmt, args in [("csr", ()), ("ell", ()), ("sell", ()), ("dia", ()), ("bdia", ()),
                      ("b4csr", (4, 4)), ("b4ell", (4, 4)), ("sbell", (4, 4)), ("bcsr", (3, 5)), ("bell", (3, 5))]:
        check_pair(fmt, coo, *args)


@pytest.mark.parametrize("seed", [0, 1])
def test_device_sort_matches_host_stable_sort(seed):
    h, w, r, c, v, _ = _with_duplicates("random_empty_rows", seed=seed)
    perm = np.random.default_rng(seed + 10).permutation(r.size)
    host = F.coo_matrix(h, w, r[perm], c[perm], v[perm])
    dev = F.DeviceMatrix(host)
    F.device_sort_coo(dev)
    F.sort_coo(host)
    for field in ("coo_row_id", "coo_col_id", "coo_data"):
        assert np.array_equal(dev.tensors[field].cpu().numpy().view(np.uint32), host.array(field).view(np.uint32))


def test_large_powerlaw_and_blocks():
    """Sizes where the device work spans many blocks (about 1M entries)."""
    coo = F.coo_matrix(*synth.powerlaw(1 << 16, maxlen=4000, seed=2))
    for fmt, args in [("csr", ()), ("sell", ()), ("ell", ())]:
        assert check_pair(fmt, coo, *args) == _abi.OK
    blk = F.coo_matrix(*synth.block_rows(20000, 8, 4, 4, seed=3))
    for fmt, args in [("b4csr", (4, 4)), ("b4ell", (4, 4)), ("sbell", (4, 4)), ("b4csr", (8, 2))]:
        assert check_pair(fmt, blk, *args) == _abi.OK
    st = F.coo_matrix(*synth.stencil_27pt(24))
    assert check_pair("dia", st) == _abi.OK
    assert check_pair("bdia", st) == _abi.OK


def test_converted_matrix_runs():
    """A device-converted SELL runs through the SpMV entry point like an uploaded one."""
    coo = coo_of("powerlaw3k")
    dev = F.device_convert(device_coo(coo), "sell")
    up = F.DeviceMatrix(F.coo2sell(coo))
    x = torch.randn(coo.shape[1], device="cuda")
    y1 = torch.ones(coo.shape[0], device="cuda")
    y2 = y1.clone()
    dev.spmv(x, y1)
    up.spmv(x, y2)
    torch.cuda.synchronize()
    # the column-balanced SELL kernel adds shared slices with atomics, so two
    # runs may differ in summation order only
    assert torch.allclose(y1, y2, rtol=1e-5, atol=1e-5)
