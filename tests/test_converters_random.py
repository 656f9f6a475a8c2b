"""Randomised converter and serial-SpMV parity against the reference's own
templates (compiled from its sources into oracle/_ref), beside the named
matrices of test_converters.py: hypothesis draws small matrices of any
shape — empty rows and columns, a single row or column, widths and heights
that are not multiples of the block or slice sizes, banded, block-clustered
and scattered patterns — and every converter's arrays and scalars must be
byte-identical to the reference's (including the same refusals), and the
oracle's csr_spmv / coo_spmv bit-identical to the reference's."""
import numpy as np
import pytest
from hypothesis import HealthCheck, given, settings
from hypothesis import strategies as st

from clspmv_mic_b200 import _abi
from clspmv_mic_b200 import formats as F
from oracle import oracle as O
from tests.conftest import ref_or_skip
from tests.test_converters import assert_same

SETTINGS = settings(max_examples=40, deadline=None, derandomize=True,
                    suppress_health_check=[HealthCheck.too_slow, HealthCheck.data_too_large])


@st.composite
def coo_matrices(draw):
    h = draw(st.integers(1, 70))
    w = draw(st.integers(1, 70))
    kind = draw(st.sampled_from(["scattered", "banded", "blocks", "rows"]))
    seed = draw(st.integers(0, 2 ** 31 - 1))
    rng = np.random.default_rng(seed)
    if kind == "scattered":
        dens = draw(st.floats(0.0, 0.3))
        mask = rng.random((h, w)) < dens
    elif kind == "banded":
        offs = rng.choice(np.arange(-min(h, w) + 1, max(h, w)), size=min(5, h + w - 1), replace=False)
        r = np.arange(h)[:, None]
        c = np.arange(w)[None, :]
        mask = np.isin(c - r, offs) & (rng.random((h, w)) < 0.95)
    elif kind == "blocks":
        bh, bw = draw(st.sampled_from([(1, 4), (2, 4), (4, 4), (4, 8), (8, 8), (3, 5)]))
        mask = np.zeros((h, w), bool)
        for _ in range(rng.integers(0, 12)):
            r0, c0 = rng.integers(0, h), rng.integers(0, w)
            mask[r0:r0 + bh, c0:c0 + bw] = True
    else:   # a few long rows, the rest empty
        mask = np.zeros((h, w), bool)
        for r in rng.choice(h, size=min(h, 3), replace=False):
            mask[r] = rng.random(w) < 0.8
    rows, cols = np.nonzero(mask)
    vals = rng.standard_normal(rows.size).astype(np.float32)
    vals[vals == 0] = 1.0
    return F.coo_matrix(h, w, rows, cols, vals)


def _rows_past_diagonals(coo, alignment=32):
    """The reference's coo2dia writes row r of every diagonal at index r of an
    aligned(min(w, h)) array: an entry at or below that row overflows it."""
    h, w = coo.shape
    rows = coo.array("coo_row_id")
    return h > w and rows.size > 0 and rows.max() >= -(-w // alignment) * alignment


def _same_or_both_refuse(fmt, mine_fn, ref_args, coo):
    if fmt in ("dia", "bdia") and _rows_past_diagonals(coo):
        # undefined in the reference (writes past its arrays): refused here as a bad argument
        with pytest.raises(_abi.ClspmvError) as e:
            mine_fn()
        assert e.value.status == _abi.ERR_ARG
        return
    if fmt == "bdia" and coo.nnz == 0:
        # the reference reads the first offset of an empty diagonal list and
        # emits one band over no diagonal; here an empty matrix has no bands
        m = mine_fn()
        assert m.scalars()["bdia_band_num"] == 0
        return
    ok, r = O.ref_convert(fmt, coo, *ref_args)
    if not ok:
        with pytest.raises(_abi.ClspmvError) as e:
            mine_fn()
        assert e.value.status == _abi.ERR_REFUSED
        return
    assert_same(fmt, mine_fn(), r)


@SETTINGS
@given(coo=coo_matrices())
def test_row_and_diagonal_formats(coo):
    ref_or_skip()
    ok, r = O.ref_convert("csr", coo)
    assert ok
    assert_same("csr", F.coo2csr(coo), r)
    _same_or_both_refuse("dia", lambda: F.coo2dia(coo, 32), (32,), coo)
    _same_or_both_refuse("bdia", lambda: F.coo2bdia(coo, 32), (32,), coo)
    ok, r = O.ref_convert("ell", coo, 32, 0)
    assert_same("ell", F.coo2ell(coo, 32, 0), r)
    for sh in (32, 4):
        ok, r = O.ref_convert("sell", coo, sh)
        assert_same("sell", F.coo2sell(coo, sh), r)


@SETTINGS
@given(coo=coo_matrices(), shape=st.sampled_from(F.BLOCK_SHAPES))
def test_block_formats(coo, shape):
    ref_or_skip()
    bh, bw = shape
    _same_or_both_refuse("b4csr", lambda: F.coo2b4csr(coo, bw, bh, 32), (bw, bh, 32), coo)
    _same_or_both_refuse("b4ell", lambda: F.coo2b4ell(coo, bw, bh, 32, 0), (bw, bh, 32, 0), coo)
    _same_or_both_refuse("sbell", lambda: F.coo2sbell(coo, bw, bh, 32), (bw, bh, 32), coo)
    ok, r = O.ref_convert("bcsr", coo, bw, bh, 32)
    assert_same("bcsr", F.coo2bcsr(coo, bw, bh, 32), r)


@SETTINGS
@given(coo=coo_matrices(), seed=st.integers(0, 1000))
def test_serial_spmv_matches_reference(coo, seed):
    """The oracle's C restatement of every <fmt>_spmv against the
    reference's own, bit for bit, on the converted arrays (result += A x on
    a random starting result)."""
    ref_or_skip()
    rng = np.random.default_rng(seed)
    x = rng.uniform(-1, 1, coo.shape[1]).astype(np.float32)
    y0 = rng.uniform(-1, 1, coo.shape[0]).astype(np.float32)
    mats = [coo, F.coo2csr(coo), F.coo2ell(coo, 32, 0), F.coo2sell(coo, 32), F.coo2sbell(coo, 4, 4, 32),
            F.coo2bcsr(coo, 4, 4, 32), F.coo2bell(coo, 4, 2, 32, 0)]
    for fmt, fn in (("dia", lambda: F.coo2dia(coo, 32)), ("bdia", lambda: F.coo2bdia(coo, 32))):
        if fmt == "bdia" and coo.nnz == 0:
            continue   # no bands here, a band over no diagonal in the reference (see above)
        try:
            mats.append(fn())
        except _abi.ClspmvError:
            pass
    for m in mats:
        mine = O.spmv_port(m, x, y0)
        theirs = O.spmv_ref(m, x, y0)
        assert np.array_equal(mine.view(np.uint32), theirs.view(np.uint32)), m.fmt


@SETTINGS
@given(coo=coo_matrices())
def test_inverse_converters_match_reference(coo):
    """<fmt>2coo of the library against the reference's inverse on the same
    converted arrays. The reference's dia2coo / bdia2coo keep only columns
    below dia_length (= min(width, height)), so a wider-than-tall matrix
    loses the entries right of column `height`; the reference then reports
    the source's nnz with those slots left uninitialised, while here nnz is
    the number of entries written. The entries written are the same."""
    L = ref_or_skip()
    import ctypes as C
    h, w = coo.shape
    for fmt, args in [("dia", (32,)), ("bdia", (32,)), ("ell", (32, 0)), ("bcsr", (4, 4, 32)), ("bcsr", (2, 8, 32)),
                      ("bell", (4, 2, 32, 0)), ("bell", (1, 4, 32, 0))]:
        try:
            m = getattr(F, f"coo2{fmt}")(coo, *args)
        except _abi.ClspmvError:
            continue
        mine = F.to_coo(m)
        out = _abi.Coo()
        getattr(L, f"ref_{fmt}2coo")(C.byref(m.struct), C.byref(out))
        theirs = O.RefMatrix("coo", out)
        theirs._ref_owned = True
        n = mine.nnz
        for f in ("coo_row_id", "coo_col_id", "coo_data"):
            assert np.array_equal(mine.array(f)[:n], theirs.array(f)[:n]), (fmt, args, f)
        if fmt in ("dia", "bdia") and w > h:
            assert n <= theirs.nnz and np.all(mine.array("coo_col_id") < h)
        else:
            assert mine.scalars() == theirs.scalars(), (fmt, args)


@SETTINGS
@given(h=st.integers(1, 60), w=st.integers(1, 60), n=st.integers(0, 400), seed=st.integers(0, 10 ** 6))
def test_sort_coo_matches_reference_without_duplicates(h, w, n, seed):
    """sort_coo on shuffled duplicate-free input: the same arrays as the
    reference's quicksort (any order of distinct keys sorts to one result)."""
    L = ref_or_skip()
    import ctypes as C
    rng = np.random.default_rng(seed)
    keys = rng.permutation(np.unique(rng.integers(0, h * w, n)))
    r, c = keys // w, keys % w
    v = rng.standard_normal(keys.size).astype(np.float32)
    a = F.coo_matrix(h, w, r, c, v)
    b = a.copy()
    F.sort_coo(a)
    assert L.ref_sort_coo(C.byref(b.struct)) == 1
    for f in ("coo_row_id", "coo_col_id", "coo_data"):
        assert np.array_equal(a.array(f).view(np.uint32), b.array(f).view(np.uint32))


def test_sort_coo_is_stable_on_repeated_keys():
    """Repeated (row, col) keys, outside the COO contract of both libraries,
    keep their input order here (the device sort does the same); the
    reference's quicksort leaves them in an order set by its pivoting."""
    rng = np.random.default_rng(5)
    r = rng.integers(0, 6, 200)
    c = rng.integers(0, 5, 200)
    v = np.arange(1, 201, dtype=np.float32)   # input position, to check the order of equal keys
    order = np.lexsort((np.arange(200), c, r))   # by key, then by input position
    a = F.coo_matrix(6, 5, r.copy(), c.copy(), v.copy())   # sorted in place
    F.sort_coo(a)
    assert np.array_equal(a.array("coo_data"), v[order])


@SETTINGS
@given(coo=coo_matrices(), align=st.sampled_from([1, 2, 4, 16, 32]))
def test_pad_csr_matches_reference(coo, align):
    """pad_csr (src/util.cpp:31-72) against the reference's. A matrix without
    nonzeros is not given to the reference, whose pad_csr crashes on it
    (segmentation fault); here it pads to an empty CSR with zero row lengths."""
    L = ref_or_skip()
    import ctypes as C
    csr = F.coo2csr(coo)
    mine = F.pad_csr(csr, align)
    if coo.nnz == 0:
        assert mine.nnz == 0 and not np.any(mine.array("csr_row_ptr"))
        return
    out = _abi.Csr()
    L.ref_pad_csr(C.byref(csr.struct), C.byref(out), align)
    theirs = O.RefMatrix("csr", out)
    theirs._ref_owned = True
    assert_same("csr", mine, theirs)
