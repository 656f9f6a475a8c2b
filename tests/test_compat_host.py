"""The reference-compatible host surface, without a GPU.

* every function include/clspmv_b200.h declares is exported by the library;
* ReadMMF / clspmv_read_mmf_f32 reads Matrix Market files exactly as the
  reference's src/fileio.cpp:10-109 (checked against it compiled from its
  own sources), including pattern and symmetric files, and rejects what it
  cannot read with a status;
* a C++ caller written against the compat headers (tests/compat/
  serial_check.cpp) compiles, links every compat entry point, and its host
  serial templates (include/spmv_serial.h) give the reference's results
  bit for bit.
"""
import ctypes as C
import re
import shutil
import subprocess

import numpy as np
import pytest

from clspmv_mic_b200 import _abi
from clspmv_mic_b200 import formats as F
from clspmv_mic_b200.drivers import read_mmf
from oracle import oracle as O

from conftest import ROOT, ref_or_skip
from matrices import cases


def header_functions():
    text = (ROOT / "include" / "clspmv_b200.h").read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(clspmv_\w+)\s*\(", text)))


def test_library_exports_every_header_function():
    names = header_functions()
    assert len(names) >= 80
    L = C.CDLL(str(_abi.LIB_PATH))
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing


def write_mtx(path, h, w, rows, cols, vals, field="real", symmetry="general", comments=("a comment",), order=None):
    rows, cols, vals = np.asarray(rows), np.asarray(cols), np.asarray(vals, dtype=np.float64)
    idx = np.arange(rows.size) if order is None else order
    with open(path, "w") as f:
        f.write(f"%%MatrixMarket matrix coordinate {field} {symmetry}\n")
        for c in comments:
            f.write(f"% {c}\n")
        f.write(f"{h} {w} {rows.size}\n")
        for i in idx:
            if field == "pattern":
                f.write(f"{rows[i] + 1} {cols[i] + 1}\n")
            else:
                f.write(f"{rows[i] + 1} {cols[i] + 1} {float(vals[i])!r}\n")


def ref_read(path):
    L = ref_or_skip()
    out = _abi.Coo()
    L.ref_read_mmf(str(path).encode(), C.byref(out))
    m = O.RefMatrix("coo", out)
    m._ref_owned = True
    return m


def assert_same_coo(a, b):
    assert a.scalars() == b.scalars()
    for k in ("coo_row_id", "coo_col_id", "coo_data"):
        np.testing.assert_array_equal(a.array(k), b.array(k), err_msg=k)


@pytest.mark.parametrize("kind", ["general_unsorted", "pattern", "symmetric", "symmetric_pattern", "rect"])
def test_read_mmf_matches_reference(tmp_path, kind):
    rng = np.random.default_rng(3)
    if kind == "rect":
        h, w, r, c, v = cases()["random_sparse"]
        w = w + 17
    else:
        h, w, r, c, v = cases()["random_empty_rows"]
    r, c, v = np.asarray(r), np.asarray(c), np.asarray(v)
    if kind.startswith("symmetric"):
        keep = r >= c                     # lower triangle with the diagonal
        r, c, v = r[keep], c[keep], v[keep]
        diag = np.arange(0, min(h, w), 5)
        extra = ~np.isin(diag, r[r == c])
        r, c, v = np.r_[r, diag[extra]], np.r_[c, diag[extra]], np.r_[v, np.full(extra.sum(), 2.5)]
    field = "pattern" if "pattern" in kind else "real"
    symmetry = "symmetric" if kind.startswith("symmetric") else "general"
    order = rng.permutation(r.size) if kind != "rect" else None
    p = tmp_path / f"{kind}.mtx"
    write_mtx(p, h, w, r, c, v, field=field, symmetry=symmetry, order=order, comments=("one", "two  words", ""))
    ours = read_mmf(p)
    assert F.if_sorted_coo(ours)
    assert_same_coo(ours, ref_read(p))


def test_read_mmf_values_and_expansion(tmp_path):
    p = tmp_path / "s.mtx"
    write_mtx(p, 3, 3, [0, 2, 1], [0, 0, 1], [1.5, -2.0, 4.0], symmetry="symmetric")
    m = read_mmf(p)
    a = m.arrays()
    assert m.shape == (3, 3) and m.nnz == 4
    assert a["coo_row_id"].tolist() == [0, 0, 1, 2]
    assert a["coo_col_id"].tolist() == [0, 2, 1, 0]
    assert a["coo_data"].tolist() == [1.5, -2.0, 4.0, -2.0]


@pytest.mark.parametrize("body,status", [
    ("%%MatrixMarket matrix coordinate complex general\n2 2 1\n1 1 1.0 0.0\n", _abi.ERR_UNSUPPORTED),
    ("%%MatrixMarket matrix array real general\n2 2\n1\n2\n3\n4\n", _abi.ERR_UNSUPPORTED),
    ("%%MatrixMarket matrix coordinate real general\n2 2 1\n3 1 1.0\n", _abi.ERR_ARG),
    ("%%MatrixMarket matrix coordinate real general\n2 2 2\n1 1 1.0\n", _abi.ERR_ARG),
    ("%%MatrixMarket matrix coordinate real general\n", _abi.ERR_ARG),
])
def test_read_mmf_rejects(tmp_path, body, status):
    p = tmp_path / "bad.mtx"
    p.write_text(body)
    with pytest.raises(_abi.ClspmvError) as e:
        read_mmf(p)
    assert e.value.status == status


def test_read_mmf_missing_file(tmp_path):
    with pytest.raises(_abi.ClspmvError) as e:
        read_mmf(tmp_path / "nope.mtx")
    assert e.value.status == _abi.ERR_ARG


def _compile_check(tmp_path):
    if shutil.which("g++") is None:
        pytest.skip("g++ not available")
    exe = tmp_path / "serial_check"
    libdir = _abi.LIB_PATH.parent
    cmd = ["g++", "-O2", "-std=c++17", "-ffp-contract=off", "-I", str(ROOT / "include"),
           str(ROOT / "tests" / "compat" / "serial_check.cpp"), "-L", str(libdir), "-lclspmv_b200",
           f"-Wl,-rpath,{libdir}", "-o", str(exe)]
    res = subprocess.run(cmd, capture_output=True, text=True)
    assert res.returncode == 0, res.stderr
    return exe


def _read_outputs(path, h):
    raw = path.read_bytes()
    out, off = {}, 0
    while off < len(raw):
        name = raw[off:off + 16].split(b"\0")[0].decode()
        off += 16
        out[name] = np.frombuffer(raw[off:off + 4 * h], dtype=np.float32)
        off += 4 * h
    return out


# format -> (converter arguments, result length from the converted struct)
_SERIAL = {
    "csr": ((), lambda s: s.matinfo.height),
    "dia": ((32,), lambda s: s.dia_length_aligned),
    "bdia": ((32,), lambda s: s.bdia_length_aligned),
    "ell": ((32, 0), lambda s: s.matinfo.height),
    "sell": ((32,), lambda s: s.matinfo.height),
    "sbell": ((4, 2, 32), lambda s: s.matinfo.height),
    "bcsr": ((4, 4, 32), lambda s: s.bcsr_row_num * 4),
    "bell": ((4, 2, 32, 0), lambda s: s.bell_row_num * 2),
}


@pytest.mark.parametrize("name", ["laplace33", "stencil6", "powerlaw3k", "blocks_odd", "random_empty_rows"])
def test_cpp_compat_serial_templates_match_reference(tmp_path, name):
    exe = _compile_check(tmp_path)
    _check_serial_program(exe, tmp_path, name, *cases()[name])


def test_cpp_compat_serial_templates_random(tmp_path):
    """The same program on seeded random matrices of every shape (square,
    wide, tall, single row or column, empty rows): each format the headers
    convert gives the reference's serial result bit for bit."""
    ref_or_skip()
    exe = _compile_check(tmp_path)
    for it in range(24):
        rng = np.random.default_rng(100 + it)
        h, w = int(rng.integers(1, 90)), int(rng.integers(1, 90))
        mask = rng.random((h, w)) < rng.uniform(0.01, 0.3)
        mask[int(rng.integers(h)), int(rng.integers(w))] = True   # at least one nonzero
        r, c = np.nonzero(mask)
        v = rng.standard_normal(r.size).astype(np.float32)
        _check_serial_program(exe, tmp_path, f"r{it}", h, w, r, c, v, require=("coo", "csr"))


def _check_serial_program(exe, tmp_path, name, h, w, r, c, v, require=("coo", "csr", "sell", "bcsr")):
    p = tmp_path / f"{name}.mtx"
    write_mtx(p, h, w, r, c, v)
    out = tmp_path / "y.bin"
    res = subprocess.run([str(exe), str(p), str(out)], capture_output=True, text=True)
    assert res.returncode == 0, res.stdout + res.stderr
    assert "MatInfo: Width" in res.stdout and "Correctness Check" in res.stdout
    got = _read_outputs(out, h)
    coo = read_mmf(p)
    x = ((np.arange(w) * 7) % 13 - 6).astype(np.float32) * np.float32(0.375)
    use_ref = O.ref() is not None
    expect_coo = (O.spmv_ref if use_ref else O.spmv_port)(coo, x)
    np.testing.assert_array_equal(got["coo"], expect_coo)
    checked = ["coo"]
    for fmt, (args, out_len) in _SERIAL.items():
        if fmt not in got:
            continue
        if use_ref:
            ok, m = O.ref_convert(fmt, coo, *args)
            assert ok
            y = O.spmv_ref(m, x, out_len=out_len(m.struct))
        else:
            m = getattr(F, f"coo2{fmt}")(coo, *args)
            y = O.spmv_port(m, x, out_len=out_len(m.struct))
        want = np.zeros(h, np.float32)   # a diagonal format of a tall matrix has fewer than h rows
        want[:min(h, y.size)] = y[:h]
        np.testing.assert_array_equal(got[fmt], want, err_msg=fmt)
        checked.append(fmt)
    assert set(require) <= set(checked)


def test_read_mmf_random_files_match_reference(tmp_path):
    """Seeded random MatrixMarket files (general and symmetric, real and
    pattern, shuffled entry order, values at several magnitudes and printed
    precisions, 0-2 comment lines): identical COO to the reference's ReadMMF."""
    ref_or_skip()
    for it in range(60):
        rng = np.random.default_rng(it)
        h, w = int(rng.integers(1, 40)), int(rng.integers(1, 40))
        sym = bool(rng.random() < 0.4)
        if sym:
            w = h
        mask = rng.random((h, w)) < rng.uniform(0, 0.3)
        if sym:
            mask = np.tril(mask)
        r, c = np.nonzero(mask)
        v = np.round(rng.standard_normal(r.size) * 10.0 ** int(rng.integers(-3, 4)), int(rng.integers(0, 6)))
        field = "pattern" if rng.random() < 0.25 else "real"
        p = tmp_path / f"m{it}.mtx"
        write_mtx(p, h, w, r, c, v, field=field, symmetry="symmetric" if sym else "general",
                  order=rng.permutation(r.size), comments=tuple(["c"] * int(rng.integers(0, 3))))
        assert_same_coo(read_mmf(p), ref_read(p))


@pytest.mark.parametrize("h,w", [(7, 19), (19, 7), (1, 40)])
def test_read_mmf_nonsquare_symmetric_matches_reference(tmp_path, h, w):
    """A 'symmetric' file that is not square, with entries above the
    diagonal: each mirrored entry takes its column as its row, which reaches
    past the declared height when width > height. Read without writing out
    of bounds, and sorted into the same COO as the reference's ReadMMF."""
    ref_or_skip()
    rng = np.random.default_rng(h * 100 + w)
    mask = np.triu(rng.random((h, w)) < 0.4, k=1)      # strictly above the diagonal: no mirrored duplicates
    d = np.arange(0, min(h, w), 3)
    mask[d, d] = True                                  # some diagonal entries (not mirrored)
    r, c = np.nonzero(mask)
    v = np.round(rng.standard_normal(r.size), 3)
    p = tmp_path / "nonsquare_sym.mtx"
    write_mtx(p, h, w, r, c, v, symmetry="symmetric", order=rng.permutation(r.size))
    ours = read_mmf(p)
    assert ours.nnz == r.size + int((r != c).sum())
    assert_same_coo(ours, ref_read(p))


@pytest.mark.parametrize("field,symmetry", [("real", "general"), ("pattern", "general"), ("real", "symmetric")])
def test_read_mmf_large_files_match_reference(tmp_path, field, symmetry):
    """Files of several MB, so the entry text is cut into ranges parsed on
    separate threads, with irregular whitespace (tabs, runs of blanks, CRLF
    line ends, entries split over lines) and shuffled entries: the same COO
    as the reference's ReadMMF."""
    ref_or_skip()
    rng = np.random.default_rng(7)
    n = 3000
    m = 250_000
    r = rng.integers(0, n, m)
    c = rng.integers(0, n, m)
    if symmetry == "symmetric":
        r, c = np.maximum(r, c), np.minimum(r, c)
    key = np.unique(r.astype(np.int64) * n + c)
    key = key[rng.permutation(key.size)]
    r, c = key // n, key % n
    v = rng.standard_normal(key.size) * 10.0 ** rng.integers(-4, 5, key.size)
    seps = [" ", "\t", "   ", " \t "]
    ends = ["\n", "\r\n", "\n\n"]
    parts = [f"%%MatrixMarket matrix coordinate {field} {symmetry}\n% generated\n{n} {n} {key.size}\n"]
    for i in range(key.size):
        s1, s2 = seps[i % 4], seps[(i // 4) % 4]
        tail = "" if field == "pattern" else f"{s2}{v[i]:.8g}"
        split = "\n" if i % 997 == 0 else s1   # now and then an entry over two lines
        parts.append(f"{r[i] + 1}{split}{c[i] + 1}{tail}{ends[i % 3]}")
    p = tmp_path / "big.mtx"
    p.write_bytes("".join(parts).encode())
    assert p.stat().st_size > 2_500_000   # at least three 1 MB ranges
    assert_same_coo(read_mmf(p), ref_read(p))
