"""Helpers comparing the library's Cocktail partition with the reference's."""
import ctypes as C
import os
import sys

import numpy as np

from clspmv_mic_b200 import _abi
from clspmv_mic_b200 import cocktail as CK
from clspmv_mic_b200.formats import HostMatrix

PART_NAMES = [p for p, _ in _abi.COCKTAIL_PARTS]


def ref_analyze(coo, table_root, mult=1.0, partial=True, full=False):
    """The reference's analyze_matrix on a private copy of `coo`, with its
    console output discarded. Returns a CocktailMatrix whose arrays are owned
    by the reference library (released with free())."""
    from oracle import oracle as O
    L = O.ref()
    src = coo.copy()
    out = _abi.Cocktail()
    sys.stdout.flush()
    saved = os.dup(1)
    devnull = os.open(os.devnull, os.O_WRONLY)
    os.dup2(devnull, 1)
    try:
        L.ref_analyze_matrix(C.byref(src.struct), C.byref(out), str(table_root).encode(), mult, int(partial), int(full))
    finally:
        os.dup2(saved, 1)
        os.close(saved)
        os.close(devnull)

    def release(s):
        for p, fmt in _abi.COCKTAIL_PARTS:
            part = getattr(s, p)
            for field, _, _ in _abi.FORMATS[fmt][1]:
                ptr = getattr(part, field)
                if ptr and getattr(s, f"ifuse{p}"):
                    L.ref_free(ptr)
    return CK.CocktailMatrix(out, owner=None, releaser=release)


def defined_mask(fmt, m: HostMatrix, field):
    """Entries the reference writes (it leaves some padding uninitialised:
    sbell column ids of block rows past sbell_row_num, src/analyze.cpp:1840;
    bell column ids past the block-row count, :2062)."""
    arr = m.array(field)
    mask = np.ones(arr.size, dtype=bool)
    s = m.struct
    if fmt == "b4ell" and field == "b4ell_col_id" and s.b4ell_height_aligned > 0:
        mask = (np.arange(arr.size) % s.b4ell_height_aligned) < s.b4ell_row_num
    if fmt == "sbell" and field == "sbell_col_id" and s.sbell_slice_num > 0:
        sp = m.array("sbell_slice_ptr")
        sh = s.sbell_slice_height
        for sl in range(s.sbell_slice_num):
            a, b = int(sp[sl]), int(sp[sl + 1])
            lr = (np.arange(b - a) % sh)
            mask[a:b] = (sl * sh + lr) < s.sbell_row_num
    return mask


def compare_cocktails(mine, theirs):
    """List of differences (empty when byte-identical on defined entries)."""
    diffs = []
    a, b = mine.struct, theirs.struct
    for k in ("mat_width", "mat_height", "mat_nnz"):
        if getattr(a, k) != getattr(b, k):
            diffs.append(f"{k}: {getattr(a, k)} != {getattr(b, k)}")
    for p in PART_NAMES:
        ua, ub = bool(getattr(a, f"ifuse{p}")), bool(getattr(b, f"ifuse{p}"))
        if ua != ub:
            diffs.append(f"ifuse{p}: {ua} != {ub}")
            continue
        if not ua:
            continue
        if getattr(a, f"{p}_meth_num") != getattr(b, f"{p}_meth_num"):
            diffs.append(f"{p}_meth_num: {getattr(a, f'{p}_meth_num')} != {getattr(b, f'{p}_meth_num')}")
        if p in ("csr", "coo") and getattr(a, f"{p}_group_num") != getattr(b, f"{p}_group_num"):
            diffs.append(f"{p}_group_num differs")
        ma, mb = mine.part(p), theirs.part(p)
        sa, sb = ma.scalars(), mb.scalars()
        for k in sa:
            if sa[k] != sb[k]:
                diffs.append(f"{p}.{k}: {sa[k]} != {sb[k]}")
        if any(d.startswith(p + ".") for d in diffs):
            continue
        for field, _, _ in _abi.FORMATS[ma.fmt][1]:
            xa, xb = ma.array(field), mb.array(field)
            if xa.shape != xb.shape:
                diffs.append(f"{p}.{field}: length {xa.shape} != {xb.shape}")
                continue
            mask = defined_mask(ma.fmt, mb, field)
            if not np.array_equal(xa.view(np.uint32)[mask], xb.view(np.uint32)[mask]):
                bad = np.nonzero(xa.view(np.uint32)[mask] != xb.view(np.uint32)[mask])[0]
                diffs.append(f"{p}.{field}: {bad.size} entries differ (first {bad[:5]})")
    return diffs
