"""Regenerates tests/golden/ from the reference compiled from its sources
(oracle/_ref/libclspmv_ref.so; build it with `make -C oracle ref`).

    python tests/golden/make_golden.py

Writes:
  inputs.npz       the small seeded COO inputs and x vectors
  converters.json  per (matrix, converter, args): the reference's scalars and
                   the sha256 of every array (entries it defines)
  spmv.npz         the reference's serial <fmt>_spmv results (y += A x, y = 0)
  cocktail.json    the reference's analyze_matrix partitions (flags, variants,
                   part scalars, array hashes) for model tables given by
                   their clspmv_mic_b200.tables.model_tables arguments
"""
import hashlib
import json
import sys
import tempfile
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE.parent.parent))

from clspmv_mic_b200 import formats as F  # noqa: E402
from clspmv_mic_b200 import synth, tables  # noqa: E402
from clspmv_mic_b200 import _abi  # noqa: E402
from oracle import oracle as O  # noqa: E402

MATRICES = {
    "laplace16": lambda: synth.laplacian_2d(16),
    "stencil6": lambda: synth.stencil_27pt(6),
    "powerlaw600": lambda: synth.powerlaw(600, maxlen=200, seed=11),
    "blocks60": lambda: synth.block_rows(60, 8, seed=5),
    "random_empty": lambda: synth.random_coo(200, 200, 0.03, seed=3, empty_row_frac=0.3),
    "wide": lambda: synth.random_coo(90, 250, 0.04, seed=21),
}
CONVERTERS = [("csr", ()), ("dia", (32,)), ("bdia", (32,)), ("ell", (32, 0)), ("sell", (32,)), ("sell", (128,)),
              ("bcsr", (4, 2, 32)), ("b4csr", (4, 4, 32)), ("b4csr", (8, 2, 32)), ("bell", (4, 4, 32, 0)),
              ("b4ell", (4, 4, 32, 0)), ("b4ell", (8, 1, 32, 0)), ("sbell", (4, 4, 32)), ("sbell", (8, 2, 32))]
COCKTAIL_TABLES = {
    "plain": {},
    "dia_flat": {"seed": 1, "launch_us": 0.2, "gather_per_s": 2e12,
                 "scale": {"sell": 0.5, "ell": 0.5, "csr": 0.5, "coo": 0.5, "dia": 6, "bdia": 6}},
    "block_partial": {"seed": 1, "launch_us": 0.05, "gather_per_s": 1e13, "scale": {"dia": 6, "bdia": 6}},
    "sell_ell_fast": {"seed": 3, "scale": {"sell": 4, "ell": 4, "csr": 0.5, "coo": 0.5, "dia": 0.3, "bdia": 0.3,
                                           "sbell": 0.3, "bell": 0.3, "bcsr": 0.3}},
}
COCKTAIL_MATRICES = {
    "mixed": lambda: synth.cocktail_mixed(3000, 2400, 2000, seed=4),
    "powerlaw2k": lambda: synth.powerlaw(2000, maxlen=400, seed=5),
    "band_noise": lambda: _union(synth.banded(2000, 9, seed=3), synth.random_coo(2000, 2000, 0.002, seed=7)),
}


def _union(*ts):
    h, w = ts[0][0], ts[0][1]
    r = np.concatenate([t[2] for t in ts]).astype(np.int64)
    c = np.concatenate([t[3] for t in ts]).astype(np.int64)
    v = np.concatenate([t[4] for t in ts])
    key, idx = np.unique(r * w + c, return_index=True)
    return (h, w, (key // w).astype(np.int32), (key % w).astype(np.int32), v[idx])


def digest(fmt, m):
    """Scalars and sha256 of each array over the entries the reference
    defines (shared with tests/test_golden.py)."""
    from tests.test_converters import _defined_mask
    out = {"scalars": m.scalars(), "arrays": {}}
    for field, _, _ in _abi.FORMATS[fmt][1]:
        a = m.array(field)
        mask = _defined_mask(fmt, m, field)
        out["arrays"][field] = [int(a.size), hashlib.sha256(np.ascontiguousarray(a[mask]).tobytes()).hexdigest()]
    return out


def cocktail_digest(ck):
    from tests.cocktail_util import defined_mask
    s = ck.struct
    out = {"mat": [s.mat_height, s.mat_width, s.mat_nnz], "parts": {}}
    for p, fmt in _abi.COCKTAIL_PARTS:
        if not getattr(s, f"ifuse{p}"):
            continue
        m = ck.part(p)
        d = {"meth": getattr(s, f"{p}_meth_num"), "scalars": m.scalars(), "arrays": {}}
        if p in ("csr", "coo"):
            d["group"] = getattr(s, f"{p}_group_num")
        for field, _, _ in _abi.FORMATS[fmt][1]:
            a = m.array(field)
            mask = defined_mask(fmt, m, field)
            d["arrays"][field] = [int(a.size), hashlib.sha256(np.ascontiguousarray(a[mask]).tobytes()).hexdigest()]
        out["parts"][p] = d
    return out


def main():
    assert O.ref() is not None, "build oracle/_ref first: make -C oracle ref"
    inputs, conv, ys = {}, {}, {}
    for name, gen in MATRICES.items():
        h, w, r, c, v = gen()
        x = synth.x_vector(w)
        inputs[f"{name}__shape"] = np.array([h, w], np.int64)
        inputs[f"{name}__r"], inputs[f"{name}__c"], inputs[f"{name}__v"], inputs[f"{name}__x"] = r, c, v, x
        coo = F.coo_matrix(h, w, r, c, v)
        ys[f"{name}__coo"] = O.spmv_ref(coo, x)
        for fmt, args in CONVERTERS:
            ok, m = O.ref_convert(fmt, coo, *args)
            key = f"{name}|{fmt}|{','.join(map(str, args))}"
            if not ok:
                conv[key] = {"refused": True}
                continue
            conv[key] = digest(fmt, m)
            if fmt in ("csr", "ell", "sell", "sbell", "bcsr"):
                ys[f"{name}__{fmt}_{'_'.join(map(str, args))}"] = O.spmv_ref(m, x)
            elif fmt in ("dia", "bdia"):
                n = m.struct.dia_length_aligned if fmt == "dia" else m.struct.bdia_length_aligned
                ys[f"{name}__{fmt}_{'_'.join(map(str, args))}"] = O.spmv_ref(m, x, out_len=n)
            elif fmt == "bell":
                ys[f"{name}__{fmt}_{'_'.join(map(str, args))}"] = O.spmv_ref(m, x, out_len=m.struct.bell_row_num * m.struct.bell_bheight)
    ck = {}
    from tests.cocktail_util import ref_analyze
    for tname, kw in COCKTAIL_TABLES.items():
        d = tempfile.mkdtemp()
        tables.model_tables(d, **kw)
        for mname, gen in COCKTAIL_MATRICES.items():
            t = gen()
            coo = F.coo_matrix(*t)
            for mode in [(1.0, True, False), (1.0, False, False)]:
                ck[f"{tname}|{mname}|{mode[0]},{int(mode[1])},{int(mode[2])}"] = cocktail_digest(ref_analyze(coo, d, *mode))
            if tname == "plain":
                inputs[f"ck_{mname}__shape"] = np.array([t[0], t[1]], np.int64)
                inputs[f"ck_{mname}__r"], inputs[f"ck_{mname}__c"], inputs[f"ck_{mname}__v"] = t[2], t[3], t[4]
    np.savez_compressed(HERE / "inputs.npz", **inputs)
    np.savez_compressed(HERE / "spmv.npz", **ys)
    (HERE / "converters.json").write_text(json.dumps({"converters": conv, "cocktail_tables": COCKTAIL_TABLES,
                                                       "cocktail": ck}, indent=0, sort_keys=True))
    print("golden written:", len(conv), "converter cases,", len(ys), "spmv results,", len(ck), "partitions")


if __name__ == "__main__":
    main()
