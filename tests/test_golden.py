"""Parity against the committed golden fixtures (tests/golden/, produced by
the reference compiled from its sources; see make_golden.py). These run
without the reference checkout: the library's converters and Cocktail
partitioner must reproduce the reference's array hashes, and the C oracle
must reproduce the reference's serial SpMV results bit for bit."""
import json
import tempfile
from pathlib import Path

import numpy as np
import pytest

from clspmv_mic_b200 import _abi
from clspmv_mic_b200 import cocktail as CK
from clspmv_mic_b200 import formats as F
from clspmv_mic_b200 import tables
from oracle import oracle as O
from tests.golden.make_golden import CONVERTERS, MATRICES, cocktail_digest, digest

HERE = Path(__file__).resolve().parent / "golden"
GOLD = json.loads((HERE / "converters.json").read_text())
INPUTS = np.load(HERE / "inputs.npz")
YS = np.load(HERE / "spmv.npz")


def _coo(name):
    h, w = INPUTS[f"{name}__shape"]
    return F.coo_matrix(int(h), int(w), INPUTS[f"{name}__r"], INPUTS[f"{name}__c"], INPUTS[f"{name}__v"])


CONVERT = {"csr": F.coo2csr, "dia": F.coo2dia, "bdia": F.coo2bdia, "ell": F.coo2ell, "sell": F.coo2sell,
           "bcsr": F.coo2bcsr, "b4csr": F.coo2b4csr, "bell": F.coo2bell, "b4ell": F.coo2b4ell, "sbell": F.coo2sbell}


@pytest.mark.parametrize("name", sorted(MATRICES))
@pytest.mark.parametrize("fmt,args", CONVERTERS)
def test_converter_matches_golden(name, fmt, args):
    key = f"{name}|{fmt}|{','.join(map(str, args))}"
    want = GOLD["converters"][key]
    coo = _coo(name)
    if want.get("refused"):
        with pytest.raises(_abi.ClspmvError) as e:
            CONVERT[fmt](coo, *args)
        assert e.value.status == _abi.ERR_REFUSED
        return
    got = digest(fmt, CONVERT[fmt](coo, *args))
    skip = {"bell_float4_aligned"} if fmt == "bell" else set()
    for k, v in want["scalars"].items():
        if k not in skip:
            assert got["scalars"][k] == v, (key, k)
    assert got["arrays"] == want["arrays"], key


@pytest.mark.parametrize("name", sorted(MATRICES))
def test_oracle_matches_golden(name):
    """The C restatement reproduces the reference's serial SpMV outputs."""
    coo = _coo(name)
    x = INPUTS[f"{name}__x"]
    assert np.array_equal(O.spmv_port(coo, x).view(np.uint32), YS[f"{name}__coo"].view(np.uint32))
    for fmt, args in CONVERTERS:
        key = f"{name}__{fmt}_{'_'.join(map(str, args))}"
        if key not in YS:
            continue
        m = CONVERT[fmt](coo, *args)
        n = YS[key].size
        got = O.spmv_port(m, x, out_len=n)
        assert np.array_equal(got.view(np.uint32), YS[key].view(np.uint32)), key


@pytest.fixture(scope="module")
def table_dirs():
    out = {}
    for name, kw in GOLD["cocktail_tables"].items():
        d = tempfile.mkdtemp(prefix=f"golden_tables_{name}_")
        tables.model_tables(d, **kw)
        out[name] = d
    return out


def test_cocktail_matches_golden(table_dirs):
    mats = {k.split("ck_")[1].split("__")[0] for k in INPUTS.files if k.startswith("ck_")}
    n = 0
    for key, want in GOLD["cocktail"].items():
        tname, mname, mode = key.split("|")
        mult, part, full = mode.split(",")
        assert mname in mats
        h, w = INPUTS[f"ck_{mname}__shape"]
        coo = F.coo_matrix(int(h), int(w), INPUTS[f"ck_{mname}__r"], INPUTS[f"ck_{mname}__c"], INPUTS[f"ck_{mname}__v"])
        got = cocktail_digest(CK.analyze(coo, table_dirs[tname], float(mult), part == "1", full == "1"))
        assert got == want, key
        n += 1
    assert n == len(GOLD["cocktail"])
