"""Several right-hand sides (Y = alpha*A*X + beta*Y) and 16-bit value storage.

Oracle: the FP64 restatement of the reference's csr_spmv (oracle/) applied
column by column. FP32 values must be within 1e-5 * (|alpha| sum_j |a_ij x_jc|
+ |beta y_ic|) per entry, the bound of the single-vector kernels. BF16 / FP16
values are checked against their own rounding bound (2^-8 and 2^-10 of the
same row scale, one rounding per stored value) and their error against FP64
is what the bench reports.
"""
import numpy as np
import pytest

from clspmv_mic_b200 import formats as F
from clspmv_mic_b200 import synth
from oracle import oracle as O

from matrices import coo_of

pytestmark = pytest.mark.gpu

RTOL = {"f32": 1e-5, "bf16": 2.0 ** -8, "f16": 2.0 ** -10}


def spmm_reference(coo, X, Y0, alpha, beta):
    csr = F.coo2csr(coo)
    m, k = coo.shape[0], X.shape[1]
    ref = np.zeros((m, k))
    bound = np.zeros((m, k))
    for c in range(k):
        y64, sc = O.csr_f64(csr, np.ascontiguousarray(X[:, c]))
        ref[:, c] = alpha * y64 + beta * Y0[:, c].astype(np.float64)
        bound[:, c] = abs(alpha) * sc + abs(beta) * np.abs(Y0[:, c].astype(np.float64))
    return ref, bound


def device_of(coo, fmt, *args):
    host = coo if fmt == "coo" else getattr(F, f"coo2{fmt}")(coo, *args)
    return F.DeviceMatrix(host)


CASES = [
    ("laplace33", "csr", ()), ("laplace33", "coo", ()), ("laplace33", "dia", ()), ("laplace33", "bdia", ()),
    ("laplace33", "ell", ()), ("laplace33", "sell", (32,)), ("stencil6", "dia", ()), ("stencil6", "bdia", ()),
    ("powerlaw3k", "csr", ()), ("powerlaw3k", "coo", ()), ("powerlaw3k", "sell", (128,)), ("powerlaw3k", "ell", ()),
    ("random_empty_rows", "csr", ()), ("random_empty_rows", "coo", ()), ("blocks_odd", "b4csr", (4, 4)),
    ("blocks_odd", "b4ell", (8, 2)), ("blocks_odd", "sbell", (4, 4)), ("blocks300", "b4csr", (8, 8)),
    ("blocks300", "sbell", (4, 1)), ("blocks300", "b4ell", (4, 4)), ("wide", "csr", ()), ("tall", "sell", (32,)),
]


def _run(name, fmt, args, k, alpha, beta, value_type="f32", ld_pad=0):
    import torch
    coo = coo_of(name)
    m, n = coo.shape
    rng = np.random.default_rng(k * 31 + len(name))
    X = rng.uniform(-1, 1, (n, k)).astype(np.float32)
    Y0 = rng.uniform(-1, 1, (m, k)).astype(np.float32)
    dev = device_of(coo, fmt, *args)
    Xd = torch.zeros((n, k + ld_pad), dtype=torch.float32, device="cuda")
    Xd[:, :k] = torch.from_numpy(X)
    Yd = torch.zeros((m, k + ld_pad), dtype=torch.float32, device="cuda")
    Yd[:, :k] = torch.from_numpy(Y0)
    packed = None if value_type == "f32" else dev.pack(value_type)
    dev.spmm(Xd[:, :k], Yd[:, :k], alpha, beta, packed=packed)
    torch.cuda.synchronize()
    got = Yd[:, :k].cpu().numpy().astype(np.float64)
    ref, bound = spmm_reference(coo, X, Y0, alpha, beta)
    err = np.abs(got - ref)
    lim = RTOL[value_type] * bound + 1e-30
    bad = np.argwhere(err > lim)
    assert bad.size == 0, f"{name}/{fmt}{args} k={k} {value_type}: {len(bad)} entries off, first {bad[:3].tolist()}"
    return float(np.max(err / np.where(bound > 0, bound, 1.0))) if err.size else 0.0


@pytest.mark.parametrize("name,fmt,args", CASES)
@pytest.mark.parametrize("k", [1, 4, 16, 32])
def test_spmm_f32(name, fmt, args, k):
    _run(name, fmt, args, k, 1.0, 0.0)


@pytest.mark.parametrize("name,fmt,args", [c for c in CASES if c[0] in ("laplace33", "blocks_odd", "powerlaw3k")])
@pytest.mark.parametrize("k,ld_pad,alpha,beta", [(3, 1, 0.5, 2.0), (5, 0, -1.0, 1.0), (64, 0, 1.0, -0.5),
                                                 (128, 4, 2.0, 0.0), (7, 2, 1.0, 1.0)])
def test_spmm_shapes_and_scalars(name, fmt, args, k, ld_pad, alpha, beta):
    _run(name, fmt, args, k, alpha, beta, ld_pad=ld_pad)


@pytest.mark.parametrize("value_type", ["bf16", "f16"])
@pytest.mark.parametrize("name,fmt,args", CASES[::2])
@pytest.mark.parametrize("k", [1, 16])
def test_spmm_reduced_precision(name, fmt, args, k, value_type):
    _run(name, fmt, args, k, 1.0, 0.0, value_type=value_type)


@pytest.mark.parametrize("value_type", ["bf16", "f16"])
def test_pack_values_scaled_rounding(value_type):
    import torch
    coo = coo_of("powerlaw3k")
    a = coo.arrays()
    rows, vals = a["coo_row_id"], a["coo_data"].astype(np.float64) * np.exp(np.linspace(-20, 20, coo.nnz))
    big = F.coo_matrix(coo.shape[0], coo.shape[1], rows, a["coo_col_id"], vals.astype(np.float32))
    csr = F.coo2csr(big)          # kept alive: its arrays are viewed below
    dev = F.DeviceMatrix(csr)
    p = dev.pack(value_type)
    torch.cuda.synchronize()
    dt = torch.bfloat16 if value_type == "bf16" else torch.float16
    packed = p.values.view(dt).float().cpu().numpy().astype(np.float64)[:big.nnz]
    scale = p.row_scale.cpu().numpy().astype(np.float64)
    ref = csr.array("csr_data").astype(np.float64)
    row_of = np.repeat(np.arange(big.shape[0]), np.diff(csr.array("csr_row_ptr")))
    mx = np.zeros(big.shape[0])
    np.maximum.at(mx, row_of, np.abs(ref))
    assert np.all(np.log2(scale) == np.round(np.log2(scale)))            # powers of two
    assert np.all((scale >= mx) & ((mx == 0) | (scale < 2 * mx)))
    rel = np.abs(packed * scale[row_of] - ref) / np.maximum(scale[row_of], 1e-300)
    assert rel.max() <= RTOL[value_type] / 2 + 1e-12


def test_spmm_k1_matches_spmv():
    import torch
    coo = coo_of("powerlaw3k")
    m, n = coo.shape
    dev = F.DeviceMatrix(F.coo2csr(coo))
    x = torch.from_numpy(synth.x_vector(n)).cuda()
    y1 = torch.zeros(m, device="cuda")
    dev.spmv(x, y1, 1.0, 0.0)
    y2 = torch.zeros((m, 1), device="cuda")
    dev.spmm(x.view(n, 1), y2, 1.0, 0.0)
    torch.cuda.synchronize()
    _, _, bound = __import__("gpu_util").reference_y(coo, x.cpu().numpy(), None, 1.0, 0.0)
    assert np.all(np.abs(y1.cpu().numpy() - y2[:, 0].cpu().numpy()) <= 2e-5 * bound + 1e-30)


def test_spmm_rejects():
    import torch
    from clspmv_mic_b200 import _abi
    dev = F.DeviceMatrix(F.coo2csr(coo_of("laplace16")))
    n = dev.shape[1]
    with pytest.raises(_abi.ClspmvError):
        dev.spmm(torch.zeros((n, 129), device="cuda"), torch.zeros((dev.shape[0], 129), device="cuda"))
    X = torch.zeros((n, 40), device="cuda")[:, 1:]      # k = 39 > 32 without 16-byte rows
    with pytest.raises(_abi.ClspmvError) as e:
        dev.spmm(X, torch.zeros((dev.shape[0], 39), device="cuda"))
    assert e.value.status == _abi.ERR_ALIGN


PACKED_CASES = [("laplace33", "csr", ()), ("powerlaw3k", "coo", ()), ("laplace33", "dia", ()), ("stencil6", "bdia", ()),
                ("powerlaw3k", "ell", ()), ("powerlaw3k", "sell", (32,)), ("random_empty_rows", "sell", (20,)),
                ("blocks_odd", "b4csr", (8, 4)), ("blocks300", "b4ell", (4, 2)), ("blocks300", "sbell", (4, 8)),
                ("random_empty_rows", "csr", ()), ("random_empty_rows", "coo", ())]


@pytest.mark.parametrize("value_type", ["bf16", "f16"])
@pytest.mark.parametrize("name,fmt,args", PACKED_CASES)
def test_spmv_packed_dedicated(name, fmt, args, value_type):
    """Single-vector SpMV with 16-bit values in each format's own kernel."""
    import torch
    coo = coo_of(name)
    m, n = coo.shape
    dev = device_of(coo, fmt, *args)
    p = dev.pack(value_type)
    x = synth.x_vector(n, seed=3)
    y0 = np.random.default_rng(2).uniform(-1, 1, m).astype(np.float32)
    for alpha, beta in [(1.0, 0.0), (-0.5, 1.5)]:
        xd = torch.from_numpy(x).cuda()
        yd = torch.from_numpy(y0.copy()).cuda()
        n0 = F.launch_count()
        dev.spmv(xd, yd, alpha, beta, packed=p)
        torch.cuda.synchronize()
        assert F.launch_count() > n0
        ref, bound = spmm_reference(coo, x[:, None], y0[:, None], alpha, beta)
        err = np.abs(yd.cpu().numpy().astype(np.float64) - ref[:, 0])
        lim = RTOL[value_type] * bound[:, 0] + 1e-6 * abs(beta) * np.abs(y0) + 1e-30
        assert np.all(err <= lim), (name, fmt, args, value_type, alpha, beta, float((err / (bound[:, 0] + 1e-30)).max()))


@pytest.mark.parametrize("value_type", ["bf16", "f16"])
@pytest.mark.parametrize("name,sh", [("powerlaw3k", 32), ("powerlaw3k", 8), ("powerlaw3k", 128), ("random_empty_rows", 32),
                                     ("random_empty_rows", 20), ("one_entry", 4)])
def test_sell_planned_packed(name, sh, value_type):
    """SELL through its length plan with 16-bit values (heads column-balanced,
    long tails from the compact column ids; slice height 20 takes the padded
    16-bit read) against the FP64 oracle at the 16-bit bound, and against
    the padded 16-bit read."""
    import torch
    coo = coo_of(name)
    m, n = coo.shape
    dev = device_of(coo, "sell", sh)
    p = dev.pack(value_type)
    x = synth.x_vector(n, seed=6)
    y0 = np.random.default_rng(5).uniform(-1, 1, m).astype(np.float32)
    for alpha, beta in [(1.0, 0.0), (-0.5, 1.5)]:
        ys = {}
        for variant in ("planned", "padded"):
            xd, yd = torch.from_numpy(x).cuda(), torch.from_numpy(y0.copy()).cuda()
            dev.spmv(xd, yd, alpha, beta, packed=p, variant=variant)
            torch.cuda.synchronize()
            ys[variant] = yd.cpu().numpy().astype(np.float64)
        ref, bound = spmm_reference(coo, x[:, None], y0[:, None], alpha, beta)
        lim = RTOL[value_type] * bound[:, 0] + 1e-6 * abs(beta) * np.abs(y0) + 1e-30
        for variant, y in ys.items():
            assert np.all(np.abs(y - ref[:, 0]) <= lim), (name, sh, value_type, variant)
        assert np.all(np.abs(ys["planned"] - ys["padded"]) <= 2e-5 * bound[:, 0] + 1e-6 * abs(beta) * np.abs(y0) + 1e-30)


@pytest.mark.parametrize("value_type", ["bf16", "f16"])
@pytest.mark.parametrize("variant", ["chunk", "merge"])
def test_csr_packed_both_kernels(value_type, variant):
    """16-bit CSR values in the chunked and the merge-path kernel."""
    import torch
    coo = coo_of("powerlaw3k")
    m, n = coo.shape
    dev = device_of(coo, "csr")
    p = dev.pack(value_type)
    x = synth.x_vector(n, seed=4)
    y0 = np.random.default_rng(3).uniform(-1, 1, m).astype(np.float32)
    xd, yd = torch.from_numpy(x).cuda(), torch.from_numpy(y0.copy()).cuda()
    dev.spmv(xd, yd, 0.5, 1.0, packed=p, variant=variant)
    torch.cuda.synchronize()
    ref, bound = spmm_reference(coo, x[:, None], y0[:, None], 0.5, 1.0)
    err = np.abs(yd.cpu().numpy().astype(np.float64) - ref[:, 0])
    assert np.all(err <= RTOL[value_type] * bound[:, 0] + 1e-6 * np.abs(y0) + 1e-30)


@pytest.mark.parametrize("k", [4, 8, 16, 32, 64])
@pytest.mark.parametrize("value_type", ["f32", "bf16"])
def test_csr_long_rows_warp_kernel(k, value_type):
    """CSR rows averaging 128 or more nonzeros take the warp-per-row kernel
    at k a power of two times 4: against the FP64 oracle, with alpha / beta,
    empty rows included."""
    import torch
    coo = F.coo_matrix(*synth.random_coo(300, 4000, 0.08, seed=21, empty_row_frac=0.1))
    assert coo.nnz >= 128 * coo.shape[0]
    m, n = coo.shape
    dev = device_of(coo, "csr")
    p = None if value_type == "f32" else dev.pack(value_type)
    rng = np.random.default_rng(k)
    X = rng.uniform(-1, 1, (n, k)).astype(np.float32)
    Y0 = rng.uniform(-1, 1, (m, k)).astype(np.float32)
    for alpha, beta in [(1.0, 0.0), (0.5, -1.5)]:
        Xd, Yd = torch.from_numpy(X).cuda(), torch.from_numpy(Y0.copy()).cuda()
        dev.spmm(Xd, Yd, alpha, beta, packed=p)
        torch.cuda.synchronize()
        ref, bound = spmm_reference(coo, X, Y0, alpha, beta)
        err = np.abs(Yd.cpu().numpy().astype(np.float64) - ref)
        assert np.all(err <= RTOL[value_type] * bound + 1e-6 * abs(beta) * np.abs(Y0) + 1e-30), (k, value_type, alpha, beta)


_BLOCK_WALK_SCRIPT = r"""
import sys
import numpy as np
import torch
sys.path.insert(0, sys.argv[2])
from clspmv_mic_b200 import formats as F
from tests.matrices import coo_of
out = {}
for name in ("blocks_odd", "blocks300", "ragged_tail"):
    coo = coo_of(name)
    m, n = coo.shape
    for fmt in ("b4csr", "b4ell", "sbell"):
        for bw, bh in [(4, 1), (4, 2), (4, 4), (4, 8), (8, 1), (8, 2), (8, 4), (8, 8)]:
            dev = F.DeviceMatrix(getattr(F, "coo2" + fmt)(coo, bw, bh))
            for k, vt in [(16, "f32"), (32, "f32"), (8, "bf16"), (128, "f16")]:
                rng = np.random.default_rng(k + bw * 3 + bh)
                X = torch.from_numpy(rng.uniform(-1, 1, (n, k)).astype(np.float32)).cuda()
                Y = torch.from_numpy(rng.uniform(-1, 1, (m, k)).astype(np.float32)).cuda()
                dev.spmm(X, Y, 0.75, -0.5, packed=None if vt == "f32" else dev.pack(vt))
                out[f"{name}-{fmt}-{bw}x{bh}-{k}-{vt}"] = Y.cpu().numpy()
np.savez(sys.argv[1], **out)
"""


def test_block_rows_kernel_matches_row_walk(tmp_path):
    """The block-row SpMM kernel of the 4-wide block formats (X slice loaded
    once per block, all rows of the block from registers) gives the same
    bits as the row walk (CLSPMV_SPMM_BLOCK_ROWS=0) for all 8 block shapes of
    b4csr / b4ell / SBELL, FP32 and 16-bit values, alpha and beta."""
    import os
    import subprocess
    import sys
    from pathlib import Path
    root = str(Path(__file__).resolve().parents[1])
    script = tmp_path / "walk.py"
    script.write_text(_BLOCK_WALK_SCRIPT)
    res = {}
    for flag in ("1", "0"):
        env = dict(os.environ, CLSPMV_SPMM_BLOCK_ROWS=flag)
        out = tmp_path / f"y{flag}.npz"
        subprocess.run([sys.executable, str(script), str(out), root], env=env, check=True, cwd=root, timeout=600)
        res[flag] = np.load(out)
    assert sorted(res["1"].files) == sorted(res["0"].files) and len(res["1"].files) == 3 * 3 * 8 * 4
    for key in res["1"].files:
        assert np.array_equal(res["1"][key].view(np.uint32), res["0"][key].view(np.uint32)), key
