"""Cocktail runtime on the GPU: a partitioned matrix's SpMV over all its
parts (running concurrently, accumulating atomically into y) against the
oracle's csr_spmv on the unpartitioned matrix, within the 1e-5 row bound;
plus replay under CUDA-graph capture (the A^k x loop of src/eval.cpp:19-72
without host synchronisation)."""
import numpy as np
import pytest

from clspmv_mic_b200 import cocktail as CK
from clspmv_mic_b200 import formats as F
from clspmv_mic_b200 import synth, tables
from tests.gpu_util import assert_close, reference_y
from tests.test_cocktail_partition import _matrices, _table_configs

pytestmark = pytest.mark.gpu

CASES = [("block_partial", "mixed", (1.0, False, False)), ("block_partial", "blocks_noise", (1.0, False, False)),
         ("dia_flat", "band_noise", (1.0, True, False)), ("random0", "band_blocks_noise", (1.0, True, False)),
         ("sbell_bell", "blocks_noise", (1.0, True, False)), ("sell_ell_fast", "powerlaw", (1.0, True, False)),
         ("plain", "laplace128", (1.0, True, False)), ("fl1_bl8_dia6", "mixed", (1.0, True, False)),
         ("plain", "wide", (1.0, True, False))]


@pytest.fixture(scope="module", autouse=True)
def _cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


@pytest.fixture(scope="module")
def setup(tmp_path_factory):
    cfgs = dict(_table_configs())
    mats = _matrices()
    out = {}
    for cfg, mname, mode in CASES:
        d = tmp_path_factory.mktemp(f"t_{cfg}")
        tables.model_tables(d, **cfgs[cfg])
        coo = F.coo_matrix(*mats[mname])
        out[(cfg, mname)] = (coo, CK.analyze(coo, d, *mode))
    return out


@pytest.mark.parametrize("cfg,mname,mode", CASES)
@pytest.mark.parametrize("alpha,beta", [(1.0, 1.0), (2.0, -0.5), (1.0, 0.0)])
@pytest.mark.parametrize("schedule", ["auto", "fused"])
def test_cocktail_spmv(setup, cfg, mname, mode, alpha, beta, schedule):
    """Both schedules: one launch per part (auto) and the fused persistent
    launch over all parts (partitions of two or more parts)."""
    import torch
    coo, ck = setup[(cfg, mname)]
    dev = ck.to_device()
    if schedule == "fused" and len(dev.parts) < 2:
        pytest.skip("one part: nothing to fuse")
    dev.set_schedule(schedule)
    x = synth.x_vector(coo.shape[1])
    y0 = np.random.default_rng(3).standard_normal(coo.shape[0]).astype(np.float32)
    xd = torch.from_numpy(x).cuda()
    yd = torch.from_numpy(y0.copy()).cuda()
    dev.spmv(xd, yd, alpha, beta)
    torch.cuda.synchronize()
    y_ref, _, bound = reference_y(coo, x, y0, alpha, beta)
    assert_close(yd.cpu().numpy(), y_ref, bound, f"cocktail {cfg}/{mname} parts={dev.parts}")


def test_cocktail_fused_covers_multi_part_cases(setup):
    """Every multi-part partition of the test configurations gets a fused
    work list (their block shapes are among those the fused kernel covers),
    and "fused" can be required; a single part keeps its own launch."""
    seen = 0
    for (cfg, mname), (coo, ck) in setup.items():
        dev = ck.to_device()
        if len(dev.parts) >= 2:
            assert dev.fused_items >= len(dev.parts), (cfg, mname, dev.parts)
            dev.set_schedule("fused")
            seen += 1
        else:
            assert dev.fused_items == 0
    assert seen >= 3


def test_cocktail_fused_graph_replay_and_repeat(setup):
    """The fused schedule replayed from a captured graph and called back to
    back (the work counter is reset by the launch before it each time): y =
    y0 + k A x."""
    import torch
    coo, ck = setup[("block_partial", "mixed")]
    dev = ck.to_device()
    assert dev.fused_items > 0, dev.parts
    dev.set_schedule("fused")
    x = synth.x_vector(coo.shape[1])
    xd = torch.from_numpy(x).cuda()
    yd = torch.zeros(coo.shape[0], dtype=torch.float32, device="cuda")
    s = torch.cuda.Stream()
    s.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(s):
        dev.spmv(xd, yd, 1.0, 1.0, stream=s)
    torch.cuda.synchronize()
    yd.zero_()
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g, stream=s):
        dev.spmv(xd, yd, 1.0, 1.0, stream=s)
    yd.zero_()
    for _ in range(3):
        g.replay()
    for _ in range(2):
        dev.spmv(xd, yd, 1.0, 1.0)
    torch.cuda.synchronize()
    y_ref, _, bound = reference_y(coo, x)
    assert_close(yd.cpu().numpy() / 5, y_ref, bound, "fused replay")


def hand_partition(layout, seed=3, scatter=30000):
    """A matrix of n rows (tridiagonal band + 4x4 blocks + scattered
    entries) split by hand into the Cocktail slots of `layout`
    ({slot: converter}), every entry in exactly one slot: the band to the
    first slot, the blocks to the second, the scattered entries dealt out by
    row to the rest. Returns (COO of the whole matrix, CocktailMatrix)."""
    from clspmv_mic_b200 import _abi
    rng = np.random.default_rng(seed)
    n = 4096
    r = np.arange(n)
    band = [(r, r, np.full(n, 2.0))] + [(r[1:], r[1:] - 1, -np.ones(n - 1)), (r[:-1], r[:-1] + 1, -np.ones(n - 1))]
    br = rng.choice(n // 4, 600, replace=False)
    bc = rng.integers(0, n // 4, 600)
    bi, bj = np.meshgrid(np.arange(4), np.arange(4), indexing="ij")
    blk_r = (br[:, None] * 4 + bi.ravel()[None, :]).ravel()
    blk_c = (bc[:, None] * 4 + bj.ravel()[None, :]).ravel()
    sr = rng.integers(0, n, scatter)
    sc = rng.integers(0, n, scatter)
    groups = {"band": (np.concatenate([b[0] for b in band]), np.concatenate([b[1] for b in band])),
              "blocks": (blk_r, blk_c), "scatter": (sr, sc)}
    # distinct (row, col): an entry keeps the first group that claims it
    taken = set()
    split = {}
    for g, (gr, gc) in groups.items():
        keys = gr.astype(np.int64) * n + gc
        keys = np.unique(keys)
        keys = np.array([k for k in keys if k not in taken], dtype=np.int64)
        taken.update(keys.tolist())
        split[g] = keys
    slots = list(layout)
    pieces = {slots[0]: split["band"], slots[1]: split["blocks"]}
    rest = slots[2:]
    srow = split["scatter"] // n
    for i, sl in enumerate(rest):
        pieces[sl] = split["scatter"][srow % len(rest) == i]
    st = _abi.Cocktail()
    st.mat_width = st.mat_height = n
    keep = []
    allk = []
    for sl, keys in pieces.items():
        keys = np.sort(keys)
        allk.append(keys)
        vals = rng.standard_normal(keys.size).astype(np.float32)
        part_coo = F.coo_matrix(n, n, keys // n, keys % n, vals)
        host = layout[sl](part_coo)
        keep.append((part_coo, host))
        setattr(st, f"ifuse{sl}", True)
        setattr(st, sl, type(getattr(st, sl)).from_buffer_copy(host.struct))
    st.mat_nnz = int(sum(k.size for k in allk))
    ck = CK.CocktailMatrix(st, owner=None)
    ck._keep = keep
    # the whole matrix: every slot's entries, with the values each slot holds
    rows = np.concatenate([pc.array("coo_row_id") for pc, _ in keep])
    cols = np.concatenate([pc.array("coo_col_id") for pc, _ in keep])
    vals = np.concatenate([pc.array("coo_data") for pc, _ in keep])
    o = np.lexsort((cols, rows))
    return F.coo_matrix(n, n, rows[o], cols[o], vals[o]), ck


HAND_LAYOUTS = {
    "dia_sbell_ell_sell_csr_coo": {"dia": F.coo2dia, "sbell": lambda c: F.coo2sbell(c, 4, 4, 32),
                                   "ell": lambda c: F.coo2ell(c), "sell": lambda c: F.coo2sell(c, 32),
                                   "csr": F.coo2csr, "coo": lambda c: c},
    "bdia_bell_bcsr_sell8_coo": {"bdia": F.coo2bdia, "bell": lambda c: F.coo2b4ell(c, 4, 2),
                                 "bcsr": lambda c: F.coo2b4csr(c, 8, 1), "sell": lambda c: F.coo2sell(c, 8),
                                 "coo": lambda c: c},
    "dia_bcsr_sell20": {"dia": F.coo2dia, "bcsr": lambda c: F.coo2b4csr(c, 4, 4), "sell": lambda c: F.coo2sell(c, 20)},
    # dense scattered part: SELL by slice columns; slice height 7: SELL row by row
    "dia_bcsr_sell32_dense": {"dia": F.coo2dia, "bcsr": lambda c: F.coo2b4csr(c, 4, 4), "sell": lambda c: F.coo2sell(c, 32)},
    "bdia_sbell82_sell7": {"bdia": F.coo2bdia, "sbell": lambda c: F.coo2sbell(c, 8, 2, 32), "sell": lambda c: F.coo2sell(c, 7)},
}
HAND_SCATTER = {"dia_bcsr_sell32_dense": 90000}


@pytest.mark.parametrize("layout", sorted(HAND_LAYOUTS))
@pytest.mark.parametrize("schedule", ["fused", "per_part"])
def test_cocktail_hand_partitions(layout, schedule):
    """Hand-made partitions using all nine slots between them (several flat
    parts at once, every fused kernel kind: DIA, BDIA, SBELL, BELL, BCSR with
    8-wide blocks, SELL by columns and by rows, ELL, CSR, COO): the fused
    launch and the per-part launches against the oracle."""
    import torch
    coo, ck = hand_partition(HAND_LAYOUTS[layout], scatter=HAND_SCATTER.get(layout, 30000))
    dev = ck.to_device()
    assert dev.fused_items >= len(dev.parts)
    dev.set_schedule(schedule)
    x = synth.x_vector(coo.shape[1])
    y0 = np.random.default_rng(2).standard_normal(coo.shape[0]).astype(np.float32)
    for alpha, beta in [(1.0, 0.0), (1.5, -0.5)]:
        xd, yd = torch.from_numpy(x).cuda(), torch.from_numpy(y0.copy()).cuda()
        dev.spmv(xd, yd, alpha, beta)
        torch.cuda.synchronize()
        y_ref, _, bound = reference_y(coo, x, y0, alpha, beta)
        assert_close(yd.cpu().numpy(), y_ref, bound, f"{layout} {schedule} parts={dev.parts}")


@pytest.mark.parametrize("lanes", [0, 1, 4, 32])
def test_cocktail_csr_part_lanes(setup, lanes):
    """The CSR part run as nonzero chunks (0) or CSR-vector with 1..32 lanes
    per row (the tuner's threads-per-row choice): the same y within the
    1e-5 row bound."""
    import torch
    coo, ck = setup[("block_partial", "blocks_noise")]
    dev = ck.to_device()
    assert "csr" in dev.parts, dev.parts
    dev.set_csr_lanes(lanes)
    x = synth.x_vector(coo.shape[1])
    y0 = np.random.default_rng(4).standard_normal(coo.shape[0]).astype(np.float32)
    xd, yd = torch.from_numpy(x).cuda(), torch.from_numpy(y0.copy()).cuda()
    dev.spmv(xd, yd, 1.0, 0.5)
    torch.cuda.synchronize()
    y_ref, _, bound = reference_y(coo, x, y0, 1.0, 0.5)
    assert_close(yd.cpu().numpy(), y_ref, bound, f"csr lanes {lanes}")


def test_cocktail_graph_replay(setup):
    """Capture y <- A x + y once, replay it k times: y = y0 + k A x."""
    import torch
    coo, ck = setup[("block_partial", "mixed")]
    dev = ck.to_device()
    assert len(dev.parts) >= 2, dev.parts
    x = synth.x_vector(coo.shape[1])
    xd = torch.from_numpy(x).cuda()
    yd = torch.zeros(coo.shape[0], dtype=torch.float32, device="cuda")
    s = torch.cuda.Stream()
    s.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(s):
        dev.spmv(xd, yd, 1.0, 1.0, stream=s)   # warm-up outside capture
    torch.cuda.synchronize()
    yd.zero_()
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g, stream=s):
        dev.spmv(xd, yd, 1.0, 1.0, stream=s)
    yd.zero_()
    k = 5
    for _ in range(k):
        g.replay()
    torch.cuda.synchronize()
    y_ref, _, bound = reference_y(coo, x)
    assert_close(yd.cpu().numpy() / k, y_ref, bound * 1.0, "graph replay")


def test_cocktail_parts_alone_sum_to_whole(setup):
    """Each part alone, added up, gives the partitioned result."""
    import torch
    coo, ck = setup[("fl1_bl8_dia6", "mixed")]
    x = synth.x_vector(coo.shape[1])
    xd = torch.from_numpy(x).cuda()
    total = np.zeros(coo.shape[0], np.float64)
    for name, part in ck.parts().items():
        yd = torch.zeros(coo.shape[0], dtype=torch.float32, device="cuda")
        kw = {"variant": "merge"} if part.fmt == "csr" else {}
        F.DeviceMatrix(part).spmv(xd, yd, 1.0, 1.0, **kw)
        torch.cuda.synchronize()
        total += yd.cpu().numpy()
    y_ref, _, bound = reference_y(coo, x)
    assert_close(total.astype(np.float32), y_ref, bound * 2, "sum of parts")


def _iterate_by_steps(dev, x, y, k, alpha, beta):
    """The reference's loop (src/eval.cpp:44-50): one SpMV, then x[:rows] <- y."""
    rows = y.shape[0]
    for _ in range(k):
        dev.spmv(x, y, alpha, beta)
        x[:rows].copy_(y)


@pytest.mark.parametrize("cfg,mname", [("plain", "laplace128"), ("block_partial", "mixed"),
                                       ("sell_ell_fast", "powerlaw")])
@pytest.mark.parametrize("k", [1, 5, 16, 21, 48])
def test_cocktail_iterate_matches_step_loop(setup, cfg, mname, k):
    """clspmv_cocktail_iterate_f32 (graph-replayed groups of 16 steps plus
    direct steps) against the step-by-step loop on the same device: equal
    bit for bit for a single part whose kernel has no atomics, within FP32
    summation-order noise otherwise."""
    import torch
    coo, ck = setup[(cfg, mname)]
    dev = ck.to_device()
    h, w = coo.shape
    a = coo.arrays()
    rowsum = np.zeros(h)
    np.add.at(rowsum, a["coo_row_id"], np.abs(a["coo_data"]))
    alpha = float(1.0 / max(rowsum.max(), 1.0))          # keeps ||x|| bounded over the steps
    x0 = torch.from_numpy(synth.x_vector(w)).cuda()
    y0 = torch.from_numpy(np.random.default_rng(7).standard_normal(h).astype(np.float32)).cuda()
    x1, y1 = x0.clone(), y0.clone()
    dev.iterate(x1, y1, k, alpha, 0.5)
    x2, y2 = x0.clone(), y0.clone()
    _iterate_by_steps(dev, x2, y2, k, alpha, 0.5)
    torch.cuda.synchronize()
    assert torch.equal(x1[:h], y1)
    exact = len(dev.parts) == 1 and dev.parts[0] in ("dia", "bdia", "ell", "bell", "sbell", "bcsr")
    if exact:
        assert torch.equal(y1, y2), dev.parts
    else:
        scale = float(y2.abs().max()) + 1e-30
        assert float((y1 - y2).abs().max()) <= 1e-4 * scale, dev.parts


def test_cocktail_iterate_against_oracle(setup):
    """Three reference steps (alpha = beta = 1) against the oracle's csr_spmv
    run three times on the host."""
    import torch
    coo, ck = setup[("block_partial", "mixed")]
    dev = ck.to_device()
    h, w = coo.shape
    x = synth.x_vector(w) * np.float32(0.05)
    y = np.zeros(h, np.float32)
    xd, yd = torch.from_numpy(x.copy()).cuda(), torch.from_numpy(y.copy()).cuda()
    dev.iterate(xd, yd, 3)
    torch.cuda.synchronize()
    xs, ys = x.copy(), y.copy()
    for _ in range(3):
        y_ref, _, bound = reference_y(coo, xs, ys)
        ys = y_ref.astype(np.float32)
        xs[:h] = ys
    scale = np.abs(ys).max() + 1e-30
    assert np.abs(yd.cpu().numpy() - ys).max() <= 1e-4 * scale


def test_cocktail_iterate_rejects_aliasing(setup):
    import torch
    from clspmv_mic_b200 import _abi
    coo, ck = setup[("plain", "laplace128")]
    dev = ck.to_device()
    v = torch.zeros(max(coo.shape), device="cuda")
    with pytest.raises(_abi.ClspmvError) as e:
        dev.iterate(v, v, 2)
    assert e.value.status == _abi.ERR_ARG


@pytest.mark.parametrize("cfg,mname", [("block_partial", "mixed"), ("dia_flat", "band_noise")])
def test_cocktail_flat_part_as_csr(setup, cfg, mname):
    """The tuner's CSR storage of the flat part runs through the Cocktail
    runtime (chunked CSR kernel) to the same y within the 1e-5 row bound."""
    import torch
    coo, ck = setup[(cfg, mname)]
    alt = ck.with_flat_as_csr()
    if alt is None:
        pytest.skip(f"no COO part: {ck.summary()}")
    dev = alt.to_device()
    x = synth.x_vector(coo.shape[1])
    y0 = np.random.default_rng(5).standard_normal(coo.shape[0]).astype(np.float32)
    xd, yd = torch.from_numpy(x).cuda(), torch.from_numpy(y0.copy()).cuda()
    dev.spmv(xd, yd, 1.0, 1.0)
    torch.cuda.synchronize()
    y_ref, _, bound = reference_y(coo, x, y0, 1.0, 1.0)
    assert_close(yd.cpu().numpy(), y_ref, bound, f"flat as csr {cfg}/{mname} parts={dev.parts}")


def _cocktail_of(pieces, converters, n, seed=8):
    """CocktailMatrix whose slots hold the given (row, col) key sets
    (key = row * n + col), converted by `converters`; and the whole matrix."""
    from clspmv_mic_b200 import _abi
    rng = np.random.default_rng(seed)
    st = _abi.Cocktail()
    st.mat_width = st.mat_height = n
    keep = []
    for sl, keys in pieces.items():
        keys = np.sort(keys)
        part_coo = F.coo_matrix(n, n, keys // n, keys % n, rng.standard_normal(keys.size).astype(np.float32))
        host = converters[sl](part_coo)
        keep.append((part_coo, host))
        setattr(st, f"ifuse{sl}", True)
        setattr(st, sl, type(getattr(st, sl)).from_buffer_copy(host.struct))
    st.mat_nnz = int(sum(k.size for k in pieces.values()))
    ck = CK.CocktailMatrix(st, owner=None)
    ck._keep = keep
    rows = np.concatenate([pc.array("coo_row_id") for pc, _ in keep])
    cols = np.concatenate([pc.array("coo_col_id") for pc, _ in keep])
    vals = np.concatenate([pc.array("coo_data") for pc, _ in keep])
    o = np.lexsort((cols, rows))
    return F.coo_matrix(n, n, rows[o], cols[o], vals[o]), ck


@pytest.mark.parametrize("with_dia", [False, True])
@pytest.mark.parametrize("sh", [32, 8])
def test_cocktail_sell_part_planned(with_dia, sh):
    """A SELL part of uneven rows (24 rows of 500-900 entries among rows of
    0-3) runs through its length plan, made at upload, alone (its own y
    update) and beside a DIA part (atomic adds into a y with beta applied
    first), against the oracle; a SELL part of even rows keeps the padded
    read."""
    import torch
    n = 4096
    rng = np.random.default_rng(sh + with_dia)
    r = np.arange(n)
    band = np.unique(np.concatenate([r * n + r, r[1:] * n + r[1:] - 1, r[:-1] * n + r[:-1] + 1]))
    keys = []
    for row in rng.choice(n, 24, replace=False):
        keys.append(row * n + rng.choice(n, int(rng.integers(500, 900)), replace=False))
    keys.append(r * n + rng.integers(0, n, n))
    sell = np.unique(np.concatenate(keys))
    sell = sell[~np.isin(sell, band)]
    pieces = {"dia": band, "sell": sell} if with_dia else {"sell": sell}
    conv = {"dia": F.coo2dia, "sell": lambda c: F.coo2sell(c, sh)}
    coo, ck = _cocktail_of(pieces, conv, n)
    dev = ck.to_device()
    assert dev.sell_planned
    x = synth.x_vector(n)
    y0 = np.random.default_rng(2).standard_normal(n).astype(np.float32)
    for alpha, beta in [(1.0, 0.0), (1.5, -0.5)]:
        xd, yd = torch.from_numpy(x).cuda(), torch.from_numpy(y0.copy()).cuda()
        dev.spmv(xd, yd, alpha, beta)
        torch.cuda.synchronize()
        y_ref, _, bound = reference_y(coo, x, y0, alpha, beta)
        assert_close(yd.cpu().numpy(), y_ref, bound, f"sell{sh} planned, dia={with_dia}")
    even = np.unique(r * n + (r * 7) % n)
    _, ck2 = _cocktail_of({"sell": even}, conv, n)
    assert not ck2.to_device().sell_planned
