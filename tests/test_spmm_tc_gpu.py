"""b4csr (4 x 4 blocks) times k >= 16 right-hand sides on the tensor cores.

Same oracle and bound as the other SpMM tests: the FP64 restatement of the
reference's csr_spmv (oracle/) column by column, every entry within
1e-5 * (|alpha| sum_j |a_ij x_jc| + |beta y_ic|). The TF32 head-and-remainder
split keeps each product to about 2^-21 of |a x|, so the test also states
the largest error seen. Covers ragged edges (rows and columns not multiples
of 4), empty block rows, right-hand sides over the 64 of one launch, padded
leading dimensions, alpha / beta, and that no bounded wait ran out.
"""
import numpy as np
import pytest

from clspmv_mic_b200 import formats as F
from clspmv_mic_b200 import _abi

from matrices import coo_of
from test_spmm_gpu import RTOL, spmm_reference

pytestmark = pytest.mark.gpu

MATRICES = ["blocks300", "blocks_odd", "laplace33", "random_empty_rows", "ragged_tail", "one_entry", "tall"]


def _tc(name, k, alpha=1.0, beta=0.0, ldx_pad=0, ldy_pad=0, seed=0):
    import torch
    coo = coo_of(name)
    m, n = coo.shape
    rng = np.random.default_rng(seed + k)
    X = rng.uniform(-1, 1, (n, k)).astype(np.float32)
    Y0 = rng.uniform(-1, 1, (m, k)).astype(np.float32)
    host = F.coo2b4csr(coo, 4, 4)
    dev = F.DeviceMatrix(host)
    Xd = torch.zeros((n, k + ldx_pad), dtype=torch.float32, device="cuda")
    Xd[:, :k] = torch.from_numpy(X)
    Yd = torch.zeros((m, k + ldy_pad), dtype=torch.float32, device="cuda")
    Yd[:, :k] = torch.from_numpy(Y0)
    F.device_spmm_tc(dev, Xd[:, :k], Yd[:, :k], alpha, beta)
    torch.cuda.synchronize()
    assert F.tensor_timeouts() == 0
    got = Yd[:, :k].cpu().numpy().astype(np.float64)
    ref, bound = spmm_reference(coo, X, Y0, alpha, beta)
    err = np.abs(got - ref)
    bad = np.argwhere(err > RTOL["f32"] * bound + 1e-30)
    assert bad.size == 0, f"{name} k={k}: {len(bad)} entries off, first {bad[:3].tolist()}"
    if ldy_pad:   # the padding columns of Y are not touched
        assert np.all(Yd[:, k:].cpu().numpy() == 0)
    return float(np.max(err / np.where(bound > 0, bound, 1.0)))


@pytest.mark.parametrize("name", MATRICES)
@pytest.mark.parametrize("k", [16, 32, 48, 64])
def test_tc_matches_oracle(name, k):
    rel = _tc(name, k)
    assert rel < 1e-6   # the split leaves about 2^-21 per product


@pytest.mark.parametrize("k,alpha,beta,ldx_pad,ldy_pad", [(80, 1.0, 1.0, 0, 0), (128, 0.5, -2.0, 4, 3),
                                                          (16, -1.0, 0.25, 8, 1), (96, 2.0, 0.0, 0, 0)])
def test_tc_scalars_and_leading_dims(k, alpha, beta, ldx_pad, ldy_pad):
    _tc("blocks300", k, alpha, beta, ldx_pad, ldy_pad)
    _tc("random_empty_rows", k, alpha, beta, ldx_pad, ldy_pad, seed=1)


def test_tc_agrees_with_cuda_core_kernel():
    """The same product through clspmv_spmm's lane-group kernel: both FP32-accurate."""
    import torch
    coo = coo_of("blocks300")
    dev = F.DeviceMatrix(F.coo2b4csr(coo, 4, 4))
    n, m = coo.shape[1], coo.shape[0]
    X = torch.rand((n, 32), device="cuda") * 2 - 1
    Y1 = torch.zeros((m, 32), device="cuda")
    Y2 = torch.zeros((m, 32), device="cuda")
    F.device_spmm_tc(dev, X, Y1)
    dev.spmm(X, Y2)
    torch.cuda.synchronize()
    _, bound = spmm_reference(coo, X.cpu().numpy(), np.zeros((m, 32), np.float32), 1.0, 0.0)
    assert np.all(np.abs(Y1.cpu().numpy() - Y2.cpu().numpy()) <= 2e-5 * bound + 1e-30)


def test_tc_many_tiles_and_repeats():
    """Enough block rows for every CTA to run several tiles (stage reuse
    across tiles), run twice: identical results (no atomics, fixed order)."""
    import torch
    from clspmv_mic_b200 import synth
    coo = F.coo_matrix(*synth.block_rows(40_000, 6, 4, 4, seed=8))
    dev = F.DeviceMatrix(F.coo2b4csr(coo, 4, 4))
    n, m = coo.shape[1], coo.shape[0]
    g = torch.Generator(device="cuda").manual_seed(3)
    X = torch.rand((n, 32), device="cuda", generator=g) * 2 - 1
    Y1 = torch.zeros((m, 32), device="cuda")
    Y2 = torch.zeros((m, 32), device="cuda")
    F.device_spmm_tc(dev, X, Y1)
    F.device_spmm_tc(dev, X, Y2)
    torch.cuda.synchronize()
    assert F.tensor_timeouts() == 0
    assert torch.equal(Y1, Y2)
    Xh = X.cpu().numpy()
    rows = np.arange(0, m, 997)
    ref, bound = spmm_reference(coo, Xh, np.zeros((m, 32), np.float32), 1.0, 0.0)
    err = np.abs(Y1.cpu().numpy()[rows] - ref[rows])
    assert np.all(err <= RTOL["f32"] * bound[rows] + 1e-30)


def test_tc_rejects_unsupported():
    import torch
    coo = coo_of("blocks300")
    dev = F.DeviceMatrix(F.coo2b4csr(coo, 4, 4))
    n, m = coo.shape[1], coo.shape[0]
    for k in (8, 20):
        with pytest.raises(_abi.ClspmvError):
            F.device_spmm_tc(dev, torch.zeros((n, k), device="cuda"), torch.zeros((m, k), device="cuda"))
    wide = F.DeviceMatrix(F.coo2b4csr(coo, 8, 4))
    with pytest.raises(_abi.ClspmvError):
        F.device_spmm_tc(wide, torch.zeros((n, 16), device="cuda"), torch.zeros((m, 16), device="cuda"))
