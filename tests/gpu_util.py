"""Helpers for the -m gpu parity tests."""
import numpy as np

from clspmv_mic_b200 import formats as F
from clspmv_mic_b200 import synth
from oracle import oracle as O

RTOL = 1e-5   # per-row bound: |y - y_ref| <= RTOL * sum_j |a_ij x_j|


def run_device(host, x, y0, alpha=1.0, beta=1.0, **kw):
    import torch
    dev = F.DeviceMatrix(host)
    xd = torch.from_numpy(np.ascontiguousarray(x, dtype=np.float32)).cuda()
    yd = torch.from_numpy(np.ascontiguousarray(y0, dtype=np.float32)).cuda()
    dev.spmv(xd, yd, alpha, beta, **kw)
    torch.cuda.synchronize()
    return yd.cpu().numpy()


def reference_y(coo, x, y0=None, alpha=1.0, beta=1.0):
    """y_ref = alpha * csr_spmv(A, x) + beta * y0 (csr_spmv of the C oracle,
    FP32, result initialised to 0), the FP64 values and the row scale."""
    csr = F.coo2csr(coo)
    ax = O.spmv_port(csr, x)
    y64, scale = O.csr_f64(csr, x)
    h = coo.shape[0]
    y0 = np.zeros(h, np.float32) if y0 is None else y0
    y_ref = (np.float32(alpha) * ax + (np.float32(beta) * y0 if beta != 0 else 0)).astype(np.float32)
    y64 = alpha * y64 + (beta * y0.astype(np.float64) if beta != 0 else 0)
    bound = abs(alpha) * scale + (abs(beta) * np.abs(y0.astype(np.float64)) if beta != 0 else 0)
    return y_ref, y64, bound


def assert_close(y, y_ref, bound, what=""):
    err = np.abs(y.astype(np.float64) - y_ref.astype(np.float64))
    lim = RTOL * bound + 1e-30
    bad = np.nonzero(err > lim)[0]
    assert bad.size == 0, f"{what}: {bad.size} rows outside 1e-5 bound, first {bad[:5]}, err {err[bad[:5]]}, lim {lim[bad[:5]]}"


def fp64_error(y, y64, bound):
    """max over rows of |y - y64| / sum|a x| (reported, not asserted)."""
    with np.errstate(divide="ignore", invalid="ignore"):
        r = np.abs(y.astype(np.float64) - y64) / np.where(bound > 0, bound, 1.0)
    return float(np.max(r)) if r.size else 0.0
