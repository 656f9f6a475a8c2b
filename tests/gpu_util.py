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


def columns_reference(coo, X, alpha=1.0):
    """Per column j of X: y32 = alpha * csr_spmv(A, X[:, j]) (the oracle's
    FP32 routine), y64 (FP64) and the row scale |alpha| sum_i |a_ri X[i, j]|;
    arrays of shape (rows, k)."""
    csr = F.coo2csr(coo)
    X = np.asarray(X, dtype=np.float32)
    y32, y64, sc = [], [], []
    for j in range(X.shape[1]):
        xj = np.ascontiguousarray(X[:, j])
        y32.append(np.float32(alpha) * O.spmv_port(csr, xj))
        a, b = O.csr_f64(csr, xj)
        y64.append(alpha * a)
        sc.append(abs(alpha) * b)
    return np.stack(y32, 1), np.stack(y64, 1), np.stack(sc, 1)


# per-row bounds by value type: FP32 values against the FP32 oracle; 16-bit
# values (rounded to 2^-9 / 2^-11 relative with a per-row power-of-two
# scale) against FP64
VALUE_RTOL = {"f32": RTOL, "bf16": 2.0 ** -8, "f16": 2.0 ** -10}


def assert_columns_close(got, ref, value_type="f32", what=""):
    """got (rows x k) within the per-row, per-column bound of `ref` =
    columns_reference(...): |got - y32| <= 1e-5 scale for FP32 values,
    |got - y64| <= 2^-8 / 2^-10 scale for BF16 / FP16."""
    y32, y64, sc = ref
    g = np.asarray(got, dtype=np.float64)
    err = np.abs(g - (y32.astype(np.float64) if value_type == "f32" else y64))
    lim = VALUE_RTOL[value_type] * sc + 1e-30
    bad = np.argwhere(err > lim)
    assert bad.size == 0, f"{what}: {len(bad)} entries outside the {value_type} row bound, first {bad[:3].tolist()}"
