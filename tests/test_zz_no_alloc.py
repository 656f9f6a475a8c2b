"""The merge-path CSR entry point that keeps its tile plan in a static
device array (clspmv_csr_merge_spmv_noalloc_f32), called through the C ABI.

It must give the same y as clspmv_csr_merge_spmv_f32 with a caller-made
plan, on two calls in a row (the second reusing the array the first one
filled), and reject matrices beyond its fixed plan size before launching
anything. This file is named to be collected last, so it also runs after
every other GPU test in the same process; it passes on its own as well.
"""
import ctypes as C

import numpy as np
import pytest

from clspmv_mic_b200 import _abi
from clspmv_mic_b200 import formats as F
from clspmv_mic_b200 import synth

from gpu_util import assert_close, reference_y
from matrices import coo_of

pytestmark = pytest.mark.gpu


def _entry():
    L = _abi.lib()
    fn = L.clspmv_csr_merge_spmv_noalloc_f32
    fn.restype = C.c_int
    fn.argtypes = [C.POINTER(_abi.Csr), C.c_void_p, C.c_void_p, C.c_float, C.c_float, C.c_void_p]
    L.clspmv_csr_merge_noalloc_max_tiles.restype = C.c_int
    return fn, L.clspmv_csr_merge_noalloc_max_tiles()


def _device_csr(coo):
    return F.DeviceMatrix(F.coo2csr(coo))


@pytest.mark.parametrize("name,alpha,beta", [("powerlaw3k", 1.0, 1.0), ("laplace33", 1.5, 0.0),
                                             ("random_empty_rows", -0.5, 2.0), ("blocks_odd", 1.0, 1.0)])
def test_noalloc_matches_merge_twice(name, alpha, beta):
    import torch
    fn, _ = _entry()
    coo = coo_of(name)
    h, w = coo.shape
    dev = _device_csr(coo)
    x = torch.from_numpy(synth.x_vector(w, seed=5)).cuda()
    y0 = np.random.default_rng(8).uniform(-1, 1, h).astype(np.float32)
    y_ref, _, bound = reference_y(coo, x.cpu().numpy(), y0, alpha, beta)
    ya = torch.from_numpy(y0).cuda()
    dev.spmv(x, ya, alpha, beta, variant="merge")
    s = torch.cuda.current_stream().cuda_stream
    for call in range(2):
        yb = torch.from_numpy(y0).cuda()
        assert fn(C.byref(dev.struct), x.data_ptr(), yb.data_ptr(), alpha, beta, s) == _abi.OK
        torch.cuda.synchronize()
        got, base = yb.cpu().numpy(), ya.cpu().numpy()
        assert_close(got, base, bound, f"{name} call {call + 1} vs clspmv_csr_merge_spmv_f32")
        assert_close(got, y_ref, bound, f"{name} call {call + 1} vs oracle")


def test_noalloc_large_matrix_fills_more_of_the_plan():
    import torch
    fn, max_tiles = _entry()
    h, w, r, c, v = synth.powerlaw(1 << 18, maxlen=4000, seed=21)
    coo = F.coo_matrix(h, w, r, c, v)
    assert F.if_sorted_coo(coo)
    tiles = _abi.lib().clspmv_csr_merge_tiles(h, coo.nnz)
    assert 100 < tiles <= max_tiles
    dev = _device_csr(coo)
    x = torch.from_numpy(synth.x_vector(w, seed=2)).cuda()
    ya = torch.zeros(h, device="cuda")
    dev.spmv(x, ya, 1.0, 0.0, variant="merge")
    s = torch.cuda.current_stream().cuda_stream
    _, _, bound = reference_y(coo, x.cpu().numpy(), None, 1.0, 0.0)
    for _ in range(2):
        yb = torch.full((h,), 7.0, device="cuda")
        assert fn(C.byref(dev.struct), x.data_ptr(), yb.data_ptr(), 1.0, 0.0, s) == _abi.OK
        torch.cuda.synchronize()
        assert_close(yb.cpu().numpy(), ya.cpu().numpy(), bound, "large")


def test_noalloc_rejects_beyond_plan_size():
    import torch
    fn, max_tiles = _entry()
    dev = _device_csr(coo_of("laplace16"))
    big = type(dev.struct).from_buffer_copy(dev.struct)
    big.matinfo.height = 1 << 26
    big.matinfo.nnz = max_tiles * 2048      # rows + nnz beyond max_tiles * 2048
    x = torch.zeros(4, device="cuda")
    y = torch.zeros(4, device="cuda")
    n0 = F.launch_count()
    assert fn(C.byref(big), x.data_ptr(), y.data_ptr(), 1.0, 1.0, None) == _abi.ERR_UNSUPPORTED
    assert F.launch_count() == n0
    assert fn(None, x.data_ptr(), y.data_ptr(), 1.0, 1.0, None) == _abi.ERR_ARG
