"""Argument checks of the tensor-core b4csr product, without a GPU: every
refusal is decided on the host before any CUDA call, so fake device pointers
are never dereferenced."""
import ctypes as C

import pytest

from clspmv_mic_b200 import _abi
from clspmv_mic_b200.formats import lib


def _struct(bw=4, bh=4, rows=64, aligned=256, data=0x1000):
    s = _abi.B4csr()
    s.matinfo.width = s.matinfo.height = rows
    s.b4csr_bwidth, s.b4csr_bheight = bw, bh
    s.b4csr_row_num, s.b4csr_aligned_size, s.b4csr_block_num = rows // 4, aligned, 16
    s.b4csr_row_ptr, s.b4csr_col_id, s.b4csr_data = 0x2000, 0x3000, data
    return s


@pytest.mark.parametrize("kw,k,ldx,ldy,x,status", [
    ({}, 8, 8, 8, 0x4000, _abi.ERR_UNSUPPORTED),          # fewer than 16 right-hand sides
    ({}, 20, 20, 20, 0x4000, _abi.ERR_UNSUPPORTED),       # not a multiple of 16
    ({}, 144, 144, 144, 0x4000, _abi.ERR_UNSUPPORTED),    # more than 128
    ({"bw": 8}, 16, 16, 16, 0x4000, _abi.ERR_UNSUPPORTED),
    ({"bh": 2}, 16, 16, 16, 0x4000, _abi.ERR_UNSUPPORTED),
    ({}, 16, 18, 16, 0x4000, _abi.ERR_ALIGN),             # ldx not a multiple of 4
    ({}, 16, 16, 16, 0x4004, _abi.ERR_ALIGN),             # X not 16-byte aligned
    ({"data": 0x1008}, 16, 16, 16, 0x4000, _abi.ERR_ALIGN),
    ({"aligned": 258}, 16, 16, 16, 0x4000, _abi.ERR_ALIGN),
    ({}, 16, 8, 16, 0x4000, _abi.ERR_ARG),                # ldx < k
    ({}, 16, 16, 16, 0, _abi.ERR_ARG),                    # no X
])
def test_refusals(kw, k, ldx, ldy, x, status):
    s = _struct(**kw)
    rc = lib().clspmv_b4csr_spmm_tc_f32(C.byref(s), k, C.c_void_p(x), ldx, C.c_void_p(0x5000), ldy,
                                        C.c_float(1.0), C.c_float(0.0), None)
    assert rc == status


def test_empty_matrix_is_a_no_op():
    s = _struct(rows=0)
    rc = lib().clspmv_b4csr_spmm_tc_f32(C.byref(s), 16, C.c_void_p(0x4000), 16, C.c_void_p(0x5000), 16,
                                        C.c_float(1.0), C.c_float(0.0), None)
    assert rc == _abi.OK
