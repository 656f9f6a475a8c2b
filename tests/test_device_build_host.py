"""Device-side format builders, run on the CPU device: array lengths and
index ranges match what the kernels and the library's host code read."""
import numpy as np
import pytest

from clspmv_mic_b200 import device_build as D
from clspmv_mic_b200 import formats as F


def _np(m, f):
    return m.tensors[f].numpy()


@pytest.mark.parametrize("rows", [1000, 1023, 4096])
def test_diagonal_and_flat(rows):
    m = D.dia(rows, 7, device="cpu")
    s = m.struct
    assert s.dia_length_aligned % 4 == 0 and s.dia_length_aligned >= rows
    assert _np(m, "dia_data").size == 7 * s.dia_length_aligned
    b = D.bdia(rows, 11, device="cpu")
    bp = _np(b, "bdia_bptr")
    assert bp[0] == 0 and bp[-1] == 11 and np.all(np.diff(bp) > 0) and b.struct.bdia_band_num == len(bp) - 1
    assert _np(b, "bdia_data").size == bp[-1] * b.struct.bdia_length_aligned
    e = D.ell(rows, 5, device="cpu")
    assert _np(e, "ell_col_id").size == 5 * e.struct.ell_height_aligned and _np(e, "ell_col_id").max() < rows
    for sh in (32, 128):
        sl = D.sell(rows, 6, sh, device="cpu")
        ptr = _np(sl, "sell_slice_ptr")
        assert sl.struct.sell_slice_num * sh >= rows and ptr[-1] == _np(sl, "sell_data").size
        assert np.all(np.diff(ptr) == sh * 6)
    c = D.coo(rows, 9, device="cpu")
    r = _np(c, "coo_row_id")
    assert c.nnz == rows * 9 and np.all(np.diff(r) >= 0) and r[-1] == rows - 1


@pytest.mark.parametrize("bh,bw", F.BLOCK_SHAPES)
def test_block_formats(bh, bw):
    rows, blocks = 2000, 3
    nbr = (rows + bh - 1) // bh
    m = D.b4csr(rows, blocks, bh, bw, device="cpu")
    s = m.struct
    nb = s.b4csr_block_num
    assert nb == nbr * blocks and s.b4csr_aligned_size >= 4 * nb and s.b4csr_aligned_size % 4 == 0
    assert _np(m, "b4csr_data").size == (bw // 4) * bh * s.b4csr_aligned_size
    c4 = _np(m, "b4csr_col_id")
    assert c4.min() >= 0 and (c4.max() + bw // 4) * 4 <= rows + bw and np.all(c4 % (bw // 4) == 0)
    e = D.b4ell(rows, blocks, bh, bw, device="cpu")
    s = e.struct
    assert s.b4ell_height_aligned >= nbr and s.b4ell_float4_aligned >= 4 * nbr and s.b4ell_float4_aligned % 4 == 0
    assert _np(e, "b4ell_col_id").size == blocks * s.b4ell_height_aligned
    assert _np(e, "b4ell_data").size == blocks * s.b4ell_float4_aligned * (bw // 4) * bh
    sb = D.sbell(rows, blocks, bh, bw, device="cpu")
    s = sb.struct
    ptr = _np(sb, "sbell_slice_ptr")
    assert s.sbell_slice_num * s.sbell_slice_height >= nbr
    assert _np(sb, "sbell_col_id").size == ptr[-1] and _np(sb, "sbell_data").size == ptr[-1] * bw * bh
