"""Device-side generators, run on the CPU device (no GPU needed)."""
import pytest

from clspmv_mic_b200 import synth


@pytest.mark.parametrize("structure", ["random", "banded", "blocked"])
def test_device_csr_structure(structure):
    import torch
    m = synth.device_csr(777, 901, 3, 17, structure, seed=5, device="cpu")
    rp, col, val = m.tensors["csr_row_ptr"], m.tensors["csr_col_id"], m.tensors["csr_data"]
    assert rp.dtype == torch.int32 and col.dtype == torch.int32 and val.dtype == torch.float32
    assert int(rp[0]) == 0 and int(rp[-1]) == m.nnz == col.numel() == val.numel()
    lens = rp[1:] - rp[:-1]
    assert bool((lens >= 3).all()) and bool((lens <= 20).all())
    assert int(col.min()) >= 0 and int(col.max()) < 901
    assert m.shape == (777, 901)
    assert m.stored_bytes == 4 * (778 + 2 * m.nnz)
    if structure == "blocked":
        assert bool((lens % 4 == 0).all())
    again = synth.device_csr(777, 901, 3, 17, structure, seed=5, device="cpu")
    assert torch.equal(again.tensors["csr_col_id"], col)
