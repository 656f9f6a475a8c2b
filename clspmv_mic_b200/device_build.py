"""Format matrices built directly on the device, in the converters' layouts.

The benchmark-table measurements need hundreds of matrices of every format
at sizes up to millions of rows; converting each on the host would take
longer than measuring it. These builders write the device arrays of a
regular synthetic matrix of each format straight away (random values,
random or banded columns), with the same array lengths, alignments and
index conventions as the host converters of include/matrix_storage.h, so
the library's kernels read them exactly as they read converted matrices.
"""
from __future__ import annotations

from .formats import DeviceMatrix

ALIGN = 32   # GPU_ALIGNMENT (include/constant.h:17)


def _al(n: int, a: int = ALIGN) -> int:
    return (n + a - 1) // a * a


def _gen(seed, device):
    import torch
    g = torch.Generator(device=device)
    g.manual_seed(int(seed))
    return g


def dia(rows: int, ndiag: int, seed: int = 1, device="cuda") -> DeviceMatrix:
    """ndiag diagonals centred on the main one."""
    import torch
    g = _gen(seed, device)
    ln = _al(rows)
    offs = torch.arange(ndiag, dtype=torch.int32, device=device) - ndiag // 2
    data = torch.randn(ndiag * ln, generator=g, device=device)
    return DeviceMatrix.from_device_arrays("dia", dict(width=rows, height=rows, nnz=rows * ndiag, dia_num=ndiag,
                                                       dia_length=rows, dia_length_aligned=ln),
                                           dict(dia_offsets=offs, dia_data=data))


def bdia(rows: int, ndiag: int, band: int = 3, seed: int = 1, device="cuda") -> DeviceMatrix:
    """ndiag diagonals in bands of `band` adjacent diagonals, bands spread
    around the main diagonal."""
    import torch
    g = _gen(seed, device)
    ln = _al(rows)
    nb = (ndiag + band - 1) // band
    widths = [band] * (ndiag // band) + ([ndiag % band] if ndiag % band else [])
    offs, bptr, start = [], [0], -(nb // 2) * (band + 4)
    for w in widths:
        offs.append(start)
        bptr.append(bptr[-1] + w)
        start += w + 4
    data = torch.randn(ndiag * ln, generator=g, device=device)
    return DeviceMatrix.from_device_arrays(
        "bdia", dict(width=rows, height=rows, nnz=rows * ndiag, bdia_band_num=len(widths), bdia_length=rows,
                     bdia_length_aligned=ln),
        dict(bdia_offsets=torch.tensor(offs, dtype=torch.int32, device=device),
             bdia_bptr=torch.tensor(bptr, dtype=torch.int32, device=device), bdia_data=data))


def ell(rows: int, width: int, seed: int = 1, device="cuda") -> DeviceMatrix:
    import torch
    g = _gen(seed, device)
    ln = _al(rows)
    col = torch.randint(0, rows, (width * ln,), generator=g, device=device, dtype=torch.int32)
    data = torch.randn(width * ln, generator=g, device=device)
    return DeviceMatrix.from_device_arrays("ell", dict(width=rows, height=rows, nnz=rows * width, ell_num=width,
                                                       ell_height_aligned=ln),
                                           dict(ell_col_id=col, ell_data=data))


def sell(rows: int, width: int, slice_height: int = 32, seed: int = 1, device="cuda") -> DeviceMatrix:
    import torch
    g = _gen(seed, device)
    ns = (rows + slice_height - 1) // slice_height
    ptr = torch.arange(ns + 1, dtype=torch.int32, device=device) * (slice_height * width)
    n = ns * slice_height * width
    col = torch.randint(0, rows, (n,), generator=g, device=device, dtype=torch.int32)
    data = torch.randn(n, generator=g, device=device)
    return DeviceMatrix.from_device_arrays("sell", dict(width=rows, height=rows, nnz=rows * width,
                                                        sell_slice_height=slice_height, sell_slice_num=ns),
                                           dict(sell_slice_ptr=ptr, sell_col_id=col, sell_data=data))


def csr(rows: int, width: int, seed: int = 1, device="cuda") -> DeviceMatrix:
    from .synth import device_csr
    return device_csr(rows, rows, width, width, "random", seed=seed, device=device)


def coo(rows: int, width: int, seed: int = 1, device="cuda") -> DeviceMatrix:
    """Row-sorted COO with `width` entries per row."""
    import torch
    m = csr(rows, width, seed, device)
    rp = m.tensors["csr_row_ptr"].long()
    row = torch.repeat_interleave(torch.arange(rows, device=device, dtype=torch.int32), rp[1:] - rp[:-1])
    return DeviceMatrix.from_device_arrays("coo", dict(width=rows, height=rows, nnz=m.nnz),
                                           dict(coo_row_id=row, coo_col_id=m.tensors["csr_col_id"],
                                                coo_data=m.tensors["csr_data"]))


def _block_cols(nbrow: int, per_row: int, cols: int, bw: int, g, device):
    import torch
    nbc = max(1, cols // bw)
    return (torch.randint(0, nbc, (nbrow * per_row,), generator=g, device=device, dtype=torch.int32) * (bw // 4))


def b4csr(rows: int, blocks: int, bh: int, bw: int, seed: int = 1, device="cuda") -> DeviceMatrix:
    """`blocks` bh x bw blocks per block row (column ids in float4 units)."""
    import torch
    g = _gen(seed, device)
    nbr = (rows + bh - 1) // bh
    nb = nbr * blocks
    ln = _al(4 * nb)
    rp = torch.arange(nbr + 1, dtype=torch.int32, device=device) * blocks
    col = _block_cols(nbr, blocks, rows, bw, g, device)
    data = torch.randn((bw // 4) * bh * ln, generator=g, device=device)
    return DeviceMatrix.from_device_arrays(
        "b4csr", dict(width=rows, height=rows, nnz=rows * blocks * bw, b4csr_bwidth=bw, b4csr_bheight=bh,
                      b4csr_row_num=nbr, b4csr_aligned_size=ln, b4csr_block_num=nb),
        dict(b4csr_row_ptr=rp, b4csr_col_id=col, b4csr_data=data))


def b4ell(rows: int, blocks: int, bh: int, bw: int, seed: int = 1, device="cuda") -> DeviceMatrix:
    import torch
    g = _gen(seed, device)
    nbr = (rows + bh - 1) // bh
    ln, f4 = _al(nbr), _al(4 * nbr)
    col = _block_cols(ln, blocks, rows, bw, g, device)
    data = torch.randn(blocks * f4 * (bw // 4) * bh, generator=g, device=device)
    return DeviceMatrix.from_device_arrays(
        "b4ell", dict(width=rows, height=rows, nnz=rows * blocks * bw, b4ell_bwidth=bw, b4ell_bheight=bh,
                      b4ell_row_num=nbr, b4ell_block_num=blocks, b4ell_height_aligned=ln, b4ell_float4_aligned=f4),
        dict(b4ell_col_id=col, b4ell_data=data))


def sbell(rows: int, blocks: int, bh: int, bw: int, slice_height: int = 32, seed: int = 1, device="cuda") -> DeviceMatrix:
    import torch
    g = _gen(seed, device)
    nbr = (rows + bh - 1) // bh
    ns = (nbr + slice_height - 1) // slice_height
    ptr = torch.arange(ns + 1, dtype=torch.int32, device=device) * (slice_height * blocks)
    nblk = ns * slice_height * blocks
    col = _block_cols(ns * slice_height, blocks, rows, bw, g, device)
    data = torch.randn(nblk * bw * bh, generator=g, device=device)
    return DeviceMatrix.from_device_arrays(
        "sbell", dict(width=rows, height=rows, nnz=rows * blocks * bw, sbell_bwidth=bw, sbell_bheight=bh,
                      sbell_slice_height=slice_height, sbell_slice_num=ns, sbell_row_num=nbr),
        dict(sbell_slice_ptr=ptr, sbell_col_id=col, sbell_data=data))
