"""Seeded synthetic matrices of the benchmark shapes (row-sorted COO).

No public matrix collection is used by the reference's benchmarks (its
sample matrix is not shipped), so these generators are the workloads:

* laplacian_2d(256)        2D 5-point Laplacian, values 4 / -1
* stencil_27pt(128)        3D 27-point stencil, N(0,1) values
* powerlaw(2**20)          Zipf(2.0) row lengths on [1, 10000] rescaled to
                           mean 16, uniform random columns, N(0,1) values
* block_rows(500_000)      dense 4x4 blocks, 8 per block row, N(0,1)
* cocktail_mixed(...)      banded + blocked + power-law regions stacked

All return (height, width, row_id, col_id, data) numpy arrays sorted by
(row, col) without duplicates, plus the x vector helper.
"""
from __future__ import annotations

import numpy as np

SEED = 1234


def x_vector(n: int, seed: int = SEED) -> np.ndarray:
    """x ~ U[-1, 1] (float32)."""
    return np.random.default_rng(seed + 7).uniform(-1.0, 1.0, size=n).astype(np.float32)


def sorted_unique(a: np.ndarray) -> np.ndarray:
    """The distinct values of an integer array in ascending order (what
    np.unique returns; a sort and a neighbour compare, which at tens of
    millions of keys is many times faster than np.unique here)."""
    s = np.sort(a)
    if s.size == 0:
        return s
    keep = np.empty(s.size, dtype=bool)
    keep[0] = True
    np.not_equal(s[1:], s[:-1], out=keep[1:])
    return s[keep]


def _finish(h, w, rows, cols, vals):
    return (int(h), int(w), np.ascontiguousarray(rows, dtype=np.int32), np.ascontiguousarray(cols, dtype=np.int32),
            np.ascontiguousarray(vals, dtype=np.float32))


def laplacian_2d(n: int = 256):
    """5-point Laplacian on an n x n grid: 4 on the diagonal, -1 off it."""
    m = n * n
    r = np.arange(m, dtype=np.int64)
    i, j = r // n, r % n
    offs = np.array([-n, -1, 0, 1, n], dtype=np.int64)
    valid = np.stack([i > 0, j > 0, np.ones(m, bool), j < n - 1, i < n - 1], axis=1)
    cols = r[:, None] + offs[None, :]
    vals = np.where(offs == 0, 4.0, -1.0)[None, :].repeat(m, axis=0)
    rows = np.broadcast_to(r[:, None], cols.shape)
    return _finish(m, m, rows[valid], cols[valid], vals[valid])


def stencil_27pt(n: int = 128, seed: int = SEED):
    """27-point stencil on an n^3 grid (offsets dk*n^2 + dj*n + di), N(0,1)."""
    m = n ** 3
    r = np.arange(m, dtype=np.int64)
    k, j, i = r // (n * n), (r // n) % n, r % n
    d = np.array([-1, 0, 1])
    dk, dj, di = [a.ravel() for a in np.meshgrid(d, d, d, indexing="ij")]
    offs = dk * n * n + dj * n + di          # ascending in (dk, dj, di) order
    order = np.argsort(offs, kind="stable")
    dk, dj, di, offs = dk[order], dj[order], di[order], offs[order]
    valid = np.ones((m, 27), dtype=bool)
    for t in range(27):
        valid[:, t] = ((k + dk[t]) >= 0) & ((k + dk[t]) < n) & ((j + dj[t]) >= 0) & ((j + dj[t]) < n) & \
                      ((i + di[t]) >= 0) & ((i + di[t]) < n)
    cols = (r[:, None] + offs[None, :])[valid]
    rows = np.broadcast_to(r[:, None], valid.shape)[valid]
    vals = np.random.default_rng(seed).standard_normal(cols.size, dtype=np.float32)
    return _finish(m, m, rows, cols, vals)


def stencil_27pt_rows(n: int, r0: int, r1: int, seed: int = SEED):
    """Rows [r0, r1) of the 27-point stencil on an n^3 grid as CSR arrays
    (row_ptr rebased to 0, global column ids ascending in each row, values
    uniform in [-1, 1) from a generator seeded by (seed, r0)): one rank's
    slab, made without the rest of the matrix."""
    r = np.arange(r0, r1, dtype=np.int64)
    k, j, i = r // (n * n), (r // n) % n, r % n
    d = np.array([-1, 0, 1])
    dk, dj, di = [a.ravel() for a in np.meshgrid(d, d, d, indexing="ij")]
    offs = dk * n * n + dj * n + di
    order = np.argsort(offs, kind="stable")
    dk, dj, di, offs = dk[order], dj[order], di[order], offs[order]
    valid = np.ones((r.size, 27), dtype=bool)
    for t in range(27):
        valid[:, t] = ((k + dk[t]) >= 0) & ((k + dk[t]) < n) & ((j + dj[t]) >= 0) & ((j + dj[t]) < n) & \
                      ((i + di[t]) >= 0) & ((i + di[t]) < n)
    cols = (r[:, None] + offs[None, :])[valid]
    row_ptr = np.zeros(r.size + 1, dtype=np.int64)
    np.cumsum(valid.sum(axis=1), out=row_ptr[1:])
    vals = np.random.default_rng([seed, int(r0)]).uniform(-1.0, 1.0, size=cols.size).astype(np.float32)
    return row_ptr, cols.astype(np.int32), vals


def zipf_lengths(m: int, s: float, mean: float, maxlen: int, rng) -> np.ndarray:
    """Row lengths: k ~ Zipf(s) truncated to [1, maxlen], scaled by
    mean / E[k] and rounded, clipped to [1, maxlen]."""
    k = np.arange(1, maxlen + 1, dtype=np.float64)
    pmf = k ** (-s)
    pmf /= pmf.sum()
    scale = mean / float((pmf * k).sum())
    draw = rng.choice(np.arange(1, maxlen + 1), size=m, p=pmf)
    return np.clip(np.rint(draw * scale), 1, maxlen).astype(np.int64)


def powerlaw(m: int = 1 << 20, n: int | None = None, s: float = 2.0, mean: float = 16.0, maxlen: int = 10000,
             seed: int = SEED):
    """Power-law rows with uniform random distinct columns, N(0,1) values."""
    n = m if n is None else n
    rng = np.random.default_rng(seed)
    lens = zipf_lengths(m, s, mean, min(maxlen, n), rng)
    rows = np.repeat(np.arange(m, dtype=np.int64), lens)
    cols = rng.integers(0, n, size=rows.size, dtype=np.int64)
    key = sorted_unique(rows * n + cols)
    vals = rng.standard_normal(key.size, dtype=np.float32)
    return _finish(m, n, key // n, key % n, vals)


def block_rows(brows: int = 500_000, blocks_per_row: int = 8, bh: int = 4, bw: int = 4, seed: int = SEED):
    """Dense bh x bw blocks at bw-aligned block columns, blocks_per_row per
    block row. Block columns are drawn one per equal band of the block-column
    range, so they are distinct and sorted."""
    rng = np.random.default_rng(seed)
    n = brows * bh
    nbc = n // bw
    band = nbc // blocks_per_row
    bc = np.arange(blocks_per_row, dtype=np.int64)[None, :] * band + rng.integers(0, band, size=(brows, blocks_per_row))
    cols = (bc[:, None, :, None] * bw + np.arange(bw)[None, None, None, :])
    cols = np.broadcast_to(cols, (brows, bh, blocks_per_row, bw))
    rows = (np.arange(brows, dtype=np.int64)[:, None] * bh + np.arange(bh)[None, :])[:, :, None, None]
    rows = np.broadcast_to(rows, cols.shape)
    vals = rng.standard_normal(cols.size, dtype=np.float32)
    return _finish(n, n, rows.ravel(), cols.ravel(), vals)


def banded(m: int, ndiag: int = 7, seed: int = SEED):
    """ndiag consecutive diagonals centred on the main one, N(0,1)."""
    half = ndiag // 2
    r = np.arange(m, dtype=np.int64)
    offs = np.arange(-half, ndiag - half)
    cols = r[:, None] + offs[None, :]
    valid = (cols >= 0) & (cols < m)
    rows = np.broadcast_to(r[:, None], cols.shape)[valid]
    vals = np.random.default_rng(seed).standard_normal(int(valid.sum()), dtype=np.float32)
    return _finish(m, m, rows, cols[valid], vals)


def cocktail_mixed(band_rows: int = 1_500_000, block_region_rows: int = 1_500_000, power_rows: int = 1_000_000,
                   blocks_per_row: int = 6, power_s: float = 1.8, power_mean: float = 20.0, seed: int = SEED):
    """One square matrix stacking a 7-diagonal band region, a 4x4-block
    region (blocks_per_row blocks per block row, columns inside the region)
    and a power-law region (columns anywhere in the matrix)."""
    rng = np.random.default_rng(seed)
    m = band_rows + block_region_rows + power_rows
    parts = []
    # banded region: rows [0, band_rows)
    _, _, r, c, v = banded(band_rows, 7, seed)
    parts.append((r.astype(np.int64), c.astype(np.int64), v))
    # block region: rows [band_rows, band_rows + block_region_rows)
    o = band_rows
    brows = block_region_rows // 4
    _, _, r, c, v = block_rows(brows, blocks_per_row, 4, 4, seed + 1)
    parts.append((r.astype(np.int64) + o, c.astype(np.int64) + o, v))
    # power-law region: rows [o2, m), columns over the whole matrix
    o2 = band_rows + block_region_rows
    lens = zipf_lengths(power_rows, power_s, power_mean, 10000, rng)
    rows = np.repeat(np.arange(power_rows, dtype=np.int64), lens)
    cols = rng.integers(0, m, size=rows.size, dtype=np.int64)
    key = sorted_unique(rows * m + cols)
    parts.append((key // m + o2, key % m, rng.standard_normal(key.size, dtype=np.float32)))
    rows = np.concatenate([p[0] for p in parts])
    cols = np.concatenate([p[1] for p in parts])
    vals = np.concatenate([p[2] for p in parts])
    return _finish(m, m, rows, cols, vals)


def random_coo(m: int, n: int, density: float, seed: int = SEED, empty_row_frac: float = 0.0, value_dist: str = "normal"):
    """Uniform random sparsity with optional empty rows (test matrices)."""
    rng = np.random.default_rng(seed)
    nnz = int(round(m * n * density))
    key = sorted_unique(rng.integers(0, m * n, size=nnz, dtype=np.int64))
    rows, cols = key // n, key % n
    if empty_row_frac > 0:
        dead = rng.random(m) < empty_row_frac
        keep = ~dead[rows]
        rows, cols = rows[keep], cols[keep]
    if value_dist == "ones":
        vals = np.ones(rows.size, dtype=np.float32)
    else:
        vals = rng.standard_normal(rows.size, dtype=np.float32)
        vals[vals == 0] = 1.0
    return _finish(m, n, rows, cols, vals)


def device_csr(rows: int, cols: int, lo: int, hi: int, structure: str = "random", seed: int = SEED,
               device="cuda"):
    """A CSR matrix generated on the device (for workloads too large to
    build on the host): row lengths uniform in [lo, hi]; columns
    "random" (uniform; unsorted within a row and possibly repeated, both
    allowed by every CSR kernel), "banded" (a contiguous run centred on the
    diagonal, shifted to stay inside the matrix: sorted, distinct) or
    "blocked" (4 x 4 blocks: rows of a group of 4 share their block columns,
    lengths rounded up to whole blocks, block columns of a group ascending
    and distinct, so that the matrix converts exactly to the block formats);
    values N(0, 1)."""
    import torch
    from .formats import DeviceMatrix
    g = torch.Generator(device=device)
    g.manual_seed(int(seed))
    lens = torch.randint(lo, hi + 1, (rows,), generator=g, device=device, dtype=torch.int64)
    if structure == "blocked":
        lens = (lens + 3) // 4 * 4
    lens.clamp_(max=cols if structure != "blocked" else (cols // 4) * 4)
    row_ptr = torch.zeros(rows + 1, dtype=torch.int64, device=device)
    torch.cumsum(lens, 0, out=row_ptr[1:])
    nnz = int(row_ptr[-1].item())
    if nnz >= 2 ** 31:
        raise ValueError("more than 2^31 - 1 nonzeros")
    row_of = torch.repeat_interleave(torch.arange(rows, device=device), lens)
    pos = torch.arange(nnz, device=device) - row_ptr[:-1][row_of]
    if structure == "random":
        col = torch.randint(0, cols, (nnz,), generator=g, device=device, dtype=torch.int64)
    elif structure == "banded":
        centre = row_of * cols // rows
        start = (centre - lens[row_of] // 2).clamp_(min=0)
        start = torch.minimum(start, cols - lens[row_of])
        col = start + pos
    elif structure == "blocked":
        nbc = max(1, cols // 4)
        maxnb = max(1, (hi + 3) // 4)
        step = max(1, nbc // (2 * maxnb))
        span = min(nbc - 1, (maxnb - 1) * step)
        groups = (rows + 3) // 4
        base = torch.randint(0, max(1, nbc - span), (groups,), generator=g, device=device, dtype=torch.int64)
        bc = base[row_of // 4] + (pos // 4) * step
        col = bc * 4 + pos % 4
    else:
        raise ValueError(structure)
    vals = torch.randn(nnz, generator=g, device=device, dtype=torch.float32)
    del row_of, pos
    return DeviceMatrix.from_device_arrays("csr", dict(width=cols, height=rows, nnz=nnz),
                                           dict(csr_row_ptr=row_ptr.to(torch.int32), csr_col_id=col.to(torch.int32),
                                                csr_data=vals))
