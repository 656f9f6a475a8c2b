"""Row-sharded CSR SpMV and the A^k x loop across the ranks of a process group.

The reference iterates y <- A x + y, x <- y on one device (src/eval.cpp:19-72,
with cpy_vector_from_gpu of src/spmv_cocktail.cpp:1510-1556 between steps).
Here each rank (one per GPU) holds a block of consecutive rows of A, split so
that every rank gets about the same number of nonzeros, with all columns.
One step is the local SpMV into the rank's rows of y, then one all-gather of
every rank's y block into every rank's x (NCCL over NVLink / NVSwitch; gloo
on the CPU). The column ids of each rank's slab are renumbered once into the
all-gather's padded layout (rank q's rows sit at x[q * block : q * block +
rows_q], block = the largest slab), so the collective writes x in place and
no step copies or reorders x. Rows of a slab run through the library's CSR
kernel (nonzero chunks), so y is the same as one device's y row for row.
"""
from __future__ import annotations

from typing import Callable, Optional

import numpy as np

from . import formats as F


def split_rows(row_ptr: np.ndarray, world: int) -> list:
    """Contiguous row ranges [r0, r1), one per rank, with about nnz / world
    nonzeros each (boundaries at the row where the running count passes
    q * nnz / world)."""
    row_ptr = np.asarray(row_ptr, dtype=np.int64)
    m, nnz = row_ptr.size - 1, int(row_ptr[-1])
    cuts = [0]
    for q in range(1, world):
        target = nnz * q / world
        r = int(np.searchsorted(row_ptr, target, side="left"))
        cuts.append(min(max(r, cuts[-1]), m))
    cuts.append(m)
    return [(cuts[q], cuts[q + 1]) for q in range(world)]


def padded_columns(col: np.ndarray, bounds: list, block: int) -> np.ndarray:
    """Column ids in the all-gather layout: column c owned by rank q (rows
    bounds[q]) becomes q * block + (c - bounds[q][0])."""
    starts = np.array([b[0] for b in bounds], dtype=np.int64)
    col = np.asarray(col, dtype=np.int64)
    q = np.searchsorted(starts, col, side="right") - 1
    # empty ranks share their start with the next one; searchsorted picks the last
    return (q * block + (col - starts[q])).astype(np.int32)


def slab(csr: F.HostMatrix, bounds: list, rank: int) -> F.HostMatrix:
    """Rows bounds[rank] of a square CSR matrix, columns renumbered into the
    padded layout (width = world * block)."""
    a = csr.arrays()
    rp, col, val = a["csr_row_ptr"], a["csr_col_id"], a["csr_data"]
    r0, r1 = bounds[rank]
    block = max(1, max(b1 - b0 for b0, b1 in bounds))
    lo, hi = int(rp[r0]), int(rp[r1])
    return F.from_arrays("csr", dict(width=len(bounds) * block, height=r1 - r0, nnz=hi - lo),
                         dict(csr_row_ptr=(rp[r0:r1 + 1] - lo).astype(np.int32),
                              csr_col_id=padded_columns(col[lo:hi], bounds, block),
                              csr_data=np.array(val[lo:hi], dtype=np.float32)))


def split_rows_even(m: int, world: int) -> list:
    """Contiguous row ranges with m / world rows each (for matrices whose
    rows hold about the same number of nonzeros, such as stencils, where no
    rank needs the whole row-pointer array to balance the split)."""
    cuts = [m * q // world for q in range(world + 1)]
    return [(cuts[q], cuts[q + 1]) for q in range(world)]


def slab_from_rows(row_ptr, col, val, bounds: list, rank: int) -> F.HostMatrix:
    """This rank's slab in the padded layout from its own rows only:
    row_ptr (rebased to 0) / col (global ids) / val of rows bounds[rank]."""
    r0, r1 = bounds[rank]
    block = max(1, max(b1 - b0 for b0, b1 in bounds))
    row_ptr = np.asarray(row_ptr, dtype=np.int64)
    if row_ptr.size != r1 - r0 + 1 or row_ptr[0] != 0:
        raise ValueError("row_ptr must hold the rank's rows, starting at 0")
    nnz = int(row_ptr[-1])
    return F.from_arrays("csr", dict(width=len(bounds) * block, height=r1 - r0, nnz=nnz),
                         dict(csr_row_ptr=row_ptr.astype(np.int32),
                              csr_col_id=padded_columns(np.asarray(col)[:nnz], bounds, block),
                              csr_data=np.asarray(val, dtype=np.float32)[:nnz]))


class ShardedCsr:
    """This rank's slab of a square CSR matrix and the buffers of the loop.

    `x` is the padded all-gather buffer (world * block floats), `y` this
    rank's rows padded to `block`. `local_spmv(x, y_rows, alpha, beta)`
    replaces the device SpMV (the CPU tests pass the oracle); by default the
    slab is uploaded and run by DeviceMatrix.spmv."""

    def __init__(self, csr: Optional[F.HostMatrix], group=None, device="cuda",
                 local_spmv: Optional[Callable] = None, *, n: Optional[int] = None,
                 make_rows: Optional[Callable] = None):
        """From the whole host matrix `csr` (every rank holds it; rows split
        by nonzeros), or, with `n` and `make_rows(r0, r1) -> (row_ptr, col,
        val)` (the rows [r0, r1) with row_ptr rebased to 0 and global column
        ids), from this rank's rows alone (rows split evenly): no rank then
        holds more of A than its slab."""
        import torch
        import torch.distributed as dist
        self.group = group
        self.world = dist.get_world_size(group) if dist.is_initialized() else 1
        self.rank = dist.get_rank(group) if dist.is_initialized() else 0
        if csr is not None:
            h, w = csr.shape
            if h != w:
                raise ValueError("x <- y needs a square matrix")
            self.bounds = split_rows(csr.array("csr_row_ptr"), self.world)
        else:
            if n is None or make_rows is None:
                raise ValueError("give the matrix, or its size and a row generator")
            self.bounds = split_rows_even(int(n), self.world)
        self.block = max(1, max(b1 - b0 for b0, b1 in self.bounds))
        self.rows = self.bounds[self.rank][1] - self.bounds[self.rank][0]
        if csr is not None:
            self.host = slab(csr, self.bounds, self.rank)
        else:
            r0, r1 = self.bounds[self.rank]
            self.host = slab_from_rows(*make_rows(r0, r1), self.bounds, self.rank)
        self.nnz = self.host.nnz
        self.device = torch.device(device)
        self.x = torch.zeros(self.world * self.block, dtype=torch.float32, device=self.device)
        self.y = torch.zeros(self.block, dtype=torch.float32, device=self.device)
        if local_spmv is None:
            dev = F.DeviceMatrix(self.host, device=self.device)
            self._dev = dev
            local_spmv = lambda x, y, alpha, beta: dev.spmv(x, y, alpha, beta)
        self.local_spmv = local_spmv
        self._into_tensor = True

    # -- layout --------------------------------------------------------------
    def scatter_global(self, v: np.ndarray, out) -> None:
        """Writes a global length-n vector into the padded layout `out`."""
        import torch
        v = np.asarray(v, dtype=np.float32)
        pad = np.zeros(self.world * self.block, np.float32)
        for q, (r0, r1) in enumerate(self.bounds):
            pad[q * self.block:q * self.block + (r1 - r0)] = v[r0:r1]
        out.copy_(torch.from_numpy(pad))

    def global_x(self) -> np.ndarray:
        """x in row order (host copy)."""
        pad = self.x.cpu().numpy()
        return np.concatenate([pad[q * self.block:q * self.block + (r1 - r0)]
                               for q, (r0, r1) in enumerate(self.bounds)])

    def load(self, x: np.ndarray, y: np.ndarray) -> None:
        """Global x and y (every rank passes the same vectors)."""
        import torch
        self.scatter_global(x, self.x)
        r0, r1 = self.bounds[self.rank]
        yy = np.zeros(self.block, np.float32)
        yy[:r1 - r0] = np.asarray(y, dtype=np.float32)[r0:r1]
        self.y.copy_(torch.from_numpy(yy))

    # -- the loop ------------------------------------------------------------
    def _all_gather(self) -> None:
        import torch.distributed as dist
        if self.world == 1:
            self.x.copy_(self.y)
            return
        if self._into_tensor:
            try:
                dist.all_gather_into_tensor(self.x, self.y, group=self.group)
                return
            except (RuntimeError, AttributeError, NotImplementedError):
                self._into_tensor = False   # a backend without it (older gloo): views of x
        dist.all_gather(list(self.x.view(self.world, self.block)), self.y, group=self.group)

    def step(self, alpha: float = 1.0, beta: float = 1.0) -> None:
        """y_rows <- alpha * A_rows x + beta * y_rows, then x <- y (all ranks)."""
        if self.rows > 0:
            self.local_spmv(self.x, self.y[:self.rows], alpha, beta)
        self._all_gather()

    def iterate(self, k: int, alpha: float = 1.0, beta: float = 1.0) -> None:
        for _ in range(int(k)):
            self.step(alpha, beta)
