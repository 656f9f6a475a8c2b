"""Host and device matrices in the reference's storage formats.

The converters are the library's own C++ (include/matrix_storage.h of this
repository), reached through the C ABI; their names follow the reference
(coo2csr, coo2dia, ... of include/matrix_storage.h in clSpMV), and they
return HostMatrix objects whose numpy arrays are views of the library-owned
buffers. DeviceMatrix copies a HostMatrix into device memory (torch tensors,
used purely as allocations) and runs the CUDA SpMV through the C ABI.
"""
from __future__ import annotations

import ctypes as C
from typing import Optional

import numpy as np

from . import _abi
from ._abi import FORMATS, check, lib

GPU_ALIGNMENT = 32       # include/constant.h:17 of the reference
SELL_GROUP_SIZE = 128    # include/constant.h:42
WARPSIZE = 32            # include/constant.h:21
BLOCK_SHAPES = [(bh, bw) for bw in (4, 8) for bh in (1, 2, 4, 8)]   # src/spmv_bell.cpp:362-363 order


class HostMatrix:
    """A format struct whose arrays live in host memory.

    `owner` is "lib" when the arrays were malloc'ed by the library (released
    with clspmv_free_<fmt>_f32), otherwise the numpy arrays are kept alive
    here."""

    def __init__(self, fmt: str, struct, keep=None, lib_owned: bool = False):
        self.fmt = fmt
        self.struct = struct
        self._keep = keep
        self._lib_owned = lib_owned

    def __del__(self):
        if getattr(self, "_lib_owned", False):
            try:
                getattr(lib(), f"clspmv_free_{self.fmt}_f32")(C.byref(self.struct))
            except Exception:
                pass
            self._lib_owned = False

    # -- views -------------------------------------------------------------
    def array(self, field: str) -> np.ndarray:
        for f, dt, n in FORMATS[self.fmt][1]:
            if f == field:
                count = int(n(self.struct))
                ptr = getattr(self.struct, field)
                if count <= 0 or not ptr:
                    return np.zeros(0, dtype=dt)
                ctype = C.c_int if dt == np.int32 else C.c_float
                return np.ctypeslib.as_array(C.cast(ptr, C.POINTER(ctype)), shape=(count,))
        raise KeyError(field)

    def arrays(self) -> dict:
        return {f: self.array(f) for f, _, _ in FORMATS[self.fmt][1]}

    def scalars(self) -> dict:
        out = {}
        for name, _ in self.struct._fields_:
            if name == "matinfo":
                mi = self.struct.matinfo
                out.update(width=mi.width, height=mi.height, nnz=mi.nnz)
            elif not any(name == f for f, _, _ in FORMATS[self.fmt][1]):
                out[name] = int(getattr(self.struct, name))
        return out

    @property
    def shape(self):
        return (self.struct.matinfo.height, self.struct.matinfo.width)

    @property
    def nnz(self) -> int:
        return self.struct.matinfo.nnz

    def stored_bytes(self) -> int:
        return int(sum(a.nbytes for a in self.arrays().values()))

    def copy(self) -> "HostMatrix":
        """Deep copy into numpy-owned arrays."""
        arrays = {k: np.array(v, copy=True) for k, v in self.arrays().items()}
        return from_arrays(self.fmt, self.scalars(), arrays)


def from_arrays(fmt: str, scalars: dict, arrays: dict) -> HostMatrix:
    """Builds a HostMatrix whose struct points at the given numpy arrays."""
    struct_t, spec = FORMATS[fmt]
    s = struct_t()
    keep = {}
    s.matinfo.width = int(scalars.get("width", 0))
    s.matinfo.height = int(scalars.get("height", 0))
    s.matinfo.nnz = int(scalars.get("nnz", 0))
    for name, _ in struct_t._fields_:
        if name in scalars and name not in ("width", "height", "nnz"):
            setattr(s, name, int(scalars[name]))
    for field, dt, _ in spec:
        a = np.ascontiguousarray(arrays[field], dtype=dt)
        if a.size == 0:
            a = np.zeros(4, dtype=dt)   # non-null pointer for empty arrays
        keep[field] = a
        setattr(s, field, a.ctypes.data)
    return HostMatrix(fmt, s, keep=keep)


def coo_matrix(height: int, width: int, row_id, col_id, data) -> HostMatrix:
    """COO matrix (coo_matrix<int,float>, include/matrix_storage.h:141-152)."""
    row_id = np.ascontiguousarray(row_id, dtype=np.int32)
    col_id = np.ascontiguousarray(col_id, dtype=np.int32)
    data = np.ascontiguousarray(data, dtype=np.float32)
    if not (row_id.shape == col_id.shape == data.shape):
        raise ValueError("row_id, col_id and data must have the same length")
    return from_arrays("coo", dict(width=width, height=height, nnz=row_id.size),
                       dict(coo_row_id=row_id, coo_col_id=col_id, coo_data=data))


# ---------------------------------------------------------------------------
# Converters (names as in the reference's matrix_storage.h)
# ---------------------------------------------------------------------------
def if_sorted_coo(coo: HostMatrix) -> bool:
    return bool(lib().clspmv_is_sorted_coo_f32(C.byref(coo.struct)))


def sort_coo(coo: HostMatrix) -> HostMatrix:
    check(lib().clspmv_sort_coo_f32(C.byref(coo.struct)), "sort_coo")
    return coo


def _convert(fmt: str, cname: str, coo: HostMatrix, *args) -> HostMatrix:
    out = FORMATS[fmt][0]()
    status = getattr(lib(), cname)(C.byref(coo.struct), C.byref(out), *args)
    m = HostMatrix(fmt, out, lib_owned=(status == _abi.OK))
    check(status, cname)
    return m


def coo2csr(coo):
    return _convert("csr", "clspmv_coo2csr_f32", coo)


def coo2dia(coo, alignment=GPU_ALIGNMENT):
    return _convert("dia", "clspmv_coo2dia_f32", coo, alignment)


def coo2bdia(coo, alignment=GPU_ALIGNMENT):
    return _convert("bdia", "clspmv_coo2bdia_f32", coo, alignment)


def coo2ell(coo, alignment=GPU_ALIGNMENT, ellnum=0):
    return _convert("ell", "clspmv_coo2ell_f32", coo, alignment, ellnum)


def coo2sell(coo, slice_height=WARPSIZE):
    return _convert("sell", "clspmv_coo2sell_f32", coo, slice_height)


def coo2bcsr(coo, bwidth, bheight, alignment=GPU_ALIGNMENT):
    return _convert("bcsr", "clspmv_coo2bcsr_f32", coo, bwidth, bheight, alignment)


def coo2b4csr(coo, bwidth, bheight, alignment=GPU_ALIGNMENT):
    return _convert("b4csr", "clspmv_coo2b4csr_f32", coo, bwidth, bheight, alignment)


def coo2bell(coo, bwidth, bheight, alignment=GPU_ALIGNMENT, ellnum=0):
    return _convert("bell", "clspmv_coo2bell_f32", coo, bwidth, bheight, alignment, ellnum)


def coo2b4ell(coo, bwidth, bheight, alignment=GPU_ALIGNMENT, ellnum=0):
    return _convert("b4ell", "clspmv_coo2b4ell_f32", coo, bwidth, bheight, alignment, ellnum)


def coo2sbell(coo, bwidth, bheight, slice_height=WARPSIZE):
    return _convert("sbell", "clspmv_coo2sbell_f32", coo, bwidth, bheight, slice_height)


def pad_csr(csr: HostMatrix, alignment: int) -> HostMatrix:
    out = FORMATS["csr"][0]()
    status = lib().clspmv_pad_csr_f32(C.byref(csr.struct), C.byref(out), alignment)
    m = HostMatrix("csr", out, lib_owned=(status == _abi.OK))
    check(status, "pad_csr")
    return m


def to_coo(m: HostMatrix) -> HostMatrix:
    """Inverse conversion <fmt>2coo (row-sorted output)."""
    out = FORMATS["coo"][0]()
    status = getattr(lib(), f"clspmv_{m.fmt}2coo_f32")(C.byref(m.struct), C.byref(out))
    res = HostMatrix("coo", out, lib_owned=(status == _abi.OK))
    check(status, f"{m.fmt}2coo")
    return res


# ---------------------------------------------------------------------------
# Device residency and SpMV
# ---------------------------------------------------------------------------
_SPMV = {
    "coo": "clspmv_coo_spmv_f32",
    "dia": "clspmv_dia_spmv_f32",
    "bdia": "clspmv_bdia_spmv_f32",
    "ell": "clspmv_ell_spmv_f32",
    "sell": "clspmv_sell_spmv_f32",
    "b4ell": "clspmv_b4ell_spmv_f32",
    "sbell": "clspmv_sbell_spmv_f32",
    "b4csr": "clspmv_b4csr_spmv_f32",
}
CSR_VARIANTS = ("merge", "vector", "scalar")


def _torch_dtype(dt):
    import torch
    return torch.float32 if dt == np.float32 else torch.int32


def _stream_handle(stream) -> Optional[int]:
    import torch
    if stream is None:
        stream = torch.cuda.current_stream()
    return stream.cuda_stream


class DeviceMatrix:
    """A format struct whose arrays are device copies (torch allocations)."""

    def __init__(self, host: HostMatrix, device="cuda"):
        import torch
        self.fmt = host.fmt
        self.struct = type(host.struct).from_buffer_copy(host.struct)
        self.tensors = {}
        for field, arr in host.arrays().items():
            if arr.size:
                t = torch.from_numpy(arr).to(device)   # host view -> one device copy
            else:
                t = torch.zeros(4, dtype=torch.float32 if arr.dtype == np.float32 else torch.int32, device=device)
            self.tensors[field] = t
            setattr(self.struct, field, t.data_ptr())
        self.shape = host.shape
        self.nnz = host.nnz
        self.stored_bytes = host.stored_bytes()
        self._plan = None

    @classmethod
    def from_device_arrays(cls, fmt: str, scalars: dict, tensors: dict) -> "DeviceMatrix":
        """A device matrix whose arrays were made on the device (e.g. by a
        device-side generator): `tensors` maps each array field of the
        format to a CUDA tensor of the right dtype."""
        self = cls.__new__(cls)
        struct_t, spec = FORMATS[fmt]
        self.fmt = fmt
        self.struct = struct_t()
        self.struct.matinfo.width = int(scalars["width"])
        self.struct.matinfo.height = int(scalars["height"])
        self.struct.matinfo.nnz = int(scalars["nnz"])
        for name, _ in struct_t._fields_:
            if name in scalars and name not in ("width", "height", "nnz"):
                setattr(self.struct, name, int(scalars[name]))
        self.tensors = {}
        for field, dt, _ in spec:
            t = tensors[field]
            if t.dtype != (_torch_dtype(dt)):
                raise TypeError(f"{field} must be {dt}")
            self.tensors[field] = t
            setattr(self.struct, field, t.data_ptr())
        self.shape = (self.struct.matinfo.height, self.struct.matinfo.width)
        self.nnz = self.struct.matinfo.nnz
        self.stored_bytes = int(sum(t.numel() * t.element_size() for t in self.tensors.values()))
        self._plan = None
        return self

    def sell_plan(self):
        """Row lengths and tail items of a SELL matrix for the padding-free
        SpMV (clspmv_sell_plan_create, made once)."""
        if getattr(self, "_sell_plan", None) is None:
            h = C.c_void_p()
            check(lib().clspmv_sell_plan_create(C.byref(self.struct), C.byref(h)), "sell_plan_create")
            self._sell_plan = h
        return self._sell_plan

    def sell_plan_entries(self) -> int:
        """Stored entries the padding-free SELL SpMV reads."""
        return int(lib().clspmv_sell_plan_entries(self.sell_plan()))

    def sell_plan_line_bytes(self) -> int:
        """Bytes the planned SpMV must read in 128-byte lines (clspmv_sell_plan_line_bytes)."""
        return int(lib().clspmv_sell_plan_line_bytes(self.sell_plan()))

    def sell_plan_sector_bytes(self) -> int:
        """col + data bytes of the 32-byte sectors holding real entries (what
        the padding-free SELL SpMV must move from the matrix arrays)."""
        return int(lib().clspmv_sell_plan_sector_bytes(self.sell_plan()))

    def __del__(self):
        p = getattr(self, "_sell_plan", None)
        if p:
            try:
                lib().clspmv_sell_plan_free(p)
            except Exception:
                pass
            self._sell_plan = None

    def merge_plan(self, stream=None):
        """Tile coordinates for the merge-path CSR kernel (computed once)."""
        import torch
        if self._plan is None:
            ntiles = lib().clspmv_csr_merge_tiles(self.shape[0], self.nnz)
            plan = torch.empty(2 * (ntiles + 1), dtype=torch.int32, device=self.tensors["csr_row_ptr"].device)
            check(lib().clspmv_csr_merge_plan(C.byref(self.struct), plan.data_ptr(), _stream_handle(stream)), "csr_merge_plan")
            self._plan = plan
        return self._plan

    def chunk_plan(self, stream=None):
        """First row of every 256-nonzero chunk for the chunked CSR kernel (computed once)."""
        import torch
        if getattr(self, "_chunk_plan", None) is None:
            n = lib().clspmv_csr_chunk_plan_size(self.nnz)
            plan = torch.empty(max(n, 1), dtype=torch.int32, device=self.tensors["csr_row_ptr"].device)
            check(lib().clspmv_csr_chunk_plan(C.byref(self.struct), plan.data_ptr(), _stream_handle(stream)), "csr_chunk_plan")
            self._chunk_plan = plan
        return self._chunk_plan

    def spmv(self, x, y, alpha: float = 1.0, beta: float = 1.0, stream=None, variant: str = "chunk",
             threads_per_row: int = 0, packed: "PackedValues | None" = None) -> None:
        """y <- alpha * A x + beta * y on the device (asynchronous on `stream`);
        with `packed`, from the 16-bit values of self.pack(). `variant`: CSR
        "chunk" (default; "merge" when col_id / data are not 16-byte aligned),
        "merge", "vector" or "scalar"; DIA / BDIA "bulk" stages the diagonals
        in shared memory by bulk copies; SELL "planned" reads only each
        row's real entries (its length plan), which on B200 is slower than the
        padded read for power-law slices: the tails of long rows are strided
        column-major reads."""
        L = lib()
        s = _stream_handle(stream)
        _computable(self.fmt)
        if packed is not None:
            if self.fmt == "csr" and variant == "chunk" and not ((self.struct.csr_col_id or 0) % 16
                                                                 or packed.values.data_ptr() % 8):
                check(L.clspmv_csr_chunk_spmv_packed(C.byref(self.struct), _abi.VALUE_TYPES[packed.value_type],
                                                     packed.values.data_ptr(), packed.row_scale.data_ptr(),
                                                     self.chunk_plan(stream).data_ptr(), x.data_ptr(), y.data_ptr(),
                                                     alpha, beta, s), "csr_chunk_spmv_packed")
                return
            if self.fmt == "sell" and variant == "planned":
                check(L.clspmv_sell_plan_spmv_packed(C.byref(self.struct), self.sell_plan(),
                                                     _abi.VALUE_TYPES[packed.value_type], packed.values.data_ptr(),
                                                     packed.row_scale.data_ptr(), x.data_ptr(), y.data_ptr(), alpha, beta,
                                                     s), "sell_plan_spmv_packed")
                return
            plan = self.merge_plan(stream).data_ptr() if self.fmt == "csr" else None
            check(L.clspmv_spmv_packed(_abi.FORMAT_IDS[self.fmt], C.byref(self.struct), _abi.VALUE_TYPES[packed.value_type],
                                       packed.values.data_ptr(), packed.row_scale.data_ptr(), plan, x.data_ptr(),
                                       y.data_ptr(), alpha, beta, s), "spmv_packed")
            return
        if self.fmt == "csr":
            if variant == "merge":
                plan = self.merge_plan(stream)
                check(L.clspmv_csr_merge_spmv_f32(C.byref(self.struct), plan.data_ptr(), x.data_ptr(), y.data_ptr(),
                                                  alpha, beta, s), "csr_merge_spmv")
            elif variant == "chunk":
                if (self.struct.csr_col_id or 0) % 16 or (self.struct.csr_data or 0) % 16:
                    return self.spmv(x, y, alpha, beta, stream, variant="merge")
                plan = self.chunk_plan(stream)
                check(L.clspmv_csr_chunk_spmv_f32(C.byref(self.struct), plan.data_ptr(), x.data_ptr(), y.data_ptr(),
                                                  alpha, beta, s), "csr_chunk_spmv")
            elif variant == "vector":
                check(L.clspmv_csr_vector_spmv_f32(C.byref(self.struct), x.data_ptr(), y.data_ptr(), alpha, beta,
                                                   threads_per_row, s), "csr_vector_spmv")
            elif variant == "scalar":
                check(L.clspmv_csr_scalar_spmv_f32(C.byref(self.struct), x.data_ptr(), y.data_ptr(), alpha, beta, s),
                      "csr_scalar_spmv")
            else:
                raise ValueError(variant)
            return
        if self.fmt == "sell" and variant == "planned":
            check(L.clspmv_sell_plan_spmv_f32(C.byref(self.struct), self.sell_plan(), x.data_ptr(), y.data_ptr(),
                                              alpha, beta, s), "sell_plan_spmv")
            return
        if self.fmt in ("dia", "bdia") and variant == "bulk":
            name = f"clspmv_{self.fmt}_bulk_spmv_f32"
            check(getattr(L, name)(C.byref(self.struct), x.data_ptr(), y.data_ptr(), alpha, beta, s), name)
            return
        name = _SPMV[self.fmt]
        check(getattr(L, name)(C.byref(self.struct), x.data_ptr(), y.data_ptr(), alpha, beta, s), name)

    def pack(self, value_type: str = "bf16", stream=None) -> "PackedValues":
        """16-bit values ("bf16" or "f16") with per-row scales, for spmm."""
        return device_pack(self, value_type, stream)

    def spmm(self, X, Y, alpha: float = 1.0, beta: float = 0.0, packed: "PackedValues | None" = None,
             stream=None) -> None:
        """Y <- alpha * A X + beta * Y for k = X.shape[1] right-hand sides.
        A CSR product with one contiguous column runs the single-vector
        chunked kernel (the fastest CSR kernel; the SpMM kernels split each
        row's k columns between lanes, which at k = 1 leaves lanes idle)."""
        if (self.fmt == "csr" and X.dim() == 2 and Y.dim() == 2 and X.shape[1] == 1 and Y.shape[1] == 1
                and X.is_contiguous() and Y.is_contiguous()):
            self.spmv(X.view(-1), Y.view(-1), alpha, beta, stream=stream, packed=packed)
            return
        device_spmm(self, X, Y, alpha, beta, packed, stream)


def _computable(fmt: str) -> None:
    """The generic BCSR / BELL (any block shape) are storage formats: only
    the reference's serial bcsr_spmv / bell_spmv read them, and no GPU kernel
    does (the device kernels take b4csr / b4ell / SBELL)."""
    if fmt in ("bcsr", "bell"):
        raise ValueError(f"no GPU kernel reads the generic {fmt}; convert to b4{fmt[1:]} for SpMV")


class _DeviceArrays:
    """Arrays a device converter cudaMalloc'ed, released with
    clspmv_device_free_<fmt>_f32 when the last tensor viewing them is gone."""

    def __init__(self, fmt: str, struct):
        self.fmt = fmt
        self.struct = struct

    def __del__(self):
        try:
            getattr(lib(), f"clspmv_device_free_{self.fmt}_f32")(C.byref(self.struct))
        except Exception:
            pass


class _CudaView:
    """__cuda_array_interface__ of one converter-owned array; keeps the owner alive."""

    def __init__(self, owner: _DeviceArrays, ptr: int, count: int, dt):
        self._owner = owner
        self.__cuda_array_interface__ = {"shape": (count,), "typestr": "<i4" if dt == np.int32 else "<f4",
                                         "data": (ptr, False), "version": 3, "strides": None}


# format -> (C entry point, default trailing arguments after the required ones)
_DEVICE_CONVERT = {
    "csr": ("clspmv_device_coo2csr_f32", 0, ()),
    "dia": ("clspmv_device_coo2dia_f32", 0, (GPU_ALIGNMENT,)),
    "bdia": ("clspmv_device_coo2bdia_f32", 0, (GPU_ALIGNMENT,)),
    "ell": ("clspmv_device_coo2ell_f32", 0, (GPU_ALIGNMENT, 0)),
    "sell": ("clspmv_device_coo2sell_f32", 0, (WARPSIZE,)),
    "bcsr": ("clspmv_device_coo2bcsr_f32", 2, (GPU_ALIGNMENT,)),
    "bell": ("clspmv_device_coo2bell_f32", 2, (GPU_ALIGNMENT, 0)),
    "b4csr": ("clspmv_device_coo2b4csr_f32", 2, (GPU_ALIGNMENT,)),
    "b4ell": ("clspmv_device_coo2b4ell_f32", 2, (GPU_ALIGNMENT, 0)),
    "sbell": ("clspmv_device_coo2sbell_f32", 2, (WARPSIZE,)),
}


def device_convert_raw(coo: DeviceMatrix, fmt: str, *args, stream=None):
    """(status, struct) of clspmv_device_coo2<fmt>_f32 on a device COO; the
    arguments after the format are those of the host coo2<fmt> (bwidth,
    bheight first for the block formats; the rest default as there)."""
    if coo.fmt != "coo":
        raise ValueError("device conversion starts from a device COO")
    name, required, defaults = _DEVICE_CONVERT[fmt]
    if len(args) < required:
        raise TypeError(f"device coo2{fmt} needs {required} leading arguments")
    full = tuple(args) + defaults[len(args) - required:]
    out = FORMATS[fmt][0]()
    status = getattr(lib(), name)(C.byref(coo.struct), C.byref(out), *full, _stream_handle(stream))
    return status, out


def device_convert(coo: DeviceMatrix, fmt: str, *args, stream=None) -> DeviceMatrix:
    """coo2<fmt> on the device: a DeviceMatrix equal array for array to
    DeviceMatrix(coo2<fmt>(host COO, *args)), converted where the COO already
    is (clspmv_device_coo2<fmt>_f32). Raises ClspmvError with the host
    converter's status where it would refuse or reject the input."""
    import torch
    status, out = device_convert_raw(coo, fmt, *args, stream=stream)
    check(status, f"device_coo2{fmt}")
    owner = _DeviceArrays(fmt, out)
    dev = coo.tensors["coo_row_id"].device
    self = DeviceMatrix.__new__(DeviceMatrix)
    self.fmt, self.struct, self.tensors, self._plan = fmt, out, {}, None
    total = None   # slots of a sliced format: its last slice pointer, read from the device
    for field, dt, n in FORMATS[fmt][1]:
        if field.endswith("_slice_ptr"):
            ns = out.sell_slice_num if fmt == "sell" else out.sbell_slice_num
            count = ns + 1
        elif fmt in ("sell", "sbell") and field.endswith("_col_id"):
            count = total
        elif fmt == "sell" and field == "sell_data":
            count = total
        elif fmt == "sbell" and field == "sbell_data":
            count = total * out.sbell_bwidth * out.sbell_bheight
        elif field == "bdia_data":
            ndiag = int(self.tensors["bdia_bptr"][-1].item()) if out.bdia_band_num > 0 else 0
            count = ndiag * out.bdia_length_aligned
        else:
            count = int(n(out))
        if count > 0:
            t = torch.as_tensor(_CudaView(owner, getattr(out, field), count, dt), device=dev)
        else:
            t = torch.empty(0, dtype=_torch_dtype(dt), device=dev)
        if field.endswith("_slice_ptr"):
            total = int(t[-1].item())
        self.tensors[field] = t
    self.shape = (out.matinfo.height, out.matinfo.width)
    self.nnz = out.matinfo.nnz
    self.stored_bytes = int(sum(t.numel() * t.element_size() for t in self.tensors.values()))
    self._owner = owner
    return self


def device_sort_coo(coo: DeviceMatrix, stream=None) -> DeviceMatrix:
    """Stable in-place sort of a device COO by (row, col) (clspmv_device_sort_coo_f32)."""
    check(lib().clspmv_device_sort_coo_f32(C.byref(coo.struct), _stream_handle(stream)), "device_sort_coo")
    return coo


class PackedValues:
    """16-bit copy of a device matrix's values with per-row power-of-two
    scales (clspmv_pack_values); indices stay those of the FP32 matrix."""

    def __init__(self, values, row_scale, value_type: str):
        self.values = values
        self.row_scale = row_scale
        self.value_type = value_type

    @property
    def nbytes(self) -> int:
        return self.values.numel() * 2 + self.row_scale.numel() * 4


def _spmm_dev(m: "DeviceMatrix"):
    if m.fmt not in _abi.FORMAT_IDS:
        raise ValueError(f"no SpMM for format {m.fmt}")
    return _abi.FORMAT_IDS[m.fmt]


def device_pack(m: "DeviceMatrix", value_type: str = "bf16", stream=None) -> PackedValues:
    import torch
    fid = _spmm_dev(m)
    n = C.c_size_t()
    check(lib().clspmv_stored_values(fid, C.byref(m.struct), C.byref(n)), "stored_values")
    dev = next(iter(m.tensors.values())).device
    vals = torch.zeros(max(int(n.value), 1), dtype=torch.int16, device=dev)
    scale = torch.ones(max(m.shape[0], 1), dtype=torch.float32, device=dev)
    check(lib().clspmv_pack_values(fid, C.byref(m.struct), _abi.VALUE_TYPES[value_type], vals.data_ptr(),
                                   scale.data_ptr(), _stream_handle(stream)), "pack_values")
    return PackedValues(vals, scale, value_type)


def device_spmm(m: "DeviceMatrix", X, Y, alpha: float = 1.0, beta: float = 0.0, packed: PackedValues | None = None,
                stream=None) -> None:
    """Y <- alpha * A X + beta * Y; X (width, k) and Y (height, k) float32
    CUDA tensors with unit column stride."""
    fid = _spmm_dev(m)
    if X.dim() != 2 or Y.dim() != 2 or X.stride(1) != 1 or Y.stride(1) != 1:
        raise ValueError("X and Y must be 2-D with unit column stride")
    k = X.shape[1]
    if Y.shape[1] != k or X.shape[0] < m.shape[1] or Y.shape[0] < m.shape[0]:
        raise ValueError("shape mismatch")
    vt = 0 if packed is None else _abi.VALUE_TYPES[packed.value_type]
    check(lib().clspmv_spmm(fid, C.byref(m.struct), vt, None if packed is None else packed.values.data_ptr(),
                            None if packed is None else packed.row_scale.data_ptr(), k, X.data_ptr(), X.stride(0),
                            Y.data_ptr(), Y.stride(0), alpha, beta, _stream_handle(stream)), "spmm")


def device_spmm_tc(m: "DeviceMatrix", X, Y, alpha: float = 1.0, beta: float = 0.0, stream=None) -> None:
    """Y <- alpha * A X + beta * Y for a b4csr matrix of 4 x 4 blocks on the
    tensor cores (tcgen05, TF32 head and remainder of every value, FP32
    accumulation); k = X.shape[1] a multiple of 16 up to 128."""
    if m.fmt != "b4csr":
        raise ValueError("the tensor-core product takes b4csr matrices")
    if X.dim() != 2 or Y.dim() != 2 or X.stride(1) != 1 or Y.stride(1) != 1:
        raise ValueError("X and Y must be 2-D with unit column stride")
    k = X.shape[1]
    if Y.shape[1] != k or X.shape[0] < m.shape[1] or Y.shape[0] < m.shape[0]:
        raise ValueError("shape mismatch")
    check(lib().clspmv_b4csr_spmm_tc_f32(C.byref(m.struct), k, X.data_ptr(), X.stride(0), Y.data_ptr(), Y.stride(0),
                                         alpha, beta, _stream_handle(stream)), "spmm_tc")


def pipeline_timeouts() -> int:
    """Bounded waits of the bulk-copy pipeline kernels that ran out since the last call (synchronous; resets)."""
    n = C.c_uint(0)
    check(lib().clspmv_pipeline_timeouts(C.byref(n)), "pipeline_timeouts")
    return int(n.value)


def tensor_timeouts() -> int:
    """Bounded waits of the tensor-core kernels that ran out since the last call (synchronous; resets)."""
    n = C.c_uint(0)
    check(lib().clspmv_tensor_timeouts(C.byref(n)), "tensor_timeouts")
    return int(n.value)


def launch_count() -> int:
    return int(lib().clspmv_launch_count())
