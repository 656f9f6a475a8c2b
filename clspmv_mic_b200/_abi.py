"""ctypes view of the C ABI in include/clspmv_b200.h.

The structs mirror the reference's matrix_storage.h templates instantiated
with int/float (include/matrix_storage.h:15-365 of clSpMV). Pointer members
are declared as c_void_p so that one struct type carries host or device
addresses.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

import numpy as np

PKG_DIR = Path(__file__).resolve().parent
LIB_PATH = PKG_DIR / "libclspmv_b200.so"

VP = C.c_void_p
I32 = C.c_int
U32 = C.c_uint


class MatInfo(C.Structure):
    _fields_ = [("width", I32), ("height", I32), ("nnz", I32)]


class Coo(C.Structure):
    _fields_ = [("matinfo", MatInfo), ("coo_row_id", VP), ("coo_col_id", VP), ("coo_data", VP)]


class Csr(C.Structure):
    _fields_ = [("matinfo", MatInfo), ("csr_row_ptr", VP), ("csr_col_id", VP), ("csr_data", VP)]


class Dia(C.Structure):
    _fields_ = [("matinfo", MatInfo), ("dia_num", I32), ("dia_length", I32), ("dia_length_aligned", I32),
                ("dia_offsets", VP), ("dia_data", VP)]


class Bdia(C.Structure):
    _fields_ = [("matinfo", MatInfo), ("bdia_band_num", I32), ("bdia_length", I32), ("bdia_length_aligned", I32),
                ("bdia_offsets", VP), ("bdia_bptr", VP), ("bdia_data", VP)]


class Ell(C.Structure):
    _fields_ = [("matinfo", MatInfo), ("ell_num", I32), ("ell_height_aligned", I32),
                ("ell_col_id", VP), ("ell_data", VP)]


class Sell(C.Structure):
    _fields_ = [("matinfo", MatInfo), ("sell_slice_height", U32), ("sell_slice_num", I32),
                ("sell_slice_ptr", VP), ("sell_col_id", VP), ("sell_data", VP)]


class Bcsr(C.Structure):
    _fields_ = [("matinfo", MatInfo), ("bcsr_bwidth", U32), ("bcsr_bheight", U32), ("bcsr_row_num", I32),
                ("bcsr_aligned_size", I32), ("bcsr_block_num", I32),
                ("bcsr_row_ptr", VP), ("bcsr_col_id", VP), ("bcsr_data", VP)]


class Bell(C.Structure):
    _fields_ = [("matinfo", MatInfo), ("bell_bwidth", U32), ("bell_bheight", U32), ("bell_row_num", I32),
                ("bell_block_num", I32), ("bell_height_aligned", I32), ("bell_float4_aligned", I32),
                ("bell_col_id", VP), ("bell_data", VP)]


class B4csr(C.Structure):
    _fields_ = [("matinfo", MatInfo), ("b4csr_bwidth", U32), ("b4csr_bheight", U32), ("b4csr_row_num", I32),
                ("b4csr_aligned_size", I32), ("b4csr_block_num", I32),
                ("b4csr_row_ptr", VP), ("b4csr_col_id", VP), ("b4csr_data", VP)]


class B4ell(C.Structure):
    _fields_ = [("matinfo", MatInfo), ("b4ell_bwidth", U32), ("b4ell_bheight", U32), ("b4ell_row_num", I32),
                ("b4ell_block_num", I32), ("b4ell_height_aligned", I32), ("b4ell_float4_aligned", I32),
                ("b4ell_col_id", VP), ("b4ell_data", VP)]


class Sbell(C.Structure):
    _fields_ = [("matinfo", MatInfo), ("sbell_bwidth", U32), ("sbell_bheight", U32), ("sbell_slice_height", U32),
                ("sbell_slice_num", I32), ("sbell_row_num", I32),
                ("sbell_slice_ptr", VP), ("sbell_col_id", VP), ("sbell_data", VP)]


COCKTAIL_PARTS = [("bdia", "bdia"), ("dia", "dia"), ("sbell", "sbell"), ("bell", "b4ell"), ("bcsr", "b4csr"),
                  ("sell", "sell"), ("ell", "ell"), ("csr", "csr"), ("coo", "coo")]


class Cocktail(C.Structure):
    """cocktail<int,int,float> (include/analyze.h:105-144 of clSpMV)."""
    _fields_ = ([(f"ifuse{n}", C.c_bool) for n in ("bdia", "dia", "sbell", "bell", "bcsr", "sell", "ell", "csr", "coo")] +
                [(f"{n}_meth_num", I32) for n in ("bdia", "dia", "sbell", "bell", "bcsr", "sell", "ell", "csr", "coo")] +
                [("csr_group_num", I32), ("coo_group_num", I32), ("mat_width", I32), ("mat_height", I32), ("mat_nnz", I32),
                 ("bdia", Bdia), ("dia", Dia), ("sbell", Sbell), ("bell", B4ell), ("bcsr", B4csr), ("sell", Sell),
                 ("ell", Ell), ("csr", Csr), ("coo", Coo)])


FORMAT_IDS = {"csr": 0, "coo": 1, "dia": 2, "bdia": 3, "ell": 4, "sell": 5, "b4csr": 6, "b4ell": 7, "sbell": 8}
VALUE_TYPES = {"f32": 0, "bf16": 1, "f16": 2}
BENCH_MAX_VARIANTS = 16
METHODS = {"bandwidth": 0, "csr_scalar": 1, "csr_vector": 2, "bdia": 3, "dia": 4, "ell": 5, "coo": 6, "bell": 7,
           "bcsr": 8, "sell": 9, "sbell": 10, "csr_merge": 11}


class BenchVariant(C.Structure):
    """clspmv_bench_variant: one timed variant of a benchmark driver."""
    _fields_ = [("status", I32), ("param0", I32), ("param1", I32), ("ms", C.c_double), ("gflops", C.c_double),
                ("distance", C.c_double), ("max_diff", C.c_double), ("max_diff_ratio", C.c_double)]


class BenchResult(C.Structure):
    """clspmv_bench_result: every variant a driver ran and the fastest."""
    _fields_ = [("method", I32), ("nvariants", I32), ("best", I32), ("best_ms", C.c_double),
                ("best_gflops", C.c_double), ("v", BenchVariant * BENCH_MAX_VARIANTS)]


class SpmmJob(C.Structure):
    """clspmv_spmm_job: one Y <- alpha*A*X + beta*Y of a batch."""
    _fields_ = [("format", I32), ("dev", VP), ("value_type", I32), ("values", VP), ("row_scale", VP), ("k", I32),
                ("X", VP), ("ldx", I32), ("Y", VP), ("ldy", I32), ("alpha", C.c_float), ("beta", C.c_float)]


def _n_bdia_data(s):
    if s.bdia_band_num <= 0:
        return 0
    bptr = np.ctypeslib.as_array(C.cast(s.bdia_bptr, C.POINTER(C.c_int)), shape=(s.bdia_band_num + 1,))
    return int(bptr[-1]) * s.bdia_length_aligned


def _ptr_last(ptr, n):
    if not ptr or n < 0:
        return 0
    return int(np.ctypeslib.as_array(C.cast(ptr, C.POINTER(C.c_int)), shape=(n + 1,))[-1])


# name -> (struct, [(field, numpy dtype, length(struct) on the host)])
FORMATS = {
    "coo": (Coo, [("coo_row_id", np.int32, lambda s: s.matinfo.nnz),
                  ("coo_col_id", np.int32, lambda s: s.matinfo.nnz),
                  ("coo_data", np.float32, lambda s: s.matinfo.nnz)]),
    "csr": (Csr, [("csr_row_ptr", np.int32, lambda s: s.matinfo.height + 1),
                  ("csr_col_id", np.int32, lambda s: s.matinfo.nnz),
                  ("csr_data", np.float32, lambda s: s.matinfo.nnz)]),
    "dia": (Dia, [("dia_offsets", np.int32, lambda s: s.dia_num),
                  ("dia_data", np.float32, lambda s: s.dia_num * s.dia_length_aligned)]),
    "bdia": (Bdia, [("bdia_offsets", np.int32, lambda s: s.bdia_band_num),
                    ("bdia_bptr", np.int32, lambda s: s.bdia_band_num + 1 if s.bdia_band_num > 0 else 0),
                    ("bdia_data", np.float32, _n_bdia_data)]),
    "ell": (Ell, [("ell_col_id", np.int32, lambda s: s.ell_num * s.ell_height_aligned),
                  ("ell_data", np.float32, lambda s: s.ell_num * s.ell_height_aligned)]),
    "sell": (Sell, [("sell_slice_ptr", np.int32, lambda s: s.sell_slice_num + 1),
                    ("sell_col_id", np.int32, lambda s: _ptr_last(s.sell_slice_ptr, s.sell_slice_num)),
                    ("sell_data", np.float32, lambda s: _ptr_last(s.sell_slice_ptr, s.sell_slice_num))]),
    "bcsr": (Bcsr, [("bcsr_row_ptr", np.int32, lambda s: s.bcsr_row_num + 1),
                    ("bcsr_col_id", np.int32, lambda s: s.bcsr_block_num),
                    ("bcsr_data", np.float32, lambda s: s.bcsr_aligned_size * s.bcsr_bwidth * s.bcsr_bheight)]),
    "bell": (Bell, [("bell_col_id", np.int32, lambda s: s.bell_height_aligned * s.bell_block_num),
                    ("bell_data", np.float32,
                     lambda s: s.bell_height_aligned * s.bell_block_num * s.bell_bwidth * s.bell_bheight)]),
    "b4csr": (B4csr, [("b4csr_row_ptr", np.int32, lambda s: s.b4csr_row_num + 1),
                      ("b4csr_col_id", np.int32, lambda s: s.b4csr_block_num),
                      ("b4csr_data", np.float32,
                       lambda s: s.b4csr_aligned_size * s.b4csr_bheight * (s.b4csr_bwidth // 4))]),
    "b4ell": (B4ell, [("b4ell_col_id", np.int32, lambda s: s.b4ell_height_aligned * s.b4ell_block_num),
                      ("b4ell_data", np.float32,
                       lambda s: s.b4ell_float4_aligned * s.b4ell_bheight * (s.b4ell_bwidth // 4) * s.b4ell_block_num)]),
    "sbell": (Sbell, [("sbell_slice_ptr", np.int32, lambda s: s.sbell_slice_num + 1),
                      ("sbell_col_id", np.int32, lambda s: _ptr_last(s.sbell_slice_ptr, s.sbell_slice_num)),
                      ("sbell_data", np.float32,
                       lambda s: _ptr_last(s.sbell_slice_ptr, s.sbell_slice_num) * s.sbell_bwidth * s.sbell_bheight)]),
}

STATUS = {0: "ok", 1: "invalid argument", 2: "allocation failed", 3: "unsupported shape", 4: "CUDA error",
          5: "refused by the format's size rule", 6: "misaligned pointer or length",
          7: "COO input is not sorted by (row, col)", 8: "bounded device wait timed out"}
OK, ERR_ARG, ERR_ALLOC, ERR_UNSUPPORTED, ERR_CUDA, ERR_REFUSED, ERR_ALIGN, ERR_NOT_SORTED, ERR_TIMEOUT = range(9)


class ClspmvError(RuntimeError):
    def __init__(self, status: int, where: str, detail: str = ""):
        self.status = status
        msg = f"{where}: {STATUS.get(status, 'status %d' % status)}"
        if detail:
            msg += f" ({detail})"
        super().__init__(msg)


_lib = None


def _declare(lib):
    P = C.POINTER
    S = {name: P(spec[0]) for name, spec in FORMATS.items()}
    f32 = C.c_float
    sigs = {
        "clspmv_version": (C.c_char_p, []),
        "clspmv_status_string": (C.c_char_p, [I32]),
        "clspmv_last_cuda_error": (C.c_char_p, []),
        "clspmv_launch_count": (C.c_longlong, []),
        "clspmv_sort_coo_f32": (I32, [S["coo"]]),
        "clspmv_is_sorted_coo_f32": (I32, [S["coo"]]),
        "clspmv_coo2csr_f32": (I32, [S["coo"], S["csr"]]),
        "clspmv_pad_csr_f32": (I32, [S["csr"], S["csr"], I32]),
        "clspmv_coo2dia_f32": (I32, [S["coo"], S["dia"], I32]),
        "clspmv_coo2bdia_f32": (I32, [S["coo"], S["bdia"], I32]),
        "clspmv_coo2ell_f32": (I32, [S["coo"], S["ell"], I32, I32]),
        "clspmv_coo2sell_f32": (I32, [S["coo"], S["sell"], U32]),
        "clspmv_coo2bcsr_f32": (I32, [S["coo"], S["bcsr"], U32, U32, I32]),
        "clspmv_coo2b4csr_f32": (I32, [S["coo"], S["b4csr"], U32, U32, I32]),
        "clspmv_coo2bell_f32": (I32, [S["coo"], S["bell"], U32, U32, I32, I32]),
        "clspmv_coo2b4ell_f32": (I32, [S["coo"], S["b4ell"], U32, U32, I32, I32]),
        "clspmv_coo2sbell_f32": (I32, [S["coo"], S["sbell"], U32, U32, U32]),
        "clspmv_csr_scalar_spmv_f32": (I32, [S["csr"], VP, VP, f32, f32, VP]),
        "clspmv_csr_vector_spmv_f32": (I32, [S["csr"], VP, VP, f32, f32, I32, VP]),
        "clspmv_csr_merge_tiles": (I32, [I32, I32]),
        "clspmv_csr_merge_plan": (I32, [S["csr"], VP, VP]),
        "clspmv_csr_merge_spmv_f32": (I32, [S["csr"], VP, VP, VP, f32, f32, VP]),
        "clspmv_csr_chunk_plan_size": (I32, [I32]),
        "clspmv_csr_chunk_plan": (I32, [S["csr"], VP, VP]),
        "clspmv_csr_chunk_spmv_f32": (I32, [S["csr"], VP, VP, VP, f32, f32, VP]),
        "clspmv_csr_chunk_spmv_packed": (I32, [S["csr"], I32, VP, VP, VP, VP, VP, f32, f32, VP]),
        "clspmv_coo_spmv_f32": (I32, [S["coo"], VP, VP, f32, f32, VP]),
        "clspmv_dia_spmv_f32": (I32, [S["dia"], VP, VP, f32, f32, VP]),
        "clspmv_bdia_spmv_f32": (I32, [S["bdia"], VP, VP, f32, f32, VP]),
        "clspmv_dia_bulk_spmv_f32": (I32, [S["dia"], VP, VP, f32, f32, VP]),
        "clspmv_bdia_bulk_spmv_f32": (I32, [S["bdia"], VP, VP, f32, f32, VP]),
        "clspmv_pipeline_timeouts": (I32, [C.POINTER(C.c_uint)]),
        "clspmv_ell_spmv_f32": (I32, [S["ell"], VP, VP, f32, f32, VP]),
        "clspmv_sell_spmv_f32": (I32, [S["sell"], VP, VP, f32, f32, VP]),
        "clspmv_b4ell_spmv_f32": (I32, [S["b4ell"], VP, VP, f32, f32, VP]),
        "clspmv_sbell_spmv_f32": (I32, [S["sbell"], VP, VP, f32, f32, VP]),
        "clspmv_b4csr_spmv_f32": (I32, [S["b4csr"], VP, VP, f32, f32, VP]),
        "clspmv_analyze_matrix_f32": (I32, [S["coo"], P(Cocktail), C.c_char_p, f32, I32, I32]),
        "clspmv_free_cocktail_f32": (None, [P(Cocktail)]),
        "clspmv_cocktail_upload_f32": (I32, [P(Cocktail), P(VP)]),
        "clspmv_cocktail_spmv_f32": (I32, [VP, VP, VP, f32, f32, VP]),
        "clspmv_cocktail_device_view": (I32, [VP, P(Cocktail)]),
        "clspmv_cocktail_iterate_f32": (I32, [VP, VP, VP, f32, f32, I32, VP]),
        "clspmv_cocktail_set_schedule": (I32, [VP, I32]),
        "clspmv_cocktail_fused_items": (I32, [VP]),
        "clspmv_cocktail_sell_planned": (I32, [VP]),
        "clspmv_cocktail_set_csr_lanes": (I32, [VP, I32]),
        "clspmv_cocktail_free": (I32, [VP]),
        "clspmv_run_method_f32": (I32, [S["coo"], I32, I32, I32, P(BenchResult)]),
        "clspmv_bandwidth_test": (I32, [C.c_size_t, I32, I32, P(C.c_double), P(C.c_double)]),
        "clspmv_gather_test": (I32, [I32, C.c_longlong, I32, I32, P(C.c_double)]),
        "clspmv_cocktail_evaluate_f32": (I32, [P(Cocktail), VP, VP, VP, I32, I32, P(C.c_double), P(C.c_double),
                                               P(C.c_double)]),
        "clspmv_read_mmf_f32": (I32, [C.c_char_p, S["coo"]]),
        "clspmv_spmm": (I32, [I32, VP, I32, VP, VP, I32, VP, I32, VP, I32, f32, f32, VP]),
        "clspmv_b4csr_spmm_tc_f32": (I32, [VP, I32, VP, I32, VP, I32, f32, f32, VP]),
        "clspmv_tensor_timeouts": (I32, [P(C.c_uint)]),
        "clspmv_stored_values": (I32, [I32, VP, P(C.c_size_t)]),
        "clspmv_spmv_packed": (I32, [I32, VP, I32, VP, VP, VP, VP, VP, f32, f32, VP]),
        "clspmv_sell_plan_create": (I32, [S["sell"], P(VP)]),
        "clspmv_sell_plan_spmv_f32": (I32, [S["sell"], VP, VP, VP, f32, f32, VP]),
        "clspmv_sell_plan_spmv_packed": (I32, [S["sell"], VP, I32, VP, VP, VP, VP, f32, f32, VP]),
        "clspmv_sell_plan_entries": (C.c_longlong, [VP]),
        "clspmv_sell_plan_items": (C.c_longlong, [VP]),
        "clspmv_sell_plan_sector_bytes": (C.c_longlong, [VP]),
        "clspmv_sell_plan_line_bytes": (C.c_longlong, [VP]),
        "clspmv_sell_plan_free": (I32, [VP]),
        "clspmv_pack_values": (I32, [I32, VP, I32, VP, VP, VP]),
        "clspmv_batch_create": (I32, [I32, P(VP)]),
        "clspmv_batch_set": (I32, [VP, P(SpmmJob), I32, VP, P(I32)]),
        "clspmv_batch_run": (I32, [VP, VP]),
        "clspmv_batch_free": (I32, [VP]),
    }
    for fmt in ("csr", "dia", "bdia", "ell", "sell", "bcsr", "bell", "b4csr", "b4ell", "sbell", "coo"):
        sigs[f"clspmv_{fmt}2coo_f32"] = (I32, [S[fmt], S["coo"]])
    for fmt in FORMATS:
        sigs[f"clspmv_free_{fmt}_f32"] = (None, [S[fmt]])
    for fmt in ("coo", "csr", "dia", "bdia", "ell", "sell", "bcsr", "bell", "b4csr", "b4ell", "sbell"):
        sigs[f"clspmv_upload_{fmt}_f32"] = (I32, [S[fmt], S[fmt]])
        sigs[f"clspmv_device_free_{fmt}_f32"] = (I32, [S[fmt]])
    sigs.update({
        "clspmv_device_sort_coo_f32": (I32, [S["coo"], VP]),
        "clspmv_device_coo2csr_f32": (I32, [S["coo"], S["csr"], VP]),
        "clspmv_device_coo2dia_f32": (I32, [S["coo"], S["dia"], I32, VP]),
        "clspmv_device_coo2bdia_f32": (I32, [S["coo"], S["bdia"], I32, VP]),
        "clspmv_device_coo2ell_f32": (I32, [S["coo"], S["ell"], I32, I32, VP]),
        "clspmv_device_coo2sell_f32": (I32, [S["coo"], S["sell"], U32, VP]),
        "clspmv_device_coo2b4csr_f32": (I32, [S["coo"], S["b4csr"], U32, U32, I32, VP]),
        "clspmv_device_coo2bcsr_f32": (I32, [S["coo"], S["bcsr"], U32, U32, I32, VP]),
        "clspmv_device_coo2bell_f32": (I32, [S["coo"], S["bell"], U32, U32, I32, I32, VP]),
        "clspmv_device_coo2b4ell_f32": (I32, [S["coo"], S["b4ell"], U32, U32, I32, I32, VP]),
        "clspmv_device_coo2sbell_f32": (I32, [S["coo"], S["sbell"], U32, U32, U32, VP]),
    })
    for name, (res, args) in sigs.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    return lib


def lib():
    """Loads libclspmv_b200.so (built in-tree by clspmv_mic_b200/build.py).

    There is no fallback: a missing library raises, so nothing can silently
    run on another code path."""
    global _lib
    if _lib is None:
        path = Path(os.environ.get("CLSPMV_LIB", str(LIB_PATH)))
        if not path.exists():
            raise ClspmvError(ERR_ARG, "load", f"{path} is missing; run `python -m clspmv_mic_b200.build`")
        _lib = _declare(C.CDLL(str(path)))
    return _lib


def check(status: int, where: str) -> None:
    if status != OK:
        detail = ""
        if status == ERR_CUDA:
            detail = lib().clspmv_last_cuda_error().decode()
        raise ClspmvError(status, where, detail)
