"""Small seeded test matrices shared by the test modules (row-sorted COO)."""
import numpy as np

from clspmv_mic_b200 import synth


def _coo(t):
    from clspmv_mic_b200 import formats as F
    h, w, r, c, v = t
    return F.coo_matrix(h, w, r, c, v)


def cases():
    """name -> (height, width, rows, cols, vals) tuples; square unless noted."""
    out = {
        "laplace16": synth.laplacian_2d(16),
        "laplace33": synth.laplacian_2d(33),
        "stencil6": synth.stencil_27pt(6),
        "stencil9": synth.stencil_27pt(9),
        "powerlaw3k": synth.powerlaw(3000, maxlen=600, seed=11),
        "blocks300": synth.block_rows(300, 8, 4, 4, seed=5),
        "blocks_odd": synth.block_rows(75, 5, 4, 4, seed=6),
        "banded7": synth.banded(1001, 7),
        "random_empty_rows": synth.random_coo(517, 517, 0.02, seed=3, empty_row_frac=0.3),
        "random_sparse": synth.random_coo(1000, 1000, 0.002, seed=4, empty_row_frac=0.1),
        "one_entry": (7, 7, np.array([3]), np.array([5]), np.array([2.5])),
        "single_row": (1, 50, np.zeros(13, int), np.arange(0, 50, 4)[:13], np.arange(1, 14, dtype=np.float32)),
        "diag_only": (64, 64, np.arange(64), np.arange(64), np.linspace(1, 2, 64)),
        "ragged_tail": synth.random_coo(1023, 1023, 0.01, seed=9, empty_row_frac=0.05),
    }
    return out


def rect_cases():
    """Non-square matrices (formats other than DIA/BDIA)."""
    return {
        "wide": synth.random_coo(200, 777, 0.02, seed=21),
        "tall": synth.random_coo(901, 130, 0.03, seed=22, empty_row_frac=0.2),
    }


def coo_of(name):
    allc = {**cases(), **rect_cases()}
    return _coo(allc[name])
