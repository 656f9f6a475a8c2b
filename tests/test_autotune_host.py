"""Matrix signatures of the partition tuner (host only)."""
import numpy as np

from clspmv_mic_b200 import formats as F
from clspmv_mic_b200.autotune import KNOBS, signature

from matrices import cases, coo_of


def test_signature_is_structural():
    a = signature(coo_of("laplace33"))
    assert a == signature(coo_of("laplace33"))
    h, w, r, c, v = cases()["laplace33"]
    same_pattern = F.coo_matrix(h, w, r, c, np.asarray(v) * 3.0)      # values do not matter
    assert signature(same_pattern) == a
    assert signature(coo_of("powerlaw3k")) != a
    assert signature(coo_of("blocks300")) != signature(coo_of("blocks_odd"))


def test_knobs_start_with_the_reference_defaults():
    assert KNOBS[0] == {}
    assert all(set(k) <= {"dia_priority_multiplier", "estimate_flat_partial", "estimate_flat_full"} for k in KNOBS)
