"""bench.py's output contract on the CPU: the headline JSON line is compact
(callers keep only the last few KB of stdout) and comes last; the reference
arm runs the reference's own code and maps no library of this package."""
import json
import subprocess
import sys

from conftest import ROOT


def _full_headline():
    sys.path.insert(0, str(ROOT))
    import bench
    keys = ["dia", "bdia", "csr_chunk", "coo", "ell", "ell_tail_coo", "sell32", "bell", "sbell", "bcsr"]
    fracs = {k: 0.123 for k in keys}
    roofline = {"bound": "hbm", "kernel": "sell32", "achieved": 5539.1, "peak": 6548.5, "peak_kind": "measured",
                "unit": "GB/s", "frac": 0.846, "frac_useful": 0.075, "min_frac": 0.249,
                "min_frac_kernel": "csr_chunk", "traffic": 2337618692.0, "alg_bytes_per_launch": 2337618692,
                "share_of_step": 0.43}
    e2e = {"value": 483.21, "unit": bench.UNIT, "h2d_bytes_per_step": 62914560, "d2h_bytes_per_step": 62914560,
           "ms_per_step": 1.5123}
    clocks = {"sm_mhz": 1965.0, "sm_max_mhz": 1965.0, "reasons": ["sw_power_cap"], "samples": 120}
    cpu = {"value": 1.712, "unit": bench.UNIT, "cores": 1, "kind": "reference",
           "sample": "csr_spmv on stencil27 best of 50, powerlaw best of 50, blocks4x4 best of 50, 1 thread"}
    parity = {"checked": keys[:4] + keys[5:] + ["csr_merge", "csr_vector", "csr_scalar", "sell32_padded"],
              "rows_over_bound": 0, "max_err_fp64": 2.34e-07, "ref_err_fp64": 3.1e-07,
              "bound": "per row |y - csr_spmv y| <= 1e-5 sum|a x|, full-size matrices"}
    return bench.headline(value=747.51, world=8, steps=200, warmup=5, ms_per_step=0.98582, small=False,
                          roofline=roofline, e2e=e2e, launches=2000, clocks=clocks, cpu_baseline=cpu,
                          parity=parity, fracs=fracs, ell_width=5, gather_peak=264.1)


def test_headline_line_is_compact():
    line = json.dumps(_full_headline())
    assert len(line) < 2048, len(line)
    d = json.loads(line)
    for k in ("metric", "value", "unit", "ms_per_step", "roofline", "e2e", "cpu_baseline", "clocks", "parity"):
        assert k in d
    assert {"frac", "frac_useful", "min_frac"} <= set(d["roofline"])


def test_reference_arm_last_line_and_no_package_library():
    res = subprocess.run([sys.executable, str(ROOT / "bench.py"), "--impl", "reference", "--small", "--steps", "1",
                          "--warmup", "0"], capture_output=True, text=True, timeout=600, cwd=str(ROOT))
    assert res.returncode == 0, res.stderr[-2000:]
    last = res.stdout.strip().splitlines()[-1]
    d = json.loads(last)
    assert d["impl"] == "reference" and d["value"] > 0
    assert d["e2e"]["h2d_bytes_per_step"] == 0 and d["cpu_baseline"]["cores"] >= 1
    assert all(n.startswith("oracle/") for n in d["native_libs"]), d["native_libs"]
    assert len(last) < 2048
