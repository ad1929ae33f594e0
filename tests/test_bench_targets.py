"""The bench line's `targets` summary (no GPU): which engine meets which half
of the target, from the legs' measured figures."""

import importlib.util
from pathlib import Path

ROOT = Path(__file__).resolve().parent.parent


def bench():
    spec = importlib.util.spec_from_file_location("bench_for_test", ROOT / "bench.py")
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def legs(fp32_max, exact_max):
    err = lambda m: None if m is None else {"rel_max": m}
    return {"plain_fp32_sweep": {"value": 12e12, "surfaces_vs_fp64": err(fp32_max)},
            "exact32_engine": {"value": 9e12, "surfaces_vs_fp64": err(exact_max),
                               "identical_to_plain_port": True},
            "plain_port": {"value": 0.5e12, "surfaces_vs_fp64": err(exact_max)}}


def test_targets_of_the_mixed_headline():
    t = bench().targets(6e12, legs(2e-2, 2e-2), "mixed64")
    assert t["surface_rel_error_le_1e-5_vs_fp64"] == {"headline": True, "fp32_form": False,
                                                     "exact32": False}
    assert t["headline_over_plain_port"] == 12.0
    assert t["headline_over_fp32_form"] == 0.5
    assert "exact32" in t["reference_cpu_ring_records_bit_for_bit"]


def test_targets_without_an_fp64_reference():
    """An exact-f32 headline has no FP64 surfaces to compare the legs with."""
    t = bench().targets(9e12, legs(None, None), "exact32")
    assert t["surface_rel_error_le_1e-5_vs_fp64"] == {"headline": False, "fp32_form": None,
                                                     "exact32": None}
