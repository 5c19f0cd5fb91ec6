"""Host-side pieces of bench.py that need no GPU: the metric's summary of the batched
comparison and the digest that compares two batches bit for bit."""
import numpy as np

import bench


def test_metric_summary_reads_the_comparison():
    mc = {"plain_fp64": {"value": 166.3e6}, "plain_fp64_one_event_at_a_time": {"value": 55.5e6},
          "learned_deferred_fp32_lockstep": {"value": 185.0e6, "L2_T": 1.8e-7, "L2_pibar": 1.3e-6,
                                             "meets_L2T_1e-6": True},
          "fp32_lockstep": {"value": 190.4e6}, "best_form": "fp32_lockstep", "events": 256}
    s = bench.metric_summary(mc)
    assert s["form"] == "learned_deferred_fp32_lockstep"
    assert abs(s["vs_plain_unbatched"] - 185.0 / 55.5) < 1e-12
    assert abs(s["vs_plain_batched"] - 185.0 / 166.3) < 1e-12
    assert s["best_form"] == "fp32_lockstep" and s["best_value"] == 190.4e6
    assert s["meets_L2T_1e-6"] and s["L2_T"] == 1.8e-7


def test_metric_summary_tolerates_missing_forms():
    s = bench.metric_summary({"plain_fp64": {"value": 1.0}})
    assert s["value"] is None and "vs_plain_unbatched" not in s and s["best_value"] is None


def test_fields_digest_is_bitwise():
    rng = np.random.default_rng(3)
    f = {"T": rng.random(100), "pibar": rng.random(100), "pi": rng.random((100, 3))}
    g = {k: v.copy() for k, v in f.items()}
    assert bench._fields_digest(f) == bench._fields_digest(g)
    g["T"][17] = np.nextafter(g["T"][17], 2.0)         # one ulp
    assert bench._fields_digest(f) != bench._fields_digest(g)
