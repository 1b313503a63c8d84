"""Host logic of bench.py that needs no GPU: the section list and the compact summary object that
ends the JSON line (it must survive a line with any subset of sections)."""
import os
import sys

import pytest

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
import bench  # noqa: E402


class Args:
    def __init__(self, sections):
        self.sections = sections


def test_wanted_sections():
    assert bench.wanted_sections(Args("all")) == set(bench.SECTIONS)
    assert bench.wanted_sections(Args("none")) == set()
    assert bench.wanted_sections(Args("serving, bvh")) == {"serving", "bvh"}
    with pytest.raises(SystemExit):
        bench.wanted_sections(Args("serving,unknown"))


def headline():
    return {"value": 1.26e9, "e2e": {"value": 1.25e9}, "roofline": {"frac": 0.5, "dram_frac": 0.04}}


def test_summary_of_a_headline_only_line():
    s = bench.summary(headline())
    assert s["value"] == 1.26e9 and s["e2e"] == 1.25e9 and s["roofline_frac"] == 0.5
    for key in ("plain_form_speedup_of_value", "reference_build_b200_value", "batched_speedup_vs_plain_form", "cpu_baseline_value"):
        assert s[key] is None
    assert s["bvh_build_s_host_device"] == {}
    assert "serving_latency_s" not in s


def test_summary_of_a_line_with_sections():
    line = headline() | {
        "plain_form": {"speedup_of_value": 2.2},
        "reference_build_b200": {"value": 1.13e8, "speedup_of_value": 11.1},
        "batched": {"speedup_vs_plain_form": 2.02},
        "cpu_baseline": {"value": 9.7e5},
        "bvh_build": {"spheres-1m": {"host": {"bvh_build_s": 0.9}, "device": {"bvh_build_s": 0.024}}},
        "serving": {"jobs_per_rate": 200,
                    "served": {"20_jobs_per_s": {"p50_latency_s": 0.07, "p99_latency_s": 5.5}, "admitted_high_water_bytes": 1},
                    "plain": {"20_jobs_per_s": {"p50_latency_s": 3.4, "p99_latency_s": 5.6}}},
    }
    s = bench.summary(line)
    assert s["plain_form_speedup_of_value"] == 2.2
    assert s["reference_build_b200_speedup_of_value"] == 11.1
    assert s["batched_speedup_vs_plain_form"] == 2.02
    assert s["bvh_build_s_host_device"] == {"spheres-1m": [0.9, 0.024]}
    assert s["serving_jobs_per_rate"] == 200
    # only the modes that ran appear; non-dict entries of a mode (high-water bytes) are skipped
    assert s["serving_latency_s"] == {"20_jobs_per_s": {"served_p50": 0.07, "served_p99": 5.5, "plain_p50": 3.4, "plain_p99": 5.6}}
