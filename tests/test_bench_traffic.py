"""bench.py's DRAM traffic of the gather comes from a recorded reduced-case capture and is tied to the kernel
sources it was taken on: reported, scaled by node-taps, while they are unchanged; null with the reason once they
differ (so a kernel change never leaves a stale figure in the bench line)."""

import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

import bench  # noqa: E402


def test_traffic_scales_with_node_taps_on_the_captured_sources(monkeypatch):
    g = dict(bench.GATHER_TRAFFIC, sources_sha256=bench.gather_sources_sha256())
    monkeypatch.setattr(bench, "GATHER_TRAFFIC", g)
    t1, hit, why = bench.gather_traffic(1.0e9)
    t2, _, _ = bench.gather_traffic(2.0e9)
    assert why is None and hit == g["l2_read_hit_rate"]
    assert t1 == g["dram_bytes_per_node_tap"] * 1.0e9 and t2 == 2 * t1


def test_traffic_is_null_when_the_sources_changed(monkeypatch):
    g = dict(bench.GATHER_TRAFFIC, sources_sha256="0" * 64)
    monkeypatch.setattr(bench, "GATHER_TRAFFIC", g)
    t, hit, why = bench.gather_traffic(1.0e9)
    assert t is None and hit is None and "changed" in why


def test_hash_covers_the_gather_and_tap_sources():
    assert set(bench.GATHER_SOURCES) == {"exmarg_b200/csrc/gather.cu", "exmarg_b200/csrc/taps.cu",
                                         "exmarg_b200/csrc/kernels.cuh"}
    assert len(bench.gather_sources_sha256()) == 64
