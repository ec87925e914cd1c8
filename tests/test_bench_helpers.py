"""bench.py's host-side helpers (CPU only): the committed ncu summaries parse into the figures the bench
line reads, and the source stamp that ties a summary to a library build is stable and covers the
CUDA sources."""
import os
import re

import bench

PROFILES = [bench.PROFILE, bench.GRID_PROFILE, os.path.join(bench.ROOT, "profiles", "ns_shade_soup_1080p.md")]


def test_profiles_carry_the_figures_the_bench_reads():
    for path in PROFILES:
        prof = bench.profile_figures(path)
        assert re.fullmatch(r"[0-9a-f]{16}", str(prof["source_sha16"])), path
        assert prof["rays_per_launch"] == 1920 * 16 * (1080 // 16), path
        assert prof["dram_bytes_per_launch"] > 0, path
        for k in ("l1_hit_pct", "l2_hit_pct", "l1_throughput_pct", "dram_throughput_pct", "alu_pipe_pct",
                  "lanes_active_per_inst", "issue_active_pct"):
            assert isinstance(prof[k], float), (path, k)
        assert 0.0 < prof["lanes_active_per_inst"] <= 32.0


def test_source_stamp_is_stable_and_tracks_the_sources(tmp_path, monkeypatch):
    a, b = bench.source_stamp(), bench.source_stamp()
    assert a == b and re.fullmatch(r"[0-9a-f]{16}", a)
    # a copy of the sources with one byte changed gives another stamp
    from mobileraytracer_b200 import build
    src = tmp_path / "csrc"
    src.mkdir()
    for f in os.listdir(build.CSRC):
        if f.endswith((".cu", ".cuh", ".h")):
            (src / f).write_bytes(open(os.path.join(build.CSRC, f), "rb").read())
    monkeypatch.setattr(build, "CSRC", str(src))
    assert bench.source_stamp() == a
    first = sorted(os.listdir(src))[0]
    (src / first).write_bytes((src / first).read_bytes() + b"\n")
    assert bench.source_stamp() != a


def test_measured_peak_is_read_from_the_peaks_file():
    peak, kind = bench.measured_peak()
    assert peak > 1000.0 and kind in ("measured", "fallback")
