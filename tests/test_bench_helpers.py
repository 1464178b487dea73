"""Host-side helpers of bench.py (no GPU): the workload definitions the bench
line reports and the launch counts it claims."""
import pathlib
import sys

import numpy as np

ROOT = pathlib.Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT))
import bench  # noqa: E402


def test_mixed_workload_matches_its_definition():
    # L=12 x 512 samples (16 T), L=14 x 384 (20 T), L=16 x 256 (24 T), 2 copies
    assert [(l, 32 * w, t) for l, w, t in bench.MIXED] == [(12, 512, 16), (14, 384, 20),
                                                           (16, 256, 24)]
    per_sweep = bench.MIXED_WORDS_PER_SWEEP * 32
    assert per_sweep == 120_791_040  # spin-flip attempts per sweep of every member
    cfg = bench.mixed_config(1, *bench.REF_SCHEDULE)
    assert [m["L"] for m in cfg["members"]] == [12, 14, 16]
    assert (cfg["swap_every"], cfg["measure_every"]) == (16, 1024)
    assert "sweeps_per_step" not in cfg  # the step size is reported beside the config


def test_rank_shards_offset_the_sample_words():
    a = bench.mixed_members(16, 1024, rank=0)
    b = bench.mixed_members(16, 1024, rank=3)
    for m0, m3 in zip(a, b):
        assert m0["word0"] == 0 and m3["word0"] == 3 * m3["n_words"]
        assert m0["seed"] == m3["seed"]  # one run, split by word ranges
        np.testing.assert_array_equal(m0["betas"], m3["betas"])


def test_ladder_is_geometric_in_temperature():
    b = bench.ladder(24)
    temps = 1.0 / b
    assert np.isclose(temps[0], bench.T_MIN) and np.isclose(temps[-1], bench.T_MAX)
    ratios = temps[1:] / temps[:-1]
    np.testing.assert_allclose(ratios, ratios[0])


def test_production_config_shares_the_reference_arm():
    ours = bench.workload_config(1, 1, 1, "auto", 0.0)
    assert ours == bench.workload_config(1)  # what the reference arm reports
    assert "sweeps_per_step" not in ours


def test_streaming_launch_counts_follow_the_schedule():
    # every sweep exchanges and measures: 2 colour launches, decisions,
    # exchange with overlaps, measurement
    assert bench.stream_launches(0, 8, 1, 1) == 8 * 5
    # no exchange, no measurement: the colour launches only
    assert bench.stream_launches(0, 8, 0, 0) == 8 * 2
    # the reference schedule over 32 sweeps from 0: two exchanges (after
    # sweeps 15 and 31), no measurement
    assert bench.stream_launches(0, 32, 16, 1024) == 32 * 2 + 2 * 2
    # a measurement without an exchange: decisions, overlaps, measurement
    assert bench.stream_launches(1023, 1, 0, 1024) == 2 + 3
