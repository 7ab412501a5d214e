"""Host-side bookkeeping of bench.py: the stage the roofline entry reports and
the algorithmic bytes per stage call."""
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

import bench  # noqa: E402


def test_dominant_stage_follows_the_launch_list_share():
    # per-stage CUDA events overlap between the two clouds' streams (sampling
    # looks longest); the launch list's serialised share picks the forward
    events = {"s2_sample": 0.164, "spatial_fwd": 0.139, "fuse_z": 0.138, "so3_synth": 0.062}
    assert bench.dominant_stage(events, True) == "spatial_fwd"
    assert bench.dominant_stage(events, False) == "s2_sample"
    # the shares cover every stage and, with the one-time Legendre table
    # (2.9 %), the whole capture
    assert abs(sum(bench.NCU_SHARE_B100_N200.values()) + 2.9 - 100.0) < 0.5
    assert set(bench.NCU_SHARE_B100_N200) == set(bench.NCU_TRAFFIC_B100_N200)


def test_stage_bytes_per_call():
    bw, N, C, P = 100, 200, 3, 131072
    n = 2 * bw
    # one SHT call transforms both clouds' channels
    assert bench.stage_bytes("sht", bw, N, C, P) == 2 * (C * n * n * 4 + C * bw * bw * 8)
    # per-cloud stages count one cloud
    assert bench.stage_bytes("s2_sample", bw, N, C, P) == P * 20 + 4 * n * n * 4
    assert bench.stage_bytes("unknown", bw, N, C, P) is None
