"""Host-side bookkeeping of bench.py: the stage the roofline entry reports and
the algorithmic bytes per stage call."""
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

import bench  # noqa: E402


def test_config_is_identical_across_arms():
    # the reference arm and the GPU arm print the same `config`
    a = bench.config_desc("B=100 ...", 1)
    b = bench.config_desc("B=100 ...", 1)
    assert a == b and "pairs_per_step" not in a


def test_traffic_table_parsed_per_stage(tmp_path):
    # the committed traffic table maps onto known stages
    for k in bench.ncu_traffic():
        assert bench.stage_bytes(k, 100, 200, 3, 131072) is not None
    # kernels of one stage are summed; template arguments are ignored
    p = tmp_path / "t.md"
    p.write_text("| kernel | launches | us / launch | DRAM read MB / launch | DRAM write MB / launch |\n"
                 "|---|---|---|---|---|\n"
                 "| `k_so3_fft_a<200, 4>` | 1 | 22.0 | 31.50 | 0.50 |\n"
                 "| `void k_so3_c2r_tail<200>` | 1 | 33.0 | 32.00 | 0.00 |\n"
                 "| `k_fuse_z<200>` | 1 | 130.0 | 200.00 | 24.00 |\n")
    t = bench.ncu_traffic(str(p))
    assert t == {"so3_fft": 64_000_000, "fuse_z": 224_000_000}


def test_stage_bytes_per_call():
    bw, N, C, P = 100, 200, 3, 131072
    n = 2 * bw
    # one SHT call transforms both clouds' channels
    assert bench.stage_bytes("sht", bw, N, C, P) == 2 * (C * n * n * 4 + C * bw * bw * 8)
    # per-cloud stages count one cloud
    assert bench.stage_bytes("s2_sample", bw, N, C, P) == P * 20 + 4 * n * n * 4
    assert bench.stage_bytes("unknown", bw, N, C, P) is None
