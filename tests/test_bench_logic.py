"""Host logic of bench.py (no GPU): composite stages, the traffic table, the
algorithmic byte model and the reference arm's unavailable line."""
import json
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
import bench  # noqa: E402


def test_composite_stages_are_summed():
    stages = [("k_render_forward", 0.5), ("k_backward_paths", 4.0), ("k_primary_shade", 1.5),
              ("k_primary_grad", 1.0), ("k_edge_traverse", 5.0), ("k_edge_line_rays", 5.0), ("k_edge_shade", 4.0),
              ("k_dp_propagate", 0.5)]
    merged = dict(bench.merge_stages(stages))
    assert merged["k_primary_edges"] == pytest.approx(2.5)
    assert merged["k_edge_eval"] == pytest.approx(9.0)
    assert "k_edge_shade" not in merged and "k_primary_grad" not in merged
    assert sum(merged.values()) == pytest.approx(sum(ms for _, ms in stages))
    split = dict(bench.merge_stages([("k_edge_expand", 4.0), ("k_edge_tasks", 170.0), ("k_edge_line", 14.0),
                                     ("k_edge_rays", 114.0), ("k_edge_shade", 17.0)]))
    assert split == pytest.approx({"k_edge_traverse": 174.0, "k_edge_eval": 145.0})


def test_traffic_table_and_byte_model():
    bench.WORKLOAD = bench.WORKLOADS["soft_shadow"]
    eval_bytes = bench.load_traffic("k_edge_eval")
    assert eval_bytes and eval_bytes > 1e9  # the committed capture of the evaluation kernels
    assert bench.load_traffic("k_primary_edges") > 0
    bench.WORKLOAD = bench.WORKLOADS["heightfield"]
    assert bench.load_traffic("k_edge_eval") is None  # captured on another workload
    bench.WORKLOAD = bench.WORKLOADS["soft_shadow"]

    class Wl:
        resolution = (512, 512)
        spp, max_bounces, num_triangles = 16, 1, 8
    counts = (3_579_904, 39_038_077)
    for stage in ("k_render_forward", "k_backward_paths", "k_edge_traverse", "k_edge_eval", "k_dp_propagate",
                  "k_primary_edges"):
        assert bench.stage_bytes(stage, Wl, counts) > 0, stage


def test_reference_arm_reports_ggx_workload_unavailable():
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--workload",
                          "heightfield_ggx", "--steps", "1", "--warmup", "0"], capture_output=True, text=True,
                         cwd=ROOT, timeout=600)
    assert out.returncode == 0, out.stderr[-2000:]
    line = json.loads(out.stdout.strip().splitlines()[-1])
    assert line["impl"] == "reference" and "GGX" in line["unavailable"]
