"""Host logic of bench.py (no GPU): the per-kernel algorithmic byte model, the
profile table reader, the workload labels and the reference arm's unavailable
line."""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
import bench  # noqa: E402


class _Wl:
    resolution = (640, 480)
    spp, max_bounces, num_triangles = 4, 3, 130054


WORK = {"points": 1_000_000, "items": 1_100_000_000, "survivors": 500_000_000, "shaded": 100_000_000,
        "tasks": 20_000_000, "items_first_stage": 1_000_000, "visits_walk": 400_000_000,
        "visits_tasks": 3_000_000_000, "candidates": 120_000_000}


def test_every_kernel_of_a_step_has_model_bytes():
    for k in ("k_render_forward", "k_backward_paths", "k_primary_shade", "k_primary_grad", "k_edge_traverse",
              "k_edge_expand", "k_edge_tasks", "k_walk_ctx", "k_edge_level", "k_edge_leaves", "k_edge_line",
              "k_edge_connect", "k_edge_pairs", "k_edge_line_rays",
              "k_edge_shade",
              "k_dp_propagate"):
        assert bench.kernel_bytes(k, _Wl, WORK) > 0, k
    assert bench.kernel_bytes("host_queue_check", _Wl, WORK) == 0


def test_byte_model_counts_nodes_and_rays():
    """Node visits cost 40 B each in the traversal kernels; a ray costs
    24 + 16 + 36 + 64 ceil(log2 T) bytes."""
    w2 = dict(WORK, visits_tasks=WORK["visits_tasks"] + 1000)
    assert bench.kernel_bytes("k_edge_tasks", _Wl, w2) - bench.kernel_bytes("k_edge_tasks", _Wl, WORK) == 40_000
    assert bench.kernel_bytes("k_edge_level", _Wl, w2) - bench.kernel_bytes("k_edge_level", _Wl, WORK) == 40_000
    assert bench.ray_bytes(130054) == 24 + 16 + 36 + 64 * 17
    assert bench.ray_bytes(8) == 24 + 16 + 36 + 64 * 3
    w3 = dict(WORK, survivors=WORK["survivors"] + 10)
    assert bench.kernel_bytes("k_edge_connect", _Wl, w3) - bench.kernel_bytes("k_edge_connect", _Wl, WORK) == \
        10 * (32 + 2 * bench.ray_bytes(130054))


def test_default_workload_is_the_glossy_heightfield_configuration():
    w = bench.WORKLOADS[bench.DEFAULT_WORKLOAD]
    assert w["resolution"] == (640, 480) and w["spp"] == 64 and w["max_bounces"] == 3
    assert w["spp"] % w["step_spp"] == 0
    bench.WORKLOAD = w
    label = bench.workload_label()
    assert "640x480" in label and "64 spp" in label and "16 steps of 4 spp" in label


def test_profile_table_reader(tmp_path, monkeypatch):
    prof = tmp_path / "profiles"
    prof.mkdir()
    (prof / "kernels_heightfield.txt").write_text("# comment\nk_edge_tasks 123456 87.5 41.0 76800\n")
    monkeypatch.setattr(bench, "ROOT", str(tmp_path))
    monkeypatch.setattr(bench, "WORKLOAD_KEY", "heightfield")
    p = bench.load_profile("k_edge_tasks")
    assert p["dram_bytes"] == 123456 and p["l2_hit_pct"] == 87.5 and p["units"] == 76800
    assert bench.load_profile("k_edge_connect") is None


def test_reference_arm_reports_ggx_workload_unavailable():
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--workload",
                          "heightfield_ggx", "--steps", "1", "--warmup", "0"], capture_output=True, text=True,
                         cwd=ROOT, timeout=600)
    assert out.returncode == 0, out.stderr[-2000:]
    line = json.loads(out.stdout.strip().splitlines()[-1])
    assert line["impl"] == "reference" and "GGX" in line["unavailable"]
