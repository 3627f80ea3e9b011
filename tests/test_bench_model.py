"""CPU checks of bench.py: the roofline arithmetic (the compulsory-bytes model
of the compositor launches and the measured-traffic lookup, which applies to
the workload it was measured on only) and the reference arm's JSON line."""
import os
import types

import torch

import bench


def test_compositor_bytes_model():
    C, N, H, W, R, D, s_t = 2, 10, 16, 24, 8, 3, 2
    radii = torch.zeros((C, N), dtype=torch.int32)
    radii[0, :7] = 3
    radii[1, 2:5] = 1
    meta = {"radii": radii, "isect_ids": torch.zeros(123, dtype=torch.int64), "tile_width": 2, "tile_height": 1}
    fwd, bwd, counts = bench.compositor_bytes(meta, D, R, s_t, N, C, H, W)
    V, I, T, P = 10, 123, 4, C * H * W
    assert counts == dict(visible=V, isects=I, tiles=T, pixels=P)
    per_splat = 60 + 4 * D + 4 * R * R * s_t
    assert fwd == V * per_splat + 4 * I + 4 * T + P * (4 * D + 32)
    assert bwd == (V * per_splat + 4 * I + 4 * T + P * (8 * D + 56) + V * (68 + 4 * D) + N * 4 * R * R * 4 * 2)


def test_measured_traffic_applies_to_its_workload_only():
    args = types.SimpleNamespace(traffic_bytes=None, workload="mixture1m")
    t = bench.traffic_bytes(args, 1_000_000, 4, 32, 8, 64)
    assert t == bench.ADJOINT_KERNEL_DRAM_BYTES + 1_000_000 * 32 * 32 * 16
    assert abs(t - 80.198e9) < 0.01e9
    assert bench.traffic_bytes(args, 1_000_000, 4, 32, 16, 0) is None  # another tile size
    assert bench.traffic_bytes(args, 500_000, 4, 32, 8, 64) is None
    args.traffic_bytes = 1.5e9
    assert bench.traffic_bytes(args, 3, 1, 8, 16, 0) == 1.5e9


def test_reference_arm_prints_the_contract_line():
    """``bench.py --impl reference`` times the CPU oracle (no GPU needed); a reduced workload keeps this quick."""
    import json
    import subprocess
    import sys

    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    out = subprocess.run([sys.executable, os.path.join(root, "bench.py"), "--impl", "reference", "--steps", "2",
                          "--warmup", "0", "--splats", "20000", "--cameras", "1"], capture_output=True, text=True,
                         cwd=root, timeout=600)
    assert out.returncode == 0, out.stderr[-2000:]
    line = json.loads(out.stdout.strip().splitlines()[-1])
    assert line["impl"] == "reference" and line["metric"] == bench.METRIC and line["unit"] == "Mpix/s"
    assert line["higher_is_better"] is True and line["steps"] == 2 and line["value"] > 0
    cb = line["cpu_baseline"]
    assert cb["kind"] == "port" and cb["cores"] >= 1 and cb["value"] == line["value"] and cb["sample"]
    assert line["e2e"] == {"value": line["value"], "unit": "Mpix/s", "h2d_bytes_per_step": 0,
                           "d2h_bytes_per_step": 0}
