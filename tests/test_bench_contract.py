"""bench.py's reference arm on CPU: it times the reference's CPU build (or the
C oracle where that build is absent) on the host cores and prints one JSON
line with the contract's keys."""
import json
import os
import subprocess
import sys

from conftest import ROOT


def test_reference_arm_prints_one_json_line():
    env = dict(os.environ)
    for k in ("WORLD_SIZE", "RANK", "LOCAL_RANK"):
        env.pop(k, None)
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "2",
                          "--warmup", "1", "--cpu-sample", "16", "--nn", "2"], env=env, stdout=subprocess.PIPE,
                         stderr=subprocess.PIPE, check=True, timeout=600)
    lines = [l for l in out.stdout.decode().splitlines() if l.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    for k in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better", "scaling",
              "vs_baseline", "dtype", "data", "config", "cpu_baseline", "e2e"):
        assert k in d, k
    assert d["impl"] == "reference" and d["metric"] == "cell-steps/s" and d["value"] > 0
    assert d["cpu_baseline"]["kind"] in ("reference", "port") and d["cpu_baseline"]["cores"] >= 1
    assert d["e2e"]["value"] == d["value"] and d["e2e"]["h2d_bytes_per_step"] == 0
    assert d["config"]["workload"].startswith("RK4 step")


def test_reference_arm_under_torchrun_two_ranks():
    """Launched like the multi-GPU driver (torchrun, 2 ranks; gloo on CPU):
    rank 0 alone times the reference and prints the line, rank 1 exits 0."""
    import socket
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    env = dict(os.environ)
    for k in ("WORLD_SIZE", "RANK", "LOCAL_RANK", "MASTER_ADDR", "MASTER_PORT"):
        env.pop(k, None)
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2", "--master-addr",
           "127.0.0.1", "--master-port", str(port), os.path.join(ROOT, "bench.py"), "--impl", "reference", "--gpus",
           "2", "--steps", "2", "--warmup", "1", "--cpu-sample", "16", "--nn", "2"]
    out = subprocess.run(cmd, env=env, stdout=subprocess.PIPE, stderr=subprocess.PIPE, check=True, timeout=600)
    lines = [l for l in out.stdout.decode().splitlines() if l.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["n_gpus"] == 2 and d["value"] > 0


def test_step_traffic_from_profiles():
    """The roofline's per-step DRAM bytes are the four stage launches' ncu
    figures; sizes without a capture give None."""
    sys.path.insert(0, ROOT)
    import bench
    with open(os.path.join(ROOT, "profiles", "traffic.json")) as f:
        t = json.load(f)
    for dt in ("f64", "f32"):
        keys = ["stage_%s_%s_1024_642" % (k, dt) for k in ("s1", "s2", "s3", "s4")]
        if not all(k in t for k in keys):
            assert bench.step_traffic(dt, 1024, 642) is None
            continue
        want = sum(t[k] for k in keys)
        assert bench.step_traffic(dt, 1024, 642) == want
        # within 10 % of the bytes the 12-pass step moves (768 / 384 B per cell-step)
        moved = bench.MOVED_BYTES_PER_CELL_STEP[dt] * 1024 * 1024 * 642
        assert 1.0 <= want / moved < 1.1
    assert bench.step_traffic("f64", 512, 642) is None


def test_reference_arm_names_its_sample():
    """The reference arm's config names the sample it timed, not the full grid."""
    env = dict(os.environ)
    for k in ("WORLD_SIZE", "RANK", "LOCAL_RANK"):
        env.pop(k, None)
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "2",
                          "--warmup", "1", "--cpu-sample", "16", "--nn", "2", "--cpu-seconds-1t", "2"], env=env,
                         stdout=subprocess.PIPE, stderr=subprocess.PIPE, check=True, timeout=600)
    d = json.loads([l for l in out.stdout.decode().splitlines() if l.startswith("{")][0])
    assert d["config"]["nx"] == 16 and d["config"]["nv"] == 42
    assert "16x16 cells x 42 velocities sample" in d["config"]["workload"]
    one = d["cpu_baseline"]["one_thread"]
    assert one["cores"] == 1 and one["value"] > 0
