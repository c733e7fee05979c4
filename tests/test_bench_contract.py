"""bench.py's reference arm on the CPU: the JSON line's keys and meaning (the oracle port timed on host cores, the same
metric, unit, direction and config as the CUDA arm), alone and under torchrun, where rank 0 alone prints and the other
ranks exit 0 without work. CPU only: the arm never touches a GPU."""
import json
import os
import socket
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)


def _lines(out):
    return [json.loads(x) for x in out.splitlines() if x.startswith("{")]


def _check(line, world):
    import bench
    assert line["impl"] == "reference"
    assert line["metric"] == bench.METRIC and line["unit"] == "s" and line["higher_is_better"] is False
    assert line["config"] == dict(bench.CONFIG, parallelism=f"replicas x{world}")
    assert line["value"] > 0 and line["ms_per_step"] == 1000.0 * line["value"]
    cpu = line["cpu_baseline"]
    assert cpu["kind"] == "port" and cpu["cores"] >= 1 and cpu["value"] == line["value"] and "oracle" in cpu["sample"]
    assert line["e2e"] == {"value": line["value"], "unit": "s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}
    assert line["n_gpus"] == world and line["steps"] == 1 and line["warmup"] == 0


def test_reference_arm_line():
    r = subprocess.run([sys.executable, "bench.py", "--impl", "reference", "--steps", "1", "--warmup", "0"], cwd=ROOT,
                       capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = _lines(r.stdout)
    assert len(lines) == 1
    _check(lines[0], 1)


def test_reference_arm_under_torchrun_prints_once():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2", "--master-addr", "127.0.0.1",
           "--master-port", str(port), "bench.py", "--impl", "reference", "--gpus", "2", "--steps", "1", "--warmup", "0"]
    env = dict(os.environ, OMP_NUM_THREADS="1")
    r = subprocess.run(cmd, cwd=ROOT, capture_output=True, text=True, timeout=900, env=env)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = _lines(r.stdout)
    assert len(lines) == 1, r.stdout[-2000:]
    _check(lines[0], 2)


def test_cpu_baseline_entry():
    """The CUDA arm's cpu_baseline (computed on the CPU): the all-threads figure, the single-thread one and the
    per-stage times, all positive, with the single-thread sample on one core."""
    import bench
    cpu = bench.cpu_baseline_entry()
    assert cpu["kind"] == "port" and cpu["unit"] == "s" and cpu["cores"] == (os.cpu_count() or 1) and cpu["value"] > 0
    one = cpu["single_thread"]
    assert one["cores"] == 1 and one["value"] > 0 and "oracle" in one["sample"]
    assert set(cpu["stage_s"]) == {"lobpcg_iteration_k5", "poisson_cg_iteration", "lobpcg_iteration_k5_1t",
                                   "poisson_cg_iteration_1t", "hpsi_one_vector_1t"}
    assert all(t > 0 for t in cpu["stage_s"].values())
    json.dumps(cpu)


def test_profiled_traffic_scales_the_committed_capture():
    """The roofline's traffic: the committed ncu capture (profiles/stencil_hpsi_95.md, 48 vectors) scaled to the
    bench's 64-vector launch, and within 5 % of the algorithmic (8k + 4) N^3 bytes (0.98: no re-reads; some of the
    output is still in L2 at the kernel's end); None without a summary."""
    import bench
    t = bench.profiled_traffic(64)
    algo = (8 * 64 + 4) * 95 ** 3
    assert t is not None and abs(t / algo - 1.0) < 0.05, (t, algo)
    assert bench.profiled_traffic(64, prof="/nonexistent/summary.md") is None
