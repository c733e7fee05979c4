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


def _check(line, world, n=25):
    import bench
    assert line["impl"] == "reference"
    assert line["metric"] == bench.METRIC and line["unit"] == "s" and line["higher_is_better"] is False
    config = dict(bench.CONFIG, parallelism=f"replicas x{world}", grid=n)
    config["workload"] = bench.CONFIG["workload"].replace("95^3", f"{n}^3")
    assert line["config"] == config
    assert line["requested"] == {"steps": 3, "warmup": 2}
    acc = line["accuracy"]
    assert acc["status"] == 0 and acc["energy_ha"] < 0 and len(acc["forces"]) == 3
    assert line["value"] > 0 and line["ms_per_step"] == 1000.0 * line["value"]
    cpu = line["cpu_baseline"]
    assert cpu["kind"] == "port" and cpu["cores"] >= 1 and cpu["value"] == line["value"] and "oracle" in cpu["sample"]
    assert "not extrapolated" in cpu["sample"]
    assert line["e2e"] == {"value": line["value"], "unit": "s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}
    assert line["n_gpus"] == world and line["steps"] == 1 and line["warmup"] == 0


def test_reference_arm_line():
    """One full (small-grid) oracle solve timed as one step, whatever K and W were asked for; they are echoed."""
    r = subprocess.run([sys.executable, "bench.py", "--impl", "reference", "--steps", "3", "--warmup", "2", "--ref-grid", "25"], cwd=ROOT,
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
           "--master-port", str(port), "bench.py", "--impl", "reference", "--gpus", "2", "--steps", "3", "--warmup", "2",
           "--ref-grid", "25"]
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
    assert cpu["method"] == "extrapolated" and 0 < cpu["measured_sample_s"] < cpu["value"]
    one = cpu["single_thread"]
    assert one["cores"] == 1 and one["value"] > 0 and "oracle" in one["sample"]
    assert set(cpu["stage_s"]) == {"lobpcg_iteration_k5", "poisson_cg_iteration", "lobpcg_iteration_k5_1t",
                                   "poisson_cg_iteration_1t", "hpsi_one_vector_1t"}
    assert all(t > 0 for t in cpu["stage_s"].values())
    json.dumps(cpu)


def test_roofline_traffic_constant():
    """The roofline's traffic: the ncu-measured DRAM bytes per vector of the H psi launch scaled to the bench's
    64-vector launch: no re-reads above the algorithmic (8k + 4) N^3 bytes (at most 5 % over), and not far below
    them (part of the output is still in L2 when the kernel ends: 0.94 in the committed capture)."""
    import bench
    t = bench.HPSI_DRAM_BYTES_PER_VECTOR * 64
    algo = (8 * 64 + 4) * 95 ** 3
    assert 0.85 < t / algo < 1.05, (t, algo)


def test_in_scf_rooflines_from_kernel_times():
    """The bench's in-SCF rooflines: per shape the mean launch time, the achieved algorithmic GB/s and its fraction of
    the peak, sorted by total device time; the dominant shape is the first."""
    import bench
    kt = [{"kernel": "jacobi", "count": 8, "aux": 0, "launches": 10, "total_ms": 0.4, "mean_us": 40.0, "bytes": 8.0e7, "gbs": 2000.0},
          {"kernel": "gram", "count": 24, "aux": 24, "launches": 5, "total_ms": 0.5, "mean_us": 100.0, "bytes": 1.6e8, "gbs": 1600.0},
          {"kernel": "hpsi", "count": 8, "aux": 0, "launches": 0, "total_ms": 0.0, "mean_us": 0.0, "bytes": 5.0e7, "gbs": 0.0}]
    r = bench.in_scf_rooflines(kt, 6400.0, "measured")
    assert [k["kernel"] for k in r["kernels"]] == ["gram", "jacobi"]
    d = r["dominant"]
    assert d["kernel"] == "gram" and d["bound"] == "hbm" and abs(d["frac"] - 0.25) < 1e-12 and d["peak_source"] == "measured"
    assert bench.in_scf_rooflines([], 6400.0, "measured") == {"kernels": [], "dominant": None}
