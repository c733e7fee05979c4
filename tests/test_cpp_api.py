"""The C++ mirror of the reference's GpuSolver API (include/ks_solver.hpp) compiled against the library and run on
the CPU (tests/cpp/host_api_check.cpp): argument errors, the host algebra on the reference's known answers and, on a
machine without a CUDA device, the loud failure of a valid solver. CPU only."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIBDIR = os.path.join(ROOT, "atomic-sandbox_b200")


def _no_device():
    try:
        import torch
        return not torch.cuda.is_available()
    except Exception:
        return True


@pytest.mark.skipif(shutil.which("g++") is None, reason="no C++ compiler")
def test_cpp_mirror_host_checks(ks, tmp_path):
    exe = str(tmp_path / "host_api_check")
    cmd = ["g++", "-std=c++17", "-O1", "-Wall", "-Wextra", "-Werror", "-I", os.path.join(ROOT, "include"),
           os.path.join(ROOT, "tests", "cpp", "host_api_check.cpp"), "-L", LIBDIR, "-lks_b200", f"-Wl,-rpath,{LIBDIR}", "-o", exe]
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr[-3000:]
    args = [exe, os.path.join(ROOT, "tests", "golden")] + (["--no-device"] if _no_device() else [])
    r = subprocess.run(args, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout[-3000:] + r.stderr[-2000:]
    oks = [x for x in r.stdout.splitlines() if x.startswith("ok ")]
    assert len(oks) >= 16 and "FAIL" not in r.stdout
