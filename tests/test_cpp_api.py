"""The C++ mirror of the reference's GpuSolver API (include/ks_solver.hpp) compiled against the library
(tests/cpp/host_api_check.cpp): on the CPU, argument errors, the host algebra on the reference's known answers and, on
a machine without a CUDA device, the loud failure of a valid solver; on the B200 (marked gpu), the H2 33^3 SCF and
forces through qm_gpu::GpuSolver against the reference's pins and the solver's contract (warm start, abort, the step
cap, coincident nuclei)."""
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


def _build(tmp_path):
    exe = str(tmp_path / "host_api_check")
    cmd = ["g++", "-std=c++17", "-O1", "-Wall", "-Wextra", "-Werror", "-I", os.path.join(ROOT, "include"),
           os.path.join(ROOT, "tests", "cpp", "host_api_check.cpp"), "-L", LIBDIR, "-lks_b200", f"-Wl,-rpath,{LIBDIR}", "-o", exe]
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr[-3000:]
    return exe


@pytest.mark.skipif(shutil.which("g++") is None, reason="no C++ compiler")
def test_cpp_mirror_host_checks(ks, tmp_path):
    exe = _build(tmp_path)
    args = [exe, os.path.join(ROOT, "tests", "golden")] + (["--no-device"] if _no_device() else [])
    r = subprocess.run(args, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout[-3000:] + r.stderr[-2000:]
    oks = [x for x in r.stdout.splitlines() if x.startswith("ok ")]
    assert len(oks) >= 16 and "FAIL" not in r.stdout


@pytest.mark.gpu
@pytest.mark.skipif(shutil.which("g++") is None, reason="no C++ compiler")
def test_cpp_mirror_scf_on_the_gpu(ks, tmp_path):
    """The mirror's solve path on the B200: the reference's H2 33^3 energy and force pins through qm_gpu::GpuSolver,
    a warm start, should_abort, the step cap and coincident nuclei as the mirror's exceptions."""
    exe = _build(tmp_path)
    r = subprocess.run([exe, os.path.join(ROOT, "tests", "golden"), "--scf"], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout[-3000:] + r.stderr[-2000:]
    assert "FAIL" not in r.stdout and "ok solve: the H2 33^3 energy pin" in r.stdout, r.stdout[-3000:]
