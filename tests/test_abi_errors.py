"""Argument errors at the C ABI and in its Python mirror, checked before any device work, and the loud failure of a
valid solver on a machine without a CUDA device (there is no CPU fallback). CPU only: none of these reach a GPU.

The reference panics on these programming errors (crates/qm-gpu/src/scf.rs:1083 grid checks); the boundary returns
KS_INVALID with a message instead (ks_last_error), and the mirror raises ValueError."""
import ctypes
import math

import numpy as np
import pytest


def _no_device():
    try:
        import torch
        return not torch.cuda.is_available()
    except Exception:
        return True


@pytest.mark.parametrize("n,h", [(4, 0.25), (1025, 0.25), (33, 0.0), (33, -0.1), (33, math.nan), (33, math.inf)])
def test_bad_grid_is_refused_before_any_device_work(ks, n, h):
    lib = ks.lib()
    opts = ks._Options(0, 0, 0, 0)
    assert not lib.ks_solver_create(n, h, ctypes.byref(opts))
    assert b"grid" in lib.ks_last_error(None)
    with pytest.raises(ValueError, match="grid"):
        ks.GpuSolver(n, h)


@pytest.mark.parametrize("opts", [(2, 0, 0), (-1, 0, 0), (0, -1, 0), (0, 0, 2)])
def test_bad_options_are_refused(ks, opts):
    lib = ks.lib()
    o = ks._Options(*opts, 0)
    assert not lib.ks_solver_create(33, 0.25, ctypes.byref(o))
    assert b"invalid options" in lib.ks_last_error(None)
    with pytest.raises(ValueError, match="invalid options"):
        ks.GpuSolver(33, 0.25, gram_mode=opts[0], n_extra=opts[1], init_mode=opts[2])


def test_null_handles_and_bad_sizes_return_invalid(ks):
    """Every entry point answers a null handle or an impossible size with a status, never a trap: KS_INVALID with a
    message, and KS_NO_STATE from the state getters (no converged state behind a null handle)."""
    lib = ks.lib()
    nuc = ks.nuclei_array([(0.0, 0.0, 0.0, 1)])
    out = np.zeros(64)
    p = out.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
    assert lib.ks_forces(None, nuc, 1, 0.5, p) == ks.KS_INVALID
    assert lib.ks_state_evals(None, p, p) == ks.KS_NO_STATE
    assert lib.ks_vjp(None, nuc, 1, 0.5, 1.0, p, p) == ks.KS_INVALID
    settings, stats = ks._Settings(), ks._Stats()
    no_abort = ctypes.cast(None, ks.ABORT_FN)
    assert lib.ks_solve(None, nuc, 1, 1, 0, ctypes.byref(settings), 0, no_abort, None, ctypes.byref(stats)) == ks.KS_INVALID
    assert lib.ks_apply_laplacian(3, 0.25, p, p) == ks.KS_INVALID
    assert lib.ks_gram(33, 0, p, 0, p, 0, p) == ks.KS_INVALID
    assert lib.ks_gram(33, 2, p, 0, p, 1, p) == ks.KS_INVALID  # the tensor-core form needs mt >= 1
    assert lib.ks_hpsi_device(None, 33, 0.25, 0, None, None, None) == ks.KS_INVALID
    assert lib.ks_rayleigh_ritz(4, p, p, 5, p, p, p) == ks.KS_INVALID  # nk > m
    # the guarded LOBPCG: head > checked, checked > k, and a tail tolerance below tol
    assert lib.ks_lobpcg_guarded(33, 0.25, p, 3, p, p, 1e-5, 1.5e-5, 3, 1e-3, 2, 10, 1, 0, p, None) == ks.KS_INVALID
    assert lib.ks_lobpcg_guarded(33, 0.25, p, 3, p, p, 1e-5, 1.5e-5, 2, 1e-3, 4, 10, 1, 0, p, None) == ks.KS_INVALID
    assert lib.ks_lobpcg_guarded(33, 0.25, p, 3, p, p, 1e-5, 1.5e-5, 2, 1e-6, 3, 10, 1, 0, p, None) == ks.KS_INVALID
    assert lib.ks_footprint_bytes(4, 1, 1, None, 6, 0) == -1
    assert lib.ks_footprint_bytes(33, -1, 1, None, 6, 0) == -1
    assert lib.ks_set_kernel_timing(None, 1) == ks.KS_INVALID
    assert lib.ks_kernel_times(None, None, 0) < 0
    assert lib.ks_state_import(None, 1, 0, 1, p, p, 0, p, p, p, p, p, 0, None, None) == ks.KS_INVALID
    assert lib.ks_test_poison_parked_density(None) == ks.KS_INVALID
    assert lib.ks_test_fail_readbacks(None, 0, 1) == ks.KS_INVALID
    assert lib.ks_last_error(None)  # a message for the last refusal


@pytest.mark.skipif(not _no_device(), reason="a CUDA device is present")
def test_no_device_fails_loudly(ks):
    """With valid arguments but no CUDA device the solver is not built: ks_solver_create returns NULL with the CUDA
    error, and the mirror raises Device. Nothing falls back to the CPU."""
    lib = ks.lib()
    opts = ks._Options(1, 3, 1, 0)
    assert not lib.ks_solver_create(33, 0.25, ctypes.byref(opts))
    assert lib.ks_last_error(None)
    with pytest.raises(ks.Device):
        ks.GpuSolver(33, 0.25, gram_mode=1, n_extra=3, init_mode=1)
    with pytest.raises(ks.Device):
        ks.apply_laplacian(33, 0.25, np.zeros(33 ** 3))
    # the wait-timeout status of the device-pointer calls needs a device too: a status, not a trap
    assert lib.ks_device_status(None) == ks.KS_DEVICE


def test_autotuner_arguments_are_refused_before_any_device_work(ks):
    """The stencil autotuner and its table refuse bad grids, vector counts and entries with KS_INVALID (ValueError)."""
    with pytest.raises(ValueError):
        ks.autotune_stencil(4, [8])        # grid below 5
    with pytest.raises(ValueError):
        ks.autotune_stencil(95, [0])       # vector counts are 1..64
    with pytest.raises(ValueError):
        ks.autotune_stencil(95, [65])
    with pytest.raises(ValueError):
        ks.set_stencil_tuning([(95, 8, 3, 5)])   # only H psi (1) and the sweep (2) are tuned
    with pytest.raises(ValueError):
        ks.set_stencil_tuning([(95, 8, 1, 96)])  # more chunks than planes
    with pytest.raises(ValueError):
        ks.set_stencil_tuning([(95, 0, 1, 5)])
