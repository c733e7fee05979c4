"""Analytic pseudised species for the pseudopotential tests (test infrastructure).

The reference generates its tables with its own radial atom solver (crates/qm/src/radial, Troullier-Martins +
Kleinman-Bylander + band-limit filter), which is Rust and cannot run here. The GPU path and the oracle take any
tables in the same format (uniform spacing du = h/256, even functions, 0 beyond the radius), so the tests use smooth
analytic ones: Gaussians times the compact bump (1 - (d/rc)^2)^3, which vanishes with two derivatives at rc."""
import math
import os
import sys

import numpy as np

sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "atomic-sandbox_b200"))
from ks_b200 import Projector, Species  # noqa: E402  (plain dataclasses; loading them needs no GPU)


def bump_gauss(amp, width, rc):
    def f(d):
        d = np.asarray(d, dtype=np.float64)
        x = np.clip(d / rc, 0.0, 1.0)
        return np.where(d < rc, amp * np.exp(-d * d / (2 * width * width)) * (1 - x * x) ** 3, 0.0)
    return f


def table(f, du, radius):
    k = int(math.ceil(radius / du)) + 4
    return f(np.arange(k) * du)


def oxygen_like(h, with_core=True, with_projectors=True):
    """A six-valence-electron ion (Z = 8): sigma_LR = 2h, a repulsive short-range core, an optional partial core and
    an s (E_KB > 0) and a p (E_KB < 0) projector."""
    du = h / 256
    proj = []
    if with_projectors:
        proj = [Projector(0, 1.2, 1.6, table(bump_gauss(1.5, 0.40, 1.6), du, 1.6)),
                Projector(1, -0.6, 1.6, table(bump_gauss(2.0, 0.45, 1.6), du, 1.6))]
    return Species(z=8, z_v=6.0, sigma_lr=2 * h, du=du, v_sr=table(bump_gauss(3.0, 0.35, 1.5), du, 1.5), r_sr=1.5,
                   rho_pc=table(bump_gauss(0.8, 0.30, 1.2), du, 1.2) if with_core else None,
                   pc_radius=1.2 if with_core else 0.0, projectors=proj)


def bare_hydrogen(h, sigma):
    """Z = 1 with Z_v = 1, the all-electron width, no short range, no core, no projectors: V_loc is exactly the
    all-electron smeared nucleus."""
    return Species(z=1, z_v=1.0, sigma_lr=sigma, du=h / 256, v_sr=np.zeros(0), r_sr=0.0)


WATER = [(0.0, 0.0, 0.0, 8), (1.43, 1.11, 0.0, 1), (-1.43, 1.11, 0.0, 1)]
