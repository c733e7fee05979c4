"""Generates oracle_h3plus_49.json: a full oracle SCF (f64 C++ restatement of crates/qm) of the all-electron H3+ whose
0-2 pair is stretched to 1.6 r0 (r0 = 2.1174 Bohr, the equilateral bond; atom 2 moved along the 0-2 axis), the case of
the reference's gpu_fd_stretched_h3plus_converges_cold (crates/qm-gpu/src/scf.rs:2014-2043): 49^3, h = 0.25,
sigma = h, Fermi-Dirac at kT = 5e-3 Ha, tol 1e-6, 1 + 1 electrons, 4 extra levels per channel.

    python tests/golden/make_oracle_h3plus.py [threads]
"""
import json
import math
import os
import sys
import time

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "..", "..", "oracle"))
import ks_oracle as O  # noqa: E402


def h3plus_stretched(r0=2.1174, stretch=1.6):
    p0, p1 = (-0.5 * r0, -0.3, 0.0), (0.5 * r0, -0.3, 0.0)
    apex = (0.0, -0.3 + r0 * math.sqrt(3.0) / 2.0, 0.0)
    u = [(apex[k] - p0[k]) / r0 for k in range(3)]
    p2 = (p0[0] + stretch * r0 * u[0], p0[1] + stretch * r0 * u[1], 0.0)
    return [(*p0, 1), (*p1, 1), (*p2, 1)]


if __name__ == "__main__":
    threads = int(sys.argv[1]) if len(sys.argv) > 1 else 8
    O.set_threads(threads)
    nuc = h3plus_stretched()
    t = time.time()
    st, stats = O.scf(49, 0.25, nuc, 1, 1, sigma=0.25, tol=1e-6, kt=5e-3, n_extra=4)
    eu, ed = st.evals()
    fu, fd = st.occupations()
    out = {"grid": 49, "h": 0.25, "sigma": 0.25, "kt": 5e-3, "n_extra": 4, "tol": 1e-6, "nuclei": nuc, "n_up": 1, "n_dn": 1,
           "wall_s": time.time() - t, "threads": threads, "stats": stats, "evals_up": eu.tolist(), "evals_dn": ed.tolist(),
           "occ_up": fu.tolist(), "occ_dn": fd.tolist(), "forces": O.forces(st, nuc, 0.25).tolist()}
    with open(os.path.join(HERE, "oracle_h3plus_49.json"), "w") as fh:
        json.dump(out, fh, indent=1)
    print(json.dumps(out)[:1500])
