"""Generates oracle_h2_81.json: a full oracle SCF (f64 C++ restatement of crates/qm) of the last geometry of the
reference's warm_displaced_steps_take_the_lowest_converged_witness chain (crates/qm-gpu/src/scf.rs:2057-2085):
all-electron H2 at R = 1.45 with the displacement (0.12, 0.03, 0.08), nuclei at (R/2 + d0, d1, d2) and
(-R/2, -d1, 0.3 d2), 81^3 x 0.25, sigma = h, Fermi-Dirac at kT = 5e-3 Ha, tol 1e-6, 1 + 1 electrons, 4 extra levels.

    python tests/golden/make_oracle_h2_81.py [threads]
"""
import json
import os
import sys
import time

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "..", "..", "oracle"))
import ks_oracle as O  # noqa: E402

# the chain of the reference's test: (R, displacement of atom 0; atom 1 gets (-d1, 0.3 d2))
PATH = [(1.4, (0.0, 0.0, 0.0)), (1.5, (0.1, -0.08, 0.05)), (1.35, (-0.05, 0.1, -0.1)), (1.45, (0.12, 0.03, 0.08))]


def geometry(r, d):
    return [(0.5 * r + d[0], d[1], d[2], 1), (-0.5 * r, -d[1], 0.3 * d[2], 1)]


if __name__ == "__main__":
    threads = int(sys.argv[1]) if len(sys.argv) > 1 else 8
    O.set_threads(threads)
    nuc = geometry(*PATH[3])
    t = time.time()
    st, stats = O.scf(81, 0.25, nuc, 1, 1, sigma=0.25, tol=1e-6, kt=5e-3, n_extra=4)
    eu, ed = st.evals()
    out = {"grid": 81, "h": 0.25, "sigma": 0.25, "kt": 5e-3, "n_extra": 4, "tol": 1e-6, "path": PATH, "nuclei": nuc,
           "n_up": 1, "n_dn": 1, "wall_s": time.time() - t, "threads": threads, "stats": stats, "evals_up": eu.tolist(),
           "evals_dn": ed.tolist(), "forces": O.forces(st, nuc, 0.25).tolist()}
    with open(os.path.join(HERE, "oracle_h2_81.json"), "w") as fh:
        json.dump(out, fh, indent=1)
    print(json.dumps(out)[:1500])
