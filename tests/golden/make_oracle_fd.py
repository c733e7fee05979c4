"""Generates oracle_fd.json: full oracle SCFs (f64 C++ restatement of crates/qm) under Fermi-Dirac
occupations at kT = 5e-3 Ha (crates/qm/src/occupations.rs) on a 33^3 grid, h = 0.25, sigma = h:
the B atom (3 + 2 electrons; its 2p triple is fractionally occupied, 2/3 and 1/3) and LiH (gapped,
F within ~1e-6 of the Aufbau energy), each with 4 extra levels per channel.

    python tests/golden/make_oracle_fd.py [threads]
"""
import json
import os
import sys
import time

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "..", "..", "oracle"))
import ks_oracle as O  # noqa: E402

threads = int(sys.argv[1]) if len(sys.argv) > 1 else 8
O.set_threads(threads)
cases = {"B": ([(0.0, 0.0, 0.0, 5)], 3, 2), "LiH": ([(1.5075, 0.0, 0.0, 3), (-1.5075, 0.0, 0.0, 1)], 2, 2)}
out = {"grid": 33, "h": 0.25, "sigma": 0.25, "kt": 5e-3, "n_extra": 4, "tol": 1e-6, "cases": {}}
for name, (nuc, nu, nd) in cases.items():
    t = time.time()
    st, stats = O.scf(33, 0.25, nuc, nu, nd, sigma=0.25, tol=1e-6, kt=5e-3, n_extra=4)
    eu, ed = st.evals()
    fu, fd = st.occupations()
    out["cases"][name] = {"nuclei": nuc, "n_up": nu, "n_dn": nd, "wall_s": time.time() - t, "stats": stats,
                          "evals_up": eu.tolist(), "evals_dn": ed.tolist(), "occ_up": fu.tolist(), "occ_dn": fd.tolist(),
                          "forces": O.forces(st, nuc, 0.25).tolist()}
with open(os.path.join(HERE, "oracle_fd.json"), "w") as fh:
    json.dump(out, fh, indent=1)
print(json.dumps(out)[:2000])
