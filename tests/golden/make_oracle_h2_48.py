"""Generates oracle_h2_48.json: a full oracle SCF (f64 C++ restatement of crates/qm) of the H2
workload -- two H 1.4 Bohr apart along x about the centre of a 48^3 grid, h = 0.25 Bohr, sigma =
0.5, 1 + 1 electrons, LSDA, tol 1e-6 -- with its energies, eigenvalues and forces.

    python tests/golden/make_oracle_h2_48.py [threads]
"""
import json
import os
import sys
import time

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "..", "..", "oracle"))
import ks_oracle as O  # noqa: E402

threads = int(sys.argv[1]) if len(sys.argv) > 1 else 6
O.set_threads(threads)
nuc = [(0.7, 0.0, 0.0, 1), (-0.7, 0.0, 0.0, 1)]
t = time.time()
st, stats = O.scf(48, 0.25, nuc, 1, 1, sigma=0.5, tol=1e-6)
dt = time.time() - t
f = O.forces(st, nuc, 0.5)
eu, ed = st.evals()
rec = {"workload": "H2 48^3 h=0.25 sigma=0.5 tol=1e-6", "wall_s": dt, "threads": threads, "stats": stats,
       "forces": f.tolist(), "evals_up": eu.tolist(), "evals_dn": ed.tolist()}
with open(os.path.join(HERE, "oracle_h2_48.json"), "w") as fh:
    json.dump(rec, fh, indent=1)
print(json.dumps(rec))
