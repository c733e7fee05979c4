"""Generates oracle_h2o95.json: a full oracle SCF (f64 C++ restatement of crates/qm) of the bench
workload -- H2O on a 95^3 grid, h = 0.25 bohr, sigma = 0.5, 5 + 5 electrons, tol 1e-6 -- with its
energies, eigenvalues, forces and work counts (LOBPCG and Poisson iterations).

The record is test/bench infrastructure: the bench reports its GPU energy against it and scales the
timed CPU sample by its iteration counts. About 20 minutes on 6 host threads.

    python tests/golden/make_oracle_h2o95.py [threads]
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
nuc = [(0.0, 0.0, 0.0, 8), (1.43, 1.11, 0.0, 1), (-1.43, 1.11, 0.0, 1)]
t = time.time()
st, stats = O.scf(95, 0.25, nuc, 5, 5, sigma=0.5, tol=1e-6)
dt = time.time() - t
f = O.forces(st, nuc, 0.5)
eu, ed = st.evals()
rec = {"workload": "H2O 95^3 h=0.25 sigma=0.5 tol=1e-6", "wall_s": dt, "threads": threads, "stats": stats,
       "forces": f.tolist(), "evals_up": eu.tolist(), "evals_dn": ed.tolist()}
with open(os.path.join(HERE, "oracle_h2o95.json"), "w") as fh:
    json.dump(rec, fh, indent=1)
print(json.dumps(rec))
