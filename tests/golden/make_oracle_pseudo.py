"""Generates oracle_pseudo.json: full oracle SCFs (f64 C++ restatement of crates/qm) under an ionic setup
(crates/qm/src/scf.rs:114-140): water with its O pseudised by the analytic species of tests/synthetic_species.py
(Z_v = 6, sigma_LR = 2h, short-range core, partial core, s and p Kleinman-Bylander projectors) and the two H
all-electron at sigma = 0.5, 8 valence electrons (4 + 4), 33^3 grid, h = 0.3, tol 1e-6, Aufbau. A second case
drops the partial core and the projectors (the local pseudopotential alone).

    python tests/golden/make_oracle_pseudo.py [threads]
"""
import json
import os
import sys
import time

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "..", "..", "oracle"))
sys.path.insert(0, os.path.join(HERE, ".."))
import ks_oracle as O  # noqa: E402
import synthetic_species as ss  # noqa: E402

threads = int(sys.argv[1]) if len(sys.argv) > 1 else 8
O.set_threads(threads)
n, h, sigma = 33, 0.3, 0.5
out = {"grid": n, "h": h, "sigma": sigma, "tol": 1e-6, "nuclei": ss.WATER, "n_up": 4, "n_dn": 4, "cases": {}}
for name, kw in (("full", {}), ("local", {"with_core": False, "with_projectors": False})):
    sp = [ss.oxygen_like(h, **kw)]
    t = time.time()
    st, stats = O.scf_ionic(n, h, ss.WATER, 4, 4, sp, sigma=sigma, tol=1e-6)
    eu, ed = st.evals()
    out["cases"][name] = {"species": kw, "wall_s": time.time() - t, "stats": stats, "evals_up": eu.tolist(), "evals_dn": ed.tolist(),
                          "forces": O.forces_ionic(st, ss.WATER, sigma, sp).tolist()}
with open(os.path.join(HERE, "oracle_pseudo.json"), "w") as fh:
    json.dump(out, fh, indent=1)
print(json.dumps(out)[:1500])
