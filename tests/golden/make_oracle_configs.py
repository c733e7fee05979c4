"""Generates full oracle SCF records (f64 C++ restatement of crates/qm) for three workloads beyond
the timed H2O one, so that the GPU solver's results on them are checked against an all-f64 run:

  nh3      NH3 on 96^3 at h = 0.22 (N at the origin, three H at 1.91 Bohr, 106.7 deg, seeded
           0.05 Bohr jitter), sigma = h = 0.22, 5 + 5 electrons, tol 1e-6
           -> oracle_nh3_96.json (energies, eigenvalues, forces)
  butane   n-butane, anti conformer (C-C 2.91, C-H 2.06 Bohr, seeded 0.02 Bohr jitter) on 128^3
           at h = 0.2, sigma = 0.5, 17 + 17 electrons (all-electron), tol 1e-6
           -> oracle_butane_128.json
  batch    the first eight molecules of the seeded batch workload on 48^3..64^3 grids (h = 0.25,
           sigma = 0.5, neutral, tol 1e-6) -> oracle_batch8.json (one record per molecule)

The geometries come from the package's workload builders (ks_drivers), so the GPU tests and the
records share one definition. Runs on the CPU only: nh3 takes about 20 minutes on 4 threads,
butane a few hours, batch a few minutes.

    python tests/golden/make_oracle_configs.py {nh3|butane|batch} [threads]
"""
import json
import os
import sys
import time

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.join(HERE, "..", "..")
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, os.path.join(ROOT, "atomic-sandbox_b200"))
import ks_oracle as O  # noqa: E402
import ks_drivers as D  # noqa: E402


def record(name, n, h, nuc, n_up, n_dn, sigma, tol=1e-6):
    t = time.time()
    st, stats = O.scf(n, h, nuc, n_up, n_dn, sigma=sigma, tol=tol)
    dt = time.time() - t
    if st is None:
        raise RuntimeError(f"{name}: oracle SCF failed: {stats}")
    f = O.forces(st, nuc, sigma)
    eu, ed = st.evals()
    return {"workload": f"{name} {n}^3 h={h} sigma={sigma} tol={tol}", "n": n, "h": h, "sigma": sigma,
            "n_up": n_up, "n_dn": n_dn, "nuclei": [list(a) for a in nuc], "wall_s": dt, "stats": stats,
            "forces": f.tolist(), "evals_up": eu.tolist(), "evals_dn": ed.tolist()}


def main():
    which = sys.argv[1]
    threads = int(sys.argv[2]) if len(sys.argv) > 2 else 4
    O.set_threads(threads)
    if which == "nh3":
        nuc = D.nh3(jitter=0.05, seed=0x5EED + 3)
        rec = record("NH3", 96, 0.22, nuc, 5, 5, 0.22)
        out = "oracle_nh3_96.json"
    elif which == "butane":
        nuc = D.butane_anti(jitter=0.02, seed=0x5EED + 2)
        rec = record("C4H10", 128, 0.2, nuc, 17, 17, 0.5)
        out = "oracle_butane_128.json"
    elif which == "batch":
        jobs = D.batch_workload(count=8, n_min=48, n_max=64)
        mols = []
        for j in jobs:
            ne = sum(int(a[3]) for a in j["nuclei"])
            r = record(j["name"], j["n"], j["h"], j["nuclei"], ne - ne // 2, ne // 2, 0.5)
            print(j["name"], j["n"], r["stats"]["total"], r["wall_s"], flush=True)
            mols.append(r)
        rec = {"workload": "batch: first 8 molecules of batch_workload(count=8, n_min=48, n_max=64)", "molecules": mols}
        out = "oracle_batch8.json"
    else:
        raise SystemExit(__doc__)
    rec["threads"] = threads
    with open(os.path.join(HERE, out), "w") as fh:
        json.dump(rec, fh, indent=1)
    print(json.dumps(rec)[:2000])


if __name__ == "__main__":
    main()
