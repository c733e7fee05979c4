"""Regenerates the golden fixtures of this directory from the reference's own sources (read as
text; nothing of the reference is executed). Run from the repository root, naming the checkout of the
reference (ItsKodas/atomic-sandbox) to read:

    python tests/golden/make_pins.py PATH_TO_REFERENCE_CHECKOUT

- reference_pins.json: the reference's known answers for the Kohn-Sham path -- the bitwise-pinned
  33^3 Aufbau energies and forces of H2 and LiH (crates/qm/src/scf.rs:1276-1279, geometry :1304-1305),
  the published 49^3 CPU energies and forces (crates/validate/references.md:156-160, :180-188, geometries
  crates/validate/tests/gpu_vs_cpu.rs:76-92), the PW92 values (crates/qm/src/xc.rs:236-243) and the
  analytic limits the reference's tests assert.
- rr_i1_a.txt / rr_i1_b.txt: the 23 x 23 Rayleigh-Ritz matrices of crates/qm-gpu/testdata (theta_0 =
  -0.8686699, crates/qm-gpu/src/eigen.rs:1188-1201).
"""
import json
import os
import re
import struct
import sys

HERE = os.path.dirname(os.path.abspath(__file__))


def bits(hexstr):
    return struct.unpack("<d", struct.pack("<Q", int(hexstr, 16)))[0]


def main(ref):
    scf = open(os.path.join(ref, "crates/qm/src/scf.rs")).read()
    pins = {}
    for name in ("BASE_H2_E", "BASE_H2_FX", "BASE_LIH_E", "BASE_LIH_FX"):
        m = re.search(r"const %s: u64 = (0x[0-9a-f]+);" % name, scf)
        pins[name] = {"bits": m.group(1), "value": bits(m.group(1))}
    refs = open(os.path.join(ref, "crates/validate/references.md")).read()
    energies = {}
    for label, key in (("| H |", "H"), ("| He |", "He"), ("| H₂ R = 1.4 |", "H2"), ("| LiH R = 3.0", "LiH"), ("| H₂O (`h2o` preset) |", "H2O")):
        line = next(l for l in refs.splitlines() if l.startswith(label))
        energies[key] = float(line.split("|")[2].replace("−", "-").strip())
    forces = {}
    for l in refs.splitlines():
        m = re.match(r"\| H₂ R = ([0-9.]+) \| 0 \(x\) \| ([^|]+) \| ([^|]+) \|", l)
        if m:
            forces["H2_R%s_F0x" % m.group(1)] = float(m.group(3).replace("−", "-").strip())
        if l.startswith("| H₂O | O (y) |"):
            forces["H2O_O_y"] = float(l.split("|")[4].replace("−", "-").strip())
        if l.startswith("| H₂O | H (x, y) |"):
            xs = l.split("|")[4].replace("−", "-").split(",")
            forces["H2O_H_x"], forces["H2O_H_y"] = float(xs[0]), float(xs[1])
    out = {
        "pins_33": {
            "grid": {"n": 33, "h": 0.25}, "settings": {"sigma": 0.25, "tol": 1e-6, "occupations": "aufbau"},
            "H2": {"nuclei": [[0.7, 0.0, 0.0, 1], [-0.7, 0.0, 0.0, 1]], "n_up": 1, "n_dn": 1,
                   "energy": pins["BASE_H2_E"]["value"], "energy_bits": pins["BASE_H2_E"]["bits"],
                   "force_x0": pins["BASE_H2_FX"]["value"], "force_x0_bits": pins["BASE_H2_FX"]["bits"], "steps": 10},
            "LiH": {"nuclei": [[-0.8, 0.1, 0.0, 3], [2.2, 0.0, 0.0, 1]], "n_up": 2, "n_dn": 2,
                    "energy": pins["BASE_LIH_E"]["value"], "energy_bits": pins["BASE_LIH_E"]["bits"],
                    "force_x0": pins["BASE_LIH_FX"]["value"], "force_x0_bits": pins["BASE_LIH_FX"]["bits"], "steps": 13},
            "source": "crates/qm/src/scf.rs:1276-1305 (none_policy_is_bitwise_today)",
        },
        "cpu_49": {
            "grid": {"n": 49, "h": 0.25}, "settings": {"sigma": 0.25, "tol": 1e-6, "occupations": "aufbau"},
            "systems": {
                "H": {"nuclei": [[0.0, 0.0, 0.0, 1]], "n_up": 1, "n_dn": 0},
                "He": {"nuclei": [[0.0, 0.0, 0.0, 2]], "n_up": 1, "n_dn": 1},
                "H2": {"nuclei": [[0.7, 0.0, 0.0, 1], [-0.7, 0.0, 0.0, 1]], "n_up": 1, "n_dn": 1},
                "LiH": {"nuclei": [[-0.8, 0.0, 0.0, 3], [2.2, 0.0, 0.0, 1]], "n_up": 2, "n_dn": 2},
                "H2O": {"nuclei": [[0.0, 0.0, 0.0, 8], [1.43, 1.11, 0.0, 1], [-1.43, 1.11, 0.0, 1]], "n_up": 5, "n_dn": 5},
            },
            "energy": energies, "forces": forces,
            "source": "crates/validate/references.md:156-188; geometries crates/validate/tests/gpu_vs_cpu.rs:76-92",
        },
        "pw92": {"eps_c_rs2": -0.044760, "eps_c_rs10": -0.018572, "tol": 2e-5, "source": "crates/qm/src/xc.rs:236-243"},
        "analytic": {
            "oscillator_49": {"levels": [1.5, 2.5, 2.5, 2.5], "tol": 1e-4, "source": "crates/qm/src/eigen.rs:394-404"},
            "gaussian_poisson_49": {"max_err": 1e-4, "hartree": 1.0 / (2.0 * 0.5 * 3.141592653589793 ** 0.5), "hartree_tol": 1e-4,
                                    "source": "crates/qm/src/poisson.rs:291-315"},
            "coulomb_far_49": {"z": 6, "sigma": 0.2, "far_index": [44, 24, 24], "far_value": -1.2, "tol": 1e-12,
                               "source": "crates/qm/src/nuclear.rs:500-509"},
        },
    }
    with open(os.path.join(HERE, "reference_pins.json"), "w") as f:
        json.dump(out, f, indent=1)
    for name in ("rr_i1_a.txt", "rr_i1_b.txt"):
        src = open(os.path.join(ref, "crates/qm-gpu/testdata", name)).read()
        with open(os.path.join(HERE, name), "w") as f:
            f.write(src)
    print("wrote", os.listdir(HERE))


if __name__ == "__main__":
    if len(sys.argv) != 2:
        raise SystemExit("usage: python tests/golden/make_pins.py PATH_TO_REFERENCE_CHECKOUT")
    main(sys.argv[1])
