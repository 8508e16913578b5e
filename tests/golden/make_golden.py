#!/usr/bin/env python3
"""Extract the reference's GFN-FF golden vectors into small committed fixtures.

Sources (curcuma test suite, read from a checkout given on the command line):
* ``test_cases/reference_data/*.ref.json``: geometry (bohr), per-term energies, Phase-2
  charges, CN, hybridisation, gradient norm for 15 molecules (xtb GFN-FF values that
  curcuma's test_gfnff_validation.cpp checks against, tolerances at :175-215), and the
  per-term parameter lists of the same files: bonds (atoms, r0 in Angstrom from the set-up
  formula (ra + rb) ff + shift, kbond = the exponent, prefactor = the force constant),
  angles (centre first, phi0 in degrees, fc), torsions (atoms, n, phi0, V).
* ``test_cases/molecules/larger/{complex,caffeine}.xyz`` with the CLI golden totals of
  ``test_cases/cli/gfnff/01_complex_gfnff_singlepoint/run_test.sh:19-30`` and
  ``test_cases/cli/gfnff_gpu/01_gfnff_gpu_singlepoint/run_test.sh:17-18``.

Output: one JSON per molecule in this directory with Z, xyz (Angstrom) and the
reference values.  Usage: ``python make_golden.py /path/to/curcuma`` (the checkout is a
required argument).
"""
import json
import re
import sys
from pathlib import Path

BOHR_A = 0.529177210903
EL = ["H", "He", "Li", "Be", "B", "C", "N", "O", "F", "Ne", "Na", "Mg", "Al", "Si", "P", "S", "Cl",
      "Ar", "K", "Ca", "Sc", "Ti", "V", "Cr", "Mn", "Fe", "Co", "Ni", "Cu", "Zn", "Ga", "Ge", "As",
      "Se", "Br", "Kr", "Rb", "Sr", "Y", "Zr", "Nb", "Mo", "Tc", "Ru", "Rh", "Pd", "Ag", "Cd", "In",
      "Sn", "Sb", "Te", "I", "Xe"]
ZOF = {s: i + 1 for i, s in enumerate(EL)}


def read_cli_value(path: Path, key: str) -> float:
    m = re.search(key + r'="([-0-9.]+)"', path.read_text())
    return float(m.group(1))


def main(root: str):
    root = Path(root)
    out = Path(__file__).resolve().parent
    refdir = root / "test_cases" / "reference_data"
    for f in sorted(refdir.glob("*.ref.json")):
        d = json.loads(f.read_text())
        at = d["molecule"]["atoms"]
        rec = {
            "name": f.name.replace(".ref.json", ""),
            "source": f"test_cases/reference_data/{f.name}",
            "Z": [ZOF[a["element"]] for a in at],
            "xyz_angstrom": [[a["x"] * BOHR_A, a["y"] * BOHR_A, a["z"] * BOHR_A] for a in at],
            "energy_components": d.get("energy_components", {}),
            "energy_charges": d.get("energy_charges", []),
            "gradient_norm": d.get("gradients", {}).get("norm"),
            "cn": d.get("topology", {}).get("coordination_numbers", []),
            "hybridization": d.get("topology", {}).get("hybridizations", []),
            "bonds": [[b["atoms"][0], b["atoms"][1], b["r0"], b["kbond"], b["prefactor"]] for b in d.get("bonds", [])],
            "angles": [[a["atoms"][0], a["atoms"][1], a["atoms"][2], a["phi0"], a["fc"]] for a in d.get("angles", [])],
            "torsions": [[*t["atoms"], t["n"], t["phi0"], t["V"]] for t in d.get("torsions", [])],
        }
        text = json.dumps({k: v for k, v in rec.items() if k not in ("bonds", "angles", "torsions")}, indent=1)
        # parameter lists one record per line
        lists = ",\n".join(f' "{k}": [' + ",".join(json.dumps(r) for r in rec[k]) + "]"
                            for k in ("bonds", "angles", "torsions"))
        (out / f"{rec['name']}.json").write_text(text[:-2] + ",\n" + lists + "\n}")
    cli = [("complex", "test_cases/cli/gfnff/01_complex_gfnff_singlepoint/run_test.sh",
            "REFERENCE_TOTAL_ENERGY", 5e-6),
           ("caffeine", "test_cases/cli/gfnff_gpu/01_gfnff_gpu_singlepoint/run_test.sh", None, 2e-5)]
    for name, script, key, tol in cli:
        lines = (root / "test_cases" / "molecules" / "larger" / f"{name}.xyz").read_text().split("\n")
        n = int(lines[0])
        rows = [l.split() for l in lines[2:2 + n]]
        text = (root / script).read_text()
        if key:
            total = read_cli_value(root / script, key)
        else:
            total = float(re.search(r"(-4\.672736999448)", text).group(1))
        rec = {"name": f"cli_{name}", "source": script, "Z": [ZOF[r[0]] for r in rows],
               "xyz_angstrom": [[float(v) for v in r[1:4]] for r in rows], "total_energy": total,
               "tolerance": tol}
        (out / f"cli_{name}.json").write_text(json.dumps(rec, indent=1))


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: make_golden.py /path/to/curcuma-checkout")
    main(sys.argv[1])
