#!/usr/bin/env python3
"""Extract the reference's GFN-FF + ALPB golden totals into a small committed fixture.

Sources (curcuma test suite, read from a checkout given on the command line):
* ``test_cases/sqm_reference/reference_data/gfnff_alpb_xtb.ref.json``: total energies of
  ``xtb 6.7.1 --gfnff --alpb SOLVENT`` (gsolv reference state) for 7 molecules in 4
  solvents, which curcuma's ``validate_gfnff_solvation.py`` checks at 1e-7 Eh
  (``test_cases/sqm_reference/CMakeLists.txt:335-351``);
* ``test_cases/sqm_reference/molecules/<mol>.xyz``: the geometries (Angstrom).

Output: ``alpb/gfnff_alpb_xtb.json`` beside this script with, per molecule, Z, xyz and the
total per solvent.  Usage: ``python make_alpb_golden.py /path/to/curcuma``.
"""
import json
import sys
from pathlib import Path

ZOF = {"H": 1, "C": 6, "N": 7, "O": 8}
MOLS = ["H2O", "NH3", "CH4", "HCN", "C6H6", "acetic_acid_dimer", "caffeine"]
SOLVENTS = ["water", "dmso", "acetone", "chloroform"]


def main(root: str):
    root = Path(root) / "test_cases" / "sqm_reference"
    ref = json.loads((root / "reference_data" / "gfnff_alpb_xtb.ref.json").read_text())
    out = {"source": "test_cases/sqm_reference/reference_data/gfnff_alpb_xtb.ref.json",
           "generator": ref["_generator"], "tolerance": 1e-7, "molecules": {}}
    for mol in MOLS:
        lines = (root / "molecules" / f"{mol}.xyz").read_text().split("\n")
        n = int(lines[0])
        rows = [l.split() for l in lines[2:2 + n]]
        out["molecules"][mol] = {"Z": [ZOF[r[0]] for r in rows],
                                 "xyz_angstrom": [[float(v) for v in r[1:4]] for r in rows],
                                 "total": {s: ref["data"][f"{mol}_{s}"] for s in SOLVENTS}}
    dst = Path(__file__).resolve().parent / "alpb"
    dst.mkdir(exist_ok=True)
    (dst / "gfnff_alpb_xtb.json").write_text(json.dumps(out, indent=1))


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: make_alpb_golden.py /path/to/curcuma-checkout")
    main(sys.argv[1])
