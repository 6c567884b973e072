"""Writes tests/golden/argon_lattice.json, the known answer of MDIR's
test/Driver/argon.test:9-14: the 864-atom argon lattice of
examples/argon/argon.{toml,pdb} (box 34.7786 Å, LJ sigma 3.4 Å and epsilon
0.238465 kcal/mol, switched from 7.5 to 8.5 Å, no charges), whose potential
energy at step 0 argon.test checks as -1304.88... kcal/mol, and
examples/argon/argon.mlir states as -5459.64 kJ/mol.

Run in a checkout that has the reference next to it:

    python tests/golden/make_argon_lattice.py /path/to/mdir

The fixture holds the positions (nm, as the PDB prints them), the box (nm),
the LJ parameters (nm, kJ/mol), the switch and cutoff (nm) and the expected
potential in kcal/mol with the digits argon.test checks."""

import json
import re
import sys
from pathlib import Path

KJ_PER_KCAL = 4.184


def main(ref):
    ex = Path(ref) / "examples" / "argon"
    toml = (ex / "argon.toml").read_text()

    def value(key):
        return float(re.search(rf"^\s*{key}\s*=\s*([-0-9.eE]+)", toml, flags=re.M).group(1))

    box = [float(v) for v in re.search(r"box\s*=\s*\[([^\]]*)\]", toml).group(1).split(",")]
    positions = []
    for line in (ex / "argon.pdb").read_text().splitlines():
        if line.startswith(("ATOM", "HETATM")):
            positions.append([float(line[30:38]) / 10.0, float(line[38:46]) / 10.0, float(line[46:54]) / 10.0])
    out = {
        "source": "examples/argon/argon.{toml,pdb}; expected: test/Driver/argon.test:9-14",
        "positions_nm": positions,
        "box_nm": [b / 10.0 for b in box],
        "sigma_nm": value("sigma") / 10.0,
        "epsilon_kj_mol": value("epsilon") * KJ_PER_KCAL,
        "switch_nm": value("switch_distance") / 10.0,
        "cutoff_nm": value("cutoff") / 10.0,
        "potential_kcal_mol_prefix": "-1304.88",
        "potential_kj_mol_argon_mlir": -5459.64,
    }
    dest = Path(__file__).resolve().parent / "argon_lattice.json"
    dest.write_text(json.dumps(out, indent=0) + "\n")
    print(f"{dest}: {len(positions)} atoms")


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: make_argon_lattice.py <path of an MDIR checkout>")
    main(sys.argv[1])
