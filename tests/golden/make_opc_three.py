"""Writes tests/golden/opc_three.json, the known-answer case of MDIR's
test/Driver/pme.test:21-29: three four-site OPC waters in a 4 nm cube, cutoff
0.9 nm, beta 3.47045919371208278 nm^-1, PME on 64^3 points with splines of
order 8.

Run in a checkout that has the reference next to it:

    python tests/golden/make_opc_three.py /path/to/mdir

It reads test/Driver/Inputs/opc/three.{prmtop,inpcrd}, places each extra
point on the H-O-H bisector at the length of its bond (the placement that
test/Driver/Inputs/ewald_reference.py uses), and runs that script itself to
record the expected terms.  The fixture holds positions (nm), charges (e),
the box, the residue of each atom (pairs within a residue are excluded) and
the expected terms in kcal/mol as pme.test prints them."""

import json
import math
import subprocess
import sys
from pathlib import Path


def read_prmtop(path):
    sections, flag, width = {}, None, None
    for line in open(path):
        if line.startswith("%FLAG"):
            flag = line.split()[1]
            sections[flag] = []
        elif line.startswith("%FORMAT"):
            fmt = line[line.index("(") + 1: line.index(")")]
            digits = ""
            for c in fmt:
                if c.isalpha():
                    digits = ""
                elif c.isdigit():
                    digits += c
                elif c == ".":
                    break
            width = int(digits)
        elif line.startswith("%"):
            continue
        elif flag:
            text = line.rstrip("\n")
            for i in range(0, len(text), width):
                field = text[i: i + width].strip()
                if field:
                    sections[flag].append(field)
    return sections


def main():
    if len(sys.argv) != 2:
        sys.exit("usage: make_opc_three.py <path of an MDIR checkout>")
    root = Path(sys.argv[1])
    inputs = root / "test/Driver/Inputs"
    top = read_prmtop(inputs / "opc/three.prmtop")
    charges = [float(v) / 18.2223 for v in top["CHARGE"]]
    n = len(charges)
    types = top["AMBER_ATOM_TYPE"]
    starts = [int(s) - 1 for s in top["RESIDUE_POINTER"]] + [n]
    lines = open(inputs / "opc/three.inpcrd").read().splitlines()
    numbers = []
    for line in lines[2:]:
        numbers += [float(line[i: i + 12]) for i in range(0, len(line), 12) if line[i: i + 12].strip()]
    x = [[0.1 * numbers[3 * i + k] for k in range(3)] for i in range(n)]
    box = [0.1 * numbers[3 * n + k] for k in range(3)]
    bonds = [int(v) for v in top["BONDS_WITHOUT_HYDROGEN"]]
    lengths = [0.1 * float(v) for v in top["BOND_EQUIL_VALUE"]]
    for b in range(0, len(bonds), 3):
        i, j, t = bonds[b] // 3, bonds[b + 1] // 3, bonds[b + 2] - 1
        site, owner = (i, j) if types[i] == "EP" else (j, i)
        if types[site] != "EP":
            continue
        units = []
        for a in (owner + 1, owner + 2):
            d = [x[a][k] - x[owner][k] for k in range(3)]
            norm = math.sqrt(sum(c * c for c in d))
            units.append([c / norm for c in d])
        s = [units[0][k] + units[1][k] for k in range(3)]
        norm = math.sqrt(sum(c * c for c in s))
        x[site] = [x[owner][k] + lengths[t] * s[k] / norm for k in range(3)]
    residue = [0] * n
    for r in range(len(starts) - 1):
        for i in range(starts[r], starts[r + 1]):
            residue[i] = r
    out = subprocess.run(
        [sys.executable, str(inputs / "ewald_reference.py"), str(inputs / "opc/three.prmtop"),
         str(inputs / "opc/three.inpcrd"), "9.0", "3.47045919371208278"],
        check=True, capture_output=True, text=True).stdout
    terms = {line.split()[0]: float(line.split()[1]) for line in out.splitlines() if line.strip()}
    fixture = {
        "source": "MDIR test/Driver/pme.test:21-29, test/Driver/Inputs/opc/three.{prmtop,inpcrd}; "
                  "expected terms printed by test/Driver/Inputs/ewald_reference.py",
        "positions_nm": x,
        "charges_e": charges,
        "box_nm": box,
        "residue": residue,
        "cutoff_nm": 0.9,
        "beta_per_nm": 3.47045919371208278,
        "pme_grid": [64, 64, 64],
        "pme_order": 8,
        "expected_kcal": terms,
        "pme_test_printed_kcal": {"direct": -14.357298, "excluded": 535.126068,
                                  "reciprocal": 4.697241, "self": -539.792827},
    }
    path = Path(__file__).with_name("opc_three.json")
    path.write_text(json.dumps(fixture, indent=1) + "\n")
    print(f"wrote {path}: {terms}")


if __name__ == "__main__":
    main()
