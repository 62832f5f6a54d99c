"""Extract the Gaussian basis-set data this engine needs from Psi4-format .gbs files.

The exponents and contraction coefficients are the published basis-set data
(Basis Set Exchange); hfscf ships them as .gbs files.  This script reads those
files and writes a compact JSON table per basis set for the elements used
here, keeping the two facts that change results: the header line
(``cartesian``/``spherical``, src/basis/hfscf_basis.cpp:53-60) and the shell
order inside each element block, with ``SP`` shells split into an S shell
followed by a P shell (src/basis/hfscf_basis.cpp:175-184).

Usage: python extract_gbs.py /path/to/basis/dir
"""
import json
import os
import sys

BASES = {
    "sto-3g": "sto-3g.gbs",
    "6-31g*": "6-31g_st_.gbs",
    "6-31g**": "6-31g_st__st_.gbs",
    "cc-pvdz": "cc-pvdz.gbs",
}
ELEMENTS = ("H", "C", "N", "O")
AM = {"S": 0, "P": 1, "D": 2, "F": 3, "G": 4}


def parse_gbs(path):
    with open(path) as f:
        lines = f.read().splitlines()
    header = lines[0].strip().replace(" ", "")
    coord = header if header in ("cartesian", "spherical") else "spherical"
    out = {}
    i = 1
    while i < len(lines):
        line = lines[i].strip()
        i += 1
        if not line or line.startswith("!") or line.startswith("*"):
            continue
        sym = line.split()[0]
        shells = []
        while i < len(lines):
            head = lines[i].split()
            i += 1
            if not head or head[0].startswith("*"):
                break
            kind, nprim = head[0].upper(), int(head[1])
            rows = [lines[i + k].replace("D", "E").split() for k in range(nprim)]
            i += nprim
            exps = [float(r[0]) for r in rows]
            if kind == "SP":
                shells.append({"L": 0, "exps": exps, "coefs": [float(r[1]) for r in rows]})
                shells.append({"L": 1, "exps": exps, "coefs": [float(r[2]) for r in rows]})
            else:
                shells.append({"L": AM[kind], "exps": exps, "coefs": [float(r[1]) for r in rows]})
        out[sym] = shells
    return coord, out


def main(src):
    here = os.path.dirname(os.path.abspath(__file__))
    for name, fname in BASES.items():
        coord, data = parse_gbs(os.path.join(src, fname))
        table = {"name": name, "coord_type": coord,
                 "elements": {e: data[e] for e in ELEMENTS if e in data}}
        dst = os.path.join(here, name.replace("*", "s") + ".json")
        with open(dst, "w") as f:
            json.dump(table, f, indent=1)
        print(dst, coord, {e: len(v) for e, v in table["elements"].items()})


if __name__ == "__main__":
    src = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("HFSCF_BASIS_DIR")
    if not src:
        sys.exit("usage: extract_gbs.py BASIS_DIR  (the reference's basis/ folder of .gbs files; "
                 "or set HFSCF_BASIS_DIR)")
    main(src)
