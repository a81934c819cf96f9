"""Extract the Gaussian-format basis-set files shipped with QUICK into compact JSON.

The reference reads ``basis/<NAME>.BAS`` at run time (``src/basis.f90:65-120``:
an element header ``"<Sym>  0"``, then shell headers ``"<S|P|SP|D|F> nprim 1.00"``
each followed by ``nprim`` rows of ``exponent coeff [coeff_p]``, then ``****``).
These files are Basis Set Exchange data.  This script turns the subset of basis
sets and elements this package needs into ``quick_b200/basis_data/<NAME>.json``,
so that the package never reads the reference tree at run time.

Usage (in a checkout that has the reference mounted)::

    python tests/golden/extract_basis.py /path/to/QUICK/basis
"""
import json
import os
import sys

# keyword (as written in QUICK inputs, cf. basis/basis_link) -> file name
BASIS_FILES = {
    "STO-3G": "STO-3G.BAS",
    "3-21G": "3-21G.BAS",
    "6-31G": "6-31G.BAS",
    "6-31G*": "6-31GD.BAS",
    "6-31G**": "6-31GDP.BAS",
    "CC-PVDZ": "CC-PVDZ.BAS",
    "CC-PVTZ": "CC-PVTZ.BAS",
    "DEF2-TZVP": "DEF2-TZVP.BAS",
}

ELEMENTS = ["H", "He", "Li", "Be", "B", "C", "N", "O", "F", "Ne", "Na", "Mg",
            "Al", "Si", "P", "S", "Cl", "Ar", "K", "Ca", "Br", "I"]


def _num(tok):
    return float(tok.replace("D", "E").replace("d", "e"))


def parse_bas(path):
    """Return {element: [[shell_type, [[exp, c(, cp)], ...]], ...]} for one file."""
    out = {}
    with open(path) as f:
        lines = [ln.rstrip("\n") for ln in f]
    i = 0
    n = len(lines)
    while i < n:
        tok = lines[i].split()
        i += 1
        if len(tok) >= 2 and tok[1] == "0" and tok[0].isalpha() and len(tok[0]) <= 2:
            sym = tok[0].capitalize()
            shells = []
            while i < n:
                t = lines[i].split()
                if len(t) < 2 or t[0].upper() not in ("S", "P", "SP", "D", "F", "G"):
                    break
                kind = t[0].upper()
                nprim = int(t[1])
                i += 1
                prims = []
                for _ in range(nprim):
                    prims.append([_num(x) for x in lines[i].split()])
                    i += 1
                shells.append([kind, prims])
            out[sym] = shells
    return out


def main(src_dir, dst_dir):
    for key, fname in BASIS_FILES.items():
        data = parse_bas(os.path.join(src_dir, fname))
        keep = {el: data[el] for el in ELEMENTS if el in data}
        name = key.replace("*", "s")
        with open(os.path.join(dst_dir, name + ".json"), "w") as f:
            json.dump({"name": key, "source_file": fname, "elements": keep}, f,
                      separators=(",", ":"))
        print(key, len(keep), "elements")


if __name__ == "__main__":
    if len(sys.argv) != 2:
        raise SystemExit("usage: extract_basis.py <QUICK source tree>/basis")
    here = os.path.dirname(os.path.abspath(__file__))
    main(sys.argv[1], os.path.join(os.path.dirname(os.path.dirname(here)), "quick_b200", "basis_data"))
