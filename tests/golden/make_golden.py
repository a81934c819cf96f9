"""Generate tests/golden/rhf_energies.json from QUICK's own regression tests.

Reads every closed-shell RHF energy test ``test/ene_*_rhf_*.in`` of the QUICK
source tree (keyword line, charge, geometry in Angstrom) and the saved output
``test/saved/<name>.out`` (``TOTAL ENERGY`` and ``ELECTRONIC ENERGY`` lines,
printed with 9 decimals by ``src/getEnergy.f90:161-162``), plus the f-function
RHF energy of ``grad_nma_rhf_def2tzvp`` (a CPU-build golden).  Only basis sets
packaged under ``quick_b200/basis_data`` are kept.  The open-shell tests
``test/*_uhf_*.in`` give ``uhf_energies.json`` (their first TOTAL ENERGY).

Usage::

    python tests/golden/make_golden.py /path/to/QUICK
"""
import glob
import json
import os
import re
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
PACKAGED = {"STO-3G", "3-21G", "6-31G", "6-31G*", "6-31G**", "CC-PVDZ", "CC-PVTZ", "DEF2-TZVP"}


def parse_input(path):
    with open(path) as f:
        lines = f.read().splitlines()
    kw = lines[0].upper()
    basis = re.search(r"BASIS=(\S+)", kw).group(1)
    charge = re.search(r"CHARGE=(-?\d+)", kw)
    charge = int(charge.group(1)) if charge else 0
    mult = re.search(r"MULT=(\d+)", kw)
    mult = int(mult.group(1)) if mult else 1
    atoms = []
    for ln in lines[1:]:
        t = ln.split()
        if not t:
            if atoms:
                break
            continue
        if len(t) >= 4 and t[0].isalpha():
            atoms.append([t[0].capitalize(), float(t[1]), float(t[2]), float(t[3])])
        elif atoms:
            break
    return kw, basis, charge, mult, atoms


def parse_output(path):
    tot = el = None
    with open(path) as f:
        for ln in f:
            if "TOTAL ENERGY" in ln and "=" in ln:
                tot = float(ln.split("=")[1].split()[0])
            if "ELECTRONIC ENERGY" in ln and "=" in ln:
                el = float(ln.split("=")[1].split()[0])
    return tot, el


def main(root):
    cases = []
    names = sorted(glob.glob(os.path.join(root, "test", "ene_*_rhf_*.in")))
    names.append(os.path.join(root, "test", "grad_nma_rhf_def2tzvp.in"))
    for inp in names:
        name = os.path.basename(inp)[:-3]
        out = os.path.join(root, "test", "saved", name + ".out")
        if not os.path.exists(out):
            continue
        kw, basis, charge, mult, atoms = parse_input(inp)
        if basis not in PACKAGED or mult != 1 or "UHF" in kw or "DFT" in kw or "B3LYP" in kw:
            continue
        tot, el = parse_output(out)
        if tot is None:
            continue
        cases.append({"name": name, "basis": basis, "charge": charge, "atoms": atoms,
                      "total_energy": tot, "electronic_energy": el,
                      "source": f"test/{name}.in, test/saved/{name}.out"})
    with open(os.path.join(HERE, "rhf_energies.json"), "w") as f:
        json.dump(cases, f, indent=1)
    print(len(cases), "cases")
    # open-shell: the UHF energy at the input geometry (the first TOTAL ENERGY line of
    # the reference's only UHF regression output, a geometry optimisation)
    uhf = []
    for inp in sorted(glob.glob(os.path.join(root, "test", "*_uhf_*.in"))):
        name = os.path.basename(inp)[:-3]
        out = os.path.join(root, "test", "saved", name + ".out")
        if not os.path.exists(out):
            continue
        kw, basis, charge, mult, atoms = parse_input(inp)
        if basis not in PACKAGED or "DFT" in kw or "B3LYP" in kw:
            continue
        first = None
        with open(out) as f:
            for ln in f:
                if "TOTAL ENERGY" in ln and "=" in ln:
                    first = float(ln.split("=")[1].split()[0])
                    break
        if first is None:
            continue
        uhf.append({"name": name, "basis": basis, "charge": charge, "mult": mult, "atoms": atoms,
                    "total_energy": first, "source": f"test/{name}.in, test/saved/{name}.out (step 1)"})
    with open(os.path.join(HERE, "uhf_energies.json"), "w") as f:
        json.dump(uhf, f, indent=1)
    print(len(uhf), "UHF cases")


if __name__ == "__main__":
    if len(sys.argv) != 2:
        raise SystemExit("usage: make_golden.py <QUICK source tree>")
    main(sys.argv[1])
