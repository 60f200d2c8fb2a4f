"""Extracts the reference's own lattice fixture into tests/golden/.

FermiPhaseSpace ships one usable piece of data for this path: grid_10.xyz, the
positions file `makeSitesSystem grid_10 <folder> grid 10` writes (a 10-site
chain, spacing 1).  This script reads it from the reference tree and stores the
site count and positions as JSON, so that the generator test can compare the
engine's own `grid 10` output with it site by site without the reference tree.
Run it where the reference is mounted:  python tests/golden/make_reference_fixtures.py
"""
from __future__ import annotations

import json
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
REF = sys.argv[1] if len(sys.argv) > 1 else "/root/reference"


def read_xyz(path: str) -> dict:
    """The reference's xyz convention (src/FHLattice.cpp:646-683): line 1 = number
    of sites, line 2 = comment, then `name x y z` per site."""
    with open(path) as fh:
        lines = fh.read().split("\n")
    n = int(lines[0].split()[0])
    names, pos = [], []
    for ln in lines[2:2 + n]:
        f = ln.split()
        names.append(f[0])
        pos.append([float(f[1]), float(f[2]), float(f[3])])
    return {"n": n, "names": names, "positions": pos}


def main() -> None:
    src = os.path.join(REF, "grid_10.xyz")
    d = read_xyz(src)
    d["source"] = "grid_10.xyz of FermiPhaseSpace (generated by makeSitesSystem grid 10)"
    with open(os.path.join(HERE, "reference_grid_10.json"), "w") as fh:
        json.dump(d, fh, indent=1)
        fh.write("\n")


if __name__ == "__main__":
    main()
