"""Extracts the e-Ar and Ar+-Ar cross-section tables of the reference's
Pegasus gas data into pic_b200/data/ar_pegasus.json.

Input: MCC_jw/gas/pegasus/Ar/{ElectronAr.txt, Ar(+)Ar.txt, 1800xx} of the
PIC-IFE_GEC project (weqwoueu/pic-).  Each reaction file holds, after '#'
comment lines: index, equation, threshold (eV), number of species, species
codes, number changes, reaction type, number of points, then (E [eV],
sigma [cm^2]) pairs (format read by LoadReactionOnePegasus,
mc/ReactionOnePegasus.f90:92-110).  The JSON keeps the numbers as read; the
table builder in pic_b200/mcc_tables.py does the unit conversion.

Usage: python pic_b200/data/make_xsec.py /path/to/PIC-IFE_GEC
"""
from __future__ import annotations

import json
import os
import sys


def _data_lines(path):
    with open(path) as f:
        for line in f:
            s = line.strip()
            if not s or s.startswith("#"):
                continue
            yield s


def read_reaction(path):
    it = _data_lines(path)
    index = int(next(it).split()[0])
    name = next(it).split()[0]
    threshold = float(next(it).split()[0])
    nspecy = int(next(it).split()[0])
    species = [int(v) for v in next(it).split()[:nspecy]]
    change = [int(v) for v in next(it).split()[:nspecy]]
    rtype = int(next(it).split()[0])
    npts = int(next(it).split()[0])
    table = []
    for _ in range(npts):
        e, s = next(it).split()[:2]
        table.append([float(e), float(s)])
    return {"index": index, "name": name, "threshold": threshold, "species": species,
            "number_change": change, "pegasus_type": rtype, "table": table}


def read_bundle(gasdir, listfile):
    with open(os.path.join(gasdir, listfile)) as f:
        lines = [l.split() for l in f if l.strip()]
    model, nreact = int(lines[0][0]), int(lines[0][1])
    reactions = [read_reaction(os.path.join(gasdir, row[0])) for row in lines[1:1 + nreact]]
    return {"model": model, "reactions": reactions}


def main(root):
    gasdir = os.path.join(root, "MCC_jw", "gas", "pegasus", "Ar")
    out = {
        "source": "weqwoueu/pic- PIC-IFE_GEC/MCC_jw/gas/pegasus/Ar",
        "electron": read_bundle(gasdir, "ElectronAr.txt"),
        "ion": read_bundle(gasdir, "Ar(+)Ar.txt"),
    }
    dst = os.path.join(os.path.dirname(os.path.abspath(__file__)), "ar_pegasus.json")
    with open(dst, "w") as f:
        json.dump(out, f, indent=1)
    print(dst)


if __name__ == "__main__":
    # the PIC-IFE_GEC project directory of a checkout of weqwoueu/pic-
    _root = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("PIC_REFERENCE_ROOT")
    if not _root:
        sys.exit(f"usage: python {os.path.basename(__file__)} <path to PIC-IFE_GEC> "
                 "(or set PIC_REFERENCE_ROOT)")
    main(_root)
