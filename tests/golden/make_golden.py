"""Generates the golden fixtures of tests/golden from the reference's own
committed outputs (weqwoueu/pic-, PIC-IFE_GEC):

  physics_parameter.json  <- OUTPUT/physics_parameter.inp:38-70 (reference
                             scales at n_ref = 1e21 m^-3, T_ref = 1 eV, and the
                             1-amu ion mass in units of m_e)
  norm_error.json         <- Norm_Error_{0064,0128,0256}.txt (IFE L2/H1 errors)
  philox4x32_10_kat.json  <- known-answer vectors of Philox4x32-10 published
                             with the Random123 library (Salmon et al., SC'11)
  pegasus_ar_digest.json  <- MCC_jw/gas/pegasus/Ar: per reaction of the e-Ar and
                             Ar+-Ar bundles, the header fields and the raw
                             (E, sigma) points summarised (count, sums, first and
                             last rows) and the SHA-256 of the file, read with a
                             token stream of its own (not the extractor's parser)

Usage: python tests/golden/make_golden.py [/path/to/PIC-IFE_GEC]
"""
import json
import os
import re
import sys

HERE = os.path.dirname(os.path.abspath(__file__))


def numbers(line):
    return [float(v.replace("D", "E")) for v in re.findall(r"[-+]?\d+\.\d*(?:[EeDd][-+]?\d+)?", line)]


def _tokens(path):
    """Whitespace tokens of a Pegasus file after its '#' comment lines, the
    order LoadReactionOnePegasus (mc/ReactionOnePegasus.f90:92-110) reads."""
    out = []
    for line in open(path):
        if line.lstrip().startswith("#"):
            continue
        out.extend(line.split())
    return out


def pegasus_digest(root):
    import hashlib
    gas = os.path.join(root, "MCC_jw", "gas", "pegasus", "Ar")
    out = {}
    for bundle in ("ElectronAr.txt", "Ar(+)Ar.txt"):
        tok = open(os.path.join(gas, bundle)).read().split()
        model, nr = int(tok[0]), int(tok[1])
        files = [tok[2 + 3 * k] for k in range(nr)]
        reactions = []
        for f in files:
            path = os.path.join(gas, f)
            t = _tokens(path)
            # Index, Name, Threshold, NSpecy, species(NSpecy), changes(NSpecy), type, n, pairs
            ns = int(t[3])
            rtype = int(t[4 + 2 * ns])
            n = int(t[5 + 2 * ns])
            vals = [float(v) for v in t[6 + 2 * ns:6 + 2 * ns + 2 * n]]
            e, sg = vals[0::2], vals[1::2]
            reactions.append({"file": f, "index": int(t[0]), "threshold": float(t[2]), "type": rtype,
                              "n": n, "sum_e": sum(e), "sum_sigma_cm2": sum(sg), "first": [e[0], sg[0]],
                              "last": [e[-1], sg[-1]],
                              "sha256": hashlib.sha256(open(path, "rb").read()).hexdigest()})
        out[bundle] = {"model": model, "reactions": reactions}
    json.dump(out, open(os.path.join(HERE, "pegasus_ar_digest.json"), "w"), indent=1)


def main(root):
    txt = open(os.path.join(root, "OUTPUT", "physics_parameter.inp")).read().splitlines()
    def after(label):
        for l in txt:
            if l.strip().startswith(label):
                return numbers(l)[-1]
        raise KeyError(label)
    phys = {
        "n_ref": after("density ref"),
        "T_ref_eV": after("temperature ref") / 11605.0,
        "L_ref": after("length ref"),
        "time_ref": after("time ref"),
        "v_ref": after("velocity ref"),
        "Phi_ref": after("potential ref"),
    }
    masses = [numbers(l)[-1] for l in txt if l.strip().startswith("mass:")]
    phys["ion_mass_over_me"] = [m for m in masses if m > 100.0][0]
    phys["ion_mass_kg"] = [m for m in masses if 1e-28 < m < 1e-25][0]
    json.dump(phys, open(os.path.join(HERE, "physics_parameter.json"), "w"), indent=1)
    ne = {}
    for n in (64, 128, 256):
        lines = open(os.path.join(root, "Norm_Error_%04d.txt" % n)).read().splitlines()
        l2, h1 = numbers(lines[2])[:2]
        ne[str(n)] = {"L2": l2, "H1": h1}
    json.dump(ne, open(os.path.join(HERE, "norm_error.json"), "w"), indent=1)
    kat = [
        {"ctr": [0, 0, 0, 0], "key": [0, 0],
         "out": [0x6627e8d5, 0xe169c58d, 0xbc57ac4c, 0x9b00dbd8]},
        {"ctr": [0xffffffff] * 4, "key": [0xffffffff] * 2,
         "out": [0x408f276d, 0x41c83b0e, 0xa20bc7c6, 0x6d5451fd]},
        {"ctr": [0x243f6a88, 0x85a308d3, 0x13198a2e, 0x03707344], "key": [0xa4093822, 0x299f31d0],
         "out": [0xd16cfe09, 0x94fdcceb, 0x5001e420, 0x24126ea1]},
    ]
    json.dump(kat, open(os.path.join(HERE, "philox4x32_10_kat.json"), "w"), indent=1)
    pegasus_digest(root)


if __name__ == "__main__":
    # the PIC-IFE_GEC project directory of a checkout of weqwoueu/pic-
    _root = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("PIC_REFERENCE_ROOT")
    if not _root:
        sys.exit(f"usage: python {os.path.basename(__file__)} <path to PIC-IFE_GEC> "
                 "(or set PIC_REFERENCE_ROOT)")
    main(_root)
