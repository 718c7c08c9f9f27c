"""Extracts the per-state rows of the reference's own QSGW test outputs
(Samples/TestInstall/*/QPU, written by main_hqpe.sc.f90:167-169 with the
format (3f9.5,1x,i3,1x,10f8.3,f5.2,f10.5,3x,f10.5)) into
tests/golden/qpu_rows.npz, the known answers of the QP-energy step:

    columns  SEx SExcore SEc vxc  0  dSEnoZ eLDA 0 0 eHF  Z  FWHM  ReS(elda)

with dSEnoZ = SEx + SExcore + SEc - vxc, eHF = eLDA + SEx + SExcore - vxc and
ReS(elda) = SEx + SExcore + SEc (eV, main_hqpe.sc.f90:154-166).

The values are stored as the integers the fixed-point fields print (the ten
energy fields x 10^decimals, decimals = 3 for f8.3 or 2 for the older f7.2
layout, per case; Z x 100; FWHM and ReS(elda) x 100000), so the fixture holds
exactly what the files hold.  Run from the repository root with the reference checked out:

    python tests/golden/make_qpu_rows.py <reference root>
"""
import os
import sys

import numpy as np

CASES = ["si_gwsc", "gas_gwsc", "gas_gwsc666", "fe_gwsc", "nio_gwsc", "nio_gwsc444", "pdo_gwsc443",
         "yh3fcc_gwsc666", "cugase2_gwsc222"]
# The two layouts the reference has written: the current one and the one its
# comment keeps, (3f9.5,1x,i2,1x,10f7.2,f5.2,f10.5,3x,f10.5) (main_hqpe.sc.f90:166).
LAYOUTS = {
    "   SEx    SExcore   SEc     vxc     ---    dSEnoZ": dict(istate=(28, 31), start=32, width=8, dec=3),
    "  SEx   SExcore SEc    vxc   ---   dSEnoZ": dict(istate=(28, 30), start=31, width=7, dec=2),
}


def parse_row(line, lay):
    """One state row -> [state, ten fields x 10^dec, f5.2 x 100, FWHM x 1e5, ReS x 1e5] or None."""
    body = line.rstrip("\n")
    w, at = lay["width"], lay["start"]
    if len(body) < at + 10 * w + 5 + 10 + 3 + 10:
        return None
    try:
        [float(body[9 * i:9 * i + 9]) for i in range(3)]
        out = [int(body[lay["istate"][0]:lay["istate"][1]])]
        for i in range(10):
            out.append(int(round(float(body[at + w * i:at + w * (i + 1)]) * 10 ** lay["dec"])))
        at += 10 * w
        out.append(int(round(float(body[at:at + 5]) * 100)))
        out.append(int(round(float(body[at + 5:at + 15]) * 1e5)))
        out.append(int(round(float(body[at + 18:at + 28]) * 1e5)))
    except ValueError:
        return None
    return out


def read_qpu(path):
    with open(path) as fh:
        text = fh.readlines()
    lay = next((v for k, v in LAYOUTS.items() if any(k in t for t in text)), None)
    if lay is None:
        raise ValueError(f"{path}: not an hqpe QPU layout")
    rows = [r for r in (parse_row(t, lay) for t in text) if r is not None]
    return np.array(rows, dtype=np.int64), lay["dec"]


def main(ref_root):
    allrows, case_of, decs = [], [], []
    for i, c in enumerate(CASES):
        a, dec = read_qpu(os.path.join(ref_root, "Samples", "TestInstall", c, "QPU"))
        allrows.append(a)
        case_of.append(np.full(len(a), i, np.int32))
        decs.append(dec)
    rows = np.concatenate(allrows)
    out = os.path.join(os.path.dirname(os.path.abspath(__file__)), "qpu_rows.npz")
    np.savez_compressed(out, rows=rows.astype(np.int32), case=np.concatenate(case_of), cases=np.array(CASES),
                        decimals=np.array(decs, np.int32))
    print(out, rows.shape)


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python tests/golden/make_qpu_rows.py <reference root>")
    main(sys.argv[1])
