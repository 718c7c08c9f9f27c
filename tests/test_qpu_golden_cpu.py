"""The QP-energy step pinned against the reference's own outputs: every
state row of Samples/TestInstall/*/QPU (extracted by
tests/golden/make_qpu_rows.py) prints the inputs SEx, SExcore, SEc, vxc, eLDA
and the results dSEnoZ = eQP - eLDA, eHF and ReS(elda) of
main_hqpe.sc.f90:154-169.  The oracle's qp_energies must reproduce them to the
rounding of the printed fields."""
import os

import numpy as np

from oracle import hqpe

HERE = os.path.dirname(os.path.abspath(__file__))


def load_rows():
    """Rows with SEx != 0 (the reference prints 0 for dSEnoZ and eHF otherwise) as eV floats:
    dict of arrays SEx, SExcore, SEc, vxc, dSEnoZ, eLDA, eHF, Z, ReS and the field half-step."""
    d = np.load(os.path.join(HERE, "golden", "qpu_rows.npz"))
    r, case = d["rows"].astype(np.float64), d["case"]
    step = 10.0 ** -d["decimals"][case].astype(np.float64)
    f = lambda i: r[:, i] * step                      # noqa: E731  the ten energy fields
    out = dict(SEx=f(1), SExcore=f(2), SEc=f(3), vxc=f(4), dSEnoZ=f(6), eLDA=f(7), eHF=f(10),
               Z=r[:, 11] / 100.0, ReS=r[:, 13] / 1e5, half=0.5 * step, case=case, cases=d["cases"])
    keep = out["SEx"] != 0.0
    return {k: (v[keep] if isinstance(v, np.ndarray) and v.shape == keep.shape else v) for k, v in out.items()}


def test_fixture_covers_the_test_install_cases():
    g = load_rows()
    assert len(g["SEx"]) > 2500
    assert set(np.unique(g["case"])) == set(range(len(g["cases"])))
    assert np.all(g["Z"] == 1.0)                       # hqpe_sc prints Z = 1 (no renormalisation)


def test_qp_energies_reproduce_reference_rows():
    g = load_rows()
    h = hqpe.HARTREE_EV
    eqp = hqpe.qp_energies(g["eLDA"], np.diag(g["SEx"] / h), np.diag(g["SExcore"] / h), np.diag(g["SEc"] / h),
                           g["vxc"])
    # four rounded inputs and one rounded output: |error| <= 5 half-steps
    err = np.abs((eqp - g["eLDA"]) - g["dSEnoZ"])
    assert np.all(err <= 5 * g["half"] + 1e-9), err.max()
    ehf = g["eLDA"] + g["SEx"] + g["SExcore"] - g["vxc"]
    assert np.all(np.abs(ehf - g["eHF"]) <= 5 * g["half"] + 1e-9)
    res = g["SEx"] + g["SExcore"] + g["SEc"]
    assert np.all(np.abs(res - g["ReS"]) <= 3 * g["half"] + 0.5e-5 + 1e-9)
    # the sign convention is visible: flipping vxc's sign breaks most rows
    bad = np.abs((g["SEx"] + g["SExcore"] + g["SEc"] + g["vxc"]) - g["dSEnoZ"]) > 5 * g["half"]
    assert bad.mean() > 0.9
