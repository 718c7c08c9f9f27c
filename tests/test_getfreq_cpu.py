"""The frequency meshes of Getfreq (m_freq.f90:94-133) as ecalj_b200.synth
restates them: the histogram bins frhis(i) = bb (exp(aa (i-1)) - 1) with
aa = HistBin_ratio - 1, bb = HistBin_dw / aa, the bin count from omg2max, the
real-axis point count from wemax, and freq_r at the bin midpoints."""
import math

import numpy as np
import pytest

from ecalj_b200 import synth


@pytest.mark.parametrize("omg2max,wemax,oratio,dw", [(1.0, 0.8, 1.03, 1e-5), (2.5, 3.0, 1.08, 1e-3),
                                                     (0.3, 0.05, 1.03, 1e-5)])
def test_getfreq_rules(omg2max, wemax, oratio, dw):
    m = synth.getfreq(omg2max, wemax, oratio, dw)
    fr, nwhis, nw = m["frhis"], m["nwhis"], m["nw"]
    aa = oratio - 1.0
    assert len(fr) == nwhis + 1 and fr[0] == 0.0
    np.testing.assert_allclose(fr, dw / aa * np.expm1(aa * np.arange(nwhis + 1)), rtol=1e-12, atol=0)
    # nwhis - 2 is the first 1-based iw whose edge passes omg2max (+1e-6)
    assert fr[nwhis - 3] > omg2max + 1e-6 >= fr[nwhis - 4]
    # nw: the first iw >= 3 whose midpoint (frhis(iw-2) + frhis(iw-1))/2 passes wemax/2
    mid = lambda iw: 0.5 * (fr[iw - 3] + fr[iw - 2])        # noqa: E731
    assert mid(nw) > wemax / 2.0 and (nw == 3 or mid(nw - 1) <= wemax / 2.0)
    assert nw <= nwhis - 1
    f = m["freq_r"]
    assert len(f) == nw + 1 and f[0] == 0.0 and np.all(np.diff(f) > 0)
    np.testing.assert_array_equal(f[1:], 0.5 * (fr[:nw] + fr[1:nw + 1]))


def test_getfreq_known_sizes_and_epsmode():
    # aa = 0.03, bb = 1e-5 / 0.03: exp(0.03 (iw-1)) > 1 + 1.000001 / bb first at iw = 268
    m = synth.getfreq(1.0, 0.8)
    assert m["nwhis"] == 270
    assert math.isclose(m["frhis"][1], 1e-5 / 0.03 * math.expm1(0.03), rel_tol=1e-12)
    e = synth.getfreq(1.0, 0.8, epsmode=True)
    assert e["nw"] == e["nwhis"] - 1 and len(e["freq_r"]) == e["nwhis"]
    with pytest.raises(ValueError):
        synth.getfreq(0.1, 5.0)                            # wemax/2 past every bin: nw undefined


def test_chain_tests_mesh_is_getfreq_form():
    """The bins the tetrahedron chain tests use are Getfreq's with ratio 1.08, dw 1e-3."""
    m = synth.getfreq(1.4, 0.05, oratio=1.08, dw=1e-3)
    ref = 1e-3 / 0.08 * (np.exp(0.08 * np.arange(61)) - 1.0)
    assert m["nwhis"] >= 60
    np.testing.assert_allclose(m["frhis"][:61], ref, rtol=1e-13, atol=1e-17)
