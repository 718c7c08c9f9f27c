"""qsgw_dpsion_chiq_d (Hilbert transform of the chi0 histogram) against
oracle/dpsion.py: relative Frobenius error <= 1e-11 on chi0(i w) and
chi0(w_r), with and without the Gaussian cut ecut and the SmearX0 filter,
odd sizes, the imaginary axis alone, and the reference's argument checks."""
import numpy as np
import pytest

from ecalj_b200 import synth
from oracle import dpsion as dp
from tests.conftest import rel_fro

pytestmark = pytest.mark.gpu
TOL = 1e-11


def _case(npr, npr_col, nwhis, niw, nw, seed):
    rng = np.random.default_rng(seed)
    aa = 0.05
    frhis = 1e-3 / aa * (np.exp(aa * np.arange(nwhis + 1)) - 1.0)
    rcxq = rng.standard_normal((npr, npr_col, nwhis + 1)) + 1j * rng.standard_normal((npr, npr_col, nwhis + 1))
    freq_i = synth.imag_mesh(niw)['freq_i'] if niw else np.zeros(0)
    freq_r = None
    if nw >= 0:
        freq_r = np.zeros(nw + 1)
        freq_r[1:] = 0.5 * (frhis[:nw] + frhis[1:nw + 1])
    return frhis, rcxq, freq_i, freq_r


def _run(qsgw, npr, npr_col, nwhis, frhis, rcxq, freq_i, freq_r, ecut, smear=0.0):
    import torch
    d = torch.from_numpy(np.asfortranarray(rcxq).reshape(-1, order='F')).to('cuda')
    zi, zr = qsgw.dpsion_chiq_d(d, npr, npr_col, nwhis, frhis, freq_i, freq_r, ecut, smearx0=smear)
    qsgw.synchronize()
    niw = len(freq_i)
    gi = zi.cpu().numpy().reshape((npr, npr_col, niw), order='F') if zi is not None else None
    gr = zr.cpu().numpy().reshape((npr, npr_col, len(freq_r)), order='F') if zr is not None else None
    return gi, gr


@pytest.mark.parametrize("npr,npr_col,nwhis,niw,nw,ecut,smear", [
    (37, 29, 40, 12, 15, 1e10, 0.0),
    (37, 29, 40, 12, 15, 0.03, 0.0),
    (37, 29, 40, 12, 15, 1e10, 0.005),
    (64, 1, 7, 3, 0, 1e10, 0.0),
    (200, 200, 150, 24, 60, 1e10, 0.0),
])
def test_dpsion_vs_oracle(qsgw, npr, npr_col, nwhis, niw, nw, ecut, smear):
    frhis, rcxq, freq_i, freq_r = _case(npr, npr_col, nwhis, niw, nw, seed=npr + nwhis)
    ri, rr = dp.dpsion_chiq(rcxq, frhis, freq_i, freq_r, ecut, smear)
    gi, gr = _run(qsgw, npr, npr_col, nwhis, frhis, rcxq, freq_i, freq_r, ecut, smear)
    print(f"dpsion {npr}x{npr_col} nwhis={nwhis}: imag {rel_fro(gi, ri):.2e} real {rel_fro(gr, rr):.2e}")
    assert rel_fro(gi, ri) < TOL
    assert rel_fro(gr, rr) < TOL


def test_dpsion_imaginary_axis_only(qsgw):
    frhis, rcxq, freq_i, _ = _case(20, 17, 30, 8, -1, seed=3)
    ri, _ = dp.dpsion_chiq(rcxq, frhis, freq_i)
    gi, gr = _run(qsgw, 20, 17, 30, frhis, rcxq, freq_i, None, 1e10)
    assert gr is None
    assert rel_fro(gi, ri) < TOL


def test_dpsion_argument_checks(qsgw):
    import torch
    frhis, rcxq, freq_i, freq_r = _case(8, 8, 10, 4, 10, seed=5)     # nw = nwhis: dpsion5.f90:208
    d = torch.zeros(8 * 8 * 11, dtype=torch.complex128, device='cuda')
    with pytest.raises(qsgw.QSGWError):
        qsgw.dpsion_chiq_d(d, 8, 8, 10, frhis, freq_i, freq_r)
    fr = np.array([0.01, 0.02])                                       # freq_r(0) /= 0: dpsion5.f90:209
    with pytest.raises(qsgw.QSGWError):
        qsgw.dpsion_chiq_d(d, 8, 8, 10, frhis, freq_i, fr)
