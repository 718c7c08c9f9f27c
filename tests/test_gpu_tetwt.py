"""Tetrahedron histogram weights on the GPU against the oracle (FP64,
relative Frobenius <= 1e-11), the volume sum rule, and the status word for
excitation energies outside the histogram."""
import numpy as np
import pytest

from ecalj_b200 import synth
from oracle import tetwt as tw
from tests.conftest import rel_fro

pytestmark = pytest.mark.gpu


def test_tetwt_vs_oracle(qsgw):
    import torch
    lib = qsgw
    idt, qbzw, ek, ekq = synth.tetra_mesh(3)
    nocc, nunocc, ef = 3, 6, 0.0
    fr = np.linspace(-0.4, 1.6, 41)
    nk = qbzw.shape[0]
    w = torch.zeros(nk * nocc * nunocc * (len(fr) - 1), dtype=torch.float64, device="cuda")
    vt = lib.tetwt_hist_d(w, idt, qbzw, ek, ekq, ef, fr, nocc, nunocc)
    lib.synchronize()
    ref, vref = tw.tetwt_hist(idt, qbzw, ek, ekq, ef, fr, nocc, nunocc)
    assert abs(vt - vref) <= 1e-13 and abs(vt - 1.0) <= 1e-12
    got = w.cpu().numpy().reshape(nk, nocc, nunocc, len(fr) - 1)
    assert np.abs(ref).sum() > 0
    assert rel_fro(got, ref) <= 1e-11          # cbrt vs **(1/3), det by cofactors, atomic order


def test_tetwt_out_of_histogram_sets_status(qsgw):
    import torch
    lib = qsgw
    idt, qbzw, ek, ekq = synth.tetra_mesh(2)
    fr = np.linspace(0.0, 0.05, 6)                        # far narrower than the excitation energies
    w = torch.zeros(qbzw.shape[0] * 3 * 6 * 5, dtype=torch.float64, device="cuda")
    lib.tetwt_hist_d(w, idt, qbzw, ek, ekq, 0.0, fr, 3, 6)
    with pytest.raises(lib.QSGWError) as e:
        lib.synchronize()
    assert e.value.code == -5
    with pytest.raises(lib.QSGWError):                  # corner index outside the mesh
        lib.tetwt_hist_d(w, idt + 1000, qbzw, ek, ekq, 0.0, fr, 3, 6)
