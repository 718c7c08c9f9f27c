"""Real frequency axis: pivoted batched inverse, chi0 of the Lorentzian model
on real frequencies and W - v (WVRllwR) against the oracle (FP64, <= 1e-11)."""
import numpy as np
import pytest

from ecalj_b200 import synth
from oracle import llw, x0
from tests.conftest import rel_fro

pytestmark = pytest.mark.gpu
TOL = 1e-11


def _pairs(p):
    de = np.concatenate([(np.asarray(eu)[None, :] - np.asarray(eo)[:, None]).T.ravel() * 0.5
                         for eo, eu in zip(p["eocc_ry"], p["eun_ry"])])
    return de


@pytest.mark.parametrize("n,nbatch", [(70, 3), (33, 2), (96, 1)])
def test_zminv_batched_pivoted(qsgw, n, nbatch):
    lib = qsgw
    rng = np.random.default_rng(n)
    a = rng.standard_normal((n, n, nbatch)) + 1j * rng.standard_normal((n, n, nbatch))
    a[:5, :5, :] *= 1e-8                                # small leading block: pivoting is required
    lda = n + 3
    buf = np.zeros((lda, n, nbatch), complex, order="F")
    buf[:n] = a
    d = lib.to_device(buf)
    lib.zminv_batched_d(d, n, lda, nbatch)
    lib.synchronize()
    got = lib.from_device(d, (lda, n, nbatch))
    for b in range(nbatch):
        assert rel_fro(got[:n, :, b], np.linalg.inv(a[:, :, b])) <= 1e-10
        np.testing.assert_array_equal(got[n:, :, b], 0)   # padding rows untouched


def test_zminv_batched_singular_sets_status(qsgw):
    lib = qsgw
    a = np.zeros((8, 8), complex, order="F")
    a[:4, :4] = np.eye(4)                                # rank 4
    d = lib.to_device(a)
    lib.zminv_batched_d(d, 8, 8, 1)
    with pytest.raises(lib.QSGWError) as e:
        lib.synchronize()
    assert e.value.code == -5
    lib.synchronize()                                    # the status was cleared by the report


def test_chi0_real_vs_oracle_and_imaginary_limit(qsgw):
    import torch
    lib = qsgw
    p = synth.chi0_problem(N=48, nk=3, nocc=2, nun=(5, 8), niw=4, seed=21)
    N, nk = p["N"], p["nk"]
    fr = synth.freq_r_mesh(7, wmax=1.5)                  # includes w = 0
    eta = 0.02
    z = lib.to_device(p["zcols"])
    chi = torch.zeros(N * N * len(fr), dtype=torch.complex128, device="cuda")
    lib.chi0_lorentz_real_d(chi, N, len(fr), fr, eta, nk, p["nocc"], p["nun"], p["eocc_h"], p["eun_h"], z)
    got = lib.from_device(chi, (N, N, len(fr)))
    ref = x0.chi0_real(p["zcols"], _pairs(p), nk, fr, eta)
    assert rel_fro(got, ref) <= TOL
    # eta = 0 at w = 0 is the imaginary-axis chi0 at nu = 0
    chi0 = torch.zeros(N * N, dtype=torch.complex128, device="cuda")
    lib.chi0_lorentz_real_d(chi0, N, 1, [0.0], 0.0, nk, p["nocc"], p["nun"], p["eocc_h"], p["eun_h"], z)
    chii = torch.zeros(N * N, dtype=torch.complex128, device="cuda")
    lib.chi0_lorentz_d(chii, N, 1, [0.0], nk, p["nocc"], p["nun"], p["eocc_h"], p["eun_h"], z)
    assert rel_fro(chi0.cpu().numpy(), chii.cpu().numpy()) <= 1e-13


@pytest.mark.parametrize("is_wc_m", [True, False])
def test_wvr_vs_oracle(qsgw, is_wc_m):
    import torch
    lib = qsgw
    p = synth.chi0_problem(N=40, nk=3, nocc=2, nun=(5, 8), niw=4, seed=23)
    N, nk = p["N"], p["nk"]
    fr = synth.freq_r_mesh(6, wmax=1.5)
    nw = len(fr)
    vsq, q = synth.coulomb(N, 24)
    vsq = vsq * 0.3                                      # keep eps~ comfortably invertible on the real axis
    chi = x0.chi0_real(p["zcols"], _pairs(p), nk, fr, 0.05)
    ref = llw.wvr_llw(np.asfortranarray(chi.copy()), 2, vsq, q, True, is_wc_m, 2)
    d = lib.to_device(np.asfortranarray(chi))
    zw = torch.zeros(N * N * nw, dtype=torch.complex128, device="cuda")
    lib.wvr_llw_d(d, N, nw, 2, vsq, lib.to_device(q), True, is_wc_m, 2, zw)
    lib.synchronize()
    assert rel_fro(lib.from_device(zw, (N, N, nw)), ref) <= TOL
