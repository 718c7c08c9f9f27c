"""chi0 at the full N = 600 workload (nk = 216, nocc = 9, nunocc U{100..300},
390 834 pairs, 24 iw): too large for the oracle, so checked through
properties that do not depend on the size.  The split-FP16 result equals the
plain FP64 result to the split path's gate (relative Frobenius <= 5e-5;
measured about 1e-6); both are Hermitian in (G, G') and negative
definite at every iw checked, as chi0(iw) = -sum |z><z| 2 de / (de^2 + w^2) / nk
with far more pairs than rows must be.  Collected after the other GPU tests:
it grows the library's device scratch to the full workload, after which the
graph test's refusal to grow scratch while recording would have nothing to
refuse."""
import math

import numpy as np
import pytest

from ecalj_b200 import synth

pytestmark = pytest.mark.gpu


def test_chi0_n600_split_equals_fp64_and_keeps_its_properties(qsgw):
    import torch
    c = synth.CONFIGS["chi0_n600"]
    rng = np.random.default_rng(c["seed"])
    nocc, nun, eocc, eun = synth.chi0_spectrum(rng, c["nk"], c["nocc"], c["nun"])
    mesh = synth.imag_mesh(c["niw"])
    N, niw, nk = c["N"], c["niw"], c["nk"]
    npair = int(np.sum(nocc * nun))
    assert npair > 350000
    g = torch.Generator(device="cuda")
    g.manual_seed(c["seed"])
    zc = torch.empty(2 * N * npair, dtype=torch.float64, device="cuda")
    zc.normal_(0.0, 1.0 / math.sqrt(N), generator=g)
    zc = zc.view(torch.complex128)
    eo, eu = np.concatenate(eocc) * 0.5, np.concatenate(eun) * 0.5
    out = {}
    try:
        for prec in (qsgw.PREC_FP64, qsgw.PREC_SPLIT_F16):
            qsgw.set_precision(prec, 2 if prec == qsgw.PREC_SPLIT_F16 else 1)
            chi = torch.zeros(N * N * niw, dtype=torch.complex128, device="cuda")
            qsgw.chi0_lorentz_d(chi, N, niw, mesh["freq_i"], nk, nocc, nun, eo, eu, zc)
            qsgw.synchronize()
            out[prec] = chi.view(niw, N, N)          # slot j: column-major (N, N) = row-major transposed
    finally:
        qsgw.set_precision(qsgw.PREC_FP64, 1)
    ref, got = out[qsgw.PREC_FP64], out[qsgw.PREC_SPLIT_F16]
    err = float(torch.linalg.vector_norm(got - ref) / torch.linalg.vector_norm(ref))
    print(f"chi0 N=600 full size: split vs FP64 relative Frobenius {err:.2e}")
    assert err < 5e-5
    for m, tol in ((ref, 1e-12), (got, 5e-5)):      # the split diagonal tiles need not be bitwise Hermitian
        herm = float(torch.linalg.vector_norm(m - m.conj().transpose(1, 2)) / torch.linalg.vector_norm(m))
        assert herm < tol
    for j in (0, niw // 2, niw - 1):
        for m in (ref, got):
            a = m[j]
            ev = torch.linalg.eigvalsh(0.5 * (a + a.conj().T)).cpu().numpy()
            assert ev.max() < 0.0                        # 390 834 pairs >> N: negative definite
