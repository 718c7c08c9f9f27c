"""chi0 at N = 1500 (nk = 512, nocc = 40, nunocc U{300..1200}, 32 iw): its zmel
cannot be resident (369 GB for 512 k), so chi0 is accumulated k by k with
qsgw_chi0_lorentz_acc_d.  Four k-points of the 512-point mesh are streamed one
at a time and compared with one call over the same four k (FP64), in FP64 and
in split precision."""
import math

import numpy as np
import pytest

from ecalj_b200 import synth
from tests.conftest import rel_fro

pytestmark = pytest.mark.gpu


def test_n1500_streamed_chi0(qsgw):
    import torch
    lib = qsgw
    c = synth.CONFIGS["chi0_n1500_streamed"]
    N, niw, nkb = c["N"], c["niw"], 4
    rng = np.random.default_rng(c["seed"])
    nocc, nun, eocc, eun = synth.chi0_spectrum(rng, nkb, c["nocc"], c["nun"])
    fi = synth.imag_mesh(niw)["freq_i"]
    eo = [e * 0.5 for e in eocc]
    eu = [e * 0.5 for e in eun]
    g = torch.Generator(device="cuda")
    zk = []
    for k in range(nkb):                                   # zmel of one k, generated on the device
        g.manual_seed(c["seed"] * 7919 + k)
        n = N * int(nocc[k]) * int(nun[k])
        z = torch.randn(2 * n, dtype=torch.float64, device="cuda", generator=g) / math.sqrt(N)
        zk.append(torch.view_as_complex(z.view(-1, 2)).contiguous())
    zall = torch.cat(zk)
    ref = torch.zeros(N * N * niw, dtype=torch.complex128, device="cuda")
    lib.set_precision(lib.PREC_FP64)
    lib.chi0_lorentz_acc_d(ref, N, niw, fi, c["nk"], nocc, nun, np.concatenate(eo), np.concatenate(eu), zall)
    for prec, tol in ((lib.PREC_FP64, 1e-13), (lib.PREC_SPLIT_F16, 2e-5)):
        lib.set_precision(prec)
        chi = torch.zeros_like(ref)
        for k in range(nkb):
            lib.chi0_lorentz_acc_d(chi, N, niw, fi, c["nk"], nocc[k:k + 1], nun[k:k + 1], eo[k], eu[k], zk[k])
        lib.synchronize()
        e = float(torch.linalg.vector_norm(chi - ref) / torch.linalg.vector_norm(ref))
        assert e <= tol, (prec, e)
    lib.set_precision(lib.PREC_FP64)
    # chi0(iw) <= 0 and Hermitian: a property of the full-size result
    c0 = ref.view(niw, N, N)[0]
    assert float(torch.linalg.vector_norm(c0 - c0.conj().T) / torch.linalg.vector_norm(c0)) <= 1e-13
    assert float(torch.real(torch.diagonal(c0)).max()) < 0
