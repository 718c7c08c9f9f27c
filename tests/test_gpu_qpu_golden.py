"""qsgw_hqpe_d against the reference's own QPU rows (Samples/TestInstall/*,
extracted into tests/golden/qpu_rows.npz): the states are packed 64 per
q-point as diagonal Hartree matrices, and eQP - eLDA must reproduce dSEnoZ to
the rounding of the printed fields, as the oracle does."""
import numpy as np
import pytest

from oracle import hqpe
from tests.test_qpu_golden_cpu import load_rows

pytestmark = pytest.mark.gpu
NTQ = 64


def test_hqpe_reproduces_reference_rows(qsgw):
    import torch
    g = load_rows()
    n = len(g["SEx"])
    nq = (n + NTQ - 1) // NTQ
    h = hqpe.HARTREE_EV

    def stack(v):                                     # diagonal (NTQ, NTQ, nq) Hartree matrices
        m = np.zeros((NTQ, NTQ, nq), complex, order='F')
        for i in range(n):
            m[i % NTQ, i % NTQ, i // NTQ] = v[i] / h
        return m

    def col(v):                                       # (NTQ, nq) eV, zero padded
        c = np.zeros(NTQ * nq)
        c[:n] = v
        return np.asfortranarray(c.reshape(NTQ, nq, order='F'))

    mats = [stack(g["SEx"]), stack(g["SExcore"]), stack(g["SEc"]), np.zeros((NTQ, NTQ, nq), complex, order='F')]
    d = [qsgw.to_device(m) for m in mats]
    de, dv = qsgw.to_device(col(g["eLDA"])), qsgw.to_device(col(g["vxc"]))
    eqp = torch.zeros(NTQ * nq, dtype=torch.float64, device='cuda')
    seh = torch.zeros(NTQ * NTQ * nq, dtype=torch.complex128, device='cuda')
    qsgw.hqpe_d(d[0], d[1], d[2], d[3], de, dv, NTQ, NTQ, nq, eqp, seh)
    qsgw.synchronize()
    e = eqp.cpu().numpy()[:n]
    err = np.abs((e - g["eLDA"]) - g["dSEnoZ"])
    assert np.all(err <= 5 * g["half"] + 1e-9), err.max()
