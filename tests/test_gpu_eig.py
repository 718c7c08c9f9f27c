"""Hand-written FP64 Jacobi eigensolver for the Coulomb matrix against the
oracle (LAPACK zhegvx) and against the defining identities."""
import numpy as np
import pytest

from oracle import llw
from ecalj_b200 import synth
from tests.conftest import rel_fro

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("n,overlap", [(1, False), (2, False), (37, False), (160, False), (64, True)])
def test_zhegv_vs_oracle(qsgw, n, overlap):
    vsq, q = synth.coulomb(n, 40 + n)
    v = np.asfortranarray(q @ np.diag(vsq ** 2) @ q.conj().T)
    v = 0.5 * (v + v.conj().T)
    o = None
    if overlap:
        rng = np.random.default_rng(n)
        g = rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))
        o = np.asfortranarray(np.eye(n) + 0.2 * g @ g.conj().T / n)
    ref_l, ref_z = llw.coulomb_eig(v, o)
    dv = qsgw.to_device(np.asfortranarray(v))
    do = qsgw.to_device(o) if overlap else None
    lam = qsgw.zhegv_d(dv, n, o=do)
    z = qsgw.from_device(dv, (n, n))
    assert rel_fro(lam, np.sort(ref_l)[::-1]) < 1e-12
    ob = np.eye(n) if o is None else o
    assert rel_fro(v @ z, ob @ z @ np.diag(lam)) < 1e-11                   # v z = lambda O z
    assert np.abs(z.conj().T @ ob @ z - np.eye(n)).max() < 1e-11           # O-orthonormal
