"""The tetrahedron chi0 chain on the GPU, as x0kf_zxq runs it for npm = 1:
tetrahedron histogram weights (qsgw_tetwt_hist_d) -> pair/bin lists
(qsgw_x0_lists) -> x0gemm per k (qsgw_x0gemm_d) -> Hilbert transform
(qsgw_dpsion_chiq_d) -> chi0(i w) and chi0(w_r).  Checked against the oracle
chain with the dense contraction in place of the lists: with the same
weights, lists + x0gemm + Hilbert transform to relative Frobenius <= 1e-11;
with the oracle's own weights to <= 1e-10 (the weights agree to ~3e-12, and
the real-axis chi0 takes single bins, Im part included, without smoothing);
and chi0(i w) Hermitian negative semidefinite.  The same with bands that
touch at some k, the weights symmetrised over the degenerate bands."""
import numpy as np
import pytest

from ecalj_b200 import synth
from oracle import dpsion as dp
from oracle import tetwt as tw
from tests.conftest import rel_fro

pytestmark = pytest.mark.gpu


def test_tetra_chain_vs_oracle(qsgw):
    _chain(qsgw, degenerate=False)


@pytest.mark.parametrize("ns,tol", [(3, 3e-5), (4, 3e-7)])
def test_tetra_chain_int8(qsgw, ns, tol):
    """The same chain with x0gemm on the int8 Ozaki path (the reference's own
    chi0 boundary: the pair/bin lists of the tetrahedron weights, accumulated
    per k into rcxq), against the oracle chain with the same weights."""
    try:
        qsgw.set_precision(qsgw.PREC_SPLIT_I8, ns)
        _chain(qsgw, degenerate=False, tol=tol)
    finally:
        qsgw.set_precision(qsgw.PREC_FP64, 1)


def test_tetra_chain_degenerate_bands(qsgw):
    """Bands that touch at some k: the host copy of the GPU weights is
    symmetrised (qsgw_tetwt_symmetrize) before the lists are built, as
    tetwt5x_dtet4 does; the oracle chain symmetrises its own weights."""
    _chain(qsgw, degenerate=True)


def _chain(qsgw, degenerate, tol=None):
    """tol: the gate of a split-precision x0gemm (None: the FP64 gates)."""
    import torch
    idt, qbzw, ek, ekq = synth.tetra_mesh(3)
    if degenerate:
        ek[::3, 2] = ek[::3, 1] + 2e-5                  # occupied bands 1, 2 touch at every third k
        ekq[::2, 4] = ekq[::2, 3]                       # bands 3, 4 at k+q at every second k
    nocc, nunocc, ef, npr = 3, 6, 0.0, 24
    frhis = 1e-3 / 0.08 * (np.exp(0.08 * np.arange(61)) - 1.0)
    nwhis = len(frhis) - 1
    nk = qbzw.shape[0]
    rng = np.random.default_rng(21)
    z = [np.asfortranarray(rng.standard_normal((npr, nocc, nunocc)) + 1j * rng.standard_normal((npr, nocc, nunocc)))
         for _ in range(nk)]
    freq_i = synth.imag_mesh(10)['freq_i']
    nw = 20
    freq_r = np.concatenate([[0.0], 0.5 * (frhis[:nw] + frhis[1:nw + 1])])

    # GPU chain
    wd = torch.zeros(nk * nocc * nunocc * nwhis, dtype=torch.float64, device='cuda')
    qsgw.tetwt_hist_d(wd, idt, qbzw, ek, ekq, ef, frhis, nocc, nunocc)
    qsgw.synchronize()
    w = wd.cpu().numpy().reshape(nk, nocc, nunocc, nwhis)
    if degenerate:
        raw = w.copy()
        w = qsgw.tetwt_symmetrize(w.copy(), ek, ekq)
        assert np.array_equal(w, tw.symmetrize_degenerate(raw, ek, ekq))
        assert not np.array_equal(w, raw)
    t = qsgw.x0_lists(w)
    rcxq = torch.zeros(npr * npr * (nwhis + 1), dtype=torch.complex128, device='cuda')
    for k in range(nk):
        zk = torch.from_numpy(z[k].reshape(-1, order='F')).to('cuda')
        qsgw.x0gemm(rcxq, npr, 1, npr, nwhis, 1, 1, nocc, zk, 1, int(t["icounkmin"][k]), int(t["icounkmax"][k]),
                    t["itc"], t["itpc"], t["jpmc"], t["iwini"], t["iwend"], t["icouini"], t["whwc"],
                    zmel_shape=(npr, nocc, nunocc), device=True)
    zi, zr = qsgw.dpsion_chiq_d(rcxq, npr, npr, nwhis, frhis, freq_i, freq_r)
    qsgw.synchronize()
    gi = zi.cpu().numpy().reshape((npr, npr, len(freq_i)), order='F')
    gr = zr.cpu().numpy().reshape((npr, npr, nw + 1), order='F')

    # oracle chain: dense contraction (no lists), Hilbert transform
    def oracle_chain(wts):
        r = np.zeros((npr, npr, nwhis + 1), complex)
        for k in range(nk):
            zz = z[k].reshape(npr, -1)                           # column p = ib * nunocc + jb
            r[:, :, 1:] += np.einsum('ap,bp,ph->abh', zz.conj(), zz, wts[k].reshape(-1, nwhis))
        return dp.dpsion_chiq(r, frhis, freq_i, freq_r)

    ri, rr = oracle_chain(w)                                     # the GPU's weights
    print(f"tetra chain, same weights: imag {rel_fro(gi, ri):.2e} real {rel_fro(gr, rr):.2e}")
    if tol is not None:
        assert rel_fro(gi, ri) < tol and rel_fro(gr, rr) < tol
        return
    assert rel_fro(gi, ri) < 1e-11
    assert rel_fro(gr, rr) < 1e-11
    wref, _ = tw.tetwt_hist(idt, qbzw, ek, ekq, ef, frhis, nocc, nunocc)
    if degenerate:
        wref = tw.symmetrize_degenerate(wref, ek, ekq)
    ri, rr = oracle_chain(wref)                                  # the oracle's weights
    print(f"tetra chain, oracle weights: imag {rel_fro(gi, ri):.2e} real {rel_fro(gr, rr):.2e}")
    assert rel_fro(gi, ri) < 1e-10
    assert rel_fro(gr, rr) < 1e-10
    # chi0(i w) is Hermitian and negative semidefinite
    for j in range(len(freq_i)):
        m = gi[:, :, j]
        assert np.allclose(m, m.conj().T, atol=1e-12 * np.abs(m).max())
        assert np.linalg.eigvalsh(0.5 * (m + m.conj().T)).max() <= 1e-12 * np.abs(m).max()
