"""Degenerate-band symmetrisation of the tetrahedron weights
(qsgw_tetwt_symmetrize, host-only) against the oracle restatement of
tetwt5.f90:347-423 and chkdgn (:868-912): bit-exact on random weights with
planted degeneracies and on the weights of a tetrahedron mesh, plus the
properties the averaging must keep."""
import numpy as np
import pytest

from ecalj_b200 import lib, synth
from oracle import tetwt as tw


def test_chkdgn_groups():
    assert tw.chkdgn([]) == []
    assert tw.chkdgn([0.3]) == [(0, 0)]
    e = [0.0, 5e-5, 0.5, 0.5, 0.5 + 2e-4, 0.9]
    assert tw.chkdgn(e) == [(0, 1), (2, 3), (4, 4), (5, 5)]
    # neighbours, not the group's first level: a slow drift stays one group
    assert tw.chkdgn([0.0, 0.9e-4, 1.8e-4, 2.7e-4]) == [(0, 3)]


def _levels(rng, nk, nband):
    e = np.sort(rng.uniform(-1.0, 1.0, (nk, nband)), axis=1)
    for k in range(nk):                    # plant degenerate runs at some k
        if k % 2 == 0:
            e[k, 1:4] = e[k, 1] + np.array([0.0, 3e-5, 6e-5])
        if k % 3 == 0:
            e[k, 5:7] = e[k, 5]
    return e


def test_matches_oracle_bitwise():
    rng = np.random.default_rng(21)
    nk, nband, nocc, nunocc, nwhis = 6, 8, 5, 7, 9
    ek, ekq = _levels(rng, nk, nband), _levels(rng, nk, nband)
    w = rng.uniform(0.0, 1.0, (nk, nocc, nunocc, nwhis))
    w[rng.uniform(size=w.shape) < 0.4] = 0.0
    ref = tw.symmetrize_degenerate(w, ek, ekq)
    got = lib.tetwt_symmetrize(w.copy(), ek, ekq)
    np.testing.assert_array_equal(got, ref)
    # the block sums are kept; members of a block are equal; other pairs untouched
    for k in range(nk):
        for (i0, i1) in tw.chkdgn(ek[k, :nocc]):
            for (j0, j1) in tw.chkdgn(ekq[k, :nunocc]):
                blk, orig = got[k, i0:i1 + 1, j0:j1 + 1], w[k, i0:i1 + 1, j0:j1 + 1]
                np.testing.assert_allclose(blk.sum(axis=(0, 1)), orig.sum(axis=(0, 1)), rtol=1e-14, atol=0)
                assert np.all(blk == blk[0, 0])
                if blk.shape[:2] == (1, 1):
                    assert np.array_equal(blk, orig)


def test_mesh_weights_chain():
    """tetwt weights of a mesh whose bands touch at some k, symmetrised, then
    turned into x0gemm lists: every member of a degenerate block is listed."""
    idt, q, ek, ekq = synth.tetra_mesh(2, nband=6, seed=4)
    ek[::3, 2] = ek[::3, 1] + 2e-5                  # touching bands at every third k
    ekq[::2, 4] = ekq[::2, 3]
    fr = np.linspace(0.0, 1.2, 25)
    w, _ = tw.tetwt_hist(idt, q, ek, ekq, 0.0, fr, 4, 6)
    ref = tw.symmetrize_degenerate(w, ek, ekq)
    got = lib.tetwt_symmetrize(w.copy(), ek, ekq)            # in place: keep w
    np.testing.assert_array_equal(got, ref)
    assert not np.array_equal(got, w)               # the planted degeneracies changed something
    np.testing.assert_allclose(got.sum(), w.sum(), rtol=1e-13)
    t = lib.x0_lists(got)
    listed = {(k, int(t["itc"][c]) - 1, int(t["itpc"][c]) - 1)
              for k in range(got.shape[0])
              for c in range(int(t["icounkmin"][k]) - 1, int(t["icounkmax"][k]))}
    nz = {tuple(int(v) for v in i) for i in zip(*np.nonzero(got.any(axis=3)))}
    assert listed == nz


def test_arguments():
    w = np.zeros((2, 3, 3, 4))
    with pytest.raises(lib.QSGWError, match='nband=2'):
        lib.tetwt_symmetrize(w, np.zeros((2, 2)), np.zeros((2, 2)))
    with pytest.raises(ValueError):
        lib.tetwt_symmetrize(w.astype(np.float32), np.zeros((2, 3)), np.zeros((2, 3)))
