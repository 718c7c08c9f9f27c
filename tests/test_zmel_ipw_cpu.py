"""CPU check of the plane-wave zmel oracle: its single-formula definition
against the reference's two evaluation orders restated step by step."""
import numpy as np

from ecalj_b200 import synth
from oracle import zmel as oz


def _lookup(vecs):
    return {tuple(int(c) for c in vecs[:, i]): i for i in range(vecs.shape[1])}


def _branch_g1_first(t):
    """m_zmel.f90:439-480: gggmat(c, G1) -> ggitp = gggmat geigq -> gather
    rows Gc+G2 -> times dgeigqk, per itp."""
    lg, lc = _lookup(t["nvggg"]), _lookup(t["nvgcgp2"])
    comp = t["nvgcgp2"]
    M = np.zeros((comp.shape[1], t["ngvecpB1"].shape[1]), complex)
    for c in range(comp.shape[1]):
        for g in range(M.shape[1]):
            k = lg.get(tuple(int(x) for x in t["ngvecpB1"][:, g] - comp[:, c] - t["nadd"]))
            if k is not None:
                M[c, g] = t["ggg"][k]
    T = M @ t["geigq"]
    ngc = t["ngveccR"].shape[1]
    idx = np.array([[lc[tuple(int(x) for x in t["ngveccR"][:, c] + t["ngvecpB2"][:, g])]
                     for g in range(t["ngvecpB2"].shape[1])] for c in range(ngc)])
    out = np.stack([T[idx, itp] @ t["dgeigqk"] for itp in range(T.shape[1])], axis=-1)
    return t["phase"][:, None, None] * out


def _branch_g2_first(t):
    """m_zmel.f90:481-524: gggmat(c, G2) -> ggit = gggmat dgeigqk -> gather
    rows Gc-G1 -> times geigq, per it."""
    lg, lc = _lookup(t["nvggg"]), _lookup(t["nvgcgp2"])
    comp = t["nvgcgp2"]
    M = np.zeros((comp.shape[1], t["ngvecpB2"].shape[1]), complex)
    for c in range(comp.shape[1]):
        for g in range(M.shape[1]):
            k = lg.get(tuple(int(x) for x in -t["ngvecpB2"][:, g] - comp[:, c] - t["nadd"]))
            if k is not None:
                M[c, g] = t["ggg"][k]
    T = M @ t["dgeigqk"]
    ngc = t["ngveccR"].shape[1]
    idx = np.array([[lc[tuple(int(x) for x in t["ngveccR"][:, c] - t["ngvecpB1"][:, g])]
                     for g in range(t["ngvecpB1"].shape[1])] for c in range(ngc)])
    out = np.stack([T[idx, it] @ t["geigq"] for it in range(T.shape[1])], axis=1)
    return t["phase"][:, None, None] * out


def test_ipw_definition_matches_both_reference_orders():
    t = synth.ipw_tables(3, ngc=9, ngp1=8, ngp2=7, ntp0=3, nmv=4)
    ref = oz.zmel_ipw(t["geigq"], t["dgeigqk"], t["ngvecpB1"], t["ngvecpB2"], t["ngveccR"], t["nvggg"], t["ggg"],
                      t["nadd"], t["phase"])
    for f in (_branch_g1_first, _branch_g2_first):
        got = f(t)
        assert np.linalg.norm(got - ref) <= 1e-12 * np.linalg.norm(ref)
    assert np.abs(ref).max() > 0
