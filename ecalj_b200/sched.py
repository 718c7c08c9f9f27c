"""Sigma_c task scheduling on the host: the real-axis window and pole-state
bounds of ``get_nwx`` (sxcf_fal2_count.sc.f90:238-298) and the pole-entry
census the library's correlation kernel will use (m_sxcf_gemm.f90:511-552).
Vectorised numpy; energies in Ry, we in Hartree.
"""
import numpy as np
from scipy.special import erfc

WFACCUT = 1e-8
DDW = 10.0


def _wfacx2(e1, e2, ek, esmr):
    el, eh = np.minimum(e1, e2), np.maximum(e1, e2)
    w = 0.5 * erfc(-(eh - ek) / np.sqrt(2.0) / esmr) - 0.5 * erfc(-(el - ek) / np.sqrt(2.0) / esmr)
    return np.where(eh - el < 1e-6, 0.0, w)


def _weavx2(e1, e2, ek, esmr):
    el, eh = np.minimum(e1, e2), np.maximum(e1, e2)
    wtt = 0.5 * erfc(-(eh - ek) / np.sqrt(2.0) / esmr) - 0.5 * erfc(-(el - ek) / np.sqrt(2.0) / esmr)
    sig2 = 2.0 * esmr ** 2
    return ek + esmr / np.sqrt(2.0 * np.pi) * (-np.exp(-(eh - ek) ** 2 / sig2)
                                               + np.exp(-(el - ek) ** 2 / sig2)) / wtt


def _wfac_levels(omg, ef, e, it, nctot, esmr):
    """wfacx2(omg, ef, e, esmrx) per level (wfacx.f90:19-36): core levels (it <= nctot) take
    esmrx = 0, the sharp window el <= e < eh; both vanish when |omg - ef| < 1e-6."""
    el, eh = min(omg, ef), max(omg, ef)
    if eh - el < 1e-6:
        return np.zeros(len(e))
    sharp = ((el <= e) & (e < eh)).astype(float)
    return np.where(it <= nctot, sharp, _wfacx2(omg, ef, e, esmr))


def nt0pm(ekc, ef, esmr):
    ekc = np.asarray(ekc)
    return int(np.sum(ekc < ef + DDW * esmr)), int(np.sum(ekc < ef - DDW * esmr))


def get_nwx(omega, ekc, freq_r, ef, esmr, nctot=0, nstate=None):
    """(nwxi, nwx, nt_max) for nw_i = 0 (valence smearing esmr; cores sharp)."""
    omega = np.asarray(omega); ekc = np.asarray(ekc); fr = np.asarray(freq_r)
    nw = len(fr) - 1
    nstate = len(ekc) if nstate is None else nstate
    nt0p, nt0m = nt0pm(ekc, ef, esmr)
    ixsmx = ixsmin = 0
    for omg in omega:
        lo, hi = (1, nt0p) if omg < ef else (nt0m + 1, nstate)
        if hi < lo:
            continue
        it = np.arange(lo, hi + 1)
        e = ekc[it - 1]
        keep = _wfac_levels(omg, ef, e, it, nctot, esmr) >= WFACCUT
        if not np.any(keep):
            continue
        we = np.abs(0.5 * (_weavx2(omg, ef, e[keep], esmr) - omg))
        ixs = np.minimum(np.searchsorted(fr[1:nw + 1], we, side='right') + 1, nw)
        m = int(ixs.max())
        if omg >= ef:
            ixsmx = max(ixsmx, m)
        else:
            ixsmin = max(ixsmin, m)
    nwx = max(ixsmx + 1, ixsmin + 1)
    if nwx > nw:
        raise ValueError("get_nwx: |w-e| beyond the real-axis mesh")
    nt_max = nt0p
    for omg in omega:
        if omg > ef:
            it = np.arange(nt0m + 1, nstate + 1)
            wf = _wfacx2(ef, omg, ekc[it - 1], esmr)
            hit = it[wf > WFACCUT]
            if len(hit):
                nt_max = max(nt_max, int(hit.max()))
    return 0, nwx, nt_max


def pole_bins(omega, ekc, freq_r, ef, esmr, nwxi, nwx, ns2r, nm, ntq, ns1=1, nctot=0, wkkr=1.0):
    """List of (column, ixs) of the pole entries (itp outer, it inner) and
    the real-axis records they touch inside [nwxi, nwx]."""
    omega = np.asarray(omega); ekc = np.asarray(ekc); fr = np.asarray(freq_r)
    nw = len(fr) - 1
    nt0p, nt0m = nt0pm(ekc, ef, esmr)
    ent = []
    for itp in range(1, ntq + 1):
        omg = omega[itp - 1]
        itini = max(ns1, nt0m + 1) if omg >= ef else ns1
        itend = ns2r if omg >= ef else min(nt0p, ns2r)
        if itend < itini:
            continue
        it = np.arange(itini, itend + 1)
        e = ekc[it - 1]
        keep = _wfac_levels(omg, ef, e, it, nctot, esmr) >= WFACCUT
        we = 0.5 * np.abs(omg - _weavx2(omg, ef, e[keep], esmr))
        ixs = np.searchsorted(fr[1:nw + 1], we, side='right') + 1
        for i, x in zip(it[keep], ixs):
            ent.append(((i - ns1) + nm * (itp - 1), int(x)))
    recs = sorted({x - 1 + j for _, x in ent for j in range(3) if nwxi <= x - 1 + j <= nwx})
    return ent, recs
