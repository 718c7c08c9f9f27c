"""Sigma task scheduling on the host, as sxcf_scz_count prepares it: the task
list over (kx, irot, ip, isp) with its middle-state batches and their size
from the memory budget (sxcf_fal2_count.sc.f90:86-230), the real-axis window
and pole-state bounds of ``get_nwx`` (:238-298), and the pole-entry census the
library's correlation kernel will use (m_sxcf_gemm.f90:511-552).  Vectorised
numpy; energies in Ry, we in Hartree.
"""
import math

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


def nmbatch_size(nstatemax_max, mmax_gb, ngcgp, nbandmx_max, nbloch, ngcmx):
    """Middle states per batch from the MEMnmbatch budget (GWinput, GB; default 2),
    sxcf_fal2_count.sc.f90:130-141: the budget less 16 ngcgp max(nbandmx) bytes,
    over max(nbandmx) (nbloch + 2 ngcmx) complex(8), at most max(nstatemax)."""
    k3 = 1000.0 ** 3
    mmm = max(mmax_gb - 16.0 * (ngcgp * nbandmx_max) / k3, 0.0)
    n = math.floor(min(nstatemax_max + 1e-8, mmm * k3 / (nbandmx_max * (nbloch + ngcmx + ngcmx) * 16) + 1e-8))
    if n == 0:
        raise ValueError("nmbatch = 0: the MEMnmbatch budget is too small")
    return n


def middle_batches(nnn, nmbatch):
    """The [nstti, nstte] ranges (1-based, inclusive) that cut nnn middle states
    into max((nnn-1)/nmbatch + 1, 1) nearly equal batches, the first nnn mod ndiv
    of them one state larger (sxcf_fal2_count.sc.f90:147-159)."""
    ndiv = max(int((nnn - 1) / nmbatch) + 1, 1)          # Fortran division truncates toward zero
    nloadav = nnn // ndiv
    nrem = nnn - ndiv * nloadav
    nload = [nloadav + 1] * nrem + [nloadav] * (ndiv - nrem)
    ends = np.cumsum(nload)
    return [(int(e - n + 1), int(e)) for n, e in zip(nload, ends)]


def sigma_tasks(irkip, nstatemax, nmbatch):
    """The icount list of sxcf_scz_count (sxcf_fal2_count.sc.f90:86-230): every
    nonzero irkip(isp, kx, irot, ip) (a numpy array of that Fortran index order,
    0-based here) in the loop order kx, irot, ip, isp, each cut into its
    middle-state batches.  nstatemax(isp, kx, irot, ip, kr) gives the middle-state
    count of a task (nt0p for exchange, nctot + min(nband, ...) for correlation).
    Returns dicts with 1-based isp, kx, irot, ip, kr, nstti, nstte."""
    irkip = np.asarray(irkip)
    nspin, nqibz, ngrp, nqip = irkip.shape
    tasks = []
    for kx in range(nqibz):
        if not irkip[:, kx].any():
            continue
        for irot in range(ngrp):
            if not irkip[:, kx, irot].any():
                continue
            for ip in range(nqip):
                for isp in range(nspin):
                    kr = int(irkip[isp, kx, irot, ip])
                    if kr == 0:
                        continue
                    nnn = nstatemax(isp + 1, kx + 1, irot + 1, ip + 1, kr)
                    for (a, b) in middle_batches(nnn, nmbatch):
                        tasks.append(dict(isp=isp + 1, kx=kx + 1, irot=irot + 1, ip=ip + 1, kr=kr, nstti=a, nstte=b))
    return tasks
