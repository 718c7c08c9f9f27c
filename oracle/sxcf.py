"""Correlation self-energy: restatement of the ``get_correlation_block`` of
``sxcf_scz_correlation`` plus ``wfacx2``/``weavx2``, ``get_nwx`` and the
exchange block.  Test infrastructure only (see package doc).

Units follow the reference: eigenvalues ``omega``/``ekc``/``ef``/``esmr`` in
Ry, ``we = (omega - e)/2`` in Hartree (m_sxcf_gemm.f90:436), Sigma in Hartree.
"""
import math
import numpy as np
from scipy.special import erfc

PI = 4.0 * math.atan(1.0)
RMAX = 2.0          # m_sxcf_gemm.f90:120
WFACCUT = 1e-8      # m_sxcf_gemm.f90:408
DDW = 10.0          # m_sxcf_gemm.f90:264


def _sign1(x):
    """Fortran dsign(1d0, x)."""
    return -1.0 if math.copysign(1.0, x) < 0 else 1.0


def wfacx2(e1, e2, ek, esmr):
    """SRC/subroutines/wfacx.f90:19-36."""
    el, eh = min(e1, e2), max(e1, e2)
    if eh - el < 1e-6:
        return 0.0
    if esmr == 0.0:
        return 1.0 if (el <= ek < eh) else 0.0
    return (0.5 * erfc(-(eh - ek) / math.sqrt(2.0) / esmr)
            - 0.5 * erfc(-(el - ek) / math.sqrt(2.0) / esmr))


def weavx2(e1, e2, ek, esmr):
    """SRC/subroutines/wfacx.f90:39-49."""
    el, eh = min(e1, e2), max(e1, e2)
    wtt = (0.5 * erfc(-(eh - ek) / math.sqrt(2.0) / esmr)
           - 0.5 * erfc(-(el - ek) / math.sqrt(2.0) / esmr))
    sig2 = 2.0 * esmr ** 2
    pi = 3.1415926535897932
    return ek + esmr / math.sqrt(2.0 * pi) * (-math.exp(-(eh - ek) ** 2 / sig2)
                                              + math.exp(-(el - ek) ** 2 / sig2)) / wtt


def wgtim(omega, ekc, nctot, ns1, ns2, ntqxx, esmr, wkkr, ua, x, wt, expa):
    """Imaginary-axis weights wgtim(0:niw, ns1:ns2, ntqxx), npm = 1
    (SRC/subroutines/m_sxcf_gemm.f90:432-458).  Returns float64
    (niw+1, ns2-ns1+1, ntqxx)."""
    x = np.asarray(x, np.float64); wt = np.asarray(wt, np.float64)
    expa = np.asarray(expa, np.float64)
    niw = len(x)
    sig2 = 2.0 * (0.5 * esmr) ** 2                                  # :433
    out = np.zeros((niw + 1, ns2 - ns1 + 1, ntqxx))
    for itp in range(1, ntqxx + 1):
        for it in range(ns1, ns2 + 1):
            we = 0.5 * (omega[itp - 1] - ekc[it - 1])               # :436
            aw = abs(ua * we); aw2 = aw * aw
            w = np.zeros(niw + 1)
            if it <= nctot:                                          # :439
                cons = 1.0 / (we ** 2 * x ** 2 + (1.0 - x) ** 2)
                w[1:] = we * cons * wt * (-1.0 / PI)
                if abs(we) < RMAX / ua:
                    w[0] = (-np.sum(w[1:] * expa) - 0.5 * _sign1(we)
                            * math.exp(we ** 2 * ua ** 2) * erfc(ua * abs(we)))
                else:
                    w[0] = 0.0
            else:
                omd = 1.0 / x - 1.0                                   # :446
                omd2w = omd ** 2 + we ** 2
                r = omd2w / sig2
                cons = np.where(r > 5e-3, (1.0 - np.exp(-r)) / omd2w,
                                (1.0 / sig2 - omd2w / sig2 ** 2 / 2.0
                                 + omd2w ** 2 / sig2 ** 3 / 6.0
                                 - omd2w ** 3 / sig2 ** 4 / 24.0
                                 + omd2w ** 4 / sig2 ** 5 / 120.0
                                 - omd2w ** 5 / sig2 ** 6 / 720.0))
                w[1:] = -we * cons * wt / (x ** 2) / PI              # :451
                w[0] = (we * np.sum(cons * expa * wt / (x ** 2)) / PI
                        + _sign1(we) * 0.5 * math.exp(aw2)
                        * (erfc(math.sqrt(aw2 + we ** 2 / sig2)) - erfc(aw)))
            out[:, it - ns1, itp - 1] = wkkr * w                      # :456
    return out


def inverse33(m):
    """m_sxcf_gemm.f90:658-668 (cofactor inverse)."""
    inv = np.empty((3, 3))
    inv[:, 0] = np.cross(m[:, 1], m[:, 2])
    inv[:, 1] = np.cross(m[:, 2], m[:, 0])
    inv[:, 2] = np.cross(m[:, 0], m[:, 1])
    det = np.sum(m[:, 0] * inv[:, 0])
    return inv.T / det


def nt0pm(ekc, ef, esmr):
    """nt0p, nt0m of m_sxcf_gemm.f90:382-383."""
    ekc = np.asarray(ekc)
    return int(np.sum(ekc < ef + DDW * esmr)), int(np.sum(ekc < ef - DDW * esmr))


def pole_table(omega, ekc, nctot, ns1, ns2r, ntqxx, ef, esmr, wkkr, freq_r):
    """Real-axis pole entries (m_sxcf_gemm.f90:529-552): list of
    (it, itp, ixs, wgt3[3]) in the reference's (itp, it) loop order; the three
    weights land on freq_r indices ixs-1, ixs, ixs+1 (0-based = Fortran)."""
    freq_r = np.asarray(freq_r)
    nw = len(freq_r) - 1
    nt0p, nt0m = nt0pm(ekc, ef, esmr)
    ent = []
    for itp in range(1, ntqxx + 1):
        omg = omega[itp - 1]
        itini = max(ns1, nt0m + 1) if omg >= ef else ns1            # :532
        itend = ns2r if omg >= ef else min(nt0p, ns2r)              # :533
        for it in range(itini, itend + 1):
            wf = wfacx2(omg, ef, ekc[it - 1], 0.0 if it <= nctot else esmr)
            if wf < WFACCUT:
                continue
            wf = wf * wkkr * _sign1(omg - ef)                        # :537
            we = 0.5 * abs(omg - weavx2(omg, ef, ekc[it - 1], esmr))
            hit = np.nonzero(freq_r[1:nw + 1] > we)[0]
            if len(hit) == 0:
                raise ValueError("pole frequency beyond freq_r(nw)")
            ixs = int(hit[0]) + 1                                    # findloc, 1-based in 1..nw
            xi = freq_r[ixs - 1:ixs + 2]
            amat = np.stack([np.ones(3), xi ** 2, xi ** 4], axis=1)
            w3 = wf * (np.array([1.0, we ** 2, we ** 4]) @ inverse33(amat))
            ent.append((it, itp, ixs, w3))
    return ent


def get_nwx(omega, ntqxx, nt0p, nt0m, nstate, freq_r, esmr, ef, ekc, nctot):
    """SRC/subroutines/sxcf_fal2_count.sc.f90:238-298 (nw_i = 0).
    Returns (nwxi, nwx, nt_max)."""
    freq_r = np.asarray(freq_r)
    nw = len(freq_r) - 1
    ixsmx = 0; ixsmin = 0; ixs = -9999
    for itp in range(1, ntqxx + 1):
        omg = omega[itp - 1]
        if omg < ef:
            itini, itend = 1, nt0p
        else:
            itini, itend = nt0m + 1, nstate
        for it in range(itini, itend + 1):
            esmrx = 0.0 if it <= nctot else esmr
            wf = wfacx2(omg, ef, ekc[it - 1], esmrx)
            if wf < WFACCUT:
                continue
            we = 0.5 * (weavx2(omg, ef, ekc[it - 1], esmr) - omg)
            for iwp in range(1, nw + 1):
                ixs = iwp
                if freq_r[iwp] > abs(we):
                    break
            if ixs > ixsmx and omg >= ef:
                ixsmx = ixs
            if ixs > ixsmin and omg < ef:
                ixsmin = ixs
    nwxi = 0
    nwx = max(ixsmx + 1, ixsmin + 1)
    if nwx > nw:
        raise ValueError("get_nwx: |w-e| > max(w)")
    nt_max = nt0p
    for itp in range(1, ntqxx + 1):
        omg = omega[itp - 1]
        if omg > ef:
            for it in range(nt0m + 1, nstate + 1):
                if wfacx2(ef, omg, ekc[it - 1], esmr) > WFACCUT and it > nt_max:
                    nt_max = it
    return nwxi, nwx, nt_max


def correlation_block(zsec, zmel, ns1, ns2, ns2r, nwxi, nwx, ntqxx,
                      wc_imag, wc_real, omega, ekc, nctot, ef, esmr, wkkr,
                      ua, x, wt, expa, freq_r, keepwv=False):
    """In-place restatement of m_sxcf_gemm.f90:407-612 for one task.

    zsec     complex128 (ntq, ntq), accumulated, diagonal Im clamped <= 0
    zmel     complex128 (ngb, ns2-ns1+1, ntqxx), M basis, not conjugated
    wc_imag  complex128 (ngb, ngb, niw+1): slot 0 = W(omega=0)-v (the first
             __WVR record), slots 1..niw = __WVI records
    wc_real  complex128 (ngb, ngb, nw+1): __WVR records (symmetrised here)
    keepwv   True reproduces the packed-upper-triangle path (:327-358, 467-475)
    """
    if ns1 > ns2:
        return zsec
    ngb = zmel.shape[0]
    niw = len(x)
    nm = ns2 - ns1 + 1
    wg = wgtim(omega, ekc, nctot, ns1, ns2, ntqxx, esmr, wkkr, ua, x, wt, expa)
    iu = np.triu_indices(ngb)
    czmelwc = np.zeros(zmel.shape, np.complex128, order='F')
    for iw in range(0, niw + 1):                                        # :463
        wv = wc_imag[:, :, iw]
        if keepwv:
            up = wv[iu]
            wc = np.zeros((ngb, ngb), np.complex128)
            wc[iu] = up
            wc[(iu[1], iu[0])] = np.conj(up)
        else:
            wc = wv
        wzmel = np.asfortranarray(zmel * wg[iw][None, :, :])              # :485
        czmelwc += (wc.conj().T @ wzmel.reshape(ngb, -1, order='F')).reshape(
            zmel.shape, order='F')                                        # :492
    ent = pole_table(omega, ekc, nctot, ns1, ns2r, ntqxx, ef, esmr, wkkr, freq_r)
    bins = {}
    for (it, itp, ixs, w3) in ent:
        for i in range(3):
            bins.setdefault(ixs - 1 + i, []).append((it, itp, w3[i]))
    nw = wc_real.shape[2] - 1
    for iw in range(0, nw + 1):                                           # :556
        if iw < nwxi or iw > nwx or iw not in bins:
            continue
        wv = wc_real[:, :, iw]
        wc = (wv + wv.conj().T) * 0.5                                     # :573
        for (it, itp, w) in bins[iw]:                                     # :578-588
            czmelwc[:, it - ns1, itp - 1] += wc.conj().T @ (w * zmel[:, it - ns1, itp - 1])
    k = ngb * nm
    zsec[:ntqxx, :ntqxx] += (czmelwc.reshape(k, ntqxx, order='F').conj().T
                             @ zmel.reshape(k, ntqxx, order='F'))          # :599
    for itp in range(ntqxx):                                              # :602-607
        im = zsec[itp, itp].imag
        if im > 0.0:
            im = 0.0
        zsec[itp, itp] = complex(zsec[itp, itp].real, im)
    return zsec


def wfacx(el, eh, ek, esmr):
    """SRC/subroutines/wfacx.f90:3-13."""
    if esmr == 0.0:
        return 1.0 if (el <= ek < eh) else 0.0
    return (0.5 * erfc(-(eh - ek) / math.sqrt(2.0) / esmr)
            - 0.5 * erfc(-(el - ek) / math.sqrt(2.0) / esmr))


def exchange_block(zsec, zmel, ns1, ns2, ntqxx, vcoud, ekc, nctot, ef, esmr, wkkr):
    """In-place restatement of get_exchange_block (m_sxcf_gemm.f90:203-231):

        wtff(it) = 1 (core) | wfacx(-1d99, ef, ekc(it+nctot), esmr) (valence)
        zsec += -wkkr * zmel^H (wtff * vcoud * zmel)   over K = (ngb, it)

    zmel is (ngb, ns2-ns1+1, ntqxx) in the E basis (is_m_basis=.false.);
    ``vcoud`` is the effective Coulomb eigenvalue vector (the caller applies
    the kx == 1 head replacement of :218)."""
    if ns1 > ns2:
        return zsec
    nm = ns2 - ns1 + 1
    wtff = np.array([1.0 if it <= nctot else wfacx(-1e99, ef, ekc[it + nctot - 1], esmr)
                     for it in range(ns1, ns2 + 1)])
    vz = zmel * np.asarray(vcoud)[:, None, None] * wtff[None, :, None]
    k = zmel.shape[0] * nm
    zsec[:ntqxx, :ntqxx] += -wkkr * (zmel.reshape(k, ntqxx, order='F').conj().T
                                     @ vz.reshape(k, ntqxx, order='F'))
    return zsec
