"""chi0 rank-k accumulation: restatement of ``x0gemm`` and of the pair tables
that ``X0kf_v4hz_init`` hands it.  Test infrastructure only (see package doc).

Conventions: every array is a numpy array whose axes are the Fortran axes in
the same order; Fortran lower bounds are passed explicitly and subtracted.
"""
import numpy as np


def rcxq_slab(iw, jpm, nwhis, npm):
    """Python index of slab ``rcxq(:,:,iw*(3-2*jpm))`` of an array declared
    ``rcxq(npr,npr_col,(1-npm)*nwhis:nwhis)`` (x0gemm.f90:27,88)."""
    return iw * (3 - 2 * jpm) - (1 - npm) * nwhis


def x0gemm(rcxq, npr, ipr_col, npr_col, nwhis, npm, ns1, ns2,
           zmel, nm1, icounkmink, icounkmaxk,
           itc, itpc, jpmc, iwini, iwend, icouini, whwc):
    """In-place restatement of SRC/subroutines/x0gemm.f90:2-97.

    rcxq    complex128 (npr, npr_col, nslab), accumulated (beta = 1, :88-89)
    zmel    complex128 (nbb, nm2-nm1+1, nqtot); Fortran second index starts at nm1
    icoun*  1-based pair indices, itc/itpc/jpmc/iwini/iwend/icouini are the
            1-based Fortran integer tables of m_x0kf; whwc the weights.

    The pair order inside each (jpm, iw) bin is the icoun order (:52-64); the
    bin product is rcxq(:,:,slab) += zw^H wzw with zw(ittp, igb1) =
    zmel(igb1, it, itp) and wzw(ittp, igb2) = zmel(igb2+ipr_col-1, it, itp) *
    whw(ittp) (:72-89).
    """
    itc = np.asarray(itc); itpc = np.asarray(itpc); jpmc = np.asarray(jpmc)
    iwini = np.asarray(iwini); iwend = np.asarray(iwend)
    icouini = np.asarray(icouini); whwc = np.asarray(whwc, dtype=np.float64)
    lists = {}
    for icoun in range(icounkmink, icounkmaxk + 1):        # :52
        c = icoun - 1
        jpm = int(jpmc[c]); it = int(itc[c]); itp = int(itpc[c])
        if it < ns1 or it > ns2:                            # :56
            continue
        for iw in range(int(iwini[c]), int(iwend[c]) + 1):  # :57
            w = whwc[iw - iwini[c] + icouini[c] - 1]        # :62
            lists.setdefault((jpm, iw), []).append((it, itp, w))
    for jpm in range(1, npm + 1):                           # :69
        for iw in range(1, nwhis + 1):                      # :70
            lst = lists.get((jpm, iw))
            if not lst:                                     # :71
                continue
            its = np.array([e[0] - nm1 for e in lst])
            itps = np.array([e[1] - 1 for e in lst])
            ws = np.array([e[2] for e in lst])
            zcols = zmel[:, its, itps]                      # (nbb, nttp)
            zw = zcols[:npr, :].T                           # (nttp, npr)   :76
            wzw = (zcols[ipr_col - 1:ipr_col - 1 + npr_col, :] * ws).T   # :84
            rcxq[:, :, rcxq_slab(iw, jpm, nwhis, npm)] += zw.conj().T @ wzw  # :88
    return rcxq


def lorentz_pair_tables(eocc, eunocc, niw, freq_i, nk):
    """Pair tables in the ``m_x0kf`` format for the direct imaginary-axis
    Lorentzian form used by the synthetic configs: every (k, occ, unocc) pair
    covers all niw "bins" (iwini=1, iwend=niw, jpm=1) with weight

        whw(pair, iw) = -2 de / (de^2 + w_iw^2) / nk,   de = e_unocc - e_occ

    (the minus sign is the reference's sign convention, chi0(iw) <= 0,
    dpsion5.f90:215-220).  This is the stand-in for the tetrahedron weights
    of m_tetwt.f90:36-256 (index layout of x0kf_v4h.f90:118-133).

    eocc    list over k of (nocc_k,) arrays,  eunocc list over k of (nun_k,)
    Returns per-k dicts with itc, itpc, jpmc, iwini, iwend, icouini, whwc
    (1-based, one dict per k, icoun restarting at 1).
    """
    out = []
    for k in range(len(eocc)):
        eo = np.asarray(eocc[k]); eu = np.asarray(eunocc[k])
        no, nu = len(eo), len(eu)
        it = np.repeat(np.arange(1, no + 1), nu)
        itp = np.tile(np.arange(1, nu + 1), no)
        de = (eu[itp - 1] - eo[it - 1])
        w = -2.0 * de[:, None] / (de[:, None] ** 2 + np.asarray(freq_i)[None, :] ** 2) / nk
        npair = no * nu
        out.append(dict(itc=it.astype(np.int32), itpc=itp.astype(np.int32),
                        jpmc=np.ones(npair, np.int32),
                        iwini=np.ones(npair, np.int32),
                        iwend=np.full(npair, niw, np.int32),
                        icouini=(np.arange(npair) * niw + 1).astype(np.int32),
                        whwc=w.reshape(-1).copy()))
    return out


def chi0_direct(zmels, tables, npr, niw):
    """chi0(iw) for all k: loops x0gemm over k (x0kf_v4h.f90:233-290 with a
    single NMBATCH batch and npm=1).  zmels: list of (npr, nocc, nun) arrays
    (conjugated as get_zmel_init_gemm(zmelconjg=.true.) leaves them).
    Returns complex128 (npr, npr, niw+1); slab 0 stays zero (:190, 206)."""
    rcxq = np.zeros((npr, npr, niw + 1), np.complex128, order='F')
    for z, t in zip(zmels, tables):
        ncoun = len(t['itc'])
        x0gemm(rcxq, npr, 1, npr, niw, 1, 1, z.shape[1], z, 1, 1, ncoun,
               t['itc'], t['itpc'], t['jpmc'], t['iwini'], t['iwend'],
               t['icouini'], t['whwc'])
    return rcxq


def chi0_real(zcols, de, nk, freq_r, eta):
    """chi0 of the Lorentzian model on real frequencies (the stand-in for the
    histogram + Hilbert transform of dpsion5.f90:243-292):
        chi0(w) = conj(Z) diag(f) Z^T,  f = [1/(w - de + i eta) - 1/(w + de + i eta)] / nk,
    whose value at w = i nu is the imaginary-axis weight -2 de/(de^2 + nu^2)/nk.
    zcols (npr, npair) complex, de (npair,) Hartree; returns (npr, npr, nw)."""
    z = np.asarray(zcols)
    out = np.empty((z.shape[0], z.shape[0], len(freq_r)), np.complex128, order='F')
    for iw, w in enumerate(freq_r):
        f = (1.0 / (w - de + 1j * eta) - 1.0 / (w + de + 1j * eta)) / nk
        out[:, :, iw] = (z.conj() * f) @ z.T
    return out
