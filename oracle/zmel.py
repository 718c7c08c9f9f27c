"""Product-basis matrix elements <psi|psi M>: restatement of the muffin-tin
part, the interstitial plane-wave part and the M->E change of
get_zmel_init_gemm.  Test infrastructure only."""
import numpy as np


def zmel_mt(cphim, cphiq, ppb, atoms, nbloch, nm1, nm2, nctot, ntp0, phase):
    """SRC/subroutines/m_zmel.f90:323-390 (ncc = 0).

    cphim  complex128 (ndima, nm2v-nm1v+1) valence coefficients at q-k for
           states nm1v..nm2v (rows: all atoms' l,n,m valence channels)
    cphiq  complex128 (ndima, ntp0) at q
    ppb    list over atoms of float64/complex (nlnm, nlnm, mdim): rows/cols are
           core channels 1..nc followed by valence nc+1..nc+nv (:110-145)
    atoms  list of dicts with keys nc, nv, ias (1-based start of the atom's
           valence rows in cphim/cphiq), ics (core offset), ims (1-based start
           of its product-basis rows), ncore (core states of the atom)
    phase  complex (natom,) = exp(-i 2pi kvec.tr) (:325)
    Returns zmelt complex128 (nbloch, nm2-nm1+1, ntp0) with the MT rows set.
    """
    nm = nm2 - nm1 + 1
    zt = np.zeros((nbloch, nm, ntp0), np.complex128)
    if nm1 > nctot:
        nm1c, nm2c, nm1v, nm2v = 0, -1, nm1, nm2
    elif nm2 > nctot:
        nm1c, nm2c, nm1v, nm2v = nm1, nctot, nctot + 1, nm2
    else:
        nm1c, nm2c, nm1v, nm2v = nm1, nm2, 0, -1
    for ia, at in enumerate(atoms):
        nc, nv, ias, ics, ims = at['nc'], at['nv'], at['ias'], at['ics'], at['ims']
        p = ppb[ia]
        mdim = p.shape[2]
        cq = cphiq[ias - 1:ias - 1 + nv, :]                                 # (nv, ntp0)
        if nm2v >= nm1v:                                                     # :355
            cm = cphim[ias - 1:ias - 1 + nv, nm1v - nm1v: nm2v - nm1v + 1]  # (nv, nmv)
            pv = p[nc:nc + nv, nc:nc + nv, :]                                # ppb(nc1:ncnv, nc1:ncnv, i)
            t = np.einsum('bai,bq->aqi', pv, cq)                            # ppbv^T cphiq   :358
            z = phase[ia] * np.einsum('at,aqi->tqi', cm.conj(), t)          # :365
            for i in range(mdim):
                zt[ims - 1 + i, nm1v - nm1:nm2v - nm1 + 1, :] = z[:, :, i]
        ncorec = at['ncore'] if nctot > 0 else 0
        nm1cc = max(nm1c, ics + 1); nm2cc = min(nm2c, ics + ncorec)         # :376
        if nm2cc >= nm1cc:
            for it in range(nm1cc, nm2cc + 1):
                pc = p[nc:nc + nv, it - ics - 1, :]                          # ppb(nc1:ncnv, it-ics, i)
                z = phase[ia] * np.einsum('bi,bq->iq', pc, cq)              # :383
                zt[ims - 1:ims - 1 + mdim, it - nm1, :] = z
    return zt


def zmel_m2e(zmelt, m2e, is_m_basis, zmelconjg):
    """m_zmel.f90:546-563 and 590-594: zmel = m2e^H zmelt (E basis) or a copy
    (M basis), then conj when zmelconjg."""
    ngb, nm, nt = zmelt.shape
    if is_m_basis:
        z = zmelt.copy()
    else:
        z = (m2e.conj().T @ zmelt.reshape(ngb, nm * nt, order='F')).reshape(
            m2e.shape[1], nm, nt, order='F')
    return z.conj() if zmelconjg else z


def zmel_ipw(geigq, dgeigqk, ngvecpB1, ngvecpB2, ngveccR, nvggg, ggg, nadd, phase):
    """SRC/subroutines/m_zmel.f90:418-535, the definition both of its branches
    (G1 integral first, :439-480, or G2 first, :481-524) evaluate:

        zmelp0(igc, it, itp) = sum_{G1, G2} ggg(G1 - (Gc + G2) - nadd)
                                * geigq(G1, itp) * dgeigqk(G2, it)
        rows nbloch+igc of zmelt = phase(igc) * zmelp0            (:528-532)

    ggg(v) is the entry of nvggg equal to v, zero when v is absent (the
    reference skips igggi <= 0, :453-454).
    geigq (ngp1, ntp0), dgeigqk (ngp2, nmv) complex (dgeigqk already conj'ed);
    ngvecpB1 (3, ngp1), ngvecpB2 (3, ngp2), ngveccR (3, ngc), nvggg (3, nggg)
    integer; returns (ngc, nmv, ntp0) complex128."""
    lut = {tuple(int(c) for c in nvggg[:, i]): ggg[i] for i in range(nvggg.shape[1])}
    ngc, ngp1, ngp2 = ngveccR.shape[1], ngvecpB1.shape[1], ngvecpB2.shape[1]
    nadd = np.asarray(nadd)
    out = np.zeros((ngc, dgeigqk.shape[1], geigq.shape[1]), np.complex128)
    for igc in range(ngc):
        m = np.zeros((ngp1, ngp2), np.complex128)               # m(G1, G2) = ggg(G1 - Gc - G2 - nadd)
        for a in range(ngp1):
            for b in range(ngp2):
                v = ngvecpB1[:, a] - ngveccR[:, igc] - ngvecpB2[:, b] - nadd
                m[a, b] = lut.get(tuple(int(c) for c in v), 0.0)
        out[igc] = phase[igc] * (dgeigqk.T @ m.T @ geigq)      # (nmv, ntp0)
    return out
