"""Generates tests/golden/golden.npz: small seeded cases of every oracle
routine (x0gemm, WVIllwI, the Sigma_c correlation block, the imaginary-axis
weights).  The reference Fortran cannot be built here, so these fixtures are
outputs of the oracle restatement; they pin the oracle (and, in the GPU
tests, the kernels) against regressions.

    python -m tests.golden.make_golden
"""
import os

import numpy as np

from oracle import llw, sxcf, x0
from ecalj_b200 import synth

HERE = os.path.dirname(os.path.abspath(__file__))


def inputs():
    """The seeded inputs shared by the golden computation and the GPU tests."""
    rng = np.random.default_rng(2026)
    d = {}
    # x0gemm, npm = 2 with a partial column range
    nbb, nm1, nm2, nqtot, nwhis, ncoun = 70, 1, 9, 11, 5, 120
    z = np.asfortranarray(rng.standard_normal((nbb, nm2 - nm1 + 1, nqtot))
                          + 1j * rng.standard_normal((nbb, nm2 - nm1 + 1, nqtot)))
    itc = rng.integers(nm1, nm2 + 1, ncoun).astype(np.int32)
    itpc = rng.integers(1, nqtot + 1, ncoun).astype(np.int32)
    jpmc = rng.integers(1, 3, ncoun).astype(np.int32)
    iwini = rng.integers(1, nwhis + 1, ncoun).astype(np.int32)
    iwend = np.minimum(nwhis, iwini + rng.integers(0, 3, ncoun)).astype(np.int32)
    nh = iwend - iwini + 1
    icouini = np.concatenate([[1], np.cumsum(nh)[:-1] + 1]).astype(np.int32)
    whwc = rng.uniform(-1, 1, int(nh.sum()))
    d['x0'] = dict(z=z, itc=itc, itpc=itpc, jpmc=jpmc, iwini=iwini, iwend=iwend, icouini=icouini,
                   whwc=whwc, nbb=nbb, nm1=nm1, nqtot=nqtot, nwhis=nwhis, ncoun=ncoun,
                   npr=70, ipr_col=1, npr_col=70, ns1=2, ns2=8)
    # W
    n, niw = 48, 4
    vsq, q = synth.coulomb(n, 31)
    g = rng.standard_normal((n, 12)) + 1j * rng.standard_normal((n, 12))
    chi = np.zeros((n, n, niw), complex, order='F')
    for iw in range(niw):
        gg = g * 0.05 / (iw + 1)
        chi[:, :, iw] = -gg @ gg.conj().T
    d['wv'] = dict(chi=chi, vsq=vsq, q=q)
    # Sigma_c
    ngb, ntq, nm, nreal = 40, 6, 25, 30
    t = synth.sigc_task(ngb, ntq, nm, niw, nreal, seed=77, nctot=2, esmr=0.02, ef=0.05)
    wi = np.asfortranarray(rng.standard_normal((ngb, ngb, niw + 1)) + 1j * rng.standard_normal((ngb, ngb, niw + 1))) * 0.1
    wr = np.asfortranarray(rng.standard_normal((ngb, ngb, nreal)) + 1j * rng.standard_normal((ngb, ngb, nreal))) * 0.1
    zz = np.asfortranarray(rng.standard_normal((ngb, nm + 2, ntq)) + 1j * rng.standard_normal((ngb, nm + 2, ntq)))
    d['sc'] = dict(t=t, wi=wi, wr=wr, z=zz, ngb=ngb, ntq=ntq, nm=nm + 2, niw=niw)
    return d


def sigc_window(t, ntq):
    ekc = t['ekc']
    nt0p, nt0m = sxcf.nt0pm(ekc, t['ef'], t['esmr'])
    nwxi, nwx, ntmax = sxcf.get_nwx(t['omega'], ntq, nt0p, nt0m, len(ekc), t['freq_r'], t['esmr'],
                                    t['ef'], ekc, t['nctot'])
    return nwxi, nwx, ntmax


def compute_all():
    d = inputs()
    out = {}
    a = d['x0']
    r = np.zeros((a['npr'], a['npr_col'], 2 * a['nwhis'] + 1), complex, order='F')
    x0.x0gemm(r, a['npr'], a['ipr_col'], a['npr_col'], a['nwhis'], 2, a['ns1'], a['ns2'], a['z'], a['nm1'],
              1, a['ncoun'], a['itc'], a['itpc'], a['jpmc'], a['iwini'], a['iwend'], a['icouini'], a['whwc'])
    out['x0_rcxq'] = r
    w = d['wv']
    out['wv_zw'] = llw.wvi_llw(w['chi'].copy(order='F'), 2, w['vsq'], w['q'], True, True, 3)
    s = d['sc']; t = s['t']
    nwxi, nwx, ntmax = sigc_window(t, s['ntq'])
    zs = np.zeros((s['ntq'], s['ntq']), complex, order='F')
    sxcf.correlation_block(zs, s['z'], 1, s['nm'], min(s['nm'], ntmax), nwxi, nwx, s['ntq'], s['wi'], s['wr'],
                           t['omega'], t['ekc'], t['nctot'], t['ef'], t['esmr'], 1.0 / 64, t['ua'],
                           t['x'], t['wx'], t['expa'], t['freq_r'])
    out['sc_zsec'] = zs
    out['sc_wgtim'] = sxcf.wgtim(t['omega'], t['ekc'], t['nctot'], 1, s['nm'], s['ntq'], t['esmr'], 1.0 / 64,
                                 t['ua'], t['x'], t['wx'], t['expa'])
    return out


if __name__ == "__main__":
    np.savez_compressed(os.path.join(HERE, "golden.npz"), **compute_all())
    print("wrote", os.path.join(HERE, "golden.npz"))
