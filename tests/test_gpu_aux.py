"""FP64 parity of Sigma_x, the QP-energy / Hermitian-Sigma step and the
muffin-tin zmel kernel against the oracle (relative Frobenius <= 1e-11)."""
import numpy as np
import pytest

from oracle import hqpe, sxcf, zmel
from tests.conftest import rel_fro

pytestmark = pytest.mark.gpu
TOL = 1e-11


def _rc(rng, *shape):
    return np.asfortranarray(rng.standard_normal(shape) + 1j * rng.standard_normal(shape))


@pytest.mark.parametrize("nctot,esmr", [(0, 0.01), (3, 0.02), (2, 0.0)])
def test_exchange_vs_oracle(qsgw, nctot, esmr):
    rng = np.random.default_rng(7 + nctot)
    ngb, ntq, ntqxx, ns1, ns2 = 70, 9, 7, 1, 23
    z = _rc(rng, ngb, ns2 - ns1 + 1, ntqxx)
    vcoud = 10 ** rng.uniform(-2, 3, ngb)
    ekc = np.sort(rng.uniform(-1.5, 3.0, ns2 + nctot + 2))
    ef = 0.1
    ref = _rc(rng, ntq, ntq)
    got = qsgw.to_device(ref)
    sxcf.exchange_block(ref, z, ns1, ns2, ntqxx, vcoud, ekc, nctot, ef, esmr, 0.125)
    qsgw.sxcf_exchange_d(got, ntq, qsgw.to_device(z), ngb, ns1, ns2, ntqxx, vcoud, ekc, nctot, ef, esmr, 0.125)
    qsgw.synchronize()
    assert rel_fro(qsgw.from_device(got, (ntq, ntq)), ref) < TOL


def test_hqpe_vs_oracle(qsgw):
    rng = np.random.default_rng(3)
    ntq, ld, nq = 11, 13, 3
    mats = [_rc(rng, ld, ld, nq) * 0.1 for _ in range(4)]
    elda = np.asfortranarray(rng.uniform(-10, 10, (ntq, nq)))
    vxc = np.asfortranarray(rng.uniform(-5, 0, (ntq, nq)))
    d = [qsgw.to_device(m) for m in mats]
    de, dv = qsgw.to_device(elda), qsgw.to_device(vxc)
    import torch
    eqp = torch.zeros(ntq * nq, dtype=torch.float64, device='cuda')
    seh = torch.zeros(ld * ld * nq, dtype=torch.complex128, device='cuda')
    qsgw.hqpe_d(d[0], d[1], d[2], d[3], de, dv, ntq, ld, nq, eqp, seh)
    qsgw.synchronize()
    eqp = eqp.cpu().numpy().reshape(ntq, nq, order='F')
    seh = qsgw.from_device(seh, (ld, ld, nq))
    for q in range(nq):
        s = [m[:ntq, :ntq, q] for m in mats]
        assert rel_fro(eqp[:, q], hqpe.qp_energies(elda[:, q], s[0], s[1], s[2], vxc[:, q])) < TOL
        assert rel_fro(seh[:ntq, :ntq, q], hqpe.hermitian_sigma(s[0], s[1], s[2], s[3])) < TOL


def _zmel_case(rng, nctot):
    atoms = [dict(nc=2, nv=9, ias=1, ics=0, ims=1, ncore=2), dict(nc=1, nv=13, ias=10, ics=2, ims=31, ncore=1),
             dict(nc=0, nv=4, ias=23, ics=3, ims=56, ncore=0)]
    mdims = [30, 25, 12]
    nbloch = 75
    ppb = [rng.standard_normal((a['nc'] + a['nv'] + 1, a['nc'] + a['nv'] + 1, md)) for a, md in zip(atoms, mdims)]
    ph = np.exp(1j * rng.uniform(0, 6.28, len(atoms)))
    return atoms, nbloch, ppb, ph


@pytest.mark.parametrize("nm1,nm2,nctot", [(1, 37, 3), (5, 20, 3), (1, 3, 3), (1, 40, 0)])
def test_zmel_mt_and_m2e_vs_oracle(qsgw, nm1, nm2, nctot):
    import torch
    rng = np.random.default_rng(nm1 * 10 + nm2)
    atoms, nbloch, ppb, ph = _zmel_case(rng, nctot)
    ndima, ntp0 = 26, 21
    nm1v = max(nm1, nctot + 1)
    nmv = max(0, nm2 - nm1v + 1)
    cphim = _rc(rng, ndima, max(nmv, 1))
    cphiq = _rc(rng, ndima, ntp0)
    ref = zmel.zmel_mt(cphim, cphiq, ppb, atoms, nbloch, nm1, nm2, nctot, ntp0, ph)
    nm = nm2 - nm1 + 1
    zt = torch.zeros(nbloch * nm * ntp0, dtype=torch.complex128, device='cuda')
    dat = []
    for a, p_, f in zip(atoms, ppb, ph):
        d = dict(a); d['nlnm'] = p_.shape[0]; d['mdim'] = p_.shape[2]; d['phase'] = f
        d['ppb_d'] = torch.from_numpy(p_.reshape(-1, order='F').copy()).cuda()
        dat.append(d)
    qsgw.zmel_mt_d(zt, nbloch, nm1, nm2, nctot, ntp0, qsgw.to_device(cphim), ndima, qsgw.to_device(cphiq), ndima, dat)
    qsgw.synchronize()
    got = qsgw.from_device(zt, (nbloch, nm, ntp0))
    assert rel_fro(got, ref) < TOL
    # M -> E and conj
    m2e = _rc(rng, nbloch, nbloch - 4)
    out = torch.zeros((nbloch - 4) * nm * ntp0, dtype=torch.complex128, device='cuda')
    qsgw.zmel_m2e_d(out, zt, nbloch, nbloch - 4, nm, ntp0, qsgw.to_device(m2e), False, True)
    qsgw.synchronize()
    assert rel_fro(qsgw.from_device(out, (nbloch - 4, nm, ntp0)), zmel.zmel_m2e(ref, m2e, False, True)) < TOL


@pytest.mark.parametrize("ntp0,nmv", [(5, 9), (8, 3)])          # G1-first and G2-first orders
def test_zmel_ipw_vs_oracle(qsgw, ntp0, nmv):
    import torch
    from ecalj_b200 import synth
    lib = qsgw
    t = synth.ipw_tables(11 + nmv, ngc=37, ngp1=29, ngp2=31, ntp0=ntp0, nmv=nmv)
    nbloch, nm1, nm1v = 6, 1, 3
    nm2 = nm1v + nmv - 1 + 2                                         # two middle states past the valence range
    nmtot = nm2 - nm1 + 1
    ngc = t["ngveccR"].shape[1]
    ldz, ldgq, ldgk = nbloch + ngc + 1, 29 + 3, 31 + 2
    gq = np.zeros((ldgq, ntp0), complex, order="F")
    gq[:29] = t["geigq"]
    gk = np.zeros((ldgk, nmv), complex, order="F")
    gk[:31] = t["dgeigqk"]
    z0 = _rc(np.random.default_rng(1), ldz, nmtot, ntp0)
    zd = lib.to_device(z0)
    lib.zmel_ipw_d(zd, ldz, nbloch, nm1, nm2, nm1v, nm1v + nmv - 1, ntp0, lib.to_device(gq), ldgq,
                   lib.to_device(gk), ldgk, t["ngvecpB1"], t["ngvecpB2"], t["ngveccR"], t["nvgcgp2"], t["nvggg"],
                   t["ggg"], t["nadd"], t["phase"])
    got = lib.from_device(zd, (ldz, nmtot, ntp0))
    ref = zmel.zmel_ipw(t["geigq"], t["dgeigqk"], t["ngvecpB1"], t["ngvecpB2"], t["ngveccR"], t["nvggg"],
                        t["ggg"], t["nadd"], t["phase"])
    it0 = nm1v - nm1
    assert rel_fro(got[nbloch:nbloch + ngc, it0:it0 + nmv, :], ref) <= TOL
    mask = np.ones(got.shape, bool)                                  # nothing else is touched
    mask[nbloch:nbloch + ngc, it0:it0 + nmv, :] = False
    np.testing.assert_array_equal(got[mask], z0[mask])


def test_zmel_ipw_missing_composite_vector(qsgw):
    """A Gc+G2 vector absent from nvgcgp2 is an argument error, found on the host."""
    from ecalj_b200 import synth
    lib = qsgw
    t = synth.ipw_tables(4, ngc=9, ngp1=8, ngp2=7, ntp0=3, nmv=4)
    need = t["ngveccR"][:, 0] + t["ngvecpB2"][:, 0]
    keep = ~np.all(t["nvgcgp2"] == need[:, None], axis=0)
    z = lib.to_device(np.zeros((20, 4, 3), complex, order="F"))
    with pytest.raises(lib.QSGWError) as e:
        lib.zmel_ipw_d(z, 20, 6, 1, 4, 1, 4, 3, lib.to_device(np.asfortranarray(t["geigq"])), 8,
                       lib.to_device(np.asfortranarray(t["dgeigqk"])), 7, t["ngvecpB1"], t["ngvecpB2"], t["ngveccR"],
                       t["nvgcgp2"][:, keep], t["nvggg"], t["ggg"], t["nadd"], t["phase"])
    assert e.value.code == -1 and "nvgcgp2" in str(e.value)
