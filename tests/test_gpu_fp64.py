"""Parity of the FP64 CUDA path against the oracle, through the C ABI.
Tolerance: relative Frobenius error <= 1e-11 on chi0, W and Sigma_c, the
parity bar of the plain complex-FP64 path."""
import numpy as np
import pytest

from oracle import llw, sxcf, x0
from ecalj_b200 import synth
from tests.conftest import rel_fro
from tests.golden.make_golden import inputs, sigc_window

pytestmark = pytest.mark.gpu
TOL = 1e-11


def _rc(rng, *shape):
    return np.asfortranarray(rng.standard_normal(shape) + 1j * rng.standard_normal(shape))


@pytest.mark.parametrize("m,n,k,opa,opb", [(70, 45, 33, 0, 0), (64, 64, 64, 2, 0), (17, 130, 300, 1, 2),
                                           (5, 7, 3000, 2, 1), (129, 65, 1, 0, 2)])
def test_zmm_host(qsgw, m, n, k, opa, opb):
    rng = np.random.default_rng(m * 7 + n)
    a = _rc(rng, m, k) if opa == 0 else _rc(rng, k, m)
    b = _rc(rng, k, n) if opb == 0 else _rc(rng, n, k)
    c = _rc(rng, m, n)
    op = lambda x, o: x if o == 0 else (x.T if o == 1 else x.conj().T)
    alpha, beta = 0.7 - 0.2j, 0.3 + 0.1j
    ref = alpha * op(a, opa) @ op(b, opb) + beta * c
    qsgw.zmm(a, b, c, m, n, k, opa, opb, alpha, beta)
    assert rel_fro(c, ref) < TOL


def test_x0gemm_golden(qsgw):
    a = inputs()['x0']
    gold = np.load(__file__.replace("test_gpu_fp64.py", "golden/golden.npz"))['x0_rcxq']
    r = np.zeros((a['npr'], a['npr_col'], 2 * a['nwhis'] + 1), complex, order='F')
    qsgw.x0gemm(r, a['npr'], a['ipr_col'], a['npr_col'], a['nwhis'], 2, a['ns1'], a['ns2'], a['z'], a['nm1'],
                1, a['ncoun'], a['itc'], a['itpc'], a['jpmc'], a['iwini'], a['iwend'], a['icouini'], a['whwc'])
    assert rel_fro(r, gold) < TOL


@pytest.mark.parametrize("npr,ipr_col,npr_col,npm", [(13, 1, 13, 1), (200, 1, 200, 2), (131, 40, 61, 1),
                                                     (64, 1, 64, 1), (65, 1, 65, 2)])
def test_x0gemm_vs_oracle(qsgw, npr, ipr_col, npr_col, npm):
    rng = np.random.default_rng(npr + npm)
    nbb, nm1, nm2, nqtot, nwhis, ncoun = max(npr, ipr_col - 1 + npr_col) + 3, 3, 12, 17, 6, 400
    z = _rc(rng, nbb, nm2 - nm1 + 1, nqtot)
    itc = rng.integers(nm1, nm2 + 1, ncoun); itpc = rng.integers(1, nqtot + 1, ncoun)
    jpmc = rng.integers(1, npm + 1, ncoun); iwini = rng.integers(1, nwhis + 1, ncoun)
    iwend = np.minimum(nwhis, iwini + rng.integers(0, 4, ncoun))
    nh = iwend - iwini + 1
    icouini = np.concatenate([[1], np.cumsum(nh)[:-1] + 1]); whwc = rng.uniform(-1, 1, int(nh.sum()))
    nslab = nwhis + 1 if npm == 1 else 2 * nwhis + 1
    r0 = _rc(rng, npr, npr_col, nslab)
    ref = r0.copy(order='F')
    x0.x0gemm(ref, npr, ipr_col, npr_col, nwhis, npm, 4, 11, z, nm1, 5, ncoun - 3,
              itc, itpc, jpmc, iwini, iwend, icouini, whwc)
    got = r0.copy(order='F')
    qsgw.x0gemm(got, npr, ipr_col, npr_col, nwhis, npm, 4, 11, z, nm1, 5, ncoun - 3,
                itc, itpc, jpmc, iwini, iwend, icouini, whwc)
    assert rel_fro(got, ref) < TOL


def test_x0gemm_device_and_empty_range(qsgw):
    import torch
    a = inputs()['x0']
    gold = np.load(__file__.replace("test_gpu_fp64.py", "golden/golden.npz"))['x0_rcxq']
    shape = (a['npr'], a['npr_col'], 2 * a['nwhis'] + 1)
    r = qsgw.to_device(np.zeros(shape, complex, order='F'))
    z = qsgw.to_device(a['z'])
    qsgw.x0gemm(r, a['npr'], a['ipr_col'], a['npr_col'], a['nwhis'], 2, a['ns1'], a['ns2'], z, a['nm1'],
                1, a['ncoun'], a['itc'], a['itpc'], a['jpmc'], a['iwini'], a['iwend'], a['icouini'], a['whwc'],
                zmel_shape=a['z'].shape, device=True)
    # an empty icoun range leaves rcxq untouched
    qsgw.x0gemm(r, a['npr'], a['ipr_col'], a['npr_col'], a['nwhis'], 2, a['ns1'], a['ns2'], z, a['nm1'],
                4, 3, a['itc'], a['itpc'], a['jpmc'], a['iwini'], a['iwend'], a['icouini'], a['whwc'],
                zmel_shape=a['z'].shape, device=True)
    torch.cuda.synchronize()
    qsgw.synchronize()
    assert rel_fro(qsgw.from_device(r, shape), gold) < TOL


def test_x0gemm_rejects_bad_index(qsgw):
    a = inputs()['x0']
    r = np.zeros((a['npr'], a['npr_col'], 2 * a['nwhis'] + 1), complex, order='F')
    itpc = a['itpc'].copy(); itpc[3] = a['nqtot'] + 5
    with pytest.raises(qsgw.QSGWError) as e:
        qsgw.x0gemm(r, a['npr'], a['ipr_col'], a['npr_col'], a['nwhis'], 2, 1, 9, a['z'], a['nm1'],
                    1, a['ncoun'], a['itc'], itpc, a['jpmc'], a['iwini'], a['iwend'], a['icouini'], a['whwc'])
    assert e.value.code == -1


def _chi0_oracle(p):
    nk = p['nk']
    eo, eu, zs = [], [], []
    oo = uo = c0 = 0
    for k in range(nk):
        no, nu = int(p['nocc'][k]), int(p['nun'][k])
        eo.append(p['eocc_h'][oo:oo + no]); eu.append(p['eun_h'][uo:uo + nu])
        zs.append(p['zcols'][:, c0:c0 + no * nu].reshape(p['N'], no, nu, order='F'))
        oo += no; uo += nu; c0 += no * nu
    tabs = x0.lorentz_pair_tables(eo, eu, p['niw'], p['freq_i'], nk)
    return x0.chi0_direct(zs, tabs, p['N'], p['niw'])[:, :, 1:]


@pytest.mark.parametrize("cfg", ["small", "n260"])
def test_chi0_lorentz_vs_oracle(qsgw, cfg):
    import torch
    if cfg == "n260":
        c = synth.CONFIGS["chi0_w_n260"]
        p = synth.chi0_problem(c['N'], c['nk'], c['nocc'], c['nun'], c['niw'], c['seed'])
    else:
        p = synth.chi0_problem(N=97, nk=5, nocc=3, nun=(7, 19), niw=5, seed=3)
    ref = _chi0_oracle(p)
    N, niw = p['N'], p['niw']
    chi = torch.zeros(N * N * niw, dtype=torch.complex128, device='cuda')
    z = qsgw.to_device(p['zcols'])
    qsgw.chi0_lorentz_d(chi, N, niw, p['freq_i'], p['nk'], p['nocc'], p['nun'], p['eocc_h'], p['eun_h'], z)
    qsgw.synchronize()
    got = qsgw.from_device(chi, (N, N, niw))
    assert rel_fro(got, ref) < TOL


@pytest.mark.parametrize("n", [1, 31, 32, 33, 100, 257])
def test_zminv_hpd(qsgw, n):
    rng = np.random.default_rng(n)
    nb = 3
    a = np.zeros((n, n, nb), complex, order='F')
    for b in range(nb):
        g = rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))
        a[:, :, b] = np.eye(n) + 0.3 * g @ g.conj().T / n
    d = qsgw.to_device(a)
    qsgw.zminv_hpd_batched_d(d, n, n, nb)
    qsgw.synchronize()
    got = qsgw.from_device(d, a.shape)
    for b in range(nb):
        assert rel_fro(got[:, :, b], np.linalg.inv(a[:, :, b])) < TOL


@pytest.mark.parametrize("iq,nspin,xm,wm", [(3, 2, True, True), (1, 1, True, True), (2, 2, False, False)])
def test_wvi_llw_vs_oracle(qsgw, iq, nspin, xm, wm):
    w = inputs()['wv']
    ref_in = w['chi'].copy(order='F')
    ref = llw.wvi_llw(ref_in, nspin, w['vsq'], w['q'], xm, wm, iq, nblochpmx=53)
    got_in = w['chi'].copy(order='F')
    got = qsgw.wvi_llw(got_in, nspin, w['vsq'], w['q'], xm, wm, iq, nblochpmx=53)
    assert rel_fro(got, ref) < TOL
    assert rel_fro(got_in, ref_in) < 1e-15          # the in-place spin doubling


def test_wvi_golden(qsgw):
    w = inputs()['wv']
    gold = np.load(__file__.replace("test_gpu_fp64.py", "golden/golden.npz"))['wv_zw']
    got = qsgw.wvi_llw(w['chi'].copy(order='F'), 2, w['vsq'], w['q'], True, True, 3)
    assert rel_fro(got, gold) < TOL


def test_wvi_not_positive_definite_reports_error(qsgw):
    """chi = 1, v^1/2 = 1 makes eps~ = 0: the pivot blocks are singular and
    the call must come back with ERR_NUMERIC (the kernels only compute with
    the resulting inf/nan values; nothing faults)."""
    w = inputs()['wv']
    chi = np.asfortranarray(np.repeat(np.eye(48)[:, :, None], 4, axis=2).astype(complex))
    with pytest.raises(qsgw.QSGWError) as e:
        qsgw.wvi_llw(chi, 2, np.ones(48), w['q'], False, False, 2)
    assert e.value.code == -5


def _sigc_case(keepwv, nblochpmx=None):
    s = inputs()['sc']
    t = s['t']
    nwxi, nwx, ntmax = sigc_window(t, s['ntq'])
    return s, t, nwxi, nwx, min(s['nm'], ntmax)


def _pack_upper(w):
    n = w.shape[0]
    iu = np.triu_indices(n)
    order = np.lexsort((iu[0], iu[1]))         # column-major over the upper triangle
    idx = (iu[0][order], iu[1][order])
    return np.asfortranarray(np.stack([w[:, :, m][idx] for m in range(w.shape[2])], axis=1))


def test_sigc_golden(qsgw):
    s, t, nwxi, nwx, ns2r = _sigc_case(False)
    gold = np.load(__file__.replace("test_gpu_fp64.py", "golden/golden.npz"))['sc_zsec']
    zs = np.zeros((s['ntq'], s['ntq']), complex, order='F')
    qsgw.sxcf_correlation(zs, s['z'], 1, s['nm'], ns2r, nwxi, nwx, s['ntq'], s['wi'], s['wr'], t['omega'],
                          t['ekc'], t['nctot'], t['ef'], t['esmr'], 1.0 / 64, t['ua'], t['x'], t['wx'],
                          t['expa'], t['freq_r'])
    assert rel_fro(zs, gold) < TOL


@pytest.mark.parametrize("keepwv", [False, True])
def test_sigc_vs_oracle_accumulates(qsgw, keepwv):
    s, t, nwxi, nwx, ns2r = _sigc_case(keepwv)
    rng = np.random.default_rng(5)
    ntq = s['ntq'] + 2                       # zsec leading dimension larger than ntqxx
    z0 = _rc(rng, ntq, ntq)
    ref = z0.copy(order='F'); got = z0.copy(order='F')
    wi, wr = s['wi'], s['wr']
    for task in range(2):
        sxcf.correlation_block(ref, s['z'], 1, s['nm'], ns2r, nwxi, nwx, s['ntq'], wi, wr, t['omega'],
                               t['ekc'], t['nctot'], t['ef'], t['esmr'], 0.25 * (task + 1), t['ua'], t['x'],
                               t['wx'], t['expa'], t['freq_r'], keepwv=keepwv)
        if keepwv:
            wrh = np.asfortranarray(0.5 * (wr + np.conj(np.transpose(wr, (1, 0, 2)))))
            wi_in, wr_in = _pack_upper(wi), _pack_upper(wrh)
        else:
            wi_in, wr_in = wi, wr
        qsgw.sxcf_correlation(got, s['z'], 1, s['nm'], ns2r, nwxi, nwx, s['ntq'], wi_in, wr_in, t['omega'],
                              t['ekc'], t['nctot'], t['ef'], t['esmr'], 0.25 * (task + 1), t['ua'], t['x'],
                              t['wx'], t['expa'], t['freq_r'], keepwv=keepwv)
    assert rel_fro(got, ref) < TOL


def test_sigc_wgtim_device(qsgw):
    import torch
    s, t, *_ = _sigc_case(False)
    gold = np.load(__file__.replace("test_gpu_fp64.py", "golden/golden.npz"))['sc_wgtim']
    out = torch.zeros(gold.size, dtype=torch.float64, device='cuda')
    qsgw.sxcf_wgtim_d(out, s['niw'], 1, s['nm'], s['ntq'], t['nctot'], t['omega'], t['ekc'], t['esmr'],
                      1.0 / 64, t['ua'], t['x'], t['wx'], t['expa'])
    qsgw.synchronize()
    got = out.cpu().numpy().reshape(gold.shape, order='F')
    assert rel_fro(got, gold) < 1e-13
