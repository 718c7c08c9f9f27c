"""The int8 Ozaki-scheme tensor-core path (qsgw_set_precision(SPLIT_I8, ns)).

Two kinds of check:
* against tests/ozaki_emul.py, a CPU emulation of exactly the same scheme
  (same scales, slices and kept slice pairs, exact integer products): the GPU
  must match it to FP64 rounding -- this pins the kernels themselves;
* against the FP64 oracle: the error the slicing leaves, gated per slice count
  (about 2^-(7 ns) relative to the largest element of a row or column for the
  chi0 kernel's base-128 digits, 2^-(8 ns) for the Sigma_c kernel's base-256
  ones, and unbiased, since the integer products accumulate exactly).
"""
import numpy as np
import pytest

from oracle import sxcf, x0
from ecalj_b200 import synth
from tests import ozaki_emul
from tests.conftest import rel_fro
from tests.test_gpu_fp64 import _chi0_oracle, _rc
from tests.test_gpu_split import _sigc_problem
from tests.golden.make_golden import sigc_window

pytestmark = pytest.mark.gpu
HARTREE_MEV = 27211.386245988
# gate on the relative Frobenius error against the FP64 oracle, per slice count: chi0 (base-128
# digits) and the Sigma_c kernel (base-256 digits; also the zmel M -> E product), the latter
# about 5x above the measured 6.8e-5 / 3.2e-7 / 1.6e-9
GATE = {2: 5e-3, 3: 2e-5, 4: 2e-7}
GATE8 = {2: 3e-4, 3: 2e-6, 4: 1e-8}
EXACT = 1e-12      # against the emulation of the same scheme


@pytest.fixture()
def i8(qsgw):
    yield qsgw
    qsgw.set_precision(qsgw.PREC_FP64, 1)


def _sigc_args(s):
    t = s['t']
    nwxi, nwx, ntmax = sigc_window(t, s['ntq'])
    ns2r = min(s['nm'], ntmax)
    return (1, s['nm'], ns2r, nwxi, nwx, s['ntq'], s['wi'], s['wr'], t['omega'], t['ekc'], t['nctot'], t['ef'],
            t['esmr'], 1.0 / 64, t['ua'], t['x'], t['wx'], t['expa'], t['freq_r'])


@pytest.mark.parametrize("ns", [2, 3, 4])
@pytest.mark.parametrize("ngb", [150, 256])
def test_sigc_i8_matches_emulation_and_oracle(i8, ns, ngb):
    s = _sigc_problem(ngb, 8, 60, 6, 12, seed=ngb + ns)
    args = _sigc_args(s)
    ref = np.zeros((s['ntq'], s['ntq']), complex, order='F')
    sxcf.correlation_block(ref, s['z'], *args)
    emu = np.zeros((s['ntq'], s['ntq']), complex, order='F')
    ozaki_emul.correlation_block(emu, s['z'], *args, ns=ns)
    i8.set_precision(i8.PREC_SPLIT_I8, ns)
    got = np.zeros((s['ntq'], s['ntq']), complex, order='F')
    i8.sxcf_correlation(got, s['z'], *args)
    e_emu, e_ref = rel_fro(got, emu), rel_fro(got, ref)
    dqp = np.max(np.abs(np.real(np.diag(got) - np.diag(ref)))) * HARTREE_MEV
    print(f"sigc i8x{ns} ngb={ngb}: vs emulation {e_emu:.2e}, vs FP64 oracle {e_ref:.2e} "
          f"(emulation vs oracle {rel_fro(emu, ref):.2e}), max QP shift {dqp:.3e} meV")
    assert e_emu < EXACT
    assert e_ref < GATE8[ns]


@pytest.mark.parametrize("ngb", [129, 160, 161])
def test_sigc_i8_paired_tail_edges(i8, ngb):
    """The last row tile runs segment pairs when it holds 1..32 of its 64 rows: ngb = 129 (1 row),
    160 (32 rows, both halves full) paired, 161 (33 rows) not.  Each equals the emulation."""
    s = _sigc_problem(ngb, 8, 40, 5, 10, seed=ngb)
    args = _sigc_args(s)
    emu = np.zeros((s['ntq'], s['ntq']), complex, order='F')
    ozaki_emul.correlation_block(emu, s['z'], *args, ns=4)
    i8.set_precision(i8.PREC_SPLIT_I8, 4)
    got = np.zeros((s['ntq'], s['ntq']), complex, order='F')
    i8.sxcf_correlation(got, s['z'], *args)
    e = rel_fro(got, emu)
    print(f"sigc i8x4 ngb={ngb} (last tile {ngb % 64} rows): vs emulation {e:.2e}")
    assert e < EXACT


@pytest.mark.parametrize("keepwv", [False, True])
def test_sigc_i8_golden_case_vs_oracle(i8, keepwv):
    """The golden Sigma_c case, W given in full or as the packed upper
    triangles of the reference's keepwv mode (m_sxcf_gemm.f90:327-358, 467-475)."""
    from tests.golden.make_golden import inputs
    from tests.test_gpu_fp64 import _pack_upper
    s = inputs()['sc']
    t = s['t']
    nwxi, nwx, ntmax = sigc_window(t, s['ntq'])
    ns2r = min(s['nm'], ntmax)
    wi, wr = s['wi'], s['wr']
    if keepwv:
        wrh = np.asfortranarray(0.5 * (wr + np.conj(np.transpose(wr, (1, 0, 2)))))
        wi_in, wr_in = _pack_upper(wi), _pack_upper(wrh)
    else:
        wi_in, wr_in = wi, wr
    ref = np.zeros((s['ntq'], s['ntq']), complex, order='F')
    sxcf.correlation_block(ref, s['z'], 1, s['nm'], ns2r, nwxi, nwx, s['ntq'], wi, wr, t['omega'], t['ekc'],
                           t['nctot'], t['ef'], t['esmr'], 1.0 / 64, t['ua'], t['x'], t['wx'], t['expa'],
                           t['freq_r'], keepwv=keepwv)
    i8.set_precision(i8.PREC_SPLIT_I8, 3)
    got = np.zeros((s['ntq'], s['ntq']), complex, order='F')
    i8.sxcf_correlation(got, s['z'], 1, s['nm'], ns2r, nwxi, nwx, s['ntq'], wi_in, wr_in, t['omega'],
                        t['ekc'], t['nctot'], t['ef'], t['esmr'], 1.0 / 64, t['ua'], t['x'], t['wx'],
                        t['expa'], t['freq_r'], keepwv=keepwv)
    err = rel_fro(got, ref)
    dqp = np.max(np.abs(np.real(np.diag(got) - np.diag(ref)))) * HARTREE_MEV
    print(f"sigc i8x3 golden keepwv={keepwv}: rel err {err:.2e}, max QP shift {dqp:.3e} meV")
    assert err < GATE8[3]
    assert dqp < 1.0


@pytest.mark.parametrize("ns", [2, 3, 4])
@pytest.mark.parametrize("cfg", ["small", "odd"])
def test_chi0_i8_matches_emulation_and_oracle(i8, ns, cfg):
    import torch
    if cfg == "odd":
        p = synth.chi0_problem(N=131, nk=3, nocc=5, nun=(11, 29), niw=7, seed=8)
    else:
        p = synth.chi0_problem(N=64, nk=2, nocc=2, nun=(8, 8), niw=4, seed=4)
    ref = _chi0_oracle(p)
    N, niw = p['N'], p['niw']
    oo = np.concatenate([[0], np.cumsum(p['nocc'])]); uo = np.concatenate([[0], np.cumsum(p['nun'])])
    # zcols order per k: (it - 1) + nocc_k (itp - 1), occupied index fastest
    de = np.concatenate([(p['eun_h'][uo[k]:uo[k + 1]][None, :] - p['eocc_h'][oo[k]:oo[k + 1]][:, None])
                         .reshape(-1, order='F') for k in range(p['nk'])])
    w = -2.0 * de[None, :] / (de[None, :] ** 2 + p['freq_i'][:, None] ** 2) / p['nk']
    emu = ozaki_emul.chi0_dense(p['zcols'], w, ns)
    i8.set_precision(i8.PREC_SPLIT_I8, ns)
    chi = torch.zeros(N * N * niw, dtype=torch.complex128, device='cuda')
    i8.chi0_lorentz_d(chi, N, niw, p['freq_i'], p['nk'], p['nocc'], p['nun'], p['eocc_h'], p['eun_h'],
                      i8.to_device(p['zcols']))
    i8.synchronize()
    got = i8.from_device(chi, (N, N, niw))
    e_emu, e_ref = rel_fro(got, emu), rel_fro(got, ref)
    print(f"chi0 i8x{ns} {cfg}: vs emulation {e_emu:.2e}, vs FP64 oracle {e_ref:.2e} "
          f"(emulation vs oracle {rel_fro(emu, ref):.2e})")
    assert e_emu < EXACT
    assert e_ref < GATE[ns]


@pytest.mark.parametrize("npr,ipr_col,npr_col,npm", [(200, 1, 200, 2), (131, 40, 61, 1), (65, 1, 65, 2)])
def test_x0gemm_i8_vs_oracle(i8, npr, ipr_col, npr_col, npm):
    """The reference's own chi0 boundary (pair/bin lists, jpm, ragged bins,
    ipr_col column blocks, weights of both signs, accumulation into rcxq) on the
    int8 path."""
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
    i8.set_precision(i8.PREC_SPLIT_I8, 4)
    got = r0.copy(order='F')
    i8.x0gemm(got, npr, ipr_col, npr_col, nwhis, npm, 4, 11, z, nm1, 5, ncoun - 3,
              itc, itpc, jpmc, iwini, iwend, icouini, whwc)
    err = rel_fro(got - r0, ref - r0)
    print(f"x0gemm i8x4 npr={npr} ipr_col={ipr_col} npr_col={npr_col} npm={npm}: added part vs oracle {err:.2e}")
    assert err < GATE[4] * 10


def test_set_precision_validates_i8_slices(qsgw):
    for bad in (1, 5):
        with pytest.raises(qsgw.QSGWError):
            qsgw.set_precision(qsgw.PREC_SPLIT_I8, bad)
    qsgw.set_precision(qsgw.PREC_SPLIT_I8, 3)
    assert qsgw.get_precision() == (qsgw.PREC_SPLIT_I8, 3)
    qsgw.set_precision(qsgw.PREC_FP64, 1)


def test_automatic_slice_count_meets_the_targets(i8):
    """set_precision(SPLIT_I8, 0): the first call of a shape tries 2 and 3
    slices against 4 and keeps the smallest within the target; the report
    lists the choice and the estimates, and the result honours the target."""
    s = _sigc_problem(150, 8, 60, 6, 12, seed=11)
    args = _sigc_args(s)
    tol_ha = 1e-3 / 27.211386245988
    i8.set_accuracy(tol_ha, 2e-5)
    i8.set_precision(i8.PREC_SPLIT_I8, 4)
    ref4 = np.zeros((s['ntq'], s['ntq']), complex, order='F')
    i8.sxcf_correlation(ref4, s['z'], *args)
    i8.set_precision(i8.PREC_SPLIT_I8, 0)
    got = np.zeros((s['ntq'], s['ntq']), complex, order='F')
    i8.sxcf_correlation(got, s['z'], *args)
    rep = i8.autotune_report()
    key = next(k for k in rep if k.startswith("sigc_i8 slices ngb=150") and "err@" not in k)
    ns = rep[key]
    errs = {int(k.rsplit("@", 1)[1]): v for k, v in rep.items() if k.startswith(key + " err@")}
    print(f"automatic Sigma_c slices: {ns}, estimates {errs}")
    assert ns in (2, 3, 4) and all(errs[c] > 0.25 * tol_ha for c in errs if c < ns)
    if ns < 4:
        assert errs[ns] <= 0.25 * tol_ha
    assert np.max(np.abs(np.real(np.diag(got) - np.diag(ref4)))) <= tol_ha * 1.01
    # chi0
    import torch
    p = synth.chi0_problem(N=131, nk=3, nocc=5, nun=(11, 29), niw=7, seed=8)
    N, niw = p['N'], p['niw']
    chi = torch.zeros(N * N * niw, dtype=torch.complex128, device='cuda')
    i8.chi0_lorentz_d(chi, N, niw, p['freq_i'], p['nk'], p['nocc'], p['nun'], p['eocc_h'], p['eun_h'],
                      i8.to_device(p['zcols']))
    i8.synchronize()
    rep = i8.autotune_report()
    key = next(k for k in rep if k.startswith("chi0_i8 slices npr=131") and "err@" not in k)
    print(f"automatic chi0 slices: {rep[key]}, report {rep}")
    ref = _chi0_oracle(p)
    assert rel_fro(i8.from_device(chi, (N, N, niw)), ref) < 4e-5


@pytest.mark.parametrize("ns", [3, 4])
@pytest.mark.parametrize("conj", [0, 1])
def test_zmel_m2e_i8_matches_emulation(i8, ns, conj):
    """zmel = m2e^H zmelt (m_zmel.f90:559-560), then conj (:590-594), on the
    int8 path: a non-square product (nbb = 130 E-basis rows from ngb = 150)."""
    rng = np.random.default_rng(40 + ns)
    ngb, nbb, nmtot, nqtot = 150, 130, 7, 23
    m2e = _rc(rng, ngb, nbb)
    zmelt = _rc(rng, ngb, nmtot, nqtot)
    ref = (m2e.conj().T @ zmelt.reshape(ngb, -1, order='F')).reshape(nbb, nmtot, nqtot, order='F')
    emu = ozaki_emul.complex_product(m2e.conj().T, zmelt.reshape(ngb, -1, order='F'), ns, bits=8)
    emu = emu.reshape(nbb, nmtot, nqtot, order='F')
    if conj:
        ref, emu = ref.conj(), emu.conj()
    i8.set_precision(i8.PREC_SPLIT_I8, ns)
    out = i8.to_device(np.zeros((nbb, nmtot, nqtot), complex, order='F'))
    i8.zmel_m2e_d(out, i8.to_device(zmelt), ngb, nbb, nmtot, nqtot, i8.to_device(m2e), 0, conj)
    i8.synchronize()
    got = i8.from_device(out, (nbb, nmtot, nqtot))
    e_emu, e_ref = rel_fro(got, emu), rel_fro(got, ref)
    print(f"zmel m2e i8x{ns} conj={conj}: vs emulation {e_emu:.2e}, vs FP64 {e_ref:.2e}")
    assert e_emu < EXACT
    assert e_ref < GATE8[ns]
