"""Split-FP16 tcgen05 path against the FP64 oracle.  Three FP16 slice
products with FP32 accumulation carry ~22 significant bits, so the gate is
a relative Frobenius error <= 5e-5 on chi0 and Sigma_c (not the 1e-11 of
the plain FP64 path), and the quasiparticle-energy error of Sigma_c must
stay far below 1 meV."""
import numpy as np
import pytest

from oracle import sxcf
from ecalj_b200 import synth
from tests.conftest import rel_fro
from tests.golden.make_golden import inputs, sigc_window
from tests.test_gpu_fp64 import _chi0_oracle

pytestmark = pytest.mark.gpu
TOL = 5e-5
HARTREE_MEV = 27211.386245988


@pytest.fixture()
def split(qsgw):
    qsgw.set_precision(qsgw.PREC_SPLIT_F16, 2)
    yield qsgw
    qsgw.set_precision(qsgw.PREC_FP64, 1)


@pytest.mark.parametrize("cfg", ["small", "odd", "n260"])
def test_chi0_split_vs_oracle(split, cfg):
    import torch
    if cfg == "n260":
        c = synth.CONFIGS["chi0_w_n260"]
        p = synth.chi0_problem(c['N'], c['nk'], c['nocc'], c['nun'], c['niw'], c['seed'])
    elif cfg == "odd":
        p = synth.chi0_problem(N=131, nk=3, nocc=5, nun=(11, 29), niw=7, seed=8)
    else:
        p = synth.chi0_problem(N=64, nk=2, nocc=2, nun=(8, 8), niw=4, seed=4)
    ref = _chi0_oracle(p)
    N, niw = p['N'], p['niw']
    chi = torch.zeros(N * N * niw, dtype=torch.complex128, device='cuda')
    split.chi0_lorentz_d(chi, N, niw, p['freq_i'], p['nk'], p['nocc'], p['nun'], p['eocc_h'], p['eun_h'],
                         split.to_device(p['zcols']))
    split.synchronize()
    got = split.from_device(chi, (N, N, niw))
    err = rel_fro(got, ref)
    print(f"chi0 split {cfg}: rel Frobenius error {err:.2e}")
    assert err < TOL


@pytest.mark.parametrize("keepwv", [False, True])
def test_sigc_split_vs_oracle(split, keepwv):
    s = inputs()['sc']
    t = s['t']
    nwxi, nwx, ntmax = sigc_window(t, s['ntq'])
    ns2r = min(s['nm'], ntmax)
    wi, wr = s['wi'], s['wr']
    if keepwv:
        from tests.test_gpu_fp64 import _pack_upper
        wrh = np.asfortranarray(0.5 * (wr + np.conj(np.transpose(wr, (1, 0, 2)))))
        wi_in, wr_in = _pack_upper(wi), _pack_upper(wrh)
    else:
        wi_in, wr_in = wi, wr
    ref = np.zeros((s['ntq'], s['ntq']), complex, order='F')
    sxcf.correlation_block(ref, s['z'], 1, s['nm'], ns2r, nwxi, nwx, s['ntq'], wi, wr, t['omega'], t['ekc'],
                           t['nctot'], t['ef'], t['esmr'], 1.0 / 64, t['ua'], t['x'], t['wx'], t['expa'],
                           t['freq_r'], keepwv=keepwv)
    got = np.zeros((s['ntq'], s['ntq']), complex, order='F')
    split.sxcf_correlation(got, s['z'], 1, s['nm'], ns2r, nwxi, nwx, s['ntq'], wi_in, wr_in, t['omega'],
                           t['ekc'], t['nctot'], t['ef'], t['esmr'], 1.0 / 64, t['ua'], t['x'], t['wx'],
                           t['expa'], t['freq_r'], keepwv=keepwv)
    err = rel_fro(got, ref)
    dqp = np.max(np.abs(np.real(np.diag(got) - np.diag(ref)))) * HARTREE_MEV
    print(f"sigc split keepwv={keepwv}: rel err {err:.2e}, max QP shift {dqp:.3e} meV")
    assert err < TOL
    assert dqp < 1.0          # QP energies within 1 meV of the FP64 oracle


def _sigc_problem(ngb, ntq, nm, niw, nreal, seed):
    """A Sigma_c task with several 64-row tiles of the product basis (the
    golden case has one), random W on the imaginary and real axes."""
    rng = np.random.default_rng(seed)
    t = synth.sigc_task(ngb, ntq, nm, niw, nreal, seed=seed, nctot=2, esmr=0.02, ef=0.05)
    wi = np.asfortranarray(rng.standard_normal((ngb, ngb, niw + 1))
                           + 1j * rng.standard_normal((ngb, ngb, niw + 1))) * 0.1
    wr = np.asfortranarray(rng.standard_normal((ngb, ngb, nreal)) + 1j * rng.standard_normal((ngb, ngb, nreal))) * 0.1
    zz = np.asfortranarray(rng.standard_normal((ngb, nm + 2, ntq)) + 1j * rng.standard_normal((ngb, nm + 2, ntq)))
    return dict(t=t, wi=wi, wr=wr, z=zz, ngb=ngb, ntq=ntq, nm=nm + 2)


@pytest.mark.parametrize("ngb", [150, 256])
def test_sigc_split_kernels_multi_tile(split, ngb):
    """The three split Sigma_c kernels (64 x 256 tiles, CTA pairs over two
    row tiles of 128 columns, 64 x 128 tiles) against the oracle and each
    other; 150 rows = 3 row tiles, so one pair has a padding tile."""
    s = _sigc_problem(ngb, 8, 60, 6, 12, seed=ngb)
    t = s['t']
    nwxi, nwx, ntmax = sigc_window(t, s['ntq'])
    ns2r = min(s['nm'], ntmax)
    ref = np.zeros((s['ntq'], s['ntq']), complex, order='F')
    sxcf.correlation_block(ref, s['z'], 1, s['nm'], ns2r, nwxi, nwx, s['ntq'], s['wi'], s['wr'], t['omega'],
                           t['ekc'], t['nctot'], t['ef'], t['esmr'], 1.0 / 64, t['ua'], t['x'], t['wx'], t['expa'],
                           t['freq_r'])
    outs = {}
    try:
        for kind in (split.SIGC_WIDE, split.SIGC_PAIR, split.SIGC_NARROW):
            split.set_sigc_kernel(kind)
            got = np.zeros((s['ntq'], s['ntq']), complex, order='F')
            split.sxcf_correlation(got, s['z'], 1, s['nm'], ns2r, nwxi, nwx, s['ntq'], s['wi'], s['wr'],
                                   t['omega'], t['ekc'], t['nctot'], t['ef'], t['esmr'], 1.0 / 64, t['ua'], t['x'],
                                   t['wx'], t['expa'], t['freq_r'])
            outs[kind] = got
    finally:
        split.set_sigc_kernel(split.SIGC_WIDE)
    for kind, got in outs.items():
        err = rel_fro(got, ref)
        dqp = np.max(np.abs(np.real(np.diag(got) - np.diag(ref)))) * HARTREE_MEV
        print(f"sigc split ngb={ngb} kernel={kind}: rel err {err:.2e}, max QP shift {dqp:.3e} meV")
        assert err < TOL
        assert dqp < 1.0
    for kind in (split.SIGC_PAIR, split.SIGC_WIDE):
        d = rel_fro(outs[kind], outs[split.SIGC_NARROW])
        print(f"kernel {kind} vs 64 x 128 tiles: rel difference {d:.2e}")
        assert d < 1e-6
