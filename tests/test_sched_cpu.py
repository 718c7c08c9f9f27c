"""The host scheduler (ecalj_b200/sched.py, vectorised) against the oracle's
scalar restatements of get_nwx (sxcf_fal2_count.sc.f90:238-298) and of the
pole-entry loop (m_sxcf_gemm.f90:529-552), with and without core states."""
import numpy as np
import pytest

from ecalj_b200 import sched, synth
from oracle import sxcf


def _case(seed, nctot):
    rng = np.random.default_rng(seed)
    ntq, nband = 12, 40
    ef, esmr = 0.05, 0.01
    core = np.sort(rng.uniform(-3.0, -1.5, nctot))
    val = np.sort(rng.uniform(-1.0, 3.0, nband))
    ekc = np.concatenate([core, val])
    omega = np.sort(rng.uniform(-0.9, 0.9, ntq))
    omega[3] = ef                                   # a target exactly at the Fermi level
    omega[7] = ef + 4e-7                            # inside wfacx2's 1e-6 cut-off
    if nctot:
        omega[0] = core[1] - 0.01                   # a target below two core levels
        omega[1] = core[2] + 0.005                  # half a smearing width above a core level
    fr = synth.freq_r_mesh(60, wmax=3.0)
    return omega, ekc, fr, ef, esmr


@pytest.mark.parametrize("nctot", [0, 3])
@pytest.mark.parametrize("seed", [1, 2, 3])
def test_get_nwx_matches_oracle(seed, nctot):
    omega, ekc, fr, ef, esmr = _case(seed, nctot)
    nt0p, nt0m = sxcf.nt0pm(ekc, ef, esmr)
    assert sched.nt0pm(ekc, ef, esmr) == (nt0p, nt0m)
    ref = sxcf.get_nwx(omega, len(omega), nt0p, nt0m, len(ekc), fr, esmr, ef, ekc, nctot)
    assert sched.get_nwx(omega, ekc, fr, ef, esmr, nctot=nctot) == ref


@pytest.mark.parametrize("nctot", [0, 3])
@pytest.mark.parametrize("seed", [4, 5])
def test_pole_bins_match_oracle_entries(seed, nctot):
    omega, ekc, fr, ef, esmr = _case(seed, nctot)
    ntq, ns1, nm = len(omega), 1, len(ekc)
    nt0p, nt0m = sxcf.nt0pm(ekc, ef, esmr)
    nwxi, nwx, _ = sxcf.get_nwx(omega, ntq, nt0p, nt0m, len(ekc), fr, esmr, ef, ekc, nctot)
    ref = sxcf.pole_table(omega, ekc, nctot, ns1, nm, ntq, ef, esmr, 1.0, fr)
    ent, recs = sched.pole_bins(omega, ekc, fr, ef, esmr, nwxi, nwx, nm, nm, ntq, ns1=ns1, nctot=nctot)
    assert [(c, x) for c, x in ent] == [((it - ns1) + nm * (itp - 1), ixs) for it, itp, ixs, _ in ref]
    want = sorted({x - 1 + j for _, _, x, _ in ref for j in range(3) if nwxi <= x - 1 + j <= nwx})
    assert recs == want
    if nctot:
        assert any(it <= nctot for it, _, _, _ in ref)      # the core window was exercised


@pytest.mark.parametrize("nnn,nmb", [(0, 5), (1, 5), (5, 5), (6, 5), (17, 5), (400, 64), (400, 400), (401, 400)])
def test_middle_batches(nnn, nmb):
    b = sched.middle_batches(nnn, nmb)
    ndiv = max((nnn - 1) // nmb + 1, 1) if nnn >= 1 else 1
    assert len(b) == ndiv
    sizes = [e - s + 1 for s, e in b]
    assert sum(sizes) == nnn and max(sizes) <= max(nmb, 1) and max(sizes) - min(sizes) <= 1
    assert sizes == sorted(sizes, reverse=True)                 # the remainder goes to the first batches
    assert b[0][0] == 1 and all(b[i + 1][0] == b[i][1] + 1 for i in range(len(b) - 1))


def test_middle_batches_known():
    assert sched.middle_batches(17, 5) == [(1, 5), (6, 9), (10, 13), (14, 17)]
    assert sched.middle_batches(0, 5) == [(1, 0)]               # one empty batch, as the reference keeps


def test_nmbatch_size():
    # 2 GB less 16 * 3000 * 60 bytes, over 60 * (500 + 2 * 800) * 16 bytes per state
    n = sched.nmbatch_size(400, 2.0, 3000, 60, 500, 800)
    assert n == min(400, int((2.0e9 - 16 * 3000 * 60) / (60 * 2100 * 16)))
    assert sched.nmbatch_size(50, 2.0, 3000, 60, 500, 800) == 50
    with pytest.raises(ValueError):
        sched.nmbatch_size(400, 1e-6, 3000, 60, 500, 800)


def test_sigma_task_order():
    """Loop order kx, irot, ip, isp over the nonzero irkip, each task cut into batches."""
    irkip = np.zeros((2, 3, 2, 3), int)             # (isp, kx, irot, ip)
    irkip[0, 0, 0, 1] = 4
    irkip[1, 0, 0, 1] = 4
    irkip[0, 0, 1, 0] = 7
    irkip[1, 2, 0, 2] = 9
    t = sched.sigma_tasks(irkip, lambda isp, kx, irot, ip, kr: 10 * kr % 13 + 1, 4)
    keys = [(d['kx'], d['irot'], d['ip'], d['isp']) for d in t]
    order = [(1, 1, 2, 1), (1, 1, 2, 2), (1, 2, 1, 1), (3, 1, 3, 2)]
    assert sorted(set(keys), key=keys.index) == order
    for d in t:
        n = 10 * d['kr'] % 13 + 1
        assert 1 <= d['nstti'] <= d['nstte'] <= n
    assert len([d for d in t if d['kr'] == 7]) == len(sched.middle_batches(10 * 7 % 13 + 1, 4))
