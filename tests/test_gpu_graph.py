"""CUDA graph of a recorded call sequence: chi0 -> W -> Sigma_c recorded once
and replayed gives the eager results, reads device inputs at replay time, and
refuses to grow scratch while recording."""
import numpy as np
import pytest

from ecalj_b200 import synth
from oracle import sxcf
from tests.conftest import rel_fro

pytestmark = pytest.mark.gpu


def _problem(lib, torch):
    p = synth.chi0_problem(N=96, nk=4, nocc=3, nun=(10, 20), niw=6, seed=31)
    N, niw = p["N"], p["niw"]
    vsq, q = synth.coulomb(N, 32)
    t = synth.sigc_task(N, 6, 20, niw, 30, seed=33, esmr=0.02, ef=0.05)
    nt0p, nt0m = sxcf.nt0pm(t["ekc"], t["ef"], t["esmr"])
    nwxi, nwx, ntmax = sxcf.get_nwx(t["omega"], 6, nt0p, nt0m, 20, t["freq_r"], t["esmr"], t["ef"], t["ekc"], 0)
    freqs = np.concatenate([[0.0], p["freq_i"]])
    d = dict(p=p, t=t, N=N, niw=niw, vsq=vsq, freqs=freqs, nwxi=nwxi, nwx=nwx, ns2r=min(20, ntmax),
             z=lib.to_device(p["zcols"]), m2e=lib.to_device(q), zmel=lib.to_device(t["zmel"]),
             chi=torch.zeros(N * N * (niw + 1), dtype=torch.complex128, device="cuda"),
             zw=torch.zeros(N * N * (niw + 1), dtype=torch.complex128, device="cuda"),
             wr=torch.zeros(N * N * len(t["freq_r"]), dtype=torch.complex128, device="cuda"),
             zsec=torch.zeros(36, dtype=torch.complex128, device="cuda"))
    return d


def _step(lib, d):
    p, t, N, niw = d["p"], d["t"], d["N"], d["niw"]
    d["zsec"].zero_()
    lib.chi0_lorentz_d(d["chi"], N, niw + 1, d["freqs"], p["nk"], p["nocc"], p["nun"], p["eocc_h"], p["eun_h"], d["z"])
    lib.wvi_llw(d["chi"], 2, d["vsq"], d["m2e"], True, True, 2, zw=d["zw"], device=True, ngb=N, niw=niw + 1)
    d["wr"].view(-1, N * N)[:] = d["zw"][:N * N]          # real-axis W = W(0) on every record
    lib.sxcf_correlation(d["zsec"], d["zmel"], 1, 20, d["ns2r"], d["nwxi"], d["nwx"], 6, d["zw"], d["wr"],
                         t["omega"], t["ekc"], 0, t["ef"], t["esmr"], 1.0 / 8, t["ua"], t["x"], t["wx"], t["expa"],
                         t["freq_r"], nblochpmx=N, device=True, ngb=N, ntq=6)


@pytest.mark.parametrize("prec", ["fp64", "split"])
def test_graph_replay_matches_eager(qsgw, prec):
    import torch
    lib = qsgw
    lib.set_precision(lib.PREC_SPLIT_F16 if prec == "split" else lib.PREC_FP64)
    try:
        d = _problem(lib, torch)
        _step(lib, d)                                     # eager (also sizes every scratch buffer)
        lib.synchronize()
        ref = {k: d[k].clone() for k in ("chi", "zw", "zsec")}
        lib.graph_begin()
        _step(lib, d)
        lib.graph_end()
        for k in ("chi", "zw", "zsec"):
            d[k].fill_(7.0)                               # the replay must rewrite everything
        for _ in range(2):
            lib.graph_launch()
        lib.synchronize()
        tol = 1e-12 if prec == "fp64" else 1e-9
        for k in ("chi", "zw", "zsec"):
            assert rel_fro(d[k].cpu().numpy(), ref[k].cpu().numpy()) <= tol, k
        # device inputs are read at replay time: z -> 2 z gives chi0 -> 4 chi0
        d["z"].mul_(2.0)
        lib.graph_launch()
        lib.synchronize()
        assert rel_fro(d["chi"].cpu().numpy(), 4 * ref["chi"].cpu().numpy()) <= tol
        lib.graph_destroy()
    finally:
        lib.set_precision(lib.PREC_FP64)


def test_graph_refuses_scratch_growth(qsgw):
    import torch
    lib = qsgw
    # more pairs x frequencies than any test collected before this one (the full-size chi0
    # test is collected after it): the weight scratch must grow
    p = synth.chi0_problem(N=64, nk=64, nocc=8, nun=(100, 120), niw=12, seed=35)
    N, niw = p["N"], p["niw"]
    chi = torch.zeros(N * N * niw, dtype=torch.complex128, device="cuda")
    z = lib.to_device(p["zcols"])
    lib.graph_begin()
    with pytest.raises(lib.QSGWError) as e:
        lib.chi0_lorentz_d(chi, N, niw, p["freq_i"], p["nk"], p["nocc"], p["nun"], p["eocc_h"], p["eun_h"], z)
    assert e.value.code == -7 and "graph" in str(e.value)
    try:
        lib.graph_end()
    except lib.QSGWError:
        pass
    lib.graph_destroy()
    # eager use works again and sizes the buffers
    lib.chi0_lorentz_d(chi, N, niw, p["freq_i"], p["nk"], p["nocc"], p["nun"], p["eocc_h"], p["eun_h"], z)
    lib.synchronize()
    assert float(torch.linalg.vector_norm(chi)) > 0
