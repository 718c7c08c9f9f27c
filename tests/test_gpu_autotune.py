"""Autotuner: tuned split-K choices give the same chi0 (within each path's
parity tolerance), are cached per shape and written to the JSON cache."""
import json

import numpy as np
import pytest

from ecalj_b200 import synth
from oracle import x0
from tests.conftest import rel_fro

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("prec,tol", [("fp64", 1e-11), ("split", 5e-5)])
def test_autotuned_chi0(qsgw, tmp_path, prec, tol):
    import torch
    lib = qsgw
    p = synth.chi0_problem(N=130, nk=6, nocc=3, nun=(30, 50), niw=5, seed=41 if prec == "fp64" else 42)
    N, niw = p["N"], p["niw"]
    eo, eu, zs, oo, uo, c0 = [], [], [], 0, 0, 0
    for k in range(p["nk"]):
        no, nu = int(p["nocc"][k]), int(p["nun"][k])
        eo.append(p["eocc_h"][oo:oo + no]); eu.append(p["eun_h"][uo:uo + nu])
        zs.append(p["zcols"][:, c0:c0 + no * nu].reshape(N, no, nu, order="F"))
        oo += no; uo += nu; c0 += no * nu
    ref = x0.chi0_direct(zs, x0.lorentz_pair_tables(eo, eu, niw, p["freq_i"], p["nk"]), N, niw)[:, :, 1:]
    cache = tmp_path / "tune.json"
    lib.set_precision(lib.PREC_SPLIT_F16 if prec == "split" else lib.PREC_FP64)
    lib.set_autotune(1, cache)
    try:
        z = lib.to_device(p["zcols"])
        for _ in range(2):                       # first call tunes, second reuses the choice
            chi = torch.zeros(N * N * niw, dtype=torch.complex128, device="cuda")
            lib.chi0_lorentz_d(chi, N, niw, p["freq_i"], p["nk"], p["nocc"], p["nun"], p["eocc_h"], p["eun_h"], z)
            lib.synchronize()
            assert rel_fro(lib.from_device(chi, (N, N, niw)), ref) <= tol
        rep = lib.autotune_report()
        keys = [k for k in rep if f"npr={N} " in k and ("split" in k) == (prec == "split")]
        assert len(keys) == 1 and rep[keys[0]] >= 1
        assert json.loads(cache.read_text())[keys[0]] == rep[keys[0]]
    finally:
        lib.set_autotune(0, None)
        lib.set_precision(lib.PREC_FP64)


def test_autotuned_sigc_f16_kernel(qsgw, tmp_path):
    """Split-FP16 Sigma_c: with tuning on and no kernel fixed by the caller, the first call of a
    shape times the three kernels (64 x 128, CTA pairs, 64 x 256) and keeps the fastest; the
    result matches the oracle with every choice.  Run in a fresh process, since a
    qsgw_set_sigc_kernel call earlier in the session fixes the kernel for good."""
    import pathlib
    import subprocess
    import sys
    import textwrap
    root = str(pathlib.Path(__file__).resolve().parents[1])
    code = textwrap.dedent(f"""
        import json, sys
        import numpy as np
        sys.path.insert(0, {root!r})
        from ecalj_b200 import lib
        from oracle import sxcf
        from tests.conftest import rel_fro
        from tests.test_gpu_split import _sigc_problem
        from tests.test_gpu_ozaki import _sigc_args
        lib.load(); lib.init(0)
        s = _sigc_problem(150, 8, 60, 6, 12, seed=77)
        args = _sigc_args(s)
        ref = np.zeros((8, 8), complex, order='F')
        sxcf.correlation_block(ref, s['z'], *args)
        lib.set_precision(lib.PREC_SPLIT_F16)
        lib.set_autotune(1, {str(tmp_path / 'tune.json')!r})
        errs = []
        for _ in range(2):
            got = np.zeros((8, 8), complex, order='F')
            lib.sxcf_correlation(got, s['z'], *args)
            errs.append(rel_fro(got, ref))
        print(json.dumps({{"errs": errs, "report": lib.autotune_report()}}))
    """)
    r = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=600, cwd=root)
    assert r.returncode == 0, r.stderr[-2000:]
    out = json.loads(r.stdout.strip().splitlines()[-1])
    print(out)
    keys = [k for k in out["report"] if k.startswith("sigc_f16 kernel ngb=150")]
    assert len(keys) == 1 and out["report"][keys[0]] in (0, 1, 2)
    assert max(out["errs"]) < 2e-5
