"""qsgw_sxcf_correlation_batch_d: several Sigma_c tasks in one call.

The batch must give what the same tasks give one call at a time (the int8
path runs the same tiles with the same slices and scales, so the results
agree to the FP64 rounding of the final product), in every precision, with
tasks of different shapes (the int8 launches are cut where ngb changes), an
empty task (no intermediate states), two tasks accumulating into one zsec,
and packed (keepwv) W.  The batch is also checked against the FP64 oracle.
"""
import numpy as np
import pytest

from oracle import sxcf
from tests.conftest import rel_fro
from tests.test_gpu_split import _sigc_problem
from tests.test_gpu_ozaki import _sigc_args

pytestmark = pytest.mark.gpu


def _tasks():
    """Five tasks: three of ngb = 150 (the first and third share zsec), one of
    ngb = 128 (a new int8 launch) and one with no intermediate states."""
    import torch
    from ecalj_b200 import lib
    probs = [_sigc_problem(150, 8, 60, 6, 12, seed=31), _sigc_problem(150, 8, 44, 6, 12, seed=32),
             _sigc_problem(150, 8, 60, 6, 12, seed=33), _sigc_problem(128, 8, 30, 6, 12, seed=34)]
    host, dev = [], []
    zsec_shared = None
    for k, s in enumerate(probs):
        args = list(_sigc_args(s))
        ntq = s['ntq']
        zs = np.zeros((ntq, ntq), complex, order='F')
        host.append(dict(s=s, args=args, zsec=zs))
        if k == 2:
            zd = zsec_shared                                   # accumulates after task 0
        else:
            zd = torch.zeros(ntq * ntq, dtype=torch.complex128, device='cuda')
        if k == 0:
            zsec_shared = zd
        dev.append(dict(zsec=zd, zmel=lib.to_device(s['z']), ns1=args[0], ns2=args[1], ns2r=args[2], nwxi=args[3],
                        nwx=args[4], ntqxx=args[5], wc_imag=lib.to_device(args[6]), wc_real=lib.to_device(args[7]),
                        omega=args[8], ekc=args[9], nctot=args[10], ef=args[11], esmr=args[12], wkkr=args[13],
                        ua=args[14], freqx=args[15], wwx=args[16], expa=args[17], freq_r=args[18],
                        ngb=s['ngb'], ntq=ntq))
    # an empty task (ns1 > ns2) between two non-empty ones: skipped, zsec untouched
    e = dict(dev[1])
    e['zsec'] = torch.zeros(8 * 8, dtype=torch.complex128, device='cuda')
    e['ns1'], e['ns2'], e['ns2r'] = 5, 4, 4
    dev.insert(2, e)
    return probs, host, dev


def _reset(dev):
    for t in dev:
        t['zsec'].zero_()


def _one_by_one(q, dev):
    for t in dev:
        q.sxcf_correlation(**dict(t, device=True))
    q.synchronize()
    return [t['zsec'].clone() for t in dev]


def _batched(q, dev):
    q.sxcf_correlation_batch_d(dev)
    q.synchronize()
    return [t['zsec'].clone() for t in dev]


@pytest.mark.parametrize("mode", ["fp64", "split-f16", "i8x3", "i8x4", "i8auto"])
def test_batch_equals_task_by_task(qsgw, mode):
    probs, host, dev = _tasks()
    prec = {"fp64": (qsgw.PREC_FP64, 1), "split-f16": (qsgw.PREC_SPLIT_F16, 2), "i8x3": (qsgw.PREC_SPLIT_I8, 3),
            "i8x4": (qsgw.PREC_SPLIT_I8, 4), "i8auto": (qsgw.PREC_SPLIT_I8, 0)}[mode]
    try:
        qsgw.set_precision(*prec)
        _reset(dev)
        one = _one_by_one(qsgw, dev)
        _reset(dev)
        bat = _batched(qsgw, dev)
        n0 = qsgw.launch_count()
        _reset(dev)
        bat2 = _batched(qsgw, dev)
        launches = qsgw.launch_count() - n0
    finally:
        qsgw.set_precision(qsgw.PREC_FP64, 1)
    for k, (a, b, c) in enumerate(zip(one, bat, bat2)):
        den = max(float(a.abs().max()), 1e-300)
        d = float((a - b).abs().max()) / den
        print(f"{mode} task {k}: batch vs one by one {d:.2e}")
        assert d < 1e-13
        assert float((b - c).abs().max()) / den < 1e-13
    assert float(bat[2].abs().max()) == 0.0            # the empty task
    # against the FP64 oracle: task 0 and task 2 (of the problem list) accumulate into one zsec
    ref = [np.zeros((8, 8), complex, order='F') for _ in probs]
    for k, s in enumerate(probs):
        sxcf.correlation_block(ref[k], s['z'], *host[k]['args'])
    tol = {"fp64": 1e-11, "split-f16": 2e-5, "i8x3": 1e-4, "i8x4": 1e-6, "i8auto": 5e-3}[mode]
    got = [bat[0], bat[1], bat[4]]
    want = [ref[0] + ref[2], ref[1], ref[3]]
    for g, w in zip(got, want):
        e = rel_fro(g.cpu().numpy().reshape(8, 8, order='F'), w)
        print(f"{mode}: batch vs oracle {e:.2e}")
        assert e < tol
    if mode.startswith("i8") and mode != "i8auto":
        print(f"{mode}: {launches} launches for the batch of {len(dev)} tasks")


def test_batch_keepwv_and_validation(qsgw):
    """Packed W (keepwv) in a batch, and the argument checks."""
    from ecalj_b200 import lib
    from tests.test_gpu_fp64 import _pack_upper
    probs, host, dev = _tasks()
    dev = [t for t in dev if t['ns1'] <= t['ns2']][:2]
    for t, k in zip(dev, (0, 1)):
        args = host[k]['args']
        wr = args[7]
        t['wc_imag'] = lib.to_device(_pack_upper(args[6]))
        t['wc_real'] = lib.to_device(_pack_upper(np.asfortranarray(0.5 * (wr + np.conj(np.transpose(wr, (1, 0, 2)))))))
        t['keepwv'] = True
    try:
        qsgw.set_precision(qsgw.PREC_SPLIT_I8, 4)
        _reset(dev)
        one = _one_by_one(qsgw, dev)
        _reset(dev)
        bat = _batched(qsgw, dev)
        for a, b in zip(one, bat):
            assert float((a - b).abs().max()) / float(a.abs().max()) < 1e-13
        for k in (0, 1):
            ref = np.zeros((8, 8), complex, order='F')
            sxcf.correlation_block(ref, probs[k]['z'], *host[k]['args'], keepwv=True)
            e = rel_fro(bat[k].cpu().numpy().reshape(8, 8, order='F'), ref)
            print(f"keepwv batch task {k} vs oracle {e:.2e}")
            assert e < 1e-6
        # a task with a bad size is refused before any work
        bad = dict(dev[1]); bad['ngb'] = 0
        with pytest.raises(qsgw.QSGWError):
            qsgw.sxcf_correlation_batch_d([dev[0], bad])
        qsgw.sxcf_correlation_batch_d([])                  # an empty batch is a no-op
    finally:
        qsgw.set_precision(qsgw.PREC_FP64, 1)
