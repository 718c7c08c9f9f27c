"""Asynchronous mode of the host-pointer entry points (qsgw_set_host_async):
calls return once their copies and kernels are enqueued, the inputs travel on
a copy stream into two device slots, and a zsec array accumulated by several
calls keeps one device image until qsgw_synchronize.  The results must equal
those of the synchronous calls to rounding (the kernels add partial sums with
atomics, so the last bit may differ between any two runs)."""
import numpy as np
import pytest

from ecalj_b200 import synth
from tests.golden.make_golden import inputs, sigc_window

pytestmark = pytest.mark.gpu
TOL = 1e-13


def _same(a, b):
    return np.linalg.norm(a - b) <= TOL * np.linalg.norm(b)


def _pinned(torch, keep, a):
    """A pinned-memory copy of a (column-major), so the copies are truly asynchronous."""
    t = torch.empty(a.size, dtype=torch.complex128 if np.iscomplexobj(a) else torch.float64, pin_memory=True)
    keep.append(t)
    v = t.numpy().reshape(a.shape, order='F')
    v[...] = a
    return v


def _sigc_call(qsgw, zsec, s, z, wi, wr, wkkr):
    t = s['t']
    nwxi, nwx, ntmax = sigc_window(t, s['ntq'])
    qsgw.sxcf_correlation(zsec, z, 1, s['nm'], min(s['nm'], ntmax), nwxi, nwx, s['ntq'], wi, wr, t['omega'],
                          t['ekc'], t['nctot'], t['ef'], t['esmr'], wkkr, t['ua'], t['x'], t['wx'], t['expa'],
                          t['freq_r'])


def test_sigc_async_accumulates(qsgw):
    import torch
    s = inputs()['sc']
    keep = []
    z, wi, wr = (_pinned(torch, keep, s[k]) for k in ('z', 'wi', 'wr'))
    rng = np.random.default_rng(3)
    ntq = s['ntq']
    z0 = np.asfortranarray(rng.standard_normal((ntq, ntq)) + 1j * rng.standard_normal((ntq, ntq)))
    ref = z0.copy(order='F')
    for task in range(3):
        _sigc_call(qsgw, ref, s, s['z'], s['wi'], s['wr'], 0.25 * (task + 1))
    got = _pinned(torch, keep, z0)
    qsgw.set_host_async(True)
    try:
        for task in range(3):                 # the same host zsec: one device image accumulates
            _sigc_call(qsgw, got, s, z, wi, wr, 0.25 * (task + 1))
        qsgw.synchronize()
        assert _same(got, ref)
        # after a synchronisation the image is made again from the (changed) host array
        got[...] = 0.0
        _sigc_call(qsgw, got, s, z, wi, wr, 1.0 / 64)
        qsgw.synchronize()
    finally:
        qsgw.set_host_async(False)
    ref2 = np.zeros((ntq, ntq), complex, order='F')
    _sigc_call(qsgw, ref2, s, s['z'], s['wi'], s['wr'], 1.0 / 64)
    assert _same(got, ref2)


def test_chi0_and_sigc_async_interleaved(qsgw):
    """Two chi0 calls into two outputs and Sigma_c calls into two zsec arrays,
    all enqueued before one synchronisation (both staging slots in use)."""
    import torch
    keep = []
    probs = [synth.chi0_problem(N=64, nk=2, nocc=2, nun=(8, 8), niw=4, seed=sd) for sd in (4, 9)]

    def chi0(out, p):
        qsgw.chi0_lorentz_d(out, p['N'], p['niw'], p['freq_i'], p['nk'], p['nocc'], p['nun'], p['eocc_h'],
                            p['eun_h'], p['zc_host'], host=True)

    refs = []
    for p in probs:
        p['zc_host'] = np.asfortranarray(p['zcols'])
        r = np.zeros(p['N'] * p['N'] * p['niw'], complex)
        chi0(r, p)
        refs.append(r)
    s = inputs()['sc']
    ntq = s['ntq']
    zref = [np.zeros((ntq, ntq), complex, order='F') for _ in range(2)]
    for i, zr in enumerate(zref):
        _sigc_call(qsgw, zr, s, s['z'], s['wi'], s['wr'], 0.5 + i)

    outs = [_pinned(torch, keep, np.zeros(p['N'] * p['N'] * p['niw'], complex)) for p in probs]
    for p in probs:
        p['zc_host'] = _pinned(torch, keep, np.asfortranarray(p['zcols']))
    z, wi, wr = (_pinned(torch, keep, s[k]) for k in ('z', 'wi', 'wr'))
    zgot = [_pinned(torch, keep, np.zeros((ntq, ntq), complex)) for _ in range(2)]
    qsgw.set_host_async(True)
    try:
        chi0(outs[0], probs[0])
        _sigc_call(qsgw, zgot[0], s, z, wi, wr, 0.5)
        chi0(outs[1], probs[1])
        _sigc_call(qsgw, zgot[1], s, z, wi, wr, 1.5)
        qsgw.synchronize()
    finally:
        qsgw.set_host_async(False)
    for o, r in zip(outs, refs):
        assert _same(o, r)
    for zg, zr in zip(zgot, zref):
        assert _same(zg, zr)


def test_async_with_pageable_arrays(qsgw):
    """Plain numpy (pageable) host arrays in the asynchronous mode: the copies
    stop overlapping, the results stay those of the synchronous calls."""
    s = inputs()['sc']
    ntq = s['ntq']
    ref = np.zeros((ntq, ntq), complex, order='F')
    for task in range(2):
        _sigc_call(qsgw, ref, s, s['z'], s['wi'], s['wr'], 0.5 * (task + 1))
    got = np.zeros((ntq, ntq), complex, order='F')
    qsgw.set_host_async(True)
    try:
        for task in range(2):
            _sigc_call(qsgw, got, s, s['z'], s['wi'], s['wr'], 0.5 * (task + 1))
        qsgw.synchronize()
    finally:
        qsgw.set_host_async(False)
    assert _same(got, ref)
