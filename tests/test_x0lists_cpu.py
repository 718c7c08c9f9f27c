"""qsgw_x0_lists (host-only) against the dense contraction: the pair/bin
lists it builds, fed to the x0gemm oracle k by k, must reproduce
rcxq(:, :, bin) = sum_{k, ib, jb} w[k, ib, jb, bin] conj(z) z^T."""
import numpy as np
import pytest

from ecalj_b200 import lib
from oracle import x0


def _weights(rng, nk, nocc, nunocc, nwhis):
    w = rng.uniform(0.0, 1.0, (nk, nocc, nunocc, nwhis))
    w[rng.uniform(size=w.shape) < 0.6] = 0.0      # holes inside the bin ranges
    w[:, :, 1, :] = 0.0                             # a band pair that never contributes
    w[2] = 0.0                                      # a k-point without pairs
    return w


def test_lists_reproduce_dense_contraction():
    rng = np.random.default_rng(11)
    nk, nocc, nunocc, nwhis, npr = 5, 3, 4, 12, 7
    w = _weights(rng, nk, nocc, nunocc, nwhis)
    t = lib.x0_lists(w)
    assert t["icounkmin"][2] == t["icounkmax"][2] + 1          # empty k
    z = [np.asfortranarray(rng.standard_normal((npr, nocc, nunocc)) + 1j * rng.standard_normal((npr, nocc, nunocc)))
         for _ in range(nk)]
    got = np.zeros((npr, npr, nwhis + 1), complex, order='F')
    for k in range(nk):
        x0.x0gemm(got, npr, 1, npr, nwhis, 1, 1, nocc, z[k], 1, int(t["icounkmin"][k]), int(t["icounkmax"][k]),
                  t["itc"], t["itpc"], t["jpmc"], t["iwini"], t["iwend"], t["icouini"], t["whwc"])
    ref = np.zeros_like(got)
    for k in range(nk):
        for ib in range(nocc):
            for jb in range(nunocc):
                zz = z[k][:, ib, jb]
                for h in range(nwhis):
                    ref[:, :, h + 1] += w[k, ib, jb, h] * np.outer(zz.conj(), zz)
    assert np.allclose(got, ref, rtol=0, atol=1e-12 * np.abs(ref).max())
    assert np.all(t["itpc"][:t["ncoun"]] != 2)                  # jb = 1 never listed


def test_lists_empty_and_capacity():
    w = np.zeros((3, 2, 2, 5))
    t = lib.x0_lists(w)
    assert t["ncoun"] == 0 and t["ncount"] == 0
    assert np.all(t["icounkmin"] == 1) and np.all(t["icounkmax"] == 0)
    w[1, 0, 1, 2] = 0.5
    import ctypes
    nc, nt = ctypes.c_int(0), ctypes.c_int(0)          # job 1 with no room: an argument error, no write
    arr = np.zeros(1, np.int32)
    rc = lib.load().qsgw_x0_lists(w.ctypes.data, 3, 2, 2, 5, 1, ctypes.byref(nc), ctypes.byref(nt),
                                  *[arr.ctypes.data] * 6, np.zeros(1).ctypes.data, arr.ctypes.data, arr.ctypes.data)
    assert lib.STATUS[rc] == "ERR_ARG"


def test_lists_argument_checks():
    import ctypes
    w = np.zeros((2, 2, 2, 3))
    nc, nt = ctypes.c_int(0), ctypes.c_int(0)
    f = lib.load().qsgw_x0_lists
    assert lib.STATUS[f(w.ctypes.data, 2, 2, 2, 3, 2, ctypes.byref(nc), ctypes.byref(nt), *([None] * 9))] == "ERR_ARG"
    assert lib.STATUS[f(w.ctypes.data, 0, 2, 2, 3, 0, ctypes.byref(nc), ctypes.byref(nt), *([None] * 9))] == "ERR_ARG"
    assert lib.STATUS[f(w.ctypes.data, 2, 2, 2, 3, 1, ctypes.byref(nc), ctypes.byref(nt), *([None] * 9))] == "ERR_ARG"
