"""The allocation-free batched HPD inverse (qsgw_zminv_hpd_batched_noalloc_d),
for callers that cannot allocate device memory, checked through the C ABI
against the allocating entry point, on two calls in a row.  This file is
collected last so that a stop-at-first-failure run has run everything else."""
import numpy as np
import pytest

from tests.conftest import rel_fro

pytestmark = pytest.mark.gpu
TOL = 1e-11          # the FP64 parity tolerance of the other GPU tests


def _hpd_batch(n, nb, seed):
    rng = np.random.default_rng(seed)
    a = np.zeros((n, n, nb), complex, order='F')
    for b in range(nb):
        g = rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))
        a[:, :, b] = np.eye(n) + 0.4 * g @ g.conj().T / n
    return a


def test_noalloc_matches_allocating_entry_point_twice(qsgw):
    import torch
    stream = torch.cuda.current_stream().cuda_stream
    for n, nb, seed in [(100, 4, 1), (257, 3, 2)]:      # two calls in a row, different shapes
        a = _hpd_batch(n, nb, seed)
        ref = qsgw.to_device(a)
        qsgw.zminv_hpd_batched_d(ref, n, n, nb)
        qsgw.synchronize()
        got = qsgw.to_device(a)
        torch.cuda.synchronize()
        qsgw.zminv_hpd_batched_noalloc_d(got, n, n, nb, stream)
        torch.cuda.synchronize()
        assert rel_fro(qsgw.from_device(got, a.shape), qsgw.from_device(ref, a.shape)) < TOL


def test_noalloc_status_is_cleared_between_calls(qsgw):
    import torch
    n, nb = 48, 2
    sing = qsgw.to_device(np.zeros((n, n, nb), complex, order='F'))
    with pytest.raises(qsgw.QSGWError) as e:
        qsgw.zminv_hpd_batched_noalloc_d(sing, n, n, nb)
    assert e.value.code == -5
    a = _hpd_batch(n, nb, 3)
    got = qsgw.to_device(a)
    qsgw.zminv_hpd_batched_noalloc_d(got, n, n, nb)
    torch.cuda.synchronize()
    inv = qsgw.from_device(got, a.shape)
    for b in range(nb):
        assert rel_fro(inv[:, :, b], np.linalg.inv(a[:, :, b])) < TOL


def test_noalloc_rejects_sizes_beyond_the_limit(qsgw):
    import torch
    t = torch.zeros(4, dtype=torch.complex128, device='cuda')
    with pytest.raises(qsgw.QSGWError) as e:
        qsgw.zminv_hpd_batched_noalloc_d(t, 8193, 8193, 2)
    assert e.value.code == -1 and "16384" in str(e.value)


_NO_INIT_SCRIPT = r"""
import sys
import numpy as np
import torch
sys.path.insert(0, {root!r})
from ecalj_b200 import lib
from tests.test_zz_no_alloc import _hpd_batch
dev = {dev}
torch.cuda.set_device(dev)
lib.load()                                   # no qsgw_init: the call needs no library context
assert not lib.initialized()
side = torch.cuda.Stream()                   # not the default stream
for n, nb, seed in [(64, 3, 5), (130, 2, 6)]:
    a = _hpd_batch(n, nb, seed)
    with torch.cuda.stream(side):
        t = torch.from_numpy(a.reshape(-1, order='F').copy()).to('cuda')
    side.synchronize()
    lib.zminv_hpd_batched_noalloc_d(t, n, n, nb, side.cuda_stream)
    got = t.cpu().numpy().reshape(a.shape, order='F')
    for b in range(nb):
        ref = np.linalg.inv(a[:, :, b])
        err = np.linalg.norm(got[:, :, b] - ref) / np.linalg.norm(ref)
        assert err < 1e-11, (n, b, err)
print("ok")
"""


def _run_fresh(dev):
    import os
    import subprocess
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    code = _NO_INIT_SCRIPT.format(root=root, dev=dev)
    r = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=600, cwd=root)
    assert r.returncode == 0 and r.stdout.strip().endswith("ok"), r.stdout[-2000:] + r.stderr[-2000:]


def test_noalloc_without_init_on_a_side_stream_in_a_fresh_process():
    """The documented use: a caller that never ran qsgw_init, on a stream of
    its own, in a process where nothing else touched the library."""
    _run_fresh(0)


def test_noalloc_on_a_second_device():
    """The static array and the raised shared-memory limit of the GEMM kernel
    are per device: the first call on device 1 must set both up there."""
    import torch
    if torch.cuda.device_count() < 2:
        pytest.skip("one visible GPU")
    _run_fresh(1)


def test_noalloc_refuses_a_capturing_stream(qsgw):
    import torch
    n, nb = 32, 1
    t = qsgw.to_device(_hpd_batch(n, nb, 7))
    s = torch.cuda.Stream()
    g = torch.cuda.CUDAGraph()
    err = None
    with torch.cuda.stream(s):
        g.capture_begin()
        try:
            qsgw.zminv_hpd_batched_noalloc_d(t, n, n, nb, s.cuda_stream)
        except qsgw.QSGWError as e:
            err = e
        finally:
            g.capture_end()
    assert err is not None and err.code == -7          # QSGW_ERR_UNSUPPORTED
