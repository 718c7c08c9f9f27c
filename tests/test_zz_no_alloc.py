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
