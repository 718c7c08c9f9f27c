"""__WVI/__WVR record files: byte layout of the reference (fixed records of
nblochpmx^2 complex, record rec at (rec-1)*recl) and the packed forms the
Sigma_c step keeps (m_sxcf_gemm.f90:325-354)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _stack(rng, n, nrec):
    return rng.standard_normal((n, n, nrec)) + 1j * rng.standard_normal((n, n, nrec))


def _upper(w, ngb):
    i, j = np.triu_indices(ngb)                  # row-major order of (i, j) with i <= j
    order = np.lexsort((i, j))                   # column by column: j major, i minor
    return w[i[order], j[order]]


@pytest.mark.parametrize("kind4", [False, True])
def test_wv_records_roundtrip(qsgw, tmp_path, kind4):
    import torch
    lib = qsgw
    rng = np.random.default_rng(5)
    n, nrec, rec0, ngb = 37, 5, 3, 30
    w = _stack(rng, n, nrec)
    path = tmp_path / "__WVI.7"
    lib.wv_write_d(path, lib.to_device(np.asfortranarray(w)), n, rec0, nrec, kind4)
    dt = np.complex64 if kind4 else np.complex128
    raw = np.fromfile(path, dtype=dt)
    assert raw.size == (rec0 - 1 + nrec) * n * n                     # records 1..rec0-1 are holes
    assert not raw[:(rec0 - 1) * n * n].any()
    rec = raw[(rec0 - 1) * n * n:].reshape(nrec, n * n)
    for r in range(nrec):
        np.testing.assert_array_equal(rec[r], w[:, :, r].astype(dt).ravel(order="F"))
    # full read of records rec0+1 .. rec0+3
    out = torch.zeros(3 * n * n, dtype=torch.complex128, device="cuda")
    lib.wv_read_d(path, out, n, rec0 + 1, 3, kind4)
    got = lib.from_device(out, (n, n, 3))
    np.testing.assert_array_equal(got, w[:, :, 1:4].astype(dt).astype(np.complex128))
    # packed forms of the leading ngb block
    ntri = ngb * (ngb + 1) // 2
    for pack in (1, 2):
        out = torch.zeros(nrec * ntri, dtype=torch.complex128, device="cuda")
        lib.wv_read_d(path, out, n, rec0, nrec, kind4, pack=pack, ngb=ngb)
        got = out.cpu().numpy().reshape(nrec, ntri)
        for r in range(nrec):
            m = w[:, :, r].astype(dt).astype(np.complex128)
            ref = _upper(m if pack == 1 else 0.5 * (m + m.conj().T), ngb)
            np.testing.assert_allclose(got[r], ref, rtol=0, atol=1e-15 * np.abs(ref).max())


def test_wv_read_errors(qsgw, tmp_path):
    import torch
    lib = qsgw
    out = torch.zeros(16, dtype=torch.complex128, device="cuda")
    with pytest.raises(lib.QSGWError):
        lib.wv_read_d(tmp_path / "missing", out, 4, 1, 1)
    p = tmp_path / "__WVR.1"
    lib.wv_write_d(p, out, 4, 1, 1)
    with pytest.raises(lib.QSGWError) as e:                          # record 2 is past the end
        lib.wv_read_d(p, out, 4, 2, 1)
    assert "short file" in str(e.value)
