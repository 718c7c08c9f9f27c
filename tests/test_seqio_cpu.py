"""Sequential unformatted files of the QSGW chain (host-only, no GPU):
__Vcoud.<iq> (main_hvccfp0.f90:396-400 / m_readVcoud.f90:30-40) and the
SEX2U / SEC2U self-energy files (main_hsfp0.sc.f90:322-359 /
main_hqpe.sc.f90:132-148).  The byte layout is checked against an
independent numpy writer and parser of Fortran records (a 4-byte length,
the payload, the length again), in both directions."""
import ctypes
import struct

import numpy as np
import pytest

from ecalj_b200 import lib


def _records(path):
    """Splits a sequential unformatted file into its record payloads."""
    data = open(path, 'rb').read()
    out, at = [], 0
    while at < len(data):
        (n,) = struct.unpack_from('<i', data, at)
        payload = data[at + 4:at + 4 + n]
        (n2,) = struct.unpack_from('<i', data, at + 4 + n)
        assert n2 == n and len(payload) == n
        out.append(payload)
        at += n + 8
    return out


def _write_records(path, payloads):
    with open(path, 'wb') as f:
        for p in payloads:
            f.write(struct.pack('<i', len(p)) + p + struct.pack('<i', len(p)))


def _vcoud_case(rng, ngb):
    q = rng.standard_normal(3)
    v = 10 ** rng.uniform(-2, 3, ngb)
    z = np.asfortranarray(rng.standard_normal((ngb, ngb)) + 1j * rng.standard_normal((ngb, ngb)))
    return q, v, z


def test_vcoud_write_layout(tmp_path):
    rng = np.random.default_rng(5)
    q, v, z = _vcoud_case(rng, 7)
    p = tmp_path / '__Vcoud.3'
    lib.vcoud_write(p, q, v, z)
    r = _records(p)
    assert len(r) == 4
    assert struct.unpack('<i', r[0]) == (7,)
    np.testing.assert_array_equal(np.frombuffer(r[1], '<f8'), q)
    np.testing.assert_array_equal(np.frombuffer(r[2], '<f8'), v)
    np.testing.assert_array_equal(np.frombuffer(r[3], '<c16').reshape(7, 7, order='F'), z)


def test_vcoud_read_of_fortran_layout(tmp_path):
    """A file laid out as the reference writes it reads back bit for bit; vcousq = sqrt(vcoud)."""
    rng = np.random.default_rng(6)
    q, v, z = _vcoud_case(rng, 9)
    p = tmp_path / '__Vcoud.1'
    _write_records(p, [struct.pack('<i', 9), q.astype('<f8').tobytes(), v.astype('<f8').tobytes(),
                       z.astype('<c16').tobytes(order='F')])
    q2, v2, vs, z2 = lib.vcoud_read(p)
    np.testing.assert_array_equal(q2, q)
    np.testing.assert_array_equal(v2, v)
    np.testing.assert_array_equal(vs, np.sqrt(v))
    np.testing.assert_array_equal(z2, z)


def test_vcoud_read_rejects_other_layouts(tmp_path):
    rng = np.random.default_rng(7)
    q, v, z = _vcoud_case(rng, 4)
    p = tmp_path / 'v'
    # complex(4) eigenvectors: the file is shorter than its header implies
    _write_records(p, [struct.pack('<i', 4), q.tobytes(), v.tobytes(), z.astype('<c8').tobytes(order='F')])
    with pytest.raises(lib.QSGWError, match='holds 220 bytes, its header implies 348'):
        lib.vcoud_read(p)
    # the right total but records cut elsewhere: the record lengths are checked too
    zb = z.astype('<c16').tobytes(order='F')
    _write_records(p, [struct.pack('<i', 4), q.tobytes(), v.tobytes() + zb[:16], zb[16:]])
    with pytest.raises(lib.QSGWError, match='record 3 holds 48 bytes, expected 32'):
        lib.vcoud_read(p)
    # 8-byte record markers (another compiler's option)
    with open(p, 'wb') as f:
        f.write(struct.pack('<q', 4) + struct.pack('<i', 4) + struct.pack('<q', 4))
    with pytest.raises(lib.QSGWError, match='holds 4 bytes, expected 24'):
        lib.vcoud_read(p)
    # a file cut short inside the eigenvector record
    lib.vcoud_write(p, q, v, z)
    data = open(p, 'rb').read()
    open(p, 'wb').write(data[:-40])
    with pytest.raises(lib.QSGWError, match='its header implies'):
        lib.vcoud_read(p)
    with pytest.raises(lib.QSGWError, match='cannot open'):
        lib.vcoud_read(tmp_path / 'missing')


def test_vcoud_capacity_and_query(tmp_path):
    rng = np.random.default_rng(8)
    q, v, z = _vcoud_case(rng, 6)
    p = tmp_path / 'v'
    lib.vcoud_write(p, q, v, z)
    f = lib.load().qsgw_vcoud_read
    n = ctypes.c_int(0)
    qq = np.zeros(3)
    assert f(bytes(p), 0, ctypes.byref(n), qq.ctypes.data, None, None, None) == 0    # size query
    assert n.value == 6 and np.array_equal(qq, q)
    small = np.zeros(5)
    assert f(bytes(p), 5, ctypes.byref(n), None, small.ctypes.data, None, None) == -1
    assert 'ngb = 6' in lib.last_error()
    # vcousq alone (vcoud NULL): the square roots, eigenvectors skipped
    vs = np.zeros(6)
    assert f(bytes(p), 6, ctypes.byref(n), None, None, vs.ctypes.data, None) == 0
    np.testing.assert_array_equal(vs, np.sqrt(v))


def _sigma_case(rng, nq, ntq):
    head = np.array([1, nq, ntq, 64, nq, 4, 4, 4], np.int32)
    qibz = np.asfortranarray(rng.standard_normal((3, nq)))
    zsec = np.asfortranarray(rng.standard_normal((ntq, ntq, nq)) + 1j * rng.standard_normal((ntq, ntq, nq)))
    return head, qibz, zsec


def test_sigma_write_layout(tmp_path):
    rng = np.random.default_rng(9)
    head, qibz, zsec = _sigma_case(rng, 3, 5)
    p = tmp_path / 'SEC2U'
    lib.sigma_write(p, head, 1, qibz, zsec)
    r = _records(p)
    assert len(r) == 1 + 3
    assert struct.unpack('<8i', r[0]) == tuple(int(h) for h in head)
    for ip in range(3):
        assert len(r[1 + ip]) == 4 + 24 + 16 * 25
        assert struct.unpack_from('<i', r[1 + ip]) == (1,)
        np.testing.assert_array_equal(np.frombuffer(r[1 + ip], '<f8', 3, 4), qibz[:, ip])
        np.testing.assert_array_equal(np.frombuffer(r[1 + ip], '<c16', 25, 28).reshape(5, 5, order='F'),
                                      zsec[:, :, ip])


def test_sigma_read_of_fortran_layout(tmp_path):
    rng = np.random.default_rng(10)
    head, qibz, zsec = _sigma_case(rng, 4, 3)
    head[0] = 2
    p = tmp_path / 'SEX2D'
    recs = [head.astype('<i4').tobytes()]
    for ip in range(4):
        recs.append(struct.pack('<i', 2) + qibz[:, ip].astype('<f8').tobytes()
                    + zsec[:, :, ip].astype('<c16').tobytes(order='F'))
    _write_records(p, recs)
    h, isx, q, z = lib.sigma_read(p)
    np.testing.assert_array_equal(h, head)
    assert list(isx) == [2] * 4
    np.testing.assert_array_equal(q, qibz)
    np.testing.assert_array_equal(z, zsec)


def test_sigma_round_trip_and_errors(tmp_path):
    rng = np.random.default_rng(11)
    head, qibz, zsec = _sigma_case(rng, 2, 4)
    p = tmp_path / 'SEXcore2U'
    lib.sigma_write(p, head, 1, qibz, zsec)
    h, isx, q, z = lib.sigma_read(p)
    np.testing.assert_array_equal(h, head)
    np.testing.assert_array_equal(z, zsec)
    # no q records (nq = 0): the header alone
    h0 = head.copy()
    h0[1] = 0
    lib.sigma_write(p, h0, 1, np.zeros((3, 0)), np.zeros((4, 4, 0), complex))
    h, isx, q, z = lib.sigma_read(p)
    assert h[1] == 0 and z.shape == (4, 4, 0) and len(_records(p)) == 1
    # header promising more q records than the file holds
    lib.sigma_write(p, head, 1, qibz, zsec)
    data = open(p, 'rb').read()
    rec = 8 + 4 + 24 + 16 * 16
    open(p, 'wb').write(data[:len(data) - rec])
    with pytest.raises(lib.QSGWError, match='holds 332 bytes, its header implies 624'):
        lib.sigma_read(p)
    # a header claiming 10^9 q records is refused before any array is sized from it
    h_big = head.copy()
    h_big[1] = 10 ** 9
    data = open(p, 'rb').read()
    open(p, 'wb').write(struct.pack('<i', 32) + h_big.astype('<i4').tobytes() + struct.pack('<i', 32) + data[40:])
    with pytest.raises(lib.QSGWError, match='its header implies'):
        lib.sigma_read(p)
    with pytest.raises(ValueError):
        lib.sigma_write(p, head, 1, qibz, zsec[:, :, :1])
