"""Index map of presplit_z_kernel (ecalj_b200/csrc/split_f16.cu), emulated on
the CPU block by block and thread by thread: the kernel loads a 64-row x 32-k
tile of Z into shared memory along m and stores it along k.  Every half2 word
of the A' layout of the chi0 split GEMM -- slice s in {hi, lo}, row
t*128 + mm holding [Re a, -Im a] and row t*128 + 64 + mm holding [Im a, Re a]
of a(m, k) = conj(Z(m, k)), m = t*64 + mm, zero where m >= M or k >= K --
must be written exactly once, inside the two slices, from the right element."""
import itertools

import pytest


def _emulate(M, K, T, Ta, Kp):
    KH = Kp // 2
    gx, gy = (KH + 31) // 32, min(T, 65535)
    slice_elems = Ta * 128 * Kp
    writes = {}
    for bx, by in itertools.product(range(gx), range(gy)):
        k0 = bx * 32
        for t in range(by, T, gy):
            st = {}
            for tx, ty, j, it in itertools.product(range(32), range(8), range(4), range(2)):
                kk, mm = ty + 8 * j, tx + 32 * it
                assert 0 <= kk < 32 and 0 <= mm < 64                       # shared-memory bounds
                m, k = t * 64 + mm, k0 + kk
                elem = (m, k) if (m < M and k < K) else None
                for q in range(4):
                    st[(q, mm, kk)] = (elem, q)
            for tx, ty in itertools.product(range(32), range(8)):
                k = k0 + tx
                if k >= KH:
                    continue
                for r in range(ty, 64, 8):
                    row0 = t * 128 + r
                    for q, (row, sl) in enumerate(((row0, 0), (row0, 1), (row0 + 64, 0), (row0 + 64, 1))):
                        idx = sl * slice_elems + row * Kp + 2 * k
                        assert 0 <= idx and idx + 1 < 2 * slice_elems            # global bounds
                        assert idx not in writes                                # written once
                        writes[idx] = st[(q, r, tx)]
    return writes, slice_elems


@pytest.mark.parametrize("M,npair", [(131, 77), (64, 32), (200, 150), (70, 5)])
def test_presplit_z_map(M, npair):
    KC = 64
    Kp = ((2 * npair + KC - 1) // KC) * KC
    T, Tn = (M + 63) // 64, (M + 127) // 128
    Ta = max(T, 2 * Tn)
    writes, slice_elems = _emulate(M, npair, T, Ta, Kp)
    assert len(writes) == 2 * T * 128 * (Kp // 2)          # every word of the T converted tiles
    for t, r, k in itertools.product(range(T), range(64), range(Kp // 2)):
        m = t * 64 + r
        elem = (m, k) if (m < M and k < npair) else None
        for q, (row, sl) in enumerate(((t * 128 + r, 0), (t * 128 + r, 1), (t * 128 + 64 + r, 0),
                                       (t * 128 + 64 + r, 1))):
            assert writes[sl * slice_elems + row * Kp + 2 * k] == (elem, q)
