"""The CPU emulation of the int8 Ozaki scheme (tests/ozaki_emul.py), which
the GPU tests use as the exact reference of the SPLIT_I8 kernels: its slices
stay in int8 range and rebuild each element to 2^-(7 ns) of the row scale,
and its products converge to the FP64 product as the slice count grows."""
import numpy as np

from tests import ozaki_emul


def test_slices_fit_int8_and_rebuild_the_value():
    rng = np.random.default_rng(3)
    x = rng.standard_normal((40, 300)) * 10.0 ** rng.uniform(-3, 3, (40, 1))
    mu = ozaki_emul.pow2_at_least(np.abs(x).max(axis=1))[:, None]
    for ns in (2, 3, 4):
        s = ozaki_emul.slices(x, mu, ns)
        assert all(np.abs(si).max() <= 64 for si in s)
        back = sum(si * 2.0 ** (-6 - 7 * i) for i, si in enumerate(s)) * mu
        assert np.max(np.abs(back - x) / mu) <= 2.0 ** (-7 * ns)
        # negation commutes with the slicing (rint is symmetric)
        sn = ozaki_emul.slices(-x, mu, ns)
        assert all(np.array_equal(a, -b) for a, b in zip(s, sn))


def test_powers_of_two_bound_the_maximum():
    m = np.array([0.0, 1.0, 0.75, 3.0, 1e-300, 2.0 ** 40])
    p = ozaki_emul.pow2_at_least(m)
    assert np.all(p >= m) and np.all(np.log2(p) == np.round(np.log2(p)))
    assert np.all(p[m > 0] <= 2 * m[m > 0])


def test_complex_product_converges_with_the_slice_count():
    rng = np.random.default_rng(5)
    a = rng.standard_normal((33, 200)) + 1j * rng.standard_normal((33, 200))
    b = rng.standard_normal((200, 21)) + 1j * rng.standard_normal((200, 21))
    ref = a @ b
    errs = [np.linalg.norm(ozaki_emul.complex_product(a, b, ns) - ref) / np.linalg.norm(ref) for ns in (2, 3, 4)]
    assert errs[0] < 1e-3 and errs[1] < 1e-5 and errs[2] < 1e-7
    assert errs[0] > errs[1] > errs[2]


def test_chi0_emulation_matches_the_direct_sum():
    rng = np.random.default_rng(7)
    z = (rng.standard_normal((24, 150)) + 1j * rng.standard_normal((24, 150))) / 5.0
    w = -rng.uniform(0.1, 3.0, (3, 150))
    w[2, :40] *= -1.0                          # one slot with weights of both signs
    ref = np.stack([(np.conj(z) * w[j]) @ z.T for j in range(3)], axis=2)
    got = ozaki_emul.chi0_dense(z, w, 4)
    assert np.linalg.norm(got - ref) / np.linalg.norm(ref) < 1e-6
