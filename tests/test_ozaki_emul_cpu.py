"""The CPU emulation of the int8 Ozaki scheme (tests/ozaki_emul.py), which
the GPU tests use as the exact reference of the SPLIT_I8 kernels: its slices
stay in int8 range and rebuild each element to 2^-(7 ns) (base-128 digits) or
about 2^-(8 ns) (base-256 digits) of the row scale, and its products converge
to the FP64 product as the slice count grows."""
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


def test_base256_slices_use_the_whole_int8_range_and_rebuild_the_value():
    rng = np.random.default_rng(4)
    x = rng.standard_normal((40, 300)) * 10.0 ** rng.uniform(-3, 3, (40, 1))
    x[0, :4] = [1.0, -1.0, 0.5, -0.75]              # values at the scale itself
    mu = ozaki_emul.pow2_at_least(np.abs(x).max(axis=1))[:, None]
    for ns in (2, 3, 4):
        u = ozaki_emul.unit(ns, 8)
        assert u < 2.0 ** (8 * ns - 1) and u > 0.98 * 2.0 ** (8 * ns - 1)
        s = ozaki_emul.slices(x, mu, ns, bits=8)
        lo = min(si.min() for si in s)
        hi = max(si.max() for si in s)
        assert lo >= -128 and hi <= 127 and lo == -128 and hi == 127
        back = sum(si * 256.0 ** (ns - 1 - i) for i, si in enumerate(s)) * (mu / u)
        assert np.max(np.abs(back - x) / mu) <= 0.5 / u * (1 + 1e-12)


def test_base256_top_digit_stays_in_range_at_the_extremes():
    # every integer V with |V| <= U has digits in [-128, 127]: the extremes and their neighbours
    for ns in (2, 3, 4):
        u = int(ozaki_emul.unit(ns, 8))
        v = np.array([u, u - 1, -u, -u + 1, 0, 127, -128, 128, -129], np.float64)
        s = ozaki_emul.slices(v, u, ns, bits=8)          # mu = U: V = v exactly
        assert all(si.min() >= -128 and si.max() <= 127 for si in s)
        back = sum(si * 256 ** (ns - 1 - i) for i, si in enumerate(s))
        assert np.array_equal(back, v.astype(np.int64))


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
    # base-256 digits: one bit more per slice, so each count is several times closer
    e8 = [np.linalg.norm(ozaki_emul.complex_product(a, b, ns, bits=8) - ref) / np.linalg.norm(ref)
          for ns in (2, 3, 4)]
    assert e8[0] > e8[1] > e8[2]
    assert all(e8[i] < errs[i] / 3 for i in range(3))


def test_chi0_emulation_matches_the_direct_sum():
    rng = np.random.default_rng(7)
    z = (rng.standard_normal((24, 150)) + 1j * rng.standard_normal((24, 150))) / 5.0
    w = -rng.uniform(0.1, 3.0, (3, 150))
    w[2, :40] *= -1.0                          # one slot with weights of both signs
    ref = np.stack([(np.conj(z) * w[j]) @ z.T for j in range(3)], axis=2)
    got = ozaki_emul.chi0_dense(z, w, 4)
    assert np.linalg.norm(got - ref) / np.linalg.norm(ref) < 1e-6


def test_base256_product_equals_exact_integer_sum_of_the_kept_pairs():
    """The emulated base-256 product against the same sum formed in exact
    integers: (mu_m nu_n / U^2) sum_k sum_{p + q <= ns - 1} A_p B_q 256^(2 (ns - 1) - p - q),
    with the A' rows [Re a, -Im a] and [Im a, Re a] sliced value by value."""
    from fractions import Fraction
    rng = np.random.default_rng(11)
    a = rng.standard_normal((3, 7)) + 1j * rng.standard_normal((3, 7))
    b = rng.standard_normal((7, 2)) + 1j * rng.standard_normal((7, 2))
    for ns in (2, 3):
        got = ozaki_emul.complex_product(a, b, ns, bits=8)
        mu = ozaki_emul.max_scale(np.maximum(np.abs(a.real), np.abs(a.imag)).max(axis=1))
        nu = ozaki_emul.max_scale(np.maximum(np.abs(b.real), np.abs(b.imag)).max(axis=0))
        u = int(ozaki_emul.unit(ns, 8))
        sl = {name: ozaki_emul.slices(x, sc, ns, bits=8) for name, x, sc in
              (("ar", a.real, mu[:, None]), ("ai", a.imag, mu[:, None]), ("an", -a.imag, mu[:, None]),
               ("br", b.real, nu[None, :]), ("bi", b.imag, nu[None, :]))}

        def level_sum(x, y, m, n):
            return sum(int(sl[x][p][m, k]) * int(sl[y][q][k, n]) * 256 ** (2 * (ns - 1) - p - q)
                       for k in range(7) for p in range(ns) for q in range(ns - p))
        for m in range(3):
            for n in range(2):
                f = Fraction(float(mu[m])) * Fraction(float(nu[n])) / (u * u)
                re = f * (level_sum("ar", "br", m, n) + level_sum("an", "bi", m, n))
                im = f * (level_sum("ai", "br", m, n) + level_sum("ar", "bi", m, n))
                assert abs(got[m, n].real - float(re)) <= 1e-14 * abs(float(re)) + 1e-300
                assert abs(got[m, n].imag - float(im)) <= 1e-14 * abs(float(im)) + 1e-300
