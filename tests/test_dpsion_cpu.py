"""Oracle of the histogram Hilbert transform (oracle/dpsion.py) pinned to
its mathematical definition: hilbertmat's weights against adaptive
quadrature of int f(w) / (w - z) dw for the piecewise-linear f the reference
assumes, and chi0(i w) of one narrow transition against the analytic
-2 W De / (De^2 + w^2), the Lorentzian form of the direct imaginary-axis path."""
import numpy as np
import pytest
from scipy.integrate import quad

from oracle import dpsion as dp


def _mesh(nwhis, dw=0.02, ratio=1.15):
    """frhis(i) = bb (exp(aa (i-1)) - 1) as m_freq.f90:98-108."""
    aa = ratio - 1.0
    return dw / aa * (np.exp(aa * np.arange(nwhis + 1)) - 1.0)


def _quad_hilbert(z, L, C, R, f):
    nwhis = (len(C) - 1) // 2
    xs = np.concatenate([[L[0]], C[:nwhis], [0.0], C[nwhis + 1:], [R[-1]]])
    ys = np.concatenate([[0.0], f[:nwhis], [0.0], f[nwhis + 1:], [0.0]])
    tot = 0j
    for a, b, fa, fb in zip(xs[:-1], xs[1:], ys[:-1], ys[1:]):
        def g(w):
            return (fa + (fb - fa) * (w - a) / (b - a)) / (w - z)
        tot += quad(lambda w: g(w).real, a, b, epsabs=1e-14, epsrel=1e-12)[0]
        tot += 1j * quad(lambda w: g(w).imag, a, b, epsabs=1e-14, epsrel=1e-12)[0]
    return tot


def test_bins_mirror():
    fr = _mesh(9)
    L, C, R = dp.histogram_bins(fr)
    assert np.allclose(L[10:], fr[:9]) and np.allclose(R[10:], fr[1:])
    assert np.allclose(L[:9], -fr[9:0:-1]) and np.allclose(R[:9], -fr[8::-1])
    assert np.allclose(C[:9], -C[10:][::-1])


@pytest.mark.parametrize("z", [0.05j, 0.3j, 1.7j, 2.5, -3.0])
def test_hilbertmat_vs_quadrature(z):
    fr = _mesh(14)
    L, C, R = dp.histogram_bins(fr)
    f = np.random.default_rng(1).standard_normal(len(C))
    f[14] = 0.0
    got = np.dot(dp.hilbertmat(z, L, C, R), f)
    ref = _quad_hilbert(z, L, C, R, f)
    assert abs(got - ref) <= 1e-10 * abs(ref)


def test_narrow_transition_lorentzian():
    """A transition of weight W (|z|^2 / nk) at De in a fine bin: x0gemm stores rcxq = pi W (positive;
    -rcxq / (R - L) is the bin average of Im chi0), and chi0(i w) -> -2 W De / (De^2 + w^2)."""
    fr = _mesh(400, dw=1e-3, ratio=1.01)
    nwhis = len(fr) - 1
    b = 250
    de = 0.5 * (fr[b - 1] + fr[b])
    W = 0.7
    rcxq = np.zeros((1, 1, nwhis + 1), complex)
    rcxq[0, 0, b] = W * np.pi
    wi = np.array([0.01, 0.1, 0.5, 2.0])
    zxqi, _ = dp.dpsion_chiq(rcxq, fr, wi)
    ref = -2.0 * W * de / (de ** 2 + wi ** 2)
    assert np.allclose(zxqi[0, 0].real, ref, rtol=2e-2)
    assert np.allclose(zxqi[0, 0].imag, 0.0, atol=1e-12)


def test_real_axis_imaginary_part_is_the_bin_average():
    fr = _mesh(30)
    nwhis = len(fr) - 1
    rng = np.random.default_rng(4)
    rcxq = rng.standard_normal((3, 2, nwhis + 1)) + 1j * rng.standard_normal((3, 2, nwhis + 1))
    freq_r = np.concatenate([[0.0], 0.5 * (fr[:10] + fr[1:11])])
    zxqi, zxq = dp.dpsion_chiq(rcxq, fr, np.array([0.2]), freq_r)
    L, C, R = dp.histogram_bins(fr)
    imatt, rmatt = dp.transform_matrices(fr, [0.2], freq_r)
    for t in range(1, 11):
        norm = -1.0 / (R[nwhis + t] - L[nwhis + t])
        hil = np.einsum('abk,k->ab', rcxq[:, :, 1:] * (-1.0 / (R[nwhis + 1:] - L[nwhis + 1:])), rmatt[t])
        assert np.allclose(zxq[:, :, t], 1j * norm * rcxq[:, :, t] + hil)
    assert np.allclose(zxq[:, :, 0], 1j * rcxq[:, :, 0] + np.einsum(
        'abk,k->ab', rcxq[:, :, 1:] * (-1.0 / (R[nwhis + 1:] - L[nwhis + 1:])), rmatt[0]))


@pytest.mark.parametrize("ecut", [1e10, 0.05])
def test_library_transform_matrix_vs_oracle(ecut):
    """qsgw_dpsion_matrix (host C++, the matrix the GPU contraction applies)
    against the oracle's imatt, rmatt and bin normalisation."""
    from ecalj_b200 import lib
    fr = _mesh(25)
    nwhis = len(fr) - 1
    freq_i = np.array([0.01, 0.2, 1.5])
    freq_r = np.concatenate([[0.0], 0.5 * (fr[:8] + fr[1:9])])
    b = lib.dpsion_matrix(fr, freq_i, freq_r, ecut)
    L, C, R = dp.histogram_bins(fr)
    imatt, rmatt = dp.transform_matrices(fr, freq_i, freq_r)
    c = C[nwhis + 1:]
    f = -(np.exp(-(c / ecut) ** 2) if ecut < 1e9 else 1.0) / (R[nwhis + 1:] - L[nwhis + 1:])
    niw = len(freq_i)
    assert np.all(b[0, :niw] == 0)
    assert np.allclose(b[1:, :niw], (f[:, None] * imatt.T), rtol=1e-13, atol=0)
    real = f[:, None] * rmatt.T + 0j
    for t in range(1, len(freq_r)):
        real[t - 1, t] += 1j * f[t - 1]
    assert np.allclose(b[1:, niw:], real, rtol=1e-13, atol=1e-300)
    assert b[0, niw] == 1j and np.all(b[0, niw + 1:] == 0)


def test_library_matrix_with_smear_applies_the_filter():
    """With SmearX0 the library matrix applied to rcxq equals the oracle's filtered transform."""
    from ecalj_b200 import lib
    fr = _mesh(30)
    nwhis = len(fr) - 1
    rng = np.random.default_rng(8)
    rcxq = rng.standard_normal((3, 2, nwhis + 1)) + 1j * rng.standard_normal((3, 2, nwhis + 1))
    freq_i = np.array([0.05, 0.4])
    freq_r = np.concatenate([[0.0], 0.5 * (fr[:9] + fr[1:10])])
    smear = 0.01
    b = lib.dpsion_matrix(fr, freq_i, freq_r, 1e10, smear)
    got = np.einsum('abk,kj->abj', rcxq, b)
    ri, rr = dp.dpsion_chiq(rcxq, fr, freq_i, freq_r, smear=smear)
    ref = np.concatenate([ri, rr], axis=2)
    assert np.allclose(got, ref, rtol=1e-12, atol=1e-12 * np.abs(ref).max())
    g = dp.gaussian_filter(fr, smear)
    assert np.allclose(g.sum(axis=0), 1.0)


def test_library_matrix_argument_checks():
    """The reference's checks (dpsion5.f90:208-209) and the mesh's: errors, no output."""
    from ecalj_b200 import lib
    fr = _mesh(10)
    with pytest.raises(lib.QSGWError):                       # nwhis <= nw
        lib.dpsion_matrix(fr, [0.1], np.concatenate([[0.0], fr[:10]]))
    with pytest.raises(lib.QSGWError):                       # freq_r(0) /= 0
        lib.dpsion_matrix(fr, [0.1], np.array([0.01, 0.02]))
    with pytest.raises(lib.QSGWError):                       # bins not increasing
        lib.dpsion_matrix(fr[::-1].copy(), [0.1])
