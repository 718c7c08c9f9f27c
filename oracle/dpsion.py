"""Hilbert transform of the chi0 histogram (test infrastructure): a plain
numpy restatement of

* hilbertmat (SRC/subroutines/hilbertmat.f90:14-79): weights rmat(i) with
  H(z) = int f(w) / (w - z) dw = sum_{i != 0} rmat(i) f(i) for f linear
  between the bin centres, zero at w = 0 and at the outer edges;
* dpsion_init (SRC/subroutines/dpsion5.f90:77-137), time reversal (npm = 1):
  the bins [his_L, his_R] on both sides of zero, imatt(j, i) =
  Re[rmat(i) - rmat(-i)] / pi at z = i freq_i(j), rmatt(it, i) =
  Re[rmat(i) - rmat(-i)] / pi at z = freq_r(it);
* dpsion_chiq (dpsion5.f90:174-292), npm = 1, no chi+-: the optional SmearX0
  filter rcxq(bins) <- rcxq(bins) . gfmat^T (:174-193, gaussianfilterhis
  :459-483), rcxq(bin) <- -wfac / (R - L) rcxq(bin) for bins 1..nwhis, then
  zxqi = rcxq . imatt^T and, on the real axis, chi0(freq_r(it)) =
  i rcxq(it) + rcxq . rmatt(it, :)^T.

Energies in Hartree as the reference's m_freq (frhis, freq_r, freq_i)."""
import numpy as np

EPS = 1e-8          # hilbertmat2's |z - a|, |z - b| threshold
EPSZ = 1e-13        # the small positive imaginary part added to z


def histogram_bins(frhis):
    """his_L, his_C, his_R over bins -nwhis..nwhis (index i + nwhis), as
    dpsion5.f90:87-89: bin i > 0 is [frhis(i), frhis(i+1)], bin -i its mirror,
    bin 0 a placeholder at zero."""
    frhis = np.asarray(frhis, dtype=np.float64)
    nwhis = len(frhis) - 1
    L = np.concatenate([-frhis[nwhis:0:-1], [0.0], frhis[:nwhis]])
    R = np.concatenate([-frhis[nwhis - 1::-1], [0.0], frhis[1:nwhis + 1]])
    return L, 0.5 * (L + R), R


def _hm2(z, a, b):
    """int_a^b (m w + n) / (w - z) dw = m facm + n facn (hilbertmat.f90:57-69)."""
    db, da = z - b, z - a
    if abs(da) > EPS and abs(db) > EPS:
        facn = np.log(db / da)
        return z * facn + (b - a), facn
    return 0.0 + 0.0j, 0.0 + 0.0j


def hilbertmat(z, L, C, R):
    """rmat over bins -nwhis..nwhis (index i + nwhis); rmat at bin 0 unused."""
    nwhis = (len(C) - 1) // 2
    rmat = np.zeros(2 * nwhis + 1, dtype=np.complex128)
    zz = complex(z) + 1j * EPSZ
    for iw in range(-nwhis, nwhis + 1):
        if iw == 0:
            continue
        k = iw + nwhis
        ci = C[k]
        cim = L[k] if iw == -nwhis else (0.0 if iw == 1 else C[k - 1])
        facm, facn = _hm2(zz, L[k], C[k])
        rmat[k] += (facm - facn * cim) / (ci - cim)
        if iw != -nwhis and iw != 1:
            rmat[k - 1] += (-facm + facn * ci) / (ci - cim)
        cip = R[k] if iw == nwhis else (0.0 if iw == -1 else C[k + 1])
        facm, facn = _hm2(zz, C[k], R[k])
        rmat[k] += (-facm + facn * cip) / (cip - ci)
        if iw != nwhis and iw != -1:
            rmat[k + 1] += (facm - facn * ci) / (cip - ci)
    return rmat


def transform_matrices(frhis, freq_i, freq_r=None):
    """imatt (niw, nwhis) and rmatt (nw+1, nwhis) of dpsion_init, npm = 1."""
    L, C, R = histogram_bins(frhis)
    nwhis = len(frhis) - 1
    pos = np.arange(nwhis + 1, 2 * nwhis + 1)          # bins 1..nwhis
    neg = np.arange(nwhis - 1, -1, -1)                 # bins -1..-nwhis
    imatt = np.empty((len(freq_i), nwhis))
    for j, w in enumerate(freq_i):
        r = hilbertmat(1j * w, L, C, R)
        imatt[j] = np.real(r[pos] - r[neg]) / np.pi
    rmatt = None
    if freq_r is not None:
        rmatt = np.empty((len(freq_r), nwhis))
        for it, w in enumerate(freq_r):
            r = hilbertmat(w, L, C, R)
            rmatt[it] = np.real(r[pos]) / np.pi - np.real(r[neg]) / np.pi
    return imatt, rmatt


def gaussian_filter(frhis, smear):
    """gfmat (nwhis, nwhis) of gaussianfilterhis (dpsion5.f90:459-483): column i is
    exp(-(c_i - c_j)^2 / (2 smear^2)) over j, normalised to sum 1, c = bin centres."""
    frhis = np.asarray(frhis, dtype=np.float64)
    c = 0.5 * (frhis[:-1] + frhis[1:])
    g = np.exp(-(c[None, :] - c[:, None]) ** 2 / (2.0 * smear ** 2))   # g[j, i]
    return g / g.sum(axis=0)[None, :]


def dpsion_chiq(rcxq, frhis, freq_i, freq_r=None, ecut=1e10, smear=0.0):
    """rcxq (npr, npr_col, nwhis+1): the x0gemm histogram, slots 0..nwhis.
    Returns zxqi (npr, npr_col, niw) and, with freq_r, zxq (npr, npr_col,
    nw+1) = the real-axis chi0 the reference leaves in rcxq(:, :, 0:nw)."""
    L, C, R = histogram_bins(frhis)
    nwhis = len(frhis) - 1
    r = np.array(rcxq, dtype=np.complex128, copy=True)
    if abs(smear) > 1e-15:                              # :174-193: rcxq(:, :, 1:) . gfmat^T
        r[:, :, 1:] = np.einsum('abk,jk->abj', r[:, :, 1:], gaussian_filter(frhis, smear))
    for iw in range(1, nwhis + 1):
        k = iw + nwhis
        wfac = np.exp(-(C[k] / ecut) ** 2) if ecut < 1e9 else 1.0
        r[:, :, iw] *= -wfac / (R[k] - L[k])
    imatt, rmatt = transform_matrices(frhis, freq_i, freq_r)
    zxqi = np.einsum('abk,jk->abj', r[:, :, 1:], imatt)
    if freq_r is None:
        return zxqi, None
    nw = len(freq_r) - 1
    zxq = 1j * r[:, :, :nw + 1] + np.einsum('abk,tk->abt', r[:, :, 1:], rmatt)
    return zxqi, zxq
