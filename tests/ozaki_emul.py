"""CPU emulation of the int8 Ozaki-scheme products of the library's SPLIT_I8
mode (test infrastructure).  It computes exactly what the tensor-core kernels
compute -- the same power-of-two scales, the same slices, the same kept slice
pairs, integer products summed exactly -- so the GPU results must match it to
FP64 rounding, independently of how close either is to the FP64 product.

Scheme: mu = 2^e >= max |x| over a row of A (a column of B), over both the real
and the imaginary parts; V = rint(x / mu 2^(6 + 7 (ns - 1))) is written in base
128 with digits in [-64, 64] (the top digit s_1 first); x ~ mu sum_i s_i 2^-(6 + 7 (i-1)).  The product keeps the slice pairs
(p, q) with p + q <= ns + 1 (1-based), each pair's integer product weighted
2^-(12 + 7 (p + q - 2)).
"""
import numpy as np


def pow2_at_least(m):
    """Elementwise smallest power of two >= m (1 where m is 0)."""
    m = np.asarray(m, np.float64)
    out = np.ones_like(m)
    nz = m > 0
    _, e = np.frexp(m[nz])
    out[nz] = np.ldexp(1.0, e)
    return out


def slices(x, mu, ns):
    """int64 slices of x / mu (mu broadcast against x), list of ns arrays, top first:
    V = rint(x / mu 2^(6 + 7 (ns - 1))) written in base 128 from the bottom, each digit
    sign(V) r with r = |V| mod 128 taken in [-63, 64], the top digit holding the rest."""
    v = np.rint(np.asarray(x, np.float64) / mu * 2.0 ** (6 + 7 * (ns - 1))).astype(np.int64)
    out = [None] * ns
    for i in range(ns - 1, 0, -1):
        r = np.abs(v) & 127
        r = np.where(r > 64, r - 128, r)
        d = np.where(v < 0, -r, r)
        out[i] = d
        v = (v - d) >> 7
    out[0] = v
    return out


def _level_weight(p, q):
    return np.ldexp(1.0, -(12 + 7 * (p + q)))            # p, q 0-based


def complex_product(a, b, ns, mu_rows=None, nu_cols=None):
    """Emulated C = a @ b for complex a (M, K), b (K, N): rows of a scaled per
    row, columns of b per column (scales computed here unless given)."""
    a = np.asarray(a); b = np.asarray(b)
    if mu_rows is None:
        mu_rows = pow2_at_least(np.maximum(np.abs(a.real), np.abs(a.imag)).max(axis=1))
    if nu_cols is None:
        nu_cols = pow2_at_least(np.maximum(np.abs(b.real), np.abs(b.imag)).max(axis=0))
    ar = slices(a.real, mu_rows[:, None], ns)
    ai = slices(a.imag, mu_rows[:, None], ns)
    br = slices(b.real, nu_cols[None, :], ns)
    bi = slices(b.imag, nu_cols[None, :], ns)
    re = np.zeros((a.shape[0], b.shape[1]))
    im = np.zeros((a.shape[0], b.shape[1]))
    for p in range(ns):
        for q in range(ns - p):
            f = _level_weight(p, q)
            # integer products: exact in float64 (|s| <= 64, K well below 2^40)
            re += f * ((ar[p].astype(np.float64) @ br[q].astype(np.float64))
                       - (ai[p].astype(np.float64) @ bi[q].astype(np.float64)))
            im += f * ((ai[p].astype(np.float64) @ br[q].astype(np.float64))
                       + (ar[p].astype(np.float64) @ bi[q].astype(np.float64)))
    return (re + 1j * im) * mu_rows[:, None] * nu_cols[None, :]


def chi0_dense(zcols, w, ns):
    """Emulated chi0(:, :, j) = sum_p w[j, p] conj(z_p) z_p^T of the SPLIT_I8
    path for weights of one sign per slot: y = sqrt(|w|) z, rows scaled by
    2^e >= sqrt(max |w_j|) max_p |z(m, p)| (max over Re and Im)."""
    z = np.asarray(zcols)
    zmax = np.maximum(np.abs(z.real), np.abs(z.imag)).max(axis=1)
    out = np.zeros((z.shape[0], z.shape[0], w.shape[0]), np.complex128, order='F')
    for j in range(w.shape[0]):
        wj = np.asarray(w[j])
        for sign in (-1.0, 1.0):
            f = np.sqrt(np.maximum(sign * wj, 0.0))
            if not np.any(f > 0):
                continue
            mu = pow2_at_least(np.sqrt(f.max() ** 2) * zmax)
            y = z * f[None, :]
            out[:, :, j] += sign * complex_product(np.conj(y), y.T, ns, mu_rows=mu, nu_cols=mu)
    return out


def correlation_block(zsec, zmel, ns1, ns2, ns2r, nwxi, nwx, ntqxx, wc_imag, wc_real, omega, ekc, nctot, ef,
                      esmr, wkkr, ua, x, wt, expa, freq_r, ns):
    """The oracle's correlation block (m_sxcf_gemm.f90:407-612) with every
    W^H z product of the imaginary axis and the poles replaced by the emulated
    int8 product (the weights multiply the product afterwards, per column, as
    the kernel applies them); the final contraction stays FP64."""
    from oracle import sxcf
    if ns1 > ns2:
        return zsec
    ngb = zmel.shape[0]
    niw = len(x)
    nm = ns2 - ns1 + 1
    zf = zmel.reshape(ngb, -1, order='F')
    wg = sxcf.wgtim(omega, ekc, nctot, ns1, ns2, ntqxx, esmr, wkkr, ua, x, wt, expa)
    cz = np.zeros(zf.shape, np.complex128)
    for iw in range(niw + 1):
        prod = complex_product(wc_imag[:, :, iw].conj().T, zf, ns)
        cz += prod * wg[iw].reshape(-1, order='F')[None, :]
    ent = sxcf.pole_table(omega, ekc, nctot, ns1, ns2r, ntqxx, ef, esmr, wkkr, freq_r)
    bins = {}
    for (it, itp, ixs, w3) in ent:
        for i in range(3):
            bins.setdefault(ixs - 1 + i, []).append(((it - ns1) + nm * (itp - 1), w3[i]))
    nw = wc_real.shape[2] - 1
    for iw in range(nw + 1):
        if iw < nwxi or iw > nwx or iw not in bins:
            continue
        wv = wc_real[:, :, iw]
        wc = (wv + wv.conj().T) * 0.5
        prod = complex_product(wc.conj().T, zf, ns)
        for (c, w) in bins[iw]:
            cz[:, c] += prod[:, c] * w
    k = ngb * nm
    zsec[:ntqxx, :ntqxx] += (cz.reshape(k, ntqxx, order='F').conj().T @ zmel.reshape(k, ntqxx, order='F'))
    for itp in range(ntqxx):
        im = zsec[itp, itp].imag
        zsec[itp, itp] = complex(zsec[itp, itp].real, min(im, 0.0))
    return zsec
