"""CPU emulation of the int8 Ozaki-scheme products of the library's SPLIT_I8
mode (test infrastructure).  It computes exactly what the tensor-core kernels
compute -- the same power-of-two scales, the same slices, the same kept slice
pairs, integer products summed exactly -- so the GPU results must match it to
FP64 rounding, independently of how close either is to the FP64 product.

Scheme: mu = 2^e >= max |x| over a row of A (a column of B), over both the real
and the imaginary parts (bits = 8: mu = that max itself); V = rint(x U / mu) is
written in ns digits of base
2^bits, the top digit s_1 first, x ~ (mu / U) sum_i s_i 2^(bits (ns - i)).  Two
digit sets:
* bits = 7 (chi0): U = 2^(6 + 7 (ns - 1)), digits in [-64, 64], symmetric, so
  negation commutes with the slicing (the chi0 kernel negates slices);
* bits = 8 (the Sigma_c kernel, also behind the zmel M -> E product):
  U = 127 256^(ns-1) - 128 (256^(ns-1) - 1) / 255, digits in [-128, 127] (every
  int8 value; U keeps the top digit in range), one bit more per slice; -x is
  sliced on its own where the kernel needs it.
The product keeps the slice pairs (p, q) with p + q <= ns + 1 (1-based), each
pair's integer product weighted 2^(bits (2 ns - p - q)) / U^2.
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


def max_scale(m):
    """The Sigma_c kernel's scale: the max itself (1 where it is 0 or not finite)."""
    m = np.asarray(m, np.float64)
    return np.where((m > 0) & np.isfinite(m), m, 1.0)


def unit(ns, bits=7):
    """U: x / mu in [-1, 1] times U is the integer V that the ns digits hold."""
    if bits == 7:
        return float(1 << (6 + 7 * (ns - 1)))
    b = 256 ** (ns - 1)
    return float(127 * b - 128 * ((b - 1) // 255))


def slices(x, mu, ns, bits=7):
    """int64 slices of x / mu (mu broadcast against x), list of ns arrays, top first.
    bits = 7: V = rint(x / mu 2^(6 + 7 (ns - 1))) written in base 128 from the bottom, each
    digit sign(V) r with r = |V| mod 128 taken in [-63, 64], the top digit holding the rest.
    bits = 8: V = rint(x (U / mu)) (one rounded multiply, as the kernel does it) written in
    base 256 from the bottom with digits in [-128, 127], the top digit holding the rest."""
    x = np.asarray(x, np.float64)
    out = [None] * ns
    if bits == 7:
        v = np.rint(x / mu * 2.0 ** (6 + 7 * (ns - 1))).astype(np.int64)
        for i in range(ns - 1, 0, -1):
            r = np.abs(v) & 127
            r = np.where(r > 64, r - 128, r)
            d = np.where(v < 0, -r, r)
            out[i] = d
            v = (v - d) >> 7
    else:
        v = np.rint(x * (unit(ns, 8) / mu)).astype(np.int64)
        for i in range(ns - 1, 0, -1):
            q = (v + 128) >> 8
            out[i] = v - (q << 8)
            v = q
    out[0] = v
    return out


def _level_weight(p, q, ns=None, bits=7):
    if bits == 7:
        return np.ldexp(1.0, -(12 + 7 * (p + q)))            # p, q 0-based
    return np.ldexp(1.0, 8 * (2 * (ns - 1) - p - q)) / unit(ns, 8) ** 2


def complex_product(a, b, ns, mu_rows=None, nu_cols=None, bits=7):
    """Emulated C = a @ b for complex a (M, K), b (K, N): rows of a scaled per
    row, columns of b per column (scales computed here unless given).  The real
    part pairs Re a with Re b and -Im a with Im b; with bits = 8 -Im a is sliced
    on its own (the Sigma_c kernel's A' rows [Re a, -Im a] and [Im a, Re a])."""
    a = np.asarray(a); b = np.asarray(b)
    scale = pow2_at_least if bits == 7 else max_scale
    if mu_rows is None:
        mu_rows = scale(np.maximum(np.abs(a.real), np.abs(a.imag)).max(axis=1))
    if nu_cols is None:
        nu_cols = scale(np.maximum(np.abs(b.real), np.abs(b.imag)).max(axis=0))
    ar = slices(a.real, mu_rows[:, None], ns, bits)
    ai = slices(a.imag, mu_rows[:, None], ns, bits)
    an = slices(-a.imag, mu_rows[:, None], ns, bits)       # = -ai when bits = 7
    br = slices(b.real, nu_cols[None, :], ns, bits)
    bi = slices(b.imag, nu_cols[None, :], ns, bits)
    re = np.zeros((a.shape[0], b.shape[1]))
    im = np.zeros((a.shape[0], b.shape[1]))
    for p in range(ns):
        for q in range(ns - p):
            f = _level_weight(p, q, ns, bits)
            # integer products: exact in float64 (|s| <= 128, K well below 2^30)
            re += f * ((ar[p].astype(np.float64) @ br[q].astype(np.float64))
                       + (an[p].astype(np.float64) @ bi[q].astype(np.float64)))
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
    int8 product in base-256 digits (the weights multiply the product
    afterwards, per column, as the kernel applies them); the final contraction
    stays FP64."""
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
        prod = complex_product(wc_imag[:, :, iw].conj().T, zf, ns, bits=8)
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
        prod = complex_product(wc.conj().T, zf, ns, bits=8)
        for (c, w) in bins[iw]:
            cz[:, c] += prod[:, c] * w
    k = ngb * nm
    zsec[:ntqxx, :ntqxx] += (cz.reshape(k, ntqxx, order='F').conj().T @ zmel.reshape(k, ntqxx, order='F'))
    for itp in range(ntqxx):
        im = zsec[itp, itp].imag
        zsec[itp, itp] = complex(zsec[itp, itp].real, min(im, 0.0))
    return zsec
