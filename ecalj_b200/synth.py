"""Seeded synthetic inputs with the shapes and value distributions of the
benchmark configurations (the reference publishes no datasets for this path).

Energies are generated in Ry as the configurations state them and handed to
the kernels in the unit the reference uses there: Hartree for the chi0
weights and the imaginary-axis mesh (x0kf / m_freq work in a.u.), Ry for the
Sigma_c energies (omega, ekc, ef, esmr), with we = (omega - e)/2 in Hartree
inside the weights (m_sxcf_gemm.f90:436).
"""
import math

import numpy as np

CONFIGS = {
    # plain FP64 chi0 + W, Si-diamond-like size
    "chi0_w_n260": dict(N=260, nk=64, nocc=4, nun=(40, 60), niw=12, seed=20260),
    # split chi0, GaAs-like shape
    "chi0_n600": dict(N=600, nk=216, nocc=9, nun=(100, 300), niw=24, seed=20261),
    # Sigma_c band sum
    "sigc_n600": dict(N=600, nq=64, niw=24, ntq=40, nm=400, nreal=50, seed=20262,
               chi_nk=64, chi_nocc=4, chi_nun=(40, 60)),
    # all-in: zmel of all k is 369 GB, so it is streamed through the GPU k by k
    "chi0_n1500_streamed": dict(N=1500, nk=512, nocc=40, nun=(300, 1200), niw=32, seed=20264),
}


def gauss_legendre01(n):
    """Gauss-Legendre nodes/weights on (0,1), ascending (the nodes the
    reference's tabulated ``gauss`` returns, mate.f90:1-206)."""
    t, w = np.polynomial.legendre.leggauss(n)
    return (t + 1.0) * 0.5, w * 0.5


def imag_mesh(niw, ua=1.0):
    """freq01 (m_freq.f90:164-186): x, wx, freq_i = (1-x)/x (Hartree), expa."""
    x, wx = gauss_legendre01(niw)
    fi = (1.0 - x) / x
    return dict(x=x, wx=wx, freq_i=fi, expa=np.exp(-ua * ua * fi * fi), ua=ua)


def chi0_spectrum(rng, nk, nocc, nun_range):
    """Band counts and energies (Ry) per k: occupied U[-0.9, 0], unoccupied U[0.05, 4]."""
    nun = rng.integers(nun_range[0], nun_range[1] + 1, size=nk)
    nocc_a = np.full(nk, nocc, dtype=np.int64)
    eocc = [rng.uniform(-0.9, 0.0, nocc) for _ in range(nk)]
    eun = [rng.uniform(0.05, 4.0, int(n)) for n in nun]
    return nocc_a, nun, eocc, eun


def zmel_columns(rng, N, ncol):
    """complex128 (N, ncol), re and im ~ N(0,1)/sqrt(N), Fortran order."""
    s = 1.0 / math.sqrt(N)
    z = np.empty((N, ncol), np.complex128, order='F')
    z.real = rng.standard_normal((N, ncol)) * s
    z.imag = rng.standard_normal((N, ncol)) * s
    return z


def chi0_problem(N, nk, nocc, nun, niw, seed):
    """All inputs of one chi0(q, iw) evaluation (numpy, host)."""
    rng = np.random.default_rng(seed)
    nocc_a, nun_a, eocc, eun = chi0_spectrum(rng, nk, nocc, nun)
    npair = int(np.sum(nocc_a * nun_a))
    z = zmel_columns(rng, N, npair)
    mesh = imag_mesh(niw)
    return dict(N=N, nk=nk, niw=niw, nocc=nocc_a, nun=nun_a,
                eocc_ry=eocc, eun_ry=eun,
                eocc_h=np.concatenate(eocc) * 0.5, eun_h=np.concatenate(eun) * 0.5,
                zcols=z, npair=npair, **mesh)


def coulomb(N, seed):
    """v = Q diag(lam) Q^H, Q Haar unitary, lam log-uniform in [1e-2, 1e3].
    Returns vcousq = sqrt(lam) and the M->E matrix Q (= zcousq)."""
    rng = np.random.default_rng(seed)
    g = rng.standard_normal((N, N)) + 1j * rng.standard_normal((N, N))
    q, r = np.linalg.qr(g)
    q = q * (np.diag(r) / np.abs(np.diag(r)))[None, :]
    lam = 10.0 ** rng.uniform(-2.0, 3.0, N)
    return np.sqrt(lam), np.asfortranarray(q.astype(np.complex128))


def freq_r_mesh(nreal, wmax=2.0):
    """Real-axis mesh of the reference's form (m_freq.f90:95-134):
    frhis(i) = bb (exp(aa (i-1)) - 1), freq_r(0) = 0,
    freq_r(i) = (frhis(i) + frhis(i+1))/2, with aa, bb chosen so that nreal
    points reach wmax (Hartree)."""
    nw = nreal - 1
    aa = 0.08
    bb = wmax / (math.exp(aa * nw) - 1.0)
    frhis = bb * (np.exp(aa * np.arange(nw + 1)) - 1.0)
    fr = np.zeros(nw + 1)
    fr[1:] = 0.5 * (frhis[:nw] + frhis[1:nw + 1])
    return fr


def getfreq(omg2max, wemax, oratio=1.03, dw=1e-5, epsmode=False):
    """The histogram bins and the real-axis mesh of Getfreq (m_freq.f90:94-133),
    Hartree: aa = HistBin_ratio - 1, bb = HistBin_dw / aa; nwhis = (the first
    iw with bb (exp(aa (iw-1)) - 1) > omg2max + 1e-6) + 2; frhis(iw) =
    bb (exp(aa (iw-1)) - 1), iw = 1..nwhis+1; nw = the first iw >= 3 with
    (frhis(iw-2) + frhis(iw-1))/2 > wemax/2, at most nwhis - 1 (nwhis - 1
    in epsmode); freq_r(0) = 0, freq_r(i) = (frhis(i) + frhis(i+1))/2.
    Returns dict(frhis (nwhis+1), freq_r (nw+1), nwhis, nw)."""
    aa = oratio - 1.0
    bb = dw / aa
    iw = 0
    while True:
        iw += 1
        if bb * (math.exp(aa * (iw - 1)) - 1.0) > omg2max + 1e-6:
            break
    nwhis = iw + 2
    frhis = bb * (np.exp(aa * np.arange(nwhis + 1)) - 1.0)        # frhis(1..nwhis+1), 0-based here
    nw = None
    for iw in range(3, nwhis + 1):
        if 0.5 * (frhis[iw - 3] + frhis[iw - 2]) > wemax / 2.0:
            nw = iw
            break
    if epsmode:
        nw = nwhis - 1
    elif nw is None:
        raise ValueError("getfreq: wemax/2 beyond the histogram (the reference leaves nw unset)")
    else:
        nw = min(nw, nwhis - 1)
    freq_r = np.zeros(nw + 1)
    freq_r[1:] = 0.5 * (frhis[:nw] + frhis[1:nw + 1])
    return dict(frhis=frhis, freq_r=freq_r, nwhis=nwhis, nw=nw)


def sigc_task(N, ntq, nm, niw, nreal, seed, nctot=0, esmr=0.01, ef=0.0):
    """Energies and zmel of one Sigma_c task (Ry).  Target energies
    omega = eq(1:ntq) in [-1, 1] Ry; intermediate energies U[-1, 4] Ry."""
    rng = np.random.default_rng(seed)
    omega = np.sort(rng.uniform(-1.0, 1.0, ntq))
    ekc = np.sort(rng.uniform(-1.0, 4.0, nctot + nm))
    z = zmel_columns(rng, N, nm * ntq).reshape(N, nm, ntq, order='F')
    mesh = imag_mesh(niw)
    fr = freq_r_mesh(nreal)
    return dict(omega=omega, ekc=ekc, zmel=np.asfortranarray(z), ef=ef, esmr=esmr,
                nctot=nctot, freq_r=fr, **mesh)


def real_axis_model(wc0, freq_r, wp=0.5):
    """Synthetic Hermitian W_c on the real mesh (the configurations give W
    only on the imaginary axis): W_c(w) = W_c(0) / (1 + (w/wp)^2)."""
    g = 1.0 / (1.0 + (np.asarray(freq_r) / wp) ** 2)
    return np.asfortranarray(wc0[:, :, None] * g[None, None, :])


def ipw_tables(seed, ngc=37, ngp1=29, ngp2=31, ntp0=5, nmv=7, span=2, gbox=6, fill=0.8):
    """G-vector tables of the interstitial plane-wave part of zmel with the
    structure getppx2 reads (rppovl.f90:40-66): plane waves at q (ngvecpB1)
    and q-k (ngvecpB2), product-basis G (ngveccR), composite vectors nvgcgp2
    holding every Gc+G2 and Gc-G1, and a ggg table on a box with a fraction
    `fill` of its vectors present (the rest read as zero)."""
    rng = np.random.default_rng(seed)
    pts = np.array(np.meshgrid(*[np.arange(-span, span + 1)] * 3, indexing="ij")).reshape(3, -1)

    def pick(n):
        return pts[:, rng.choice(pts.shape[1], n, replace=False)].astype(np.int32)

    b1, b2, gc = pick(ngp1), pick(ngp2), pick(ngc)
    comp = {tuple(gc[:, c] + b2[:, g]) for c in range(ngc) for g in range(ngp2)}
    comp |= {tuple(gc[:, c] - b1[:, g]) for c in range(ngc) for g in range(ngp1)}
    comp = np.array(sorted(comp), np.int32).T
    comp = comp[:, rng.permutation(comp.shape[1])]
    box = np.array(np.meshgrid(*[np.arange(-gbox, gbox + 1)] * 3, indexing="ij")).reshape(3, -1)
    keep = rng.random(box.shape[1]) < fill
    nvggg = box[:, keep][:, rng.permutation(int(keep.sum()))].astype(np.int32)
    ggg = rng.standard_normal(nvggg.shape[1]) + 1j * rng.standard_normal(nvggg.shape[1])
    geigq = rng.standard_normal((ngp1, ntp0)) + 1j * rng.standard_normal((ngp1, ntp0))
    dgeigqk = rng.standard_normal((ngp2, nmv)) + 1j * rng.standard_normal((ngp2, nmv))
    phase = np.exp(-2j * np.pi * rng.random(ngc))
    return dict(ngvecpB1=b1, ngvecpB2=b2, ngveccR=gc, nvgcgp2=comp, nvggg=nvggg, ggg=ggg, geigq=geigq,
                dgeigqk=dgeigqk, phase=phase, nadd=np.array([1, 0, -1], np.int32))


def tetra_mesh(n, nband=6, q=(0.13, 0.05, -0.08), seed=0):
    """A k mesh of the unit cube (n^3 cells, (n+1)^3 corner points) cut into
    6 tetrahedra per cell, and smooth bands e_b(k) (Ry) crossing e = 0 at k
    and at k+q: idtet (6 n^3, 4), qbzw ((n+1)^3, 3), ek, ekq ((n+1)^3, nband)."""
    rng = np.random.default_rng(seed)
    g = np.arange(n + 1) / n
    kx, ky, kz = np.meshgrid(g, g, g, indexing="ij")
    qbzw = np.stack([kx.ravel(), ky.ravel(), kz.ravel()], axis=1)
    idx = lambda i, j, k: (i * (n + 1) + j) * (n + 1) + k
    # Freudenthal split of a cube along its main diagonal: 6 tetrahedra
    paths = [(0, 1, 2), (0, 2, 1), (1, 0, 2), (1, 2, 0), (2, 0, 1), (2, 1, 0)]
    tets = []
    for i in range(n):
        for j in range(n):
            for k in range(n):
                for p in paths:
                    c = [i, j, k]
                    corners = [idx(*c)]
                    for d in p:
                        c = list(c)
                        c[d] += 1
                        corners.append(idx(*c))
                    tets.append(corners)
    phase = rng.uniform(0, 2 * np.pi, (nband, 3))
    amp = rng.uniform(0.15, 0.3, nband)
    base = np.linspace(-0.7, 0.8, nband)

    def bands(kp):
        return base[None, :] + amp[None, :] * np.cos(2 * np.pi * kp[:, None, :] + phase[None, :, :]).sum(-1)

    return np.array(tets, np.int32), qbzw, bands(qbzw), bands(qbzw + np.asarray(q)[None, :])
