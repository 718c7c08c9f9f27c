"""Tetrahedron histogram weights of chi0 (test infrastructure): a plain
restatement of the Rath-Freeman microcell integral the reference uses,
SRC/subroutines/tetwt5.f90 (lindtet6 :514-600, inttetra6 :601-672,
inttetrac6 :673-713, intttvc6 :714-787, midk3 :848-857, midk :913-919),
integtetn (m_tetrakbt.f90:441-466) and sortea (util.f90:574-594), with
tetrahedron_matrix_linear = F (its default, switch.f90:253-263), and the
per-corner accumulation of tetwt5x_dtet4 (:304-341, npm = 1, one micro
tetrahedron per tetrahedron, wtet = 1/4).

    wtthis(ihis) = int_{frhis(ihis)}^{frhis(ihis+1)} d omega int_tet d^3k
                   f(ea(k)) (1 - f(eb(k))) delta(omega + x(k)),  x = (ea - eb)/2
"""
import numpy as np


def sortea(ea):
    """Insertion sort of util.f90:574-594: the index order of ea, ascending."""
    n = len(ea)
    order = list(range(n))
    for ix in range(1, n):
        i = ix
        while i >= 1 and ea[order[i - 1]] > ea[order[i]]:
            order[i - 1], order[i] = order[i], order[i - 1]
            i -= 1
    return order


def integtetn(e, ee):
    """m_tetrakbt.f90:441-466: normalised cumulative integral of the cross
    section of a tetrahedron with corner values e (ascending) below ee."""
    e1, e2, e3, e4 = e[0] - 3e-8, e[1] - 2e-8, e[2] - 1e-8, e[3]
    v1, v2, v4 = ee - e1, ee - e2, ee - e4
    if ee < e1:
        return 0.0
    if ee < e2:
        return v1 ** 3 / ((e4 - e1) * (e3 - e1) * (e2 - e1))
    if ee < e3:
        a = v1 / ((e4 - e1) * (e3 - e1) * (e2 - e1)) ** (1.0 / 3.0)
        b = v2 / (-(e4 - e2) * (e3 - e2) * (e1 - e2)) ** (1.0 / 3.0)
        return (a - b) * (a * a + a * b + b * b)
    if ee < e4:
        return 1.0 - v4 ** 3 / ((e1 - e4) * (e2 - e4) * (e3 - e4))
    if ee == e4:
        return 1.0
    raise ValueError("integtetn: ee > e4")


def det33(a):
    return float(np.linalg.det(np.asarray(a, dtype=np.float64)))


def intttvc6(v, voltet, frhis, wt):
    """:714-787 with matrix_linear = F: add this tetrahedron's histogram of
    omega = -v into wt (nwhis,)."""
    order = sortea([-x for x in v])
    ww = [-v[i] for i in order]                     # ascending
    nwhis = len(frhis) - 1
    inihis = iedhis = None
    ix = 0
    for ihis in range(nwhis):
        if ix == 0 and ww[0] < frhis[ihis + 1]:
            inihis = ihis
            ix = 3
        if ix == 3 and ww[3] < frhis[ihis + 1]:
            iedhis = ihis
            break
    if inihis is None or iedhis is None:
        raise ValueError("intttvc6: excitation energies outside the histogram")
    norm = integtetn(ww, ww[3])
    pvn = voltet / norm
    intega = 0.0
    for ihis in range(inihis, iedhis + 1):
        integb = norm if frhis[ihis + 1] > ww[3] else integtetn(ww, frhis[ihis + 1])
        wt[ihis] += pvn * (integb - intega)
        intega = integb


def inttetrac6(kk, xx, itetx, frhis, wt):
    """:673-713: volume of the sub-tetrahedron itetx (0-based corners of the
    8-point sets kk, xx) and its histogram."""
    kin = [np.asarray(kk[i], dtype=np.float64) for i in itetx]
    am = np.stack([kin[i] - kin[3] for i in range(3)], axis=1)
    voltet = abs(det33(am) / 6.0)
    intttvc6([xx[i] for i in itetx], voltet, frhis, wt)


def _mid(kk, ee, xx, i, j, yy=None):
    r = ee[i] / (ee[i] - ee[j])
    k = kk[i] + r * (kk[j] - kk[i])
    x = xx[i] + r * (xx[j] - xx[i])
    y = None if yy is None else yy[i] + r * (yy[j] - yy[i])
    return k, x, y


def inttetra6(kk8, xx8, ebf8, itetx, frhis, wt):
    """:601-672: the part of a sub-tetrahedron where eb > ef (ebf > 0)."""
    kin = [np.asarray(kk8[i], dtype=np.float64) for i in itetx]
    xin = [xx8[i] for i in itetx]
    ein = [ebf8[i] for i in itetx]
    order = sortea(ein)                             # ascending: ee[3] largest
    kk = [kin[i] for i in order] + [None] * 4
    ee = [ein[i] for i in order]
    xx = [xin[i] for i in order] + [0.0] * 4

    def mid(i, j, slot):
        kk[4 + slot], xx[4 + slot], _ = _mid(kk, ee, xx, i, j)

    # corner numbers of the reference are 1-based: k(n) -> index n-1, K(n) -> index 3+n
    if 0.0 >= ee[3]:
        return
    if ee[3] > 0.0 >= ee[2]:                        # Fig 1
        mid(3, 1, 0); mid(3, 0, 1); mid(3, 2, 2)
        inttetrac6(kk, xx, (3, 4, 5, 6), frhis, wt)
    elif ee[2] > 0.0 >= ee[1]:                      # Fig 2
        mid(3, 1, 0); mid(3, 0, 1); mid(2, 0, 2); mid(2, 1, 3)
        inttetrac6(kk, xx, (3, 2, 4, 5), frhis, wt)
        inttetrac6(kk, xx, (2, 5, 6, 4), frhis, wt)
        inttetrac6(kk, xx, (2, 4, 6, 7), frhis, wt)
    elif ee[1] > 0.0 >= ee[0]:                      # Fig 3
        mid(0, 3, 0); mid(0, 1, 1); mid(0, 2, 2)
        inttetrac6(kk, xx, (2, 3, 6, 1), frhis, wt)
        inttetrac6(kk, xx, (3, 4, 5, 6), frhis, wt)
        inttetrac6(kk, xx, (3, 1, 5, 6), frhis, wt)
    else:                                           # Fig 4
        inttetrac6(kk, xx, (0, 1, 2, 3), frhis, wt)


def lindtet6(kvec, ea, eb, x, efa, efb, frhis):
    """:514-600: histogram weights (nwhis,) of one tetrahedron (corners kvec
    (4, 3), occupied energies ea, unoccupied eb, x = (ea - eb)/2)."""
    order = sortea(list(ea))[::-1]                  # descending: ee[3] smallest
    kk = [np.asarray(kvec[i], dtype=np.float64) for i in order] + [None] * 4
    ee = [ea[i] - efa for i in order]
    xx = [x[i] for i in order] + [0.0] * 4
    ebf = [eb[i] - efb for i in order] + [0.0] * 4
    wt = np.zeros(len(frhis) - 1)

    def mid(i, j, slot):
        kk[4 + slot], xx[4 + slot], ebf[4 + slot] = _mid(kk, ee, xx, i, j, ebf)

    if 0.0 <= ee[3]:
        return wt
    if ee[3] < 0.0 <= ee[2]:                        # Fig 1
        mid(3, 1, 0); mid(3, 0, 1); mid(3, 2, 2)
        inttetra6(kk, xx, ebf, (3, 4, 5, 6), frhis, wt)
    elif ee[2] < 0.0 <= ee[1]:                      # Fig 2
        mid(3, 1, 0); mid(3, 0, 1); mid(2, 0, 2); mid(2, 1, 3)
        inttetra6(kk, xx, ebf, (3, 2, 4, 5), frhis, wt)
        inttetra6(kk, xx, ebf, (2, 5, 6, 4), frhis, wt)
        inttetra6(kk, xx, ebf, (2, 4, 6, 7), frhis, wt)
    elif ee[1] < 0.0 <= ee[0]:                      # Fig 3
        mid(0, 3, 0); mid(0, 1, 1); mid(0, 2, 2)
        inttetra6(kk, xx, ebf, (2, 3, 6, 1), frhis, wt)
        inttetra6(kk, xx, ebf, (3, 4, 5, 6), frhis, wt)
        inttetra6(kk, xx, ebf, (3, 1, 5, 6), frhis, wt)
    else:                                           # Fig 4
        inttetra6(kk, xx, ebf, (0, 1, 2, 3), frhis, wt)
    return wt


def tetwt_hist(idtet, qbzw, ek, ekq, efermi, frhis, nocc, nunocc):
    """Per-k histogram weights of every (occupied ib < nocc at k, unoccupied
    jb < nunocc at k+q) pair, tetwt5x_dtet4 :304-341 with npm = 1 and a dense
    output w[k, ib, jb, ihis] += wtthis(ihis) * pi / (4 voltot) per corner.
    idtet (ntet, 4) corner indices into qbzw (nk, 3) and into the band tables
    ek, ekq (nk, nband), energies in Ry (x in Hartree as the reference)."""
    nk = ek.shape[0]
    nwhis = len(frhis) - 1
    vols = []
    for t in range(idtet.shape[0]):
        kv = qbzw[idtet[t]]
        vols.append(abs(det33(np.stack([kv[i] - kv[3] for i in range(3)], axis=1)) / 6.0))
    voltot = float(np.sum(vols))
    f = np.pi / (4.0 * voltot)
    w = np.zeros((nk, nocc, nunocc, nwhis))
    for t in range(idtet.shape[0]):
        kk = idtet[t]
        kv = qbzw[kk]
        for ib in range(nocc):
            for jb in range(nunocc):
                eocc = ek[kk, ib]
                eunocc = ekq[kk, jb]
                if not (eocc.min() <= efermi and eunocc.max() >= efermi):
                    continue
                if np.max(eunocc - eocc) < 0.0:
                    continue
                x = 0.5 * (eocc - eunocc)
                wt = lindtet6(kv, eocc, eunocc, x, efermi, efermi, frhis)
                for c in range(4):
                    w[kk[c], ib, jb] += wt * f
    return w, voltot


def chkdgn(ene, epsx=1e-4):
    """tetwt5.f90:868-912: groups of consecutive levels, a new group wherever
    |ene(i) - ene(i-1)| > epsx; returns (first, last) pairs, 0-based inclusive."""
    n = len(ene)
    if n < 1:
        return []
    groups, first = [], 0
    for i in range(1, n):
        if abs(ene[i] - ene[i - 1]) > epsx:
            groups.append((first, i - 1))
            first = i
    groups.append((first, n - 1))
    return groups


def symmetrize_degenerate(w, ek, ekq, epsx=1e-4):
    """tetwt5.f90:347-423, job 1, npm = 1, no core states, on the dense
    w[k, ib, jb, ihis] of tetwt_hist: for every k, every degenerate group of
    ek[k, :nocc] and every one of ekq[k, :nunocc], each (ib, jb) of the block
    gets the block's mean histogram, summed ib-major, jb-minor and divided by
    the block size as the reference does.  Returns a new array."""
    w = np.array(w, dtype=np.float64, copy=True)
    nk, nocc, nunocc, _ = w.shape
    for k in range(nk):
        for (i0, i1) in chkdgn(ek[k, :nocc], epsx):
            for (j0, j1) in chkdgn(ekq[k, :nunocc], epsx):
                cnt = (i1 - i0 + 1) * (j1 - j0 + 1)
                if cnt == 1:
                    continue
                acc = np.zeros(w.shape[3])
                for ib in range(i0, i1 + 1):
                    for jb in range(j0, j1 + 1):
                        acc = acc + w[k, ib, jb]
                acc = acc / cnt
                w[k, i0:i1 + 1, j0:j1 + 1] = acc
    return w
