"""W on the imaginary axis: restatement of ``WVIllwI`` (q /= 0 branch) and of
``zminv_h``.  Test infrastructure only (see package doc)."""
import numpy as np
from scipy.linalg import lapack


def zminv_h(a):
    """SRC/subroutines/m_lapack.f90:21-47: in-place inverse by zgetrf+zgetri.
    Returns (inverse, info)."""
    lu, piv, info = lapack.zgetrf(a)
    if info != 0:
        return a, info
    inv, info = lapack.zgetri(lu, piv)
    return inv, info


def wvi_llw(zxqi, nspin, vcousq, m2e, is_x0_m_basis, is_wc_m_basis, iq,
            nblochpmx=None):
    """SRC/subroutines/m_llw.f90:265-376 (iq <= nqibz branch).

    zxqi   complex128 (ngb, ngb, niw); doubled in place when nspin == 1 (:299-303)
    vcousq float64 (ngb,) = sqrt(vcoud) (m_readVcoud.f90:42)
    m2e    complex128 (ngb, ngb) product-basis M->E matrix (m_zmel.f90:46-68)
    iq     1-based q index; iq == 1 skips the head row/column (ix = 1, :309)
    Returns zw complex128 (nblochpmx, nblochpmx, niw) = W - v per iw (:315-373).
    """
    ngb, _, niw = zxqi.shape
    if nblochpmx is None:
        nblochpmx = ngb
    if nspin == 1:
        zxqi *= 2.0                                          # :301
    ix = 1 if iq == 1 else 0                                 # :309
    out = np.zeros((nblochpmx, nblochpmx, niw), np.complex128, order='F')
    v = np.asarray(vcousq, dtype=np.float64)
    for iw in range(niw):
        zxqw = zxqi[:, :, iw].copy()                         # :320
        if is_x0_m_basis:                                    # :333-340
            x_m2e = zxqw @ m2e
            zxqw = m2e.conj().T @ x_m2e
        s = slice(ix, ngb)
        eps = -v[s, None] * zxqw[s, s] * v[None, s]          # :344
        eps[np.diag_indices_from(eps)] += 1.0                # :345
        einv, info = zminv_h(eps)                            # :350
        if info != 0:
            raise np.linalg.LinAlgError(f"zgetrf/zgetri info={info}")
        zw = np.zeros((nblochpmx, nblochpmx), np.complex128)
        blk = v[s, None] * einv * v[None, s]                 # :356
        blk[np.diag_indices_from(blk)] -= v[s] * v[s]        # :357
        zw[s, s] = blk
        if is_wc_m_basis and iq != 1:                        # :363-370
            x_m2e = zw[:ngb, :ngb] @ m2e.conj().T
            zw[:ngb, :ngb] = m2e @ x_m2e
        out[:, :, iw] = zw
    return out


def coulomb_eig(vmat, omat=None):
    """SRC/subroutines/main_hvccfp0.f90:322-367 with zhgv_h (m_lapack.f90:64-104):
    generalized Hermitian eigenproblem (-v) z = lambda O z, vcoud = -lambda,
    i.e. eigenvalues of v in descending order with O-orthonormal vectors.
    Returns (vcoud, zcousq)."""
    from scipy.linalg import eigh
    n = vmat.shape[0]
    b = np.eye(n, dtype=np.complex128) if omat is None else omat
    lam, z = eigh(-vmat, b, lower=False, driver='gvx')
    return -lam, z


def wvr_llw(zxq, nspin, vcousq, m2e, is_x0_m_basis, is_wc_m_basis, iq, nblochpmx=None):
    """SRC/subroutines/m_llw.f90:49-264 (WVRllwR): the per-frequency block
    :125-170 is the one of WVIllwI with eps~ general; zminv_h is LAPACK's
    pivoted zgetrf + zgetri, so the same restatement applies."""
    return wvi_llw(zxq, nspin, vcousq, m2e, is_x0_m_basis, is_wc_m_basis, iq, nblochpmx)
