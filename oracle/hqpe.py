"""QP energies and the Hermitian self-energy: restatement of
SRC/subroutines/main_hqpe.sc.f90:160-180.  Test infrastructure only."""
import numpy as np

HARTREE_EV = 27.211386245988   # conversion used for the eV columns (m_lgunit hartree)


def qp_energies(elda_ev, sex2, sexcore2, sec2, vxc_ev):
    """e_QP = e_LDA + SEx + SExcore + Re SEc - vxc in eV with Z = 1
    (main_hqpe.sc.f90:150-161).  sex2/sexcore2/sec2 are the ntq x ntq
    Hartree matrices; only their diagonals enter."""
    h = HARTREE_EV
    sex = np.real(np.diag(sex2)) * h
    sexc = np.real(np.diag(sexcore2)) * h
    rsec = np.real(np.diag(sec2)) * h
    return np.asarray(elda_ev) + sex + sexc + rsec - np.asarray(vxc_ev)


def hermitian_sigma(sex2, sexcore2, sec2, vxc_band_ry):
    """Sigma_ij = SEx + SExcore + (SEc + SEc^H)/2 - vxc/2 (Hartree; vxc given
    in Ry in the band basis, i.e. evec^H v_xc evec), main_hqpe.sc.f90:178-180."""
    return sex2 + sexcore2 + 0.5 * (sec2 + sec2.conj().T) - 0.5 * vxc_band_ry
