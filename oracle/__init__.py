"""CPU oracle for the QSGW inner loops (chi0 -> W -> Sigma_c).

TEST INFRASTRUCTURE ONLY.  Nothing in the product (the ``ecalj_b200``
package and ``libqsgw_b200.so``) imports, links or calls this package.  Only
``tests/``, ``__graft_entry__.smoke()`` and the ``cpu_baseline`` /
``--impl reference`` legs of ``bench.py`` use it, always as the checker or as
the timed CPU stand-in for the reference, never as the thing that is measured
on the GPU.

Every function is a float64 numpy restatement of one routine of tkotani/ecalj
(Fortran 90) and cites the file:line it follows.  The reference cannot be
compiled here (no Fortran compiler, no MPI, no MKL) and its own test-suite
holds no kernel-level golden vectors (its only pins are end-to-end QPU tables
that need the whole DFT+GW pipeline).  Those tables do pin one step: each
QPU row prints the QP-energy inputs beside its results, and ``hqpe`` is
checked against 2663 such rows of the reference's TestInstall cases
(``tests/golden/qpu_rows.npz``, ``tests/test_qpu_golden_cpu.py``).  For every
other routine PARITY IS UNPINNED: the restatement is checked against analytic
known answers (``tests/test_oracle.py``) and the committed fixtures in
``tests/golden/golden.npz`` are generated from this restatement, not from the
reference binary.

Linear algebra goes through numpy/scipy (OpenBLAS zgemm, LAPACK zgetrf/zgetri,
zhegvx), the same LAPACK routines the reference's CPU path calls
(SRC/subroutines/m_lapack.f90:21-47, 64-104; m_blas.f90 zmm_h).
"""
