! ISO_C_BINDING interface to libqsgw_b200 (include/qsgw_b200.h) for ecalj's
! own drivers.  Selected in place of the m_blas / m_lapack aliases by a
! -D__B200 build; every function returns 0 or a negative qsgw_status.
module m_qsgw_b200
  use, intrinsic :: iso_c_binding
  implicit none
  integer(c_int), parameter :: QSGW_PREC_FP64 = 0, QSGW_PREC_SPLIT_F16 = 1, QSGW_PREC_SPLIT_I8 = 2
  type, bind(C) :: qsgw_sxcf_args
    integer(c_int) :: ngb, nblochpmx, ns1, ns2, ns2r, ntqxx, ntq, niw, nw, nwxi, nwx, nctot, nekc, keepwv
    real(c_double) :: ef, esmr, wkkr, ua
    type(c_ptr) :: omega, ekc, freqx, wwx, expa, freq_r
    type(c_ptr) :: zmel, wc_imag, wc_real, zsec
  end type
  type, bind(C) :: qsgw_zmel_atom
    type(c_ptr) :: ppb_d
    integer(c_int) :: nlnm, nc, nv, ias, ics, ims, mdim, ncore
    real(c_double) :: phase_re, phase_im
  end type
  type, bind(C) :: qsgw_zmel_ipw_args
    integer(c_int) :: ngc, ngp1, ngp2, ngcgp, nggg
    integer(c_int) :: ntp0, nm1, nm2, nm1v, nm2v
    integer(c_int) :: ldz, row0
    integer(c_int) :: nadd(3)
    type(c_ptr) :: ngvecpB1, ngvecpB2, ngveccR, nvgcgp2, nvggg, ggg, phase, geigq_d
    integer(c_int) :: ldgq
    type(c_ptr) :: dgeigqk_d
    integer(c_int) :: ldgk
    type(c_ptr) :: zmelt_d
  end type
  interface
    integer(c_int) function qsgw_init(device) bind(C, name='qsgw_init')
      import :: c_int
      integer(c_int), value :: device
    end function
    integer(c_int) function qsgw_finalize() bind(C, name='qsgw_finalize')
      import :: c_int
    end function
    integer(c_int) function qsgw_synchronize() bind(C, name='qsgw_synchronize')
      import :: c_int
    end function
    integer(c_int) function qsgw_set_precision(mode, nslices) bind(C, name='qsgw_set_precision')
      import :: c_int
      integer(c_int), value :: mode, nslices
    end function
    integer(c_int) function qsgw_set_accuracy(sigc_qp_tol_ha, chi0_rel_tol) bind(C, name='qsgw_set_accuracy')
      import :: c_int, c_double
      real(c_double), value :: sigc_qp_tol_ha, chi0_rel_tol
    end function
    integer(c_int) function qsgw_set_host_async(on) bind(C, name='qsgw_set_host_async')
      import :: c_int
      integer(c_int), value :: on
    end function
    integer(c_int) function qsgw_set_sigc_kernel(kind) bind(C, name='qsgw_set_sigc_kernel')
      import :: c_int
      integer(c_int), value :: kind
    end function
    integer(c_int) function qsgw_last_error(buf, len) bind(C, name='qsgw_last_error')
      import :: c_int, c_char
      character(kind=c_char) :: buf(*)
      integer(c_int), value :: len
    end function
    integer(c_int) function qsgw_zmm_d(a, b, c, m, n, k, opa, opb, alpha, beta, lda, ldb, ldc) &
         bind(C, name='qsgw_zmm_d')
      import :: c_int, c_double, c_ptr
      type(c_ptr), value :: a, b, c
      integer(c_int), value :: m, n, k, opa, opb, lda, ldb, ldc
      real(c_double), intent(in) :: alpha(2), beta(2)
    end function
    integer(c_int) function qsgw_zminv_hpd_batched_d(a, n, lda, nbatch) bind(C, name='qsgw_zminv_hpd_batched_d')
      import :: c_int, c_ptr
      type(c_ptr), value :: a
      integer(c_int), value :: n, lda, nbatch
    end function
    integer(c_int) function qsgw_x0gemm_d(rcxq, npr, ipr_col, npr_col, nwhis, npm, ns1, ns2, &
         zmel, nbb, nm1, nm2, nqtot, icounkmink, icounkmaxk, itc, itpc, jpmc, iwini, iwend, &
         icouini, whwc, ncount) bind(C, name='qsgw_x0gemm_d')
      import :: c_int, c_double, c_ptr
      type(c_ptr), value :: rcxq, zmel
      integer(c_int), value :: npr, ipr_col, npr_col, nwhis, npm, ns1, ns2, nbb, nm1, nm2, nqtot
      integer(c_int), value :: icounkmink, icounkmaxk, ncount
      integer(c_int), intent(in) :: itc(*), itpc(*), jpmc(*), iwini(*), iwend(*), icouini(*)
      real(c_double), intent(in) :: whwc(*)
    end function
    integer(c_int) function qsgw_chi0_lorentz_d(chi0, npr, niw, freq_i, nk, nocc, nun, eocc, eunocc, &
         zcols, ldz) bind(C, name='qsgw_chi0_lorentz_d')
      import :: c_int, c_double, c_ptr
      type(c_ptr), value :: chi0, zcols
      integer(c_int), value :: npr, niw, nk, ldz
      real(c_double), intent(in) :: freq_i(*), eocc(*), eunocc(*)
      integer(c_int), intent(in) :: nocc(*), nun(*)
    end function
    ! degenerate-band averaging of the dense tetrahedron weights (host arrays, in place)
    integer(c_int) function qsgw_tetwt_symmetrize(w, nk, nocc, nunocc, nwhis, ek, ekq, nband) &
         bind(C, name='qsgw_tetwt_symmetrize')
      import :: c_int, c_double
      real(c_double), intent(inout) :: w(*)
      integer(c_int), value :: nk, nocc, nunocc, nwhis, nband
      real(c_double), intent(in) :: ek(*), ekq(*)
    end function
    ! x0gemm pair/bin lists from dense tetrahedron weights (host arrays, no GPU needed)
    integer(c_int) function qsgw_x0_lists(w, nk, nocc, nunocc, nwhis, job, ncoun, ncount, itc, itpc, jpmc, &
         iwini, iwend, icouini, whwc, icounkmin, icounkmax) bind(C, name='qsgw_x0_lists')
      import :: c_int, c_double
      real(c_double), intent(in) :: w(*)
      integer(c_int), value :: nk, nocc, nunocc, nwhis, job
      integer(c_int), intent(inout) :: ncoun, ncount
      integer(c_int), intent(out) :: itc(*), itpc(*), jpmc(*), iwini(*), iwend(*), icouini(*)
      integer(c_int), intent(out) :: icounkmin(*), icounkmax(*)
      real(c_double), intent(out) :: whwc(*)
    end function
    ! Hilbert transform of the chi0 histogram (dpsion_init + dpsion_chiq, npm = 1)
    integer(c_int) function qsgw_dpsion_chiq_d(rcxq, npr, npr_col, nwhis, frhis, niw, freq_i, nw, freq_r, &
         ecut, smearx0, zxqi, zxq) bind(C, name='qsgw_dpsion_chiq_d')
      import :: c_int, c_double, c_ptr
      type(c_ptr), value :: rcxq, zxqi, zxq
      integer(c_int), value :: npr, npr_col, nwhis, niw, nw
      real(c_double), intent(in) :: frhis(*), freq_i(*), freq_r(*)
      real(c_double), value :: ecut, smearx0
    end function
    ! its transform matrix on the host (complex (nwhis+1) x (niw+nw+1); no GPU needed)
    integer(c_int) function qsgw_dpsion_matrix(nwhis, frhis, niw, freq_i, nw, freq_r, ecut, smearx0, b) &
         bind(C, name='qsgw_dpsion_matrix')
      import :: c_int, c_double, c_ptr
      integer(c_int), value :: nwhis, niw, nw
      real(c_double), intent(in) :: frhis(*), freq_i(*), freq_r(*)
      real(c_double), value :: ecut, smearx0
      type(c_ptr), value :: b
    end function
    ! the same with host chi0 and zcols (c_loc of the Fortran arrays)
    integer(c_int) function qsgw_chi0_lorentz(chi0, npr, niw, freq_i, nk, nocc, nun, eocc, eunocc, &
         zcols, ldz) bind(C, name='qsgw_chi0_lorentz')
      import :: c_int, c_double, c_ptr
      type(c_ptr), value :: chi0, zcols
      integer(c_int), value :: npr, niw, nk, ldz
      real(c_double), intent(in) :: freq_i(*), eocc(*), eunocc(*)
      integer(c_int), intent(in) :: nocc(*), nun(*)
    end function
    integer(c_int) function qsgw_wvi_llw_d(zxqi, ngb, niw, nspin, vcousq, m2e, is_x0_m_basis, &
         is_wc_m_basis, iq, zw, nblochpmx) bind(C, name='qsgw_wvi_llw_d')
      import :: c_int, c_double, c_ptr
      type(c_ptr), value :: zxqi, m2e, zw
      integer(c_int), value :: ngb, niw, nspin, is_x0_m_basis, is_wc_m_basis, iq, nblochpmx
      real(c_double), intent(in) :: vcousq(*)
    end function
    integer(c_int) function qsgw_sxcf_correlation_d(args) bind(C, name='qsgw_sxcf_correlation_d')
      import :: c_int, qsgw_sxcf_args
      type(qsgw_sxcf_args), intent(in) :: args
    end function
    ! the same with host arrays in args (zmel, wc_imag, wc_real, zsec): copies in and out
    integer(c_int) function qsgw_sxcf_correlation(args) bind(C, name='qsgw_sxcf_correlation')
      import :: c_int, qsgw_sxcf_args
      type(qsgw_sxcf_args), intent(in) :: args
    end function
    integer(c_int) function qsgw_wvr_llw_d(zxq, ngb, nw, nspin, vcousq, m2e, is_x0_m_basis, &
         is_wc_m_basis, iq, zw, nblochpmx) bind(C, name='qsgw_wvr_llw_d')
      import :: c_int, c_double, c_ptr
      type(c_ptr), value :: zxq, m2e, zw
      integer(c_int), value :: ngb, nw, nspin, is_x0_m_basis, is_wc_m_basis, iq, nblochpmx
      real(c_double), intent(in) :: vcousq(*)
    end function
    integer(c_int) function qsgw_zminv_batched_d(a, n, lda, nbatch) bind(C, name='qsgw_zminv_batched_d')
      import :: c_int, c_ptr
      type(c_ptr), value :: a
      integer(c_int), value :: n, lda, nbatch
    end function
    integer(c_int) function qsgw_sxcf_exchange_d(zsec, ntq, zmel, ngb, ns1, ns2, ntqxx, vcoud, ekc, nekc, &
         nctot, ef, esmr, wkkr) bind(C, name='qsgw_sxcf_exchange_d')
      import :: c_int, c_double, c_ptr
      type(c_ptr), value :: zsec, zmel
      integer(c_int), value :: ntq, ngb, ns1, ns2, ntqxx, nekc, nctot
      real(c_double), intent(in) :: vcoud(*), ekc(*)
      real(c_double), value :: ef, esmr, wkkr
    end function
    integer(c_int) function qsgw_zhegv_d(v, o, n, lda, vcoud) bind(C, name='qsgw_zhegv_d')
      import :: c_int, c_double, c_ptr
      type(c_ptr), value :: v, o
      integer(c_int), value :: n, lda
      real(c_double), intent(out) :: vcoud(*)
    end function
    integer(c_int) function qsgw_tetwt_hist_d(w, nk, nocc, nunocc, nwhis, idtet, ntet, qbzw, ek, ekq, &
         nband, efermi, frhis, voltot) bind(C, name='qsgw_tetwt_hist_d')
      import :: c_int, c_double, c_ptr
      type(c_ptr), value :: w
      integer(c_int), value :: nk, nocc, nunocc, nwhis, ntet, nband
      integer(c_int), intent(in) :: idtet(*)
      real(c_double), intent(in) :: qbzw(*), ek(*), ekq(*), frhis(*)
      real(c_double), value :: efermi
      real(c_double), intent(out) :: voltot
    end function
    integer(c_int) function qsgw_wv_write_d(path, zw, nblochpmx, rec0, nrec, kind4) bind(C, name='qsgw_wv_write_d')
      import :: c_int, c_char, c_ptr
      character(kind=c_char), intent(in) :: path(*)
      type(c_ptr), value :: zw
      integer(c_int), value :: nblochpmx, rec0, nrec, kind4
    end function
    integer(c_int) function qsgw_wv_read_d(path, out, nblochpmx, rec0, nrec, kind4, pack, ngb) &
         bind(C, name='qsgw_wv_read_d')
      import :: c_int, c_char, c_ptr
      character(kind=c_char), intent(in) :: path(*)
      type(c_ptr), value :: out
      integer(c_int), value :: nblochpmx, rec0, nrec, kind4, pack, ngb
    end function
    ! __Vcoud.<iq> and SEX2U / SEXcore2U / SEC2U: the same 4-byte-marker records
    ! the Fortran sequential unformatted writes of these files produce, so
    ! either side can write a file the other reads
    integer(c_int) function qsgw_vcoud_write(path, ngb, q, vcoud, zcousq) bind(C, name='qsgw_vcoud_write')
      import :: c_int, c_char, c_double, c_double_complex
      character(kind=c_char), intent(in) :: path(*)
      integer(c_int), value :: ngb
      real(c_double), intent(in) :: q(3), vcoud(*)
      complex(c_double_complex), intent(in) :: zcousq(*)
    end function
    integer(c_int) function qsgw_vcoud_read(path, ngb_cap, ngb, q, vcoud, vcousq, zcousq) &
         bind(C, name='qsgw_vcoud_read')
      import :: c_int, c_char, c_double, c_ptr
      character(kind=c_char), intent(in) :: path(*)
      integer(c_int), value :: ngb_cap
      integer(c_int), intent(out) :: ngb
      real(c_double), intent(out) :: q(3)
      type(c_ptr), value :: vcoud, vcousq, zcousq
    end function
    integer(c_int) function qsgw_sigma_write(path, head, is, qibz, zsec) bind(C, name='qsgw_sigma_write')
      import :: c_int, c_char, c_double, c_double_complex
      character(kind=c_char), intent(in) :: path(*)
      integer(c_int), intent(in) :: head(8)
      integer(c_int), value :: is
      real(c_double), intent(in) :: qibz(3, *)
      complex(c_double_complex), intent(in) :: zsec(*)
    end function
    integer(c_int) function qsgw_sigma_read(path, head, nq_cap, ntq_cap, isx, qibz, zsec) &
         bind(C, name='qsgw_sigma_read')
      import :: c_int, c_char, c_ptr
      character(kind=c_char), intent(in) :: path(*)
      integer(c_int), intent(out) :: head(8)
      integer(c_int), value :: nq_cap, ntq_cap
      type(c_ptr), value :: isx, qibz, zsec
    end function
    integer(c_int) function qsgw_graph_begin() bind(C, name='qsgw_graph_begin')
      import :: c_int
    end function
    integer(c_int) function qsgw_graph_end() bind(C, name='qsgw_graph_end')
      import :: c_int
    end function
    integer(c_int) function qsgw_graph_launch() bind(C, name='qsgw_graph_launch')
      import :: c_int
    end function
    integer(c_int) function qsgw_set_autotune(mode, cache_path) bind(C, name='qsgw_set_autotune')
      import :: c_int, c_char
      integer(c_int), value :: mode
      character(kind=c_char), intent(in) :: cache_path(*)
    end function
    ! ---- the remaining entry points (the W_c interpolator's qsgw_wsurr_* have no
    ! counterpart in ecalj's drivers and are not bound here)
    integer(c_int) function qsgw_set_stream(stream) bind(C, name='qsgw_set_stream')
      import :: c_int, c_ptr
      type(c_ptr), value :: stream
    end function
    integer(c_int) function qsgw_get_precision(mode, nslices) bind(C, name='qsgw_get_precision')
      import :: c_int
      integer(c_int), intent(out) :: mode, nslices
    end function
    integer(c_long_long) function qsgw_launch_count() bind(C, name='qsgw_launch_count')
      import :: c_long_long
    end function
    integer(c_int) function qsgw_profile(enable) bind(C, name='qsgw_profile')
      import :: c_int
      integer(c_int), value :: enable
    end function
    integer(c_int) function qsgw_profile_get(tag, ms, launches) bind(C, name='qsgw_profile_get')
      import :: c_int, c_char, c_double, c_long_long
      character(kind=c_char), intent(in) :: tag(*)
      real(c_double), intent(out) :: ms
      integer(c_long_long), intent(out) :: launches
    end function
    integer(c_int) function qsgw_autotune_report(buf, len) bind(C, name='qsgw_autotune_report')
      import :: c_int, c_char
      character(kind=c_char), intent(out) :: buf(*)
      integer(c_int), value :: len
    end function
    integer(c_int) function qsgw_graph_destroy() bind(C, name='qsgw_graph_destroy')
      import :: c_int
    end function
    ! zmm_h (m_blas.f90:198) with host arrays
    integer(c_int) function qsgw_zmm(a, b, c, m, n, k, opa, opb, alpha, beta, lda, ldb, ldc) &
         bind(C, name='qsgw_zmm')
      import :: c_int, c_double, c_double_complex
      complex(c_double_complex), intent(in) :: a(*), b(*)
      complex(c_double_complex), intent(inout) :: c(*)
      integer(c_int), value :: m, n, k, opa, opb, lda, ldb, ldc
      real(c_double), intent(in) :: alpha(2), beta(2)
    end function
    integer(c_int) function qsgw_zminv_hpd_batched_noalloc_d(a, n, lda, nbatch, stream) &
         bind(C, name='qsgw_zminv_hpd_batched_noalloc_d')
      import :: c_int, c_ptr
      type(c_ptr), value :: a, stream
      integer(c_int), value :: n, lda, nbatch
    end function
    ! x0gemm (x0gemm.f90:2-97) with host arrays
    integer(c_int) function qsgw_x0gemm(rcxq, npr, ipr_col, npr_col, nwhis, npm, ns1, ns2, &
         zmel, nbb, nm1, nm2, nqtot, icounkmink, icounkmaxk, itc, itpc, jpmc, iwini, iwend, &
         icouini, whwc, ncount) bind(C, name='qsgw_x0gemm')
      import :: c_int, c_double, c_double_complex
      complex(c_double_complex), intent(inout) :: rcxq(*)
      complex(c_double_complex), intent(in) :: zmel(*)
      integer(c_int), value :: npr, ipr_col, npr_col, nwhis, npm, ns1, ns2, nbb, nm1, nm2, nqtot
      integer(c_int), value :: icounkmink, icounkmaxk, ncount
      integer(c_int), intent(in) :: itc(*), itpc(*), jpmc(*), iwini(*), iwend(*), icouini(*)
      real(c_double), intent(in) :: whwc(*)
    end function
    ! chi0 of one batch of k added into chi0 (zmel streamed k by k)
    integer(c_int) function qsgw_chi0_lorentz_acc_d(chi0, npr, niw, freq_i, nk_total, nkb, nocc, nun, &
         eocc, eunocc, zcols, ldz) bind(C, name='qsgw_chi0_lorentz_acc_d')
      import :: c_int, c_double, c_ptr
      type(c_ptr), value :: chi0, zcols
      integer(c_int), value :: npr, niw, nk_total, nkb, ldz
      real(c_double), intent(in) :: freq_i(*), eocc(*), eunocc(*)
      integer(c_int), intent(in) :: nocc(*), nun(*)
    end function
    ! real-axis chi0 of the Lorentzian model (broadening eta)
    integer(c_int) function qsgw_chi0_lorentz_real_d(chi0, npr, nw, freq_r, eta, nk, nocc, nun, &
         eocc, eunocc, zcols, ldz) bind(C, name='qsgw_chi0_lorentz_real_d')
      import :: c_int, c_double, c_ptr
      type(c_ptr), value :: chi0, zcols
      integer(c_int), value :: npr, nw, nk, ldz
      real(c_double), value :: eta
      real(c_double), intent(in) :: freq_r(*), eocc(*), eunocc(*)
      integer(c_int), intent(in) :: nocc(*), nun(*)
    end function
    ! WVIllwI per-iw block (m_llw.f90:318-373) with host arrays
    integer(c_int) function qsgw_wvi_llw(zxqi, ngb, niw, nspin, vcousq, m2e, is_x0_m_basis, &
         is_wc_m_basis, iq, zw, nblochpmx) bind(C, name='qsgw_wvi_llw')
      import :: c_int, c_double, c_double_complex
      complex(c_double_complex), intent(inout) :: zxqi(*)
      complex(c_double_complex), intent(in) :: m2e(*)
      complex(c_double_complex), intent(inout) :: zw(*)
      integer(c_int), value :: ngb, niw, nspin, is_x0_m_basis, is_wc_m_basis, iq, nblochpmx
      real(c_double), intent(in) :: vcousq(*)
    end function
    ! imaginary-axis weights of Sigma_c (m_sxcf_gemm.f90:423-458) on the device
    integer(c_int) function qsgw_sxcf_wgtim_d(wgtim, niw, ns1, ns2, ntqxx, nctot, omega, ekc, nekc, &
         esmr, wkkr, ua, freqx, wwx, expa) bind(C, name='qsgw_sxcf_wgtim_d')
      import :: c_int, c_double, c_ptr
      type(c_ptr), value :: wgtim
      integer(c_int), value :: niw, ns1, ns2, ntqxx, nctot, nekc
      real(c_double), value :: esmr, wkkr, ua
      real(c_double), intent(in) :: omega(*), ekc(*), freqx(*), wwx(*), expa(*)
    end function
    ! QP energies and Hermitian Sigma (main_hqpe.sc.f90:150-161, 178-180), device arrays
    integer(c_int) function qsgw_hqpe_d(sex2, sexcore2, sec2, vxc_band, elda, vxc, ntq, ld, nq, &
         eqp, sigma_herm) bind(C, name='qsgw_hqpe_d')
      import :: c_int, c_ptr
      type(c_ptr), value :: sex2, sexcore2, sec2, vxc_band, elda, vxc, eqp, sigma_herm
      integer(c_int), value :: ntq, ld, nq
    end function
    ! get_zmel_init_gemm: muffin-tin part (m_zmel.f90:323-415)
    integer(c_int) function qsgw_zmel_mt_d(zmelt, nbloch, nm1, nm2, nctot, ntp0, cphim, ldm, cphiq, &
         ldq, natom, atoms) bind(C, name='qsgw_zmel_mt_d')
      import :: c_int, c_ptr, qsgw_zmel_atom
      type(c_ptr), value :: zmelt, cphim, cphiq
      integer(c_int), value :: nbloch, nm1, nm2, nctot, ntp0, ldm, ldq, natom
      type(qsgw_zmel_atom), intent(in) :: atoms(*)
    end function
    ! interstitial plane-wave part (m_zmel.f90:418-535)
    integer(c_int) function qsgw_zmel_ipw_d(args) bind(C, name='qsgw_zmel_ipw_d')
      import :: c_int, qsgw_zmel_ipw_args
      type(qsgw_zmel_ipw_args), intent(in) :: args
    end function
    ! M -> E and conjugation (m_zmel.f90:546-563, 590-594)
    integer(c_int) function qsgw_zmel_m2e_d(zmel, zmelt, ngb, nbb, nmtot, nqtot, m2e, is_m_basis, &
         zmelconjg) bind(C, name='qsgw_zmel_m2e_d')
      import :: c_int, c_ptr
      type(c_ptr), value :: zmel, zmelt, m2e
      integer(c_int), value :: ngb, nbb, nmtot, nqtot, is_m_basis, zmelconjg
    end function
  end interface
end module m_qsgw_b200
