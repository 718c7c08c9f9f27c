/*
 * libqsgw_b200 -- C ABI of the B200 implementation of ecalj's QSGW inner
 * loops (chi0 -> W -> Sigma_c).  Every entry point replaces one routine of
 * tkotani/ecalj (Fortran) at its call site and keeps that routine's argument
 * layout:
 *
 *   - complex(8) arrays are interleaved (re, im) doubles, column-major, with
 *     the Fortran leading dimensions passed explicitly;
 *   - Fortran lower bounds (ns1:ns2, (1-npm)*nwhis:nwhis, 0:niw ...) are
 *     passed explicitly and indices are 1-based where the reference's are;
 *   - accumulated outputs (rcxq, zsec) are read-modify-write, as the
 *     reference's beta = CONE GEMMs are.
 *
 * Functions without a suffix take HOST pointers and copy in and out.  The
 * "_d" variants take DEVICE pointers for the large arrays (the reference
 * passes those under `host_data use_device`); small tables stay on the host.
 * "_d" calls are ordered on the library stream (qsgw_set_stream) and return
 * before the GPU finishes; qsgw_synchronize() waits and reports any deferred
 * device-side status.
 *
 * Return value: 0 on success, a negative qsgw_status on failure; the
 * library never aborts.  qsgw_last_error() gives the message.  The library is
 * not re-entrant: one caller thread per process (one MPI rank per GPU in the
 * reference, m_gpu.f90:44).
 */
#ifndef QSGW_B200_H
#define QSGW_B200_H
#ifdef __cplusplus
extern "C" {
#endif

enum qsgw_status {
  QSGW_OK = 0,
  QSGW_ERR_ARG = -1,         /* bad shape / bound / pointer */
  QSGW_ERR_CUDA = -2,        /* CUDA runtime error */
  QSGW_ERR_OOM = -3,         /* device allocation failed */
  QSGW_ERR_NOTINIT = -4,     /* qsgw_init not called */
  QSGW_ERR_NUMERIC = -5,     /* non-finite value or non-positive pivot */
  QSGW_ERR_TIMEOUT = -6,     /* a bounded device wait ran out */
  QSGW_ERR_UNSUPPORTED = -7  /* mode not built for this shape */
};

enum qsgw_precision {
  QSGW_PREC_FP64 = 0,        /* complex FP64 on the FP64 tensor pipe (DMMA) */
  QSGW_PREC_SPLIT_F16 = 1,   /* split-FP16 slices on tcgen05, FP32 accumulate */
  QSGW_PREC_SPLIT_I8 = 2     /* Ozaki int8 slices on tcgen05, exact INT32 accumulate */
};

/* ---- context (replaces m_gpu.f90:14-68 gpu_init / cuBLAS+cuSOLVER handles,
 *      m_lapack.f90:230-255 cusolver_init/cusolver_finalize) ---------------- */
int qsgw_init(int device);
int qsgw_finalize(void);
/* Launch stream for every later call (a cudaStream_t; 0 = library stream). */
int qsgw_set_stream(void *stream);
int qsgw_synchronize(void);
/* Host-pointer calls (qsgw_chi0_lorentz, qsgw_sxcf_correlation) copy their
 * inputs on a copy stream into one of two device slots.  on = 0 (default):
 * each call returns with its outputs written, like the reference's Fortran
 * calls.  on = 1: each call returns once its copies and kernels are enqueued,
 * so the copy of one call overlaps the computation of the previous one; the
 * host outputs are valid, and the host inputs may be changed, only after
 * qsgw_synchronize().  zsec arrays accumulated by several calls are kept on
 * the device between synchronisations (one image per host array). */
int qsgw_set_host_async(int on);
/* Runtime precision switch; the reference's is the compile-time -D__MP
 * (m_kind.f90:3-11).  nslices: FP16 slices per operand for SPLIT_F16 (2);
 * int8 slices per operand for SPLIT_I8 (2, 3 or 4: about 14, 21 or 28 bits
 * relative to the largest element of a row / column, products accumulated
 * exactly).  Applies to the chi0 (qsgw_chi0_lorentz*, qsgw_x0gemm*), Sigma_c
 * (qsgw_sxcf_correlation*) and zmel M->E (qsgw_zmel_m2e_d) contractions. */
int qsgw_set_precision(int mode, int nslices);
/* Targets of the automatic slice count (SPLIT_I8 with nslices = 0): on the
 * first call of each problem shape the contraction runs at 4 slices and at 2
 * and 3, and keeps the smallest count whose change against 4 slices stays
 * within the target -- Sigma_c: largest |Re Sigma_c,nn| change of the call's
 * contribution in Hartree (default 1 meV = 3.675e-5 Ha, the QP-energy gate),
 * with a factor 4 of margin for the other calls of the shape; chi0: relative
 * Frobenius norm (default 2e-5) -- else 4.  Choices and estimates are listed by
 * qsgw_autotune_report.  Calls that accumulate into an output the caller
 * holds (qsgw_chi0_lorentz_acc_d, qsgw_x0gemm*) take the choice already made
 * for their shape, else 3 (chi0) / 4 (x0gemm) slices.  No counterpart in the
 * reference (its precision is fixed at compile time).                     */
int qsgw_set_accuracy(double sigc_qp_tol_ha, double chi0_rel_tol);
int qsgw_get_precision(int *mode, int *nslices);
/* Kernel of the split-precision Sigma_c contraction: 0 = one CTA per
 * 64 x 128 output tile, 1 = CTA pairs over 128-column tiles (tcgen05
 * cta_group::2, M = 256 over two SMs, each loading half of the B tile), 2 =
 * one CTA per 64 x 256 tile (N = 256 MMAs, FP64 sums in a global scratch
 * tile; the default, the fastest on B200).  All compute the same sums; the
 * environment variable QSGW_SIGC_KERNEL=<kind> sets it at load time. */
int qsgw_set_sigc_kernel(int kind);
/* Copies the last error message (NUL-terminated, truncated to len). */
int qsgw_last_error(char *buf, int len);
/* Number of kernels this library has launched since qsgw_init. */
long long qsgw_launch_count(void);
/* Per-kernel timing (replaces the reference's m_stopwatch laps,
 * m_stopwatch.f90:1-133): enable != 0 clears the record and starts putting
 * CUDA events around every hot kernel on the launch stream; qsgw_profile_get
 * waits for the stream and returns the summed milliseconds and the launch
 * count of one kernel tag ("chi0_dmma", "sigc_seg_dmma", "gemm_dmma",
 * "chi0_tc", "sigc_seg_tc").                                              */
int qsgw_profile(int enable);
int qsgw_profile_get(const char *tag, double *ms, long long *launches);

/* ---- BLAS shim: ZGEMM (m_blas.f90:198 zmm_h, :469 zmm_d) ----------------
 * C = alpha op(A) op(B) + beta C; op = 0 'N', 1 'T', 2 'C' (m_op_n/t/c).
 * alpha/beta are complex given as (re, im) pairs.  Always FP64.            */
int qsgw_zmm(const double *a, const double *b, double *c, int m, int n, int k,
             int opa, int opb, const double *alpha, const double *beta,
             int lda, int ldb, int ldc);
int qsgw_zmm_d(const double *a, const double *b, double *c, int m, int n,
               int k, int opa, int opb, const double *alpha,
               const double *beta, int lda, int ldb, int ldc);

/* ---- Inverse of a batch of Hermitian positive definite matrices in place
 * (replaces zminv_d, m_lapack.f90:108-176, on the imaginary axis where
 * eps~ = 1 - v^1/2 chi0 v^1/2 is HPD because chi0(iw) <= 0).  Blocked
 * Gauss-Jordan, FP64.  a: device, nbatch matrices at stride lda*n.
 * Returns QSGW_ERR_NUMERIC (after the batch completes) if a pivot block is
 * not invertible.                                                          */
int qsgw_zminv_hpd_batched_d(double *a, int n, int lda, int nbatch);
/* The same inverse without any device allocation (no counterpart in the
 * reference; it is an addition of this library).  For callers that cannot
 * call cudaMalloc at this point: a driver that already keeps the device full
 * with resident W(iw) stacks (the reference's --keepwv mode does this, and
 * hvccfp0 sleeps and retries when device memory runs out), or a caller whose
 * stream pipeline must not meet the implicit device synchronisation of
 * cudaMalloc / cudaFree.  Needs no qsgw_init; runs on the current device and
 * on `stream` (a cudaStream_t, 0 = default stream) and returns when the batch
 * is done.  Limit: n * nbatch <= 16384 (larger sizes return QSGW_ERR_ARG).
 * The Gauss-Jordan panels and the status word live in one static device
 * array of 16 MiB that every GPU loading the library holds until exit; the
 * first call on a device looks up that array's device address.  Every call
 * waits for its stream to read the status word, so no call can be recorded
 * into a CUDA graph: on a capturing stream it returns QSGW_ERR_UNSUPPORTED
 * before enqueuing anything.  All calls share the array: calls that overlap
 * on the GPU race and must not be issued concurrently.                     */
int qsgw_zminv_hpd_batched_noalloc_d(double *a, int n, int lda, int nbatch,
                                     void *stream);

/* ---- Hilbert transform of the chi0 histogram: drop-in for dpsion_init +
 * dpsion_chiq (dpsion5.f90:77-137, 174-292; hilbertmat.f90:14-79), time
 * reversal (npm = 1), no chi+-.
 * rcxq (device, npr*npr_col x (nwhis+1) complex, slots 0..nwhis as x0gemm
 * leaves them), frhis (host, nwhis+1 increasing bin edges, Hartree), freq_i
 * (host, niw), freq_r (host, nw+1, freq_r[0] = 0; nw = -1 skips the real
 * axis), ecut (>= 1e9: no Gaussian cut), smearx0 (GWinput SmearX0: the
 * Gaussian filter of the bins, gaussianfilterhis dpsion5.f90:459-483; 0 =
 * off).  zxqi (device, npr*npr_col x niw)
 * = chi0(i freq_i), zxq (device, npr*npr_col x (nw+1)) = chi0(freq_r): the
 * reference leaves the latter in rcxq(:, :, 0:nw); rcxq is not modified here. */
int qsgw_dpsion_chiq_d(const double *rcxq, int npr, int npr_col, int nwhis,
                       const double *frhis, int niw, const double *freq_i,
                       int nw, const double *freq_r, double ecut,
                       double smearx0, double *zxqi, double *zxq);
/* The transform matrix that call applies, on the host (no GPU needed): b
 * (complex, (nwhis+1) x (niw + nw + 1), column-major) with b(0, j) = 0 and
 * b(i, j) = f_i imatt(j, i) for the imaginary columns, b(i, niw + t) =
 * f_i rmatt(t, i) + i f_i [i == t] (f_0 = 1) for the real ones, f_i =
 * -wfac / (R_i - L_i) the bin normalisation, then (smearx0 != 0) rows 1..
 * nwhis replaced by gfmat^T b: chi0 = rcxq . b.                            */
int qsgw_dpsion_matrix(int nwhis, const double *frhis, int niw,
                       const double *freq_i, int nw, const double *freq_r,
                       double ecut, double smearx0, double *b);

/* ---- chi0 rank-k accumulation: drop-in for x0gemm (x0gemm.f90:2-97) ----
 * rcxq(npr, npr_col, (1-npm)*nwhis : nwhis) += sum over pairs of
 *   conj(zmel(:,it,itp)) * whw * zmel(ipr_col-1+:, it, itp)^T
 * per (jpm, iw) bin, the bin landing in slab iw*(3-2*jpm).
 * zmel(nbb, nm1:nm2, nqtot) as get_zmel_init_gemm leaves it (conjugated).
 * Pair tables are m_x0kf's (x0kf_v4h.f90:40-41,118-133), 1-based, read in
 * icoun = icounkmink..icounkmaxk; only pairs with ns1 <= it <= ns2 count.
 * whwc has ncount entries.  Index tables are host arrays in both variants. */
int qsgw_x0gemm(double *rcxq, int npr, int ipr_col, int npr_col, int nwhis,
                int npm, int ns1, int ns2, const double *zmel, int nbb,
                int nm1, int nm2, int nqtot, int icounkmink, int icounkmaxk,
                const int *itc, const int *itpc, const int *jpmc,
                const int *iwini, const int *iwend, const int *icouini,
                const double *whwc, int ncount);
int qsgw_x0gemm_d(double *rcxq_d, int npr, int ipr_col, int npr_col,
                  int nwhis, int npm, int ns1, int ns2, const double *zmel_d,
                  int nbb, int nm1, int nm2, int nqtot, int icounkmink,
                  int icounkmaxk, const int *itc, const int *itpc,
                  const int *jpmc, const int *iwini, const int *iwend,
                  const int *icouini, const double *whwc, int ncount);

/* ---- chi0 for all k-points and all imaginary frequencies in one call
 * (the k-loop of x0kf_zxq, x0kf_v4h.f90:233-290, with the direct iw
 * Lorentzian weights that stand in for the tetrahedron weights):
 *   chi0(:,:,iw) = sum_k sum_{pairs of k} w(pair,iw) conj(z) z^T,
 *   w = -2 de / (de^2 + freq_i(iw)^2) / nk,   de = e_unocc - e_occ.
 * zcols_d: device, complex (npr, ncol) = the zmel columns of every k
 * (zmel(:, it, itp) of k stored at column col0[k] + (it-1) + nocc_k*(itp-1)).
 * eocc/eunocc: host, concatenated per k (offsets by prefix sums of nocc/nun).
 * chi0_d: device complex (npr, npr, niw), overwritten.  The weights are
 * formed on the GPU in FP64.  Uses the precision set by qsgw_set_precision. */
int qsgw_chi0_lorentz_d(double *chi0_d, int npr, int niw, const double *freq_i,
                        int nk, const int *nocc, const int *nun,
                        const double *eocc, const double *eunocc,
                        const double *zcols_d, int ldz);
/* The same chi0 added into chi0_d (not cleared) for a batch of nkb k-points
 * of an nk_total mesh (weights carry 1/nk_total): calling it once per batch
 * streams the zmel columns through the GPU when all k cannot be resident
 * (N = 1500 with 512 k and up to 48 000 pairs per k: 369 GB of zmel).  No
 * autotuning trials.                                                       */
int qsgw_chi0_lorentz_acc_d(double *chi0_d, int npr, int niw, const double *freq_i,
                            int nk_total, int nkb, const int *nocc, const int *nun,
                            const double *eocc, const double *eunocc,
                            const double *zcols_d, int ldz);
/* Same with host chi0 / zcols (copied in and out inside the call). */
int qsgw_chi0_lorentz(double *chi0, int npr, int niw, const double *freq_i,
                      int nk, const int *nocc, const int *nun,
                      const double *eocc, const double *eunocc,
                      const double *zcols, int ldz);

/* ---- W - v on the imaginary axis: drop-in for the per-iw block of
 * WVIllwI (m_llw.f90:265-376, q /= 0 branch, iq <= nqibz):
 *   chi *= 2 if nspin == 1 (in place, :299-303); chi -> m2e^H chi m2e if
 *   is_x0_m_basis; eps~ = 1 - v^1/2 chi v^1/2; zw = v^1/2 (eps~^-1 - 1)
 *   v^1/2; zw -> m2e zw m2e^H if is_wc_m_basis and iq /= 1.
 * iq == 1 skips the head row/column (ix = 1).  zw(nblochpmx,nblochpmx,niw)
 * is overwritten (rows/cols beyond ngb zero).  All iw in one batch.        */
int qsgw_wvi_llw(double *zxqi, int ngb, int niw, int nspin,
                 const double *vcousq, const double *m2e, int is_x0_m_basis,
                 int is_wc_m_basis, int iq, double *zw, int nblochpmx);
int qsgw_wvi_llw_d(double *zxqi_d, int ngb, int niw, int nspin,
                   const double *vcousq, const double *m2e_d,
                   int is_x0_m_basis, int is_wc_m_basis, int iq,
                   double *zw_d, int nblochpmx);

/* ---- Sigma_c band sum: drop-in for get_correlation_block of
 * sxcf_scz_correlation (m_sxcf_gemm.f90:407-612) for one task
 * (kx, irot, ip, isp, icount).                                            */
typedef struct qsgw_sxcf_args {
  int ngb;          /* product-basis size = nbb (zmel rows)                 */
  int nblochpmx;    /* leading dimension of the W records                   */
  int ns1, ns2;     /* middle states [ns1, ns2] (nstti/nstte)               */
  int ns2r;         /* last middle state of the pole part (nstte2)          */
  int ntqxx, ntq;   /* target states used; leading dimension of zsec        */
  int niw, nw;      /* imaginary points; real-axis records 0..nw            */
  int nwxi, nwx;    /* real-axis window (nwxic, nwxc)                       */
  int nctot;        /* core states at the head of ekc                       */
  int nekc;         /* length of ekc (nctot + nband)                        */
  int keepwv;       /* 1: W given as packed upper triangles (--keepwv)      */
  double ef, esmr, wkkr, ua;
  const double *omega;   /* host (ntq): eq(1:ntq), Ry                       */
  const double *ekc;     /* host (nekc): [ecore; e(q-k)], Ry                */
  const double *freqx;   /* host (niw): Gauss points x in (0,1)             */
  const double *wwx;     /* host (niw): their weights                       */
  const double *expa;    /* host (niw): exp(-ua^2 w^2)                      */
  const double *freq_r;  /* host (nw+1): real-axis mesh, freq_r(0) = 0      */
  const double *zmel;    /* complex (ngb, ns2-ns1+1, ntqxx), M basis        */
  const double *wc_imag; /* complex (nblochpmx,nblochpmx,niw+1): slot 0 is
                            W(w=0)-v (first __WVR record), 1..niw __WVI; with
                            keepwv: (ngb(ngb+1)/2, niw+1) packed upper      */
  const double *wc_real; /* complex (nblochpmx,nblochpmx,nw+1) __WVR records;
                            with keepwv: packed (ngb(ngb+1)/2, nw+1) of the
                            already symmetrised (W+W^H)/2                   */
  double *zsec;          /* complex (ntq, ntq), accumulated                 */
} qsgw_sxcf_args;
/* Host pointers for every array. */
int qsgw_sxcf_correlation(const qsgw_sxcf_args *args);
/* zmel, wc_imag, wc_real, zsec are device pointers; the tables stay host. */
int qsgw_sxcf_correlation_d(const qsgw_sxcf_args *args);
/* ntask tasks (device pointers, as qsgw_sxcf_correlation_d): the same result
 * as calling qsgw_sxcf_correlation_d on tasks[0], tasks[1], ... in order
 * (tasks may share zsec; it accumulates in that order).  It replaces the
 * loop over (irot, ip, isp, icount) of sxcf_scz_correlation
 * (m_sxcf_gemm.f90:369-384).  With QSGW_PREC_SPLIT_I8, consecutive tasks of
 * equal ngb and slice count share one launch of the int8 contraction (up to
 * 8 GiB of slice scratch per launch; the first task of a shape whose slice
 * count is automatic runs alone to choose it); every other precision runs
 * the tasks one by one. */
int qsgw_sxcf_correlation_batch_d(const qsgw_sxcf_args *tasks, int ntask);

/* Imaginary-axis weights wgtim(0:niw, ns1:ns2, ntqxx), FP64 on the GPU
 * (m_sxcf_gemm.f90:432-458, npm = 1).  wgtim_d: device (niw+1, nm, ntqxx). */
int qsgw_sxcf_wgtim_d(double *wgtim_d, int niw, int ns1, int ns2, int ntqxx,
                      int nctot, const double *omega, const double *ekc,
                      int nekc, double esmr, double wkkr, double ua,
                      const double *freqx, const double *wwx,
                      const double *expa);

/* ---- Sigma_x block of sxcf_scz_exchange (m_sxcf_gemm.f90:203-231):
 *   zsec += -wkkr * zmel^H (wtff * vcoud * zmel), K = (ngb, it)
 * wtff(it) = 1 for cores, wfacx(-1d99, ef, ekc(it+nctot), esmr) for valence
 * (the reference's index).  zmel: device (ngb, ns2-ns1+1, ntqxx) in the E
 * basis; zsec: device (ntq, ntq); vcoud (effective, the kx == 1 head
 * replacement of :218 applied by the caller) and ekc are host arrays.      */
int qsgw_sxcf_exchange_d(double *zsec_d, int ntq, const double *zmel_d, int ngb,
                         int ns1, int ns2, int ntqxx, const double *vcoud,
                         const double *ekc, int nekc, int nctot, double ef,
                         double esmr, double wkkr);

/* ---- QP energies and the Hermitian self-energy of hqpe_sc
 * (main_hqpe.sc.f90:150-161, 178-180), nq q-points at once, FP64:
 *   eqp(i) = elda(i) + [SEx + SExcore + Re SEc](i,i) * Hartree - vxc(i)   (eV)
 *   Sigma_h = SEx + SExcore + (SEc + SEc^H)/2 - vxc_band/2                 (Ha)
 * Matrices (ntq, ntq) with leading dimension ld, nq of them at stride ld*ld;
 * vxc_band in Ry (evec^H v_xc evec); elda, vxc, eqp (ntq, nq) in eV; all
 * device arrays.                                                           */
int qsgw_hqpe_d(const double *sex2_d, const double *sexcore2_d,
                const double *sec2_d, const double *vxc_band_ry_d,
                const double *elda_ev_d, const double *vxc_ev_d, int ntq, int ld,
                int nq, double *eqp_ev_d, double *sigma_herm_d);

/* ---- Product-basis matrix elements <psi|psi M>, muffin-tin part of
 * get_zmel_init_gemm (m_zmel.f90:323-390, ncc = 0): every atom in one launch.
 * zmelt: device (nbloch, nm1:nm2, ntp0); only the rows of the atoms' product
 * functions are written (zero zmelt first).  cphim: device (ldm, nm1v:nm2v)
 * valence coefficients at q-k, cphiq: device (ldq, ntp0) at q.            */
typedef struct qsgw_zmel_atom {
  const double *ppb_d;   /* device (nlnm, nlnm, mdim) radial integrals x rotated
                            Gaunt coefficients: rows/cols core 1..nc then
                            valence nc+1..nc+nv (set_ppb, m_zmel.f90:110-145) */
  int nlnm, nc, nv;      /* channels: total, core, valence (nv <= 96)        */
  int ias;               /* 1-based first row of the atom in cphim/cphiq     */
  int ics;               /* core-state offset of the atom                    */
  int ims;               /* 1-based first product-basis row (of iatomp)      */
  int mdim;              /* product functions of the atom                    */
  int ncore;             /* core states of the atom                          */
  double phase_re, phase_im;   /* exp(-i 2 pi k.tau)  (m_zmel.f90:325)       */
} qsgw_zmel_atom;
int qsgw_zmel_mt_d(double *zmelt_d, int nbloch, int nm1, int nm2, int nctot,
                   int ntp0, const double *cphim_d, int ldm,
                   const double *cphiq_d, int ldq, int natom,
                   const qsgw_zmel_atom *atoms);
/* Interstitial plane-wave part of get_zmel_init_gemm (m_zmel.f90:418-535):
 *   zmelt(row0+igc, it, itp) = phase(igc) * sum_{G1,G2} ggg(G1 - (Gc+G2) - nadd)
 *                              * geigq(G1, itp) * dgeigqk(G2, it)
 * for it = nm1v..nm2v (middle index of zmelt nm1..nm2), itp = 1..ntp0.
 * The G-vector tables are the reference's (getppx2, rppovl.f90:40-66):
 * nvggg/ggg (the ggg table), nvgcgp2 (composite vectors Gc+G2 and Gc-G1),
 * ngvecpB1/ngvecpB2 (plane waves at q and q-k), ngveccR (rotated Gc); the
 * inverse tables are built here.  The G1-first or G2-first order follows
 * the reference's choice (:439).  A composite vector missing from nvgcgp2
 * is an argument error.                                                    */
typedef struct qsgw_zmel_ipw_args {
  int ngc, ngp1, ngp2, ngcgp, nggg;
  int ntp0, nm1, nm2, nm1v, nm2v;
  int ldz, row0;               /* zmelt_d (ldz, nm1:nm2, ntp0); row0 = nbloch    */
  int nadd[3];
  const int *ngvecpB1;         /* host (3, ngp1) */
  const int *ngvecpB2;         /* host (3, ngp2) */
  const int *ngveccR;          /* host (3, ngc)  */
  const int *nvgcgp2;          /* host (3, ngcgp) */
  const int *nvggg;            /* host (3, nggg) */
  const double *ggg;           /* host complex (nggg) */
  const double *phase;         /* host complex (ngc) */
  const double *geigq_d;       /* device complex (ldgq, ntp0) */
  int ldgq;
  const double *dgeigqk_d;     /* device complex (ldgk, nm1v:nm2v), conjugated */
  int ldgk;
  double *zmelt_d;
} qsgw_zmel_ipw_args;
int qsgw_zmel_ipw_d(const qsgw_zmel_ipw_args *args);
/* M->E change and conjugation (m_zmel.f90:546-563, 590-594):
 * zmel(nbb, nmtot*nqtot) = m2e^H zmelt (or a copy when is_m_basis), then
 * conj when zmelconjg.  m2e: device (ngb, nbb).                            */
int qsgw_zmel_m2e_d(double *zmel_d, const double *zmelt_d, int ngb, int nbb,
                    int nmtot, int nqtot, const double *m2e_d, int is_m_basis,
                    int zmelconjg);

/* ---- Coulomb-matrix eigenproblem (main_hvccfp0.f90:322-367 with zhgv_d,
 * m_lapack.f90:203-229): (-v) z = lambda O z, vcoud = -lambda, i.e. the
 * eigenvalues of v in descending order with O-orthonormal eigenvectors.
 * v_d: device (lda, n) Hermitian, overwritten by the eigenvectors z (column
 * j belongs to vcoud[j]); o_d: device (lda, n) overlap or NULL (identity);
 * vcoud: host (n).  FP64 parallel cyclic Jacobi.                          */
int qsgw_zhegv_d(double *v_d, const double *o_d, int n, int lda, double *vcoud);

/* ---- Autotuner.  mode 0: launch parameters from heuristics (default);
 * mode 1: the first call with a new problem shape times the candidates of a
 * tunable parameter (today the split-K count of the chi0 contractions, FP64
 * and split precision) on the caller's data and keeps the fastest; later
 * calls with that shape reuse it.  cache_path (may be NULL) names a JSON file
 * {"shape key": choice} read now and rewritten when a choice is added.
 * No tuning while a graph is being recorded (cached choices still apply).
 * report: the current choices as JSON text (QSGW_ERR_ARG if len is short).  */
int qsgw_set_autotune(int mode, const char *cache_path);
int qsgw_autotune_report(char *buf, int len);

/* ---- CUDA graph of a recorded call sequence (no reference counterpart: the
 * reference launches every kernel from the host each time).  Between
 * qsgw_graph_begin and qsgw_graph_end the device entry points
 * (qsgw_chi0_lorentz_d, qsgw_wvi_llw_d, qsgw_sxcf_correlation_d, ... and any
 * other work the caller puts on the library stream) are recorded instead of
 * run; qsgw_graph_launch replays them.  Host tables passed during recording
 * (frequencies, energies, band counts, pole tables) are copied into pinned
 * memory owned by the graph and replayed as recorded; device arrays are read
 * at replay time.  Record only after the same calls ran once (scratch must
 * not grow while recording: such a call fails with QSGW_ERR_UNSUPPORTED).
 * One graph per context; begin replaces the previous one.  The library
 * stream must not be the legacy default stream.                          */
int qsgw_graph_begin(void);
int qsgw_graph_end(void);
int qsgw_graph_launch(void);
int qsgw_graph_destroy(void);

/* ---- Real frequency axis (WVRllwR, m_llw.f90:49-264).
 * chi0 of the Lorentzian model on real frequencies:
 *   chi0(w) = conj(Z) diag(f) Z^T,  f = [1/(w - de + i eta) - 1/(w + de + i eta)] / nk
 * (its value at w = i nu is the weight of qsgw_chi0_lorentz_d), computed as
 * two Hermitian parts (Re f, Im f) on the chi0 engine; freq_r host (nw),
 * Hartree; output (npr, npr, nw) complex, overwritten.                     */
int qsgw_chi0_lorentz_real_d(double *chi0_d, int npr, int nw, const double *freq_r,
                             double eta, int nk, const int *nocc, const int *nun,
                             const double *eocc, const double *eunocc,
                             const double *zcols_d, int ldz);
/* W - v on real frequencies: the WVIllwI block with eps~ general, inverted
 * by Gauss-Jordan with partial pivoting (zminv, m_lapack.f90:108-176);
 * arguments as qsgw_wvi_llw_d.  A singular eps~ sets the status word
 * (qsgw_synchronize returns QSGW_ERR_NUMERIC).                              */
int qsgw_wvr_llw_d(double *zxq_d, int ngb, int nw, int nspin, const double *vcousq,
                   const double *m2e_d, int is_x0_m_basis, int is_wc_m_basis, int iq,
                   double *zw_d, int nblochpmx);
/* in-place inverses of nbatch general complex n x n matrices (lda, batch
 * stride lda*n), partial pivoting; a zero pivot sets the status word.      */
int qsgw_zminv_batched_d(double *a, int n, int lda, int nbatch);

/* ---- Tetrahedron histogram weights of chi0 (tetwt5x_dtet4 with lindtet6,
 * SRC/subroutines/tetwt5.f90:9-787, tetrahedron_matrix_linear = F, npm = 1,
 * one micro tetrahedron): for every tetrahedron and every pair (occupied
 * band ib < nocc at k, band jb < nunocc at k+q) the Rath-Freeman integral
 *   wtthis(ihis) = int_bin d omega int_tet d^3k f(e_k)(1 - f(e_k+q)) delta(omega - (e_k+q - e_k)/2)
 * is added to each corner k: w_d(ihis, jb, ib, k) += wtthis * pi / (4 voltot)
 * (w_d device, nwhis x nunocc x nocc x nk, accumulated: zero it first).
 * idtet: host (4, ntet) 0-based corner k indices; qbzw: host (3, nk) k
 * vectors; ek/ekq: host (nband, nk) energies at k and k+q (Ry, as the
 * reference; omega in Hartree); frhis: host (nwhis + 1) increasing bin
 * edges (Hartree).  voltot (host, may be NULL) <- total volume.  A pair
 * whose excitation energies leave the histogram sets the status word
 * (qsgw_synchronize returns QSGW_ERR_NUMERIC); the reference stops there.
 * Dense output instead of the reference's (ibjb, ihw, nhw, jhw, whw)
 * storage; its symmetrisation over degenerate bands is
 * qsgw_tetwt_symmetrize below.                                             */
int qsgw_tetwt_hist_d(double *w_d, int nk, int nocc, int nunocc, int nwhis,
                      const int *idtet, int ntet, const double *qbzw,
                      const double *ek, const double *ekq, int nband,
                      double efermi, const double *frhis, double *voltot);
/* The reference's symmetrisation over degenerate bands (tetwt5.f90:347-423,
 * job 1, npm = 1, no core states) on the host copy of those weights (w:
 * nwhis x nunocc x nocc x nk, in place): for every k, the levels ek(1:nocc, k)
 * and ekq(1:nunocc, k) (nband x nk, Ry) are cut into groups wherever two
 * neighbours differ by more than 1e-4 (chkdgn, :868-912), and every (ib, jb)
 * of a group pair gets the pair's mean histogram (summed ib-major, divided
 * by the group-pair size, as the reference).  A group cut by nocc or nunocc
 * is averaged over its members inside the array.  Host-only.              */
int qsgw_tetwt_symmetrize(double *w, int nk, int nocc, int nunocc, int nwhis,
                          const double *ek, const double *ekq, int nband);
/* Pair/bin lists of qsgw_x0gemm from those weights copied to the host
 * (w: nwhis x nunocc x nocc x nk): the index accumulation of X0kf_v4hz_init
 * (x0kf_v4h.f90:48-142), npm = 1, no core states, no cRPA.  A pair with any
 * nonzero bin gets one entry (k-major, then ib, then jb): itc = ib+1, itpc =
 * jb+1, jpmc = 1, the bin range [iwini, iwend] from its first to its last
 * nonzero bin, icouini = 1-based start of its weights in whwc; icounkmin/max
 * (nk each) = the entries of each k, 1-based.  job 0 sets *ncoun, *ncount;
 * job 1 fills arrays of those sizes (*ncoun, *ncount = their capacities).
 * Host-only: needs no GPU and no qsgw_init.                                */
int qsgw_x0_lists(const double *w, int nk, int nocc, int nunocc, int nwhis,
                  int job, int *ncoun, int *ncount, int *itc, int *itpc,
                  int *jpmc, int *iwini, int *iwend, int *icouini,
                  double *whwc, int *icounkmin, int *icounkmax);

/* ---- W record files __WVI.<iq> / __WVR.<iq> in the reference's layout:
 * fixed records without markers, record rec at byte (rec-1)*recl, one
 * nblochpmx x nblochpmx column-major matrix per record, complex(8)
 * (recl = 16 nblochpmx^2) or complex(4) when kind4 != 0 (m_mpiio.f90:12-73,
 * written at m_llw.f90:177, 373; read at m_sxcf_gemm.f90:317-354).
 * write: records rec0..rec0+nrec-1 from the device stack zw_d (nrec
 * matrices); the file is created when missing, other records are kept.
 * read: pack = 0 -> full matrices into out_d (nrec x nblochpmx^2);
 * pack = 1 -> upper triangle (i <= j, column by column) of the leading
 * ngb x ngb block, the WVI form of keepwv; pack = 2 -> the same of
 * (W + W^H)/2, the WVR form (m_sxcf_gemm.f90:337-354); out_d then holds
 * nrec x ngb(ngb+1)/2 values.                                              */
int qsgw_wv_write_d(const char *path, const double *zw_d, int nblochpmx, int rec0,
                    int nrec, int kind4);
int qsgw_wv_read_d(const char *path, double *out_d, int nblochpmx, int rec0,
                   int nrec, int kind4, int pack, int ngb);

/* ---- Sequential unformatted files (host memory, no GPU needed): a record
 * is a 4-byte length, the payload and the length again (the gfortran /
 * ifort / nvfortran default), 4-byte integers, at most 2^31-1 bytes.
 *
 * __Vcoud.<iq>, the Coulomb eigenproblem's output: records ngb | q(3) |
 * vcoud(ngb) | zcousq(ngb, ngb) complex(8), as main_hvccfp0.f90:396-400
 * writes them and Readvcoud (m_readVcoud.f90:30-40) reads them.
 * read: *ngb and q (if non-NULL) from the first two records; with vcoud,
 * vcousq and zcousq all NULL it stops there (a size query), else ngb <=
 * ngb_cap is required and each non-NULL array is filled; vcousq =
 * sqrt(vcoud) as Readvcoud forms it.  A file whose length is not the one
 * its header implies, or a record whose length does not match this layout,
 * is an error (QSGW_ERR_ARG), found before any array is sized from the
 * header.                                                                  */
int qsgw_vcoud_write(const char *path, int ngb, const double *q,
                     const double *vcoud, const double *zcousq);
int qsgw_vcoud_read(const char *path, int ngb_cap, int *ngb, double *q,
                    double *vcoud, double *vcousq, double *zcousq);
/* SEX2U, SEXcore2U, SEC2U (D for spin 2), the self-energy matrices: a
 * header record head[8] = nspin, nq, ntq, nqbz, nqibz, n1, n2, n3, then for
 * ip = 1..nq one record is, qibz(1:3, ip), zsec(1:ntq, 1:ntq, ip)
 * (main_hsfp0.sc.f90:322, 333, 340, 359; read at main_hqpe.sc.f90:132-148).
 * write: nq = head[1], ntq = head[2]; qibz (3, nq) real(8); zsec (ntq, ntq,
 * nq) complex(8); every record carries the spin index is.
 * read: head from the header; with isx, qibz and zsec all NULL it stops
 * there, else nq <= nq_cap and ntq <= ntq_cap are required and the non-NULL
 * arrays are filled (isx (nq): each record's spin index).  The file length
 * is checked against the header first, as for __Vcoud.                    */
int qsgw_sigma_write(const char *path, const int *head, int is,
                     const double *qibz, const double *zsec);
int qsgw_sigma_read(const char *path, int *head, int nq_cap, int ntq_cap,
                    int *isx, double *qibz, double *zsec);

/* ---- Learned W_c(q, i w) frequency interpolator.  No counterpart in the
 * reference: it stands in for computing chi0 and W at every frequency of
 * the imaginary grid.  One sample = one real channel of one element of
 * W_c(q) at one target frequency; features (16) = the channel at the na
 * anchor frequencies / s (s = their largest magnitude), the target's
 * Gauss-Legendre x, 1; output (normalised by s) = C[h] . x + MLP(x), with a
 * linear head row h per target (FP32, 128 rows; rows >= 64 take no MLP
 * term) and an MLP 16-256-256-1 (ReLU, BF16 weights with an FP32 master
 * copy, FP32 accumulation).  Trained with Adam on the s^2-weighted squared
 * error, the head rows first set by least squares.
 * Parameters live in the library (one network per process).              */
int qsgw_wsurr_init(unsigned long long seed);
int qsgw_wsurr_nparam(void);
/* host FP32 parameter vector: set != 0 writes it (and the BF16 copy), else reads */
int qsgw_wsurr_params(float *host, int set);
/* proj_d (nslot, 2 nb nb) float <- W_c(ridx[i], cidx[j]) re/im of each slot
 * (channel 2 (i + nb j) + c); wc_d: device slots of ld x ld complex, slot
 * stride ld*ld; ridx, cidx: host (nb), cidx NULL = ridx.                   */
int qsgw_wsurr_project_d(const double *wc_d, int ld, int nslot, const int *ridx,
                         const int *cidx, int nb, float *proj_d);
/* samples of every (q, channel, target), target fastest: proj_d (nq, nw, ne)
 * float; anchors/targets: host slot indices into nw (na <= 10); thead: host
 * head row of each target (< 128); xcoord: host (nw) Gauss-Legendre x.
 * Element features (x[na+2..na+5]): ftab[row], ftab[col], re/im, diagonal,
 * for the block rows rid and columns cid (host, nb each, ne = 2 nb nb);
 * ftab: host (nftab) per-index feature, NULL = no element features.
 * Outputs (device): x_d (samples, 16), tix_d (samples); optional y_d
 * (normalised value at the target), wgt_d (s^2), scale_d (s).              */
int qsgw_wsurr_features_d(const float *proj_d, int nq, int nw, int ne,
                          const int *anchors, int na, const int *targets,
                          const int *thead, int nt, const float *xcoord,
                          const int *rid, const int *cid, int nb,
                          const float *ftab, int nftab, float *x_d, int *tix_d,
                          float *y_d, float *wgt_d, float *scale_d);
/* least squares of the head rows: accumulate the s^2-weighted normal
 * equations of n samples in the features order (nt targets, thead: host
 * head row of each), then solve them (ridge * trace/16 added to the
 * diagonal) into the head rows that received samples, clearing the sums.  */
int qsgw_wsurr_lsq_accumulate_d(const float *x_d, const float *y_d,
                                const float *wgt_d, long long n, int nt,
                                const int *thead);
int qsgw_wsurr_lsq_solve(double ridge, int *rows_solved);
/* inference: y_d <- network output (normalised) for batch samples */
int qsgw_wsurr_forward_d(const float *x_d, const int *tix_d, float *y_d, int batch);
/* gradient only (no update): grad_host <- dL/dparams, loss_host <- L;
 * wgt_d NULL = unweighted mean squared error                               */
int qsgw_wsurr_grad_d(const float *x_d, const int *tix_d, const float *y_d,
                      const float *wgt_d, int batch, float *loss_host,
                      float *grad_host);
/* nsteps Adam steps on random mini-batches of `batch` rows drawn from the n
 * samples (counter-based hash of seed and step); loss_host <- last batch's L */
int qsgw_wsurr_train_d(const float *x_d, const int *tix_d, const float *y_d,
                       const float *wgt_d, long long n, int batch, int nsteps,
                       float lr, unsigned long long seed, float *loss_host);
/* full matrix, linear head only: slot tslot[t] of wc_d (nslot slots of ld x
 * ld, n x n used) <- s * C[thead[t]] . x built from the anchor slots aslot;
 * txc: host Gauss-Legendre x of each target; ftab: host (n) per-index
 * feature as in qsgw_wsurr_features_d, or NULL.                            */
int qsgw_wsurr_head_full_d(double *wc_d, int n, int ld, int nslot,
                           const int *aslot, int na, const int *tslot,
                           const int *thead, const float *txc, int nt,
                           const float *ftab);
/* block (idx x idx) of the target slots <- pred_d * scale_d; pred_d and
 * scale_d hold 2 nb nb nt samples of one q in the features order (target
 * fastest, then channel 2 (i + nb j) + re/im)                              */
int qsgw_wsurr_scatter_d(double *wc_d, int ld, int nslot, const int *idx, int nb,
                         const int *tslot, int nt, const float *pred_d,
                         const float *scale_d);

#ifdef __cplusplus
}
#endif
#endif /* QSGW_B200_H */
