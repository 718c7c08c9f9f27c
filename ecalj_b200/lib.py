"""ctypes binding of libqsgw_b200.so, mirroring the reference routines the
C ABI replaces (names, argument meaning, 1-based Fortran indices).

Host-array calls take numpy arrays (complex128 / float64 / int32, Fortran
order where the reference array is multi-dimensional).  Device calls take
torch CUDA tensors.  Every failure raises ``QSGWError`` with the library's
status code and message; there is no CPU fallback: if the shared library is
missing the import of this module fails.
"""
import ctypes
import os

import numpy as np

from . import build as _build

_PKG = os.path.dirname(os.path.abspath(__file__))
LIBPATH = os.path.join(_PKG, "libqsgw_b200.so")

c_int = ctypes.c_int
c_dbl = ctypes.c_double
c_vp = ctypes.c_void_p
c_ip = ctypes.POINTER(ctypes.c_int)
c_dp = ctypes.POINTER(ctypes.c_double)

STATUS = {0: "OK", -1: "ERR_ARG", -2: "ERR_CUDA", -3: "ERR_OOM", -4: "ERR_NOTINIT",
          -5: "ERR_NUMERIC", -6: "ERR_TIMEOUT", -7: "ERR_UNSUPPORTED"}
PREC_FP64 = 0
PREC_SPLIT_F16 = 1
PREC_SPLIT_I8 = 2


class QSGWError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"{STATUS.get(code, code)}: {msg}")
        self.code = code


class SxcfArgs(ctypes.Structure):
    """Mirror of ``qsgw_sxcf_args`` (include/qsgw_b200.h)."""
    _fields_ = [("ngb", c_int), ("nblochpmx", c_int), ("ns1", c_int), ("ns2", c_int),
                ("ns2r", c_int), ("ntqxx", c_int), ("ntq", c_int), ("niw", c_int),
                ("nw", c_int), ("nwxi", c_int), ("nwx", c_int), ("nctot", c_int),
                ("nekc", c_int), ("keepwv", c_int),
                ("ef", c_dbl), ("esmr", c_dbl), ("wkkr", c_dbl), ("ua", c_dbl),
                ("omega", c_vp), ("ekc", c_vp), ("freqx", c_vp), ("wwx", c_vp),
                ("expa", c_vp), ("freq_r", c_vp),
                ("zmel", c_vp), ("wc_imag", c_vp), ("wc_real", c_vp), ("zsec", c_vp)]


class ZmelAtom(ctypes.Structure):
    """Mirror of ``qsgw_zmel_atom``."""
    _fields_ = [("ppb_d", c_vp), ("nlnm", c_int), ("nc", c_int), ("nv", c_int), ("ias", c_int),
                ("ics", c_int), ("ims", c_int), ("mdim", c_int), ("ncore", c_int),
                ("phase_re", c_dbl), ("phase_im", c_dbl)]


class ZmelIpwArgs(ctypes.Structure):
    """Mirror of ``qsgw_zmel_ipw_args``."""
    _fields_ = [("ngc", c_int), ("ngp1", c_int), ("ngp2", c_int), ("ngcgp", c_int), ("nggg", c_int),
                ("ntp0", c_int), ("nm1", c_int), ("nm2", c_int), ("nm1v", c_int), ("nm2v", c_int),
                ("ldz", c_int), ("row0", c_int), ("nadd", c_int * 3),
                ("ngvecpB1", c_vp), ("ngvecpB2", c_vp), ("ngveccR", c_vp), ("nvgcgp2", c_vp), ("nvggg", c_vp),
                ("ggg", c_vp), ("phase", c_vp), ("geigq_d", c_vp), ("ldgq", c_int), ("dgeigqk_d", c_vp),
                ("ldgk", c_int), ("zmelt_d", c_vp)]


_SIGS = {
    "qsgw_init": [c_int],
    "qsgw_finalize": [],
    "qsgw_set_stream": [c_vp],
    "qsgw_synchronize": [],
    "qsgw_set_precision": [c_int, c_int],
    "qsgw_set_sigc_kernel": [c_int],
    "qsgw_set_host_async": [c_int],
    "qsgw_x0_lists": [c_vp, c_int, c_int, c_int, c_int, c_int, c_vp, c_vp, c_vp, c_vp, c_vp, c_vp, c_vp, c_vp,
                      c_vp, c_vp, c_vp],
    "qsgw_tetwt_symmetrize": [c_vp, c_int, c_int, c_int, c_int, c_vp, c_vp, c_int],
    "qsgw_dpsion_matrix": [c_int, c_vp, c_int, c_vp, c_int, c_vp, c_dbl, c_dbl, c_vp],
    "qsgw_dpsion_chiq_d": [c_vp, c_int, c_int, c_int, c_vp, c_int, c_vp, c_int, c_vp, c_dbl, c_dbl, c_vp, c_vp],
    "qsgw_get_precision": [c_ip, c_ip],
    "qsgw_set_accuracy": [c_dbl, c_dbl],
    "qsgw_last_error": [ctypes.c_char_p, c_int],
    "qsgw_profile": [c_int],
    "qsgw_profile_get": [ctypes.c_char_p, c_dp, ctypes.POINTER(ctypes.c_longlong)],
    "qsgw_zmm": [c_vp, c_vp, c_vp, c_int, c_int, c_int, c_int, c_int, c_dp, c_dp, c_int, c_int, c_int],
    "qsgw_zmm_d": [c_vp, c_vp, c_vp, c_int, c_int, c_int, c_int, c_int, c_dp, c_dp, c_int, c_int, c_int],
    "qsgw_zminv_hpd_batched_d": [c_vp, c_int, c_int, c_int],
    "qsgw_zminv_hpd_batched_noalloc_d": [c_vp, c_int, c_int, c_int, c_vp],
    "qsgw_x0gemm": [c_vp, c_int, c_int, c_int, c_int, c_int, c_int, c_int, c_vp, c_int, c_int, c_int,
                    c_int, c_int, c_int, c_vp, c_vp, c_vp, c_vp, c_vp, c_vp, c_vp, c_int],
    "qsgw_x0gemm_d": [c_vp, c_int, c_int, c_int, c_int, c_int, c_int, c_int, c_vp, c_int, c_int, c_int,
                      c_int, c_int, c_int, c_vp, c_vp, c_vp, c_vp, c_vp, c_vp, c_vp, c_int],
    "qsgw_chi0_lorentz_d": [c_vp, c_int, c_int, c_vp, c_int, c_vp, c_vp, c_vp, c_vp, c_vp, c_int],
    "qsgw_chi0_lorentz": [c_vp, c_int, c_int, c_vp, c_int, c_vp, c_vp, c_vp, c_vp, c_vp, c_int],
    "qsgw_wvi_llw": [c_vp, c_int, c_int, c_int, c_vp, c_vp, c_int, c_int, c_int, c_vp, c_int],
    "qsgw_wvi_llw_d": [c_vp, c_int, c_int, c_int, c_vp, c_vp, c_int, c_int, c_int, c_vp, c_int],
    "qsgw_sxcf_correlation": [ctypes.POINTER(SxcfArgs)],
    "qsgw_sxcf_correlation_d": [ctypes.POINTER(SxcfArgs)],
    "qsgw_sxcf_correlation_batch_d": [ctypes.POINTER(SxcfArgs), c_int],
    "qsgw_sxcf_wgtim_d": [c_vp, c_int, c_int, c_int, c_int, c_int, c_vp, c_vp, c_int, c_dbl, c_dbl,
                          c_dbl, c_vp, c_vp, c_vp],
    "qsgw_sxcf_exchange_d": [c_vp, c_int, c_vp, c_int, c_int, c_int, c_int, c_vp, c_vp, c_int, c_int, c_dbl,
                             c_dbl, c_dbl],
    "qsgw_hqpe_d": [c_vp, c_vp, c_vp, c_vp, c_vp, c_vp, c_int, c_int, c_int, c_vp, c_vp],
    "qsgw_zmel_mt_d": [c_vp, c_int, c_int, c_int, c_int, c_int, c_vp, c_int, c_vp, c_int, c_int,
                       ctypes.POINTER(ZmelAtom)],
    "qsgw_zmel_m2e_d": [c_vp, c_vp, c_int, c_int, c_int, c_int, c_vp, c_int, c_int],
    "qsgw_zmel_ipw_d": [c_vp],
    "qsgw_zhegv_d": [c_vp, c_vp, c_int, c_int, c_vp],
    "qsgw_set_autotune": [c_int, ctypes.c_char_p],
    "qsgw_autotune_report": [ctypes.c_char_p, c_int],
    "qsgw_graph_begin": [],
    "qsgw_graph_end": [],
    "qsgw_graph_launch": [],
    "qsgw_graph_destroy": [],
    "qsgw_chi0_lorentz_acc_d": [c_vp, c_int, c_int, c_vp, c_int, c_int, c_vp, c_vp, c_vp, c_vp, c_vp, c_int],
    "qsgw_chi0_lorentz_real_d": [c_vp, c_int, c_int, c_vp, ctypes.c_double, c_int, c_vp, c_vp, c_vp, c_vp, c_vp,
                                 c_int],
    "qsgw_wvr_llw_d": [c_vp, c_int, c_int, c_int, c_vp, c_vp, c_int, c_int, c_int, c_vp, c_int],
    "qsgw_zminv_batched_d": [c_vp, c_int, c_int, c_int],
    "qsgw_tetwt_hist_d": [c_vp, c_int, c_int, c_int, c_int, c_vp, c_int, c_vp, c_vp, c_vp, c_int, ctypes.c_double,
                          c_vp, c_vp],
    "qsgw_wv_write_d": [ctypes.c_char_p, c_vp, c_int, c_int, c_int, c_int],
    "qsgw_wv_read_d": [ctypes.c_char_p, c_vp, c_int, c_int, c_int, c_int, c_int, c_int],
    "qsgw_vcoud_write": [ctypes.c_char_p, c_int, c_vp, c_vp, c_vp],
    "qsgw_vcoud_read": [ctypes.c_char_p, c_int, c_ip, c_vp, c_vp, c_vp, c_vp],
    "qsgw_sigma_write": [ctypes.c_char_p, c_vp, c_int, c_vp, c_vp],
    "qsgw_sigma_read": [ctypes.c_char_p, c_vp, c_int, c_int, c_vp, c_vp, c_vp],
    "qsgw_wsurr_init": [ctypes.c_ulonglong],
    "qsgw_wsurr_nparam": [],
    "qsgw_wsurr_params": [c_vp, c_int],
    "qsgw_wsurr_project_d": [c_vp, c_int, c_int, c_vp, c_vp, c_int, c_vp],
    "qsgw_wsurr_lsq_accumulate_d": [c_vp, c_vp, c_vp, ctypes.c_longlong, c_int, c_vp],
    "qsgw_wsurr_lsq_solve": [ctypes.c_double, c_vp],
    "qsgw_wsurr_features_d": [c_vp, c_int, c_int, c_int, c_vp, c_int, c_vp, c_vp, c_int, c_vp, c_vp, c_vp, c_int,
                              c_vp, c_int, c_vp, c_vp, c_vp, c_vp, c_vp],
    "qsgw_wsurr_forward_d": [c_vp, c_vp, c_vp, c_int],
    "qsgw_wsurr_grad_d": [c_vp, c_vp, c_vp, c_vp, c_int, c_vp, c_vp],
    "qsgw_wsurr_train_d": [c_vp, c_vp, c_vp, c_vp, ctypes.c_longlong, c_int, c_int, ctypes.c_float,
                           ctypes.c_ulonglong, c_vp],
    "qsgw_wsurr_head_full_d": [c_vp, c_int, c_int, c_int, c_vp, c_int, c_vp, c_vp, c_vp, c_int, c_vp],
    "qsgw_wsurr_scatter_d": [c_vp, c_int, c_int, c_vp, c_int, c_vp, c_int, c_vp, c_vp],
}


def exported_symbols():
    """Names the header declares (kept in sync with include/qsgw_b200.h)."""
    return sorted(list(_SIGS) + ["qsgw_launch_count"])


_lib = None


def load(build_if_missing=False):
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIBPATH):
        if build_if_missing:
            _build.build()
        else:
            raise ImportError(f"{LIBPATH} is missing: run `python -m ecalj_b200.build`")
    lib = ctypes.CDLL(LIBPATH)
    for name, args in _SIGS.items():
        f = getattr(lib, name)
        f.argtypes = args
        f.restype = c_int
    lib.qsgw_launch_count.argtypes = []
    lib.qsgw_launch_count.restype = ctypes.c_longlong
    _lib = lib
    return lib


def last_error():
    buf = ctypes.create_string_buffer(1024)
    load().qsgw_last_error(buf, 1024)
    return buf.value.decode(errors="replace")


def _chk(rc):
    if rc != 0:
        raise QSGWError(rc, last_error())
    return rc


def _p(a):
    """Pointer of a numpy array or torch tensor (None passes NULL)."""
    if a is None:
        return None
    if isinstance(a, np.ndarray):
        return a.ctypes.data
    return a.data_ptr()


def _host_c128(a):
    a = np.asarray(a)
    if a.dtype != np.complex128 or not a.flags.f_contiguous:
        raise ValueError("expected a Fortran-ordered complex128 array")
    return a


def _i32(a):
    return np.ascontiguousarray(np.asarray(a, dtype=np.int32))


def _f64(a):
    return np.ascontiguousarray(np.asarray(a, dtype=np.float64))


# ---------------------------------------------------------------- context
_initialized = False


def init(device=0):
    global _initialized
    _chk(load().qsgw_init(device))
    _initialized = True


def finalize():
    global _initialized
    _chk(load().qsgw_finalize())
    _initialized = False


def initialized():
    """True between init() and finalize() in this process."""
    return _initialized


def set_stream(stream_handle):
    _chk(load().qsgw_set_stream(stream_handle))


def share_torch_stream():
    """Run torch and this library on one stream: a new torch stream becomes
    torch's current stream and the library's launch stream (the legacy
    default stream, handle 0, does not order work against the library's own
    non-blocking stream).  Returns the torch stream."""
    import torch
    s = torch.cuda.Stream()
    torch.cuda.set_stream(s)
    set_stream(s.cuda_stream)
    return s


def synchronize():
    _chk(load().qsgw_synchronize())


def set_precision(mode, nslices=2):
    _chk(load().qsgw_set_precision(mode, nslices))


def set_accuracy(sigc_qp_tol_ha=1e-3 / 27.211386245988, chi0_rel_tol=2e-5):
    """Targets of the automatic int8 slice count (set_precision(PREC_SPLIT_I8, 0))."""
    _chk(load().qsgw_set_accuracy(sigc_qp_tol_ha, chi0_rel_tol))


def set_host_async(on):
    """Host-pointer calls return once enqueued (True) or with their outputs written (False, default);
    in the asynchronous mode outputs are valid after synchronize()."""
    _chk(load().qsgw_set_host_async(1 if on else 0))


SIGC_NARROW, SIGC_PAIR, SIGC_WIDE = 0, 1, 2


def set_sigc_kernel(kind):
    """Split-precision Sigma_c kernel: SIGC_NARROW (one CTA per 64 x 128 tile), SIGC_PAIR
    (CTA pairs over 128-column tiles), SIGC_WIDE (one CTA per 64 x 256 tile, default)."""
    _chk(load().qsgw_set_sigc_kernel(int(kind)))


def get_precision():
    m, n = c_int(), c_int()
    _chk(load().qsgw_get_precision(ctypes.byref(m), ctypes.byref(n)))
    return m.value, n.value


def launch_count():
    return int(load().qsgw_launch_count())


def profile(enable=True):
    """Start (clearing old records) or stop per-kernel event timing."""
    _chk(load().qsgw_profile(int(enable)))


def profile_get(tag):
    """(milliseconds, launches) summed over the recorded launches of ``tag``."""
    ms, n = c_dbl(), ctypes.c_longlong()
    _chk(load().qsgw_profile_get(tag.encode(), ctypes.byref(ms), ctypes.byref(n)))
    return ms.value, n.value


# ---------------------------------------------------------------- BLAS shim
def _alpha(x):
    x = complex(x)
    return (c_dbl * 2)(x.real, x.imag)


def zmm(a, b, c, m, n, k, opa=0, opb=0, alpha=1.0, beta=0.0, lda=None, ldb=None, ldc=None, device=False):
    """m_blas.f90 zmm_h / zmm_d: c = alpha op(a) op(b) + beta c (c updated in place)."""
    lda = lda or (m if opa == 0 else k)
    ldb = ldb or (k if opb == 0 else n)
    ldc = ldc or m
    f = load().qsgw_zmm_d if device else load().qsgw_zmm
    _chk(f(_p(a), _p(b), _p(c), m, n, k, opa, opb, _alpha(alpha), _alpha(beta), lda, ldb, ldc))
    return c


def zminv_hpd_batched_d(a, n, lda, nbatch):
    _chk(load().qsgw_zminv_hpd_batched_d(_p(a), n, lda, nbatch))


def zminv_hpd_batched_noalloc_d(a, n, lda, nbatch, stream=None):
    """Allocation-free batched HPD inverse (static device scratch, n*nbatch <=
    16384); synchronous on ``stream`` (a raw cudaStream_t handle, None = 0)."""
    _chk(load().qsgw_zminv_hpd_batched_noalloc_d(_p(a), n, lda, nbatch, stream))


# ---------------------------------------------------------------- chi0
def x0gemm(rcxq, npr, ipr_col, npr_col, nwhis, npm, ns1, ns2, zmel, nm1,
           icounkmink, icounkmaxk, itc, itpc, jpmc, iwini, iwend, icouini, whwc,
           zmel_shape=None, device=False):
    """x0gemm.f90:2-97.  Host: rcxq (npr, npr_col, nslab) and zmel (nbb, nm,
    nqtot) Fortran-ordered complex128 numpy arrays, rcxq updated in place.
    Device: flat torch tensors holding the same column-major memory, with
    ``zmel_shape = (nbb, nm, nqtot)``."""
    if device:
        nbb, nmz, nqtot = zmel_shape
    else:
        rcxq = _host_c128(rcxq)
        zmel = _host_c128(zmel)
        nbb, nmz, nqtot = zmel.shape
    t = [_i32(itc), _i32(itpc), _i32(jpmc), _i32(iwini), _i32(iwend), _i32(icouini)]
    w = _f64(whwc)
    f = load().qsgw_x0gemm_d if device else load().qsgw_x0gemm
    _chk(f(_p(rcxq), npr, ipr_col, npr_col, nwhis, npm, ns1, ns2, _p(zmel), nbb, nm1, nm1 + nmz - 1,
           nqtot, icounkmink, icounkmaxk, *[_p(x) for x in t], _p(w), len(w)))
    return rcxq


def to_device(a):
    """Flat torch CUDA tensor with the column-major memory of numpy array ``a``."""
    import torch
    return torch.from_numpy(np.asarray(a).reshape(-1, order='F').copy()).cuda()


def from_device(t, shape):
    """Inverse of ``to_device``: Fortran-ordered numpy array of ``shape``."""
    return t.cpu().numpy().reshape(shape, order='F')


def chi0_lorentz_d(chi0, npr, niw, freq_i, nk, nocc, nun, eocc, eunocc, zcols, ldz=None, host=False):
    """All-k chi0 with device-built Lorentzian weights (include/qsgw_b200.h).
    host=True: chi0/zcols are host arrays (numpy, column-major memory)."""
    fi, no, nu = _f64(freq_i), _i32(nocc), _i32(nun)
    eo, eu = _f64(eocc), _f64(eunocc)
    f = load().qsgw_chi0_lorentz if host else load().qsgw_chi0_lorentz_d
    _chk(f(_p(chi0), npr, niw, _p(fi), nk, _p(no), _p(nu), _p(eo), _p(eu), _p(zcols), ldz or npr))
    return chi0


def dpsion_matrix(frhis, freq_i, freq_r=None, ecut=1e10, smearx0=0.0):
    """The Hilbert transform matrix of dpsion_chiq_d on the host (no GPU): complex
    (nwhis+1, niw + nw + 1), chi0 = rcxq . b."""
    fh, fi = _f64(frhis), _f64(freq_i)
    nwhis, niw = len(fh) - 1, len(fi)
    nw = -1 if freq_r is None else len(freq_r) - 1
    fr = _f64(freq_r) if freq_r is not None else np.zeros(1)
    b = np.zeros((nwhis + 1, niw + nw + 1), np.complex128, order='F')
    _chk(load().qsgw_dpsion_matrix(nwhis, _p(fh), niw, _p(fi), nw, _p(fr), ecut, smearx0, _p(b)))
    return b


def dpsion_chiq_d(rcxq, npr, npr_col, nwhis, frhis, freq_i, freq_r=None, ecut=1e10, zxqi=None, zxq=None,
                  smearx0=0.0):
    """Hilbert transform of the chi0 histogram (dpsion5.f90:77-137, 215-292), npm = 1.
    rcxq, zxqi, zxq: device complex128 tensors (zxqi, zxq allocated when None).
    Returns (zxqi, zxq); zxq is None without freq_r."""
    import torch
    fh, fi = _f64(frhis), _f64(freq_i)
    niw = len(fi)
    nw = -1 if freq_r is None else len(freq_r) - 1
    fr = _f64(freq_r) if freq_r is not None else np.zeros(1)
    M = npr * npr_col
    if zxqi is None and niw > 0:
        zxqi = torch.empty(M * niw, dtype=torch.complex128, device=rcxq.device)
    if zxq is None and nw >= 0:
        zxq = torch.empty(M * (nw + 1), dtype=torch.complex128, device=rcxq.device)
    _chk(load().qsgw_dpsion_chiq_d(_p(rcxq), npr, npr_col, nwhis, _p(fh), niw, _p(fi), nw, _p(fr), ecut, smearx0,
                                   _p(zxqi) if zxqi is not None else None, _p(zxq) if zxq is not None else None))
    return zxqi, zxq


# ---------------------------------------------------------------- W
def wvi_llw(zxqi, nspin, vcousq, m2e, is_x0_m_basis, is_wc_m_basis, iq, nblochpmx=None,
            zw=None, device=False, ngb=None, niw=None):
    """m_llw.f90:265-376 (q /= 0 branch): returns zw (nblochpmx, nblochpmx, niw)."""
    v = _f64(vcousq)
    if device:
        assert zw is not None and ngb is not None and niw is not None
        nbl = nblochpmx or ngb
        _chk(load().qsgw_wvi_llw_d(_p(zxqi), ngb, niw, nspin, _p(v), _p(m2e), int(is_x0_m_basis),
                                   int(is_wc_m_basis), iq, _p(zw), nbl))
        return zw
    zxqi = _host_c128(zxqi)
    ngb, _, niw = zxqi.shape
    nbl = nblochpmx or ngb
    if zw is None:
        zw = np.zeros((nbl, nbl, niw), np.complex128, order='F')
    m = None if m2e is None else _host_c128(m2e)
    _chk(load().qsgw_wvi_llw(_p(zxqi), ngb, niw, nspin, _p(v), _p(m), int(is_x0_m_basis),
                             int(is_wc_m_basis), iq, _p(zw), nbl))
    return zw


# ---------------------------------------------------------------- Sigma_c
def _sxcf_args(zsec, zmel, ns1, ns2, ns2r, nwxi, nwx, ntqxx, wc_imag, wc_real,
               omega, ekc, nctot, ef, esmr, wkkr, ua, freqx, wwx, expa, freq_r,
               keepwv=False, nblochpmx=None, device=False, ngb=None, ntq=None):
    """(SxcfArgs, arrays to keep alive, zsec) of one task."""
    tabs = dict(omega=_f64(omega), ekc=_f64(ekc), freqx=_f64(freqx), wwx=_f64(wwx),
                expa=_f64(expa), freq_r=_f64(freq_r))
    if device:
        assert ngb is not None and ntq is not None
    else:
        zsec = _host_c128(zsec); zmel = _host_c128(zmel)
        wc_imag = _host_c128(wc_imag); wc_real = _host_c128(wc_real)
        ngb = zmel.shape[0]; ntq = zsec.shape[0]
    niw = len(tabs['freqx']); nw = len(tabs['freq_r']) - 1
    a = SxcfArgs(ngb=ngb, nblochpmx=nblochpmx or ngb, ns1=ns1, ns2=ns2, ns2r=ns2r, ntqxx=ntqxx,
                 ntq=ntq, niw=niw, nw=nw, nwxi=nwxi, nwx=nwx, nctot=nctot,
                 nekc=len(tabs['ekc']), keepwv=int(keepwv), ef=ef, esmr=esmr, wkkr=wkkr, ua=ua,
                 omega=_p(tabs['omega']), ekc=_p(tabs['ekc']), freqx=_p(tabs['freqx']),
                 wwx=_p(tabs['wwx']), expa=_p(tabs['expa']), freq_r=_p(tabs['freq_r']),
                 zmel=_p(zmel), wc_imag=_p(wc_imag), wc_real=_p(wc_real), zsec=_p(zsec))
    return a, (tabs, zmel, wc_imag, wc_real), zsec


def sxcf_correlation(zsec, zmel, ns1, ns2, ns2r, nwxi, nwx, ntqxx, wc_imag, wc_real,
                     omega, ekc, nctot, ef, esmr, wkkr, ua, freqx, wwx, expa, freq_r,
                     keepwv=False, nblochpmx=None, device=False, ngb=None, ntq=None):
    """get_correlation_block (m_sxcf_gemm.f90:407-612) for one task; zsec updated in place."""
    a, keep, zsec = _sxcf_args(zsec, zmel, ns1, ns2, ns2r, nwxi, nwx, ntqxx, wc_imag, wc_real, omega, ekc, nctot,
                               ef, esmr, wkkr, ua, freqx, wwx, expa, freq_r, keepwv, nblochpmx, device, ngb, ntq)
    f = load().qsgw_sxcf_correlation_d if device else load().qsgw_sxcf_correlation
    _chk(f(ctypes.byref(a)))
    return zsec


def sxcf_correlation_batch_d(tasks):
    """qsgw_sxcf_correlation_batch_d: ``tasks`` is a list of keyword dicts of
    sxcf_correlation (device arrays, ngb and ntq given); the same result as
    calling sxcf_correlation(..., device=True) on each in order."""
    built = [_sxcf_args(**dict(t, device=True)) for t in tasks]
    arr = (SxcfArgs * len(built))()
    for i, (a, _, _) in enumerate(built):
        arr[i] = a
    _chk(load().qsgw_sxcf_correlation_batch_d(arr, len(built)))
    return [z for _, _, z in built]


def sxcf_wgtim_d(out, niw, ns1, ns2, ntqxx, nctot, omega, ekc, esmr, wkkr, ua, freqx, wwx, expa):
    o, e = _f64(omega), _f64(ekc)
    x, w, ex = _f64(freqx), _f64(wwx), _f64(expa)
    _chk(load().qsgw_sxcf_wgtim_d(_p(out), niw, ns1, ns2, ntqxx, nctot, _p(o), _p(e), len(e), esmr,
                                  wkkr, ua, _p(x), _p(w), _p(ex)))
    return out


# ---------------------------------------------------------------- Sigma_x, hqpe, zmel
def sxcf_exchange_d(zsec, ntq, zmel, ngb, ns1, ns2, ntqxx, vcoud, ekc, nctot, ef, esmr, wkkr):
    """sxcf_scz_exchange block (m_sxcf_gemm.f90:203-231); device zsec/zmel."""
    v, e = _f64(vcoud), _f64(ekc)
    _chk(load().qsgw_sxcf_exchange_d(_p(zsec), ntq, _p(zmel), ngb, ns1, ns2, ntqxx, _p(v), _p(e), len(e),
                                     nctot, ef, esmr, wkkr))
    return zsec


def hqpe_d(sex2, sexcore2, sec2, vxc_band_ry, elda_ev, vxc_ev, ntq, ld, nq, eqp_ev, sigma_herm):
    """main_hqpe.sc.f90:150-161,178-180 for nq q-points (all device arrays)."""
    _chk(load().qsgw_hqpe_d(_p(sex2), _p(sexcore2), _p(sec2), _p(vxc_band_ry), _p(elda_ev), _p(vxc_ev), ntq, ld,
                            nq, _p(eqp_ev), _p(sigma_herm)))


def zmel_mt_d(zmelt, nbloch, nm1, nm2, nctot, ntp0, cphim, ldm, cphiq, ldq, atoms):
    """Muffin-tin part of get_zmel_init_gemm; ``atoms`` is a list of dicts with
    the qsgw_zmel_atom fields (ppb_d a device tensor)."""
    arr = (ZmelAtom * len(atoms))()
    keep = []
    for i, a in enumerate(atoms):
        keep.append(a["ppb_d"])
        arr[i] = ZmelAtom(_p(a["ppb_d"]), a["nlnm"], a["nc"], a["nv"], a["ias"], a["ics"], a["ims"], a["mdim"],
                          a["ncore"], float(np.real(a["phase"])), float(np.imag(a["phase"])))
    _chk(load().qsgw_zmel_mt_d(_p(zmelt), nbloch, nm1, nm2, nctot, ntp0, _p(cphim), ldm, _p(cphiq), ldq,
                               len(atoms), arr))
    return zmelt


def zmel_ipw_d(zmelt, ldz, row0, nm1, nm2, nm1v, nm2v, ntp0, geigq, ldgq, dgeigqk, ldgk, ngvecpB1, ngvecpB2,
               ngveccR, nvgcgp2, nvggg, ggg, nadd, phase):
    """Interstitial plane-wave rows of zmelt (m_zmel.f90:418-535).  Integer
    vector tables are (3, n) arrays; ggg, phase complex host arrays."""
    iv = [np.asfortranarray(np.asarray(v, dtype=np.int32)) for v in (ngvecpB1, ngvecpB2, ngveccR, nvgcgp2, nvggg)]
    for v in iv:
        if v.ndim != 2 or v.shape[0] != 3:
            raise ValueError("G-vector tables must be (3, n)")
    g = np.ascontiguousarray(ggg, dtype=np.complex128)
    ph = np.ascontiguousarray(phase, dtype=np.complex128)
    a = ZmelIpwArgs(ngc=iv[2].shape[1], ngp1=iv[0].shape[1], ngp2=iv[1].shape[1], ngcgp=iv[3].shape[1],
                    nggg=iv[4].shape[1], ntp0=ntp0, nm1=nm1, nm2=nm2, nm1v=nm1v, nm2v=nm2v, ldz=ldz, row0=row0,
                    nadd=(c_int * 3)(*[int(x) for x in nadd]), ngvecpB1=iv[0].ctypes.data, ngvecpB2=iv[1].ctypes.data,
                    ngveccR=iv[2].ctypes.data, nvgcgp2=iv[3].ctypes.data, nvggg=iv[4].ctypes.data,
                    ggg=g.ctypes.data, phase=ph.ctypes.data, geigq_d=_p(geigq), ldgq=ldgq, dgeigqk_d=_p(dgeigqk),
                    ldgk=ldgk, zmelt_d=_p(zmelt))
    _chk(load().qsgw_zmel_ipw_d(ctypes.byref(a)))
    return zmelt


def zmel_m2e_d(zmel, zmelt, ngb, nbb, nmtot, nqtot, m2e, is_m_basis, zmelconjg):
    _chk(load().qsgw_zmel_m2e_d(_p(zmel), _p(zmelt), ngb, nbb, nmtot, nqtot, _p(m2e), int(is_m_basis),
                                int(zmelconjg)))
    return zmel


def zhegv_d(v, n, lda=None, o=None):
    """Coulomb eigenproblem: v (device, Hermitian) -> eigenvectors in place;
    returns vcoud (descending eigenvalues of v, O-orthonormal vectors)."""
    out = np.zeros(n)
    _chk(load().qsgw_zhegv_d(_p(v), _p(o), n, lda or n, out.ctypes.data))
    return out


# ---------------------------------------------------------------- autotuner
def set_autotune(mode=1, cache_path=None):
    _chk(load().qsgw_set_autotune(mode, None if cache_path is None else os.fsencode(cache_path)))


def autotune_report():
    """The tuned choices, {shape key: value}."""
    import json
    buf = ctypes.create_string_buffer(1 << 16)
    _chk(load().qsgw_autotune_report(buf, len(buf)))
    return json.loads(buf.value.decode())


# ---------------------------------------------------------------- CUDA graph of a call sequence
def graph_begin():
    _chk(load().qsgw_graph_begin())


def graph_end():
    _chk(load().qsgw_graph_end())


def graph_launch():
    _chk(load().qsgw_graph_launch())


def graph_destroy():
    _chk(load().qsgw_graph_destroy())


def chi0_lorentz_acc_d(chi0, npr, niw, freq_i, nk_total, nocc, nun, eocc, eunocc, zcols, ldz=None):
    """chi0 += the contribution of one batch of k-points (len(nocc) of them)."""
    fi, no, nu = _f64(freq_i), _i32(nocc), _i32(nun)
    eo, eu = _f64(eocc), _f64(eunocc)
    _chk(load().qsgw_chi0_lorentz_acc_d(_p(chi0), npr, niw, _p(fi), nk_total, len(no), _p(no), _p(nu), _p(eo),
                                        _p(eu), _p(zcols), ldz or npr))
    return chi0


# ---------------------------------------------------------------- real frequency axis
def chi0_lorentz_real_d(chi0, npr, nw, freq_r, eta, nk, nocc, nun, eocc, eunocc, zcols, ldz=None):
    fr, no, nu = _f64(freq_r), _i32(nocc), _i32(nun)
    eo, eu = _f64(eocc), _f64(eunocc)
    _chk(load().qsgw_chi0_lorentz_real_d(_p(chi0), npr, nw, _p(fr), float(eta), nk, _p(no), _p(nu), _p(eo), _p(eu),
                                         _p(zcols), ldz or npr))
    return chi0


def wvr_llw_d(zxq, ngb, nw, nspin, vcousq, m2e, is_x0_m_basis, is_wc_m_basis, iq, zw, nblochpmx=None):
    """m_llw.f90:49-264: W - v on real frequencies (device arrays)."""
    v = _f64(vcousq)
    _chk(load().qsgw_wvr_llw_d(_p(zxq), ngb, nw, nspin, _p(v), _p(m2e), int(is_x0_m_basis), int(is_wc_m_basis), iq,
                               _p(zw), nblochpmx or ngb))
    return zw


def zminv_batched_d(a, n, lda, nbatch):
    _chk(load().qsgw_zminv_batched_d(_p(a), n, lda, nbatch))


# ---------------------------------------------------------------- tetrahedron weights
def x0_lists(w):
    """x0gemm pair/bin lists from dense histogram weights w (nk, nocc, nunocc, nwhis), numpy, the
    layout of tetwt_hist_d's output (x0kf_v4h.f90:48-142, npm = 1).  Returns a dict of the 1-based
    tables itc, itpc, jpmc, iwini, iwend, icouini, whwc, icounkmin, icounkmax (host, no GPU needed)."""
    w = np.ascontiguousarray(np.asarray(w, dtype=np.float64))
    nk, nocc, nunocc, nwhis = w.shape
    nc, nt = ctypes.c_int(0), ctypes.c_int(0)
    f = load().qsgw_x0_lists
    _chk(f(_p(w), nk, nocc, nunocc, nwhis, 0, ctypes.byref(nc), ctypes.byref(nt), *([None] * 9)))
    t = {k: np.zeros(max(nc.value, 1), np.int32) for k in ("itc", "itpc", "jpmc", "iwini", "iwend", "icouini")}
    t["whwc"] = np.zeros(max(nt.value, 1))
    t["icounkmin"] = np.zeros(nk, np.int32)
    t["icounkmax"] = np.zeros(nk, np.int32)
    _chk(f(_p(w), nk, nocc, nunocc, nwhis, 1, ctypes.byref(nc), ctypes.byref(nt), _p(t["itc"]), _p(t["itpc"]),
           _p(t["jpmc"]), _p(t["iwini"]), _p(t["iwend"]), _p(t["icouini"]), _p(t["whwc"]), _p(t["icounkmin"]),
           _p(t["icounkmax"])))
    t["ncoun"], t["ncount"] = nc.value, nt.value
    return t


def tetwt_symmetrize(w, ek, ekq):
    """In place on the host weights w (nk, nocc, nunocc, nwhis) (numpy, the layout of tetwt_hist_d's
    output): the degenerate-band symmetrisation of tetwt5.f90:347-423; ek, ekq (nk, nband) in Ry."""
    if not (isinstance(w, np.ndarray) and w.dtype == np.float64 and w.flags.c_contiguous and w.ndim == 4):
        raise ValueError("w must be a C-contiguous float64 array (nk, nocc, nunocc, nwhis)")
    a = np.ascontiguousarray(np.asarray(ek, dtype=np.float64))
    b = np.ascontiguousarray(np.asarray(ekq, dtype=np.float64))
    nk, nocc, nunocc, nwhis = w.shape
    if a.shape != b.shape or a.shape[0] != nk:
        raise ValueError(f"ek {a.shape} / ekq {b.shape} must both be (nk={nk}, nband)")
    _chk(load().qsgw_tetwt_symmetrize(_p(w), nk, nocc, nunocc, nwhis, _p(a), _p(b), a.shape[1]))
    return w


def tetwt_hist_d(w, idtet, qbzw, ek, ekq, efermi, frhis, nocc, nunocc):
    """w (device, nwhis x nunocc x nocc x nk, accumulated) += tetrahedron
    histogram weights; idtet (ntet, 4) 0-based, qbzw (nk, 3), ek/ekq (nk, nband).
    Returns the total tetrahedron volume."""
    it = np.ascontiguousarray(np.asarray(idtet, dtype=np.int32))
    q = np.ascontiguousarray(np.asarray(qbzw, dtype=np.float64))
    a = np.ascontiguousarray(np.asarray(ek, dtype=np.float64))       # (nk, nband) C order = (nband, nk) F order
    b = np.ascontiguousarray(np.asarray(ekq, dtype=np.float64))
    fr = _f64(frhis)
    vt = ctypes.c_double(0.0)
    _chk(load().qsgw_tetwt_hist_d(_p(w), a.shape[0], nocc, nunocc, len(fr) - 1, it.ctypes.data, it.shape[0],
                                  q.ctypes.data, a.ctypes.data, b.ctypes.data, a.shape[1], float(efermi),
                                  fr.ctypes.data, ctypes.byref(vt)))
    return vt.value


# ---------------------------------------------------------------- W record files
def wv_write_d(path, zw, nblochpmx, rec0, nrec, kind4=False):
    """Write records rec0.. of a __WVI/__WVR file from a device W stack."""
    _chk(load().qsgw_wv_write_d(os.fsencode(path), _p(zw), nblochpmx, rec0, nrec, int(kind4)))


def wv_read_d(path, out, nblochpmx, rec0, nrec, kind4=False, pack=0, ngb=0):
    """Read records into a device buffer: full (pack 0), upper triangle (1) or
    upper triangle of (W + W^H)/2 (2) of the leading ngb x ngb block."""
    _chk(load().qsgw_wv_read_d(os.fsencode(path), _p(out), nblochpmx, rec0, nrec, int(kind4), pack, ngb))
    return out


# ---------------------------------------------------------------- sequential unformatted files (host)
def vcoud_write(path, q, vcoud, zcousq):
    """__Vcoud.<iq>: ngb | q(3) | vcoud(ngb) | zcousq(ngb, ngb) (main_hvccfp0.f90:396-400)."""
    v = _f64(vcoud)
    z = np.asfortranarray(np.asarray(zcousq, dtype=np.complex128))
    n = v.size
    if z.shape != (n, n):
        raise ValueError(f"zcousq must be ({n}, {n}), got {z.shape}")
    _chk(load().qsgw_vcoud_write(os.fsencode(path), n, _p(_f64(q)), _p(v), _p(z)))


def vcoud_read(path):
    """Readvcoud (m_readVcoud.f90:30-40): returns q, vcoud, vcousq, zcousq (Fortran order)."""
    f = load().qsgw_vcoud_read
    n = ctypes.c_int(0)
    q = np.zeros(3)
    _chk(f(os.fsencode(path), 0, ctypes.byref(n), _p(q), None, None, None))
    v, vs = np.zeros(n.value), np.zeros(n.value)
    z = np.zeros((n.value, n.value), np.complex128, order='F')
    _chk(f(os.fsencode(path), n.value, ctypes.byref(n), _p(q), _p(v), _p(vs), _p(z)))
    return q, v, vs, z


def sigma_write(path, head, is_, qibz, zsec):
    """SEX2U / SEXcore2U / SEC2U: head (nspin, nq, ntq, nqbz, nqibz, n1, n2, n3), qibz (3, nq),
    zsec (ntq, ntq, nq) complex (main_hsfp0.sc.f90:322, 333, 340, 359)."""
    h = np.ascontiguousarray(np.asarray(head, dtype=np.int32))
    if h.size != 8:
        raise ValueError("head holds 8 integers")
    nq, ntq = int(h[1]), int(h[2])
    q = np.asfortranarray(np.asarray(qibz, dtype=np.float64))
    z = np.asfortranarray(np.asarray(zsec, dtype=np.complex128))
    if q.shape != (3, nq) or z.shape != (ntq, ntq, nq):
        raise ValueError(f"qibz {q.shape} / zsec {z.shape} do not match nq={nq} ntq={ntq}")
    _chk(load().qsgw_sigma_write(os.fsencode(path), _p(h), is_, _p(q), _p(z)))


def sigma_read(path):
    """Returns head, isx (nq), qibz (3, nq), zsec (ntq, ntq, nq) (main_hqpe.sc.f90:132-148)."""
    f = load().qsgw_sigma_read
    h = np.zeros(8, np.int32)
    _chk(f(os.fsencode(path), _p(h), 0, 0, None, None, None))
    nq, ntq = int(h[1]), int(h[2])
    isx = np.zeros(max(nq, 1), np.int32)
    q = np.zeros((3, max(nq, 1)), order='F')
    z = np.zeros((max(ntq, 1), max(ntq, 1), max(nq, 1)), np.complex128, order='F')
    _chk(f(os.fsencode(path), _p(h), nq, ntq, _p(isx), _p(q), _p(z)))
    return h, isx[:nq], q[:, :nq], z[:, :, :nq]


# ---------------------------------------------------------------- W_c frequency surrogate
def _f32(a):
    return np.ascontiguousarray(np.asarray(a, dtype=np.float32))


def wsurr_init(seed=1234):
    _chk(load().qsgw_wsurr_init(seed))


def wsurr_nparam():
    return load().qsgw_wsurr_nparam()


def wsurr_params(values=None):
    """Read (values None) or write the FP32 parameter vector."""
    n = wsurr_nparam()
    if values is None:
        out = np.zeros(n, np.float32)
        _chk(load().qsgw_wsurr_params(out.ctypes.data, 0))
        return out
    v = _f32(values)
    if v.size != n:
        raise ValueError(f"expected {n} parameters, got {v.size}")
    _chk(load().qsgw_wsurr_params(v.ctypes.data, 1))


def wsurr_project_d(wc, ld, nslot, ridx, proj, cidx=None):
    r = _i32(ridx)
    c = None if cidx is None else _i32(cidx)
    if c is not None and len(c) != len(r):
        raise ValueError("ridx and cidx differ in length")
    _chk(load().qsgw_wsurr_project_d(_p(wc), ld, nslot, r.ctypes.data, None if c is None else c.ctypes.data, len(r),
                                     _p(proj)))


def wsurr_lsq_accumulate_d(x, y, wgt, n, thead):
    h = _i32(thead)
    _chk(load().qsgw_wsurr_lsq_accumulate_d(_p(x), _p(y), _p(wgt), n, len(h), h.ctypes.data))


def wsurr_lsq_solve(ridge=1e-9):
    """Solve the accumulated normal equations into the head rows; returns the rows solved."""
    k = ctypes.c_int(0)
    _chk(load().qsgw_wsurr_lsq_solve(ridge, ctypes.byref(k)))
    return k.value


def wsurr_features_d(proj, nq, nw, ne, anchors, targets, thead, xcoord, x, tix, y=None, wgt=None, scale=None,
                     rid=None, cid=None, ftab=None):
    a, t, h, xc = _i32(anchors), _i32(targets), _i32(thead), _f32(xcoord)
    if len(h) != len(t) or len(xc) != nw:
        raise ValueError("thead must match targets and xcoord must have nw entries")
    if ftab is None:
        r = c = f = None
        nb = nf = 0
    else:
        r, c, f = _i32(rid), _i32(cid), _f32(ftab)
        nb, nf = len(r), len(f)
        if len(c) != nb:
            raise ValueError("rid and cid differ in length")
    _chk(load().qsgw_wsurr_features_d(_p(proj), nq, nw, ne, a.ctypes.data, len(a), t.ctypes.data, h.ctypes.data,
                                      len(t), xc.ctypes.data, _p(r), _p(c), nb, _p(f), nf, _p(x), _p(tix), _p(y),
                                      _p(wgt), _p(scale)))


def wsurr_forward_d(x, tix, y, batch):
    _chk(load().qsgw_wsurr_forward_d(_p(x), _p(tix), _p(y), batch))


def wsurr_grad_d(x, tix, y, batch, wgt=None):
    """Returns (loss, gradient) without updating the parameters."""
    loss = np.zeros(1, np.float32)
    grad = np.zeros(wsurr_nparam(), np.float32)
    _chk(load().qsgw_wsurr_grad_d(_p(x), _p(tix), _p(y), _p(wgt), batch, loss.ctypes.data, grad.ctypes.data))
    return float(loss[0]), grad


def wsurr_train_d(x, tix, y, wgt, n, batch, nsteps, lr, seed=0):
    """nsteps Adam steps; returns the last mini-batch's loss."""
    loss = np.zeros(1, np.float32)
    _chk(load().qsgw_wsurr_train_d(_p(x), _p(tix), _p(y), _p(wgt), n, batch, nsteps, lr, seed, loss.ctypes.data))
    return float(loss[0])


def wsurr_head_full_d(wc, n, ld, nslot, aslot, tslot, thead, txc, ftab=None):
    a, t, h, x = _i32(aslot), _i32(tslot), _i32(thead), _f32(txc)
    f = None if ftab is None else _f32(ftab)
    if f is not None and len(f) != n:
        raise ValueError("ftab must have n entries")
    _chk(load().qsgw_wsurr_head_full_d(_p(wc), n, ld, nslot, a.ctypes.data, len(a), t.ctypes.data, h.ctypes.data,
                                       x.ctypes.data, len(t), _p(f)))


def wsurr_scatter_d(wc, ld, nslot, idx, tslot, pred, scale):
    i, t = _i32(idx), _i32(tslot)
    if pred.numel() < 2 * len(i) ** 2 * len(t) or scale.numel() < pred.numel():
        raise ValueError("pred/scale hold fewer than 2 nb^2 nt samples")
    _chk(load().qsgw_wsurr_scatter_d(_p(wc), ld, nslot, i.ctypes.data, len(i), t.ctypes.data, len(t), _p(pred),
                                     _p(scale)))
