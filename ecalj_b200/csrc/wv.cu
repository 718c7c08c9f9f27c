// W - v on the imaginary axis (WVIllwI, m_llw.f90:265-376) and the batched
// inverse of the Hermitian positive definite eps~ (stands in for zminv_d,
// m_lapack.f90:108-176).
//
// Inverse: blocked Gauss-Jordan exchange without pivoting (valid because
// eps~ = 1 - v^1/2 chi0 v^1/2 >= 1 on the imaginary axis).  Per block column
// p of width nb:
//     [[P, Q], [R, S]]  ->  [[P^-1, -P^-1 Q], [R P^-1, S - R P^-1 Q]]
// which after all blocks leaves A^-1.  Each step is one small kernel that
// inverts P in shared memory and writes the two panels
//     Rb = [R P^-1 ; I + P^-1]   (n x nb),   Qb = [Q  with  P - I in block p]
// followed by ONE rank-nb update A <- A - Rb Qb on the DMMA engine, which
// produces all four blocks of the exchange at once.
#include "zgemm_f64.cuh"

namespace qsgw {

constexpr int GJ_NB = 32;

__global__ void gj_panel_kernel(double2* __restrict__ A, int n, long long lda, long long a_bs,
                                double2* __restrict__ Rb, double2* __restrict__ Qb, int c0, int w,
                                int* __restrict__ flag) {
  __shared__ double2 P[GJ_NB][GJ_NB + 1];
  const int b = blockIdx.y;
  double2* Ab = A + b * a_bs;
  double2* Rbb = Rb + static_cast<long long>(b) * n * GJ_NB;
  double2* Qbb = Qb + static_cast<long long>(b) * n * GJ_NB;
  const int tid = threadIdx.x;
  for (int e = tid; e < GJ_NB * GJ_NB; e += blockDim.x) {
    const int i = e % GJ_NB, j = e / GJ_NB;
    P[i][j] = (i < w && j < w) ? Ab[(c0 + i) + (c0 + j) * lda] : make_double2(0.0, 0.0);
  }
  __syncthreads();
  // in-place exchange inverse of the w x w pivot block
  bool bad = false;
  for (int k = 0; k < w; ++k) {
    const double2 pk = P[k][k];
    const double den = pk.x * pk.x + pk.y * pk.y;
    if (!(den > 1e-300) || !isfinite(den)) bad = true;
    const double2 inv = make_double2(pk.x / den, -pk.y / den);
    double2 nv[GJ_NB * GJ_NB / 128];
    int cnt = 0;
    for (int e = tid; e < w * w; e += blockDim.x, ++cnt) {
      const int i = e % w, j = e / w;
      double2 r;
      if (i == k && j == k) {
        r = inv;
      } else if (i == k) {            // -P_kj / P_kk
        const double2 a = P[k][j];
        r = make_double2(-(a.x * inv.x - a.y * inv.y), -(a.x * inv.y + a.y * inv.x));
      } else if (j == k) {            //  P_ik / P_kk
        const double2 a = P[i][k];
        r = make_double2(a.x * inv.x - a.y * inv.y, a.x * inv.y + a.y * inv.x);
      } else {                        //  P_ij - P_ik P_kj / P_kk
        const double2 a = P[i][k], c = P[k][j];
        const double2 t = make_double2(a.x * inv.x - a.y * inv.y, a.x * inv.y + a.y * inv.x);
        const double2 o = P[i][j];
        r = make_double2(o.x - (t.x * c.x - t.y * c.y), o.y - (t.x * c.y + t.y * c.x));
      }
      nv[cnt] = r;
    }
    __syncthreads();
    cnt = 0;
    for (int e = tid; e < w * w; e += blockDim.x, ++cnt) P[e % w][e / w] = nv[cnt];
    __syncthreads();
  }
  if (bad && tid == 0) atomicExch(flag, 1);
  // Rb rows of this CTA's row block
  const int r0 = blockIdx.x * 64;
  for (int e = tid; e < 64 * GJ_NB; e += blockDim.x) {
    const int ii = e % 64, j = e / 64;
    const int row = r0 + ii;
    if (row >= n || j >= w) continue;
    double2 acc;
    if (row >= c0 && row < c0 + w) {
      acc = P[row - c0][j];
      if (row - c0 == j) acc.x += 1.0;
    } else {
      acc = make_double2(0.0, 0.0);
      for (int l = 0; l < w; ++l) {
        const double2 a = Ab[row + (c0 + l) * lda];
        const double2 c = P[l][j];
        acc.x += a.x * c.x - a.y * c.y;
        acc.y += a.x * c.y + a.y * c.x;
      }
    }
    Rbb[row + static_cast<long long>(j) * n] = acc;
  }
  // Qb columns of the same index range
  for (int e = tid; e < 64 * GJ_NB; e += blockDim.x) {
    const int l = e % GJ_NB, jj = e / GJ_NB;
    const int col = r0 + jj;
    if (col >= n || l >= w) continue;
    double2 v = Ab[(c0 + l) + static_cast<long long>(col) * lda];
    if (col - c0 == l) v.x -= 1.0;
    Qbb[l + static_cast<long long>(col) * GJ_NB] = v;
  }
}

static DevBuf g_gj_r, g_gj_q;

int zminv_hpd_batched(double2* A, int n, long long lda, long long a_bs, int nbatch, cudaStream_t s) {
  if (n <= 0 || nbatch <= 0) return QSGW_OK;
  const size_t pbytes = static_cast<size_t>(n) * GJ_NB * nbatch * sizeof(double2);
  int rc = g_gj_r.ensure(pbytes);
  if (rc) return rc;
  rc = g_gj_q.ensure(pbytes);
  if (rc) return rc;
  const dim3 pg((n + 63) / 64, nbatch);
  QSGW_CUDA(cudaMemsetAsync(ctx().d_flags, 0, sizeof(int), s));
  for (int c0 = 0; c0 < n; c0 += GJ_NB) {
    const int w = std::min(GJ_NB, n - c0);
    gj_panel_kernel<<<pg, 256, 0, s>>>(A, n, lda, a_bs, g_gj_r.as<double2>(), g_gj_q.as<double2>(),
                                       c0, w, ctx().d_flags);
    count_launch();
    QSGW_LAUNCH_CHECK("gj_panel_kernel");
    rc = zgemm_f64(0, 0, n, n, w, make_double2(-1.0, 0.0), g_gj_r.as<double2>(), n,
                   static_cast<long long>(n) * GJ_NB, g_gj_q.as<double2>(), GJ_NB,
                   static_cast<long long>(n) * GJ_NB, make_double2(1.0, 0.0), A, lda, a_bs, nbatch, s);
    if (rc) return rc;
  }
  return QSGW_OK;
}

// Same blocked Gauss-Jordan with caller-provided panel scratch (rb, qb: each
// n*32*nbatch complex) and status word; allocates nothing.
int zminv_hpd_batched_explicit(double2* A, int n, long long lda, long long a_bs, int nbatch, double2* rb,
                               double2* qb, int* flag, cudaStream_t s) {
  if (n <= 0 || nbatch <= 0) return QSGW_OK;
  const dim3 pg((n + 63) / 64, nbatch);
  for (int c0 = 0; c0 < n; c0 += GJ_NB) {
    const int w = std::min(GJ_NB, n - c0);
    gj_panel_kernel<<<pg, 256, 0, s>>>(A, n, lda, a_bs, rb, qb, c0, w, flag);
    count_launch();
    QSGW_LAUNCH_CHECK("gj_panel_kernel");
    int rc = zgemm_f64(0, 0, n, n, w, make_double2(-1.0, 0.0), rb, n, static_cast<long long>(n) * GJ_NB, qb,
                       GJ_NB, static_cast<long long>(n) * GJ_NB, make_double2(1.0, 0.0), A, lda, a_bs, nbatch, s);
    if (rc) return rc;
  }
  return QSGW_OK;
}

// eps~(i,j) = delta_ij - v_i chi(i,j) v_j on the (ngb-ix) x (ngb-ix) block (m_llw.f90:341-348)
__global__ void eps_build_kernel(double2* __restrict__ eps, const double2* __restrict__ chi,
                                 const double* __restrict__ v, int ngb, int ix, long long ldchi,
                                 long long chi_bs, int niw) {
  const int n = ngb - ix;
  const long long tot = static_cast<long long>(n) * n * niw;
  for (long long e = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; e < tot;
       e += static_cast<long long>(gridDim.x) * blockDim.x) {
    const int i = static_cast<int>(e % n);
    const long long r = e / n;
    const int j = static_cast<int>(r % n);
    const int iw = static_cast<int>(r / n);
    const double2 c = chi[iw * chi_bs + (i + ix) + (j + ix) * ldchi];
    const double f = v[i + ix] * v[j + ix];
    double2 o = make_double2(-f * c.x, -f * c.y);
    if (i == j) o.x += 1.0;
    eps[e] = o;
  }
}

// zw(i,j) = v_i einv v_j - delta_ij v_i v_j inside [ix, ngb), zero elsewhere (:353-360)
__global__ void wc_build_kernel(double2* __restrict__ zw, const double2* __restrict__ einv,
                                const double* __restrict__ v, int ngb, int ix, int ldzw, int niw) {
  const int n = ngb - ix;
  const long long tot = static_cast<long long>(ldzw) * ldzw * niw;
  for (long long e = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; e < tot;
       e += static_cast<long long>(gridDim.x) * blockDim.x) {
    const int i = static_cast<int>(e % ldzw);
    const long long r = e / ldzw;
    const int j = static_cast<int>(r % ldzw);
    const int iw = static_cast<int>(r / ldzw);
    double2 o = make_double2(0.0, 0.0);
    if (i >= ix && i < ngb && j >= ix && j < ngb) {
      const double2 a = einv[static_cast<long long>(iw) * n * n + (i - ix) + static_cast<long long>(j - ix) * n];
      const double f = v[i] * v[j];
      o = make_double2(f * a.x, f * a.y);
      if (i == j) o.x -= f;
    }
    zw[e] = o;
  }
}

__global__ void zscale_real_kernel(double2* a, long long n, double f) {
  for (long long e = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; e < n;
       e += static_cast<long long>(gridDim.x) * blockDim.x) {
    double2 v = a[e];
    v.x *= f; v.y *= f;
    a[e] = v;
  }
}

static DevBuf g_wv_v, g_wv_e, g_wv_x, g_wv_chi, g_wv_m2e, g_wv_zw;

static int grid_for(long long n) {
  return static_cast<int>(std::max<long long>(1, std::min<long long>((n + 255) / 256, 16LL * ctx().sm_count)));
}

// general = false: imaginary axis, eps~ Hermitian positive definite (WVIllwI);
// general = true: real axis, eps~ general, inverted with partial pivoting (WVRllwR,
// m_llw.f90:49-264, the same per-frequency block :125-170).
static int wvi_device(double2* zxqi, int ngb, int niw, int nspin, const double* vcousq,
                      const double2* m2e, int is_x0_m, int is_wc_m, int iq, double2* zw, int ldzw,
                      bool general = false) {
  cudaStream_t s = ctx().stream;
  const long long nn = static_cast<long long>(ngb) * ngb;
  int rc = g_wv_v.ensure(ngb * sizeof(double));
  if (rc) return rc;
  if ((rc = h2d(g_wv_v.p, vcousq, ngb * sizeof(double), s))) return rc;
  if (nspin == 1) {   // zxqi = 2 zxqi in place (m_llw.f90:299-303)
    zscale_real_kernel<<<grid_for(nn * niw), 256, 0, s>>>(zxqi, nn * niw, 2.0);
    count_launch();
    QSGW_LAUNCH_CHECK("zscale_real_kernel");
  }
  const double2* chi = zxqi;
  if (is_x0_m) {      // chi_E = m2e^H chi m2e (:333-340)
    rc = g_wv_x.ensure(nn * niw * sizeof(double2));
    if (rc) return rc;
    rc = g_wv_chi.ensure(nn * niw * sizeof(double2));
    if (rc) return rc;
    rc = zgemm_f64(0, 0, ngb, ngb, ngb, make_double2(1, 0), zxqi, ngb, nn, m2e, ngb, 0,
                   make_double2(0, 0), g_wv_x.as<double2>(), ngb, nn, niw, s);
    if (rc) return rc;
    rc = zgemm_f64(2, 0, ngb, ngb, ngb, make_double2(1, 0), m2e, ngb, 0, g_wv_x.as<double2>(), ngb, nn,
                   make_double2(0, 0), g_wv_chi.as<double2>(), ngb, nn, niw, s);
    if (rc) return rc;
    chi = g_wv_chi.as<double2>();
  }
  const int ix = (iq == 1) ? 1 : 0;
  const int n = ngb - ix;
  const long long en = static_cast<long long>(n) * n;
  rc = g_wv_e.ensure(std::max<long long>(en, 1) * niw * sizeof(double2));
  if (rc) return rc;
  if (n > 0) {
    eps_build_kernel<<<grid_for(en * niw), 256, 0, s>>>(g_wv_e.as<double2>(), chi, g_wv_v.as<double>(),
                                                        ngb, ix, ngb, nn, niw);
    count_launch();
    QSGW_LAUNCH_CHECK("eps_build_kernel");
    rc = general ? zminv_general_batched(g_wv_e.as<double2>(), n, n, en, niw, s)    // :139
                 : zminv_hpd_batched(g_wv_e.as<double2>(), n, n, en, niw, s);       // :350
    if (rc) return rc;
  }
  wc_build_kernel<<<grid_for(static_cast<long long>(ldzw) * ldzw * niw), 256, 0, s>>>(
      zw, g_wv_e.as<double2>(), g_wv_v.as<double>(), ngb, ix, ldzw, niw);
  count_launch();
  QSGW_LAUNCH_CHECK("wc_build_kernel");
  if (is_wc_m && iq != 1) {   // W_M = m2e W_E m2e^H (:363-370)
    const long long zs = static_cast<long long>(ldzw) * ldzw;
    rc = g_wv_x.ensure(nn * niw * sizeof(double2));
    if (rc) return rc;
    rc = zgemm_f64(0, 2, ngb, ngb, ngb, make_double2(1, 0), zw, ldzw, zs, m2e, ngb, 0,
                   make_double2(0, 0), g_wv_x.as<double2>(), ngb, nn, niw, s);
    if (rc) return rc;
    rc = zgemm_f64(0, 0, ngb, ngb, ngb, make_double2(1, 0), m2e, ngb, 0, g_wv_x.as<double2>(), ngb, nn,
                   make_double2(0, 0), zw, ldzw, zs, niw, s);
    if (rc) return rc;
  }
  return QSGW_OK;
}

static int wvi_check(int ngb, int niw, int nspin, int iq, int ldzw, const void* zxqi, const void* zw,
                     const void* v) {
  QSGW_ARG(ngb >= 1 && niw >= 1, "wvi_llw: ngb=%d niw=%d", ngb, niw);
  QSGW_ARG(nspin == 1 || nspin == 2, "wvi_llw: nspin=%d", nspin);
  QSGW_ARG(iq >= 1, "wvi_llw: iq=%d (1-based)", iq);
  QSGW_ARG(ldzw >= ngb, "wvi_llw: nblochpmx=%d < ngb=%d", ldzw, ngb);
  QSGW_ARG(zxqi && zw && v, "wvi_llw: null pointer");
  QSGW_ARG((reinterpret_cast<uintptr_t>(zxqi) & 15) == 0 && (reinterpret_cast<uintptr_t>(zw) & 15) == 0,
           "wvi_llw: complex arrays must be 16-byte aligned");
  return QSGW_OK;
}

}  // namespace qsgw

using namespace qsgw;

extern "C" int qsgw_zminv_hpd_batched_d(double* a, int n, int lda, int nbatch) {
  int rc = require_init();
  if (rc) return rc;
  QSGW_ARG(a && n >= 0 && lda >= std::max(1, n) && nbatch >= 0, "zminv_hpd: n=%d lda=%d nbatch=%d", n, lda, nbatch);
  QSGW_ARG((reinterpret_cast<uintptr_t>(a) & 15) == 0, "zminv_hpd: array must be 16-byte aligned");
  return zminv_hpd_batched(reinterpret_cast<double2*>(a), n, lda, static_cast<long long>(lda) * n, nbatch,
                           ctx().stream);
}

extern "C" int qsgw_wvi_llw_d(double* zxqi_d, int ngb, int niw, int nspin, const double* vcousq,
                              const double* m2e_d, int is_x0_m_basis, int is_wc_m_basis, int iq,
                              double* zw_d, int nblochpmx) {
  int rc = require_init();
  if (rc) return rc;
  rc = wvi_check(ngb, niw, nspin, iq, nblochpmx, zxqi_d, zw_d, vcousq);
  if (rc) return rc;
  QSGW_ARG(!(is_x0_m_basis || is_wc_m_basis) || m2e_d, "wvi_llw: m2e required for basis changes");
  return wvi_device(reinterpret_cast<double2*>(zxqi_d), ngb, niw, nspin, vcousq,
                    reinterpret_cast<const double2*>(m2e_d), is_x0_m_basis, is_wc_m_basis, iq,
                    reinterpret_cast<double2*>(zw_d), nblochpmx);
}

extern "C" int qsgw_wvr_llw_d(double* zxq_d, int ngb, int nw, int nspin, const double* vcousq,
                              const double* m2e_d, int is_x0_m_basis, int is_wc_m_basis, int iq,
                              double* zw_d, int nblochpmx) {
  int rc = require_init();
  if (rc) return rc;
  rc = wvi_check(ngb, nw, nspin, iq, nblochpmx, zxq_d, zw_d, vcousq);
  if (rc) return rc;
  QSGW_ARG(!(is_x0_m_basis || is_wc_m_basis) || m2e_d, "wvr_llw: m2e required for basis changes");
  return wvi_device(reinterpret_cast<double2*>(zxq_d), ngb, nw, nspin, vcousq,
                    reinterpret_cast<const double2*>(m2e_d), is_x0_m_basis, is_wc_m_basis, iq,
                    reinterpret_cast<double2*>(zw_d), nblochpmx, true);
}

extern "C" int qsgw_wvi_llw(double* zxqi, int ngb, int niw, int nspin, const double* vcousq,
                            const double* m2e, int is_x0_m_basis, int is_wc_m_basis, int iq, double* zw,
                            int nblochpmx) {
  int rc = require_init();
  if (rc) return rc;
  rc = wvi_check(ngb, niw, nspin, iq, nblochpmx, zxqi, zw, vcousq);
  if (rc) return rc;
  const bool need_m2e = is_x0_m_basis || (is_wc_m_basis && iq != 1);
  QSGW_ARG(!need_m2e || m2e, "wvi_llw: m2e required for basis changes");
  cudaStream_t s = ctx().stream;
  const size_t cb = static_cast<size_t>(ngb) * ngb * niw * 16;
  const size_t zb = static_cast<size_t>(nblochpmx) * nblochpmx * niw * 16;
  rc = g_wv_zw.ensure(cb + zb);
  if (rc) return rc;
  double2* dchi = g_wv_zw.as<double2>();
  double2* dzw = dchi + static_cast<size_t>(ngb) * ngb * niw;
  QSGW_CUDA(cudaMemcpyAsync(dchi, zxqi, cb, cudaMemcpyHostToDevice, s));
  if (need_m2e) {
    rc = g_wv_m2e.ensure(static_cast<size_t>(ngb) * ngb * 16);
    if (rc) return rc;
    QSGW_CUDA(cudaMemcpyAsync(g_wv_m2e.p, m2e, static_cast<size_t>(ngb) * ngb * 16, cudaMemcpyHostToDevice, s));
  }
  QSGW_CUDA(cudaMemsetAsync(ctx().d_flags, 0, sizeof(int), s));
  rc = wvi_device(dchi, ngb, niw, nspin, vcousq, need_m2e ? g_wv_m2e.as<double2>() : nullptr,
                  is_x0_m_basis, is_wc_m_basis, iq, dzw, nblochpmx);
  if (rc) return rc;
  QSGW_CUDA(cudaMemcpyAsync(zw, dzw, zb, cudaMemcpyDeviceToHost, s));
  if (nspin == 1) QSGW_CUDA(cudaMemcpyAsync(zxqi, dchi, cb, cudaMemcpyDeviceToHost, s));
  int flag = 0;
  QSGW_CUDA(cudaMemcpyAsync(&flag, ctx().d_flags, sizeof(int), cudaMemcpyDeviceToHost, s));
  QSGW_CUDA(cudaStreamSynchronize(s));
  if (flag) {
    QSGW_CUDA(cudaMemset(ctx().d_flags, 0, sizeof(int)));   // reported here, not again by qsgw_synchronize
    set_error("wvi_llw: eps~ is not positive definite (singular pivot block)");
    return QSGW_ERR_NUMERIC;
  }
  return QSGW_OK;
}
