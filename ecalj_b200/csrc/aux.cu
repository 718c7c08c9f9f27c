// Smaller FP64 steps around the Sigma_c band sum:
//   qsgw_sxcf_exchange_d : Sigma_x block of sxcf_scz_exchange (m_sxcf_gemm.f90:203-231)
//   qsgw_hqpe_d          : QP energies and the Hermitian self-energy of hqpe_sc
//                          (main_hqpe.sc.f90:150-161, 178-180)
#include <cmath>
#include <vector>
#include "zgemm_f64.cuh"

namespace qsgw {

// vz(G, it, itp) = wtff(it) * vcoud(G) * zmel(G, it, itp)   (m_sxcf_gemm.f90:220-226)
__global__ void exchange_scale_kernel(double2* __restrict__ vz, const double2* __restrict__ z,
                                      const double* __restrict__ vcoud, const double* __restrict__ wtff, int ngb,
                                      int nm, long long ncol) {
  const long long tot = static_cast<long long>(ngb) * ncol;
  for (long long e = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; e < tot;
       e += static_cast<long long>(gridDim.x) * blockDim.x) {
    const int g = static_cast<int>(e % ngb);
    const long long c = e / ngb;
    const int it = static_cast<int>(c % nm);
    const double f = wtff[it] * vcoud[g];
    const double2 v = z[e];
    vz[e] = make_double2(f * v.x, f * v.y);
  }
}

// e_QP = e_LDA + SEx + SExcore + Re SEc - vxc (eV), Sigma_h = SEx + SExcore + (SEc + SEc^H)/2 - vxc_band/2 (Ha)
__global__ void hqpe_kernel(const double2* __restrict__ sex, const double2* __restrict__ sexc,
                            const double2* __restrict__ sec, const double2* __restrict__ vxcm,
                            const double* __restrict__ elda, const double* __restrict__ vxcd, int ntq, int ld,
                            int nq, double hartree, double* __restrict__ eqp, double2* __restrict__ seh) {
  const long long tot = static_cast<long long>(ntq) * ntq * nq;
  for (long long e = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; e < tot;
       e += static_cast<long long>(gridDim.x) * blockDim.x) {
    const int i = static_cast<int>(e % ntq);
    const long long r = e / ntq;
    const int j = static_cast<int>(r % ntq);
    const int q = static_cast<int>(r / ntq);
    const long long base = static_cast<long long>(q) * ld * ld;
    const long long ij = base + i + static_cast<long long>(j) * ld, ji = base + j + static_cast<long long>(i) * ld;
    const double2 a = sex[ij], b = sexc[ij], c = sec[ij], ct = sec[ji], v = vxcm[ij];
    double2 o;
    o.x = a.x + b.x + 0.5 * (c.x + ct.x) - 0.5 * v.x;
    o.y = a.y + b.y + 0.5 * (c.y - ct.y) - 0.5 * v.y;
    seh[ij] = o;
    if (i == j) {
      const long long d = static_cast<long long>(q) * ntq + i;
      eqp[d] = elda[d] + (a.x + b.x + c.x) * hartree - vxcd[d];
    }
  }
}

static DevBuf g_ex_vz, g_ex_tab;

static int grid_for(long long n) {
  return static_cast<int>(std::max<long long>(1, std::min<long long>((n + 255) / 256, 16LL * ctx().sm_count)));
}

}  // namespace qsgw

using namespace qsgw;

extern "C" int qsgw_sxcf_exchange_d(double* zsec_d, int ntq, const double* zmel_d, int ngb, int ns1, int ns2,
                                    int ntqxx, const double* vcoud, const double* ekc, int nekc, int nctot,
                                    double ef, double esmr, double wkkr) {
  int rc = require_init();
  if (rc) return rc;
  QSGW_ARG(zsec_d && zmel_d && vcoud && ekc, "sxcf_exchange: null pointer");
  QSGW_ARG(ngb >= 1 && ntq >= ntqxx && ntqxx >= 0, "sxcf_exchange: ngb=%d ntq=%d ntqxx=%d", ngb, ntq, ntqxx);
  if (ns1 > ns2 || ntqxx == 0) return QSGW_OK;                    // :211 guard
  QSGW_ARG(ns1 >= 1, "sxcf_exchange: ns1=%d", ns1);
  const int nm = ns2 - ns1 + 1;
  // occupations wtff (:212-216): 1 for cores, wfacx(-1d99, ef, ekc(it+nctot), esmr) for valence
  std::vector<double> wtff(nm);
  for (int it = ns1; it <= ns2; ++it) {
    double w = 1.0;
    if (it > nctot) {
      const int idx = it + nctot;                                 // the reference indexes ekc(is1+nctot)
      QSGW_ARG(idx >= 1 && idx <= nekc, "sxcf_exchange: ekc(%d) outside 1..%d", idx, nekc);
      const double ek = ekc[idx - 1];
      if (esmr == 0.0) w = (-1e99 <= ek && ek < ef) ? 1.0 : 0.0;
      else w = 0.5 * std::erfc(-(ef - ek) / std::sqrt(2.0) / esmr) - 0.5 * std::erfc(-(-1e99 - ek) / std::sqrt(2.0) / esmr);
    }
    wtff[it - ns1] = w;
  }
  cudaStream_t s = ctx().stream;
  const long long ncol = static_cast<long long>(nm) * ntqxx;
  rc = g_ex_vz.ensure(static_cast<size_t>(ngb) * ncol * sizeof(double2));
  if (rc) return rc;
  rc = g_ex_tab.ensure((ngb + nm) * sizeof(double));
  if (rc) return rc;
  double* dv = g_ex_tab.as<double>();
  QSGW_CUDA(cudaMemcpyAsync(dv, vcoud, ngb * sizeof(double), cudaMemcpyHostToDevice, s));
  QSGW_CUDA(cudaMemcpyAsync(dv + ngb, wtff.data(), nm * sizeof(double), cudaMemcpyHostToDevice, s));
  exchange_scale_kernel<<<grid_for(static_cast<long long>(ngb) * ncol), 256, 0, s>>>(
      g_ex_vz.as<double2>(), reinterpret_cast<const double2*>(zmel_d), dv, dv + ngb, ngb, nm, ncol);
  count_launch();
  QSGW_LAUNCH_CHECK("exchange_scale_kernel");
  // zsec += -wkkr zmel^H vzmel over K = ngb * nm (:227-229)
  const long long kk = static_cast<long long>(ngb) * nm;
  return zgemm_f64(2, 0, ntqxx, ntqxx, static_cast<int>(kk), make_double2(-wkkr, 0.0),
                   reinterpret_cast<const double2*>(zmel_d), kk, 0, g_ex_vz.as<double2>(), kk, 0,
                   make_double2(1.0, 0.0), reinterpret_cast<double2*>(zsec_d), ntq, 0, 1, s);
}

extern "C" int qsgw_hqpe_d(const double* sex2_d, const double* sexcore2_d, const double* sec2_d,
                           const double* vxc_band_ry_d, const double* elda_ev_d, const double* vxc_ev_d, int ntq,
                           int ld, int nq, double* eqp_ev_d, double* sigma_herm_d) {
  int rc = require_init();
  if (rc) return rc;
  QSGW_ARG(sex2_d && sexcore2_d && sec2_d && vxc_band_ry_d && elda_ev_d && vxc_ev_d && eqp_ev_d && sigma_herm_d,
           "hqpe: null pointer");
  QSGW_ARG(ntq >= 1 && ld >= ntq && nq >= 1, "hqpe: ntq=%d ld=%d nq=%d", ntq, ld, nq);
  cudaStream_t s = ctx().stream;
  const double hartree = 27.211386245988;
  hqpe_kernel<<<grid_for(static_cast<long long>(ntq) * ntq * nq), 256, 0, s>>>(
      reinterpret_cast<const double2*>(sex2_d), reinterpret_cast<const double2*>(sexcore2_d),
      reinterpret_cast<const double2*>(sec2_d), reinterpret_cast<const double2*>(vxc_band_ry_d), elda_ev_d, vxc_ev_d,
      ntq, ld, nq, hartree, eqp_ev_d, reinterpret_cast<double2*>(sigma_herm_d));
  count_launch();
  QSGW_LAUNCH_CHECK("hqpe_kernel");
  return QSGW_OK;
}
