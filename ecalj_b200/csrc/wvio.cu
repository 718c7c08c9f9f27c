// W(iw) / W(w) record files in the reference's layout.
//
// __WVI.<iq> and __WVR.<iq> are fixed-length records without markers
// (m_mpiio.f90:12-73 writes them with MPI_File_write_at at offset
// (rec-1)*recl; m_sxcf_gemm.f90:317-318 reads them as Fortran direct-access
// unformatted files): record rec holds one nblochpmx x nblochpmx column-major
// matrix, complex(8) (recl = 16 nblochpmx^2) or complex(4) with the mixed
// precision build (writem_kind4, recl = 8 nblochpmx^2).  WVI record iw = W(i w_iw)
// - v, iw = 1..niw (m_llw.f90:373); WVR record iw - nw_i + 1 = W(w_iw) - v
// (m_llw.f90:177).  Reading can also produce the packed upper triangles the
// Sigma_c step keeps resident (m_sxcf_gemm.f90:325-354).
#include <fcntl.h>
#include <unistd.h>
#include <cerrno>
#include <cstring>
#include <vector>
#include "common.cuh"

namespace qsgw {

// packed(t, r) for t over the upper triangle i <= j of the leading ngb x ngb block, column by column
// (t = i + j (j + 1) / 2, 0-based): mode 1 = W(i, j), mode 2 = (W(i, j) + conj(W(j, i))) / 2.
__global__ void pack_upper_kernel(double2* __restrict__ out, const double2* __restrict__ w, int ld, int ngb,
                                  int nrec, int mode) {
  const long long ntri = static_cast<long long>(ngb) * (ngb + 1) / 2;
  const long long tot = ntri * nrec;
  for (long long e = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; e < tot;
       e += static_cast<long long>(gridDim.x) * blockDim.x) {
    const long long t = e % ntri;
    const int r = static_cast<int>(e / ntri);
    // column j: first t of column j is j (j + 1) / 2
    int j = static_cast<int>((sqrt(8.0 * static_cast<double>(t) + 1.0) - 1.0) * 0.5);
    while (static_cast<long long>(j) * (j + 1) / 2 > t) --j;
    while (static_cast<long long>(j + 1) * (j + 2) / 2 <= t) ++j;
    const int i = static_cast<int>(t - static_cast<long long>(j) * (j + 1) / 2);
    const double2* m = w + static_cast<long long>(r) * ld * ld;
    const double2 a = m[i + static_cast<long long>(ld) * j];
    double2 v = a;
    if (mode == 2) {
      const double2 b = m[j + static_cast<long long>(ld) * i];
      v = make_double2(0.5 * (a.x + b.x), 0.5 * (a.y - b.y));
    }
    out[e] = v;
  }
}

__global__ void widen_kernel(double2* __restrict__ out, const float2* __restrict__ in, long long n) {
  for (long long e = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; e < n;
       e += static_cast<long long>(gridDim.x) * blockDim.x) {
    const float2 v = in[e];
    out[e] = make_double2(v.x, v.y);
  }
}

__global__ void narrow_kernel(float2* __restrict__ out, const double2* __restrict__ in, long long n) {
  for (long long e = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; e < n;
       e += static_cast<long long>(gridDim.x) * blockDim.x) {
    const double2 v = in[e];
    out[e] = make_float2(static_cast<float>(v.x), static_cast<float>(v.y));
  }
}

static DevBuf g_wv_dev;

static int io_grid(long long n) {
  return static_cast<int>(std::max<long long>(1, std::min<long long>((n + 255) / 256, 16LL * ctx().sm_count)));
}

static int full_io(int fd, char* buf, size_t bytes, off_t off, bool wr, const char* path) {
  size_t done = 0;
  while (done < bytes) {
    const ssize_t k = wr ? pwrite(fd, buf + done, bytes - done, off + static_cast<off_t>(done))
                         : pread(fd, buf + done, bytes - done, off + static_cast<off_t>(done));
    if (k < 0 && errno == EINTR) continue;
    if (k <= 0) {
      set_error("wv file %s: %s at byte %lld", path, k < 0 ? std::strerror(errno) : "short file",
                static_cast<long long>(off) + static_cast<long long>(done));
      return QSGW_ERR_ARG;
    }
    done += static_cast<size_t>(k);
  }
  return QSGW_OK;
}

}  // namespace qsgw

using namespace qsgw;

extern "C" int qsgw_wv_write_d(const char* path, const double* zw_d, int nblochpmx, int rec0, int nrec, int kind4) {
  int rc = require_init();
  if (rc) return rc;
  QSGW_ARG(path && zw_d && nblochpmx >= 1 && rec0 >= 1 && nrec >= 0, "wv_write: bad arguments");
  if (nrec == 0) return QSGW_OK;
  cudaStream_t s = ctx().stream;
  const long long nel = static_cast<long long>(nblochpmx) * nblochpmx;
  const size_t esz = kind4 ? sizeof(float2) : sizeof(double2);
  const size_t recl = static_cast<size_t>(nel) * esz;
  const int fd = open(path, O_RDWR | O_CREAT, 0644);
  QSGW_ARG(fd >= 0, "wv_write: cannot open %s: %s", path, std::strerror(errno));
  std::vector<char> host(recl);
  for (int r = 0; r < nrec && rc == QSGW_OK; ++r) {
    const double2* src = reinterpret_cast<const double2*>(zw_d) + static_cast<long long>(r) * nel;
    if (kind4) {
      rc = g_wv_dev.ensure(recl);
      if (rc) break;
      narrow_kernel<<<io_grid(nel), 256, 0, s>>>(g_wv_dev.as<float2>(), src, nel);
      count_launch();
      if (cudaGetLastError() != cudaSuccess) {
        set_error("wv_write: narrow_kernel launch failed");
        rc = QSGW_ERR_CUDA;
        break;
      }
      src = nullptr;
    }
    const cudaError_t e = cudaMemcpyAsync(host.data(), kind4 ? g_wv_dev.p : static_cast<const void*>(src), recl,
                                          cudaMemcpyDeviceToHost, s);
    if (e != cudaSuccess || cudaStreamSynchronize(s) != cudaSuccess) {
      set_error("wv_write: device to host copy failed");
      rc = QSGW_ERR_CUDA;
      break;
    }
    rc = full_io(fd, host.data(), recl, static_cast<off_t>(rec0 - 1 + r) * static_cast<off_t>(recl), true, path);
  }
  close(fd);
  return rc;
}

extern "C" int qsgw_wv_read_d(const char* path, double* out_d, int nblochpmx, int rec0, int nrec, int kind4,
                              int pack, int ngb) {
  int rc = require_init();
  if (rc) return rc;
  QSGW_ARG(path && out_d && nblochpmx >= 1 && rec0 >= 1 && nrec >= 0 && pack >= 0 && pack <= 2,
           "wv_read: bad arguments");
  QSGW_ARG(pack == 0 || (ngb >= 1 && ngb <= nblochpmx), "wv_read: ngb=%d outside 1..%d", ngb, nblochpmx);
  if (nrec == 0) return QSGW_OK;
  cudaStream_t s = ctx().stream;
  const long long nel = static_cast<long long>(nblochpmx) * nblochpmx;
  const size_t esz = kind4 ? sizeof(float2) : sizeof(double2);
  const size_t recl = static_cast<size_t>(nel) * esz;
  const int fd = open(path, O_RDONLY);
  QSGW_ARG(fd >= 0, "wv_read: cannot open %s: %s", path, std::strerror(errno));
  std::vector<char> host(recl);
  // staging on the device: the raw record (kind4) and, 256-byte aligned after it, the widened record (packing)
  const size_t raw_bytes = kind4 ? ((recl + 255) / 256) * 256 : 0;
  const size_t need = raw_bytes + (pack ? static_cast<size_t>(nel) * sizeof(double2) : 0);
  if (need) rc = g_wv_dev.ensure(need);
  const long long ntri = static_cast<long long>(ngb) * (ngb + 1) / 2;
  for (int r = 0; r < nrec && rc == QSGW_OK; ++r) {
    rc = full_io(fd, host.data(), recl, static_cast<off_t>(rec0 - 1 + r) * static_cast<off_t>(recl), false, path);
    if (rc) break;
    double2* full = pack ? reinterpret_cast<double2*>(g_wv_dev.as<char>() + raw_bytes)
                         : reinterpret_cast<double2*>(out_d) + static_cast<long long>(r) * nel;
    cudaError_t e;
    if (kind4) {
      e = cudaMemcpyAsync(g_wv_dev.p, host.data(), recl, cudaMemcpyHostToDevice, s);
      if (e == cudaSuccess) {
        widen_kernel<<<io_grid(nel), 256, 0, s>>>(full, g_wv_dev.as<float2>(), nel);
        count_launch();
        e = cudaGetLastError();
      }
    } else {
      e = cudaMemcpyAsync(full, host.data(), recl, cudaMemcpyHostToDevice, s);
    }
    if (e == cudaSuccess && pack) {
      pack_upper_kernel<<<io_grid(ntri), 256, 0, s>>>(reinterpret_cast<double2*>(out_d) + static_cast<long long>(r) * ntri,
                                                      full, nblochpmx, ngb, 1, pack);
      count_launch();
      e = cudaGetLastError();
    }
    // the host record buffer is reused: finish its copy first
    if (e != cudaSuccess || cudaStreamSynchronize(s) != cudaSuccess) {
      set_error("wv_read: host to device copy or kernel failed");
      rc = QSGW_ERR_CUDA;
    }
  }
  close(fd);
  return rc;
}
