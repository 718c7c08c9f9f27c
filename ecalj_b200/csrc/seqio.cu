// Fortran sequential unformatted files of the QSGW chain (host memory, no GPU):
//
// * __Vcoud.<iq>: the Coulomb eigenproblem's output, four records
//   ngb | q(3) | vcoud(ngb) | zcousq(ngb, ngb)  (written at
//   main_hvccfp0.f90:396-400 with vcoud = -eb, read by Readvcoud,
//   m_readVcoud.f90:30-40, which also forms vcousq = sqrt(vcoud));
// * SEX2U / SEXcore2U / SEC2U (D for spin 2): the self-energy matrices,
//   a header record nspin, nq, ntq, nqbz, nqibz, n1, n2, n3 and one record
//   is, q(3), zsec(ntq, ntq) per q (main_hsfp0.sc.f90:322, 333, 340, 359;
//   read at main_hqpe.sc.f90:132-148).
//
// A record is the gfortran / ifort / nvfortran default layout: a 4-byte
// length, the payload, the same length again.  Default integers are 4 bytes
// (the reference is built without a default-integer-8 flag).  Records are
// limited to 2^31 - 1 bytes (ngb <= 11585 for zcousq); longer records would
// need the compilers' continuation markers and are refused.
#include <cerrno>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include "common.cuh"

namespace qsgw {
namespace {

struct Piece {
  void* p;        // read target (nullptr: skip these bytes) or write source
  size_t bytes;
};

constexpr size_t MAX_RECORD = 0x7fffffff;

class SeqFile {
 public:
  SeqFile(const char* path, bool write) : path_(path) {
    f_ = std::fopen(path, write ? "wb" : "rb");
    err_ = f_ ? 0 : errno;
  }
  ~SeqFile() {
    if (f_) std::fclose(f_);
  }
  SeqFile(const SeqFile&) = delete;
  SeqFile& operator=(const SeqFile&) = delete;

  int open_status(const char* what) const {
    QSGW_ARG(f_, "%s: cannot open %s: %s", what, path_, std::strerror(err_));
    return QSGW_OK;
  }

  // The file must hold exactly `want` bytes (the layout its header implies), checked before
  // a caller sizes arrays from that header.
  int check_length(const char* what, long double want) {
    const long here = std::ftell(f_);
    QSGW_ARG(here >= 0 && std::fseek(f_, 0, SEEK_END) == 0, "%s: %s: cannot seek", what, path_);
    const long total = std::ftell(f_);
    QSGW_ARG(std::fseek(f_, here, SEEK_SET) == 0, "%s: %s: cannot seek", what, path_);
    QSGW_ARG(static_cast<long double>(total) == want,
             "%s: %s holds %ld bytes, its header implies %.0Lf (not a file of this layout, or cut short)", what,
             path_, total, want);
    return QSGW_OK;
  }

  int put(const char* what, const Piece* pc, int n) {
    size_t len = 0;
    for (int i = 0; i < n; ++i) len += pc[i].bytes;
    QSGW_ARG(len <= MAX_RECORD, "%s: %s: record of %zu bytes exceeds 2^31-1", what, path_, len);
    const int32_t m = static_cast<int32_t>(len);
    bool ok = std::fwrite(&m, 4, 1, f_) == 1;
    for (int i = 0; ok && i < n; ++i)
      ok = pc[i].bytes == 0 || std::fwrite(pc[i].p, 1, pc[i].bytes, f_) == pc[i].bytes;
    ok = ok && std::fwrite(&m, 4, 1, f_) == 1;
    QSGW_ARG(ok, "%s: %s: write failed: %s", what, path_, std::strerror(errno));
    ++nrec_;
    return QSGW_OK;
  }

  // Reads one record into the pieces; their sizes must add up to its length.
  int get(const char* what, const Piece* pc, int n) {
    size_t want = 0;
    for (int i = 0; i < n; ++i) want += pc[i].bytes;
    int32_t m = 0, m2 = 0;
    QSGW_ARG(std::fread(&m, 4, 1, f_) == 1, "%s: %s: record %d missing (end of file)", what, path_, nrec_ + 1);
    QSGW_ARG(m >= 0 && static_cast<size_t>(m) == want,
             "%s: %s: record %d holds %d bytes, expected %zu (a 4-byte-marker sequential file of this layout)",
             what, path_, nrec_ + 1, m, want);
    for (int i = 0; i < n; ++i) {
      if (pc[i].bytes == 0) continue;
      bool ok;
      if (pc[i].p)
        ok = std::fread(pc[i].p, 1, pc[i].bytes, f_) == pc[i].bytes;
      else
        ok = std::fseek(f_, static_cast<long>(pc[i].bytes), SEEK_CUR) == 0;
      QSGW_ARG(ok, "%s: %s: record %d is cut short", what, path_, nrec_ + 1);
    }
    QSGW_ARG(std::fread(&m2, 4, 1, f_) == 1 && m2 == m, "%s: %s: record %d has no matching end marker", what,
             path_, nrec_ + 1);
    ++nrec_;
    return QSGW_OK;
  }

 private:
  const char* path_;
  FILE* f_ = nullptr;
  int err_ = 0;
  int nrec_ = 0;
};

}  // namespace
}  // namespace qsgw

using namespace qsgw;

extern "C" int qsgw_vcoud_write(const char* path, int ngb, const double* q, const double* vcoud,
                                const double* zcousq) {
  QSGW_ARG(path && q && vcoud && zcousq && ngb >= 1, "vcoud_write: bad arguments (ngb=%d)", ngb);
  SeqFile f(path, true);
  int rc = f.open_status("vcoud_write");
  if (rc) return rc;
  int32_t n = ngb;
  const size_t nn = static_cast<size_t>(ngb);
  Piece r1{&n, 4}, r2{const_cast<double*>(q), 24}, r3{const_cast<double*>(vcoud), 8 * nn},
      r4{const_cast<double*>(zcousq), 16 * nn * nn};
  if ((rc = f.put("vcoud_write", &r1, 1)) || (rc = f.put("vcoud_write", &r2, 1)) ||
      (rc = f.put("vcoud_write", &r3, 1)) || (rc = f.put("vcoud_write", &r4, 1)))
    return rc;
  return QSGW_OK;
}

extern "C" int qsgw_vcoud_read(const char* path, int ngb_cap, int* ngb, double* q, double* vcoud, double* vcousq,
                               double* zcousq) {
  QSGW_ARG(path && ngb, "vcoud_read: bad arguments");
  SeqFile f(path, false);
  int rc = f.open_status("vcoud_read");
  if (rc) return rc;
  int32_t n = 0;
  double qv[3];
  Piece r1{&n, 4}, r2{qv, 24};
  if ((rc = f.get("vcoud_read", &r1, 1)) || (rc = f.get("vcoud_read", &r2, 1))) return rc;
  QSGW_ARG(n >= 1, "vcoud_read: %s: ngb = %d", path, n);
  const long double ln = n;
  if ((rc = f.check_length("vcoud_read", (4 + 8) + (24 + 8) + (8 * ln + 8) + (16 * ln * ln + 8)))) return rc;
  *ngb = n;
  if (q) std::memcpy(q, qv, sizeof qv);
  if (!vcoud && !vcousq && !zcousq) return QSGW_OK;        // header query
  QSGW_ARG(n <= ngb_cap, "vcoud_read: %s holds ngb = %d, the arrays take %d", path, n, ngb_cap);
  const size_t nn = static_cast<size_t>(n);
  double* v = vcoud;
  if (!v && vcousq) v = vcousq;                             // sqrt formed in place below
  Piece r3{v, 8 * nn}, r4{zcousq, 16 * nn * nn};
  if ((rc = f.get("vcoud_read", &r3, 1)) || (rc = f.get("vcoud_read", &r4, 1))) return rc;
  if (vcousq)
    for (size_t i = 0; i < nn; ++i) vcousq[i] = std::sqrt(v[i]);
  return QSGW_OK;
}

extern "C" int qsgw_sigma_write(const char* path, const int* head, int is, const double* qibz,
                                const double* zsec) {
  QSGW_ARG(path && head && qibz && zsec, "sigma_write: bad arguments");
  const int nq = head[1], ntq = head[2];
  QSGW_ARG(nq >= 0 && ntq >= 1, "sigma_write: nq=%d ntq=%d", nq, ntq);
  SeqFile f(path, true);
  int rc = f.open_status("sigma_write");
  if (rc) return rc;
  int32_t h[8];
  for (int i = 0; i < 8; ++i) h[i] = head[i];
  Piece r1{h, 32};
  if ((rc = f.put("sigma_write", &r1, 1))) return rc;
  int32_t isx = is;
  const size_t mat = static_cast<size_t>(ntq) * ntq;
  for (int ip = 0; ip < nq; ++ip) {
    Piece r[3] = {{&isx, 4}, {const_cast<double*>(qibz + 3 * static_cast<size_t>(ip)), 24},
                  {const_cast<double*>(zsec + 2 * mat * ip), 16 * mat}};
    if ((rc = f.put("sigma_write", r, 3))) return rc;
  }
  return QSGW_OK;
}

extern "C" int qsgw_sigma_read(const char* path, int* head, int nq_cap, int ntq_cap, int* isx, double* qibz,
                               double* zsec) {
  QSGW_ARG(path && head, "sigma_read: bad arguments");
  SeqFile f(path, false);
  int rc = f.open_status("sigma_read");
  if (rc) return rc;
  int32_t h[8];
  Piece r1{h, 32};
  if ((rc = f.get("sigma_read", &r1, 1))) return rc;
  const int nq = h[1], ntq = h[2];
  QSGW_ARG(nq >= 0 && ntq >= 1, "sigma_read: %s: header nq=%d ntq=%d", path, nq, ntq);
  const long double lt = ntq;
  if ((rc = f.check_length("sigma_read", (32 + 8) + static_cast<long double>(nq) * (4 + 24 + 16 * lt * lt + 8))))
    return rc;
  for (int i = 0; i < 8; ++i) head[i] = h[i];
  if (!zsec && !qibz && !isx) return QSGW_OK;               // header query
  QSGW_ARG(nq <= nq_cap && ntq <= ntq_cap, "sigma_read: %s holds nq=%d ntq=%d, the arrays take %d, %d", path, nq,
           ntq, nq_cap, ntq_cap);
  const size_t mat = static_cast<size_t>(ntq) * ntq;
  for (int ip = 0; ip < nq; ++ip) {
    int32_t s = 0;
    Piece r[3] = {{&s, 4}, {qibz ? qibz + 3 * static_cast<size_t>(ip) : nullptr, 24},
                  {zsec ? zsec + 2 * mat * ip : nullptr, 16 * mat}};
    if ((rc = f.get("sigma_read", r, 3))) return rc;
    if (isx) isx[ip] = s;
  }
  return QSGW_OK;
}
