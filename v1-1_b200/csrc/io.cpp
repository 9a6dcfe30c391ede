// Orbital and A-vector files in the reference's layout: Fortran unformatted
// sequential records as gfortran writes them (a 4-byte little-endian length
// before and after each record; records must stay below 2 GiB).
//
//   orbital file  (save_vector / write_spf / spf_header_write,
//                  MCTDH.SRC/loadstuff.f90:9-180):
//     record 1: spfdims(3), number of orbitals, cflag (=1 complex)   5 x int32
//     record 2: orbitals (spfsize x num) complex*16, column-major
//   A-vector file (avector_header_write / write_avector,
//                  MCTDH.SRC/configload.f90:221-249, 850-863):
//     record 1: numvects                                               int32
//     record 2: num2part, numr, numconfig, restrictflag, restrictms,
//               allspinproject, spinrestrictval, 0 ... (100 x int32)
//     record 3: icomplex (=1)                                          int32
//     then per vector and configuration: configlist(num2part) int32,
//               avector(numr) complex*16
// Loading an A-vector (easy_load_avectors, configload.f90:801-847) reorders
// each stored determinant to the canonical order, multiplies by the phase of
// that reordering and places it at its index in the walk tables' configuration
// list; determinants not in the list are an error.
#include <algorithm>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <memory>
#include <unordered_map>
#include <vector>
#include "walks.hpp"
#include "common.cuh"
#include "../../include/sincgpu.h"

namespace sincgpu {
namespace {

struct File {
  FILE* f = nullptr;
  ~File() {
    if (f) fclose(f);
  }
};

int write_record(FILE* f, const void* a, size_t na, const void* b = nullptr, size_t nb = 0) {
  const size_t len = na + nb;
  SG_CHECK(len < 0x7fffffffULL, SINCGPU_ERANGE, "record of %zu bytes exceeds 2 GiB", len);
  const int32_t m = (int32_t)len;
  SG_CHECK(fwrite(&m, 4, 1, f) == 1 && (na == 0 || fwrite(a, 1, na, f) == na) &&
               (nb == 0 || fwrite(b, 1, nb, f) == nb) && fwrite(&m, 4, 1, f) == 1,
           SINCGPU_ECUDA, "write failed");
  return SINCGPU_OK;
}

// reads one record into buf (resized to the record length)
int read_record(FILE* f, std::vector<char>& buf) {
  int32_t m = 0, t = 0;
  SG_CHECK(fread(&m, 4, 1, f) == 1, SINCGPU_EINVAL, "unexpected end of file");
  SG_CHECK(m >= 0, SINCGPU_ERANGE, "continued (> 2 GiB) records are not supported");
  buf.resize((size_t)m);
  SG_CHECK(m == 0 || fread(buf.data(), 1, (size_t)m, f) == (size_t)m, SINCGPU_EINVAL, "truncated record");
  SG_CHECK(fread(&t, 4, 1, f) == 1 && t == m, SINCGPU_EINVAL, "record markers do not match (%d, %d)", m, t);
  return SINCGPU_OK;
}

inline int iind(int orb, int spin) { return (orb - 1) * 2 + spin; }

int reorder_phase(int* c, int numpart) {
  int phase = 1;
  bool done = false;
  while (!done) {
    done = true;
    for (int j = 0; j < numpart - 1; ++j)
      if (iind(c[2 * j], c[2 * j + 1]) > iind(c[2 * j + 2], c[2 * j + 3])) {
        phase = -phase;
        done = false;
        std::swap(c[2 * j], c[2 * j + 2]);
        std::swap(c[2 * j + 1], c[2 * j + 3]);
      }
  }
  return phase;
}

}  // namespace
}  // namespace sincgpu

using namespace sincgpu;

extern "C" {

int sincgpu_save_spfs(const char* path, const int* dims, int numspf, const double* spfs) {
  SG_CHECK(path && dims && spfs && numspf >= 1, SINCGPU_EINVAL, "bad argument");
  File fh;
  fh.f = fopen(path, "wb");
  SG_CHECK(fh.f, SINCGPU_EINVAL, "cannot open %s for writing", path);
  const int32_t head[5] = {dims[0], dims[1], dims[2], numspf, 1};
  SG_TRY(write_record(fh.f, head, sizeof(head)));
  const size_t n = (size_t)dims[0] * dims[1] * dims[2] * numspf;
  return write_record(fh.f, spfs, sizeof(double) * 2 * n);
}

int sincgpu_load_spfs(const char* path, int* dims, int* numspf, double* spfs, long long capacity) {
  SG_CHECK(path && dims && numspf, SINCGPU_EINVAL, "bad argument");
  File fh;
  fh.f = fopen(path, "rb");
  SG_CHECK(fh.f, SINCGPU_EINVAL, "cannot open %s", path);
  std::vector<char> buf;
  SG_TRY(read_record(fh.f, buf));
  SG_CHECK(buf.size() == 20, SINCGPU_EINVAL, "orbital header of %zu bytes, expected 20", buf.size());
  int32_t head[5];
  std::memcpy(head, buf.data(), 20);
  SG_CHECK(head[4] == 1, SINCGPU_EINVAL, "real-valued orbital files are not supported");
  for (int i = 0; i < 3; ++i) dims[i] = head[i];
  *numspf = head[3];
  if (!spfs) return SINCGPU_OK;  // header only
  const long long n = (long long)head[0] * head[1] * head[2] * head[3];
  SG_CHECK(n <= capacity, SINCGPU_ERANGE, "file holds %lld complex values, buffer %lld", n, capacity);
  SG_TRY(read_record(fh.f, buf));
  SG_CHECK((long long)buf.size() == 16 * n, SINCGPU_EINVAL, "orbital record of %zu bytes, expected %lld",
           buf.size(), 16 * n);
  std::memcpy(spfs, buf.data(), buf.size());
  return SINCGPU_OK;
}

int sincgpu_save_avector(const char* path, sincgpu_walks* walks, int numvects, const double* avectors,
                         int allspinproject, int spinrestrictval) {
  SG_CHECK(path && walks && avectors && numvects >= 1, SINCGPU_EINVAL, "bad argument");
  const Walks& w = walks->w;
  File fh;
  fh.f = fopen(path, "wb");
  SG_CHECK(fh.f, SINCGPU_EINVAL, "cannot open %s for writing", path);
  const int32_t nv = numvects;
  SG_TRY(write_record(fh.f, &nv, 4));
  int32_t arr[100] = {0};
  arr[0] = 2 * w.numpart;  // num2part
  arr[1] = 1;              // numr
  arr[2] = w.numconfig;
  arr[3] = 1;              // restrictflag
  arr[4] = w.restrictms;
  arr[5] = allspinproject;
  arr[6] = spinrestrictval;
  SG_TRY(write_record(fh.f, arr, sizeof(arr)));
  const int32_t icomplex = 1;
  SG_TRY(write_record(fh.f, &icomplex, 4));
  std::vector<int32_t> cfg(2 * w.numpart);
  for (int v = 0; v < numvects; ++v)
    for (int c = 0; c < w.numconfig; ++c) {
      for (int k = 0; k < 2 * w.numpart; ++k) cfg[k] = w.configlist[(size_t)c * 2 * w.numpart + k];
      SG_TRY(write_record(fh.f, cfg.data(), 4 * cfg.size(), avectors + 2 * ((size_t)v * w.numconfig + c), 16));
    }
  return SINCGPU_OK;
}

int sincgpu_load_avector(const char* path, sincgpu_walks* walks, int maxvects, double* avectors, int* numvects) {
  SG_CHECK(path && walks && avectors && numvects && maxvects >= 1, SINCGPU_EINVAL, "bad argument");
  const Walks& w = walks->w;
  const int np = w.numpart;
  File fh;
  fh.f = fopen(path, "rb");
  SG_CHECK(fh.f, SINCGPU_EINVAL, "cannot open %s", path);
  std::vector<char> buf;
  SG_TRY(read_record(fh.f, buf));
  SG_CHECK(buf.size() == 4, SINCGPU_EINVAL, "bad A-vector header");
  int32_t nv;
  std::memcpy(&nv, buf.data(), 4);
  SG_TRY(read_record(fh.f, buf));
  SG_CHECK(buf.size() == 400, SINCGPU_EINVAL, "A-vector header of %zu bytes, expected 400", buf.size());
  int32_t arr[100];
  std::memcpy(arr, buf.data(), 400);
  const int num2part = arr[0], numr = arr[1], nconf = arr[2];
  SG_CHECK(num2part == 2 * np, SINCGPU_EINVAL, "file has %d electrons, the tables %d", num2part / 2, np);
  SG_CHECK(numr == 1, SINCGPU_EINVAL, "numr %d: only numr = 1 files are supported", numr);
  SG_TRY(read_record(fh.f, buf));
  int32_t icomplex;
  std::memcpy(&icomplex, buf.data(), 4);
  SG_CHECK(icomplex == 1, SINCGPU_EINVAL, "real-valued A-vector files are not supported");
  std::unordered_map<uint64_t, int> index;
  for (int c = 0; c < w.numconfig; ++c) {
    uint64_t m = 0;
    for (int j = 0; j < np; ++j)
      m |= 1ull << (iind(w.configlist[(size_t)c * 2 * np + 2 * j], w.configlist[(size_t)c * 2 * np + 2 * j + 1]) - 1);
    index[m] = c;
  }
  const int nread = std::min<int>(nv, maxvects);
  std::memset(avectors, 0, sizeof(double) * 2 * (size_t)nread * w.numconfig);
  std::vector<int> cfg(2 * np);
  for (int v = 0; v < nread; ++v)
    for (int k = 0; k < nconf; ++k) {
      SG_TRY(read_record(fh.f, buf));
      SG_CHECK(buf.size() == 4 * (size_t)num2part + 16, SINCGPU_EINVAL, "bad A-vector record");
      std::memcpy(cfg.data(), buf.data(), 4 * (size_t)num2part);
      double val[2];
      std::memcpy(val, buf.data() + 4 * (size_t)num2part, 16);
      const int phase = reorder_phase(cfg.data(), np);
      uint64_t m = 0;
      bool ok = true;
      for (int j = 0; j < np && ok; ++j) {
        if (cfg[2 * j] < 1 || cfg[2 * j] > w.nspf || cfg[2 * j + 1] < 1 || cfg[2 * j + 1] > 2) {
          ok = false;
        } else {
          const uint64_t bit = 1ull << (iind(cfg[2 * j], cfg[2 * j + 1]) - 1);
          if (m & bit) ok = false;  // two electrons in one spin-orbital
          m |= bit;
        }
      }
      auto it = ok ? index.find(m) : index.end();
      SG_CHECK(it != index.end(), SINCGPU_EINVAL, "determinant %d of vector %d is not in the configuration list",
               k + 1, v + 1);
      double* dst = avectors + 2 * ((size_t)v * w.numconfig + it->second);
      dst[0] = val[0] * phase;
      dst[1] = val[1] * phase;
    }
  *numvects = nread;
  return SINCGPU_OK;
}

}  // extern "C"
