// Determinant list, walk and hop tables (host side; uploaded once to the device).
#pragma once
#include <cstdint>
#include <vector>

namespace sincgpu {

struct Walks {
  int numelec = 0, numpart = 0, nspf = 0, restrictms = 0;
  int numconfig = 0;
  // configlist(2*numpart, numconfig), 1-based orbital and spin values
  std::vector<int> configlist;
  // per-config counts and offsets (scol/dcol: walks before config c, 0-based)
  std::vector<int> numsinglewalks, numdoublewalks;
  std::vector<long long> scol, dcol;
  // walk tables, walk-major
  std::vector<int> singlewalkopspf;   // 2 per walk: [ispf, jspf]
  std::vector<int> singlewalkdirphase;
  std::vector<int> singlewalk;        // target config (1-based)
  std::vector<int> doublewalkdirspf;  // 4 per walk: [jjspf, iispf, jspf, ispf]
  std::vector<int> doublewalkdirphase;
  std::vector<int> doublewalk;
  // hops: CSR over configs; start/end are 1-based walk positions inside the config
  std::vector<long long> singlehop_off, doublehop_off;
  std::vector<int> singlehop, singlehopwalkstart, singlehopwalkend;
  std::vector<int> doublehop, doublehopwalkstart, doublehopwalkend;
  std::vector<int> singlediaghop, doublediaghop;  // 1-based hop index or -1
};

int build_walks(Walks& w, int numelec, int nspf, int restrictms, int nthreads);

}  // namespace sincgpu
