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

  // ---- spin projection (allspinproject=1); spinrestrictval < 0: not built ----
  int spinrestrictval = -1;                 // 2S
  std::vector<int> numspinwalks;            // per config
  std::vector<long long> spinwalk_off;      // CSR over configs
  std::vector<int> spinwalk, spinwalkdirphase;  // 1-based target, phase
  std::vector<long long> spinset_off;       // kept sets (rank > 0), CSR
  std::vector<int> spinsets;                // 1-based configs in discovery order
  std::vector<int> spinsetrank;
  std::vector<long long> spinproj_off;      // offset of each set's size^2 projector
  std::vector<double> spinproj;             // row-major P(ii,jj) = sum_k v_k(ii) v_k(jj)
  std::vector<int> spin_eliminated;         // 1-based configs of rank-0 sets
  long long numspinconfig = 0;              // total rank
  int maxspinsetsize = 0;
};

int build_walks(Walks& w, int numelec, int nspf, int restrictms, int nthreads);
// spin walks, sets and S^2 projectors; spinrestrictval < 0 selects |restrictms|
int build_spin(Walks& w, int spinrestrictval);

}  // namespace sincgpu

// opaque handle of the C ABI (include/sincgpu.h)
struct sincgpu_walks {
  sincgpu::Walks w;
};
