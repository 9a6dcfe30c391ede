// Determinant list, walks and hops, restated from the reference so that every
// integer table (indices, phases, order) is identical:
//   fast_newconfiglist   MCTDH.SRC/newconfig.f90:349-1040  (numshells=1 full CI,
//                        restrictflag=1, spfrestrictflag=0, holeflag=0, dflevel 0)
//   reorder              MCTDH.SRC/newconfig.f90:140-161
//   allowedconfig0       MCTDH.SRC/newconfig.f90:167-261
//   walks / getnumwalks  MCTDH.SRC/walks.f90:149-506, 510-759 (per-config sort
//                        getlistorder 453-483: ascending target, ties last-first)
//   hops                 MCTDH.SRC/walks.f90:761-993
//   spin projection      MCTDH.SRC/spinwalks.f90 (getnumspinwalks 302-388,
//                        spinwalks 86-153, spinsets_first 156-299,
//                        configspin_matel 390-414, configspinset_projector
//                        432-642); the S^2 eigenproblem of each set is solved
//                        by cyclic Jacobi rotations instead of LAPACK dsyev
//                        (the projector onto an eigenspace does not depend on
//                        the solver beyond rounding)
// getconfiguration (newconfig.f90:49-131) returns the unique index of an
// allowed, ordered configuration; here that lookup is a hash of the set of
// occupied spin-orbitals (a 64-bit mask, nspf <= 32).
#include <algorithm>
#include <cmath>
#include <thread>
#include <functional>
#include <unordered_map>
#include "walks.hpp"
#include "common.cuh"

namespace sincgpu {

namespace {

inline int iind(int orb, int spin) { return (orb - 1) * 2 + spin; }
inline void aarr(int index, int& orb, int& spin) {
  int ind = index - 1;
  orb = ind / 2 + 1;
  spin = ind % 2 + 1;
}

int reorder(int* c, int numpart) {
  int phase = 1;
  bool flag = false;
  while (!flag) {
    flag = true;
    for (int j = 0; j < numpart - 1; ++j) {
      if (iind(c[2 * j], c[2 * j + 1]) > iind(c[2 * j + 2], c[2 * j + 3])) {
        phase = -phase;
        flag = false;
        std::swap(c[2 * j], c[2 * j + 2]);
        std::swap(c[2 * j + 1], c[2 * j + 3]);
      }
    }
  }
  return phase;
}

struct Builder {
  Walks& w;
  std::unordered_map<uint64_t, int> index;

  explicit Builder(Walks& ww) : w(ww) {}

  bool allowed(const int* c) const {
    const int n = w.numpart;
    for (int j = 0; j < n; ++j)
      for (int i = j + 1; i < n; ++i)
        if (c[2 * i] == c[2 * j] && c[2 * i + 1] == c[2 * j + 1]) return false;
    for (int j = 0; j < n; ++j)
      if (c[2 * j] < 1 || c[2 * j] > w.nspf) return false;
    int s = 0;
    for (int j = 0; j < n; ++j) s += c[2 * j + 1] * 2 - 3;
    if (s != w.restrictms) return false;
    // single shell with numexcite=999, minocc=-999, maxocc=999 (parameters.f90:152-158)
    if (n < 2 * w.nspf - 999) return false;
    return true;
  }

  static uint64_t mask(const int* c, int n) {
    uint64_t m = 0;
    for (int j = 0; j < n; ++j) m |= 1ull << (iind(c[2 * j], c[2 * j + 1]) - 1);
    return m;
  }

  int lookup(const int* c) const {
    auto it = index.find(mask(c, w.numpart));
    return it == index.end() ? -1 : it->second;
  }

  void configlist() {
    const int n = w.numpart, nspf = w.nspf;
    std::vector<int> lower(n + 2, 0), upper(n + 2, 0);
    const int numdoubly = n - std::abs(w.restrictms);
    for (int ii = 1; ii <= numdoubly; ++ii) lower[ii] = (ii + 1) / 2;
    for (int ii = 1; ii <= std::abs(w.restrictms); ++ii) lower[ii + numdoubly] = numdoubly / 2 + ii;
    for (int ii = 1; ii <= n; ++ii) upper[ii] = nspf + 1 - lower[n + 1 - ii];
    // single shell: mynumexcite = min(999, max(0,2nspf-numelec), 2nspf); mm = 2nspf - min(.,2nspf-n)
    const int isums = std::max(0, 2 * nspf - std::max(0, w.numelec));
    const int mynumexcite = std::min(std::min(999, isums), std::max(0, 2 * nspf));
    const int mm = 2 * nspf - std::min(mynumexcite, 2 * nspf - n);
    for (int jj = 1; jj <= mm && jj <= n; ++jj) upper[jj] = std::min(upper[jj], nspf - (mm - jj) / 2);
    std::vector<int> iii(n + 1, 0);
    std::vector<int> cfg(2 * n), c(2 * n);
    std::vector<int> single(n + 1);
    // nested loops ii1..iin (newconfig.f90:629-716)
    auto emit = [&]() {
      for (int k = 1; k <= n; ++k) cfg[2 * k - 2] = iii[k];
      for (int k = 1; k <= n; ++k) single[k] = 1;
      for (int k = 2; k <= n; ++k)
        if (iii[k] == iii[k - 1]) {
          cfg[2 * (k - 1) - 1] = 1;
          cfg[2 * k - 1] = 2;
          single[k - 1] = 0;
          single[k] = 0;
        }
      std::vector<int> singles;
      for (int k = 1; k <= n; ++k)
        if (single[k]) singles.push_back(k);
      const int ns = (int)singles.size();
      for (long long bits = 0; bits < (1LL << ns); ++bits) {  // jj1 outermost
        c = cfg;
        for (int pos = 0; pos < ns; ++pos) {
          int jj = (int)((bits >> (ns - 1 - pos)) & 1);
          c[2 * singles[pos] - 1] = jj + 1;
        }
        if (allowed(c.data())) {
          reorder(c.data(), n);
          w.configlist.insert(w.configlist.end(), c.begin(), c.end());
        }
      }
    };
    // nested loops over the electrons' orbitals
    std::function<void(int)> rec = [&](int k) {
      if (k > n) {
        emit();
        return;
      }
      int lo = lower[k];
      if (k >= 2) lo = std::max(lo, iii[k - 1]);
      if (k >= 3) lo = std::max(lo, iii[k - 2] + 1);
      for (int v = lo; v <= upper[k]; ++v) {
        iii[k] = v;
        rec(k + 1);
      }
    };
    rec(1);
    w.numconfig = (int)(w.configlist.size() / (2 * n));
    index.reserve(w.numconfig * 2);
    for (int i = 0; i < w.numconfig; ++i) index[mask(&w.configlist[(size_t)2 * n * i], n)] = i + 1;
  }

  struct SW { int c2, ph, a, b; };
  struct DW { int c2, ph, d1, d2, d3, d4; };

  template <class T>
  static void listsort(std::vector<T>& v) {
    // ascending target; equal targets in reverse order of generation
    std::vector<int> order(v.size());
    for (size_t i = 0; i < v.size(); ++i) order[i] = (int)i;
    std::stable_sort(order.begin(), order.end(), [&](int x, int y) {
      if (v[x].c2 != v[y].c2) return v[x].c2 < v[y].c2;
      return x > y;
    });
    std::vector<T> out(v.size());
    for (size_t i = 0; i < v.size(); ++i) out[i] = v[order[i]];
    v.swap(out);
  }

  void walks_for(int c1, std::vector<SW>& sw, std::vector<DW>& dw) const {
    const int n = w.numpart, nspf = w.nspf;
    const int* th = &w.configlist[(size_t)2 * n * (c1 - 1)];
    std::vector<int> that(2 * n);
    sw.clear();
    dw.clear();
    for (int idof = 0; idof < n; ++idof) {
      const int ispf = th[2 * idof], ispin = th[2 * idof + 1];
      for (int jindex = 1; jindex <= 2 * nspf; ++jindex) {
        int jspf, jspin;
        aarr(jindex, jspf, jspin);
        if (ispin != jspin) continue;
        bool flag = false;
        for (int jdof = 0; jdof < n; ++jdof)
          if (jdof != idof && iind(th[2 * jdof], th[2 * jdof + 1]) == jindex) flag = true;
        if (flag) continue;
        std::copy(th, th + 2 * n, that.begin());
        that[2 * idof] = jspf;
        that[2 * idof + 1] = jspin;
        const int ph = reorder(that.data(), n);
        if (!allowed(that.data())) continue;
        const int c2 = lookup(that.data());
        sw.push_back({c2, ph, ispf, jspf});
      }
    }
    for (int idof = 0; idof < n; ++idof)
      for (int iidof = idof + 1; iidof < n; ++iidof) {
        const int ispf = th[2 * idof], ispin = th[2 * idof + 1];
        const int iispf = th[2 * iidof], iispin = th[2 * iidof + 1];
        for (int jindex = 1; jindex <= 2 * nspf; ++jindex) {
          int jspf, jspin;
          aarr(jindex, jspf, jspin);
          if (ispin != jspin) continue;
          for (int jjindex = 1; jjindex <= 2 * nspf; ++jjindex) {
            if (jjindex == jindex) continue;
            int jjspf, jjspin;
            aarr(jjindex, jjspf, jjspin);
            if (iispin != jjspin) continue;
            bool flag = false;
            for (int jdof = 0; jdof < n && !flag; ++jdof)
              if (jdof != idof && jdof != iidof) {
                const int k = iind(th[2 * jdof], th[2 * jdof + 1]);
                if (k == jindex || k == jjindex) flag = true;
              }
            if (flag) continue;
            std::copy(th, th + 2 * n, that.begin());
            that[2 * idof] = jspf;
            that[2 * idof + 1] = jspin;
            that[2 * iidof] = jjspf;
            that[2 * iidof + 1] = jjspin;
            const int ph = reorder(that.data(), n);
            if (!allowed(that.data())) continue;
            const int c2 = lookup(that.data());
            dw.push_back({c2, ph, jjspf, iispf, jspf, ispf});  // walks.f90:343-345
          }
        }
      }
    listsort(sw);
    listsort(dw);
  }
};

template <class T>
void group_hops(const std::vector<int>& target, const std::vector<long long>& col,
                const std::vector<int>& num, int nc, std::vector<long long>& off, std::vector<int>& hop,
                std::vector<int>& st, std::vector<int>& en, std::vector<int>& diag) {
  off.assign(1, 0);
  hop.clear();
  st.clear();
  en.clear();
  diag.assign(nc, -1);
  for (int c = 0; c < nc; ++c) {
    const long long b = col[c];
    for (int iw = 0; iw < num[c]; ++iw) {
      const int t = target[b + iw];
      if (iw == 0 || t != target[b + iw - 1]) {
        hop.push_back(t);
        st.push_back(iw + 1);
        en.push_back(iw + 1);
        if (t == c + 1) diag[c] = (int)(hop.size() - off.back());
      } else {
        en.back() = iw + 1;
      }
    }
    off.push_back((long long)hop.size());
  }
}

}  // namespace

int build_walks(Walks& w, int numelec, int nspf, int restrictms, int nthreads) {
  SG_CHECK(numelec >= 1 && numelec <= 16, SINCGPU_ERANGE, "numelec %d outside [1,16]", numelec);
  SG_CHECK(nspf >= 1 && nspf <= 32, SINCGPU_ERANGE, "nspf %d outside [1,32]", nspf);
  SG_CHECK((numelec - std::abs(restrictms)) % 2 == 0 && std::abs(restrictms) <= numelec, SINCGPU_EINVAL,
           "restrictms %d not compatible with %d electrons", restrictms, numelec);
  w = Walks();
  w.numelec = w.numpart = numelec;
  w.nspf = nspf;
  w.restrictms = restrictms;
  Builder b(w);
  b.configlist();
  SG_CHECK(w.numconfig > 0, SINCGPU_EINVAL, "no configurations");
  const int nc = w.numconfig;
  if (nthreads <= 0) nthreads = (int)std::max(1u, std::thread::hardware_concurrency());
  nthreads = std::min(nthreads, nc);
  std::vector<std::vector<Builder::SW>> sws(nc);
  std::vector<std::vector<Builder::DW>> dws(nc);
  std::vector<std::thread> pool;
  for (int t = 0; t < nthreads; ++t)
    pool.emplace_back([&, t]() {
      for (int c = t; c < nc; c += nthreads) b.walks_for(c + 1, sws[c], dws[c]);
    });
  for (auto& th : pool) th.join();
  w.numsinglewalks.resize(nc);
  w.numdoublewalks.resize(nc);
  w.scol.assign(nc + 1, 0);
  w.dcol.assign(nc + 1, 0);
  for (int c = 0; c < nc; ++c) {
    w.numsinglewalks[c] = (int)sws[c].size();
    w.numdoublewalks[c] = (int)dws[c].size();
    w.scol[c + 1] = w.scol[c] + w.numsinglewalks[c];
    w.dcol[c + 1] = w.dcol[c] + w.numdoublewalks[c];
  }
  const long long ts = w.scol[nc], td = w.dcol[nc];
  w.singlewalkopspf.resize(2 * ts);
  w.singlewalkdirphase.resize(ts);
  w.singlewalk.resize(ts);
  w.doublewalkdirspf.resize(4 * td);
  w.doublewalkdirphase.resize(td);
  w.doublewalk.resize(td);
  for (int c = 0; c < nc; ++c) {
    for (size_t i = 0; i < sws[c].size(); ++i) {
      const long long k = w.scol[c] + (long long)i;
      const auto& e = sws[c][i];
      SG_CHECK(e.c2 > 0, SINCGPU_ESTATE, "walk target not in the configuration list");
      w.singlewalk[k] = e.c2;
      w.singlewalkdirphase[k] = e.ph;
      w.singlewalkopspf[2 * k] = e.a;
      w.singlewalkopspf[2 * k + 1] = e.b;
    }
    for (size_t i = 0; i < dws[c].size(); ++i) {
      const long long k = w.dcol[c] + (long long)i;
      const auto& e = dws[c][i];
      SG_CHECK(e.c2 > 0, SINCGPU_ESTATE, "walk target not in the configuration list");
      w.doublewalk[k] = e.c2;
      w.doublewalkdirphase[k] = e.ph;
      w.doublewalkdirspf[4 * k] = e.d1;
      w.doublewalkdirspf[4 * k + 1] = e.d2;
      w.doublewalkdirspf[4 * k + 2] = e.d3;
      w.doublewalkdirspf[4 * k + 3] = e.d4;
    }
  }
  group_hops<int>(w.singlewalk, w.scol, w.numsinglewalks, nc, w.singlehop_off, w.singlehop,
                  w.singlehopwalkstart, w.singlehopwalkend, w.singlediaghop);
  group_hops<int>(w.doublewalk, w.dcol, w.numdoublewalks, nc, w.doublehop_off, w.doublehop,
                  w.doublehopwalkstart, w.doublehopwalkend, w.doublediaghop);
  return SINCGPU_OK;
}

namespace {

// cyclic Jacobi eigen-decomposition of a real symmetric m x m matrix (row-major);
// on return vals holds the eigenvalues and column k of V the k-th eigenvector
void jacobi_eigen(int m, std::vector<double>& A, std::vector<double>& V, std::vector<double>& vals) {
  V.assign((size_t)m * m, 0.0);
  for (int i = 0; i < m; ++i) V[(size_t)i * m + i] = 1.0;
  double norm = 0.0;
  for (double x : A) norm += x * x;
  for (int sweep = 0; sweep < 100; ++sweep) {
    double off = 0.0;
    for (int p = 0; p < m; ++p)
      for (int q = p + 1; q < m; ++q) off += A[(size_t)p * m + q] * A[(size_t)p * m + q];
    if (off <= 1e-32 * norm || off == 0.0) break;
    for (int p = 0; p < m; ++p)
      for (int q = p + 1; q < m; ++q) {
        const double apq = A[(size_t)p * m + q];
        if (apq == 0.0) continue;
        const double theta = (A[(size_t)q * m + q] - A[(size_t)p * m + p]) / (2.0 * apq);
        const double t = (theta >= 0 ? 1.0 : -1.0) / (std::fabs(theta) + std::sqrt(theta * theta + 1.0));
        const double c = 1.0 / std::sqrt(t * t + 1.0), sn = t * c;
        for (int k = 0; k < m; ++k) {  // columns p, q
          const double akp = A[(size_t)k * m + p], akq = A[(size_t)k * m + q];
          A[(size_t)k * m + p] = c * akp - sn * akq;
          A[(size_t)k * m + q] = sn * akp + c * akq;
        }
        for (int k = 0; k < m; ++k) {  // rows p, q
          const double apk = A[(size_t)p * m + k], aqk = A[(size_t)q * m + k];
          A[(size_t)p * m + k] = c * apk - sn * aqk;
          A[(size_t)q * m + k] = sn * apk + c * aqk;
        }
        for (int k = 0; k < m; ++k) {
          const double vkp = V[(size_t)k * m + p], vkq = V[(size_t)k * m + q];
          V[(size_t)k * m + p] = c * vkp - sn * vkq;
          V[(size_t)k * m + q] = sn * vkp + c * vkq;
        }
      }
  }
  vals.resize(m);
  for (int i = 0; i < m; ++i) vals[i] = A[(size_t)i * m + i];
}

}  // namespace

int build_spin(Walks& w, int spinrestrictval) {
  SG_CHECK(w.numconfig > 0, SINCGPU_ESTATE, "walk tables not built");
  const int n = w.numpart, nc = w.numconfig;
  int srv = spinrestrictval < 0 ? std::abs(w.restrictms) : spinrestrictval;
  if (srv < std::abs(w.restrictms)) srv = std::abs(w.restrictms);  // getparams.f90:190-192
  SG_CHECK((srv - std::abs(w.restrictms)) % 2 == 0 && srv <= n, SINCGPU_EINVAL,
           "2S = %d not reachable with %d electrons and 2Ms = %d", srv, n, w.restrictms);
  // index of every configuration by its spin-orbital mask
  std::unordered_map<uint64_t, int> index;
  index.reserve((size_t)nc * 2);
  for (int c = 0; c < nc; ++c) {
    uint64_t m = 0;
    const int* cf = &w.configlist[(size_t)c * 2 * n];
    for (int j = 0; j < n; ++j) m |= 1ull << (iind(cf[2 * j], cf[2 * j + 1]) - 1);
    index[m] = c + 1;
  }
  Builder b(w);
  std::vector<int> msvalue(nc);
  std::vector<std::vector<int>> unpaired(nc);
  for (int c = 0; c < nc; ++c) {
    const int* cf = &w.configlist[(size_t)c * 2 * n];
    int ms = 0;
    for (int i = 0; i < n; ++i) {
      ms += cf[2 * i + 1] * 2 - 3;
      bool paired = false;
      for (int j = 0; j < n; ++j)
        if (j != i && cf[2 * j] == cf[2 * i]) {
          paired = true;
          break;
        }
      if (!paired) unpaired[c].push_back(i + 1);
    }
    msvalue[c] = ms;
  }
  // spin walks: flip one pair of unpaired electrons with opposite spins
  w.spinrestrictval = srv;
  w.numspinwalks.assign(nc, 0);
  w.spinwalk_off.assign(nc + 1, 0);
  w.spinwalk.clear();
  w.spinwalkdirphase.clear();
  std::vector<int> cfg(2 * n), that(2 * n);
  for (int c = 0; c < nc; ++c) {
    const auto& up = unpaired[c];
    for (size_t ii = 0; ii < up.size(); ++ii) {
      cfg.assign(&w.configlist[(size_t)c * 2 * n], &w.configlist[(size_t)c * 2 * n] + 2 * n);
      const int idof = up[ii];
      const int first = cfg[2 * idof - 1];
      cfg[2 * idof - 1] = cfg[2 * idof - 1] % 2 + 1;
      for (size_t jj = ii + 1; jj < up.size(); ++jj) {
        that = cfg;
        const int jdof = up[jj];
        if (that[2 * jdof - 1] == first) continue;
        that[2 * jdof - 1] = that[2 * jdof - 1] % 2 + 1;
        const int ph = reorder(that.data(), n);
        if (!b.allowed(that.data())) continue;
        uint64_t m = 0;
        for (int j = 0; j < n; ++j) m |= 1ull << (iind(that[2 * j], that[2 * j + 1]) - 1);
        auto it = index.find(m);
        SG_CHECK(it != index.end(), SINCGPU_ESTATE, "spin walk target not in the configuration list");
        w.spinwalk.push_back(it->second);
        w.spinwalkdirphase.push_back(ph);
        ++w.numspinwalks[c];
      }
    }
    w.spinwalk_off[c + 1] = (long long)w.spinwalk.size();
  }
  // spin sets: components grown level by level from the lowest untaken config
  std::vector<char> taken(nc + 1, 0);
  std::vector<std::vector<int>> sets;
  for (int i = 1; i <= nc; ++i) {
    if (taken[i]) continue;
    taken[i] = 1;
    std::vector<int> temp{i};
    size_t prev = 0, cur = 1;
    while (true) {
      size_t add = 0;
      for (size_t j = prev; j < cur; ++j) {
        const int cj = temp[j] - 1;
        for (long long k = w.spinwalk_off[cj]; k < w.spinwalk_off[cj + 1]; ++k) {
          const int t = w.spinwalk[k];
          if (std::find(temp.begin(), temp.begin() + (cur + add), t) == temp.begin() + (cur + add)) {
            SG_CHECK(!taken[t], SINCGPU_ESTATE, "spin set overlap at config %d", t);
            temp.push_back(t);
            taken[t] = 1;
            ++add;
          }
        }
      }
      prev = cur;
      cur += add;
      if (add == 0) break;
    }
    sets.push_back(std::move(temp));
  }
  // S^2 per set, eigenvectors with S(S+1), projector
  const double target = srv / 2.0 * (srv / 2.0 + 1.0);
  w.spinset_off.assign(1, 0);
  w.spinsets.clear();
  w.spinsetrank.clear();
  w.spinproj_off.assign(1, 0);
  w.spinproj.clear();
  w.spin_eliminated.clear();
  w.numspinconfig = 0;
  w.maxspinsetsize = 0;
  std::vector<double> A, V, vals;
  for (const auto& st : sets) {
    const int m = (int)st.size();
    w.maxspinsetsize = std::max(w.maxspinsetsize, m);
    A.assign((size_t)m * m, 0.0);
    for (int jj = 0; jj < m; ++jj) {
      const int cj = st[jj] - 1;
      A[(size_t)jj * m + jj] = msvalue[cj] * (double)msvalue[cj] / 4.0 + unpaired[cj].size() / 2.0;
      for (int ii = 0; ii < m; ++ii) {
        if (ii == jj) continue;
        for (long long k = w.spinwalk_off[cj]; k < w.spinwalk_off[cj + 1]; ++k)
          if (w.spinwalk[k] == st[ii]) {
            A[(size_t)ii * m + jj] = w.spinwalkdirphase[k];
            break;
          }
      }
    }
    jacobi_eigen(m, A, V, vals);
    std::vector<int> keep;
    for (int k = 0; k < m; ++k)
      if (std::fabs(vals[k] - target) < 1e-3) keep.push_back(k);
    if (keep.empty()) {
      w.spin_eliminated.insert(w.spin_eliminated.end(), st.begin(), st.end());
      continue;
    }
    w.spinsets.insert(w.spinsets.end(), st.begin(), st.end());
    w.spinset_off.push_back((long long)w.spinsets.size());
    w.spinsetrank.push_back((int)keep.size());
    w.numspinconfig += (long long)keep.size();
    const size_t base = w.spinproj.size();
    w.spinproj.resize(base + (size_t)m * m, 0.0);
    for (int ii = 0; ii < m; ++ii)
      for (int jj = 0; jj < m; ++jj) {
        double s = 0.0;
        for (int k : keep) s += V[(size_t)ii * m + k] * V[(size_t)jj * m + k];
        w.spinproj[base + (size_t)ii * m + jj] = s;
      }
    w.spinproj_off.push_back((long long)w.spinproj.size());
  }
  return SINCGPU_OK;
}

}  // namespace sincgpu
