// CI side of the orbital RHS on the device, over the uploaded walk tables:
//   1-RDM            getdenmat00   MCTDH.SRC/denmat.f90:177-274
//   regularised inv  invmatsmooth  MCTDH.SRC/utils.f90:533-611 (denreg, denmat.f90:353)
//   2-RDM            get_tworeducedx MCTDH.SRC/mean.f90:14-152
//   one-body matels  sparseops_matel / pot_matel / pulse_matel MCTDH.SRC/matel.f90:113-293
//   sparse matrices  assemble_sparsemats MCTDH.SRC/matel.f90:393-475, 674-729
//   sigma            sparsesparsemult_byproc MCTDH.SRC/walkmult.f90:735-907
// All reductions are gathers in a fixed order (no atomics), so results are
// bit-identical from run to run.  The RDM gathers use per-element contribution
// lists built once on the host when the tables are attached.
#include <algorithm>
#include <cmath>
#include <vector>
#include "context.hpp"
#include "jacobi_svd.cuh"
#include "walks.hpp"

namespace sincgpu {

// ---------------------------------------------------------------------------
// host: per-element contribution lists and hop ranges, uploaded once
// ---------------------------------------------------------------------------


int ci_attach(Ctx& c, const Walks& w) {
  SG_CHECK(w.nspf == c.nspf, SINCGPU_EINVAL, "walk tables for %d orbitals, context has %d", w.nspf, c.nspf);
  CIState& s = c.ci;
  const int n = w.nspf, nc = w.numconfig;
  s.nc = nc;
  s.nsh = (long long)w.singlehop.size();
  s.ndh = (long long)w.doublehop.size();
  // 1-RDM lists: element (ispf,jspf) <- (config1, config2, phase) for every single walk
  {
    const long long nw = w.scol[nc];
    std::vector<long long> off((size_t)n * n + 1, 0);
    for (long long k = 0; k < nw; ++k)
      off[(w.singlewalkopspf[2 * k] - 1) + (size_t)n * (w.singlewalkopspf[2 * k + 1] - 1) + 1]++;
    for (size_t e = 0; e < (size_t)n * n; ++e) off[e + 1] += off[e];
    std::vector<int2> ent(nw);
    std::vector<long long> pos(off.begin(), off.end() - 1);
    for (int c1 = 0; c1 < nc; ++c1)
      for (long long k = w.scol[c1]; k < w.scol[c1 + 1]; ++k) {
        size_t e = (w.singlewalkopspf[2 * k] - 1) + (size_t)n * (w.singlewalkopspf[2 * k + 1] - 1);
        ent[pos[e]++] = make_int2(c1, w.singlewalkdirphase[k] > 0 ? w.singlewalk[k] - 1 : -w.singlewalk[k]);
      }
    SG_TRY(dupload(c, (void**)&s.den_off, off.data(), sizeof(long long) * off.size()));
    SG_TRY(dupload(c, (void**)&s.den_ent, ent.data(), sizeof(int2) * ent.size()));
  }
  // 2-RDM lists: each double walk feeds (d1,d2,d3,d4) and (d3,d4,d1,d2)
  {
    const long long nw = w.dcol[nc];
    const size_t n4 = (size_t)n * n * n * n;
    auto e1 = [&](long long k) {
      const int* d = &w.doublewalkdirspf[4 * k];
      return (size_t)(d[0] - 1) + n * ((size_t)(d[1] - 1) + n * ((size_t)(d[2] - 1) + (size_t)n * (d[3] - 1)));
    };
    auto e2 = [&](long long k) {
      const int* d = &w.doublewalkdirspf[4 * k];
      return (size_t)(d[2] - 1) + n * ((size_t)(d[3] - 1) + n * ((size_t)(d[0] - 1) + (size_t)n * (d[1] - 1)));
    };
    std::vector<long long> off(n4 + 1, 0);
    for (long long k = 0; k < nw; ++k) {
      off[e1(k) + 1]++;
      off[e2(k) + 1]++;
    }
    for (size_t e = 0; e < n4; ++e) off[e + 1] += off[e];
    std::vector<int2> ent(2 * nw);
    std::vector<long long> pos(off.begin(), off.end() - 1);
    for (int c1 = 0; c1 < nc; ++c1)
      for (long long k = w.dcol[c1]; k < w.dcol[c1 + 1]; ++k) {
        int2 v = make_int2(c1, w.doublewalkdirphase[k] > 0 ? w.doublewalk[k] - 1 : -w.doublewalk[k]);
        ent[pos[e1(k)]++] = v;
        ent[pos[e2(k)]++] = v;
      }
    SG_TRY(dupload(c, (void**)&s.tal_off, off.data(), sizeof(long long) * off.size()));
    SG_TRY(dupload(c, (void**)&s.tal_ent, ent.data(), sizeof(int2) * ent.size()));
  }
  // walks (compact) and hop ranges for assembly and sigma
  {
    const long long ns = w.scol[nc], nd = w.dcol[nc];
    std::vector<int> sidx(ns), didx(nd);  // packed indices with the phase in the sign
    for (long long k = 0; k < ns; ++k) {
      int e = (w.singlewalkopspf[2 * k] - 1) + n * (w.singlewalkopspf[2 * k + 1] - 1);
      sidx[k] = w.singlewalkdirphase[k] > 0 ? e : -(e + 1);
    }
    for (long long k = 0; k < nd; ++k) {
      const int* d = &w.doublewalkdirspf[4 * k];
      int e = (d[0] - 1) + n * ((d[1] - 1) + n * ((d[2] - 1) + n * (d[3] - 1)));
      didx[k] = w.doublewalkdirphase[k] > 0 ? e : -(e + 1);
    }
    SG_TRY(dupload(c, (void**)&s.sidx, sidx.data(), sizeof(int) * ns));
    SG_TRY(dupload(c, (void**)&s.didx, didx.data(), sizeof(int) * nd));
    std::vector<long long> swb(s.nsh), dwb(s.ndh);
    std::vector<int> swn(s.nsh), dwn(s.ndh), shop(s.nsh), dhop(s.ndh);
    for (int c1 = 0; c1 < nc; ++c1) {
      for (long long h = w.singlehop_off[c1]; h < w.singlehop_off[c1 + 1]; ++h) {
        swb[h] = w.scol[c1] + w.singlehopwalkstart[h] - 1;
        swn[h] = w.singlehopwalkend[h] - w.singlehopwalkstart[h] + 1;
        shop[h] = w.singlehop[h] - 1;
      }
      for (long long h = w.doublehop_off[c1]; h < w.doublehop_off[c1 + 1]; ++h) {
        dwb[h] = w.dcol[c1] + w.doublehopwalkstart[h] - 1;
        dwn[h] = w.doublehopwalkend[h] - w.doublehopwalkstart[h] + 1;
        dhop[h] = w.doublehop[h] - 1;
      }
    }
    SG_TRY(dupload(c, (void**)&s.swb, swb.data(), sizeof(long long) * s.nsh));
    SG_TRY(dupload(c, (void**)&s.dwb, dwb.data(), sizeof(long long) * s.ndh));
    SG_TRY(dupload(c, (void**)&s.swn, swn.data(), sizeof(int) * s.nsh));
    SG_TRY(dupload(c, (void**)&s.dwn, dwn.data(), sizeof(int) * s.ndh));
    SG_TRY(dupload(c, (void**)&s.shop, shop.data(), sizeof(int) * s.nsh));
    SG_TRY(dupload(c, (void**)&s.dhop, dhop.data(), sizeof(int) * s.ndh));
    SG_TRY(dupload(c, (void**)&s.shop_off, w.singlehop_off.data(), sizeof(long long) * (nc + 1)));
    SG_TRY(dupload(c, (void**)&s.dhop_off, w.doublehop_off.data(), sizeof(long long) * (nc + 1)));
    dfree(c, s.xpot);
    dfree(c, s.xone);
    dfree(c, s.xz);
    s.xpot = s.xone = s.xz = nullptr;
    SG_TRY(dalloc(c, &s.xpot, sizeof(double2) * std::max(1LL, s.ndh)));
    SG_TRY(dalloc(c, &s.xone, sizeof(double2) * std::max(1LL, s.nsh)));
    SG_TRY(dalloc(c, &s.xz, sizeof(double2) * std::max(1LL, s.nsh)));
  }
  // spin sets and projectors (allspinproject=1), when built
  s.spin = false;
  if (w.spinrestrictval >= 0) {
    std::vector<int> sets0(w.spinsets.size()), elim0(w.spin_eliminated.size());
    for (size_t i = 0; i < sets0.size(); ++i) sets0[i] = w.spinsets[i] - 1;
    for (size_t i = 0; i < elim0.size(); ++i) elim0[i] = w.spin_eliminated[i] - 1;
    s.nspinsets = (int)w.spinsetrank.size();
    s.numspinconfig = w.numspinconfig;
    s.nspinelim = (int)elim0.size();
    s.maxspinset = w.maxspinsetsize;
    SG_CHECK(s.maxspinset <= 4096, SINCGPU_ERANGE, "spin set of %d configurations exceeds 4096",
             s.maxspinset);
    SG_TRY(dupload(c, (void**)&s.sp_set_off, w.spinset_off.data(), sizeof(long long) * w.spinset_off.size()));
    // empty tables stay null (upload of 0 bytes); the kernel touches only non-empty ones
    SG_TRY(dupload(c, (void**)&s.sp_sets, sets0.data(), sizeof(int) * sets0.size()));
    SG_TRY(dupload(c, (void**)&s.sp_proj_off, w.spinproj_off.data(), sizeof(long long) * w.spinproj_off.size()));
    SG_TRY(dupload(c, (void**)&s.sp_proj, w.spinproj.data(), sizeof(double) * w.spinproj.size()));
    SG_TRY(dupload(c, (void**)&s.sp_elim, elim0.data(), sizeof(int) * elim0.size()));
    s.spin = true;
  }
  // the tables are complete before any other stream (a batch graph) reads them
  SG_CUDA(cudaStreamSynchronize(c.stream));
  s.attached = true;
  s.assembled = false;
  return SINCGPU_OK;
}

// basis_project with allspinproject=1 (configspin_project_general,
// MCTDH.SRC/spin.f90:339-375): a(set) <- P_set a(set) for every kept spin set,
// one CTA per set; configurations of eliminated (rank-0) sets become zero.
__global__ void __launch_bounds__(256) spin_project_kernel(const long long* __restrict__ set_off,
                                                           const int* __restrict__ sets,
                                                           const long long* __restrict__ proj_off,
                                                           const double* __restrict__ proj, int nsets,
                                                           const int* __restrict__ elim, int nelim,
                                                           double2* __restrict__ a) {
  extern __shared__ double2 v[];
  const int sidx = blockIdx.x;
  if (sidx >= nsets) {  // trailing CTAs zero the eliminated configurations
    for (int i = (sidx - nsets) * blockDim.x + threadIdx.x; i < nelim; i += (gridDim.x - nsets) * blockDim.x)
      a[elim[i]] = make_double2(0.0, 0.0);
    return;
  }
  const long long b = set_off[sidx];
  const int m = (int)(set_off[sidx + 1] - b);
  for (int i = threadIdx.x; i < m; i += blockDim.x) v[i] = a[sets[b + i]];
  __syncthreads();
  const double* P = proj + proj_off[sidx];
  for (int i = threadIdx.x; i < m; i += blockDim.x) {
    double2 acc = make_double2(0.0, 0.0);
    for (int j = 0; j < m; ++j) {
      const double p = P[(long long)i * m + j];
      acc.x = fma(p, v[j].x, acc.x);
      acc.y = fma(p, v[j].y, acc.y);
    }
    a[sets[b + i]] = acc;
  }
}

int ci_spin_project(Ctx& c, double2* a) {
  CIState& s = c.ci;
  SG_CHECK(s.attached && s.spin, SINCGPU_ESTATE, "no spin projectors attached (build them with sincgpu_walks_spin)");
  const int zb = s.nspinelim > 0 ? std::min(ceil_div(s.nspinelim, 256), 64) : 0;
  if (s.nspinsets + zb == 0) return SINCGPU_OK;
  // process-wide attribute, one fixed value, set once (thread-safe static init)
  static const cudaError_t attr = cudaFuncSetAttribute(
      spin_project_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)(sizeof(double2) * 4096));
  SG_CUDA(attr);
  spin_project_kernel<<<s.nspinsets + zb, 256, sizeof(double2) * std::max(1, s.maxspinset), c.stream>>>(
      s.sp_set_off, s.sp_sets, s.sp_proj_off, s.sp_proj, s.nspinsets, s.sp_elim, s.nspinelim, a);
  SG_LAUNCHED();
  return SINCGPU_OK;
}

void CIState::release(cudaStream_t stream) {
  void* ptrs[] = {den_off, den_ent, tal_off, tal_ent, sidx, didx, swb, dwb, swn, dwn,
                  shop, dhop, shop_off, dhop_off, xpot, xone, xz,
                  sp_set_off, sp_sets, sp_proj_off, sp_proj, sp_elim};
  for (void* p : ptrs)
    if (p) cudaFreeAsync(p, stream);
  *this = CIState();
}

// ---------------------------------------------------------------------------
// RDM gathers
// ---------------------------------------------------------------------------
__device__ __forceinline__ double2 warp_sum(double2 v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    v.x += __shfl_down_sync(0xffffffffu, v.x, o);
    v.y += __shfl_down_sync(0xffffffffu, v.y, o);
  }
  return v;
}

// denmat(e) = sum phase * conj(A(c2)) * A(c1)           (denmat.f90:227-236)
// tally(e)  = sum phase * conj(A1(c1)) * A2(c2)         (mean.f90:72-90)
template <bool DEN>
__global__ void __launch_bounds__(128) rdm_gather_kernel(const long long* __restrict__ off,
                                                         const int2* __restrict__ ent,
                                                         const double2* __restrict__ a1,
                                                         const double2* __restrict__ a2, long long nel,
                                                         double2* __restrict__ out) {
  const long long e = blockIdx.x * 4LL + (threadIdx.x >> 5);
  const int lane = threadIdx.x & 31;
  if (e >= nel) return;
  double2 acc = make_double2(0.0, 0.0);
  for (long long k = off[e] + lane; k < off[e + 1]; k += 32) {
    const int2 v = ent[k];
    const int c2 = v.y >= 0 ? v.y : -v.y - 1;
    const double ph = v.y >= 0 ? 1.0 : -1.0;
    double2 t = DEN ? cmulc(a1[v.x], a1[c2]) : cmulc(a2[c2], a1[v.x]);
    acc.x = fma(ph, t.x, acc.x);
    acc.y = fma(ph, t.y, acc.y);
  }
  acc = warp_sum(acc);
  if (lane == 0) out[e] = acc;
}

// Fast path of the regularised inverse: Gauss-Jordan with partial pivoting on
// [A | I] (n <= 32) by one CTA of 256 threads: warp 0 finds the pivot (largest
// modulus, lowest row on ties), then the row swap, the pivot-row scaling and the
// elimination are spread over all threads (one element each, n * 2n elements).
// Same arithmetic per element as a one-row-per-lane elimination.  When every
// singular value is far above the regularisation threshold the SVD formula is
// the plain inverse, and sigma_min >= 1/||A^-1||_F certifies that; need_svd is
// set otherwise.
__global__ void __launch_bounds__(256) inverse_gj_kernel(const double2* __restrict__ A_in, int n,
                                                         double safe_sigma, double2* __restrict__ inv,
                                                         int* __restrict__ need_svd) {
  __shared__ double2 M[32][65];
  __shared__ double2 fcol[32];
  __shared__ int piv, sing;
  __shared__ double fro_part[8];
  const int tid = threadIdx.x, n2 = 2 * n;
  for (int e = tid; e < n * n2; e += 256) {
    const int r = e / n2, j = e - r * n2;
    M[r][j] = j < n ? A_in[r + n * j] : make_double2(j - n == r ? 1.0 : 0.0, 0.0);
  }
  if (tid == 0) sing = 0;
  __syncthreads();
  for (int k = 0; k < n; ++k) {
    if (tid < 32) {
      const int r = tid;
      double mag = (r >= k && r < n) ? M[r][k].x * M[r][k].x + M[r][k].y * M[r][k].y : -1.0;
      int arg = r;
      for (int o = 16; o > 0; o >>= 1) {  // argmax, lowest row on ties
        const double m2 = __shfl_xor_sync(0xffffffffu, mag, o);
        const int a2 = __shfl_xor_sync(0xffffffffu, arg, o);
        if (m2 > mag || (m2 == mag && a2 < arg)) {
          mag = m2;
          arg = a2;
        }
      }
      if (r == 0) {
        piv = arg;
        if (mag <= 0.0) sing = 1;
      }
    }
    __syncthreads();
    if (sing) break;
    const int arg = piv;
    if (arg != k)
      for (int j = tid; j < n2; j += 256) {
        const double2 t = M[k][j];
        M[k][j] = M[arg][j];
        M[arg][j] = t;
      }
    __syncthreads();
    const double2 pv = M[k][k];
    const double pm = pv.x * pv.x + pv.y * pv.y;
    const double2 pinv = make_double2(pv.x / pm, -pv.y / pm);
    if (tid < n) fcol[tid] = M[tid][k];
    __syncthreads();
    for (int j = tid; j < n2; j += 256) M[k][j] = cmul(M[k][j], pinv);
    __syncthreads();
    for (int e = tid; e < n * n2; e += 256) {
      const int r = e / n2, j = e - r * n2;
      if (r != k) M[r][j] = csub(M[r][j], cmul(fcol[r], M[k][j]));
    }
    __syncthreads();
  }
  double fro = 0.0;
  if (!sing)
    for (int e = tid; e < n * n; e += 256) {
      const int r = e % n, j = e / n;  // column-major output
      const double2 v = M[r][n + j];
      fro += v.x * v.x + v.y * v.y;
      inv[r + n * j] = v;
    }
  for (int o = 16; o > 0; o >>= 1) fro += __shfl_xor_sync(0xffffffffu, fro, o);
  if ((tid & 31) == 0) fro_part[tid >> 5] = fro;
  __syncthreads();
  if (tid == 0) {
    double f = 0.0;
    for (int w = 0; w < 8; ++w) f += fro_part[w];
    *need_svd = (sing || !(f * safe_sigma * safe_sigma < 1.0)) ? 1 : 0;
  }
}

// Regularised inverse of an n x n complex matrix by one-sided (Hestenes) Jacobi
// SVD: A = U S V^H, inv = V f(S) U^H with f(s) = 1/s, 1/tol below tol, 0 at 0.
// One warp, lane k owns row k.  Skipped when `need_svd` is 0.
__global__ void __launch_bounds__(32) invmatsmooth_kernel(const double2* __restrict__ A_in, int n,
                                                          double tol, double2* __restrict__ inv,
                                                          const int* __restrict__ need_svd) {
  if (need_svd && *need_svd == 0) return;
  __shared__ double2 A[32 * 32], V[32 * 32];
  __shared__ double sv[32];
  const int k = threadIdx.x;
  hestenes_svd_warp(A_in, n, A, V, sv);
  // inv(i,j) = sum_m V(i,m) f(s_m) conj(U(j,m)),  U(j,m) = A(j,m)/s_m
  if (k < n) {
    for (int j = 0; j < n; ++j) {
      double2 acc = make_double2(0.0, 0.0);
      for (int m = 0; m < n; ++m) {
        const double s = sv[m];
        if (s == 0.0) continue;
        const double f = (s < tol ? 1.0 / tol : 1.0 / s) / s;
        double2 t = cmulc(V[k + 32 * m], A[j + 32 * m]);  // V(i,m) conj(A(j,m))
        acc.x = fma(f, t.x, acc.x);
        acc.y = fma(f, t.y, acc.y);
      }
      inv[k + n * j] = acc;
    }
  }
}

int ci_denmat(Ctx& c, const double2* avec, double2* denmat, double2* invdenmat, double denreg) {
  CIState& s = c.ci;
  SG_CHECK(s.attached, SINCGPU_ESTATE, "no walk tables attached");
  const int n = c.nspf;
  ProfScope ps(c, ST_CI);
  rdm_gather_kernel<true><<<ceil_div((long long)n * n, 4), 128, 0, c.stream>>>(s.den_off, s.den_ent, avec,
                                                                              avec, (long long)n * n, denmat);
  SG_LAUNCHED();
  if (invdenmat) {
    SG_TRY(c.ws_ci2.ensure(sizeof(double2) * n * n + 256));
    int* flag = (int*)((char*)c.ws_ci2.ptr + sizeof(double2) * n * n);
    // plain inverse is the SVD formula when sigma_min >= 1e-6 >> denreg
    inverse_gj_kernel<<<1, 256, 0, c.stream>>>(denmat, n, std::max(1e-6, 1e4 * denreg), invdenmat, flag);
    SG_LAUNCHED();
    invmatsmooth_kernel<<<1, 32, 0, c.stream>>>(denmat, n, denreg, invdenmat, flag);
    SG_LAUNCHED();
  }
  return SINCGPU_OK;
}

int ci_tally(Ctx& c, const double2* a1, const double2* a2, double2* tally) {
  CIState& s = c.ci;
  SG_CHECK(s.attached, SINCGPU_ESTATE, "no walk tables attached");
  const long long n4 = (long long)c.nspf * c.nspf * c.nspf * c.nspf;
  ProfScope ps(c, ST_CI);
  rdm_gather_kernel<false><<<ceil_div(n4, 4), 128, 0, c.stream>>>(s.tal_off, s.tal_ent, a1, a2, n4, tally);
  SG_LAUNCHED();
  return SINCGPU_OK;
}

// ---------------------------------------------------------------------------
// one-body matrix elements: M(i,j) = sum_x conj(phi_i) (op phi_j)
//   pot (mult_pot), KE (mult_ke), z (lenmultiply z part)
// ---------------------------------------------------------------------------
constexpr int OX = 32;
__global__ void __launch_bounds__(256) onebody_kernel(const double2* __restrict__ phi,
                                                      const double2* __restrict__ kephi,
                                                      const double* __restrict__ pot,
                                                      const double* __restrict__ zdip, int n, long long G,
                                                      long long xper, double2* __restrict__ part) {
  __shared__ double2 sp[32][OX], sk[32][OX];
  __shared__ double spot[OX], sz[OX];
  const long long xb = blockIdx.x * xper, xe = min(G, xb + xper);
  const int nn = n * n;
  double2 a1[4], a2[4], a3[4];
#pragma unroll
  for (int r = 0; r < 4; ++r) a1[r] = a2[r] = a3[r] = make_double2(0.0, 0.0);
  for (long long x0 = xb; x0 < xe; x0 += OX) {
    __syncthreads();
    for (int i = threadIdx.x; i < n * OX; i += blockDim.x) {
      int o = i / OX, k = i % OX;
      long long x = x0 + k;
      bool ok = x < xe;
      sp[o][k] = ok ? phi[(long long)o * G + x] : make_double2(0, 0);
      sk[o][k] = ok ? kephi[(long long)o * G + x] : make_double2(0, 0);
    }
    for (int k = threadIdx.x; k < OX; k += blockDim.x) {
      long long x = x0 + k;
      spot[k] = x < xe ? pot[x] : 0.0;
      sz[k] = x < xe ? zdip[x] : 0.0;
    }
    __syncthreads();
#pragma unroll
    for (int r = 0; r < 4; ++r) {
      int e = threadIdx.x + 256 * r;
      if (e < nn) {
        int i = e % n, j = e / n;  // M(i,j) = <phi_i| op |phi_j>
        for (int k = 0; k < OX; ++k) {
          double2 t = cmulc(sp[j][k], sp[i][k]);  // conj(phi_i) phi_j
          a1[r].x = fma(spot[k], t.x, a1[r].x);
          a1[r].y = fma(spot[k], t.y, a1[r].y);
          a3[r].x = fma(sz[k], t.x, a3[r].x);
          a3[r].y = fma(sz[k], t.y, a3[r].y);
          double2 u = cmulc(sk[j][k], sp[i][k]);
          a2[r].x += u.x;
          a2[r].y += u.y;
        }
      }
    }
  }
#pragma unroll
  for (int r = 0; r < 4; ++r) {
    int e = threadIdx.x + 256 * r;
    if (e < nn) {
      double2* p = part + (long long)blockIdx.x * 3 * nn;
      p[e] = a1[r];
      p[nn + e] = a2[r];
      p[2 * nn + e] = a3[r];
    }
  }
}

__global__ void __launch_bounds__(128) onebody_reduce_kernel(const double2* __restrict__ partial, int nblk,
                                                             int nel, double2* __restrict__ out) {
  __shared__ double2 red[128];
  const int e = blockIdx.x;
  double2 s = make_double2(0.0, 0.0);
  for (int b = threadIdx.x; b < nblk; b += 128) s = cadd(s, partial[(long long)b * nel + e]);
  red[threadIdx.x] = s;
  __syncthreads();
  for (int w = 64; w > 0; w >>= 1) {
    if (threadIdx.x < w) red[threadIdx.x] = cadd(red[threadIdx.x], red[threadIdx.x + w]);
    __syncthreads();
  }
  if (threadIdx.x == 0) out[e] = red[0];
}

int ci_onebody(Ctx& c, const double2* phi, double2* mats /* potmat, kemat, zmat: 3 n^2 */) {
  const int n = c.nspf;
  const long long G = c.G;
  const int nblk = 2 * 148;
  const long long xper = ((G + nblk - 1) / nblk + OX - 1) / OX * OX;
  const int nb = ceil_div(G, xper);
  SG_TRY(c.ws_ci.ensure(sizeof(double2) * ((size_t)n * G + (size_t)nb * 3 * n * n)));
  double2* kephi = (double2*)c.ws_ci.ptr;
  double2* part = kephi + (size_t)n * G;
  SG_TRY(mult_ke(c, phi, kephi, n, false, 0.0));
  ProfScope ps(c, ST_CI);
  onebody_kernel<<<nb, 256, 0, c.stream>>>(phi, kephi, c.d_pot, c.d_zdip, n, G, xper, part);
  SG_LAUNCHED();
  onebody_reduce_kernel<<<3 * n * n, 128, 0, c.stream>>>(part, nb, 3 * n * n, mats);
  SG_LAUNCHED();
  return SINCGPU_OK;
}

// ---------------------------------------------------------------------------
// assembled sparse matrices (per config1 and hop) and sigma
// ---------------------------------------------------------------------------
__global__ void assemble_kernel(const long long* __restrict__ wb, const int* __restrict__ wn,
                                const int* __restrict__ idx, long long nhop,
                                const double2* __restrict__ mat1, const double2* __restrict__ mat2,
                                double2* __restrict__ out1, double2* __restrict__ out2) {
  const long long h = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (h >= nhop) return;
  double2 s1 = make_double2(0.0, 0.0), s2 = make_double2(0.0, 0.0);
  const long long b = wb[h];
  for (int k = 0; k < wn[h]; ++k) {
    const int v = idx[b + k];
    const int e = v >= 0 ? v : -v - 1;
    const double ph = v >= 0 ? 1.0 : -1.0;
    const double2 m = mat1[e];
    s1.x = fma(ph, m.x, s1.x);
    s1.y = fma(ph, m.y, s1.y);
    if (mat2) {
      const double2 m2 = mat2[e];
      s2.x = fma(ph, m2.x, s2.x);
      s2.y = fma(ph, m2.y, s2.y);
    }
  }
  out1[h] = s1;
  if (out2) out2[h] = s2;
}

__global__ void add_mats_kernel(const double2* __restrict__ a, const double2* __restrict__ b, int nel,
                                double2* __restrict__ out) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < nel) out[i] = cadd(a[i], b[i]);
}

int ci_assemble(Ctx& c, const double2* twoematel, const double2* mats) {
  CIState& s = c.ci;
  SG_CHECK(s.attached, SINCGPU_ESTATE, "no walk tables attached");
  const int n = c.nspf, nn = n * n;
  SG_TRY(c.ws_ci2.ensure(sizeof(double2) * nn));
  double2* one = (double2*)c.ws_ci2.ptr;
  ProfScope ps(c, ST_CI);
  add_mats_kernel<<<ceil_div(nn, 256), 256, 0, c.stream>>>(mats, mats + nn, nn, one);  // pot + KE
  SG_LAUNCHED();
  if (s.ndh > 0) {
    assemble_kernel<<<ceil_div(s.ndh, 128), 128, 0, c.stream>>>(s.dwb, s.dwn, s.didx, s.ndh, twoematel,
                                                                nullptr, s.xpot, nullptr);
    SG_LAUNCHED();
  }
  if (s.nsh > 0) {
    assemble_kernel<<<ceil_div(s.nsh, 128), 128, 0, c.stream>>>(s.swb, s.swn, s.sidx, s.nsh, one,
                                                                mats + 2 * nn, s.xone, s.xz);
    SG_LAUNCHED();
  }
  s.assembled = true;
  return SINCGPU_OK;
}

// sigma(c1) = const A(c1) + sum_dhops xpot A(dhop) + sum_shops (xone + ez xz) A(shop) + ez nucdip A(c1)
__global__ void __launch_bounds__(128) sigma_kernel(const long long* __restrict__ doff,
                                                    const int* __restrict__ dhop,
                                                    const double2* __restrict__ xpot,
                                                    const long long* __restrict__ soff,
                                                    const int* __restrict__ shop,
                                                    const double2* __restrict__ xone,
                                                    const double2* __restrict__ xz, double ez,
                                                    double diag, const double2* __restrict__ in,
                                                    int nc, double2* __restrict__ out) {
  const int c1 = blockIdx.x * 4 + (threadIdx.x >> 5);
  const int lane = threadIdx.x & 31;
  if (c1 >= nc) return;
  double2 acc = make_double2(0.0, 0.0);
  if (xpot)
    for (long long h = doff[c1] + lane; h < doff[c1 + 1]; h += 32) {
      const double2 t = cmul(xpot[h], in[dhop[h]]);
      acc = cadd(acc, t);
    }
  double2 acc1 = make_double2(0.0, 0.0);
  for (long long h = soff[c1] + lane; h < soff[c1 + 1]; h += 32) {
    double2 m = xone ? xone[h] : make_double2(0.0, 0.0);
    if (ez != 0.0) {
      m.x = fma(ez, xz[h].x, m.x);
      m.y = fma(ez, xz[h].y, m.y);
    }
    acc1 = cadd(acc1, cmul(m, in[shop[h]]));
  }
  acc = warp_sum(acc);
  acc1 = warp_sum(acc1);
  if (lane == 0) {
    const double2 a = in[c1];
    double2 r = make_double2(diag * a.x, diag * a.y);
    r = cadd(r, acc);
    r = cadd(r, acc1);
    out[c1] = r;
  }
}

// z-dipole expectation (dipolesub_one, MCTDH.SRC/dipolesub.f90:20-125, z part):
// <A| Z A> with Z the singles of <phi_i|z|phi_j>, plus nucdip <A|A>; also <A|A>
int ci_dipole_z(Ctx& c, const double2* a, double2* tmp, double nucdipz, double2* dip, double* normsq) {
  CIState& s = c.ci;
  SG_CHECK(s.attached && s.assembled, SINCGPU_ESTATE, "sparse CI matrices not assembled");
  sigma_kernel<<<ceil_div(s.nc, 4), 128, 0, c.stream>>>(s.dhop_off, s.dhop, nullptr, s.shop_off, s.shop, nullptr,
                                                        s.xz, 1.0, 0.0, a, s.nc, tmp);
  SG_LAUNCHED();
  std::vector<double2> ha(s.nc), za(s.nc);
  SG_CUDA(cudaMemcpyAsync(ha.data(), a, sizeof(double2) * s.nc, cudaMemcpyDeviceToHost, c.stream));
  SG_CUDA(cudaMemcpyAsync(za.data(), tmp, sizeof(double2) * s.nc, cudaMemcpyDeviceToHost, c.stream));
  SG_CUDA(cudaStreamSynchronize(c.stream));
  double2 d = make_double2(0.0, 0.0);
  double nn = 0.0;
  for (int i = 0; i < s.nc; ++i) {  // hermdot: sum conj(a) b
    d.x += ha[i].x * za[i].x + ha[i].y * za[i].y;
    d.y += ha[i].x * za[i].y - ha[i].y * za[i].x;
    nn += ha[i].x * ha[i].x + ha[i].y * ha[i].y;
  }
  dip->x = d.x + nucdipz * nn;
  dip->y = d.y;
  *normsq = nn;
  return SINCGPU_OK;
}

int ci_sigma(Ctx& c, const double2* in, double2* out, double constant, double ez, double nucdipz) {
  CIState& s = c.ci;
  SG_CHECK(s.attached && s.assembled, SINCGPU_ESTATE, "sparse CI matrices not assembled");
  ProfScope ps(c, ST_CI);
  sigma_kernel<<<ceil_div(s.nc, 4), 128, 0, c.stream>>>(s.dhop_off, s.dhop, s.xpot, s.shop_off, s.shop, s.xone,
                                                        s.xz, ez, constant + ez * nucdipz, in, s.nc, out);
  SG_LAUNCHED();
  return SINCGPU_OK;
}

}  // namespace sincgpu
