// Pair densities -> Toeplitz/FFT Coulomb solve -> reduced two-electron potentials.
//
// Reference: call_twoe_matel00 (SINCDVR/coreproject.f90:945-1194) builds
// rho_ab = phi1_a * conj(phi2_b) (line 1063), op_tinv (lines 366-537) embeds it at
// octant (1,1,1) of a (2N)^3 grid, circ3d_sub (SINCDVR/toeplitz_subs.f90:561-589)
// convolves it circularly with threed_two and octant (2,2,2) is returned.  That is
// exactly the linear convolution R(x) = sum_y T(x-y) rho(y) for x,y in [0,N)^3.
//
// Here the same convolution runs on a padded P^3 grid (P >= 2N-1, from the table
// in coulomb_kernels.cuh) with the kernel spectrum precomputed once, as five
// global passes (coulomb_kernels.cuh):
//   CX : rho rows -> DFT along x          (N^2 rows, N nonzero inputs each)
//   CY : DFT along y                      (N*P columns, N nonzero inputs each)
//   CZ : DFT along z, * khat, inverse DFT (P^2 columns, only z<N kept)
//   CYI: inverse DFT along y              (N*P columns, only y<N kept)
//   CXI: inverse DFT along x              (N^2 rows, only x<N kept) -> R
// Pruned inputs/outputs never touch memory.  Pairs are processed in chunks whose
// intermediates W1 (N*N*P) and W2 (N*P*P) fit a 2 GB budget: the passes are
// bound by FP64 issue and latency, not by HBM, so few launches over many pairs
// beat L2-sized chunks (measured on the 41^3 / 10-orbital workload: 0.89 ms per
// evaluation with 48 MB chunks of 7 pairs, 0.75 ms with one chunk of all 55).
// The passes run in FP64 (double2) or, with the context option coulomb_fp32,
// in FP32 (float2) with FP64 inputs and outputs.
#include <algorithm>
#include <vector>
#include <cudaTypedefs.h>
#include "coulomb_kernels.cuh"

namespace sincgpu {

int fft_length_for(int min_len, int* p1, int* p2) {
  struct L { int P, a, b; };
  static const L table[] = {
#define SINCGPU_TABLE_ENTRY(P, A, B) {P, A, B},
      SINCGPU_FFT_LENGTHS(SINCGPU_TABLE_ENTRY)
#undef SINCGPU_TABLE_ENTRY
  };
  for (const L& e : table)
    if (e.P >= min_len) {
      if (p1) *p1 = e.a;
      if (p2) *p2 = e.b;
      return e.P;
    }
  return -1;
}

template <class C>
static int coul_dispatch(Ctx& c, const CoulArgs<C>& ca, int np, bool dens, const double2* s1,
                         const double2* s2, double* Rpl, double2* full, bool herm,
                         const CUtensorMap* zmap = nullptr, int* err = nullptr) {
  switch (c.P) {
#define SINCGPU_CASE(P, A, B) \
  case P:                     \
    return coul_launch<A, B, C>(c, ca, np, dens, s1, s2, Rpl, full, herm, zmap, err);
    SINCGPU_FFT_LENGTHS(SINCGPU_CASE)
#undef SINCGPU_CASE
    default:
      set_error("no Coulomb kernels for FFT length %d", c.P);
      return SINCGPU_ERANGE;
  }
}

template <class C>
static const C* roots_of(const Ctx& c);
template <>
const double2* roots_of<double2>(const Ctx& c) { return c.d_roots; }
template <>
const float2* roots_of<float2>(const Ctx& c) { return c.d_roots32; }
template <class C>
static const C* khat_of(const Ctx& c);
template <>
const double2* khat_of<double2>(const Ctx& c) { return c.d_khat; }
template <>
const float2* khat_of<float2>(const Ctx& c) { return c.d_khat32; }

template <class C>
static const typename CplxTraits<C>::Real* khr_of(const Ctx& c);
template <>
const double* khr_of<double2>(const Ctx& c) { return c.d_khr; }
template <>
const float* khr_of<float2>(const Ctx& c) { return c.d_khr32; }
template <class C>
static const typename CplxTraits<C>::Real* khT_of(const Ctx& c);
template <>
const double* khT_of<double2>(const Ctx& c) { return c.d_khT; }
template <>
const float* khT_of<float2>(const Ctx& c) { return c.d_khT32; }

// cuTensorMapEncodeTiled from the driver (no link-time dependency on libcuda).
static PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess)
      p = nullptr;
    return reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
  }();
  return fn;
}

// Tensor map of a W2 chunk for the TMA-staged z pass: [pair < np][z < N][2 P^2
// reals], box (2 TL reals, N, 1).  False when the layout breaks a TMA rule (row
// stride or base not 16-byte aligned, box too tall) or the driver has no encoder.
template <class C>
static bool make_zmap(const Ctx& c, const C* W2, int np, CUtensorMap* map) {
  using R = typename CplxTraits<C>::Real;
  const int N = c.N, P = c.P;
  const int TL = lines_for_ztma<C>(P);
  const size_t plane = sizeof(C) * (size_t)P * P;
  if (plane % 16 || reinterpret_cast<uintptr_t>(W2) % 16 || N > 256 || 2 * TL > 256) return false;
  PFN_cuTensorMapEncodeTiled_v12000 enc = encode_fn();
  if (!enc) return false;
  const cuuint64_t dims[3] = {2ull * P * P, (cuuint64_t)N, (cuuint64_t)np};
  const cuuint64_t strides[2] = {plane, plane * N};
  const cuuint32_t box[3] = {(cuuint32_t)(2 * TL), (cuuint32_t)N, 1};
  const cuuint32_t estr[3] = {1, 1, 1};
  const CUresult r = enc(map, sizeof(R) == 8 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3,
                         const_cast<C*>(W2), dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                         CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                         CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS;
}

template <class C>
static int coul_run_t(Ctx& c, const double2* src1, const double2* src2, const int* h_pa,
                      const int* h_pb, int npair, double* Rpl, double2* full, bool herm, bool dens) {
  const int N = c.N, P = c.P;
  // three-pass form (plane kernel on chip, no W2) where its plane fits shared memory
  int fused = 0;
  if (c.coul_fused != 0 && c.coul_tma <= 0) {
    int p1 = 0, p2 = 0;
    if (fft_length_for(P, &p1, &p2) == P) fused = yzy_cluster<C>(p1, p2, N);
  }
  const long long per_pair = (long long)sizeof(C) * ((long long)N * N * P + (fused ? 0LL : (long long)N * P * P));
  int chunk = c.coul_chunk;
  if (chunk <= 0) {
    const long long budget = kCoulChunkBudget;
    chunk = (int)std::max(1LL, budget / per_pair);
  }
  chunk = std::min(chunk, npair);
  SG_TRY(c.ws_fft.ensure((size_t)per_pair * chunk));
  const int* d_pa = nullptr;
  const int* d_pb = nullptr;
  if (!dens) {
    SG_TRY(cached_ints(c, IC_PA, h_pa, npair, &d_pa));
    SG_TRY(cached_ints(c, IC_PB, h_pb, npair, &d_pb));
  }
  CoulArgs<C> ca{};
  ca.N = N;
  ca.P = P;
  ca.nspf = c.nspf;
  ca.G = c.G;
  ca.roots = roots_of<C>(c);
  ca.khat = khat_of<C>(c);
  ca.khr = khr_of<C>(c);
  ca.W1 = (C*)c.ws_fft.ptr;
  ca.W2 = fused ? nullptr : ca.W1 + (long long)chunk * N * N * P;
  ca.npair_total = npair;
  ca.fused = fused;
  if (fused) {
    SG_TRY(ensure_khT(c, sizeof(C) == 8));
    ca.khT = khT_of<C>(c);
  }
  // TMA-staged z pass: one map over the chunk's W2 (the last, shorter chunk
  // only addresses its first pairs)
  // automatic choice: the plain pass.  With chunks of a few pairs the staged pass
  // was faster for P >= 128 (162: 9.9 -> 8.1 ms per evaluation); with the
  // whole-pair-list chunks the plain pass wins at every measured length (162:
  // 4.8 vs 5.4 ms FP64, 2.1 vs 2.5 ms FP32; 81: 0.16 vs 0.18 ms), its three
  // resident CTAs per SM hiding the W2 latency better than two staged ones
  CUtensorMap zmap;
  const bool want_tma = c.coul_tma > 0 && !fused;
  const bool use_tma = want_tma && make_zmap<C>(c, ca.W2, chunk, &zmap);
  int* err = nullptr;
  if (use_tma) {
    SG_TRY(timeout_flags(c, &err));
    err += 1;
  }
  // orbitals arriving in groups (host-array entry): the hermitian pair list is
  // b-major (a <= b), so the pairs of orbitals below e are its first e (e + 1) / 2;
  // a chunk never crosses a group's end and the first chunk of each group waits for it
  const bool grouped = !dens && herm && c.up_n > 0;
  auto pairs_below = [](int e) { return e * (e + 1) / 2; };
  int g = -1;
  for (int p0 = 0; p0 < npair;) {
    int np = std::min(chunk, npair - p0);
    if (grouped) {
      int gg = 0;
      while (gg < c.up_n - 1 && pairs_below(c.up_end[gg]) <= p0) ++gg;
      if (gg != g) {
        SG_CUDA(cudaStreamWaitEvent(c.stream, c.ev_up[gg], 0));
        g = gg;
      }
      np = std::max(1, std::min(np, pairs_below(c.up_end[gg]) - p0));
    }
    ca.pair0 = p0;
    ca.pa = d_pa ? d_pa + p0 : nullptr;
    ca.pb = d_pb ? d_pb + p0 : nullptr;
    SG_TRY(coul_dispatch(c, ca, np, dens, src1, src2, Rpl, full, herm, use_tma ? &zmap : nullptr, err));
    p0 += np;
  }
  // every group has been waited for (the last group ends at the last orbital)
  if (grouped && g != c.up_n - 1) SG_CUDA(cudaStreamWaitEvent(c.stream, c.ev_up[c.up_n - 1], 0));
  return SINCGPU_OK;
}

static int coul_run(Ctx& c, const double2* src1, const double2* src2, const int* h_pa,
                    const int* h_pb, int npair, double* Rpl, double2* full, bool herm, bool dens) {
  if (c.coul_fp32) {
    SG_TRY(ensure_fp32_tables(c));
    return coul_run_t<float2>(c, src1, src2, h_pa, h_pb, npair, Rpl, full, herm, dens);
  }
  return coul_run_t<double2>(c, src1, src2, h_pa, h_pb, npair, Rpl, full, herm, dens);
}

int coulomb_pairs(Ctx& c, const double2* phi1, const double2* phi2, const int* h_pa,
                  const int* h_pb, int npair, double* Rpl, double2* full, bool herm) {
  return coul_run(c, phi1, phi2, h_pa, h_pb, npair, Rpl, full, herm, false);
}

int coulomb_dens(Ctx& c, const double2* dens, int m, double2* red) {
  return coul_run(c, dens, nullptr, nullptr, nullptr, m, nullptr, red, false, true);
}

// op_tinv on explicit densities with caller-provided scratch: no allocation.
// The densities are processed in chunks that fit `scratch_bytes`.
template <class C>
static int coulomb_dens_scratch_t(Ctx& c, const double2* dens, int m, double2* red, void* scratch,
                                  size_t scratch_bytes) {
  const int N = c.N, P = c.P;
  const size_t per_dens = sizeof(C) * ((size_t)N * N * P + (size_t)N * P * P);
  SG_CHECK(per_dens <= scratch_bytes, SINCGPU_ERANGE,
           "one density on a %d^3 grid (FFT length %d) needs %zu bytes of scratch; the fixed "
           "scratch holds %zu bytes", N, P, per_dens, scratch_bytes);
  const int chunk = (int)std::min<size_t>(scratch_bytes / per_dens, (size_t)m);
  CoulArgs<C> ca{};
  ca.N = N;
  ca.P = P;
  ca.nspf = c.nspf;
  ca.G = c.G;
  ca.roots = roots_of<C>(c);
  ca.khat = khat_of<C>(c);
  ca.khr = khr_of<C>(c);
  ca.W1 = (C*)scratch;
  ca.W2 = ca.W1 + (size_t)chunk * N * N * P;
  ca.npair_total = m;
  ca.pa = nullptr;
  ca.pb = nullptr;
  for (int p0 = 0; p0 < m; p0 += chunk) {
    ca.pair0 = p0;
    SG_TRY(coul_dispatch(c, ca, std::min(chunk, m - p0), true, dens, nullptr, nullptr, red, false));
  }
  return SINCGPU_OK;
}

int coulomb_dens_scratch(Ctx& c, const double2* dens, int m, double2* red, double2* scratch,
                         size_t scratch_bytes) {
  if (c.coul_fp32) {
    SG_CHECK(c.d_khat32 && c.d_roots32 && c.d_khr32, SINCGPU_ESTATE, "FP32 Coulomb tables are missing");
    return coulomb_dens_scratch_t<float2>(c, dens, m, red, scratch, scratch_bytes);
  }
  return coulomb_dens_scratch_t<double2>(c, dens, m, red, scratch, scratch_bytes);
}

}  // namespace sincgpu
