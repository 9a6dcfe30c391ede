// Tensor-core (tcgen05, kind::tf32) contractions of the precision form.
//
// C[m][n] = sum_k A[m][k] B[n][k] with FP64 inputs split as v = hi + lo (both
// tf32) and three MMAs per K step, hi*hi + hi*lo + lo*hi, accumulated in FP32 in
// tensor memory ("3xTF32": about 2^-21 relative per product, the FP32 level of the
// precision form's Coulomb potentials).  One CTA of 256 threads owns a 128-row x
// NT-column tile (NT <= 256, a multiple of 16): the threads stage K chunks of A
// and B into shared memory (two stages, the split done while staging), thread 0
// issues the MMAs and commits them to an mbarrier, and the epilogue reads the
// accumulator back from tensor memory (a row per thread, half the columns per
// warpgroup).
//
// Used for get_reducedpot0's contraction (SRC/mean.f90:556-558, reducedpot =
// R x Gamma) when the context option contract_tf32 is set.
#include <algorithm>
#include "context.hpp"
#include "tma.cuh"
#include "umma.cuh"
#include "../../include/sincgpu.h"

namespace sincgpu {

namespace {

constexpr uint32_t kWaitLimit = 1u << 26;  // mbarrier polls before a wait is declared stuck

// Generic epilogue: C[m * ldm + n * ldn] = D[m][n] (FP64), for the self test.
struct StoreEpi {
  double* C;
  long long ldm, ldn;
  __device__ void operator()(long long m, int n, float v) const { C[m * ldm + (long long)n * ldn] = (double)v; }
};

// reducedpot epilogue: columns 2t, 2t+1 are Re, Im of the orbital pair t; with
// `tmap` only pairs kk <= ii are computed and reducedpot(x, ii, kk) is the
// conjugate of reducedpot(x, kk, ii).
struct RedpotEpi {
  double2* out;
  long long G;
  const int* tmap;
  int n;
};

// Row m of A starts at (m % Mlo) lam + (m / Mlo) lam2 (two-level rows: the lines
// of a 3-D grid along one axis); element k of the row is k lak further.
struct ARows {
  long long lam, Mlo, lam2, lak;
  __device__ __forceinline__ long long row(long long m) const { return (m % Mlo) * lam + (m / Mlo) * lam2; }
};

// kinetic epilogue: element (m, j) of one axis's contraction at out[row(m) + j lak]
// (the same addressing as the input lines); `first` writes it, adding the
// potential and z-field terms times the input when `extra`, otherwise it adds
struct KeEpi {
  double* out;
  const double* in;
  ARows ar;
  int first, extra;
  const double* pot;
  const double* zdip;
  double zfield;
  long long G;
};

template <int KC>
struct TileSmem {
  static constexpr int kA = KC * 128;  // u32 per A tile (hi or lo)
  __host__ __device__ static constexpr size_t bytes(int NT) {
    return sizeof(uint32_t) * 2 * (2 * (size_t)kA + 2 * (size_t)KC * NT);
  }
};

// Stages rows m0.. of A and columns n0.. of B, K range [k0, k0 + KC), split into
// tf32 hi / lo, in the chunk-major K-major core-matrix layout of umma.cuh.  Warps
// 0-3 stage A (one row per thread), warps 4-7 stage B; every thread issues all of
// its global loads before the first split, so a warp has KC loads in flight.
template <int KC>
__device__ __forceinline__ void stage_tile(uint32_t* base, int NT, const double* __restrict__ A, ARows ar,
                                           long long M, long long m0, const double* __restrict__ B,
                                           long long lbn, long long lbk, int Ntot, int n0, int K, int k0) {
  uint32_t* Ahi = base;
  uint32_t* Alo = Ahi + TileSmem<KC>::kA;
  uint32_t* Bhi = Alo + TileSmem<KC>::kA;
  uint32_t* Blo = Bhi + KC * NT;
  const int tid = threadIdx.x;
  if (tid < 128) {
    const long long m = m0 + tid;
    const long long rb = m < M ? ar.row(m) : 0;
    double v[KC];
#pragma unroll
    for (int k = 0; k < KC; ++k) v[k] = (m < M && k0 + k < K) ? A[rb + (long long)(k0 + k) * ar.lak] : 0.0;
#pragma unroll
    for (int c = 0; c < KC / 4; ++c) {
      uint4 h, l;
      umma::split_tf32(v[4 * c + 0], h.x, l.x);
      umma::split_tf32(v[4 * c + 1], h.y, l.y);
      umma::split_tf32(v[4 * c + 2], h.z, l.z);
      umma::split_tf32(v[4 * c + 3], h.w, l.w);
      *reinterpret_cast<uint4*>(Ahi + (c * 128 + tid) * 4) = h;
      *reinterpret_cast<uint4*>(Alo + (c * 128 + tid) * 4) = l;
    }
  } else {
    constexpr int kMaxIt = KC * 256 / 4 / 128;  // (KC / 4) * NT / 128 for NT <= 256
    const int t2 = tid - 128;
    const int nit = ((KC / 4) * NT + 127) / 128;
    double v[kMaxIt][4];
#pragma unroll
    for (int it = 0; it < kMaxIt; ++it) {
      const int idx = t2 + 128 * it;
      const int c = idx / NT, r = idx - c * NT;
      const int nn = n0 + r;
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        const int k = k0 + 4 * c + j;
        v[it][j] = (it < nit && c < KC / 4 && nn < Ntot && k < K) ? B[(long long)nn * lbn + (long long)k * lbk]
                                                                 : 0.0;
      }
    }
#pragma unroll
    for (int it = 0; it < kMaxIt; ++it) {
      const int idx = t2 + 128 * it;
      const int c = idx / NT, r = idx - c * NT;
      if (it < nit && c < KC / 4) {
        uint4 h, l;
        umma::split_tf32(v[it][0], h.x, l.x);
        umma::split_tf32(v[it][1], h.y, l.y);
        umma::split_tf32(v[it][2], h.z, l.z);
        umma::split_tf32(v[it][3], h.w, l.w);
        *reinterpret_cast<uint4*>(Bhi + (c * NT + r) * 4) = h;
        *reinterpret_cast<uint4*>(Blo + (c * NT + r) * 4) = l;
      }
    }
  }
}

template <class Epi>
__device__ __forceinline__ void apply_epi(const Epi& e, long long m, long long M, int n, int Ntot,
                                          const float (&v)[8]);

template <>
__device__ __forceinline__ void apply_epi<StoreEpi>(const StoreEpi& e, long long m, long long M, int n, int Ntot,
                                                    const float (&v)[8]) {
  if (m >= M) return;
#pragma unroll
  for (int j = 0; j < 8; ++j)
    if (n + j < Ntot) e(m, n + j, v[j]);
}

template <>
__device__ __forceinline__ void apply_epi<KeEpi>(const KeEpi& e, long long m, long long M, int n, int Ntot,
                                                 const float (&v)[8]) {
  if (m >= M) return;
  const long long rb = e.ar.row(m);
#pragma unroll
  for (int j = 0; j < 8; ++j) {
    if (n + j >= Ntot) break;
    const long long a = rb + (long long)(n + j) * e.ar.lak;
    if (e.first) {
      double w = (double)v[j];
      if (e.extra) {
        const long long gidx = (a >> 1) % e.G;  // grid point of the complex element
        w = fma(e.pot[gidx] + e.zfield * e.zdip[gidx], e.in[a], w);
      }
      e.out[a] = w;
    } else {
      e.out[a] += (double)v[j];
    }
  }
}

template <>
__device__ __forceinline__ void apply_epi<RedpotEpi>(const RedpotEpi& e, long long m, long long M, int n,
                                                     int Ntot, const float (&v)[8]) {
  if (m >= M) return;
#pragma unroll
  for (int j = 0; j < 8; j += 2) {
    const int col = n + j;
    if (col >= Ntot) break;
    const int t = col / 2;
    const double2 z = make_double2((double)v[j], (double)v[j + 1]);
    if (e.tmap) {
      const int kk = e.tmap[2 * t], ii = e.tmap[2 * t + 1];
      e.out[(long long)(kk + e.n * ii) * e.G + m] = z;
      if (kk != ii) e.out[(long long)(ii + e.n * kk) * e.G + m] = make_double2(z.x, -z.y);
    } else {
      e.out[(long long)t * e.G + m] = z;
    }
  }
}

template <int KC, class Epi>
__global__ void __launch_bounds__(256) gemm_tf32x3_kernel(const double* __restrict__ A, ARows ar, long long M,
                                                          const double* __restrict__ B, long long lbn,
                                                          long long lbk, int Ntot, int K, int NT,
                                                          uint32_t tmem_cols, Epi epi, int* __restrict__ err) {
  extern __shared__ __align__(128) uint32_t tsm[];
  __shared__ __align__(8) uint64_t mbar[2];
  __shared__ uint32_t tmem_base;
  const int tid = threadIdx.x, warp = tid / 32, lane = tid % 32;
  const long long m0 = (long long)blockIdx.x * 128;
  const int n0 = blockIdx.y * NT;
  const size_t stage_u32 = TileSmem<KC>::bytes(NT) / sizeof(uint32_t) / 2;
  uint32_t* st[2] = {tsm, tsm + stage_u32};
  if (warp == 0) umma::tmem_alloc(&tmem_base, tmem_cols);
  if (tid == 0) {
    umma::mbar_init(&mbar[0], 1);
    umma::mbar_init(&mbar[1], 1);
  }
  const int nch = (K + KC - 1) / KC;
  stage_tile<KC>(st[0], NT, A, ar, M, m0, B, lbn, lbk, Ntot, n0, K, 0);
  umma::fence_smem_to_async();
  umma::fence_before_sync();
  __syncthreads();
  umma::fence_after_sync();
  const uint32_t tmem = tmem_base;
  const uint32_t idesc = umma::idesc_tf32(128, NT);
  bool ok = true;
  for (int ch = 0; ch < nch; ++ch) {
    const int s = ch & 1;
    if (tid == 0) {
      const uint32_t a_hi = umma::smem_u32(st[s]);
      const uint32_t a_lo = a_hi + 4u * TileSmem<KC>::kA;
      const uint32_t b_hi = a_lo + 4u * TileSmem<KC>::kA;
      const uint32_t b_lo = b_hi + 4u * KC * NT;
#pragma unroll
      for (int ks = 0; ks < KC / 8; ++ks) {
        const uint32_t ao = ks * 2 * 128 * 16, bo = ks * 2 * NT * 16;
        const uint64_t ah = umma::desc_kmajor(a_hi + ao, 128 * 16, 128);
        const uint64_t al = umma::desc_kmajor(a_lo + ao, 128 * 16, 128);
        const uint64_t bh = umma::desc_kmajor(b_hi + bo, NT * 16, 128);
        const uint64_t bl = umma::desc_kmajor(b_lo + bo, NT * 16, 128);
        umma::mma_tf32(tmem, ah, bh, idesc, ch > 0 || ks > 0);
        umma::mma_tf32(tmem, ah, bl, idesc, true);
        umma::mma_tf32(tmem, al, bh, idesc, true);
      }
      umma::commit(&mbar[s]);
    }
    if (ch + 1 < nch) {
      // the other stage was read by the MMAs of chunk ch - 1
      if (ch >= 1 && ok) ok = umma::mbar_wait(&mbar[s ^ 1], ((ch - 1) >> 1) & 1, kWaitLimit);
      if (ok) stage_tile<KC>(st[s ^ 1], NT, A, ar, M, m0, B, lbn, lbk, Ntot, n0, K, (ch + 1) * KC);
      umma::fence_smem_to_async();
    }
    umma::fence_before_sync();
    __syncthreads();
    umma::fence_after_sync();
  }
  // MMAs complete in issue order: the last commit covers all of them
  if (ok) ok = umma::mbar_wait(&mbar[(nch - 1) & 1], ((nch - 1) >> 1) & 1, kWaitLimit);
  if (!ok) {
    atomicExch(err, 1);
    umma::mbar_wait(&mbar[(nch - 1) & 1], ((nch - 1) >> 1) & 1, kWaitLimit);
  }
  umma::fence_after_sync();
  if (ok) {
    // warp w reads accumulator rows 32 (w % 4) .. + 31 (its tensor-memory lane
    // quarter) and columns [h NT / 2, (h + 1) NT / 2), h = w / 4
    const int q = warp & 3, h = warp >> 2;
    const long long m = m0 + 32 * q + lane;
    for (int c0 = h * (NT / 2); c0 < (h + 1) * (NT / 2); c0 += 8) {
      float v[8];
      umma::tmem_ld8(tmem + ((uint32_t)(32 * q) << 16) + (uint32_t)c0, v);
      umma::tmem_ld_wait();
      apply_epi(epi, m, M, n0 + c0, Ntot, v);
    }
  }
  umma::fence_before_sync();
  __syncthreads();
  if (warp == 0) umma::tmem_dealloc(tmem, tmem_cols);
}

// Pipelined form of gemm_tf32x3_kernel: the 256 staging threads (warps 0-3: A
// rows, warps 4-7: B columns) fill a ring of ST stages ahead of the tensor core,
// and a ninth warp issues the MMAs.  Stage s is handed over by mbarriers: the
// staging threads arrive on full[s] after their shared-memory stores (with the
// async-proxy fence), the issuing thread waits on it, issues the stage's MMAs and
// commits them to empty[s], which the staging threads wait on before refilling
// the stage.  No block-wide barrier inside the K loop, so global loads of the
// next stages overlap the MMAs of the current one.  Every wait is bounded; a
// timeout sets *err and the CTA skips the rest of its work (no hang).
template <int KC, int ST, class Epi>
__global__ void __launch_bounds__(288) gemm_tf32x3_ws_kernel(const double* __restrict__ A, ARows ar, long long M,
                                                             const double* __restrict__ B, long long lbn,
                                                             long long lbk, int Ntot, int K, int NT,
                                                             uint32_t tmem_cols, Epi epi, int* __restrict__ err) {
  extern __shared__ __align__(128) uint32_t tsm[];
  __shared__ __align__(8) uint64_t full[ST], empty[ST], done;
  __shared__ uint32_t tmem_base;
  __shared__ int fail;
  const int tid = threadIdx.x, warp = tid / 32, lane = tid % 32;
  const long long m0 = (long long)blockIdx.x * 128;
  const int n0 = blockIdx.y * NT;
  const size_t stage_u32 = TileSmem<KC>::bytes(NT) / sizeof(uint32_t) / 2;
  if (warp == 0) umma::tmem_alloc(&tmem_base, tmem_cols);
  if (tid == 0) {
    for (int s = 0; s < ST; ++s) {
      umma::mbar_init(&full[s], 256);
      umma::mbar_init(&empty[s], 1);
    }
    umma::mbar_init(&done, 1);
    fail = 0;
  }
  umma::fence_before_sync();
  __syncthreads();
  umma::fence_after_sync();
  const uint32_t tmem = tmem_base;
  const int nch = (K + KC - 1) / KC;
  if (warp < 8) {
    // staging threads
    for (int ch = 0; ch < nch; ++ch) {
      const int s = ch % ST;
      if (ch >= ST && !umma::mbar_wait(&empty[s], ((ch / ST) - 1) & 1, kWaitLimit)) {
        atomicExch(&fail, 1);
        break;
      }
      if (fail) break;
      stage_tile<KC>(tsm + (size_t)s * stage_u32, NT, A, ar, M, m0, B, lbn, lbk, Ntot, n0, K, ch * KC);
      umma::fence_smem_to_async();
      umma::mbar_arrive(&full[s]);
    }
  } else if (lane == 0) {
    // the issuing thread
    const uint32_t idesc = umma::idesc_tf32(128, NT);
    for (int ch = 0; ch < nch; ++ch) {
      const int s = ch % ST;
      if (!umma::mbar_wait(&full[s], (ch / ST) & 1, kWaitLimit)) {
        atomicExch(&fail, 1);
        break;
      }
      umma::fence_after_sync();
      const uint32_t a_hi = umma::smem_u32(tsm + (size_t)s * stage_u32);
      const uint32_t a_lo = a_hi + 4u * TileSmem<KC>::kA;
      const uint32_t b_hi = a_lo + 4u * TileSmem<KC>::kA;
      const uint32_t b_lo = b_hi + 4u * KC * NT;
#pragma unroll
      for (int ks = 0; ks < KC / 8; ++ks) {
        const uint32_t ao = ks * 2 * 128 * 16, bo = ks * 2 * NT * 16;
        const uint64_t ah = umma::desc_kmajor(a_hi + ao, 128 * 16, 128);
        const uint64_t al = umma::desc_kmajor(a_lo + ao, 128 * 16, 128);
        const uint64_t bh = umma::desc_kmajor(b_hi + bo, NT * 16, 128);
        const uint64_t bl = umma::desc_kmajor(b_lo + bo, NT * 16, 128);
        umma::mma_tf32(tmem, ah, bh, idesc, ch > 0 || ks > 0);
        umma::mma_tf32(tmem, ah, bl, idesc, true);
        umma::mma_tf32(tmem, al, bh, idesc, true);
      }
      umma::commit(&empty[s]);
    }
    umma::commit(&done);  // arrives when every MMA issued above has completed
  }
  // everyone: the accumulator is final once `done` completes (bounded)
  bool ok = umma::mbar_wait(&done, 0, kWaitLimit);
  __syncthreads();
  ok = ok && !fail;
  if (!ok && tid == 0) atomicExch(err, 1);
  umma::fence_after_sync();
  if (ok && warp < 8) {
    const int q = warp & 3, h = warp >> 2;
    const long long m = m0 + 32 * q + lane;
    for (int c0 = h * (NT / 2); c0 < (h + 1) * (NT / 2); c0 += 8) {
      float v[8];
      umma::tmem_ld8(tmem + ((uint32_t)(32 * q) << 16) + (uint32_t)c0, v);
      umma::tmem_ld_wait();
      apply_epi(epi, m, M, n0 + c0, Ntot, v);
    }
  }
  umma::fence_before_sync();
  __syncthreads();
  if (warp == 0) umma::tmem_dealloc(tmem, tmem_cols);
}

// Pre-split operands for the bulk-copy form: each K chunk of each 128-row tile of
// A (and of each NT-column tile of B) is written once, split into tf32 hi and lo,
// in the exact shared-memory layout of stage_tile (core matrices, K-major), hi
// then lo, so that one 1-D bulk copy moves it.  Rows, columns and K beyond the
// operand are zero.
// A: block (mt, ch) at u32 offset (mt nch + ch) 2 * 128 KC.
template <int KC>
__global__ void __launch_bounds__(128) split_a_tiles_kernel(const double* __restrict__ A, ARows ar, long long M,
                                                            int K, int nch, uint32_t* __restrict__ out) {
  const long long mt = blockIdx.x;
  const int ch = blockIdx.y, r = threadIdx.x;
  const long long m = mt * 128 + r;
  const long long rb = m < M ? ar.row(m) : 0;
  double v[KC];
#pragma unroll
  for (int k = 0; k < KC; ++k) {
    const int kk = ch * KC + k;
    v[k] = (m < M && kk < K) ? A[rb + (long long)kk * ar.lak] : 0.0;
  }
  uint32_t* hi = out + (size_t)(mt * nch + ch) * 2 * 128 * KC;
  uint32_t* lo = hi + 128 * KC;
#pragma unroll
  for (int c = 0; c < KC / 4; ++c) {
    uint4 h, l;
    umma::split_tf32(v[4 * c + 0], h.x, l.x);
    umma::split_tf32(v[4 * c + 1], h.y, l.y);
    umma::split_tf32(v[4 * c + 2], h.z, l.z);
    umma::split_tf32(v[4 * c + 3], h.w, l.w);
    *reinterpret_cast<uint4*>(hi + (c * 128 + r) * 4) = h;
    *reinterpret_cast<uint4*>(lo + (c * 128 + r) * 4) = l;
  }
}

// B: block (nt, ch) at u32 offset (nt nch + ch) 2 NT KC; element (column n, k) =
// B[n lbn + k lbk].
template <int KC>
__global__ void split_b_tiles_kernel(const double* __restrict__ B, long long lbn, long long lbk, int Ntot, int K,
                                     int NT, int nch, uint32_t* __restrict__ out) {
  const int nt = blockIdx.x, ch = blockIdx.y;
  uint32_t* hi = out + (size_t)(nt * nch + ch) * 2 * NT * KC;
  uint32_t* lo = hi + NT * KC;
  for (int idx = threadIdx.x; idx < (KC / 4) * NT; idx += blockDim.x) {
    const int c = idx / NT, r = idx - c * NT;
    const int n = nt * NT + r;
    double v[4];
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const int k = ch * KC + 4 * c + j;
      v[j] = (n < Ntot && k < K) ? B[(long long)n * lbn + (long long)k * lbk] : 0.0;
    }
    uint4 h, l;
    umma::split_tf32(v[0], h.x, l.x);
    umma::split_tf32(v[1], h.y, l.y);
    umma::split_tf32(v[2], h.z, l.z);
    umma::split_tf32(v[3], h.w, l.w);
    *reinterpret_cast<uint4*>(hi + (c * NT + r) * 4) = h;
    *reinterpret_cast<uint4*>(lo + (c * NT + r) * 4) = l;
  }
}

// The bulk-copy form: one thread moves each K chunk of the pre-split A and B tiles
// into a ring of ST stages with two 1-D bulk copies (announced on the stage's
// `full` mbarrier with their byte count), another issues the MMAs and commits them
// to the stage's `empty` mbarrier; four warps read the accumulator back.  Every
// wait is bounded; on a timeout the CTA records it in *err, waits (bounded) for
// the copies it issued, frees its tensor memory and returns.
template <int KC, int ST, class Epi>
__global__ void __launch_bounds__(128) gemm_tf32x3_bulk_kernel(const uint32_t* __restrict__ As,
                                                               const uint32_t* __restrict__ Bs, long long M, int Ntot,
                                                               int nch, int NT, uint32_t tmem_cols, Epi epi,
                                                               int* __restrict__ err) {
  extern __shared__ __align__(128) uint32_t tsm[];
  __shared__ __align__(8) uint64_t full[ST], empty[ST], done;
  __shared__ uint32_t tmem_base;
  __shared__ int fail;
  const int tid = threadIdx.x, warp = tid / 32, lane = tid % 32;
  const long long mt = blockIdx.x;
  const int nt = blockIdx.y;
  const uint32_t a_bytes = 2u * 128u * KC * 4u, b_bytes = 2u * (uint32_t)NT * KC * 4u;
  const size_t stage_u32 = (a_bytes + b_bytes) / 4;
  if (warp == 0) umma::tmem_alloc(&tmem_base, tmem_cols);
  if (tid == 0) {
    for (int s = 0; s < ST; ++s) {
      umma::mbar_init(&full[s], 1);
      umma::mbar_init(&empty[s], 1);
    }
    umma::mbar_init(&done, 1);
    fail = 0;
  }
  umma::fence_before_sync();
  __syncthreads();
  umma::fence_after_sync();
  const uint32_t tmem = tmem_base;
  int issued = 0;  // chunks whose copies the producer issued
  if (tid == 0) {
    // producer
    for (int ch = 0; ch < nch; ++ch) {
      const int s = ch % ST;
      if (ch >= ST && !umma::mbar_wait(&empty[s], ((ch / ST) - 1) & 1, kWaitLimit)) {
        atomicExch(&fail, 1);
        break;
      }
      if (fail) break;
      uint32_t* dst = tsm + (size_t)s * stage_u32;
      tma::mbar_arrive_expect_tx(&full[s], a_bytes + b_bytes);
      tma::load_1d(dst, As + (size_t)(mt * nch + ch) * (a_bytes / 4), a_bytes, &full[s]);
      tma::load_1d(dst + a_bytes / 4, Bs + (size_t)(nt * nch + ch) * (b_bytes / 4), b_bytes, &full[s]);
      issued = ch + 1;
    }
  } else if (tid == 32) {
    // MMA issue
    const uint32_t idesc = umma::idesc_tf32(128, NT);
    for (int ch = 0; ch < nch; ++ch) {
      const int s = ch % ST;
      if (!umma::mbar_wait(&full[s], (ch / ST) & 1, kWaitLimit)) {
        atomicExch(&fail, 1);
        break;
      }
      umma::fence_after_sync();
      const uint32_t a_hi = umma::smem_u32(tsm + (size_t)s * stage_u32);
      const uint32_t a_lo = a_hi + 4u * 128u * KC;
      const uint32_t b_hi = a_hi + a_bytes;
      const uint32_t b_lo = b_hi + 4u * (uint32_t)NT * KC;
#pragma unroll
      for (int ks = 0; ks < KC / 8; ++ks) {
        const uint32_t ao = ks * 2 * 128 * 16, bo = ks * 2 * NT * 16;
        const uint64_t ah = umma::desc_kmajor(a_hi + ao, 128 * 16, 128);
        const uint64_t al = umma::desc_kmajor(a_lo + ao, 128 * 16, 128);
        const uint64_t bh = umma::desc_kmajor(b_hi + bo, NT * 16, 128);
        const uint64_t bl = umma::desc_kmajor(b_lo + bo, NT * 16, 128);
        umma::mma_tf32(tmem, ah, bh, idesc, ch > 0 || ks > 0);
        umma::mma_tf32(tmem, ah, bl, idesc, true);
        umma::mma_tf32(tmem, al, bh, idesc, true);
      }
      umma::commit(&empty[s]);
    }
    umma::commit(&done);
  }
  bool ok = umma::mbar_wait(&done, 0, kWaitLimit);
  __syncthreads();
  ok = ok && !fail;
  if (!ok) {
    if (tid == 0) {
      atomicExch(err, 1);
      // the copies of the last ST issued chunks may still be landing: wait for them
      for (int ch = issued > ST ? issued - ST : 0; ch < issued; ++ch)
        umma::mbar_wait(&full[ch % ST], (ch / ST) & 1, kWaitLimit);
    }
    __syncthreads();
  }
  umma::fence_after_sync();
  if (ok) {
    const long long m = mt * 128 + 32 * warp + lane;
    for (int c0 = 0; c0 < NT; c0 += 8) {
      float v[8];
      umma::tmem_ld8(tmem + ((uint32_t)(32 * warp) << 16) + (uint32_t)c0, v);
      umma::tmem_ld_wait();
      apply_epi(epi, m, M, nt * NT + c0, Ntot, v);
    }
  }
  umma::fence_before_sync();
  __syncthreads();
  if (warp == 0) umma::tmem_dealloc(tmem, tmem_cols);
}

constexpr int kSmemDyn = 224 * 1024;  // dynamic limit (the static mbarriers take the rest of 227 KB)

template <int KC, class Epi>
int launch_tf32x3_kc(Ctx& c, const double* A, ARows ar, long long M, const double* B, long long lbn, long long lbk,
                     int Ntot, int K, const Epi& epi, size_t smem_min) {
  const int ntile = ceil_div(Ntot, 256);
  const int NT = ceil_div(ceil_div(Ntot, ntile), 16) * 16;
  const uint32_t cols = NT <= 32 ? 32 : NT <= 64 ? 64 : NT <= 128 ? 128 : 256;
  const size_t smem = std::max(TileSmem<KC>::bytes(NT), std::min<size_t>(smem_min, kSmemDyn));
  SG_CHECK(smem <= (size_t)kSmemDyn, SINCGPU_ERANGE, "tensor-core tile needs %zu bytes of shared memory", smem);
  // process-wide attribute, one fixed value (thread-safe static initialisation)
  static const cudaError_t attr = cudaFuncSetAttribute(gemm_tf32x3_kernel<KC, Epi>,
                                                       cudaFuncAttributeMaxDynamicSharedMemorySize, kSmemDyn);
  SG_CUDA(attr);
  int* err = nullptr;
  SG_TRY(timeout_flags(c, &err));
  const dim3 grid((unsigned)ceil_div(M, 128), (unsigned)ntile);
  gemm_tf32x3_kernel<KC, Epi><<<grid, 256, smem, c.stream>>>(A, ar, M, B, lbn, lbk, Ntot, K, NT, cols, epi, err);
  SG_LAUNCHED();
  return SINCGPU_OK;
}

template <int KC, int ST, class Epi>
int launch_tf32x3_ws(Ctx& c, const double* A, ARows ar, long long M, const double* B, long long lbn, long long lbk,
                     int Ntot, int K, const Epi& epi, size_t smem_min) {
  const int ntile = ceil_div(Ntot, 256);
  const int NT = ceil_div(ceil_div(Ntot, ntile), 16) * 16;
  const uint32_t cols = NT <= 32 ? 32 : NT <= 64 ? 64 : NT <= 128 ? 128 : 256;
  const size_t smem = std::max(ST * TileSmem<KC>::bytes(NT) / 2, std::min<size_t>(smem_min, kSmemDyn));
  SG_CHECK(smem <= (size_t)kSmemDyn, SINCGPU_ERANGE, "tensor-core stages need %zu bytes of shared memory", smem);
  static const cudaError_t attr = cudaFuncSetAttribute(gemm_tf32x3_ws_kernel<KC, ST, Epi>,
                                                       cudaFuncAttributeMaxDynamicSharedMemorySize, kSmemDyn);
  SG_CUDA(attr);
  int* err = nullptr;
  SG_TRY(timeout_flags(c, &err));
  const dim3 grid((unsigned)ceil_div(M, 128), (unsigned)ntile);
  gemm_tf32x3_ws_kernel<KC, ST, Epi><<<grid, 288, smem, c.stream>>>(A, ar, M, B, lbn, lbk, Ntot, K, NT, cols, epi,
                                                                      err);
  SG_LAUNCHED();
  return SINCGPU_OK;
}

// Bulk-copy form: pre-split A and B (workspace ws_tc), then the ring kernel.
template <int KC, int ST, class Epi>
int launch_tf32x3_bulk(Ctx& c, const double* A, ARows ar, long long M, const double* B, long long lbn,
                       long long lbk, int Ntot, int K, const Epi& epi) {
  const int ntile = ceil_div(Ntot, 256);
  const int NT = ceil_div(ceil_div(Ntot, ntile), 16) * 16;
  const uint32_t cols = NT <= 32 ? 32 : NT <= 64 ? 64 : NT <= 128 ? 128 : 256;
  const int nch = ceil_div(K, KC);
  const long long mtiles = (M + 127) / 128;
  if constexpr (ST > 3) {  // wide tiles: fewer stages where ST of them do not fit
    if ((size_t)ST * (2 * 128 * KC + 2 * NT * KC) * sizeof(uint32_t) > (size_t)kSmemDyn)
      return launch_tf32x3_bulk<KC, 3>(c, A, ar, M, B, lbn, lbk, Ntot, K, epi);
  }
  const size_t a_u32 = (size_t)mtiles * nch * 2 * 128 * KC, b_u32 = (size_t)ntile * nch * 2 * NT * KC;
  SG_TRY(c.ws_tc.ensure(sizeof(uint32_t) * (a_u32 + b_u32)));
  uint32_t* As = (uint32_t*)c.ws_tc.ptr;
  uint32_t* Bs = As + a_u32;
  SG_CHECK(mtiles < (1LL << 31), SINCGPU_ERANGE, "too many row tiles");
  split_a_tiles_kernel<KC><<<dim3((unsigned)mtiles, nch), 128, 0, c.stream>>>(A, ar, M, K, nch, As);
  SG_LAUNCHED();
  split_b_tiles_kernel<KC><<<dim3(ntile, nch), 256, 0, c.stream>>>(B, lbn, lbk, Ntot, K, NT, nch, Bs);
  SG_LAUNCHED();
  const size_t smem = (size_t)ST * (2 * 128 * KC + 2 * NT * KC) * sizeof(uint32_t);
  SG_CHECK(smem <= (size_t)kSmemDyn, SINCGPU_ERANGE, "tensor-core stages need %zu bytes of shared memory", smem);
  static const cudaError_t attr = cudaFuncSetAttribute(gemm_tf32x3_bulk_kernel<KC, ST, Epi>,
                                                       cudaFuncAttributeMaxDynamicSharedMemorySize, kSmemDyn);
  SG_CUDA(attr);
  int* err = nullptr;
  SG_TRY(timeout_flags(c, &err));
  gemm_tf32x3_bulk_kernel<KC, ST, Epi><<<dim3((unsigned)mtiles, ntile), 128, smem, c.stream>>>(
      As, Bs, M, Ntot, nch, NT, cols, epi, err);
  SG_LAUNCHED();
  return SINCGPU_OK;
}

// smem_min: dynamic shared memory to reserve at least (the self test reserves
// more than its tiles need, so that every descriptor address stays inside the
// CTA's allocation).  K chunks of 16 (two CTAs per SM) or, with the context
// option tc_kc = 32, of 32 (one CTA per SM, twice the MMAs per commit).
template <class Epi>
int launch_tf32x3(Ctx& c, const double* A, ARows ar, long long M, const double* B, long long lbn, long long lbk,
                  int Ntot, int K, const Epi& epi, size_t smem_min = 0) {
  SG_CHECK(M >= 1 && Ntot >= 1 && K >= 1, SINCGPU_EINVAL, "empty tensor-core contraction");
  if (c.tc_pipe == 4) return launch_tf32x3_bulk<16, 3>(c, A, ar, M, B, lbn, lbk, Ntot, K, epi);
  if (c.tc_pipe == 5) return launch_tf32x3_bulk<16, 5>(c, A, ar, M, B, lbn, lbk, Ntot, K, epi);
  if (c.tc_pipe == 1) return launch_tf32x3_ws<16, 3>(c, A, ar, M, B, lbn, lbk, Ntot, K, epi, smem_min);
  if (c.tc_pipe == 2) return launch_tf32x3_ws<16, 4>(c, A, ar, M, B, lbn, lbk, Ntot, K, epi, smem_min);
  if (c.tc_pipe == 3) return launch_tf32x3_ws<8, 6>(c, A, ar, M, B, lbn, lbk, Ntot, K, epi, smem_min);
  if (c.tc_kc == 32) return launch_tf32x3_kc<32>(c, A, ar, M, B, lbn, lbk, Ntot, K, epi, smem_min);
  return launch_tf32x3_kc<16>(c, A, ar, M, B, lbn, lbk, Ntot, K, epi, smem_min);
}

}  // namespace

int timeout_flags(Ctx& c, int** flags) {
  if (!c.ws_tcerr.ptr) {
    SG_TRY(c.ws_tcerr.ensure(64));
    SG_CUDA(cudaMemsetAsync(c.ws_tcerr.ptr, 0, 64, c.stream));
  }
  *flags = (int*)c.ws_tcerr.ptr;
  return SINCGPU_OK;
}

int tc_error_reset(Ctx& c) {
  int* f = nullptr;
  SG_TRY(timeout_flags(c, &f));
  SG_CUDA(cudaMemsetAsync(f, 0, sizeof(int), c.stream));
  return SINCGPU_OK;
}

int tc_error_read(Ctx& c, int* flag) {
  *flag = 0;
  if (!c.ws_tcerr.ptr) return SINCGPU_OK;
  SG_CUDA(cudaMemcpyAsync(flag, c.ws_tcerr.ptr, sizeof(int), cudaMemcpyDeviceToHost, c.stream));
  SG_CUDA(cudaStreamSynchronize(c.stream));
  return SINCGPU_OK;
}

// reducedpot[(kk + n ii) G + x] = sum_k Rpl[k G + x] Wm[k NC + col] (col = 2t + re/im)
int rp_gemm_tf32(Ctx& c, const double* Rpl, const double* Wm, int K, int NC, const int* d_tmap,
                 double2* reducedpot) {
  RedpotEpi e{reducedpot, c.G, d_tmap, c.nspf};
  return launch_tf32x3(c, Rpl, ARows{1, c.G, 0, c.G}, c.G, Wm, 1, NC, NC, K, e);
}

// The per-axis kinetic contraction on the tensor cores (precision form, option
// ke_tf32): out(.., j, ..) = sum_l K(j, l) in(.., l, ..) along x, y and z, real and
// imaginary parts as separate lines, one 3xTF32 GEMM per axis (lines x N x N
// against ketile, FP32 accumulation, FP64 sums across the axes), the potential
// and z-field terms added in the first axis's epilogue.  Same result as mult_ke to
// about 1e-7 of the kinetic term.
int mult_ke_tf32(Ctx& c, const double2* in, double2* out, int howmany, bool extra, double zfield) {
  const long long N = c.N, NN = N * N, G = c.G;
  const double* A = reinterpret_cast<const double*>(in);
  double* O = reinterpret_cast<double*>(out);
  // line = (re/im, the other two coordinates, orbital); element l along the axis
  const ARows ax{1, 2, 2 * N, 2}, ay{1, 2 * N, 2 * NN, 2 * N}, az{1, 2 * NN, 2 * G, 2 * NN};
  const long long M = 2 * NN * howmany;
  {
    ProfScope ps(c, ST_KE_XY);
    SG_TRY(launch_tf32x3(c, A, ax, M, c.d_ketile, c.ke_stride, 1, c.N, c.N,
                         KeEpi{O, A, ax, 1, extra ? 1 : 0, c.d_pot, c.d_zdip, zfield, G}));
    SG_TRY(launch_tf32x3(c, A, ay, M, c.d_ketile, c.ke_stride, 1, c.N, c.N,
                         KeEpi{O, A, ay, 0, 0, nullptr, nullptr, 0.0, G}));
  }
  ProfScope ps(c, ST_KE_Z);
  return launch_tf32x3(c, A, az, M, c.d_ketile, c.ke_stride, 1, c.N, c.N, KeEpi{O, A, az, 0, 0, nullptr, nullptr, 0.0, G});
}

}  // namespace sincgpu

using namespace sincgpu;

extern "C" int sincgpu_kernel_timeouts(sincgpu_ctx* h, int* flags) {
  CTX_CHECK(h);
  Ctx& c = h->c;
  SG_CHECK(flags, SINCGPU_EINVAL, "null flags");
  flags[0] = flags[1] = 0;
  if (!c.ws_tcerr.ptr) return SINCGPU_OK;
  SG_CUDA(cudaMemcpyAsync(flags, c.ws_tcerr.ptr, 2 * sizeof(int), cudaMemcpyDeviceToHost, c.stream));
  SG_CUDA(cudaStreamSynchronize(c.stream));
  return SINCGPU_OK;
}

extern "C" int sincgpu_gemm_tf32x3_dev(sincgpu_ctx* h, const double* A, const double* B, double* C, long long M,
                                       int N, int K, int* timed_out) {
  CTX_CHECK(h);
  Ctx& c = h->c;
  SG_CHECK(A && B && C, SINCGPU_EINVAL, "null matrix");
  SG_CHECK(M >= 1 && N >= 1 && K >= 1, SINCGPU_EINVAL, "bad sizes");
  SG_TRY(tc_error_reset(c));
  StoreEpi e{C, N, 1};
  SG_TRY(launch_tf32x3(c, A, ARows{K, M, 0, 1}, M, B, K, 1, N, K, e, 200 * 1024));
  int flag = 0;
  SG_TRY(tc_error_read(c, &flag));
  if (timed_out) *timed_out = flag;
  SG_CHECK(!flag, SINCGPU_ECUDA, "tensor-core contraction timed out waiting for its MMAs");
  return SINCGPU_OK;
}
