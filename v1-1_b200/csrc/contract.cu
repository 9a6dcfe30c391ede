// Dense contractions of the mean-field build, on FP64 CUDA cores.
//
// twoematel (SINCDVR/coreproject.f90:1089-1100):
//   twoematel(a1,b1,a2,b2) = sum_x rho_{a1b1}(x) R_{a2b2}(x),  rho = phi1_a conj(phi2_b)
// reducedpot (MCTDH.SRC/mean.f90:556-558, ZGEMM):
//   reducedpot(x,k,i) = sum_{c,d} R_{cd}(x) Gamma(c,d,k,i)
//
// Both are recast as REAL tall-skinny GEMMs over planar real/imag rows.
// With hermitian orbitals (phi1 == phi2) rho_ba = conj(rho_ab) and, the kernel
// being real, R_ba = conj(R_ab); only the U = n(n+1)/2 pairs a<=b are stored:
//   twoematel: C = [u|v]^T [r|s]  (2U x 2U, K = G), then
//       M(p,q)       = (UR-VS) + i(US+VR)      M(pbar,q)    = (UR+VS) + i(US-VR)
//       M(p,qbar)    = (UR+VS) + i(VR-US)      M(pbar,qbar) = conj M(p,q)
//   reducedpot: out = sum_p r_p A_p + s_p B_p with A_p = G(c,d)+G(d,c),
//       B_p = i(G(c,d)-G(d,c)) for c<d and A_p = G(c,c), B_p = iG(c,c) for c=d,
//   i.e. [r|s] (G x 2U) times a real 2U x 2n^2 matrix.
// Compared with the complex contractions of the reference this is 4x (twoematel)
// and 2x (reducedpot) fewer flops.  Without the symmetry (phi1 != phi2) all n^2
// ordered pairs are used with the plain complex identities.
#include <algorithm>
#include <vector>
#include "context.hpp"

namespace sincgpu {

constexpr int kMaxOrb = 32;
constexpr int TK = 16;  // x points per K stage of the twoematel GEMM

// 8-byte asynchronous global->shared copy (zero-fill when !valid)
__device__ __forceinline__ void cp_async8(void* smem, const void* gmem, bool valid) {
  unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  int n = valid ? 8 : 0;
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(s), "l"(gmem), "r"(n));
}
// 16-byte asynchronous global->shared copy (zero-fill when !valid)
__device__ __forceinline__ void cp_async16(void* smem, const void* gmem, bool valid) {
  unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  int n = valid ? 16 : 0;
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(s), "l"(gmem), "r"(n));
}
// D (8 x 8, two values per lane) += A (8 x 4) B (4 x 8) on the FP64 tensor cores;
// lane g * 4 + t holds A[g][t], B[t][g] and D[g][2t], D[g][2t + 1]
__device__ __forceinline__ void dmma_884(double (&d)[2], double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
               : "+d"(d[0]), "+d"(d[1])
               : "d"(a), "d"(b));
}

__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N)); }

// ---------------------------------------------------------------------------
// C_part[split][m][n] = sum_{x in split} A(x,m) B(x,n)
// A(x,m): m <  npair -> Re(phi1_{pa} conj(phi2_{pb}))(x),  m >= npair -> Im
// B(x,n): Rpl[n*G + x]
// ---------------------------------------------------------------------------
// twoematel GEMM with square 16R x 16R tiles (R x R register blocks, 256
// threads): for 2U <= 16R one tile covers all outputs (R = 7 gives 112 x 112,
// enough for U = 55), so neither the pair products nor the orbital
// tiles are recomputed per column tile and padding stays small.  Split-K over x
// across the SMs; cp.async double buffering of the orbital values and Rpl rows.
// DMMA = true: the same tiles on the FP64 tensor cores (mma.sync m8n8k4 f64):
// 2R warps, warp w owns rows 16 (w / 2) .. + 15 of the tile and half of its
// columns (2 x R fragments of 8 x 8), shared-memory rows padded to TK + 4 doubles
// (4 mod 16) so the fragment loads are conflict-free.
template <int R, bool DMMA>
__global__ void __launch_bounds__(DMMA ? 64 * R : 256, 1) twoe_gemm3_kernel(const double2* __restrict__ phi1,
                                                            const double2* __restrict__ phi2,
                                                            const int* __restrict__ pa,
                                                            const int* __restrict__ pb,
                                                            const double* __restrict__ Rpl, int npair,
                                                            int nspf, long long G, int ntn,
                                                            long long xper, double* __restrict__ part) {
  constexpr int TT = 16 * R;
  constexpr int TS = DMMA ? TK + 4 : TK + 1;  // shared-memory row stride (doubles)
  constexpr int NTH = DMMA ? 64 * R : 256;
  extern __shared__ __align__(16) double dsm[];
  double* As = dsm;                                   // [TT][TS]
  double* Bs = As + TT * TS;                          // [2][TT][TS]
  double2* fsm = reinterpret_cast<double2*>(Bs + 2 * TT * TS);  // [2][2][nspf][TK]
  int* sa = reinterpret_cast<int*>(fsm + 4 * nspf * TK);
  int* sb = sa + TT;
  int* sc = sb + TT;
  auto f1 = [&](int st, int o, int k) -> double2& { return fsm[((st * 2 + 0) * nspf + o) * TK + k]; };
  auto f2 = [&](int st, int o, int k) -> double2& { return fsm[((st * 2 + 1) * nspf + o) * TK + k]; };
  const int M = 2 * npair;
  // upper-triangle tiles only (tm <= tn): C = A^T K A is symmetric, the lower
  // tiles are mirrored in split_reduce_kernel
  int tm = 0, rem = blockIdx.x;
  while (rem >= ntn - tm) {
    rem -= ntn - tm;
    ++tm;
  }
  const int tn = tm + rem;
  const int m0 = tm * TT, n0 = tn * TT;
  const long long xb = blockIdx.y * xper;
  const long long xe = min(G, xb + xper);
  const int tid = threadIdx.x, tx = tid % 16, ty = tid / 16;
  for (int i = tid; i < TT; i += NTH) {
    const int m = m0 + i;
    if (m < M) {
      const int p = m % npair;
      sa[i] = pa[p];
      sb[i] = pb[p];
      sc[i] = m / npair;
    } else {
      sa[i] = 0;
      sb[i] = 0;
      sc[i] = -1;
    }
  }
  auto load = [&](int st, long long x0) {
    for (int i = tid; i < nspf * TK; i += NTH) {
      const int o = i / TK, k = i % TK;
      const long long x = x0 + k;
      const bool ok = x < xe;
      const double2* g1 = ok ? phi1 + (long long)o * G + x : phi1;
      const double2* g2 = ok ? phi2 + (long long)o * G + x : phi2;
      cp_async8(&f1(st, o, k), g1, ok);
      cp_async8(reinterpret_cast<double*>(&f1(st, o, k)) + 1, reinterpret_cast<const double*>(g1) + 1, ok);
      cp_async8(&f2(st, o, k), g2, ok);
      cp_async8(reinterpret_cast<double*>(&f2(st, o, k)) + 1, reinterpret_cast<const double*>(g2) + 1, ok);
    }
    for (int i = tid; i < TK * TT; i += NTH) {
      const int nn = i / TK, k = i % TK;
      const int n = n0 + nn;
      const long long x = x0 + k;
      const bool ok = n < M && x < xe;
      cp_async8(&Bs[(st * TT + nn) * TS + k], ok ? (const void*)(Rpl + (long long)n * G + x) : (const void*)Rpl, ok);
    }
    cp_async_commit();
  };
  double acc[DMMA ? 1 : R][DMMA ? 1 : R];
  double dacc[DMMA ? 2 : 1][DMMA ? R : 1][2];
#pragma unroll
  for (int i = 0; i < (DMMA ? 1 : R); ++i)
#pragma unroll
    for (int j = 0; j < (DMMA ? 1 : R); ++j) acc[i][j] = 0.0;
#pragma unroll
  for (int i = 0; i < (DMMA ? 2 : 1); ++i)
#pragma unroll
    for (int j = 0; j < (DMMA ? R : 1); ++j) dacc[i][j][0] = dacc[i][j][1] = 0.0;
  const int wrow = 16 * ((tid >> 5) >> 1), wcol = 8 * R * ((tid >> 5) & 1);
  const int g8 = (tid & 31) >> 2, t4 = tid & 3;
  const long long nk = (xe - xb + TK - 1) / TK;
  __syncthreads();  // sa/sb/sc visible
  if (nk > 0) load(0, xb);
  for (long long t = 0; t < nk; ++t) {
    const int st = (int)(t & 1);
    if (t + 1 < nk) {
      load(st ^ 1, xb + (t + 1) * TK);
      cp_async_wait<1>();
    } else {
      cp_async_wait<0>();
    }
    __syncthreads();
    for (int i = tid; i < TK * TT; i += NTH) {
      const int mm = i / TK, k = i % TK;
      double v = 0.0;
      const int comp = sc[mm];
      if (comp >= 0) {
        const double2 r = cmulc(f1(st, sa[mm], k), f2(st, sb[mm], k));
        v = comp == 0 ? r.x : r.y;
      }
      As[mm * TS + k] = v;
    }
    __syncthreads();
    const double* Bst = Bs + st * TT * TS;
    if constexpr (DMMA) {
#pragma unroll
      for (int k4 = 0; k4 < TK; k4 += 4) {
        double a[2], b[R];
#pragma unroll
        for (int r = 0; r < 2; ++r) a[r] = As[(wrow + 8 * r + g8) * TS + k4 + t4];
#pragma unroll
        for (int j = 0; j < R; ++j) b[j] = Bst[(wcol + 8 * j + g8) * TS + k4 + t4];
#pragma unroll
        for (int r = 0; r < 2; ++r)
#pragma unroll
          for (int j = 0; j < R; ++j) dmma_884(dacc[r][j], a[r], b[j]);
      }
    } else {
#pragma unroll 4
      for (int k = 0; k < TK; ++k) {
        double a[R], b[R];
#pragma unroll
        for (int i = 0; i < R; ++i) a[i] = As[(tx + 16 * i) * TS + k];
#pragma unroll
        for (int j = 0; j < R; ++j) b[j] = Bst[(ty + 16 * j) * TS + k];
#pragma unroll
        for (int i = 0; i < R; ++i)
#pragma unroll
          for (int j = 0; j < R; ++j) acc[i][j] = fma(a[i], b[j], acc[i][j]);
      }
    }
    __syncthreads();
  }
  double* out = part + (long long)blockIdx.y * M * M;
  if constexpr (DMMA) {
#pragma unroll
    for (int r = 0; r < 2; ++r) {
      const int m = m0 + wrow + 8 * r + g8;
#pragma unroll
      for (int j = 0; j < R; ++j) {
        const int n = n0 + wcol + 8 * j + 2 * t4;
        if (m < M && n < M) out[(long long)m * M + n] = dacc[r][j][0];
        if (m < M && n + 1 < M) out[(long long)m * M + n + 1] = dacc[r][j][1];
      }
    }
  } else {
#pragma unroll
    for (int i = 0; i < R; ++i) {
      const int m = m0 + tx + 16 * i;
#pragma unroll
      for (int j = 0; j < R; ++j) {
        const int n = n0 + ty + 16 * j;
        if (m < M && n < M) out[(long long)m * M + n] = acc[i][j];
      }
    }
  }
}

// twoematel GEMM on the FP64 tensor cores, software-pipelined: the same tiles,
// warps and fragments as twoe_gemm3_kernel<R, true> (2R warps, warp w owns rows
// 16 (w / 2) .. + 15 of the 16R x 16R tile and half of its columns), but the pair
// products of stage t + 1 are formed between the MMAs of stage t (one product per
// thread after each K = 4 step: 16R x TK products over 64R threads is exactly 4
// per thread), the product tile is double-buffered and the raw orbital values and
// Rpl rows triple-buffered, so one barrier per stage separates the stages and the
// tensor pipe is not idle while the products are formed.
// SYM (one tile holds all 2U rows and columns): C is symmetric, so only the 8 x 8
// blocks on and below the diagonal are computed, R (2R + 1) of the (2R)^2; each
// off-diagonal block is also stored transposed in place of its mirror.  Row blocks p and 2R - 1 - p form a pair
// with 2R + 1 blocks; warp 2p takes the first R + 1 of them, warp 2p + 1 the rest.
template <int R, bool SYM, int KT>
__global__ void __launch_bounds__(64 * R, 1) twoe_dmma_kernel(const double2* __restrict__ phi1,
                                                              const double2* __restrict__ phi2,
                                                              const int* __restrict__ pa, const int* __restrict__ pb,
                                                              const double* __restrict__ Rpl, int npair, int nspf,
                                                              long long G, int ntn, long long xper,
                                                              double* __restrict__ part, int strict) {
  constexpr int TT = 16 * R;
  constexpr int TS = KT + 4;  // shared-memory row stride (doubles), 4 mod 16
  constexpr int NTH = 64 * R;
  static_assert(TT * KT == (KT / 4) * NTH, "one product per thread and K = 4 step");
  extern __shared__ __align__(16) double dsm[];
  double* As = dsm;                                             // [2][TT][TS]
  double* Bs = As + 2 * TT * TS;                                // [3][TT][TS]
  double2* fsm = reinterpret_cast<double2*>(Bs + 3 * TT * TS);  // [3][2][nspf][KT]
  int* sa = reinterpret_cast<int*>(fsm + 6 * nspf * KT);
  int* sb = sa + TT;
  int* sc = sb + TT;
  const int M = 2 * npair;
  // tile (tm, tn): SYM CTAs take the diagonal tiles (blockIdx.x = tm = tn); the
  // others the upper-triangle tiles, the diagonal included unless `strict`
  int tm = 0, tn = 0;
  if constexpr (SYM) {
    tm = tn = blockIdx.x;
  } else {
    int rem = blockIdx.x;
    while (rem >= ntn - tm - strict) {
      rem -= ntn - tm - strict;
      ++tm;
    }
    tn = tm + strict + rem;
  }
  const int m0 = tm * TT, n0 = tn * TT;
  const long long xb = blockIdx.y * xper;
  const long long xe = min(G, xb + xper);
  const int tid = threadIdx.x;
  for (int i = tid; i < TT; i += NTH) {
    const int m = m0 + i;
    if (m < M) {
      const int p = m % npair;
      sa[i] = pa[p];
      sb[i] = pb[p];
      sc[i] = m / npair;
    } else {
      sa[i] = 0;
      sb[i] = 0;
      sc[i] = -1;
    }
  }
  auto load = [&](int st, long long x0) {
    double2* f = fsm + st * 2 * nspf * KT;
    for (int i = tid; i < nspf * KT; i += NTH) {
      const int o = i / KT, k = i % KT;
      const long long x = x0 + k;
      const bool ok = x < xe;
      const double* g1 = reinterpret_cast<const double*>(ok ? phi1 + (long long)o * G + x : phi1);
      const double* g2 = reinterpret_cast<const double*>(ok ? phi2 + (long long)o * G + x : phi2);
      double* d1 = reinterpret_cast<double*>(f + o * KT + k);
      double* d2 = reinterpret_cast<double*>(f + (nspf + o) * KT + k);
      cp_async16(d1, g1, ok);
      cp_async16(d2, g2, ok);
    }
    double* b = Bs + st * TT * TS;
    for (int i = tid; i < KT * TT; i += NTH) {
      const int nn = i / KT, k = i % KT;
      const int n = n0 + nn;
      const long long x = x0 + k;
      const bool ok = n < M && x < xe;
      cp_async8(&b[nn * TS + k], ok ? (const void*)(Rpl + (long long)n * G + x) : (const void*)Rpl, ok);
    }
    cp_async_commit();
  };
  // product q (0..3) of this thread for stage st into product buffer ab
  auto product = [&](int st, int ab, int q) {
    const int i = tid + q * NTH;
    const int mm = i / KT, k = i % KT;
    const double2* f = fsm + st * 2 * nspf * KT;
    double v = 0.0;
    const int comp = sc[mm];
    if (comp >= 0) {
      const double2 r = cmulc(f[sa[mm] * KT + k], f[(nspf + sb[mm]) * KT + k]);
      v = comp == 0 ? r.x : r.y;
    }
    As[(ab * TT + mm) * TS + k] = v;
  };
  double dacc[2][R][2];
#pragma unroll
  for (int i = 0; i < 2; ++i)
#pragma unroll
    for (int j = 0; j < R; ++j) dacc[i][j][0] = dacc[i][j][1] = 0.0;
  const int wrow = 16 * ((tid >> 5) >> 1), wcol = 8 * R * ((tid >> 5) & 1);
  const int g8 = (tid & 31) >> 2, t4 = tid & 3;
  // SYM: this warp's blocks (row block sr[j] in {rA, rB}, column block sb8[j])
  constexpr int NS = SYM ? R + 1 : 1;
  const int pr = (tid >> 5) >> 1, rA = pr, rB = 2 * R - 1 - pr;
  bool sok[NS], sisA[NS];
  int sb8[NS];
  double sacc[NS][2];
#pragma unroll
  for (int j = 0; j < NS; ++j) {
    const int s = ((tid >> 5) & 1) * (R + 1) + j;  // slot within the pair's 2R + 1 blocks
    sok[j] = s <= 2 * R;
    sisA[j] = s <= pr;
    sb8[j] = s <= pr ? s : s - pr - 1;
    sacc[j][0] = sacc[j][1] = 0.0;
  }
  const long long nk = (xe - xb + KT - 1) / KT;
  __syncthreads();  // sa/sb/sc visible
  if (nk > 0) {
    load(0, xb);
    if (nk > 1) {
      load(1, xb + KT);
      cp_async_wait<1>();
    } else {
      cp_async_wait<0>();
    }
    __syncthreads();
#pragma unroll
    for (int q = 0; q < KT / 4; ++q) product(0, 0, q);
  }
  for (long long t = 0; t < nk; ++t) {
    const int st = (int)(t % 3), ab = (int)(t & 1);
    if (t + 1 < nk) cp_async_wait<0>();  // raw stage t + 1 (the only group in flight)
    __syncthreads();  // products of t and raw t + 1 visible; stage t - 1 fully consumed
    if (t + 2 < nk) load((int)((t + 2) % 3), xb + (t + 2) * KT);
    const double* Ast = As + ab * TT * TS;
    const double* Bst = Bs + st * TT * TS;
    const bool next = t + 1 < nk;
#pragma unroll
    for (int k4 = 0; k4 < KT; k4 += 4) {
      if constexpr (SYM) {
        const double aA = Ast[(8 * rA + g8) * TS + k4 + t4], aB = Ast[(8 * rB + g8) * TS + k4 + t4];
#pragma unroll
        for (int j = 0; j < NS; ++j)
          if (sok[j]) dmma_884(sacc[j], sisA[j] ? aA : aB, Bst[(8 * sb8[j] + g8) * TS + k4 + t4]);
      } else {
        double a[2], b[R];
#pragma unroll
        for (int r = 0; r < 2; ++r) a[r] = Ast[(wrow + 8 * r + g8) * TS + k4 + t4];
#pragma unroll
        for (int j = 0; j < R; ++j) b[j] = Bst[(wcol + 8 * j + g8) * TS + k4 + t4];
#pragma unroll
        for (int r = 0; r < 2; ++r)
#pragma unroll
          for (int j = 0; j < R; ++j) dmma_884(dacc[r][j], a[r], b[j]);
      }
      if (next) product((int)((t + 1) % 3), ab ^ 1, k4 / 4);
    }
  }
  double* out = part + (long long)blockIdx.y * M * M;
  if constexpr (SYM) {
#pragma unroll
    for (int j = 0; j < NS; ++j) {
      if (!sok[j]) continue;
      const int rb = sisA[j] ? rA : rB;
      const int m = m0 + 8 * rb + g8, n = n0 + 8 * sb8[j] + 2 * t4;
      if (m < M && n < M) out[(long long)m * M + n] = sacc[j][0];
      if (m < M && n + 1 < M) out[(long long)m * M + n + 1] = sacc[j][1];
      if (sb8[j] != rb) {  // the transposed block above the diagonal (never computed)
        if (m < M && n < M) out[(long long)n * M + m] = sacc[j][0];
        if (m < M && n + 1 < M) out[(long long)(n + 1) * M + m] = sacc[j][1];
      }
    }
    return;
  }
#pragma unroll
  for (int r = 0; r < 2; ++r) {
    const int m = m0 + wrow + 8 * r + g8;
#pragma unroll
    for (int j = 0; j < R; ++j) {
      const int n = n0 + wcol + 8 * j + 2 * t4;
      if (m < M && n < M) out[(long long)m * M + n] = dacc[r][j][0];
      if (m < M && n + 1 < M) out[(long long)m * M + n + 1] = dacc[r][j][1];
    }
  }
}

// C[m][n] = sum_s part[s][m][n] (deterministic): a CTA owns 32 consecutive
// elements; its 8 warps sum interleaved eighths of the split range (warp g takes
// splits g, g + 8, ...) in a fixed order and warp 0 adds the eight partial sums in
// order.  Elements of the lower-triangle tiles (tile(m) > tile(n), never computed)
// are read mirrored.
__global__ void __launch_bounds__(256) split_reduce_kernel(const double* __restrict__ part, int nsplit, int M,
                                                           int TT, double* __restrict__ C) {
  __shared__ double acc[8][32];
  const int lane = threadIdx.x & 31, g = threadIdx.x >> 5;
  const long long MM = (long long)M * M;
  const long long i = (long long)blockIdx.x * 32 + lane;
  long long src = i;
  if (i < MM && TT < M) {
    const int m = (int)(i / M), n = (int)(i % M);
    if (m / TT > n / TT) src = (long long)n * M + m;
  }
  double s = 0.0;
  if (i < MM)
    for (int k = g; k < nsplit; k += 8) s += part[(long long)k * MM + src];
  acc[g][lane] = s;
  __syncthreads();
  if (g == 0 && i < MM) {
    double t = acc[0][lane];
#pragma unroll
    for (int q = 1; q < 8; ++q) t += acc[q][lane];
    C[i] = t;
  }
}

// twoematel(a1,b1,a2,b2) from C = [[UR,US],[VR,VS]]
// lut[a + n*b] = 2*p + conj  (hermitian pairs a<=b), or p for the general list.
__global__ void twoe_assemble_kernel(const double* __restrict__ C, const int* __restrict__ lut,
                                     int npair, int n, int herm, double2* __restrict__ out) {
  long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  const long long n4 = (long long)n * n * n * n;
  if (idx >= n4) return;
  int a1 = (int)(idx % n), b1 = (int)((idx / n) % n);
  int a2 = (int)((idx / ((long long)n * n)) % n), b2 = (int)(idx / ((long long)n * n * n));
  const int M = 2 * npair;
  int lp = lut[a1 + n * b1], lq = lut[a2 + n * b2];
  int p, q, cp = 0, cq = 0;
  if (herm) {
    p = lp >> 1;
    cp = lp & 1;
    q = lq >> 1;
    cq = lq & 1;
  } else {
    p = lp;
    q = lq;
  }
  double UR = C[(long long)p * M + q], US = C[(long long)p * M + npair + q];
  double VR = C[(long long)(npair + p) * M + q], VS = C[(long long)(npair + p) * M + npair + q];
  double2 r;
  if (!cp && !cq)
    r = make_double2(UR - VS, US + VR);
  else if (cp && !cq)
    r = make_double2(UR + VS, US - VR);
  else if (!cp && cq)
    r = make_double2(UR + VS, VR - US);
  else
    r = make_double2(UR - VS, -(US + VR));
  out[idx] = r;
}

// shared memory of twoe_dmma_kernel<R, *, KT>: product tiles, Rpl stages, raw
// orbital stages, the pair tables
static size_t twoe_pipe_smem(int R, int KT, int n) {
  return sizeof(double) * 5 * (size_t)(16 * R) * (KT + 4) + sizeof(double2) * 6 * (size_t)n * KT +
         sizeof(int) * 3 * (size_t)(16 * R);
}
constexpr int kTwoeSmemMax = 227 * 1024;

template <int RR, bool SYM, int KT>
static int launch_twoe_pipe_t(Ctx& c, dim3 grid, size_t bytes, const double2* phi1, const double2* phi2,
                              const int* d_pa, const int* d_pb, const double* Rpl, int npair, int ntn,
                              long long xper, double* part, int strict) {
  // process-wide attribute, one fixed value (thread-safe static initialisation)
  static const cudaError_t attr = cudaFuncSetAttribute(twoe_dmma_kernel<RR, SYM, KT>,
                                                       cudaFuncAttributeMaxDynamicSharedMemorySize, kTwoeSmemMax);
  SG_CUDA(attr);
  twoe_dmma_kernel<RR, SYM, KT><<<grid, 64 * RR, bytes, c.stream>>>(phi1, phi2, d_pa, d_pb, Rpl, npair, c.nspf,
                                                                     c.G, ntn, xper, part, strict);
  return SINCGPU_OK;
}

// K stages of 32 points where the shared memory allows (half the stages and
// barriers of 16-point stages; the same bits), else 16
template <int RR>
static int launch_twoe_pipe(Ctx& c, dim3 grid, bool sym, const double2* phi1, const double2* phi2,
                            const int* d_pa, const int* d_pb, const double* Rpl, int npair, int ntn,
                            long long xper, double* part, int strict = 0) {
  const size_t b32 = twoe_pipe_smem(RR, 32, c.nspf), b16 = twoe_pipe_smem(RR, 16, c.nspf);
  if (b32 <= (size_t)kTwoeSmemMax)
    return sym ? launch_twoe_pipe_t<RR, true, 32>(c, grid, b32, phi1, phi2, d_pa, d_pb, Rpl, npair, ntn, xper, part,
                                                  0)
               : launch_twoe_pipe_t<RR, false, 32>(c, grid, b32, phi1, phi2, d_pa, d_pb, Rpl, npair, ntn, xper,
                                                   part, strict);
  return sym ? launch_twoe_pipe_t<RR, true, 16>(c, grid, b16, phi1, phi2, d_pa, d_pb, Rpl, npair, ntn, xper, part,
                                                0)
             : launch_twoe_pipe_t<RR, false, 16>(c, grid, b16, phi1, phi2, d_pa, d_pb, Rpl, npair, ntn, xper, part,
                                                 strict);
}

static void pair_lut(int n, const int* pa, const int* pb, int npair, bool herm, std::vector<int>& lut) {
  lut.assign((size_t)n * n, 0);
  for (int p = 0; p < npair; ++p) {
    if (herm) {
      lut[pa[p] + n * pb[p]] = 2 * p;
      if (pa[p] != pb[p]) lut[pb[p] + n * pa[p]] = 2 * p + 1;
    } else {
      lut[pa[p] + n * pb[p]] = p;
    }
  }
}

int twoe_matel(Ctx& c, const double2* phi1, const double2* phi2, const int* h_pa, const int* h_pb,
               int npair, const double* Rpl, bool herm, double2* twoematel) {
  const int n = c.nspf;
  SG_CHECK(n <= kMaxOrb, SINCGPU_ERANGE, "at most %d orbitals (got %d)", kMaxOrb, n);
  const int M = 2 * npair;
  // register block R: the smallest of 2..9 whose 16R tile holds M, else 8 (multi-tile)
  // tile edge 16R with the least padding of M (ties: the larger tile)
  int R = 2;
  for (int r = 2; r <= 9; ++r)
    if (ceil_div(M, 16 * r) * 16 * r <= ceil_div(M, 16 * R) * 16 * R) R = r;
  if (c.twoe_tile >= 2 && c.twoe_tile <= 9) R = c.twoe_tile;
  const int TT = 16 * R;
  const int ntm = ceil_div(M, TT), ntn = ntm;
  const int ntiles = ntm * (ntm + 1) / 2;  // upper triangle
  long long target = 148;  // one 256-thread CTA per SM (R x R accumulators per thread)
  int nsplit = (int)std::max(1LL, std::min((long long)ceil_div(c.G, TK), std::max(1LL, target / ntiles)));
  long long xper = ((c.G + nsplit - 1) / nsplit + TK - 1) / TK * TK;
  nsplit = ceil_div(c.G, xper);
  const long long MM = (long long)M * M;
  size_t need = sizeof(double) * (MM * nsplit + MM);
  SG_TRY(c.ws_twoe.ensure(need));
  double* part = (double*)c.ws_twoe.ptr;
  double* C = part + MM * nsplit;
  const int *d_pa, *d_pb, *d_lut;
  std::vector<int> lut;
  pair_lut(n, h_pa, h_pb, npair, herm, lut);
  SG_TRY(cached_ints(c, IC_PA, h_pa, npair, &d_pa));
  SG_TRY(cached_ints(c, IC_PB, h_pb, npair, &d_pb));
  SG_TRY(cached_ints(c, IC_LUT, lut.data(), (size_t)n * n, &d_lut));
  bool sym = false;
  {
    ProfScope ps(c, ST_TWOE_GEMM);
    const int TS = c.twoe_dmma ? TK + 4 : TK + 1;
    const size_t sbytes = sizeof(double) * 3 * (size_t)TT * TS + sizeof(double2) * 4 * (size_t)n * TK +
                          sizeof(int) * 3 * (size_t)TT;
    const dim3 grid(ntiles, nsplit);
    // the pipelined kernel copies whole complex values (16 bytes)
    const bool pipe = ((uintptr_t)phi1 % 16 == 0) && ((uintptr_t)phi2 % 16 == 0);
    // hermitian pairs make the pair matrix symmetric: a diagonal tile needs only
    // its blocks on and below the diagonal (the SYM kernel); with several tiles
    // (option twoe_symdiag) the diagonal tiles take that kernel and the strictly
    // upper ones the full one
    sym = pipe && herm && c.twoe_dmma && (ntm == 1 || c.twoe_symdiag);
#define SG_TWOE_LAUNCH(RR, DM)                                                                             \
  if (DM && pipe && sym && ntm > 1) {                                                                      \
    SG_TRY(launch_twoe_pipe<RR>(c, dim3(ntm, nsplit), true, phi1, phi2, d_pa, d_pb, Rpl, npair, ntn, xper,  \
                                part));                                                                    \
    SG_TRY(launch_twoe_pipe<RR>(c, dim3(ntm * (ntm - 1) / 2, nsplit), false, phi1, phi2, d_pa, d_pb, Rpl,   \
                                npair, ntn, xper, part, 1));                                               \
  } else if (DM && pipe) {                                                                                 \
    SG_TRY(launch_twoe_pipe<RR>(c, grid, sym, phi1, phi2, d_pa, d_pb, Rpl, npair, ntn, xper, part));        \
  } else {                                                                                                 \
    static const cudaError_t attr = cudaFuncSetAttribute(                                                  \
        twoe_gemm3_kernel<RR, DM>, cudaFuncAttributeMaxDynamicSharedMemorySize,                            \
        (int)(sizeof(double) * 3 * 16 * RR * (TK + 4) + sizeof(double2) * 4 * kMaxOrb * TK +                \
              sizeof(int) * 3 * 16 * RR));                                                                 \
    SG_CUDA(attr);                                                                                         \
    twoe_gemm3_kernel<RR, DM><<<grid, DM ? 64 * RR : 256, sbytes, c.stream>>>(phi1, phi2, d_pa, d_pb, Rpl,   \
                                                                          npair, n, c.G, ntn, xper, part); \
  }
#define SG_TWOE_CASE(RR)                \
  case RR:                              \
    if (c.twoe_dmma)                    \
      SG_TWOE_LAUNCH(RR, true)          \
    else                                \
      SG_TWOE_LAUNCH(RR, false)         \
    break;
    switch (R) {
      SG_TWOE_CASE(2)
      SG_TWOE_CASE(3)
      SG_TWOE_CASE(4)
      SG_TWOE_CASE(5)
      SG_TWOE_CASE(6)
      SG_TWOE_CASE(7)
      SG_TWOE_CASE(8)
      SG_TWOE_CASE(9)
      default:
        break;
    }
#undef SG_TWOE_CASE
#undef SG_TWOE_LAUNCH
    SG_LAUNCHED();
  }
  ProfScope ps(c, ST_TWOE_FINISH);
  split_reduce_kernel<<<ceil_div(MM, 32), 256, 0, c.stream>>>(part, nsplit, M, TT, C);
  SG_LAUNCHED();
  const long long n4 = (long long)n * n * n * n;
  twoe_assemble_kernel<<<ceil_div(n4, 256), 256, 0, c.stream>>>(C, d_lut, npair, n, herm ? 1 : 0,
                                                                 twoematel);
  SG_LAUNCHED();
  return SINCGPU_OK;
}

// ---------------------------------------------------------------------------
// reducedpot
// ---------------------------------------------------------------------------
// Wm[k][c], k < 2*npair, c < 2n^2 (column c = 2*(kk + n*ii) + re/im)
__global__ void build_w_kernel(const double2* __restrict__ tally, const int* __restrict__ pa,
                               const int* __restrict__ pb, int npair, int n, int herm,
                               double* __restrict__ Wm) {
  const int NC = 2 * n * n;
  long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (idx >= 2LL * npair * NC) return;
  int k = (int)(idx / NC), col = (int)(idx % NC);
  int p = k % npair, comp = k / npair;
  int cc = pa[p], d = pb[p];
  int ki = col / 2, kk = ki % n, ii = ki / n;
  long long tail = (long long)n * n * (kk + (long long)n * ii);
  double2 g1 = tally[cc + n * d + tail];
  double2 A, B;
  if (herm && cc != d) {
    double2 g2 = tally[d + n * cc + tail];
    A = cadd(g1, g2);
    double2 df = csub(g1, g2);
    B = make_double2(-df.y, df.x);
  } else {
    A = g1;
    B = make_double2(-g1.y, g1.x);
  }
  double2 v = comp == 0 ? A : B;
  Wm[idx] = (col & 1) ? v.y : v.x;
}

// Half-column W: columns c = 2t + {re, im} for the orbital pairs t = (kk, ii),
// kk <= ii, listed in tmap (kk, ii interleaved).  With a hermitian pair list and a
// 2-RDM of one A-vector (Gamma(c,d,k,i) = conj Gamma(d,c,i,k)), reducedpot(x,i,k)
// = conj reducedpot(x,k,i), so these columns determine all of it.
__global__ void build_w_half_kernel(const double2* __restrict__ tally, const int* __restrict__ pa,
                                    const int* __restrict__ pb, const int* __restrict__ tmap, int npair, int n,
                                    int nt, double* __restrict__ Wm) {
  const int NC = 2 * nt;
  long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (idx >= 2LL * npair * NC) return;
  int k = (int)(idx / NC), col = (int)(idx % NC);
  int p = k % npair, comp = k / npair;
  int cc = pa[p], d = pb[p];
  const int t = col / 2, kk = tmap[2 * t], ii = tmap[2 * t + 1];
  long long tail = (long long)n * n * (kk + (long long)n * ii);
  double2 g1 = tally[cc + n * d + tail];
  double2 A, B;
  if (cc != d) {
    double2 g2 = tally[d + n * cc + tail];
    A = cadd(g1, g2);
    double2 df = csub(g1, g2);
    B = make_double2(-df.y, df.x);
  } else {
    A = g1;
    B = make_double2(-g1.y, g1.x);
  }
  double2 v = comp == 0 ? A : B;
  Wm[idx] = (col & 1) ? v.y : v.x;
}

constexpr int RM = 128, RK = 16;

// reducedpot GEMM with 128 (x) x 4CG (columns) tiles, 16 x CG threads of 8x4
// register blocks; CG is chosen per call so that the 2n^2 columns pad least.
template <int CG, bool HALF>
__global__ void __launch_bounds__(16 * CG) rp_gemm3_kernel(const double* __restrict__ Rpl,
                                                           const double* __restrict__ Wm, int K, int NC,
                                                           long long G, double2* __restrict__ out,
                                                           const int* __restrict__ tmap, int n) {
  constexpr int NT = 16 * CG, TNC = 4 * CG;
  __shared__ __align__(16) double As[2][RK][RM];
  __shared__ __align__(16) double Bs[2][RK][TNC];
  const int tid = threadIdx.x, tx = tid % 16, ty = tid / 16;
  const long long x0 = (long long)blockIdx.x * RM;
  const int c0 = blockIdx.y * TNC;
  auto load = [&](int st, int k0) {
    for (int i = tid; i < RK * RM; i += NT) {
      const int k = i / RM, xx = i % RM;
      const long long x = x0 + xx;
      const bool ok = (k0 + k < K) && x < G;
      cp_async8(&As[st][k][xx], ok ? (const void*)(Rpl + (long long)(k0 + k) * G + x) : (const void*)Rpl, ok);
    }
    for (int i = tid; i < RK * TNC; i += NT) {
      const int k = i / TNC, cc = i % TNC;
      const bool ok = (k0 + k < K) && (c0 + cc < NC);
      cp_async8(&Bs[st][k][cc], ok ? (const void*)(Wm + (long long)(k0 + k) * NC + c0 + cc) : (const void*)Wm, ok);
    }
    cp_async_commit();
  };
  double acc[8][4];
#pragma unroll
  for (int i = 0; i < 8; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) acc[i][j] = 0.0;
  const int nk = (K + RK - 1) / RK;
  load(0, 0);
  for (int t = 0; t < nk; ++t) {
    const int st = t & 1;
    if (t + 1 < nk) {
      load(st ^ 1, (t + 1) * RK);
      cp_async_wait<1>();
    } else {
      cp_async_wait<0>();
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < RK; ++k) {
      double a[8], b[4];
#pragma unroll
      for (int i = 0; i < 8; ++i) a[i] = As[st][k][tx + 16 * i];
      const double2 b01 = *reinterpret_cast<const double2*>(&Bs[st][k][4 * ty]);
      const double2 b23 = *reinterpret_cast<const double2*>(&Bs[st][k][4 * ty + 2]);
      b[0] = b01.x;
      b[1] = b01.y;
      b[2] = b23.x;
      b[3] = b23.y;
#pragma unroll
      for (int i = 0; i < 8; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) acc[i][j] = fma(a[i], b[j], acc[i][j]);
    }
    __syncthreads();
  }
#pragma unroll
  for (int i = 0; i < 8; ++i) {
    const long long x = x0 + tx + 16 * i;
    if (x >= G) continue;
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const int col = c0 + 4 * ty + 2 * h;
      if (col >= NC) continue;
      const double2 v = make_double2(acc[i][2 * h], acc[i][2 * h + 1]);
      if (HALF) {
        const int t = col / 2, kk = tmap[2 * t], ii = tmap[2 * t + 1];
        out[(long long)(kk + n * ii) * G + x] = v;
        if (kk != ii) out[(long long)(ii + n * kk) * G + x] = make_double2(v.x, -v.y);
      } else {
        out[(long long)(col / 2) * G + x] = v;
      }
    }
  }
}

// reducedpot GEMM on the FP64 tensor cores (mma.sync m8n8k4 f64, the FP64 tensor
// path of sm_100a): CTA tile 64 (x) x 16 FN (columns), 8 warps (4 x 2) of
// 16 x 8 FN (2 x FN MMA tiles, 4 FN accumulators per thread), three CTAs per SM,
// K in chunks of 16 with a two-stage cp.async pipeline (deeper chunks and the
// third CTA measured faster than 8-deep chunks in three stages at two CTAs per
// SM).  One column tile covers all n(n+1) columns of the hermitian half for
// n <= 10 (FN = 7: 112 columns), so every Rpl row is read once.  Shared-memory rows are padded to 4 (mod 16) doubles so that
// the fragment loads (lane g + 4t reads row t, column g) are free of bank
// conflicts.  The accumulator pair (2t, 2t+1) of a fragment is one complex column
// pair (Re, Im) of reducedpot.
constexpr int DM = 64, DK = 16, DST = 2;
constexpr int DAS = DM + 4;


// the K loop of rp_dmma_kernel: acc (2 x FN fragments per warp) of the CTA's 64-point tile
template <int FN>
__device__ __forceinline__ void rp_dmma_mainloop(double (*As)[DK][DAS], double (*Bs)[DK][16 * FN + 4],
                                                 const double* __restrict__ Rpl, const double* __restrict__ Wm,
                                                 int K, int NC, long long G, long long x0, int c0,
                                                 double (&acc)[2][FN][2]) {
  constexpr int DN = 16 * FN;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int g = lane >> 2, t = lane & 3;
  const int wm = (warp & 3) * 16, wn = (warp >> 2) * 8 * FN;
  const int nk = (K + DK - 1) / DK;
  // Wm rows hold NC (even) doubles, so column pairs start on 16-byte boundaries
  auto load = [&](int st, int k0) {
#pragma unroll
    for (int q = 0; q < DK * DM / 256; ++q) {
      const int i = tid + 256 * q;
      const int k = i / DM, xx = i % DM;
      const long long x = x0 + xx;
      const bool ok = (k0 + k < K) && x < G;
      cp_async8(&As[st][k][xx], ok ? (const void*)(Rpl + (long long)(k0 + k) * G + x) : (const void*)Rpl, ok);
    }
    for (int i = tid; i < DK * DN / 2; i += 256) {
      const int k = i / (DN / 2), cc = 2 * (i % (DN / 2));
      const bool ok = (k0 + k < K) && (c0 + cc < NC);
      cp_async16(&Bs[st][k][cc], ok ? (const void*)(Wm + (long long)(k0 + k) * NC + c0 + cc) : (const void*)Wm,
                 ok);
    }
    cp_async_commit();
  };
#pragma unroll
  for (int i = 0; i < 2; ++i)
#pragma unroll
    for (int j = 0; j < FN; ++j) acc[i][j][0] = acc[i][j][1] = 0.0;
  load(0, 0);
  for (int kc = 0; kc < nk; ++kc) {
    const int st = kc % DST;
    cp_async_wait<0>();
    __syncthreads();  // chunk kc visible; every warp is done with chunk kc - 1
    if (kc + 1 < nk) load((kc + 1) % DST, (kc + 1) * DK);
#pragma unroll
    for (int k4 = 0; k4 < DK; k4 += 4) {
      double a[2], b[FN];
#pragma unroll
      for (int i = 0; i < 2; ++i) a[i] = As[st][k4 + t][wm + 8 * i + g];
#pragma unroll
      for (int j = 0; j < FN; ++j) b[j] = Bs[st][k4 + t][wn + 8 * j + g];
#pragma unroll
      for (int i = 0; i < 2; ++i)
#pragma unroll
        for (int j = 0; j < FN; ++j) dmma_884(acc[i][j], a[i], b[j]);
    }
  }
}

// reducedpot from the accumulators: column 2 tt + re/im; with HALF the pair
// tt = (kk <= ii) of tmap and its mirror (ii, kk) = conj
template <bool HALF, int FN>
__device__ __forceinline__ void rp_dmma_store(const double (&acc)[2][FN][2], long long G, long long x0, int c0,
                                              int NC, const int* __restrict__ tmap, int n,
                                              double2* __restrict__ out) {
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int g = lane >> 2, t = lane & 3;
  const int wm = (warp & 3) * 16, wn = (warp >> 2) * 8 * FN;
#pragma unroll
  for (int i = 0; i < 2; ++i) {
    const long long x = x0 + wm + 8 * i + g;
    if (x >= G) continue;
#pragma unroll
    for (int j = 0; j < FN; ++j) {
      const int col = c0 + wn + 8 * j + 2 * t;
      if (col >= NC) continue;
      const double2 v = make_double2(acc[i][j][0], acc[i][j][1]);
      if (HALF) {
        const int tt = col / 2, kk = tmap[2 * tt], ii = tmap[2 * tt + 1];
        out[(long long)(kk + n * ii) * G + x] = v;
        if (kk != ii) out[(long long)(ii + n * kk) * G + x] = make_double2(v.x, -v.y);
      } else {
        out[(long long)(col / 2) * G + x] = v;
      }
    }
  }
}

template <bool HALF, int FN>
__global__ void __launch_bounds__(256, 3) rp_dmma_kernel(const double* __restrict__ Rpl, const double* __restrict__ Wm,
                                                      int K, int NC, long long G, double2* __restrict__ out,
                                                      const int* __restrict__ tmap, int n) {
  __shared__ __align__(16) double As[DST][DK][DAS];
  __shared__ __align__(16) double Bs[DST][DK][16 * FN + 4];
  const long long x0 = (long long)blockIdx.x * DM;
  const int c0 = blockIdx.y * 16 * FN;
  double acc[2][FN][2];
  rp_dmma_mainloop<FN>(As, Bs, Rpl, Wm, K, NC, G, x0, c0, acc);
  rp_dmma_store<HALF, FN>(acc, G, x0, c0, NC, tmap, n, out);
}

// rp_dmma_kernel<true, FN> with the reduced-potential apply of actreduced00 in its
// epilogue (all n(n+1) half columns in the CTA's one column tile, n(n+1) <= 16 FN):
// after writing reducedpot the CTA keeps its 64 x n(n+1) tile in shared memory and
// forms, per point and orbital i, s_i = S_i + sum_k reducedpot(x,k,i) phi_k(x)
// (k ascending; the k > i terms from the mirrored pair) and then
// T_i = timefac sum_j s_j inv(j,i): redpot_kernel's arithmetic in its order, so
// the same bits, without reading the reducedpot it has just written back from
// HBM.  Dynamic shared memory: the K loop's stages, then the epilogue's tile.
constexpr int RPV = DM + 2;  // tile row stride (doubles): conflict-free accumulator stores
template <int FN>
__global__ void __launch_bounds__(256, 3) rp_apply_kernel(const double* __restrict__ Rpl, const double* __restrict__ Wm,
                                                       int K, int NC, long long G, double2* __restrict__ out,
                                                       const int* __restrict__ tmap, int n,
                                                       const double2* __restrict__ phi,
                                                       const double2* __restrict__ S,
                                                       const double2* __restrict__ inv, double2 timefac,
                                                       double2* __restrict__ T, const double2* __restrict__ proj,
                                                       double2* __restrict__ part) {
  extern __shared__ __align__(16) double rp_sm[];
  auto As = reinterpret_cast<double (*)[DK][DAS]>(rp_sm);
  auto Bs = reinterpret_cast<double (*)[DK][16 * FN + 4]>(rp_sm + DST * DK * DAS);
  const long long x0 = (long long)blockIdx.x * DM;
  double acc[2][FN][2];
  rp_dmma_mainloop<FN>(As, Bs, Rpl, Wm, K, NC, G, x0, 0, acc);
  rp_dmma_store<true, FN>(acc, G, x0, 0, NC, tmap, n, out);
  __syncthreads();  // every warp is done with the stages
  double* Vt = rp_sm;                                           // [NC][RPV]
  double2* ss = reinterpret_cast<double2*>(Vt + NC * RPV);      // [n][DM]
  double2* sinv = ss + n * DM;                                  // n*n
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int g = lane >> 2, t = lane & 3;
  const int wm = (warp & 3) * 16, wn = (warp >> 2) * 8 * FN;
#pragma unroll
  for (int i = 0; i < 2; ++i)
#pragma unroll
    for (int j = 0; j < FN; ++j) {
      const int col = wn + 8 * j + 2 * t, xx = wm + 8 * i + g;
      if (col < NC) {
        Vt[col * RPV + xx] = acc[i][j][0];
        Vt[(col + 1) * RPV + xx] = acc[i][j][1];
      }
    }
  for (int e = tid; e < n * n; e += 256) sinv[e] = inv[e];
  // this thread's point is the same for all its items (256 threads over 64 points):
  // its orbital values once, all loads in flight together (n <= kApplyOrb)
  static_assert(256 % DM == 0, "one point per thread");
  constexpr int kApplyOrb = 10;  // n(n+1) <= 16 FN <= 112
  const int pxx = tid % DM;
  const long long px = x0 + pxx;
  double2 ph[kApplyOrb];
#pragma unroll
  for (int k = 0; k < kApplyOrb; ++k)
    ph[k] = (k < n && px < G) ? phi[(long long)k * G + px] : make_double2(0.0, 0.0);
  __syncthreads();
  for (int it = tid; it < n * DM; it += 256) {
    const int i = it / DM, xx = it % DM;  // xx == pxx
    const long long x = x0 + xx;
    if (x >= G) continue;
    double2 a = S[(long long)i * G + x];
#pragma unroll
    for (int k = 0; k < kApplyOrb; ++k) {
      if (k < n) {
        const int tt = k <= i ? i * (i + 1) / 2 + k : k * (k + 1) / 2 + i;
        const double re = Vt[2 * tt * RPV + xx], im = Vt[(2 * tt + 1) * RPV + xx];
        cfma(a, make_double2(re, k <= i ? im : -im), ph[k]);
      }
    }
    ss[i * DM + xx] = a;
  }
  __syncthreads();  // the s values complete; every read of the reducedpot tile done
  // T of the tile, kept for the projector dots over the spent reducedpot tile
  double2* Tt = reinterpret_cast<double2*>(rp_sm);  // [n][DM]
  for (int it = tid; it < n * DM; it += 256) {
    const int i = it / DM, xx = it % DM;
    const long long x = x0 + xx;
    if (x >= G) {
      if (part) Tt[i * DM + xx] = make_double2(0.0, 0.0);
      continue;
    }
    double2 a = make_double2(0.0, 0.0);
    for (int j = 0; j < n; ++j) cfma(a, ss[j * DM + xx], sinv[j + n * i]);
    a = cmul(timefac, a);
    T[(long long)i * G + x] = a;
    if (part) Tt[i * DM + xx] = a;
  }
  if (!part) return;
  // projector-dot partials of this 64-point tile with dots_kernel's lane
  // assignment (two 32-point halves per lane), FMA order and shuffle tree
  __syncthreads();
  const int nn = n * n;
  for (int j = warp; j < n; j += 8) {
    double2 pv[DM / 32];
#pragma unroll
    for (int r = 0; r < DM / 32; ++r) {
      const long long x = x0 + r * 32 + lane;
      pv[r] = x < G ? proj[(long long)j * G + x] : make_double2(0.0, 0.0);
    }
    for (int i = 0; i < n; ++i) {
      double2 a = make_double2(0.0, 0.0);
#pragma unroll
      for (int r = 0; r < DM / 32; ++r) {  // conj(p) t
        const double2 p = pv[r], tv = Tt[i * DM + r * 32 + lane];
        a.x = fma(p.x, tv.x, fma(p.y, tv.y, a.x));
        a.y = fma(p.x, tv.y, fma(-p.y, tv.x, a.y));
      }
      for (int o = 16; o > 0; o >>= 1) {
        a.x += __shfl_down_sync(0xffffffffu, a.x, o);
        a.y += __shfl_down_sync(0xffffffffu, a.y, o);
      }
      if (lane == 0) part[(long long)blockIdx.x * nn + j + n * i] = a;
    }
  }
}

static size_t rp_apply_smem(int n, int NC, int FN) {
  const size_t stages = sizeof(double) * DST * DK * ((size_t)DAS + 16 * FN + 4);
  const size_t epi = sizeof(double) * (size_t)NC * RPV + sizeof(double2) * ((size_t)n * DM + (size_t)n * n);
  return std::max(stages, epi);
}

// column fragments per warp (CTA width 16 FN, FN <= 7 for the static shared
// memory) with the fewest padded columns of NC, the widest on ties
static int rp_dmma_fn(int NC) {
  int best = 7;
  long long waste = -1;
  for (int fn : {7, 6, 5, 4}) {
    const long long w = (long long)ceil_div(NC, 16 * fn) * 16 * fn - NC;
    if (waste < 0 || w < waste) {
      waste = w;
      best = fn;
    }
  }
  return best;
}

static int reduced_pot_impl(Ctx& c, const double* Rpl, const int* h_pa, const int* h_pb, int npair,
                            bool herm, const double2* tally, double2* reducedpot, bool half, RpApply* apply) {
  if (apply) apply->done = false;
  const int n = c.nspf;
  half = half && herm;
  const int nt = n * (n + 1) / 2;
  const int K = 2 * npair, NC = half ? 2 * nt : 2 * n * n;
  size_t need = sizeof(double) * (size_t)K * NC;
  SG_TRY(c.ws_gemm.ensure(need));
  double* Wm = (double*)c.ws_gemm.ptr;
  const int *d_pa, *d_pb, *d_tmap = nullptr;
  SG_TRY(cached_ints(c, IC_PA, h_pa, npair, &d_pa));
  SG_TRY(cached_ints(c, IC_PB, h_pb, npair, &d_pb));
  if (half) {
    std::vector<int> tm;
    tm.reserve(2 * (size_t)nt);
    for (int ii = 0; ii < n; ++ii)
      for (int kk = 0; kk <= ii; ++kk) {
        tm.push_back(kk);
        tm.push_back(ii);
      }
    SG_TRY(cached_ints(c, IC_TMAP, tm.data(), tm.size(), &d_tmap));
  }
  {
    ProfScope ps(c, ST_RP_W);
    if (half)
      build_w_half_kernel<<<ceil_div((long long)K * NC, 256), 256, 0, c.stream>>>(tally, d_pa, d_pb, d_tmap,
                                                                                  npair, n, nt, Wm);
    else
      build_w_kernel<<<ceil_div((long long)K * NC, 256), 256, 0, c.stream>>>(tally, d_pa, d_pb, npair, n,
                                                                             herm ? 1 : 0, Wm);
    SG_LAUNCHED();
  }
  // column groups: the CG in {8, 10, 12, 14, 16} (tiles of 4 CG columns) with the
  // fewest padded columns, the widest on ties
  int best = 16;
  long long waste = -1;
  for (int cg : {16, 14, 12, 10, 8}) {
    const long long w = (long long)ceil_div(NC, 4 * cg) * 4 * cg - NC;
    if (waste < 0 || w < waste) {
      waste = w;
      best = cg;
    }
  }
  ProfScope ps(c, ST_RP_GEMM);
  if (c.contract_tf32) return rp_gemm_tf32(c, Rpl, Wm, K, NC, half ? d_tmap : nullptr, reducedpot);
  if (c.rp_dmma) {
    const int fn = rp_dmma_fn(NC);
    const dim3 grid((unsigned)ceil_div(c.G, DM), (unsigned)ceil_div(NC, 16 * fn));
    // one column tile (n(n+1) <= 112, so n <= 10: the epilogue's per-thread orbital registers)
    if (apply && half && grid.y == 1 && n <= 10) {
      // process-wide attributes, one fixed value each (thread-safe static initialisation)
      static const cudaError_t attr = [] {
        const void* ks[] = {(const void*)rp_apply_kernel<4>, (const void*)rp_apply_kernel<5>,
                            (const void*)rp_apply_kernel<6>, (const void*)rp_apply_kernel<7>};
        for (const void* k : ks) {
          const cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                     (int)rp_apply_smem(10, 112, 7));
          if (e != cudaSuccess) return e;
        }
        return cudaSuccess;
      }();
      SG_CUDA(attr);
      if (apply->ready) SG_CUDA(cudaStreamWaitEvent(c.stream, apply->ready, 0));
      const size_t sm = rp_apply_smem(n, NC, fn);
#define SG_RP_APPLY(FN)                                                                                  \
  case FN:                                                                                               \
    rp_apply_kernel<FN><<<grid, 256, sm, c.stream>>>(Rpl, Wm, K, NC, c.G, reducedpot, d_tmap, n, apply->phi, \
                                                     apply->S, apply->inv, apply->timefac, apply->T,     \
                                                     apply->proj, apply->part);                          \
    break;
      switch (fn) {
        SG_RP_APPLY(4)
        SG_RP_APPLY(5)
        SG_RP_APPLY(6)
        default:
          SG_RP_APPLY(7)
      }
#undef SG_RP_APPLY
      SG_LAUNCHED();
      apply->done = true;
      return SINCGPU_OK;
    }
#define SG_RP_DMMA(FN)                                                                                   \
  case FN:                                                                                               \
    if (half)                                                                                            \
      rp_dmma_kernel<true, FN><<<grid, 256, 0, c.stream>>>(Rpl, Wm, K, NC, c.G, reducedpot, d_tmap, n);  \
    else                                                                                                 \
      rp_dmma_kernel<false, FN><<<grid, 256, 0, c.stream>>>(Rpl, Wm, K, NC, c.G, reducedpot, nullptr, n); \
    break;
    switch (fn) {
      SG_RP_DMMA(4)
      SG_RP_DMMA(5)
      SG_RP_DMMA(6)
      default:
        SG_RP_DMMA(7)
    }
#undef SG_RP_DMMA
    SG_LAUNCHED();
    return SINCGPU_OK;
  }
  const int gx = ceil_div(c.G, RM);
#define SG_RP_LAUNCH(CG)                                                                                   \
  if (half)                                                                                                \
    rp_gemm3_kernel<CG, true><<<dim3(gx, ceil_div(NC, 4 * CG)), 16 * CG, 0, c.stream>>>(Rpl, Wm, K, NC, c.G, \
                                                                                        reducedpot, d_tmap, n); \
  else                                                                                                     \
    rp_gemm3_kernel<CG, false><<<dim3(gx, ceil_div(NC, 4 * CG)), 16 * CG, 0, c.stream>>>(Rpl, Wm, K, NC, c.G, \
                                                                                         reducedpot, nullptr, n);
  switch (best) {
    case 8: SG_RP_LAUNCH(8) break;
    case 10: SG_RP_LAUNCH(10) break;
    case 12: SG_RP_LAUNCH(12) break;
    case 14: SG_RP_LAUNCH(14) break;
    default: SG_RP_LAUNCH(16) break;
  }
#undef SG_RP_LAUNCH
  SG_LAUNCHED();
  return SINCGPU_OK;
}

int reduced_pot(Ctx& c, const double* Rpl, const int* h_pa, const int* h_pb, int npair, bool herm,
                const double2* tally, double2* reducedpot, bool tally_herm, RpApply* apply) {
  return reduced_pot_impl(c, Rpl, h_pa, h_pb, npair, herm, tally, reducedpot, tally_herm, apply);
}

// twoereduced(G, n^2) interleaved -> planar rows for all ordered pairs
__global__ void to_planar_kernel(const double2* __restrict__ R, long long total, long long Gn2,
                                 double* __restrict__ Rpl) {
  long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= total) return;
  double2 v = R[i];
  Rpl[i] = v.x;
  Rpl[Gn2 + i] = v.y;
}

int reduced_pot_full(Ctx& c, const double2* twoereduced, const double2* tally, double2* reducedpot) {
  const int n = c.nspf;
  const int npair = n * n;
  std::vector<int> pa(npair), pb(npair);
  for (int b = 0; b < n; ++b)
    for (int a = 0; a < n; ++a) {
      pa[a + n * b] = a;
      pb[a + n * b] = b;
    }
  const long long total = c.G * npair;
  SG_TRY(c.ws_conv.ensure(sizeof(double) * 2 * total));
  double* Rpl = (double*)c.ws_conv.ptr;
  to_planar_kernel<<<ceil_div(total, 256), 256, 0, c.stream>>>(twoereduced, total, total, Rpl);
  SG_LAUNCHED();
  return reduced_pot_impl(c, Rpl, pa.data(), pb.data(), npair, false, tally, reducedpot, false, nullptr);
}

}  // namespace sincgpu
