// Coulomb pass kernels on the register two-step FFT (fft_reg.cuh), templated on
// the padded length P = P1*P2 and on the complex type C of the transforms:
// double2 (FP64 form) or float2 (FP32 precision form: pair products are formed
// in FP64 and rounded once, the spectra W1/W2, twiddles and kernel spectrum are
// FP32, and the potentials are widened back to FP64 on output).  See coulomb.cu
// for the algorithm and the passes.
#pragma once
#include <algorithm>
#include "context.hpp"
#include "fft_reg.cuh"
#include "tma.cuh"

namespace sincgpu {

// lines (rows or columns) per CTA of the x and y passes: fewer for long lines to
// stay within 48 KB of static shared memory
__host__ __device__ constexpr int lines_for(int P) { return P <= 128 ? 16 : 8; }

// lines per CTA of the z pass (forward, spectrum multiply, inverse: the most
// arithmetic per loaded line): the most of 32, 16, 8 whose exchange buffer and
// twiddle table fit in 46 KB, so that a CTA is a whole number of warps where the
// line length allows (measured: 9.9 vs 11.8 ms per evaluation on the 162-point
// grid, neutral on the 81-point one; the x and y passes were slower with more).
template <class C>
__host__ __device__ constexpr int lines_for_z(int P) {
  return ((P + 1) * 32 + P) * (int)sizeof(C) <= 46 * 1024   ? 32
         : ((P + 1) * 16 + P) * (int)sizeof(C) <= 46 * 1024 ? 16
                                                             : 8;
}
// lines per tile of the TMA-staged z pass (measured: capping it at 16 made the FP32
// pass on the 162-point grid slower, 4.1 -> 5.1 ms, and did not rescue P = 81)
template <class C>
__host__ __device__ constexpr int lines_for_ztma(int P) {
  return lines_for_z<C>(P);
}

template <class C>
struct CoulArgs {
  int N, P, nspf;
  long long G;
  const C* roots;
  const C* khat;
  C* W1;  // [pair][z][y<N][kx]
  C* W2;  // [pair][z<N][ky][kx]
  const int* pa;
  const int* pb;
  int pair0;        // index of the chunk's first pair in the full list
  int npair_total;  // planar output: Re at pair p, Im at npair_total + p
  int fused;        // 0: five passes (W1, W2); 1, 2, 4, 8: three passes (W1T), plane kernel on clusters of that size
  const typename CplxTraits<C>::Real* khT;  // real kernel spectrum [kx][kz][ky] (three-pass form)
  const typename CplxTraits<C>::Real* khr;  // real kernel spectrum: the octant k <= P/2 ((P/2+1)^3) for P <= 128, else all P^3
};

template <class C>
__device__ __forceinline__ void load_roots(C* roots, const C* g, int P) {
  for (int i = threadIdx.x; i < P; i += blockDim.x) roots[i] = g[i];
}

// CX: rows of rho -> DFT along x -> W1
template <int P1, int P2, bool DENS, class C>
__global__ void __launch_bounds__((P1 > P2 ? P1 : P2) * lines_for(P1 * P2)) coul_fwd_x_t(
    const double2* __restrict__ phi1, const double2* __restrict__ phi2, CoulArgs<C> ca) {
  constexpr int P = P1 * P2, S = P1 > P2 ? P1 : P2, TL = lines_for(P);
  __shared__ C roots[P];
  __shared__ C ex[(P + 1) * TL];
  load_roots(roots, ca.roots, P);
  const int N = ca.N;
  const int s = threadIdx.x % S, l = threadIdx.x / S;
  // pairs run fastest over the grid: the CTAs of one row block for all the
  // chunk's pairs run together and read the orbitals' rows from L2, so each
  // orbital is read from DRAM about once per launch instead of once per pair
  const int p = blockIdx.x, f = blockIdx.y * TL + l;  // row f = z*N + y
  const bool row = f < N * N;
  const long long off = (long long)f * N;
  const double2* s1;
  const double2* s2 = nullptr;
  if (DENS) {
    s1 = phi1 + (long long)(ca.pair0 + p) * ca.G + off;
  } else {
    s1 = phi1 + (long long)ca.pa[p] * ca.G + off;
    s2 = phi2 + (long long)ca.pb[p] * ca.G + off;
  }
  C a[P1], b[P2];
#pragma unroll
  for (int n1 = 0; n1 < P1; ++n1) {
    const int x = s + P2 * n1;
    double2 v = make_double2(0.0, 0.0);
    if (row && s < P2 && x < N) v = DENS ? s1[x] : cmulc(s1[x], s2[x]);
    a[n1] = cvt<C>(v);
  }
  __syncthreads();
  dft_in_to_out<P1, P2, false, C, true, false>(a, b, s, l, TL, ex, roots);
  if (row && s < P1) {
    C* dst = ca.W1 + ((long long)p * N * N + f) * P;
#pragma unroll
    for (int k2 = 0; k2 < P2; ++k2) dst[s + P1 * k2] = b[k2];
  }
}

// CY: W1 columns (y < N) -> DFT along y -> W2
template <int P1, int P2, class C>
__global__ void __launch_bounds__((P1 > P2 ? P1 : P2) * lines_for(P1 * P2)) coul_fwd_y_t(CoulArgs<C> ca) {
  constexpr int P = P1 * P2, TL = lines_for(P);
  __shared__ C roots[P];
  __shared__ C ex[P * TL];
  load_roots(roots, ca.roots, P);
  const int N = ca.N;
  const int l = threadIdx.x % TL, s = threadIdx.x / TL;
  const int p = blockIdx.z, f = blockIdx.x * TL + l;  // column f = z*P + kx
  const bool col = f < N * P;
  const int z = f / P, kx = f - z * P;
  const C* src = ca.W1 + ((long long)p * N + z) * N * P + kx;
  C a[P1], b[P2];
#pragma unroll
  for (int n1 = 0; n1 < P1; ++n1) {
    const int y = s + P2 * n1;
    a[n1] = (col && s < P2 && y < N) ? src[(long long)y * P] : CplxTraits<C>::make(0.0, 0.0);
  }
  __syncthreads();
  dft_in_to_out<P1, P2, false, C, false, false>(a, b, s, l, TL, ex, roots);
  if (col && s < P1) {
    C* dst = ca.W2 + ((long long)p * N + z) * P * P + kx;
#pragma unroll
    for (int k2 = 0; k2 < P2; ++k2) dst[(long long)(s + P1 * k2) * P] = b[k2];
  }
}

// CZ: W2 columns along z (z < N): forward, * khat, inverse, z < N written back.
// (At P = 162 in FP64 the kernel is register bound at two CTAs per SM; forcing
// three with spilled registers measured slower, 4.8 -> 5.9 ms per evaluation.)
template <int P1, int P2, class C>
__global__ void __launch_bounds__((P1 > P2 ? P1 : P2) * lines_for_z<C>(P1 * P2)) coul_z_t(CoulArgs<C> ca) {
  constexpr int P = P1 * P2, TL = lines_for_z<C>(P);
  __shared__ C roots[P];
  __shared__ C ex[P * TL];
  load_roots(roots, ca.roots, P);
  const int N = ca.N;
  const int l = threadIdx.x % TL, s = threadIdx.x / TL;
  const int p = blockIdx.z, f = blockIdx.x * TL + l;  // column f = ky*P + kx
  const long long zs = (long long)P * P;
  const bool col = f < zs;
  C* base = ca.W2 + (long long)p * N * zs + f;
  C a[P1], b[P2];
#pragma unroll
  for (int n1 = 0; n1 < P1; ++n1) {
    const int z = s + P2 * n1;
    a[n1] = (col && s < P2 && z < N) ? base[z * zs] : CplxTraits<C>::make(0.0, 0.0);
  }
  __syncthreads();
  dft_in_to_out<P1, P2, false, C>(a, b, s, l, TL, ex, roots);
  if (col && s < P1) {
    if constexpr (P <= 128) {
      // the spectrum is real and even in each axis: read it on the octant (a table
      // of (P/2+1)^3 values that stays in L2 while the W2 slab streams through).
      // Measured on the 41^3 grid (P = 81): z pass 0.165 -> 0.148 ms; on the 81^3
      // grid (P = 162) it was slower (4.8 -> 6.7 ms), so longer lines read the
      // real part of the whole table (below)
      using R = typename CplxTraits<C>::Real;
      constexpr int H = P / 2 + 1;
      const int ky = f / P, kx = f - ky * P;
      const R* kh = ca.khr + ((ky <= P - ky ? ky : P - ky) * H + (kx <= P - kx ? kx : P - kx));
#pragma unroll
      for (int k2 = 0; k2 < P2; ++k2) {
        const int kz = s + P1 * k2;
        const R w = kh[(kz <= P - kz ? kz : P - kz) * H * H];
        b[k2] = CplxTraits<C>::make(b[k2].x * w, b[k2].y * w);
      }
    } else {
      // longer lines: the real spectrum over the whole table, P^3 values with the
      // indexing of the complex one (P = 162: 34 MB, half the complex table's DRAM
      // re-reads per pair; z pass 4.80 -> 4.44 ms per evaluation on the 81^3 grid)
      using R = typename CplxTraits<C>::Real;
      const R* kh = ca.khr + f;
#pragma unroll
      for (int k2 = 0; k2 < P2; ++k2) {
        const R w = kh[(long long)(s + P1 * k2) * zs];
        b[k2] = CplxTraits<C>::make(b[k2].x * w, b[k2].y * w);
      }
    }
  }
  dft_out_to_in<P1, P2, true, C, false, false>(b, a, s, l, TL, ex, roots);
  if (col && s < P2) {
#pragma unroll
    for (int m1 = 0; m1 < P1; ++m1) {
      const int z = s + P2 * m1;
      if (z < N) base[z * zs] = a[m1];
    }
  }
}

// CZ for lengths P = P1 * P2 with P1 = 2 P2 (162 = 18 x 9): the plain z pass
// gives each line max(P1, P2) = P1 threads, and half of them idle in the steps
// with P2 sub-transforms (the loads, the first forward step, the last inverse
// step, the stores) while the others wait at the exchange barrier.  Here a line
// has P2 threads: thread s does sub-transform s of length P1 in those steps and
// the two sub-transforms s and s + P2 of length P2 in the others, so every
// thread works in every step and a CTA holds twice the lines for the same
// threads.  Same arithmetic in the same order as coul_z_t.
template <int P1, int P2>
__host__ __device__ constexpr int lines_for_z2() { return 32; }

template <int P1, int P2, class C>
__global__ void __launch_bounds__(P2 * lines_for_z2<P1, P2>(), 2) coul_z2_t(CoulArgs<C> ca) {
  static_assert(P1 == 2 * P2, "paired z pass needs P1 = 2 P2");
  constexpr int P = P1 * P2, TL = lines_for_z2<P1, P2>();
  extern __shared__ __align__(16) unsigned char z2_raw[];
  C* roots = reinterpret_cast<C*>(z2_raw);
  C* ex = roots + P;
  load_roots(roots, ca.roots, P);
  const int N = ca.N;
  const int l = threadIdx.x % TL, s = threadIdx.x / TL;  // s < P2
  const int p = blockIdx.z, f = blockIdx.x * TL + l;    // column f = ky*P + kx
  const long long zs = (long long)P * P;
  const bool col = f < zs;
  C* base = ca.W2 + (long long)p * N * zs + f;
  const C zero = CplxTraits<C>::make(0.0, 0.0);
  auto X = [&](int e) -> C& { return ex[e * TL + l]; };
  C a[P1], b0[P2], b1[P2];
#pragma unroll
  for (int n1 = 0; n1 < P1; ++n1) {
    const int z = s + P2 * n1;
    a[n1] = (col && z < N) ? base[z * zs] : zero;
  }
  __syncthreads();  // twiddles
  // forward step 1: sub-transform s of length P1
  RegFFT<P1, 1, false, C>::run(a, ConstRoots<P, C>{}, P);
#pragma unroll
  for (int k1 = 0; k1 < P1; ++k1) {
    C v = a[k1];
    if (k1 > 0 && s > 0) v = cmul(v, root<false>(roots, s * k1));
    X(k1 * P2 + s) = v;
  }
  __syncthreads();
  // forward step 2: sub-transforms t = s and t = s + P2 of length P2
#pragma unroll
  for (int n2 = 0; n2 < P2; ++n2) {
    b0[n2] = X(s * P2 + n2);
    b1[n2] = X((s + P2) * P2 + n2);
  }
  RegFFT<P2, 1, false, C>::run(b0, ConstRoots<P, C>{}, P);
  RegFFT<P2, 1, false, C>::run(b1, ConstRoots<P, C>{}, P);
  if (col) {
    // the real spectrum over the whole table, as coul_z_t reads it at these lengths
    using R = typename CplxTraits<C>::Real;
    const R* kh = ca.khr + f;
#pragma unroll
    for (int k2 = 0; k2 < P2; ++k2) {
      const R w0 = kh[(long long)(s + P1 * k2) * zs], w1 = kh[(long long)(s + P2 + P1 * k2) * zs];
      b0[k2] = CplxTraits<C>::make(b0[k2].x * w0, b0[k2].y * w0);
      b1[k2] = CplxTraits<C>::make(b1[k2].x * w1, b1[k2].y * w1);
    }
  }
  __syncthreads();  // the exchange is read before the inverse writes it
  // inverse step 1: sub-transforms t = s and t = s + P2 of length P2
  RegFFT<P2, 1, true, C>::run(b0, ConstRoots<P, C>{}, P);
  RegFFT<P2, 1, true, C>::run(b1, ConstRoots<P, C>{}, P);
#pragma unroll
  for (int m2 = 0; m2 < P2; ++m2) {
    C v0 = b0[m2], v1 = b1[m2];
    if (m2 > 0) {
      if (s > 0) v0 = cmul(v0, root<true>(roots, s * m2));
      v1 = cmul(v1, root<true>(roots, (s + P2) * m2));
    }
    X(m2 * P1 + s) = v0;
    X(m2 * P1 + s + P2) = v1;
  }
  __syncthreads();
  // inverse step 2: sub-transform s of length P1; z = s + P2 m1
#pragma unroll
  for (int k1 = 0; k1 < P1; ++k1) a[k1] = X(s * P1 + k1);
  RegFFT<P1, 1, true, C>::run(a, ConstRoots<P, C>{}, P);
  if (col) {
#pragma unroll
    for (int m1 = 0; m1 < P1; ++m1) {
      const int z = s + P2 * m1;
      if (z < N) base[z * zs] = a[m1];
    }
  }
}

// CZ with TMA-staged slabs: a persistent CTA walks its tiles of TL consecutive
// (ky, kx) columns; the tile's N z-planes (an N x TL slab of W2) arrive in shared
// memory by one tiled bulk tensor load, two tiles ahead of the computation (two
// buffers, one mbarrier each), so the transforms never wait on global loads of
// W2.  The kernel spectrum is real (the Coulomb kernel is real and even): its
// real part for the thread's frequencies is loaded before the slab is awaited.
// Same arithmetic as coul_z_t otherwise.  `err` is set when a slab never
// arrives (bounded waits; the CTA then stops instead of hanging).
template <int P1, int P2, class C>
__global__ void __launch_bounds__((P1 > P2 ? P1 : P2) * lines_for_ztma<C>(P1 * P2))
    coul_z_tma_t(CoulArgs<C> ca, const __grid_constant__ CUtensorMap zmap, int ntiles_f, int ntiles,
                 size_t slab_stride, int* __restrict__ err) {
  using R = typename CplxTraits<C>::Real;
  constexpr int P = P1 * P2, TL = lines_for_ztma<C>(P);
  constexpr uint32_t kLimit = 1u << 26;
  __shared__ C roots[P];
  __shared__ C ex[P * TL];
  __shared__ __align__(8) uint64_t full[2];
  extern __shared__ __align__(128) unsigned char slab_raw[];
  load_roots(roots, ca.roots, P);
  const int N = ca.N;
  const int tid = threadIdx.x, l = tid % TL, s = tid / TL;
  const long long zs = (long long)P * P;
  const uint32_t slab_bytes = (uint32_t)(N * TL * sizeof(C));
  auto slab = [&](int b) { return reinterpret_cast<C*>(slab_raw + b * slab_stride); };
  auto issue = [&](int t, int b) {
    const int p = t / ntiles_f, f0 = (t - p * ntiles_f) * TL;
    tma::mbar_arrive_expect_tx(&full[b], slab_bytes);
    tma::load_3d(slab(b), &zmap, 2 * f0, 0, p, &full[b]);
  };
  if (tid == 0) {
    tma::mbar_init(&full[0], 1);
    tma::mbar_init(&full[1], 1);
  }
  __syncthreads();
  if (tid == 0) {
    if (blockIdx.x < ntiles) issue(blockIdx.x, 0);
    if (blockIdx.x + gridDim.x < ntiles) issue(blockIdx.x + gridDim.x, 1);
  }
  int i = 0;
  for (int t = blockIdx.x; t < ntiles; t += gridDim.x, ++i) {
    const int b = i & 1;
    const int p = t / ntiles_f, f = (t - p * ntiles_f) * TL + l;
    const bool col = f < zs;
    R kh[P2];
    if (col && s < P1) {
      if constexpr (P > 128) {
        // the real table over all P^3 frequencies (built at these lengths)
        const R* khr = ca.khr + f;
#pragma unroll
        for (int k2 = 0; k2 < P2; ++k2) kh[k2] = khr[(long long)(s + P1 * k2) * zs];
      } else {
        const R* khr = reinterpret_cast<const R*>(ca.khat + f);
#pragma unroll
        for (int k2 = 0; k2 < P2; ++k2) kh[k2] = khr[2 * (long long)(s + P1 * k2) * zs];
      }
    }
    const bool arrived = tma::mbar_wait(&full[b], (i >> 1) & 1, kLimit);
    if (__syncthreads_or(!arrived)) {
      if (tid == 0) {
        atomicExch(err, 1);
        // let the other buffer's load (if any) land before the CTA leaves
        tma::mbar_wait(&full[b ^ 1], ((i + 1) >> 1) & 1, kLimit);
      }
      return;
    }
    C a[P1], bb[P2];
    const C* sl = slab(b);
#pragma unroll
    for (int n1 = 0; n1 < P1; ++n1) {
      const int z = s + P2 * n1;
      a[n1] = (col && s < P2 && z < N) ? sl[z * TL + l] : CplxTraits<C>::make(0.0, 0.0);
    }
    __syncthreads();  // the slab is read: its buffer takes the tile two steps ahead
    if (tid == 0 && t + 2 * (int)gridDim.x < ntiles) {
      tma::fence_proxy_async();
      issue(t + 2 * gridDim.x, b);
    }
    dft_in_to_out<P1, P2, false, C>(a, bb, s, l, TL, ex, roots);
    if (col && s < P1) {
#pragma unroll
      for (int k2 = 0; k2 < P2; ++k2) bb[k2] = CplxTraits<C>::make(bb[k2].x * kh[k2], bb[k2].y * kh[k2]);
    }
    dft_out_to_in<P1, P2, true, C, false, false>(bb, a, s, l, TL, ex, roots);
    if (col && s < P2) {
      C* base = ca.W2 + (long long)p * N * zs + f;
#pragma unroll
      for (int m1 = 0; m1 < P1; ++m1) {
        const int z = s + P2 * m1;
        if (z < N) base[z * zs] = a[m1];
      }
    }
  }
}

// CYI: W2 columns along ky (all P) -> inverse DFT -> W1 (y < N)
template <int P1, int P2, class C>
__global__ void __launch_bounds__((P1 > P2 ? P1 : P2) * lines_for(P1 * P2)) coul_inv_y_t(CoulArgs<C> ca) {
  constexpr int P = P1 * P2, TL = lines_for(P);
  __shared__ C roots[P];
  __shared__ C ex[P * TL];
  load_roots(roots, ca.roots, P);
  const int N = ca.N;
  const int l = threadIdx.x % TL, s = threadIdx.x / TL;
  const int p = blockIdx.z, f = blockIdx.x * TL + l;  // column f = z*P + kx
  const bool col = f < N * P;
  const int z = f / P, kx = f - z * P;
  const C* src = ca.W2 + ((long long)p * N + z) * P * P + kx;
  C a[P1], b[P2];
#pragma unroll
  for (int n1 = 0; n1 < P1; ++n1)
    a[n1] = (col && s < P2) ? src[(long long)(s + P2 * n1) * P] : CplxTraits<C>::make(0.0, 0.0);
  __syncthreads();
  dft_in_to_out<P1, P2, true, C, false, false>(a, b, s, l, TL, ex, roots);
  if (col && s < P1) {
    C* dst = ca.W1 + ((long long)p * N + z) * N * P + kx;
#pragma unroll
    for (int k2 = 0; k2 < P2; ++k2) {
      const int y = s + P1 * k2;
      if (y < N) dst[(long long)y * P] = b[k2];
    }
  }
}

// CXI: W1 rows along kx -> inverse DFT -> R (x < N)
template <int P1, int P2, bool DENS, class C>
__global__ void __launch_bounds__((P1 > P2 ? P1 : P2) * lines_for(P1 * P2)) coul_inv_x_t(
    CoulArgs<C> ca, double* __restrict__ Rpl, double2* __restrict__ full, int herm) {
  constexpr int P = P1 * P2, S = P1 > P2 ? P1 : P2, TL = lines_for(P);
  __shared__ C roots[P];
  __shared__ C ex[(P + 1) * TL];
  load_roots(roots, ca.roots, P);
  const int N = ca.N;
  const int s = threadIdx.x % S, l = threadIdx.x / S;
  const int p = blockIdx.z, f = blockIdx.x * TL + l;  // row f = z*N + y
  const bool row = f < N * N;
  const C* src = ca.W1 + ((long long)p * N * N + f) * P;
  C a[P1], b[P2];
#pragma unroll
  for (int n1 = 0; n1 < P1; ++n1)
    a[n1] = (row && s < P2) ? src[s + P2 * n1] : CplxTraits<C>::make(0.0, 0.0);
  __syncthreads();
  dft_in_to_out<P1, P2, true, C, true, false>(a, b, s, l, TL, ex, roots);
  if (!(row && s < P1)) return;
  const long long G = ca.G;
  const long long g0 = (long long)f * N;
  const int gp = ca.pair0 + p;
  long long off_ab, off_ba = 0;
  bool mirror = false;
  if (DENS) {
    off_ab = G * gp;
  } else {
    const int pa = ca.pa[p], pb = ca.pb[p];
    off_ab = G * ((long long)pa + (long long)ca.nspf * pb);
    off_ba = G * ((long long)pb + (long long)ca.nspf * pa);
    mirror = herm && pa != pb;
  }
#pragma unroll
  for (int k2 = 0; k2 < P2; ++k2) {
    const int x = s + P1 * k2;
    if (x < N) {
      const double2 v = widen(b[k2]);
      const long long g = g0 + x;
      if (Rpl) {
        Rpl[(long long)gp * G + g] = v.x;
        Rpl[(long long)(ca.npair_total + gp) * G + g] = v.y;
      }
      if (full) {
        full[off_ab + g] = v;
        if (mirror) full[off_ba + g] = cconj(v);
      }
    }
  }
}

}  // namespace sincgpu
#include "coulomb_fused.cuh"
namespace sincgpu {

// Launches the five passes for one chunk of np pairs (or, with ca.fused, the
// three passes of coulomb_fused.cuh).  With `zmap` (a tensor map
// of the chunk's W2 as [pair][z][2 P^2 reals]) the z pass is the TMA-staged
// persistent kernel, else the plain one.
template <int P1, int P2, class C>
int coul_launch(Ctx& c, const CoulArgs<C>& ca, int np, bool dens, const double2* src1,
                const double2* src2, double* Rpl, double2* full, bool herm, const CUtensorMap* zmap,
                int* err) {
  constexpr int P = P1 * P2, S = P1 > P2 ? P1 : P2, TL = lines_for(P);
  const int N = ca.N;
  const int nthr = S * TL;
  // lines are flattened over the two outer axes so that no lane idles past the
  // end of a row of lines: rows f = z*N + y (x passes), columns f = z*P + kx
  // (y passes) and f = ky*P + kx (z pass)
  constexpr int TLZ = lines_for_z<C>(P);
  const int nrow = ceil_div(N * N, TL), ncol = ceil_div(N * P, TL), nzc = ceil_div(P * P, TLZ);
  if (ca.fused) {
    {
      ProfScope ps(c, ST_COUL_FWD_X);
      if (dens)
        coul_fwd_xT_t<P1, P2, true, C><<<dim3(nrow, 1, np), nthr, 0, c.stream>>>(src1, nullptr, ca);
      else
        coul_fwd_xT_t<P1, P2, false, C><<<dim3(nrow, 1, np), nthr, 0, c.stream>>>(src1, src2, ca);
      SG_LAUNCHED();
    }
    {
      ProfScope ps(c, ST_COUL_YZY);
      switch (ca.fused) {
        case 1: SG_TRY((launch_yzy<P1, P2, C, 1>(c, ca, np, ca.khT))); break;
        case 2: SG_TRY((launch_yzy<P1, P2, C, 2>(c, ca, np, ca.khT))); break;
        case 4: SG_TRY((launch_yzy<P1, P2, C, 4>(c, ca, np, ca.khT))); break;
        default: SG_TRY((launch_yzy<P1, P2, C, 8>(c, ca, np, ca.khT))); break;
      }
      SG_LAUNCHED();
    }
    {
      ProfScope ps(c, ST_COUL_INV_X);
      if (dens)
        coul_inv_xT_t<P1, P2, true, C><<<dim3(nrow, 1, np), nthr, 0, c.stream>>>(ca, Rpl, full, 0);
      else
        coul_inv_xT_t<P1, P2, false, C><<<dim3(nrow, 1, np), nthr, 0, c.stream>>>(ca, Rpl, full, herm ? 1 : 0);
      SG_LAUNCHED();
    }
    return SINCGPU_OK;
  }
  {
    ProfScope ps(c, ST_COUL_FWD_X);
    if (dens)
      coul_fwd_x_t<P1, P2, true, C><<<dim3(np, nrow), nthr, 0, c.stream>>>(src1, nullptr, ca);
    else
      coul_fwd_x_t<P1, P2, false, C><<<dim3(np, nrow), nthr, 0, c.stream>>>(src1, src2, ca);
    SG_LAUNCHED();
  }
  {
    ProfScope ps(c, ST_COUL_FWD_Y);
    coul_fwd_y_t<P1, P2, C><<<dim3(ncol, 1, np), nthr, 0, c.stream>>>(ca);
    SG_LAUNCHED();
  }
  {
    ProfScope ps(c, ST_COUL_Z);
    if (zmap) {
      constexpr int TLT = lines_for_ztma<C>(P);
      const size_t slab_stride = ((size_t)N * TLT * sizeof(C) + 127) / 128 * 128;
      const size_t dyn = 2 * slab_stride;
      static const cudaError_t attr = [] {
        cudaFuncAttributes fa{};
        cudaError_t e = cudaFuncGetAttributes(&fa, coul_z_tma_t<P1, P2, C>);
        if (e == cudaSuccess)
          e = cudaFuncSetAttribute(coul_z_tma_t<P1, P2, C>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   (int)(227 * 1024 - fa.sharedSizeBytes));
        return e;
      }();
      SG_CUDA(attr);
      int occ = 0;  // resident CTAs per SM at this slab size
      SG_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, coul_z_tma_t<P1, P2, C>, S * TLT, dyn));
      occ = std::max(occ, 1);
      int nsm = 148;
      cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, c.device);
      const int ntf = ceil_div(P * P, TLT), ntiles = ntf * np;
      const int grid = std::min(ntiles, nsm * occ);
      coul_z_tma_t<P1, P2, C><<<grid, S * TLT, dyn, c.stream>>>(ca, *zmap, ntf, ntiles, slab_stride, err);
    } else if constexpr (P1 == 2 * P2 && P > 128) {
      // (the paired pass reads the whole real spectrum table, built above 128)
      if (c.coul_z2) {
        constexpr int TL2 = lines_for_z2<P1, P2>();
        const size_t dyn = sizeof(C) * ((size_t)P + (size_t)P * TL2);
        static const cudaError_t attr = cudaFuncSetAttribute(
            coul_z2_t<P1, P2, C>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)dyn);
        SG_CUDA(attr);
        coul_z2_t<P1, P2, C><<<dim3(ceil_div(P * P, TL2), 1, np), P2 * TL2, dyn, c.stream>>>(ca);
      } else {
        coul_z_t<P1, P2, C><<<dim3(nzc, 1, np), S * TLZ, 0, c.stream>>>(ca);
      }
    } else {
      coul_z_t<P1, P2, C><<<dim3(nzc, 1, np), S * TLZ, 0, c.stream>>>(ca);
    }
    SG_LAUNCHED();
  }
  {
    ProfScope ps(c, ST_COUL_INV_Y);
    coul_inv_y_t<P1, P2, C><<<dim3(ncol, 1, np), nthr, 0, c.stream>>>(ca);
    SG_LAUNCHED();
  }
  {
    ProfScope ps(c, ST_COUL_INV_X);
    if (dens)
      coul_inv_x_t<P1, P2, true, C><<<dim3(nrow, 1, np), nthr, 0, c.stream>>>(ca, Rpl, full, 0);
    else
      coul_inv_x_t<P1, P2, false, C><<<dim3(nrow, 1, np), nthr, 0, c.stream>>>(ca, Rpl, full, herm ? 1 : 0);
    SG_LAUNCHED();
  }
  return SINCGPU_OK;
}


#define SINCGPU_DECLARE_LAUNCH(P, A, B)                                                             \
  extern template int coul_launch<A, B, double2>(Ctx&, const CoulArgs<double2>&, int, bool,         \
                                                 const double2*, const double2*, double*, double2*, \
                                                 bool, const CUtensorMap*, int*);                  \
  extern template int coul_launch<A, B, float2>(Ctx&, const CoulArgs<float2>&, int, bool,           \
                                                const double2*, const double2*, double*, double2*,  \
                                                bool, const CUtensorMap*, int*);
SINCGPU_FFT_LENGTHS(SINCGPU_DECLARE_LAUNCH)
#undef SINCGPU_DECLARE_LAUNCH

#define SINCGPU_INSTANTIATE_LAUNCH(P, A, B)                                                       \
  template int coul_launch<A, B, double2>(Ctx&, const CoulArgs<double2>&, int, bool,              \
                                          const double2*, const double2*, double*, double2*, bool,  \
                                          const CUtensorMap*, int*);                                \
  template int coul_launch<A, B, float2>(Ctx&, const CoulArgs<float2>&, int, bool,                \
                                         const double2*, const double2*, double*, double2*, bool,   \
                                         const CUtensorMap*, int*);

}  // namespace sincgpu
