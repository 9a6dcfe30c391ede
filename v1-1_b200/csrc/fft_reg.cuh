// Register-resident two-step FFT for the Coulomb passes.
//
// A line of length P = P1*P2 is transformed by P2 (or P1) threads with one
// exchange through shared memory (four-step Cooley-Tukey):
//   X[k1 + P1 k2] = sum_n2 W_P2^(n2 k2) W_P^(n2 k1) sum_n1 x[n2 + P2 n1] W_P1^(n1 k1)
// Distribution D_in : thread s = n2 (< P2) holds x[n2 + P2*n1], n1 = 0..P1-1
// Distribution D_out: thread s = k1 (< P1) holds X[k1 + P1*k2], k2 = 0..P2-1
//   dft_in_to_out : D_in  -> D_out   (forward or inverse)
//   dft_out_to_in : D_out -> D_in    (inverse of the above layout, forward or inverse)
// The sub-transforms of length P1 / P2 run fully unrolled in registers
// (compile-time mixed radix 2/3/4/5/7 Stockham), twiddles come from the table
// roots[m] = exp(-2 pi i m / P) in shared memory.  The complex type C is double2
// (the FP64 form) or float2 (the FP32 precision form).
#pragma once
#include <cmath>
#include <vector>
#include "fft_engine.cuh"
#include "fft_lengths.h"

namespace sincgpu {

// Twiddle tables of every FFT length in constant memory (this translation unit's
// copy): the sub-transforms' twiddles have compile-time indices, so they become
// constant-bank operands instead of shared-memory loads.  The table holds the
// same values as the contexts' shared-memory roots (long-double cos/sin rounded to
// double; the FP32 table rounds those doubles).
namespace {
__constant__ double2 c_roots64[root_total()];
__constant__ float2 c_roots32[root_total()];

int upload_roots_here() {
  std::vector<double2> h64(root_total());
  std::vector<float2> h32(root_total());
  for (int i = 0; i < kNumFftLens; ++i) {
    const int P = kFftLens[i], o = root_offset(P);
    for (int m = 0; m < P; ++m) {
      const long double ang = -2.0L * 3.14159265358979323846264338327950288L * (long double)m / (long double)P;
      h64[o + m] = make_double2((double)cosl(ang), (double)sinl(ang));
      h32[o + m] = make_float2((float)h64[o + m].x, (float)h64[o + m].y);
    }
  }
  if (cudaMemcpyToSymbol(c_roots64, h64.data(), sizeof(double2) * h64.size()) != cudaSuccess) return 1;
  if (cudaMemcpyToSymbol(c_roots32, h32.data(), sizeof(float2) * h32.size()) != cudaSuccess) return 1;
  return 0;
}
const int c_roots_registered = register_const_roots(&upload_roots_here);

template <class C>
struct CRootTable;
template <>
struct CRootTable<double2> {
  __device__ __forceinline__ static double2 at(int i) { return c_roots64[i]; }
};
template <>
struct CRootTable<float2> {
  __device__ __forceinline__ static float2 at(int i) { return c_roots32[i]; }
};
}  // namespace

// roots of length P from constant memory: ConstRoots<P, C>{}[m] = exp(-2 pi i m / P)
template <int P, class C>
struct ConstRoots {
  static constexpr int kOff = root_offset(P);
  static_assert(kOff >= 0, "FFT length missing from the twiddle table");
  __device__ __forceinline__ C operator[](int m) const { return CRootTable<C>::at(kOff + m); }
};

constexpr int first_radix(int m) {
  return m % 4 == 0 ? 4 : (m % 2 == 0 ? 2 : (m % 3 == 0 ? 3 : (m % 5 == 0 ? 5 : 7)));
}

// In-register DFT of compile-time length M (M divides P), stages from span L on.
template <int M, int L, bool INV, class C>
struct RegFFT {
  static constexpr int R = first_radix(M / L);
  template <class RT>
  __device__ __forceinline__ static void run(C (&a)[M], const RT& roots, int P) {
    C b[M];
    const int rstep = P / M;
#pragma unroll
    for (int j = 0; j < M / R; ++j) {
      const int k = j % L;
      C t[R];
#pragma unroll
      for (int q = 0; q < R; ++q) {
        C v = a[j + q * (M / R)];
        if (q > 0 && k > 0) v = cmul(v, root<INV>(roots, (q * k * (M / (L * R))) * rstep));
        t[q] = v;
      }
      Butterfly<R, INV, C>::run(t, roots, P);
#pragma unroll
      for (int q = 0; q < R; ++q) b[(j / L) * L * R + k + q * L] = t[q];
    }
#pragma unroll
    for (int i = 0; i < M; ++i) a[i] = b[i];
    RegFFT<M, L * R, INV, C>::run(a, roots, P);
  }
};
template <int M, bool INV, class C>
struct RegFFT<M, M, INV, C> {
  template <class RT>
  __device__ __forceinline__ static void run(C (&)[M], const RT&, int) {}
};

// ex: exchange buffer for TL lines.  Element e of line l sits at ex[e*TL + l]
// (element-major, for kernels whose lanes run over lines: column passes) or, with
// ROW, at ex[l*(P+1) + e] (line-major, for kernels whose lanes run along a line:
// row passes), so that consecutive lanes touch consecutive addresses either way.
// Threads with s >= P2 (step 1) or s >= P1 (step 2) idle in that step.
// On entry a[] holds D_in (valid for s < P2); on exit b[] holds D_out (valid for s < P1).
template <int P, bool ROW>
__device__ __forceinline__ int ex_at(int e, int l, int TL) {
  return ROW ? l * (P + 1) + e : e * TL + l;
}

// TRAIL = false drops the closing barrier where the caller never writes the
// exchange buffer again (or passes another barrier first).
template <int P1, int P2, bool INV, class C, bool ROW = false, bool TRAIL = true>
__device__ __forceinline__ void dft_in_to_out(C (&a)[P1], C (&b)[P2], int s, int l, int TL, C* ex,
                                              const C* roots) {
  constexpr int P = P1 * P2;
  if (s < P2) {
    RegFFT<P1, 1, INV, C>::run(a, ConstRoots<P, C>{}, P);
#pragma unroll
    for (int k1 = 0; k1 < P1; ++k1) {
      C v = a[k1];
      if (k1 > 0 && s > 0) v = cmul(v, root<INV>(roots, s * k1));
      ex[ex_at<P, ROW>(k1 * P2 + s, l, TL)] = v;
    }
  }
  __syncthreads();
  if (s < P1) {
#pragma unroll
    for (int n2 = 0; n2 < P2; ++n2) b[n2] = ex[ex_at<P, ROW>(s * P2 + n2, l, TL)];
    RegFFT<P2, 1, INV, C>::run(b, ConstRoots<P, C>{}, P);
  }
  if (TRAIL) __syncthreads();
}

// On entry b[] holds D_out (valid for s < P1); on exit a[] holds D_in (valid for s < P2).
template <int P1, int P2, bool INV, class C, bool ROW = false, bool TRAIL = true>
__device__ __forceinline__ void dft_out_to_in(C (&b)[P2], C (&a)[P1], int s, int l, int TL, C* ex,
                                              const C* roots) {
  constexpr int P = P1 * P2;
  if (s < P1) {
    RegFFT<P2, 1, INV, C>::run(b, ConstRoots<P, C>{}, P);
#pragma unroll
    for (int m2 = 0; m2 < P2; ++m2) {
      C v = b[m2];
      if (m2 > 0 && s > 0) v = cmul(v, root<INV>(roots, s * m2));
      ex[ex_at<P, ROW>(m2 * P1 + s, l, TL)] = v;
    }
  }
  __syncthreads();
  if (s < P2) {
#pragma unroll
    for (int k1 = 0; k1 < P1; ++k1) a[k1] = ex[ex_at<P, ROW>(s * P1 + k1, l, TL)];
    RegFFT<P1, 1, INV, C>::run(a, ConstRoots<P, C>{}, P);
  }
  if (TRAIL) __syncthreads();
}

}  // namespace sincgpu
