// In-shared-memory batched line FFT (Stockham auto-sort, mixed radix 2/3/4/5/7)
// and the radix butterflies shared with the register FFT (fft_reg.cuh).
//
// The Toeplitz Coulomb solve of the reference (SINCDVR/toeplitz_subs.f90:561-589)
// needs forward-unnormalised 3-D DFTs on a doubled grid (COREPROJECT/ftcore.f90
// uses DFFTPACK zfftf / FFTW_FORWARD).  The Stockham engine transforms a tile of
// lines held in shared memory (used at set-up for the kernel spectrum).
//
// Stage with radix r after a span L (product of the earlier radices):
//   for j in [0, P/r):  k = j mod L
//     y_q = sum_t x[j + t*P/r] * w^(t*k) * W_r^(t*q),   w = exp(-+2*pi*i/(L*r))
//     out[(j/L)*L*r + k + q*L] = y_q
// which ends in natural order with no bit reversal.  The butterflies are
// templates over the radix and the complex type (double2, or float2 for the
// precision form).
#pragma once
#include "common.cuh"

namespace sincgpu {

constexpr int kMaxRadices = 12;
constexpr int kMaxFftLen = 256;

struct FftPlan {
  int P;                    // transform length
  int nrad;                 // number of stages
  int rad[kMaxRadices];     // radix of each stage
};

// roots[m] = exp(-2*pi*i*m/P), m in [0,P).  Inverse transforms use conj(roots).
// `roots` is a shared-memory table or a constant-memory accessor (fft_reg.cuh).
template <bool INV, class RT>
__device__ __forceinline__ auto root(const RT& roots, int m) {
  auto w = roots[m];
  if (INV) w.y = -w.y;
  return w;
}

// -i*z (forward) or +i*z (inverse)
template <bool INV, class C>
__device__ __forceinline__ C mul_mi(C z) {
  C r;
  if (INV) {
    r.x = -z.y;
    r.y = z.x;
  } else {
    r.x = z.y;
    r.y = -z.x;
  }
  return r;
}

template <int R, bool INV, class C>
struct Butterfly;

template <bool INV, class C>
struct Butterfly<2, INV, C> {
  template <class RT>
  __device__ __forceinline__ static void run(C* a, const RT&, int) {
    C t0 = a[0], t1 = a[1];
    a[0] = cadd(t0, t1);
    a[1] = csub(t0, t1);
  }
};

template <bool INV, class C>
struct Butterfly<3, INV, C> {
  template <class RT>
  __device__ __forceinline__ static void run(C* a, const RT& roots, int P) {
    using Re = typename CplxTraits<C>::Real;
    // W_3 = exp(-+2 pi i/3) = (-1/2, s),  s = -+ sin(2 pi/3)
    const Re s = INV ? -roots[P / 3].y : roots[P / 3].y;
    const Re h = (Re)-0.5;
    C sum = cadd(a[1], a[2]);
    C dif = csub(a[1], a[2]);
    C m;
    m.x = fma(h, sum.x, a[0].x);
    m.y = fma(h, sum.y, a[0].y);
    a[0] = cadd(a[0], sum);
    a[1].x = fma(-s, dif.y, m.x);
    a[1].y = fma(s, dif.x, m.y);
    a[2].x = fma(s, dif.y, m.x);
    a[2].y = fma(-s, dif.x, m.y);
  }
};

template <bool INV, class C>
struct Butterfly<4, INV, C> {
  template <class RT>
  __device__ __forceinline__ static void run(C* a, const RT&, int) {
    C s02 = cadd(a[0], a[2]), d02 = csub(a[0], a[2]);
    C s13 = cadd(a[1], a[3]), d13 = csub(a[1], a[3]);
    C rot = mul_mi<INV>(d13);
    a[0] = cadd(s02, s13);
    a[2] = csub(s02, s13);
    a[1] = cadd(d02, rot);
    a[3] = csub(d02, rot);
  }
};

// odd prime radices: direct DFT with the symmetric pairing t <-> r-t
template <int R, bool INV, class C>
struct ButterflyOdd {
  template <class RT>
  __device__ __forceinline__ static void run(C* a, const RT& roots, int P) {
    const int step = P / R;
    C sp[(R - 1) / 2], sm[(R - 1) / 2];
#pragma unroll
    for (int t = 1; t <= (R - 1) / 2; ++t) {
      sp[t - 1] = cadd(a[t], a[R - t]);
      sm[t - 1] = csub(a[t], a[R - t]);
    }
    C y[R];
    C y0 = a[0];
#pragma unroll
    for (int t = 0; t < (R - 1) / 2; ++t) y0 = cadd(y0, sp[t]);
    y[0] = y0;
#pragma unroll
    for (int q = 1; q <= (R - 1) / 2; ++q) {
      C re = a[0];  // sum_t cos(2 pi t q / R) sp_t
      C im;         // sum_t sin-part of sm_t
      im.x = 0;
      im.y = 0;
#pragma unroll
      for (int t = 1; t <= (R - 1) / 2; ++t) {
        const C w = root<INV>(roots, ((t * q) % R) * step);  // (cos, -+sin)
        re.x = fma(w.x, sp[t - 1].x, re.x);
        re.y = fma(w.x, sp[t - 1].y, re.y);
        im.x = fma(w.y, sm[t - 1].x, im.x);
        im.y = fma(w.y, sm[t - 1].y, im.y);
      }
      // y_q = re + i*im,  y_{R-q} = re - i*im
      y[q].x = re.x - im.y;
      y[q].y = re.y + im.x;
      y[R - q].x = re.x + im.y;
      y[R - q].y = re.y - im.x;
    }
#pragma unroll
    for (int q = 0; q < R; ++q) a[q] = y[q];
  }
};
template <bool INV, class C>
struct Butterfly<5, INV, C> : ButterflyOdd<5, INV, C> {};
template <bool INV, class C>
struct Butterfly<7, INV, C> : ButterflyOdd<7, INV, C> {};

template <int R, bool INV>
__device__ __forceinline__ void fft_stage(const double2* __restrict__ src, double2* __restrict__ dst,
                                          int nlines, int lstride, int estride, int P, int L,
                                          const double2* roots, bool lines_fast) {
  const int Pr = P / R;
  const int tw = P / (L * R);
  const int nitems = nlines * Pr;
  for (int it = threadIdx.x; it < nitems; it += blockDim.x) {
    int l, j;
    if (lines_fast) {
      j = it / nlines;
      l = it - j * nlines;
    } else {
      l = it / Pr;
      j = it - l * Pr;
    }
    const int jL = j / L;
    const int k = j - jL * L;
    double2 a[R];
    const double2* sl = src + l * lstride;
#pragma unroll
    for (int t = 0; t < R; ++t) {
      double2 v = sl[(j + t * Pr) * estride];
      if (t > 0 && k > 0) v = cmul(v, root<INV>(roots, t * k * tw));
      a[t] = v;
    }
    Butterfly<R, INV, double2>::run(a, roots, P);
    double2* dl = dst + l * lstride;
    const int base = jL * L * R + k;
#pragma unroll
    for (int q = 0; q < R; ++q) dl[(base + q * L) * estride] = a[q];
  }
}

// Transforms `nlines` lines of length plan.P held in shared memory.
// Element (line l, index j) lives at buf[l*lstride + j*estride].
// `lines_fast` selects the work-item order: consecutive threads on consecutive
// lines (column tiles) or on consecutive indices of one line (row tiles).
// Returns the buffer holding the result (A or B); both must be distinct.
// The caller synchronises the block before the call; the call ends synchronised.
template <bool INV>
__device__ double2* fft_lines(double2* A, double2* B, int nlines, int lstride, int estride,
                              const FftPlan& plan, const double2* roots, bool lines_fast) {
  const int P = plan.P;
  int L = 1;
  double2* src = A;
  double2* dst = B;
  for (int s = 0; s < plan.nrad; ++s) {
    const int r = plan.rad[s];
    switch (r) {
      case 2: fft_stage<2, INV>(src, dst, nlines, lstride, estride, P, L, roots, lines_fast); break;
      case 3: fft_stage<3, INV>(src, dst, nlines, lstride, estride, P, L, roots, lines_fast); break;
      case 4: fft_stage<4, INV>(src, dst, nlines, lstride, estride, P, L, roots, lines_fast); break;
      case 5: fft_stage<5, INV>(src, dst, nlines, lstride, estride, P, L, roots, lines_fast); break;
      default: fft_stage<7, INV>(src, dst, nlines, lstride, estride, P, L, roots, lines_fast); break;
    }
    __syncthreads();
    double2* t = src;
    src = dst;
    dst = t;
    L *= r;
  }
  return src;
}

}  // namespace sincgpu
