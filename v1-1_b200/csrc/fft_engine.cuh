// In-shared-memory batched line FFT (Stockham auto-sort, mixed radix 2/3/4/5/7).
//
// The Toeplitz Coulomb solve of the reference (SINCDVR/toeplitz_subs.f90:561-589)
// needs forward-unnormalised 3-D DFTs on a doubled grid (COREPROJECT/ftcore.f90
// uses DFFTPACK zfftf / FFTW_FORWARD).  Here each CTA transforms a tile of lines
// that already sits in shared memory; the global-memory passes (coulomb.cu) decide
// which axis the lines run along.
//
// Stage with radix r after a span L (product of the earlier radices):
//   for j in [0, P/r):  k = j mod L
//     y_q = sum_t x[j + t*P/r] * w^(t*k) * W_r^(t*q),   w = exp(-+2*pi*i/(L*r))
//     out[(j/L)*L*r + k + q*L] = y_q
// which ends in natural order with no bit reversal.
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
template <bool INV>
__device__ __forceinline__ double2 root(const double2* roots, int m) {
  double2 w = roots[m];
  if (INV) w.y = -w.y;
  return w;
}

// One radix-r butterfly on r inputs already multiplied by their twiddles.
template <bool INV>
__device__ __forceinline__ void dft_small(double2* a, int r, const double2* roots, int P) {
  if (r == 2) {
    double2 t0 = a[0], t1 = a[1];
    a[0] = cadd(t0, t1);
    a[1] = csub(t0, t1);
  } else if (r == 3) {
    // W_3 = exp(-+2 pi i/3) = (-1/2, -+s)
    const double s = INV ? -roots[P / 3].y : roots[P / 3].y;  // = -+ sin(2pi/3)
    double2 sum = cadd(a[1], a[2]);
    double2 dif = csub(a[1], a[2]);
    double2 m = make_double2(a[0].x - 0.5 * sum.x, a[0].y - 0.5 * sum.y);
    // i*s*dif = (-s*dif.y, s*dif.x)
    a[0] = cadd(a[0], sum);
    a[1] = make_double2(m.x - s * dif.y, m.y + s * dif.x);
    a[2] = make_double2(m.x + s * dif.y, m.y - s * dif.x);
  } else if (r == 4) {
    double2 s02 = cadd(a[0], a[2]), d02 = csub(a[0], a[2]);
    double2 s13 = cadd(a[1], a[3]), d13 = csub(a[1], a[3]);
    // forward: W_4 = -i;  -i*d13 = (d13.y, -d13.x)
    double2 rot = INV ? make_double2(-d13.y, d13.x) : make_double2(d13.y, -d13.x);
    a[0] = cadd(s02, s13);
    a[2] = csub(s02, s13);
    a[1] = cadd(d02, rot);
    a[3] = csub(d02, rot);
  } else {
    double2 in[8];
#pragma unroll
    for (int t = 0; t < 8; ++t)
      if (t < r) in[t] = a[t];
    const int step = P / r;
    for (int q = 0; q < r; ++q) {
      double2 acc = in[0];
      for (int t = 1; t < r; ++t) {
        int e = (t * q) % r;
        acc = cadd(acc, cmul(in[t], root<INV>(roots, e * step)));
      }
      a[q] = acc;
    }
  }
}

// Transforms `nlines` lines of length plan.P held in shared memory.
// Element (line l, index j) lives at buf[l*lstride + j*estride].
// `lines_fast` selects the work-item order: consecutive threads on consecutive
// lines (column tiles) or on consecutive indices of one line (row tiles).
// Returns the buffer holding the result (A or B); both must be distinct.
template <bool INV>
__device__ double2* fft_lines(double2* A, double2* B, int nlines, int lstride, int estride,
                              const FftPlan& plan, const double2* roots, bool lines_fast) {
  const int P = plan.P;
  int L = 1;
  double2* src = A;
  double2* dst = B;
  for (int s = 0; s < plan.nrad; ++s) {
    const int r = plan.rad[s];
    const int Pr = P / r;
    const int tw = P / (L * r);
    const int nitems = nlines * Pr;
    for (int it = threadIdx.x; it < nitems; it += blockDim.x) {
      int l, j;
      if (lines_fast) {
        l = it % nlines;
        j = it / nlines;
      } else {
        j = it % Pr;
        l = it / Pr;
      }
      const int k = j % L;
      double2 a[8];
      const double2* sl = src + l * lstride;
#pragma unroll
      for (int t = 0; t < 8; ++t) {
        if (t < r) {
          double2 v = sl[(j + t * Pr) * estride];
          if (t > 0 && k > 0) v = cmul(v, root<INV>(roots, t * k * tw));
          a[t] = v;
        }
      }
      dft_small<INV>(a, r, roots, P);
      double2* dl = dst + l * lstride;
      const int base = (j / L) * L * r + k;
#pragma unroll
      for (int q = 0; q < 8; ++q)
        if (q < r) dl[(base + q * L) * estride] = a[q];
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
