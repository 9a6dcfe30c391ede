// One-sided (Hestenes) Jacobi SVD of a small complex matrix by one warp.
//
// A (n x n, n <= 32, column-major, leading dimension n) is copied to shared
// memory (leading dimension 32) and rotated in place by plane rotations of
// column pairs until every pair is orthogonal to 1e-15; V accumulates the same
// rotations from the identity.  On return A holds U S (column m = U_m s_m),
// V the right singular vectors and sv the singular values (column norms), so
// that A_in = (A S^-1) S V^H.  Lane k owns row k; the whole warp must call it.
#pragma once
#include "common.cuh"

namespace sincgpu {

__device__ __forceinline__ void hestenes_svd_warp(const double2* __restrict__ A_in, int n, double2* A,
                                                  double2* V, double* sv) {
  const int k = threadIdx.x;
  for (int j = 0; j < n; ++j) {
    if (k < n) {
      A[k + 32 * j] = A_in[k + n * j];
      V[k + 32 * j] = make_double2(k == j ? 1.0 : 0.0, 0.0);
    }
  }
  __syncwarp();
  for (int sweep = 0; sweep < 60; ++sweep) {
    int rotated = 0;
    for (int p = 0; p < n - 1; ++p)
      for (int q = p + 1; q < n; ++q) {
        double2 ap = k < n ? A[k + 32 * p] : make_double2(0, 0);
        double2 aq = k < n ? A[k + 32 * q] : make_double2(0, 0);
        double al = ap.x * ap.x + ap.y * ap.y;
        double be = aq.x * aq.x + aq.y * aq.y;
        double2 ga = cmulc(aq, ap);  // conj(ap) * aq
        for (int o = 16; o > 0; o >>= 1) {
          al += __shfl_xor_sync(0xffffffffu, al, o);
          be += __shfl_xor_sync(0xffffffffu, be, o);
          ga.x += __shfl_xor_sync(0xffffffffu, ga.x, o);
          ga.y += __shfl_xor_sync(0xffffffffu, ga.y, o);
        }
        const double g = sqrt(ga.x * ga.x + ga.y * ga.y);
        if (g <= 1e-15 * sqrt(al * be) || g == 0.0) continue;
        rotated = 1;
        const double zeta = (be - al) / (2.0 * g);
        const double t = (zeta >= 0 ? 1.0 : -1.0) / (fabs(zeta) + sqrt(1.0 + zeta * zeta));
        const double cs = 1.0 / sqrt(1.0 + t * t), sn = cs * t;
        const double2 ph = make_double2(ga.x / g, -ga.y / g);  // exp(-i phi)
        if (k < n) {
          double2 aqr = cmul(aq, ph);
          A[k + 32 * p] = make_double2(cs * ap.x - sn * aqr.x, cs * ap.y - sn * aqr.y);
          A[k + 32 * q] = make_double2(sn * ap.x + cs * aqr.x, sn * ap.y + cs * aqr.y);
          double2 vp = V[k + 32 * p], vq = cmul(V[k + 32 * q], ph);
          V[k + 32 * p] = make_double2(cs * vp.x - sn * vq.x, cs * vp.y - sn * vq.y);
          V[k + 32 * q] = make_double2(sn * vp.x + cs * vq.x, sn * vp.y + cs * vq.y);
        }
        __syncwarp();
      }
    if (!rotated) break;
  }
  for (int j = 0; j < n; ++j) {
    double2 a = k < n ? A[k + 32 * j] : make_double2(0, 0);
    double s2 = a.x * a.x + a.y * a.y;
    for (int o = 16; o > 0; o >>= 1) s2 += __shfl_xor_sync(0xffffffffu, s2, o);
    if (k == 0) sv[j] = sqrt(s2);
  }
  __syncwarp();
}

}  // namespace sincgpu
