// Per-axis sinc-DVR kinetic contraction on the FP64 tensor cores (DMMA).
//
// Reference: mult_ke (SINCDVR/coreproject.f90:2104-2116) -> mult_general_withbcast
// (1321-1390) -> mult_all0 (2070-2097), one ZGEMM per axis with the real matrix
// ketot(l,j) = K(j-l) stored as complex:
//   out(x,y,z) = sum_l K(x-l) in(l,y,z) + sum_l K(y-l) in(x,l,z) + sum_l K(z-l) in(x,y,l)
//
// Pass 1 (one CTA per xy plane):  O = X K + K X for the real and imaginary planes
//   of a z slice, both products accumulated into the same 8x8 tiles.
// Pass 2 (one CTA per xz plane):  O += K X' along z, read-modify-write.
// The real K is applied to real and imaginary parts separately (no 2x complex
// waste).  Tensor-core instruction: mma.sync.aligned.m8n8k4.row.col.f64
// (tcgen05 has no f64 kind; this is the FP64 tensor path of sm_100a).
// Pass 1 optionally fuses the diagonal terms of the orbital RHS:
//   + pot(x) in + zfield * z(x) in        (mult_pot, lenmultiply)
#include "context.hpp"

namespace sincgpu {

__device__ __forceinline__ void dmma884(double& d0, double& d1, double a, double b) {
  asm volatile(
      "mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
      : "+d"(d0), "+d"(d1)
      : "d"(a), "d"(b));
}

struct KeArgs {
  int N, S, n8, k4;
  long long G;
  const double* ketile;  // S x S, K(j-l) at [j*S + l], zero outside N
  const double* pot;
  const double* zdip;
  double zfield;
  int extra;
};

// pass 1: xy planes
__global__ void __launch_bounds__(256) ke_xy_kernel(const double2* __restrict__ in,
                                                    double2* __restrict__ out, KeArgs ka) {
  extern __shared__ double sm[];
  const int N = ka.N, S = ka.S, n8 = ka.n8;
  double* Ks = sm;             // n8 x S
  double* Xr = Ks + n8 * S;    // n8 x S
  double* Xi = Xr + n8 * S;    // n8 x S
  const int z = blockIdx.x, orb = blockIdx.y;
  const double2* src = in + (long long)orb * ka.G + (long long)z * N * N;
  // staged in batches of 8 elements per thread: all 8 loads are in flight before
  // the first shared-memory store
  for (int i0 = threadIdx.x; i0 < n8 * S; i0 += 8 * blockDim.x) {
    double kv[8];
    double2 xv[8];
#pragma unroll
    for (int r = 0; r < 8; ++r) {
      const int i = i0 + r * blockDim.x;
      const int y = i / S, x = i - y * S;
      kv[r] = i < n8 * S ? ka.ketile[i] : 0.0;
      xv[r] = (i < n8 * S && y < N && x < N) ? src[y * N + x] : make_double2(0.0, 0.0);
    }
#pragma unroll
    for (int r = 0; r < 8; ++r) {
      const int i = i0 + r * blockDim.x;
      if (i < n8 * S) {
        Ks[i] = kv[r];
        Xr[i] = xv[r].x;
        Xi[i] = xv[r].y;
      }
    }
  }
  __syncthreads();
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int g = lane >> 2, t = lane & 3;
  const int T = n8 >> 3;
  double2* dst = out + (long long)orb * ka.G + (long long)z * N * N;
  for (int job = warp; job < T * T; job += blockDim.x >> 5) {
    const int y0 = (job / T) * 8, x0 = (job % T) * 8;
    double r0 = 0, r1 = 0, i0 = 0, i1 = 0;
    for (int k = 0; k < ka.k4; k += 4) {
      // X K : A = X[y0+g][k+t], B = K[k+t][x0+g]
      double bK = Ks[(k + t) * S + x0 + g];
      dmma884(r0, r1, Xr[(y0 + g) * S + k + t], bK);
      dmma884(i0, i1, Xi[(y0 + g) * S + k + t], bK);
      // K X : A = K[y0+g][k+t], B = X[k+t][x0+g]
      double aK = Ks[(y0 + g) * S + k + t];
      dmma884(r0, r1, aK, Xr[(k + t) * S + x0 + g]);
      dmma884(i0, i1, aK, Xi[(k + t) * S + x0 + g]);
    }
    const int y = y0 + g;
    if (y < N) {
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const int x = x0 + 2 * t + h;
        if (x < N) {
          double vr = h ? r1 : r0, vi = h ? i1 : i0;
          if (ka.extra) {
            long long gidx = (long long)z * N * N + (long long)y * N + x;
            double f = ka.pot[gidx] + ka.zfield * ka.zdip[gidx];
            vr = fma(f, Xr[y * S + x], vr);
            vi = fma(f, Xi[y * S + x], vi);
          }
          dst[y * N + x] = make_double2(vr, vi);
        }
      }
    }
  }
}

// pass 2: xz planes, O'[z][x] = sum_l K[z][l] X'[l][x], added into out
__global__ void __launch_bounds__(256) ke_z_kernel(const double2* __restrict__ in,
                                                   double2* __restrict__ out, KeArgs ka) {
  extern __shared__ double sm[];
  const int N = ka.N, S = ka.S, n8 = ka.n8;
  double* Ks = sm;
  double* Xr = Ks + n8 * S;
  double* Xi = Xr + n8 * S;
  const int y = blockIdx.x, orb = blockIdx.y;
  const long long NN = (long long)N * N;
  const double2* src = in + (long long)orb * ka.G + (long long)y * N;
  for (int i0 = threadIdx.x; i0 < n8 * S; i0 += 8 * blockDim.x) {
    double kv[8];
    double2 xv[8];
#pragma unroll
    for (int r = 0; r < 8; ++r) {
      const int i = i0 + r * blockDim.x;
      const int zz = i / S, x = i - zz * S;
      kv[r] = i < n8 * S ? ka.ketile[i] : 0.0;
      xv[r] = (i < n8 * S && zz < N && x < N) ? src[zz * NN + x] : make_double2(0.0, 0.0);
    }
#pragma unroll
    for (int r = 0; r < 8; ++r) {
      const int i = i0 + r * blockDim.x;
      if (i < n8 * S) {
        Ks[i] = kv[r];
        Xr[i] = xv[r].x;
        Xi[i] = xv[r].y;
      }
    }
  }
  __syncthreads();
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int g = lane >> 2, t = lane & 3;
  const int T = n8 >> 3;
  double2* dst = out + (long long)orb * ka.G + (long long)y * N;
  for (int job = warp; job < T * T; job += blockDim.x >> 5) {
    const int z0 = (job / T) * 8, x0 = (job % T) * 8;
    const int zz = z0 + g;
    // the pass-1 values this lane adds to, loaded before the MMA chain so that
    // their latency overlaps it
    double2 prev[2];
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const int x = x0 + 2 * t + h;
      prev[h] = (zz < N && x < N) ? dst[zz * NN + x] : make_double2(0.0, 0.0);
    }
    double r0 = 0, r1 = 0, i0 = 0, i1 = 0;
    for (int k = 0; k < ka.k4; k += 4) {
      double aK = Ks[(z0 + g) * S + k + t];
      dmma884(r0, r1, aK, Xr[(k + t) * S + x0 + g]);
      dmma884(i0, i1, aK, Xi[(k + t) * S + x0 + g]);
    }
    if (zz < N) {
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const int x = x0 + 2 * t + h;
        if (x < N) {
          double2 v = prev[h];
          v.x += h ? r1 : r0;
          v.y += h ? i1 : i0;
          dst[zz * NN + x] = v;
        }
      }
    }
  }
}

int mult_ke_tf32(Ctx& c, const double2* in, double2* out, int howmany, bool extra, double zfield);  // contract_tc.cu

int mult_ke(Ctx& c, const double2* in, double2* out, int howmany, bool extra, double zfield) {
  if (c.ke_tf32) return mult_ke_tf32(c, in, out, howmany, extra, zfield);
  const int N = c.N;
  KeArgs ka{};
  ka.N = N;
  ka.S = c.ke_stride;
  ka.n8 = (N + 7) / 8 * 8;
  ka.k4 = (N + 3) / 4 * 4;
  ka.G = c.G;
  ka.ketile = c.d_ketile;
  ka.pot = c.d_pot;
  ka.zdip = c.d_zdip;
  ka.zfield = zfield;
  ka.extra = extra ? 1 : 0;
  const size_t smem = sizeof(double) * 3 * (size_t)ka.n8 * ka.S;
  SG_CHECK(smem <= 227 * 1024, SINCGPU_ERANGE, "kinetic kernel needs %zu bytes of shared memory (N=%d)",
           smem, N);
  SG_CHECK(howmany <= 65535, SINCGPU_ERANGE, "howmany %d too large", howmany);
  // process-wide attributes, one fixed value, set once (thread-safe static init)
  static const cudaError_t attr = [] {
    cudaError_t e = cudaFuncSetAttribute(ke_xy_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024);
    if (e == cudaSuccess)
      e = cudaFuncSetAttribute(ke_z_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024);
    return e;
  }();
  SG_CUDA(attr);
  {
    ProfScope ps(c, ST_KE_XY);
    ke_xy_kernel<<<dim3(N, howmany), 256, smem, c.stream>>>(in, out, ka);
    SG_LAUNCHED();
  }
  ProfScope ps(c, ST_KE_Z);
  ke_z_kernel<<<dim3(N, howmany), 256, smem, c.stream>>>(in, out, ka);
  SG_LAUNCHED();
  return SINCGPU_OK;
}

}  // namespace sincgpu
