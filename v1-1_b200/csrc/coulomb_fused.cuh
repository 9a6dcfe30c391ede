// Three-pass form of the Coulomb convolution: the y, z and inverse-y transforms
// of one (pair, kx) plane run in one kernel with the plane held on chip, so the
// W2 slab of the five-pass form (N P^2 values per pair, written once, read and
// written by the z pass, read once more) never reaches HBM.
//
//   XT : rows of rho -> DFT along x -> W1T[pair][kx][z][y]     (N^2 P values)
//   YZY: per (pair, kx): N rows along y (N nonzero inputs) -> plane[z < N][ky < P]
//        in shared memory; P columns along z: forward, * real kernel spectrum,
//        inverse, z < N back into the plane; N rows inverse along y (y < N kept)
//        -> W1T in place
//   XTI: W1T rows along kx -> inverse DFT -> R (x < N)
//
// The plane (N x P values) is split over a thread-block cluster of CL CTAs when
// it does not fit one CTA: CTA r owns rows [r NR, (r+1) NR) with NR = ceil(N/CL)
// for the two y transforms, and columns [r PC, (r+1) PC) with PC = ceil(P/CL)
// for the z transforms, which read and write the other CTAs' rows through
// distributed shared memory (cluster barriers between the phases).  41^3 grid
// (P = 81) in FP64: one CTA per plane (108 KB, two per SM); 81^3 grid (P = 162):
// clusters of 4 in FP64 (112 KB per CTA), of 2 in FP32.
//
// The transforms are those of the five-pass form (the same register FFTs and
// twiddles, fft_reg.cuh); the kernel spectrum is taken real (the Coulomb kernel
// is real and even, the imaginary part of its DFT is rounding noise), as the
// TMA-staged z pass does, so results agree with the five-pass form to rounding.
#pragma once
#include <cooperative_groups.h>

namespace sincgpu {

// largest N a length-P plan serves (P >= 2N - 1)
__host__ __device__ constexpr int yzy_nmax(int P) { return (P + 1) / 2; }
// threads of the plane kernel for lines of length P1*P2 split over CL CTAs
__host__ __device__ constexpr int yzy_threads(int P1, int P2, int CL) {
  return (P1 > P2 ? P1 : P2) * ((yzy_nmax(P1 * P2) + CL - 1) / CL);
}
__host__ __device__ constexpr int yzy_bound(int P1, int P2, int CL) {
  return yzy_threads(P1, P2, CL) < 1024 ? yzy_threads(P1, P2, CL) : 1024;
}
// dynamic shared memory of one CTA: twiddles, NR plane rows, the z exchange
template <class C>
__host__ __device__ constexpr size_t yzy_smem(int P, int N, int CL) {
  return sizeof(C) * ((size_t)P + 2ull * (size_t)((N + CL - 1) / CL) * P);
}
// registers per thread the plane kernel is planned with: the FP64 transforms of
// lines with more than 12 values per thread need about 170 without spilling
template <class C>
__host__ __device__ constexpr int yzy_regs(int P1, int P2) {
  return (sizeof(C) == 16 && (P1 > 12 || P2 > 12)) ? 168 : 80;
}
// CTAs per SM that T threads of yzy_regs registers allow (1 or 2)
template <class C>
__host__ __device__ constexpr int yzy_min_blocks(int P1, int P2, int T) {
  return 65536 / (((T + 31) / 32 * 32) * yzy_regs<C>(P1, P2)) >= 2 ? 2 : 1;
}

// XT: rows of rho -> DFT along x -> W1T (transposed through shared memory so
// that each kx writes TL consecutive rows)
template <int P1, int P2, bool DENS, class C>
__global__ void __launch_bounds__((P1 > P2 ? P1 : P2) * lines_for(P1 * P2)) coul_fwd_xT_t(
    const double2* __restrict__ phi1, const double2* __restrict__ phi2, CoulArgs<C> ca) {
  constexpr int P = P1 * P2, S = P1 > P2 ? P1 : P2, TL = lines_for(P);
  __shared__ C roots[P];
  __shared__ C ex[(P + 1) * TL];
  load_roots(roots, ca.roots, P);
  const int N = ca.N;
  const long long NN = (long long)N * N;
  const int s = threadIdx.x % S, l = threadIdx.x / S;
  const int p = blockIdx.z;
  const long long f0 = (long long)blockIdx.x * TL, f = f0 + l;  // row f = z*N + y
  const bool row = f < NN;
  const long long off = f * N;
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
  dft_in_to_out<P1, P2, false, C, true, true>(a, b, s, l, TL, ex, roots);
  if (s < P1) {
#pragma unroll
    for (int k2 = 0; k2 < P2; ++k2) ex[(s + P1 * k2) * TL + l] = b[k2];
  }
  __syncthreads();
  C* dst = ca.W1 + (long long)p * P * NN + f0;
  for (int it = threadIdx.x; it < P * TL; it += blockDim.x) {
    const int kx = it / TL, ll = it - kx * TL;
    if (f0 + ll < NN) dst[kx * NN + ll] = ex[it];
  }
}

// YZY: one (pair, kx) plane, or its share of rows and columns in a cluster of CL
template <int P1, int P2, class C, int CL>
__global__ void __launch_bounds__(yzy_bound(P1, P2, CL), yzy_min_blocks<C>(P1, P2, yzy_bound(P1, P2, CL)))
    coul_yzy_t(CoulArgs<C> ca, const typename CplxTraits<C>::Real* __restrict__ khT) {
  using R = typename CplxTraits<C>::Real;
  constexpr int P = P1 * P2, S = P1 > P2 ? P1 : P2;
  extern __shared__ __align__(16) unsigned char yzy_raw[];
  const int N = ca.N;
  const int NR = (N + CL - 1) / CL;  // rows per CTA = lines per round
  C* roots = reinterpret_cast<C*>(yzy_raw);
  C* plane = roots + P;              // NR x P: row z - r NR, column ky
  C* zex = plane + NR * P;           // exchange of the z transforms, element-major (e * NR + line)
  const int tid = threadIdx.x, s = tid % S, l = tid / S;
  int r = 0;
  if constexpr (CL > 1) r = (int)cooperative_groups::this_cluster().block_rank();
  const int kx = blockIdx.x / CL, p = blockIdx.y;
  const long long NN = (long long)N * N;
  C* W = ca.W1 + ((long long)p * P + kx) * NN;  // the plane in HBM: (z, y), y fastest
  const int z = r * NR + l;
  const bool rowok = z < N;
  C* row = plane + l * P;
  load_roots(roots, ca.roots, P);
  const C zero = CplxTraits<C>::make(0.0, 0.0);

  // ---- phase 1: forward DFT along y of the CTA's rows; the row is its own exchange
  C a[P1], b[P2];
#pragma unroll
  for (int n1 = 0; n1 < P1; ++n1) {
    const int y = s + P2 * n1;
    a[n1] = (rowok && s < P2 && y < N) ? W[(long long)z * N + y] : zero;
  }
  __syncthreads();  // twiddles
  if (s < P2) {
    RegFFT<P1, 1, false, C>::run(a, ConstRoots<P, C>{}, P);
#pragma unroll
    for (int k1 = 0; k1 < P1; ++k1) {
      C v = a[k1];
      if (k1 > 0 && s > 0) v = cmul(v, root<false>(roots, s * k1));
      row[k1 * P2 + s] = v;
    }
  }
  __syncthreads();
  if (s < P1) {
#pragma unroll
    for (int n2 = 0; n2 < P2; ++n2) b[n2] = row[s * P2 + n2];
    RegFFT<P2, 1, false, C>::run(b, ConstRoots<P, C>{}, P);
  }
  __syncthreads();
  if (s < P1) {
#pragma unroll
    for (int k2 = 0; k2 < P2; ++k2) row[s + P1 * k2] = b[k2];
  }
  // element (z, ky) of the plane, in the shared memory of the CTA that owns row z
  auto at = [&](int zz, int ky) -> C* {
    if constexpr (CL > 1) {
      const int q = zz / NR;
      return cooperative_groups::this_cluster().map_shared_rank(plane, q) + (zz - q * NR) * P + ky;
    } else {
      return plane + zz * P + ky;
    }
  };
  if constexpr (CL > 1) {
    cooperative_groups::this_cluster().sync();
  } else {
    __syncthreads();
  }

  // ---- phase 2: the CTA's columns along z: forward, * kernel spectrum, inverse
  constexpr int PCmax = (P + CL - 1) / CL;
  const int k0 = r * PCmax, kend = min(P, k0 + PCmax);
  const R* kh = khT + (long long)kx * P * P;  // [kz][ky] at this kx
  for (int kb = k0; kb < kend; kb += NR) {
    const int ky = kb + l;
    const bool colok = ky < kend;
#pragma unroll
    for (int n1 = 0; n1 < P1; ++n1) {
      const int zz = s + P2 * n1;
      a[n1] = (colok && s < P2 && zz < N) ? *at(zz, ky) : zero;
    }
    dft_in_to_out<P1, P2, false, C, false, true>(a, b, s, l, NR, zex, roots);
    if (colok && s < P1) {
#pragma unroll
      for (int k2 = 0; k2 < P2; ++k2) {
        const R w = kh[(long long)(s + P1 * k2) * P + ky];
        b[k2] = CplxTraits<C>::make(b[k2].x * w, b[k2].y * w);
      }
    }
    dft_out_to_in<P1, P2, true, C, false, true>(b, a, s, l, NR, zex, roots);
    if (colok && s < P2) {
#pragma unroll
      for (int m1 = 0; m1 < P1; ++m1) {
        const int zz = s + P2 * m1;
        if (zz < N) *at(zz, ky) = a[m1];
      }
    }
  }
  if constexpr (CL > 1) {
    cooperative_groups::this_cluster().sync();  // no remote access after this point
  } else {
    __syncthreads();
  }

  // ---- phase 3: inverse DFT along y of the CTA's rows (y < N kept) -> W1T
#pragma unroll
  for (int n1 = 0; n1 < P1; ++n1) a[n1] = s < P2 ? row[s + P2 * n1] : zero;
  __syncthreads();  // the row is read before it serves as exchange
  if (s < P2) {
    RegFFT<P1, 1, true, C>::run(a, ConstRoots<P, C>{}, P);
#pragma unroll
    for (int k1 = 0; k1 < P1; ++k1) {
      C v = a[k1];
      if (k1 > 0 && s > 0) v = cmul(v, root<true>(roots, s * k1));
      row[k1 * P2 + s] = v;
    }
  }
  __syncthreads();
  if (s < P1) {
#pragma unroll
    for (int n2 = 0; n2 < P2; ++n2) b[n2] = row[s * P2 + n2];
    RegFFT<P2, 1, true, C>::run(b, ConstRoots<P, C>{}, P);
    if (rowok) {
#pragma unroll
      for (int k2 = 0; k2 < P2; ++k2) {
        const int y = s + P1 * k2;
        if (y < N) W[(long long)z * N + y] = b[k2];
      }
    }
  }
}

// XTI: W1T rows along kx -> inverse DFT -> R (x < N); the tile of TL rows is read
// kx by kx (TL consecutive values each) and transposed through shared memory
template <int P1, int P2, bool DENS, class C>
__global__ void __launch_bounds__((P1 > P2 ? P1 : P2) * lines_for(P1 * P2)) coul_inv_xT_t(
    CoulArgs<C> ca, double* __restrict__ Rpl, double2* __restrict__ full, int herm) {
  constexpr int P = P1 * P2, S = P1 > P2 ? P1 : P2, TL = lines_for(P);
  __shared__ C roots[P];
  __shared__ C ex[(P + 1) * TL];
  load_roots(roots, ca.roots, P);
  const int N = ca.N;
  const long long NN = (long long)N * N;
  const int s = threadIdx.x % S, l = threadIdx.x / S;
  const int p = blockIdx.z;
  const long long f0 = (long long)blockIdx.x * TL, f = f0 + l;  // row f = z*N + y
  const bool row = f < NN;
  const C* src = ca.W1 + (long long)p * P * NN + f0;
  for (int it = threadIdx.x; it < P * TL; it += blockDim.x) {
    const int kx = it / TL, ll = it - kx * TL;
    ex[ll * (P + 1) + kx] = (f0 + ll < NN) ? src[kx * NN + ll] : CplxTraits<C>::make(0.0, 0.0);
  }
  __syncthreads();
  C a[P1], b[P2];
#pragma unroll
  for (int n1 = 0; n1 < P1; ++n1)
    a[n1] = s < P2 ? ex[l * (P + 1) + s + P2 * n1] : CplxTraits<C>::make(0.0, 0.0);
  __syncthreads();
  dft_in_to_out<P1, P2, true, C, true, false>(a, b, s, l, TL, ex, roots);
  if (!(row && s < P1)) return;
  const long long G = ca.G;
  const long long g0 = f * N;
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

// cluster size of the plane kernel for an N^3 grid on a length-P1*P2 plan with
// complex type C: the smallest of 1, 2, 4, 8 whose CTA (S ceil(N/CL) threads of
// yzy_regs registers) fits the register file and whose share of the plane fits
// shared memory at the CTAs per SM the registers allow; 0 when none does
template <class C>
inline int yzy_cluster(int P1, int P2, int N) {
  const int P = P1 * P2, S = P1 > P2 ? P1 : P2;
  if (N > yzy_nmax(P)) return 0;
  for (int cl : {1, 2, 4, 8}) {
    const int T = S * ((N + cl - 1) / cl);
    if (T > yzy_bound(P1, P2, cl) || (size_t)((T + 31) / 32 * 32) * yzy_regs<C>(P1, P2) > 65536) continue;
    const size_t limit = yzy_min_blocks<C>(P1, P2, T) == 2 ? 112 * 1024 : 226 * 1024;
    if (yzy_smem<C>(P, N, cl) <= limit) return cl;
  }
  return 0;
}

template <int P1, int P2, class C, int CL>
int launch_yzy(Ctx& c, const CoulArgs<C>& ca, int np, const typename CplxTraits<C>::Real* khT) {
  constexpr int S = P1 > P2 ? P1 : P2;
  if constexpr (yzy_threads(P1, P2, CL) > 1024) {
    set_error("fused Coulomb plane kernel: no %d-CTA form for length %d", CL, P1 * P2);
    return SINCGPU_ERANGE;
  } else {
    const int NR = (ca.N + CL - 1) / CL;
    const size_t smem = yzy_smem<C>(P1 * P2, ca.N, CL);
    static const cudaError_t attr = cudaFuncSetAttribute(
        coul_yzy_t<P1, P2, C, CL>, cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024);
    SG_CUDA(attr);
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)(P1 * P2 * CL), (unsigned)np, 1);
    cfg.blockDim = dim3((unsigned)(S * NR), 1, 1);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = c.stream;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeClusterDimension;
    at[0].val.clusterDim.x = CL;
    at[0].val.clusterDim.y = 1;
    at[0].val.clusterDim.z = 1;
    cfg.attrs = at;
    cfg.numAttrs = CL > 1 ? 1 : 0;
    SG_CUDA(cudaLaunchKernelEx(&cfg, coul_yzy_t<P1, P2, C, CL>, ca, khT));
    return SINCGPU_OK;
  }
}

}  // namespace sincgpu
