// Orbital right-hand side (MCTDH.SRC/derivs.f90:629-852, actreduced00) for the sinc
// project (numr=1, bondpoints=1, nonuc_checkflag=1, no frozen core):
//   Y      = phi x denmat                                   (lines 674-676)
//   S      = KE(Y) + pot*Y + E_z(t) z*Y                     (lines 712-752)
//   S     += sum_k reducedpot(:,k,i) phi_k                  (line 763, mult_reducedpot)
//   S      = timefac * S x invdenmat        (dentimeflag)   (lines 788-790)
//   out    = S - proj x <proj|S>            (projflag)      (lines 806-807, project00)
// Kernels: mix (pointwise n x n), KE (ke.cu, fused pot/pulse), reducedpot apply +
// invdenmat mix (one pass over reducedpot, the dominant HBM stream), projector
// dots (split-K, deterministic), projector subtraction.
//
// The per-point kernels work on tiles of 32 consecutive grid points (one per
// lane) by all orbitals: each warp handles a subset of output orbitals, reads
// every (orbital, tile) row as one coalesced 512-byte segment, and the small
// per-point vectors (phi, the partial sums) and n x n matrices sit in shared
// memory, so no thread keeps an n-vector in registers.
#include <algorithm>
#include "context.hpp"

namespace sincgpu {

constexpr int TXO = 32;          // grid points per tile (lanes)
constexpr int kMaxOrbRhs = 32;   // largest orbital count of these kernels
constexpr int kRhsSmemMax = 64 * 1024;

// out(x,i) = sum_j in(x,j) mat(j,i)   (column-major n x n complex mat)
__global__ void __launch_bounds__(TXO * kMaxOrbRhs) mix_kernel(const double2* __restrict__ in,
                                                        const double2* __restrict__ mat, int n, long long G,
                                                        double2* __restrict__ out) {
  extern __shared__ double2 rsm[];
  double2* sm = rsm;            // n*n
  double2* tin = rsm + n * n;   // n x TXO
  const int lx = threadIdx.x, ty = threadIdx.y, tid = ty * TXO + lx;
  for (int e = tid; e < n * n; e += TXO * blockDim.y) sm[e] = mat[e];
  const long long x = blockIdx.x * (long long)TXO + lx;
  const bool ok = x < G;
  for (int j = ty; j < n; j += blockDim.y) tin[j * TXO + lx] = ok ? in[(long long)j * G + x] : make_double2(0.0, 0.0);
  __syncthreads();
  if (!ok) return;
  for (int i = ty; i < n; i += blockDim.y) {
    double2 acc = make_double2(0.0, 0.0);
    for (int j = 0; j < n; ++j) cfma(acc, tin[j * TXO + lx], sm[j + n * i]);
    out[(long long)i * G + x] = acc;
  }
}

// s_i = acc(x,i) + sum_k V(x,k,i) phi_k(x) over i in [i0, i0+ni); then, when
// `dentime`, t_i = timefac * sum_j s_j inv(j,i) (all n orbitals present).
__global__ void __launch_bounds__(TXO * kMaxOrbRhs) redpot_kernel(const double2* __restrict__ phi,
                                                           const double2* __restrict__ V,
                                                           const double2* __restrict__ acc_in,
                                                           const double2* __restrict__ inv, double2 timefac,
                                                           int n, int i0, int ni, int dentime, long long G,
                                                           double2* __restrict__ out) {
  extern __shared__ double2 rsm[];
  double2* sinv = rsm;                 // n*n (dentime)
  double2* sph = rsm + n * n;          // n x TXO
  double2* ss = sph + n * TXO;         // n x TXO (dentime)
  const int lx = threadIdx.x, ty = threadIdx.y, tid = ty * TXO + lx;
  if (dentime)
    for (int e = tid; e < n * n; e += TXO * blockDim.y) sinv[e] = inv[e];
  const long long x = blockIdx.x * (long long)TXO + lx;
  const bool ok = x < G;
  for (int k = ty; k < n; k += blockDim.y) sph[k * TXO + lx] = ok ? phi[(long long)k * G + x] : make_double2(0.0, 0.0);
  __syncthreads();
  if (ok) {
    for (int ii = ty; ii < ni; ii += blockDim.y) {
      double2 a = acc_in ? acc_in[(long long)ii * G + x] : make_double2(0.0, 0.0);
      const double2* Vi = V + (long long)n * ii * G + x;  // V(x,k,i): column k + n*ii
#pragma unroll 4
      for (int k = 0; k < n; ++k) cfma(a, Vi[(long long)k * G], sph[k * TXO + lx]);
      if (dentime) ss[ii * TXO + lx] = a;
      else out[(long long)ii * G + x] = a;
    }
    (void)i0;
  }
  if (!dentime) return;
  __syncthreads();
  if (!ok) return;
  for (int i = ty; i < n; i += blockDim.y) {
    double2 a = make_double2(0.0, 0.0);
    for (int j = 0; j < n; ++j) cfma(a, ss[j * TXO + lx], sinv[j + n * i]);
    out[(long long)i * G + x] = cmul(timefac, a);
  }
}

// actreduced blended over two mean-field slots without projection (the orbital
// Jacobian): out = f0 A_0 + f1 A_1 with A_s = timefac ((Y D_s + V_s . x) I_s) and
// Y = KE(x) (+ potential and field), per point in one pass: mix_kernel,
// redpot_kernel (dentime) and axpby_kernel's arithmetic in their order, so the
// same bits as those launches, without the per-slot temporaries.
__global__ void __launch_bounds__(TXO * kMaxOrbRhs) blend2_kernel(
    const double2* __restrict__ xin, const double2* __restrict__ Y, const double2* __restrict__ V0,
    const double2* __restrict__ V1, const double2* __restrict__ D0, const double2* __restrict__ D1,
    const double2* __restrict__ I0, const double2* __restrict__ I1, double2 timefac, double f0, double f1, int n,
    long long G, double2* __restrict__ out) {
  extern __shared__ double2 rsm[];
  double2* sD = rsm;            // [2][n*n]
  double2* sI = sD + 2 * n * n;  // [2][n*n]
  double2* sx = sI + 2 * n * n;  // n x TXO
  double2* sy = sx + n * TXO;    // n x TXO
  double2* ss = sy + n * TXO;    // n x TXO
  const int lx = threadIdx.x, ty = threadIdx.y, tid = ty * TXO + lx;
  for (int e = tid; e < n * n; e += TXO * blockDim.y) {
    sD[e] = D0[e];
    sD[n * n + e] = D1[e];
    sI[e] = I0[e];
    sI[n * n + e] = I1[e];
  }
  const long long x = blockIdx.x * (long long)TXO + lx;
  const bool ok = x < G;
  for (int j = ty; j < n; j += blockDim.y) {
    sx[j * TXO + lx] = ok ? xin[(long long)j * G + x] : make_double2(0.0, 0.0);
    sy[j * TXO + lx] = ok ? Y[(long long)j * G + x] : make_double2(0.0, 0.0);
  }
  const int ii = ty;  // one warp per orbital
  double2 res = make_double2(0.0, 0.0);
  for (int s = 0; s < 2; ++s) {
    __syncthreads();  // tiles loaded (s = 0); the previous slot's ss reads done (s = 1)
    if (ok) {
      const double2* Ds = sD + s * n * n;
      double2 a = make_double2(0.0, 0.0);
      for (int j = 0; j < n; ++j) cfma(a, sy[j * TXO + lx], Ds[j + n * ii]);
      const double2* Vi = (s ? V1 : V0) + (long long)n * ii * G + x;
#pragma unroll 4
      for (int k = 0; k < n; ++k) cfma(a, Vi[(long long)k * G], sx[k * TXO + lx]);
      ss[ii * TXO + lx] = a;
    }
    __syncthreads();
    if (ok) {
      const double2* Is = sI + s * n * n;
      double2 t = make_double2(0.0, 0.0);
      for (int j = 0; j < n; ++j) cfma(t, ss[j * TXO + lx], Is[j + n * ii]);
      t = cmul(timefac, t);
      res = s == 0 ? make_double2(f0 * t.x, f0 * t.y) : make_double2(fma(f1, t.x, 1.0 * res.x), fma(f1, t.y, 1.0 * res.y));
    }
  }
  if (ok) out[(long long)ii * G + x] = res;
}

// M(j,i) = sum_s f_s sum_l D_s(j,l) I_s(l,i): one thread per element (n*n <= 1024)
__global__ void blendq_m_kernel(const double2* __restrict__ D0, const double2* __restrict__ D1,
                                const double2* __restrict__ I0, const double2* __restrict__ I1, double f0, double f1,
                                int n, double2* __restrict__ M) {
  const int e = threadIdx.x;
  if (e >= n * n) return;
  const int j = e % n, i = e / n;
  double2 a0 = make_double2(0.0, 0.0), a1 = make_double2(0.0, 0.0);
  for (int l = 0; l < n; ++l) {
    cfma(a0, D0[j + n * l], I0[l + n * i]);
    cfma(a1, D1[j + n * l], I1[l + n * i]);
  }
  M[e] = make_double2(fma(f1, a1.x, f0 * a0.x), fma(f1, a1.y, f0 * a0.y));
}

// Q(x,k,i) = sum_s sum_j V_s(x,k,j) (f_s I_s(j,i)), reducedpot layout (x fastest,
// then k, then i): per tile of TXO points the rows V_s(., k, j) of one k are staged
// (warp j loads row j of both slots), then warp i forms Q(., k, i)
__global__ void __launch_bounds__(TXO * kMaxOrbRhs) blendq_build_kernel(
    const double2* __restrict__ V0, const double2* __restrict__ V1, const double2* __restrict__ I0,
    const double2* __restrict__ I1, double f0, double f1, int n, long long G, double2* __restrict__ Q) {
  extern __shared__ double2 rsm[];
  double2* sJ = rsm;             // [2][n*n]
  double2* sV = sJ + 2 * n * n;  // [2][n][TXO]
  const int lx = threadIdx.x, ty = threadIdx.y, tid = ty * TXO + lx;
  for (int e = tid; e < n * n; e += TXO * blockDim.y) {
    const double2 a = I0[e], b = I1[e];
    sJ[e] = make_double2(f0 * a.x, f0 * a.y);
    sJ[n * n + e] = make_double2(f1 * b.x, f1 * b.y);
  }
  const long long x = blockIdx.x * (long long)TXO + lx;
  const bool ok = x < G;
  for (int k = 0; k < n; ++k) {
    __syncthreads();  // the previous k's rows are used (and sJ is staged)
    for (int j = ty; j < n; j += blockDim.y) {
      const long long o = (long long)(k + n * j) * G + x;
      sV[j * TXO + lx] = ok ? V0[o] : make_double2(0.0, 0.0);
      sV[(n + j) * TXO + lx] = ok ? V1[o] : make_double2(0.0, 0.0);
    }
    __syncthreads();
    if (ok) {
      for (int i = ty; i < n; i += blockDim.y) {
        double2 a = make_double2(0.0, 0.0);
        for (int j = 0; j < n; ++j) cfma(a, sV[j * TXO + lx], sJ[j + n * i]);
        for (int j = 0; j < n; ++j) cfma(a, sV[(n + j) * TXO + lx], sJ[n * n + j + n * i]);
        Q[(long long)(k + n * i) * G + x] = a;
      }
    }
  }
}

// out(x,i) = timefac (sum_j Y(x,j) M(j,i) + sum_k Q(x,k,i) xin(x,k))
__global__ void __launch_bounds__(TXO * kMaxOrbRhs) blendq_apply_kernel(
    const double2* __restrict__ xin, const double2* __restrict__ Y, const double2* __restrict__ Q,
    const double2* __restrict__ M, double2 timefac, int n, long long G, double2* __restrict__ out) {
  extern __shared__ double2 rsm[];
  double2* sM = rsm;            // n*n
  double2* sx = sM + n * n;     // n x TXO
  double2* sy = sx + n * TXO;   // n x TXO
  const int lx = threadIdx.x, ty = threadIdx.y, tid = ty * TXO + lx;
  for (int e = tid; e < n * n; e += TXO * blockDim.y) sM[e] = M[e];
  const long long x = blockIdx.x * (long long)TXO + lx;
  const bool ok = x < G;
  for (int j = ty; j < n; j += blockDim.y) {
    sx[j * TXO + lx] = ok ? xin[(long long)j * G + x] : make_double2(0.0, 0.0);
    sy[j * TXO + lx] = ok ? Y[(long long)j * G + x] : make_double2(0.0, 0.0);
  }
  __syncthreads();
  if (!ok) return;
  for (int i = ty; i < n; i += blockDim.y) {
    double2 a = make_double2(0.0, 0.0);
    for (int j = 0; j < n; ++j) cfma(a, sy[j * TXO + lx], sM[j + n * i]);
    const double2* Qi = Q + (long long)n * i * G + x;
#pragma unroll 4
    for (int k = 0; k < n; ++k) cfma(a, Qi[(long long)k * G], sx[k * TXO + lx]);
    out[(long long)i * G + x] = cmul(timefac, a);
  }
}

// partial[blk][j + n*i] = sum_{x in blk} conj(P_j(x)) T_i(x); block blk covers
// DCH consecutive points, warp w the rows j = w, w + (warps per block), ...
// BL points per block: 64 (DCH) where the reducedpot GEMM's epilogue forms the same
// partials for its 64-point tiles, 256 for the orbital Jacobian's dots (eight terms
// per lane before the shuffle tree, a quarter of the partials to reduce)
constexpr int DCH = 64;
template <int BL>
__global__ void __launch_bounds__(TXO * kMaxOrbRhs) dots_kernel(const double2* __restrict__ Pm,
                                                         const double2* __restrict__ Tm, int n, long long G,
                                                         double2* __restrict__ partial) {
  extern __shared__ double2 rsm[];
  double2* tt = rsm;  // n x BL
  const int lx = threadIdx.x, ty = threadIdx.y, tid = ty * TXO + lx;
  const long long x0 = blockIdx.x * (long long)BL;
  const int nth = TXO * blockDim.y;
  // staged in batches of 8 elements per thread: the 8 loads are in flight together
  for (int e0 = tid; e0 < n * BL; e0 += 8 * nth) {
    double2 v[8];
#pragma unroll
    for (int r = 0; r < 8; ++r) {
      const int e = e0 + r * nth;
      const int i = e / BL, k = e % BL;
      const long long x = x0 + k;
      v[r] = (e < n * BL && x < G) ? Tm[(long long)i * G + x] : make_double2(0.0, 0.0);
    }
#pragma unroll
    for (int r = 0; r < 8; ++r) {
      const int e = e0 + r * nth;
      if (e < n * BL) tt[e] = v[r];
    }
  }
  __syncthreads();
  const int nn = n * n;
  for (int j = ty; j < n; j += blockDim.y) {
    double2 pv[BL / TXO];
#pragma unroll
    for (int r = 0; r < BL / TXO; ++r) {
      const long long x = x0 + r * TXO + lx;
      pv[r] = x < G ? Pm[(long long)j * G + x] : make_double2(0.0, 0.0);
    }
    for (int i = 0; i < n; ++i) {
      double2 a = make_double2(0.0, 0.0);
#pragma unroll
      for (int r = 0; r < BL / TXO; ++r) {  // conj(p) t
        const double2 p = pv[r], t = tt[i * BL + r * TXO + lx];
        a.x = fma(p.x, t.x, fma(p.y, t.y, a.x));
        a.y = fma(p.x, t.y, fma(-p.y, t.x, a.y));
      }
      for (int o = 16; o > 0; o >>= 1) {
        a.x += __shfl_down_sync(0xffffffffu, a.x, o);
        a.y += __shfl_down_sync(0xffffffffu, a.y, o);
      }
      if (lx == 0) partial[(long long)blockIdx.x * nn + j + n * i] = a;
    }
  }
}

// one CTA per element: strided partial sums then a fixed-shape tree (deterministic)
__global__ void __launch_bounds__(128) dots_reduce_kernel(const double2* __restrict__ partial,
                                                          int nblk, int nn, double2* __restrict__ D) {
  __shared__ double2 red[128];
  const int e = blockIdx.x;
  double2 s = make_double2(0.0, 0.0);
  for (int b = threadIdx.x; b < nblk; b += 128) s = cadd(s, partial[(long long)b * nn + e]);
  red[threadIdx.x] = s;
  __syncthreads();
  for (int w = 64; w > 0; w >>= 1) {
    if (threadIdx.x < w) red[threadIdx.x] = cadd(red[threadIdx.x], red[threadIdx.x + w]);
    __syncthreads();
  }
  if (threadIdx.x == 0) D[e] = red[0];
}

// out(x,i) = T(x,i) - sum_j P_j(x) D(j,i)
__global__ void __launch_bounds__(TXO * kMaxOrbRhs) project_kernel(const double2* __restrict__ Tm,
                                                            const double2* __restrict__ Pm,
                                                            const double2* __restrict__ D, int n, long long G,
                                                            double2* __restrict__ out) {
  extern __shared__ double2 rsm[];
  double2* sd = rsm;            // n*n
  double2* sp = rsm + n * n;    // n x TXO
  const int lx = threadIdx.x, ty = threadIdx.y, tid = ty * TXO + lx;
  for (int e = tid; e < n * n; e += TXO * blockDim.y) sd[e] = D[e];
  const long long x = blockIdx.x * (long long)TXO + lx;
  const bool ok = x < G;
  for (int j = ty; j < n; j += blockDim.y) sp[j * TXO + lx] = ok ? Pm[(long long)j * G + x] : make_double2(0.0, 0.0);
  __syncthreads();
  if (!ok) return;
  for (int i = ty; i < n; i += blockDim.y) {
    double2 a = make_double2(0.0, 0.0);
    for (int j = 0; j < n; ++j) cfma(a, sp[j * TXO + lx], sd[j + n * i]);
    out[(long long)i * G + x] = csub(Tm[(long long)i * G + x], a);
  }
}

// out(x,i) = T(x,i) - sum_j P_j(x) (M1(j,i) + M2(j,i)) - sum_j X_j(x) D2(j,i)
// (the projector and projector-derivative terms of the orbital Jacobian)
__global__ void __launch_bounds__(TXO * kMaxOrbRhs) jac_combine_kernel(const double2* __restrict__ Tm,
                                                                const double2* __restrict__ Pm,
                                                                const double2* __restrict__ M1,
                                                                const double2* __restrict__ M2,
                                                                const double2* __restrict__ Xm,
                                                                const double2* __restrict__ D2, int n,
                                                                long long G, double2* __restrict__ out) {
  extern __shared__ double2 rsm[];
  double2* sm = rsm;               // n*n: M1 + M2
  double2* sd = sm + n * n;        // n*n: D2
  double2* sp = sd + n * n;        // n x TXO
  double2* sx = sp + n * TXO;      // n x TXO
  const int lx = threadIdx.x, ty = threadIdx.y, tid = ty * TXO + lx;
  for (int e = tid; e < n * n; e += TXO * blockDim.y) {
    sm[e] = cadd(M1[e], M2[e]);
    sd[e] = D2[e];
  }
  const long long x = blockIdx.x * (long long)TXO + lx;
  const bool ok = x < G;
  for (int j = ty; j < n; j += blockDim.y) {
    sp[j * TXO + lx] = ok ? Pm[(long long)j * G + x] : make_double2(0.0, 0.0);
    sx[j * TXO + lx] = ok ? Xm[(long long)j * G + x] : make_double2(0.0, 0.0);
  }
  __syncthreads();
  if (!ok) return;
  for (int i = ty; i < n; i += blockDim.y) {
    double2 a = make_double2(0.0, 0.0);
    for (int j = 0; j < n; ++j) {
      cfma(a, sp[j * TXO + lx], sm[j + n * i]);
      cfma(a, sx[j * TXO + lx], sd[j + n * i]);
    }
    out[(long long)i * G + x] = csub(Tm[(long long)i * G + x], a);
  }
}

// acc = a * acc + b * in  (or acc = b * in when `first`)
__global__ void axpby_kernel(double2* __restrict__ acc, const double2* __restrict__ in, double a, double b,
                             long long len, int first) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < len;
       i += (long long)gridDim.x * blockDim.x) {
    const double2 v = in[i];
    if (first) {
      acc[i] = make_double2(b * v.x, b * v.y);
    } else {
      const double2 w = acc[i];
      acc[i] = make_double2(fma(b, v.x, a * w.x), fma(b, v.y, a * w.y));
    }
  }
}

namespace {

// the kernels' shared-memory limit: one fixed value (race-free across threads)
int rhs_attrs() {
  static const cudaError_t attr = [] {
    for (const void* k : {(const void*)mix_kernel, (const void*)redpot_kernel, (const void*)dots_kernel<DCH>,
                          (const void*)dots_kernel<4 * DCH>,
                          (const void*)project_kernel, (const void*)jac_combine_kernel,
                          (const void*)blend2_kernel, (const void*)blendq_build_kernel,
                          (const void*)blendq_apply_kernel}) {
      const cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, kRhsSmemMax);
      if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
  }();
  SG_CUDA(attr);
  return SINCGPU_OK;
}

// one warp per orbital (n <= 32): every warp of a block has the same share of
// the per-orbital loops
dim3 tile_for(int n) { return dim3(TXO, (unsigned)std::max(1, std::min(n, kMaxOrbRhs))); }

size_t smem_mix(int n) { return sizeof(double2) * ((size_t)n * n + (size_t)n * TXO); }
size_t smem_redpot(int n) { return sizeof(double2) * ((size_t)n * n + 2 * (size_t)n * TXO); }
size_t smem_dots(int n, int bl = DCH) { return sizeof(double2) * (size_t)n * bl; }
size_t smem_jac(int n) { return sizeof(double2) * (2 * (size_t)n * n + 2 * (size_t)n * TXO); }

int launch_dots(Ctx& c, const double2* P, const double2* T, double2* D, double2* part, bool wide = false) {
  const int n = c.nspf;
  wide = wide && smem_dots(n, 4 * DCH) <= (size_t)kRhsSmemMax;
  const int nb = ceil_div(c.G, wide ? 4 * DCH : DCH);
  if (wide)
    dots_kernel<4 * DCH><<<nb, tile_for(n), smem_dots(n, 4 * DCH), c.stream>>>(P, T, n, c.G, part);
  else
    dots_kernel<DCH><<<nb, tile_for(n), smem_dots(n), c.stream>>>(P, T, n, c.G, part);
  SG_LAUNCHED();
  dots_reduce_kernel<<<n * n, 128, 0, c.stream>>>(part, nb, n * n, D);
  SG_LAUNCHED();
  return SINCGPU_OK;
}

}  // namespace

int orbital_dots_scratch(const Ctx& c) { return ceil_div(c.G, DCH); }

int orbital_dots(Ctx& c, const double2* P, const double2* T, double2* D, double2* part) {
  SG_CHECK(c.nspf <= kMaxOrbRhs, SINCGPU_ERANGE, "at most %d orbitals", kMaxOrbRhs);
  SG_TRY(rhs_attrs());
  return launch_dots(c, P, T, D, part, true);
}

int orbital_mix(Ctx& c, const double2* in, const double2* mat, double2* out) {
  const int n = c.nspf;
  SG_CHECK(n <= kMaxOrbRhs, SINCGPU_ERANGE, "at most %d orbitals", kMaxOrbRhs);
  SG_TRY(rhs_attrs());
  mix_kernel<<<ceil_div(c.G, TXO), tile_for(n), smem_mix(n), c.stream>>>(in, mat, n, c.G, out);
  SG_LAUNCHED();
  return SINCGPU_OK;
}

int jac_combine(Ctx& c, const double2* T, const double2* P, const double2* M1, const double2* M2,
                const double2* X, const double2* D2, double2* out) {
  const int n = c.nspf;
  SG_CHECK(n <= kMaxOrbRhs, SINCGPU_ERANGE, "at most %d orbitals", kMaxOrbRhs);
  SG_TRY(rhs_attrs());
  jac_combine_kernel<<<ceil_div(c.G, TXO), tile_for(n), smem_jac(n), c.stream>>>(T, P, M1, M2, X, D2, n, c.G, out);
  SG_LAUNCHED();
  return SINCGPU_OK;
}

int axpby(Ctx& c, double2* acc, const double2* in, double a, double b, long long len, bool first) {
  axpby_kernel<<<std::min<long long>(ceil_div(len, 256), 148 * 8), 256, 0, c.stream>>>(acc, in, a, b, len,
                                                                                        first ? 1 : 0);
  SG_LAUNCHED();
  return SINCGPU_OK;
}

int mult_reducedpot_range(Ctx& c, const double2* phi, const double2* redpot, int i0, int ni,
                          double2* out) {
  const int n = c.nspf;
  SG_CHECK(n <= kMaxOrbRhs, SINCGPU_ERANGE, "at most %d orbitals", kMaxOrbRhs);
  SG_TRY(rhs_attrs());
  ProfScope ps(c, ST_RHS_REDPOT);
  redpot_kernel<<<ceil_div(c.G, TXO), tile_for(n), smem_redpot(n), c.stream>>>(
      phi, redpot, nullptr, nullptr, make_double2(1, 0), n, i0, ni, 0, c.G, out);
  SG_LAUNCHED();
  return SINCGPU_OK;
}

int mult_reducedpot(Ctx& c, const double2* phi, const double2* redpot, double2* out) {
  return mult_reducedpot_range(c, phi, redpot, 0, c.nspf, out);
}

namespace {
// actreduced temporaries in ws_rhs: Y = phi denmat, S = KE(Y), T, split-K partials, D
struct RhsTemps {
  double2 *Y, *S, *T, *part, *D;
};
int rhs_temps(Ctx& c, RhsTemps& t) {
  const int n = c.nspf;
  SG_CHECK(n <= kMaxOrbRhs, SINCGPU_ERANGE, "at most %d orbitals", kMaxOrbRhs);
  SG_TRY(rhs_attrs());
  const long long G = c.G;
  const int nb = ceil_div(G, DCH);
  const size_t need = sizeof(double2) * (3 * (size_t)n * G + (size_t)nb * n * n + (size_t)n * n);
  SG_TRY(c.ws_rhs.ensure(need));
  t.Y = (double2*)c.ws_rhs.ptr;
  t.S = t.Y + (size_t)n * G;
  t.T = t.S + (size_t)n * G;
  t.part = t.T + (size_t)n * G;
  t.D = t.part + (size_t)nb * n * n;
  return SINCGPU_OK;
}
}  // namespace

int actreduced(Ctx& c, const double2* phi, const double2* proj, const double2* denmat,
               const double2* invdenmat, const double2* redpot, double2 timefac, int dentimeflag,
               int projflag, double zfield, double2* out) {
  SG_TRY(actreduced_pre(c, phi, denmat, zfield));
  return actreduced_post(c, phi, proj, invdenmat, redpot, timefac, dentimeflag, projflag, out);
}

int actreduced_pre(Ctx& c, const double2* phi, const double2* denmat, double zfield) {
  RhsTemps t;
  SG_TRY(rhs_temps(c, t));
  const int n = c.nspf;
  {
    ProfScope ps(c, ST_RHS_MIX);
    mix_kernel<<<ceil_div(c.G, TXO), tile_for(n), smem_mix(n), c.stream>>>(phi, denmat, n, c.G, t.Y);
    SG_LAUNCHED();
  }
  return mult_ke(c, t.Y, t.S, n, true, zfield);
}

int actreduced_ke(Ctx& c, const double2* phi, double zfield) {
  RhsTemps t;
  SG_TRY(rhs_temps(c, t));
  return mult_ke(c, phi, t.Y, c.nspf, true, zfield);
}

int actreduced_mix_ke(Ctx& c, const double2* denmat) {
  RhsTemps t;
  SG_TRY(rhs_temps(c, t));
  const int n = c.nspf;
  ProfScope ps(c, ST_RHS_MIX);
  mix_kernel<<<ceil_div(c.G, TXO), tile_for(n), smem_mix(n), c.stream>>>(t.Y, denmat, n, c.G, t.S);
  SG_LAUNCHED();
  return SINCGPU_OK;
}

bool actreduced_blend2_fits(int n) {
  return n <= kMaxOrbRhs && sizeof(double2) * (4 * (size_t)n * n + 3 * (size_t)n * TXO) <= (size_t)kRhsSmemMax;
}

int actreduced_blend2(Ctx& c, const double2* x, const double2* const* denmat, const double2* const* invdenmat,
                      const double2* const* redpot, const double* facs, double2 timefac, double zfield,
                      double2* out) {
  RhsTemps t;
  SG_TRY(rhs_temps(c, t));
  const int n = c.nspf;
  SG_TRY(mult_ke(c, x, t.Y, n, true, zfield));
  ProfScope ps(c, ST_RHS_REDPOT);
  const size_t sm = sizeof(double2) * (4 * (size_t)n * n + 3 * (size_t)n * TXO);
  blend2_kernel<<<ceil_div(c.G, TXO), tile_for(n), sm, c.stream>>>(x, t.Y, redpot[0], redpot[1], denmat[0],
                                                                    denmat[1], invdenmat[0], invdenmat[1], timefac,
                                                                    facs[0], facs[1], n, c.G, out);
  SG_LAUNCHED();
  return SINCGPU_OK;
}

size_t smem_bq_build(int n) { return sizeof(double2) * (2 * (size_t)n * n + 2 * (size_t)n * TXO); }
size_t smem_bq_apply(int n) { return sizeof(double2) * ((size_t)n * n + 2 * (size_t)n * TXO); }

bool actreduced_blendq_fits(int n) {
  return n <= kMaxOrbRhs && smem_bq_build(n) <= (size_t)kRhsSmemMax && smem_bq_apply(n) <= (size_t)kRhsSmemMax;
}

int blendq_prepare(Ctx& c, const double2* const* denmat, const double2* const* invdenmat,
                   const double2* const* redpot, const double* facs) {
  const int n = c.nspf;
  SG_CHECK(actreduced_blendq_fits(n), SINCGPU_ERANGE, "blended reduced potential: at most %d orbitals", kMaxOrbRhs);
  SG_TRY(rhs_attrs());
  const size_t nq = (size_t)c.G * n * n;
  SG_TRY(c.ws_bq.ensure(sizeof(double2) * (nq + (size_t)n * n)));
  double2* Q = (double2*)c.ws_bq.ptr;
  ProfScope ps(c, ST_RHS_REDPOT);
  blendq_m_kernel<<<1, 1024, 0, c.stream>>>(denmat[0], denmat[1], invdenmat[0], invdenmat[1], facs[0], facs[1], n,
                                            Q + nq);
  SG_LAUNCHED();
  blendq_build_kernel<<<ceil_div(c.G, TXO), tile_for(n), smem_bq_build(n), c.stream>>>(
      redpot[0], redpot[1], invdenmat[0], invdenmat[1], facs[0], facs[1], n, c.G, Q);
  SG_LAUNCHED();
  return SINCGPU_OK;
}

int actreduced_blendq(Ctx& c, const double2* x, double2 timefac, double zfield, double2* out) {
  RhsTemps t;
  SG_TRY(rhs_temps(c, t));
  const int n = c.nspf;
  const double2* Q = (const double2*)c.ws_bq.ptr;
  SG_CHECK(Q, SINCGPU_ESTATE, "blended reduced potential not prepared");
  SG_TRY(mult_ke(c, x, t.Y, n, true, zfield));
  ProfScope ps(c, ST_RHS_REDPOT);
  blendq_apply_kernel<<<ceil_div(c.G, TXO), tile_for(n), smem_bq_apply(n), c.stream>>>(
      x, t.Y, Q, Q + (size_t)c.G * n * n, timefac, n, c.G, out);
  SG_LAUNCHED();
  return SINCGPU_OK;
}

int actreduced_temps(Ctx& c, double2** S, double2** T, double2** part) {
  RhsTemps t;
  SG_TRY(rhs_temps(c, t));
  *S = t.S;
  *T = t.T;
  if (part) *part = t.part;
  return SINCGPU_OK;
}

int actreduced_post(Ctx& c, const double2* phi, const double2* proj, const double2* invdenmat,
                    const double2* redpot, double2 timefac, int dentimeflag, int projflag, double2* out,
                    bool t_ready, bool dots_ready) {
  RhsTemps t;
  SG_TRY(rhs_temps(c, t));
  const int n = c.nspf;
  const long long G = c.G;
  const int bt = ceil_div(G, TXO);
  double2 *S = t.S, *T = t.T, *part = t.part, *D = t.D;
  double2* dst = projflag == 1 ? T : out;
  if (!t_ready) {
    ProfScope ps(c, ST_RHS_REDPOT);
    redpot_kernel<<<bt, tile_for(n), smem_redpot(n), c.stream>>>(phi, redpot, S, invdenmat, timefac, n, 0, n,
                                                           dentimeflag ? 1 : 0, G, dst);
    SG_LAUNCHED();
  }
  if (projflag == 1) {
    ProfScope ps(c, ST_RHS_PROJ);
    if (dots_ready) {
      dots_reduce_kernel<<<n * n, 128, 0, c.stream>>>(part, ceil_div(G, DCH), n * n, D);
      SG_LAUNCHED();
    } else {
      // above 10 orbitals no GEMM epilogue forms 64-point partials, so the dots
      // take 256-point blocks (a quarter of the partials; 81^3, 16 orbitals: the
      // 64-point form took 0.27 ms)
      SG_TRY(launch_dots(c, proj, T, D, part, n > 10));
    }
    project_kernel<<<bt, tile_for(n), smem_mix(n), c.stream>>>(T, proj, D, n, G, out);
    SG_LAUNCHED();
  }
  return SINCGPU_OK;
}

}  // namespace sincgpu
