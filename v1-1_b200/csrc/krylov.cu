// Krylov exponential propagator of the A-vector on the device.
//
// Restates Sidje's Expokit DGEXPV as the reference's variant DGEXPVxxx20
// (MCTDH.SRC/expokit.f90:2222-2660) that expoavecprop calls
// (MCTDH.SRC/expo_driver.f90:827-1055): w = exp(t A) v for the real-ified
// A-vector (complex nc-vector viewed as 2*nc reals), A = timefac * H with H the
// CI sigma operator (sparsesparsemult_byproc, ci.cu).  Full (modified
// Gram-Schmidt) Arnoldi, happy-breakdown test, (6,6) Pade with scaling and
// squaring of the small Hessenberg (DGPADM, expokit.f90:526-713), local error
// estimate and step-size control with the reference's modification that the next
// step is never shorter than the accepted one, and the returned step guess.
// All vector and matrix arithmetic runs on the GPU in FP64; the host only reads
// the few scalars that decide step acceptance.
#include <algorithm>
#include <cmath>
#include <vector>
#include <cooperative_groups.h>
#include "context.hpp"

namespace sincgpu {

constexpr int kKryThreads = 1024;
constexpr int kMaxKry = 124;  // Krylov dimension limit (Pade order m + 2 <= 126)

// block reduction (fixed shape -> deterministic)
__device__ double block_sum(double v, double* red) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  __syncthreads();
  if (l == 0) red[w] = v;
  __syncthreads();
  double s = 0.0;
  if (threadIdx.x < 32) {
    s = threadIdx.x < (blockDim.x >> 5) ? red[threadIdx.x] : 0.0;
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
    if (threadIdx.x == 0) red[32] = s;
  }
  __syncthreads();
  return red[32];
}

struct KryState {  // device scalars
  double beta;     // |w|
  double avnorm;   // |A v_{m+1}|
  int mbrk;        // 0 = no breakdown, else breakdown dimension
};

// V[0] = w / beta (beta computed here and stored)
__global__ void __launch_bounds__(kKryThreads) kry_start_kernel(const double* __restrict__ w, long long n,
                                                                double* __restrict__ V, KryState* st,
                                                                int compute_beta) {
  __shared__ double red[33];
  double s = 0.0;
  if (compute_beta) {
    for (long long i = threadIdx.x; i < n; i += blockDim.x) s += w[i] * w[i];
    s = block_sum(s, red);
    if (threadIdx.x == 0) st->beta = sqrt(s);
  }
  __syncthreads();
  const double b = compute_beta ? sqrt(s) : st->beta;
  const double inv = 1.0 / b;
  for (long long i = threadIdx.x; i < n; i += blockDim.x) V[i] = inv * w[i];
  if (threadIdx.x == 0) st->mbrk = 0;
}

// modified Gram-Schmidt of p = V[j+1] (the matvec of V[j]) against V[0..j],
// Hessenberg column j, breakdown test, normalisation (expokit.f90:2327-2346).
__global__ void __launch_bounds__(kKryThreads) kry_mgs_kernel(double* __restrict__ V, long long n, int j,
                                                              double* __restrict__ Hm, int mh,
                                                              double break_tol, KryState* st) {
  __shared__ double red[33];
  if (st->mbrk) return;
  double* p = V + (long long)(j + 1) * n;
  for (int i = 0; i <= j; ++i) {
    const double* vi = V + (long long)i * n;
    double s = 0.0;
    for (long long k = threadIdx.x; k < n; k += blockDim.x) s += vi[k] * p[k];
    const double hij = block_sum(s, red);
    for (long long k = threadIdx.x; k < n; k += blockDim.x) p[k] -= hij * vi[k];
    if (threadIdx.x == 0) Hm[(long long)j * mh + i] = hij;
    __syncthreads();
  }
  double s = 0.0;
  for (long long k = threadIdx.x; k < n; k += blockDim.x) s += p[k] * p[k];
  const double h = sqrt(block_sum(s, red));
  if (h <= break_tol) {
    if (threadIdx.x == 0) st->mbrk = j + 1;
    return;
  }
  if (threadIdx.x == 0) Hm[(long long)j * mh + j + 1] = h;
  const double inv = 1.0 / h;
  for (long long k = threadIdx.x; k < n; k += blockDim.x) p[k] *= inv;
}

// kry_mgs_kernel with p held in registers (the same elements per thread,
// k = threadIdx.x + e blockDim.x, and the same sums in the same order: the same
// bits) and v_{i+1} loaded while v_i's projection is being reduced, so that no
// global access sits inside the sequential loop.  n <= E * kKryThreads.
template <int E>
__global__ void __launch_bounds__(kKryThreads) kry_mgs_reg_kernel(double* __restrict__ V, long long n, int j,
                                                                  double* __restrict__ Hm, int mh,
                                                                  double break_tol, KryState* st) {
  __shared__ double red[33];
  if (st->mbrk) return;
  double* p = V + (long long)(j + 1) * n;
  double x[E], a[E], an[E];
#pragma unroll
  for (int e = 0; e < E; ++e) {
    const long long k = threadIdx.x + (long long)e * blockDim.x;
    x[e] = k < n ? p[k] : 0.0;
    a[e] = k < n ? V[k] : 0.0;
    an[e] = 0.0;
  }
  for (int i = 0; i <= j; ++i) {
    if (i < j) {
      const double* vn = V + (long long)(i + 1) * n;
#pragma unroll
      for (int e = 0; e < E; ++e) {
        const long long k = threadIdx.x + (long long)e * blockDim.x;
        an[e] = k < n ? vn[k] : 0.0;
      }
    }
    double s = 0.0;
#pragma unroll
    for (int e = 0; e < E; ++e)
      if (threadIdx.x + (long long)e * blockDim.x < n) s += a[e] * x[e];
    const double hij = block_sum(s, red);
#pragma unroll
    for (int e = 0; e < E; ++e)
      if (threadIdx.x + (long long)e * blockDim.x < n) x[e] -= hij * a[e];
    if (threadIdx.x == 0) Hm[(long long)j * mh + i] = hij;
    __syncthreads();
#pragma unroll
    for (int e = 0; e < E; ++e) a[e] = an[e];
  }
  double s = 0.0;
#pragma unroll
  for (int e = 0; e < E; ++e)
    if (threadIdx.x + (long long)e * blockDim.x < n) s += x[e] * x[e];
  const double h = sqrt(block_sum(s, red));
  const bool brk = h <= break_tol;
  if (threadIdx.x == 0) {
    if (brk) st->mbrk = j + 1;
    else Hm[(long long)j * mh + j + 1] = h;
  }
  const double inv = 1.0 / h;
#pragma unroll
  for (int e = 0; e < E; ++e) {
    const long long k = threadIdx.x + (long long)e * blockDim.x;
    if (k < n) p[k] = brk ? x[e] : x[e] * inv;
  }
}

// kry_mgs_reg_kernel over a thread-block cluster of kMgsCluster CTAs, for vectors
// longer than one CTA holds in registers (n > 4 kKryThreads): CTA r of the cluster
// keeps the slice [r S, r S + S) of p in registers (S = ceil(n / kMgsCluster),
// E elements per thread), each projection's dot is summed per CTA (block_sum) and
// then over the cluster's partials in rank order through distributed shared memory
// (so every CTA gets the same value, and the sums have a fixed shape), one cluster
// barrier per sum (the partials alternate between two slots).  The modified
// Gram-Schmidt order of expokit.f90:2327-2346 is kept; only the shape of each sum
// differs from the single-CTA kernels.  A single CTA took 0.37 ms per call at
// 28800 reals (14400 determinants): its loads of V sat behind one SM's bandwidth.
constexpr int kMgsCluster = 8;

template <int E>
__global__ void __launch_bounds__(kKryThreads) kry_mgs_cluster_kernel(double* __restrict__ V, long long n, int j,
                                                                      double* __restrict__ Hm, int mh,
                                                                      double break_tol, KryState* st) {
  namespace cg = cooperative_groups;
  cg::cluster_group cl = cg::this_cluster();
  __shared__ double red[33];
  __shared__ double cpart[2];
  if (st->mbrk) return;  // the same value in every CTA of the cluster
  const long long S = (n + kMgsCluster - 1) / kMgsCluster;
  const long long lo = (long long)cl.block_rank() * S, hi = min(n, lo + S);
  double* p = V + (long long)(j + 1) * n;
  int nsum = 0;
  // sum over the cluster: this CTA's block sum, then the kMgsCluster partials in rank order
  auto cluster_sum = [&](double v) {
    const double b = block_sum(v, red);
    const int slot = nsum++ & 1;
    if (threadIdx.x == 0) cpart[slot] = b;
    cl.sync();
    double t = 0.0;
#pragma unroll
    for (int q = 0; q < kMgsCluster; ++q) t += *cl.map_shared_rank(&cpart[slot], q);
    return t;
  };
  double x[E], a[E], an[E];
#pragma unroll
  for (int e = 0; e < E; ++e) {
    const long long k = lo + threadIdx.x + (long long)e * blockDim.x;
    x[e] = k < hi ? p[k] : 0.0;
    a[e] = k < hi ? V[k] : 0.0;
    an[e] = 0.0;
  }
  for (int i = 0; i <= j; ++i) {
    if (i < j) {
      const double* vn = V + (long long)(i + 1) * n;
#pragma unroll
      for (int e = 0; e < E; ++e) {
        const long long k = lo + threadIdx.x + (long long)e * blockDim.x;
        an[e] = k < hi ? vn[k] : 0.0;
      }
    }
    double s = 0.0;
#pragma unroll
    for (int e = 0; e < E; ++e) s += a[e] * x[e];  // zero outside the slice
    const double hij = cluster_sum(s);
#pragma unroll
    for (int e = 0; e < E; ++e) x[e] -= hij * a[e];
    if (cl.block_rank() == 0 && threadIdx.x == 0) Hm[(long long)j * mh + i] = hij;
#pragma unroll
    for (int e = 0; e < E; ++e) a[e] = an[e];
  }
  double s = 0.0;
#pragma unroll
  for (int e = 0; e < E; ++e) s += x[e] * x[e];
  const double h = sqrt(cluster_sum(s));
  const bool brk = h <= break_tol;
  if (cl.block_rank() == 0 && threadIdx.x == 0) {
    if (brk) st->mbrk = j + 1;
    else Hm[(long long)j * mh + j + 1] = h;
  }
  const double inv = 1.0 / h;
#pragma unroll
  for (int e = 0; e < E; ++e) {
    const long long k = lo + threadIdx.x + (long long)e * blockDim.x;
    if (k < hi) p[k] = brk ? x[e] : x[e] * inv;
  }
  cl.sync();  // no CTA leaves while another may still read its partials
}

template <int E>
static int launch_mgs_cluster(Ctx& c, double* V, long long n, int j, double* Hm, int mh, double break_tol,
                              KryState* st) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(kMgsCluster, 1, 1);
  cfg.blockDim = dim3(kKryThreads, 1, 1);
  cfg.dynamicSmemBytes = 0;
  cfg.stream = c.stream;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeClusterDimension;
  at[0].val.clusterDim.x = kMgsCluster;
  at[0].val.clusterDim.y = 1;
  at[0].val.clusterDim.z = 1;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  SG_CUDA(cudaLaunchKernelEx(&cfg, kry_mgs_cluster_kernel<E>, V, n, j, Hm, mh, break_tol, st));
  return SINCGPU_OK;
}

__global__ void __launch_bounds__(kKryThreads) kry_avnorm_kernel(const double* __restrict__ p, long long n,
                                                                 KryState* st) {
  __shared__ double red[33];
  if (st->mbrk) return;
  double s = 0.0;
  for (long long k = threadIdx.x; k < n; k += blockDim.x) s += p[k] * p[k];
  s = block_sum(s, red);
  if (threadIdx.x == 0) st->avnorm = sqrt(s);
}

// (6,6) Pade exp(t H) with scaling and squaring (DGPADM), H = Hm[0:mx,0:mx]
// (column-major, leading dimension mh); writes column `col` of exp(t H) to exph
// and, when Efull is given, the whole matrix (column-major, leading dimension mx).
// One CTA; mx <= kMaxPade.  The five mx^2 work matrices live in dynamic shared
// memory, or in `gscratch` (global, 5 mx^2 doubles) when it is given.
constexpr int kMaxPade = 128;
__global__ void __launch_bounds__(kKryThreads) kry_padm_kernel(const double* __restrict__ Hm, int mh, int mx,
                                                               double t, double* __restrict__ exph,
                                                               int* __restrict__ ns_out, int col,
                                                               double* __restrict__ Efull,
                                                               double* __restrict__ gscratch) {
  constexpr int ideg = 6;
  extern __shared__ double psm[];  // H, A, B, C, T: 5 mx^2 doubles
  __shared__ double coef[ideg + 1];
  __shared__ double rows[kMaxPade];
  __shared__ int piv_s;
  const int m = mx, mm = m * m, tid = threadIdx.x;
  double* H = gscratch ? gscratch : psm;
  double* A = H + mm;
  double* B = A + mm;
  double* C = B + mm;
  double* T = C + mm;
  for (int i = tid; i < mm; i += blockDim.x) H[i] = Hm[(i / m) * mh + (i % m)];
  __syncthreads();
  // infinity norm: max row sum of |H|
  for (int r = tid; r < m; r += blockDim.x) {
    double s = 0.0;
    for (int j = 0; j < m; ++j) s += fabs(H[r + m * j]);
    rows[r] = s;
  }
  __syncthreads();
  __shared__ double hnorm_s;
  if (tid == 0) {
    double hn = 0.0;
    for (int i = 0; i < m; ++i) hn = fmax(hn, rows[i]);
    hnorm_s = fabs(t * hn);
  }
  __syncthreads();
  const double hnorm = hnorm_s;
  if (hnorm == 0.0) {
    for (int i = tid; i < m; i += blockDim.x) exph[i] = i == col ? 1.0 : 0.0;
    if (Efull)
      for (int e = tid; e < mm; e += blockDim.x) Efull[e] = (e % m) == (e / m) ? 1.0 : 0.0;
    if (tid == 0) *ns_out = 0;
    return;
  }
  const int ns = max(0, (int)(log(hnorm) / log(2.0)) + 2);
  const double scale = t / (double)(1LL << ns);
  const double scale2 = scale * scale;
  if (tid == 0) {
    const int ii = ideg + 1, jj = 2 * ideg + 1;
    coef[0] = 1.0;
    for (int k = 1; k <= ideg; ++k) coef[k] = (coef[k - 1] * (double)(ii - k)) / (double)(k * (jj - k));
  }
  __syncthreads();
  // A = scale2 * H*H  (H2);  B = cp I (p);  C = cq I (q)
  for (int e = tid; e < mm; e += blockDim.x) {
    const int i = e % m, j = e / m;
    double s = 0.0;
    for (int k = 0; k < m; ++k) s += H[i + m * k] * H[k + m * j];
    A[e] = scale2 * s;
    B[e] = i == j ? coef[ideg - 1] : 0.0;
    C[e] = i == j ? coef[ideg] : 0.0;
  }
  __syncthreads();
  double* P = B;
  double* Q = C;
  int iodd = 1;
  for (int k = ideg - 1; k > 0; --k) {
    double* src = iodd ? Q : P;
    for (int e = tid; e < mm; e += blockDim.x) {
      const int i = e % m, j = e / m;
      double s = 0.0;
      for (int kk = 0; kk < m; ++kk) s += src[i + m * kk] * A[kk + m * j];
      T[e] = s + (i == j ? coef[k - 1] : 0.0);
    }
    __syncthreads();
    for (int e = tid; e < mm; e += blockDim.x) src[e] = T[e];
    __syncthreads();
    iodd = 1 - iodd;
  }
  {  // last factor: scale * (q or p) * H
    double* src = iodd ? Q : P;
    for (int e = tid; e < mm; e += blockDim.x) {
      const int i = e % m, j = e / m;
      double s = 0.0;
      for (int kk = 0; kk < m; ++kk) s += src[i + m * kk] * H[kk + m * j];
      T[e] = scale * s;
    }
    __syncthreads();
    for (int e = tid; e < mm; e += blockDim.x) src[e] = T[e];
    __syncthreads();
  }
  // Q = Q - P; solve Q X = P (LU, partial pivoting, first maximum on ties)
  for (int e = tid; e < mm; e += blockDim.x) Q[e] -= P[e];
  __syncthreads();
  for (int k = 0; k < m; ++k) {
    if (tid == 0) {
      int ip = k;
      double best = fabs(Q[k + m * k]);
      for (int i = k + 1; i < m; ++i)
        if (fabs(Q[i + m * k]) > best) {
          best = fabs(Q[i + m * k]);
          ip = i;
        }
      piv_s = ip;
    }
    __syncthreads();
    const int ip = piv_s;
    if (ip != k)
      for (int j = tid; j < 2 * m; j += blockDim.x) {
        double* M = j < m ? Q : P;
        const int jj = j < m ? j : j - m;
        double tmp = M[k + m * jj];
        M[k + m * jj] = M[ip + m * jj];
        M[ip + m * jj] = tmp;
      }
    __syncthreads();
    const double pv = Q[k + m * k];
    // eliminate below the pivot (row operations on Q and P)
    for (int e = tid; e < (m - k - 1) * (m - k - 1 + m); e += blockDim.x) {
      const int w = m - k - 1 + m;
      const int i = k + 1 + e / w, c = e % w;
      const double l = Q[i + m * k] / pv;
      if (c < m - k - 1) {
        const int j = k + 1 + c;
        Q[i + m * j] -= l * Q[k + m * j];
      } else {
        const int j = c - (m - k - 1);
        P[i + m * j] -= l * P[k + m * j];
      }
    }
    __syncthreads();
  }
  // back substitution, one column of P per thread
  for (int j = tid; j < m; j += blockDim.x)
    for (int i = m - 1; i >= 0; --i) {
      double s = P[i + m * j];
      for (int kk = i + 1; kk < m; ++kk) s -= Q[i + m * kk] * P[kk + m * j];
      P[i + m * j] = s / Q[i + m * i];
    }
  __syncthreads();
  for (int e = tid; e < mm; e += blockDim.x) P[e] = 2.0 * P[e] + ((e % m) == (e / m) ? 1.0 : 0.0);
  __syncthreads();
  if (ns == 0 && iodd == 1) {
    for (int i = tid; i < m; i += blockDim.x) exph[i] = -P[i + m * col];
    if (Efull)
      for (int e = tid; e < mm; e += blockDim.x) Efull[e] = -P[e];
    if (tid == 0) *ns_out = ns;
    return;
  }
  for (int s = 0; s < ns; ++s) {  // squaring removes the sign of the iodd==1 case
    for (int e = tid; e < mm; e += blockDim.x) {
      const int i = e % m, j = e / m;
      double acc = 0.0;
      for (int kk = 0; kk < m; ++kk) acc += P[i + m * kk] * P[kk + m * j];
      T[e] = acc;
    }
    __syncthreads();
    for (int e = tid; e < mm; e += blockDim.x) P[e] = T[e];
    __syncthreads();
  }
  for (int i = tid; i < m; i += blockDim.x) exph[i] = P[i + m * col];
  if (Efull)
    for (int e = tid; e < mm; e += blockDim.x) Efull[e] = P[e];
  if (tid == 0) *ns_out = ns;
}

// w = beta * V[0:mx]^T exph[0:mx]; beta <- |w|
__global__ void __launch_bounds__(kKryThreads) kry_update_kernel(const double* __restrict__ V, long long n,
                                                                 int mx, const double* __restrict__ exph,
                                                                 double* __restrict__ w, KryState* st) {
  __shared__ double red[33];
  const double beta = st->beta;
  double s = 0.0;
  for (long long k = threadIdx.x; k < n; k += blockDim.x) {
    double acc = 0.0;
    for (int i = 0; i < mx; ++i) acc += V[(long long)i * n + k] * exph[i];
    const double v = beta * acc;
    w[k] = v;
    s += v * v;
  }
  s = block_sum(s, red);
  if (threadIdx.x == 0) st->beta = sqrt(s);
}

// out = scale * in (complex), used to apply timefac after the sigma product
__global__ void cscale_kernel(const double2* __restrict__ in, double2 s, int nc, double2* __restrict__ out,
                              const KryState* st) {
  if (st && st->mbrk) return;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < nc) out[i] = cmul(s, in[i]);
}

int pade_expm(Ctx& c, const double* Hm, int mh, int mx, double t, int col, double* exph, double* Efull,
              double* gscratch, int* d_ns) {
  SG_CHECK(mx >= 1 && mx <= kMaxPade, SINCGPU_ERANGE, "Pade order %d outside [1,%d]", mx, kMaxPade);
  // process-wide attribute, one fixed value, set once (thread-safe static init)
  static const cudaError_t attr = cudaFuncSetAttribute(
      kry_padm_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)(sizeof(double) * 5 * 64 * 64));
  SG_CUDA(attr);
  const bool smem = mx <= 64;
  SG_CHECK(smem || gscratch, SINCGPU_EINVAL, "Pade order %d needs global scratch", mx);
  const size_t psmem = smem ? sizeof(double) * 5 * (size_t)mx * mx : 0;
  kry_padm_kernel<<<1, kKryThreads, psmem, c.stream>>>(Hm, mh, mx, t, exph, d_ns, col, Efull,
                                                       smem ? nullptr : gscratch);
  SG_LAUNCHED();
  return SINCGPU_OK;
}

static double fortran_nint(double x) { return x >= 0 ? std::floor(x + 0.5) : -std::floor(-x + 0.5); }

int expv_avector(Ctx& c, const double2* v, double2* w, double t, double2 timefac, int m, double tol,
                 double anorm, double* stepguess, int* nstep_out, double ez, double nucdipz, int maxdim_in,
                 int* nmult_out) {
  CIState& s = c.ci;
  SG_CHECK(s.attached && s.assembled, SINCGPU_ESTATE, "sparse CI matrices not assembled");
  const int nc = s.nc;
  const long long n = 2LL * nc;
  // the reference checks m < maxdim (DGEXPVxxx2's maxdim argument; n by default)
  const long long maxdim = maxdim_in > 0 ? maxdim_in : n;
  SG_CHECK(m > 0 && m < maxdim && m <= kMaxKry, SINCGPU_ERANGE, "Krylov dimension %d outside [1,%lld)", m,
           std::min<long long>(maxdim, kMaxKry + 1));
  const int mh = m + 2;
  const size_t need = sizeof(double) * ((size_t)(m + 2) * n + (size_t)mh * mh + 128 + 5 * (size_t)mh * mh) +
                      sizeof(double2) * nc + sizeof(KryState) + 64;
  SG_TRY(c.ws_kry.ensure(need));
  double* V = (double*)c.ws_kry.ptr;
  double* Hm = V + (size_t)(m + 2) * n;
  double* exph = Hm + (size_t)mh * mh;
  double* pscr = exph + 128;
  double2* tmp = (double2*)(pscr + 5 * (size_t)mh * mh);
  KryState* dst = (KryState*)(tmp + nc);
  int* d_ns = (int*)(dst + 1);
  int nmult = 0;
  const double delta = 1.2, gamma = 0.9, break_tol = 1.0e-7;
  double eps = std::fabs((4.0 / 3.0 - 1.0) * 3.0 - 1.0);
  if (tol <= eps) tol = std::sqrt(eps);
  const double rndoff = eps * anorm;
  (void)rndoff;
  const double sgn = t >= 0 ? 1.0 : -1.0;
  const double t_out = std::fabs(t);
  const double sqr1 = std::sqrt(0.1);
  double t_now = 0.0, t_step = 0.0, t_last = 0.0, t_new = *stepguess;
  double xm = 1.0 / m;
  int nstep = 0;
  // w = v; beta = |w|
  SG_CUDA(cudaMemcpyAsync(w, v, sizeof(double2) * nc, cudaMemcpyDeviceToDevice, c.stream));
  KryState hst{};
  bool have_beta = false;
  ProfScope ps(c, ST_CI);
  const int cb = ceil_div(nc, 256);
  while (t_now < t_out) {
    ++nstep;
    t_last = t_step;
    t_step = std::min(t_out - t_now, t_new);
    SG_CUDA(cudaMemsetAsync(Hm, 0, sizeof(double) * mh * mh, c.stream));
    kry_start_kernel<<<1, kKryThreads, 0, c.stream>>>((const double*)w, n, V, dst, have_beta ? 0 : 1);
    SG_LAUNCHED();
    for (int j = 0; j < m; ++j) {
      ++nmult;
      SG_TRY(ci_sigma(c, (const double2*)(V + (size_t)j * n), tmp, c.nucrepulsion, ez, nucdipz));
      cscale_kernel<<<cb, 256, 0, c.stream>>>(tmp, timefac, nc, (double2*)(V + (size_t)(j + 1) * n), dst);
      SG_LAUNCHED();
      if (n <= kKryThreads)
        kry_mgs_reg_kernel<1><<<1, kKryThreads, 0, c.stream>>>(V, n, j, Hm, mh, break_tol, dst);
      else if (n <= 2 * kKryThreads)
        kry_mgs_reg_kernel<2><<<1, kKryThreads, 0, c.stream>>>(V, n, j, Hm, mh, break_tol, dst);
      else if (n <= 4 * kKryThreads)
        kry_mgs_reg_kernel<4><<<1, kKryThreads, 0, c.stream>>>(V, n, j, Hm, mh, break_tol, dst);
      else if (!c.kry_cluster)
        kry_mgs_kernel<<<1, kKryThreads, 0, c.stream>>>(V, n, j, Hm, mh, break_tol, dst);
      else if (n <= 1LL * kMgsCluster * kKryThreads)
        SG_TRY(launch_mgs_cluster<1>(c, V, n, j, Hm, mh, break_tol, dst));
      else if (n <= 2LL * kMgsCluster * kKryThreads)
        SG_TRY(launch_mgs_cluster<2>(c, V, n, j, Hm, mh, break_tol, dst));
      else if (n <= 4LL * kMgsCluster * kKryThreads)
        SG_TRY(launch_mgs_cluster<4>(c, V, n, j, Hm, mh, break_tol, dst));
      else if (n <= 8LL * kMgsCluster * kKryThreads)
        SG_TRY(launch_mgs_cluster<8>(c, V, n, j, Hm, mh, break_tol, dst));
      else
        kry_mgs_kernel<<<1, kKryThreads, 0, c.stream>>>(V, n, j, Hm, mh, break_tol, dst);
      SG_LAUNCHED();
    }
    ++nmult;
    SG_TRY(ci_sigma(c, (const double2*)(V + (size_t)m * n), tmp, c.nucrepulsion, ez, nucdipz));
    cscale_kernel<<<cb, 256, 0, c.stream>>>(tmp, timefac, nc, (double2*)(V + (size_t)(m + 1) * n), dst);
    SG_LAUNCHED();
    kry_avnorm_kernel<<<1, kKryThreads, 0, c.stream>>>(V + (size_t)(m + 1) * n, n, dst);
    SG_LAUNCHED();
    SG_CUDA(cudaMemcpyAsync(&hst, dst, sizeof(KryState), cudaMemcpyDeviceToHost, c.stream));
    SG_CUDA(cudaStreamSynchronize(c.stream));
    have_beta = true;
    int k1 = 2, mbrkdwn = m;
    if (hst.mbrk) {
      k1 = 0;
      mbrkdwn = hst.mbrk;
      t_step = t_out - t_now;
    }
    {  // Hm(m+2, m+1) = 1  (expokit.f90:2356)
      const double one = 1.0;
      SG_CUDA(cudaMemcpyAsync(Hm + (size_t)m * mh + m + 1, &one, sizeof(double), cudaMemcpyHostToDevice, c.stream));
    }
    double err_loc = tol;
    double ex[2] = {0.0, 0.0};
    while (true) {
      const int mx = mbrkdwn + k1;
      SG_TRY(pade_expm(c, Hm, mh, mx, sgn * t_step, 0, exph, nullptr, pscr, d_ns));
      if (k1 == 0) {
        err_loc = tol;
        break;
      }
      SG_CUDA(cudaMemcpyAsync(ex, exph + m, sizeof(double) * 2, cudaMemcpyDeviceToHost, c.stream));
      SG_CUDA(cudaStreamSynchronize(c.stream));
      const double p1 = std::fabs(ex[0]) * hst.beta;
      const double p2 = std::fabs(ex[1]) * hst.beta * hst.avnorm;
      if (p1 > 10.0 * p2) {
        err_loc = p2;
        xm = 1.0 / m;
      } else {
        err_loc = p1;
        xm = 1.0 / (m - 1);
      }
      if (err_loc > delta * t_step * tol) {  // reject, step down (mxreject = 0)
        t_step = gamma * t_step * std::pow(t_step * tol / err_loc, xm);
        const double q = std::pow(10.0, fortran_nint(std::log10(t_step) - sqr1) - 1);
        t_step = std::trunc(t_step / q + 0.55) * q;
        continue;
      }
      break;
    }
    const int mxu = mbrkdwn + std::max(0, k1 - 1);
    kry_update_kernel<<<1, kKryThreads, 0, c.stream>>>(V, n, mxu, exph, (double*)w, dst);
    SG_LAUNCHED();
    SG_CUDA(cudaMemcpyAsync(&hst, dst, sizeof(KryState), cudaMemcpyDeviceToHost, c.stream));
    SG_CUDA(cudaStreamSynchronize(c.stream));
    t_new = gamma * t_step * std::pow(t_step * tol / err_loc, xm);
    const double q = std::pow(10.0, fortran_nint(std::log10(t_new) - sqr1) - 1);
    t_new = std::trunc(t_new / q + 0.55) * q;
    if (t_new < t_step) t_new = t_step;
    t_now += t_step;
    if (nstep >= 1000) break;
  }
  *stepguess = nstep == 1 ? t_step : t_last;
  if (nstep_out) *nstep_out = nstep;
  if (nmult_out) *nmult_out = nmult;
  return SINCGPU_OK;
}

}  // namespace sincgpu
