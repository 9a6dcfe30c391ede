// Pair densities -> Toeplitz/FFT Coulomb solve -> reduced two-electron potentials.
//
// Reference: call_twoe_matel00 (SINCDVR/coreproject.f90:945-1194) builds
// rho_ab = phi1_a * conj(phi2_b) (line 1063), op_tinv (lines 366-537) embeds it at
// octant (1,1,1) of a (2N)^3 grid, circ3d_sub (SINCDVR/toeplitz_subs.f90:561-589)
// convolves it circularly with threed_two and octant (2,2,2) is returned.  That is
// exactly the linear convolution R(x) = sum_y T(x-y) rho(y) for x,y in [0,N)^3.
//
// Here the same convolution runs on a padded P^3 grid (P >= 2N-1, 7-smooth) with
// the kernel spectrum precomputed once, as five global passes:
//   CX : rho rows -> DFT along x          (N^2 rows, N nonzero inputs each)
//   CY : DFT along y                      (N*P columns, N nonzero inputs each)
//   CZ : DFT along z, * khat, inverse DFT (P^2 columns, only z<N kept)
//   CYI: inverse DFT along y              (N*P columns, only y<N kept)
//   CXI: inverse DFT along x              (N^2 rows, only x<N kept) -> R
// Pruned inputs/outputs never touch memory.  Pairs are processed in chunks
// sized so that the intermediate W1 (N*N*P) and W2 (N*P*P) stay L2 resident.
#include <algorithm>
#include <vector>
#include "context.hpp"

namespace sincgpu {

constexpr int kRowTile = 8;  // rows per CTA in the x passes
constexpr int kThreads = 128;

struct CoulArgs {
  int N, P, tx, nspf;
  long long G;
  FftPlan plan;
  const double2* roots;
  const double2* khat;
  double2* W1;  // [pair][z][y][kx]   y < N
  double2* W2;  // [pair][z][ky][kx]  z < N
  const int* pa;
  const int* pb;
  int pair0;        // index of the chunk's first pair in the full list
  int npair_total;  // planar output: Re at pair p, Im at npair_total + p
};

__device__ __forceinline__ void load_roots(double2* roots, const double2* g, int P) {
  for (int i = threadIdx.x; i < P; i += blockDim.x) roots[i] = g[i];
}

// CX.  DENS: the densities are given (op_tinv entry); else rho = phi1_a conj(phi2_b).
template <bool DENS>
__global__ void __launch_bounds__(kThreads) coul_fwd_x(const double2* __restrict__ phi1,
                                                       const double2* __restrict__ phi2,
                                                       CoulArgs ca) {
  extern __shared__ double2 sm[];
  const int N = ca.N, P = ca.P;
  double2* roots = sm;
  double2* A = sm + P;
  double2* B = A + kRowTile * P;
  load_roots(roots, ca.roots, P);
  const int p = blockIdx.z, z = blockIdx.y, y0 = blockIdx.x * kRowTile;
  const int nrow = min(kRowTile, N - y0);
  const long long plane = (long long)z * N * N;
  const double2* s1;
  const double2* s2 = nullptr;
  if (DENS) {
    s1 = phi1 + (long long)(ca.pair0 + p) * ca.G + plane;
  } else {
    s1 = phi1 + (long long)ca.pa[p] * ca.G + plane;
    s2 = phi2 + (long long)ca.pb[p] * ca.G + plane;
  }
  for (int i = threadIdx.x; i < kRowTile * P; i += blockDim.x) {
    int r = i / P, x = i - r * P;
    double2 v = make_double2(0.0, 0.0);
    if (r < nrow && x < N) {
      long long o = (long long)(y0 + r) * N + x;
      v = DENS ? s1[o] : cmulc(s1[o], s2[o]);
    }
    A[i] = v;
  }
  __syncthreads();
  double2* res = fft_lines<false>(A, B, kRowTile, P, 1, ca.plan, roots, false);
  double2* dst = ca.W1 + (((long long)p * N + z) * N + y0) * P;
  for (int i = threadIdx.x; i < nrow * P; i += blockDim.x) dst[i] = res[i];
}

// CY: W1[p][z][y<N][kx] -> W2[p][z][ky][kx]
__global__ void __launch_bounds__(kThreads) coul_fwd_y(CoulArgs ca) {
  extern __shared__ double2 sm[];
  const int N = ca.N, P = ca.P, tx = ca.tx;
  double2* roots = sm;
  double2* A = sm + P;
  double2* B = A + P * tx;
  load_roots(roots, ca.roots, P);
  const int p = blockIdx.z, z = blockIdx.y, x0 = blockIdx.x * tx;
  const double2* src = ca.W1 + ((long long)p * N + z) * N * P;
  for (int i = threadIdx.x; i < P * tx; i += blockDim.x) {
    int j = i / tx, l = i - j * tx, kx = x0 + l;
    A[i] = (j < N && kx < P) ? src[(long long)j * P + kx] : make_double2(0.0, 0.0);
  }
  __syncthreads();
  double2* res = fft_lines<false>(A, B, tx, 1, tx, ca.plan, roots, true);
  double2* dst = ca.W2 + ((long long)p * N + z) * P * P;
  for (int i = threadIdx.x; i < P * tx; i += blockDim.x) {
    int j = i / tx, l = i - j * tx, kx = x0 + l;
    if (kx < P) dst[(long long)j * P + kx] = res[i];
  }
}

// CZ: along z: forward, * khat, inverse; in place on W2 (z < N kept)
__global__ void __launch_bounds__(kThreads) coul_z(CoulArgs ca) {
  extern __shared__ double2 sm[];
  const int N = ca.N, P = ca.P, tx = ca.tx;
  double2* roots = sm;
  double2* A = sm + P;
  double2* B = A + P * tx;
  load_roots(roots, ca.roots, P);
  const int p = blockIdx.z, ky = blockIdx.y, x0 = blockIdx.x * tx;
  double2* col = ca.W2 + (long long)p * N * P * P + (long long)ky * P;
  const long long zs = (long long)P * P;
  for (int i = threadIdx.x; i < P * tx; i += blockDim.x) {
    int j = i / tx, l = i - j * tx, kx = x0 + l;
    A[i] = (j < N && kx < P) ? col[j * zs + kx] : make_double2(0.0, 0.0);
  }
  __syncthreads();
  double2* res = fft_lines<false>(A, B, tx, 1, tx, ca.plan, roots, true);
  double2* other = (res == A) ? B : A;
  const double2* kh = ca.khat + (long long)ky * P;
  for (int i = threadIdx.x; i < P * tx; i += blockDim.x) {
    int j = i / tx, l = i - j * tx, kx = x0 + l;
    if (kx < P) res[i] = cmul(res[i], kh[j * zs + kx]);
  }
  __syncthreads();
  double2* out = fft_lines<true>(res, other, tx, 1, tx, ca.plan, roots, true);
  for (int i = threadIdx.x; i < N * tx; i += blockDim.x) {
    int j = i / tx, l = i - j * tx, kx = x0 + l;
    if (kx < P) col[j * zs + kx] = out[i];
  }
}

// CYI: W2[p][z][ky][kx] -> inverse along y -> W1[p][z][y<N][kx]
__global__ void __launch_bounds__(kThreads) coul_inv_y(CoulArgs ca) {
  extern __shared__ double2 sm[];
  const int N = ca.N, P = ca.P, tx = ca.tx;
  double2* roots = sm;
  double2* A = sm + P;
  double2* B = A + P * tx;
  load_roots(roots, ca.roots, P);
  const int p = blockIdx.z, z = blockIdx.y, x0 = blockIdx.x * tx;
  const double2* src = ca.W2 + ((long long)p * N + z) * P * P;
  for (int i = threadIdx.x; i < P * tx; i += blockDim.x) {
    int j = i / tx, l = i - j * tx, kx = x0 + l;
    A[i] = kx < P ? src[(long long)j * P + kx] : make_double2(0.0, 0.0);
  }
  __syncthreads();
  double2* res = fft_lines<true>(A, B, tx, 1, tx, ca.plan, roots, true);
  double2* dst = ca.W1 + ((long long)p * N + z) * N * P;
  for (int i = threadIdx.x; i < N * tx; i += blockDim.x) {
    int j = i / tx, l = i - j * tx, kx = x0 + l;
    if (kx < P) dst[(long long)j * P + kx] = res[i];
  }
}

// CXI: inverse along x, keep x < N, write R.
//   Rpl (optional): planar Re/Im rows of the pair list
//   full (optional): twoereduced(x,a,b) interleaved; herm adds (b,a) = conj.
//   DENS: full[g + G*(pair0+p)] (op_tinv layout).
template <bool DENS>
__global__ void __launch_bounds__(kThreads) coul_inv_x(CoulArgs ca, double* __restrict__ Rpl,
                                                       double2* __restrict__ full, int herm) {
  extern __shared__ double2 sm[];
  const int N = ca.N, P = ca.P;
  double2* roots = sm;
  double2* A = sm + P;
  double2* B = A + kRowTile * P;
  load_roots(roots, ca.roots, P);
  const int p = blockIdx.z, z = blockIdx.y, y0 = blockIdx.x * kRowTile;
  const int nrow = min(kRowTile, N - y0);
  const double2* src = ca.W1 + (((long long)p * N + z) * N + y0) * P;
  for (int i = threadIdx.x; i < kRowTile * P; i += blockDim.x) {
    int r = i / P;
    A[i] = r < nrow ? src[i] : make_double2(0.0, 0.0);
  }
  __syncthreads();
  double2* res = fft_lines<true>(A, B, kRowTile, P, 1, ca.plan, roots, false);
  const long long G = ca.G;
  const long long gbase = (long long)z * N * N + (long long)y0 * N;
  const int gp = ca.pair0 + p;
  long long off_ab = 0, off_ba = 0;
  bool mirror = false;
  if (!DENS) {
    const int a = ca.pa[p], b = ca.pb[p];
    off_ab = G * ((long long)a + (long long)ca.nspf * b);
    off_ba = G * ((long long)b + (long long)ca.nspf * a);
    mirror = herm && a != b;
  } else {
    off_ab = G * gp;
  }
  for (int i = threadIdx.x; i < nrow * N; i += blockDim.x) {
    int r = i / N, x = i - r * N;
    double2 v = res[r * P + x];
    long long g = gbase + (long long)r * N + x;
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

static int coul_run(Ctx& c, const double2* src1, const double2* src2, const int* h_pa,
                    const int* h_pb, int npair, double* Rpl, double2* full, bool herm, bool dens) {
  const int N = c.N, P = c.P, tx = c.tx;
  const long long per_pair = 16LL * ((long long)N * N * P + (long long)N * P * P);
  int chunk = c.coul_chunk;
  if (chunk <= 0) {
    const long long budget = 48LL << 20;
    chunk = (int)std::max(1LL, budget / per_pair);
  }
  chunk = std::min(chunk, npair);
  const size_t ws_fft = (size_t)per_pair * chunk;
  const size_t ws_pair = sizeof(int) * 2 * (size_t)npair;
  SG_TRY(c.ws_fft.ensure(ws_fft));
  SG_TRY(c.ws_pairs.ensure(ws_pair));
  int* d_pa = (int*)c.ws_pairs.ptr;
  int* d_pb = d_pa + npair;
  if (!dens) {
    SG_CUDA(cudaMemcpyAsync(d_pa, h_pa, sizeof(int) * npair, cudaMemcpyHostToDevice, c.stream));
    SG_CUDA(cudaMemcpyAsync(d_pb, h_pb, sizeof(int) * npair, cudaMemcpyHostToDevice, c.stream));
  }
  CoulArgs ca{};
  ca.N = N;
  ca.P = P;
  ca.tx = tx;
  ca.nspf = c.nspf;
  ca.G = c.G;
  ca.plan = c.plan;
  ca.roots = c.d_roots;
  ca.khat = c.d_khat;
  ca.W1 = (double2*)c.ws_fft.ptr;
  ca.W2 = ca.W1 + (long long)chunk * N * N * P;
  ca.npair_total = npair;

  const size_t smx = sizeof(double2) * (P + 2 * kRowTile * P);
  const size_t smc = sizeof(double2) * (P + 2 * P * tx);
  static bool attr_done = false;
  if (!attr_done) {
    SG_CUDA(cudaFuncSetAttribute(coul_fwd_y, cudaFuncAttributeMaxDynamicSharedMemorySize, 160 * 1024));
    SG_CUDA(cudaFuncSetAttribute(coul_z, cudaFuncAttributeMaxDynamicSharedMemorySize, 160 * 1024));
    SG_CUDA(cudaFuncSetAttribute(coul_inv_y, cudaFuncAttributeMaxDynamicSharedMemorySize, 160 * 1024));
    SG_CUDA(cudaFuncSetAttribute(coul_fwd_x<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, 160 * 1024));
    SG_CUDA(cudaFuncSetAttribute(coul_fwd_x<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, 160 * 1024));
    SG_CUDA(cudaFuncSetAttribute(coul_inv_x<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, 160 * 1024));
    SG_CUDA(cudaFuncSetAttribute(coul_inv_x<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, 160 * 1024));
    attr_done = true;
  }
  SG_CHECK(smc <= 160 * 1024, SINCGPU_ERANGE, "column tile needs %zu bytes of shared memory", smc);
  const int nyb = ceil_div(N, kRowTile), nxt = ceil_div(P, tx);
  for (int p0 = 0; p0 < npair; p0 += chunk) {
    const int np = std::min(chunk, npair - p0);
    ca.pair0 = p0;
    ca.pa = d_pa + p0;
    ca.pb = d_pb + p0;
    {
      ProfScope ps(c, ST_COUL_FWD_X);
      if (dens)
        coul_fwd_x<true><<<dim3(nyb, N, np), kThreads, smx, c.stream>>>(src1, nullptr, ca);
      else
        coul_fwd_x<false><<<dim3(nyb, N, np), kThreads, smx, c.stream>>>(src1, src2, ca);
      SG_LAUNCHED();
    }
    {
      ProfScope ps(c, ST_COUL_FWD_Y);
      coul_fwd_y<<<dim3(nxt, N, np), kThreads, smc, c.stream>>>(ca);
      SG_LAUNCHED();
    }
    {
      ProfScope ps(c, ST_COUL_Z);
      coul_z<<<dim3(nxt, P, np), kThreads, smc, c.stream>>>(ca);
      SG_LAUNCHED();
    }
    {
      ProfScope ps(c, ST_COUL_INV_Y);
      coul_inv_y<<<dim3(nxt, N, np), kThreads, smc, c.stream>>>(ca);
      SG_LAUNCHED();
    }
    {
      ProfScope ps(c, ST_COUL_INV_X);
      if (dens)
        coul_inv_x<true><<<dim3(nyb, N, np), kThreads, smx, c.stream>>>(ca, Rpl, full, 0);
      else
        coul_inv_x<false><<<dim3(nyb, N, np), kThreads, smx, c.stream>>>(ca, Rpl, full, herm ? 1 : 0);
      SG_LAUNCHED();
    }
  }
  return SINCGPU_OK;
}

int coulomb_pairs(Ctx& c, const double2* phi1, const double2* phi2, const int* h_pa,
                  const int* h_pb, int npair, double* Rpl, double2* full, bool herm) {
  return coul_run(c, phi1, phi2, h_pa, h_pb, npair, Rpl, full, herm, false);
}

int coulomb_dens(Ctx& c, const double2* dens, int m, double2* red) {
  return coul_run(c, dens, nullptr, nullptr, nullptr, m, nullptr, red, false, true);
}

}  // namespace sincgpu
