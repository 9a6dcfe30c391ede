// Set-up of the sinc-DVR tables on the device:
//   * 1-D kinetic Toeplitz vector K(d)           SINCDVR/SineDVR.f90:11-44
//   * inverse 3-D kinetic operator (Coulomb)      SINCDVR/tooth.f90:12-231
//   * threed_two / nuclear potential              SINCDVR/sincproject.f90:119-256
//   * DFT of the zero-padded Coulomb kernel, computed once (the reference
//     recomputes FFT(threed_two) inside every circ3d_sub call,
//     SINCDVR/toeplitz_subs.f90:574).
#include <cmath>
#include <cstring>
#include <vector>
#include <algorithm>
#include <mutex>
#include <set>
#include "context.hpp"
#include "fft_lengths.h"

namespace sincgpu {

static std::vector<int (*)()>& root_uploaders() {
  static std::vector<int (*)()> v;
  return v;
}

int register_const_roots(int (*upload)()) {
  root_uploaders().push_back(upload);
  return 1;
}

int upload_const_roots(int device) {
  static std::mutex mu;
  static std::set<int> done;
  std::lock_guard<std::mutex> lk(mu);
  if (done.count(device)) return SINCGPU_OK;
  for (int (*f)() : root_uploaders())
    SG_CHECK(f() == 0, SINCGPU_ECUDA, "upload of the constant twiddle tables failed");
  done.insert(device);
  return SINCGPU_OK;
}


static const double kPi = 3.14159265358979323846264338327950288;

// ---------------------------------------------------------------------------
// FFT plan: P >= 2N-1 with prime factors <= 7.  Any such P gives exactly the
// linear convolution the reference computes on its 2N grid (density support
// [0,N), kernel support [1-N,N-1]).
// ---------------------------------------------------------------------------
static bool smooth7(int p) {
  for (int r : {2, 3, 5, 7})
    while (p % r == 0) p /= r;
  return p == 1;
}

int fft_length_for(int min_len, int* p1, int* p2);  // coulomb.cu

int choose_plan(Ctx& c) {
  int P = fft_length_for(2 * c.N - 1, nullptr, nullptr);
  SG_CHECK(P > 0 && P <= kMaxFftLen && smooth7(P), SINCGPU_ERANGE,
           "no supported padded FFT length >= %d (N=%d)", 2 * c.N - 1, c.N);
  FftPlan pl{};
  pl.P = P;
  int p = P, k = 0;
  for (int r : {4, 2, 3, 5, 7}) {
    while (p % r == 0) {
      SG_CHECK(k < kMaxRadices, SINCGPU_ERANGE, "too many FFT stages");
      pl.rad[k++] = r;
      p /= r;
    }
  }
  pl.nrad = k;
  c.plan = pl;
  c.P = P;
  // column tile: largest divisor of P in [8,32] whose double buffer fits 100 KB
  int tx = 0;
  for (int t = 32; t >= 8; --t)
    if (P % t == 0 && 2LL * P * t * 16 <= 100 * 1024) {
      tx = t;
      break;
    }
  if (tx == 0) tx = 16;
  c.tx = tx;
  std::vector<double2> roots(P);
  for (int m = 0; m < P; ++m) {
    long double ang = -2.0L * 3.14159265358979323846264338327950288L * (long double)m / (long double)P;
    roots[m] = make_double2((double)cosl(ang), (double)sinl(ang));
  }
  SG_TRY(dupload(c, (void**)&c.d_roots, roots.data(), sizeof(double2) * P));
  return SINCGPU_OK;
}

// ---------------------------------------------------------------------------
// 1-D sinc-DVR kinetic vector (SineDVR.f90:22-34): K(0) = pi^2/3, K(d) =
// 2(-1)^d/d^2, all / (2 spacing^2); and the padded S x S tile K(j-l) used by the
// DMMA kinetic kernels (rows/cols >= N are zero).
// ---------------------------------------------------------------------------
static int build_kinetic(Ctx& c) {
  const int N = c.N;
  std::vector<double> ke(2 * N - 1);
  const double mypi = 4.0 * std::atan(1.0);
  for (int i = 1 - N; i <= N - 1; ++i) {
    double v;
    if (i == 0)
      v = mypi * mypi / 3.0;
    else
      v = 2.0 / ((double)i * (double)i) * ((i % 2) ? -1.0 : 1.0);
    ke[i + N - 1] = v / 2.0 / (c.spacing * c.spacing);
  }
  // row stride: multiple of 8 rows/cols rounded to 4 (mod 16) doubles so that
  // the m8n8k4 fragment loads are free of bank conflicts
  int n8 = (N + 7) / 8 * 8;
  int S = n8;
  while (S % 16 != 4) ++S;
  c.ke_stride = S;
  std::vector<double> tile((size_t)S * S, 0.0);
  for (int j = 0; j < N; ++j)
    for (int l = 0; l < N; ++l) tile[(size_t)j * S + l] = ke[(j - l) + N - 1];
  SG_TRY(dupload(c, (void**)&c.d_kevect, ke.data(), sizeof(double) * ke.size()));
  SG_TRY(dupload(c, (void**)&c.d_ketile, tile.data(), sizeof(double) * tile.size()));
  return SINCGPU_OK;
}

// ---------------------------------------------------------------------------
// getinverse (tooth.f90:12-95)
// ---------------------------------------------------------------------------

// DELTA^3/SQRT(PPOS(a)**2+PPOS(b)**2+PPOS(c)**2), rounded exactly as written:
// no fused multiply-add, left-to-right association (tooth.f90:141).
__device__ __forceinline__ double rcoul(int a, int b, int cc, double delta, double d3) {
  double pa = __dmul_rn((double)a, delta), pb = __dmul_rn((double)b, delta),
         pc = __dmul_rn((double)cc, delta);
  double s = __dadd_rn(__dmul_rn(pa, pa), __dmul_rn(pb, pb));
  s = __dadd_rn(s, __dmul_rn(pc, pc));
  return __ddiv_rn(d3, __dsqrt_rn(s));
}

// TR(I,J,K) = -sum_p [ALLTT(p-I) R(p,J,K) + ALLTT(p-J) R(I,p,K) + ALLTT(p-K) R(I,J,p)]
// + 2 pi delta_{IJK,0}   (tooth.f90:44, 158-181; line 165 in its intended,
// conformable form ALLTT(-NBIG-J:NBIG-J)).
__global__ void tr_kernel(double* __restrict__ tr, const double* __restrict__ alltt, int ns,
                          int nbig, double delta, double d3) {
  const int NS = 2 * ns + 1;
  long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (idx >= (long long)NS * NS * NS) return;
  int i = (int)(idx % NS) - ns;
  int j = (int)((idx / NS) % NS) - ns;
  int k = (int)(idx / ((long long)NS * NS)) - ns;
  const int off = ns + nbig;
  double acc = 0.0;
  for (int p = -nbig; p <= nbig; ++p) {
    double r1 = (p == 0 && j == 0 && k == 0) ? 0.0 : rcoul(p, j, k, delta, d3);
    double r2 = (i == 0 && p == 0 && k == 0) ? 0.0 : rcoul(i, p, k, delta, d3);
    double r3 = (i == 0 && j == 0 && p == 0) ? 0.0 : rcoul(i, j, p, delta, d3);
    double t = __dadd_rn(__dmul_rn(alltt[p - i + off], r1), __dmul_rn(alltt[p - j + off], r2));
    t = __dadd_rn(t, __dmul_rn(alltt[p - k + off], r3));
    acc = __dadd_rn(acc, t);
  }
  double v = -acc;
  if (i == 0 && j == 0 && k == 0) v = __dadd_rn(v, 2.0 * 3.14159265358979323846);
  tr[idx] = v;
}

// Y = (mode-`axis` product with M) X on an NS^3 cube; M(a,b) column-major.
// TOOTHEIGMULT (tooth.f90:191-231) applies axis 3, then 2, then 1.
__global__ void mode_mult_kernel(const double* __restrict__ X, double* __restrict__ Y,
                                 const double* __restrict__ M, int NS, int axis) {
  long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (idx >= (long long)NS * NS * NS) return;
  int c0 = (int)(idx % NS), c1 = (int)((idx / NS) % NS), c2 = (int)(idx / ((long long)NS * NS));
  int a = axis == 0 ? c0 : (axis == 1 ? c1 : c2);
  long long stride = axis == 0 ? 1 : (axis == 1 ? NS : (long long)NS * NS);
  long long base = idx - (long long)a * stride;
  double acc = 0.0;
  for (int b = 0; b < NS; ++b) acc = fma(M[a + (long long)NS * b], X[base + b * stride], acc);
  Y[idx] = acc;
}

__global__ void divide_eigs_kernel(double* __restrict__ QQ, const double* __restrict__ E, int NS) {
  long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (idx >= (long long)NS * NS * NS) return;
  int c0 = (int)(idx % NS), c1 = (int)((idx / NS) % NS), c2 = (int)(idx / ((long long)NS * NS));
  QQ[idx] = QQ[idx] / (E[c0] + E[c1] + E[c2]);
}

// tempcoulomb(d) = TINV(d)/spacing^3 on [1-N,N-1]^3 with TINV = R (+ Q on the
// small grid)  (tooth.f90:83-89, sincproject.f90:155-156, 182-187).
__global__ void assemble_t_kernel(double* __restrict__ T, const double* __restrict__ Q, int N,
                                  int ns, double delta, double d3) {
  const int W = 2 * N - 1;
  long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (idx >= (long long)W * W * W) return;
  int a = (int)(idx % W) - (N - 1), b = (int)((idx / W) % W) - (N - 1),
      cc = (int)(idx / ((long long)W * W)) - (N - 1);
  double v = (a == 0 && b == 0 && cc == 0) ? 0.0 : rcoul(a, b, cc, delta, d3);
  if (abs(a) <= ns && abs(b) <= ns && abs(cc) <= ns) {
    const int NS = 2 * ns + 1;
    v = __dadd_rn(v, Q[(a + ns) + (long long)NS * ((b + ns) + (long long)NS * (cc + ns))]);
  }
  T[idx] = __ddiv_rn(v, d3);
}

// Cyclic Jacobi eigen-solver for the small symmetric 1-D matrix T (NS x NS).
// The reference calls LAPACK DSYEV (tooth.f90:64); Q = V (V^T TR / EIGS) V^T
// does not depend on eigenvector signs or order.
static void jacobi_eigen(std::vector<double>& A, int n, std::vector<double>& E,
                         std::vector<double>& V) {
  V.assign((size_t)n * n, 0.0);
  for (int i = 0; i < n; ++i) V[(size_t)i * n + i] = 1.0;
  for (int sweep = 0; sweep < 100; ++sweep) {
    double off = 0.0;
    for (int q = 0; q < n; ++q)
      for (int p = 0; p < q; ++p) off += A[(size_t)p + (size_t)n * q] * A[(size_t)p + (size_t)n * q];
    if (off < 1e-30) break;
    for (int p = 0; p < n - 1; ++p)
      for (int q = p + 1; q < n; ++q) {
        double apq = A[p + (size_t)n * q];
        if (apq == 0.0) continue;
        double app = A[p + (size_t)n * p], aqq = A[q + (size_t)n * q];
        double theta = (aqq - app) / (2.0 * apq);
        double t = (theta >= 0 ? 1.0 : -1.0) / (std::fabs(theta) + std::sqrt(theta * theta + 1.0));
        double cs = 1.0 / std::sqrt(t * t + 1.0), sn = t * cs;
        for (int k = 0; k < n; ++k) {  // columns p,q
          double akp = A[k + (size_t)n * p], akq = A[k + (size_t)n * q];
          A[k + (size_t)n * p] = cs * akp - sn * akq;
          A[k + (size_t)n * q] = sn * akp + cs * akq;
        }
        for (int k = 0; k < n; ++k) {  // rows p,q
          double apk = A[p + (size_t)n * k], aqk = A[q + (size_t)n * k];
          A[p + (size_t)n * k] = cs * apk - sn * aqk;
          A[q + (size_t)n * k] = sn * apk + cs * aqk;
        }
        for (int k = 0; k < n; ++k) {
          double vkp = V[k + (size_t)n * p], vkq = V[k + (size_t)n * q];
          V[k + (size_t)n * p] = cs * vkp - sn * vkq;
          V[k + (size_t)n * q] = sn * vkp + cs * vkq;
        }
      }
  }
  E.resize(n);
  for (int i = 0; i < n; ++i) E[i] = A[i + (size_t)n * i];
}

static int build_tcoul(Ctx& c, int nbig, int ns) {
  const int N = c.N;
  const double delta = c.spacing;
  const double d3 = (delta * delta) * delta;
  SG_CHECK(nbig > ns, SINCGPU_EINVAL, "toothnbig (%d) must exceed toothnsmall (%d)", nbig, ns);
  const int NS = 2 * ns + 1;
  const long long ncube = (long long)NS * NS * NS;
  // ALLTT (tooth.f90:152-156)
  std::vector<double> alltt(2 * (ns + nbig) + 1);
  const double d2inv = 1.0 / (delta * delta);
  for (int m = -(ns + nbig); m <= ns + nbig; ++m) {
    double v = (m == 0) ? (kPi * kPi / (6.0 * delta * delta))
                        : ((m % 2) ? -1.0 : 1.0) * d2inv / ((double)m * (double)m);
    alltt[m + ns + nbig] = v;
  }
  // 1-D T_small (tooth.f90:48-53)
  std::vector<double> Tm((size_t)NS * NS);
  for (int j = -ns; j <= ns; ++j)
    for (int i = -ns; i <= ns; ++i) {
      int d = i - j;
      double v = (d == 0) ? (kPi / delta) * (kPi / delta) / 6.0
                          : ((d % 2) ? -1.0 : 1.0) / (delta * delta * (double)d * (double)d);
      Tm[(i + ns) + (size_t)NS * (j + ns)] = v;
    }
  std::vector<double> E, V;
  jacobi_eigen(Tm, NS, E, V);
  std::vector<double> VT((size_t)NS * NS);
  for (int a = 0; a < NS; ++a)
    for (int b = 0; b < NS; ++b) VT[a + (size_t)NS * b] = V[b + (size_t)NS * a];

  double *d_alltt = nullptr, *d_x = nullptr, *d_y = nullptr, *d_V = nullptr, *d_VT = nullptr,
         *d_E = nullptr;
  int rc = SINCGPU_OK;
  auto cleanup = [&]() {
    for (double* p : {d_alltt, d_x, d_y, d_V, d_VT, d_E}) dfree(c, p);
  };
  do {
    if (dupload(c, (void**)&d_alltt, alltt.data(), sizeof(double) * alltt.size()) != SINCGPU_OK ||
        dalloc(c, &d_x, sizeof(double) * ncube) != SINCGPU_OK ||
        dalloc(c, &d_y, sizeof(double) * ncube) != SINCGPU_OK ||
        dupload(c, (void**)&d_V, V.data(), sizeof(double) * NS * NS) != SINCGPU_OK ||
        dupload(c, (void**)&d_VT, VT.data(), sizeof(double) * NS * NS) != SINCGPU_OK ||
        dupload(c, (void**)&d_E, E.data(), sizeof(double) * NS) != SINCGPU_OK) {
      set_error("device allocation failed in getinverse");
      rc = SINCGPU_ENOMEM;
      break;
    }
    const int tb = 256;
    const int gb = ceil_div(ncube, tb);
    cudaStream_t st = c.stream;
    tr_kernel<<<gb, tb, 0, st>>>(d_x, d_alltt, ns, nbig, delta, d3);
    // QQ = TOOTHEIGMULT(TR, W^T): axis 3, 2, 1
    mode_mult_kernel<<<gb, tb, 0, st>>>(d_x, d_y, d_VT, NS, 2);
    mode_mult_kernel<<<gb, tb, 0, st>>>(d_y, d_x, d_VT, NS, 1);
    mode_mult_kernel<<<gb, tb, 0, st>>>(d_x, d_y, d_VT, NS, 0);
    divide_eigs_kernel<<<gb, tb, 0, st>>>(d_y, d_E, NS);
    mode_mult_kernel<<<gb, tb, 0, st>>>(d_y, d_x, d_V, NS, 2);
    mode_mult_kernel<<<gb, tb, 0, st>>>(d_x, d_y, d_V, NS, 1);
    mode_mult_kernel<<<gb, tb, 0, st>>>(d_y, d_x, d_V, NS, 0);  // Q in d_x
    const int W = 2 * N - 1;
    const long long nw = (long long)W * W * W;
    dfree(c, c.d_tcoul);
    c.d_tcoul = nullptr;
    if (dalloc(c, &c.d_tcoul, sizeof(double) * nw) != SINCGPU_OK) {
      set_error("device allocation failed for the Coulomb table");
      rc = SINCGPU_ENOMEM;
      break;
    }
    assemble_t_kernel<<<ceil_div(nw, tb), tb, 0, st>>>(c.d_tcoul, d_x, N, ns, delta, d3);
    cudaError_t e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) {
      set_error("getinverse kernels: %s", cudaGetErrorString(e));
      rc = SINCGPU_ECUDA;
    }
  } while (0);
  cleanup();
  return rc;
}

// ---------------------------------------------------------------------------
// nuclear potential (sincproject.f90:192-250) and z dipole (init_sinc_new.f90:619-645)
// ---------------------------------------------------------------------------
struct Centers {
  int n;
  int pp[3 * 16];
  double z[16];
};

__global__ void pot_kernel(double* __restrict__ pot, const double* __restrict__ T, Centers cen,
                           int N, double spacing, int sqrt32) {
  long long g = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  const long long G = (long long)N * N * N;
  if (g >= G) return;
  int ix = (int)(g % N), iy = (int)((g / N) % N), iz = (int)(g / ((long long)N * N));
  const int W = 2 * N - 1;
  double acc = 0.0;
  for (int c = 0; c < cen.n; ++c) {
    int a = cen.pp[3 * c] + ix, b = cen.pp[3 * c + 1] + iy, cc = cen.pp[3 * c + 2] + iz;
    double v;
    if (abs(a) <= N - 1 && abs(b) <= N - 1 && abs(cc) <= N - 1) {
      v = T[(a + N - 1) + (long long)W * ((b + N - 1) + (long long)W * (cc + N - 1))];
    } else {
      int isq = a * a + b * b + cc * cc;
      double rt = sqrt32 ? (double)sqrtf((float)isq) : __dsqrt_rn((double)isq);
      v = __ddiv_rn(1.0, __dmul_rn(spacing, rt));
    }
    acc = __dsub_rn(acc, __dmul_rn(1.0 * cen.z[c], v));
  }
  pot[g] = acc;
}

__global__ void zdip_kernel(double* __restrict__ zdip, const double* __restrict__ points, int N) {
  long long g = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  const long long G = (long long)N * N * N;
  if (g >= G) return;
  zdip[g] = points[g / ((long long)N * N)];
}

static int fortran_div2(int a) { return a / 2; }  // C++ truncates toward zero like Fortran
static int fortran_mod2(int a) { return a % 2; }   // sign follows the dividend like Fortran MOD

static int build_pot(Ctx& c, int sqrt32) {
  const int N = c.N;
  SG_CHECK(c.numcenters <= 16, SINCGPU_EINVAL, "at most 16 nuclear centers (got %d)", c.numcenters);
  Centers cen{};
  cen.n = c.numcenters;
  for (int i = 0; i < c.numcenters; ++i) {
    for (int k = 0; k < 3; ++k) {
      int cs = c.centershift[3 * i + k];
      int pp = -N + cs + 1, qq = N + cs - 1;
      SG_CHECK(!(fortran_mod2(qq) == 1 || fortran_mod2(pp) == 1), SINCGPU_EINVAL,
               "nucleus %d axis %d: centershift %d has the wrong parity for %d points "
               "(must be even for odd N, odd for even N)", i + 1, k + 1, cs, N);
      cen.pp[3 * i + k] = fortran_div2(pp);
    }
    cen.z[i] = c.nuccharges[i];
  }
  // grid coordinates (SineDVR.f90:15-19)
  std::vector<double> pts(N);
  for (int i = 0; i < N; ++i) pts[i] = (i + 1) * c.spacing;
  double mid = (pts[0] + pts[N - 1]) / 2.0;
  for (int i = 0; i < N; ++i) pts[i] -= mid;
  double* d_pts = nullptr;
  SG_TRY(dupload(c, (void**)&d_pts, pts.data(), sizeof(double) * N));
  dfree(c, c.d_pot);
  dfree(c, c.d_zdip);
  c.d_pot = c.d_zdip = nullptr;
  SG_TRY(dalloc(c, &c.d_pot, sizeof(double) * c.G));
  SG_TRY(dalloc(c, &c.d_zdip, sizeof(double) * c.G));
  pot_kernel<<<ceil_div(c.G, 256), 256, 0, c.stream>>>(c.d_pot, c.d_tcoul, cen, N, c.spacing, sqrt32);
  zdip_kernel<<<ceil_div(c.G, 256), 256, 0, c.stream>>>(c.d_zdip, d_pts, N);
  dfree(c, d_pts);
  cudaError_t e = cudaStreamSynchronize(c.stream);
  SG_CHECK(e == cudaSuccess, SINCGPU_ECUDA, "potential kernels: %s", cudaGetErrorString(e));
  // nuclear repulsion (sinc_extraproject.f90:290-300)
  double nr = 0.0;
  for (int i = 0; i < c.numcenters; ++i)
    for (int j = i + 1; j < c.numcenters; ++j) {
      double rsq[3];
      for (int k = 0; k < 3; ++k) {
        double d = (c.centershift[3 * i + k] - c.centershift[3 * j + k]) * c.spacing / 2;
        rsq[k] = d * d;
      }
      nr += c.nuccharges[i] * c.nuccharges[j] / std::sqrt(rsq[0] + rsq[1] + rsq[2]);
    }
  c.nucrepulsion = nr;
  return SINCGPU_OK;
}

// ---------------------------------------------------------------------------
// kernel spectrum: khat = DFT_P^3( T(d) at d mod P ) / P^3
// ---------------------------------------------------------------------------
__global__ void embed_kernel(double2* __restrict__ out, const double* __restrict__ T, int N, int P) {
  long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  const long long P3 = (long long)P * P * P;
  if (idx >= P3) return;
  int m0 = (int)(idx % P), m1 = (int)((idx / P) % P), m2 = (int)(idx / ((long long)P * P));
  auto dof = [&](int m) { return m <= N - 1 ? m : (m >= P - (N - 1) ? m - P : 1 << 20); };
  int a = dof(m0), b = dof(m1), cc = dof(m2);
  double v = 0.0;
  if (a != (1 << 20) && b != (1 << 20) && cc != (1 << 20)) {
    const int W = 2 * N - 1;
    v = T[(a + N - 1) + (long long)W * ((b + N - 1) + (long long)W * (cc + N - 1))];
  }
  out[idx] = make_double2(v, 0.0);
}

// In-place forward DFT of a full P^3 array along one axis.
// axis 0: rows of P contiguous points; axes 1,2: column tiles of `tx` lines.
__global__ void fft_full_axis_kernel(double2* __restrict__ data, FftPlan plan,
                                     const double2* __restrict__ roots_g, int axis, int tx,
                                     double scale) {
  extern __shared__ double2 smem[];
  const int P = plan.P;
  double2* roots = smem;
  for (int i = threadIdx.x; i < P; i += blockDim.x) roots[i] = roots_g[i];
  double2* A = smem + P;
  if (axis == 0) {
    // one block = 8 rows
    const int rows = 8, ls = P + 1;
    double2* B = A + rows * ls;
    long long row0 = (long long)blockIdx.x * rows;
    const long long nrows = (long long)P * P;
    for (int i = threadIdx.x; i < rows * P; i += blockDim.x) {
      int r = i / P, j = i % P;
      long long row = row0 + r;
      A[r * ls + j] = row < nrows ? data[row * P + j] : make_double2(0, 0);
    }
    __syncthreads();
    double2* res = fft_lines<false>(A, B, rows, ls, 1, plan, roots, false);
    for (int i = threadIdx.x; i < rows * P; i += blockDim.x) {
      int r = i / P, j = i % P;
      long long row = row0 + r;
      if (row < nrows) data[row * P + j] = cscale(res[r * ls + j], scale);
    }
  } else {
    // lines along axis (stride sl), tile of tx consecutive x, outer index o
    const long long sl = axis == 1 ? P : (long long)P * P;
    const long long so = axis == 1 ? (long long)P * P : P;
    double2* B = A + P * tx;
    int x0 = blockIdx.x * tx;
    int o = blockIdx.y;
    for (int i = threadIdx.x; i < P * tx; i += blockDim.x) {
      int j = i / tx, l = i % tx;
      int x = x0 + l;
      A[j * tx + l] = x < P ? data[o * so + j * sl + x] : make_double2(0, 0);
    }
    __syncthreads();
    double2* res = fft_lines<false>(A, B, tx, 1, tx, plan, roots, true);
    for (int i = threadIdx.x; i < P * tx; i += blockDim.x) {
      int j = i / tx, l = i % tx;
      int x = x0 + l;
      if (x < P) data[o * so + j * sl + x] = cscale(res[j * tx + l], scale);
    }
  }
}

// khr[(fz H + fy) H + fx] = Re khat[(fz P + fy) P + fx] for f <= P/2, H = P/2 + 1
// (P <= 128), or khr[i] = Re khat[i] over the whole table (longer lengths)
__global__ void khat_real_kernel(double* __restrict__ out, const double2* __restrict__ in, int P) {
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (P > 128) {
    if (i < (long long)P * P * P) out[i] = in[i].x;
    return;
  }
  const int H = P / 2 + 1;
  if (i >= (long long)H * H * H) return;
  const int fx = (int)(i % H), fy = (int)((i / H) % H), fz = (int)(i / ((long long)H * H));
  out[i] = in[((long long)fz * P + fy) * P + fx].x;
}

__global__ void narrow_real_kernel(float* __restrict__ out, const double* __restrict__ in, long long n) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x)
    out[i] = (float)in[i];
}

int make_khat(Ctx& c) {
  const int P = c.P;
  const long long P3 = (long long)P * P * P;
  dfree(c, c.d_khat);
  dfree(c, c.d_khat32);  // FP32 copies and the transposed spectra follow the FP64 tables
  dfree(c, c.d_roots32);
  dfree(c, c.d_khT);
  dfree(c, c.d_khT32);
  dfree(c, c.d_khr);
  dfree(c, c.d_khr32);
  c.d_khr = nullptr;
  c.d_khr32 = nullptr;
  c.d_khat = nullptr;
  c.d_khat32 = nullptr;
  c.d_roots32 = nullptr;
  c.d_khT = nullptr;
  c.d_khT32 = nullptr;
  SG_TRY(dalloc(c, &c.d_khat, sizeof(double2) * P3));
  embed_kernel<<<ceil_div(P3, 256), 256, 0, c.stream>>>(c.d_khat, c.d_tcoul, c.N, P);
  SG_LAUNCHED();
  size_t sm0 = sizeof(double2) * (P + 2 * 8 * (P + 1));
  size_t sm1 = sizeof(double2) * (P + 2 * P * c.tx);
  size_t smax = std::max(sm0, sm1);
  // the attribute is process-wide: always the same (largest) value, so contexts
  // created concurrently on several threads never lower it under each other
  constexpr int kSmemOptIn = 227 * 1024;
  SG_CHECK(smax <= (size_t)kSmemOptIn, SINCGPU_ERANGE, "kernel-spectrum FFT needs %zu bytes of shared memory", smax);
  SG_CUDA(cudaFuncSetAttribute(fft_full_axis_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, kSmemOptIn));
  fft_full_axis_kernel<<<ceil_div((long long)P * P, 8), 128, sm0, c.stream>>>(c.d_khat, c.plan, c.d_roots, 0,
                                                                              c.tx, 1.0);
  SG_LAUNCHED();
  dim3 g1(ceil_div(P, c.tx), P);
  fft_full_axis_kernel<<<g1, 128, sm1, c.stream>>>(c.d_khat, c.plan, c.d_roots, 1, c.tx, 1.0);
  SG_LAUNCHED();
  const double inv = 1.0 / ((double)P * (double)P * (double)P);
  fft_full_axis_kernel<<<g1, 128, sm1, c.stream>>>(c.d_khat, c.plan, c.d_roots, 2, c.tx, inv);
  SG_LAUNCHED();
  const long long nkr = khr_len(P);
  SG_TRY(dalloc(c, &c.d_khr, sizeof(double) * nkr));
  khat_real_kernel<<<ceil_div(nkr, 256), 256, 0, c.stream>>>(c.d_khr, c.d_khat, P);
  SG_LAUNCHED();
  SG_CUDA(cudaStreamSynchronize(c.stream));
  return SINCGPU_OK;
}

__global__ void narrow_kernel(float2* __restrict__ out, const double2* __restrict__ in, long long n) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x)
    out[i] = make_float2((float)in[i].x, (float)in[i].y);
}

int ensure_fp32_tables(Ctx& c) {
  if (c.d_khat32 && c.d_roots32 && c.d_khr32) return SINCGPU_OK;  // no stream work once built (graph capture)
  const long long P3 = (long long)c.P * c.P * c.P;
  if (!c.d_khr32) {
    const long long nkr = khr_len(c.P);
    SG_TRY(dalloc(c, &c.d_khr32, sizeof(float) * nkr));
    narrow_real_kernel<<<std::min<long long>(ceil_div(nkr, 256), 148 * 16), 256, 0, c.stream>>>(c.d_khr32, c.d_khr,
                                                                                               nkr);
    SG_LAUNCHED();
  }
  if (!c.d_khat32) {
    SG_TRY(dalloc(c, &c.d_khat32, sizeof(float2) * P3));
    narrow_kernel<<<std::min<long long>(ceil_div(P3, 256), 148 * 16), 256, 0, c.stream>>>(c.d_khat32,
                                                                                        c.d_khat, P3);
    SG_LAUNCHED();
  }
  if (!c.d_roots32) {
    SG_TRY(dalloc(c, &c.d_roots32, sizeof(float2) * c.P));
    narrow_kernel<<<1, 256, 0, c.stream>>>(c.d_roots32, c.d_roots, c.P);
    SG_LAUNCHED();
  }
  SG_CUDA(cudaStreamSynchronize(c.stream));
  return SINCGPU_OK;
}

// khT[(kx P + kz) P + ky] = Re khat[(kz P + ky) P + kx], and its FP32 rounding
template <class R>
__global__ void khat_transpose_kernel(R* __restrict__ out, const double2* __restrict__ in, int P) {
  const long long P3 = (long long)P * P * P;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < P3;
       i += (long long)gridDim.x * blockDim.x) {
    const long long kx = i / ((long long)P * P);
    const long long rem = i - kx * P * P;
    const long long kz = rem / P, ky = rem - kz * P;
    out[i] = (R)in[(kz * P + ky) * P + kx].x;
  }
}

int ensure_khT(Ctx& c, bool fp32) {
  if (fp32 ? c.d_khT32 != nullptr : c.d_khT != nullptr) return SINCGPU_OK;  // no stream work once built
  const long long P3 = (long long)c.P * c.P * c.P;
  const int grid = (int)std::min<long long>(ceil_div(P3, 256), 148 * 16);
  if (fp32) {
    SG_TRY(dalloc(c, &c.d_khT32, sizeof(float) * P3));
    khat_transpose_kernel<float><<<grid, 256, 0, c.stream>>>(c.d_khT32, c.d_khat, c.P);
  } else {
    SG_TRY(dalloc(c, &c.d_khT, sizeof(double) * P3));
    khat_transpose_kernel<double><<<grid, 256, 0, c.stream>>>(c.d_khT, c.d_khat, c.P);
  }
  SG_LAUNCHED();
  SG_CUDA(cudaStreamSynchronize(c.stream));
  return SINCGPU_OK;
}

int build_tables(Ctx& c, int toothnbig, int toothnsmall, int flags) {
  if (toothnbig < c.N - 1) toothnbig = c.N - 1;  // sinc_extraproject.f90:273-276
  SG_TRY(choose_plan(c));
  SG_TRY(build_kinetic(c));
  SG_TRY(build_tcoul(c, toothnbig, toothnsmall));
  SG_TRY(build_pot(c, (flags & 1) ? 1 : 0));
  if (flags & 2) {  // notwoflag (sincproject.f90:330-332)
    const long long W = 2LL * c.N - 1;
    SG_CUDA(cudaMemsetAsync(c.d_tcoul, 0, sizeof(double) * W * W * W, c.stream));
  }
  SG_TRY(make_khat(c));
  return SINCGPU_OK;
}

// threed_two(-N:N-1)^3 (complex, real valued) and pot supplied by the caller,
// i.e. by the unchanged Fortran init_project (init_sinc_new.f90:533).
__global__ void take_threed_kernel(double* __restrict__ T, const double2* __restrict__ t2, int N) {
  const int W = 2 * N - 1;
  long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (idx >= (long long)W * W * W) return;
  int a = (int)(idx % W), b = (int)((idx / W) % W), cc = (int)(idx / ((long long)W * W));
  const long long M = 2LL * N;
  T[idx] = t2[(a + 1) + M * ((b + 1) + M * (cc + 1))].x;
}

int build_tables_from_arrays(Ctx& c, const double2* threed_two_host, const double* pot_host) {
  SG_TRY(choose_plan(c));
  SG_TRY(build_kinetic(c));
  const int N = c.N;
  const long long M3 = 8LL * N * N * N;
  const long long W = 2LL * N - 1;
  double2* d_t2 = nullptr;
  SG_TRY(dupload(c, (void**)&d_t2, threed_two_host, sizeof(double2) * M3));
  dfree(c, c.d_tcoul);
  c.d_tcoul = nullptr;
  SG_TRY(dalloc(c, &c.d_tcoul, sizeof(double) * W * W * W));
  take_threed_kernel<<<ceil_div(W * W * W, 256), 256, 0, c.stream>>>(c.d_tcoul, d_t2, N);
  dfree(c, d_t2);
  cudaError_t e = cudaStreamSynchronize(c.stream);
  SG_CHECK(e == cudaSuccess, SINCGPU_ECUDA, "threed_two upload: %s", cudaGetErrorString(e));
  dfree(c, c.d_zdip);
  c.d_zdip = nullptr;
  SG_TRY(dupload(c, (void**)&c.d_pot, pot_host, sizeof(double) * c.G));
  SG_TRY(dalloc(c, &c.d_zdip, sizeof(double) * c.G));
  std::vector<double> pts(N);
  for (int i = 0; i < N; ++i) pts[i] = (i + 1) * c.spacing;
  double mid = (pts[0] + pts[N - 1]) / 2.0;
  for (int i = 0; i < N; ++i) pts[i] -= mid;
  double* d_pts = nullptr;
  SG_TRY(dupload(c, (void**)&d_pts, pts.data(), sizeof(double) * N));
  zdip_kernel<<<ceil_div(c.G, 256), 256, 0, c.stream>>>(c.d_zdip, d_pts, N);
  dfree(c, d_pts);
  e = cudaStreamSynchronize(c.stream);
  SG_CHECK(e == cudaSuccess, SINCGPU_ECUDA, "zdip: %s", cudaGetErrorString(e));
  SG_TRY(make_khat(c));
  return SINCGPU_OK;
}

}  // namespace sincgpu
