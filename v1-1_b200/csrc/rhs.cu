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
#include <algorithm>
#include "context.hpp"

namespace sincgpu {

// out(x,i) = sum_j in(x,j) mat(j,i)   (column-major n x n complex mat)
template <int NMAX>
__global__ void __launch_bounds__(256) mix_kernel(const double2* __restrict__ in,
                                                  const double2* __restrict__ mat, int n,
                                                  long long G, double2* __restrict__ out) {
  __shared__ double2 sm[NMAX * NMAX];
  for (int i = threadIdx.x; i < n * n; i += blockDim.x) sm[i] = mat[i];
  __syncthreads();
  long long x = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (x >= G) return;
  double2 v[NMAX];
#pragma unroll
  for (int j = 0; j < NMAX; ++j)
    if (j < n) v[j] = in[(long long)j * G + x];
  for (int i = 0; i < n; ++i) {
    double2 acc = make_double2(0.0, 0.0);
#pragma unroll
    for (int j = 0; j < NMAX; ++j)
      if (j < n) {
        double2 m = sm[j + n * i];
        acc.x = fma(v[j].x, m.x, fma(-v[j].y, m.y, acc.x));
        acc.y = fma(v[j].x, m.y, fma(v[j].y, m.x, acc.y));
      }
    out[(long long)i * G + x] = acc;
  }
}

// s_i = acc(x,i) + sum_k V(x,k,i) phi_k(x) over i in [i0, i0+ni); then, when
// `dentime`, t_i = timefac * sum_j s_j inv(j,i) (all n orbitals present).
template <int NMAX>
__global__ void __launch_bounds__(128) redpot_kernel(const double2* __restrict__ phi,
                                                     const double2* __restrict__ V,
                                                     const double2* __restrict__ acc_in,
                                                     const double2* __restrict__ inv,
                                                     double2 timefac, int n, int i0, int ni,
                                                     int dentime, long long G,
                                                     double2* __restrict__ out) {
  __shared__ double2 sinv[NMAX * NMAX];
  if (dentime)
    for (int i = threadIdx.x; i < n * n; i += blockDim.x) sinv[i] = inv[i];
  __syncthreads();
  long long x = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (x >= G) return;
  double2 ph[NMAX];
#pragma unroll
  for (int k = 0; k < NMAX; ++k)
    if (k < n) ph[k] = phi[(long long)k * G + x];
  double2 s[NMAX];
#pragma unroll
  for (int ii = 0; ii < NMAX; ++ii) {
    if (ii < ni) {
      const int i = i0 + ii;
      double2 a = acc_in ? acc_in[(long long)ii * G + x] : make_double2(0.0, 0.0);
      const double2* Vi = V + (long long)n * ii * G + x;  // V(x,k,i): column k + n*ii
#pragma unroll
      for (int k = 0; k < NMAX; ++k)
        if (k < n) {
          double2 v = Vi[(long long)k * G];
          a.x = fma(v.x, ph[k].x, fma(-v.y, ph[k].y, a.x));
          a.y = fma(v.x, ph[k].y, fma(v.y, ph[k].x, a.y));
        }
      s[ii] = a;
      (void)i;
    }
  }
  if (!dentime) {
    for (int ii = 0; ii < ni; ++ii) out[(long long)ii * G + x] = s[ii];
    return;
  }
  for (int i = 0; i < n; ++i) {
    double2 a = make_double2(0.0, 0.0);
#pragma unroll
    for (int j = 0; j < NMAX; ++j)
      if (j < n) {
        double2 m = sinv[j + n * i];
        a.x = fma(s[j].x, m.x, fma(-s[j].y, m.y, a.x));
        a.y = fma(s[j].x, m.y, fma(s[j].y, m.x, a.y));
      }
    out[(long long)i * G + x] = cmul(timefac, a);
  }
}

// partial[blk][j + n*i] = sum_{x in blk} conj(P_j(x)) T_i(x)
constexpr int DX = 32;
__global__ void __launch_bounds__(256) dots_kernel(const double2* __restrict__ Pm,
                                                   const double2* __restrict__ Tm, int n,
                                                   long long G, long long xper,
                                                   double2* __restrict__ partial) {
  __shared__ double2 sp[32][DX];
  __shared__ double2 st[32][DX];
  const long long xb = blockIdx.x * xper, xe = min(G, xb + xper);
  const int nn = n * n;
  double2 acc[4];
#pragma unroll
  for (int r = 0; r < 4; ++r) acc[r] = make_double2(0.0, 0.0);
  for (long long x0 = xb; x0 < xe; x0 += DX) {
    __syncthreads();
    for (int i = threadIdx.x; i < n * DX; i += blockDim.x) {
      int o = i / DX, k = i % DX;
      long long x = x0 + k;
      bool ok = x < xe;
      sp[o][k] = ok ? Pm[(long long)o * G + x] : make_double2(0.0, 0.0);
      st[o][k] = ok ? Tm[(long long)o * G + x] : make_double2(0.0, 0.0);
    }
    __syncthreads();
#pragma unroll
    for (int r = 0; r < 4; ++r) {
      int e = threadIdx.x + 256 * r;
      if (e < nn) {
        int j = e % n, i = e / n;
        double2 a = acc[r];
        for (int k = 0; k < DX; ++k) {
          double2 p = sp[j][k], t = st[i][k];
          a.x = fma(p.x, t.x, fma(p.y, t.y, a.x));
          a.y = fma(p.x, t.y, fma(-p.y, t.x, a.y));
        }
        acc[r] = a;
      }
    }
  }
#pragma unroll
  for (int r = 0; r < 4; ++r) {
    int e = threadIdx.x + 256 * r;
    if (e < nn) partial[(long long)blockIdx.x * nn + e] = acc[r];
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
template <int NMAX>
__global__ void __launch_bounds__(256) project_kernel(const double2* __restrict__ Tm,
                                                      const double2* __restrict__ Pm,
                                                      const double2* __restrict__ D, int n,
                                                      long long G, double2* __restrict__ out) {
  __shared__ double2 sd[NMAX * NMAX];
  for (int i = threadIdx.x; i < n * n; i += blockDim.x) sd[i] = D[i];
  __syncthreads();
  long long x = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (x >= G) return;
  double2 p[NMAX];
#pragma unroll
  for (int j = 0; j < NMAX; ++j)
    if (j < n) p[j] = Pm[(long long)j * G + x];
  for (int i = 0; i < n; ++i) {
    double2 a = make_double2(0.0, 0.0);
#pragma unroll
    for (int j = 0; j < NMAX; ++j)
      if (j < n) {
        double2 d = sd[j + n * i];
        a.x = fma(p[j].x, d.x, fma(-p[j].y, d.y, a.x));
        a.y = fma(p[j].x, d.y, fma(p[j].y, d.x, a.y));
      }
    double2 t = Tm[(long long)i * G + x];
    out[(long long)i * G + x] = csub(t, a);
  }
}

#define SG_DISPATCH_N(n, KERNEL, ...)                                     \
  do {                                                                    \
    if ((n) <= 8)                                                         \
      KERNEL<8> __VA_ARGS__;                                              \
    else if ((n) <= 16)                                                   \
      KERNEL<16> __VA_ARGS__;                                             \
    else                                                                  \
      KERNEL<32> __VA_ARGS__;                                             \
  } while (0)

// out(x,i) = T(x,i) - sum_j P_j(x) (M1(j,i) + M2(j,i)) - sum_j X_j(x) D2(j,i)
// (the projector and projector-derivative terms of the orbital Jacobian)
template <int NMAX>
__global__ void __launch_bounds__(256) jac_combine_kernel(const double2* __restrict__ Tm,
                                                          const double2* __restrict__ Pm,
                                                          const double2* __restrict__ M1,
                                                          const double2* __restrict__ M2,
                                                          const double2* __restrict__ Xm,
                                                          const double2* __restrict__ D2, int n,
                                                          long long G, double2* __restrict__ out) {
  __shared__ double2 sm[NMAX * NMAX], sd[NMAX * NMAX];
  for (int i = threadIdx.x; i < n * n; i += blockDim.x) {
    sm[i] = cadd(M1[i], M2[i]);
    sd[i] = D2[i];
  }
  __syncthreads();
  long long x = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (x >= G) return;
  double2 p[NMAX], q[NMAX];
#pragma unroll
  for (int j = 0; j < NMAX; ++j)
    if (j < n) {
      p[j] = Pm[(long long)j * G + x];
      q[j] = Xm[(long long)j * G + x];
    }
  for (int i = 0; i < n; ++i) {
    double2 a = make_double2(0.0, 0.0);
#pragma unroll
    for (int j = 0; j < NMAX; ++j)
      if (j < n) {
        const double2 m = sm[j + n * i], d = sd[j + n * i];
        a.x = fma(p[j].x, m.x, fma(-p[j].y, m.y, a.x));
        a.y = fma(p[j].x, m.y, fma(p[j].y, m.x, a.y));
        a.x = fma(q[j].x, d.x, fma(-q[j].y, d.y, a.x));
        a.y = fma(q[j].x, d.y, fma(q[j].y, d.x, a.y));
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

int orbital_dots_scratch(const Ctx& c) {
  const int nblk_dots = 4 * 148;
  const long long xper = ((c.G + nblk_dots - 1) / nblk_dots + DX - 1) / DX * DX;
  return ceil_div(c.G, xper);
}

int orbital_dots(Ctx& c, const double2* P, const double2* T, double2* D, double2* part) {
  const int n = c.nspf;
  const long long G = c.G;
  const int nblk_dots = 4 * 148;
  const long long xper = ((G + nblk_dots - 1) / nblk_dots + DX - 1) / DX * DX;
  const int nb = ceil_div(G, xper);
  dots_kernel<<<nb, 256, 0, c.stream>>>(P, T, n, G, xper, part);
  SG_LAUNCHED();
  dots_reduce_kernel<<<n * n, 128, 0, c.stream>>>(part, nb, n * n, D);
  SG_LAUNCHED();
  return SINCGPU_OK;
}

int orbital_mix(Ctx& c, const double2* in, const double2* mat, double2* out) {
  const int n = c.nspf;
  SG_CHECK(n <= 32, SINCGPU_ERANGE, "at most 32 orbitals");
  SG_DISPATCH_N(n, mix_kernel, <<<ceil_div(c.G, 256), 256, 0, c.stream>>>(in, mat, n, c.G, out));
  SG_LAUNCHED();
  return SINCGPU_OK;
}

int jac_combine(Ctx& c, const double2* T, const double2* P, const double2* M1, const double2* M2,
                const double2* X, const double2* D2, double2* out) {
  const int n = c.nspf;
  SG_CHECK(n <= 32, SINCGPU_ERANGE, "at most 32 orbitals");
  SG_DISPATCH_N(n, jac_combine_kernel, <<<ceil_div(c.G, 256), 256, 0, c.stream>>>(T, P, M1, M2, X, D2, n,
                                                                                  c.G, out));
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
  SG_CHECK(n <= 32, SINCGPU_ERANGE, "at most 32 orbitals");
  const int blocks = ceil_div(c.G, 128);
  ProfScope ps(c, ST_RHS_REDPOT);
  SG_DISPATCH_N(n, redpot_kernel, <<<blocks, 128, 0, c.stream>>>(phi, redpot, nullptr, nullptr,
                                                               make_double2(1, 0), n, i0, ni, 0, c.G,
                                                               out));
  SG_LAUNCHED();
  return SINCGPU_OK;
}

int mult_reducedpot(Ctx& c, const double2* phi, const double2* redpot, double2* out) {
  return mult_reducedpot_range(c, phi, redpot, 0, c.nspf, out);
}

int actreduced(Ctx& c, const double2* phi, const double2* proj, const double2* denmat,
               const double2* invdenmat, const double2* redpot, double2 timefac, int dentimeflag,
               int projflag, double zfield, double2* out) {
  const int n = c.nspf;
  SG_CHECK(n <= 32, SINCGPU_ERANGE, "at most 32 orbitals");
  const long long G = c.G;
  const int nblk_dots = 4 * 148;
  const long long xper = ((G + nblk_dots - 1) / nblk_dots + DX - 1) / DX * DX;
  const int nb = ceil_div(G, xper);
  const size_t need = sizeof(double2) * (3 * (size_t)n * G + (size_t)nb * n * n + (size_t)n * n);
  SG_TRY(c.ws_rhs.ensure(need));
  double2* Y = (double2*)c.ws_rhs.ptr;
  double2* S = Y + (size_t)n * G;
  double2* T = S + (size_t)n * G;
  double2* part = T + (size_t)n * G;
  double2* D = part + (size_t)nb * n * n;
  const int b256 = ceil_div(G, 256), b128 = ceil_div(G, 128);
  {
    ProfScope ps(c, ST_RHS_MIX);
    SG_DISPATCH_N(n, mix_kernel, <<<b256, 256, 0, c.stream>>>(phi, denmat, n, G, Y));
    SG_LAUNCHED();
  }
  SG_TRY(mult_ke(c, Y, S, n, true, zfield));
  double2* dst = projflag == 1 ? T : out;
  {
    ProfScope ps(c, ST_RHS_REDPOT);
    SG_DISPATCH_N(n, redpot_kernel, <<<b128, 128, 0, c.stream>>>(phi, redpot, S, invdenmat, timefac, n, 0,
                                                               n, dentimeflag ? 1 : 0, G, dst));
    SG_LAUNCHED();
  }
  if (projflag == 1) {
    ProfScope ps(c, ST_RHS_PROJ);
    dots_kernel<<<nb, 256, 0, c.stream>>>(proj, T, n, G, xper, part);
    SG_LAUNCHED();
    dots_reduce_kernel<<<n * n, 128, 0, c.stream>>>(part, nb, n * n, D);
    SG_LAUNCHED();
    SG_DISPATCH_N(n, project_kernel, <<<b256, 256, 0, c.stream>>>(T, proj, D, n, G, out));
    SG_LAUNCHED();
  }
  return SINCGPU_OK;
}

}  // namespace sincgpu
