// Exponential orbital propagation on the device (intopt=3 of the reference).
//
// expospfprop (MCTDH.SRC/expo_driver.f90:482-771, DGPHIV branch):
//   jacvect    = phi0,  jacvectout = blend_s actreduced00(phi0, slot s, no projection)
//                                    (jacinit0, expo_driver.f90:429-467)
//   u          = blend_s actreduced00(phi0, slot s, projected)
//                                    (spf_linear_derivs, derivs.f90:1037-1186)
//   w          = t phi_1(t J) u      (DGPHIV, expokit.f90:3904-4310: Krylov on the
//                                     3-extended Hessenberg, (6,6) Pade, local error
//                                     estimate, step-down by 0.8 on rejection)
//   phi        = spf_orthogit(phi0 + w)   (two Loewdin passes, spfs.f90:120-196)
// with J = jacoperate00 (expo_driver.f90:40-259, jacsymflag=0, no frozen core,
// no constraint, no driving):
//   J x = T - jacvect <jacvect|T> - jacvect <x|jacvectout> - x <jacvect|jacvectout>,
//   T   = blend_s actreduced00(x, slot s, no projection)
// where blend_s uses weights ((t-first)/(last-first), 1 - that) over the two
// mean-field slots when the linear flag is set (effective_cmf_linearflag), else
// slot 0 alone.  The saved Krylov dimension / step-size state of expospfprop
// (expo_driver.f90:498-509, 560-580, 743-767) lives in the context.
//
// Krylov vectors are the orbitals viewed as 2*G*n reals.  Dots and norms are
// split over a fixed grid of 296 CTAs; every consumer sums the 296 partials in
// the same fixed order, so results are deterministic.  Modified Gram-Schmidt
// runs one fused kernel per projection: it applies the previous projection and
// accumulates the partials of the next dot in the same pass.
#include <algorithm>
#include <cmath>
#include "context.hpp"
#include "jacobi_svd.cuh"

namespace sincgpu {

constexpr int kLvBlocks = 2 * 148;
constexpr int kLvThreads = 512;
constexpr int kMaxPadeOrb = 128;  // largest Pade order of pade_expm (Krylov dimension + 3)

struct OrbKryState {
  double beta;    // |p| of the start vector
  double avnorm;  // |J v_{m+1}|
  double hlast;   // last h(j+1,j) (the breakdown value when mbrk != 0)
  int mbrk;       // 0, or the breakdown dimension
  int gfail;      // 1: a grid barrier of lv_arnoldi_orth_kernel gave up
};

__device__ __forceinline__ double lv_block_sum(double v, double* red) {
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

// the same fixed-order total of the kLvBlocks partials in every CTA
__device__ __forceinline__ double lv_total(const double* __restrict__ part, double* red) {
  const double v = threadIdx.x < kLvBlocks ? part[threadIdx.x] : 0.0;
  return lv_block_sum(v, red);
}

// part[b] = sum over CTA b's share of a.b (as reals)
__global__ void __launch_bounds__(kLvThreads) lv_dot_kernel(const double2* __restrict__ a,
                                                            const double2* __restrict__ b, long long nv,
                                                            double* __restrict__ part) {
  __shared__ double red[33];
  double s = 0.0;
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < nv;
       k += (long long)gridDim.x * blockDim.x) {
    const double2 x = a[k], y = b[k];
    s = fma(x.x, y.x, s);
    s = fma(x.y, y.y, s);
  }
  s = lv_block_sum(s, red);
  if (threadIdx.x == 0) part[blockIdx.x] = s;
}

// p += u and the partials of |p|^2
__global__ void __launch_bounds__(kLvThreads) lv_add_norm_kernel(double2* __restrict__ p,
                                                                 const double2* __restrict__ u, long long nv,
                                                                 double* __restrict__ part) {
  __shared__ double red[33];
  double s = 0.0;
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < nv;
       k += (long long)gridDim.x * blockDim.x) {
    double2 x = p[k];
    const double2 y = u[k];
    x.x += y.x;
    x.y += y.y;
    p[k] = x;
    s = fma(x.x, x.x, s);
    s = fma(x.y, x.y, s);
  }
  s = lv_block_sum(s, red);
  if (threadIdx.x == 0) part[blockIdx.x] = s;
}

// start vector: beta = sqrt(total); v = p / beta (p == v allowed)
__global__ void __launch_bounds__(kLvThreads) lv_start_kernel(double2* __restrict__ v, long long nv,
                                                              const double* __restrict__ part,
                                                              OrbKryState* st) {
  __shared__ double red[33];
  const double beta = sqrt(lv_total(part, red));
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    st->beta = beta;
    st->mbrk = 0;
  }
  if (beta == 0.0) return;
  const double inv = 1.0 / beta;
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < nv;
       k += (long long)gridDim.x * blockDim.x) {
    double2 x = v[k];
    v[k] = make_double2(x.x * inv, x.y * inv);
  }
}

// one modified Gram-Schmidt projection: h = <v_i, p> (from part_in);
// p -= h v_i; then the partials of <v_{i+1}, p> (i < j) or |p|^2 (i == j)
__global__ void __launch_bounds__(kLvThreads) lv_mgs_kernel(const double2* __restrict__ V, double2* __restrict__ p,
                                                            long long nv, int i, int j,
                                                            const double* __restrict__ part_in,
                                                            double* __restrict__ part_out, double* __restrict__ Hm,
                                                            int mh) {
  __shared__ double red[33];
  const double h = lv_total(part_in, red);
  if (blockIdx.x == 0 && threadIdx.x == 0) Hm[(long long)j * mh + i] = h;
  const double2* vi = V + (long long)i * nv;
  const double2* vn = i < j ? V + (long long)(i + 1) * nv : nullptr;
  double s = 0.0;
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < nv;
       k += (long long)gridDim.x * blockDim.x) {
    const double2 a = vi[k];
    double2 x = p[k];
    x.x = fma(-h, a.x, x.x);
    x.y = fma(-h, a.y, x.y);
    p[k] = x;
    const double2 b = vn ? vn[k] : x;
    s = fma(b.x, x.x, s);
    s = fma(b.y, x.y, s);
  }
  s = lv_block_sum(s, red);
  if (threadIdx.x == 0) part_out[blockIdx.x] = s;
}

// Grid-wide barrier of a cooperative launch (all CTAs resident): bar[0] counts
// the arrivals of the current generation, bar[1] is the generation.  The last
// CTA to arrive clears the count and advances the generation; the others poll
// the generation at most kGridPolls times.  Returns false when the limit was
// reached, after raising st->gfail (the caller's CTA then leaves the kernel and
// the host reports SINCGPU_ETIMEOUT).
constexpr unsigned kGridPolls = 1u << 22;

__device__ __forceinline__ bool grid_barrier(unsigned* bar, OrbKryState* st, int* ok) {
  __syncthreads();
  if (threadIdx.x == 0) {
    volatile unsigned* vb = bar;
    const unsigned gen = vb[1];
    __threadfence();
    int done = 1;
    if (atomicAdd(&bar[0], 1u) == gridDim.x - 1) {
      atomicExch(&bar[0], 0u);
      __threadfence();
      atomicAdd(&bar[1], 1u);
    } else {
      done = 0;
      for (unsigned it = 0; it < kGridPolls; ++it)
        if (vb[1] != gen) {
          done = 1;
          break;
        }
      if (!done) atomicExch(&st->gfail, 1);
    }
    __threadfence();
    *ok = done;
  }
  __syncthreads();
  return *ok != 0;
}

// lv_total over partials written earlier in the same launch (read through L2)
__device__ __forceinline__ double lv_total_l2(const double* part, double* red) {
  const double v = threadIdx.x < kLvBlocks ? __ldcg(part + threadIdx.x) : 0.0;
  return lv_block_sum(v, red);
}

// The whole orthogonalisation of Arnoldi step j in one cooperative launch:
// lv_dot_kernel (<v_0, p>), the j + 1 lv_mgs_kernel projections and
// lv_arnoldi_norm_kernel, with the same grid, element assignment, partial sums
// and fixed-order totals (so the same bits), p held in registers throughout and
// a grid barrier where the separate launches had a kernel boundary.  p is read
// once and written once; v_i comes from L2 the second time (it was v_{i+1} of
// the projection before).  E elements per thread: nv <= E * kLvBlocks * kLvThreads.
template <int E>
__global__ void __launch_bounds__(kLvThreads, 2) lv_arnoldi_orth_kernel(const double2* __restrict__ V, double2* p,
                                                                         long long nv, int j, double* part0,
                                                                         double* part1, double* __restrict__ Hm,
                                                                         int mh, double break_tol, OrbKryState* st,
                                                                         unsigned* bar) {
  __shared__ double red[33];
  __shared__ int ok;
  const long long stride = (long long)gridDim.x * blockDim.x;
  const long long k0 = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  double2 x[E];
  double s = 0.0;
#pragma unroll
  for (int e = 0; e < E; ++e) {
    const long long k = k0 + e * stride;
    x[e] = make_double2(0.0, 0.0);
    if (k < nv) {
      x[e] = p[k];
      const double2 a = V[k];
      s = fma(a.x, x[e].x, s);
      s = fma(a.y, x[e].y, s);
    }
  }
  s = lv_block_sum(s, red);
  if (threadIdx.x == 0) part0[blockIdx.x] = s;
  if (!grid_barrier(bar, st, &ok)) return;
  for (int i = 0; i <= j; ++i) {
    const double* pin = (i & 1) ? part1 : part0;
    double* pout = (i & 1) ? part0 : part1;
    const double h = lv_total_l2(pin, red);
    if (blockIdx.x == 0 && threadIdx.x == 0) Hm[(long long)j * mh + i] = h;
    const double2* vi = V + (long long)i * nv;
    const double2* vn = i < j ? V + (long long)(i + 1) * nv : nullptr;
    s = 0.0;
#pragma unroll
    for (int e = 0; e < E; ++e) {
      const long long k = k0 + e * stride;
      if (k < nv) {
        const double2 a = vi[k];
        x[e].x = fma(-h, a.x, x[e].x);
        x[e].y = fma(-h, a.y, x[e].y);
        const double2 b = vn ? vn[k] : x[e];
        s = fma(b.x, x[e].x, s);
        s = fma(b.y, x[e].y, s);
      }
    }
    s = lv_block_sum(s, red);
    if (threadIdx.x == 0) pout[blockIdx.x] = s;
    if (!grid_barrier(bar, st, &ok)) return;
  }
  const double h = sqrt(lv_total_l2(((j + 1) & 1) ? part1 : part0, red));
  const bool brk = h <= break_tol;
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    st->hlast = h;
    if (brk) st->mbrk = j + 1;
    else Hm[(long long)j * mh + j + 1] = h;
  }
  const double inv = 1.0 / h;
#pragma unroll
  for (int e = 0; e < E; ++e) {
    const long long k = k0 + e * stride;
    if (k < nv) p[k] = brk ? x[e] : make_double2(x[e].x * inv, x[e].y * inv);
  }
}

constexpr int kOrthE = 5;  // register-resident elements per thread of the one-launch orthogonalisation

// whether all kLvBlocks CTAs of lv_arnoldi_orth_kernel fit on the device at once
// (the cooperative launch needs it); evaluated once per process
static bool orth_fits() {
  static const bool fits = [] {
    int dev = 0, sms = 0, per_sm = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return false;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) return false;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, lv_arnoldi_orth_kernel<kOrthE>, kLvThreads, 0) !=
        cudaSuccess)
      return false;
    return (long long)per_sm * sms >= kLvBlocks;
  }();
  return fits;
}

// h(j+1,j) = |p|; breakdown test; p /= h (expokit.f90 Arnoldi loop)
__global__ void __launch_bounds__(kLvThreads) lv_arnoldi_norm_kernel(double2* __restrict__ p, long long nv, int j,
                                                                     const double* __restrict__ part,
                                                                     double* __restrict__ Hm, int mh,
                                                                     double break_tol, OrbKryState* st) {
  __shared__ double red[33];
  const double h = sqrt(lv_total(part, red));
  const bool brk = h <= break_tol;
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    st->hlast = h;
    if (brk) st->mbrk = j + 1;
    else Hm[(long long)j * mh + j + 1] = h;
  }
  if (brk) return;
  const double inv = 1.0 / h;
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < nv;
       k += (long long)gridDim.x * blockDim.x) {
    double2 x = p[k];
    p[k] = make_double2(x.x * inv, x.y * inv);
  }
}

__global__ void __launch_bounds__(kLvThreads) lv_avnorm_kernel(const double* __restrict__ part, OrbKryState* st) {
  __shared__ double red[33];
  const double a = sqrt(lv_total(part, red));
  if (threadIdx.x == 0) st->avnorm = a;
}

// w += beta * V[0:mx] phih[0:mx]  (DGEMV 'n' with beta_blas = 1)
__global__ void __launch_bounds__(256) lv_update_kernel(const double2* __restrict__ V, long long nv, int mx,
                                                        const double* __restrict__ phih,
                                                        const OrbKryState* __restrict__ st,
                                                        double2* __restrict__ w) {
  __shared__ double c[128];
  const double beta = st->beta;
  for (int i = threadIdx.x; i < mx; i += blockDim.x) c[i] = beta * phih[i];
  __syncthreads();
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < nv;
       k += (long long)gridDim.x * blockDim.x) {
    double2 acc = w[k];
    for (int i = 0; i < mx; ++i) {
      const double2 v = V[(long long)i * nv + k];
      acc.x = fma(c[i], v.x, acc.x);
      acc.y = fma(c[i], v.y, acc.y);
    }
    w[k] = acc;
  }
}

__global__ void lv_add_kernel(double2* __restrict__ a, const double2* __restrict__ b, long long nv) {
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < nv;
       k += (long long)gridDim.x * blockDim.x)
    a[k] = cadd(a[k], b[k]);
}

// S^(-1/2) of the overlap by SVD with singular values below 1e-10 dropped
// (symorthogmat, MCTDH.SRC/utils.f90:947-1023: out = U diag(f(s)) V^H), and
// the orthonormality error max|S - 1| of the overlap on input.
__global__ void __launch_bounds__(32) orthogmat_kernel(const double2* __restrict__ S_in, int n,
                                                       double2* __restrict__ out, double* __restrict__ err) {
  __shared__ double2 A[32 * 32], V[32 * 32];
  __shared__ double sv[32];
  const int k = threadIdx.x;
  double e = 0.0;
  if (k < n)
    for (int j = 0; j < n; ++j) {
      double2 d = S_in[k + n * j];
      if (k == j) d.x -= 1.0;
      e = fmax(e, sqrt(d.x * d.x + d.y * d.y));
    }
  for (int o = 16; o > 0; o >>= 1) e = fmax(e, __shfl_xor_sync(0xffffffffu, e, o));
  if (k == 0 && err) *err = e;
  if (!out) return;
  hestenes_svd_warp(S_in, n, A, V, sv);
  // out(i,j) = sum_m U(i,m) f(s_m) conj(V(j,m)),  U(i,m) = A(i,m) / s_m
  if (k < n)
    for (int j = 0; j < n; ++j) {
      double2 acc = make_double2(0.0, 0.0);
      for (int m = 0; m < n; ++m) {
        const double s = sv[m];
        if (s < 1e-10) continue;
        const double f = 1.0 / sqrt(s) / s;
        const double2 t = cmulc(A[k + 32 * m], V[j + 32 * m]);  // A(i,m) conj(V(j,m))
        acc.x = fma(f, t.x, acc.x);
        acc.y = fma(f, t.y, acc.y);
      }
      out[k + n * j] = acc;
    }
}

namespace {

// device scratch of one orbital propagation
struct OrbWork {
  double2 *V, *jv, *jvo, *u, *w, *T, *tmp, *dpart;
  double2 *D2, *M1, *M2, *ovl, *smh;
  double *part0, *part1, *Hm, *exph, *Efull, *pscratch, *err;
  OrbKryState* st;
  int* ns;
  unsigned* gbar;  // lv_arnoldi_orth_kernel's grid barrier (count, generation)
  bool blendq = false;  // the unprojected blends read the prepared Q and M (blendq_prepare)
};

size_t al256(size_t b) { return (b + 255) / 256 * 256; }

int orb_work(Ctx& c, int m, OrbWork& o) {
  const long long nv = c.G * c.nspf;
  const int n = c.nspf, nn = n * n;
  const int mh = m + 3;
  const size_t vb = sizeof(double2) * (size_t)nv;
  const size_t dpart = sizeof(double2) * (size_t)orbital_dots_scratch(c) * nn;
  const size_t mat = sizeof(double2) * nn;
  size_t need = al256(vb) * ((size_t)m + 2 + 6) + al256(dpart) + 5 * al256(mat) +
                2 * al256(sizeof(double) * kLvBlocks) + al256(sizeof(double) * mh * mh) +
                al256(sizeof(double) * 130) + al256(sizeof(double) * kMaxPadeOrb * kMaxPadeOrb) +
                al256(sizeof(double) * 5 * kMaxPadeOrb * kMaxPadeOrb) + 4 * 256;
  SG_TRY(c.ws_orb.ensure(need));
  char* p = (char*)c.ws_orb.ptr;
  auto take = [&](size_t b) {
    char* r = p;
    p += al256(b);
    return r;
  };
  o.V = (double2*)take(vb * (m + 2));
  o.jv = (double2*)take(vb);
  o.jvo = (double2*)take(vb);
  o.u = (double2*)take(vb);
  o.w = (double2*)take(vb);
  o.T = (double2*)take(vb);
  o.tmp = (double2*)take(vb);
  o.dpart = (double2*)take(dpart);
  o.D2 = (double2*)take(mat);
  o.M1 = (double2*)take(mat);
  o.M2 = (double2*)take(mat);
  o.ovl = (double2*)take(mat);
  o.smh = (double2*)take(mat);
  o.part0 = (double*)take(sizeof(double) * kLvBlocks);
  o.part1 = (double*)take(sizeof(double) * kLvBlocks);
  o.Hm = (double*)take(sizeof(double) * mh * mh);
  o.exph = (double*)take(sizeof(double) * 130);
  o.Efull = (double*)take(sizeof(double) * kMaxPadeOrb * kMaxPadeOrb);
  o.pscratch = (double*)take(sizeof(double) * 5 * kMaxPadeOrb * kMaxPadeOrb);
  o.err = (double*)take(sizeof(double));
  o.st = (OrbKryState*)take(sizeof(OrbKryState));
  o.ns = (int*)take(sizeof(int));
  o.gbar = (unsigned*)take(2 * sizeof(unsigned));
  return SINCGPU_OK;
}

// page-locked host copy of OrbKryState and its event, made once per context (the
// block comes from the process's recycled page-locked blocks)
int orb_state_host(Ctx& c, OrbKryState** h) {
  if (!c.orb_state_h) {
    SG_TRY(pinned_get(sizeof(OrbKryState), &c.orb_state_h));
    c.orb_state_bytes = sizeof(OrbKryState);
    SG_CUDA(cudaEventCreateWithFlags(&c.ev_orb_state, cudaEventDisableTiming));
  }
  *h = static_cast<OrbKryState*>(c.orb_state_h);
  return SINCGPU_OK;
}

// blended unprojected (proj == nullptr) or projected actreduced00 over the slots
int blend_actreduced(Ctx& c, const double2* x, const double2* proj, const MeanFieldSlot* slots,
                     const double* facs, int nslot, double2 timefac, double ez, double2* tmp, double2* out,
                     bool blendq = false) {
  const long long len = c.G * c.nspf;
  if (blendq && nslot == 2 && !proj) return actreduced_blendq(c, x, timefac, ez, out);
  if (nslot == 2 && !proj && actreduced_blend2_fits(c.nspf)) {
    const double2* den[2] = {slots[0].denmat, slots[1].denmat};
    const double2* inv[2] = {slots[0].invdenmat, slots[1].invdenmat};
    const double2* rp[2] = {slots[0].reducedpot, slots[1].reducedpot};
    return actreduced_blend2(c, x, den, inv, rp, facs, timefac, ez, out);
  }
  if (nslot > 1) SG_TRY(actreduced_ke(c, x, ez));  // KE(x) once for all slots
  for (int s = 0; s < nslot; ++s) {
    if (nslot > 1) {
      SG_TRY(actreduced_mix_ke(c, slots[s].denmat));
      SG_TRY(actreduced_post(c, x, proj, slots[s].invdenmat, slots[s].reducedpot, timefac, 1, proj ? 1 : 0, tmp));
    } else {
      SG_TRY(actreduced(c, x, proj, slots[s].denmat, slots[s].invdenmat, slots[s].reducedpot, timefac, 1,
                        proj ? 1 : 0, ez, tmp));
    }
    SG_TRY(axpby(c, out, tmp, 1.0, facs[s], len, s == 0));
  }
  return SINCGPU_OK;
}

int jacoperate(Ctx& c, OrbWork& o, const double2* x, const MeanFieldSlot* slots, const double* facs, int nslot,
               double2 timefac, double ez, double2* y) {
  SG_TRY(blend_actreduced(c, x, nullptr, slots, facs, nslot, timefac, ez, o.tmp, o.T, o.blendq));
  SG_TRY(orbital_dots(c, o.jv, o.T, o.M1, o.dpart));   // <jacvect|T>
  SG_TRY(orbital_dots(c, x, o.jvo, o.M2, o.dpart));    // <x|jacvectout>
  return jac_combine(c, o.T, o.jv, o.M1, o.M2, x, o.D2, y);
}

double fortran_nint(double x) { return x >= 0 ? std::floor(x + 0.5) : -std::floor(-x + 0.5); }

}  // namespace

int spf_orthogit(Ctx& c, double2* phi, double* error) {
  const int n = c.nspf;
  SG_CHECK(n <= 32, SINCGPU_ERANGE, "at most 32 orbitals");
  OrbWork o;
  SG_TRY(orb_work(c, 1, o));
  const long long nv = c.G * n;
  for (int ii = 0; ii < 3; ++ii) {
    SG_TRY(orbital_dots(c, phi, phi, o.ovl, o.dpart));
    orthogmat_kernel<<<1, 32, 0, c.stream>>>(o.ovl, n, ii < 2 ? o.smh : nullptr, o.err);
    SG_LAUNCHED();
    if (ii < 2) {
      SG_TRY(orbital_mix(c, phi, o.smh, o.tmp));
      SG_CUDA(cudaMemcpyAsync(phi, o.tmp, sizeof(double2) * nv, cudaMemcpyDeviceToDevice, c.stream));
    }
  }
  if (error) {
    SG_CUDA(cudaMemcpyAsync(error, o.err, sizeof(double), cudaMemcpyDeviceToHost, c.stream));
    SG_CUDA(cudaStreamSynchronize(c.stream));
  }
  return SINCGPU_OK;
}

int expospfprop(Ctx& c, double2* phi, const MeanFieldSlot* slots, double tin, double tout, double firsttime,
                double lasttime, bool linear, double2 timefac, double ez, double expotol, int* numiters) {
  OrbPropState& S = c.orb;
  const int n = c.nspf;
  SG_CHECK(n <= 32, SINCGPU_ERANGE, "at most 32 orbitals");
  const long long nv = c.G * n;
  const long long idim = 2 * nv;
  const int maxexpodim = (int)std::min<long long>(S.maxexpodim, idim - 1);
  const double tdiff = tout - tin, midtime = 0.5 * (tin + tout);
  double facs[2] = {1.0, 0.0};
  const int nslot = linear ? 2 : 1;
  if (linear) {
    SG_CHECK(lasttime != firsttime, SINCGPU_EINVAL, "linear blend needs lasttime != firsttime");
    facs[0] = (midtime - firsttime) / (lasttime - firsttime);
    facs[1] = 1.0 - facs[0];
  }
  // saved-variable bookkeeping before the Krylov call (expo_driver.f90:560-580)
  ++S.icalled;
  if (S.icalled == 1) {
    S.tempstepsize = S.first_stepsize;
    S.thisexpodim = std::min(S.expodim, maxexpodim);
  }
  if (S.icalled % 12 == 0) S.exposet = 0;
  if (S.thisexpodim < maxexpodim) S.tempstepsize *= 4;
  else S.tempstepsize *= S.expostepfac;
  const int m = S.thisexpodim;
  SG_CHECK(m >= 1 && m + 3 <= kMaxPadeOrb, SINCGPU_ERANGE, "Krylov dimension %d outside [1,%d]", m,
           kMaxPadeOrb - 3);
  OrbWork o;
  SG_TRY(orb_work(c, m, o));
  const int mh = m + 3;
  ProfScope ps(c, ST_OTHER);

  // jacinit: jacvect = phi, jacvectout = blend (gridtime, 1-gridtime) of the
  // unprojected actreduced at midtime; D2 = <jacvect|jacvectout>
  SG_CUDA(cudaMemcpyAsync(o.jv, phi, sizeof(double2) * nv, cudaMemcpyDeviceToDevice, c.stream));
  // with two slots the blend factors and mean fields are fixed for this call: fold
  // the slots' reduced potentials and density matrices once
  if (nslot == 2 && c.orb_blendq && actreduced_blendq_fits(n)) {
    const double2* den[2] = {slots[0].denmat, slots[1].denmat};
    const double2* inv[2] = {slots[0].invdenmat, slots[1].invdenmat};
    const double2* rp[2] = {slots[0].reducedpot, slots[1].reducedpot};
    SG_TRY(blendq_prepare(c, den, inv, rp, facs));
    o.blendq = true;
  }
  SG_TRY(blend_actreduced(c, o.jv, nullptr, slots, facs, nslot, timefac, ez, o.tmp, o.jvo, o.blendq));
  SG_TRY(orbital_dots(c, o.jv, o.jvo, o.D2, o.dpart));
  // u = spf_linear_derivs(midtime, phi)
  SG_TRY(blend_actreduced(c, o.jv, o.jv, slots, facs, nslot, timefac, ez, o.tmp, o.u));

  // DGPHIV0 with v = 0: w = tdiff * phi_1(tdiff J) u
  const double delta = 1.2, gamma = 0.8, break_tol = 1.0e-7;
  double tol = expotol;
  const double eps = std::fabs((4.0 / 3.0 - 1.0) * 3.0 - 1.0);
  if (tol <= eps) tol = std::sqrt(eps);
  const double sgn = tdiff >= 0 ? 1.0 : -1.0, t_out = std::fabs(tdiff), sqr1 = std::sqrt(0.1);
  double t_now = 0.0, t_step = 0.0, t_last = 0.0, t_new = 0.0, xm = 0.0;
  int nstep = 0, nmult = 0;
  bool w_zero = true;
  SG_CUDA(cudaMemsetAsync(o.w, 0, sizeof(double2) * nv, c.stream));
  const int lvg = kLvBlocks;
  const bool orth_fused = c.orth_fused && nv <= (long long)kOrthE * lvg * kLvThreads && orth_fits();
  SG_CUDA(cudaMemsetAsync(o.gbar, 0, 2 * sizeof(unsigned), c.stream));
  SG_CUDA(cudaMemsetAsync(o.st, 0, sizeof(OrbKryState), c.stream));
  const int ub = std::min<long long>(ceil_div(nv, 256), 148 * 8);
  OrbKryState hst{};
  while (t_now < t_out) {
    // p = J w + u into V[0]; J 0 = 0 exactly, so the product is skipped while w is zero
    ++nmult;
    double2* V0 = o.V;
    if (w_zero) {
      SG_CUDA(cudaMemsetAsync(V0, 0, sizeof(double2) * nv, c.stream));
    } else {
      SG_TRY(jacoperate(c, o, o.w, slots, facs, nslot, timefac, ez, V0));
    }
    lv_add_norm_kernel<<<lvg, kLvThreads, 0, c.stream>>>(V0, o.u, nv, o.part0);
    SG_LAUNCHED();
    lv_start_kernel<<<lvg, kLvThreads, 0, c.stream>>>(V0, nv, o.part0, o.st);
    SG_LAUNCHED();
    SG_CUDA(cudaMemcpyAsync(&hst, o.st, sizeof(OrbKryState), cudaMemcpyDeviceToHost, c.stream));
    SG_CUDA(cudaStreamSynchronize(c.stream));
    if (hst.beta == 0.0) break;
    SG_CUDA(cudaMemsetAsync(o.Hm, 0, sizeof(double) * mh * mh, c.stream));
    if (nstep == 0) {
      t_new = S.tempstepsize;
      xm = 1.0 / m;
    }
    ++nstep;
    t_last = t_step;
    t_step = std::min(t_out - t_now, t_new);
    int k1 = 3, mbrkdwn = m;
    // The product J v_{j+1} is issued before step j's breakdown test is read back,
    // so the device does not idle during the host round trip; after a breakdown it
    // is dropped (it writes only v_{j+2} and the product's scratch, which the rest
    // of the step does not read) and not counted.
    OrbKryState* hst_pin = nullptr;
    SG_TRY(orb_state_host(c, &hst_pin));
    bool have_next = false;  // p = V[j + 1] already holds J V[j]
    for (int j = 0; j < m; ++j) {
      ++nmult;
      double2* p = o.V + (size_t)(j + 1) * nv;
      if (!have_next) SG_TRY(jacoperate(c, o, o.V + (size_t)j * nv, slots, facs, nslot, timefac, ez, p));
      if (orth_fused) {
        const double2* Vc = o.V;
        double *P0 = o.part0, *P1 = o.part1, *H = o.Hm;
        OrbKryState* S = o.st;
        unsigned* B = o.gbar;
        int jj = j, mhh = mh;
        long long nvv = nv;
        double bt = break_tol;
        void* args[] = {(void*)&Vc, (void*)&p,   (void*)&nvv, (void*)&jj, (void*)&P0, (void*)&P1,
                        (void*)&H,  (void*)&mhh, (void*)&bt,  (void*)&S,  (void*)&B};
        SG_CUDA(cudaLaunchCooperativeKernel((const void*)lv_arnoldi_orth_kernel<kOrthE>, dim3(lvg),
                                            dim3(kLvThreads), args, 0, c.stream));
        count_launch();
      } else {
        lv_dot_kernel<<<lvg, kLvThreads, 0, c.stream>>>(o.V, p, nv, o.part0);
        SG_LAUNCHED();
        double* pin = o.part0;
        double* pout = o.part1;
        for (int i = 0; i <= j; ++i) {
          lv_mgs_kernel<<<lvg, kLvThreads, 0, c.stream>>>(o.V, p, nv, i, j, pin, pout, o.Hm, mh);
          SG_LAUNCHED();
          std::swap(pin, pout);
        }
        lv_arnoldi_norm_kernel<<<lvg, kLvThreads, 0, c.stream>>>(p, nv, j, pin, o.Hm, mh, break_tol, o.st);
        SG_LAUNCHED();
      }
      SG_CUDA(cudaMemcpyAsync(hst_pin, o.st, sizeof(OrbKryState), cudaMemcpyDeviceToHost, c.stream));
      SG_CUDA(cudaEventRecord(c.ev_orb_state, c.stream));
      SG_TRY(jacoperate(c, o, p, slots, facs, nslot, timefac, ez, o.V + (size_t)(j + 2) * nv));
      have_next = true;
      SG_CUDA(cudaEventSynchronize(c.ev_orb_state));
      hst = *hst_pin;
      SG_CHECK(!hst.gfail, SINCGPU_ETIMEOUT, "grid barrier of the Arnoldi orthogonalisation timed out");
      if (hst.mbrk) {  // happy breakdown
        k1 = 0;
        mbrkdwn = hst.mbrk;
        t_step = t_out - t_now;
        break;
      }
    }
    if (k1 != 0) {
      ++nmult;
      double2* p = o.V + (size_t)(m + 1) * nv;
      if (!have_next) SG_TRY(jacoperate(c, o, o.V + (size_t)m * nv, slots, facs, nslot, timefac, ez, p));
      lv_dot_kernel<<<lvg, kLvThreads, 0, c.stream>>>(p, p, nv, o.part0);
      SG_LAUNCHED();
      lv_avnorm_kernel<<<1, kLvThreads, 0, c.stream>>>(o.part0, o.st);
      SG_LAUNCHED();
      SG_CUDA(cudaMemcpyAsync(&hst, o.st, sizeof(OrbKryState), cudaMemcpyDeviceToHost, c.stream));
      SG_CUDA(cudaStreamSynchronize(c.stream));
    }
    const double hj1j = hst.hlast;
    {  // the 3-extended scheme (expokit.f90, label 300)
      const double one = 1.0, zero = 0.0;
      SG_CUDA(cudaMemcpyAsync(o.Hm + (size_t)mh * mbrkdwn, &one, sizeof(double), cudaMemcpyHostToDevice,
                              c.stream));
      SG_CUDA(cudaMemcpyAsync(o.Hm + (size_t)(m - 1) * mh + m, &zero, sizeof(double), cudaMemcpyHostToDevice,
                              c.stream));
      for (int i = 1; i < k1; ++i)
        SG_CUDA(cudaMemcpyAsync(o.Hm + (size_t)(m + i) * mh + m + i - 1, &one, sizeof(double),
                                cudaMemcpyHostToDevice, c.stream));
    }
    double err_loc = tol;
    while (true) {
      const int mx = mbrkdwn + std::max(1, k1);
      SG_TRY(pade_expm(c, o.Hm, mh, mx, sgn * t_step, mbrkdwn, o.exph, o.Efull, o.pscratch, o.ns));
      if (k1 == 0) {
        err_loc = tol;
        break;
      }
      // phih(m) = hj1j E(m-1, m+1), phih(m+1) = hj1j E(m-1, m+2)
      double e2[2];
      SG_CUDA(cudaMemcpyAsync(&e2[0], o.Efull + (size_t)(m + 1) * mx + (m - 1), sizeof(double),
                              cudaMemcpyDeviceToHost, c.stream));
      SG_CUDA(cudaMemcpyAsync(&e2[1], o.Efull + (size_t)(m + 2) * mx + (m - 1), sizeof(double),
                              cudaMemcpyDeviceToHost, c.stream));
      SG_CUDA(cudaStreamSynchronize(c.stream));
      const double ph_m = hj1j * e2[0], ph_m1 = hj1j * e2[1];
      const double p1 = std::fabs(ph_m) * hst.beta;
      const double p2 = std::fabs(ph_m1) * hst.beta * hst.avnorm;
      if (p1 > 10.0 * p2) {
        err_loc = p2;
        xm = 1.0 / (m + 1);
      } else {
        err_loc = p1;
        xm = 1.0 / m;
      }
      if (err_loc > delta * t_step * tol) {  // reject (mxreject = 0): step down and retry
        t_step = gamma * t_step;
        continue;
      }
      SG_CUDA(cudaMemcpyAsync(o.exph + m, &ph_m, sizeof(double), cudaMemcpyHostToDevice, c.stream));
      break;
    }
    const int mxu = mbrkdwn + std::max(0, k1 - 2);
    lv_update_kernel<<<ub, 256, 0, c.stream>>>(o.V, nv, mxu, o.exph, o.st, o.w);
    SG_LAUNCHED();
    w_zero = false;
    t_new = gamma * t_step * std::pow(t_step * tol / err_loc, xm);
    const double q = std::pow(10.0, fortran_nint(std::log10(t_new) - sqr1) - 1);
    t_new = std::trunc(t_new / q + 0.55) * q;
    if (t_new < t_step) t_new = t_step;
    t_now += t_step;
    if (nstep >= 1000) break;
  }
  S.tempstepsize = nstep == 1 ? t_step : t_last;
  if (nstep > 1) {
    S.thisexpodim = std::min(maxexpodim, std::max(S.thisexpodim + 5, (int)std::ceil(S.thisexpodim * 1.2)));
    S.exposet = 1;
  }
  // phi = orthonormalised (phi0 + w)
  lv_add_kernel<<<ub, 256, 0, c.stream>>>(phi, o.w, nv);
  SG_LAUNCHED();
  SG_TRY(spf_orthogit(c, phi, nullptr));
  if (S.exposet == 0) S.thisexpodim = std::max(5, (int)std::floor(S.thisexpodim * 0.95));
  if (numiters) *numiters = nmult;
  SG_CUDA(cudaStreamSynchronize(c.stream));
  return SINCGPU_OK;
}

}  // namespace sincgpu
