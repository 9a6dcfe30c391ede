// Constant-mean-field (CMF) propagation step on the device.
//
// cmf_prop_wfn (MCTDH.SRC/prop.f90:230-574) with the reference's defaults
// prepropflag=1, step_flag=2, postpropflag=2, improvedrelaxflag=0, for the sinc
// project (numr=1, mcscfnum=1, no frozen core, constraints or driving term):
//   slot 1 <- slot 0 (orbitals, A-vector, denmat, invdenmat, reducedpot, 2-RDM,
//                     assembled CI matrices)
//   pre-prop : A(tout) = exp(-i dt H0) A(tin); get_allden; get_reducedpot
//   2 x      : orbitals tin -> tout (expospfprop, mean fields blended between the
//              slots) and spf_orthogit (propspfs0, prop.f90:160-228);
//              A(tout) = exp(-i dt (H1+H0)/2) A(tin) (cmf_prop_avector0 with
//              linearflag=1, prop.f90:633-776); get_allden, all_matel,
//              get_reducedpot (get_stuff0, proputils.f90:264-300)
//   post-prop: A-vector again (postpropflag=2); get_allden; get_reducedpot
// then the spin projection of A and the energy <A|P H0 A>/<A|A>
// (prop_loop, prop.f90:926-955).  Each A-vector propagation is expoavecprop
// (expo_driver.f90:827-1055: DGEXPVxxx2 with t = 1 on timefac dt H, its saved
// Krylov order and step guess) followed by basis_project (myconfigprop,
// configstuff.f90:235-265).  The Krylov runs on the configuration basis; for a
// spin-projected start vector and the spin-free Hamiltonian its Krylov space is
// that of the reference's spin-adapted basis.
//
// Length-gauge pulses along z (MCTDH.SRC/pulse.f90 tdpotlen0 with pulsetypes
// 1-5) enter the orbital equation and the CI Hamiltonian at each sub-step
// midpoint.
#include <algorithm>
#include <cmath>
#include <vector>
#include "context.hpp"
#include "../../include/sincgpu.h"

namespace sincgpu {

double pulse_ez(const std::vector<PulseParams>& pulses, double t) {
  const double pi = 3.14159265358979323846;
  double e = 0.0;
  for (const PulseParams& p : pulses) {
    const double fac = std::cos(p.theta);
    if (fac == 0.0) continue;
    const double w = p.omega, w2 = p.omega2, tau = t - p.start;
    double v = 0.0;
    switch (p.type) {
      case 1:  // simplepulselen
        if (t >= p.start && tau <= pi / w)
          v = p.strength * w *
              (std::sin(tau * w) * std::cos(tau * w + p.phaseshift) +
               std::sin(tau * w + p.phaseshift) * std::cos(tau * w));
        break;
      case 2:  // pulselen: E = -dA/dt of A = strength sin^2(w tau) sin((tau - pi/2w) w2 + phase)
        if (t >= p.start && tau <= pi / w) {
          const double arg = (tau - pi / w / 2) * w2 + p.phaseshift;
          v = p.strength * (2 * w * std::sin(tau * w) * std::cos(tau * w) * std::sin(arg) +
                            std::sin(tau * w) * std::sin(tau * w) * w2 * std::cos(arg));
        }
        break;
      case 3: {  // longpulselen
        if (t >= p.start && tau <= pi / w) {
          const double k = 2 * p.longstep + 1, edge = pi / 2.0 / w / k;
          double f, f2;
          if (tau <= edge || tau >= pi / w - edge) {
            f = 2 * w * k * std::sin(tau * w * k) * std::cos(tau * w * k);
            f2 = std::sin(tau * w * k) * std::sin(tau * w * k);
          } else {
            f = 0.0;
            f2 = 1.0;
          }
          v = p.strength * (f * std::sin(tau * w2 + p.phaseshift) + f2 * w2 * std::cos(tau * w2 + p.phaseshift));
        }
        break;
      }
      case 4:  // cwpulselen
        if (t < pi / w) v = p.strength * w2 * std::cos(t * w2 + p.phaseshift);
        break;
      case 5: {  // monopulselen
        const double pp = t * w - pi / 2;
        if (pp < pi / 2) v = p.strength * (0.75 * std::cos(pp) + std::cos(3 * pp) / 4.0);
        break;
      }
      default:
        break;
    }
    e += v * fac;
  }
  return e;
}

// a = w1 * x1 + w0 * x0 (complex arrays)
__global__ void blend_kernel(double2* __restrict__ a, const double2* __restrict__ x1,
                             const double2* __restrict__ x0, double w1, double w0, long long len) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < len;
       i += (long long)gridDim.x * blockDim.x) {
    const double2 u = x1[i], v = x0[i];
    a[i] = make_double2(w1 * u.x + w0 * v.x, w1 * u.y + w0 * v.y);
  }
}

namespace {

size_t al256(size_t b) { return (b + 255) / 256 * 256; }

int cmf_alloc(Ctx& c) {
  CmfState& m = c.cmf;
  CIState& s = c.ci;
  const size_t G = c.G, n = c.nspf, nc = s.nc;
  const size_t bspf = sizeof(double2) * G * n, ba = sizeof(double2) * nc, bm = sizeof(double2) * n * n;
  const size_t b4 = bm * n * n, brp = sizeof(double2) * G * n * n;
  const size_t bh = sizeof(double2) * std::max<long long>(1, s.ndh), bs = sizeof(double2) * std::max<long long>(1, s.nsh);
  const size_t per = al256(bspf) + al256(ba) + 2 * al256(bm) + al256(b4) + al256(brp) + al256(bh) + 2 * al256(bs);
  const size_t need = 2 * per + al256(b4) + al256(3 * bm) + 3 * al256(ba);
  SG_TRY(m.ws.ensure(need));
  char* p = (char*)m.ws.ptr;
  auto take = [&](size_t b) {
    char* r = p;
    p += al256(b);
    return (double2*)r;
  };
  for (int k = 0; k < 2; ++k) {
    m.spfs[k] = take(bspf);
    m.avec[k] = take(ba);
    m.den[k] = take(bm);
    m.inv[k] = take(bm);
    m.tally[k] = take(b4);
    m.rp[k] = take(brp);
    m.xpot[k] = take(bh);
    m.xone[k] = take(bs);
    m.xz[k] = take(bs);
  }
  m.mat = take(b4);
  m.mats = take(3 * bm);
  m.ta = take(ba);
  m.tb = take(ba);
  m.tc = take(ba);
  return SINCGPU_OK;
}

int d2d(Ctx& c, void* dst, const void* src, size_t b) {
  SG_CUDA(cudaMemcpyAsync(dst, src, b, cudaMemcpyDeviceToDevice, c.stream));
  return SINCGPU_OK;
}

int get_allden(Ctx& c) {
  CmfState& m = c.cmf;
  SG_TRY(ci_denmat(c, m.avec[0], m.den[0], m.inv[0], m.p.denreg));
  return ci_tally(c, m.avec[0], m.avec[0], m.tally[0]);
}

int all_matel(Ctx& c) {
  CmfState& m = c.cmf;
  CIState& s = c.ci;
  SG_TRY(twoe_core(c, m.spfs[0], m.spfs[0], m.mat, nullptr, m.pa, m.pb, m.herm));
  SG_TRY(ci_onebody(c, m.spfs[0], m.mats));
  SG_TRY(ci_assemble(c, m.mat, m.mats));
  SG_TRY(d2d(c, m.xpot[0], s.xpot, sizeof(double2) * s.ndh));
  SG_TRY(d2d(c, m.xone[0], s.xone, sizeof(double2) * s.nsh));
  return d2d(c, m.xz[0], s.xz, sizeof(double2) * s.nsh);
}

int get_reducedpot(Ctx& c) {
  CmfState& m = c.cmf;
  return reduced_pot(c, (const double*)c.ws_red.ptr, m.pa.data(), m.pb.data(), (int)m.pa.size(), m.herm,
                     m.tally[0], m.rp[0], true);  // 2-RDM of one A-vector
}

// the CI matrices the sigma product uses: slot 0, or w1 slot1 + w0 slot0
int set_hamiltonian(Ctx& c, bool blend, double w1, double w0) {
  CmfState& m = c.cmf;
  CIState& s = c.ci;
  if (!blend) {
    SG_TRY(d2d(c, s.xpot, m.xpot[0], sizeof(double2) * s.ndh));
    SG_TRY(d2d(c, s.xone, m.xone[0], sizeof(double2) * s.nsh));
    return d2d(c, s.xz, m.xz[0], sizeof(double2) * s.nsh);
  }
  auto bl = [&](double2* a, const double2* x1, const double2* x0, long long len) -> int {
    if (len <= 0) return SINCGPU_OK;
    blend_kernel<<<std::min<long long>(ceil_div(len, 256), 148 * 8), 256, 0, c.stream>>>(a, x1, x0, w1, w0, len);
    SG_LAUNCHED();
    return SINCGPU_OK;
  };
  SG_TRY(bl(s.xpot, m.xpot[1], m.xpot[0], s.ndh));
  SG_TRY(bl(s.xone, m.xone[1], m.xone[0], s.nsh));
  return bl(s.xz, m.xz[1], m.xz[0], s.nsh);
}

// expoavecprop's saved order / step state around one Krylov call
int expoavecprop_step(Ctx& c, const double2* in, double2* out, double dt, double midtime) {
  CmfState& m = c.cmf;
  AvecPropState& a = m.a;
  ++a.icalled;
  if (a.icalled == 1) {
    a.tempstep = m.p.par_timestep / m.p.littlesteps;
    a.dim = std::min(a.maxorder, m.p.aorder);
  }
  if (a.icalled % 20 == 0) a.set = 0;
  a.tempstep *= a.dim < a.maxorder ? 4.0 : 1.1;
  const double ez = pulse_ez(m.pulses, midtime);
  const double2 tf = make_double2(m.p.timefac.x * dt, m.p.timefac.y * dt);
  int nstep = 0, nmult = 0;
  SG_TRY(expv_avector(c, in, out, 1.0, tf, a.dim, m.p.aerror, m.p.par_timestep / m.p.littlesteps, &a.tempstep,
                      &nstep, ez, m.nucdipz, a.maxorder + 1, &nmult));
  if (a.set == 0 && nstep == 1 && a.dim > 2) a.dim = std::max(2, a.dim - 1);
  if (nstep > 1) {
    a.set = 1;
    a.dim = std::min((int)std::floor(a.dim * 1.2) + 5, a.maxorder);
  }
  m.avec_iters += nmult;
  return SINCGPU_OK;
}

int cmf_prop_avector(Ctx& c, int linearflag, double tin, double tout) {
  CmfState& m = c.cmf;
  const size_t ba = sizeof(double2) * c.ci.nc;
  const double2* src = m.avec[1];
  for (int k = 1; k <= m.p.littlesteps; ++k) {
    const double ta = tin + (tout - tin) * (k - 1) / m.p.littlesteps;
    const double tb = tin + (tout - tin) * k / m.p.littlesteps;
    const double dt = tb - ta, mid = 0.5 * (ta + tb);
    if (linearflag == 0) {
      SG_TRY(set_hamiltonian(c, false, 0.0, 1.0));
    } else {
      const double s0 = (mid - m.first) / (m.last - m.first), s1 = (m.last - mid) / (m.last - m.first);
      SG_TRY(set_hamiltonian(c, true, s1, s0));
    }
    double2* dst = (k & 1) ? m.ta : m.tb;
    SG_TRY(expoavecprop_step(c, src, dst, dt, mid));
    if (c.ci.spin) SG_TRY(ci_spin_project(c, dst));
    src = dst;
  }
  return d2d(c, m.avec[0], src, ba);
}

int propspfs(Ctx& c, int linearflag, double tin, double tout) {
  CmfState& m = c.cmf;
  SG_TRY(d2d(c, m.spfs[0], m.spfs[1], sizeof(double2) * c.G * c.nspf));
  MeanFieldSlot slots[2] = {{m.den[0], m.inv[0], m.rp[0]}, {m.den[1], m.inv[1], m.rp[1]}};
  for (int k = 1; k <= m.p.littlesteps; ++k) {
    const double ta = tin + (tout - tin) * (k - 1) / m.p.littlesteps;
    const double tb = tin + (tout - tin) * k / m.p.littlesteps;
    const double ez = pulse_ez(m.pulses, 0.5 * (ta + tb));
    int it = 0;
    SG_TRY(expospfprop(c, m.spfs[0], slots, ta, tb, m.first, m.last, linearflag == 1, m.p.timefac, ez,
                       m.p.expotol, &it));
    SG_TRY(spf_orthogit(c, m.spfs[0], nullptr));
    m.orb_iters += it;
  }
  return SINCGPU_OK;
}

// <A|P H0 A>/<A|A> (project: apply the spin projector to H A) and |A|
int energy(Ctx& c, double ez, bool project, double* e, double* norm) {
  CmfState& m = c.cmf;
  const int nc = c.ci.nc;
  SG_TRY(set_hamiltonian(c, false, 0.0, 1.0));
  SG_TRY(ci_sigma(c, m.avec[0], m.tc, c.nucrepulsion, ez, m.nucdipz));
  if (project && c.ci.spin) SG_TRY(ci_spin_project(c, m.tc));
  std::vector<double2> a(nc), ha(nc);
  SG_CUDA(cudaMemcpyAsync(a.data(), m.avec[0], sizeof(double2) * nc, cudaMemcpyDeviceToHost, c.stream));
  SG_CUDA(cudaMemcpyAsync(ha.data(), m.tc, sizeof(double2) * nc, cudaMemcpyDeviceToHost, c.stream));
  SG_CUDA(cudaStreamSynchronize(c.stream));
  double sr = 0.0, s2 = 0.0;
  for (int i = 0; i < nc; ++i) {  // dot(a, Ha) = sum conj(a) Ha (real part), dot(a, a)
    sr += a[i].x * ha[i].x + a[i].y * ha[i].y;
    s2 += a[i].x * a[i].x + a[i].y * a[i].y;
  }
  *e = sr / s2;
  *norm = std::sqrt(s2);
  return SINCGPU_OK;
}

}  // namespace

int cmf_init(Ctx& c, const double2* phi, const double2* avec, double* e0) {
  CmfState& m = c.cmf;
  CIState& s = c.ci;
  SG_CHECK(s.attached, SINCGPU_ESTATE, "no walk tables attached");
  SG_CHECK(m.configured, SINCGPU_ESTATE, "call sincgpu_cmf_setup first");
  SG_TRY(cmf_alloc(c));
  const long long basis = s.spin ? s.numspinconfig : (long long)s.nc;
  m.a = AvecPropState();
  m.nucdipz = nucdip_z(c);
  m.a.maxorder = (int)std::max(1LL, std::min<long long>(2 * basis - 1, m.p.maxaorder));
  c.orb.expodim = m.p.expodim;
  c.orb.maxexpodim = m.p.maxexpodim;
  c.orb.expostepfac = m.p.expostepfac;
  c.orb.first_stepsize = m.p.par_timestep / m.p.littlesteps;
  c.orb.icalled = c.orb.thisexpodim = c.orb.exposet = 0;
  c.orb.tempstepsize = -1.0;
  SG_TRY(d2d(c, m.spfs[0], phi, sizeof(double2) * c.G * c.nspf));
  SG_TRY(d2d(c, m.avec[0], avec, sizeof(double2) * s.nc));
  if (s.spin) SG_TRY(ci_spin_project(c, m.avec[0]));
  // get_stuff(0): get_allden, all_matel, get_reducedpot
  SG_TRY(get_allden(c));
  SG_TRY(all_matel(c));
  SG_TRY(get_reducedpot(c));
  m.ready = true;
  double norm;
  SG_TRY(energy(c, pulse_ez(m.pulses, 0.0), false, e0, &norm));
  m.energy = *e0;
  m.norm = norm;
  return SINCGPU_OK;
}

// FP64 Coulomb passes and contractions while alive (the precision form's
// correction pass), the context's precision options restored after
struct Fp64Scope {
  Ctx& c;
  const int coul, tf32;
  bool on;
  Fp64Scope(Ctx& cc, bool enable) : c(cc), coul(cc.coul_fp32), tf32(cc.contract_tf32), on(enable) {
    if (on) {
      c.coul_fp32 = 0;
      c.contract_tf32 = 0;
    }
  }
  ~Fp64Scope() {
    if (on) {
      c.coul_fp32 = coul;
      c.contract_tf32 = tf32;
    }
  }
};

int cmf_step(Ctx& c, double tin, double tout) {
  CmfState& m = c.cmf;
  CIState& s = c.ci;
  SG_CHECK(m.ready, SINCGPU_ESTATE, "call sincgpu_cmf_init_dev first");
  SG_CHECK(tout != tin, SINCGPU_EINVAL, "empty time step");
  m.first = tin;
  m.last = tout;
  m.orb_iters = m.avec_iters = 0;
  // advance: slot 1 <- slot 0
  const size_t bspf = sizeof(double2) * c.G * c.nspf, ba = sizeof(double2) * s.nc;
  const size_t bm = sizeof(double2) * c.nspf * c.nspf, b4 = bm * c.nspf * c.nspf;
  SG_TRY(d2d(c, m.spfs[1], m.spfs[0], bspf));
  SG_TRY(d2d(c, m.avec[1], m.avec[0], ba));
  SG_TRY(d2d(c, m.den[1], m.den[0], bm));
  SG_TRY(d2d(c, m.inv[1], m.inv[0], bm));
  SG_TRY(d2d(c, m.tally[1], m.tally[0], b4));
  SG_TRY(d2d(c, m.rp[1], m.rp[0], bspf * c.nspf));
  SG_TRY(d2d(c, m.xpot[1], m.xpot[0], sizeof(double2) * s.ndh));
  SG_TRY(d2d(c, m.xone[1], m.xone[0], sizeof(double2) * s.nsh));
  SG_TRY(d2d(c, m.xz[1], m.xz[0], sizeof(double2) * s.nsh));
  // pre-prop
  SG_TRY(cmf_prop_avector(c, 0, tin, tout));
  SG_TRY(get_allden(c));
  SG_TRY(get_reducedpot(c));
  // main steps
  for (int ii = 0; ii < m.p.step_flag; ++ii) {
    SG_TRY(propspfs(c, 1, tin, tout));
    SG_TRY(cmf_prop_avector(c, 1, tin, tout));
    Fp64Scope fp64(c, m.fp64_last && ii == m.p.step_flag - 1);
    SG_TRY(get_allden(c));
    SG_TRY(all_matel(c));
    SG_TRY(get_reducedpot(c));
  }
  // post-prop (postpropflag=2)
  SG_TRY(cmf_prop_avector(c, 1, tin, tout));
  Fp64Scope fp64(c, m.fp64_last);
  SG_TRY(get_allden(c));
  SG_TRY(get_reducedpot(c));
  // prop_loop: spin projection, energy
  if (s.spin) SG_TRY(ci_spin_project(c, m.avec[0]));
  SG_TRY(energy(c, 0.0, true, &m.energy, &m.norm));
  return SINCGPU_OK;
}

}  // namespace sincgpu

using namespace sincgpu;

extern "C" {

int sincgpu_cmf_setup(sincgpu_ctx* h, double par_timestep, int littlesteps, double expotol, double aerror,
                      int aorder, int maxaorder, int expodim, int maxexpodim, double expostepfac, double denreg,
                      double timefac_re, double timefac_im) {
  CTX_CHECK(h);
  SG_CHECK(par_timestep > 0 && littlesteps >= 1, SINCGPU_EINVAL, "bad time step");
  SG_CHECK(aorder >= 1 && maxaorder >= 1 && maxaorder <= 124, SINCGPU_EINVAL,
           "aorder %d / maxaorder %d outside [1,124]", aorder, maxaorder);
  SG_CHECK(expodim >= 1 && maxexpodim >= 1 && maxexpodim <= 125, SINCGPU_EINVAL,
           "expodim %d / maxexpodim %d outside [1,125]", expodim, maxexpodim);
  CmfState& m = h->c.cmf;
  m.p.par_timestep = par_timestep;
  m.p.littlesteps = littlesteps;
  m.p.expotol = expotol;
  m.p.aerror = aerror;
  m.p.aorder = aorder;
  m.p.maxaorder = maxaorder;
  m.p.expodim = expodim;
  m.p.maxexpodim = maxexpodim;
  m.p.expostepfac = expostepfac;
  m.p.denreg = denreg;
  m.p.timefac = make_double2(timefac_re, timefac_im);
  m.configured = true;
  m.ready = false;
  return SINCGPU_OK;
}

int sincgpu_cmf_pulses(sincgpu_ctx* h, int npulses, const int* pulsetype, const double* params) {
  CTX_CHECK(h);
  SG_CHECK(npulses >= 0 && (npulses == 0 || (pulsetype && params)), SINCGPU_EINVAL, "bad pulse list");
  std::vector<PulseParams> v;
  for (int i = 0; i < npulses; ++i) {
    const double* q = params + 8 * i;
    PulseParams p;
    p.type = pulsetype[i];
    p.omega = q[0];
    p.omega2 = q[1];
    p.start = q[2];
    p.phaseshift = q[3];
    p.strength = q[4];
    p.longstep = q[5];
    p.theta = q[6];
    SG_CHECK(p.type >= 1 && p.type <= 5, SINCGPU_EINVAL, "pulse type %d outside [1,5]", p.type);
    SG_CHECK(p.omega > 0, SINCGPU_EINVAL, "pulse omega must be positive");
    SG_CHECK(std::fabs(std::sin(p.theta)) < 1e-12, SINCGPU_ERANGE,
             "only z-polarised pulses (pulsetheta = 0 or pi) are supported");
    v.push_back(p);
  }
  h->c.cmf.pulses = v;
  return SINCGPU_OK;
}

int sincgpu_pulse_ez(sincgpu_ctx* h, double t, double* ez) {
  CTX_CHECK(h);
  SG_CHECK(ez, SINCGPU_EINVAL, "null argument");
  *ez = pulse_ez(h->c.cmf.pulses, t);
  return SINCGPU_OK;
}

int sincgpu_cmf_init_dev(sincgpu_ctx* h, const double* phi, const double* avector, double* energy0) {
  CTX_CHECK(h);
  SG_CHECK(phi && avector && energy0, SINCGPU_EINVAL, "null argument");
  return cmf_init(h->c, (const double2*)phi, (const double2*)avector, energy0);
}

int sincgpu_cmf_step(sincgpu_ctx* h, double tin, double tout, double* energy, double* norm, int* orb_iters,
                     int* avec_iters) {
  CTX_CHECK(h);
  SG_TRY(cmf_step(h->c, tin, tout));
  const CmfState& m = h->c.cmf;
  if (energy) *energy = m.energy;
  if (norm) *norm = m.norm;
  if (orb_iters) *orb_iters = m.orb_iters;
  if (avec_iters) *avec_iters = m.avec_iters;
  return SINCGPU_OK;
}

int sincgpu_cmf_dipole_z(sincgpu_ctx* h, double* dipole, double* normsq) {
  CTX_CHECK(h);
  Ctx& c = h->c;
  SG_CHECK(c.cmf.ready && dipole && normsq, SINCGPU_EINVAL, "no CMF state or null argument");
  SG_TRY(set_hamiltonian(c, false, 0.0, 1.0));
  double2 d;
  SG_TRY(ci_dipole_z(c, c.cmf.avec[0], c.cmf.tc, c.cmf.nucdipz, &d, normsq));
  dipole[0] = d.x;
  dipole[1] = d.y;
  return SINCGPU_OK;
}

int sincgpu_cmf_state_dev(sincgpu_ctx* h, double* phi, double* avector) {
  CTX_CHECK(h);
  Ctx& c = h->c;
  SG_CHECK(c.cmf.ready, SINCGPU_ESTATE, "no CMF state");
  if (phi)
    SG_CUDA(cudaMemcpyAsync(phi, c.cmf.spfs[0], sizeof(double2) * c.G * c.nspf, cudaMemcpyDeviceToDevice,
                            c.stream));
  if (avector)
    SG_CUDA(cudaMemcpyAsync(avector, c.cmf.avec[0], sizeof(double2) * c.ci.nc, cudaMemcpyDeviceToDevice,
                            c.stream));
  SG_CUDA(cudaStreamSynchronize(c.stream));
  return SINCGPU_OK;
}

}  // extern "C"
