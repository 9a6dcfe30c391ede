// C ABI of the CI side: walk tables, RDMs, one-body matrix elements, assembled
// sparse matrices and the sigma product (declarations: include/sincgpu.h).
#include <cstring>
#include <vector>
#include "context.hpp"
#include "walks.hpp"
#include "../../include/sincgpu.h"


namespace sincgpu {
double nucdip_z(const Ctx& c) {  // nucdipvalue (SINCDVR/init_sinc_new.f90:652-662), z component
  double d = 0.0;
  for (int i = 0; i < c.numcenters; ++i) d += c.nuccharges[i] * c.centershift[3 * i + 2] / 2.0 * c.spacing;
  return d;
}
}  // namespace sincgpu

using namespace sincgpu;

namespace {

int up(Ctx& c, void* dst, const void* src, size_t bytes) {
  SG_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, c.stream));
  return SINCGPU_OK;
}
int down(Ctx& c, void* dst, const void* src, size_t bytes) {
  SG_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, c.stream));
  return SINCGPU_OK;
}


template <class T>
void copy_out(const std::vector<T>& v, int* out) {
  for (size_t i = 0; i < v.size(); ++i) out[i] = (int)v[i];
}

}  // namespace

extern "C" {

int sincgpu_walks_create(sincgpu_walks** out, int numelec, int nspf, int restrictms, int nthreads) {
  SG_CHECK(out, SINCGPU_EINVAL, "null output pointer");
  *out = nullptr;
  sincgpu_walks* h = new sincgpu_walks();
  int rc = build_walks(h->w, numelec, nspf, restrictms, nthreads);
  if (rc != SINCGPU_OK) {
    delete h;
    return rc;
  }
  *out = h;
  return SINCGPU_OK;
}

int sincgpu_walks_destroy(sincgpu_walks* h) {
  delete h;
  return SINCGPU_OK;
}

int sincgpu_walks_sizes(sincgpu_walks* h, long long* s, int n) {
  SG_CHECK(h && s, SINCGPU_EINVAL, "null argument");
  const Walks& w = h->w;
  long long v[6] = {w.numconfig, w.numpart, w.scol.back(), w.dcol.back(), (long long)w.singlehop.size(),
                    (long long)w.doublehop.size()};
  for (int i = 0; i < n && i < 6; ++i) s[i] = v[i];
  return SINCGPU_OK;
}

int sincgpu_walks_table(sincgpu_walks* h, int which, int* out) {
  SG_CHECK(h && out, SINCGPU_EINVAL, "null argument");
  const Walks& w = h->w;
  switch (which) {
    case SINCGPU_T_CONFIGLIST: copy_out(w.configlist, out); break;
    case SINCGPU_T_NUMSINGLEWALKS: copy_out(w.numsinglewalks, out); break;
    case SINCGPU_T_NUMDOUBLEWALKS: copy_out(w.numdoublewalks, out); break;
    case SINCGPU_T_SINGLEWALKOPSPF: copy_out(w.singlewalkopspf, out); break;
    case SINCGPU_T_SINGLEWALKDIRPHASE: copy_out(w.singlewalkdirphase, out); break;
    case SINCGPU_T_SINGLEWALK: copy_out(w.singlewalk, out); break;
    case SINCGPU_T_DOUBLEWALKDIRSPF: copy_out(w.doublewalkdirspf, out); break;
    case SINCGPU_T_DOUBLEWALKDIRPHASE: copy_out(w.doublewalkdirphase, out); break;
    case SINCGPU_T_DOUBLEWALK: copy_out(w.doublewalk, out); break;
    case SINCGPU_T_SINGLEHOPOFF: copy_out(w.singlehop_off, out); break;
    case SINCGPU_T_SINGLEHOP: copy_out(w.singlehop, out); break;
    case SINCGPU_T_SINGLEHOPWALKSTART: copy_out(w.singlehopwalkstart, out); break;
    case SINCGPU_T_SINGLEHOPWALKEND: copy_out(w.singlehopwalkend, out); break;
    case SINCGPU_T_DOUBLEHOPOFF: copy_out(w.doublehop_off, out); break;
    case SINCGPU_T_DOUBLEHOP: copy_out(w.doublehop, out); break;
    case SINCGPU_T_DOUBLEHOPWALKSTART: copy_out(w.doublehopwalkstart, out); break;
    case SINCGPU_T_DOUBLEHOPWALKEND: copy_out(w.doublehopwalkend, out); break;
    case SINCGPU_T_SINGLEDIAGHOP: copy_out(w.singlediaghop, out); break;
    case SINCGPU_T_DOUBLEDIAGHOP: copy_out(w.doublediaghop, out); break;
    case SINCGPU_T_NUMSPINWALKS: copy_out(w.numspinwalks, out); break;
    case SINCGPU_T_SPINWALK: copy_out(w.spinwalk, out); break;
    case SINCGPU_T_SPINWALKDIRPHASE: copy_out(w.spinwalkdirphase, out); break;
    case SINCGPU_T_SPINSETOFF: copy_out(w.spinset_off, out); break;
    case SINCGPU_T_SPINSETS: copy_out(w.spinsets, out); break;
    case SINCGPU_T_SPINSETRANK: copy_out(w.spinsetrank, out); break;
    case SINCGPU_T_SPINELIMINATED: copy_out(w.spin_eliminated, out); break;
    default:
      set_error("unknown walk table id %d", which);
      return SINCGPU_EINVAL;
  }
  return SINCGPU_OK;
}

int sincgpu_walks_spin(sincgpu_walks* h, int spinrestrictval) {
  SG_CHECK(h, SINCGPU_EINVAL, "null argument");
  return build_spin(h->w, spinrestrictval);
}

int sincgpu_walks_spin_sizes(sincgpu_walks* h, long long* s, int n) {
  SG_CHECK(h && s, SINCGPU_EINVAL, "null argument");
  const Walks& w = h->w;
  SG_CHECK(w.spinrestrictval >= 0, SINCGPU_ESTATE, "spin tables not built");
  long long v[6] = {(long long)w.spinsetrank.size(), w.numspinconfig, (long long)w.spinwalk.size(),
                    (long long)w.spinproj.size(), (long long)w.spin_eliminated.size(), w.maxspinsetsize};
  for (int i = 0; i < n && i < 6; ++i) s[i] = v[i];
  return SINCGPU_OK;
}

int sincgpu_walks_spinprojectors(sincgpu_walks* h, double* out) {
  SG_CHECK(h && out, SINCGPU_EINVAL, "null argument");
  SG_CHECK(h->w.spinrestrictval >= 0, SINCGPU_ESTATE, "spin tables not built");
  std::memcpy(out, h->w.spinproj.data(), sizeof(double) * h->w.spinproj.size());
  return SINCGPU_OK;
}

int sincgpu_dipole_z_dev(sincgpu_ctx* h, const double* avector, double* dipole, double* normsq) {
  CTX_CHECK(h);
  Ctx& c = h->c;
  SG_CHECK(avector && dipole && normsq, SINCGPU_EINVAL, "null argument");
  SG_TRY(c.ws_ci2.ensure(sizeof(double2) * c.ci.nc));
  double2 d;
  SG_TRY(ci_dipole_z(c, (const double2*)avector, (double2*)c.ws_ci2.ptr, nucdip_z(c), &d, normsq));
  dipole[0] = d.x;
  dipole[1] = d.y;
  return SINCGPU_OK;
}

int sincgpu_dipole_z(sincgpu_ctx* h, const double* avector, double* dipole, double* normsq) {
  CTX_CHECK(h);
  Ctx& c = h->c;
  SG_CHECK(c.ci.attached, SINCGPU_ESTATE, "no walk tables attached");
  SG_CHECK(avector, SINCGPU_EINVAL, "null argument");
  const size_t b = sizeof(double2) * c.ci.nc;
  SG_TRY(c.ws_io.ensure(b));
  SG_CUDA(cudaMemcpyAsync(c.ws_io.ptr, avector, b, cudaMemcpyHostToDevice, c.stream));
  return sincgpu_dipole_z_dev(h, (const double*)c.ws_io.ptr, dipole, normsq);
}

int sincgpu_spin_project_dev(sincgpu_ctx* h, double* avector) {
  CTX_CHECK(h);
  SG_CHECK(avector, SINCGPU_EINVAL, "null argument");
  return ci_spin_project(h->c, (double2*)avector);
}

int sincgpu_spin_project(sincgpu_ctx* h, const double* in, double* out) {
  CTX_CHECK(h);
  Ctx& c = h->c;
  SG_CHECK(c.ci.attached, SINCGPU_ESTATE, "no walk tables attached");
  SG_CHECK(in && out, SINCGPU_EINVAL, "null argument");
  const size_t b = sizeof(double2) * c.ci.nc;
  SG_TRY(c.ws_io.ensure(b));
  SG_CUDA(cudaMemcpyAsync(c.ws_io.ptr, in, b, cudaMemcpyHostToDevice, c.stream));
  SG_TRY(ci_spin_project(c, (double2*)c.ws_io.ptr));
  SG_CUDA(cudaMemcpyAsync(out, c.ws_io.ptr, b, cudaMemcpyDeviceToHost, c.stream));
  SG_CUDA(cudaStreamSynchronize(c.stream));
  return SINCGPU_OK;
}

int sincgpu_ci_attach(sincgpu_ctx* h, sincgpu_walks* w) {
  CTX_CHECK(h);
  SG_CHECK(w, SINCGPU_EINVAL, "null walk tables");
  return ci_attach(h->c, w->w);
}

// ----------------------------------------------------------------- device forms
int sincgpu_getdenmat_dev(sincgpu_ctx* h, const double* avector, double* denmat, double* invdenmat,
                          double denreg) {
  CTX_CHECK(h);
  SG_CHECK(avector && denmat, SINCGPU_EINVAL, "null argument");
  return ci_denmat(h->c, (const double2*)avector, (double2*)denmat, (double2*)invdenmat, denreg);
}

int sincgpu_get_tworeducedx_dev(sincgpu_ctx* h, const double* a1, const double* a2, double* tally) {
  CTX_CHECK(h);
  SG_CHECK(a1 && tally, SINCGPU_EINVAL, "null argument");
  return ci_tally(h->c, (const double2*)a1, (const double2*)(a2 ? a2 : a1), (double2*)tally);
}

int sincgpu_onebody_matel_dev(sincgpu_ctx* h, const double* phi, double* mats) {
  CTX_CHECK(h);
  SG_CHECK(phi && mats, SINCGPU_EINVAL, "null argument");
  return ci_onebody(h->c, (const double2*)phi, (double2*)mats);
}

int sincgpu_assemble_sparsemats_dev(sincgpu_ctx* h, const double* twoematel, const double* mats) {
  CTX_CHECK(h);
  SG_CHECK(twoematel && mats, SINCGPU_EINVAL, "null argument");
  return ci_assemble(h->c, (const double2*)twoematel, (const double2*)mats);
}

int sincgpu_sparseconfigmult_dev(sincgpu_ctx* h, const double* in, double* out, double ezfield) {
  CTX_CHECK(h);
  SG_CHECK(in && out && in != out, SINCGPU_EINVAL, "in/out must be distinct, non-null");
  return ci_sigma(h->c, (const double2*)in, (double2*)out, h->c.nucrepulsion, ezfield, nucdip_z(h->c));
}

namespace {
// avec_ready (or nullptr): the A-vector reached the device before the orbitals (the
// host-array entry), so the side stream's RDMs start on it while the orbitals are
// still being copied; the mix and kinetic contraction wait for the orbitals.
// host_out (or nullptr): the host-array entry's RHS buffer; the RHS is copied there
// as soon as it is final, and twoematel, which that entry does not return, is formed
// on the side stream while the copy runs
int orbital_rhs_avec_impl(sincgpu_ctx* h, const double* phi, const double* avector, double tre, double tim,
                          double ztdpot, double* denmat, double* invdenmat, double* tally, double* twoematel,
                          double* reducedpot, double* out, cudaEvent_t avec_ready, double* host_out = nullptr) {
  SG_CHECK(phi && avector && denmat && invdenmat && tally && reducedpot && out, SINCGPU_EINVAL,
           "null argument");
  SG_CHECK(out != phi, SINCGPU_EINVAL, "out must not alias phi");
  Ctx& c = h->c;
  const double2 *P = (const double2*)phi, *A = (const double2*)avector;
  const double2 tf = make_double2(tre, tim);
  const size_t bout = sizeof(double2) * (size_t)c.G * c.nspf;
  if (!c.rhs_overlap) {
    SG_TRY(sincgpu_getdenmat_dev(h, avector, denmat, invdenmat, 1e-10));
    SG_TRY(sincgpu_get_tworeducedx_dev(h, avector, avector, tally));
    // the 2-RDM of one A-vector: reducedpot(x,i,k) = conj reducedpot(x,k,i)
    SG_TRY(orbital_rhs(c, P, (const double2*)tally, (const double2*)denmat, (const double2*)invdenmat, tf, ztdpot,
                       (double2*)twoematel, (double2*)reducedpot, (double2*)out, true));
    if (host_out) SG_CUDA(cudaMemcpyAsync(host_out, out, bout, cudaMemcpyDeviceToHost, c.stream));
    return SINCGPU_OK;
  }
  // The RDMs, the density-matrix inverse, the mix with denmat and the kinetic
  // contraction depend on the A-vector or the orbitals alone: they run on the
  // side stream while this stream runs the Coulomb passes.  The side stream starts
  // after everything issued so far (ev_fork); reducedpot waits for the tally
  // (ev_ci) and the reduced-potential apply for the kinetic result (ev_join).
  // twoematel, which nothing here reads, then runs on the side stream beside
  // reducedpot, the apply and the projection (mean_field), and joins last.  Workspaces grown meanwhile are ordered on the side stream (their
  // owner is c.stream, swapped below).  The same fork and join hold under graph
  // capture.
  SG_TRY(side_stream(c));
  SG_CUDA(cudaEventRecord(c.ev_fork, c.stream));
  SG_CUDA(cudaStreamWaitEvent(c.side, avec_ready ? avec_ready : c.ev_fork, 0));
  const cudaStream_t main_stream = c.stream;
  c.stream = c.side;
  const int rc_side = [&]() -> int {
    SG_TRY(ci_denmat(c, A, (double2*)denmat, (double2*)invdenmat, 1e-10));
    SG_TRY(ci_tally(c, A, A, (double2*)tally));
    SG_CUDA(cudaEventRecord(c.ev_ci, c.side));
    if (avec_ready) SG_CUDA(cudaStreamWaitEvent(c.side, c.up_n ? c.ev_up[c.up_n - 1] : c.ev_fork, 0));
    return actreduced_pre(c, P, (const double2*)denmat, ztdpot);
  }();
  c.stream = main_stream;
  SG_CUDA(cudaEventRecord(c.ev_join, c.side));
  if (rc_side != SINCGPU_OK) {
    cudaStreamWaitEvent(c.stream, c.ev_join, 0);
    return rc_side;
  }
  // reducedpot applies itself to the orbitals in its epilogue where it can
  // (after the kinetic result: ev_join); otherwise actreduced_post applies it
  double2 *S = nullptr, *T = nullptr, *part = nullptr;
  int rc = actreduced_temps(c, &S, &T, &part);
  RpApply ap{P, S, (const double2*)invdenmat, tf, T, c.ev_join, false, P, part};
  const bool deferred = host_out && twoematel;
  TwoeDefer defer;
  if (rc == SINCGPU_OK)
    rc = mean_field(c, P, (const double2*)tally, deferred ? nullptr : (double2*)twoematel, (double2*)reducedpot,
                    true, c.ev_ci, twoematel ? c.side : nullptr, &ap, deferred ? &defer : nullptr);
  SG_CUDA(cudaStreamWaitEvent(c.stream, c.ev_join, 0));
  int rc2 = rc == SINCGPU_OK ? actreduced_post(c, P, P, (const double2*)invdenmat, (const double2*)reducedpot, tf,
                                               1, 1, (double2*)out, ap.done, ap.done)
                             : rc;
  if (rc2 == SINCGPU_OK && host_out) {
    // the RHS is final: its copy to the host overlaps the deferred twoematel (issued
    // first: a copy to pageable memory returns only when it is done)
    SG_CUDA(cudaEventRecord(c.ev_rhs, c.stream));
    if (deferred) rc2 = twoe_deferred(c, P, defer, (double2*)twoematel, c.ev_rhs, c.side);
    SG_CUDA(cudaMemcpyAsync(host_out, out, bout, cudaMemcpyDeviceToHost, c.stream));
  }
  // twoematel (side stream) joins last
  if (twoematel) SG_CUDA(cudaStreamWaitEvent(c.stream, c.ev_twoe, 0));
  return rc2;
}
}  // namespace

int sincgpu_orbital_rhs_avec_dev(sincgpu_ctx* h, const double* phi, const double* avector, double tre,
                                 double tim, double ztdpot, double* denmat, double* invdenmat, double* tally,
                                 double* twoematel, double* reducedpot, double* out) {
  CTX_CHECK(h);
  return orbital_rhs_avec_impl(h, phi, avector, tre, tim, ztdpot, denmat, invdenmat, tally, twoematel, reducedpot,
                               out, nullptr);
}

int sincgpu_expoavecprop_dev(sincgpu_ctx* h, const double* avec_in, double* avec_out, double t,
                             double tre, double tim, int krylovdim, double tol, double anorm, double ezfield,
                             double* stepguess, int* nstep) {
  CTX_CHECK(h);
  SG_CHECK(avec_in && avec_out && stepguess && avec_in != avec_out, SINCGPU_EINVAL, "bad argument");
  SG_CHECK(*stepguess > 0.0, SINCGPU_EINVAL, "stepguess must be positive");
  return expv_avector(h->c, (const double2*)avec_in, (double2*)avec_out, t, make_double2(tre, tim), krylovdim,
                      tol, anorm, stepguess, nstep, ezfield, nucdip_z(h->c));
}

int sincgpu_expoavecprop(sincgpu_ctx* h, const double* avec_in, double* avec_out, double t, double tre,
                         double tim, int krylovdim, double tol, double anorm, double ezfield, double* stepguess,
                         int* nstep) {
  CTX_CHECK(h);
  Ctx& c = h->c;
  SG_CHECK(c.ci.attached, SINCGPU_ESTATE, "no walk tables attached");
  SG_CHECK(avec_in && avec_out, SINCGPU_EINVAL, "null argument");
  const size_t ba = sizeof(double2) * c.ci.nc, pa = (ba + 255) / 256 * 256;
  SG_TRY(c.ws_io.ensure(2 * pa));
  double* di = (double*)c.ws_io.ptr;
  double* dout = (double*)((char*)c.ws_io.ptr + pa);
  SG_TRY(up(c, di, avec_in, ba));
  SG_TRY(sincgpu_expoavecprop_dev(h, di, dout, t, tre, tim, krylovdim, tol, anorm, ezfield, stepguess, nstep));
  SG_TRY(down(c, avec_out, dout, ba));
  SG_CUDA(cudaStreamSynchronize(c.stream));
  return SINCGPU_OK;
}

// ----------------------------------------------------------------- host forms
int sincgpu_orbital_rhs_avec(sincgpu_ctx* h, const double* phi, const double* avector, double tre,
                             double tim, double ztdpot, double* outspfs) {
  CTX_CHECK(h);
  Ctx& c = h->c;
  SG_CHECK(c.ci.attached, SINCGPU_ESTATE, "no walk tables attached");
  SG_CHECK(phi && avector && outspfs, SINCGPU_EINVAL, "null argument");
  const int n = c.nspf;
  const size_t bphi = sizeof(double2) * (size_t)c.G * n, ba = sizeof(double2) * c.ci.nc;
  const size_t bm = sizeof(double2) * n * n, b4 = sizeof(double2) * (size_t)n * n * n * n;
  auto pad = [](size_t b) { return (b + 255) / 256 * 256; };
  const size_t total = 2 * pad(bphi) + pad(ba) + 2 * pad(bm) + 2 * pad(b4);
  SG_TRY(c.ws_io.ensure(total));
  SG_TRY(c.ws_state.ensure(sizeof(double2) * (size_t)c.G * n * n));
  char* p = (char*)c.ws_io.ptr;
  double* dphi = (double*)p;
  p += pad(bphi);
  double* dout = (double*)p;
  p += pad(bphi);
  double* da = (double*)p;
  p += pad(ba);
  double* dden = (double*)p;
  p += pad(bm);
  double* dinv = (double*)p;
  p += pad(bm);
  double* dtal = (double*)p;
  p += pad(b4);
  double* dmat = (double*)p;
  // the A-vector first: the RDMs start on it while the orbitals are copied.  With
  // rhs_upload_groups > 1 the orbitals go up in groups on the copy stream and the
  // Coulomb pair loop starts on the first group while the others are in flight
  if (c.rhs_overlap) SG_TRY(side_stream(c));
  SG_TRY(up(c, da, avector, ba));
  if (c.rhs_overlap) SG_CUDA(cudaEventRecord(c.ev_avec, c.stream));
  int ng = 0;
  if (c.rhs_overlap && c.up_groups > 1 && n > 1) {
    // group ends ceil(n (g + 1) / groups), repeated ends dropped
    for (int g = 0; g < c.up_groups; ++g) {
      const int e = (n * (g + 1) + c.up_groups - 1) / c.up_groups;
      if (ng == 0 || e > c.up_end[ng - 1]) c.up_end[ng++] = e;
    }
  }
  if (ng > 1) {
    // the copies wait for everything issued so far (workspace growth included)
    SG_CUDA(cudaEventRecord(c.ev_entry, c.stream));
    SG_CUDA(cudaStreamWaitEvent(c.copy, c.ev_entry, 0));
    const size_t borb = sizeof(double2) * (size_t)c.G;
    for (int g = 0, b = 0; g < ng; b = c.up_end[g++]) {
      SG_CUDA(cudaMemcpyAsync((char*)dphi + borb * b, (const char*)phi + borb * b, borb * (c.up_end[g] - b),
                              cudaMemcpyHostToDevice, c.copy));
      SG_CUDA(cudaEventRecord(c.ev_up[g], c.copy));
    }
    c.up_n = ng;
  } else {
    SG_TRY(up(c, dphi, phi, bphi));
  }
  const int rc = orbital_rhs_avec_impl(h, dphi, da, tre, tim, ztdpot, dden, dinv, dtal, dmat,
                                       (double*)c.ws_state.ptr, dout, c.rhs_overlap ? c.ev_avec : nullptr, outspfs);
  if (c.up_n) {
    // the last group is joined here too, whatever the evaluation did
    c.up_n = 0;
    cudaStreamWaitEvent(c.stream, c.ev_up[ng - 1], 0);
  }
  if (rc != SINCGPU_OK) {
    // no copy may still use the caller's buffers once this returns
    cudaStreamSynchronize(c.stream);
    return rc;
  }
  SG_CUDA(cudaStreamSynchronize(c.stream));
  return SINCGPU_OK;
}

int sincgpu_getdenmat(sincgpu_ctx* h, const double* avector, double* denmat, double* invdenmat) {
  CTX_CHECK(h);
  Ctx& c = h->c;
  SG_CHECK(c.ci.attached, SINCGPU_ESTATE, "no walk tables attached");
  SG_CHECK(avector && denmat, SINCGPU_EINVAL, "null argument");
  const int n = c.nspf;
  const size_t ba = sizeof(double2) * c.ci.nc, bm = sizeof(double2) * n * n;
  SG_TRY(c.ws_io.ensure(ba + 2 * bm + 512));
  char* base = (char*)c.ws_io.ptr;
  double2* da = (double2*)base;
  double2* dd = (double2*)(base + (ba + 255) / 256 * 256);
  double2* di = dd + n * n;
  SG_TRY(up(c, da, avector, ba));
  SG_TRY(ci_denmat(c, da, dd, invdenmat ? di : nullptr, 1e-10));
  SG_TRY(down(c, denmat, dd, bm));
  if (invdenmat) SG_TRY(down(c, invdenmat, di, bm));
  SG_CUDA(cudaStreamSynchronize(c.stream));
  return SINCGPU_OK;
}

int sincgpu_get_tworeducedx(sincgpu_ctx* h, const double* a1, const double* a2, double* tally) {
  CTX_CHECK(h);
  Ctx& c = h->c;
  SG_CHECK(c.ci.attached, SINCGPU_ESTATE, "no walk tables attached");
  SG_CHECK(a1 && tally, SINCGPU_EINVAL, "null argument");
  const int n = c.nspf;
  const size_t ba = sizeof(double2) * c.ci.nc, bt = sizeof(double2) * (size_t)n * n * n * n;
  const size_t pa = (ba + 255) / 256 * 256;
  SG_TRY(c.ws_io.ensure(2 * pa + bt));
  char* base = (char*)c.ws_io.ptr;
  double2* d1 = (double2*)base;
  double2* d2 = (double2*)(base + pa);
  double2* dt = (double2*)(base + 2 * pa);
  SG_TRY(up(c, d1, a1, ba));
  if (a2 && a2 != a1) SG_TRY(up(c, d2, a2, ba));
  SG_TRY(ci_tally(c, d1, (a2 && a2 != a1) ? d2 : d1, dt));
  SG_TRY(down(c, tally, dt, bt));
  SG_CUDA(cudaStreamSynchronize(c.stream));
  return SINCGPU_OK;
}

int sincgpu_onebody_matel(sincgpu_ctx* h, const double* phi, double* potmatel, double* kematel,
                          double* zmatel) {
  CTX_CHECK(h);
  Ctx& c = h->c;
  SG_CHECK(phi && potmatel && kematel && zmatel, SINCGPU_EINVAL, "null argument");
  const int n = c.nspf;
  const size_t bphi = sizeof(double2) * (size_t)c.G * n, bm = sizeof(double2) * n * n;
  SG_TRY(c.ws_io.ensure(bphi + 3 * bm + 256));
  double2* dp = (double2*)c.ws_io.ptr;
  double2* dm = dp + (size_t)c.G * n;
  SG_TRY(up(c, dp, phi, bphi));
  SG_TRY(ci_onebody(c, dp, dm));
  SG_TRY(down(c, potmatel, dm, bm));
  SG_TRY(down(c, kematel, dm + n * n, bm));
  SG_TRY(down(c, zmatel, dm + 2 * n * n, bm));
  SG_CUDA(cudaStreamSynchronize(c.stream));
  return SINCGPU_OK;
}

int sincgpu_assemble_sparsemats(sincgpu_ctx* h, const double* twoematel, const double* potmatel,
                                const double* kematel, const double* zmatel) {
  CTX_CHECK(h);
  Ctx& c = h->c;
  SG_CHECK(twoematel && potmatel && kematel && zmatel, SINCGPU_EINVAL, "null argument");
  const int n = c.nspf;
  const size_t b4 = sizeof(double2) * (size_t)n * n * n * n, bm = sizeof(double2) * n * n;
  SG_TRY(c.ws_io.ensure(b4 + 3 * bm + 256));
  double2* dt = (double2*)c.ws_io.ptr;
  double2* dm = dt + (size_t)n * n * n * n;
  SG_TRY(up(c, dt, twoematel, b4));
  SG_TRY(up(c, dm, potmatel, bm));
  SG_TRY(up(c, dm + n * n, kematel, bm));
  SG_TRY(up(c, dm + 2 * n * n, zmatel, bm));
  SG_TRY(ci_assemble(c, dt, dm));
  SG_CUDA(cudaStreamSynchronize(c.stream));
  return SINCGPU_OK;
}

int sincgpu_sparseconfigmult(sincgpu_ctx* h, const double* in, double* out, double ezfield) {
  CTX_CHECK(h);
  Ctx& c = h->c;
  SG_CHECK(c.ci.attached, SINCGPU_ESTATE, "no walk tables attached");
  SG_CHECK(in && out, SINCGPU_EINVAL, "null argument");
  const size_t ba = sizeof(double2) * c.ci.nc, pa = (ba + 255) / 256 * 256;
  SG_TRY(c.ws_io.ensure(2 * pa));
  double2* di = (double2*)c.ws_io.ptr;
  double2* dout = (double2*)((char*)c.ws_io.ptr + pa);
  SG_TRY(up(c, di, in, ba));
  SG_TRY(ci_sigma(c, di, dout, c.nucrepulsion, ezfield, nucdip_z(c)));
  SG_TRY(down(c, out, dout, ba));
  SG_CUDA(cudaStreamSynchronize(c.stream));
  return SINCGPU_OK;
}

}  // extern "C"
