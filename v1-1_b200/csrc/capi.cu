// C ABI of the sinc-DVR orbital-RHS library (declarations: include/sincgpu.h).
#include <atomic>
#include <cstdarg>
#include <cstring>
#include <mutex>
#include <algorithm>
#include <vector>
#include <string>
#include "context.hpp"
#include "fft_lengths.h"
#include "../../include/sincgpu.h"

namespace sincgpu {

static thread_local char g_err[512] = "";
static std::atomic<long long> g_launches{0};

void count_launch() { g_launches.fetch_add(1, std::memory_order_relaxed); }

void set_error(const char* fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_err, sizeof(g_err), fmt, ap);
  va_end(ap);
}

int Workspace::ensure(size_t need) {
  if (need <= bytes) return SINCGPU_OK;
  if (owner) {
    cudaStreamCaptureStatus st = cudaStreamCaptureStatusNone;
    if (cudaStreamIsCapturing(*owner, &st) == cudaSuccess && st != cudaStreamCaptureStatusNone) {
      set_error("a workspace would grow to %zu bytes during graph capture (run the call once before capturing)",
                need);
      return SINCGPU_ESTATE;
    }
  }
  release();
  size_t want = need + need / 8;
  const cudaError_t e = owner ? cudaMallocAsync(&ptr, want, *owner) : cudaMalloc(&ptr, want);
  if (e != cudaSuccess) {
    cudaGetLastError();
    ptr = nullptr;
    set_error("cudaMalloc of %zu bytes failed", want);
    return SINCGPU_ENOMEM;
  }
  bytes = want;
  return SINCGPU_OK;
}

void Workspace::release() {
  if (ptr) {
    if (owner)
      cudaFreeAsync(ptr, *owner);
    else
      cudaFree(ptr);
  }
  ptr = nullptr;
  bytes = 0;
}

namespace {
std::mutex g_pin_mu;
std::vector<std::pair<size_t, void*>> g_pin_free;
}  // namespace

int pinned_get(size_t bytes, void** p) {
  {
    std::lock_guard<std::mutex> lk(g_pin_mu);
    for (auto it = g_pin_free.begin(); it != g_pin_free.end(); ++it)
      if (it->first == bytes) {
        *p = it->second;
        g_pin_free.erase(it);
        return SINCGPU_OK;
      }
  }
  SG_CUDA(cudaMallocHost(p, bytes));
  return SINCGPU_OK;
}

void pinned_put(size_t bytes, void* p) {
  std::lock_guard<std::mutex> lk(g_pin_mu);
  g_pin_free.emplace_back(bytes, p);
}

int dalloc(Ctx& c, void** p, size_t bytes) {
  *p = nullptr;
  if (cudaMallocAsync(p, std::max<size_t>(bytes, 16), c.stream) != cudaSuccess) {
    cudaGetLastError();
    *p = nullptr;
    set_error("device allocation of %zu bytes failed", bytes);
    return SINCGPU_ENOMEM;
  }
  return SINCGPU_OK;
}

void dfree(Ctx& c, void* p) {
  if (p) cudaFreeAsync(p, c.stream);
}

int dupload(Ctx& c, void** dst, const void* src, size_t bytes) {
  dfree(c, *dst);
  *dst = nullptr;
  if (bytes == 0) return SINCGPU_OK;
  SG_TRY(dalloc(c, dst, bytes));
  SG_CUDA(cudaMemcpyAsync(*dst, src, bytes, cudaMemcpyHostToDevice, c.stream));
  return SINCGPU_OK;
}

void Ctx::bind_workspaces() {
  for (Workspace* w : {&ws_fft, &ws_pairs, &ws_gemm, &ws_twoe, &ws_rhs, &ws_io, &ws_red, &ws_conv, &ws_state, &ws_ci,
                       &ws_ci2, &ws_kry, &ws_orb, &ws_tcerr, &ws_tc, &ws_bq, &cmf.ws})
    w->owner = &stream;
}

Ctx::~Ctx() {
  // stream-ordered frees below follow the context's own work; work that a batch
  // graph ran on another stream is waited for here
  if (side) cudaStreamSynchronize(side);
  if (stream) cudaStreamSynchronize(stream);
  if (rhs_graph) cudaDeviceSynchronize();
  for (void* p : {(void*)d_kevect, (void*)d_ketile, (void*)d_pot, (void*)d_zdip, (void*)d_tcoul, (void*)d_khat,
                  (void*)d_roots, (void*)d_khat32, (void*)d_roots32, (void*)d_khT, (void*)d_khT32, (void*)d_khr, (void*)d_khr32})
    dfree(*this, p);
  ws_fft.release();
  ws_pairs.release();
  ws_gemm.release();
  ws_twoe.release();
  ws_rhs.release();
  ws_io.release();
  ws_red.release();
  ws_conv.release();
  ws_state.release();
  ws_ci.release();
  ws_ci2.release();
  ws_kry.release();
  ws_orb.release();
  ws_tcerr.release();
  ws_tc.release();
  ws_bq.release();
  cmf.ws.release();
  for (IntCache& ic : icache) dfree(*this, ic.dev);
  if (rhs_exec) cudaGraphExecDestroy(rhs_exec);
  if (rhs_graph) cudaGraphDestroy(rhs_graph);
  ci.release(stream);
  if (side) cudaStreamDestroy(side);
  if (orb_state_h) pinned_put(orb_state_bytes, orb_state_h);
  for (cudaEvent_t e : {ev_fork, ev_ci, ev_join, ev_coul, ev_twoe, ev_rhs, ev_avec, ev_orb_state, ev_entry})
    if (e) cudaEventDestroy(e);
  for (cudaEvent_t e : ev_up)
    if (e) cudaEventDestroy(e);
  if (copy) cudaStreamDestroy(copy);
  if (stream && own_stream) cudaStreamDestroy(stream);
}

int cached_ints(Ctx& c, int slot, const int* h, size_t n, const int** d) {
  IntCache& ic = c.icache[slot];
  if (ic.dev && ic.host.size() == n && std::equal(h, h + n, ic.host.begin())) {
    *d = ic.dev;
    return SINCGPU_OK;
  }
  if (n > ic.cap) {
    dfree(c, ic.dev);
    ic.dev = nullptr;
    ic.cap = 0;
    SG_TRY(dalloc(c, &ic.dev, sizeof(int) * std::max<size_t>(n, 1)));
    ic.cap = n;
  }
  ic.host.assign(h, h + n);
  if (n) SG_CUDA(cudaMemcpyAsync(ic.dev, ic.host.data(), sizeof(int) * n, cudaMemcpyHostToDevice, c.stream));
  *d = ic.dev;
  return SINCGPU_OK;
}

// hermitian pair list a <= b (0-based), b-major
static void herm_pairs(int n, std::vector<int>& pa, std::vector<int>& pb) {
  pa.clear();
  pb.clear();
  for (int b = 0; b < n; ++b)
    for (int a = 0; a <= b; ++a) {
      pa.push_back(a);
      pb.push_back(b);
    }
}
static void all_pairs(int n, std::vector<int>& pa, std::vector<int>& pb) {
  pa.clear();
  pb.clear();
  for (int b = 0; b < n; ++b)
    for (int a = 0; a < n; ++a) {
      pa.push_back(a);
      pb.push_back(b);
    }
}

// Coulomb pair solves + twoematel (+ optional full twoereduced); leaves the planar
// reduced potentials of the pair list in ws_red.
int twoe_core(Ctx& c, const double2* phi1, const double2* phi2, double2* twoematel, double2* full,
              std::vector<int>& pa, std::vector<int>& pb, bool& herm) {
  herm = (phi1 == phi2);
  if (herm)
    herm_pairs(c.nspf, pa, pb);
  else
    all_pairs(c.nspf, pa, pb);
  const int npair = (int)pa.size();
  SG_TRY(c.ws_red.ensure(sizeof(double) * 2 * (size_t)npair * c.G));
  double* Rpl = (double*)c.ws_red.ptr;
  SG_TRY(coulomb_pairs(c, phi1, phi2, pa.data(), pb.data(), npair, Rpl, full, herm));
  if (twoematel) SG_TRY(twoe_matel(c, phi1, phi2, pa.data(), pb.data(), npair, Rpl, herm, twoematel));
  return SINCGPU_OK;
}

// twoematel and reducedpot of one orbital set; tally_herm when the 2-RDM is the one
// of a single A-vector (the library built it), which lets reducedpot be mirrored
int side_stream(Ctx& c) {
  if (c.side) return SINCGPU_OK;
  int cur = 0;
  SG_CUDA(cudaGetDevice(&cur));
  if (cur != c.device) SG_CUDA(cudaSetDevice(c.device));
  cudaError_t e = cudaStreamCreateWithFlags(&c.side, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&c.copy, cudaStreamNonBlocking);
  for (cudaEvent_t* ev : {&c.ev_fork, &c.ev_ci, &c.ev_join, &c.ev_coul, &c.ev_twoe, &c.ev_rhs, &c.ev_avec,
                          &c.ev_entry})
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(ev, cudaEventDisableTiming);
  for (cudaEvent_t& ev : c.ev_up)
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&ev, cudaEventDisableTiming);
  if (cur != c.device) cudaSetDevice(cur);
  SG_CUDA(e);
  return SINCGPU_OK;
}

int mean_field(Ctx& c, const double2* phi, const double2* tally, double2* twoematel, double2* reducedpot,
               bool tally_herm, cudaEvent_t tally_ready, cudaStream_t side, RpApply* apply, TwoeDefer* defer) {
  std::vector<int> pa, pb;
  bool herm;
  if (defer && !twoematel) {
    SG_TRY(twoe_core(c, phi, phi, nullptr, nullptr, pa, pb, herm));
    defer->pa = pa;
    defer->pb = pb;
    defer->herm = herm;
  } else if (side && twoematel) {
    // twoematel feeds nothing below, so it runs on `side` beside reducedpot and the
    // apply; the pair tables both read are uploaded here first (on this stream)
    SG_TRY(twoe_core(c, phi, phi, nullptr, nullptr, pa, pb, herm));
    const int* d;
    SG_TRY(cached_ints(c, IC_PA, pa.data(), pa.size(), &d));
    SG_TRY(cached_ints(c, IC_PB, pb.data(), pb.size(), &d));
    SG_CUDA(cudaEventRecord(c.ev_coul, c.stream));
    SG_CUDA(cudaStreamWaitEvent(side, c.ev_coul, 0));
    const cudaStream_t main_stream = c.stream;
    c.stream = side;
    const int rc = twoe_matel(c, phi, phi, pa.data(), pb.data(), (int)pa.size(), (const double*)c.ws_red.ptr, herm,
                              twoematel);
    c.stream = main_stream;
    SG_CUDA(cudaEventRecord(c.ev_twoe, side));
    if (rc != SINCGPU_OK) {
      cudaStreamWaitEvent(c.stream, c.ev_twoe, 0);
      return rc;
    }
  } else {
    SG_TRY(twoe_core(c, phi, phi, twoematel, nullptr, pa, pb, herm));
  }
  if (tally_ready) SG_CUDA(cudaStreamWaitEvent(c.stream, tally_ready, 0));
  return reduced_pot(c, (const double*)c.ws_red.ptr, pa.data(), pb.data(), (int)pa.size(), herm, tally,
                     reducedpot, tally_herm, apply);
}

int twoe_deferred(Ctx& c, const double2* phi, const TwoeDefer& defer, double2* twoematel, cudaEvent_t after,
                  cudaStream_t side) {
  SG_CUDA(cudaStreamWaitEvent(side, after, 0));
  const cudaStream_t main_stream = c.stream;
  c.stream = side;
  const int rc = twoe_matel(c, phi, phi, defer.pa.data(), defer.pb.data(), (int)defer.pa.size(),
                            (const double*)c.ws_red.ptr, defer.herm, twoematel);
  c.stream = main_stream;
  SG_CUDA(cudaEventRecord(c.ev_twoe, side));
  return rc;
}

int orbital_rhs(Ctx& c, const double2* phi, const double2* tally, const double2* denmat, const double2* invdenmat,
                double2 timefac, double ztdpot, double2* twoematel, double2* reducedpot, double2* out,
                bool tally_herm) {
  SG_TRY(mean_field(c, phi, tally, twoematel, reducedpot, tally_herm));
  return actreduced(c, phi, phi, denmat, invdenmat, reducedpot, timefac, 1, 1, ztdpot, out);
}

}  // namespace sincgpu

using namespace sincgpu;

extern "C" {

const char* sincgpu_last_error(void) { return g_err; }
int sincgpu_version(void) { return 100; }

static int ctx_common(sincgpu_ctx* h, int numpoints, double spacing, int numspf, int device) {
  Ctx& c = h->c;
  SG_CHECK(numpoints >= 2 && numpoints <= 128, SINCGPU_ERANGE, "numpoints %d outside [2,128]", numpoints);
  SG_CHECK(spacing > 0.0, SINCGPU_EINVAL, "spacing must be positive");
  SG_CHECK(numspf >= 1 && numspf <= 32, SINCGPU_ERANGE, "numspf %d outside [1,32]", numspf);
  c.N = numpoints;
  c.G = (long long)numpoints * numpoints * numpoints;
  c.spacing = spacing;
  c.nspf = numspf;
  c.device = device;
  SG_CUDA(cudaSetDevice(device));
  SG_TRY(upload_const_roots(device));
  SG_CUDA(cudaStreamCreateWithFlags(&c.stream, cudaStreamNonBlocking));
  c.own_stream = true;
  c.bind_workspaces();
  // memory the contexts release stays cached in the device's stream-ordered pool
  // for the next allocations instead of going back to the driver
  cudaMemPool_t pool;
  if (cudaDeviceGetDefaultMemPool(&pool, device) == cudaSuccess) {
    uint64_t keep = ~0ull;
    cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
  }
  return SINCGPU_OK;
}

int sincgpu_create(sincgpu_ctx** out, int numpoints, double spacing, int numcenters,
                   const int* centershift, const double* nuccharges, int numspf, int toothnbig,
                   int toothnsmall, int flags, int device) {
  SG_CHECK(out, SINCGPU_EINVAL, "null output pointer");
  *out = nullptr;
  SG_CHECK(numcenters >= 0 && numcenters <= 16, SINCGPU_ERANGE, "numcenters %d outside [0,16]", numcenters);
  SG_CHECK(numcenters == 0 || (centershift && nuccharges), SINCGPU_EINVAL, "null nuclear arrays");
  SG_CHECK(toothnsmall >= 1, SINCGPU_EINVAL, "toothnsmall must be >= 1");
  sincgpu_ctx* h = new sincgpu_ctx();
  int rc = ctx_common(h, numpoints, spacing, numspf, device);
  if (rc == SINCGPU_OK) {
    h->c.numcenters = numcenters;
    h->c.centershift.assign(centershift, centershift + 3 * numcenters);
    h->c.nuccharges.assign(nuccharges, nuccharges + numcenters);
    rc = build_tables(h->c, toothnbig, toothnsmall, flags);
  }
  if (rc != SINCGPU_OK) {
    delete h;
    return rc;
  }
  *out = h;
  return SINCGPU_OK;
}

int sincgpu_create_from_tables(sincgpu_ctx** out, int numpoints, double spacing, int numspf,
                               const double* threed_two, const double* pot, int device) {
  SG_CHECK(out && threed_two && pot, SINCGPU_EINVAL, "null argument");
  *out = nullptr;
  sincgpu_ctx* h = new sincgpu_ctx();
  int rc = ctx_common(h, numpoints, spacing, numspf, device);
  if (rc == SINCGPU_OK) rc = build_tables_from_arrays(h->c, (const double2*)threed_two, pot);
  if (rc != SINCGPU_OK) {
    delete h;
    return rc;
  }
  *out = h;
  return SINCGPU_OK;
}

int sincgpu_destroy(sincgpu_ctx* h) {
  if (!h) return SINCGPU_OK;
  cudaSetDevice(h->c.device);
  delete h;
  return SINCGPU_OK;
}

int sincgpu_get_tables(sincgpu_ctx* h, double* tempcoulomb, double* pot, double* kevect,
                       double* nucrepulsion) {
  CTX_CHECK(h);
  Ctx& c = h->c;
  SG_CUDA(cudaStreamSynchronize(c.stream));
  const long long W = 2LL * c.N - 1;
  if (tempcoulomb) SG_CUDA(cudaMemcpy(tempcoulomb, c.d_tcoul, sizeof(double) * W * W * W, cudaMemcpyDeviceToHost));
  if (pot) SG_CUDA(cudaMemcpy(pot, c.d_pot, sizeof(double) * c.G, cudaMemcpyDeviceToHost));
  if (kevect) SG_CUDA(cudaMemcpy(kevect, c.d_kevect, sizeof(double) * W, cudaMemcpyDeviceToHost));
  if (nucrepulsion) *nucrepulsion = c.nucrepulsion;
  return SINCGPU_OK;
}

int sincgpu_fft_length(sincgpu_ctx* h) { return h ? h->c.P : -1; }

int sincgpu_get_option(sincgpu_ctx* h, const char* name, long long* value) {
  CTX_CHECK(h);
  SG_CHECK(name && value, SINCGPU_EINVAL, "null argument");
  const Ctx& c = h->c;
  const struct {
    const char* n;
    long long v;
  } opts[] = {{"coul_chunk", c.coul_chunk},       {"coulomb_fp32", c.coul_fp32}, {"contract_tf32", c.contract_tf32},
              {"coul_tma", c.coul_tma},           {"twoe_tile", c.twoe_tile},    {"orth_fused", c.orth_fused},
              {"rhs_overlap", c.rhs_overlap},     {"coul_fused", c.coul_fused},  {"coul_z2", c.coul_z2},
              {"cmf_fp64_last", c.cmf.fp64_last ? 1 : 0}, {"rhs_upload_groups", c.up_groups}, {"kry_cluster", c.kry_cluster}, {"orb_blendq", c.orb_blendq}, {"ke_tf32", c.ke_tf32}, {"tc_kc", c.tc_kc}, {"tc_pipe", c.tc_pipe}, {"twoe_symdiag", c.twoe_symdiag}, {"twoe_dmma", c.twoe_dmma}, {"rp_dmma", c.rp_dmma}};
  for (const auto& o : opts)
    if (!strcmp(name, o.n)) {
      *value = o.v;
      return SINCGPU_OK;
    }
  SG_CHECK(false, SINCGPU_EINVAL, "unknown option '%s'", name);
  return SINCGPU_EINVAL;
}

int sincgpu_set_option(sincgpu_ctx* h, const char* name, long long value) {
  CTX_CHECK(h);
  SG_CHECK(name, SINCGPU_EINVAL, "null option name");
  if (!strcmp(name, "coul_chunk")) {
    SG_CHECK(value >= 0, SINCGPU_EINVAL, "coul_chunk must be >= 0");
    h->c.coul_chunk = (int)value;
    return SINCGPU_OK;
  }
  if (!strcmp(name, "coulomb_fp32")) {
    SG_CHECK(value == 0 || value == 1, SINCGPU_EINVAL, "coulomb_fp32 must be 0 or 1");
    if (value) SG_TRY(ensure_fp32_tables(h->c));
    h->c.coul_fp32 = (int)value;
    return SINCGPU_OK;
  }
  if (!strcmp(name, "rhs_overlap")) {
    SG_CHECK(value == 0 || value == 1, SINCGPU_EINVAL, "rhs_overlap must be 0 or 1");
    h->c.rhs_overlap = (int)value;
    return SINCGPU_OK;
  }
  if (!strcmp(name, "orb_blendq")) {
    SG_CHECK(value == 0 || value == 1, SINCGPU_EINVAL, "orb_blendq must be 0 or 1");
    h->c.orb_blendq = (int)value;
    return SINCGPU_OK;
  }
  if (!strcmp(name, "kry_cluster")) {
    SG_CHECK(value == 0 || value == 1, SINCGPU_EINVAL, "kry_cluster must be 0 or 1");
    h->c.kry_cluster = (int)value;
    return SINCGPU_OK;
  }
  if (!strcmp(name, "rhs_upload_groups")) {
    SG_CHECK(value >= 1 && value <= Ctx::kUpGroups, SINCGPU_EINVAL, "rhs_upload_groups must be 1..%d",
             Ctx::kUpGroups);
    h->c.up_groups = (int)value;
    return SINCGPU_OK;
  }
  if (!strcmp(name, "orth_fused")) {
    SG_CHECK(value == 0 || value == 1, SINCGPU_EINVAL, "orth_fused must be 0 or 1");
    h->c.orth_fused = (int)value;
    return SINCGPU_OK;
  }
  if (!strcmp(name, "twoe_tile")) {
    SG_CHECK(value == 0 || (value >= 2 && value <= 9), SINCGPU_EINVAL, "twoe_tile must be 0 or 2..9");
    h->c.twoe_tile = (int)value;
    return SINCGPU_OK;
  }
  if (!strcmp(name, "twoe_dmma")) {
    SG_CHECK(value == 0 || value == 1, SINCGPU_EINVAL, "twoe_dmma must be 0 or 1");
    h->c.twoe_dmma = (int)value;
    return SINCGPU_OK;
  }
  if (!strcmp(name, "rp_dmma")) {
    SG_CHECK(value == 0 || value == 1, SINCGPU_EINVAL, "rp_dmma must be 0 or 1");
    h->c.rp_dmma = (int)value;
    return SINCGPU_OK;
  }
  if (!strcmp(name, "twoe_symdiag")) {
    SG_CHECK(value == 0 || value == 1, SINCGPU_EINVAL, "twoe_symdiag must be 0 or 1");
    h->c.twoe_symdiag = (int)value;
    return SINCGPU_OK;
  }
  if (!strcmp(name, "tc_pipe")) {
    SG_CHECK(value >= 0 && value <= 5, SINCGPU_EINVAL, "tc_pipe must be 0 (two stages, no ring), 1 (ring of 3 x 16), "
             "2 (4 x 16), 3 (6 x 8), 4 or 5 (pre-split operands, bulk copies into 3 or 5 stages)");
    h->c.tc_pipe = (int)value;
    return SINCGPU_OK;
  }
  if (!strcmp(name, "tc_kc")) {
    SG_CHECK(value == 16 || value == 32, SINCGPU_EINVAL, "tc_kc must be 16 or 32");
    h->c.tc_kc = (int)value;
    return SINCGPU_OK;
  }
  if (!strcmp(name, "ke_tf32")) {
    SG_CHECK(value == 0 || value == 1, SINCGPU_EINVAL, "ke_tf32 must be 0 or 1");
    h->c.ke_tf32 = (int)value;
    return SINCGPU_OK;
  }
  if (!strcmp(name, "coul_z2")) {
    SG_CHECK(value == 0 || value == 1, SINCGPU_EINVAL, "coul_z2 must be 0 or 1");
    h->c.coul_z2 = (int)value;
    return SINCGPU_OK;
  }
  if (!strcmp(name, "coul_fused")) {
    SG_CHECK(value >= -1 && value <= 1, SINCGPU_EINVAL, "coul_fused must be -1, 0 or 1");
    h->c.coul_fused = (int)value;
    return SINCGPU_OK;
  }
  if (!strcmp(name, "coul_tma")) {
    SG_CHECK(value >= -1 && value <= 1, SINCGPU_EINVAL, "coul_tma must be -1, 0 or 1");
    h->c.coul_tma = (int)value;
    return SINCGPU_OK;
  }
  if (!strcmp(name, "cmf_fp64_last")) {
    SG_CHECK(value == 0 || value == 1, SINCGPU_EINVAL, "cmf_fp64_last must be 0 or 1");
    h->c.cmf.fp64_last = value != 0;
    return SINCGPU_OK;
  }
  if (!strcmp(name, "contract_tf32")) {
    SG_CHECK(value == 0 || value == 1, SINCGPU_EINVAL, "contract_tf32 must be 0 or 1");
    h->c.contract_tf32 = (int)value;
    return SINCGPU_OK;
  }
  set_error("unknown option '%s'", name);
  return SINCGPU_EINVAL;
}

int sincgpu_synchronize(sincgpu_ctx* h) {
  CTX_CHECK(h);
  SG_CUDA(cudaStreamSynchronize(h->c.stream));
  return SINCGPU_OK;
}

int sincgpu_set_sync_mode(int device, int mode) {
  static const unsigned flags[] = {cudaDeviceScheduleAuto, cudaDeviceScheduleSpin, cudaDeviceScheduleYield,
                                   cudaDeviceScheduleBlockingSync};
  SG_CHECK(mode >= 0 && mode <= 3, SINCGPU_EINVAL, "sync mode %d outside [0,3]", mode);
  SG_CUDA(cudaSetDevice(device));
  SG_CUDA(cudaSetDeviceFlags(flags[mode]));
  return SINCGPU_OK;
}

int sincgpu_set_stream(sincgpu_ctx* h, void* stream) {
  CTX_CHECK(h);
  Ctx& c = h->c;
  // workspaces are stream-ordered on the context's stream: finish the old
  // stream's work before later frees are ordered on the new one
  if (c.stream) SG_CUDA(cudaStreamSynchronize(c.stream));
  if (c.own_stream && c.stream) SG_CUDA(cudaStreamDestroy(c.stream));
  c.own_stream = false;
  c.stream = (cudaStream_t)stream;
  return SINCGPU_OK;
}

long long sincgpu_launch_count(void) { return g_launches.load(); }

int sincgpu_profile(sincgpu_ctx* h, int enable) {
  CTX_CHECK(h);
  h->c.prof.on = enable != 0;
  return SINCGPU_OK;
}

int sincgpu_profile_read(sincgpu_ctx* h, double* ms, long long* launches, int nstage) {
  CTX_CHECK(h);
  Ctx& c = h->c;
  SG_CUDA(cudaStreamSynchronize(c.stream));
  for (auto& r : c.prof.recs) {
    float t = 0.f;
    cudaEventElapsedTime(&t, r.a, r.b);
    c.prof.ms[r.stage] += t;
    c.prof.launches[r.stage] += 1;
    cudaEventDestroy(r.a);
    cudaEventDestroy(r.b);
  }
  c.prof.recs.clear();
  for (int i = 0; i < nstage && i < ST_COUNT; ++i) {
    if (ms) ms[i] = c.prof.ms[i];
    if (launches) launches[i] = c.prof.launches[i];
    c.prof.ms[i] = 0.0;
    c.prof.launches[i] = 0;
  }
  return SINCGPU_OK;
}

int sincgpu_host_register(void* ptr, long long bytes) {
  SG_CHECK(ptr && bytes > 0, SINCGPU_EINVAL, "bad host range");
  SG_CUDA(cudaHostRegister(ptr, (size_t)bytes, cudaHostRegisterDefault));
  return SINCGPU_OK;
}
int sincgpu_host_unregister(void* ptr) {
  SG_CUDA(cudaHostUnregister(ptr));
  return SINCGPU_OK;
}

// ---------------------------------------------------------------------------
// device-resident forms
// ---------------------------------------------------------------------------
int sincgpu_twoe_matel_dev(sincgpu_ctx* h, const double* phi1, const double* phi2, double* twoematel,
                           double* twoereduced) {
  CTX_CHECK(h);
  SG_CHECK(phi1 && phi2 && twoematel, SINCGPU_EINVAL, "null argument");
  std::vector<int> pa, pb;
  bool herm;
  return twoe_core(h->c, (const double2*)phi1, (const double2*)phi2, (double2*)twoematel,
                   (double2*)twoereduced, pa, pb, herm);
}

int sincgpu_mult_ke_dev(sincgpu_ctx* h, const double* in, double* out, int howmany) {
  CTX_CHECK(h);
  SG_CHECK(in && out && in != out, SINCGPU_EINVAL, "in/out must be distinct, non-null");
  SG_CHECK(howmany >= 0, SINCGPU_EINVAL, "howmany < 0");
  if (howmany == 0) return SINCGPU_OK;
  return mult_ke(h->c, (const double2*)in, (double2*)out, howmany, false, 0.0);
}

int sincgpu_mult_reducedpot_dev(sincgpu_ctx* h, const double* inspfs, double* outspfs,
                                const double* reducedpot) {
  CTX_CHECK(h);
  SG_CHECK(inspfs && outspfs && reducedpot, SINCGPU_EINVAL, "null argument");
  return mult_reducedpot(h->c, (const double2*)inspfs, (const double2*)reducedpot, (double2*)outspfs);
}


int sincgpu_mean_field_dev(sincgpu_ctx* h, const double* phi, const double* tally, double* twoematel,
                           double* reducedpot) {
  CTX_CHECK(h);
  SG_CHECK(phi && tally && reducedpot, SINCGPU_EINVAL, "null argument");
  return mean_field(h->c, (const double2*)phi, (const double2*)tally, (double2*)twoematel, (double2*)reducedpot,
                    false);
}

int sincgpu_actreduced_dev(sincgpu_ctx* h, int dentimeflag, const double* inspfs, const double* projspfs,
                           const double* denmat, const double* invdenmat, const double* reducedpot,
                           double tre, double tim, int projflag, double ztdpot, double* out) {
  CTX_CHECK(h);
  SG_CHECK(inspfs && denmat && reducedpot && out, SINCGPU_EINVAL, "null argument");
  SG_CHECK(!dentimeflag || invdenmat, SINCGPU_EINVAL, "invdenmat required with dentimeflag");
  SG_CHECK(projflag != 1 || projspfs, SINCGPU_EINVAL, "projspfs required with projflag=1");
  SG_CHECK(out != inspfs, SINCGPU_EINVAL, "outspfs must not alias inspfs");
  return actreduced(h->c, (const double2*)inspfs, (const double2*)projspfs, (const double2*)denmat,
                    (const double2*)invdenmat, (const double2*)reducedpot, make_double2(tre, tim),
                    dentimeflag, projflag, ztdpot, (double2*)out);
}

int sincgpu_orbital_rhs_dev(sincgpu_ctx* h, const double* phi, const double* tally, const double* denmat,
                            const double* invdenmat, double tre, double tim, double ztdpot,
                            double* twoematel, double* reducedpot, double* out) {
  CTX_CHECK(h);
  SG_CHECK(phi && tally && denmat && invdenmat && reducedpot && out, SINCGPU_EINVAL, "null argument");
  SG_CHECK(out != phi, SINCGPU_EINVAL, "out must not alias phi");
  return orbital_rhs(h->c, (const double2*)phi, (const double2*)tally, (const double2*)denmat,
                     (const double2*)invdenmat, make_double2(tre, tim), ztdpot, (double2*)twoematel,
                     (double2*)reducedpot, (double2*)out, false);
}

// ---------------------------------------------------------------------------
// host-array drop-ins: stage through ws_io
// ---------------------------------------------------------------------------
struct Staging {
  Ctx& c;
  size_t off = 0;
  explicit Staging(Ctx& cc) : c(cc) {}
  size_t add(size_t bytes) {
    size_t o = off;
    off += (bytes + 255) / 256 * 256;
    return o;
  }
  char* at(size_t o) { return (char*)c.ws_io.ptr + o; }
};

static int up(Ctx& c, void* dst, const void* src, size_t bytes) {
  SG_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, c.stream));
  return SINCGPU_OK;
}
static int down(Ctx& c, void* dst, const void* src, size_t bytes) {
  SG_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, c.stream));
  return SINCGPU_OK;
}

int sincgpu_call_twoe_matel00(sincgpu_ctx* h, int lowspf, int highspf, const double* in10,
                              const double* in20, double* twoematel, double* twoereduced) {
  CTX_CHECK(h);
  Ctx& c = h->c;
  const int n = c.nspf;
  SG_CHECK(in10 && in20 && twoematel && twoereduced, SINCGPU_EINVAL, "null argument");
  if (highspf - lowspf + 1 <= 0) return SINCGPU_OK;  // coreproject.f90:968-971
  SG_CHECK(lowspf == 1 && highspf == n, SINCGPU_EINVAL,
           "orbital range %d:%d must be 1:%d (single-rank build)", lowspf, highspf, n);
  const bool same = (in10 == in20);
  const size_t bphi = sizeof(double2) * (size_t)c.G * n;
  const size_t bmat = sizeof(double2) * (size_t)n * n * n * n;
  const size_t bred = sizeof(double2) * (size_t)c.G * n * n;
  Staging s(c);
  size_t o1 = s.add(bphi), o2 = same ? o1 : s.add(bphi), om = s.add(bmat), orr = s.add(bred);
  SG_TRY(c.ws_io.ensure(s.off));
  double2* d1 = (double2*)s.at(o1);
  double2* d2 = (double2*)s.at(o2);
  SG_TRY(up(c, d1, in10, bphi));
  if (!same) SG_TRY(up(c, d2, in20, bphi));
  std::vector<int> pa, pb;
  bool herm;
  SG_TRY(twoe_core(c, d1, d2, (double2*)s.at(om), (double2*)s.at(orr), pa, pb, herm));
  SG_TRY(down(c, twoematel, s.at(om), bmat));
  SG_TRY(down(c, twoereduced, s.at(orr), bred));
  SG_CUDA(cudaStreamSynchronize(c.stream));
  return SINCGPU_OK;
}

int sincgpu_op_tinv(sincgpu_ctx* h, const double* dens, double* red, int allsize, int circsize) {
  CTX_CHECK(h);
  Ctx& c = h->c;
  SG_CHECK(dens && red, SINCGPU_EINVAL, "null argument");
  SG_CHECK(allsize >= 0 && circsize >= 1 && allsize % circsize == 0, SINCGPU_EINVAL,
           "SIZE ERROR OP_TINV %d %d", allsize, circsize);  // coreproject.f90:389-391
  if (allsize == 0) return SINCGPU_OK;
  const size_t b = sizeof(double2) * (size_t)c.G * allsize;
  Staging s(c);
  size_t oi = s.add(b), oo = s.add(b);
  SG_TRY(c.ws_io.ensure(s.off));
  SG_TRY(up(c, s.at(oi), dens, b));
  SG_TRY(coulomb_dens(c, (const double2*)s.at(oi), allsize, (double2*)s.at(oo)));
  SG_TRY(down(c, red, s.at(oo), b));
  SG_CUDA(cudaStreamSynchronize(c.stream));
  return SINCGPU_OK;
}

int sincgpu_mult_ke(sincgpu_ctx* h, const double* in, double* out, int howmany) {
  CTX_CHECK(h);
  Ctx& c = h->c;
  SG_CHECK(in && out, SINCGPU_EINVAL, "null argument");
  SG_CHECK(howmany >= 0, SINCGPU_EINVAL, "howmany < 0");
  if (howmany == 0) return SINCGPU_OK;
  const size_t b = sizeof(double2) * (size_t)c.G * howmany;
  Staging s(c);
  size_t oi = s.add(b), oo = s.add(b);
  SG_TRY(c.ws_io.ensure(s.off));
  SG_TRY(up(c, s.at(oi), in, b));
  SG_TRY(mult_ke(c, (const double2*)s.at(oi), (double2*)s.at(oo), howmany, false, 0.0));
  SG_TRY(down(c, out, s.at(oo), b));
  SG_CUDA(cudaStreamSynchronize(c.stream));
  return SINCGPU_OK;
}

int sincgpu_mult_reducedpot(sincgpu_ctx* h, int firstspf, int lastspf, const double* inspfs,
                            double* outspfs, const double* reducedpot) {
  CTX_CHECK(h);
  Ctx& c = h->c;
  const int n = c.nspf;
  SG_CHECK(inspfs && outspfs && reducedpot, SINCGPU_EINVAL, "null argument");
  SG_CHECK(firstspf >= 1 && lastspf <= n, SINCGPU_EINVAL, "orbital range %d:%d outside 1:%d", firstspf,
           lastspf, n);
  const int ni = lastspf - firstspf + 1;
  if (ni <= 0) return SINCGPU_OK;
  const size_t bphi = sizeof(double2) * (size_t)c.G * n;
  const size_t bout = sizeof(double2) * (size_t)c.G * ni;
  const size_t bv = sizeof(double2) * (size_t)c.G * n * ni;
  Staging s(c);
  size_t op = s.add(bphi), oo = s.add(bout), ov = s.add(bv);
  SG_TRY(c.ws_io.ensure(s.off));
  SG_TRY(up(c, s.at(op), inspfs, bphi));
  SG_TRY(up(c, s.at(ov), reducedpot, bv));
  SG_TRY(mult_reducedpot_range(c, (const double2*)s.at(op), (const double2*)s.at(ov), firstspf - 1, ni,
                               (double2*)s.at(oo)));
  SG_TRY(down(c, outspfs, s.at(oo), bout));
  SG_CUDA(cudaStreamSynchronize(c.stream));
  return SINCGPU_OK;
}

int sincgpu_get_reducedpot(sincgpu_ctx* h, const double* twoereduced, const double* tally,
                           double* reducedpot) {
  CTX_CHECK(h);
  Ctx& c = h->c;
  const int n = c.nspf;
  SG_CHECK(twoereduced && tally && reducedpot, SINCGPU_EINVAL, "null argument");
  const size_t bred = sizeof(double2) * (size_t)c.G * n * n;
  const size_t bt = sizeof(double2) * (size_t)n * n * n * n;
  Staging s(c);
  size_t orr = s.add(bred), ot = s.add(bt), oo = s.add(bred);
  SG_TRY(c.ws_io.ensure(s.off));
  SG_TRY(up(c, s.at(orr), twoereduced, bred));
  SG_TRY(up(c, s.at(ot), tally, bt));
  SG_TRY(reduced_pot_full(c, (const double2*)s.at(orr), (const double2*)s.at(ot), (double2*)s.at(oo)));
  SG_TRY(down(c, reducedpot, s.at(oo), bred));
  SG_CUDA(cudaStreamSynchronize(c.stream));
  return SINCGPU_OK;
}

int sincgpu_actreduced00(sincgpu_ctx* h, int dentimeflag, const double* inspfs, const double* projspfs,
                         const double* denmat, const double* invdenmat, const double* reducedpot,
                         double tre, double tim, int projflag, double ztdpot, double* outspfs) {
  CTX_CHECK(h);
  Ctx& c = h->c;
  const int n = c.nspf;
  SG_CHECK(inspfs && denmat && reducedpot && outspfs, SINCGPU_EINVAL, "null argument");
  SG_CHECK(!dentimeflag || invdenmat, SINCGPU_EINVAL, "invdenmat required with dentimeflag");
  SG_CHECK(projflag != 1 || projspfs, SINCGPU_EINVAL, "projspfs required with projflag=1");
  const size_t bphi = sizeof(double2) * (size_t)c.G * n;
  const size_t bm = sizeof(double2) * (size_t)n * n;
  const size_t bv = sizeof(double2) * (size_t)c.G * n * n;
  Staging s(c);
  size_t oi = s.add(bphi), op = s.add(bphi), od = s.add(bm), oinv = s.add(bm), ov = s.add(bv),
         oo = s.add(bphi);
  SG_TRY(c.ws_io.ensure(s.off));
  SG_TRY(up(c, s.at(oi), inspfs, bphi));
  if (projflag == 1) SG_TRY(up(c, s.at(op), projspfs, bphi));
  SG_TRY(up(c, s.at(od), denmat, bm));
  if (dentimeflag) SG_TRY(up(c, s.at(oinv), invdenmat, bm));
  SG_TRY(up(c, s.at(ov), reducedpot, bv));
  SG_TRY(actreduced(c, (const double2*)s.at(oi), (const double2*)s.at(op), (const double2*)s.at(od),
                    (const double2*)s.at(oinv), (const double2*)s.at(ov), make_double2(tre, tim),
                    dentimeflag, projflag, ztdpot, (double2*)s.at(oo)));
  SG_TRY(down(c, outspfs, s.at(oo), bphi));
  SG_CUDA(cudaStreamSynchronize(c.stream));
  return SINCGPU_OK;
}

}  // extern "C"

extern "C" int sincgpu_orbital_rhs(sincgpu_ctx* h, const double* phi, const double* tally,
                                   const double* denmat, const double* invdenmat, double tre,
                                   double tim, double ztdpot, double* twoematel, double* out) {
  CTX_CHECK(h);
  Ctx& c = h->c;
  const int n = c.nspf;
  SG_CHECK(phi && tally && denmat && invdenmat && out, SINCGPU_EINVAL, "null argument");
  const size_t bphi = sizeof(double2) * (size_t)c.G * n;
  const size_t bt = sizeof(double2) * (size_t)n * n * n * n;
  const size_t bm = sizeof(double2) * (size_t)n * n;
  Staging s(c);
  size_t op = s.add(bphi), ot = s.add(bt), od = s.add(bm), oi = s.add(bm), om = s.add(bt), oo = s.add(bphi);
  SG_TRY(c.ws_io.ensure(s.off));
  SG_TRY(c.ws_state.ensure(sizeof(double2) * (size_t)c.G * n * n));
  SG_TRY(up(c, s.at(op), phi, bphi));
  SG_TRY(up(c, s.at(ot), tally, bt));
  SG_TRY(up(c, s.at(od), denmat, bm));
  SG_TRY(up(c, s.at(oi), invdenmat, bm));
  SG_TRY(sincgpu_orbital_rhs_dev(h, (const double*)s.at(op), (const double*)s.at(ot), (const double*)s.at(od),
                                 (const double*)s.at(oi), tre, tim, ztdpot, (double*)s.at(om),
                                 (double*)c.ws_state.ptr, (double*)s.at(oo)));
  if (twoematel) SG_TRY(down(c, twoematel, s.at(om), bt));
  SG_TRY(down(c, out, s.at(oo), bphi));
  SG_CUDA(cudaStreamSynchronize(c.stream));
  return SINCGPU_OK;
}
