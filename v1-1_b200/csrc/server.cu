// Device-resident request loop (the served form of the CMF propagation).
//
// Clients submit propagation requests (grid, nuclei, orbitals, electrons,
// pulses, number of steps, initial orbitals and A-vector).  A fixed pool of
// worker threads admits pending requests while both a slot and the HBM budget
// allow it (continuous batching: a request that arrives while others run is
// admitted as soon as one finishes and frees its slot and memory), builds its
// context (tables, walk tables with spin sets, CMF state) and steps it to the
// end.  Every live request owns a context with its own non-blocking stream and
// device buffers, so the requests' kernels overlap on the device, and the
// deterministic kernels give each request the same result alone or in a mix.
// Per-step latency is the host wall time of each CMF step (which ends in a
// synchronisation); the server keeps all step latencies for p50/p99.
#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <thread>
#include <vector>
#include "context.hpp"
#include "walks.hpp"
#include "../../include/sincgpu.h"

namespace {

struct Req {
  int id = 0;
  int N = 0;
  double spacing = 0.0;
  std::vector<int> cs;
  std::vector<double> z;
  int nspf = 0, numelec = 0, restrictms = 0, spinrestrictval = -1;
  std::vector<int> ptype;
  std::vector<double> pparams;
  int nsteps = 0;
  double dt = 0.05;
  int fp32 = 0, keep_state = 0;
  std::vector<double> phi, avec;
  long long est = 0;
  double t_submit = 0.0;
};

struct Res {
  int status = SINCGPU_OK;
  char err[256] = "";
  double energy0 = 0.0, energy = 0.0, norm = 0.0, dipole = 0.0, wait_ms = 0.0;
  double t_submit = 0.0, t_admit = 0.0, t_ready = 0.0, t_end = 0.0;  // ms since server creation
  std::vector<double> step_ms, energies, step_start;
  std::vector<double> phi, avec;
  bool done = false;
};

double now_ms() {
  using namespace std::chrono;
  return duration<double, std::milli>(steady_clock::now().time_since_epoch()).count();
}

long long binom(int n, int k) {
  if (k < 0 || k > n) return 0;
  long long r = 1;
  for (int i = 1; i <= k; ++i) r = r * (n - k + i) / i;
  return r;
}

// device bytes a request will hold (dominant terms, generous)
long long estimate_bytes(const Req& r) {
  const long long G = (long long)r.N * r.N * r.N, n = r.nspf;
  const long long npair = n * (n + 1) / 2;
  const int na = (r.numelec + r.restrictms) / 2, nb = r.numelec - na;
  const long long nc = binom(r.nspf, na) * binom(r.nspf, nb);
  long long P = 2 * r.N;  // upper bound of the padded length
  long long b = 0;
  b += 16 * G * n * (2 + 25);                 // orbitals (2 slots) + Krylov basis and Jacobian state
  b += 16 * G * n * n * 4;                    // reducedpot (2 slots), their blend for the Jacobian, scratch
  b += 8 * 2 * npair * G;                     // planar reduced potentials
  b += std::min(sincgpu::kCoulChunkBudget, npair * 16 * (r.N * r.N * P + r.N * P * P));  // Coulomb W1/W2 chunk
  b += 16 * P * P * P;                        // kernel spectrum
  b += 16 * G * n * 6;                        // RHS temporaries
  const long long walks = nc * (long long)(r.numelec * r.nspf + r.numelec * r.numelec * r.nspf * r.nspf / 2);
  b += walks * 24 + nc * 16 * 260;            // walk tables, assembled matrices, A-vector Krylov
  return b + (64ll << 20);
}

}  // namespace

struct sincgpu_server {
  int device = 0;
  long long budget = 0, reserved = 0;
  int max_active = 1, active = 0, peak_active = 0;
  std::mutex mu;
  std::condition_variable cv_work, cv_done;
  std::deque<Req*> pending;
  std::map<int, std::unique_ptr<Req>> reqs;
  std::map<int, std::unique_ptr<Res>> res;
  std::vector<std::thread> workers;
  bool stop = false;
  int next_id = 1;
  double t0 = 0.0;  // creation time (now_ms)
  long long admitted = 0, completed = 0;
  double t_first = -1.0, t_last = 0.0;

  void worker();
  void run(Req& r, Res& out);
};

void sincgpu_server::run(Req& r, Res& out) {
  using namespace sincgpu;
  sincgpu_ctx* ctx = nullptr;
  sincgpu_walks* walks = nullptr;
  double* dphi = nullptr;
  double* davec = nullptr;
  auto fail = [&](int rc) {
    out.status = rc;
    std::snprintf(out.err, sizeof(out.err), "%s", sincgpu_last_error());
  };
  int rc = sincgpu_create(&ctx, r.N, r.spacing, (int)r.z.size(), r.cs.data(), r.z.data(), r.nspf, 240, 40, 0,
                          device);
  // the walk-table build of one request uses its share of the host cores, so that
  // the other requests' host loops (one synchronisation per Arnoldi step) are not
  // starved while it runs
  const int host_threads = std::max(1, (int)std::thread::hardware_concurrency() / std::max(1, max_active));
  if (rc == SINCGPU_OK) rc = sincgpu_walks_create(&walks, r.numelec, r.nspf, r.restrictms, host_threads);
  if (rc == SINCGPU_OK) rc = sincgpu_walks_spin(walks, r.spinrestrictval);
  if (rc == SINCGPU_OK) rc = sincgpu_ci_attach(ctx, walks);
  const long long G = (long long)r.N * r.N * r.N;
  const int nc = walks ? walks->w.numconfig : 0;
  if (rc == SINCGPU_OK && r.fp32) rc = sincgpu_set_option(ctx, "coulomb_fp32", 1);
  if (rc == SINCGPU_OK && r.fp32) rc = sincgpu_set_option(ctx, "contract_tf32", 1);
  // requests share the GPU: a cooperative launch waits until all of its CTAs fit
  // at once, which would hold every other request's kernels back
  if (rc == SINCGPU_OK) rc = sincgpu_set_option(ctx, "orth_fused", 0);
  if (rc == SINCGPU_OK)
    rc = sincgpu_cmf_setup(ctx, r.dt, 1, 1e-8, 1e-9, 30, 100, 10, 100, 1.2, 1e-10, 0.0, -1.0);
  if (rc == SINCGPU_OK)
    rc = sincgpu_cmf_pulses(ctx, (int)r.ptype.size(), r.ptype.data(), r.pparams.data());
  // the request's state buffers are stream-ordered on its context's stream, so
  // neither their allocation nor their release synchronises the other requests
  if (rc == SINCGPU_OK) {
    if (dalloc(ctx->c, &dphi, sizeof(double) * 2 * G * r.nspf) != SINCGPU_OK ||
        dalloc(ctx->c, &davec, sizeof(double) * 2 * nc) != SINCGPU_OK) {
      set_error("out of device memory for the initial state");
      rc = SINCGPU_ENOMEM;
    }
  }
  if (rc == SINCGPU_OK && (long long)r.phi.size() != 2 * G * r.nspf) {
    set_error("initial orbitals have %zu doubles, expected %lld", r.phi.size(), 2 * G * r.nspf);
    rc = SINCGPU_EINVAL;
  }
  if (rc == SINCGPU_OK && (long long)r.avec.size() != 2LL * nc) {
    set_error("initial A-vector has %zu doubles, expected %d", r.avec.size(), 2 * nc);
    rc = SINCGPU_EINVAL;
  }
  if (rc == SINCGPU_OK) {
    cudaMemcpyAsync(dphi, r.phi.data(), sizeof(double) * r.phi.size(), cudaMemcpyHostToDevice, ctx->c.stream);
    cudaMemcpyAsync(davec, r.avec.data(), sizeof(double) * r.avec.size(), cudaMemcpyHostToDevice,
                    ctx->c.stream);
    rc = sincgpu_cmf_init_dev(ctx, dphi, davec, &out.energy0);
  }
  out.t_ready = now_ms() - this->t0;
  for (int k = 0; rc == SINCGPU_OK && k < r.nsteps; ++k) {
    const double t0 = now_ms();
    out.step_start.push_back(t0 - this->t0);
    double e = 0.0, nn = 0.0;
    rc = sincgpu_cmf_step(ctx, r.dt * k, r.dt * (k + 1), &e, &nn, nullptr, nullptr);
    out.step_ms.push_back(now_ms() - t0);
    out.energies.push_back(e);
    out.energy = e;
    out.norm = nn;
  }
  if (rc == SINCGPU_OK) {
    // a tensor-core contraction or a staged Coulomb pass that gave up a bounded
    // wait has left a wrong result behind: the request fails
    int flags[2] = {0, 0};
    rc = sincgpu_kernel_timeouts(ctx, flags);
    if (rc == SINCGPU_OK && (flags[0] || flags[1])) {
      set_error("a %s gave up a bounded wait during the request",
                flags[0] ? "tensor-core contraction" : "staged Coulomb pass");
      rc = SINCGPU_ETIMEOUT;
    }
  }
  if (rc == SINCGPU_OK) {
    double d[2], nn;
    rc = sincgpu_cmf_dipole_z(ctx, d, &nn);
    out.dipole = nn > 0 ? d[0] / nn : 0.0;
  }
  if (rc == SINCGPU_OK && r.keep_state) {
    out.phi.resize(2 * G * r.nspf);
    out.avec.resize(2 * (size_t)nc);
    rc = sincgpu_cmf_state_dev(ctx, dphi, davec);
    if (rc == SINCGPU_OK) {
      cudaMemcpyAsync(out.phi.data(), dphi, sizeof(double) * out.phi.size(), cudaMemcpyDeviceToHost,
                      ctx->c.stream);
      cudaMemcpyAsync(out.avec.data(), davec, sizeof(double) * out.avec.size(), cudaMemcpyDeviceToHost,
                      ctx->c.stream);
      cudaStreamSynchronize(ctx->c.stream);
    }
  }
  if (rc != SINCGPU_OK) fail(rc);
  if (ctx) {
    dfree(ctx->c, dphi);
    dfree(ctx->c, davec);
  }
  if (walks) sincgpu_walks_destroy(walks);
  if (ctx) sincgpu_destroy(ctx);
}

void sincgpu_server::worker() {
  cudaSetDevice(device);
  while (true) {
    Req* r = nullptr;
    {
      std::unique_lock<std::mutex> lk(mu);
      cv_work.wait(lk, [&] {
        if (stop && pending.empty()) return true;
        for (Req* q : pending)
          if (reserved + q->est <= budget || active == 0) return true;
        return false;
      });
      if (stop && pending.empty()) return;
      // first pending request that fits the budget (any request when nothing runs)
      for (auto it = pending.begin(); it != pending.end(); ++it)
        if (reserved + (*it)->est <= budget || active == 0) {
          r = *it;
          pending.erase(it);
          break;
        }
      if (!r) continue;
      reserved += r->est;
      ++active;
      ++admitted;
      peak_active = std::max(peak_active, active);
      if (t_first < 0) t_first = now_ms();
    }
    auto out = std::make_unique<Res>();
    out->wait_ms = now_ms() - r->t_submit;
    out->t_submit = r->t_submit - t0;
    out->t_admit = now_ms() - t0;
    run(*r, *out);
    out->t_end = now_ms() - t0;
    {
      std::lock_guard<std::mutex> lk(mu);
      reserved -= r->est;
      --active;
      ++completed;
      t_last = now_ms();
      out->done = true;
      res[r->id] = std::move(out);
      r->phi.clear();
      r->phi.shrink_to_fit();
      r->avec.clear();
      r->avec.shrink_to_fit();
    }
    cv_done.notify_all();
    cv_work.notify_all();
  }
}

extern "C" {

int sincgpu_server_create(sincgpu_server** out, int device, long long hbm_budget, int max_active) {
  using namespace sincgpu;
  SG_CHECK(out && max_active >= 1 && max_active <= 64, SINCGPU_EINVAL, "bad argument");
  SG_CUDA(cudaSetDevice(device));
  // memory cached in the stream-ordered pool by earlier contexts counts as free
  cudaMemPool_t pool = nullptr;
  if (cudaDeviceGetDefaultMemPool(&pool, device) == cudaSuccess) {
    SG_CUDA(cudaDeviceSynchronize());
    cudaMemPoolTrimTo(pool, 0);
  } else {
    pool = nullptr;
  }
  size_t fr = 0, tot = 0;
  SG_CUDA(cudaMemGetInfo(&fr, &tot));
  auto s = std::make_unique<sincgpu_server>();
  s->device = device;
  s->budget = hbm_budget > 0 ? std::min<long long>(hbm_budget, (long long)fr) : (long long)(0.85 * fr);
  // The budget is reserved in the stream-ordered pool up front: the requests'
  // device allocations are then carved out of memory the pool already holds.
  // Growing the pool maps new physical memory in a driver call that can take tens
  // of milliseconds, during which the other requests' host threads stalled.
  if (pool) {
    uint64_t keep = ~0ull;
    cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
    cudaStream_t st = nullptr;
    void* p = nullptr;
    if (cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) == cudaSuccess) {
      if (cudaMallocFromPoolAsync(&p, (size_t)s->budget, pool, st) == cudaSuccess) cudaFreeAsync(p, st);
      cudaStreamSynchronize(st);
      cudaStreamDestroy(st);
    }
    cudaGetLastError();
  }
  s->max_active = max_active;
  s->t0 = now_ms();
  for (int i = 0; i < max_active; ++i) s->workers.emplace_back([p = s.get()] { p->worker(); });
  *out = s.release();
  return SINCGPU_OK;
}

int sincgpu_server_submit(sincgpu_server* s, const sincgpu_request* q, int* id) {
  using namespace sincgpu;
  SG_CHECK(s && q && id && q->phi && q->avector && q->numcenters >= 1, SINCGPU_EINVAL, "bad argument");
  SG_CHECK(q->numelec >= 1 && q->numspf >= 1 && q->nsteps >= 0 && q->dt > 0, SINCGPU_EINVAL, "bad request");
  auto r = std::make_unique<Req>();
  r->N = q->numpoints;
  r->spacing = q->spacing;
  r->cs.assign(q->centershift, q->centershift + 3 * q->numcenters);
  r->z.assign(q->nuccharges, q->nuccharges + q->numcenters);
  r->nspf = q->numspf;
  r->numelec = q->numelec;
  r->restrictms = q->restrictms;
  r->spinrestrictval = q->spinrestrictval;
  if (q->npulses > 0) {
    SG_CHECK(q->pulsetype && q->pulseparams, SINCGPU_EINVAL, "pulse arrays missing");
    r->ptype.assign(q->pulsetype, q->pulsetype + q->npulses);
    r->pparams.assign(q->pulseparams, q->pulseparams + 8 * q->npulses);
  }
  r->nsteps = q->nsteps;
  r->dt = q->dt;
  r->fp32 = q->coulomb_fp32;
  r->keep_state = q->keep_state;
  const long long G = (long long)q->numpoints * q->numpoints * q->numpoints;
  r->phi.assign(q->phi, q->phi + 2 * G * q->numspf);
  const int na = (q->numelec + q->restrictms) / 2, nb = q->numelec - na;
  const long long nc = binom(q->numspf, na) * binom(q->numspf, nb);
  r->avec.assign(q->avector, q->avector + 2 * nc);
  r->est = estimate_bytes(*r);
  r->t_submit = now_ms();
  {
    std::lock_guard<std::mutex> lk(s->mu);
    SG_CHECK(!s->stop, SINCGPU_ESTATE, "server is shutting down");
    r->id = s->next_id++;
    *id = r->id;
    s->pending.push_back(r.get());
    s->reqs[r->id] = std::move(r);
  }
  s->cv_work.notify_all();
  return SINCGPU_OK;
}

int sincgpu_server_wait(sincgpu_server* s, int id, double* energy0, double* energy, double* norm,
                        double* dipole_z, int* nsteps_done) {
  using namespace sincgpu;
  SG_CHECK(s, SINCGPU_EINVAL, "null server");
  std::unique_lock<std::mutex> lk(s->mu);
  SG_CHECK(s->reqs.count(id), SINCGPU_EINVAL, "unknown request %d", id);
  s->cv_done.wait(lk, [&] { return s->res.count(id) && s->res[id]->done; });
  const Res& r = *s->res[id];
  if (energy0) *energy0 = r.energy0;
  if (energy) *energy = r.energy;
  if (norm) *norm = r.norm;
  if (dipole_z) *dipole_z = r.dipole;
  if (nsteps_done) *nsteps_done = (int)r.step_ms.size();
  if (r.status != SINCGPU_OK) {
    set_error("request %d failed: %s", id, r.err);
    return r.status;
  }
  return SINCGPU_OK;
}

int sincgpu_server_result_arrays(sincgpu_server* s, int id, double* step_ms, double* energies, double* phi,
                                 double* avector) {
  using namespace sincgpu;
  SG_CHECK(s, SINCGPU_EINVAL, "null server");
  std::lock_guard<std::mutex> lk(s->mu);
  SG_CHECK(s->res.count(id) && s->res[id]->done, SINCGPU_ESTATE, "request %d not finished", id);
  const Res& r = *s->res[id];
  if (step_ms) std::copy(r.step_ms.begin(), r.step_ms.end(), step_ms);
  if (energies) std::copy(r.energies.begin(), r.energies.end(), energies);
  if (phi) {
    SG_CHECK(!r.phi.empty(), SINCGPU_ESTATE, "request %d kept no state", id);
    std::copy(r.phi.begin(), r.phi.end(), phi);
  }
  if (avector) {
    SG_CHECK(!r.avec.empty(), SINCGPU_ESTATE, "request %d kept no state", id);
    std::copy(r.avec.begin(), r.avec.end(), avector);
  }
  return SINCGPU_OK;
}

int sincgpu_server_timeline(sincgpu_server* s, int id, double* times, double* step_start) {
  using namespace sincgpu;
  SG_CHECK(s, SINCGPU_EINVAL, "null server");
  std::lock_guard<std::mutex> lk(s->mu);
  SG_CHECK(s->res.count(id) && s->res[id]->done, SINCGPU_ESTATE, "request %d not finished", id);
  const Res& r = *s->res[id];
  if (times) {
    times[0] = r.t_submit;
    times[1] = r.t_admit;
    times[2] = r.t_ready;
    times[3] = r.t_end;
  }
  if (step_start) std::copy(r.step_start.begin(), r.step_start.end(), step_start);
  return SINCGPU_OK;
}

int sincgpu_server_stats(sincgpu_server* s, long long* counts, double* p50_ms, double* p99_ms,
                         double* steps_per_s) {
  using namespace sincgpu;
  SG_CHECK(s, SINCGPU_EINVAL, "null server");
  std::lock_guard<std::mutex> lk(s->mu);
  std::vector<double> all;
  for (auto& kv : s->res)
    if (kv.second->done) all.insert(all.end(), kv.second->step_ms.begin(), kv.second->step_ms.end());
  std::sort(all.begin(), all.end());
  auto pct = [&](double p) {
    if (all.empty()) return 0.0;
    const size_t k = (size_t)std::min<double>(all.size() - 1, std::ceil(p * all.size()) - 1);
    return all[k];
  };
  if (p50_ms) *p50_ms = pct(0.50);
  if (p99_ms) *p99_ms = pct(0.99);
  const double span = s->t_last - s->t_first;
  if (steps_per_s) *steps_per_s = span > 0 ? all.size() / (span / 1e3) : 0.0;
  if (counts) {
    counts[0] = s->admitted;
    counts[1] = s->completed;
    counts[2] = (long long)all.size();
    counts[3] = s->peak_active;
    counts[4] = (long long)s->pending.size();
  }
  return SINCGPU_OK;
}

int sincgpu_server_destroy(sincgpu_server* s) {
  if (!s) return SINCGPU_OK;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    s->stop = true;
  }
  s->cv_work.notify_all();
  for (auto& t : s->workers) t.join();
  // the pool gives the reservation back (what live contexts hold stays theirs)
  cudaMemPool_t pool;
  if (cudaSetDevice(s->device) == cudaSuccess && cudaDeviceGetDefaultMemPool(&pool, s->device) == cudaSuccess &&
      cudaDeviceSynchronize() == cudaSuccess)
    cudaMemPoolTrimTo(pool, 0);
  cudaGetLastError();
  delete s;
  return SINCGPU_OK;
}

}  // extern "C"
