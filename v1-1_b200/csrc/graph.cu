// Captured CUDA graphs of the orbital-RHS evaluation and batches of them.
//
// A context captures one sincgpu_orbital_rhs_avec_dev call (1-RDM, inverse,
// 2-RDM, Coulomb pair solves, twoematel, reducedpot, actreduced00) into a graph
// after a warm-up run that sizes every workspace and uploads every host table,
// so the captured work is kernels and device copies only.  A batch adds the
// graphs of many contexts (instances of different grids, orbitals and electron
// counts) as independent child nodes of one parent graph: one launch runs them
// all and lets the device overlap them.
//
// The autotuner times the Coulomb pair-chunk size (pairs per pass sequence,
// which sets how much of W1/W2 stays in L2) for an instance and keeps the
// fastest.
#include <algorithm>
#include <memory>
#include <vector>
#include "context.hpp"
#include "../../include/sincgpu.h"

struct sincgpu_batch {
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  int count = 0;
};

using namespace sincgpu;

namespace {

struct RhsArgs {
  const double *phi, *avec;
  double tre, tim, ztd;
  double *den, *inv, *tally, *mat, *rp, *out;
};

int run_rhs(sincgpu_ctx* h, const RhsArgs& a) {
  return sincgpu_orbital_rhs_avec_dev(h, a.phi, a.avec, a.tre, a.tim, a.ztd, a.den, a.inv, a.tally, a.mat, a.rp,
                                      a.out);
}

}  // namespace

extern "C" {

int sincgpu_rhs_graph_capture(sincgpu_ctx* h, const double* phi, const double* avector, double tre, double tim,
                              double ztdpot, double* denmat, double* invdenmat, double* tally, double* twoematel,
                              double* reducedpot, double* outspfs) {
  CTX_CHECK(h);
  Ctx& c = h->c;
  SG_CHECK(!c.prof.on, SINCGPU_ESTATE, "turn profiling off before capturing");
  RhsArgs a{phi, avector, tre, tim, ztdpot, denmat, invdenmat, tally, twoematel, reducedpot, outspfs};
  // warm-up: sizes the workspaces, uploads the tables, sets kernel attributes
  SG_TRY(run_rhs(h, a));
  SG_CUDA(cudaStreamSynchronize(c.stream));
  if (c.rhs_exec) cudaGraphExecDestroy(c.rhs_exec);
  if (c.rhs_graph) cudaGraphDestroy(c.rhs_graph);
  c.rhs_exec = nullptr;
  c.rhs_graph = nullptr;
  cudaStream_t cap;
  SG_CUDA(cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking));
  cudaStream_t saved = c.stream;
  c.stream = cap;
  int rc = SINCGPU_OK;
  cudaError_t e = cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal);
  if (e == cudaSuccess) {
    rc = run_rhs(h, a);
    cudaGraph_t g = nullptr;
    cudaError_t e2 = cudaStreamEndCapture(cap, &g);
    if (rc == SINCGPU_OK && e2 != cudaSuccess) {
      set_error("graph capture failed: %s", cudaGetErrorString(e2));
      rc = SINCGPU_ECUDA;
    }
    if (rc == SINCGPU_OK) c.rhs_graph = g;
    else if (g) cudaGraphDestroy(g);
  } else {
    set_error("cudaStreamBeginCapture: %s", cudaGetErrorString(e));
    rc = SINCGPU_ECUDA;
  }
  c.stream = saved;
  cudaStreamDestroy(cap);
  if (rc != SINCGPU_OK) return rc;
  SG_CUDA(cudaGraphInstantiate(&c.rhs_exec, c.rhs_graph, 0));
  return SINCGPU_OK;
}

int sincgpu_rhs_graph_launch(sincgpu_ctx* h) {
  CTX_CHECK(h);
  Ctx& c = h->c;
  SG_CHECK(c.rhs_exec, SINCGPU_ESTATE, "no captured graph");
  SG_CUDA(cudaGraphLaunch(c.rhs_exec, c.stream));
  count_launch();
  return SINCGPU_OK;
}

int sincgpu_batch_create(sincgpu_batch** out, sincgpu_ctx** ctxs, int n) {
  SG_CHECK(out && ctxs && n >= 1, SINCGPU_EINVAL, "bad argument");
  std::unique_ptr<sincgpu_batch> b(new sincgpu_batch());
  SG_CUDA(cudaGraphCreate(&b->graph, 0));
  for (int i = 0; i < n; ++i) {
    SG_CHECK(ctxs[i] && ctxs[i]->c.rhs_graph, SINCGPU_ESTATE, "instance %d has no captured graph", i);
    SG_CHECK(ctxs[i]->c.device == ctxs[0]->c.device, SINCGPU_EINVAL, "instances on different devices");
    cudaGraphNode_t node;
    SG_CUDA(cudaGraphAddChildGraphNode(&node, b->graph, nullptr, 0, ctxs[i]->c.rhs_graph));
  }
  SG_CUDA(cudaGraphInstantiate(&b->exec, b->graph, 0));
  b->count = n;
  *out = b.release();
  return SINCGPU_OK;
}

int sincgpu_batch_launch(sincgpu_batch* b, void* stream) {
  SG_CHECK(b && b->exec, SINCGPU_EINVAL, "bad batch");
  SG_CUDA(cudaGraphLaunch(b->exec, (cudaStream_t)stream));
  count_launch();
  return SINCGPU_OK;
}

int sincgpu_batch_destroy(sincgpu_batch* b) {
  if (!b) return SINCGPU_OK;
  if (b->exec) cudaGraphExecDestroy(b->exec);
  if (b->graph) cudaGraphDestroy(b->graph);
  delete b;
  return SINCGPU_OK;
}

int sincgpu_autotune_rhs(sincgpu_ctx* h, const double* phi, const double* avector, double* denmat,
                         double* invdenmat, double* tally, double* twoematel, double* reducedpot, double* outspfs,
                         int* best_chunk, float* best_ms) {
  CTX_CHECK(h);
  Ctx& c = h->c;
  const int n = c.nspf, npair = n * (n + 1) / 2;
  RhsArgs a{phi, avector, 0.0, -1.0, 0.0, denmat, invdenmat, tally, twoematel, reducedpot, outspfs};
  cudaEvent_t e0, e1;
  SG_CUDA(cudaEventCreate(&e0));
  SG_CUDA(cudaEventCreate(&e1));
  int rc = SINCGPU_OK;
  // one configuration: a warm-up evaluation (sizes the workspaces), then three timed
  auto timed = [&](float* ms) -> int {
    SG_TRY(run_rhs(h, a));
    cudaEventRecord(e0, c.stream);
    for (int r = 0; r < 3; ++r) SG_TRY(run_rhs(h, a));
    cudaEventRecord(e1, c.stream);
    SG_CUDA(cudaEventSynchronize(e1));
    cudaEventElapsedTime(ms, e0, e1);
    *ms /= 3.f;
    return SINCGPU_OK;
  };
  // coordinate descent over three knobs, each kept at its best before the next:
  // (1) the Coulomb pair chunk (pairs per pass launch); pair chunks whose W1/W2
  //     scratch would exceed 512 MiB are not tried
  // (2) the twoematel tile edge 16R (the register block R of the FP64 tensor-core
  //     GEMM: fewer, larger tiles against less padding and fewer triangle tiles)
  // (3) the Coulomb z pass plain or with TMA-staged slabs
  float bms = 1e30f;
  int best = 0;
  const int saved_chunk = c.coul_chunk, saved_tile = c.twoe_tile, saved_tma = c.coul_tma;
  std::vector<int> cand = {0, npair, (npair + 1) / 2, (npair + 3) / 4, 16, 8};
  std::sort(cand.begin(), cand.end());
  cand.erase(std::unique(cand.begin(), cand.end()), cand.end());
  const size_t csz = c.coul_fp32 ? sizeof(float2) : sizeof(double2);
  const size_t per_pair = csz * ((size_t)c.N * c.N * c.P + (size_t)c.N * c.P * c.P);
  for (int ch : cand) {
    if (ch < 0 || ch > npair) continue;
    if (ch > 0 && per_pair * (size_t)ch > (512ull << 20)) continue;
    c.coul_chunk = ch;
    float ms = 0.f;
    if ((rc = timed(&ms)) != SINCGPU_OK) break;
    if (ms < bms) {
      bms = ms;
      best = ch;
    }
  }
  if (rc == SINCGPU_OK) {
    c.coul_chunk = best;
    int best_tile = 0;
    for (int t : {4, 5, 6, 7, 8, 9}) {
      c.twoe_tile = t;
      float ms = 0.f;
      if ((rc = timed(&ms)) != SINCGPU_OK) break;
      if (ms < 0.98f * bms) {  // a fixed tile must beat the automatic one clearly
        bms = ms;
        best_tile = t;
      }
    }
    c.twoe_tile = best_tile;
  }
  if (rc == SINCGPU_OK) {
    c.coul_tma = 1;
    float ms = 0.f;
    rc = timed(&ms);
    if (rc == SINCGPU_OK && ms < 0.98f * bms) {
      bms = ms;
    } else {
      c.coul_tma = saved_tma;
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (rc != SINCGPU_OK) {
    c.coul_chunk = saved_chunk;
    c.twoe_tile = saved_tile;
    c.coul_tma = saved_tma;
  }
  if (best_chunk) *best_chunk = c.coul_chunk;
  if (best_ms) *best_ms = bms;
  return rc;
}

}  // extern "C"
