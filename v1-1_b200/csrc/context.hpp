// Device-resident state of one sinc-DVR system (the GPU counterpart of the
// SINCDVR project module state, SINCDVR/sincproject.f90:4-43).
#pragma once
#include <cuda_runtime.h>
#include <vector>
#include "common.cuh"
#include "fft_engine.cuh"

namespace sincgpu {

// Device scratch that grows on demand.  With an owner stream (every context
// workspace) the memory is stream-ordered (cudaMallocAsync / cudaFreeAsync on the
// context's stream): growing it neither synchronises the device nor stalls the
// other contexts' streams, which a plain cudaFree would.  Growth is refused while
// the owner stream is being captured into a graph.
// Device bytes of Coulomb pass intermediates (W1 + W2) per pair chunk when the
// chunk size is automatic.
constexpr long long kCoulChunkBudget = 2LL << 30;
// values in the real kernel-spectrum table d_khr for FFT length P (octant up to 128)
inline long long khr_len(int P) {
  const long long H = P / 2 + 1;
  return P <= 128 ? H * H * H : (long long)P * P * P;
}

struct Workspace {
  void* ptr = nullptr;
  size_t bytes = 0;
  cudaStream_t* owner = nullptr;
  int ensure(size_t need);
  void release();
};

// Per-kernel CUDA-event timing (off by default; sincgpu_profile).
enum Stage {
  ST_COUL_FWD_X = 0, ST_COUL_FWD_Y, ST_COUL_Z, ST_COUL_INV_Y, ST_COUL_INV_X,
  ST_TWOE_GEMM, ST_TWOE_FINISH, ST_RP_W, ST_RP_GEMM, ST_KE_XY, ST_KE_Z,
  ST_RHS_MIX, ST_RHS_REDPOT, ST_RHS_PROJ, ST_CI, ST_OTHER, ST_COUL_YZY, ST_COUNT
};

struct Prof {
  bool on = false;
  struct Rec { int stage; cudaEvent_t a, b; };
  std::vector<Rec> recs;
  double ms[ST_COUNT] = {};
  long long launches[ST_COUNT] = {};
};

// Device copies of the walk tables (ci.cu).
struct CIState {
  bool attached = false, assembled = false;
  int nc = 0;
  long long nsh = 0, ndh = 0;              // single / double hops (all configs)
  long long *den_off = nullptr, *tal_off = nullptr;
  int2 *den_ent = nullptr, *tal_ent = nullptr;  // (config1, +-config2) per RDM element
  int *sidx = nullptr, *didx = nullptr;     // packed matrix index, sign = phase
  long long *swb = nullptr, *dwb = nullptr; // first walk of each hop
  int *swn = nullptr, *dwn = nullptr;       // walks in each hop
  int *shop = nullptr, *dhop = nullptr;     // hop target config (0-based)
  long long *shop_off = nullptr, *dhop_off = nullptr;  // hops of each config
  double2 *xpot = nullptr, *xone = nullptr, *xz = nullptr;  // assembled per-hop values
  // spin sets (allspinproject=1): CSR of 0-based configs, row-major projectors
  bool spin = false;
  int nspinsets = 0, nspinelim = 0, maxspinset = 0;
  long long *sp_set_off = nullptr, *sp_proj_off = nullptr;
  int *sp_sets = nullptr, *sp_elim = nullptr;
  double* sp_proj = nullptr;
  long long numspinconfig = 0;              // spin-adapted dimension
  void release(cudaStream_t stream);  // stream-ordered frees
};

// Host integer tables (pair lists, lookup tables) kept on the device and
// uploaded only when their content changes, so that steady-state evaluations
// issue no host-to-device copies (which CUDA graph capture requires).
struct IntCache {
  std::vector<int> host;
  int* dev = nullptr;
  size_t cap = 0;
};
enum IntSlot { IC_PA = 0, IC_PB, IC_LUT, IC_TMAP, IC_COUNT };

// saved variables of the orbital exponential propagator (expospfprop)
struct OrbPropState {
  int expodim = 10;          // starting Krylov dimension
  int maxexpodim = 100;      // largest Krylov dimension
  double expostepfac = 1.2;  // step growth once the dimension is at its maximum
  double first_stepsize = 0.1;  // par_timestep / littlesteps
  int icalled = 0;
  int thisexpodim = 0;
  int exposet = 0;
  double tempstepsize = -1.0;
};

// one length-gauge pulse (MCTDH.SRC/parameters.f90:105-125)
struct PulseParams {
  int type = 2;
  double omega = 1.0, omega2 = 1.0, start = 0.0, phaseshift = 0.0, strength = 0.5, longstep = 1.0, theta = 0.0;
};
// z component of the field of all pulses at time t (tdpotlen0, which=3)
double pulse_ez(const std::vector<PulseParams>& pulses, double t);

struct CmfParams {
  double par_timestep = 0.05;
  int littlesteps = 1;
  double expotol = 1e-8, aerror = 1e-9;
  int aorder = 30, maxaorder = 100, expodim = 10, maxexpodim = 100;
  double expostepfac = 1.2, denreg = 1e-10;
  int step_flag = 2;
  double2 timefac = {0.0, -1.0};
};

// saved variables of expoavecprop (expo_driver.f90:842-866)
struct AvecPropState {
  int icalled = 0;
  double tempstep = -1.0;
  int dim = -1, set = 0, maxorder = 0;
};

// two time slots of the propagated state and its mean fields (cmf.cu)
struct CmfState {
  bool configured = false, ready = false;
  CmfParams p;
  std::vector<PulseParams> pulses;
  AvecPropState a;
  double first = 0.0, last = 0.0, energy = 0.0, norm = 0.0, nucdipz = 0.0;
  int orb_iters = 0, avec_iters = 0;
  // precision form: the last mean-field build of each step (whose matrices give the
  // energy and dipole and start the next step) and the post-prop reducedpot in FP64
  bool fp64_last = false;
  std::vector<int> pa, pb;  // pair list of the resident planar reduced potentials
  bool herm = true;
  Workspace ws;
  double2 *spfs[2] = {}, *avec[2] = {}, *den[2] = {}, *inv[2] = {}, *tally[2] = {}, *rp[2] = {};
  double2 *xpot[2] = {}, *xone[2] = {}, *xz[2] = {};
  double2 *mat = nullptr, *mats = nullptr, *ta = nullptr, *tb = nullptr, *tc = nullptr;
};

struct Ctx {
  // ---- problem parameters -------------------------------------------------
  int N = 0;             // points per axis (numpoints == gridpoints, nbox=1)
  long long G = 0;       // totpoints = N^3
  int nspf = 0;          // orbitals
  double spacing = 0.0;
  int numcenters = 0;
  std::vector<int> centershift;     // 3*numcenters
  std::vector<double> nuccharges;
  double nucrepulsion = 0.0;
  int device = 0;
  cudaStream_t stream = nullptr;
  bool own_stream = false;

  // ---- FFT plan for the padded Toeplitz grid ------------------------------
  FftPlan plan{};
  int P = 0;             // padded axis length, P >= 2N-1, 7-smooth
  int tx = 0;            // column-tile width of the y/z passes

  // ---- device tables --------------------------------------------------------
  double* d_kevect = nullptr;   // K(d), d in [1-N, N-1]           (2N-1)
  double* d_ketile = nullptr;   // K(j-l) padded S x S for the DMMA KE kernels
  int ke_stride = 0;            // S (row stride of d_ketile)
  double* d_pot = nullptr;      // nuclear potential              (G)
  double* d_zdip = nullptr;     // z coordinate of each point      (G)
  double* d_tcoul = nullptr;    // threed_two on [1-N,N-1]^3 (real) ((2N-1)^3)
  double2* d_khat = nullptr;    // DFT of the padded kernel / P^3  (P^3)
  double2* d_roots = nullptr;   // exp(-2 pi i m / P)              (P)
  float2* d_khat32 = nullptr;   // FP32 copies for the precision form, made on demand
  float2* d_roots32 = nullptr;
  double* d_khT = nullptr;      // real part of d_khat as [kx][kz][ky], three-pass Coulomb form (on demand)
  // real part of d_khat (the kernel is real and even in each axis, so its spectrum
  // is too: khat(P-k) = khat(k)): for P <= 128 on the octant k <= P/2 of each axis,
  // (P/2+1)^3 values; for longer lengths the full P^3 table (khr_len(P) values)
  double* d_khr = nullptr;
  float* d_khr32 = nullptr;
  float* d_khT32 = nullptr;

  // ---- scratch --------------------------------------------------------------
  Workspace ws_fft;     // W1 + W2 of the Coulomb passes
  Workspace ws_pairs;   // pair lists
  Workspace ws_gemm;    // reducedpot W matrix
  Workspace ws_twoe;    // twoematel split-K partials (may run beside reducedpot)
  Workspace ws_rhs;     // RHS temporaries
  Workspace ws_io;      // staging for host-pointer entry points
  Workspace ws_red;     // planar reduced potentials of the last build
  Workspace ws_conv;    // layout conversion scratch
  Workspace ws_state;   // resident mean-field state of the fused orbital-RHS entry
  Workspace ws_ci, ws_ci2;  // CI scratch (KE phi + partials; summed one-body matrix)
  Workspace ws_kry;         // Krylov basis, Hessenberg, Pade output
  Workspace ws_orb;         // orbital Krylov basis and Jacobian state
  Workspace ws_tcerr;       // timeout flags: [0] tensor-core contractions, [1] TMA z pass
  Workspace ws_tc;          // pre-split tf32 operand tiles of the bulk-copy tensor-core GEMM
  Workspace ws_bq;          // blended reduced potential Q and matrix M of an orbital Krylov call
  OrbPropState orb;
  CIState ci;
  CmfState cmf;
  IntCache icache[IC_COUNT];
  cudaGraph_t rhs_graph = nullptr;         // captured orbital-RHS evaluation (graph.cu)
  cudaGraphExec_t rhs_exec = nullptr;
  int coul_chunk = 0;   // pairs per pass sequence (0 = automatic)
  int coul_fp32 = 0;    // 1: Coulomb passes in FP32 (precision form), 0: FP64
  int contract_tf32 = 0;  // 1: reducedpot contraction as 3xTF32 on the tensor cores
  int coul_tma = -1;      // TMA-staged persistent z pass: 1 on, 0 off, -1 automatic (off)
  int tc_pipe = 4;        // tcgen05 3xTF32 GEMM with a staging ring and an MMA-issuing warp: 1: 3 stages of
                          // K = 16, 2: 4 x 16, 3: 6 x 8; 4, 5: pre-split operands moved by bulk copies
                          // into 3 or 5 stages; 0: two stages, block barriers
  int tc_kc = 16;         // K chunk of the tcgen05 3xTF32 GEMM: 16 or 32
  int ke_tf32 = 0;        // 1: kinetic contraction on the tcgen05 tensor cores, 3xTF32 (precision form)
  int coul_z2 = 0;        // z pass with P2 threads per line where P1 = 2 P2 (coul_z2_t): 1 on, 0 off
  int coul_fused = 0;     // three-pass Coulomb form (y, z, inverse y per plane on chip): 1 on where it fits, 0 off, -1 automatic
  int rp_dmma = 1;        // 1: FP64 reducedpot GEMM on the FP64 tensor cores (DMMA), 0: DFMA tiles
  int twoe_dmma = 1;      // 1: FP64 twoematel GEMM on the FP64 tensor cores (DMMA), 0: DFMA tiles
  int twoe_symdiag = 0;   // 1: multi-tile twoematel computes its diagonal tiles' lower blocks only
  int twoe_tile = 0;      // twoematel tile edge 16R: 0 = least padding, 2..9 = that R
  int orth_fused = 1;     // 1: an orbital Arnoldi step's orthogonalisation in one cooperative launch
  int kry_cluster = 1;    // 1: A-vector Gram-Schmidt beyond 4096 reals on a cluster of CTAs (0: one CTA)
  int orb_blendq = 1;     // 1: the orbital Jacobian reads one blended reduced potential (0: both slots')
  int rhs_overlap = 1;    // 1: the fused orbital-RHS entry runs its CI part and the mix + kinetic
                          //    contraction on `side`, beside the Coulomb passes and twoematel
  cudaStream_t side = nullptr;  // the second stream of the fused orbital-RHS entry (own, non-blocking;
                                //   made with its events on first use, side_stream)
  cudaEvent_t ev_fork = nullptr, ev_ci = nullptr, ev_join = nullptr, ev_coul = nullptr, ev_twoe = nullptr,
              ev_rhs = nullptr;
  cudaEvent_t ev_avec = nullptr;  // host-array entry: the A-vector is on the device
  // host-array orbital-RHS entry: the orbitals are copied in up to kUpGroups groups on
  // `copy` (made with its events by side_stream); while that entry runs, up_n > 0 and
  // orbital index < up_end[g] is on the device once ev_up[g] has fired, and the
  // Coulomb pair loop waits for each group before the pairs that need it
  static constexpr int kUpGroups = 8;
  int up_groups = 4;      // option rhs_upload_groups (1: one copy before the evaluation)
  cudaStream_t copy = nullptr;
  cudaEvent_t ev_up[kUpGroups] = {};
  cudaEvent_t ev_entry = nullptr;
  int up_n = 0;
  int up_end[kUpGroups] = {};
  void* orb_state_h = nullptr;    // page-locked copy of the orbital Krylov state (orbprop.cu)
  size_t orb_state_bytes = 0;
  cudaEvent_t ev_orb_state = nullptr;
  Prof prof;

  ~Ctx();
  void bind_workspaces();  // makes every workspace stream-ordered on `stream`
};

// Tensor-core (3xTF32) contractions of the precision form (contract_tc.cu).
int rp_gemm_tf32(Ctx& c, const double* Rpl, const double* Wm, int K, int NC, const int* d_tmap,
                 double2* reducedpot);
int tc_error_reset(Ctx& c);
// Device flags (zeroed once) that kernels with bounded waits set when a wait gave
// up: [0] tensor-core contractions, [1] TMA-staged Coulomb z pass.
int timeout_flags(Ctx& c, int** flags);
int tc_error_read(Ctx& c, int* flag);

// Stream-ordered device memory on the context's stream (cudaMallocAsync /
// cudaFreeAsync): allocating and freeing the context's tables neither
// synchronises the device nor stalls other contexts' streams.
int dalloc(Ctx& c, void** p, size_t bytes);
template <class T>
int dalloc(Ctx& c, T** p, size_t bytes) {
  return dalloc(c, reinterpret_cast<void**>(p), bytes);
}
void dfree(Ctx& c, void* p);
// (Re)allocates *dst and copies `bytes` from host memory on the context stream
// (the host buffer may be released on return).
int dupload(Ctx& c, void** dst, const void* src, size_t bytes);

// Brackets one kernel launch with events on the context stream when profiling.
struct ProfScope {
  Ctx& c;
  int stage;
  cudaEvent_t a = nullptr;
  ProfScope(Ctx& cc, int st) : c(cc), stage(st) {
    if (c.prof.on) {
      cudaEventCreate(&a);
      cudaEventRecord(a, c.stream);
    }
  }
  ~ProfScope() {
    if (c.prof.on) {
      cudaEvent_t b;
      cudaEventCreate(&b);
      cudaEventRecord(b, c.stream);
      c.prof.recs.push_back({stage, a, b});
    }
  }
};

// device copy of a host integer table (capi.cu); uploads only on a content change
int cached_ints(Ctx& c, int slot, const int* h, size_t n, const int** d);

// setup.cu
int build_tables(Ctx& c, int toothnbig, int toothnsmall, int flags);
int build_tables_from_arrays(Ctx& c, const double2* threed_two_host, const double* pot_host);
int choose_plan(Ctx& c);
int make_khat(Ctx& c);
// FP32 roots and kernel spectrum (rounded once from the FP64 tables)
int ensure_fp32_tables(Ctx& c);
// real kernel spectrum transposed to [kx][kz][ky] (FP64, and FP32 with fp32)
int ensure_khT(Ctx& c, bool fp32);

// coulomb.cu: R_p = T * (phi1_a conj(phi2_b)) for pairs p=(a_p,b_p).
// Rpl (device) receives the planar real/imag parts: Rpl[p*G+x] = Re, Rpl[(npair+p)*G+x] = Im.
// full (device, optional) receives twoereduced(x,a,b) interleaved; when `herm` the
// conjugate pair (b,a) is written too.
int coulomb_pairs(Ctx& c, const double2* phi1, const double2* phi2, const int* h_pa,
                  const int* h_pb, int npair, double* Rpl, double2* full, bool herm);
// op_tinv on explicit densities: dens(G, m) -> red(G, m)
int coulomb_dens(Ctx& c, const double2* dens, int m, double2* red);

// contract.cu
int twoe_matel(Ctx& c, const double2* phi1, const double2* phi2, const int* h_pa,
               const int* h_pb, int npair, const double* Rpl, bool herm, double2* twoematel);
// tally_herm: the 2-RDM has Gamma(c,d,k,i) = conj Gamma(d,c,i,k) (one A-vector);
// with a hermitian pair list only the k <= i half of reducedpot is computed and
// the rest mirrored
// The reduced-potential apply of actreduced00 folded into the reducedpot GEMM's
// epilogue: T = timefac (S + sum_k reducedpot(.,k,.) phi_k) inv, when reducedpot
// is a hermitian half whose columns fit one CTA tile (n <= 10) on the FP64 tensor
// path; `done` reports whether it was (else the caller applies reducedpot itself).
struct RpApply {
  const double2* phi;
  const double2* S;
  const double2* inv;
  double2 timefac;
  double2* T;
  cudaEvent_t ready;  // S and inv are written on another stream (or nullptr)
  bool done;
  // when set: also the projector-dot partials part[b][j + n i] = sum over the 64
  // points of tile b of conj(proj_j) T_i, as dots_kernel forms them (same bits)
  const double2* proj;
  double2* part;
};
int reduced_pot(Ctx& c, const double* Rpl, const int* h_pa, const int* h_pb, int npair,
                bool herm, const double2* tally, double2* reducedpot, bool tally_herm = false,
                RpApply* apply = nullptr);
int reduced_pot_full(Ctx& c, const double2* twoereduced, const double2* tally, double2* reducedpot);

// capi.cu: twoematel + reducedpot of one orbital set, and that followed by
// actreduced00 (tally_herm: see reduced_pot)
// Small page-locked host blocks, recycled across contexts: pinning and unpinning
// are driver calls that can take milliseconds while other contexts' threads run
int pinned_get(size_t bytes, void** p);
void pinned_put(size_t bytes, void* p);
// creates c.side and the fork/join events on the context's device if not yet made
int side_stream(Ctx& c);
// tally_ready: when set, reducedpot waits for it (the tally is written on another
// stream); side: when set, twoematel runs on that stream after the Coulomb passes
// and c.ev_twoe marks its end (the caller joins it)
// defer: when set (and twoematel null), the pair lists the twoematel GEMM needs are
// kept there and twoe_deferred forms twoematel later from the same reduced potentials
struct TwoeDefer {
  std::vector<int> pa, pb;
  bool herm = false;
};
int mean_field(Ctx& c, const double2* phi, const double2* tally, double2* twoematel, double2* reducedpot,
               bool tally_herm, cudaEvent_t tally_ready = nullptr, cudaStream_t side = nullptr,
               RpApply* apply = nullptr, TwoeDefer* defer = nullptr);
// twoematel of a deferred mean-field build on `side` once `after` has fired; c.ev_twoe
// marks its end (the caller joins it).  The reduced potentials in c.ws_red must
// still be the build's.
int twoe_deferred(Ctx& c, const double2* phi, const TwoeDefer& defer, double2* twoematel, cudaEvent_t after,
                  cudaStream_t side);
int orbital_rhs(Ctx& c, const double2* phi, const double2* tally, const double2* denmat, const double2* invdenmat,
                double2 timefac, double ztdpot, double2* twoematel, double2* reducedpot, double2* out,
                bool tally_herm);

// ke.cu: out = KE(in) [+ pot*in + zfield*z*in when `extra`]
int mult_ke(Ctx& c, const double2* in, double2* out, int howmany, bool extra, double zfield);

// ci.cu (walk tables: walks.hpp)
struct Walks;
int ci_attach(Ctx& c, const Walks& w);
int ci_denmat(Ctx& c, const double2* avec, double2* denmat, double2* invdenmat, double denreg);
int ci_tally(Ctx& c, const double2* a1, const double2* a2, double2* tally);
int ci_onebody(Ctx& c, const double2* phi, double2* mats);
int ci_assemble(Ctx& c, const double2* twoematel, const double2* mats);
int ci_sigma(Ctx& c, const double2* in, double2* out, double constant, double ez, double nucdipz);
int ci_dipole_z(Ctx& c, const double2* a, double2* tmp, double nucdipz, double2* dip, double* normsq);

// krylov.cu: w = exp(t * timefac * H) v on the real-ified A-vector
// maxdim: the reference's DGEXPVxxx2 maxdim (Krylov dimension must stay below it;
// 0 selects the vector length); nmult_out: number of sigma products
int expv_avector(Ctx& c, const double2* v, double2* w, double t, double2 timefac, int m, double tol,
                 double anorm, double* stepguess, int* nstep_out, double ez, double nucdipz, int maxdim = 0,
                 int* nmult_out = nullptr);
// twoematel and the Coulomb pair solves of (phi1, phi2); leaves the planar reduced
// potentials of the pair list (pa, pb) in ws_red (capi.cu)
int twoe_core(Ctx& c, const double2* phi1, const double2* phi2, double2* twoematel, double2* full,
              std::vector<int>& pa, std::vector<int>& pb, bool& herm);

// rhs.cu
int mult_reducedpot(Ctx& c, const double2* phi, const double2* redpot, double2* out);
// orbitals [i0, i0+ni) only; redpot/out hold just that window
int mult_reducedpot_range(Ctx& c, const double2* phi, const double2* redpot, int i0, int ni,
                          double2* out);
int actreduced(Ctx& c, const double2* phi, const double2* proj, const double2* denmat,
               const double2* invdenmat, const double2* redpot, double2 timefac,
               int dentimeflag, int projflag, double zfield, double2* out);
// actreduced in two halves: the mix with denmat and the kinetic (+ potential and
// field) contraction, which need no reduced potentials, then the reduced-potential
// apply and the projection; the temporaries between them live in ws_rhs
// (t_ready: T, the apply's result before the projection, is already in ws_rhs)
int actreduced_pre(Ctx& c, const double2* phi, const double2* denmat, double zfield);
int actreduced_post(Ctx& c, const double2* phi, const double2* proj, const double2* invdenmat,
                    const double2* redpot, double2 timefac, int dentimeflag, int projflag, double2* out,
                    bool t_ready = false, bool dots_ready = false);
// the kinetic result S of actreduced_pre, the apply target T and the projector-dot
// partials (orbital_dots_scratch(c) blocks of 64 points) in ws_rhs
int actreduced_temps(Ctx& c, double2** S, double2** T, double2** part = nullptr);
// actreduced_pre for several density matrices of one phi: the kinetic, potential
// and field operators act on each orbital alike and so commute with the orbital
// mixing, KE(phi denmat) = KE(phi) denmat; actreduced_ke forms KE(phi) once (ws_rhs
// Y), actreduced_mix_ke then S = Y denmat for each denmat before actreduced_post
int actreduced_ke(Ctx& c, const double2* phi, double zfield);
// out = facs[0] A_0 + facs[1] A_1, A_s = actreduced without projection for slot s
// (denmat[s], invdenmat[s], redpot[s]), in one pass after one kinetic contraction
bool actreduced_blend2_fits(int n);  // its shared memory (n <= 20)
int actreduced_blend2(Ctx& c, const double2* x, const double2* const* denmat, const double2* const* invdenmat,
                      const double2* const* redpot, const double* facs, double2 timefac, double zfield,
                      double2* out);
// The same blend with the slots folded once per orbital Krylov call: the
// propagation's blend factors and mean fields are fixed during the call, so
// A = timefac (Y M + sum_k x_k Q(:, k, :)) with M = sum_s f_s D_s I_s and
// Q(x, k, i) = sum_s f_s sum_j V_s(x, k, j) I_s(j, i); blendq_prepare forms Q and M
// in c.ws_bq (one pass over both slots' reducedpot), after which each product
// reads one reduced potential instead of two.  Same algebra as actreduced_blend2,
// rounding differs.
bool actreduced_blendq_fits(int n);
int blendq_prepare(Ctx& c, const double2* const* denmat, const double2* const* invdenmat,
                   const double2* const* redpot, const double* facs);
int actreduced_blendq(Ctx& c, const double2* x, double2 timefac, double zfield, double2* out);
int actreduced_mix_ke(Ctx& c, const double2* denmat);
// D(j,i) = <P_j|T_i> over the grid (split-K, deterministic); part holds
// orbital_dots_scratch(c) * nspf^2 partial sums
int orbital_dots_scratch(const Ctx& c);
int orbital_dots(Ctx& c, const double2* P, const double2* T, double2* D, double2* part);
// out = in x mat (n x n, column-major)
int orbital_mix(Ctx& c, const double2* in, const double2* mat, double2* out);
// out = T - P (M1 + M2) - X D2
int jac_combine(Ctx& c, const double2* T, const double2* P, const double2* M1, const double2* M2,
                const double2* X, const double2* D2, double2* out);
// acc = a acc + b in  (acc = b in when `first`)
int axpby(Ctx& c, double2* acc, const double2* in, double a, double b, long long len, bool first);

// ci.cu: spin projection of an A-vector in place (basis_project, allspinproject=1)
int ci_spin_project(Ctx& c, double2* a);

// krylov.cu: (6,6) Pade exponential of a small Hessenberg (mx <= 128)
int pade_expm(Ctx& c, const double* Hm, int mh, int mx, double t, int col, double* exph, double* Efull,
              double* gscratch, int* d_ns);

// orbprop.cu: one orbital propagation over [tin, tout] (expospfprop) and the
// Loewdin re-orthonormalisation (spf_orthogit)
struct MeanFieldSlot {
  const double2* denmat;
  const double2* invdenmat;
  const double2* reducedpot;
};
int expospfprop(Ctx& c, double2* phi, const MeanFieldSlot* slots, double tin, double tout,
                double firsttime, double lasttime, bool linear, double2 timefac, double ez, double expotol,
                int* numiters);
int spf_orthogit(Ctx& c, double2* phi, double* error);

// cmf.cu: constant-mean-field step (cmf_prop_wfn) and its initialisation
int cmf_init(Ctx& c, const double2* phi, const double2* avec, double* e0);
int cmf_step(Ctx& c, double tin, double tout);
// z component of the nuclear dipole (capi_ci.cu)
double nucdip_z(const Ctx& c);

}  // namespace sincgpu

// Opaque handle of the C ABI.
struct sincgpu_ctx {
  sincgpu::Ctx c;
};

#define CTX_CHECK(ctx)                                                                   \
  do {                                                                                   \
    if (!(ctx)) {                                                                        \
      ::sincgpu::set_error("null context");                                              \
      return SINCGPU_EINVAL;                                                             \
    }                                                                                    \
    SG_CUDA(cudaSetDevice((ctx)->c.device));                                             \
  } while (0)
