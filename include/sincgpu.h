/*
 * sincgpu -- B200 (sm_100a) implementation of the LBNL-AMO-MCTDHF polyatomic
 * sinc-DVR orbital right-hand side, behind a plain C ABI.
 *
 * Conventions
 *   - Every array is a Fortran array passed by address: column-major, the grid
 *     index x fastest (x + N*y + N*N*z), then the orbital index.
 *   - "complex" arrays are complex*16: interleaved (re, im) doubles.  Their
 *     element count below is in complex numbers.
 *   - Orbital indices in argument lists are 1-based, as in the Fortran caller.
 *   - Every function returns SINCGPU_OK (0) or an error code; the message of the
 *     last failure on the calling thread is available from sincgpu_last_error().
 *     The library never aborts the process; the Fortran shim turns a non-zero
 *     status into the reference's abort (OFLWR ... CFLST).
 *   - Functions without the _dev suffix take HOST arrays (they upload, compute
 *     and download before returning).  _dev functions take DEVICE pointers and
 *     enqueue on the context stream; call sincgpu_synchronize() before reading
 *     results on the host.
 *   - A context is not re-entrant: callers serialise calls on one context.
 *
 * Citations are to the reference project (MCTDH.SRC/...).
 */
#ifndef SINCGPU_H
#define SINCGPU_H

#ifdef __cplusplus
extern "C" {
#endif

#define SINCGPU_OK 0
#define SINCGPU_EINVAL 1   /* bad argument */
#define SINCGPU_ECUDA 2    /* CUDA runtime failure */
#define SINCGPU_ENOMEM 3   /* device allocation failed */
#define SINCGPU_ESTATE 4   /* call made in the wrong state */
#define SINCGPU_ETIMEOUT 5 /* bounded device wait expired */
#define SINCGPU_ERANGE 6   /* size outside the supported range */

typedef struct sincgpu_ctx sincgpu_ctx;

/* Message of the last failure on this thread ("" if none). */
const char* sincgpu_last_error(void);
int sincgpu_version(void);

/* ---------------------------------------------------------------------------
 * Set-up
 * ------------------------------------------------------------------------- */

/* Builds the project state on the device: 1-D kinetic vector (SINCDVR/SineDVR.f90:11-44,
 * init_sinc_new.f90:441-464), the inverse-kinetic Coulomb kernel threed_two
 * (SINCDVR/tooth.f90:12-231, sincproject.f90:119-188), the nuclear potential
 * (sincproject.f90:190-250) and nucrepulsion (sinc_extraproject.f90:288-300).
 * Replaces the get_twoe_new part of init_project (init_sinc_new.f90:533).
 *   centershift(3,numcenters) in units of spacing/2; flags bit0: single-precision
 *   sqrt in the far-field nuclear potential (sincproject.f90:220 without -r8);
 *   bit1: notwoflag (zero Coulomb kernel, sincproject.f90:330-332). */
int sincgpu_create(sincgpu_ctx** ctx, int numpoints, double spacing, int numcenters,
                   const int* centershift, const double* nuccharges, int numspf, int toothnbig,
                   int toothnsmall, int flags, int device);

/* Same, but takes threed_two(-N:N-1,-N:N-1,-N:N-1) (complex, real valued) and
 * pot(totpoints) already built by the Fortran init_project. */
int sincgpu_create_from_tables(sincgpu_ctx** ctx, int numpoints, double spacing, int numspf,
                               const double* threed_two, const double* pot, int device);

int sincgpu_destroy(sincgpu_ctx* ctx);

/* Copies back tempcoulomb(1-N:N-1)^3 = threed_two on that range (real),
 * pot(totpoints), kevect(1-N:N-1) and nucrepulsion.  Any pointer may be NULL. */
int sincgpu_get_tables(sincgpu_ctx* ctx, double* tempcoulomb, double* pot, double* kevect,
                       double* nucrepulsion);

/* Padded FFT length P (>= 2N-1) used for the Toeplitz convolution. */
int sincgpu_fft_length(sincgpu_ctx* ctx);

/* Options: "coul_chunk" (pairs per Coulomb pass sequence, 0 = auto);
 * "coulomb_fp32" (1: the Coulomb passes in FP32, the precision form);
 * "contract_tf32" (1: the reducedpot contraction on the tensor cores as 3xTF32
 * with FP32 accumulation, the precision form); "coul_tma" (the Coulomb z pass
 * with TMA-staged slabs: 1 on, 0 off, -1 automatic = off: the plain pass was
 * faster at every measured length once whole pair lists go in one launch);
 * "twoe_tile" (twoematel tile edge 16R: 0 = least padding, 2..9 = R);
 * "orth_fused" (1: the orbital Arnoldi orthogonalisation of one Krylov step in
 * one cooperative launch with bounded grid barriers, 0: one launch per dot,
 * projection and norm; the results are bitwise the same); "rhs_overlap" (1: the
 * A-vector orbital-RHS entry runs the RDMs, the density-matrix inverse and the
 * kinetic contraction on a second stream of the context beside the Coulomb
 * passes, then twoematel there beside reducedpot and the apply, joined by
 * events; 0: one stream; bitwise the same); "coul_fused" (1: the Coulomb
 * solve as three passes, the y, z and inverse-y transforms of each (pair, kx)
 * plane in one kernel with the plane in shared memory, split over a
 * thread-block cluster where it does not fit one CTA; 0: five passes through
 * HBM; results agree to rounding); "cmf_fp64_last" (1: in the precision form,
 * the last mean-field build of each CMF step and its post-prop reducedpot run
 * in FP64, so that the energy, the dipole and the next step start from FP64
 * matrices); "ke_tf32" (1: the per-axis kinetic contraction on the tcgen05
 * tensor cores, one 3xTF32 GEMM per axis with FP32 accumulation, the precision
 * form; 0: FP64 tensor cores); "rhs_upload_groups" (1..8, default 4: the
 * host-array orbital-RHS entry copies the orbitals up in that many groups on
 * a copy stream, and the Coulomb pair loop starts on the pairs of the first
 * group while the others are in flight; 1: one copy before the evaluation;
 * bitwise the same); "kry_cluster" (1, default: the A-vector Krylov's
 * Gram-Schmidt step on vectors longer than 4096 reals runs on a cluster of 8
 * CTAs with the dot products summed through distributed shared memory; 0: one
 * CTA; results agree to rounding); "orb_blendq" (1, default: an orbital Krylov
 * call with two mean-field slots folds their reduced potentials and density
 * matrices into one blended potential once, and each Jacobian product reads
 * that; 0: each product reads both slots; results agree to rounding). */
int sincgpu_set_option(sincgpu_ctx* ctx, const char* name, long long value);
/* Current value of an option of sincgpu_set_option (SINCGPU_EINVAL for an unknown name). */
int sincgpu_get_option(sincgpu_ctx* ctx, const char* name, long long* value);

/* C(M x N, row-major) = A(M x K, row-major) * B(N x K, row-major)^T on the
 * tensor cores (tcgen05 kind::tf32, 3xTF32 split, FP32 accumulation), device
 * pointers.  The contraction kernel of the precision form, exposed for checks;
 * *timed_out (may be NULL) is set when the kernel gave up waiting for its MMAs. */
/* flags[0..1]: 1 when a tensor-core contraction / a TMA-staged Coulomb z pass gave
 * up waiting for its MMAs or slab loads (bounded waits) since the context was
 * created; synchronises the context's stream. */
int sincgpu_kernel_timeouts(sincgpu_ctx* ctx, int* flags);

int sincgpu_gemm_tf32x3_dev(sincgpu_ctx* ctx, const double* A, const double* B, double* C, long long M, int N,
                            int K, int* timed_out);

int sincgpu_synchronize(sincgpu_ctx* ctx);
/* How host threads wait for the device (process-wide, per device): 0 = CUDA's
 * default heuristic, 1 = spin, 2 = yield, 3 = block on an OS primitive.  Blocking
 * keeps many host threads that each wait on their own stream (the request loop's
 * workers) from burning the host's cores while they wait. */
int sincgpu_set_sync_mode(int device, int mode);

/* Makes the context enqueue on a caller-owned cudaStream_t (passed as void*).
 * The caller keeps the stream alive for the life of the context. */
int sincgpu_set_stream(sincgpu_ctx* ctx, void* stream);

/* Number of kernels this library has launched in the process so far. */
long long sincgpu_launch_count(void);

/* Per-kernel CUDA-event timing on the context stream (off by default).
 * sincgpu_profile_read synchronises, returns the accumulated milliseconds and
 * launch counts per stage (indices: 0 coul_fwd_x, 1 coul_fwd_y, 2 coul_z,
 * 3 coul_inv_y, 4 coul_inv_x, 5 twoe_gemm, 6 twoe_finish, 7 rp_w, 8 rp_gemm,
 * 9 ke_xy, 10 ke_z, 11 rhs_mix, 12 rhs_redpot, 13 rhs_proj, 14 ci, 15 other)
 * and resets them. */
int sincgpu_profile(sincgpu_ctx* ctx, int enable);
int sincgpu_profile_read(sincgpu_ctx* ctx, double* ms, long long* launches, int nstage);

/* Page-locks a caller's host array so that host-array entry points copy at full
 * PCIe/C2C speed.  Optional. */
int sincgpu_host_register(void* ptr, long long bytes);
int sincgpu_host_unregister(void* ptr);

/* ---------------------------------------------------------------------------
 * Drop-ins for the SINCDVR project interface (host arrays)
 * ------------------------------------------------------------------------- */

/* call_twoe_matel00 (SINCDVR/coreproject.f90:945-1194; caller MCTDH.SRC/matel.f90:95-96):
 *   twoereduced(x,a,b) = sum_y threed_two(x-y) inspfs10(y,a) conj(inspfs20(y,b))
 *   twoematel(a1,b1,a2,b2) = sum_x inspfs10(x,a1) conj(inspfs20(x,b1)) twoereduced(x,a2,b2)
 * inspfs10/20(totpoints,numspf), twoematel(numspf^4), twoereduced(totpoints,numspf,numspf).
 * lowspf/highspf must span all orbitals (single-rank build).  When inspfs10 and
 * inspfs20 are the same array the hermitian pair symmetry halves the work. */
int sincgpu_call_twoe_matel00(sincgpu_ctx* ctx, int lowspf, int highspf, const double* inspfs10,
                              const double* inspfs20, double* twoematel, double* twoereduced);

/* op_tinv (SINCDVR/coreproject.f90:250-539, serial path): twoereduced(:,i) =
 * threed_two (*) twoeden03(:,i), i=1..allsize.  circsize only has to divide allsize
 * (it selects batching in the reference and does not change the result). */
int sincgpu_op_tinv(sincgpu_ctx* ctx, const double* twoeden03, double* twoereduced, int allsize,
                    int circsize);

/* mult_ke (SINCDVR/coreproject.f90:2104-2116): in/out(totpoints,howmany). */
int sincgpu_mult_ke(sincgpu_ctx* ctx, const double* in, double* out, int howmany);

/* mult_reducedpot (SINCDVR/coreproject.f90:1200-1235):
 * outspfs(:,i) = sum_k reducedpot(:,k,i) inspfs(:,k), i = firstspf..lastspf;
 * reducedpot(totpoints,numspf,firstspf:lastspf), outspfs(totpoints,firstspf:lastspf). */
int sincgpu_mult_reducedpot(sincgpu_ctx* ctx, int firstspf, int lastspf, const double* inspfs,
                            double* outspfs, const double* reducedpot);

/* get_reducedpot0 (MCTDH.SRC/mean.f90:503-588): reducedpot(G,n^2) =
 * twoereduced(G,n^2) x reducedpottally(n^2,n^2). */
int sincgpu_get_reducedpot(sincgpu_ctx* ctx, const double* twoereduced,
                           const double* reducedpottally, double* reducedpot);

/* actreduced00 (MCTDH.SRC/derivs.f90:629-852) for numr=1, no frozen core, length
 * gauge: out = (1-P) timefac [KE + pot + ztdpot z + W] (inspfs denmat) invdenmat,
 * where W is the mult_reducedpot term on inspfs.  denmat/invdenmat(numspf,numspf). */
int sincgpu_actreduced00(sincgpu_ctx* ctx, int dentimeflag, const double* inspfs,
                         const double* projspfs, const double* denmat, const double* invdenmat,
                         const double* reducedpot, double timefac_re, double timefac_im,
                         int projflag, double ztdpot, double* outspfs);

/* ---------------------------------------------------------------------------
 * Device-resident forms (device pointers, context stream)
 * ------------------------------------------------------------------------- */
int sincgpu_twoe_matel_dev(sincgpu_ctx* ctx, const double* phi1, const double* phi2,
                           double* twoematel, double* twoereduced);
int sincgpu_mult_ke_dev(sincgpu_ctx* ctx, const double* in, double* out, int howmany);
int sincgpu_mult_reducedpot_dev(sincgpu_ctx* ctx, const double* inspfs, double* outspfs,
                                const double* reducedpot);
/* Mean-field build from orbitals and a 2-RDM tally: Coulomb pair solves,
 * twoematel and reducedpot (MCTDH.SRC/matel.f90:72-111 + mean.f90:484-590). */
int sincgpu_mean_field_dev(sincgpu_ctx* ctx, const double* phi, const double* reducedpottally,
                           double* twoematel, double* reducedpot);

/* Allocation-free op_tinv; no counterpart in the reference.  For callers that
 * cannot call cudaMalloc when they need the solve (a process whose device memory
 * is partitioned once at start-up, a latency-critical loop that cannot accept
 * the synchronisation cudaMalloc/cudaFree may cause).  Same result as
 * sincgpu_op_tinv, on DEVICE arrays twoeden03(totpoints,allsize) ->
 * twoereduced(totpoints,allsize), enqueued on the context stream.  The FFT
 * scratch is a fixed 64 MiB device array inside the library (held on every GPU
 * that loads it until exit); one density needs 16*(N*N*P + N*P*P) bytes of it
 * in the FP64 form and 8*(N*N*P + N*P*P) with the context option coulomb_fp32
 * (P = sincgpu_fft_length); larger grids are rejected with SINCGPU_ERANGE.
 * The FP32 form also needs the context's FP32 twiddle and kernel-spectrum
 * tables: sincgpu_set_option("coulomb_fp32", 1) allocates them when the option
 * is set, so this entry itself never does.  All calls share the array: calls
 * that overlap on the GPU race.  The first call on a device looks up the array's address; make it
 * before any stream capture. */
int sincgpu_op_tinv_noalloc_dev(sincgpu_ctx* ctx, const double* twoeden03, double* twoereduced,
                                int allsize);
int sincgpu_actreduced_dev(sincgpu_ctx* ctx, int dentimeflag, const double* inspfs,
                           const double* projspfs, const double* denmat, const double* invdenmat,
                           const double* reducedpot, double timefac_re, double timefac_im,
                           int projflag, double ztdpot, double* outspfs);

/* One orbital-RHS evaluation = mean-field build (Coulomb pair solves, twoematel,
 * reducedpot from the 2-RDM tally) + actreduced00 with projspfs = inspfs,
 * dentimeflag = projflag = 1 (MCTDH.SRC/derivs.f90:629-852).  Device pointers;
 * reducedpot(totpoints,n,n) receives the reduced potentials; twoematel may be NULL. */
int sincgpu_orbital_rhs_dev(sincgpu_ctx* ctx, const double* phi, const double* reducedpottally,
                            const double* denmat, const double* invdenmat, double timefac_re,
                            double timefac_im, double ztdpot, double* twoematel,
                            double* reducedpot, double* outspfs);

/* Host-array form of the same evaluation: only phi, the tally and the two n x n
 * matrices go up and only outspfs (and twoematel, if non-NULL) come back; the
 * reduced potentials stay on the device.  A Fortran driver replaces the sequence
 * twoe_matel + get_reducedpot + actreduced0 with this call. */
int sincgpu_orbital_rhs(sincgpu_ctx* ctx, const double* phi, const double* reducedpottally,
                        const double* denmat, const double* invdenmat, double timefac_re,
                        double timefac_im, double ztdpot, double* twoematel, double* outspfs);

/* ---------------------------------------------------------------------------
 * CI side: determinant list, walks, hops (host tables) and their device use
 * ------------------------------------------------------------------------- */
typedef struct sincgpu_walks sincgpu_walks;

/* Builds the determinant list and the walk/hop tables exactly as
 * fast_newconfiglist (MCTDH.SRC/newconfig.f90:349-1040), walks/getnumwalks
 * (MCTDH.SRC/walks.f90:149-759) and hops (walks.f90:761-993) do for a full CI of
 * numelec electrons in nspf orbitals at 2*M_s = restrictms (restrictflag=1,
 * numshells=1, holeflag=0, single rank).  nthreads <= 0: all host cores. */
int sincgpu_walks_create(sincgpu_walks** walks, int numelec, int nspf, int restrictms, int nthreads);
int sincgpu_walks_destroy(sincgpu_walks* walks);
/* sizes[0..5] = numconfig, numpart, total single walks, total double walks,
 * total single hops, total double hops. */
int sincgpu_walks_sizes(sincgpu_walks* walks, long long* sizes, int nsizes);

/* Copies one table as int32, 1-based values as in the reference:
 *   CONFIGLIST        configlist(2*numpart, numconfig)
 *   NUMSINGLEWALKS    (numconfig)          NUMDOUBLEWALKS (numconfig)
 *   SINGLEWALKOPSPF   (2, totsingle)       SINGLEWALKDIRPHASE, SINGLEWALK (totsingle)
 *   DOUBLEWALKDIRSPF  (4, totdouble)       DOUBLEWALKDIRPHASE, DOUBLEWALK (totdouble)
 *   SINGLEHOPOFF      (numconfig+1) CSR offsets into the flat hop arrays (0-based)
 *   SINGLEHOP, SINGLEHOPWALKSTART, SINGLEHOPWALKEND (totsinglehops), likewise DOUBLE*
 *   SINGLEDIAGHOP, DOUBLEDIAGHOP (numconfig): 1-based hop of config1 itself, -1 if none */
#define SINCGPU_T_CONFIGLIST 0
#define SINCGPU_T_NUMSINGLEWALKS 1
#define SINCGPU_T_NUMDOUBLEWALKS 2
#define SINCGPU_T_SINGLEWALKOPSPF 3
#define SINCGPU_T_SINGLEWALKDIRPHASE 4
#define SINCGPU_T_SINGLEWALK 5
#define SINCGPU_T_DOUBLEWALKDIRSPF 6
#define SINCGPU_T_DOUBLEWALKDIRPHASE 7
#define SINCGPU_T_DOUBLEWALK 8
#define SINCGPU_T_SINGLEHOPOFF 9
#define SINCGPU_T_SINGLEHOP 10
#define SINCGPU_T_SINGLEHOPWALKSTART 11
#define SINCGPU_T_SINGLEHOPWALKEND 12
#define SINCGPU_T_DOUBLEHOPOFF 13
#define SINCGPU_T_DOUBLEHOP 14
#define SINCGPU_T_DOUBLEHOPWALKSTART 15
#define SINCGPU_T_DOUBLEHOPWALKEND 16
#define SINCGPU_T_SINGLEDIAGHOP 17
#define SINCGPU_T_DOUBLEDIAGHOP 18
int sincgpu_walks_table(sincgpu_walks* walks, int which, int* out);

/* Spin walks, spin sets and S^2 projectors of the allspinproject=1 path
 * (MCTDH.SRC/spinwalks.f90: getnumspinwalks :302-388, spinwalks :86-153,
 * spinsets_first :156-299, configspin_matel :390-414, configspinset_projector
 * :432-642).  spinrestrictval is 2S; a negative value selects |restrictms| (the
 * reference's default high spin, MCTDH.SRC/getparams.f90:190-192).  Sets whose
 * projector has rank 0 are eliminated, as the reference does.  Call before
 * sincgpu_ci_attach so that the projectors are uploaded. */
int sincgpu_walks_spin(sincgpu_walks* walks, int spinrestrictval);

/* sizes[0..5] = number of kept spin sets, total spin rank (numspinconfig), total
 * spin walks, projector entries (sum of set size^2), eliminated configurations,
 * largest set size. */
int sincgpu_walks_spin_sizes(sincgpu_walks* walks, long long* sizes, int nsizes);

/* Spin tables as int32 (1-based configurations as in the reference): */
#define SINCGPU_T_NUMSPINWALKS 19     /* numconfig */
#define SINCGPU_T_SPINWALK 20         /* total spin walks, per config in order */
#define SINCGPU_T_SPINWALKDIRPHASE 21 /* total spin walks */
#define SINCGPU_T_SPINSETOFF 22       /* kept sets + 1 (CSR offsets into SPINSETS) */
#define SINCGPU_T_SPINSETS 23         /* configurations of the kept sets */
#define SINCGPU_T_SPINSETRANK 24      /* kept sets */
#define SINCGPU_T_SPINELIMINATED 25   /* configurations of eliminated sets */

/* Projectors of the kept sets, concatenated, each size x size row-major. */
int sincgpu_walks_spinprojectors(sincgpu_walks* walks, double* out);

/* Uploads the tables to the context's device (walk_init after hops in
 * MCTDH.SRC/mctdhf.f90:837-853).  The walks handle may be destroyed afterwards. */
int sincgpu_ci_attach(sincgpu_ctx* ctx, sincgpu_walks* walks);

/* getdenmatstuff (MCTDH.SRC/denmat.f90:312-378): denmat(n,n) from the A-vector
 * (getdenmat00, 177-274) and its regularised inverse invmatsmooth(denmat, denreg)
 * (MCTDH.SRC/utils.f90:533-611, denreg 1e-10).  invdenmat may be NULL. */
int sincgpu_getdenmat(sincgpu_ctx* ctx, const double* avector, double* denmat, double* invdenmat);
/* get_tworeducedx (MCTDH.SRC/mean.f90:14-152): reducedpottally(n,n,n,n). */
int sincgpu_get_tworeducedx(sincgpu_ctx* ctx, const double* avector1, const double* avector2,
                            double* reducedpottally);
/* One-body matrix elements <phi_i|op|phi_j>: potential (pot_matel, MCTDH.SRC/matel.f90:113-169),
 * kinetic (sparseops_matel, 241-293) and z (pulse_matel zz, 173-238). */
int sincgpu_onebody_matel(sincgpu_ctx* ctx, const double* phi, double* potmatel, double* kematel,
                          double* zmatel);
/* assemble_sparsemats (MCTDH.SRC/matel.f90:674-729; doubles 393-475): per
 * (config, hop) sums of the matrix elements over the hop's walks. */
int sincgpu_assemble_sparsemats(sincgpu_ctx* ctx, const double* twoematel, const double* potmatel,
                                const double* kematel, const double* zmatel);
/* sparseconfigmult with sparseopt=1 (MCTDH.SRC/walkmult.f90:735-907, boflag=1,
 * numr=1): out = nucrepulsion*in + doubles + one-body singles, plus with a
 * length-gauge z field ezfield: ezfield*(z singles + nuclear dipole*in). */
int sincgpu_sparseconfigmult(sincgpu_ctx* ctx, const double* invector, double* outvector, double ezfield);

/* Device forms of the above.  mats = [potmatel | kematel | zmatel] (3*n*n complex). */
int sincgpu_getdenmat_dev(sincgpu_ctx* ctx, const double* avector, double* denmat, double* invdenmat,
                          double denreg);
int sincgpu_get_tworeducedx_dev(sincgpu_ctx* ctx, const double* avector1, const double* avector2,
                                double* reducedpottally);
int sincgpu_onebody_matel_dev(sincgpu_ctx* ctx, const double* phi, double* mats);
int sincgpu_assemble_sparsemats_dev(sincgpu_ctx* ctx, const double* twoematel, const double* mats);
int sincgpu_sparseconfigmult_dev(sincgpu_ctx* ctx, const double* invector, double* outvector,
                                 double ezfield);

/* A-vector Krylov propagation, the expoavecprop -> DGEXPVxxx2 path
 * (MCTDH.SRC/expo_driver.f90:827-1055, MCTDH.SRC/expokit.f90:2222-2688):
 * avec_out = exp(t * timefac * H) avec_in with H the assembled CI Hamiltonian
 * (sparseconfigmult, including nucrepulsion and, for ezfield != 0, the z field),
 * Arnoldi of dimension krylovdim on the real-ified vector, (6,6) Pade of the
 * Hessenberg, local error control at tolerance tol (aerror).  *stepguess is the
 * first trial step on entry and the next call's guess on exit (the reference's
 * saved tempstepsize); *nstep receives the number of internal steps.  Config-basis
 * form: the spin-adapted basis transformation is not applied.  The reference scales
 * the operator by the step (cmf_prop_avector0, MCTDH.SRC/prop.f90:688-693) and calls
 * with t = 1, anorm = dt: pass timefac*dt and t = 1 to take the same decisions. */
int sincgpu_expoavecprop_dev(sincgpu_ctx* ctx, const double* avec_in, double* avec_out, double t,
                             double timefac_re, double timefac_im, int krylovdim, double tol, double anorm,
                             double ezfield, double* stepguess, int* nstep);
int sincgpu_expoavecprop(sincgpu_ctx* ctx, const double* avec_in, double* avec_out, double t,
                         double timefac_re, double timefac_im, int krylovdim, double tol, double anorm,
                         double ezfield, double* stepguess, int* nstep);

/* basis_project with allspinproject=1 (MCTDH.SRC/spin.f90:643-660 ->
 * configspin_project_general :339-375): each spin set's coefficients are
 * replaced by P_set times them; configurations of eliminated sets are zeroed.
 * Needs walk tables with spin sets attached. */
int sincgpu_spin_project_dev(sincgpu_ctx* ctx, double* avector);
int sincgpu_spin_project(sincgpu_ctx* ctx, const double* avector_in, double* avector_out);

/* z-dipole expectation (dipolesub_one, MCTDH.SRC/dipolesub.f90:20-125, the z
 * component with bra = ket): dipole = <A| Z A> + nucdipvalue_z <A|A> (complex, 2
 * doubles) with Z the configuration singles of <phi_i|z|phi_j> assembled by
 * sincgpu_assemble_sparsemats, and normsq = <A|A>; divide by normsq for the
 * normalised expectation. */
int sincgpu_dipole_z_dev(sincgpu_ctx* ctx, const double* avector, double* dipole, double* normsq);
int sincgpu_dipole_z(sincgpu_ctx* ctx, const double* avector, double* dipole, double* normsq);

/* One orbital-RHS evaluation from the A-vector: denmat, invdenmat and the 2-RDM
 * (get_allden, MCTDH.SRC/mean.f90:467-477), then sincgpu_orbital_rhs_dev. */
int sincgpu_orbital_rhs_avec_dev(sincgpu_ctx* ctx, const double* phi, const double* avector,
                                 double timefac_re, double timefac_im, double ztdpot, double* denmat,
                                 double* invdenmat, double* reducedpottally, double* twoematel,
                                 double* reducedpot, double* outspfs);

/* Host-array form: orbitals and A-vector in, orbital RHS out; the mean fields stay
 * on the device.  This is the call a Fortran driver makes per RHS evaluation when
 * it keeps the GPU state between calls.  The copies overlap the evaluation: the
 * A-vector goes up first (the RDMs start on it), the orbitals in groups (option
 * "rhs_upload_groups") under the Coulomb pair loop, and the RHS comes down while
 * twoematel, formed after it, runs; page-locked host buffers let the copies run
 * asynchronously.  Returns when the RHS is in outspfs. */
int sincgpu_orbital_rhs_avec(sincgpu_ctx* ctx, const double* phi, const double* avector,
                             double timefac_re, double timefac_im, double ztdpot, double* outspfs);

/* Orbital propagation, the expospfprop -> DGPHIV path of intopt=3
 * (MCTDH.SRC/expo_driver.f90:482-771 with jacinit0 :429-467 and jacoperate00
 * :40-259; MCTDH.SRC/expokit.f90:3904-4310; spf_linear_derivs
 * MCTDH.SRC/derivs.f90:1037-1186; spf_orthogit MCTDH.SRC/spfs.f90:120-196).
 * phi (device, totpoints x numspf complex) is advanced in place from tin to tout:
 * phi <- orthonormalised(phi + dt phi_1(dt J) f(phi)), J the orbital Jacobian.
 * The mean fields come as two slots (0: the end of the mean-field interval,
 * 1: its start), each denmat, invdenmat (numspf^2) and reducedpot
 * (totpoints x numspf^2); with linearflag they are blended with weights
 * ((t-firsttime)/(lasttime-firsttime), 1 - that) at the interval midpoint (the
 * reference's effective_cmf_linearflag), otherwise slot 0 alone is used and the
 * slot-1 pointers may be NULL.  ezfield is the z field at the midpoint.
 * *numiters receives the number of Jacobian products (iwsp(1)).  The Krylov
 * dimension and step guess persist in the context between calls, as the
 * reference's saved variables do; sincgpu_orbprop_setup resets them. */
int sincgpu_expospfprop_dev(sincgpu_ctx* ctx, double* phi, const double* denmat0, const double* invdenmat0,
                            const double* reducedpot0, const double* denmat1, const double* invdenmat1,
                            const double* reducedpot1, double tin, double tout, double firsttime,
                            double lasttime, int linearflag, double timefac_re, double timefac_im,
                            double ezfield, double expotol, int* numiters);

/* Parameters of the orbital propagator (expodim, maxexpodim, expostepfac and
 * par_timestep/littlesteps, MCTDH.SRC/parameters.f90:271-290); resets the saved
 * state.  maxexpodim must be at most 125. */
int sincgpu_orbprop_setup(sincgpu_ctx* ctx, int expodim, int maxexpodim, double expostepfac,
                          double first_stepsize);

/* Saved state of the orbital propagator: current Krylov dimension, next step
 * guess, the exposet flag and the call count. */
int sincgpu_orbprop_state(sincgpu_ctx* ctx, int* thisexpodim, double* tempstepsize, int* exposet,
                          int* icalled);

/* spf_orthogit (MCTDH.SRC/spfs.f90:120-196): two Loewdin passes
 * phi <- phi S^(-1/2), S = <phi|phi>, S^(-1/2) by SVD with singular values below
 * 1e-10 dropped (symorthogmat, MCTDH.SRC/utils.f90:947-1023).  *error (optional)
 * receives max|S - 1| of the final overlap. */
int sincgpu_spf_orthogit_dev(sincgpu_ctx* ctx, double* phi, double* error);

/* Orbital and A-vector files in the reference's format (gfortran unformatted
 * sequential records; save_vector / write_spf / spf_header_write,
 * MCTDH.SRC/loadstuff.f90:9-180; avector_header_write / write_avector /
 * easy_load_avectors, MCTDH.SRC/configload.f90:221-249, 801-863).  Host arrays;
 * dims are spfdims(3) (numpoints per axis for the sinc project).  Loading an
 * A-vector reorders each stored determinant, applies the reordering phase and
 * maps it onto the walk tables' configuration list (numr = 1, complex files).
 * sincgpu_load_spfs with spfs = NULL reads the header only. */
int sincgpu_save_spfs(const char* path, const int* dims, int numspf, const double* spfs);
int sincgpu_load_spfs(const char* path, int* dims, int* numspf, double* spfs, long long capacity);
int sincgpu_save_avector(const char* path, sincgpu_walks* walks, int numvects, const double* avectors,
                         int allspinproject, int spinrestrictval);
int sincgpu_load_avector(const char* path, sincgpu_walks* walks, int maxvects, double* avectors, int* numvects);

/* CUDA-graph form of sincgpu_orbital_rhs_avec_dev: one warm-up evaluation, then
 * the same call captured into a graph kept in the context (all arguments are
 * device pointers baked into the graph).  sincgpu_rhs_graph_launch replays it on
 * the context stream. */
int sincgpu_rhs_graph_capture(sincgpu_ctx* ctx, const double* phi, const double* avector, double timefac_re,
                              double timefac_im, double ztdpot, double* denmat, double* invdenmat,
                              double* reducedpottally, double* twoematel, double* reducedpot, double* outspfs);
int sincgpu_rhs_graph_launch(sincgpu_ctx* ctx);

/* A batch: the captured graphs of n contexts (instances of any size on one
 * device) as independent child nodes of one parent graph, launched at once. */
typedef struct sincgpu_batch sincgpu_batch;
int sincgpu_batch_create(sincgpu_batch** batch, sincgpu_ctx** ctxs, int n);
int sincgpu_batch_launch(sincgpu_batch* batch, void* stream);
int sincgpu_batch_destroy(sincgpu_batch* batch);

/* Autotuner: times the orbital-RHS evaluation (a warm-up, then the mean of
 * three) and tunes three launch-shape options in turn, each kept at its fastest
 * value in the context before the next: the Coulomb pair chunk (automatic, all
 * pairs, 1/2, 1/4, 16, 8; "coul_chunk"), the twoematel tile edge 16R (automatic,
 * R = 4..9; "twoe_tile") and the TMA-staged z pass ("coul_tma").  A fixed value
 * must beat the current one by 2 %.  Returns the chunk and the best time; the
 * others are read with sincgpu_get_option. */
int sincgpu_autotune_rhs(sincgpu_ctx* ctx, const double* phi, const double* avector, double* denmat,
                         double* invdenmat, double* reducedpottally, double* twoematel, double* reducedpot,
                         double* outspfs, int* best_chunk, float* best_ms);

/* Constant-mean-field propagation (cmf_prop_wfn, MCTDH.SRC/prop.f90:230-574, with
 * prepropflag=1, step_flag=2, postpropflag=2; orbitals by expospfprop/DGPHIV,
 * A-vector by expoavecprop/DGEXPVxxx2 followed by the spin projection, mean fields
 * and CI matrices in two time slots blended linearly).  Parameters as the
 * reference's namelist: par_timestep, littlesteps, expotol, aerror, aorder,
 * maxaorder (<= 124), expodim, maxexpodim (<= 125), expostepfac, denreg
 * (MCTDH.SRC/parameters.f90:244-295) and timefac (-i for real time). */
int sincgpu_cmf_setup(sincgpu_ctx* ctx, double par_timestep, int littlesteps, double expotol, double aerror,
                      int aorder, int maxaorder, int expodim, int maxexpodim, double expostepfac, double denreg,
                      double timefac_re, double timefac_im);

/* Length-gauge pulses (MCTDH.SRC/pulse.f90:8-52 tdpotlen0 and pulse types 1-5,
 * :149-372).  params holds 8 doubles per pulse: omega, omega2, pulsestart,
 * phaseshift, pulsestrength, longstep, pulsetheta, (unused).  Only z-polarised
 * pulses (sin(pulsetheta) = 0) are supported. */
int sincgpu_cmf_pulses(sincgpu_ctx* ctx, int npulses, const int* pulsetype, const double* params);
/* z component of the field at time t. */
int sincgpu_pulse_ez(sincgpu_ctx* ctx, double t, double* ez);

/* Start of a propagation (prop_loop, MCTDH.SRC/prop.f90:811-852): the A-vector is
 * spin projected, the mean fields and CI matrices of (phi, avector) are built
 * (get_stuff) and *energy0 receives <A|H A>/<A|A> with the field at t = 0.
 * phi and avector are device arrays; the context keeps its own copies.  Needs
 * walk tables attached (with spin sets for allspinproject=1). */
int sincgpu_cmf_init_dev(sincgpu_ctx* ctx, const double* phi, const double* avector, double* energy0);

/* One CMF step from tin to tout on the resident state; *energy = <A|P H A>/<A|A>
 * at tout without the field (timedepexpect=0), *norm = |A|, and the numbers of
 * Jacobian products (orbitals) and sigma products (A-vector) in the step. */
int sincgpu_cmf_step(sincgpu_ctx* ctx, double tin, double tout, double* energy, double* norm, int* orb_iters,
                     int* avec_iters);

/* z dipole of the current CMF state (as sincgpu_dipole_z, with the CI matrices of
 * the current orbitals). */
int sincgpu_cmf_dipole_z(sincgpu_ctx* ctx, double* dipole, double* normsq);

/* Copies the current orbitals and A-vector to device arrays (either may be NULL). */
int sincgpu_cmf_state_dev(sincgpu_ctx* ctx, double* phi, double* avector);

/* Served form: a device-resident request loop.  Requests (a sinc-DVR system,
 * electrons and 2Ms, pulses, number of CMF steps of length dt, initial orbitals
 * (totpoints x numspf complex) and A-vector (host arrays, copied at submit)) are
 * admitted by max_active worker threads while the HBM budget (0: 85% of the free
 * memory) allows; each live request keeps its orbitals, A-vector, mean fields
 * and walk tables on the device in its own context and stream until it finishes,
 * so requests arriving while others run join as slots and memory free up and
 * their work overlaps on the device.  Results are deterministic: a request gives
 * the same numbers alone or in a mix.  The server reserves its HBM budget in the
 * device's stream-ordered memory pool when it is created (the requests' device
 * allocations come out of that reservation, so that none of them waits in the
 * driver for new memory while other requests run) and gives it back when it is
 * destroyed.  A request whose tensor-core contraction or staged Coulomb pass gave
 * up a bounded wait fails with SINCGPU_ETIMEOUT. */
typedef struct sincgpu_request {
  int numpoints;
  double spacing;
  int numcenters;
  const int* centershift;    /* 3 x numcenters, half-grid units */
  const double* nuccharges;  /* numcenters */
  int numspf, numelec, restrictms, spinrestrictval;  /* spinrestrictval < 0: |restrictms| */
  int npulses;
  const int* pulsetype;      /* as sincgpu_cmf_pulses */
  const double* pulseparams; /* 8 per pulse */
  int nsteps;
  double dt;
  int coulomb_fp32;          /* precision form: FP32 Coulomb passes and 3xTF32 tensor-core reducedpot */
  int keep_state;            /* keep the final orbitals and A-vector for sincgpu_server_result_arrays */
  const double* phi;
  const double* avector;
} sincgpu_request;
typedef struct sincgpu_server sincgpu_server;
int sincgpu_server_create(sincgpu_server** server, int device, long long hbm_budget, int max_active);
int sincgpu_server_submit(sincgpu_server* server, const sincgpu_request* request, int* id);
/* Blocks until request id finished: initial and final energy, norm, normalised z
 * dipole, steps done; non-zero status if the request failed. */
int sincgpu_server_wait(sincgpu_server* server, int id, double* energy0, double* energy, double* norm,
                        double* dipole_z, int* nsteps_done);
/* Per-step latencies (ms) and energies of a finished request; final orbitals and
 * A-vector when it was submitted with keep_state.  Any pointer may be NULL. */
int sincgpu_server_result_arrays(sincgpu_server* server, int id, double* step_ms, double* energies, double* phi,
                                 double* avector);
/* Timeline of a finished request in ms since the server was created: times[0] =
 * submitted, times[1] = admitted to a slot, times[2] = context and CMF state ready
 * (set-up done), times[3] = finished; step_start[k] = start of CMF step k.  Any
 * pointer may be NULL. */
int sincgpu_server_timeline(sincgpu_server* server, int id, double* times, double* step_start);
/* counts[0..4] = admitted, completed, steps, peak concurrent requests, pending;
 * p50 / p99 of all finished steps' latencies (ms); steps per second between the
 * first admission and the last completion. */
int sincgpu_server_stats(sincgpu_server* server, long long* counts, double* p50_ms, double* p99_ms,
                         double* steps_per_s);
/* Finishes all submitted requests, stops the workers and frees the server. */
int sincgpu_server_destroy(sincgpu_server* server);

#ifdef __cplusplus
}
#endif
#endif /* SINCGPU_H */
