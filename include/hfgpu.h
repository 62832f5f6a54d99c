/* hfgpu: B200 two-electron engine for hfscf -- C ABI.
 *
 * The entry points replace the reference's two-electron hot path:
 *   - ERIOS::Erios (src/integrals/hfscf_oseri.hpp:27-123): Obara-Saika ERIs,
 *     Schwarz diagonal, first-derivative ERIs;
 *   - Mol::hf_solver::update_fock_matrix (src/scfsolver/hfscf_hf_solver.cpp:254-286)
 *     and Mol::uhf_solver::update_fock_matrix (src/scfsolver/hfscf_uhf_solver.cpp:155-191);
 *   - the two-electron term of Mol::scf_gradient::calc_scf_gradient_rhf/uhf
 *     (src/gradient/hfscf_grad_rhf.cpp:76-141, src/gradient/hfscf_grad_uhf.cpp:124-150).
 *
 * Conventions (all as in the reference):
 *   - matrices are n x n, row-major, FP64; n = number of pure or Cartesian functions;
 *   - function order: atoms in input order, shells in basis-file order, Cartesian
 *     components l = L-i, m = i-j, n = j, pure components m = -L..L;
 *   - densities carry no factor 2 (RHF D = C_occ C_occ^T), F = H + 2J[D] - K[D];
 *   - J[D]_ij = sum_kl D_kl (ij|kl), K[D]_ij = sum_kl D_kl (ik|jl).
 *
 * Every call returns an hfgpu_status (0 = success) and never exits the process.
 * A handle is not thread-safe: serialise calls on one handle.  Host-pointer entry
 * points copy inputs to the device and results back, synchronising the handle's
 * stream; *_device entry points take device pointers and enqueue on that stream.
 */
#ifndef HFGPU_H
#define HFGPU_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct hfgpu_handle hfgpu_handle;

typedef enum {
  HFGPU_OK = 0,
  HFGPU_ERR_INVALID = 1,     /* bad argument or basis (e.g. L > 2, non-finite exponent) */
  HFGPU_ERR_NOMEM = 2,       /* device or host allocation failed */
  HFGPU_ERR_CUDA = 3,        /* CUDA runtime error; see hfgpu_last_error */
  HFGPU_ERR_STATE = 4,       /* call out of order (e.g. no geometry set) */
  HFGPU_ERR_NONFINITE = 5,   /* a result was NaN or Inf */
  HFGPU_ERR_UNSUPPORTED = 6  /* feature not available in this build */
} hfgpu_status;

typedef enum { HFGPU_FP64 = 0, HFGPU_MIXED = 1 } hfgpu_precision;

/* Basis description: flat arrays, as BASIS::Shell takes them
 * (src/integrals/hfscf_shell.hpp:21-57).  Coefficients are the UNNORMALISED
 * values of the basis file; the engine normalises them as the reference's
 * Shell constructor does (src/integrals/hfscf_shell.cpp:44-54). */
typedef struct {
  int nshell;
  int natoms;
  int pure;                /* 1 = spherical functions, 0 = Cartesian */
  const int* L;            /* [nshell] angular momentum, 0..2 */
  const int* shell_atom;   /* [nshell] atom of each shell */
  const int* nprim;        /* [nshell] primitives per shell */
  const double* exps;      /* [sum nprim] exponents */
  const double* coefs;     /* [sum nprim] contraction coefficients */
} hfgpu_basis;

typedef struct {
  double schwarz_tol;      /* quartets with Q_ab Q_cd below this are never computed (default 1e-12,
                              the reference's screen_tol = 100 * integral_tol, hfscf_oseri.hpp:31-32) */
  double density_tol;      /* J/K: skip quartets whose density-weighted bound is below this (default 1e-12; 0 = off) */
  double mixed_fp32_bound; /* mixed precision: quartets with Q_ab Q_cd below this run in FP32 (default 1e-4) */
  double mixed_density_tol;/* density-weighted threshold of mixed-precision Delta-D builds (hfgpu_fock_delta
                              with HFGPU_MIXED; default 1e-12 as for full builds: a looser 1e-10 made the
                              incremental SCF of n-octane take 44 iterations instead of 24) */
  int device;              /* CUDA device ordinal (default 0) */
  int warp_max_quartets;   /* (dd|dp), (dd|dd): one warp per quartet when the class has at most this many
                              quartets, one thread per quartet otherwise (default 2^30 = always; -1 = never) */
  int grad_warp_max_waves;    /* gradient of (dp|dp) (dd|pp) (dd|ds) (dd|dp) (dd|dd) before any
                                 hfgpu_autotune_grad / hfgpu_set_grad_forms: > 0 (default 48) one block of
                                 four warps per quartet over shared-memory tables (form 3), 0 = one thread
                                 per quartet on global scratch (form 0) */
  int reserved[5];          /* reserved[0] = 1: arm every shared-memory staging wait without issuing its copy,
                              so that the bounded wait runs out (tests the timeout path; builds then report
                              status 2); 0 otherwise.  reserved[1] > 0: at most this many blocks per
                              straight-line gradient launch (default 2048; the launch loops over the rest).
                              reserved[2..4]: 0. */
} hfgpu_opts;

int hfgpu_default_opts(hfgpu_opts* opts);

/* Replaces constructing Erios + Molecule::create_shell_pairs
 * (src/integrals/hfscf_oseri.hpp:30-32, src/molecule/hfscf_molecule.cpp:661-669). */
int hfgpu_create(const hfgpu_basis* basis, const hfgpu_opts* opts, hfgpu_handle** out);
int hfgpu_destroy(hfgpu_handle* h);
const char* hfgpu_last_error(const hfgpu_handle* h);
int hfgpu_nbf(const hfgpu_handle* h, int* nbf);
/* Stream for all device work of this handle (cudaStream_t passed as void*; NULL = handle's own). */
int hfgpu_set_stream(hfgpu_handle* h, void* stream);

/* Atom coordinates in bohr, natoms x 3.  Rebuilds primitive-pair data, the Schwarz
 * factors and the screened quartet lists (replaces ShellPair::set_params,
 * src/integrals/hfscf_shellpair.cpp:33-61, and Erios::compute_screen_matrix,
 * src/integrals/hfscf_oseri_screen.cpp:22-181). */
int hfgpu_set_geometry(hfgpu_handle* h, const double* xyz_bohr, int natoms);

/* Shell-pair Schwarz factors sqrt(max |(ab|ab)|), nshell x nshell (symmetric). */
int hfgpu_schwarz(hfgpu_handle* h, double* Q_out);

/* Every unique ERI into the reference's packed 8-fold vector of length
 * n(n+1)(n^2+n+2)/8, indexed by hfscfmath::index_ijkl (src/math/hfscf_math.hpp:90-101).
 * Replaces Mol::hf_solver::create_repulsion_matrix (src/scfsolver/hfscf_hf_hamiltonian.cpp:67-112).
 * No screening is applied. */
int hfgpu_eri_packed(hfgpu_handle* h, double* eri_out, long long eri_len);

/* J[DJ] (if DJ != NULL) and K[DK[m]] for m < nK.  J: n x n, K: nK x n x n. */
int hfgpu_jk(hfgpu_handle* h, const double* DJ, int nK, const double* DK, double* J, double* K, int precision);

/* RHF: F = H + 2 J[D] - K[D] (src/scfsolver/hfscf_hf_solver.cpp:261-278). */
int hfgpu_fock_rhf(hfgpu_handle* h, const double* D, const double* H, double* F, int precision);

/* UHF: F_a = H + J[Da+Db] - K[Da], F_b = H + J[Da+Db] - K[Db]
 * (src/scfsolver/hfscf_uhf_solver.cpp:160-180). */
int hfgpu_fock_uhf(hfgpu_handle* h, const double* Da, const double* Db, const double* H, double* Fa, double* Fb,
                   int precision);

/* Incremental RHF build: F_inout += 2 J[dD] - K[dD], with density screening on |dD|. */
int hfgpu_fock_delta(hfgpu_handle* h, const double* dD, double* F_inout, int precision);

/* Autograd-shaped pair for the two-electron energy E2 = sum_ij D_ij (2J[D] - K[D])_ij.
 * forward: E2 at the current geometry.
 * backward: dE_dR (natoms x 3) += scale * dE2/dR at fixed D, contracting first-derivative
 * ERIs with the density on the fly; derivative integrals are recomputed, never stored. */
int hfgpu_energy_forward(hfgpu_handle* h, const double* D, double* E2, int precision);
int hfgpu_grad2e_backward(hfgpu_handle* h, const double* D, double scale, double* dE_dR, int precision);
/* UHF: E2 = 1/2 [sum Dt J[Dt] - sum Da K[Da] - sum Db K[Db]], Dt = Da + Db. */
int hfgpu_grad2e_uhf_backward(hfgpu_handle* h, const double* Da, const double* Db, double scale, double* dE_dR,
                              int precision);

/* Two-electron part of the analytic Hessian at a fixed density, replacing the reference's
 * second-derivative ERI tensors and their contraction in Mol::scf_hessian::calc_scf_hessian_tei
 * (src/hessian/hfscf_hessian_ints.cpp:20-303; Erios::compute_contracted_shell_quartet_deriv2_qq/_pq,
 * src/integrals/hfscf_oserideriv2qq.cpp:28-853, hfscf_oserideriv2pq.cpp:23-891).
 * hess (3 natoms x 3 natoms, row-major) += scale * d2E2/dX dY with E2 as for
 * hfgpu_grad2e_backward: for RHF the reference's m_hessianC + m_hessianEx.  Second-derivative
 * integrals are recomputed per quartet and contracted with the density on the fly, never stored.
 * FP64 only; single-molecule handles (HFGPU_ERR_UNSUPPORTED for a batched handle). */
int hfgpu_hess2e(hfgpu_handle* h, const double* D, double scale, double* hess);
int hfgpu_hess2e_uhf(hfgpu_handle* h, const double* Da, const double* Db, double scale, double* hess);
/* Launch form of the Hessian classes: -1 (default) one thread per quartet on straight-line
 * register code for the many-quartet classes that have it ((ss|ss), (ps|ss), (ps|ps), (pp|ss),
 * (pp|ps), (ds|ss), (ds|ps), (dp|ss)), else one block of 128
 * threads per quartet for the classes with large op tables or few quartets and one warp per
 * quartet for the others; 0 one thread per quartet on global scratch everywhere, 1 one block per
 * quartet everywhere, 2 one warp per quartet wherever four quartets' tables fit one block (the
 * block form elsewhere), 3 the straight-line form wherever the class has it (the default
 * elsewhere).  The results agree to rounding. */
int hfgpu_set_hess_form(hfgpu_handle* h, int form);
/* Per class (HFGPU_NUM_CLASSES ints: 0 thread, 1 block, 2 warp, 3 straight-line, -1 the rule of
 * hfgpu_set_hess_form), as hfgpu_autotune_hess returns them. */
int hfgpu_set_hess_forms(hfgpu_handle* h, const int* forms);
/* Times every class alone in each form on RHF weights of the device density D (median of
 * `repeats` runs, L2 flushed before each) and keeps the faster per class; forms (may be NULL)
 * receives the choice.  No counterpart in the reference (which has one CPU code path). */
int hfgpu_autotune_hess(hfgpu_handle* h, const double* D, int repeats, int* forms);

/* Device-pointer variants (enqueue on the handle's stream, no host synchronisation). */
/* hess (device, 3 natoms x 3 natoms) += sum W d2(ab|cd)/dX dY with the weights of
 * hfgpu_grad2e_device (RHF: DJ = D, cJ = 2, DK = D, cK = 1). */
int hfgpu_hess2e_device(hfgpu_handle* h, const double* DJ, double cJ, int nK, const double* DK, double cK,
                        double* hess);
int hfgpu_jk_device(hfgpu_handle* h, const double* DJ, int nK, const double* DK, double* J, double* K,
                    int precision);
int hfgpu_grad2e_device(hfgpu_handle* h, const double* DJ, double cJ, int nK, const double* DK, double cK,
                        double* grad, int precision);

/* Same result as hfgpu_grad2e_device, for callers that cannot allocate device memory
 * while they run (their allocator owns the device, or allocation is forbidden after
 * start-up).  No counterpart in the reference.  Allocates nothing: the scratch of the
 * large gradient classes comes from a fixed array of hfgpu_noalloc_scratch_bytes()
 * (32 MiB) inside the library, held on every device that loads it until exit; a
 * class whose smallest launch does not fit returns HFGPU_ERR_INVALID.  The first call
 * on a device looks up the array's address (make it before any stream capture); all
 * calls share the array, so calls that overlap on the GPU race.  Runs on the handle's
 * stream; grad is accumulated into, as in hfgpu_grad2e_device. */
int hfgpu_grad2e_device_noalloc(hfgpu_handle* h, const double* DJ, double cJ, int nK, const double* DK, double cK,
                                double* grad, int precision);
long long hfgpu_noalloc_scratch_bytes(void);

/* Batched handles: many independent molecules in one handle (hundreds of small molecules,
 * e.g. water clusters, methane, ethane and ammonia in STO-3G or 6-31G*).  No counterpart in
 * the reference, which runs one molecule per process.
 * Shell pairs and quartets are formed within each molecule only; every per-class kernel
 * launch covers all molecules.  Matrices live in a block storage: molecule m's n_m x n_m
 * row-major block starts at mat_off[m].  Molecules must be Cartesian (pure = 0); for s and
 * p shells the two are the same functions.  RHF only (one density).  Atoms are numbered
 * consecutively over the molecules for the gradient. */
int hfgpu_batch_create(int nmol, const hfgpu_basis* bases, const double* const* xyz_bohr, const hfgpu_opts* opts,
                       hfgpu_handle** out);
int hfgpu_batch_layout(const hfgpu_handle* h, int* nbf, long long* mat_off, long long* mat_total);
/* J[D], K[D] for every molecule; D, J, K device pointers to block storage. */
int hfgpu_batch_jk_device(hfgpu_handle* h, const double* D, double* J, double* K, int precision);
/* grad (device, total atoms x 3) += two-electron RHF gradient of every molecule. */
int hfgpu_batch_grad2e_device(hfgpu_handle* h, const double* D, double* grad, int precision);
/* Eigenvalues W (nmol x nmax, ascending) and eigenvectors V (nmol x nmax x nmax, columns) of
 * every molecule's symmetric matrix in A (nmol x nmax x nmax, padded; nmax = the largest
 * molecule's function count, at most 118), for the batched SCF's diagonalisation step; the
 * reference diagonalises one molecule with Eigen (src/scfsolver/hfscf_hf_solver.cpp:206-242).
 * Cyclic Jacobi, one thread block per molecule; entries outside a molecule's block pass
 * through as identity eigenvectors.  sweeps (device, nmol ints, may be NULL) receives the
 * Jacobi sweeps each molecule took.  Device pointers, enqueued on the handle's stream. */
int hfgpu_batch_eigh(hfgpu_handle* h, const double* A, double* W, double* V, int* sweeps);
/* The batched SCF's density step without a diagonalisation: P (nmol x nmax x nmax, padded, zero
 * outside each block) = the projector onto the nocc[b] lowest eigenvectors of every molecule's
 * orthonormal-basis Fock block in Fo (same layout), by trace-correcting purification, one thread
 * block per molecule with the matrix in shared memory (molecules of up to 116 functions); each
 * stops at its own converged step.  err[b] (device) = tr P - tr P^2 there, or 1 when max_steps did
 * not converge (diagonalise that iteration instead).  nocc: device ints.  Replaces, for a
 * closed-shell density, the diagonalisation of Mol::hf_solver::calc_density_matrix
 * (src/scfsolver/hfscf_hf_solver.cpp:206-231).  Enqueued on the handle's stream. */
int hfgpu_batch_purify_device(hfgpu_handle* h, const double* Fo, const int* nocc, int max_steps, double* P,
                              double* err);

/* One-electron matrices S, T, V (n x n) for the basis at xyz (bohr), on the host CPU.
 * Z: nuclear charges per atom.  Needs no handle and no GPU (the reference's
 * OSOverlap/OSKinetic/OSNuclear, src/integrals/hfscf_osoverlap.cpp:10, hfscf_osnuclear.cpp:17);
 * the handle-based device versions follow below. */
int hfgpu_one_electron(const hfgpu_basis* basis, const double* xyz_bohr, const double* Z, double* S, double* T,
                       double* V);
/* grad (natoms x 3) += cH sum D_ij d(T+V)_ij/dX + cS sum W_ij dS_ij/dX, including the
 * Hellmann-Feynman term of every nucleus.  The reference's RHF gradient
 * (src/gradient/hfscf_grad_rhf.cpp:140-167) is cH = 2 with D and cS = -2 with Q = D F D. */
int hfgpu_one_electron_grad(const hfgpu_basis* basis, const double* xyz_bohr, const double* Z, const double* D,
                            const double* W, double cH, double cS, double* grad);

/* The same one-electron matrices and gradient on the GPU, for the handle's basis and current
 * geometry (reference routines as above, and the per-atom assembly of
 * src/gradient/hfscf_grad_ints.cpp:14-77,153-199).  Z: nuclear charge per atom (host array;
 * a batched handle takes every molecule's atoms in order).  S, T, V, D, W and grad are device
 * pointers: n x n matrices (block storage for a batched handle) and natoms x 3; V is
 * overwritten, grad accumulated.  Enqueued on the handle's stream. */
int hfgpu_one_electron_device(hfgpu_handle* h, const double* Z, double* S, double* T, double* V);
int hfgpu_one_electron_grad_device(hfgpu_handle* h, const double* Z, const double* D, const double* W, double cH,
                                   double cS, double* grad);

/* SCF density without a diagonalisation: P (n x n, device) = the projector onto the nocc lowest
 * eigenvectors of the symmetric orthonormal-basis Fock matrix Fo (device), by trace-correcting
 * purification (at most max_steps <= 256 squarings; it stops changing P once tr P - tr P^2 <
 * 1e-11).  *err (device double) receives that tr P - tr P^2 at convergence, or 1 if it did not
 * converge in max_steps (then diagonalise instead).  Replaces the diagonalisation of
 * Mol::hf_solver::calc_density_matrix (src/scfsolver/hfscf_hf_solver.cpp:206-231) for a
 * closed-shell density: C_occ C_occ^T is that projector.  Enqueued on the handle's stream. */
int hfgpu_purify_device(hfgpu_handle* h, const double* Fo, int n, int nocc, int max_steps, double* P, double* err);
/* Launch form of hfgpu_purify_device: 1 (default) one cooperative launch whose blocks meet at a
 * grid-wide barrier between the phases of a step and all stop at the step that converged (when
 * the device supports cooperative launches), 0 two launches per step for every step. */
int hfgpu_set_purify_mode(hfgpu_handle* h, int cooperative);

/* Counters of the last J/K build: quartets launched and quartets skipped by density screening. */
int hfgpu_last_counts(const hfgpu_handle* h, long long* launched, long long* skipped);

/* Measurement hooks (no counterpart in the reference, which has no GPU path).
 * set_timing: record CUDA events around every per-class kernel of later J/K builds.
 * class_stats(cls, out[9]): la lb lc ld, screened quartets, quartets at/above the mixed-precision
 *   bound, and from the last J/K build: quartets computed, skipped by density, primitive quartets computed.
 * class_time: event time (ms) of that class's kernels in the last J/K build.
 * last_launches: kernel launches of the last J/K (or Fock) build.
 * fp64_peak: FP64 FMA throughput of the device in TFLOP/s, from a register-only FMA kernel.
 * setup_times(ms[4]): host wall time (ms) of the last hfgpu_set_geometry (or create): primitive
 *   pairs, Schwarz factors, quartet lists built on the host, their upload to the device. */
int hfgpu_set_timing(hfgpu_handle* h, int on);
int hfgpu_class_stats(hfgpu_handle* h, int cls, long long* out);
int hfgpu_class_time(hfgpu_handle* h, int cls, float* ms);
/* Work of class cls in the current geometry's lists, independent of any build: out[0] =
 * Schwarz-screened quartets (all of them are computed by a gradient), out[1] = their primitive
 * quartets (kept primitive pairs of the bra times those of the ket).  No host synchronisation. */
int hfgpu_class_work(const hfgpu_handle* h, int cls, long long* out);
/* Partition of one molecule's work over nparts devices (or passes): later J/K builds and
 * two-electron gradients of this handle process only the quartets numbered part, part + nparts,
 * part + 2 nparts, ... of every class list (the lists are ordered by bound and primitive count,
 * so the parts cost about the same), and their J, K, E2 and gradient outputs are this part's
 * terms; summed over the nparts parts they equal the unpartitioned outputs up to FP64 summation
 * order (the density screening decides on the same device bounds in every part).  The Fock
 * entry points (fock_rhf, fock_uhf, fock_delta), which add H, return HFGPU_ERR_STATE on a
 * partitioned handle.  nparts = 1 (the default) ends the partition.  No reference counterpart
 * (the reference's Fock build and gradient are one OpenMP loop on one host). */
int hfgpu_set_partition(hfgpu_handle* h, int part, int nparts);
int hfgpu_last_launches(const hfgpu_handle* h, int* kernels);
/* Device status word of the handle's kernels since the last call, then cleared (synchronises
 * the handle's stream): 0 = fine; 2 = a block's wait for its shared-memory staging copy ran
 * out (bounded at about 0.1 s; the block skipped its quartets, so that build is incomplete);
 * 3 = a persistent launch stopped at a host abort request.  The host-pointer entry points
 * check it themselves and return HFGPU_ERR_CUDA for status 2 and HFGPU_ERR_STATE for status 3.  No reference
 * counterpart (the reference has no device code and exits on errors). */
int hfgpu_device_status(hfgpu_handle* h, int* status);
/* Host abort flag (on = 1) or its reset (on = 0), written on a stream of its own so that it
 * lands while builds run: the persistent launches (schedule variant 2) stop between two chunks
 * of 32 quartets and record status 3; a build running then is incomplete.  The flag stays set
 * until reset.  No reference counterpart. */
int hfgpu_request_abort(hfgpu_handle* h, int on);
int hfgpu_fp64_peak(int device, double* tflops);
/* Boys function F_0..F_m (m <= 10) at count points T >= 0 (host arrays; F is count x (m+1)),
 * through the same table and evaluation the quartet kernels use, in FP64 (HFGPU_FP64) or in
 * the FP32 form of the mixed-precision kernels (HFGPU_MIXED; T is rounded to float first).
 * The reference's counterpart is extramath::F_nu (src/math/gamma.cpp:18-24), which evaluates
 * T < 1e-8 at T = 1e-8; this routine does not clamp. */
int hfgpu_boys(hfgpu_handle* h, int precision, int m, const double* T, long long count, double* F);
int hfgpu_setup_times(const hfgpu_handle* h, double* ms);

/* Launch schedule of the J/K build (no reference counterpart: the reference has one CPU
 * code path).  Four ints per quartet class, HFGPU_NUM_CLASSES classes in the order of
 * hfgpu_class_stats:
 *   [0] threads per block of the thread-per-quartet form (32, 64, 128);
 *   [1] lanes per quartet of the primitive-split form used for quartets with at least 16
 *       primitive quartets (4, 8, 16, 32; 1 = 32; 0 = thread form; classes without that
 *       form ignore it);
 *   [2] 2/1/0/-1 = block-per-quartet form (128 threads per quartet) / warp-per-quartet form
 *       (four quartets per 128-thread block) for the classes that have one, (dp|pp) (dp|ds)
 *       (dp|dp) (dd|pp) (dd|ds) (dd|dp) (dd|dd) / thread forms (-1 = follow
 *       opts.warp_max_quartets with the warp form);
 *   [3] variant of the thread-per-quartet form: 0 plain; 1 register-capped, for more warps
 *       per SM (the small classes (ps|ss) ... (dp|ss) have one); 2 persistent, with the
 *       class's Boys table staged into shared memory by one bulk (TMA) copy per block (the
 *       classes of total angular momentum <= 4 have one); 3 at most two blocks per SM, so that
 *       the spilled registers of the large classes stay in L2 (classes with 250 or more VRR
 *       values have one); classes without the variant ignore it.
 * Default: 64, 0, -1 for (dd|dp) and (dd|dd) else 0, 0.
 * autotune: times every form of every class on the current geometry with device density D
 * (n x n; `repeats` builds per candidate, one class at a time on the handle's stream),
 * keeps the fastest; then, on whole builds, tries per class the best candidate of each other
 * kind of form (thread, primitive-split, warp or block) and keeps it where the build gets at least 1%
 * faster; keeps the result only if whole builds with it beat whole builds with the schedule
 * it started from, and returns the schedule in `schedule` (may be NULL).  Last, it times the
 * classes of a build one after another on one stream against concurrently on six and keeps
 * the serial order where it is at least 1% faster (the handle keeps that choice; it is not
 * part of the schedule array).  Every timing is the median of separately timed runs, each
 * after an L2 flush.
 * Results of later builds do not depend on the schedule beyond FP64 summation order. */
#define HFGPU_NUM_CLASSES 21
int hfgpu_autotune(hfgpu_handle* h, const double* D, int precision, int repeats, int* schedule);
int hfgpu_set_schedule(hfgpu_handle* h, const int* schedule);
/* Gradient form per class for the classes that have several (the op-table classes (dp|dp) (dd|pp)
 * (dd|ds) (dd|dp) (dd|dd)): times one warp or one 128- or 256-thread block per quartet (whole or split
 * per set) against one thread per quartet for each class alone on the handle's lists and the
 * given device density D (RHF weights), keeps the fastest; then, on whole gradients, tries the
 * other forms per class and keeps one where it makes the gradient at least 1% faster (the
 * classes run concurrently; last, one after another on one stream against concurrently, as for
 * the J/K build), and returns the forms in forms[HFGPU_NUM_CLASSES] (0 thread, 1 warp,
 * 2 warp split into four launches of one accumulator set each, 3 block of four warps, 4 block
 * split into four launches, 5 and 6 the same with blocks of eight warps, -1 class without a
 * choice; may be NULL).  Until it runs, the
 * classes use form 3 (opts.grad_warp_max_waves > 0) or form 0 (opts.grad_warp_max_waves = 0).
 * Results do not depend on the form beyond FP64 summation order. */
int hfgpu_autotune_grad(hfgpu_handle* h, const double* D, int precision, int repeats, int* forms);
/* Sets the gradient forms directly (HFGPU_NUM_CLASSES ints, -1 .. 6, as hfgpu_autotune_grad returns them;
 * -1 = the default of opts.grad_warp_max_waves; ignored for classes without a choice). */
int hfgpu_set_grad_forms(hfgpu_handle* h, const int* forms);
int hfgpu_get_schedule(const hfgpu_handle* h, int* schedule);

#ifdef __cplusplus
}
#endif
#endif
