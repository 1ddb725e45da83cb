/*
 * dss.h -- C ABI of the B200 Fock-build engine for DollarStoreSCF.
 *
 * All matrices crossing this boundary on the host are symmetric n x n matrices in
 * the reference's packed-upper column-major layout (LAPACK 'U' packed): element
 * (y <= x) lives at index x*(x+1)/2 + y (lalib/Matrix.ipp:332-356).  The caller
 * owns every host array; no pointer is kept after a call returns.  Every call
 * returns DSS_OK (0) or a negative status and records a message readable with
 * dss_last_error(); nothing aborts the process.  One context per host thread.
 *
 * Function order matches scf::constructBasis (chem/scf/SCFBasis.cpp:120-139):
 * shells in the order given, m = -l..l inside a spherical shell (the reference's
 * real solid harmonics, chem/GTO.cpp:15-94); inside a Cartesian (6D) shell the
 * monomials x^a y^b z^c are ordered a descending then b descending, each scaled
 * to unit self-overlap.
 */
#ifndef DSS_H
#define DSS_H

#ifdef __cplusplus
extern "C" {
#endif

#define DSS_OK 0
#define DSS_ERR_INVALID (-1)     /* bad argument or call order */
#define DSS_ERR_OOM (-2)         /* device or host allocation failed */
#define DSS_ERR_CUDA (-3)        /* CUDA runtime / launch error */
#define DSS_ERR_NOCONV (-4)      /* SCF reached its iteration cap */
#define DSS_ERR_UNSUPPORTED (-6) /* e.g. angular momentum above the compiled maximum */

#define DSS_BOYS_REF 0  /* the reference's truncated series (parity mode) */
#define DSS_BOYS_FAST 1 /* accurate tabulated Boys function */

typedef struct dss_ctx dss_ctx;

typedef struct dss_opts {
  int device;                 /* CUDA device ordinal */
  double schwarz_threshold;   /* drop shell quartets with Q_ab Q_cd below this (0: keep all) */
  int boys_mode;              /* DSS_BOYS_REF or DSS_BOYS_FAST */
  double primitive_threshold; /* drop primitive pairs with |K_ab| (pi/p)^1.5 below this (0: keep all) */
} dss_opts;

/* Defaults: device 0, Schwarz threshold 1e-12, reference Boys, primitive-pair
 * threshold 1e-18 (each dropped pair changes any integral by < ~1e-15). */
void dss_default_opts(dss_opts* opts);

/* Creates a context on opts->device (opts may be NULL for the defaults).
 * Replaces the reference's global two-electron state (chem/scf/ExactCoulomb.cpp:13-15). */
int dss_create(dss_ctx** ctx, const dss_opts* opts);

void dss_destroy(dss_ctx* ctx);

/* Message of the last failed call on ctx ("" if none).  With ctx == NULL: the
 * last dss_create failure. */
const char* dss_last_error(const dss_ctx* ctx);

/* Basis of one molecule as shells.  l[s], nprim[s]; exps/coefs concatenated in
 * shell order; coefs are the basis file's contraction coefficients (the library
 * applies the reference's primitive normalisation, chem/GTO.cpp:90-93, and no
 * contraction renormalisation).  centers_bohr[3*s].  pure = 1: spherical (5D)
 * functions as in the reference; pure = 0: Cartesian (6D).
 * Computes Schwarz factors on the device and the screened quartet work lists.
 * Replaces the set-up half of assignExactRepulsionTensor (ExactCoulomb.cpp:41-52). */
int dss_set_basis(dss_ctx* ctx, int n_shell, const int* l, const int* nprim, const double* exps,
                  const double* coefs, const double* centers_bohr, int pure);

/* Number of basis functions of the current basis. */
int dss_nbf(const dss_ctx* ctx);

/* Coulomb and exchange matrices of one symmetric density D (packed-U, n(n+1)/2):
 *   J[m][n] = sum_st D[s][t] (mn|st)      (getExactCoulombMatrix, ExactCoulomb.cpp:103-112)
 *   K[m][n] = sum_st D[s][t] (mt|sn)      (getExactExchangeMatrix, ExactCoulomb.cpp:114-123)
 * The reference's RHF two-electron Fock part G = J[D_total] - K[D_alpha]
 * (SCFSolver.cpp:29-43) is J - K/2 of one call with D = D_total.
 * Either output may be NULL.  Host arrays; returns after the results are copied back. */
int dss_build_jk(dss_ctx* ctx, const double* D_packed, double* J_packed, double* K_packed);

/* Same build on device-resident dense row-major n x n matrices (device
 * pointers, symmetric D); enqueued on the context's stream, which the caller
 * synchronises with dss_sync().  For callers that keep densities in HBM. */
int dss_build_jk_device(dss_ctx* ctx, const double* D_dense_dev, double* J_dense_dev, double* K_dense_dev);

/* Mixed-precision, density-screened build (the incremental form's kernel):
 * quartets whose bound Q_ab Q_cd max|D| (over the six density blocks they
 * touch) is below skip_threshold are skipped; a warp of quartets whose bounds
 * are all below fp32_threshold runs the recurrences in FP32.  The Boys
 * function, the Schwarz factors and all accumulation stay FP64; the Boys
 * function is the accurate one.  Device-resident dense matrices as above. */
int dss_build_jk_mixed_device(dss_ctx* ctx, const double* D_dense_dev, double* J_dense_dev, double* K_dense_dev,
                              double fp32_threshold, double skip_threshold);

/* Largest basis dss_build_jk_device_noalloc accepts. */
#define DSS_NOALLOC_MAX_NBF 512

/* dss_build_jk_device without any device allocation during the call (no
 * counterpart in the reference, which has no GPU).  For callers that may not
 * allocate device memory while they run: code that must not let cudaMalloc /
 * cudaFree synchronise the device, processes whose device memory is owned by
 * a pool or budget, latency-bound loops.  The two n x n accumulators live in a
 * fixed 4 MiB array inside the library (held on every GPU that loads the
 * library until the process exits), so n may not exceed DSS_NOALLOC_MAX_NBF;
 * larger bases are rejected with DSS_ERR_INVALID.  dss_create looks up the
 * array's device address (with lazy module loading this is when the array
 * reaches the device), and dss_set_basis / dss_set_class_variant load the
 * kernels a build launches, so the call itself loads and allocates nothing,
 * its first call included.  The array is zeroed at the start of every call and
 * keeps the last call's accumulators afterwards; every call on a device shares
 * it, so calls whose GPU work overlaps (other streams or contexts on the same
 * device) race.  Inputs, outputs and the basis context are the caller's, as
 * for dss_build_jk_device; single-molecule contexts only. */
int dss_build_jk_device_noalloc(dss_ctx* ctx, const double* D_dense_dev, double* J_dense_dev, double* K_dense_dev);

/* Waits for the context's stream. */
int dss_sync(dss_ctx* ctx);

/* Work statistics of the current basis: unique shell quartets kept by the
 * Schwarz screen, primitive quartets they hold, and the warp tasks. */
int dss_work_stats(const dss_ctx* ctx, long long* shell_quartets, long long* prim_quartets, long long* warp_tasks);

/* Uses the caller's CUDA stream (a cudaStream_t passed as void*) for all
 * later work on ctx; NULL restores the context's own stream. */
int dss_set_stream(dss_ctx* ctx, void* stream);

/* The stream ctx currently enqueues on (a cudaStream_t as void*). */
void* dss_get_stream(const dss_ctx* ctx);

/* Shell-quartet classes (la lb|lc ld) the library was compiled with. */
int dss_num_classes(void);

/* Class i: its angular momenta and, for the current basis, the screened shell
 * and primitive quartets and warp tasks it holds. */
int dss_class_info(const dss_ctx* ctx, int i, int* l4, long long* shell_quartets, long long* prim_quartets,
                   long long* warp_tasks);

/* Kernel variant of class i: 0 one thread per shell quartet, 1 one warp per
 * shell quartet (shared-memory programs; only for the classes compiled with it),
 * 2 and 3 one thread per shell quartet with one and two fewer resident blocks
 * per SM and so more registers per thread (classes of total angular momentum
 * <= 4; the plain FP64 reference-Boys build, other forms run variant 0's
 * kernel), 4 one thread per shell quartet in persistent blocks that stage the
 * reference-mode Boys records of the class's orders in shared memory (classes
 * of total angular momentum <= 2; the plain FP64 reference-Boys build of an
 * unsplit launch, otherwise variant 0's kernel), 5, 6, 7 variants 0, 2, 3
 * launched as one wave (the blocks the SMs hold at once, the warps striding
 * over the work; 6 and 7 where 2 and 3 exist), 8 variant 0's kernel on one
 * block per SM of a third of the SMs (a class whose per-thread arrays spill to
 * local memory then keeps that memory within L2 while the other SMs run the
 * classes beside it), -1 the library default
 * (variant 0: in a build the classes run concurrently, and the warp-cooperative
 * kernels' large shared-memory blocks slow the classes beside them more than
 * they gain, measured on the (H2O)16 6-31G* build 8.51 -> 7.21 ms).  Used
 * by the autotuner; persists across bases. */
int dss_set_class_variant(dss_ctx* ctx, int i, int variant);

/* The variant class i currently runs with (-1 before a basis is set). */
int dss_get_class_variant(const dss_ctx* ctx, int i);

/* The list schedule of a plain build's class launches (host only): n launch
 * times ms[] and nstreams side streams; order[k] is the index of the k-th
 * launch (longest first, ties in index order) and stream[k] its side stream,
 * the one with the least work so far (lowest index on ties). */
int dss_list_schedule(const float* ms, int n, int nstreams, int* order, int* stream);

/* Kernel launches one dss_build_jk_device call enqueues. */
int dss_kernels_per_build(const dss_ctx* ctx);

/* One dss_build_jk_device with a CUDA event pair around every class launch;
 * ms_per_class[dss_num_classes()] receives each launch's device time (0 for
 * classes without work).  Synchronises the stream.  The context keeps the times
 * per class and kernel shape (until the next dss_set_basis): once every class
 * of a build has one for its current shape, plain builds launch the classes
 * longest first, each onto the side stream with the least work so far. */
int dss_profile_build(dss_ctx* ctx, const double* D_dense_dev, double* J_dense_dev, double* K_dense_dev,
                      float* ms_per_class);

/* Persistent grouped launches (on = 1; 0 restores one launch per class, the
 * default): the unsplit thread-per-quartet classes of total angular momentum
 * <= 2, and those of 3..4, each share one persistent kernel whose warps take
 * warp tasks of every class of the group from a device work queue (an atomic
 * head, zeroed before each launch); warp-cooperative, split and heavier
 * classes keep their own launches.  Plain FP64 reference-Boys builds and the
 * mixed-precision form; other builds run per class.  No counterpart in the
 * reference; chosen by the autotuner (dss_time_build). */
int dss_set_persistent(dss_ctx* ctx, int on);
int dss_get_persistent(const dss_ctx* ctx);

/* One dss_build_jk_device (every class, in the launch shape the context is set
 * to) timed with one CUDA event pair; *ms receives its device time.
 * Synchronises the stream. */
int dss_time_build(dss_ctx* ctx, const double* D_dense_dev, double* J_dense_dev, double* K_dense_dev, float* ms);

/* Device Boys function F_0..F_L (L <= 12) at n points x[] into F[n*(L+1)]:
 * mode DSS_BOYS_REF (the reference's truncated series, evaluated from the
 * accurate function and the tabulated truncation points), DSS_BOYS_FAST, or 2
 * (the reference's series summed term by term).  For tests and diagnostics. */
int dss_eval_boys(dss_ctx* ctx, int mode, int L, const double* x, int n, double* F);

/* Measures the device's double-precision FMA throughput with a register-only
 * loop (the FP64 CUDA-core roofline the ERI kernels are reported against). */
int dss_probe_fp64_peak(dss_ctx* ctx, double* tflops);

/* One-electron matrices of the current basis for the given nuclei (Z[natom],
 * xyz_bohr[3*natom]), packed-U: overlap S, kinetic T and nuclear attraction V
 * (H = T + V), and the nuclear repulsion energy.  Replaces
 * scf::assignOverlapMatrix / assignCoreHamiltonian (chem/scf/SCFBasis.cpp:56-83).
 * Any output may be NULL.  Computed on the device (one warp per shell pair). */
int dss_one_electron(dss_ctx* ctx, int natom, const int* Z, const double* xyz_bohr, double* S_packed,
                     double* T_packed, double* V_packed, double* e_nuc);

/* ---------------------------------------------------------------- SCF on the device */

typedef struct dss_scf_opts {
  double conv;   /* converged when |E_elec - E_prev| < conv (scf::energy_threshold) */
  int diis_size; /* Pulay DIIS ring length, 1..9 */
  int max_iter;  /* iteration cap (the reference loops until converged) */
  int use_guess; /* 0: core guess D = 0 (scf::useCoreGuess); 1: start from D_alpha_inout */
  /* Mixed-precision incremental form (incremental = 1): G(D_k) = G(D_k-1) +
   * G(D_k - D_k-1), each increment built by dss_build_jk_mixed_device with the
   * thresholds below; a full FP64 build every rebuild_every iterations and for
   * every iteration once |dE| < final_switch (so the last two iterations and the
   * energy are FP64).  incremental = 0 is the plain form: a full FP64 build with
   * the context's Boys mode every iteration. */
  int incremental;
  double fp32_threshold; /* default 1e-7 */
  double skip_threshold; /* default 1e-12 */
  int rebuild_every;     /* default 16 */
  double final_switch;   /* default 1e-8 Eh */
} dss_scf_opts;

/* Defaults: conv 1e-8 (chem/scf/SCFSolver.cpp:26), diis_size 8 (:214),
 * max_iter 128, core guess, plain form. */
void dss_default_scf_opts(dss_scf_opts* opts);

/* Closed-shell RHF on the device for the current basis, replacing
 * scf::useCoreGuess + scf::solveMOs + scf::getTotalEnergy
 * (chem/scf/SCFSolver.cpp:179-237, chem/scf/Energy.cpp:21-78).
 * H (core Hamiltonian) and S (overlap) packed-U; n_alpha occupied orbitals;
 * e_nuc the nuclear repulsion added to the final energy.  On return
 * *E_total holds the converged total energy, D_alpha_inout (if not NULL) the
 * final alpha density (packed-U), *iterations the SCF iterations.
 * Returns DSS_ERR_NOCONV when max_iter is reached (outputs still written). */
int dss_scf_solve(dss_ctx* ctx, const double* H_packed, const double* S_packed, int n_alpha, double e_nuc,
                  const dss_scf_opts* opts, double* E_total, double* D_alpha_inout, int* iterations);

/* Open-shell UHF on the device for the current basis (multiplicity > 1 in
 * scf::assignMolecule, chem/scf/SCFBasis.cpp:17-37), replacing the
 * unrestricted branch of scf::solveMOs + scf::calculateEnergies
 * (chem/scf/SCFSolver.cpp:120-172,196-237; chem/scf/Energy.cpp:21-50):
 * G_s = J[D_a + D_b] - K[D_s] from one unrestricted J/K build per iteration (each
 * integral evaluated once for J and both exchange matrices; two builds with the
 * accurate Boys mode), one Pulay DIIS
 * ring per spin (chem/scf/SCFDIIS.cpp:14-52), one eigensolve per spin,
 * E_elec = sum eps_a + sum eps_b - (tr(D_a G_a) + tr(D_b G_b))/2.  n_alpha and
 * n_beta occupied orbitals (electron_count[0], electron_count[1]).  Plain FP64
 * form only (opts->incremental must be 0).  D_alpha_inout / D_beta_inout: the
 * guess when opts->use_guess, and the final spin densities (packed-U). */
int dss_uhf_solve(dss_ctx* ctx, const double* H_packed, const double* S_packed, int n_alpha, int n_beta,
                  double e_nuc, const dss_scf_opts* opts, double* E_total, double* D_alpha_inout,
                  double* D_beta_inout, int* iterations);

/* MO coefficients (n x n row-major: AO row, MO column, ascending orbital
 * energy) and orbital energies of spin 0 (alpha; the RHF orbitals) or 1 (beta,
 * after dss_uhf_solve) from the last solve in this context: the reference's
 * scf::coefficient_matrix[spin] and scf::mo_levels[spin]
 * (chem/scf/SCFCommon.hpp:28-29).  Either output may be NULL. */
int dss_scf_orbitals(const dss_ctx* ctx, int spin, double* C, double* eps);

/* Molden file of the last solve, replacing scf::writeOrbitalsMolden
 * (chem/scf/WriteOrbitals.cpp:17-137): nuclei Z[natom] / xyz_bohr (the shells'
 * centres), the basis with its file coefficients, the orbitals (all of them when
 * write_virtual, else the occupied ones), alpha then beta.  5D bases only. */
int dss_write_molden(dss_ctx* ctx, const char* path, int natom, const int* Z, const double* xyz_bohr,
                     int write_virtual);

/* WFX file of the last solve, replacing scf::writeOrbitalsWFX
 * (chem/scf/WriteOrbitals.cpp:139-458): the same sections (nuclei, electron
 * counts, Cartesian primitives per atom in WFX type order, occupations,
 * energies, spin types, orbital coefficients on the primitives), all orbitals
 * when write_virtual, else the occupied ones, alpha then beta.  Beta
 * occupations count the beta electrons (the reference's loop counts alpha
 * electrons there, WriteOrbitals.cpp:350).  5D bases, l <= 2. */
int dss_write_wfx(dss_ctx* ctx, const char* path, int natom, const int* Z, const double* xyz_bohr,
                  int write_virtual);

/* Density checkpoint (restart file) of the last dss_scf_solve / dss_uhf_solve:
 * the spin densities (packed-U; D_alpha only for a restricted solve), the
 * electron counts and a checksum.  The reference has no restart file of its
 * own (chem/scf/WriteOrbitals.cpp writes viewer output only); the file feeds
 * the guess of a later solve (dss_scf_opts.use_guess). */
int dss_save_density(dss_ctx* ctx, const char* path);

/* Reads a density checkpoint for a basis of nbf functions into D_alpha and (if
 * not NULL) D_beta (a restricted file gives D_beta = D_alpha); *spins,
 * *n_alpha, *n_beta (each optional) receive the file's spin count and electron
 * counts.  Host only.  Rejects a file of another basis size, a truncated file
 * and a checksum mismatch (DSS_ERR_INVALID; the message goes to ctx, which may
 * be NULL). */
int dss_load_density(dss_ctx* ctx, const char* path, int nbf, int* spins, int* n_alpha, int* n_beta,
                     double* D_alpha, double* D_beta);

/* Nuclear gradient dE/dR (grad[3*natom], hartree/bohr) of the last
 * dss_scf_solve / dss_uhf_solve, the quantity of scf::getEnergyGradient
 * (chem/scf/Gradient.cpp:14-133, chem/scf/ExactCoulomb.cpp:125-195):
 * tr(D dH) + 1/2 sum Gamma d(ij|kl) - tr(W dS) + dV_nn, W the energy-weighted
 * density of the final orbitals.  step = 0: every term analytic on the device
 * (the four-centre term as dss_eri_gradient; shifted overlap, kinetic and
 * nuclear-attraction integrals with the Hellmann-Feynman term).  step > 0: the
 * one-electron terms instead by central differences of step bohr of the device
 * one-electron integrals at fixed D and W (a cross-check; O(step^2)). */
int dss_gradient(dss_ctx* ctx, int natom, const int* Z, const double* xyz_bohr, double step, double* grad);

/* Analytic four-centre term of the nuclear gradient, added into grad[3*natom]:
 * 1/2 sum_{ijkl} Gamma_ijkl d(ij|kl)/dR with Gamma_ijkl = D_ij D_kl -
 * sum_s D^s_ik D^s_jl, over the Schwarz-screened quartets of the current basis
 * (derivative integrals from the 2 zeta-weighted shifted classes, digested with
 * the two-particle density on the device).  Replaces addExactTwoElectronGradient
 * (chem/scf/ExactCoulomb.cpp:125-195).  D_packed: total density; Da_packed and
 * Db_packed: the spin densities for an unrestricted determinant, both NULL for a
 * closed shell (D^s = D/2).  shell_atom[s]: the nucleus (0..natom-1) of shell s.
 * Packed-U host arrays; single-molecule contexts. */
int dss_eri_gradient(dss_ctx* ctx, const double* D_packed, const double* Da_packed, const double* Db_packed,
                     int natom, const int* shell_atom, double* grad);

/* ---------------------------------------------------------------- batches of molecules */
/* Many closed-shell molecules of uneven size solved together: each ERI class
 * is one launch over every molecule of the batch, and one SCF iteration of all
 * molecules (the steps of dss_scf_solve, plain form) is a captured CUDA graph
 * whose per-molecule control (iteration count, DIIS ring, convergence) lives on
 * the device.  Molecules may be added and removed between steps (continuous
 * batching); each occupies a region of a device arena fixed at creation, and a
 * molecule that does not fit is not admitted (DSS_ERR_OOM).  The reference has
 * no batch mode; per molecule the iteration is the reference's solveMOs loop. */
typedef struct dss_batch dss_batch;

/* arena_bytes: device memory for molecule regions (0: a quarter of the free
 * memory); diis_size 1..9 (0: 8). */
int dss_batch_create(dss_batch** batch, const dss_opts* opts, size_t arena_bytes, int diis_size);
void dss_batch_destroy(dss_batch* batch);
const char* dss_batch_last_error(const dss_batch* batch);

/* Admits one molecule (shells as in dss_set_basis, nuclei Z/xyz_bohr, total
 * charge); D_guess (packed-U alpha density, may be NULL) warm-starts it, as the
 * reference's frequency driver does by not resetting the density
 * (chem/scf/Frequency.cpp:121-133).  *handle identifies it. */
int dss_batch_add(dss_batch* batch, int n_shell, const int* l, const int* nprim, const double* exps,
                  const double* coefs, const double* centers_bohr, int pure, int natom, const int* Z,
                  const double* xyz_bohr, int charge, const double* D_guess, int* handle);

/* Runs up to `iterations` SCF iterations of every unfinished molecule, then
 * computes the final energies of those that finished.  *n_active: molecules
 * still iterating.  opts->incremental = 1 runs the mixed-precision incremental
 * form per molecule exactly as dss_scf_solve does (full FP64 builds at the start,
 * every rebuild_every iterations and in the final phase; FP32 / skipped quartets
 * by the Schwarz x |dD| bound otherwise; accurate Boys function). */
int dss_batch_step(dss_batch* batch, const dss_scf_opts* opts, int iterations, int* n_active);

/* Steps until every molecule finished (converged or reached max_iter). */
int dss_batch_solve(dss_batch* batch, const dss_scf_opts* opts);

/* Result of a finished molecule: total energy, final alpha density (packed-U,
 * may be NULL), iterations, status (DSS_OK or DSS_ERR_NOCONV). */
int dss_batch_result(dss_batch* batch, int handle, double* E_total, double* D_packed, int* iterations,
                     int* status);

/* Handles of the molecules whose results the last dss_batch_step produced
 * (converged or stopped in it); *count is their number, at most cap are written.
 * One call replaces polling dss_batch_result per molecule. */
int dss_batch_finished(const dss_batch* batch, int* handles, int cap, int* count);

/* One J/K accumulation over every live molecule's current density with CUDA
 * events around each class launch (classes one after another on one stream):
 * ms[i] = milliseconds of class i in dss_class_info order, 0 for classes without
 * work.  Overwrites the molecules' J/K scratch only; for the batch autotuner. */
int dss_batch_profile(dss_batch* batch, float* ms);

/* One FP64 J/K accumulation over every live molecule in the batch's launch
 * shape (per class, or persistent groups), timed as a whole: *ms. */
int dss_batch_time_build(dss_batch* batch, float* ms);

/* dss_set_persistent for the batch's builds (the captured iteration is re-made). */
int dss_batch_set_persistent(dss_batch* batch, int on);

/* Releases a molecule's region. */
int dss_batch_remove(dss_batch* batch, int handle);

/* Live molecules, largest free arena block in bytes, and (in/out) the region
 * bytes a molecule of *region_bytes_of_n functions needs. */
int dss_batch_info(const dss_batch* batch, int* n_live, long long* free_bytes, long long* region_bytes_of_n);

/* Kernel variant of class i for the batch (see dss_set_class_variant). */
int dss_batch_set_class_variant(dss_batch* batch, int i, int variant);

/* The batch's Fock-build context (for dss_class_info / dss_get_class_variant). */
void* dss_batch_context(dss_batch* batch);

#ifdef __cplusplus
}
#endif
#endif /* DSS_H */
