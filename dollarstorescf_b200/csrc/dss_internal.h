// Internal state of a dss_ctx (the C ABI's opaque handle).
#pragma once
#include <cuda_runtime.h>

#include <array>
#include <string>
#include <vector>

#include "dss.h"

struct PrimPair;

// Device buffer that grows on demand and frees on destruction.
template <class T>
struct DevBuf {
  T* ptr = nullptr;
  size_t n = 0;
  DevBuf() = default;
  DevBuf(const DevBuf&) = delete;
  DevBuf& operator=(const DevBuf&) = delete;
  DevBuf(DevBuf&& o) noexcept : ptr(o.ptr), n(o.n) {
    o.ptr = nullptr;
    o.n = 0;
  }
  DevBuf& operator=(DevBuf&& o) noexcept {
    if (this != &o) {
      free();
      ptr = o.ptr;
      n = o.n;
      o.ptr = nullptr;
      o.n = 0;
    }
    return *this;
  }
  ~DevBuf() { free(); }
  cudaError_t resize(size_t count) {
    if (count <= n && ptr) return cudaSuccess;
    free();
    if (count == 0) return cudaSuccess;
    cudaError_t e = cudaMalloc((void**)&ptr, count * sizeof(T));
    if (e != cudaSuccess) {
      ptr = nullptr;
      n = 0;
      return e;
    }
    n = count;
    return cudaSuccess;
  }
  void free() {
    if (ptr) cudaFree(ptr);
    ptr = nullptr;
    n = 0;
  }
};

struct BasisHost {
  int pure = 1;
  int nbf = 0;
  std::vector<int> l, nprim, prim0, f0;
  std::vector<double> xyz, exps, wts;
  std::vector<double> coefs;  // the file's contraction coefficients (unnormalised)
  std::vector<int> mol;  // per shell: molecule of a batch (empty: one molecule); f0 is then molecule-local
};

// Device scratch of the one-electron kernels (grow-only, reused across calls).
struct OneEScratch {
  DevBuf<int2> pairs;
  DevBuf<int> ints;
  DevBuf<double> dbl;
};

struct ClassTasks {
  int la = 0, lb = 0, lc = 0, ld = 0;
  int ntasks = 0;
  int variant = 0;  // 0: thread per quartet, 1: warp-cooperative
  int split = 1;    // thread-per-quartet launches: slices of the bra primitive pairs
  long long shell_quartets = 0, prim_quartets = 0;
  DevBuf<int4> d_tasks;
};

struct ScfBuffers {
  DevBuf<double> pool;
  DevBuf<int> ibuf;
};

struct dss_ctx {
  dss_opts opts{};
  const double* boys_cell = nullptr;  // device address of the Boys cell records on opts.device
  double* noalloc_acc = nullptr;      // device address of the allocation-free build's accumulators
  cudaStream_t stream = nullptr;      // the stream work is enqueued on
  cudaStream_t own_stream = nullptr;  // created with the context
  // Side streams: the class launches of one build fork onto them so that the
  // long-running, low-occupancy high-angular-momentum classes overlap the rest.
  static constexpr int kSideStreams = 16;  // capacity; nside are used
  int nside = 8;
  cudaStream_t side[kSideStreams] = {};
  cudaEvent_t fork_ev = nullptr;
  cudaEvent_t join_ev[kSideStreams] = {};
  std::string err;

  // basis
  int nbf = 0, pure = 1, nshell = 0;
  BasisHost basis;
  DevBuf<PrimPair> d_pp;
  const PrimPair* ext_pp = nullptr;  // batch mode: the batch's device pool of primitive pairs (used instead of d_pp)
  DevBuf<int> d_pair_a, d_pair_b, d_pair_pp0, d_pair_npp, d_sh_f0;
  DevBuf<double> d_sh_xyz, d_Q, d_Qs;  // Schwarz factors: computation order, sorted pair order
  DevBuf<int> d_sh_nf;                  // functions per shell
  DevBuf<float> d_dmax;
  // Set-up scratch, grow-only so that admitting molecule after molecule does not
  // allocate and free device memory every time: Schwarz-factor inputs and outputs
  // (dss_pairs_make) and the one-electron kernels' inputs.
  DevBuf<PrimPair> sch_pp;
  DevBuf<int> sch_pa, sch_pb, sch_p0, sch_pn;
  DevBuf<double> sch_xyz, sch_Q;
  OneEScratch oe_scratch;
  std::vector<int> h_pair_a, h_pair_b, h_pair_npp, h_pair_cls;
  std::vector<double> h_Q;
  std::vector<int> class_pair0, class_pair1;
  std::vector<ClassTasks> tasks;
  // Milliseconds of each class launch timed alone by the last profile, per kernel shape.
  std::vector<std::array<float, 9>> class_ms;
  std::vector<int> class_variant;  // per class: -1 default, 0 thread, 1 warp-cooperative
  // Persistent grouped launches (dss_set_persistent) and their queue heads.
  bool persist = false;
  DevBuf<int> d_persist_head;
  std::vector<int> h_pair_mol;

  // Batch mode (nmol > 0, set by the batch engine): per-shell matrix offsets
  // into the batch arena and per-molecule sizes; see EriArgs.
  int nmol = 0;
  DevBuf<long long> d_sh_mbase, d_sh_jbase, d_sh_kbase, d_sh_dbase;
  DevBuf<int> d_sh_n, d_sh_mol, d_sh_loc, d_sh_nsm;
  const int* d_mol_active = nullptr;
  long long n_shell_quartets = 0, n_prim_quartets = 0, n_warp_tasks = 0;

  // build scratch
  DevBuf<double> packed_in, packed_j, packed_k, Ddense, Jacc, Kacc;
  ScfBuffers scf;
  // Orbitals of the last dss_scf_solve / dss_uhf_solve (host copies): per spin
  // C (n x n row-major, AO row, MO column) and the orbital energies.
  std::vector<double> last_C[2], last_eps[2];
  int last_nocc[2] = {0, 0};
  int last_spins = 0;  // 0: none, 1: RHF, 2: UHF

  void release_basis() {
    d_pp.free();
    d_pair_a.free();
    d_pair_b.free();
    d_pair_pp0.free();
    d_pair_npp.free();
    d_sh_f0.free();
    d_sh_xyz.free();
    d_Q.free();
    d_Qs.free();
    d_sh_nf.free();
    d_dmax.free();
    d_sh_mbase.free();
    d_sh_jbase.free();
    d_sh_kbase.free();
    d_sh_dbase.free();
    d_sh_n.free();
    d_sh_mol.free();
    d_sh_loc.free();
    d_sh_nsm.free();
    tasks.clear();
    nbf = 0;
  }
  void release() {
    release_basis();
    packed_in.free();
    packed_j.free();
    packed_k.free();
    Ddense.free();
    Jacc.free();
    Kacc.free();
    scf.pool.free();
    scf.ibuf.free();
  }
};

int dss_fail(dss_ctx* ctx, int code, const std::string& msg);
// Device address of the allocation-free build's accumulator array on the current
// device; loads the array and its kernels (dss_create calls it, so that
// dss_build_jk_device_noalloc itself loads and allocates nothing).
cudaError_t dss_noalloc_attach(double** acc);
// Loads the kernels a plain build of the context's basis launches (see
// dss_preload_eri_variant).
void dss_preload_build(dss_ctx* ctx);
// Device address of the reference-mode Boys cell records on the current device
// (defined once in the generated boys_cell_data.cu).
cudaError_t dss_boys_cell_table(const double** out);
int dss_cuda_check(dss_ctx* ctx, cudaError_t e, const char* what);
// Shell pairs of a basis with their primitive pairs and Schwarz factors, sorted
// by (pair class, molecule, primitive-pair count descending, Q descending).
// Work lists of a pair set on the host, per quartet class (DSS_FOR_EACH_CLASS
// order): warp tasks {bra pair, first ket pair, ket count, molecule} and the
// shell / primitive quartets they cover.
struct HostTasks {
  std::vector<std::vector<int4>> tasks;
  std::vector<long long> shell_quartets, prim_quartets;
};

struct PairSet {
  std::vector<int> pa, pb, p0, pn, cls, mol;  // shells, first primitive pair, primitive pairs, class, molecule
  std::vector<double> Q;
  std::vector<double> pp;  // primitive pairs, 10 doubles each (the PrimPair record)
  // Batch molecules: the molecule's own work lists (pair indices local to this
  // set, molecule 0), made once at admission and offset into a batch's lists.
  HostTasks tasks;
  bool have_tasks = false;
};
// Pairs of one basis (Schwarz factors computed on the device, synchronously).
int dss_pairs_make(dss_ctx* ctx, const BasisHost& B, PairSet* out, bool with_tasks = false);
// Concatenation of per-molecule pair sets in batch order: part m's shells start
// at shell_offset[m] and its pairs become molecule m's.
// pp_offset (optional): each part's primitive pairs already sit on the device
// at that record offset of one pool; the merged set then carries no pp records
// and its p0 index that pool.
void dss_pairs_merge(const std::vector<const PairSet*>& parts, const std::vector<int>& shell_offset, PairSet* out,
                     const std::vector<long long>* pp_offset = nullptr);
// Exponent of the first shell's primitive of every primitive pair of the
// context's basis (one molecule), in the order of its device primitive pairs.
void dss_pair_alphas(const dss_ctx* ctx, std::vector<double>* alpha);
// Makes B and P the context's basis: uploads, class ranges, work lists.
// no_tasks: install only the pairs (the caller installs the work lists).
int dss_pairs_install(dss_ctx* ctx, BasisHost&& B, PairSet&& P, const HostTasks* tasks = nullptr,
                      bool no_tasks = false);
int dss_setup_pairs(dss_ctx* ctx, BasisHost&& B);
// Shells from the C-ABI arrays: validation and the reference's primitive normalisation.
int dss_make_basis(int n_shell, const int* l, const int* nprim, const double* exps, const double* coefs,
                   const double* centers, int pure, BasisHost* out, std::string* err);
// One-electron S, T, V (packed-U, device buffers) of one molecule's basis,
// computed on the device on stream s (synchronous).  V == NULL: T receives
// T + V, the core Hamiltonian.
// One-electron part of the nuclear gradient, analytic (synchronous): grad_host
// [3 natom] = sum D dH/dR - sum W dS/dR for dense n x n device densities D, W
// (Hellmann-Feynman term included; the nuclear repulsion is not).
int dss_one_electron_gradient(cudaStream_t s, const BasisHost& B, int natom, const int* Z, const double* xyz_bohr,
                              const int* shell_atom, const double* D_dev, const double* W_dev, double* grad_host,
                              std::string* errp, OneEScratch* scratch = nullptr);
int dss_one_electron_device(cudaStream_t s, const BasisHost& B, int natom, const int* Z, const double* xyz,
                            double* S, double* T, double* V, std::string* err, OneEScratch* scratch = nullptr);
// The same into host packed-U arrays (any may be NULL), plus the nuclear repulsion.
int dss_one_electron_basis(cudaStream_t s, const BasisHost& B, int natom, const int* Z, const double* xyz,
                           double* S, double* T, double* V, double* e_nuc, std::string* err,
                           OneEScratch* scratch = nullptr);
// sum_{A<B} Z_A Z_B / R_AB.
double dss_nuclear_repulsion(int natom, const int* Z, const double* xyz);
int dss_build_tasks(dss_ctx* ctx);
// Work lists for pairs sorted by (class, molecule, npp, Q): class ranges
// [c0[c], c1[c]), Schwarz factors, primitive-pair counts and molecules.
void dss_make_tasks(const std::vector<int>& c0, const std::vector<int>& c1, const std::vector<double>& Q,
                    const std::vector<int>& npp, const std::vector<int>& pmol, int nmol, double thr, HostTasks* out);
// Uploads work lists as the context's (device buffers reused, grow-only).
int dss_install_tasks(dss_ctx* ctx, const HostTasks& ht);
// Work lists of the given per-class counts and statistics whose device buffers
// (ctx->tasks[i].d_tasks, grow-only) the caller fills on the context's stream.
int dss_install_task_counts(dss_ctx* ctx, const std::vector<int>& counts, const std::vector<long long>& sq,
                            const std::vector<long long>& pq);
// Number of shell-pair classes; bra and ket pair classes of quartet class i
// (DSS_FOR_EACH_CLASS order).
int dss_num_pair_classes();
int dss_quartet_bra_class(int i);
int dss_quartet_ket_class(int i);
// Per-class pair ranges of a pair set.
void dss_class_ranges(const std::vector<int>& cls, std::vector<int>* c0, std::vector<int>* c1);
// G = (Jacc + Jacc^T) - (Kacc + Kacc^T) / 2, dense n x n.
void dss_symmetrize_combine(cudaStream_t s, int n, const double* Jacc, const double* Kacc, double* G);
// How one J/K accumulation runs: Boys mode and, for the mixed-precision form,
// the density-weighted screen (dmax: per shell block max |D|, device).
struct BuildMode {
  int boys = 0;
  int mixed = 0;
  const float* dmax = nullptr;
  double skip_thr = 0.0, fp32_thr = 0.0;
  bool no_zero = false;  // the caller has zeroed the accumulators (batch mode)
  // Unrestricted build (one molecule): J from D = D_a + D_b, K from Da into
  // Kacc and from Db into K2 (zeroed here unless no_zero).
  bool uhf = false;
  const double* Da = nullptr;
  const double* Db = nullptr;
  double* K2 = nullptr;
};

// Enqueues one J/K accumulation; with events != NULL records events[2i], events[2i+1]
// around the launch of class i.  mode == NULL: the context's Boys mode, FP64.
int dss_enqueue_jk(dss_ctx* ctx, const double* D, double* Jacc, double* Kacc, cudaEvent_t* events = nullptr,
                   const BuildMode* mode = nullptr);
// Analytic two-electron gradient of the context's basis (one molecule) into
// grad_host[3 natom] (overwritten): densities dense n x n on the device, D the
// total, X (and Y) the exchange densities with factor xfac (RHF: X = D, Y = NULL,
// 1/4; UHF: D_alpha, D_beta, 1/2); shell_atom[s] the nucleus of shell s (host).
int dss_eri_gradient_dense(dss_ctx* ctx, const double* D_dev, const double* X_dev, const double* Y_dev, double xfac,
                           int natom, const int* shell_atom, double* grad_host);
// Keeps class i's launch time alone (ms) for its current kernel shape; the
// class launches of later builds are ordered by these times (dss_enqueue_jk).
void dss_record_class_ms(dss_ctx* ctx, int i, float ms);
// Per shell-pair block maximum of |D| (dense n x n, device) into dmax [nshell^2].
void dss_block_max(dss_ctx* ctx, const double* D, float* dmax);
