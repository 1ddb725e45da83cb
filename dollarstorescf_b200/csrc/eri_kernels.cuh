// ERI + J/K digest kernels and the Schwarz diagonal kernel, templated on the
// shell-quartet class.  The per-class integral code comes from eri_gen.cuh.
//
// Work decomposition: a warp owns one bra shell pair (ab) and up to 32 ket shell
// pairs (cd), one per lane (a "warp task").  Ket pairs of a task are consecutive
// in the class's pair list, which is sorted by primitive-pair count and then by
// Schwarz bound, so all lanes of a warp run the same primitive loop trip counts.
//
// Digest (the J/K of chem/scf/ExactCoulomb.cpp:103-123 over the 8-fold unique
// quartets of :54-68): for a unique shell quartet every function quartet
// (ij|kl) is scaled by s = 1/2 per coincidence (a == b, c == d, ab == cd) and
// contributes
//   Jacc[i][j] += 2 s (ij|kl) D[k][l],   Jacc[k][l] += 2 s (ij|kl) D[i][j],
//   Kacc[i][l] += s (ij|kl) D[j][k],     Kacc[j][l] += s (ij|kl) D[i][k],
//   Kacc[i][k] += s (ij|kl) D[j][l],     Kacc[j][k] += s (ij|kl) D[i][l],
// and finally J = Jacc + Jacc^T, K = Kacc + Kacc^T, so that
//   J[m][n] = sum_st D[s][t] (mn|st),   K[m][n] = sum_st D[s][t] (mt|sn).
// Each thread first sums its quartet's contributions per target element; the
// Jacc[i][j] sums, shared by the whole warp (same bra pair), are reduced with
// warp shuffles before a single atomic per element.
#pragma once
#include <atomic>

#include "common.cuh"
#include "eri_gen.cuh"

struct EriArgs {
  const int4* tasks;      // {bra pair, first ket pair, ket count, molecule}
  int ntasks;
  int split;              // thread-per-quartet kernel: blockIdx.y of split slices
                          // evaluates its share of the bra primitive pairs
  const int* pair_a;      // shell index of a (pair order: l_a >= l_b)
  const int* pair_b;
  const int* pair_pp0;    // first primitive pair
  const int* pair_npp;    // primitive pairs in the pair
  const PrimPair* pp;
  const double* sh_xyz;   // [nshell][3] bohr
  const int* sh_f0;       // first basis function of each shell
  const double* D;        // dense n x n density (row-major, symmetric)
  double* J;              // dense n x n accumulators (Jacc, Kacc above)
  double* K;
  int n;
  // Density-weighted screening (mixed-precision form only): a quartet is
  // skipped when Q_ab Q_cd max|D| over its six density blocks is below skip_thr,
  // and a warp runs its quartets in FP32 when every bound is below fp32_thr.
  const double* Qp;   // Schwarz factor per pair
  const float* dmax;  // [nshell * nshell] max |D| per shell block
  int ns;
  double skip_thr, fp32_thr;
  // Batches of molecules (NULL for one molecule): every shell carries the
  // offsets of its molecule's n x n matrices from D, J and K, the molecule's n,
  // its molecule index, its index among the molecule's shells, and the offset
  // and shell count of the molecule's dmax block.  Quartets of molecules whose
  // mol_active flag is 0 are skipped.
  const long long* sh_mbase;
  const long long* sh_jbase;
  const long long* sh_kbase;
  const int* sh_n;
  const int* sh_mol;
  const int* sh_loc;
  const long long* sh_dbase;
  const int* sh_nsm;
  const int* mol_active;
  const double* boys_cell;  // reference-mode Boys records (dss_boys_cell_table)
  // Unrestricted builds (the UHF kernel variant, one molecule): J from D (the
  // total density D_a + D_b), K from Da into K and from Db into K2.
  const double* Da;
  const double* Db;
  double* K2;
};

struct SchwarzArgs {
  int pair0, npair;       // pair range of one pair class
  const int* pair_a;
  const int* pair_b;
  const int* pair_pp0;
  const int* pair_npp;
  const PrimPair* pp;
  const double* sh_xyz;
  double* Q;              // out: sqrt(max |(ij|ij)|) per pair
  const double* boys_cell;  // reference-mode Boys records (dss_boys_cell_table)
};

__host__ __device__ constexpr int dss_ncart(int l) { return (l + 1) * (l + 2) / 2; }
__host__ __device__ constexpr int dss_nfunc(int l, bool pure) { return pure ? 2 * l + 1 : dss_ncart(l); }

template <int LA, int LB, int LC, int LD>
struct EriClass;

#define DSS_DEFINE_ERI_CLASS(la, lb, lc, ld, bc, kc)                                                    \
  template <>                                                                                           \
  struct EriClass<la, lb, lc, ld> {                                                                     \
    template <int BOYS, bool PURE, typename R>                                                          \
    __device__ __forceinline__ static void evalr(const PrimPair* bra, int nb, const PrimPair* ket, int nk, \
                                                 double ABx, double ABy, double ABz, double CDx,        \
                                                 double CDy, double CDz, R* I, const double* cells) {   \
      eri_##la##lb##lc##ld<BOYS, PURE, R>(bra, nb, ket, nk, ABx, ABy, ABz, CDx, CDy, CDz, I, cells);   \
    }                                                                                                   \
    template <int BOYS, bool PURE>                                                                      \
    __device__ __forceinline__ static void eval(const PrimPair* bra, int nb, const PrimPair* ket, int nk, \
                                                double ABx, double ABy, double ABz, double CDx,         \
                                                double CDy, double CDz, double* I, const double* cells) { \
      eri_##la##lb##lc##ld<BOYS, PURE, double>(bra, nb, ket, nk, ABx, ABy, ABz, CDx, CDy, CDz, I, cells); \
    }                                                                                                   \
  };
DSS_FOR_EACH_CLASS(DSS_DEFINE_ERI_CLASS)
#undef DSS_DEFINE_ERI_CLASS

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Density bound of a quartet for the mixed-precision screen.
__device__ __forceinline__ double quartet_dbound(const EriArgs& a, int sa, int sb, int sc, int sd) {
  const float* dm = a.dmax;
  int ns = a.ns;
  if (a.sh_mbase) {
    dm += a.sh_dbase[sa];
    ns = a.sh_nsm[sa];
    sa = a.sh_loc[sa];
    sb = a.sh_loc[sb];
    sc = a.sh_loc[sc];
    sd = a.sh_loc[sd];
  }
  float m = dm[sc * ns + sd];
  m = fmaxf(m, dm[sa * ns + sb]);
  m = fmaxf(m, dm[sa * ns + sd]);
  m = fmaxf(m, dm[sb * ns + sd]);
  m = fmaxf(m, dm[sa * ns + sc]);
  m = fmaxf(m, dm[sb * ns + sc]);
  return (double)m;
}

// Resident blocks the compiler must allow (caps registers): the light classes
// are latency bound and want more warps; the heavy ones keep their registers.
__host__ __device__ constexpr int dss_min_blocks(int L) { return L == 0 ? 8 : (L <= 2 ? 6 : (L <= 4 ? 4 : 1)); }

// Register tiers of the plain-form thread-per-quartet kernel (the autotuner's
// shape choice, class variants 0, 2, 3): tier 0 is dss_min_blocks; tiers 1 and 2
// allow fewer resident 128-thread blocks and so more registers per thread
// (64/80/128 -> 80/96/168 -> 128/128/255 for L = 0 / 1..2 / 3..4), trading
// occupancy for fewer spills.  Classes with L >= 5 have one tier.
__host__ __device__ constexpr int dss_min_blocks_tier(int L, int tier) {
  return tier == 0 ? dss_min_blocks(L)
                   : (tier == 1 ? (L == 0 ? 6 : (L <= 2 ? 5 : (L <= 4 ? 3 : 1)))
                                : (L == 0 ? 4 : (L <= 2 ? 4 : (L <= 4 ? 2 : 1))));
}
__host__ __device__ constexpr bool dss_has_tiers(int L) { return L <= 4; }

// The four exchange target blocks of one quartet (Kacc[i][l] += s (ij|kl) D[j][k]
// and the three others), one block at a time, from density D into Km.
template <int NA, int NB, int NC, int ND>
__device__ __forceinline__ void digest_k(const double* I, double s, const double* __restrict__ D, double* Km, int n,
                                         int fa, int fb, int fc, int fd) {
  // Kacc[i][l] += s (ij|kl) D[j][k]
  {
    double d[NB * NC];
#pragma unroll
    for (int j = 0; j < NB; ++j)
#pragma unroll
      for (int k = 0; k < NC; ++k) d[j * NC + k] = __ldg(D + (size_t)(fb + j) * n + fc + k);
#pragma unroll
    for (int i = 0; i < NA; ++i)
#pragma unroll
      for (int l = 0; l < ND; ++l) {
        double v = 0.0;
#pragma unroll
        for (int j = 0; j < NB; ++j)
#pragma unroll
          for (int k = 0; k < NC; ++k) v += I[((i * NB + j) * NC + k) * ND + l] * d[j * NC + k];
        atomicAdd(Km + (size_t)(fa + i) * n + fd + l, s * v);
      }
  }
  // Kacc[j][l] += s (ij|kl) D[i][k]
  {
    double d[NA * NC];
#pragma unroll
    for (int i = 0; i < NA; ++i)
#pragma unroll
      for (int k = 0; k < NC; ++k) d[i * NC + k] = __ldg(D + (size_t)(fa + i) * n + fc + k);
#pragma unroll
    for (int j = 0; j < NB; ++j)
#pragma unroll
      for (int l = 0; l < ND; ++l) {
        double v = 0.0;
#pragma unroll
        for (int i = 0; i < NA; ++i)
#pragma unroll
          for (int k = 0; k < NC; ++k) v += I[((i * NB + j) * NC + k) * ND + l] * d[i * NC + k];
        atomicAdd(Km + (size_t)(fb + j) * n + fd + l, s * v);
      }
  }
  // Kacc[i][k] += s (ij|kl) D[j][l]
  {
    double d[NB * ND];
#pragma unroll
    for (int j = 0; j < NB; ++j)
#pragma unroll
      for (int l = 0; l < ND; ++l) d[j * ND + l] = __ldg(D + (size_t)(fb + j) * n + fd + l);
#pragma unroll
    for (int i = 0; i < NA; ++i)
#pragma unroll
      for (int k = 0; k < NC; ++k) {
        double v = 0.0;
#pragma unroll
        for (int j = 0; j < NB; ++j)
#pragma unroll
          for (int l = 0; l < ND; ++l) v += I[((i * NB + j) * NC + k) * ND + l] * d[j * ND + l];
        atomicAdd(Km + (size_t)(fa + i) * n + fc + k, s * v);
      }
  }
  // Kacc[j][k] += s (ij|kl) D[i][l]
  {
    double d[NA * ND];
#pragma unroll
    for (int i = 0; i < NA; ++i)
#pragma unroll
      for (int l = 0; l < ND; ++l) d[i * ND + l] = __ldg(D + (size_t)(fa + i) * n + fd + l);
#pragma unroll
    for (int j = 0; j < NB; ++j)
#pragma unroll
      for (int k = 0; k < NC; ++k) {
        double v = 0.0;
#pragma unroll
        for (int i = 0; i < NA; ++i)
#pragma unroll
          for (int l = 0; l < ND; ++l) v += I[((i * NB + j) * NC + k) * ND + l] * d[i * ND + l];
        atomicAdd(Km + (size_t)(fb + j) * n + fc + k, s * v);
      }
  }
}

// One warp task (warp = task index): the bra pair against up to 32 ket pairs,
// one per lane, evaluated and digested.  slice: the bra-primitive slice of a
// split launch (a.split > 1), else 0.
// UHF = true: the unrestricted variant (one molecule): J from a.D = D_a + D_b,
// K from a.Da into a.K and from a.Db into a.K2, from one evaluation of the integrals.
template <int LA, int LB, int LC, int LD, int BOYS, bool PURE, bool MIXED, bool UHF>
__device__ __forceinline__ void eri_jk_task(const EriArgs& a, const int4* __restrict__ tasks, int warp, int lane,
                                            int slice) {
  constexpr int NA = dss_nfunc(LA, PURE), NB = dss_nfunc(LB, PURE);
  constexpr int NC = dss_nfunc(LC, PURE), ND = dss_nfunc(LD, PURE);
  const int4 t = __ldg(tasks + warp);
  bool active = lane < t.z;
  const int bra = t.x;
  const int ket = t.y + (active ? lane : 0);
  // Bra primitive pairs of this slice: all of them, or with split > 1 the
  // blockIdx.y-th of split equal parts.  The digest is linear in the integrals,
  // so every slice digests its partial sum and J/K add up to the full quartet.
  int bpp0 = __ldg(a.pair_pp0 + bra), bnpp = __ldg(a.pair_npp + bra);
  if (a.split > 1) {
    const int lo = bnpp * slice / a.split, hi = bnpp * (slice + 1) / a.split;
    if (lo == hi) return;  // uniform per warp
    bpp0 += lo;
    bnpp = hi - lo;
  }
  const int sa = __ldg(a.pair_a + bra), sb = __ldg(a.pair_b + bra);
  const int sc = __ldg(a.pair_a + ket), sd = __ldg(a.pair_b + ket);
  const double* __restrict__ Dm = a.D;
  double* Jm = a.J;
  double* Km = a.K;
  int n = a.n;
  if (a.sh_mbase) {  // uniform per warp: the bra pair fixes the molecule
    if (a.mol_active && !__ldg(a.mol_active + __ldg(a.sh_mol + sa))) return;
    n = __ldg(a.sh_n + sa);
    Dm += __ldg(a.sh_mbase + sa);
    Jm += __ldg(a.sh_jbase + sa);
    Km += __ldg(a.sh_kbase + sa);
  }
  bool fp32 = false;
  if constexpr (MIXED) {
    const double bound = __ldg(a.Qp + bra) * __ldg(a.Qp + ket) * quartet_dbound(a, sa, sb, sc, sd);
    active = active && bound >= a.skip_thr;
    fp32 = __all_sync(0xffffffffu, !active || bound < a.fp32_thr);
  }
  const double Ax = __ldg(a.sh_xyz + 3 * sa), Ay = __ldg(a.sh_xyz + 3 * sa + 1), Az = __ldg(a.sh_xyz + 3 * sa + 2);
  const double Bx = __ldg(a.sh_xyz + 3 * sb), By = __ldg(a.sh_xyz + 3 * sb + 1), Bz = __ldg(a.sh_xyz + 3 * sb + 2);
  const double Cx = __ldg(a.sh_xyz + 3 * sc), Cy = __ldg(a.sh_xyz + 3 * sc + 1), Cz = __ldg(a.sh_xyz + 3 * sc + 2);
  const double Dx = __ldg(a.sh_xyz + 3 * sd), Dy = __ldg(a.sh_xyz + 3 * sd + 1), Dz = __ldg(a.sh_xyz + 3 * sd + 2);

  double I[NA * NB * NC * ND];
  bool done = false;
  if constexpr (MIXED) {
    if (active && fp32) {
      float If[NA * NB * NC * ND];
      EriClass<LA, LB, LC, LD>::template evalr<BOYS, PURE, float>(
          a.pp + bpp0, bnpp, a.pp + __ldg(a.pair_pp0 + ket),
          __ldg(a.pair_npp + ket), Ax - Bx, Ay - By, Az - Bz, Cx - Dx, Cy - Dy, Cz - Dz, If, a.boys_cell);
#pragma unroll
      for (int q = 0; q < NA * NB * NC * ND; ++q) I[q] = (double)If[q];
      done = true;
    }
  }
  if (done) {
  } else if (active) {
    EriClass<LA, LB, LC, LD>::template eval<BOYS, PURE>(
        a.pp + bpp0, bnpp, a.pp + __ldg(a.pair_pp0 + ket),
        __ldg(a.pair_npp + ket), Ax - Bx, Ay - By, Az - Bz, Cx - Dx, Cy - Dy, Cz - Dz, I, a.boys_cell);
  } else {
#pragma unroll
    for (int q = 0; q < NA * NB * NC * ND; ++q) I[q] = 0.0;
  }
  double s = 1.0;
  if (sa == sb) s *= 0.5;
  if (sc == sd) s *= 0.5;
  if (bra == ket) s *= 0.5;
  const int fa = __ldg(a.sh_f0 + sa), fb = __ldg(a.sh_f0 + sb);
  const int fc = __ldg(a.sh_f0 + sc), fd = __ldg(a.sh_f0 + sd);
  const double* __restrict__ D = Dm;
  const double s2 = 2.0 * s;

  // One target block at a time: its density block in, its sums out, so only
  // I, one density block and one accumulator block are live together.
  // Bra-pair J block (Jacc[i][j] += 2 s (ij|kl) D[k][l]): the whole warp shares
  // the target, so the lanes' sums are reduced before one atomic.
  {
    double d[NC * ND];
#pragma unroll
    for (int k = 0; k < NC; ++k)
#pragma unroll
      for (int l = 0; l < ND; ++l) d[k * ND + l] = __ldg(D + (size_t)(fc + k) * n + fd + l);
#pragma unroll
    for (int i = 0; i < NA; ++i)
#pragma unroll
      for (int j = 0; j < NB; ++j) {
        double v = 0.0;
#pragma unroll
        for (int q = 0; q < NC * ND; ++q) v += I[(i * NB + j) * NC * ND + q] * d[q];
        v = warp_sum(s2 * v);
        if (lane == 0) atomicAdd(Jm + (size_t)(fa + i) * n + fb + j, v);
      }
  }
  if (!active) return;
  // Jacc[k][l] += 2 s (ij|kl) D[i][j]
  {
    double d[NA * NB];
#pragma unroll
    for (int i = 0; i < NA; ++i)
#pragma unroll
      for (int j = 0; j < NB; ++j) d[i * NB + j] = __ldg(D + (size_t)(fa + i) * n + fb + j);
#pragma unroll
    for (int k = 0; k < NC; ++k)
#pragma unroll
      for (int l = 0; l < ND; ++l) {
        double v = 0.0;
#pragma unroll
        for (int q = 0; q < NA * NB; ++q) v += I[q * NC * ND + k * ND + l] * d[q];
        atomicAdd(Jm + (size_t)(fc + k) * n + fd + l, s2 * v);
      }
  }
  if constexpr (UHF) {
    digest_k<NA, NB, NC, ND>(I, s, a.Da, Km, n, fa, fb, fc, fd);
    digest_k<NA, NB, NC, ND>(I, s, a.Db, a.K2, n, fa, fb, fc, fd);
  } else {
    digest_k<NA, NB, NC, ND>(I, s, D, Km, n, fa, fb, fc, fd);
  }
}

// Thread per shell quartet, warp per task.  TIER: register tier (dss_min_blocks_tier).
// The warps stride over the tasks, so a launch may use fewer blocks than tasks
// (the one-wave grids of class variants 5-7).
template <int LA, int LB, int LC, int LD, int BOYS, bool PURE, bool MIXED = false, bool UHF = false, int TIER = 0>
__global__ void __launch_bounds__(128, dss_min_blocks_tier(LA + LB + LC + LD, TIER)) eri_jk_kernel(EriArgs a) {
  const int nwarps = (int)((gridDim.x * blockDim.x) >> 5);
  for (int warp = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5); warp < a.ntasks; warp += nwarps)
    eri_jk_task<LA, LB, LC, LD, BOYS, PURE, MIXED, UHF>(a, a.tasks, warp, threadIdx.x & 31, (int)blockIdx.y);
}

// Multiprocessors of the current device (read once per device).
inline int dss_sm_count() {
  static std::atomic<int> cache[64] = {};
  int dev = 0;
  cudaGetDevice(&dev);
  int n = (dev >= 0 && dev < 64) ? cache[dev].load() : 0;
  if (!n) {
    cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
    if (n < 1) n = 1;
    if (dev >= 0 && dev < 64) cache[dev].store(n);
  }
  return n;
}

// The shared-memory Boys shape (class variant 4; plain form, reference Boys,
// total angular momentum L <= 2, unsplit launches): persistent blocks of
// DSS_SMEM_WARPS warps first copy the block-A cell records of orders 0..L
// (35 KB per order) into shared memory with coalesced 16-byte loads, then walk
// the warp tasks with a grid stride; each lane's Boys lookups read the staged
// records instead of gathering them through L1/L2.  Resident blocks per SM are
// set by the staged bytes: 4 / 3 / 2 for L = 0 / 1 / 2.
#define DSS_SMEM_WARPS 8
__host__ __device__ constexpr int dss_smem_min_blocks(int L) { return L == 0 ? 4 : (L == 1 ? 3 : 2); }
__host__ __device__ constexpr bool dss_has_smem_variant(int L) { return L <= 2; }

template <int LA, int LB, int LC, int LD, bool PURE>
__global__ void __launch_bounds__(32 * DSS_SMEM_WARPS, dss_smem_min_blocks(LA + LB + LC + LD))
    eri_jk_smem_kernel(EriArgs a) {
  dss_boys_smem_stage<LA + LB + LC + LD>(a.boys_cell);
  const int lane = threadIdx.x & 31;
  for (int w = (int)blockIdx.x * DSS_SMEM_WARPS + (int)(threadIdx.x >> 5); w < a.ntasks;
       w += (int)gridDim.x * DSS_SMEM_WARPS)
    eri_jk_task<LA, LB, LC, LD, DSS_BOYS_REF_SMEM, PURE, false, false>(a, a.tasks, w, lane, 0);
}

// Persistent grouped launch: one kernel runs the warp tasks of several classes
// (a group of classes with one register budget) from a device work queue.
// Items are the classes' warp tasks concatenated in launch order (highest
// total angular momentum first); each warp takes DSS_PERSIST_CHUNK consecutive
// items per atomicAdd on the queue head and runs each through its class's task
// body, so the classes of a group share the SMs and no class waits for another
// class's launch to drain.
#define DSS_PERSIST_MAX 10
#define DSS_PERSIST_CHUNK 4
struct PersistArgs {
  EriArgs a;                       // common arguments (a.tasks / a.ntasks unused)
  const int4* tasks[DSS_PERSIST_MAX];
  int start[DSS_PERSIST_MAX + 1];  // class k owns items [start[k], start[k + 1])
  int slot[DSS_PERSIST_MAX];       // class k's position in the group's class list
  int ncls;
  int* head;                       // queue head, zeroed before the launch
};

// Host launcher of the shared-memory Boys shape: sets the kernel's dynamic
// shared-memory limit and reads its resident blocks per SM once per device, and
// launches at most that many blocks per SM.
template <int LA, int LB, int LC, int LD, bool PURE>
inline void dss_launch_eri_smem(const EriArgs& a, cudaStream_t s) {
  constexpr int L = LA + LB + LC + LD;
  const size_t smem = dss_boys_smem_bytes<L>();
  static std::atomic<int> grid_dev[64] = {};  // resident blocks x SMs, per device (0: not yet read)
  int dev = 0;
  cudaGetDevice(&dev);
  int g = (dev >= 0 && dev < 64) ? grid_dev[dev].load() : 0;
  if (!g) {
    cudaFuncSetAttribute(eri_jk_smem_kernel<LA, LB, LC, LD, PURE>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)smem);
    int per = 0, nsm = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, eri_jk_smem_kernel<LA, LB, LC, LD, PURE>,
                                                  32 * DSS_SMEM_WARPS, smem);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    g = (per > 0 ? per : 1) * (nsm > 0 ? nsm : 1);
    if (dev >= 0 && dev < 64) grid_dev[dev].store(g);
  }
  const long long need = ((long long)a.ntasks + DSS_SMEM_WARPS - 1) / DSS_SMEM_WARPS;
  const unsigned blocks = (unsigned)(need < g ? need : g);
  if (!blocks) return;
  eri_jk_smem_kernel<LA, LB, LC, LD, PURE><<<blocks, 32 * DSS_SMEM_WARPS, smem, s>>>(a);
}

// Schwarz factors Q_ab = sqrt(max_ij |(ij|ij)|) for the pairs of one class: one
// warp per shell pair, the lanes splitting the bra primitive pairs (each lane
// sums its bra primitive pairs against every ket primitive pair), the diagonal
// integrals summed across the warp.
template <int LA, int LB, int BOYS, bool PURE>
__global__ void __launch_bounds__(128) schwarz_kernel(SchwarzArgs a) {
  constexpr int NA = dss_nfunc(LA, PURE), NB = dss_nfunc(LB, PURE);
  const int w = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5);
  const int lane = threadIdx.x & 31;
  if (w >= a.npair) return;
  const int pr = a.pair0 + w;
  const int sa = a.pair_a[pr], sb = a.pair_b[pr];
  const double ABx = a.sh_xyz[3 * sa] - a.sh_xyz[3 * sb];
  const double ABy = a.sh_xyz[3 * sa + 1] - a.sh_xyz[3 * sb + 1];
  const double ABz = a.sh_xyz[3 * sa + 2] - a.sh_xyz[3 * sb + 2];
  const PrimPair* pp = a.pp + a.pair_pp0[pr];
  const int npp = a.pair_npp[pr];
  double diag[NA * NB];
#pragma unroll
  for (int q = 0; q < NA * NB; ++q) diag[q] = 0.0;
  for (int ib = lane; ib < npp; ib += 32) {
    double I[NA * NB * NA * NB];
    EriClass<LA, LB, LA, LB>::template eval<BOYS, PURE>(pp + ib, 1, pp, npp, ABx, ABy, ABz, ABx, ABy, ABz, I,
                                                        a.boys_cell);
#pragma unroll
    for (int q = 0; q < NA * NB; ++q) diag[q] += I[q * NA * NB + q];
  }
  double mx = 0.0;
#pragma unroll
  for (int q = 0; q < NA * NB; ++q) mx = fmax(mx, fabs(warp_sum(diag[q])));
  if (lane == 0) a.Q[pr] = sqrt(mx);
}

// Host-side launchers (one translation unit per class defines them).
#define DSS_DECLARE_LAUNCHERS(la, lb, lc, ld, bc, kc) \
  void dss_launch_eri_jk_##la##lb##lc##ld(int boys, int pure, int mixed, int uhf, int tier, const EriArgs& a, \
                                          cudaStream_t s);
DSS_FOR_EACH_CLASS(DSS_DECLARE_LAUNCHERS)
#undef DSS_DECLARE_LAUNCHERS

void dss_launch_schwarz(int la, int lb, int boys, int pure, const SchwarzArgs& a, cudaStream_t s);
// variant 0: one thread per quartet; 1: warp-cooperative (when compiled for the class);
// 2, 3: one thread per quartet in register tier 1, 2 (plain form: reference Boys,
// FP64; other forms run tier 0); 4: the shared-memory Boys shape (plain form,
// L <= 2; split launches and other forms run tier 0); 5, 6, 7: variants 0, 2, 3
// on a one-wave grid.  uhf = 1: the unrestricted variant (thread per
// quartet, reference Boys only).
void dss_launch_eri_variant(int la, int lb, int lc, int ld, int boys, int pure, int mixed, int uhf, int variant,
                            const EriArgs& a, cudaStream_t s);
bool dss_has_coop(int la, int lb, int lc, int ld);
// Persistent grouped launches: group * 100 + the class's slot in its group, or
// -1 for a class that has none; the launcher of a group's kernel (false when
// the group has no kernel for this Boys mode / form).
int dss_persist_group(int la, int lb, int lc, int ld);
bool dss_launch_persist(int group, int boys, int pure, int mixed, const PersistArgs& p, cudaStream_t s);
// Loads the FP64 kernel of a plain build of the class (variant as above) if the
// CUDA runtime loads modules lazily, so that its first launch allocates nothing.
void dss_preload_eri_variant(int la, int lb, int lc, int ld, int boys, int pure, int variant);
void dss_launch_eri_jk(int la, int lb, int lc, int ld, int boys, int pure, int mixed, int uhf, int tier,
                       const EriArgs& a, cudaStream_t s);
