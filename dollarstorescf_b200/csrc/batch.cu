// Batched RHF: many molecules of uneven size in one set of launches.
//
// Every admitted molecule owns one region of a device arena: a small header
// (energies, iteration counter, DIIS state) followed by its n x n matrices and
// DIIS rings.  Regions stay in place while their molecule is in the batch, so
// molecules can join and leave between iterations (the serving loop's
// continuous batching) without moving the others.  Admission is by arena space.
//
// The batch's shells form one basis whose shell pairs and work lists never mix
// molecules (dss_setup_pairs with per-shell molecule ids); each ERI class is one
// launch over all molecules, reading and writing every molecule's own matrices
// through per-shell offsets.  The SCF steps run as batched kernels (one grid
// dimension over molecules): the reference's iteration (chem/scf/SCFSolver.cpp:
// 145-177: G, F, Pulay DIIS, X F X, eigenvectors, density, energy, convergence)
// with all per-molecule control (iteration count, DIIS ring, convergence flag)
// on the device, so one captured CUDA graph replays the same iteration for
// every molecule whatever its stage.  The eigensolver is the cyclic Jacobi
// method with one thread block per molecule, the matrix held in shared memory
// when it fits, warm-started from the previous iteration's vectors.
#include <atomic>
#include <cuda_runtime.h>

#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "dss.h"
#include "dss_internal.h"
#include "linalg.cuh"

namespace {

// Region layout (doubles): header, then matrices of n*n each, then rings, eps.
constexpr int kHdr = 256;
// M_GP, M_DP: G and D of the previous build (incremental form).
enum Mat { M_H, M_S, M_X, M_D, M_DT, M_J, M_K, M_G, M_FN, M_F, M_T1, M_T2, M_CP, M_C, M_V, M_T3, M_GP, M_DP, M_NMAT };
// Header slots
constexpr int H_E = 0, H_EPREV = 1, H_TRDG = 2, H_ENUC = 3, H_DOTS = 4, H_COEF = 16, H_B = 32, H_TRDH = 140,
              H_EFINAL = 141, H_XSCALE = 142, H_INT = 200;
// Integer header (as int view of doubles from H_INT): iteration, done, diis count, diis slot, nocc, n, status,
// final energy present; incremental form: iteration of the last full build, full builds in a row, final
// phase reached, the current iteration is a full build.
constexpr int I_IT = 0, I_DONE = 1, I_CNT = 2, I_SLOT = 3, I_NOCC = 4, I_N = 5, I_STATUS = 6, I_FINAL = 7,
              I_LASTFULL = 8, I_STREAK = 9, I_FPHASE = 10, I_FULL = 11;

__host__ __device__ inline size_t region_size(int n, int ds) {
  const size_t n2 = (size_t)n * n;
  size_t s = kHdr + (size_t)M_NMAT * n2 + 2 * (size_t)ds * n2 + (size_t)n + 8;
  return (s + 31) & ~(size_t)31;  // 256-byte granules
}
__device__ __forceinline__ double* mat(double* base, int n, int k) { return base + kHdr + (size_t)k * n * n; }
__device__ __forceinline__ double* ring_f(double* base, int n, int ds, int slot) {
  return base + kHdr + (size_t)M_NMAT * n * n + (size_t)slot * n * n;
}
__device__ __forceinline__ double* ring_e(double* base, int n, int ds, int slot) {
  return base + kHdr + (size_t)(M_NMAT + ds) * n * n + (size_t)slot * n * n;
}
__device__ __forceinline__ double* eps_of(double* base, int n, int ds) {
  return base + kHdr + (size_t)(M_NMAT + 2 * ds) * n * n;
}
__device__ __forceinline__ int* ihdr(double* base) { return reinterpret_cast<int*>(base + H_INT); }

struct BatchView {
  double* arena;
  const long long* region;  // per batch slot
  const int* nvec;
  const int* active;        // per batch slot
  int nb, ds;
};

#define BV_BEGIN()                                   \
  const int b = blockIdx.y;                          \
  if (b >= v.nb || !v.active[b]) return;             \
  const int n = v.nvec[b];                           \
  double* base = v.arena + v.region[b];              \
  const long long n2 = (long long)n * n;             \
  (void)n2;

// Dt = 2 D, J = K = 0
__global__ void k_prep(BatchView v) {
  BV_BEGIN();
  for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < n2; t += (long long)gridDim.x * blockDim.x) {
    mat(base, n, M_DT)[t] = 2.0 * mat(base, n, M_D)[t];
    mat(base, n, M_J)[t] = 0.0;
    mat(base, n, M_K)[t] = 0.0;
  }
}

// Incremental form: which molecules run a full build this iteration (the
// single-molecule rule of dss_scf_solve: the first two iterations, every
// rebuild_every-th, and all of the final phase), then Dt = 2 D (full) or
// 2 (D - D_prev), J = K = 0.
__global__ void k_mode(BatchView v, int rebuild_every) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= v.nb || !v.active[b]) return;
  int* ih = ihdr(v.arena + v.region[b]);
  const int it = ih[I_IT] + 1;
  const int full = ih[I_FPHASE] || it <= 2 || it - ih[I_LASTFULL] >= rebuild_every;
  ih[I_FULL] = full;
  if (full) {
    ih[I_LASTFULL] = it;
    ih[I_STREAK] += 1;
  } else {
    ih[I_STREAK] = 0;
  }
}

__global__ void k_force_full(BatchView v) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= v.nb) return;
  int* ih = ihdr(v.arena + v.region[b]);
  ih[I_LASTFULL] = -(1 << 30);
  ih[I_STREAK] = 0;
}

__global__ void k_prep_inc(BatchView v) {
  BV_BEGIN();
  const bool full = ihdr(base)[I_FULL] != 0;
  const double* D = mat(base, n, M_D);
  const double* Dp = mat(base, n, M_DP);
  for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < n2; t += (long long)gridDim.x * blockDim.x) {
    mat(base, n, M_DT)[t] = full ? 2.0 * D[t] : 2.0 * (D[t] - Dp[t]);
    mat(base, n, M_J)[t] = 0.0;
    mat(base, n, M_K)[t] = 0.0;
  }
}

// Per shell block max |Dt| of every active molecule (the density-weighted
// screen's bound); FLT_MAX for a full build, so that its quartets all run in FP64.
// Shells of a molecule are consecutive in the batch basis; entry (a, b) of the
// molecule's ns x ns block sits at sh_dbase + loc(a) ns + loc(b).
struct BlockMaxArgs {
  const int *sh_mol, *sh_loc, *sh_nsm, *sh_f0, *sh_nf;
  const long long *sh_mbase, *sh_dbase;
  float* dmax;
  int nshell;
};
__global__ void k_block_max(BatchView v, BlockMaxArgs a) {
  for (int g = blockIdx.x; g < a.nshell; g += gridDim.x) {
    const int slot = a.sh_mol[g];
    if (!v.active[slot]) continue;
    const double* base = v.arena + v.region[slot];
    const bool full = reinterpret_cast<const int*>(base + H_INT)[I_FULL] != 0;
    const int n = v.nvec[slot], ns = a.sh_nsm[g], la = a.sh_loc[g], g0 = g - la;
    const double* Dt = v.arena + a.sh_mbase[g];
    const int fa = a.sh_f0[g], na = a.sh_nf[g];
    for (int sb = threadIdx.x; sb < ns; sb += blockDim.x) {
      float out = FLT_MAX;
      if (!full) {
        const int fb = a.sh_f0[g0 + sb], nbf = a.sh_nf[g0 + sb];
        double m = 0.0;
        for (int i = 0; i < na; ++i)
          for (int j = 0; j < nbf; ++j) m = fmax(m, fabs(Dt[(long long)(fa + i) * n + fb + j]));
        out = (float)(m * (1.0 + 1e-6));  // round up: the bound stays a bound in float
      }
      a.dmax[a.sh_dbase[g] + (long long)la * ns + sb] = out;
    }
  }
}

// G = (J + J^T) - (K + K^T)/2 (+ G_prev after an incremental build), F_new = H + G;
// the incremental form keeps G and D as the next iteration's G_prev, D_prev.
__global__ void k_fock_inc(BatchView v) {
  BV_BEGIN();
  const bool full = ihdr(base)[I_FULL] != 0;
  const double* J = mat(base, n, M_J);
  const double* K = mat(base, n, M_K);
  double* Gp = mat(base, n, M_GP);
  for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < n2; t += (long long)gridDim.x * blockDim.x) {
    const int r = (int)(t / n), c = (int)(t % n);
    const long long u = (long long)c * n + r;
    double g = (J[t] + J[u]) - 0.5 * (K[t] + K[u]);
    if (!full) g += Gp[t];
    Gp[t] = g;
    mat(base, n, M_DP)[t] = mat(base, n, M_D)[t];
    mat(base, n, M_G)[t] = g;
    mat(base, n, M_FN)[t] = mat(base, n, M_H)[t] + g;
  }
}

// G = (J + J^T) - (K + K^T)/2, F_new = H + G
__global__ void k_fock(BatchView v) {
  BV_BEGIN();
  const double* J = mat(base, n, M_J);
  const double* K = mat(base, n, M_K);
  for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < n2; t += (long long)gridDim.x * blockDim.x) {
    const int r = (int)(t / n), c = (int)(t % n);
    const long long u = (long long)c * n + r;
    const double g = (J[t] + J[u]) - 0.5 * (K[t] + K[u]);
    mat(base, n, M_G)[t] = g;
    mat(base, n, M_FN)[t] = mat(base, n, M_H)[t] + g;
  }
}

// C = alpha op(A) op(B) + beta C per molecule (matrix indices into the region).
__global__ void k_gemm(BatchView v, int ka, int kb, int kc, int ta, int tb, double alpha, double beta) {
  const int b = blockIdx.z;
  if (b >= v.nb || !v.active[b]) return;
  const int n = v.nvec[b];
  const int row0 = blockIdx.y * 32, col0 = blockIdx.x * 32;
  if (row0 >= n || col0 >= n) return;
  double* base = v.arena + v.region[b];
  const double* A = mat(base, n, ka);
  const double* B = mat(base, n, kb);
  double* C = mat(base, n, kc);
  __shared__ double As[32][33];
  __shared__ double Bs[32][33];
  const int tx = threadIdx.x, ty = threadIdx.y;
  double acc[4] = {0.0, 0.0, 0.0, 0.0};
  for (int k0 = 0; k0 < n; k0 += 32) {
    for (int r = ty; r < 32; r += 8) {
      const int i = row0 + r, k = k0 + tx;
      As[r][tx] = (i < n && k < n) ? (ta ? A[(size_t)k * n + i] : A[(size_t)i * n + k]) : 0.0;
      const int kk = k0 + r, j = col0 + tx;
      Bs[r][tx] = (kk < n && j < n) ? (tb ? B[(size_t)j * n + kk] : B[(size_t)kk * n + j]) : 0.0;
    }
    __syncthreads();
#pragma unroll 8
    for (int k = 0; k < 32; ++k) {
      const double bv = Bs[k][tx];
#pragma unroll
      for (int q = 0; q < 4; ++q) acc[q] += As[ty + 8 * q][k] * bv;
    }
    __syncthreads();
  }
  for (int q = 0; q < 4; ++q) {
    const int i = row0 + ty + 8 * q, j = col0 + tx;
    if (i < n && j < n) {
      const size_t o = (size_t)i * n + j;
      C[o] = alpha * acc[q] + (beta == 0.0 ? 0.0 : beta * C[o]);
    }
  }
}

// DIIS slot choice (lalib/DIIS.ipp:19-62) for molecules in their second or later iteration.
__global__ void k_diis_choose(BatchView v) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= v.nb || !v.active[b]) return;
  double* base = v.arena + v.region[b];
  int* ih = ihdr(base);
  for (int i = 0; i < 10; ++i) base[H_DOTS + i] = 0.0;
  if (ih[I_IT] < 1) return;  // first iteration: F = F_new
  int count = ih[I_CNT], slot = 0;
  if (count < v.ds) {
    slot = count;
    ++count;
  } else {
    double mx = 0.0;
    for (int i = 0; i < v.ds; ++i) {
      const double e = base[H_B + i * 10 + i];
      if (e > mx) {
        mx = e;
        slot = i;
      }
    }
  }
  ih[I_CNT] = count;
  ih[I_SLOT] = slot;
}

// e = T2 - T2^T and F_new into the chosen ring slots.
__global__ void k_diis_store(BatchView v) {
  BV_BEGIN();
  int* ih = ihdr(base);
  if (ih[I_IT] < 1) return;
  const int slot = ih[I_SLOT];
  const double* T2 = mat(base, n, M_T2);
  double* e = ring_e(base, n, v.ds, slot);
  double* f = ring_f(base, n, v.ds, slot);
  for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < n2; t += (long long)gridDim.x * blockDim.x) {
    const int r = (int)(t / n), c = (int)(t % n);
    e[t] = T2[t] - T2[(long long)c * n + r];
    f[t] = mat(base, n, M_FN)[t];
  }
}

// dots[i] = <e_i, e_slot>; blockIdx.z = ring entry.
__global__ void k_diis_dots(BatchView v) {
  BV_BEGIN();
  int* ih = ihdr(base);
  const int i = blockIdx.z;
  if (ih[I_IT] < 1 || i >= ih[I_CNT]) return;
  const double* a = ring_e(base, n, v.ds, i);
  const double* c = ring_e(base, n, v.ds, ih[I_SLOT]);
  double acc = 0.0;
  for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < n2; t += (long long)gridDim.x * blockDim.x)
    acc += a[t] * c[t];
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
  __shared__ double red[32];
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    double s = 0.0;
    for (int k = 0; k < (int)(blockDim.x >> 5); ++k) s += red[k];
    atomicAdd(base + H_DOTS + i, s);
  }
}

// Bordered B c = (0,..,0,1) by Gaussian elimination with partial pivoting; a
// singular system keeps only the newest Fock matrix.
__global__ void k_diis_solve(BatchView v) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= v.nb || !v.active[b]) return;
  double* base = v.arena + v.region[b];
  int* ih = ihdr(base);
  if (ih[I_IT] < 1) return;
  const int count = ih[I_CNT], slot = ih[I_SLOT];
  double* B = base + H_B;
  double* coef = base + H_COEF;
  for (int i = 0; i < count; ++i) {
    B[slot * 10 + i] = base[H_DOTS + i];
    B[i * 10 + slot] = base[H_DOTS + i];
  }
  const int m = count + 1;
  double M[10][11];
  for (int i = 0; i < m; ++i) {
    for (int j = 0; j < m; ++j) M[i][j] = (i < count && j < count) ? B[i * 10 + j] : ((i == count && j == count) ? 0.0 : 1.0);
    M[i][m] = (i == count) ? 1.0 : 0.0;
  }
  bool singular = false;
  for (int k = 0; k < m; ++k) {
    int piv = k;
    for (int i = k + 1; i < m; ++i)
      if (fabs(M[i][k]) > fabs(M[piv][k])) piv = i;
    if (M[piv][k] == 0.0) {
      singular = true;
      break;
    }
    if (piv != k)
      for (int j = 0; j <= m; ++j) {
        const double t = M[k][j];
        M[k][j] = M[piv][j];
        M[piv][j] = t;
      }
    for (int i = k + 1; i < m; ++i) {
      const double f = M[i][k] / M[k][k];
      for (int j = k; j <= m; ++j) M[i][j] -= f * M[k][j];
    }
  }
  if (!singular) {
    double x[10];
    for (int i = m - 1; i >= 0; --i) {
      double s = M[i][m];
      for (int j = i + 1; j < m; ++j) s -= M[i][j] * x[j];
      x[i] = s / M[i][i];
    }
    for (int i = 0; i < count; ++i) coef[i] = x[i];
  } else {
    for (int i = 0; i < count; ++i) coef[i] = (i == slot) ? 1.0 : 0.0;
  }
}

// F = sum_i c_i F_i (iteration >= 2) or F = F_new (first iteration)
__global__ void k_diis_combine(BatchView v) {
  BV_BEGIN();
  int* ih = ihdr(base);
  const int count = ih[I_CNT];
  const bool first = ih[I_IT] < 1;
  double* F = mat(base, n, M_F);
  for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < n2; t += (long long)gridDim.x * blockDim.x) {
    if (first) {
      F[t] = mat(base, n, M_FN)[t];
    } else {
      double s = 0.0;
      for (int i = 0; i < count; ++i) s += base[H_COEF + i] * ring_f(base, n, v.ds, i)[t];
      F[t] = s;
    }
  }
}

// Cyclic Jacobi, one block per molecule: A (matrix ka, overwritten) -> eigenvalues
// ascending in eps, eigenvectors as columns of matrix kv (rotations accumulate in
// the spare matrix kt, transposed).  MODE 0: A (packed upper triangle) and VT in
// shared memory; 1: packed A in shared memory, VT in global memory; 2: both dense
// in global memory.  A launch takes the molecules with n_lo < n <= n_hi.
template <int MODE>
__global__ void __launch_bounds__(512) k_jacobi(BatchView v, int ka, int kv, int kt, int max_sweeps, double tol,
                                                int n_lo, int n_hi) {
  const int b = blockIdx.x;
  if (b >= v.nb || !v.active[b]) return;
  const int n = v.nvec[b];
  if (n <= n_lo || n > n_hi) return;
  double* base = v.arena + v.region[b];
  extern __shared__ double sm[];
  const size_t nn = (size_t)n * n, np = dss_packed_size(n);
  const int tid = threadIdx.x, nt = blockDim.x;
  double* src = mat(base, n, ka);
  if (MODE <= 1) {
    double* VT = MODE == 0 ? sm + np : mat(base, n, kt);
    void* aux = sm + np + (MODE == 0 ? nn : 0);
    DssPackedSym A{sm, n};
    for (int i = tid >> 5; i < n; i += nt >> 5)
      for (int jj = i + (tid & 31); jj < n; jj += 32) A.at(i, jj) = src[(size_t)i * n + jj];
    for (int t = tid; t < (int)nn; t += nt) VT[t] = (t / n == t % n) ? 1.0 : 0.0;
    __syncthreads();
    dss_block_jacobi(A, VT, aux, max_sweeps, tol);
    __syncthreads();
    dss_block_jacobi_sorted(A, VT, eps_of(base, n, v.ds), mat(base, n, kv));
  } else {
    double* VT = mat(base, n, kt);
    DssDenseSym A{src, n};
    for (int t = tid; t < (int)nn; t += nt) VT[t] = (t / n == t % n) ? 1.0 : 0.0;
    __syncthreads();
    dss_block_jacobi(A, VT, sm, max_sweeps, tol);
    __syncthreads();
    dss_block_jacobi_sorted(A, VT, eps_of(base, n, v.ds), mat(base, n, kv));
  }
}

__global__ void k_copy(BatchView v, int ksrc, int kdst) {
  BV_BEGIN();
  for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < n2; t += (long long)gridDim.x * blockDim.x)
    mat(base, n, kdst)[t] = mat(base, n, ksrc)[t];
}

// D = C_occ C_occ^T
__global__ void k_density(BatchView v) {
  BV_BEGIN();
  const int nocc = ihdr(base)[I_NOCC];
  const double* C = mat(base, n, M_C);
  for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < n2; t += (long long)gridDim.x * blockDim.x) {
    const int r = (int)(t / n), c = (int)(t % n);
    double s = 0.0;
    for (int k = 0; k < nocc; ++k) s += C[(size_t)r * n + k] * C[(size_t)c * n + k];
    mat(base, n, M_D)[t] = s;
  }
}

// tr(D X) into header slot hs (one block per molecule).
__global__ void k_trace(BatchView v, int kx, int hs) {
  const int b = blockIdx.x;
  if (b >= v.nb || !v.active[b]) return;
  const int n = v.nvec[b];
  double* base = v.arena + v.region[b];
  const double* D = mat(base, n, M_D);
  const double* X = mat(base, n, kx);
  double acc = 0.0;
  for (long long t = threadIdx.x; t < (long long)n * n; t += blockDim.x) acc += D[t] * X[t];
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
  __shared__ double red[32];
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    double s = 0.0;
    for (int k = 0; k < (int)(blockDim.x >> 5); ++k) s += red[k];
    base[hs] = s;
  }
}

// E_elec = 2 sum_occ eps - tr(D G); iteration count, convergence (checkConvergence),
// iteration cap; active flags for the next iteration; counts molecules still active.
// Incremental form (inc != 0): convergence also needs the last two builds to have
// been full ones, and |dE| < final_switch starts the final (all full) phase.
__global__ void k_energy(BatchView v, double conv, int max_iter, int inc, double final_switch, int* active_out,
                         int* n_active) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= v.nb) return;
  if (!v.active[b]) {
    active_out[b] = 0;
    return;
  }
  const int n = v.nvec[b];
  double* base = v.arena + v.region[b];
  int* ih = ihdr(base);
  const double* w = eps_of(base, n, v.ds);
  double e = 0.0;
  for (int i = 0; i < ih[I_NOCC]; ++i) e += 2.0 * w[i];
  e -= base[H_TRDG];
  base[H_EPREV] = base[H_E];
  base[H_E] = e;
  ih[I_IT] += 1;
  int act = 1;
  const double de = fabs(e - base[H_EPREV]);
  if (inc && de < final_switch) ih[I_FPHASE] = 1;
  if (!isfinite(e)) {
    ih[I_DONE] = 1;
    ih[I_STATUS] = DSS_ERR_NOCONV;
    act = 0;
  } else if (de < conv && (!inc || ih[I_STREAK] >= 2)) {
    ih[I_DONE] = 1;
    ih[I_STATUS] = DSS_OK;
    act = 0;
  } else if (ih[I_IT] >= max_iter) {
    ih[I_DONE] = 1;
    ih[I_STATUS] = DSS_ERR_NOCONV;
    act = 0;
  }
  active_out[b] = act;
  atomicAdd(n_active + (act ? 0 : 1), 1);  // [0] still iterating, [1] finished in this iteration
}

// Final energy E = 2 tr(D H) + tr(D G) + E_nuc (calculateEnergies, Energy.cpp:21-50).
__global__ void k_final(BatchView v) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= v.nb || !v.active[b]) return;
  double* base = v.arena + v.region[b];
  base[H_EFINAL] = 2.0 * base[H_TRDH] + base[H_TRDG] + base[H_ENUC];
  ihdr(base)[I_FINAL] = 1;
}

// Admission set-up of one molecule's region (single block per matrix op).
__global__ void k_admit_init(double* base, int n, const double* Hp, const double* Sp, const double* Dp, int nocc,
                             double e_nuc) {
  const long long n2 = (long long)n * n;
  for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < n2; t += (long long)gridDim.x * blockDim.x) {
    const int r = (int)(t / n), c = (int)(t % n);
    const int x = r > c ? r : c, y = r > c ? c : r;
    const long long pi = (long long)x * (x + 1) / 2 + y;
    mat(base, n, M_H)[t] = Hp[pi];
    mat(base, n, M_S)[t] = Sp[pi];
    mat(base, n, M_T1)[t] = Sp[pi];
    mat(base, n, M_D)[t] = Dp ? Dp[pi] : 0.0;
    mat(base, n, M_CP)[t] = (r == c) ? 1.0 : 0.0;
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    for (int i = 0; i < kHdr; ++i) base[i] = 0.0;
    base[H_ENUC] = e_nuc;
    int* ih = ihdr(base);
    ih[I_NOCC] = nocc;
    ih[I_N] = n;
  }
}

// out = V diag(eps)^-1/2 per molecule (eps: the molecule's eigenvalue slot).
// X = S^-1/2 by the coupled Newton-Schulz iteration (Higham, Functions of
// Matrices, 2008, eq. 6.35): Y0 = S/c, Z0 = I, T = (3 I - Z Y)/2, Y <- Y T,
// Z <- T Z; Z -> (S/c)^-1/2 quadratically once Z Y is near I.  c = the largest
// absolute row sum of S bounds its largest eigenvalue, so the iteration
// converges.  One block per molecule sets c, Y0 and Z0.
__global__ void k_ns_init(BatchView v, int ks, int ky, int kz) {
  BV_BEGIN();
  __shared__ double red[256];
  const double* S = mat(base, n, ks);
  double m = 0.0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    double r = 0.0;
    for (int j = 0; j < n; ++j) r += fabs(S[(size_t)i * n + j]);
    m = fmax(m, r);
  }
  red[threadIdx.x] = m;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w) red[threadIdx.x] = fmax(red[threadIdx.x], red[threadIdx.x + w]);
    __syncthreads();
  }
  const double c = red[0];
  for (long long t = threadIdx.x; t < n2; t += blockDim.x) {
    mat(base, n, ky)[t] = S[t] / c;
    mat(base, n, kz)[t] = (t / n == t % n) ? 1.0 : 0.0;
  }
  if (threadIdx.x == 0) base[H_XSCALE] = c;
}

// T = 1.5 I - 0.5 P, in place.
__global__ void k_ns_t(BatchView v, int kp) {
  BV_BEGIN();
  double* P = mat(base, n, kp);
  for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < n2; t += (long long)gridDim.x * blockDim.x)
    P[t] = (t / n == t % n ? 1.5 : 0.0) - 0.5 * P[t];
}

// X = Z / sqrt(c); *bad set when max |X S X - I| = max |P / c - I| exceeds tol
// (P = Z S Z).
__global__ void k_ns_finish(BatchView v, int kp, int kz, int kx, double tol, int* bad) {
  BV_BEGIN();
  const double* P = mat(base, n, kp);
  const double c = base[H_XSCALE];
  const double r = 1.0 / sqrt(c);
  bool off = false;
  for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < n2; t += (long long)gridDim.x * blockDim.x) {
    mat(base, n, kx)[t] = mat(base, n, kz)[t] * r;
    off = off || !(fabs(P[t] / c - (t / n == t % n ? 1.0 : 0.0)) <= tol);
  }
  if (off) atomicOr(bad, 1);
}

__global__ void k_scale_cols_eps(BatchView v, int kv, int kout) {
  BV_BEGIN();
  const double* w = eps_of(base, n, v.ds);
  for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < n2; t += (long long)gridDim.x * blockDim.x)
    mat(base, n, kout)[t] = mat(base, n, kv)[t] / sqrt(w[t % n]);
}

inline dim3 grid2(long long per_mol, int nb) {
  long long bx = (per_mol + 255) / 256;
  if (bx > 64) bx = 64;
  if (bx < 1) bx = 1;
  return dim3((unsigned)bx, (unsigned)nb);
}

}  // namespace

struct dss_batch_mol {
  bool live = false;
  int n = 0, nocc = 0, natom = 0;
  long long region = -1;
  size_t size = 0;
  BasisHost basis;  // molecule-local
  PairSet pairs;    // its shell pairs and Schwarz factors, made once at admission
  bool needs_x = true;  // X = S^-1/2 not computed yet (done for all new molecules at the next step)
  long long pp_off = 0;  // its primitive pairs' first record in the batch's device pool
  // Its work lists in the batch's device task pool: class i's tasks at
  // task_off + task_cls_off[i], task_cnt[i] of them (pair indices local to the
  // molecule; the host copies are dropped after the upload).
  long long task_off = 0;
  size_t task_n = 0;
  std::vector<int> task_cnt;
  std::vector<long long> task_cls_off;
};

// Device pool of the live molecules' primitive-pair records (10 doubles each),
// filled at admission, so a change of composition moves no primitive pairs:
// the merged pair list indexes the pool.  Removal leaves a hole; the pool is
// compacted when it grows.
struct PpPool {
  double* ptr = nullptr;
  size_t cap = 0, used = 0;  // records
  PpPool() = default;
  PpPool(const PpPool&) = delete;
  PpPool& operator=(const PpPool&) = delete;
  ~PpPool() {
    if (ptr) cudaFree(ptr);
  }
};

// Device pool of the live molecules' own work lists (int4 tasks), filled at
// admission; a change of composition gathers the batch's lists from it on the
// device (k_gather_tasks) instead of merging and uploading them from the host.
// Removal leaves a hole; the pool is compacted when it grows.
struct TaskPool {
  int4* ptr = nullptr;
  size_t cap = 0, used = 0;  // tasks
  TaskPool() = default;
  TaskPool(const TaskPool&) = delete;
  TaskPool& operator=(const TaskPool&) = delete;
  ~TaskPool() {
    if (ptr) cudaFree(ptr);
  }
};

// One run of a molecule's class-i tasks copied into the batch's class-i list,
// its pair indices moved by (dx, dy) into the merged pair order, w = its slot.
struct TaskSeg {
  const int4* src;
  int4* dst;
  int n, dx, dy, slot;
};

struct dss_batch {
  dss_ctx* ctx = nullptr;
  std::string err;
  int ds = 8;
  DevBuf<double> arena;
  size_t arena_doubles = 0;
  std::vector<std::pair<size_t, size_t>> free_list;  // (offset, size) in doubles
  std::vector<dss_batch_mol> mols;
  bool dirty = true;
  // current composition
  std::vector<int> slot_mol;  // batch slot -> molecule handle
  DevBuf<long long> d_region;
  DevBuf<int> d_n, d_active, d_active_next, d_nact;
  DevBuf<int> d_pending;  // per slot: 1 while the molecule's X is not computed
  DevBuf<int> d_nsbad;    // set when the Newton-Schulz X of a new molecule did not converge
  DevBuf<double> admit_tmp;  // admission scratch (packed H, S, guess), grow-only
  PpPool pp_pool;
  TaskPool task_pool;
  DevBuf<TaskSeg> d_segs;       // the gather's segment table, grow-only
  std::vector<TaskSeg> h_segs;  // its host image (kept until the next rebuild)
  int nmax = 0;
  int* h_nact = nullptr;  // pinned: molecules still iterating, molecules finished in the last iteration
  std::vector<int> last_finished;  // handles whose results the last dss_batch_step produced
  cudaGraphExec_t graph = nullptr;
  bool have_graph_opts = false;
  bool eager_ran = false;     // an eager iteration ran since the last change (next one captures)
  dss_scf_opts graph_opts{};  // the options the captured iteration was built with
  int inc = 0;                // the last step ran the incremental form (finalize follows it)
  ~dss_batch() {
    if (graph) cudaGraphExecDestroy(graph);
    if (h_nact) cudaFreeHost(h_nact);
    if (ctx) dss_destroy(ctx);
  }
};

namespace {

int bfail(dss_batch* b, int code, const std::string& m) {
  b->err = m;
  return code;
}

bool arena_alloc(dss_batch* b, size_t want, size_t* off) {
  for (size_t i = 0; i < b->free_list.size(); ++i) {
    if (b->free_list[i].second >= want) {
      *off = b->free_list[i].first;
      b->free_list[i].first += want;
      b->free_list[i].second -= want;
      if (!b->free_list[i].second) b->free_list.erase(b->free_list.begin() + i);
      return true;
    }
  }
  return false;
}

void arena_free(dss_batch* b, size_t off, size_t size) {
  b->free_list.push_back({off, size});
  std::sort(b->free_list.begin(), b->free_list.end());
  std::vector<std::pair<size_t, size_t>> merged;
  for (auto& f : b->free_list) {
    if (!merged.empty() && merged.back().first + merged.back().second == f.first) merged.back().second += f.second;
    else merged.push_back(f);
  }
  b->free_list = merged;
}

BatchView view(dss_batch* b, const int* active) {
  BatchView v;
  v.arena = b->arena.ptr;
  v.region = b->d_region.ptr;
  v.nvec = b->d_n.ptr;
  v.active = active;
  v.nb = (int)b->slot_mol.size();
  v.ds = b->ds;
  return v;
}

// Uploads a new molecule's primitive pairs into the pool (growing and compacting
// it over the live molecules when full) and records their offset.
int pool_put(dss_batch* b, dss_batch_mol* m) {
  PpPool& pool = b->pp_pool;
  cudaStream_t s = b->ctx->stream;
  const size_t rec = m->pairs.pp.size() / 10;
  if (pool.used + rec > pool.cap) {
    size_t live = rec;
    for (const auto& o : b->mols)
      if (o.live) live += o.pairs.pp.size() / 10;
    const size_t cap = std::max<size_t>(std::max<size_t>(2 * pool.cap, live + live / 2), 1 << 16);
    double* np = nullptr;
    if (cudaMalloc((void**)&np, cap * 10 * sizeof(double)) != cudaSuccess) return DSS_ERR_OOM;
    size_t at = 0;
    for (auto& o : b->mols) {
      if (!o.live) continue;
      const size_t r = o.pairs.pp.size() / 10;
      if (r && cudaMemcpyAsync(np + at * 10, pool.ptr + (size_t)o.pp_off * 10, r * 10 * sizeof(double),
                               cudaMemcpyDeviceToDevice, s) != cudaSuccess) {
        cudaFree(np);
        return DSS_ERR_CUDA;
      }
      o.pp_off = (long long)at;
      at += r;
    }
    if (cudaStreamSynchronize(s) != cudaSuccess) {
      cudaFree(np);
      return DSS_ERR_CUDA;
    }
    if (pool.ptr) cudaFree(pool.ptr);
    pool.ptr = np;
    pool.cap = cap;
    pool.used = at;
    b->dirty = true;  // the live molecules' offsets moved
  }
  if (rec && cudaMemcpyAsync(pool.ptr + pool.used * 10, m->pairs.pp.data(), rec * 10 * sizeof(double),
                             cudaMemcpyHostToDevice, s) != cudaSuccess)
    return DSS_ERR_CUDA;
  m->pp_off = (long long)pool.used;
  pool.used += rec;
  return DSS_OK;
}

// Uploads a new molecule's work lists (all classes, one run) into the task
// pool, growing and compacting it over the live molecules when full, and drops
// the host copies.
int task_put(dss_batch* b, dss_batch_mol* m) {
  TaskPool& pool = b->task_pool;
  cudaStream_t s = b->ctx->stream;
  HostTasks& ht = m->pairs.tasks;
  const size_t nq = ht.tasks.size();
  m->task_cnt.assign(nq, 0);
  m->task_cls_off.assign(nq, 0);
  size_t rec = 0;
  for (size_t ci = 0; ci < nq; ++ci) {
    m->task_cls_off[ci] = (long long)rec;
    m->task_cnt[ci] = (int)ht.tasks[ci].size();
    rec += ht.tasks[ci].size();
  }
  if (pool.used + rec > pool.cap) {
    size_t live = rec;
    for (const auto& o : b->mols)
      if (o.live) live += o.task_n;
    const size_t cap = std::max<size_t>(std::max<size_t>(2 * pool.cap, live + live / 2), 1 << 16);
    int4* np = nullptr;
    if (cudaMalloc((void**)&np, cap * sizeof(int4)) != cudaSuccess) return DSS_ERR_OOM;
    size_t at = 0;
    for (auto& o : b->mols) {
      if (!o.live) continue;
      if (o.task_n && cudaMemcpyAsync(np + at, pool.ptr + o.task_off, o.task_n * sizeof(int4),
                                      cudaMemcpyDeviceToDevice, s) != cudaSuccess) {
        cudaFree(np);
        return DSS_ERR_CUDA;
      }
      o.task_off = (long long)at;
      at += o.task_n;
    }
    if (cudaStreamSynchronize(s) != cudaSuccess) {
      cudaFree(np);
      return DSS_ERR_CUDA;
    }
    if (pool.ptr) cudaFree(pool.ptr);
    pool.ptr = np;
    pool.cap = cap;
    pool.used = at;
    b->dirty = true;  // the live molecules' offsets moved
  }
  for (size_t ci = 0; ci < nq; ++ci) {
    const std::vector<int4>& t = ht.tasks[ci];
    if (!t.empty() && cudaMemcpyAsync(pool.ptr + pool.used + m->task_cls_off[ci], t.data(), t.size() * sizeof(int4),
                                      cudaMemcpyHostToDevice, s) != cudaSuccess)
      return DSS_ERR_CUDA;
  }
  m->task_off = (long long)pool.used;
  m->task_n = rec;
  pool.used += rec;
  // The copies above are from pageable memory, so they have left the host
  // vectors when cudaMemcpyAsync returns.
  for (auto& t : ht.tasks) std::vector<int4>().swap(t);
  return DSS_OK;
}

__global__ void k_gather_tasks(const TaskSeg* __restrict__ segs, int nseg) {
  for (int g = blockIdx.x; g < nseg; g += gridDim.x) {
    const TaskSeg sg = segs[g];
    for (int i = threadIdx.x; i < sg.n; i += blockDim.x) {
      const int4 t = sg.src[i];
      sg.dst[i] = make_int4(t.x + sg.dx, t.y + sg.dy, t.z, sg.slot);
    }
  }
}

// Rebuilds the batch basis (pairs, Schwarz factors, work lists) and the
// per-slot tables for the live molecules.
int rebuild(dss_batch* b) {
  dss_ctx* ctx = b->ctx;
  b->slot_mol.clear();
  for (size_t h = 0; h < b->mols.size(); ++h)
    if (b->mols[h].live) b->slot_mol.push_back((int)h);
  const int nb = (int)b->slot_mol.size();
  if (b->graph) {
    cudaGraphExecDestroy(b->graph);
    b->graph = nullptr;
  }
  b->eager_ran = false;
  if (!nb) {
    b->dirty = false;
    return DSS_OK;
  }
  BasisHost B;
  B.pure = b->mols[b->slot_mol[0]].basis.pure;
  std::vector<long long> mbase, jbase, kbase, dbase;
  std::vector<int> shn, shmol, shloc, shnsm;
  std::vector<long long> region(nb);
  std::vector<int> nv(nb);
  long long dtot = 0;
  b->nmax = 0;
  for (int s = 0; s < nb; ++s) {
    const dss_batch_mol& m = b->mols[b->slot_mol[s]];
    const BasisHost& mb = m.basis;
    region[s] = m.region;
    nv[s] = m.n;
    b->nmax = std::max(b->nmax, m.n);
    const long long n2 = (long long)m.n * m.n;
    const int ns = (int)mb.l.size();
    const int p0 = (int)B.exps.size();
    for (int q = 0; q < ns; ++q) {
      B.l.push_back(mb.l[q]);
      B.nprim.push_back(mb.nprim[q]);
      B.prim0.push_back(p0 + mb.prim0[q]);
      B.f0.push_back(mb.f0[q]);
      for (int k = 0; k < 3; ++k) B.xyz.push_back(mb.xyz[3 * q + k]);
      B.mol.push_back(s);
      mbase.push_back(m.region + kHdr + (long long)M_DT * n2);
      jbase.push_back(m.region + kHdr + (long long)M_J * n2);
      kbase.push_back(m.region + kHdr + (long long)M_K * n2);
      dbase.push_back(dtot);
      shn.push_back(m.n);
      shmol.push_back(s);
      shloc.push_back(q);
      shnsm.push_back(ns);
    }
    dtot += (long long)ns * ns;
    B.exps.insert(B.exps.end(), mb.exps.begin(), mb.exps.end());
    B.wts.insert(B.wts.end(), mb.wts.begin(), mb.wts.end());
  }
  B.nbf = 0;
  ctx->nmol = nb;
  std::vector<const PairSet*> parts(nb);
  std::vector<int> shell_off(nb);
  for (int s = 0, off = 0; s < nb; ++s) {
    parts[s] = &b->mols[b->slot_mol[s]].pairs;
    shell_off[s] = off;
    off += (int)b->mols[b->slot_mol[s]].basis.l.size();
  }
  PairSet P;
  std::vector<long long> pp_off(nb);
  for (int sl = 0; sl < nb; ++sl) pp_off[sl] = b->mols[b->slot_mol[sl]].pp_off;
  dss_pairs_merge(parts, shell_off, &P, &pp_off);
  ctx->ext_pp = reinterpret_cast<const PrimPair*>(b->pp_pool.ptr);
  // Work lists: every molecule's own lists (made at admission), their pair
  // indices moved to the merged (class, molecule) order: no search over the
  // batch's pairs when its composition changes.
  const int ncls = dss_num_pair_classes();
  std::vector<std::vector<int>> lc0(nb), lc1(nb);
  std::vector<int> mc0(ncls, 0);
  std::vector<std::vector<int>> off(nb, std::vector<int>(ncls, 0));
  for (int sl = 0; sl < nb; ++sl) dss_class_ranges(parts[sl]->cls, &lc0[sl], &lc1[sl]);
  for (int c = 0, acc = 0; c < ncls; ++c) {
    mc0[c] = acc;
    for (int sl = 0; sl < nb; ++sl) {
      off[sl][c] = acc - mc0[c];
      acc += lc1[sl][c] - lc0[sl][c];
    }
  }
  const size_t nq = parts[0]->tasks.shell_quartets.size();
  std::vector<int> cnt(nq, 0);
  std::vector<long long> sq(nq, 0), pq(nq, 0);
  for (size_t ci = 0; ci < nq; ++ci)
    for (int sl = 0; sl < nb; ++sl) {
      const dss_batch_mol& m = b->mols[b->slot_mol[sl]];
      cnt[ci] += m.task_cnt[ci];
      sq[ci] += parts[sl]->tasks.shell_quartets[ci];
      pq[ci] += parts[sl]->tasks.prim_quartets[ci];
    }
  int rc = dss_pairs_install(ctx, std::move(B), std::move(P), nullptr, true);
  if (rc != DSS_OK) return bfail(b, rc, ctx->err);
  if ((rc = dss_install_task_counts(ctx, cnt, sq, pq)) != DSS_OK) return bfail(b, rc, ctx->err);
  // The batch's lists, gathered on the device from the molecules' own lists in
  // (class, slot) order.
  b->h_segs.clear();
  for (size_t ci = 0; ci < nq; ++ci) {
    const int bc = dss_quartet_bra_class((int)ci), kc = dss_quartet_ket_class((int)ci);
    int at = 0;
    for (int sl = 0; sl < nb; ++sl) {
      const dss_batch_mol& m = b->mols[b->slot_mol[sl]];
      const int n = m.task_cnt[ci];
      if (!n) continue;
      TaskSeg sg;
      sg.src = b->task_pool.ptr + m.task_off + m.task_cls_off[ci];
      sg.dst = ctx->tasks[ci].d_tasks.ptr + at;
      sg.n = n;
      sg.dx = mc0[bc] + off[sl][bc] - lc0[sl][bc];
      sg.dy = mc0[kc] + off[sl][kc] - lc0[sl][kc];
      sg.slot = sl;
      b->h_segs.push_back(sg);
      at += n;
    }
  }
  if (!b->h_segs.empty()) {
    if (b->d_segs.resize(b->h_segs.size()) != cudaSuccess) return bfail(b, DSS_ERR_OOM, "batch: device tables");
    if (cudaMemcpyAsync(b->d_segs.ptr, b->h_segs.data(), b->h_segs.size() * sizeof(TaskSeg), cudaMemcpyHostToDevice,
                        ctx->stream) != cudaSuccess)
      return bfail(b, DSS_ERR_CUDA, "batch: device tables");
    const int nseg = (int)b->h_segs.size();
    k_gather_tasks<<<(unsigned)std::min(nseg, 8192), 256, 0, ctx->stream>>>(b->d_segs.ptr, nseg);
    if (cudaGetLastError() != cudaSuccess) return bfail(b, DSS_ERR_CUDA, "batch: task gather launch");
  }
  ctx->nbf = 1;  // batch mode: accumulators are addressed per molecule
  if (ctx->d_dmax.resize((size_t)std::max<long long>(dtot, 1)) != cudaSuccess)
    return bfail(b, DSS_ERR_OOM, "batch: device tables");
  auto up = [&](auto& buf, const auto& host) -> int {
    if (buf.resize(host.size()) != cudaSuccess) return DSS_ERR_OOM;
    if (cudaMemcpyAsync(buf.ptr, host.data(), host.size() * sizeof(host[0]), cudaMemcpyHostToDevice, ctx->stream) !=
        cudaSuccess)
      return DSS_ERR_CUDA;
    return DSS_OK;
  };
  if ((rc = up(ctx->d_sh_mbase, mbase)) || (rc = up(ctx->d_sh_jbase, jbase)) || (rc = up(ctx->d_sh_kbase, kbase)) ||
      (rc = up(ctx->d_sh_dbase, dbase)) || (rc = up(ctx->d_sh_n, shn)) || (rc = up(ctx->d_sh_mol, shmol)) ||
      (rc = up(ctx->d_sh_loc, shloc)) || (rc = up(ctx->d_sh_nsm, shnsm)) || (rc = up(b->d_region, region)) ||
      (rc = up(b->d_n, nv)))
    return bfail(b, rc, "batch: device tables");
  if (b->d_active.resize(nb) != cudaSuccess || b->d_active_next.resize(nb) != cudaSuccess ||
      b->d_nact.resize(2) != cudaSuccess)
    return bfail(b, DSS_ERR_OOM, "batch: device tables");
  b->dirty = false;
  return DSS_OK;
}

__global__ void k_active_from_hdr(BatchView v, int* active, int want_final) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= v.nb) return;
  int* ih = ihdr(v.arena + v.region[b]);
  active[b] = want_final ? (ih[I_DONE] && !ih[I_FINAL]) : !ih[I_DONE];
}

bool same_opts(const dss_scf_opts& a, const dss_scf_opts& c) {
  return a.conv == c.conv && a.max_iter == c.max_iter && a.incremental == c.incremental &&
         a.fp32_threshold == c.fp32_threshold && a.skip_threshold == c.skip_threshold &&
         a.rebuild_every == c.rebuild_every && a.final_switch == c.final_switch;
}

// Eigensolver, one block of 512 threads per molecule, in up to three launches
// by size: matrix and rotations in shared memory, matrix only, neither.
// Eigenvalues go to each molecule's eps slot, eigenvectors (columns) to kv.
void launch_jacobi(dss_batch* b, const BatchView& v, int ka, int kv, int kt, int max_sweeps) {
  cudaStream_t s = b->ctx->stream;
  const int nb = (int)b->slot_mol.size();
  // Shared-memory opt-in per device (the function attribute is per context);
  // batches on several host threads may both set it, which is harmless.
  static std::atomic<int> optin_dev[64] = {};
  int dev = 0;
  cudaGetDevice(&dev);
  int optin = 0;
  if (dev >= 0 && dev < 64 && optin_dev[dev].load()) {
    optin = optin_dev[dev].load();
  } else {
    cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    cudaFuncSetAttribute(k_jacobi<0>, cudaFuncAttributeMaxDynamicSharedMemorySize, optin);
    cudaFuncSetAttribute(k_jacobi<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, optin);
    if (dev >= 0 && dev < 64) optin_dev[dev].store(optin);
  }
  auto fits = [&](int nn_, bool vt) {
    return (dss_packed_size(nn_) + (vt ? (size_t)nn_ * nn_ : 0)) * 8 + dss_block_jacobi_smem(nn_) <= (size_t)optin;
  };
  int n1 = 0, n2 = 0;
  while (fits(n1 + 1, true)) ++n1;
  while (fits(n2 + 1, false)) ++n2;
  int top[3] = {0, 0, 0};
  for (int k = 0; k < nb; ++k) {
    const int nk = b->mols[b->slot_mol[k]].n;
    const int mode = nk <= n1 ? 0 : (nk <= n2 ? 1 : 2);
    top[mode] = std::max(top[mode], nk);
  }
  if (top[0])
    k_jacobi<0><<<nb, 512, (dss_packed_size(top[0]) + (size_t)top[0] * top[0]) * 8 + dss_block_jacobi_smem(top[0]),
                  s>>>(v, ka, kv, kt, max_sweeps, DSS_JACOBI_TOL, 0, n1);
  if (top[1])
    k_jacobi<1><<<nb, 512, dss_packed_size(top[1]) * 8 + dss_block_jacobi_smem(top[1]), s>>>(
        v, ka, kv, kt, max_sweeps, DSS_JACOBI_TOL, n1, n2);
  if (top[2])
    k_jacobi<2><<<nb, 512, dss_block_jacobi_smem(top[2]), s>>>(v, ka, kv, kt, max_sweeps, DSS_JACOBI_TOL, n2,
                                                               1 << 30);
}

// X = U s^-1/2 U^T (assignOrthogonalization, chem/scf/SCFBasis.cpp:85-100) for
// every molecule admitted since the last step, all in one batched eigensolve:
// admission stays cheap and a burst of new molecules shares the launches.
int prepare_x(dss_batch* b) {
  const int nb = (int)b->slot_mol.size();
  std::vector<int> pend(nb, 0);
  bool any = false;
  for (int k = 0; k < nb; ++k)
    if (b->mols[b->slot_mol[k]].needs_x) pend[k] = 1, any = true;
  if (!any) return DSS_OK;
  cudaStream_t s = b->ctx->stream;
  if (b->d_pending.resize(std::max(nb, 1)) != cudaSuccess) return DSS_ERR_OOM;
  if (cudaMemcpyAsync(b->d_pending.ptr, pend.data(), nb * sizeof(int), cudaMemcpyHostToDevice, s) != cudaSuccess)
    return DSS_ERR_CUDA;
  BatchView v = view(b, b->d_pending.ptr);
  const long long nn = (long long)b->nmax * b->nmax;
  const int tiles = (b->nmax + 31) / 32;
  const dim3 gg(tiles, tiles, nb), gb(32, 8);
  // Newton-Schulz (batched GEMMs, no per-molecule serial sweeps): M_T1 holds S
  // since admission; Y and Z alternate between (M_T2, M_T3) and (M_C, M_F),
  // P = Z Y and T in M_V.  32 iterations converge for cond(S) c / lambda_max up
  // to ~1e8; a molecule whose X S X is not I to 1e-11 afterwards sends the
  // new molecules to the eigen-decomposition X = U s^-1/2 U^T below.
  k_ns_init<<<dim3(1, nb), 256, 0, s>>>(v, M_T1, M_T2, M_T3);
  int y = M_T2, z = M_T3, y2 = M_C, z2 = M_F;
  for (int it = 0; it < 32; ++it) {
    k_gemm<<<gg, gb, 0, s>>>(v, z, y, M_V, 0, 0, 1.0, 0.0);
    k_ns_t<<<grid2(nn, nb), 256, 0, s>>>(v, M_V);
    k_gemm<<<gg, gb, 0, s>>>(v, y, M_V, y2, 0, 0, 1.0, 0.0);
    k_gemm<<<gg, gb, 0, s>>>(v, M_V, z, z2, 0, 0, 1.0, 0.0);
    std::swap(y, y2);
    std::swap(z, z2);
  }
  // The check is on X S X = Z S Z / c itself: S Z into the free buffer, then Z (S Z).
  k_gemm<<<gg, gb, 0, s>>>(v, M_T1, z, y2, 0, 0, 1.0, 0.0);
  k_gemm<<<gg, gb, 0, s>>>(v, z, y2, M_V, 0, 0, 1.0, 0.0);
  if (b->d_nsbad.resize(1) != cudaSuccess) return DSS_ERR_OOM;
  if (cudaMemsetAsync(b->d_nsbad.ptr, 0, sizeof(int), s) != cudaSuccess) return DSS_ERR_CUDA;
  k_ns_finish<<<grid2(nn, nb), 256, 0, s>>>(v, M_V, z, M_X, 1e-11, b->d_nsbad.ptr);
  int bad = 0;
  if (cudaMemcpyAsync(&bad, b->d_nsbad.ptr, sizeof(int), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
      cudaStreamSynchronize(s) != cudaSuccess)
    return DSS_ERR_CUDA;
  if (bad) {
    launch_jacobi(b, v, M_T1, M_V, M_T3, 60);
    k_scale_cols_eps<<<grid2(nn, nb), 256, 0, s>>>(v, M_V, M_T2);
    k_gemm<<<gg, gb, 0, s>>>(v, M_T2, M_V, M_X, 0, 1, 1.0, 0.0);
  }
  if (cudaStreamSynchronize(s) != cudaSuccess) return DSS_ERR_CUDA;  // pend is freed on return
  for (int k = 0; k < nb; ++k) b->mols[b->slot_mol[k]].needs_x = false;
  return DSS_OK;
}

// One SCF iteration for the active molecules (the captured body).  The
// incremental form (o.incremental) follows dss_scf_solve's: G = G_prev +
// G[2 dD] with the density-weighted screen (FP32 quartets below fp32_threshold,
// skipped below skip_threshold), full FP64 builds per molecule at the start,
// every rebuild_every iterations and in the final phase, accurate Boys function.
int enqueue_iteration(dss_batch* b, const dss_scf_opts& o) {
  dss_ctx* ctx = b->ctx;
  cudaStream_t s = ctx->stream;
  const int nb = (int)b->slot_mol.size();
  BatchView v = view(b, b->d_active.ptr);
  const long long nn = (long long)b->nmax * b->nmax;
  ctx->d_mol_active = b->d_active.ptr;
  BuildMode bm;
  bm.boys = ctx->opts.boys_mode;
  bm.no_zero = true;
  if (o.incremental) {
    k_mode<<<(nb + 127) / 128, 128, 0, s>>>(v, o.rebuild_every);
    k_prep_inc<<<grid2(nn, nb), 256, 0, s>>>(v);
    BlockMaxArgs ba;
    ba.sh_mol = ctx->d_sh_mol.ptr;
    ba.sh_loc = ctx->d_sh_loc.ptr;
    ba.sh_nsm = ctx->d_sh_nsm.ptr;
    ba.sh_f0 = ctx->d_sh_f0.ptr;
    ba.sh_nf = ctx->d_sh_nf.ptr;
    ba.sh_mbase = ctx->d_sh_mbase.ptr;
    ba.sh_dbase = ctx->d_sh_dbase.ptr;
    ba.dmax = ctx->d_dmax.ptr;
    ba.nshell = ctx->nshell;
    k_block_max<<<(unsigned)std::min(ctx->nshell, 4096), 64, 0, s>>>(v, ba);
    bm.boys = DSS_BOYS_FAST;
    bm.mixed = 1;
    bm.dmax = ctx->d_dmax.ptr;
    bm.fp32_thr = o.fp32_threshold;
    bm.skip_thr = o.skip_threshold;
  } else {
    k_prep<<<grid2(nn, nb), 256, 0, s>>>(v);
  }
  int rc = dss_enqueue_jk(ctx, b->arena.ptr, b->arena.ptr, b->arena.ptr, nullptr, &bm);
  if (rc != DSS_OK) return rc;
  if (o.incremental) {
    k_fock_inc<<<grid2(nn, nb), 256, 0, s>>>(v);
  } else {
    k_fock<<<grid2(nn, nb), 256, 0, s>>>(v);
  }
  const int tiles = (b->nmax + 31) / 32;
  const dim3 gg(tiles, tiles, nb), gb(32, 8);
  // DIIS error e = S D F_new - (S D F_new)^T
  k_gemm<<<gg, gb, 0, s>>>(v, M_D, M_FN, M_T1, 0, 0, 1.0, 0.0);
  k_gemm<<<gg, gb, 0, s>>>(v, M_S, M_T1, M_T2, 0, 0, 1.0, 0.0);
  k_diis_choose<<<(nb + 127) / 128, 128, 0, s>>>(v);
  k_diis_store<<<grid2(nn, nb), 256, 0, s>>>(v);
  k_diis_dots<<<dim3(grid2(nn, nb).x, nb, b->ds), 256, 0, s>>>(v);
  k_diis_solve<<<(nb + 127) / 128, 128, 0, s>>>(v);
  k_diis_combine<<<grid2(nn, nb), 256, 0, s>>>(v);
  // F' = X F X, rotated into the previous eigenvector basis: A = C'^T F' C'
  k_gemm<<<gg, gb, 0, s>>>(v, M_F, M_X, M_T1, 0, 0, 1.0, 0.0);
  k_gemm<<<gg, gb, 0, s>>>(v, M_X, M_T1, M_T2, 0, 0, 1.0, 0.0);
  k_gemm<<<gg, gb, 0, s>>>(v, M_T2, M_CP, M_T1, 0, 0, 1.0, 0.0);
  k_gemm<<<gg, gb, 0, s>>>(v, M_CP, M_T1, M_T2, 1, 0, 1.0, 0.0);
  launch_jacobi(b, v, M_T2, M_V, M_T3, 40);
  // C' <- C' V (through T1), C = X C', D = C_occ C_occ^T
  k_gemm<<<gg, gb, 0, s>>>(v, M_CP, M_V, M_T1, 0, 0, 1.0, 0.0);
  k_copy<<<grid2(nn, nb), 256, 0, s>>>(v, M_T1, M_CP);
  k_gemm<<<gg, gb, 0, s>>>(v, M_X, M_CP, M_C, 0, 0, 1.0, 0.0);
  k_density<<<grid2(nn, nb), 256, 0, s>>>(v);
  // E_elec = 2 sum eps_occ - tr(D G), G from the previous density
  k_trace<<<nb, 256, 0, s>>>(v, M_G, H_TRDG);
  if (cudaMemsetAsync(b->d_nact.ptr, 0, 2 * sizeof(int), s) != cudaSuccess) return DSS_ERR_CUDA;
  k_energy<<<(nb + 127) / 128, 128, 0, s>>>(v, o.conv, o.max_iter, o.incremental, o.final_switch,
                                            b->d_active_next.ptr, b->d_nact.ptr);
  if (cudaMemcpyAsync(b->d_active.ptr, b->d_active_next.ptr, nb * sizeof(int), cudaMemcpyDeviceToDevice, s) !=
      cudaSuccess)
    return DSS_ERR_CUDA;
  if (cudaGetLastError() != cudaSuccess) return DSS_ERR_CUDA;
  return DSS_OK;
}

// Final energies for molecules that finished but have no final energy yet.
int finalize(dss_batch* b) {
  dss_ctx* ctx = b->ctx;
  cudaStream_t s = ctx->stream;
  const int nb = (int)b->slot_mol.size();
  if (!nb) return DSS_OK;
  BatchView v0 = view(b, b->d_active.ptr);
  k_active_from_hdr<<<(nb + 127) / 128, 128, 0, s>>>(v0, b->d_active.ptr, 1);
  std::vector<int> fin(nb);
  if (cudaMemcpyAsync(fin.data(), b->d_active.ptr, nb * sizeof(int), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
      cudaStreamSynchronize(s) != cudaSuccess)
    return DSS_ERR_CUDA;
  for (int k = 0; k < nb; ++k)
    if (fin[k]) b->last_finished.push_back(b->slot_mol[k]);
  BatchView v = view(b, b->d_active.ptr);
  const long long nn = (long long)b->nmax * b->nmax;
  k_prep<<<grid2(nn, nb), 256, 0, s>>>(v);
  ctx->d_mol_active = b->d_active.ptr;
  BuildMode bm;
  bm.boys = b->inc ? DSS_BOYS_FAST : ctx->opts.boys_mode;  // FP64 build; the incremental form's Boys function
  bm.no_zero = true;
  int rc = dss_enqueue_jk(ctx, b->arena.ptr, b->arena.ptr, b->arena.ptr, nullptr, &bm);
  if (rc != DSS_OK) return rc;
  k_fock<<<grid2(nn, nb), 256, 0, s>>>(v);
  k_trace<<<nb, 256, 0, s>>>(v, M_H, H_TRDH);
  k_trace<<<nb, 256, 0, s>>>(v, M_G, H_TRDG);
  k_final<<<(nb + 127) / 128, 128, 0, s>>>(v);
  if (cudaGetLastError() != cudaSuccess) return DSS_ERR_CUDA;
  return DSS_OK;
}

}  // namespace

extern "C" {

int dss_batch_create(dss_batch** out, const dss_opts* opts, size_t arena_bytes, int diis_size) {
  if (!out) return DSS_ERR_INVALID;
  *out = nullptr;
  dss_batch* b = new (std::nothrow) dss_batch();
  if (!b) return DSS_ERR_OOM;
  int rc = dss_create(&b->ctx, opts);
  if (rc != DSS_OK) {
    delete b;
    return rc;
  }
  b->ds = (diis_size >= 1 && diis_size <= 9) ? diis_size : 8;
  if (!arena_bytes) {
    size_t fr = 0, tot = 0;
    cudaMemGetInfo(&fr, &tot);
    arena_bytes = fr / 4;
  }
  b->arena_doubles = arena_bytes / 8;
  if (b->arena.resize(b->arena_doubles) != cudaSuccess) {
    delete b;
    return DSS_ERR_OOM;
  }
  b->free_list.push_back({0, b->arena_doubles});
  if (cudaMallocHost((void**)&b->h_nact, 2 * sizeof(int)) != cudaSuccess) {
    delete b;
    return DSS_ERR_OOM;
  }
  *out = b;
  return DSS_OK;
}

void dss_batch_destroy(dss_batch* b) {
  if (!b) return;
  if (b->ctx) cudaStreamSynchronize(b->ctx->stream);
  delete b;
}

const char* dss_batch_last_error(const dss_batch* b) { return b ? b->err.c_str() : ""; }

}  // extern "C"

namespace {

__global__ void k_pack_d(const double* D, double* p, int n) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long long)n * n) return;
  const int r = (int)(t / n), c = (int)(t % n);
  if (r <= c) p[(long long)c * (c + 1) / 2 + r] = D[t];
}

int capture_graph(dss_batch* b, const dss_scf_opts& o) {
  cudaStream_t s = b->ctx->stream;
  if (b->graph) {
    cudaGraphExecDestroy(b->graph);
    b->graph = nullptr;
  }
  cudaGraph_t g = nullptr;
  if (cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal) != cudaSuccess)
    return bfail(b, DSS_ERR_CUDA, "batch: stream capture failed to start");
  const int rc = enqueue_iteration(b, o);
  const cudaError_t e = cudaStreamEndCapture(s, &g);
  if (rc != DSS_OK || e != cudaSuccess || !g) {
    if (g) cudaGraphDestroy(g);
    cudaGetLastError();
    return bfail(b, DSS_ERR_CUDA, std::string("batch: graph capture: ") + cudaGetErrorString(e));
  }
  const cudaError_t ie = cudaGraphInstantiate(&b->graph, g, 0);
  cudaGraphDestroy(g);
  if (ie != cudaSuccess) return bfail(b, DSS_ERR_CUDA, std::string("batch: graph instantiate: ") + cudaGetErrorString(ie));
  b->graph_opts = o;
  b->have_graph_opts = true;
  return DSS_OK;
}

}  // namespace

extern "C" {

int dss_batch_add(dss_batch* b, int n_shell, const int* l, const int* nprim, const double* exps, const double* coefs,
                  const double* centers, int pure, int natom, const int* Z, const double* xyz, int charge,
                  const double* D_guess, int* handle) {
  if (!b || !handle) return DSS_ERR_INVALID;
  b->err.clear();
  if (n_shell <= 0 || !l || !nprim || !exps || !coefs || !centers || natom <= 0 || !Z || !xyz)
    return bfail(b, DSS_ERR_INVALID, "dss_batch_add: empty molecule or NULL array");
  for (const auto& m : b->mols)
    if (m.live && m.basis.pure != (pure ? 1 : 0))
      return bfail(b, DSS_ERR_INVALID, "dss_batch_add: all molecules of a batch share the 5D/6D choice");
  dss_batch_mol m;
  std::string err;
  int rc = dss_make_basis(n_shell, l, nprim, exps, coefs, centers, pure, &m.basis, &err);
  if (rc != DSS_OK) return bfail(b, rc, err);
  int ne = -charge;
  for (int a = 0; a < natom; ++a) ne += Z[a];
  if (ne < 0 || ne % 2) return bfail(b, DSS_ERR_INVALID, "dss_batch_add: closed-shell RHF needs an even electron count");
  m.n = m.basis.nbf;
  m.nocc = ne / 2;
  m.natom = natom;
  if (m.nocc > m.n) return bfail(b, DSS_ERR_INVALID, "dss_batch_add: more occupied orbitals than functions");
  const size_t np = (size_t)m.n * (m.n + 1) / 2;
  const double e_nuc = dss_nuclear_repulsion(natom, Z, xyz);
  cudaSetDevice(b->ctx->opts.device);
  rc = dss_pairs_make(b->ctx, m.basis, &m.pairs, true);  // with its own work lists
  if (rc != DSS_OK) return bfail(b, rc, std::string("dss_batch_add: shell pairs: ") + b->ctx->err);
  rc = pool_put(b, &m);
  if (rc != DSS_OK) return bfail(b, rc, "dss_batch_add: primitive-pair pool allocation failed");
  rc = task_put(b, &m);
  if (rc != DSS_OK) return bfail(b, rc, "dss_batch_add: task pool allocation failed");
  m.size = region_size(m.n, b->ds);
  size_t off = 0;
  if (!arena_alloc(b, m.size, &off))
    return bfail(b, DSS_ERR_OOM, "dss_batch_add: not admitted, the batch arena has no room for this molecule");
  m.region = (long long)off;
  cudaStream_t s = b->ctx->stream;
  cudaSetDevice(b->ctx->opts.device);
  DevBuf<double>& tmp = b->admit_tmp;
  const int n = m.n;
  const size_t n2 = (size_t)n * n;
  if (tmp.resize(3 * np) != cudaSuccess) {
    arena_free(b, off, m.size);
    return bfail(b, DSS_ERR_OOM, "dss_batch_add: device allocation failed");
  }
  double* dH = tmp.ptr;
  double* dS = dH + np;
  double* dD = dS + np;
  // S and H = T + V straight into the scratch (device one-electron kernels).
  rc = dss_one_electron_device(s, m.basis, natom, Z, xyz, dS, dH, nullptr, &err, &b->ctx->oe_scratch);
  if (rc != DSS_OK) {
    arena_free(b, off, m.size);
    return bfail(b, rc, err);
  }
  if (D_guess) cudaMemcpyAsync(dD, D_guess, np * 8, cudaMemcpyHostToDevice, s);
  double* base = b->arena.ptr + off;
  k_admit_init<<<(unsigned)std::min<size_t>((n2 + 255) / 256, 1024), 256, 0, s>>>(base, n, dH, dS,
                                                                                  D_guess ? dD : nullptr, m.nocc,
                                                                                  e_nuc);
  // X is computed for all new molecules together at the next dss_batch_step.
  const cudaError_t e = cudaStreamSynchronize(s);  // the scratch is reused by the next admission
  if (e != cudaSuccess) {
    arena_free(b, off, m.size);
    return bfail(b, DSS_ERR_CUDA, std::string("dss_batch_add: ") + cudaGetErrorString(e));
  }
  m.live = true;
  b->mols.push_back(std::move(m));
  *handle = (int)b->mols.size() - 1;
  b->dirty = true;
  return DSS_OK;
}

int dss_batch_step(dss_batch* b, const dss_scf_opts* opts, int iterations, int* n_active) {
  if (!b) return DSS_ERR_INVALID;
  b->err.clear();
  dss_scf_opts o;
  dss_default_scf_opts(&o);
  if (opts) o = *opts;
  if (o.incremental && (o.rebuild_every < 1 || !(o.fp32_threshold >= 0.0) || !(o.skip_threshold >= 0.0)))
    return bfail(b, DSS_ERR_INVALID, "dss_batch_step: incremental form needs rebuild_every >= 1 and thresholds >= 0");
  cudaSetDevice(b->ctx->opts.device);
  cudaStream_t s = b->ctx->stream;
  bool fresh = false;
  if (b->dirty) {
    const int rc = rebuild(b);
    if (rc != DSS_OK) return rc;
    fresh = true;
  }
  const int nb = (int)b->slot_mol.size();
  if (n_active) *n_active = 0;
  if (!nb) return DSS_OK;
  {
    const int rc = prepare_x(b);
    if (rc != DSS_OK) return bfail(b, rc, "dss_batch_step: orthogonalisation of new molecules failed");
  }
  if (fresh) {
    BatchView v = view(b, b->d_active.ptr);
    k_active_from_hdr<<<(nb + 127) / 128, 128, 0, s>>>(v, b->d_active.ptr, 0);
  }
  if ((o.incremental != 0) != (b->inc != 0)) {
    // Switching forms: G_prev / D_prev may be stale, the next build is a full one.
    BatchView v = view(b, b->d_active.ptr);
    k_force_full<<<(nb + 127) / 128, 128, 0, s>>>(v);
  }
  b->inc = o.incremental != 0;
  int act = nb, newly_done = 0;
  b->last_finished.clear();
  for (int it = 0; it < iterations && act > 0; ++it) {
    const bool graph_ok = b->graph && b->have_graph_opts && same_opts(b->graph_opts, o);
    if (!graph_ok && !(b->eager_ran && b->have_graph_opts && same_opts(b->graph_opts, o))) {
      // First iteration after a change of composition or options runs eagerly
      // (it also sets kernel attributes); the graph is captured only when a
      // second iteration follows without a change, so a serving loop whose
      // composition changes every step does not pay for captures it never replays.
      if (b->graph) {
        cudaGraphExecDestroy(b->graph);
        b->graph = nullptr;
      }
      int rc = enqueue_iteration(b, o);
      if (rc != DSS_OK) return bfail(b, rc, "dss_batch_step: launch failed");
      b->graph_opts = o;
      b->have_graph_opts = true;
      b->eager_ran = true;
    } else {
      if (!graph_ok) {
        const int rc = capture_graph(b, o);
        if (rc != DSS_OK) return rc;
      }
      if (cudaGraphLaunch(b->graph, s) != cudaSuccess) return bfail(b, DSS_ERR_CUDA, "dss_batch_step: graph launch");
    }
    cudaMemcpyAsync(b->h_nact, b->d_nact.ptr, 2 * sizeof(int), cudaMemcpyDeviceToHost, s);
    const cudaError_t e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return bfail(b, DSS_ERR_CUDA, std::string("dss_batch_step: ") + cudaGetErrorString(e));
    act = b->h_nact[0];
    newly_done += b->h_nact[1];
  }
  if (newly_done > 0) {  // final energies only when some molecule finished
    const int rc = finalize(b);
    if (rc != DSS_OK) return bfail(b, rc, "dss_batch_step: final energies");
  }
  // Restore the iteration flags for the next step.
  BatchView v = view(b, b->d_active.ptr);
  k_active_from_hdr<<<(nb + 127) / 128, 128, 0, s>>>(v, b->d_active.ptr, 0);
  const cudaError_t e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return bfail(b, DSS_ERR_CUDA, std::string("dss_batch_step: ") + cudaGetErrorString(e));
  if (n_active) *n_active = act;
  return DSS_OK;
}

int dss_batch_solve(dss_batch* b, const dss_scf_opts* opts) {
  dss_scf_opts o;
  dss_default_scf_opts(&o);
  if (opts) o = *opts;
  int act = 0;
  return dss_batch_step(b, &o, o.max_iter + 1, &act);
}

int dss_batch_result(dss_batch* b, int handle, double* E_total, double* D_packed, int* iterations, int* status) {
  if (!b || handle < 0 || handle >= (int)b->mols.size() || !b->mols[handle].live) return DSS_ERR_INVALID;
  const dss_batch_mol& m = b->mols[handle];
  double hdr[kHdr];
  cudaStream_t s = b->ctx->stream;
  double* base = b->arena.ptr + m.region;
  if (cudaMemcpyAsync(hdr, base, sizeof(hdr), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
      cudaStreamSynchronize(s) != cudaSuccess)
    return bfail(b, DSS_ERR_CUDA, "dss_batch_result: copy");
  const int* ih = reinterpret_cast<const int*>(hdr + H_INT);
  if (!ih[I_FINAL]) return bfail(b, DSS_ERR_INVALID, "dss_batch_result: molecule not finished");
  if (E_total) *E_total = hdr[H_EFINAL];
  if (iterations) *iterations = ih[I_IT];
  if (status) *status = ih[I_STATUS];
  if (D_packed) {
    const int n = m.n;
    const size_t np = (size_t)n * (n + 1) / 2;
    DevBuf<double> tmp;
    if (tmp.resize(np) != cudaSuccess) return bfail(b, DSS_ERR_OOM, "dss_batch_result: allocation");
    k_pack_d<<<(unsigned)(((size_t)n * n + 255) / 256), 256, 0, s>>>(base + kHdr + (size_t)M_D * n * n, tmp.ptr, n);
    if (cudaMemcpyAsync(D_packed, tmp.ptr, np * 8, cudaMemcpyDeviceToHost, s) != cudaSuccess ||
        cudaStreamSynchronize(s) != cudaSuccess)
      return bfail(b, DSS_ERR_CUDA, "dss_batch_result: copy D");
  }
  return DSS_OK;
}

int dss_batch_remove(dss_batch* b, int handle) {
  if (!b || handle < 0 || handle >= (int)b->mols.size() || !b->mols[handle].live) return DSS_ERR_INVALID;
  cudaStreamSynchronize(b->ctx->stream);
  dss_batch_mol& m = b->mols[handle];
  arena_free(b, (size_t)m.region, m.size);
  m.live = false;
  m.basis = BasisHost();
  m.pairs = PairSet();
  b->dirty = true;
  return DSS_OK;
}

int dss_batch_info(const dss_batch* b, int* n_live, long long* free_bytes, long long* region_bytes_of_n) {
  if (!b) return DSS_ERR_INVALID;
  if (n_live) {
    int c = 0;
    for (const auto& m : b->mols) c += m.live ? 1 : 0;
    *n_live = c;
  }
  if (free_bytes) {
    size_t mx = 0;
    for (const auto& f : b->free_list) mx = std::max(mx, f.second);
    *free_bytes = (long long)mx * 8;
  }
  if (region_bytes_of_n && *region_bytes_of_n > 0) *region_bytes_of_n = (long long)region_size((int)*region_bytes_of_n, b->ds) * 8;
  return DSS_OK;
}

int dss_batch_set_class_variant(dss_batch* b, int i, int variant) {
  if (!b) return DSS_ERR_INVALID;
  const int rc = dss_set_class_variant(b->ctx, i, variant);
  if (rc == DSS_OK && b->graph) {
    cudaGraphExecDestroy(b->graph);
    b->graph = nullptr;
  }
  b->eager_ran = false;
  return rc;
}

int dss_batch_profile(dss_batch* b, float* ms) {
  if (!b || !ms) return DSS_ERR_INVALID;
  b->err.clear();
  const int ncls = dss_num_classes();
  for (int i = 0; i < ncls; ++i) ms[i] = 0.0f;
  cudaSetDevice(b->ctx->opts.device);
  if (b->dirty) {
    const int rc = rebuild(b);
    if (rc != DSS_OK) return rc;
  }
  const int nb = (int)b->slot_mol.size();
  if (!nb) return DSS_OK;
  dss_ctx* ctx = b->ctx;
  cudaStream_t s = ctx->stream;
  // Every live molecule takes part (J and K are scratch: the next iteration rebuilds them).
  DevBuf<int> all;
  if (all.resize(nb) != cudaSuccess) return bfail(b, DSS_ERR_OOM, "dss_batch_profile: allocation");
  std::vector<int> ones(nb, 1);
  cudaMemcpyAsync(all.ptr, ones.data(), nb * sizeof(int), cudaMemcpyHostToDevice, s);
  BatchView v = view(b, all.ptr);
  const long long nn = (long long)b->nmax * b->nmax;
  k_prep<<<grid2(nn, nb), 256, 0, s>>>(v);
  ctx->d_mol_active = all.ptr;
  const int nc = (int)ctx->tasks.size();
  std::vector<cudaEvent_t> ev(2 * nc);
  for (auto& e : ev) cudaEventCreate(&e);
  BuildMode bm;
  bm.boys = ctx->opts.boys_mode;
  bm.no_zero = true;
  int rc = dss_enqueue_jk(ctx, b->arena.ptr, b->arena.ptr, b->arena.ptr, ev.data(), &bm);
  const cudaError_t e = cudaStreamSynchronize(s);
  if (rc == DSS_OK && e == cudaSuccess)
    for (int i = 0; i < nc && i < ncls; ++i)
      if (ctx->tasks[i].ntasks) {
        cudaEventElapsedTime(&ms[i], ev[2 * i], ev[2 * i + 1]);
        dss_record_class_ms(ctx, i, ms[i]);
      }
  for (auto& x : ev) cudaEventDestroy(x);
  ctx->d_mol_active = b->d_active.ptr;
  if (rc != DSS_OK) return bfail(b, rc, "dss_batch_profile: launch failed");
  if (e != cudaSuccess) return bfail(b, DSS_ERR_CUDA, std::string("dss_batch_profile: ") + cudaGetErrorString(e));
  return DSS_OK;
}

int dss_batch_time_build(dss_batch* b, float* ms) {
  if (!b || !ms) return DSS_ERR_INVALID;
  b->err.clear();
  *ms = 0.0f;
  cudaSetDevice(b->ctx->opts.device);
  if (b->dirty) {
    const int rc = rebuild(b);
    if (rc != DSS_OK) return rc;
  }
  const int nb = (int)b->slot_mol.size();
  if (!nb) return DSS_OK;
  dss_ctx* ctx = b->ctx;
  cudaStream_t s = ctx->stream;
  DevBuf<int> all;
  if (all.resize(nb) != cudaSuccess) return bfail(b, DSS_ERR_OOM, "dss_batch_time_build: allocation");
  std::vector<int> ones(nb, 1);
  cudaMemcpyAsync(all.ptr, ones.data(), nb * sizeof(int), cudaMemcpyHostToDevice, s);
  BatchView v = view(b, all.ptr);
  const long long nn = (long long)b->nmax * b->nmax;
  k_prep<<<grid2(nn, nb), 256, 0, s>>>(v);
  ctx->d_mol_active = all.ptr;
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  BuildMode bm;
  bm.boys = ctx->opts.boys_mode;
  bm.no_zero = true;
  cudaEventRecord(e0, s);
  int rc = dss_enqueue_jk(ctx, b->arena.ptr, b->arena.ptr, b->arena.ptr, nullptr, &bm);
  cudaEventRecord(e1, s);
  const cudaError_t e = cudaStreamSynchronize(s);
  if (rc == DSS_OK && e == cudaSuccess) cudaEventElapsedTime(ms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  ctx->d_mol_active = b->d_active.ptr;
  if (rc != DSS_OK) return bfail(b, rc, "dss_batch_time_build: launch failed");
  if (e != cudaSuccess) return bfail(b, DSS_ERR_CUDA, std::string("dss_batch_time_build: ") + cudaGetErrorString(e));
  return DSS_OK;
}

int dss_batch_set_persistent(dss_batch* b, int on) {
  if (!b) return DSS_ERR_INVALID;
  const int rc = dss_set_persistent(b->ctx, on);
  if (rc == DSS_OK && b->graph) {
    cudaGraphExecDestroy(b->graph);
    b->graph = nullptr;
  }
  b->eager_ran = false;
  return rc;
}

int dss_batch_finished(const dss_batch* b, int* handles, int cap, int* count) {
  if (!b || !count || (cap > 0 && !handles)) return DSS_ERR_INVALID;
  const int n = (int)b->last_finished.size();
  for (int i = 0; i < n && i < cap; ++i) handles[i] = b->last_finished[i];
  *count = n;
  return DSS_OK;
}

void* dss_batch_context(dss_batch* b) { return b ? (void*)b->ctx : nullptr; }

}  // extern "C"
