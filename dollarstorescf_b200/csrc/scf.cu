// Device RHF SCF: the reference's solveMOs loop (chem/scf/SCFSolver.cpp:196-237)
// with every matrix step on the GPU.
//
// Per iteration (runSCFIteration, SCFSolver.cpp:145-172):
//   G = J[2 D] - K[2 D] / 2                 (computeCoulombTerms/ExchangeTerms :29-43)
//   F_new = H + G                            (updateFockMatrix :45-62)
//   iteration 1: F = F_new; later: Pulay DIIS (SCFDIIS.cpp:19-52, lalib/DIIS.ipp):
//     e = S D F_new - (S D F_new)^T, B_ii = |e|^2, B_ij = <e_i, e_j>, bordered by
//     ones; ring of diis_size entries, when full the entry with the largest B_ii
//     is replaced; F = sum_i c_i F_i from B c = (0,..,0,1).
//   F' = X F X, X = S^-1/2 (Loewdin, SCFBasis.cpp:85-100); F' C' = C' eps
//   (cyclic Jacobi on the device, warm-started from the previous C'); C = X C'
//   D = C_occ C_occ^T                        (computeDensityMatrix :77-94)
//   E_elec = 2 sum_occ eps - tr(D G)         (getTotalElectronicEnergy :118-130)
//   converged when |E_elec - E_prev| < conv  (checkConvergence :174-177)
// Final energy from the final density (calculateEnergies, Energy.cpp:21-50):
//   E = 2 tr(D H) + tr(D G[D]) + E_nuc.
// Unlike the reference the loop has an iteration cap (DSS_ERR_NOCONV), and a
// singular DIIS system falls back to the newest Fock matrix instead of the
// reference's behaviour (LAPACK reports the error, the coefficients stay the
// right-hand side and F becomes 0, lalib/Lapack.cpp:164-169).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <string>
#include <vector>

#include "dss.h"
#include "dss_internal.h"
#include "linalg.cuh"

namespace {

__global__ void unpack_sym(const double* __restrict__ p, double* __restrict__ d, int n) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long long)n * n) return;
  const int r = (int)(t / n), c = (int)(t % n);
  const int x = r > c ? r : c, y = r > c ? c : r;
  d[t] = p[(long long)x * (x + 1) / 2 + y];
}

__global__ void pack_sym(const double* __restrict__ d, double* __restrict__ p, int n) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long long)n * n) return;
  const int r = (int)(t / n), c = (int)(t % n);
  if (r <= c) p[(long long)c * (c + 1) / 2 + r] = d[t];
}

// out = a*X + b*Y (+ c*Z if Z)
__global__ void axpby(long long N, double a, const double* X, double b, const double* Y, double c, const double* Z,
                      double* out) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= N) return;
  double v = a * X[t] + b * Y[t];
  if (Z) v += c * Z[t];
  out[t] = v;
}

// e = T - T^T
__global__ void antisym(const double* __restrict__ T, double* __restrict__ e, int n) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long long)n * n) return;
  const int r = (int)(t / n), c = (int)(t % n);
  e[t] = T[t] - T[(long long)c * n + r];
}

// X = U diag(s^-1/2) U^T helper: scale columns of U by f(s).
__global__ void scale_cols(const double* __restrict__ U, const double* __restrict__ s, double* __restrict__ out,
                           int n, int power_neg_half) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long long)n * n) return;
  const int c = (int)(t % n);
  const double v = power_neg_half ? 1.0 / sqrt(s[c]) : sqrt(s[c]);
  out[t] = U[t] * v;
}

// D = C[:, :nocc] C[:, :nocc]^T
__global__ void density_kernel(const double* __restrict__ C, double* __restrict__ D, int n, int nocc) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long long)n * n) return;
  const int r = (int)(t / n), c = (int)(t % n);
  double v = 0.0;
  for (int k = 0; k < nocc; ++k) v += C[(size_t)r * n + k] * C[(size_t)c * n + k];
  D[t] = v;
}

// Block sums of x*y (and optional second pair) into out[] via atomics.
__global__ void dot_kernel(long long N, const double* __restrict__ x, const double* __restrict__ y, double* out) {
  double acc = 0.0;
  for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < N; t += (long long)gridDim.x * blockDim.x)
    acc += x[t] * y[t];
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
  __shared__ double red[32];
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    double s = 0.0;
    for (int k = 0; k < (int)(blockDim.x >> 5); ++k) s += red[k];
    atomicAdd(out, s);
  }
}

// DIIS slot choice (lalib/DIIS.ipp:19-62): state[0] = count, state[1] = slot.
__global__ void diis_choose(int* state, const double* B, int size, int ld) {
  int count = state[0];
  int slot = 0;
  if (count < size) {
    slot = count;
    count += 1;
  } else {
    double mx = 0.0;
    for (int i = 0; i < size; ++i) {
      const double e = B[i * ld + i];
      if (e > mx) {
        mx = e;
        slot = i;
      }
    }
  }
  state[0] = count;
  state[1] = slot;
}

// B row/column of the new slot from the dot products, then the bordered solve
// B c = (0,..,0,1) by Gaussian elimination with partial pivoting.
__global__ void diis_solve(int* state, double* B, int ld, const double* dots, double* coef) {
  const int count = state[0], slot = state[1];
  for (int i = 0; i < count; ++i) {
    B[slot * ld + i] = dots[i];
    B[i * ld + slot] = dots[i];
  }
  const int m = count + 1;
  double M[10][11];
  for (int i = 0; i < m; ++i) {
    for (int j = 0; j < m; ++j) {
      double v;
      if (i < count && j < count) v = B[i * ld + j];
      else if (i == count && j == count) v = 0.0;
      else v = 1.0;
      M[i][j] = v;
    }
    M[i][m] = (i == count) ? 1.0 : 0.0;
  }
  bool singular = false;
  for (int k = 0; k < m && !singular; ++k) {
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
    for (int i = m - 1; i >= 0; --i) {
      double v = M[i][m];
      for (int j = i + 1; j < m; ++j) v -= M[i][j] * coef[j];
      coef[i] = v / M[i][i];
    }
  }
  for (int i = 0; i < count; ++i) {
    if (singular) coef[i] = (i == slot) ? 1.0 : 0.0;
  }
  state[2] = singular ? 1 : 0;
}

// F = sum_i coef[i] F_i
__global__ void diis_combine(int n2, const double* __restrict__ Fring, const double* __restrict__ coef,
                             const int* __restrict__ state, double* __restrict__ F) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n2) return;
  const int count = state[0];
  double v = 0.0;
  for (int i = 0; i < count; ++i) v += coef[i] * Fring[(size_t)i * n2 + t];
  F[t] = v;
}

__global__ void copy_slot(int n2, const double* __restrict__ src, double* __restrict__ ring, const int* state) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n2) return;
  ring[(size_t)state[1] * n2 + t] = src[t];
}

// dots[i] = <e_i, e_new> for the ring entries (i < count), after the new entry is stored.
__global__ void ring_dots(int n2, const double* __restrict__ ering, const int* __restrict__ state,
                          double* __restrict__ dots) {
  const int i = blockIdx.y;
  if (i >= state[0]) return;
  const double* a = ering + (size_t)i * n2;
  const double* b = ering + (size_t)state[1] * n2;
  double acc = 0.0;
  for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < n2; t += (long long)gridDim.x * blockDim.x)
    acc += a[t] * b[t];
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
  __shared__ double red[32];
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    double s = 0.0;
    for (int k = 0; k < (int)(blockDim.x >> 5); ++k) s += red[k];
    atomicAdd(dots + i, s);
  }
}

// E_elec = 2 sum_{i<nocc} eps_i - tr(D G)  ->  out[0]; tr(D G) comes in trDG.
__global__ void energy_kernel(const double* eps, int nocc, const double* trDG, double* out) {
  double s = 0.0;
  for (int i = 0; i < nocc; ++i) s += 2.0 * eps[i];
  out[0] = s - trDG[0];
}

inline unsigned nb(long long N, int t = 256) { return (unsigned)((N + t - 1) / t); }

// UHF two-electron parts from the J/K accumulators of the two spin densities:
// G_a = J[D_a + D_b] - K[D_a], G_b = J[D_a + D_b] - K[D_b], with
// J = Ja + Ja^T + Jb + Jb^T and K_s = Ks + Ks^T.  Also J itself (for the energy).
__global__ void uhf_combine(const double* __restrict__ Ja, const double* __restrict__ Ka,
                            const double* __restrict__ Jb, const double* __restrict__ Kb, double* __restrict__ Ga,
                            double* __restrict__ Gb, double* __restrict__ Jt, int n) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long long)n * n) return;
  const int r = (int)(t / n), c = (int)(t % n);
  const long long u = (long long)c * n + r;
  const double J = Ja[t] + Ja[u] + Jb[t] + Jb[u];
  Ga[t] = J - (Ka[t] + Ka[u]);
  Gb[t] = J - (Kb[t] + Kb[u]);
  if (Jt) Jt[t] = J;
}

// The same from one unrestricted build: J accumulated from D_a + D_b, one
// exchange accumulator per spin.
__global__ void uhf_combine_one(const double* __restrict__ Jacc, const double* __restrict__ Ka,
                                const double* __restrict__ Kb, double* __restrict__ Ga, double* __restrict__ Gb,
                                double* __restrict__ Jt, int n) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long long)n * n) return;
  const int r = (int)(t / n), c = (int)(t % n);
  const long long u = (long long)c * n + r;
  const double J = Jacc[t] + Jacc[u];
  Ga[t] = J - (Ka[t] + Ka[u]);
  Gb[t] = J - (Kb[t] + Kb[u]);
  if (Jt) Jt[t] = J;
}

// E_elec = sum_{i<na} eps_a_i + sum_{i<nb} eps_b_i - (tr(Da Ga) + tr(Db Gb)) / 2
// (getTotalElectronicEnergy, unrestricted branch, SCFSolver.cpp:131-142).
__global__ void uhf_energy_kernel(const double* eps_a, int na, const double* eps_b, int nbeta, const double* tr,
                                  double* out) {
  double s = 0.0;
  for (int i = 0; i < na; ++i) s += eps_a[i];
  for (int i = 0; i < nbeta; ++i) s += eps_b[i];
  out[0] = s - 0.5 * tr[0] - 0.5 * tr[1];
}



}  // namespace

extern "C" {

void dss_default_scf_opts(dss_scf_opts* o) {
  if (!o) return;
  o->conv = 1e-8;  // scf::energy_threshold, chem/scf/SCFSolver.cpp:26
  o->diis_size = 8;  // diis::setIterationCount(8), SCFSolver.cpp:214
  o->max_iter = 128;
  o->use_guess = 0;
  o->incremental = 0;
  o->fp32_threshold = 1e-7;
  o->skip_threshold = 1e-12;
  // Measured on the 256-alkane batch and (H2O)32 6-31G*: rebuilding every 16
  // iterations and switching to full builds at |dE| < 1e-8 is the fastest of
  // final_switch 1e-5..1e-9 x rebuild_every 8/16, with the same energies.
  o->rebuild_every = 16;
  o->final_switch = 1e-8;
}

int dss_scf_solve(dss_ctx* ctx, const double* Hp, const double* Sp, int n_alpha, double e_nuc,
                  const dss_scf_opts* opts_in, double* E_total, double* Dp, int* iterations) {
  if (!ctx) return DSS_ERR_INVALID;
  ctx->err.clear();
  if (!ctx->nbf) return dss_fail(ctx, DSS_ERR_INVALID, "dss_scf_solve: no basis set");
  if (!Hp || !Sp || !E_total) return dss_fail(ctx, DSS_ERR_INVALID, "dss_scf_solve: NULL argument");
  const int n = ctx->nbf;
  if (n_alpha < 0 || n_alpha > n) return dss_fail(ctx, DSS_ERR_INVALID, "dss_scf_solve: occupied count out of range");
  dss_scf_opts o;
  dss_default_scf_opts(&o);
  if (opts_in) o = *opts_in;
  if (o.diis_size < 1 || o.diis_size > 9)
    return dss_fail(ctx, DSS_ERR_INVALID, "dss_scf_solve: diis_size must be 1..9");
  if (o.use_guess && !Dp) return dss_fail(ctx, DSS_ERR_INVALID, "dss_scf_solve: use_guess needs D");
  if (cudaSetDevice(ctx->opts.device) != cudaSuccess) return dss_fail(ctx, DSS_ERR_CUDA, "dss_scf_solve: cudaSetDevice");
  const size_t n2 = (size_t)n * n, np = (size_t)n * (n + 1) / 2;
  cudaStream_t s = ctx->stream;
  // Device buffers (kept in the context so repeated solves reuse them).
  ScfBuffers& b = ctx->scf;
  const int ds = o.diis_size;
  const size_t need = n2 * (16 + 2 * (size_t)ds) + 3 * n2 + 8 * (size_t)n + 256;
  if (b.pool.resize(need) != cudaSuccess || b.ibuf.resize(8 + 2 * (size_t)n) != cudaSuccess)
    return dss_fail(ctx, DSS_ERR_OOM, "dss_scf_solve: device allocation failed");
  double* base = b.pool.ptr;
  double *H = base, *S = H + n2, *X = S + n2, *D = X + n2, *Dt = D + n2, *J = Dt + n2, *K = J + n2, *G = K + n2,
         *F = G + n2, *Fn = F + n2, *T1 = Fn + n2, *T2 = T1 + n2, *Cp = T2 + n2, *C = Cp + n2;
  double* Gprev = C + n2;  // incremental form: G and D of the previous build
  double* Dprev = Gprev + n2;
  double* Fring = Dprev + n2;
  double* Ering = Fring + (size_t)ds * n2;
  double* work = Ering + (size_t)ds * n2;           // 3 n^2 + 64 + n ints
  double* eps = work + 3 * n2 + 64 + (size_t)n;    // n
  double* small = eps + n;                           // scalars: [0]=E, [1]=trDG, [2..11] dots, [16..35] coef
  double* Bm = small + 64;                           // 10 x 10
  int* state = b.ibuf.ptr;
  auto fail_cuda = [&](cudaError_t e, const char* what) {
    return dss_fail(ctx, DSS_ERR_CUDA, std::string("dss_scf_solve: ") + what + ": " + cudaGetErrorString(e));
  };
  cudaError_t e;
#define SCF_CHECK(call, what)                      \
  do {                                             \
    e = (call);                                    \
    if (e != cudaSuccess) return fail_cuda(e, what); \
  } while (0)
  // Inputs.
  DevBuf<double> packed;
  SCF_CHECK(packed.resize(np), "alloc");
  SCF_CHECK(cudaMemcpyAsync(packed.ptr, Hp, np * 8, cudaMemcpyHostToDevice, s), "H2D H");
  unpack_sym<<<nb(n2), 256, 0, s>>>(packed.ptr, H, n);
  SCF_CHECK(cudaMemcpyAsync(packed.ptr, Sp, np * 8, cudaMemcpyHostToDevice, s), "H2D S");
  unpack_sym<<<nb(n2), 256, 0, s>>>(packed.ptr, S, n);
  // X = U s^-1/2 U^T from the eigen-decomposition of S (assignOrthogonalization).
  SCF_CHECK(cudaMemcpyAsync(T1, S, n2 * 8, cudaMemcpyDeviceToDevice, s), "copy S");
  SCF_CHECK(dss_jacobi_eigh(s, n, T1, T2, eps, work, 60, DSS_JACOBI_TOL, false), "eigh(S)");
  scale_cols<<<nb(n2), 256, 0, s>>>(T2, eps, T1, n, 1);
  dss_gemm(s, n, false, true, 1.0, T1, T2, 0.0, X);
  // Initial density.
  if (o.use_guess) {
    SCF_CHECK(cudaMemcpyAsync(packed.ptr, Dp, np * 8, cudaMemcpyHostToDevice, s), "H2D D");
    unpack_sym<<<nb(n2), 256, 0, s>>>(packed.ptr, D, n);
  } else {
    SCF_CHECK(cudaMemsetAsync(D, 0, n2 * 8, s), "zero D");  // useCoreGuess, SCFSolver.cpp:179-194
  }
  SCF_CHECK(cudaMemsetAsync(state, 0, 8 * sizeof(int), s), "zero state");
  SCF_CHECK(cudaMemsetAsync(Bm, 0, 100 * 8, s), "zero B");
  bool have_cp = false;
  double E = 0.0, E_prev = 0.0;
  int it = 0;
  int rc = DSS_OK;
  // Full builds: the plain form always; the incremental form at the start, every
  // rebuild_every iterations and throughout the final phase.
  BuildMode full_mode;
  full_mode.boys = o.incremental ? DSS_BOYS_FAST : ctx->opts.boys_mode;
  int last_full = -1000, full_streak = 0;
  bool final_phase = !o.incremental;
  if (o.incremental) {
    if (ctx->d_dmax.resize((size_t)ctx->nshell * ctx->nshell) != cudaSuccess)
      return dss_fail(ctx, DSS_ERR_OOM, "dss_scf_solve: device allocation failed");
  }
  while (true) {
    if (it && std::fabs(E - E_prev) < o.conv && full_streak >= (o.incremental ? 2 : 0)) break;
    if (o.incremental && it && std::fabs(E - E_prev) < o.final_switch) final_phase = true;
    if (it >= o.max_iter) {
      rc = dss_fail(ctx, DSS_ERR_NOCONV, "dss_scf_solve: no convergence within max_iter iterations");
      break;
    }
    ++it;
    const bool full = !o.incremental || final_phase || it <= 2 || it - last_full >= o.rebuild_every;
    if (full) {
      // G = J[2D] - K[2D]/2
      axpby<<<nb(n2), 256, 0, s>>>((long long)n2, 2.0, D, 0.0, D, 0.0, nullptr, Dt);
      int r2 = dss_enqueue_jk(ctx, Dt, J, K, nullptr, &full_mode);
      if (r2 != DSS_OK) return r2;
      // J, K hold the accumulators: G = (J + J^T) - (K + K^T)/2
      dss_symmetrize_combine(s, n, J, K, G);
      last_full = it;
      ++full_streak;
    } else {
      // G = G_prev + G[2 (D - D_prev)] with the screened mixed-precision kernels.
      axpby<<<nb(n2), 256, 0, s>>>((long long)n2, 2.0, D, -2.0, Dprev, 0.0, nullptr, Dt);
      dss_block_max(ctx, Dt, ctx->d_dmax.ptr);
      BuildMode mm;
      mm.boys = DSS_BOYS_FAST;
      mm.mixed = 1;
      mm.dmax = ctx->d_dmax.ptr;
      mm.fp32_thr = o.fp32_threshold;
      mm.skip_thr = o.skip_threshold;
      int r2 = dss_enqueue_jk(ctx, Dt, J, K, nullptr, &mm);
      if (r2 != DSS_OK) return r2;
      dss_symmetrize_combine(s, n, J, K, T1);
      axpby<<<nb(n2), 256, 0, s>>>((long long)n2, 1.0, Gprev, 1.0, T1, 0.0, nullptr, G);
      full_streak = 0;
    }
    if (o.incremental) {
      SCF_CHECK(cudaMemcpyAsync(Gprev, G, n2 * 8, cudaMemcpyDeviceToDevice, s), "copy G");
      SCF_CHECK(cudaMemcpyAsync(Dprev, D, n2 * 8, cudaMemcpyDeviceToDevice, s), "copy D");
    }
    axpby<<<nb(n2), 256, 0, s>>>((long long)n2, 1.0, H, 1.0, G, 0.0, nullptr, Fn);
    if (it == 1) {
      SCF_CHECK(cudaMemcpyAsync(F, Fn, n2 * 8, cudaMemcpyDeviceToDevice, s), "copy F");
    } else {
      // e = S D F_new - (S D F_new)^T
      dss_gemm(s, n, false, false, 1.0, D, Fn, 0.0, T1);
      dss_gemm(s, n, false, false, 1.0, S, T1, 0.0, T2);
      diis_choose<<<1, 1, 0, s>>>(state, Bm, ds, 10);
      antisym<<<nb(n2), 256, 0, s>>>(T2, T1, n);
      copy_slot<<<nb(n2), 256, 0, s>>>((int)n2, T1, Ering, state);
      copy_slot<<<nb(n2), 256, 0, s>>>((int)n2, Fn, Fring, state);
      SCF_CHECK(cudaMemsetAsync(small + 2, 0, 10 * 8, s), "zero dots");
      ring_dots<<<dim3(64, ds), 256, 0, s>>>((int)n2, Ering, state, small + 2);
      diis_solve<<<1, 1, 0, s>>>(state, Bm, 10, small + 2, small + 16);
      diis_combine<<<nb(n2), 256, 0, s>>>((int)n2, Fring, small + 16, state, F);
    }
    // F' = X F X, eigen-decomposition (warm start from the previous C').
    dss_gemm(s, n, false, false, 1.0, F, X, 0.0, T1);
    dss_gemm(s, n, false, false, 1.0, X, T1, 0.0, T2);  // T2 = F'
    if (have_cp) {
      dss_gemm(s, n, false, false, 1.0, T2, Cp, 0.0, T1);
      dss_gemm(s, n, true, false, 1.0, Cp, T1, 0.0, T2);  // Cp^T F' Cp
      SCF_CHECK(dss_jacobi_eigh(s, n, T2, T1, eps, work, 40, DSS_JACOBI_TOL, false), "eigh(F')");
      dss_gemm(s, n, false, false, 1.0, Cp, T1, 0.0, T2);
      SCF_CHECK(cudaMemcpyAsync(Cp, T2, n2 * 8, cudaMemcpyDeviceToDevice, s), "copy C'");
    } else {
      SCF_CHECK(dss_jacobi_eigh(s, n, T2, Cp, eps, work, 60, DSS_JACOBI_TOL, false), "eigh(F')");
      have_cp = true;
    }
    dss_gemm(s, n, false, false, 1.0, X, Cp, 0.0, C);
    density_kernel<<<nb(n2), 256, 0, s>>>(C, D, n, n_alpha);
    // E_elec = 2 sum eps_occ - tr(D G), G from the previous density.
    SCF_CHECK(cudaMemsetAsync(small + 1, 0, 8, s), "zero tr");
    dot_kernel<<<64, 256, 0, s>>>((long long)n2, D, G, small + 1);
    energy_kernel<<<1, 1, 0, s>>>(eps, n_alpha, small + 1, small);
    SCF_CHECK(cudaGetLastError(), "launch");
    double Eh = 0.0;
    SCF_CHECK(cudaMemcpyAsync(&Eh, small, 8, cudaMemcpyDeviceToHost, s), "D2H E");
    SCF_CHECK(cudaStreamSynchronize(s), "sync");
    E_prev = E;
    E = Eh;
    if (!std::isfinite(E)) {
      rc = dss_fail(ctx, DSS_ERR_NOCONV, "dss_scf_solve: energy is not finite");
      break;
    }
  }
  // Final energy from the final density (calculateEnergies), FP64.
  axpby<<<nb(n2), 256, 0, s>>>((long long)n2, 2.0, D, 0.0, D, 0.0, nullptr, Dt);
  int r3 = dss_enqueue_jk(ctx, Dt, J, K, nullptr, &full_mode);
  if (r3 != DSS_OK) return r3;
  dss_symmetrize_combine(s, n, J, K, G);
  SCF_CHECK(cudaMemsetAsync(small + 1, 0, 16, s), "zero tr");
  dot_kernel<<<64, 256, 0, s>>>((long long)n2, D, H, small + 1);
  dot_kernel<<<64, 256, 0, s>>>((long long)n2, D, G, small + 2);
  double tr[2];
  SCF_CHECK(cudaMemcpyAsync(tr, small + 1, 16, cudaMemcpyDeviceToHost, s), "D2H tr");
  if (Dp) {
    pack_sym<<<nb(n2), 256, 0, s>>>(D, packed.ptr, n);
    SCF_CHECK(cudaMemcpyAsync(Dp, packed.ptr, np * 8, cudaMemcpyDeviceToHost, s), "D2H D");
  }
  // The final orbitals, for dss_scf_orbitals / dss_write_molden.
  ctx->last_C[0].resize(n2);
  ctx->last_eps[0].resize(n);
  SCF_CHECK(cudaMemcpyAsync(ctx->last_C[0].data(), C, n2 * 8, cudaMemcpyDeviceToHost, s), "D2H C");
  SCF_CHECK(cudaMemcpyAsync(ctx->last_eps[0].data(), eps, (size_t)n * 8, cudaMemcpyDeviceToHost, s), "D2H eps");
  SCF_CHECK(cudaStreamSynchronize(s), "sync");
  ctx->last_nocc[0] = n_alpha;
  ctx->last_nocc[1] = 0;
  ctx->last_spins = 1;
  *E_total = 2.0 * tr[0] + tr[1] + e_nuc;
  if (iterations) *iterations = it;
#undef SCF_CHECK
  return rc;
}


int dss_uhf_solve(dss_ctx* ctx, const double* Hp, const double* Sp, int n_alpha, int n_beta, double e_nuc,
                  const dss_scf_opts* opts_in, double* E_total, double* Dap, double* Dbp, int* iterations) {
  if (!ctx) return DSS_ERR_INVALID;
  ctx->err.clear();
  if (!ctx->nbf || ctx->nmol > 0) return dss_fail(ctx, DSS_ERR_INVALID, "dss_uhf_solve: no single-molecule basis set");
  if (!Hp || !Sp || !E_total) return dss_fail(ctx, DSS_ERR_INVALID, "dss_uhf_solve: NULL argument");
  const int n = ctx->nbf;
  if (n_alpha < 0 || n_alpha > n || n_beta < 0 || n_beta > n)
    return dss_fail(ctx, DSS_ERR_INVALID, "dss_uhf_solve: occupied count out of range");
  dss_scf_opts o;
  dss_default_scf_opts(&o);
  if (opts_in) o = *opts_in;
  if (o.diis_size < 1 || o.diis_size > 9)
    return dss_fail(ctx, DSS_ERR_INVALID, "dss_uhf_solve: diis_size must be 1..9");
  if (o.incremental) return dss_fail(ctx, DSS_ERR_UNSUPPORTED, "dss_uhf_solve: the incremental form is RHF only");
  if (o.use_guess && (!Dap || !Dbp)) return dss_fail(ctx, DSS_ERR_INVALID, "dss_uhf_solve: use_guess needs both D");
  if (cudaSetDevice(ctx->opts.device) != cudaSuccess) return dss_fail(ctx, DSS_ERR_CUDA, "dss_uhf_solve: cudaSetDevice");
  const size_t n2 = (size_t)n * n, np = (size_t)n * (n + 1) / 2;
  cudaStream_t s = ctx->stream;
  ScfBuffers& b = ctx->scf;
  const int ds = o.diis_size;
  const size_t need = n2 * (20 + 4 * (size_t)ds) + 3 * n2 + 16 * (size_t)n + 512;
  if (b.pool.resize(need) != cudaSuccess || b.ibuf.resize(16 + 2 * (size_t)n) != cudaSuccess)
    return dss_fail(ctx, DSS_ERR_OOM, "dss_uhf_solve: device allocation failed");
  double* base = b.pool.ptr;
  double *H = base, *S = H + n2, *X = S + n2, *Jt = X + n2, *T1 = Jt + n2, *T2 = T1 + n2, *Fn = T2 + n2;
  double* Jacc[2] = {Fn + n2, Fn + 2 * n2};
  double* Kacc[2] = {Fn + 3 * n2, Fn + 4 * n2};
  double* D[2] = {Fn + 5 * n2, Fn + 6 * n2};
  double* G[2] = {Fn + 7 * n2, Fn + 8 * n2};
  double* F[2] = {Fn + 9 * n2, Fn + 10 * n2};
  double* Cp[2] = {Fn + 11 * n2, Fn + 12 * n2};
  double* C = Fn + 13 * n2;
  double* Fring[2] = {C + n2, C + n2 + (size_t)ds * n2};
  double* Ering[2] = {C + n2 + 2 * (size_t)ds * n2, C + n2 + 3 * (size_t)ds * n2};
  double* work = C + n2 + 4 * (size_t)ds * n2;  // 3 n^2 + 64 + n ints
  double* eps[2] = {work + 3 * n2 + 64 + (size_t)n, work + 3 * n2 + 64 + 2 * (size_t)n};
  double* small = eps[1] + n;  // [0] E, [1..2] traces, [2..11]/[16..35] per-spin dots/coef below
  double* dots[2] = {small + 64, small + 80};
  double* coef[2] = {small + 96, small + 112};
  double* Bm[2] = {small + 128, small + 228};
  int* state[2] = {b.ibuf.ptr, b.ibuf.ptr + 8};
  const int nocc[2] = {n_alpha, n_beta};
  auto fail_cuda = [&](cudaError_t e, const char* what) {
    return dss_fail(ctx, DSS_ERR_CUDA, std::string("dss_uhf_solve: ") + what + ": " + cudaGetErrorString(e));
  };
  cudaError_t e;
#define UHF_CHECK(call, what)                        \
  do {                                               \
    e = (call);                                      \
    if (e != cudaSuccess) return fail_cuda(e, what); \
  } while (0)
  DevBuf<double> packed;
  UHF_CHECK(packed.resize(np), "alloc");
  UHF_CHECK(cudaMemcpyAsync(packed.ptr, Hp, np * 8, cudaMemcpyHostToDevice, s), "H2D H");
  unpack_sym<<<nb(n2), 256, 0, s>>>(packed.ptr, H, n);
  UHF_CHECK(cudaMemcpyAsync(packed.ptr, Sp, np * 8, cudaMemcpyHostToDevice, s), "H2D S");
  unpack_sym<<<nb(n2), 256, 0, s>>>(packed.ptr, S, n);
  // X = U s^-1/2 U^T (assignOrthogonalization).
  UHF_CHECK(cudaMemcpyAsync(T1, S, n2 * 8, cudaMemcpyDeviceToDevice, s), "copy S");
  UHF_CHECK(dss_jacobi_eigh(s, n, T1, T2, eps[0], work, 60, DSS_JACOBI_TOL, false), "eigh(S)");
  scale_cols<<<nb(n2), 256, 0, s>>>(T2, eps[0], T1, n, 1);
  dss_gemm(s, n, false, true, 1.0, T1, T2, 0.0, X);
  for (int sp = 0; sp < 2; ++sp) {
    if (o.use_guess) {
      UHF_CHECK(cudaMemcpyAsync(packed.ptr, sp ? Dbp : Dap, np * 8, cudaMemcpyHostToDevice, s), "H2D D");
      unpack_sym<<<nb(n2), 256, 0, s>>>(packed.ptr, D[sp], n);
    } else {
      UHF_CHECK(cudaMemsetAsync(D[sp], 0, n2 * 8, s), "zero D");  // useCoreGuess, SCFSolver.cpp:179-194
    }
    UHF_CHECK(cudaMemsetAsync(Bm[sp], 0, 100 * 8, s), "zero B");
  }
  UHF_CHECK(cudaMemsetAsync(b.ibuf.ptr, 0, 16 * sizeof(int), s), "zero state");
  BuildMode mode;
  mode.boys = ctx->opts.boys_mode;
  // J of the total density and K of each spin density, combined into G_a, G_b
  // (and J).  With the reference Boys function one unrestricted build evaluates
  // every integral once for both exchange matrices; otherwise one build per spin.
  auto two_electron = [&]() -> int {
    if (mode.boys == DSS_BOYS_REF) {
      axpby<<<nb(n2), 256, 0, s>>>((long long)n2, 1.0, D[0], 1.0, D[1], 0.0, nullptr, T1);  // D_a + D_b
      BuildMode um = mode;
      um.uhf = true;
      um.Da = D[0];
      um.Db = D[1];
      um.K2 = Kacc[1];
      int r = dss_enqueue_jk(ctx, T1, Jacc[0], Kacc[0], nullptr, &um);
      if (r != DSS_OK) return r;
      uhf_combine_one<<<nb(n2), 256, 0, s>>>(Jacc[0], Kacc[0], Kacc[1], G[0], G[1], Jt, n);
      return DSS_OK;
    }
    for (int sp = 0; sp < 2; ++sp) {
      int r = dss_enqueue_jk(ctx, D[sp], Jacc[sp], Kacc[sp], nullptr, &mode);
      if (r != DSS_OK) return r;
    }
    uhf_combine<<<nb(n2), 256, 0, s>>>(Jacc[0], Kacc[0], Jacc[1], Kacc[1], G[0], G[1], Jt, n);
    return DSS_OK;
  };
  bool have_cp[2] = {false, false};
  double E = 0.0, E_prev = 0.0;
  int it = 0;
  int rc = DSS_OK;
  while (true) {
    if (it && std::fabs(E - E_prev) < o.conv) break;
    if (it >= o.max_iter) {
      rc = dss_fail(ctx, DSS_ERR_NOCONV, "dss_uhf_solve: no convergence within max_iter iterations");
      break;
    }
    ++it;
    int r2 = two_electron();
    if (r2 != DSS_OK) return r2;
    for (int sp = 0; sp < 2; ++sp) {
      // F_new = H + G_s; DIIS per spin (solvers[spin], SCFDIIS.cpp:14-52).
      axpby<<<nb(n2), 256, 0, s>>>((long long)n2, 1.0, H, 1.0, G[sp], 0.0, nullptr, Fn);
      if (it == 1) {
        UHF_CHECK(cudaMemcpyAsync(F[sp], Fn, n2 * 8, cudaMemcpyDeviceToDevice, s), "copy F");
      } else {
        dss_gemm(s, n, false, false, 1.0, D[sp], Fn, 0.0, T1);
        dss_gemm(s, n, false, false, 1.0, S, T1, 0.0, T2);
        diis_choose<<<1, 1, 0, s>>>(state[sp], Bm[sp], ds, 10);
        antisym<<<nb(n2), 256, 0, s>>>(T2, T1, n);
        copy_slot<<<nb(n2), 256, 0, s>>>((int)n2, T1, Ering[sp], state[sp]);
        copy_slot<<<nb(n2), 256, 0, s>>>((int)n2, Fn, Fring[sp], state[sp]);
        UHF_CHECK(cudaMemsetAsync(dots[sp], 0, 10 * 8, s), "zero dots");
        ring_dots<<<dim3(64, ds), 256, 0, s>>>((int)n2, Ering[sp], state[sp], dots[sp]);
        diis_solve<<<1, 1, 0, s>>>(state[sp], Bm[sp], 10, dots[sp], coef[sp]);
        diis_combine<<<nb(n2), 256, 0, s>>>((int)n2, Fring[sp], coef[sp], state[sp], F[sp]);
      }
    }
    for (int sp = 0; sp < 2; ++sp) {
      // F' = X F X, eigen-decomposition (warm start from the previous C'), C = X C'.
      dss_gemm(s, n, false, false, 1.0, F[sp], X, 0.0, T1);
      dss_gemm(s, n, false, false, 1.0, X, T1, 0.0, T2);
      if (have_cp[sp]) {
        dss_gemm(s, n, false, false, 1.0, T2, Cp[sp], 0.0, T1);
        dss_gemm(s, n, true, false, 1.0, Cp[sp], T1, 0.0, T2);
        UHF_CHECK(dss_jacobi_eigh(s, n, T2, T1, eps[sp], work, 40, DSS_JACOBI_TOL, false), "eigh(F')");
        dss_gemm(s, n, false, false, 1.0, Cp[sp], T1, 0.0, T2);
        UHF_CHECK(cudaMemcpyAsync(Cp[sp], T2, n2 * 8, cudaMemcpyDeviceToDevice, s), "copy C'");
      } else {
        UHF_CHECK(dss_jacobi_eigh(s, n, T2, Cp[sp], eps[sp], work, 60, DSS_JACOBI_TOL, false), "eigh(F')");
        have_cp[sp] = true;
      }
      dss_gemm(s, n, false, false, 1.0, X, Cp[sp], 0.0, C);
      density_kernel<<<nb(n2), 256, 0, s>>>(C, D[sp], n, nocc[sp]);
    }
    UHF_CHECK(cudaMemsetAsync(small + 1, 0, 16, s), "zero tr");
    dot_kernel<<<64, 256, 0, s>>>((long long)n2, D[0], G[0], small + 1);
    dot_kernel<<<64, 256, 0, s>>>((long long)n2, D[1], G[1], small + 2);
    uhf_energy_kernel<<<1, 1, 0, s>>>(eps[0], n_alpha, eps[1], n_beta, small + 1, small);
    UHF_CHECK(cudaGetLastError(), "launch");
    double Eh = 0.0;
    UHF_CHECK(cudaMemcpyAsync(&Eh, small, 8, cudaMemcpyDeviceToHost, s), "D2H E");
    UHF_CHECK(cudaStreamSynchronize(s), "sync");
    E_prev = E;
    E = Eh;
    if (!std::isfinite(E)) {
      rc = dss_fail(ctx, DSS_ERR_NOCONV, "dss_uhf_solve: energy is not finite");
      break;
    }
  }
  // Final energy from the final densities (calculateEnergies, Energy.cpp:21-50):
  // tr(Dt H) + tr(Dt J)/2 - (tr(Da Ka) + tr(Db Kb))/2 + E_nuc, Dt = Da + Db.
  int r3 = two_electron();
  if (r3 != DSS_OK) return r3;
  axpby<<<nb(n2), 256, 0, s>>>((long long)n2, 1.0, D[0], 1.0, D[1], 0.0, nullptr, T1);  // Dt
  UHF_CHECK(cudaMemsetAsync(small + 1, 0, 40, s), "zero tr");
  dot_kernel<<<64, 256, 0, s>>>((long long)n2, T1, H, small + 1);
  dot_kernel<<<64, 256, 0, s>>>((long long)n2, T1, Jt, small + 2);
  dot_kernel<<<64, 256, 0, s>>>((long long)n2, D[0], G[0], small + 3);  // tr(Da (J - Ka))
  dot_kernel<<<64, 256, 0, s>>>((long long)n2, D[1], G[1], small + 4);
  double tr[4];
  UHF_CHECK(cudaMemcpyAsync(tr, small + 1, 32, cudaMemcpyDeviceToHost, s), "D2H tr");
  for (int sp = 0; sp < 2; ++sp) {
    double* out = sp ? Dbp : Dap;
    if (!out) continue;
    pack_sym<<<nb(n2), 256, 0, s>>>(D[sp], packed.ptr, n);
    UHF_CHECK(cudaMemcpyAsync(out, packed.ptr, np * 8, cudaMemcpyDeviceToHost, s), "D2H D");
    UHF_CHECK(cudaStreamSynchronize(s), "sync");
  }
  for (int sp = 0; sp < 2; ++sp) {  // the final orbitals, for dss_scf_orbitals / dss_write_molden
    dss_gemm(s, n, false, false, 1.0, X, Cp[sp], 0.0, C);
    ctx->last_C[sp].resize(n2);
    ctx->last_eps[sp].resize(n);
    UHF_CHECK(cudaMemcpyAsync(ctx->last_C[sp].data(), C, n2 * 8, cudaMemcpyDeviceToHost, s), "D2H C");
    UHF_CHECK(cudaMemcpyAsync(ctx->last_eps[sp].data(), eps[sp], (size_t)n * 8, cudaMemcpyDeviceToHost, s),
              "D2H eps");
    UHF_CHECK(cudaStreamSynchronize(s), "sync");
  }
  ctx->last_nocc[0] = n_alpha;
  ctx->last_nocc[1] = n_beta;
  ctx->last_spins = 2;
  UHF_CHECK(cudaStreamSynchronize(s), "sync");
  // tr(Ds Gs) = tr(Ds J) - tr(Ds Ks); summed over the spins: tr(Dt J) - sum tr(Ds Ks).
  const double exch = tr[1] - (tr[2] + tr[3]);  // sum_s tr(Ds Ks)
  *E_total = tr[0] + 0.5 * tr[1] - 0.5 * exch + e_nuc;
  if (iterations) *iterations = it;
#undef UHF_CHECK
  return rc;
}

}  // extern "C"
