// Dense FP64 kernels of the device SCF (see linalg.cuh).
#include <cooperative_groups.h>
#include <cuda_runtime.h>

#include <atomic>

#include "linalg.cuh"

namespace cg = cooperative_groups;

namespace {

constexpr int TS = 32;  // GEMM tile

__global__ void gemm_kernel(int n, bool ta, bool tb, double alpha, const double* __restrict__ A,
                            const double* __restrict__ B, double beta, double* __restrict__ C) {
  __shared__ double As[TS][TS + 1];
  __shared__ double Bs[TS][TS + 1];
  const int tx = threadIdx.x, ty = threadIdx.y;  // 32 x 8
  const int row0 = blockIdx.y * TS, col0 = blockIdx.x * TS;
  double acc[4] = {0.0, 0.0, 0.0, 0.0};
  for (int k0 = 0; k0 < n; k0 += TS) {
    for (int r = ty; r < TS; r += 8) {
      const int i = row0 + r, k = k0 + tx;
      // op(A)[i][k]
      double a = 0.0;
      if (i < n && k < n) a = ta ? A[(size_t)k * n + i] : A[(size_t)i * n + k];
      As[r][tx] = a;
      const int kk = k0 + r, j = col0 + tx;
      double b = 0.0;
      if (kk < n && j < n) b = tb ? B[(size_t)j * n + kk] : B[(size_t)kk * n + j];
      Bs[r][tx] = b;
    }
    __syncthreads();
#pragma unroll 8
    for (int k = 0; k < TS; ++k) {
      const double b = Bs[k][tx];
#pragma unroll
      for (int q = 0; q < 4; ++q) acc[q] += As[ty + 8 * q][k] * b;
    }
    __syncthreads();
  }
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    const int i = row0 + ty + 8 * q, j = col0 + tx;
    if (i < n && j < n) {
      const size_t o = (size_t)i * n + j;
      C[o] = alpha * acc[q] + (beta == 0.0 ? 0.0 : beta * C[o]);
    }
  }
}

__global__ void __launch_bounds__(256) jacobi_kernel(int n, int m, double* A0, double* A1, double* V0, double* V1,
                                                     double* w, double* scratch, int* rank, int max_sweeps,
                                                     double tol) {
  cg::grid_group grid = cg::this_grid();
  extern __shared__ double rot[];  // [m/2] c, [m/2] s
  const int half = m / 2;
  double* cs_c = rot;
  double* cs_s = rot + half;
  const long long gtid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long gsz = (long long)gridDim.x * blockDim.x;
  double* A = A0;
  double* An = A1;
  double* Vc = V0;
  double* Vn = V1;
  __shared__ double red[2][8];
  double off_prev = 0.0;
  for (int sweep = 0; sweep <= max_sweeps; ++sweep) {
    // Off-diagonal and total Frobenius norms (slots alternate between sweeps).
    double* slot = scratch + 2 * (sweep & 1);
    double off = 0.0, dia = 0.0;
    for (long long t = gtid; t < (long long)n * n; t += gsz) {
      const int i = (int)(t / n), j = (int)(t % n);
      const double v = A[t];
      if (i == j) dia += v * v;
      else off += v * v;
    }
    for (int o = 16; o > 0; o >>= 1) {
      off += __shfl_xor_sync(0xffffffffu, off, o);
      dia += __shfl_xor_sync(0xffffffffu, dia, o);
    }
    if ((threadIdx.x & 31) == 0) {
      red[0][threadIdx.x >> 5] = off;
      red[1][threadIdx.x >> 5] = dia;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      double o = 0.0, d = 0.0;
      for (int k = 0; k < (int)(blockDim.x >> 5); ++k) {
        o += red[0][k];
        d += red[1][k];
      }
      atomicAdd(slot, o);
      atomicAdd(slot + 1, d);
    }
    // Clear the other slot for the next sweep.
    if (gtid == 0) {
      double* other = scratch + 2 * ((sweep + 1) & 1);
      other[0] = 0.0;
      other[1] = 0.0;
    }
    grid.sync();
    const double offv = slot[0], tot = slot[0] + slot[1];
    if (gtid == 0) scratch[4] = (double)sweep;
    if (dss_jacobi_done(offv, tot, off_prev, sweep, max_sweeps, tol)) break;
    off_prev = offv;
    for (int r = 0; r < m - 1; ++r) {
      for (int k = threadIdx.x; k < half; k += blockDim.x) {
        int p, q;
        dss_rr_pair(m, r, k, p, q);
        double c = 1.0, s = 0.0;
        if (q < n) {
          const double apq = A[(size_t)p * n + q];
          if (fabs(apq) > 1e-300) {
            const double app = A[(size_t)p * n + p], aqq = A[(size_t)q * n + q];
            const double tau = (aqq - app) / (2.0 * apq);
            const double t = (tau >= 0.0 ? 1.0 : -1.0) / (fabs(tau) + sqrt(1.0 + tau * tau));
            c = 1.0 / sqrt(1.0 + t * t);
            s = t * c;
          }
        }
        cs_c[k] = c;
        cs_s[k] = s;
      }
      __syncthreads();
      // A' = R^T A R on 2x2 blocks (pair k1 rows, pair k2 columns).
      for (long long t = gtid; t < (long long)half * half; t += gsz) {
        const int k1 = (int)(t / half), k2 = (int)(t % half);
        int p1, q1, p2, q2;
        dss_rr_pair(m, r, k1, p1, q1);
        dss_rr_pair(m, r, k2, p2, q2);
        const double c1 = cs_c[k1], s1 = cs_s[k1], c2 = cs_c[k2], s2 = cs_s[k2];
        const bool q1v = q1 < n, q2v = q2 < n;
        const double b00 = A[(size_t)p1 * n + p2];
        const double b01 = q2v ? A[(size_t)p1 * n + q2] : 0.0;
        const double b10 = q1v ? A[(size_t)q1 * n + p2] : 0.0;
        const double b11 = (q1v && q2v) ? A[(size_t)q1 * n + q2] : 0.0;
        // X = R1^T B
        const double x00 = c1 * b00 - s1 * b10, x01 = c1 * b01 - s1 * b11;
        const double x10 = s1 * b00 + c1 * b10, x11 = s1 * b01 + c1 * b11;
        // X R2
        An[(size_t)p1 * n + p2] = x00 * c2 - x01 * s2;
        if (q2v) An[(size_t)p1 * n + q2] = x00 * s2 + x01 * c2;
        if (q1v) An[(size_t)q1 * n + p2] = x10 * c2 - x11 * s2;
        if (q1v && q2v) An[(size_t)q1 * n + q2] = x10 * s2 + x11 * c2;
      }
      // V' = V R
      for (long long t = gtid; t < (long long)n * half; t += gsz) {
        const int i = (int)(t / half), k = (int)(t % half);
        int p, q;
        dss_rr_pair(m, r, k, p, q);
        const double c = cs_c[k], s = cs_s[k];
        const double vp = Vc[(size_t)i * n + p];
        if (q < n) {
          const double vq = Vc[(size_t)i * n + q];
          Vn[(size_t)i * n + p] = c * vp - s * vq;
          Vn[(size_t)i * n + q] = s * vp + c * vq;
        } else {
          Vn[(size_t)i * n + p] = vp;
        }
      }
      grid.sync();
      double* tA = A;
      A = An;
      An = tA;
      double* tV = Vc;
      Vc = Vn;
      Vn = tV;
    }
  }
  // Eigenvalues in ascending order (ties by index), vectors permuted alike.
  for (long long t = gtid; t < n; t += gsz) {
    const int i = (int)t;
    const double wi = A[(size_t)i * n + i];
    int r = 0;
    for (int j = 0; j < n; ++j) {
      const double wj = A[(size_t)j * n + j];
      if (wj < wi || (wj == wi && j < i)) ++r;
    }
    rank[i] = r;
    w[r] = wi;
  }
  grid.sync();
  for (long long t = gtid; t < (long long)n * n; t += gsz) {
    const int i = (int)(t / n), j = (int)(t % n);
    Vn[(size_t)i * n + rank[j]] = Vc[t];
  }
  grid.sync();
  if (Vn != V0)
    for (long long t = gtid; t < (long long)n * n; t += gsz) V0[t] = Vn[t];
}

// One thread block for a matrix that fits in shared memory as a packed upper
// triangle (no grid-wide synchronisation between the rounds); VT_SMEM: the
// rotations in shared memory too, else in VTg.
template <bool VT_SMEM>
__global__ void __launch_bounds__(512) jacobi_block_kernel(int n, const double* A0, double* V, double* w, double* VTg,
                                                            int max_sweeps, double tol, int v_init) {
  extern __shared__ double sm[];
  const size_t nn = (size_t)n * n, np = dss_packed_size(n);
  DssPackedSym A{sm, n};
  double* VT = VT_SMEM ? sm + np : VTg;
  void* aux = sm + np + (VT_SMEM ? nn : 0);
  const int tid = threadIdx.x, nt = blockDim.x;
  for (int i = tid >> 5; i < n; i += nt >> 5)
    for (int j = i + (tid & 31); j < n; j += 32) A.at(i, j) = A0[(size_t)i * n + j];
  for (int t = tid; t < (int)nn; t += nt) {
    const int i = t / n, j = t % n;
    VT[t] = v_init ? V[(size_t)j * n + i] : (i == j ? 1.0 : 0.0);
  }
  __syncthreads();
  dss_block_jacobi(A, VT, aux, max_sweeps, tol);
  __syncthreads();
  dss_block_jacobi_sorted(A, VT, w, V);
}

__global__ void set_identity(int n, double* V) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t < (long long)n * n) V[t] = (t / n == t % n) ? 1.0 : 0.0;
}

}  // namespace

void dss_gemm(cudaStream_t s, int n, bool ta, bool tb, double alpha, const double* A, const double* B, double beta,
              double* C) {
  dim3 block(32, 8);
  dim3 grid((n + TS - 1) / TS, (n + TS - 1) / TS);
  gemm_kernel<<<grid, block, 0, s>>>(n, ta, tb, alpha, A, B, beta, C);
}

cudaError_t dss_jacobi_eigh(cudaStream_t s, int n, double* A, double* V, double* w, double* work, int max_sweeps,
                            double tol, bool v_init) {
  int dev = 0;
  cudaGetDevice(&dev);
  // Per device: the shared-memory opt-in and the kernels' attribute (set per
  // context).  Contexts on several host threads may both set it, which is harmless.
  static std::atomic<int> optin_cache[64] = {};
  int optin = 0;
  if (dev >= 0 && dev < 64) {
    optin = optin_cache[dev].load();
    if (!optin) {
      cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
      cudaFuncSetAttribute(jacobi_block_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, optin);
      cudaFuncSetAttribute(jacobi_block_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, optin);
      optin_cache[dev].store(optin);
    }
  }
  const size_t one = dss_packed_size(n) * 8 + dss_block_jacobi_smem(n), two = one + (size_t)n * n * 8;
  if (two <= (size_t)optin) {
    // Small matrices: one block, matrix and rotations in shared memory.
    jacobi_block_kernel<true><<<1, 512, two, s>>>(n, A, V, w, work, max_sweeps, tol, v_init ? 1 : 0);
    return cudaGetLastError();
  }
  if (one <= (size_t)optin) {
    // Medium: the matrix in shared memory, the rotations in work.
    jacobi_block_kernel<false><<<1, 512, one, s>>>(n, A, V, w, work, max_sweeps, tol, v_init ? 1 : 0);
    return cudaGetLastError();
  }
  const int m = (n % 2) ? n + 1 : n;
  double* A1 = work;
  double* V1 = work + (size_t)n * n;
  double* scratch = work + 2 * (size_t)n * n;
  int* rank = reinterpret_cast<int*>(scratch + 64);
  if (!v_init) {
    set_identity<<<(unsigned)(((long long)n * n + 255) / 256), 256, 0, s>>>(n, V);
  }
  cudaError_t e = cudaMemsetAsync(scratch, 0, 8 * sizeof(double), s);
  if (e != cudaSuccess) return e;
  int nsm = 0;
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  const int threads = 256;
  const size_t shmem = (size_t)m * sizeof(double);
  int per_sm = 0;
  e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, jacobi_kernel, threads, shmem);
  if (e != cudaSuccess) return e;
  if (per_sm < 1) return cudaErrorInvalidConfiguration;
  long long need = ((long long)(m / 2) * (m / 2) + threads - 1) / threads;
  int blocks = nsm * (per_sm < 2 ? per_sm : 2);
  if (need < blocks) blocks = (int)(need > 0 ? need : 1);
  void* args[] = {(void*)&n, (void*)&m, (void*)&A, (void*)&A1, (void*)&V, (void*)&V1, (void*)&w, (void*)&scratch,
                  (void*)&rank, (void*)&max_sweeps, (void*)&tol};
  return cudaLaunchCooperativeKernel((void*)jacobi_kernel, blocks, threads, args, shmem, s);
}
