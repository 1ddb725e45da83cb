// Dense FP64 building blocks of the device SCF: a tiled GEMM, the parallel
// cyclic Jacobi eigensolver, and small helpers.  All matrices are row-major
// n x n in device memory.
#pragma once
#include <cuda_runtime.h>

// Jacobi stops when the off-diagonal Frobenius norm is below this fraction of
// the whole, or at the rounding floor (dss_jacobi_done).
#define DSS_JACOBI_TOL 1e-14

// C = alpha * op(A) * op(B) + beta * C, op = transpose when the flag is set.
void dss_gemm(cudaStream_t s, int n, bool ta, bool tb, double alpha, const double* A, const double* B, double beta,
              double* C);

// Symmetric eigensolver (cyclic Jacobi, round-robin parallel ordering): one
// thread block with the matrix in shared memory when it fits, else one
// cooperative launch over the GPU: on return w[n] holds the eigenvalues in ascending order
// and V (n x n, row-major) the eigenvectors as columns.  A is overwritten.
// work must hold 3 n^2 + 4 n + 64 doubles.  Returns cudaSuccess or the launch
// error; *sweeps receives the sweep count when non-NULL (device pointer ok: NULL).
cudaError_t dss_jacobi_eigh(cudaStream_t s, int n, double* A, double* V, double* w, double* work, int max_sweeps,
                            double tol, bool v_init);

// Round-robin (circle method) pairing of m (even) indices: round r, slot k -> (p < q).
__device__ __forceinline__ void dss_rr_pair(int m, int r, int k, int& p, int& q) {
  if (k == 0) {
    p = m - 1;
    q = r;
  } else {
    p = (r + k) % (m - 1);
    q = (r - k + (m - 1)) % (m - 1);
  }
  if (p > q) {
    const int t = p;
    p = q;
    q = t;
  }
}

// Stopping rule of the Jacobi sweeps, from the squared off-diagonal and total
// Frobenius norms at the start of a sweep: off <= tol^2 total, or the rounding
// floor is reached -- off is already below 1e-24 total (relative 1e-12) and the
// last sweep did not cut it by 4x, where a sweep above the floor cuts it
// quadratically.  The floor grows like sqrt(n) eps max|lambda| / rms(lambda), so
// for large n or a wide spectrum it lies above tol = 1e-14 and the first test
// alone would run every sweep up to max_sweeps.
__host__ __device__ __forceinline__ bool dss_jacobi_done(double off, double tot, double off_prev, int sweep,
                                                         int max_sweeps, double tol) {
  if (off <= tol * tol * tot || sweep >= max_sweeps) return true;
  return sweep >= 2 && off <= 1e-24 * tot && off > 0.25 * off_prev;
}

// Shared memory (bytes) dss_block_jacobi needs besides the matrix.
__host__ __device__ constexpr size_t dss_block_jacobi_smem(int n) {
  return (size_t)((n + 1) / 2) * 2 * (sizeof(int) + sizeof(double)) + 64 * sizeof(double) + 16;
}
// Doubles of a packed upper triangle.
__host__ __device__ constexpr size_t dss_packed_size(int n) { return (size_t)n * (n + 1) / 2; }

// Symmetric matrix views for dss_block_jacobi.  DssPackedSym: upper triangle
// packed by rows (shared memory; element (i, j) and (j, i) are one word, so a
// rotation writes each element once).  DssDenseSym: full row-major n x n (global
// memory; every 2x2 block is updated, rows stay contiguous for coalescing).
struct DssPackedSym {
  double* a;
  int n;
  static constexpr bool kPacked = true;
  __device__ __forceinline__ int row(int i) const { return i * n - (i * (i - 1)) / 2; }
  __device__ __forceinline__ double& at(int i, int j) const {
    const int lo = i < j ? i : j, hi = i < j ? j : i;
    return a[row(lo) + (hi - lo)];
  }
};
struct DssDenseSym {
  double* a;
  int n;
  static constexpr bool kPacked = false;
  __device__ __forceinline__ double& at(int i, int j) const { return a[(size_t)i * n + j]; }
};

// Cyclic Jacobi run by one thread block (blockDim.x a multiple of 32): the
// symmetric matrix A is rotated to diagonal form in sweeps of m - 1 rounds of
// m/2 disjoint rotations (m = n rounded up to even; round-robin order).  The
// rotations accumulate into VT (n x n row-major, shared or global memory), whose
// row j ends as the eigenvector belonging to A's diagonal entry j.  Each round
// stores its pairs and (c, s) in shared memory (sh, dss_block_jacobi_smem(n)
// bytes), then updates the 2x2 blocks of A (packed: the blocks at or above the
// block diagonal, each element once; dense: all blocks, rows contiguous) and
// rotates rows p, q of VT with the loads of two pairs and up to eight elements
// per lane issued before their stores, so a global VT exposes one memory latency
// per two pairs (n <= 256).  Stops when the off-diagonal Frobenius norm is at most tol times the
// whole, or after max_sweeps sweeps; returns the sweeps run.
template <class M>
static __device__ __noinline__ int dss_block_jacobi(M A, double* VT, void* sh, int max_sweeps, double tol) {
  const int n = A.n;
  const int m = (n & 1) ? n + 1 : n, half = m / 2;
  double* C = reinterpret_cast<double*>(sh);
  double* S = C + half;
  double* red = S + half;  // 64
  int* P = reinterpret_cast<int*>(red + 64);
  int* Q = P + half;
  const int tid = threadIdx.x, nt = blockDim.x, lane = tid & 31, warp = tid >> 5, nw = nt >> 5;
  int sweep = 0;
  double so_prev = 0.0;
  for (;; ++sweep) {
    double off = 0.0, dia = 0.0;
    for (int i = warp; i < n; i += nw)
      for (int j = (M::kPacked ? i : 0) + lane; j < n; j += 32) {
        const double x = A.at(i, j);
        if (i == j) dia += x * x;
        else off += (M::kPacked ? 2.0 : 1.0) * x * x;
      }
    for (int o = 16; o > 0; o >>= 1) {
      off += __shfl_xor_sync(0xffffffffu, off, o);
      dia += __shfl_xor_sync(0xffffffffu, dia, o);
    }
    if (lane == 0) {
      red[warp] = off;
      red[32 + warp] = dia;
    }
    __syncthreads();
    double so = 0.0, sd = 0.0;
    for (int k = 0; k < nw; ++k) {
      so += red[k];
      sd += red[32 + k];
    }
    __syncthreads();
    if (dss_jacobi_done(so, so + sd, so_prev, sweep, max_sweeps, tol)) break;
    so_prev = so;
    for (int r = 0; r < m - 1; ++r) {
      for (int k = tid; k < half; k += nt) {
        int p, q;
        dss_rr_pair(m, r, k, p, q);
        double c = 1.0, s = 0.0;
        if (q < n) {
          const double apq = A.at(p, q);
          if (fabs(apq) > 1e-300) {
            // t = tan of the rotation angle, the smaller root of t^2 + 2 tau t - 1 = 0,
            // tau = (a_qq - a_pp) / (2 a_pq): t = sgn(d) 2 a_pq / (|d| + sqrt(d^2 + 4 a_pq^2)).
            const double d = A.at(q, q) - A.at(p, p);
            const double t = (d >= 0.0 ? 2.0 : -2.0) * apq / (fabs(d) + sqrt(d * d + 4.0 * apq * apq));
            c = rsqrt(1.0 + t * t);
            s = t * c;
          }
        }
        P[k] = p;
        Q[k] = q;
        C[k] = c;
        S[k] = s;
      }
      __syncthreads();
      // A <- R^T A R, R = [[c, s], [-s, c]] on every pair (p, q).
      for (int k1 = warp; k1 < half; k1 += nw) {
        const int p1 = P[k1], q1 = Q[k1];
        const double c1 = C[k1], s1 = S[k1];
        const bool q1v = q1 < n;
        for (int k2 = (M::kPacked ? k1 : 0) + lane; k2 < half; k2 += 32) {
          const int p2 = P[k2], q2 = Q[k2];
          const double c2 = C[k2], s2 = S[k2];
          const bool q2v = q2 < n;
          const bool diag = k2 == k1;
          const double b00 = A.at(p1, p2);
          const double b01 = q2v ? A.at(p1, q2) : 0.0;
          const double b10 = q1v ? A.at(q1, p2) : 0.0;
          const double b11 = (q1v && q2v) ? A.at(q1, q2) : 0.0;
          const double x00 = c1 * b00 - s1 * b10, x01 = c1 * b01 - s1 * b11;
          const double x10 = s1 * b00 + c1 * b10, x11 = s1 * b01 + c1 * b11;
          const double y00 = x00 * c2 - x01 * s2, y01 = x00 * s2 + x01 * c2;
          const double y10 = x10 * c2 - x11 * s2, y11 = x10 * s2 + x11 * c2;
          A.at(p1, p2) = y00;
          if (q2v) A.at(p1, q2) = y01;
          // Packed: on a diagonal block (q1, p2) is the word just written.
          if (q1v && !(M::kPacked && diag)) A.at(q1, p2) = y10;
          if (q1v && q2v) A.at(q1, q2) = y11;
        }
      }
      // Rows p, q of VT (columns of V): V <- V R.  Two pairs per pass, all loads of
      // a pass before its stores, so a global VT exposes one latency per pass.
      for (int k0 = warp; k0 < half; k0 += 2 * nw) {
        int pp[2], qq[2];
        double cc[2], ss[2];
#pragma unroll
        for (int h = 0; h < 2; ++h) {
          const int k = k0 + h * nw;
          const bool ok = k < half && Q[k < half ? k : 0] < n;
          pp[h] = ok ? P[k] : 0;
          qq[h] = ok ? Q[k] : 0;
          cc[h] = ok ? C[k] : 1.0;
          ss[h] = ok ? S[k] : 0.0;
          if (!ok) pp[h] = qq[h] = -1;
        }
        for (int i0 = lane; i0 < n; i0 += 256) {
          double a[2][8], b[2][8];
#pragma unroll
          for (int h = 0; h < 2; ++h)
#pragma unroll
            for (int u = 0; u < 8; ++u) {
              const int i = i0 + 32 * u;
              const bool ok = pp[h] >= 0 && i < n;
              a[h][u] = ok ? VT[(size_t)pp[h] * n + i] : 0.0;
              b[h][u] = ok ? VT[(size_t)qq[h] * n + i] : 0.0;
            }
#pragma unroll
          for (int h = 0; h < 2; ++h)
#pragma unroll
            for (int u = 0; u < 8; ++u) {
              const int i = i0 + 32 * u;
              if (pp[h] >= 0 && i < n) {
                VT[(size_t)pp[h] * n + i] = cc[h] * a[h][u] - ss[h] * b[h][u];
                VT[(size_t)qq[h] * n + i] = ss[h] * a[h][u] + cc[h] * b[h][u];
              }
            }
        }
      }
      __syncthreads();
    }
  }
  return sweep;
}

// After dss_block_jacobi: eigenvalues of A's diagonal in ascending order (ties
// by index) into w, and V (n x n row-major) with the eigenvectors as columns in
// the same order, from VT.  One thread block.
template <class M>
static __device__ __forceinline__ void dss_block_jacobi_sorted(M A, const double* VT, double* w, double* V) {
  const int n = A.n;
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    const double wi = A.at(i, i);
    int rk = 0;
    for (int j = 0; j < n; ++j) {
      const double wj = A.at(j, j);
      if (wj < wi || (wj == wi && j < i)) ++rk;
    }
    w[rk] = wi;
    for (int r = 0; r < n; ++r) V[(size_t)r * n + rk] = VT[(size_t)i * n + r];
  }
}

