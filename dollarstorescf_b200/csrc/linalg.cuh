// Dense FP64 building blocks of the device SCF: a tiled GEMM, the parallel
// cyclic Jacobi eigensolver, and small helpers.  All matrices are row-major
// n x n in device memory.
#pragma once
#include <cuda_runtime.h>

// Jacobi stops when the off-diagonal Frobenius norm is below this fraction of
// the whole; double rounding leaves a floor near sqrt(n) * 1.1e-16 (2.7e-15 at
// n = 608), so a tighter target would only burn sweeps.
#define DSS_JACOBI_TOL 1e-14

// C = alpha * op(A) * op(B) + beta * C, op = transpose when the flag is set.
void dss_gemm(cudaStream_t s, int n, bool ta, bool tb, double alpha, const double* A, const double* B, double beta,
              double* C);

// Symmetric eigensolver (cyclic Jacobi, round-robin parallel ordering, one
// cooperative launch): on return w[n] holds the eigenvalues in ascending order
// and V (n x n, row-major) the eigenvectors as columns.  A is overwritten.
// work must hold 3 n^2 + 4 n + 64 doubles.  Returns cudaSuccess or the launch
// error; *sweeps receives the sweep count when non-NULL (device pointer ok: NULL).
cudaError_t dss_jacobi_eigh(cudaStream_t s, int n, double* A, double* V, double* w, double* work, int max_sweeps,
                            double tol, bool v_init);
