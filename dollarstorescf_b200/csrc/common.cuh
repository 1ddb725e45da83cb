// Shared device-side types and the per-primitive-quartet set-up used by every
// generated ERI class (eri_gen.cuh).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "boys.cuh"

// One primitive pair of a shell pair (a, b): exponent sum p = alpha + beta, 1/p,
// the Gaussian product centre P, P - A, the pair prefactor
// K = w_a w_b exp(-alpha beta / p |A - B|^2), w the normalised primitive weights
// (chem/GTO.cpp:90-93 times the file coefficient), and Kp = sqrt(2 pi^2.5) K / p,
// the pair's share of the ERI prefactor.  80 bytes, 16-byte aligned, so a lane
// fetches one with five 16-byte loads.
struct __align__(16) PrimPair {
  double p, inv_p;
  double Px, Py, Pz;
  double PAx, PAy, PAz;
  double K;
  double Kp;
};

__device__ __forceinline__ PrimPair load_pp(const PrimPair* __restrict__ src) {
  const double2* s = reinterpret_cast<const double2*>(src);
  double2 a = __ldg(s), b = __ldg(s + 1), c = __ldg(s + 2), d = __ldg(s + 3), e = __ldg(s + 4);
  PrimPair r;
  r.p = a.x; r.inv_p = a.y;
  r.Px = b.x; r.Py = b.y;
  r.Pz = c.x; r.PAx = c.y;
  r.PAy = d.x; r.PAz = d.y;
  r.K = e.x; r.Kp = e.y;
  return r;
}

// 2 pi^2.5 with the reference's PI = 3.14159265358979 (lalib/MathUtil.hpp:8),
// the ERI prefactor of chem/GaussianIntegral.cpp:632.
#define DSS_TWO_PI_25 34.98683665524963

// Primitive-quartet set-up (cells: the reference-mode Boys records, see
// boys_ref_cells): Boys values scaled by the prefactor
//   2 pi^2.5 / (p q sqrt(p+q)) K_ab K_cd F_m(T),  T = rho |P-Q|^2,
// and the Obara-Saika coefficients used by the vertical recursion.
template <int BOYS, int L>
__device__ __forceinline__ void prim_quartet(const PrimPair& b, const PrimPair& k, double* F, double& PAx,
                                             double& PAy, double& PAz, double& WPx, double& WPy, double& WPz,
                                             double& QCx, double& QCy, double& QCz, double& WQx, double& WQy,
                                             double& WQz, double& oo2p, double& oo2q, double& oo2pq,
                                             double& rho_p, double& rho_q, const double* __restrict__ cells) {
  const double p = b.p, q = k.p;
  const double pq = p + q;
  const double r_pq = rsqrt(pq);  // 1/sqrt(p+q); its square is 1/(p+q) to ~2 ulp
  const double inv_pq = r_pq * r_pq;
  const double PQx = b.Px - k.Px, PQy = b.Py - k.Py, PQz = b.Pz - k.Pz;
  const double rho = p * q * inv_pq;
  const double T = rho * (PQx * PQx + PQy * PQy + PQz * PQz);
  rho_p = q * inv_pq;  // rho / p
  rho_q = p * inv_pq;  // rho / q
  PAx = b.PAx; PAy = b.PAy; PAz = b.PAz;
  QCx = k.PAx; QCy = k.PAy; QCz = k.PAz;
  WPx = -rho_p * PQx; WPy = -rho_p * PQy; WPz = -rho_p * PQz;
  WQx = rho_q * PQx; WQy = rho_q * PQy; WQz = rho_q * PQz;
  oo2p = 0.5 * b.inv_p;
  oo2q = 0.5 * k.inv_p;
  oo2pq = 0.5 * inv_pq;
  const double pref = b.Kp * k.Kp * r_pq;  // 2 pi^2.5 K_ab K_cd / (p q sqrt(p+q))
  boys_eval<BOYS, L>(T, F, cells);
#pragma unroll
  for (int m = 0; m <= L; ++m) F[m] *= pref;
}
