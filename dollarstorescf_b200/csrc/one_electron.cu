// One-electron matrices on the device: overlap, kinetic energy and nuclear
// attraction of a basis, replacing scf::assignOverlapMatrix /
// scf::assignCoreHamiltonian (chem/scf/SCFBasis.cpp:56-83) and the integrals
// they call (overlapIntegral, kineticEnergyIntegral, nuclearPotentialIntegral,
// chem/GaussianIntegral.cpp:29-332).
//
// One warp per shell pair, kernels templated on the pair class (l_a >= l_b).
// The lanes split the primitive pairs (overlap, kinetic) and the (primitive
// pair, nucleus) combinations (nuclear attraction); the sums are reduced with
// warp shuffles, after which every lane holds them, runs the horizontal
// transfer and the Cartesian -> function transform, and writes its share of the
// packed outputs.
//
// Obara-Saika for one centre pair (p = a + b, P the product centre):
//   overlap, per Cartesian direction:
//     S(i+1, j) = PA S(i, j) + (i S(i-1, j) + j S(i, j-1)) / (2p),  and likewise in j,
//     S(0, 0) = sqrt(pi/p) exp(-ab/p X_AB^2)
//   kinetic: -1/2 <a| d^2/dx^2 |b> per direction,
//     d^2/dx^2 x^j e^(-b x^2) = j(j-1) x^(j-2) - 2b(2j+1) x^j + 4b^2 x^(j+2)
//   nuclear attraction (nucleus C, charge Z, -Z <a| 1/r_C |b>):
//     [e+1_i]^(m) = PA_i [e]^(m) - PC_i [e]^(m+1) + e_i/(2p) ([e-1_i]^(m) - [e-1_i]^(m+1)),
//     [0]^(m) = 2 pi / p exp(-ab/p AB^2) F_m(p PC^2), then the horizontal transfer
//     (a|b+1_i) = (a+1_i|b) + AB_i (a|b); F_m are the reference's values
//     (boys_ref, the parity mode of the Boys function).
#include <cmath>
#include <algorithm>
#include <cstring>
#include <string>
#include <vector>

#include "boys.cuh"
#include "dss.h"
#include "dss_internal.h"
#include "sph_tab.h"

namespace {

constexpr double kPiRef = 3.14159265358979;  // lalib/MathUtil.hpp:8
constexpr int kLmaxOne = 2;                  // per shell, as the ERI kernels

__host__ __device__ constexpr int oe_ncart(int l) { return (l + 1) * (l + 2) / 2; }
__host__ __device__ constexpr int oe_coff(int l) { return l * (l + 1) * (l + 2) / 6; }
// Exponents of the k-th Cartesian monomial of degree l (x-major: x power
// descending, then y power descending).
__host__ __device__ constexpr int oe_cx(int l, int k) {
  int idx = 0;
  for (int a = l; a >= 0; --a)
    for (int b = l - a; b >= 0; --b) {
      if (idx == k) return a;
      ++idx;
    }
  return 0;
}
__host__ __device__ constexpr int oe_cy(int l, int k) {
  int idx = 0;
  for (int a = l; a >= 0; --a)
    for (int b = l - a; b >= 0; --b) {
      if (idx == k) return b;
      ++idx;
    }
  return 0;
}
// Index of x^a y^b z^c among all monomials of degree <= a + b + c.
__host__ __device__ constexpr int oe_idx(int a, int b, int c) {
  int pos = oe_coff(a + b + c);
  for (int ap = a + b + c; ap > a; --ap) pos += a + b + c - ap + 1;
  return pos + c;
}

struct OneEArgs {
  const int2* pairs;  // (shell with the larger l, other shell)
  int npair;
  const int* sh_l;
  const int* sh_nprim;
  const int* sh_prim0;
  const int* sh_f0;
  const double* sh_xyz;
  const double* exps;
  const double* wts;
  int natom;
  const double* atom_xyz;
  const double* atom_z;
  const double* tr;  // [l][function][Cartesian], 6 x 6 per l
  int pure;
  double* S;  // packed-U outputs; V == NULL: T receives T + V (the core Hamiltonian)
  double* T;
  double* V;
  const double* boys_cell;  // reference-mode Boys records (dss_boys_cell_table)
  // Gradient kernels: dense n x n densities D (contracted with dH) and W (with
  // dS), the nucleus of each shell, and the gradient accumulator [3 natom].
  const double* D;
  const double* W;
  const int* sh_atom;
  int n;
  double* grad;
};

__device__ __forceinline__ double oe_warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

template <int LA, int LB>
__global__ void __launch_bounds__(128) one_e_kernel(OneEArgs a) {
  constexpr int NA = oe_ncart(LA), NB = oe_ncart(LB);
  constexpr int E = LA + LB;
  constexpr int NE = oe_coff(E + 1);
  constexpr int NBC = oe_coff(LB + 1);
  const int warp = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5);
  const int lane = threadIdx.x & 31;
  if (warp >= a.npair) return;  // uniform per warp
  const int2 pr = a.pairs[warp];
  const int sa = pr.x, sb = pr.y;
  const double A[3] = {a.sh_xyz[3 * sa], a.sh_xyz[3 * sa + 1], a.sh_xyz[3 * sa + 2]};
  const double B[3] = {a.sh_xyz[3 * sb], a.sh_xyz[3 * sb + 1], a.sh_xyz[3 * sb + 2]};
  const double AB[3] = {A[0] - B[0], A[1] - B[1], A[2] - B[2]};
  const double AB2 = AB[0] * AB[0] + AB[1] * AB[1] + AB[2] * AB[2];
  const int npa = a.sh_nprim[sa], npb = a.sh_nprim[sb];
  const int pa0 = a.sh_prim0[sa], pb0 = a.sh_prim0[sb];
  const int npp = npa * npb;

  double S[NA * NB], T[NA * NB], Vacc[NE];
#pragma unroll
  for (int q = 0; q < NA * NB; ++q) S[q] = T[q] = 0.0;
#pragma unroll
  for (int q = 0; q < NE; ++q) Vacc[q] = 0.0;

  // Overlap and kinetic energy: lanes over primitive pairs.
  for (int t = lane; t < npp; t += 32) {
    const int i = t / npb, j = t - (t / npb) * npb;
    const double al = a.exps[pa0 + i], be = a.exps[pb0 + j];
    const double w = a.wts[pa0 + i] * a.wts[pb0 + j];
    const double p = al + be, mu = al * be / p;
    double PA[3], PB[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      const double P = (al * A[d] + be * B[d]) / p;
      PA[d] = P - A[d];
      PB[d] = P - B[d];
    }
    double Sd[3][LA + 1][LB + 3];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      Sd[d][0][0] = sqrt(kPiRef / p) * exp(-mu * AB[d] * AB[d]);
#pragma unroll
      for (int ii = 0; ii <= LA; ++ii)
#pragma unroll
        for (int jj = 0; jj <= LB + 2; ++jj) {
          if (ii == 0 && jj == 0) continue;
          double v;
          if (ii > 0) {
            v = PA[d] * Sd[d][ii - 1][jj];
            if (ii > 1) v += (ii - 1) * Sd[d][ii - 2][jj] / (2.0 * p);
            if (jj > 0) v += jj * Sd[d][ii - 1][jj - 1] / (2.0 * p);
          } else {
            v = PB[d] * Sd[d][0][jj - 1];
            if (jj > 1) v += (jj - 1) * Sd[d][0][jj - 2] / (2.0 * p);
          }
          Sd[d][ii][jj] = v;
        }
    }
#pragma unroll
    for (int ia = 0; ia < NA; ++ia)
#pragma unroll
      for (int ib = 0; ib < NB; ++ib) {
        const int ea[3] = {oe_cx(LA, ia), oe_cy(LA, ia), LA - oe_cx(LA, ia) - oe_cy(LA, ia)};
        const int eb[3] = {oe_cx(LB, ib), oe_cy(LB, ib), LB - oe_cx(LB, ib) - oe_cy(LB, ib)};
        const double sx = Sd[0][ea[0]][eb[0]], sy = Sd[1][ea[1]][eb[1]], sz = Sd[2][ea[2]][eb[2]];
        S[ia * NB + ib] += w * sx * sy * sz;
        double tk = 0.0;
#pragma unroll
        for (int d = 0; d < 3; ++d) {
          const int jj = eb[d], ii = ea[d];
          double k = -2.0 * be * (2 * jj + 1) * Sd[d][ii][jj] + 4.0 * be * be * Sd[d][ii][jj + 2];
          if (jj > 1) k += jj * (jj - 1) * Sd[d][ii][jj - 2];
          double o = 1.0;
#pragma unroll
          for (int d2 = 0; d2 < 3; ++d2)
            if (d2 != d) o *= Sd[d2][ea[d2]][eb[d2]];
          tk += -0.5 * k * o;
        }
        T[ia * NB + ib] += w * tk;
      }
  }

  // Nuclear attraction: lanes over (primitive pair, nucleus).
  const int nwork = npp * a.natom;
  for (int t = lane; t < nwork; t += 32) {
    const int q = t / a.natom, c = t - (t / a.natom) * a.natom;
    const int i = q / npb, j = q - (q / npb) * npb;
    const double al = a.exps[pa0 + i], be = a.exps[pb0 + j];
    const double w = a.wts[pa0 + i] * a.wts[pb0 + j];
    const double p = al + be, mu = al * be / p;
    double PA[3], PC[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      const double P = (al * A[d] + be * B[d]) / p;
      PA[d] = P - A[d];
      PC[d] = P - a.atom_xyz[3 * c + d];
    }
    const double pref = 2.0 * kPiRef / p * exp(-mu * AB2) * w;
    const double x = p * (PC[0] * PC[0] + PC[1] * PC[1] + PC[2] * PC[2]);
    double F[E + 1];
    boys_ref<E>(x, F, a.boys_cell);
    double Vt[E + 1][NE];
#pragma unroll
    for (int m = 0; m <= E; ++m) Vt[m][0] = pref * F[m];
#pragma unroll
    for (int e = 1; e <= E; ++e)
#pragma unroll
      for (int k = 0; k < oe_ncart(e); ++k) {
        const int qx = oe_cx(e, k), qy = oe_cy(e, k), qz = e - qx - qy;
        const int dir = qx ? 0 : (qy ? 1 : 2);
        const int mx = qx - (dir == 0), my = qy - (dir == 1), mz = qz - (dir == 2);
        const int edir = dir == 0 ? mx : (dir == 1 ? my : mz);
        const int i1 = oe_idx(mx, my, mz);
        const int it = oe_idx(qx, qy, qz);
#pragma unroll
        for (int m = 0; m <= E - e; ++m) {
          double v = PA[dir] * Vt[m][i1] - PC[dir] * Vt[m + 1][i1];
          if (edir > 0) {
            const int i2 = oe_idx(mx - (dir == 0), my - (dir == 1), mz - (dir == 2));
            v += edir / (2.0 * p) * (Vt[m][i2] - Vt[m + 1][i2]);
          }
          Vt[m][it] = v;
        }
      }
    const double z = a.atom_z[c];
#pragma unroll
    for (int e = 0; e < NE; ++e) Vacc[e] += -z * Vt[0][e];
  }

#pragma unroll
  for (int q = 0; q < NA * NB; ++q) {
    S[q] = oe_warp_sum(S[q]);
    T[q] = oe_warp_sum(T[q]);
  }
#pragma unroll
  for (int q = 0; q < NE; ++q) Vacc[q] = oe_warp_sum(Vacc[q]);

  // Horizontal transfer of the nuclear integrals to (a|b).
  double br[NE][NBC];
#pragma unroll
  for (int e = 0; e < NE; ++e) br[e][0] = Vacc[e];
#pragma unroll
  for (int bd = 1; bd <= LB; ++bd)
#pragma unroll
    for (int k = 0; k < oe_ncart(bd); ++k) {
      const int qx = oe_cx(bd, k), qy = oe_cy(bd, k), qz = bd - qx - qy;
      const int dir = qx ? 0 : (qy ? 1 : 2);
      const int ibm = oe_idx(qx - (dir == 0), qy - (dir == 1), qz - (dir == 2));
      const int ibt = oe_idx(qx, qy, qz);
#pragma unroll
      for (int ed = 0; ed <= E - bd; ++ed)
#pragma unroll
        for (int r = 0; r < oe_ncart(ed); ++r) {
          const int rx = oe_cx(ed, r), ry = oe_cy(ed, r), rz = ed - rx - ry;
          const int ie = oe_idx(rx, ry, rz);
          const int iep = oe_idx(rx + (dir == 0), ry + (dir == 1), rz + (dir == 2));
          br[ie][ibt] = br[iep][ibm] + AB[dir] * br[ie][ibm];
        }
    }

  // Functions: pure (m = -l..l) or Cartesian, through the transform table.
  const int nfa = a.pure ? 2 * LA + 1 : NA, nfb = a.pure ? 2 * LB + 1 : NB;
  const int fa0 = a.sh_f0[sa], fb0 = a.sh_f0[sb];
  const double* ta = a.tr + LA * 36;
  const double* tb = a.tr + LB * 36;
  for (int o = lane; o < nfa * nfb; o += 32) {
    const int fa = o / nfb, fb = o - (o / nfb) * nfb;
    const int i = fa0 + fa, j = fb0 + fb;
    if (sa == sb && j > i) continue;
    double s = 0.0, tt = 0.0, v = 0.0;
#pragma unroll
    for (int ca = 0; ca < NA; ++ca) {
      const double wa = ta[fa * 6 + ca];
      if (wa == 0.0) continue;
#pragma unroll
      for (int cb = 0; cb < NB; ++cb) {
        const double wgt = wa * tb[fb * 6 + cb];
        if (wgt == 0.0) continue;
        s += wgt * S[ca * NB + cb];
        tt += wgt * T[ca * NB + cb];
        v += wgt * br[oe_coff(LA) + ca][oe_coff(LB) + cb];
      }
    }
    const int x = i > j ? i : j, y = i > j ? j : i;
    const size_t idx = (size_t)x * (x + 1) / 2 + y;
    if (a.S) a.S[idx] = s;
    if (a.V) {
      a.T[idx] = tt;
      a.V[idx] = v;
    } else {
      a.T[idx] = tt + v;
    }
  }
}

// Analytic one-electron part of the nuclear gradient for one shell-pair class:
//   sum_mn D_mn dH_mn/dR - sum_mn W_mn dS_mn/dR,
// H = T + V.  A primitive Cartesian Gaussian moves with its centre, so
//   d/dA_x <a|O|b> = 2 alpha <a+1_x|O|b> - a_x <a-1_x|O|b>
// (chem/GaussianIntegral.cpp:1052-1459 differentiates the same way).  S and T
// depend on A - B only (d/dB = -d/dA); the nuclear attraction of nucleus C is
// invariant under moving A, B and C together, so its C derivative (the
// Hellmann-Feynman term) is -(d/dA + d/dB).  One warp per shell pair: lanes over
// primitive pairs (S, T) and over (primitive pair, nucleus) (V), the pair's
// densities carried to the Cartesian basis first; the A and B sums are reduced
// over the warp, the C terms added per item.
__device__ __forceinline__ double oe_binom(int n, int k) {
  double r = 1.0;
  for (int i = 1; i <= k; ++i) r = r * (n - k + i) / i;
  return r;
}

template <int LA, int LB>
__global__ void __launch_bounds__(128) one_e_grad_kernel(OneEArgs a) {
  constexpr int NA = oe_ncart(LA), NB = oe_ncart(LB);
  constexpr int E1 = LA + LB + 1;
  constexpr int NE1 = oe_coff(E1 + 1);
  const int warp = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5);
  const int lane = threadIdx.x & 31;
  if (warp >= a.npair) return;  // uniform per warp
  const int2 pr = a.pairs[warp];
  const int sa = pr.x, sb = pr.y;
  const double A[3] = {a.sh_xyz[3 * sa], a.sh_xyz[3 * sa + 1], a.sh_xyz[3 * sa + 2]};
  const double B[3] = {a.sh_xyz[3 * sb], a.sh_xyz[3 * sb + 1], a.sh_xyz[3 * sb + 2]};
  const double AB[3] = {A[0] - B[0], A[1] - B[1], A[2] - B[2]};
  const double AB2 = AB[0] * AB[0] + AB[1] * AB[1] + AB[2] * AB[2];
  const int npa = a.sh_nprim[sa], npb = a.sh_nprim[sb];
  const int pa0 = a.sh_prim0[sa], pb0 = a.sh_prim0[sb];
  const int npp = npa * npb;
  // The pair's densities in the Cartesian basis (both orders of an unlike pair).
  const int nfa = a.pure ? 2 * LA + 1 : NA, nfb = a.pure ? 2 * LB + 1 : NB;
  const int fa0 = a.sh_f0[sa], fb0 = a.sh_f0[sb];
  const double* ta = a.tr + LA * 36;
  const double* tb = a.tr + LB * 36;
  const double fac = sa == sb ? 1.0 : 2.0;
  double Pc[NA * NB], Qc[NA * NB];
#pragma unroll
  for (int ca = 0; ca < NA; ++ca)
#pragma unroll
    for (int cb = 0; cb < NB; ++cb) {
      double p = 0.0, q = 0.0;
      for (int fa = 0; fa < nfa; ++fa)
        for (int fb = 0; fb < nfb; ++fb) {
          const double w = ta[fa * 6 + ca] * tb[fb * 6 + cb];
          if (w == 0.0) continue;
          const size_t ij = (size_t)(fa0 + fa) * a.n + fb0 + fb;
          p += w * a.D[ij];
          q += w * a.W[ij];
        }
      Pc[ca * NB + cb] = fac * p;
      Qc[ca * NB + cb] = fac * q;
    }
  double gA[3] = {0.0, 0.0, 0.0}, gB[3] = {0.0, 0.0, 0.0};

  // Overlap and kinetic energy.
  for (int t = lane; t < npp; t += 32) {
    const int i = t / npb, j = t - (t / npb) * npb;
    const double al = a.exps[pa0 + i], be = a.exps[pb0 + j];
    const double w = a.wts[pa0 + i] * a.wts[pb0 + j];
    const double p = al + be, mu = al * be / p;
    double PA[3], PB[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      const double P = (al * A[d] + be * B[d]) / p;
      PA[d] = P - A[d];
      PB[d] = P - B[d];
    }
    double Sd[3][LA + 2][LB + 3];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      Sd[d][0][0] = sqrt(kPiRef / p) * exp(-mu * AB[d] * AB[d]);
#pragma unroll
      for (int ii = 0; ii <= LA + 1; ++ii)
#pragma unroll
        for (int jj = 0; jj <= LB + 2; ++jj) {
          if (ii == 0 && jj == 0) continue;
          double v;
          if (ii > 0) {
            v = PA[d] * Sd[d][ii - 1][jj];
            if (ii > 1) v += (ii - 1) * Sd[d][ii - 2][jj] / (2.0 * p);
            if (jj > 0) v += jj * Sd[d][ii - 1][jj - 1] / (2.0 * p);
          } else {
            v = PB[d] * Sd[d][0][jj - 1];
            if (jj > 1) v += (jj - 1) * Sd[d][0][jj - 2] / (2.0 * p);
          }
          Sd[d][ii][jj] = v;
        }
    }
    // 1-D kinetic factor -1/2 <i| d^2/dx^2 |j> of direction d.
    auto kin = [&](int d, int ii, int jj) {
      double k = -2.0 * be * (2 * jj + 1) * Sd[d][ii][jj] + 4.0 * be * be * Sd[d][ii][jj + 2];
      if (jj > 1) k += jj * (jj - 1) * Sd[d][ii][jj - 2];
      return -0.5 * k;
    };
#pragma unroll
    for (int ia = 0; ia < NA; ++ia)
#pragma unroll
      for (int ib = 0; ib < NB; ++ib) {
        const int ea[3] = {oe_cx(LA, ia), oe_cy(LA, ia), LA - oe_cx(LA, ia) - oe_cy(LA, ia)};
        const int eb[3] = {oe_cx(LB, ib), oe_cy(LB, ib), LB - oe_cx(LB, ib) - oe_cy(LB, ib)};
        const double pc = Pc[ia * NB + ib], qc = Qc[ia * NB + ib];
        double s1[3], k1[3], ds[3], dk[3];
#pragma unroll
        for (int d = 0; d < 3; ++d) {
          s1[d] = Sd[d][ea[d]][eb[d]];
          k1[d] = kin(d, ea[d], eb[d]);
          ds[d] = 2.0 * al * Sd[d][ea[d] + 1][eb[d]];
          dk[d] = 2.0 * al * kin(d, ea[d] + 1, eb[d]);
          if (ea[d] > 0) {
            ds[d] -= ea[d] * Sd[d][ea[d] - 1][eb[d]];
            dk[d] -= ea[d] * kin(d, ea[d] - 1, eb[d]);
          }
        }
#pragma unroll
        for (int d = 0; d < 3; ++d) {
          const int d1 = (d + 1) % 3, d2 = (d + 2) % 3;
          const double dS = ds[d] * s1[d1] * s1[d2];
          const double dT = dk[d] * s1[d1] * s1[d2] + ds[d] * (k1[d1] * s1[d2] + s1[d1] * k1[d2]);
          gA[d] += w * (pc * dT - qc * dS);
        }
      }
  }
#pragma unroll
  for (int d = 0; d < 3; ++d) gB[d] = -gA[d];

  // Nuclear attraction: lanes over (primitive pair, nucleus).
  const int nwork = npp * a.natom;
  for (int t = lane; t < nwork; t += 32) {
    const int q = t / a.natom, c = t - (t / a.natom) * a.natom;
    const int i = q / npb, j = q - (q / npb) * npb;
    const double al = a.exps[pa0 + i], be = a.exps[pb0 + j];
    const double w = a.wts[pa0 + i] * a.wts[pb0 + j];
    const double p = al + be, mu = al * be / p;
    double PA[3], PC[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      const double P = (al * A[d] + be * B[d]) / p;
      PA[d] = P - A[d];
      PC[d] = P - a.atom_xyz[3 * c + d];
    }
    const double z = a.atom_z[c];
    const double pref = -z * 2.0 * kPiRef / p * exp(-mu * AB2) * w;
    const double x = p * (PC[0] * PC[0] + PC[1] * PC[1] + PC[2] * PC[2]);
    double F[E1 + 1];
    boys_ref<E1>(x, F, a.boys_cell);
    double Vt[E1 + 1][NE1];
#pragma unroll
    for (int m = 0; m <= E1; ++m) Vt[m][0] = pref * F[m];
#pragma unroll
    for (int e = 1; e <= E1; ++e)
#pragma unroll
      for (int k = 0; k < oe_ncart(e); ++k) {
        const int qx = oe_cx(e, k), qy = oe_cy(e, k), qz = e - qx - qy;
        const int dir = qx ? 0 : (qy ? 1 : 2);
        const int mx = qx - (dir == 0), my = qy - (dir == 1), mz = qz - (dir == 2);
        const int edir = dir == 0 ? mx : (dir == 1 ? my : mz);
        const int i1 = oe_idx(mx, my, mz);
        const int it = oe_idx(qx, qy, qz);
#pragma unroll
        for (int m = 0; m <= E1 - e; ++m) {
          double v = PA[dir] * Vt[m][i1] - PC[dir] * Vt[m + 1][i1];
          if (edir > 0) {
            const int i2 = oe_idx(mx - (dir == 0), my - (dir == 1), mz - (dir == 2));
            v += edir / (2.0 * p) * (Vt[m][i2] - Vt[m + 1][i2]);
          }
          Vt[m][it] = v;
        }
      }
    // (a|V_C|b) by the horizontal transfer written out:
    // (a|b) = sum_{k <= b} prod_i C(b_i, k_i) AB_i^(b_i - k_i) [a + k].
    auto vab = [&](int ax, int ay, int az, int bx, int by, int bz) {
      double s = 0.0;
      for (int kx = 0; kx <= bx; ++kx)
        for (int ky = 0; ky <= by; ++ky)
          for (int kz = 0; kz <= bz; ++kz) {
            double f = oe_binom(bx, kx) * oe_binom(by, ky) * oe_binom(bz, kz);
            for (int r = kx; r < bx; ++r) f *= AB[0];
            for (int r = ky; r < by; ++r) f *= AB[1];
            for (int r = kz; r < bz; ++r) f *= AB[2];
            s += f * Vt[0][oe_idx(ax + kx, ay + ky, az + kz)];
          }
      return s;
    };
    double cA[3] = {0.0, 0.0, 0.0}, cB[3] = {0.0, 0.0, 0.0};
    for (int ia = 0; ia < NA; ++ia)
      for (int ib = 0; ib < NB; ++ib) {
        const int ea[3] = {oe_cx(LA, ia), oe_cy(LA, ia), LA - oe_cx(LA, ia) - oe_cy(LA, ia)};
        const int eb[3] = {oe_cx(LB, ib), oe_cy(LB, ib), LB - oe_cx(LB, ib) - oe_cy(LB, ib)};
        const double pc = Pc[ia * NB + ib];
        for (int d = 0; d < 3; ++d) {
          const int u[3] = {d == 0, d == 1, d == 2};
          double dA = 2.0 * al * vab(ea[0] + u[0], ea[1] + u[1], ea[2] + u[2], eb[0], eb[1], eb[2]);
          if (ea[d] > 0) dA -= ea[d] * vab(ea[0] - u[0], ea[1] - u[1], ea[2] - u[2], eb[0], eb[1], eb[2]);
          double dB = 2.0 * be * vab(ea[0], ea[1], ea[2], eb[0] + u[0], eb[1] + u[1], eb[2] + u[2]);
          if (eb[d] > 0) dB -= eb[d] * vab(ea[0], ea[1], ea[2], eb[0] - u[0], eb[1] - u[1], eb[2] - u[2]);
          cA[d] += pc * dA;
          cB[d] += pc * dB;
        }
      }
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      gA[d] += cA[d];
      gB[d] += cB[d];
      atomicAdd(a.grad + 3 * c + d, -(cA[d] + cB[d]));
    }
  }
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    gA[d] = oe_warp_sum(gA[d]);
    gB[d] = oe_warp_sum(gB[d]);
  }
  if (lane == 0) {
    const int ata = a.sh_atom[sa], atb = a.sh_atom[sb];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      atomicAdd(a.grad + 3 * ata + d, gA[d]);
      atomicAdd(a.grad + 3 * atb + d, gB[d]);
    }
  }
}

template <int LA, int LB>
void launch_one_e_grad(const OneEArgs& a, cudaStream_t s) {
  const unsigned blocks = (unsigned)(((long long)a.npair * 32 + 127) / 128);
  if (blocks) one_e_grad_kernel<LA, LB><<<blocks, 128, 0, s>>>(a);
}

void launch_one_e_grad_class(int la, int lb, const OneEArgs& a, cudaStream_t s) {
  switch (la * 3 + lb) {
    case 0: return launch_one_e_grad<0, 0>(a, s);
    case 3: return launch_one_e_grad<1, 0>(a, s);
    case 4: return launch_one_e_grad<1, 1>(a, s);
    case 6: return launch_one_e_grad<2, 0>(a, s);
    case 7: return launch_one_e_grad<2, 1>(a, s);
    case 8: return launch_one_e_grad<2, 2>(a, s);
    default: return;
  }
}

template <int LA, int LB>
void launch_one_e(const OneEArgs& a, cudaStream_t s) {
  const unsigned blocks = (unsigned)(((long long)a.npair * 32 + 127) / 128);
  if (blocks) one_e_kernel<LA, LB><<<blocks, 128, 0, s>>>(a);
}

void launch_one_e_class(int la, int lb, const OneEArgs& a, cudaStream_t s) {
  switch (la * 3 + lb) {
    case 0: return launch_one_e<0, 0>(a, s);
    case 3: return launch_one_e<1, 0>(a, s);
    case 4: return launch_one_e<1, 1>(a, s);
    case 6: return launch_one_e<2, 0>(a, s);
    case 7: return launch_one_e<2, 1>(a, s);
    case 8: return launch_one_e<2, 2>(a, s);
    default: return;
  }
}

}  // namespace

namespace {

// Uploads the inputs of the one-electron kernels (shells, primitives, nuclei,
// function transforms, shell-pair lists by class, and the nucleus of each shell
// when shell_atom is given) and fills the common kernel arguments; c0[c] is the
// first pair of class c (la * 3 + lb) in the pair list.
int one_e_stage(cudaStream_t s, const BasisHost& B, int natom, const int* Z, const double* xyz_bohr,
                const int* shell_atom, std::string* errp, OneEScratch& sc, OneEArgs* out, std::vector<size_t>* c0) {
  const int ns = (int)B.l.size();
  for (int q = 0; q < ns; ++q)
    if (B.l[q] < 0 || B.l[q] > kLmaxOne) {
      if (errp) *errp = "dss_one_electron: l above 2";
      return DSS_ERR_UNSUPPORTED;
    }
  // Transform tables [l][function][Cartesian] for the basis' 5D/6D choice.
  std::vector<double> tr((kLmaxOne + 1) * 36, 0.0);
  for (int t = 0; t < kDssSphTermCount; ++t) {
    const DssSphTerm& q = kDssSphTerms[t];
    if (q.pure == B.pure && q.l <= kLmaxOne) tr[q.l * 36 + q.func * 6 + q.cart] = q.w;
  }
  // Shell pairs grouped by class, the larger l first.
  std::vector<std::vector<int2>> cls(9);
  for (int x = 0; x < ns; ++x)
    for (int y = 0; y <= x; ++y) {
      const int a = B.l[y] > B.l[x] ? y : x, b = a == x ? y : x;
      cls[B.l[a] * 3 + B.l[b]].push_back(make_int2(a, b));
    }
  std::vector<int2> pairs;
  c0->assign(10, 0);
  for (int c = 0; c < 9; ++c) {
    (*c0)[c] = pairs.size();
    pairs.insert(pairs.end(), cls[c].begin(), cls[c].end());
  }
  (*c0)[9] = pairs.size();
  std::vector<double> zd(natom);
  for (int c = 0; c < natom; ++c) zd[c] = (double)Z[c];
  // One upload of every input.
  const size_t ni = 5 * (size_t)ns, nd = 3 * (size_t)ns + 2 * B.exps.size() + 4 * (size_t)natom + tr.size();
  std::vector<int> hi(ni, 0);
  std::vector<double> hd;
  hd.reserve(nd);
  for (int q = 0; q < ns; ++q) {
    hi[q] = B.l[q];
    hi[ns + q] = B.nprim[q];
    hi[2 * ns + q] = B.prim0[q];
    hi[3 * ns + q] = B.f0[q];
    hi[4 * ns + q] = shell_atom ? shell_atom[q] : 0;
  }
  hd.insert(hd.end(), B.xyz.begin(), B.xyz.end());
  hd.insert(hd.end(), B.exps.begin(), B.exps.end());
  hd.insert(hd.end(), B.wts.begin(), B.wts.end());
  hd.insert(hd.end(), xyz_bohr, xyz_bohr + 3 * (size_t)natom);
  hd.insert(hd.end(), zd.begin(), zd.end());
  hd.insert(hd.end(), tr.begin(), tr.end());
  DevBuf<int2>& d_pairs = sc.pairs;
  DevBuf<int>& d_i = sc.ints;
  DevBuf<double>& d_d = sc.dbl;
  cudaError_t e = d_pairs.resize(std::max<size_t>(pairs.size(), 1));
  if (e == cudaSuccess) e = d_i.resize(std::max<size_t>(ni, 1));
  if (e == cudaSuccess) e = d_d.resize(std::max<size_t>(hd.size(), 1));
  if (e == cudaSuccess && !pairs.empty())
    e = cudaMemcpyAsync(d_pairs.ptr, pairs.data(), pairs.size() * sizeof(int2), cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess && ni) e = cudaMemcpyAsync(d_i.ptr, hi.data(), ni * sizeof(int), cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess && !hd.empty())
    e = cudaMemcpyAsync(d_d.ptr, hd.data(), hd.size() * sizeof(double), cudaMemcpyHostToDevice, s);
  if (e != cudaSuccess) {
    if (errp) *errp = std::string("dss_one_electron: ") + cudaGetErrorString(e);
    return e == cudaErrorMemoryAllocation ? DSS_ERR_OOM : DSS_ERR_CUDA;
  }
  OneEArgs a{};
  a.pairs = d_pairs.ptr;
  a.sh_l = d_i.ptr;
  a.sh_nprim = d_i.ptr + ns;
  a.sh_prim0 = d_i.ptr + 2 * ns;
  a.sh_f0 = d_i.ptr + 3 * ns;
  a.sh_atom = d_i.ptr + 4 * ns;
  a.sh_xyz = d_d.ptr;
  a.exps = a.sh_xyz + 3 * ns;
  a.wts = a.exps + B.exps.size();
  a.atom_xyz = a.wts + B.exps.size();
  a.atom_z = a.atom_xyz + 3 * (size_t)natom;
  a.tr = a.atom_z + natom;
  a.natom = natom;
  a.pure = B.pure;
  a.n = B.nbf;
  e = dss_boys_cell_table(&a.boys_cell);
  if (e != cudaSuccess) {
    if (errp) *errp = std::string("dss_one_electron: ") + cudaGetErrorString(e);
    return DSS_ERR_CUDA;
  }
  *out = a;
  return DSS_OK;
}

}  // namespace

int dss_one_electron_device(cudaStream_t s, const BasisHost& B, int natom, const int* Z, const double* xyz_bohr,
                            double* dS, double* dT, double* dV, std::string* errp, OneEScratch* scratch) {
  OneEScratch local;
  OneEScratch& sc = scratch ? *scratch : local;
  OneEArgs a;
  std::vector<size_t> c0;
  int rc = one_e_stage(s, B, natom, Z, xyz_bohr, nullptr, errp, sc, &a, &c0);
  if (rc != DSS_OK) return rc;
  a.S = dS;
  a.T = dT;
  a.V = dV;
  const int2* all = a.pairs;
  for (int c = 0; c < 9; ++c) {
    if (c0[c + 1] == c0[c]) continue;
    a.pairs = all + c0[c];
    a.npair = (int)(c0[c + 1] - c0[c]);
    launch_one_e_class(c / 3, c % 3, a, s);
  }
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);  // the inputs are freed or reused after return
  if (e != cudaSuccess) {
    if (errp) *errp = std::string("dss_one_electron: ") + cudaGetErrorString(e);
    return DSS_ERR_CUDA;
  }
  return DSS_OK;
}

int dss_one_electron_gradient(cudaStream_t s, const BasisHost& B, int natom, const int* Z, const double* xyz_bohr,
                              const int* shell_atom, const double* D_dev, const double* W_dev, double* grad_host,
                              std::string* errp, OneEScratch* scratch) {
  OneEScratch local;
  OneEScratch& sc = scratch ? *scratch : local;
  OneEArgs a;
  std::vector<size_t> c0;
  int rc = one_e_stage(s, B, natom, Z, xyz_bohr, shell_atom, errp, sc, &a, &c0);
  if (rc != DSS_OK) return rc;
  DevBuf<double> g;
  cudaError_t e = g.resize(std::max(3 * natom, 1));
  if (e == cudaSuccess) e = cudaMemsetAsync(g.ptr, 0, 3 * (size_t)natom * sizeof(double), s);
  if (e != cudaSuccess) {
    if (errp) *errp = std::string("dss_one_electron_gradient: ") + cudaGetErrorString(e);
    return e == cudaErrorMemoryAllocation ? DSS_ERR_OOM : DSS_ERR_CUDA;
  }
  a.D = D_dev;
  a.W = W_dev;
  a.grad = g.ptr;
  const int2* all = a.pairs;
  for (int c = 0; c < 9; ++c) {
    if (c0[c + 1] == c0[c]) continue;
    a.pairs = all + c0[c];
    a.npair = (int)(c0[c + 1] - c0[c]);
    launch_one_e_grad_class(c / 3, c % 3, a, s);
  }
  e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaMemcpyAsync(grad_host, g.ptr, 3 * (size_t)natom * sizeof(double), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) {
    if (errp) *errp = std::string("dss_one_electron_gradient: ") + cudaGetErrorString(e);
    return DSS_ERR_CUDA;
  }
  return DSS_OK;
}

double dss_nuclear_repulsion(int natom, const int* Z, const double* xyz_bohr) {
  // sum_{A<B} Z_A Z_B / R_AB (chem/scf/Energy.cpp:44-49)
  double e = 0.0;
  for (int i = 0; i < natom; ++i)
    for (int j = i + 1; j < natom; ++j) {
      const double dx = xyz_bohr[3 * i] - xyz_bohr[3 * j], dy = xyz_bohr[3 * i + 1] - xyz_bohr[3 * j + 1],
                   dz = xyz_bohr[3 * i + 2] - xyz_bohr[3 * j + 2];
      e += (double)Z[i] * Z[j] / std::sqrt(dx * dx + dy * dy + dz * dz);
    }
  return e;
}

int dss_one_electron_basis(cudaStream_t s, const BasisHost& B, int natom, const int* Z, const double* xyz_bohr,
                           double* S_packed, double* T_packed, double* V_packed, double* e_nuc, std::string* errp,
                           OneEScratch* scratch) {
  const size_t np = (size_t)B.nbf * (B.nbf + 1) / 2;
  DevBuf<double> d;
  cudaError_t e = d.resize(std::max<size_t>(3 * np, 1));
  if (e != cudaSuccess) {
    if (errp) *errp = std::string("dss_one_electron: ") + cudaGetErrorString(e);
    return DSS_ERR_OOM;
  }
  int rc = dss_one_electron_device(s, B, natom, Z, xyz_bohr, d.ptr, d.ptr + np, d.ptr + 2 * np, errp, scratch);
  if (rc != DSS_OK) return rc;
  double* outs[3] = {S_packed, T_packed, V_packed};
  for (int k = 0; k < 3 && e == cudaSuccess; ++k)
    if (outs[k] && np) e = cudaMemcpyAsync(outs[k], d.ptr + k * np, np * 8, cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) {
    if (errp) *errp = std::string("dss_one_electron: ") + cudaGetErrorString(e);
    return DSS_ERR_CUDA;
  }
  if (e_nuc) *e_nuc = dss_nuclear_repulsion(natom, Z, xyz_bohr);
  return DSS_OK;
}

extern "C" int dss_one_electron(dss_ctx* ctx, int natom, const int* Z, const double* xyz_bohr, double* S_packed,
                                double* T_packed, double* V_packed, double* e_nuc) {
  if (!ctx) return DSS_ERR_INVALID;
  ctx->err.clear();
  if (!ctx->nbf || ctx->nmol > 0) return dss_fail(ctx, DSS_ERR_INVALID, "dss_one_electron: no single-molecule basis set");
  if (natom < 0 || (natom > 0 && (!Z || !xyz_bohr)))
    return dss_fail(ctx, DSS_ERR_INVALID, "dss_one_electron: bad atom arrays");
  cudaSetDevice(ctx->opts.device);
  std::string err;
  const int rc = dss_one_electron_basis(ctx->stream, ctx->basis, natom, Z, xyz_bohr, S_packed, T_packed, V_packed,
                                        e_nuc, &err, &ctx->oe_scratch);
  if (rc != DSS_OK) return dss_fail(ctx, rc, err);
  return DSS_OK;
}
