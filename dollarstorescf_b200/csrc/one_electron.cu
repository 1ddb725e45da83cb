// One-electron matrices on the host (C++, threads over shell pairs): overlap,
// kinetic energy and nuclear attraction of the current basis, replacing
// scf::assignOverlapMatrix / scf::assignCoreHamiltonian
// (chem/scf/SCFBasis.cpp:56-83) and the integrals they call
// (overlapIntegral, kineticEnergyIntegral, nuclearPotentialIntegral,
// chem/GaussianIntegral.cpp:29-332).
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
//     (a|b+1_i) = (a+1_i|b) + AB_i (a|b); F_m with the reference's series (parity).
#include <cmath>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

#include "dss.h"
#include "dss_internal.h"
#include "sph_tab.h"

namespace {

constexpr double kPiRef = 3.14159265358979;  // lalib/MathUtil.hpp:8
constexpr int kLmax = 4;                     // per shell on the host path
constexpr int kNC = (kLmax + 1) * (kLmax + 2) / 2;

int ncart(int l) { return (l + 1) * (l + 2) / 2; }
int coff(int l) { return l * (l + 1) * (l + 2) / 6; }
int cidx(int a, int b, int c) {
  const int l = a + b + c;
  int pos = 0;
  for (int ap = l; ap > a; --ap) pos += l - ap + 1;
  return pos + (l - a - b);
}
int call_idx(int a, int b, int c) { return coff(a + b + c) + cidx(a, b, c); }

struct Cart3 {
  int x, y, z;
};
std::vector<std::vector<Cart3>> cart_tables() {
  std::vector<std::vector<Cart3>> t(2 * kLmax + 2);
  for (int l = 0; l < (int)t.size(); ++l)
    for (int a = l; a >= 0; --a)
      for (int b = l - a; b >= 0; --b) t[l].push_back({a, b, l - a - b});
  return t;
}

// The reference's Boys function (chem/GaussianIntegral.cpp:209-223).
double boys_ref_host(double x, unsigned m) {
  if (x > (double)m * 1.1 + 25.0) {
    unsigned int dfi = 1u;
    for (int j = 2 * (int)m - 1; j > 0; j -= 2) dfi *= (unsigned int)j;
    double p2 = 1.0;
    for (unsigned j = 0; j < m + 1; ++j) p2 *= 2.0;
    // integer power in the reference's square-and-multiply order
    unsigned p = 2 * m + 1;
    double fac[8];
    int nf = 0;
    double tail;
    while (true) {
      if (p == 0) { tail = 1.0; break; }
      if (p == 1) { tail = x; break; }
      double y = x;
      unsigned l = 2;
      for (; l < p; l *= 2) y = y * y;
      fac[nf++] = y;
      p -= l / 2;
    }
    double r = tail;
    for (int i = nf - 1; i >= 0; --i) r = fac[i] * r;
    return (double)(int)dfi / p2 * std::sqrt(kPiRef / r);
  }
  double F = 1.0, a = 1.0;
  for (int i = 1; a > 0.000000001; ++i) {
    a = 2.0 * x / (double)(2 * (int)m + 2 * i + 1) * a;
    F += a;
  }
  return std::exp(-x) / (double)(2 * m + 1) * F;
}

struct PairOut {
  // Cartesian blocks [ncart(la)][ncart(lb)]
  double S[kNC * kNC], T[kNC * kNC], V[kNC * kNC];
};

void pair_integrals(const BasisHost& B, int sa, int sb, int natom, const int* Z, const double* xyz,
                    const std::vector<std::vector<Cart3>>& ct, PairOut& out) {
  const int la = B.l[sa], lb = B.l[sb];
  const int na = ncart(la), nb = ncart(lb);
  std::memset(&out, 0, sizeof(out));
  const double* A = &B.xyz[3 * sa];
  const double* Bc = &B.xyz[3 * sb];
  const double AB[3] = {A[0] - Bc[0], A[1] - Bc[1], A[2] - Bc[2]};
  const double AB2 = AB[0] * AB[0] + AB[1] * AB[1] + AB[2] * AB[2];
  const int E = la + lb;
  const int nE = coff(E + 1);
  const int nBc = coff(lb + 1);
  std::vector<double> Vt((size_t)(E + 1) * nE), acc(nE, 0.0), br((size_t)nE * nBc);
  for (int i = 0; i < B.nprim[sa]; ++i)
    for (int j = 0; j < B.nprim[sb]; ++j) {
      const double al = B.exps[B.prim0[sa] + i], be = B.exps[B.prim0[sb] + j];
      const double w = B.wts[B.prim0[sa] + i] * B.wts[B.prim0[sb] + j];
      const double p = al + be, mu = al * be / p;
      double P[3], PA[3], PB[3];
      for (int k = 0; k < 3; ++k) {
        P[k] = (al * A[k] + be * Bc[k]) / p;
        PA[k] = P[k] - A[k];
        PB[k] = P[k] - Bc[k];
      }
      // 1-D overlaps up to (la, lb + 2)
      double Sd[3][kLmax + 2][kLmax + 4];
      for (int d = 0; d < 3; ++d) {
        Sd[d][0][0] = std::sqrt(kPiRef / p) * std::exp(-mu * AB[d] * AB[d]);
        for (int ii = 0; ii <= la + 1; ++ii)
          for (int jj = 0; jj <= lb + 2; ++jj) {
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
      for (int ia = 0; ia < na; ++ia)
        for (int ib = 0; ib < nb; ++ib) {
          const int ea[3] = {ct[la][ia].x, ct[la][ia].y, ct[la][ia].z};
          const int eb[3] = {ct[lb][ib].x, ct[lb][ib].y, ct[lb][ib].z};
          const double sx = Sd[0][ea[0]][eb[0]], sy = Sd[1][ea[1]][eb[1]], sz = Sd[2][ea[2]][eb[2]];
          out.S[ia * nb + ib] += w * sx * sy * sz;
          double t = 0.0;
          for (int d = 0; d < 3; ++d) {
            const int jj = eb[d], ii = ea[d];
            double k = -2.0 * be * (2 * jj + 1) * Sd[d][ii][jj] + 4.0 * be * be * Sd[d][ii][jj + 2];
            if (jj > 1) k += jj * (jj - 1) * Sd[d][ii][jj - 2];
            double o = 1.0;
            for (int d2 = 0; d2 < 3; ++d2)
              if (d2 != d) o *= Sd[d2][ea[d2]][eb[d2]];
            t += -0.5 * k * o;
          }
          out.T[ia * nb + ib] += w * t;
        }
      // nuclear attraction
      const double pref = 2.0 * kPiRef / p * std::exp(-mu * AB2) * w;
      for (int c = 0; c < natom; ++c) {
        const double* C = &xyz[3 * c];
        double PC[3] = {P[0] - C[0], P[1] - C[1], P[2] - C[2]};
        const double x = p * (PC[0] * PC[0] + PC[1] * PC[1] + PC[2] * PC[2]);
        for (int m = 0; m <= E; ++m) Vt[(size_t)m * nE] = pref * boys_ref_host(x, (unsigned)m);
        for (int e = 1; e <= E; ++e)
          for (const Cart3& q : ct[e]) {
            int em[3] = {q.x, q.y, q.z};
            const int dir = q.x ? 0 : (q.y ? 1 : 2);
            em[dir] -= 1;
            const int i1 = call_idx(em[0], em[1], em[2]);
            int i2 = -1;
            if (em[dir] > 0) {
              int e2[3] = {em[0], em[1], em[2]};
              e2[dir] -= 1;
              i2 = call_idx(e2[0], e2[1], e2[2]);
            }
            const int it = call_idx(q.x, q.y, q.z);
            for (int m = 0; m <= E - e; ++m) {
              double v = PA[dir] * Vt[(size_t)m * nE + i1] - PC[dir] * Vt[(size_t)(m + 1) * nE + i1];
              if (i2 >= 0) v += em[dir] / (2.0 * p) * (Vt[(size_t)m * nE + i2] - Vt[(size_t)(m + 1) * nE + i2]);
              Vt[(size_t)m * nE + it] = v;
            }
          }
        for (int e = 0; e < nE; ++e) acc[e] += -(double)Z[c] * Vt[e];
      }
    }
  // horizontal transfer of the accumulated nuclear integrals
  for (int e = 0; e < nE; ++e) br[(size_t)e * nBc] = acc[e];
  for (int bd = 1; bd <= lb; ++bd)
    for (const Cart3& q : ct[bd]) {
      int bm[3] = {q.x, q.y, q.z};
      const int dir = q.x ? 0 : (q.y ? 1 : 2);
      bm[dir] -= 1;
      const int ibm = call_idx(bm[0], bm[1], bm[2]), ibt = call_idx(q.x, q.y, q.z);
      for (int ed = 0; ed <= E - bd; ++ed)
        for (const Cart3& r : ct[ed]) {
          int ec[3] = {r.x, r.y, r.z};
          const int ie = call_idx(r.x, r.y, r.z);
          ec[dir] += 1;
          const int iep = call_idx(ec[0], ec[1], ec[2]);
          br[(size_t)ie * nBc + ibt] = br[(size_t)iep * nBc + ibm] + AB[dir] * br[(size_t)ie * nBc + ibm];
        }
    }
  for (int ia = 0; ia < na; ++ia)
    for (int ib = 0; ib < nb; ++ib)
      out.V[ia * nb + ib] = br[(size_t)(coff(la) + ia) * nBc + coff(lb) + ib];
}

}  // namespace

extern "C" int dss_one_electron(dss_ctx* ctx, int natom, const int* Z, const double* xyz_bohr, double* S_packed,
                                double* T_packed, double* V_packed, double* e_nuc) {
  if (!ctx) return DSS_ERR_INVALID;
  ctx->err.clear();
  if (!ctx->nbf || ctx->nmol > 0) return dss_fail(ctx, DSS_ERR_INVALID, "dss_one_electron: no single-molecule basis set");
  if (natom < 0 || (natom > 0 && (!Z || !xyz_bohr)))
    return dss_fail(ctx, DSS_ERR_INVALID, "dss_one_electron: bad atom arrays");
  std::string err;
  const int rc = dss_one_electron_basis(ctx->basis, natom, Z, xyz_bohr, S_packed, T_packed, V_packed, e_nuc, &err);
  if (rc != DSS_OK) return dss_fail(ctx, rc, err);
  return DSS_OK;
}

int dss_one_electron_basis(const BasisHost& B, int natom, const int* Z, const double* xyz_bohr, double* S_packed,
                           double* T_packed, double* V_packed, double* e_nuc, std::string* errp) {
  const int ns = (int)B.l.size();
  for (int s = 0; s < ns; ++s)
    if (B.l[s] > kLmax) {
      if (errp) *errp = "dss_one_electron: l above 4";
      return DSS_ERR_UNSUPPORTED;
    }
  // Function transforms per (l, pure).
  std::vector<std::vector<std::vector<std::pair<int, double>>>> tr(kLmax + 1);
  for (int l = 0; l <= kLmax; ++l) tr[l].resize(B.pure ? 2 * l + 1 : ncart(l));
  for (int t = 0; t < kDssSphTermCount; ++t) {
    const DssSphTerm& q = kDssSphTerms[t];
    if (q.pure == B.pure && q.l <= kLmax) tr[q.l][q.func].push_back({q.cart, q.w});
  }
  const auto ct = cart_tables();
  const int n = B.nbf;
  const size_t np = (size_t)n * (n + 1) / 2;
  std::vector<double> S(np, 0.0), T(np, 0.0), V(np, 0.0);
  // Shell pairs (a >= b) split over host threads.
  std::vector<std::pair<int, int>> pairs;
  for (int a = 0; a < ns; ++a)
    for (int b = 0; b <= a; ++b) pairs.push_back({a, b});
  unsigned nth = std::thread::hardware_concurrency();
  if (nth == 0) nth = 1;
  if (nth > 32) nth = 32;
  auto work = [&](unsigned tid) {
    PairOut po;
    for (size_t k = tid; k < pairs.size(); k += nth) {
      const int sa = pairs[k].first, sb = pairs[k].second;
      pair_integrals(B, sa, sb, natom, Z, xyz_bohr, ct, po);
      const int la = B.l[sa], lb = B.l[sb];
      const int nca = ncart(la), ncb = ncart(lb);
      const auto& ta = tr[la];
      const auto& tb = tr[lb];
      for (size_t fa = 0; fa < ta.size(); ++fa)
        for (size_t fb = 0; fb < tb.size(); ++fb) {
          const int i = B.f0[sa] + (int)fa, j = B.f0[sb] + (int)fb;
          if (sa == sb && j > i) continue;
          double s = 0.0, t = 0.0, v = 0.0;
          for (const auto& xa : ta[fa])
            for (const auto& xb : tb[fb]) {
              const double wgt = xa.second * xb.second;
              const int q = xa.first * ncb + xb.first;
              s += wgt * po.S[q];
              t += wgt * po.T[q];
              v += wgt * po.V[q];
            }
          (void)nca;
          const int x = i > j ? i : j, y = i > j ? j : i;
          const size_t idx = (size_t)x * (x + 1) / 2 + y;
          S[idx] = s;
          T[idx] = t;
          V[idx] = v;
        }
    }
  };
  std::vector<std::thread> th;
  for (unsigned t = 1; t < nth; ++t) th.emplace_back(work, t);
  work(0);
  for (auto& t : th) t.join();
  if (S_packed) std::memcpy(S_packed, S.data(), np * 8);
  if (T_packed) std::memcpy(T_packed, T.data(), np * 8);
  if (V_packed) std::memcpy(V_packed, V.data(), np * 8);
  if (e_nuc) {
    // sum_{A<B} Z_A Z_B / R_AB (chem/scf/Energy.cpp:44-49)
    double e = 0.0;
    for (int i = 0; i < natom; ++i)
      for (int j = i + 1; j < natom; ++j) {
        const double dx = xyz_bohr[3 * i] - xyz_bohr[3 * j], dy = xyz_bohr[3 * i + 1] - xyz_bohr[3 * j + 1],
                     dz = xyz_bohr[3 * i + 2] - xyz_bohr[3 * j + 2];
        e += (double)Z[i] * Z[j] / std::sqrt(dx * dx + dy * dy + dz * dz);
      }
    *e_nuc = e;
  }
  return DSS_OK;
}
