// Drop-in replacement for DollarStoreSCF's chem/scf/ExactCoulomb.cpp: the same
// four functions (chem/scf/ExactCoulomb.hpp:9-15), backed by the B200 engine
// through the C ABI (include/dss.h).  Link this file instead of ExactCoulomb.cpp
// and add libdss.so; no other reference file changes.
//
//   assignExactRepulsionTensor()  (ExactCoulomb.cpp:41-72): instead of storing
//       the N^4/8 tensor, packs scf::basis into shells and hands them to the
//       engine, which computes Schwarz factors and screened work lists on the
//       GPU (direct SCF: integrals are recomputed per Fock build).
//   getExactCoulombMatrix(mu, nu)  (:103-112) and
//   getExactExchangeMatrix(mu, nu, spin)  (:114-123): the reference's callers
//       (computeCoulombTerms / computeExchangeTerms, SCFSolver.cpp:29-43, and
//       calculateEnergies, Energy.cpp:26-36) sweep mu from 0 and nu from mu, so
//       the first request of every sweep is (0, 0).  On that request the shim
//       runs one GPU build from the current density (scf::total_density_matrix
//       for J, scf::density_matrix[spin] for K) and then serves elements from
//       the cached matrices.  For RHF the exchange of D_alpha is K[D_total]/2,
//       so one build per Fock matrix serves both sweeps.
//   addExactTwoElectronGradient(v)  (:125-195): adds the analytic four-centre
//       term of dss_eri_gradient (derivative ERIs digested with the two-particle
//       density of scf::total_density_matrix and, for UHF, density_matrix[0/1])
//       to v, with the nucleus of each shell from scf::basis_atoms.
//
// Errors follow the reference's convention (lalib/Lapack.cpp:33-38): a message
// on stderr and the run continues; the affected matrix elements read as NaN.
#include <cmath>
#include <cstdlib>
#include <iostream>
#include <limits>
#include <vector>

#include "chem/scf/ExactCoulomb.hpp"
#include "chem/scf/SCFCommon.hpp"
#include "dss.h"

namespace {

dss_ctx* g_ctx = nullptr;
int g_n = 0;
std::vector<double> g_J, g_K[2];  // packed-U caches
bool g_k_from_total = false;      // g_K[0] holds K[D_total]/2 from the last Coulomb build
std::vector<double> g_Dp, g_Jtmp, g_Ktmp;
std::vector<int> g_shell_f0;  // first basis function of each shell

const double kNaN = std::numeric_limits<double>::quiet_NaN();

size_t pidx(uint y, uint x) {
  if (y > x) std::swap(x, y);
  return (size_t)x * (x + 1) / 2 + y;
}

void report(const char* what) {
  std::cerr << "ERROR (GPU Fock build): " << what << ": " << dss_last_error(g_ctx) << '\n';
}

void pack_density(const flo::SymmetricMatrixNd& D) {
  g_Dp.resize((size_t)g_n * (g_n + 1) / 2);
  for (uint x = 0; x < (uint)g_n; ++x)
    for (uint y = 0; y <= x; ++y) g_Dp[pidx(y, x)] = D(y, x);
}

bool same_shell(const flo::ContractedGaussian& a, const flo::ContractedGaussian& b) {
  if (a.l != b.l || a.primitives.size() != b.primitives.size()) return false;
  if (a.center.x != b.center.x || a.center.y != b.center.y || a.center.z != b.center.z) return false;
  for (size_t p = 0; p < a.primitives.size(); ++p)
    if (a.primitives[p].zeta != b.primitives[p].zeta ||
        a.primitives[p].unnormalized_weight != b.primitives[p].unnormalized_weight)
      return false;
  return true;
}

}  // namespace

namespace scf {

void assignExactRepulsionTensor() {
  if (!g_ctx) {
    dss_opts o;
    dss_default_opts(&o);
    if (const char* dev = std::getenv("DSS_DEVICE")) o.device = std::atoi(dev);
    if (const char* thr = std::getenv("DSS_SCHWARZ")) o.schwarz_threshold = std::atof(thr);
    if (dss_create(&g_ctx, &o) != DSS_OK) {
      std::cerr << "ERROR (GPU Fock build): " << dss_last_error(nullptr) << '\n';
      g_ctx = nullptr;
      return;
    }
  }
  // scf::basis holds 2l+1 consecutive functions per shell (SCFBasis.cpp:129-136).
  std::vector<int> l, nprim;
  std::vector<double> exps, coefs, centers;
  g_shell_f0.clear();
  for (size_t f = 0; f < basis.size();) {
    const flo::ContractedGaussian& g = basis[f];
    size_t e = f + 1;
    while (e < basis.size() && e - f < 2 * g.l + 1 && same_shell(basis[e], g)) ++e;
    g_shell_f0.push_back((int)f);
    l.push_back((int)g.l);
    nprim.push_back((int)g.primitives.size());
    for (const flo::GTOPrimitive& p : g.primitives) {
      exps.push_back(p.zeta);
      coefs.push_back(p.unnormalized_weight);
    }
    centers.push_back(g.center.x);
    centers.push_back(g.center.y);
    centers.push_back(g.center.z);
    f = e;
  }
  if (dss_set_basis(g_ctx, (int)l.size(), l.data(), nprim.data(), exps.data(), coefs.data(), centers.data(), 1) !=
      DSS_OK) {
    report("dss_set_basis");
    g_n = 0;
    return;
  }
  g_n = dss_nbf(g_ctx);
  g_J.assign((size_t)g_n * (g_n + 1) / 2, kNaN);
  g_K[0] = g_J;
  g_K[1] = g_J;
  g_k_from_total = false;
}

double getExactCoulombMatrix(uint mu, uint nu) {
  if (!g_ctx || !g_n) return kNaN;
  if (mu == 0 && nu == 0) {
    pack_density(total_density_matrix);
    g_Jtmp.resize(g_Dp.size());
    g_Ktmp.resize(g_Dp.size());
    if (dss_build_jk(g_ctx, g_Dp.data(), g_Jtmp.data(), g_Ktmp.data()) != DSS_OK) {
      report("dss_build_jk");
      std::fill(g_J.begin(), g_J.end(), kNaN);
      g_k_from_total = false;
    } else {
      g_J = g_Jtmp;
      if (spin_treatment == SpinTreatment::restricted) {
        // D_total = 2 D_alpha exactly (SCFSolver.cpp:92), so K[D_alpha] = K[D_total] / 2.
        for (size_t i = 0; i < g_Ktmp.size(); ++i) g_K[0][i] = 0.5 * g_Ktmp[i];
        g_k_from_total = true;
      } else {
        g_k_from_total = false;
      }
    }
  }
  return g_J[pidx(mu, nu)];
}

double getExactExchangeMatrix(uint mu, uint nu, Spin spin) {
  if (!g_ctx || !g_n) return kNaN;
  const int s = (int)spin;
  if (mu == 0 && nu == 0 && !(s == 0 && g_k_from_total)) {
    pack_density(density_matrix[s]);
    g_Ktmp.resize(g_Dp.size());
    if (dss_build_jk(g_ctx, g_Dp.data(), nullptr, g_Ktmp.data()) != DSS_OK) {
      report("dss_build_jk");
      std::fill(g_K[s].begin(), g_K[s].end(), kNaN);
    } else {
      g_K[s] = g_Ktmp;
    }
  }
  const double v = g_K[s][pidx(mu, nu)];
  // The cache from a Coulomb build serves exactly one exchange sweep.
  if (s == 0 && mu + 1 == (uint)g_n && nu + 1 == (uint)g_n) g_k_from_total = false;
  return v;
}

void addExactTwoElectronGradient(VectorNd& target) {
  if (!g_ctx || !g_n) return;
  const int natom = (int)(target.size() / 3);
  std::vector<int> shell_atom(g_shell_f0.size());
  for (size_t q = 0; q < g_shell_f0.size(); ++q) shell_atom[q] = (int)basis_atoms[g_shell_f0[q]];
  pack_density(total_density_matrix);
  const std::vector<double> Dt = g_Dp;
  std::vector<double> Da, Db;
  if (spin_treatment == SpinTreatment::unrestricted) {
    pack_density(density_matrix[0]);
    Da = g_Dp;
    pack_density(density_matrix[1]);
    Db = g_Dp;
  }
  std::vector<double> g(3 * (size_t)natom, 0.0);
  if (dss_eri_gradient(g_ctx, Dt.data(), Da.empty() ? nullptr : Da.data(), Db.empty() ? nullptr : Db.data(), natom,
                       shell_atom.data(), g.data()) != DSS_OK) {
    report("dss_eri_gradient");
    for (size_t i = 0; i < g.size(); ++i) target[i] = kNaN;
    return;
  }
  for (size_t i = 0; i < g.size(); ++i) target[i] += g[i];
}

}  // namespace scf
