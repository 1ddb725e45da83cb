// Nuclear gradient of the last RHF/UHF solve in a context, the quantity of the
// reference's scf::getEnergyGradient (chem/scf/Gradient.cpp:14-133, with the
// two-electron part of chem/scf/ExactCoulomb.cpp:125-195):
//
//   dE/dR = sum D_mn dH_mn/dR + 1/2 sum Gamma dERI/dR - sum W_mn dS_mn/dR + dV_nn/dR
//
// with the density D, the energy-weighted density W = sum_s sum_occ eps_i C_i C_i^T
// (RHF: twice the alpha sum) and the two-particle density of the converged
// determinant.  The two-electron term is analytic: derivative ERIs fused with the
// two-particle-density digest on the device (dss_eri_gradient_dense,
// eri_gradient.cu).  The one-electron terms are analytic too
// (dss_one_electron_gradient: shifted overlap, kinetic and nuclear-attraction
// integrals contracted with D and W, Hellmann-Feynman term included), and the
// nuclear repulsion's derivative is added on the host.  With step > 0 the
// one-electron terms are instead central differences of step bohr of the device
// one-electron integrals at fixed D and W (6 natom evaluations; a cross-check).
#include <algorithm>
#include <cmath>
#include <string>
#include <vector>

#include "dss.h"
#include "dss_internal.h"

namespace {

// tr(A X) for dense symmetric A (n x n) and packed-upper X.
double trace_dense_packed(const std::vector<double>& A, const std::vector<double>& Xp, int n) {
  double s = 0.0;
  for (int j = 0; j < n; ++j)
    for (int i = 0; i <= j; ++i) {
      const double x = Xp[(size_t)j * (j + 1) / 2 + i];
      s += (i == j ? 1.0 : 2.0) * A[(size_t)i * n + j] * x;
    }
  return s;
}

}  // namespace

extern "C" int dss_gradient(dss_ctx* ctx, int natom, const int* Z, const double* xyz_bohr, double step,
                            double* grad) {
  if (!ctx) return DSS_ERR_INVALID;
  ctx->err.clear();
  if (natom <= 0 || !Z || !xyz_bohr || !grad || !(step >= 0.0))
    return dss_fail(ctx, DSS_ERR_INVALID, "dss_gradient: empty molecule, NULL array or negative step");
  if (ctx->last_spins == 0 || ctx->nmol > 0)
    return dss_fail(ctx, DSS_ERR_INVALID, "dss_gradient: no solved single molecule in this context");
  const BasisHost& B0 = ctx->basis;
  const int n = B0.nbf;
  const int ns = (int)B0.l.size();
  const size_t n2 = (size_t)n * n;
  if (ctx->last_C[0].size() != n2) return dss_fail(ctx, DSS_ERR_INVALID, "dss_gradient: orbitals do not match the basis");
  const bool uhf = ctx->last_spins == 2;
  // Shell -> nucleus by centre.
  std::vector<int> owner(ns, -1);
  for (int s = 0; s < ns; ++s)
    for (int a = 0; a < natom && owner[s] < 0; ++a)
      if (B0.xyz[3 * s] == xyz_bohr[3 * a] && B0.xyz[3 * s + 1] == xyz_bohr[3 * a + 1] &&
          B0.xyz[3 * s + 2] == xyz_bohr[3 * a + 2])
        owner[s] = a;
  for (int s = 0; s < ns; ++s)
    if (owner[s] < 0) return dss_fail(ctx, DSS_ERR_INVALID, "dss_gradient: a shell centre is not on any nucleus");
  // Spin densities and the energy-weighted density from the last orbitals.
  std::vector<double> Ds[2], Dt(n2, 0.0), W(n2, 0.0);
  for (int sp = 0; sp < (uhf ? 2 : 1); ++sp) {
    const std::vector<double>& C = ctx->last_C[sp];
    const std::vector<double>& eps = ctx->last_eps[sp];
    const int nocc = ctx->last_nocc[sp];
    const double occ = uhf ? 1.0 : 2.0;
    Ds[sp].assign(n2, 0.0);
    for (int i = 0; i < n; ++i)
      for (int j = 0; j < n; ++j) {
        double d = 0.0, w = 0.0;
        for (int k = 0; k < nocc; ++k) {
          const double c = C[(size_t)i * n + k] * C[(size_t)j * n + k];
          d += c;
          w += eps[k] * c;
        }
        Ds[sp][(size_t)i * n + j] = d;
        Dt[(size_t)i * n + j] += occ * d;
        W[(size_t)i * n + j] += occ * w;
      }
  }
  cudaStream_t s = ctx->stream;
  DevBuf<double> dmat, pk;
  if (dmat.resize(3 * n2) != cudaSuccess || pk.resize((size_t)n * (n + 1)) != cudaSuccess)
    return dss_fail(ctx, DSS_ERR_OOM, "dss_gradient: device allocation failed");
  double* dDt = dmat.ptr;
  double* dDa = dmat.ptr + n2;
  double* dDb = dmat.ptr + 2 * n2;
  cudaError_t e = cudaMemcpyAsync(dDt, Dt.data(), n2 * 8, cudaMemcpyHostToDevice, s);
  if (uhf && e == cudaSuccess) e = cudaMemcpyAsync(dDa, Ds[0].data(), n2 * 8, cudaMemcpyHostToDevice, s);
  if (uhf && e == cudaSuccess) e = cudaMemcpyAsync(dDb, Ds[1].data(), n2 * 8, cudaMemcpyHostToDevice, s);
  if (e != cudaSuccess) return dss_fail(ctx, DSS_ERR_CUDA, std::string("dss_gradient: ") + cudaGetErrorString(e));
  // Two-electron part: analytic.
  std::vector<double> g2(3 * (size_t)natom, 0.0);
  int rc = uhf ? dss_eri_gradient_dense(ctx, dDt, dDa, dDb, 0.5, natom, owner.data(), g2.data())
           : dss_eri_gradient_dense(ctx, dDt, dDt, nullptr, 0.25, natom, owner.data(), g2.data());
  if (rc != DSS_OK) return rc;
  if (step == 0.0) {
    // One-electron part analytic, nuclear repulsion on the host.
    DevBuf<double> dW;
    if (dW.resize(n2) != cudaSuccess) return dss_fail(ctx, DSS_ERR_OOM, "dss_gradient: device allocation failed");
    e = cudaMemcpyAsync(dW.ptr, W.data(), n2 * 8, cudaMemcpyHostToDevice, s);
    if (e != cudaSuccess) return dss_fail(ctx, DSS_ERR_CUDA, std::string("dss_gradient: ") + cudaGetErrorString(e));
    std::vector<double> g1(3 * (size_t)natom, 0.0);
    std::string err;
    rc = dss_one_electron_gradient(s, B0, natom, Z, xyz_bohr, owner.data(), dDt, dW.ptr, g1.data(), &err,
                                   &ctx->oe_scratch);
    if (rc != DSS_OK) return dss_fail(ctx, rc, "dss_gradient: " + err);
    for (int a = 0; a < natom; ++a)
      for (int d = 0; d < 3; ++d) {
        // d/dR_a of sum_{b<c} Z_b Z_c / R_bc (chem/scf/Gradient.cpp:118-130)
        double vn = 0.0;
        for (int b = 0; b < natom; ++b) {
          if (b == a) continue;
          const double rx = xyz_bohr[3 * a] - xyz_bohr[3 * b], ry = xyz_bohr[3 * a + 1] - xyz_bohr[3 * b + 1],
                       rz = xyz_bohr[3 * a + 2] - xyz_bohr[3 * b + 2];
          const double r = std::sqrt(rx * rx + ry * ry + rz * rz);
          vn -= (double)Z[a] * Z[b] * (xyz_bohr[3 * a + d] - xyz_bohr[3 * b + d]) / (r * r * r);
        }
        grad[3 * a + d] = g1[3 * a + d] + vn + g2[3 * a + d];
      }
    return DSS_OK;
  }
  // One-electron part: E_1(R) = tr(D H(R)) - tr(W S(R)) + V_nn(R) at displaced nuclei.
  const size_t np = (size_t)n * (n + 1) / 2;
  std::vector<double> Sp(np), Hp(np);
  std::vector<double> xyz(xyz_bohr, xyz_bohr + 3 * (size_t)natom);
  auto energy1 = [&](int a, int d, double delta, double* E) -> int {
    BasisHost B = B0;
    for (int q = 0; q < ns; ++q)
      if (owner[q] == a) B.xyz[3 * q + d] += delta;
    xyz[3 * a + d] = xyz_bohr[3 * a + d] + delta;
    std::string err;
    int r = dss_one_electron_device(s, B, natom, Z, xyz.data(), pk.ptr, pk.ptr + np, nullptr, &err, &ctx->oe_scratch);
    if (r != DSS_OK) return dss_fail(ctx, r, "dss_gradient: one-electron integrals: " + err);
    cudaError_t ce = cudaMemcpyAsync(Sp.data(), pk.ptr, np * 8, cudaMemcpyDeviceToHost, s);
    if (ce == cudaSuccess) ce = cudaMemcpyAsync(Hp.data(), pk.ptr + np, np * 8, cudaMemcpyDeviceToHost, s);
    if (ce == cudaSuccess) ce = cudaStreamSynchronize(s);
    if (ce != cudaSuccess) return dss_fail(ctx, DSS_ERR_CUDA, std::string("dss_gradient: ") + cudaGetErrorString(ce));
    *E = trace_dense_packed(Dt, Hp, n) - trace_dense_packed(W, Sp, n) + dss_nuclear_repulsion(natom, Z, xyz.data());
    xyz[3 * a + d] = xyz_bohr[3 * a + d];
    return DSS_OK;
  };
  for (int a = 0; a < natom; ++a)
    for (int d = 0; d < 3; ++d) {
      double Ep = 0.0, Em = 0.0;
      rc = energy1(a, d, step, &Ep);
      if (rc == DSS_OK) rc = energy1(a, d, -step, &Em);
      if (rc != DSS_OK) return rc;
      grad[3 * a + d] = (Ep - Em) / (2.0 * step) + g2[3 * a + d];
    }
  return DSS_OK;
}
