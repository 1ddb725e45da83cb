// Nuclear gradient of the last RHF/UHF solve in a context, the quantity of the
// reference's scf::getEnergyGradient (chem/scf/Gradient.cpp:14-133, with the
// two-electron part of chem/scf/ExactCoulomb.cpp:125-195):
//
//   dE/dR = sum D_mn dH_mn/dR + 1/2 sum Gamma dERI/dR - sum W_mn dS_mn/dR + dV_nn/dR
//
// with the density D, the energy-weighted density W = sum_s sum_occ eps_i C_i C_i^T
// (RHF: twice the alpha sum) and the two-particle density of the converged
// determinant.  Every term differentiates integrals at fixed D and W, so this
// function evaluates the fixed-density expression
//
//   E_fix(R) = tr(D H(R)) + E_2e[D](R) - tr(W S(R)) + V_nn(R)
//
// at R +- h along each nuclear coordinate (the basis functions move with their
// nucleus) with the device one-electron kernels and one device J/K build per
// point, and takes the central difference.  It is not an analytic derivative:
// the truncation error is O(h^2) (h = 1e-4 bohr: ~1e-9 Eh/bohr), and each point
// costs a basis set-up and a build (6 natom of them).
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

// tr(A (Acc + Acc^T)) for dense A (symmetric) and an accumulator Acc.
double trace_sym_acc(const std::vector<double>& A, const std::vector<double>& acc, int n) {
  double s = 0.0;
  for (size_t t = 0; t < (size_t)n * n; ++t) s += 2.0 * A[t] * acc[t];
  return s;
}

}  // namespace

extern "C" int dss_gradient(dss_ctx* ctx, int natom, const int* Z, const double* xyz_bohr, double step,
                            double* grad) {
  if (!ctx) return DSS_ERR_INVALID;
  ctx->err.clear();
  if (natom <= 0 || !Z || !xyz_bohr || !grad || !(step > 0.0))
    return dss_fail(ctx, DSS_ERR_INVALID, "dss_gradient: empty molecule, NULL array or step <= 0");
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
  // A private context for the displaced geometries (the caller's basis stays).
  dss_opts o = ctx->opts;
  o.schwarz_threshold = std::min(o.schwarz_threshold, 1e-15);  // no quartet flips in or out between points
  dss_ctx* g = nullptr;
  int rc = dss_create(&g, &o);
  if (rc != DSS_OK) return dss_fail(ctx, rc, std::string("dss_gradient: ") + dss_last_error(nullptr));
  struct Guard {
    dss_ctx* c;
    ~Guard() { dss_destroy(c); }
  } guard{g};
  cudaStream_t s = g->stream;
  DevBuf<double> dmat, acc, pk;
  if (dmat.resize(3 * n2) != cudaSuccess || acc.resize(3 * n2) != cudaSuccess ||
      pk.resize((size_t)n * (n + 1)) != cudaSuccess)
    return dss_fail(ctx, DSS_ERR_OOM, "dss_gradient: device allocation failed");
  double* dDt = dmat.ptr;
  double* dDa = dmat.ptr + n2;
  double* dDb = dmat.ptr + 2 * n2;
  cudaError_t e = cudaMemcpyAsync(dDt, Dt.data(), n2 * 8, cudaMemcpyHostToDevice, s);
  if (uhf && e == cudaSuccess) e = cudaMemcpyAsync(dDa, Ds[0].data(), n2 * 8, cudaMemcpyHostToDevice, s);
  if (uhf && e == cudaSuccess) e = cudaMemcpyAsync(dDb, Ds[1].data(), n2 * 8, cudaMemcpyHostToDevice, s);
  if (e != cudaSuccess) return dss_fail(ctx, DSS_ERR_CUDA, std::string("dss_gradient: ") + cudaGetErrorString(e));
  const size_t np = (size_t)n * (n + 1) / 2;
  std::vector<double> Sp(np), Hp(np), Jh(n2), Kh(n2), K2h(n2);
  std::vector<double> xyz(xyz_bohr, xyz_bohr + 3 * (size_t)natom);
  // E_fix at the geometry with nucleus a moved by delta along axis d.
  auto energy = [&](int a, int d, double delta, double* E) -> int {
    BasisHost B = B0;
    for (int q = 0; q < ns; ++q)
      if (owner[q] == a) B.xyz[3 * q + d] += delta;
    xyz[3 * a + d] = xyz_bohr[3 * a + d] + delta;
    int r = dss_setup_pairs(g, std::move(B));
    if (r != DSS_OK) return r;
    std::string err;
    r = dss_one_electron_device(s, g->basis, natom, Z, xyz.data(), pk.ptr, pk.ptr + np, nullptr, &err, &g->oe_scratch);
    if (r != DSS_OK) return r;
    BuildMode m;
    m.boys = o.boys_mode;
    if (uhf && o.boys_mode == DSS_BOYS_REF) {
      m.uhf = true;
      m.Da = dDa;
      m.Db = dDb;
      m.K2 = acc.ptr + 2 * n2;
    }
    r = dss_enqueue_jk(g, uhf && !m.uhf ? dDa : dDt, acc.ptr, acc.ptr + n2, nullptr, &m);
    if (r != DSS_OK) return r;
    cudaError_t ce = cudaMemcpyAsync(Sp.data(), pk.ptr, np * 8, cudaMemcpyDeviceToHost, s);
    if (ce == cudaSuccess) ce = cudaMemcpyAsync(Hp.data(), pk.ptr + np, np * 8, cudaMemcpyDeviceToHost, s);
    if (ce == cudaSuccess) ce = cudaMemcpyAsync(Jh.data(), acc.ptr, n2 * 8, cudaMemcpyDeviceToHost, s);
    if (ce == cudaSuccess) ce = cudaMemcpyAsync(Kh.data(), acc.ptr + n2, n2 * 8, cudaMemcpyDeviceToHost, s);
    if (uhf && m.uhf && ce == cudaSuccess)
      ce = cudaMemcpyAsync(K2h.data(), acc.ptr + 2 * n2, n2 * 8, cudaMemcpyDeviceToHost, s);
    if (ce == cudaSuccess) ce = cudaStreamSynchronize(s);
    if (ce != cudaSuccess) return DSS_ERR_CUDA;
    double E2;
    if (!uhf) {
      // J[Dt], K[Dt]: E_2e = tr(Dt J)/2 - tr(Dt K)/4.
      E2 = 0.5 * trace_sym_acc(Dt, Jh, n) - 0.25 * trace_sym_acc(Dt, Kh, n);
    } else if (m.uhf) {
      // J[Dt], K[Da], K[Db]: E_2e = tr(Dt J)/2 - (tr(Da Ka) + tr(Db Kb))/2.
      E2 = 0.5 * trace_sym_acc(Dt, Jh, n) - 0.5 * (trace_sym_acc(Ds[0], Kh, n) + trace_sym_acc(Ds[1], K2h, n));
    } else {
      // Accurate Boys mode: J and K of each spin from two builds.
      const std::vector<double> Ja = Jh, Ka = Kh;
      r = dss_enqueue_jk(g, dDb, acc.ptr, acc.ptr + n2, nullptr, &m);
      if (r != DSS_OK) return r;
      ce = cudaMemcpyAsync(Jh.data(), acc.ptr, n2 * 8, cudaMemcpyDeviceToHost, s);
      if (ce == cudaSuccess) ce = cudaMemcpyAsync(Kh.data(), acc.ptr + n2, n2 * 8, cudaMemcpyDeviceToHost, s);
      if (ce == cudaSuccess) ce = cudaStreamSynchronize(s);
      if (ce != cudaSuccess) return DSS_ERR_CUDA;
      E2 = 0.5 * (trace_sym_acc(Dt, Ja, n) + trace_sym_acc(Dt, Jh, n)) -
           0.5 * (trace_sym_acc(Ds[0], Ka, n) + trace_sym_acc(Ds[1], Kh, n));
    }
    *E = trace_dense_packed(Dt, Hp, n) + E2 - trace_dense_packed(W, Sp, n) +
         dss_nuclear_repulsion(natom, Z, xyz.data());
    xyz[3 * a + d] = xyz_bohr[3 * a + d];
    return DSS_OK;
  };
  for (int a = 0; a < natom; ++a)
    for (int d = 0; d < 3; ++d) {
      double Ep = 0.0, Em = 0.0;
      rc = energy(a, d, step, &Ep);
      if (rc == DSS_OK) rc = energy(a, d, -step, &Em);
      if (rc != DSS_OK) return dss_fail(ctx, rc, std::string("dss_gradient: displaced point failed: ") + g->err);
      grad[3 * a + d] = (Ep - Em) / (2.0 * step);
    }
  return DSS_OK;
}
