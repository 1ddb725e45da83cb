// Orbital output of a solved molecule: the MO coefficients and energies of the
// last dss_scf_solve / dss_uhf_solve, and a Molden file with the layout of the
// reference's scf::writeOrbitalsMolden (chem/scf/WriteOrbitals.cpp:17-137):
// [Atoms] in bohr, [GTO] with the file's contraction coefficients per atom, [MO]
// with every orbital (or only the occupied ones), alpha then beta, and the
// reference's Molden order of the real solid harmonics inside a shell
// (p: x, y, z; d: m = 0, +1, -1, +2, -2 in Molden's naming), which permutes this
// library's m = -l..l order exactly as the reference permutes its own.
// Numbers are written with more digits than the reference prints.
#include <cmath>
#include <cstdio>
#include <string>
#include <vector>

#include "dss.h"
#include "dss_internal.h"

namespace {

const char* const kSymbols[] = {"H",  "He", "Li", "Be", "B",  "C",  "N",  "O",  "F",  "Ne", "Na", "Mg", "Al", "Si",
                                "P",  "S",  "Cl", "Ar", "K",  "Ca", "Sc", "Ti", "V",  "Cr", "Mn", "Fe", "Co", "Ni",
                                "Cu", "Zn", "Ga", "Ge", "As", "Se", "Br", "Kr"};

// Position inside a shell (m = -l..l order) of the k-th Molden function.
const int kMoldenPerm[3][5] = {{0, 0, 0, 0, 0}, {0, 2, 1, 0, 0}, {2, 1, 3, 0, 4}};
const char kShellLabel[3] = {'s', 'p', 'd'};

}  // namespace

extern "C" {

int dss_scf_orbitals(const dss_ctx* ctx, int spin, double* C, double* eps) {
  if (!ctx || spin < 0 || spin > 1) return DSS_ERR_INVALID;
  if (ctx->last_spins == 0 || (spin == 1 && ctx->last_spins < 2)) return DSS_ERR_INVALID;
  const size_t n = (size_t)ctx->nbf;
  if (ctx->last_C[spin].size() != n * n || ctx->last_eps[spin].size() != n) return DSS_ERR_INVALID;
  if (C)
    for (size_t i = 0; i < n * n; ++i) C[i] = ctx->last_C[spin][i];
  if (eps)
    for (size_t i = 0; i < n; ++i) eps[i] = ctx->last_eps[spin][i];
  return DSS_OK;
}

int dss_write_molden(dss_ctx* ctx, const char* path, int natom, const int* Z, const double* xyz_bohr,
                     int write_virtual) {
  if (!ctx) return DSS_ERR_INVALID;
  ctx->err.clear();
  if (!path || natom <= 0 || !Z || !xyz_bohr)
    return dss_fail(ctx, DSS_ERR_INVALID, "dss_write_molden: NULL path or empty molecule");
  if (ctx->last_spins == 0 || ctx->nmol > 0)
    return dss_fail(ctx, DSS_ERR_INVALID, "dss_write_molden: no solved single molecule in this context");
  const BasisHost& B = ctx->basis;
  if (!B.pure) return dss_fail(ctx, DSS_ERR_UNSUPPORTED, "dss_write_molden: 5D (spherical) bases only, as [5D]");
  const int ns = (int)B.l.size();
  const int n = B.nbf;
  for (int a = 0; a < natom; ++a)
    if (Z[a] < 1 || Z[a] > (int)(sizeof(kSymbols) / sizeof(kSymbols[0])))
      return dss_fail(ctx, DSS_ERR_UNSUPPORTED, "dss_write_molden: element without a symbol here");
  // Shells of each atom: those centred on it, in basis order.
  std::vector<std::vector<int>> atom_shells(natom);
  for (int s = 0; s < ns; ++s) {
    if (B.l[s] > 2) return dss_fail(ctx, DSS_ERR_UNSUPPORTED, "dss_write_molden: l above 2");
    int owner = -1;
    for (int a = 0; a < natom && owner < 0; ++a)
      if (B.xyz[3 * s] == xyz_bohr[3 * a] && B.xyz[3 * s + 1] == xyz_bohr[3 * a + 1] &&
          B.xyz[3 * s + 2] == xyz_bohr[3 * a + 2])
        owner = a;
    if (owner < 0) return dss_fail(ctx, DSS_ERR_INVALID, "dss_write_molden: a shell centre is not on any nucleus");
    atom_shells[owner].push_back(s);
  }
  FILE* f = std::fopen(path, "wb");
  if (!f) return dss_fail(ctx, DSS_ERR_INVALID, std::string("dss_write_molden: cannot open ") + path);
  std::fprintf(f, "[Molden Format]\n[5D]\n[9G]\n[Atoms] AU\n");
  for (int a = 0; a < natom; ++a)
    std::fprintf(f, " %-2s %5d %4d %17.10f %17.10f %17.10f\n", kSymbols[Z[a] - 1], a + 1, Z[a], xyz_bohr[3 * a],
                 xyz_bohr[3 * a + 1], xyz_bohr[3 * a + 2]);
  std::fprintf(f, "[GTO]\n");
  for (int a = 0; a < natom; ++a) {
    std::fprintf(f, "%d 0\n", a + 1);
    for (int s : atom_shells[a]) {
      std::fprintf(f, "%c %d 1.00\n", kShellLabel[B.l[s]], B.nprim[s]);
      for (int p = 0; p < B.nprim[s]; ++p)
        std::fprintf(f, " %20.12E %20.12E\n", B.exps[B.prim0[s] + p], B.coefs[B.prim0[s] + p]);
    }
    std::fprintf(f, "\n");
  }
  std::fprintf(f, "[MO]\n");
  const bool unrestricted = ctx->last_spins == 2;
  for (int sp = 0; sp < (unrestricted ? 2 : 1); ++sp) {
    const int nocc = ctx->last_nocc[sp];
    const std::vector<double>& C = ctx->last_C[sp];
    const std::vector<double>& eps = ctx->last_eps[sp];
    const int nmo = write_virtual ? n : nocc;
    for (int i = 0; i < nmo; ++i) {
      const int occ = (i < nocc) ? (unrestricted ? 1 : 2) : 0;
      std::fprintf(f, "Sym=   %c%d\nEne=   %.12f\nSpin=  %s\nOccup= %d\n", sp ? 'b' : 'a', i, eps[i],
                   sp ? "Beta" : "Alpha", occ);
      int ao = 0;
      for (int a = 0; a < natom; ++a)
        for (int s : atom_shells[a])
          for (int m = 0; m <= 2 * B.l[s]; ++m) {
            ++ao;
            const int row = B.f0[s] + kMoldenPerm[B.l[s]][m];
            std::fprintf(f, "%6d %20.12E\n", ao, C[(size_t)row * n + i]);
          }
    }
  }
  const bool ok = std::fclose(f) == 0;
  if (!ok) return dss_fail(ctx, DSS_ERR_INVALID, "dss_write_molden: write failed");
  return DSS_OK;
}

}  // extern "C"
