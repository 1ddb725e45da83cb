// Orbital output of a solved molecule: the MO coefficients and energies of the
// last dss_scf_solve / dss_uhf_solve, and a Molden file with the layout of the
// reference's scf::writeOrbitalsMolden (chem/scf/WriteOrbitals.cpp:17-137):
// [Atoms] in bohr, [GTO] with the file's contraction coefficients per atom, [MO]
// with every orbital (or only the occupied ones), alpha then beta, and the
// reference's Molden order of the real solid harmonics inside a shell
// (p: x, y, z; d: m = 0, +1, -1, +2, -2 in Molden's naming), which permutes this
// library's m = -l..l order exactly as the reference permutes its own.
// Numbers are written with more digits than the reference prints.
//
// The WFX file (dss_write_wfx) has the sections of the reference's
// scf::writeOrbitalsWFX (chem/scf/WriteOrbitals.cpp:139-458): every contracted
// shell expanded into unnormalised Cartesian primitives x^a y^b z^c exp(-zeta r^2)
// per atom, in the WFX type order (s; x, y, z; xx, yy, zz, xy, xz, yz), and each
// orbital's coefficient on each primitive = sum over the shell's functions of
// C(function, orbital) x solid-harmonic term weight x normalised primitive weight.
#include <cmath>
#include <cstdio>
#include <string>
#include <vector>

#include "dss.h"
#include "dss_internal.h"
#include "sph_tab.h"

namespace {

const char* const kSymbols[] = {"H",  "He", "Li", "Be", "B",  "C",  "N",  "O",  "F",  "Ne", "Na", "Mg", "Al", "Si",
                                "P",  "S",  "Cl", "Ar", "K",  "Ca", "Sc", "Ti", "V",  "Cr", "Mn", "Fe", "Co", "Ni",
                                "Cu", "Zn", "Ga", "Ge", "As", "Se", "Br", "Kr"};

// Position inside a shell (m = -l..l order) of the k-th Molden function.
const int kMoldenPerm[3][5] = {{0, 0, 0, 0, 0}, {0, 2, 1, 0, 0}, {2, 1, 3, 0, 4}};
const char kShellLabel[3] = {'s', 'p', 'd'};

// WFX primitive types of l = 0..2 (1-based type = kWfxType0[l] + position):
// the Cartesian exponents at each position of the format's order.
const int kWfxType0[3] = {1, 2, 5};
const int kWfxCart[3][6][3] = {{{0, 0, 0}},
                               {{1, 0, 0}, {0, 1, 0}, {0, 0, 1}},
                               {{2, 0, 0}, {0, 2, 0}, {0, 0, 2}, {1, 1, 0}, {1, 0, 1}, {0, 1, 1}}};

// Exponents of this library's Cartesian index c of angular momentum l (x-major order).
void cart_exponents(int l, int c, int* a, int* b, int* z) {
  int i = 0;
  for (int x = l; x >= 0; --x)
    for (int y = l - x; y >= 0; --y, ++i)
      if (i == c) {
        *a = x;
        *b = y;
        *z = l - x - y;
        return;
      }
}

// Shells of each atom (those centred on it, in basis order); false if a shell
// centre is on no nucleus.
bool shells_by_atom(const BasisHost& B, int natom, const double* xyz, std::vector<std::vector<int>>* out) {
  out->assign(natom, {});
  for (int s = 0; s < (int)B.l.size(); ++s) {
    int owner = -1;
    for (int a = 0; a < natom && owner < 0; ++a)
      if (B.xyz[3 * s] == xyz[3 * a] && B.xyz[3 * s + 1] == xyz[3 * a + 1] && B.xyz[3 * s + 2] == xyz[3 * a + 2])
        owner = a;
    if (owner < 0) return false;
    (*out)[owner].push_back(s);
  }
  return true;
}

// Writes vals `per` to a line in right-aligned columns (the reference's layout).
void write_rows(FILE* f, const std::vector<double>& vals, int per, const char* fmt) {
  for (size_t i = 0; i < vals.size(); ++i) {
    std::fprintf(f, fmt, vals[i]);
    if (i % per == (size_t)per - 1 || i + 1 == vals.size()) std::fputc('\n', f);
  }
}

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
  for (int s = 0; s < ns; ++s)
    if (B.l[s] > 2) return dss_fail(ctx, DSS_ERR_UNSUPPORTED, "dss_write_molden: l above 2");
  std::vector<std::vector<int>> atom_shells;
  if (!shells_by_atom(B, natom, xyz_bohr, &atom_shells))
    return dss_fail(ctx, DSS_ERR_INVALID, "dss_write_molden: a shell centre is not on any nucleus");
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

int dss_write_wfx(dss_ctx* ctx, const char* path, int natom, const int* Z, const double* xyz_bohr,
                  int write_virtual) {
  if (!ctx) return DSS_ERR_INVALID;
  ctx->err.clear();
  if (!path || natom <= 0 || !Z || !xyz_bohr)
    return dss_fail(ctx, DSS_ERR_INVALID, "dss_write_wfx: NULL path or empty molecule");
  if (ctx->last_spins == 0 || ctx->nmol > 0)
    return dss_fail(ctx, DSS_ERR_INVALID, "dss_write_wfx: no solved single molecule in this context");
  const BasisHost& B = ctx->basis;
  if (!B.pure) return dss_fail(ctx, DSS_ERR_UNSUPPORTED, "dss_write_wfx: 5D (spherical) bases only");
  const int n = B.nbf;
  int zsum = 0;
  for (int a = 0; a < natom; ++a) {
    if (Z[a] < 1 || Z[a] > (int)(sizeof(kSymbols) / sizeof(kSymbols[0])))
      return dss_fail(ctx, DSS_ERR_UNSUPPORTED, "dss_write_wfx: element without a symbol here");
    zsum += Z[a];
  }
  for (int l : B.l)
    if (l > 2) return dss_fail(ctx, DSS_ERR_UNSUPPORTED, "dss_write_wfx: l above 2");
  std::vector<std::vector<int>> atom_shells;
  if (!shells_by_atom(B, natom, xyz_bohr, &atom_shells))
    return dss_fail(ctx, DSS_ERR_INVALID, "dss_write_wfx: a shell centre is not on any nucleus");
  const bool unrestricted = ctx->last_spins == 2;
  const int na = ctx->last_nocc[0];
  const int nb = unrestricted ? ctx->last_nocc[1] : ctx->last_nocc[0];

  // Primitive list: per atom, per shell, per primitive, per WFX type.
  struct Prim {
    int shell, p, pos;
  };
  std::vector<Prim> prims;
  std::vector<double> centers, types, exps;
  for (int a = 0; a < natom; ++a)
    for (int s : atom_shells[a]) {
      const int l = B.l[s], nc = (l + 1) * (l + 2) / 2;
      for (int p = 0; p < B.nprim[s]; ++p)
        for (int t = 0; t < nc; ++t) {
          prims.push_back({s, p, t});
          centers.push_back(a + 1);
          types.push_back(kWfxType0[l] + t);
          exps.push_back(B.exps[B.prim0[s] + p]);
        }
    }
  // For each shell function (m = -l..l) and WFX position: the solid-harmonic weight.
  double sph[3][5][6] = {};
  for (int t = 0; t < kDssSphTermCount; ++t) {
    const DssSphTerm& q = kDssSphTerms[t];
    if (!q.pure || q.l > 2) continue;
    int x, y, z;
    cart_exponents(q.l, q.cart, &x, &y, &z);
    for (int pos = 0; pos < (q.l + 1) * (q.l + 2) / 2; ++pos)
      if (kWfxCart[q.l][pos][0] == x && kWfxCart[q.l][pos][1] == y && kWfxCart[q.l][pos][2] == z)
        sph[q.l][q.func][pos] += q.w;
  }

  FILE* f = std::fopen(path, "wb");
  if (!f) return dss_fail(ctx, DSS_ERR_INVALID, std::string("dss_write_wfx: cannot open ") + path);
  std::fprintf(f, "<Title>\nDollarStoreSCF B200 output\n</Title>\n\n<Keywords>\nGTO\n</Keywords>\n\n");
  std::fprintf(f, "<Number of Nuclei>\n%d\n</Number of Nuclei>\n\n", natom);
  std::fprintf(f, "<Net Charge>\n%d\n</Net Charge>\n\n", zsum - na - nb);
  std::fprintf(f, "<Number of Electrons>\n%d\n</Number of Electrons>\n\n", na + nb);
  std::fprintf(f, "<Number of Alpha Electrons>\n%d\n</Number of Alpha Electrons>\n\n", na);
  std::fprintf(f, "<Number of Beta Electrons>\n%d\n</Number of Beta Electrons>\n\n", nb);
  std::fprintf(f, "<Electronic Spin Multiplicity>\n%d\n</Electronic Spin Multiplicity>\n\n", na - nb + 1);
  std::fprintf(f, "<Nuclear Names>\n");
  for (int a = 0; a < natom; ++a) std::fprintf(f, "%s%d\n", kSymbols[Z[a] - 1], a + 1);
  std::fprintf(f, "</Nuclear Names>\n\n<Atomic Numbers>\n");
  for (int a = 0; a < natom; ++a) std::fprintf(f, "%d\n", Z[a]);
  std::fprintf(f, "</Atomic Numbers>\n\n<Nuclear Cartesian Coordinates>\n");
  for (int a = 0; a < natom; ++a)
    std::fprintf(f, " %20.12E %20.12E %20.12E\n", xyz_bohr[3 * a], xyz_bohr[3 * a + 1], xyz_bohr[3 * a + 2]);
  std::fprintf(f, "</Nuclear Cartesian Coordinates>\n\n");
  std::fprintf(f, "<Number of Primitives>\n%zu\n</Number of Primitives>\n\n", prims.size());
  std::fprintf(f, "<Primitive Centers>\n");
  write_rows(f, centers, 10, " %4.0f");
  std::fprintf(f, "</Primitive Centers>\n\n<Primitive Types>\n");
  write_rows(f, types, 10, " %4.0f");
  std::fprintf(f, "</Primitive Types>\n\n<Primitive Exponents>\n");
  write_rows(f, exps, 5, " %20.12E");
  std::fprintf(f, "</Primitive Exponents>\n\n");

  const int nmo_a = write_virtual ? n : na;
  const int nmo_b = unrestricted ? (write_virtual ? n : nb) : 0;
  std::fprintf(f, "<Molecular Orbital Occupation Numbers>\n");
  for (int i = 0; i < nmo_a; ++i) std::fprintf(f, "%d\n", i < na ? (unrestricted ? 1 : 2) : 0);
  for (int i = 0; i < nmo_b; ++i) std::fprintf(f, "%d\n", i < nb ? 1 : 0);
  std::fprintf(f, "</Molecular Orbital Occupation Numbers>\n\n<Molecular Orbital Energies>\n");
  for (int i = 0; i < nmo_a; ++i) std::fprintf(f, "%.12E\n", ctx->last_eps[0][i]);
  for (int i = 0; i < nmo_b; ++i) std::fprintf(f, "%.12E\n", ctx->last_eps[1][i]);
  std::fprintf(f, "</Molecular Orbital Energies>\n\n<Molecular Orbital Spin Types>\n");
  for (int i = 0; i < nmo_a; ++i) std::fprintf(f, "%s\n", unrestricted ? "Alpha" : "Alpha and Beta");
  for (int i = 0; i < nmo_b; ++i) std::fprintf(f, "Beta\n");
  std::fprintf(f, "</Molecular Orbital Spin Types>\n\n<Molecular Orbital Primitive Coefficients>\n");
  std::vector<double> w(prims.size());
  for (int sp = 0; sp < (unrestricted ? 2 : 1); ++sp) {
    const std::vector<double>& C = ctx->last_C[sp];
    for (int i = 0; i < (sp ? nmo_b : nmo_a); ++i) {
      std::fprintf(f, "<MO Number>\n%d\n</MO Number>\n", i + 1 + (sp ? nmo_a : 0));
      for (size_t k = 0; k < prims.size(); ++k) {
        const Prim& q = prims[k];
        const int l = B.l[q.shell];
        double v = 0.0;
        for (int m = 0; m <= 2 * l; ++m) v += C[(size_t)(B.f0[q.shell] + m) * n + i] * sph[l][m][q.pos];
        w[k] = v * B.wts[B.prim0[q.shell] + q.p];
      }
      write_rows(f, w, 5, " %20.12E");
    }
  }
  std::fprintf(f, "</Molecular Orbital Primitive Coefficients>\n");
  const bool ok = std::fclose(f) == 0;
  if (!ok) return dss_fail(ctx, DSS_ERR_INVALID, "dss_write_wfx: write failed");
  return DSS_OK;
}

}  // extern "C"
