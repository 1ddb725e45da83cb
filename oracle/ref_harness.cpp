// Test infrastructure (oracle): a C-ABI driver around the unmodified DollarStoreSCF
// sources, compiled by oracle/build_ref.sh into oracle/_ref/libdssref.so.
// The reference ships no main() and no tests; this file is the driver its README
// expects a user to write.  It is never linked into the product library.
//
// Every entry point drives the reference's own functions:
//   molecule / basis      scf::assignMolecule      chem/scf/SCFBasis.cpp:17-37
//   spherical basis       scf::constructBasis      chem/scf/SCFBasis.cpp:107-171
//   Cartesian (6D) basis  the same steps with one Cartesian term per function
//                         (the reference has no 6D mode; chem/GTO.cpp:15-94 builds
//                         only real solid harmonics)
//   SCF                   scf::useCoreGuess + scf::solveMOs + scf::getTotalEnergy
//                         chem/scf/SCFSolver.cpp:179-237, chem/scf/Energy.cpp:21-78
//   Fock two-electron     scf::computeCoulombTerms / computeExchangeTerms
//                         chem/scf/SCFSolver.cpp:29-43 over the stored tensor of
//                         chem/scf/ExactCoulomb.cpp:41-72
//   single ERI            flo::electronRepulsionIntegral chem/GaussianIntegral.cpp:561-642
//   Boys                  flo::boysFunctionExact     chem/GaussianIntegral.cpp:209-223
#include <sys/mman.h>
#include <sys/wait.h>
#include <unistd.h>

#include <chrono>
#include <cmath>
#include <cstring>
#include <iostream>
#include <sstream>
#include <vector>

#include "chem/GTO.hpp"
#include "chem/GaussianIntegral.hpp"
#include "chem/Molecule.hpp"
#include "chem/scf/Energy.hpp"
#include "chem/scf/ExactCoulomb.hpp"
#include "chem/scf/SCFBasis.hpp"
#include "chem/scf/SCFCommon.hpp"
#include "chem/scf/SCFDIIS.hpp"
#include "chem/scf/SCFSolver.hpp"
#include "chem/scf/WriteOrbitals.hpp"
#include "chem/scf/Gradient.hpp"

namespace flo {
double boysFunctionExact(double x, uint m);
}
namespace scf {
extern flo::Molecule molecule;
extern std::vector<flo::AtomicBasis> atom_bases;
extern double energy_threshold;
extern uint iteration;
void assignOverlapMatrix();
void assignCoreHamiltonian();
void assignOrthogonalization();
// Non-static definitions of chem/scf/ExactCoulomb.cpp:13-15, SCFSolver.cpp and
// Energy.cpp:13-18 that the parallel drivers below reuse.  The tensor globals
// are weak references: the drop-in variant of this library replaces
// ExactCoulomb.cpp with the GPU shim and has no stored tensor (the parallel
// fill then reports failure instead of running).
extern std::vector<double> repulsion_tensor __attribute__((weak));
extern size_t diagonal_size __attribute__((weak));
extern size_t tensor_size __attribute__((weak));
extern double previous_electronic_energy;
extern double total_electronic_energy;
extern double kinetic_energy, nuclear_attraction_energy, electron_repulsion_energy, exchange_energy,
    correlation_energy, nuclear_energy;
void updateFockMatrix(Spin spin);
void solveRoothaanHall(Spin spin);
void computeDensityMatrix(const Spin spin);
bool checkConvergence();
}  // namespace scf

namespace {
std::stringstream g_sink;
std::streambuf* g_saved = nullptr;
void quiet_on() {
  if (!g_saved) g_saved = std::cout.rdbuf(g_sink.rdbuf());
  g_sink.str("");
}
void quiet_off() {
  if (g_saved) std::cout.rdbuf(g_saved);
  g_saved = nullptr;
}

double dfact(int n) {
  double r = 1.0;
  for (int i = n; i > 0; i -= 2) r *= i;
  return r;
}

bool g_have_tensor = false;

// Fill scf::basis the way constructBasis() does (SCFBasis.cpp:120-139), but with
// one Cartesian monomial per function in 6D mode.  Monomials of a shell are
// ordered x-major: for l=2 xx, xy, xz, yy, yz, zz.
void build_basis_6d() {
  using namespace scf;
  basis.clear();
  basis_atoms.clear();
  atom_basis.clear();
  atom_basis.push_back(0);
  for (size_t i = 0; i < molecule.size(); ++i) {
    flo::vec3 center = molecule[i].position;
    for (flo::GTOShell& shell : atom_bases[i]) {
      int l = (int)shell.l;
      for (int a = l; a >= 0; --a) {
        for (int b = l - a; b >= 0; --b) {
          int c = l - a - b;
          flo::ContractedGaussian g(shell.primitives, (uint)l, 0, center);
          double w = std::sqrt(dfact(2 * l + 1) /
                               (4.0 * PI * dfact(2 * a - 1) * dfact(2 * b - 1) * dfact(2 * c - 1)));
          g.spherical_harmonic.clear();
          g.spherical_harmonic.push_back(flo::CartesianPolynomialTerm(w, (uint)a, (uint)b, (uint)c));
          basis.push_back(g);
          basis_atoms.push_back((uint)i);
        }
      }
    }
    atom_basis.push_back((uint)basis.size());
  }
}

// Buffer sizing of constructBasis() (SCFBasis.cpp:142-162), then S, H, X.
void size_state_and_one_electron() {
  using namespace scf;
  matrix_size = (uint)basis.size();
  buffer.resize(5);
  asymmetric_buffer.resize(5);
  for (int i = 0; i < 5; ++i) {
    buffer[i].resize(basis.size());
    asymmetric_buffer[i].resize(basis.size(), basis.size());
  }
  fock_matrix[0].resize(matrix_size);
  two_electron_hamiltonian[0].resize(matrix_size);
  coefficient_matrix[0].resize(matrix_size, matrix_size);
  density_matrix[0].resize(basis.size());
  total_density_matrix.resize(basis.size());
  assignOverlapMatrix();
  assignCoreHamiltonian();
  assignOrthogonalization();
}

void copy_packed(const flo::SymmetricMatrixNd& m, double* out) {
  size_t n = m.getWidth();
  for (size_t x = 0; x < n; ++x)
    for (size_t y = 0; y <= x; ++y) out[x * (x + 1) / 2 + y] = m.at((uint)y, (uint)x);
}
void load_packed(flo::SymmetricMatrixNd& m, const double* in) {
  size_t n = m.getWidth();
  for (size_t x = 0; x < n; ++x)
    for (size_t y = 0; y <= x; ++y) m.at((uint)y, (uint)x) = in[x * (x + 1) / 2 + y];
}

// ---------------------------------------------------------------- parallel drivers
// The reference is single-threaded with global state (chem/GaussianIntegral.cpp:10,
// chem/scf/SCFCommon.hpp), so threads are ruled out.  For bases whose serial run
// takes hours ((H2O)16 in 6-31G*), the drivers below fork worker processes that
// call the same reference functions on disjoint items and return results through
// shared anonymous mappings; the parent then stores them exactly where the
// reference's own loops would.  Every value is the reference's own, computed by
// the same function with the same arguments, so the results are bitwise those of
// the serial loops.
int g_workers = 1;

void* shared_alloc(size_t bytes) {
  void* p = mmap(nullptr, bytes, PROT_READ | PROT_WRITE, MAP_SHARED | MAP_ANONYMOUS, -1, 0);
  return p == MAP_FAILED ? nullptr : p;
}

// body(item) for item in [0, count), items pulled from a shared counter by
// g_workers forked processes.  Returns 0 when every worker exited cleanly.
template <class F>
int fork_for(long long count, F body) {
  long long* ctr = static_cast<long long*>(shared_alloc(4096));
  if (!ctr) return -1;
  *ctr = 0;
  std::cout.flush();
  std::cerr.flush();
  std::vector<pid_t> kids;
  int rc = 0;
  for (int w = 0; w < g_workers; ++w) {
    pid_t p = fork();
    if (p == 0) {
      for (;;) {
        long long it = __atomic_fetch_add(ctr, 1LL, __ATOMIC_RELAXED);
        if (it >= count) break;
        body(it);
      }
      _exit(0);
    }
    if (p < 0) {
      rc = -1;
      break;
    }
    kids.push_back(p);
  }
  for (pid_t p : kids) {
    int st = 0;
    if (waitpid(p, &st, 0) < 0 || !WIFEXITED(st) || WEXITSTATUS(st) != 0) rc = -1;
  }
  munmap(ctr, 4096);
  return rc;
}

void decode_pair(size_t m, uint& i, uint& j) {
  i = (uint)((std::sqrt(8.0 * (double)m + 1.0) - 1.0) / 2.0);
  while ((size_t)i * (i + 1) / 2 > m) --i;
  while ((size_t)(i + 1) * (i + 2) / 2 <= m) ++i;
  j = (uint)(m - (size_t)i * (i + 1) / 2);
}

// assignExactRepulsionTensor (chem/scf/ExactCoulomb.cpp:41-72) over workers: the
// same diagonal screen, index formula and electronRepulsionIntegral arguments;
// one item is one bra pair m = pair(i, j) with every ket pair n >= m.
int fill_tensor_parallel() {
  using namespace scf;
  if (!&repulsion_tensor || !&diagonal_size || !&tensor_size) return -1;
  const uint nb = (uint)basis.size();
  flo::SymmetricMatrixNd diagonal_terms(nb);
  for (uint a = 0; a < nb; ++a)
    for (uint b = 0; b <= a; ++b)
      diagonal_terms.at(b, a) = flo::electronRepulsionIntegral(basis[a], basis[b], basis[a], basis[b]);
  diagonal_size = (size_t)nb * (nb + 1) / 2;
  tensor_size = diagonal_size * (diagonal_size + 1) / 2;
  double* sh = static_cast<double*>(shared_alloc(tensor_size * sizeof(double)));
  if (!sh) return -1;
  const double thr = 0.00000001 * 0.00000001;  // INTEGRAL_THRESHOLD^2 (ExactCoulomb.cpp:11,63)
  int rc = fork_for((long long)diagonal_size, [&](long long item) {
    const size_t m = (size_t)item;
    uint i, j;
    decode_pair(m, i, j);
    for (size_t n = m; n < diagonal_size; ++n) {
      uint k, l;
      decode_pair(n, k, l);
      const size_t index = tensor_size - (diagonal_size - m) * (diagonal_size - m + 1) / 2 + n - m;
      if (diagonal_terms(i, j) * diagonal_terms(k, l) > thr)
        sh[index] = flo::electronRepulsionIntegral(basis[i], basis[k], basis[j], basis[l]);
    }
  });
  if (rc == 0) {
    repulsion_tensor.clear();
    repulsion_tensor.shrink_to_fit();
    repulsion_tensor.assign(sh, sh + tensor_size);
  }
  munmap(sh, tensor_size * sizeof(double));
  return rc;
}

// computeCoulombTerms(spin) followed by computeExchangeTerms(spin)
// (SCFSolver.cpp:29-43): G(mu,nu) = getExactCoulombMatrix(mu,nu), then
// -= getExactExchangeMatrix(mu,nu,spin).  With workers, rows mu are spread over
// processes and the parent performs the same two stores.
int two_electron_terms(scf::Spin spin, bool coulomb, bool exchange) {
  using namespace scf;
  const uint n = matrix_size;
  if (g_workers <= 1) {
    if (coulomb) computeCoulombTerms(spin);
    if (exchange) computeExchangeTerms(spin);
    return 0;
  }
  const size_t P = (size_t)n * (n + 1) / 2;
  double* sh = static_cast<double*>(shared_alloc(2 * P * sizeof(double)));
  if (!sh) return -1;
  double* J = sh;
  double* K = sh + P;
  int rc = fork_for((long long)n, [&](long long item) {
    const uint mu = (uint)item;
    for (uint nu = mu; nu < n; ++nu) {
      const size_t idx = (size_t)nu * (nu + 1) / 2 + mu;
      if (coulomb) J[idx] = getExactCoulombMatrix(mu, nu);
      if (exchange) K[idx] = getExactExchangeMatrix(mu, nu, spin);
    }
  });
  if (rc == 0) {
    flo::SymmetricMatrixNd& G = two_electron_hamiltonian[(int)spin];
    if (coulomb)
      for (uint mu = 0; mu < n; ++mu)
        for (uint nu = mu; nu < n; ++nu) G.at(mu, nu) = J[(size_t)nu * (nu + 1) / 2 + mu];
    if (exchange)
      for (uint mu = 0; mu < n; ++mu)
        for (uint nu = mu; nu < n; ++nu) G.at(mu, nu) -= K[(size_t)nu * (nu + 1) / 2 + mu];
  }
  munmap(sh, 2 * P * sizeof(double));
  return rc;
}
}  // namespace

extern "C" {

// Molecule and basis.  Z[natom], xyz_bohr[3*natom]; shells in atom order with
// shell_atom[s], shell_l[s], shell_nprim[s], then exps/coefs concatenated.
// cartesian: 0 = the reference's spherical (5D) functions, 1 = 6D monomials.
// build_tensor: 1 = also build the stored ERI tensor (needed for SCF/Fock).
// Returns the number of basis functions.
int ref_setup(int natom, const int* Z, const double* xyz_bohr, int nshell, const int* shell_atom,
              const int* shell_l, const int* shell_nprim, const double* exps, const double* coefs,
              int charge, int multiplicity, int cartesian, int build_tensor, int quiet) {
  if (quiet) quiet_on();
  flo::Molecule mol;
  for (int i = 0; i < natom; ++i) {
    flo::vec3 p(xyz_bohr[3 * i], xyz_bohr[3 * i + 1], xyz_bohr[3 * i + 2]);
    mol.atoms.push_back(flo::Atom(p, (flo::Element)Z[i]));
  }
  scf::assignMolecule(mol, charge, (uint)multiplicity);
  int off = 0;
  for (int s = 0; s < nshell; ++s) {
    std::vector<flo::GTOPrimitive> prims;
    for (int k = 0; k < shell_nprim[s]; ++k) prims.push_back(flo::GTOPrimitive(exps[off + k], coefs[off + k]));
    off += shell_nprim[s];
    scf::atom_bases[shell_atom[s]].push_back(flo::GTOShell((uint)shell_l[s], prims));
  }
  g_have_tensor = false;
  // Parallel tensor fill for closed-shell set-ups only (the unrestricted state
  // arrays are sized by constructBasis itself).
  const bool par = g_workers > 1 && multiplicity == 1;
  if (!cartesian && build_tensor && !par) {
    scf::constructBasis();
    g_have_tensor = true;
  } else {
    if (cartesian) {
      build_basis_6d();
    } else {
      // constructBasis() without the tensor: the same function list.
      scf::basis.clear();
      scf::basis_atoms.clear();
      scf::atom_basis.clear();
      scf::atom_basis.push_back(0);
      for (size_t i = 0; i < scf::molecule.size(); ++i) {
        for (flo::GTOShell& sh : scf::atom_bases[i])
          for (int m = -(int)sh.l; m <= (int)sh.l; ++m) {
            scf::basis.push_back(flo::ContractedGaussian(sh.primitives, sh.l, m, scf::molecule[i].position));
            scf::basis_atoms.push_back((uint)i);
          }
        scf::atom_basis.push_back((uint)scf::basis.size());
      }
    }
    size_state_and_one_electron();
    if (build_tensor) {
      if (par) {
        if (fill_tensor_parallel() != 0) {
          if (quiet) quiet_off();
          return -1;
        }
      } else {
        scf::assignExactRepulsionTensor();
      }
      g_have_tensor = true;
    }
  }
  if (quiet) quiet_off();
  return (int)scf::basis.size();
}

int ref_nbf() { return (int)scf::basis.size(); }

// Packed-upper (LAPACK 'U') one-electron matrices.
void ref_get_overlap(double* out) { copy_packed(scf::overlap_matrix, out); }
void ref_get_core_hamiltonian(double* out) { copy_packed(scf::core_hamiltonian, out); }

// Cartesian terms of basis function f: returns the count, fills (weight, x, y, z).
int ref_basis_terms(int f, double* weight, int* xyz) {
  const flo::ContractedGaussian& g = scf::basis[f];
  for (size_t t = 0; t < g.spherical_harmonic.size(); ++t) {
    weight[t] = g.spherical_harmonic[t].weight;
    xyz[3 * t] = (int)g.spherical_harmonic[t].x;
    xyz[3 * t + 1] = (int)g.spherical_harmonic[t].y;
    xyz[3 * t + 2] = (int)g.spherical_harmonic[t].z;
  }
  return (int)g.spherical_harmonic.size();
}
// Normalised primitive weights of basis function f (chem/GTO.cpp:90-93).
int ref_basis_prims(int f, double* zeta, double* weight) {
  const flo::ContractedGaussian& g = scf::basis[f];
  for (size_t p = 0; p < g.primitives.size(); ++p) {
    zeta[p] = g.primitives[p].zeta;
    weight[p] = g.primitives[p].weight;
  }
  return (int)g.primitives.size();
}

// SCF from the core guess to |dE| < conv (RHF, or UHF when ref_setup had
// multiplicity > 1).  Returns the iteration count; fills E_total and the final
// alpha density (packed-U).
int ref_scf(double conv, double* E_total, double* D_alpha_packed, double* seconds, int quiet) {
  if (!g_have_tensor) return -1;
  if (quiet) quiet_on();
  scf::energy_threshold = conv;
  auto t0 = std::chrono::steady_clock::now();
  scf::useCoreGuess();
  scf::solveMOs();
  auto t1 = std::chrono::steady_clock::now();
  *E_total = scf::getTotalEnergy();
  if (D_alpha_packed) copy_packed(scf::density_matrix[0], D_alpha_packed);
  if (seconds) *seconds = std::chrono::duration<double>(t1 - t0).count();
  if (quiet) quiet_off();
  return (int)scf::iteration;
}

// Nuclear gradient dE/dR [natom*3] (hartree/bohr) at the last ref_scf's density
// (scf::getEnergyGradient, chem/scf/Gradient.cpp:14-133).
int ref_gradient(double* out, int quiet) {
  if (!g_have_tensor) return -1;
  if (quiet) quiet_on();
  flo::VectorNd g;
  scf::getEnergyGradient(g);
  for (size_t i = 0; i < g.size(); ++i) out[i] = g[i];
  if (quiet) quiet_off();
  return (int)g.size();
}

// Molden file of the last ref_scf (scf::writeOrbitalsMolden, chem/scf/WriteOrbitals.cpp:17-137).
void ref_write_molden(const char* path, int write_virtual, int quiet) {
  if (quiet) quiet_on();
  scf::writeOrbitalsMolden(std::string(path), write_virtual != 0);
  if (quiet) quiet_off();
}

// WFX file of the last ref_scf (scf::writeOrbitalsWFX, chem/scf/WriteOrbitals.cpp:139-458).
void ref_write_wfx(const char* path, int write_virtual, int quiet) {
  if (quiet) quiet_on();
  scf::writeOrbitalsWFX(std::string(path), write_virtual != 0);
  if (quiet) quiet_off();
}

// Spin density (0 = alpha, 1 = beta; packed-U) after ref_scf, and the
// electron counts scf::assignMolecule derived from charge and multiplicity.
void ref_get_density(int spin, double* D_packed) { copy_packed(scf::density_matrix[spin ? 1 : 0], D_packed); }
void ref_electron_counts(int* n_alpha, int* n_beta) {
  *n_alpha = (int)scf::electron_count[0];
  *n_beta = (int)scf::electron_count[1];
}

// Two-electron Fock part for a given alpha density: G = J[2 D_alpha] - K[D_alpha]
// (the RHF G of SCFSolver.cpp:29-43, computeDensityMatrix :92).
int ref_fock_2e(const double* D_alpha_packed, double* G_packed) {
  if (!g_have_tensor) return -1;
  load_packed(scf::density_matrix[0], D_alpha_packed);
  scf::total_density_matrix = 2.0 * scf::density_matrix[0];
  scf::computeCoulombTerms(scf::Spin::alpha);
  scf::computeExchangeTerms(scf::Spin::alpha);
  copy_packed(scf::two_electron_hamiltonian[0], G_packed);
  return 0;
}

// J[D_total] and K[D_alpha] separately (packed-U), from the stored tensor.
int ref_jk(const double* D_alpha_packed, double* J_packed, double* K_packed) {
  if (!g_have_tensor) return -1;
  size_t n = scf::basis.size();
  load_packed(scf::density_matrix[0], D_alpha_packed);
  scf::total_density_matrix = 2.0 * scf::density_matrix[0];
  if (g_workers > 1) {
    const size_t P = n * (n + 1) / 2;
    double* sh = static_cast<double*>(shared_alloc(2 * P * sizeof(double)));
    if (!sh) return -1;
    int rc = fork_for((long long)n, [&](long long item) {
      const uint mu = (uint)item;
      for (uint nu = mu; nu < n; ++nu) {
        sh[(size_t)nu * (nu + 1) / 2 + mu] = scf::getExactCoulombMatrix(mu, nu);
        sh[P + (size_t)nu * (nu + 1) / 2 + mu] = scf::getExactExchangeMatrix(mu, nu, scf::Spin::alpha);
      }
    });
    if (rc == 0) {
      std::memcpy(J_packed, sh, P * sizeof(double));
      std::memcpy(K_packed, sh + P, P * sizeof(double));
    }
    munmap(sh, 2 * P * sizeof(double));
    return rc;
  }
  for (uint mu = 0; mu < n; ++mu)
    for (uint nu = mu; nu < n; ++nu) {
      J_packed[(size_t)nu * (nu + 1) / 2 + mu] = scf::getExactCoulombMatrix(mu, nu);
      K_packed[(size_t)nu * (nu + 1) / 2 + mu] = scf::getExactExchangeMatrix(mu, nu, scf::Spin::alpha);
    }
  return 0;
}

// Worker processes for the drivers above (1: the reference's serial loops).
// Closed-shell only: ref_setup fills the tensor in parallel for multiplicity 1,
// and ref_scf_capped runs the restricted iteration.
void ref_set_workers(int n) { g_workers = n > 1 ? n : 1; }

// scf::useCoreGuess + scf::solveMOs + scf::calculateEnergies for a closed-shell
// set-up (chem/scf/SCFSolver.cpp:145-237, chem/scf/Energy.cpp:21-50), step by
// step with the reference's own functions: the same iteration (two-electron
// terms, updateFockMatrix, solveRoothaanHall, computeDensityMatrix,
// getTotalElectronicEnergy), the same stop (checkConvergence) and the same final
// energy terms.  Two differences, both outside the arithmetic: the two-electron
// terms may be spread over worker processes (ref_set_workers), and the loop
// stops after max_iter iterations (the reference has no cap; 0 = none), in
// which case the return value is -(iterations) and E_total is the energy of
// the last iterate.  Returns the iteration count otherwise.
int ref_scf_capped(double conv, int max_iter, double* E_total, double* D_alpha_packed, double* seconds,
                   double* E_trace, int quiet) {
  using namespace scf;
  if (!g_have_tensor || spin_treatment != SpinTreatment::restricted) return -1000000;
  if (quiet) quiet_on();
  energy_threshold = conv;
  auto t0 = std::chrono::steady_clock::now();
  useCoreGuess();
  iteration = 0;
  diis::setIterationCount(8);
  total_electronic_energy = 0.0;
  previous_electronic_energy = 0.0;
  bool capped = false;
  int rc = 0;
  while (!checkConvergence()) {
    if (max_iter > 0 && (int)iteration >= max_iter) {
      capped = true;
      break;
    }
    ++iteration;
    rc |= two_electron_terms(Spin::alpha, true, true);
    updateFockMatrix(Spin::alpha);
    solveRoothaanHall(Spin::alpha);
    computeDensityMatrix(Spin::alpha);
    previous_electronic_energy = total_electronic_energy;
    total_electronic_energy = getTotalElectronicEnergy();
    if (E_trace && iteration <= 4096) E_trace[iteration - 1] = total_electronic_energy;
  }
  // calculateEnergies (Energy.cpp:21-50), restricted branch.
  kinetic_energy = flo::trace(total_density_matrix * kinetic_energy_matrix);
  nuclear_attraction_energy = flo::trace(total_density_matrix * nuclear_attraction_matrix);
  rc |= two_electron_terms(Spin::alpha, true, false);
  electron_repulsion_energy = 0.5 * flo::trace(density_matrix[0] * two_electron_hamiltonian[0]);
  electron_repulsion_energy *= 2.0;
  two_electron_hamiltonian[0] = 0.0;
  rc |= two_electron_terms(Spin::alpha, false, true);
  exchange_energy = 0.5 * flo::trace(density_matrix[0] * two_electron_hamiltonian[0]);
  exchange_energy *= 2.0;
  correlation_energy = 0.0;
  nuclear_energy = 0.0;
  for (int i = 0; i < (int)molecule.size(); ++i)
    for (int j = i + 1; j < (int)molecule.size(); ++j)
      nuclear_energy += (int)molecule[i].element * (int)molecule[j].element /
                        flo::length(molecule[i].position - molecule[j].position);
  auto t1 = std::chrono::steady_clock::now();
  *E_total = getTotalEnergy();
  if (D_alpha_packed) copy_packed(density_matrix[0], D_alpha_packed);
  if (seconds) *seconds = std::chrono::duration<double>(t1 - t0).count();
  if (quiet) quiet_off();
  if (rc) return -1000000;
  return capped ? -(int)iteration : (int)iteration;
}

// (mu nu | sigma tau) in chemist notation; argument order of the reference is
// (mu, sigma, nu, tau) (GaussianIntegral.cpp:561-565).
double ref_eri(int mu, int nu, int sigma, int tau) {
  return flo::electronRepulsionIntegral(scf::basis[mu], scf::basis[sigma], scf::basis[nu], scf::basis[tau]);
}

double ref_boys(double x, unsigned m) { return flo::boysFunctionExact(x, m); }

// Timed sample of the ERI phase: the canonical function quartets
// (i>=j, k>=l, ij<=kl) of assignExactRepulsionTensor (ExactCoulomb.cpp:54-68)
// whose first index i lies in [i_begin, i_end).  Returns the quartet count and
// the seconds spent; a checksum of the integrals guards against dead-code removal.
long long ref_time_eri_rows(int i_begin, int i_end, double* seconds, double* checksum) {
  size_t n = scf::basis.size();
  long long count = 0;
  double sum = 0.0;
  auto t0 = std::chrono::steady_clock::now();
  for (uint i = (uint)i_begin; i < (uint)i_end && i < n; ++i)
    for (uint j = 0; j <= i; ++j)
      for (uint k = 0; k < n; ++k)
        for (uint l = 0; l <= k; ++l) {
          uint m = j + i * (i + 1) / 2;
          uint nn = l + k * (k + 1) / 2;
          if (m > nn) continue;
          sum += flo::electronRepulsionIntegral(scf::basis[i], scf::basis[k], scf::basis[j], scf::basis[l]);
          ++count;
        }
  auto t1 = std::chrono::steady_clock::now();
  *seconds = std::chrono::duration<double>(t1 - t0).count();
  *checksum = sum;
  return count;
}

// Timed random sample of the ERI phase: canonical quartets (ij|kl) with pair
// indices m = i(i+1)/2 + j <= n = k(k+1)/2 + l drawn uniformly (xorshift64 from
// seed) until max_seconds have passed.  The mean cost per quartet times the
// quartet count gives the reference's ERI-phase time for the whole tensor.
long long ref_time_eri_random(double max_seconds, unsigned long long seed, double* seconds, double* checksum) {
  const size_t n = scf::basis.size();
  const unsigned long long P = (unsigned long long)n * (n + 1) / 2;
  unsigned long long st = seed ? seed : 88172645463325252ull;
  auto next = [&]() {
    st ^= st << 13;
    st ^= st >> 7;
    st ^= st << 17;
    return st;
  };
  auto decode = [](unsigned long long m, uint& i, uint& j) {
    i = (uint)((std::sqrt(8.0 * (double)m + 1.0) - 1.0) / 2.0);
    while ((unsigned long long)i * (i + 1) / 2 > m) --i;
    while ((unsigned long long)(i + 1) * (i + 2) / 2 <= m) ++i;
    j = (uint)(m - (unsigned long long)i * (i + 1) / 2);
  };
  long long count = 0;
  double sum = 0.0;
  auto t0 = std::chrono::steady_clock::now();
  double el = 0.0;
  while (el < max_seconds) {
    for (int rep = 0; rep < 64; ++rep) {
      unsigned long long a = next() % P, b = next() % P;
      if (a > b) std::swap(a, b);
      uint i, j, k, l;
      decode(a, i, j);
      decode(b, k, l);
      sum += flo::electronRepulsionIntegral(scf::basis[i], scf::basis[k], scf::basis[j], scf::basis[l]);
      ++count;
    }
    el = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  }
  *seconds = el;
  *checksum = sum;
  return count;
}

// Timed J+K digest over the stored tensor for one density (the per-iteration
// Fock work of the reference, SCFSolver.cpp:29-43).  Returns seconds.
double ref_time_jk(const double* D_alpha_packed) {
  size_t n = scf::basis.size();
  std::vector<double> G(n * (n + 1) / 2);
  auto t0 = std::chrono::steady_clock::now();
  ref_fock_2e(D_alpha_packed, G.data());
  auto t1 = std::chrono::steady_clock::now();
  return std::chrono::duration<double>(t1 - t0).count();
}

}  // extern "C"
