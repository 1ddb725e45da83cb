// Density checkpoint: a restart file holding the spin densities of the last
// dss_scf_solve / dss_uhf_solve, read back as the guess of a later solve
// (use_guess), so a resumed job starts from the converged density instead of
// the core guess.  The reference writes no restart file of its own (its Molden
// and WFX output is for viewers; chem/scf/WriteOrbitals.cpp:17,196), so the
// format is this library's.
//
// File layout, little-endian:
//   bytes  0..7   magic "DSSDENS1"
//   bytes  8..23  int32 nbf, int32 spins (1: restricted, 2: unrestricted),
//                 int32 n_alpha, int32 n_beta
//   then          spins x nbf(nbf+1)/2 doubles: D_alpha (then D_beta), packed
//                 upper triangle (element (i, j), i <= j, at j(j+1)/2 + i), the
//                 layout of every packed matrix of this library
//   last 8 bytes  uint64 FNV-1a hash of bytes 8 .. end-8
// A restricted file holds D_alpha only (D_beta = D_alpha).
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "dss.h"
#include "dss_internal.h"

namespace {

const char kMagic[8] = {'D', 'S', 'S', 'D', 'E', 'N', 'S', '1'};

uint64_t fnv1a(const unsigned char* p, size_t n, uint64_t h = 1469598103934665603ull) {
  for (size_t i = 0; i < n; ++i) {
    h ^= p[i];
    h *= 1099511628211ull;
  }
  return h;
}

}  // namespace

extern "C" {

int dss_save_density(dss_ctx* ctx, const char* path) {
  if (!ctx) return DSS_ERR_INVALID;
  ctx->err.clear();
  if (!path) return dss_fail(ctx, DSS_ERR_INVALID, "dss_save_density: path is NULL");
  if (ctx->last_spins == 0 || ctx->nmol > 0)
    return dss_fail(ctx, DSS_ERR_INVALID, "dss_save_density: no solved single molecule in this context");
  const int n = ctx->nbf;
  const int spins = ctx->last_spins;
  if (ctx->last_C[0].size() != (size_t)n * n || (spins == 2 && ctx->last_C[1].size() != (size_t)n * n))
    return dss_fail(ctx, DSS_ERR_INVALID, "dss_save_density: orbitals do not match the basis");
  const size_t np = (size_t)n * (n + 1) / 2;
  const int32_t head[4] = {n, spins, ctx->last_nocc[0], spins == 2 ? ctx->last_nocc[1] : ctx->last_nocc[0]};
  std::vector<unsigned char> body(sizeof(head) + spins * np * sizeof(double));
  std::memcpy(body.data(), head, sizeof(head));
  for (int sp = 0; sp < spins; ++sp) {
    const std::vector<double>& C = ctx->last_C[sp];
    const int nocc = ctx->last_nocc[sp];
    std::vector<double> D(np);
    for (int j = 0; j < n; ++j)
      for (int i = 0; i <= j; ++i) {
        double d = 0.0;
        for (int k = 0; k < nocc; ++k) d += C[(size_t)i * n + k] * C[(size_t)j * n + k];
        D[(size_t)j * (j + 1) / 2 + i] = d;
      }
    std::memcpy(body.data() + sizeof(head) + sp * np * sizeof(double), D.data(), np * sizeof(double));
  }
  const uint64_t h = fnv1a(body.data(), body.size());
  FILE* f = std::fopen(path, "wb");
  if (!f) return dss_fail(ctx, DSS_ERR_INVALID, std::string("dss_save_density: cannot open ") + path);
  bool ok = std::fwrite(kMagic, 1, 8, f) == 8 && std::fwrite(body.data(), 1, body.size(), f) == body.size() &&
            std::fwrite(&h, 1, 8, f) == 8;
  ok = (std::fclose(f) == 0) && ok;
  if (!ok) return dss_fail(ctx, DSS_ERR_INVALID, "dss_save_density: write failed");
  return DSS_OK;
}

int dss_load_density(dss_ctx* ctx, const char* path, int nbf, int* spins, int* n_alpha, int* n_beta,
                     double* D_alpha, double* D_beta) {
  if (ctx) ctx->err.clear();
  if (!path || nbf <= 0 || !D_alpha)
    return dss_fail(ctx, DSS_ERR_INVALID, "dss_load_density: NULL path or output, or nbf <= 0");
  FILE* f = std::fopen(path, "rb");
  if (!f) return dss_fail(ctx, DSS_ERR_INVALID, std::string("dss_load_density: cannot open ") + path);
  std::vector<unsigned char> all;
  unsigned char buf[1 << 16];
  size_t got;
  while ((got = std::fread(buf, 1, sizeof(buf), f)) > 0) all.insert(all.end(), buf, buf + got);
  std::fclose(f);
  int32_t head[4];
  if (all.size() < 8 + sizeof(head) + 8 || std::memcmp(all.data(), kMagic, 8) != 0)
    return dss_fail(ctx, DSS_ERR_INVALID, "dss_load_density: not a density checkpoint");
  std::memcpy(head, all.data() + 8, sizeof(head));
  const size_t np = (size_t)nbf * (nbf + 1) / 2;
  if (head[0] != nbf)
    return dss_fail(ctx, DSS_ERR_INVALID, "dss_load_density: the file's basis has " + std::to_string(head[0]) +
                                              " functions, not " + std::to_string(nbf));
  if (head[1] != 1 && head[1] != 2) return dss_fail(ctx, DSS_ERR_INVALID, "dss_load_density: bad spin count");
  const size_t body = sizeof(head) + (size_t)head[1] * np * sizeof(double);
  if (all.size() != 8 + body + 8) return dss_fail(ctx, DSS_ERR_INVALID, "dss_load_density: truncated or oversized file");
  uint64_t h;
  std::memcpy(&h, all.data() + 8 + body, 8);
  if (h != fnv1a(all.data() + 8, body)) return dss_fail(ctx, DSS_ERR_INVALID, "dss_load_density: checksum mismatch");
  const unsigned char* d = all.data() + 8 + sizeof(head);
  std::memcpy(D_alpha, d, np * sizeof(double));
  if (D_beta) std::memcpy(D_beta, head[1] == 2 ? d + np * sizeof(double) : d, np * sizeof(double));
  if (spins) *spins = head[1];
  if (n_alpha) *n_alpha = head[2];
  if (n_beta) *n_beta = head[3];
  return DSS_OK;
}

}  // extern "C"
