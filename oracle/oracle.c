/*
 * Test infrastructure (oracle): a plain-C restatement of DollarStoreSCF's
 * electron-repulsion arithmetic, used only by tests/, the smoke check and
 * bench.py's CPU-baseline leg to check the CUDA path.  It is not linked into,
 * and never called by, the product library.
 *
 * What it restates (file:line in the reference):
 *   orc_boys_ref   flo::boysFunctionExact       chem/GaussianIntegral.cpp:209-223
 *                  (series truncated at a term <= 1e-9; asymptotic form when
 *                  x > 1.1 m + 25; PI = 3.14159265358979, lalib/MathUtil.hpp:8;
 *                  integer powers by the reference's own square-and-multiply
 *                  order, lalib/MathUtil.hpp:56-73)
 *   orc_eri_shell  the primitive/Cartesian sums of electronRepulsionIntegral
 *                  chem/GaussianIntegral.cpp:561-642 (prefactor :585-586,632)
 *                  evaluated per Cartesian shell quartet.  The reference's
 *                  separable 1-D Obara-Saika chain (OSRepulsion :334-559) is
 *                  replaced by the textbook 3-D Obara-Saika vertical recursion
 *                  plus the Head-Gordon-Pople horizontal transfer; both are exact
 *                  linear maps of the same F_m values, so results agree to
 *                  rounding.
 *
 * Cartesian monomials of a shell of angular momentum l are ordered x-major
 * (a descending, then b descending) -- xx, xy, xz, yy, yz, zz for l = 2.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>

#define ORC_PI 3.14159265358979
#define ORC_LMAX 4                /* per shell */
#define ORC_LTOT (4 * ORC_LMAX)   /* total angular momentum of a quartet */
#define ORC_NC(l) (((l) + 1) * ((l) + 2) / 2)

/* Integer power by the reference's recursion (lalib/MathUtil.hpp:56-66). */
static double ref_ipow(double x, unsigned p) {
  if (p == 1) return x;
  if (p == 0) return 1.0;
  double y = x;
  unsigned l = 2;
  for (; l < p; l *= 2) y = y * y;
  return y * ref_ipow(x, p - l / 2);
}

/* (2m-1)!! as the reference evaluates it: in 32-bit int arithmetic
 * (doubleFactorial<int>, lalib/MathUtil.hpp:36-42), which wraps for m >= 11. */
static double dfact_int32(int n) {
  unsigned int r = 1u;
  for (int i = n; i > 0; i -= 2) r *= (unsigned int)i;
  return (double)(int)r;
}

double orc_boys_ref(double x, unsigned m) {
  if (x > (double)m * 1.1 + 25.0) {
    double pw2 = 1.0;
    for (unsigned i = 0; i < m + 1; ++i) pw2 *= 2.0;
    return dfact_int32(2 * (int)m - 1) / pw2 * sqrt(ORC_PI / ref_ipow(x, 2 * m + 1));
  }
  double F = 1.0, a = 1.0;
  for (int i = 1; a > 0.000000001; ++i) {
    a = 2.0 * x / (double)(2 * (int)m + 2 * i + 1) * a;
    F += a;
  }
  return exp(-x) / (double)(2 * m + 1) * F;
}

/* Cartesian index tables: monomials of total degree l, x-major. */
static int g_tab_ready = 0;
static int g_cx[ORC_LTOT + 2][ORC_NC(ORC_LTOT + 1)];
static int g_cy[ORC_LTOT + 2][ORC_NC(ORC_LTOT + 1)];
static int g_cz[ORC_LTOT + 2][ORC_NC(ORC_LTOT + 1)];
/* index of (a,b,c) with a+b+c = l */
static int cidx(int a, int b, int c) {
  int l = a + b + c;
  /* x-major: position = sum over larger a' of (l - a' + 1) + (l - a - b) */
  int pos = 0;
  for (int ap = l; ap > a; --ap) pos += l - ap + 1;
  return pos + (l - a - b);
}
static void init_tabs(void) {
  if (g_tab_ready) return;
  for (int l = 0; l <= ORC_LTOT + 1; ++l) {
    int n = 0;
    for (int a = l; a >= 0; --a)
      for (int b = l - a; b >= 0; --b) {
        g_cx[l][n] = a;
        g_cy[l][n] = b;
        g_cz[l][n] = l - a - b;
        ++n;
      }
  }
  g_tab_ready = 1;
}

/* Offsets for the cumulative index over all monomials with degree <= L. */
static int coff(int l) { return l * (l + 1) * (l + 2) / 6; }
static int call_idx(int a, int b, int c) { return coff(a + b + c) + cidx(a, b, c); }

/*
 * One Cartesian shell quartet (ab|cd), contracted.  exps/w are the primitive
 * exponents and normalised weights (norm * coefficient) per shell.  out has
 * NC(la)*NC(lb)*NC(lc)*NC(ld) entries in row-major [a][b][c][d] order.
 */
void orc_eri_shell(int la, int lb, int lc, int ld, const double* A, const double* B, const double* C,
                   const double* D, int na, const double* ea, const double* wa, int nb, const double* eb,
                   const double* wb, int nc, const double* ec, const double* wc, int nd, const double* ed,
                   const double* wd, double* out) {
  init_tabs();
  const int E = la + lb, F = lc + ld, L = E + F;
  const int nE = coff(E + 1), nF = coff(F + 1);
  /* contracted [e0|f0] for all e <= E, f <= F */
  double* acc = (double*)calloc((size_t)nE * nF, sizeof(double));
  /* primitive table V[m][e][f] */
  double* V = (double*)malloc((size_t)(L + 1) * nE * nF * sizeof(double));
  double Fm[ORC_LTOT + 1];
  double AB2 = 0, CD2 = 0;
  for (int k = 0; k < 3; ++k) {
    AB2 += (A[k] - B[k]) * (A[k] - B[k]);
    CD2 += (C[k] - D[k]) * (C[k] - D[k]);
  }
#define VV(m, e, f) V[((size_t)(m) * nE + (e)) * nF + (f)]
  for (int ia = 0; ia < na; ++ia)
    for (int ib = 0; ib < nb; ++ib)
      for (int ic = 0; ic < nc; ++ic)
        for (int id = 0; id < nd; ++id) {
          double al = ea[ia], be = eb[ib], ga = ec[ic], de = ed[id];
          double p = al + be, q = ga + de;
          double P[3], Q[3], W[3];
          for (int k = 0; k < 3; ++k) {
            P[k] = (al * A[k] + be * B[k]) / p;
            Q[k] = (ga * C[k] + de * D[k]) / q;
          }
          double rho = p * q / (p + q);
          double PQ2 = 0;
          for (int k = 0; k < 3; ++k) {
            W[k] = (p * P[k] + q * Q[k]) / (p + q);
            PQ2 += (P[k] - Q[k]) * (P[k] - Q[k]);
          }
          double T = p * q * PQ2 / (p + q);
          for (int m = 0; m <= L; ++m) Fm[m] = orc_boys_ref(T, (unsigned)m);
          double pref = 2.0 * pow(ORC_PI, 2.5) / (p * q * sqrt(p + q)) * exp(-al * be / p * AB2) *
                        exp(-ga * de / q * CD2) * wa[ia] * wb[ib] * wc[ic] * wd[id];
          for (int m = 0; m <= L; ++m) VV(m, 0, 0) = pref * Fm[m];
          /* bra vertical recursion, f = 0 */
          for (int e = 1; e <= L; ++e) {
            if (e > E) break;
            for (int n = 0; n < ORC_NC(e); ++n) {
              int ex = g_cx[e][n], ey = g_cy[e][n], ez = g_cz[e][n];
              int dir = ex ? 0 : (ey ? 1 : 2);
              int em[3] = {ex, ey, ez};
              em[dir] -= 1;
              int i1 = call_idx(em[0], em[1], em[2]);
              int i2 = -1;
              if (em[dir] > 0) {
                int e2[3] = {em[0], em[1], em[2]};
                e2[dir] -= 1;
                i2 = call_idx(e2[0], e2[1], e2[2]);
              }
              int it = call_idx(ex, ey, ez);
              double pa = P[dir] - A[dir], wp = W[dir] - P[dir];
              for (int m = 0; m <= L - e; ++m) {
                double v = pa * VV(m, i1, 0) + wp * VV(m + 1, i1, 0);
                if (i2 >= 0) v += em[dir] / (2.0 * p) * (VV(m, i2, 0) - rho / p * VV(m + 1, i2, 0));
                VV(m, it, 0) = v;
              }
            }
          }
          /* ket vertical recursion */
          for (int f = 1; f <= F; ++f) {
            for (int n = 0; n < ORC_NC(f); ++n) {
              int fx = g_cx[f][n], fy = g_cy[f][n], fz = g_cz[f][n];
              int dir = fx ? 0 : (fy ? 1 : 2);
              int fm[3] = {fx, fy, fz};
              fm[dir] -= 1;
              int j1 = call_idx(fm[0], fm[1], fm[2]);
              int j2 = -1;
              if (fm[dir] > 0) {
                int f2[3] = {fm[0], fm[1], fm[2]};
                f2[dir] -= 1;
                j2 = call_idx(f2[0], f2[1], f2[2]);
              }
              int jt = call_idx(fx, fy, fz);
              double qc = Q[dir] - C[dir], wq = W[dir] - Q[dir];
              for (int e = 0; e <= E; ++e) {
                for (int ne = 0; ne < ORC_NC(e); ++ne) {
                  int ie = coff(e) + ne;
                  int ecomp[3] = {g_cx[e][ne], g_cy[e][ne], g_cz[e][ne]};
                  int ik = -1;
                  if (ecomp[dir] > 0) {
                    int e2[3] = {ecomp[0], ecomp[1], ecomp[2]};
                    e2[dir] -= 1;
                    ik = call_idx(e2[0], e2[1], e2[2]);
                  }
                  for (int m = 0; m <= L - e - f; ++m) {
                    double v = qc * VV(m, ie, j1) + wq * VV(m + 1, ie, j1);
                    if (j2 >= 0) v += fm[dir] / (2.0 * q) * (VV(m, ie, j2) - rho / q * VV(m + 1, ie, j2));
                    if (ik >= 0) v += ecomp[dir] / (2.0 * (p + q)) * VV(m + 1, ik, j1);
                    VV(m, ie, jt) = v;
                  }
                }
              }
            }
          }
          for (int e = 0; e < nE; ++e)
            for (int f = 0; f < nF; ++f) acc[(size_t)e * nF + f] += VV(0, e, f);
        }
#undef VV
  /* Horizontal transfer on the bra: (a, b+1_i| = (a+1_i, b| + AB_i (a, b| */
  /* H1[a-comp (deg la..E-lb')][b-comp][f] built degree by degree in b. */
  {
    double AB[3] = {A[0] - B[0], A[1] - B[1], A[2] - B[2]};
    double CD[3] = {C[0] - D[0], C[1] - D[1], C[2] - D[2]};
    /* bra[(ea, b)] for ea over all monomials deg <= E, b over deg <= lb */
    int nB = coff(lb + 1);
    double* bra = (double*)calloc((size_t)nE * nB * nF, sizeof(double));
#define BR(e, b, f) bra[((size_t)(e) * nB + (b)) * nF + (f)]
    for (int e = 0; e < nE; ++e)
      for (int f = 0; f < nF; ++f) BR(e, 0, f) = acc[(size_t)e * nF + f];
    for (int bdeg = 1; bdeg <= lb; ++bdeg)
      for (int nbb = 0; nbb < ORC_NC(bdeg); ++nbb) {
        int bx = g_cx[bdeg][nbb], by = g_cy[bdeg][nbb], bz = g_cz[bdeg][nbb];
        int dir = bx ? 0 : (by ? 1 : 2);
        int bm[3] = {bx, by, bz};
        bm[dir] -= 1;
        int ibm = call_idx(bm[0], bm[1], bm[2]);
        int ibt = call_idx(bx, by, bz);
        for (int edeg = 0; edeg <= E - bdeg; ++edeg)
          for (int ne = 0; ne < ORC_NC(edeg); ++ne) {
            int ec3[3] = {g_cx[edeg][ne], g_cy[edeg][ne], g_cz[edeg][ne]};
            int ie = coff(edeg) + ne;
            ec3[dir] += 1;
            int iep = call_idx(ec3[0], ec3[1], ec3[2]);
            for (int f = 0; f < nF; ++f) BR(ie, ibt, f) = BR(iep, ibm, f) + AB[dir] * BR(ie, ibm, f);
          }
      }
    /* ket: |c, d+1_i) = |c+1_i, d) + CD_i |c, d) */
    int nD = coff(ld + 1);
    int nAc = ORC_NC(la), nBc = ORC_NC(lb), nCc = ORC_NC(lc), nDc = ORC_NC(ld);
    double* ket = (double*)calloc((size_t)nF * nD, sizeof(double));
    for (int a = 0; a < nAc; ++a)
      for (int b = 0; b < nBc; ++b) {
        int ia = coff(la) + a, ibb = coff(lb) + b;
        memset(ket, 0, sizeof(double) * (size_t)nF * nD);
        for (int f = 0; f < nF; ++f) ket[(size_t)f * nD + 0] = BR(ia, ibb, f);
        for (int ddeg = 1; ddeg <= ld; ++ddeg)
          for (int ndd = 0; ndd < ORC_NC(ddeg); ++ndd) {
            int dx = g_cx[ddeg][ndd], dy = g_cy[ddeg][ndd], dz = g_cz[ddeg][ndd];
            int dir = dx ? 0 : (dy ? 1 : 2);
            int dm[3] = {dx, dy, dz};
            dm[dir] -= 1;
            int idm = call_idx(dm[0], dm[1], dm[2]);
            int idt = call_idx(dx, dy, dz);
            for (int fdeg = 0; fdeg <= F - ddeg; ++fdeg)
              for (int nf = 0; nf < ORC_NC(fdeg); ++nf) {
                int fc3[3] = {g_cx[fdeg][nf], g_cy[fdeg][nf], g_cz[fdeg][nf]};
                int jf = coff(fdeg) + nf;
                fc3[dir] += 1;
                int jfp = call_idx(fc3[0], fc3[1], fc3[2]);
                ket[(size_t)jf * nD + idt] = ket[(size_t)jfp * nD + idm] + CD[dir] * ket[(size_t)jf * nD + idm];
              }
          }
        for (int c = 0; c < nCc; ++c)
          for (int d = 0; d < nDc; ++d)
            out[(((size_t)a * nBc + b) * nCc + c) * nDc + d] = ket[(size_t)(coff(lc) + c) * nD + coff(ld) + d];
      }
#undef BR
    free(ket);
    free(bra);
  }
  free(V);
  free(acc);
}
