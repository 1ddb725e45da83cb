// Boys function F_m(x) = int_0^1 t^(2m) exp(-x t^2) dt, m = 0..L, in two modes.
//
// DSS_BOYS_REF reproduces the reference's flo::boysFunctionExact
// (chem/GaussianIntegral.cpp:209-223) value for value: for x > 1.1 m + 25 the
// asymptotic form (2m-1)!!/2^(m+1) sqrt(PI/x^(2m+1)) with PI = 3.14159265358979,
// otherwise exp(-x)/(2m+1) * sum_i a_i with a_0 = 1, a_i = a_(i-1) 2x/(2m+2i+1),
// summed up to and including the first term <= 1e-9.  That truncation leaves
// an absolute error of up to ~1.5e-11 which moves (H2O)_16 energies by ~1e-9 Eh,
// so this mode is the one that meets 1e-9 Eh parity with the reference.  The
// per-m series share one sequence: the m-series is the (m+1)-series scaled by
// 2x/(2m+3) plus a leading 1, so the top m runs the full series and each lower m
// only adjusts its truncation point by a few terms (the stopping rule is applied
// to the m-series' own terms, exactly as the reference applies it).  The series
// itself only runs next to a truncation breakpoint and near x = 0; elsewhere
// the values come from per-cell Taylor records (boys_ref_cells) or, beyond
// their orders, from the accurate function corrected by the truncated tail
// (boys_ref_walk).
//
// DSS_BOYS_FAST is the accurate function: a 7-term Taylor expansion of F_L
// about the nearest point of a 1/16-spaced table (boys_tab.cuh), downward
// recursion F_m = (2x F_(m+1) + exp(-x)) / (2m+1), and for x >= 36 the
// asymptotic F_0 = sqrt(pi/x)/2 with upward recursion.  Relative error ~1e-14.
#pragma once
#include <cuda_runtime.h>

#include "boys_tab.cuh"

#define DSS_BOYS_REF 0
#define DSS_BOYS_FAST 1
// Reference values as DSS_BOYS_REF, with the block-A cell records of orders
// 0..L read from dynamic shared memory (dss_boys_smem_stage); only kernels that
// stage them may instantiate this mode.
#define DSS_BOYS_REF_SMEM 2

#define DSS_PI_REF 3.14159265358979

// The reference's switch to the asymptotic form, x > 1.1 m + 25, evaluated in
// double precision as it does (1.1 m rounded, then + 25 rounded): the values for
// m = 0..12 as exact literals, so that the test costs no arithmetic per call.
__host__ __device__ constexpr double dss_boys_asym_thr(int m) {
  switch (m) {
    case 0: return 0x1.9000000000000p+4;
    case 1: return 0x1.a19999999999ap+4;
    case 2: return 0x1.b333333333333p+4;
    case 3: return 0x1.c4ccccccccccdp+4;
    case 4: return 0x1.d666666666666p+4;
    case 5: return 0x1.e800000000000p+4;
    case 6: return 0x1.f99999999999ap+4;
    case 7: return 0x1.059999999999ap+5;
    case 8: return 0x1.0e66666666666p+5;
    case 9: return 0x1.1733333333333p+5;
    case 10: return 0x1.2000000000000p+5;
    case 11: return 0x1.28ccccccccccdp+5;
    default: return 0x1.319999999999ap+5;
  }
}

// 1/(2k+1) for k = 0..255 (g_odd_inv in boys_tab.cuh): the series divides
// 2x/(2m+2i+1) become products with a correctly rounded reciprocal.
__device__ __forceinline__ double odd_inv(int k) { return g_odd_inv[k]; }

// The reference's integer power (lalib/MathUtil.hpp:56-66): square-and-multiply
// in its own order, so the asymptotic branch rounds the same way.
__device__ __forceinline__ double ref_ipow(double x, unsigned p) {
  // Iterative form of: if p==1 return x; if p==0 return 1; y=x; l=2;
  // while l<p: y=y*y, l*=2; return y * pow(x, p - l/2) -- the factors are
  // multiplied innermost first, as the recursion does.
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
    p = p - l / 2;
  }
  double r = tail;
  for (int i = nf - 1; i >= 0; --i) r = fac[i] * r;
  return r;
}

template <int L>
static __device__ __noinline__ void boys_ref_series(double x, double* F) {
  const double ex = exp(-x);
  // m values with x > 1.1 m + 25 take the asymptotic branch; they are the lowest m.
  // Series for the remaining m are built from the top down.
  int m_series_lo = L + 1;
#pragma unroll
  for (int m = L; m >= 0; --m) {
    const double thr = dss_boys_asym_thr(m);
    if (!(x > thr)) m_series_lo = m;
  }
  // Top series (m = L) when it is needed.
  double S = 0.0, last = 0.0;
  int n = 0;  // index of the last term included
  if (m_series_lo <= L) {
    const double x2 = 2.0 * x;
    double a = 1.0;
    S = 1.0;
    int i = 1;
    do {
      a = x2 * odd_inv(L + i) * a;
      S += a;
      ++i;
    } while (a > 0.000000001);
    n = i - 1;
    last = a;
    F[L] = ex * odd_inv(L) * S;
  }
  // Downward: the m-series terms are t^(m)_i = c_m t^(m+1)_(i-1) with
  // c_m = 2x/(2m+3); the reference stops at the first i >= 1 with t^(m)_i <= 1e-9.
#pragma unroll
  for (int m = L - 1; m >= 0; --m) {
    if (m < m_series_lo) break;
    const double c = 2.0 * x * odd_inv(m + 1);
    // (m+1)-series: S = sum_{k=0..n} t_k, last = t_n.  Find the first k >= 0 with
    // c * t_k <= 1e-9 (the m-series stop index is k + 1).
    double Sm1 = S, t = last;
    int k = n;
    if (c * t <= 0.000000001) {
      // Walk back while the previous term also satisfies the stop rule.
      while (k > 0) {
        const double tp = t * (double)(2 * (m + 1) + 2 * k + 1) / (2.0 * x);
        if (c * tp <= 0.000000001) {
          Sm1 -= t;
          t = tp;
          --k;
        } else {
          break;
        }
      }
    } else {
      // Extend the (m+1)-series forward until the stop rule holds.
      do {
        t = t * 2.0 * x * odd_inv(m + 1 + k + 1);
        Sm1 += t;
        ++k;
      } while (c * t > 0.000000001);
    }
    // m-series: 1 + c * (sum of (m+1)-terms 0..k), last term c * t_k, stop index k + 1.
    S = 1.0 + c * Sm1;
    last = c * t;
    n = k + 1;
    F[m] = ex * odd_inv(m) * S;
  }
  // Asymptotic branch for the low m.
#pragma unroll
  for (int m = 0; m <= L; ++m) {
    if (m < m_series_lo) {
      // (2m-1)!! in 32-bit int arithmetic as the reference evaluates it
      // (doubleFactorial<int>, lalib/MathUtil.hpp:36-42); it wraps for m >= 11.
      unsigned int dfi = 1u;
      for (int j = 2 * m - 1; j > 0; j -= 2) dfi *= (unsigned int)j;
      const double df = (double)(int)dfi;
      double p2 = 1.0;
      for (int j = 0; j < m + 1; ++j) p2 *= 2.0;
      F[m] = df / p2 * sqrt(DSS_PI_REF / ref_ipow(x, 2 * m + 1));
    }
  }
}

template <int L>
__device__ __forceinline__ void boys_fast(double x, double* F) {
  static_assert(L + 6 < DSS_BOYS_NM, "Boys table too narrow for this order");
  if (x < 35.9) {
    const int k = __double2int_rn(x * (double)DSS_BOYS_STEP);
    const double dx = (double)k * (1.0 / DSS_BOYS_STEP) - x;  // x0 - x
    const double* row = g_boys_tab + k * DSS_BOYS_NM + L;
    // Taylor: F_L(x) = sum_j F_(L+j)(x0) (x0 - x)^j / j!
    double f = row[6] * (1.0 / 720.0);
    f = f * dx + row[5] * (1.0 / 120.0);
    f = f * dx + row[4] * (1.0 / 24.0);
    f = f * dx + row[3] * (1.0 / 6.0);
    f = f * dx + row[2] * 0.5;
    f = f * dx + row[1];
    f = f * dx + row[0];
    F[L] = f;
    if (L > 0) {
      const double ex = exp(-x);
      const double x2 = 2.0 * x;
#pragma unroll
      for (int m = L - 1; m >= 0; --m) F[m] = (x2 * F[m + 1] + ex) * (1.0 / (double)(2 * m + 1));
    }
  } else {
    const double ex = exp(-x);
    const double inv2x = 0.5 / x;
    F[0] = 0.5 * sqrt(3.141592653589793 / x);
#pragma unroll
    for (int m = 0; m < L; ++m) F[m + 1] = ((double)(2 * m + 1) * F[m] - ex) * inv2x;
  }
}

// Reference-mode Boys for orders beyond the interval tables (see boys_ref).  The
// m = L series the reference would sum is  S = sum_{i<=n} t_i,  t_i = (2x)^i / prod_{j<=i}(2L+2j+1),
// stopped at n = first i >= 1 with t_i <= 1e-9.  Then
//   S = e^x (2L+1) F_L(x) - sum_{i>n} t_i,
// with F_L from the accurate table (boys_fast), n from the tabulated truncation
// breakpoints (n = 1 + #{k : B_L[k] < x}, boys_tab.cuh), t_n = exp(n ln 2x - LP_L[n])
// and the short geometric tail summed directly.  The lower orders follow by the
// same truncation-adjusting downward step as boys_ref_series.  When x lies within
// a relative 4e-14 of a breakpoint (where rounding decides the reference's stop),
// or L exceeds the tables, the series itself runs.
template <int L>
__device__ __forceinline__ void boys_ref_walk(double x, double* F) {
  int m_series_lo = L + 1;
#pragma unroll
  for (int m = L; m >= 0; --m) {
    const double thr = dss_boys_asym_thr(m);
    if (!(x > thr)) m_series_lo = m;
  }
  // The reference's asymptotic form (2m-1)!!/2^(m+1) sqrt(PI/x^(2m+1)) for the low
  // orders, as (2m-1)!!/2^(m+1) sqrt(PI) * rsqrt(x)^(2m+1); (2m-1)!! is the
  // reference's 32-bit value.  Same numbers to ~1e-15 relative, no loops.
  double asym[L + 1];
  if (m_series_lo > 0) {
    const double y = rsqrt(x);
    const double y2 = y * y;
    double pw = y * 1.7724538509055152;  // sqrt(PI_REF) * x^-(1/2)
#pragma unroll
    for (int m = 0; m <= L; ++m) {
      unsigned int dfi = 1u;
      for (int j = 2 * m - 1; j > 0; j -= 2) dfi *= (unsigned int)j;
      double p2 = 1.0;
      for (int j = 0; j < m + 1; ++j) p2 *= 2.0;
      asym[m] = ((double)(int)dfi / p2) * pw;
      pw *= y2;
    }
  }
  if (m_series_lo > L) {
#pragma unroll
    for (int m = 0; m <= L; ++m) F[m] = asym[m];
    return;
  }
  // One code path for all lanes of a warp (their x differ): the series runs only
  // for orders outside the tables, x ~ 0, x beyond the table, or next to a stop.
  bool use_series = L >= DSS_BOYS_NLB || L + 6 >= DSS_BOYS_NM || !(x > 1e-280) || !(x < 35.9);
  int n = 1;
  if (!use_series) {
    // Truncation index of the m = L series.
    const double* bp = g_boys_bp + L * (DSS_BOYS_NB + 1);
    n = 1 + (int)g_boys_idx[L * DSS_BOYS_NG + (int)(x * 4.0)];
    while (n <= DSS_BOYS_NB && bp[n] < x) ++n;
    if (n > DSS_BOYS_NB) {
      use_series = true;
    } else {
      const double lo_b = bp[n - 1], hi_b = bp[n];  // lo_b < x <= hi_b (bp[0] = 0)
      use_series = fabs(x - hi_b) <= 4e-14 * x || fabs(x - lo_b) <= 4e-14 * x;
    }
  }
  if (use_series) {
    double Fs[L + 1];
    boys_ref_series<L>(x, Fs);
#pragma unroll
    for (int m = 0; m <= L; ++m) F[m] = Fs[m];
    return;
  }
  // Accurate F_L (7-term Taylor about the nearest table point).
  const int k = __double2int_rn(x * (double)DSS_BOYS_STEP);
  const double dx = (double)k * (1.0 / DSS_BOYS_STEP) - x;
  const double* row = g_boys_tab + k * DSS_BOYS_NM + L;
  double fl = row[6] * (1.0 / 720.0);
  fl = fl * dx + row[5] * (1.0 / 120.0);
  fl = fl * dx + row[4] * (1.0 / 24.0);
  fl = fl * dx + row[3] * (1.0 / 6.0);
  fl = fl * dx + row[2] * 0.5;
  fl = fl * dx + row[1];
  fl = fl * dx + row[0];
  const double ex = exp(-x);
  const double x2 = 2.0 * x;
  const double tn = exp((double)n * log(x2) - g_boys_lp[L * (DSS_BOYS_NB + 1) + n]);
  // Tail beyond the stop: t_n <= 1e-9 and the term ratio 2x/(2L+2n+2j+1) stays
  // below 0.37 there; scanning x in (0, 1.1 L + 25] shows that what is left
  // after 8 + floor(L/2) further terms is below 1e-17 S (L <= 8), so 10 + L/2 terms
  // leave S unchanged at double precision (orders above 8, not scanned, keep 20).
  // A fixed trip count keeps the warp's lanes together.
  constexpr int kTail = L <= 8 ? 10 + L / 2 : 20;
  double tail = 0.0, t = tn;
#pragma unroll
  for (int j = 1; j <= kTail; ++j) {
    t = t * x2 * odd_inv(L + n + j);
    tail += t;
  }
  double S = fl * (double)(2 * L + 1) / ex - tail;
  double last = tn;
  F[L] = fl - ex * tail * odd_inv(L);
#pragma unroll
  for (int m = L - 1; m >= 0; --m) {
    if (m < m_series_lo) break;
    const double c = 2.0 * x * odd_inv(m + 1);
    double Sm1 = S, tt = last;
    int kk = n;
    if (c * tt <= 0.000000001) {
      while (kk > 0) {
        const double tp = tt * (double)(2 * (m + 1) + 2 * kk + 1) / x2;
        if (c * tp <= 0.000000001) {
          Sm1 -= tt;
          tt = tp;
          --kk;
        } else {
          break;
        }
      }
    } else {
      do {
        tt = tt * x2 * odd_inv(m + 1 + kk + 1);
        Sm1 += tt;
        ++kk;
      } while (c * tt > 0.000000001);
    }
    S = 1.0 + c * Sm1;
    last = c * tt;
    n = kk + 1;
    F[m] = ex * odd_inv(m) * S;
  }
#pragma unroll
  for (int m = 0; m <= L; ++m)
    if (m < m_series_lo) F[m] = asym[m];
}

// Reference-mode Boys from the cell records (cells = the library's copy of
// g_boys_cell, boys_cell_data.cu, passed in the kernel arguments): per order m
// and grid point k = round(16 x) a 64-byte record holds the Taylor
// coefficients, about k/16, of the reference's value up to the one truncation
// breakpoint b the cell may contain (b = 1e300 when it has none) and b itself;
// a second record at the same index of block B holds the piece past b.
// Orders with x > 1.1 m + 25 take the asymptotic form (one rsqrt for all of
// them); every other order reads its A record (two 32-byte loads, b included),
// the B record only when x > b, and evaluates seven FMAs: no search.  The
// series itself (a separate function) runs only for x < 1/32 (cell 0 holds
// several breakpoints) and within 4e-14 (relative) of a breakpoint, where the
// rounding of the reference's own sum decides its stop.
// Block-A records of orders 0..L staged in shared memory: record r (order-major,
// as in the global table) keeps its four 16-byte chunks at r*4 + ((j + (r >> 1)) & 3),
// so the first chunks of random records spread over all eight 16-byte bank groups.
extern __shared__ __align__(16) double2 dss_boys_smem[];

__device__ __forceinline__ int dss_boys_smem_slot(int r, int j) { return r * 4 + ((j + (r >> 1)) & 3); }

// Copies the block-A records of orders 0..L into dss_boys_smem (every thread of
// the block takes part; ends with a block barrier).
template <int L>
__device__ __forceinline__ void dss_boys_smem_stage(const double* __restrict__ cells) {
  const double2* src = reinterpret_cast<const double2*>(cells);
  const int nchunk = (L + 1) * DSS_BOYS_NCELL * 4;
  for (int i = threadIdx.x; i < nchunk; i += blockDim.x) dss_boys_smem[dss_boys_smem_slot(i >> 2, i & 3)] = __ldg(src + i);
  __syncthreads();
}

template <int L>
__host__ __device__ constexpr size_t dss_boys_smem_bytes() { return (size_t)(L + 1) * DSS_BOYS_NCELL * 64; }

// One 32-byte read-only load (four doubles, 32-byte aligned address): a cell
// record takes two of them instead of four 16-byte loads.
__device__ __forceinline__ void dss_ld4(const double* __restrict__ p, double& a, double& b, double& c, double& d) {
  asm("ld.global.nc.v4.f64 {%0, %1, %2, %3}, [%4];" : "=d"(a), "=d"(b), "=d"(c), "=d"(d) : "l"(p));
}

template <int L, bool SMEM = false>
__device__ __forceinline__ void boys_ref_cells(double x, double* F, const double* __restrict__ cells) {
  static_assert(L < DSS_BOYS_NMC, "cell records too narrow for this order");
  // Orders m < m_lo take the asymptotic form (x > 1.1 m + 25; the thresholds
  // grow with m, so these are the lowest orders).
  int m_lo = L + 1;
#pragma unroll
  for (int m = L; m >= 0; --m)
    if (!(x > dss_boys_asym_thr(m))) m_lo = m;
  if (m_lo > 0) {
    // (2m-1)!!/2^(m+1) sqrt(PI) x^-(m+1/2), (2m-1)!! as the reference's 32-bit int.
    const double y = rsqrt(x);
    const double y2 = y * y;
    double pw = y * 1.7724538509055152;  // sqrt(PI_REF) * x^-(1/2)
#pragma unroll
    for (int m = 0; m <= L; ++m) {
      unsigned int dfi = 1u;
      for (int j = 2 * m - 1; j > 0; j -= 2) dfi *= (unsigned int)j;
      double p2 = 1.0;
      for (int j = 0; j < m + 1; ++j) p2 *= 2.0;
      if (m < m_lo) F[m] = ((double)(int)dfi / p2) * pw;
      pw *= y2;
    }
  }
  if (m_lo > L) return;
  const int k = max(0, min(__double2int_rn(x * (double)DSS_BOYS_STEP), DSS_BOYS_NCELL - 1));
  const double dx = x - (double)k * (1.0 / DSS_BOYS_STEP);
  bool series = !(x >= 1.0 / 32.0);
#pragma unroll
  for (int m = 0; m <= L; ++m) {
    if (m < m_lo) continue;
    const double* r = cells + ((size_t)m * DSS_BOYS_NCELL + k) * 8;
    double2 c01, c23, c45, c6b;
    if constexpr (SMEM) {
      const int rec = m * DSS_BOYS_NCELL + k;
      c01 = dss_boys_smem[dss_boys_smem_slot(rec, 0)];
      c23 = dss_boys_smem[dss_boys_smem_slot(rec, 1)];
      c45 = dss_boys_smem[dss_boys_smem_slot(rec, 2)];
      c6b = dss_boys_smem[dss_boys_smem_slot(rec, 3)];
    } else {
      dss_ld4(r, c01.x, c01.y, c23.x, c23.y);
      dss_ld4(r + 4, c45.x, c45.y, c6b.x, c6b.y);
    }
    const double b = c6b.y;
    if (x > b) {  // the piece past the cell's breakpoint, same index in block B
      r += (size_t)DSS_BOYS_NMC * DSS_BOYS_NCELL * 8;
      dss_ld4(r, c01.x, c01.y, c23.x, c23.y);
      dss_ld4(r + 4, c45.x, c45.y, c6b.x, c6b.y);
    }
    double f = c6b.x;
    f = f * dx + c45.y;
    f = f * dx + c45.x;
    f = f * dx + c23.y;
    f = f * dx + c23.x;
    f = f * dx + c01.y;
    f = f * dx + c01.x;
    F[m] = f;
    series = series || fabs(x - b) <= 4e-14 * x;
  }
  if (series) {
    // A private array for the (non-inlined) series, so that F itself stays in
    // registers on the common path.
    double Fs[L + 1];
    boys_ref_series<L>(x, Fs);
#pragma unroll
    for (int m = 0; m <= L; ++m) F[m] = Fs[m];
  }
}

#ifndef DSS_BOYS_CELL_LMAX
#define DSS_BOYS_CELL_LMAX 8
#endif

// Reference-mode Boys (the reference's flo::boysFunctionExact values): the cell
// records for L <= DSS_BOYS_CELL_LMAX, boys_ref_walk above.
template <int L>
__device__ __forceinline__ void boys_ref(double x, double* F, const double* __restrict__ cells) {
  if constexpr (L <= DSS_BOYS_CELL_LMAX && L < DSS_BOYS_NMC) {
    boys_ref_cells<L>(x, F, cells);
  } else {
    boys_ref_walk<L>(x, F);
  }
}

template <int BOYS, int L>
__device__ __forceinline__ void boys_eval(double x, double* F, const double* __restrict__ cells) {
  if constexpr (BOYS == DSS_BOYS_REF_SMEM) {
    static_assert(L <= DSS_BOYS_CELL_LMAX && L < DSS_BOYS_NMC, "shared-memory records need the cell table");
    boys_ref_cells<L, true>(x, F, cells);
  } else if constexpr (BOYS == DSS_BOYS_REF) {
    boys_ref<L>(x, F, cells);
  } else {
    boys_fast<L>(x, F);
  }
}
