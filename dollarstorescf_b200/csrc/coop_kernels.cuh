// Warp-cooperative ERI + J/K digest for the high-angular-momentum classes.
//
// One warp evaluates one shell quartet: warp task t (one bra pair, up to 32 kets)
// is spread over DSS_COOP_SPLIT warps, one ket each.  The recurrences are the same as the thread-per-quartet kernels but
// run as the generated operation programs of coop_gen.cuh over a per-warp
// shared-memory value array: the VRR program once per primitive quartet
// (accumulating into the contracted [e0|f0]), then the HRR + function-transform
// program once per contracted quartet.  Lanes execute the operations of one
// dependency level in parallel.  Up to 8 primitive-quartet records (Boys values
// times prefactor and the Obara-Saika coefficients) are prepared in parallel by
// lanes 0..7 before the VRR passes.  The digest gives each J/K target element to
// one lane, which sums its products from shared memory.
#pragma once
#include "coop_gen.cuh"
#include "eri_kernels.cuh"

#define DSS_COOP_WARPS 1   // warps per block: small blocks let shared memory set occupancy
#define DSS_COOP_SPLIT 32  // warps per warp task: each warp takes one ket of the task
#define DSS_COOP_BATCH 8   // primitive-quartet records prepared per pass

template <int LA, int LB, int LC, int LD, bool PURE>
struct CoopProg;

#define DSS_DEFINE_COOP_PROG(la, lb, lc, ld)                                             \
  template <>                                                                           \
  struct CoopProg<la, lb, lc, ld, true> {                                               \
    static constexpr int NSLOTS = DSS_COOP_##la##lb##lc##ld##_s_NSLOTS;                 \
    static constexpr int NACC = DSS_COOP_##la##lb##lc##ld##_s_NACC;                     \
    static constexpr int ACC_BASE = DSS_COOP_##la##lb##lc##ld##_s_ACC_BASE;             \
    static constexpr int NVLV = DSS_COOP_##la##lb##lc##ld##_s_NVLV;                     \
    static constexpr int NHLV = DSS_COOP_##la##lb##lc##ld##_s_NHLV;                     \
    __device__ static const uint4* vrr() { return kCoopVrr_##la##lb##lc##ld##_s; }      \
    __device__ static const uint4* acc() { return kCoopAcc_##la##lb##lc##ld##_s; }      \
    __device__ static const uint4* hrr() { return kCoopHrr_##la##lb##lc##ld##_s; }      \
    __device__ static const unsigned short* vlv() { return kCoopVrrLv_##la##lb##lc##ld##_s; } \
    __device__ static const unsigned short* hlv() { return kCoopHrrLv_##la##lb##lc##ld##_s; } \
    __device__ static const double* w() { return kCoopW_##la##lb##lc##ld##_s; }         \
    __device__ static const unsigned short* out() { return kCoopOut_##la##lb##lc##ld##_s; } \
  };                                                                                    \
  template <>                                                                           \
  struct CoopProg<la, lb, lc, ld, false> {                                              \
    static constexpr int NSLOTS = DSS_COOP_##la##lb##lc##ld##_c_NSLOTS;                 \
    static constexpr int NACC = DSS_COOP_##la##lb##lc##ld##_c_NACC;                     \
    static constexpr int ACC_BASE = DSS_COOP_##la##lb##lc##ld##_c_ACC_BASE;             \
    static constexpr int NVLV = DSS_COOP_##la##lb##lc##ld##_c_NVLV;                     \
    static constexpr int NHLV = DSS_COOP_##la##lb##lc##ld##_c_NHLV;                     \
    __device__ static const uint4* vrr() { return kCoopVrr_##la##lb##lc##ld##_c; }      \
    __device__ static const uint4* acc() { return kCoopAcc_##la##lb##lc##ld##_c; }      \
    __device__ static const uint4* hrr() { return kCoopHrr_##la##lb##lc##ld##_c; }      \
    __device__ static const unsigned short* vlv() { return kCoopVrrLv_##la##lb##lc##ld##_c; } \
    __device__ static const unsigned short* hlv() { return kCoopHrrLv_##la##lb##lc##ld##_c; } \
    __device__ static const double* w() { return kCoopW_##la##lb##lc##ld##_c; }         \
    __device__ static const unsigned short* out() { return kCoopOut_##la##lb##lc##ld##_c; } \
  };
DSS_FOR_EACH_COOP_CLASS(DSS_DEFINE_COOP_PROG)
#undef DSS_DEFINE_COOP_PROG

// Record layout (doubles): F_m * prefactor at 0..L; PA 12-14, WP 15-17, QC 18-20,
// WQ 21-23, 1/2p 24, 1/2q 25, 1/2(p+q) 26, rho/p 27, rho/q 28.
#define DSS_REC 32

__device__ __forceinline__ double coop_get(const double* __restrict__ rec, const double* __restrict__ vals,
                                           unsigned idx) {
  return idx < 32u ? rec[idx] : vals[idx - 32u];
}

// The operations of one dependency level are independent, so a lane takes
// several at a time: their records and all their operands are read before any
// result is stored, which overlaps the dependent load chains.
__device__ __forceinline__ void coop_vrr_fetch(const uint4& op, const double* __restrict__ r,
                                               const double* __restrict__ vals, double (&x)[5]) {
  const unsigned s0 = op.x >> 16, s1 = op.y & 0xFFFFu, s2 = op.y >> 16, s3 = op.z & 0xFFFFu, s4 = op.z >> 16;
  x[0] = coop_get(r, vals, s0);
  x[1] = coop_get(r, vals, s1);
  x[2] = s2 != 0xFFFFu ? coop_get(r, vals, s2) : 0.0;
  x[3] = s2 != 0xFFFFu ? coop_get(r, vals, s3) : 0.0;
  x[4] = s4 != 0xFFFFu ? coop_get(r, vals, s4) : 0.0;
}

__device__ __forceinline__ double coop_vrr_value(const uint4& op, const double* __restrict__ r, const double (&x)[5]) {
  const unsigned kind = op.w & 15u, ax = (op.w >> 4) & 3u;
  const double k1 = (double)((op.w >> 8) & 0xFFu), k2 = (double)((op.w >> 16) & 0xFFu);
  const bool has2 = (op.y >> 16) != 0xFFFFu, has4 = (op.z >> 16) != 0xFFFFu;
  double v;
  if (kind == 0u) {
    v = r[12 + ax] * x[0] + r[15 + ax] * x[1];
    if (has2) v += k1 * r[24] * (x[2] - r[27] * x[3]);
  } else {
    v = r[18 + ax] * x[0] + r[21 + ax] * x[1];
    if (has2) v += k1 * r[25] * (x[2] - r[28] * x[3]);
    if (has4) v += k2 * r[26] * x[4];
  }
  return v;
}

// One level of the VRR program over the primitive-quartet record r, four
// operations per lane in flight (records and operands of all four read first).
__device__ __forceinline__ void coop_vrr_level(const uint4* __restrict__ prog, int o0, int o1, int lane,
                                               const double* __restrict__ r, double* vals) {
  int o = o0 + lane;
  for (; o + 96 < o1; o += 128) {
    uint4 op[4];
    double x[4][5];
#pragma unroll
    for (int u = 0; u < 4; ++u) op[u] = __ldg(prog + o + 32 * u);
#pragma unroll
    for (int u = 0; u < 4; ++u) coop_vrr_fetch(op[u], r, vals, x[u]);
    double v[4];
#pragma unroll
    for (int u = 0; u < 4; ++u) v[u] = coop_vrr_value(op[u], r, x[u]);
#pragma unroll
    for (int u = 0; u < 4; ++u) vals[(op[u].x & 0xFFFFu) - 32u] = v[u];
  }
  for (; o < o1; o += 32) {
    const uint4 a = __ldg(prog + o);
    double xa[5];
    coop_vrr_fetch(a, r, vals, xa);
    vals[(a.x & 0xFFFFu) - 32u] = coop_vrr_value(a, r, xa);
  }
}

// HRR (kind 2) and function-transform (kind 3) operations over the value array.
__device__ __forceinline__ void coop_hrr_fetch(const uint4& op, const double* __restrict__ vals, double (&x)[3]) {
  const unsigned s0 = op.x >> 16, s1 = op.y & 0xFFFFu, s2 = op.y >> 16;
  x[0] = vals[s0 - 32u];
  x[1] = s1 != 0xFFFFu ? vals[s1 - 32u] : 0.0;
  x[2] = s2 != 0xFFFFu ? vals[s2 - 32u] : 0.0;
}

__device__ __forceinline__ double coop_hrr_value(const uint4& op, const double* __restrict__ hdr,
                                                 const double* __restrict__ wts, const double (&x)[3]) {
  if ((op.w & 15u) == 2u) {
    const unsigned ax = (op.w >> 4) & 3u, side = (op.w >> 6) & 1u;
    return x[0] + hdr[3 * side + ax] * x[1];
  }
  double v = __ldg(wts + (op.z & 0xFFFFu)) * x[0];
  if ((op.y & 0xFFFFu) != 0xFFFFu) v += __ldg(wts + (op.z >> 16)) * x[1];
  if ((op.y >> 16) != 0xFFFFu) v += __ldg(wts + (op.w >> 16)) * x[2];
  return v;
}

__device__ __forceinline__ void coop_hrr_level(const uint4* __restrict__ prog, int o0, int o1, int lane,
                                               const double* __restrict__ hdr, const double* __restrict__ wts,
                                               double* vals) {
  int o = o0 + lane;
  for (; o + 96 < o1; o += 128) {
    uint4 op[4];
    double x[4][3];
#pragma unroll
    for (int u = 0; u < 4; ++u) op[u] = __ldg(prog + o + 32 * u);
#pragma unroll
    for (int u = 0; u < 4; ++u) coop_hrr_fetch(op[u], vals, x[u]);
    double v[4];
#pragma unroll
    for (int u = 0; u < 4; ++u) v[u] = coop_hrr_value(op[u], hdr, wts, x[u]);
#pragma unroll
    for (int u = 0; u < 4; ++u) vals[(op[u].x & 0xFFFFu) - 32u] = v[u];
  }
  for (; o < o1; o += 32) {
    const uint4 a = __ldg(prog + o);
    double xa[3];
    coop_hrr_fetch(a, vals, xa);
    vals[(a.x & 0xFFFFu) - 32u] = coop_hrr_value(a, hdr, wts, xa);
  }
}

template <int LA, int LB, int LC, int LD, bool PURE>
__host__ __device__ constexpr size_t coop_smem_per_warp() {
  constexpr int NA = dss_nfunc(LA, PURE), NB = dss_nfunc(LB, PURE), NC = dss_nfunc(LC, PURE),
                ND = dss_nfunc(LD, PURE);
  return (size_t)CoopProg<LA, LB, LC, LD, PURE>::NSLOTS + DSS_COOP_BATCH * DSS_REC + 8 +
         (NA * NB) * 2 + NC * ND + NA * ND + NB * ND + NA * NC + NB * NC;
}

template <int LA, int LB, int LC, int LD, int BOYS, bool PURE, bool MIXED = false>
__global__ void __launch_bounds__(32 * DSS_COOP_WARPS) eri_coop_kernel(EriArgs a) {
  using P = CoopProg<LA, LB, LC, LD, PURE>;
  constexpr int NA = dss_nfunc(LA, PURE), NB = dss_nfunc(LB, PURE);
  constexpr int NC = dss_nfunc(LC, PURE), ND = dss_nfunc(LD, PURE);
  constexpr int L = LA + LB + LC + LD;
  constexpr size_t PER_WARP = coop_smem_per_warp<LA, LB, LC, LD, PURE>();
  extern __shared__ double smem[];
  const int wib = threadIdx.x >> 5;
  const int lane = threadIdx.x & 31;
  const long long gw = (long long)blockIdx.x * DSS_COOP_WARPS + wib;
  const int warp = (int)(gw / DSS_COOP_SPLIT);
  const int part = (int)(gw % DSS_COOP_SPLIT);
  if (warp >= a.ntasks) return;  // uniform per warp
  double* vals = smem + PER_WARP * wib;
  double* recs = vals + P::NSLOTS;
  double* hdr = recs + DSS_COOP_BATCH * DSS_REC;
  double* jab = hdr + 8;        // [NA*NB] J sums for the bra pair over the task
  double* dab = jab + NA * NB;  // density blocks
  double* dcd = dab + NA * NB;
  double* dad = dcd + NC * ND;
  double* dbd = dad + NA * ND;
  double* dac = dbd + NB * ND;
  double* dbc = dac + NA * NC;

  const int4 t = __ldg(a.tasks + warp);
  const int k_begin = part * ((t.z + DSS_COOP_SPLIT - 1) / DSS_COOP_SPLIT);
  const int k_end = min(t.z, k_begin + (t.z + DSS_COOP_SPLIT - 1) / DSS_COOP_SPLIT);
  if (k_begin >= k_end) return;  // uniform per warp
  const int bra = t.x;
  const int sa = __ldg(a.pair_a + bra), sb = __ldg(a.pair_b + bra);
  const double* __restrict__ Dm = a.D;
  double* Jm = a.J;
  double* Km = a.K;
  int n = a.n;
  if (a.sh_mbase) {  // batches: the bra pair fixes the molecule
    if (a.mol_active && !__ldg(a.mol_active + __ldg(a.sh_mol + sa))) return;
    n = __ldg(a.sh_n + sa);
    Dm += __ldg(a.sh_mbase + sa);
    Jm += __ldg(a.sh_jbase + sa);
    Km += __ldg(a.sh_kbase + sa);
  }
  const int fa = __ldg(a.sh_f0 + sa), fb = __ldg(a.sh_f0 + sb);
  const PrimPair* bpp = a.pp + __ldg(a.pair_pp0 + bra);
  const int nbp = __ldg(a.pair_npp + bra);
  for (int q = lane; q < NA * NB; q += 32) {
    jab[q] = 0.0;
    dab[q] = __ldg(Dm + (size_t)(fa + q / NB) * n + fb + q % NB);
  }
  const uint4* __restrict__ vrr = P::vrr();
  const uint4* __restrict__ accp = P::acc();
  const uint4* __restrict__ hrr = P::hrr();
  const unsigned short* __restrict__ vlv = P::vlv();
  const unsigned short* __restrict__ hlv = P::hlv();
  const double* __restrict__ wts = P::w();
  const unsigned short* __restrict__ outs = P::out();

  for (int kq = k_begin; kq < k_end; ++kq) {
    const int ket = t.y + kq;
    const int sc = __ldg(a.pair_a + ket), sd = __ldg(a.pair_b + ket);
    const int fc = __ldg(a.sh_f0 + sc), fd = __ldg(a.sh_f0 + sd);
    const PrimPair* kpp = a.pp + __ldg(a.pair_pp0 + ket);
    const int nkp = __ldg(a.pair_npp + ket);
    if constexpr (MIXED) {  // uniform across the warp
      if (__ldg(a.Qp + bra) * __ldg(a.Qp + ket) * quartet_dbound(a, sa, sb, sc, sd) < a.skip_thr) continue;
    }
    if (lane < 6) {
      const int s0 = lane < 3 ? sa : sc, s1 = lane < 3 ? sb : sd, ax = lane % 3;
      hdr[lane] = __ldg(a.sh_xyz + 3 * s0 + ax) - __ldg(a.sh_xyz + 3 * s1 + ax);
    }
    for (int q = lane; q < P::NACC; q += 32) vals[P::ACC_BASE + q] = 0.0;
    const int nprim = nbp * nkp;
    for (int b0 = 0; b0 < nprim; b0 += DSS_COOP_BATCH) {
      const int nb = min(DSS_COOP_BATCH, nprim - b0);
      if (lane < nb) {
        const int pi = b0 + lane;
        const PrimPair bp = load_pp(bpp + pi % nbp);
        const PrimPair kp = load_pp(kpp + pi / nbp);
        double F[L + 1];
        double* r = recs + lane * DSS_REC;
        prim_quartet<BOYS, L>(bp, kp, F, r[12], r[13], r[14], r[15], r[16], r[17], r[18], r[19], r[20], r[21],
                              r[22], r[23], r[24], r[25], r[26], r[27], r[28], a.boys_cell);
#pragma unroll
        for (int m = 0; m <= L; ++m) r[m] = F[m];
      }
      __syncwarp();
      for (int j = 0; j < nb; ++j) {
        const double* __restrict__ r = recs + j * DSS_REC;
        for (int lv = 0; lv < P::NVLV; ++lv) {
          coop_vrr_level(vrr, __ldg(vlv + lv), __ldg(vlv + lv + 1), lane, r, vals);
          __syncwarp();
        }
        // Accumulation: distinct targets, sources among the VRR outputs, four per lane in flight.
        int o = lane;
        for (; o + 96 < P::NACC; o += 128) {
          unsigned dst[4];
          double add[4], cur[4];
#pragma unroll
          for (int u = 0; u < 4; ++u) {
            const uint4 op = __ldg(accp + o + 32 * u);
            dst[u] = (op.x & 0xFFFFu) - 32u;
            add[u] = coop_get(r, vals, op.x >> 16);
            cur[u] = vals[dst[u]];
          }
#pragma unroll
          for (int u = 0; u < 4; ++u) vals[dst[u]] = cur[u] + add[u];
        }
        for (; o < P::NACC; o += 32) {
          const uint4 op = __ldg(accp + o);
          vals[(op.x & 0xFFFFu) - 32u] += coop_get(r, vals, op.x >> 16);
        }
        __syncwarp();
      }
    }
    // HRR + transform
    for (int lv = 0; lv < P::NHLV; ++lv) {
      coop_hrr_level(hrr, __ldg(hlv + lv), __ldg(hlv + lv + 1), lane, hdr, wts, vals);
      __syncwarp();
    }
    // Digest (same algebra as eri_jk_kernel).
    double s = 1.0;
    if (sa == sb) s *= 0.5;
    if (sc == sd) s *= 0.5;
    if (bra == ket) s *= 0.5;
    for (int q = lane; q < NC * ND; q += 32) dcd[q] = __ldg(Dm + (size_t)(fc + q / ND) * n + fd + q % ND);
    for (int q = lane; q < NA * ND; q += 32) dad[q] = __ldg(Dm + (size_t)(fa + q / ND) * n + fd + q % ND);
    for (int q = lane; q < NB * ND; q += 32) dbd[q] = __ldg(Dm + (size_t)(fb + q / ND) * n + fd + q % ND);
    for (int q = lane; q < NA * NC; q += 32) dac[q] = __ldg(Dm + (size_t)(fa + q / NC) * n + fc + q % NC);
    for (int q = lane; q < NB * NC; q += 32) dbc[q] = __ldg(Dm + (size_t)(fb + q / NC) * n + fc + q % NC);
    __syncwarp();
#define DSS_I(i, j, k, l) vals[__ldg(outs + (((i) * NB + (j)) * NC + (k)) * ND + (l)) - 32u]
    // J over the bra pair: accumulated in shared memory across the task's kets.
    for (int q = lane; q < NA * NB; q += 32) {
      const int i = q / NB, j = q % NB;
      double acc = 0.0;
      for (int k = 0; k < NC; ++k)
        for (int l = 0; l < ND; ++l) acc += DSS_I(i, j, k, l) * dcd[k * ND + l];
      jab[q] += s * acc;
    }
    for (int q = lane; q < NC * ND; q += 32) {
      const int k = q / ND, l = q % ND;
      double acc = 0.0;
      for (int i = 0; i < NA; ++i)
        for (int j = 0; j < NB; ++j) acc += DSS_I(i, j, k, l) * dab[i * NB + j];
      atomicAdd(Jm + (size_t)(fc + k) * n + fd + l, 2.0 * s * acc);
    }
    for (int q = lane; q < NA * ND; q += 32) {  // K[i][l] += (ij|kl) D[j][k]
      const int i = q / ND, l = q % ND;
      double acc = 0.0;
      for (int j = 0; j < NB; ++j)
        for (int k = 0; k < NC; ++k) acc += DSS_I(i, j, k, l) * dbc[j * NC + k];
      atomicAdd(Km + (size_t)(fa + i) * n + fd + l, s * acc);
    }
    for (int q = lane; q < NB * ND; q += 32) {  // K[j][l] += (ij|kl) D[i][k]
      const int j = q / ND, l = q % ND;
      double acc = 0.0;
      for (int i = 0; i < NA; ++i)
        for (int k = 0; k < NC; ++k) acc += DSS_I(i, j, k, l) * dac[i * NC + k];
      atomicAdd(Km + (size_t)(fb + j) * n + fd + l, s * acc);
    }
    for (int q = lane; q < NA * NC; q += 32) {  // K[i][k] += (ij|kl) D[j][l]
      const int i = q / NC, k = q % NC;
      double acc = 0.0;
      for (int j = 0; j < NB; ++j)
        for (int l = 0; l < ND; ++l) acc += DSS_I(i, j, k, l) * dbd[j * ND + l];
      atomicAdd(Km + (size_t)(fa + i) * n + fc + k, s * acc);
    }
    for (int q = lane; q < NB * NC; q += 32) {  // K[j][k] += (ij|kl) D[i][l]
      const int j = q / NC, k = q % NC;
      double acc = 0.0;
      for (int i = 0; i < NA; ++i)
        for (int l = 0; l < ND; ++l) acc += DSS_I(i, j, k, l) * dad[i * ND + l];
      atomicAdd(Km + (size_t)(fb + j) * n + fc + k, s * acc);
    }
#undef DSS_I
    __syncwarp();
  }
  for (int q = lane; q < NA * NB; q += 32)
    atomicAdd(Jm + (size_t)(fa + q / NB) * n + fb + q % NB, 2.0 * jab[q]);
}
