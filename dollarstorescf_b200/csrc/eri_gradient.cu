// Analytic two-electron nuclear gradient: derivative ERIs fused with the
// two-particle-density digest (the four-centre term of
// chem/scf/ExactCoulomb.cpp:125-195, differentiated as chem/GaussianIntegral.cpp:
// 1052-1459 differentiates the primitives).
//
//   dE_2e/dX = sum over unique shell quartets q of 4 s_q sum_{ijkl in q} d(ij|kl)/dX Gamma_ijkl,
//   Gamma_ijkl = D_ij D_kl - x (X_ik X_jl + X_il X_jk) - x (Y_ik Y_jl + Y_il Y_jk),
//
// D the total density; RHF: X = D, x = 1/4, no Y; UHF: X = D_alpha, Y = D_beta,
// x = 1/2; s_q = 1/2 per coincidence (a = b, c = d, ab = cd) as in the J/K digest.
// One warp per shell quartet runs the class's generated programs (gen_grad.py):
// per primitive quartet the Obara-Saika VRR and four accumulations (unweighted
// and weighted by 2 alpha, 2 beta, 2 gamma), then per contracted quartet the HRR
// to the shifted classes and the contraction with Gamma carried to the Cartesian
// basis (Gc), into the derivatives along A, B and C; D's is minus their sum.
// The warp tasks, shell pairs and primitive pairs are the context's J/K work
// lists (Schwarz-screened); quartets whose four shells sit on one nucleus add
// nothing and are skipped.
#include <atomic>
#include <cuda_runtime.h>

#include <string>
#include <vector>

#include "common.cuh"
#include "dss.h"
#include "dss_internal.h"
#include "eri_kernels.cuh"

struct DssCartFun {
  int f;
  double w;
};
#include "grad_gen.cuh"

namespace {

constexpr int kGradSplit = 32;  // warps per warp task: one ket each
constexpr int kGradBatch = 8;   // primitive-quartet records prepared per pass
constexpr int kRec = 32;

struct GradArgs {
  const int4* tasks;
  int ntasks;
  const int* pair_a;
  const int* pair_b;
  const int* pair_pp0;
  const int* pair_npp;
  const PrimPair* pp;
  const double* pp_alpha;  // exponent of the pair's first primitive
  const double* sh_xyz;
  const int* sh_f0;
  const int* sh_atom;
  const double* D;  // dense n x n: total density
  const double* X;  // exchange density (RHF: D)
  const double* Y;  // second exchange density (UHF: D_beta) or NULL
  double xfac;
  int n, pure, boys;
  double* grad;  // [3 natom]
  const double* boys_cell;
};

template <int LA, int LB, int LC, int LD>
struct GradProg;

#define DSS_DEFINE_GRAD_PROG(la, lb, lc, ld)                                              \
  template <>                                                                            \
  struct GradProg<la, lb, lc, ld> {                                                      \
    static constexpr int NSLOTS = DSS_GRAD_##la##lb##lc##ld##_NSLOTS;                    \
    static constexpr int NACC = DSS_GRAD_##la##lb##lc##ld##_NACC;                        \
    static constexpr int NVLV = DSS_GRAD_##la##lb##lc##ld##_NVLV;                        \
    static constexpr int NPLV = DSS_GRAD_##la##lb##lc##ld##_NPLV;                        \
    __device__ static const uint4* vrr() { return kGradVrr_##la##lb##lc##ld; }           \
    __device__ static const uint4* acc() { return kGradAcc_##la##lb##lc##ld; }           \
    __device__ static const uint4* post() { return kGradPost_##la##lb##lc##ld; }         \
    __device__ static const unsigned short* vlv() { return kGradVrrLv_##la##lb##lc##ld; } \
    __device__ static const unsigned short* plv() { return kGradPostLv_##la##lb##lc##ld; } \
  };
DSS_FOR_EACH_GRAD_CLASS(DSS_DEFINE_GRAD_PROG)
#undef DSS_DEFINE_GRAD_PROG

__device__ __forceinline__ const DssCartFun* cart_fun(int l, int pure) {
  if (pure) return l == 0 ? kGradCF_s0[0] : (l == 1 ? kGradCF_s1[0] : kGradCF_s2[0]);
  return l == 0 ? kGradCF_c0[0] : (l == 1 ? kGradCF_c1[0] : kGradCF_c2[0]);
}

__device__ __forceinline__ double gget(const double* __restrict__ rec, const double* __restrict__ vals, unsigned idx) {
  return idx < 32u ? rec[idx] : vals[idx - 32u];
}

template <int LA, int LB, int LC, int LD>
__host__ __device__ constexpr size_t grad_smem_doubles() {
  constexpr int CA = dss_ncart(LA), CB = dss_ncart(LB), CC = dss_ncart(LC), CD = dss_ncart(LD);
  // values, records, AB/CD, Gc, density blocks (function basis, at most Cartesian sizes)
  return (size_t)GradProg<LA, LB, LC, LD>::NSLOTS + kGradBatch * kRec + 8 + CA * CB * CC * CD +
         2 * (CA * CB + CC * CD + 2 * (CA * CC + CA * CD + CB * CC + CB * CD));
}

template <int LA, int LB, int LC, int LD>
__global__ void __launch_bounds__(32) eri_grad_kernel(GradArgs a) {
  using P = GradProg<LA, LB, LC, LD>;
  constexpr int L = LA + LB + LC + LD + 1;
  constexpr int CA = dss_ncart(LA), CB = dss_ncart(LB), CC = dss_ncart(LC), CD = dss_ncart(LD);
  constexpr int NGC = CA * CB * CC * CD;
  extern __shared__ double smem[];
  const int lane = threadIdx.x & 31;
  const long long gw = blockIdx.x;
  const int task = (int)(gw / kGradSplit);
  const int part = (int)(gw % kGradSplit);
  if (task >= a.ntasks) return;
  double* vals = smem;
  double* recs = vals + P::NSLOTS;
  double* hdr = recs + kGradBatch * kRec;
  double* gc = hdr + 8;
  double* dab = gc + NGC;
  double* dcd = dab + CA * CB;
  double* xac = dcd + CC * CD;
  double* xad = xac + CA * CC;
  double* xbc = xad + CA * CD;
  double* xbd = xbc + CB * CC;
  double* yac = xbd + CB * CD;
  double* yad = yac + CA * CC;
  double* ybc = yad + CA * CD;
  double* ybd = ybc + CB * CC;

  const int4 t = __ldg(a.tasks + task);
  const int per = (t.z + kGradSplit - 1) / kGradSplit;
  const int k_begin = part * per, k_end = min(t.z, k_begin + per);
  if (k_begin >= k_end) return;
  const int pure = a.pure, n = a.n;
  const int NA = pure ? 2 * LA + 1 : CA, NB = pure ? 2 * LB + 1 : CB;
  const int NC = pure ? 2 * LC + 1 : CC, ND = pure ? 2 * LD + 1 : CD;
  const int bra = t.x;
  const int sa = __ldg(a.pair_a + bra), sb = __ldg(a.pair_b + bra);
  const int fa = __ldg(a.sh_f0 + sa), fb = __ldg(a.sh_f0 + sb);
  const int ata = __ldg(a.sh_atom + sa), atb = __ldg(a.sh_atom + sb);
  const int bpp0 = __ldg(a.pair_pp0 + bra), nbp = __ldg(a.pair_npp + bra);
  const DssCartFun* cfa = cart_fun(LA, pure);
  const DssCartFun* cfb = cart_fun(LB, pure);
  const DssCartFun* cfc = cart_fun(LC, pure);
  const DssCartFun* cfd = cart_fun(LD, pure);
  for (int q = lane; q < NA * NB; q += 32) dab[q] = __ldg(a.D + (size_t)(fa + q / NB) * n + fb + q % NB);

  for (int kq = k_begin; kq < k_end; ++kq) {
    const int ket = t.y + kq;
    const int sc = __ldg(a.pair_a + ket), sd = __ldg(a.pair_b + ket);
    const int atc = __ldg(a.sh_atom + sc), atd = __ldg(a.sh_atom + sd);
    if (ata == atb && atb == atc && atc == atd) continue;  // one nucleus: no net force (uniform per warp)
    const int fc = __ldg(a.sh_f0 + sc), fd = __ldg(a.sh_f0 + sd);
    const int kpp0 = __ldg(a.pair_pp0 + ket), nkp = __ldg(a.pair_npp + ket);
    if (lane < 6) {
      const int s0 = lane < 3 ? sa : sc, s1 = lane < 3 ? sb : sd, ax = lane % 3;
      hdr[lane] = __ldg(a.sh_xyz + 3 * s0 + ax) - __ldg(a.sh_xyz + 3 * s1 + ax);
    }
    for (int q = lane; q < P::NACC; q += 32) vals[P::NSLOTS - P::NACC + q] = 0.0;
    __syncwarp();
    const int nprim = nbp * nkp;
    for (int b0 = 0; b0 < nprim; b0 += kGradBatch) {
      const int nb = min(kGradBatch, nprim - b0);
      if (lane < nb) {
        const int pi = b0 + lane;
        const int ib = pi % nbp, ik = pi / nbp;
        const PrimPair bp = load_pp(a.pp + bpp0 + ib);
        const PrimPair kp = load_pp(a.pp + kpp0 + ik);
        double F[L + 1];
        double* r = recs + lane * kRec;
        if (a.boys == DSS_BOYS_REF)
          prim_quartet<DSS_BOYS_REF, L>(bp, kp, F, r[12], r[13], r[14], r[15], r[16], r[17], r[18], r[19], r[20],
                                        r[21], r[22], r[23], r[24], r[25], r[26], r[27], r[28], a.boys_cell);
        else
          prim_quartet<DSS_BOYS_FAST, L>(bp, kp, F, r[12], r[13], r[14], r[15], r[16], r[17], r[18], r[19], r[20],
                                         r[21], r[22], r[23], r[24], r[25], r[26], r[27], r[28], a.boys_cell);
#pragma unroll
        for (int m = 0; m <= L; ++m) r[m] = F[m];
        const double al = __ldg(a.pp_alpha + bpp0 + ib);
        r[29] = 2.0 * al;
        r[30] = 2.0 * (bp.p - al);
        r[31] = 2.0 * __ldg(a.pp_alpha + kpp0 + ik);
      }
      __syncwarp();
      for (int j = 0; j < nb; ++j) {
        const double* __restrict__ r = recs + j * kRec;
        for (int lv = 0; lv < P::NVLV; ++lv) {
          const int o1 = P::vlv()[lv + 1];
          for (int o = P::vlv()[lv] + lane; o < o1; o += 32) {
            const uint4 op = P::vrr()[o];
            const unsigned dst = op.x & 0xFFFFu, s0 = op.x >> 16, s1 = op.y & 0xFFFFu, s2 = op.y >> 16;
            const unsigned s3 = op.z & 0xFFFFu, s4 = op.z >> 16;
            const unsigned kind = op.w & 15u, ax = (op.w >> 4) & 3u;
            const double k1 = (double)((op.w >> 8) & 0xFFu), k2 = (double)((op.w >> 16) & 0xFFu);
            double v;
            if (kind == 0u) {
              v = r[12 + ax] * gget(r, vals, s0) + r[15 + ax] * gget(r, vals, s1);
              if (s2 != 0xFFFFu) v += k1 * r[24] * (gget(r, vals, s2) - r[27] * gget(r, vals, s3));
            } else {
              v = r[18 + ax] * gget(r, vals, s0) + r[21 + ax] * gget(r, vals, s1);
              if (s2 != 0xFFFFu) v += k1 * r[25] * (gget(r, vals, s2) - r[28] * gget(r, vals, s3));
              if (s4 != 0xFFFFu) v += k2 * r[26] * gget(r, vals, s4);
            }
            vals[dst - 32u] = v;
          }
          __syncwarp();
        }
        for (int o = lane; o < P::NACC; o += 32) {
          const uint4 op = P::acc()[o];
          const unsigned w = op.y & 0xFFFFu;
          const double v = gget(r, vals, op.x >> 16);
          vals[(op.x & 0xFFFFu) - 32u] += (w == 0xFFFFu ? v : r[w] * v);
        }
        __syncwarp();
      }
    }
    // Two-particle density of the quartet, function basis -> Cartesian (Gc).
    double s = 4.0;
    if (sa == sb) s *= 0.5;
    if (sc == sd) s *= 0.5;
    if (bra == ket) s *= 0.5;
    for (int q = lane; q < NC * ND; q += 32) dcd[q] = __ldg(a.D + (size_t)(fc + q / ND) * n + fd + q % ND);
    for (int q = lane; q < NA * NC; q += 32) xac[q] = __ldg(a.X + (size_t)(fa + q / NC) * n + fc + q % NC);
    for (int q = lane; q < NA * ND; q += 32) xad[q] = __ldg(a.X + (size_t)(fa + q / ND) * n + fd + q % ND);
    for (int q = lane; q < NB * NC; q += 32) xbc[q] = __ldg(a.X + (size_t)(fb + q / NC) * n + fc + q % NC);
    for (int q = lane; q < NB * ND; q += 32) xbd[q] = __ldg(a.X + (size_t)(fb + q / ND) * n + fd + q % ND);
    if (a.Y) {
      for (int q = lane; q < NA * NC; q += 32) yac[q] = __ldg(a.Y + (size_t)(fa + q / NC) * n + fc + q % NC);
      for (int q = lane; q < NA * ND; q += 32) yad[q] = __ldg(a.Y + (size_t)(fa + q / ND) * n + fd + q % ND);
      for (int q = lane; q < NB * NC; q += 32) ybc[q] = __ldg(a.Y + (size_t)(fb + q / NC) * n + fc + q % NC);
      for (int q = lane; q < NB * ND; q += 32) ybd[q] = __ldg(a.Y + (size_t)(fb + q / ND) * n + fd + q % ND);
    }
    __syncwarp();
    const double xf = a.xfac;
    const bool uy = a.Y != nullptr;
    for (int g = lane; g < NGC; g += 32) {
      const int cd_ = g % CD, cc_ = (g / CD) % CC, cb_ = (g / (CD * CC)) % CB, ca_ = g / (CD * CC * CB);
      double acc = 0.0;
      for (int u = 0; u < 3; ++u) {
        const DssCartFun ea = cfa[3 * ca_ + u];
        if (ea.f < 0) break;
        for (int v = 0; v < 3; ++v) {
          const DssCartFun eb = cfb[3 * cb_ + v];
          if (eb.f < 0) break;
          for (int x = 0; x < 3; ++x) {
            const DssCartFun ec = cfc[3 * cc_ + x];
            if (ec.f < 0) break;
            for (int y = 0; y < 3; ++y) {
              const DssCartFun ed = cfd[3 * cd_ + y];
              if (ed.f < 0) break;
              const int i = ea.f, j = eb.f, k = ec.f, l = ed.f;
              double gm = dab[i * NB + j] * dcd[k * ND + l] -
                          xf * (xac[i * NC + k] * xbd[j * ND + l] + xad[i * ND + l] * xbc[j * NC + k]);
              if (uy) gm -= xf * (yac[i * NC + k] * ybd[j * ND + l] + yad[i * ND + l] * ybc[j * NC + k]);
              acc += ea.w * eb.w * ec.w * ed.w * gm;
            }
          }
        }
      }
      gc[g] = s * acc;
    }
    __syncwarp();
    // HRR to the shifted classes and the contraction into the nine sums.
    double gsum[9];
#pragma unroll
    for (int d = 0; d < 9; ++d) gsum[d] = 0.0;
    for (int lv = 0; lv < P::NPLV; ++lv) {
      const int o1 = P::plv()[lv + 1];
      for (int o = P::plv()[lv] + lane; o < o1; o += 32) {
        const uint4 op = P::post()[o];
        const unsigned kind = op.w & 15u;
        if (kind == 2u) {
          const unsigned dst = op.x & 0xFFFFu, s0 = op.x >> 16, s1 = op.y & 0xFFFFu;
          const unsigned ax = (op.w >> 4) & 3u, side = (op.w >> 6) & 1u;
          vals[dst - 32u] = vals[s0 - 32u] + hdr[3 * side + ax] * vals[s1 - 32u];
        } else {
          const unsigned dir = op.x & 0xFFFFu, sp = op.x >> 16, sm = op.y & 0xFFFFu, gi = op.y >> 16;
          double v = vals[sp - 32u];
          if (sm != 0xFFFFu) v -= (double)((op.w >> 8) & 0xFFu) * vals[sm - 32u];
          const double c = gc[gi] * v;
#pragma unroll
          for (int d = 0; d < 9; ++d) gsum[d] += (dir == (unsigned)d) ? c : 0.0;
        }
      }
      __syncwarp();
    }
#pragma unroll
    for (int d = 0; d < 9; ++d) gsum[d] = warp_sum(gsum[d]);
    if (lane == 0) {
      const int at[3] = {ata, atb, atc};
#pragma unroll
      for (int c = 0; c < 3; ++c)
#pragma unroll
        for (int i = 0; i < 3; ++i) atomicAdd(a.grad + 3 * at[c] + i, gsum[3 * c + i]);
#pragma unroll
      for (int i = 0; i < 3; ++i) atomicAdd(a.grad + 3 * atd + i, -(gsum[i] + gsum[3 + i] + gsum[6 + i]));
    }
    __syncwarp();
  }
}

template <int LA, int LB, int LC, int LD>
cudaError_t launch_grad(const GradArgs& a, cudaStream_t s) {
  const size_t smem = grad_smem_doubles<LA, LB, LC, LD>() * sizeof(double);
  static std::atomic<bool> attr[64] = {};
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev < 0 || dev >= 64 || !attr[dev].load()) {
    const cudaError_t e =
        cudaFuncSetAttribute(eri_grad_kernel<LA, LB, LC, LD>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    if (dev >= 0 && dev < 64) attr[dev].store(true);
  }
  const long long blocks = (long long)a.ntasks * kGradSplit;
  if (blocks <= 0) return cudaSuccess;
  eri_grad_kernel<LA, LB, LC, LD><<<(unsigned)blocks, 32, smem, s>>>(a);
  return cudaGetLastError();
}

cudaError_t launch_grad_class(int la, int lb, int lc, int ld, const GradArgs& a, cudaStream_t s) {
#define DSS_GRAD_DISPATCH(la_, lb_, lc_, ld_) \
  if (la == la_ && lb == lb_ && lc == lc_ && ld == ld_) return launch_grad<la_, lb_, lc_, ld_>(a, s);
  DSS_FOR_EACH_GRAD_CLASS(DSS_GRAD_DISPATCH)
#undef DSS_GRAD_DISPATCH
  return cudaErrorInvalidValue;
}

__global__ void unpack_packed(const double* __restrict__ p, double* __restrict__ d, int n) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long long)n * n) return;
  const int r = (int)(t / n), c = (int)(t % n);
  const int lo = r < c ? r : c, hi = r < c ? c : r;
  d[t] = p[(size_t)hi * (hi + 1) / 2 + lo];
}

}  // namespace

int dss_eri_gradient_dense(dss_ctx* ctx, const double* D_dev, const double* X_dev, const double* Y_dev, double xfac,
                           int natom, const int* shell_atom, double* grad_host) {
  if (ctx->nmol > 0 || ctx->nbf == 0)
    return dss_fail(ctx, DSS_ERR_INVALID, "dss_eri_gradient: needs a context with one molecule's basis");
  if (DSS_GEN_LMAX > 2) return dss_fail(ctx, DSS_ERR_UNSUPPORTED, "dss_eri_gradient: compiled for l <= 2 only");
  const int ns = ctx->nshell;
  for (int s = 0; s < ns; ++s)
    if (shell_atom[s] < 0 || shell_atom[s] >= natom)
      return dss_fail(ctx, DSS_ERR_INVALID, "dss_eri_gradient: shell_atom out of range");
  cudaStream_t s = ctx->stream;
  std::vector<double> alpha;
  dss_pair_alphas(ctx, &alpha);
  DevBuf<double> d_alpha, d_grad;
  DevBuf<int> d_atom;
  if (d_alpha.resize(std::max<size_t>(alpha.size(), 1)) != cudaSuccess || d_grad.resize(3 * (size_t)natom) != cudaSuccess ||
      d_atom.resize(ns) != cudaSuccess)
    return dss_fail(ctx, DSS_ERR_OOM, "dss_eri_gradient: device allocation failed");
  cudaError_t e = cudaMemcpyAsync(d_alpha.ptr, alpha.data(), alpha.size() * 8, cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess) e = cudaMemcpyAsync(d_atom.ptr, shell_atom, ns * sizeof(int), cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess) e = cudaMemsetAsync(d_grad.ptr, 0, 3 * (size_t)natom * 8, s);
  if (e != cudaSuccess) return dss_fail(ctx, DSS_ERR_CUDA, std::string("dss_eri_gradient: ") + cudaGetErrorString(e));
  GradArgs a{};
  a.pair_a = ctx->d_pair_a.ptr;
  a.pair_b = ctx->d_pair_b.ptr;
  a.pair_pp0 = ctx->d_pair_pp0.ptr;
  a.pair_npp = ctx->d_pair_npp.ptr;
  a.pp = ctx->d_pp.ptr;
  a.pp_alpha = d_alpha.ptr;
  a.sh_xyz = ctx->d_sh_xyz.ptr;
  a.sh_f0 = ctx->d_sh_f0.ptr;
  a.sh_atom = d_atom.ptr;
  a.D = D_dev;
  a.X = X_dev;
  a.Y = Y_dev;
  a.xfac = xfac;
  a.n = ctx->nbf;
  a.pure = ctx->pure;
  a.boys = ctx->opts.boys_mode;
  a.grad = d_grad.ptr;
  a.boys_cell = ctx->boys_cell;
  for (const ClassTasks& ct : ctx->tasks) {
    if (!ct.ntasks) continue;
    a.tasks = ct.d_tasks.ptr;
    a.ntasks = ct.ntasks;
    e = launch_grad_class(ct.la, ct.lb, ct.lc, ct.ld, a, s);
    if (e != cudaSuccess)
      return dss_fail(ctx, DSS_ERR_CUDA, std::string("dss_eri_gradient: launch: ") + cudaGetErrorString(e));
  }
  e = cudaMemcpyAsync(grad_host, d_grad.ptr, 3 * (size_t)natom * 8, cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return dss_fail(ctx, DSS_ERR_CUDA, std::string("dss_eri_gradient: ") + cudaGetErrorString(e));
  return DSS_OK;
}

extern "C" int dss_eri_gradient(dss_ctx* ctx, const double* D_packed, const double* Da_packed,
                                const double* Db_packed, int natom, const int* shell_atom, double* grad) {
  if (!ctx) return DSS_ERR_INVALID;
  ctx->err.clear();
  if (!D_packed || !shell_atom || !grad || natom <= 0)
    return dss_fail(ctx, DSS_ERR_INVALID, "dss_eri_gradient: NULL array or no nuclei");
  if ((Da_packed == nullptr) != (Db_packed == nullptr))
    return dss_fail(ctx, DSS_ERR_INVALID, "dss_eri_gradient: give both spin densities or neither");
  const int n = ctx->nbf;
  if (n == 0 || ctx->nmol > 0) return dss_fail(ctx, DSS_ERR_INVALID, "dss_eri_gradient: no single-molecule basis set");
  const size_t n2 = (size_t)n * n, np = (size_t)n * (n + 1) / 2;
  const bool uhf = Da_packed != nullptr;
  DevBuf<double> packed, dense;
  if (packed.resize(np) != cudaSuccess || dense.resize((uhf ? 3 : 1) * n2) != cudaSuccess)
    return dss_fail(ctx, DSS_ERR_OOM, "dss_eri_gradient: device allocation failed");
  cudaStream_t s = ctx->stream;
  const double* srcs[3] = {D_packed, Da_packed, Db_packed};
  for (int k = 0; k < (uhf ? 3 : 1); ++k) {
    cudaError_t e = cudaMemcpyAsync(packed.ptr, srcs[k], np * 8, cudaMemcpyHostToDevice, s);
    if (e != cudaSuccess) return dss_fail(ctx, DSS_ERR_CUDA, std::string("dss_eri_gradient: ") + cudaGetErrorString(e));
    unpack_packed<<<(unsigned)((n2 + 255) / 256), 256, 0, s>>>(packed.ptr, dense.ptr + k * n2, n);
  }
  std::vector<double> g(3 * (size_t)natom);
  const int rc = uhf ? dss_eri_gradient_dense(ctx, dense.ptr, dense.ptr + n2, dense.ptr + 2 * n2, 0.5, natom,
                                              shell_atom, g.data())
                     : dss_eri_gradient_dense(ctx, dense.ptr, dense.ptr, nullptr, 0.25, natom, shell_atom, g.data());
  if (rc != DSS_OK) return rc;
  for (size_t i = 0; i < g.size(); ++i) grad[i] += g[i];
  return DSS_OK;
}
