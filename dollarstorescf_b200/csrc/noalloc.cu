// J/K build that allocates no device memory during the call.
//
// dss_build_jk_device keeps its Coulomb/exchange accumulators in buffers the
// context allocates on first use.  Some callers cannot allow any device
// allocation while they run: code that must not synchronise the device the way
// cudaMalloc/cudaFree can, callers running under a memory pool or budget that
// owns all device memory, and real-time loops that have to stay free of
// allocator latency.  dss_build_jk_device_noalloc gives them the same build with
// the accumulators in a fixed array that is part of the loaded library image
// (every GPU that loads the library holds it until the process exits).
//
// With lazy module loading (the CUDA default since 12.2) the array and a
// kernel's code reach the device on first use, which allocates.  dss_create
// therefore looks up the array's address here (loading it and the symmetrise
// kernel), and dss_set_basis loads the class kernels a build launches, so the
// entry point itself loads and allocates nothing.
#include <cuda_runtime.h>

#include "dss.h"
#include "dss_internal.h"

namespace {

// Two n x n accumulators, n <= DSS_NOALLOC_MAX_NBF (4 MiB).
static __device__ __align__(256) double g_noalloc_acc[2 * DSS_NOALLOC_MAX_NBF * DSS_NOALLOC_MAX_NBF];

__global__ void noalloc_symmetrize(const double* __restrict__ acc, double* __restrict__ out, int n) {
  const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (long long)n * n) return;
  const int r = (int)(idx / n), c = (int)(idx % n);
  out[idx] = acc[(long long)r * n + c] + acc[(long long)c * n + r];
}

}  // namespace

// Set-up with the context's device current (called by dss_create): the array's
// name is a host-side stand-in, the kernels need its device address.  The
// address is kept per context, so a context made after a device reset looks it
// up again.
cudaError_t dss_noalloc_attach(double** acc) {
  void* p = nullptr;
  cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_acc);
  if (e != cudaSuccess) return e;
  cudaFuncAttributes fa;
  e = cudaFuncGetAttributes(&fa, noalloc_symmetrize);
  if (e != cudaSuccess) return e;
  *acc = static_cast<double*>(p);
  return cudaSuccess;
}

extern "C" int dss_build_jk_device_noalloc(dss_ctx* ctx, const double* D, double* J, double* K) {
  if (!ctx) return DSS_ERR_INVALID;
  ctx->err.clear();
  if (!ctx->nbf || ctx->nmol > 0)
    return dss_fail(ctx, DSS_ERR_INVALID, "dss_build_jk_device_noalloc: no single-molecule basis set");
  if (!D) return dss_fail(ctx, DSS_ERR_INVALID, "dss_build_jk_device_noalloc: D is NULL");
  const int n = ctx->nbf;
  if (n > DSS_NOALLOC_MAX_NBF)
    return dss_fail(ctx, DSS_ERR_INVALID,
                    "dss_build_jk_device_noalloc: " + std::to_string(n) + " basis functions exceed the maximum of " +
                        std::to_string(DSS_NOALLOC_MAX_NBF) + " for the built-in accumulators");
  if (!ctx->noalloc_acc)
    return dss_fail(ctx, DSS_ERR_INVALID, "dss_build_jk_device_noalloc: accumulator array not attached");
  cudaError_t e = cudaSetDevice(ctx->opts.device);
  if (e != cudaSuccess) return dss_cuda_check(ctx, e, "dss_build_jk_device_noalloc: cudaSetDevice");
  double* Jacc = ctx->noalloc_acc;
  double* Kacc = ctx->noalloc_acc + (size_t)n * n;
  // dss_enqueue_jk zeroes both accumulators before the ERI launches, so nothing
  // left from an earlier call reaches the result.
  int rc = dss_enqueue_jk(ctx, D, Jacc, Kacc);
  if (rc != DSS_OK) return rc;
  const long long nn = (long long)n * n;
  const unsigned blocks = (unsigned)((nn + 255) / 256);
  if (J) noalloc_symmetrize<<<blocks, 256, 0, ctx->stream>>>(Jacc, J, n);
  if (K) noalloc_symmetrize<<<blocks, 256, 0, ctx->stream>>>(Kacc, K, n);
  e = cudaGetLastError();
  if (e != cudaSuccess) return dss_cuda_check(ctx, e, "dss_build_jk_device_noalloc: launch");
  return DSS_OK;
}
