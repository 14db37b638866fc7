// dsax_probe.cu -- dense tensor-core throughput of this GPU, measured with
// the instruction forms the kernels use, so that the correlator's int8 and
// the beamformer's FP8 work can be stated as a fraction of a measured peak
// (the pool measures only HBM copy bandwidth and cuBLAS BF16).
//
// One CTA per SM (its dynamic shared memory keeps a second one off the SM)
// issues back-to-back tcgen05.mma M=128 N=256 from a 48 KB operand tile into
// two 256-column TMEM accumulators, then waits for the last one (bounded)
// and frees TMEM.  kind::i8 uses K = 32 bytes, kind::f16 (BF16) K = 16,
// kind::f8f6f4 (E4M3) K = 32 per instruction.  ops = 2 M N K per MMA.
#include <cstdint>
#include <cuda_runtime.h>

#include "../../include/dsax.h"
#include "dsax_ctx.h"
#include "dsax_internal.h"
#include "dsax_ptx.cuh"

namespace dsax {
namespace probe {
constexpr int kThreads = 128;
constexpr int kOperandBytes = 48 * 1024;     // A: 128 x 128 B, B: 256 x 128 B
constexpr int kSmemBytes = 1024 + 120 * 1024;  // > half an SM: one CTA per SM
}  // namespace probe

template <int KIND>
__global__ void __launch_bounds__(probe::kThreads, 1) probe_mma_kernel(int nmma, int *err,
                                                                        uint64_t limit_ns) {
  extern __shared__ uint8_t smem_raw[];
  __shared__ __align__(8) uint64_t bar;
  __shared__ uint32_t tbase;
  __shared__ volatile int abort_sh;
  const int tid = threadIdx.x, warp = tid >> 5;
  const uint32_t base = (smem_u32(smem_raw) + 1023u) & ~1023u;
  uint8_t *g = smem_raw + (base - smem_u32(smem_raw));
  // small operand values (finite in BF16 and E4M3), so the pipe does real work
  for (int i = tid; i < probe::kOperandBytes; i += probe::kThreads)
    g[i] = (uint8_t)((i * 37 + 11) & 0x3F);
  if (tid == 0) {
    mbar_init(&bar, 1);
    abort_sh = 0;
    mbar_fence_init();
  }
  if (warp == 0) {
    tmem_alloc(&tbase, 512);
    tmem_relinquish();
  }
  fence_proxy_async_smem();
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = tbase;
  if (tid == 0) {
    constexpr uint32_t idesc = KIND == 0 ? umma_idesc(2, 1, 1, 128, 256)    // s8 -> s32
                               : KIND == 1 ? umma_idesc(1, 1, 1, 128, 256)  // bf16 -> f32
                                           : umma_idesc(1, 0, 0, 128, 256); // e4m3 -> f32
    const uint32_t a = base, b = base + 16384u;
    for (int i = 0; i < nmma; ++i) {
      const uint32_t d = tmem + 256u * (uint32_t)(i & 1);
      const uint32_t koff = 32u * (uint32_t)((i >> 1) & 3);
      const uint64_t ad = umma_desc_sw128(a + koff, 1024u), bd = umma_desc_sw128(b + koff, 1024u);
      if constexpr (KIND == 0)
        umma_i8(d, ad, bd, idesc, i >= 2);
      else if constexpr (KIND == 1)
        umma_f16(d, ad, bd, idesc, i >= 2);
      else
        umma_f8(d, ad, bd, idesc, i >= 2);
    }
    umma_commit(&bar);
    volatile int no_abort = 0;
    mbar_wait_bounded(&bar, 0u, &no_abort, err, DEV_ERR_WAIT_ACCUM, drain_limit(limit_ns));
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  if (warp == 0) tmem_dealloc(tmem, 512);
}

// A wait on an mbarrier that nothing arrives on: the bounded wait must give
// up after limit_ns, record DEV_ERR_WAIT_FULL in the error word and return.
__global__ void wait_check_kernel(int *err, uint64_t limit_ns) {
  __shared__ __align__(8) uint64_t bar;
  __shared__ volatile int abort_sh;
  if (threadIdx.x == 0) {
    mbar_init(&bar, 1);
    abort_sh = 0;
    mbar_fence_init();
    mbar_wait_bounded(&bar, 0u, &abort_sh, err, DEV_ERR_WAIT_FULL, limit_ns);
  }
}

template <int KIND>
static int probe_launch(int grid, int nmma, int *err, uint64_t limit, cudaStream_t st) {
  static SmemAttrOnce attr;
  if (smem_attr_once(attr, probe_mma_kernel<KIND>, probe::kSmemBytes) != cudaSuccess) return -2;
  probe_mma_kernel<KIND><<<grid, probe::kThreads, probe::kSmemBytes, st>>>(nmma, err, limit);
  return cudaGetLastError() == cudaSuccess ? 0 : -2;
}

}  // namespace dsax

using namespace dsax;

extern "C" int dsax_probe_tensor_peak(dsax_ctx *c, int kind, int reps, double *ops_per_s) {
  if (!c || !ops_per_s || kind < 0 || kind > 2 || reps < 1) return DSAX_ERR_ARG;
  DeviceGuard g(c->device);
  const int nmma = 8192, grid = c->num_sms;
  const double k = kind == 1 ? 16.0 : 32.0;
  const double ops = 2.0 * 128.0 * 256.0 * k * nmma * grid;
  auto launch = [&]() {
    return kind == 0 ? probe_launch<0>(grid, nmma, c->d_err, c->cfg.wait_limit_ns, c->stream)
           : kind == 1 ? probe_launch<1>(grid, nmma, c->d_err, c->cfg.wait_limit_ns, c->stream)
                       : probe_launch<2>(grid, nmma, c->d_err, c->cfg.wait_limit_ns, c->stream);
  };
  cudaEvent_t e0, e1;
  if (cudaEventCreate(&e0) != cudaSuccess) return cuda_check(c, cudaGetLastError(), "event");
  if (cudaEventCreate(&e1) != cudaSuccess) {
    cudaEventDestroy(e0);
    return cuda_check(c, cudaGetLastError(), "event");
  }
  double best = 0.0;
  int rc = DSAX_OK;
  for (int r = 0; r <= reps && rc == DSAX_OK; ++r) {   // the first launch warms up
    cudaEventRecord(e0, c->stream);
    if (launch() != 0) {
      rc = cuda_check(c, cudaGetLastError(), "probe launch");
      break;
    }
    cudaEventRecord(e1, c->stream);
    if ((rc = dsax_sync(c)) != DSAX_OK) break;
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    if (r > 0 && ms > 0.f && ops / (ms * 1e-3) > best) best = ops / (ms * 1e-3);
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  *ops_per_s = best;
  return rc;
}

extern "C" int dsax_check_wait_limit(dsax_ctx *c, unsigned long long limit_ns) {
  if (!c || limit_ns == 0 || limit_ns > 10000000000ull) return DSAX_ERR_ARG;
  DeviceGuard g(c->device);
  wait_check_kernel<<<1, 32, 0, c->stream>>>(c->d_err, limit_ns);
  const int rc = cuda_check(c, cudaGetLastError(), "wait check launch");
  if (rc != DSAX_OK) return rc;
  return dsax_sync(c);
}
