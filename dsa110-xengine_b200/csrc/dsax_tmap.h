// dsax_tmap.h -- the driver's tensor-map encoder (cuTensorMapEncodeTiled),
// reached through the runtime's driver entry point so that the library does
// not link libcuda directly.
#pragma once
#include <cuda.h>
#include <cuda_runtime.h>

namespace dsax {

typedef CUresult (*EncodeTiledFn)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *,
                                  const cuuint64_t *, const cuuint64_t *, const cuuint32_t *,
                                  const cuuint32_t *, CUtensorMapInterleave, CUtensorMapSwizzle,
                                  CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

// The encoder, looked up once (null if the driver does not provide it).
inline EncodeTiledFn tensor_map_encoder() {
  static EncodeTiledFn fn = [] {
    void *p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      return reinterpret_cast<EncodeTiledFn>(p);
    return static_cast<EncodeTiledFn>(nullptr);
  }();
  return fn;
}

}  // namespace dsax
