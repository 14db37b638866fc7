/*
 * xgpu_dsax.h -- the xGPU call shapes used by the reference, implemented by
 * libdsax.so on sm_100a tensor cores.
 *
 * Names, argument order and meanings follow the call sites only
 * (src/dsaX_xgpu.cu:253-287,312-340 and src/cuda_correlator.cu:161-294 of
 * dsa110-xengine; the dsa110 fork of xGPU takes the device input pointer as
 * the second argument of xgpuCudaXengine).  No xGPU code is used.  Geometry
 * is the one the reference builds xGPU with (README.md:38-55):
 * NPOL 2, NSTATION 64, NFREQUENCY 768, NTIME 2048, triangular output.
 *
 * Input (device): ComplexInput [NTIME][NFREQUENCY][NSTATION][NPOL]
 * (8-bit real, imag) -- what the reference's promoter writes.
 * Output: triangular [NFREQUENCY][2080][NPOL][NPOL] Complex (float),
 * V_ij = sum_t x_i conj(x_j), j <= i, integrated on the device across calls
 * until xgpuClearDeviceIntegrationBuffer.
 */
#ifndef XGPU_DSAX_H
#define XGPU_DSAX_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct { int8_t real, imag; } ComplexInput;
typedef struct { float real, imag; } Complex;

#define SYNCOP_NONE 0
#define SYNCOP_DUMP 1
#define SYNCOP_SYNC_TRANSFER 2
#define SYNCOP_SYNC_COMPUTE 3

#define TRIANGULAR_ORDER 1000

typedef struct XGPUInfo {
    unsigned int npol, nstation, nbaseline, nfrequency, ntime, ntimepipe;
    size_t vecLength;     /* ComplexInput elements per integration   */
    size_t vecLengthPipe; /* per transfer (ntimepipe time samples)   */
    size_t matLength;     /* Complex elements of the output matrix   */
    size_t triLength;     /* same (triangular order)                 */
    int matrix_order;     /* TRIANGULAR_ORDER                        */
} XGPUInfo;

typedef struct XGPUContext {
    ComplexInput *array_h; /* pinned host input buffer (array_len elements) */
    Complex *matrix_h;     /* pinned host output matrix (matrix_len)        */
    size_t array_len, matrix_len;
    void *internal;        /* library state                                 */
} XGPUContext;

/* xgpuInfo: sizes of the compiled geometry (src/dsaX_xgpu.cu:256). */
void xgpuInfo(XGPUInfo *info);
/* xgpuInit: device buffers, pinned array_h / matrix_h (allocated here when
 * NULL), integration buffer cleared.  Returns 0 or a nonzero error. */
int xgpuInit(XGPUContext *context, int device_flags);
/* xgpuCudaXengine: correlate one integration from device memory and add it
 * to the device integration buffer; SYNCOP_DUMP copies the buffer to
 * matrix_h and waits (src/dsaX_xgpu.cu:318).  Returns 0 or an error. */
int xgpuCudaXengine(XGPUContext *context, ComplexInput *array_d, int syncOp);
/* xgpuClearDeviceIntegrationBuffer: zero the integration (src/dsaX_xgpu.cu:336). */
void xgpuClearDeviceIntegrationBuffer(XGPUContext *context);
/* xgpuReorderMatrix: no-op -- the output is already in triangular order. */
void xgpuReorderMatrix(Complex *matrix);
/* xgpuFree: release everything xgpuInit allocated. */
void xgpuFree(XGPUContext *context);

#ifdef __cplusplus
}
#endif
#endif /* XGPU_DSAX_H */
