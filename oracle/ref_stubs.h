/*
 * ref_stubs.h -- what the reference functions lifted by oracle/make_ref.py
 * need from the headers that are absent here (psrdada, xGPU, CUDA).
 * TEST INFRASTRUCTURE ONLY.
 *
 *  - ipcio_t: only its `curbuf` member is used, by massage()
 *    (src/dsaX_reorder_raw.c:163) to write into the current ring block.
 *  - Complex: xGPU's {float real; float imag;} visibility element, used by
 *    simple_extract() (src/dsaX_wrangle.c:74-93).
 *  - DEBUG, cores[]: globals the reorder threads read
 *    (src/dsaX_reorder_raw.c:53-54); defined in ref_harness.cpp.
 *  - For the flagger's element kernels compiled as host C++: __global__
 *    is empty, blockIdx/threadIdx are per-thread globals the harness sets
 *    before each (block, thread) call, and __float2uint_rn is CUDA's
 *    float -> unsigned int conversion (round to nearest even, saturating
 *    at 0 and UINT_MAX, NaN -> 0).
 */
#ifndef REF_STUBS_H
#define REF_STUBS_H
#ifndef _GNU_SOURCE
#define _GNU_SOURCE
#endif
#include <math.h>
#include <pthread.h>
#include <sched.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <syslog.h>

typedef struct { char *curbuf; } ipcio_t;
typedef struct { float real; float imag; } Complex;

#ifdef __cplusplus
extern "C" {
#endif
extern int DEBUG;
extern int cores[16];
#ifdef __cplusplus
}
#endif

#ifdef __cplusplus
#define __global__
struct ref_dim3 { int x; };
extern thread_local ref_dim3 blockIdx, threadIdx;
static inline unsigned int __float2uint_rn(float v) {
  if (!(v > 0.0f)) return 0u;                       /* negative, zero, NaN */
  if (v >= 4294967296.0f) return 4294967295u;
  return (unsigned int)nearbyint((double)v);        /* default rounding: nearest even */
}
#endif

#endif
