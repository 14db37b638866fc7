/*
 * ref_harness.cpp -- stable C entry points around the reference functions
 * that oracle/make_ref.py lifts out of the reference tree into
 * oracle/_ref/ (see that script for the list and the shapes).
 * TEST INFRASTRUCTURE ONLY: the tests load oracle/_ref/libref.so to pin the
 * oracle restatement (oracle/*.c, oracle/oracle.py) to the reference's own
 * code, and bench.py's reference arm times the reorders with it.  The
 * product library never loads it.
 *
 * The flagger's element kernels (scaley, flag, flagts) and the cuBLAS
 * beamformer's populate_weights_matrix are CUDA kernels in the reference;
 * they read only blockIdx.x / threadIdx.x and global memory (no shared
 * memory, no barriers), so running every (block, thread) pair in turn on
 * the host computes what their launches compute (up to the device's float
 * cos/sin, which differ from the host's in the last bits).
 */
#include "ref_stubs.h"

extern "C" {
int DEBUG = 0;
// The reference pins reorder thread i to cores[i] of its production hosts
// (src/dsaX_reorder_raw.c:54); here thread i goes to core i.
int cores[16] = {0, 1, 2, 3, 4, 5, 6, 7, 8, 9, 10, 11, 12, 13, 14, 15};
}
thread_local ref_dim3 blockIdx, threadIdx;

// reference functions (src/gpu_flagger.cu), compiled in ref_flagger.cpp
float medval(float *a, int n);
void channflag(float *spec, float Thr, int *mask);
void simple_channflag(float *spec, float Thr, int *mask);
void simple_tsflag(float *spec, float Thr, int *mask);
void gather_mask(int *h_idx, int *h_mask, int *n_mask);
void gather_tsmask(int *h_idx, int *h_mask, int *n_mask);
void calc_bpwr(float *h_spec, float *h_bpwr);
void median_calc(float *arr);
void scaley(unsigned char *data, float *spectrum, float *varspec);
// src/dsaX_bfCorr.cu, compiled in ref_bfcorr.cpp (half stored as float)
void populate_weights_matrix(float *antpos_e, float *antpos_n, float *calibs, float *wr, float *wi,
                             float *fqs, float dec);
void flag(unsigned char *data, int *midx, unsigned char *repval, float *bpwr);
void flagts(unsigned char *data, int *midx, unsigned char *repval, float *bpwr);

extern "C" {
// src/dsaX_wrangle.c, src/dsaX_wrangleAndWrite.c (ref_wrangle.c)
void auto_extract(float *output, float *specs);
void simple_extract(Complex *mat, float *output);
void gen_lookup(int *idx_xgpu_in_greg);
void reorder_gh(float *input, float *output, int *idx_xgpu_in_greg);
// src/dsaX_reorder_raw.c(.bak) massage(), run on nthreads threads
int massage_run_raw(const char *in, char *out, int nthreads);
int massage_run_bak(const char *in, char *out, int nthreads);

void ref_flag_shape(int *nbeam, int *ntime, int *nchan) {
  *nbeam = NBEAMS_P;
  *ntime = NTIMES_P;
  *nchan = NCHAN_P;
}
int ref_npackets(void) { return NPACKETS; }
int ref_nants(void) { return NANTS; }

float ref_medval(float *a, int n) { return medval(a, n); }
void ref_channflag(float *spec, float thr, int *mask) { channflag(spec, thr, mask); }
void ref_simple_channflag(float *spec, float thr, int *mask) { simple_channflag(spec, thr, mask); }
void ref_simple_tsflag(float *ts, float thr, int *mask) { simple_tsflag(ts, thr, mask); }
void ref_gather_mask(int *idx, int *mask, int *n) { gather_mask(idx, mask, n); }
void ref_gather_tsmask(int *idx, int *mask, int *n) { gather_tsmask(idx, mask, n); }
void ref_calc_bpwr(float *spec, float *bpwr) { calc_bpwr(spec, bpwr); }
void ref_median_calc(float *arr) { median_calc(arr); }

// scaley<<<NBEAMS_P*NTIMES_P*NCHAN_P/32, 32>>> (src/gpu_flagger.cu:1297)
void ref_scaley(unsigned char *data, float *spec0, float *var0) {
  const long long nblk = (long long)NBEAMS_P * NTIMES_P * NCHAN_P / 32;
  for (long long b = 0; b < nblk; ++b)
    for (int t = 0; t < 32; ++t) {
      blockIdx.x = (int)b;
      threadIdx.x = t;
      scaley(data, spec0, var0);
    }
}
// flag<<<n_mask*NTIMES_P/32, 32>>> (src/gpu_flagger.cu:1379)
void ref_flag(unsigned char *data, int *midx, int n_mask, float *bpwr) {
  const long long nblk = (long long)n_mask * NTIMES_P / 32;
  for (long long b = 0; b < nblk; ++b)
    for (int t = 0; t < 32; ++t) {
      blockIdx.x = (int)b;
      threadIdx.x = t;
      flag(data, midx, nullptr, bpwr);
    }
}
// flagts<<<n_tsmask*(NCHAN_P-256)/32, 32>>> (src/gpu_flagger.cu:1395)
void ref_flagts(unsigned char *data, int *midx, int n_mask, float *bpwr) {
  const long long nblk = (long long)n_mask * (NCHAN_P - 256) / 32;
  for (long long b = 0; b < nblk; ++b)
    for (int t = 0; t < 32; ++t) {
      blockIdx.x = (int)b;
      threadIdx.x = t;
      flagts(data, midx, nullptr, bpwr);
    }
}

// populate_weights_matrix<<<2*(NCHAN_PER_PACKET/8)*(NBEAMS/2)*128*(NANTS/2)/128, 128>>>
// (src/dsaX_bfCorr.cu:921): wr / wi [2 arms][NCHAN_PER_PACKET/8][NBEAMS/2]
// [4 t][NANTS/2][8 ch][2 t][2 pol]
void ref_bfcorr_shape(int *nants, int *ngrp, int *nbeams) {
  *nants = NANTS_BF;
  *ngrp = NCHAN_PER_PACKET / 8;
  *nbeams = NBEAMS;
}
void ref_populate_weights(float *antpos_e, float *antpos_n, float *calibs, float *wr, float *wi,
                          float *fqs, float dec) {
  const long long nblk = 2LL * (NCHAN_PER_PACKET / 8) * (NBEAMS / 2) * 128 * (NANTS_BF / 2) / 128;
  for (long long b = 0; b < nblk; ++b)
    for (int t = 0; t < 128; ++t) {
      blockIdx.x = (int)b;
      threadIdx.x = t;
      populate_weights_matrix(antpos_e, antpos_n, calibs, wr, wi, fqs, dec);
    }
}

void ref_auto_extract(float *output, float *specs) { auto_extract(output, specs); }
void ref_simple_extract(Complex *mat, float *output) { simple_extract(mat, output); }
void ref_gen_lookup(int *idx) { gen_lookup(idx); }
void ref_reorder_gh(float *in, float *out, int *idx) { reorder_gh(in, out, idx); }
int ref_massage_raw(const char *in, char *out, int nthreads) {
  return massage_run_raw(in, out, nthreads);
}
int ref_massage_bak(const char *in, char *out, int nthreads) {
  return massage_run_bak(in, out, nthreads);
}
}
