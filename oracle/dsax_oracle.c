/*
 * dsax_oracle.c -- CPU restatement of the DSA-110 X-engine hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker that the CUDA library
 * is compared against.  Nothing in the product path (libdsax.so, the C-ABI,
 * the dsax_xengine host program) links, loads or calls it; only tests/,
 * __graft_entry__.smoke() and bench.py's CPU-baseline leg do.
 *
 * Parity status (which outputs are pinned by what):
 *  - 4-bit decode: pinned by the reference's own decoder (utils/gen_packet.py
 *    make_spectrum/make_histogram) run on utils/packet.out; fixture in
 *    tests/golden/packet_decode.json.
 *  - reorder/fluff layout: pinned by utils/test.out (the 8-bit reorder
 *    output of a tone packet); fixture in tests/golden/reorder_tone.json.
 *  - correlator arithmetic: the xGPU library that computes it is not in the
 *    reference tree (un-vendored dsa110-xGPU, no pinned version).  The
 *    convention restated here (V_ij = sum_t x_i conj(x_j), i >= j,
 *    pol product index 2*pol_i + pol_j, triangular baseline i(i+1)/2 + j,
 *    f' = 2*chan + time) follows the reference's own restatement in
 *    src/dsaX_bfCorr.cu:442-447,509-552 and the consumers
 *    src/dsaX_writevis.c:55-74, src/dsaX_wrangleAndWrite.c:46-57.  The
 *    cross-hand ordering (pp=1 vs 2) is pinned by convention only.
 *  - beamformer: src/dsaX_beamformer.cu:267-416 (beam = sum_a w*x, no
 *    conjugate; power summed over 8 channels x 2 times x 2 pols x packets).
 *  - plain flagger: src/gpu_flagger.cu:175-798 (statistics and host
 *    median/MAD flagging), parameterised for other shapes.
 *
 * Build: gcc -O3 -march=native -fopenmp -shared -fPIC (oracle/Makefile).
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#ifdef _OPENMP
#include <omp.h>
#endif

#define NST 64             /* stations in the xGPU products */
#define NBL (NST * (NST + 1) / 2)  /* 2080 baselines */

/* ------------------------------------------------------------------ */
/* a1: sample decode. src/dsaX_xgpu.cu:74-75: real = low nibble,      */
/* imag = high nibble, both 4-bit two's complement.                   */
/* ------------------------------------------------------------------ */
static inline int lo4(uint8_t b) { return (int)((b & 0x0F) ^ 0x08) - 8; }
static inline int hi4(uint8_t b) { return (int)((b >> 4) ^ 0x08) - 8; }

int oracle_version(void) { return 1; }

int oracle_nthreads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

/* The xGPU-stage promoter, src/dsaX_xgpu.cu:67-77: byte i -> out[2i] =
 * real, out[2i+1] = imag. */
void oracle_promote(const uint8_t *in, int8_t *out, int64_t n) {
    for (int64_t i = 0; i < n; i++) {
        out[2 * i] = (int8_t)lo4(in[i]);
        out[2 * i + 1] = (int8_t)hi4(in[i]);
    }
}

/* a3: massage(), src/dsaX_reorder_raw.c:153-169.  Captured layout
 * [pkt][nant_in][nchan][2 t][2 pol] (one packed byte per sample) is byte-
 * reordered to the xGPU input order [pkt][2*nchan][64][2 pol], still 4-bit
 * packed.  Antennas >= nant_in are zero-filled here; the reference leaves
 * them as whatever the ring buffer held (zero in a fresh buffer). */
void oracle_massage(const uint8_t *in, uint8_t *out, int npkt, int nant_in,
                    int nchan) {
    const int64_t nk = 2 * (int64_t)nchan;
#pragma omp parallel for schedule(static)
    for (int p = 0; p < npkt; p++) {
        uint8_t *o = out + (int64_t)p * nk * NST * 2;
        memset(o, 0, (size_t)(nk * NST * 2));
        for (int a = 0; a < nant_in; a++) {
            const uint8_t *s = in + ((int64_t)p * nant_in + a) * nk * 2;
            for (int64_t k = 0; k < nk; k++) {
                o[(k * NST + a) * 2 + 0] = s[k * 2 + 0];
                o[(k * NST + a) * 2 + 1] = s[k * 2 + 1];
            }
        }
    }
}

/* a4: AVX-512 fluff + word transpose, src/dsaX_reorder_raw.c.bak:184-258
 * (and src/dsaX_reorder.c:96-252).  Output [pkt][2*nchan][64][2 pol]
 * [re, im] int8 -- the 8-bit ComplexInput vector xGPU consumes. */
void oracle_fluff_reorder(const uint8_t *in, int8_t *out, int npkt,
                          int nant_in, int nchan) {
    const int64_t nk = 2 * (int64_t)nchan;
#pragma omp parallel for schedule(static)
    for (int p = 0; p < npkt; p++) {
        int8_t *o = out + (int64_t)p * nk * NST * 4;
        memset(o, 0, (size_t)(nk * NST * 4));
        for (int a = 0; a < nant_in; a++) {
            const uint8_t *s = in + ((int64_t)p * nant_in + a) * nk * 2;
            for (int64_t k = 0; k < nk; k++) {
                for (int pol = 0; pol < 2; pol++) {
                    uint8_t b = s[k * 2 + pol];
                    o[((k * NST + a) * 2 + pol) * 2 + 0] = (int8_t)lo4(b);
                    o[((k * NST + a) * 2 + pol) * 2 + 1] = (int8_t)hi4(b);
                }
            }
        }
    }
}

/* Accumulate the 128x128 complex Gram matrix of one frequency.
 * xr/xi: [ntime][128] (row index = 2*station + pol).  accR/accI [128][128].
 * V[a][b] = sum_t x_a * conj(x_b):  re = ra rb + ia ib,  im = ia rb - ra ib. */
static void gram128(const int32_t *xr, const int32_t *xi, int ntime,
                    int32_t *accR, int32_t *accI) {
    memset(accR, 0, sizeof(int32_t) * 128 * 128);
    memset(accI, 0, sizeof(int32_t) * 128 * 128);
    for (int t = 0; t < ntime; t++) {
        const int32_t *r = xr + (int64_t)t * 128;
        const int32_t *m = xi + (int64_t)t * 128;
        for (int a = 0; a < 128; a++) {
            const int32_t ra = r[a], ia = m[a];
            if ((ra | ia) == 0) continue;
            int32_t *R = accR + a * 128, *I = accI + a * 128;
            for (int b = 0; b < 128; b++) {
                R[b] += ra * r[b] + ia * m[b];
                I[b] += ia * r[b] - ra * m[b];
            }
        }
    }
}

/* Scatter one frequency's Gram matrix to the xGPU triangular layout:
 * vis[((tri(i,j))*4 + 2*pi + pj)*2 + {0,1}], tri(i,j) = i(i+1)/2 + j, j<=i.
 * (src/dsaX_wrangleAndWrite.c:50-57, src/dsaX_writevis.c:66-70.) */
static void scatter_tri(const int32_t *accR, const int32_t *accI, float *vis) {
    for (int i = 0; i < NST; i++)
        for (int j = 0; j <= i; j++) {
            int64_t bl = (int64_t)i * (i + 1) / 2 + j;
            for (int pi = 0; pi < 2; pi++)
                for (int pj = 0; pj < 2; pj++) {
                    int a = 2 * i + pi, b = 2 * j + pj;
                    float *v = vis + (bl * 4 + 2 * pi + pj) * 2;
                    v[0] = (float)accR[a * 128 + b];
                    v[1] = (float)accI[a * 128 + b];
                }
        }
}

/* a6: the X-engine on the captured 4-bit block (unpack + reorder + xGPU
 * arithmetic in one).  Computes channels [ch0, ch0+nch) only; vis holds
 * 2*nch frequencies f' = 2*(ch-ch0) + t in xGPU triangular order.
 * Exact: every partial sum is an integer below 2^24, so the int32 result
 * converted to float equals xGPU's FP32 accumulation in any order. */
int oracle_correlate(const uint8_t *blk, int npkt, int nant_in, int nchan,
                     int ch0, int nch, float *vis) {
    if (nant_in < 1 || nant_in > NST || npkt < 1 || nchan < 1 || ch0 < 0 ||
        nch < 1 || ch0 + nch > nchan || npkt > (1 << 23))
        return -1;
    const int64_t ant_stride = (int64_t)nchan * 4;
    const int64_t pkt_stride = (int64_t)nant_in * ant_stride;
    int err = 0;
#pragma omp parallel
    {
        int32_t *xr = (int32_t *)malloc(sizeof(int32_t) * npkt * 128);
        int32_t *xi = (int32_t *)malloc(sizeof(int32_t) * npkt * 128);
        int32_t *accR = (int32_t *)malloc(sizeof(int32_t) * 128 * 128);
        int32_t *accI = (int32_t *)malloc(sizeof(int32_t) * 128 * 128);
        if (!xr || !xi || !accR || !accI) {
#pragma omp atomic write
            err = -2;
        } else {
#pragma omp for schedule(dynamic)
            for (int fq = 0; fq < 2 * nch; fq++) {
                const int ch = ch0 + fq / 2, t = fq % 2;
                memset(xr, 0, sizeof(int32_t) * npkt * 128);
                memset(xi, 0, sizeof(int32_t) * npkt * 128);
                for (int p = 0; p < npkt; p++)
                    for (int a = 0; a < nant_in; a++)
                        for (int pol = 0; pol < 2; pol++) {
                            uint8_t b = blk[p * pkt_stride + a * ant_stride +
                                            ch * 4 + t * 2 + pol];
                            xr[(int64_t)p * 128 + 2 * a + pol] = lo4(b);
                            xi[(int64_t)p * 128 + 2 * a + pol] = hi4(b);
                        }
                gram128(xr, xi, npkt, accR, accI);
                scatter_tri(accR, accI, vis + (int64_t)fq * NBL * 8);
            }
        }
        free(xr); free(xi); free(accR); free(accI);
    }
    return err;
}

/* The same X-engine on xGPU's own 8-bit input vector
 * [ntime][nfreq][64][2 pol][re,im] (what dsaX_xgpu.cu hands to
 * xgpuCudaXengine after its promoter).  Used to pin that
 * massage/fluff + X-engine == oracle_correlate on the captured block. */
int oracle_xengine_int8(const int8_t *xin, int ntime, int nfreq, float *vis) {
    int err = 0;
#pragma omp parallel
    {
        int32_t *xr = (int32_t *)malloc(sizeof(int32_t) * ntime * 128);
        int32_t *xi = (int32_t *)malloc(sizeof(int32_t) * ntime * 128);
        int32_t *accR = (int32_t *)malloc(sizeof(int32_t) * 128 * 128);
        int32_t *accI = (int32_t *)malloc(sizeof(int32_t) * 128 * 128);
        if (!xr || !xi || !accR || !accI) {
#pragma omp atomic write
            err = -2;
        } else {
#pragma omp for schedule(dynamic)
            for (int f = 0; f < nfreq; f++) {
                for (int t = 0; t < ntime; t++) {
                    const int8_t *s = xin + ((int64_t)t * nfreq + f) * 256;
                    for (int a = 0; a < 128; a++) {
                        xr[(int64_t)t * 128 + a] = s[2 * a];
                        xi[(int64_t)t * 128 + a] = s[2 * a + 1];
                    }
                }
                gram128(xr, xi, ntime, accR, accI);
                scatter_tri(accR, accI, vis + (int64_t)f * NBL * 8);
            }
        }
        free(xr); free(xi); free(accR); free(accI);
    }
    return err;
}

/* a7: simple_extract, src/dsaX_writevis.c:55-74: XX and YY (pp = 0, 3),
 * averaged over the two time slots f' = 2f, 2f+1 -> [2080][nchan][2][re,im]. */
void oracle_simple_extract(const float *vis, int nchan, float *out) {
    for (int bl = 0; bl < NBL; bl++)
        for (int pol = 0; pol < 2; pol++)
            for (int f = 0; f < nchan; f++) {
                int64_t o = 2 * (((int64_t)bl * nchan + f) * 2 + pol);
                int64_t i0 = ((2 * (int64_t)f * NBL + bl) * 4 + pol * 3) * 2;
                int64_t i1 = (((2 * (int64_t)f + 1) * NBL + bl) * 4 + pol * 3) * 2;
                out[o] = 0.5f * (vis[i0] + vis[i1]);
                out[o + 1] = 0.5f * (vis[i0 + 1] + vis[i1 + 1]);
            }
}

/* ------------------------------------------------------------------ */
/* Beamformer (src/dsaX_beamformer.cu:121-449), FP64.                  */
/* ------------------------------------------------------------------ */

/* a11/a12: Stokes-I beam power.
 *  blk  : captured block [npkt][nant_in][nchan][2 t][2 pol] 4-bit complex
 *  wre/wim : weights [ngrp = nchan/8][2 pol][nbeam][64 ants] (double)
 *  pkt_per_out : packets summed per output time (16 -> 32 samples)
 *  power: [npkt/pkt_per_out][nbeam][ngrp] (double)
 * P[to][b][g] = sum_{pol} sum_{p in to} sum_{c<8, t<2}
 *               | sum_a w[g][pol][b][a] * x[p][a][8g+c][t][pol] |^2
 * The beam is sum_a w*x with no conjugate (src/dsaX_beamformer.cu:376-378). */
int oracle_beamform(const uint8_t *blk, int npkt, int nant_in, int nchan,
                    const double *wre, const double *wim, int nbeam,
                    int pkt_per_out, int g0, int ng, double *power) {
    if (nchan % 8 || npkt % pkt_per_out || nant_in > NST || g0 < 0 ||
        g0 + ng > nchan / 8)
        return -1;
    const int nout = npkt / pkt_per_out;
    const int64_t ant_stride = (int64_t)nchan * 4;
    const int64_t pkt_stride = (int64_t)nant_in * ant_stride;
#pragma omp parallel for collapse(2) schedule(dynamic)
    for (int gi = 0; gi < ng; gi++)
        for (int to = 0; to < nout; to++) {
            const int g = g0 + gi;
            double xr[NST], xi[NST];
            for (int b = 0; b < nbeam; b++)
                power[((int64_t)to * nbeam + b) * ng + gi] = 0.0;
            for (int pol = 0; pol < 2; pol++) {
                const double *Wr = wre + ((int64_t)g * 2 + pol) * nbeam * NST;
                const double *Wi = wim + ((int64_t)g * 2 + pol) * nbeam * NST;
                for (int p = to * pkt_per_out; p < (to + 1) * pkt_per_out; p++)
                    for (int c = 0; c < 8; c++)
                        for (int t = 0; t < 2; t++) {
                            for (int a = 0; a < NST; a++) {
                                if (a < nant_in) {
                                    uint8_t v = blk[p * pkt_stride + a * ant_stride +
                                                    (8 * g + c) * 4 + t * 2 + pol];
                                    xr[a] = lo4(v);
                                    xi[a] = hi4(v);
                                } else {
                                    xr[a] = xi[a] = 0.0;
                                }
                            }
                            for (int b = 0; b < nbeam; b++) {
                                const double *wr = Wr + (int64_t)b * NST;
                                const double *wi = Wi + (int64_t)b * NST;
                                double br = 0.0, bi = 0.0;
                                for (int a = 0; a < NST; a++) {
                                    br += wr[a] * xr[a] - wi[a] * xi[a];
                                    bi += wi[a] * xr[a] + wr[a] * xi[a];
                                }
                                power[((int64_t)to * nbeam + b) * ng + gi] +=
                                    br * br + bi * bi;
                            }
                        }
            }
        }
    return 0;
}

/* a10: geometric weights, src/dsaX_beamformer.cu:421-449 (calc_weights)
 * with the normalisation of init_weights (:559-602), in FP64.
 *  antpos[64] easting (m); cal[64][ngrp][2 pol][re,im]; flagged ants -> 0.
 *  freq of group g = (fch1_mhz - (8g+4) * 250/8192) MHz;
 *  theta_b = sep_arcmin * (127 - b) * pi / 10800;
 *  w = (cos(afac*pos) + i sin(afac*pos)) * cal / |cal|^2,
 *  afac = -2 pi nu theta / c.
 * Output wre/wim [ngrp][2][nbeam][64]. */
void oracle_geometric_weights(const double *antpos, const double *cal,
                              const int *flagged, int ngrp, int nbeam,
                              double fch1_mhz, double sep_arcmin,
                              double *wre, double *wim) {
    const double PI_ = 3.14159265358979323846, CVAC_ = 299792458.0;
    for (int g = 0; g < ngrp; g++)
        for (int pol = 0; pol < 2; pol++)
            for (int b = 0; b < nbeam; b++)
                for (int a = 0; a < NST; a++) {
                    const double *c = cal + (((int64_t)a * ngrp + g) * 2 + pol) * 2;
                    double cr = c[0], ci = c[1];
                    double n2 = cr * cr + ci * ci;
                    if (n2 != 0.0) { cr /= n2; ci /= n2; }
                    if (flagged && flagged[a]) { cr = 0.0; ci = 0.0; }
                    double nu = (fch1_mhz - (8.0 * g + 4.0) * 250.0 / 8192.0) * 1e6;
                    double theta = sep_arcmin * (127.0 - b) * PI_ / 10800.0;
                    double afac = -2.0 * PI_ * nu * theta / CVAC_;
                    double tr = cos(afac * antpos[a]), ti = sin(afac * antpos[a]);
                    int64_t o = (((int64_t)g * 2 + pol) * nbeam + b) * NST + a;
                    wre[o] = tr * cr - ti * ci;
                    wim[o] = ti * cr + tr * ci;
                }
}
