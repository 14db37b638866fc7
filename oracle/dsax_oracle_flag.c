/*
 * dsax_oracle_flag.c -- CPU restatement of the plain RFI flagger
 * (src/gpu_flagger.cu).  TEST INFRASTRUCTURE ONLY: the checker for the CUDA
 * flagger and the label source for the learned flagger's training tests.
 *
 * Reference shapes are hard-coded to [64 beams][16384 t][1024 ch] uint8
 * (src/gpu_flagger.cu:71-77); this restatement takes any
 * [nbeam][ntime][nchan] float32 filterbank and the constants that the
 * reference hard-codes (guard band ZeroChannels, median window nFiltSize,
 * TBIN, FBIN, time-series baseline length T/16) as parameters.
 *
 * Two modes:
 *  parity   : reproduces src/gpu_flagger.cu as written where it is
 *             deterministic -- the "max" spectrum is the mean spectrum
 *             (:1334 calls calc_spectrum into d_max) and simple_channflag
 *             averages spec[j] FBIN times instead of spec[j+k] (:594).
 *  intended : true per-channel max, and FBIN-channel boxcar in
 *             simple_channflag.
 * calc_ppspec's in-place max/min reductions race (:354-372), so pp is
 * defined in both modes as max - min of the TBIN-sample bin means.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

typedef struct {
    int nbeam, ntime, nchan;
    int guard;        /* ZeroChannels (128 at 1024 ch)            */
    int filt;         /* nFiltSize, forward median window (21)    */
    int tbin;         /* TBIN (128)                               */
    int fbin;         /* FBIN (8)                                 */
    int ts_base;      /* samples used for the ts median (T/16)    */
    int tsflag;       /* 1: time-series flagging on               */
    int parity;       /* 1: parity mode, 0: intended mode         */
    float thresh;     /* -t (5.0)                                 */
    float var_add;    /* var threshold = thresh + var_add (0.5)   */
    float ts_thresh;  /* -s (10.0)                                */
    int nperm;        /* permanent flag channels                  */
    int perm[8];
} oracle_flag_params;

/* lower median as medval() (src/gpu_flagger.cu:534-556):
 * sorted[(n+1)/2 - 1]. */
static int cmpf(const void *a, const void *b) {
    float x = *(const float *)a, y = *(const float *)b;
    return (x > y) - (x < y);
}
static float medval(const float *a, int n, float *tmp) {
    memcpy(tmp, a, sizeof(float) * n);
    qsort(tmp, n, sizeof(float), cmpf);
    return tmp[(n + 1) / 2 - 1];
}

/* Per-(beam, chan) statistics in one pass (calc_spectrum :175-223,
 * calc_varspec :229-278, calc_maxspec :283-319, calc_ppspec :324-376) and
 * the per-(beam, t) channel-mean time series (make_ts :414-453).
 * Accumulated in double; stored float. */
void oracle_flag_stats(const float *x, const oracle_flag_params *P,
                       float *spec, float *var, float *maxs, float *pp,
                       float *ts) {
    const int B = P->nbeam, T = P->ntime, C = P->nchan;
    const int nb = T / P->tbin;
#pragma omp parallel for schedule(static)
    for (int b = 0; b < B; b++) {
        const float *xb = x + (int64_t)b * T * C;
        double *s = (double *)calloc(C, sizeof(double));
        double *bmax = (double *)malloc(sizeof(double) * C);
        double *bmin = (double *)malloc(sizeof(double) * C);
        double *bsum = (double *)calloc(C, sizeof(double));
        float *mx = (float *)malloc(sizeof(float) * C);
        for (int c = 0; c < C; c++) { bmax[c] = -1e300; bmin[c] = 1e300; mx[c] = -INFINITY; }
        for (int t = 0; t < T; t++) {
            double tsum = 0.0;
            for (int c = 0; c < C; c++) {
                float v = xb[(int64_t)t * C + c];
                s[c] += v;
                bsum[c] += v;
                tsum += v;
                if (v > mx[c]) mx[c] = v;
            }
            ts[(int64_t)b * T + t] = (float)(tsum / C);
            if ((t + 1) % P->tbin == 0) {
                for (int c = 0; c < C; c++) {
                    double m = bsum[c] / P->tbin;
                    if (m > bmax[c]) bmax[c] = m;
                    if (m < bmin[c]) bmin[c] = m;
                    bsum[c] = 0.0;
                }
            }
        }
        for (int c = 0; c < C; c++) {
            double mean = s[c] / T;
            double acc = 0.0;
            for (int t = 0; t < T; t++) {
                double d = xb[(int64_t)t * C + c] - mean;
                acc += d * d;
            }
            spec[b * C + c] = (float)mean;
            var[b * C + c] = (float)(acc / T);
            maxs[b * C + c] = P->parity ? (float)mean : mx[c];
            pp[b * C + c] = nb > 0 ? (float)(bmax[c] - bmin[c]) : 0.0f;
        }
        free(s); free(bmax); free(bmin); free(bsum); free(mx);
    }
}

/* channflag (src/gpu_flagger.cu:655-720): forward median detrend over
 * nFiltSize channels, then flag |x| > Thr * MAD inside the guard band
 * (note: compared against 0, not against the median), plus permanent
 * flag channels.  Also returns the detrended spectrum and |x|/MAD margin
 * when requested (for tests that skip near-threshold decisions). */
void oracle_channflag(const float *spec, float thr,
                      const oracle_flag_params *P, int *mask,
                      float *margin) {
    const int B = P->nbeam, C = P->nchan, G = P->guard, F = P->filt;
    const int n = C - 2 * G;
#pragma omp parallel for schedule(static)
    for (int b = 0; b < B; b++) {
        float *corr = (float *)malloc(sizeof(float) * C);
        float *tmp = (float *)malloc(sizeof(float) * (C + F));
        float *nrm = (float *)malloc(sizeof(float) * C);
        const float *sb = spec + (int64_t)b * C;
        for (int j = G; j < C - G; j++) {
            if (C - G - j >= F)
                corr[j] = sb[j] - medval(sb + j, F, tmp);
            else
                corr[j] = sb[j] - medval(sb + C - G - F, F, tmp);
        }
        float med = medval(corr + G, n, tmp);
        for (int j = G; j < C - G; j++) nrm[j - G] = fabsf(corr[j] - med);
        float mad = medval(nrm, n, tmp);
        for (int j = G; j < C - G; j++) {
            if (corr[j] > thr * mad || corr[j] < -thr * mad) mask[b * C + j] = 1;
            if (margin) {
                float m = mad > 0 ? fabsf(fabsf(corr[j]) - thr * mad) / mad : INFINITY;
                if (m < margin[b * C + j]) margin[b * C + j] = m;
            }
            for (int k = 0; k < P->nperm; k++)
                if (j == P->perm[k]) mask[b * C + j] = 1;
        }
        free(corr); free(tmp); free(nrm);
    }
}

/* simple_channflag (src/gpu_flagger.cu:562-610): one-sided,
 * Thr/sqrt(FBIN) (evaluated in double and stored float, as there), over
 * channels [G, C-G-FBIN). */
void oracle_simple_channflag(const float *spec, float thr,
                             const oracle_flag_params *P, int *mask,
                             float *margin) {
    const int B = P->nbeam, C = P->nchan, G = P->guard, FB = P->fbin;
    const int n = C - 2 * G;
    const float mythr = (float)((double)thr / sqrt((double)FB));
#pragma omp parallel for schedule(static)
    for (int b = 0; b < B; b++) {
        float *tmp = (float *)malloc(sizeof(float) * C);
        float *nrm = (float *)malloc(sizeof(float) * C);
        const float *sb = spec + (int64_t)b * C;
        float med = medval(sb + G, n, tmp);
        for (int j = G; j < C - G; j++) nrm[j - G] = fabsf(sb[j] - med);
        float mad = medval(nrm, n, tmp);
        for (int j = G; j < C - G - FB; j++) {
            float vv = 0.0f;
            for (int k = 0; k < FB; k++) vv += P->parity ? sb[j] : sb[j + k];
            vv = vv / (float)FB - med;
            if (vv > mythr * mad) mask[b * C + j] = 1;
            if (margin) {
                float m = mad > 0 ? fabsf(vv - mythr * mad) / mad : INFINITY;
                if (m < margin[b * C + j]) margin[b * C + j] = m;
            }
        }
        free(tmp); free(nrm);
    }
}

/* simple_tsflag (src/gpu_flagger.cu:612-653): median and MAD over the
 * first ts_base samples, one-sided threshold. */
void oracle_simple_tsflag(const float *ts, float thr,
                          const oracle_flag_params *P, int *mask,
                          float *margin) {
    const int B = P->nbeam, T = P->ntime, n = P->ts_base;
#pragma omp parallel for schedule(static)
    for (int b = 0; b < B; b++) {
        float *tmp = (float *)malloc(sizeof(float) * n);
        float *nrm = (float *)malloc(sizeof(float) * n);
        const float *tb = ts + (int64_t)b * T;
        float med = medval(tb, n, tmp);
        for (int j = 0; j < n; j++) nrm[j] = fabsf(tb[j] - med);
        float mad = medval(nrm, n, tmp);
        for (int t = 0; t < T; t++) {
            float vv = tb[t] - med;
            if (vv > thr * mad) mask[(int64_t)b * T + t] = 1;
            if (margin) {
                float m = mad > 0 ? fabsf(vv - thr * mad) / mad : INFINITY;
                if (m < margin[(int64_t)b * T + t]) margin[(int64_t)b * T + t] = m;
            }
        }
        free(tmp); free(nrm);
    }
}

/* The channel-mean time series after flag() (:459-474) has set the flagged
 * columns of each beam to level[beam] (make_ts, :414-453, runs on the
 * replaced data at :1384): accumulated in double, stored float. */
void oracle_ts_replaced(const float *x, const oracle_flag_params *P, const int *chanmask,
                        const float *level, float *ts) {
    const int B = P->nbeam, T = P->ntime, C = P->nchan;
#pragma omp parallel for schedule(static)
    for (int b = 0; b < B; b++) {
        const float *xb = x + (int64_t)b * T * C;
        const int *mb = chanmask + (int64_t)b * C;
        for (int t = 0; t < T; t++) {
            double s = 0.0;
            for (int c = 0; c < C; c++) s += mb[c] ? (double)level[b] : (double)xb[(int64_t)t * C + c];
            ts[(int64_t)b * T + t] = (float)(s / C);
        }
    }
}

/* The channel decisions of :1340-1347 on given statistics:
 * channflag(spec - oldspec, Thr), channflag(var, Thr + 0.5),
 * channflag(max, Thr), simple_channflag(pp, Thr), plus the permanent flag
 * channels.  chanmask is overwritten (0/1). */
void oracle_chan_flags(const float *spec, const float *var, const float *mx, const float *pp,
                       const float *oldspec, const oracle_flag_params *P, int *chanmask,
                       float *chan_margin) {
    const int B = P->nbeam, C = P->nchan;
    float *sub = (float *)malloc(sizeof(float) * B * C);
    for (int i = 0; i < B * C; i++) {
        chanmask[i] = 0;
        sub[i] = spec[i] - (oldspec ? oldspec[i] : 0.0f);
        if (chan_margin) chan_margin[i] = INFINITY;
    }
    oracle_channflag(sub, P->thresh, P, chanmask, chan_margin);
    oracle_channflag(var, P->thresh + P->var_add, P, chanmask, chan_margin);
    oracle_channflag(mx, P->thresh, P, chanmask, chan_margin);
    oracle_simple_channflag(pp, P->thresh, P, chanmask, chan_margin);
    free(sub);
}

/* The per-block decision chain of src/gpu_flagger.cu:1340-1398:
 * channflag(spec - oldspec, Thr), channflag(var, Thr + 0.5),
 * channflag(max, Thr), simple_channflag(pp, Thr), then (if enabled)
 * simple_tsflag(ts, TsThr) on the time series of the data with the flagged
 * columns set to `level` (MN x bpwr, the same for every beam here).
 * oldspec may be NULL (first block: zeros).  chanmask [B][C] and tsmask
 * [B][T] are overwritten (0/1).  Returns the number of flagged (beam, chan)
 * columns. */
int oracle_plain_flag(const float *x, const oracle_flag_params *P,
                      const float *oldspec, int *chanmask, int *tsmask,
                      float *chan_margin, float *ts_margin, float *stats_out, float level) {
    const int B = P->nbeam, T = P->ntime, C = P->nchan;
    float *spec = (float *)malloc(sizeof(float) * B * C);
    float *var = (float *)malloc(sizeof(float) * B * C);
    float *mx = (float *)malloc(sizeof(float) * B * C);
    float *pp = (float *)malloc(sizeof(float) * B * C);
    float *sub = (float *)malloc(sizeof(float) * B * C);
    float *ts = (float *)malloc(sizeof(float) * (int64_t)B * T);
    oracle_flag_stats(x, P, spec, var, mx, pp, ts);
    for (int i = 0; i < B * C; i++) sub[i] = spec[i] - (oldspec ? oldspec[i] : 0.0f);
    oracle_chan_flags(spec, var, mx, pp, oldspec, P, chanmask, chan_margin);
    float *lev = (float *)malloc(sizeof(float) * B);
    for (int b = 0; b < B; b++) lev[b] = level;
    oracle_ts_replaced(x, P, chanmask, lev, ts);
    free(lev);
    for (int64_t i = 0; i < (int64_t)B * T; i++) {
        tsmask[i] = 0;
        if (ts_margin) ts_margin[i] = INFINITY;
    }
    if (P->tsflag) oracle_simple_tsflag(ts, P->ts_thresh, P, tsmask, ts_margin);
    int n = 0;
    for (int i = 0; i < B * C; i++) n += chanmask[i];
    if (stats_out) {
        /* [5][B*C] spec, var, max, pp, sub then [B*T] ts */
        memcpy(stats_out, spec, sizeof(float) * B * C);
        memcpy(stats_out + B * C, var, sizeof(float) * B * C);
        memcpy(stats_out + 2 * B * C, mx, sizeof(float) * B * C);
        memcpy(stats_out + 3 * B * C, pp, sizeof(float) * B * C);
        memcpy(stats_out + 4 * B * C, sub, sizeof(float) * B * C);
        memcpy(stats_out + 5 * B * C, ts, sizeof(float) * (int64_t)B * T);
    }
    free(spec); free(var); free(mx); free(pp); free(sub); free(ts);
    return n;
}
