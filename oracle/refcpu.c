/*
 * refcpu.c -- float32 C restatement of MetalMom's CPU front end.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the CPU baseline that bench.py times
 * (`cpu_baseline`, `--impl reference`) and a second checker for the tests.
 * The shipped CUDA library never links or calls it.
 *
 * MetalMom's own CPU path is Swift + Apple Accelerate and cannot be built on
 * Linux, so this port restates the same per-clip algorithm, step for step, in
 * the same precision (float32 data, float64 mel band edges):
 *
 *   zero padding by n_fft/2 and the frame count      STFT.swift:241-254
 *   periodic Hann built from a float32 ramp + cosf    Windows.swift:14-48
 *   window placement for win != n_fft                 STFT.swift:44-57
 *   per-frame radix-2 real FFT, x0.5 rescale, |X|^2   STFT.swift:287-329
 *   Slaney filterbank, float64 edges cast to float32  FilterBank.swift:23-73
 *   dense mel GEMM  [n_mels x nFreqs][nFreqs x T]     MelSpectrogram.swift:127-138
 *   power_to_db with the clip-global top_db floor     Scaling.swift:73-118
 *   DCT-II ortho basis via cosf, GEMM, truncation     MFCC.swift:65-106
 *
 * The FFT is a textbook iterative radix-2 transform of n_fft/2 complex points
 * followed by the standard split into the real spectrum, i.e. the published
 * algorithm vDSP_fft_zrip implements (its 2x output scale is undone exactly
 * as the reference does).  Batches run one clip per worker thread.
 */
#include <math.h>
#include <pthread.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define RC_OK 0
#define RC_ERR -1

static int is_pow2(int64_t n) { return n > 0 && (n & (n - 1)) == 0; }

int64_t refcpu_n_frames(int64_t length, int n_fft, int hop, int center) {
    int64_t padded = center ? length + 2 * (int64_t)(n_fft / 2) : length;
    if (padded < n_fft || !is_pow2(n_fft) || hop <= 0) return 0;
    return 1 + (padded - n_fft) / hop;
}

/* Windows.hann(periodic:) -- float32 ramp 0, step, 2*step ... then cosf. */
static void hann_f32(int length, float *w) {
    if (length <= 0) return;
    if (length == 1) { w[0] = 1.0f; return; }
    int M = length + 1;
    float step = 2.0f * (float)M_PI / (float)(M - 1);
    for (int i = 0; i < length; i++) {
        float ramp = (float)i * step;
        w[i] = cosf(ramp) * -0.5f + 0.5f;
    }
}

/* prepareWindow (STFT.swift:44-57). */
static void prepare_window_f32(int win, int n_fft, float *out) {
    memset(out, 0, sizeof(float) * (size_t)n_fft);
    if (win <= 0) return;
    float *w = (float *)malloc(sizeof(float) * (size_t)win);
    hann_f32(win, w);
    if (win < n_fft) {
        int before = (n_fft - win) / 2;
        memcpy(out + before, w, sizeof(float) * (size_t)win);
    } else if (win > n_fft) {
        int start = (win - n_fft) / 2;
        memcpy(out, w + start, sizeof(float) * (size_t)n_fft);
    } else {
        memcpy(out, w, sizeof(float) * (size_t)n_fft);
    }
    free(w);
}

/* ---------------- FFT plan: radix-2 complex FFT of h = n_fft/2 points ---- */
typedef struct {
    int n, h, log2h;
    int *rev;        /* bit reversal over h */
    float *twr, *twi; /* exp(-2 pi i t / h), t < h/2 */
    float *pwr, *pwi; /* exp(-2 pi i k / n), k <= h/2, for the real split */
} fft_plan;

static int fft_plan_init(fft_plan *p, int n) {
    memset(p, 0, sizeof(*p));
    p->n = n;
    p->h = n / 2;
    int h = p->h;
    p->log2h = 0;
    while ((1 << p->log2h) < h) p->log2h++;
    p->rev = (int *)malloc(sizeof(int) * (size_t)(h > 0 ? h : 1));
    p->twr = (float *)malloc(sizeof(float) * (size_t)(h / 2 + 1));
    p->twi = (float *)malloc(sizeof(float) * (size_t)(h / 2 + 1));
    p->pwr = (float *)malloc(sizeof(float) * (size_t)(h / 2 + 1));
    p->pwi = (float *)malloc(sizeof(float) * (size_t)(h / 2 + 1));
    if (!p->rev || !p->twr || !p->twi || !p->pwr || !p->pwi) return RC_ERR;
    for (int i = 0; i < h; i++) {
        int r = 0;
        for (int b = 0; b < p->log2h; b++) r |= ((i >> b) & 1) << (p->log2h - 1 - b);
        p->rev[i] = r;
    }
    for (int t = 0; t <= h / 2; t++) {
        double a = -2.0 * M_PI * (double)t / (double)(h > 0 ? h : 1);
        p->twr[t] = (float)cos(a);
        p->twi[t] = (float)sin(a);
        double b = -2.0 * M_PI * (double)t / (double)n;
        p->pwr[t] = (float)cos(b);
        p->pwi[t] = (float)sin(b);
    }
    return RC_OK;
}

static void fft_plan_free(fft_plan *p) {
    free(p->rev); free(p->twr); free(p->twi); free(p->pwr); free(p->pwi);
}

/* In-place forward complex FFT (decimation in time) on h points. */
static void cfft(const fft_plan *p, float *re, float *im) {
    int h = p->h;
    for (int i = 0; i < h; i++) {
        int j = p->rev[i];
        if (j > i) {
            float t = re[i]; re[i] = re[j]; re[j] = t;
            t = im[i]; im[i] = im[j]; im[j] = t;
        }
    }
    for (int len = 2; len <= h; len <<= 1) {
        int half = len >> 1, stride = h / len;
        for (int s = 0; s < h; s += len) {
            for (int j = 0; j < half; j++) {
                float wr = p->twr[j * stride], wi = p->twi[j * stride];
                int a = s + j, b = a + half;
                float xr = re[b] * wr - im[b] * wi;
                float xi = re[b] * wi + im[b] * wr;
                re[b] = re[a] - xr; im[b] = im[a] - xi;
                re[a] += xr; im[a] += xi;
            }
        }
    }
}

/* Power spectrum of one windowed real frame: P[k] = |X[k]|^2, k <= n/2. */
static void real_power(const fft_plan *p, const float *frame, float *re, float *im,
                       float *P, int magnitude) {
    int n = p->n, h = p->h;
    if (n == 1) { P[0] = magnitude ? fabsf(frame[0]) : frame[0] * frame[0]; return; }
    for (int i = 0; i < h; i++) { re[i] = frame[2 * i]; im[i] = frame[2 * i + 1]; }
    cfft(p, re, im);
    /* DC and Nyquist (vDSP packs them in realp[0]/imagp[0]). */
    float dc = re[0] + im[0], ny = re[0] - im[0];
    P[0] = magnitude ? fabsf(dc) : dc * dc;
    P[h] = magnitude ? fabsf(ny) : ny * ny;
    for (int k = 1; k <= h / 2; k++) {
        int q = h - k;
        for (int pass = 0; pass < (k == q ? 1 : 2); pass++) {
            int a = pass ? q : k, b = pass ? k : q;
            /* E = (Z[a] + conj Z[b]) / 2 ; O = (Z[a] - conj Z[b]) / 2i */
            float er = 0.5f * (re[a] + re[b]), ei = 0.5f * (im[a] - im[b]);
            float orr = 0.5f * (im[a] + im[b]), oi = -0.5f * (re[a] - re[b]);
            float wr, wi;
            if (a <= h / 2) { wr = p->pwr[a]; wi = p->pwi[a]; }
            else { wr = -p->pwr[h - a]; wi = p->pwi[h - a]; }
            float xr = er + (orr * wr - oi * wi);
            float xi = ei + (orr * wi + oi * wr);
            float pw = xr * xr + xi * xi;
            P[a] = magnitude ? sqrtf(pw) : pw;
        }
    }
}

/* ---------------- mel filterbank (FilterBank.swift:23-73) ---------------- */
static double hz_to_mel_d(double hz) {
    double f_sp = 200.0 / 3.0, mel = hz / f_sp;
    double min_log_mel = 1000.0 / f_sp, logstep = log(6.4) / 27.0;
    if (hz >= 1000.0) mel = min_log_mel + log(hz / 1000.0) / logstep;
    return mel;
}
static double mel_to_hz_d(double mel) {
    double f_sp = 200.0 / 3.0, min_log_mel = 1000.0 / f_sp, logstep = log(6.4) / 27.0;
    if (mel < min_log_mel) return mel * f_sp;
    return 1000.0 * exp((mel - min_log_mel) * logstep);
}

static void mel_fb_f32(int sr, int n_fft, int n_mels, float fmin, float fmax, float *W) {
    int nf = n_fft / 2 + 1;
    float fmax_a = fmax > 0 ? fmax : (float)sr / 2.0f;
    double lo = hz_to_mel_d((double)fmin), hi = hz_to_mel_d((double)fmax_a);
    float *pts = (float *)malloc(sizeof(float) * (size_t)(n_mels + 2));
    for (int i = 0; i < n_mels + 2; i++)
        pts[i] = (float)mel_to_hz_d(lo + (double)i * (hi - lo) / (double)(n_mels + 1));
    for (int m = 0; m < n_mels; m++) {
        float fl = pts[m], fc = pts[m + 1], fr = pts[m + 2];
        float enorm = 2.0f / (pts[m + 2] - pts[m]);
        for (int k = 0; k < nf; k++) {
            float f = (float)k * (float)sr / (float)n_fft, w = 0.0f;
            if (f >= fl && f <= fc && fc != fl) w = (f - fl) / (fc - fl);
            else if (f > fc && f <= fr && fr != fc) w = (fr - f) / (fr - fc);
            W[(size_t)m * nf + k] = w * enorm;
        }
    }
    free(pts);
}

/* vDSP_vthr: x >= t ? x : t */
static inline float vthr(float x, float t) { return x >= t ? x : t; }

/* ---------------- per-clip pipeline -------------------------------------- */
typedef struct {
    int sr, n_mfcc, n_fft, hop, win, n_mels, center;
    float fmin, fmax, top_db;
} rc_params;

/* MFCC [min(n_mfcc,n_mels) x T] (or mel-dB [n_mels x T] when mel_db_out). */
static int clip_mfcc(const rc_params *q, const float *y, int64_t L, float *out,
                     float *mel_db_out) {
    int n = q->n_fft, nf = n / 2 + 1;
    int64_t T = refcpu_n_frames(L, n, q->hop, q->center);
    if (T == 0) return RC_OK;
    int pad = q->center ? n / 2 : 0;
    float *win = (float *)malloc(sizeof(float) * (size_t)n);
    float *frame = (float *)malloc(sizeof(float) * (size_t)n);
    float *re = (float *)malloc(sizeof(float) * (size_t)(n / 2 + 1));
    float *im = (float *)malloc(sizeof(float) * (size_t)(n / 2 + 1));
    float *P = (float *)malloc(sizeof(float) * (size_t)nf * (size_t)T);
    float *W = (float *)malloc(sizeof(float) * (size_t)nf * (size_t)q->n_mels);
    float *D = (float *)malloc(sizeof(float) * (size_t)q->n_mels * (size_t)T);
    fft_plan plan;
    if (!win || !frame || !re || !im || !P || !W || !D || fft_plan_init(&plan, n) != RC_OK) {
        free(win); free(frame); free(re); free(im); free(P); free(W); free(D);
        return RC_ERR;
    }
    prepare_window_f32(q->win, n, win);
    for (int64_t t = 0; t < T; t++) {
        int64_t s0 = t * q->hop - pad;
        for (int i = 0; i < n; i++) {
            int64_t s = s0 + i;
            float v = (s >= 0 && s < L) ? y[s] : 0.0f;
            frame[i] = v * win[i];
        }
        real_power(&plan, frame, re, im, P + (size_t)t * nf, 0);
    }
    /* dense mel GEMM on the frame-major power (same sums as vDSP_mmul) */
    mel_fb_f32(q->sr, n, q->n_mels, q->fmin, q->fmax, W);
    for (int m = 0; m < q->n_mels; m++) {
        const float *wr = W + (size_t)m * nf;
        for (int64_t t = 0; t < T; t++) {
            const float *pr = P + (size_t)t * nf;
            float acc = 0.0f;
            for (int k = 0; k < nf; k++) acc += wr[k] * pr[k];
            D[(size_t)m * T + t] = acc;
        }
    }
    /* power_to_db(ref=1, amin=1e-10, top_db) */
    size_t cnt = (size_t)q->n_mels * (size_t)T;
    float vmax = -INFINITY;
    for (size_t i = 0; i < cnt; i++) {
        float v = 10.0f * log10f(vthr(D[i], 1e-10f) / 1.0f);
        D[i] = v;
        if (v > vmax) vmax = v;
    }
    if (q->top_db > 0) {
        float floor_db = vmax - q->top_db;
        for (size_t i = 0; i < cnt; i++) D[i] = vthr(D[i], floor_db);
    }
    if (mel_db_out) memcpy(mel_db_out, D, sizeof(float) * cnt);
    if (out) {
        int K = q->n_mfcc < q->n_mels ? q->n_mfcc : q->n_mels, N = q->n_mels;
        float norm0 = sqrtf(1.0f / (float)N), normk = sqrtf(2.0f / (float)N);
        float *B = (float *)malloc(sizeof(float) * (size_t)(K > 0 ? K : 1) * (size_t)N);
        for (int k = 0; k < K; k++)
            for (int j = 0; j < N; j++) {
                float ang = (float)M_PI * (float)k * (2.0f * (float)j + 1.0f) / (2.0f * (float)N);
                B[(size_t)k * N + j] = cosf(ang) * (k == 0 ? norm0 : normk);
            }
        for (int k = 0; k < K; k++)
            for (int64_t t = 0; t < T; t++) {
                float acc = 0.0f;
                for (int j = 0; j < N; j++) acc += B[(size_t)k * N + j] * D[(size_t)j * T + t];
                out[(size_t)k * T + t] = acc;
            }
        free(B);
    }
    fft_plan_free(&plan);
    free(win); free(frame); free(re); free(im); free(P); free(W); free(D);
    return RC_OK;
}

int refcpu_mfcc(const float *y, int64_t L, int sr, int n_mfcc, int n_fft, int hop,
                int win, int n_mels, float fmin, float fmax, int center, float top_db,
                float *out_mfcc, float *out_mel_db) {
    rc_params q = {sr, n_mfcc, n_fft, hop, win, n_mels, center, fmin, fmax, top_db};
    if (!y || L <= 0 || n_fft <= 0 || hop <= 0 || n_mels < 0 || n_mfcc < 0) return RC_ERR;
    return clip_mfcc(&q, y, L, out_mfcc, out_mel_db);
}

/* STFT magnitude or power [n_fft/2+1 x T], row-major (reference layout). */
int refcpu_stft(const float *y, int64_t L, int n_fft, int hop, int win, int center,
                int magnitude, float *out) {
    if (!y || L <= 0 || !is_pow2(n_fft) || hop <= 0) return RC_ERR;
    int n = n_fft, nf = n / 2 + 1, pad = center ? n / 2 : 0;
    int64_t T = refcpu_n_frames(L, n, hop, center);
    float *w = (float *)malloc(sizeof(float) * (size_t)n);
    float *frame = (float *)malloc(sizeof(float) * (size_t)n);
    float *re = (float *)malloc(sizeof(float) * (size_t)(n / 2 + 1));
    float *im = (float *)malloc(sizeof(float) * (size_t)(n / 2 + 1));
    float *P = (float *)malloc(sizeof(float) * (size_t)nf);
    fft_plan plan;
    if (!w || !frame || !re || !im || !P || fft_plan_init(&plan, n) != RC_OK) {
        free(w); free(frame); free(re); free(im); free(P);
        return RC_ERR;
    }
    prepare_window_f32(win, n, w);
    for (int64_t t = 0; t < T; t++) {
        int64_t s0 = t * hop - pad;
        for (int i = 0; i < n; i++) {
            int64_t s = s0 + i;
            frame[i] = ((s >= 0 && s < L) ? y[s] : 0.0f) * w[i];
        }
        real_power(&plan, frame, re, im, P, magnitude);
        for (int k = 0; k < nf; k++) out[(size_t)k * T + t] = P[k];
    }
    fft_plan_free(&plan);
    free(w); free(frame); free(re); free(im); free(P);
    return RC_OK;
}

/* ---------------- threaded batch ----------------------------------------- */
typedef struct {
    const rc_params *q;
    const float *const *ys;
    const int64_t *lens;
    float *const *outs;
    int n;
    int next;
    int err;
    pthread_mutex_t mu;
} batch_job;

static void *batch_worker(void *arg) {
    batch_job *j = (batch_job *)arg;
    for (;;) {
        pthread_mutex_lock(&j->mu);
        int i = j->next++;
        pthread_mutex_unlock(&j->mu);
        if (i >= j->n) break;
        if (clip_mfcc(j->q, j->ys[i], j->lens[i], j->outs[i], NULL) != RC_OK) j->err = 1;
    }
    return NULL;
}

int refcpu_mfcc_batch(const float *const *ys, const int64_t *lens, int n_clips, int sr,
                      int n_mfcc, int n_fft, int hop, int win, int n_mels, float fmin,
                      float fmax, int center, float top_db, float *const *outs,
                      int n_threads) {
    rc_params q = {sr, n_mfcc, n_fft, hop, win, n_mels, center, fmin, fmax, top_db};
    if (n_threads < 1) n_threads = 1;
    batch_job job = {&q, ys, lens, outs, n_clips, 0, 0, PTHREAD_MUTEX_INITIALIZER};
    pthread_t *th = (pthread_t *)malloc(sizeof(pthread_t) * (size_t)n_threads);
    int started = 0;
    for (int i = 0; i < n_threads; i++)
        if (pthread_create(&th[started], NULL, batch_worker, &job) == 0) started++;
    if (started == 0) batch_worker(&job);
    for (int i = 0; i < started; i++) pthread_join(th[i], NULL);
    free(th);
    return job.err ? RC_ERR : RC_OK;
}
