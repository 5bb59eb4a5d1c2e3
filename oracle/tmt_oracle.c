/*
 * tmt_oracle.c -- CPU oracle for the tomotopy LDA collapsed-Gibbs path.
 * TEST INFRASTRUCTURE ONLY: see tmt_oracle.h for scope, citations and the
 * parity status.  Build with -ffp-contract=off so that float expressions
 * round exactly as written (the device code spells out the same operations
 * with round-to-nearest intrinsics).
 */
#include "tmt_oracle.h"
#include <math.h>
#include <stdlib.h>
#include <string.h>
#include <pthread.h>

/* ------------------------------------------------------------------------ */
/* Philox4x32-10                                                            */
/* ------------------------------------------------------------------------ */
static inline void mulhilo32(uint32_t a, uint32_t b, uint32_t* hi, uint32_t* lo)
{
    uint64_t p = (uint64_t)a * (uint64_t)b;
    *hi = (uint32_t)(p >> 32);
    *lo = (uint32_t)p;
}

void orc_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4])
{
    uint32_t c0 = ctr[0], c1 = ctr[1], c2 = ctr[2], c3 = ctr[3];
    uint32_t k0 = key[0], k1 = key[1];
    for (int r = 0; r < 10; ++r) {
        uint32_t hi0, lo0, hi1, lo1;
        mulhilo32(0xD2511F53u, c0, &hi0, &lo0);
        mulhilo32(0xCD9E8D57u, c2, &hi1, &lo1);
        uint32_t n0 = hi1 ^ c1 ^ k0;
        uint32_t n1 = lo1;
        uint32_t n2 = hi0 ^ c3 ^ k1;
        uint32_t n3 = lo0;
        c0 = n0; c1 = n1; c2 = n2; c3 = n3;
        k0 += 0x9E3779B9u;
        k1 += 0xBB67AE85u;
    }
    out[0] = c0; out[1] = c1; out[2] = c2; out[3] = c3;
}

float orc_u01(uint32_t x)
{
    return (float)(x >> 8) * (1.0f / 16777216.0f);
}

static inline uint32_t philox_first(uint32_t c0, uint32_t c1, uint32_t c2, uint32_t c3, uint64_t seed)
{
    uint32_t ctr[4] = { c0, c1, c2, c3 };
    uint32_t key[2] = { (uint32_t)seed, (uint32_t)(seed >> 32) };
    uint32_t out[4];
    orc_philox4x32_10(ctr, key, out);
    return out[0];
}

/* ------------------------------------------------------------------------ */
/* Float LUTs (restating src/Utils/LUT.hpp:11-70 and math.h:119-153)        */
/* ------------------------------------------------------------------------ */
/* LUT3<F, float, N, S, M, T, L, U>: three linear-interpolation segments,
 * [0, N/S) step 1/S, [N/S, N/S + M/T) step 1/T, then step 1/U for L points;
 * below smallThreshold and above the last point a closed form is used. */
typedef struct {
    float* points;
    size_t N, M, L;
    float P, Q, R;
} lut3;

static const float ORC_PI = 3.14159265f;

/* tomotopy's F_lgamma calls the unqualified lgamma / log, which resolve to
 * the double overloads: the table holds (float)lgamma((double)x) and the
 * closed forms are evaluated in double, then rounded to float. */
static float F_lgamma_small(float x)
{
    if (x == 0) return INFINITY;
    return (float)((x + 0.5f) * log((double)(x + 1)) - (double)(x + 1) + log((double)(2 * ORC_PI)) / 2
                   + (double)(1 / 12.f / (x + 1)) - log((double)x));
}
static float F_lgamma_large(float x)
{
    return (float)((x - 0.5f) * log((double)x) - (double)x + log((double)(2 * ORC_PI)) / 2
                   + (double)(1 / 12.f / x));
}
static float F_lgamma_nonfinite(float x)
{
    if (isnan(x)) return NAN;
    if (x > 0) return INFINITY;
    return -INFINITY;
}

static float F_digamma_small(float x)
{
    if (x == 0) return -INFINITY;
    return logf(x + 2) - 0.5f / (x + 2) - 1 / 12.f / powf(x + 2, 2) - 1 / (x + 1) - 1 / x;
}
static float F_digamma_large(float x)
{
    return logf(x) - 0.5f / x - 1 / 12.f / powf(x, 2);
}
static float F_digamma_nonfinite(float x)
{
    if (isnan(x) || x < 0) return NAN;
    return INFINITY;
}

/* digammaf: the float recursion + Chebyshev series of math.h:72-115 */
float orc_digammaf(float x)
{
    static const float gam = 0.577215664f, ln2 = 0.693147180f;
    if (x < 0.0f)
        return orc_digammaf(1.0f - x) + ORC_PI / tanf(ORC_PI * (1.0f - x));
    else if (x < 1.0f)
        return orc_digammaf(1.0f + x) - 1.0f / x;
    else if (x == 1.0f)
        return -gam;
    else if (x == 2.0f)
        return (float)(1.0L - gam);
    else if (x == 3.0f)
        return (float)(1.5L - gam);
    else if (x > 3.0f)
        return 0.5f * (orc_digammaf(x / 2.0f) + orc_digammaf((x + 1.0f) / 2.0f)) + ln2;
    else {
        static const float kn[] = { .304591985f,
            .720379774f, -.124549592f,
            .277694573e-1f, -.677623714e-2f,
            .172387551e-2f, -.448176990e-3f,
            .117936600e-3f, -.312538942e-4f,
            .831739970e-5f, -.221914276e-5f,
            .593022667e-6f, -.158630511e-6f,
            .424592039e-7f, -.113691296e-7f,
            .304502217e-8f, -.815684550e-9f, };
        float Tn_1 = 1.0f;
        float Tn = (float)(x - 2.0);
        float resul = kn[0] + kn[1] * Tn;
        x = (float)(x - 2.0L);
        for (size_t n = 2; n < sizeof(kn) / sizeof(float); n++) {
            const float Tn1 = (float)(2.0L * x * Tn - Tn_1);
            resul += kn[n] * Tn1;
            Tn_1 = Tn;
            Tn = Tn1;
        }
        return resul;
    }
}

static lut3 g_lgamma, g_digamma;
static pthread_once_t g_lut_once = PTHREAD_ONCE_INIT;

static void lut3_build(lut3* t, int which, size_t N, size_t S, size_t M, size_t T, size_t L, size_t U)
{
    t->N = N; t->M = M; t->L = L;
    t->P = (float)(1. / S); t->Q = (float)(1. / T); t->R = (float)(1. / U);
    t->points = (float*)calloc(N + M + L, sizeof(float));
    for (size_t i = 0; i < N; i++) {
        float x = i ? i * t->P : (float)0.0001;
        t->points[i] = which ? orc_digammaf(x) : (float)lgamma((double)x);
    }
    for (size_t i = 0; i < M; i++) {
        float x = i * t->Q + N * t->P;
        t->points[i + N] = which ? orc_digammaf(x) : (float)lgamma((double)x);
    }
    for (size_t i = 0; i < L; i++) {
        float x = i * t->R + N * t->P + M * t->Q;
        t->points[i + N + M] = which ? orc_digammaf(x) : (float)lgamma((double)x);
    }
}

static void luts_init(void)
{
    lut3_build(&g_lgamma, 0, 1 * 1024, 1024, 100 * 64, 64, 1000 * 8, 8);
    lut3_build(&g_digamma, 1, 1 * 1024, 1024, 100 * 64, 64, 1000 * 4, 4);
}

static float lut3_get(const lut3* t, float x, int which)
{
    if (!isfinite(x)) return which ? F_digamma_nonfinite(x) : F_lgamma_nonfinite(x);
    if (x < 0) return NAN;
    if (x < (float)0.001) return which ? F_digamma_small(x) : F_lgamma_small(x);
    const size_t N = t->N, M = t->M, L = t->L;
    const float P = t->P, Q = t->Q, R = t->R;
    if (x >= N * P + M * Q + (L - 1) * R) return which ? F_digamma_large(x) : F_lgamma_large(x);
    size_t idx;
    float a;
    float nx = x;
    if (x < N * P) {
        idx = (size_t)(nx / P);
        a = (nx - idx * P) / P;
    } else {
        nx -= N * P;
        if (nx < M * Q) {
            idx = (size_t)(nx / Q);
            a = (nx - idx * Q) / Q;
            idx += N;
        } else {
            nx -= M * Q;
            idx = (size_t)(nx / R);
            a = (nx - idx * R) / R;
            idx += N + M;
        }
    }
    return t->points[idx] + a * (t->points[idx + 1] - t->points[idx]);
}

float orc_lgammaT(float x)
{
    pthread_once(&g_lut_once, luts_init);
    return lut3_get(&g_lgamma, x, 0);
}

float orc_digammaT(float x)
{
    pthread_once(&g_lut_once, luts_init);
    return lut3_get(&g_digamma, x, 1);
}

/* digammaApprox (math.h:170-176) evaluated in float, as it is over Eigen float arrays */
float orc_digammaApprox(float z)
{
    return logf(z + 4) - 1.f / 2.f / (z + 4) - 1.f / 12.f / ((z + 4) * (z + 4))
        - 1.f / z - 1.f / (z + 1) - 1.f / (z + 2) - 1.f / (z + 3);
}

/* ------------------------------------------------------------------------ */
/* Sampling primitives                                                      */
/* ------------------------------------------------------------------------ */
/* prefixSum, SSE2 path (sample.hpp:62-86): groups of four are scanned as
 * x + (x<<1 lane), then + (x<<2 lanes), then offset by the previous group's
 * last value; the tail (n % 4) is a sequential running sum. */
void orc_prefix_sum_sse(float* arr, int n)
{
    int n4 = n & ~3;
    float offset = 0.f;
    for (int i = 0; i < n4; i += 4) {
        float x0 = arr[i], x1 = arr[i + 1], x2 = arr[i + 2], x3 = arr[i + 3];
        float y0 = x0, y1 = x1 + x0, y2 = x2 + x1, y3 = x3 + x2;
        float s0 = y0, s1 = y1, s2 = y2 + y0, s3 = y3 + y1;
        arr[i] = s0 + offset;
        arr[i + 1] = s1 + offset;
        arr[i + 2] = s2 + offset;
        arr[i + 3] = s3 + offset;
        offset = arr[i + 3];
    }
    if (!n4) n4 = 1;
    for (int i = n4; i < n; ++i) arr[i] += arr[i - 1];
}

/* sampleFromDiscreteAcc (sample.hpp:133-189): r = u * cum[K-1]; first z with
 * r < cum[z]; K-1 if none. */
size_t orc_sample_acc(const float* cum, size_t K, float u01)
{
    float r = u01 * cum[K - 1];
    for (size_t z = 0; z < K; ++z)
        if (r < cum[z]) return z;
    return K - 1;
}

/* forShuffled (Utils.hpp:157-178) */
void orc_shuffled_order(size_t N, size_t seed, uint64_t* out)
{
    static const size_t primes[16] = {
        65537, 65539, 65543, 65551, 65557, 65563,
        65579, 65581, 65587, 65599, 65609, 65617,
        65629, 65633, 65647, 65651
    };
    if (!N) return;
    size_t P = primes[seed & 0xF];
    if (N % P == 0) {
        P = primes[(seed + 1) & 0xF];
        if (N % P == 0) P = primes[(seed + 2) & 0xF];
        if (N % P == 0) P = primes[(seed + 3) & 0xF];
    }
    P %= N;
    for (size_t i = 0; i < N; ++i) out[i] = ((i + seed) * P) % N;
}

/* ------------------------------------------------------------------------ */
/* Corpus preparation                                                       */
/* ------------------------------------------------------------------------ */
typedef struct { uint64_t cf, df; uint32_t idx; } cfdf;
static uint64_t g_min_cf, g_min_df;

static int cfdf_bad(const cfdf* a) { return a->cf < g_min_cf || a->df < g_min_df; }
/* the comparator of removeStopwords (TopicModel.hpp:538-551): valid words
 * first, each group by (cf, df) descending */
static int cfdf_less(const cfdf* a, const cfdf* b)
{
    int ab = cfdf_bad(a), bb = cfdf_bad(b);
    if (ab) {
        if (bb) return (a->cf > b->cf) || (a->cf == b->cf && a->df > b->df);
        return 0;
    }
    if (bb) return 1;
    return (a->cf > b->cf) || (a->cf == b->cf && a->df > b->df);
}

/* stable merge sort of cfdf (std::stable_sort semantics) */
static void cfdf_msort(cfdf* a, cfdf* tmp, size_t n)
{
    if (n < 2) return;
    size_t h = n / 2;
    cfdf_msort(a, tmp, h);
    cfdf_msort(a + h, tmp, n - h);
    size_t i = 0, j = h, k = 0;
    while (i < h && j < n) {
        if (cfdf_less(&a[j], &a[i])) tmp[k++] = a[j++];
        else tmp[k++] = a[i++];
    }
    while (i < h) tmp[k++] = a[i++];
    while (j < n) tmp[k++] = a[j++];
    memcpy(a, tmp, n * sizeof(cfdf));
}

uint64_t orc_remove_stopwords(uint64_t nv, uint64_t* cf, uint64_t* df,
                              uint64_t min_cf, uint64_t min_df, uint64_t rm_top,
                              uint32_t* order)
{
    cfdf* v = (cfdf*)malloc((nv + 1) * sizeof(cfdf));
    cfdf* tmp = (cfdf*)malloc((nv + 1) * sizeof(cfdf));
    g_min_cf = min_cf; g_min_df = min_df;
    for (uint64_t i = 0; i < nv; ++i) { v[i].cf = cf[i]; v[i].df = df[i]; v[i].idx = (uint32_t)i; }
    cfdf_msort(v, tmp, nv);
    /* std::rotate(begin, begin + rm_top, end) */
    if (rm_top && nv) {
        uint64_t r = rm_top < nv ? rm_top : nv;
        memcpy(tmp, v, r * sizeof(cfdf));
        memmove(v, v + r, (nv - r) * sizeof(cfdf));
        memcpy(v + (nv - r), tmp, r * sizeof(cfdf));
    }
    uint64_t lim = nv - (rm_top < nv ? rm_top : nv);
    uint64_t realV = lim;
    for (uint64_t i = 0; i < lim; ++i) {
        if (cfdf_bad(&v[i])) { realV = i; break; }
    }
    for (uint64_t i = 0; i < nv; ++i) {
        order[v[i].idx] = (uint32_t)i;
        cf[i] = v[i].cf;
        df[i] = v[i].df;
    }
    free(v); free(tmp);
    return realV;
}

typedef struct { uint32_t w; uint32_t i; } wpair;
static void wpair_msort(wpair* a, wpair* tmp, size_t n)
{
    if (n < 2) return;
    size_t h = n / 2;
    wpair_msort(a, tmp, h);
    wpair_msort(a + h, tmp, n - h);
    size_t i = 0, j = h, k = 0;
    while (i < h && j < n) {
        if (a[j].w < a[i].w) tmp[k++] = a[j++];
        else tmp[k++] = a[i++];
    }
    while (i < h) tmp[k++] = a[i++];
    while (j < n) tmp[k++] = a[j++];
    memcpy(a, tmp, n * sizeof(wpair));
}

void orc_sort_doc(uint32_t* words, size_t n, uint32_t* w_order)
{
    wpair* pv = (wpair*)malloc((n + 1) * sizeof(wpair));
    wpair* tmp = (wpair*)malloc((n + 1) * sizeof(wpair));
    for (size_t i = 0; i < n; ++i) { pv[i].w = words[i]; pv[i].i = (uint32_t)i; }
    wpair_msort(pv, tmp, n);
    for (size_t i = 0; i < n; ++i) {
        words[i] = pv[i].w;
        w_order[pv[i].i] = (uint32_t)i;
    }
    free(pv); free(tmp);
}

void orc_init_z(uint64_t N, const uint32_t* words, uint32_t V, uint32_t K,
                const float* alpha, uint64_t seed, uint16_t* z)
{
    float* cum = (float*)malloc(K * sizeof(float));
    float s = 0.f;
    for (uint32_t k = 0; k < K; ++k) { s = s + alpha[k]; cum[k] = s; }
    for (uint64_t i = 0; i < N; ++i) {
        if (words[i] >= V) { z[i] = 0xFFFF; continue; }
        float u = orc_u01(philox_first((uint32_t)i, (uint32_t)(i >> 32), ORC_STREAM_INIT, 0, seed));
        z[i] = (uint16_t)orc_sample_acc(cum, K, u);
    }
    free(cum);
}

void orc_counts_from_z(uint64_t D, const uint64_t* doc_off, const uint32_t* words,
                       const uint16_t* z, uint32_t V, uint32_t K,
                       int32_t* ndk, int32_t* nkw, int32_t* nk)
{
    memset(ndk, 0, D * K * sizeof(int32_t));
    memset(nkw, 0, (size_t)V * K * sizeof(int32_t));
    memset(nk, 0, K * sizeof(int32_t));
    for (uint64_t d = 0; d < D; ++d) {
        for (uint64_t i = doc_off[d]; i < doc_off[d + 1]; ++i) {
            uint32_t w = words[i];
            if (w >= V) continue;
            uint16_t k = z[i];
            ndk[d * K + k]++;
            nkw[(size_t)w * K + k]++;
            nk[k]++;
        }
    }
}

uint64_t orc_word_major(uint64_t D, const uint64_t* doc_off, const uint32_t* words,
                        uint32_t V, uint64_t* w_off, uint32_t* tok_doc, uint64_t* tok_pos)
{
    memset(w_off, 0, (V + 1) * sizeof(uint64_t));
    uint64_t N = doc_off[D];
    for (uint64_t i = 0; i < N; ++i)
        if (words[i] < V) w_off[words[i] + 1]++;
    for (uint32_t v = 0; v < V; ++v) w_off[v + 1] += w_off[v];
    uint64_t* cur = (uint64_t*)malloc((V + 1) * sizeof(uint64_t));
    memcpy(cur, w_off, (V + 1) * sizeof(uint64_t));
    for (uint64_t d = 0; d < D; ++d) {
        for (uint64_t i = doc_off[d]; i < doc_off[d + 1]; ++i) {
            uint32_t w = words[i];
            if (w >= V) continue;
            uint64_t t = cur[w]++;
            tok_doc[t] = (uint32_t)d;
            if (tok_pos) tok_pos[t] = i;
        }
    }
    free(cur);
    return w_off[V];
}

/* ------------------------------------------------------------------------ */
/* The device sampler's semantics                                           */
/* ------------------------------------------------------------------------ */
/* Segmented warp scan + strict search, the order the dense device kernel
 * uses: c = ceil(K/32) topics per lane; lane l sums its segment
 * sequentially; lane totals get a Hillis-Steele inclusive scan over 32
 * lanes (offsets 1,2,4,8,16); lane l's exclusive offset is lane l-1's
 * inclusive value; cum[j] = excl[lane(j)] + loc[j]; r = u * incl[31];
 * result = first j with r < cum[j], else K-1. */
static uint32_t seg_scan_draw(const float* w, uint32_t K, float u, float* loc)
{
    uint32_t c = (K + 31) / 32;
    float T[32], x[32], y[32], excl[32];
    for (uint32_t l = 0; l < 32; ++l) {
        float s = 0.f;
        uint32_t b = l * c, e = b + c < K ? b + c : K;
        for (uint32_t j = b; j < e; ++j) { s = s + w[j]; loc[j] = s; }
        T[l] = s;
        x[l] = s;
    }
    for (uint32_t off = 1; off < 32; off <<= 1) {
        for (uint32_t l = 0; l < 32; ++l) y[l] = (l >= off) ? x[l] + x[l - off] : x[l];
        memcpy(x, y, sizeof(x));
    }
    for (uint32_t l = 0; l < 32; ++l) excl[l] = l ? x[l - 1] : 0.f;
    float total = x[31];
    float r = u * total;
    (void)T;
    for (uint32_t j = 0; j < K; ++j) {
        float cj = excl[j / c] + loc[j];
        if (r < cj) return j;
    }
    return K - 1;
}

void orc_sweep_snapshot(uint32_t K, uint32_t V, const float* alpha, float eta,
                        uint64_t seed, uint32_t iter,
                        const uint64_t* w_off, const uint32_t* tok_doc,
                        const int32_t* ndk, const int32_t* nkw, const int32_t* nk,
                        const uint16_t* z_old, uint16_t* z_new)
{
    float veta = eta * (float)V;
    float* R = (float*)malloc(K * sizeof(float));
    float* w = (float*)malloc(K * sizeof(float));
    float* loc = (float*)malloc(K * sizeof(float));
    for (uint32_t k = 0; k < K; ++k) R[k] = 1.0f / ((float)nk[k] + veta);
    for (uint32_t v = 0; v < V; ++v) {
        const int32_t* col = nkw + (size_t)v * K;
        for (uint64_t t = w_off[v]; t < w_off[v + 1]; ++t) {
            uint32_t d = tok_doc[t];
            uint16_t zo = z_old[t];
            const int32_t* row = ndk + (size_t)d * K;
            for (uint32_t k = 0; k < K; ++k) {
                int own = (k == zo);
                float a = (float)(row[k] - own) + alpha[k];
                float b = (float)(col[k] - own) + eta;
                float r = own ? 1.0f / ((float)(nk[k] - 1) + veta) : R[k];
                w[k] = (a * b) * r;
            }
            float u = orc_u01(philox_first((uint32_t)t, (uint32_t)(t >> 32), ORC_STREAM_SWEEP, iter, seed));
            z_new[t] = (uint16_t)seg_scan_draw(w, K, u, loc);
        }
    }
    free(R); free(w); free(loc);
}

void orc_conditional_f64(uint32_t K, uint32_t V, const float* alpha, float eta,
                         const int32_t* ndk_row, const int32_t* nkw_col, const int32_t* nk,
                         uint16_t z_own, double* p)
{
    double veta = (double)eta * (double)V, s = 0;
    for (uint32_t k = 0; k < K; ++k) {
        int own = (k == z_own);
        p[k] = ((double)(ndk_row[k] - own) + alpha[k]) * ((double)(nkw_col[k] - own) + eta)
             / ((double)(nk[k] - own) + veta);
        s += p[k];
    }
    for (uint32_t k = 0; k < K; ++k) p[k] /= s;
}

void orc_apply_sweep(uint32_t K, uint32_t V, const uint64_t* w_off, const uint32_t* tok_doc,
                     int32_t* ndk, int32_t* nkw, int32_t* nk,
                     uint16_t* z_old, const uint16_t* z_new)
{
    for (uint32_t v = 0; v < V; ++v) {
        for (uint64_t t = w_off[v]; t < w_off[v + 1]; ++t) {
            uint16_t zo = z_old[t], zn = z_new[t];
            if (zo == zn) continue;
            uint32_t d = tok_doc[t];
            ndk[(size_t)d * K + zo]--; ndk[(size_t)d * K + zn]++;
            nkw[(size_t)v * K + zo]--; nkw[(size_t)v * K + zn]++;
            nk[zo]--; nk[zn]++;
            z_old[t] = zn;
        }
    }
}

/* ------------------------------------------------------------------------ */
/* The reference's sequential sampler                                       */
/* ------------------------------------------------------------------------ */
static inline uint64_t splitmix64(uint64_t* s)
{
    uint64_t z = (*s += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}
static inline float sm_u01(uint64_t* s) { return (float)(splitmix64(s) >> 40) * (1.0f / 16777216.0f); }

/* sampleDocument for tokens [b, e) of one doc (LDAModel.hpp:326-354) with
 * getZLikelihoods (:273-285) and addWordTo (:287-299). */
static void sample_doc_range(uint32_t K, uint32_t V, const float* alpha, float eta, float veta,
                             const uint32_t* words, uint16_t* z, uint64_t b, uint64_t e,
                             int32_t* ndk_row, int32_t* nkw, int32_t* nk, float* dist, uint64_t* rng)
{
    for (uint64_t i = b; i < e; ++i) {
        uint32_t v = words[i];
        if (v >= V) continue;
        uint16_t k0 = z[i];
        int32_t* col = nkw + (size_t)v * K;
        ndk_row[k0]--; nk[k0]--; col[k0]--;
        for (uint32_t k = 0; k < K; ++k)
            dist[k] = ((float)ndk_row[k] + alpha[k]) * ((float)col[k] + eta) / ((float)nk[k] + veta);
        orc_prefix_sum_sse(dist, (int)K);
        uint16_t k1 = (uint16_t)orc_sample_acc(dist, K, sm_u01(rng));
        z[i] = k1;
        ndk_row[k1]++; nk[k1]++; col[k1]++;
    }
}

void orc_gibbs_none(uint64_t D, const uint64_t* doc_off, const uint32_t* words,
                    uint32_t V, uint32_t K, const float* alpha, float eta,
                    uint16_t* z, int32_t* ndk, int32_t* nkw, int32_t* nk,
                    uint64_t* rng_state)
{
    float veta = eta * (float)V;
    float* dist = (float*)malloc(K * sizeof(float));
    uint64_t* order = (uint64_t*)malloc((D + 1) * sizeof(uint64_t));
    orc_shuffled_order(D, (size_t)(splitmix64(rng_state) & 0xFFFFFFFFu), order);
    for (uint64_t j = 0; j < D; ++j) {
        uint64_t d = order[j];
        sample_doc_range(K, V, alpha, eta, veta, words, z, doc_off[d], doc_off[d + 1],
                         ndk + d * K, nkw, nk, dist, rng_state);
    }
    free(dist); free(order);
}

/* ------------------------------------------------------------------------ */
/* PARTITION scheme on host threads (CPU baseline)                          */
/* ------------------------------------------------------------------------ */
struct orc_partition {
    uint64_t D; const uint64_t* doc_off; const uint32_t* words;
    uint32_t V, K, W; const float* alpha; float eta, veta;
    uint16_t* z; int32_t* ndk; int32_t* nkw; int32_t* nk;
    uint32_t* vchunk;      /* W chunk ends */
    uint64_t* chunk_off;   /* (W+1) x D */
    int32_t** local_nk;    /* W private n_k */
    float** dist;
    uint64_t* rng;         /* W splitmix states */
    pthread_t* th;
    void* args;
    pthread_barrier_t bar;
    uint32_t iters, stop;
};

typedef struct { orc_partition* p; uint32_t id; } part_arg;

static void* partition_worker(void* a_)
{
    part_arg* a = (part_arg*)a_;
    orc_partition* p = a->p;
    uint32_t pid = a->id, W = p->W;
    uint64_t* order = (uint64_t*)malloc((p->D / W + 2) * sizeof(uint64_t));
    for (;;) {
        pthread_barrier_wait(&p->bar);          /* start of a train() call */
        if (p->stop) break;
        for (uint32_t it = 0; it < p->iters; ++it) {
            for (uint32_t i = 0; i < W; ++i) {
                uint32_t didx = (i + pid) % W;
                uint64_t n = (p->D + (W - 1) - didx) / W;
                orc_shuffled_order(n, (size_t)(splitmix64(&p->rng[pid]) & 0xFFFFFFFFu), order);
                for (uint64_t j = 0; j < n; ++j) {
                    uint64_t d = order[j] * W + didx;
                    uint64_t b = p->doc_off[d] + p->chunk_off[(uint64_t)pid * p->D + d];
                    uint64_t e = p->doc_off[d] + p->chunk_off[(uint64_t)(pid + 1) * p->D + d];
                    sample_doc_range(p->K, p->V, p->alpha, p->eta, p->veta, p->words, p->z, b, e,
                                     p->ndk + d * p->K, p->nkw, p->local_nk[pid], p->dist[pid], &p->rng[pid]);
                }
                pthread_barrier_wait(&p->bar);  /* the round's join */
            }
            /* mergeState (rowsum) by worker 0, distributeMergedState by all */
            if (pid == 0) {
                memset(p->nk, 0, p->K * sizeof(int32_t));
                for (uint32_t v = 0; v < p->V; ++v) {
                    const int32_t* col = p->nkw + (size_t)v * p->K;
                    for (uint32_t k = 0; k < p->K; ++k) p->nk[k] += col[k];
                }
            }
            pthread_barrier_wait(&p->bar);
            memcpy(p->local_nk[pid], p->nk, p->K * sizeof(int32_t));
            pthread_barrier_wait(&p->bar);
        }
        pthread_barrier_wait(&p->bar);          /* end of the train() call */
    }
    free(order);
    return NULL;
}

orc_partition* orc_partition_create(uint64_t D, const uint64_t* doc_off, const uint32_t* words,
                                    uint32_t V, uint32_t K, const float* alpha, float eta,
                                    uint16_t* z, int32_t* ndk, int32_t* nkw, int32_t* nk,
                                    const uint64_t* vocab_cf, uint32_t nthreads, uint64_t seed)
{
    orc_partition* p = (orc_partition*)calloc(1, sizeof(orc_partition));
    uint32_t W = nthreads ? nthreads : 1;
    uint32_t maxw = (V + 3) / 4;          /* estimateMaxThreads (LDAModel.hpp:494-497) */
    if (maxw < 1) maxw = 1;
    if (W > maxw) W = maxw;
    p->D = D; p->doc_off = doc_off; p->words = words; p->V = V; p->K = K; p->W = W;
    p->alpha = alpha; p->eta = eta; p->veta = eta * (float)V;
    p->z = z; p->ndk = ndk; p->nkw = nkw; p->nk = nk;
    /* updatePartition (LDAModel.hpp:437-472): chunk ends by cumulative cf */
    p->vchunk = (uint32_t*)malloc(W * sizeof(uint32_t));
    uint64_t tot = 0, cum = 0;
    uint32_t nch = 0;
    for (uint32_t v = 0; v < V; ++v) tot += vocab_cf[v];
    for (uint32_t v = 0; v < V && nch < W; ++v) {
        cum += vocab_cf[v];
        if (cum * W >= tot * (nch + 1)) p->vchunk[nch++] = v + 1;
    }
    while (nch < W) p->vchunk[nch++] = V;
    p->chunk_off = (uint64_t*)malloc((uint64_t)(W + 1) * D * sizeof(uint64_t));
    for (uint64_t d = 0; d < D; ++d) {
        uint64_t len = doc_off[d + 1] - doc_off[d];
        const uint32_t* ws = words + doc_off[d];
        p->chunk_off[d] = 0;
        uint32_t g = 0;
        for (uint64_t j = 0; j < len; ++j)
            for (; g < W && ws[j] >= p->vchunk[g]; ++g) p->chunk_off[(uint64_t)(g + 1) * D + d] = j;
        for (; g < W; ++g) p->chunk_off[(uint64_t)(g + 1) * D + d] = len;
    }
    p->local_nk = (int32_t**)malloc(W * sizeof(int32_t*));
    p->dist = (float**)malloc(W * sizeof(float*));
    p->rng = (uint64_t*)malloc(W * sizeof(uint64_t));
    for (uint32_t i = 0; i < W; ++i) {
        p->local_nk[i] = (int32_t*)malloc(K * sizeof(int32_t));
        memcpy(p->local_nk[i], nk, K * sizeof(int32_t));
        p->dist[i] = (float*)aligned_alloc(64, ((K + 15) / 16) * 64);
        p->rng[i] = seed * 0x9E3779B97F4A7C15ull + i + 1;
    }
    pthread_barrier_init(&p->bar, NULL, W);
    p->th = (pthread_t*)malloc(W * sizeof(pthread_t));
    part_arg* args = (part_arg*)malloc(W * sizeof(part_arg));
    for (uint32_t i = 1; i < W; ++i) {
        args[i].p = p; args[i].id = i;
        pthread_create(&p->th[i], NULL, partition_worker, &args[i]);
    }
    args[0].p = p; args[0].id = 0;   /* worker 0 is the calling thread */
    p->args = args;
    return p;
}

void orc_partition_train(orc_partition* p, uint32_t iters)
{
    p->iters = iters;
    p->stop = 0;
    /* worker 0 runs on the calling thread: one train() call = one pass of
     * the worker loop body, bracketed by the start/end barriers. */
    uint32_t W = p->W;
    uint64_t* order = (uint64_t*)malloc((p->D / W + 2) * sizeof(uint64_t));
    if (W > 1) pthread_barrier_wait(&p->bar);
    for (uint32_t it = 0; it < iters; ++it) {
        for (uint32_t i = 0; i < W; ++i) {
            uint32_t didx = i % W;
            uint64_t n = (p->D + (W - 1) - didx) / W;
            orc_shuffled_order(n, (size_t)(splitmix64(&p->rng[0]) & 0xFFFFFFFFu), order);
            for (uint64_t j = 0; j < n; ++j) {
                uint64_t d = order[j] * W + didx;
                uint64_t b = p->doc_off[d] + p->chunk_off[d];
                uint64_t e = p->doc_off[d] + p->chunk_off[(uint64_t)1 * p->D + d];
                sample_doc_range(p->K, p->V, p->alpha, p->eta, p->veta, p->words, p->z, b, e,
                                 p->ndk + d * p->K, p->nkw, p->local_nk[0], p->dist[0], &p->rng[0]);
            }
            if (W > 1) pthread_barrier_wait(&p->bar);
        }
        memset(p->nk, 0, p->K * sizeof(int32_t));
        for (uint32_t v = 0; v < p->V; ++v) {
            const int32_t* col = p->nkw + (size_t)v * p->K;
            for (uint32_t k = 0; k < p->K; ++k) p->nk[k] += col[k];
        }
        if (W > 1) pthread_barrier_wait(&p->bar);
        memcpy(p->local_nk[0], p->nk, p->K * sizeof(int32_t));
        if (W > 1) pthread_barrier_wait(&p->bar);
    }
    if (W > 1) pthread_barrier_wait(&p->bar);
    free(order);
}

void orc_partition_destroy(orc_partition* p)
{
    if (!p) return;
    if (p->W > 1) {
        p->stop = 1;
        pthread_barrier_wait(&p->bar);
        for (uint32_t i = 1; i < p->W; ++i) pthread_join(p->th[i], NULL);
    }
    pthread_barrier_destroy(&p->bar);
    for (uint32_t i = 0; i < p->W; ++i) { free(p->local_nk[i]); free(p->dist[i]); }
    free(p->local_nk); free(p->dist); free(p->rng); free(p->vchunk); free(p->chunk_off);
    free(p->th); free(p->args); free(p);
}

/* ------------------------------------------------------------------------ */
/* Log-likelihood                                                           */
/* ------------------------------------------------------------------------ */
static float alpha_sum_f(uint32_t K, const float* alpha)
{
    float s = 0.f;
    for (uint32_t k = 0; k < K; ++k) s += alpha[k];
    return s;
}

double orc_ll_docs_lut(uint64_t D, uint32_t K, const int32_t* ndk, const int32_t* doc_len,
                       const float* alpha)
{
    double ll = 0;
    float as = alpha_sum_f(K, alpha);
    for (uint64_t d = 0; d < D; ++d) {
        ll -= orc_lgammaT((float)doc_len[d] + as) - orc_lgammaT(as);
        for (uint32_t k = 0; k < K; ++k)
            ll += orc_lgammaT((float)ndk[d * K + k] + alpha[k]) - orc_lgammaT(alpha[k]);
    }
    return ll;
}

double orc_ll_rest_lut(uint32_t K, uint32_t V, const int32_t* nkw, const int32_t* nk, float eta)
{
    double ll = 0;
    float lge = orc_lgammaT(eta);
    float veta = (float)V * eta;
    ll += orc_lgammaT(veta) * K;
    for (uint32_t k = 0; k < K; ++k) {
        ll -= orc_lgammaT((float)nk[k] + veta);
        for (uint32_t v = 0; v < V; ++v) {
            int32_t c = nkw[(size_t)v * K + k];
            if (!c) continue;
            ll += orc_lgammaT((float)c + eta) - lge;
        }
    }
    return ll;
}

double orc_ll_docs_f64(uint64_t D, uint32_t K, const int32_t* ndk, const int32_t* doc_len,
                       const float* alpha)
{
    double ll = 0, as = 0;
    for (uint32_t k = 0; k < K; ++k) as += (double)alpha[k];
    double lgas = lgamma(as);
    for (uint64_t d = 0; d < D; ++d) {
        double s = 0;
        for (uint32_t k = 0; k < K; ++k) {
            int32_t c = ndk[d * K + k];
            if (!c) continue;
            s += lgamma((double)c + (double)alpha[k]) - lgamma((double)alpha[k]);
        }
        ll += s - (lgamma((double)doc_len[d] + as) - lgas);
    }
    return ll;
}

double orc_ll_rest_f64(uint32_t K, uint32_t V, const int32_t* nkw, const int32_t* nk, float eta)
{
    double ll = 0, e = (double)eta, veta = (double)V * (double)eta;
    double lge = lgamma(e);
    ll += lgamma(veta) * K;
    for (uint32_t k = 0; k < K; ++k) ll -= lgamma((double)nk[k] + veta);
    for (uint64_t i = 0; i < (uint64_t)V * K; ++i) {
        if (!nkw[i]) continue;
        ll += lgamma((double)nkw[i] + e) - lge;
    }
    return ll;
}

/* ------------------------------------------------------------------------ */
/* optimizeParameters (LDAModel.hpp:221-265)                                */
/* ------------------------------------------------------------------------ */
void orc_optimize_alpha(uint64_t D, uint32_t K, const int32_t* ndk, const int32_t* doc_len,
                        float* alpha)
{
    for (int it = 0; it < 10; ++it) {
        float as = alpha_sum_f(K, alpha);
        float dsum = orc_digammaT(as);
        double denom = 0;
        for (uint64_t d = 0; d < D; ++d)
            denom += (double)(orc_digammaApprox((float)doc_len[d] + as) - dsum);
        for (uint32_t k = 0; k < K; ++k) {
            float dk = orc_digammaT(alpha[k]);
            double nom = 0;
            for (uint64_t d = 0; d < D; ++d)
                nom += (double)(orc_digammaApprox((float)ndk[d * K + k] + alpha[k]) - dk);
            float a = (float)nom / (float)denom * alpha[k];
            alpha[k] = a > 1e-5f ? a : 1e-5f;
        }
    }
}

/* ------------------------------------------------------------------------ */
/* Per-document infer (LDAModel.hpp:920-953)                                */
/* ------------------------------------------------------------------------ */
static uint32_t blocked_draw(const float* A, const float* phi, uint32_t K, uint32_t zo, float phi_own, float u);

/* The device's infer semantics for one (vid-sorted) document:
 *   z0 ~ Discrete(alpha) (u = Philox(j, 0xFFFFFFFF, doc_key)), added to the doc's counts;
 *   `iters` sweeps over the tokens in order; for token j of word v (own assignment removed):
 *     A_k = (float)n_dk[k] + alpha_k
 *     B_k = (float)(n_kw[k,v] + own[k]) + eta      own = the doc's other tokens of word v
 *     R_k = 1 / ((float)(n_k[k] + n_dk[k]) + V*eta)
 *     weight A_k * (B_k * R_k), drawn with blocked_draw (no own-topic term),
 *     u = Philox(j, sweep, doc_key) under key seed ^ 'INFR';
 *   theta_k = ((float)n_dk[k] + alpha_k) / ((float)N_d + sum(alpha))   (_getTopicsByDoc)
 *   ll = LLRest(model + doc) - LLRest(model) + LLDocs(doc) in FP64 (only touched cells). */
double orc_infer_doc(uint32_t K, uint32_t V, const float* alpha, float eta,
                     const int32_t* nkw, const int32_t* nk,
                     const uint32_t* words, uint32_t len, uint32_t iters,
                     uint64_t seed, uint64_t doc_key, uint16_t* z, int32_t* ndk, float* theta)
{
    float veta = eta * (float)V;
    uint64_t key = seed ^ (uint64_t)ORC_STREAM_INFER;
    uint32_t klo = (uint32_t)doc_key, khi = (uint32_t)(doc_key >> 32);
    int32_t* own = (int32_t*)calloc(K, sizeof(int32_t));
    float* A = (float*)malloc(K * sizeof(float));
    float* BR = (float*)malloc(K * sizeof(float));
    float* acum = (float*)malloc(K * sizeof(float));
    float s = 0.f;
    for (uint32_t k = 0; k < K; ++k) { s = s + alpha[k]; acum[k] = s; }
    memset(ndk, 0, K * sizeof(int32_t));
    for (uint32_t j = 0; j < len; ++j) {
        if (words[j] >= V) { z[j] = 0xFFFF; continue; }
        float u = orc_u01(philox_first(j, 0xFFFFFFFFu, klo, khi, key));
        uint16_t k = (uint16_t)orc_sample_acc(acum, K, u);
        z[j] = k;
        ndk[k]++;
    }
    for (uint32_t it = 0; it < iters; ++it) {
        uint32_t rb = 0;
        while (rb < len) {
            uint32_t re = rb + 1;
            while (re < len && words[re] == words[rb]) ++re;
            uint32_t v = words[rb];
            if (v < V) {
                for (uint32_t j = rb; j < re; ++j) own[z[j]]++;
                const int32_t* g = nkw + (size_t)v * K;
                for (uint32_t j = rb; j < re; ++j) {
                    uint16_t zo = z[j];
                    own[zo]--;
                    ndk[zo]--;
                    for (uint32_t k = 0; k < K; ++k) {
                        A[k] = (float)ndk[k] + alpha[k];
                        float B = (float)(g[k] + own[k]) + eta;
                        float R = 1.0f / ((float)(nk[k] + ndk[k]) + veta);
                        BR[k] = B * R;
                    }
                    float u = orc_u01(philox_first(j, it, klo, khi, key));
                    uint16_t zn = (uint16_t)blocked_draw(A, BR, K, 0xFFFFFFFFu, 0.f, u);
                    z[j] = zn;
                    ndk[zn]++;
                    own[zn]++;
                }
                for (uint32_t j = rb; j < re; ++j) own[z[j]]--;
            }
            rb = re;
        }
    }
    /* ll over touched cells, FP64 */
    double e = (double)eta, vd = (double)V * (double)eta, ll = 0, as = 0;
    float asf = 0.f;
    uint32_t n = 0;
    for (uint32_t k = 0; k < K; ++k) { as += (double)alpha[k]; asf = asf + alpha[k]; }
    for (uint32_t j = 0; j < len; ++j) n += words[j] < V;
    for (uint32_t k = 0; k < K; ++k) {
        if (!ndk[k]) continue;
        ll += lgamma((double)nk[k] + vd) - lgamma((double)(nk[k] + ndk[k]) + vd);
        ll += lgamma((double)ndk[k] + alpha[k]) - lgamma((double)alpha[k]);
    }
    ll -= lgamma((double)n + as) - lgamma(as);
    uint32_t rb = 0;
    while (rb < len) {
        uint32_t re = rb + 1;
        while (re < len && words[re] == words[rb]) ++re;
        uint32_t v = words[rb];
        if (v < V) {
            const int32_t* g = nkw + (size_t)v * K;
            for (uint32_t j = rb; j < re; ++j) own[z[j]]++;
            for (uint32_t j = rb; j < re; ++j) {
                uint32_t k = z[j];
                int32_t c = own[k];
                if (!c) continue;          /* cell already counted */
                double after = lgamma((double)(g[k] + c) + e);
                double before = g[k] ? lgamma((double)g[k] + e) : lgamma(e);
                ll += after - before;
                own[k] = 0;
            }
        }
        rb = re;
    }
    if (theta)
        for (uint32_t k = 0; k < K; ++k) theta[k] = ((float)ndk[k] + alpha[k]) / ((float)n + asf);
    free(own); free(A); free(BR); free(acum);
    return ll;
}

/* ------------------------------------------------------------------------ */
/* Doc-major sweep: live n_dk, snapshot n_kw / n_k  (the device semantics)  */
/* ------------------------------------------------------------------------ */
/* tomotopy's COPY_MERGE with one worker per document (LDAModel.hpp:401-423,
 * 555-570): each document is sampled sequentially with its own n_dk live;
 * n_kw and n_k are the start-of-sweep copy with the token's own assignment
 * removed; every count delta lands in the next state after the sweep.
 *
 * Arithmetic (each operation rounded to nearest, no contraction unless fma):
 *   R_k      = 1 / ((float)n_k[k] + V*eta)
 *   phi_k    = ((float)n_kw[k,v] + eta) * R_k             (per word, per sweep)
 *   phi_own  = ((float)(n_kw[zo,v]-1) + eta) * (1 / ((float)(n_k[zo]-1) + V*eta))
 *   A_k      = (float)n_dk[k] + alpha_k                    (own token removed)
 * Topics are dealt to 32 lanes in blocks of four: lane l owns the topics
 * k = 128*j + 4*l + i (j = 0, 1, ..., i = 0..3, k < K), in that order.
 * Pass 1: T_l = fma-chain of A_k * phi_k over lane l's topics (s = fma(A, phi,
 * s) from s = 0), the own topic zo contributing fma(0, phi_zo, s) = s; the
 * lane owning zo then adds T_l = T_l + A_zo*phi_own (no subtraction, so no
 * cancellation when A_zo*phi_zo would dominate the lane).  X = Hillis-Steele inclusive scan of T over 32 lanes,
 * E_l = X_{l-1} (E_0 = 0), r = u * X_31, u = Philox(token index, step).
 * h = first lane owning a topic with r < E_h + T_h (none: K-1).
 * Pass 2: x_t = A_k * phi_k (phi_own at zo) over lane h's topics in order,
 * in chunks of 32, each Hillis-Steele scanned and offset by the running
 * sum of the previous chunks: P_t; result = lane h's t-th topic for the
 * first t with r < E_h + P_t, else lane h's last topic.  Any fixed topic
 * order draws from the same distribution; this one makes each warp-wide
 * load a contiguous 512-byte run. */
static void hs32(float* x)   /* Hillis-Steele inclusive scan of 32 values */
{
    float y[32];
    for (uint32_t off = 1; off < 32; off <<= 1) {
        for (uint32_t l = 0; l < 32; ++l) y[l] = (l >= off) ? x[l] + x[l - off] : x[l];
        memcpy(x, y, sizeof(y));
    }
}

/* the t-th topic of lane l, or -1 */
static inline int64_t lane_topic(uint32_t l, uint32_t t, uint32_t K)
{
    uint64_t k = 128ull * (t >> 2) + 4ull * l + (t & 3);
    return k < K ? (int64_t)k : -1;
}

static inline uint32_t lane_count(uint32_t l, uint32_t K)
{
    uint32_t n = 0;
    for (uint32_t j = 0; 128 * j + 4 * l < K; ++j) {
        uint32_t b = 128 * j + 4 * l;
        n += (K - b) >= 4 ? 4 : (K - b);
    }
    return n;
}

/* A: doc row A_k; phi: word weights; zo, phi_own: the own topic */
static uint32_t blocked_draw(const float* A, const float* phi, uint32_t K, uint32_t zo, float phi_own, float u)
{
    float T[32], X[32];
    uint32_t cl[32];
    for (uint32_t l = 0; l < 32; ++l) {
        float s = 0.f;
        cl[l] = lane_count(l, K);
        /* the own topic is left out of the chain (its document weight reads 0:
         * fmaf(0, phi, s) == s) and added last by its lane: no subtraction */
        for (uint32_t t = 0; t < cl[l]; ++t) {
            int64_t k = lane_topic(l, t, K);
            s = fmaf((uint32_t)k == zo ? 0.f : A[k], phi[k], s);
        }
        if (zo < K && ((zo >> 2) & 31) == l) s = s + A[zo] * phi_own;
        T[l] = s;
        X[l] = s;
    }
    hs32(X);
    float total = X[31];
    float r = u * total;
    int h = -1;
    float E = 0.f;
    for (uint32_t l = 0; l < 32; ++l) {
        float El = l ? X[l - 1] : 0.f;
        if (cl[l] && r < El + T[l]) { h = (int)l; E = El; break; }
    }
    if (h < 0) return K - 1;
    uint32_t n = cl[h];
    float carry = 0.f;
    for (uint32_t m = 0; m < n; m += 32) {
        float x[32];
        for (uint32_t t = 0; t < 32; ++t) {
            if (m + t < n) {
                int64_t k = lane_topic((uint32_t)h, m + t, K);
                x[t] = A[k] * ((zo < K && (uint32_t)k == zo) ? phi_own : phi[k]);
            } else {
                x[t] = 0.f;
            }
        }
        hs32(x);
        for (uint32_t t = 0; t < 32 && m + t < n; ++t)
            if (r < E + (carry + x[t])) return (uint32_t)lane_topic((uint32_t)h, m + t, K);
        carry = carry + x[31];
    }
    return (uint32_t)lane_topic((uint32_t)h, n - 1, K);
}

/* The conditional blocked_draw implies: width[k] = the length of the set of
 * r = u * total in [0, total) that the draw maps to topic k, formed from the
 * same float lane totals, lane scan and pass-2 prefix sums (a lane is hit for
 * r below fl(E_h + T_h); inside it, topic t for r below fl(E_h + P_t), the
 * lane's last topic taking the rest; r past every lane goes to K-1).
 * start[k] (may be NULL): where topic k's interval begins (-1 if empty;
 * every interval but K-1's is one contiguous range).
 * Returns total; width sums to total.  Test infrastructure for the 1e-5
 * gate on the kernel's own arithmetic. */
float orc_draw_intervals(const float* A, const float* phi, uint32_t K, uint32_t zo, float phi_own,
                         double* width, double* start)
{
    float T[32], X[32];
    uint32_t cl[32];
    for (uint32_t k = 0; k < K; ++k) { width[k] = 0.0; if (start) start[k] = -1.0; }
    for (uint32_t l = 0; l < 32; ++l) {
        float s = 0.f;
        cl[l] = lane_count(l, K);
        for (uint32_t t = 0; t < cl[l]; ++t) {
            int64_t k = lane_topic(l, t, K);
            s = fmaf((uint32_t)k == zo ? 0.f : A[k], phi[k], s);
        }
        if (zo < K && ((zo >> 2) & 31) == l) s = s + A[zo] * phi_own;
        T[l] = s;
        X[l] = s;
    }
    hs32(X);
    const float total = X[31];
    double lo = 0.0;                         /* r below lo is taken by earlier lanes */
    for (uint32_t l = 0; l < 32; ++l) {
        if (!cl[l]) continue;
        const float E = l ? X[l - 1] : 0.f;
        const double b = (double)(E + T[l]);
        const double lane_hi = b < (double)total ? b : (double)total;
        if (lane_hi > lo) {
            double tlo = lo;
            float carry = 0.f;
            const uint32_t n = cl[l];
            for (uint32_t m = 0; m < n; m += 32) {
                float x[32];
                for (uint32_t t = 0; t < 32; ++t) {
                    if (m + t < n) {
                        int64_t k = lane_topic(l, m + t, K);
                        x[t] = A[k] * ((uint32_t)k == zo ? phi_own : phi[k]);
                    } else {
                        x[t] = 0.f;
                    }
                }
                hs32(x);
                for (uint32_t t = 0; t < 32 && m + t < n; ++t) {
                    const int64_t k = lane_topic(l, m + t, K);
                    double hi = (m + t == n - 1) ? lane_hi : (double)(E + (carry + x[t]));
                    if (hi > lane_hi) hi = lane_hi;
                    if (hi > tlo) { if (start) start[k] = tlo; width[k] += hi - tlo; tlo = hi; }
                }
                carry = carry + x[31];
            }
        }
        if (b > lo) lo = b;
    }
    if ((double)total > lo) {
        if (start && width[K - 1] == 0.0) start[K - 1] = lo;
        width[K - 1] += (double)total - lo;
    }
    return total;
}

/* blocked_draw itself, for tests: the topic drawn for u (and *total) */
uint32_t orc_blocked_draw(const float* A, const float* phi, uint32_t K, uint32_t zo, float phi_own, float u)
{
    return blocked_draw(A, phi, K, zo, phi_own, u);
}

/* The same for tomotopy's draw (getZLikelihoods + prefixSum + sampleFromDiscreteAcc,
 * LDAModel.hpp:273-285, sample.hpp:69-86, 133-189): dist_k = (A_k * B_k) / C_k
 * in float, the SSE-order prefix sum cum, r = u * cum[K-1], first k with
 * r < cum[k]; width[k] from cum's running maximum.  A, B, C: the three
 * factors with the token removed. */
float orc_ref_draw_intervals(const float* A, const float* B, const float* C, uint32_t K, double* width)
{
    float* cum = (float*)aligned_alloc(64, ((K + 15) / 16) * 64);
    for (uint32_t k = 0; k < K; ++k) cum[k] = (A[k] * B[k]) / C[k];
    orc_prefix_sum_sse(cum, (int)K);
    const float total = cum[K - 1];
    double lo = 0.0;
    for (uint32_t k = 0; k < K; ++k) {
        double hi = (double)cum[k] < (double)total ? (double)cum[k] : (double)total;
        width[k] = hi > lo ? hi - lo : 0.0;
        if (hi > lo) lo = hi;
    }
    if ((double)total > lo) width[K - 1] += (double)total - lo;
    free(cum);
    return total;
}

void orc_sweep_doc_live_subset(uint32_t K, uint32_t V, const float* alpha, float eta,
                        uint64_t seed, uint32_t iter, uint64_t D, const uint64_t* doc_off,
                        const uint32_t* words, int32_t* ndk,
                        const int32_t* nkw, const int32_t* nk,
                        int32_t* nkw_next, int32_t* nk_next, uint16_t* z,
                        const uint64_t* docs, uint64_t n_docs)
{
    (void)D;
    float veta = eta * (float)V;
    float* R = (float*)malloc(K * sizeof(float));
    float* A = (float*)malloc(K * sizeof(float));
    float* phi = (float*)malloc(K * sizeof(float));
    for (uint32_t k = 0; k < K; ++k) R[k] = 1.0f / ((float)nk[k] + veta);
    for (uint64_t di = 0; di < n_docs; ++di) {
        uint64_t d = docs ? docs[di] : di;
        int32_t* row = ndk + d * K;
        for (uint32_t k = 0; k < K; ++k) A[k] = (float)row[k] + alpha[k];
        for (uint64_t i = doc_off[d]; i < doc_off[d + 1]; ++i) {
            uint32_t v = words[i];
            if (v >= V) continue;
            uint16_t zo = z[i];
            const int32_t* col = nkw + (size_t)v * K;
            row[zo]--;
            A[zo] = (float)row[zo] + alpha[zo];
            for (uint32_t k = 0; k < K; ++k) phi[k] = ((float)col[k] + eta) * R[k];
            float phi_own = ((float)(col[zo] - 1) + eta) * (1.0f / ((float)(nk[zo] - 1) + veta));
            float u = orc_u01(philox_first((uint32_t)i, (uint32_t)(i >> 32), ORC_STREAM_SWEEP, iter, seed));
            uint16_t zn = (uint16_t)blocked_draw(A, phi, K, zo, phi_own, u);
            row[zn]++;
            A[zn] = (float)row[zn] + alpha[zn];
            z[i] = zn;
            if (zn != zo) {
                nkw_next[(size_t)v * K + zo]--; nkw_next[(size_t)v * K + zn]++;
                nk_next[zo]--; nk_next[zn]++;
            }
        }
    }
    free(R); free(A); free(phi);
}

/* One document group of the device sweep, generic over the conditional's
 * options (word priors, per-document alphas and masks) and with the
 * long-document split.  A document of at least split_len tokens (all ids
 * counted) is cut into `slices` contiguous position ranges, slice w =
 * [b + w*L/slices, b + (w+1)*L/slices) (integer division); they are sampled
 * side by side in steps of `step` positions: in step s every slice samples its
 * positions [s*step, (s+1)*step) in order with a private copy of the
 * document's n_dk row -- the row as of the start of the step plus its own
 * changes -- and after the step the row gains every slice's changes.  A
 * shorter document is sampled in order with its row live (split_len = 0:
 * every document).  Draws, n_kw / n_k snapshots and deltas as
 * orc_sweep_doc_live_subset. */
/* orc_sweep_spec: see tmt_oracle.h */
static inline float mask_bit(const uint32_t* mask, uint32_t mw, uint64_t d, uint32_t k);

typedef struct {
    const orc_sweep_spec* sp;
    const float* al; uint64_t d;
    float* R; float* phi; float veta; uint32_t mw;
} sweep_ctx;

static inline float sweep_afold(const sweep_ctx* c, int32_t n, uint32_t k)
{
    const float x = (float)n + c->al[k];
    return c->sp->mask ? x * mask_bit(c->sp->mask, c->mw, c->d, k) : x;
}

/* tokens [tb, te) of document c->d with the row `row` (and A) live; the
 * row's changes are also added to dlt when dlt != NULL */
static void sweep_tokens(const sweep_ctx* c, uint64_t tb, uint64_t te, int32_t* row, float* A, int32_t* dlt)
{
    const orc_sweep_spec* sp = c->sp;
    const uint32_t K = sp->K;
    for (uint64_t i = tb; i < te; ++i) {
        uint32_t v = sp->words[i];
        if (v >= sp->V) continue;
        uint16_t zo = sp->z[i];
        const int32_t* col = sp->nkw + (size_t)v * K;
        const float* pe = (sp->pidx && sp->pidx[v] >= 0) ? sp->prior + (size_t)sp->pidx[v] * K : NULL;
        row[zo]--;
        A[zo] = sweep_afold(c, row[zo], zo);
        for (uint32_t k = 0; k < K; ++k) c->phi[k] = ((float)col[k] + (pe ? pe[k] : sp->eta)) * c->R[k];
        const float so = sp->esum ? sp->esum[zo] : c->veta;
        float phi_own = ((float)(col[zo] - 1) + (pe ? pe[zo] : sp->eta)) * (1.0f / ((float)(sp->nk[zo] - 1) + so));
        float u = orc_u01(philox_first((uint32_t)i, (uint32_t)(i >> 32), ORC_STREAM_SWEEP, sp->iter, sp->seed));
        uint16_t zn = (uint16_t)blocked_draw(A, c->phi, K, zo, phi_own, u);
        row[zn]++;
        A[zn] = sweep_afold(c, row[zn], zn);
        sp->z[i] = zn;
        if (zn != zo) {
            sp->nkw_next[(size_t)v * K + zo]--; sp->nkw_next[(size_t)v * K + zn]++;
            sp->nk_next[zo]--; sp->nk_next[zn]++;
            if (dlt) { dlt[zo]--; dlt[zn]++; }
        }
    }
}

void orc_sweep_docs(const orc_sweep_spec* sp, const uint64_t* docs, uint64_t n_docs)
{
    const uint32_t K = sp->K;
    sweep_ctx c;
    c.sp = sp;
    c.veta = sp->eta * (float)sp->V;
    c.mw = (K + 31) / 32;
    c.R = (float*)malloc(K * sizeof(float));
    c.phi = (float*)malloc(K * sizeof(float));
    float* A = (float*)malloc(K * sizeof(float));
    int32_t* P = (int32_t*)malloc(K * sizeof(int32_t));
    int32_t* dlt = (int32_t*)malloc(K * sizeof(int32_t));
    for (uint32_t k = 0; k < K; ++k) c.R[k] = 1.0f / ((float)sp->nk[k] + (sp->esum ? sp->esum[k] : c.veta));
    for (uint64_t di = 0; di < n_docs; ++di) {
        const uint64_t d = docs ? docs[di] : di;
        c.d = d;
        c.al = sp->arow ? sp->alpha_rows + (size_t)sp->arow[d] * K : sp->alpha;
        int32_t* row = sp->ndk + d * K;
        if (sp->unit_off) {              /* a shared row: its documents in order, the row live */
            for (uint32_t k = 0; k < K; ++k) A[k] = sweep_afold(&c, row[k], k);
            for (uint64_t u = sp->unit_off[d]; u < sp->unit_off[d + 1]; ++u) {
                const uint64_t dd = sp->unit_docs[u];
                sweep_tokens(&c, sp->doc_off[dd], sp->doc_off[dd + 1], row, A, NULL);
            }
            continue;
        }
        const uint64_t b = sp->doc_off[d], e = sp->doc_off[d + 1], L = e - b;
        if (!sp->split_len || L < sp->split_len || sp->slices < 2) {
            for (uint32_t k = 0; k < K; ++k) A[k] = sweep_afold(&c, row[k], k);
            sweep_tokens(&c, b, e, row, A, NULL);
            continue;
        }
        const uint32_t S = sp->slices, m = sp->step;
        uint64_t longest = 0;
        for (uint32_t w = 0; w < S; ++w) {
            const uint64_t n = (uint64_t)(w + 1) * L / S - (uint64_t)w * L / S;
            if (n > longest) longest = n;
        }
        for (uint64_t s = 0; s * m < longest; ++s) {
            for (uint32_t k = 0; k < K; ++k) dlt[k] = 0;
            for (uint32_t w = 0; w < S; ++w) {
                const uint64_t sb = b + (uint64_t)w * L / S, se = b + (uint64_t)(w + 1) * L / S;
                uint64_t tb = sb + s * m, te = tb + m;
                if (tb >= se) continue;
                if (te > se) te = se;
                for (uint32_t k = 0; k < K; ++k) { P[k] = row[k]; A[k] = sweep_afold(&c, P[k], k); }
                sweep_tokens(&c, tb, te, P, A, dlt);
            }
            for (uint32_t k = 0; k < K; ++k) row[k] += dlt[k];
        }
    }
    free(c.R); free(c.phi); free(A); free(P); free(dlt);
}

void orc_sweep_doc_live(uint32_t K, uint32_t V, const float* alpha, float eta,
                        uint64_t seed, uint32_t iter, uint64_t D, const uint64_t* doc_off,
                        const uint32_t* words, int32_t* ndk,
                        const int32_t* nkw, const int32_t* nk,
                        int32_t* nkw_next, int32_t* nk_next, uint16_t* z)
{
    orc_sweep_doc_live_subset(K, V, alpha, eta, seed, iter, D, doc_off, words, ndk, nkw, nk,
                              nkw_next, nk_next, z, NULL, D);
}

/* ------------------------------------------------------------------------ */
/* Weighted counts: TermWeight IDF / PMI (LDAModel.hpp:287-299, 795-809,     */
/* 1093-1122; Utils.hpp:132-155)                                            */
/* ------------------------------------------------------------------------ */
/* Every token carries a float weight (IDF: vocabWeights[v]; PMI: the
 * per-document formula); n_dk, n_kw and n_k are float sums of weights and a
 * decrement clamps at 0 (updateCnt<true>).  The device semantics restated
 * here: a document's n_dk row is updated in float in token order by its
 * warp; the model counts are float states that change only between document
 * groups, by folding the group's deltas, which accumulate as integers in
 * units of 2^-24 (each token weight rounded to that grid), so the fold is
 * independent of the order of the atomic adds. */
int64_t orc_wq(float w)
{
    return (int64_t)llrintf(w * 16777216.0f);
}

float orc_fold(float n, int64_t q)
{
    float d = (float)q * 5.9604644775390625e-8f;   /* 2^-24 */
    float s = n + d;
    return s > 0.f ? s : 0.f;
}

void orc_fold_w(uint32_t K, uint32_t V, float* nkw, float* nk, int64_t* dkw, int64_t* dk)
{
    for (uint32_t k = 0; k < K; ++k) { nk[k] = orc_fold(nk[k], dk[k]); dk[k] = 0; }
    for (uint64_t i = 0; i < (uint64_t)V * K; ++i) { nkw[i] = orc_fold(nkw[i], dkw[i]); dkw[i] = 0; }
}

void orc_counts_from_z_w(uint64_t D, const uint64_t* doc_off, const uint32_t* words,
                         const uint16_t* z, const float* wt, uint32_t V, uint32_t K,
                         float* ndk, float* doc_wlen, float* nkw, float* nk)
{
    int64_t* qkw = (int64_t*)calloc((size_t)V * K, sizeof(int64_t));
    int64_t* qk = (int64_t*)calloc(K, sizeof(int64_t));
    memset(ndk, 0, (size_t)D * K * sizeof(float));
    for (uint64_t d = 0; d < D; ++d) {
        float len = 0.f;
        for (uint64_t i = doc_off[d]; i < doc_off[d + 1]; ++i) {
            uint32_t v = words[i];
            if (v >= V) continue;
            float w = wt[i];
            ndk[d * K + z[i]] += w;
            len += w;
            int64_t q = orc_wq(w);
            qkw[(size_t)v * K + z[i]] += q;
            qk[z[i]] += q;
        }
        doc_wlen[d] = len;
    }
    for (uint32_t k = 0; k < K; ++k) nk[k] = orc_fold(0.f, qk[k]);
    for (uint64_t i = 0; i < (uint64_t)V * K; ++i) nkw[i] = orc_fold(0.f, qkw[i]);
    free(qkw);
    free(qk);
}

void orc_sweep_doc_live_w_subset(uint32_t K, uint32_t V, const float* alpha, float eta,
                                 uint64_t seed, uint32_t iter, const uint64_t* doc_off,
                                 const uint32_t* words, const float* wt, float* ndk,
                                 const float* nkw, const float* nk, int64_t* dkw, int64_t* dk,
                                 uint16_t* z, const uint64_t* docs, uint64_t n_docs)
{
    float veta = eta * (float)V;
    float* R = (float*)malloc(K * sizeof(float));
    float* A = (float*)malloc(K * sizeof(float));
    float* phi = (float*)malloc(K * sizeof(float));
    for (uint32_t k = 0; k < K; ++k) R[k] = 1.0f / (nk[k] + veta);
    for (uint64_t di = 0; di < n_docs; ++di) {
        uint64_t d = docs ? docs[di] : di;
        float* row = ndk + d * K;
        for (uint32_t k = 0; k < K; ++k) A[k] = row[k] + alpha[k];
        for (uint64_t i = doc_off[d]; i < doc_off[d + 1]; ++i) {
            uint32_t v = words[i];
            if (v >= V) continue;
            uint16_t zo = z[i];
            float w = wt[i];
            const float* col = nkw + (size_t)v * K;
            float n = row[zo] - w;
            row[zo] = n > 0.f ? n : 0.f;
            A[zo] = row[zo] + alpha[zo];
            for (uint32_t k = 0; k < K; ++k) phi[k] = (col[k] + eta) * R[k];
            float co = col[zo] - w, no = nk[zo] - w;
            co = co > 0.f ? co : 0.f;
            no = no > 0.f ? no : 0.f;
            float phi_own = (co + eta) * (1.0f / (no + veta));
            float u = orc_u01(philox_first((uint32_t)i, (uint32_t)(i >> 32), ORC_STREAM_SWEEP, iter, seed));
            uint16_t zn = (uint16_t)blocked_draw(A, phi, K, zo, phi_own, u);
            row[zn] = row[zn] + w;
            A[zn] = row[zn] + alpha[zn];
            z[i] = zn;
            if (zn != zo) {
                int64_t q = orc_wq(w);
                dkw[(size_t)v * K + zo] -= q; dkw[(size_t)v * K + zn] += q;
                dk[zo] -= q; dk[zn] += q;
            }
        }
    }
    free(R); free(A); free(phi);
}

double orc_ll_docs_w_f64(uint64_t D, uint32_t K, const float* ndk, const float* doc_wlen,
                         const float* alpha)
{
    double ll = 0, as = 0;
    for (uint32_t k = 0; k < K; ++k) as += (double)alpha[k];
    double lgas = lgamma(as);
    for (uint64_t d = 0; d < D; ++d) {
        double s = 0;
        for (uint32_t k = 0; k < K; ++k) {
            float c = ndk[d * K + k];
            if (c == 0.f) continue;
            s += lgamma((double)c + (double)alpha[k]) - lgamma((double)alpha[k]);
        }
        ll += s - (lgamma((double)doc_wlen[d] + as) - lgas);
    }
    return ll;
}

double orc_ll_rest_w_f64(uint32_t K, uint32_t V, const float* nkw, const float* nk, float eta)
{
    double ll = 0, e = (double)eta, veta = (double)V * (double)eta;
    double lge = lgamma(e);
    ll += lgamma(veta) * K;
    for (uint32_t k = 0; k < K; ++k) ll -= lgamma((double)nk[k] + veta);
    for (uint64_t i = 0; i < (uint64_t)V * K; ++i) {
        if (nkw[i] == 0.f) continue;
        ll += lgamma((double)nkw[i] + e) - lge;
    }
    return ll;
}

void orc_optimize_alpha_w(uint64_t D, uint32_t K, const float* ndk, const float* doc_wlen, float* alpha)
{
    for (int it = 0; it < 10; ++it) {
        float as = alpha_sum_f(K, alpha);
        float dsum = orc_digammaT(as);
        double denom = 0;
        for (uint64_t d = 0; d < D; ++d)
            denom += (double)(orc_digammaApprox(doc_wlen[d] + as) - dsum);
        for (uint32_t k = 0; k < K; ++k) {
            float dk = orc_digammaT(alpha[k]);
            double nom = 0;
            for (uint64_t d = 0; d < D; ++d)
                nom += (double)(orc_digammaApprox(ndk[d * K + k] + alpha[k]) - dk);
            float a = (float)nom / (float)denom * alpha[k];
            alpha[k] = a > 1e-5f ? a : 1e-5f;
        }
    }
}

/* Per-document infer with weighted counts: the device's k_infer_slots<WT>.
 * n_dk starts from z0 in token order; within a run of one word (weight w),
 * B_k = (n_kw[k,v] + own_k * w) + eta, R_k = 1 / ((n_k[k] + n_dk[k]) + V*eta);
 * a removal clamps n_dk at 0; the document length is its weight sum. */
double orc_infer_doc_w(uint32_t K, uint32_t V, const float* alpha, float eta,
                       const float* nkw, const float* nk,
                       const uint32_t* words, const float* wt, uint32_t len, uint32_t iters,
                       uint64_t seed, uint64_t doc_key, uint16_t* z, float* ndk, float* theta)
{
    float veta = eta * (float)V;
    uint64_t key = seed ^ (uint64_t)ORC_STREAM_INFER;
    uint32_t klo = (uint32_t)doc_key, khi = (uint32_t)(doc_key >> 32);
    int32_t* own = (int32_t*)calloc(K, sizeof(int32_t));
    float* A = (float*)malloc(K * sizeof(float));
    float* BR = (float*)malloc(K * sizeof(float));
    float* acum = (float*)malloc(K * sizeof(float));
    float s = 0.f, wsum = 0.f;
    for (uint32_t k = 0; k < K; ++k) { s = s + alpha[k]; acum[k] = s; }
    memset(ndk, 0, K * sizeof(float));
    for (uint32_t j = 0; j < len; ++j) {
        if (words[j] >= V) { z[j] = 0xFFFF; continue; }
        float u = orc_u01(philox_first(j, 0xFFFFFFFFu, klo, khi, key));
        z[j] = (uint16_t)orc_sample_acc(acum, K, u);
    }
    for (uint32_t j = 0; j < len; ++j) {
        if (words[j] >= V) continue;
        ndk[z[j]] = ndk[z[j]] + wt[j];
        wsum = wsum + wt[j];
    }
    for (uint32_t it = 0; it < iters; ++it) {
        uint32_t rb = 0;
        while (rb < len) {
            uint32_t re = rb + 1;
            while (re < len && words[re] == words[rb]) ++re;
            uint32_t v = words[rb];
            if (v < V) {
                float w = wt[rb];
                for (uint32_t j = rb; j < re; ++j) own[z[j]]++;
                const float* g = nkw + (size_t)v * K;
                for (uint32_t j = rb; j < re; ++j) {
                    uint16_t zo = z[j];
                    own[zo]--;
                    float n = ndk[zo] - w;
                    ndk[zo] = n > 0.f ? n : 0.f;
                    for (uint32_t k = 0; k < K; ++k) {
                        A[k] = ndk[k] + alpha[k];
                        float B = (g[k] + (float)own[k] * w) + eta;
                        float R = 1.0f / ((nk[k] + ndk[k]) + veta);
                        BR[k] = B * R;
                    }
                    float u = orc_u01(philox_first(j, it, klo, khi, key));
                    uint16_t zn = (uint16_t)blocked_draw(A, BR, K, 0xFFFFFFFFu, 0.f, u);
                    z[j] = zn;
                    ndk[zn] = ndk[zn] + w;
                    own[zn]++;
                }
                for (uint32_t j = rb; j < re; ++j) own[z[j]]--;
            }
            rb = re;
        }
    }
    double e = (double)eta, vd = (double)V * (double)eta, ll = 0, as = 0;
    float asf = 0.f;
    for (uint32_t k = 0; k < K; ++k) { as += (double)alpha[k]; asf = asf + alpha[k]; }
    for (uint32_t k = 0; k < K; ++k) {
        if (ndk[k] == 0.f) continue;
        ll += lgamma((double)nk[k] + vd) - lgamma(((double)nk[k] + (double)ndk[k]) + vd);
        ll += lgamma((double)ndk[k] + alpha[k]) - lgamma((double)alpha[k]);
    }
    ll -= lgamma((double)wsum + as) - lgamma(as);
    uint32_t rb = 0;
    while (rb < len) {
        uint32_t re = rb + 1;
        while (re < len && words[re] == words[rb]) ++re;
        uint32_t v = words[rb];
        if (v < V) {
            const float* g = nkw + (size_t)v * K;
            float w = wt[rb];
            for (uint32_t j = rb; j < re; ++j) own[z[j]]++;
            for (uint32_t j = rb; j < re; ++j) {
                uint32_t k = z[j];
                int32_t c = own[k];
                if (!c) continue;
                double after = lgamma(((double)g[k] + (double)((float)c * w)) + e);
                double before = g[k] != 0.f ? lgamma((double)g[k] + e) : lgamma(e);
                ll += after - before;
                own[k] = 0;
            }
        }
        rb = re;
    }
    if (theta)
        for (uint32_t k = 0; k < K; ++k) theta[k] = (ndk[k] + alpha[k]) / (wsum + asf);
    free(own); free(A); free(BR); free(acum);
    return ll;
}

/* ------------------------------------------------------------------------ */
/* Word priors: set_word_prior (LDAModel.hpp:1031-1045, 724-737, 99-117)     */
/* ------------------------------------------------------------------------ */
/* etaByTopicWord is eta everywhere except the columns of prior words (pidx[v]
 * >= 0 names row pidx[v] of `prior`, K floats); esum[k] = its row sums:
 * (V - P) * eta plus the prior words' values in ascending word id, summed
 * in double and rounded once to float.  z0 of every token
 * ~ Discrete(its word's column) (updateStateWithDoc, :765-779), drawn like
 * orc_init_z from the column's sequential float cumulative sum. */
void orc_prior_esum(uint32_t K, uint32_t V, const int32_t* pidx, const float* prior, float eta, float* esum)
{
    uint32_t P = 0;
    for (uint32_t v = 0; v < V; ++v) P += pidx[v] >= 0;
    for (uint32_t k = 0; k < K; ++k) {
        double s = (double)(V - P) * (double)eta;
        for (uint32_t v = 0; v < V; ++v)
            if (pidx[v] >= 0) s += (double)prior[(size_t)pidx[v] * K + k];
        esum[k] = (float)s;
    }
}

static void column_cum(uint32_t K, const float* col, float eta, float* cum)
{
    float s = 0.f;
    for (uint32_t k = 0; k < K; ++k) { s = s + (col ? col[k] : eta); cum[k] = s; }
}

void orc_init_z_p(uint64_t N, const uint32_t* words, uint32_t V, uint32_t K, const int32_t* pidx,
                  const float* prior, float eta, uint64_t seed, uint16_t* z)
{
    float* cum = (float*)malloc(K * sizeof(float));
    for (uint64_t i = 0; i < N; ++i) {
        uint32_t v = words[i];
        if (v >= V) { z[i] = 0xFFFF; continue; }
        column_cum(K, pidx[v] >= 0 ? prior + (size_t)pidx[v] * K : NULL, eta, cum);
        float u = orc_u01(philox_first((uint32_t)i, (uint32_t)(i >> 32), ORC_STREAM_INIT, 0, seed));
        z[i] = (uint16_t)orc_sample_acc(cum, K, u);
    }
    free(cum);
}

/* one document group of the doc-major sweep with word priors:
 *   R_k = 1 / ((float)n_k[k] + esum_k), phi_k = ((float)n_kw[k,v] + eta_kv) * R_k,
 *   phi_own = ((float)(n_kw[zo,v] - 1) + eta_{zo,v}) * (1 / ((float)(n_k[zo] - 1) + esum_zo)) */
void orc_sweep_doc_live_p_subset(uint32_t K, uint32_t V, const float* alpha, float eta,
                                 const int32_t* pidx, const float* prior, const float* esum,
                                 uint64_t seed, uint32_t iter, const uint64_t* doc_off,
                                 const uint32_t* words, int32_t* ndk,
                                 const int32_t* nkw, const int32_t* nk,
                                 int32_t* nkw_next, int32_t* nk_next, uint16_t* z,
                                 const uint64_t* docs, uint64_t n_docs)
{
    float* R = (float*)malloc(K * sizeof(float));
    float* A = (float*)malloc(K * sizeof(float));
    float* phi = (float*)malloc(K * sizeof(float));
    for (uint32_t k = 0; k < K; ++k) R[k] = 1.0f / ((float)nk[k] + esum[k]);
    for (uint64_t di = 0; di < n_docs; ++di) {
        uint64_t d = docs ? docs[di] : di;
        int32_t* row = ndk + d * K;
        for (uint32_t k = 0; k < K; ++k) A[k] = (float)row[k] + alpha[k];
        for (uint64_t i = doc_off[d]; i < doc_off[d + 1]; ++i) {
            uint32_t v = words[i];
            if (v >= V) continue;
            uint16_t zo = z[i];
            const int32_t* col = nkw + (size_t)v * K;
            const float* pe = pidx[v] >= 0 ? prior + (size_t)pidx[v] * K : NULL;
            row[zo]--;
            A[zo] = (float)row[zo] + alpha[zo];
            for (uint32_t k = 0; k < K; ++k) phi[k] = ((float)col[k] + (pe ? pe[k] : eta)) * R[k];
            float phi_own = ((float)(col[zo] - 1) + (pe ? pe[zo] : eta)) * (1.0f / ((float)(nk[zo] - 1) + esum[zo]));
            float u = orc_u01(philox_first((uint32_t)i, (uint32_t)(i >> 32), ORC_STREAM_SWEEP, iter, seed));
            uint16_t zn = (uint16_t)blocked_draw(A, phi, K, zo, phi_own, u);
            row[zn]++;
            A[zn] = (float)row[zn] + alpha[zn];
            z[i] = zn;
            if (zn != zo) {
                nkw_next[(size_t)v * K + zo]--; nkw_next[(size_t)v * K + zn]++;
                nk_next[zo]--; nk_next[zn]++;
            }
        }
    }
    free(R); free(A); free(phi);
}

/* getLLRest with etaByTopicWord (LDAModel.hpp:636-651), FP64 */
double orc_ll_rest_p_f64(uint32_t K, uint32_t V, const int32_t* nkw, const int32_t* nk, float eta,
                         const int32_t* pidx, const float* prior, const float* esum)
{
    double ll = 0, e = (double)eta, lge = lgamma(e);
    for (uint32_t k = 0; k < K; ++k) ll += lgamma((double)esum[k]) - lgamma((double)nk[k] + (double)esum[k]);
    for (uint32_t v = 0; v < V; ++v) {
        const float* pe = pidx[v] >= 0 ? prior + (size_t)pidx[v] * K : NULL;
        for (uint32_t k = 0; k < K; ++k) {
            int32_t c = nkw[(size_t)v * K + k];
            if (!c) continue;
            if (pe) ll += lgamma((double)c + (double)pe[k]) - lgamma((double)pe[k]);
            else ll += lgamma((double)c + e) - lge;
        }
    }
    return ll;
}

/* per-document infer with word priors: z0 from the word's column, R_k =
 * 1 / ((float)(n_k + n_dk) + esum_k), B_k = (float)(n_kw + own) + eta_kv */
double orc_infer_doc_p(uint32_t K, uint32_t V, const float* alpha, float eta,
                       const int32_t* pidx, const float* prior, const float* esum,
                       const int32_t* nkw, const int32_t* nk,
                       const uint32_t* words, uint32_t len, uint32_t iters,
                       uint64_t seed, uint64_t doc_key, uint16_t* z, int32_t* ndk, float* theta)
{
    uint64_t key = seed ^ (uint64_t)ORC_STREAM_INFER;
    uint32_t klo = (uint32_t)doc_key, khi = (uint32_t)(doc_key >> 32);
    int32_t* own = (int32_t*)calloc(K, sizeof(int32_t));
    float* A = (float*)malloc(K * sizeof(float));
    float* BR = (float*)malloc(K * sizeof(float));
    float* cum = (float*)malloc(K * sizeof(float));
    memset(ndk, 0, K * sizeof(int32_t));
    for (uint32_t j = 0; j < len; ++j) {
        uint32_t v = words[j];
        if (v >= V) { z[j] = 0xFFFF; continue; }
        column_cum(K, pidx[v] >= 0 ? prior + (size_t)pidx[v] * K : NULL, eta, cum);
        float u = orc_u01(philox_first(j, 0xFFFFFFFFu, klo, khi, key));
        uint16_t k = (uint16_t)orc_sample_acc(cum, K, u);
        z[j] = k;
        ndk[k]++;
    }
    for (uint32_t it = 0; it < iters; ++it) {
        uint32_t rb = 0;
        while (rb < len) {
            uint32_t re = rb + 1;
            while (re < len && words[re] == words[rb]) ++re;
            uint32_t v = words[rb];
            if (v < V) {
                const float* pe = pidx[v] >= 0 ? prior + (size_t)pidx[v] * K : NULL;
                for (uint32_t j = rb; j < re; ++j) own[z[j]]++;
                const int32_t* g = nkw + (size_t)v * K;
                for (uint32_t j = rb; j < re; ++j) {
                    uint16_t zo = z[j];
                    own[zo]--;
                    ndk[zo]--;
                    for (uint32_t k = 0; k < K; ++k) {
                        A[k] = (float)ndk[k] + alpha[k];
                        float B = (float)(g[k] + own[k]) + (pe ? pe[k] : eta);
                        float R = 1.0f / ((float)(nk[k] + ndk[k]) + esum[k]);
                        BR[k] = B * R;
                    }
                    float u = orc_u01(philox_first(j, it, klo, khi, key));
                    uint16_t zn = (uint16_t)blocked_draw(A, BR, K, 0xFFFFFFFFu, 0.f, u);
                    z[j] = zn;
                    ndk[zn]++;
                    own[zn]++;
                }
                for (uint32_t j = rb; j < re; ++j) own[z[j]]--;
            }
            rb = re;
        }
    }
    double e = (double)eta, ll = 0, as = 0;
    float asf = 0.f;
    uint32_t n = 0;
    for (uint32_t k = 0; k < K; ++k) { as += (double)alpha[k]; asf = asf + alpha[k]; }
    for (uint32_t j = 0; j < len; ++j) n += words[j] < V;
    for (uint32_t k = 0; k < K; ++k) {
        if (!ndk[k]) continue;
        double es = (double)esum[k];
        ll += lgamma((double)nk[k] + es) - lgamma((double)(nk[k] + ndk[k]) + es);
        ll += lgamma((double)ndk[k] + alpha[k]) - lgamma((double)alpha[k]);
    }
    ll -= lgamma((double)n + as) - lgamma(as);
    uint32_t rb = 0;
    while (rb < len) {
        uint32_t re = rb + 1;
        while (re < len && words[re] == words[rb]) ++re;
        uint32_t v = words[rb];
        if (v < V) {
            const int32_t* g = nkw + (size_t)v * K;
            const float* pe = pidx[v] >= 0 ? prior + (size_t)pidx[v] * K : NULL;
            for (uint32_t j = rb; j < re; ++j) own[z[j]]++;
            for (uint32_t j = rb; j < re; ++j) {
                uint32_t k = z[j];
                int32_t c = own[k];
                if (!c) continue;
                double ek = pe ? (double)pe[k] : e;
                double after = lgamma((double)(g[k] + c) + ek);
                double before = g[k] ? lgamma((double)g[k] + ek) : lgamma(ek);
                ll += after - before;
                own[k] = 0;
            }
        }
        rb = re;
    }
    if (theta)
        for (uint32_t k = 0; k < K; ++k) theta[k] = ((float)ndk[k] + alpha[k]) / ((float)n + asf);
    free(own); free(A); free(BR); free(cum);
    return ll;
}

/* ------------------------------------------------------------------------ */
/* Per-document topic masks and alphas: the derived models' conditionals    */
/* ------------------------------------------------------------------------ */
/* LLDA / PLDA multiply the conditional by the document's label mask
 * (LLDAModel.hpp:37-48, PLDAModel.hpp:39); DMR replaces alpha by the
 * document's alpha (getCachedAlpha, DMRModel.hpp:193-206).  Device
 * semantics: A_k = ((float)n_dk + alpha_dk) * m_dk with m_dk in {0, 1}; a
 * masked topic's weight is exactly 0 and an unmasked one's is unchanged.
 * mask: D rows of ceil(K/32) words (bit k of row d), NULL = all topics;
 * arow: D indices into alpha_rows (M x K), NULL = the model's alpha. */
static inline float mask_bit(const uint32_t* mask, uint32_t mw, uint64_t d, uint32_t k)
{
    return mask ? (float)((mask[d * mw + (k >> 5)] >> (k & 31)) & 1u) : 1.f;
}

void orc_sweep_doc_live_m_subset(uint32_t K, uint32_t V, const float* alpha, const float* alpha_rows,
                                 const uint32_t* arow, const uint32_t* mask, float eta,
                                 uint64_t seed, uint32_t iter, const uint64_t* doc_off,
                                 const uint32_t* words, int32_t* ndk,
                                 const int32_t* nkw, const int32_t* nk,
                                 int32_t* nkw_next, int32_t* nk_next, uint16_t* z,
                                 const uint64_t* docs, uint64_t n_docs)
{
    float veta = eta * (float)V;
    uint32_t mw = (K + 31) / 32;
    float* R = (float*)malloc(K * sizeof(float));
    float* A = (float*)malloc(K * sizeof(float));
    float* phi = (float*)malloc(K * sizeof(float));
    for (uint32_t k = 0; k < K; ++k) R[k] = 1.0f / ((float)nk[k] + veta);
    for (uint64_t di = 0; di < n_docs; ++di) {
        uint64_t d = docs ? docs[di] : di;
        const float* al = arow ? alpha_rows + (size_t)arow[d] * K : alpha;
        int32_t* row = ndk + d * K;
        for (uint32_t k = 0; k < K; ++k) A[k] = ((float)row[k] + al[k]) * mask_bit(mask, mw, d, k);
        for (uint64_t i = doc_off[d]; i < doc_off[d + 1]; ++i) {
            uint32_t v = words[i];
            if (v >= V) continue;
            uint16_t zo = z[i];
            const int32_t* col = nkw + (size_t)v * K;
            row[zo]--;
            A[zo] = ((float)row[zo] + al[zo]) * mask_bit(mask, mw, d, zo);
            for (uint32_t k = 0; k < K; ++k) phi[k] = ((float)col[k] + eta) * R[k];
            float phi_own = ((float)(col[zo] - 1) + eta) * (1.0f / ((float)(nk[zo] - 1) + veta));
            float u = orc_u01(philox_first((uint32_t)i, (uint32_t)(i >> 32), ORC_STREAM_SWEEP, iter, seed));
            uint16_t zn = (uint16_t)blocked_draw(A, phi, K, zo, phi_own, u);
            row[zn]++;
            A[zn] = ((float)row[zn] + al[zn]) * mask_bit(mask, mw, d, zn);
            z[i] = zn;
            if (zn != zo) {
                nkw_next[(size_t)v * K + zo]--; nkw_next[(size_t)v * K + zn]++;
                nk_next[zo]--; nk_next[zn]++;
            }
        }
    }
    free(R); free(A); free(phi);
}

/* getLLDocs with per-document alphas (DMR's getLLDocTopic, DMRModel.hpp:208-224), FP64 */
double orc_ll_docs_m_f64(uint64_t D, uint32_t K, const int32_t* ndk, const int32_t* doc_len,
                         const float* alpha_rows, const uint32_t* arow)
{
    double ll = 0;
    for (uint64_t d = 0; d < D; ++d) {
        const float* al = alpha_rows + (size_t)arow[d] * K;
        double as = 0, s = 0;
        for (uint32_t k = 0; k < K; ++k) as += (double)al[k];
        for (uint32_t k = 0; k < K; ++k) {
            int32_t c = ndk[d * K + k];
            if (!c) continue;
            s += lgamma((double)c + (double)al[k]) - lgamma((double)al[k]);
        }
        ll += s - (lgamma((double)doc_len[d] + as) - lgamma(as));
    }
    return ll;
}

/* ------------------------------------------------------------------------ */
/* The reference's sequential sampler (ParallelScheme::NONE) with weighted    */
/* counts or word priors: the statistical gate for those paths               */
/* ------------------------------------------------------------------------ */
/* Weighted: addWordTo with float weights, decrements clamped at 0
 * (LDAModel.hpp:287-299, Utils.hpp:132-155); the conditional of
 * getZLikelihoods (:273-285) in tomotopy's (A*B)/C order. */
void orc_gibbs_none_w(uint64_t D, const uint64_t* doc_off, const uint32_t* words, const float* wt,
                      uint32_t V, uint32_t K, const float* alpha, float eta,
                      uint16_t* z, float* ndk, float* nkw, float* nk, uint64_t* rng_state)
{
    float veta = eta * (float)V;
    float* dist = (float*)malloc(K * sizeof(float));
    uint64_t* order = (uint64_t*)malloc((D + 1) * sizeof(uint64_t));
    orc_shuffled_order(D, (size_t)(splitmix64(rng_state) & 0xFFFFFFFFu), order);
    for (uint64_t j = 0; j < D; ++j) {
        uint64_t d = order[j];
        float* row = ndk + d * K;
        for (uint64_t i = doc_off[d]; i < doc_off[d + 1]; ++i) {
            uint32_t v = words[i];
            if (v >= V) continue;
            float w = wt[i];
            uint16_t k0 = z[i];
            float* col = nkw + (size_t)v * K;
            row[k0] = fmaxf(row[k0] - w, 0.f);
            nk[k0] = fmaxf(nk[k0] - w, 0.f);
            col[k0] = fmaxf(col[k0] - w, 0.f);
            for (uint32_t k = 0; k < K; ++k) dist[k] = (row[k] + alpha[k]) * (col[k] + eta) / (nk[k] + veta);
            orc_prefix_sum_sse(dist, (int)K);
            uint16_t k1 = (uint16_t)orc_sample_acc(dist, K, sm_u01(rng_state));
            z[i] = k1;
            row[k1] += w; nk[k1] += w; col[k1] += w;
        }
    }
    free(dist); free(order);
}

/* Word priors: getZLikelihoods<true> with etaByTopicWord / etaSumByTopic. */
void orc_gibbs_none_p(uint64_t D, const uint64_t* doc_off, const uint32_t* words,
                      uint32_t V, uint32_t K, const float* alpha, float eta,
                      const int32_t* pidx, const float* prior, const float* esum,
                      uint16_t* z, int32_t* ndk, int32_t* nkw, int32_t* nk, uint64_t* rng_state)
{
    float* dist = (float*)malloc(K * sizeof(float));
    uint64_t* order = (uint64_t*)malloc((D + 1) * sizeof(uint64_t));
    orc_shuffled_order(D, (size_t)(splitmix64(rng_state) & 0xFFFFFFFFu), order);
    for (uint64_t j = 0; j < D; ++j) {
        uint64_t d = order[j];
        int32_t* row = ndk + d * K;
        for (uint64_t i = doc_off[d]; i < doc_off[d + 1]; ++i) {
            uint32_t v = words[i];
            if (v >= V) continue;
            uint16_t k0 = z[i];
            int32_t* col = nkw + (size_t)v * K;
            const float* pe = pidx[v] >= 0 ? prior + (size_t)pidx[v] * K : NULL;
            row[k0]--; nk[k0]--; col[k0]--;
            for (uint32_t k = 0; k < K; ++k)
                dist[k] = ((float)row[k] + alpha[k]) * ((float)col[k] + (pe ? pe[k] : eta)) / ((float)nk[k] + esum[k]);
            orc_prefix_sum_sse(dist, (int)K);
            uint16_t k1 = (uint16_t)orc_sample_acc(dist, K, sm_u01(rng_state));
            z[i] = k1;
            row[k1]++; nk[k1]++; col[k1]++;
        }
    }
    free(dist); free(order);
}


/* ------------------------------------------------------------------------ */
/* The benchmark workload, without the engine: the seeded synthetic corpus  */
/* and its preparation, for the timed CPU baseline                          */
/* ------------------------------------------------------------------------ */
/* The generator of tomotopy_b200/csrc/synth.cpp restated (the workload of
 * both bench arms, so the CPU arm needs no engine code): Philox4x32-10
 * streams keyed by seed ^ 0x5EEDC0DE5EEDC0DE with counters (owner a, owner b,
 * 'SYNT', draw index); lengths Poisson (a sum of pieces of mean <= 50, Knuth)
 * or round(lognormal) clipped; topic-word distributions Dirichlet(beta V
 * Zipf(s)) drawn as log-Gamma (Marsaglia-Tsang, the a < 1 boost in log
 * space), words 40 nats below a topic's top word dropped, Vose alias tables;
 * tokens by the Polya urn of Dirichlet(doc_alpha * 1_T).  Identical output
 * for any thread count. */
typedef struct { uint64_t key; uint32_t a, b, n, buf[4]; int left; } syn_rng;

static void syn_init(syn_rng* r, uint64_t seed, uint32_t a, uint32_t b)
{
    r->key = seed ^ 0x5EEDC0DE5EEDC0DEull; r->a = a; r->b = b; r->n = 0; r->left = 0;
}
static uint32_t syn_next(syn_rng* r)
{
    if (!r->left) {
        uint32_t ctr[4] = { r->a, r->b, 0x53594E54u, r->n++ }, key[2] = { (uint32_t)r->key, (uint32_t)(r->key >> 32) };
        orc_philox4x32_10(ctr, key, r->buf);
        r->left = 4;
    }
    return r->buf[--r->left];
}
static double syn_uniform(syn_rng* r)      /* (0, 1], 53 bits */
{
    uint64_t hi = syn_next(r), lo = syn_next(r);
    uint64_t m = ((hi << 32) | lo) >> 11;
    return ((double)m + 1.0) * (1.0 / 9007199254740992.0);
}
static double syn_normal(syn_rng* r)
{
    double u1 = syn_uniform(r), u2 = syn_uniform(r);
    return sqrt(-2.0 * log(u1)) * cos(6.283185307179586 * u2);
}
static double syn_log_gamma(syn_rng* r, double a)
{
    double boost = 0.0;
    if (a < 1.0) { boost = log(syn_uniform(r)) / a; a += 1.0; }
    const double d = a - 1.0 / 3.0, c = 1.0 / sqrt(9.0 * d);
    for (;;) {
        double x = syn_normal(r), v = 1.0 + c * x;
        if (v <= 0) continue;
        v = v * v * v;
        double u = syn_uniform(r);
        if (log(u) < 0.5 * x * x + d - d * v + d * log(v)) return log(d * v) + boost;
    }
}
static uint32_t syn_poisson_small(syn_rng* r, double lam)
{
    double L = exp(-lam), p = 1.0;
    uint32_t k = 0;
    do { ++k; p *= syn_uniform(r); } while (p > L);
    return k - 1;
}

typedef struct { uint32_t n; uint32_t* word; float* prob; uint32_t* alias; } syn_alias;

/* Vose's alias method with the generator's stack order */
static void syn_build_alias(const double* p, const uint32_t* ids, uint32_t n, syn_alias* out)
{
    out->n = n;
    out->word = (uint32_t*)malloc((n + 1) * sizeof(uint32_t));
    out->prob = (float*)calloc(n + 1, sizeof(float));
    out->alias = (uint32_t*)calloc(n + 1, sizeof(uint32_t));
    memcpy(out->word, ids, n * sizeof(uint32_t));
    double s = 0;
    for (uint32_t i = 0; i < n; ++i) s += p[i];
    double* q = (double*)malloc((n + 1) * sizeof(double));
    uint32_t* small = (uint32_t*)malloc((n + 1) * sizeof(uint32_t));
    uint32_t* large = (uint32_t*)malloc((n + 1) * sizeof(uint32_t));
    uint32_t ns = 0, nl = 0;
    for (uint32_t i = 0; i < n; ++i) {
        q[i] = p[i] / s * (double)n;
        if (q[i] < 1.0) small[ns++] = i; else large[nl++] = i;
    }
    while (ns && nl) {
        uint32_t l = small[--ns], g = large[--nl];
        out->prob[l] = (float)q[l];
        out->alias[l] = g;
        q[g] = (q[g] + q[l]) - 1.0;
        if (q[g] < 1.0) small[ns++] = g; else large[nl++] = g;
    }
    for (uint32_t i = 0; i < nl; ++i) { out->prob[large[i]] = 1.f; out->alias[large[i]] = large[i]; }
    for (uint32_t i = 0; i < ns; ++i) { out->prob[small[i]] = 1.f; out->alias[small[i]] = small[i]; }
    free(q); free(small); free(large);
}

typedef struct {
    const orc_synth_spec* s; uint64_t b, e; int phase;
    uint32_t* len; const uint64_t* doc_off; uint32_t* words;
    const double* zipf; double zs; syn_alias* topics;
} syn_job;

static uint32_t syn_doc_length(const orc_synth_spec* s, syn_rng* r)
{
    double L;
    if (s->len_kind == 0) {
        double lam = s->len_a, acc = 0;
        uint32_t m = (uint32_t)ceil(lam / 50.0);
        if (m < 1) m = 1;
        for (uint32_t i = 0; i < m; ++i) acc += syn_poisson_small(r, lam / m);
        L = acc;
    } else {
        L = floor(exp(s->len_a + s->len_b * syn_normal(r)) + 0.5);
    }
    if (L < s->len_min) L = s->len_min;
    if (L > s->len_max) L = s->len_max;
    return (uint32_t)L;
}

static void* syn_work(void* arg)
{
    syn_job* j = (syn_job*)arg;
    const orc_synth_spec* s = j->s;
    if (j->phase == 0) {
        for (uint64_t d = j->b; d < j->e; ++d) {
            const uint64_t dd = d + s->doc_offset;
            syn_rng r;
            syn_init(&r, s->seed, (uint32_t)dd, 0x4C454E00u | (uint32_t)(dd >> 32));
            j->len[d] = syn_doc_length(s, &r);
        }
    } else if (j->phase == 1) {
        double* lg = (double*)malloc(s->V * sizeof(double));
        double* p = (double*)malloc(s->V * sizeof(double));
        uint32_t* ids = (uint32_t*)malloc(s->V * sizeof(uint32_t));
        for (uint64_t t = j->b; t < j->e; ++t) {
            syn_rng r;
            syn_init(&r, s->seed, (uint32_t)t, 0x50484900u);
            double mx = -INFINITY;
            for (uint32_t v = 0; v < s->V; ++v) {
                double a = s->topic_beta * (double)s->V * j->zipf[v] / j->zs;
                lg[v] = syn_log_gamma(&r, a);
                if (lg[v] > mx) mx = lg[v];
            }
            uint32_t n = 0;
            for (uint32_t v = 0; v < s->V; ++v) {
                double x = lg[v] - mx;
                if (x < -40.0) continue;
                p[n] = exp(x);
                ids[n++] = v;
            }
            syn_build_alias(p, ids, n, &j->topics[t]);
        }
        free(lg); free(p); free(ids);
    } else {
        const double conc = s->doc_alpha * (double)s->T;
        uint32_t cap = 0;
        uint32_t* zt = NULL;
        for (uint64_t d = j->b; d < j->e; ++d) {
            const uint64_t dd = d + s->doc_offset;
            syn_rng r;
            syn_init(&r, s->seed, (uint32_t)dd, 0x544F4B00u | (uint32_t)(dd >> 32));
            const uint32_t L = (uint32_t)(j->doc_off[d + 1] - j->doc_off[d]);
            if (L > cap) { free(zt); cap = L; zt = (uint32_t*)malloc(cap * sizeof(uint32_t)); }
            uint32_t* out = j->words + j->doc_off[d];
            for (uint32_t i = 0; i < L; ++i) {
                double u = syn_uniform(&r) * ((double)i + conc);
                uint32_t z;
                if (u < conc || i == 0) z = syn_next(&r) % s->T;
                else { uint32_t q = (uint32_t)(u - conc); z = zt[q < i - 1 ? q : i - 1]; }
                zt[i] = z;
                const syn_alias* A = &j->topics[z];
                uint32_t jj = (uint32_t)(((uint64_t)syn_next(&r) * A->n) >> 32);
                float f = (float)(syn_next(&r) >> 8) * (1.0f / 16777216.0f);
                out[i] = A->word[f < A->prob[jj] ? jj : A->alias[jj]];
            }
        }
        free(zt);
    }
    return NULL;
}

static void syn_parallel(syn_job* proto, uint64_t n, uint32_t threads)
{
    if (threads < 1) threads = 1;
    if (n < 64) threads = 1;
    pthread_t* th = (pthread_t*)malloc(threads * sizeof(pthread_t));
    syn_job* jobs = (syn_job*)malloc(threads * sizeof(syn_job));
    for (uint32_t i = 0; i < threads; ++i) {
        jobs[i] = *proto;
        jobs[i].b = n * i / threads;
        jobs[i].e = n * (i + 1) / threads;
        if (threads > 1) pthread_create(&th[i], NULL, syn_work, &jobs[i]);
        else syn_work(&jobs[i]);
    }
    if (threads > 1) for (uint32_t i = 0; i < threads; ++i) pthread_join(th[i], NULL);
    free(th); free(jobs);
}

int orc_synth_corpus(const orc_synth_spec* s, uint64_t* doc_off, uint32_t* words, uint64_t capacity,
                     uint64_t* n_tokens, uint32_t threads)
{
    if (!s || !doc_off || !n_tokens || !s->V || !s->T || !s->D || s->len_min > s->len_max || !s->len_max) return -1;
    uint32_t* len = (uint32_t*)malloc(s->D * sizeof(uint32_t));
    syn_job job = { s, 0, 0, 0, len, doc_off, words, NULL, 0, NULL };
    syn_parallel(&job, s->D, threads);
    doc_off[0] = 0;
    for (uint64_t d = 0; d < s->D; ++d) doc_off[d + 1] = doc_off[d] + len[d];
    free(len);
    *n_tokens = doc_off[s->D];
    if (!words) return 0;
    if (capacity < *n_tokens) return -1;
    double* zipf = (double*)malloc(s->V * sizeof(double));
    double zs = 0;
    for (uint32_t v = 0; v < s->V; ++v) { zipf[v] = pow((double)(v + 1), -s->zipf_s); zs += zipf[v]; }
    syn_alias* topics = (syn_alias*)calloc(s->T, sizeof(syn_alias));
    job.phase = 1; job.zipf = zipf; job.zs = zs; job.topics = topics;
    syn_parallel(&job, s->T, threads);
    job.phase = 2;
    syn_parallel(&job, s->D, threads);
    for (uint32_t t = 0; t < s->T; ++t) { free(topics[t].word); free(topics[t].prob); free(topics[t].alias); }
    free(topics); free(zipf);
    return 0;
}

/* removeStopwords + prepareDoc over a whole corpus (the restated functions
 * above), threaded over documents: words are renumbered in place and sorted
 * within each document; order[old id] = new id; returns realV. */
typedef struct { const uint64_t* doc_off; uint32_t* words; uint64_t b, e; uint64_t nv; uint64_t* df;
                 const uint32_t* order; int phase; } prep_job;

static void* prep_work(void* arg)
{
    prep_job* j = (prep_job*)arg;
    uint32_t* tmp = NULL; uint32_t* wo = NULL; size_t cap = 0;
    for (uint64_t d = j->b; d < j->e; ++d) {
        const uint64_t b = j->doc_off[d], n = j->doc_off[d + 1] - b;
        if (n > cap) { free(tmp); free(wo); cap = n; tmp = (uint32_t*)malloc(cap * 4); wo = (uint32_t*)malloc(cap * 4); }
        if (j->phase == 0) {          /* df: distinct words of the document */
            memcpy(tmp, j->words + b, n * 4);
            orc_sort_doc(tmp, n, wo);
            for (uint64_t i = 0; i < n; ++i)
                if (i == 0 || tmp[i] != tmp[i - 1]) j->df[tmp[i]]++;
        } else {                      /* renumber, then sort by the new ids */
            uint32_t* w = j->words + b;
            for (uint64_t i = 0; i < n; ++i) w[i] = j->order[w[i]];
            orc_sort_doc(w, n, wo);
        }
    }
    free(tmp); free(wo);
    return NULL;
}

uint64_t orc_prepare_corpus(uint64_t D, const uint64_t* doc_off, uint32_t* words, uint64_t nv,
                            uint64_t min_cf, uint64_t min_df, uint64_t rm_top, uint32_t* order, uint32_t threads)
{
    if (threads < 1) threads = 1;
    uint64_t* cf = (uint64_t*)calloc(nv + 1, sizeof(uint64_t));
    uint64_t* df = (uint64_t*)calloc(nv + 1, sizeof(uint64_t));
    for (uint64_t i = 0; i < doc_off[D]; ++i) cf[words[i]]++;
    uint64_t** dfs = (uint64_t**)malloc(threads * sizeof(uint64_t*));
    pthread_t* th = (pthread_t*)malloc(threads * sizeof(pthread_t));
    prep_job* jobs = (prep_job*)malloc(threads * sizeof(prep_job));
    for (int phase = 0; phase < 2; ++phase) {
        for (uint32_t i = 0; i < threads; ++i) {
            dfs[i] = phase == 0 ? (uint64_t*)calloc(nv + 1, sizeof(uint64_t)) : NULL;
            prep_job pj = { doc_off, words, D * i / threads, D * (i + 1) / threads, nv, dfs[i], order, phase };
            jobs[i] = pj;
            pthread_create(&th[i], NULL, prep_work, &jobs[i]);
        }
        for (uint32_t i = 0; i < threads; ++i) pthread_join(th[i], NULL);
        if (phase == 0) {
            for (uint32_t i = 0; i < threads; ++i) {
                for (uint64_t v = 0; v < nv; ++v) df[v] += dfs[i][v];
                free(dfs[i]);
            }
            uint64_t rv = orc_remove_stopwords(nv, cf, df, min_cf, min_df, rm_top, order);
            cf[nv] = rv;        /* kept for the return */
        }
    }
    const uint64_t rv = cf[nv];
    free(cf); free(df); free(dfs); free(th); free(jobs);
    return rv;
}
