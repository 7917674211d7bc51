/*
 * dmst_oracle.c -- TEST INFRASTRUCTURE ONLY (see dmst_oracle.h).
 *
 * A scalar restatement, one (read, profile) pair at a time, of the
 * reference's FP32 scoring path.  A reference batch runs up to eight pairs
 * in SIMD lanes, but a lane's result never depends on its batch mates
 * (columns past a lane's length are masked to zero and read the zero_idx pad
 * code), so one pair in isolation gives that lane's result.
 *
 * Arithmetic follows the reference operation by operation:
 *   - every float recurrence in the association order of the reference
 *     source, with the fused multiply-adds that GCC forms from it at -O3 on
 *     x86-64-v3 written out as fmaf() (this file is built with
 *     -ffp-contract=off so that no other contraction happens);
 *   - FTZ/DAZ on for the duration of each call, as the reference sets on
 *     every thread (dummest-core.hh:143-154);
 *   - the ExpScore algebra in double with the reference's rounding points
 *     (dummest-score.hh, dummest-batch.hh), and the same libm calls (frexp,
 *     ldexp, log2, exp2).
 */
#include "dmst_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#include <xmmintrin.h>

#define NCODE_PAD 24      /* zero_idx = alphabet size + 4 (dummest-dp.hh:91-95) */
#define WIDTH 29          /* floats per profile row (dummest-core.hh:231) */
#define NPARAM 11         /* floats per Params (dummest-core.hh:233-239) */
#define RESCALE_BITS 64   /* dummest-score.hh:80-84 */
#define RESCALE_THRESH 1e30f /* FP32 engine, dummest-score.hh:93 */
#define EXP2_HI 120       /* FP32 engine, dummest-score.hh:214-218 */

typedef dmsto_score xs;
static const xs XS0 = {0.0f, 0};

static _Thread_local int g_last_bwd, g_last_fwd;

void dmsto_last_rescales(int *backward, int *forward) {
    if (backward) *backward = g_last_bwd;
    if (forward) *forward = g_last_fwd;
}

/* FTZ (bit 15) and DAZ (bit 6) of MXCSR for one call. */
static unsigned ftz_enter(void) {
    unsigned old = _mm_getcsr();
    _mm_setcsr(old | 0x8040u);
    return old;
}
static void ftz_leave(unsigned old) { _mm_setcsr(old); }

/* ---------------------------------------------------------------------------
 * ExpScore algebra
 * ------------------------------------------------------------------------- */

/* normalizeScore (dummest-score.hh:59-67). */
static xs normalize(double m, int e) {
    if (m == 0.0) return XS0;
    int ex = 0;
    m = frexp(m, &ex);
    xs r = {(float)m, e + ex};
    return r;
}

/* splitNormalizedDouble (dummest-batch.hh:42-53). */
static void split_norm(double x, float *m, int *e) {
    if (x == 0.0) {
        *m = 0.0f;
        *e = 0;
        return;
    }
    uint64_t u;
    memcpy(&u, &x, sizeof u);
    const int ef = (int)((u >> 52) & 0x7FFu);
    if (ef == 0x7FF) {
        *m = (float)x;
        *e = 0;
        return;
    }
    if (ef == 0) {
        *m = 0.0f;
        *e = 0;
        return;
    }
    *e = ef - 1022;
    const uint64_t v = (u & 0xFFFFFFFFFFFFFull) | (1022ull << 52);
    double d;
    memcpy(&d, &v, sizeof d);
    *m = (float)d;
}

/* scoreLess (dummest-score.hh:70-76). */
static int score_less(xs a, xs b) {
    if (a.m == 0.0f) return b.m != 0.0f;
    if (b.m == 0.0f) return 0;
    if (a.e != b.e) return a.e < b.e;
    return a.m < b.m;
}

/* pow2Score (dummest-score.hh:197-199). */
static xs pow2s(int e2) {
    xs r = {0.5f, e2 + 1};
    return r;
}

/* scaleScore (dummest-score.hh:155-160). */
static xs scale_score(xs a, double f) {
    if (a.m == 0.0f) return XS0;
    if (!(f > 0.0) || !isfinite(f)) return XS0;
    return normalize((double)a.m * f, a.e);
}

/* One lane of batchScaleScores (dummest-batch.hh:114-130). */
static xs batch_scale(xs a, double f) {
    const int a0 = (a.m == 0.0f);
    const int fok = (f > 0.0) && isfinite(f);
    float m;
    int ex;
    split_norm(a0 ? 0.0 : (double)a.m * (fok ? f : 1.0), &m, &ex);
    if (a0 || !fok) return XS0;
    xs r = {m, a.e + ex};
    return r;
}

/* One lane of batchMulScores / batchMulScorePlanes with eFold = 0
 * (dummest-batch.hh:58-72, :216-235). */
static xs batch_mul(xs a, xs b) {
    const int nz = (a.m != 0.0f) && (b.m != 0.0f);
    double p = (double)a.m * (double)b.m;
    int e = a.e + b.e;
    if (p < 0.5) {
        p *= 2.0;
        e -= 1;
    }
    if (!nz) return XS0;
    xs r = {(float)p, e};
    return r;
}

/* One lane of batchAddScores (dummest-batch.hh:78-108). */
static xs batch_add(xs a, xs b) {
    if (a.m == 0.0f) return b;
    if (b.m == 0.0f) return a;
    const int agebe = a.e >= b.e;
    const float mh = agebe ? a.m : b.m, ml = agebe ? b.m : a.m;
    const int eh = agebe ? a.e : b.e, el = agebe ? b.e : a.e;
    int d = eh - el;
    d = d > 60 ? 60 : d;
    double s = (double)mh + (double)ml * (1.0 / (double)(1ull << (unsigned)d));
    int e = eh;
    if (s >= 1.0) {
        s *= 0.5;
        e += 1;
    }
    xs r = {(float)s, e};
    return r;
}

/* addScores (dummest-score.hh:169-181). */
static xs add_scores(xs a, xs b) {
    if (a.m == 0.0f) return b;
    if (b.m == 0.0f) return a;
    if (a.e >= b.e) {
        const int d = a.e - b.e;
        if (d > 60) return a;
        return normalize((double)a.m + ldexp((double)b.m, -d), a.e);
    }
    const int d = b.e - a.e;
    if (d > 60) return b;
    return normalize((double)b.m + ldexp((double)a.m, -d), b.e);
}

/* mulScores (dummest-score.hh:184-188). */
static xs mul_scores(xs a, xs b) {
    if (a.m == 0.0f || b.m == 0.0f) return XS0;
    return normalize((double)a.m * (double)b.m, a.e + b.e);
}

/* scoreToFloatClamped (dummest-score.hh:224-230). */
static float pack(xs a) {
    if (a.m == 0.0f) return 0.0f;
    const int e = a.e > EXP2_HI ? EXP2_HI : a.e;
    return ldexpf(a.m, e);
}

/* clampRescaleCount (dummest-score.hh:97-102). */
static int clamp_count(int c) { return c > 1000000 ? 1000000 : (c < -1000000 ? -1000000 : c); }

/* One lane of batchPromoteRescaled (dummest-batch.hh:146-213): subnormals
 * flush, then promoteRescaledScore (dummest-score.hh:107-116). */
static xs promote(float v, int cum) {
    if (fpclassify(v) == FP_SUBNORMAL) return XS0;
    if (!(v > 0.0f)) return XS0;
    cum = clamp_count(cum);
    if (!(v < INFINITY)) {
        xs r = {nextafterf(1.0f, 0.0f), 1023 + RESCALE_BITS * cum};
        return r;
    }
    return normalize((double)v, RESCALE_BITS * cum);
}

/* rowRescaleVector lane (dummest-score.hh:145-152) times the static scale 1. */
static float row_scale(int cnt) { return 1.0f * ldexpf(1.0f, -RESCALE_BITS * clamp_count(cnt)); }

/* Kokkos::max on AVX2 lanes: (a > b) ? a : b. */
static float vmax(float a, float b) { return a > b ? a : b; }

/* ---------------------------------------------------------------------------
 * Null model (dummest-dp-backward.hh:6-165)
 * ------------------------------------------------------------------------- */

typedef struct null_out {
    float *pre;  /* prefixSeed, L */
    float *suf;  /* suffixSeedFromNext, L */
    float s1, s2, sC;
} null_out;

/* bg_probs + 4 indexed by the code at column j; columns outside the read
 * hold the zero_idx pad code (buildTransposedDecoded, dummest-dp.hh:67-77). */
static float bg_at(const float *bg4, const uint8_t *codes, int L, int j) {
    return bg4[(j >= 0 && j < L) ? codes[j] : NCODE_PAD];
}

static int null_model(const float *bg, const uint8_t *codes, int L, dmsto_rates r, null_out *o) {
    const float *bg4 = bg + 4;
    xs *prefix = (xs *)calloc((size_t)L + 4, sizeof(xs));
    xs *suffix = (xs *)calloc((size_t)L + 4, sizeof(xs));
    if (!prefix || !suffix) {
        free(prefix);
        free(suffix);
        return -1;
    }
    /* buildBatchNullModels (dummest-dp-backward.hh:167-188). */
    const double sr = (double)r.single, dr = (double)r.dbl;
    const double keep = 1 - sr - dr;
    const double sNE = sr * 0.25, dNE = dr * 0.0625;
    const double frame = 1.0 / 3.0;

    /* buildNullSuffix (dummest-dp-backward.hh:6-55). */
    float tm;
    int te;
    split_norm(0.5 * keep, &tm, &te);
    suffix[L] = pow2s(0);
    for (int i = L - 1; i >= 0; --i) {
        const double codonScale = (double)bg_at(bg4, codes, L, i) * keep;
        const xs singleIn = suffix[i + 1];
        const xs doubleIn = (i + 1 < L) ? suffix[i + 2] : pow2s(2);
        const xs codonRaw = batch_scale(suffix[i + 3], codonScale);
        const xs single = batch_scale(singleIn, sNE);
        const xs dbl = batch_scale(doubleIn, dNE);
        xs codon = codonRaw;
        if (!(i + 2 < L)) {
            codon.m = tm;
            codon.e = te - 2 * (L - i) + 1;
        }
        suffix[i] = batch_add(codon, batch_add(single, dbl));
    }

    /* buildNullPrefixFirstCodon (dummest-dp-backward.hh:58-100). */
    for (int i = 0; i < L; ++i) {
        const float bgc = bg_at(bg4, codes, L, i - 2);
        const double codonScale = (double)bgc * keep;
        const xs ps = i > 0 ? prefix[i - 1] : XS0;
        const xs pd = i >= 2 ? prefix[i - 2] : XS0;
        xs codon;
        if (i >= 3)
            codon = batch_scale(prefix[i - 3], codonScale);
        else if (i == 2)
            codon = scale_score(normalize((double)bgc, 0), frame);
        else if (i == 1)
            codon = scale_score(pow2s(-4), frame);
        else
            codon = scale_score(pow2s(-2), frame);
        prefix[i] = batch_add(codon, batch_add(batch_scale(ps, sNE), batch_scale(pd, dNE)));
    }

    /* buildNullTotalAndScales (dummest-dp-backward.hh:103-129). */
    const double keepSingle = 1.0 - sr;
    const double keepBoth = keepSingle - dr;
    const xs ts = scale_score(prefix[L - 2], keepSingle * 0.25);
    const xs td = scale_score(prefix[L - 3], keepBoth * 0.0625);
    const xs total = add_scores(add_scores(prefix[L - 1], ts), td);
    const float nullLog = (float)(total.m == 0.0f ? -INFINITY : log2((double)total.m) + (double)total.e);
    double pbl = -(double)nullLog / (double)L;
    if (!(pbl < (double)EXP2_HI)) pbl = (double)EXP2_HI;
    const double raw = exp2(pbl);
    const xs perBase = normalize(raw, 0);
    const xs perBaseInv = normalize(1.0 / raw, 0);
    const xs quarter = normalize(0.25, 0), sixteenth = normalize(0.0625, 0);
    o->s1 = pack(mul_scores(perBase, quarter));
    o->s2 = pack(mul_scores(mul_scores(perBase, perBase), sixteenth));
    o->sC = pack(mul_scores(mul_scores(perBase, perBase), perBase));

    /* buildNullSeedModels (dummest-dp-backward.hh:133-165). */
    xs running = pow2s(0);
    for (int t = 0; t < L - 1; ++t) running = batch_mul(running, perBase);
    for (int j = 0; j < L; ++j) {
        o->suf[j] = pack(batch_mul(suffix[j + 1], running));
        running = batch_mul(running, perBaseInv);
    }
    running = perBase;
    for (int j = 0; j < L; ++j) {
        o->pre[j] = pack(batch_mul(prefix[j], running));
        running = batch_mul(running, perBase);
    }
    free(prefix);
    free(suffix);
    return 0;
}

int dmsto_null_model(const float *bg, const uint8_t *codes, int L, dmsto_rates r, float *prefix_seed,
                     float *suffix_seed, float *scales3) {
    if (!bg || !codes || L < 3 || !prefix_seed || !suffix_seed || !scales3) return -1;
    const unsigned csr = ftz_enter();
    null_out o = {prefix_seed, suffix_seed, 0, 0, 0};
    const int st = null_model(bg, codes, L, r, &o);
    scales3[0] = o.s1;
    scales3[1] = o.s2;
    scales3[2] = o.sC;
    ftz_leave(csr);
    return st;
}

/* ---------------------------------------------------------------------------
 * The backward recurrence of one row (dummest-dp-backward.hh:473-548 and the
 * filter's copy at :367-427).  Writes row i of W1 (`row`) from row i+1
 * (`below`), Y of row i into ycur from ynext, and returns the row maximum
 * over W1 and Y (the rescale test; the filter ignores it).
 * ------------------------------------------------------------------------- */
typedef struct pair_ctx {
    const float *values, *params, *bg4;
    const uint8_t *codes;
    int M, L;
    float s1, s2, sC;
    const float *pre, *suf;
} pair_ctx;

static int code_at(const pair_ctx *p, int j) { return (j >= 0 && j < p->L) ? p->codes[j] : NCODE_PAD; }

static float backward_row(const pair_ctx *p, int i, float rs, float *row, const float *below, float *ycur,
                          const float *ynext, float *filt_best) {
    const float *q = p->params + (size_t)i * NPARAM;
    const float *erow = p->values + (size_t)i * WIDTH + 4;
    const int L = p->L;
    const float enter = q[10] * p->sC, d0 = q[6], d1 = q[7] * p->s2, d2 = q[8] * p->s1;
    const float a0 = q[0] * p->sC, a1 = q[1] * p->s1, a2 = q[2] * p->s2, b0 = q[3] * p->sC, eps = q[9];
    float z[4] = {0.0f, 0.0f, 0.0f, 0.0f};
    float nJ3 = below[L + 2], nJ2 = below[L + 1], nJ1 = below[L];
    float cJ2 = row[L + 1], cJ1 = row[L];
    float rowMax = 0.0f;
    for (int j = L - 1; j >= 0; --j) {
        const float e = erow[code_at(p, j + 1)];
        const float bgv = p->bg4[code_at(p, j + 1)];
        const float nAt = below[j];
        float acc = (nJ3 * e) * enter;
        acc = fmaf(ynext[j], d0, acc);
        acc = fmaf(nJ2, d1, acc);
        acc = fmaf(nJ1, d2, acc);
        const float zbg = z[(j + 3) & 3] * bgv;
        acc = fmaf(zbg, a0, acc);
        acc = fmaf(cJ2, a2, acc);
        acc = fmaf(cJ1, a1, acc);
        const float wv = fmaf(p->suf[j], rs, acc);
        row[j] = wv;
        if (filt_best) *filt_best = vmax(*filt_best, wv * p->pre[j]);
        rowMax = vmax(rowMax, wv);
        ycur[j] = fmaf(eps, ynext[j], wv);
        rowMax = vmax(rowMax, ycur[j]);
        z[j & 3] = fmaf(b0, zbg, wv);
        nJ3 = nJ2;
        nJ2 = nJ1;
        nJ1 = nAt;
        cJ2 = cJ1;
        cJ1 = wv;
    }
    return rowMax;
}

static void scale_range(float *v, int n, float f) {
    for (int k = 0; k < n; ++k) v[k] *= f;
}

static int setup_pair(pair_ctx *p, const float *values, const float *params, const float *bg, int M,
                      const uint8_t *codes, int L, dmsto_rates r, float **seeds) {
    p->values = values;
    p->params = params;
    p->bg4 = bg + 4;
    p->codes = codes;
    p->M = M;
    p->L = L;
    float *s = (float *)calloc(2 * (size_t)L + 8, sizeof(float));
    if (!s) return -1;
    null_out o = {s, s + L + 4, 0, 0, 0};
    if (null_model(bg, codes, L, r, &o)) {
        free(s);
        return -1;
    }
    p->pre = o.pre;
    p->suf = o.suf;
    p->s1 = o.s1;
    p->s2 = o.s2;
    p->sC = o.sC;
    *seeds = s;
    return 0;
}

/* backwardPass rows M..0 (dummest-dp-backward.hh:473-574) into W1
 * ((M+2) x (L+4), zeroed by the caller: row M+1 and columns L..L+3 stay zero
 * as setupBatch leaves them, :271-276) with the per-row rescale counts.
 * Returns the sum of the counts. */
static int backward_full(const pair_ctx *p, float *W1, int *cntB, float *ybuf) {
    const size_t W = (size_t)p->L + 4;
    const float step = ldexpf(1.0f, -RESCALE_BITS);
    float *ynext = ybuf, *ycur = ybuf + W;
    int sum = 0;
    cntB[p->M + 1] = 0;
    for (int i = p->M; i >= 0; --i) {
        cntB[i] = cntB[i + 1];
        float *row = W1 + (size_t)i * W;
        const float rowMax = backward_row(p, i, row_scale(cntB[i]), row, row + W, ycur, ynext, NULL);
        float *t = ycur;
        ycur = ynext;
        ynext = t;
        if (rowMax > RESCALE_THRESH) {
            cntB[i]++;
            scale_range(row, (int)W, step);
            scale_range(ynext, (int)W, step);
            scale_range(ycur, (int)W, step);
        }
        sum += cntB[i];
    }
    return sum;
}

int dmsto_backward_matrix(const float *values, const float *params, const float *bg, int M, const uint8_t *codes,
                          int L, dmsto_rates r, float *w1_out, int *counts) {
    if (!values || !params || !bg || !codes || M < 1 || L < 3 || !w1_out || !counts) return -1;
    const unsigned csr = ftz_enter();
    pair_ctx p;
    float *seeds = NULL;
    const size_t W = (size_t)L + 4;
    float *W1 = (float *)calloc((size_t)(M + 2) * W, sizeof(float));
    float *ybuf = (float *)calloc(2 * W, sizeof(float));
    int *cntB = (int *)calloc((size_t)M + 2, sizeof(int));
    int st = -1;
    if (W1 && ybuf && cntB && !setup_pair(&p, values, params, bg, M, codes, L, r, &seeds)) {
        backward_full(&p, W1, cntB, ybuf);
        for (int i = 0; i <= M; ++i) {
            memcpy(w1_out + (size_t)i * L, W1 + (size_t)i * W, (size_t)L * sizeof(float));
            counts[i] = cntB[i];
        }
        st = 0;
    }
    free(W1);
    free(ybuf);
    free(cntB);
    free(seeds);
    ftz_leave(csr);
    return st;
}

/* findSimilarities' scores, and (colBest/colRow non-NULL) the per-column
 * anchors of its hit path: for each column j the largest wMid over the rows
 * and its row, rows in ascending order with a strict comparison, so the
 * first row wins ties (dummest-dp-forward.hh:196-206). */
static int score_pair_impl(const float *values, const float *params, const float *bg, int M, const uint8_t *codes,
                           int L, dmsto_rates r, dmsto_score *mid, dmsto_score *filter, dmsto_score *colBest,
                           int *colRow) {
    if (!values || !params || !bg || !codes || M < 1 || L < 3 || !mid || !filter) return -1;
    if (colBest)
        for (int j = 0; j < L; ++j) {
            colBest[j] = XS0;
            colRow[j] = 0;
        }
    const unsigned csr = ftz_enter();
    pair_ctx p;
    float *seeds = NULL;
    const size_t W = (size_t)L + 4;
    float *W1 = (float *)calloc((size_t)(M + 2) * W, sizeof(float));
    float *ybuf = (float *)calloc(4 * W, sizeof(float));
    int *cntB = (int *)calloc((size_t)M + 2, sizeof(int));
    int *cntF = (int *)calloc((size_t)M + 2, sizeof(int));
    int st = -1;
    if (!W1 || !ybuf || !cntB || !cntF || setup_pair(&p, values, params, bg, M, codes, L, r, &seeds)) goto done;
    {
        const float step = ldexpf(1.0f, -RESCALE_BITS);
        const int sumB = backward_full(&p, W1, cntB, ybuf);
        /* bestOut: exact max over promote(W1, cnt) * prefixSeed, columns
         * outer, rows M..0 inner (dummest-dp-backward.hh:579-609). */
        xs bestFilt = XS0;
        for (int j = 0; j < L; ++j) {
            const double nd = (double)p.pre[j];
            for (int i = M; i >= 0; --i) {
                const xs cand = batch_scale(promote(W1[(size_t)i * W + j], cntB[i]), nd);
                if (score_less(bestFilt, cand)) bestFilt = cand;
            }
        }

        /* forwardPass rows 0..M (dummest-dp-forward.hh:63-250) with the mid
         * score max over promote(W0, cntF) * promote(W1, cntB). */
        memset(ybuf, 0, 4 * W * sizeof(float));
        float *ynext = ybuf, *ycur = ybuf + W;
        float *w0cur = ybuf + 2 * W, *w0nxt = ybuf + 3 * W;
        xs best = XS0;
        int sumF = 0;
        for (int i = 0; i <= M; ++i) {
            if (i > 0) cntF[i] = cntF[i - 1];
            const float *q = params + (size_t)i * NPARAM;
            const float *erow = values + (size_t)i * WIDTH + 4;
            const float enter = q[10] * p.sC, a0 = q[0], a1 = q[1] * p.s1, a2 = q[2] * p.s2, b0 = q[3];
            const float d0 = q[6], d1 = q[7] * p.s2, d2 = q[8] * p.s1, eps = q[9];
            const float rs = row_scale(cntF[i]);
            const float *w1row = W1 + (size_t)i * W;
            float z0[4] = {0.0f, 0.0f, 0.0f, 0.0f};
            float ws0 = 0.0f, ws1 = 0.0f, ws2 = 0.0f;
            float rowMax = 0.0f;
            for (int j = 0; j < L; ++j) {
                const float w1 = ws0, w2 = ws1, w3 = ws2;
                const int c = code_at(&p, j - 2);
                const float X = (enter * erow[c]) * w3;
                /* GCC forms these at -O3 (its widening_mul dump of the
                 * reference): Z0 = (bg*sC) * fma(b0, Z0[j-3], a0*w3); the Z1/Z2
                 * ring stores are dead, so their products fuse into the sum:
                 * w0 = W0in + fma(pre, rs, fma(a2, w2, fma(a1, w1, Z0))). */
                const float Z0 = (p.bg4[c] * p.sC) * fmaf(b0, z0[(j - 3) & 3], a0 * w3);
                z0[j & 3] = Z0;
                const float w0 = w0cur[j] + fmaf(p.pre[j], rs, fmaf(a2, w2, fmaf(a1, w1, Z0)));
                rowMax = vmax(rowMax, w0);
                const xs wm = batch_mul(promote(w0, cntF[i]), promote(w1row[j], cntB[i]));
                if (score_less(best, wm)) best = wm;
                if (colBest && score_less(colBest[j], wm)) {
                    colBest[j] = wm;
                    colRow[j] = i;
                }
                w0cur[j] = w0;
                ws2 = ws1;
                ws1 = ws0;
                ws0 = w0;
                ycur[j] = fmaf(eps, ynext[j], d0 * w0);
                rowMax = vmax(rowMax, ycur[j]);
                if (i < M) w0nxt[j] = w0nxt[j] + fmaf(d2, w1, fmaf(d1, w2, X + ycur[j]));
            }
            if (rowMax > RESCALE_THRESH) {
                cntF[i]++;
                if (i < M) scale_range(w0nxt, (int)W, step);
                scale_range(ynext, (int)W, step);
                scale_range(ycur, (int)W, step);
            }
            sumF += cntF[i];
            float *t = ycur;
            ycur = ynext;
            ynext = t;
            t = w0cur;
            w0cur = w0nxt;
            w0nxt = t;
            memset(w0nxt, 0, W * sizeof(float));
        }
        *mid = best;
        *filter = bestFilt;
        g_last_bwd = sumB;
        g_last_fwd = sumF;
        st = 0;
    }
done:
    free(W1);
    free(ybuf);
    free(cntB);
    free(cntF);
    free(seeds);
    ftz_leave(csr);
    return st;
}

int dmsto_score_pair(const float *values, const float *params, const float *bg, int M, const uint8_t *codes, int L,
                     dmsto_rates r, dmsto_score *mid, dmsto_score *filter) {
    return score_pair_impl(values, params, bg, M, codes, L, r, mid, filter, NULL, NULL);
}

int dmsto_anchors(const float *values, const float *params, const float *bg, int M, const uint8_t *codes, int L,
                  dmsto_rates r, dmsto_score *colBest, int *colRow) {
    if (!colBest || !colRow) return -1;
    dmsto_score mid, filter;
    return score_pair_impl(values, params, bg, M, codes, L, r, &mid, &filter, colBest, colRow);
}

int dmsto_filter_pair(const float *values, const float *params, const float *bg, int M, const uint8_t *codes, int L,
                      dmsto_rates r, float *best) {
    if (!values || !params || !bg || !codes || M < 1 || L < 3 || !best) return -1;
    const unsigned csr = ftz_enter();
    pair_ctx p;
    float *seeds = NULL;
    const size_t W = (size_t)L + 4;
    float *buf = (float *)calloc(4 * W, sizeof(float));
    int st = -1;
    if (buf && !setup_pair(&p, values, params, bg, M, codes, L, r, &seeds)) {
        /* Two rolling W1 rows and two Y rows, no rescaling, static scale 1
         * (dummest-dp-backward.hh:345-427). */
        float *rows[2] = {buf, buf + W};
        float *ynext = buf + 2 * W, *ycur = buf + 3 * W;
        float b = 0.0f;
        for (int i = M; i >= 0; --i) {
            backward_row(&p, i, 1.0f, rows[i & 1], rows[(i + 1) & 1], ycur, ynext, &b);
            float *t = ycur;
            ycur = ynext;
            ynext = t;
        }
        *best = b;
        st = 0;
    }
    free(buf);
    free(seeds);
    ftz_leave(csr);
    return st;
}

/* ---------------------------------------------------------------------------
 * log T in FP64 (the finite-difference oracle of the library's gradient): T
 * is the total weight of all local alignments of the read, the sum over cells
 * of prefixSeed[j] * W1[i][j], W1 the backward recurrence
 * (dummest-dp-backward.hh:473-574) evaluated in double on double-precision
 * profile values (values: (M+1) x 29, params: (M+2) x 11).  The null model is
 * the reference's, computed from the float background (it is held fixed).
 * Rows are scaled by 2^-512 when their maximum passes 2^512 (exact powers of
 * two), and T is summed as a mantissa with a binary exponent.
 * ------------------------------------------------------------------------- */
int dmsto_log_total(const double *values, const double *params, const float *bg, int M, const uint8_t *codes,
                    int L, dmsto_rates r, double *logT) {
    if (!values || !params || !bg || !codes || M < 1 || L < 3 || !logT) return -1;
    const unsigned csr = ftz_enter();
    float *seeds = (float *)calloc(2 * (size_t)L + 8, sizeof(float));
    const size_t W = (size_t)L + 4;
    double *rows = (double *)calloc(4 * W, sizeof(double));
    int st = -1;
    null_out o = {seeds, seeds + L + 4, 0, 0, 0};
    if (seeds && rows && !null_model(bg, codes, L, r, &o)) {
        const double s1 = o.s1, s2 = o.s2, sC = o.sC;
        const float *bg4 = bg + 4;
        double *below = rows, *row = rows + W, *ynext = rows + 2 * W, *ycur = rows + 3 * W;
        int cnt = 0;
        double tm = 0.0;  /* T = tm * 2^te */
        int te = 0;
        for (int i = M; i >= 0; --i) {
            const double *q = params + (size_t)i * NPARAM;
            const double *erow = values + (size_t)i * WIDTH + 4;
            const double enter = q[10] * sC, d0 = q[6], d1 = q[7] * s2, d2 = q[8] * s1;
            const double a0 = q[0] * sC, a1 = q[1] * s1, a2 = q[2] * s2, b0 = q[3] * sC, eps = q[9];
            double z[4] = {0, 0, 0, 0};
            double n3 = below[L + 2], n2 = below[L + 1], n1 = below[L], c2 = 0, c1 = 0;
            double mx = 0, part = 0;
            for (int j = L; j < L + 4; ++j) row[j] = 0;
            for (int j = L - 1; j >= 0; --j) {
                const int c = (j + 1 < L) ? codes[j + 1] : NCODE_PAD;
                const double zbg = z[(j + 3) & 3] * (double)bg4[c];
                const double w = n3 * erow[c] * enter + ynext[j] * d0 + n2 * d1 + n1 * d2 + zbg * a0 + c2 * a2 +
                                 c1 * a1 + ldexp((double)o.suf[j], -512 * cnt);
                row[j] = w;
                ycur[j] = eps * ynext[j] + w;
                z[j & 3] = b0 * zbg + w;
                part += (double)o.pre[j] * w;
                if (ycur[j] > mx) mx = ycur[j];
                n3 = n2; n2 = n1; n1 = below[j];
                c2 = c1; c1 = w;
            }
            /* add part * 2^(512 cnt) to T */
            if (part > 0) {
                int pe;
                const double pm = frexp(part, &pe);
                pe += 512 * cnt;
                if (tm == 0 || pe > te + 60) {
                    tm = pm;
                    te = pe;
                } else if (pe >= te - 60) {
                    int e2;
                    tm = frexp(tm + ldexp(pm, pe - te), &e2);  /* keep tm in [0.5, 1) */
                    te += e2;
                }
            }
            if (mx > 0x1p512) {  /* this row and the Y rows the next one reads */
                ++cnt;
                for (size_t k = 0; k < W; ++k) {
                    row[k] = ldexp(row[k], -512);
                    ycur[k] = ldexp(ycur[k], -512);
                }
            }
            double *t = below;
            below = row;
            row = t;
            t = ynext;
            ynext = ycur;
            ycur = t;
        }
        *logT = tm > 0 ? log(tm) + te * 0.6931471805599453 : -INFINITY;
        st = 0;
    }
    free(seeds);
    free(rows);
    ftz_leave(csr);
    return st;
}

/* ---------------------------------------------------------------------------
 * Posterior tables in FP64.  The forward recurrence (dummest-dp-forward.hh:
 * 63-250) and the backward one (dummest-dp-backward.hh:473-574) evaluated in
 * double on double profile arrays, without anchoring:
 *   forward, row i:  W0in[i][j] = X(i-1,j) + Y0[i-1][j] + d'1 s2 W0[i-1][j-2] + d'2 s1 W0[i-1][j-1],
 *                    X(i,j) = enter_i sC e_i(c_{j-2}) W0[i][j-3],
 *                    Z0[j] = bg[j-2] sC (a'0 W0[i][j-3] + b'0 Z0[j-3]),
 *                    W0[i][j] = W0in + Z0 + a'1 s1 W0[i][j-1] + a'2 s2 W0[i][j-2] + pre[j],
 *                    Y0[i][j] = d'0 W0[i][j] + eps' Y0[i-1][j];
 *   backward:        as dmsto_log_total.
 * Each row is held at its own power-of-two offset (the exponent of the
 * maximum of the row it reads from), so values far below a row's maximum
 * flush to zero as in the reference's per-row rescaling, in double range.
 * Outputs (each (M+1) x L, row-major): cell[i][j] = W0[i][j] W1[i][j] / T and
 * match[i][j] = X(i,j) W1[i+1][j] / T (the match-state posterior of the
 * combined table, dummest-dp-forward.hh:125-157); log T from the forward
 * total sum W0 suf and, as a self-check, from the backward total sum pre W1.
 * ------------------------------------------------------------------------- */
typedef struct { double m; int e; } dx;  /* m * 2^e, m in [0.5, 1) or 0 */

static void dx_add(dx *a, double v, int ve) {
    if (!(v > 0)) return;
    int pe;
    const double pm = frexp(v, &pe);
    pe += ve;
    if (a->m == 0 || pe > a->e + 60) {
        a->m = pm;
        a->e = pe;
    } else if (pe >= a->e - 60) {
        int e2;
        a->m = frexp(a->m + ldexp(pm, pe - a->e), &e2);
        a->e += e2;
    }
}

static int row_exponent(const double *a, const double *b, int n) {
    double mx = 0;
    for (int k = 0; k < n; ++k) {
        if (a[k] > mx) mx = a[k];
        if (b && b[k] > mx) mx = b[k];
    }
    int e = 0;
    if (mx > 0) frexp(mx, &e);
    return e;
}

int dmsto_posteriors(const double *values, const double *params, const float *bg, int M, const uint8_t *codes,
                     int L, dmsto_rates r, double *logT_fwd, double *logT_bwd, double *cell, double *match) {
    if (!values || !params || !bg || !codes || M < 1 || L < 3) return -1;
    const unsigned csr = ftz_enter();
    const size_t R = (size_t)M + 1;
    float *seeds = (float *)calloc(2 * (size_t)L + 8, sizeof(float));
    double *W0 = (double *)calloc(R * (size_t)L, sizeof(double));
    double *Y0 = (double *)calloc(R * (size_t)L, sizeof(double));
    int *eF = (int *)calloc(R, sizeof(int));
    const size_t W = (size_t)L + 4;
    double *rows = (double *)calloc(4 * W, sizeof(double));
    int st = -1;
    null_out o = {seeds, seeds + L + 4, 0, 0, 0};
    if (seeds && W0 && Y0 && eF && rows && !null_model(bg, codes, L, r, &o)) {
        const double s1 = o.s1, s2 = o.s2, sC = o.sC;
        const float *bg4 = bg + 4;
#define CODE(j) (((j) >= 0 && (j) < L) ? codes[(j)] : NCODE_PAD)
        dx Tf = {0, 0}, Tb = {0, 0};
        /* forward */
        for (int i = 0; i <= M; ++i) {
            const double *q = params + (size_t)i * NPARAM;
            const double *qp = params + (size_t)(i > 0 ? i - 1 : 0) * NPARAM;
            const double *eprev = values + (size_t)(i > 0 ? i - 1 : 0) * WIDTH + 4;
            double *w = W0 + (size_t)i * L, *y = Y0 + (size_t)i * L;
            const double *wp = i > 0 ? W0 + (size_t)(i - 1) * L : NULL, *yp = i > 0 ? Y0 + (size_t)(i - 1) * L : NULL;
            const int sh = i > 0 ? row_exponent(wp, yp, L) : 0;
            eF[i] = i > 0 ? eF[i - 1] + sh : 0;
            const double f = ldexp(1.0, -sh);
            double z[3] = {0, 0, 0};
            double part = 0;
            for (int j = 0; j < L; ++j) {
                double in = 0;
                if (i > 0) {
                    const double u3 = j >= 3 ? wp[j - 3] : 0, u2 = j >= 2 ? wp[j - 2] : 0, u1 = j >= 1 ? wp[j - 1] : 0;
                    in = (qp[10] * sC * eprev[CODE(j - 2)] * u3 + yp[j] + qp[7] * s2 * u2 + qp[8] * s1 * u1) * f;
                }
                const double w3 = j >= 3 ? w[j - 3] : 0, w2 = j >= 2 ? w[j - 2] : 0, w1 = j >= 1 ? w[j - 1] : 0;
                const double zz = (double)bg4[CODE(j - 2)] * sC * (q[0] * w3 + q[3] * z[j % 3]);
                w[j] = in + zz + q[1] * s1 * w1 + q[2] * s2 * w2 + ldexp((double)o.pre[j], -eF[i]);
                y[j] = q[6] * w[j] + q[9] * (i > 0 ? yp[j] * f : 0);
                z[j % 3] = zz;
                part += w[j] * (double)o.suf[j];
            }
            dx_add(&Tf, part, eF[i]);
        }
        /* backward */
        const double invT = Tf.m > 0 ? 1.0 / Tf.m : 0.0;
        double *below = rows, *row = rows + W, *ynext = rows + 2 * W, *ycur = rows + 3 * W;
        int eBn = 0; /* offset of row i+1 */
        for (int i = M; i >= 0; --i) {
            const double *q = params + (size_t)i * NPARAM;
            const double *erow = values + (size_t)i * WIDTH + 4;
            const int sh = i < M ? row_exponent(below, ynext, L) : 0;
            const int eB = eBn + sh;
            const double f = ldexp(1.0, -sh);
            const double enter = q[10] * sC, d0 = q[6], d1 = q[7] * s2, d2 = q[8] * s1;
            const double a0 = q[0] * sC, a1 = q[1] * s1, a2 = q[2] * s2, b0 = q[3] * sC, eps = q[9];
            double z[4] = {0, 0, 0, 0};
            double n3 = below[L + 2] * f, n2 = below[L + 1] * f, n1 = below[L] * f, c2 = 0, c1 = 0, part = 0;
            for (int j = L; j < L + 4; ++j) row[j] = ycur[j] = 0;
            for (int j = L - 1; j >= 0; --j) {
                const int c = CODE(j + 1);
                const double zbg = z[(j + 3) & 3] * (double)bg4[c];
                const double yn = ynext[j] * f;
                const double wv = n3 * erow[c] * enter + yn * d0 + n2 * d1 + n1 * d2 + zbg * a0 + c2 * a2 +
                                  c1 * a1 + ldexp((double)o.suf[j], -eB);
                row[j] = wv;
                ycur[j] = eps * yn + wv;
                z[j & 3] = b0 * zbg + wv;
                part += (double)o.pre[j] * wv;
                if (cell) cell[(size_t)i * L + j] = ldexp(W0[(size_t)i * L + j] * wv * invT, eF[i] + eB - Tf.e);
                if (match && j + 3 < L)  /* X(i, j+3) W1[i+1][j+3]; row i+1 unscaled, offset eBn */
                    match[(size_t)i * L + j + 3] =
                        ldexp(enter * erow[c] * W0[(size_t)i * L + j] * below[j + 3] * invT, eF[i] + eBn - Tf.e);
                n3 = n2;
                n2 = n1;
                n1 = below[j] * f;
                c2 = c1;
                c1 = wv;
            }
            if (match)
                for (int j = 0; j < 3 && j < L; ++j) match[(size_t)i * L + j] = 0;
            dx_add(&Tb, part, eB);
            eBn = eB;
            double *t = below;
            below = row;
            row = t;
            t = ynext;
            ynext = ycur;
            ycur = t;
        }
#undef CODE
        if (logT_fwd) *logT_fwd = Tf.m > 0 ? log(Tf.m) + Tf.e * 0.6931471805599453 : -INFINITY;
        if (logT_bwd) *logT_bwd = Tb.m > 0 ? log(Tb.m) + Tb.e * 0.6931471805599453 : -INFINITY;
        st = 0;
    }
    free(seeds);
    free(W0);
    free(Y0);
    free(eF);
    free(rows);
    ftz_leave(csr);
    return st;
}
