// The exact row-rescaled DP for pairs whose values leave the fast path's
// range: one thread per pair, rows in sequence, the reference's dynamic row
// rescaling (2^-64 whenever a row maximum exceeds RESCALE_THRESH) and exact
// (mantissa, exponent) products for the mid and filter scores.
//
// It restates for one lane
//   backwardPass          dummest-dp-backward.hh:444-615 (incl. bestOut :579-609)
//   forwardPass scores    dummest-dp-forward.hh:9-250, :536-544
//   row rescale helpers   dummest-score.hh:78-152
//   promote / product     dummest-batch.hh:146-235
// Only pairs whose reported scores exceed ~100 bits (or whose null seeds are
// extreme) come here, so the kernel favours exactness over speed.
#pragma once

#include "dp_common.cuh"
#include "dp_wavefront.cuh"
#include "null_model.cuh"

namespace dmst {

__device__ __forceinline__ int clampCount(int c) {
    return c > 1000000 ? 1000000 : (c < -1000000 ? -1000000 : c);
}

// promoteRescaledScore (dummest-score.hh:107-116) with the subnormal flush of
// batchPromoteRescaled's scalar path (dummest-batch.hh:201-210).
__device__ __forceinline__ XS promote(float v, int cum) {
    if (!(v > 0.0f)) return xsZero();
    if (v < 1.17549435e-38f) return xsZero();  // subnormal input flushes
    cum = clampCount(cum);
    if (!(v < INFINITY)) return XS{0.99999994f, 1023 + kRescaleBits * cum};
    return splitNorm((double)v, kRescaleBits * cum);
}

// scoreLess (dummest-score.hh:70-76): zero sorts below everything positive.
__device__ __forceinline__ bool scoreLess(XS a, XS b) {
    if (a.m == 0.0f) return b.m != 0.0f;
    if (b.m == 0.0f) return false;
    if (a.e != b.e) return a.e < b.e;
    return a.m < b.m;
}

// batchMulScorePlanes with eFold = STATIC_SHIFT = 0 (dummest-batch.hh:216-235).
__device__ __forceinline__ XS planeMul(XS a, XS b) { return batchMul(a, b); }

__device__ __forceinline__ float rowScale(int cnt) {
    // rowRescaleVector (dummest-score.hh:145-152): 2^(-64 * count), a float.
    return ldexpf(1.0f, -kRescaleBits * clampCount(cnt));
}

struct ExactJob {
    int pair;             // index into the pair arrays
    long long scratchOff; // float offset of this job's scratch
};

struct ExactOut {
    XS mid;
    XS filt;
    int failed;  // the pipelined kernel gave up a wait (the scores are not valid)
    int pad;
};

// Scratch per job (floats): W1 (M+2) x (L+4), then four rows of L+4
// (Y0a, Y0b, W0a, W0b), then 2 x (M+2) ints of rescale counts.
__host__ __device__ inline long long exactScratchFloats(int M, int L) {
    return (long long)(M + 2) * (L + 4) + 4LL * (L + 4) + 2LL * (M + 2);
}

__global__ void exactKernel(const ExactJob *jobs, int n, const DevPair *pairs, const DevProfile *profiles,
                            const float *emit, const float *params, const uint8_t *codes, const float *seeds,
                            const PairScales *scales, float *scratch, ExactOut *out) {
    const int ji = blockIdx.x * blockDim.x + threadIdx.x;
    if (ji >= n) return;
    const ExactJob job = jobs[ji];
    const DevPair p = pairs[job.pair];
    const DevProfile &pr = profiles[p.prof];
    const PairScales sc = scales[job.pair];
    const int L = p.L, M = p.M, W = L + 4;
    const uint8_t *cd = codes + p.codeOff;
    const float *pre = seeds + p.seedOff;
    const float *suf = pre + L;
    const float *E = emit + pr.emitOff;
    const int rowPad = pr.rowPad;
    const float *par = params + pr.paramOff;
    float *W1 = scratch + job.scratchOff;
    float *Ya = W1 + (size_t)(M + 2) * W;
    float *Yb = Ya + W;
    float *Wa = Yb + W;
    float *Wb = Wa + W;
    int *cntB = reinterpret_cast<int *>(Wb + W);
    int *cntF = cntB + (M + 2);
    const float *bg = pr.bg;
    auto code = [&](int j) -> int { return (j >= 0 && j < L) ? (int)cd[j] : kPad; };
    const float RESCALE_STEP = ldexpf(1.0f, -kRescaleBits);

    // ---- backward (dummest-dp-backward.hh:249-263, :473-574) ----
    for (int j = 0; j < W; ++j) {
        W1[(size_t)(M + 1) * W + j] = 0.0f;
        Ya[j] = 0.0f;
        Yb[j] = 0.0f;
        Wa[j] = 0.0f;
        Wb[j] = 0.0f;
    }
    for (int i = 0; i <= M; ++i)
        for (int j = L; j < W; ++j) W1[(size_t)i * W + j] = 0.0f;
    for (int i = 0; i < M + 2; ++i) cntB[i] = cntF[i] = 0;
    float *Ynext = Ya, *Ycur = Yb;
    for (int i = M; i >= 0; --i) {
        if (i < M) cntB[i] = cntB[i + 1];
        const float *q = par + (size_t)i * kParamFloats;
        const float enter = q[10] * sc.sC, d0 = q[6], d1 = q[7] * sc.s2, d2 = q[8] * sc.s1;
        const float a0 = q[0] * sc.sC, a1 = q[1] * sc.s1, a2 = q[2] * sc.s2, b0 = q[3] * sc.sC, eps = q[9];
        const float rs = 1.0f * rowScale(cntB[i]);
        float rowMax = 0.0f;
        float *row = W1 + (size_t)i * W;
        const float *below = W1 + (size_t)(i + 1) * W;
        float nJ3 = below[L + 2], nJ2 = below[L + 1], nJ1 = below[L];
        float cJ2 = row[L + 1], cJ1 = row[L];
        float z[4] = {0.0f, 0.0f, 0.0f, 0.0f};
        for (int j = L - 1; j >= 0; --j) {
            const int c = code(j + 1);
            const float e = E[(size_t)c * rowPad + i];
            const float bgv = bg[c];
            const float nAt = below[j];
            float acc = (nJ3 * e) * enter;
            acc = __fmaf_rn(Ynext[j], d0, acc);
            acc = __fmaf_rn(nJ2, d1, acc);
            acc = __fmaf_rn(nJ1, d2, acc);
            const float zbg = z[(j + 3) & 3] * bgv;
            acc = __fmaf_rn(zbg, a0, acc);
            acc = __fmaf_rn(cJ2, a2, acc);
            acc = __fmaf_rn(cJ1, a1, acc);
            const float wv = __fmaf_rn(suf[j], rs, acc);
            row[j] = wv;
            rowMax = fmaxf(rowMax, wv);
            Ycur[j] = __fmaf_rn(eps, Ynext[j], wv);
            rowMax = fmaxf(rowMax, Ycur[j]);
            z[j & 3] = __fmaf_rn(b0, zbg, wv);
            nJ3 = nJ2;
            nJ2 = nJ1;
            nJ1 = nAt;
            cJ2 = cJ1;
            cJ1 = wv;
        }
        float *tmp = Ycur;
        Ycur = Ynext;
        Ynext = tmp;
        if (rowMax > kRescaleThresh) {
            cntB[i]++;
            for (int j = 0; j < W; ++j) row[j] *= RESCALE_STEP;
            for (int j = 0; j < W; ++j) {
                Ynext[j] *= RESCALE_STEP;
                Ycur[j] *= RESCALE_STEP;
            }
        }
    }

    // ---- exact filter best (dummest-dp-backward.hh:579-609) ----
    XS bestFilt = xsZero();
    for (int j = 0; j < L; ++j) {
        const double nd = (double)pre[j];
        for (int i = M; i >= 0; --i) {
            const XS r = promote(W1[(size_t)i * W + j], cntB[i]);
            const XS cand = scaleScore(r, nd);
            if (scoreLess(bestFilt, cand)) bestFilt = cand;
        }
    }

    // ---- forward with the mid score (dummest-dp-forward.hh:30, :63-250) ----
    for (int j = 0; j < W; ++j) {
        Ya[j] = 0.0f;
        Yb[j] = 0.0f;
        Wa[j] = 0.0f;
        Wb[j] = 0.0f;
    }
    Ynext = Ya;
    Ycur = Yb;
    float *W0cur = Wa, *W0nxt = Wb;
    XS best = xsZero();
    for (int i = 0; i <= M; ++i) {
        if (i > 0) cntF[i] = cntF[i - 1];
        const float *q = par + (size_t)i * kParamFloats;
        const float enter = q[10] * sc.sC, a0 = q[0], a1 = q[1] * sc.s1, a2 = q[2] * sc.s2, b0 = q[3];
        const float d0 = q[6], d1 = q[7] * sc.s2, d2 = q[8] * sc.s1, eps = q[9];
        const float rs = 1.0f * rowScale(cntF[i]);
        float rowMax = 0.0f;
        float z0[4] = {0.0f, 0.0f, 0.0f, 0.0f};
        float ws0 = 0.0f, ws1 = 0.0f, ws2 = 0.0f;
        const float *w1row = W1 + (size_t)i * W;
        for (int j = 0; j < L; ++j) {
            const float w1 = ws0, w2 = ws1, w3 = ws2;
            const int c = code(j - 2);
            const float e = E[(size_t)c * rowPad + i];
            const float bgv = bg[c];
            const float X = (enter * e) * w3;
            // GCC's contraction of dummest-dp-forward.hh:148-166 at -O3.
            const float Z0 = (bgv * sc.sC) * __fmaf_rn(b0, z0[(j - 3) & 3], a0 * w3);
            z0[j & 3] = Z0;
            const float w0 = W0cur[j] + __fmaf_rn(pre[j], rs, __fmaf_rn(a2, w2, __fmaf_rn(a1, w1, Z0)));
            rowMax = fmaxf(rowMax, w0);
            const XS f = promote(w0, cntF[i]);
            const XS b = promote(w1row[j], cntB[i]);
            const XS wm = planeMul(f, b);
            if (scoreLess(best, wm)) best = wm;
            W0cur[j] = w0;
            ws2 = ws1;
            ws1 = ws0;
            ws0 = w0;
            Ycur[j] = __fmaf_rn(eps, Ynext[j], d0 * w0);
            rowMax = fmaxf(rowMax, Ycur[j]);
            if (i < M) W0nxt[j] = W0nxt[j] + __fmaf_rn(d2, w1, __fmaf_rn(d1, w2, X + Ycur[j]));
        }
        if (rowMax > kRescaleThresh) {
            cntF[i]++;
            if (i < M)
                for (int j = 0; j < W; ++j) W0nxt[j] *= RESCALE_STEP;
            for (int j = 0; j < W; ++j) {
                Ynext[j] *= RESCALE_STEP;
                Ycur[j] *= RESCALE_STEP;
            }
        }
        float *t = Ycur;
        Ycur = Ynext;
        Ynext = t;
        t = W0cur;
        W0cur = W0nxt;
        W0nxt = t;
        for (int j = 0; j < W; ++j) W0nxt[j] = 0.0f;
    }
    out[ji].mid = best;
    out[ji].filt = bestFilt;
    out[ji].failed = 0;
}

}  // namespace dmst
