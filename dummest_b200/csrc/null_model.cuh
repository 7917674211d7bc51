// Per-pair null model on the device: the codon/frameshift background prefix
// and suffix probabilities, the whole-sequence null total, the per-base
// scales and the seed vectors that the DP consumes.
//
// Restates, for one sequence (single-lane semantics), the reference's
//   buildNullSuffix            dummest-dp-backward.hh:6-55
//   buildNullPrefixFirstCodon  dummest-dp-backward.hh:58-100
//   buildNullTotalAndScales    dummest-dp-backward.hh:103-129
//   buildNullSeedModels        dummest-dp-backward.hh:133-165
// with the exact score algebra of dummest-score.hh / dummest-batch.hh: each
// step rounds a double to a float mantissa exactly where the reference does,
// so the seeds are bit-identical to the reference's (up to the last-ulp
// behaviour of log2/exp2 in double, which feeds one float rounding).
// A sequence's per-lane result in the reference does not depend on the batch
// it was scored in (lanes past their length are forced to 0 or 1), so the
// single-sequence form is the reference's result for that lane.
#pragma once

#include "dp_common.cuh"

namespace dmst {

struct XS {  // ExpScore (dummest-score.hh:28-33)
    float m;
    int e;
};

__device__ __forceinline__ XS xsZero() { return XS{0.0f, 0}; }
__device__ __forceinline__ XS pow2Score(int e2) { return XS{0.5f, e2 + 1}; }  // dummest-score.hh:197-199

// splitNormalizedDouble (dummest-batch.hh:42-53); also normalizeScore's frexp
// for every non-subnormal double (products here never reach double
// subnormals).
__device__ __forceinline__ XS splitNorm(double x, int eAdd) {
    if (x == 0.0) return xsZero();
    unsigned long long u = (unsigned long long)__double_as_longlong(x);
    int ef = (int)((u >> 52) & 0x7FFULL);
    if (ef == 0x7FF) return XS{__double2float_rn(x), eAdd};
    if (ef == 0) return xsZero();
    double m = __longlong_as_double((long long)((u & 0xFFFFFFFFFFFFFULL) | (1022ULL << 52)));
    return XS{__double2float_rn(m), eAdd + ef - 1022};
}

// scaleScore / batchScaleScores (dummest-score.hh:155-160, dummest-batch.hh:114-130).
__device__ __forceinline__ XS scaleScore(XS a, double f) {
    if (a.m == 0.0f) return xsZero();
    if (!(f > 0.0) || !isfinite(f)) return xsZero();
    return splitNorm(__dmul_rn((double)a.m, f), a.e);
}

// scaleScore by a positive finite factor below 1 (the frameshift emission
// rates): the product of a float mantissa in [0.5, 1] and f is 0 or a normal
// double, so splitNorm's infinity and subnormal cases cannot occur; the
// result is scaleScore's.
__device__ __forceinline__ XS scaleByRate(XS a, double f) {
    if (a.m == 0.0f) return xsZero();
    const double x = __dmul_rn((double)a.m, f);
    const unsigned long long u = (unsigned long long)__double_as_longlong(x);
    const int ef = (int)((u >> 52) & 0x7FFULL);
    const double m = __longlong_as_double((long long)((u & 0xFFFFFFFFFFFFFULL) | (1022ULL << 52)));
    return XS{__double2float_rn(m), a.e + ef - 1022};
}

// batchAddScores (dummest-batch.hh:78-108).
__device__ __forceinline__ XS batchAdd(XS a, XS b) {
    if (a.m == 0.0f) return b;
    if (b.m == 0.0f) return a;
    const bool agebe = a.e >= b.e;
    const float mh = agebe ? a.m : b.m, ml = agebe ? b.m : a.m;
    const int eh = agebe ? a.e : b.e, el = agebe ? b.e : a.e;
    int d = eh - el;
    d = d > 60 ? 60 : d;
    // 1 / 2^d is the exact power 2^-d (0 <= d <= 60), built from its exponent
    // bits instead of a double division; ml * 2^-d is exact, so the sum
    // rounds once, as the reference's does.
    const double inv = __longlong_as_double((long long)(1023 - d) << 52);
    double s = __dadd_rn((double)mh, __dmul_rn((double)ml, inv));
    int e = eh;
    if (s >= 1.0) {
        s *= 0.5;
        e += 1;
    }
    return XS{__double2float_rn(s), e};
}

// addScores, the scalar form (dummest-score.hh:169-181).  ldexp(m, -d) for
// 0 <= d <= 60 is the product of m and the power 2^-d built from its exponent
// bits: both exact, so the same bits.
__device__ __forceinline__ XS scalarAdd(XS a, XS b) {
    if (a.m == 0.0f) return b;
    if (b.m == 0.0f) return a;
    const bool agebe = a.e >= b.e;
    const XS h = agebe ? a : b, l = agebe ? b : a;
    const int d = h.e - l.e;
    if (d > 60) return h;
    const double inv = __longlong_as_double((long long)(1023 - d) << 52);
    return splitNorm(__dadd_rn((double)h.m, __dmul_rn((double)l.m, inv)), h.e);
}

// batchMulScores with eFold = 0 (dummest-batch.hh:58-72).
__device__ __forceinline__ XS batchMul(XS a, XS b) {
    if (a.m == 0.0f || b.m == 0.0f) return xsZero();
    double p = __dmul_rn((double)a.m, (double)b.m);
    int e = a.e + b.e;
    if (p < 0.5) {
        p *= 2.0;
        e -= 1;
    }
    return XS{__double2float_rn(p), e};
}

// mulScores, the scalar form (dummest-score.hh:184-188).
__device__ __forceinline__ XS scalarMul(XS a, XS b) {
    if (a.m == 0.0f || b.m == 0.0f) return xsZero();
    return splitNorm(__dmul_rn((double)a.m, (double)b.m), a.e + b.e);
}

// scoreToFloatClamped (dummest-score.hh:224-230), FP32 engine: exponent capped
// at 120.  With the mantissa in [0.5, 1], m 2^e is a normal float for
// -125 <= e <= 120, where it is the exact product of m and the power of two
// built from its exponent bits; smaller exponents (subnormal or zero results)
// go through ldexpf.
__device__ __forceinline__ float packScore(XS a) {
    if (a.m == 0.0f) return 0.0f;
    const int e = a.e > 120 ? 120 : a.e;
    if (e >= -125) return __fmul_rn(a.m, __int_as_float((e + 127) << 23));
    return ldexpf(a.m, e);
}

struct NullRates {
    double single;      // BACKGROUND_FRAMESHIFT_RATE (a float value)
    double dbl;         // BACKGROUND_FRAMESHIFT_RATE_2 (a float value)
};

__device__ __forceinline__ float bgAt(const float *bg, const uint8_t *codes, int L, int j) {
    return (j >= 0 && j < L) ? bg[codes[j]] : 0.0f;  // beyond the sequence: zero_idx, bg 0
}

// Prefix recurrence (dummest-dp-backward.hh:66-99) step i, given the three
// previous prefix values.
__device__ __forceinline__ XS prefixStep(int i, const float *bg, const uint8_t *codes, int L, XS p1, XS p2, XS p3,
                                         double keep, double sNE, double dNE) {
    const float bgc = bgAt(bg, codes, L, i - 2);
    const double codonScale = __dmul_rn((double)bgc, keep);
    const double frame = 1.0 / 3.0;
    XS codon;
    if (i >= 3)
        codon = scaleScore(p3, codonScale);
    else if (i == 2)
        codon = scaleScore(splitNorm((double)bgc, 0), frame);
    else if (i == 1)
        codon = scaleScore(pow2Score(-4), frame);
    else
        codon = scaleScore(pow2Score(-2), frame);
    XS single = scaleByRate(i > 0 ? p1 : xsZero(), sNE);
    XS dbl = scaleByRate(i >= 2 ? p2 : xsZero(), dNE);
    return batchAdd(codon, batchAdd(single, dbl));
}

// Pairs whose reads have one length are scored by one warp, one lane per
// pair (the pairs of one read side by side, so that their codon loads are
// broadcasts): the lanes run in lock step over the L columns, keep the
// suffix recurrence in registers, store the temporary prefix and suffix
// probabilities interleaved (one coalesced 256-byte store per column), and
// write their seed vectors through a shared-memory transpose, so that each
// store instruction writes 32 consecutive seeds of one pair.
// Temporary ExpScores of one null-model job: the prefix [L][32] and the
// suffix [L+1][32] probabilities of its (up to) 32 pairs, interleaved.
__host__ __device__ constexpr long long nullTmpEntries(long long L) { return 2 * 32 * (L + 1); }

struct NullJob {
    int first;  // index of the job's first pair in the pair-index array
    int count;  // pairs in the job (<= 32), all with the same read
};

constexpr int kNullWarps = 4;

__device__ __forceinline__ void flushSeeds(float (*stage)[33], float *const *dst, int count, int j0, int ncol,
                                           int lane) {
    // stage[c][p] holds column j0 + c of pair p; write pair p's columns with
    // lanes over columns.
    __syncwarp();
    for (int p = 0; p < count; ++p)
        if (lane < ncol) dst[p][j0 + lane] = stage[lane][p];
    __syncwarp();
}

__global__ void __launch_bounds__(kNullWarps * 32) nullModelKernel(const NullJob *jobs, int nJobs, const int *jobPairs,
                                                                   const DevPair *pairs, const DevProfile *profiles,
                                                                   const uint8_t *codes, float *seeds, XS *tmp,
                                                                   const long long *tmpOff, PairScales *scales,
                                                                   NullRates r) {
    __shared__ float stageAll[kNullWarps][32][33];
    __shared__ float *dstAll[kNullWarps][2][32];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    float (*stage)[33] = stageAll[warp];
    const double keep = 1.0 - r.single - r.dbl;  // codonKeepProbability
    const double sNE = r.single * 0.25;          // singleNucleotideEmission
    const double dNE = r.dbl * 0.0625;           // doubleNucleotideEmission
    for (int ji = blockIdx.x * kNullWarps + warp; ji < nJobs; ji += gridDim.x * kNullWarps) {
        const NullJob job = jobs[ji];
        const bool on = lane < job.count;
        const int pi = jobPairs[job.first + (on ? lane : 0)];
        const DevPair p = pairs[pi];
        const int L = p.L;
        const uint8_t *cd = codes + p.codeOff;
        const float *bg = profiles[p.prof].bg;
        float *pre = seeds + p.seedOff;
        dstAll[warp][0][lane] = on ? pre : nullptr;
        dstAll[warp][1][lane] = on ? pre + L : nullptr;
        XS *pfx = tmp + tmpOff[ji];           // [L x 32] interleaved prefix probabilities
        XS *sfx = pfx + 32 * ((size_t)L + 1);  // [(L+1) x 32] interleaved suffix probabilities

        // Pass 1: the prefix recurrence (dummest-dp-backward.hh:58-100, i = 0..L-1)
        // and the suffix recurrence (:6-55, i = L-1..0, from suffix[L] = 1 and
        // suffix[L+1..L+3] = 0), two independent chains run side by side; both
        // sequences are kept for the seed passes.
        XS p1 = xsZero(), p2 = xsZero(), p3 = xsZero();
        const XS trailing = splitNorm(0.5 * keep, 0);
        XS s1 = pow2Score(0), s2 = xsZero(), s3 = xsZero();  // suffix[i+1], [i+2], [i+3]
        for (int k = 0; k < L; ++k) {
            const XS q = prefixStep(k, bg, cd, L, p1, p2, p3, keep, sNE, dNE);
            pfx[(size_t)k * 32 + lane] = q;
            p3 = p2;
            p2 = p1;
            p1 = q;
            const int i = L - 1 - k;
            const double codonScale = __dmul_rn((double)bgAt(bg, cd, L, i), keep);
            const XS single = scaleByRate(s1, sNE);
            const XS dIn = (i + 1 < L) ? s2 : pow2Score(2);
            const XS dbl = scaleByRate(dIn, dNE);
            const XS codon = (i + 2 < L) ? scaleScore(s3, codonScale) : XS{trailing.m, trailing.e - 2 * (L - i) + 1};
            const XS v = batchAdd(codon, batchAdd(single, dbl));
            sfx[(size_t)i * 32 + lane] = v;
            s3 = s2;
            s2 = s1;
            s1 = v;
        }
        // Total and scales (dummest-dp-backward.hh:103-129).
        const double keepSingle = 1.0 - r.single;
        const double keepBoth = keepSingle - r.dbl;
        const XS trailingSingle = scaleScore(p2, keepSingle * 0.25);
        const XS trailingDouble = scaleScore(p3, keepBoth * 0.0625);
        const XS total = scalarAdd(scalarAdd(p1, trailingSingle), trailingDouble);
        const float nullLog = (total.m == 0.0f) ? -INFINITY : (float)(log2((double)total.m) + (double)total.e);
        double perBaseLog = -(double)nullLog / (double)L;
        if (!(perBaseLog < 120.0)) perBaseLog = 120.0;
        const double perBaseRaw = exp2(perBaseLog);
        const XS perBase = splitNorm(perBaseRaw, 0);
        const XS perBaseInv = splitNorm(1.0 / perBaseRaw, 0);
        const XS quarter = splitNorm(0.25, 0), sixteenth = splitNorm(0.0625, 0);
        if (on) {
            PairScales sc;
            sc.s1 = packScore(scalarMul(perBase, quarter));
            sc.s2 = packScore(scalarMul(scalarMul(perBase, perBase), sixteenth));
            sc.sC = packScore(scalarMul(scalarMul(perBase, perBase), perBase));
            sc.pad = 0.0f;
            scales[pi] = sc;
        }

        // Pass 2: prefix seeds (dummest-dp-backward.hh:155-164) from the kept
        // prefix, beside the L-1 multiplications that start the suffix seeds'
        // running scale (:137-145).
        XS running = pow2Score(0);
        XS runPre = perBase;
        for (int j0 = 0; j0 < L; j0 += 32) {
            const int ncol = L - j0 < 32 ? L - j0 : 32;
            for (int c0 = 0; c0 < ncol; c0 += 8) {
                // the kept prefix values of 8 columns, loaded before the chain uses them
                XS v[8];
#pragma unroll
                for (int u = 0; u < 8; ++u)
                    v[u] = (c0 + u < ncol) ? pfx[(size_t)(j0 + c0 + u) * 32 + lane] : xsZero();
#pragma unroll
                for (int u = 0; u < 8; ++u) {
                    const int c = c0 + u;
                    if (c >= ncol) break;
                    const int j = j0 + c;
                    stage[c][lane] = packScore(batchMul(v[u], runPre));
                    runPre = batchMul(runPre, perBase);
                    if (j < L - 1) running = batchMul(running, perBase);
                }
            }
            flushSeeds(stage, dstAll[warp][0], job.count, j0, ncol, lane);
        }

        // Pass 3: suffix seeds (dummest-dp-backward.hh:146-154).
        for (int j0 = 0; j0 < L; j0 += 32) {
            const int ncol = L - j0 < 32 ? L - j0 : 32;
            for (int c0 = 0; c0 < ncol; c0 += 8) {
                XS v[8];
#pragma unroll
                for (int u = 0; u < 8; ++u) {
                    const int j = j0 + c0 + u;
                    v[u] = (c0 + u < ncol && j + 1 < L) ? sfx[(size_t)(j + 1) * 32 + lane] : pow2Score(0);
                }
#pragma unroll
                for (int u = 0; u < 8; ++u) {
                    const int c = c0 + u;
                    if (c >= ncol) break;
                    stage[c][lane] = packScore(batchMul(v[u], running));
                    running = batchMul(running, perBaseInv);
                }
            }
            flushSeeds(stage, dstAll[warp][1], job.count, j0, ncol, lane);
        }
        __syncwarp();
    }
}

}  // namespace dmst
