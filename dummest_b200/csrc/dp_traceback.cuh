// Traceback of the hit path (dummest-dp-forward.hh:276-453, :471-535,
// dummest-dp.hh:119-268, dummest-traceback.hh:6-118), for the jobs of
// dp_traceback_job.cuh, after the exact kernel's replay stored each job's W0,
// W1 and rescale counts:
//
//   sidesKernel     column masses: reverseSide[j] = sum over rows (M..0) of W1
//                   and forwardSide[j] = sum over rows (0..M) of W0, each
//                   scaled down with its rows' rescales (the reference's
//                   per-cell fma(1, w, side) and per-row rescaleRow);
//   flank*Kernel    buildFlankEVs: the entry and exit flank totals as exact
//                   scores, and their largest exponents;
//   xTableKernel    X(i, j) = promote(X_ij, cntF_i) * promote(W1[i+1][j],
//                   cntB_{i+1}), the forward's combined match scores, and
//                   each row's largest exponent;
//   optimalKernel   the prefix- and suffix-optimal tables in the row-scaled
//                   float form of dummest-scalerow.hh: each row is a running
//                   maximum (a block-wide max scan) of candidates read from
//                   the row before;
//   spanKernel      the forward and reverse walks of every candidate anchor
//                   at once (they do not depend on which anchors are kept):
//                   each walk's sequence span and match counts; the host
//                   then takes the anchors in the reference's sorted order,
//                   skipping those inside or overlapping kept ones;
//   storeWalkKernel the kept anchors' walks again, writing their segments.
//
// Columns at or past a pair's length are not built: the reference's values
// there are zero (W1 is masked, so X and the exit flank totals are 0) or
// never read (the prefix table right of the anchor), so a per-pair width L
// gives the reference's tables and walks whatever its batch width.
#pragma once

#include "dp_common.cuh"
#include "dp_exact.cuh"
#include "dp_traceback_job.cuh"
#include "null_model.cuh"

namespace dmst {

// promoteRescaledScore, the scalar form (dummest-score.hh:107-116).
__device__ __forceinline__ XS promoteScalar(float v, int cum) {
    if (!(v > 0.0f)) return xsZero();
    cum = clampCount(cum);
    if (!(v < INFINITY)) return XS{0.99999994f, 1023 + kRescaleBits * cum};
    return splitNorm((double)v, kRescaleBits * cum);
}

// scoreToRowScale / scoreFromRowScale (dummest-scalerow.hh:26-55): the score
// moved to row exponent E by rewriting the exponent field, and back.
__device__ __forceinline__ float toRow(XS s, int E) {
    const unsigned u = __float_as_uint(s.m);
    int d = s.e - E;
    d = d > 0 ? 0 : (d < -1000 ? -1000 : d);
    const int ne = 126 + d;
    const float r = __uint_as_float((u & 0x807FFFFFu) | ((unsigned)(ne > 0 ? ne : 0) << 23));
    return (s.m == 0.0f || ne <= 0) ? 0.0f : r;
}
__device__ __forceinline__ XS fromRow(float s, int E) {
    const unsigned u = __float_as_uint(s);
    const unsigned ef = (u >> 23) & 0xFFu;
    const bool live = (s > 0.0f) && ef != 0;
    const XS o{__uint_as_float((u & 0x807FFFFFu) | (126u << 23)), (int)ef - 126 + E};
    return live ? o : xsZero();
}

__device__ __forceinline__ XS ldXS(const XS *p) {
    const float2 v = *reinterpret_cast<const float2 *>(p);
    return XS{v.x, __float_as_int(v.y)};
}
__device__ __forceinline__ void stXS(XS *p, XS s) {
    *reinterpret_cast<float2 *>(p) = make_float2(s.m, __int_as_float(s.e));
}

// Column masses, one thread per (job, column).  Block 0 of a job also resets
// the X table's row maxima (INT_MIN, dummest-dp-backward.hh:265-269).
__global__ void sidesKernel(const AlignJob *jobs, const float *cells, int *rows, float *colR, float *colF) {
    const AlignJob jb = jobs[blockIdx.y];
    const int M = jb.M, L = jb.L;
    int *cntB = rows + jb.rowOff, *cntF = cntB + (M + 2), *rowMaxX = cntF + (M + 2);
    if (blockIdx.x == 0)
        for (int i = threadIdx.x; i < M + 2; i += blockDim.x) rowMaxX[i] = INT_MIN;
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= L) return;
    const float *W0 = cells + 2 * jb.cellOff;
    const float *W1 = W0 + (size_t)(M + 1) * L;
    float r = 0.0f;
    for (int i = M; i >= 0; --i) {
        r = __fadd_rn(r, W1[(size_t)i * L + j]);
        if (cntB[i] != cntB[i + 1]) r = __fmul_rn(r, stepsDown(cntB[i] - cntB[i + 1]));
    }
    float f = 0.0f;
    for (int i = 0; i <= M; ++i) {
        f = __fadd_rn(f, W0[(size_t)i * L + j]);
        if (cntF[i + 1] != cntF[i]) f = __fmul_rn(f, stepsDown(cntF[i + 1] - cntF[i]));
    }
    colR[jb.colOff + j] = r;
    colF[jb.colOff + j] = f;
}

// buildFlankEVs (dummest-dp.hh:137-256) in four kernels.  The reference's
// per-lane loops hold three independent recurrences (the middle entry masses
// and the suffix rest masses, run backward; the arrival masses, run forward),
// an elementwise combination and two running sums; each recurrence stays one
// sequential chain (ExpScore sums round at every step), but the chains run
// side by side, and whatever depends on the column alone is computed in
// parallel first.  Per job, work holds kFlankArrays arrays of L + 4 scores.
constexpr int kFlankArrays = 9;
enum FlankArray { kFBg = 0, kFPre, kFColR, kFColF, kFWeighted, kFMid, kFRest, kFArrival, kFUnified };

struct FlankRates {
    double sr, dr, keep, third;
};
__device__ __forceinline__ FlankRates flankRates(NullRates nr) {
    FlankRates f;
    f.sr = nr.single;
    f.dr = nr.dbl;
    f.keep = 1.0 - nr.single - nr.dbl;
    f.third = 1.0 / 3.0;
    return f;
}
__device__ __forceinline__ XS *flankArray(XS *work, const AlignJob &jb, int job, int a) {
    return work + (size_t)kFlankArrays * (jb.colOff + 4LL * job) + (size_t)a * (jb.L + 4);
}

// Per column: the background codon score bgc(j), the prefix seed's score,
// both column masses as exact scores, and the entry tiles' weighted sum.
__global__ void flankPrepKernel(const AlignJob *jobs, const DevPair *pairs, const DevProfile *profiles,
                                const uint8_t *codes, const float *seeds, const PairScales *scales, NullRates nr,
                                const float *colR, const float *colF, const int *rows, XS *work) {
    const int t = blockIdx.y;
    const AlignJob jb = jobs[t];
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    const int L = jb.L;
    if (j >= L + 4) return;
    XS *bgx = flankArray(work, jb, t, kFBg), *prex = flankArray(work, jb, t, kFPre);
    if (j >= L) {  // the arrays' tails stay zero
        for (int a = 0; a < kFlankArrays; ++a) flankArray(work, jb, t, a)[j] = xsZero();
        return;
    }
    const DevPair p = pairs[jb.pair];
    const float *bg = profiles[p.prof].bg;
    const uint8_t *cd = codes + p.codeOff;
    const float *pre = seeds + p.seedOff;
    const PairScales sc = scales[jb.pair];
    const int M = jb.M;
    const int *cntB = rows + jb.rowOff, *cntF = cntB + (M + 2);
    const FlankRates r = flankRates(nr);
    auto bgc = [&](int pos) { return (pos >= 0 && pos < L) ? splitNorm((double)bg[cd[pos]], 0) : xsZero(); };
    auto preS = [&](int pos) { return splitNorm((double)pre[pos], 0); };
    const XS aS1 = splitNorm((double)sc.s1, 0), aS2 = splitNorm((double)sc.s2, 0), aSC = splitNorm((double)sc.sC, 0);
    bgx[j] = bgc(j);
    prex[j] = preS(j);
    flankArray(work, jb, t, kFColR)[j] = promoteScalar(colR[jb.colOff + j], cntB[0]);
    flankArray(work, jb, t, kFColF)[j] = promoteScalar(colF[jb.colOff + j], cntF[M + 1]);
    // entry tiles ending at j (the first piece weighs 1/3)
    XS single = xsZero(), dbl = xsZero(), codon = xsZero();
    if (j == 0) single = preS(0);
    else single = scalarMul(scaleScore(preS(j - 1), r.sr), aS1);
    if (j == 1) dbl = scaleScore(aS2, r.third);
    else if (j >= 2) dbl = scalarMul(scaleScore(preS(j - 2), r.dr), aS2);
    if (j == 2) codon = scalarMul(scaleScore(aSC, r.third), bgc(0));
    else if (j >= 3) codon = scalarMul(scaleScore(scalarMul(preS(j - 3), aSC), r.keep), bgc(j - 2));
    flankArray(work, jb, t, kFWeighted)[j] =
        scalarAdd(single, scalarAdd(scaleScore(dbl, 2.0), scaleScore(codon, 3.0)));
}

// The three recurrences, one per warp (thread 0 of warps 0, 1, 2), inputs
// loaded kFlankAhead columns at a time ahead of the chain.
constexpr int kFlankAhead = 8;
__global__ void flankChainKernel(const AlignJob *jobs, const PairScales *scales, NullRates nr, XS *work) {
    const int t = blockIdx.x;
    if ((threadIdx.x & 31) != 0) return;
    const int w = threadIdx.x >> 5;
    const AlignJob jb = jobs[t];
    const int L = jb.L;
    const PairScales sc = scales[jb.pair];
    const FlankRates r = flankRates(nr);
    const XS aS1 = splitNorm((double)sc.s1, 0), aS2 = splitNorm((double)sc.s2, 0), aSC = splitNorm((double)sc.sC, 0);
    const XS *__restrict__ bgx = flankArray(work, jb, t, kFBg);
    if (w == 0) {
        // middle entry masses, backward: mid[j] = colR[j] + cover of j+1.. continued
        const XS *__restrict__ cR = flankArray(work, jb, t, kFColR);
        XS *__restrict__ mid = flankArray(work, jb, t, kFMid);
        XS m1 = xsZero(), m2 = xsZero(), m3 = xsZero();  // mid[j+1], mid[j+2], mid[j+3]
        for (int q = L; q < L + 4; ++q) mid[q] = xsZero();
        for (int hi = L - 1; hi >= 0; hi -= kFlankAhead) {
            XS vc[kFlankAhead], vb[kFlankAhead];
#pragma unroll
            for (int u = 0; u < kFlankAhead; ++u) {
                const int j = hi - u;
                vc[u] = j >= 0 ? ldXS(cR + j) : xsZero();
                vb[u] = j >= 0 ? ldXS(bgx + j + 1) : xsZero();
            }
#pragma unroll
            for (int u = 0; u < kFlankAhead; ++u) {
                const int j = hi - u;
                if (j < 0) break;
                XS c = scalarMul(scaleScore(m1, r.sr), aS1);
                c = scalarAdd(c, scalarMul(scaleScore(m2, r.dr), aS2));
                c = scalarAdd(c, scalarMul(scaleScore(scalarMul(m3, aSC), r.keep), vb[u]));
                const XS m = scalarAdd(vc[u], c);
                stXS(mid + j, m);
                m3 = m2;
                m2 = m1;
                m1 = m;
            }
        }
    } else if (w == 1) {
        // cover of [j, end): the empty rest at the end counts 1
        XS *__restrict__ rest = flankArray(work, jb, t, kFRest);
        const XS bS1 = scaleScore(aS1, 4.0), bS2 = scaleScore(aS2, 16.0);
        for (int q = L; q < L + 4; ++q) rest[q] = xsZero();
        rest[L] = pow2Score(0);
        XS r1 = pow2Score(0), r2 = xsZero(), r3 = xsZero();  // rest[j+1], rest[j+2], rest[j+3]
        for (int hi = L - 1; hi >= 0; hi -= kFlankAhead) {
            XS vb[kFlankAhead];
#pragma unroll
            for (int u = 0; u < kFlankAhead; ++u) vb[u] = hi - u >= 0 ? ldXS(bgx + hi - u) : xsZero();
#pragma unroll
            for (int u = 0; u < kFlankAhead; ++u) {
                const int j = hi - u;
                if (j < 0) break;
                const XS one = scalarMul(scaleScore(r1, r.sr), aS1);
                const XS two = (j + 1 <= L - 1) ? scalarMul(scaleScore(r2, r.dr), aS2) : scaleScore(bS1, r.dr * 0.25);
                XS three;
                if (j + 2 <= L - 1)
                    three = scalarMul(scaleScore(scalarMul(r3, aSC), r.keep), vb[u]);
                else if (j + 1 <= L - 1)
                    three = scaleScore(bS2, r.keep * 0.0625);
                else
                    three = scaleScore(bS1, r.keep * 0.25);
                const XS v = scalarAdd(one, scalarAdd(two, three));
                stXS(rest + j, v);
                r3 = r2;
                r2 = r1;
                r1 = v;
            }
        }
    } else if (w == 2) {
        // arrival masses, forward: cover ending at j grown from the cut masses
        const XS *__restrict__ cF = flankArray(work, jb, t, kFColF);
        XS *__restrict__ fa = flankArray(work, jb, t, kFArrival);
        XS f1 = xsZero(), f2 = xsZero(), f3 = xsZero();  // arrival at j-1, j-2, j-3
        for (int lo = 0; lo < L; lo += kFlankAhead) {
            XS vc[kFlankAhead], vb[kFlankAhead];
#pragma unroll
            for (int u = 0; u < kFlankAhead; ++u) {
                const int j = lo + u;
                vc[u] = j < L ? ldXS(cF + j) : xsZero();
                vb[u] = (j < L && j >= 2) ? ldXS(bgx + j - 2) : xsZero();
            }
#pragma unroll
            for (int u = 0; u < kFlankAhead; ++u) {
                const int j = lo + u;
                if (j >= L) break;
                XS a = vc[u];
                if (j >= 1) a = scalarAdd(a, scalarMul(scaleScore(f1, r.sr), aS1));
                if (j >= 2) a = scalarAdd(a, scalarMul(scaleScore(f2, r.dr), aS2));
                if (j >= 3) a = scalarAdd(a, scalarMul(scaleScore(scalarMul(f3, aSC), r.keep), vb[u]));
                stXS(fa + j, a);
                f3 = f2;
                f2 = f1;
                f1 = a;
            }
        }
    }
}

// Per-base amounts (start pieces plus end pieces), one thread per column.
__global__ void flankUnifyKernel(const AlignJob *jobs, const PairScales *scales, NullRates nr, XS *work) {
    const int t = blockIdx.y;
    const AlignJob jb = jobs[t];
    const int L = jb.L;
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= L) return;
    const PairScales sc = scales[jb.pair];
    const FlankRates r = flankRates(nr);
    const XS aS1 = splitNorm((double)sc.s1, 0), aS2 = splitNorm((double)sc.s2, 0), aSC = splitNorm((double)sc.sC, 0);
    const XS bS1 = scaleScore(aS1, 4.0), bS2 = scaleScore(aS2, 16.0);
    const XS *bgx = flankArray(work, jb, t, kFBg);
    const XS *mid = flankArray(work, jb, t, kFMid), *rest = flankArray(work, jb, t, kFRest);
    const XS *fa = flankArray(work, jb, t, kFArrival);
    XS total = scalarMul(ldXS(mid + j), ldXS(flankArray(work, jb, t, kFWeighted) + j));
    const XS rn = ldXS(rest + j + 1);
    if (j >= 1) {
        const XS exit1 = scalarMul(scaleScore(rn, r.sr), aS1);
        total = scalarAdd(total, scalarMul(ldXS(fa + j - 1), exit1));
    }
    if (j >= 2) {
        const XS exit2 = scalarMul(scaleScore(rn, r.dr), aS2);
        total = scalarAdd(total, scaleScore(scalarMul(ldXS(fa + j - 2), exit2), 2.0));
    }
    if (j >= 3) {
        const XS exit3 = scalarMul(scaleScore(scalarMul(rn, aSC), r.keep), ldXS(bgx + j - 2));
        total = scalarAdd(total, scaleScore(scalarMul(ldXS(fa + j - 3), exit3), 3.0));
    }
    if (j == L - 1) {  // leftover endings at the last base
        const XS f1 = ldXS(fa + j - 1);
        total = scalarAdd(total, scaleScore(scalarMul(f1, scaleScore(bS1, r.dr * 0.25)), 2.0));
        total = scalarAdd(total, scaleScore(scalarMul(f1, scaleScore(bS1, r.keep * 0.25)), 3.0));
        if (j - 2 >= 0)
            total = scalarAdd(total, scaleScore(scalarMul(ldXS(fa + j - 2), scaleScore(bS2, r.keep * 0.0625)), 3.0));
    }
    stXS(flankArray(work, jb, t, kFUnified) + j, scaleScore(total, r.third));
}

// The entry totals (running forward, warp 0) and the exit totals (running
// backward, warp 1) with their largest exponents.
__global__ void flankSumKernel(const AlignJob *jobs, const XS *work, int *rows, XS *revEv, XS *fwdEv) {
    const int t = blockIdx.x;
    if ((threadIdx.x & 31) != 0) return;
    const int w = threadIdx.x >> 5;
    const AlignJob jb = jobs[t];
    const int L = jb.L;
    const XS *__restrict__ u = flankArray(const_cast<XS *>(work), jb, t, kFUnified);
    int *sideMax = rows + jb.rowOff + 3 * (jb.M + 2);
    XS cum = xsZero();
    int mx = INT_MIN;
    if (w == 0) {
        XS *__restrict__ rev = revEv + jb.colOff;
        for (int lo = 0; lo < L; lo += kFlankAhead) {
            XS v[kFlankAhead];
#pragma unroll
            for (int q = 0; q < kFlankAhead; ++q) v[q] = lo + q < L ? ldXS(u + lo + q) : xsZero();
#pragma unroll
            for (int q = 0; q < kFlankAhead; ++q) {
                if (lo + q >= L) break;
                cum = scalarAdd(cum, v[q]);
                stXS(rev + lo + q, cum);
                if (cum.m != 0.0f && cum.e > mx) mx = cum.e;
            }
        }
        sideMax[0] = mx;
    } else if (w == 1) {
        XS *__restrict__ fwd = fwdEv + jb.colOff;
        for (int hi = L - 1; hi >= 0; hi -= kFlankAhead) {
            XS v[kFlankAhead];
#pragma unroll
            for (int q = 0; q < kFlankAhead; ++q) v[q] = hi - q >= 0 ? ldXS(u + hi - q) : xsZero();
#pragma unroll
            for (int q = 0; q < kFlankAhead; ++q) {
                if (hi - q < 0) break;
                cum = scalarAdd(cum, v[q]);
                stXS(fwd + hi - q, cum);
                if (cum.m != 0.0f && cum.e > mx) mx = cum.e;
            }
        }
        sideMax[1] = mx;
    }
}

// X table, one thread per (job, column, group of kXRows rows).
constexpr int kXRows = 8;
__global__ void xTableKernel(const AlignJob *jobs, const DevPair *pairs, const DevProfile *profiles, const float *emit,
                             const float *params, const uint8_t *codes, const PairScales *scales, const float *cells,
                             int *rows, XS *X) {
    const AlignJob jb = jobs[blockIdx.z];
    const int M = jb.M, L = jb.L;
    const int i0 = blockIdx.y * kXRows;
    if (i0 > M) return;
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    const DevPair p = pairs[jb.pair];
    const DevProfile &pr = profiles[p.prof];
    const float sC = scales[jb.pair].sC;
    const int *cntB = rows + jb.rowOff, *cntF = cntB + (M + 2);
    int *rowMaxX = rows + jb.rowOff + 2 * (M + 2);
    const float *W0 = cells + 2 * jb.cellOff;
    const float *W1 = W0 + (size_t)(M + 1) * L;
    const int code = (j >= 2 && j < L) ? (int)codes[p.codeOff + j - 2] : kPad;
    const float *em = emit + pr.emitOff + (size_t)code * pr.rowPad;
    for (int i = i0; i < i0 + kXRows && i <= M; ++i) {
        int e = INT_MIN;
        if (j < L) {
            const float enter = __fmul_rn(params[pr.paramOff + (size_t)i * kParamFloats + 10], sC);
            const float w3 = j >= 3 ? W0[(size_t)i * L + j - 3] : 0.0f;
            const float xf = __fmul_rn(__fmul_rn(enter, em[i]), w3);
            float w1n = 0.0f;
            if (i + 1 <= M) w1n = __fmul_rn(W1[(size_t)(i + 1) * L + j], stepsDown(cntB[i + 1] - cntB[i + 2]));
            const XS x = planeMul(promote(xf, cntF[i]), promote(w1n, cntB[i + 1]));
            stXS(X + jb.cellOff + (size_t)i * L + j, x);
            if (x.m != 0.0f) e = x.e;
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) e = max(e, __shfl_xor_sync(0xffffffffu, e, o));
        if ((threadIdx.x & 31) == 0 && e != INT_MIN) atomicMax(rowMaxX + i, e);
    }
}

// Max scans over a row of kOptThreads x kOptPer columns at a time.
constexpr int kOptThreads = 512;
constexpr int kOptPer = 8;

// Exclusive max of the threads' values in thread order (reverse: from the
// last thread down); all values >= 0, and 0 where nothing comes before.
__device__ __forceinline__ float blockExclusiveMax(float v, float *sm, bool reverse) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    constexpr int nw = kOptThreads / 32;
    float incl = v;
    if (!reverse) {
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const float t = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl = fmaxf(incl, t);
        }
    } else {
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const float t = __shfl_down_sync(0xffffffffu, incl, o);
            if (lane + o < 32) incl = fmaxf(incl, t);
        }
    }
    if (reverse ? lane == 0 : lane == 31) sm[warp] = incl;
    __syncthreads();
    float before = 0.0f;
    if (!reverse) {
        for (int w = 0; w < warp; ++w) before = fmaxf(before, sm[w]);
        const float t = __shfl_up_sync(0xffffffffu, incl, 1);
        if (lane >= 1) before = fmaxf(before, t);
    } else {
        for (int w = warp + 1; w < nw; ++w) before = fmaxf(before, sm[w]);
        const float t = __shfl_down_sync(0xffffffffu, incl, 1);
        if (lane + 1 < 32) before = fmaxf(before, t);
    }
    __syncthreads();
    return before;
}

// Prefix- and suffix-optimal tables of one job per CTA
// (dummest-dp-forward.hh:295-451).  The prefix table overwrites the job's W0
// and W1 (no longer read); the suffix table has its own array.
__global__ void __launch_bounds__(kOptThreads) optimalKernel(const AlignJob *jobs, float *cells, const int *rows,
                                                             const XS *X, const XS *revEv, const XS *fwdEv,
                                                             XS *suffix) {
    __shared__ float sm[kOptThreads / 32];
    __shared__ float carry;
    const AlignJob jb = jobs[blockIdx.x];
    const int M = jb.M, L = jb.L;
    const int *rowMaxX = rows + jb.rowOff + 2 * (M + 2);
    const int revMax = rows[jb.rowOff + 3 * (M + 2)], fwdMax = rows[jb.rowOff + 3 * (M + 2) + 1];
    XS *pre = reinterpret_cast<XS *>(cells + 2 * jb.cellOff);
    const XS *Xj = X + jb.cellOff;
    XS *suf = suffix + jb.cellOff;
    const XS *rev = revEv + jb.colOff, *fwd = fwdEv + jb.colOff;
    constexpr int chunk = kOptThreads * kOptPer;

    // prefix-optimal: rows 0..M, each a running maximum left to right
    int runMax = INT_MIN;
    for (int i = 0; i <= M; ++i) {
        runMax = max(runMax, rowMaxX[i]);
        const int E = max(runMax, revMax) + 1;
        if (threadIdx.x == 0) carry = 0.0f;
        __syncthreads();
        for (int c0 = 0; c0 < L; c0 += chunk) {
            float v[kOptPer];
            float run = 0.0f;
            const int jb0 = c0 + threadIdx.x * kOptPer;
#pragma unroll
            for (int q = 0; q < kOptPer; ++q) {
                const int j = jb0 + q;
                float cand = 0.0f;
                if (j < L) {
                    const float comb = toRow(ldXS(Xj + (size_t)i * L + j), E);
                    const float rs = toRow(ldXS(rev + j), E);
                    if (i == 0) {
                        cand = fmaxf(comb, rs);
                    } else {
                        const XS *pp = pre + (size_t)(i - 1) * L;
                        const float up = toRow(ldXS(pp + j), E);
                        const float succ = j >= 3 ? toRow(ldXS(pp + j - 3), E) : 0.0f;
                        cand = fmaxf(fmaxf(up, __fadd_rn(comb, succ)), rs);
                    }
                }
                run = fmaxf(run, cand);
                v[q] = run;
            }
            const float before = fmaxf(blockExclusiveMax(run, sm, false), carry);
            __syncthreads();  // every thread has read carry
#pragma unroll
            for (int q = 0; q < kOptPer; ++q) {
                const int j = jb0 + q;
                if (j < L) stXS(pre + (size_t)i * L + j, fromRow(fmaxf(before, v[q]), E));
            }
            if (threadIdx.x == kOptThreads - 1) carry = fmaxf(before, run);
            __syncthreads();
        }
    }
    // suffix-optimal: rows M..0, each a running maximum right to left
    runMax = INT_MIN;
    const int nChunks = (L + chunk - 1) / chunk;
    for (int i = M; i >= 0; --i) {
        runMax = max(runMax, rowMaxX[i]);
        const int E = max(runMax, fwdMax) + 1;
        if (threadIdx.x == 0) carry = 0.0f;
        __syncthreads();
        for (int cc = nChunks - 1; cc >= 0; --cc) {
            const int c0 = cc * chunk;
            float v[kOptPer];
            float run = 0.0f;
            const int jb0 = c0 + threadIdx.x * kOptPer;
#pragma unroll
            for (int q = kOptPer - 1; q >= 0; --q) {
                const int j = jb0 + q;
                float cand = 0.0f;
                if (j < L) {
                    const float fs = toRow(ldXS(fwd + j), E);
                    if (i == M) {
                        cand = fs;
                    } else {
                        const XS *np = suf + (size_t)(i + 1) * L;
                        const float down = toRow(ldXS(np + j), E);
                        float cps = 0.0f;
                        if (j + 3 < L)
                            cps = __fadd_rn(toRow(ldXS(Xj + (size_t)i * L + j + 3), E), toRow(ldXS(np + j + 3), E));
                        cand = fmaxf(fmaxf(down, fs), cps);
                    }
                }
                run = fmaxf(run, cand);
                v[q] = run;
            }
            const float after = fmaxf(blockExclusiveMax(run, sm, true), carry);
            __syncthreads();
#pragma unroll
            for (int q = 0; q < kOptPer; ++q) {
                const int j = jb0 + q;
                if (j < L) stXS(suf + (size_t)i * L + j, fromRow(fmaxf(after, v[q]), E));
            }
            if (threadIdx.x == 0) carry = fmaxf(after, run);
            __syncthreads();
        }
    }
}

struct Seg {
    int start1, start2, length;
};

// A candidate's walks in brief: its sequence span [beg, end) (before the
// clamp to [0, L)) and its forward and reverse match counts.
struct WalkSpan {
    int beg, end, nf, nr;
};

// One anchor's walks (dummest-traceback.hh:35-118): forward from (anchor1,
// anchor2) over the suffix-optimal table, then backward from (anchor1 - 1,
// anchor2) over the prefix-optimal table, with the reference's merging of
// adjacent matches.  The alignment is the reverse matches, last found first,
// then the forward ones; addForwardMatch consults only the last forward
// match and addReverseMatch only the current first segment, so the walk keeps
// those in registers.  STORE: the segments go to out[0, nr + nf), with nrKnown
// the reverse match count (from the span pass): forward match q at
// out[nrKnown + q], reverse match q at out[nrKnown - 1 - q].
template <bool STORE>
__device__ WalkSpan walkAnchor(const AlignJob &jb, int a1, int a2, const XS *pre, const XS *Xj, const XS *suf,
                               const XS *rev, const XS *fwd, Seg *out, int nrKnown) {
    const int M = jb.M, L = jb.L;
    auto S = [&](int i, int j) { return (i <= M && j < L) ? ldXS(suf + (size_t)i * L + j) : xsZero(); };
    auto P = [&](int i, int j) { return ldXS(pre + (size_t)i * L + j); };
    Seg fFirst{0, 0, 0}, fLast{0, 0, 0}, rFirst{0, 0, 0}, rFront{0, 0, 0};
    int nf = 0, nr = 0;
    {
        int i = a1, pos = a2;
        while (i <= M && pos < L) {
            XS best = xsZero();
            int bi = INT_MAX, bj = INT_MAX;
            bool emit = false;
            if (pos + 3 < L) {
                const XS cd = scalarAdd(ldXS(Xj + (size_t)i * L + pos + 3), S(i + 1, pos + 3));
                if (scoreLess(best, cd)) { best = cd; bi = i + 1; bj = pos + 3; emit = true; }
            }
            XS cd = S(i + 1, pos);
            if (scoreLess(best, cd)) { best = cd; bi = i + 1; bj = pos; emit = false; }
            cd = S(i, pos + 1);
            if (scoreLess(best, cd)) { best = cd; bi = i; bj = pos + 1; emit = false; }
            cd = ldXS(fwd + pos);
            if (scoreLess(best, cd)) { best = cd; bi = INT_MAX; bj = INT_MAX; emit = false; }
            if (emit) {  // addForwardMatch(i, pos + 1)
                const int p1 = i, p2 = pos + 1;
                bool add = true;
                if (nf > 0) {
                    Seg &x = fLast;
                    if (x.start1 + x.length == p1 && x.start2 + x.length == p2) ++x.length;
                    if (x.start1 + x.length > p1 || x.start2 + x.length > p2) add = false;
                    if (nf == 1) fFirst = fLast;
                    if (STORE) out[nrKnown + nf - 1] = fLast;
                }
                if (add) {
                    const Seg s{p1, p2, 1};
                    if (nf == 0) fFirst = s;
                    fLast = s;
                    if (STORE) out[nrKnown + nf] = s;
                    ++nf;
                }
            }
            i = bi;
            pos = bj;
        }
    }
    {
        int i = a1 - 1, pos = a2;
        while (i >= 0 && pos >= 0) {
            XS best = xsZero();
            int bi = -1, bj = -1;
            bool emit = false;
            if (pos >= 3) {
                const XS succ = i >= 1 ? P(i - 1, pos - 3) : xsZero();
                const XS cd = scalarAdd(ldXS(Xj + (size_t)i * L + pos), succ);
                if (scoreLess(best, cd)) { best = cd; bi = i - 1; bj = pos - 3; emit = true; }
            }
            if (i >= 1) {
                const XS cd = P(i - 1, pos);
                if (scoreLess(best, cd)) { best = cd; bi = i - 1; bj = pos; emit = false; }
            }
            if (pos > 0) {
                const XS cd = P(i, pos - 1);
                if (scoreLess(best, cd)) { best = cd; bi = i; bj = pos - 1; emit = false; }
            }
            const XS cd = ldXS(rev + pos);
            if (scoreLess(best, cd)) { best = cd; bi = -1; bj = -1; emit = false; }
            if (emit) {  // addReverseMatch(i, pos - 2)
                const int p1 = i, p2 = pos - 2;
                bool add = true;
                if (nr > 0 || nf > 0) {
                    Seg &x = nr > 0 ? rFront : fFirst;
                    if (x.start1 - 1 == p1 && x.start2 - 1 == p2) {
                        --x.start1;
                        --x.start2;
                        ++x.length;
                    }
                    if (x.start1 <= p1 || x.start2 <= p2) add = false;
                    if (nr > 0) {
                        if (nr == 1) rFirst = rFront;
                        if (STORE) out[nrKnown - nr] = rFront;
                    } else {
                        if (nf == 1) fLast = fFirst;
                        if (STORE) out[nrKnown] = fFirst;
                    }
                }
                if (add) {
                    const Seg s{p1, p2, 1};
                    if (nr == 0) rFirst = s;
                    rFront = s;
                    ++nr;
                    if (STORE) out[nrKnown - nr] = s;
                }
            }
            i = bi;
            pos = bj;
        }
    }
    WalkSpan w;
    w.nf = nf;
    w.nr = nr;
    if (nf + nr == 0) {
        w.beg = w.end = a2;
    } else {
        w.beg = nr > 0 ? rFront.start2 : fFirst.start2;
        w.end = nf > 0 ? fLast.start2 + fLast.length : rFirst.start2 + rFirst.length;
    }
    return w;
}

// The span pass: every candidate of every job at once, one thread each
// (grid.y = job); spans[colOff + c] for candidate c.
__global__ void spanKernel(const AlignJob *jobs, const int *cand, const int *anchorRow, const float *cells,
                           const XS *X, const XS *suffix, const XS *revEv, const XS *fwdEv, WalkSpan *spans) {
    const AlignJob jb = jobs[blockIdx.y];
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= jb.nCand) return;
    const int a2 = cand[jb.colOff + c];
    const int a1 = anchorRow[jb.colOff + a2];
    spans[jb.colOff + c] = walkAnchor<false>(jb, a1, a2, reinterpret_cast<const XS *>(cells + 2 * jb.cellOff),
                                             X + jb.cellOff, suffix + jb.cellOff, revEv + jb.colOff,
                                             fwdEv + jb.colOff, nullptr, 0);
}

// An accepted candidate whose segments are written.
struct WalkItem {
    int job, anchor2, nr, pad;
    long long segOff;  // in the output segment list
};

// The store pass: the accepted candidates' walks again, segments written in
// place (the walks are deterministic, so the counts are the span pass's).
__global__ void storeWalkKernel(const AlignJob *jobs, const WalkItem *items, int nItems, const int *anchorRow,
                                const float *cells, const XS *X, const XS *suffix, const XS *revEv,
                                const XS *fwdEv, Seg *segOut) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= nItems) return;
    const WalkItem it = items[t];
    const AlignJob jb = jobs[it.job];
    const int a1 = anchorRow[jb.colOff + it.anchor2];
    walkAnchor<true>(jb, a1, it.anchor2, reinterpret_cast<const XS *>(cells + 2 * jb.cellOff), X + jb.cellOff,
                     suffix + jb.cellOff, revEv + jb.colOff, fwdEv + jb.colOff, segOut + it.segOff, it.nr);
}

}  // namespace dmst
