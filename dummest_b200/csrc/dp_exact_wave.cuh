// Exact row-rescaled DP on the wavefront, one warp per pair (one row per
// lane), for the pairs the fast kernel cannot score exactly (a row maximum
// above RESCALE_THRESH, or a product beyond float range).
//
// The reference decides each row's rescale after the whole row is known
// (dummest-dp-backward.hh:560-573, dummest-dp-forward.hh:228-242), which a
// wavefront cannot wait for.  So each direction runs twice:
//
//  1. discovery: the same recurrence with a per-lane scale count that rises
//     by one (values x 2^-64, exact) whenever a value passes 2^100, and that
//     lanes align when they exchange values.  Every operation then sees the
//     reference's operands up to an exact power of two, so each row's
//     maximum is the reference's up to that power; the row's (max, count)
//     is recorded.  A scan over the rows turns these into the reference's
//     own counts: cnt_i = cnt_prev + [max_i * 2^(64 (count_i - cnt_prev)) > 1e30].
//  2. replay: the reference's arithmetic exactly, with those counts known in
//     advance: row i computes at the scale of the row it reads, seeds times
//     2^(-64 cnt_prev), and multiplies everything it hands on (stored W1, the
//     values sent to the next row) by 2^-64 when its own count rose.
//
// Mid and filter maxima are taken over exact double products (the reference
// forms them in double and rounds the mantissa to float,
// dummest-batch.hh:146-235) and folded with the row's count sum into an
// exact (mantissa, exponent) best.
#pragma once

#include "dp_wavefront.cuh"

namespace dmst {

constexpr float kBump = 0x1p100f;          // discovery: rescale a lane above this
constexpr float kStep = 0x1p-64f;           // one rescale step, RESCALE_STEP

__device__ __forceinline__ float stepsDown(int d) {  // 2^(-64 d), d >= 0, flushes to 0 past float range
    return d == 0 ? 1.0f : (d == 1 ? kStep : 0.0f);
}

// Seed coefficient of a row at scale count c: scale * 2^(-64 c), a float that
// flushes to zero from c = 2 on (rowRescaleVector, dummest-score.hh:145-152).
__device__ __forceinline__ float seedCoef(float rs, int c) { return rs * (c == 0 ? 1.0f : (c == 1 ? kStep : 0.0f)); }

struct ExactBest {  // exact (double mantissa, binary exponent) maximum
    double m;
    int e;
};

__device__ __forceinline__ void foldBest(ExactBest &b, double v, int countSum) {
    if (!(v > 0.0)) return;
    int e;
    double m = frexp(v, &e);
    e += kRescaleBits * countSum;
    if (b.m == 0.0 || e > b.e || (e == b.e && m > b.m)) {
        b.m = m;
        b.e = e;
    }
}

struct ExactArgs {
    SweepArgs a;          // R = 1 geometry; a.w1 / a.ring point into the pair's scratch
    float *rowMax;        // M+1 (discovery)
    int *rowCnt;          // M+1 (discovery)
    int *cntB;            // M+2: reference backward counts (cntB[M+1] = 0)
    int *cntF;            // M+2: reference forward counts, cntF[i+1] holds row i (cntF[0] = 0)
};

// ---------------------------------------------------------------------------
// Backward sweep, R = 1.  DISCOVER: dynamic counts, record row maxima.
// Otherwise replay with cntB, store W1, exact filter best.
// ---------------------------------------------------------------------------
template <bool DISCOVER>
__device__ void exactBackward(const ExactArgs &x, int lane, ExactBest &filt) {
    const SweepArgs &a = x.a;
    Coef<1> c;
    float h1 = 0, h2 = 0, h3 = 0, z1 = 0, z2 = 0, z3 = 0, rb1 = 0, rb2 = 0, rb3 = 0, rmax = 0;
    int cnt = 0, cOut = 0;
    float rs = 0, fOut = 1;
    double rowBestF = 0;  // replay: this row's max W1*prefixSeed
    float sendW = 0, sendY = 0;
    int sendC = 0;
    const int L = a.L, P = a.P, nS = a.nS;
    const int T = nS * P + (kLanes - 1);
    int u = -(kLanes - 1 - lane), sp = 0, jj = 0;
    for (int t = 0; t < T; ++t, ++u) {
        float inW = __shfl_down_sync(kFull, sendW, 1);
        float inY = __shfl_down_sync(kFull, sendY, 1);
        int inC = __shfl_down_sync(kFull, sendC, 1);
        const bool act = (u >= 0) && (sp < nS) && (jj < L);
        if (act) {
            const int s = nS - 1 - sp;
            const int j = L - 1 - jj;
            const int i = s * kLanes + lane;  // this lane's row
            if (jj == 0) {
                loadBackwardCoef<1>(c, a, i);
                h1 = h2 = h3 = z1 = z2 = z3 = rb1 = rb2 = rb3 = rmax = 0;
                rowBestF = 0;
                if (DISCOVER) {
                    cnt = 0;
                } else {
                    const int ci = i <= a.M ? i : a.M + 1;
                    cnt = x.cntB[ci + 1 <= a.M + 1 ? ci + 1 : a.M + 1];
                    cOut = x.cntB[ci];
                    fOut = stepsDown(cOut - cnt);
                }
                rs = seedCoef(c.rs[0], cnt);
            }
            if (lane == kLanes - 1) {
                if (sp > 0) {
                    inW = __ldcg(a.ring + 3 * jj);
                    inY = __ldcg(a.ring + 3 * jj + 1);
                    inC = __float_as_int(__ldcg(a.ring + 3 * jj + 2));
                } else {
                    inW = inY = 0.0f;
                    inC = 0;
                }
            }
            if (DISCOVER) {
                if (inC > cnt) {
                    const float f = stepsDown(inC - cnt);
                    h1 *= f; h2 *= f; h3 *= f; z1 *= f; z2 *= f; z3 *= f;
                    rb1 *= f; rb2 *= f; rb3 *= f; rmax *= f;
                    cnt = inC;
                    rs = seedCoef(c.rs[0], cnt);
                } else if (inC < cnt) {
                    const float f = stepsDown(cnt - inC);
                    inW *= f;
                    inY *= f;
                }
            }
            const int code = (j + 1 < L) ? (int)__ldg(a.codes + j + 1) : kPad;
            const float bgv = a.smBg[code];
            const float e = a.smE[code * a.rowPad + i];
            const float sufv = __ldg(a.suf + j);
            float acc = (rb3 * e) * c.enter[0];
            acc = __fmaf_rn(inY, c.d0[0], acc);
            acc = __fmaf_rn(rb2, c.d1[0], acc);
            acc = __fmaf_rn(rb1, c.d2[0], acc);
            const float zbg = z3 * bgv;
            acc = __fmaf_rn(zbg, c.a0[0], acc);
            acc = __fmaf_rn(h2, c.a2[0], acc);
            acc = __fmaf_rn(h1, c.a1[0], acc);
            float W = __fmaf_rn(sufv, rs, acc);
            float Y = __fmaf_rn(c.eps[0], inY, W);
            const float Z = __fmaf_rn(c.b0[0], zbg, W);
            rb3 = rb2; rb2 = rb1; rb1 = inW;
            h3 = h2; h2 = h1; h1 = W;
            z3 = z2; z2 = z1; z1 = Z;
            if (DISCOVER) {
                rmax = fmaxf(rmax, fmaxf(W, Y));
                if (fmaxf(W, Y) > kBump) {
                    h1 *= kStep; h2 *= kStep; h3 *= kStep; z1 *= kStep; z2 *= kStep; z3 *= kStep;
                    rb1 *= kStep; rb2 *= kStep; rb3 *= kStep; rmax *= kStep;
                    W *= kStep;
                    Y *= kStep;
                    ++cnt;
                    rs = seedCoef(c.rs[0], cnt);
                }
                sendW = W;
                sendY = Y;
                sendC = cnt;
                if (jj == L - 1 && i <= a.M) {
                    x.rowMax[i] = rmax;
                    x.rowCnt[i] = cnt;
                }
            } else {
                const float Wo = W * fOut, Yo = Y * fOut;
                a.w1[((size_t)s * a.D + jj + (kLanes - 1 - lane)) * kLanes + lane] = Wo;
                rowBestF = fmax(rowBestF, (double)Wo * (double)__ldg(a.pre + j));
                if (jj == L - 1 && i <= a.M) foldBest(filt, rowBestF, cOut);
                sendW = Wo;
                sendY = Yo;
                sendC = cOut;
            }
            if (lane == 0 && sp < nS - 1) {
                __stcg(a.ring + 3 * jj, sendW);
                __stcg(a.ring + 3 * jj + 1, sendY);
                __stcg(a.ring + 3 * jj + 2, __int_as_float(sendC));
            }
        } else {
            sendW = sendY = 0.0f;
            sendC = 0;
        }
        if (u >= 0 && ++jj == P) {
            jj = 0;
            ++sp;
        }
        __syncwarp();
    }
}

// ---------------------------------------------------------------------------
// Forward sweep, R = 1.  DISCOVER: dynamic counts, record row maxima of W0/Y0.
// Otherwise replay with cntF and take the exact mid maximum.
// ---------------------------------------------------------------------------
template <bool DISCOVER>
__device__ void exactForward(const ExactArgs &x, int lane, ExactBest &mid) {
    const SweepArgs &a = x.a;
    Coef<1> c;
    float w1 = 0, w2 = 0, w3 = 0, z1 = 0, z2 = 0, z3 = 0, rmax = 0;
    int cnt = 0, cOut = 0, cB = 0;
    float rs = 0, fOut = 1;
    double rowBest = 0;
    float sendIn = 0, sendY = 0;
    int sendC = 0;
    const int L = a.L, P = a.P, nS = a.nS;
    const int T = nS * P + (kLanes - 1);
    int u = -lane, s = 0, j = 0;
    for (int t = 0; t < T; ++t, ++u) {
        float inW = __shfl_up_sync(kFull, sendIn, 1);
        float inY = __shfl_up_sync(kFull, sendY, 1);
        int inC = __shfl_up_sync(kFull, sendC, 1);
        const bool act = (u >= 0) && (s < nS) && (j < L);
        if (act) {
            const int i = s * kLanes + lane;
            if (j == 0) {
                loadForwardCoef<1>(c, a, i);
                w1 = w2 = w3 = z1 = z2 = z3 = rmax = 0;
                rowBest = 0;
                if (DISCOVER) {
                    cnt = 0;
                } else {
                    const int ci = i <= a.M ? i : a.M;
                    cnt = x.cntF[ci];      // count of row i-1 (inherited)
                    cOut = x.cntF[ci + 1]; // count of row i after its decision
                    fOut = stepsDown(cOut - cnt);
                    cB = x.cntB[ci];
                }
                rs = seedCoef(c.rs[0], cnt);
            }
            if (lane == 0) {
                if (s > 0) {
                    inW = __ldcg(a.ring + 3 * j);
                    inY = __ldcg(a.ring + 3 * j + 1);
                    inC = __float_as_int(__ldcg(a.ring + 3 * j + 2));
                } else {
                    inW = inY = 0.0f;
                    inC = 0;
                }
            }
            if (DISCOVER) {
                if (inC > cnt) {
                    const float f = stepsDown(inC - cnt);
                    w1 *= f; w2 *= f; w3 *= f; z1 *= f; z2 *= f; z3 *= f; rmax *= f;
                    cnt = inC;
                    rs = seedCoef(c.rs[0], cnt);
                } else if (inC < cnt) {
                    const float f = stepsDown(cnt - inC);
                    inW *= f;
                    inY *= f;
                }
            }
            const int code = (j >= 2) ? (int)__ldg(a.codes + j - 2) : kPad;
            const float bgsC = a.smBg[code] * a.sc.sC;
            const float e = a.smE[code * a.rowPad + i];
            const float prev = __ldg(a.pre + j);
            const float X = (c.enter[0] * e) * w3;
            const float Z0 = bgsC * __fmaf_rn(c.a0[0], w3, c.b0[0] * z3);
            const float Z1 = c.a1[0] * w1;
            const float Z2 = c.a2[0] * w2;
            const float W0 = inW + __fmaf_rn(prev, rs, (Z0 + Z1) + Z2);
            float Y0 = __fmaf_rn(c.d0[0], W0, c.eps[0] * inY);
            float nin = __fmaf_rn(c.d2[0], w1, __fmaf_rn(c.d1[0], w2, X + Y0));
            if (!DISCOVER) {
                const float wb = __ldcg(a.w1 + ((size_t)s * a.D + (L - 1 - j) + (kLanes - 1 - lane)) * kLanes + lane);
                rowBest = fmax(rowBest, (double)W0 * (double)wb);
            }
            w3 = w2; w2 = w1; w1 = W0;
            z3 = z2; z2 = z1; z1 = Z0;
            if (DISCOVER) {
                rmax = fmaxf(rmax, fmaxf(W0, Y0));
                if (fmaxf(fmaxf(W0, Y0), nin) > kBump) {
                    w1 *= kStep; w2 *= kStep; w3 *= kStep; z1 *= kStep; z2 *= kStep; z3 *= kStep;
                    rmax *= kStep;
                    nin *= kStep;
                    Y0 *= kStep;
                    ++cnt;
                    rs = seedCoef(c.rs[0], cnt);
                }
                sendIn = nin;
                sendY = Y0;
                sendC = cnt;
                if (j == L - 1 && i <= a.M) {
                    x.rowMax[i] = rmax;
                    x.rowCnt[i] = cnt;
                }
            } else {
                if (j == L - 1 && i <= a.M) foldBest(mid, rowBest, cnt + cB);
                sendIn = nin * fOut;
                sendY = Y0 * fOut;
                sendC = cOut;
            }
            if (lane == kLanes - 1 && s < nS - 1) {
                __stcg(a.ring + 3 * j, sendIn);
                __stcg(a.ring + 3 * j + 1, sendY);
                __stcg(a.ring + 3 * j + 2, __int_as_float(sendC));
            }
        } else {
            sendIn = sendY = 0.0f;
            sendC = 0;
        }
        if (u >= 0 && ++j == P) {
            j = 0;
            ++s;
        }
        __syncwarp();
    }
}

__device__ __forceinline__ ExactBest warpBest(ExactBest b) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        double m = __shfl_xor_sync(kFull, b.m, o);
        int e = __shfl_xor_sync(kFull, b.e, o);
        if (m != 0.0 && (b.m == 0.0 || e > b.e || (e == b.e && m > b.m))) {
            b.m = m;
            b.e = e;
        }
    }
    return b;
}

// Reference counts from the discovery maxima, scanned in the reference's row
// order (backward: M..0 from cnt = 0; forward: 0..M).  One lane.
__device__ void scanCounts(const float *rowMax, const int *rowCnt, int *cnt, int M, bool backward) {
    if (backward) {
        cnt[M + 1] = 0;
        for (int i = M; i >= 0; --i) {
            int d = rowCnt[i] - cnt[i + 1];
            d = d > 15 ? 15 : (d < -15 ? -15 : d);
            const double pre = ldexp((double)rowMax[i], kRescaleBits * d);
            cnt[i] = cnt[i + 1] + (pre > (double)kRescaleThresh ? 1 : 0);
        }
    } else {
        cnt[0] = 0;
        for (int i = 0; i <= M; ++i) {
            int d = rowCnt[i] - cnt[i];
            d = d > 15 ? 15 : (d < -15 ? -15 : d);
            const double pre = ldexp((double)rowMax[i], kRescaleBits * d);
            cnt[i + 1] = cnt[i] + (pre > (double)kRescaleThresh ? 1 : 0);
        }
    }
}

struct ExactWaveJob {
    int pair;
    int pad;
    long long scratchOff;  // float offset of this job's scratch
};

// Scratch per job (floats): W1 nS*D*32, ring 3*P, rowMax M+1, rowCnt M+1,
// cntB M+2, cntF M+2.
__host__ __device__ inline long long exactWaveScratch(int M, int L) {
    const long long nS = (M + 1 + kLanes - 1) / kLanes;
    const long long P = L > kLanes ? L : kLanes;
    const long long D = P + kLanes - 1;
    return nS * D * kLanes + 3 * P + 2LL * (M + 1) + 2LL * (M + 2) + 64;
}

__global__ void __launch_bounds__(kLanes) exactWaveKernel(const ExactWaveJob *jobs, int n, const DevPair *pairs,
                                                           const DevProfile *profiles, const float *emit,
                                                           const float *params, const uint8_t *codes,
                                                           const float *seeds, const PairScales *scales,
                                                           float *scratch, ExactOut *out) {
    extern __shared__ float4 smRaw[];
    float *smE = reinterpret_cast<float *>(smRaw);
    __shared__ float smBg[32];
    const int lane = threadIdx.x;
    for (int ji = blockIdx.x; ji < n; ji += gridDim.x) {
        const ExactWaveJob job = jobs[ji];
        const DevPair p = pairs[job.pair];
        const DevProfile &pr = profiles[p.prof];
        const int rowPad = pr.rowPad;
        __syncwarp();
        {
            const float4 *src = reinterpret_cast<const float4 *>(emit + pr.emitOff);
            const int n4 = kNumCodes * rowPad / 4;
            for (int k = lane; k < n4; k += kLanes) smRaw[k] = __ldg(src + k);
            smBg[lane] = lane < kNumCodes ? pr.bg[lane] : 0.0f;
        }
        __syncwarp();
        ExactArgs x;
        SweepArgs &a = x.a;
        a.codes = codes + p.codeOff;
        a.pre = seeds + p.seedOff;
        a.suf = a.pre + p.L;
        a.params = params + pr.paramOff;
        a.smE = smE;
        a.smBg = smBg;
        a.sc = scales[job.pair];
        a.L = p.L;
        a.M = p.M;
        a.rowPad = rowPad;
        a.nS = (p.M + 1 + kLanes - 1) / kLanes;
        a.P = p.L > kLanes ? p.L : kLanes;
        a.D = a.P + kLanes - 1;
        float *base = scratch + job.scratchOff;
        a.w1 = base;
        a.ring = base + (size_t)a.nS * a.D * kLanes;
        x.rowMax = a.ring + 3 * (size_t)a.P;
        x.rowCnt = reinterpret_cast<int *>(x.rowMax + (p.M + 1));
        x.cntB = x.rowCnt + (p.M + 1);
        x.cntF = x.cntB + (p.M + 2);
        ExactBest filt{0.0, 0}, mid{0.0, 0};
        exactBackward<true>(x, lane, filt);
        __syncwarp();
        if (lane == 0) scanCounts(x.rowMax, x.rowCnt, x.cntB, p.M, true);
        __syncwarp();
        exactForward<true>(x, lane, mid);
        __syncwarp();
        if (lane == 0) scanCounts(x.rowMax, x.rowCnt, x.cntF, p.M, false);
        __syncwarp();
        exactBackward<false>(x, lane, filt);
        __syncwarp();
        exactForward<false>(x, lane, mid);
        filt = warpBest(filt);
        mid = warpBest(mid);
        if (lane == 0) {
            ExactOut o;
            o.mid = mid.m == 0.0 ? xsZero() : XS{__double2float_rn(mid.m), mid.e};
            o.filt = filt.m == 0.0 ? xsZero() : XS{__double2float_rn(filt.m), filt.e};
            out[ji] = o;
        }
        __syncwarp();
    }
}

}  // namespace dmst
