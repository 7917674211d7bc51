// The batched wavefront DP: one warp per (read, profile) pair.
//
// Layout.  The profile's rows are striped across the 32 lanes of a warp: a
// stripe is S = 32*R consecutive rows, lane l owns rows l*R .. l*R+R-1 of the
// stripe (R = 1, 2 or 4).  All R rows of a lane sit at the same column in a
// step, and lane l lags lane l-1 (forward) or l+1 (backward) by one column,
// so every cell's row-boundary inputs arrive from the neighbouring lane's
// previous step through one warp shuffle per value.  When a lane finishes a
// stripe it starts the next one at once (a continuous wavefront); the rows
// crossing from one stripe to the next go through a small per-warp ring in
// global memory.  Per pair there is one fill and one drain of 31 steps.
//
// Per-column operands (codon code, background, seeds, and the ring values of
// the stripe boundary) are staged in a per-warp shared-memory window indexed
// by lane-local time, refilled once every 32 steps by one coalesced load per
// lane; a step reads its column with one 16-byte shared load.  The forward
// reads W1 two steps ahead into registers.
//
// The recurrences are the reference's, term for term and in the same
// association order (so that the float rounding matches):
//   backward  dummest-dp-backward.hh:473-574 (and the float filter :367-430)
//   forward   dummest-dp-forward.hh:63-250
// The forward reads W1 from the warp's slot, written by the backward in
// diagonal-major order ([stripe][diagonal][lane][R]) so that both the store
// and the load of one step are one contiguous 32*R*4-byte access.
//
// Row rescaling.  The kernel computes with every rescale count at zero, which
// is exactly the reference's arithmetic for a pair whose row maxima never
// exceed RESCALE_THRESH.  It reports the largest backward Y (Y >= W1 at every
// cell) and the largest forward W0/Y0, so the host can tell whether the
// reference would have rescaled; such pairs are re-scored by the exact
// row-rescaled path (dp_exact_wave.cuh).
//
// Mid score.  The reference forms promote(W0)*promote(W1) in double and
// rounds the mantissa to float (dummest-batch.hh:216-235); with both counts
// zero that is the float product W0*W1 whenever it is a normal float, so the
// per-cell product is one FMUL.  Overflow (a score above 2^128) is reported
// as +inf and routed to the exact path.
#pragma once

#include "dp_common.cuh"

namespace dmst {

struct SweepArgs {
    const uint8_t *codes;   // codon codes of the read
    const float *pre;       // prefixSeed[L]
    const float *suf;       // suffixSeedFromNext[L]
    const float *params;    // the profile's (M+2) x 11 Params
    const float *smE;       // emission table in shared memory, [25][rowPad]
    const float *smBg;      // bg_probs[4 + c] in shared memory
    float *w1;              // this warp's W1 slot
    float *ring;            // this warp's stripe-boundary ring (4 floats per column)
    PairScales sc;
    int L, M, rowPad, nS, P, D;
};

template <int R>
struct Coef {
    float enter[R], a0[R], a1[R], a2[R], b0[R], d0[R], d1[R], d2[R], eps[R], rs[R];
};

// Backward coefficients of rows rowBase..rowBase+R-1 (dummest-dp-backward.hh:481-494).
template <int R>
__device__ __forceinline__ void loadBackwardCoef(Coef<R> &c, const SweepArgs &a, int rowBase) {
#pragma unroll
    for (int k = 0; k < R; ++k) {
        const int i = rowBase + k;
        if (i <= a.M) {
            const float *q = a.params + (size_t)i * kParamFloats;
            c.enter[k] = q[10] * a.sc.sC;
            c.d0[k] = q[6];
            c.d1[k] = q[7] * a.sc.s2;
            c.d2[k] = q[8] * a.sc.s1;
            c.a0[k] = q[0] * a.sc.sC;
            c.a1[k] = q[1] * a.sc.s1;
            c.a2[k] = q[2] * a.sc.s2;
            c.b0[k] = q[3] * a.sc.sC;
            c.eps[k] = q[9];
            c.rs[k] = 1.0f;
        } else {
            c.enter[k] = c.d0[k] = c.d1[k] = c.d2[k] = c.a0[k] = c.a1[k] = c.a2[k] = c.b0[k] = c.eps[k] = 0.0f;
            c.rs[k] = 0.0f;
        }
    }
}

// Forward coefficients (dummest-dp-forward.hh:72-83): alpha'0 and beta'0 stay
// unscaled here, the codon scale multiplies the background term instead.
template <int R>
__device__ __forceinline__ void loadForwardCoef(Coef<R> &c, const SweepArgs &a, int rowBase) {
#pragma unroll
    for (int k = 0; k < R; ++k) {
        const int i = rowBase + k;
        if (i <= a.M) {
            const float *q = a.params + (size_t)i * kParamFloats;
            c.enter[k] = q[10] * a.sc.sC;
            c.a0[k] = q[0];
            c.a1[k] = q[1] * a.sc.s1;
            c.a2[k] = q[2] * a.sc.s2;
            c.b0[k] = q[3];
            c.d0[k] = q[6];
            c.d1[k] = q[7] * a.sc.s2;
            c.d2[k] = q[8] * a.sc.s1;
            c.eps[k] = q[9];
            c.rs[k] = 1.0f;
        } else {
            c.enter[k] = c.d0[k] = c.d1[k] = c.d2[k] = c.a0[k] = c.a1[k] = c.a2[k] = c.b0[k] = c.eps[k] = 0.0f;
            c.rs[k] = 0.0f;
        }
    }
}

template <int R>
__device__ __forceinline__ void loadEmit(float (&e)[R], const float *p) {
    if constexpr (R == 4) {
        float4 v = *reinterpret_cast<const float4 *>(p);
        e[0] = v.x; e[1] = v.y; e[2] = v.z; e[3] = v.w;
    } else if constexpr (R == 2) {
        float2 v = *reinterpret_cast<const float2 *>(p);
        e[0] = v.x; e[1] = v.y;
    } else {
        e[0] = p[0];
    }
}

template <int R>
__device__ __forceinline__ void storeW1(float *p, const float (&w)[R]) {
    if constexpr (R == 4) {
        *reinterpret_cast<float4 *>(p) = make_float4(w[0], w[1], w[2], w[3]);
    } else if constexpr (R == 2) {
        *reinterpret_cast<float2 *>(p) = make_float2(w[0], w[1]);
    } else {
        p[0] = w[0];
    }
}

// W1 values are read once, by the warp that wrote them: bypass L1 (the slot is
// rewritten by the warp's next pair).
template <int R>
__device__ __forceinline__ void loadW1(float (&w)[R], const float *p) {
    if constexpr (R == 4) {
        float4 v = __ldcg(reinterpret_cast<const float4 *>(p));
        w[0] = v.x; w[1] = v.y; w[2] = v.z; w[3] = v.w;
    } else if constexpr (R == 2) {
        float2 v = __ldcg(reinterpret_cast<const float2 *>(p));
        w[0] = v.x; w[1] = v.y;
    } else {
        w[0] = __ldcg(p);
    }
}

// ---------------------------------------------------------------------------
// Wavefront geometry.  The period P of a lane (steps per stripe) is at least
// kMinPeriod, so that a stripe-boundary value is written by one lane at least
// 64 steps before the window refill that hands it to the other lane.
// ---------------------------------------------------------------------------
constexpr int kMinPeriod = 96;
constexpr int kWin = 128;  // window entries (lane-local times), a power of two

__host__ __device__ inline int wavePeriod(int L) { return L > kMinPeriod ? L : kMinPeriod; }

// Per-warp staging window: entry t & (kWin-1) holds the column operands of
// lane-local time t.
struct Window {
    float4 col[kWin];   // backward: {code, bg, suf, pre}; forward: {code, bg*sC, pre, unused}
    float4 ring[kWin];  // stripe-boundary (W, Y, scale count) for the lane that reads the ring
};

// The stripe-boundary ring in global memory: 4 floats per column.
__device__ __forceinline__ float4 ringLoad(const float *ring, int col) {
    return __ldcg(reinterpret_cast<const float4 *>(ring) + col);
}
__device__ __forceinline__ void ringStore(float *ring, int col, float w, float y, int cnt) {
    __stcg(reinterpret_cast<float4 *>(ring) + col, make_float4(w, y, __int_as_float(cnt), 0.0f));
}
__device__ __forceinline__ void ringStore(float *ring, int col, float w, float y) {
    __stcg(reinterpret_cast<float2 *>(ring) + 2 * col, make_float2(w, y));
}

// Backward window entry for local time u (the column of u is L-1 - u mod P).
__device__ __forceinline__ void fillBackward(Window &w, const SweepArgs &a, int u) {
    const int e = u & (kWin - 1);
    float4 c = make_float4(__int_as_float(kPad), 0.0f, 0.0f, 0.0f);
    float4 r = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    if (u >= 0 && u < a.nS * a.P) {
        const int sp = u / a.P, jj = u - sp * a.P;
        if (jj < a.L) {
            const int j = a.L - 1 - jj;
            const int code = (j + 1 < a.L) ? (int)__ldg(a.codes + j + 1) : kPad;
            c = make_float4(__int_as_float(code), a.smBg[code], __ldg(a.suf + j), __ldg(a.pre + j));
            if (sp > 0) r = ringLoad(a.ring, jj);
        }
    }
    w.col[e] = c;
    w.ring[e] = r;
}

// Forward window entry for local time u (the column of u is u mod P).
__device__ __forceinline__ void fillForward(Window &w, const SweepArgs &a, int u) {
    const int e = u & (kWin - 1);
    float4 c = make_float4(__int_as_float(kPad), 0.0f, 0.0f, 0.0f);
    float4 r = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    if (u >= 0 && u < a.nS * a.P) {
        const int s = u / a.P, j = u - s * a.P;
        if (j < a.L) {
            const int code = (j >= 2) ? (int)__ldg(a.codes + j - 2) : kPad;
            c = make_float4(__int_as_float(code), a.smBg[code] * a.sc.sC, __ldg(a.pre + j), 0.0f);
            if (s > 0) r = ringLoad(a.ring, j);
        }
    }
    w.col[e] = c;
    w.ring[e] = r;
}

// ---------------------------------------------------------------------------
// Sweep modes.
//   kFilter    fast backward, no W1 kept: findSimilaritiesBackwardOnly
//   kMid       fast backward keeping W1 / fast forward with the float mid
//   kDiscover  exact path, pass 1: per-lane scale counts, row maxima
//   kReplay    exact path, pass 2: the reference's counts, exact maxima
// The fast modes compute with every rescale count at zero.
// ---------------------------------------------------------------------------
enum SweepMode { kFilter = 0, kMid = 1, kDiscover = 2, kReplay = 3 };

constexpr float kBump = 0x1p100f;  // discovery: rescale a lane above this
constexpr float kStep = 0x1p-64f;  // one rescale step, RESCALE_STEP (dummest-score.hh:87)
constexpr int kRescaleBits = 64;   // RESCALE_BITS (dummest-score.hh:83)

__device__ __forceinline__ float stepsDown(int d) {  // 2^(-64 d), d >= 0; 0 past float range
    return d == 0 ? 1.0f : (d == 1 ? kStep : 0.0f);
}

// Seed coefficient at scale count c: scale * 2^(-64 c) as the float the
// reference builds (rowRescaleVector, dummest-score.hh:145-152; FTZ makes it 0
// from c = 2 on).
__device__ __forceinline__ float seedCoef(bool realRow, int c) {
    return realRow ? (c == 0 ? 1.0f : (c == 1 ? kStep : 0.0f)) : 0.0f;
}

// Exact (double mantissa, binary exponent) maximum of the exact path.
struct ExactBest {
    double m;
    int e;
};

__device__ __forceinline__ void foldBest(ExactBest &b, double v, int countSum) {
    if (!(v > 0.0)) return;
    int e;
    const double m = frexp(v, &e);
    e += kRescaleBits * countSum;
    if (b.m == 0.0 || e > b.e || (e == b.e && m > b.m)) {
        b.m = m;
        b.e = e;
    }
}

// Per-pair rows of the exact path (global scratch).
struct ExactRows {
    float *rowMax;  // M+1: discovery row maxima
    int *rowCnt;    // M+1: discovery counts at the row ends
    int *cntB;      // M+2: reference backward counts, cntB[M+1] = 0
    int *cntF;      // M+2: reference forward counts, cntF[i+1] = row i, cntF[0] = 0
};

// ---------------------------------------------------------------------------
// Backward sweep (dummest-dp-backward.hh:473-574; the float filter :367-430).
// ---------------------------------------------------------------------------
template <int R, int MODE>
__device__ void backwardSweep(const SweepArgs &a, Window &win, int lane, float &filtOut, float &maxYOut,
                              const ExactRows *x = nullptr, ExactBest *exact = nullptr) {
    constexpr int S = kLanes * R;
    constexpr bool kStore = MODE == kMid || MODE == kReplay;
    Coef<R> c;
    float h1[R], h2[R], h3[R], z1[R], z2[R], z3[R];
#pragma unroll
    for (int k = 0; k < R; ++k) h1[k] = h2[k] = h3[k] = z1[k] = z2[k] = z3[k] = 0.0f;
    float rb1 = 0.0f, rb2 = 0.0f, rb3 = 0.0f;  // row below (other lane) at j+1..j+3
    float sendW = 0.0f, sendY = 0.0f;
    int sendC = 0;
    float filt = 0.0f, maxY = 0.0f;
    // exact-path state
    int cnt = 0;                  // discovery: this lane's scale count
    float rmax[R];                // discovery: per-row maxima at count cnt
    int cOut[R];                  // replay: count of each row after its decision
    float fOut[R];                // replay: 1 or 2^-64, the row's own rescale
    double rowBest[R];            // replay: per-row max of W1 * prefixSeed
    if constexpr (MODE == kDiscover || MODE == kReplay) {
#pragma unroll
        for (int k = 0; k < R; ++k) {
            rmax[k] = 0.0f;
            cOut[k] = 0;
            fOut[k] = 1.0f;
            rowBest[k] = 0.0;
        }
    }
    const int L = a.L, P = a.P, nS = a.nS;
    const int total = nS * P;
    const int T = total + (kLanes - 1);
    const int lag = kLanes - 1 - lane;  // lane 31 leads
    int u = -lag;                       // local time
    int sp = 0, jj = 0;                 // stripe from the bottom, column from the right
    float *wp = a.w1;                   // W1 store pointer of the current step
    // Window: local times [0, 64) now, then 32 ahead at every block start.
    __syncwarp();
    fillBackward(win, a, lane);
    fillBackward(win, a, lane + 32);
    for (int t0 = 0; t0 < T; t0 += 32) {
        __syncwarp();
        if (t0 > 0) fillBackward(win, a, t0 + 32 + lane);
        const int tEnd = t0 + 32 < T ? t0 + 32 : T;
        for (int t = t0; t < tEnd; ++t) {
            float inW = __shfl_down_sync(kFull, sendW, 1);
            float inY = __shfl_down_sync(kFull, sendY, 1);
            int inC = 0;
            if (MODE == kDiscover) inC = __shfl_down_sync(kFull, sendC, 1);
            if (u >= 0 && u < total && jj < L) {
                const int s = nS - 1 - sp;
                const int rowBase = s * S + lane * R;
                if (jj == 0) {
                    loadBackwardCoef<R>(c, a, rowBase);
#pragma unroll
                    for (int k = 0; k < R; ++k) h1[k] = h2[k] = h3[k] = z1[k] = z2[k] = z3[k] = 0.0f;
                    rb1 = rb2 = rb3 = 0.0f;
                    wp = a.w1 + (((size_t)s * a.D + lag) * kLanes + lane) * R;
                    if (MODE == kDiscover) {
                        cnt = 0;
#pragma unroll
                        for (int k = 0; k < R; ++k) rmax[k] = 0.0f;
                    }
                    if (MODE == kReplay) {
#pragma unroll
                        for (int k = 0; k < R; ++k) {
                            const int i = rowBase + k;
                            const int ci = i <= a.M ? i : a.M + 1;
                            const int cIn = x->cntB[ci + 1 <= a.M + 1 ? ci + 1 : a.M + 1];
                            cOut[k] = x->cntB[ci];
                            fOut[k] = stepsDown(cOut[k] - cIn);
                            c.rs[k] = seedCoef(i <= a.M, cIn);
                            rowBest[k] = 0.0;
                        }
                    }
                }
                const int slot = u & (kWin - 1);
                const float4 col = win.col[slot];
                if (lane == kLanes - 1) {
                    const float4 r = win.ring[slot];
                    inW = r.x;
                    inY = r.y;
                    if (MODE == kDiscover) inC = __float_as_int(r.z);
                }
                if (MODE == kDiscover) {
                    // Align the incoming values and this lane to one scale.
                    if (inC > cnt) {
                        const float f = stepsDown(inC - cnt);
#pragma unroll
                        for (int k = 0; k < R; ++k) {
                            h1[k] *= f; h2[k] *= f; h3[k] *= f;
                            z1[k] *= f; z2[k] *= f; z3[k] *= f;
                            rmax[k] *= f;
                            c.rs[k] = seedCoef(rowBase + k <= a.M, inC);
                        }
                        rb1 *= f; rb2 *= f; rb3 *= f;
                        cnt = inC;
                    } else if (inC < cnt) {
                        const float f = stepsDown(cnt - inC);
                        inW *= f;
                        inY *= f;
                    }
                }
                const int code = __float_as_int(col.x);
                const float bgv = col.y, sufv = col.z, prev = col.w;
                float e[R];
                loadEmit<R>(e, a.smE + code * a.rowPad + rowBase);
                float bW1 = rb1, bW2 = rb2, bW3 = rb3, bY = inY;
                float wv[R];
                float stepMax = 0.0f;
#pragma unroll
                for (int k = R - 1; k >= 0; --k) {
                    float acc = (bW3 * e[k]) * c.enter[k];
                    acc = __fmaf_rn(bY, c.d0[k], acc);
                    acc = __fmaf_rn(bW2, c.d1[k], acc);
                    acc = __fmaf_rn(bW1, c.d2[k], acc);
                    const float zbg = z3[k] * bgv;
                    acc = __fmaf_rn(zbg, c.a0[k], acc);
                    acc = __fmaf_rn(h2[k], c.a2[k], acc);
                    acc = __fmaf_rn(h1[k], c.a1[k], acc);
                    const float W = __fmaf_rn(sufv, c.rs[k], acc);
                    const float Y = __fmaf_rn(c.eps[k], bY, W);
                    const float Z = __fmaf_rn(c.b0[k], zbg, W);
                    if (MODE == kFilter || MODE == kMid) {
                        maxY = fmaxf(maxY, Y);
                        filt = fmaxf(filt, W * prev);
                    }
                    if (MODE == kDiscover) {
                        rmax[k] = fmaxf(rmax[k], Y);  // Y >= W1 at every cell
                        stepMax = fmaxf(stepMax, Y);
                    }
                    if (MODE == kReplay) {
                        // What leaves the row is scaled by the row's own decision.
                        const float Wo = W * fOut[k];
                        rowBest[k] = fmax(rowBest[k], (double)Wo * (double)prev);
                        bW1 = h1[k] * fOut[k];
                        bW2 = h2[k] * fOut[k];
                        bW3 = h3[k] * fOut[k];
                        bY = Y * fOut[k];
                        wv[k] = Wo;
                    } else {
                        bW1 = h1[k];
                        bW2 = h2[k];
                        bW3 = h3[k];
                        bY = Y;
                        wv[k] = W;
                    }
                    h3[k] = h2[k];
                    h2[k] = h1[k];
                    h1[k] = W;
                    z3[k] = z2[k];
                    z2[k] = z1[k];
                    z1[k] = Z;
                }
                rb3 = rb2;
                rb2 = rb1;
                rb1 = inW;
                sendW = wv[0];
                sendY = bY;
                if (MODE == kDiscover) {
                    if (stepMax > kBump) {
#pragma unroll
                        for (int k = 0; k < R; ++k) {
                            h1[k] *= kStep; h2[k] *= kStep; h3[k] *= kStep;
                            z1[k] *= kStep; z2[k] *= kStep; z3[k] *= kStep;
                            rmax[k] *= kStep;
                            c.rs[k] = seedCoef(rowBase + k <= a.M, cnt + 1);
                        }
                        rb1 *= kStep; rb2 *= kStep; rb3 *= kStep;
                        sendW *= kStep;
                        sendY *= kStep;
                        ++cnt;
                    }
                    sendC = cnt;
                }
                if (kStore) {
                    storeW1<R>(wp, wv);
                    wp += kLanes * R;
                }
                if (lane == 0 && sp < nS - 1) {
                    if (MODE == kDiscover)
                        ringStore(a.ring, jj, sendW, sendY, sendC);
                    else
                        ringStore(a.ring, jj, sendW, sendY);
                }
                if (jj == L - 1) {
                    // the last column of these rows
#pragma unroll
                    for (int k = 0; k < R; ++k) {
                        const int i = rowBase + k;
                        if (i > a.M) continue;
                        if (MODE == kDiscover) {
                            x->rowMax[i] = rmax[k];
                            x->rowCnt[i] = cnt;
                        }
                        if (MODE == kReplay) foldBest(*exact, rowBest[k], cOut[k]);
                    }
                }
            } else {
                sendW = 0.0f;
                sendY = 0.0f;
                sendC = 0;
            }
            if (u >= 0 && ++jj == P) {
                jj = 0;
                ++sp;
            }
            ++u;
        }
    }
    filtOut = filt;
    maxYOut = maxY;
}

// W1 read-ahead for the forward sweep: a cursor two steps ahead of the lane.
template <int R>
struct W1Ahead {
    int u, s, j;
    __device__ __forceinline__ void next(const SweepArgs &a, int lane, int total, float (&q)[R]) {
        if (u >= 0 && u < total && j < a.L) {
            const int db = (a.L - 1 - j) + (kLanes - 1 - lane);
            loadW1<R>(q, a.w1 + (((size_t)s * a.D + db) * kLanes + lane) * R);
        }
        if (u >= 0 && ++j == a.P) {
            j = 0;
            ++s;
        }
        ++u;
    }
};

template <int R, int MODE>
struct FwdState {
    Coef<R> c;
    float w1[R], w2[R], w3[R], z1[R], z2[R], z3[R];
    float sendIn, sendY, best, mx;
    int sendC;
    int u, s, j;
    // exact-path state (see backwardSweep)
    int cnt;
    float rmax[R];
    int cIn[R], cB[R];
    float fOut[R];
    double rowBest[R];
};

// One forward step of a lane (dummest-dp-forward.hh:112-223); q holds the W1
// values of this step.
template <int R, int MODE>
__device__ __forceinline__ void forwardStep(FwdState<R, MODE> &f, const SweepArgs &a, Window &win, int lane,
                                            int total, const float (&q)[R], const ExactRows *x, ExactBest *exact) {
    constexpr int S = kLanes * R;
    float inW = __shfl_up_sync(kFull, f.sendIn, 1);
    float inY = __shfl_up_sync(kFull, f.sendY, 1);
    int inC = 0;
    if (MODE == kDiscover) inC = __shfl_up_sync(kFull, f.sendC, 1);
    if (f.u >= 0 && f.u < total && f.j < a.L) {
        const int rowBase = f.s * S + lane * R;
        if (f.j == 0) {
            loadForwardCoef<R>(f.c, a, rowBase);
#pragma unroll
            for (int k = 0; k < R; ++k) f.w1[k] = f.w2[k] = f.w3[k] = f.z1[k] = f.z2[k] = f.z3[k] = 0.0f;
            if (MODE == kDiscover) {
                f.cnt = 0;
#pragma unroll
                for (int k = 0; k < R; ++k) f.rmax[k] = 0.0f;
            }
            if (MODE == kReplay) {
#pragma unroll
                for (int k = 0; k < R; ++k) {
                    const int i = rowBase + k;
                    const int ci = i <= a.M ? i : a.M;
                    f.cIn[k] = x->cntF[ci];
                    f.fOut[k] = stepsDown(x->cntF[ci + 1] - f.cIn[k]);
                    f.cB[k] = x->cntB[ci];
                    f.c.rs[k] = seedCoef(i <= a.M, f.cIn[k]);
                    f.rowBest[k] = 0.0;
                }
            }
        }
        const int slot = f.u & (kWin - 1);
        const float4 col = win.col[slot];
        if (lane == 0) {
            const float4 r = win.ring[slot];
            inW = r.x;
            inY = r.y;
            if (MODE == kDiscover) inC = __float_as_int(r.z);
        }
        if (MODE == kDiscover) {
            if (inC > f.cnt) {
                const float g = stepsDown(inC - f.cnt);
#pragma unroll
                for (int k = 0; k < R; ++k) {
                    f.w1[k] *= g; f.w2[k] *= g; f.w3[k] *= g;
                    f.z1[k] *= g; f.z2[k] *= g; f.z3[k] *= g;
                    f.rmax[k] *= g;
                    f.c.rs[k] = seedCoef(rowBase + k <= a.M, inC);
                }
                f.cnt = inC;
            } else if (inC < f.cnt) {
                const float g = stepsDown(f.cnt - inC);
                inW *= g;
                inY *= g;
            }
        }
        const int code = __float_as_int(col.x);
        const float bgsC = col.y, prev = col.z;
        float e[R];
        loadEmit<R>(e, a.smE + code * a.rowPad + rowBase);
        float win0 = inW, yab = inY;
        float stepMax = 0.0f;
#pragma unroll
        for (int k = 0; k < R; ++k) {
            // The reference's operations as GCC contracts them at -O3
            // (dummest-dp-forward.hh:116-222): Z0 = (bg*sC)*fma(b0, Z0[j-3],
            // a0*w3); the alpha1/alpha2 products fuse into the W0 sum, and
            // Y0 = fma(eps, Y0[i-1], d0*W0).
            const float X = (f.c.enter[k] * e[k]) * f.w3[k];
            const float Z0 = bgsC * __fmaf_rn(f.c.b0[k], f.z3[k], f.c.a0[k] * f.w3[k]);
            const float zs = __fmaf_rn(f.c.a2[k], f.w2[k], __fmaf_rn(f.c.a1[k], f.w1[k], Z0));
            // fma(prev, 1, x) is prev + x; in the fast mode every row takes the
            // seed: padding rows (past M, zero coefficients) then hold only
            // their seed, which reaches no real row and multiplies a zero W1.
            const float W0 = (MODE == kMid) ? win0 + __fadd_rn(zs, prev) : win0 + __fmaf_rn(prev, f.c.rs[k], zs);
            if (MODE == kMid) f.best = fmaxf(f.best, W0 * q[k]);
            if (MODE == kReplay) f.rowBest[k] = fmax(f.rowBest[k], (double)W0 * (double)q[k]);
            const float Y0 = __fmaf_rn(f.c.eps[k], yab, f.c.d0[k] * W0);
            if (MODE == kMid) f.mx = fmaxf(f.mx, fmaxf(W0, Y0));
            const float nin = __fmaf_rn(f.c.d2[k], f.w1[k], __fmaf_rn(f.c.d1[k], f.w2[k], X + Y0));
            if (MODE == kDiscover) {
                f.rmax[k] = fmaxf(f.rmax[k], fmaxf(W0, Y0));
                stepMax = fmaxf(stepMax, fmaxf(fmaxf(W0, Y0), nin));
            }
            f.w3[k] = f.w2[k];
            f.w2[k] = f.w1[k];
            f.w1[k] = W0;
            f.z3[k] = f.z2[k];
            f.z2[k] = f.z1[k];
            f.z1[k] = Z0;
            if (MODE == kReplay) {
                win0 = nin * f.fOut[k];
                yab = Y0 * f.fOut[k];
            } else {
                win0 = nin;
                yab = Y0;
            }
        }
        if (MODE == kDiscover) {
            if (stepMax > kBump) {
#pragma unroll
                for (int k = 0; k < R; ++k) {
                    f.w1[k] *= kStep; f.w2[k] *= kStep; f.w3[k] *= kStep;
                    f.z1[k] *= kStep; f.z2[k] *= kStep; f.z3[k] *= kStep;
                    f.rmax[k] *= kStep;
                    f.c.rs[k] = seedCoef(rowBase + k <= a.M, f.cnt + 1);
                }
                win0 *= kStep;
                yab *= kStep;
                ++f.cnt;
            }
            f.sendC = f.cnt;
        }
        f.sendIn = win0;
        f.sendY = yab;
        if (lane == kLanes - 1 && f.s < a.nS - 1) {
            if (MODE == kDiscover)
                ringStore(a.ring, f.j, f.sendIn, f.sendY, f.sendC);
            else
                ringStore(a.ring, f.j, f.sendIn, f.sendY);
        }
        if (f.j == a.L - 1) {
#pragma unroll
            for (int k = 0; k < R; ++k) {
                const int i = rowBase + k;
                if (i > a.M) continue;
                if (MODE == kDiscover) {
                    x->rowMax[i] = f.rmax[k];
                    x->rowCnt[i] = f.cnt;
                }
                if (MODE == kReplay) foldBest(*exact, f.rowBest[k], f.cIn[k] + f.cB[k]);
            }
        }
    } else {
        f.sendIn = 0.0f;
        f.sendY = 0.0f;
        f.sendC = 0;
    }
    if (f.u >= 0 && ++f.j == a.P) {
        f.j = 0;
        ++f.s;
    }
    ++f.u;
}

// ---------------------------------------------------------------------------
// Forward sweep (reads W1 written by the backward sweep of the same mode).
// ---------------------------------------------------------------------------
template <int R, int MODE>
__device__ void forwardSweep(const SweepArgs &a, Window &win, int lane, float &bestOut, float &maxOut,
                             const ExactRows *x = nullptr, ExactBest *exact = nullptr) {
    FwdState<R, MODE> f;
#pragma unroll
    for (int k = 0; k < R; ++k) {
        f.w1[k] = f.w2[k] = f.w3[k] = f.z1[k] = f.z2[k] = f.z3[k] = 0.0f;
        if constexpr (MODE == kDiscover || MODE == kReplay) {
            f.rmax[k] = 0.0f;
            f.cIn[k] = f.cB[k] = 0;
            f.fOut[k] = 1.0f;
            f.rowBest[k] = 0.0;
        }
    }
    f.sendIn = f.sendY = f.best = f.mx = 0.0f;
    f.sendC = f.cnt = 0;
    f.u = -lane;  // lane 0 leads
    f.s = f.j = 0;
    const int total = a.nS * a.P;
    const int T = total + (kLanes - 1);
    constexpr bool kReadW1 = MODE == kMid || MODE == kReplay;
    W1Ahead<R> ah{-lane, 0, 0};
    float qa[R], qb[R];
#pragma unroll
    for (int k = 0; k < R; ++k) qa[k] = qb[k] = 0.0f;
    if (kReadW1) {
        ah.next(a, lane, total, qa);
        ah.next(a, lane, total, qb);
    }
    __syncwarp();
    fillForward(win, a, lane);
    fillForward(win, a, lane + 32);
    for (int t0 = 0; t0 < T; t0 += 32) {
        __syncwarp();
        if (t0 > 0) fillForward(win, a, t0 + 32 + lane);
        // Blocks are 32 steps (even) except the last; its odd tail step is
        // handled after the pairwise loop.
        const int n = (t0 + 32 < T ? 32 : T - t0);
        int k = 0;
        for (; k + 1 < n; k += 2) {
            forwardStep<R, MODE>(f, a, win, lane, total, qa, x, exact);
            if (kReadW1) ah.next(a, lane, total, qa);
            forwardStep<R, MODE>(f, a, win, lane, total, qb, x, exact);
            if (kReadW1) ah.next(a, lane, total, qb);
        }
        if (k < n) {
            forwardStep<R, MODE>(f, a, win, lane, total, qa, x, exact);
            if (kReadW1) ah.next(a, lane, total, qa);
        }
    }
    bestOut = f.best;
    maxOut = f.mx;
}

__device__ __forceinline__ float warpMax(float v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmaxf(v, __shfl_xor_sync(kFull, v, o));
    return v;
}

struct DpArgs {
    const Chunk *chunks;
    int nChunks;
    int *chunkCounter;
    const DevPair *pairs;
    const DevProfile *profiles;
    const float *emit;
    const float *params;
    const uint8_t *codes;
    const float *seeds;
    const PairScales *scales;
    float *w1;
    size_t w1SlotFloats;
    float *ring;
    size_t ringSlotFloats;
    PairOut *out;
};

template <int R, bool MID>
__device__ void scorePair(const DpArgs &g, int pi, const float *smE, int rowPad, const float *smBg, Window &win,
                          float *w1, float *ring, int lane) {
    const DevPair p = g.pairs[pi];
    SweepArgs a;
    a.codes = g.codes + p.codeOff;
    a.pre = g.seeds + p.seedOff;
    a.suf = a.pre + p.L;
    a.params = g.params + g.profiles[p.prof].paramOff;
    a.smE = smE;
    a.smBg = smBg;
    a.w1 = w1;
    a.ring = ring;
    a.sc = g.scales[pi];
    a.L = p.L;
    a.M = p.M;
    a.rowPad = rowPad;
    a.nS = (p.M + 1 + kLanes * R - 1) / (kLanes * R);
    a.P = wavePeriod(p.L);
    a.D = a.P + kLanes - 1;
    float filt, maxYb, mid = 0.0f, maxFw = 0.0f;
    if (MID) {
        backwardSweep<R, kMid>(a, win, lane, filt, maxYb);
        forwardSweep<R, kMid>(a, win, lane, mid, maxFw);
    } else {
        backwardSweep<R, kFilter>(a, win, lane, filt, maxYb);
    }
    filt = warpMax(filt);
    maxYb = warpMax(maxYb);
    mid = warpMax(mid);
    maxFw = warpMax(maxFw);
    if (lane == 0) {
        PairOut o;
        o.mid = mid;
        o.filt = filt;
        o.maxYb = maxYb;
        o.maxFw = maxFw;
        g.out[pi] = o;
    }
}

// CTA shape: kCtaWarps warps share one shared-memory copy of the profile's
// emission table; at most 128 registers per thread.
#ifndef DMST_CTA_WARPS
#define DMST_CTA_WARPS 16
#endif
constexpr int kCtaWarps = DMST_CTA_WARPS;

// Persistent kernel for one rows-per-lane value: CTAs pull chunks
// (same-profile runs of pairs, costliest first) from a global counter, stage
// the chunk's profile emission table in shared memory, and their warps pull
// pairs from the chunk.  Dynamic shared memory: the table (tableFloats), then
// one Window per warp.
template <int R, bool MID>
__global__ void __launch_bounds__(kCtaWarps * kLanes, 1) dpKernel(DpArgs g, int tableFloats) {
    extern __shared__ float4 smRaw[];
    float *smE = reinterpret_cast<float *>(smRaw);
    Window *wins = reinterpret_cast<Window *>(smE + tableFloats);
    __shared__ float smBg[32];
    __shared__ int smChunk, smNext;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const size_t slot = (size_t)blockIdx.x * kCtaWarps + warp;
    float *w1 = g.w1 + slot * g.w1SlotFloats;
    float *ring = g.ring + slot * g.ringSlotFloats;
    Window &win = wins[warp];
    int loaded = -1;
    for (;;) {
        if (threadIdx.x == 0) {
            smChunk = atomicAdd(g.chunkCounter, 1);
            smNext = 0;
        }
        __syncthreads();
        const int ci = smChunk;
        if (ci >= g.nChunks) break;
        const Chunk ch = g.chunks[ci];
        const int rowPad = ch.rowPad;
        if (ch.prof != loaded) {
            const DevProfile *pr = g.profiles + ch.prof;
            const float4 *src = reinterpret_cast<const float4 *>(g.emit + pr->emitOff);
            const int n4 = kNumCodes * rowPad / 4;
            for (int i = threadIdx.x; i < n4; i += blockDim.x) smRaw[i] = __ldg(src + i);
            if (threadIdx.x < 32) smBg[threadIdx.x] = threadIdx.x < kNumCodes ? pr->bg[threadIdx.x] : 0.0f;
            loaded = ch.prof;
        }
        __syncthreads();
        for (;;) {
            int k = 0;
            if (lane == 0) k = atomicAdd(&smNext, 1);
            k = __shfl_sync(kFull, k, 0);
            if (k >= ch.count) break;
            scorePair<R, MID>(g, ch.first + k, smE, rowPad, smBg, win, w1, ring, lane);
        }
        __syncthreads();
    }
}

}  // namespace dmst
