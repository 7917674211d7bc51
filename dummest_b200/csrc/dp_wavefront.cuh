// The row-contiguous stripe wavefront: the step functions of the exact
// row-rescaled path (dp_exact_wave.cuh, dp_exact.cuh) and of the plain
// one-pair-per-launch schedule (dp_plain.cuh).  The batched kernel of the
// fast path is dp_stagger.cuh.
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
// by lane-local time, refilled once every 48 steps by coalesced loads; a step
// reads its column with one 16-byte shared load.  The forward copies W1 five
// steps ahead into a shared-memory ring with cp.async, so that the DRAM
// latency of the W1 round trip is hidden without holding registers.
//
// Steps run in groups of three (six in the forward): the three-column
// histories of each row live in register slots whose roles rotate with the
// step's phase, so the history shifts by renaming instead of copying.
//
// The recurrences are the reference's, term for term and in the same
// association order (so that the float rounding matches):
//   backward  dummest-dp-backward.hh:473-574 (and the float filter :367-430)
//   forward   dummest-dp-forward.hh:63-250
// The forward reads W1 from the warp's slot, written by the backward in
// diagonal-major order ([stripe][diagonal][lane][R]) so that both the store
// and the load of one step are one contiguous 32*R*4-byte access.
//
// Row rescaling.  The fast modes compute with every rescale count at zero,
// which is exactly the reference's arithmetic for a pair whose row maxima
// never exceed RESCALE_THRESH.  They report the largest backward Y (Y >= W1
// at every cell) and the largest forward W0/Y0, so the host can tell whether
// the reference would have rescaled; such pairs are re-scored by the exact
// row-rescaled path (dp_exact_wave.cuh), whose modes apply the reference's
// rescale counts.
//
// Mid score.  The reference forms promote(W0)*promote(W1) in double and
// rounds the mantissa to float (dummest-batch.hh:216-235); with both counts
// zero that is the float product W0*W1 whenever it is a normal float, so the
// per-cell product is one FMUL.  Overflow (a score above 2^128) is reported
// as +inf and routed to the exact path.
#pragma once

#include "dp_common.cuh"

namespace dmst {

// Fields of the pair that the sweeps read only at window refills and stripe
// starts.  They sit in the warp's shared memory and are read through volatile
// loads, so that the compiler re-reads them instead of holding them in
// registers across the sweeps.
struct PairCold {
    const uint8_t *codes;   // codon codes of the read
    const float *pre;       // prefixSeed[L]
    const float *suf;       // suffixSeedFromNext[L]
    const float *coef;      // the profile's DP coefficient planes (coefOffOf)
    const float *smBg;      // bg_probs[4 + c] in shared memory
    PairScales sc;
    int M;
    int coefStride;         // floats between planes (the profile's rowPad)
    int pad[2];
};

struct SweepArgs {
    PairCold *cold;         // in shared memory
    const float *smE;       // emission table, [25][rowPad] (shared memory; the exact path reads it from global)
    float *w1;              // this warp's W1 slot
    float *ring;            // this warp's stripe-boundary ring (4 floats per column)
    int L, rowPad, nS, P, D;
    // Stripes of this warp, in processing order: sFirst, sFirst + sStep, ...
    // (nMine of them; the fast path: 0, 1, ..., nS-1).  The exact path runs a
    // pair's stripes on several warps: the ring of stripe sp (processing
    // order) is then ring + (sp % ringSlots) * ringStride.
    int sFirst, sStep, nMine, ringSlots;
    long long ringStride;
    // Exact replay for the traceback: the row-major (M+1) x L matrix that takes
    // each cell's value before its row's rescale (backward: W1, forward: W0),
    // or null.
    float *alignOut;

    __device__ __forceinline__ const uint8_t *codes() const {
        return *reinterpret_cast<const uint8_t *const volatile *>(&cold->codes);
    }
    __device__ __forceinline__ const float *pre() const {
        return *reinterpret_cast<const float *const volatile *>(&cold->pre);
    }
    __device__ __forceinline__ const float *suf() const {
        return *reinterpret_cast<const float *const volatile *>(&cold->suf);
    }
    __device__ __forceinline__ const float *coef() const {
        return *reinterpret_cast<const float *const volatile *>(&cold->coef);
    }
    __device__ __forceinline__ int coefStride() const {
        return *reinterpret_cast<const volatile int *>(&cold->coefStride);
    }
    __device__ __forceinline__ const float *smBg() const {
        return *reinterpret_cast<const float *const volatile *>(&cold->smBg);
    }
    __device__ __forceinline__ PairScales sc() const {
        const volatile PairScales *v = &cold->sc;
        return PairScales{v->s1, v->s2, v->sC, 0.0f};
    }
    __device__ __forceinline__ int M() const { return *reinterpret_cast<const volatile int *>(&cold->M); }
};

template <int R>
struct Coef {
    float enter[R], a0[R], a1[R], a2[R], b0[R], d0[R], d1[R], d2[R], eps[R], rs[R];
};

// R consecutive rows of a coefficient plane (read-only in every kernel).
template <int R>
__device__ __forceinline__ void loadRows(float (&v)[R], const float *p) {
    if constexpr (R == 4) {
        const float4 t = __ldg(reinterpret_cast<const float4 *>(p));
        v[0] = t.x; v[1] = t.y; v[2] = t.z; v[3] = t.w;
    } else if constexpr (R == 2) {
        const float2 t = __ldg(reinterpret_cast<const float2 *>(p));
        v[0] = t.x; v[1] = t.y;
    } else {  // R = 1 or 3 (rows not 8-byte aligned for R = 3)
#pragma unroll
        for (int k = 0; k < R; ++k) v[k] = __ldg(p + k);
    }
}

// v[k] = plane[row k] * s, rounded as the reference's float product; a
// padding row (plane value 0) gives 0, as the scales are finite.
template <int R>
__device__ __forceinline__ void loadScaled(float (&v)[R], const float *p, float s) {
    loadRows<R>(v, p);
#pragma unroll
    for (int k = 0; k < R; ++k) v[k] = v[k] * s;
}

// Backward coefficients of rows rowBase..rowBase+R-1 (dummest-dp-backward.hh:481-494):
// the Params products with the pair's scales; rows past M get 0 (rs 0).
template <int R>
__device__ __forceinline__ void loadBackwardCoef(Coef<R> &c, const SweepArgs &a, int rowBase) {
    const float *q = a.coef() + rowBase;
    const int st = a.coefStride();
    const PairScales sc = a.sc();
    loadScaled<R>(c.enter, q + kPEnter * st, sc.sC);
    loadRows<R>(c.d0, q + kPD0 * st);
    loadScaled<R>(c.d1, q + kPD1 * st, sc.s2);
    loadScaled<R>(c.d2, q + kPD2 * st, sc.s1);
    loadScaled<R>(c.a0, q + kPA0 * st, sc.sC);
    loadScaled<R>(c.a1, q + kPA1 * st, sc.s1);
    loadScaled<R>(c.a2, q + kPA2 * st, sc.s2);
    loadScaled<R>(c.b0, q + kPB0 * st, sc.sC);
    loadRows<R>(c.eps, q + kPEps * st);
    loadRows<R>(c.rs, q + kPRs * st);
}

// Forward coefficients (dummest-dp-forward.hh:72-83): alpha'0 and beta'0 stay
// unscaled here, the codon scale multiplies the background term instead.
template <int R>
__device__ __forceinline__ void loadForwardCoef(Coef<R> &c, const SweepArgs &a, int rowBase) {
    const float *q = a.coef() + rowBase;
    const int st = a.coefStride();
    const PairScales sc = a.sc();
    loadScaled<R>(c.enter, q + kPEnter * st, sc.sC);
    loadRows<R>(c.a0, q + kPA0 * st);
    loadScaled<R>(c.a1, q + kPA1 * st, sc.s1);
    loadScaled<R>(c.a2, q + kPA2 * st, sc.s2);
    loadRows<R>(c.b0, q + kPB0 * st);
    loadRows<R>(c.d0, q + kPD0 * st);
    loadScaled<R>(c.d1, q + kPD1 * st, sc.s2);
    loadScaled<R>(c.d2, q + kPD2 * st, sc.s1);
    loadRows<R>(c.eps, q + kPEps * st);
    loadRows<R>(c.rs, q + kPRs * st);
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
#pragma unroll
        for (int k = 0; k < R; ++k) e[k] = p[k];
    }
}

// The same load from a 32-bit shared-memory address (the emission table in
// the CTA's shared memory): a plain shared load, no generic-address check.
// The table is written before the chunk's barrier and only read in the
// sweeps, and the address depends on the step's window entry, so the load
// cannot move above the barrier.
template <int R>
__device__ __forceinline__ void loadEmitS(float (&e)[R], unsigned addr) {
    if constexpr (R == 4) {
        asm("ld.shared.v4.f32 {%0, %1, %2, %3}, [%4];" : "=f"(e[0]), "=f"(e[1]), "=f"(e[2]), "=f"(e[3]) : "r"(addr));
    } else if constexpr (R == 2) {
        asm("ld.shared.v2.f32 {%0, %1}, [%2];" : "=f"(e[0]), "=f"(e[1]) : "r"(addr));
    } else {
#pragma unroll
        for (int k = 0; k < R; ++k) asm("ld.shared.f32 %0, [%1];" : "=f"(e[k]) : "r"(addr + 4u * k));
    }
}

template <int R>
__device__ __forceinline__ void storeW1(float *p, const float (&w)[R]) {
    if constexpr (R == 4) {
        *reinterpret_cast<float4 *>(p) = make_float4(w[0], w[1], w[2], w[3]);
    } else if constexpr (R == 2) {
        *reinterpret_cast<float2 *>(p) = make_float2(w[0], w[1]);
    } else {
#pragma unroll
        for (int k = 0; k < R; ++k) p[k] = w[k];
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
// Wavefront geometry.  Steps run in blocks of kBlock (a multiple of three);
// the window holds the column operands of local times [t0 - 31, t0 + 2 kBlock)
// around a block starting at t0 (127 entries), and each block start refills
// the kBlock entries of the next block.  The period P of a lane (steps per
// stripe) is at least kMinPeriod, so that a stripe-boundary value is written
// by one lane before the window refill that hands it to the other lane
// (31 + s P + j < (s+1) P + j - 2 kBlock + 1 for every stripe s and column j).
// ---------------------------------------------------------------------------
constexpr int kBlock = 48;
constexpr int kMinPeriod = 128;
constexpr int kWin = 128;  // window entries (lane-local times), a power of two
static_assert(kBlock % 6 == 0 && kBlock <= kWin - 31 - kBlock, "window geometry");
static_assert(kMinPeriod >= 31 + 2 * kBlock, "stripe hand-off before the refill that reads it");

__host__ __device__ inline int wavePeriod(int L) { return L > kMinPeriod ? L : kMinPeriod; }

// Per-warp staging window: entry t & (kWin-1) holds the column operands of
// lane-local time t.
// W1 staging of the forward sweep: each lane copies its R values of W1 for
// the step kW1Ahead steps ahead into a ring of kW1Slots slots (cp.async, one
// commit group per step), so that a step waits on shared memory, not DRAM.
constexpr int kW1Slots = 6;
constexpr int kW1Ahead = kW1Slots - 1;

struct Window {
    float4 col[kWin];   // backward: {code*rowPad, bg, suf, pre}; forward: {code*rowPad, bg*sC, pre, unused}
    float4 ring[kWin];  // stripe-boundary (W, Y, scale count) for the lane that reads the ring
    float4 w1[kW1Slots][kLanes];  // forward W1 staging ring (lane l uses [slot][l], R floats)
    PairCold cold;      // the pair in flight: fields read only at refills and stripe starts
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

// max(a, b, c) in one instruction (the three-input max.f32 of sm_100).
__device__ __forceinline__ float fmax3(float a, float b, float c) {
    float r;
    asm("max.f32 %0, %1, %2, %3;" : "=f"(r) : "f"(a), "f"(b), "f"(c));
    return r;
}

// The step's share of the float filter best, max over the lane's rows of
// W1 * prefixSeed[j] (fast modes).  A correctly rounded product by prev >= 0
// is monotone in W (with flush to zero as well), so the largest product is
// the product of the largest W, and a NaN W (an overflowed value times a zero
// factor) is passed over by the max in both forms: the same bits with R - 2
// fewer multiplies at R = 4.
template <int R>
__device__ __forceinline__ float stepFilt(float filt, const float (&wv)[R], float prev) {
    if constexpr (R == 4)
        return fmax3(filt, fmax3(wv[0], wv[1], wv[2]) * prev, wv[3] * prev);
    else if constexpr (R == 2)
        return fmax3(filt, wv[0] * prev, wv[1] * prev);
    else
        return fmaxf(filt, wv[0] * prev);
}

// The ring a stripe reads (written by the stripe before it in processing order).
template <bool EXACT>
__device__ __forceinline__ const float *ringOfPrev(const SweepArgs &a, int k) {
    if (!EXACT) return a.ring;
    const int sp = a.sFirst + k * a.sStep;
    return a.ring + (size_t)((sp - 1) % a.ringSlots) * a.ringStride;
}
template <bool EXACT>
__device__ __forceinline__ int stripeOf(const SweepArgs &a, int k) {
    return EXACT ? a.sFirst + k * a.sStep : k;
}

// Backward window entry for local time u (the column of u is L-1 - u mod P).
template <bool EXACT>
__device__ __forceinline__ void fillBackward(Window &w, const SweepArgs &a, int u) {
    const int e = u & (kWin - 1);
    float4 c = make_float4(__int_as_float(kPad * a.rowPad), 0.0f, 0.0f, 0.0f);
    float4 r = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    if (u >= 0 && u < a.nMine * a.P) {
        const int k = u / a.P, jj = u - k * a.P;
        if (jj < a.L) {
            const int j = a.L - 1 - jj;
            const int code = (j + 1 < a.L) ? (int)__ldg(a.codes() + j + 1) : kPad;
            c = make_float4(__int_as_float(code * a.rowPad), a.smBg()[code], __ldg(a.suf() + j), __ldg(a.pre() + j));
            if (stripeOf<EXACT>(a, k) > 0) r = ringLoad(ringOfPrev<EXACT>(a, k), jj);
        }
    }
    w.col[e] = c;
    w.ring[e] = r;
}

// Forward window entry for local time u (the column of u is u mod P).
template <bool EXACT>
__device__ __forceinline__ void fillForward(Window &w, const SweepArgs &a, int u) {
    const int e = u & (kWin - 1);
    float4 c = make_float4(__int_as_float(kPad * a.rowPad), 0.0f, 0.0f, 0.0f);
    float4 r = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    if (u >= 0 && u < a.nMine * a.P) {
        const int k = u / a.P, j = u - k * a.P;
        if (j < a.L) {
            const int code = (j >= 2) ? (int)__ldg(a.codes() + j - 2) : kPad;
            c = make_float4(__int_as_float(code * a.rowPad), a.smBg()[code] * a.sc().sC, __ldg(a.pre() + j), 0.0f);
            if (stripeOf<EXACT>(a, k) > 0) r = ringLoad(ringOfPrev<EXACT>(a, k), j);
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
    float *anchorPart;  // replay with anchors: [stripe][column] x (mantissa, exponent, row), 3 words
};

// scoreLess (dummest-score.hh:70-76) on (mantissa, exponent) pairs.
__device__ __forceinline__ bool xsLessMe(float am, int ae, float bm, int be) {
    if (am == 0.0f) return bm != 0.0f;
    if (bm == 0.0f) return false;
    if (ae != be) return ae < be;
    return am < bm;
}

// ---------------------------------------------------------------------------
// Backward sweep (dummest-dp-backward.hh:473-574; the float filter :367-430).
//
// Steps run in groups of three.  A row's history (W1 and Z at columns j+1,
// j+2, j+3) lives in three register slots whose roles rotate with the step's
// phase PH = t mod 3: slot (3-PH)%3 holds column j+1, (4-PH)%3 column j+2 and
// (5-PH)%3 column j+3, and the new value of column j replaces column j+3.  The
// history then shifts by renaming, with no register copies.
// ---------------------------------------------------------------------------
template <int R, int MODE>
struct BwdState {
    Coef<R> c;
    float h[3][R], z[3][R];  // this lane's rows: W1 and Z history slots
    float rb[3];             // the row below (the next lane's top row): W1 history slots
    float sendW, sendY, filt, maxY;
    int sendC;
    int u, sp, jj;           // lane-local time, stripe from the bottom, column from the right
    float *wp;               // W1 store pointer of the current step
    // exact-path state
    int cnt;                 // discovery: this lane's scale count
    float rmax[R];           // discovery: per-row maxima at count cnt
    int cOut[R];             // replay: count of each row after its decision
    float fOut[R];           // replay: 1 or 2^-64, the row's own rescale
    double rowBest[R];       // replay: per-row max of W1 * prefixSeed
};

// PIPE: the sweep runs one of several warps' stripes of a pair (a stripe
// pipeline: stripes sFirst, sFirst + sStep, ...; ring slot per stripe).
template <int R, int MODE, int PH, bool PIPE = (MODE == kDiscover || MODE == kReplay), bool SH = false>
__device__ __forceinline__ void backwardStep(BwdState<R, MODE> &b, const SweepArgs &a, Window &win, int lane,
                                             int total, const ExactRows *x, ExactBest *exact) {
    constexpr int S = kLanes * R;
    constexpr bool kStore = MODE == kMid || MODE == kReplay;
    constexpr bool kExactMode = MODE == kDiscover || MODE == kReplay;
    constexpr int I1 = (3 - PH) % 3, I2 = (4 - PH) % 3, I3 = (5 - PH) % 3;
    float inW = __shfl_down_sync(kFull, b.sendW, 1);
    float inY = __shfl_down_sync(kFull, b.sendY, 1);
    int inC = 0;
    if (MODE == kDiscover) inC = __shfl_down_sync(kFull, b.sendC, 1);
    const int lag = kLanes - 1 - lane;
    if (b.u >= 0 && b.u < total && b.jj < a.L) {
        const int s = a.nS - 1 - b.sp;
        const int rowBase = s * S + lane * R;
        if (b.jj == 0) {
            loadBackwardCoef<R>(b.c, a, rowBase);
#pragma unroll
            for (int q = 0; q < 3; ++q) {
#pragma unroll
                for (int k = 0; k < R; ++k) b.h[q][k] = b.z[q][k] = 0.0f;
                b.rb[q] = 0.0f;
            }
            b.wp = a.w1 + (((size_t)s * a.D + lag) * kLanes + lane) * R;
            if (MODE == kDiscover) {
                b.cnt = 0;
#pragma unroll
                for (int k = 0; k < R; ++k) b.rmax[k] = 0.0f;
            }
            if (MODE == kReplay) {
#pragma unroll
                for (int k = 0; k < R; ++k) {
                    const int i = rowBase + k;
                    const int ci = i <= a.M() ? i : a.M() + 1;
                    const int cIn = x->cntB[ci + 1 <= a.M() + 1 ? ci + 1 : a.M() + 1];
                    b.cOut[k] = x->cntB[ci];
                    b.fOut[k] = stepsDown(b.cOut[k] - cIn);
                    b.c.rs[k] = seedCoef(i <= a.M(), cIn);
                    b.rowBest[k] = 0.0;
                }
            }
        }
        const int slot = b.u & (kWin - 1);
        const float4 col = win.col[slot];
        if (lane == kLanes - 1) {
            const float4 r = win.ring[slot];
            inW = r.x;
            inY = r.y;
            if (MODE == kDiscover) inC = __float_as_int(r.z);
        }
        if (MODE == kDiscover) {
            // Align the incoming values and this lane to one scale.
            if (inC > b.cnt) {
                const float f = stepsDown(inC - b.cnt);
#pragma unroll
                for (int k = 0; k < R; ++k) {
#pragma unroll
                    for (int q = 0; q < 3; ++q) {
                        b.h[q][k] *= f;
                        b.z[q][k] *= f;
                    }
                    b.rmax[k] *= f;
                    b.c.rs[k] = seedCoef(rowBase + k <= a.M(), inC);
                }
#pragma unroll
                for (int q = 0; q < 3; ++q) b.rb[q] *= f;
                b.cnt = inC;
            } else if (inC < b.cnt) {
                const float f = stepsDown(b.cnt - inC);
                inW *= f;
                inY *= f;
            }
        }
        const int eOff = __float_as_int(col.x);  // code * rowPad
        const float bgv = col.y, sufv = col.z, prev = col.w;
        float e[R];
        if (SH)  // the table in shared memory: a plain shared load
            loadEmitS<R>(e, (unsigned)__cvta_generic_to_shared(a.smE) + 4u * (unsigned)(eOff + rowBase));
        else
            loadEmit<R>(e, a.smE + eOff + rowBase);
        // First products (W1[i+1][j+3] * e) * enter, taken before any row of
        // this step overwrites its column-j+3 slot.
        float p[R];
        p[R - 1] = (b.rb[I3] * e[R - 1]) * b.c.enter[R - 1];
#pragma unroll
        for (int k = 0; k < R - 1; ++k) {
            const float h3 = (MODE == kReplay) ? b.h[I3][k + 1] * b.fOut[k + 1] : b.h[I3][k + 1];
            p[k] = (h3 * e[k]) * b.c.enter[k];
        }
        float bW1 = b.rb[I1], bW2 = b.rb[I2], bY = inY;
        float wv[R], yv[R];
        float stepMax = 0.0f;
#pragma unroll
        for (int k = R - 1; k >= 0; --k) {
            float acc = p[k];
            acc = __fmaf_rn(bY, b.c.d0[k], acc);
            acc = __fmaf_rn(bW2, b.c.d1[k], acc);
            acc = __fmaf_rn(bW1, b.c.d2[k], acc);
            const float zbg = b.z[I3][k] * bgv;
            acc = __fmaf_rn(zbg, b.c.a0[k], acc);
            acc = __fmaf_rn(b.h[I2][k], b.c.a2[k], acc);
            acc = __fmaf_rn(b.h[I1][k], b.c.a1[k], acc);
            // Seed term fma(suf, rs, acc): in the fast modes rs is 1 on real
            // rows, where the fma is the exact sum suf + acc (one rounding, as
            // the reference's add), and 0 on rows past M, which accumulate
            // exactly 0 and must stay 0.
            const float W = __fmaf_rn(sufv, b.c.rs[k], acc);
            const float Y = __fmaf_rn(b.c.eps[k], bY, W);
            const float Z = __fmaf_rn(b.c.b0[k], zbg, W);
            if (MODE == kFilter || MODE == kMid) yv[k] = Y;
            if (MODE == kDiscover) {
                b.rmax[k] = fmaxf(b.rmax[k], Y);  // Y >= W1 at every cell
                stepMax = fmaxf(stepMax, Y);
            }
            if (MODE == kReplay) {
                if (a.alignOut != nullptr && rowBase + k <= a.M())
                    a.alignOut[(size_t)(rowBase + k) * a.L + (a.L - 1 - b.jj)] = W;
                // What leaves the row is scaled by the row's own decision.
                const float Wo = W * b.fOut[k];
                b.rowBest[k] = fmax(b.rowBest[k], (double)Wo * (double)prev);
                bW1 = b.h[I1][k] * b.fOut[k];
                bW2 = b.h[I2][k] * b.fOut[k];
                bY = Y * b.fOut[k];
                wv[k] = Wo;
            } else {
                bW1 = b.h[I1][k];
                bW2 = b.h[I2][k];
                bY = Y;
                wv[k] = W;
            }
            b.h[I3][k] = W;
            b.z[I3][k] = Z;
        }
        if (MODE == kFilter || MODE == kMid) {
            // running maxima, two rows per three-input max
#pragma unroll
            for (int k = 0; k < R; k += 2) b.maxY = (k + 1 < R) ? fmax3(b.maxY, yv[k], yv[k + 1]) : fmaxf(b.maxY, yv[k]);
            b.filt = stepFilt<R>(b.filt, wv, prev);
        }
        b.rb[I3] = inW;
        b.sendW = wv[0];
        b.sendY = bY;
        if (MODE == kDiscover) {
            if (stepMax > kBump) {
#pragma unroll
                for (int k = 0; k < R; ++k) {
#pragma unroll
                    for (int q = 0; q < 3; ++q) {
                        b.h[q][k] *= kStep;
                        b.z[q][k] *= kStep;
                    }
                    b.rmax[k] *= kStep;
                    b.c.rs[k] = seedCoef(rowBase + k <= a.M(), b.cnt + 1);
                }
#pragma unroll
                for (int q = 0; q < 3; ++q) b.rb[q] *= kStep;
                b.sendW *= kStep;
                b.sendY *= kStep;
                ++b.cnt;
            }
            b.sendC = b.cnt;
        }
        if (kStore) {
            storeW1<R>(b.wp, wv);
            b.wp += kLanes * R;
        }
        if (lane == 0 && b.sp < a.nS - 1) {
            float *rg = PIPE ? a.ring + (size_t)(b.sp % a.ringSlots) * a.ringStride : a.ring;
            if (MODE == kDiscover)
                ringStore(rg, b.jj, b.sendW, b.sendY, b.sendC);
            else
                ringStore(rg, b.jj, b.sendW, b.sendY);
        }
        if (b.jj == a.L - 1) {
            // the last column of these rows
#pragma unroll
            for (int k = 0; k < R; ++k) {
                const int i = rowBase + k;
                if (i > a.M()) continue;
                if (MODE == kDiscover) {
                    x->rowMax[i] = b.rmax[k];
                    x->rowCnt[i] = b.cnt;
                }
                if (MODE == kReplay) foldBest(*exact, b.rowBest[k], b.cOut[k]);
            }
        }
    } else {
        b.sendW = 0.0f;
        b.sendY = 0.0f;
        b.sendC = 0;
    }
    if (b.u >= 0 && ++b.jj == a.P) {
        b.jj = 0;
        b.sp += PIPE ? a.sStep : 1;
    }
    ++b.u;
}

// Window refills for a block of kBlock steps starting at t0: local times
// [t0 + kBlock, t0 + 2 kBlock), one entry per lane and pass.
template <bool BACKWARD, bool EXACT = false>
__device__ __forceinline__ void fillBlock(Window &win, const SweepArgs &a, int first, int lane) {
#pragma unroll
    for (int o = 0; o < kBlock; o += kLanes) {
        if (o + lane < kBlock) {
            if (BACKWARD)
                fillBackward<EXACT>(win, a, first + o + lane);
            else
                fillForward<EXACT>(win, a, first + o + lane);
        }
    }
}

// Asynchronous global-to-shared copies of W1 (cp.async: the copy bypasses the
// registers; cp.async.wait_group orders it before the lane's own reads).
template <int R>
__device__ __forceinline__ void cpAsyncW1(float4 *dst, const float *src) {
    const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
    if constexpr (R == 4)
        asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(d), "l"(src) : "memory");
    else
        asm volatile("cp.async.ca.shared.global [%0], [%1], %2;" ::"r"(d), "l"(src), "n"(4 * R) : "memory");
}
__device__ __forceinline__ void cpAsyncCommit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cpAsyncWait() {
    asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

// W1 staging cursor of the forward sweep: the lane-local time whose W1 is
// copied next (kW1Ahead steps ahead of the lane).  Every call commits one
// group, empty for steps the lane does not compute.
template <int R, bool EXACT = false>
struct W1Stage {
    int u, s, j;
    __device__ __forceinline__ void issue(const SweepArgs &a, Window &win, int slot, int lane, int total) {
        if (u >= 0 && u < total && j < a.L) {
            const int db = (a.L - 1 - j) + (kLanes - 1 - lane);
            cpAsyncW1<R>(&win.w1[slot][lane], a.w1 + (((size_t)s * a.D + db) * kLanes + lane) * R);
        }
        cpAsyncCommit();
        if (u >= 0 && ++j == a.P) {
            j = 0;
            s += EXACT ? a.sStep : 1;
        }
        ++u;
    }
};

template <int R, int MODE>
struct FwdState {
    Coef<R> c;
    float w[3][R], z[3][R];  // W0 and Z0 history slots (rotating roles, see backwardStep)
    float sendIn, sendY, best, mx;
    int sendC;
    // anchors: the column's best wMid over the rows below and this lane's (mantissa, exponent, row)
    float sendAM;
    int sendAE, sendAR;
    int u, s, j;
    // exact-path state (see BwdState)
    int cnt;
    float rmax[R];
    int cIn[R], cB[R];
    float fOut[R];
    double rowBest[R];
};

// One forward step of a lane (dummest-dp-forward.hh:112-223) at phase PH;
// q holds the W1 values of this step.  Slot (3-PH)%3 holds column j-1,
// (4-PH)%3 column j-2, (5-PH)%3 column j-3, which the new column j replaces.
// ANCH (replay only): also the per-column anchors of the hit path
// (dummest-dp-forward.hh:196-206): each column's best wMid over the rows and
// its row passes up the lanes with the column, each lane folding its rows in
// ascending order with scoreLess (the first row wins ties); the stripe's top
// lane writes the stripe's partial, and the stripes are folded in order after
// the sweep.
template <int R, int MODE, int PH, bool ANCH = false, bool PIPE = (MODE == kDiscover || MODE == kReplay),
          bool SH = false>
__device__ __forceinline__ void forwardStep(FwdState<R, MODE> &f, const SweepArgs &a, Window &win, int lane,
                                            int total, const float (&q)[R], const ExactRows *x, ExactBest *exact) {
    constexpr int S = kLanes * R;
    constexpr bool kExactMode = MODE == kDiscover || MODE == kReplay;
    constexpr int I1 = (3 - PH) % 3, I2 = (4 - PH) % 3, I3 = (5 - PH) % 3;
    float inW = __shfl_up_sync(kFull, f.sendIn, 1);
    float inY = __shfl_up_sync(kFull, f.sendY, 1);
    float aM = 0.0f;
    int aE = 0, aR = 0;
    if (ANCH) {
        aM = __shfl_up_sync(kFull, f.sendAM, 1);
        aE = __shfl_up_sync(kFull, f.sendAE, 1);
        aR = __shfl_up_sync(kFull, f.sendAR, 1);
        if (lane == 0) {  // the rows below are the previous stripe's: a partial of this stripe
            aM = 0.0f;
            aE = aR = 0;
        }
    }
    int inC = 0;
    if (MODE == kDiscover) inC = __shfl_up_sync(kFull, f.sendC, 1);
    if (f.u >= 0 && f.u < total && f.j < a.L) {
        const int rowBase = f.s * S + lane * R;
        if (f.j == 0) {
            loadForwardCoef<R>(f.c, a, rowBase);
#pragma unroll
            for (int h = 0; h < 3; ++h)
#pragma unroll
                for (int k = 0; k < R; ++k) f.w[h][k] = f.z[h][k] = 0.0f;
            if (MODE == kDiscover) {
                f.cnt = 0;
#pragma unroll
                for (int k = 0; k < R; ++k) f.rmax[k] = 0.0f;
            }
            if (MODE == kReplay) {
#pragma unroll
                for (int k = 0; k < R; ++k) {
                    const int i = rowBase + k;
                    const int ci = i <= a.M() ? i : a.M();
                    f.cIn[k] = x->cntF[ci];
                    f.fOut[k] = stepsDown(x->cntF[ci + 1] - f.cIn[k]);
                    f.cB[k] = x->cntB[ci];
                    f.c.rs[k] = seedCoef(i <= a.M(), f.cIn[k]);
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
#pragma unroll
                    for (int h = 0; h < 3; ++h) {
                        f.w[h][k] *= g;
                        f.z[h][k] *= g;
                    }
                    f.rmax[k] *= g;
                    f.c.rs[k] = seedCoef(rowBase + k <= a.M(), inC);
                }
                f.cnt = inC;
            } else if (inC < f.cnt) {
                const float g = stepsDown(f.cnt - inC);
                inW *= g;
                inY *= g;
            }
        }
        const int eOff = __float_as_int(col.x);  // code * rowPad
        const float bgsC = col.y, prev = col.z;
        float e[R];
        if (SH)  // the table in shared memory: a plain shared load
            loadEmitS<R>(e, (unsigned)__cvta_generic_to_shared(a.smE) + 4u * (unsigned)(eOff + rowBase));
        else
            loadEmit<R>(e, a.smE + eOff + rowBase);
        float win0 = inW, yab = inY;
        float stepMax = 0.0f;
        float bv[R];
#pragma unroll
        for (int k = 0; k < R; ++k) {
            const float w1 = f.w[I1][k], w2 = f.w[I2][k], w3 = f.w[I3][k];
            // The reference's operations as GCC contracts them at -O3
            // (dummest-dp-forward.hh:116-222): Z0 = (bg*sC)*fma(b0, Z0[j-3],
            // a0*w3); the alpha1/alpha2 products fuse into the W0 sum, and
            // Y0 = fma(eps, Y0[i-1], d0*W0).
            const float X = (f.c.enter[k] * e[k]) * w3;
            const float Z0 = bgsC * __fmaf_rn(f.c.b0[k], f.z[I3][k], f.c.a0[k] * w3);
            const float zs = __fmaf_rn(f.c.a2[k], w2, __fmaf_rn(f.c.a1[k], w1, Z0));
            // fma(prev, 1, x) is prev + x; in the fast mode every row takes the
            // seed: padding rows (past M, zero coefficients) then hold only
            // their seed, which reaches no real row and multiplies a zero W1.
            const float W0 = (MODE == kMid) ? win0 + __fadd_rn(zs, prev) : win0 + __fmaf_rn(prev, f.c.rs[k], zs);
            if (MODE == kMid) bv[k] = W0 * q[k];
            if (MODE == kReplay) {
                f.rowBest[k] = fmax(f.rowBest[k], (double)W0 * (double)q[k]);
                if (a.alignOut != nullptr && rowBase + k <= a.M()) a.alignOut[(size_t)(rowBase + k) * a.L + f.j] = W0;
            }
            if (ANCH) {
                // wMid = promote(W0) * promote(W1): the exact double product,
                // its mantissa rounded to float (dummest-batch.hh:216-235)
                const double v = (double)W0 * (double)q[k];
                if (rowBase + k <= a.M() && v > 0.0) {
                    // frexp of v from its bits: v, a product of two positive
                    // normal floats, is a normal double
                    const unsigned long long u = (unsigned long long)__double_as_longlong(v);
                    const int ev = (int)((u >> 52) & 0x7FFULL) - 1022;
                    const double mv = __longlong_as_double((long long)((u & 0xFFFFFFFFFFFFFULL) | (1022ULL << 52)));
                    const float cm = __double2float_rn(mv);
                    const int ce = ev + kRescaleBits * (f.cIn[k] + f.cB[k]);
                    if (xsLessMe(aM, aE, cm, ce)) {
                        aM = cm;
                        aE = ce;
                        aR = rowBase + k;
                    }
                }
            }
            const float Y0 = __fmaf_rn(f.c.eps[k], yab, f.c.d0[k] * W0);
            if (MODE == kMid) f.mx = fmax3(f.mx, W0, Y0);
            const float nin = __fmaf_rn(f.c.d2[k], w1, __fmaf_rn(f.c.d1[k], w2, X + Y0));
            if (MODE == kDiscover) {
                f.rmax[k] = fmaxf(f.rmax[k], fmaxf(W0, Y0));
                stepMax = fmaxf(stepMax, fmaxf(fmaxf(W0, Y0), nin));
            }
            f.w[I3][k] = W0;
            f.z[I3][k] = Z0;
            if (MODE == kReplay) {
                win0 = nin * f.fOut[k];
                yab = Y0 * f.fOut[k];
            } else {
                win0 = nin;
                yab = Y0;
            }
        }
        if (MODE == kMid) {
#pragma unroll
            for (int k = 0; k < R; k += 2) f.best = (k + 1 < R) ? fmax3(f.best, bv[k], bv[k + 1]) : fmaxf(f.best, bv[k]);
        }
        if (MODE == kDiscover) {
            if (stepMax > kBump) {
#pragma unroll
                for (int k = 0; k < R; ++k) {
#pragma unroll
                    for (int h = 0; h < 3; ++h) {
                        f.w[h][k] *= kStep;
                        f.z[h][k] *= kStep;
                    }
                    f.rmax[k] *= kStep;
                    f.c.rs[k] = seedCoef(rowBase + k <= a.M(), f.cnt + 1);
                }
                win0 *= kStep;
                yab *= kStep;
                ++f.cnt;
            }
            f.sendC = f.cnt;
        }
        f.sendIn = win0;
        f.sendY = yab;
        if (ANCH) {
            f.sendAM = aM;
            f.sendAE = aE;
            f.sendAR = aR;
            if (lane == kLanes - 1) {
                float *pp = x->anchorPart + ((size_t)f.s * a.L + f.j) * 3;
                pp[0] = aM;
                pp[1] = __int_as_float(aE);
                pp[2] = __int_as_float(aR);
            }
        }
        if (lane == kLanes - 1 && f.s < a.nS - 1) {
            float *rg = PIPE ? a.ring + (size_t)(f.s % a.ringSlots) * a.ringStride : a.ring;
            if (MODE == kDiscover)
                ringStore(rg, f.j, f.sendIn, f.sendY, f.sendC);
            else
                ringStore(rg, f.j, f.sendIn, f.sendY);
        }
        if (f.j == a.L - 1) {
#pragma unroll
            for (int k = 0; k < R; ++k) {
                const int i = rowBase + k;
                if (i > a.M()) continue;
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
        if (ANCH) {
            f.sendAM = 0.0f;
            f.sendAE = f.sendAR = 0;
        }
    }
    if (f.u >= 0 && ++f.j == a.P) {
        f.j = 0;
        f.s += PIPE ? a.sStep : 1;
    }
    ++f.u;
}

// One forward step at position P6 of a six-step group: wait for this step's
// W1 copy, read it from the staging ring, run the step, and stage the W1 of
// the step kW1Ahead later into the slot this lane read one step ago.
template <int R, int MODE, int P6, bool ANCH = false, bool PIPE = (MODE == kDiscover || MODE == kReplay),
          bool SH = false>
__device__ __forceinline__ void forwardStaged(FwdState<R, MODE> &f, const SweepArgs &a, Window &win, int lane,
                                              int total, W1Stage<R, PIPE> &st,
                                              const ExactRows *x, ExactBest *exact) {
    constexpr bool kReadW1 = MODE == kMid || MODE == kReplay;
    float q[R];
    if (kReadW1) {
        cpAsyncWait<kW1Ahead - 1>();
        const float4 v = win.w1[P6][lane];
        q[0] = v.x;
        if constexpr (R > 1) q[1] = v.y;
        if constexpr (R > 2) {
            q[2] = v.z;
            q[3] = v.w;
        }
    } else {
#pragma unroll
        for (int k = 0; k < R; ++k) q[k] = 0.0f;
    }
    forwardStep<R, MODE, P6 % 3, ANCH, PIPE, SH>(f, a, win, lane, total, q, x, exact);
    if (kReadW1) st.issue(a, win, (P6 + kW1Ahead) % kW1Slots, lane, total);
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
    const int *pairIdx;  // null: chunk c holds pairs first .. first+count-1; else pairIdx[first + k]
};

// CTA shapes: WARPS warps share one shared-memory copy of the profile's
// emission table, one CTA per SM; 16 warps leave 128 registers per thread,
// 12 warps 168 and 8 warps 255.  The autotuner picks the shape per
// rows-per-lane value.
constexpr int kCtaWarps = 16;       // the default (and widest) shape
constexpr int kCtaWarpsNarrow = 8;
constexpr int kCtaWarpsMid = 12;

}  // namespace dmst
