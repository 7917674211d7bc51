// The batched wavefront DP with staggered rows: one warp per (read, profile)
// pair, R rows per lane, and the R rows of a lane one column apart.
//
// Layout.  As in the stripe layout of dp_wavefront.cuh, lane l owns rows
// l*R .. l*R+R-1 of a stripe of S = 32 R rows.  Here every row lags the row it
// depends on by exactly one step (backward: row i+1 leads row i; forward: row
// i-1 leads row i), inside a lane as well as across lanes: lane l's row k lags
// the stripe's leading row by
//   backward  (31 - l) R + (R - 1 - k)      forward  l R + k.
// A row's operands from the neighbouring row were then produced one or more
// steps earlier, so the R rows of a lane are independent within a step: four
// dependency chains of one row each instead of one chain through four rows,
// which is what bounds the row-contiguous layout (the reference's FMA order
// puts the row below's Y first, so a row cannot start before the row below
// has finished).  The arithmetic per cell is unchanged, term for term, so the
// results are the same bits.
//
// Values crossing rows inside a lane are register histories; the lane's
// boundary row crosses lanes through one warp shuffle per value, and the
// stripe's boundary row crosses stripes through a per-warp ring in global
// memory.  Only a lane's leading row reads the staging window; its other
// rows take the same column operands one to R-1 steps later from register
// delay lines (the roles rotate with the step's phase, so nothing is copied).
//
// Stripes follow each other with no bubble (a lane starts its next stripe as
// soon as its leading row finishes the last column).  The period P of a stripe
// is at least L + 3: the last three steps of a row's stripe are idle and
// write zeros, so that every history entry a row reads at the start of its
// next stripe is zero, and a lane's other rows are idle while its leading row
// takes the next stripe's coefficients.  Idle steps are handled by masks in
// the general steps; the interior steps (every row of every lane inside one
// stripe) run without them.
//
// W1 is stored by warp step: the backward's step t writes the lane's R values
// (its rows, each at its own column) to group t of the warp's slot, and the
// forward's step t' = (nS-1) P + L + S - 2 - t needs exactly those cells, so a
// step's store and load are each one contiguous access of 32 lanes x R floats
// (at R = 3 each lane's three values take a 16-byte entry, so that the store,
// the forward's staging copy and its shared load are one instruction each).
//
// The recurrences are the reference's, term for term and in the same
// association order:
//   backward  dummest-dp-backward.hh:473-574 (and the float filter :367-430)
//   forward   dummest-dp-forward.hh:63-250
#pragma once

#include "dp_wavefront.cuh"

namespace dmst {

constexpr int kSBlock = 32;     // steps per block: one window entry per lane per block
constexpr int kSWin = 256;      // column window entries (lane-local times), a power of two
constexpr int kSRingWin = 128;  // ring window entries (read by the stripe's leading lane only)
constexpr int kSW1Slots = 8;    // forward W1 staging slots (cp.async, one group per step)
constexpr int kSW1Ahead = kSW1Slots - 1;

// Period of a stripe: L + 3 (three idle steps per row and stripe), and at
// least S + 2 kSBlock + 31, so that the ring value a stripe's lowest row
// writes is stored at least one block before the window refill that loads it
// for the next stripe's leading row (which happens two blocks ahead).
__host__ __device__ inline int stagPeriod(int L, int R) {
    const int lo = kLanes * R + 2 * kSBlock + kLanes - 1;
    return L + 3 > lo ? L + 3 : lo;
}
// Steps of one sweep: the last cell is the stripe's lagging row (lag S - 1)
// at column L - 1 of the last stripe.
__host__ __device__ inline long long stagSteps(int M, int L, int R) {
    const int S = kLanes * R;
    const long long nS = (M + 1 + S - 1) / S;
    return (nS - 1) * stagPeriod(L, R) + L - 1 + S;
}
// Floats per lane in a W1 group: R, and 4 at R = 3, so that a lane's values
// are one 16-byte store, copy and load (the fourth float is padding).
__host__ __device__ constexpr int stagLaneStride(int R) { return R == 3 ? 4 : R; }
// W1 slot of one pair: one group of 32 stagLaneStride(R) floats per step,
// steps rounded up to the forward's eight-step groups.
__host__ __device__ inline long long stagSlotFloats(int M, int L, int R) {
    return (stagSteps(M, L, R) + kSW1Slots - 1) / kSW1Slots * kSW1Slots * (long long)(kLanes * stagLaneStride(R));
}

// Per-warp staging: the column operands by lane-local time, the ring values
// of the leading lane, and the forward's W1 staging ring.  Entry e of each
// circular window is also kept at e + size for e < kSBlock (a mirrored tail),
// so that the up to kSBlock entries a lane reads in one block are consecutive
// from the block's first one: the interior steps address them from one base
// with constant offsets.
template <int R>
struct WindowS {
    float4 col[kSWin + kSBlock];  // backward {code*rowPad, bg, suf, pre}; forward {code*rowPad, bg*sC, pre, 0}
    float2 ring[kSRingWin + kSBlock];
    float w1[kSW1Slots][kLanes * stagLaneStride(R)];
    PairCold cold;
};

// A window entry as loaded from global memory (one per lane per block, held
// in registers for a block so that the loads' latency is off the steps).
struct FillRegs {
    int code;
    float suf, pre, rw, ry;
};

template <bool BACKWARD>
__device__ __forceinline__ FillRegs fillLoadS(const SweepArgs &a, int u) {
    FillRegs f{kPad, 0.0f, 0.0f, 0.0f, 0.0f};
    if (u >= 0 && u < a.nS * a.P) {
        const int k = u / a.P, jj = u - k * a.P;
        if (jj < a.L) {
            if (BACKWARD) {
                const int j = a.L - 1 - jj;
                f.code = (j + 1 < a.L) ? (int)__ldg(a.codes() + j + 1) : kPad;
                f.suf = __ldg(a.suf() + j);
                f.pre = __ldg(a.pre() + j);
            } else {
                f.code = (jj >= 2) ? (int)__ldg(a.codes() + jj - 2) : kPad;
                f.pre = __ldg(a.pre() + jj);
            }
            if (k > 0) {
                const float2 r = __ldcg(reinterpret_cast<const float2 *>(a.ring) + jj);
                f.rw = r.x;
                f.ry = r.y;
            }
        }
    }
    return f;
}

template <bool BACKWARD, int R>
__device__ __forceinline__ void fillStoreS(WindowS<R> &w, const SweepArgs &a, const FillRegs &f, int u) {
    const float bg = a.smBg()[f.code];
    const float4 c = BACKWARD ? make_float4(__int_as_float(f.code * a.rowPad), bg, f.suf, f.pre)
                              : make_float4(__int_as_float(f.code * a.rowPad), bg * a.sc().sC, f.pre, 0.0f);
    const float2 r = make_float2(f.rw, f.ry);
    const int e = u & (kSWin - 1), e2 = u & (kSRingWin - 1);
    w.col[e] = c;
    if (e < kSBlock) w.col[e + kSWin] = c;
    w.ring[e2] = r;
    if (e2 < kSBlock) w.ring[e2 + kSRingWin] = r;
}

// A lane's R values of one W1 group (R = 3: one 16-byte store, padding last).
template <int R>
__device__ __forceinline__ void storeW1S(float *p, const float (&w)[R]) {
    if constexpr (R == 3)
        *reinterpret_cast<float4 *>(p) = make_float4(w[0], w[1], w[2], 0.0f);
    else
        storeW1<R>(p, w);
}

__device__ __forceinline__ void ringStoreS(float *ring, int col, float w, float y) {
    __stcg(reinterpret_cast<float2 *>(ring) + col, make_float2(w, y));
}

// The window's first entries: local times [-S, kSBlock) now (the leading rows
// of the lanes read from -(31 R) on), and the block after into registers.
template <bool BACKWARD, int R>
__device__ __forceinline__ FillRegs fillPrologueS(WindowS<R> &win, const SweepArgs &a, int lane) {
    constexpr int S = kLanes * R;
    for (int v = -S + lane; v < kSBlock; v += kLanes) fillStoreS<BACKWARD, R>(win, a, fillLoadS<BACKWARD>(a, v), v);
    return fillLoadS<BACKWARD>(a, kSBlock + lane);
}

// The interior steps of a block starting at t0 with n steps: [gA, gB) relative
// to t0, in groups of G steps.  A step t is interior when every row of every
// lane is inside stripe sp and active, and no lane starts the stripe at t:
// sp P + S <= t <= sp P + L - 1 (the same bounds in both sweeps; the last lane
// to start a stripe starts it at sp P + S - R).  At most one stripe's interior
// meets a block (between two interiors lie P - L + S > kSBlock general steps).
template <int G>
__device__ __forceinline__ int interiorRunS(const SweepArgs &a, int S, int t0, int n, int &gA, int &gB) {
    gA = gB = 0;
    const int last = t0 + n - 1 - S;
    if (last < 0) return -1;
    const int sp = last / a.P;
    if (sp >= a.nS) return -1;
    const int lo = max(t0, sp * a.P + S), hi = min(t0 + n - 1, sp * a.P + a.L - 1);
    if (lo > hi) return -1;
    gA = (lo - t0 + G - 1) / G * G;
    gB = (hi - t0 + 1) / G * G;
    if (gB <= gA) {
        gA = gB = 0;
        return -1;
    }
    return sp;
}

// ---------------------------------------------------------------------------
// Backward sweep.  Phase PH = t mod 4: slot (PH - d) & 3 of a row's W1 and Z
// histories holds its value from d steps ago.  Row k (k < R - 1) reads row
// k+1's W1 at columns j+1, j+2, j+3 (that row's values from 2, 3 and 4 steps
// ago) and its Y at column j (from the previous step); the lane's leading row
// reads the lane below through the shuffled values of the last four steps.
// ---------------------------------------------------------------------------
// Addresses of an interior run: the window entries of its first step (the
// mirrored tails keep a block's entries consecutive), the W1 group of its
// first step and the ring column its stripe-boundary writer starts at.  The
// steps of a group address them with constant offsets; the run advances them
// once per group.
struct RunPtrs {
    const float4 *col;
    const float2 *ring;
    float *w1;           // backward: W1 store; forward: the W1 group staged next
    float2 *ringOut;
};

template <int R>
struct BwdS {
    Coef<R> c;
    float h[4][R], z[4][R], rb[4], yPrev[R];
    float bgH[4], sufH[4], preH[4], evH[4][R];
    float sendW, sendY, filt, maxY;
    int u, jj, sp;
    float *wp;        // W1 group of the current step (this lane's R values)
    unsigned eS;      // emission rows of the lane: 32-bit shared address (table in shared memory)
    const float *eG;  // or the global address (tall profiles)
};

template <int R, bool MID, int PH, bool GEN, bool SH>
__device__ __forceinline__ void bwdStepS(BwdS<R> &b, const SweepArgs &a, WindowS<R> &win, int lane,
                                         bool ringWriter, const RunPtrs &ip) {
    constexpr int S = kLanes * R;
    constexpr int SW = kLanes * stagLaneStride(R);  // floats per W1 group
    float inW = __shfl_down_sync(kFull, b.sendW, 1);
    float inY = __shfl_down_sync(kFull, b.sendY, 1);
    if (GEN && b.u >= 0 && b.jj == 0 && b.sp < a.nS) {
        // the leading row starts a stripe; the lane's other rows are idle
        const int rowBase = (a.nS - 1 - b.sp) * S + lane * R;
        loadBackwardCoef<R>(b.c, a, rowBase);
        if (SH)
            b.eS = (unsigned)__cvta_generic_to_shared(a.smE + rowBase);
        else
            b.eG = a.smE + rowBase;
    }
    const float4 col = GEN ? win.col[b.u & (kSWin - 1)] : ip.col[PH];
    if (lane == kLanes - 1) {
        const float2 r = GEN ? win.ring[b.u & (kSRingWin - 1)] : ip.ring[PH];
        inW = r.x;
        inY = r.y;
    }
    float ev[R];
    if (SH)
        loadEmitS<R>(ev, b.eS + 4u * (unsigned)__float_as_int(col.x));
    else
        loadEmit<R>(ev, b.eG + __float_as_int(col.x));
    b.bgH[PH] = col.y;
    b.sufH[PH] = col.z;
    b.preH[PH] = col.w;
#pragma unroll
    for (int k = 0; k < R; ++k) b.evH[PH][k] = ev[k];
    b.rb[PH] = inW;
    float nW[R], nY[R], nZ[R], pv[R];
#pragma unroll
    for (int k = 0; k < R; ++k) {
        const int D = R - 1 - k;      // steps behind the lane's leading row
        const int Q = (PH + 4 - D) & 3;
        const float e = b.evH[Q][k], bgv = b.bgH[Q], sufv = b.sufH[Q];
        pv[k] = b.preH[Q];
        float Wb1, Wb2, Wb3, Yb;  // the row below: W1 at columns j+1, j+2, j+3 and Y at j
        if (k == R - 1) {
            Wb1 = b.rb[(PH + 3) & 3];
            Wb2 = b.rb[(PH + 2) & 3];
            Wb3 = b.rb[(PH + 1) & 3];
            Yb = inY;
        } else {
            Wb1 = b.h[(PH + 2) & 3][k + 1];
            Wb2 = b.h[(PH + 1) & 3][k + 1];
            Wb3 = b.h[PH][k + 1];
            Yb = b.yPrev[k + 1];
        }
        const float h1 = b.h[(PH + 3) & 3][k], h2 = b.h[(PH + 2) & 3][k], z3 = b.z[(PH + 1) & 3][k];
        const float p = (Wb3 * e) * b.c.enter[k];
        float acc = __fmaf_rn(Yb, b.c.d0[k], p);
        acc = __fmaf_rn(Wb2, b.c.d1[k], acc);
        acc = __fmaf_rn(Wb1, b.c.d2[k], acc);
        const float zbg = z3 * bgv;
        acc = __fmaf_rn(zbg, b.c.a0[k], acc);
        acc = __fmaf_rn(h2, b.c.a2[k], acc);
        acc = __fmaf_rn(h1, b.c.a1[k], acc);
        // seed term: rs is 1 on real rows (the fma is the exact sum) and 0 on
        // padding rows, which stay 0
        float W = __fmaf_rn(sufv, b.c.rs[k], acc);
        float Y = __fmaf_rn(b.c.eps[k], Yb, W);
        float Z = __fmaf_rn(b.c.b0[k], zbg, W);
        if (GEN) {
            const bool act = b.u >= 0 && b.sp < a.nS && b.jj >= D && b.jj < a.L + D;
            if (!act) W = Y = Z = 0.0f;
        }
        nW[k] = W;
        nY[k] = Y;
        nZ[k] = Z;
    }
    if constexpr (R == 4) {
        b.maxY = fmax3(b.maxY, nY[0], nY[1]);
        b.maxY = fmax3(b.maxY, nY[2], nY[3]);
        b.filt = fmax3(b.filt, nW[0] * pv[0], nW[1] * pv[1]);
        b.filt = fmax3(b.filt, nW[2] * pv[2], nW[3] * pv[3]);
    } else if constexpr (R == 3) {
        b.maxY = fmax3(b.maxY, nY[0], nY[1]);
        b.maxY = fmaxf(b.maxY, nY[2]);
        b.filt = fmax3(b.filt, nW[0] * pv[0], nW[1] * pv[1]);
        b.filt = fmaxf(b.filt, nW[2] * pv[2]);
    } else if constexpr (R == 2) {
        b.maxY = fmax3(b.maxY, nY[0], nY[1]);
        b.filt = fmax3(b.filt, nW[0] * pv[0], nW[1] * pv[1]);
    } else {
        b.maxY = fmaxf(b.maxY, nY[0]);
        b.filt = fmaxf(b.filt, nW[0] * pv[0]);
    }
#pragma unroll
    for (int k = 0; k < R; ++k) {
        b.h[PH][k] = nW[k];
        b.z[PH][k] = nZ[k];
        b.yPrev[k] = nY[k];
    }
    b.sendW = nW[0];
    b.sendY = nY[0];
    // the stripe's lowest row (lane 0, row 0) hands its row to the next stripe
    if (GEN) {
        if (MID) storeW1S<R>(b.wp, nW);
        b.wp += SW;
        if (lane == 0 && b.u >= 0 && b.sp < a.nS - 1 && b.jj >= R - 1 && b.jj < a.L + R - 1)
            ringStoreS(a.ring, b.jj - (R - 1), nW[0], nY[0]);
        if (b.u >= 0 && ++b.jj == a.P) {
            b.jj = 0;
            ++b.sp;
        }
        ++b.u;
    } else {  // the run advances u, jj and the W1 pointer
        if (MID) storeW1S<R>(ip.w1 + PH * SW, nW);
        if (ringWriter) __stcg(ip.ringOut + PH, make_float2(nW[0], nY[0]));
    }
}

template <int R, bool MID, bool SH>
__device__ void backwardSweepS(const SweepArgs &a, WindowS<R> &win, int lane, float &filtOut, float &maxYOut) {
    constexpr int S = kLanes * R;
    constexpr int SW = kLanes * stagLaneStride(R);  // floats per W1 group
    BwdS<R> b;
#pragma unroll
    for (int q = 0; q < 4; ++q) {
#pragma unroll
        for (int k = 0; k < R; ++k) b.h[q][k] = b.z[q][k] = b.evH[q][k] = 0.0f;
        b.rb[q] = b.bgH[q] = b.sufH[q] = b.preH[q] = 0.0f;
    }
#pragma unroll
    for (int k = 0; k < R; ++k) {
        b.yPrev[k] = 0.0f;
        b.c.enter[k] = b.c.a0[k] = b.c.a1[k] = b.c.a2[k] = b.c.b0[k] = 0.0f;
        b.c.d0[k] = b.c.d1[k] = b.c.d2[k] = b.c.eps[k] = b.c.rs[k] = 0.0f;
    }
    b.sendW = b.sendY = b.filt = b.maxY = 0.0f;
    b.u = -(kLanes - 1 - lane) * R;  // lane 31's leading row leads
    b.jj = b.sp = 0;
    b.wp = a.w1 + lane * stagLaneStride(R);
    {
        const int rowBase = (a.nS - 1) * S + lane * R;  // in bounds before the lane's first stripe
        b.eS = SH ? (unsigned)__cvta_generic_to_shared(a.smE + rowBase) : 0u;
        b.eG = a.smE + rowBase;
    }
    const int steps = (a.nS - 1) * a.P + a.L - 1 + S;
    const int T = (steps + 3) / 4 * 4;
    __syncwarp();
    FillRegs pf = fillPrologueS<true, R>(win, a, lane);
    for (int t0 = 0; t0 < T; t0 += kSBlock) {
        __syncwarp();
        fillStoreS<true, R>(win, a, pf, t0 + kSBlock + lane);
        pf = fillLoadS<true>(a, t0 + 2 * kSBlock + lane);
        const int n = min(kSBlock, T - t0);
        int gA, gB;
        const int sp = interiorRunS<4>(a, S, t0, n, gA, gB);
        const bool ringWriter = lane == 0 && sp >= 0 && sp < a.nS - 1;
        int g = 0;
        RunPtrs ip{nullptr, nullptr, nullptr, nullptr};
#pragma unroll 1
        for (; g < gA; g += 4) {
            bwdStepS<R, MID, 0, true, SH>(b, a, win, lane, false, ip);
            bwdStepS<R, MID, 1, true, SH>(b, a, win, lane, false, ip);
            bwdStepS<R, MID, 2, true, SH>(b, a, win, lane, false, ip);
            bwdStepS<R, MID, 3, true, SH>(b, a, win, lane, false, ip);
        }
        if (gB > gA) {
            ip.col = win.col + (b.u & (kSWin - 1));
            ip.ring = win.ring + (b.u & (kSRingWin - 1));
            ip.w1 = b.wp;
            ip.ringOut = reinterpret_cast<float2 *>(a.ring) + (b.jj - (R - 1));  // used by lane 0 only
#pragma unroll 1
            for (; g < gB; g += 4) {
                bwdStepS<R, MID, 0, false, SH>(b, a, win, lane, ringWriter, ip);
                bwdStepS<R, MID, 1, false, SH>(b, a, win, lane, ringWriter, ip);
                bwdStepS<R, MID, 2, false, SH>(b, a, win, lane, ringWriter, ip);
                bwdStepS<R, MID, 3, false, SH>(b, a, win, lane, ringWriter, ip);
                ip.col += 4;
                ip.ring += 4;
                ip.w1 += 4 * SW;
                ip.ringOut += 4;
            }
            b.u += gB - gA;
            b.jj += gB - gA;
            b.wp += (gB - gA) * SW;
        }
#pragma unroll 1
        for (; g < n; g += 4) {
            bwdStepS<R, MID, 0, true, SH>(b, a, win, lane, false, ip);
            bwdStepS<R, MID, 1, true, SH>(b, a, win, lane, false, ip);
            bwdStepS<R, MID, 2, true, SH>(b, a, win, lane, false, ip);
            bwdStepS<R, MID, 3, true, SH>(b, a, win, lane, false, ip);
        }
    }
    filtOut = b.filt;
    maxYOut = b.maxY;
}

// ---------------------------------------------------------------------------
// Forward sweep.  Phase PH = t mod 8 (the W1 staging slot); the histories use
// H = PH mod 4 as the backward's.  Row k takes W0's input and Y0 of row k-1 at
// its own column from the previous step (registers); the lane's leading row
// takes them from lane l-1 by shuffle, lane 0's from the ring.
// ---------------------------------------------------------------------------
template <int R>
struct FwdS {
    Coef<R> c;
    float w[4][R], z[4][R], ninPrev[R], yPrev[R];
    float bgH[4], preH[4], evH[4][R];
    float sendIn, sendY, best, mx;
    int u, jj, sp;
    unsigned eS;
    const float *eG;
    const float *w1src;  // W1 group of the step kSW1Ahead ahead (this lane's R values)
    int gAhead;          // its group index; no copy below 0
};

template <int R>
__device__ __forceinline__ void cpAsyncStage(float *dst, const float *src) {
    const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
    if constexpr (R == 4 || R == 3) {  // R = 3: the lane's 16-byte group entry, padding included
        asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(d), "l"(src) : "memory");
    } else {
        asm volatile("cp.async.ca.shared.global [%0], [%1], %2;" ::"r"(d), "l"(src), "n"(4 * R) : "memory");
    }
}

template <int R, int PH, bool GEN, bool SH>
__device__ __forceinline__ void fwdStepS(FwdS<R> &f, const SweepArgs &a, WindowS<R> &win, int lane,
                                         bool ringWriter, const RunPtrs &ip) {
    constexpr int S = kLanes * R;
    constexpr int SW = kLanes * stagLaneStride(R);  // floats per W1 group
    constexpr int H = PH & 3;
    float q[R];
    cpAsyncWait<kSW1Ahead - 1>();
    if constexpr (R == 4) {
        const float4 v = *reinterpret_cast<const float4 *>(&win.w1[PH][lane * 4]);
        q[0] = v.x;
        q[1] = v.y;
        q[2] = v.z;
        q[3] = v.w;
    } else if constexpr (R == 3) {
        const float4 v = *reinterpret_cast<const float4 *>(&win.w1[PH][lane * 4]);
        q[0] = v.x;
        q[1] = v.y;
        q[2] = v.z;
    } else if constexpr (R == 2) {
        const float2 v = *reinterpret_cast<const float2 *>(&win.w1[PH][lane * 2]);
        q[0] = v.x;
        q[1] = v.y;
    } else {
#pragma unroll
        for (int k = 0; k < R; ++k) q[k] = win.w1[PH][lane * R + k];
    }
    float inW = __shfl_up_sync(kFull, f.sendIn, 1);
    float inY = __shfl_up_sync(kFull, f.sendY, 1);
    if (GEN && f.u >= 0 && f.jj == 0 && f.sp < a.nS) {
        const int rowBase = f.sp * S + lane * R;
        loadForwardCoef<R>(f.c, a, rowBase);
        if (SH)
            f.eS = (unsigned)__cvta_generic_to_shared(a.smE + rowBase);
        else
            f.eG = a.smE + rowBase;
    }
    const float4 col = GEN ? win.col[f.u & (kSWin - 1)] : ip.col[PH];
    if (lane == 0) {
        const float2 r = GEN ? win.ring[f.u & (kSRingWin - 1)] : ip.ring[PH];
        inW = r.x;
        inY = r.y;
    }
    float ev[R];
    if (SH)
        loadEmitS<R>(ev, f.eS + 4u * (unsigned)__float_as_int(col.x));
    else
        loadEmit<R>(ev, f.eG + __float_as_int(col.x));
    f.bgH[H] = col.y;
    f.preH[H] = col.z;
#pragma unroll
    for (int k = 0; k < R; ++k) f.evH[H][k] = ev[k];
    float nW[R], nZ[R], nN[R], nY[R], bv[R];
#pragma unroll
    for (int k = 0; k < R; ++k) {
        const int Q = (H + 4 - k) & 3;  // row k is k steps behind the lane's leading row
        const float e = f.evH[Q][k], bgsC = f.bgH[Q], prev = f.preH[Q];
        const float win0 = k == 0 ? inW : f.ninPrev[k - 1];
        const float yab = k == 0 ? inY : f.yPrev[k - 1];
        const float w1 = f.w[(H + 3) & 3][k], w2 = f.w[(H + 2) & 3][k], w3 = f.w[(H + 1) & 3][k];
        const float z3 = f.z[(H + 1) & 3][k];
        // the reference's operations as GCC contracts them at -O3
        // (dummest-dp-forward.hh:116-222)
        const float X = (f.c.enter[k] * e) * w3;
        float Z0 = bgsC * __fmaf_rn(f.c.b0[k], z3, f.c.a0[k] * w3);
        const float zs = __fmaf_rn(f.c.a2[k], w2, __fmaf_rn(f.c.a1[k], w1, Z0));
        float W0 = win0 + __fadd_rn(zs, prev);
        float b = W0 * q[k];
        float Y0 = __fmaf_rn(f.c.eps[k], yab, f.c.d0[k] * W0);
        float nin = __fmaf_rn(f.c.d2[k], w1, __fmaf_rn(f.c.d1[k], w2, X + Y0));
        if (GEN) {
            const bool act = f.u >= 0 && f.sp < a.nS && f.jj >= k && f.jj < a.L + k;
            if (!act) W0 = Y0 = nin = Z0 = b = 0.0f;
        }
        f.mx = fmax3(f.mx, W0, Y0);
        nW[k] = W0;
        nZ[k] = Z0;
        nN[k] = nin;
        nY[k] = Y0;
        bv[k] = b;
    }
    if constexpr (R == 4) {
        f.best = fmax3(f.best, bv[0], bv[1]);
        f.best = fmax3(f.best, bv[2], bv[3]);
    } else if constexpr (R == 3) {
        f.best = fmax3(f.best, bv[0], bv[1]);
        f.best = fmaxf(f.best, bv[2]);
    } else if constexpr (R == 2) {
        f.best = fmax3(f.best, bv[0], bv[1]);
    } else {
        f.best = fmaxf(f.best, bv[0]);
    }
#pragma unroll
    for (int k = 0; k < R; ++k) {
        f.w[H][k] = nW[k];
        f.z[H][k] = nZ[k];
        f.ninPrev[k] = nN[k];
        f.yPrev[k] = nY[k];
    }
    f.sendIn = nN[R - 1];
    f.sendY = nY[R - 1];
    // the stage for the step kSW1Ahead later goes into the slot read one step ago
    if (GEN) {
        if (lane == kLanes - 1 && f.u >= 0 && f.sp < a.nS - 1 && f.jj >= R - 1 && f.jj < a.L + R - 1)
            ringStoreS(a.ring, f.jj - (R - 1), nN[R - 1], nY[R - 1]);
        if (f.gAhead >= 0) cpAsyncStage<R>(&win.w1[(PH + kSW1Ahead) % kSW1Slots][lane * stagLaneStride(R)], f.w1src);
        cpAsyncCommit();
        f.w1src -= SW;
        --f.gAhead;
        if (f.u >= 0 && ++f.jj == a.P) {
            f.jj = 0;
            ++f.sp;
        }
        ++f.u;
    } else {  // the run advances u, jj and the staging cursor
        if (ringWriter) __stcg(ip.ringOut + PH, make_float2(nN[R - 1], nY[R - 1]));
        cpAsyncStage<R>(&win.w1[(PH + kSW1Ahead) % kSW1Slots][lane * stagLaneStride(R)], ip.w1 - PH * SW);
        cpAsyncCommit();
    }
}

template <int R, bool SH>
__device__ void forwardSweepS(const SweepArgs &a, WindowS<R> &win, int lane, float &bestOut, float &maxOut) {
    constexpr int S = kLanes * R;
    constexpr int SW = kLanes * stagLaneStride(R);  // floats per W1 group
    FwdS<R> f;
#pragma unroll
    for (int q = 0; q < 4; ++q) {
#pragma unroll
        for (int k = 0; k < R; ++k) f.w[q][k] = f.z[q][k] = f.evH[q][k] = 0.0f;
        f.bgH[q] = f.preH[q] = 0.0f;
    }
#pragma unroll
    for (int k = 0; k < R; ++k) {
        f.ninPrev[k] = f.yPrev[k] = 0.0f;
        f.c.enter[k] = f.c.a0[k] = f.c.a1[k] = f.c.a2[k] = f.c.b0[k] = 0.0f;
        f.c.d0[k] = f.c.d1[k] = f.c.d2[k] = f.c.eps[k] = f.c.rs[k] = 0.0f;
    }
    f.sendIn = f.sendY = f.best = f.mx = 0.0f;
    f.u = -lane * R;  // lane 0's row 0 leads
    f.jj = f.sp = 0;
    {
        const int rowBase = lane * R;
        f.eS = SH ? (unsigned)__cvta_generic_to_shared(a.smE + rowBase) : 0u;
        f.eG = a.smE + rowBase;
    }
    const int steps = (a.nS - 1) * a.P + a.L - 1 + S;
    const int T = (steps + kSW1Slots - 1) / kSW1Slots * kSW1Slots;
    // step t reads the backward's group steps - 1 - t
    {
        const float *src = a.w1 + (size_t)(steps - 1) * SW + lane * stagLaneStride(R);
#pragma unroll
        for (int k = 0; k < kSW1Ahead; ++k) {
            cpAsyncStage<R>(&win.w1[k][lane * stagLaneStride(R)], src);
            cpAsyncCommit();
            src -= SW;
        }
        f.w1src = src;
        f.gAhead = steps - 1 - kSW1Ahead;
    }
    __syncwarp();
    FillRegs pf = fillPrologueS<false, R>(win, a, lane);
    for (int t0 = 0; t0 < T; t0 += kSBlock) {
        __syncwarp();
        fillStoreS<false, R>(win, a, pf, t0 + kSBlock + lane);
        pf = fillLoadS<false>(a, t0 + 2 * kSBlock + lane);
        const int n = min(kSBlock, T - t0);
        int gA, gB;
        const int sp = interiorRunS<8>(a, S, t0, n, gA, gB);
        const bool ringWriter = lane == kLanes - 1 && sp >= 0 && sp < a.nS - 1;
        int g = 0;
        RunPtrs ip{nullptr, nullptr, nullptr, nullptr};
#pragma unroll 1
        for (; g < gA; g += 8) {
            fwdStepS<R, 0, true, SH>(f, a, win, lane, false, ip);
            fwdStepS<R, 1, true, SH>(f, a, win, lane, false, ip);
            fwdStepS<R, 2, true, SH>(f, a, win, lane, false, ip);
            fwdStepS<R, 3, true, SH>(f, a, win, lane, false, ip);
            fwdStepS<R, 4, true, SH>(f, a, win, lane, false, ip);
            fwdStepS<R, 5, true, SH>(f, a, win, lane, false, ip);
            fwdStepS<R, 6, true, SH>(f, a, win, lane, false, ip);
            fwdStepS<R, 7, true, SH>(f, a, win, lane, false, ip);
        }
        if (gB > gA) {
            ip.col = win.col + (f.u & (kSWin - 1));
            ip.ring = win.ring + (f.u & (kSRingWin - 1));
            ip.w1 = const_cast<float *>(f.w1src);
            ip.ringOut = reinterpret_cast<float2 *>(a.ring) + (f.jj - (R - 1));  // used by lane 31 only
#pragma unroll 1
            for (; g < gB; g += 8) {
                fwdStepS<R, 0, false, SH>(f, a, win, lane, ringWriter, ip);
                fwdStepS<R, 1, false, SH>(f, a, win, lane, ringWriter, ip);
                fwdStepS<R, 2, false, SH>(f, a, win, lane, ringWriter, ip);
                fwdStepS<R, 3, false, SH>(f, a, win, lane, ringWriter, ip);
                fwdStepS<R, 4, false, SH>(f, a, win, lane, ringWriter, ip);
                fwdStepS<R, 5, false, SH>(f, a, win, lane, ringWriter, ip);
                fwdStepS<R, 6, false, SH>(f, a, win, lane, ringWriter, ip);
                fwdStepS<R, 7, false, SH>(f, a, win, lane, ringWriter, ip);
                ip.col += 8;
                ip.ring += 8;
                ip.w1 -= 8 * SW;
                ip.ringOut += 8;
            }
            f.u += gB - gA;
            f.jj += gB - gA;
            f.w1src -= (gB - gA) * SW;
            f.gAhead -= gB - gA;
        }
#pragma unroll 1
        for (; g < n; g += 8) {
            fwdStepS<R, 0, true, SH>(f, a, win, lane, false, ip);
            fwdStepS<R, 1, true, SH>(f, a, win, lane, false, ip);
            fwdStepS<R, 2, true, SH>(f, a, win, lane, false, ip);
            fwdStepS<R, 3, true, SH>(f, a, win, lane, false, ip);
            fwdStepS<R, 4, true, SH>(f, a, win, lane, false, ip);
            fwdStepS<R, 5, true, SH>(f, a, win, lane, false, ip);
            fwdStepS<R, 6, true, SH>(f, a, win, lane, false, ip);
            fwdStepS<R, 7, true, SH>(f, a, win, lane, false, ip);
        }
    }
    cpAsyncWait<0>();  // no copy outlives the sweep (the staging slots are reused)
    bestOut = f.best;
    maxOut = f.mx;
}


// One pair on one warp: the backward (and, for the mid score, the forward)
// sweep, then the warp maxima as the pair's raw results.
template <int R, bool MID, bool SH>
__device__ void scorePairS(const DpArgs &g, int pi, const float *smE, int rowPad, const float *smBg,
                           WindowS<R> &win, float *w1, float *ring, int lane) {
    const DevPair p = g.pairs[pi];
    __syncwarp();
    if (lane == 0) {
        PairCold &c = win.cold;
        c.codes = g.codes + p.codeOff;
        c.pre = g.seeds + p.seedOff;
        c.suf = c.pre + p.L;
        const DevProfile &pr = g.profiles[p.prof];
        c.coef = g.params + coefOffOf(pr.paramOff, pr.M);
        c.coefStride = pr.rowPad;
        c.smBg = smBg;
        c.sc = g.scales[pi];
        c.M = p.M;
    }
    __syncwarp();
    SweepArgs a;
    a.alignOut = nullptr;
    a.cold = &win.cold;
    a.smE = smE;
    a.w1 = w1;
    a.ring = ring;
    a.L = p.L;
    a.rowPad = rowPad;
    a.nS = (p.M + 1 + kLanes * R - 1) / (kLanes * R);
    a.P = stagPeriod(p.L, R);
    a.D = 0;
    a.sFirst = 0;
    a.sStep = 1;
    a.nMine = a.nS;
    a.ringSlots = 1;
    a.ringStride = 0;
    float filt, maxYb, mid = 0.0f, maxFw = 0.0f;
    backwardSweepS<R, MID, SH>(a, win, lane, filt, maxYb);
    if (MID) {
        __syncwarp();  // the window is refilled for the forward sweep
        forwardSweepS<R, SH>(a, win, lane, mid, maxFw);
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

// Persistent kernel for one rows-per-lane value: CTAs pull chunks
// (same-profile runs of pairs, costliest first) from a global counter, stage
// the chunk's profile emission table in shared memory, and their warps pull
// pairs from the chunk.  Dynamic shared memory: the table (tableFloats), then
// one WindowS per warp (the launch may use fewer than WARPS warps when the
// table leaves no room; W1 slots are indexed by the launched warps).  With
// GT (tall profiles) the table stays in global memory, read through L1 (a
// stripe's 32 R rows of 25 codes), and the shared memory holds the windows
// of all WARPS warps.
template <int R, bool MID, int WARPS, bool GT>
__global__ void __launch_bounds__(WARPS * kLanes, 1) dpKernel(DpArgs g, int tableFloats) {
    extern __shared__ float4 smRaw[];
    const float *smE = reinterpret_cast<const float *>(smRaw);
    WindowS<R> *wins = reinterpret_cast<WindowS<R> *>(reinterpret_cast<float *>(smRaw) + tableFloats);
    __shared__ float smBg[32];
    __shared__ int smChunk, smNext;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const size_t slot = (size_t)blockIdx.x * (blockDim.x >> 5) + warp;  // launched warps, not WARPS
    float *w1 = g.w1 + slot * g.w1SlotFloats;
    float *ring = g.ring + slot * g.ringSlotFloats;
    WindowS<R> &win = wins[warp];
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
        if (ch.count == 0) {  // a chunk of the second search wave with no survivors
            __syncthreads();
            continue;
        }
        const int rowPad = ch.rowPad;
        if (ch.prof != loaded) {
            const DevProfile *pr = g.profiles + ch.prof;
            if (GT) {
                smE = g.emit + pr->emitOff;
            } else {
                const float4 *src = reinterpret_cast<const float4 *>(g.emit + pr->emitOff);
                const int n4 = kNumCodes * rowPad / 4;
                for (int i = threadIdx.x; i < n4; i += blockDim.x) smRaw[i] = __ldg(src + i);
            }
            if (threadIdx.x < 32) smBg[threadIdx.x] = threadIdx.x < kNumCodes ? pr->bg[threadIdx.x] : 0.0f;
            loaded = ch.prof;
        }
        __syncthreads();
        for (;;) {
            int k = 0;
            if (lane == 0) k = atomicAdd(&smNext, 1);
            k = __shfl_sync(kFull, k, 0);
            if (k >= ch.count) break;
            const int pi = g.pairIdx ? g.pairIdx[ch.first + k] : ch.first + k;
            scorePairS<R, MID, !GT>(g, pi, smE, rowPad, smBg, win, w1, ring, lane);
        }
        __syncthreads();
    }
}

// Shared memory of one warp's staging (host side: launch sizes).
inline size_t stagWindowBytes(int R) {
    return R == 4 ? sizeof(WindowS<4>)
                  : (R == 3 ? sizeof(WindowS<3>) : (R == 2 ? sizeof(WindowS<2>) : sizeof(WindowS<1>)));
}

}  // namespace dmst
