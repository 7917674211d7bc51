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
// row-rescaled kernel (dp_exact.cuh).
//
// Mid score.  The reference forms promote(W0)*promote(W1) in double and
// rounds the mantissa to float (dummest-batch.hh:216-235); with both counts
// zero that is the float product W0*W1 whenever it is a normal float, so the
// per-cell product is one FMUL.  Overflow (a score above 2^128) is reported
// as +inf and routed to the exact kernel.
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
    float *ring;            // this warp's stripe-boundary ring (2 floats per column)
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

// Steps of look-ahead for the per-step global operands (codon code, seeds,
// W1, ring): each step issues the loads of step t + kPF into a register FIFO,
// so their latency overlaps kPF steps of arithmetic.
constexpr int kPF = 4;

// Per-lane position in the wavefront: local time u and (stripe, column).
struct Cursor {
    int u, sp, jj;
    __device__ __forceinline__ void advance(int P) {
        if (u >= 0 && ++jj == P) {
            jj = 0;
            ++sp;
        }
        ++u;
    }
    __device__ __forceinline__ bool active(int nS, int L) const { return u >= 0 && sp < nS && jj < L; }
};

// Backward sweep.  STORE: keep W1 for the forward sweep (mid mode); without
// it this is the lean float filter (findSimilaritiesBackwardOnly), whose
// arithmetic is the same with every rescale count at zero.
template <int R, bool STORE>
__device__ void backwardSweep(const SweepArgs &a, int lane, float &filtOut, float &maxYOut) {
    constexpr int S = kLanes * R;
    Coef<R> c;
    float h1[R], h2[R], h3[R], z1[R], z2[R], z3[R];
#pragma unroll
    for (int k = 0; k < R; ++k) h1[k] = h2[k] = h3[k] = z1[k] = z2[k] = z3[k] = 0.0f;
    float rb1 = 0.0f, rb2 = 0.0f, rb3 = 0.0f;  // row below (other lane) at j+1..j+3
    float sendW = 0.0f, sendY = 0.0f;
    float filt = 0.0f, maxY = 0.0f;
    const int L = a.L, P = a.P, nS = a.nS;
    const int T = nS * P + (kLanes - 1);
    const bool ringAhead = P > kLanes + kPF;  // ring entries are written > kPF steps before use
    Cursor cur{-(kLanes - 1 - lane), 0, 0}, ahead = cur;
    int qc[kPF];
    float qs[kPF], qp[kPF], qw[kPF], qy[kPF];
    auto fetch = [&](const Cursor &x, int &code, float &suf, float &pre, float &rw, float &ry) {
        code = kPad;
        suf = pre = rw = ry = 0.0f;
        if (x.active(nS, L)) {
            const int j = L - 1 - x.jj;
            code = (j + 1 < L) ? (int)__ldg(a.codes + j + 1) : kPad;
            suf = __ldg(a.suf + j);
            pre = __ldg(a.pre + j);
            if (ringAhead && lane == kLanes - 1 && x.sp > 0) {
                rw = __ldcg(a.ring + 2 * x.jj);
                ry = __ldcg(a.ring + 2 * x.jj + 1);
            }
        }
    };
#pragma unroll
    for (int k = 0; k < kPF; ++k) {
        fetch(ahead, qc[k], qs[k], qp[k], qw[k], qy[k]);
        ahead.advance(P);
    }
    for (int t = 0; t < T; ++t) {
        int nc;
        float ns, np, nw, ny;
        fetch(ahead, nc, ns, np, nw, ny);
        ahead.advance(P);
        float inW = __shfl_down_sync(kFull, sendW, 1);
        float inY = __shfl_down_sync(kFull, sendY, 1);
        if (cur.active(nS, L)) {
            const int sp = cur.sp, jj = cur.jj;
            const int s = nS - 1 - sp;
            const int rowBase = s * S + lane * R;
            if (jj == 0) {
                loadBackwardCoef<R>(c, a, rowBase);
#pragma unroll
                for (int k = 0; k < R; ++k) h1[k] = h2[k] = h3[k] = z1[k] = z2[k] = z3[k] = 0.0f;
                rb1 = rb2 = rb3 = 0.0f;
            }
            if (lane == kLanes - 1) {
                if (sp == 0) {
                    inW = inY = 0.0f;
                } else if (ringAhead) {
                    inW = qw[0];
                    inY = qy[0];
                } else {
                    inW = __ldcg(a.ring + 2 * jj);
                    inY = __ldcg(a.ring + 2 * jj + 1);
                }
            }
            const int code = qc[0];
            const float bgv = a.smBg[code];
            float e[R];
            loadEmit<R>(e, a.smE + code * a.rowPad + rowBase);
            const float sufv = qs[0];
            const float prev = qp[0];
            float bW1 = rb1, bW2 = rb2, bW3 = rb3, bY = inY;
            float wv[R];
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
                maxY = fmaxf(maxY, Y);
                filt = fmaxf(filt, W * prev);
                bW1 = h1[k];
                bW2 = h2[k];
                bW3 = h3[k];
                bY = Y;
                h3[k] = h2[k];
                h2[k] = h1[k];
                h1[k] = W;
                z3[k] = z2[k];
                z2[k] = z1[k];
                z1[k] = Z;
                wv[k] = W;
            }
            rb3 = rb2;
            rb2 = rb1;
            rb1 = inW;
            sendW = wv[0];
            sendY = bY;
            if (STORE) {
                const int d = jj + (kLanes - 1 - lane);
                storeW1<R>(a.w1 + (((size_t)s * a.D + d) * kLanes + lane) * R, wv);
            }
            if (lane == 0 && sp < nS - 1) {
                __stcg(a.ring + 2 * jj, sendW);
                __stcg(a.ring + 2 * jj + 1, sendY);
            }
        } else {
            sendW = 0.0f;
            sendY = 0.0f;
        }
#pragma unroll
        for (int k = 0; k < kPF - 1; ++k) {
            qc[k] = qc[k + 1];
            qs[k] = qs[k + 1];
            qp[k] = qp[k + 1];
            qw[k] = qw[k + 1];
            qy[k] = qy[k + 1];
        }
        qc[kPF - 1] = nc;
        qs[kPF - 1] = ns;
        qp[kPF - 1] = np;
        qw[kPF - 1] = nw;
        qy[kPF - 1] = ny;
        cur.advance(P);
        __syncwarp();
    }
    filtOut = filt;
    maxYOut = maxY;
}

// Forward sweep with the mid-anchored product (reads W1 written above).
template <int R>
__device__ void forwardSweep(const SweepArgs &a, int lane, float &bestOut, float &maxOut) {
    constexpr int S = kLanes * R;
    Coef<R> c;
    float w1[R], w2[R], w3[R], z1[R], z2[R], z3[R];
#pragma unroll
    for (int k = 0; k < R; ++k) w1[k] = w2[k] = w3[k] = z1[k] = z2[k] = z3[k] = 0.0f;
    float sendIn = 0.0f, sendY = 0.0f;
    float best = 0.0f, mx = 0.0f;
    const int L = a.L, P = a.P, nS = a.nS;
    const int T = nS * P + (kLanes - 1);
    const bool ringAhead = P > kLanes + kPF;
    Cursor cur{-lane, 0, 0}, ahead = cur;
    int qc[kPF];
    float qp[kPF], qw[kPF], qy[kPF], qb[kPF][R];
    auto fetch = [&](const Cursor &x, int &code, float &pre, float &rw, float &ry, float (&wb)[R]) {
        code = kPad;
        pre = rw = ry = 0.0f;
#pragma unroll
        for (int k = 0; k < R; ++k) wb[k] = 0.0f;
        if (x.active(nS, L)) {
            const int s = x.sp, j = x.jj;
            code = (j >= 2) ? (int)__ldg(a.codes + j - 2) : kPad;
            pre = __ldg(a.pre + j);
            const int db = (L - 1 - j) + (kLanes - 1 - lane);
            loadW1<R>(wb, a.w1 + (((size_t)s * a.D + db) * kLanes + lane) * R);
            if (ringAhead && lane == 0 && s > 0) {
                rw = __ldcg(a.ring + 2 * j);
                ry = __ldcg(a.ring + 2 * j + 1);
            }
        }
    };
#pragma unroll
    for (int k = 0; k < kPF; ++k) {
        fetch(ahead, qc[k], qp[k], qw[k], qy[k], qb[k]);
        ahead.advance(P);
    }
    for (int t = 0; t < T; ++t) {
        int nc;
        float np, nw, ny, nb[R];
        fetch(ahead, nc, np, nw, ny, nb);
        ahead.advance(P);
        float inW = __shfl_up_sync(kFull, sendIn, 1);
        float inY = __shfl_up_sync(kFull, sendY, 1);
        if (cur.active(nS, L)) {
            const int s = cur.sp, j = cur.jj;
            const int rowBase = s * S + lane * R;
            if (j == 0) {
                loadForwardCoef<R>(c, a, rowBase);
#pragma unroll
                for (int k = 0; k < R; ++k) w1[k] = w2[k] = w3[k] = z1[k] = z2[k] = z3[k] = 0.0f;
            }
            if (lane == 0) {
                if (s == 0) {
                    inW = inY = 0.0f;
                } else if (ringAhead) {
                    inW = qw[0];
                    inY = qy[0];
                } else {
                    inW = __ldcg(a.ring + 2 * j);
                    inY = __ldcg(a.ring + 2 * j + 1);
                }
            }
            const int code = qc[0];
            const float bgsC = a.smBg[code] * a.sc.sC;
            float e[R];
            loadEmit<R>(e, a.smE + code * a.rowPad + rowBase);
            const float prev = qp[0];
            float win = inW, yab = inY;
#pragma unroll
            for (int k = 0; k < R; ++k) {
                const float X = (c.enter[k] * e[k]) * w3[k];
                const float Z0 = bgsC * __fmaf_rn(c.a0[k], w3[k], c.b0[k] * z3[k]);
                const float Z1 = c.a1[k] * w1[k];
                const float Z2 = c.a2[k] * w2[k];
                const float W0 = win + __fmaf_rn(prev, c.rs[k], (Z0 + Z1) + Z2);
                mx = fmaxf(mx, W0);
                best = fmaxf(best, W0 * qb[0][k]);
                const float Y0 = __fmaf_rn(c.d0[k], W0, c.eps[k] * yab);
                mx = fmaxf(mx, Y0);
                const float nin = __fmaf_rn(c.d2[k], w1[k], __fmaf_rn(c.d1[k], w2[k], X + Y0));
                w3[k] = w2[k];
                w2[k] = w1[k];
                w1[k] = W0;
                z3[k] = z2[k];
                z2[k] = z1[k];
                z1[k] = Z0;
                win = nin;
                yab = Y0;
            }
            sendIn = win;
            sendY = yab;
            if (lane == kLanes - 1 && s < nS - 1) {
                __stcg(a.ring + 2 * j, sendIn);
                __stcg(a.ring + 2 * j + 1, sendY);
            }
        } else {
            sendIn = 0.0f;
            sendY = 0.0f;
        }
#pragma unroll
        for (int k = 0; k < kPF - 1; ++k) {
            qc[k] = qc[k + 1];
            qp[k] = qp[k + 1];
            qw[k] = qw[k + 1];
            qy[k] = qy[k + 1];
#pragma unroll
            for (int r = 0; r < R; ++r) qb[k][r] = qb[k + 1][r];
        }
        qc[kPF - 1] = nc;
        qp[kPF - 1] = np;
        qw[kPF - 1] = nw;
        qy[kPF - 1] = ny;
#pragma unroll
        for (int r = 0; r < R; ++r) qb[kPF - 1][r] = nb[r];
        cur.advance(P);
        __syncwarp();
    }
    bestOut = best;
    maxOut = mx;
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
__device__ void scorePair(const DpArgs &g, int pi, const float *smE, int rowPad, const float *smBg, float *w1,
                          float *ring, int lane) {
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
    a.P = p.L > kLanes ? p.L : kLanes;
    a.D = a.P + kLanes - 1;
    float filt, maxYb, mid = 0.0f, maxFw = 0.0f;
    backwardSweep<R, MID>(a, lane, filt, maxYb);
    if (MID) forwardSweep<R>(a, lane, mid, maxFw);
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

// Warps per CTA by rows per lane: tall profiles (R = 4) carry the largest
// shared emission tables, so more warps share one copy.
template <int R>
struct KernelShape {
    static constexpr int warps = R == 4 ? 6 : 4;
    static constexpr int minBlocks = R == 4 ? 2 : 3;
};

// Persistent kernel for one rows-per-lane value: CTAs pull chunks
// (same-profile runs of pairs, costliest first) from a global counter, stage
// the chunk's profile emission table in shared memory, and their warps pull
// pairs from the chunk.
template <int R, bool MID>
__global__ void __launch_bounds__(KernelShape<R>::warps * kLanes, KernelShape<R>::minBlocks) dpKernel(DpArgs g) {
    constexpr int NW = KernelShape<R>::warps;
    extern __shared__ float4 smRaw[];
    float *smE = reinterpret_cast<float *>(smRaw);
    __shared__ float smBg[32];
    __shared__ int smChunk, smNext;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const size_t slot = (size_t)blockIdx.x * NW + warp;
    float *w1 = g.w1 + slot * g.w1SlotFloats;
    float *ring = g.ring + slot * g.ringSlotFloats;
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
            scorePair<R, MID>(g, ch.first + k, smE, rowPad, smBg, w1, ring, lane);
        }
        __syncthreads();
    }
}

}  // namespace dmst
