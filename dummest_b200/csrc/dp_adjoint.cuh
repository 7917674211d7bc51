// Log-likelihood, its gradient (the adjoint) and posterior tables of the DNA x
// profile model.
//
// The objective of a pair is log T, T the total weight of all local
// alignments: every alignment starts once (prefixSeed) and ends once
// (suffixSeedFromNext), so
//     T = sum_{i,j} prefixSeed[j] * W1[i][j] = sum_{i,j} W0[i][j] * suffixSeed[j]
// with W1 the backward recurrence (dummest-dp-backward.hh:473-574) and W0 the
// forward one (dummest-dp-forward.hh:63-250).  The forward recurrence is
// exactly the adjoint of the backward one: W0[i][j] = dT/dW1[i][j],
// Y0[i-1][j] = dT/dY[i][j] and Z0[i][j] = dT/dZ[i][j] (the backward's delete
// and insert states).  The derivative of T with respect to a coefficient of
// row i is therefore the sum over the row of that adjoint times the operand
// the coefficient multiplies in the backward recurrence:
//     dT/d(enter)  = sum_j W0[i][j] * W1[i+1][j+3] * e_i(c_{j+1}) * sC
//     dT/de_i(c)   = sum_{j: c_{j+1}=c} W0[i][j] * W1[i+1][j+3] * enter * sC
//     dT/d(delta'0)= sum_j W0[i][j] * Y[i+1][j]            (delta'1: W1[i+1][j+2] s2,
//                                                              delta'2: W1[i+1][j+1] s1)
//     dT/d(alpha'0)= sum_j W0[i][j] * Z[i][j+3] bg[j+1] sC  (alpha'1: W1[i][j+1] s1,
//                                                              alpha'2: W1[i][j+2] s2)
//     dT/d(eps')   = sum_j Y0[i-1][j] * Y[i+1][j]
//     dT/d(beta'0) = sum_j Z0[i][j] * Z[i][j+3] bg[j+1] sC
// The null model (seeds, per-base scales, background) is held fixed.  The
// posterior tables are cell[i][j] = W0[i][j] W1[i][j] / T and match[i][j] =
// X(i,j) W1[i+1][j] / T, X(i,j) = enter_i sC e_i(c_{j-2}) W0[i][j-3] (the
// match term of the forward, dummest-dp-forward.hh:125-157).
//
// Layout of the work: one warp per pair, FP64 throughout, as a wavefront over
// stripes of 32 profile rows (lane l holds one row of the stripe; at step k
// it works on column k - l in the forward and L-1-(k-l) in the backward, the
// row it depends on being the neighbouring lane's, one step earlier, passed
// by a shuffle).  Phase A sweeps the stripes upward and stores (W0, Y0, Z0)
// of every cell indexed by (stripe, step, lane), so that each step of the
// warp writes one contiguous block; phase B sweeps them downward, and at
// backward step k every lane reads the forward values of its cell from the
// single forward step L+30-k of the same stripe: again one contiguous block.
// The first lane of a stripe reads the row below (forward: from the store)
// or above (backward: from a two-row boundary buffer) through a coalesced
// load of 32 columns per lane group, passed on by shuffles.
//
// Scaling: every stripe is held at its own power-of-two offset, the binary
// exponent of the largest value of the row it reads from (the previous
// stripe's boundary row), accumulated along the sweep.  Products of a
// forward and a backward value stay in double range for any score (homologs
// reach 2^2000 and more; a row grows by at most ~2^6 over the one below, so a
// stripe spans ~2^200); values more than ~1000 binades below the boundary
// row's maximum flush to zero, the double-range counterpart of the
// reference's float row rescaling.  T is a mantissa with a binary exponent.
#pragma once

#include "dp_common.cuh"

namespace dmst {

constexpr int kAdjWarps = 4;  // warps (pairs) per CTA

struct AdjointJob {
    int pair;         // index into the pair descriptors
    int pad;
    long long fOff;   // double offset of the pair's forward store
    long long bOff;   // double offset of the pair's boundary rows
    long long pOff;   // double offset of the pair's posterior tables, -1 for none
};
static_assert(sizeof(AdjointJob) == 32, "AdjointJob layout");

__host__ __device__ __forceinline__ int adjStripes(int M) { return (M + 1 + 31) / 32; }
// Forward store of a pair: stripes x (L + 31) steps x 32 lanes x (W0, Y0, Z0),
// then one offset per stripe.
__host__ __device__ __forceinline__ long long adjStoreDoubles(int M, int L) {
    return (long long)adjStripes(M) * (L + 31) * 32 * 3 + adjStripes(M);
}
__device__ __forceinline__ size_t adjF(int L, int s, int k, int lane) {
    return (((size_t)s * (L + 31) + k) * 32 + lane) * 3;
}
// Checkpointed store of a pair (CKPT): the forward pass keeps only what the
// backward pass needs to recompute the forward blocks it reads, kAdjCk steps
// at a time: each stripe's top row (W0, Y0 per column, which the next stripe
// reads), the warp's state at every kAdjCk-th step of each stripe (per lane
// its own row's W0 and Z0 at the three columns before, the row below's W0 at
// the three columns before and the two values it publishes), the per-stripe
// offsets, then the backward's two recompute buffers of kAdjCk forward blocks.
constexpr int kAdjCk = 64;       // forward steps per checkpoint (64 columns)
constexpr int kAdjCkVals = 11;   // doubles of a lane's state
__host__ __device__ __forceinline__ int adjChunks(int L) { return (L + 31 + kAdjCk - 1) / kAdjCk; }
__host__ __device__ __forceinline__ long long adjCkTopOff(int M, int L) { return 0; }
__host__ __device__ __forceinline__ long long adjCkStateOff(int M, int L) { return (long long)adjStripes(M) * L * 2; }
__host__ __device__ __forceinline__ long long adjCkOffsetsOff(int M, int L) {
    return adjCkStateOff(M, L) + (long long)adjStripes(M) * adjChunks(L) * 32 * kAdjCkVals;
}
__host__ __device__ __forceinline__ long long adjCkBufOff(int M, int L) {
    return adjCkOffsetsOff(M, L) + ((adjStripes(M) + 1) & ~1);
}
__host__ __device__ __forceinline__ long long adjCkptDoubles(int M, int L) {
    return adjCkBufOff(M, L) + 2LL * kAdjCk * 96;
}
// Boundary rows of a pair: parity x (W1, Y) x (L + 4) columns.
__host__ __device__ __forceinline__ long long adjBoundDoubles(int L) { return 2LL * 2 * (L + 4); }

// Binary exponent of x > 0 (x = m 2^e, m in [0.5, 1)); 0 for x = 0.
__device__ __forceinline__ int binExp(double x) {
    int e = 0;
    if (x > 0.0) frexp(x, &e);
    return e;
}

// T += v 2^ve with T = tm 2^te, tm in [0.5, 1) (terms 60 binades below drop).
__device__ __forceinline__ void dxAdd(double &tm, int &te, double v, int ve) {
    if (!(v > 0.0)) return;
    int pe;
    const double pm = frexp(v, &pe);
    pe += ve;
    if (tm == 0.0 || pe > te + 60) {
        tm = pm;
        te = pe;
    } else if (pe >= te - 60) {
        int e2;
        tm = frexp(tm + ldexp(pm, pe - te), &e2);
        te += e2;
    }
}

__device__ __forceinline__ double warpSumD(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Shared memory of a warp: the backward's ring of forward blocks (one block =
// one forward step of a stripe: 32 lanes x (W0, Y0, Z0), plus the Y0 of the
// row below the stripe that the block's step needs), then the per-lane
// emission sums of the stripe.
constexpr int kAdjRing = 8;          // slots (a power of two)
constexpr int kAdjAhead = 6;         // blocks copied ahead of use
constexpr int kAdjSlot = 32 * 3 + 2; // doubles per slot (16-byte multiple)
constexpr size_t kAdjSmemWarp = (size_t)(kAdjRing * kAdjSlot + kNumCodes * 32) * sizeof(double);
constexpr size_t kAdjSmem = kAdjWarps * kAdjSmemWarp;

__device__ __forceinline__ void adjCp16(double *dst, const double *src) {
    const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(d), "l"(src) : "memory");
}
__device__ __forceinline__ void adjCp8(double *dst, const double *src) {
    const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(d), "l"(src) : "memory");
}
__device__ __forceinline__ void adjCommit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void adjWait() {
    asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

// The forward coefficients of a lane's row (row 32 s + lane) and its history
// (own row at j-1, j-2, j-3; the row below at j-1, j-2, j-3; the values
// published at the previous step).
struct AdjRow {
    double a0, a1, a2, b0, d0, eps, pEnter, pd1, pd2;
    const float *Eprev;
    bool rowOK;
};
struct AdjHist {
    double w1, w2, w3, z1, z2, z3, u1, u2, u3, pubW, pubY;
};
__device__ __forceinline__ AdjRow adjRow(int s, int lane, int M, const float *par, const float *E, double sC,
                                         double s1, double s2) {
    AdjRow r;
    const int i = 32 * s + lane;
    r.rowOK = i <= M;
    const int ir = r.rowOK ? i : M;
    const float *q = par + (size_t)ir * kParamFloats;
    const float *qp = par + (size_t)(ir > 0 ? ir - 1 : 0) * kParamFloats;
    r.a0 = q[0];
    r.a1 = (double)q[1] * s1;
    r.a2 = (double)q[2] * s2;
    r.b0 = q[3];
    r.d0 = q[6];
    r.eps = q[9];
    r.pEnter = ir > 0 ? (double)qp[10] * sC : 0.0;
    r.pd1 = ir > 0 ? (double)qp[7] * s2 : 0.0;
    r.pd2 = ir > 0 ? (double)qp[8] * s1 : 0.0;
    r.Eprev = E + (ir > 0 ? ir - 1 : 0);
    return r;
}
// Forward step k of a stripe (lane l at column k - l): the row below comes
// from lane l-1's previous step, or for lane 0 from (cW, cY), lane k mod 32
// of which holds the row below the stripe at column k.  live: the cell is in
// the matrix.
__device__ __forceinline__ void adjFwdStep(const AdjRow &r, AdjHist &h, int k, int lane, int L, double cW, double cY,
                                           const uint8_t *cd, const float *pre, const float *bg, int rowPad,
                                           double sC, double seedScale, double &W0, double &Y0, double &Z0,
                                           bool &live) {
    const int j = k - lane;
    double uj = __shfl_up_sync(0xffffffffu, h.pubW, 1);
    double yPrev = __shfl_up_sync(0xffffffffu, h.pubY, 1);
    const double bw = __shfl_sync(0xffffffffu, cW, k & 31);
    const double by = __shfl_sync(0xffffffffu, cY, k & 31);
    if (lane == 0) {
        uj = bw;
        yPrev = by;
    }
    W0 = Y0 = Z0 = 0.0;
    live = r.rowOK && j >= 0 && j < L;
    if (live) {
        const int c = (j - 2 >= 0 && j - 2 < L) ? (int)cd[j - 2] : kPad;
        const double win = fma(r.pEnter * (double)r.Eprev[(size_t)c * rowPad], h.u3,
                               fma(r.pd1, h.u2, fma(r.pd2, h.u1, yPrev)));
        Z0 = ((double)bg[c] * sC) * fma(r.a0, h.w3, r.b0 * h.z3);
        W0 = fma(r.a1, h.w1, fma(r.a2, h.w2, fma((double)pre[j], seedScale, win + Z0)));
        Y0 = fma(r.d0, W0, r.eps * yPrev);
    }
    h.w3 = h.w2; h.w2 = h.w1; h.w1 = W0;
    h.z3 = h.z2; h.z2 = h.z1; h.z1 = Z0;
    h.u3 = h.u2; h.u2 = h.u1; h.u1 = uj;
    h.pubW = W0;
    h.pubY = Y0;
}

// grad: (M+2) x 11 Params gradients then (M+1) x 25 emission gradients of
// the profile, accumulated over the pairs (each term already divided by the
// pair's T).  logT: per job, natural log.  post: posterior tables (POST).
// The forward store must start 16-byte aligned (the host pads each pair's).
// CKPT: the checkpointed store (adjCkptDoubles per pair) instead of the full
// one; the backward pass recomputes each kAdjCk-step chunk of forward blocks
// from its checkpoint (the same step function, so the same values) into one
// of two buffers before its look-ahead reads the chunk.
template <bool POST, bool CKPT = false>
__global__ void __launch_bounds__(kAdjWarps * 32, 3) adjointKernel(
    const AdjointJob *jobs, int nJobs, const DevPair *pairs, const DevProfile *profiles, const float *emit,
    const float *params, const uint8_t *codes, const float *seeds, const PairScales *scales, double *fstore,
    double *bstore, double *grad, double *logT, double *post) {
    extern __shared__ __align__(16) double adjSmem[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    double *ring = adjSmem + (size_t)warp * (kAdjSmemWarp / sizeof(double));
    double *geS = ring + kAdjRing * kAdjSlot;  // [25][32]
    const int ji = blockIdx.x * kAdjWarps + warp;
    if (ji >= nJobs) return;  // whole warps only
    const AdjointJob job = jobs[ji];
    const DevPair p = pairs[job.pair];
    const DevProfile &pr = profiles[p.prof];
    const int L = p.L, M = p.M, rowPad = pr.rowPad, nS = adjStripes(M);
    const uint8_t *cd = codes + p.codeOff;
    const float *pre = seeds + p.seedOff;
    const float *suf = pre + L;
    const float *E = emit + pr.emitOff;
    const float *par = params + pr.paramOff;
    const PairScales sc = scales[job.pair];
    const double sC = sc.sC, s1 = sc.s1, s2 = sc.s2;
    double *F = fstore + job.fOff;
    double *Foff = CKPT ? F + adjCkOffsetsOff(M, L) : F + (size_t)nS * (L + 31) * 32 * 3;  // per-stripe offsets
    double *Ftop = F + adjCkTopOff(M, L);      // CKPT: [stripe][column] x (W0, Y0)
    double *Fck = F + adjCkStateOff(M, L);     // CKPT: [stripe][chunk][lane] x kAdjCkVals
    double *Fbuf = F + adjCkBufOff(M, L);      // CKPT: [2][kAdjCk][96]
    const int nCk = adjChunks(L);
    double *Bnd = bstore + job.bOff;
    double *cellP = POST ? post + job.pOff : nullptr;
    double *matchP = POST ? cellP + (size_t)(M + 1) * L : nullptr;
    auto code = [&](int j) -> int { return (j >= 0 && j < L) ? (int)cd[j] : kPad; };
    auto bnd = [&](int par2, int t, int j) -> double * { return Bnd + ((size_t)(par2 * 2 + t) * (L + 4) + j); };
    const int nSteps = L + 31;

    // ---- phase A: forward (the adjoint), stripes upward ----
    double tm = 0.0;
    int te = 0, eS = 0;
    double lastMax = 0.0;  // lane 31: maximum of its row's W0 and Y0
    for (int s = 0; s < nS; ++s) {
        const int sh = s > 0 ? binExp(__shfl_sync(0xffffffffu, lastMax, 31)) : 0;
        eS += sh;
        const double f = ldexp(1.0, -sh), seedScale = ldexp(1.0, -eS);
        if (lane == 0) Foff[s] = (double)eS;
        const AdjRow r = adjRow(s, lane, M, par, E, sC, s1, s2);
        AdjHist h = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
        double part = 0.0, rowMax = 0.0;
        // lane c holds column 32b + c of row 32s-1 for the current block b
        // (cW, cY) and the next one (nW, nY)
        auto fetch = [&](int b, double &W, double &Y) {
            const int jc = 32 * b + lane;
            W = Y = 0.0;
            if (s > 0 && jc < L) {
                if (CKPT) {
                    const double *a = Ftop + ((size_t)(s - 1) * L + jc) * 2;
                    W = a[0] * f;
                    Y = a[1] * f;
                } else {
                    const size_t a = adjF(L, s - 1, jc + 31, 31);
                    W = F[a] * f;
                    Y = F[a + 1] * f;
                }
            }
        };
        double cW = 0.0, cY = 0.0, nW, nY;
        fetch(0, nW, nY);
        for (int k = 0; k < nSteps; ++k) {
            const int j = k - lane;
            if ((k & 31) == 0) {
                cW = nW;
                cY = nY;
                fetch((k >> 5) + 1, nW, nY);
            }
            if (CKPT && k % kAdjCk == 0) {  // the state the recompute starts from
                double *ck = Fck + (((size_t)s * nCk + k / kAdjCk) * 32 + lane) * kAdjCkVals;
                ck[0] = h.w1; ck[1] = h.w2; ck[2] = h.w3; ck[3] = h.z1; ck[4] = h.z2; ck[5] = h.z3;
                ck[6] = h.u1; ck[7] = h.u2; ck[8] = h.u3; ck[9] = h.pubW; ck[10] = h.pubY;
            }
            double W0, Y0, Z0;
            bool live;
            adjFwdStep(r, h, k, lane, L, cW, cY, cd, pre, pr.bg, rowPad, sC, seedScale, W0, Y0, Z0, live);
            if (live) {
                if (CKPT) {
                    if (lane == 31) {  // the top row, for the next stripe
                        double *a = Ftop + ((size_t)s * L + j) * 2;
                        a[0] = W0;
                        a[1] = Y0;
                    }
                } else {
                    const size_t a = adjF(L, s, k, lane);
                    F[a] = W0;
                    F[a + 1] = Y0;
                    F[a + 2] = Z0;
                }
                part = fma(W0, (double)suf[j], part);
                rowMax = fmax(rowMax, fmax(W0, Y0));
            }
        }
        dxAdd(tm, te, warpSumD(part), eS);
        lastMax = rowMax;
        __syncwarp();  // the stripe's stores before the next stripe's loads
    }
    if (lane == 0) logT[ji] = log(tm) + te * 0.6931471805599453;
    const double invT = tm > 0.0 ? 1.0 / tm : 0.0;

    // ---- phase B: backward, stripes downward, with the gradient sums ----
    double *gP = grad;                                    // (M+2) x 11
    double *gE = grad + (size_t)(M + 2) * kParamFloats;  // (M+1) x 25
    for (int j = lane; j < L + 4; j += 32) {  // the row above the top stripe is zero
        *bnd(nS & 1, 0, j) = 0.0;
        *bnd(nS & 1, 1, j) = 0.0;
    }
    __syncwarp();
    int eB = 0;
    double lastMaxB = 0.0;  // lane 31: maximum of its row's W1 and Y
    for (int s = nS - 1; s >= 0; --s) {
        const int i = 32 * s + 31 - lane;
        const bool rowOK = i <= M;
        const int sh = s < nS - 1 ? binExp(__shfl_sync(0xffffffffu, lastMaxB, 31)) : 0;
        eB += sh;
        const double f = ldexp(1.0, -sh), seedScale = ldexp(1.0, -eB);
        const int eF = (int)Foff[s];
        const int eFp = s > 0 ? (int)Foff[s - 1] : 0;
        const int rowExp = eF + eB - te;
        const int epsExp = (lane == 31 ? eFp : eF) + eB - te;  // Y0[i-1]: row 32s-1 is in stripe s-1
        const int ir = rowOK ? i : M;
        const float *q = par + (size_t)ir * kParamFloats;
        const double enter = (double)q[10] * sC, d0 = q[6], d1 = (double)q[7] * s2, d2 = (double)q[8] * s1;
        const double a0 = (double)q[0] * sC, a1 = (double)q[1] * s1, a2 = (double)q[2] * s2;
        const double b0 = (double)q[3] * sC, eps = q[9], q10 = q[10];
        const float *Erow = E + ir;
        const int rd = (s + 1) & 1, wr = s & 1;  // boundary parity read (row 32s+32) and written (row 32s)
        double gEnter = 0, gD0 = 0, gD1 = 0, gD2 = 0, gA0 = 0, gA1 = 0, gA2 = 0, gEps = 0, gB0 = 0;
#pragma unroll
        for (int c = 0; c < kNumCodes; ++c) geS[c * 32 + lane] = 0.0;
        // Forward blocks of this stripe into the ring: the block of forward
        // step t holds every lane's (W0, Y0, Z0) of that step, and (lane 0's
        // copy) the Y0 of row 32s-1 at forward step t + 31 of stripe s-1.
        const bool below = s > 0;
        // CKPT: the forward blocks of chunk cc of this stripe, recomputed from
        // its checkpoint into buffer cc & 1 (forward lane mapping: lane l is
        // row 32 s + l), as the forward pass computed them.
        int curChunk = -1;
        auto recompute = [&](int cc) {
            const AdjRow r = adjRow(s, lane, M, par, E, sC, s1, s2);
            const double fF = s > 0 ? ldexp(1.0, -(eF - eFp)) : 1.0, seedF = ldexp(1.0, -eF);
            const double *ck = Fck + (((size_t)s * nCk + cc) * 32 + lane) * kAdjCkVals;
            AdjHist h = {ck[0], ck[1], ck[2], ck[3], ck[4], ck[5], ck[6], ck[7], ck[8], ck[9], ck[10]};
            auto fetchTop = [&](int b, double &W, double &Y) {
                const int jc = 32 * b + lane;
                W = Y = 0.0;
                if (s > 0 && jc < L) {
                    const double *a = Ftop + ((size_t)(s - 1) * L + jc) * 2;
                    W = a[0] * fF;
                    Y = a[1] * fF;
                }
            };
            const int k0 = cc * kAdjCk, k1 = min(k0 + kAdjCk, nSteps);
            double *buf = Fbuf + (size_t)(cc & 1) * kAdjCk * 96;
            double cW = 0.0, cY = 0.0, nW, nY;
            fetchTop(k0 >> 5, nW, nY);
            for (int k = k0; k < k1; ++k) {
                if ((k & 31) == 0) {
                    cW = nW;
                    cY = nY;
                    fetchTop((k >> 5) + 1, nW, nY);
                }
                double W0, Y0, Z0;
                bool live;
                adjFwdStep(r, h, k, lane, L, cW, cY, cd, pre, pr.bg, rowPad, sC, seedF, W0, Y0, Z0, live);
                double *o = buf + (size_t)(k - k0) * 96 + 3 * lane;
                o[0] = W0;
                o[1] = Y0;
                o[2] = Z0;
            }
            __threadfence_block();
            __syncwarp();  // the buffer before the copies that read it
        };
        auto issue = [&](int t) {
            if (t >= 0 && t <= L + 30) {
                if (CKPT && t / kAdjCk != curChunk) {  // t descends: each chunk once, in order
                    curChunk = t / kAdjCk;
                    recompute(curChunk);
                }
                double *dst = ring + (t & (kAdjRing - 1)) * kAdjSlot;
                const double *src = CKPT ? Fbuf + ((size_t)((t / kAdjCk) & 1) * kAdjCk + t % kAdjCk) * 96
                                         : F + adjF(L, s, t, 0);
                adjCp16(dst + 2 * lane, src + 2 * lane);
                if (lane < 16) adjCp16(dst + 64 + 2 * lane, src + 64 + 2 * lane);
                if (lane == 16 && below && t + 31 <= L + 30)
                    adjCp8(dst + 96, CKPT ? Ftop + ((size_t)(s - 1) * L + t) * 2 + 1 : F + adjF(L, s - 1, t + 31, 31) + 1);
            }
            adjCommit();
        };
        const int t0 = L + 30;  // the forward step of backward step 0
#pragma unroll
        for (int d = 0; d < kAdjAhead; ++d) issue(t0 - d);
        double n1 = 0, n2 = 0, n3 = 0;     // row i+1 at j+1, j+2, j+3
        double c1 = 0, c2 = 0;             // own row at j+1, j+2
        double zz1 = 0, zz2 = 0, zz3 = 0;  // own Z at j+1, j+2, j+3
        double pubW = 0, pubY = 0;
        double rowMax = 0.0;
        // lane c holds column L-1-(32b+c) of row 32s+32 for the current block
        // b (cW, cY) and the next one (nW, nY)
        auto fetch = [&](int b, double &W, double &Y) {
            const int jc = L - 1 - (32 * b + lane);
            W = Y = 0.0;
            if (jc >= 0) {
                W = *bnd(rd, 0, jc) * f;
                Y = *bnd(rd, 1, jc) * f;
            }
        };
        double cW, cY, nW, nY;
        fetch(0, nW, nY);
        for (int k = 0; k < nSteps; ++k) {
            const int j = L - 1 - (k - lane);
            const int t = t0 - k;
            issue(t - kAdjAhead);
            if ((k & 31) == 0) {
                cW = nW;
                cY = nY;
                fetch((k >> 5) + 1, nW, nY);
            }
            double nj = __shfl_up_sync(0xffffffffu, pubW, 1);
            double ynj = __shfl_up_sync(0xffffffffu, pubY, 1);
            const double bw = __shfl_sync(0xffffffffu, cW, k & 31);
            const double by = __shfl_sync(0xffffffffu, cY, k & 31);
            if (lane == 0) {
                nj = bw;
                ynj = by;
            }
            adjWait<kAdjAhead - 1>();  // blocks t and t-1 are in
            __syncwarp();
            double W = 0.0, Y = 0.0, Z = 0.0;
            if (rowOK && j >= 0 && j < L) {
                const int c = code(j + 1);
                const double ec = (double)Erow[(size_t)c * rowPad];
                const double zbg = zz3 * (double)pr.bg[c];
                W = fma(n3 * ec, enter,
                        fma(ynj, d0, fma(n2, d1, fma(n1, d2, fma(zbg, a0, fma(c2, a2, fma(c1, a1,
                            (double)suf[j] * seedScale)))))));
                Y = fma(eps, ynj, W);
                Z = fma(b0, zbg, W);
                rowMax = fmax(rowMax, Y);  // Y >= W
                if (lane == 31) {          // row 32s: the boundary for the stripe below
                    *bnd(wr, 0, j) = W;
                    *bnd(wr, 1, j) = Y;
                }
                // forward values of the cell: block t, lane 31-lane; Y0 of the
                // row below: block t-1, lane 30-lane (row 32s-1: block t's extra)
                const double *bt = ring + (t & (kAdjRing - 1)) * kAdjSlot;
                const double wA = bt[3 * (31 - lane)], zA = bt[3 * (31 - lane) + 2];
                double yA = 0.0;
                if (lane < 31)
                    yA = ring[((t - 1) & (kAdjRing - 1)) * kAdjSlot + 3 * (30 - lane) + 1];
                else if (below)
                    yA = bt[96];
                const double me = wA * n3 * sC;  // d/d(enter * e) without the other factor
                gEnter = fma(me, ec, gEnter);
                geS[c * 32 + lane] = fma(me, q10, geS[c * 32 + lane]);
                gD0 = fma(wA, ynj, gD0);
                gD1 = fma(wA, n2, gD1);
                gD2 = fma(wA, n1, gD2);
                gA0 = fma(wA, zbg, gA0);
                gA1 = fma(wA, c1, gA1);
                gA2 = fma(wA, c2, gA2);
                gEps = fma(yA, ynj, gEps);
                gB0 = fma(zA, zbg, gB0);
                if (POST) {
                    cellP[(size_t)i * L + j] = ldexp(wA * W * invT, rowExp);
                    if (j + 3 < L) matchP[(size_t)i * L + j + 3] = ldexp(me * ec * q10 * invT, rowExp);
                    if (j < 3) matchP[(size_t)i * L + j] = 0.0;
                }
            }
            n3 = n2; n2 = n1; n1 = nj;
            c2 = c1; c1 = W;
            zz3 = zz2; zz2 = zz1; zz1 = Z;
            pubW = W;
            pubY = Y;
        }
        adjWait<0>();  // no copy outlives the stripe (the ring is reused)
        if (lane == 31)  // columns L..L+3 of the boundary row stay zero
            for (int j = L; j < L + 4; ++j) {
                *bnd(wr, 0, j) = 0.0;
                *bnd(wr, 1, j) = 0.0;
            }
        lastMaxB = rowMax;
        __syncwarp();  // the boundary row before the next stripe reads it; ring and geS complete
        // d log T = dT / T: each lane adds its row's sums times 2^(offsets) / T
        // (the per-base scale of each coefficient applied here, once per row)
        if (rowOK) {
            double *g = gP + (size_t)i * kParamFloats;
            const double v[9] = {gA0 * sC, gA1 * s1, gA2 * s2, gB0 * sC, gD0, gD1 * s2, gD2 * s1, gEps, gEnter};
            const int slot[9] = {0, 1, 2, 3, 6, 7, 8, 9, 10};
#pragma unroll
            for (int k = 0; k < 9; ++k) {
                const double x = ldexp(v[k] * invT, k == 7 ? epsExp : rowExp);
                if (x != 0.0) atomicAdd(g + slot[k], x);
            }
            double *gr = gE + (size_t)i * kNumCodes;
            for (int cc = 0; cc < kNumCodes; ++cc) {
                const double x = ldexp(geS[cc * 32 + lane] * invT, rowExp);
                if (x != 0.0) atomicAdd(gr + cc, x);
            }
        }
        __syncwarp();
    }
}

}  // namespace dmst
