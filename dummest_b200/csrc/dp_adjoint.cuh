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
// One thread per pair, FP64 throughout.  Every row is held at its own
// power-of-two offset: a row reads the row before it (forward) or after it
// (backward) multiplied by 2^-e, e the binary exponent of that row's maximum,
// and the offsets add up along the sweep.  Products of a forward and a
// backward value then stay in double range for any score (homologs reach
// 2^2000 and more); values more than ~1000 binades below their row's maximum
// flush to zero, the double-range counterpart of the reference's float row
// rescaling.  T is kept as a mantissa and a binary exponent.
//
// Phase A runs the forward and keeps (W0, Y0, Z0) of every cell and each
// row's offset; phase B runs the backward, accumulates the row sums (reduced
// over the warp before the atomics: the 32 pairs of a warp share the profile
// and step through its rows together) and writes the posteriors if asked.
// The 32 pairs of a warp store their cells interleaved: one coalesced
// 256-byte access per value and step.
#pragma once

#include "dp_common.cuh"

namespace dmst {

struct AdjointJob {
    int pair;         // index into the pair descriptors
    int Lw;           // longest read of the warp (store row length)
    long long fOff;   // double offset of the warp's forward store (lane-interleaved)
    long long bOff;   // double offset of the warp's backward row buffers
    long long pOff;   // double offset of the pair's posterior tables, -1 for none
};
static_assert(sizeof(AdjointJob) == 32, "AdjointJob layout");

// Forward store of a warp: (M+1) x Lw cells x 3 values, then the M+1 row
// offsets, each entry lane-interleaved.
__host__ __device__ __forceinline__ long long adjStoreDoubles(int M, int Lw) {
    return ((long long)(M + 1) * Lw * 3 + (M + 1)) * 32;
}
__device__ __forceinline__ size_t adjF(int Lw, int i, int j, int t, int lane) {
    return ((((size_t)i * Lw + j) * 3 + t) << 5) + lane;
}
__device__ __forceinline__ size_t adjE(int Lw, int M, int i, int lane) {
    return (((size_t)(M + 1) * Lw * 3 + i) << 5) + lane;
}
// Backward two-row buffer of a warp: parity p, column j (0..Lw+3), value t (W1 or Y).
__host__ __device__ __forceinline__ long long adjRowDoubles(int Lw) { return 2LL * (Lw + 4) * 2 * 32; }
__device__ __forceinline__ size_t adjB(int Lw, int p, int j, int t, int lane) {
    return ((((size_t)p * (Lw + 4) + j) * 2 + t) << 5) + lane;
}

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

__device__ __forceinline__ double warpSum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// grad: (M+2) x 11 Params gradients then (M+1) x 25 emission gradients of
// the profile, accumulated over the pairs (each term already divided by the
// pair's T).  logT: per job, natural log.  post: posterior tables (jobs with
// pOff >= 0).  Launched with whole warps; lanes past nJobs step through the
// rows with no columns so that the warp reductions see every lane.
__global__ void __launch_bounds__(128) adjointKernel(const AdjointJob *jobs, int nJobs, const DevPair *pairs,
                                                      const DevProfile *profiles, const float *emit,
                                                      const float *params, const uint8_t *codes, const float *seeds,
                                                      const PairScales *scales, double *fstore, double *bstore,
                                                      double *grad, double *logT, double *post) {
    const int ji = blockIdx.x * blockDim.x + threadIdx.x;
    const int lane = threadIdx.x & 31;
    const int first = ji - lane;  // the warp's first job
    if (first >= nJobs) return;   // whole warps only
    const bool valid = ji < nJobs;
    const AdjointJob job = jobs[valid ? ji : first];
    const DevPair p = pairs[job.pair];
    const DevProfile &pr = profiles[p.prof];
    const int L = valid ? p.L : 0, M = p.M, Lw = job.Lw, rowPad = pr.rowPad;
    const uint8_t *cd = codes + p.codeOff;
    const float *pre = seeds + p.seedOff;
    const float *suf = pre + p.L;
    const float *E = emit + pr.emitOff;
    const float *par = params + pr.paramOff;
    const PairScales sc = scales[job.pair];
    const double sC = sc.sC, s1 = sc.s1, s2 = sc.s2;
    double *F = fstore + job.fOff;
    double *B = bstore + job.bOff;
    double *cellP = (valid && job.pOff >= 0) ? post + job.pOff : nullptr;
    double *matchP = cellP ? cellP + (size_t)(M + 1) * L : nullptr;
    auto code = [&](int j) -> int { return (j >= 0 && j < L) ? (int)cd[j] : kPad; };
    auto bgc = [&](int j) -> double { return (double)pr.bg[code(j)]; };
    auto e = [&](int i, int c) -> double { return (double)E[(size_t)c * rowPad + i]; };

    // ---- phase A: forward (the adjoint), rows 0..M ----
    double tm = 0.0;
    int te = 0;
    int eF = 0;
    double maxPrev = 0.0;  // maximum of the previous row's W0 and Y0
    for (int i = 0; i <= M; ++i) {
        const float *q = par + (size_t)i * kParamFloats;
        const float *qp = par + (size_t)(i > 0 ? i - 1 : 0) * kParamFloats;
        const double a0 = q[0], a1 = (double)q[1] * s1, a2 = (double)q[2] * s2, b0 = q[3];
        const double d0 = q[6], eps = q[9];
        // the previous row's coefficients feed this row's incoming sums
        const double pEnter = i > 0 ? (double)qp[10] * sC : 0.0, pd1 = i > 0 ? (double)qp[7] * s2 : 0.0;
        const double pd2 = i > 0 ? (double)qp[8] * s1 : 0.0;
        const int sh = i > 0 ? binExp(maxPrev) : 0;
        eF += sh;
        const double f = ldexp(1.0, -sh), seedScale = ldexp(1.0, -eF);
        if (valid) F[adjE(Lw, M, i, lane)] = (double)eF;
        double w1 = 0, w2 = 0, w3 = 0, z1 = 0, z2 = 0, z3 = 0;  // this row at j-1, j-2, j-3
        double u1 = 0, u2 = 0, u3 = 0;                          // previous row's W0 at j-1, j-2, j-3
        double part = 0.0, rowMax = 0.0;
        for (int j = 0; j < L; ++j) {
            double uj = 0.0, yPrev = 0.0;
            if (i > 0) {
                uj = F[adjF(Lw, i - 1, j, 0, lane)] * f;
                yPrev = F[adjF(Lw, i - 1, j, 1, lane)] * f;
            }
            const int c = code(j - 2);
            const double win = pEnter * (i > 0 ? e(i - 1, c) : 0.0) * u3 + yPrev + pd1 * u2 + pd2 * u1;
            const double Z0 = bgc(j - 2) * sC * (a0 * w3 + b0 * z3);
            const double W0 = win + Z0 + a1 * w1 + a2 * w2 + (double)pre[j] * seedScale;
            const double Y0 = d0 * W0 + eps * yPrev;
            F[adjF(Lw, i, j, 0, lane)] = W0;
            F[adjF(Lw, i, j, 1, lane)] = Y0;
            F[adjF(Lw, i, j, 2, lane)] = Z0;
            part += W0 * (double)suf[j];
            rowMax = fmax(rowMax, fmax(W0, Y0));
            w3 = w2; w2 = w1; w1 = W0;
            z3 = z2; z2 = z1; z1 = Z0;
            u3 = u2; u2 = u1; u1 = uj;
        }
        dxAdd(tm, te, part, eF);
        maxPrev = rowMax;
    }
    if (valid) logT[ji] = log(tm) + te * 0.6931471805599453;
    const double invT = tm > 0.0 ? 1.0 / tm : 0.0;

    // ---- phase B: backward, rows M..0, with the gradient sums ----
    for (int j = 0; j < L + 4; ++j) {  // row M+1 is zero
        B[adjB(Lw, (M + 1) & 1, j, 0, lane)] = 0.0;
        B[adjB(Lw, (M + 1) & 1, j, 1, lane)] = 0.0;
    }
    double *gP = grad;                                    // (M+2) x 11
    double *gE = grad + (size_t)(M + 2) * kParamFloats;  // (M+1) x 25
    int eB = 0;
    double maxNext = 0.0;  // maximum of the next row's W1 and Y
    for (int i = M; i >= 0; --i) {
        const float *q = par + (size_t)i * kParamFloats;
        const double enter = (double)q[10] * sC, d0 = q[6], d1 = (double)q[7] * s2, d2 = (double)q[8] * s1;
        const double a0 = (double)q[0] * sC, a1 = (double)q[1] * s1, a2 = (double)q[2] * s2;
        const double b0 = (double)q[3] * sC, eps = q[9];
        const int cur = i & 1, nxt = (i + 1) & 1;
        const int sh = i < M ? binExp(maxNext) : 0;
        eB += sh;
        const double f = ldexp(1.0, -sh), seedScale = ldexp(1.0, -eB);
        // offsets of this row's products relative to T
        const int eFi = valid ? (int)F[adjE(Lw, M, i, lane)] : 0;
        const int eFp = (valid && i > 0) ? (int)F[adjE(Lw, M, i - 1, lane)] : 0;
        const int rowExp = eFi + eB - te, epsExp = eFp + eB - te;
        double gEnter = 0, gD0 = 0, gD1 = 0, gD2 = 0, gA0 = 0, gA1 = 0, gA2 = 0, gEps = 0, gB0 = 0;
        double ge[kNumCodes];
#pragma unroll
        for (int c = 0; c < kNumCodes; ++c) ge[c] = 0.0;
        double n1 = B[adjB(Lw, nxt, L, 0, lane)] * f, n2 = B[adjB(Lw, nxt, L + 1, 0, lane)] * f;
        double n3 = B[adjB(Lw, nxt, L + 2, 0, lane)] * f;  // row i+1 at j+1, j+2, j+3
        double c1 = 0, c2 = 0;                              // this row at j+1, j+2
        double zz1 = 0, zz2 = 0, zz3 = 0;                   // Z of this row at j+1, j+2, j+3
        double rowMax = 0.0;
        for (int j = L - 1; j >= 0; --j) {
            const double nj = B[adjB(Lw, nxt, j, 0, lane)] * f;
            const double ynj = B[adjB(Lw, nxt, j, 1, lane)] * f;
            const int c = code(j + 1);
            const double ec = e(i, c), bg1 = bgc(j + 1);
            const double zbg = zz3 * bg1;
            const double W = n3 * ec * enter + ynj * d0 + n2 * d1 + n1 * d2 + zbg * a0 + c2 * a2 + c1 * a1 +
                             (double)suf[j] * seedScale;
            const double Y = eps * ynj + W;
            const double Z = b0 * zbg + W;
            B[adjB(Lw, cur, j, 0, lane)] = W;
            B[adjB(Lw, cur, j, 1, lane)] = Y;
            rowMax = fmax(rowMax, Y);  // Y >= W
            const double wA = F[adjF(Lw, i, j, 0, lane)];
            const double zA = F[adjF(Lw, i, j, 2, lane)];
            const double yA = i > 0 ? F[adjF(Lw, i - 1, j, 1, lane)] : 0.0;
            const double me = wA * n3 * sC;  // d/d(enter * e) without the other factor
            gEnter += me * ec;
            ge[c] += me * (double)q[10];
            gD0 += wA * ynj;
            gD1 += wA * n2 * s2;
            gD2 += wA * n1 * s1;
            gA0 += wA * zbg * sC;
            gA1 += wA * c1 * s1;
            gA2 += wA * c2 * s2;
            gEps += yA * ynj;
            gB0 += zA * zbg * sC;
            if (cellP) {
                cellP[(size_t)i * L + j] = ldexp(wA * W * invT, rowExp);
                if (j + 3 < L) matchP[(size_t)i * L + j + 3] = ldexp(me * ec * (double)q[10] * invT, rowExp);
                if (j < 3) matchP[(size_t)i * L + j] = 0.0;
            }
            n3 = n2; n2 = n1; n1 = nj;
            c2 = c1; c1 = W;
            zz3 = zz2; zz2 = zz1; zz1 = Z;
        }
        // the row's columns L..L+3 stay zero for the row above
        for (int j = L; j < L + 4; ++j) {
            B[adjB(Lw, cur, j, 0, lane)] = 0.0;
            B[adjB(Lw, cur, j, 1, lane)] = 0.0;
        }
        maxNext = rowMax;
        // d log T = dT / T: scale each sum by 2^(offsets) / T, then reduce the warp
        const double sRow = invT, sEps = invT;
        double v[10] = {gA0, gA1, gA2, gB0, gD0, gD1, gD2, gEps, gEnter, 0.0};
        const int slot[9] = {0, 1, 2, 3, 6, 7, 8, 9, 10};
#pragma unroll
        for (int k = 0; k < 9; ++k) {
            const double x = ldexp(v[k] * (k == 7 ? sEps : sRow), k == 7 ? epsExp : rowExp);
            const double s = warpSum(valid ? x : 0.0);
            if (lane == 0 && s != 0.0) atomicAdd(gP + (size_t)i * kParamFloats + slot[k], s);
        }
        double *gr = gE + (size_t)i * kNumCodes;
#pragma unroll
        for (int cc = 0; cc < kNumCodes; ++cc) {
            const double s = warpSum(valid ? ldexp(ge[cc] * sRow, rowExp) : 0.0);
            if (lane == 0 && s != 0.0) atomicAdd(gr + cc, s);
        }
    }
}

}  // namespace dmst
