// Exact row-rescaled DP on the wavefront, one warp per pair, for the pairs
// the fast kernel cannot score exactly (a row maximum above RESCALE_THRESH,
// or a product beyond float range).
//
// The reference decides each row's rescale after the whole row is known
// (dummest-dp-backward.hh:560-573, dummest-dp-forward.hh:228-242), which a
// wavefront cannot wait for.  So each direction runs twice (the kDiscover
// and kReplay modes of the sweeps in dp_wavefront.cuh):
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

#include "dp_exact.cuh"
#include "dp_wavefront.cuh"

namespace dmst {

constexpr int kExactR = 4;  // rows per lane of the exact path

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

// Scratch per job (floats): W1 nS*D*32R, ring 4P, rowMax M+1, rowCnt M+1,
// cntB M+2, cntF M+2.
__host__ __device__ inline long long exactWaveScratch(int M, int L) {
    const long long S = (long long)kLanes * kExactR;
    const long long nS = (M + 1 + S - 1) / S;
    const long long P = wavePeriod(L);
    const long long D = P + kLanes - 1;
    return nS * D * S + 4 * P + 2LL * (M + 1) + 2LL * (M + 2) + 64;
}

// One warp per CTA; dynamic shared memory = the emission table (tableFloats)
// and one Window.
__global__ void __launch_bounds__(kLanes) exactWaveKernel(const ExactWaveJob *jobs, int n, const DevPair *pairs,
                                                           const DevProfile *profiles, const float *emit,
                                                           const float *params, const uint8_t *codes,
                                                           const float *seeds, const PairScales *scales,
                                                           float *scratch, ExactOut *out, int tableFloats) {
    extern __shared__ float4 smRaw[];
    float *smE = reinterpret_cast<float *>(smRaw);
    Window &win = *reinterpret_cast<Window *>(smE + tableFloats);
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
        if (lane == 0) {
            PairCold &c = win.cold;
            c.codes = codes + p.codeOff;
            c.pre = seeds + p.seedOff;
            c.suf = c.pre + p.L;
            c.params = params + pr.paramOff;
            c.smBg = smBg;
            c.sc = scales[job.pair];
            c.M = p.M;
        }
        __syncwarp();
        SweepArgs a;
        a.cold = &win.cold;
        a.smE = smE;
        a.L = p.L;
        a.rowPad = rowPad;
        a.nS = (p.M + 1 + kLanes * kExactR - 1) / (kLanes * kExactR);
        a.P = wavePeriod(p.L);
        a.D = a.P + kLanes - 1;
        float *base = scratch + job.scratchOff;
        a.w1 = base;
        a.ring = base + (size_t)a.nS * a.D * kLanes * kExactR;
        ExactRows x;
        x.rowMax = a.ring + 4 * (size_t)a.P;
        x.rowCnt = reinterpret_cast<int *>(x.rowMax + (p.M + 1));
        x.cntB = x.rowCnt + (p.M + 1);
        x.cntF = x.cntB + (p.M + 2);
        ExactBest filt{0.0, 0}, mid{0.0, 0};
        float f0, f1;
        backwardSweep<kExactR, kDiscover>(a, win, lane, f0, f1, &x, nullptr);
        __syncwarp();
        if (lane == 0) scanCounts(x.rowMax, x.rowCnt, x.cntB, p.M, true);
        __syncwarp();
        forwardSweep<kExactR, kDiscover>(a, win, lane, f0, f1, &x, nullptr);
        __syncwarp();
        if (lane == 0) scanCounts(x.rowMax, x.rowCnt, x.cntF, p.M, false);
        __syncwarp();
        backwardSweep<kExactR, kReplay>(a, win, lane, f0, f1, &x, &filt);
        __syncwarp();
        forwardSweep<kExactR, kReplay>(a, win, lane, f0, f1, &x, &mid);
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
