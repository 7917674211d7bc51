// The plain schedule: one (read, profile) pair per kernel launch, the
// baseline the batched persistent kernel is measured against.  The launch is
// one CTA whose warps share the pair: its stripes (32 R profile rows each)
// are dealt to the warps round-robin and run as a stripe pipeline (the
// exact path's protocol, dp_exact_wave.cuh: each warp waits, bounded, until
// the stripe before its own has written the boundary row it needs), with
// the batched kernel's fast-path arithmetic (kMid or kFilter).  A pair of
// nS stripes keeps min(nS, 8) warps busy, so its time is that of the one
// pair alone on the GPU, with none of the batching across pairs.  The
// results are those of the batched kernel bit for bit; a pair whose wait
// ran out is handed to the exact path (its mid is set to NaN, which the
// flag kernel routes there).
#pragma once

#include "dp_exact_wave.cuh"

namespace dmst {

constexpr int kPlainWarps = kPipeWarps;

// Scratch of one pair (floats): W1 of every stripe (nS x D x 32 R) and the
// 2W boundary rings of 4 P floats.
__host__ __device__ inline long long plainScratchFloats(int M, int L, int R) {
    const long long S = (long long)kLanes * R;
    const long long nS = (M + 1 + S - 1) / S;
    const long long Pw = wavePeriod(L);
    const long long D = Pw + kLanes - 1;
    const long long W = nS < kPlainWarps ? nS : kPlainWarps;
    return nS * D * S + 2LL * W * 4 * Pw;
}

template <int R, bool MID>
__global__ void __launch_bounds__(kPlainWarps * kLanes, 1)
    plainKernel(const DevPair *pairs, int pi, const DevProfile *profiles, const float *emit, const float *params,
                const uint8_t *codes, const float *seeds, const PairScales *scales, float *scratch, PairOut *out,
                int spinLimit) {
    extern __shared__ float4 smRaw[];
    Window *wins = reinterpret_cast<Window *>(smRaw);
    __shared__ float smBg[32];
    __shared__ int progress[kPlainWarps];
    __shared__ int abortFlag;
    __shared__ float part[4][kPlainWarps];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const DevPair p = pairs[pi];
    const DevProfile &pr = profiles[p.prof];
    constexpr int S = kLanes * R;
    const int nS = (p.M + 1 + S - 1) / S;
    const int W = min(nS, kPlainWarps);
    Window &win = wins[warp];
    if (warp == 0) smBg[lane] = lane < kNumCodes ? pr.bg[lane] : 0.0f;
    if (threadIdx.x == 0) abortFlag = 0;
    if (lane == 0) {
        PairCold &c = win.cold;
        c.codes = codes + p.codeOff;
        c.pre = seeds + p.seedOff;
        c.suf = c.pre + p.L;
        c.coef = params + coefOffOf(pr.paramOff, pr.M);
        c.coefStride = pr.rowPad;
        c.smBg = smBg;
        c.sc = scales[pi];
        c.M = p.M;
    }
    PipeSync ps;
    ps.progress = progress;
    ps.abort = &abortFlag;
    ps.W = W;
    ps.spinLimit = spinLimit > 0 ? spinLimit : kPipeSpinLimit;
    SweepArgs a;
    a.cold = &win.cold;
    a.smE = emit + pr.emitOff;
    a.L = p.L;
    a.rowPad = pr.rowPad;
    a.nS = nS;
    const int Pw = wavePeriod(p.L);
    a.P = Pw + kPipeExtra;
    a.D = Pw + kLanes - 1;
    a.sFirst = warp;
    a.sStep = W;
    a.nMine = warp < W ? (nS - warp + W - 1) / W : 0;
    a.ringSlots = 2 * W;
    a.ringStride = 4LL * Pw;
    a.w1 = scratch;
    a.ring = scratch + (size_t)nS * a.D * S;
    a.alignOut = nullptr;
    float filt = 0.0f, maxY = 0.0f, mid = 0.0f, maxFw = 0.0f;
    bool ok = true;
    if (lane == 0) progress[warp] = warp < W ? pipePos(a, -1) : INT_MAX;
    __syncthreads();
    if (warp < W) ok = backwardSweepPipe<R, MID ? kMid : kFilter>(a, win, warp, lane, ps, nullptr, nullptr, &filt, &maxY);
    __syncthreads();  // every stripe's W1 is stored; the rings are free
    ok = ok && abortFlag == 0;
    if (MID) {
        if (lane == 0) progress[warp] = warp < W ? pipePos(a, -1) : INT_MAX;
        __syncthreads();
        if (warp < W && ok) ok = forwardSweepPipe<R, kMid>(a, win, warp, lane, ps, nullptr, nullptr, &mid, &maxFw);
        __syncthreads();
        ok = ok && abortFlag == 0;
    }
    filt = warpMax(filt);
    maxY = warpMax(maxY);
    mid = warpMax(mid);
    maxFw = warpMax(maxFw);
    if (lane == 0) {
        part[0][warp] = filt;
        part[1][warp] = maxY;
        part[2][warp] = mid;
        part[3][warp] = maxFw;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        PairOut o{0.0f, 0.0f, 0.0f, 0.0f};
        for (int w = 0; w < kPlainWarps; ++w) {
            o.filt = fmaxf(o.filt, part[0][w]);
            o.maxYb = fmaxf(o.maxYb, part[1][w]);
            o.mid = fmaxf(o.mid, part[2][w]);
            o.maxFw = fmaxf(o.maxFw, part[3][w]);
        }
        if (!ok) {  // a wait ran out: NaN results (the flag kernel queues a NaN mid for the exact path)
            o.mid = __int_as_float(0x7fc00000);
            o.filt = __int_as_float(0x7fc00000);
        }
        out[pi] = o;
    }
}

}  // namespace dmst
