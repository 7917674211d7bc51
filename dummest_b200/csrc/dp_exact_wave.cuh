// Exact row-rescaled DP on the wavefront, for the pairs the fast kernel
// cannot score exactly (a row maximum above RESCALE_THRESH, or a product
// beyond float range).  One CTA per pair; its warps split the pair's stripes
// (below).
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
//
// Stripe pipeline.  A pair's stripes (32 R rows each) are dealt round-robin
// to the CTA's W warps: warp w runs stripes w, w + W, ... in processing order
// (top-down in the backward, bottom-up in the forward).  The rows crossing
// from stripe sp to sp+1 go through ring (sp mod 2W) in global memory.  Every
// warp publishes, in shared memory, how far its ring-writing lane has got
// (the position sp P' + column of the next column it computes), and before
// each refill of its staging window a warp waits until the stripe before
// each stripe it stages has written the ring columns the refill reads, and
// until the ring slot it is about to overwrite has been read.  Every wait is
// on a stripe earlier in processing order, and the stripe period P' = P + 128
// is long enough that a warp's window never reaches its next stripe before
// its current stripe's columns are all computed and published, so the waits
// cannot form a cycle.  Every wait is bounded: past the limit it sets the
// CTA's abort flag, all warps leave their sweeps at the next block, and the
// pair's result is marked failed.
#pragma once

#include "dp_exact.cuh"
#include "dp_traceback_job.cuh"
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

constexpr int kPipeWarps = 8;        // warps per CTA of the exact path
constexpr int kPipeExtra = 128;      // stripe period P' = P + kPipeExtra
constexpr int kPipeSpinLimit = 1 << 24;  // default iterations of a wait (64 ns sleeps) before it gives up
static_assert(kPipeExtra >= kLanes - 1 + 2 * kBlock, "a window never reaches the next stripe early");

__host__ __device__ inline int pipePeriod(int L) { return wavePeriod(L) + kPipeExtra; }

// Scratch per job (floats): W1 nS*D*32R, rings 2W x 4P, rowMax M+1, rowCnt
// M+1, cntB M+2, cntF M+2, and with anchors the stripes' column partials
// nS x L x 3.
__host__ __device__ inline long long exactWaveScratch(int M, int L, int W, bool anchors = false) {
    const long long S = (long long)kLanes * kExactR;
    const long long nS = (M + 1 + S - 1) / S;
    const long long P = wavePeriod(L);
    const long long D = P + kLanes - 1;
    return nS * D * S + 2LL * W * 4 * P + 2LL * (M + 1) + 2LL * (M + 2) + 64 + (anchors ? nS * L * 3 : 0);
}

struct PipeSync {
    volatile int *progress;  // [kPipeWarps]: ring-writer position of each warp
    volatile int *abort;     // the CTA's abort flag
    int W;                   // warps running stripes
    int spinLimit;           // iterations of a wait before it gives up (sets the abort flag)
};

// Position of this warp's ring-writing lane (local time t0 - 31) at block
// boundary t0, and publication of it (after the lane's ring stores).
__device__ __forceinline__ int pipePos(const SweepArgs &a, int lt) {
    if (lt < 0) return a.sFirst * a.P;
    const int k = lt / a.P;
    if (k >= a.nMine) return INT_MAX;
    return (a.sFirst + k * a.sStep) * a.P + (lt - k * a.P);
}
__device__ __forceinline__ void pipePublish(const PipeSync &ps, int warp, int pos, int lane) {
    __threadfence_block();  // each lane's ring stores (lane 0 backward, lane 31 forward) ...
    __syncwarp();
    if (lane == 0) ps.progress[warp] = pos;  // ... before the position
}

// Lane 0 waits until warp w's position reaches target; false on abort.
__device__ __forceinline__ bool pipeWaitOne(const PipeSync &ps, int w, int target) {
    int it = 0;
    while (ps.progress[w] < target) {
        if (*ps.abort) return false;
        if (++it > ps.spinLimit) {
            *ps.abort = 1;
            return false;
        }
        __nanosleep(64);
    }
    return true;
}

// Before the block of local times [t0, t0 + kBlock) and the refill of the
// window entries [fill, fill + kBlock): the ring columns the refill reads are
// written, and the ring slots this block writes have been read.  Warp-uniform.
__device__ __forceinline__ bool pipeReady(const PipeSync &ps, const SweepArgs &a, int t0, int fill, int lane) {
    bool ok = true;
    if (lane == 0) {
        const int total = a.nMine * a.P;
        // readers: the last entry of each stripe the refill touches
        for (int u = fill; ok && u < fill + kBlock && u < total;) {
            const int k = u / a.P;
            const int kEnd = min(min(fill + kBlock, total), (k + 1) * a.P) - 1;  // last entry in stripe k
            const int sp = a.sFirst + k * a.sStep;
            const int jj = min(kEnd - k * a.P, a.L - 1);
            if (sp > 0 && u - k * a.P < a.L) ok = pipeWaitOne(ps, (sp - 1) % ps.W, (sp - 1) * a.P + jj + 1);
            u = (k + 1) * a.P;
        }
        // writers: before overwriting ring slot (sp mod 2W), stripe r = sp - 2W + 1 (which
        // reads the slot's previous contents) has staged all its columns: its writer lane
        // is past column L, and a warp's refills run at least 78 steps ahead of it
        for (int lt = max(t0 - (kLanes - 1), 0); ok && lt < t0 + kBlock - (kLanes - 1) && lt < total;) {
            const int k = lt / a.P;
            const int sp = a.sFirst + k * a.sStep;
            const int r = sp - a.ringSlots + 1;
            if (sp < a.nS - 1 && r >= 1) ok = pipeWaitOne(ps, r % ps.W, r * a.P + a.L);
            lt = (k + 1) * a.P;
        }
    }
    ok = __shfl_sync(kFull, ok, 0);
    __syncwarp();
    __threadfence_block();  // the positions seen before the refill's ring loads
    return ok;
}

// The sweeps of one warp in a stripe pipeline.  The fast mode (kMid) also
// gives the warp's share of the float maxima (filter best and largest Y in
// the backward, mid and largest W0 / Y0 in the forward) through the optional
// outputs; warps reduce them afterwards.
template <int R, int MODE>
__device__ bool backwardSweepPipe(const SweepArgs &a, Window &win, int warp, int lane, const PipeSync &ps,
                                  const ExactRows *x, ExactBest *exact, float *filtOut = nullptr,
                                  float *maxYOut = nullptr) {
    BwdState<R, MODE> b;
#pragma unroll
    for (int q = 0; q < 3; ++q) {
#pragma unroll
        for (int k = 0; k < R; ++k) b.h[q][k] = b.z[q][k] = 0.0f;
        b.rb[q] = 0.0f;
    }
#pragma unroll
    for (int k = 0; k < R; ++k) {
        b.rmax[k] = 0.0f;
        b.cOut[k] = 0;
        b.fOut[k] = 1.0f;
        b.rowBest[k] = 0.0;
    }
    b.sendW = b.sendY = b.filt = b.maxY = 0.0f;
    b.sendC = b.cnt = 0;
    b.u = -(kLanes - 1 - lane);  // lane 31 leads
    b.sp = a.sFirst;
    b.jj = 0;
    b.wp = a.w1;
    const int total = a.nMine * a.P;
    const int T = (total + (kLanes - 1) + 2) / 3 * 3;
    if (!pipeReady(ps, a, -kBlock, 0, lane)) return false;
    fillBlock<true, true>(win, a, 0, lane);
    for (int t0 = 0; t0 < T; t0 += kBlock) {
        pipePublish(ps, warp, pipePos(a, t0 - (kLanes - 1)), lane);
        if (!pipeReady(ps, a, t0, t0 + kBlock, lane)) return false;
        fillBlock<true, true>(win, a, t0 + kBlock, lane);
        const int n = (t0 + kBlock < T ? kBlock : T - t0);
#pragma unroll 1
        for (int g = 0; g < n; g += 3) {
            backwardStep<R, MODE, 0, true>(b, a, win, lane, total, x, exact);
            backwardStep<R, MODE, 1, true>(b, a, win, lane, total, x, exact);
            backwardStep<R, MODE, 2, true>(b, a, win, lane, total, x, exact);
        }
    }
    pipePublish(ps, warp, INT_MAX, lane);
    if (filtOut) *filtOut = b.filt;
    if (maxYOut) *maxYOut = b.maxY;
    return true;
}

template <int R, int MODE, bool ANCH = false>
__device__ bool forwardSweepPipe(const SweepArgs &a, Window &win, int warp, int lane, const PipeSync &ps,
                                 const ExactRows *x, ExactBest *exact, float *bestOut = nullptr,
                                 float *maxOut = nullptr) {
    FwdState<R, MODE> f;
#pragma unroll
    for (int h = 0; h < 3; ++h)
#pragma unroll
        for (int k = 0; k < R; ++k) f.w[h][k] = f.z[h][k] = 0.0f;
#pragma unroll
    for (int k = 0; k < R; ++k) {
        f.rmax[k] = 0.0f;
        f.cIn[k] = f.cB[k] = 0;
        f.fOut[k] = 1.0f;
        f.rowBest[k] = 0.0;
    }
    f.sendIn = f.sendY = f.best = f.mx = 0.0f;
    f.sendC = f.cnt = 0;
    f.sendAM = 0.0f;
    f.sendAE = f.sendAR = 0;
    f.u = -lane;  // lane 0 leads
    f.s = a.sFirst;
    f.j = 0;
    const int total = a.nMine * a.P;
    const int T = (total + (kLanes - 1) + 5) / 6 * 6;
    constexpr bool kReadW1 = MODE == kReplay || MODE == kMid;
    W1Stage<R, true> st{-lane, a.sFirst, 0};
    if (kReadW1) {
#pragma unroll
        for (int k = 0; k < kW1Ahead; ++k) st.issue(a, win, k, lane, total);
    }
    bool ok = pipeReady(ps, a, -kBlock, 0, lane);
    if (ok) fillBlock<false, true>(win, a, 0, lane);
    for (int t0 = 0; ok && t0 < T; t0 += kBlock) {
        pipePublish(ps, warp, pipePos(a, t0 - (kLanes - 1)), lane);
        ok = pipeReady(ps, a, t0, t0 + kBlock, lane);
        if (!ok) break;
        fillBlock<false, true>(win, a, t0 + kBlock, lane);
        const int n = (t0 + kBlock < T ? kBlock : T - t0);
#pragma unroll 1
        for (int g = 0; g < n; g += 6) {
            forwardStaged<R, MODE, 0, ANCH, true>(f, a, win, lane, total, st, x, exact);
            forwardStaged<R, MODE, 1, ANCH, true>(f, a, win, lane, total, st, x, exact);
            forwardStaged<R, MODE, 2, ANCH, true>(f, a, win, lane, total, st, x, exact);
            forwardStaged<R, MODE, 3, ANCH, true>(f, a, win, lane, total, st, x, exact);
            forwardStaged<R, MODE, 4, ANCH, true>(f, a, win, lane, total, st, x, exact);
            forwardStaged<R, MODE, 5, ANCH, true>(f, a, win, lane, total, st, x, exact);
        }
    }
    if (kReadW1) cpAsyncWait<0>();  // no copy outlives the sweep (the slots are reused)
    if (ok) pipePublish(ps, warp, INT_MAX, lane);
    if (bestOut) *bestOut = f.best;
    if (maxOut) *maxOut = f.mx;
    return ok;
}

// Warps running a pair's stripes: one per stripe, at most kPipeWarps.
__host__ __device__ inline int exactWarps(int M) {
    const int nS = (M + 1 + kLanes * kExactR - 1) / (kLanes * kExactR);
    return nS < kPipeWarps ? nS : kPipeWarps;
}

// Pairs the fast kernel could not score exactly (a row maximum above
// RESCALE_THRESH in either sweep, a score beyond float range, or a mid
// product too small for a normal float), or every pair when force is set, go
// to the queue of the exact path.  queueCount[0] counts them.  With `only`,
// pairs whose entry is 0 are skipped.
__global__ void flagKernel(const PairOut *po, int n, int force, int *queue, int *queueCount, const uint8_t *only) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n || (only && !only[k])) return;  // only: the pairs that have mid scores (search survivors)
    const PairOut o = po[k];
    const bool ok = !force && o.maxYb <= kRescaleThresh && o.maxFw <= kRescaleThresh && o.mid < INFINITY &&
                    o.filt < INFINITY && o.mid >= 0x1p-100f;
    if (!ok) queue[atomicAdd(queueCount, 1)] = k;
}

// Orders the exact-path queue costliest pair first ((M + 1) L cells, ties by
// pair position), so that the persistent CTAs that take pairs in queue order
// end on the cheapest ones, and the order no longer depends on the flag
// kernel's atomics.  One CTA of 1024 threads, a bitonic sort of up to
// kQueueSortMax entries in shared memory; a longer queue keeps its order.
constexpr int kQueueSortMax = 4096;
__global__ void __launch_bounds__(1024) queueSortKernel(int *queue, const int *queueCount, const DevPair *pairs) {
    __shared__ unsigned long long key[kQueueSortMax];
    const int cnt = *queueCount;
    if (cnt < 2 || cnt > kQueueSortMax) return;
    int n = 2;
    while (n < cnt) n *= 2;
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        unsigned long long v = 0;  // padding sorts last
        if (i < cnt) {
            const int k = queue[i];
            const DevPair p = pairs[k];
            const long long cells = (long long)(p.M + 1) * p.L;
            const unsigned long long c = cells < 0xffffffffLL ? (unsigned long long)cells : 0xffffffffULL;
            // descending cost, then ascending position (complemented)
            v = (c << 32) | (unsigned long long)(0x7fffffffu - (unsigned)k);
        }
        key[i] = v;
    }
    __syncthreads();
    for (int size = 2; size <= n; size *= 2) {
        for (int stride = size / 2; stride > 0; stride /= 2) {
            for (int i = threadIdx.x; i < n / 2; i += blockDim.x) {
                const int lo = 2 * i - (i & (stride - 1)), hi = lo + stride;
                const bool desc = (lo & size) == 0;  // the final merge (size == n) is descending
                const unsigned long long a = key[lo], b = key[hi];
                if (desc ? a < b : a > b) {
                    key[lo] = b;
                    key[hi] = a;
                }
            }
            __syncthreads();
        }
    }
    for (int i = threadIdx.x; i < cnt; i += blockDim.x) queue[i] = (int)(0x7fffffffu - (unsigned)(key[i] & 0xffffffffULL));
}

// Persistent CTAs of kPipeWarps warps take the queued pairs one at a time
// (queueCount[1] is the next queue position) and score each with its stripes
// spread over the CTA's warps; CTA b uses scratch slot b (slotFloats floats).
// Dynamic shared memory = one Window per warp.  The emission table is read
// from global memory (a stripe's 32 R rows x 25 codes stay in L1), so tall
// profiles leave the shared memory to the windows.
// ANCH: also the per-column anchors of each pair (anchorOff[pair] >= 0: the
// offset of its L columns in anchorM / anchorE / anchorRow).
// ALIGN (with ANCH): pairs with a traceback job (jobOf[pair] >= 0) also keep
// what the traceback tables are built from: the replay sweeps' row-major W0
// and W1 before each row's rescale (at float offset 2 AlignJob::cellOff in
// alignCells: W0 at [0, (M+1) L), W1 at [(M+1) L, 2 (M+1) L)) and the
// reference's rescale counts (AlignJob::rowOff in alignRows: cntB at
// [0, M+2), cntF at [M+2, 2 (M+2))).
// GROUPS = 2: the CTA's warps form two groups of kPipeWarps / 2 that run
// pairs independently (each its own queue position, shared state, scratch
// slot blockIdx.x * 2 + group and named barrier), a pair taking at most
// kPipeWarps / 2 warps: for calls whose pairs have at most that many stripes,
// twice the pairs per CTA, the same per-pair work.
template <bool ANCH, bool ALIGN = false, int GROUPS = 1>
__global__ void __launch_bounds__(kPipeWarps * kLanes, 1)
    exactWaveKernel(const int *queue, int *queueCount, const DevPair *pairs, const DevProfile *profiles,
                    const float *emit, const float *params, const uint8_t *codes, const float *seeds,
                    const PairScales *scales, float *pool, long long slotFloats, ExactOut *out,
                    const long long *anchorOff, float *anchorM, int *anchorE, int *anchorRow,
                    const int *jobOf = nullptr, const AlignJob *jobs = nullptr, float *alignCells = nullptr,
                    int *alignRows = nullptr, int spinLimit = kPipeSpinLimit) {
    static_assert(GROUPS == 1 || GROUPS == 2, "one or two groups");
    constexpr int GW = kPipeWarps / GROUPS;  // warps of a group
    constexpr int GT = GW * kLanes;          // threads of a group
    extern __shared__ float4 smRaw[];
    Window *wins = reinterpret_cast<Window *>(smRaw);
    __shared__ float smBgG[GROUPS][32];
    __shared__ int progressG[GROUPS][GW];
    __shared__ int abortG[GROUPS];
    __shared__ ExactBest bestFG[GROUPS][GW], bestMG[GROUPS][GW];
    __shared__ int smNextG[GROUPS];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int group = warp / GW, gw = warp % GW, gt = threadIdx.x % GT;
    float *smBg = smBgG[group];
    int *progress = progressG[group];
    int &abortFlag = abortG[group];
    ExactBest *bestF = bestFG[group], *bestM = bestMG[group];
    int &smNext = smNextG[group];
    auto gsync = [&]() {
        if (GROUPS == 1)
            __syncthreads();
        else
            asm volatile("bar.sync %0, %1;" ::"r"(1 + group), "r"(GT) : "memory");
    };
    Window &win = wins[warp];
    PipeSync ps;
    ps.progress = progress;
    ps.abort = &abortFlag;
    ps.spinLimit = spinLimit > 0 ? spinLimit : kPipeSpinLimit;
    // Queue positions: with two groups, group g of CTA b first takes position
    // g * gridDim.x + b (so every CTA holds a pair before any holds two, which
    // matters when there are fewer pairs than CTAs), then positions from
    // 2 * gridDim.x on, dynamically.
    bool first = true;
    for (;;) {
        gsync();  // the previous pair is done with the shared state
        if (gt == 0)
            smNext = GROUPS == 1 ? atomicAdd(queueCount + 1, 1)
                                 : (first ? group * (int)gridDim.x + (int)blockIdx.x
                                          : 2 * (int)gridDim.x + atomicAdd(queueCount + 1, 1));
        first = false;
        gsync();
        const int qi = smNext;
        if (qi >= queueCount[0]) break;
        const int pi = queue[qi];
        const DevPair p = pairs[pi];
        const DevProfile &pr = profiles[p.prof];
        const int W = min(exactWarps(p.M), GW);
        ps.W = W;
        if (gw == 0) smBg[lane] = lane < kNumCodes ? pr.bg[lane] : 0.0f;
        if (gt == 0) abortFlag = 0;
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
            bestF[gw] = ExactBest{0.0, 0};
            bestM[gw] = ExactBest{0.0, 0};
        }
        SweepArgs a;
        a.cold = &win.cold;
        a.smE = emit + pr.emitOff;
        a.L = p.L;
        a.rowPad = pr.rowPad;
        a.nS = (p.M + 1 + kLanes * kExactR - 1) / (kLanes * kExactR);
        const int Pw = wavePeriod(p.L);
        a.P = Pw + kPipeExtra;
        a.D = Pw + kLanes - 1;
        a.sFirst = gw;
        a.sStep = W;
        a.nMine = gw < W ? (a.nS - gw + W - 1) / W : 0;
        a.ringSlots = 2 * W;
        a.ringStride = 4LL * Pw;
        float *base = pool + (size_t)(blockIdx.x * GROUPS + group) * slotFloats;
        a.w1 = base;
        a.ring = base + (size_t)a.nS * a.D * kLanes * kExactR;
        ExactRows x;
        x.rowMax = a.ring + (size_t)a.ringSlots * a.ringStride;
        x.rowCnt = reinterpret_cast<int *>(x.rowMax + (p.M + 1));
        x.cntB = x.rowCnt + (p.M + 1);
        x.cntF = x.cntB + (p.M + 2);
        x.anchorPart = reinterpret_cast<float *>(x.cntF + (p.M + 2));
        ExactBest filt{0.0, 0}, mid{0.0, 0};
        bool ok = true;
        float *alignW0 = nullptr, *alignW1 = nullptr;
        int *alignCnt = nullptr;
        if (ALIGN && jobOf[pi] >= 0) {
            const AlignJob &jb = jobs[jobOf[pi]];
            alignW0 = alignCells + 2 * jb.cellOff;  // two floats per cell
            alignW1 = alignW0 + (size_t)(p.M + 1) * p.L;
            alignCnt = alignRows + jb.rowOff;
        }
        // Four sweeps, each over every warp; the counts scan between them.
        for (int phase = 0; phase < 4; ++phase) {
            if (lane == 0) progress[gw] = gw < W ? pipePos(a, -1) : INT_MAX;
            gsync();
            a.alignOut = phase == 2 ? alignW1 : (phase == 3 ? alignW0 : nullptr);
            if (gw < W && ok) {
                switch (phase) {
                case 0: ok = backwardSweepPipe<kExactR, kDiscover>(a, win, gw, lane, ps, &x, nullptr); break;
                case 1: ok = forwardSweepPipe<kExactR, kDiscover>(a, win, gw, lane, ps, &x, nullptr); break;
                case 2: ok = backwardSweepPipe<kExactR, kReplay>(a, win, gw, lane, ps, &x, &filt); break;
                default: ok = forwardSweepPipe<kExactR, kReplay, ANCH>(a, win, gw, lane, ps, &x, &mid); break;
                }
            }
            gsync();
            ok = ok && abortFlag == 0;
            if (phase < 2 && gt == 0 && ok) scanCounts(x.rowMax, x.rowCnt, phase == 0 ? x.cntB : x.cntF, p.M, phase == 0);
        }
        if (ALIGN && ok && alignCnt != nullptr) {
            for (int i = gt; i < p.M + 2; i += GT) {
                alignCnt[i] = x.cntB[i];
                alignCnt[p.M + 2 + i] = x.cntF[i];
            }
        }
        if (ANCH && ok && anchorOff[pi] >= 0) {
            // fold the stripes' partials of each column in row order
            const long long o = anchorOff[pi];
            for (int j = gt; j < p.L; j += GT) {
                float bm = 0.0f;
                int be = 0, br = 0;
                for (int s2 = 0; s2 < a.nS; ++s2) {
                    const float *pp = x.anchorPart + ((size_t)s2 * p.L + j) * 3;
                    const float cm = pp[0];
                    const int ce = __float_as_int(pp[1]);
                    if (xsLessMe(bm, be, cm, ce)) {
                        bm = cm;
                        be = ce;
                        br = __float_as_int(pp[2]);
                    }
                }
                anchorM[o + j] = bm;
                anchorE[o + j] = be;
                anchorRow[o + j] = br;
            }
        }
        filt = warpBest(filt);
        mid = warpBest(mid);
        if (lane == 0) {
            bestF[gw] = filt;
            bestM[gw] = mid;
        }
        gsync();
        if (gt == 0) {
            ExactBest f{0.0, 0}, m{0.0, 0};
            for (int w = 0; w < W; ++w) {
                const ExactBest bf = bestF[w], bm = bestM[w];
                if (bf.m != 0.0 && (f.m == 0.0 || bf.e > f.e || (bf.e == f.e && bf.m > f.m))) f = bf;
                if (bm.m != 0.0 && (m.m == 0.0 || bm.e > m.e || (bm.e == m.e && bm.m > m.m))) m = bm;
            }
            ExactOut o;
            o.mid = m.m == 0.0 ? xsZero() : XS{__double2float_rn(m.m), m.e};
            o.filt = f.m == 0.0 ? xsZero() : XS{__double2float_rn(f.m), f.e};
            o.failed = abortFlag != 0;
            out[pi] = o;
        }
    }
}

}  // namespace dmst
