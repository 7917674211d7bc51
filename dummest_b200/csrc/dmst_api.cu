// C ABI of the B200 search path (include/dummest_b200.h): context, device
// memory, profile and sequence upload, pair scheduling and kernel launches.
#include "dummest_b200.h"

#include "dp_common.cuh"
#include "dp_exact.cuh"
#include "dp_adjoint.cuh"
#include "dp_posterior.cuh"
#include "dp_plain.cuh"
#include "dp_exact_wave.cuh"
#include "dp_search.cuh"
#include "dp_stagger.cuh"
#include "dp_traceback.cuh"
#include "dp_wavefront.cuh"
#include "host_model.h"
#include "null_model.cuh"

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstdarg>
#include <cstddef>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <new>
#include <numeric>
#include <string>
#include <thread>
#include <vector>

using namespace dmst;

namespace {

__constant__ uint8_t cCodonTable[64];

// ---------------------------------------------------------------------------
// Device decode: DNA -> codon codes (decodeSequence, dummest-sequence.hh:181-204)
// One CTA per sequence.  Bases are 0..3 (ACGT) or 4 (anything else / masked).
// ---------------------------------------------------------------------------
__device__ __forceinline__ int asciiBase(unsigned char ch) {
    switch (ch | 0x20) {
    case 'a': return 0;
    case 'c': return 1;
    case 'g': return 2;
    case 't': return 3;
    default: return 4;
    }
}

__global__ void decodeAsciiKernel(const char *ascii, const long long *inOff, const long long *outOff, const int *lens,
                                  uint8_t *codes) {
    const int s = blockIdx.x;
    const int L = lens[s];
    const char *in = ascii + inOff[s];
    uint8_t *out = codes + outOff[s];
    for (int i = threadIdx.x; i < L; i += blockDim.x) {
        uint8_t c = 0;
        if (i + 2 < L) {
            int b0 = asciiBase(in[i]), b1 = asciiBase(in[i + 1]), b2 = asciiBase(in[i + 2]);
            c = (b0 > 3 || b1 > 3 || b2 > 3) ? (uint8_t)kMaskCode : cCodonTable[16 * b0 + 4 * b1 + b2];
        }
        out[i] = c;
    }
}

// 2-bit packed input: 16 bases per 32-bit word, optional masked-base bitmap.
__global__ void decodePackedKernel(const uint32_t *words, const uint32_t *mask, const long long *wordOff,
                                   const long long *maskOff, const long long *outOff, const int *lens,
                                   uint8_t *codes) {
    const int s = blockIdx.x;
    const int L = lens[s];
    const uint32_t *w = words + wordOff[s];
    const uint32_t *mk = mask ? mask + maskOff[s] : nullptr;
    uint8_t *out = codes + outOff[s];
    for (int i = threadIdx.x; i < L; i += blockDim.x) {
        uint8_t c = 0;
        if (i + 2 < L) {
            int b[3];
            bool masked = false;
#pragma unroll
            for (int t = 0; t < 3; ++t) {
                const int k = i + t;
                b[t] = (int)((__ldg(w + (k >> 4)) >> (2 * (k & 15))) & 3u);
                if (mk && ((__ldg(mk + (k >> 5)) >> (k & 31)) & 1u)) masked = true;
            }
            c = masked ? (uint8_t)kMaskCode : cCodonTable[16 * b[0] + 4 * b[1] + b[2]];
        }
        out[i] = c;
    }
}

// One contig of a window of the resident genome: the record's packed words
// and mask words, the contig's first position in the record and its length;
// rev: the sequence is the reverse complement (its base k is the complement of
// the record's base pos + len - 1 - k).
struct WinSeg {
    long long wordOff, maskOff, outOff;
    int pos, len, rev;
    int chunk;  // its first 16-code chunk: the call's sequences are consecutive whole chunks
};

// Words of padding before the first and after the last record of the resident
// genome: a window's lanes read up to two words before and after its contig.
constexpr long long kGenomePad = 2;

// Windows of the resident genome -> codon codes, as decodePackedKernel decodes
// the same letters uploaded packed (the last two codes 0).  The call's
// sequences lie back to back in whole 16-byte chunks (starts 16-byte aligned,
// lengths reserved in 16-byte units), and each thread makes one chunk: 16
// codes from the 18 bases they need (three 2-bit words and two mask words,
// funnel-shifted into place), written with one 16-byte store, so every thread
// has the same work whatever the contigs' lengths.  A block finds its threads'
// contigs from the first contig of its first chunk (blockSeg, from the host).
// The codon table sits in shared memory: the lanes' lookups differ, which a
// constant-memory table would serialise.
constexpr int kWinThreads = 256;
__global__ void __launch_bounds__(kWinThreads)
windowDecodeKernel(const uint32_t *words, const uint32_t *mask, const WinSeg *segs, const int *blockSeg, int nseg,
                   long long nChunks, uint8_t *codes) {
    // table[64 rev + y]: the code of the triplet whose three bases, in record
    // order, are the 2-bit fields of y (lowest first): forward the codon
    // (b0, b1, b2) = (y & 3, y >> 2 & 3, y >> 4); reverse-complemented the
    // codon (3 - b2, 3 - b1, 3 - b0), whose codon-table index is 63 - y.
    // nib[n]: 0xFF in the bytes whose bit of n is set.
    __shared__ uint8_t table[128];
    __shared__ uint32_t nib[16];
    if (threadIdx.x < 64) {
        const int y = threadIdx.x;
        table[y] = cCodonTable[16 * (y & 3) + 4 * ((y >> 2) & 3) + (y >> 4)];
        table[64 + y] = cCodonTable[63 - y];
    } else if (threadIdx.x < 80) {
        const int n = threadIdx.x - 64;
        nib[n] = (n & 1 ? 0xFFu : 0u) | (n & 2 ? 0xFF00u : 0u) | (n & 4 ? 0xFF0000u : 0u) | (n & 8 ? 0xFF000000u : 0u);
    }
    __syncthreads();
    const long long g = (long long)blockIdx.x * kWinThreads + threadIdx.x;
    if (g >= nChunks) return;
    int s = blockSeg[blockIdx.x];
    while (s + 1 < nseg && segs[s + 1].chunk <= g) ++s;
    const WinSeg sg = segs[s];
    const uint32_t *w = words + sg.wordOff;
    const uint32_t *mk = mask + sg.maskOff;
    const int q0 = 16 * (int)(g - sg.chunk);
    // the sequence's bases q0 .. q0 + 17 are the record's g0 .. g0 + 17
    // (reversed and complemented for rev); g0 >= pos - 17 and the words read
    // end at most two past the record's last
    const int g0 = sg.rev ? sg.pos + sg.len - 18 - q0 : sg.pos + q0;
    const int wi = g0 >> 4, o = g0 & 15, mi = g0 >> 5, mo = g0 & 31;
    const uint32_t w0 = __ldg(w + wi), w1 = __ldg(w + wi + 1), w2 = __ldg(w + wi + 2);
    const uint32_t lo = __funnelshift_r(w0, w1, 2 * o);  // bases g0 .. g0 + 15
    const uint32_t hi = __funnelshift_r(w1, w2, 2 * o);  // bases g0 + 16 .. g0 + 31
    const uint32_t m = __funnelshift_r(__ldg(mk + mi), __ldg(mk + mi + 1), mo);  // mask bits g0 .. g0 + 31
    // the triplets at record positions g0 + j, j = 0 .. 15: forward the
    // sequence's codes in order, reverse-complemented in reverse order
    const uint32_t base = sg.rev ? 64u : 0u;
    const uint32_t mm = m | (m >> 1) | (m >> 2);  // bit j: a base of triplet j is not A, C, G or T
    uint32_t ow[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        uint32_t v = 0;
#pragma unroll
        for (int r = 0; r < 4; ++r) {
            const int j = 4 * q + r;
            v |= (uint32_t)table[(__funnelshift_r(lo, hi, 2 * j) & 63u) | base] << (8 * r);
        }
        const uint32_t mb = nib[(mm >> (4 * q)) & 15u];
        ow[q] = (v & ~mb) | ((uint32_t)kMaskCode * 0x01010101u & mb);
    }
    if (sg.rev) {  // bytes in sequence order
        const uint32_t t0 = __byte_perm(ow[3], 0, 0x0123), t1 = __byte_perm(ow[2], 0, 0x0123);
        ow[2] = __byte_perm(ow[1], 0, 0x0123);
        ow[3] = __byte_perm(ow[0], 0, 0x0123);
        ow[0] = t0;
        ow[1] = t1;
    }
    const int valid = sg.len - 2 - q0;  // codes k < valid are codons, the rest 0
    if (valid < 16) {
#pragma unroll
        for (int k = 0; k < 16; ++k)
            if (k >= valid) ow[k >> 2] &= ~(0xFFu << (8 * (k & 3)));
    }
    *reinterpret_cast<uint4 *>(codes + sg.outOff + q0) = make_uint4(ow[0], ow[1], ow[2], ow[3]);
}

// ---------------------------------------------------------------------------
// Buffers replaced while calls may be in flight.  cudaFree and cudaFreeHost
// synchronise the whole device, so freeing a buffer that a call outgrew would
// make the host wait for every queued call (with calls submitted one ahead of
// their completion, a whole call's device time).  The old buffer is kept here
// instead and freed when its context has no call in flight (drainCalls,
// dmst_ctx_destroy), or at once when the kept bytes pass graveLimit(): 40% of
// the device's memory, at least 16 GB.  The W1 slots of the default batch
// take 20-30 GB, so a lower limit made every growth of them (a call whose
// longest pairs need longer slots) wait for the call in flight and leave the
// device idle while the host finished preparing.  An allocation that fails
// for want of memory frees the kept buffers and tries again (devAlloc).
// ---------------------------------------------------------------------------
struct Grave {
    void *p;
    bool host;
    int device;
    size_t bytes;
};
std::mutex gGraveMutex;
std::vector<Grave> gGraves;
size_t gGraveBytes = 0;
size_t graveLimit() {
    static const size_t limit = [] {
        size_t v = (size_t)16 << 30, freeB = 0, totalB = 0;
        if (cudaMemGetInfo(&freeB, &totalB) == cudaSuccess)
            v = std::max(v, (size_t)(0.4 * (double)totalB));
        else
            cudaGetLastError();
        return v;
    }();
    return limit;
}

void reapGraves() {
    std::vector<Grave> g;
    {
        std::lock_guard<std::mutex> lock(gGraveMutex);
        g.swap(gGraves);
        gGraveBytes = 0;
    }
    if (g.empty()) return;
    int cur = -1;
    cudaGetDevice(&cur);
    for (const Grave &x : g) {
        if (x.host) {
            cudaFreeHost(x.p);
        } else {
            cudaSetDevice(x.device);
            cudaFree(x.p);
        }
    }
    if (cur >= 0) cudaSetDevice(cur);
}

void bury(void *p, bool host, size_t bytes) {
    int dev = 0;
    cudaGetDevice(&dev);
    const size_t limit = graveLimit();
    bool full;
    {
        std::lock_guard<std::mutex> lock(gGraveMutex);
        gGraves.push_back(Grave{p, host, dev, bytes});
        gGraveBytes += bytes;
        full = gGraveBytes > limit;
    }
    if (full) reapGraves();  // frees synchronise the device, as before the graveyard
}

// cudaMalloc / cudaMallocHost that, when the device (or host) is out of
// memory, frees the graveyard (synchronising the device) and tries once more:
// kept buffers never make an allocation fail that would fit without them.
cudaError_t devAlloc(void **p, size_t bytes) {
    cudaError_t e = cudaMalloc(p, bytes);
    if (e == cudaErrorMemoryAllocation) {
        bool kept;
        {
            std::lock_guard<std::mutex> lock(gGraveMutex);
            kept = !gGraves.empty();
        }
        if (kept) {
            cudaGetLastError();
            reapGraves();
            e = cudaMalloc(p, bytes);
        }
    }
    return e;
}

cudaError_t hostAlloc(void **p, size_t bytes) {
    cudaError_t e = cudaMallocHost(p, bytes);
    if (e == cudaErrorMemoryAllocation) {
        bool kept;
        {
            std::lock_guard<std::mutex> lock(gGraveMutex);
            kept = !gGraves.empty();
        }
        if (kept) {
            cudaGetLastError();
            reapGraves();
            e = cudaMallocHost(p, bytes);
        }
    }
    return e;
}

// ---------------------------------------------------------------------------
// Small device buffer helper
// ---------------------------------------------------------------------------
template <typename T>
struct DevBuf {
    T *p = nullptr;
    size_t cap = 0;  // elements
    // Capacity for n elements, contents not kept.  Growth is geometric (x1.25,
    // or n x (1 + headroom) for buffers whose need varies from call to call)
    // so that calls whose sizes vary a little do not reallocate; the old
    // buffer, which a call in flight may still read, goes to the graveyard.
    cudaError_t ensure(size_t n, double headroom = 0.0) {
        if (n <= cap && p) return cudaSuccess;
        const size_t want = std::max<size_t>({n, cap + cap / 4, (size_t)((double)n * (1.0 + headroom)), 1});
        if (p) bury(p, false, cap * sizeof(T));
        p = nullptr;
        cap = 0;
        cudaError_t e = devAlloc((void **)&p, want * sizeof(T));
        if (e != cudaSuccess && want > n) {  // the headroom did not fit: the exact size
            cudaGetLastError();
            e = devAlloc((void **)&p, std::max<size_t>(n, 1) * sizeof(T));
            if (e == cudaSuccess) cap = std::max<size_t>(n, 1);
            return e;
        }
        if (e == cudaSuccess) cap = want;
        return e;
    }
    // Grow keeping the first `keep` elements.
    cudaError_t grow(size_t n, size_t keep, cudaStream_t st) {
        if (n <= cap && p) return cudaSuccess;
        size_t want = std::max(n, cap * 2);
        T *q = nullptr;
        cudaError_t e = devAlloc((void **)&q, want * sizeof(T));
        if (e != cudaSuccess) return e;
        if (p && keep) {
            e = cudaMemcpyAsync(q, p, keep * sizeof(T), cudaMemcpyDeviceToDevice, st);
            if (e != cudaSuccess) {
                cudaFree(q);
                return e;
            }
        }
        if (p) bury(p, false, cap * sizeof(T));  // the copy, and calls in flight, still read it
        p = q;
        cap = want;
        return cudaSuccess;
    }
    void release() {
        if (p) cudaFree(p);
        p = nullptr;
        cap = 0;
    }
};

// Page-locked host staging (uploads and downloads that run asynchronously).
template <class T>
struct PinnedBuf {
    T *p = nullptr;
    size_t cap = 0;
    cudaError_t ensure(size_t n) {
        if (n <= cap && p) return cudaSuccess;
        const size_t want = std::max<size_t>({n, cap + cap / 2, 64});
        if (p) bury(p, true, cap * sizeof(T));  // an async copy in flight may still use it
        p = nullptr;
        cap = 0;
        cudaError_t e = hostAlloc((void **)&p, want * sizeof(T));
        if (e == cudaSuccess) cap = want;
        return e;
    }
    void release() {
        if (p) cudaFreeHost(p);
        p = nullptr;
        cap = 0;
    }
};

struct HostProfile {
    int M;
    int rowPad;
    std::vector<float> emit;    // [25][rowPad]
    std::vector<float> params;  // (M+2) x 11
    float bg[26];
    std::vector<float> values;  // (M+1) x 29 (kept for calibration letter freqs)
};

const char *statusText(int s) {
    switch (s) {
    case DMST_OK: return "ok";
    case DMST_EINVAL: return "invalid argument";
    case DMST_ENOMEM: return "out of memory";
    case DMST_EDEVICE: return "CUDA device error";
    case DMST_ETIMEOUT: return "kernel iteration budget exceeded";
    case DMST_EPARSE: return "parse error";
    case DMST_ERANGE: return "size beyond a documented limit";
    default: return "unknown status";
    }
}

// Kernel shapes the autotuner chooses among: rows per lane (the stripe is
// 32 R rows) and warps per CTA.
constexpr int kNumR = 4;
constexpr int kShapeR[kNumR] = {4, 3, 2, 1};
constexpr int kShapeWarps[3] = {kCtaWarps, kCtaWarpsNarrow, kCtaWarpsMid};
inline int rIndex(int R) { return R == 4 ? 0 : (R == 3 ? 1 : (R == 2 ? 2 : 3)); }

using DpKern = void (*)(DpArgs, int);
template <bool MID, int W, bool GT>
DpKern kernByR(int R) {
    return R == 4 ? dpKernel<4, MID, W, GT>
                  : (R == 3 ? dpKernel<3, MID, W, GT> : (R == 2 ? dpKernel<2, MID, W, GT> : dpKernel<1, MID, W, GT>));
}
template <bool GT>
DpKern dpKernelShape(int R, bool mid, int warps) {
    if (warps == kCtaWarpsNarrow)
        return mid ? kernByR<true, kCtaWarpsNarrow, GT>(R) : kernByR<false, kCtaWarpsNarrow, GT>(R);
    if (warps == kCtaWarpsMid)
        return mid ? kernByR<true, kCtaWarpsMid, GT>(R) : kernByR<false, kCtaWarpsMid, GT>(R);
    return mid ? kernByR<true, kCtaWarps, GT>(R) : kernByR<false, kCtaWarps, GT>(R);
}
// gt: the emission table stays in global memory (profiles whose table would
// leave shared memory for fewer than `warps` staging windows).
DpKern dpKernelFor(int R, bool mid, int warps, bool gt) {
    return gt ? dpKernelShape<true>(R, mid, warps) : dpKernelShape<false>(R, mid, warps);
}

using PlainKern = void (*)(const DevPair *, int, const DevProfile *, const float *, const float *, const uint8_t *,
                          const float *, const PairScales *, float *, PairOut *, int);
template <bool MID>
PlainKern plainKernelByR(int R) {
    return R == 4 ? plainKernel<4, MID> : (R == 2 ? plainKernel<2, MID> : plainKernel<1, MID>);
}
// The plain schedule's kernel for R rows per lane; its dynamic shared memory
// (a window per warp) is allowed once.
PlainKern plainKernelFor(int R, bool mid) {
    static bool attrSet = false;
    if (!attrSet) {
        for (int r : {4, 2, 1})
            for (bool m : {true, false})
                cudaFuncSetAttribute(m ? plainKernelByR<true>(r) : plainKernelByR<false>(r),
                                     cudaFuncAttributeMaxDynamicSharedMemorySize, (int)(kPlainWarps * sizeof(Window)));
        attrSet = true;
    }
    return mid ? plainKernelByR<true>(R) : plainKernelByR<false>(R);
}

// Rows of a profile as the kernel with R rows per lane computes them.
inline long long paddedRows(int M, int R) {
    const long long S = (long long)kLanes * R;
    return (M + 1 + S - 1) / S * S;
}

// Kernel shapes: (R, W) pairs, index rIndex(R) * 3 + wIndex(W).
constexpr int kNumShapes = kNumR * 3;
inline int wIndex(int W) { return W == kShapeWarps[0] ? 0 : (W == kShapeWarps[1] ? 1 : 2); }
// Reads shorter than this form the short length class: the autotuner times
// every shape on each class of its sample, and a pair takes the shape with
// the least expected time for its class (16-warp CTAs of three rows per lane
// are fastest on short reads, 8- or 12-warp CTAs of four rows on long ones).
constexpr int kShortRead = 700;
inline int lengthClass(int L) { return L < kShortRead ? 1 : 0; }

// What the autotuner measured: per length class (0: long, 1: short) and
// rows-per-lane value, the faster CTA shape and its rate in computed (padded)
// cells per millisecond.
struct Tuning {
    bool tuned = false;
    int warps[2][kNumR] = {{kCtaWarps, kCtaWarps, kCtaWarps, kCtaWarps}, {kCtaWarps, kCtaWarps, kCtaWarps, kCtaWarps}};
    double rate[2][kNumR] = {};
    double rates[2][kNumR][3] = {};  // per class, R, kShapeWarps: the measured rates (cells per ms)
    int forceR = 0, forceWarps = 0;  // set while the autotuner measures one shape
};

// The kernel shape of a pair of a profile of length M and a read of length L.
void shapeOf(int M, int L, int forced, const Tuning &t, int &R, int &W) {
    const int c = lengthClass(L);
    if (forced >= 1 && forced <= 4) {
        R = forced;
    } else if (t.forceR) {
        R = t.forceR;
    } else if (!t.tuned) {
        // Untuned default: four rows per lane.
        R = 4;
    } else {
        // Tuned: the R with the least expected time (computed rows / rate).
        R = 4;
        double bestT = 1e300;
        for (int q = 0; q < kNumR; ++q) {
            if (!(t.rate[c][q] > 0)) continue;
            const double time = (double)paddedRows(M, kShapeR[q]) / t.rate[c][q];
            if (time < bestT) {
                bestT = time;
                R = kShapeR[q];
            }
        }
    }
    W = t.forceWarps ? t.forceWarps : t.warps[c][rIndex(R)];
}

}  // namespace

// The per-call state of a scoring call in flight.  A context has two, so
// that one call's host work overlaps the other's device work: the buffers the
// call reads after its DP kernels (pairs, seeds, scales, for the exact path)
// and its page-locked staging are per slot; buffers used only by the call's
// own stream-ordered kernels are shared.
struct CallSlot {
    DevBuf<DevPair> dPairs;
    DevBuf<float> dSeeds;
    DevBuf<PairScales> dScales;
    DevBuf<PairOut> dOut;
    DevBuf<ExactOut> dExOut;  // exact-path results, by pair position
    DevBuf<int> dQueue;       // exact-path queue, by queue position
    DevBuf<int> dQueueCount;  // [0] queued pairs, [1] next queue position
    DevBuf<PairOut> dOutF;    // search: the filter wave's results
    DevBuf<uint8_t> dMask;    // search: survivors
    PinnedBuf<PairOut> hOutF;
    PinnedBuf<uint8_t> hMask;
    PinnedBuf<float> hMinBest;
    DevBuf<long long> dAnchorOff;  // anchors: per pair position, the offset of its columns
    DevBuf<float> dAnchorM;
    DevBuf<int> dAnchorE, dAnchorRow;
    PinnedBuf<long long> hAnchorOff;
    PinnedBuf<float> hAnchorM;
    PinnedBuf<int> hAnchorE, hAnchorRow;
    PinnedBuf<DevPair> hPairs;
    PinnedBuf<Chunk> hChunks;
    PinnedBuf<NullJob> hNullJobs;
    PinnedBuf<int> hJobPairs;
    PinnedBuf<long long> hNullTmpOff;
    PinnedBuf<PairOut> hOut;
    PinnedBuf<ExactOut> hExOut;
    cudaEvent_t ev[5] = {};  // null start, DP start, DP end, exact end, results copied
    cudaEvent_t evFork = nullptr;  // the flag kernel done: the exact path may start
    cudaGraphExec_t graphExec = nullptr;
    std::vector<uintptr_t> graphKey;
    int graphLaunches = 0;
    // the pending call
    bool pending = false;
    size_t n = 0;
    int mode = 0;
    bool mid = false, nullOnly = false, sequentialExact = false, exactOnDevice = false, search = false;
    dmst_score *anchorBest = nullptr;  // anchors: the caller's outputs (columns in the caller's pair order)
    int *anchorRowOut = nullptr;
    long long anchorCols = 0;
    dmst_result *out = nullptr;
    std::vector<int> order;
    std::vector<DevPair> dp;
    int launches = 0;
    double hostMs = 0;
    std::chrono::steady_clock::time_point t0;
};

struct dmst_ctx {
    dmst_opts opts;
    Rates rates;
    Tuning tune;
    cudaGraphExec_t graphExec = nullptr;  // DMST_MODE_GRAPH: the instantiated launch graph
    bool exactAttrSet = false;            // the exact kernel's shared-memory attribute is set
    std::vector<uintptr_t> graphKey;      // the launch shape and buffers it was captured with
    int graphLaunches = 0;                // kernel launches in it
    int graphCaptures = 0;                // captures so far (replays reuse the last)
    int device = 0;
    int smCount = 0;
    int maxSmemOptin = 0;
    int nullBlocksPerSm = 0;  // resident null-model blocks per SM (queried on first use)
    cudaStream_t stream = nullptr;
    cudaStream_t stream2 = nullptr;  // the exact path and result copies of scoring calls
    PinnedBuf<char> hSeqStage[2];    // dmst_seqs_add_packed: host staging blocks, in turn
    cudaEvent_t evSeqStage[2] = {};  // ... each block's copy done
    int seqStageNext = 0;
    cudaEvent_t ev[6] = {};
    std::string err;

    std::vector<HostProfile> profiles;
    bool profilesDirty = false;
    DevBuf<float> dEmit, dParams;
    DevBuf<DevProfile> dProfiles;
    int maxRowPad = 0;

    std::vector<long long> seqOff;  // code offsets (device buffer)
    std::vector<int> seqLen;
    long long codeBytes = 0;
    DevBuf<uint8_t> dCodes;
    DevBuf<char> dStage;
    DevBuf<long long> dStageOff;
    DevBuf<int> dStageLen;

    // the genome of dmst_genome_load: per record its name in the text, its
    // length, its packed words and mask words (offsets in buffers that hold
    // kGenomePad words before the first record and after the last), and its
    // contigs (start, length)
    struct GenomeRecord {
        size_t nameOff;
        int nameLen;
        int length;
        long long wordOff, maskOff;
        std::vector<std::pair<int, int>> contigs;
    };
    std::vector<GenomeRecord> genome;
    DevBuf<uint32_t> dGenomeWords, dGenomeMask;
    DevBuf<WinSeg> dWinSegs;
    cudaEvent_t evWin[2] = {};  // around the last window decode kernel
    bool winTimed = false;

    // per call (shared by the slots: used only by a call's stream-ordered kernels)
    DevBuf<XS> dNullTmp;
    DevBuf<NullJob> dNullJobs;
    DevBuf<int> dNullJobPairs;
    DevBuf<long long> dNullTmpOff;
    DevBuf<Chunk> dChunks;
    DevBuf<int> dCounter;
    DevBuf<float> dW1, dRing;
    DevBuf<ExactJob> dJobs;
    DevBuf<AdjointJob> dAdjJobs;             // dmst_loglik_grad, dmst_posteriors
    int adjCheckpoint = DMST_ADJ_CKPT_AUTO;   // dmst_adjoint_checkpoint
    bool lastAdjCheckpointed = false;
    DevBuf<double> dPost;                    // dmst_posteriors: the batch's posterior tables
    DevBuf<PostSumJob> dPostJobs;            // dmst_posterior_summary: the batch's reductions
    DevBuf<double> dColPost, dRowMatch;      // dmst_posterior_summary outputs (the call's pairs)
    DevBuf<int> dColRow;
    DevBuf<double> dAdjF, dAdjB, dGrad, dLogT;
    std::vector<int> lastOrder;              // sorted position -> caller's pair index of the last call
    CallSlot slot[2];
    int nextSlot = 0;                        // the slot the next submit uses
    int oldest = 0;                          // the oldest pending call's slot
    int lastSlot = 0;                        // the slot of the last completed call
    DevBuf<float> dExactPool;                // exact-path scratch: one slot per CTA
    DevBuf<Chunk> dMidChunks;                // search: the survivors' chunks
    DevBuf<int> dSurvivors;                  // search: survivor pair indices by chunk
    DevBuf<float> dMinBest;                  // search: per-profile filter gate
    DevBuf<float> dExactScratch;
    DevBuf<ExactOut> dExactOut;
    // dmst_align: the traceback buffers (dp_traceback.cuh) and the last call's results
    DevBuf<AlignJob> dAlignJobs;
    DevBuf<int> dAlignJobOf, dAlignRows, dAlignCand;
    DevBuf<float> dAlignCells, dAlignColR, dAlignColF;
    DevBuf<XS> dAlignX, dAlignSuf, dAlignWork, dAlignRev, dAlignFwd;
    DevBuf<WalkSpan> dAlignSpan;
    DevBuf<WalkItem> dAlignItems;
    DevBuf<Seg> dAlignSegOut;
    std::vector<dmst_alignment> alignOut;
    std::vector<dmst_segment> alignSegOut;
    double alignMs[9] = {};  // dmst_last_align_timing

    double lastTotalMs = 0, lastDpMs = 0, lastNullMs = 0, lastExactMs = 0, lastHostMs = 0;
    double lastPostMs = 0, lastWallMs = 0;
    int lastExactPairs = 0;
    int lastLaunches = 0;
    int lastFlagged = 0;  // pairs the last completed mid-score call sent to the exact path
    int waitLimit = 0;    // exact path: iterations of a stripe wait before it gives up (0: the default)

    int fail(int status, const char *fmt, ...) {
        char buf[512];
        va_list ap;
        va_start(ap, fmt);
        vsnprintf(buf, sizeof buf, fmt, ap);
        va_end(ap);
        err = buf;
        return status;
    }
    int cudaFail(cudaError_t e, const char *what) {
        if (e == cudaErrorMemoryAllocation) {
            cudaGetLastError();
            return fail(DMST_ENOMEM, "%s: %s", what, cudaGetErrorString(e));
        }
        return fail(DMST_EDEVICE, "%s: %s", what, cudaGetErrorString(e));
    }
};

#define CK(call, what)                                  \
    do {                                                \
        cudaError_t e_ = (call);                        \
        if (e_ != cudaSuccess) return ctx->cudaFail(e_, what); \
    } while (0)

extern "C" {

static int drainCalls(dmst_ctx *ctx);

void dmst_opts_default(dmst_opts *o) {
    if (!o) return;
    o->insert1 = 0.0171;  // OPT_insert1 (dummest-core.hh:66-71)
    o->insert2 = 0.0018;
    o->delete1 = 0.0328;
    o->delete2 = 0.0083;
    o->stop_codon_prob = 0.0005;
    o->bg_stop_codon_prob = 0.046875;
    o->device = 0;
    o->rows_per_lane = 0;
    o->device_budget_bytes = 0;
    o->tantan_threshold = 0.5;
}

const char *dmst_strerror(int status) { return statusText(status); }

const char *dmst_last_error(const dmst_ctx *ctx) { return ctx ? ctx->err.c_str() : ""; }

void *dmst_ctx_stream(const dmst_ctx *ctx) { return ctx ? (void *)ctx->stream : nullptr; }

int dmst_ctx_create(const dmst_opts *opts, dmst_ctx **out) {
    if (!out) return DMST_EINVAL;
    *out = nullptr;
    dmst_opts o;
    dmst_opts_default(&o);
    if (opts) o = *opts;
    if (!(o.insert1 >= 0 && o.insert1 < 1 && o.insert2 >= 0 && o.insert2 < 1 && o.delete1 >= 0 && o.delete1 < 1 &&
          o.delete2 >= 0 && o.delete2 < 1 && o.insert1 + o.insert2 + o.delete1 + o.delete2 < 1 &&
          o.stop_codon_prob >= 0 && o.stop_codon_prob < 1 && o.bg_stop_codon_prob >= 0 &&
          o.bg_stop_codon_prob < 1))
        return DMST_EINVAL;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev <= o.device || o.device < 0) {
        cudaGetLastError();
        return DMST_EDEVICE;
    }
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, o.device) != cudaSuccess) return DMST_EDEVICE;
    if (prop.major < 10) return DMST_EDEVICE;  // built for sm_100a only
    dmst_ctx *ctx = new (std::nothrow) dmst_ctx();
    if (!ctx) return DMST_ENOMEM;
    ctx->opts = o;
    ctx->rates.insert1 = (float)o.insert1;
    ctx->rates.insert2 = (float)o.insert2;
    ctx->rates.delete1 = (float)o.delete1;
    ctx->rates.delete2 = (float)o.delete2;
    ctx->rates.stop = (float)o.stop_codon_prob;
    ctx->rates.bgStop = (float)o.bg_stop_codon_prob;
    ctx->device = o.device;
    ctx->smCount = prop.multiProcessorCount;
    ctx->maxSmemOptin = (int)prop.sharedMemPerBlockOptin;
    if (cudaSetDevice(o.device) != cudaSuccess || cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaStreamCreateWithFlags(&ctx->stream2, cudaStreamNonBlocking) != cudaSuccess) {
        delete ctx;
        return DMST_EDEVICE;
    }
    for (auto &e : ctx->ev) cudaEventCreate(&e);
    for (auto &e : ctx->evSeqStage) cudaEventCreateWithFlags(&e, cudaEventDisableTiming);
    for (auto &sl : ctx->slot) {
        for (auto &e : sl.ev) cudaEventCreate(&e);
        cudaEventCreateWithFlags(&sl.evFork, cudaEventDisableTiming);
    }
    uint8_t table[64];
    standardCodeTable(table);
    if (cudaMemcpyToSymbol(cCodonTable, table, 64) != cudaSuccess) {
        delete ctx;
        return DMST_EDEVICE;
    }
    *out = ctx;
    return DMST_OK;
}

void dmst_ctx_destroy(dmst_ctx *ctx) {
    if (!ctx) return;
    cudaSetDevice(ctx->device);
    cudaStreamSynchronize(ctx->stream);
    if (ctx->stream2) cudaStreamSynchronize(ctx->stream2);
    reapGraves();
    if (ctx->graphExec) cudaGraphExecDestroy(ctx->graphExec);
    for (auto &sl : ctx->slot) {
        if (sl.graphExec) cudaGraphExecDestroy(sl.graphExec);
        sl.dPairs.release();
        sl.dSeeds.release();
        sl.dScales.release();
        sl.dOut.release();
        sl.dExOut.release();
        sl.dQueue.release();
        sl.dQueueCount.release();
        sl.hPairs.release();
        sl.hChunks.release();
        sl.hNullJobs.release();
        sl.hJobPairs.release();
        sl.hNullTmpOff.release();
        sl.hOut.release();
        sl.hExOut.release();
        sl.dOutF.release();
        sl.dMask.release();
        sl.hOutF.release();
        sl.hMask.release();
        sl.hMinBest.release();
        sl.dAnchorOff.release();
        sl.dAnchorM.release();
        sl.dAnchorE.release();
        sl.dAnchorRow.release();
        sl.hAnchorOff.release();
        sl.hAnchorM.release();
        sl.hAnchorE.release();
        sl.hAnchorRow.release();
        for (auto &e : sl.ev)
            if (e) cudaEventDestroy(e);
        if (sl.evFork) cudaEventDestroy(sl.evFork);
    }
    ctx->dExactPool.release();
    for (auto &hb : ctx->hSeqStage) hb.release();
    for (auto &e : ctx->evSeqStage)
        if (e) cudaEventDestroy(e);
    ctx->dAlignJobs.release();
    ctx->dAlignJobOf.release();
    ctx->dAlignRows.release();
    ctx->dAlignCand.release();
    ctx->dAlignCells.release();
    ctx->dAlignColR.release();
    ctx->dAlignColF.release();
    ctx->dAlignX.release();
    ctx->dAlignSuf.release();
    ctx->dAlignWork.release();
    ctx->dAlignRev.release();
    ctx->dAlignFwd.release();
    ctx->dAlignSpan.release();
    ctx->dAlignItems.release();
    ctx->dAlignSegOut.release();
    ctx->dMidChunks.release();
    ctx->dSurvivors.release();
    ctx->dMinBest.release();
    ctx->dEmit.release();
    ctx->dParams.release();
    ctx->dProfiles.release();
    ctx->dCodes.release();
    ctx->dStage.release();
    ctx->dStageOff.release();
    ctx->dStageLen.release();
    ctx->dNullTmp.release();
    ctx->dNullJobs.release();
    ctx->dNullJobPairs.release();
    ctx->dNullTmpOff.release();
    ctx->dChunks.release();
    ctx->dCounter.release();
    ctx->dW1.release();
    ctx->dRing.release();
    ctx->dJobs.release();
    ctx->dAdjJobs.release();
    ctx->dAdjF.release();
    ctx->dAdjB.release();
    ctx->dGrad.release();
    ctx->dLogT.release();
    ctx->dPost.release();
    ctx->dPostJobs.release();
    ctx->dColPost.release();
    ctx->dColRow.release();
    ctx->dRowMatch.release();
    ctx->dExactScratch.release();
    ctx->dExactOut.release();
    ctx->dGenomeWords.release();
    ctx->dGenomeMask.release();
    ctx->dWinSegs.release();
    for (auto &e : ctx->evWin)
        if (e) cudaEventDestroy(e);
    for (auto &e : ctx->ev)
        if (e) cudaEventDestroy(e);
    if (ctx->stream) cudaStreamDestroy(ctx->stream);
    if (ctx->stream2) cudaStreamDestroy(ctx->stream2);
    delete ctx;
}

// ---------------------------------------------------------------------------
// Profiles
// ---------------------------------------------------------------------------
static HostProfile makeHostProfile(const float *values, int width, int M, const dmst_params *params,
                                   const float *bg) {
    HostProfile hp;
    hp.M = M;
    hp.rowPad = rowPadOf(M);
    hp.emit.assign((size_t)kNumCodes * hp.rowPad, 0.0f);
    for (int i = 0; i <= M; ++i)
        for (int c = 0; c < kNumCodes; ++c) hp.emit[(size_t)c * hp.rowPad + i] = values[(size_t)i * width + 4 + c];
    hp.params.resize((size_t)(M + 2) * kParamFloats);
    std::memcpy(hp.params.data(), params, hp.params.size() * sizeof(float));
    for (int c = 0; c < 26; ++c) hp.bg[c] = (c < kNumCodes) ? bg[4 + c] : 0.0f;
    hp.bg[kPad] = 0.0f;  // zero_idx pad reads as 0
    hp.values.assign(values, values + (size_t)(M + 1) * width);
    return hp;
}

int dmst_profile_add(dmst_ctx *ctx, const float *values, int width, int M, const dmst_params *params,
                     const float *bg, int *id) {
    if (!ctx || !values || !params || !bg || width != kWidth || M < 2) return DMST_EINVAL;
    ctx->profiles.push_back(makeHostProfile(values, width, M, params, bg));
    ctx->profilesDirty = true;
    if (id) *id = (int)ctx->profiles.size() - 1;
    return DMST_OK;
}

int dmst_profile_set(dmst_ctx *ctx, int id, const float *values, int width, int M, const dmst_params *params,
                     const float *bg) {
    if (!ctx || !values || !params || !bg || width != kWidth || M < 2 || id < 0 ||
        id >= (int)ctx->profiles.size())
        return DMST_EINVAL;
    ctx->profiles[id] = makeHostProfile(values, width, M, params, bg);
    ctx->profilesDirty = true;
    return DMST_OK;
}

int dmst_hmm_finalize(const char *text, size_t len, int index, int background_type, const dmst_opts *opts, int *M,
                      float *values, dmst_params *params, float *bg, char *name, size_t name_cap) {
    if (!text || !M) return DMST_EINVAL;
    dmst_opts o;
    dmst_opts_default(&o);
    if (opts) o = *opts;
    std::vector<RawProfile> raws;
    if (parseHmmText(text, len, raws, nullptr) < 0) return DMST_EPARSE;
    if (index < 0 || index >= (int)raws.size()) return DMST_EINVAL;
    *M = raws[index].M;
    if (!values) return DMST_OK;
    Rates r{(float)o.insert1, (float)o.insert2, (float)o.delete1, (float)o.delete2, (float)o.stop_codon_prob,
            (float)o.bg_stop_codon_prob};
    FinalProfile f;
    const int type = background_type & 0xff;
    const double maskAt = (background_type & DMST_HMM_MASK) ? o.tantan_threshold : -1.0;
    if (finalizeProfile(raws[index], r, type ? type : 'G', f, nullptr, maskAt) < 0) return DMST_EPARSE;
    std::memcpy(values, f.values.data(), f.values.size() * sizeof(float));
    if (params) std::memcpy(params, f.params.data(), f.params.size() * sizeof(Params));
    if (bg) std::memcpy(bg, f.bg.data(), f.bg.size() * sizeof(float));
    if (name && name_cap) {
        std::snprintf(name, name_cap, "%s", f.name.c_str());
    }
    return DMST_OK;
}

int dmst_profile_load_hmm(dmst_ctx *ctx, const char *text, size_t len, int background_type, int *first_id,
                          int *count) {
    if (!ctx || !text) return DMST_EINVAL;
    std::vector<RawProfile> raws;
    std::string e;
    if (parseHmmText(text, len, raws, &e) < 0) return ctx->fail(DMST_EPARSE, "HMMER3: %s", e.c_str());
    int first = (int)ctx->profiles.size();
    const int type = background_type & 0xff;
    const double maskAt = (background_type & DMST_HMM_MASK) ? ctx->opts.tantan_threshold : -1.0;
    for (auto &raw : raws) {
        FinalProfile f;
        if (finalizeProfile(raw, ctx->rates, type ? type : 'G', f, &e, maskAt) < 0)
            return ctx->fail(DMST_EPARSE, "profile %s: %s", raw.name.c_str(), e.c_str());
        int st = dmst_profile_add(ctx, f.values.data(), f.width, f.M,
                                  reinterpret_cast<const dmst_params *>(f.params.data()), f.bg.data(), nullptr);
        if (st) return st;
    }
    if (first_id) *first_id = first;
    if (count) *count = (int)raws.size();
    return DMST_OK;
}

int dmst_profile_count(const dmst_ctx *ctx) { return ctx ? (int)ctx->profiles.size() : 0; }
int dmst_profile_length(const dmst_ctx *ctx, int id) {
    if (!ctx || id < 0 || id >= (int)ctx->profiles.size()) return DMST_EINVAL;
    return ctx->profiles[id].M;
}

static int uploadProfiles(dmst_ctx *ctx) {
    if (!ctx->profilesDirty) return DMST_OK;
    // Per profile: its (M+2) x 11 Params, then its DP coefficient planes
    // (coefOffOf).
    size_t nE = 0, nP = 0;
    for (auto &p : ctx->profiles) {
        nE += p.emit.size();
        nP = (size_t)coefOffOf((long long)nP, p.M) + (size_t)kCoefPlanes * p.rowPad;
    }
    std::vector<float> emit(nE), par(nP, 0.0f);
    std::vector<DevProfile> desc(ctx->profiles.size());
    size_t oE = 0, oP = 0;
    ctx->maxRowPad = 0;
    for (size_t i = 0; i < ctx->profiles.size(); ++i) {
        auto &p = ctx->profiles[i];
        std::copy(p.emit.begin(), p.emit.end(), emit.begin() + oE);
        std::copy(p.params.begin(), p.params.end(), par.begin() + oP);
        const size_t oC = (size_t)coefOffOf((long long)oP, p.M);
        for (int r = 0; r <= p.M; ++r) {
            for (int q = 0; q < kCoefPlanes - 1; ++q)
                par[oC + (size_t)q * p.rowPad + r] = p.params[(size_t)r * kParamFloats + kCoefParam[q]];
            par[oC + (size_t)kPRs * p.rowPad + r] = 1.0f;
        }
        DevProfile &d = desc[i];
        d.M = p.M;
        d.rowPad = p.rowPad;
        d.emitOff = (long long)oE;
        d.paramOff = (long long)oP;
        std::memcpy(d.bg, p.bg, sizeof d.bg);
        oE += p.emit.size();
        oP = oC + (size_t)kCoefPlanes * p.rowPad;
        ctx->maxRowPad = std::max(ctx->maxRowPad, p.rowPad);
    }
    CK(ctx->dEmit.ensure(nE), "alloc emission tables");
    CK(ctx->dParams.ensure(nP), "alloc params");
    CK(ctx->dProfiles.ensure(desc.size()), "alloc profiles");
    CK(cudaMemcpy(ctx->dEmit.p, emit.data(), nE * sizeof(float), cudaMemcpyHostToDevice), "upload emission");
    CK(cudaMemcpy(ctx->dParams.p, par.data(), nP * sizeof(float), cudaMemcpyHostToDevice), "upload params");
    CK(cudaMemcpy(ctx->dProfiles.p, desc.data(), desc.size() * sizeof(DevProfile), cudaMemcpyHostToDevice),
       "upload profiles");
    ctx->profilesDirty = false;
    return DMST_OK;
}

// ---------------------------------------------------------------------------
// Sequences
// ---------------------------------------------------------------------------
static int checkOffsets(const int64_t *offsets, int nseq) {
    if (!offsets || nseq < 0) return DMST_EINVAL;
    for (int i = 0; i < nseq; ++i) {
        int64_t L = offsets[i + 1] - offsets[i];
        if (L < 3 || L > (1 << 30)) return DMST_EINVAL;
    }
    return DMST_OK;
}

// Reserve device code space for nseq new sequences; fills the new offsets.
static int reserveSeqs(dmst_ctx *ctx, const int64_t *offsets, int nseq, std::vector<long long> &outOff,
                       std::vector<int> &lens) {
    long long total = 0;
    outOff.resize(nseq);
    lens.resize(nseq);
    for (int i = 0; i < nseq; ++i) {
        lens[i] = (int)(offsets[i + 1] - offsets[i]);
        outOff[i] = ctx->codeBytes + total;
        total += (lens[i] + 15) / 16 * 16;  // 16-byte aligned starts
    }
    CK(ctx->dCodes.grow((size_t)(ctx->codeBytes + total), (size_t)ctx->codeBytes, ctx->stream), "alloc codes");
    return DMST_OK;
}

static void commitSeqs(dmst_ctx *ctx, const std::vector<long long> &off, const std::vector<int> &lens, int *first) {
    if (first) *first = (int)ctx->seqLen.size();
    for (size_t i = 0; i < lens.size(); ++i) {
        ctx->seqOff.push_back(off[i]);
        ctx->seqLen.push_back(lens[i]);
        ctx->codeBytes = off[i] + (lens[i] + 15) / 16 * 16;
    }
}

int dmst_seqs_add_decoded(dmst_ctx *ctx, const uint8_t *codes, const int64_t *offsets, int nseq, int *first_id) {
    if (!ctx || (!codes && nseq > 0)) return DMST_EINVAL;
    int st = checkOffsets(offsets, nseq);
    if (st) return ctx->fail(st, "every sequence needs length >= 3");
    for (int64_t k = offsets[0]; k < offsets[nseq]; ++k)
        if (codes[k] >= kNumCodes) return ctx->fail(DMST_EINVAL, "codon code out of range at %lld", (long long)k);
    CK(cudaSetDevice(ctx->device), "set device");
    std::vector<long long> off;
    std::vector<int> lens;
    if ((st = reserveSeqs(ctx, offsets, nseq, off, lens))) return st;
    for (int i = 0; i < nseq; ++i)
        CK(cudaMemcpyAsync(ctx->dCodes.p + off[i], codes + offsets[i], lens[i], cudaMemcpyHostToDevice, ctx->stream),
           "upload codes");
    CK(cudaStreamSynchronize(ctx->stream), "upload codes");
    commitSeqs(ctx, off, lens, first_id);
    return DMST_OK;
}

int dmst_seqs_add_dna(dmst_ctx *ctx, const char *ascii, const int64_t *offsets, int nseq, int *first_id) {
    if (!ctx || (!ascii && nseq > 0)) return DMST_EINVAL;
    int st = checkOffsets(offsets, nseq);
    if (st) return ctx->fail(st, "every sequence needs length >= 3");
    if (nseq == 0) {
        if (first_id) *first_id = (int)ctx->seqLen.size();
        return DMST_OK;
    }
    CK(cudaSetDevice(ctx->device), "set device");
    std::vector<long long> off;
    std::vector<int> lens;
    if ((st = reserveSeqs(ctx, offsets, nseq, off, lens))) return st;
    const size_t nbytes = (size_t)(offsets[nseq] - offsets[0]);
    std::vector<long long> inOff(nseq);
    for (int i = 0; i < nseq; ++i) inOff[i] = offsets[i] - offsets[0];
    CK(ctx->dStage.ensure(nbytes), "alloc staging");
    CK(ctx->dStageOff.ensure(2 * (size_t)nseq), "alloc staging");
    CK(ctx->dStageLen.ensure(nseq), "alloc staging");
    CK(cudaMemcpyAsync(ctx->dStage.p, ascii + offsets[0], nbytes, cudaMemcpyHostToDevice, ctx->stream), "upload dna");
    CK(cudaMemcpyAsync(ctx->dStageOff.p, inOff.data(), nseq * sizeof(long long), cudaMemcpyHostToDevice, ctx->stream),
       "upload offsets");
    CK(cudaMemcpyAsync(ctx->dStageOff.p + nseq, off.data(), nseq * sizeof(long long), cudaMemcpyHostToDevice,
                       ctx->stream),
       "upload offsets");
    CK(cudaMemcpyAsync(ctx->dStageLen.p, lens.data(), nseq * sizeof(int), cudaMemcpyHostToDevice, ctx->stream),
       "upload lengths");
    decodeAsciiKernel<<<nseq, 256, 0, ctx->stream>>>(ctx->dStage.p, ctx->dStageOff.p, ctx->dStageOff.p + nseq,
                                                       ctx->dStageLen.p, ctx->dCodes.p);
    CK(cudaGetLastError(), "decode kernel");
    CK(cudaStreamSynchronize(ctx->stream), "decode kernel");
    commitSeqs(ctx, off, lens, first_id);
    return DMST_OK;
}

static void fillContig(dmst_contig &o, const FastaContig &c, int seqId) {
    o.record = c.record;
    o.start = c.start;
    o.length = c.length;
    o.seq_id = seqId;
    o.name_off = (int64_t)c.nameOff;
    o.name_len = c.nameLen;
    o.seq_id_rc = -1;
    o.letter_off = (int64_t)c.letterOff;
    o.record_length = c.recordLength;
    o.pipeline = (c.hasPipeline ? 1 : 0) | (c.isPlus ? 2 : 0);
    o.w_start = c.wStart;
    o.w_end = c.wEnd;
    o.true_length = c.trueLength;
    o.profile_off = (int64_t)c.profileOff;
    o.profile_len = c.profileLen;
    o.pad = 0;
}

int dmst_fasta_contigs(const char *text, size_t len, int flags, dmst_contig *contigs, size_t cap_contigs,
                       size_t *n_contigs, char *letters, size_t cap_letters, size_t *n_letters) {
    if ((!text && len) || !n_contigs || !n_letters || (flags & ~(DMST_FASTA_REVCOMP | DMST_FASTA_PIPELINE)))
        return DMST_EINVAL;
    std::vector<FastaContig> cs;
    std::string lt;
    if (fastaContigs(text, len, cs, lt, nullptr, (flags & DMST_FASTA_PIPELINE) != 0)) return DMST_EPARSE;
    *n_contigs = cs.size();
    *n_letters = lt.size();
    if (cap_contigs < cs.size() || cap_letters < lt.size()) return DMST_ERANGE;
    if ((cs.size() && !contigs) || (lt.size() && !letters)) return DMST_EINVAL;
    for (size_t k = 0; k < cs.size(); ++k) fillContig(contigs[k], cs[k], -1);
    if (!lt.empty()) std::memcpy(letters, lt.data(), lt.size());
    return DMST_OK;
}

int dmst_seqs_add_fasta(dmst_ctx *ctx, const char *text, size_t len, int flags, dmst_contig *contigs,
                        size_t cap_contigs, size_t *n_contigs) {
    if (!ctx || (!text && len) || !n_contigs || (flags & ~(DMST_FASTA_REVCOMP | DMST_FASTA_PIPELINE)))
        return DMST_EINVAL;
    std::vector<FastaContig> cs;
    std::string lt, perr;
    if (fastaContigs(text, len, cs, lt, &perr, (flags & DMST_FASTA_PIPELINE) != 0))
        return ctx->fail(DMST_EPARSE, "FASTA: %s", perr.c_str());
    *n_contigs = cs.size();
    if (cap_contigs < cs.size()) return ctx->fail(DMST_ERANGE, "FASTA: %zu contigs, capacity %zu", cs.size(), cap_contigs);
    if (cs.size() && !contigs) return DMST_EINVAL;
    const bool rc = (flags & DMST_FASTA_REVCOMP) != 0;
    // The sequences in id order: per record its contigs of >= 3 letters, then
    // (rc) their reverse complements, last contig first.  Each is packed 2
    // bits per base (A 0, C 1, G 2, T 3; each sequence on a fresh word) with
    // the other letters in the bitmap.
    std::vector<uint32_t> words, mask;
    std::vector<int64_t> off(1, 0);
    std::vector<std::pair<int, bool>> which;  // (contig, reverse complement)
    auto base2 = [](char v) { return v == 0 ? 0 : v == 1 ? 1 : v == 5 ? 2 : v == 16 ? 3 : -1; };
    auto pack = [&](size_t k, bool rev) {
        const FastaContig &c = cs[k];
        const size_t w0 = words.size(), m0 = mask.size();
        words.resize(w0 + (c.length + 15) / 16, 0u);
        mask.resize(m0 + (c.length + 31) / 32, 0u);
        for (int q = 0; q < c.length; ++q) {
            int b = base2(lt[c.letterOff + (rev ? c.length - 1 - q : q)]);
            if (rev && b >= 0) b = 3 - b;  // A-T, C-G
            if (b < 0)
                mask[m0 + q / 32] |= 1u << (q % 32);
            else
                words[w0 + q / 16] |= (uint32_t)b << (2 * (q % 16));
        }
        off.push_back(off.back() + c.length);
        which.emplace_back((int)k, rev);
    };
    for (size_t k0 = 0; k0 < cs.size();) {
        size_t k1 = k0;
        while (k1 < cs.size() && cs[k1].record == cs[k0].record) ++k1;
        for (size_t k = k0; k < k1; ++k)
            if (cs[k].length >= 3) pack(k, false);
        if (rc)
            for (size_t k = k1; k-- > k0;)
                if (cs[k].length >= 3) pack(k, true);
        k0 = k1;
    }
    int first = (int)ctx->seqLen.size();
    if (!which.empty()) {
        const int st = dmst_seqs_add_packed(ctx, words.data(), mask.data(), off.data(), (int)which.size(), &first);
        if (st) return st;
    }
    for (size_t k = 0; k < cs.size(); ++k) fillContig(contigs[k], cs[k], -1);
    for (size_t q = 0; q < which.size(); ++q) {
        dmst_contig &o = contigs[which[q].first];
        (which[q].second ? o.seq_id_rc : o.seq_id) = first + (int)q;
    }
    return DMST_OK;
}

int dmst_seqs_add_packed(dmst_ctx *ctx, const uint32_t *words, const uint32_t *mask_bits, const int64_t *offsets,
                         int nseq, int *first_id) {
    if (!ctx || (!words && nseq > 0)) return DMST_EINVAL;
    int st = checkOffsets(offsets, nseq);
    if (st) return ctx->fail(st, "every sequence needs length >= 3");
    if (nseq == 0) {
        if (first_id) *first_id = (int)ctx->seqLen.size();
        return DMST_OK;
    }
    CK(cudaSetDevice(ctx->device), "set device");
    std::vector<long long> off;
    std::vector<int> lens;
    if ((st = reserveSeqs(ctx, offsets, nseq, off, lens))) return st;
    // word / mask-word offsets per sequence: each sequence starts on a fresh word.
    std::vector<long long> wOff(nseq), mOff(nseq);
    long long nw = 0, nm = 0;
    for (int i = 0; i < nseq; ++i) {
        wOff[i] = nw;
        mOff[i] = nm;
        nw += (lens[i] + 15) / 16;
        nm += (lens[i] + 31) / 32;
    }
    // One pinned host block (words, mask words, the three offset arrays,
    // lengths) per call, two of them in turn: the copy and the decode are
    // queued on the context's stream without waiting, so a scoring call
    // queued before keeps running while the host goes on (every later call on
    // the stream finds the codes decoded).
    auto up16 = [](size_t x) { return (x + 15) & ~(size_t)15; };
    const size_t bW = (size_t)nw * 4, bM = mask_bits ? (size_t)nm * 4 : 0, bO = (size_t)nseq * 8;
    const size_t oM = up16(bW), oO = oM + up16(bM), oL = oO + up16(3 * bO), total = oL + (size_t)nseq * 4;
    const int b = ctx->seqStageNext;
    ctx->seqStageNext ^= 1;
    CK(cudaEventSynchronize(ctx->evSeqStage[b]), "sequence staging");  // its previous copy is done
    CK(ctx->hSeqStage[b].ensure(total), "alloc sequence staging");
    char *h = ctx->hSeqStage[b].p;
    std::memcpy(h, words, bW);
    if (mask_bits) std::memcpy(h + oM, mask_bits, bM);
    std::memcpy(h + oO, wOff.data(), bO);
    std::memcpy(h + oO + bO, mOff.data(), bO);
    std::memcpy(h + oO + 2 * bO, off.data(), bO);
    std::memcpy(h + oL, lens.data(), (size_t)nseq * 4);
    CK(ctx->dStage.ensure(total), "alloc staging");
    char *dv = ctx->dStage.p;
    CK(cudaMemcpyAsync(dv, h, total, cudaMemcpyHostToDevice, ctx->stream), "upload packed");
    CK(cudaEventRecord(ctx->evSeqStage[b], ctx->stream), "event");
    const long long *dOff = reinterpret_cast<const long long *>(dv + oO);
    decodePackedKernel<<<nseq, 256, 0, ctx->stream>>>(
        reinterpret_cast<const uint32_t *>(dv), mask_bits ? reinterpret_cast<const uint32_t *>(dv + oM) : nullptr,
        dOff, dOff + nseq, dOff + 2 * nseq, reinterpret_cast<const int *>(dv + oL), ctx->dCodes.p);
    CK(cudaGetLastError(), "decode kernel");
    commitSeqs(ctx, off, lens, first_id);
    return DMST_OK;
}

int dmst_windows_from_hits(const char *hits, size_t len, int flags, const char *const *record_names,
                           const int64_t *record_lengths, int n_records, const char *const *profile_names,
                           const int64_t *profile_lengths, int n_profiles, dmst_window *windows, size_t cap,
                           size_t *n_windows, size_t *n_malformed, size_t *n_dropped) {
    if ((!hits && len) || !n_windows || n_records < 0 || n_profiles < 0 || (n_records && (!record_names ||
        !record_lengths)) || (n_profiles && (!profile_names || !profile_lengths)) ||
        (flags & ~DMST_HITS_TARGET_IS_CONTIG))
        return DMST_EINVAL;
    std::vector<std::string> rn(n_records), pn(n_profiles);
    std::vector<long long> rl(n_records), pl(n_profiles);
    for (int k = 0; k < n_records; ++k) {
        if (!record_names[k]) return DMST_EINVAL;
        rn[k] = record_names[k];
        rl[k] = record_lengths[k];
    }
    for (int k = 0; k < n_profiles; ++k) {
        if (!profile_names[k]) return DMST_EINVAL;
        pn[k] = profile_names[k];
        pl[k] = profile_lengths[k];
    }
    std::vector<HitWindow> ws;
    size_t malformed = 0, dropped = 0;
    if (windowsFromHits(hits, len, (flags & DMST_HITS_TARGET_IS_CONTIG) != 0, rn, rl, pn, pl, ws, malformed, dropped,
                        nullptr))
        return DMST_EPARSE;
    *n_windows = ws.size();
    if (n_malformed) *n_malformed = malformed;
    if (n_dropped) *n_dropped = dropped;
    if (cap < ws.size()) return DMST_ERANGE;
    if (ws.size() && !windows) return DMST_EINVAL;
    for (size_t k = 0; k < ws.size(); ++k) {
        dmst_window &o = windows[k];
        o.record = ws[k].record;
        o.strand = ws[k].strand;
        o.start = ws[k].start;
        o.end = ws[k].end;
        o.profile_off = (int64_t)ws[k].profileOff;
        o.profile_len = ws[k].profileLen;
        o.profile = ws[k].profile;
    }
    return DMST_OK;
}

int dmst_genome_load(dmst_ctx *ctx, const char *text, size_t len, size_t *n_records, int64_t *record_lengths,
                     size_t cap_records) {
    if (!ctx || (!text && len) || !n_records) return DMST_EINVAL;
    std::vector<FastaContig> cs;
    std::vector<FastaRecord> recs;
    std::string lt, perr;
    if (fastaContigs(text, len, cs, lt, &perr, false, &recs)) return ctx->fail(DMST_EPARSE, "FASTA: %s", perr.c_str());
    *n_records = recs.size();
    if (record_lengths)
        for (size_t k = 0; k < recs.size() && k < cap_records; ++k) record_lengths[k] = recs[k].length;
    // every position of a record (its contigs' letters and its cutting
    // characters) 2 bits, each record on fresh words; the positions that are
    // not A, C, G or T (cutting characters included) set in the bitmap
    std::vector<dmst_ctx::GenomeRecord> g(recs.size());
    long long nw = kGenomePad, nm = kGenomePad;
    for (size_t r = 0; r < recs.size(); ++r) {
        g[r].nameOff = recs[r].nameOff;
        g[r].nameLen = recs[r].nameLen;
        g[r].length = recs[r].length;
        g[r].wordOff = nw;
        g[r].maskOff = nm;
        nw += (recs[r].length + 15) / 16;
        nm += (recs[r].length + 31) / 32;
    }
    std::vector<uint32_t> words((size_t)(nw + kGenomePad), 0u), mask((size_t)(nm + kGenomePad), ~0u);
    for (const FastaContig &c : cs) {
        dmst_ctx::GenomeRecord &gr = g[c.record];
        gr.contigs.emplace_back(c.start, c.length);
        for (int q = 0; q < c.length; ++q) {
            const int p = c.start + q;
            const char v = lt[c.letterOff + q];
            const int b = v == 0 ? 0 : v == 1 ? 1 : v == 5 ? 2 : v == 16 ? 3 : -1;
            if (b < 0) continue;
            words[gr.wordOff + p / 16] |= (uint32_t)b << (2 * (p % 16));
            mask[gr.maskOff + p / 32] &= ~(1u << (p % 32));
        }
    }
    CK(cudaSetDevice(ctx->device), "set device");
    CK(ctx->dGenomeWords.ensure(words.size()), "alloc genome");
    CK(ctx->dGenomeMask.ensure(mask.size()), "alloc genome");
    CK(cudaMemcpyAsync(ctx->dGenomeWords.p, words.data(), words.size() * 4, cudaMemcpyHostToDevice, ctx->stream),
       "upload genome");
    CK(cudaMemcpyAsync(ctx->dGenomeMask.p, mask.data(), mask.size() * 4, cudaMemcpyHostToDevice, ctx->stream),
       "upload genome");
    CK(cudaStreamSynchronize(ctx->stream), "upload genome");
    ctx->genome = std::move(g);
    return DMST_OK;
}

int dmst_seqs_add_windows(dmst_ctx *ctx, const dmst_window *windows, size_t n, dmst_contig *contigs,
                          size_t cap_contigs, size_t *n_contigs) {
    if (!ctx || (!windows && n) || !n_contigs) return DMST_EINVAL;
    for (size_t k = 0; k < n; ++k) {
        const dmst_window &w = windows[k];
        if (w.record < 0 || w.record >= (int)ctx->genome.size() || (w.strand != 1 && w.strand != -1) ||
            w.start < 0 || w.start > w.end || w.end > ctx->genome[w.record].length || w.profile_len < 0)
            return ctx->fail(DMST_EINVAL, "window %zu outside its record (or no genome loaded)", k);
    }
    // per window the record's contigs it overlaps, in the window's text order
    struct Piece {
        int window, start, length;  // start in the window
        int pos;                    // its first position in the record
    };
    std::vector<Piece> pieces;
    for (size_t k = 0; k < n; ++k) {
        const dmst_window &w = windows[k];
        const auto &cl = ctx->genome[w.record].contigs;
        auto it = std::upper_bound(cl.begin(), cl.end(), w.start,
                                   [](long long s, const std::pair<int, int> &c) { return s < (long long)c.first + c.second; });
        const size_t first = pieces.size();
        for (; it != cl.end() && it->first < w.end; ++it) {
            const long long a = std::max<long long>(w.start, it->first);
            const long long b = std::min<long long>(w.end, (long long)it->first + it->second);
            if (b <= a) continue;
            const long long st = w.strand > 0 ? a - w.start : w.end - b;
            pieces.push_back({(int)k, (int)st, (int)(b - a), (int)a});
        }
        if (w.strand < 0) std::reverse(pieces.begin() + first, pieces.end());
    }
    *n_contigs = pieces.size();
    if (cap_contigs < pieces.size())
        return ctx->fail(DMST_ERANGE, "windows: %zu contigs, capacity %zu", pieces.size(), cap_contigs);
    if (pieces.size() && !contigs) return DMST_EINVAL;
    std::vector<int64_t> off(1, 0);
    std::vector<size_t> which;
    for (size_t q = 0; q < pieces.size(); ++q)
        if (pieces[q].length >= 3) {
            off.push_back(off.back() + pieces[q].length);
            which.push_back(q);
        }
    int first = (int)ctx->seqLen.size();
    if (!which.empty()) {
        CK(cudaSetDevice(ctx->device), "set device");
        std::vector<long long> sOff;
        std::vector<int> lens;
        int st = reserveSeqs(ctx, off.data(), (int)which.size(), sOff, lens);
        if (st) return st;
        // the sequences are reserved back to back in whole 16-byte chunks
        std::vector<WinSeg> segs(which.size());
        long long nChunks = 0;
        for (size_t i = 0; i < which.size(); ++i) {
            const Piece &pc = pieces[which[i]];
            const dmst_window &w = windows[pc.window];
            const dmst_ctx::GenomeRecord &gr = ctx->genome[w.record];
            if (sOff[i] != sOff[0] + 16 * nChunks) return ctx->fail(DMST_EINVAL, "window sequences not contiguous");
            segs[i] = {gr.wordOff, gr.maskOff, sOff[i], pc.pos, pc.length, w.strand < 0 ? 1 : 0, (int)nChunks};
            nChunks += (pc.length + 15) / 16;
        }
        if (nChunks >= INT32_MAX) return ctx->fail(DMST_EINVAL, "windows: %lld chunks of 16 nt, too many", nChunks);
        const long long blocks = (nChunks + kWinThreads - 1) / kWinThreads;
        std::vector<int> blockSeg((size_t)blocks);
        for (long long bk = 0, sgi = 0; bk < blocks; ++bk) {  // the contig of each block's first chunk
            while (sgi + 1 < (long long)segs.size() && segs[sgi + 1].chunk <= bk * kWinThreads) ++sgi;
            blockSeg[bk] = (int)sgi;
        }
        // one upload: the descriptors, then the blocks' first contigs
        const size_t segBytes = segs.size() * sizeof(WinSeg), total = segBytes + blockSeg.size() * sizeof(int);
        CK(ctx->dWinSegs.ensure((total + sizeof(WinSeg) - 1) / sizeof(WinSeg), 0.3), "alloc window segments");
        std::vector<char> up(total);
        std::memcpy(up.data(), segs.data(), segBytes);
        std::memcpy(up.data() + segBytes, blockSeg.data(), blockSeg.size() * sizeof(int));
        CK(cudaMemcpyAsync(ctx->dWinSegs.p, up.data(), total, cudaMemcpyHostToDevice, ctx->stream),
           "upload window segments");
        for (auto &e : ctx->evWin)
            if (!e) CK(cudaEventCreate(&e), "event");
        CK(cudaEventRecord(ctx->evWin[0], ctx->stream), "event");
        windowDecodeKernel<<<(unsigned)blocks, kWinThreads, 0, ctx->stream>>>(
            ctx->dGenomeWords.p, ctx->dGenomeMask.p, ctx->dWinSegs.p,
            reinterpret_cast<const int *>(reinterpret_cast<const char *>(ctx->dWinSegs.p) + segBytes),
            (int)segs.size(), nChunks, ctx->dCodes.p);
        CK(cudaGetLastError(), "window decode kernel");
        CK(cudaEventRecord(ctx->evWin[1], ctx->stream), "event");
        ctx->winTimed = true;
        commitSeqs(ctx, sOff, lens, &first);
    }
    size_t next = 0;
    for (size_t q = 0; q < pieces.size(); ++q) {
        const Piece &pc = pieces[q];
        const dmst_window &w = windows[pc.window];
        const dmst_ctx::GenomeRecord &gr = ctx->genome[w.record];
        dmst_contig &o = contigs[q];
        o.record = pc.window;
        o.start = pc.start;
        o.length = pc.length;
        o.seq_id = pc.length >= 3 ? first + (int)next++ : -1;
        o.name_off = (int64_t)gr.nameOff;
        o.name_len = gr.nameLen;
        o.seq_id_rc = -1;
        o.letter_off = -1;
        o.record_length = (int32_t)(w.end - w.start);
        o.pipeline = 1 | (w.strand > 0 ? 2 : 0);
        o.w_start = w.start + 1;
        o.w_end = w.end;
        o.true_length = gr.length;
        o.profile_off = w.profile_off;
        o.profile_len = w.profile_len;
        o.pad = 0;
    }
    return DMST_OK;
}

int dmst_last_windows_ms(dmst_ctx *ctx, double *ms) {
    if (!ctx || !ms) return DMST_EINVAL;
    *ms = -1.0;
    if (!ctx->winTimed) return DMST_OK;
    CK(cudaEventSynchronize(ctx->evWin[1]), "window timing");
    float t = 0.f;
    CK(cudaEventElapsedTime(&t, ctx->evWin[0], ctx->evWin[1]), "window timing");
    *ms = t;
    return DMST_OK;
}

int dmst_seqs_clear(dmst_ctx *ctx) {
    if (ctx && ctx->slot[ctx->oldest].pending) {  // pending calls read the sequences being dropped
        const int ds = drainCalls(ctx);
        if (ds) return ds;
    }
    if (!ctx) return DMST_EINVAL;
    ctx->seqOff.clear();
    ctx->seqLen.clear();
    ctx->codeBytes = 0;
    return DMST_OK;
}

int dmst_seq_count(const dmst_ctx *ctx) { return ctx ? (int)ctx->seqLen.size() : 0; }

int dmst_seq_length(const dmst_ctx *ctx, int id) {
    return (ctx && id >= 0 && id < (int)ctx->seqLen.size()) ? ctx->seqLen[id] : -1;
}

int dmst_decode_letters(const char *letters, int L, uint8_t *codes) {
    if (!letters || !codes || L < 0) return DMST_EINVAL;
    decodeLetters(letters, L, codes);
    return DMST_OK;
}

int dmst_encode_dna(const char *ascii, int L, char *letters) {
    if (!ascii || !letters || L < 0) return DMST_EINVAL;
    return encodeDna(ascii, L, letters) < 0 ? DMST_EPARSE : DMST_OK;
}

// ---------------------------------------------------------------------------
// Scoring
// ---------------------------------------------------------------------------
// scoreToLog (dummest-score.hh:202-207): std::log of the float mantissa is the
// float overload, so the logarithm is taken in single precision and then
// added to e * ln 2 in double, as the reference's logProbRatio is.
// scoreToLog (dummest-score.hh:203-208) as the reference's x86-64-v3 build
// evaluates it: the float log of the mantissa, then e ln 2 added in one fused
// multiply-add (GCC contracts the expression at -O3).
static double scoreLn(float m, int e) { return std::fma((double)e, 0.6931471805599453, (double)std::log(m)); }

static void fillResult(dmst_result &r, float v, bool isFilterF, dmst_score *dst, double *ln) {
    (void)isFilterF;
    (void)r;
    if (!(v > 0.0f)) {
        dst->m = 0.0f;
        dst->e = 0;
        *ln = -INFINITY;
        return;
    }
    int e = 0;
    float m = std::frexp(v, &e);
    if (std::isinf(v)) {
        m = 0.0f;
        e = 0;
    }
    dst->m = m;
    dst->e = e;
    *ln = (m == 0.0f) ? (std::isinf(v) ? INFINITY : -INFINITY) : scoreLn(m, e);
}

static void scoreToResult(XS s, dmst_score *dst, double *ln) {
    dst->m = s.m;
    dst->e = s.e;
    *ln = (s.m == 0.0f) ? -INFINITY : scoreLn(s.m, s.e);
}

// Milliseconds between two recorded events; a timing failure is noted in the
// context's error text and cleared (it must not surface as the error of a
// later launch check), and reads as -1.
static float elapsedMs(dmst_ctx *ctx, cudaEvent_t a, cudaEvent_t b) {
    float ms = -1.0f;
    const cudaError_t e = cudaEventElapsedTime(&ms, a, b);
    if (e != cudaSuccess) {
        cudaGetLastError();
        ctx->err = std::string("event timing: ") + cudaGetErrorString(e);
        return -1.0f;
    }
    return ms;
}

// Internal mode bit: set up the pairs and run the null model only (the
// device pair descriptors, seeds and scales of the call stay in the context).
constexpr int kModeNullOnly = 0x10000;

// Host setup, uploads and the launches of a call into slot ctx->nextSlot
// (which must be free); the call completes in completeCall.
// minBest (search only): per profile id, the filter wave's gate (the smallest
// float best that survives); the call then runs both waves.
// anchorBest/anchorRow (anchors only): the per-column anchors of every pair,
// scored on the exact path.  alignJobs (with anchors): every pair is a
// traceback job (job k = pair k; the exact kernel keeps its W0, W1 and
// rescale counts); the jobs' pair fields become the pairs' internal positions
// and the jobs go to ctx->dAlignJobs.
static int submitCall(dmst_ctx *ctx, const dmst_pair *pairs, size_t n, int mode, dmst_result *out,
                      const float *minBest = nullptr, dmst_score *anchorBest = nullptr, int *anchorRow = nullptr,
                      std::vector<AlignJob> *alignJobs = nullptr) {
    const bool nullOnly = (mode & kModeNullOnly) != 0;
    const bool search = minBest != nullptr;
    const bool anchors = anchorBest != nullptr;
    if (anchors) mode |= DMST_MODE_FORCE_EXACT;
    if (!ctx || (n && (!pairs || (!out && !nullOnly)))) return DMST_EINVAL;
    const int base = mode & 0xff;
    const bool plain = (mode & (DMST_MODE_PLAIN | DMST_MODE_PLAIN_1WARP)) != 0;
    // the plain schedule's kernel: the pair's stripes on the CTA's warps, or
    // (DMST_MODE_PLAIN_1WARP) the batched kernel's one warp per pair
    const bool plainStriped = plain && !(mode & DMST_MODE_PLAIN_1WARP);
    const bool forceExact = (mode & (DMST_MODE_FORCE_EXACT | DMST_MODE_EXACT_SEQUENTIAL)) != 0;
    const bool sequentialExact = (mode & DMST_MODE_EXACT_SEQUENTIAL) != 0;
    if (base != DMST_MODE_MID && base != DMST_MODE_FILTER) return DMST_EINVAL;
    const bool mid = base == DMST_MODE_MID;
    const auto hostT0 = std::chrono::steady_clock::now();
    const int si = ctx->nextSlot;
    CallSlot &S = ctx->slot[si];
    if (S.pending) return ctx->fail(DMST_EINVAL, "scoring call: no free slot");
    if (n > (size_t)INT32_MAX / 2) return ctx->fail(DMST_ERANGE, "too many pairs");
    CK(cudaSetDevice(ctx->device), "set device");
    int st = uploadProfiles(ctx);
    if (st) return st;

    // Pair descriptors, ordered by profile then by cost (costliest first).
    std::vector<int> order(n);
    std::iota(order.begin(), order.end(), 0);
    for (size_t i = 0; i < n; ++i) {
        const dmst_pair &q = pairs[i];
        if (q.seq < 0 || q.seq >= (int)ctx->seqLen.size() || q.profile < 0 || q.profile >= (int)ctx->profiles.size())
            return ctx->fail(DMST_EINVAL, "pair %zu: unknown sequence or profile id", i);
    }
    {
        // Profile-major, longest read first, input order breaking ties.  Two
        // stable counting sorts (by length, descending, then by profile) when
        // the length range is small against n; one key sort otherwise.
        int maxLen = 0;
        for (size_t i = 0; i < n; ++i) maxLen = std::max(maxLen, ctx->seqLen[pairs[i].seq]);
        const size_t nProf = ctx->profiles.size();
        if ((size_t)maxLen <= 4 * n + 65536) {
            std::vector<int> cnt((size_t)maxLen + 2, 0), byLen(n);
            for (size_t i = 0; i < n; ++i) ++cnt[(size_t)(maxLen - ctx->seqLen[pairs[i].seq]) + 1];
            for (size_t v = 1; v < cnt.size(); ++v) cnt[v] += cnt[v - 1];
            for (size_t i = 0; i < n; ++i) byLen[cnt[(size_t)(maxLen - ctx->seqLen[pairs[i].seq])]++] = (int)i;
            std::vector<int> start(nProf + 1, 0);
            for (size_t i = 0; i < n; ++i) ++start[(size_t)pairs[i].profile + 1];
            for (size_t q = 0; q < nProf; ++q) start[q + 1] += start[q];
            for (size_t k = 0; k < n; ++k) order[start[pairs[byLen[k]].profile]++] = byLen[k];
        } else {
            std::vector<std::pair<uint64_t, int>> keys(n);
            for (size_t i = 0; i < n; ++i) {
                const uint32_t inv = 0xFFFFFFFFu - (uint32_t)ctx->seqLen[pairs[i].seq];
                keys[i] = {((uint64_t)(uint32_t)pairs[i].profile << 32) | inv, (int)i};
            }
            std::sort(keys.begin(), keys.end());
            for (size_t i = 0; i < n; ++i) order[i] = keys[i].second;
        }
    }
    // The kernel shape of every pair (rows per lane and warps per CTA, from
    // the profile's length and the read's length class).  With tuned shapes,
    // a shape group too small to give every CTA two chunks would run as its
    // own underfilled launch; its pairs join the largest group instead.
    std::vector<int> pairShape(n);
    {
        // the shape depends on the profile and the read's length class only
        const size_t nProf = ctx->profiles.size();
        std::vector<int> shapeTab(2 * nProf);
        for (size_t q = 0; q < nProf; ++q)
            for (int c = 0; c < 2; ++c) {
                int R, W;
                shapeOf(ctx->profiles[q].M, c ? 0 : kShortRead, ctx->opts.rows_per_lane, ctx->tune, R, W);
                if (plainStriped && R == 3) R = 4;  // the plain schedule's stripes take R = 4, 2 or 1
                shapeTab[2 * q + c] = rIndex(R) * 3 + wIndex(W);
            }
        long long groupPairs[kNumShapes] = {};
        for (size_t i = 0; i < n; ++i) {
            pairShape[i] = shapeTab[2 * (size_t)pairs[i].profile + lengthClass(ctx->seqLen[pairs[i].seq])];
            ++groupPairs[pairShape[i]];
        }
        if (ctx->tune.tuned && !ctx->tune.forceR && ctx->opts.rows_per_lane == 0 && !plain) {
            int big = 0;
            for (int q = 1; q < kNumShapes; ++q)
                if (groupPairs[q] > groupPairs[big]) big = q;
            int remap[kNumShapes];
            bool any = false;
            for (int q = 0; q < kNumShapes; ++q) {
                const long long fill = 2LL * ctx->smCount * 4 * kShapeWarps[q % 3];
                remap[q] = (q != big && groupPairs[q] > 0 && groupPairs[q] < fill) ? big : q;
                any |= remap[q] != q;
            }
            if (any)
                for (int &sh : pairShape) sh = remap[sh];
        }
    }
    std::vector<DevPair> dp(n);
    long long seedFloats = 0;
    size_t w1Max = 0, ringMax = 0;
    for (size_t k = 0; k < n; ++k) {
        const dmst_pair &q = pairs[order[k]];
        DevPair &d = dp[k];
        d.codeOff = ctx->seqOff[q.seq];
        d.L = ctx->seqLen[q.seq];
        d.M = ctx->profiles[q.profile].M;
        d.prof = q.profile;
        d.R = kShapeR[pairShape[order[k]] / 3];
        d.seedOff = seedFloats;
        seedFloats += 2LL * d.L;
        // the staggered kernel's W1 groups (one per step) and its ring (W, Y per column)
        if (mid) w1Max = std::max(w1Max, (size_t)stagSlotFloats(d.M, d.L, d.R));
        ringMax = std::max(ringMax, 2 * (size_t)stagPeriod(d.L, d.R));
    }
    // Kernel groups by shape.  Chunks: runs of pairs of one profile and shape,
    // costliest first within each group.
    struct Group {
        int R, warps;     // warps launched per CTA (<= kernWarps when shared memory is short)
        int kernWarps;    // the kernel's CTA shape (warp slots per CTA)
        DpKern kern;
        DpKern kernF = nullptr;  // search: the filter wave's kernel of the same shape
        bool gt = false;  // emission table read from global memory
        std::vector<Chunk> chunks;
        std::vector<double> cost;
        int maxRowPad = 0;
        size_t smem = 0;
        int grid = 0;
        size_t chunkBase = 0;
    };
    Group groups[kNumShapes];
    for (int q = 0; q < kNumShapes; ++q) {
        const int W = kShapeWarps[q % 3];
        groups[q].R = kShapeR[q / 3];
        groups[q].kernWarps = W;
        groups[q].warps = W;
        groups[q].kern = dpKernelFor(groups[q].R, mid, W, false);
    }
    auto groupOf = [&](size_t k) { return pairShape[order[k]]; };  // the group of sorted position k
    // Warps per CTA: tall profiles leave less shared memory for the windows
    // (or keep their table in global memory), and long pairs of tall profiles
    // are capped by the device memory their W1 slots take.
    const size_t smemLimit = (size_t)ctx->maxSmemOptin - 1024;
    long long groupPairs[kNumShapes] = {};
    for (size_t k = 0; k < n && !nullOnly; ++k) {
        Group &G = groups[groupOf(k)];
        G.maxRowPad = std::max(G.maxRowPad, ctx->profiles[dp[k].prof].rowPad);
        ++groupPairs[groupOf(k)];
    }
    // Slot sizes rounded up to one of eight levels per power of two (at most
    // 12.5% larger), so that calls of similar shape keep the same slot layout
    // (and replay the same launch graph under DMST_MODE_GRAPH).
    auto slotLevel = [](size_t v) {
        v = std::max<size_t>(v, 64);
        const int hb = 63 - __builtin_clzll((unsigned long long)v);
        const size_t q = std::max<size_t>((size_t)1 << std::max(hb - 3, 6), 64);
        return (v + q - 1) / q * q;
    };
    const size_t w1Slot = slotLevel(w1Max);
    const size_t ringSlot = slotLevel(ringMax);
    // Every launched warp holds one W1 slot: at most maxSlots of them fit the
    // device budget (the call's budget, or 60% of the free memory counting the
    // slots the context already holds).  Long pairs of tall profiles (80 MB of
    // W1 at M = 2000 x 10 kb) then run fewer warps per CTA, or fewer CTAs.
    // The stores of an earlier posterior or gradient call (dmst_posteriors
    // and the like keep them for the next such call) are given up when the
    // slots of a full GPU (every SM at the widest CTA) would not fit without them.
    size_t maxSlots = SIZE_MAX;
    if (mid && !nullOnly) {
        size_t freeB = 0, totalB = 0;
        CK(cudaMemGetInfo(&freeB, &totalB), "memory info");
        const size_t held = (ctx->dW1.cap + ctx->dRing.cap) * sizeof(float);
        const size_t slotBytes = (w1Slot + ringSlot) * sizeof(float);
        const size_t adjHeld = (ctx->dAdjF.cap + ctx->dAdjB.cap + ctx->dPost.cap) * sizeof(double);
        const size_t fullGpu = (size_t)ctx->smCount * kCtaWarps * slotBytes;
        if (!ctx->opts.device_budget_bytes && adjHeld && 0.6 * (double)(freeB + held) < (double)fullGpu) {
            ctx->dAdjF.release();  // synchronises the device, once
            ctx->dAdjB.release();
            ctx->dPost.release();
            CK(cudaMemGetInfo(&freeB, &totalB), "memory info");
        }
        const size_t budget =
            ctx->opts.device_budget_bytes ? ctx->opts.device_budget_bytes : (size_t)(0.6 * (double)(freeB + held));
        maxSlots = std::max<size_t>(1, budget / slotBytes);
    }
    int chunkPairsOf[kNumShapes];
    for (int q = 0; q < kNumShapes; ++q) {
        chunkPairsOf[q] = 1;
        Group &G = groups[q];
        if (!groupPairs[q]) continue;
        const size_t table = (size_t)kNumCodes * G.maxRowPad * sizeof(float);
        // A table that would leave room for fewer than the shape's warps stays
        // in global memory instead (read through L1), and every warp runs.
        const size_t winBytes = stagWindowBytes(G.R);
        G.gt = table + (size_t)G.kernWarps * winBytes > smemLimit;
        if (G.gt) G.kern = dpKernelFor(G.R, mid, G.kernWarps, true);
        if (search) G.kernF = dpKernelFor(G.R, false, G.kernWarps, G.gt);
        G.warps = G.gt ? G.kernWarps : (int)std::min<size_t>(G.kernWarps, (smemLimit - table) / winBytes);
        G.warps = (int)std::max<size_t>(1, std::min<size_t>(G.warps, maxSlots / ctx->smCount));
        // Chunks of up to four pairs per launched warp, fewer when the group is
        // too small to give each CTA four chunks, but never fewer pairs than the
        // CTA's warps while there are that many pairs per SM (a chunk of fewer
        // pairs leaves warps idle until the chunk's barrier).
        const long long perCta = groupPairs[q] / (4LL * ctx->smCount);
        const long long perSm = (groupPairs[q] + ctx->smCount - 1) / ctx->smCount;
        const long long floorPairs = std::min<long long>(G.warps, perSm);
        chunkPairsOf[q] =
            plain ? 1 : (int)std::max<long long>(1, std::min<long long>(4LL * G.warps, std::max(floorPairs, perCta)));
    }
    for (size_t k = 0; k < n && !nullOnly;) {
        Group &G = groups[groupOf(k)];
        size_t e = k;
        double cost = 0;
        const int chunkPairs = chunkPairsOf[groupOf(k)];
        while (e < n && dp[e].prof == dp[k].prof && groupOf(e) == groupOf(k) && (int)(e - k) < chunkPairs) {
            cost += (double)(dp[e].M + 1) * dp[e].L;
            ++e;
        }
        const int rowPad = ctx->profiles[dp[k].prof].rowPad;
        G.chunks.push_back(Chunk{(int)k, (int)(e - k), dp[k].prof, rowPad});
        G.cost.push_back(cost);
        k = e;
    }
    std::vector<Chunk> allChunks;
    size_t slotsMax = 0;
    for (Group &G : groups) {
        if (G.chunks.empty()) continue;
        if (!plain) {
            std::vector<int> co(G.chunks.size());
            std::iota(co.begin(), co.end(), 0);
            std::stable_sort(co.begin(), co.end(), [&](int a, int b) { return G.cost[a] > G.cost[b]; });
            std::vector<Chunk> sorted(co.size());
            for (size_t i = 0; i < co.size(); ++i) sorted[i] = G.chunks[co[i]];
            G.chunks.swap(sorted);
        }
        G.chunkBase = allChunks.size();
        allChunks.insert(allChunks.end(), G.chunks.begin(), G.chunks.end());
        // Shared memory: the emission table, then one staging window per warp.
        const size_t table = (size_t)kNumCodes * G.maxRowPad * sizeof(float);
        G.smem = (G.gt ? 0 : table) + (size_t)G.warps * stagWindowBytes(G.R);
        CK(cudaFuncSetAttribute(G.kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)G.smem),
           "smem attribute");
        if (search)
            CK(cudaFuncSetAttribute(G.kernF, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)G.smem),
               "smem attribute");
        int perSm = 0;
        CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSm, G.kern, G.warps * kLanes, G.smem), "occupancy");
        if (perSm < 1) return ctx->fail(DMST_ERANGE, "kernel does not fit on an SM");
        G.grid = plain ? 1 : (int)std::min<long long>((long long)perSm * ctx->smCount, (long long)G.chunks.size());
        G.grid = (int)std::max<size_t>(1, std::min<size_t>(G.grid, maxSlots / G.warps));
        slotsMax = std::max(slotsMax, (size_t)G.grid * G.warps);
    }

    // Uploads go through the slot's page-locked staging, so that they queue
    // behind the previous call's kernels without waiting for them.
    auto upload = [&](auto &pinned, auto *dst, const auto *src, size_t cnt, const char *what) -> int {
        if (!cnt) return DMST_OK;
        CK(pinned.ensure(cnt), what);
        std::memcpy(pinned.p, src, cnt * sizeof(*src));
        CK(cudaMemcpyAsync(dst, pinned.p, cnt * sizeof(*src), cudaMemcpyHostToDevice, ctx->stream), what);
        return DMST_OK;
    };
    CK(S.dPairs.ensure(n), "alloc pairs");
    CK(S.dSeeds.ensure((size_t)seedFloats, 0.1), "alloc seeds");
    CK(S.dScales.ensure(n), "alloc scales");
    CK(S.dOut.ensure(n), "alloc out");
    CK(ctx->dChunks.ensure(allChunks.size(), 0.25), "alloc chunks");
    if ((st = upload(S.hPairs, S.dPairs.p, dp.data(), n, "upload pairs"))) return st;
    if ((st = upload(S.hChunks, ctx->dChunks.p, allChunks.data(), allChunks.size(), "upload chunks"))) return st;
    // The groups run one after another on the stream, so they share the slots.
    size_t plainScratch = 0;
    if (plainStriped)
        for (size_t k = 0; k < n; ++k)
            plainScratch = std::max(plainScratch, (size_t)plainScratchFloats(dp[k].M, dp[k].L, dp[k].R));
    // 25% headroom: the slot size follows the call's longest pairs and their
    // kernel shapes, so calls of one workload vary, and a grown W1 buffer
    // (tens of GB) costs the host a long allocation
    CK(ctx->dW1.ensure(std::max<size_t>(std::max(slotsMax * w1Slot, plainScratch), 1), 0.25), "alloc W1 slots");
    CK(ctx->dRing.ensure(std::max<size_t>(slotsMax * ringSlot, 1), 0.25), "alloc ring slots");
    // one counter per group (search: the second wave's after them; the one-warp plain schedule: one per chunk)
    const size_t nCounters = std::max<size_t>(allChunks.size() + kNumShapes, 2 * kNumShapes);
    CK(ctx->dCounter.ensure(nCounters), "alloc counters");

    // Null-model jobs: up to 32 pairs of reads of one length per warp (the
    // lanes run in lock step over the columns), the pairs of one read
    // side by side, the longest reads first: the kernel's warps take the jobs
    // round-robin, so that each warp ends on short jobs and the kernel has no
    // tail of long reads started last.
    std::vector<int> jobPairs(n);
    {
        // A counting sort of the (profile-major) pair slots by read, with the
        // call's reads taken in (length descending, id) order.
        const size_t nSeq = ctx->seqLen.size();
        std::vector<int> start(nSeq, 0);  // pairs of each read, then where they start
        for (size_t k = 0; k < n; ++k) ++start[pairs[order[k]].seq];
        std::vector<int> used;
        for (size_t q = 0; q < nSeq; ++q)
            if (start[q]) used.push_back((int)q);
        std::sort(used.begin(), used.end(), [&](int x, int y) {
            return ctx->seqLen[x] != ctx->seqLen[y] ? ctx->seqLen[x] > ctx->seqLen[y] : x < y;
        });
        int at = 0;
        for (int q : used) {
            const int c = start[q];
            start[q] = at;
            at += c;
        }
        for (size_t k = 0; k < n; ++k) jobPairs[start[pairs[order[k]].seq]++] = (int)k;
    }
    std::vector<NullJob> nullJobs;
    std::vector<long long> nullTmpOff;
    long long nullTmpEntries = 0;
    for (size_t k = 0; k < n;) {
        size_t e = k;
        while (e < n && e - k < 32 && dp[jobPairs[e]].L == dp[jobPairs[k]].L) ++e;
        nullJobs.push_back(NullJob{(int)k, (int)(e - k)});
        nullTmpOff.push_back(nullTmpEntries);
        nullTmpEntries += dmst::nullTmpEntries(dp[jobPairs[k]].L);
        k = e;
    }
    CK(ctx->dNullJobs.ensure(nullJobs.size(), 0.25), "alloc null jobs");
    CK(ctx->dNullJobPairs.ensure(n), "alloc null jobs");
    CK(ctx->dNullTmp.ensure((size_t)nullTmpEntries, 0.1), "alloc null tmp");
    CK(ctx->dNullTmpOff.ensure(nullJobs.size(), 0.25), "alloc null tmp");
    if ((st = upload(S.hNullJobs, ctx->dNullJobs.p, nullJobs.data(), nullJobs.size(), "upload null jobs"))) return st;
    if ((st = upload(S.hJobPairs, ctx->dNullJobPairs.p, jobPairs.data(), n, "upload null jobs"))) return st;
    if ((st = upload(S.hNullTmpOff, ctx->dNullTmpOff.p, nullTmpOff.data(), nullTmpOff.size(), "upload null jobs")))
        return st;

    // The exact path on the device: flagged pairs go to a queue that
    // persistent CTAs of the exact kernel drain, each CTA (or, when no pair of
    // the call has more than kPipeWarps / 2 stripes and more pairs than SMs are
    // expected, each half of a CTA) with a scratch slot sized for the largest
    // pair of the call.
    const bool exactOnDevice = mid && !nullOnly && !sequentialExact;
    long long poolSlot = 0;
    int exactGrid = 0, exactGroups = 1;
    if (exactOnDevice) {
        int maxWarps = 1;
        for (size_t k = 0; k < n; ++k) maxWarps = std::max(maxWarps, exactWarps(dp[k].M));
        // two groups pay only with more exact-path pairs than SMs (the
        // grouped kernel holds more per thread; with fewer pairs, one pair per
        // SM is faster): a forced call sends every pair, otherwise the last
        // call's count stands in
        const long long exactPairsExpected = forceExact ? (long long)n : (long long)ctx->lastFlagged;
        exactGroups = maxWarps <= kPipeWarps / 2 && exactPairsExpected > ctx->smCount ? 2 : 1;
        for (size_t k = 0; k < n; ++k)
            poolSlot = std::max(poolSlot, exactWaveScratch(dp[k].M, dp[k].L,
                                                           std::min(exactWarps(dp[k].M), kPipeWarps / exactGroups),
                                                           anchors));
        poolSlot = (poolSlot + 63) / 64 * 64;
        size_t freeB = 0, totalB = 0;
        CK(cudaMemGetInfo(&freeB, &totalB), "memory info");
        const size_t poolBudget = std::max<size_t>((freeB + ctx->dExactPool.cap * sizeof(float)) / 4, (size_t)256 << 20);
        exactGrid = (int)std::max<size_t>(
            1, std::min<size_t>((size_t)ctx->smCount,
                                poolBudget / ((size_t)poolSlot * exactGroups * sizeof(float))));
        CK(ctx->dExactPool.ensure((size_t)exactGrid * exactGroups * poolSlot), "alloc exact scratch");
        CK(S.dExOut.ensure(n), "alloc exact out");
        CK(S.dQueue.ensure(n), "alloc exact queue");
        CK(S.dQueueCount.ensure(2), "alloc exact queue");
        CK(S.hExOut.ensure(n), "alloc exact out");
        if (!ctx->exactAttrSet) {
            CK(cudaFuncSetAttribute(exactWaveKernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)(kPipeWarps * sizeof(Window))),
               "smem attribute");
            CK(cudaFuncSetAttribute(exactWaveKernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)(kPipeWarps * sizeof(Window))),
               "smem attribute");
            CK(cudaFuncSetAttribute(exactWaveKernel<true, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)(kPipeWarps * sizeof(Window))),
               "smem attribute");
            CK(cudaFuncSetAttribute(exactWaveKernel<false, false, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)(kPipeWarps * sizeof(Window))),
               "smem attribute");
            CK(cudaFuncSetAttribute(exactWaveKernel<true, false, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)(kPipeWarps * sizeof(Window))),
               "smem attribute");
            CK(cudaFuncSetAttribute(exactWaveKernel<true, true, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)(kPipeWarps * sizeof(Window))),
               "smem attribute");
            ctx->exactAttrSet = true;
        }
    }
    CK(S.hOut.ensure(n), "alloc results");
    long long anchorCols = 0;
    if (anchors) {
        // columns of each pair, in the caller's order; pair position k -> offset
        std::vector<long long> callerOff(n);
        for (size_t i = 0; i < n; ++i) {
            callerOff[i] = anchorCols;
            anchorCols += ctx->seqLen[pairs[i].seq];
        }
        std::vector<long long> off(n);
        for (size_t k = 0; k < n; ++k) off[k] = callerOff[order[k]];
        CK(S.dAnchorM.ensure((size_t)anchorCols, 0.3), "alloc anchors");
        CK(S.dAnchorE.ensure((size_t)anchorCols, 0.3), "alloc anchors");
        CK(S.dAnchorRow.ensure((size_t)anchorCols, 0.3), "alloc anchors");
        CK(S.hAnchorM.ensure((size_t)anchorCols), "alloc anchors");
        CK(S.hAnchorE.ensure((size_t)anchorCols), "alloc anchors");
        CK(S.hAnchorRow.ensure((size_t)anchorCols), "alloc anchors");
        CK(S.dAnchorOff.ensure(n), "alloc anchors");
        if ((st = upload(S.hAnchorOff, S.dAnchorOff.p, off.data(), n, "upload anchors"))) return st;
    }
    const bool align = anchors && alignJobs != nullptr;
    if (align) {
        std::vector<int> pos(n), jobOf(n);
        for (size_t k = 0; k < n; ++k) {
            pos[order[k]] = (int)k;
            jobOf[k] = order[k];
        }
        for (AlignJob &jb : *alignJobs) jb.pair = pos[jb.pair];
        CK(ctx->dAlignJobs.ensure(n), "alloc traceback jobs");
        CK(ctx->dAlignJobOf.ensure(n), "alloc traceback jobs");
        CK(cudaMemcpyAsync(ctx->dAlignJobs.p, alignJobs->data(), n * sizeof(AlignJob), cudaMemcpyHostToDevice,
                           ctx->stream),
           "upload traceback jobs");
        CK(cudaMemcpyAsync(ctx->dAlignJobOf.p, jobOf.data(), n * sizeof(int), cudaMemcpyHostToDevice, ctx->stream),
           "upload traceback jobs");
        CK(cudaStreamSynchronize(ctx->stream), "upload traceback jobs");  // the host vectors go out of scope
    }
    int chunkStride = 1;
    if (search) {
        for (const Chunk &c : allChunks) chunkStride = std::max(chunkStride, c.count);
        const size_t nProf = ctx->profiles.size();
        CK(S.dOutF.ensure(n), "alloc filter results");
        CK(S.dMask.ensure(n), "alloc survivors");
        CK(S.hOutF.ensure(n), "alloc filter results");
        CK(S.hMask.ensure(n), "alloc survivors");
        CK(ctx->dMidChunks.ensure(std::max<size_t>(allChunks.size(), 1)), "alloc survivor chunks");
        CK(ctx->dSurvivors.ensure(std::max<size_t>(allChunks.size() * chunkStride, 1)), "alloc survivors");
        CK(ctx->dMinBest.ensure(nProf), "alloc filter gates");
        if ((st = upload(S.hMinBest, ctx->dMinBest.p, minBest, nProf, "upload filter gates"))) return st;
    }

    S.hostMs = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - hostT0).count();
    NullRates nr;
    nr.single = (double)(ctx->rates.insert1 + ctx->rates.delete2);
    nr.dbl = (double)(ctx->rates.insert2 + ctx->rates.delete1);
    const int nj = (int)nullJobs.size();
    // One wave of null-model blocks: as many as fit on the GPU at once.
    if (!ctx->nullBlocksPerSm) {
        int perSm = 0;
        CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSm, nullModelKernel, kNullWarps * 32, 0),
           "null-model occupancy");
        ctx->nullBlocksPerSm = std::max(1, perSm);
    }
    const int nullBlocks =
        std::max(1, std::min((nj + kNullWarps - 1) / kNullWarps, ctx->smCount * ctx->nullBlocksPerSm));
    DpArgs g;
    g.pairs = S.dPairs.p;
    g.profiles = ctx->dProfiles.p;
    g.emit = ctx->dEmit.p;
    g.params = ctx->dParams.p;
    g.codes = ctx->dCodes.p;
    g.seeds = S.dSeeds.p;
    g.scales = S.dScales.p;
    g.w1 = ctx->dW1.p;
    g.w1SlotFloats = w1Slot;
    g.ring = ctx->dRing.p;
    g.ringSlotFloats = ringSlot;
    g.out = S.dOut.p;
    g.pairIdx = nullptr;
    // The device work of the call up to the DP results: counter reset,
    // null-model kernel, the DP kernels of each rows-per-lane group, and the
    // timing events between them.
    int launches = 0;
    // Inside a stream capture the timing events become external event-record
    // nodes, which (unlike internal ones) can be read with cudaEventElapsedTime.
    bool capturing = false;
    auto record = [&](cudaEvent_t ev) {
        return capturing ? cudaEventRecordWithFlags(ev, ctx->stream, cudaEventRecordExternal)
                         : cudaEventRecord(ev, ctx->stream);
    };
    auto enqueue = [&]() -> int {
        launches = 0;
        CK(cudaMemsetAsync(ctx->dCounter.p, 0, nCounters * sizeof(int), ctx->stream), "zero counters");
        if (exactOnDevice) CK(cudaMemsetAsync(S.dQueueCount.p, 0, 2 * sizeof(int), ctx->stream), "zero queue");
        CK(record(S.ev[0]), "event");
        nullModelKernel<<<nullBlocks, kNullWarps * 32, 0, ctx->stream>>>(
            ctx->dNullJobs.p, nj, ctx->dNullJobPairs.p, S.dPairs.p, ctx->dProfiles.p, ctx->dCodes.p,
            S.dSeeds.p, ctx->dNullTmp.p, ctx->dNullTmpOff.p, S.dScales.p, nr);
        CK(cudaGetLastError(), "null-model kernel");
        ++launches;
        CK(record(S.ev[1]), "event");
        if (search) {
            // the filter wave over every pair, then each chunk's survivors
            for (int gi = 0; gi < kNumShapes; ++gi) {
                Group &G = groups[gi];
                if (G.chunks.empty()) continue;
                DpArgs gk = g;
                gk.out = S.dOutF.p;
                gk.chunks = ctx->dChunks.p + G.chunkBase;
                gk.nChunks = (int)G.chunks.size();
                gk.chunkCounter = ctx->dCounter.p + gi;
                G.kernF<<<G.grid, G.warps * kLanes, G.smem, ctx->stream>>>(gk, G.gt ? 0 : kNumCodes * G.maxRowPad);
                CK(cudaGetLastError(), "filter kernel");
                ++launches;
            }
            const int nc = (int)allChunks.size();
            survivorKernel<<<(nc + 7) / 8, 256, 0, ctx->stream>>>(ctx->dChunks.p, nc, S.dOutF.p, ctx->dMinBest.p,
                                                                  ctx->dMidChunks.p, ctx->dSurvivors.p, chunkStride,
                                                                  S.dMask.p);
            CK(cudaGetLastError(), "survivor kernel");
            ++launches;
        }
        if (!forceExact && !nullOnly) {
            for (int gi = 0; gi < kNumShapes; ++gi) {
                Group &G = groups[gi];
                if (G.chunks.empty()) continue;
                if (plainStriped) {
                    // One pair per launch, its stripes on the CTA's warps.
                    auto pk = plainKernelFor(G.R, mid);
                    for (size_t k = 0; k < G.chunks.size(); ++k) {
                        pk<<<1, kPlainWarps * kLanes, kPlainWarps * sizeof(Window), ctx->stream>>>(
                            S.dPairs.p, G.chunks[k].first, ctx->dProfiles.p, ctx->dEmit.p, ctx->dParams.p,
                            ctx->dCodes.p, S.dSeeds.p, S.dScales.p, ctx->dW1.p, S.dOut.p, ctx->waitLimit);
                        ++launches;
                    }
                } else if (plain) {
                    // One pair per launch: a one-CTA grid over a one-pair chunk.
                    for (size_t k = 0; k < G.chunks.size(); ++k) {
                        DpArgs gk = g;
                        gk.chunks = ctx->dChunks.p + G.chunkBase + k;
                        gk.nChunks = 1;
                        gk.chunkCounter = ctx->dCounter.p + kNumShapes + G.chunkBase + k;
                        G.kern<<<1, G.warps * kLanes, G.smem, ctx->stream>>>(gk, G.gt ? 0 : kNumCodes * G.maxRowPad);
                        ++launches;
                    }
                } else {
                    DpArgs gk = g;
                    gk.chunks = (search ? ctx->dMidChunks.p : ctx->dChunks.p) + G.chunkBase;
                    gk.nChunks = (int)G.chunks.size();
                    gk.chunkCounter = ctx->dCounter.p + (search ? kNumShapes : 0) + gi;
                    if (search) gk.pairIdx = ctx->dSurvivors.p;
                    G.kern<<<G.grid, G.warps * kLanes, G.smem, ctx->stream>>>(gk, G.gt ? 0 : kNumCodes * G.maxRowPad);
                    ++launches;
                }
                CK(cudaGetLastError(), "DP kernel");
            }
        }
        CK(record(S.ev[2]), "event");
        if (exactOnDevice) {
            flagKernel<<<(int)((n + 255) / 256), 256, 0, ctx->stream>>>(S.dOut.p, (int)n, forceExact ? 1 : 0,
                                                                        S.dQueue.p, S.dQueueCount.p,
                                                                        search ? S.dMask.p : nullptr);
            CK(cudaGetLastError(), "flag kernel");
            ++launches;
            queueSortKernel<<<1, 1024, 0, ctx->stream>>>(S.dQueue.p, S.dQueueCount.p, S.dPairs.p);
            CK(cudaGetLastError(), "queue sort kernel");
            ++launches;
        }
        return DMST_OK;
    };
    if ((mode & DMST_MODE_GRAPH) && !plain && !nullOnly && !sequentialExact && !search) {
        // Replay the captured graph when the launch shape and the buffers are
        // those of the last capture; otherwise capture again and update the
        // executable graph (or instantiate a new one).
        std::vector<uintptr_t> key = {(uintptr_t)nCounters, (uintptr_t)nj, (uintptr_t)nullBlocks,
                                      (uintptr_t)forceExact, (uintptr_t)ctx->dCounter.p, (uintptr_t)ctx->dNullJobs.p,
                                      (uintptr_t)ctx->dNullJobPairs.p, (uintptr_t)S.dPairs.p,
                                      (uintptr_t)ctx->dProfiles.p, (uintptr_t)ctx->dCodes.p, (uintptr_t)S.dSeeds.p,
                                      (uintptr_t)ctx->dNullTmp.p, (uintptr_t)ctx->dNullTmpOff.p,
                                      (uintptr_t)S.dScales.p, (uintptr_t)ctx->dEmit.p, (uintptr_t)ctx->dParams.p,
                                      (uintptr_t)ctx->dW1.p, (uintptr_t)ctx->dRing.p, (uintptr_t)S.dOut.p,
                                      (uintptr_t)ctx->dChunks.p, (uintptr_t)w1Slot, (uintptr_t)ringSlot,
                                      (uintptr_t)n, (uintptr_t)exactOnDevice, (uintptr_t)forceExact,
                                      (uintptr_t)exactGrid, (uintptr_t)poolSlot, (uintptr_t)ctx->dExactPool.p,
                                      (uintptr_t)exactGroups,
                                      (uintptr_t)S.dExOut.p, (uintptr_t)S.dQueue.p, (uintptr_t)S.dQueueCount.p,
                                      (uintptr_t)S.hOut.p, (uintptr_t)S.hExOut.p};
        for (const Group &G : groups) {
            const uintptr_t v[8] = {(uintptr_t)G.kern, (uintptr_t)G.grid,         (uintptr_t)G.warps,
                                    (uintptr_t)G.smem, (uintptr_t)G.chunks.size(), (uintptr_t)G.chunkBase,
                                    (uintptr_t)G.maxRowPad, (uintptr_t)G.kernWarps};
            key.insert(key.end(), v, v + 8);
        }
        if (!S.graphExec || key != S.graphKey) {
            cudaGraph_t graph = nullptr;
            CK(cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal), "begin capture");
            capturing = true;
            const int st = enqueue();
            capturing = false;
            const cudaError_t ce = cudaStreamEndCapture(ctx->stream, &graph);
            if (st) {
                if (graph) cudaGraphDestroy(graph);
                return st;
            }
            CK(ce, "end capture");
            if (S.graphExec) {
                cudaGraphExecUpdateResultInfo info;
                if (cudaGraphExecUpdate(S.graphExec, graph, &info) != cudaSuccess) {
                    cudaGetLastError();
                    cudaGraphExecDestroy(S.graphExec);
                    S.graphExec = nullptr;
                }
            }
            cudaError_t ie = cudaSuccess;
            if (!S.graphExec) ie = cudaGraphInstantiate(&S.graphExec, graph, 0);
            cudaGraphDestroy(graph);
            CK(ie, "instantiate graph");
            S.graphKey = key;
            S.graphLaunches = launches;
            ++ctx->graphCaptures;
        }
        CK(cudaGraphLaunch(S.graphExec, ctx->stream), "graph launch");
        launches = S.graphLaunches;
    } else {
        const int st = enqueue();
        if (st) return st;
    }
    // The exact path and the result copies go on the second stream, after the
    // flag kernel, when the exact path is expected to leave SMs idle (the
    // previous call flagged fewer pairs than three quarters of the SMs, each
    // pair taking one CTA): the next call's null model and DP kernels (first
    // stream) then fill them.  A larger exact path keeps the stream order.
    const bool overlapExact = exactOnDevice && !align && ctx->lastFlagged * 4 < ctx->smCount * 3;
    cudaStream_t tail = overlapExact ? ctx->stream2 : ctx->stream;
    if (exactOnDevice) {
        if (overlapExact) {
            CK(cudaEventRecord(S.evFork, ctx->stream), "event");
            CK(cudaStreamWaitEvent(ctx->stream2, S.evFork, 0), "stream dependency");
        }
        auto ek = exactGroups == 2
                      ? (align ? exactWaveKernel<true, true, 2>
                               : (anchors ? exactWaveKernel<true, false, 2> : exactWaveKernel<false, false, 2>))
                      : (align ? exactWaveKernel<true, true> : (anchors ? exactWaveKernel<true> : exactWaveKernel<false>));
        ek<<<exactGrid, kPipeWarps * kLanes, kPipeWarps * sizeof(Window), tail>>>(
            S.dQueue.p, S.dQueueCount.p, S.dPairs.p, ctx->dProfiles.p, ctx->dEmit.p, ctx->dParams.p,
            ctx->dCodes.p, S.dSeeds.p, S.dScales.p, ctx->dExactPool.p, poolSlot, S.dExOut.p,
            anchors ? S.dAnchorOff.p : nullptr, S.dAnchorM.p, S.dAnchorE.p, S.dAnchorRow.p,
            align ? ctx->dAlignJobOf.p : nullptr, align ? ctx->dAlignJobs.p : nullptr,
            align ? ctx->dAlignCells.p : nullptr, align ? ctx->dAlignRows.p : nullptr, ctx->waitLimit);
        CK(cudaGetLastError(), "exact kernel");
        ++launches;
    }
    CK(cudaEventRecord(S.ev[3], tail), "event");
    if (!nullOnly) {
        CK(cudaMemcpyAsync(S.hOut.p, S.dOut.p, n * sizeof(PairOut), cudaMemcpyDeviceToHost, tail),
           "download results");
        if (exactOnDevice)
            CK(cudaMemcpyAsync(S.hExOut.p, S.dExOut.p, n * sizeof(ExactOut), cudaMemcpyDeviceToHost, tail),
               "download exact results");
        if (anchors) {
            CK(cudaMemcpyAsync(S.hAnchorM.p, S.dAnchorM.p, anchorCols * sizeof(float), cudaMemcpyDeviceToHost,
                               tail),
               "download anchors");
            CK(cudaMemcpyAsync(S.hAnchorE.p, S.dAnchorE.p, anchorCols * sizeof(int), cudaMemcpyDeviceToHost, tail),
               "download anchors");
            CK(cudaMemcpyAsync(S.hAnchorRow.p, S.dAnchorRow.p, anchorCols * sizeof(int), cudaMemcpyDeviceToHost,
                               tail),
               "download anchors");
        }
        if (search) {
            CK(cudaMemcpyAsync(S.hOutF.p, S.dOutF.p, n * sizeof(PairOut), cudaMemcpyDeviceToHost, tail),
               "download filter results");
            CK(cudaMemcpyAsync(S.hMask.p, S.dMask.p, n, cudaMemcpyDeviceToHost, tail), "download survivors");
        }
    }
    CK(cudaEventRecord(S.ev[4], tail), "event");
    S.pending = true;
    S.n = n;
    S.mode = mode;
    S.mid = mid;
    S.nullOnly = nullOnly;
    S.sequentialExact = sequentialExact;
    S.exactOnDevice = exactOnDevice;
    S.search = search;
    S.anchorBest = anchorBest;
    S.anchorRowOut = anchorRow;
    S.anchorCols = anchorCols;
    S.out = out;
    S.order.swap(order);
    S.dp.swap(dp);
    S.launches = launches;
    S.t0 = hostT0;
    ctx->nextSlot = si ^ 1;
    return DMST_OK;
}

// Waits for the oldest pending call and writes its results.
static int completeCall(dmst_ctx *ctx) {
    const int si = ctx->oldest;
    CallSlot &S = ctx->slot[si];
    if (!S.pending) return DMST_OK;
    S.pending = false;
    ctx->oldest = si ^ 1;
    ctx->lastSlot = si;
    ctx->lastOrder = S.order;
    const size_t n = S.n;
    const bool mid = S.mid, nullOnly = S.nullOnly;
    const bool forceExact = (S.mode & (DMST_MODE_FORCE_EXACT | DMST_MODE_EXACT_SEQUENTIAL)) != 0;
    const std::vector<int> &order = S.order;
    const std::vector<DevPair> &dp = S.dp;
    dmst_result *out = S.out;
    int launches = S.launches;
    const auto hostT0 = S.t0;
    ctx->lastHostMs = S.hostMs;
    ctx->lastExactMs = 0;
    ctx->lastExactPairs = 0;
    CK(cudaEventSynchronize(S.ev[4]), "scoring kernels");
    if (nullOnly) {
        ctx->lastNullMs = elapsedMs(ctx, S.ev[0], S.ev[1]);
        ctx->lastDpMs = 0;
        ctx->lastTotalMs = ctx->lastNullMs;
        ctx->lastLaunches = launches;
        return DMST_OK;
    }
    const PairOut *po = S.hOut.p;
    const bool search = S.search;
    const uint8_t *survived = search ? S.hMask.p : nullptr;
    const PairOut *pf = search ? S.hOutF.p : nullptr;
    // Pairs outside the fast path's exact range go to the row-rescaled kernel.
    std::vector<int> flagged;
    for (size_t k = 0; k < n; ++k) {
        if (!mid || (survived && !survived[k])) continue;
        const PairOut &o = po[k];
        const bool ok = !forceExact && o.maxYb <= kRescaleThresh && o.maxFw <= kRescaleThresh &&
                        o.mid < INFINITY && o.filt < INFINITY && o.mid >= 0x1p-100f;
        if (!ok) flagged.push_back((int)k);
    }
    std::vector<ExactOut> eo;
    float exactMs = 0;
    if (S.exactOnDevice) {
        exactMs = elapsedMs(ctx, S.ev[2], S.ev[3]);
        eo.resize(flagged.size());
        for (size_t f = 0; f < flagged.size(); ++f) eo[f] = S.hExOut.p[flagged[f]];
    } else if (!flagged.empty()) {
        // The one-thread-per-pair restatement (DMST_MODE_EXACT_SEQUENTIAL), in
        // batches under a scratch budget.
        size_t free = 0, total = 0;
        cudaMemGetInfo(&free, &total);
        const size_t budget = std::max<size_t>(free / 2, (size_t)256 << 20);
        eo.resize(flagged.size());
        CK(cudaEventRecord(ctx->ev[3], ctx->stream), "event");
        size_t i0 = 0;
        while (i0 < flagged.size()) {
            std::vector<ExactJob> jobs;
            long long used = 0;
            size_t i1 = i0;
            while (i1 < flagged.size()) {
                const DevPair &d = dp[flagged[i1]];
                long long need = (exactScratchFloats(d.M, d.L) + 63) / 64 * 64;
                if (i1 > i0 && (size_t)(used + need) * 4 > budget) break;
                jobs.push_back(ExactJob{flagged[i1], used});
                used += need;
                ++i1;
            }
            const size_t nj = i1 - i0;
            CK(ctx->dExactScratch.ensure((size_t)used, 0.5), "alloc exact scratch");
            CK(ctx->dExactOut.ensure(nj), "alloc exact out");
            CK(ctx->dJobs.ensure(nj), "alloc exact jobs");
            CK(cudaMemcpyAsync(ctx->dJobs.p, jobs.data(), nj * sizeof(ExactJob), cudaMemcpyHostToDevice, ctx->stream),
               "upload jobs");
            const int tpb = 32;
            exactKernel<<<(int)((nj + tpb - 1) / tpb), tpb, 0, ctx->stream>>>(
                ctx->dJobs.p, (int)nj, S.dPairs.p, ctx->dProfiles.p, ctx->dEmit.p, ctx->dParams.p, ctx->dCodes.p,
                S.dSeeds.p, S.dScales.p, ctx->dExactScratch.p, ctx->dExactOut.p);
            CK(cudaGetLastError(), "exact kernel");
            ++launches;
            CK(cudaMemcpyAsync(eo.data() + i0, ctx->dExactOut.p, nj * sizeof(ExactOut), cudaMemcpyDeviceToHost,
                               ctx->stream),
               "download exact");
            CK(cudaStreamSynchronize(ctx->stream), "exact kernel");
            i0 = i1;
        }
        CK(cudaEventRecord(ctx->ev[4], ctx->stream), "event");
        CK(cudaEventSynchronize(ctx->ev[4]), "event");
        exactMs = elapsedMs(ctx, ctx->ev[3], ctx->ev[4]);
    }
    for (size_t f = 0; f < eo.size(); ++f)
        if (eo[f].failed)
            return ctx->fail(DMST_ETIMEOUT, "exact path: the stripe pipeline of pair %d gave up a wait",
                             order[flagged[f]]);
    ctx->lastExactMs = exactMs;
    ctx->lastExactPairs = (int)flagged.size();
    if (mid) ctx->lastFlagged = (int)flagged.size();

    float nullMs = 0, dpMs = 0;
    nullMs = elapsedMs(ctx, S.ev[0], S.ev[1]);
    dpMs = elapsedMs(ctx, S.ev[1], S.ev[2]);
    ctx->lastNullMs = nullMs;
    ctx->lastDpMs = dpMs;
    ctx->lastTotalMs = nullMs + dpMs + exactMs;
    ctx->lastLaunches = launches;

    const auto postT0 = std::chrono::steady_clock::now();
    std::vector<int> flagAt(n, -1);
    for (size_t f = 0; f < flagged.size(); ++f) flagAt[flagged[f]] = (int)f;
    for (size_t k = 0; k < n; ++k) {
        dmst_result &r = out[order[k]];
        std::memset(&r, 0, sizeof r);
        if (search && !survived[k]) {  // filtered out: the filter wave's score only
            const float f = pf[k].filt;
            r.filter_f = f;
            r.filter_ln = std::log((double)f);
            r.mid_ln = -INFINITY;
        } else if (mid) {
            if (flagAt[k] >= 0) {
                scoreToResult(eo[flagAt[k]].mid, &r.mid, &r.mid_ln);
                scoreToResult(eo[flagAt[k]].filt, &r.filter, &r.filter_ln);
                r.flags |= DMST_RES_EXACT_PATH;
            } else {
                fillResult(r, po[k].mid, false, &r.mid, &r.mid_ln);
                fillResult(r, po[k].filt, false, &r.filter, &r.filter_ln);
            }
            r.filter_f = po[k].filt;
            if (search) {
                r.filter_f = pf[k].filt;  // the float filter of the first wave
                r.flags |= DMST_RES_SURVIVOR;
            }
        } else {
            const float f = po[k].filt;
            r.filter_f = f;
            r.filter_ln = std::log((double)f);
            r.mid_ln = -INFINITY;
        }
    }
    if (S.anchorBest) {
        for (long long c = 0; c < S.anchorCols; ++c) {
            S.anchorBest[c].m = S.hAnchorM.p[c];
            S.anchorBest[c].e = S.hAnchorE.p[c];
            S.anchorRowOut[c] = S.hAnchorRow.p[c];
        }
        S.anchorBest = nullptr;
        S.anchorRowOut = nullptr;
    }
    const auto endT = std::chrono::steady_clock::now();
    ctx->lastPostMs = std::chrono::duration<double, std::milli>(endT - postT0).count();
    ctx->lastWallMs = std::chrono::duration<double, std::milli>(endT - hostT0).count();
    return DMST_OK;
}

// Completes every pending call (before anything that changes what pending
// calls read: sequences, profiles, the shared buffers of another entry point).
static int drainCalls(dmst_ctx *ctx) {
    int first = DMST_OK;
    while (ctx->slot[ctx->oldest].pending) {
        const int st = completeCall(ctx);
        if (st && !first) first = st;
    }
    reapGraves();  // no call of this context is in flight
    return first;
}

int dmst_score_pairs_submit(dmst_ctx *ctx, const dmst_pair *pairs, size_t n, int mode, dmst_result *out) {
    const bool nullOnly = (mode & kModeNullOnly) != 0;
    if (!ctx || (n && (!pairs || (!out && !nullOnly)))) return DMST_EINVAL;
    ctx->lastTotalMs = ctx->lastDpMs = ctx->lastNullMs = ctx->lastExactMs = ctx->lastHostMs = 0;
    ctx->lastPostMs = ctx->lastWallMs = 0;
    ctx->lastLaunches = 0;
    ctx->lastExactPairs = 0;
    if (n == 0) return DMST_OK;
    // Modes that run the exact path on the host, or profiles to re-upload,
    // need the pending calls done first; otherwise a third call waits for
    // the oldest.
    if ((mode & DMST_MODE_EXACT_SEQUENTIAL) || ctx->profilesDirty) {
        const int st = drainCalls(ctx);
        if (st) return st;
    }
    if (ctx->slot[ctx->nextSlot].pending) {
        const int st = completeCall(ctx);
        if (st) return st;
    }
    const int st = submitCall(ctx, pairs, n, mode, out);
    if (st) {
        // a failed submit leaves nothing pending in its slot; drop the others' launches too
        drainCalls(ctx);
    }
    return st;
}

int dmst_search_submit(dmst_ctx *ctx, const dmst_pair *pairs, size_t n, const float *filter_min_best, int mode,
                       dmst_result *out) {
    if (!ctx || !filter_min_best || (n && (!pairs || !out))) return DMST_EINVAL;
    if ((mode & 0xff) != DMST_MODE_MID || (mode & (DMST_MODE_PLAIN | DMST_MODE_EXACT_SEQUENTIAL | kModeNullOnly)))
        return ctx->fail(DMST_EINVAL, "dmst_search: mode must be DMST_MODE_MID (with FORCE_EXACT or GRAPH at most)");
    ctx->lastTotalMs = ctx->lastDpMs = ctx->lastNullMs = ctx->lastExactMs = ctx->lastHostMs = 0;
    ctx->lastPostMs = ctx->lastWallMs = 0;
    ctx->lastLaunches = 0;
    ctx->lastExactPairs = 0;
    if (n == 0) return DMST_OK;
    if (ctx->profilesDirty) {
        const int st = drainCalls(ctx);
        if (st) return st;
    }
    if (ctx->slot[ctx->nextSlot].pending) {
        const int st = completeCall(ctx);
        if (st) return st;
    }
    const int st = submitCall(ctx, pairs, n, mode, out, filter_min_best);
    if (st) drainCalls(ctx);
    return st;
}

int dmst_search(dmst_ctx *ctx, const dmst_pair *pairs, size_t n, const float *filter_min_best, int mode,
                dmst_result *out) {
    if (!ctx) return DMST_EINVAL;
    int st = drainCalls(ctx);
    if (st) return st;
    ctx->nextSlot = ctx->oldest = 0;
    st = dmst_search_submit(ctx, pairs, n, filter_min_best, mode, out);
    if (st || n == 0) return st;
    return completeCall(ctx);
}

int dmst_anchors(dmst_ctx *ctx, const dmst_pair *pairs, size_t n, dmst_score *best, int *row, dmst_result *out) {
    if (!ctx || (n && (!pairs || !best || !row))) return DMST_EINVAL;
    int st = drainCalls(ctx);
    if (st) return st;
    ctx->nextSlot = ctx->oldest = 0;
    if (n == 0) return DMST_OK;
    std::vector<dmst_result> tmp;
    if (!out) {
        tmp.resize(n);
        out = tmp.data();
    }
    if (ctx->profilesDirty) {
        st = drainCalls(ctx);
        if (st) return st;
    }
    st = submitCall(ctx, pairs, n, DMST_MODE_MID, out, nullptr, best, row);
    if (st) {
        drainCalls(ctx);
        return st;
    }
    return completeCall(ctx);
}

// The traceback of the hit path.  The call's pairs are scored; the hits go,
// in batches whose traceback buffers fit half the free device memory, through
// the exact kernel (anchors, W0, W1 and rescale counts kept), the table
// kernels of dp_traceback.cuh, the reference's anchor sort on the host, the
// span pass over every candidate, the reference's sequential choice of
// anchors on the host (from the spans), and the store pass for the kept ones.
static size_t alignJobBytes(int M, int L) {
    const size_t cells = (size_t)(M + 1) * L;
    return cells * (8 + 8 + 8) + (size_t)L * (4 + 4 + 8 * kFlankArrays + 8 + 8 + 4 + sizeof(WalkSpan) + 2 * sizeof(Seg)) +
           (size_t)alignRowInts(M) * 4 + 256;
}

static bool lessScore(dmst_score a, dmst_score b) {  // scoreLess (dummest-score.hh:70-76)
    if (a.m == 0.0f) return b.m != 0.0f;
    if (b.m == 0.0f) return false;
    if (a.e != b.e) return a.e < b.e;
    return a.m < b.m;
}

int dmst_align(dmst_ctx *ctx, const dmst_pair *pairs, size_t n, dmst_result *out, size_t *n_alignments,
               size_t *n_segments) {
    if (!ctx || (n && !pairs) || !n_alignments || !n_segments) return DMST_EINVAL;
    int st = drainCalls(ctx);
    if (st) return st;
    using Clock = std::chrono::steady_clock;
    auto msSince = [](Clock::time_point t) {
        return std::chrono::duration<double, std::milli>(Clock::now() - t).count();
    };
    const auto tCall = Clock::now();
    double *tm = ctx->alignMs;
    for (int q = 0; q < 9; ++q) tm[q] = 0.0;
    ctx->nextSlot = ctx->oldest = 0;
    ctx->alignOut.clear();
    ctx->alignSegOut.clear();
    *n_alignments = *n_segments = 0;
    if (n == 0) return DMST_OK;
    std::vector<dmst_result> tmp;
    if (!out) {
        tmp.resize(n);
        out = tmp.data();
    }
    st = submitCall(ctx, pairs, n, DMST_MODE_MID, out);
    if (st) {
        drainCalls(ctx);
        return st;
    }
    if ((st = completeCall(ctx))) return st;
    tm[1] = msSince(tCall);
    tm[8] = ctx->lastLaunches;

    // hits: laneHit with a report (dummest-dp-forward.hh:262-274, :489-490);
    // the gate is normalizeScore((double)minProbRatio, 0)
    std::vector<int> hits;
    std::vector<dmst_score> gates;
    for (size_t k = 0; k < n; ++k) {
        if (!(pairs[k].min_prob_ratio >= 0.0f)) continue;
        dmst_score g{0.0f, 0};
        if (pairs[k].min_prob_ratio != 0.0f) {
            int ex = 0;
            const double m = std::frexp((double)pairs[k].min_prob_ratio, &ex);
            g = dmst_score{(float)m, ex};
        }
        if (out[k].mid.m != 0.0f && !lessScore(out[k].mid, g)) {
            hits.push_back((int)k);
            gates.push_back(g);
        }
    }
    tm[7] = (double)hits.size();
    if (hits.empty()) {
        tm[0] = msSince(tCall);
        return DMST_OK;
    }

    size_t freeB = 0, totalB = 0;
    CK(cudaMemGetInfo(&freeB, &totalB), "memory info");
    const size_t held = ctx->dAlignCells.cap * sizeof(float) + (ctx->dAlignX.cap + ctx->dAlignSuf.cap) * sizeof(XS);
    const size_t budget = std::max<size_t>((freeB + held) / 2, (size_t)256 << 20);
    NullRates nr;
    nr.single = (double)(ctx->rates.insert1 + ctx->rates.delete2);
    nr.dbl = (double)(ctx->rates.insert2 + ctx->rates.delete1);
    for (size_t b0 = 0; b0 < hits.size();) {
        // the batch: hits b0 .. b1-1
        size_t b1 = b0, bytes = 0;
        while (b1 < hits.size() && b1 - b0 < 65535) {
            const dmst_pair &pp = pairs[hits[b1]];
            const size_t jb = alignJobBytes(ctx->profiles[pp.profile].M, ctx->seqLen[pp.seq]);
            if (b1 > b0 && bytes + jb > budget) break;
            bytes += jb;
            ++b1;
        }
        const int nb = (int)(b1 - b0);
        std::vector<AlignJob> jobs(nb);
        std::vector<dmst_pair> bp(nb);
        long long cells = 0, cols = 0, rowsN = 0;
        int maxL = 0, maxM = 0;
        for (int j = 0; j < nb; ++j) {
            const dmst_pair &pp = pairs[hits[b0 + j]];
            bp[j] = pp;
            AlignJob &jb = jobs[j];
            jb.pair = j;
            jb.M = ctx->profiles[pp.profile].M;
            jb.L = ctx->seqLen[pp.seq];
            jb.nCand = 0;
            jb.cellOff = cells;
            jb.colOff = cols;
            jb.rowOff = rowsN;
            jb.minM = gates[b0 + j].m;
            jb.minE = gates[b0 + j].e;
            cells += (long long)(jb.M + 1) * jb.L;
            cols += jb.L;
            rowsN += alignRowInts(jb.M);
            maxL = std::max(maxL, jb.L);
            maxM = std::max(maxM, jb.M);
        }
        // headroom: calls whose hits differ a little reuse the buffers (a
        // reallocation synchronises the device and costs a cudaMalloc of GBs)
        CK(ctx->dAlignCells.ensure((size_t)cells * 2, 0.3), "alloc traceback tables");
        CK(ctx->dAlignX.ensure((size_t)cells, 0.3), "alloc traceback tables");
        CK(ctx->dAlignSuf.ensure((size_t)cells, 0.3), "alloc traceback tables");
        CK(ctx->dAlignRows.ensure((size_t)rowsN, 0.3), "alloc traceback rows");
        CK(ctx->dAlignColR.ensure((size_t)cols, 0.3), "alloc traceback columns");
        CK(ctx->dAlignColF.ensure((size_t)cols, 0.3), "alloc traceback columns");
        CK(ctx->dAlignWork.ensure((size_t)kFlankArrays * (cols + 4LL * nb), 0.3), "alloc traceback columns");
        CK(ctx->dAlignRev.ensure((size_t)cols, 0.3), "alloc traceback columns");
        CK(ctx->dAlignFwd.ensure((size_t)cols, 0.3), "alloc traceback columns");
        CK(ctx->dAlignCand.ensure((size_t)cols, 0.3), "alloc traceback columns");
        CK(ctx->dAlignSpan.ensure((size_t)cols, 0.3), "alloc traceback columns");

        // the exact path with the traceback stores, then the tables
        std::vector<dmst_score> best((size_t)cols);
        std::vector<int> row((size_t)cols);
        std::vector<dmst_result> bres(nb);
        const int si = ctx->nextSlot;
        auto tPhase = Clock::now();
        st = submitCall(ctx, bp.data(), nb, DMST_MODE_MID, bres.data(), nullptr, best.data(), row.data(), &jobs);
        if (st) {
            drainCalls(ctx);
            return st;
        }
        CallSlot &S = ctx->slot[si];
        sidesKernel<<<dim3((maxL + 127) / 128, nb), 128, 0, ctx->stream>>>(
            ctx->dAlignJobs.p, ctx->dAlignCells.p, ctx->dAlignRows.p, ctx->dAlignColR.p, ctx->dAlignColF.p);
        flankPrepKernel<<<dim3((maxL + 4 + 127) / 128, nb), 128, 0, ctx->stream>>>(
            ctx->dAlignJobs.p, S.dPairs.p, ctx->dProfiles.p, ctx->dCodes.p, S.dSeeds.p, S.dScales.p, nr,
            ctx->dAlignColR.p, ctx->dAlignColF.p, ctx->dAlignRows.p, ctx->dAlignWork.p);
        flankChainKernel<<<nb, 96, 0, ctx->stream>>>(ctx->dAlignJobs.p, S.dScales.p, nr, ctx->dAlignWork.p);
        flankUnifyKernel<<<dim3((maxL + 127) / 128, nb), 128, 0, ctx->stream>>>(ctx->dAlignJobs.p, S.dScales.p, nr,
                                                                                 ctx->dAlignWork.p);
        flankSumKernel<<<nb, 64, 0, ctx->stream>>>(ctx->dAlignJobs.p, ctx->dAlignWork.p, ctx->dAlignRows.p,
                                                   ctx->dAlignRev.p, ctx->dAlignFwd.p);
        xTableKernel<<<dim3((maxL + 127) / 128, (maxM + 1 + kXRows - 1) / kXRows, nb), 128, 0, ctx->stream>>>(
            ctx->dAlignJobs.p, S.dPairs.p, ctx->dProfiles.p, ctx->dEmit.p, ctx->dParams.p, ctx->dCodes.p, S.dScales.p,
            ctx->dAlignCells.p, ctx->dAlignRows.p, ctx->dAlignX.p);
        optimalKernel<<<nb, kOptThreads, 0, ctx->stream>>>(ctx->dAlignJobs.p, ctx->dAlignCells.p, ctx->dAlignRows.p,
                                                          ctx->dAlignX.p, ctx->dAlignRev.p, ctx->dAlignFwd.p,
                                                          ctx->dAlignSuf.p);
        CK(cudaGetLastError(), "traceback table kernels");
        if ((st = completeCall(ctx))) return st;
        CK(cudaStreamSynchronize(ctx->stream), "traceback tables");
        tm[2] += msSince(tPhase);
        tm[8] += ctx->lastLaunches + 7;  // the traceback call's, then sides, 4 flank, X and optimal kernels
        tPhase = Clock::now();

        // The reference's sort of each hit's anchors (std::ranges::sort with
        // std::greater<>, dummest-dp-forward.hh:494, which libstdc++ runs as
        // std::sort with the same comparisons): every column, zero columns as
        // placeholders; the candidates are the leading entries at or above the
        // gate.  Entries below the gate sort after every passing one, so the
        // passing entries alone, sorted, are the candidates in order unless two
        // of them are equal scores: then where the reference's sort puts the
        // tied ones depends on all L entries, and the full sort runs.  Hits are
        // shared among host threads.
        struct Entry {
            dmst_score pair;
            int col;
        };
        std::vector<int> cand((size_t)cols);
        auto sortJob = [&](int j, std::vector<Entry> &ent) {
            AlignJob &jb = jobs[j];
            const dmst_score g{jb.minM, jb.minE};
            auto greater = [](const Entry &x, const Entry &y) { return lessScore(y.pair, x.pair); };
            ent.clear();
            for (int c = 0; c < jb.L; ++c) {
                const dmst_score a = best[jb.colOff + c];
                if (a.m != 0.0f && !lessScore(a, g)) ent.push_back(Entry{a, c});
            }
            std::sort(ent.begin(), ent.end(), greater);
            bool tie = false;
            for (size_t q = 1; q < ent.size() && !tie; ++q)
                tie = ent[q].pair.m == ent[q - 1].pair.m && ent[q].pair.e == ent[q - 1].pair.e;
            if (tie) {
                ent.resize(jb.L);
                for (int c = 0; c < jb.L; ++c) {
                    const dmst_score a = best[jb.colOff + c];
                    ent[c] = a.m != 0.0f ? Entry{a, c} : Entry{dmst_score{0.0f, 0}, 0};
                }
                std::sort(ent.begin(), ent.end(), greater);
            }
            int nc = 0;
            while (nc < (int)ent.size() && ent[nc].pair.m != 0.0f && !lessScore(ent[nc].pair, g)) {
                cand[jb.colOff + nc] = ent[nc].col;
                ++nc;
            }
            jb.nCand = nc;
        };
        {
            const int nt = std::max(1, std::min<int>((int)std::thread::hardware_concurrency(), nb / 8));
            std::atomic<int> next{0};
            auto worker = [&]() {
                std::vector<Entry> ent;
                for (int j; (j = next.fetch_add(1)) < nb;) sortJob(j, ent);
            };
            std::vector<std::thread> pool;
            for (int q = 1; q < nt; ++q) pool.emplace_back(worker);
            worker();
            for (auto &th : pool) th.join();
        }
        tm[3] += msSince(tPhase);
        tPhase = Clock::now();
        int maxCand = 1;
        for (const AlignJob &jb : jobs) maxCand = std::max(maxCand, jb.nCand);
        CK(cudaMemcpyAsync(ctx->dAlignJobs.p, jobs.data(), nb * sizeof(AlignJob), cudaMemcpyHostToDevice,
                           ctx->stream),
           "upload traceback jobs");
        CK(cudaMemcpyAsync(ctx->dAlignCand.p, cand.data(), (size_t)cols * sizeof(int), cudaMemcpyHostToDevice,
                           ctx->stream),
           "upload traceback candidates");
        spanKernel<<<dim3((maxCand + 127) / 128, nb), 128, 0, ctx->stream>>>(
            ctx->dAlignJobs.p, ctx->dAlignCand.p, S.dAnchorRow.p, ctx->dAlignCells.p, ctx->dAlignX.p,
            ctx->dAlignSuf.p, ctx->dAlignRev.p, ctx->dAlignFwd.p, ctx->dAlignSpan.p);
        CK(cudaGetLastError(), "traceback span kernel");
        std::vector<WalkSpan> spans((size_t)cols);
        CK(cudaMemcpyAsync(spans.data(), ctx->dAlignSpan.p, (size_t)cols * sizeof(WalkSpan), cudaMemcpyDeviceToHost,
                           ctx->stream),
           "download traceback spans");
        CK(cudaStreamSynchronize(ctx->stream), "traceback spans");
        tm[4] += msSince(tPhase);
        tPhase = Clock::now();

        // The reference's choice (dummest-dp-forward.hh:497-531): in sorted
        // order, an anchor inside a kept alignment is skipped, and one whose
        // clamped span meets a kept alignment's columns is dropped; the rest
        // are kept and mark their columns.  marked[] holds prefix counts of
        // the marked columns, rebuilt when a kept span marks some.
        std::vector<WalkItem> items;
        std::vector<uint8_t> mark;
        std::vector<int> marked;
        long long ng = 0;
        for (int j = 0; j < nb; ++j) {
            const AlignJob &jb = jobs[j];
            mark.assign(jb.L, 0);
            marked.assign(jb.L + 1, 0);
            for (int c = 0; c < jb.nCand; ++c) {
                const int a2 = cand[jb.colOff + c];
                if (mark[a2]) continue;
                const WalkSpan &w = spans[jb.colOff + c];
                const int beg = std::max(w.beg, 0), end = std::min(w.end, jb.L);
                if (beg < end && marked[end] - marked[beg] > 0) continue;
                if (beg < end) {
                    std::fill(mark.begin() + beg, mark.begin() + end, (uint8_t)1);
                    for (int q = 0; q < jb.L; ++q) marked[q + 1] = marked[q] + mark[q];
                }
                const int n = w.nf + w.nr;
                dmst_alignment o;
                o.pair = hits[b0 + j];
                o.score = best[jb.colOff + a2];
                o.ln_score = scoreLn(o.score.m, o.score.e);
                o.anchor1 = row[jb.colOff + a2];
                o.anchor2 = a2;
                o.seg_begin = (long long)ctx->alignSegOut.size() + ng;
                o.seg_count = n;
                o.pad = 0;
                ctx->alignOut.push_back(o);
                if (n > 0) items.push_back(WalkItem{j, a2, w.nr, 0, ng});
                ng += n;
            }
        }
        tm[5] += msSince(tPhase);
        tPhase = Clock::now();
        if (!items.empty()) {
            CK(ctx->dAlignItems.ensure(items.size(), 0.3), "alloc traceback output");
            CK(ctx->dAlignSegOut.ensure((size_t)ng, 0.3), "alloc traceback output");
            CK(cudaMemcpyAsync(ctx->dAlignItems.p, items.data(), items.size() * sizeof(WalkItem),
                               cudaMemcpyHostToDevice, ctx->stream),
               "upload traceback walks");
            storeWalkKernel<<<(int)((items.size() + 127) / 128), 128, 0, ctx->stream>>>(
                ctx->dAlignJobs.p, ctx->dAlignItems.p, (int)items.size(), S.dAnchorRow.p, ctx->dAlignCells.p,
                ctx->dAlignX.p, ctx->dAlignSuf.p, ctx->dAlignRev.p, ctx->dAlignFwd.p, ctx->dAlignSegOut.p);
            CK(cudaGetLastError(), "traceback store kernel");
            const size_t first = ctx->alignSegOut.size();
            ctx->alignSegOut.resize(first + (size_t)ng);
            static_assert(sizeof(Seg) == sizeof(dmst_segment), "segment layout");
            CK(cudaMemcpyAsync(ctx->alignSegOut.data() + first, ctx->dAlignSegOut.p, (size_t)ng * sizeof(Seg),
                               cudaMemcpyDeviceToHost, ctx->stream),
               "download segments");
            CK(cudaStreamSynchronize(ctx->stream), "traceback segments");
        }
        tm[6] += msSince(tPhase);
        tm[8] += 1 + (items.empty() ? 0 : 1);  // span and store passes
        b0 = b1;
    }
    *n_alignments = ctx->alignOut.size();
    *n_segments = ctx->alignSegOut.size();
    tm[0] = msSince(tCall);
    return DMST_OK;
}

int dmst_last_align_timing(const dmst_ctx *ctx, double *out, int n) {
    if (!ctx || !out || n < 0) return DMST_EINVAL;
    for (int i = 0; i < n && i < 9; ++i) out[i] = ctx->alignMs[i];
    return DMST_OK;
}

int dmst_align_fetch(const dmst_ctx *ctx, dmst_alignment *alignments, size_t cap_alignments, dmst_segment *segments,
                     size_t cap_segments) {
    if (!ctx) return DMST_EINVAL;
    const size_t na = ctx->alignOut.size(), ns = ctx->alignSegOut.size();
    if (cap_alignments < na || cap_segments < ns) return DMST_ERANGE;
    if ((na && !alignments) || (ns && !segments)) return DMST_EINVAL;
    if (na) std::memcpy(alignments, ctx->alignOut.data(), na * sizeof(dmst_alignment));
    if (ns) std::memcpy(segments, ctx->alignSegOut.data(), ns * sizeof(dmst_segment));
    return DMST_OK;
}

int dmst_filter_threshold(double lambda_filter, double k_filter, double total_length, double filter_evalue,
                          float *min_best) {
    if (!min_best || !(lambda_filter > 0) || !(k_filter > 0) || !(total_length > 0) || !(filter_evalue >= 0))
        return DMST_EINVAL;
    // The reference's gate for a float best b > 0 (dummest-search.hh:158-166):
    //   E(b) = K T / exp(log((double)b) * lambda) <= E_filter
    // E(b) decreases with b: the smallest passing float is found by bisection
    // over the positive floats' bit patterns (ordered like their values).
    auto passes = [&](float b) {
        const double lp = std::log((double)b);
        const double probRatio = std::exp(lp * lambda_filter);
        const double evalue = k_filter * total_length / probRatio;
        return evalue <= filter_evalue;
    };
    uint32_t lo = 1, hi = 0x7f7fffffu;  // smallest subnormal .. FLT_MAX
    float f;
    std::memcpy(&f, &hi, 4);
    if (!passes(f)) {
        *min_best = INFINITY;  // only +inf survives
        return DMST_OK;
    }
    std::memcpy(&f, &lo, 4);
    if (passes(f)) {
        *min_best = f;
        return DMST_OK;
    }
    while (hi - lo > 1) {  // passes(hi), !passes(lo)
        const uint32_t m = lo + (hi - lo) / 2;
        std::memcpy(&f, &m, 4);
        if (passes(f))
            hi = m;
        else
            lo = m;
    }
    std::memcpy(&f, &hi, 4);
    *min_best = f;
    return DMST_OK;
}

int dmst_score_pairs_complete(dmst_ctx *ctx) {
    if (!ctx) return DMST_EINVAL;
    return completeCall(ctx);
}

int dmst_pending_calls(const dmst_ctx *ctx) {
    return ctx ? (int)ctx->slot[0].pending + (int)ctx->slot[1].pending : 0;
}

int dmst_score_pairs(dmst_ctx *ctx, const dmst_pair *pairs, size_t n, int mode, dmst_result *out) {
    if (!ctx) return DMST_EINVAL;
    int st = drainCalls(ctx);
    if (st) return st;
    ctx->nextSlot = ctx->oldest = 0;  // nothing pending: synchronous calls share slot 0 (and its graph)
    st = dmst_score_pairs_submit(ctx, pairs, n, mode, out);
    if (st || n == 0) return st;
    return completeCall(ctx);
}

int dmst_last_timing_ex(const dmst_ctx *ctx, double *out, int n) {
    if (!ctx || !out || n < 0) return DMST_EINVAL;
    const double v[10] = {ctx->lastTotalMs, ctx->lastNullMs,      ctx->lastDpMs,
                          ctx->lastExactMs, ctx->lastHostMs,      (double)ctx->lastLaunches,
                          (double)ctx->lastExactPairs, ctx->lastPostMs, ctx->lastWallMs,
                          (double)ctx->graphCaptures};
    for (int i = 0; i < n && i < 10; ++i) out[i] = v[i];
    return DMST_OK;
}

int dmst_last_timing(const dmst_ctx *ctx, double *total_ms, double *dp_ms, double *null_ms, int *launches) {
    if (!ctx) return DMST_EINVAL;
    if (total_ms) *total_ms = ctx->lastTotalMs;
    if (dp_ms) *dp_ms = ctx->lastDpMs;
    if (null_ms) *null_ms = ctx->lastNullMs;
    if (launches) *launches = ctx->lastLaunches;
    return DMST_OK;
}

int dmst_set_wait_limit(dmst_ctx *ctx, int iterations) {
    if (!ctx || iterations < 0) return DMST_EINVAL;
    ctx->waitLimit = iterations;
    return DMST_OK;
}

int dmst_autotune(dmst_ctx *ctx, const dmst_pair *sample, size_t n, double *gcups6) {
    if (!ctx || !sample || n == 0) return DMST_EINVAL;
    for (size_t i = 0; i < n; ++i)
        if (sample[i].seq < 0 || sample[i].seq >= (int)ctx->seqLen.size() || sample[i].profile < 0 ||
            sample[i].profile >= (int)ctx->profiles.size())
            return ctx->fail(DMST_EINVAL, "autotune sample pair %zu: unknown sequence or profile id", i);
    // The sample's pairs by read length class; every shape is timed on each.
    std::vector<dmst_pair> cls[2];
    for (size_t i = 0; i < n; ++i) cls[lengthClass(ctx->seqLen[sample[i].seq])].push_back(sample[i]);
    Tuning t = ctx->tune;
    for (int c = 0; c < 2; ++c) {
        const std::vector<dmst_pair> &sub = cls[c];
        if (sub.empty()) continue;
        std::vector<dmst_result> res(sub.size());
        for (int q = 0; q < kNumR; ++q) {
            const int R = kShapeR[q];
            double padded = 0;
            for (const dmst_pair &pp : sub)
                padded += (double)paddedRows(ctx->profiles[pp.profile].M, R) * ctx->seqLen[pp.seq];
            double bestRate = 0;
            for (int w = 0; w < 3; ++w) {
                ctx->tune.forceR = R;
                ctx->tune.forceWarps = kShapeWarps[w];
                double ms = 0;
                int st = DMST_OK;
                for (int rep = 0; rep < 2 && st == DMST_OK; ++rep) {  // the first run warms up
                    st = dmst_score_pairs(ctx, sub.data(), sub.size(), DMST_MODE_MID, res.data());
                    ms = ctx->lastDpMs;
                }
                ctx->tune.forceR = ctx->tune.forceWarps = 0;
                if (st) {
                    ctx->tune = t;
                    return st;
                }
                const double rate = ms > 0 ? padded / ms : 0;  // padded cells per ms
                t.rates[c][q][w] = rate;
                if (rate > bestRate) {
                    bestRate = rate;
                    t.warps[c][q] = kShapeWarps[w];
                }
            }
            t.rate[c][q] = bestRate;
        }
    }
    // a class the sample does not have takes the other's shapes
    for (int c = 0; c < 2; ++c)
        if (cls[c].empty()) {
            std::memcpy(t.warps[c], t.warps[1 - c], sizeof t.warps[c]);
            std::memcpy(t.rate[c], t.rate[1 - c], sizeof t.rate[c]);
            std::memcpy(t.rates[c], t.rates[1 - c], sizeof t.rates[c]);
        }
    if (gcups6) {
        const int qs[3] = {rIndex(4), rIndex(2), rIndex(1)};
        for (int i = 0; i < 3; ++i)
            for (int w = 0; w < 2; ++w) gcups6[i * 2 + w] = t.rates[0][qs[i]][w] / 1e6;
    }
    t.tuned = true;
    t.forceR = t.forceWarps = 0;
    ctx->tune = t;
    return DMST_OK;
}

int dmst_tuned_rates(const dmst_ctx *ctx, double *gcups9) {
    if (!ctx || !gcups9) return DMST_EINVAL;
    const int qs[3] = {rIndex(4), rIndex(2), rIndex(1)};
    for (int i = 0; i < 3; ++i)
        for (int w = 0; w < 3; ++w) gcups9[i * 3 + w] = ctx->tune.rates[0][qs[i]][w] / 1e6;
    return DMST_OK;
}

int dmst_tuned_rates_ex(const dmst_ctx *ctx, double *gcups, int n) {
    if (!ctx || !gcups || n < 0 || n > 2 * kNumShapes) return DMST_EINVAL;
    for (int i = 0; i < n; ++i) {
        const int c = i / kNumShapes, k = i % kNumShapes;
        gcups[i] = ctx->tune.rates[c][k / 3][k % 3] / 1e6;
    }
    return DMST_OK;
}

// The adjoint kernel over n pairs of one profile: log T per pair, the summed
// gradient of log T (Params then emissions) and, if post is given, each
// pair's posterior tables at the offsets of dmst_posteriors.
static int runAdjoint(dmst_ctx *ctx, const dmst_pair *pairs, size_t n, double *log_t, double *grad_params,
                      double *grad_emit, double *post, const char *what, double *colPost = nullptr,
                      int *colRow = nullptr, double *rowMatch = nullptr) {
    if (!ctx || !pairs || n == 0 || (n >> 31)) return DMST_EINVAL;
    // The kernel writes the posterior tables (device) when the caller wants
    // them (post, host) or a reduction of them (the summary outputs).
    const bool summary = colPost || colRow || rowMatch;
    const bool tables = post || summary;
    const int prof = pairs[0].profile;
    for (size_t i = 0; i < n; ++i)
        if (pairs[i].profile != prof)
            return ctx->fail(DMST_EINVAL, "%s: pair %zu is for another profile (one profile per call)", what, i);
    // Pair descriptors, null models and seeds on the device, sorted longest
    // read first.
    const auto wallT0 = std::chrono::steady_clock::now();
    int st = dmst_score_pairs(ctx, pairs, n, DMST_MODE_MID | kModeNullOnly, nullptr);
    if (st) return st;
    CallSlot &S = ctx->slot[ctx->lastSlot];  // the pairs, seeds and scales of that call
    const double nullMs = elapsedMs(ctx, S.ev[0], S.ev[1]);
    double adjMs = 0.0;
    int launches = 1;
    const std::vector<int> order = ctx->lastOrder;
    const int M = ctx->profiles[prof].M;
    // Posterior offsets in the caller's order.
    std::vector<long long> postOff(n, -1);
    if (post) {
        long long o = 0;
        for (size_t i = 0; i < n; ++i) {
            postOff[i] = o;
            o += 2LL * (M + 1) * ctx->seqLen[pairs[i].seq];
        }
    }
    std::vector<AdjointJob> jobs(n);
    std::vector<long long> needF(n), needB(n), needP(n);
    // Batches of pairs under the device budget.  The full forward store is
    // 24 bytes per cell; the checkpointed one keeps the stripes' top rows and
    // a checkpoint every kAdjCk columns (about 1/12 of it) and recomputes.
    // Auto: the full store when every pair's fits the budget at once.
    size_t freeB = 0, totalB = 0;
    CK(cudaSetDevice(ctx->device), "set device");
    CK(cudaMemGetInfo(&freeB, &totalB), "memory info");
    const size_t held = (ctx->dAdjF.cap + ctx->dAdjB.cap + ctx->dPost.cap) * sizeof(double);
    const size_t budget = ctx->opts.device_budget_bytes ? ctx->opts.device_budget_bytes : (freeB + held) / 2;
    long long fullAll = 0;
    for (size_t k = 0; k < n; ++k) {
        const int L = ctx->seqLen[pairs[order[k]].seq];
        fullAll += ((adjStoreDoubles(M, L) + 31) & ~31LL) + adjBoundDoubles(L) + (tables ? 2LL * (M + 1) * L : 0);
    }
    const bool ckpt = ctx->adjCheckpoint == DMST_ADJ_CKPT_ON ||
                      (ctx->adjCheckpoint == DMST_ADJ_CKPT_AUTO && (size_t)fullAll * 8 > budget);
    ctx->lastAdjCheckpointed = ckpt;
    for (size_t k = 0; k < n; ++k) {
        const int L = ctx->seqLen[pairs[order[k]].seq];
        jobs[k] = AdjointJob{(int)k, 0, 0, 0, tables ? 0 : -1};
        // 256-byte aligned stores (cp.async)
        needF[k] = ((ckpt ? adjCkptDoubles(M, L) : adjStoreDoubles(M, L)) + 31) & ~31LL;
        needB[k] = adjBoundDoubles(L);
        needP[k] = tables ? 2LL * (M + 1) * L : 0;
    }
    const size_t gN = (size_t)(M + 2) * kParamFloats + (size_t)(M + 1) * kNumCodes;
    CK(ctx->dGrad.ensure(gN), "alloc gradient");
    CK(ctx->dLogT.ensure(n), "alloc log T");
    CK(ctx->dAdjJobs.ensure(n), "alloc adjoint jobs");
    CK(cudaMemsetAsync(ctx->dGrad.p, 0, gN * sizeof(double), ctx->stream), "zero gradient");
    // Summary outputs in the caller's order: pair i's columns at the sum of
    // the earlier pairs' lengths, its rows at i (M+1).
    std::vector<long long> colOff(n + 1, 0);
    for (size_t i = 0; i < n; ++i) colOff[i + 1] = colOff[i] + ctx->seqLen[pairs[i].seq];
    std::vector<PostSumJob> sumJobs;
    if (summary) {
        CK(ctx->dPostJobs.ensure(n), "alloc summary jobs");
        CK(ctx->dColPost.ensure((size_t)colOff[n]), "alloc column posteriors");
        CK(ctx->dColRow.ensure((size_t)colOff[n]), "alloc column rows");
        CK(ctx->dRowMatch.ensure(n * (size_t)(M + 1)), "alloc row sums");
        sumJobs.resize(n);
    }
    for (size_t k0 = 0; k0 < n;) {
        size_t k1 = k0;
        long long f = 0, b = 0, pp = 0;
        while (k1 < n && (k1 == k0 || (size_t)(f + needF[k1] + b + needB[k1] + pp + needP[k1]) * 8 <= budget)) {
            jobs[k1].fOff = f;
            jobs[k1].bOff = b;
            if (tables) jobs[k1].pOff = pp;
            f += needF[k1];
            b += needB[k1];
            pp += needP[k1];
            ++k1;
        }
        const int nj = (int)(k1 - k0);
        CK(ctx->dAdjF.ensure((size_t)f), "alloc adjoint store");
        CK(ctx->dAdjB.ensure((size_t)b), "alloc adjoint rows");
        if (tables) CK(ctx->dPost.ensure((size_t)std::max<long long>(pp, 1)), "alloc posterior tables");
        CK(cudaMemcpyAsync(ctx->dAdjJobs.p, jobs.data() + k0, nj * sizeof(AdjointJob), cudaMemcpyHostToDevice,
                           ctx->stream),
           "upload adjoint jobs");
        const int blocks = (nj + kAdjWarps - 1) / kAdjWarps;
        auto kern = ckpt ? (tables ? adjointKernel<true, true> : adjointKernel<false, true>)
                         : (tables ? adjointKernel<true> : adjointKernel<false>);
        CK(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kAdjSmem), "smem attribute");
        CK(cudaEventRecord(ctx->ev[3], ctx->stream), "event");
        kern<<<blocks, kAdjWarps * 32, kAdjSmem, ctx->stream>>>(
            ctx->dAdjJobs.p, nj, S.dPairs.p, ctx->dProfiles.p, ctx->dEmit.p, ctx->dParams.p, ctx->dCodes.p,
            S.dSeeds.p, S.dScales.p, ctx->dAdjF.p, ctx->dAdjB.p, ctx->dGrad.p, ctx->dLogT.p + k0,
            tables ? ctx->dPost.p : nullptr);
        CK(cudaGetLastError(), "adjoint kernel");
        ++launches;
        if (summary) {
            int maxL = 0;
            for (size_t k = k0; k < k1; ++k) {
                const int ci = order[k];
                const int L = ctx->seqLen[pairs[ci].seq];
                sumJobs[k] = PostSumJob{jobs[k].pOff, colOff[ci], (long long)ci * (M + 1), M, L};
                maxL = std::max(maxL, L);
            }
            CK(cudaMemcpyAsync(ctx->dPostJobs.p, sumJobs.data() + k0, nj * sizeof(PostSumJob),
                               cudaMemcpyHostToDevice, ctx->stream),
               "upload summary jobs");
            if (colPost || colRow) {
                postColumnKernel<<<dim3((maxL + kPostThreads - 1) / kPostThreads, nj), kPostThreads, 0, ctx->stream>>>(
                    ctx->dPostJobs.p, ctx->dPost.p, ctx->dColPost.p, ctx->dColRow.p);
                CK(cudaGetLastError(), "posterior column kernel");
                ++launches;
            }
            if (rowMatch) {
                const int rowsPer = kPostThreads / kLanes;
                postRowKernel<<<dim3((M + 1 + rowsPer - 1) / rowsPer, nj), kPostThreads, 0, ctx->stream>>>(
                    ctx->dPostJobs.p, ctx->dPost.p, ctx->dRowMatch.p);
                CK(cudaGetLastError(), "posterior row kernel");
                ++launches;
            }
        }
        CK(cudaEventRecord(ctx->ev[4], ctx->stream), "event");
        if (post)
            for (size_t k = k0; k < k1; ++k)
                CK(cudaMemcpyAsync(post + postOff[order[k]], ctx->dPost.p + jobs[k].pOff,
                                   (size_t)needP[k] * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream),
                   "download posterior tables");
        CK(cudaStreamSynchronize(ctx->stream), "adjoint kernel");
        adjMs += elapsedMs(ctx, ctx->ev[3], ctx->ev[4]);
        k0 = k1;
    }
    // Timing of the call: [1] null model, [2] adjoint kernels, [0] both.
    ctx->lastNullMs = nullMs;
    ctx->lastDpMs = adjMs;
    ctx->lastExactMs = 0;
    ctx->lastTotalMs = nullMs + adjMs;
    ctx->lastLaunches = launches;
    ctx->lastWallMs = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - wallT0).count();
    std::vector<double> g(gN), lt(n);
    CK(cudaMemcpy(g.data(), ctx->dGrad.p, gN * sizeof(double), cudaMemcpyDeviceToHost), "download gradient");
    CK(cudaMemcpy(lt.data(), ctx->dLogT.p, n * sizeof(double), cudaMemcpyDeviceToHost), "download log T");
    if (log_t)
        for (size_t k = 0; k < n; ++k) log_t[order[k]] = lt[k];
    if (grad_params) std::memcpy(grad_params, g.data(), (size_t)(M + 2) * kParamFloats * sizeof(double));
    if (grad_emit)
        std::memcpy(grad_emit, g.data() + (size_t)(M + 2) * kParamFloats, (size_t)(M + 1) * kNumCodes * sizeof(double));
    if (colPost)
        CK(cudaMemcpy(colPost, ctx->dColPost.p, (size_t)colOff[n] * sizeof(double), cudaMemcpyDeviceToHost),
           "download column posteriors");
    if (colRow)
        CK(cudaMemcpy(colRow, ctx->dColRow.p, (size_t)colOff[n] * sizeof(int), cudaMemcpyDeviceToHost),
           "download column rows");
    if (rowMatch)
        CK(cudaMemcpy(rowMatch, ctx->dRowMatch.p, n * (size_t)(M + 1) * sizeof(double), cudaMemcpyDeviceToHost),
           "download row sums");
    return DMST_OK;
}

int dmst_adjoint_checkpoint(dmst_ctx *ctx, int mode, int *last_checkpointed) {
    if (!ctx) return DMST_EINVAL;
    if (last_checkpointed) *last_checkpointed = ctx->lastAdjCheckpointed ? 1 : 0;
    if (mode < 0) return DMST_OK;  // query only
    if (mode != DMST_ADJ_CKPT_AUTO && mode != DMST_ADJ_CKPT_ON && mode != DMST_ADJ_CKPT_OFF) return DMST_EINVAL;
    ctx->adjCheckpoint = mode;
    return DMST_OK;
}

int dmst_loglik_grad(dmst_ctx *ctx, const dmst_pair *pairs, size_t n, double *log_t, double *grad_params,
                     double *grad_emit) {
    return runAdjoint(ctx, pairs, n, log_t, grad_params, grad_emit, nullptr, "dmst_loglik_grad");
}

int dmst_posteriors(dmst_ctx *ctx, const dmst_pair *pairs, size_t n, double *log_t, double *post) {
    if (!post) return DMST_EINVAL;
    return runAdjoint(ctx, pairs, n, log_t, nullptr, nullptr, post, "dmst_posteriors");
}

int dmst_posterior_summary(dmst_ctx *ctx, const dmst_pair *pairs, size_t n, double *log_t, double *col_post,
                           int *col_row, double *row_match) {
    if (!col_post && !col_row && !row_match) return DMST_EINVAL;
    return runAdjoint(ctx, pairs, n, log_t, nullptr, nullptr, nullptr, "dmst_posterior_summary", col_post, col_row,
                      row_match);
}

int dmst_tuned_shape(const dmst_ctx *ctx, int M, int *rows_per_lane, int *warps_per_cta) {
    if (!ctx || M < 1) return DMST_EINVAL;
    int R, W;
    shapeOf(M, kShortRead, ctx->opts.rows_per_lane, ctx->tune, R, W);  // reads of the long class
    if (rows_per_lane) *rows_per_lane = R;
    if (warps_per_cta) *warps_per_cta = W;
    return DMST_OK;
}

int dmst_null_model(dmst_ctx *ctx, int seq, int profile, float *prefix_seed, float *suffix_seed, float *scales3) {
    if (!ctx || seq < 0 || seq >= (int)ctx->seqLen.size() || profile < 0 || profile >= (int)ctx->profiles.size())
        return DMST_EINVAL;
    CK(cudaSetDevice(ctx->device), "set device");
    int st = drainCalls(ctx);
    if (st) return st;
    st = uploadProfiles(ctx);
    if (st) return st;
    DevPair d;
    d.codeOff = ctx->seqOff[seq];
    d.L = ctx->seqLen[seq];
    d.M = ctx->profiles[profile].M;
    d.prof = profile;
    d.R = 1;
    d.seedOff = 0;
    long long zero = 0;
    const int pairIndex = 0;
    const NullJob job{0, 1};
    CK(ctx->slot[0].dPairs.ensure(1), "alloc");
    CK(ctx->slot[0].dSeeds.ensure(2 * (size_t)d.L), "alloc");
    CK(ctx->dNullTmp.ensure((size_t)nullTmpEntries(d.L)), "alloc");
    CK(ctx->dNullTmpOff.ensure(1), "alloc");
    CK(ctx->dNullJobs.ensure(1), "alloc");
    CK(ctx->dNullJobPairs.ensure(1), "alloc");
    CK(ctx->slot[0].dScales.ensure(1), "alloc");
    CK(cudaMemcpy(ctx->slot[0].dPairs.p, &d, sizeof d, cudaMemcpyHostToDevice), "upload");
    CK(cudaMemcpy(ctx->dNullTmpOff.p, &zero, sizeof zero, cudaMemcpyHostToDevice), "upload");
    CK(cudaMemcpy(ctx->dNullJobs.p, &job, sizeof job, cudaMemcpyHostToDevice), "upload");
    CK(cudaMemcpy(ctx->dNullJobPairs.p, &pairIndex, sizeof pairIndex, cudaMemcpyHostToDevice), "upload");
    NullRates nr;
    nr.single = (double)(ctx->rates.insert1 + ctx->rates.delete2);
    nr.dbl = (double)(ctx->rates.insert2 + ctx->rates.delete1);
    nullModelKernel<<<1, kNullWarps * 32, 0, ctx->stream>>>(ctx->dNullJobs.p, 1, ctx->dNullJobPairs.p, ctx->slot[0].dPairs.p,
                                                           ctx->dProfiles.p, ctx->dCodes.p, ctx->slot[0].dSeeds.p,
                                                           ctx->dNullTmp.p, ctx->dNullTmpOff.p, ctx->slot[0].dScales.p, nr);
    CK(cudaGetLastError(), "null-model kernel");
    CK(cudaStreamSynchronize(ctx->stream), "null-model kernel");
    std::vector<float> s(2 * (size_t)d.L);
    PairScales sc;
    CK(cudaMemcpy(s.data(), ctx->slot[0].dSeeds.p, s.size() * 4, cudaMemcpyDeviceToHost), "download");
    CK(cudaMemcpy(&sc, ctx->slot[0].dScales.p, sizeof sc, cudaMemcpyDeviceToHost), "download");
    if (prefix_seed) std::memcpy(prefix_seed, s.data(), (size_t)d.L * 4);
    if (suffix_seed) std::memcpy(suffix_seed, s.data() + d.L, (size_t)d.L * 4);
    if (scales3) {
        scales3[0] = sc.s1;
        scales3[1] = sc.s2;
        scales3[2] = sc.sC;
    }
    return DMST_OK;
}

// ---------------------------------------------------------------------------
// Calibration
// ---------------------------------------------------------------------------
int dmst_estimate_gumbel(double *scores, int n, double seq_length, double *out8) {
    if (!scores || !out8 || n < 2) return DMST_EINVAL;
    estimateGumbel(scores, n, seq_length, out8);
    return DMST_OK;
}

int dmst_calibration_sequence(const float *letter_freqs, double bg_stop, double insert1, double insert2,
                              double delete1, double delete2, int trial, int sequence_length, int border,
                              char *letters) {
    if (!letter_freqs || !letters || sequence_length < 1 || border < 0 || trial < 0) return DMST_EINVAL;
    Rates r{(float)insert1, (float)insert2, (float)delete1, (float)delete2, 0.0f, (float)bg_stop};
    calibrationSequence(letter_freqs, (float)bg_stop, r, trial, sequence_length, border, letters);
    return DMST_OK;
}

int dmst_calibrate(dmst_ctx *ctx, int profile, int sequence_length, int border, int num_sequences, double *out4,
                   double *scores) {
    if (!ctx || profile < 0 || profile >= (int)ctx->profiles.size() || sequence_length < 1 || border < 0 ||
        num_sequences < 2 || !out4)
        return DMST_EINVAL;
    if (sequence_length + border < 3) return DMST_EINVAL;
    const HostProfile &hp = ctx->profiles[profile];
    // Letter frequencies = the background row the reference reads
    // (p.values + width * length + 4, dummest.cc:376 -> estimateK).
    const float *freqs = hp.values.data() + (size_t)kWidth * hp.M + 4;
    const int Ltot = sequence_length + border;
    std::vector<char> letters(Ltot);
    std::vector<uint8_t> codes((size_t)Ltot * num_sequences);
    std::vector<int64_t> off(num_sequences + 1);
    for (int t = 0; t < num_sequences; ++t) {
        calibrationSequence(freqs, ctx->rates.bgStop, ctx->rates, t, sequence_length, border, letters.data());
        decodeLetters(letters.data(), Ltot, codes.data() + (size_t)t * Ltot);
        off[t] = (int64_t)t * Ltot;
    }
    off[num_sequences] = (int64_t)num_sequences * Ltot;
    // Keep the caller's sequences: append, score, then drop ours.
    const size_t keepSeqs = ctx->seqLen.size();
    const long long keepBytes = ctx->codeBytes;
    int first = 0;
    int st = dmst_seqs_add_decoded(ctx, codes.data(), off.data(), num_sequences, &first);
    if (st) return st;
    std::vector<dmst_pair> pairs(num_sequences);
    for (int t = 0; t < num_sequences; ++t) pairs[t] = dmst_pair{first + t, profile, -2.0f};
    std::vector<dmst_result> res(num_sequences);
    st = dmst_score_pairs(ctx, pairs.data(), pairs.size(), DMST_MODE_MID, res.data());
    ctx->seqLen.resize(keepSeqs);
    ctx->seqOff.resize(keepSeqs);
    ctx->codeBytes = keepBytes;
    if (st) return st;
    std::vector<double> mids(num_sequences), flts(num_sequences);
    for (int t = 0; t < num_sequences; ++t) {
        mids[t] = res[t].mid_ln;
        flts[t] = res[t].filter_ln;
    }
    if (scores) {
        std::copy(mids.begin(), mids.end(), scores);
        std::copy(flts.begin(), flts.end(), scores + num_sequences);
    }
    double g[8];
    estimateGumbel(mids.data(), num_sequences, sequence_length, g);
    out4[0] = g[0];
    out4[1] = g[1];
    estimateGumbel(flts.data(), num_sequences, sequence_length, g);
    out4[2] = g[0];
    out4[3] = g[1];
    return DMST_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Null model without allocation.
//
// Some callers cannot allocate device memory at the point where they need a
// read's null-model seeds: a process whose device memory is already claimed
// by another pool (a framework's caching allocator holding nearly all HBM
// fails a fresh cudaMalloc), or a latency-bound caller whose other streams
// must not stall on cudaFree's implicit device synchronisation.  For them
// dmst_null_model_noalloc runs the same null-model kernel as dmst_null_model
// with the caller's device buffers for input and output and a fixed,
// file-scope device array for everything else.  It calls no cudaMalloc,
// cudaFree or any other allocating function.
// ---------------------------------------------------------------------------
namespace {

// Layout of the static scratch: a 2 KiB header (the kernel's profile, pair,
// job and offset records), then the interleaved prefix and suffix
// temporaries, 2 x 32 x (L+1) ExpScores.  The header is 2 KiB although its records take 192
// bytes so that a background lookup with any 8-bit code (bg[0..255] starts
// 24 bytes into the profile record) stays inside the array.
constexpr size_t kNaHeaderBytes = 2048;
constexpr size_t kNaTmpEntries = (size_t)nullTmpEntries(DMST_NOALLOC_MAX_LEN);
constexpr size_t kNaScratchBytes = kNaHeaderBytes + kNaTmpEntries * sizeof(XS);  // 8,391,168 bytes
static_assert(kNaScratchBytes == 8391168, "documented scratch size");

static __device__ __align__(256) unsigned char gNullScratch[kNaScratchBytes];

struct NaHeader {
    DevProfile profile;  // offset 0
    DevPair pair;        // offset 128
    NullJob job;         // offset 160
    int jobPair;         // offset 168
    int pad;
    long long tmpOff;    // offset 176
};
static_assert(sizeof(NaHeader) <= 192, "no-alloc header layout");
static_assert(offsetof(NaHeader, profile) + offsetof(DevProfile, bg) + 256 * sizeof(float) <= kNaHeaderBytes,
              "an 8-bit code must index inside the header");

// Writes one call's header records into the scratch from a kernel argument,
// in stream order with the null-model launch that reads them.
__global__ void naHeaderKernel(NaHeader h, NaHeader *dst) {
    if (threadIdx.x == 0) *dst = h;
}


}  // namespace

extern "C" int dmst_null_model_noalloc(const uint8_t *codes, int length, const float *bg, const dmst_opts *opts,
                                       float *seeds, float *scales4, void *stream) {
    if (!codes || !bg || !seeds || !scales4 || length < 1) return DMST_EINVAL;
    if (length > DMST_NOALLOC_MAX_LEN) return DMST_ERANGE;
    dmst_opts o;
    dmst_opts_default(&o);
    if (opts) o = *opts;
    if (!(o.insert1 >= 0 && o.insert1 < 1 && o.insert2 >= 0 && o.insert2 < 1 && o.delete1 >= 0 && o.delete1 < 1 &&
          o.delete2 >= 0 && o.delete2 < 1 && o.insert1 + o.insert2 + o.delete1 + o.delete2 < 1))
        return DMST_EINVAL;
    // An error left pending by the caller's earlier CUDA work is reported as
    // it is and left in place for the caller to read (not cleared here).
    if (cudaPeekAtLastError() != cudaSuccess) return DMST_EDEVICE;
    // The scratch's address on the current device, asked for on every call
    // (it allocates nothing once the module is loaded, and stays right after
    // a device reset, which gives module globals new addresses).
    void *base = nullptr;
    if (cudaGetSymbolAddress(&base, gNullScratch) != cudaSuccess || !base) {
        cudaGetLastError();
        return DMST_EDEVICE;
    }
    NaHeader *hdr = reinterpret_cast<NaHeader *>(base);
    XS *tmp = reinterpret_cast<XS *>(static_cast<unsigned char *>(base) + kNaHeaderBytes);

    // The records dmst_null_model builds for one pair, with offsets 0 into the
    // caller's buffers.  Every scratch word the kernel reads is written in the
    // same call (the header here, the suffix temporary before its reads), so
    // nothing has to start at zero.
    NaHeader h;
    std::memset(&h, 0, sizeof h);
    h.profile.M = 0;
    h.profile.rowPad = 0;
    for (int c = 0; c < 26; ++c) h.profile.bg[c] = (c < kNumCodes) ? bg[4 + c] : 0.0f;
    h.profile.bg[kPad] = 0.0f;  // zero_idx pad reads as 0
    h.pair.codeOff = 0;
    h.pair.seedOff = 0;
    h.pair.L = length;
    h.pair.M = 0;
    h.pair.prof = 0;
    h.pair.R = 1;
    h.job = NullJob{0, 1};
    h.jobPair = 0;
    h.tmpOff = 0;
    Rates r{};
    r.insert1 = (float)o.insert1;
    r.insert2 = (float)o.insert2;
    r.delete1 = (float)o.delete1;
    r.delete2 = (float)o.delete2;
    NullRates nr;
    nr.single = (double)(r.insert1 + r.delete2);
    nr.dbl = (double)(r.insert2 + r.delete1);

    cudaStream_t s = static_cast<cudaStream_t>(stream);
    naHeaderKernel<<<1, 32, 0, s>>>(h, hdr);
    if (cudaGetLastError() != cudaSuccess) return DMST_EDEVICE;  // nothing queued
    nullModelKernel<<<1, kNullWarps * 32, 0, s>>>(&hdr->job, 1, &hdr->jobPair, &hdr->pair, &hdr->profile, codes,
                                                  seeds, tmp, &hdr->tmpOff, reinterpret_cast<PairScales *>(scales4),
                                                  nr);
    if (cudaGetLastError() != cudaSuccess) return DMST_EDEVICE;  // the header write alone is queued
    return DMST_OK;
}
