// The two-wave search on the device (dummest-search.hh:119-193): the float
// filter (findSimilaritiesBackwardOnly) over every pair, then the full
// mid-anchored scoring over the survivors, with no host round trip.
//
// A pair survives when its float best b is positive and passes the E-value
// gate K_filter T / exp(lambda_filter ln b) <= E_filter, or when b is +inf
// ("inf always survives", dummest-search.hh:163-168).  The gate decreases in b,
// so the host turns it into the smallest float b* that passes
// (dmst_filter_threshold, evaluated with the reference's expression in
// double), and the device compares b >= b*.
//
// The survivors of each chunk of the filter wave (pairs of one profile,
// longest read first) become the pairs of the same chunk of the second wave,
// in order, so the compaction needs no scan across chunks: one warp per chunk
// packs its survivors with a ballot.
#pragma once

#include "dp_common.cuh"
#include "dp_wavefront.cuh"

namespace dmst {

__global__ void survivorKernel(const Chunk *filterChunks, int nChunks, const PairOut *fo, const float *minBest,
                               Chunk *midChunks, int *survivorIdx, int chunkStride, uint8_t *survived) {
    const int c = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (c >= nChunks) return;  // whole warps
    const Chunk ch = filterChunks[c];
    const float gate = minBest[ch.prof];
    int cnt = 0;
    for (int k0 = 0; k0 < ch.count; k0 += kLanes) {
        const int k = k0 + lane;
        bool sv = false;
        int pi = 0;
        if (k < ch.count) {
            pi = ch.first + k;
            const float b = fo[pi].filt;
            sv = b > 0.0f && (b >= gate || isinf(b));
            survived[pi] = sv ? 1 : 0;
        }
        const unsigned m = __ballot_sync(kFull, sv);
        if (sv) survivorIdx[(size_t)c * chunkStride + cnt + __popc(m & ((1u << lane) - 1u))] = pi;
        cnt += __popc(m);
    }
    if (lane == 0) midChunks[c] = Chunk{c * chunkStride, cnt, ch.prof, ch.rowPad};
}

}  // namespace dmst
