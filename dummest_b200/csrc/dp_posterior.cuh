// Reductions of the posterior tables that the adjoint kernel writes in its
// POST form (cell posteriors W0 W1 / T and match posteriors X W1 / T, each
// (M+1) x L doubles, row-major): per column, the largest cell posterior over
// the rows and its row (the first row on ties), the posterior-decoded track
// of the alignment through the window; and per row, the sum over the columns
// of the match posteriors, the expected number of match emissions of the
// profile row.  The tables stay in device memory; only these L + (M+1) values
// per pair leave it.  Both kernels read each table once, coalesced across the
// columns (HBM-bound).
#pragma once

#include "dp_common.cuh"

namespace dmst {

struct PostSumJob {
    long long pOff;    // double offset of the pair's tables in the batch's buffer
    long long colOff;  // offset of the pair's columns in the column outputs
    long long rowOff;  // offset of the pair's rows in the row output
    int M, L;
};
static_assert(sizeof(PostSumJob) == 32, "PostSumJob layout");

constexpr int kPostThreads = 256;

// Block (x, y): columns x * 256 .. of job y; a thread walks its column down
// the rows.
__global__ void __launch_bounds__(kPostThreads) postColumnKernel(const PostSumJob *jobs, const double *post,
                                                                 double *colPost, int *colRow) {
    const PostSumJob jb = jobs[blockIdx.y];
    const int j = blockIdx.x * kPostThreads + threadIdx.x;
    if (j >= jb.L) return;
    const double *cell = post + jb.pOff + j;
    double best = -1.0;
    int row = 0;
#pragma unroll 8
    for (int i = 0; i <= jb.M; ++i) {
        const double v = __ldcs(cell + (size_t)i * jb.L);
        if (v > best) {
            best = v;
            row = i;
        }
    }
    if (colPost) colPost[jb.colOff + j] = best;
    if (colRow) colRow[jb.colOff + j] = row;
}

// Block (x, y): rows x * 8 .. x * 8 + 7 of job y, one warp per row; the lanes
// sum interleaved columns and the warp folds the 32 partial sums.
__global__ void __launch_bounds__(kPostThreads) postRowKernel(const PostSumJob *jobs, const double *post,
                                                              double *rowMatch) {
    const PostSumJob jb = jobs[blockIdx.y];
    const int lane = threadIdx.x & 31;
    const int i = blockIdx.x * (kPostThreads / kLanes) + (threadIdx.x >> 5);
    if (i > jb.M) return;
    const double *m = post + jb.pOff + (size_t)(jb.M + 1) * jb.L + (size_t)i * jb.L;
    double s = 0.0;
    for (int j = lane; j < jb.L; j += kLanes) s += __ldcs(m + j);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(kFull, s, o);
    if (lane == 0) rowMatch[jb.rowOff + i] = s;
}

}  // namespace dmst
