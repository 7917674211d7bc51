// One traceback job: a hit pair (its best mid score passed the pair's gate)
// whose alignments are traced (dummest-dp-forward.hh:471-535).  The offsets
// place the job's pieces in the traceback buffers:
//   cells  (M+1) x L row-major cells: the replay's W0 and W1 (floats, written
//          by the exact kernel), later the prefix-optimal table in the same
//          bytes; the X table and the suffix-optimal table (one ExpScore per
//          cell) in their own arrays at the same cell offset;
//   cols   L entries per column array: anchors, column masses, flank scores,
//          candidates and their walks' spans;
//   rows   the reference's rescale counts cntB[M+2], cntF[M+2], the X table's
//          row maxima [M+2] and the two flank maxima.
#pragma once

namespace dmst {

struct AlignJob {
    int pair;            // the pair's index in its scoring call (internal order)
    int M, L;
    int nCand;           // columns in the reference's sorted anchor order that pass the gate
    long long cellOff;   // cells
    long long colOff;    // columns
    long long rowOff;    // ints
    float minM;          // the gate, normalizeScore(minProbRatio, 0)
    int minE;
};

__host__ __device__ inline long long alignRowInts(int M) { return 3LL * (M + 2) + 2; }

}  // namespace dmst
