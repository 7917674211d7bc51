// Shared device-side types of the B200 search path.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace dmst {

constexpr int kLanes = 32;
constexpr unsigned kFull = 0xffffffffu;
constexpr int kNumCodes = 25;    // codon codes 0..24 (24 = zero pad, dummest-dp.hh:93)
constexpr int kPad = 24;
constexpr int kRowAlign = 128;   // emission-table row padding (32 lanes x 4 rows)
// Rows of a profile's emission table and coefficient planes: M+1 rounded up
// to whole 96-row stripes (32 lanes x 3 rows), then to kRowAlign, so that the
// last stripe of every rows-per-lane shape (128, 96, 64 or 32 rows) lies in
// the zero-filled padding.
__host__ __device__ constexpr int rowPadOf(int M) {
    const int r96 = (M + 1 + 95) / 96 * 96;
    const int r = r96 > M + 1 ? r96 : M + 1;
    return (r + kRowAlign - 1) / kRowAlign * kRowAlign;
}
constexpr int kParamFloats = 11; // Params (dummest-core.hh:233-239)
// RESCALE_THRESH of the FP32 engine (dummest-score.hh:93).  The fast path is
// exact with respect to the reference only while no row maximum exceeds it.
constexpr float kRescaleThresh = 1e30f;

// One profile as the device keeps it.  The emission table is code-major,
// emit[c * rowPad + i] = values[i][4 + c] (dummest-profile.hh:208-224) for
// rows i <= M and 0 above, so four consecutive rows of one code are one
// 16-byte shared-memory load.
struct DevProfile {
    int M;
    int rowPad;
    long long emitOff;   // float offset of the [25][rowPad] table
    long long paramOff;  // float offset of the (M+2) x 11 Params
    float bg[26];        // bg_probs[4 + c], c = 0..24 (bg[24] = 0), bg[25] = 0
};
static_assert(sizeof(DevProfile) == 128, "DevProfile layout");

// The DP coefficient planes of a profile follow its Params in the params
// buffer, 16-byte aligned: kCoefPlanes planes of rowPad floats, one value per
// profile row (the Params entry the recurrences read), 0 on the padding rows
// past M; the last plane holds 1 on rows 0..M (the seed term's row factor).
// A lane loads its R consecutive rows of a plane with one vector load.
enum CoefPlane { kPA0, kPA1, kPA2, kPB0, kPD0, kPD1, kPD2, kPEps, kPEnter, kPRs, kCoefPlanes };
constexpr int kCoefParam[kCoefPlanes - 1] = {0, 1, 2, 3, 6, 7, 8, 9, 10};  // Params index of each plane
__host__ __device__ constexpr long long coefOffOf(long long paramOff, int M) {
    return (paramOff + (long long)(M + 2) * kParamFloats + 3) / 4 * 4;
}

// One (sequence, profile) pair of a scoring call.
struct DevPair {
    long long codeOff;  // byte offset of the sequence's codon codes
    long long seedOff;  // float offset of prefixSeed[L] followed by suffixSeedFromNext[L]
    int L;
    int M;
    int prof;
    int R;              // profile rows per lane (1, 2 or 4)
};
static_assert(sizeof(DevPair) == 32, "DevPair layout");

// Per-pair null-model scales (setupBatch's packed nullScale* lanes).
struct PairScales {
    float s1;  // nullScaleOneNucleotide  = perBase / 4
    float s2;  // nullScaleTwoNucleotide  = perBase^2 / 16
    float sC;  // nullScaleCodon          = perBase^3
    float pad;
};

// Raw per-pair results of the wavefront kernel (fast path).
struct PairOut {
    float mid;    // max W0*W1 over cells
    float filt;   // max W1*prefixSeed over cells
    float maxYb;  // max backward Y (>= every W1); > threshold means a row rescale
    float maxFw;  // max forward W0 / Y0
};

// A run of pairs that share a profile, scheduled on one CTA.
struct Chunk {
    int first;
    int count;
    int prof;
    int rowPad;
};

}  // namespace dmst
