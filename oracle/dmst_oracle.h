/*
 * dmst_oracle.h -- TEST INFRASTRUCTURE ONLY.
 *
 * A plain-C, one-pair-at-a-time restatement of the reference's scoring path
 * for the DNA x protein-profile search: the per-read null model, the
 * row-rescaled backward and forward recurrences, the exact mid-anchored and
 * filter scores, and the lean backward-only float filter.  It is the checker
 * of the CUDA library's parity tests and the "port" CPU baseline; nothing in
 * the product links it.
 *
 * Pinned: tests/test_oracle.py checks it against the reference compiled from
 * its own sources (oracle/_ref, oracle/ref_harness.cc) on synthetic pairs and
 * against the committed golden vectors in tests/golden/.
 *
 * Profile layout (the reference's Profile, dummest-core.hh:241-254):
 *   values  (M+1) x 29 floats, row i = transitions of node i then the match
 *           emissions used by row i (values + i*29 + 4 indexed by codon code)
 *   params  (M+2) x 11 floats, the reference Params (dummest-core.hh:233-239):
 *           alpha'[3], beta'[3], delta'[3], epsilon', enter
 *   bg      29 floats, bg_probs (bg + 4 indexed by codon code)
 * Sequences are codon codes 0..24 (decodeSequence, dummest-sequence.hh:181-204),
 * length >= 3.
 */
#ifndef DMST_ORACLE_H
#define DMST_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct dmsto_score { /* ExpScore, dummest-score.hh:28-33 */
    float m;
    int32_t e;
} dmsto_score;

/* Background frameshift rates as the reference derives them from the four
 * options (dummest-core.hh:123-131): single = INSERT1 + DELETE2,
 * dbl = INSERT2 + DELETE1, both float sums. */
typedef struct dmsto_rates {
    float single;
    float dbl;
} dmsto_rates;

/* Null model of one read (dummest-dp-backward.hh:6-165): prefixSeed[0..L),
 * suffixSeedFromNext[0..L) and the packed scales {one-nt, two-nt, codon}. */
int dmsto_null_model(const float *bg, const uint8_t *codes, int L, dmsto_rates r, float *prefix_seed,
                     float *suffix_seed, float *scales3);

/* findSimilarities(needAlign=false) for one pair: backwardPass with the exact
 * filter best (dummest-dp-backward.hh:444-615) then forwardPass's mid score
 * (dummest-dp-forward.hh:9-250).  Outputs the exact ExpScores. */
int dmsto_score_pair(const float *values, const float *params, const float *bg, int M, const uint8_t *codes, int L,
                     dmsto_rates r, dmsto_score *mid, dmsto_score *filter);

/* findSimilaritiesBackwardOnly for one pair (dummest-dp-backward.hh:300-438):
 * max W1 * prefixSeed in plain float, no row rescaling (may be +inf). */
int dmsto_filter_pair(const float *values, const float *params, const float *bg, int M, const uint8_t *codes, int L,
                      dmsto_rates r, float *best);

/* W1 of backwardPass for one pair: rows 0..M x columns 0..L-1 (row-major,
 * as stored after each row's rescale) and the per-row rescale counts. */
int dmsto_backward_matrix(const float *values, const float *params, const float *bg, int M, const uint8_t *codes,
                          int L, dmsto_rates r, float *w1, int *counts);

/* Per-column anchors of the hit path (dummest-dp-forward.hh:196-206): for
 * each column j < L the largest wMid = promote(W0) * promote(W1) over the
 * rows, and its row (the first row on ties). */
int dmsto_anchors(const float *values, const float *params, const float *bg, int M, const uint8_t *codes, int L,
                  dmsto_rates r, dmsto_score *colBest, int *colRow);

/* log T in FP64: T = sum over cells of prefixSeed * W1 (the total weight of
 * all local alignments), the backward recurrence in double on double profile
 * arrays (values (M+1) x 29, params (M+2) x 11), the reference's null model
 * from the float background.  The finite-difference oracle of the gradient. */
int dmsto_log_total(const double *values, const double *params, const float *bg, int M, const uint8_t *codes,
                    int L, dmsto_rates r, double *logT);

/* Posterior tables in FP64 ((M+1) x L each, row-major; either may be NULL):
 * cell[i][j] = W0[i][j] W1[i][j] / T, match[i][j] = X(i,j) W1[i+1][j] / T
 * (X the match term of the forward, dummest-dp-forward.hh:125-157), with
 * log T from the forward total and from the backward total. */
int dmsto_posteriors(const double *values, const double *params, const float *bg, int M, const uint8_t *codes,
                     int L, dmsto_rates r, double *logT_fwd, double *logT_bwd, double *cell, double *match);

/* Rescale counts of the last dmsto_score_pair call on this thread: sum over
 * rows of the backward and forward counts (0 when no row was rescaled). */
void dmsto_last_rescales(int *backward, int *forward);

#ifdef __cplusplus
}
#endif

#endif
