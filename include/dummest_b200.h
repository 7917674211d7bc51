/*
 * dummest_b200.h -- C ABI of the B200 (sm_100a) implementation of DUMMEST's
 * search hot path: the frameshift-aware DNA x protein-profile Forward/Backward
 * dynamic program, its mid-anchored score, the lean backward-only filter, and
 * the random-sequence scoring behind Gumbel E-value calibration.
 *
 * Plain C types only.  Every call returns a status (0 or a negative DMST_E*
 * code); nothing aborts and no exception crosses the ABI.  One context per
 * host thread (contexts are not internally locked).  All host buffers are
 * caller-owned; device memory is owned by the context.
 *
 * Reference interfaces this ABI replaces (paths relative to the reference
 * repository root):
 *   Params / Profile            dummest-core.hh:233-254
 *   ExpScore                    dummest-score.hh:28-33
 *   readProfiles/finalizeProfile dummest-profile.hh:235-329, :105-233
 *   decodeSequence              dummest-sequence.hh:181-204
 *   findSimilarities            dummest-search.hh:9-17   (needAlign=false)
 *   findSimilaritiesBackwardOnly dummest-dp-backward.hh:300-438
 *   backwardPass bestOut        dummest-dp-backward.hh:579-609
 *   estimateK / estimateGumbel  dummest-calibration.hh:338-649, :97-104
 *   rate globals                dummest-core.hh:115-131
 */
#ifndef DUMMEST_B200_H
#define DUMMEST_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes --------------------------------------------------- */
#define DMST_OK 0
#define DMST_EINVAL (-1)   /* bad argument (null pointer, L < 3, unknown id, ...) */
#define DMST_ENOMEM (-2)   /* host or device allocation failed */
#define DMST_EDEVICE (-3)  /* CUDA error, or no usable sm_100 device */
#define DMST_ETIMEOUT (-4) /* a kernel exceeded its iteration budget */
#define DMST_EPARSE (-5)   /* malformed HMMER3 / sequence text */
#define DMST_ERANGE (-6)   /* size beyond a documented limit */

/* ---- score modes for dmst_score_pairs --------------------------------- */
/* Backward then forward; mid-anchored score and the exact filter best.  The
 * GPU counterpart of findSimilarities(needAlign=false) as estimateK calls it
 * (dummest-calibration.hh:489-505, dummest-dp-forward.hh:536-544). */
#define DMST_MODE_MID 0
/* The lean float backward-only filter (findSimilaritiesBackwardOnly): plain
 * float W1 with no row rescaling, score = max W1[i][j]*prefixSeed[j], which
 * may be +inf ("inf always survives", dummest-search.hh:163-168). */
#define DMST_MODE_FILTER 1
/* Flag for either mode: run the plain schedule, one pair per kernel launch,
 * the baseline the batched persistent kernel is measured against.  The
 * launch is one CTA of 8 warps that share the pair: its stripes (32 R profile
 * rows each) are dealt to the warps and run as a stripe pipeline, with the
 * same per-cell arithmetic (results bit for bit those of the batched call).
 * No counterpart in the reference (its unit of work is a SIMD batch). */
#define DMST_MODE_PLAIN 0x100
/* With DMST_MODE_PLAIN: the earlier plain form, the batched kernel launched
 * on a one-pair chunk, where one warp computes the pair. */
#define DMST_MODE_PLAIN_1WARP 0x1000
/* Flag: route every pair through the exact row-rescaled wavefront path
 * (the path taken by pairs whose rows the reference would rescale). */
#define DMST_MODE_FORCE_EXACT 0x200
/* Flag: route every pair through the one-thread-per-pair exact kernel, a
 * direct restatement of the reference's row-at-a-time loops (a slow
 * cross-check of the wavefront paths). */
#define DMST_MODE_EXACT_SEQUENTIAL 0x400

/* Flag: launch the call's device work up to the DP results (counter reset,
 * null-model kernel, persistent DP kernels) through a captured CUDA graph.
 * The graph is captured on the first such call and replayed by later calls
 * with the same launch shape and buffers (their descriptors are uploaded into
 * the same device buffers first); a changed shape captures again and updates
 * the executable graph.  Results are those of the direct launches.  Ignored
 * with DMST_MODE_PLAIN. */
#define DMST_MODE_GRAPH 0x800

/* ---- per-result flags -------------------------------------------------- */
#define DMST_RES_EXACT_PATH 1 /* pair was scored by the exact row-rescaled kernel */
#define DMST_RES_SURVIVOR 2   /* dmst_search: the pair passed the filter wave and has a mid score */

/* Reference Params (dummest-core.hh:233-239), FP32 engine layout. */
typedef struct dmst_params {
    float alpha_prime[3];
    float beta_prime[3];
    float delta_prime[3];
    float epsilon_prime;
    float enter_match_probability;
} dmst_params;

/* Reference ExpScore (dummest-score.hh:28-33): value = m * 2^e, m in [0.5,1)
 * (the float rounding of a [0.5,1) double may give exactly 1.0, as in the
 * reference), m == 0 for zero. */
typedef struct dmst_score {
    float m;
    int32_t e;
} dmst_score;

/* Rates and limits (dummest-core.hh:60-80, :115-131). */
typedef struct dmst_opts {
    double insert1, insert2, delete1, delete2; /* frameshift rates per base */
    double stop_codon_prob;                    /* STOP_CODON_PROB */
    double bg_stop_codon_prob;                 /* BG_STOP_CODON_PROB */
    int device;                                /* CUDA device ordinal */
    int rows_per_lane;                         /* 0 = autotuned, else 1, 2, 3 or 4 */
    size_t device_budget_bytes;                /* 0 = 60% of free device memory */
    double tantan_threshold;                   /* TANTAN_MASK_THRESHOLD (OPT_tantan, 0.5) for DMST_HMM_MASK */
} dmst_opts;

/* One (sequence, profile) pair; min_prob_ratio < 0 means "report" as in the
 * calibration call (minProbRatio = -2, dummest-calibration.hh:490). */
typedef struct dmst_pair {
    int32_t seq;
    int32_t profile;
    float min_prob_ratio;
} dmst_pair;

typedef struct dmst_result {
    dmst_score mid;    /* max_{i,j} W0*W1 (exact pair)                        */
    dmst_score filter; /* max_{i,j} W1*prefixSeed (exact pair, MODE_MID)     */
    double mid_ln;     /* ln(mid) = scoreToLog(mid); -inf for zero            */
    double filter_ln;  /* ln(filter) (MODE_MID) or ln of the float filter     */
    float filter_f;    /* MODE_FILTER: the float filter score as the reference returns it */
    int32_t flags;     /* DMST_RES_*                                          */
} dmst_result;

typedef struct dmst_ctx dmst_ctx;

/* Default options: the reference's compile-time defaults. */
void dmst_opts_default(dmst_opts *opts);

int dmst_ctx_create(const dmst_opts *opts, dmst_ctx **out);
void dmst_ctx_destroy(dmst_ctx *ctx);
const char *dmst_strerror(int status);
/* Text of the last error on this context ("" if none). */
const char *dmst_last_error(const dmst_ctx *ctx);
/* The context's CUDA stream (a cudaStream_t), on which every kernel of the
 * context runs; callers may record events on it to time a sequence of calls. */
void *dmst_ctx_stream(const dmst_ctx *ctx);

/* ---- profiles ----------------------------------------------------------
 * dmst_profile_add takes an already-finalized profile exactly as the
 * reference holds it: values is (M+1) x width floats (row i = transitions of
 * node i followed by the match emissions of node i+1, width = 29 for protein,
 * dummest-profile.hh:264-313), params is M+2 Params, bg is width floats
 * (bg_probs, dummest-profile.hh:135-148).  Replaces: Profile construction. */
int dmst_profile_add(dmst_ctx *ctx, const float *values, int width, int M, const dmst_params *params,
                     const float *bg, int *id);

/* Replace profile `id` by new values, Params and background (any length);
 * later calls use the new profile.  For refining a profile in place. */
int dmst_profile_set(dmst_ctx *ctx, int id, const float *values, int width, int M, const dmst_params *params,
                     const float *bg);

/* Parse HMMER3 text and finalize each profile with the reference's semantics
 * (readProfiles + finalizeProfile without letter-probability filtering).
 * background_type: 'G', 'A' or 'M', or-ed with DMST_HMM_MASK to tantan-mask
 * each profile's consensus as the reference does by default (-m 1 or 3,
 * readProfiles' isMask; dummest-profile.hh:105-233): consensus letters whose
 * repeat probability reaches the context's tantan_threshold emit the
 * background and are left out of the background means.  Replaces:
 * readProfiles (dummest-profile.hh:235-329).  first_id/count receive the new
 * ids. */
#define DMST_HMM_MASK 0x100
int dmst_profile_load_hmm(dmst_ctx *ctx, const char *text, size_t len, int background_type, int *first_id,
                          int *count);

/* Host-side finalize without a context (for tests and tools): fills values
 * ((M+1)*29), params (M+2) and bg (29) of profile number `index` in the text
 * (background_type as for dmst_profile_load_hmm, the threshold from opts).
 * Returns its M via *M.  Call with values == NULL first to learn M. */
int dmst_hmm_finalize(const char *text, size_t len, int index, int background_type, const dmst_opts *opts,
                      int *M, float *values, dmst_params *params, float *bg, char *name, size_t name_cap);

int dmst_profile_count(const dmst_ctx *ctx);
int dmst_profile_length(const dmst_ctx *ctx, int id);

/* ---- sequences ----------------------------------------------------------
 * Sequences are kept on the device as per-base codon codes (0..24, the
 * output of decodeSequence, dummest-sequence.hh:181-204).
 *   _decoded: codes given by the caller.
 *   _dna:     ASCII DNA (ACGT any case; IUPAC ambiguity and other letters of
 *             RYSWKMBDHVN map to the masked code), decoded on the device.
 *   _packed:  2-bit packed DNA (A=0 C=1 G=2 T=3, base k of a sequence at bits
 *             2*(k%16) of 32-bit word k/16 counted from that sequence's first
 *             word), plus an optional bitmap of masked bases (bit k%32 of
 *             word k/32; NULL = none); decoded on the device.
 * offsets has nseq+1 entries (base offsets; packed: word offsets follow from
 * the base offsets rounded up to 16 per sequence).  Every sequence needs
 * L >= 3 (dummest-dp.hh:84).  first_id receives the id of the first one.
 * _packed copies its inputs into pinned staging and queues the upload and
 * decode behind the context's pending calls without waiting for them: the
 * caller's arrays may be reused at once, and every later call finds the
 * sequences decoded. */
int dmst_seqs_add_decoded(dmst_ctx *ctx, const uint8_t *codes, const int64_t *offsets, int nseq, int *first_id);
int dmst_seqs_add_dna(dmst_ctx *ctx, const char *ascii, const int64_t *offsets, int nseq, int *first_id);
int dmst_seqs_add_packed(dmst_ctx *ctx, const uint32_t *words, const uint32_t *mask_bits, const int64_t *offsets,
                         int nseq, int *first_id);
/* One contig of a FASTA text, as the reference's reader cuts it (readContig,
 * dummest-sequence.hh:6-82, with the IUPAC character classes of
 * dummest.cc:445-456): a record is '>' and a name (the first word of the
 * line); its sequence runs to the next '>' and is cut into contigs at
 * characters that are neither letters of the protein alphabet
 * ("ACDEFGHIKLMNPQRSTVWYUO?*", either case), IUPAC codes (RYSWKMBDHVN, read
 * as 22) nor characters up to ' ' (skipped); each cutting character counts
 * one position of the record. */
typedef struct dmst_contig {
    int32_t record;      /* index of its record in the text */
    int32_t start;       /* Contig::start: its position in the record */
    int32_t length;      /* letters */
    int32_t seq_id;      /* dmst_seqs_add_fasta: its sequence id (-1: shorter than 3, not added) */
    int64_t name_off;    /* the record's name in the text */
    int32_t name_len;
    int32_t seq_id_rc;   /* dmst_seqs_add_fasta with DMST_FASTA_REVCOMP: its reverse complement's id */
    int64_t letter_off;  /* dmst_fasta_contigs: its letter codes in letters */
    int32_t record_length; /* the record's length (its contigs and cutting characters) */
    int32_t pipeline;    /* DMST_FASTA_PIPELINE: bit 0 the header had pipeline fields, bit 1 plus strand */
    int64_t w_start, w_end;  /* DMST_FASTA_PIPELINE: the window of the header's name "chr/start-end" */
    int64_t true_length;     /* ... its "length=" field */
    int64_t profile_off;     /* ... its "profile=" field in the text */
    int32_t profile_len;
    int32_t pad;
} dmst_contig;

/* dmst_seqs_add_fasta flags: also add each contig's reverse complement (A-T
 * and C-G swapped, other letters kept, order reversed), as the pipeline's
 * minus_strand_revcomp record of the same sequence (bin/dummest:236-264)
 * cuts it; in that record the contig starts at record_length - start -
 * length. */
#define DMST_FASTA_REVCOMP 1
/* dmst_fasta_contigs / dmst_seqs_add_fasta flags: read the pipeline's headers
 * (">chr/start-end length=N profile=NAME plus_strand|minus_strand..." as
 * bin/dummest writes them) as the reader of the reference's PIPELINE_MODE
 * build does (dummest-sequence.hh:19-52): the name is the part before '/',
 * and fields a header lacks keep the previous record's values, as the
 * reader's reused Sequence keeps them (0 before any). */
#define DMST_FASTA_PIPELINE 2

/* The contigs of a FASTA text and their letter codes (the reader's
 * charToNumber values: A=0 C=1 G=5 T=16, IUPAC 22, other letters their
 * protein codes), host only.  *n_contigs and *n_letters get the counts; with
 * capacities below them nothing is written and DMST_ERANGE is returned.
 * A text not starting with '>' (after whitespace) or a header without a name
 * is DMST_EPARSE, as the reader fails.  A '*' inside DNA (code 23) is read
 * as a letter, which the reference's decodeSequence does not accept (it
 * asserts codes <= 22); the library decodes it as any non-ACGT letter. */
int dmst_fasta_contigs(const char *text, size_t len, int flags, dmst_contig *contigs, size_t cap_contigs,
                       size_t *n_contigs, char *letters, size_t cap_letters, size_t *n_letters);
/* Reads a FASTA text (dummest.cc:553-606's readContig loop) and adds each
 * contig of length >= 3 as one sequence, decoded as the engine decodes it
 * (decodeSequence: a triplet with any letter other than A, C, G, T is '?'),
 * uploaded 2-bit packed with a bitmap of the other letters.  Sequence ids
 * follow the text: per record its contigs, then (DMST_FASTA_REVCOMP) the
 * reverse complements in the minus record's order.
 * Masking (the reference's tantan pass, makeMaskedSequence) stays with the
 * caller: a base written as 'N' decodes as the reference's masked copy
 * does.  contigs (cap_contigs entries)
 * gets every contig with its sequence id; with too small a capacity nothing
 * is added and DMST_ERANGE is returned, *n_contigs holding the count. */
int dmst_seqs_add_fasta(dmst_ctx *ctx, const char *text, size_t len, int flags, dmst_contig *contigs,
                        size_t cap_contigs, size_t *n_contigs);
/* One window of the pipeline's prefilter hits (bin/dummest:91-183 and its
 * bedtools sort | merge | getfasta -s stage, bin/dummest:663-676): a merged
 * interval of one (target record, profile, strand). */
typedef struct dmst_window {
    int32_t record;      /* the target record: index among the record names (the genome's records) */
    int32_t strand;      /* +1 plus_strand; -1 minus_strand_revcomp: the window is reverse-complemented */
    int64_t start, end;  /* [start, end), 0-based positions of the record (the BED interval) */
    int64_t profile_off; /* the profile's name (the hit rows' query) in the hits text */
    int32_t profile_len;
    int32_t profile;     /* its index among the profile names, -1 when not among them */
} dmst_window;

/* dmst_windows_from_hits flags: the hits' targets are the records themselves
 * (the pipeline's ORF mode, coordinates in nucleotides, the strand from their
 * order) rather than their six-frame translations "record_frame=+-N". */
#define DMST_HITS_TARGET_IS_CONTIG 1

/* The windows of BLAST-tab hit rows (mmseqs convertalis output), host only.
 * Per row (12 or more fields; '#' lines and shorter rows skipped; rows whose
 * coordinates or frame do not parse as Python's int() counted in
 * *n_malformed and skipped; rows of a target not among the records, or of
 * length 0, skipped) an interval centred on the hit and padded by 3 x the
 * profile's length (0 for a profile not among profile_names) on each side,
 * clipped to the record (_stream_bed_from_convertalis, bin/dummest:91-183).
 * Per (target, query, strand), ordered as bedtools sort orders the names
 * "target|query|strand" (bytes), the intervals are sorted by start and merged
 * where the next starts at or before the current end (bedtools merge); the
 * name is split back at its last two '|' (bin/dummest:77-88).  A window whose
 * record is not among the names (a query holding '|') is skipped as bedtools
 * getfasta skips it, counted in *n_dropped.  Names that repeat: the last one
 * counts, as in the driver's dictionaries.  A row giving a start past its end
 * is DMST_EPARSE (bedtools rejects the interval).  *n_windows gets the count;
 * with cap below it nothing is written and DMST_ERANGE is returned.  A text of
 * 1 MB or more is parsed on up to 16 host threads (line-aligned parts, grouped
 * in text order, so the result does not depend on the split). */
int dmst_windows_from_hits(const char *hits, size_t len, int flags, const char *const *record_names,
                           const int64_t *record_lengths, int n_records, const char *const *profile_names,
                           const int64_t *profile_lengths, int n_profiles, dmst_window *windows, size_t cap,
                           size_t *n_windows, size_t *n_malformed, size_t *n_dropped);
/* Keep a genome on the device for dmst_seqs_add_windows: every record of a
 * FASTA text (read as dmst_fasta_contigs reads it), 2 bits per position with a
 * bitmap of the positions that are not A, C, G or T.  Replaces the previous
 * genome; the text must stay valid while windows of it are added (their
 * contigs name the record by its offset in it).  *n_records gets the record
 * count; record_lengths (cap_records entries, may be NULL) each record's
 * length (contigs and cutting characters). */
int dmst_genome_load(dmst_ctx *ctx, const char *text, size_t len, size_t *n_records, int64_t *record_lengths,
                     size_t cap_records);
/* Add the windows of the loaded genome as sequences, decoded on the device
 * from the resident genome (forward, or reverse-complemented for strand -1).
 * Sequences and contigs are those dmst_seqs_add_fasta gives, with
 * DMST_FASTA_PIPELINE, for the windowed FASTA the pipeline writes from the
 * same windows (bedtools getfasta -s -name+ and _rewrite_fasta,
 * bin/dummest:186-233): the contigs' record is the window's index, start and
 * record_length are positions in the window, name the genome record's name
 * in the genome text, w_start = start + 1, w_end = end, true_length the
 * genome record's length, profile the window's (offsets in the hits text),
 * pipeline bit 1 set for strand +1; letter_off is -1.  A window outside its
 * record is DMST_EINVAL; with cap_contigs below the count nothing is added
 * and DMST_ERANGE is returned, *n_contigs holding the count. */
int dmst_seqs_add_windows(dmst_ctx *ctx, const dmst_window *windows, size_t n, dmst_contig *contigs,
                          size_t cap_contigs, size_t *n_contigs);
/* Device ms of the last dmst_seqs_add_windows decode kernel (waits for it);
 * -1 when none has run. */
int dmst_last_windows_ms(dmst_ctx *ctx, double *ms);
/* Drop all sequences (device memory is kept for reuse). */
int dmst_seqs_clear(dmst_ctx *ctx);
int dmst_seq_count(const dmst_ctx *ctx);
/* Length in nucleotides of sequence id, -1 for an unknown id. */
int dmst_seq_length(const dmst_ctx *ctx, int id);

/* Host decode of letter codes (A=0 C=1 G=5 T=16, masked=22, the engine's
 * protein-alphabet coding of DNA) into codon codes; replaces decodeSequence. */
int dmst_decode_letters(const char *letters, int L, uint8_t *codes);
/* Host ASCII DNA -> letter codes as the engine reads FASTA (dummest.cc:437-449). */
int dmst_encode_dna(const char *ascii, int L, char *letters);

/* ---- scoring ------------------------------------------------------------
 * Score n pairs.  mode = DMST_MODE_MID or DMST_MODE_FILTER, optionally or-ed
 * with DMST_MODE_PLAIN / DMST_MODE_FORCE_EXACT.  Synchronous. */
int dmst_score_pairs(dmst_ctx *ctx, const dmst_pair *pairs, size_t n, int mode, dmst_result *out);

/* Asynchronous scoring.  dmst_score_pairs_submit does the host work of a call
 * (sorting, descriptors, uploads through page-locked staging) and queues its
 * device work: null model, DP kernels, the exact path (flagged pairs are
 * queued and re-scored on the device) and the copy of the results back; it
 * returns without waiting.  dmst_score_pairs_complete waits for the oldest
 * pending call and writes its results into the `out` array given at submit
 * (which must stay valid until then).  At most two calls are pending per
 * context: a third submit completes the oldest first, so that the host work
 * of one call overlaps the device work of the other.  Adding sequences or
 * profiles, and every other entry point, completes the pending calls first.
 * dmst_score_pairs is submit + complete.  The reference batches pairs
 * synchronously per thread (dummest-search.hh:76-285). */
int dmst_score_pairs_submit(dmst_ctx *ctx, const dmst_pair *pairs, size_t n, int mode, dmst_result *out);
int dmst_score_pairs_complete(dmst_ctx *ctx);
/* Calls submitted and not yet completed (0, 1 or 2). */
int dmst_pending_calls(const dmst_ctx *ctx);

/* Two-wave search (findFinalSimilaritiesBatched's filter pass and slow wave,
 * dummest-search.hh:119-193), both waves on the device with no host round
 * trip: the float filter (findSimilaritiesBackwardOnly) of every pair, then
 * the mid-anchored score of the survivors.  A pair survives when its float
 * best b > 0 and b >= filter_min_best[profile id] or b = +inf (one gate per
 * profile id of the context, from dmst_filter_threshold).  Every result has
 * filter_f / filter_ln (the float filter); survivors also have the mid and
 * exact filter scores of dmst_score_pairs (DMST_MODE_MID) and
 * DMST_RES_SURVIVOR set; the others have mid_ln = -inf.  mode:
 * DMST_MODE_MID, optionally with DMST_MODE_FORCE_EXACT.  dmst_search_submit
 * queues the call like dmst_score_pairs_submit (completed by
 * dmst_score_pairs_complete); dmst_search waits for it. */
int dmst_search(dmst_ctx *ctx, const dmst_pair *pairs, size_t n, const float *filter_min_best, int mode,
                dmst_result *out);
int dmst_search_submit(dmst_ctx *ctx, const dmst_pair *pairs, size_t n, const float *filter_min_best, int mode,
                       dmst_result *out);
/* Per-column anchors of the hit path (dummest-dp-forward.hh:196-206,
 * :456-469), the starting points the reference sorts (descending) and traces
 * back from (dummest-traceback.hh).  For pair k (the caller's order) and
 * column j < L_k, at offset sum_{k'<k} L_k' + j: best = the largest mid
 * product wMid = promote(W0) promote(W1) over the profile rows (ExpScore) and
 * row = its row, the first on ties; columns whose products are all 0 have
 * best = {0, 0}.  Scored on the exact path; out (may be NULL) gets the
 * pairs' scores as from dmst_score_pairs(DMST_MODE_MID).  Synchronous. */
int dmst_anchors(dmst_ctx *ctx, const dmst_pair *pairs, size_t n, dmst_score *best, int *row, dmst_result *out);

/* One alignment of the hit path: the reference's AlignedSimilarity
 * (dummest-core.hh:298-317). */
typedef struct dmst_alignment {
    int32_t pair;       /* the pair's index in the dmst_align call */
    dmst_score score;   /* the anchor's exact mid score (AlignedSimilarity::pair) */
    double ln_score;    /* scoreToLog(score) (AlignedSimilarity::logProbRatio) */
    int32_t anchor1;    /* profile row of the anchor */
    int32_t anchor2;    /* sequence column of the anchor */
    int64_t seg_begin;  /* its first segment pair in dmst_align_fetch's list */
    int32_t seg_count;  /* 0: the walks from the anchor matched nothing (no MAF record) */
    int32_t pad;
} dmst_alignment;

/* A gapless piece of an alignment (SegmentPair, dummest-core.hh:273-275):
 * profile rows start1.., sequence columns start2.., length of them. */
typedef struct dmst_segment {
    int32_t start1, start2, length;
} dmst_segment;

/* The hit path with its traceback: findSimilarities(needAlign = true)
 * (dummest-search.hh:9-17; dummest-dp-forward.hh:252-535;
 * dummest-traceback.hh:35-118; dummest-dp.hh:119-268).  Every pair is scored
 * (out, may be NULL, as from dmst_score_pairs(DMST_MODE_MID)); a pair whose
 * min_prob_ratio is >= 0 and whose mid score is nonzero and at least
 * normalizeScore(min_prob_ratio) is a hit, and its alignments are traced on
 * the device: its per-column anchors in the reference's sorted order (the
 * reference's std::ranges::sort, descending), each anchor at or above the
 * gate and not inside an earlier alignment walked forward and backward over
 * the prefix- and suffix-optimal tables, and kept unless its sequence span
 * overlaps one kept before.  The alignments are kept in the context, the
 * pairs' lists in the call's pair order, each in the reference's order;
 * *n_alignments and *n_segments get their counts (dmst_align_fetch copies
 * them).  Pairs with min_prob_ratio < 0 (the calibration call's "report")
 * and misses have none.  Synchronous. */
int dmst_align(dmst_ctx *ctx, const dmst_pair *pairs, size_t n, dmst_result *out, size_t *n_alignments,
               size_t *n_segments);
/* Copies the last dmst_align call's alignments and segment pairs (capacities
 * at least its counts, else DMST_ERANGE). */
int dmst_align_fetch(const dmst_ctx *ctx, dmst_alignment *alignments, size_t cap_alignments,
                     dmst_segment *segments, size_t cap_segments);
/* Wall-clock phases of the last dmst_align call (ms): out[0] the whole call,
 * [1] scoring every pair, [2] the hits' exact replay and traceback tables,
 * [3] the anchor sort, [4] the walks' span pass, [5] the choice of anchors,
 * [6] the kept walks and the segment copy, [7] hits traced, [8] kernel
 * launches of the call.  n <= 9. */
int dmst_last_align_timing(const dmst_ctx *ctx, double *out, int n);

/* The filter gate as a float threshold: the smallest float best b whose
 * E-value K_filter * total_length / exp(ln(b) * lambda_filter) is at most
 * filter_evalue (the reference's expression, dummest-search.hh:158-166, in
 * double); +inf when no finite best passes. */
int dmst_filter_threshold(double lambda_filter, double k_filter, double total_length, double filter_evalue,
                          float *min_best);

/* Timing of the last dmst_score_pairs call, from CUDA events on the context's
 * stream: total device ms and the ms of the main DP kernel(s). */
int dmst_last_timing(const dmst_ctx *ctx, double *total_ms, double *dp_ms, double *null_ms, int *launches);
/* The same breakdown as an array: out[0] device ms of the call, [1] null-model
 * kernel ms, [2] DP kernel ms, [3] exact-path ms, [4] host preparation ms
 * (wall clock), [5] kernel launches, [6] pairs on the exact path, [7] host ms
 * after the device work (result assembly), [8] wall ms of the whole call,
 * [9] CUDA-graph captures made by the context so far (DMST_MODE_GRAPH).
 * n = number of entries wanted (<= 10). */
int dmst_last_timing_ex(const dmst_ctx *ctx, double *out, int n);

/* ---- autotuning ------------------------------------------------------
 * Kernel shapes: R rows of the profile per lane (a stripe of 32 R rows: 4, 3,
 * 2 or 1) and 16, 8 or 12 warps per CTA.  dmst_autotune times the DP kernel of
 * every shape on the caller's sample of pairs (mode MID, each shape run twice,
 * the second timed) and keeps, per R, the fastest CTA shape and its rate in
 * computed cells per second.  Later calls with rows_per_lane == 0 then pick,
 * per profile, the R with the least expected time (computed rows / rate).
 * gcups6 (may be NULL) receives the rates in GCUPS of computed cells, for
 * R = 4, 2, 1 x 16, 8 warps; dmst_tuned_rates gives nine (R = 4, 2, 1 x 16, 8,
 * 12 warps) and dmst_tuned_rates_ex the first n <= 12 of all twelve
 * (R = 4, 3, 2, 1 x 16, 8, 12 warps).  No counterpart in the reference (its
 * SIMD width is fixed at compile time). */
int dmst_autotune(dmst_ctx *ctx, const dmst_pair *sample, size_t n, double *gcups6);
int dmst_tuned_rates(const dmst_ctx *ctx, double *gcups9);
int dmst_tuned_rates_ex(const dmst_ctx *ctx, double *gcups, int n);
/* The shape a call would use for a profile of length M. */
int dmst_tuned_shape(const dmst_ctx *ctx, int M, int *rows_per_lane, int *warps_per_cta);

/* The exact path's wait budget: a warp of the stripe-pipelined exact kernel
 * that waits for the stripe before its own (a flag in shared memory) gives up
 * after this many 64 ns sleeps, marks its pair failed and lets the CTA's
 * other warps leave at their next block; the call then returns DMST_ETIMEOUT
 * and the context stays usable.  iterations = 0 restores the default (2^24,
 * about a second); a small value makes a call with multi-stripe exact-path
 * pairs time out on purpose (the test of the timeout path).  No counterpart
 * in the reference (its threads never wait on one another inside a pair). */
int dmst_set_wait_limit(dmst_ctx *ctx, int iterations);

/* Column checkpointing of the adjoint's forward pass (dmst_loglik_grad,
 * dmst_posteriors): DMST_ADJ_CKPT_ON keeps the stripes' top rows and a
 * checkpoint every 64 columns and recomputes the forward blocks in the
 * backward pass (about 1/12 of the full store's 24 bytes per cell, one more
 * forward pass of work); DMST_ADJ_CKPT_OFF keeps every cell's forward values;
 * DMST_ADJ_CKPT_AUTO (the default) keeps them when every pair's full store
 * fits the device budget at once.  The results are the same either way.
 * mode < 0 only queries; last_checkpointed (may be NULL) gets whether the
 * last adjoint call checkpointed.  No counterpart in the reference. */
#define DMST_ADJ_CKPT_AUTO 0
#define DMST_ADJ_CKPT_ON 1
#define DMST_ADJ_CKPT_OFF 2
int dmst_adjoint_checkpoint(dmst_ctx *ctx, int mode, int *last_checkpointed);
/* ---- log-likelihood and its gradient --------------------------------------
 * For pairs of one profile: log_t[k] = log T of pair k, T the total weight of
 * all local alignments of the read under the profile, i.e. the sum over cells
 * of prefixSeed[j] * W1[i][j] (equally, of W0[i][j] * suffixSeedFromNext[j]);
 * and the gradient of sum_k log T_k with respect to the profile's Params
 * (grad_params: (M+2) x 11 doubles, the dmst_params fields in order) and its
 * emission table (grad_emit: (M+1) x 25 doubles, the entries values[i][4+c]).
 * The null model (seeds, per-base scales, background) is held fixed.  Any of
 * the outputs may be NULL.  FP64 throughout.  The reference computes no
 * gradient: its forward recurrence (dummest-dp-forward.hh:63-250) is the
 * adjoint of its backward one (dummest-dp-backward.hh:473-574), and this call
 * evaluates both, with the gradient sums of each row. */
int dmst_loglik_grad(dmst_ctx *ctx, const dmst_pair *pairs, size_t n, double *log_t, double *grad_params,
                     double *grad_emit);

/* Posterior tables of pairs of one profile, FP64.  For pair k (the caller's
 * order), at post + sum_{k'<k} 2 (M+1) L_k': (M+1) x L_k doubles of cell
 * posteriors W0[i][j] W1[i][j] / T, then (M+1) x L_k doubles of match
 * posteriors X(i,j) W1[i+1][j] / T, X(i,j) the match term of the forward
 * (enter_i sC e_i(c_{j-2}) W0[i][j-3]; the combined table of
 * dummest-dp-forward.hh:125-157, divided by T).  log_t (n, may be NULL) as in
 * dmst_loglik_grad.  The reference's search never outputs posteriors; its
 * mid score is the maximum over cells of W0 W1 (dummest-dp-forward.hh:174-206),
 * so max_ij cell * T is that score. */
int dmst_posteriors(dmst_ctx *ctx, const dmst_pair *pairs, size_t n, double *log_t, double *post);

/* The posterior pass of a genome scan's windows above threshold, reduced on
 * the device: the tables of dmst_posteriors are computed in device memory and
 * only these leave it.  For pair k (the caller's order), at
 * col_post + sum_{k'<k} L_k' (and col_row likewise): per column j the largest
 * cell posterior max_i W0[i][j] W1[i][j] / T and its row i (the first on
 * ties), the posterior-decoded track of the alignment; at row_match +
 * k (M+1): per row i the sum over the columns of the match posteriors, the
 * expected number of match emissions of profile row i.  FP64; any output
 * may be NULL, but not all three.  The reference has no posterior pass; the
 * tables follow its forward and backward recurrences
 * (dummest-dp-forward.hh:125-157, dummest-dp-backward.hh:473-574). */
int dmst_posterior_summary(dmst_ctx *ctx, const dmst_pair *pairs, size_t n, double *log_t, double *col_post,
                           int *col_row, double *row_match);

/* Per-pair null model (testing aid): prefixSeed[0..L), suffixSeedFromNext[0..L)
 * and the three per-base scales (one-nt, two-nt, codon) for one pair, computed
 * by the device prologue kernel.  Replaces the null half of setupBatch
 * (dummest-dp-backward.hh:6-188). */
int dmst_null_model(dmst_ctx *ctx, int seq, int profile, float *prefix_seed, float *suffix_seed, float *scales3);

/* ---- null model without allocation -------------------------------------
 * This entry point has no counterpart in the reference.  It serves callers
 * that cannot allocate device memory where they need a read's null model:
 * a process whose device memory is already claimed by another pool (a
 * framework's caching allocator holding nearly all HBM makes a fresh
 * cudaMalloc fail), or a latency-bound caller whose other streams must not
 * stall on cudaFree's implicit device synchronisation.
 *
 * It computes exactly what dmst_null_model computes (the same kernel), with
 * no context and no allocation of any kind: inputs and outputs are the
 * caller's DEVICE buffers, and the kernel's scratch is a fixed file-scope
 * device array of 8,391,168 bytes (a 2 KiB header plus 2 x 32 x (L+1) 8-byte
 * scores for L <= DMST_NOALLOC_MAX_LEN).
 *
 *   codes    device pointer, `length` codon codes 0..24 (dmst_decode_letters);
 *            a larger code yields meaningless seeds but reads stay in bounds
 *   length   1 .. DMST_NOALLOC_MAX_LEN; larger returns DMST_ERANGE
 *   bg       HOST pointer, 29 floats (bg_probs, as for dmst_profile_add)
 *   opts     HOST pointer to the rates (insert1..delete2 are used), or NULL
 *            for the defaults
 *   seeds    device pointer, 2*length floats: prefixSeed[0..L) then
 *            suffixSeedFromNext[0..L)
 *   scales4  device pointer, 4 floats: one-nt, two-nt and codon scales, 0
 *   stream   cudaStream_t (NULL = the legacy default stream); the work is
 *            queued there and the call returns without waiting
 *
 * The scratch is set up on the first call on each device (the current device
 * when the call is made: cudaGetSymbolAddress, return code checked), so make
 * that first call before any stream capture.  Nothing in the scratch has to
 * start at zero: the call writes every word it later reads.  Calls on one
 * device share the one scratch array, so calls whose work can overlap (two
 * streams, or two host threads) race; order them on one stream or wait for
 * the previous call's work.  The scratch address found at set-up is kept for
 * the life of the process: after cudaDeviceReset (or anything else that
 * destroys and recreates the device's primary context) it is stale, so do not
 * call this entry point again in that process.  Returns DMST_EINVAL for a null
 * pointer, a length below 1 or invalid rates, DMST_ERANGE beyond the maximum,
 * DMST_EDEVICE for a CUDA error (including set-up and launch).  An error
 * already pending from the caller's earlier CUDA work is reported as
 * DMST_EDEVICE before anything is queued, and is not cleared. */
#define DMST_NOALLOC_MAX_LEN 16384
int dmst_null_model_noalloc(const uint8_t *codes, int length, const float *bg, const dmst_opts *opts,
                            float *seeds, float *scales4, void *stream);

/* ---- calibration --------------------------------------------------------
 * Gumbel fits of the reference (estimateGumbel, dummest-calibration.hh:97-104),
 * FP64 on the host.  Sorts scores in place.  out8 = MM lambda, MM K,
 * MM K(lambda=1), ML lambda, ML K, ML K(lambda=1), L-moments lambda, L-moments K. */
int dmst_estimate_gumbel(double *scores, int n, double seq_length, double *out8);

/* The reference's random calibration sequences (estimateK's generator,
 * dummest-calibration.hh:436-483): trial t of a profile, as letter codes
 * (sequence_length + border of them).  letter_freqs = the profile's
 * background letter probabilities (bg_probs + 4). */
int dmst_calibration_sequence(const float *letter_freqs, double bg_stop_codon_prob, double insert1,
                              double insert2, double delete1, double delete2, int trial, int sequence_length,
                              int border, char *letters);

/* Calibrate a profile on the device: generate num_sequences random sequences
 * as estimateK does, score them (mode MID), and fit.  out receives
 * lambda (MM mid), K (MM mid), lambda_filter, K_filter; scores (may be NULL)
 * receives num_sequences mid ln-scores then num_sequences filter ln-scores. */
int dmst_calibrate(dmst_ctx *ctx, int profile, int sequence_length, int border, int num_sequences, double *out4,
                   double *scores);

#ifdef __cplusplus
}
#endif

#endif /* DUMMEST_B200_H */
