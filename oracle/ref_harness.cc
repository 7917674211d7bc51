// TEST INFRASTRUCTURE ONLY -- the CPU oracle built from the reference sources.
//
// This single translation unit includes the DUMMEST reference engine headers
// (they define non-inline globals, so the engine must live in exactly one TU,
// in the include order of dummest.cc:8-17) and exposes a flat C interface to
// the reference's own hot-path routines, so that tests and the CPU-baseline leg
// of bench.py can call the unmodified reference code on explicit inputs:
//
//   readProfiles / finalizeProfile        dummest-profile.hh:235-329, :105-233
//   decodeSequence                        dummest-sequence.hh:181-204
//   findSimilarities (needAlign=false)    dummest-search.hh:9-17
//     = backwardPass + forwardPass        dummest-dp-backward.hh:444-615,
//                                         dummest-dp-forward.hh:9-547
//   findSimilaritiesBackwardOnly          dummest-dp-backward.hh:300-438
//   setupBatch (null model + seeds)       dummest-dp-backward.hh:191-297
//   estimateGumbel                        dummest-calibration.hh:97-104
//
// Built by oracle/Makefile into oracle/_ref/ (git-ignored) twice: with
// Float=float (the FP32 engine, "dummestl") and with -DDOUBLE (the FP64
// engine, "dummest").  It is never linked into, or called by, the product.
#include "dummest-core.hh"
#include "dummest-sequence.hh"
#include "dummest-output.hh"
#include "dummest-dp.hh"
#include "dummest-traceback.hh"
#include "dummest-dp-backward.hh"
#include "dummest-dp-forward.hh"
#include "dummest-search.hh"
#include "dummest-calibration.hh"
#include "dummest-profile.hh"

#include <atomic>
#include <thread>
#include <unistd.h>

namespace {

std::vector<Profile> g_profiles;
std::vector<Float> g_values;
std::vector<char> g_charVec;
std::mutex g_lock;

// The reference keeps a calibration cache that it writes at exit
// (dummest-calibration.hh:163-336); point it at a scratch directory so the
// oracle never touches a user's cache.
struct CacheDirGuard {
    CacheDirGuard() {
        std::string dir = "/tmp/dmst-oracle-cache-" + std::to_string((long)getuid());
        setenv("DUMMEST_CACHE_DIR", dir.c_str(), 0);
    }
} g_cacheDirGuard;

// Flush-to-zero for the duration of one oracle call (the reference sets it on
// every engine thread, dummest-core.hh:143-154); the caller's floating-point
// mode is restored afterwards.
struct FtzScope {
    unsigned saved;
    FtzScope() : saved(_mm_getcsr()) { enableFlushToZero(); }
    ~FtzScope() { _mm_setcsr(saved); }
};

void ensureInit() {
    static bool done = [] {
        build_standard_genetic_code();
        return true;
    }();
    (void)done;
}

const Profile *getProfile(int p) {
    if (p < 0 || p >= (int)g_profiles.size()) return nullptr;
    return &g_profiles[p];
}

// Mid and filter results of one findSimilarities(needAlign=false) batch, exactly
// as estimateK consumes them (dummest-calibration.hh:489-505).
void runBatch(const Profile &prof, std::vector<std::vector<uint8_t>> &seqs, int n, DPScratch &scratch,
              ExpScore *mid, double *midLn, ExpScore *flt) {
    std::array<std::vector<uint8_t> *, simdWidth> ptrs{};
    for (int k = 0; k < n; ++k) ptrs[k] = &seqs[k];
    std::array<Float, simdWidth> minProbRatio;
    minProbRatio.fill((Float)-2.0);
    std::array<std::vector<AlignedSimilarity>, simdWidth> sims;
    std::array<ExpScore, simdWidth> filterBest{};
    findSimilarities(sims, prof, ptrs, minProbRatio, scratch, n, &filterBest, false);
    for (int k = 0; k < n; ++k) {
        if (sims[k].size() < 3) {
            mid[k] = ExpScore{0.0f, 0};
            midLn[k] = -INFINITY;
        } else {
            mid[k] = sims[k][2].pair;
            midLn[k] = sims[k][2].logProbRatio;
        }
        flt[k] = filterBest[k];
    }
}

}  // namespace

extern "C" {

int dmstref_float_bytes(void) { return (int)sizeof(Float); }
int dmstref_simd_width(void) { return (int)simdWidth; }

// Rates are mutable globals in the reference (dummest-core.hh:115-131).
void dmstref_set_rates(double insert1, double insert2, double delete1, double delete2, double stop,
                       double bgStop) {
    std::lock_guard<std::mutex> g(g_lock);
    INSERT1 = (Float)insert1;
    INSERT2 = (Float)insert2;
    DELETE1 = (Float)delete1;
    DELETE2 = (Float)delete2;
    STOP_CODON_PROB = (Float)stop;
    BG_STOP_CODON_PROB = (Float)bgStop;
    updateBackgroundFrameshiftRates();
}

void dmstref_get_rates(double *out6) {
    out6[0] = INSERT1;
    out6[1] = INSERT2;
    out6[2] = DELETE1;
    out6[3] = DELETE2;
    out6[4] = STOP_CODON_PROB;
    out6[5] = BG_STOP_CODON_PROB;
}

// Parse an HMMER3 text file with the reference reader.  Replaces any profiles
// loaded before.  Returns the number of profiles, or -1.
int dmstref_load_profiles(const char *path, int backgroundType, int maskProfiles) {
    std::lock_guard<std::mutex> g(g_lock);
    ensureInit();
    FtzScope ftz;
    g_profiles.clear();
    g_values.clear();
    g_charVec.clear();
    std::ifstream in(path);
    if (!in) return -1;
    if (!readProfiles(in, g_profiles, g_values, g_charVec, backgroundType, maskProfiles != 0, 0.0, false))
        return -1;
    // names live in g_charVec; keep Profile::name (a std::string) as is.
    return (int)g_profiles.size();
}

int dmstref_profile_dims(int p, int *M, int *width) {
    const Profile *pr = getProfile(p);
    if (!pr) return -1;
    *M = pr->length;
    *width = pr->width;
    return 0;
}

const char *dmstref_profile_name(int p) {
    const Profile *pr = getProfile(p);
    return pr ? pr->name.c_str() : "";
}

// values: (M+1)*width, params: (M+2)*11 (alpha'[3] beta'[3] delta'[3] eps' enter),
// bg: width.  Converted to float (the FP64 build rounds here).
int dmstref_profile_export(int p, float *values, float *params, float *bg) {
    const Profile *pr = getProfile(p);
    if (!pr) return -1;
    const int M = pr->length, W = pr->width;
    for (int i = 0; i < (M + 1) * W; ++i) values[i] = (float)pr->values[i];
    for (int i = 0; i < M + 2; ++i) {
        const Params &q = pr->values_v2[i];
        float *o = params + 11 * i;
        for (int t = 0; t < 3; ++t) {
            o[t] = (float)q.alpha_prime[t];
            o[3 + t] = (float)q.beta_prime[t];
            o[6 + t] = (float)q.delta_prime[t];
        }
        o[9] = (float)q.epsilon_prime;
        o[10] = (float)q.enter_match_probability;
    }
    for (int k = 0; k < W; ++k) bg[k] = (float)pr->bg_probs[k];
    return 0;
}

// ASCII DNA -> the engine's letter codes, as main() reads FASTA with IUPAC
// ambiguity mapped to the masked letter (dummest.cc:437-449).  Returns L or -1.
int dmstref_encode_dna(const char *ascii, int L, char *out) {
    ensureInit();
    FtzScope ftz;
    char charToNumber[256];
    memset(charToNumber, 127, 256);
    setCharToNumber(charToNumber, getAlphabet(20));
    for (auto c : "RYSWKMBDHVN")
        if (c != '\0') charToNumber[(unsigned char)c] = charToNumber[tolower(c)] = 22;
    for (int i = 0; i < L; ++i) {
        char v = charToNumber[(unsigned char)ascii[i]];
        if (v == 127) return -1;
        out[i] = v;
    }
    return L;
}

// Letter codes (length L) -> per-base codon codes (dummest-sequence.hh:181-204).
int dmstref_decode(const char *codes, int L, uint8_t *out) {
    ensureInit();
    FtzScope ftz;
    char charToNumber[256];
    memset(charToNumber, 0, 256);
    const char *alphabet = getAlphabet(20);
    setCharToNumber(charToNumber, alphabet);
    std::vector<uint8_t> d = decodeSequence(codes, L, alphabet, charToNumber);
    std::copy(d.begin(), d.end(), out);
    return L;
}

// tantan masking of a DNA strand (dummest-sequence.hh:206-236).  buf holds the
// L letter codes followed by room for L more; the masked copy lands there.
int dmstref_mask_sequence(char *buf, int L) {
    ensureInit();
    FtzScope ftz;
    makeMaskedSequence(buf, L, 20);
    return L;
}

// One findSimilarities(needAlign=false) call on n <= simdWidth decoded
// sequences: the calibration mid score (pair and ln) and the exact filter best.
int dmstref_find_similarities(int p, const uint8_t *const *decoded, const int *lens, int n, float *midM,
                              int *midE, double *midLn, float *fltM, int *fltE) {
    ensureInit();
    FtzScope ftz;
    const Profile *pr = getProfile(p);
    if (!pr || n < 1 || n > (int)simdWidth) return -1;
    std::vector<std::vector<uint8_t>> seqs(n);
    for (int k = 0; k < n; ++k) {
        if (lens[k] < 3) return -1;
        seqs[k].assign(decoded[k], decoded[k] + lens[k]);
    }
    thread_local DPScratch scratch;
    ExpScore mid[simdWidth], flt[simdWidth];
    double ln[simdWidth];
    runBatch(*pr, seqs, n, scratch, mid, ln, flt);
    for (int k = 0; k < n; ++k) {
        midM[k] = mid[k].m;
        midE[k] = mid[k].e;
        midLn[k] = ln[k];
        fltM[k] = flt[k].m;
        fltE[k] = flt[k].e;
    }
    return 0;
}

// The per-column anchors of one sequence's hit path, read from the
// reference's own trackers after findSimilarities: for each column j the
// largest wMid over the rows (bestMidScorePhys) and its row (bestMidRowPhys)
// (dummest-dp-forward.hh:196-206).
int dmstref_anchors(int p, const uint8_t *codes, int L, float *bestM, int *bestE, int *row) {
    ensureInit();
    FtzScope ftz;
    const Profile *pr = getProfile(p);
    if (!pr || L < 3 || !bestM || !bestE || !row) return -1;
    std::vector<std::vector<uint8_t>> seqs(1);
    seqs[0].assign(codes, codes + L);
    DPScratch scratch;
    ExpScore mid[simdWidth], flt[simdWidth];
    double ln[simdWidth];
    runBatch(*pr, seqs, 1, scratch, mid, ln, flt);
    for (int j = 0; j < L; ++j) {
        bestM[j] = scratch.bestMidScorePhys[j][0].m;
        bestE[j] = scratch.bestMidScorePhys[j][0].e;
        row[j] = scratch.bestMidRowPhys[j][0];
    }
    return 0;
}

// The hit path with alignments: findSimilarities(needAlign=true) on n <=
// simdWidth lanes with per-lane minProbRatio (dummest-search.hh:9-17,
// dummest-dp-forward.hh:471-535, dummest-traceback.hh:35-118).  Every
// AlignedSimilarity of every lane, in the order the engine produced them:
// lane[s], pair (m, e), logProbRatio, anchor1, anchor2, and its segment pairs
// segs[3 k .. 3 k + 3) = (start1, start2, length) for k in
// [segOff[s], segOff[s + 1]).  Returns the number of similarities; -1 on bad
// input; -(1 + similarities) when simCap or segCap is too small (then
// *needSegs holds the segments needed and nothing else is written).
int dmstref_align(int p, const uint8_t *const *decoded, const int *lens, const float *minProbRatio, int n,
                  int simCap, int *lane, float *pairM, int *pairE, double *logRatio, int *anchor1, int *anchor2,
                  int *segOff, int segCap, int *segs, int *needSegs) {
    ensureInit();
    FtzScope ftz;
    const Profile *pr = getProfile(p);
    if (!pr || n < 1 || n > (int)simdWidth) return -1;
    std::vector<std::vector<uint8_t>> seqs(n);
    std::array<std::vector<uint8_t> *, simdWidth> ptrs{};
    std::array<Float, simdWidth> mpr;
    mpr.fill((Float)-2.0);
    for (int k = 0; k < n; ++k) {
        if (lens[k] < 3) return -1;
        seqs[k].assign(decoded[k], decoded[k] + lens[k]);
        ptrs[k] = &seqs[k];
        mpr[k] = (Float)minProbRatio[k];
    }
    DPScratch scratch;
    std::array<std::vector<AlignedSimilarity>, simdWidth> sims;
    findSimilarities(sims, *pr, ptrs, mpr, scratch, n, nullptr, true);
    int ns = 0, nseg = 0;
    for (int k = 0; k < n; ++k)
        for (const auto &x : sims[k]) {
            ++ns;
            nseg += (int)x.alignment.size();
        }
    if (needSegs) *needSegs = nseg;
    if (ns > simCap || nseg > segCap) return -(1 + ns);
    int s = 0, g = 0;
    for (int k = 0; k < n; ++k)
        for (const auto &x : sims[k]) {
            lane[s] = k;
            pairM[s] = x.pair.m;
            pairE[s] = x.pair.e;
            logRatio[s] = x.logProbRatio;
            anchor1[s] = x.anchor1;
            anchor2[s] = x.anchor2;
            segOff[s] = g;
            for (const auto &a : x.alignment) {
                segs[3 * g] = a.start1;
                segs[3 * g + 1] = a.start2;
                segs[3 * g + 2] = a.length;
                ++g;
            }
            ++s;
        }
    segOff[s] = g;
    return ns;
}

// The reference's FASTA reader over a text: readContig (dummest-sequence.hh:6-82)
// with the IUPAC character classes the engine builds for protein profiles
// (dummest.cc:445-456), called in the engine's loop (dummest.cc:553-555).
// Per contig: its record index, Contig::start and length; letters = the
// contigs' codes concatenated; names = each record's name followed by '\n'.
// Returns the number of contigs, or -(2 + needed) when a capacity is too
// small.  The reader aborts on malformed input (dummest-util.hh:19-22): only
// well-formed texts may be given.
int dmstref_read_fasta(const char *text, long long len, int *record, int *start, int *length, int cap,
                       char *letters, long long capLetters, char *names, long long capNames) {
    ensureInit();
    const char *alphabet = getAlphabet(20);
    char charToNumber[256];
    memset(charToNumber, 127, 256);
    memset(charToNumber, 125, ' ' + 1);
    charToNumber['>'] = 126;
    setCharToNumber(charToNumber, alphabet);
    char iupac[256];
    std::copy(charToNumber, charToNumber + 256, iupac);
    for (auto c : "RYSWKMBDHVN")
        if (c != '\0') iupac[(unsigned char)c] = iupac[tolower(c)] = 22;
    std::istringstream in(std::string(text, (size_t)len));
    Sequence sequence{};
    Contig contig{0, 0};
    std::vector<char> vec;
    std::vector<int> rec, st, ln;
    std::string lt, nm;
    size_t lastName = (size_t)-1;
    int nrec = -1;
    while (readContig(in, sequence, contig, vec, iupac)) {
        if (sequence.nameIdx != lastName) {
            lastName = sequence.nameIdx;
            ++nrec;
            nm += std::string(&vec[sequence.nameIdx]) + "\n";
        }
        if (contig.length == 0) continue;
        rec.push_back(nrec);
        st.push_back(contig.start);
        ln.push_back(contig.length);
        lt.append(&vec[vec.size() - contig.length], contig.length);
    }
    if ((int)rec.size() > cap || (long long)lt.size() > capLetters || (long long)nm.size() > capNames)
        return -(2 + (int)std::max({rec.size(), lt.size(), nm.size()}));
    for (size_t k = 0; k < rec.size(); ++k) {
        record[k] = rec[k];
        start[k] = st[k];
        length[k] = ln[k];
    }
    std::memcpy(letters, lt.data(), lt.size());
    std::memcpy(names, nm.data(), nm.size());
    return (int)rec.size();
}

// The engine's sequence loop without its scoring (dummest.cc:553-606, no
// masking): every contig read (readContig with the IUPAC classes,
// dummest.cc:445-456), padded as the engine pads it and decoded
// (decodeSequence).  Returns the contigs' total length; *checksum gets the sum
// of the decoded codes times their position + 1.
long long dmstref_read_decode(const char *text, long long len, long long *checksum) {
    ensureInit();
    const char *alphabet = getAlphabet(20);
    char charToNumber[256];
    memset(charToNumber, 127, 256);
    memset(charToNumber, 125, ' ' + 1);
    charToNumber['>'] = 126;
    setCharToNumber(charToNumber, alphabet);
    char iupac[256];
    std::copy(charToNumber, charToNumber + 256, iupac);
    for (auto c : "RYSWKMBDHVN")
        if (c != '\0') iupac[(unsigned char)c] = iupac[tolower(c)] = 22;
    std::istringstream in(std::string(text, (size_t)len));
    Sequence sequence{};
    Contig contig{0, 0};
    std::vector<char> vec;
    long long total = 0, sum = 0;
    while (readContig(in, sequence, contig, vec, iupac)) {
        if (contig.length == 0) continue;
        const size_t seqIdx = vec.size() - contig.length;
        vec.resize(seqIdx + simdRoundUp(contig.length + 1));
        std::vector<uint8_t> d = decodeSequence(&vec[seqIdx], contig.length, alphabet, charToNumber);
        for (size_t k = 0; k < d.size(); ++k) sum += (long long)d[k] * (long long)(k + 1);
        total += contig.length;
        vec.resize(seqIdx);
    }
    if (checksum) *checksum = sum;
    return total;
}

#ifdef PIPELINE_MODE
// The reader of the PIPELINE_MODE build (dummest-sequence.hh:19-52): per
// contig also its record's header fields as the reader left them in
// `sequence` (fields: has_pipeline_fields, w_start, w_end, true_length,
// is_plus); names gets "name\tprofile\n" per record (name = the part before
// '/').  Only well-formed texts (the reader throws or aborts otherwise).
int dmstref_read_fasta_pipeline(const char *text, long long len, int *record, int *start, int *length,
                                long long *fields, int cap, char *names, long long capNames) {
    ensureInit();
    const char *alphabet = getAlphabet(20);
    char charToNumber[256];
    memset(charToNumber, 127, 256);
    memset(charToNumber, 125, ' ' + 1);
    charToNumber['>'] = 126;
    setCharToNumber(charToNumber, alphabet);
    char iupac[256];
    std::copy(charToNumber, charToNumber + 256, iupac);
    for (auto c : "RYSWKMBDHVN")
        if (c != '\0') iupac[(unsigned char)c] = iupac[tolower(c)] = 22;
    std::istringstream in(std::string(text, (size_t)len));
    Sequence sequence{};
    Contig contig{0, 0};
    std::vector<char> vec;
    std::string nm;
    size_t lastName = (size_t)-1;
    int nrec = -1, n = 0;
    while (readContig(in, sequence, contig, vec, iupac)) {
        if (sequence.nameIdx != lastName) {
            lastName = sequence.nameIdx;
            ++nrec;
            nm += std::string(&vec[sequence.nameIdx]) + "\t" + sequence.target_profile + "\n";
        }
        if (contig.length == 0) continue;
        if (n >= cap) return -2;
        record[n] = nrec;
        start[n] = contig.start;
        length[n] = contig.length;
        long long *f = fields + 5 * n;
        f[0] = sequence.has_pipeline_fields ? 1 : 0;
        f[1] = (long long)sequence.w_start;
        f[2] = (long long)sequence.w_end;
        f[3] = (long long)sequence.true_length;
        f[4] = sequence.is_plus ? 1 : 0;
        ++n;
    }
    if ((long long)nm.size() > capNames) return -2;
    std::memcpy(names, nm.data(), nm.size());
    return n;
}
#endif

// The lean float filter (findSimilaritiesBackwardOnly) on n <= simdWidth lanes.
int dmstref_backward_only(int p, const uint8_t *const *decoded, const int *lens, int n, float *best) {
    ensureInit();
    FtzScope ftz;
    const Profile *pr = getProfile(p);
    if (!pr || n < 1 || n > (int)simdWidth) return -1;
    std::vector<std::vector<uint8_t>> seqs(n);
    std::array<std::vector<uint8_t> *, simdWidth> ptrs{};
    for (int k = 0; k < n; ++k) {
        if (lens[k] < 3) return -1;
        seqs[k].assign(decoded[k], decoded[k] + lens[k]);
        ptrs[k] = &seqs[k];
    }
    thread_local DPScratch scratch;
    std::array<Float, simdWidth> b;
    findSimilaritiesBackwardOnly(b, *pr, ptrs, scratch, n);
    for (int k = 0; k < n; ++k) best[k] = (float)b[k];
    return 0;
}

// Many sequences against one profile, the way the reference schedules them
// (dummest-search.hh:111-117, :201-208): sorted by length (descending), cut
// into <= simdWidth-lane batches, batches pulled by nthreads workers, each
// worker with its own DPScratch and flush-to-zero set.  mode 0: backward +
// forward mid score (needAlign=false) plus the exact filter best; mode 1: the
// lean float filter only.  Outputs are per input sequence (input order).
int dmstref_score_many(int p, const uint8_t *codes, const int64_t *offsets, int nseq, int nthreads, int mode,
                       double *midLn, double *fltLn) {
    ensureInit();
    FtzScope ftz;
    const Profile *pr = getProfile(p);
    if (!pr || nseq < 0 || nthreads < 1) return -1;
    std::vector<int> order(nseq);
    for (int i = 0; i < nseq; ++i) {
        order[i] = i;
        if (offsets[i + 1] - offsets[i] < 3) return -1;
    }
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) {
        return offsets[a + 1] - offsets[a] > offsets[b + 1] - offsets[b];
    });
    const int nb = (nseq + (int)simdWidth - 1) / (int)simdWidth;
    std::atomic<int> next{0};
    auto worker = [&]() {
        enableFlushToZero();
        DPScratch scratch;
        std::vector<std::vector<uint8_t>> seqs(simdWidth);
        for (;;) {
            int b = next.fetch_add(1);
            if (b >= nb) break;
            int start = b * (int)simdWidth;
            int n = std::min((int)simdWidth, nseq - start);
            for (int k = 0; k < n; ++k) {
                int s = order[start + k];
                seqs[k].assign(codes + offsets[s], codes + offsets[s + 1]);
            }
            if (mode == 0) {
                ExpScore mid[simdWidth], flt[simdWidth];
                double ln[simdWidth];
                runBatch(*pr, seqs, n, scratch, mid, ln, flt);
                for (int k = 0; k < n; ++k) {
                    int s = order[start + k];
                    midLn[s] = ln[k];
                    fltLn[s] = scoreToLog(flt[k]);
                }
            } else {
                std::array<std::vector<uint8_t> *, simdWidth> ptrs{};
                for (int k = 0; k < n; ++k) ptrs[k] = &seqs[k];
                std::array<Float, simdWidth> best;
                findSimilaritiesBackwardOnly(best, *pr, ptrs, scratch, n);
                for (int k = 0; k < n; ++k) {
                    int s = order[start + k];
                    fltLn[s] = std::log((double)best[k]);
                    if (midLn) midLn[s] = NAN;
                }
            }
        }
    };
    std::vector<std::thread> pool;
    for (int t = 1; t < nthreads; ++t) pool.emplace_back(worker);
    worker();
    for (auto &t : pool) t.join();
    return 0;
}

// Null model of one sequence (setupBatch, dummest-dp-backward.hh:191-297):
// prefixSeed[0..L), suffixSeedFromNext[0..L) as stored Float lanes, and the
// three per-base scales (one-nt, two-nt, codon) as packed Float lanes.
int dmstref_null_model(int p, const uint8_t *decoded, int L, float *prefixSeed, float *sufSeed, float *scales) {
    ensureInit();
    FtzScope ftz;
    const Profile *pr = getProfile(p);
    if (!pr || L < 3) return -1;
    std::vector<uint8_t> seq(decoded, decoded + L);
    std::array<std::vector<uint8_t> *, simdWidth> ptrs{};
    ptrs[0] = &seq;
    thread_local DPScratch scratch;
    BackwardCtx ctx;
    setupBatch(*pr, ptrs, scratch, 1, ctx, false);
    alignas(64) Float buf[simdWidth];
    for (int j = 0; j < L; ++j) {
        Kokkos::Experimental::simd_unchecked_store(scratch.nullPrefixSeed[j], buf,
                                                   Kokkos::Experimental::simd_flag_default);
        prefixSeed[j] = (float)buf[0];
        Kokkos::Experimental::simd_unchecked_store(scratch.nullSuffixSeedFromNext[j], buf,
                                                   Kokkos::Experimental::simd_flag_default);
        sufSeed[j] = (float)buf[0];
    }
    Kokkos::Experimental::simd_unchecked_store(ctx.nullScaleOneNucleotide, buf, Kokkos::Experimental::simd_flag_default);
    scales[0] = (float)buf[0];
    Kokkos::Experimental::simd_unchecked_store(ctx.nullScaleTwoNucleotide, buf, Kokkos::Experimental::simd_flag_default);
    scales[1] = (float)buf[0];
    Kokkos::Experimental::simd_unchecked_store(ctx.nullScaleCodon, buf, Kokkos::Experimental::simd_flag_default);
    scales[2] = (float)buf[0];
    return 0;
}

// Full backward W1 matrix of one sequence (rows 0..M, columns 0..L) and the
// per-row rescale counts, for cell-by-cell comparisons on small cases.
int dmstref_backward_matrix(int p, const uint8_t *decoded, int L, float *W1, int *counts) {
    ensureInit();
    FtzScope ftz;
    const Profile *pr = getProfile(p);
    if (!pr || L < 3) return -1;
    std::vector<uint8_t> seq(decoded, decoded + L);
    std::array<std::vector<uint8_t> *, simdWidth> ptrs{};
    ptrs[0] = &seq;
    thread_local DPScratch scratch;
    BackwardCtx ctx;
    backwardPass(*pr, ptrs, scratch, 1, nullptr, ctx, false);
    alignas(64) Float buf[simdWidth];
    for (int i = 0; i <= pr->length; ++i) {
        for (int j = 0; j < L; ++j) {
            Kokkos::Experimental::simd_unchecked_store(scratch.W1.get(i, j), buf,
                                                       Kokkos::Experimental::simd_flag_default);
            W1[(size_t)i * L + j] = (float)buf[0];
        }
        counts[i] = scratch.backwardRescaleCount[i][0];
    }
    return 0;
}

// Gumbel fits of the reference (dummest-calibration.hh:97-104).  Sorts scores
// in place.  out8: MM lambda, MM K, MM K(lambda=1), ML lambda, ML K,
// ML K(lambda=1), L-moments lambda, L-moments K.
void dmstref_estimate_gumbel(double *scores, int n, double seqLength, double *out8) {
    estimateGumbel(out8[0], out8[1], out8[2], out8[3], out8[4], out8[5], out8[6], out8[7], scores, n, seqLength);
}

// The reference's own calibration of profile p, estimateK
// (dummest-calibration.hh:338-649), called the way dummest.cc:395-408 calls
// it: letter frequencies = the profile's background row, nthreads workers.
// out4 = lambda (MM, mid), K (MM, mid), lambda_filter, K_filter.  With
// scoresPath the per-trial scores go to that file (estimateK then bypasses
// its cache), as the CLI's scores option does.
int dmstref_estimate_k(int p, int seqLen, int border, int num, int nthreads, const char *scoresPath,
                       double *out4) {
    ensureInit();
    FtzScope ftz;
    const Profile *pr = getProfile(p);
    if (!pr || seqLen < 1 || border < 0 || num < 2 || nthreads < 1 || !out4) return -1;
    Profile prof = *pr;  // estimateK stores lambda/K into the profile
    const Float *bgProbs = prof.values + prof.width * prof.length + 4;
    std::vector<char> buf(seqLen + border + 64);
    std::ofstream scores;
    if (scoresPath) scores.open(scoresPath);
    {
        ThreadPool pool(nthreads);
        std::vector<DPScratch> scratches(nthreads);
        estimateK(prof, bgProbs, buf.data(), seqLen, border, num, 0, pool, scratches,
                  scoresPath ? &scores : nullptr, nullptr);
    }
    out4[0] = prof.lambda;
    out4[1] = prof.gumbelKmidAnchored;
    out4[2] = prof.lambda_filter;
    out4[3] = prof.gumbel_k_filter;
    return 0;
}

}  // extern "C"
