// Host-side model preparation for the B200 search path: HMMER3 parsing and
// profile finalization, DNA -> codon-code decoding, the reference's random
// calibration sequences, and the FP64 Gumbel fits.  Everything here runs once
// per profile / per sequence / per calibration; the per-cell work is on the
// device (dp_kernels.cuh).
//
// Each routine restates the reference's semantics in FP32 engine terms
// (Float = float) and cites the reference lines it follows.  Where the
// reference mixes float and double arithmetic, the same types are used here
// so that the finalized profile is bit-identical to the reference's.
#include "host_model.h"

#include <cerrno>
#include <climits>
#include <cstdlib>
#include <cstring>

#include <algorithm>
#include <cctype>
#include <cmath>
#include <cstring>
#include <random>
#include <sstream>
#include <string>
#include <vector>

namespace dmst {

const char kAlphabet[] = "ACDEFGHIKLMNPQRSTVWYUO?*";  // dummest-core.hh:352

// Synonymous codons per amino acid, in the reference's order
// (dummest-sequence.hh:103-124).  The order matters: the calibration generator
// picks codons by index.
static const char *codonsOf(char aa, int *n) {
    struct Entry {
        char aa;
        const char *codons;  // concatenated triplets
    };
    static const Entry table[] = {
        {'A', "GCTGCCGCAGCG"}, {'R', "CGTCGCCGACGGAGAAGG"}, {'N', "AATAAC"}, {'D', "GATGAC"},
        {'C', "TGTTGC"},       {'U', "TGTTGC"},             {'Q', "CAACAG"}, {'E', "GAAGAG"},
        {'G', "GGTGGCGGAGGG"}, {'H', "CATCAC"},             {'I', "ATTATCATA"}, {'L', "TTATTGCTTCTCCTACTG"},
        {'K', "AAAAAG"},       {'O', "AAAAAG"},             {'M', "ATG"},    {'F', "TTTTTC"},
        {'P', "CCTCCCCCACCG"}, {'S', "TCTTCCTCATCGAGTAGC"}, {'T', "ACTACCACAACG"}, {'W', "TGG"},
        {'Y', "TATTAC"},       {'V', "GTTGTCGTAGTG"},       {'*', "TAATAGTGA"}, {'?', "???"},
    };
    for (const Entry &e : table)
        if (e.aa == aa) {
            *n = (int)strlen(e.codons) / 3;
            return e.codons;
        }
    *n = 0;
    return nullptr;
}

int codonCount(char aa) {
    int n = 0;
    codonsOf(aa, &n);
    return n;
}

// The standard code as a 64-entry table over 2-bit bases A=0 C=1 G=2 T=3
// (index = 16*b0 + 4*b1 + b2), holding codon codes (alphabet indices).
// Same mapping as codonTableFlat (dummest-sequence.hh:131-178).
void standardCodeTable(uint8_t out[64]) {
    static const char bases[] = "ACGT";
    for (int b0 = 0; b0 < 4; ++b0)
        for (int b1 = 0; b1 < 4; ++b1)
            for (int b2 = 0; b2 < 4; ++b2) {
                char codon[3] = {bases[b0], bases[b1], bases[b2]};
                char aa = '?';
                for (const char *p = kAlphabet; *p && aa == '?'; ++p) {
                    int n = 0;
                    const char *cs = codonsOf(*p, &n);
                    if (*p == '?' || *p == 'U' || *p == 'O') continue;
                    for (int k = 0; k < n; ++k)
                        if (!memcmp(cs + 3 * k, codon, 3)) aa = *p;
                }
                out[16 * b0 + 4 * b1 + b2] = (uint8_t)(strchr(kAlphabet, aa) - kAlphabet);
            }
}

// ---------------------------------------------------------------------------
// HMMER3 text -> raw per-node numbers (dummest-profile.hh:235-329).
// ---------------------------------------------------------------------------

// -ln(p) text -> p; '*' is zero (dummest-profile.hh:14-19).
static double probFromText(const std::string &w) {
    if (!w.empty() && w[0] == '*') return 0;
    return std::exp(-std::strtod(w.c_str(), nullptr));
}

int parseHmmText(const char *text, size_t len, std::vector<RawProfile> &out, std::string *err) {
    // The reader's state machine: NAME and HMM lines, the column-header line,
    // an optional COMPO line, then per node an (insert line), a transition
    // line, and a match line whose numbers all contain '.'; "//" ends a
    // profile.  Values are stored as float (Float) the way the reference's
    // values vector holds them.
    std::string all(text, len);
    std::istringstream in(all);
    std::string line, word;
    RawProfile cur;
    int state = 0;
    int width = 0;
    while (std::getline(in, line)) {
        std::istringstream iss(line);
        word.clear();
        iss >> word;
        switch (state) {
        case 0:
            if (word == "NAME") {
                iss >> word;
                cur.name = word;
            } else if (word == "HMM") {
                ++state;
            }
            break;
        case 1:
            ++state;
            break;
        case 2:
            if (word != "COMPO") ++state;
            break;
        case 3: {
            std::string mi, md, im, ii, dm, dd;
            iss >> mi >> md >> im >> ii >> dm >> dd;
            if (!iss) {
                if (err) *err = "bad transition line";
                return -1;
            }
            double MtoI = probFromText(mi), MtoD = probFromText(md), ItoI = probFromText(ii),
                   DtoD = probFromText(dd);
            if (MtoI > 1 || MtoD > 1 || ItoI > 1 || DtoD > 1) {
                if (err) *err = "transition probability above 1";
                return -1;
            }
            // values row layout: MtoI, ItoI, MtoD, DtoD (dummest-profile.hh:277-280)
            cur.values.push_back((float)MtoI);
            cur.values.push_back((float)ItoI);
            cur.values.push_back((float)MtoD);
            cur.values.push_back((float)DtoD);
            ++state;
            break;
        }
        case 4:
            if (word == "//") {
                if (cur.M < 2) {
                    if (err) *err = "profile shorter than 2";
                    return -1;
                }
                cur.values.insert(cur.values.end(), width - 4, 0.0f);
                cur.width = width;
                out.push_back(cur);
                cur = RawProfile();
                width = 0;
                state = 0;
            } else {
                int k = 0;
                while (iss >> word && word.find('.') != std::string::npos) {
                    double p = probFromText(word);
                    if (p > 1) {
                        if (err) *err = "emission probability above 1";
                        return -1;
                    }
                    cur.values.push_back((float)p);
                    ++k;
                }
                cur.values.insert(cur.values.end(), kNonLetterWidth - 4, 0.0f);
                if (k == 0 || (width > 0 && k + kNonLetterWidth != width)) {
                    if (err) *err = "bad match-emission line";
                    return -1;
                }
                width = k + kNonLetterWidth;
                cur.M += 1;
                state = 2;
            }
        }
    }
    if (state != 0) {
        if (err) *err = "truncated HMMER3 text";
        return -1;
    }
    return (int)out.size();
}

// ---------------------------------------------------------------------------
// Repeat probabilities of a protein sequence: tantan (M. C. Frith, "A new
// repeat-masking method enables specific detection of homologous sequences",
// Nucleic Acids Res. 39:e23, 2011).  A hidden Markov model with a background
// state and one repeat state per offset k = 1..K, in which a letter is
// emitted with the likelihood ratio of its pair with the letter k back.  The
// forward pass runs over the sequence with the states rescaled every 16
// letters, the backward pass returns over it with the same factors, and the
// repeat probability of a letter is 1 - P(background at the letter).  The
// parameters are the ones the reference engine passes for a profile's
// consensus (tantan-wrapper.hh:13-72, the protein case): BLOSUM62 likelihood
// ratios exp(lambda s) with lambda = 0.32403216734804408 and s = -4 for
// letters outside the 20, K = 50, repeat start 0.005, repeat end 0.05, offset
// weights decaying by 0.9, no gaps.  The sums over offsets are taken as four
// interleaved partial sums, as the reference's 4-wide build takes them.
// ---------------------------------------------------------------------------
static void tantanProteinProbs(const uint8_t *seq, int n, float *prob) {
    // BLOSUM62 (Henikoff & Henikoff 1992), rows and columns in the order
    // ARNDCQEGHILKMFPSTWYV, as usually published.
    static const char kOrder[] = "ARNDCQEGHILKMFPSTWYV";
    static const signed char kBlosum[20][20] = {
        {4, -1, -2, -2, 0, -1, -1, 0, -2, -1, -1, -1, -1, -2, -1, 1, 0, -3, -2, 0},
        {-1, 5, 0, -2, -3, 1, 0, -2, 0, -3, -2, 2, -1, -3, -2, -1, -1, -3, -2, -3},
        {-2, 0, 6, 1, -3, 0, 0, 0, 1, -3, -3, 0, -2, -3, -2, 1, 0, -4, -2, -3},
        {-2, -2, 1, 6, -3, 0, 2, -1, -1, -3, -4, -1, -3, -3, -1, 0, -1, -4, -3, -3},
        {0, -3, -3, -3, 9, -3, -4, -3, -3, -1, -1, -3, -1, -2, -3, -1, -1, -2, -2, -1},
        {-1, 1, 0, 0, -3, 5, 2, -2, 0, -3, -2, 1, 0, -3, -1, 0, -1, -2, -1, -2},
        {-1, 0, 0, 2, -4, 2, 5, -2, 0, -3, -3, 1, -2, -3, -1, 0, -1, -3, -2, -2},
        {0, -2, 0, -1, -3, -2, -2, 6, -2, -4, -4, -2, -3, -3, -2, 0, -2, -2, -3, -3},
        {-2, 0, 1, -1, -3, 0, 0, -2, 8, -3, -3, -1, -2, -1, -2, -1, -2, -2, 2, -3},
        {-1, -3, -3, -3, -1, -3, -3, -4, -3, 4, 2, -3, 1, 0, -3, -2, -1, -3, -1, 3},
        {-1, -2, -3, -4, -1, -2, -3, -4, -3, 2, 4, -2, 2, 0, -3, -2, -1, -2, -1, 1},
        {-1, 2, 0, -1, -3, 1, 1, -2, -1, -3, -2, 5, -1, -3, -1, 0, -1, -3, -2, -2},
        {-1, -1, -2, -3, -1, 0, -2, -3, -2, 1, 2, -1, 5, 0, -2, -1, -1, -1, -1, 1},
        {-2, -3, -3, -3, -2, -3, -3, -3, -1, 0, 0, -3, 0, 6, -4, -2, -2, 1, 3, -1},
        {-1, -2, -2, -1, -3, -1, -1, -2, -2, -3, -3, -1, -2, -4, 7, -1, -1, -4, -3, -2},
        {1, -1, 1, 0, -1, 0, 0, 0, -1, -2, -2, 0, -1, -2, -1, 4, 1, -3, -2, -2},
        {0, -1, 0, -1, -1, -1, -1, -2, -2, -1, -1, -1, -1, -2, -1, 1, 5, -2, -2, 0},
        {-3, -3, -4, -4, -2, -2, -3, -2, -2, -3, -2, -3, -1, 1, -4, -3, -2, 11, 2, -3},
        {-2, -2, -2, -3, -2, -1, -2, -3, 2, -1, -1, -2, -1, 3, -3, -2, -2, 2, 7, -1},
        {0, -3, -3, -3, -1, -2, -2, -3, -3, 3, 1, -2, 1, -1, -2, -2, 0, -3, -1, 4},
    };
    constexpr int kLetters = 22;  // codes 20, 21 (U, O) score as the minimum
    constexpr double kLambda = 0.32403216734804408;
    constexpr int K = 50;
    constexpr double kStart = 0.005, kEnd = 0.05, kDecay = 0.9;
    constexpr int kScaleStep = 16;
    double lr[kLetters][kLetters];
    int at[20];  // the published order's index of each of our letters (ACDEFGHIKLMNPQRSTVWY)
    for (int a = 0; a < 20; ++a) at[a] = (int)(strchr(kOrder, kAlphabet[a]) - kOrder);
    for (int a = 0; a < kLetters; ++a)
        for (int b = 0; b < kLetters; ++b)
            lr[a][b] = std::exp(kLambda * (a < 20 && b < 20 ? kBlosum[at[a]][at[b]] : -4));
    auto letter = [&](int i) { return seq[i] < kLetters ? seq[i] : kLetters - 1; };

    const double b2b = 1 - kStart, f2b = kEnd, f2f = 1 - kEnd;
    std::vector<double> b2f(K), fg(K, 0.0), scale(n / kScaleStep);
    double w = kStart * ((1 - kDecay) / (1 - std::pow(kDecay, K)));  // the first offset's share
    for (int k = 0; k < K; ++k, w *= kDecay) b2f[k] = w;

    // Forward: prob[i] holds P(prefix ending in the background at i), scaled.
    double bg = 1.0;
    for (int i = 0; i < n; ++i) {
        const double *row = lr[letter(i)];
        const int off = std::min(i, K);
        double part[4] = {0, 0, 0, 0};
        int k = 0;
        for (; k + 4 <= off; k += 4)
            for (int q = 0; q < 4; ++q) {
                const double f = fg[k + q];
                part[q] += f;
                fg[k + q] = (bg * b2f[k + q] + f * f2f) * row[letter(i - k - q - 1)];
            }
        double fromFg = (part[0] + part[2]) + (part[1] + part[3]);
        for (; k < off; ++k) {
            const double f = fg[k];
            fromFg += f;
            fg[k] = (bg * b2f[k] + f * f2f) * row[letter(i - k - 1)];
        }
        bg = bg * b2b + fromFg * f2b;
        if (i % kScaleStep == kScaleStep - 1) {
            const double c = 1 / bg;
            scale[i / kScaleStep] = c;
            bg *= c;
            for (double &x : fg) x *= c;
        }
        prob[i] = (float)bg;
    }
    double fromFg = 0;
    for (double x : fg) fromFg += x;
    const double z = bg * b2b + fromFg * f2b;

    // Backward, folding each position's posterior as it passes.
    bg = b2b;
    std::fill(fg.begin(), fg.end(), f2b);
    for (int i = n - 1; i >= 0; --i) {
        const double nonRepeat = prob[i] * bg / z;
        prob[i] = 1 - (float)nonRepeat;
        if (i % kScaleStep == kScaleStep - 1) {
            const double c = scale[i / kScaleStep];
            bg *= c;
            for (double &x : fg) x *= c;
        }
        const double *row = lr[letter(i)];
        const int off = std::min(i, K);
        const double toBg = f2b * bg;
        double part[4] = {0, 0, 0, 0};
        int k = 0;
        for (; k + 4 <= off; k += 4)
            for (int q = 0; q < 4; ++q) {
                const double f = fg[k + q] * row[letter(i - k - q - 1)];
                part[q] += b2f[k + q] * f;
                fg[k + q] = toBg + f2f * f;
            }
        double toFg = (part[0] + part[2]) + (part[1] + part[3]);
        for (; k < off; ++k) {
            const double f = fg[k] * row[letter(i - k - 1)];
            toFg += b2f[k] * f;
            fg[k] = toBg + f2f * f;
        }
        bg = b2b * bg + toFg;
    }
}

// ---------------------------------------------------------------------------
// finalizeProfile (dummest-profile.hh:105-233), FP32 engine, with the
// reference's tantan masking of the consensus (isMask) and without
// letter-probability filtering.
// ---------------------------------------------------------------------------

// myMean over `length` rows at `step` (dummest-profile.hh:37-62), skipping
// the masked rows (mask may be null).
static double columnMean(const float *values, int length, int step, int meanType, const char *mask) {
    double mean = 0;
    int n = 0;
    std::vector<float> forMedian;
    for (int i = 0; i < length; ++i) {
        if (mask && mask[i]) continue;
        double v = values[(size_t)i * step];
        if (meanType == 'G') mean += std::log(std::max(v, 1e-6));
        if (meanType == 'A') mean += v;
        if (meanType == 'M') forMedian.push_back((float)v);
        ++n;
    }
    if (meanType == 'G') return std::exp(mean / n);
    if (meanType == 'A') return mean / n;
    std::sort(forMedian.begin(), forMedian.end());
    return n ? forMedian[n / 2] : 0.0;
}

int finalizeProfile(RawProfile &p, const Rates &r, int backgroundType, FinalProfile &f, std::string *err,
                    double maskThreshold) {
    const int W = p.width, M = p.M;
    const int alphabetSize = W - kNonLetterWidth;
    if (alphabetSize != 20) {
        if (err) *err = "only protein (20-letter) profiles are supported";
        return -1;
    }
    float *vals = p.values.data();
    float *end = vals + (size_t)W * M;
    const float I1 = r.insert1, I2 = r.insert2, D1 = r.delete1, D2 = r.delete2;
    const float STOP = r.stop, BGSTOP = r.bgStop;

    if (end[3] <= 0) end[3] = (float)columnMean(vals + W + 3, M - 1, W, 'G', nullptr);

    // The consensus: each match row's most probable letter, the first on
    // ties, as read (dummest-profile.hh:310-312); its letters with repeat
    // probability >= the threshold are masked (dummest-profile.hh:122-125).
    std::vector<char> masked(M, 0);
    f.maskedRows = 0;
    if (maskThreshold >= 0) {
        std::vector<uint8_t> consensus(M);
        for (int i = 0; i < M; ++i) {
            const float *letters = vals + (size_t)i * W + 4;
            consensus[i] = (uint8_t)(std::max_element(letters, letters + alphabetSize) - letters);
        }
        std::vector<float> prob(M);
        tantanProteinProbs(consensus.data(), M, prob.data());
        const float threshold = (float)maskThreshold;  // the reference's Float option
        for (int i = 0; i < M; ++i) {
            masked[i] = prob[i] >= threshold;
            f.maskedRows += masked[i];
        }
    }
    const char *mask = masked.data();

    double sumOfMeans = 0;
    for (int k = 4; k < 4 + alphabetSize; ++k) {
        double mean = columnMean(vals + k, M, W, backgroundType, mask);
        end[k] = (float)mean;
        sumOfMeans += mean;
    }
    f.bg.assign(W, 0.0f);
    for (int k = 4; k < 4 + alphabetSize; ++k) {
        end[k] = (float)((double)end[k] / sumOfMeans);
        // (1 - BG_STOP) / ncodons is float arithmetic in the FP32 engine.
        end[k] *= (1 - BGSTOP) / (float)codonCount(kAlphabet[k - 4]);
        f.bg[k] = end[k];
    }
    f.bg[4 + alphabetSize + 0] = 0;
    f.bg[4 + alphabetSize + 1] = 0;
    f.bg[4 + alphabetSize + 2] = (float)(1.0 / 64.0);
    f.bg[4 + alphabetSize + 3] = (float)(BGSTOP / 3.0);
    f.bg[4 + alphabetSize + 4] = 0;

    f.params.assign(M + 2, Params{});
    const float keepAll = 1 - I1 - I2 - D1 - D2;  // float expression, as in the reference
    for (int i = 0;; ++i) {
        float *probs = vals + (size_t)i * W;
        Params &q = f.params[i];
        double alpha = probs[0] * keepAll;  // float product
        double beta = probs[1];
        double alphaFS1 = I1, alphaFS2 = I2;
        q.alpha[0] = (float)(alpha * (1 - beta));
        q.alpha[1] = (float)alphaFS1;
        q.alpha[2] = (float)alphaFS2;
        q.beta[0] = (float)beta;
        q.beta[1] = q.beta[2] = 0;
        double delta = probs[2] * keepAll;
        double epsilon = probs[3];
        if (i == M) break;
        double epsilon1 = probs[W + 3];
        double deltaFS1 = D1, deltaFS2 = D2;
        q.delta[0] = (float)(delta * (1 - epsilon1));
        q.delta[1] = (float)deltaFS1;
        q.delta[2] = (float)deltaFS2;
        q.epsilon = (float)(epsilon * (1 - epsilon1) / (1 - epsilon));
        q.enter = (float)(1 - alpha - alphaFS1 - alphaFS2 - delta - deltaFS1 - deltaFS2);
        if (epsilon >= 1) {
            if (err) *err = "delete-to-delete probability of 1";
            return -1;
        }
        probs[2] = (float)delta;
        probs[3] = (float)epsilon;
        for (int k = 4; k < 4 + alphabetSize; ++k) {
            if (masked[i]) {  // a masked row emits the background
                probs[k] = end[k];
                continue;
            }
            double pr = probs[k];
            int nc = codonCount(kAlphabet[k - 4]);
            probs[k] = (float)((1 - STOP) * pr / nc);
        }
        probs[4 + 20] = probs[4 + 1];   // U = C
        probs[4 + 21] = probs[4 + 8];   // O = K
        probs[4 + alphabetSize + 2] = (float)(1.0 / 64.0);
        probs[4 + alphabetSize + 3] = (float)(STOP / 3.0);
        probs[4 + alphabetSize + 4] = 0.0f;
    }
    f.M = M;
    f.width = W;
    f.name = p.name;
    f.values = p.values;
    return 0;
}

// ---------------------------------------------------------------------------
// Sequences
// ---------------------------------------------------------------------------

// ASCII DNA -> letter codes (A=0 C=1 G=5 T=16, IUPAC -> 22), the FASTA reader's
// charToNumberIUPAC (dummest.cc:437-449).  Returns -1 on other characters.
int encodeDna(const char *ascii, int L, char *letters) {
    for (int i = 0; i < L; ++i) {
        int c = toupper((unsigned char)ascii[i]);
        switch (c) {
        case 'A': letters[i] = 0; break;
        case 'C': letters[i] = 1; break;
        case 'G': letters[i] = 5; break;
        case 'T': letters[i] = 16; break;
        case 'R': case 'Y': case 'S': case 'W': case 'K': case 'M':
        case 'B': case 'D': case 'H': case 'V': case 'N': letters[i] = 22; break;
        default: return -1;
        }
    }
    return L;
}

// The FASTA reader's character classes (dummest.cc:445-456): 125 for
// characters up to ' ' (skipped), 126 for '>' (a record starts), the
// protein alphabet's letter codes (either case), IUPAC ambiguity codes
// RYSWKMBDHVN as 22 (either case), 127 for everything else (ends a contig).
static const unsigned char *fastaClasses() {
    static unsigned char t[256];
    static bool built = false;
    if (!built) {
        for (int c = 0; c < 256; ++c) t[c] = c <= ' ' ? 125 : 127;
        t[(unsigned char)'>'] = 126;
        for (int i = 0; kAlphabet[i]; ++i) {
            const int c = (unsigned char)kAlphabet[i];
            t[toupper(c)] = t[tolower(c)] = (unsigned char)i;
        }
        for (const char *q = "RYSWKMBDHVN"; *q; ++q) t[(unsigned char)*q] = t[tolower((unsigned char)*q)] = 22;
        built = true;
    }
    return t;
}

// readContig (dummest-sequence.hh:6-82) over a whole text: a record is '>'
// and a name (the first word of the line); its sequence, up to the next
// '>', is cut into contigs at characters outside the classes above (each
// such character counts one position of the record, so a contig's start is
// its position in the record), with characters up to ' ' skipped.
// Empty contigs are not reported.
// std::stoi / std::stoll on text[a, b): leading whitespace, a sign, digits;
// false where they would throw (no digits, out of range).
static bool parseInteger(const char *text, size_t a, size_t b, bool asInt, long long &v) {
    std::string t(text + a, text + b);
    errno = 0;
    char *end = nullptr;
    const long long x = std::strtoll(t.c_str(), &end, 10);
    if (end == t.c_str() || errno == ERANGE) return false;
    if (asInt && (x < INT32_MIN || x > INT32_MAX)) return false;
    v = x;
    return true;
}

int fastaContigs(const char *text, size_t len, std::vector<FastaContig> &out, std::string &letters,
                 std::string *err, bool pipeline, std::vector<FastaRecord> *records) {
    const unsigned char *cls = fastaClasses();
    size_t i = 0;
    int record = -1;
    int recLen = 0;
    size_t nameOff = 0;
    int nameLen = 0;
    bool inRecord = false;
    // the pipeline fields, kept from record to record as the reader's
    // Sequence keeps them (dummest-sequence.hh:19-52)
    bool hasPipeline = false, isPlus = false;
    long long wStart = 0, wEnd = 0, trueLength = 0;
    size_t profileOff = 0;
    int profileLen = 0;
    while (i < len) {
        if (!inRecord) {
            while (i < len && isspace((unsigned char)text[i])) ++i;  // istream >> char
            if (i >= len) break;
            if (text[i] != '>') {
                if (err) *err = "bad sequence data: no '>'";
                return -1;
            }
            ++i;
            size_t lineEnd = i;
            while (lineEnd < len && text[lineEnd] != '\n') ++lineEnd;
            size_t w = i;
            while (w < lineEnd && isspace((unsigned char)text[w])) ++w;
            size_t we = w;
            while (we < lineEnd && !isspace((unsigned char)text[we])) ++we;
            if (we == w) {
                if (err) *err = "bad sequence data: no name";
                return -1;
            }
            ++record;
            nameOff = w;
            nameLen = (int)(we - w);
            size_t slash = w;
            while (slash < we && text[slash] != '/') ++slash;
            if (pipeline && slash < we) {  // "chr/start-end" then tokens
                size_t dash = slash + 1;
                while (dash < we && text[dash] != '-') ++dash;
                if (dash < we) {
                    if (!parseInteger(text, slash + 1, dash, true, wStart) ||
                        !parseInteger(text, dash + 1, we, true, wEnd)) {
                        if (err) *err = "bad window coordinates in a pipeline header";
                        return -1;
                    }
                }
                size_t lenA = 0, lenB = 0, profA = 0, profB = 0, strA = 0, strB = 0;
                bool haveLength = false, haveProfile = false, haveStrand = false;
                for (size_t t = we; t < lineEnd;) {
                    while (t < lineEnd && isspace((unsigned char)text[t])) ++t;
                    size_t te = t;
                    while (te < lineEnd && !isspace((unsigned char)text[te])) ++te;
                    if (te == t) break;
                    auto starts = [&](const char *pfx) {
                        const size_t n = strlen(pfx);
                        return te - t >= n && std::memcmp(text + t, pfx, n) == 0;
                    };
                    if (starts("length=")) {
                        lenA = t;
                        lenB = te;
                        haveLength = true;
                    } else if (starts("profile=")) {
                        profA = t;
                        profB = te;
                        haveProfile = true;
                    } else if (starts("bitscore=")) {
                    } else if (!haveStrand) {
                        strA = t;
                        strB = te;
                        haveStrand = true;
                    }
                    t = te;
                }
                if (haveLength && haveProfile && haveStrand) {
                    if (!parseInteger(text, lenA + 7, lenB, false, trueLength)) {
                        if (err) *err = "bad length in a pipeline header";
                        return -1;
                    }
                    profileOff = profA + 8;
                    profileLen = (int)(profB - profA - 8);
                    isPlus = std::string(text + strA, text + strB).find("plus_strand") != std::string::npos;
                }
                hasPipeline = true;
                nameLen = (int)(slash - w);
            }
            recLen = 0;
            if (records) records->push_back({nameOff, nameLen, 0});
            i = lineEnd < len ? lineEnd + 1 : len;
            inRecord = true;
        }
        // skip symbols that cannot start a contig, counting the visible ones
        while (i < len && text[i] != '>') {
            const unsigned char c = (unsigned char)text[i];
            if (cls[c] < 125) break;
            if (c > ' ') ++recLen;
            ++i;
        }
        const size_t first = letters.size();
        while (i < len && cls[(unsigned char)text[i]] < 126) {
            const unsigned char c = (unsigned char)text[i];
            if (c > ' ') letters.push_back((char)cls[c]);
            ++i;
        }
        const size_t n = letters.size() - first;
        if (n > (size_t)INT32_MAX / 2) {
            if (err) *err = "sequence is too long";
            return -1;
        }
        if (n == 0) {  // the record's end: the next character is '>' or the text ends
            for (size_t k = out.size(); k-- > 0 && out[k].record == record;) out[k].recordLength = recLen;
            if (records) records->back().length = recLen;
            inRecord = false;
            continue;
        }
        FastaContig fc;
        fc.record = record;
        fc.start = recLen;
        fc.length = (int)n;
        fc.nameOff = nameOff;
        fc.nameLen = nameLen;
        fc.letterOff = first;
        fc.recordLength = 0;
        fc.hasPipeline = hasPipeline;
        fc.isPlus = isPlus;
        fc.wStart = wStart;
        fc.wEnd = wEnd;
        fc.trueLength = trueLength;
        fc.profileOff = profileOff;
        fc.profileLen = profileLen;
        recLen += (int)n;
        out.push_back(fc);
    }
    for (size_t k = out.size(); k-- > 0 && out[k].record == record && out[k].recordLength == 0;)
        out[k].recordLength = recLen;  // a text ending inside its last record
    if (records && inRecord) records->back().length = recLen;
    return 0;
}

// Letter code -> 2-bit base, or -1 when it is not one of A, C, G, T.
static int letterToBase(char v) {
    switch (v) {
    case 0: return 0;
    case 1: return 1;
    case 5: return 2;
    case 16: return 3;
    default: return -1;
    }
}

// decodeSequence (dummest-sequence.hh:181-204): per base, the codon code of the
// triplet starting there; a triplet holding any non-ACGT letter is '?' (22);
// the last two bases get code 0.
int decodeLetters(const char *letters, int L, uint8_t *codes) {
    static uint8_t table[64];
    static bool built = false;
    if (!built) {
        standardCodeTable(table);
        built = true;
    }
    for (int i = 0; i < L; ++i) codes[i] = 0;
    for (int i = 0; i + 2 < L; ++i) {
        int b0 = letterToBase(letters[i]), b1 = letterToBase(letters[i + 1]), b2 = letterToBase(letters[i + 2]);
        codes[i] = (b0 < 0 || b1 < 0 || b2 < 0) ? 22 : table[16 * b0 + 4 * b1 + b2];
    }
    return L;
}

// ---------------------------------------------------------------------------
// Calibration: the random sequences of estimateK (dummest-calibration.hh:
// 365-483) and the Gumbel fits (dummest-calibration.hh:7-104).
// ---------------------------------------------------------------------------

int calibrationSequence(const float *letterFreqs, float bgStop, const Rates &r, int trial, int seqLen, int border,
                        char *out) {
    // Amino-acid frequencies: background letter prob x codon count, plus stop.
    std::vector<double> aaFreqs(21);
    for (int k = 0; k < 20; ++k) aaFreqs[k] = letterFreqs[k] * codonCount(kAlphabet[k]);
    aaFreqs[20] = bgStop;
    std::discrete_distribution<> dist(aaFreqs.begin(), aaFreqs.end());
    const float bfr1 = r.insert1 + r.delete2;  // BACKGROUND_FRAMESHIFT_RATE (float)
    const float bfr2 = r.insert2 + r.delete1;  // BACKGROUND_FRAMESHIFT_RATE_2 (float)
    const float bfr12 = bfr1 + bfr2;
    static const char letterOf[4] = {0, 1, 5, 16};  // A C G T as letter codes
    auto baseLetter = [&](char b) -> char {
        switch (b) {
        case 'A': return 0;
        case 'C': return 1;
        case 'G': return 5;
        default: return 16;
        }
    };
    std::vector<char> buf((size_t)seqLen + border + 16, 0);
    std::mt19937_64 gen(5489 + trial);
    std::uniform_int_distribution<int> distDNA(0, 3);
    std::uniform_int_distribution<int> distOffset(0, 2);
    int offset = distOffset(gen);
    for (int j = 0; j < offset; j++) buf[j] = letterOf[distDNA(gen)];
    for (int j = offset; j <= seqLen; j += 3) {
        double u = std::generate_canonical<double, 10>(gen);
        if (u < bfr1) {
            if (j <= seqLen) buf[j] = letterOf[distDNA(gen)];
            j -= 2;
            continue;
        } else if (u < bfr12) {
            if (j <= seqLen) buf[j] = letterOf[distDNA(gen)];
            if (j + 1 <= seqLen) buf[j + 1] = letterOf[distDNA(gen)];
            j -= 1;
            continue;
        }
        int x = dist(gen);
        char aa = (x < 20) ? kAlphabet[x] : '*';
        int n = 0;
        const char *cs = codonsOf(aa, &n);
        std::uniform_int_distribution<int> dist2(0, n - 1);
        const char *xx = cs + 3 * dist2(gen);
        for (int k = 0; k < 3; k++)
            if (j + k <= seqLen) buf[j + k] = baseLetter(xx[k]);
    }
    for (int j = 0; j < border; ++j) buf[seqLen + j] = buf[j];
    std::memcpy(out, buf.data(), (size_t)seqLen + border);
    return seqLen + border;
}

static double meanOf(const double *x, int n) {
    double s = 0;
    for (int i = 0; i < n; ++i) s += x[i];
    return s / n;
}

// Method of moments (dummest-calibration.hh:7-20): lambda = pi / sqrt(6 var)
// with the population variance; K = exp(lambda*mean - euler) / length.
// The reference's build (-O3, x86-64-v3) sums the squares in order but forms
// them as separate products, except the last one when n is odd, which its
// scalar loop tail fuses into the sum; and it fuses lambda*mean - euler.
static double mmLambda(const double *s, int n, double mean) {
    const double pi = 3.1415926535897932;
    double v = 0;
    for (int i = 0; i < n; ++i) {
        const double d = s[i] - mean;
        v = ((n & 1) && i == n - 1) ? std::fma(d, d, v) : v + d * d;
    }
    return pi / std::sqrt(6 * (v / n));
}
static double mmK(double mean, double lambda, double len) {
    const double euler = 0.57721566490153286;
    return std::exp(std::fma(lambda, mean, -euler)) / len;
}
// L-moments lambda (dummest-calibration.hh:22-29), on sorted scores.
static double lmLambda(const double *sorted, int n, double mean) {
    double s = 0;
    for (int i = 0; i < n; ++i) s += i * sorted[i];
    double d = 0.5 * n * (n - 1);
    return std::log(2.0) / (s / d - mean);
}
// Maximum likelihood lambda by bracketing and bisection
// (dummest-calibration.hh:31-73).
static double mlRoot(const double *s, int n, double lambda) {
    double x = 0, y = 0, z = 0;
    for (int i = 0; i < n; ++i) {
        x += s[i];
        y += std::exp(-lambda * s[i]);
        z += s[i] * std::exp(-lambda * s[i]);
    }
    return 1 / lambda - x / n + z / y;
}
static double mlLambda(const double *s, int n) {
    double lo = 1, hi = 1, x, y;
    int iters = 0;
    do {
        if (++iters > 1000) return 1.0;
        lo /= 2;
        hi *= 2;
        x = mlRoot(s, n, lo);
        y = mlRoot(s, n, hi);
    } while ((x < 0 && y < 0) || (x > 0 && y > 0));
    double gap = hi - lo;
    for (;;) {
        gap /= 2;
        double mid = lo + gap;
        if (mid <= lo) return lo;
        double z = mlRoot(s, n, mid);
        if ((x < 0 && z <= 0) || (x > 0 && z >= 0)) lo = mid;
    }
}
static double mlK(const double *s, int n, double lambda, double len) {
    double t = 0;
    for (int i = 0; i < n; ++i) t += std::exp(-lambda * s[i]);
    return n / (t * len);
}

void estimateGumbel(double *scores, int n, double len, double out[8]) {
    std::sort(scores, scores + n);
    double mean = meanOf(scores, n);
    out[0] = mmLambda(scores, n, mean);
    out[1] = mmK(mean, out[0], len);
    out[2] = mmK(mean, 1, len);
    out[3] = mlLambda(scores, n);
    out[4] = mlK(scores, n, out[3], len);
    out[5] = mlK(scores, n, 1, len);
    out[6] = lmLambda(scores, n, mean);
    out[7] = mmK(mean, out[6], len);
}

}  // namespace dmst
