// Host-side model types and preparation routines (see host_model.cpp).
#pragma once

#include <cstddef>
#include <cstdint>
#include <string>
#include <vector>

namespace dmst {

constexpr int kNonLetterWidth = 9;  // dummest-core.hh:231
constexpr int kWidth = 29;          // 20 letters + 9 (protein profiles)
constexpr int kCodes = 25;          // codon codes 0..24; 24 is the zero pad (dummest-dp.hh:93)
constexpr int kPadCode = 24;
constexpr int kMaskCode = 22;       // '?' masked / ambiguous triplet
extern const char kAlphabet[];

// FP32 engine rates (dummest-core.hh:115-124); Float = float.
struct Rates {
    float insert1, insert2, delete1, delete2;
    float stop, bgStop;
};

// Reference Params (dummest-core.hh:233-239).
struct Params {
    float alpha[3];
    float beta[3];
    float delta[3];
    float epsilon;
    float enter;
};
static_assert(sizeof(Params) == 11 * sizeof(float), "Params must be 11 floats");

struct RawProfile {
    std::string name;
    int M = 0;
    int width = 0;
    std::vector<float> values;  // (M+1) * width, the reader's layout
};

struct FinalProfile {
    std::string name;
    int M = 0;
    int width = 0;
    std::vector<float> values;  // (M+1) * width after finalize
    std::vector<Params> params; // M + 2
    std::vector<float> bg;      // width
    int maskedRows = 0;         // consensus letters masked by tantan
};

int codonCount(char aa);
void standardCodeTable(uint8_t out[64]);
int parseHmmText(const char *text, size_t len, std::vector<RawProfile> &out, std::string *err);
// maskThreshold >= 0: tantan-mask the consensus (rows whose repeat
// probability is >= the threshold emit the background and leave the means).
int finalizeProfile(RawProfile &p, const Rates &r, int backgroundType, FinalProfile &f, std::string *err,
                    double maskThreshold = -1.0);
int encodeDna(const char *ascii, int L, char *letters);

// One contig of a FASTA text (readContig, dummest-sequence.hh:6-82).
struct FastaContig {
    int record;          // index of its record
    int start;           // Contig::start: position in the record, skipped symbols counted
    int length;
    size_t nameOff;      // the record name: the first word of its header line, in the text
    int nameLen;
    size_t letterOff;    // its letter codes in the output string
    int recordLength;    // its record's length (contigs and cutting characters)
    // pipeline headers (the reader's PIPELINE_MODE): the fields as the reader
    // holds them after its record's header
    bool hasPipeline, isPlus;
    long long wStart, wEnd, trueLength;
    size_t profileOff;
    int profileLen;
};
// One record of a FASTA text: its name and length (contigs and cutting characters).
struct FastaRecord {
    size_t nameOff;
    int nameLen;
    int length;
};
int fastaContigs(const char *text, size_t len, std::vector<FastaContig> &out, std::string &letters,
                 std::string *err, bool pipeline = false, std::vector<FastaRecord> *records = nullptr);

// One window of the pipeline's prefilter hits: a merged interval of one
// (target record, profile, strand), as bedtools getfasta -s cuts it.
struct HitWindow {
    int record;          // index among the record names
    int strand;          // +1, or -1: reverse-complemented
    long long start, end;
    size_t profileOff;   // the profile name in the hits text
    int profileLen;
    int profile;         // index among the profile names, -1 when not among them
};
int windowsFromHits(const char *tab, size_t len, bool targetIsContig, const std::vector<std::string> &recordNames,
                    const std::vector<long long> &recordLengths, const std::vector<std::string> &profileNames,
                    const std::vector<long long> &profileLengths, std::vector<HitWindow> &out, size_t &malformed,
                    size_t &dropped, std::string *err);
int decodeLetters(const char *letters, int L, uint8_t *codes);
int calibrationSequence(const float *letterFreqs, float bgStop, const Rates &r, int trial, int seqLen, int border,
                        char *out);
void estimateGumbel(double *scores, int n, double len, double out[8]);

}  // namespace dmst
