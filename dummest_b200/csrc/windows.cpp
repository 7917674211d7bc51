// Windows of the pipeline's prefilter hits: the step between the prefilter
// and the engine, restated from the pipeline driver.
//
//   bin/dummest:91-183   _stream_bed_from_convertalis: one BED interval per
//                        BLAST-tab hit row, centred on the hit and padded by
//                        3 x the profile length on each side, named by the
//                        fake chromosome "target|query|strand";
//   bin/dummest:663-676  bedtools sort | bedtools merge | awk (_AWK_UNPACK,
//                        bin/dummest:77-88) | bedtools getfasta -s -name+:
//                        per fake chromosome the intervals sorted by start
//                        and merged where they overlap or touch, unpacked
//                        into (chromosome, start, end, profile, strand) and
//                        cut from the genome, reverse-complemented on '-'.
//
// bedtools is the Ubuntu 24.04 package (2.31.1) that the reference's container
// installs; the sort, merge and getfasta behaviour restated here is its
// documented behaviour: chromosomes in byte order, then start; intervals merged
// while the next start is <= the current end (book-ended ones included);
// intervals of unknown chromosomes, or past a chromosome's end, skipped with a
// warning; an interval whose start is past its end is an error.
#include "host_model.h"

#include <algorithm>
#include <cctype>
#include <climits>
#include <map>
#include <string>
#include <unordered_map>
#include <vector>

namespace dmst {

namespace {

bool isSpaceByte(unsigned char c) { return c == ' ' || (c >= '\t' && c <= '\r'); }

// Python's int() of a bytes token: an optional sign, then digits with single
// underscores between them.  False where int() raises ValueError, and for
// values outside int64 (which int() takes but no genome coordinate reaches).
bool pyInt(const char *a, const char *b, long long &v) {
    while (a < b && isSpaceByte((unsigned char)*a)) ++a;
    while (b > a && isSpaceByte((unsigned char)b[-1])) --b;
    bool neg = false;
    if (a < b && (*a == '+' || *a == '-')) neg = *a++ == '-';
    if (a == b || !isdigit((unsigned char)*a) || !isdigit((unsigned char)b[-1])) return false;
    unsigned long long x = 0;
    for (const char *p = a; p < b; ++p) {
        if (*p == '_') {
            if (!isdigit((unsigned char)p[1])) return false;  // a digit follows (p[1] < b: b[-1] is a digit)
            continue;
        }
        if (!isdigit((unsigned char)*p)) return false;
        x = x * 10 + (unsigned)(*p - '0');
        if (x > (unsigned long long)LLONG_MAX) return false;
    }
    v = neg ? -(long long)x : (long long)x;
    return true;
}

long long floorDiv2(long long x) { return x >= 0 ? x / 2 : -((-x + 1) / 2); }

struct Interval {
    long long start, end;
};

struct FakeChrom {
    std::vector<Interval> iv;
    size_t queryOff;  // the query of its first row, in the text
    size_t queryLen;
    int record;       // the target's index (-1: none)
};

}  // namespace

int windowsFromHits(const char *tab, size_t len, bool targetIsContig, const std::vector<std::string> &recordNames,
                    const std::vector<long long> &recordLengths, const std::vector<std::string> &profileNames,
                    const std::vector<long long> &profileLengths, std::vector<HitWindow> &out, size_t &malformed,
                    size_t &dropped, std::string *err) {
    // the driver's dictionaries: a later entry of the same name replaces an earlier one
    std::unordered_map<std::string, int> recIdx, profIdx;
    for (size_t k = 0; k < recordNames.size(); ++k) recIdx[recordNames[k]] = (int)k;
    for (size_t k = 0; k < profileNames.size(); ++k) profIdx[profileNames[k]] = (int)k;
    std::map<std::string, FakeChrom> chroms;  // bedtools sort: chromosomes in byte order
    malformed = 0;
    dropped = 0;
    out.clear();
    std::vector<std::pair<const char *, const char *>> f;
    for (size_t i = 0; i < len;) {
        size_t e = i;
        while (e < len && tab[e] != '\n') ++e;
        const char *ln = tab + i, *le = tab + e;
        i = e < len ? e + 1 : len;
        if (ln < le && *ln == '#') continue;
        f.clear();
        for (const char *p = ln; p < le;) {
            while (p < le && isSpaceByte((unsigned char)*p)) ++p;
            const char *q = p;
            while (q < le && !isSpaceByte((unsigned char)*q)) ++q;
            if (q > p) f.emplace_back(p, q);
            p = q;
        }
        if (f.size() < 12) continue;
        long long c6, c7, tStart, tEnd;
        if (!pyInt(f[6].first, f[6].second, c6) || !pyInt(f[7].first, f[7].second, c7) ||
            !pyInt(f[8].first, f[8].second, tStart) || !pyInt(f[9].first, f[9].second, tEnd)) {
            ++malformed;
            continue;
        }
        const std::string query(f[0].first, f[0].second), target(f[1].first, f[1].second);
        std::string targetBase;
        char strand;
        long long frameVal = 0;
        if (targetIsContig) {
            targetBase = target;
            strand = tStart <= tEnd ? '+' : '-';
        } else {
            const size_t us = target.rfind('_');  // rsplit('_', 1)
            targetBase = us == std::string::npos ? std::string() : target.substr(0, us);
            const std::string frameStr = us == std::string::npos ? target : target.substr(us + 1);
            const size_t eq = frameStr.find('=');  // split('=')[1]
            if (eq == std::string::npos) {
                ++malformed;
                continue;
            }
            size_t eq2 = frameStr.find('=', eq + 1);
            if (eq2 == std::string::npos) eq2 = frameStr.size();
            if (!pyInt(frameStr.data() + eq + 1, frameStr.data() + eq2, frameVal)) {
                ++malformed;
                continue;
            }
            strand = frameVal > 0 ? '+' : '-';
        }
        const auto ri = recIdx.find(targetBase);
        const long long L = ri == recIdx.end() ? 0 : recordLengths[ri->second];
        if (L == 0) continue;
        const auto pi = profIdx.find(query);
        const long long pad = 3 * (pi == profIdx.end() ? 0 : profileLengths[pi->second]);
        long long start, end;
        if (targetIsContig) {
            const long long center = floorDiv2(tStart + tEnd);
            start = std::max(0LL, center - 1 - pad);
            end = std::min(L, center + pad);
        } else {
            const long long pPos = std::max(1LL, floorDiv2(tStart + tEnd));
            const long long frame = frameVal < 0 ? -frameVal : frameVal;
            const long long basePos = (frame - 1) + 3 * (pPos - 1);
            if (strand == '+') {
                start = std::max(0LL, basePos - pad);
                end = std::min(L, basePos + 1 + pad);
            } else {
                start = std::max(0LL, L - basePos - 1 - pad);
                end = std::min(L, L - basePos + pad);
            }
        }
        if (start > end) {  // bedtools sort rejects the interval and the pipeline stops
            if (err)
                *err = "hit row gives a window whose start " + std::to_string(start) + " is past its end " +
                       std::to_string(end) + " (target " + target + ")";
            return -1;
        }
        const std::string fake = targetBase + "|" + query + "|" + strand;
        auto it = chroms.find(fake);
        if (it == chroms.end()) {
            FakeChrom fc;
            fc.queryOff = (size_t)(f[0].first - tab);
            fc.queryLen = query.size();
            fc.record = -1;
            it = chroms.emplace(fake, fc).first;
        }
        it->second.iv.push_back({start, end});
    }
    for (auto &kv : chroms) {
        // _AWK_UNPACK: split the fake name at '|'; the strand is the last
        // field, the profile the one before, the chromosome the rest
        const std::string &fake = kv.first;
        const size_t s2 = fake.rfind('|');
        const size_t s1 = fake.rfind('|', s2 - 1);
        const std::string chrom = fake.substr(0, s1);
        const int strand = fake[s2 + 1] == '+' ? 1 : -1;
        const std::string profile = fake.substr(s1 + 1, s2 - s1 - 1);
        const FakeChrom &fc = kv.second;
        const size_t profOff = fc.queryOff + (fc.queryLen - profile.size());
        const auto ri = recIdx.find(chrom);
        const auto pi = profIdx.find(profile);
        std::vector<Interval> iv = fc.iv;
        std::sort(iv.begin(), iv.end(), [](const Interval &a, const Interval &b) { return a.start < b.start; });
        for (size_t k = 0; k < iv.size();) {
            long long s = iv[k].start, e = iv[k].end;
            size_t j = k + 1;
            for (; j < iv.size() && iv[j].start <= e; ++j) e = std::max(e, iv[j].end);
            k = j;
            // getfasta: unknown chromosomes and intervals past the end are skipped
            if (ri == recIdx.end() || e > recordLengths[ri->second]) {
                ++dropped;
                continue;
            }
            HitWindow w;
            w.record = ri->second;
            w.strand = strand;
            w.start = s;
            w.end = e;
            w.profileOff = profOff;
            w.profileLen = (int)profile.size();
            w.profile = pi == profIdx.end() ? -1 : pi->second;
            out.push_back(w);
        }
    }
    return 0;
}

}  // namespace dmst
