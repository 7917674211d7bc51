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
#include <string>
#include <string_view>
#include <system_error>
#include <thread>
#include <unordered_map>
#include <vector>

namespace dmst {

namespace {

bool isSpaceByte(unsigned char c) { return c == ' ' || (c >= '\t' && c <= '\r'); }

// Python's int() of a bytes token: an optional sign, then digits with single
// underscores between them.  False where int() raises ValueError, and for
// values outside int64 (which int() takes but no genome coordinate reaches):
// such a row counts as malformed and gives no window.
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
        const unsigned digit = (unsigned)(*p - '0');
        // checked before the multiply, so that no intermediate wraps past 2^64
        if (x > ((unsigned long long)LLONG_MAX - digit) / 10) return false;
        x = x * 10 + digit;
    }
    v = neg ? -(long long)x : (long long)x;
    return true;
}

long long floorDiv2(long long x) { return x >= 0 ? x / 2 : -((-x + 1) / 2); }

struct Interval {
    long long start, end;
};

// The rows of one fake chromosome "target|query|strand" (bedtools sort's
// chromosome): the target's record, the query (its profile index, or its text
// for a query not among the profile names) and the strand.
struct FakeChrom {
    std::vector<Interval> iv;
    size_t queryOff;  // the query of its first row, in the text
    size_t queryLen;
    int record;
    char strand;
};

}  // namespace

int windowsFromHits(const char *tab, size_t len, bool targetIsContig, const std::vector<std::string> &recordNames,
                    const std::vector<long long> &recordLengths, const std::vector<std::string> &profileNames,
                    const std::vector<long long> &profileLengths, std::vector<HitWindow> &out, size_t &malformed,
                    size_t &dropped, std::string *err) {
    // the driver's dictionaries: a later entry of the same name replaces an
    // earlier one.  Keys view the names (and, for queries not among the
    // profile names, the text), which outlive the call's maps.
    std::unordered_map<std::string_view, int> recIdx, profIdx, otherQuery;
    for (size_t k = 0; k < recordNames.size(); ++k) recIdx[recordNames[k]] = (int)k;
    for (size_t k = 0; k < profileNames.size(); ++k) profIdx[profileNames[k]] = (int)k;
    malformed = 0;
    dropped = 0;
    out.clear();
    // the rows, parsed in line-aligned parts of the text on several threads
    // (the maps above are only read), then grouped in text order
    struct Row {
        int record, profile;  // profile -1: the query is not among the profile names
        char strand;
        size_t queryOff, queryLen;
        long long start, end;
    };
    struct Part {
        std::vector<Row> rows;
        size_t malformed = 0;
        bool failed = false;
        std::string err;
    };
    auto parseRange = [&](size_t i, size_t stop, Part &part) {
        std::vector<std::string_view> f;
        while (i < stop) {
            size_t e = i;
            while (e < stop && tab[e] != '\n') ++e;
            const char *ln = tab + i, *le = tab + e;
            i = e < stop ? e + 1 : stop;
            if (ln < le && *ln == '#') continue;
            f.clear();
            for (const char *p = ln; p < le;) {
                while (p < le && isSpaceByte((unsigned char)*p)) ++p;
                const char *q = p;
                while (q < le && !isSpaceByte((unsigned char)*q)) ++q;
                if (q > p) f.emplace_back(p, (size_t)(q - p));
                p = q;
            }
            if (f.size() < 12) continue;
            long long c6, c7, tStart, tEnd;
            auto num = [](std::string_view v, long long &x) { return pyInt(v.data(), v.data() + v.size(), x); };
            if (!num(f[6], c6) || !num(f[7], c7) || !num(f[8], tStart) || !num(f[9], tEnd)) {
                ++part.malformed;
                continue;
            }
            const std::string_view query = f[0], target = f[1];
            std::string_view targetBase;
            char strand;
            long long frameVal = 0;
            if (targetIsContig) {
                targetBase = target;
                strand = tStart <= tEnd ? '+' : '-';
            } else {
                const size_t us = target.rfind('_');  // rsplit('_', 1)
                targetBase = us == std::string_view::npos ? std::string_view() : target.substr(0, us);
                const std::string_view frameStr = us == std::string_view::npos ? target : target.substr(us + 1);
                const size_t eq = frameStr.find('=');  // split('=')[1]
                if (eq == std::string_view::npos) {
                    ++part.malformed;
                    continue;
                }
                size_t eq2 = frameStr.find('=', eq + 1);
                if (eq2 == std::string_view::npos) eq2 = frameStr.size();
                if (!pyInt(frameStr.data() + eq + 1, frameStr.data() + eq2, frameVal)) {
                    ++part.malformed;
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
                part.failed = true;
                part.err = "hit row gives a window whose start " + std::to_string(start) + " is past its end " +
                           std::to_string(end) + " (target " + std::string(target) + ")";
                return;
            }
            part.rows.push_back({ri->second, pi == profIdx.end() ? -1 : pi->second, strand,
                                 (size_t)(query.data() - tab), query.size(), start, end});
        }
    };
    const size_t nParts = len < (1u << 20) ? 1 : std::min<size_t>(16, std::max(1u, std::thread::hardware_concurrency()));
    std::vector<size_t> cut(nParts + 1, len);
    cut[0] = 0;
    for (size_t k = 1; k < nParts; ++k) {
        size_t c = std::max(cut[k - 1], len / nParts * k);
        while (c < len && tab[c - 1] != '\n') ++c;  // a line start
        cut[k] = c;
    }
    std::vector<Part> parts(nParts);
    if (nParts == 1) {
        parseRange(0, len, parts[0]);
    } else {
        std::vector<std::thread> pool;
        try {
            for (size_t k = 0; k < nParts; ++k)
                pool.emplace_back(parseRange, cut[k], cut[k + 1], std::ref(parts[k]));
        } catch (const std::system_error &) {  // no more threads: this one parses the parts left
            for (size_t k = pool.size(); k < nParts; ++k) parseRange(cut[k], cut[k + 1], parts[k]);
        }
        for (auto &t : pool) t.join();
    }
    std::unordered_map<unsigned long long, int> chromOf;  // (record, query id, strand) -> chroms index
    std::vector<FakeChrom> chroms;
    for (Part &part : parts) {
        if (part.failed) {
            if (err) *err = part.err;
            return -1;
        }
        malformed += part.malformed;
        for (const Row &r : part.rows) {
            int qid = r.profile;
            if (qid < 0)
                qid = otherQuery.emplace(std::string_view(tab + r.queryOff, r.queryLen),
                                         (int)(profileNames.size() + otherQuery.size()))
                          .first->second;
            const unsigned long long key =
                ((unsigned long long)r.record << 33) | ((unsigned long long)qid << 1) | (r.strand == '-' ? 1u : 0u);
            auto it = chromOf.find(key);
            if (it == chromOf.end()) {
                FakeChrom fc;
                fc.queryOff = r.queryOff;
                fc.queryLen = r.queryLen;
                fc.record = r.record;
                fc.strand = r.strand;
                it = chromOf.emplace(key, (int)chroms.size()).first;
                chroms.push_back(std::move(fc));
            }
            chroms[it->second].iv.push_back({r.start, r.end});
        }
    }
    // bedtools sort: the fake chromosomes "target|query|strand" in byte order
    std::vector<std::string> fakes(chroms.size());
    std::vector<int> order(chroms.size());
    for (size_t c = 0; c < chroms.size(); ++c) {
        const FakeChrom &fc = chroms[c];
        fakes[c] = recordNames[fc.record] + "|" + std::string(tab + fc.queryOff, fc.queryLen) + "|" + fc.strand;
        order[c] = (int)c;
    }
    std::sort(order.begin(), order.end(), [&](int a, int b) { return fakes[a] < fakes[b]; });
    for (size_t oi = 0; oi < order.size(); ++oi) {
        const int c = order[oi];
        // distinct (target, query) pairs can spell the same name ("a|b" + "c",
        // "a" + "b|c"): bedtools sees one chromosome
        while (oi + 1 < order.size() && fakes[order[oi + 1]] == fakes[c]) {
            auto &more = chroms[order[++oi]].iv;
            chroms[c].iv.insert(chroms[c].iv.end(), more.begin(), more.end());
        }
        // _AWK_UNPACK: split the fake name at '|'; the strand is the last
        // field, the profile the one before, the chromosome the rest
        const std::string &fake = fakes[c];
        const size_t s2 = fake.rfind('|');
        const size_t s1 = fake.rfind('|', s2 - 1);
        const std::string_view chrom(fake.data(), s1);
        const int strand = fake[s2 + 1] == '+' ? 1 : -1;
        const std::string_view profile(fake.data() + s1 + 1, s2 - s1 - 1);
        FakeChrom &fc = chroms[c];
        const size_t profOff = fc.queryOff + (fc.queryLen - profile.size());
        const auto ri = recIdx.find(chrom);
        const auto pi = profIdx.find(profile);
        std::vector<Interval> &iv = fc.iv;
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
