// TEST INFRASTRUCTURE ONLY: the reference engine bound to libdummest_b200.so.
//
// The reference's DP sits behind two functions, findSimilarities
// (dummest-search.hh:9-17) and findSimilaritiesBackwardOnly
// (dummest-dp-backward.hh:300-304).  Their callers are the survivor wave
// (findFinalSimilarities, dummest-search.hh:57-74), the filter wave
// (dummest-search.hh:146-179) and calibration (estimateK,
// dummest-calibration.hh:489-505).  make_dropin_src.py copies the reference
// sources into a build folder and makes each of the two functions begin with
// a call into this file, which answers it through the C ABI
// (include/dummest_b200.h) and returns; everything else -- option parsing,
// the FASTA reader, tantan, the thread pool and its batching, the Gumbel fit,
// the output -- is the reference's own code.  A test runs the stock engine and
// this one on the same input and compares their stdout byte for byte.
//
// Each worker thread has its own library context (a context is not locked);
// profiles are added once per context, keyed by their values array; every
// call adds its batch's decoded sequences and clears them afterwards.
#pragma once

#include <algorithm>
#include <atomic>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <iostream>
#include <unordered_map>
#include <vector>

#include "dummest_b200.h"

namespace dmst_dropin {

struct Ctx {
    dmst_ctx *h = nullptr;
    std::unordered_map<const void *, int> profileIds;
    ~Ctx() {
        if (h) dmst_ctx_destroy(h);
    }
};

[[noreturn]] inline void die(Ctx &c, int st, const char *what) {
    std::cerr << "dummest_b200 drop-in: " << what << ": " << dmst_strerror(st);
    if (c.h) std::cerr << " (" << dmst_last_error(c.h) << ")";
    std::cerr << "\n";
    std::exit(1);
}

// The calling thread's context, created on first use (after option parsing,
// so with the engine's frameshift and stop-codon rates).
inline Ctx &context() {
    thread_local Ctx c;
    if (!c.h) {
        dmst_opts o;
        dmst_opts_default(&o);
        o.insert1 = INSERT1;
        o.insert2 = INSERT2;
        o.delete1 = DELETE1;
        o.delete2 = DELETE2;
        o.stop_codon_prob = STOP_CODON_PROB;
        o.bg_stop_codon_prob = BG_STOP_CODON_PROB;
        const char *dev = std::getenv("DMST_DEVICE");
        o.device = dev ? std::atoi(dev) : 0;
        if (int st = dmst_ctx_create(&o, &c.h)) die(c, st, "dmst_ctx_create");
    }
    return c;
}

inline int profileId(Ctx &c, const Profile &p) {
    auto it = c.profileIds.find(p.values);
    if (it != c.profileIds.end()) return it->second;
    int id = -1;
    if (int st = dmst_profile_add(c.h, p.values, p.width, p.length,
                                  reinterpret_cast<const dmst_params *>(p.values_v2.data()), p.bg_probs.data(), &id))
        die(c, st, "dmst_profile_add");
    c.profileIds.emplace(p.values, id);
    return id;
}

// The batch's lanes as sequences of the context and one pair per lane.
inline std::vector<dmst_pair> addLanes(Ctx &c, const Profile &profile,
                                       const std::array<std::vector<uint8_t> *, simdWidth> &decoded, int activeCount,
                                       const Float *minProbRatio) {
    std::vector<int64_t> off(activeCount + 1, 0);
    for (int k = 0; k < activeCount; ++k) off[k + 1] = off[k] + (int64_t)decoded[k]->size();
    // The widest batch the engine has scored, which it reports at the end
    // (setupBatch keeps it, dummest-dp-backward.hh:203-209; both entry points
    // pass through setupBatch there, and through here in this build).
    size_t width = 0;
    for (int k = 0; k < activeCount; ++k) width = std::max(width, decoded[k]->size());
    size_t cur = g_maxDpWidth.load(std::memory_order_relaxed);
    while (width > cur && !g_maxDpWidth.compare_exchange_weak(cur, width, std::memory_order_relaxed))
        ;
    std::vector<uint8_t> codes((size_t)off[activeCount]);
    for (int k = 0; k < activeCount; ++k)
        std::memcpy(codes.data() + off[k], decoded[k]->data(), decoded[k]->size());
    int first = 0;
    if (int st = dmst_seqs_clear(c.h)) die(c, st, "dmst_seqs_clear");
    if (int st = dmst_seqs_add_decoded(c.h, codes.data(), off.data(), activeCount, &first))
        die(c, st, "dmst_seqs_add_decoded");
    const int pid = profileId(c, profile);
    std::vector<dmst_pair> pairs(activeCount);
    for (int k = 0; k < activeCount; ++k)
        pairs[k] = dmst_pair{first + k, pid, minProbRatio ? (float)minProbRatio[k] : -2.0f};
    return pairs;
}

// findSimilaritiesBackwardOnly: the float filter best of each lane.
inline void backwardOnly(std::array<Float, simdWidth> &bestScores, const Profile &profile,
                         const std::array<std::vector<uint8_t> *, simdWidth> &decoded, int activeCount) {
    Ctx &c = context();
    std::vector<dmst_pair> pairs = addLanes(c, profile, decoded, activeCount, nullptr);
    std::vector<dmst_result> res(activeCount);
    if (int st = dmst_score_pairs(c.h, pairs.data(), pairs.size(), DMST_MODE_FILTER, res.data()))
        die(c, st, "dmst_score_pairs (filter)");
    for (int k = 0; k < activeCount; ++k) bestScores[k] = res[k].filter_f;
}

// findSimilarities: with a non-negative minProbRatio (the survivor wave) a
// lane's alignments, each an AlignedSimilarity with its segment pairs; with
// a negative one (calibration, and searches without an E-value gate) the
// three report entries of dummest-dp-forward.hh:536-544: two placeholders
// and the lane's best column anchor with its mid score.  filterBestOut gets
// the exact filter best.
inline void similarities(std::array<std::vector<AlignedSimilarity>, simdWidth> &sims, const Profile &profile,
                         const std::array<std::vector<uint8_t> *, simdWidth> &decoded,
                         const std::array<Float, simdWidth> &minProbRatio, int activeCount,
                         std::array<ExpScore, simdWidth> *filterBestOut) {
    Ctx &c = context();
    std::vector<dmst_pair> pairs = addLanes(c, profile, decoded, activeCount, minProbRatio.data());
    std::vector<dmst_result> res(activeCount);
    bool anyGate = false, anyReport = false;
    for (int k = 0; k < activeCount; ++k) (minProbRatio[k] >= 0 ? anyGate : anyReport) = true;
    if (anyGate) {
        size_t nAl = 0, nSeg = 0;
        if (int st = dmst_align(c.h, pairs.data(), pairs.size(), res.data(), &nAl, &nSeg)) die(c, st, "dmst_align");
        std::vector<dmst_alignment> al(nAl);
        std::vector<dmst_segment> seg(nSeg);
        if (int st = dmst_align_fetch(c.h, al.data(), nAl, seg.data(), nSeg)) die(c, st, "dmst_align_fetch");
        for (const dmst_alignment &a : al) {
            AlignedSimilarity s{ExpScore{a.score.m, a.score.e}, a.ln_score, a.anchor1, a.anchor2, {}};
            for (int q = 0; q < a.seg_count; ++q) {
                const dmst_segment &g = seg[(size_t)a.seg_begin + q];
                s.alignment.push_back(SegmentPair{g.start1, g.start2, g.length});
            }
            sims[a.pair].push_back(std::move(s));
        }
    }
    if (anyReport) {
        // The per-column anchors: the lane's best column (the first one on
        // ties, as std::max_element picks) and its row.
        size_t cols = 0;
        for (int k = 0; k < activeCount; ++k) cols += decoded[k]->size();
        std::vector<dmst_score> best(cols);
        std::vector<int> row(cols);
        if (int st = dmst_anchors(c.h, pairs.data(), pairs.size(), best.data(), row.data(), res.data()))
            die(c, st, "dmst_anchors");
        size_t o = 0;
        for (int k = 0; k < activeCount; ++k) {
            const int len = (int)decoded[k]->size();
            if (minProbRatio[k] < 0) {
                AlignedSimilarity sel{ExpScore{}, -INFINITY, 0, 0, {}};
                for (int j = 0; j < len; ++j) {
                    const ExpScore e{best[o + j].m, best[o + j].e};
                    if (e.m != 0.0 && scoreLess(sel.pair, e)) sel = AlignedSimilarity{e, -INFINITY, row[o + j], j, {}};
                }
                AlignedSimilarity b = sel;
                b.logProbRatio = -INFINITY;
                sel.logProbRatio = res[k].mid_ln;  // scoreToLog(sel.pair)
                sims[k].push_back(b);
                sims[k].push_back(b);
                sims[k].push_back(sel);
            }
            o += len;
        }
    }
    if (filterBestOut)
        for (int k = 0; k < activeCount; ++k) (*filterBestOut)[k] = ExpScore{res[k].filter.m, res[k].filter.e};
}

}  // namespace dmst_dropin
