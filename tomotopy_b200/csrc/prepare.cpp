// prepare.cpp -- host-side corpus preparation of tomotopy's LDAModel::prepare
// for an integer-id corpus:
//   1. vocabulary reorder by (cf, df) descending with the min_cf / min_df /
//      rm_top rules (TopicModel::removeStopwords, TopicModel.hpp:526-571): a
//      stable sort where words failing a threshold go last, then the first
//      rm_top ids rotated to the end; realV = the ids before the first
//      failing word;
//   2. every document sorted by the new ids, remembering each token's new
//      position (prepareDoc -> sortAndWriteOrder, LDAModel.hpp:716-722,
//      Utils.hpp:227-248).
// A corpus split across processes counts (cf, df) per shard
// (tmt_corpus_counts), sums them, and prepares every shard with the summed
// counts (tmt_prepare_corpus_counted), so that all shards share one
// vocabulary order.
#include <algorithm>
#include <cstdint>
#include <numeric>
#include <thread>
#include <vector>
#include "../../include/tomotopy_b200.h"

extern "C" tmt_status tmt_corpus_counts(uint64_t D, const uint64_t* doc_off, const uint32_t* words,
                                        uint32_t n_vocab, uint64_t* vocab_cf, uint64_t* vocab_df)
{
    if (!doc_off || (doc_off[D] && !words) || (n_vocab && (!vocab_cf || !vocab_df))) return TMT_ERR_INVALID_ARGUMENT;
    try {
        std::fill(vocab_cf, vocab_cf + n_vocab, 0);
        std::fill(vocab_df, vocab_df + n_vocab, 0);
        std::vector<uint64_t> last(n_vocab, UINT64_MAX);
        for (uint64_t d = 0; d < D; ++d) {
            for (uint64_t i = doc_off[d]; i < doc_off[d + 1]; ++i) {
                const uint32_t w = words[i];
                if (w >= n_vocab) return TMT_ERR_INVALID_ARGUMENT;
                ++vocab_cf[w];
                if (last[w] != d) { last[w] = d; ++vocab_df[w]; }
            }
        }
    } catch (...) {
        return TMT_ERR_OUT_OF_MEMORY;
    }
    return TMT_OK;
}

extern "C" tmt_status tmt_prepare_corpus_counted(uint64_t D, const uint64_t* doc_off, const uint32_t* words,
                                                 uint32_t n_vocab, const uint64_t* cf, const uint64_t* df,
                                                 uint64_t min_cf, uint64_t min_df, uint64_t rm_top,
                                                 uint32_t* words_out, uint32_t* w_order, uint32_t* vocab_order,
                                                 uint32_t* real_v)
{
    if (!doc_off || (doc_off[D] && (!words || !words_out)) || !vocab_order || !real_v ||
        (n_vocab && (!cf || !df)))
        return TMT_ERR_INVALID_ARGUMENT;
    try {
        const uint64_t N = doc_off[D];
        for (uint64_t i = 0; i < N; ++i)
            if (words[i] >= n_vocab) return TMT_ERR_INVALID_ARGUMENT;
        auto bad = [&](uint32_t i) { return cf[i] < min_cf || df[i] < min_df; };
        auto gt = [&](uint32_t a, uint32_t b) { return cf[a] > cf[b] || (cf[a] == cf[b] && df[a] > df[b]); };
        std::vector<uint32_t> ids(n_vocab);
        std::iota(ids.begin(), ids.end(), 0u);
        std::stable_sort(ids.begin(), ids.end(), [&](uint32_t a, uint32_t b) {
            bool ba = bad(a), bb = bad(b);
            if (ba) return bb ? gt(a, b) : false;
            if (bb) return true;
            return gt(a, b);
        });
        const uint64_t r = std::min<uint64_t>(rm_top, n_vocab);
        if (r) std::rotate(ids.begin(), ids.begin() + r, ids.end());
        uint32_t rv = (uint32_t)(n_vocab - r);
        for (uint32_t i = 0; i < n_vocab - r; ++i)
            if (bad(ids[i])) { rv = i; break; }
        *real_v = rv;
        for (uint32_t i = 0; i < n_vocab; ++i) vocab_order[ids[i]] = i;
        if (!N) return TMT_OK;
        unsigned nt = std::max(1u, std::min(std::thread::hardware_concurrency(), 64u));
        if (D < 1024) nt = 1;
        std::vector<std::thread> th;
        for (unsigned t = 0; t < nt; ++t) {
            th.emplace_back([&, t] {
                std::vector<std::pair<uint32_t, uint32_t>> pv;
                for (uint64_t d = D * t / nt; d < D * (t + 1) / nt; ++d) {
                    const uint64_t b = doc_off[d], n = doc_off[d + 1] - b;
                    pv.resize(n);
                    for (uint64_t j = 0; j < n; ++j) pv[j] = { vocab_order[words[b + j]], (uint32_t)j };
                    std::stable_sort(pv.begin(), pv.end(),
                                     [](const auto& x, const auto& y) { return x.first < y.first; });
                    for (uint64_t j = 0; j < n; ++j) {
                        words_out[b + j] = pv[j].first;
                        if (w_order) w_order[b + pv[j].second] = (uint32_t)j;
                    }
                }
            });
        }
        for (auto& x : th) x.join();
    } catch (...) {
        return TMT_ERR_OUT_OF_MEMORY;
    }
    return TMT_OK;
}

extern "C" tmt_status tmt_prepare_corpus(uint64_t D, const uint64_t* doc_off, const uint32_t* words,
                                         uint32_t n_vocab, uint64_t min_cf, uint64_t min_df, uint64_t rm_top,
                                         uint32_t* words_out, uint32_t* w_order, uint32_t* vocab_order,
                                         uint64_t* vocab_cf, uint64_t* vocab_df, uint32_t* real_v)
{
    if (!doc_off || (doc_off[D] && (!words || !words_out)) || !vocab_order || !real_v)
        return TMT_ERR_INVALID_ARGUMENT;
    try {
        std::vector<uint64_t> cf(n_vocab), df(n_vocab);
        tmt_status st = tmt_corpus_counts(D, doc_off, words, n_vocab, cf.data(), df.data());
        if (st != TMT_OK) return st;
        st = tmt_prepare_corpus_counted(D, doc_off, words, n_vocab, cf.data(), df.data(), min_cf, min_df, rm_top,
                                        words_out, w_order, vocab_order, real_v);
        if (st != TMT_OK) return st;
        for (uint32_t w = 0; w < n_vocab; ++w) {
            if (vocab_cf) vocab_cf[vocab_order[w]] = cf[w];
            if (vocab_df) vocab_df[vocab_order[w]] = df[w];
        }
    } catch (...) {
        return TMT_ERR_OUT_OF_MEMORY;
    }
    return TMT_OK;
}
