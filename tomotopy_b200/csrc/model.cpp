// model.cpp -- the host side of tomotopy's LDAModel over the device engine:
// dictionary, documents, preparation, training, queries, inference of
// string documents and tomotopy's binary model layout (tmt_model_* in
// include/tomotopy_b200.h).
//
// What it restates (paths in the tomotopy tree):
//   add_doc            TopicModel::_addDoc / _makeFromRawDoc   TopicModel.hpp:397-449
//   prepare            LDAModel::prepare                        LDAModel.hpp:1073-1138
//                      TopicModel::removeStopwords              TopicModel.hpp:526-571
//                      LDAModel::prepareDoc                     LDAModel.hpp:716-722
//   topic-word dist    LDAModel::_getWidsByTopic                LDAModel.hpp:828-841
//   doc topic dist     LDAModel::_getTopicsByDoc                LDAModel.hpp:1145-1159
//   count by topics    LDAModel::_getTopicsCount                LDAModel.hpp:815-826
//   save / load        TopicModel::_saveModel / _loadModel      TopicModel.hpp:335-395
//                      serializer (keys, tagged blocks)         Utils/serializer.hpp:147-209, 787-853
//                      LDAModel tagged fields                   LDAModel.hpp:958-960
//                      DocumentBase / DocumentLDA fields        TopicModel.hpp:127-131, LDAModel.cpp:5-6
// The sampling, merging, log-likelihood and inference run on the device
// through the engine's C ABI.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <numeric>
#include <stdexcept>
#include <string>
#include <unordered_map>
#include <unordered_set>
#include <vector>
#include <memory>
#include <type_traits>
#include <utility>
#include "../../include/tomotopy_b200.h"

namespace {

struct ArgErr : std::runtime_error { using std::runtime_error::runtime_error; };
struct FormatErr : std::runtime_error { using std::runtime_error::runtime_error; };
struct EngineErr : std::runtime_error {
    tmt_status st;
    EngineErr(tmt_status s, const std::string& m) : std::runtime_error(m), st(s) {}
};

// ---------------------------------------------------------------------------
// tomotopy's binary layout
// ---------------------------------------------------------------------------
constexpr uint32_t kTaggedKey = 0x4b545054;   // "TPTK"
constexpr uint32_t kTaggedVersion = 0x00010001;

struct Writer {
    std::string b;
    void raw(const void* p, size_t n) { b.append(static_cast<const char*>(p), n); }
    template <class T> void pod(T v) { raw(&v, sizeof(T)); }
    // a key written as raw bytes (tomotopy's Key: no length prefix)
    void key(const char* s, size_t n) { raw(s, n); }
    template <class T> void vec(const std::vector<T>& v)
    {
        pod<uint32_t>((uint32_t)v.size());
        if (!v.empty()) raw(v.data(), v.size() * sizeof(T));
    }
    void str(const std::string& s)
    {
        pod<uint32_t>((uint32_t)s.size());
        raw(s.data(), s.size());
    }
    // one tagged block: header {key, version, totsize, keysize, trailing} +
    // key (NUL-terminated name) + data; totsize counts the last 16 header
    // bytes, the key and the data
    void tagged(const char* name, const Writer& data, uint32_t trailing)
    {
        const uint32_t keysize = (uint32_t)std::strlen(name) + 1;
        pod<uint32_t>(kTaggedKey);
        pod<uint32_t>(kTaggedVersion);
        pod<uint64_t>((uint64_t)keysize + data.b.size() + 16);
        pod<uint32_t>(keysize);
        pod<uint32_t>(trailing);
        raw(name, keysize);
        raw(data.b.data(), data.b.size());
    }
};

struct Reader {
    const uint8_t* p;
    size_t n, i = 0;
    Reader(const uint8_t* p_, size_t n_) : p(p_), n(n_) {}
    void need(size_t k) const
    {
        if (i + k > n) throw FormatErr("unexpected end of model data");
    }
    void raw(void* out, size_t k)
    {
        need(k);
        std::memcpy(out, p + i, k);
        i += k;
    }
    template <class T> T pod()
    {
        T v;
        raw(&v, sizeof(T));
        return v;
    }
    bool expect(const char* s, size_t k)
    {
        need(k);
        if (std::memcmp(p + i, s, k)) return false;
        i += k;
        return true;
    }
    template <class T> std::vector<T> vec()
    {
        const uint32_t m = pod<uint32_t>();
        std::vector<T> v(m);
        if (m) raw(v.data(), m * sizeof(T));
        return v;
    }
    std::string str()
    {
        const uint32_t m = pod<uint32_t>();
        std::string s(m, '\0');
        if (m) raw(&s[0], m);
        return s;
    }
    bool peek_tagged() const { return i + 4 <= n && std::memcmp(p + i, &kTaggedKey, 4) == 0; }
    // a chain of tagged blocks: name -> [begin, end) of the data; the reader
    // ends after the last block (trailing count 0)
    std::unordered_map<std::string, std::pair<size_t, size_t>> tagged_chain()
    {
        std::unordered_map<std::string, std::pair<size_t, size_t>> m;
        for (;;) {
            const size_t at = i;
            if (pod<uint32_t>() != kTaggedKey) throw FormatErr("tagged data key is not found");
            pod<uint32_t>();   // version
            const uint64_t tot = pod<uint64_t>();
            const uint32_t keysize = pod<uint32_t>();
            const uint32_t trailing = pod<uint32_t>();
            need(keysize);
            std::string name(reinterpret_cast<const char*>(p + i), keysize);
            while (!name.empty() && name.back() == '\0') name.pop_back();
            i += keysize;
            const size_t end = at + 8 + tot;
            if (end > n || end < i) throw FormatErr("tagged block overruns the data");
            m[name] = { i, end };
            i = end;
            if (!trailing) break;
        }
        return m;
    }
};

// ---------------------------------------------------------------------------
// the model
// ---------------------------------------------------------------------------
struct Doc {
    std::vector<uint32_t> words;     // dictionary ids; after prepare: sorted by id
    std::vector<uint32_t> wOrder;    // wOrder[original position] = sorted position (after prepare)
    std::vector<uint16_t> Zs;        // sorted order
    std::vector<float> wordWeights;  // TermWeight IDF / PMI: per token, sorted order (empty for ONE)
    float weight = 1.f;
    std::string rawStr, docUid;
    std::vector<uint32_t> origWordPos;
    std::vector<uint16_t> origWordLen;
};

} // namespace

// An allocator whose value-less construct leaves trivial elements
// uninitialised: resize() then reserves the pages without writing them, and
// the engine's threaded download is the first to touch them (a zero fill of
// a 4 GB n_dk on one thread first took seconds).
template <class T>
struct NoInit : std::allocator<T> {
    template <class U>
    struct rebind {
        using other = NoInit<U>;
    };
    NoInit() = default;
    template <class U>
    NoInit(const NoInit<U>&) noexcept {}
    template <class U>
    void construct(U* p) noexcept(std::is_nothrow_default_constructible<U>::value)
    {
        ::new (static_cast<void*>(p)) U;
    }
    template <class U, class... A>
    void construct(U* p, A&&... a)
    {
        ::new (static_cast<void*>(p)) U(std::forward<A>(a)...);
    }
};
template <class T>
using HostBuf = std::vector<T, NoInit<T>>;

struct tmt_model {
    // hyper-parameters (LDAArgs, LDAModel.hpp:962-983)
    uint32_t K = 1;
    float alpha = 0.1f, eta = 0.01f;
    std::vector<float> alphas;
    uint64_t seed = 0;
    uint64_t min_cf = 0, min_df = 0, rm_top = 0;
    uint32_t optim_interval = 10, burn_in = 0;
    int32_t device = 0;
    uint32_t sweep_groups = 0;
    int32_t tw = 0;                  // TermWeight: 0 ONE, 1 IDF, 2 PMI
    double weightedN = 0;            // the ll_per_word denominator (TopicModel::weightedN)
    // vocabulary
    std::unordered_map<std::string, uint32_t> dict;
    std::vector<std::string> id2word;
    std::vector<uint64_t> vocabCf, vocabDf;
    std::vector<Doc> docs;
    uint64_t realV = 0, realN = 0, globalStep = 0;
    bool prepared = false;
    std::vector<float> vocabWeights;
    // set_word_prior (LDAModel.hpp:1031-1045): word -> K priors, in insertion
    // (or file) order; the first call for a word wins (etaByWord.emplace)
    std::vector<std::pair<std::string, std::vector<float>>> etaByWord;
    // device state
    tmt_handle* eng = nullptr;
    // host copies, refreshed on demand
    bool host_fresh = false;
    HostBuf<int32_t> nkw, nk, ndk;
    HostBuf<float> nkw_f, nk_f, ndk_f;   // the same for weighted counts
    std::string err;

    ~tmt_model()
    {
        if (eng) tmt_destroy(eng);
    }

    uint32_t add_word(const std::string& w)
    {
        auto it = dict.find(w);
        if (it != dict.end()) return it->second;
        const uint32_t id = (uint32_t)id2word.size();
        dict.emplace(w, id);
        id2word.push_back(w);
        return id;
    }

    void check(tmt_status st)
    {
        if (st != TMT_OK) throw EngineErr(st, eng ? tmt_last_error(eng) : "engine call failed");
    }

    void refresh()
    {
        if (host_fresh || !eng) return;
        // every element is written by the downloads: sized, not filled
        HostBuf<uint16_t> z(realN_all());
        if (tw) {
            nkw_f.resize((uint64_t)K * realV);
            nk_f.resize(K);
            ndk_f.resize((uint64_t)docs.size() * K);
            check(tmt_download_state(eng, z.data(), nullptr, nullptr, alphas.data()));
            check(tmt_download_counts_f32(eng, docs.empty() ? nullptr : ndk_f.data(), nkw_f.data(), nk_f.data(),
                                          nullptr));
        } else {
            nkw.resize((uint64_t)K * realV);
            nk.resize(K);
            check(tmt_download_state(eng, z.data(), nkw.data(), nk.data(), alphas.data()));
            ndk.resize((uint64_t)docs.size() * K);
            if (!docs.empty()) check(tmt_download_doc_topic(eng, ndk.data()));
        }
        uint64_t at = 0;
        for (auto& d : docs) {
            std::copy(z.begin() + at, z.begin() + at + d.words.size(), d.Zs.begin());
            at += d.words.size();
        }
        host_fresh = true;
    }

    static const char* tw_key(int32_t t) { return t == 1 ? "idf\0\0" : t == 2 ? "pmi\0\0" : "one\0\0"; }

    // TermWeight IDF / PMI weights (LDAModel.hpp:1093-1122 vocabWeights,
    // :795-809 per token), in each document's sorted order
    void compute_weights()
    {
        const size_t V = id2word.size();
        vocabWeights.assign(V, 0.f);
        if (tw == 1) {
            std::vector<uint64_t> df(V, 0);
            for (auto& d : docs) {
                std::unordered_set<uint32_t> u(d.words.begin(), d.words.end());
                for (auto w : u)
                    if (w < realV) ++df[w];
            }
            for (size_t i = 0; i < V; ++i) vocabWeights[i] = (float)std::log(docs.size() / (double)df[i]);
        } else {
            uint64_t tot = 0;
            for (auto c : vocabCf) tot += c;
            for (size_t i = 0; i < V; ++i) vocabWeights[i] = (float)(vocabCf[i] / (double)tot);
        }
        std::vector<uint32_t> tf(realV, 0);
        for (auto& d : docs) doc_weights(d.words, d.wordWeights, tf);
    }

    // one document's token weights; tf: realV zeros on entry and exit
    void doc_weights(const std::vector<uint32_t>& words, std::vector<float>& out, std::vector<uint32_t>& tf) const
    {
        out.assign(words.size(), 0.f);
        if (tw == 2)
            for (auto w : words)
                if (w < realV) ++tf[w];
        for (size_t i = 0; i < words.size(); ++i) {
            const uint32_t w = words[i];
            if (w >= realV) continue;
            if (tw == 1) {
                out[i] = vocabWeights[w];
            } else {
                const float q = (float)tf[w] / vocabWeights[w] / (float)words.size();
                out[i] = std::max((float)std::log((double)q), 0.f);
            }
        }
        if (tw == 2)
            for (auto w : words)
                if (w < realV) tf[w] = 0;
    }

    uint64_t realN_all() const
    {
        uint64_t n = 0;
        for (auto& d : docs) n += d.words.size();
        return n;
    }

    // removeStopwords (TopicModel.hpp:526-571): ids re-numbered by (cf, df)
    // descending, words below min_cf / min_df last, the rm_top most frequent
    // rotated to the end; realV = the ids before the first removed word.
    void remove_stopwords()
    {
        const uint32_t nv = (uint32_t)id2word.size();
        vocabCf.resize(nv);
        vocabDf.resize(nv);
        auto bad = [&](uint32_t i) { return vocabCf[i] < min_cf || vocabDf[i] < min_df; };
        auto gt = [&](uint32_t a, uint32_t b) {
            return vocabCf[a] > vocabCf[b] || (vocabCf[a] == vocabCf[b] && vocabDf[a] > vocabDf[b]);
        };
        std::vector<uint32_t> ids(nv);
        std::iota(ids.begin(), ids.end(), 0u);
        std::stable_sort(ids.begin(), ids.end(), [&](uint32_t a, uint32_t b) {
            const bool ba = bad(a), bb = bad(b);
            if (ba) return bb ? gt(a, b) : false;
            if (bb) return true;
            return gt(a, b);
        });
        const uint64_t r = std::min<uint64_t>(rm_top, nv);
        if (r) std::rotate(ids.begin(), ids.begin() + r, ids.end());
        realV = nv - r;
        for (uint32_t i = 0; i < nv - r; ++i)
            if (bad(ids[i])) { realV = i; break; }
        std::vector<uint32_t> order(nv);
        std::vector<uint64_t> cf(nv), df(nv);
        std::vector<std::string> words(nv);
        for (uint32_t i = 0; i < nv; ++i) {
            order[ids[i]] = i;
            cf[i] = vocabCf[ids[i]];
            df[i] = vocabDf[ids[i]];
            words[i] = id2word[ids[i]];
        }
        vocabCf.swap(cf);
        vocabDf.swap(df);
        id2word.swap(words);
        dict.clear();
        for (uint32_t i = 0; i < nv; ++i) dict.emplace(id2word[i], i);
        for (auto& d : docs)
            for (auto& w : d.words) w = order[w];
    }

    // prepareDoc: stable sort of the doc's words, wOrder[old] = new
    static void sort_doc(Doc& d)
    {
        const size_t n = d.words.size();
        std::vector<std::pair<uint32_t, uint32_t>> pv(n);
        for (size_t i = 0; i < n; ++i) pv[i] = { d.words[i], (uint32_t)i };
        std::stable_sort(pv.begin(), pv.end(), [](const auto& a, const auto& b) { return a.first < b.first; });
        d.wOrder.assign(n, 0);
        for (size_t i = 0; i < n; ++i) {
            d.words[i] = pv[i].first;
            d.wOrder[pv[i].second] = (uint32_t)i;
        }
    }

    // prepareWordPriors (LDAModel.hpp:724-737): the prior words still in the
    // vocabulary (id < realV) get their columns
    void prior_table(std::vector<uint32_t>& ids, std::vector<float>& vals) const
    {
        ids.clear();
        vals.clear();
        for (auto& e : etaByWord) {
            auto it = dict.find(e.first);
            if (it == dict.end() || it->second >= realV) continue;
            ids.push_back(it->second);
            vals.insert(vals.end(), e.second.begin(), e.second.end());
        }
    }

    void apply_word_priors()
    {
        std::vector<uint32_t> ids;
        std::vector<float> vals;
        prior_table(ids, vals);
        check(tmt_set_word_priors(eng, (uint32_t)ids.size(), ids.data(), vals.data()));
    }

    const std::vector<float>* prior_of(const std::string& w) const
    {
        for (auto& e : etaByWord)
            if (e.first == w) return &e.second;
        return nullptr;
    }

    void make_engine()
    {
        if (eng) { tmt_destroy(eng); eng = nullptr; }
        tmt_config c{};
        c.K = K;
        c.V = (uint32_t)realV;
        c.alpha = alphas.data();
        c.eta = eta;
        c.seed = seed;
        c.optim_interval = optim_interval;
        c.burn_in = burn_in;
        c.device = device;
        c.sweep_groups = sweep_groups;
        tmt_handle* h = nullptr;
        tmt_status st = tmt_create(&c, &h);
        if (st != TMT_OK) {
            std::string m = h ? tmt_last_error(h) : "tmt_create failed";
            if (h) tmt_destroy(h);
            throw EngineErr(st, m);
        }
        eng = h;
    }

    // upload the documents; z0 from the documents' Zs when `with_z`, else drawn on the device
    void upload(bool with_z)
    {
        std::vector<uint64_t> off(docs.size() + 1, 0);
        for (size_t d = 0; d < docs.size(); ++d) off[d + 1] = off[d] + docs[d].words.size();
        std::vector<uint32_t> w(off.back());
        std::vector<uint16_t> z(with_z ? off.back() : 0);
        for (size_t d = 0; d < docs.size(); ++d) {
            std::copy(docs[d].words.begin(), docs[d].words.end(), w.begin() + off[d]);
            if (with_z) std::copy(docs[d].Zs.begin(), docs[d].Zs.end(), z.begin() + off[d]);
        }
        if (tw) {
            std::vector<float> wt(off.back());
            for (size_t d = 0; d < docs.size(); ++d)
                std::copy(docs[d].wordWeights.begin(), docs[d].wordWeights.end(), wt.begin() + off[d]);
            const float none = 0.f;    // a corpus without tokens still passes a weights array
            check(tmt_upload_corpus_weighted(eng, w.data(), off.data(), docs.size(), with_z ? z.data() : nullptr,
                                             wt.empty() ? &none : wt.data()));
        } else {
            check(tmt_upload_corpus(eng, w.data(), off.data(), docs.size(), with_z ? z.data() : nullptr));
        }
        realN = 0;
        for (auto x : w) realN += x < realV;
        host_fresh = false;
    }

    // countRealN's weighted sum (TopicModel.hpp:507-523): the tokens' weights in
    // document and token order, 1 per token without weights
    double weighted_sum() const
    {
        double s = 0;
        for (auto& d : docs)
            for (size_t i = 0; i < d.words.size(); ++i)
                if (d.words[i] < realV) s += d.wordWeights.empty() ? 1.0 : (double)d.wordWeights[i];
        return s;
    }

    void prepare()
    {
        if (prepared) return;
        remove_stopwords();
        for (auto& d : docs) {
            sort_doc(d);
            d.Zs.assign(d.words.size(), 0xFFFF);
        }
        // tomotopy counts weightedN before the weights exist (prepare calls
        // countRealN first, TopicModel.hpp:652-655): a fresh model's
        // ll_per_word divides by the token count
        weightedN = 0;
        for (auto& d : docs)
            for (auto w : d.words) weightedN += w < realV;
        if (tw) compute_weights();
        make_engine();
        apply_word_priors();
        upload(false);
        prepared = true;
    }

    // ---- serialization ----------------------------------------------------
    void save(Writer& w, bool full, const uint8_t* extra, size_t extra_len)
    {
        refresh();
        w.key("LDA\0\0", 5);
        w.key(tw_key(tw), 5);
        {   // TopicModel header fields
            Writer dic;
            dic.key("Dict", 4);
            dic.pod<uint32_t>((uint32_t)id2word.size());
            for (auto& s : id2word) dic.str(s);
            Writer cf, df, rv, gs, ex;
            cf.vec(vocabCf);
            df.vec(vocabDf);
            rv.pod<uint64_t>(realV);
            gs.pod<uint64_t>(globalStep_now());
            ex.vec(std::vector<uint8_t>(extra, extra + extra_len));
            w.tagged("dict", dic, 5);
            w.tagged("vocabCf", cf, 4);
            w.tagged("vocabDf", df, 3);
            w.tagged("realV", rv, 2);
            w.tagged("globalStep", gs, 1);
            w.tagged("extra", ex, 0);
        }
        {   // LDAModel fields, version 1 (tagged)
            Writer vw, a, as, e, k, ebw, bi, oi;
            vw.vec(vocabWeights);
            a.pod<float>(alpha);
            as.pod<uint32_t>(K);
            as.pod<uint32_t>(1);
            as.raw(alphas.data(), K * sizeof(float));
            e.pod<float>(eta);
            k.pod<uint16_t>((uint16_t)K);
            ebw.pod<uint32_t>((uint32_t)etaByWord.size());
            for (auto& e : etaByWord) {
                ebw.str(e.first);
                ebw.vec(e.second);
            }
            bi.pod<uint32_t>(burn_in);
            oi.pod<uint32_t>(optim_interval);
            w.tagged("vocabWeights", vw, 7);
            w.tagged("alpha", a, 6);
            w.tagged("alphas", as, 5);
            w.tagged("eta", e, 4);
            w.tagged("K", k, 3);
            w.tagged("etaByWord", ebw, 2);
            w.tagged("burnIn", bi, 1);
            w.tagged("optimInterval", oi, 0);
        }
        // globalState: numByTopic (K x 1), numByTopicWord (K x V column-major);
        // int32 for TermWeight ONE, float for IDF / PMI (ModelStateLDA<_tw>)
        w.pod<uint32_t>(K);
        w.pod<uint32_t>(1);
        if (tw) w.raw(nk_f.data(), K * sizeof(float));
        else w.raw(nk.data(), K * sizeof(int32_t));
        w.pod<uint32_t>(K);
        w.pod<uint32_t>((uint32_t)realV);
        if (tw) w.raw(nkw_f.data(), (uint64_t)K * realV * sizeof(float));
        else w.raw(nkw.data(), (uint64_t)K * realV * sizeof(int32_t));
        if (!full) {
            w.pod<uint32_t>(0);
            return;
        }
        w.pod<uint32_t>((uint32_t)docs.size());
        for (auto& d : docs) {
            Writer wt, ws, wo, rs, op, ol, du, zs, ww;
            wt.pod<float>(d.weight);
            ws.vec(d.words);
            wo.vec(d.wOrder);
            rs.str(d.rawStr);
            op.vec(d.origWordPos);
            ol.vec(d.origWordLen);
            du.str(d.docUid);
            zs.vec(d.Zs);
            ww.vec(d.wordWeights);
            w.tagged("weight", wt, 6);
            w.tagged("words", ws, 5);
            w.tagged("wOrder", wo, 4);
            w.tagged("rawStr", rs, 3);
            w.tagged("origWordPos", op, 2);
            w.tagged("origWordLen", ol, 1);
            w.tagged("docUid", du, 0);
            w.tagged("Zs", zs, 1);
            w.tagged("wordWeights", ww, 0);
        }
    }

    uint64_t globalStep_now() const
    {
        if (!eng) return globalStep;
        tmt_info inf{};
        tmt_get_info(eng, &inf);
        return inf.global_step;
    }

    void load(Reader& r, std::vector<uint8_t>& extra)
    {
        if (!r.expect("LDA\0\0", 5)) throw FormatErr("not an LDA model");
        tw = -1;
        for (int32_t t = 0; t < 3 && tw < 0; ++t)
            if (r.expect(tw_key(t), 5)) tw = t;
        if (tw < 0) throw FormatErr("unknown term weighting");
        auto hdr = r.tagged_chain();
        auto sub = [&](const std::string& k) -> Reader {
            auto it = hdr.find(k);
            if (it == hdr.end()) throw FormatErr("missing field " + k);
            Reader q(r.p, it->second.second);
            q.i = it->second.first;
            return q;
        };
        {
            Reader q = sub("dict");
            if (!q.expect("Dict", 4)) throw FormatErr("bad dictionary");
            const uint32_t m = q.pod<uint32_t>();
            id2word.clear();
            dict.clear();
            for (uint32_t i = 0; i < m; ++i) {
                id2word.push_back(q.str());
                dict.emplace(id2word.back(), i);
            }
        }
        { Reader q = sub("vocabCf"); vocabCf = q.vec<uint64_t>(); }
        { Reader q = sub("vocabDf"); vocabDf = q.vec<uint64_t>(); }
        { Reader q = sub("realV"); realV = q.pod<uint64_t>(); }
        { Reader q = sub("globalStep"); globalStep = q.pod<uint64_t>(); }
        if (hdr.count("extra")) { Reader q = sub("extra"); extra = q.vec<uint8_t>(); }
        // LDAModel fields: version 1 (tagged) or version 0
        if (r.peek_tagged()) {
            auto f = r.tagged_chain();
            auto g = [&](const std::string& k) -> Reader {
                auto it = f.find(k);
                if (it == f.end()) throw FormatErr("missing field " + k);
                Reader q(r.p, it->second.second);
                q.i = it->second.first;
                return q;
            };
            { Reader q = g("vocabWeights"); vocabWeights = q.vec<float>(); }
            { Reader q = g("alpha"); alpha = q.pod<float>(); }
            {
                Reader q = g("alphas");
                const uint32_t rows = q.pod<uint32_t>(), cols = q.pod<uint32_t>();
                if (cols != 1) throw FormatErr("alphas is not a vector");
                alphas.resize(rows);
                q.raw(alphas.data(), rows * sizeof(float));
            }
            { Reader q = g("eta"); eta = q.pod<float>(); }
            { Reader q = g("K"); K = q.pod<uint16_t>(); }
            if (f.count("etaByWord")) {
                Reader q = g("etaByWord");
                const uint32_t n = q.pod<uint32_t>();
                etaByWord.clear();
                for (uint32_t i = 0; i < n; ++i) {
                    std::string w = q.str();
                    std::vector<float> pr = q.vec<float>();
                    etaByWord.emplace_back(std::move(w), std::move(pr));
                }
            }
            if (f.count("burnIn")) { Reader q = g("burnIn"); burn_in = q.pod<uint32_t>(); }
            if (f.count("optimInterval")) { Reader q = g("optimInterval"); optim_interval = q.pod<uint32_t>(); }
        } else {
            vocabWeights = r.vec<float>();
            alpha = r.pod<float>();
            const uint32_t rows = r.pod<uint32_t>(), cols = r.pod<uint32_t>();
            if (cols != 1) throw FormatErr("alphas is not a vector");
            alphas.resize(rows);
            r.raw(alphas.data(), rows * sizeof(float));
            eta = r.pod<float>();
            K = r.pod<uint16_t>();
        }
        if (alphas.size() != K) throw FormatErr("alphas does not have K values");
        // globalState
        {
            const uint32_t rows = r.pod<uint32_t>(), cols = r.pod<uint32_t>();
            if (rows != K || cols != 1) throw FormatErr("numByTopic shape");
            if (tw) {
                nk_f.resize(K);
                r.raw(nk_f.data(), K * sizeof(float));
            } else {
                nk.resize(K);
                r.raw(nk.data(), K * sizeof(int32_t));
            }
            const uint32_t r2 = r.pod<uint32_t>(), c2 = r.pod<uint32_t>();
            if (r2 != K || c2 != realV) throw FormatErr("numByTopicWord shape");
            if (tw) {
                nkw_f.resize((uint64_t)K * realV);
                r.raw(nkw_f.data(), nkw_f.size() * sizeof(float));
            } else {
                nkw.resize((uint64_t)K * realV);
                r.raw(nkw.data(), nkw.size() * sizeof(int32_t));
            }
        }
        // documents
        const uint32_t nd = r.pod<uint32_t>();
        docs.assign(nd, Doc{});
        for (auto& d : docs) {
            if (r.peek_tagged()) {
                auto f = r.tagged_chain();
                auto g = [&](const char* k, auto fn) {
                    auto it = f.find(k);
                    if (it == f.end()) return;
                    Reader q(r.p, it->second.second);
                    q.i = it->second.first;
                    fn(q);
                };
                g("weight", [&](Reader& q) { d.weight = q.pod<float>(); });
                g("words", [&](Reader& q) { d.words = q.vec<uint32_t>(); });
                g("wOrder", [&](Reader& q) { d.wOrder = q.vec<uint32_t>(); });
                g("rawStr", [&](Reader& q) { d.rawStr = q.str(); });
                g("origWordPos", [&](Reader& q) { d.origWordPos = q.vec<uint32_t>(); });
                g("origWordLen", [&](Reader& q) { d.origWordLen = q.vec<uint16_t>(); });
                g("docUid", [&](Reader& q) { d.docUid = q.str(); });
                auto f2 = r.tagged_chain();
                auto it = f2.find("Zs");
                if (it == f2.end()) throw FormatErr("document without Zs");
                Reader q(r.p, it->second.second);
                q.i = it->second.first;
                d.Zs = q.vec<uint16_t>();
                auto iw = f2.find("wordWeights");
                if (iw != f2.end()) {
                    Reader q2(r.p, iw->second.second);
                    q2.i = iw->second.first;
                    d.wordWeights = q2.vec<float>();
                }
            } else {
                if (!r.expect("Docu", 4)) throw FormatErr("bad document");
                d.weight = r.pod<float>();
                d.words = r.vec<uint32_t>();
                d.wOrder = r.vec<uint32_t>();
                d.Zs = r.vec<uint16_t>();
                d.wordWeights = r.vec<float>();
            }
            if (d.Zs.size() != d.words.size()) throw FormatErr("Zs and words differ in length");
            if (tw && d.wordWeights.size() != d.words.size()) throw FormatErr("wordWeights and words differ in length");
            if (!tw) d.wordWeights.clear();
            for (size_t i = 0; i < d.words.size(); ++i)
                if (d.words[i] < realV && d.Zs[i] >= K) throw FormatErr("topic id out of range");
        }
        prepared = true;
        realN = 0;
        for (auto& d : docs)
            for (auto w : d.words) realN += w < realV;
        // countRealN after a load sees the stored weights (TopicModel.hpp:392-394)
        weightedN = weighted_sum();
        if (device < 0) {
            // parse only: the host arrays are the state; n_dk recounted from Zs
            if (tw) {
                ndk_f.assign(docs.size() * (uint64_t)K, 0.f);
                for (size_t di = 0; di < docs.size(); ++di)
                    for (size_t i = 0; i < docs[di].words.size(); ++i)
                        if (docs[di].words[i] < realV)
                            ndk_f[di * K + docs[di].Zs[i]] += docs[di].wordWeights[i];
            } else {
                ndk.assign(docs.size() * (uint64_t)K, 0);
                for (size_t di = 0; di < docs.size(); ++di)
                    for (size_t i = 0; i < docs[di].words.size(); ++i)
                        if (docs[di].words[i] < realV) ++ndk[di * K + docs[di].Zs[i]];
            }
            host_fresh = true;
            return;
        }
        for (auto& e : etaByWord)
            if (e.second.size() != K) throw FormatErr("a word prior does not have K values");
        make_engine();
        apply_word_priors();
        upload(true);
        if (tw) check(tmt_set_counts_f32(eng, nkw_f.data(), nk_f.data()));
        else check(tmt_set_counts(eng, nkw.data(), nk.data()));
        check(tmt_set_alpha(eng, alphas.data()));
        check(tmt_set_global_step(eng, globalStep));
        host_fresh = false;
    }
};

namespace {

template <class F>
tmt_status guard(tmt_model* m, F&& f)
{
    try {
        if (m) m->err.clear();
        f();
        return TMT_OK;
    } catch (const ArgErr& e) {
        if (m) m->err = e.what();
        return TMT_ERR_INVALID_ARGUMENT;
    } catch (const FormatErr& e) {
        if (m) m->err = e.what();
        return TMT_ERR_INVALID_ARGUMENT;
    } catch (const EngineErr& e) {
        if (m) m->err = e.what();
        return e.st;
    } catch (const std::bad_alloc&) {
        if (m) m->err = "host allocation failed";
        return TMT_ERR_OUT_OF_MEMORY;
    } catch (const std::exception& e) {
        if (m) m->err = e.what();
        return TMT_ERR_INTERNAL;
    }
}

// NUL-separated words -> vector
std::vector<std::string> split_words(const char* buf, uint32_t n)
{
    std::vector<std::string> out;
    out.reserve(n);
    const char* p = buf;
    for (uint32_t i = 0; i < n; ++i) {
        const size_t l = std::strlen(p);
        out.emplace_back(p, l);
        p += l + 1;
    }
    return out;
}

} // namespace

extern "C" {

tmt_status tmt_model_create(const tmt_model_args* a, tmt_model** out)
{
    if (!a || !out) return TMT_ERR_INVALID_ARGUMENT;
    *out = nullptr;
    auto* m = new (std::nothrow) tmt_model();
    if (!m) return TMT_ERR_OUT_OF_MEMORY;
    tmt_status st = guard(m, [&] {
        if (a->K == 0 || a->K > 32767) throw ArgErr("wrong K value (K = " + std::to_string(a->K) + ")");
        if (!(a->eta > 0)) throw ArgErr("wrong eta value (eta = " + std::to_string(a->eta) + ")");
        m->K = a->K;
        m->eta = a->eta;
        if (a->alpha && a->n_alpha == a->K) {
            m->alphas.assign(a->alpha, a->alpha + a->K);
            m->alpha = a->alpha[0];
        } else if (a->alpha && a->n_alpha == 1) {
            m->alphas.assign(a->K, a->alpha[0]);
            m->alpha = a->alpha[0];
        } else {
            throw ArgErr("wrong alpha value (len = " + std::to_string(a->n_alpha) + ")");
        }
        for (float x : m->alphas)
            if (!(x > 0)) throw ArgErr("wrong alpha value");
        m->seed = a->seed;
        m->min_cf = a->min_cf;
        m->min_df = a->min_df;
        m->rm_top = a->rm_top;
        m->device = a->device;
        m->sweep_groups = a->sweep_groups;
        if (a->tw < 0 || a->tw > 2) throw ArgErr("unknown term weight");
        m->tw = a->tw;
    });
    *out = m;
    return st;
}

tmt_status tmt_model_add_doc(tmt_model* m, const char* words, uint32_t n_words, int64_t* doc_id)
{
    if (!m || !doc_id || (n_words && !words)) return TMT_ERR_INVALID_ARGUMENT;
    return guard(m, [&] {
        if (m->prepared) throw ArgErr("cannot add_doc() after train()");
        *doc_id = -1;
        if (!n_words) return;             // an empty document is ignored (TopicModel.hpp:399)
        auto ws = split_words(words, n_words);
        Doc d;
        d.words.reserve(n_words);
        for (auto& w : ws) d.words.push_back(m->add_word(w));
        m->vocabCf.resize(m->id2word.size());
        m->vocabDf.resize(m->id2word.size());
        for (auto w : d.words) ++m->vocabCf[w];
        std::unordered_set<uint32_t> uniq(d.words.begin(), d.words.end());
        for (auto w : uniq) ++m->vocabDf[w];
        m->docs.push_back(std::move(d));
        *doc_id = (int64_t)m->docs.size() - 1;
    });
}

tmt_status tmt_model_set_word_prior(tmt_model* m, const char* word, const float* prior, uint32_t n)
{
    if (!m || !word || (n && !prior)) return TMT_ERR_INVALID_ARGUMENT;
    return guard(m, [&] {
        if (m->prepared) throw ArgErr("cannot set_word_prior() after train()");
        if (n != m->K) throw ArgErr("priors.size() must be equal to K.");
        for (uint32_t k = 0; k < n; ++k)
            if (!(prior[k] >= 0.f)) throw ArgErr("priors must not be less than 0.");
        const std::string w(word);
        m->add_word(w);
        m->vocabCf.resize(m->id2word.size());
        m->vocabDf.resize(m->id2word.size());
        if (!m->prior_of(w)) m->etaByWord.emplace_back(w, std::vector<float>(prior, prior + n));
    });
}

tmt_status tmt_model_get_word_prior(tmt_model* m, const char* word, float* out, uint32_t* n)
{
    if (!m || !word || !n) return TMT_ERR_INVALID_ARGUMENT;
    return guard(m, [&] {
        // getWordPrior (LDAModel.hpp:1047-1062): after preparation with any
        // prior, a word's column of etaByTopicWord (eta for words without one);
        // before, the stored priors
        *n = 0;
        const std::string w(word);
        bool any = false;
        for (auto& e : m->etaByWord) {
            auto it = m->dict.find(e.first);
            if (it != m->dict.end() && it->second < m->realV) any = true;
        }
        if (m->prepared && any) {
            auto it = m->dict.find(w);
            if (it == m->dict.end() || it->second >= m->realV) return;
            const auto* p = m->prior_of(w);
            for (uint32_t k = 0; k < m->K; ++k) if (out) out[k] = p ? (*p)[k] : m->eta;
            *n = m->K;
            return;
        }
        if (const auto* p = m->prior_of(w)) {
            if (out) std::copy(p->begin(), p->end(), out);
            *n = (uint32_t)p->size();
        }
    });
}

tmt_status tmt_model_prepare(tmt_model* m)
{
    if (!m) return TMT_ERR_INVALID_ARGUMENT;
    return guard(m, [&] { m->prepare(); });
}

tmt_status tmt_model_train(tmt_model* m, uint32_t iters)
{
    if (!m) return TMT_ERR_INVALID_ARGUMENT;
    return guard(m, [&] {
        m->prepare();
        m->check(tmt_train(m->eng, iters, 0, nullptr));
        m->host_fresh = false;
    });
}

tmt_status tmt_model_set_optim(tmt_model* m, uint32_t optim_interval, uint32_t burn_in)
{
    if (!m) return TMT_ERR_INVALID_ARGUMENT;
    return guard(m, [&] {
        m->optim_interval = optim_interval;
        m->burn_in = burn_in;
        if (m->eng) m->check(tmt_set_optim(m->eng, optim_interval, burn_in));
    });
}

tmt_status tmt_model_set_seed(tmt_model* m, uint64_t seed)
{
    if (!m) return TMT_ERR_INVALID_ARGUMENT;
    return guard(m, [&] {
        m->seed = seed;
        if (m->eng) m->check(tmt_set_seed(m->eng, seed));
    });
}

tmt_status tmt_model_get_info(tmt_model* m, tmt_model_info* out)
{
    if (!m || !out) return TMT_ERR_INVALID_ARGUMENT;
    return guard(m, [&] {
        out->K = m->K;
        out->V = (uint32_t)m->realV;
        out->n_vocab = (uint32_t)m->id2word.size();
        out->n_docs = m->docs.size();
        out->N = m->realN;
        out->global_step = m->globalStep_now();
        out->prepared = m->prepared;
        out->alpha = m->alpha;
        out->eta = m->eta;
        out->optim_interval = m->optim_interval;
        out->burn_in = m->burn_in;
        out->seed = m->seed;
        out->min_cf = m->min_cf;
        out->min_df = m->min_df;
        out->rm_top = m->rm_top;
        out->tw = m->tw;
        out->weighted_n = m->weightedN;
    });
}

tmt_status tmt_model_ll(tmt_model* m, double* ll_docs, double* ll_rest)
{
    if (!m) return TMT_ERR_INVALID_ARGUMENT;
    return guard(m, [&] {
        if (!m->eng) throw ArgErr("the model is not trained");
        m->check(tmt_ll(m->eng, ll_docs, ll_rest));
    });
}

tmt_status tmt_model_alpha(tmt_model* m, float* out)
{
    if (!m || !out) return TMT_ERR_INVALID_ARGUMENT;
    return guard(m, [&] {
        m->refresh();
        std::copy(m->alphas.begin(), m->alphas.end(), out);
    });
}

tmt_status tmt_model_topic_word_dist(tmt_model* m, uint32_t topic, int normalize, float* out)
{
    if (!m || !out) return TMT_ERR_INVALID_ARGUMENT;
    return guard(m, [&] {
        if (!m->eng && !m->host_fresh) throw ArgErr("the model is not trained");
        if (topic >= m->K) throw ArgErr("must topic_id < K");
        m->refresh();
        // _getWidsByTopic (LDAModel.hpp:828-841)
        const float nt = m->tw ? m->nk_f[topic] : (float)m->nk[topic];
        const float sum = normalize ? nt + (float)m->realV * m->eta : 1.f;
        for (uint64_t v = 0; v < m->realV; ++v) {
            const float c = m->tw ? m->nkw_f[v * m->K + topic] : (float)m->nkw[v * m->K + topic];
            out[v] = (c + m->eta) / sum;
        }
    });
}

tmt_status tmt_model_count_by_topics(tmt_model* m, uint64_t* out)
{
    if (!m || !out) return TMT_ERR_INVALID_ARGUMENT;
    return guard(m, [&] {
        if (!m->eng && !m->host_fresh) throw ArgErr("the model is not trained");
        m->refresh();
        if (m->tw) {
            // _getTopicsCount (LDAModel.hpp:815-826) counts tokens, not weights
            std::fill(out, out + m->K, 0);
            for (auto& d : m->docs)
                for (size_t i = 0; i < d.Zs.size(); ++i)
                    if (d.words[i] < m->realV) ++out[d.Zs[i]];
        } else {
            for (uint32_t k = 0; k < m->K; ++k) out[k] = (uint64_t)m->nk[k];
        }
    });
}

tmt_status tmt_model_vocab(tmt_model* m, uint32_t used_only, char* buf, uint64_t cap, uint64_t* need)
{
    if (!m || !need) return TMT_ERR_INVALID_ARGUMENT;
    return guard(m, [&] {
        const uint64_t n = used_only ? m->realV : m->id2word.size();
        uint64_t total = 0;
        for (uint64_t i = 0; i < n; ++i) total += m->id2word[i].size() + 1;
        *need = total;
        if (!buf || cap < total) return;
        char* p = buf;
        for (uint64_t i = 0; i < n; ++i) {
            std::memcpy(p, m->id2word[i].data(), m->id2word[i].size());
            p += m->id2word[i].size();
            *p++ = '\0';
        }
    });
}

tmt_status tmt_model_vocab_freq(tmt_model* m, uint64_t* cf, uint64_t* df)
{
    if (!m) return TMT_ERR_INVALID_ARGUMENT;
    return guard(m, [&] {
        for (size_t i = 0; i < m->id2word.size(); ++i) {
            if (cf) cf[i] = i < m->vocabCf.size() ? m->vocabCf[i] : 0;
            if (df) df[i] = i < m->vocabDf.size() ? m->vocabDf[i] : 0;
        }
    });
}

tmt_status tmt_model_doc(tmt_model* m, uint64_t doc, uint32_t* words, uint16_t* topics, uint32_t* len)
{
    if (!m || !len) return TMT_ERR_INVALID_ARGUMENT;
    return guard(m, [&] {
        if (doc >= m->docs.size()) throw ArgErr("document index out of range");
        if (m->prepared) m->refresh();
        const Doc& d = m->docs[doc];
        *len = (uint32_t)d.words.size();
        // original word order: tomotopy's wOrder mapping (py_LDA.cpp:613-619)
        for (size_t i = 0; i < d.words.size(); ++i) {
            const size_t j = d.wOrder.empty() ? i : d.wOrder[i];
            if (words) words[i] = d.words[j];
            if (topics) topics[i] = d.Zs.empty() ? 0xFFFF : d.Zs[j];
        }
    });
}

tmt_status tmt_model_doc_topic_dist(tmt_model* m, uint64_t doc, int normalize, float* out, double* ll)
{
    if (!m || !out) return TMT_ERR_INVALID_ARGUMENT;
    return guard(m, [&] {
        if (!m->eng && !m->host_fresh) throw ArgErr("the model is not trained");
        if (doc >= m->docs.size()) throw ArgErr("document index out of range");
        m->refresh();
        std::vector<float> row(m->K);
        float n = 0.f;    // getSumWordWeight (LDA.h:104-133): the token count, or the weights' float sum
        if (m->tw) {
            std::copy(m->ndk_f.begin() + doc * m->K, m->ndk_f.begin() + (doc + 1) * m->K, row.begin());
            for (float x : m->docs[doc].wordWeights) n += x;
        } else {
            int32_t c = 0;
            for (uint32_t k = 0; k < m->K; ++k) {
                row[k] = (float)m->ndk[doc * m->K + k];
                c += m->ndk[doc * m->K + k];
            }
            n = (float)c;
        }
        float as = 0.f;
        double asd = 0;
        for (float a : m->alphas) { as += a; asd += a; }
        // _getTopicsByDoc (LDAModel.hpp:1145-1159)
        for (uint32_t k = 0; k < m->K; ++k)
            out[k] = normalize ? (row[k] + m->alphas[k]) / (n + as) : row[k] + m->alphas[k];
        if (ll) {   // getLLDocs for this document (LDAModel.hpp:616-631), FP64
            double s = 0;
            for (uint32_t k = 0; k < m->K; ++k)
                if (row[k] != 0.f) s += std::lgamma((double)row[k] + m->alphas[k]) - std::lgamma((double)m->alphas[k]);
            *ll = s - (std::lgamma((double)n + asd) - std::lgamma(asd));
        }
    });
}

tmt_status tmt_model_infer(tmt_model* m, const char* words, const uint64_t* doc_nwords, uint64_t D, uint32_t iters,
                           uint64_t seed, float* theta, double* ll)
{
    if (!m || (D && !doc_nwords)) return TMT_ERR_INVALID_ARGUMENT;
    return guard(m, [&] {
        if (!m->eng) throw ArgErr("cannot infer with untrained model");
        // makeDoc: words outside the dictionary are dropped (TopicModel.hpp:430-438)
        std::vector<uint64_t> off(D + 1, 0);
        std::vector<uint32_t> ids;
        const char* p = words;
        for (uint64_t d = 0; d < D; ++d) {
            for (uint64_t i = 0; i < doc_nwords[d]; ++i) {
                const size_t l = std::strlen(p);
                auto it = m->dict.find(std::string(p, l));
                if (it != m->dict.end()) ids.push_back(it->second);
                p += l + 1;
            }
            off[d + 1] = ids.size();
        }
        if (m->tw) {
            // the new documents' weights (initializeDocState, LDAModel.hpp:795-809)
            std::vector<float> wt(ids.size()), one;
            std::vector<uint32_t> tf(m->realV, 0);
            for (uint64_t d = 0; d < D; ++d) {
                std::vector<uint32_t> ws(ids.begin() + off[d], ids.begin() + off[d + 1]);
                m->doc_weights(ws, one, tf);
                std::copy(one.begin(), one.end(), wt.begin() + off[d]);
            }
            const float none = 0.f;
            m->check(tmt_infer_batch_weighted(m->eng, ids.data(), off.data(), D, wt.empty() ? &none : wt.data(),
                                              iters, seed, nullptr, theta, ll));
        } else {
            m->check(tmt_infer_batch(m->eng, ids.data(), off.data(), D, iters, seed, nullptr, theta, ll));
        }
    });
}

tmt_status tmt_model_infer_together(tmt_model* m, const char* words, const uint64_t* doc_nwords, uint64_t D,
                                    uint32_t iters, uint64_t seed, float* theta, double* ll)
{
    if (!m || (D && !doc_nwords)) return TMT_ERR_INVALID_ARGUMENT;
    tmt_handle* tmp = nullptr;
    tmt_status st = guard(m, [&] {
        if (!m->eng) throw ArgErr("cannot infer with untrained model");
        m->refresh();
        // makeDoc + prepareDoc: unknown words dropped, each document sorted by id
        std::vector<uint64_t> off(D + 1, 0);
        std::vector<uint32_t> ids;
        const char* p = words;
        for (uint64_t d = 0; d < D; ++d) {
            const size_t b = ids.size();
            for (uint64_t i = 0; i < doc_nwords[d]; ++i) {
                const size_t l = std::strlen(p);
                auto it = m->dict.find(std::string(p, l));
                if (it != m->dict.end()) ids.push_back(it->second);
                p += l + 1;
            }
            std::stable_sort(ids.begin() + b, ids.end());
            off[d + 1] = ids.size();
        }
        // a private state: the model's counts plus the new documents' (LDAModel.hpp:852-893)
        tmt_config c{};
        c.K = m->K;
        c.V = (uint32_t)m->realV;
        c.alpha = m->alphas.data();
        c.eta = m->eta;
        c.seed = seed;
        c.optim_interval = 0;
        c.device = m->device;
        c.sweep_groups = m->sweep_groups;
        {
            tmt_status s2 = tmt_create(&c, &tmp);
            if (s2 != TMT_OK) throw EngineErr(s2, tmp ? tmt_last_error(tmp) : "tmt_create failed");
        }
        auto ck = [&](tmt_status s2) { if (s2 != TMT_OK) throw EngineErr(s2, tmt_last_error(tmp)); };
        {   // the model's word priors apply to the private state too
            std::vector<uint32_t> pids;
            std::vector<float> pvals;
            m->prior_table(pids, pvals);
            ck(tmt_set_word_priors(tmp, (uint32_t)pids.size(), pids.data(), pvals.data()));
        }
        if (m->tw) {
            // weighted: the new documents' weights; the private state adds the
            // model's float counts to the documents' (float adds)
            std::vector<float> wt(ids.size()), one;
            std::vector<uint32_t> tf(m->realV, 0);
            for (uint64_t d = 0; d < D; ++d) {
                std::vector<uint32_t> ws(ids.begin() + off[d], ids.begin() + off[d + 1]);
                m->doc_weights(ws, one, tf);
                std::copy(one.begin(), one.end(), wt.begin() + off[d]);
            }
            const float none = 0.f;
            ck(tmt_upload_corpus_weighted(tmp, ids.data(), off.data(), D, nullptr, wt.empty() ? &none : wt.data()));
            std::vector<float> nkw((uint64_t)m->K * m->realV), nk(m->K);
            ck(tmt_download_counts_f32(tmp, nullptr, nkw.data(), nk.data(), nullptr));
            for (size_t i = 0; i < nkw.size(); ++i) nkw[i] += m->nkw_f[i];
            for (uint32_t k = 0; k < m->K; ++k) nk[k] += m->nk_f[k];
            ck(tmt_set_counts_f32(tmp, nkw.data(), nk.data()));
        } else {
            ck(tmt_upload_corpus(tmp, ids.data(), off.data(), D, nullptr));
            std::vector<int32_t> nkw((uint64_t)m->K * m->realV), nk(m->K);
            ck(tmt_download_state(tmp, nullptr, nkw.data(), nk.data(), nullptr));
            for (size_t i = 0; i < nkw.size(); ++i) nkw[i] += m->nkw[i];
            for (uint32_t k = 0; k < m->K; ++k) nk[k] += m->nk[k];
            ck(tmt_set_counts(tmp, nkw.data(), nk.data()));
        }
        ck(tmt_train(tmp, iters, 0, nullptr));
        double d_docs = 0, d_rest = 0, m_docs = 0, m_rest = 0;
        ck(tmt_ll(tmp, &d_docs, &d_rest));
        m->check(tmt_ll(m->eng, &m_docs, &m_rest));
        if (ll) *ll = d_docs + d_rest - m_rest;
        if (theta && D && m->tw) {
            std::vector<float> ndk(D * m->K), wl(D);
            ck(tmt_download_counts_f32(tmp, ndk.data(), nullptr, nullptr, wl.data()));
            float as = 0.f;
            for (float a : m->alphas) as += a;
            for (uint64_t d = 0; d < D; ++d)
                for (uint32_t k = 0; k < m->K; ++k)
                    theta[d * m->K + k] = (ndk[d * m->K + k] + m->alphas[k]) / (wl[d] + as);
        } else if (theta && D) {
            std::vector<int32_t> ndk(D * m->K);
            ck(tmt_download_doc_topic(tmp, ndk.data()));
            float as = 0.f;
            for (float a : m->alphas) as += a;
            for (uint64_t d = 0; d < D; ++d) {
                int32_t n = 0;
                for (uint32_t k = 0; k < m->K; ++k) n += ndk[d * m->K + k];
                for (uint32_t k = 0; k < m->K; ++k)
                    theta[d * m->K + k] = ((float)ndk[d * m->K + k] + m->alphas[k]) / ((float)n + as);
            }
        }
    });
    if (tmp) tmt_destroy(tmp);
    return st;
}

tmt_status tmt_model_save(tmt_model* m, const uint8_t* extra, uint64_t extra_len, int full, uint8_t** out,
                          uint64_t* out_len)
{
    if (!m || !out || !out_len || (extra_len && !extra)) return TMT_ERR_INVALID_ARGUMENT;
    return guard(m, [&] {
        m->prepare();
        Writer w;
        m->save(w, full != 0, extra, extra_len);
        *out = static_cast<uint8_t*>(std::malloc(std::max<size_t>(1, w.b.size())));
        if (!*out) throw std::bad_alloc();
        std::memcpy(*out, w.b.data(), w.b.size());
        *out_len = w.b.size();
    });
}

void tmt_model_free_buffer(uint8_t* buf)
{
    std::free(buf);
}

tmt_status tmt_model_load(const uint8_t* data, uint64_t len, int32_t device, uint32_t sweep_groups, tmt_model** out,
                          uint8_t** extra, uint64_t* extra_len)
{
    if (!data || !out) return TMT_ERR_INVALID_ARGUMENT;
    *out = nullptr;
    auto* m = new (std::nothrow) tmt_model();
    if (!m) return TMT_ERR_OUT_OF_MEMORY;
    m->device = device;
    m->sweep_groups = sweep_groups;
    std::vector<uint8_t> ex;
    tmt_status st = guard(m, [&] {
        Reader r(data, len);
        m->load(r, ex);
    });
    if (extra && extra_len) {
        *extra = static_cast<uint8_t*>(std::malloc(std::max<size_t>(1, ex.size())));
        if (*extra) std::memcpy(*extra, ex.data(), ex.size());
        *extra_len = ex.size();
    }
    *out = m;
    return st;
}

const char* tmt_model_last_error(const tmt_model* m)
{
    return m ? m->err.c_str() : "null model";
}

void tmt_model_destroy(tmt_model* m)
{
    delete m;
}

} // extern "C"
