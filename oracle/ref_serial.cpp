/*
 * ref_serial.cpp -- writes an LDA model file with tomotopy's own serializer
 * (src/Utils/serializer.hpp/.cpp, Dictionary.cpp, SharedString.cpp,
 * tvector.hpp compiled from the tomotopy tree), in the order of
 * TopicModel::_saveModel (TopicModel.hpp:335-359) with LDAModel's tagged
 * fields (LDAModel.hpp:958-960) and the DocumentBase / DocumentLDA tagged
 * fields (TopicModel.hpp:127-131, LDAModel.cpp:5-6).  The two Eigen-typed
 * fields (alphas, numByTopic) are written as Serializer<Eigen::Matrix<T,-1,1>>
 * does (serializer.hpp:499-511): rows, cols, raw data.
 * TEST INFRASTRUCTURE ONLY (oracle/_ref).
 */
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <sstream>
#include <string>
#include <vector>
#include <unordered_map>
#include "serializer.hpp"
#include "Dictionary.h"
#include "SharedString.h"
#include "tvector.hpp"

using namespace tomoto;

namespace {
void write_vec_eigen(std::ostream& o, const float* p, uint32_t n)
{
    serializer::writeMany(o, (uint32_t)n, (uint32_t)1);
    o.write((const char*)p, sizeof(float) * n);
}
void write_vec_eigen(std::ostream& o, const int32_t* p, uint32_t n)
{
    serializer::writeMany(o, (uint32_t)n, (uint32_t)1);
    o.write((const char*)p, sizeof(int32_t) * n);
}
}

extern "C" int ref_write_lda(const char* vocab, uint32_t n_vocab, const uint64_t* cf, const uint64_t* df,
                             uint64_t realV, uint64_t globalStep, const uint8_t* extra, uint64_t extra_len,
                             float alpha, const float* alphas, float eta, uint16_t K, uint32_t burnIn,
                             uint32_t optimInterval, const int32_t* nk, const int32_t* nkw, int full,
                             uint64_t n_docs, const uint64_t* doc_off, const uint32_t* words, const uint32_t* w_order,
                             const uint16_t* zs, uint8_t** out, uint64_t* out_len)
{
    std::ostringstream w;
    Dictionary dict;
    const char* p = vocab;
    for (uint32_t i = 0; i < n_vocab; ++i) { dict.add(std::string(p)); p += std::strlen(p) + 1; }
    std::vector<uint64_t> vcf(cf, cf + n_vocab), vdf(df, df + n_vocab);
    std::vector<uint8_t> ex(extra, extra + extra_len);
    size_t gstep = (size_t)globalStep;
    serializer::writeMany(w, serializer::to_keyz(serializer::to_key("LDA\0")), serializer::to_keyz(serializer::to_key("one\0")));
    serializer::writeTaggedMany(w, 0x00010001,
        serializer::to_keyz("dict"), dict,
        serializer::to_keyz("vocabCf"), vcf,
        serializer::to_keyz("vocabDf"), vdf,
        serializer::to_keyz("realV"), realV,
        serializer::to_keyz("globalStep"), gstep,
        serializer::to_keyz("extra"), ex);
    // LDAModel tagged fields: alphas is an Eigen vector, written into a side
    // stream first so that it can be handed to writeTaggedMany as bytes
    struct EigenBytes { std::string b; void serializerWrite(std::ostream& o) const { o.write(b.data(), b.size()); }
                        void serializerRead(std::istream&) {} uint64_t computeHash(uint64_t s) const { return s; } };
    EigenBytes eb;
    { std::ostringstream t; write_vec_eigen(t, alphas, K); eb.b = t.str(); }
    std::vector<float> vocabWeights;
    std::unordered_map<std::string, std::vector<float>> etaByWord;
    serializer::writeTaggedMany(w, 0x00010001,
        serializer::to_keyz("vocabWeights"), vocabWeights,
        serializer::to_keyz("alpha"), alpha,
        serializer::to_keyz("alphas"), eb,
        serializer::to_keyz("eta"), eta,
        serializer::to_keyz("K"), K,
        serializer::to_keyz("etaByWord"), etaByWord,
        serializer::to_keyz("burnIn"), burnIn,
        serializer::to_keyz("optimInterval"), optimInterval);
    // globalState: numByTopic (Eigen vector), numByTopicWord (ShareableMatrix::serializerWrite, LDA.h:89-95)
    write_vec_eigen(w, nk, K);
    serializer::writeToStream<uint32_t>(w, (uint32_t)K);
    serializer::writeToStream<uint32_t>(w, (uint32_t)realV);
    w.write((const char*)nkw, sizeof(int32_t) * (uint64_t)K * realV);
    if (!full) {
        serializer::writeMany(w, std::vector<size_t>{});
    } else {
        serializer::writeToStream<uint32_t>(w, (uint32_t)n_docs);
        for (uint64_t d = 0; d < n_docs; ++d) {
            const uint64_t b = doc_off[d], n = doc_off[d + 1] - b;
            float weight = 1.f;
            tvector<uint32_t> dw((uint32_t*)words + b, n);
            std::vector<uint32_t> wo(w_order + b, w_order + b + n);
            SharedString rawStr, docUid;
            std::vector<uint32_t> origWordPos;
            std::vector<uint16_t> origWordLen;
            serializer::writeTaggedMany(w, 0x00010001,
                serializer::to_keyz("weight"), weight,
                serializer::to_keyz("words"), dw,
                serializer::to_keyz("wOrder"), wo,
                serializer::to_keyz("rawStr"), rawStr,
                serializer::to_keyz("origWordPos"), origWordPos,
                serializer::to_keyz("origWordLen"), origWordLen,
                serializer::to_keyz("docUid"), docUid);
            tvector<uint16_t> z((uint16_t*)zs + b, n);
            tvector<float> wordWeights;
            serializer::writeTaggedMany(w, 0x00010001,
                serializer::to_keyz("Zs"), z,
                serializer::to_keyz("wordWeights"), wordWeights);
        }
    }
    const std::string s = w.str();
    *out = (uint8_t*)std::malloc(s.size() ? s.size() : 1);
    std::memcpy(*out, s.data(), s.size());
    *out_len = s.size();
    return 0;
}

extern "C" void ref_free(uint8_t* p) { std::free(p); }
