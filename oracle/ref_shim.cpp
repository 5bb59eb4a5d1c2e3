/*
 * ref_shim.cpp -- exposes tomotopy's own numeric primitives, compiled from
 * the tomotopy source tree (src/Utils/math.h, LUT.hpp, sample.hpp,
 * Utils.hpp), through a C ABI so the oracle's restatements can be pinned
 * against them bit-exactly.  TEST INFRASTRUCTURE ONLY; built into
 * oracle/_ref/ by oracle/Makefile (REF=<tomotopy tree>); never shipped.
 */
#include <cstdint>
#include <cstddef>
#include <vector>
#include <numeric>
#include <cassert>
#include "exception.h"
#include "math.h"
#include "sample.hpp"
#include "Utils.hpp"

namespace {
struct FixedUniform {           // stands in for the RNG: uniform_real() returns u
    float u;
    float uniform_real() { return u; }
};
}

extern "C" {

float ref_lgammaT(float x) { return tomoto::math::lgammaT(x); }
float ref_digammaT(float x) { return tomoto::math::digammaT(x); }
float ref_digammaf(float x) { return tomoto::math::digammaf(x); }
/* math.h:170-176 instantiated for a scalar float (C++ promotes to double) */
double ref_digammaApprox(float x) { return (double)tomoto::math::digammaApprox(x); }

/* sample.hpp:62-86 -- arr must be 16-byte aligned */
void ref_prefix_sum(float* arr, int n) { tomoto::sample::prefixSum(arr, n); }

/* sample.hpp:133-189 -- cum must be 32-byte aligned (AVX loads) */
size_t ref_sample_acc(const float* cum, size_t K, float u)
{
    FixedUniform rg{ u };
    return tomoto::sample::sampleFromDiscreteAcc(cum, cum + K, rg);
}

/* Utils.hpp:157-178 */
void ref_shuffled_order(size_t N, size_t seed, uint64_t* out)
{
    size_t i = 0;
    tomoto::forShuffled(N, seed, [&](size_t id) { out[i++] = id; });
}

/* Utils.hpp:227-248 on a u32 vector: words sorted in place, order[old] = new */
void ref_sort_and_write_order(uint32_t* words, size_t n, uint32_t* order)
{
    std::vector<uint32_t> v(words, words + n), o;
    tomoto::sortAndWriteOrder(v, o);
    for (size_t i = 0; i < n; ++i) { words[i] = v[i]; order[i] = o[i]; }
}

/* sortAndWriteOrder over (cf, df) pairs with removeStopwords' comparator and
 * rotate (TopicModel.hpp:526-571, restated only as the call it makes into
 * Utils.hpp; the comparator lambda is the reference's rule). */
uint64_t ref_remove_stopwords(uint64_t nv, uint64_t* cf, uint64_t* df,
                              uint64_t minWordCnt, uint64_t minWordDf, uint64_t removeTopN,
                              uint32_t* order_out)
{
    std::vector<std::pair<size_t, size_t>> vocabCfDf;
    for (size_t i = 0; i < nv; ++i) vocabCfDf.emplace_back(cf[i], df[i]);
    std::vector<uint32_t> order;
    tomoto::sortAndWriteOrder(vocabCfDf, order, removeTopN, [&](const std::pair<size_t, size_t>& a, const std::pair<size_t, size_t>& b)
    {
        if (a.first < minWordCnt || a.second < minWordDf)
        {
            if (b.first < minWordCnt || b.second < minWordDf) return a > b;
            return false;
        }
        if (b.first < minWordCnt || b.second < minWordDf) return true;
        return a > b;
    });
    uint64_t realV = std::find_if(vocabCfDf.begin(), vocabCfDf.end() - std::min((size_t)removeTopN, vocabCfDf.size()),
        [&](const std::pair<size_t, size_t>& a) { return a.first < minWordCnt || a.second < minWordDf; }) - vocabCfDf.begin();
    for (size_t i = 0; i < nv; ++i) { cf[i] = vocabCfDf[i].first; df[i] = vocabCfDf[i].second; order_out[i] = order[i]; }
    return realV;
}

}
