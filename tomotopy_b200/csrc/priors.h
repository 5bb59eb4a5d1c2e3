// priors.h -- host-side tables of word priors (tomotopy's etaByTopicWord,
// LDAModel.hpp:724-737) shared by the engine and the inference server.
#pragma once
#include <algorithm>
#include <cstdint>
#include <vector>

namespace tmtk {

// ids[p] (< V, each once) has the eta column vals[p*K .. p*K+K-1].
//   idx[v]  = p for a prior word, -1 otherwise
//   esum[k] = (V - P) * eta + the prior words' values in ascending id, in
//             double, rounded once to float
//   pcum    = each prior row's sequential float cumulative sum (z0 draws)
//   ecum    = the cumulative sum of a column of eta
struct PriorTables {
    std::vector<int32_t> idx;
    std::vector<float> esum, pcum, ecum;
};

inline void build_prior_tables(uint32_t K, uint32_t V, float eta, const std::vector<uint32_t>& ids,
                               const std::vector<float>& vals, PriorTables& t)
{
    const uint32_t P = (uint32_t)ids.size();
    t.idx.assign(V, -1);
    for (uint32_t p = 0; p < P; ++p) t.idx[ids[p]] = (int32_t)p;
    std::vector<uint32_t> by_id(ids.begin(), ids.end());
    std::sort(by_id.begin(), by_id.end());
    t.esum.resize(K);
    for (uint32_t k = 0; k < K; ++k) {
        double sd = (double)(V - P) * (double)eta;
        for (uint32_t v : by_id) sd += (double)vals[(uint64_t)t.idx[v] * K + k];
        t.esum[k] = (float)sd;
    }
    t.pcum.resize((uint64_t)P * K);
    for (uint32_t p = 0; p < P; ++p) {
        float acc = 0.f;
        for (uint32_t k = 0; k < K; ++k) {
            acc = acc + vals[(uint64_t)p * K + k];
            t.pcum[(uint64_t)p * K + k] = acc;
        }
    }
    t.ecum.resize(K);
    float acc = 0.f;
    for (uint32_t k = 0; k < K; ++k) {
        acc = acc + eta;
        t.ecum[k] = acc;
    }
}

} // namespace tmtk
