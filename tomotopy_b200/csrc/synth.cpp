// synth.cpp -- seeded synthetic corpus from the LDA generative process.
//
// Stands in for corpora that are not available offline (tomotopy's
// enwiki-1000 benchmark file and the larger configurations of the same
// shape).  Process, per the workload definitions:
//   phi_t ~ Dirichlet(beta * V * zipf_s)   for t < T true topics, where zipf_s
//           is the Zipf(s) distribution over word ranks (word id = rank);
//   L_d   ~ Poisson(mean) or round(lognormal(mu, sigma)), clipped to [lo, hi];
//   z_di  ~ DirichletMultinomial(doc_alpha * 1_T), drawn with the Polya urn
//           (exactly the marginal of theta_d ~ Dirichlet(doc_alpha) followed
//           by L_d categorical draws, without materialising theta_d);
//   w_di  ~ Categorical(phi_{z_di}) through per-topic alias tables.
// Every random number is Philox4x32-10 keyed by the seed, with counters
// (document, draw index), so the corpus is identical for any thread count.
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>
#include <thread>
#include <algorithm>
#include <numeric>
#include "philox.cuh"
#include "../../include/tomotopy_b200.h"

namespace {

struct Rng {
    uint64_t key;
    uint32_t a, b;       // counter words that identify the stream owner
    uint32_t n = 0;      // draw index
    uint32_t buf[4];
    int left = 0;
    Rng(uint64_t seed, uint32_t a_, uint32_t b_) : key(seed ^ 0x5EEDC0DE5EEDC0DEull), a(a_), b(b_) {}
    uint32_t next()
    {
        if (!left) {
            tmt::u32x4 r = tmt::philox4x32_10(a, b, tmt::kStreamSynth, n++, (uint32_t)key, (uint32_t)(key >> 32));
            buf[0] = r.x; buf[1] = r.y; buf[2] = r.z; buf[3] = r.w;
            left = 4;
        }
        return buf[--left];
    }
    // (0, 1], 53-bit
    double uniform()
    {
        uint64_t hi = next(), lo = next();
        uint64_t m = ((hi << 32) | lo) >> 11;
        return ((double)m + 1.0) * (1.0 / 9007199254740992.0);
    }
    double normal()
    {
        double u1 = uniform(), u2 = uniform();
        return std::sqrt(-2.0 * std::log(u1)) * std::cos(6.283185307179586 * u2);
    }
    // log of a Gamma(a, 1) draw (Marsaglia & Tsang 2000, with the a < 1 boost
    // done in log space so that tiny shapes do not underflow).
    double log_gamma_draw(double a)
    {
        double boost = 0.0;
        if (a < 1.0) {
            boost = std::log(uniform()) / a;
            a += 1.0;
        }
        const double d = a - 1.0 / 3.0, c = 1.0 / std::sqrt(9.0 * d);
        for (;;) {
            double x = normal(), v = 1.0 + c * x;
            if (v <= 0) continue;
            v = v * v * v;
            double u = uniform();
            if (std::log(u) < 0.5 * x * x + d - d * v + d * std::log(v))
                return std::log(d * v) + boost;
        }
    }
    uint32_t poisson_small(double lam)   // Knuth; lam <= 60
    {
        double L = std::exp(-lam), p = 1.0;
        uint32_t k = 0;
        do { ++k; p *= uniform(); } while (p > L);
        return k - 1;
    }
};

struct Alias {
    std::vector<uint32_t> word;   // support
    std::vector<float> prob;
    std::vector<uint32_t> alias;
};

// Vose's alias method over a sparse support.
void build_alias(const std::vector<double>& p, const std::vector<uint32_t>& ids, Alias& out)
{
    size_t n = ids.size();
    out.word = ids;
    out.prob.assign(n, 0.f);
    out.alias.assign(n, 0);
    double s = 0;
    for (double x : p) s += x;
    std::vector<double> q(n);
    std::vector<uint32_t> small, large;
    for (size_t i = 0; i < n; ++i) {
        q[i] = p[i] / s * (double)n;
        (q[i] < 1.0 ? small : large).push_back((uint32_t)i);
    }
    while (!small.empty() && !large.empty()) {
        uint32_t l = small.back(); small.pop_back();
        uint32_t g = large.back(); large.pop_back();
        out.prob[l] = (float)q[l];
        out.alias[l] = g;
        q[g] = (q[g] + q[l]) - 1.0;
        (q[g] < 1.0 ? small : large).push_back(g);
    }
    for (uint32_t i : large) { out.prob[i] = 1.f; out.alias[i] = i; }
    for (uint32_t i : small) { out.prob[i] = 1.f; out.alias[i] = i; }
}

uint32_t doc_length(const tmt_synth_spec& s, Rng& r)
{
    double L;
    if (s.len_kind == TMT_LEN_POISSON) {
        double lam = s.len_a, acc = 0;
        // Poisson(lam) as a sum of Poisson(lam / m) pieces with lam / m <= 50
        uint32_t m = (uint32_t)std::ceil(lam / 50.0);
        if (m < 1) m = 1;
        for (uint32_t i = 0; i < m; ++i) acc += r.poisson_small(lam / m);
        L = acc;
    } else {
        L = std::floor(std::exp(s.len_a + s.len_b * r.normal()) + 0.5);
    }
    if (L < s.len_min) L = s.len_min;
    if (L > s.len_max) L = s.len_max;
    return (uint32_t)L;
}

template <class F>
void parallel_for(uint64_t n, uint32_t threads, F&& f)
{
    if (threads <= 1 || n < 64) { f(0, n); return; }
    std::vector<std::thread> th;
    for (uint32_t i = 0; i < threads; ++i) {
        uint64_t b = n * i / threads, e = n * (i + 1) / threads;
        th.emplace_back([&, b, e] { f(b, e); });
    }
    for (auto& t : th) t.join();
}

} // namespace

extern "C" tmt_status tmt_synth_corpus(const tmt_synth_spec* spec, uint64_t* doc_off,
                                       uint32_t* words, uint64_t capacity, uint64_t* n_tokens)
{
    if (!spec || !doc_off || !n_tokens) return TMT_ERR_INVALID_ARGUMENT;
    const tmt_synth_spec s = *spec;
    if (s.V == 0 || s.T == 0 || s.D == 0 || s.len_min > s.len_max || s.len_max == 0)
        return TMT_ERR_INVALID_ARGUMENT;
    uint32_t threads = s.threads ? s.threads : std::max(1u, std::thread::hardware_concurrency());
    try {
        // document lengths (stream owner: doc id, tag 0)
        std::vector<uint32_t> len(s.D);
        parallel_for(s.D, threads, [&](uint64_t b, uint64_t e) {
            for (uint64_t d = b; d < e; ++d) {
                const uint64_t dd = d + s.doc_offset;
                Rng r(s.seed, (uint32_t)dd, 0x4C454E00u | (uint32_t)(dd >> 32));
                len[d] = doc_length(s, r);
            }
        });
        doc_off[0] = 0;
        for (uint64_t d = 0; d < s.D; ++d) doc_off[d + 1] = doc_off[d] + len[d];
        *n_tokens = doc_off[s.D];
        if (!words) return TMT_OK;
        if (capacity < *n_tokens) return TMT_ERR_INVALID_ARGUMENT;

        // topic-word distributions, sparse support (stream owner: topic, tag 1)
        std::vector<double> zipf(s.V);
        double zs = 0;
        for (uint32_t v = 0; v < s.V; ++v) { zipf[v] = std::pow((double)(v + 1), -s.zipf_s); zs += zipf[v]; }
        std::vector<Alias> topics(s.T);
        parallel_for(s.T, threads, [&](uint64_t b, uint64_t e) {
            std::vector<double> lg(s.V);
            for (uint64_t t = b; t < e; ++t) {
                Rng r(s.seed, (uint32_t)t, 0x50484900u);
                double mx = -INFINITY;
                for (uint32_t v = 0; v < s.V; ++v) {
                    double a = s.topic_beta * (double)s.V * zipf[v] / zs;
                    lg[v] = r.log_gamma_draw(a);
                    mx = std::max(mx, lg[v]);
                }
                std::vector<double> p;
                std::vector<uint32_t> ids;
                for (uint32_t v = 0; v < s.V; ++v) {
                    double x = lg[v] - mx;
                    if (x < -40.0) continue;          // mass below 4e-18 of the top word
                    p.push_back(std::exp(x));
                    ids.push_back(v);
                }
                build_alias(p, ids, topics[t]);
            }
        });

        // tokens (stream owner: doc id, tag 2)
        const double conc = s.doc_alpha * (double)s.T;
        parallel_for(s.D, threads, [&](uint64_t b, uint64_t e) {
            std::vector<uint32_t> zt;
            for (uint64_t d = b; d < e; ++d) {
                const uint64_t dd = d + s.doc_offset;
                Rng r(s.seed, (uint32_t)dd, 0x544F4B00u | (uint32_t)(dd >> 32));
                uint32_t L = len[d];
                zt.resize(L);
                uint32_t* out = words + doc_off[d];
                for (uint32_t i = 0; i < L; ++i) {
                    // Polya urn: new table with prob conc / (i + conc)
                    double u = r.uniform() * ((double)i + conc);
                    uint32_t z;
                    if (u < conc || i == 0) z = r.next() % s.T;
                    else z = zt[std::min<uint32_t>((uint32_t)(u - conc), i - 1)];
                    zt[i] = z;
                    const Alias& A = topics[z];
                    uint32_t n = (uint32_t)A.word.size();
                    uint32_t j = (uint32_t)(((uint64_t)r.next() * n) >> 32);
                    float f = (float)(r.next() >> 8) * (1.0f / 16777216.0f);
                    out[i] = A.word[f < A.prob[j] ? j : A.alias[j]];
                }
            }
        });
    } catch (...) {
        return TMT_ERR_OUT_OF_MEMORY;
    }
    return TMT_OK;
}
