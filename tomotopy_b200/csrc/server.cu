// server.cu -- continuous-batching inference over frozen models resident on
// one GPU (tmt_server_* in include/tomotopy_b200.h).
//
// A worker thread runs steps.  Each step it admits queued requests into free
// slots of their model's slot pool and into free space of the shared token
// arena (the HBM budget for documents in flight), then launches the
// resumable inference kernel (infer.cuh) once per model with active slots
// (each model on its own stream, so the models of one step run concurrently),
// advancing every active document by ceil(step_token_sweeps / length) sweeps
// (at least one), so long documents do not stall a step.  Documents that have
// done all their sweeps leave with their theta and log-likelihood.  Requests
// arriving while others are on the GPU join at the next step.  A document's
// draws depend only on its model, words, seed and key, so its result is the
// same alone or in any mix.  All waits are host-side and bounded.
#include <cuda_runtime.h>
#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <thread>
#include <vector>
#include "common.cuh"
#include "infer.cuh"
#include "priors.h"
#include "philox.cuh"
#include "../../include/tomotopy_b200.h"

using namespace tmtk;
using Clock = std::chrono::steady_clock;

namespace {

// copies admitted documents from the contiguous staging buffer into the arena
__global__ void k_scatter_docs(const uint32_t* __restrict__ staging, const uint64_t* __restrict__ src,
                               const uint64_t* __restrict__ dst, const uint32_t* __restrict__ len, uint32_t n,
                               uint32_t* __restrict__ arena)
{
    for (uint32_t i = blockIdx.x; i < n; i += gridDim.x)
        for (uint32_t j = threadIdx.x; j < len[i]; j += blockDim.x) arena[dst[i] + j] = staging[src[i] + j];
}

// packs the outputs of finished slots: theta rows and ll
__global__ void k_gather_results(const float* __restrict__ theta, const double* __restrict__ ll,
                                 const uint32_t* __restrict__ slots, uint32_t n, uint32_t K,
                                 float* __restrict__ out_theta, double* __restrict__ out_ll)
{
    for (uint32_t i = blockIdx.x; i < n; i += gridDim.x) {
        const uint32_t sl = slots[i];
        for (uint32_t k = threadIdx.x; k < K; k += blockDim.x) out_theta[(uint64_t)i * K + k] = theta[(uint64_t)sl * K + k];
        if (threadIdx.x == 0) out_ll[i] = ll[sl];
    }
}

template <class T>
T* pinned(size_t n)
{
    void* p = nullptr;
    if (cudaMallocHost(&p, std::max<size_t>(16, n * sizeof(T))) != cudaSuccess) {
        cudaGetLastError();
        throw OomError("cudaMallocHost failed");
    }
    return static_cast<T*>(p);
}

struct Request {
    uint64_t id;
    uint32_t model;
    std::vector<uint32_t> words;   // sorted by id
    std::vector<float> wts;        // weighted models: the tokens' weights, in the same order
    uint32_t iters;
    uint64_t seed, key;
    Clock::time_point t_submit;
};

struct Result {
    uint64_t id;
    uint32_t model;
    std::vector<float> theta;
    double ll;
    double latency_ms, queue_ms;
};

// first-fit allocator over [0, cap) tokens
struct Arena {
    std::map<uint64_t, uint64_t> free_;   // begin -> length
    uint64_t cap = 0, used = 0;
    void init(uint64_t c) { cap = c; free_.clear(); if (c) free_[0] = c; used = 0; }
    bool alloc(uint64_t n, uint64_t& at)
    {
        if (n == 0) { at = 0; return true; }
        for (auto it = free_.begin(); it != free_.end(); ++it) {
            if (it->second >= n) {
                at = it->first;
                const uint64_t rest = it->second - n;
                free_.erase(it);
                if (rest) free_[at + n] = rest;
                used += n;
                return true;
            }
        }
        return false;
    }
    void release(uint64_t at, uint64_t n)
    {
        if (n == 0) return;
        used -= n;
        auto it = free_.emplace(at, n).first;
        auto nx = std::next(it);
        if (nx != free_.end() && it->first + it->second == nx->first) {
            it->second += nx->second;
            free_.erase(nx);
        }
        if (it != free_.begin()) {
            auto pv = std::prev(it);
            if (pv->first + pv->second == it->first) {
                pv->second += it->second;
                free_.erase(it);
            }
        }
    }
};

struct Model {
    cudaStream_t stream = nullptr;       // this model's launches; models of one step run concurrently
    cudaEvent_t ev_done = nullptr;
    uint32_t K = 0, V = 0;
    float eta = 0;
    std::vector<float> alpha;
    float asum_f = 0;
    double asum_d = 0;
    int32_t* d_nkw = nullptr;
    int32_t* d_nk = nullptr;
    float* d_alpha = nullptr;
    float* d_acum = nullptr;
    // slot pool
    uint32_t slots = 0;
    std::vector<int> active;            // request index per slot, -1 free
    std::vector<Request> req;           // request per slot
    // per-slot metadata, pinned host mirrors of the device arrays
    uint64_t* h_tok_begin = nullptr;
    uint32_t *h_tok_len = nullptr, *h_it_begin = nullptr, *h_it_end = nullptr, *h_it_total = nullptr;
    uint64_t* h_keys = nullptr;
    uint32_t* h_work = nullptr;
    uint32_t* h_fin = nullptr;
    float* h_out_theta = nullptr;
    double* h_out_ll = nullptr;
    std::vector<uint32_t> h_done;
    uint32_t* d_fin = nullptr;
    float* d_out_theta = nullptr;
    double* d_out_ll = nullptr;
    uint64_t* d_tok_begin = nullptr;
    uint32_t *d_tok_len = nullptr, *d_it_begin = nullptr, *d_it_end = nullptr, *d_it_total = nullptr;
    uint64_t* d_keys = nullptr;
    int32_t* d_ndk = nullptr;
    float* d_theta = nullptr;
    double* d_ll = nullptr;
    uint32_t* d_work = nullptr;
    uint32_t* d_counter = nullptr;
    // word priors (tmt_server_set_model_priors; all NULL: none)
    int32_t* d_pidx = nullptr;
    float* d_pval = nullptr;
    float* d_esum = nullptr;
    float* d_pcum = nullptr;
    float* d_ecum = nullptr;
    bool used = false;                  // a request was submitted: the model is frozen
    bool weighted = false;              // float counts (TermWeight IDF / PMI); requests carry weights
};

} // namespace

struct tmt_server {
    tmt_server_config cfg{};
    int device = 0, num_sms = 0;
    cudaStream_t stream = nullptr;
    std::vector<void*> allocs;
    uint32_t* d_words = nullptr;
    uint16_t* d_z = nullptr;
    uint32_t* d_staging = nullptr;               // admitted documents of one step, contiguous
    uint32_t* h_staging = nullptr;               // pinned
    // token weights beside the arena's words, allocated with the first weighted model
    float* d_wt = nullptr;
    float* d_wstaging = nullptr;
    float* h_wstaging = nullptr;
    uint64_t *h_sc_src = nullptr, *h_sc_dst = nullptr, *d_sc_src = nullptr, *d_sc_dst = nullptr;
    uint32_t *h_sc_len = nullptr, *d_sc_len = nullptr;
    std::vector<void*> pinned_allocs;
    uint64_t sc_cap = 0;                         // documents one step may admit
    Arena arena;
    std::vector<std::unique_ptr<Model>> models;

    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    std::deque<Request> queue;
    std::deque<Result> results;
    uint64_t next_id = 1;
    bool stop = false;
    std::thread worker;
    std::string err;
    tmt_status worker_status = TMT_OK;
    // statistics
    uint64_t steps = 0, completed = 0, active_sum = 0, tokens_in_flight_max = 0;
    uint64_t token_sweeps = 0;                   // token-sweeps advanced
    double alg_bytes = 0;                        // token-sweeps x (4K + 8) per model
    double kernel_ms = 0, busy_ms = 0;           // inference launches (events); whole steps (wall)
    cudaEvent_t ev_k0 = nullptr, ev_k1 = nullptr;

    template <class T>
    T* dalloc(size_t n)
    {
        void* p = nullptr;
        const size_t b = std::max<size_t>(16, n * sizeof(T));
        cudaError_t e = cudaMalloc(&p, b);
        if (e != cudaSuccess) {
            cudaGetLastError();
            throw OomError(std::string("cudaMalloc: ") + cudaGetErrorString(e));
        }
        allocs.push_back(p);
        return static_cast<T*>(p);
    }
    template <class T>
    T* palloc(size_t n)
    {
        T* p = pinned<T>(n);
        pinned_allocs.push_back(p);
        return p;
    }
    ~tmt_server()
    {
        cudaSetDevice(device);
        if (stream) cudaStreamSynchronize(stream);
        for (void* p : allocs) cudaFree(p);
        for (void* p : pinned_allocs) cudaFreeHost(p);
        for (auto& m : models) {
            if (m->ev_done) cudaEventDestroy(m->ev_done);
            if (m->stream) cudaStreamDestroy(m->stream);
        }
        if (ev_k0) cudaEventDestroy(ev_k0);
        if (ev_k1) cudaEventDestroy(ev_k1);
        if (stream) cudaStreamDestroy(stream);
    }
};

namespace {

// One step of the worker; returns false when there was nothing to do.
bool server_step(tmt_server* s)
{
    const auto t_step = Clock::now();
    std::vector<std::pair<Model*, uint32_t>> admitted;   // (model, slot)
    std::vector<Model*> models;                          // tmt_server_add_model may append meanwhile
    {
        std::lock_guard<std::mutex> lk(s->mu);
        for (auto& mp : s->models) models.push_back(mp.get());
        while (!s->queue.empty() && admitted.size() < s->sc_cap) {
            Request& r = s->queue.front();
            Model* m = s->models[r.model].get();
            auto it = std::find(m->active.begin(), m->active.end(), -1);
            if (it == m->active.end()) break;            // no slot: wait (head of line)
            uint64_t at = 0;
            if (!s->arena.alloc(r.words.size(), at)) break;   // over the budget: wait
            const uint32_t sl = (uint32_t)(it - m->active.begin());
            m->active[sl] = 1;
            m->h_tok_begin[sl] = at;
            m->h_tok_len[sl] = (uint32_t)r.words.size();
            m->h_keys[sl] = r.key;
            m->h_it_total[sl] = r.iters;
            m->h_done[sl] = 0;
            m->req[sl] = std::move(r);
            s->queue.pop_front();
            admitted.emplace_back(m, sl);
        }
        s->tokens_in_flight_max = std::max<uint64_t>(s->tokens_in_flight_max, s->arena.used);
    }
    // the admitted documents: packed into pinned staging, one copy, one scatter
    if (!admitted.empty()) {
        uint64_t off = 0;
        uint32_t n = 0;
        for (auto& [m, sl] : admitted) {
            const uint32_t len = m->h_tok_len[sl];
            if (!len) continue;
            std::memcpy(s->h_staging + off, m->req[sl].words.data(), len * sizeof(uint32_t));
            if (m->weighted) std::memcpy(s->h_wstaging + off, m->req[sl].wts.data(), len * sizeof(float));
            s->h_sc_src[n] = off;
            s->h_sc_dst[n] = m->h_tok_begin[sl];
            s->h_sc_len[n] = len;
            off += len;
            ++n;
        }
        if (n) {
            CK(cudaMemcpyAsync(s->d_staging, s->h_staging, off * sizeof(uint32_t), cudaMemcpyHostToDevice, s->stream));
            CK(cudaMemcpyAsync(s->d_sc_src, s->h_sc_src, n * sizeof(uint64_t), cudaMemcpyHostToDevice, s->stream));
            CK(cudaMemcpyAsync(s->d_sc_dst, s->h_sc_dst, n * sizeof(uint64_t), cudaMemcpyHostToDevice, s->stream));
            CK(cudaMemcpyAsync(s->d_sc_len, s->h_sc_len, n * sizeof(uint32_t), cudaMemcpyHostToDevice, s->stream));
            k_scatter_docs<<<std::min<uint32_t>(n, 4096), 128, 0, s->stream>>>(s->d_staging, s->d_sc_src, s->d_sc_dst,
                                                                              s->d_sc_len, n, s->d_words);
            CK(cudaGetLastError());
            if (s->d_wt) {
                // the weights (4-byte values, moved by the same scatter; stale for unweighted documents)
                CK(cudaMemcpyAsync(s->d_wstaging, s->h_wstaging, off * sizeof(float), cudaMemcpyHostToDevice,
                                   s->stream));
                k_scatter_docs<<<std::min<uint32_t>(n, 4096), 128, 0, s->stream>>>(
                    reinterpret_cast<const uint32_t*>(s->d_wstaging), s->d_sc_src, s->d_sc_dst, s->d_sc_len, n,
                    reinterpret_cast<uint32_t*>(s->d_wt));
                CK(cudaGetLastError());
            }
        }
    }
    bool any = false;
    std::vector<std::pair<Model*, uint32_t>> finishing;
    std::vector<uint32_t> nfin(models.size(), 0);
    std::vector<char> active_model(models.size(), 0);
    // Each document advances about step_token_sweeps token-sweeps per step.  When
    // the documents in flight cannot fill the GPU's resident warps (32 per SM),
    // each advances proportionally more, at most 4x: otherwise a tail of long
    // documents runs one sweep per step with the GPU nearly idle, while a larger
    // factor makes new arrivals wait behind long steps (64x doubled the p99 at
    // 1k requests/s on config 4).
    uint64_t n_active = 0;
    for (Model* m : models)
        for (uint32_t sl = 0; sl < m->slots; ++sl) n_active += m->active[sl] >= 0;
    const uint64_t capacity = (uint64_t)s->num_sms * 32;
    const uint64_t scale = n_active ? std::min<uint64_t>(4, std::max<uint64_t>(1, capacity / n_active)) : 1;
    const uint64_t quota = (uint64_t)s->cfg.step_token_sweeps * scale;
    for (size_t mi = 0; mi < models.size(); ++mi) {
        Model* m = models[mi];
        std::vector<uint32_t> work;
        for (uint32_t sl = 0; sl < m->slots; ++sl) {
            if (m->active[sl] < 0) continue;
            const uint32_t len = std::max(1u, m->h_tok_len[sl]);
            const uint32_t adv = (uint32_t)std::min<uint64_t>(0xFFFFFFFFu, std::max<uint64_t>(1, (quota + len - 1) / len));
            m->h_it_begin[sl] = m->h_done[sl];
            m->h_it_end[sl] = (uint32_t)std::min<uint64_t>(m->h_it_total[sl], (uint64_t)m->h_done[sl] + adv);
            const uint64_t ts = (uint64_t)(m->h_it_end[sl] - m->h_it_begin[sl]) * m->h_tok_len[sl];
            s->token_sweeps += ts;
            s->alg_bytes += (double)ts * (4.0 * m->K + 8.0);
            work.push_back(sl);
            if (m->h_it_end[sl] == m->h_it_total[sl]) {
                finishing.emplace_back(m, sl);
                m->h_fin[nfin[mi]++] = sl;
            }
        }
        if (work.empty()) continue;
        if (!any) CK(cudaEventRecord(s->ev_k0, s->stream));   // the fork: admitted documents are in place
        any = true;
        cudaStream_t ms = m->stream;
        active_model[mi] = 1;
        CK(cudaStreamWaitEvent(ms, s->ev_k0, 0));
        s->active_sum += work.size();
        const size_t S = m->slots;
        CK(cudaMemcpyAsync(m->d_tok_begin, m->h_tok_begin, S * sizeof(uint64_t), cudaMemcpyHostToDevice, ms));
        CK(cudaMemcpyAsync(m->d_tok_len, m->h_tok_len, S * sizeof(uint32_t), cudaMemcpyHostToDevice, ms));
        CK(cudaMemcpyAsync(m->d_keys, m->h_keys, S * sizeof(uint64_t), cudaMemcpyHostToDevice, ms));
        CK(cudaMemcpyAsync(m->d_it_begin, m->h_it_begin, S * sizeof(uint32_t), cudaMemcpyHostToDevice, ms));
        CK(cudaMemcpyAsync(m->d_it_end, m->h_it_end, S * sizeof(uint32_t), cudaMemcpyHostToDevice, ms));
        CK(cudaMemcpyAsync(m->d_it_total, m->h_it_total, S * sizeof(uint32_t), cudaMemcpyHostToDevice, ms));
        std::copy(work.begin(), work.end(), m->h_work);
        CK(cudaMemcpyAsync(m->d_work, m->h_work, work.size() * sizeof(uint32_t), cudaMemcpyHostToDevice, ms));
        CK(cudaMemsetAsync(m->d_counter, 0, sizeof(uint32_t), ms));
        InferArgs a{};
        a.nkw = m->d_nkw;
        a.nk = m->d_nk;
        a.alpha = m->d_alpha;
        a.acum = m->d_acum;
        a.K = m->K;
        a.V = m->V;
        a.eta = m->eta;
        a.veta = m->eta * (float)m->V;
        a.asum_f = m->asum_f;
        a.veta_d = (double)m->V * (double)m->eta;
        a.asum_d = m->asum_d;
        a.lg_asum = std::lgamma(m->asum_d);
        a.lg_eta = std::lgamma((double)m->eta);
        a.words = s->d_words;
        a.z = s->d_z;
        a.tok_begin = m->d_tok_begin;
        a.tok_len = m->d_tok_len;
        a.keys = m->d_keys;
        a.it_begin = m->d_it_begin;
        a.it_end = m->d_it_end;
        a.it_total = m->d_it_total;
        a.ndk = m->d_ndk;
        a.theta = m->d_theta;
        a.ll = m->d_ll;
        a.work = m->d_work;
        a.n_work = (uint32_t)work.size();
        a.counter = m->d_counter;
        a.wt = m->weighted ? s->d_wt : nullptr;
        a.pidx = m->d_pidx;
        a.pval = m->d_pval;
        a.esum = m->d_esum;
        a.pcum = m->d_pcum;
        a.ecum = m->d_ecum;
        // every request of a model shares the draw key base; the per-request seed is folded in below
        a.key = 0;
        // requests may carry different seeds: launch per distinct seed (usually one)
        std::map<uint64_t, std::vector<uint32_t>> by_seed;
        for (uint32_t sl : work) by_seed[m->req[sl].seed].push_back(sl);
        if (by_seed.size() == 1) {
            a.key = by_seed.begin()->first ^ (uint64_t)tmt::kStreamInfer;
            launch_infer(a, s->num_sms, ms);
        } else {
            uint32_t at = 0;
            for (auto& [seed, sls] : by_seed) {
                std::copy(sls.begin(), sls.end(), m->h_work + at);
                CK(cudaMemcpyAsync(m->d_work + at, m->h_work + at, sls.size() * sizeof(uint32_t), cudaMemcpyHostToDevice, ms));
                a.work = m->d_work + at;
                at += (uint32_t)sls.size();
                CK(cudaMemsetAsync(m->d_counter, 0, sizeof(uint32_t), ms));
                a.n_work = (uint32_t)sls.size();
                a.key = seed ^ (uint64_t)tmt::kStreamInfer;
                launch_infer(a, s->num_sms, ms);
            }
        }
    }
    if (!any) return false;
    // results of the finished documents: packed per model, one copy each
    for (size_t mi = 0; mi < models.size(); ++mi) {
        Model* m = models[mi];
        const uint32_t n = nfin[mi];
        if (n) {
            CK(cudaMemcpyAsync(m->d_fin, m->h_fin, n * sizeof(uint32_t), cudaMemcpyHostToDevice, m->stream));
            k_gather_results<<<std::min<uint32_t>(n, 4096), 128, 0, m->stream>>>(m->d_theta, m->d_ll, m->d_fin, n,
                                                                                 m->K, m->d_out_theta, m->d_out_ll);
            CK(cudaGetLastError());
            CK(cudaMemcpyAsync(m->h_out_theta, m->d_out_theta, (uint64_t)n * m->K * sizeof(float),
                               cudaMemcpyDeviceToHost, m->stream));
            CK(cudaMemcpyAsync(m->h_out_ll, m->d_out_ll, n * sizeof(double), cudaMemcpyDeviceToHost, m->stream));
        }
        if (active_model[mi]) {     // the join
            CK(cudaEventRecord(m->ev_done, m->stream));
            CK(cudaStreamWaitEvent(s->stream, m->ev_done, 0));
        }
    }
    CK(cudaEventRecord(s->ev_k1, s->stream));
    CK(cudaStreamSynchronize(s->stream));
    {
        float ms = 0.f;
        CK(cudaEventElapsedTime(&ms, s->ev_k0, s->ev_k1));
        s->kernel_ms += ms;
    }
    std::vector<Result> out(finishing.size());
    {
        std::vector<uint32_t> seen(models.size(), 0);
        for (size_t i = 0; i < finishing.size(); ++i) {
            auto [m, sl] = finishing[i];
            const size_t mi = std::find(models.begin(), models.end(), m) - models.begin();
            const uint32_t r = seen[mi]++;
            out[i].theta.assign(m->h_out_theta + (uint64_t)r * m->K, m->h_out_theta + (uint64_t)(r + 1) * m->K);
            out[i].ll = m->h_out_ll[r];
        }
    }
    const auto now = Clock::now();
    ++s->steps;
    s->busy_ms += std::chrono::duration<double, std::milli>(now - t_step).count();
    {
        std::lock_guard<std::mutex> lk(s->mu);
        for (Model* m : models)
            for (uint32_t sl = 0; sl < m->slots; ++sl)
                if (m->active[sl] >= 0) m->h_done[sl] = m->h_it_end[sl];
        for (size_t i = 0; i < finishing.size(); ++i) {
            auto [m, sl] = finishing[i];
            Request& r = m->req[sl];
            out[i].id = r.id;
            out[i].model = r.model;
            out[i].latency_ms = std::chrono::duration<double, std::milli>(now - r.t_submit).count();
            out[i].queue_ms = 0;
            s->arena.release(m->h_tok_begin[sl], m->h_tok_len[sl]);
            m->active[sl] = -1;
            r.words.clear();
            r.words.shrink_to_fit();
            s->results.push_back(std::move(out[i]));
            ++s->completed;
        }
    }
    if (!finishing.empty()) s->cv_done.notify_all();
    return true;
}

void server_loop(tmt_server* s)
{
    cudaSetDevice(s->device);
    try {
        for (;;) {
            {
                std::unique_lock<std::mutex> lk(s->mu);
                if (s->stop) break;
            }
            if (!server_step(s)) {
                std::unique_lock<std::mutex> lk(s->mu);
                if (s->stop) break;
                s->cv_work.wait_for(lk, std::chrono::milliseconds(20));
            }
        }
    } catch (const std::exception& e) {
        std::lock_guard<std::mutex> lk(s->mu);
        s->err = e.what();
        s->worker_status = TMT_ERR_CUDA;
        s->stop = true;
        s->cv_done.notify_all();
    }
}

} // namespace

extern "C" {

tmt_status tmt_server_start(const tmt_server_config* cfg, tmt_server** out)
{
    if (!cfg || !out) return TMT_ERR_INVALID_ARGUMENT;
    *out = nullptr;
    if (cfg->max_slots == 0 || cfg->token_budget == 0 || cfg->max_doc_len == 0 || cfg->max_doc_len > cfg->token_budget)
        return TMT_ERR_INVALID_ARGUMENT;
    auto* s = new (std::nothrow) tmt_server();
    if (!s) return TMT_ERR_OUT_OF_MEMORY;
    s->cfg = *cfg;
    if (!s->cfg.step_token_sweeps) s->cfg.step_token_sweeps = 4096;
    s->device = cfg->device;
    try {
        CK(cudaSetDevice(s->device));
        CK(cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking));
        CK(cudaDeviceGetAttribute(&s->num_sms, cudaDevAttrMultiProcessorCount, s->device));
        CK(cudaEventCreate(&s->ev_k0));
        CK(cudaEventCreate(&s->ev_k1));
        s->d_words = s->dalloc<uint32_t>(cfg->token_budget);
        s->d_z = s->dalloc<uint16_t>(cfg->token_budget);
        s->d_staging = s->dalloc<uint32_t>(cfg->token_budget);
        s->h_staging = s->palloc<uint32_t>(cfg->token_budget);
        const uint64_t maxdocs = cfg->token_budget;
        s->sc_cap = std::min<uint64_t>(maxdocs, 1u << 22);
        s->h_sc_src = s->palloc<uint64_t>(std::min<uint64_t>(maxdocs, 1u << 22));
        s->h_sc_dst = s->palloc<uint64_t>(std::min<uint64_t>(maxdocs, 1u << 22));
        s->h_sc_len = s->palloc<uint32_t>(std::min<uint64_t>(maxdocs, 1u << 22));
        s->d_sc_src = s->dalloc<uint64_t>(std::min<uint64_t>(maxdocs, 1u << 22));
        s->d_sc_dst = s->dalloc<uint64_t>(std::min<uint64_t>(maxdocs, 1u << 22));
        s->d_sc_len = s->dalloc<uint32_t>(std::min<uint64_t>(maxdocs, 1u << 22));
        s->arena.init(cfg->token_budget);
    } catch (const OomError&) {
        delete s;
        return TMT_ERR_OUT_OF_MEMORY;
    } catch (...) {
        delete s;
        return TMT_ERR_CUDA;
    }
    s->worker = std::thread(server_loop, s);
    *out = s;
    return TMT_OK;
}

} // extern "C"

namespace {

// n_kw / n_k: int32 counts, or floats when `weighted` (4 bytes either way)
tmt_status add_model_impl(tmt_server* s, uint32_t K, uint32_t V, const float* alpha, float eta, const void* n_kw,
                          const void* n_k, bool weighted, uint32_t* model_id)
{
    if (!s || !alpha || !n_k || (V && !n_kw) || !model_id || K == 0 || K > 32767 || !(eta > 0))
        return TMT_ERR_INVALID_ARGUMENT;
    if (infer_warps(K) == 0) return TMT_ERR_UNSUPPORTED;
    auto m = std::make_unique<Model>();
    m->K = K;
    m->V = V;
    m->eta = eta;
    m->alpha.assign(alpha, alpha + K);
    std::vector<float> acum(K);
    float sf = 0.f;
    double sd = 0;
    for (uint32_t k = 0; k < K; ++k) {
        if (!(alpha[k] > 0)) return TMT_ERR_INVALID_ARGUMENT;
        sf = sf + alpha[k];
        acum[k] = sf;
        sd += (double)alpha[k];
    }
    m->asum_f = sf;
    m->asum_d = sd;
    m->weighted = weighted;
    const uint32_t S = s->cfg.max_slots;
    m->slots = S;
    m->active.assign(S, -1);
    m->req.resize(S);
    m->h_done.assign(S, 0);
    std::lock_guard<std::mutex> lk(s->mu);      // the worker does not allocate meanwhile
    try {
        CK(cudaSetDevice(s->device));
        CK(cudaStreamCreateWithFlags(&m->stream, cudaStreamNonBlocking));
        CK(cudaEventCreateWithFlags(&m->ev_done, cudaEventDisableTiming));
        m->h_tok_begin = s->palloc<uint64_t>(S);
        m->h_keys = s->palloc<uint64_t>(S);
        m->h_tok_len = s->palloc<uint32_t>(S);
        m->h_it_begin = s->palloc<uint32_t>(S);
        m->h_it_end = s->palloc<uint32_t>(S);
        m->h_it_total = s->palloc<uint32_t>(S);
        m->h_work = s->palloc<uint32_t>(S);
        m->h_fin = s->palloc<uint32_t>(S);
        m->h_out_theta = s->palloc<float>((uint64_t)S * K);
        m->h_out_ll = s->palloc<double>(S);
        std::fill(m->h_tok_begin, m->h_tok_begin + S, 0);
        std::fill(m->h_keys, m->h_keys + S, 0);
        std::fill(m->h_tok_len, m->h_tok_len + S, 0);
        std::fill(m->h_it_begin, m->h_it_begin + S, 0);
        std::fill(m->h_it_end, m->h_it_end + S, 0);
        std::fill(m->h_it_total, m->h_it_total + S, 0);
        m->d_fin = s->dalloc<uint32_t>(S);
        m->d_out_theta = s->dalloc<float>((uint64_t)S * K);
        m->d_out_ll = s->dalloc<double>(S);
        m->d_nkw = s->dalloc<int32_t>((uint64_t)K * V);
        m->d_nk = s->dalloc<int32_t>(K);
        m->d_alpha = s->dalloc<float>(K);
        m->d_acum = s->dalloc<float>(K);
        m->d_tok_begin = s->dalloc<uint64_t>(S);
        m->d_tok_len = s->dalloc<uint32_t>(S);
        m->d_keys = s->dalloc<uint64_t>(S);
        m->d_it_begin = s->dalloc<uint32_t>(S);
        m->d_it_end = s->dalloc<uint32_t>(S);
        m->d_it_total = s->dalloc<uint32_t>(S);
        m->d_ndk = s->dalloc<int32_t>((uint64_t)S * K);
        m->d_theta = s->dalloc<float>((uint64_t)S * K);
        m->d_ll = s->dalloc<double>(S);
        m->d_work = s->dalloc<uint32_t>(S);
        m->d_counter = s->dalloc<uint32_t>(1);
        if (weighted && !s->d_wt) {
            s->d_wstaging = s->dalloc<float>(s->cfg.token_budget);
            s->h_wstaging = s->palloc<float>(s->cfg.token_budget);
            s->d_wt = s->dalloc<float>(s->cfg.token_budget);
        }
        if ((uint64_t)K * V)
            CK(cudaMemcpy(m->d_nkw, n_kw, (uint64_t)K * V * 4, cudaMemcpyHostToDevice));
        CK(cudaMemcpy(m->d_nk, n_k, K * 4, cudaMemcpyHostToDevice));
        CK(cudaMemcpy(m->d_alpha, alpha, K * sizeof(float), cudaMemcpyHostToDevice));
        CK(cudaMemcpy(m->d_acum, acum.data(), K * sizeof(float), cudaMemcpyHostToDevice));
    } catch (const OomError&) {
        return TMT_ERR_OUT_OF_MEMORY;
    } catch (...) {
        return TMT_ERR_CUDA;
    }
    *model_id = (uint32_t)s->models.size();
    s->models.push_back(std::move(m));
    return TMT_OK;
}

// a request from host arrays: sorted by word id, the weights following their
// tokens; every token of one word must carry the same weight
tmt_status make_request(tmt_server* s, const uint32_t* wid, const float* wts, uint64_t len, uint32_t iters,
                        uint64_t seed, uint64_t key, Request& r)
{
    if (len > s->cfg.max_doc_len || (len && !wid)) return TMT_ERR_INVALID_ARGUMENT;
    if (wts) {
        std::vector<std::pair<uint32_t, float>> pw(len);
        for (uint64_t i = 0; i < len; ++i) {
            if (!(wts[i] >= 0.f) || !(wts[i] <= 65536.f)) return TMT_ERR_INVALID_ARGUMENT;
            pw[i] = { wid[i], wts[i] };
        }
        std::stable_sort(pw.begin(), pw.end(), [](const auto& x, const auto& y) { return x.first < y.first; });
        r.words.resize(len);
        r.wts.resize(len);
        for (uint64_t i = 0; i < len; ++i) {
            r.words[i] = pw[i].first;
            r.wts[i] = pw[i].second;
            if (i && r.words[i] == r.words[i - 1] && r.wts[i] != r.wts[i - 1]) return TMT_ERR_INVALID_ARGUMENT;
        }
    } else {
        r.words.assign(wid, wid + len);
        std::stable_sort(r.words.begin(), r.words.end());
    }
    r.iters = iters;
    r.seed = seed;
    r.key = key;
    return TMT_OK;
}

// queue requests (under the lock): each model must match its requests' kind
tmt_status enqueue(tmt_server* s, std::vector<Request>& rs, const uint32_t* model_ids, uint64_t* request_ids)
{
    const auto now = Clock::now();
    {
        std::lock_guard<std::mutex> lk(s->mu);
        if (s->stop) return s->worker_status != TMT_OK ? s->worker_status : TMT_ERR_CANCELLED;
        for (uint64_t d = 0; d < rs.size(); ++d) {
            if (model_ids[d] >= s->models.size()) return TMT_ERR_INVALID_ARGUMENT;
            if (s->models[model_ids[d]]->weighted != !rs[d].wts.empty() && !rs[d].words.empty())
                return TMT_ERR_INVALID_ARGUMENT;
        }
        for (uint64_t d = 0; d < rs.size(); ++d) {
            Request& r = rs[d];
            r.model = model_ids[d];
            if (s->models[r.model]->weighted && r.wts.size() != r.words.size()) r.wts.assign(r.words.size(), 0.f);
            s->models[r.model]->used = true;
            r.id = s->next_id++;
            r.t_submit = now;
            request_ids[d] = r.id;
            s->queue.push_back(std::move(r));
        }
    }
    s->cv_work.notify_one();
    return TMT_OK;
}

} // namespace

extern "C" {

tmt_status tmt_server_add_model(tmt_server* s, uint32_t K, uint32_t V, const float* alpha, float eta,
                                const int32_t* n_kw, const int32_t* n_k, uint32_t* model_id)
{
    return add_model_impl(s, K, V, alpha, eta, n_kw, n_k, false, model_id);
}

tmt_status tmt_server_add_model_f32(tmt_server* s, uint32_t K, uint32_t V, const float* alpha, float eta,
                                    const float* n_kw, const float* n_k, uint32_t* model_id)
{
    return add_model_impl(s, K, V, alpha, eta, n_kw, n_k, true, model_id);
}

tmt_status tmt_server_set_model_priors(tmt_server* s, uint32_t model_id, uint32_t P, const uint32_t* word_ids,
                                       const float* priors)
{
    if (!s || (P && (!word_ids || !priors))) return TMT_ERR_INVALID_ARGUMENT;
    std::lock_guard<std::mutex> lk(s->mu);
    if (model_id >= s->models.size()) return TMT_ERR_INVALID_ARGUMENT;
    Model* m = s->models[model_id].get();
    if (m->used) return TMT_ERR_STATE;           // only before the model's first request
    const uint32_t K = m->K, V = m->V;
    std::vector<uint8_t> seen(V, 0);
    for (uint32_t p = 0; p < P; ++p) {
        if (word_ids[p] >= V || seen[word_ids[p]]++) return TMT_ERR_INVALID_ARGUMENT;
        for (uint32_t k = 0; k < K; ++k)
            if (!(priors[(uint64_t)p * K + k] >= 0.f) || !std::isfinite(priors[(uint64_t)p * K + k]))
                return TMT_ERR_INVALID_ARGUMENT;
    }
    if (P == 0) {
        m->d_pidx = nullptr;
        m->d_pval = m->d_esum = m->d_pcum = m->d_ecum = nullptr;
        return TMT_OK;
    }
    try {
        CK(cudaSetDevice(s->device));
        std::vector<uint32_t> ids(word_ids, word_ids + P);
        std::vector<float> vals(priors, priors + (uint64_t)P * K);
        PriorTables t;
        build_prior_tables(K, V, m->eta, ids, vals, t);
        m->d_pidx = s->dalloc<int32_t>(V);
        m->d_pval = s->dalloc<float>((uint64_t)P * K);
        m->d_esum = s->dalloc<float>(K);
        m->d_pcum = s->dalloc<float>((uint64_t)P * K);
        m->d_ecum = s->dalloc<float>(K);
        CK(cudaMemcpy(m->d_pidx, t.idx.data(), V * sizeof(int32_t), cudaMemcpyHostToDevice));
        CK(cudaMemcpy(m->d_pval, vals.data(), (uint64_t)P * K * sizeof(float), cudaMemcpyHostToDevice));
        CK(cudaMemcpy(m->d_esum, t.esum.data(), K * sizeof(float), cudaMemcpyHostToDevice));
        CK(cudaMemcpy(m->d_pcum, t.pcum.data(), (uint64_t)P * K * sizeof(float), cudaMemcpyHostToDevice));
        CK(cudaMemcpy(m->d_ecum, t.ecum.data(), K * sizeof(float), cudaMemcpyHostToDevice));
    } catch (const OomError&) {
        return TMT_ERR_OUT_OF_MEMORY;
    } catch (...) {
        return TMT_ERR_CUDA;
    }
    return TMT_OK;
}

tmt_status tmt_server_submit(tmt_server* s, uint32_t model_id, const uint32_t* wid, uint32_t len, uint32_t iters,
                             uint64_t seed, uint64_t key, uint64_t* request_id)
{
    if (!s || (len && !wid) || !request_id) return TMT_ERR_INVALID_ARGUMENT;
    std::vector<Request> rs(1);
    tmt_status st = make_request(s, wid, nullptr, len, iters, seed, key, rs[0]);
    if (st != TMT_OK) return st;
    return enqueue(s, rs, &model_id, request_id);
}

tmt_status tmt_server_submit_weighted(tmt_server* s, uint32_t model_id, const uint32_t* wid, const float* weights,
                                      uint32_t len, uint32_t iters, uint64_t seed, uint64_t key, uint64_t* request_id)
{
    if (!s || (len && (!wid || !weights)) || !request_id) return TMT_ERR_INVALID_ARGUMENT;
    std::vector<Request> rs(1);
    tmt_status st = make_request(s, wid, weights, len, iters, seed, key, rs[0]);
    if (st != TMT_OK) return st;
    return enqueue(s, rs, &model_id, request_id);
}

tmt_status tmt_server_poll(tmt_server* s, uint32_t wait_ms, uint64_t* request_id, uint32_t* model_id,
                           float* theta, uint32_t theta_cap, double* ll, double* latency_ms)
{
    if (!s || !request_id) return TMT_ERR_INVALID_ARGUMENT;
    std::unique_lock<std::mutex> lk(s->mu);
    s->cv_done.wait_for(lk, std::chrono::milliseconds(wait_ms), [&] { return !s->results.empty() || s->stop; });
    if (s->results.empty()) {
        if (s->worker_status != TMT_OK) return s->worker_status;
        return TMT_ERR_TIMEOUT;
    }
    if (theta && theta_cap < s->results.front().theta.size()) return TMT_ERR_INVALID_ARGUMENT;   // kept queued
    Result r = std::move(s->results.front());
    s->results.pop_front();
    lk.unlock();
    *request_id = r.id;
    if (model_id) *model_id = r.model;
    if (theta) std::memcpy(theta, r.theta.data(), r.theta.size() * sizeof(float));
    if (ll) *ll = r.ll;
    if (latency_ms) *latency_ms = r.latency_ms;
    return TMT_OK;
}

tmt_status tmt_server_submit_batch(tmt_server* s, const uint32_t* model_ids, const uint32_t* wid,
                                   const uint64_t* doc_off, uint64_t n, uint32_t iters, uint64_t seed,
                                   const uint64_t* keys, uint64_t* request_ids)
{
    return tmt_server_submit_batch_weighted(s, model_ids, wid, nullptr, doc_off, n, iters, seed, keys, request_ids);
}

tmt_status tmt_server_submit_batch_weighted(tmt_server* s, const uint32_t* model_ids, const uint32_t* wid,
                                            const float* weights, const uint64_t* doc_off, uint64_t n, uint32_t iters,
                                            uint64_t seed, const uint64_t* keys, uint64_t* request_ids)
{
    if (!s || (n && (!model_ids || !doc_off || !request_ids))) return TMT_ERR_INVALID_ARGUMENT;
    std::vector<Request> rs(n);
    for (uint64_t d = 0; d < n; ++d) {
        if (doc_off[d + 1] < doc_off[d]) return TMT_ERR_INVALID_ARGUMENT;
        const uint64_t len = doc_off[d + 1] - doc_off[d];
        if (len && weights == nullptr && !wid) return TMT_ERR_INVALID_ARGUMENT;
        tmt_status st = make_request(s, wid ? wid + doc_off[d] : nullptr, weights ? weights + doc_off[d] : nullptr,
                                     len, iters, seed, keys ? keys[d] : 0, rs[d]);
        if (st != TMT_OK) return st;
    }
    return enqueue(s, rs, model_ids, request_ids);
}

tmt_status tmt_server_poll_batch(tmt_server* s, uint32_t wait_ms, uint64_t max_n, uint64_t* request_ids,
                                 uint32_t* model_ids, float* theta, uint32_t theta_stride, double* ll,
                                 double* latency_ms, uint64_t* n_out)
{
    if (!s || !request_ids || !n_out || max_n == 0) return TMT_ERR_INVALID_ARGUMENT;
    *n_out = 0;
    std::unique_lock<std::mutex> lk(s->mu);
    s->cv_done.wait_for(lk, std::chrono::milliseconds(wait_ms), [&] { return !s->results.empty() || s->stop; });
    if (s->results.empty()) {
        if (s->worker_status != TMT_OK) return s->worker_status;
        return TMT_ERR_TIMEOUT;
    }
    uint64_t n = 0;
    while (n < max_n && !s->results.empty()) {
        const Result& r = s->results.front();
        if (theta && theta_stride < r.theta.size()) {
            if (n == 0) return TMT_ERR_INVALID_ARGUMENT;   // kept queued
            break;
        }
        request_ids[n] = r.id;
        if (model_ids) model_ids[n] = r.model;
        if (theta) std::memcpy(theta + n * theta_stride, r.theta.data(), r.theta.size() * sizeof(float));
        if (ll) ll[n] = r.ll;
        if (latency_ms) latency_ms[n] = r.latency_ms;
        s->results.pop_front();
        ++n;
    }
    *n_out = n;
    return TMT_OK;
}

tmt_status tmt_server_get_stats(tmt_server* s, tmt_server_stats* out)
{
    if (!s || !out) return TMT_ERR_INVALID_ARGUMENT;
    std::lock_guard<std::mutex> lk(s->mu);
    out->steps = s->steps;
    out->completed = s->completed;
    out->queued = s->queue.size();
    out->mean_active = s->steps ? (double)s->active_sum / (double)s->steps : 0.0;
    out->tokens_in_flight_max = s->tokens_in_flight_max;
    out->token_sweeps = s->token_sweeps;
    out->alg_bytes = s->alg_bytes;
    out->kernel_ms = s->kernel_ms;
    out->busy_ms = s->busy_ms;
    return TMT_OK;
}

const char* tmt_server_last_error(const tmt_server* s)
{
    return s ? s->err.c_str() : "null server";
}

tmt_status tmt_server_stop(tmt_server* s)
{
    if (!s) return TMT_ERR_INVALID_ARGUMENT;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->stop = true;
    }
    s->cv_work.notify_all();
    s->cv_done.notify_all();
    if (s->worker.joinable()) s->worker.join();
    const tmt_status st = s->worker_status;
    delete s;
    return st;
}

} // extern "C"
