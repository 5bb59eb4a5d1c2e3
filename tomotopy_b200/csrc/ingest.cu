// ingest.cu -- corpus preparation on the device: tomotopy's removeStopwords
// (TopicModel.hpp:526-571) and prepareDoc (LDAModel.hpp:716-722) for an
// integer-id corpus, with the same outputs as the host tmt_prepare_corpus.
//
//   1. each document's tokens sorted by (old id, position) in shared memory
//      (bitonic sort of 64-bit keys, documents bucketed by length so a block's
//      shared memory fits its documents); cf counts every token, df every run
//      start of a sorted document;
//   2. the vocabulary order from (cf, df) on the host (tmt_prepare_corpus_counted
//      with no documents: the same stable sort, thresholds and rm_top rotation);
//   3. each document re-sorted by (new id, original position): a stable sort
//      by the new ids, as sortAndWriteOrder does (Utils.hpp:227-248); w_order
//      maps every original position to its sorted position.
#include <cuda_runtime.h>
#include <algorithm>
#include <cstdint>
#include <cstring>
#include <stdexcept>
#include <string>
#include <vector>
#include "../../include/tomotopy_b200.h"

namespace {

constexpr uint32_t kMaxSortDoc = 16384;     // tokens per document sorted on chip

struct IngestError : std::runtime_error { using std::runtime_error::runtime_error; };

#define ICK(x)                                                                                   \
    do {                                                                                         \
        cudaError_t e_ = (x);                                                                    \
        if (e_ != cudaSuccess) throw IngestError(std::string(#x) + ": " + cudaGetErrorString(e_)); \
    } while (0)

// One block per listed document (all of length <= npow): keys sorted in
// shared memory, ascending.  pass 0: key = (old id << 32) | position; writes
// the sorted old ids and original positions, counts cf and df.  pass 1: key =
// (new id << 32) | original position; writes the new ids and w_order.
__global__ void k_doc_sort(const uint64_t* __restrict__ doc_off, const uint32_t* __restrict__ docs, uint32_t npow,
                           int pass, const uint32_t* __restrict__ words, const uint32_t* __restrict__ pos_in,
                           const uint32_t* __restrict__ order, uint32_t* __restrict__ words_out,
                           uint32_t* __restrict__ pos_out, unsigned long long* __restrict__ cf,
                           unsigned long long* __restrict__ df)
{
    extern __shared__ unsigned long long s_key[];
    const uint64_t d = docs[blockIdx.x];
    const uint64_t b = doc_off[d];
    const uint32_t n = (uint32_t)(doc_off[d + 1] - b);
    for (uint32_t i = threadIdx.x; i < npow; i += blockDim.x) {
        unsigned long long key = ~0ull;
        if (i < n) {
            if (pass == 0) key = ((unsigned long long)words[b + i] << 32) | i;
            else key = ((unsigned long long)order[words[b + i]] << 32) | pos_in[b + i];
        }
        s_key[i] = key;
    }
    __syncthreads();
    for (uint32_t k = 2; k <= npow; k <<= 1) {
        for (uint32_t j = k >> 1; j > 0; j >>= 1) {
            for (uint32_t i = threadIdx.x; i < npow; i += blockDim.x) {
                const uint32_t ixj = i ^ j;
                if (ixj > i) {
                    const unsigned long long x = s_key[i], y = s_key[ixj];
                    const bool up = (i & k) == 0;
                    if ((x > y) == up) {
                        s_key[i] = y;
                        s_key[ixj] = x;
                    }
                }
            }
            __syncthreads();
        }
    }
    for (uint32_t i = threadIdx.x; i < n; i += blockDim.x) {
        const unsigned long long key = s_key[i];
        const uint32_t w = (uint32_t)(key >> 32), p = (uint32_t)key;
        words_out[b + i] = w;
        if (pass == 0) {
            pos_out[b + i] = p;
            atomicAdd(cf + w, 1ull);
            if (i == 0 || (uint32_t)(s_key[i - 1] >> 32) != w) atomicAdd(df + w, 1ull);
        } else {
            pos_out[b + p] = i;
        }
    }
}

void sort_docs(const std::vector<std::vector<uint32_t>>& buckets, uint32_t* d_docs, const uint64_t* d_off, int pass,
               const uint32_t* words, const uint32_t* pos_in, const uint32_t* order, uint32_t* words_out,
               uint32_t* pos_out, unsigned long long* cf, unsigned long long* df, cudaStream_t st)
{
    uint64_t at = 0;
    for (size_t c = 0; c < buckets.size(); ++c) {
        const auto& list = buckets[c];
        if (list.empty()) continue;
        const uint32_t npow = 32u << c;
        const uint32_t threads = std::min<uint32_t>(512, std::max<uint32_t>(32, npow / 2));
        const size_t smem = (size_t)npow * 8;
        ICK(cudaFuncSetAttribute(k_doc_sort, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)(kMaxSortDoc * 8)));
        for (size_t o = 0; o < list.size(); o += 0x7FFFFFFF) {
            const uint32_t cnt = (uint32_t)std::min<size_t>(list.size() - o, 0x7FFFFFFF);
            k_doc_sort<<<cnt, threads, smem, st>>>(d_off, d_docs + at + o, npow, pass, words, pos_in, order,
                                                   words_out, pos_out, cf, df);
            ICK(cudaGetLastError());
        }
        at += list.size();
    }
}

template <class T>
T* dmalloc(std::vector<void*>& owned, size_t count)
{
    void* p = nullptr;
    ICK(cudaMalloc(&p, std::max<size_t>(count, 1) * sizeof(T)));
    owned.push_back(p);
    return static_cast<T*>(p);
}

void set_err(char* err, uint64_t err_len, const std::string& m)
{
    if (!err || !err_len) return;
    const size_t n = std::min<size_t>(m.size(), err_len - 1);
    std::memcpy(err, m.data(), n);
    err[n] = '\0';
}

} // namespace

extern "C" tmt_status tmt_prepare_corpus_device(int32_t device, uint64_t D, const uint64_t* doc_off,
                                                const uint32_t* words, uint32_t n_vocab, uint64_t min_cf,
                                                uint64_t min_df, uint64_t rm_top, uint32_t* words_out,
                                                uint32_t* w_order, uint32_t* vocab_order, uint64_t* vocab_cf,
                                                uint64_t* vocab_df, uint32_t* real_v, char* err, uint64_t err_len)
{
    set_err(err, err_len, "");
    if (!doc_off || (doc_off[D] && (!words || !words_out)) || !vocab_order || !real_v) {
        set_err(err, err_len, "NULL argument");
        return TMT_ERR_INVALID_ARGUMENT;
    }
    const uint64_t N = doc_off[D];
    // the host checks: offsets, ids, document lengths
    std::vector<std::vector<uint32_t>> buckets(10);     // npow = 32 << c, up to 16384
    for (uint64_t d = 0; d < D; ++d) {
        if (doc_off[d + 1] < doc_off[d]) {
            set_err(err, err_len, "doc_off is not non-decreasing");
            return TMT_ERR_INVALID_ARGUMENT;
        }
        const uint64_t n = doc_off[d + 1] - doc_off[d];
        if (n > kMaxSortDoc) {
            set_err(err, err_len, "document " + std::to_string(d) + " has " + std::to_string(n) +
                                      " tokens; the device preparation sorts at most 16384 per document "
                                      "(use tmt_prepare_corpus)");
            return TMT_ERR_INVALID_ARGUMENT;
        }
        if (n == 0) continue;
        uint32_t c = 0;
        while ((32ull << c) < n) ++c;
        buckets[c].push_back((uint32_t)d);
    }
    if (D > 0xFFFFFFFFull) {
        set_err(err, err_len, "too many documents");
        return TMT_ERR_INVALID_ARGUMENT;
    }
    for (uint64_t i = 0; i < N; ++i)
        if (words[i] >= n_vocab) {
            set_err(err, err_len, "word id >= n_vocab at token " + std::to_string(i));
            return TMT_ERR_INVALID_ARGUMENT;
        }
    std::vector<void*> owned;
    cudaStream_t st = nullptr;
    tmt_status status = TMT_OK;
    try {
        ICK(cudaSetDevice(device));
        ICK(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
        uint64_t* d_off = dmalloc<uint64_t>(owned, D + 1);
        uint32_t* d_words = dmalloc<uint32_t>(owned, N);
        uint32_t* d_sorted = dmalloc<uint32_t>(owned, N);
        uint32_t* d_pos = dmalloc<uint32_t>(owned, N);
        uint32_t* d_docs = dmalloc<uint32_t>(owned, D);
        uint32_t* d_order = dmalloc<uint32_t>(owned, n_vocab);
        unsigned long long* d_cf = dmalloc<unsigned long long>(owned, n_vocab);
        unsigned long long* d_df = dmalloc<unsigned long long>(owned, n_vocab);
        std::vector<uint32_t> all;
        all.reserve(D);
        for (auto& l : buckets) all.insert(all.end(), l.begin(), l.end());
        ICK(cudaMemcpyAsync(d_off, doc_off, (D + 1) * sizeof(uint64_t), cudaMemcpyHostToDevice, st));
        if (N) ICK(cudaMemcpyAsync(d_words, words, N * sizeof(uint32_t), cudaMemcpyHostToDevice, st));
        if (!all.empty()) ICK(cudaMemcpyAsync(d_docs, all.data(), all.size() * sizeof(uint32_t), cudaMemcpyHostToDevice, st));
        ICK(cudaMemsetAsync(d_cf, 0, (size_t)n_vocab * 8, st));
        ICK(cudaMemsetAsync(d_df, 0, (size_t)n_vocab * 8, st));
        // 1. sort by old id; cf, df
        sort_docs(buckets, d_docs, d_off, 0, d_words, nullptr, nullptr, d_sorted, d_pos, d_cf, d_df, st);
        std::vector<uint64_t> cf(n_vocab), df(n_vocab);
        if (n_vocab) {
            ICK(cudaMemcpyAsync(cf.data(), d_cf, (size_t)n_vocab * 8, cudaMemcpyDeviceToHost, st));
            ICK(cudaMemcpyAsync(df.data(), d_df, (size_t)n_vocab * 8, cudaMemcpyDeviceToHost, st));
        }
        ICK(cudaStreamSynchronize(st));
        // 2. the vocabulary order (the host rule, no documents)
        const uint64_t zero = 0;
        tmt_status s2 = tmt_prepare_corpus_counted(0, &zero, nullptr, n_vocab, cf.data(), df.data(), min_cf, min_df,
                                                   rm_top, nullptr, nullptr, vocab_order, real_v);
        if (s2 != TMT_OK) throw IngestError("vocabulary order failed");
        for (uint32_t w = 0; w < n_vocab; ++w) {
            if (vocab_cf) vocab_cf[vocab_order[w]] = cf[w];
            if (vocab_df) vocab_df[vocab_order[w]] = df[w];
        }
        // 3. re-sort by new id, stable in the original position
        if (n_vocab) ICK(cudaMemcpyAsync(d_order, vocab_order, (size_t)n_vocab * 4, cudaMemcpyHostToDevice, st));
        sort_docs(buckets, d_docs, d_off, 1, d_sorted, d_pos, d_order, d_words, d_pos, nullptr, nullptr, st);
        if (N) {
            ICK(cudaMemcpyAsync(words_out, d_words, N * sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
            if (w_order) ICK(cudaMemcpyAsync(w_order, d_pos, N * sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
        }
        ICK(cudaStreamSynchronize(st));
    } catch (const IngestError& e) {
        set_err(err, err_len, e.what());
        cudaGetLastError();
        status = TMT_ERR_CUDA;
    } catch (const std::bad_alloc&) {
        set_err(err, err_len, "host allocation failed");
        status = TMT_ERR_OUT_OF_MEMORY;
    }
    if (st) cudaStreamSynchronize(st);
    for (void* p : owned) cudaFree(p);
    if (st) cudaStreamDestroy(st);
    return status;
}
