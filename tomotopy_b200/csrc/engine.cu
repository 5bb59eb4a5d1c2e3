// engine.cu -- B200 collapsed-Gibbs LDA engine behind the C ABI in
// include/tomotopy_b200.h.
//
// Sampler semantics (one sweep = tomotopy's trainOne, LDAModel.hpp:505-539):
// tomotopy's COPY_MERGE scheme (LDAModel.hpp:401-423, 555-570) with one worker
// per document.  A warp owns a document and samples its tokens in order, its
// n_dk row live in shared memory, exactly as sampleDocument does
// (LDAModel.hpp:326-354).  n_kw and n_k are read from the start-of-sweep copy
// with the token's own assignment removed; count deltas go to the next copy
// with integer atomics (the merge, :555-570).  Each draw is Philox4x32-10 of
// (doc-major token index, global step), so z depends only on the seed and the
// start-of-sweep state: results are bit-identical for any scheduling.
//
// Conditional per topic k (getZLikelihoods, LDAModel.hpp:273-285):
//   w_k = A_k * phi_k,  A_k = (float)n_dk[k] + alpha_k,  phi_k = ((float)n_kw[k,v] + eta) * R_k,
//   R_k = 1 / ((float)n_k[k] + V*eta)  (phi: the group's per-word table);
//   the token's own topic zo: phi_own = ((float)(n_kw[zo,v] - 1) + eta) * (1 / ((float)(n_k[zo] - 1) + V*eta))
// each operation rounded to nearest (no contraction).  Topics are dealt to
// the 32 lanes in blocks of four (lane l owns k = 128 j + 4 l + i).  Pass 1:
// each lane's fma chain over its topics with the own topic left out, the
// owning lane then adding A_zo * phi_own; a Hillis-Steele scan over the lane
// totals.  Pass 2: the prefix sums of the hit lane's topics.  The draw is
// the first k (in that order) with u*total < cum[k], else the hit lane's
// last topic, or K-1 when no lane is hit (sampleFromDiscreteAcc,
// sample.hpp:133-189).
#include <cuda_runtime.h>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <cmath>
#include <string>
#include <vector>
#include <numeric>
#include <algorithm>
#include <stdexcept>
#include <mutex>
#include <thread>
#include "philox.cuh"
#include "special.cuh"
#include "common.cuh"
#include "infer.cuh"
#include "priors.h"
#include "../../include/tomotopy_b200.h"

namespace {

using namespace tmtk;
constexpr int kSweepWarps = 8;           // warps per sweep block
// The 16-bit-row kernels (variant 2): 5 warps a block, 5 blocks/SM.  At 8
// warps x 4 blocks the token loop gets 64 registers and spills (spilled
// registers come back from L2: the resident warps' columns keep L1 from
// holding them); smaller blocks also leave L1 more of the SM's 256 KB.
// Measured at k = 1000 (ms per sweep): 8 x 4 101.1 (before alpha moved to
// shared memory; 101.9 after, spilling), 7 x 4 97.6, 6 x 4 92.4,
// 5 x 4 94.7, 4 x 6 92.7, 4 x 7 97.1, 3 x 8 98.0, 5 x 5 91.4.
constexpr int kRow16Warps = 5;
constexpr int kRow16MinB = 5;

// One Hillis-Steele step with the lane test folded into an fma: m is 1 for
// lanes at or above `off`, else 0, and for the finite sums here fma(y, 1, x)
// rounds exactly as x + y and fma(y, 0, x) is x -- the values of the usual
// predicated add, in fewer instructions.
__device__ __forceinline__ float hs_step(float x, int off, float m)
{
    return __fmaf_rn(__shfl_up_sync(FULL, x, off), m, x);
}

// Long documents: a document of at least split_len tokens (all ids counted)
// is sampled by a whole block as kSweepWarps slices side by side, merging
// their n_dk changes every split_step positions (k_sweep_doc, phase 1).  A
// token then sees up to (kSweepWarps - 1) * split_step of its document's
// other tokens as of the step's start.  The threshold of a document group is
// max(8 * (kSweepWarps - 1) * split_step, ceil(tokens / 4096)): documents
// longer than the group's work per warp of a 4096-warp machine, and at least
// 8 stale windows long (at 16 positions per step: 896 tokens; splitting from
// 421 tokens measured 0.49% lower ll_per_word at the k=100 configuration
// after 500 sweeps, from 842 tokens 0.03%).  It depends on the corpus only,
// never on the device or on timing; integer counts with K <= kSplitMaxK (the
// kernels with phase 1 are built for up to 4 blocks of four topics per lane).
// tmt_set_doc_split overrides the threshold and the step.
constexpr uint32_t kSplitStep = 16;
constexpr uint32_t kSplitMaxK = 512;

uint64_t split_len_of(uint64_t group_tokens, uint32_t K, uint64_t min_len, uint32_t step)
{
    if (K > kSplitMaxK || min_len >= 0xFFFFFFFFull) return 0;
    if (min_len) return min_len;
    return std::max<uint64_t>(8ull * (kSweepWarps - 1) * step, (group_tokens + 4095) / 4096);
}


// ---------------------------------------------------------------------------
// word priors (set_word_prior: etaByTopicWord, LDAModel.hpp:99-117, 724-737)
// ---------------------------------------------------------------------------
// eta is per (topic, word) only for the words given a prior: idx[v] >= 0 names
// row idx[v] of val (K floats); every other word keeps the scalar eta.  esum[k]
// replaces V*eta in the denominators.  All NULL: no priors.
struct PriorArgs {
    const int32_t* idx;
    const float* val;
    const float* esum;
};

__device__ __forceinline__ const float* prior_col(const PriorArgs& pr, uint64_t v, uint32_t K)
{
    if (!pr.idx) return nullptr;
    const int p = __ldg(pr.idx + v);
    return p >= 0 ? pr.val + (uint64_t)p * K : nullptr;
}

__device__ __forceinline__ float esum_of(const PriorArgs& pr, uint32_t k, float veta)
{
    return pr.esum ? __ldg(pr.esum + k) : veta;
}

// ---------------------------------------------------------------------------
// initialisation: z0 ~ Discrete(alpha) (initializeDocState, LDAModel.hpp:781-813)
// ---------------------------------------------------------------------------
// With word priors (pidx != NULL) every token draws from its word's eta column
// instead (updateStateWithDoc, LDAModel.hpp:765-779): pcum holds the sequential
// float cumulative sums of the prior rows, ecum that of a column of eta.
__global__ void k_init_z(const uint32_t* __restrict__ words, uint64_t n_all, uint32_t V, uint32_t K,
                         const float* __restrict__ acum, uint64_t seed, uint64_t tok_offset,
                         uint16_t* __restrict__ z, const int32_t* __restrict__ pidx,
                         const float* __restrict__ pcum, const float* __restrict__ ecum)
{
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n_all;
         i += (uint64_t)gridDim.x * blockDim.x) {
        if (words[i] >= V) { z[i] = 0xFFFF; continue; }
        const uint64_t gi = i + tok_offset;      // the token's index in the whole (unsharded) corpus
        float u = tmt::u01(tmt::philox_u32((uint32_t)gi, (uint32_t)(gi >> 32), tmt::kStreamInit, 0, seed));
        if (pidx) {
            const int p = pidx[words[i]];
            acum = p >= 0 ? pcum + (uint64_t)p * K : ecum;
        }
        float r = __fmul_rn(u, acum[K - 1]);
        uint32_t lo = 0, hi = K - 1;
        while (lo < hi) {
            uint32_t mid = (lo + hi) >> 1;
            if (r < acum[mid]) hi = mid; else lo = mid + 1;
        }
        z[i] = (uint16_t)lo;
    }
}

// counts from assignments: warp per document (resetStatistics, LDAModel.hpp:301-316).
// With nk_smem the block sums n_k in shared memory (K ints) and adds its
// nonzero totals once at the end: n_k's K addresses would otherwise take one
// global atomic per token.
__global__ void k_counts(const uint64_t* __restrict__ doc_off, const uint32_t* __restrict__ words,
                         const uint16_t* __restrict__ z, uint64_t D, uint32_t K, uint32_t V,
                         int32_t* __restrict__ ndk, int32_t* __restrict__ nkw, int32_t* __restrict__ nk,
                         int32_t* __restrict__ doc_len, bool nk_smem)
{
    extern __shared__ int32_t s_nk[];
    if (nk_smem) {
        for (uint32_t k = threadIdx.x; k < K; k += blockDim.x) s_nk[k] = 0;
        __syncthreads();
    }
    const int lane = threadIdx.x & 31;
    const uint64_t warp = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
    const uint64_t nwarps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
    for (uint64_t d = warp; d < D; d += nwarps) {
        int cnt = 0;
        for (uint64_t i = doc_off[d] + lane; i < doc_off[d + 1]; i += 32) {
            uint32_t w = words[i];
            if (w >= V) continue;
            uint32_t k = z[i];
            atomicAdd(&ndk[d * K + k], 1);
            atomicAdd(&nkw[(uint64_t)w * K + k], 1);
            if (nk_smem) atomicAdd(&s_nk[k], 1);
            else atomicAdd(&nk[k], 1);
            ++cnt;
        }
#pragma unroll
        for (int o = 16; o; o >>= 1) cnt += __shfl_xor_sync(FULL, cnt, o);
        if (lane == 0 && doc_len) doc_len[d] = cnt;
    }
    if (nk_smem) {
        __syncthreads();
        for (uint32_t k = threadIdx.x; k < K; k += blockDim.x)
            if (s_nk[k]) atomicAdd(&nk[k], s_nk[k]);
    }
}

// n_dk and the valid-token counts per row from z: document d's tokens go to
// row row_of[d] (PT's pseudo-documents), or to row d when row_of is NULL.
// ndk and len must be zero on entry.
__global__ void k_counts_rows(const uint64_t* __restrict__ doc_off, const uint32_t* __restrict__ words,
                              const uint16_t* __restrict__ z, uint64_t D, uint32_t K, uint32_t V,
                              const uint32_t* __restrict__ row_of, int32_t* __restrict__ ndk,
                              int32_t* __restrict__ len)
{
    const int lane = threadIdx.x & 31;
    const uint64_t warp = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
    const uint64_t nwarps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
    for (uint64_t d = warp; d < D; d += nwarps) {
        const uint64_t r = row_of ? row_of[d] : d;
        int cnt = 0;
        for (uint64_t i = doc_off[d] + lane; i < doc_off[d + 1]; i += 32) {
            if (words[i] >= V) continue;
            atomicAdd(&ndk[r * K + z[i]], 1);
            ++cnt;
        }
#pragma unroll
        for (int o = 16; o; o >>= 1) cnt += __shfl_xor_sync(FULL, cnt, o);
        if (lane == 0 && cnt) atomicAdd(&len[r], cnt);
    }
}

// ---------------------------------------------------------------------------
// the training sweep
// ---------------------------------------------------------------------------
// Per-sweep word table: phi[v*KP + k] = ((float)n_kw[k,v] + eta) * R_k with
// R_k = 1 / ((float)n_k[k] + V*eta) and KP = K rounded up to a multiple of
// 4 (entries K..KP-1 are 0); the same pass copies n_kw and n_k into the
// next state, which the sweep then updates with the count deltas.
__global__ void k_phi_copy(const int32_t* __restrict__ nkw, const int32_t* __restrict__ nk, uint32_t V, uint32_t K,
                           uint32_t KP, float eta, float veta, float* __restrict__ phi, int32_t* __restrict__ nkw_next,
                           int32_t* __restrict__ nk_next, uint32_t smem_k, PriorArgs pr, float* __restrict__ rm1)
{
    extern __shared__ __align__(16) float s_R[];
    const bool r_smem = K <= smem_k;
    if (r_smem)
        for (uint32_t k = threadIdx.x; k < K; k += blockDim.x)
            s_R[k] = __fdiv_rn(1.0f, __fadd_rn((float)nk[k], esum_of(pr, k, veta)));
    if (blockIdx.x == 0)
        for (uint32_t k = threadIdx.x; k < K; k += blockDim.x) {
            nk_next[k] = nk[k];
            rm1[k] = __fdiv_rn(1.0f, __fadd_rn((float)(nk[k] - 1), esum_of(pr, k, veta)));
        }
    __syncthreads();
    if (r_smem && (K & 3) == 0 && !pr.idx) {
        // K a multiple of 4 (KP == K) and no word priors: 16-byte loads and
        // stores, the same values
        const uint32_t K4 = K >> 2;
        for (uint64_t v = blockIdx.x; v < V; v += gridDim.x) {
            const int4* src = reinterpret_cast<const int4*>(nkw + v * K);
            int4* dst = reinterpret_cast<int4*>(nkw_next + v * K);
            float4* ph = reinterpret_cast<float4*>(phi + v * KP);
            for (uint32_t k4 = threadIdx.x; k4 < K4; k4 += blockDim.x) {
                const int4 n = __ldg(src + k4);
                dst[k4] = n;
                const float4 R = reinterpret_cast<const float4*>(s_R)[k4];
                ph[k4] = make_float4(__fmul_rn(__fadd_rn((float)n.x, eta), R.x), __fmul_rn(__fadd_rn((float)n.y, eta), R.y),
                                     __fmul_rn(__fadd_rn((float)n.z, eta), R.z), __fmul_rn(__fadd_rn((float)n.w, eta), R.w));
            }
        }
        return;
    }
    for (uint64_t v = blockIdx.x; v < V; v += gridDim.x) {
        const int32_t* src = nkw + v * K;
        int32_t* dst = nkw_next + v * K;
        float* ph = phi + v * KP;
        const float* pe = prior_col(pr, v, K);
        for (uint32_t k = threadIdx.x; k < KP; k += blockDim.x) {
            float val = 0.f;
            if (k < K) {
                const int32_t n = src[k];
                dst[k] = n;
                const float R = r_smem ? s_R[k] : __fdiv_rn(1.0f, __fadd_rn((float)nk[k], esum_of(pr, k, veta)));
                val = __fmul_rn(__fadd_rn((float)n, pe ? pe[k] : eta), R);
            }
            ph[k] = val;
        }
    }
}

// Sharded corpus: fold the ranks' summed deltas of one group into the state.
// n_k first (one block), then n_kw and, when phi != NULL, the word table of
// the new state; the deltas are zeroed for the next group.
__global__ void k_nk_apply(int32_t* __restrict__ nk, int32_t* __restrict__ dnk, uint32_t K)
{
    for (uint32_t k = threadIdx.x; k < K; k += blockDim.x) {
        nk[k] += dnk[k];
        dnk[k] = 0;
    }
}

__global__ void k_phi_apply(int32_t* __restrict__ nkw, int32_t* __restrict__ delta, const int32_t* __restrict__ nk,
                            uint32_t V, uint32_t K, uint32_t KP, float eta, float veta, float* __restrict__ phi,
                            uint32_t smem_k, int fold, PriorArgs pr, float* __restrict__ rm1)
{
    extern __shared__ float s_R[];
    const bool r_smem = phi && K <= smem_k;
    if (r_smem)
        for (uint32_t k = threadIdx.x; k < K; k += blockDim.x)
            s_R[k] = __fdiv_rn(1.0f, __fadd_rn((float)nk[k], esum_of(pr, k, veta)));
    if (phi && rm1 && blockIdx.x == 0)
        for (uint32_t k = threadIdx.x; k < K; k += blockDim.x)
            rm1[k] = __fdiv_rn(1.0f, __fadd_rn((float)(nk[k] - 1), esum_of(pr, k, veta)));
    __syncthreads();
    for (uint64_t v = blockIdx.x; v < V; v += gridDim.x) {
        int32_t* col = nkw + v * K;
        int32_t* dcol = delta + v * K;
        float* ph = phi ? phi + v * KP : nullptr;
        const float* pe = ph ? prior_col(pr, v, K) : nullptr;
        for (uint32_t k = threadIdx.x; k < KP; k += blockDim.x) {
            float val = 0.f;
            if (k < K) {
                int32_t n = col[k];
                if (fold) {
                    n += dcol[k];
                    col[k] = n;
                    dcol[k] = 0;
                }
                if (ph) {
                    const float R = r_smem ? s_R[k] : __fdiv_rn(1.0f, __fadd_rn((float)nk[k], esum_of(pr, k, veta)));
                    val = __fmul_rn(__fadd_rn((float)n, pe ? pe[k] : eta), R);
                }
            }
            if (ph) ph[k] = val;
        }
    }
}

// ---------------------------------------------------------------------------
// weighted counts (TermWeight IDF / PMI)
// ---------------------------------------------------------------------------
// A token of weight w adds round(w * 2^24) to the integer deltas; a fold adds
// the deltas to the float state, n' = max(n + (float)q * 2^-24, 0), and zeroes
// them.  Integer deltas make the fold independent of the order of the adds.
__device__ __forceinline__ long long wq_of(float w)
{
    return __float2ll_rn(__fmul_rn(w, 16777216.f));
}

__device__ __forceinline__ float fold_w(float n, long long q)
{
    const float s = __fadd_rn(n, __fmul_rn(__ll2float_rn(q), 5.9604644775390625e-8f));
    return s > 0.f ? s : 0.f;
}

// n_k's fixed-point deltas of a group: the column sums of the word deltas
// (every token adds the same q to dkw[v][k] as to n_k's delta of k), summed
// as integers, so any order gives the same value.  Block (x, y): topics
// [256x, 256x + 256), word rows [y * rows, (y + 1) * rows).
__global__ void k_dk_sum(const long long* __restrict__ dkw, uint32_t V, uint32_t K, uint32_t rows,
                         long long* __restrict__ dk)
{
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= K) return;
    const uint64_t v0 = (uint64_t)blockIdx.y * rows;
    const uint64_t v1 = v0 + rows < (uint64_t)V ? v0 + rows : (uint64_t)V;
    unsigned long long sum = 0;
    for (uint64_t v = v0; v < v1; ++v) sum += (unsigned long long)__ldg(dkw + v * K + k);
    if (sum) atomicAdd(reinterpret_cast<unsigned long long*>(dk) + k, sum);
}

__global__ void k_nk_fold_w(float* __restrict__ nk, long long* __restrict__ dk, uint32_t K)
{
    for (uint32_t k = threadIdx.x; k < K; k += blockDim.x) {
        nk[k] = fold_w(nk[k], dk[k]);
        dk[k] = 0;
    }
}

// n_kw fold (fold != 0) and, when phi != NULL, the word table of the state
__global__ void k_phi_fold_w(float* __restrict__ nkw, long long* __restrict__ dkw, const float* __restrict__ nk,
                             uint32_t V, uint32_t K, uint32_t KP, float eta, float veta, float* __restrict__ phi,
                             uint32_t smem_k, int fold, PriorArgs pr)
{
    extern __shared__ float s_R[];
    const bool r_smem = phi && K <= smem_k;
    if (r_smem)
        for (uint32_t k = threadIdx.x; k < K; k += blockDim.x)
            s_R[k] = __fdiv_rn(1.0f, __fadd_rn(nk[k], esum_of(pr, k, veta)));
    __syncthreads();
    for (uint64_t v = blockIdx.x; v < V; v += gridDim.x) {
        float* col = nkw + v * K;
        long long* dcol = dkw + v * K;
        float* ph = phi ? phi + v * KP : nullptr;
        const float* pe = ph ? prior_col(pr, v, K) : nullptr;
        for (uint32_t k = threadIdx.x; k < KP; k += blockDim.x) {
            float val = 0.f;
            if (k < K) {
                float n = col[k];
                if (fold) {
                    n = fold_w(n, dcol[k]);
                    col[k] = n;
                    dcol[k] = 0;
                }
                if (ph) {
                    const float R = r_smem ? s_R[k] : __fdiv_rn(1.0f, __fadd_rn(nk[k], esum_of(pr, k, veta)));
                    val = __fmul_rn(__fadd_rn(n, pe ? pe[k] : eta), R);
                }
            }
            if (ph) ph[k] = val;
        }
    }
}

// Weighted counts from z, thread per document: n_dk and the document's weight
// sum accumulate in float in token order (addWordTo in initializeDocState and
// updateSumWordWeight, LDAModel.hpp:795-809, LDA.h:113-116); n_kw and n_k go
// to the integer deltas (folded afterwards).
__global__ void k_counts_w(const uint64_t* __restrict__ doc_off, const uint32_t* __restrict__ words,
                           const uint16_t* __restrict__ z, const float* __restrict__ wt, uint64_t D, uint32_t K,
                           uint32_t V, float* __restrict__ ndk, long long* __restrict__ dkw,
                           long long* __restrict__ dk, float* __restrict__ doc_wlen, bool dk_smem)
{
    // with dk_smem the block sums n_k's fixed-point deltas in shared memory
    // (integers: any order gives the same sums) and adds them once at the end
    extern __shared__ unsigned long long s_dk[];
    if (dk_smem) {
        for (uint32_t k = threadIdx.x; k < K; k += blockDim.x) s_dk[k] = 0;
        __syncthreads();
    }
    for (uint64_t d = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; d < D; d += (uint64_t)gridDim.x * blockDim.x) {
        float* row = ndk + d * K;
        float len = 0.f;
        for (uint64_t i = doc_off[d]; i < doc_off[d + 1]; ++i) {
            const uint32_t v = words[i];
            if (v >= V) continue;
            const float w = wt[i];
            const uint32_t k = z[i];
            row[k] = __fadd_rn(row[k], w);
            len = __fadd_rn(len, w);
            const unsigned long long q = (unsigned long long)wq_of(w);
            atomicAdd(reinterpret_cast<unsigned long long*>(dkw) + (uint64_t)v * K + k, q);
            if (dk_smem) atomicAdd(s_dk + k, q);
            else atomicAdd(reinterpret_cast<unsigned long long*>(dk) + k, q);
        }
        doc_wlen[d] = len;
    }
    if (dk_smem) {
        __syncthreads();
        for (uint32_t k = threadIdx.x; k < K; k += blockDim.x)
            if (s_dk[k]) atomicAdd(reinterpret_cast<unsigned long long*>(dk) + k, s_dk[k]);
    }
}

struct SweepArgs {
    const uint64_t* doc_off;
    const uint32_t* words;
    uint16_t* z;
    int32_t* ndk;
    const int32_t* nkw;     // start-of-sweep snapshot (own-topic weight)
    const int32_t* nk;
    const float* phi;       // per-word topic weights of the snapshot
    int32_t* nkw_next;
    int32_t* nk_next;
    const float* alpha;
    const uint32_t* doc_order;
    uint32_t* doc_counter;
    // weighted counts (TermWeight IDF / PMI): ndk, nkw and nk hold floats,
    // the deltas go to dkw / dk in units of 2^-24
    const float* wt;          // token weights (doc-major)
    long long* dkw;           // V x K
    long long* dk;            // K
    PriorArgs pr;             // word priors (all NULL: none)
    // integer counts: rm1[k] = 1 / ((float)(n_k[k] - 1) + esum_k), the own
    // topic's reciprocal, built with the group's word table (NULL: divide)
    const float* rm1;
    // per-document conditionals of the derived models (all NULL: none):
    // A_k = ((float)n_dk + alpha_dk) * m_dk
    const float* alpha_rows;  // M x K
    const uint32_t* arow;     // D: the document's row of alpha_rows
    const uint32_t* mask;     // D x mw words: bit k = topic k allowed
    uint32_t mw;
    uint64_t D;
    uint32_t K, V, c;
    float eta, veta;
    uint64_t seed;
    uint32_t iter;
    const uint32_t* iter_ptr; // non-null (a captured sweep): the sweep counter lives on the device
    uint64_t pos_begin, pos_end;  // this launch samples doc_order positions [pos_begin, pos_end)
    uint64_t tok_offset;     // global index of token 0 (a shard of a corpus split across GPUs)
    uint32_t scan_steps;     // Hillis-Steele steps over the lanes holding topics: ceil(log2(min(32, ceil(K/4))))
    uint32_t rowi_smem;      // 1: the int n_dk row lives in shared memory
    uint32_t dnk_smem;       // 1: n_k deltas aggregate in shared memory
    // split documents: positions [pos_begin, pos_begin + n_long) are sampled
    // one per block in slices (phase 1 of k_sweep_doc); 0: none
    uint32_t n_long;
    uint32_t split_step;     // positions per slice between merges
    uint32_t* long_counter;  // phase 1's document counter
    // shared rows (PT's pseudo-documents, tmt_set_doc_rows): doc_order holds
    // rows; row r's documents are unit_docs[unit_off[r] .. unit_off[r+1]),
    // sampled one after another with the row live.  NULL: every document is
    // its own row.
    const uint64_t* unit_off;
    const uint32_t* unit_docs;
    uint64_t max_len;        // the launch's longest document (or shared row), all ids counted
};

// Shared-memory layout of a sweep block (offsets in 4-byte words, 16-byte
// aligned regions): [alpha: KP floats] [n_k deltas: KP ints] [per warp:
// (float)n_dk + alpha, KP floats, zero padded] [per warp: n_dk, KP ints
// (floats with weighted counts)]; with weighted counts there are no n_k
// deltas here.  Static: the pass-2 column scratch.



// Topics are dealt to lanes in blocks of four: lane l owns k = 128*j + 4*l + i.
// Every warp-wide float4 load of a K-vector is one contiguous 512-byte run
// and shared-memory float4 reads are conflict-free.
//   CH > 0: at most CH blocks per lane (KP <= 128*CH <= 4096), unrolled.
//   CH == 0: any K, runtime loops.
//   WT: weighted counts (TermWeight IDF / PMI): n_dk, n_kw, n_k are floats,
//       every token carries a weight w, a removal clamps at 0 (updateCnt<true>,
//       Utils.hpp:132-155) and the count deltas are integers in units of 2^-24.
//   SPLIT: the launch's first n_long documents are split (phase 1); the
//       kernels without it carry no phase-1 code.
//   PLAIN: plain LDA with integer counts -- no word priors, per-document
//       masks or alphas, the own-topic reciprocal table and n_k deltas in
//       shared memory present -- so the token loop carries none of those
//       checks or pointers (~60 fewer warp instructions per token at K = 1000;
//       the same arithmetic).
//   ROW16: the document's count row lives in shared memory as 16-bit counts
//       (the host guarantees every document of the launch is shorter than
//       65,536 tokens), half the space of 32-bit rows: variant 1 runs 5
//       blocks of 5 warps per SM without reading the row through L1.
template <int CH, int MINB, bool WT, bool SPLIT = false, bool PLAIN = false, bool ROW16 = false>
__global__ void __launch_bounds__((ROW16 ? kRow16Warps : kSweepWarps) * 32, ROW16 ? kRow16MinB : MINB)
k_sweep_doc(SweepArgs a)
{
    static_assert(!(PLAIN && WT), "plain LDA has integer counts");
    static_assert(!(ROW16 && (WT || SPLIT)), "16-bit rows: integer counts, no split documents");
    using CT = typename std::conditional<WT, float, int>::type;
    constexpr int CHR = CH > 0 ? CH : 1;
    extern __shared__ __align__(16) int smem[];
    const int K = (int)a.K;
    const int KP = (int)round4(a.K);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
    // n_k deltas in shared memory: integer counts only (weighted counts take
    // theirs from the word deltas after the sweep, k_dk_sum)
    const bool dnk_smem = !WT && (PLAIN || a.dnk_smem);
    // alpha (read from here unless per-document alpha rows are set)
    float* s_alpha = reinterpret_cast<float*>(smem);
    // the hit lane's blocks of four of the word's column, for pass 2 (CH > 0):
    // a shared-memory read instead of a second trip to L2 for the column
    // (not in the MINB-4 kernels: in the 16-bit-row kernel it measured
    // slower, 94.9 vs 92.7 ms per sweep at k = 1000, and at 64 registers its
    // addressing spills, spilled registers coming back from L2)
    constexpr bool kScratch = CH > 0 && MINB < 4;
    __shared__ __align__(16) float s_xs[kScratch ? kSweepWarps * 4 * CHR : 4];
    int* s_dnk = smem + KP;
    float* s_rowf = reinterpret_cast<float*>(s_dnk + (dnk_smem ? KP : 0));
    float* rowf = s_rowf + warp * KP;
    int* s_rowi = reinterpret_cast<int*>(s_rowf + nwarps * KP);
    // split documents (integer counts): the document's row C and the slices'
    // merged changes of the current step, after the per-warp rows
    constexpr bool split = SPLIT && !WT;
    int* s_C = s_rowi + ((a.rowi_smem || split) ? nwarps * KP : 0);
    int* s_dlt = s_C + KP;
    __shared__ uint32_t s_q;
    for (int k = threadIdx.x; k < K; k += blockDim.x) {
        s_alpha[k] = a.alpha[k];
        if (dnk_smem) s_dnk[k] = 0;
    }
    __syncthreads();
    // blocks of four owned by this lane
    const int nch = 4 * lane < K ? ((K - 4 * lane + 127) >> 7) : 0;
    float lm[5];                         // hs_step's lane masks
#pragma unroll
    for (int i = 0; i < 5; ++i) lm[i] = lane >= (1 << i) ? 1.f : 0.f;
    auto scan32 = [&](float x) {
#pragma unroll
        for (int i = 0; i < 5; ++i) x = hs_step(x, 1 << i, lm[i]);
        return x;
    };
    auto scan_n = [&](float x, int steps) {
#pragma unroll
        for (int i = 0; i < 5; ++i)
            if (i < steps) x = hs_step(x, 1 << i, lm[i]);
        return x;
    };
    const float eta = a.eta, veta = a.veta;
    const uint32_t iter = a.iter_ptr ? *a.iter_ptr : a.iter;

    // the own topic's word weight with the token removed from n_kw and n_k,
    // phio (w: the token's weight).  A word's weights: this lane's blocks of four of its table column.  A
    // document's tokens are sorted by word, so about 40% of the tokens of the
    // benchmark corpora repeat the previous token's word: the column stays in
    // registers (the table is the group's snapshot, so it cannot change).
    auto load_col = [&](uint32_t v, float4 (&pv)[CHR]) {
        const float* ph = a.phi + (uint64_t)v * KP;
        if constexpr (CH > 0) {
#pragma unroll
            for (int jj = 0; jj < CHR; ++jj)
                if (jj < nch) pv[jj] = __ldg(reinterpret_cast<const float4*>(ph + 128 * jj + 4 * lane));
        }
    };
    // nkw_o = n_kw[zo, v] and ri = rm1[zo] of the snapshot, loaded for a batch
    // of 32 tokens at once (the table cannot change during the launch)
    auto load_word = [&](uint32_t v, int zo, float w, CT nkw_o, float ri, float& phio) {
        float eo = eta;
        if (!PLAIN && a.pr.idx) {
            const float* pe = prior_col(a.pr, v, K);
            if (pe) eo = __ldg(pe + zo);
        }
        auto so = [&]() { return (!PLAIN && a.pr.idx) ? __ldg(a.pr.esum + zo) : veta; };
        if constexpr (WT) {
            const CT nk_o = __ldg(reinterpret_cast<const CT*>(a.nk) + zo);
            float co = __fsub_rn(nkw_o, w), no = __fsub_rn(nk_o, w);
            co = co > 0.f ? co : 0.f;
            no = no > 0.f ? no : 0.f;
            phio = __fmul_rn(__fadd_rn(co, eo), __fdiv_rn(1.0f, __fadd_rn(no, so())));
        } else {
            float rinv;
            if (PLAIN || a.rm1) {
                rinv = ri;
            } else {
                const CT nk_o = __ldg(reinterpret_cast<const CT*>(a.nk) + zo);
                rinv = __fdiv_rn(1.0f, __fadd_rn((float)(nk_o - 1), so()));
            }
            phio = __fmul_rn(__fadd_rn((float)(nkw_o - 1), eo), rinv);
        }
    };

    float4 pv[CHR];                      // the column of word v_have (see load_col)
    uint32_t v_have = 0xFFFFFFFFu;
    // the current document's alphas and topic mask (the derived models' conditionals)
    const float* alpha = a.alpha;
    const uint32_t* dmask = nullptr;
    auto set_doc = [&](uint64_t d) {
        if constexpr (!PLAIN) {
            alpha = a.arow ? a.alpha_rows + (uint64_t)a.arow[d] * K : a.alpha;
            dmask = a.mask ? a.mask + d * (uint64_t)a.mw : nullptr;
        }
    };
    auto afold = [&](float n, int k) -> float {
        // (the shared copy unless the document has its own alpha row)
        const float x = __fadd_rn(n, (PLAIN || !a.arow) ? s_alpha[k] : __ldg(alpha + k));
        if constexpr (PLAIN) return x;
        else return dmask ? __fmul_rn(x, (float)((__ldg(dmask + (k >> 5)) >> (k & 31)) & 1u)) : x;
    };
    // Samples the tokens [b, e) of the current document in order with the
    // document row rowi (counts) / rowf (A_k) live; with dlt != NULL every
    // change of the row is added to dlt as well.
    const bool has_ri = !WT && (PLAIN || a.rm1 != nullptr);
    auto run_tokens = [&](uint64_t b, uint64_t e, auto* rowi, float* rowf, int* dlt) {
            for (uint64_t base = b; base < e; base += 32) {
                const uint64_t my_i = base + lane;
                uint32_t my_w = 0xFFFFFFFFu, my_z = 0xFFFF;
                float my_u = 0.f, my_wt = 0.f;
                // this lane's token's own-topic count and reciprocal in the snapshot:
                // 32 independent loads per batch instead of one on every token's chain
                CT my_nkw = CT(0);
                float my_ri = 0.f;
                if (my_i < e) {
                    my_w = a.words[my_i];
                    my_z = a.z[my_i];
                    if (WT) my_wt = a.wt[my_i];
                    if (my_w < a.V) {
                        my_nkw = __ldg(reinterpret_cast<const CT*>(a.nkw) + (uint64_t)my_w * K + my_z);
                        if (has_ri) my_ri = __ldg(a.rm1 + my_z);
                    }
                    const uint64_t gi = my_i + a.tok_offset;
                    my_u = tmt::u01(tmt::philox_u32((uint32_t)gi, (uint32_t)(gi >> 32), tmt::kStreamSweep,
                                                    iter, a.seed));
                }
                uint32_t my_new = my_z;
                unsigned vm = __ballot_sync(FULL, my_i < e && my_w < a.V);
                if (vm) {
                    int j = __ffs(vm) - 1;
                    vm &= vm - 1;
                    uint32_t v = __shfl_sync(FULL, my_w, j);
                    int zo = (int)__shfl_sync(FULL, my_z, j);
                    if (v != v_have) {
                        load_col(v, pv);
                        v_have = v;
                    }
                    float phi_own;
                    load_word(v, zo, WT ? __shfl_sync(FULL, my_wt, j) : 1.f, __shfl_sync(FULL, my_nkw, j),
                              has_ri ? __shfl_sync(FULL, my_ri, j) : 0.f, phi_own);
                    for (;;) {
                        const int jn = vm ? __ffs(vm) - 1 : -1;
                        const float u = __shfl_sync(FULL, my_u, j);
                        const float wt = WT ? __shfl_sync(FULL, my_wt, j) : 1.f;
                        const float* ph = a.phi + (uint64_t)v * KP;
                        // remove the token from its document.  The own topic's document
                        // weight Ao is held in a register and its slot of the row is 0
                        // until the draw is made, so pass 1's chain leaves the own topic
                        // out exactly and its owner adds Ao * phi_own last: no
                        // subtract-and-add that could cancel when the own topic dominates its lane
                        // (every lane forms the new count and Ao; lane 0 stores them)
                        CT n_rm;             // (from a 16-bit row: promoted, and stored back below 65,536)
                        if constexpr (WT) {
                            n_rm = __fsub_rn(rowi[zo], wt);
                            n_rm = n_rm > 0.f ? n_rm : 0.f;
                        } else {
                            n_rm = rowi[zo] - 1;
                        }
                        const float Ao = afold((float)n_rm, zo);
                        __syncwarp();
                        if (lane == 0) {
                            rowi[zo] = n_rm;
                            rowf[zo] = 0.f;
                        }
                        __syncwarp();
                        // pass 1: fma chain over this lane's topics
                        float s = 0.f;
                        if (CH > 0) {
    #pragma unroll
                            for (int jj = 0; jj < CHR; ++jj) {
                                if (jj < nch) {
                                    const float4 A4 = *reinterpret_cast<const float4*>(rowf + 128 * jj + 4 * lane);
                                    s = __fmaf_rn(A4.x, pv[jj].x, s);
                                    s = __fmaf_rn(A4.y, pv[jj].y, s);
                                    s = __fmaf_rn(A4.z, pv[jj].z, s);
                                    s = __fmaf_rn(A4.w, pv[jj].w, s);
                                }
                            }
                        } else {
                            for (int jj = 0; jj < nch; ++jj) {
                                const float4 A4 = *reinterpret_cast<const float4*>(rowf + 128 * jj + 4 * lane);
                                const float4 P4 = __ldg(reinterpret_cast<const float4*>(ph + 128 * jj + 4 * lane));
                                s = __fmaf_rn(A4.x, P4.x, s);
                                s = __fmaf_rn(A4.y, P4.y, s);
                                s = __fmaf_rn(A4.z, P4.z, s);
                                s = __fmaf_rn(A4.w, P4.w, s);
                            }
                        }
                        // the own topic, with the token excluded from n_kw and n_k
                        if (lane == ((zo >> 2) & 31)) s = __fadd_rn(s, __fmul_rn(Ao, phi_own));
                        // lanes at or above min(32, ceil(K/4)) hold no topics: a Hillis-Steele
                        // scan of scan_steps = ceil(log2(that)) steps gives the other lanes
                        // the values of the full scan, and the total sits in lane
                        // 2^scan_steps - 1
                        // (above 128 topics every lane holds topics: the five steps, unrolled)
                        const float x = CH >= 2 ? scan32(s) : scan_n(s, a.scan_steps);
                        const float E = __fmul_rn(__shfl_up_sync(FULL, x, 1), lm[0]);   // 0 in lane 0
                        const float total = __shfl_sync(FULL, x, CH >= 2 ? 31 : (1 << a.scan_steps) - 1);
                        const float r = __fmul_rn(u, total);
                        const unsigned m = __ballot_sync(FULL, nch > 0 && r < __fadd_rn(E, s));
                        int znew = K - 1;
                        if (m) {
                            // pass 2: position among lane h's topics
                            const int h = __ffs(m) - 1;
                            const float Eh = __shfl_sync(FULL, E, h);
                            const int mh = K - 4 * h;
                            const int nh = 4 * (mh >> 7) + min(mh & 127, 4);
                            int found = nh - 1;
                            if (CH > 0 && CH <= 2) {
                                // at most 8 topics: lane h forms their Hillis-Steele prefix sums
                                // (the warp-wide scan's order) from the weights in its registers
                                if (lane == h) {
                                    float c[4 * CHR];
    #pragma unroll
                                    for (int jj = 0; jj < CHR; ++jj) {
                                        const float4 A4 = jj < nch ? *reinterpret_cast<const float4*>(rowf + 128 * jj + 4 * h)
                                                                   : make_float4(0.f, 0.f, 0.f, 0.f);
                                        const float av[4] = { A4.x, A4.y, A4.z, A4.w };
                                        const float pw[4] = { pv[jj].x, pv[jj].y, pv[jj].z, pv[jj].w };
    #pragma unroll
                                        for (int i = 0; i < 4; ++i) {
                                            const int t = 4 * jj + i;
                                            const int k = 128 * jj + 4 * h + i;
                                            c[t] = t < nh ? (k == zo ? __fmul_rn(Ao, phi_own) : __fmul_rn(av[i], pw[i])) : 0.f;
                                        }
                                    }
    #pragma unroll
                                    for (int off = 1; off < 4 * CHR; off <<= 1) {
    #pragma unroll
                                        for (int t = 4 * CHR - 1; t >= off; --t) c[t] = __fadd_rn(c[t], c[t - off]);
                                    }
                                    bool hit = false;
    #pragma unroll
                                    for (int t = 0; t < 4 * CHR; ++t) {
                                        if (!hit && t < nh && r < __fadd_rn(Eh, c[t])) {
                                            found = t;
                                            hit = true;
                                        }
                                    }
                                }
                                found = __shfl_sync(FULL, found, h);
                            } else {
                                // 32 at a time; up to 16 topics (CH == 4) a 4-step scan gives the
                                // same prefix values
                                constexpr int kSteps2 = CH == 4 ? 4 : 5;
                                if (kScratch) {
                                    // lane h's column blocks into the warp's scratch (t-th topic at t)
                                    if (lane == h) {
    #pragma unroll
                                        for (int jj = 0; jj < CHR; ++jj)
                                            if (jj < nch) *reinterpret_cast<float4*>(s_xs + 4 * (CHR * warp + jj)) = pv[jj];
                                    }
                                    __syncwarp();
                                }
                                float carry = 0.f;
                                for (int mm = 0; mm < nh; mm += 32) {
                                    const int t = mm + lane;
                                    const int k = 128 * (t >> 2) + 4 * h + (t & 3);
                                    float x2 = 0.f;
                                    // rowf[zo] reads 0 until the draw: fma(sel, phi_own, 0 * phi) is
                                    // Ao * phi_own at zo and fma(0, phi_own, p) == p elsewhere
                                    if (t < nh)
                                        x2 = __fmaf_rn(k == zo ? Ao : 0.f, phi_own,
                                                       __fmul_rn(rowf[k], kScratch ? s_xs[4 * CHR * warp + t] : __ldg(ph + k)));
                                    x2 = scan_n(x2, kSteps2);
                                    const unsigned mb =
                                        __ballot_sync(FULL, t < nh && r < __fadd_rn(Eh, __fadd_rn(carry, x2)));
                                    if (mb) { found = mm + __ffs(mb) - 1; break; }
                                    carry = __fadd_rn(carry, __shfl_sync(FULL, x2, 31));
                                }
                            }
                            znew = 128 * (found >> 2) + 4 * h + (found & 3);
                        }
                        // the new topic's count: every lane forms it, lane 0 stores
                        CT n_add;
                        if constexpr (WT) n_add = __fadd_rn(rowi[znew], wt);
                        else n_add = rowi[znew] + 1;
                        const float A_add = afold((float)n_add, znew);
                        __syncwarp();
                        if (lane == 0) {
                            rowf[zo] = Ao;            // the own topic's slot back (znew's update follows)
                            rowi[znew] = n_add;
                            rowf[znew] = A_add;
                            if constexpr (WT) {
                                if (znew != zo) {
                                    const unsigned long long q = (unsigned long long)__float2ll_rn(__fmul_rn(wt, 16777216.f));
                                    unsigned long long* dw = reinterpret_cast<unsigned long long*>(a.dkw) + (uint64_t)v * K;
                                    atomicAdd(dw + zo, 0ull - q);
                                    atomicAdd(dw + znew, q);
                                    // n_k's deltas are the column sums of these (k_dk_sum)
                                }
                            } else {
                                if (znew != zo) {
                                    atomicSub(&a.nkw_next[(uint64_t)v * K + zo], 1);
                                    atomicAdd(&a.nkw_next[(uint64_t)v * K + znew], 1);
                                    if (PLAIN || a.dnk_smem) { atomicSub(&s_dnk[zo], 1); atomicAdd(&s_dnk[znew], 1); }
                                    else { atomicSub(&a.nk_next[zo], 1); atomicAdd(&a.nk_next[znew], 1); }
                                    if (dlt) { atomicSub(&dlt[zo], 1); atomicAdd(&dlt[znew], 1); }
                                }
                            }
                        }
                        __syncwarp();
                        if (lane == j) my_new = (uint32_t)znew;
                        if (jn < 0) break;
                        j = jn;
                        vm &= vm - 1;
                        v = __shfl_sync(FULL, my_w, j);
                        zo = (int)__shfl_sync(FULL, my_z, j);
                        if (v != v_have) {
                            load_col(v, pv);
                            v_have = v;
                        }
                        load_word(v, zo, WT ? __shfl_sync(FULL, my_wt, j) : 1.f, __shfl_sync(FULL, my_nkw, j),
                                  has_ri ? __shfl_sync(FULL, my_ri, j) : 0.f, phi_own);
                    }
                }
                if (my_i < e && my_w < a.V) a.z[my_i] = (uint16_t)my_new;
            }
    };

    // Phase 1: split documents, one per block.  The first n_long documents of
    // this launch hold at least split_len tokens; a block cuts one into
    // nwarps slices (slice w = [b + w*L/nwarps, b + (w+1)*L/nwarps)) and its
    // warps sample them side by side in steps of split_step positions, each
    // with a private copy of the row as of the step's start plus its own
    // changes; after each step the row C gains all slices' changes.  Only
    // integer sums are merged, so the result does not depend on timing.
    if constexpr (split) {
        CT* prow = reinterpret_cast<CT*>(s_rowi + warp * KP);
        for (;;) {
            __syncthreads();                  // the previous document is written back; s_q is free
            if (threadIdx.x == 0) s_q = atomicAdd(a.long_counter, 1u);
            __syncthreads();
            const uint32_t q = s_q;
            if (q >= a.n_long) break;
            const uint64_t d = a.doc_order[a.pos_begin + q];
            set_doc(d);
            int* grow = reinterpret_cast<int*>(a.ndk) + d * (uint64_t)K;
            for (int k = threadIdx.x; k < K; k += blockDim.x) {
                s_C[k] = grow[k];
                s_dlt[k] = 0;
            }
            __syncthreads();
            const uint64_t b = a.doc_off[d], L = a.doc_off[d + 1] - b;
            const uint64_t sb = b + (uint64_t)warp * L / nwarps, se = b + (uint64_t)(warp + 1) * L / nwarps;
            const uint64_t m = a.split_step;
            const uint64_t steps = ((L + nwarps - 1) / nwarps + m - 1) / m;   // the longest slice's steps
            for (uint64_t st = 0; st < steps; ++st) {
                for (int k = lane; k < KP; k += 32) {
                    const int n = k < K ? s_C[k] : 0;
                    prow[k] = (CT)n;
                    rowf[k] = k < K ? afold((float)n, k) : 0.f;
                }
                __syncwarp();
                const uint64_t tb = sb + st * m, te = min(tb + m, se);
                if (tb < te) run_tokens(tb, te, prow, rowf, s_dlt);
                __syncthreads();              // every slice's changes of this step are in s_dlt
                for (int k = threadIdx.x; k < K; k += blockDim.x) {
                    s_C[k] += s_dlt[k];
                    s_dlt[k] = 0;
                }
                __syncthreads();
            }
            for (int k = threadIdx.x; k < K; k += blockDim.x) grow[k] = s_C[k];
        }
    }

    // Phase 2: the other documents (or shared rows), one per warp, in order
    // with the row live.
    for (;;) {
        uint32_t q = 0;
        if (lane == 0) q = atomicAdd(a.doc_counter, 1u);
        q = __shfl_sync(FULL, q, 0);
        const uint64_t pos = a.pos_begin + (split ? a.n_long : 0) + q;
        if (pos >= a.pos_end) break;
        const uint64_t d = a.doc_order[pos];
        set_doc(d);
        CT* grow = reinterpret_cast<CT*>(a.ndk) + d * (uint64_t)K;
        using RT = typename std::conditional<ROW16, uint16_t, CT>::type;
        const bool row_smem = ROW16 || a.rowi_smem;
        RT* rowi = row_smem ? reinterpret_cast<RT*>(s_rowi) + warp * KP : reinterpret_cast<RT*>(grow);
        for (int k = lane; k < KP; k += 32) {
            float f = 0.f;
            if (k < K) {
                const CT n = grow[k];
                if (row_smem) rowi[k] = (RT)n;
                f = afold((float)n, k);
            }
            rowf[k] = f;
        }
        __syncwarp();
        if (a.unit_off) {
            for (uint64_t u = a.unit_off[d]; u < a.unit_off[d + 1]; ++u) {
                const uint64_t dd = a.unit_docs[u];
                run_tokens(a.doc_off[dd], a.doc_off[dd + 1], rowi, rowf, nullptr);
            }
        } else {
            run_tokens(a.doc_off[d], a.doc_off[d + 1], rowi, rowf, nullptr);
        }
        __syncwarp();
        if (row_smem)
            for (int k = lane; k < K; k += 32) grow[k] = (CT)rowi[k];
        __syncwarp();
    }
    if (dnk_smem) {
        __syncthreads();
        for (int k = threadIdx.x; k < K; k += blockDim.x)
            if (s_dnk[k]) atomicAdd(&a.nk_next[k], s_dnk[k]);
    }
}

// ---------------------------------------------------------------------------
// log-likelihood in FP64 (getLLDocs / getLLRest, LDAModel.hpp:616-668)
// ---------------------------------------------------------------------------

// n_dk rows and n_kw columns, each dealt to the warps in a fixed order, and
// fixed reduction trees: bit-reproducible.
// lg_alpha[k] = lgamma(alpha_k); asum[0] = sum(alpha), asum[1] = lgamma(sum(alpha))
__global__ void k_ll_prep(const float* __restrict__ alpha, uint32_t K, double* __restrict__ lg_alpha,
                          double* __restrict__ asum)
{
    for (uint32_t k = threadIdx.x; k < K; k += blockDim.x) lg_alpha[k] = lgamma((double)alpha[k]);
    if (threadIdx.x == 0) {
        double s = 0;
        for (uint32_t k = 0; k < K; ++k) s += (double)alpha[k];
        asum[0] = s;
        asum[1] = lgamma(s);
    }
}

// CT: the count type (int32 for TermWeight ONE, float for weighted counts);
// LT: the document length type (token count or weight sum).
template <typename CT, typename LT>
__global__ void k_ll_partials(const CT* __restrict__ ndk, uint64_t D, uint32_t K,
                              const double* __restrict__ lg_alpha, const float* __restrict__ alpha,
                              const LT* __restrict__ doc_len, const double* __restrict__ asum_p,
                              const CT* __restrict__ nkw, uint32_t V, double eta, double lg_eta,
                              double* __restrict__ partials, PriorArgs pr, const float* __restrict__ alpha_rows,
                              const uint32_t* __restrict__ arow, const double* __restrict__ row_asum)
{
    __shared__ double s_d[32], s_r[32];
    const double asum = asum_p[0], lg_asum = asum_p[1];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const uint64_t gw = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
    const uint64_t nw = ((uint64_t)gridDim.x * blockDim.x) >> 5;
    double accd = 0, accr = 0;
    for (uint64_t r = gw; r < D; r += nw) {
        const CT* p = ndk + r * K;
        if (arow) {
            // the document's own alphas (DMR's getLLDocTopic, DMRModel.hpp:208-224)
            const float* al = alpha_rows + (uint64_t)arow[r] * K;
            for (uint32_t k = lane; k < K; k += 32) {
                const CT n = p[k];
                if (n != CT(0)) accd += lgamma((double)n + (double)al[k]) - lgamma((double)al[k]);
            }
            const double as_r = row_asum[2 * arow[r]], lgas_r = row_asum[2 * arow[r] + 1];
            if (lane == 0) accd -= lgamma((double)doc_len[r] + as_r) - lgas_r;
            continue;
        }
        for (uint32_t k = lane; k < K; k += 32) {
            const CT n = p[k];
            if (n != CT(0)) accd += lgamma((double)n + (double)alpha[k]) - lg_alpha[k];
        }
        if (lane == 0) accd -= lgamma((double)doc_len[r] + asum) - lg_asum;
    }
    // the word rows' assignment does not depend on D: LLRest is the same bits on
    // every rank of a sharded corpus and on one GPU holding all of it
    for (uint64_t v = gw; v < V; v += nw) {
        const CT* p = nkw + v * K;
        const float* pe = prior_col(pr, v, K);
        for (uint32_t k = lane; k < K; k += 32) {
            const CT n = p[k];
            if (n == CT(0)) continue;
            if (pe) accr += lgamma((double)n + (double)pe[k]) - lgamma((double)pe[k]);
            else accr += lgamma((double)n + eta) - lg_eta;
        }
    }
    accd = warp_sum(accd);
    accr = warp_sum(accr);
    if (lane == 0) { s_d[warp] = accd; s_r[warp] = accr; }
    __syncthreads();
    if (warp == 0) {
        const int nwb = blockDim.x >> 5;
        double x = lane < nwb ? s_d[lane] : 0.0, y = lane < nwb ? s_r[lane] : 0.0;
        x = warp_sum(x);
        y = warp_sum(y);
        if (lane == 0) { partials[2 * blockIdx.x] = x; partials[2 * blockIdx.x + 1] = y; }
    }
}

// esum != NULL (word priors): the per-topic sums of eta replace V*eta
template <typename CT>
__global__ void k_ll_final(const double* __restrict__ partials, uint32_t nparts,
                           const CT* __restrict__ nk, uint32_t K, double veta, double* __restrict__ out,
                           const float* __restrict__ esum)
{
    __shared__ double s_d[32], s_r[32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    double x = 0, y = 0;
    for (uint32_t i = threadIdx.x; i < nparts; i += blockDim.x) { x += partials[2 * i]; y += partials[2 * i + 1]; }
    for (uint32_t k = threadIdx.x; k < K; k += blockDim.x) {
        const double es = esum ? (double)esum[k] : veta;
        y += lgamma(es) - lgamma((double)nk[k] + es);
    }
    x = warp_sum(x);
    y = warp_sum(y);
    if (lane == 0) { s_d[warp] = x; s_r[warp] = y; }
    __syncthreads();
    if (warp == 0) {
        const int nwb = blockDim.x >> 5;
        x = lane < nwb ? s_d[lane] : 0.0;
        y = lane < nwb ? s_r[lane] : 0.0;
        x = warp_sum(x);
        y = warp_sum(y);
        if (lane == 0) { out[0] = x; out[1] = y; }
    }
}

// ---------------------------------------------------------------------------
// log-likelihood without device allocation (tmt_ll_counts_noalloc)
// ---------------------------------------------------------------------------
// Scratch of tmt_ll_counts_noalloc: 2 partial sums per block of the partial
// kernel, lgamma(alpha_k) for up to 32767 topics, sum(alpha) and its lgamma.
// 281 KB; every GPU that loads this library holds it until the process exits.
constexpr uint32_t kNoAllocMaxBlocks = 1184;
constexpr uint32_t kNoAllocMaxK = 32767;
static __device__ __align__(256) double g_ll_scratch[2 * kNoAllocMaxBlocks + kNoAllocMaxK + 2];

// Blocks of the log-likelihood's partial-sum kernel on a GPU with `sms` SMs:
// tmt_ll and tmt_ll_counts_noalloc use the same grid, so they add the same
// terms in the same order.
inline uint32_t ll_blocks(int sms)
{
    return std::min<uint32_t>(kNoAllocMaxBlocks, (uint32_t)std::max(1, sms * 8));
}

// The unique id of the calling thread's current CUDA context (0: none, or
// the driver does not say).  The driver's cuCtxGetCurrent / cuCtxGetId are
// reached through the runtime, so the library does not link the driver
// library; ids are never reused within a process, unlike context handles.
unsigned long long current_context_id()
{
    using GetCurrent = int (*)(void**);
    using GetId = int (*)(void*, unsigned long long*);
    static GetCurrent get_current = nullptr;
    static GetId get_id = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q{};
        if (cudaGetDriverEntryPointByVersion("cuCtxGetCurrent", &p, 12000, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            get_current = reinterpret_cast<GetCurrent>(p);
        p = nullptr;
        if (cudaGetDriverEntryPointByVersion("cuCtxGetId", &p, 12000, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            get_id = reinterpret_cast<GetId>(p);
        cudaGetLastError();
    });
    void* ctx = nullptr;
    unsigned long long id = 0;
    if (!get_current || !get_id || get_current(&ctx) != 0 || !ctx || get_id(ctx, &id) != 0) return 0;
    return id;
}

// ---------------------------------------------------------------------------
// alpha optimisation (optimizeParameters / calcDigammaSum, LDAModel.hpp:221-265)
// ---------------------------------------------------------------------------
// part_nom[bx*K + k] = sum over this block's docs of digammaApprox(n_dk + alpha_k)
// part_den[bx]       = sum over this block's docs of digammaApprox(N_d + sum(alpha))
template <typename CT, typename LT>
__global__ void k_alpha_sums(const CT* __restrict__ ndk, uint64_t D, uint32_t K,
                             const float* __restrict__ alpha, const LT* __restrict__ doc_len,
                             const float* __restrict__ asum_p,
                             double* __restrict__ part_nom, double* __restrict__ part_den)
{
    __shared__ double s_red[32];
    const uint64_t per = (D + gridDim.x - 1) / gridDim.x;
    const uint64_t d0 = blockIdx.x * per, d1 = min(D, d0 + per);
    const uint32_t k = blockIdx.y * blockDim.x + threadIdx.x;
    if (k < K) {
        const float ak = alpha[k];
        double acc = 0;
        uint64_t zeros = 0;
        for (uint64_t d = d0; d < d1; ++d) {
            const CT n = ndk[d * K + k];
            if (n != CT(0)) acc += (double)tmt::digamma_approx_f(__fadd_rn((float)n, ak));
            else ++zeros;
        }
        acc += (double)zeros * (double)tmt::digamma_approx_f(ak);
        part_nom[(uint64_t)blockIdx.x * K + k] = acc;
    }
    if (blockIdx.y == 0) {
        const float as = *asum_p;
        double acc = 0;
        for (uint64_t d = d0 + threadIdx.x; d < d1; d += blockDim.x)
            acc += (double)tmt::digamma_approx_f(__fadd_rn((float)doc_len[d], as));
        acc = warp_sum(acc);
        const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
        if (lane == 0) s_red[warp] = acc;
        __syncthreads();
        if (warp == 0) {
            double x = lane < (int)(blockDim.x >> 5) ? s_red[lane] : 0.0;
            x = warp_sum(x);
            if (lane == 0) part_den[blockIdx.x] = x;
        }
    }
}

// One fixed-point step for every k, then the new sum(alpha) for the next step.
__global__ void k_alpha_update(const double* __restrict__ part_nom, const double* __restrict__ part_den,
                               uint32_t nparts, uint32_t K, uint64_t D, float* __restrict__ alpha,
                               float* __restrict__ asum_p, const float* __restrict__ dg_points)
{
    __shared__ double s_den;
    tmt::DigammaTable dg{ dg_points };
    if (threadIdx.x == 0) {
        double den = 0;
        for (uint32_t i = 0; i < nparts; ++i) den += part_den[i];
        s_den = den - (double)D * (double)dg(*asum_p);
    }
    __syncthreads();
    const double den = s_den;
    for (uint32_t k = threadIdx.x; k < K; k += blockDim.x) {
        double nom = 0;
        for (uint32_t i = 0; i < nparts; ++i) nom += part_nom[(uint64_t)i * K + k];
        const float ak = alpha[k];
        nom -= (double)D * (double)dg(ak);
        const float na = __fmul_rn(__fdiv_rn((float)nom, (float)den), ak);
        alpha[k] = na > 1e-5f ? na : 1e-5f;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        float s = 0.f;
        for (uint32_t k = 0; k < K; ++k) s = __fadd_rn(s, alpha[k]);
        *asum_p = s;
    }
}

// sums of the partial rows in the order k_alpha_update uses: out[k] (k < K) and out[K]
__global__ void k_alpha_fold(const double* __restrict__ part_nom, const double* __restrict__ part_den,
                             uint32_t nparts, uint32_t K, double* __restrict__ out)
{
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k < K) {
        double nom = 0;
        for (uint32_t i = 0; i < nparts; ++i) nom += part_nom[(uint64_t)i * K + k];
        out[k] = nom;
    } else if (k == K) {
        double den = 0;
        for (uint32_t i = 0; i < nparts; ++i) den += part_den[i];
        out[K] = den;
    }
}

// the sweep counter of captured sweeps: set before a run of graph launches,
// advanced by the last node of each
__global__ void k_set_step(uint32_t* __restrict__ step, uint32_t v)
{
    *step = v;
}

__global__ void k_next_step(uint32_t* __restrict__ step)
{
    *step += 1;
}

__global__ void k_sum_alpha(const float* __restrict__ alpha, uint32_t K, float* __restrict__ out)
{
    if (threadIdx.x == 0 && blockIdx.x == 0) {
        float s = 0.f;
        for (uint32_t k = 0; k < K; ++k) s = __fadd_rn(s, alpha[k]);
        *out = s;
    }
}

} // namespace

// ---------------------------------------------------------------------------
// the handle
// ---------------------------------------------------------------------------
struct tmt_handle {
    tmt_config cfg{};
    std::vector<float> alpha;        // host copy (after optimisation when downloaded)
    int device = 0;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    cudaEvent_t kev0 = nullptr, kev1 = nullptr;   // around the sweep kernel only
    cudaEvent_t tev0 = nullptr, tev1 = nullptr;   // around a whole tmt_train call
    double train_ms = 0;
    double sweep_kernel_ms = 0;                   // summed over the last train() call
    uint32_t sweeps_timed = 0;
    int num_sms = 0;
    std::string err;
    cudaEvent_t stage_ev[2] = {nullptr, nullptr};   // the staged transfers' chunk events

    uint64_t D = 0, N_all = 0, N = 0, global_step = 0, bytes = 0, launches = 0;
    int sampler_used = 0;
    float last_ms = 0.f;
    bool uploaded = false;

    // device buffers
    std::vector<void*> allocs;
    uint64_t* d_doc_off = nullptr;
    uint32_t* d_words = nullptr;
    uint16_t* d_z = nullptr;
    int32_t* d_ndk = nullptr;
    int32_t* d_nkw[2] = { nullptr, nullptr };
    int32_t* d_nk[2] = { nullptr, nullptr };
    float* d_phi = nullptr;          // per-word topic weights of the current snapshot
    float* d_rm1 = nullptr;          // K: the own topic's reciprocal of the snapshot
    uint32_t groups = 1;             // document groups per sweep
    std::vector<uint64_t> group_bounds;   // doc_order positions: group g = [b[g], b[g+1])
    // long documents (k_sweep_doc phase 1): per group, the tokens of the
    // global group, and the number of its first (longest) local documents
    // that are split; the lengths of the local documents in doc_order
    std::vector<uint64_t> group_tokens;
    std::vector<uint32_t> group_nlong;
    std::vector<uint64_t> order_len;
    uint64_t split_min = 0;          // 0: the rule (split_len_of); >= 2^32 - 1: never
    uint32_t split_step = kSplitStep;
    // shared rows (tmt_set_doc_rows: PT's pseudo-documents): n_rows rows of
    // n_dk replace the per-document rows; 0: one row per document
    uint64_t n_rows = 0;
    uint64_t row_cap = 0;            // rows the n_dk, length and order buffers hold
    uint64_t unit_cap = 0;           // rows d_unit_off holds
    uint64_t* d_unit_off = nullptr;  // n_rows + 1
    uint32_t* d_unit_docs = nullptr; // D
    uint32_t* d_row_of = nullptr;    // D
    // a corpus sharded across GPUs (tmt_upload_shard); world == 1: this GPU holds all of it
    uint32_t rank = 0, world = 1;
    uint64_t D_global = 0, tok_offset = 0;
    std::vector<uint64_t> gbounds;   // the groups over all ranks (document-count prefix bounds)
    tmt_allreduce_fn allreduce = nullptr;
    void* ar_user = nullptr;
    int32_t* d_delta = nullptr;      // sharded: one group's count deltas, n_kw (K*V) then n_k (K)
    // weighted counts (TermWeight IDF / PMI, tmt_upload_corpus_weighted): d_ndk,
    // d_nkw[0], d_nk[0] hold floats; deltas of a document group in units of 2^-24
    bool weighted = false;
    float* d_wt = nullptr;           // token weights, doc-major
    long long* d_dkw = nullptr;      // V x K
    long long* d_dk = nullptr;       // K
    float* d_doc_wlen = nullptr;     // per document: the sum of its token weights
    // word priors (tmt_set_word_priors): host copies, and their device tables
    // (allocated by the upload)
    std::vector<uint32_t> prior_ids;
    std::vector<float> prior_vals;   // P x K
    int32_t* d_prior_idx = nullptr;  // V: row of d_prior, -1 for no prior
    float* d_prior = nullptr;        // P x K
    float* d_esum = nullptr;         // K: sum over the words of eta_kv
    float* d_prior_cum = nullptr;    // P x K: cumulative rows (z0 draws)
    float* d_cum_eta = nullptr;      // K: cumulative column of eta
    PriorArgs prior_args() const { return PriorArgs{ d_prior_idx, d_prior, d_esum }; }
    // per-document alphas and topic masks (tmt_set_doc_alpha / tmt_set_doc_topic_mask)
    float* d_alpha_rows = nullptr;   // M x K
    uint32_t* d_arow = nullptr;      // D
    double* d_row_asum = nullptr;    // M x 2: sum of a row, lgamma of it
    uint32_t* d_mask = nullptr;      // D x ceil(K/32)
    // sweep-kernel autotuner: variants give bit-identical results, so the
    // first sweeps each time one variant and the fastest is kept.  With
    // several variants they run in the order 0, 1, .., n-1, n-1, .., 0 and
    // each group sums its two timings: sweep times still fall over the first
    // sweeps, and the mirrored order cancels a linear drift.
    int variant = 0;                 // the variant of the sweep being tuned
    int tune_step = 0;
    int n_variants = 1;
    int tuned = -1;                  // 0 once every group has its variant, -1 while tuning
    std::vector<int> group_variant;  // per document group, the fastest variant
    std::vector<std::vector<float>> group_ms;   // tuning: per group, per variant
    std::vector<cudaEvent_t> gev;    // tuning: start/end of each group's sweep kernel
    struct Occ { const void* kern; uint32_t smem; int per_sm; };
    std::vector<Occ> occ;            // blocks per SM of each sweep kernel and shared-memory size launched
    // captured sweeps (single GPU, after tuning): one graph per starting buffer parity
    bool graphs = true;
    uint32_t* d_step = nullptr;
    cudaGraphExec_t graph_exec[2] = { nullptr, nullptr };
    uint64_t graph_kernels = 0;      // kernels in one captured sweep
    int graph_flip = 0;              // buffer parity change of one sweep
    std::vector<cudaEvent_t> run_ev; // graph sweeps: start/end of each run between ll / optimiser steps
    int cur = 0;
    int32_t* d_doc_len = nullptr;
    uint32_t* d_doc_order = nullptr;
    uint32_t* d_counter = nullptr;
    float* d_alpha = nullptr;
    float* d_asum = nullptr;
    double* d_lg_alpha = nullptr;
    double* d_asum_ll = nullptr;     // sum(alpha), lgamma(sum(alpha)) in FP64
    double* d_llv = nullptr;         // tmt_ll output (2)
    double* d_partials = nullptr;
    uint32_t n_partials = 0;
    double* d_ll = nullptr;          // ll history for one train() call (2 per point)
    uint32_t ll_cap = 0;
    float* d_dg_points = nullptr;
    // inference buffers (grown on demand, kept across calls)
    struct InferBufs {
        uint64_t cap_docs = 0, cap_tokens = 0, cap_theta = 0;
        uint64_t* doc_off = nullptr;
        uint32_t* words = nullptr;
        uint16_t* z = nullptr;
        uint64_t* keys = nullptr;
        float* theta = nullptr;
        double* ll = nullptr;
        float* acum = nullptr;
        uint32_t* counter = nullptr;
        float* wt = nullptr;
        uint64_t cap_wt = 0;
    } inf;
    double* d_part_nom = nullptr;
    double* d_part_den = nullptr;
    double* d_alpha_fold = nullptr;  // sharded: K + 1 sums exchanged across ranks
    uint32_t n_apart = 0;

    template <class T>
    T* dalloc(size_t count)
    {
        size_t b = count * sizeof(T);
        if (b == 0) b = 16;
        if (cfg.hbm_budget && bytes + b > cfg.hbm_budget)
            throw OomError("HBM budget exceeded: need " + std::to_string(bytes + b) + " bytes, budget " +
                           std::to_string(cfg.hbm_budget));
        void* p = nullptr;
        cudaError_t e = cudaMalloc(&p, b);
        if (e != cudaSuccess) {
            cudaGetLastError();
            throw OomError(std::string("cudaMalloc failed: ") + cudaGetErrorString(e));
        }
        allocs.push_back(p);
        bytes += b;
        return static_cast<T*>(p);
    }

    void drop_graphs()
    {
        for (auto& g : graph_exec)
            if (g) { cudaGraphExecDestroy(g); g = nullptr; }
    }

    void release()
    {
        if (device >= 0) cudaSetDevice(device);
        drop_graphs();
        for (void* p : allocs) cudaFree(p);
        allocs.clear();
        bytes = 0;
    }

    ~tmt_handle()
    {
        release();
        for (int i = 0; i < 2; ++i)
            if (stage_ev[i]) cudaEventDestroy(stage_ev[i]);
        if (ev0) cudaEventDestroy(ev0);
        if (ev1) cudaEventDestroy(ev1);
        if (kev0) cudaEventDestroy(kev0);
        if (kev1) cudaEventDestroy(kev1);
        if (tev0) cudaEventDestroy(tev0);
        if (tev1) cudaEventDestroy(tev1);
        for (cudaEvent_t e : gev) cudaEventDestroy(e);
        for (cudaEvent_t e : run_ev) cudaEventDestroy(e);
        if (stream) cudaStreamDestroy(stream);
    }
};

namespace {

tmt_status fail(tmt_handle* h, tmt_status s, const std::string& msg)
{
    if (h) h->err = msg;
    return s;
}

template <class F>
tmt_status guarded(tmt_handle* h, F&& f)
{
    try {
        if (h) {
            h->err.clear();
            CK(cudaSetDevice(h->device));
        }
        f();
        return TMT_OK;
    } catch (const ArgError& e) {
        return fail(h, TMT_ERR_INVALID_ARGUMENT, e.what());
    } catch (const OomError& e) {
        return fail(h, TMT_ERR_OUT_OF_MEMORY, e.what());
    } catch (const StateError& e) {
        return fail(h, TMT_ERR_STATE, e.what());
    } catch (const CudaError& e) {
        return fail(h, TMT_ERR_CUDA, e.what());
    } catch (const std::bad_alloc&) {
        return fail(h, TMT_ERR_OUT_OF_MEMORY, "host allocation failed");
    } catch (const std::exception& e) {
        return fail(h, TMT_ERR_INTERNAL, e.what());
    }
}

void launch_check(tmt_handle* h)
{
    ++h->launches;
    CK(cudaGetLastError());
}

// Copies host memory with up to max_threads threads: the first touch of
// freshly allocated pageable pages (a page fault each) then runs on all of
// them.
void host_copy_parallel(char* dst, const char* src, uint64_t bytes, uint32_t max_threads = 16)
{
    const uint64_t per = 1ull << 20;
    const uint32_t hw = std::max(1u, std::thread::hardware_concurrency());
    const uint32_t T = (uint32_t)std::min<uint64_t>(std::min(max_threads, hw), (bytes + per - 1) / per);
    if (T <= 1) {
        std::memcpy(dst, src, bytes);
        return;
    }
    const uint64_t slice = ((bytes + T - 1) / T + 4095) & ~4095ull;
    std::vector<std::thread> th;
    th.reserve(T);
    for (uint32_t t = 0; t < T; ++t) {
        const uint64_t b = (uint64_t)t * slice;
        if (b >= bytes) break;
        const uint64_t n = std::min(slice, bytes - b);
        try {
            th.emplace_back([=] { std::memcpy(dst + b, src + b, n); });
        } catch (...) {
            std::memcpy(dst + b, src + b, n);     // no thread to be had: this one copies the slice
        }
    }
    for (auto& x : th) x.join();
}

constexpr uint64_t kStageChunk = 32ull << 20;   // a staging buffer; staged transfers are >= 32 MB

// true for memory CUDA knows (pinned host, device or managed memory): one
// direct copy serves it; false for plain pageable host memory
bool cuda_visible(const void* p)
{
    cudaPointerAttributes at{};
    const bool known = cudaPointerGetAttributes(&at, p) == cudaSuccess && at.type != cudaMemoryTypeUnregistered;
    cudaGetLastError();
    return known;
}

// Two 32 MB pinned staging buffers shared by every handle of the process:
// allocated on the first staged transfer and kept until the process exits
// (64 MB of pinned host memory).  Pinning took 16-56 ms and unpinning up to
// 1.2 s per pair on B200's host, too much to pay per handle.  One staged
// transfer at a time holds them (handles on other threads wait).
struct StagePool {
    std::mutex m;
    void* buf[2] = {nullptr, nullptr};
};

StagePool& stage_pool()
{
    static StagePool* p = new StagePool();   // never destroyed: outlives every handle
    return *p;
}

// with the pool's lock held: the buffers, and the handle's two events
void** ensure_stage(tmt_handle* h, StagePool& pool)
{
    for (int i = 0; i < 2; ++i) {
        if (!pool.buf[i]) {
            if (cudaHostAlloc(&pool.buf[i], kStageChunk, cudaHostAllocPortable) != cudaSuccess) {
                cudaGetLastError();
                pool.buf[i] = nullptr;
                throw OomError("pinned staging buffer allocation failed");
            }
        }
        if (!h->stage_ev[i]) CK(cudaEventCreateWithFlags(&h->stage_ev[i], cudaEventDisableTiming));
    }
    return pool.buf;
}

// Device -> host copy on the handle's stream, synchronous on return.  A
// destination CUDA knows (pinned, or device memory), or a small copy, takes
// one cudaMemcpyAsync; a large pageable one goes through the two pinned
// staging buffers, the device copy of a chunk overlapping the copy of the one
// before by 16 host threads.  Measured on B200's host, 808 MB into freshly
// mapped memory: 40-41 ms with 32 MB chunks (47-53 ms with 16 MB, 71-96 ms
// with 8 MB), against 370-380 ms for the driver's pageable path, which copies
// and takes the page faults on one thread (populating the pages with more
// threads beside the copies measured slower).
void d2h(tmt_handle* h, void* dst, const void* src, uint64_t bytes)
{
    if (!bytes) return;
    if (bytes < kStageChunk || cuda_visible(dst)) {
        CK(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDefault, h->stream));
        CK(cudaStreamSynchronize(h->stream));
        return;
    }
    StagePool& pool = stage_pool();
    std::lock_guard<std::mutex> lock(pool.m);
    void** stage = ensure_stage(h, pool);
    const uint64_t n = (bytes + kStageChunk - 1) / kStageChunk;
    auto len = [&](uint64_t c) { return std::min(kStageChunk, bytes - c * kStageChunk); };
    auto issue = [&](uint64_t c) {
        CK(cudaMemcpyAsync(stage[c & 1], static_cast<const char*>(src) + c * kStageChunk, len(c),
                           cudaMemcpyDeviceToHost, h->stream));
        CK(cudaEventRecord(h->stage_ev[c & 1], h->stream));
    };
    issue(0);
    for (uint64_t c = 0; c < n; ++c) {
        // buffer (c+1)&1 last held chunk c-1, whose host copy has finished
        if (c + 1 < n) issue(c + 1);
        CK(cudaEventSynchronize(h->stage_ev[c & 1]));
        host_copy_parallel(static_cast<char*>(dst) + c * kStageChunk, static_cast<const char*>(stage[c & 1]), len(c));
    }
}

// Host -> device copy ordered on the handle's stream.  A source CUDA knows
// (pinned, or device memory), or a small copy, takes one cudaMemcpyAsync; a
// large pageable one is copied by 16 host threads into the two pinned
// staging buffers, each chunk's device copy overlapping the host copy of the
// next (808 MB: 24 ms against 77 ms for the driver's pageable path, measured
// on B200's host).  On return the source has been read and, for a staged copy,
// the device copies have finished (the buffers are free for the next user).
void h2d(tmt_handle* h, void* dst, const void* src, uint64_t bytes)
{
    if (!bytes) return;
    if (bytes < kStageChunk || cuda_visible(src)) {
        CK(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDefault, h->stream));
        return;
    }
    StagePool& pool = stage_pool();
    std::lock_guard<std::mutex> lock(pool.m);
    void** stage = ensure_stage(h, pool);
    const uint64_t n = (bytes + kStageChunk - 1) / kStageChunk;
    for (uint64_t c = 0; c < n; ++c) {
        const uint64_t len = std::min(kStageChunk, bytes - c * kStageChunk);
        // the buffer's previous device copy (chunk c-2) has finished
        if (c >= 2) CK(cudaEventSynchronize(h->stage_ev[c & 1]));
        host_copy_parallel(static_cast<char*>(stage[c & 1]), static_cast<const char*>(src) + c * kStageChunk, len);
        CK(cudaMemcpyAsync(static_cast<char*>(dst) + c * kStageChunk, stage[c & 1], len, cudaMemcpyHostToDevice,
                           h->stream));
        CK(cudaEventRecord(h->stage_ev[c & 1], h->stream));
    }
    CK(cudaEventSynchronize(h->stage_ev[(n - 1) & 1]));   // stream order: every chunk has landed
}

struct SweepShape {
    uint32_t warps;      // warps per block
    uint32_t smem;       // dynamic shared memory bytes
    uint32_t rowi_smem, dnk_smem;
    uint32_t row16;      // the rows in shared memory as 16-bit counts (ROW16 kernels)
};

// rowi_global: the document's count row stays in global memory (L1-cached),
// halving the shared memory of a warp (the occupancy variant)
// split: the launch samples split documents (phase 1): every warp gets a
// private row in shared memory whatever the variant, and the block the
// document's row and the step's merged changes (K <= kSplitMaxK keeps the
// block at kSweepWarps warps)
// row16: with rowi_global, the rows stay in shared memory as 16-bit counts
SweepShape sweep_shape(uint32_t K, bool weighted, bool rowi_global = false, bool split = false, bool row16 = false)
{
    const uint32_t KP = round4(K);
    const uint32_t budget = 200 * 1024;
    SweepShape s{};
    // weighted counts take n_k's deltas from the word deltas after the sweep
    // (k_dk_sum): 64-bit shared-memory atomics per token cost ~17 ms a sweep
    s.dnk_smem = !weighted && K <= 16384u;
    s.rowi_smem = K <= 8192 && !rowi_global;
    s.row16 = row16 && rowi_global && !weighted && !split && K <= 8192;
    const uint32_t per_warp = 4 * KP + ((s.rowi_smem || split) ? 4 * KP : 0) + (s.row16 ? 2 * KP : 0);
    // alpha (KP floats) ahead of the n_k deltas
    const uint32_t fixed = 4 * KP + (s.dnk_smem ? 4 * KP : 0) + (split ? 8 * KP : 0);
    uint32_t w = (budget - fixed) / per_warp;
    s.warps = std::max(1u, std::min((uint32_t)(s.row16 ? kRow16Warps : kSweepWarps), w));
    s.smem = fixed + s.warps * per_warp;
    return s;
}

template <int CH, int MINB, bool WT, bool SPLIT = false, bool PLAIN = false, bool ROW16 = false>
void launch_sweep_t(tmt_handle* h, const SweepArgs& a, const SweepShape& sh)
{
    auto kern = k_sweep_doc<CH, MINB, WT, SPLIT, PLAIN, ROW16>;
    // attribute and occupancy once per kernel and shared-memory size (the
    // shapes depend on K and on whether the launch splits documents), so a
    // captured sweep makes no such call; the attribute allows the largest shape
    int per_sm = 0;
    for (const auto& e : h->occ)
        if (e.kern == (const void*)kern && e.smem == sh.smem) per_sm = e.per_sm;
    if (per_sm == 0) {
        const uint32_t KP = round4(a.K);
        const uint32_t most = std::max(sh.smem, sweep_shape(a.K, WT, false, !WT && a.K <= kSplitMaxK).smem);
        CK(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)std::max(most, 4 * KP)));
        CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, sh.warps * 32, sh.smem));
        if (per_sm < 1) throw CudaError("sweep kernel does not fit on an SM");
        h->occ.push_back({ (const void*)kern, sh.smem, per_sm });
    }
    // a split document takes a block; the others a warp each
    const uint64_t n_long = SPLIT ? a.n_long : 0;
    const uint64_t docs = a.pos_end - a.pos_begin - n_long;
    uint32_t grid = (uint32_t)std::min<uint64_t>((uint64_t)per_sm * h->num_sms,
                                                 n_long + (docs + sh.warps - 1) / sh.warps);
    if (grid == 0) grid = 1;
    kern<<<grid, sh.warps * 32, sh.smem, h->stream>>>(a);
    launch_check(h);
}

// Variants (identical results, different speed): 0 = the document row in
// shared memory as 32-bit counts, 3 blocks/SM; 1 = the row as 16-bit counts
// in shared memory (5 warps a block, 5 blocks/SM) or, for documents of
// 65,536+ tokens, in global memory (4 blocks/SM).  (Measured and dropped:
// loading the next token's column into registers during the current token,
// 2 blocks/SM -- slower at every benchmark configuration once the per-token
// loads came off the chain, e.g. 20.5 vs 11.4 ms per group at k = 1000, and
// two of the tuner's sweeps spent on it; at K = 1000, the word's column
// read from L1 every token, 6 blocks/SM, and a per-warp shared-memory copy
// of it -- fewer instructions, slower sweeps.)
int sweep_variants_for(uint32_t K)
{
    return (round4(K) + 127) / 128 > 32 ? 1 : 2;
}

template <int CH, bool WT, bool PLAIN>
void launch_sweep_cp(tmt_handle* h, const SweepArgs& a, const SweepShape& sh, int variant)
{
    // split documents: integer counts, up to 4 blocks of four topics per lane
    constexpr bool kSplit = !WT && CH >= 1 && CH <= 4;
    if (kSplit && a.n_long > 0) {
        if (variant >= 1) launch_sweep_t<CH, 4, WT, kSplit, PLAIN>(h, a, sh);
        else launch_sweep_t<CH, 3, WT, kSplit, PLAIN>(h, a, sh);
        return;
    }
    if (variant >= 1) {
        if constexpr (!WT) {
            if (sh.row16) return launch_sweep_t<CH, 4, WT, false, PLAIN, true>(h, a, sh);
        }
        launch_sweep_t<CH, 4, WT, false, PLAIN>(h, a, sh);
    }
    else launch_sweep_t<CH, 3, WT, false, PLAIN>(h, a, sh);
}

// plain: the launch has none of the conditional's options (PLAIN kernels)
template <int CH, bool WT>
void launch_sweep_ch(tmt_handle* h, const SweepArgs& a, const SweepShape& sh, int variant, bool plain)
{
    if constexpr (!WT) {
        if (plain) return launch_sweep_cp<CH, false, true>(h, a, sh, variant);
    }
    launch_sweep_cp<CH, WT, false>(h, a, sh, variant);
}

template <bool WT>
void launch_sweep_w(tmt_handle* h, const SweepArgs& b, const SweepShape& sh, uint32_t ch, int variant, bool plain)
{
    if (ch <= 1) launch_sweep_ch<1, WT>(h, b, sh, variant, plain);
    else if (ch <= 2) launch_sweep_ch<2, WT>(h, b, sh, variant, plain);
    else if (ch <= 4) launch_sweep_ch<4, WT>(h, b, sh, variant, plain);
    else if (ch <= 8) launch_sweep_ch<8, WT>(h, b, sh, variant, plain);
    else if (ch <= 16) launch_sweep_ch<16, WT>(h, b, sh, variant, plain);
    else if (ch <= 32) launch_sweep_ch<32, WT>(h, b, sh, variant, plain);
    else launch_sweep_t<0, 3, WT>(h, b, sh);
}

void launch_sweep(tmt_handle* h, const SweepArgs& a, int variant)
{
    const uint32_t KP = round4(a.K);
    const uint32_t ch = (KP + 127) / 128;
    const bool wt = a.wt != nullptr;
    const bool split = !wt && a.n_long > 0;
    // 16-bit rows when every document of the launch is shorter than 65,536 tokens
    const SweepShape sh = sweep_shape(a.K, wt, variant >= 1, split, a.max_len < 65536);
    if (!wt && a.n_long > 0 && sh.warps != (uint32_t)kSweepWarps)
        throw CudaError("split documents need a block of " + std::to_string(kSweepWarps) + " warps");
    SweepArgs b = a;
    b.rowi_smem = sh.rowi_smem;
    b.dnk_smem = sh.dnk_smem;
    // plain LDA: none of the conditional's options (results are the same either way)
    const bool plain = !wt && !a.pr.idx && !a.arow && !a.mask && a.rm1 && sh.dnk_smem;
    if (wt) launch_sweep_w<true>(h, b, sh, ch, variant, false);
    else launch_sweep_w<false>(h, b, sh, ch, variant, plain);
}

// The variant of group g: the one being tuned, else the group's fastest.
int variant_of(const tmt_handle* h, uint32_t g)
{
    return h->tuned < 0 ? h->variant : h->group_variant[g];
}

// Tuning sweeps time each group's sweep kernel with its own event pair.
void tune_mark(tmt_handle* h, uint32_t g, int end)
{
    if (h->tuned < 0) CK(cudaEventRecord(h->gev[2 * g + end], h->stream));
}

// In-place SUM over the ranks of a sharded corpus, ordered on the engine's stream.
void exchange(tmt_handle* h, void* buf, uint64_t count, int32_t dtype)
{
    if (h->world <= 1) return;
    const int32_t rc = h->allreduce(h->ar_user, buf, count, dtype, (void*)h->stream);
    if (rc != 0) throw CudaError("allreduce across ranks failed (" + std::to_string(rc) + ")");
}

// The launch arguments of document group g.
SweepArgs sweep_args(tmt_handle* h, const int32_t* nkw, const int32_t* nk, int32_t* nkw_next, int32_t* nk_next,
                     uint32_t g)
{
    const uint64_t pos_begin = h->group_bounds[g], pos_end = h->group_bounds[g + 1];
    SweepArgs a{};
    a.doc_off = h->d_doc_off;
    a.words = h->d_words;
    a.z = h->d_z;
    a.ndk = h->d_ndk;
    a.nkw = nkw;
    a.nk = nk;
    a.phi = h->d_phi;
    a.nkw_next = nkw_next;
    a.nk_next = nk_next;
    a.alpha = h->d_alpha;
    a.doc_order = h->d_doc_order;
    a.doc_counter = h->d_counter;
    a.D = h->D;
    a.K = h->cfg.K;
    a.V = h->cfg.V;
    a.c = (h->cfg.K + 31) / 32;
    {
        const uint32_t lanes = std::min<uint32_t>(32, (h->cfg.K + 3) / 4);
        uint32_t st = 0;
        while ((1u << st) < lanes) ++st;
        a.scan_steps = st;
    }
    a.eta = h->cfg.eta;
    a.veta = h->cfg.eta * (float)h->cfg.V;
    a.seed = h->cfg.seed;
    a.iter = (uint32_t)h->global_step;
    a.pos_begin = pos_begin;
    a.pos_end = pos_end;
    a.tok_offset = h->tok_offset;
    a.pr = h->prior_args();
    a.rm1 = h->weighted ? nullptr : h->d_rm1;
    a.alpha_rows = h->d_alpha_rows;
    a.arow = h->d_arow;
    a.mask = h->d_mask;
    a.mw = (h->cfg.K + 31) / 32;
    a.n_long = (h->weighted || h->n_rows) ? 0 : h->group_nlong[g];
    a.max_len = pos_end > pos_begin ? h->order_len[pos_begin] : 0;    // longest first
    a.unit_off = h->n_rows ? h->d_unit_off : nullptr;
    a.unit_docs = h->n_rows ? h->d_unit_docs : nullptr;
    a.split_step = h->split_step;
    a.long_counter = h->d_counter + 1;
    return a;
}

// A sweep of one rank of a sharded corpus: per group, the word table of the
// current (summed) state, this rank's documents of the group with their count
// deltas into d_delta, the SUM of the deltas over the ranks, and the fold of
// the summed deltas into the state (fused with the next group's table).  Every
// rank runs every group that holds documents on any rank, so the collectives
// match; n_kw is updated in place (h->cur stays 0).
void do_sweep_sharded(tmt_handle* h)
{
    const uint32_t K = h->cfg.K, V = h->cfg.V;
    const float veta = h->cfg.eta * (float)V;
    const uint64_t KV = (uint64_t)K * V;
    int32_t* dnkw = h->d_delta;
    int32_t* dnk = h->d_delta + KV;
    const uint32_t smem_k = K <= 12288 ? K : 0;
    const uint32_t grid = (uint32_t)std::max<uint64_t>(1, std::min<uint64_t>((uint64_t)h->num_sms * 16, V));
    bool pending = false, recorded = false;
    const uint32_t G = (uint32_t)h->group_bounds.size() - 1;
    for (uint32_t g = 0; g < G; ++g) {
        if (h->gbounds[g] == h->gbounds[g + 1]) continue;      // empty on every rank
        if (!recorded) { CK(cudaEventRecord(h->kev0, h->stream)); recorded = true; }
        if (pending) {
            k_nk_apply<<<1, 1024, 0, h->stream>>>(h->d_nk[0], dnk, K);
            launch_check(h);
        }
        k_phi_apply<<<grid, 256, smem_k * 4, h->stream>>>(h->d_nkw[0], dnkw, h->d_nk[0], V, K, round4(K), h->cfg.eta,
                                                        veta, h->d_phi, smem_k, pending ? 1 : 0, h->prior_args(),
                                                        h->d_rm1);
        launch_check(h);
        if (h->group_bounds[g] < h->group_bounds[g + 1]) {
            CK(cudaMemsetAsync(h->d_counter, 0, 2 * sizeof(uint32_t), h->stream));
            tune_mark(h, g, 0);
            launch_sweep(h, sweep_args(h, h->d_nkw[0], h->d_nk[0], dnkw, dnk, g), variant_of(h, g));
            tune_mark(h, g, 1);
        }
        exchange(h, h->d_delta, KV + K, TMT_I32);
        pending = true;
    }
    if (pending) {
        k_nk_apply<<<1, 1024, 0, h->stream>>>(h->d_nk[0], dnk, K);
        launch_check(h);
        k_phi_apply<<<grid, 256, 0, h->stream>>>(h->d_nkw[0], dnkw, h->d_nk[0], V, K, round4(K), h->cfg.eta, veta,
                                                nullptr, 0, 1, h->prior_args(), nullptr);
        launch_check(h);
    }
    CK(cudaEventRecord(h->kev1, h->stream));
    if (!recorded) CK(cudaEventRecord(h->kev0, h->stream));
    h->sampler_used = TMT_SAMPLER_DENSE;
}

// A sweep with weighted counts: per group, fold the previous group's deltas
// into the float state (n_k first, then n_kw fused with the word table of the
// new state), then the group's documents with their deltas going to
// d_dkw / d_dk; after the last group, a final fold.  The state is updated in
// place (h->cur stays 0).
void do_sweep_w(tmt_handle* h, bool capture)
{
    const uint32_t K = h->cfg.K, V = h->cfg.V;
    const float veta = h->cfg.eta * (float)V;
    float* nkw = reinterpret_cast<float*>(h->d_nkw[0]);
    float* nk = reinterpret_cast<float*>(h->d_nk[0]);
    const uint32_t smem_k = K <= 12288 ? K : 0;
    const uint32_t grid = (uint32_t)std::max<uint64_t>(1, std::min<uint64_t>((uint64_t)h->num_sms * 16, V));
    bool pending = false, recorded = false;
    // n_k's deltas of the group just sampled, then its fold
    const uint32_t gx = (K + 255) / 256;
    const uint32_t gy = (uint32_t)std::max<uint64_t>(1, std::min<uint64_t>((V + 63) / 64,
                                                                          (uint64_t)h->num_sms * 8 / gx + 1));
    const uint32_t rows = (V + gy - 1) / gy;
    auto fold_nk = [&] {
        k_dk_sum<<<dim3(gx, gy), 256, 0, h->stream>>>(h->d_dkw, V, K, rows, h->d_dk);
        launch_check(h);
        k_nk_fold_w<<<1, 1024, 0, h->stream>>>(nk, h->d_dk, K);
        launch_check(h);
    };
    const uint32_t G = (uint32_t)h->group_bounds.size() - 1;
    for (uint32_t g = 0; g < G; ++g) {
        if (h->group_bounds[g] == h->group_bounds[g + 1]) continue;
        if (pending) fold_nk();
        k_phi_fold_w<<<grid, 256, smem_k * 4, h->stream>>>(nkw, h->d_dkw, nk, V, K, round4(K), h->cfg.eta, veta,
                                                         h->d_phi, smem_k, pending ? 1 : 0, h->prior_args());
        launch_check(h);
        CK(cudaMemsetAsync(h->d_counter, 0, 2 * sizeof(uint32_t), h->stream));
        SweepArgs a = sweep_args(h, h->d_nkw[0], h->d_nk[0], nullptr, nullptr, g);
        a.wt = h->d_wt;
        a.dkw = h->d_dkw;
        a.dk = h->d_dk;
        if (capture) a.iter_ptr = h->d_step;
        if (!capture) {
            if (!recorded) { CK(cudaEventRecord(h->kev0, h->stream)); recorded = true; }
            tune_mark(h, g, 0);
        }
        launch_sweep(h, a, variant_of(h, g));
        if (!capture) tune_mark(h, g, 1);
        pending = true;
    }
    if (pending) {
        fold_nk();
        k_phi_fold_w<<<grid, 256, 0, h->stream>>>(nkw, h->d_dkw, nk, V, K, round4(K), h->cfg.eta, veta, nullptr, 0, 1,
                                                 h->prior_args());
        launch_check(h);
    }
    if (!capture) {
        CK(cudaEventRecord(h->kev1, h->stream));
        if (!recorded) CK(cudaEventRecord(h->kev0, h->stream));
    }
    h->sampler_used = TMT_SAMPLER_DENSE;
}

// One sweep = one launch per document group (contiguous ranges of the
// longest-first order holding equal shares of the tokens); before each, the
// word table and the next-state copy are rebuilt from the current state.
// capture: the launches are being recorded into a graph (no timing events;
// the draws read the sweep counter from d_step).
void do_sweep(tmt_handle* h, bool capture = false)
{
    if (h->world > 1) return do_sweep_sharded(h);
    if (h->weighted) return do_sweep_w(h, capture);
    const uint32_t K = h->cfg.K, V = h->cfg.V;
    const float veta = h->cfg.eta * (float)V;
    bool recorded = false;
    const uint32_t G = (uint32_t)h->group_bounds.size() - 1;
    for (uint32_t g = 0; g < G; ++g) {
        if (h->group_bounds[g] == h->group_bounds[g + 1]) continue;
        const int cur = h->cur, nxt = cur ^ 1;
        const uint32_t smem_k = K <= 12288 ? K : 0;
        uint32_t grid = (uint32_t)std::max<uint64_t>(1, std::min<uint64_t>((uint64_t)h->num_sms * 16, V));
        k_phi_copy<<<grid, 256, smem_k * 4, h->stream>>>(h->d_nkw[cur], h->d_nk[cur], V, K, round4(K), h->cfg.eta,
                                                        veta, h->d_phi, h->d_nkw[nxt], h->d_nk[nxt], smem_k,
                                                        h->prior_args(), h->d_rm1);
        launch_check(h);
        CK(cudaMemsetAsync(h->d_counter, 0, 2 * sizeof(uint32_t), h->stream));
        SweepArgs a = sweep_args(h, h->d_nkw[cur], h->d_nk[cur], h->d_nkw[nxt], h->d_nk[nxt], g);
        if (capture) a.iter_ptr = h->d_step;
        if (!capture) {
            if (!recorded) { CK(cudaEventRecord(h->kev0, h->stream)); recorded = true; }
            tune_mark(h, g, 0);
        }
        launch_sweep(h, a, variant_of(h, g));
        if (!capture) tune_mark(h, g, 1);
        h->cur = nxt;
    }
    if (!capture) {
        CK(cudaEventRecord(h->kev1, h->stream));
        if (!recorded) CK(cudaEventRecord(h->kev0, h->stream));
    }
    h->sampler_used = TMT_SAMPLER_DENSE;
}

// One sweep as a graph launch: the sweep's launches are captured once per
// starting buffer parity (after the autotuner has fixed every group's
// variant) and replayed; the last node advances the device sweep counter.
void graph_sweep(tmt_handle* h)
{
    const int p = h->cur;
    if (!h->graph_exec[p]) {
        const int cur0 = h->cur;
        const uint64_t l0 = h->launches;
        cudaGraph_t g = nullptr;
        CK(cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal));
        try {
            do_sweep(h, true);
            k_next_step<<<1, 1, 0, h->stream>>>(h->d_step);
            launch_check(h);
        } catch (...) {
            cudaStreamEndCapture(h->stream, &g);
            if (g) cudaGraphDestroy(g);
            cudaGetLastError();
            h->cur = cur0;
            h->launches = l0;
            throw;
        }
        CK(cudaStreamEndCapture(h->stream, &g));
        h->graph_kernels = h->launches - l0;
        h->launches = l0;
        h->graph_flip = h->cur ^ cur0;
        h->cur = cur0;
        const cudaError_t e = cudaGraphInstantiate(&h->graph_exec[p], g, 0);
        cudaGraphDestroy(g);
        if (e != cudaSuccess) {
            h->graph_exec[p] = nullptr;
            throw CudaError(std::string("cudaGraphInstantiate: ") + cudaGetErrorString(e));
        }
    }
    CK(cudaGraphLaunch(h->graph_exec[p], h->stream));
    h->launches += h->graph_kernels;
    h->cur ^= h->graph_flip;
    h->sampler_used = TMT_SAMPLER_DENSE;
}

void do_optimize(tmt_handle* h)
{
    const uint32_t K = h->cfg.K;
    dim3 grid(h->n_apart, (K + 255) / 256);
    k_sum_alpha<<<1, 32, 0, h->stream>>>(h->d_alpha, K, h->d_asum);
    launch_check(h);
    for (int it = 0; it < 10; ++it) {
        if (h->weighted)
            k_alpha_sums<<<grid, 256, 0, h->stream>>>(reinterpret_cast<const float*>(h->d_ndk), h->D, K, h->d_alpha,
                                                      (const float*)h->d_doc_wlen, h->d_asum, h->d_part_nom,
                                                      h->d_part_den);
        else
            k_alpha_sums<<<grid, 256, 0, h->stream>>>(h->d_ndk, h->n_rows ? h->n_rows : h->D, K, h->d_alpha,
                                                      h->d_doc_len, h->d_asum, h->d_part_nom, h->d_part_den);
        launch_check(h);
        uint32_t nparts = h->n_apart;
        const double* nom = h->d_part_nom;
        const double* den = h->d_part_den;
        if (h->world > 1) {
            // this rank's sums into one row (K digamma sums, then the length sum), summed over the ranks
            k_alpha_fold<<<(K + 256) / 256, 256, 0, h->stream>>>(h->d_part_nom, h->d_part_den, h->n_apart, K,
                                                                 h->d_alpha_fold);
            launch_check(h);
            exchange(h, h->d_alpha_fold, (uint64_t)K + 1, TMT_F64);
            nparts = 1;
            nom = h->d_alpha_fold;
            den = h->d_alpha_fold + K;
        }
        k_alpha_update<<<1, 1024, 0, h->stream>>>(nom, den, nparts, K, h->n_rows ? h->n_rows : h->D_global,
                                                  h->d_alpha, h->d_asum, h->d_dg_points);
        launch_check(h);
    }
}

// FP64 ll into d_out[0..1]; alpha read from the device copy.
// FP64 ll into d_out[0..1] (docs, rest); stream-ordered, no host sync.
void do_ll(tmt_handle* h, double* d_out)
{
    const uint32_t K = h->cfg.K;
    const double eta = (double)h->cfg.eta;
    const double veta = (double)h->cfg.V * eta;
    k_ll_prep<<<1, 256, 0, h->stream>>>(h->d_alpha, K, h->d_lg_alpha, h->d_asum_ll);
    launch_check(h);
    if (h->weighted) {
        k_ll_partials<<<h->n_partials, 256, 0, h->stream>>>(
            reinterpret_cast<const float*>(h->d_ndk), h->D, K, h->d_lg_alpha, h->d_alpha, (const float*)h->d_doc_wlen,
            h->d_asum_ll, reinterpret_cast<const float*>(h->d_nkw[0]), h->cfg.V, eta, std::lgamma(eta), h->d_partials,
            h->prior_args(), h->d_alpha_rows, h->d_arow, h->d_row_asum);
        launch_check(h);
        k_ll_final<<<1, 256, 0, h->stream>>>(h->d_partials, h->n_partials, reinterpret_cast<const float*>(h->d_nk[0]),
                                             K, veta, d_out, h->d_esum);
    } else {
        k_ll_partials<<<h->n_partials, 256, 0, h->stream>>>(h->d_ndk, h->n_rows ? h->n_rows : h->D, K,
                                                            h->d_lg_alpha, h->d_alpha,
                                                            h->d_doc_len, h->d_asum_ll,
                                                            h->d_nkw[h->cur], h->cfg.V, eta, std::lgamma(eta),
                                                            h->d_partials, h->prior_args(), h->d_alpha_rows,
                                                            h->d_arow, h->d_row_asum);
        launch_check(h);
        k_ll_final<<<1, 256, 0, h->stream>>>(h->d_partials, h->n_partials, h->d_nk[h->cur], K, veta, d_out,
                                             h->d_esum);
    }
    launch_check(h);
    exchange(h, d_out, 1, TMT_F64);     // LLDocs over every rank's documents; LLRest is replicated
}

// The document order and groups of a (possibly sharded) corpus: documents
// longest first (stable), cut into G ranges holding equal shares of the
// tokens -- position p is in group g when prefix(p) * G lies in
// [g * total, (g+1) * total).  The rank's documents keep that order.
struct ShardPlan {
    std::vector<uint32_t> order;        // local document indices, global order
    std::vector<uint64_t> bounds;       // group g = order[bounds[g] .. bounds[g+1])
    std::vector<uint64_t> gbounds;      // group g holds global positions [gbounds[g], gbounds[g+1])
    std::vector<uint64_t> gtokens;      // group g's tokens over all ranks
    uint64_t tok_offset = 0;
};

ShardPlan plan_shard(const uint64_t* len, uint64_t D_global, uint32_t groups, uint64_t doc_begin, uint64_t D_local)
{
    if (doc_begin > D_global || D_local > D_global - doc_begin) throw ArgError("shard outside the corpus");
    ShardPlan p;
    std::vector<uint64_t> gorder(D_global);
    uint64_t longest = 0;
    for (uint64_t d = 0; d < D_global; ++d) longest = std::max(longest, len[d]);
    if (longest <= 4 * D_global + 65536) {
        // stable counting sort on (longest - len): the order std::stable_sort
        // by descending length gives, in O(D + longest)
        std::vector<uint64_t> start(longest + 2, 0);
        for (uint64_t d = 0; d < D_global; ++d) ++start[longest - len[d] + 1];
        for (uint64_t b = 1; b <= longest + 1; ++b) start[b] += start[b - 1];
        for (uint64_t d = 0; d < D_global; ++d) gorder[start[longest - len[d]]++] = d;
    } else {
        std::iota(gorder.begin(), gorder.end(), (uint64_t)0);
        std::stable_sort(gorder.begin(), gorder.end(), [&](uint64_t a, uint64_t b) { return len[a] > len[b]; });
    }
    uint64_t total = 0;
    for (uint64_t d = 0; d < D_global; ++d) {
        total += len[d];
        if (d < doc_begin) p.tok_offset += len[d];
    }
    const uint64_t G = std::max<uint32_t>(1, groups);
    p.gbounds.assign(G + 1, 0);
    p.gbounds[G] = D_global;
    p.bounds.assign(G + 1, 0);
    p.order.reserve(D_local);
    p.gtokens.assign(G, 0);
    uint64_t prefix = 0, g = 1;
    for (uint64_t q = 0; q < D_global; ++q) {
        while (g < G && prefix * G >= g * total) {
            p.gbounds[g] = q;
            p.bounds[g] = p.order.size();
            ++g;
        }
        const uint64_t d = gorder[q];
        if (d >= doc_begin && d - doc_begin < D_local) p.order.push_back((uint32_t)(d - doc_begin));
        prefix += len[d];
        p.gtokens[g - 1] += len[d];
    }
    for (; g < G; ++g) {
        p.gbounds[g] = D_global;
        p.bounds[g] = p.order.size();
    }
    p.bounds[G] = p.order.size();
    return p;
}

// Per document group, how many of its first (longest) local documents are
// split: those of at least the group's split_len tokens (split_len_of over the
// global group's tokens, so every rank of a sharded corpus agrees).
void update_split(tmt_handle* h)
{
    if (h->group_bounds.empty()) return;
    const uint32_t G = (uint32_t)h->group_bounds.size() - 1;
    h->group_nlong.assign(G, 0);
    if (h->weighted || h->n_rows) return;
    for (uint32_t g = 0; g < G; ++g) {
        const uint64_t sl = split_len_of(h->group_tokens[g], h->cfg.K, h->split_min, h->split_step);
        if (!sl) continue;
        uint32_t n = 0;
        for (uint64_t q = h->group_bounds[g]; q < h->group_bounds[g + 1] && h->order_len[q] >= sl; ++q) ++n;
        h->group_nlong[g] = n;
    }
}

void validate_config(const tmt_config& c)
{
    if (c.K == 0 || c.K > 32767) throw ArgError("wrong K value (K = " + std::to_string(c.K) + ")");
    if (!(c.eta > 0)) throw ArgError("wrong eta value (eta = " + std::to_string(c.eta) + ")");
    if (c.alpha) {
        for (uint32_t k = 0; k < c.K; ++k)
            if (!(c.alpha[k] > 0)) throw ArgError("wrong alpha value");
    } else if (!(c.alpha_scalar > 0)) {
        throw ArgError("wrong alpha value");
    }
    if (c.sampler < TMT_SAMPLER_AUTO || c.sampler > TMT_SAMPLER_SPARSE) throw ArgError("unknown sampler");
}

} // namespace

// ---------------------------------------------------------------------------
// C ABI
// ---------------------------------------------------------------------------
namespace {

tmt_status upload_impl(tmt_handle* h, const uint32_t* wid, const uint64_t* doc_off, uint64_t D, const uint16_t* z0,
                       const tmt_shard* shard, const float* weights = nullptr)
{
    if (!h) return TMT_ERR_INVALID_ARGUMENT;
    return guarded(h, [&] {
        if (!doc_off) throw ArgError("doc_off is NULL");
        if (D >= 0xFFFFFFFFull) throw ArgError("too many documents");
        const uint64_t n_all = doc_off[D];
        if (n_all && !wid) throw ArgError("wid is NULL");
        for (uint64_t d = 0; d < D; ++d)
            if (doc_off[d + 1] < doc_off[d]) throw ArgError("doc_off is not non-decreasing");
        const uint32_t K = h->cfg.K, V = h->cfg.V;
        if (z0) {
            for (uint64_t i = 0; i < n_all; ++i)
                if (wid[i] < V && z0[i] >= K) throw ArgError("z0 holds a topic id >= K");
        }
        if (weights) {
            // the deltas are int64 in units of 2^-24: the weights of all tokens
            // together stay below 2^38 so no sum can overflow
            if (shard && shard->world > 1) throw ArgError("weighted counts on a corpus sharded across GPUs are not supported");
            double total = 0;
            for (uint64_t i = 0; i < n_all; ++i) {
                if (wid[i] >= V) continue;
                const float w = weights[i];
                if (!(w >= 0.f) || !(w <= 65536.f))
                    throw ArgError("token weight " + std::to_string(i) + " is negative, too large or not finite");
                total += (double)w;
            }
            if (total >= 274877906944.0) throw ArgError("the token weights sum to 2^38 or more");
        }
        h->release();
        h->uploaded = false;
        h->D = D;
        h->N_all = n_all;
        h->global_step = 0;
        h->cur = 0;
        // valid-token count per document: counted on the host for weighted
        // counts (the planner's facts are uploaded), else N is read back from
        // the device's n_k after the counts kernel
        std::vector<int32_t> len;
        uint64_t N = 0;
        if (weights) {
            len.resize(D);
            for (uint64_t d = 0; d < D; ++d) {
                int32_t c = 0;
                for (uint64_t i = doc_off[d]; i < doc_off[d + 1]; ++i) c += wid[i] < V;
                len[d] = c;
                N += c;
            }
        }
        h->N = N;
        ShardPlan plan;
        if (shard) {
            if (shard->world == 0 || shard->rank >= shard->world) throw ArgError("bad rank / world");
            if (shard->world > 1 && !shard->allreduce) throw ArgError("a sharded corpus needs an allreduce");
            if (!shard->doc_len_global && shard->D_global) throw ArgError("doc_len_global is NULL");
            if (shard->doc_begin > shard->D_global || D > shard->D_global - shard->doc_begin)
                throw ArgError("shard outside the corpus");
            for (uint64_t d = 0; d < D; ++d)
                if (shard->doc_len_global[shard->doc_begin + d] != doc_off[d + 1] - doc_off[d])
                    throw ArgError("doc_len_global disagrees with doc_off at document " + std::to_string(d));
            plan = plan_shard(shard->doc_len_global, shard->D_global, h->groups, shard->doc_begin, D);
            h->rank = shard->rank;
            h->world = shard->world;
            h->D_global = shard->D_global;
            h->allreduce = shard->allreduce;
            h->ar_user = shard->user;
        } else {
            std::vector<uint64_t> lens(D);
            for (uint64_t d = 0; d < D; ++d) lens[d] = doc_off[d + 1] - doc_off[d];
            plan = plan_shard(lens.data(), D, h->groups, 0, D);
            h->rank = 0;
            h->world = 1;
            h->D_global = D;
            h->allreduce = nullptr;
            h->ar_user = nullptr;
        }
        h->weighted = weights != nullptr;
        h->n_rows = 0;
        h->row_cap = D;
        h->unit_cap = 0;
        h->d_unit_off = nullptr;
        h->d_unit_docs = nullptr;
        h->d_row_of = nullptr;
        h->tok_offset = plan.tok_offset;
        h->group_bounds = plan.bounds;
        h->gbounds = plan.gbounds;
        h->group_tokens = plan.gtokens;
        const std::vector<uint32_t>& order = plan.order;
        h->order_len.resize(D);
        for (uint64_t q = 0; q < D; ++q) h->order_len[q] = doc_off[order[q] + 1] - doc_off[order[q]];
        update_split(h);

        h->d_doc_off = h->dalloc<uint64_t>(D + 1);
        h->d_words = h->dalloc<uint32_t>(n_all);
        h->d_z = h->dalloc<uint16_t>(n_all);
        h->d_ndk = h->dalloc<int32_t>(D * (uint64_t)K);
        h->d_nkw[0] = h->dalloc<int32_t>((uint64_t)K * V);
        h->d_nk[0] = h->dalloc<int32_t>(K);
        if (h->world > 1) {
            // the next-state buffers become one exchanged delta buffer
            h->d_delta = h->dalloc<int32_t>((uint64_t)K * V + K);
            h->d_nkw[1] = h->d_delta;
            h->d_nk[1] = h->d_delta + (uint64_t)K * V;
            h->d_alpha_fold = h->dalloc<double>((uint64_t)K + 1);
        } else if (h->weighted) {
            // the float state is updated in place; the deltas are int64
            h->d_delta = nullptr;
            h->d_alpha_fold = nullptr;
            h->d_nkw[1] = nullptr;
            h->d_nk[1] = nullptr;
            h->d_wt = h->dalloc<float>(n_all);
            h->d_dkw = h->dalloc<long long>((uint64_t)K * V);
            h->d_dk = h->dalloc<long long>(K);
            h->d_doc_wlen = h->dalloc<float>(D);
        } else {
            h->d_delta = nullptr;
            h->d_alpha_fold = nullptr;
            h->d_nkw[1] = h->dalloc<int32_t>((uint64_t)K * V);
            h->d_nk[1] = h->dalloc<int32_t>(K);
        }
        h->d_phi = h->dalloc<float>((uint64_t)round4(K) * V);
        h->d_rm1 = h->dalloc<float>(K);
        h->d_prior_idx = nullptr;
        h->d_prior = h->d_esum = h->d_prior_cum = h->d_cum_eta = nullptr;
        h->d_alpha_rows = nullptr;
        h->d_arow = nullptr;
        h->d_row_asum = nullptr;
        h->d_mask = nullptr;
        if (!h->prior_ids.empty()) {
            // etaByTopicWord as a sparse table (prepareWordPriors, LDAModel.hpp:724-737)
            const uint32_t P = (uint32_t)h->prior_ids.size();
            PriorTables t;
            build_prior_tables(K, V, h->cfg.eta, h->prior_ids, h->prior_vals, t);
            const std::vector<int32_t>& idx = t.idx;
            const std::vector<float>& esum = t.esum;
            const std::vector<float>& pcum = t.pcum;
            const std::vector<float>& ecum = t.ecum;
            h->d_prior_idx = h->dalloc<int32_t>(V);
            h->d_prior = h->dalloc<float>((uint64_t)P * K);
            h->d_esum = h->dalloc<float>(K);
            h->d_prior_cum = h->dalloc<float>((uint64_t)P * K);
            h->d_cum_eta = h->dalloc<float>(K);
            cudaStream_t s0 = h->stream;
            CK(cudaMemcpyAsync(h->d_prior_idx, idx.data(), V * sizeof(int32_t), cudaMemcpyHostToDevice, s0));
            CK(cudaMemcpyAsync(h->d_prior, h->prior_vals.data(), (uint64_t)P * K * sizeof(float), cudaMemcpyHostToDevice, s0));
            CK(cudaMemcpyAsync(h->d_esum, esum.data(), K * sizeof(float), cudaMemcpyHostToDevice, s0));
            CK(cudaMemcpyAsync(h->d_prior_cum, pcum.data(), (uint64_t)P * K * sizeof(float), cudaMemcpyHostToDevice, s0));
            CK(cudaMemcpyAsync(h->d_cum_eta, ecum.data(), K * sizeof(float), cudaMemcpyHostToDevice, s0));
            CK(cudaStreamSynchronize(s0));
        }
        {
            // the first 2 n_variants sweeps run eagerly, the variants in the
            // order 0 .. n-1, n-1 .. 0, and every group keeps its fastest
            const uint32_t G = (uint32_t)h->group_bounds.size() - 1;
            h->n_variants = sweep_variants_for(K);
            h->variant = 0;
            h->tune_step = 0;
            h->tuned = -1;
            h->group_variant.assign(G, 0);
            h->group_ms.assign(G, std::vector<float>(h->n_variants, 0.f));
            while (h->gev.size() < 2 * (size_t)G) {
                cudaEvent_t e;
                CK(cudaEventCreate(&e));
                h->gev.push_back(e);
            }
            h->d_step = h->dalloc<uint32_t>(1);
        }
        h->d_doc_len = h->dalloc<int32_t>(D);
        h->d_doc_order = h->dalloc<uint32_t>(D);
        h->d_counter = h->dalloc<uint32_t>(2);      // phase 2's (warp) and phase 1's (block) document counters
        h->d_alpha = h->dalloc<float>(K);
        h->d_asum = h->dalloc<float>(1);
        h->d_lg_alpha = h->dalloc<double>(K);
        h->d_asum_ll = h->dalloc<double>(2);
        h->d_llv = h->dalloc<double>(2);
        h->n_partials = ll_blocks(h->num_sms);
        h->d_partials = h->dalloc<double>(2 * (size_t)h->n_partials);
        h->ll_cap = 0;
        h->d_ll = nullptr;
        const std::vector<float>& dg = tmt::digamma_points();
        h->d_dg_points = h->dalloc<float>(dg.size());
        h->n_apart = (uint32_t)std::max<uint64_t>(1, std::min<uint64_t>((uint64_t)h->num_sms * 4, (D + 63) / 64));
        h->d_part_nom = h->dalloc<double>((size_t)h->n_apart * K);
        h->d_part_den = h->dalloc<double>(h->n_apart);

        cudaStream_t st = h->stream;
        CK(cudaMemcpyAsync(h->d_doc_off, doc_off, (D + 1) * sizeof(uint64_t), cudaMemcpyHostToDevice, st));
        h2d(h, h->d_words, wid, n_all * sizeof(uint32_t));
        CK(cudaMemcpyAsync(h->d_doc_order, order.data(), D * sizeof(uint32_t), cudaMemcpyHostToDevice, st));
        CK(cudaMemcpyAsync(h->d_alpha, h->alpha.data(), K * sizeof(float), cudaMemcpyHostToDevice, st));
        CK(cudaMemcpyAsync(h->d_dg_points, dg.data(), dg.size() * sizeof(float), cudaMemcpyHostToDevice, st));
        CK(cudaMemsetAsync(h->d_ndk, 0, D * (uint64_t)K * sizeof(int32_t), st));
        CK(cudaMemsetAsync(h->d_nkw[0], 0, (uint64_t)K * V * sizeof(int32_t), st));
        CK(cudaMemsetAsync(h->d_nk[0], 0, K * sizeof(int32_t), st));
        if (z0) {
            h2d(h, h->d_z, z0, n_all * sizeof(uint16_t));
        } else if (n_all) {
            std::vector<float> acum(K);
            float s = 0.f;
            for (uint32_t k = 0; k < K; ++k) { s = s + h->alpha[k]; acum[k] = s; }
            float* d_acum = h->dalloc<float>(K);
            CK(cudaMemcpyAsync(d_acum, acum.data(), K * sizeof(float), cudaMemcpyHostToDevice, st));
            uint32_t grid = (uint32_t)std::min<uint64_t>((uint64_t)h->num_sms * 16, (n_all + 255) / 256);
            k_init_z<<<grid, 256, 0, st>>>(h->d_words, n_all, V, K, d_acum, h->cfg.seed, h->tok_offset, h->d_z,
                                           h->d_prior_idx, h->d_prior_cum, h->d_cum_eta);
            launch_check(h);
        }
        if (D && h->weighted) {
            h2d(h, h->d_wt, weights, n_all * sizeof(float));
            CK(cudaMemsetAsync(h->d_dkw, 0, (uint64_t)K * V * sizeof(long long), st));
            CK(cudaMemsetAsync(h->d_dk, 0, K * sizeof(long long), st));
            uint32_t grid = (uint32_t)std::min<uint64_t>((uint64_t)h->num_sms * 16, (D + 127) / 128);
            const bool dk_smem = K <= 4096;     // at most 32 KB of shared memory
            k_counts_w<<<grid, 128, dk_smem ? K * sizeof(long long) : 0, st>>>(
                h->d_doc_off, h->d_words, h->d_z, h->d_wt, D, K, V, reinterpret_cast<float*>(h->d_ndk), h->d_dkw,
                h->d_dk, h->d_doc_wlen, dk_smem);
            launch_check(h);
            k_nk_fold_w<<<1, 1024, 0, st>>>(reinterpret_cast<float*>(h->d_nk[0]), h->d_dk, K);
            launch_check(h);
            const uint32_t g2 = (uint32_t)std::max<uint64_t>(1, std::min<uint64_t>((uint64_t)h->num_sms * 16, V));
            k_phi_fold_w<<<g2, 256, 0, st>>>(reinterpret_cast<float*>(h->d_nkw[0]), h->d_dkw,
                                             reinterpret_cast<const float*>(h->d_nk[0]), V, K, round4(K), h->cfg.eta,
                                             h->cfg.eta * (float)V, nullptr, 0, 1, h->prior_args());
            launch_check(h);
            // the token counts per document as well (the shard planner's facts)
            CK(cudaMemcpyAsync(h->d_doc_len, len.data(), D * sizeof(int32_t), cudaMemcpyHostToDevice, st));
        } else if (D) {
            uint32_t grid = (uint32_t)std::min<uint64_t>((uint64_t)h->num_sms * 16, (D * 32 + 255) / 256);
            const bool nk_smem = K <= 8192;     // at most 32 KB of shared memory
            k_counts<<<grid, 256, nk_smem ? K * sizeof(int32_t) : 0, st>>>(
                h->d_doc_off, h->d_words, h->d_z, D, K, V, h->d_ndk, h->d_nkw[0], h->d_nk[0], h->d_doc_len, nk_smem);
            launch_check(h);
            // this rank's valid tokens: the sum of its n_k, before any exchange
            std::vector<int32_t> nk_local(K);
            CK(cudaMemcpyAsync(nk_local.data(), h->d_nk[0], K * sizeof(int32_t), cudaMemcpyDeviceToHost, st));
            CK(cudaStreamSynchronize(st));
            for (uint32_t k = 0; k < K; ++k) N += (uint64_t)(uint32_t)nk_local[k];
            h->N = N;
        }
        if (h->world > 1) {
            if (h->d_delta) CK(cudaMemsetAsync(h->d_delta, 0, ((uint64_t)K * V + K) * sizeof(int32_t), st));
            // every rank counted its own documents: the model's counts are the sums
            exchange(h, h->d_nkw[0], (uint64_t)K * V, TMT_I32);
            exchange(h, h->d_nk[0], K, TMT_I32);
        }
        CK(cudaStreamSynchronize(st));
        h->uploaded = true;
    });
}

} // namespace

extern "C" {

tmt_status tmt_create(const tmt_config* cfg, tmt_handle** out)
{
    if (!cfg || !out) return TMT_ERR_INVALID_ARGUMENT;
    *out = nullptr;
    tmt_handle* h = nullptr;
    try {
        h = new tmt_handle();
    } catch (...) {
        return TMT_ERR_OUT_OF_MEMORY;
    }
    h->cfg = *cfg;
    h->cfg.alpha = nullptr;
    h->device = cfg->device;
    try {
        validate_config(*cfg);   // the ctor's argument checks, before any CUDA call
    } catch (const std::exception& e) {
        h->err = e.what();
        *out = h;
        return TMT_ERR_INVALID_ARGUMENT;
    }
    if (cfg->sampler == TMT_SAMPLER_SPARSE) {
        h->err = "the sparse-bucket sampler is not built (the dense sampler is TMT_SAMPLER_DENSE / AUTO)";
        *out = h;
        return TMT_ERR_UNSUPPORTED;
    }
    tmt_status s = guarded(h, [&] {
        h->groups = cfg->sweep_groups ? cfg->sweep_groups : 8;
        h->alpha.assign(cfg->K, cfg->alpha_scalar);
        if (cfg->alpha) std::copy(cfg->alpha, cfg->alpha + cfg->K, h->alpha.begin());
        CK(cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking));
        CK(cudaEventCreate(&h->ev0));
        CK(cudaEventCreate(&h->ev1));
        CK(cudaEventCreate(&h->kev0));
        CK(cudaEventCreate(&h->kev1));
        CK(cudaEventCreate(&h->tev0));
        CK(cudaEventCreate(&h->tev1));
        CK(cudaDeviceGetAttribute(&h->num_sms, cudaDevAttrMultiProcessorCount, h->device));
    });
    if (s != TMT_OK) {
        // keep the handle so the caller can read the message
        *out = h;
        return s;
    }
    *out = h;
    return TMT_OK;
}


tmt_status tmt_upload_corpus(tmt_handle* h, const uint32_t* wid, const uint64_t* doc_off, uint64_t D,
                             const uint16_t* z0)
{
    return upload_impl(h, wid, doc_off, D, z0, nullptr);
}

tmt_status tmt_upload_corpus_weighted(tmt_handle* h, const uint32_t* wid, const uint64_t* doc_off, uint64_t D,
                                      const uint16_t* z0, const float* weights)
{
    if (!h) return TMT_ERR_INVALID_ARGUMENT;
    if (!weights) {
        h->err = "weights is NULL";
        return TMT_ERR_INVALID_ARGUMENT;
    }
    return upload_impl(h, wid, doc_off, D, z0, nullptr, weights);
}

tmt_status tmt_upload_shard(tmt_handle* h, const uint32_t* wid, const uint64_t* doc_off, uint64_t D,
                            const uint16_t* z0, const tmt_shard* shard)
{
    if (!shard) return TMT_ERR_INVALID_ARGUMENT;
    return upload_impl(h, wid, doc_off, D, z0, shard);
}

tmt_status tmt_plan_shard(const uint64_t* doc_len_global, uint64_t D_global, uint32_t groups, uint64_t doc_begin,
                          uint64_t D_local, uint32_t* local_order, uint64_t* local_bounds, uint64_t* global_bounds,
                          uint64_t* token_offset)
{
    if ((D_global && !doc_len_global) || (D_local && !local_order) || !local_bounds) return TMT_ERR_INVALID_ARGUMENT;
    try {
        const ShardPlan p = plan_shard(doc_len_global, D_global, groups, doc_begin, D_local);
        std::copy(p.order.begin(), p.order.end(), local_order);
        std::copy(p.bounds.begin(), p.bounds.end(), local_bounds);
        if (global_bounds) std::copy(p.gbounds.begin(), p.gbounds.end(), global_bounds);
        if (token_offset) *token_offset = p.tok_offset;
        return TMT_OK;
    } catch (const ArgError&) {
        return TMT_ERR_INVALID_ARGUMENT;
    } catch (const std::bad_alloc&) {
        return TMT_ERR_OUT_OF_MEMORY;
    }
}

tmt_status tmt_train(tmt_handle* h, uint32_t iters, uint32_t ll_every, double* ll_out)
{
    if (!h) return TMT_ERR_INVALID_ARGUMENT;
    return guarded(h, [&] {
        if (!h->uploaded) throw StateError("train() before the corpus was uploaded");
        if (h->D == 0 || h->N == 0) {
            h->global_step += iters;
            return;
        }
        const uint32_t npts = (ll_every && ll_out) ? iters / ll_every : 0;
        if (npts > h->ll_cap) {
            h->d_ll = h->dalloc<double>(2 * (size_t)npts);
            h->ll_cap = npts;
        }
        uint32_t pt = 0;
        h->sweep_kernel_ms = 0;
        h->sweeps_timed = 0;
        const bool use_graphs = h->graphs && h->world == 1;
        uint32_t runs = 0;              // runs of graph sweeps between ll / optimiser steps
        bool in_run = false;
        auto run_event = [&](uint32_t idx) {
            while (h->run_ev.size() <= idx) {
                cudaEvent_t e;
                CK(cudaEventCreate(&e));
                h->run_ev.push_back(e);
            }
            return h->run_ev[idx];
        };
        auto end_run = [&] {
            if (!in_run) return;
            CK(cudaEventRecord(run_event(2 * runs + 1), h->stream));
            ++runs;
            in_run = false;
        };
        CK(cudaEventRecord(h->tev0, h->stream));
        for (uint32_t i = 0; i < iters; ++i) {
            if (use_graphs && h->tuned >= 0) {
                if (!in_run) {
                    k_set_step<<<1, 1, 0, h->stream>>>(h->d_step, (uint32_t)h->global_step);
                    launch_check(h);
                    CK(cudaEventRecord(run_event(2 * runs), h->stream));
                    in_run = true;
                }
                CK(cudaEventRecord(h->ev0, h->stream));
                graph_sweep(h);
                CK(cudaEventRecord(h->ev1, h->stream));
                ++h->sweeps_timed;
            } else {
                end_run();
                CK(cudaEventRecord(h->ev0, h->stream));
                do_sweep(h);
                CK(cudaEventRecord(h->ev1, h->stream));
                // the events of this sweep are complete before the next
                // sweep records them again: read them now
                CK(cudaEventSynchronize(h->kev1));
                float ms = 0.f;
                CK(cudaEventElapsedTime(&ms, h->kev0, h->kev1));
                h->sweep_kernel_ms += ms;
                ++h->sweeps_timed;
                if (h->tuned < 0) {
                    const uint32_t G = (uint32_t)h->group_bounds.size() - 1;
                    for (uint32_t g = 0; g < G; ++g) {
                        if (h->group_bounds[g] == h->group_bounds[g + 1]) continue;
                        float gm = 0.f;
                        CK(cudaEventElapsedTime(&gm, h->gev[2 * g], h->gev[2 * g + 1]));
                        h->group_ms[g][h->variant] += gm;
                    }
                    const int nv = h->n_variants;
                    const int steps = nv > 1 ? 2 * nv : 1;
                    if (++h->tune_step >= steps) {
                        for (uint32_t g = 0; g < G; ++g) {
                            const auto& v = h->group_ms[g];
                            h->group_variant[g] = (int)(std::min_element(v.begin(), v.end()) - v.begin());
                        }
                        h->variant = 0;
                        h->tuned = 0;
                        h->drop_graphs();
                    } else {
                        h->variant = h->tune_step < nv ? h->tune_step : 2 * nv - 1 - h->tune_step;
                    }
                }
            }
            const uint64_t gs = h->global_step;
            const bool opt = gs >= h->cfg.burn_in && h->cfg.optim_interval && (gs + 1) % h->cfg.optim_interval == 0;
            const bool llp = npts && (i + 1) % ll_every == 0 && pt < npts;
            if (opt || llp) end_run();
            if (opt && !h->d_arow) do_optimize(h);   // per-document alphas are the caller's (DMR fits lambda)
            ++h->global_step;
            if (llp) do_ll(h, h->d_ll + 2 * pt++);
        }
        end_run();
        CK(cudaEventRecord(h->tev1, h->stream));
        CK(cudaStreamSynchronize(h->stream));
        CK(cudaEventElapsedTime(&h->last_ms, h->ev0, h->ev1));
        for (uint32_t r = 0; r < runs; ++r) {
            float ms = 0.f;
            CK(cudaEventElapsedTime(&ms, h->run_ev[2 * r], h->run_ev[2 * r + 1]));
            h->sweep_kernel_ms += ms;
        }
        {
            float ms = 0.f;
            CK(cudaEventElapsedTime(&ms, h->tev0, h->tev1));
            h->train_ms = ms;
        }
        if (npts) {
            std::vector<double> tmp(2 * (size_t)npts);
            CK(cudaMemcpy(tmp.data(), h->d_ll, tmp.size() * sizeof(double), cudaMemcpyDeviceToHost));
            for (uint32_t p = 0; p < npts; ++p) ll_out[p] = tmp[2 * p] + tmp[2 * p + 1];
        }
    });
}

tmt_status tmt_ll(tmt_handle* h, double* ll_docs, double* ll_rest)
{
    if (!h) return TMT_ERR_INVALID_ARGUMENT;
    return guarded(h, [&] {
        if (!h->uploaded) throw StateError("ll before the corpus was uploaded");
        double out[2] = { 0, 0 };
        if (h->D) {
            do_ll(h, h->d_llv);
            CK(cudaMemcpyAsync(out, h->d_llv, sizeof(out), cudaMemcpyDeviceToHost, h->stream));
            CK(cudaStreamSynchronize(h->stream));
        }
        if (ll_docs) *ll_docs = out[0];
        if (ll_rest) *ll_rest = out[1];
    });
}

tmt_status tmt_download_state(tmt_handle* h, uint16_t* z, int32_t* n_kw, int32_t* n_k, float* alpha)
{
    if (!h) return TMT_ERR_INVALID_ARGUMENT;
    return guarded(h, [&] {
        if (!h->uploaded) throw StateError("no corpus uploaded");
        if (h->weighted && (n_kw || n_k))
            throw StateError("the counts are weighted (float): read them with tmt_download_counts_f32");
        const uint32_t K = h->cfg.K, V = h->cfg.V;
        if (z) d2h(h, z, h->d_z, h->N_all * sizeof(uint16_t));
        if (n_kw) d2h(h, n_kw, h->d_nkw[h->cur], (uint64_t)K * V * sizeof(int32_t));
        if (n_k) CK(cudaMemcpyAsync(n_k, h->d_nk[h->cur], K * sizeof(int32_t), cudaMemcpyDeviceToHost, h->stream));
        CK(cudaMemcpyAsync(h->alpha.data(), h->d_alpha, K * sizeof(float), cudaMemcpyDeviceToHost, h->stream));
        CK(cudaStreamSynchronize(h->stream));
        if (alpha) std::copy(h->alpha.begin(), h->alpha.end(), alpha);
    });
}

tmt_status tmt_download_counts_f32(tmt_handle* h, float* n_dk, float* n_kw, float* n_k, float* doc_wlen)
{
    if (!h) return TMT_ERR_INVALID_ARGUMENT;
    return guarded(h, [&] {
        if (!h->uploaded) throw StateError("no corpus uploaded");
        if (!h->weighted) throw StateError("the counts are integers: read them with tmt_download_state");
        const uint64_t K = h->cfg.K, V = h->cfg.V;
        if (n_dk) d2h(h, n_dk, h->d_ndk, h->D * K * sizeof(float));
        if (n_kw) d2h(h, n_kw, h->d_nkw[0], K * V * sizeof(float));
        if (n_k) CK(cudaMemcpyAsync(n_k, h->d_nk[0], K * sizeof(float), cudaMemcpyDeviceToHost, h->stream));
        if (doc_wlen && h->D)
            CK(cudaMemcpyAsync(doc_wlen, h->d_doc_wlen, h->D * sizeof(float), cudaMemcpyDeviceToHost, h->stream));
        CK(cudaStreamSynchronize(h->stream));
    });
}

tmt_status tmt_download_doc_topic(tmt_handle* h, int32_t* n_dk)
{
    if (!h) return TMT_ERR_INVALID_ARGUMENT;
    return guarded(h, [&] {
        if (!h->uploaded) throw StateError("no corpus uploaded");
        if (!n_dk) throw ArgError("n_dk is NULL");
        if (h->weighted) throw StateError("the counts are weighted (float): read them with tmt_download_counts_f32");
        d2h(h, n_dk, h->d_ndk, (h->n_rows ? h->n_rows : h->D) * (uint64_t)h->cfg.K * sizeof(int32_t));
    });
}

tmt_status tmt_set_counts(tmt_handle* h, const int32_t* n_kw, const int32_t* n_k)
{
    if (!h) return TMT_ERR_INVALID_ARGUMENT;
    return guarded(h, [&] {
        if (!h->uploaded) throw StateError("set_counts before the corpus was uploaded");
        if (!n_kw || !n_k) throw ArgError("n_kw / n_k is NULL");
        if (h->weighted) throw StateError("set_counts takes integer counts; this corpus has weighted counts");
        const uint64_t kv = (uint64_t)h->cfg.K * h->cfg.V;
        h2d(h, h->d_nkw[h->cur], n_kw, kv * sizeof(int32_t));
        CK(cudaMemcpyAsync(h->d_nk[h->cur], n_k, h->cfg.K * sizeof(int32_t), cudaMemcpyHostToDevice, h->stream));
        CK(cudaStreamSynchronize(h->stream));
    });
}

tmt_status tmt_set_doc_topic_mask(tmt_handle* h, const uint32_t* mask_bits)
{
    if (!h) return TMT_ERR_INVALID_ARGUMENT;
    return guarded(h, [&] {
        if (!h->uploaded) throw StateError("set_doc_topic_mask before the corpus was uploaded");
        if (h->world > 1) throw ArgError("per-document masks on a corpus sharded across GPUs are not supported");
        if (h->n_rows && mask_bits) throw StateError("per-document masks and shared rows do not combine");
        h->drop_graphs();
        if (!mask_bits) { h->d_mask = nullptr; return; }
        const uint64_t mw = (h->cfg.K + 31) / 32;
        if (!h->d_mask) h->d_mask = h->dalloc<uint32_t>(std::max<uint64_t>(1, h->D * mw));
        if (h->D) CK(cudaMemcpyAsync(h->d_mask, mask_bits, h->D * mw * sizeof(uint32_t), cudaMemcpyHostToDevice, h->stream));
        CK(cudaStreamSynchronize(h->stream));
    });
}

tmt_status tmt_set_doc_alpha(tmt_handle* h, uint32_t M, const float* alpha_rows, const uint32_t* doc_row)
{
    if (!h) return TMT_ERR_INVALID_ARGUMENT;
    return guarded(h, [&] {
        if (!h->uploaded) throw StateError("set_doc_alpha before the corpus was uploaded");
        if (h->world > 1) throw ArgError("per-document alphas on a corpus sharded across GPUs are not supported");
        if (h->n_rows && alpha_rows) throw StateError("per-document alphas and shared rows do not combine");
        h->drop_graphs();
        if (!alpha_rows) { h->d_arow = nullptr; h->d_alpha_rows = nullptr; h->d_row_asum = nullptr; return; }
        const uint32_t K = h->cfg.K;
        if (M == 0 || !doc_row) throw ArgError("alpha rows need M > 0 and doc_row");
        for (uint64_t i = 0; i < (uint64_t)M * K; ++i)
            if (!(alpha_rows[i] > 0.f) || !std::isfinite(alpha_rows[i])) throw ArgError("alphas must be finite and > 0");
        for (uint64_t d = 0; d < h->D; ++d)
            if (doc_row[d] >= M) throw ArgError("doc_row[" + std::to_string(d) + "] >= M");
        std::vector<double> ras(2 * (size_t)M);
        for (uint32_t m = 0; m < M; ++m) {
            double sd = 0;
            for (uint32_t k = 0; k < K; ++k) sd += (double)alpha_rows[(uint64_t)m * K + k];
            ras[2 * m] = sd;
            ras[2 * m + 1] = std::lgamma(sd);
        }
        h->d_alpha_rows = h->dalloc<float>((uint64_t)M * K);
        h->d_row_asum = h->dalloc<double>(2 * (size_t)M);
        if (!h->d_arow) h->d_arow = h->dalloc<uint32_t>(std::max<uint64_t>(1, h->D));
        CK(cudaMemcpyAsync(h->d_alpha_rows, alpha_rows, (uint64_t)M * K * sizeof(float), cudaMemcpyHostToDevice, h->stream));
        CK(cudaMemcpyAsync(h->d_row_asum, ras.data(), ras.size() * sizeof(double), cudaMemcpyHostToDevice, h->stream));
        if (h->D) CK(cudaMemcpyAsync(h->d_arow, doc_row, h->D * sizeof(uint32_t), cudaMemcpyHostToDevice, h->stream));
        CK(cudaStreamSynchronize(h->stream));
    });
}

tmt_status tmt_set_word_priors(tmt_handle* h, uint32_t P, const uint32_t* word_ids, const float* priors)
{
    if (!h) return TMT_ERR_INVALID_ARGUMENT;
    return guarded(h, [&] {
        if (h->uploaded) throw StateError("word priors must be set before the corpus is uploaded");
        if (P && (!word_ids || !priors)) throw ArgError("word_ids / priors is NULL");
        const uint32_t K = h->cfg.K, V = h->cfg.V;
        if (P > V) throw ArgError("more prior words than words");
        std::vector<uint8_t> seen(V, 0);
        for (uint32_t p = 0; p < P; ++p) {
            if (word_ids[p] >= V) throw ArgError("prior word id " + std::to_string(word_ids[p]) + " >= V");
            if (seen[word_ids[p]]++) throw ArgError("prior word id " + std::to_string(word_ids[p]) + " given twice");
            for (uint32_t k = 0; k < K; ++k) {
                const float x = priors[(uint64_t)p * K + k];
                if (!(x >= 0.f) || !std::isfinite(x)) throw ArgError("priors must be finite and not less than 0");
            }
        }
        h->prior_ids.assign(word_ids, word_ids + P);
        h->prior_vals.assign(priors, priors + (uint64_t)P * K);
    });
}

tmt_status tmt_set_counts_f32(tmt_handle* h, const float* n_kw, const float* n_k)
{
    if (!h) return TMT_ERR_INVALID_ARGUMENT;
    return guarded(h, [&] {
        if (!h->uploaded) throw StateError("set_counts before the corpus was uploaded");
        if (!n_kw || !n_k) throw ArgError("n_kw / n_k is NULL");
        if (!h->weighted) throw StateError("set_counts_f32 takes weighted counts; this corpus has integer counts");
        const uint64_t kv = (uint64_t)h->cfg.K * h->cfg.V;
        for (uint64_t i = 0; i < kv; ++i)
            if (!(n_kw[i] >= 0.f) || !std::isfinite(n_kw[i])) throw ArgError("n_kw holds a negative or non-finite value");
        for (uint32_t k = 0; k < h->cfg.K; ++k)
            if (!(n_k[k] >= 0.f) || !std::isfinite(n_k[k])) throw ArgError("n_k holds a negative or non-finite value");
        h2d(h, h->d_nkw[0], n_kw, kv * sizeof(float));
        CK(cudaMemcpyAsync(h->d_nk[0], n_k, h->cfg.K * sizeof(float), cudaMemcpyHostToDevice, h->stream));
        CK(cudaStreamSynchronize(h->stream));
    });
}

tmt_status tmt_set_alpha(tmt_handle* h, const float* alpha)
{
    if (!h || !alpha) return TMT_ERR_INVALID_ARGUMENT;
    return guarded(h, [&] {
        if (!h->uploaded) throw StateError("set_alpha before the corpus was uploaded");
        for (uint32_t k = 0; k < h->cfg.K; ++k)
            if (!(alpha[k] > 0)) throw ArgError("wrong alpha value");
        std::copy(alpha, alpha + h->cfg.K, h->alpha.begin());
        CK(cudaMemcpyAsync(h->d_alpha, h->alpha.data(), h->cfg.K * sizeof(float), cudaMemcpyHostToDevice, h->stream));
        CK(cudaStreamSynchronize(h->stream));
    });
}

tmt_status tmt_set_global_step(tmt_handle* h, uint64_t step)
{
    if (!h) return TMT_ERR_INVALID_ARGUMENT;
    h->global_step = step;
    return TMT_OK;
}

tmt_status tmt_set_seed(tmt_handle* h, uint64_t seed)
{
    if (!h) return TMT_ERR_INVALID_ARGUMENT;
    h->cfg.seed = seed;
    return guarded(h, [&] { h->drop_graphs(); });   // the seed is an argument of the captured launches
}

tmt_status tmt_get_sweep_variants(const tmt_handle* h, int32_t* out, uint32_t cap, uint32_t* n)
{
    if (!h || !n) return TMT_ERR_INVALID_ARGUMENT;
    *n = (uint32_t)h->group_variant.size();
    if (out)
        for (uint32_t g = 0; g < *n && g < cap; ++g) out[g] = h->tuned < 0 ? -1 : h->group_variant[g];
    return TMT_OK;
}

tmt_status tmt_get_sweep_timings(const tmt_handle* h, float* out, uint32_t cap, uint32_t* n_groups,
                                 uint32_t* n_variants)
{
    if (!h || !n_groups || !n_variants) return TMT_ERR_INVALID_ARGUMENT;
    *n_groups = (uint32_t)h->group_ms.size();
    *n_variants = (uint32_t)h->n_variants;
    if (out) {
        uint32_t i = 0;
        for (const auto& g : h->group_ms)
            for (float ms : g) {
                if (i < cap) out[i] = ms;
                ++i;
            }
    }
    return TMT_OK;
}

tmt_status tmt_set_doc_split(tmt_handle* h, uint64_t min_tokens, uint32_t step)
{
    if (!h) return TMT_ERR_INVALID_ARGUMENT;
    return guarded(h, [&] {
        if (step > 65536) throw ArgError("split step above 65536 positions");
        h->split_min = min_tokens;
        h->split_step = step ? step : kSplitStep;
        h->drop_graphs();          // the split is an argument of the captured launches
        update_split(h);
    });
}

tmt_status tmt_set_doc_rows(tmt_handle* h, uint64_t R, const uint32_t* row_of_doc)
{
    if (!h) return TMT_ERR_INVALID_ARGUMENT;
    return guarded(h, [&] {
        if (!h->uploaded) throw StateError("set_doc_rows before the corpus was uploaded");
        if (h->world > 1) throw ArgError("shared rows on a corpus sharded across GPUs are not supported");
        if (h->weighted) throw StateError("shared rows take integer counts; this corpus has weighted counts");
        if (row_of_doc && (h->d_mask || h->d_arow))
            throw StateError("shared rows do not combine with per-document masks or alphas");
        const uint64_t D = h->D;
        const uint32_t K = h->cfg.K, V = h->cfg.V;
        if (row_of_doc) {
            if (R == 0 || R >= 0xFFFFFFFFull) throw ArgError("R must be in 1 .. 2^32 - 2");
            for (uint64_t d = 0; d < D; ++d)
                if (row_of_doc[d] >= R) throw ArgError("row_of_doc[" + std::to_string(d) + "] >= R");
        }
        h->drop_graphs();                 // the rows are arguments of the captured launches
        std::vector<uint64_t> off(D + 1);
        CK(cudaMemcpyAsync(off.data(), h->d_doc_off, (D + 1) * sizeof(uint64_t), cudaMemcpyDeviceToHost, h->stream));
        CK(cudaStreamSynchronize(h->stream));
        const uint64_t rows = row_of_doc ? R : D;
        if (rows > h->row_cap) {
            h->d_ndk = h->dalloc<int32_t>(rows * K);
            h->d_doc_len = h->dalloc<int32_t>(rows);
            h->d_doc_order = h->dalloc<uint32_t>(rows);
            h->row_cap = rows;
        }
        ShardPlan plan;
        std::vector<uint64_t> lens;
        if (row_of_doc) {
            // row r's documents in ascending order (a counting sort on the row)
            std::vector<uint64_t> unit_off(R + 1, 0);
            lens.assign(R, 0);
            for (uint64_t d = 0; d < D; ++d) {
                ++unit_off[row_of_doc[d] + 1];
                lens[row_of_doc[d]] += off[d + 1] - off[d];
            }
            for (uint64_t r = 0; r < R; ++r) unit_off[r + 1] += unit_off[r];
            std::vector<uint32_t> docs(std::max<uint64_t>(D, 1));
            std::vector<uint64_t> fill(unit_off.begin(), unit_off.end() - 1);
            for (uint64_t d = 0; d < D; ++d) docs[fill[row_of_doc[d]]++] = (uint32_t)d;
            if (!h->d_unit_docs) {
                h->d_unit_docs = h->dalloc<uint32_t>(std::max<uint64_t>(D, 1));
                h->d_row_of = h->dalloc<uint32_t>(std::max<uint64_t>(D, 1));
            }
            if (R > h->unit_cap) {
                h->d_unit_off = h->dalloc<uint64_t>(R + 1);
                h->unit_cap = R;
            }
            CK(cudaMemcpyAsync(h->d_unit_off, unit_off.data(), (R + 1) * sizeof(uint64_t), cudaMemcpyHostToDevice,
                               h->stream));
            if (D) {
                CK(cudaMemcpyAsync(h->d_unit_docs, docs.data(), D * sizeof(uint32_t), cudaMemcpyHostToDevice,
                                   h->stream));
                CK(cudaMemcpyAsync(h->d_row_of, row_of_doc, D * sizeof(uint32_t), cudaMemcpyHostToDevice, h->stream));
            }
        } else {
            lens.resize(D);
            for (uint64_t d = 0; d < D; ++d) lens[d] = off[d + 1] - off[d];
        }
        plan = plan_shard(lens.data(), rows, h->groups, 0, rows);
        h->order_len.resize(rows);
        for (uint64_t q = 0; q < rows; ++q) h->order_len[q] = lens[plan.order[q]];
        h->n_rows = row_of_doc ? R : 0;
        h->group_bounds = plan.bounds;
        h->gbounds = plan.gbounds;
        h->group_tokens = plan.gtokens;
        update_split(h);
        if (rows)
            CK(cudaMemcpyAsync(h->d_doc_order, plan.order.data(), rows * sizeof(uint32_t), cudaMemcpyHostToDevice,
                               h->stream));
        // the rows' counts and lengths, recounted from z
        CK(cudaMemsetAsync(h->d_ndk, 0, rows * (uint64_t)K * sizeof(int32_t), h->stream));
        CK(cudaMemsetAsync(h->d_doc_len, 0, rows * sizeof(int32_t), h->stream));
        if (D) {
            const uint32_t grid = (uint32_t)std::min<uint64_t>((uint64_t)h->num_sms * 16, (D * 32 + 255) / 256);
            k_counts_rows<<<grid, 256, 0, h->stream>>>(h->d_doc_off, h->d_words, h->d_z, D, K, V,
                                                       row_of_doc ? h->d_row_of : nullptr, h->d_ndk, h->d_doc_len);
            launch_check(h);
        }
        CK(cudaStreamSynchronize(h->stream));
    });
}

tmt_status tmt_get_doc_split(const tmt_handle* h, uint32_t* n_long, uint32_t cap, uint32_t* n)
{
    if (!h || !n) return TMT_ERR_INVALID_ARGUMENT;
    *n = (uint32_t)h->group_nlong.size();
    if (n_long)
        for (uint32_t g = 0; g < *n && g < cap; ++g) n_long[g] = h->group_nlong[g];
    return TMT_OK;
}

tmt_status tmt_set_graphs(tmt_handle* h, int32_t enable)
{
    if (!h) return TMT_ERR_INVALID_ARGUMENT;
    h->graphs = enable != 0;
    return TMT_OK;
}

tmt_status tmt_set_optim(tmt_handle* h, uint32_t optim_interval, uint32_t burn_in)
{
    if (!h) return TMT_ERR_INVALID_ARGUMENT;
    h->cfg.optim_interval = optim_interval;
    h->cfg.burn_in = burn_in;
    return TMT_OK;
}

tmt_status tmt_get_info(const tmt_handle* h, tmt_info* out)
{
    if (!h || !out) return TMT_ERR_INVALID_ARGUMENT;
    out->D = h->D;
    out->N_all = h->N_all;
    out->N = h->N;
    out->global_step = h->global_step;
    out->device_bytes = h->bytes;
    out->K = h->cfg.K;
    out->V = h->cfg.V;
    out->sampler = h->sampler_used;
    out->last_sweep_ms = h->last_ms;
    out->kernel_launches = h->launches;
    out->sweep_kernel_ms = h->sweep_kernel_ms;
    out->sweeps_timed = h->sweeps_timed;
    out->sweep_groups = h->groups;
    out->train_ms = h->train_ms;
    out->rank = h->rank;
    out->world = h->world;
    return TMT_OK;
}

} // extern "C"

namespace {

// tmt_infer_batch / tmt_infer_batch_weighted (weights == NULL: integer counts)
tmt_status infer_impl(tmt_handle* h, const uint32_t* wid, const uint64_t* doc_off, uint64_t D, const float* weights,
                      uint32_t iters, uint64_t seed, const uint64_t* doc_keys, float* theta, double* ll)
{
    if (!h) return TMT_ERR_INVALID_ARGUMENT;
    return guarded(h, [&] {
        if (!h->uploaded) throw StateError("infer() before the model has a state");
        if (!doc_off) throw ArgError("doc_off is NULL");
        if (h->weighted && !weights)
            throw StateError("the model has weighted counts: infer with tmt_infer_batch_weighted");
        if (!h->weighted && weights)
            throw StateError("the model has integer counts: infer with tmt_infer_batch");
        const uint64_t n_all = doc_off[D];
        if (n_all && !wid) throw ArgError("wid is NULL");
        for (uint64_t d = 0; d < D; ++d)
            if (doc_off[d + 1] < doc_off[d]) throw ArgError("doc_off is not non-decreasing");
        if (infer_warps(h->cfg.K) == 0) throw ArgError("K too large for inference");
        if (D >= 0xFFFFFFFFull) throw ArgError("too many documents");
        if (D == 0) return;
        const uint32_t K = h->cfg.K;
        // documents sorted by word id, as prepareDoc does (LDAModel.hpp:716-722),
        // the weights following their tokens
        std::vector<uint32_t> sorted(wid, wid + n_all);
        std::vector<float> wsorted;
        if (weights) {
            std::vector<std::pair<uint32_t, float>> pw(n_all);
            for (uint64_t i = 0; i < n_all; ++i) pw[i] = { wid[i], weights[i] };
            for (uint64_t d = 0; d < D; ++d)
                std::stable_sort(pw.begin() + doc_off[d], pw.begin() + doc_off[d + 1],
                                 [](const auto& x, const auto& y) { return x.first < y.first; });
            wsorted.resize(n_all);
            for (uint64_t i = 0; i < n_all; ++i) {
                sorted[i] = pw[i].first;
                wsorted[i] = pw[i].second;
                if (sorted[i] >= h->cfg.V) continue;
                if (!(wsorted[i] >= 0.f) || !(wsorted[i] <= 65536.f))
                    throw ArgError("token weight " + std::to_string(i) + " is negative, too large or not finite");
            }
            for (uint64_t d = 0; d < D; ++d)
                for (uint64_t i = doc_off[d] + 1; i < doc_off[d + 1]; ++i)
                    if (sorted[i] == sorted[i - 1] && sorted[i] < h->cfg.V && wsorted[i] != wsorted[i - 1])
                        throw ArgError("the tokens of one word in document " + std::to_string(d) +
                                       " carry different weights");
        } else {
            for (uint64_t d = 0; d < D; ++d)
                std::stable_sort(sorted.begin() + doc_off[d], sorted.begin() + doc_off[d + 1]);
        }
        auto& B = h->inf;
        if (D > B.cap_docs) {
            B.doc_off = h->dalloc<uint64_t>(D + 1);
            B.keys = h->dalloc<uint64_t>(D);
            B.ll = h->dalloc<double>(D);
            B.cap_docs = D;
        }
        if (D * K > B.cap_theta) {
            B.theta = h->dalloc<float>(D * (uint64_t)K);
            B.cap_theta = D * (uint64_t)K;
        }
        if (n_all > B.cap_tokens) {
            B.words = h->dalloc<uint32_t>(n_all);
            B.z = h->dalloc<uint16_t>(n_all);
            B.cap_tokens = n_all;
        }
        if (weights && n_all > B.cap_wt) {
            B.wt = h->dalloc<float>(n_all);
            B.cap_wt = n_all;
        }
        if (!B.acum) {
            B.acum = h->dalloc<float>(K);
            B.counter = h->dalloc<uint32_t>(1);
        }
        // alpha of the current state (after any optimisation)
        CK(cudaMemcpyAsync(h->alpha.data(), h->d_alpha, K * sizeof(float), cudaMemcpyDeviceToHost, h->stream));
        CK(cudaStreamSynchronize(h->stream));
        std::vector<float> acum(K);
        float sf = 0.f;
        double sd = 0;
        for (uint32_t k = 0; k < K; ++k) { sf = sf + h->alpha[k]; acum[k] = sf; sd += (double)h->alpha[k]; }
        cudaStream_t st = h->stream;
        CK(cudaMemcpyAsync(B.doc_off, doc_off, (D + 1) * sizeof(uint64_t), cudaMemcpyHostToDevice, st));
        h2d(h, B.words, sorted.data(), n_all * sizeof(uint32_t));
        if (weights) h2d(h, B.wt, wsorted.data(), n_all * sizeof(float));
        if (doc_keys) CK(cudaMemcpyAsync(B.keys, doc_keys, D * sizeof(uint64_t), cudaMemcpyHostToDevice, st));
        CK(cudaMemcpyAsync(B.acum, acum.data(), K * sizeof(float), cudaMemcpyHostToDevice, st));
        CK(cudaMemsetAsync(B.counter, 0, sizeof(uint32_t), st));
        InferArgs a{};
        a.nkw = h->d_nkw[h->cur];
        a.nk = h->d_nk[h->cur];
        a.alpha = h->d_alpha;
        a.acum = B.acum;
        a.K = K;
        a.V = h->cfg.V;
        a.eta = h->cfg.eta;
        a.veta = h->cfg.eta * (float)h->cfg.V;
        a.asum_f = sf;
        a.veta_d = (double)h->cfg.V * (double)h->cfg.eta;
        a.asum_d = sd;
        a.lg_asum = std::lgamma(sd);
        a.lg_eta = std::lgamma((double)h->cfg.eta);
        a.key = seed ^ (uint64_t)tmt::kStreamInfer;
        a.words = B.words;
        a.z = B.z;
        a.tok_begin = B.doc_off;          // slot d = document d: tokens [doc_off[d], doc_off[d+1])
        a.tok_len = nullptr;
        a.keys = doc_keys ? B.keys : nullptr;
        a.it_begin = a.it_end = a.it_total = nullptr;
        a.u_begin = 0;
        a.u_end = iters;
        a.u_total = iters;
        a.ndk = nullptr;
        a.theta = B.theta;
        a.ll = B.ll;
        a.work = nullptr;
        a.n_work = (uint32_t)D;
        a.counter = B.counter;
        a.wt = weights ? B.wt : nullptr;
        a.pidx = h->d_prior_idx;
        a.pval = h->d_prior;
        a.esum = h->d_esum;
        a.pcum = h->d_prior_cum;
        a.ecum = h->d_cum_eta;
        launch_infer(a, h->num_sms, h->stream);
        ++h->launches;
        if (theta) d2h(h, theta, B.theta, D * (uint64_t)K * sizeof(float));
        if (ll) CK(cudaMemcpyAsync(ll, B.ll, D * sizeof(double), cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
    });
}

} // namespace

extern "C" {

tmt_status tmt_infer_batch(tmt_handle* h, const uint32_t* wid, const uint64_t* doc_off, uint64_t D,
                           uint32_t iters, uint64_t seed, const uint64_t* doc_keys, float* theta, double* ll)
{
    return infer_impl(h, wid, doc_off, D, nullptr, iters, seed, doc_keys, theta, ll);
}

tmt_status tmt_infer_batch_weighted(tmt_handle* h, const uint32_t* wid, const uint64_t* doc_off, uint64_t D,
                                    const float* weights, uint32_t iters, uint64_t seed, const uint64_t* doc_keys,
                                    float* theta, double* ll)
{
    if (h && !weights) {
        h->err = "weights is NULL";
        return TMT_ERR_INVALID_ARGUMENT;
    }
    return infer_impl(h, wid, doc_off, D, weights, iters, seed, doc_keys, theta, ll);
}

/* Allocation-free FP64 log-likelihood over caller-owned device counts.
 * Host code may not pass g_ll_scratch itself (its host-side name is not a
 * device address): the device address is looked up with cudaGetSymbolAddress,
 * with the device current, once per device context, and reused. */
tmt_status tmt_ll_counts_noalloc(const int32_t* n_dk, uint64_t D, uint32_t K, const int32_t* doc_len,
                                 const float* alpha, const int32_t* n_kw, uint32_t V, const int32_t* n_k,
                                 float eta, double* ll_out, void* stream, char* err, size_t err_len)
{
    auto say = [&](tmt_status st, const std::string& msg) {
        if (err && err_len) {
            const size_t n = std::min(err_len - 1, msg.size());
            std::memcpy(err, msg.data(), n);
            err[n] = '\0';
        }
        return st;
    };
    if (K == 0 || K > kNoAllocMaxK)
        return say(TMT_ERR_INVALID_ARGUMENT, "K = " + std::to_string(K) + " is outside 1.." +
                                                 std::to_string(kNoAllocMaxK) + ", the size of the static scratch");
    if (!ll_out || !alpha || !n_k || (D && (!n_dk || !doc_len)) || (V && !n_kw))
        return say(TMT_ERR_INVALID_ARGUMENT, "a required device pointer is NULL");
    if (!(eta > 0)) return say(TMT_ERR_INVALID_ARGUMENT, "eta must be > 0");
    // an error left by the caller's own earlier work is reported as such and
    // left in place; nothing is launched
    cudaError_t e = cudaPeekAtLastError();
    if (e != cudaSuccess)
        return say(TMT_ERR_CUDA, std::string("an earlier CUDA error is pending on this thread: ") +
                                     cudaGetErrorString(e));
    // every array must be device (or managed) memory: a host pointer handed
    // to the kernels would fault on the GPU instead of failing here
    const struct { const void* p; const char* name; } arrays[] = {
        { n_dk, "n_dk" }, { doc_len, "doc_len" }, { alpha, "alpha" }, { n_kw, "n_kw" }, { n_k, "n_k" },
        { ll_out, "ll_out" } };
    for (const auto& a : arrays) {
        if (!a.p) continue;
        cudaPointerAttributes at{};
        const cudaError_t pe = cudaPointerGetAttributes(&at, a.p);
        if (pe != cudaSuccess) {
            cudaGetLastError();
            return say(TMT_ERR_INVALID_ARGUMENT, std::string(a.name) + " is not memory CUDA knows: " +
                                                     cudaGetErrorString(pe));
        }
        if (at.type != cudaMemoryTypeDevice && at.type != cudaMemoryTypeManaged)
            return say(TMT_ERR_INVALID_ARGUMENT, std::string(a.name) + " is not device or managed memory");
    }
    // set-up, once per device context: the array's device address and the
    // SM count.  A new context (cudaDeviceReset, or another context made
    // current) has its own copy of the array, so the cache is keyed by the
    // context's unique id.
    struct Slot { unsigned long long ctx; double* ptr; int sms; };
    static std::mutex mu;
    static Slot slots[64] = {};
    int dev = 0;
    e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return say(TMT_ERR_CUDA, std::string("cudaGetDevice: ") + cudaGetErrorString(e));
    if (dev < 0 || dev >= 64) return say(TMT_ERR_UNSUPPORTED, "device ordinal above 63");
    double* base = nullptr;
    int sms = 0;
    {
        std::lock_guard<std::mutex> lock(mu);
        Slot& sl = slots[dev];
        const unsigned long long ctx = current_context_id();
        if (!sl.ptr || ctx == 0 || sl.ctx != ctx) {
            void* p = nullptr;
            e = cudaGetSymbolAddress(&p, g_ll_scratch);
            if (e != cudaSuccess)
                return say(TMT_ERR_CUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
            int n = 0;
            e = cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
            if (e != cudaSuccess)
                return say(TMT_ERR_CUDA, std::string("cudaDeviceGetAttribute: ") + cudaGetErrorString(e));
            sl = Slot{ current_context_id(), static_cast<double*>(p), n };
        }
        base = sl.ptr;
        sms = sl.sms;
    }
    // tmt_ll's grid on this device (ll_blocks), so both give the same sums
    const uint32_t blocks = ll_blocks(sms);
    double* partials = base;                             // 2 * blocks, every slot overwritten
    double* lg_alpha = partials + 2 * kNoAllocMaxBlocks; // K, every slot overwritten
    double* asum = lg_alpha + kNoAllocMaxK;              // 2, overwritten
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const double etad = (double)eta;
    k_ll_prep<<<1, 256, 0, st>>>(alpha, K, lg_alpha, asum);
    k_ll_partials<<<blocks, 256, 0, st>>>(n_dk, D, K, lg_alpha, alpha, doc_len, asum, n_kw, V, etad,
                                          std::lgamma(etad), partials, PriorArgs{}, nullptr, nullptr, nullptr);
    k_ll_final<<<1, 256, 0, st>>>(partials, blocks, n_k, K, (double)V * etad, ll_out, nullptr);
    // no error was pending before the launches: one now is theirs
    e = cudaGetLastError();
    if (e != cudaSuccess) return say(TMT_ERR_CUDA, std::string("launch: ") + cudaGetErrorString(e));
    return say(TMT_OK, "");
}

const char* tmt_last_error(const tmt_handle* h)
{
    return h ? h->err.c_str() : "null handle";
}

void tmt_destroy(tmt_handle* h)
{
    delete h;
}

} // extern "C"
