// infer.cuh -- inference of unseen documents against a frozen model:
// tomotopy's LDAModel::_infer<together = false> (LDAModel.hpp:920-953).
//
// Each document gets a private copy of the model with its own tokens added,
// z0 ~ Discrete(alpha), then sequential Gibbs sweeps.  Only the document's
// cells differ from the frozen model, so one warp keeps them on chip:
//   A_k = (float)n_dk[k] + alpha_k
//   R_k = 1 / ((float)(n_k[k] + n_dk[k]) + V*eta)
//   B_k = (float)(n_kw[k,v] + own[k]) + eta   (own: the document's other tokens of word v)
//   weight A_k * (B_k * R_k), drawn with the blocked two-pass draw of the training sweep.
// Documents are sorted by word id (prepareDoc, LDAModel.hpp:716-722), so the
// tokens of one word form a run and `own` is that run's topic histogram.
//
// The kernel works on "slots" and is resumable: one launch advances each
// listed slot through sweeps [it_begin, it_end); z and n_dk persist in device
// memory between launches.  Draws use the absolute (token, sweep) counter, so
// a document's result does not depend on how its sweeps are split across
// launches or on which other documents share them.
#pragma once
#include <algorithm>
#include <cmath>
#include <type_traits>
#include "common.cuh"
#include "philox.cuh"

namespace tmtk {

struct InferArgs {
    // frozen model
    const int32_t* nkw;          // K x V column-major
    const int32_t* nk;
    const float* alpha;
    const float* acum;           // sequential float cumsum of alpha
    uint32_t K, V;
    float eta, veta, asum_f;
    double veta_d, asum_d, lg_asum, lg_eta;
    uint64_t key;                // seed ^ 'INFR'
    // tokens, addressed by the slots
    const uint32_t* words;       // sorted within each document
    uint16_t* z;
    // slots
    const uint64_t* tok_begin;   // first token of each slot; with tok_len == NULL, tok_begin[s+1] ends slot s
    const uint32_t* tok_len;
    const uint64_t* keys;        // per-slot draw key; NULL: 0
    const uint32_t* it_begin;    // per-slot sweep range of this launch; NULL: the uniform values below
    const uint32_t* it_end;
    const uint32_t* it_total;
    uint32_t u_begin, u_end, u_total;
    int32_t* ndk;                // slot x K counts kept between launches; NULL when every slot finishes here
    float* theta;                // slot x K, written when a slot finishes (may be NULL)
    double* ll;                  // slot, written when a slot finishes (may be NULL)
    const uint32_t* work;        // slots advanced by this launch; NULL: 0 .. n_work-1
    uint32_t n_work;
    uint32_t* counter;           // zeroed before the launch
    // weighted counts (TermWeight IDF / PMI): nkw, nk and ndk hold floats;
    // wt[token] is the token's weight, the same for every token of one word
    // within a document (IDF: the word's weight; PMI: a function of the word's
    // count in the document)
    const float* wt;
    // word priors (etaByTopicWord): pidx[v] >= 0 names row pidx[v] of pval
    // (K floats); esum[k] replaces V*eta; z0 draws from pcum (the rows'
    // cumulative sums) or ecum (a column of eta).  pidx == NULL: no priors.
    const int32_t* pidx;
    const float* pval;
    const float* esum;
    const float* pcum;
    const float* ecum;
};

// WT: weighted counts.  The document's counts n_dk are float sums of weights
// (a removal clamps at 0, updateCnt<true>); B_k = (n_kw[k,v] + own[k] * w) + eta
// with w the weight of the current word's tokens; R_k = 1 / ((n_k[k] + n_dk[k])
// + V*eta); the document's length is its weight sum.  n_dk starts from z0 in
// token order (initializeDocState's addWordTo sequence).
template <int CH, bool WT>
__global__ void __launch_bounds__(256)
k_infer_slots(InferArgs a)
{
    using CT = typename std::conditional<WT, float, int>::type;
    using G4 = typename std::conditional<WT, float4, int4>::type;
    constexpr int CHR = CH > 0 ? CH : 1;
    extern __shared__ __align__(16) int smem[];
    const int K = (int)a.K;
    const int KP = (int)round4(a.K);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    CT* rowi = reinterpret_cast<CT*>(smem + warp * 4 * KP);
    const CT* nkw = reinterpret_cast<const CT*>(a.nkw);
    const CT* nkv = reinterpret_cast<const CT*>(a.nk);
    CT* ndk_s = reinterpret_cast<CT*>(a.ndk);
    float* rowf = reinterpret_cast<float*>(rowi + KP);
    float* rr = rowf + KP;
    int* own = reinterpret_cast<int*>(rr + KP);
    const int nch = 4 * lane < K ? ((K - 4 * lane + 127) >> 7) : 0;
    const float eta = a.eta, veta = a.veta;
    const bool vecg = (K & 3) == 0;      // n_kw columns 16-byte aligned: vector loads

    for (;;) {
        uint32_t q = 0;
        if (lane == 0) q = atomicAdd(a.counter, 1u);
        q = __shfl_sync(FULL, q, 0);
        if (q >= a.n_work) break;
        const uint32_t sl = a.work ? a.work[q] : q;
        const uint64_t b = a.tok_begin[sl];
        const uint32_t L = a.tok_len ? a.tok_len[sl] : (uint32_t)(a.tok_begin[sl + 1] - b);
        const uint64_t dk = a.keys ? a.keys[sl] : 0;
        const uint32_t klo = (uint32_t)dk, khi = (uint32_t)(dk >> 32);
        const uint32_t it0 = a.it_begin ? a.it_begin[sl] : a.u_begin;
        const uint32_t it1 = a.it_end ? a.it_end[sl] : a.u_end;
        const uint32_t itT = a.it_total ? a.it_total[sl] : a.u_total;
        for (int k = lane; k < KP; k += 32) own[k] = 0;
        int nvalid = 0;
        float wsum = 0.f;                    // WT: the document's weight sum, in token order
        if (it0 == 0) {
            // z0 ~ Discrete(alpha), added to the document's counts
            for (int k = lane; k < KP; k += 32) rowi[k] = 0;
            __syncwarp();
            for (uint32_t j = lane; j < L; j += 32) {
                const uint32_t w = a.words[b + j];
                uint16_t zz = 0xFFFF;
                if (w < a.V) {
                    const float u = tmt::u01(tmt::philox_u32(j, 0xFFFFFFFFu, klo, khi, a.key));
                    const float* cum = a.acum;
                    if (a.pidx) {
                        const int p = a.pidx[w];
                        cum = p >= 0 ? a.pcum + (uint64_t)p * K : a.ecum;
                    }
                    const float r = __fmul_rn(u, cum[K - 1]);
                    uint32_t lo = 0, hi = K - 1;
                    while (lo < hi) {
                        const uint32_t mid = (lo + hi) >> 1;
                        if (r < cum[mid]) hi = mid; else lo = mid + 1;
                    }
                    zz = (uint16_t)lo;
                    if (!WT) atomicAdd(reinterpret_cast<int*>(rowi) + lo, 1);
                    ++nvalid;
                }
                a.z[b + j] = zz;
            }
            if (WT) {
                __syncwarp();
                if (lane == 0)
                    for (uint32_t j = 0; j < L; ++j)
                        if (a.words[b + j] < a.V) {
                            const float wj = a.wt[b + j];
                            rowi[a.z[b + j]] = __fadd_rn(rowi[a.z[b + j]], wj);
                            wsum = __fadd_rn(wsum, wj);
                        }
            }
        } else {
            for (int k = lane; k < KP; k += 32) rowi[k] = k < K ? ndk_s[(uint64_t)sl * K + k] : CT(0);
            for (uint32_t j = lane; j < L; j += 32) nvalid += a.words[b + j] < a.V;
            if (WT && lane == 0)
                for (uint32_t j = 0; j < L; ++j)
                    if (a.words[b + j] < a.V) wsum = __fadd_rn(wsum, a.wt[b + j]);
        }
#pragma unroll
        for (int o = 16; o; o >>= 1) nvalid += __shfl_xor_sync(FULL, nvalid, o);
        if (WT) wsum = __shfl_sync(FULL, wsum, 0);
        __syncwarp();
        // R_k's denominator: (float)(n_k + n_dk) for integer counts, (n_k + n_dk) in float for weights
        auto rden = [&](int k, CT n) -> float {
            const float es = a.esum ? __ldg(a.esum + k) : veta;
            if constexpr (WT) return __fadd_rn(__fadd_rn(__ldg(nkv + k), n), es);
            else return __fadd_rn((float)(__ldg(nkv + k) + n), es);
        };
        for (int k = lane; k < KP; k += 32) {
            float f = 0.f, g = 0.f;
            if (k < K) {
                const CT n = rowi[k];
                f = __fadd_rn((float)n, __ldg(a.alpha + k));
                g = __frcp_rn(rden(k, n));
            }
            rowf[k] = f;
            rr[k] = g;
        }
        __syncwarp();
        // `own` holds the topics of the current run's other tokens; a word
        // that occurs once in the document never touches it.
        auto run_end = [&](uint32_t j0, uint32_t v) -> uint32_t {
            uint32_t re = j0 + 1;
            for (;;) {
                const uint32_t j = re + lane;
                const bool diff = j >= L || a.words[b + j] != v;
                const unsigned mm = __ballot_sync(FULL, diff);
                if (mm) return re + __ffs(mm) - 1;
                re += 32;
            }
        };
        // the frozen n_kw column of word `v_have`, this lane's blocks of four,
        // loaded once per run of a word.  (Loading the next token's column
        // during the current draw measured slower on B200: the extra registers
        // cost more occupancy than the hidden latency gained.)
        G4 gv[CHR];
        uint32_t v_have = 0xFFFFFFFFu;
        auto load_col = [&](uint32_t v, G4 (&g)[CHR]) {
            const CT* col = nkw + (uint64_t)v * K;
#pragma unroll
            for (int jj = 0; jj < CHR; ++jj) {
                if (jj < nch) {
                    const int k0 = 128 * jj + 4 * lane;
                    if (vecg) {
                        g[jj] = __ldg(reinterpret_cast<const G4*>(col + k0));
                    } else {
                        g[jj].x = __ldg(col + k0);
                        g[jj].y = k0 + 1 < K ? __ldg(col + k0 + 1) : 0;
                        g[jj].z = k0 + 2 < K ? __ldg(col + k0 + 2) : 0;
                        g[jj].w = k0 + 3 < K ? __ldg(col + k0 + 3) : 0;
                    }
                }
            }
        };
        for (uint32_t it = it0; it < it1; ++it) {
            uint32_t run_b = 0, run_e = 0;      // the multi-token run whose histogram is in `own`
            for (uint32_t base = 0; base < L; base += 32) {
                const uint32_t jl = base + lane;
                uint32_t my_w = 0xFFFFFFFFu, my_z = 0;
                uint32_t my_zc = 0;              // my token's current topic (updated when it is drawn)
                bool my_same = false;            // my token's word equals the next token's
                float my_u = 0.f, my_wt = 1.f;
                if (jl < L) {
                    my_w = a.words[b + jl];
                    my_z = a.z[b + jl];
                    if (WT) my_wt = a.wt[b + jl];
                    my_same = jl + 1 < L && a.words[b + jl + 1] == my_w;
                    my_u = tmt::u01(tmt::philox_u32(jl, it, klo, khi, a.key));
                }
                my_zc = my_z;
                const unsigned same_m = __ballot_sync(FULL, my_same);
                const int nb = (int)min(32u, L - base);
                for (int q2 = 0; q2 < nb; ++q2) {
                    const uint32_t j = base + q2;
                    const uint32_t v = __shfl_sync(FULL, my_w, q2);
                    const int zo = (int)__shfl_sync(FULL, my_z, q2);
                    const float u = __shfl_sync(FULL, my_u, q2);
                    const float wt = WT ? __shfl_sync(FULL, my_wt, q2) : 1.f;
                    if (v >= a.V) continue;
                    const bool in_run = j < run_e;
                    if (!in_run && ((same_m >> q2) & 1u)) {
                        // a multi-token run starts here: histogram of its tokens' topics.  A run
                        // inside this chunk of 32 tokens takes them from the lanes' registers.
                        run_b = j;
                        const unsigned rest = ~same_m & (0xFFFFFFFFu << q2);
                        if (rest) {
                            const int qe = __ffs(rest) - 1;           // the run's last token in the chunk
                            run_e = base + qe + 1;
                            if (lane >= q2 && lane <= qe) atomicAdd(&own[my_z], 1);
                        } else {
                            run_e = run_end(j, v);
                            for (uint32_t t = run_b + lane; t < run_e; t += 32) atomicAdd(&own[a.z[b + t]], 1);
                        }
                        __syncwarp();
                    }
                    const bool multi = j < run_e;
                    const CT* gcol = nkw + (uint64_t)v * K;
                    if (CH > 0 && v != v_have) { load_col(v, gv); v_have = v; }
                    const float* pe = nullptr;           // the word's prior column, if any
                    if (a.pidx) {
                        const int p = __ldg(a.pidx + v);
                        if (p >= 0) pe = a.pval + (uint64_t)p * K;
                    }
                    // B_k before the multiplication by R_k
                    auto bk = [&](CT g, int o, int k) -> float {
                        const float ek = pe ? __ldg(pe + k) : eta;
                        if constexpr (WT) return __fadd_rn(__fadd_rn(g, __fmul_rn((float)o, wt)), ek);
                        else return __fadd_rn((float)(g + o), ek);
                    };
                    if (lane == 0) {
                        if (multi) own[zo] -= 1;
                        CT n;
                        if constexpr (WT) {
                            n = __fsub_rn(rowi[zo], wt);
                            n = n > 0.f ? n : 0.f;
                        } else {
                            n = rowi[zo] - 1;
                        }
                        rowi[zo] = n;
                        rowf[zo] = __fadd_rn((float)n, __ldg(a.alpha + zo));
                        rr[zo] = __frcp_rn(rden(zo, n));
                    }
                    __syncwarp();
                    // pass 1: fma chain over this lane's topics
                    float s = 0.f;
                    if (CH > 0) {
#pragma unroll
                        for (int jj = 0; jj < CHR; ++jj) {
                            if (jj < nch) {
                                const int k0 = 128 * jj + 4 * lane;
                                const float4 A4 = *reinterpret_cast<const float4*>(rowf + k0);
                                const float4 R4 = *reinterpret_cast<const float4*>(rr + k0);
                                int4 O4 = make_int4(0, 0, 0, 0);
                                if (multi) O4 = *reinterpret_cast<const int4*>(own + k0);
                                s = __fmaf_rn(A4.x, __fmul_rn(bk(gv[jj].x, O4.x, k0), R4.x), s);
                                s = __fmaf_rn(A4.y, __fmul_rn(bk(gv[jj].y, O4.y, k0 + 1), R4.y), s);
                                s = __fmaf_rn(A4.z, __fmul_rn(bk(gv[jj].z, O4.z, k0 + 2), R4.z), s);
                                s = __fmaf_rn(A4.w, __fmul_rn(bk(gv[jj].w, O4.w, k0 + 3), R4.w), s);
                            }
                        }
                    } else {
                        for (int jj = 0; jj < nch; ++jj)
                            for (int i = 0; i < 4; ++i) {
                                const int k = 128 * jj + 4 * lane + i;
                                if (k < K) s = __fmaf_rn(rowf[k], __fmul_rn(bk(__ldg(gcol + k), own[k], k), rr[k]), s);
                            }
                    }
                    const float x = hs_scan32(s, lane);
                    float E = __shfl_up_sync(FULL, x, 1);
                    if (lane == 0) E = 0.f;
                    const float total = __shfl_sync(FULL, x, 31);
                    const float r = __fmul_rn(u, total);
                    const unsigned m = __ballot_sync(FULL, nch > 0 && r < __fadd_rn(E, s));
                    int znew = K - 1;
                    if (m) {
                        // pass 2: position among lane h's topics, 32 at a time
                        const int h = __ffs(m) - 1;
                        const float Eh = __shfl_sync(FULL, E, h);
                        const int mh = K - 4 * h;
                        const int nh = 4 * (mh >> 7) + min(mh & 127, 4);
                        float carry = 0.f;
                        int found = nh - 1;
                        for (int mm = 0; mm < nh; mm += 32) {
                            const int t = mm + lane;
                            const int k = 128 * (t >> 2) + 4 * h + (t & 3);
                            float x2 = 0.f;
                            if (t < nh)
                                x2 = __fmul_rn(rowf[k], __fmul_rn(bk(__ldg(gcol + k), multi ? own[k] : 0, k), rr[k]));
                            x2 = hs_scan32(x2, lane);
                            const unsigned mb = __ballot_sync(FULL, t < nh && r < __fadd_rn(Eh, __fadd_rn(carry, x2)));
                            if (mb) { found = mm + __ffs(mb) - 1; break; }
                            carry = __fadd_rn(carry, __shfl_sync(FULL, x2, 31));
                        }
                        znew = 128 * (found >> 2) + 4 * h + (found & 3);
                    }
                    __syncwarp();
                    if (lane == 0) {
                        if (multi) own[znew] += 1;
                        CT n;
                        if constexpr (WT) n = __fadd_rn(rowi[znew], wt);
                        else n = rowi[znew] + 1;
                        rowi[znew] = n;
                        rowf[znew] = __fadd_rn((float)n, __ldg(a.alpha + znew));
                        rr[znew] = __frcp_rn(rden(znew, n));
                        a.z[b + j] = (uint16_t)znew;
                    }
                    if (lane == q2) my_zc = (uint32_t)znew;
                    __syncwarp();
                    if (multi && j + 1 == run_e) {
                        // the run is done: clear its histogram (from the registers when the
                        // run lies inside this chunk)
                        if (run_b >= base) {
                            const uint32_t lb = run_b - base, le = run_e - base;
                            if (lane >= lb && lane < le) atomicSub(&own[my_zc], 1);
                        } else {
                            for (uint32_t t = run_b + lane; t < run_e; t += 32) atomicSub(&own[a.z[b + t]], 1);
                        }
                        __syncwarp();
                    }
                }
            }
        }
        if (it1 < itT) {            // keep the document's counts for the next launch
            for (int k = lane; k < K; k += 32) ndk_s[(uint64_t)sl * K + k] = rowi[k];
            __syncwarp();
            continue;
        }
        // finished: theta, FP64 ll over the touched cells
        double acc = 0;
        const float dlen = WT ? wsum : (float)nvalid;
        const float denom = __fadd_rn(dlen, a.asum_f);
        for (int k = lane; k < K; k += 32) {
            const CT n = rowi[k];
            if (a.theta) a.theta[(uint64_t)sl * K + k] = __fdiv_rn(__fadd_rn((float)n, __ldg(a.alpha + k)), denom);
            if (n != CT(0)) {
                const double gk = (double)__ldg(nkv + k);
                const double es = a.esum ? (double)__ldg(a.esum + k) : a.veta_d;
                acc += lgamma(gk + es) - lgamma(gk + (double)n + es);
                const double al = (double)__ldg(a.alpha + k);
                acc += lgamma((double)n + al) - lgamma(al);
            }
        }
        uint32_t rb = 0;
        while (rb < L) {            // word cells: per run, each distinct topic once
            const uint32_t v = a.words[b + rb];
            uint32_t re = rb + 1;
            for (;;) {
                const uint32_t j = re + lane;
                const bool diff = j >= L || a.words[b + j] != v;
                const unsigned mm = __ballot_sync(FULL, diff);
                if (mm) { re += __ffs(mm) - 1; break; }
                re += 32;
            }
            if (v < a.V) {
                for (uint32_t j = rb + lane; j < re; j += 32) atomicAdd(&own[a.z[b + j]], 1);
                __syncwarp();
                const float wr = WT ? a.wt[b + rb] : 1.f;    // the run's weight
                const float* pe = nullptr;
                if (a.pidx) {
                    const int p = a.pidx[v];
                    if (p >= 0) pe = a.pval + (uint64_t)p * K;
                }
                for (uint32_t j = rb + lane; j < re; j += 32) {
                    const int k = a.z[b + j];
                    const int c = atomicExch(&own[k], 0);
                    if (c) {
                        const CT gk = __ldg(nkw + (uint64_t)v * K + k);
                        const double ek = pe ? (double)pe[k] : (double)a.eta;
                        double after;
                        if constexpr (WT) after = lgamma(((double)gk + (double)__fmul_rn((float)c, wr)) + ek);
                        else after = lgamma((double)(gk + c) + ek);
                        acc += after - (gk != CT(0) ? lgamma((double)gk + ek) : (pe ? lgamma(ek) : a.lg_eta));
                    }
                }
                __syncwarp();
            }
            rb = re;
        }
        acc = warp_sum(acc);
        if (lane == 0 && a.ll) a.ll[sl] = acc - (lgamma((double)dlen + a.asum_d) - a.lg_asum);
        __syncwarp();
    }
}

// warps per block so that 16 * KP bytes of state per warp fit in 200 KB; 0: too large
inline uint32_t infer_warps(uint32_t K)
{
    const uint32_t per_warp = 16 * round4(K);
    return std::min(8u, (200u * 1024u) / per_warp);
}

template <int CH, bool WT>
inline void launch_infer_t(const InferArgs& a, uint32_t warps, int num_sms, cudaStream_t st)
{
    auto kern = k_infer_slots<CH, WT>;
    const uint32_t smem = warps * 16 * round4(a.K);
    CK(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    int per_sm = 0;
    CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, warps * 32, smem));
    if (per_sm < 1) throw CudaError("infer kernel does not fit on an SM");
    uint32_t grid = (uint32_t)std::min<uint64_t>((uint64_t)per_sm * num_sms, (a.n_work + warps - 1) / warps);
    if (grid == 0) grid = 1;
    kern<<<grid, warps * 32, smem, st>>>(a);
    CK(cudaGetLastError());
}

template <bool WT>
inline void launch_infer_w(const InferArgs& a, uint32_t warps, uint32_t ch, int num_sms, cudaStream_t st)
{
    if (ch <= 1) launch_infer_t<1, WT>(a, warps, num_sms, st);
    else if (ch <= 2) launch_infer_t<2, WT>(a, warps, num_sms, st);
    else if (ch <= 4) launch_infer_t<4, WT>(a, warps, num_sms, st);
    else if (ch <= 8) launch_infer_t<8, WT>(a, warps, num_sms, st);
    else if (ch <= 16) launch_infer_t<16, WT>(a, warps, num_sms, st);
    else if (ch <= 32) launch_infer_t<32, WT>(a, warps, num_sms, st);
    else launch_infer_t<0, WT>(a, warps, num_sms, st);
}

// One launch of the slot kernel for this K (the counter must be zeroed first);
// a.wt != NULL: weighted counts.
inline void launch_infer(const InferArgs& a, int num_sms, cudaStream_t st)
{
    const uint32_t warps = infer_warps(a.K);
    if (warps == 0) throw ArgError("K too large for on-chip inference state");
    const uint32_t ch = (round4(a.K) + 127) / 128;
    if (a.wt) launch_infer_w<true>(a, warps, ch, num_sms, st);
    else launch_infer_w<false>(a, warps, ch, num_sms, st);
}

} // namespace tmtk
