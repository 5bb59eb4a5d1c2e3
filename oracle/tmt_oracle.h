/*
 * tmt_oracle.h -- CPU oracle for the tomotopy LDA collapsed-Gibbs path.
 *
 * TEST INFRASTRUCTURE ONLY.  Nothing in the product library links, loads or
 * calls this code; only tests/, __graft_entry__.smoke() and the CPU-baseline
 * arm of bench.py use it, and only as the checker (or as the timed CPU
 * baseline).  The product path fails loudly when its CUDA library is missing.
 *
 * What it restates (reference paths are relative to the tomotopy source tree):
 *   - the float lgamma / digamma lookup tables        src/Utils/math.h:119-153, src/Utils/LUT.hpp:11-70
 *   - digammaApprox                                   src/Utils/math.h:170-176
 *   - prefixSum (SSE order) / sampleFromDiscreteAcc   src/Utils/sample.hpp:62-86, 133-189
 *   - forShuffled doc order                           src/Utils/Utils.hpp:157-178
 *   - removeStopwords vocab reorder                   src/TopicModel/TopicModel.hpp:526-571
 *   - per-doc word sort (sortAndWriteOrder)           src/Utils/Utils.hpp:227-248, LDAModel.hpp:716-722
 *   - sampleDocument / getZLikelihoods / addWordTo    src/TopicModel/LDAModel.hpp:273-354
 *   - PARTITION scheme (vocab chunks, W rounds)       src/TopicModel/LDAModel.hpp:356-399, 436-489
 *   - getLLDocs / getLLRest                           src/TopicModel/LDAModel.hpp:616-668
 *   - optimizeParameters / calcDigammaSum             src/TopicModel/LDAModel.hpp:221-265
 *   - per-document infer (together=False)             src/TopicModel/LDAModel.hpp:920-953
 *
 * Parity status: the numeric primitives (LUTs, digammaApprox, prefixSum,
 * sampleFromDiscreteAcc, forShuffled, sortAndWriteOrder) are pinned bit-exactly
 * against the reference's own sources compiled from the tomotopy tree into
 * oracle/_ref (see oracle/Makefile and tests/test_oracle_ref.py).  The full
 * sampler is NOT pinned against tomotopy itself: tomotopy's model code needs
 * Eigen 3.4.0 and EigenRand 0.5.1, neither of which exists here, and its RNG
 * (EigenRand P8_mt19937_64_32) is not restated.  Sampler parity is therefore
 * statistical (ll_per_word) plus the exact invariants below.
 *
 * The "snapshot sweep" (orc_sweep_snapshot) defines the device sampler's
 * semantics exactly: every token of a sweep reads the start-of-sweep counts
 * with its own assignment removed, draws with a counter-based Philox4x32-10
 * stream, and the count deltas are applied after the sweep.  Its float
 * arithmetic and summation order are spelled out so that the device dense
 * kernel can be checked bit-exactly against it.
 */
#ifndef TMT_ORACLE_H
#define TMT_ORACLE_H
#include <stdint.h>
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- Philox4x32-10 (Salmon, Moraes, Dror, Shaw, SC'11) ---------------- */
void orc_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]);
/* upper 24 bits of x scaled into [0, 1) */
float orc_u01(uint32_t x);

/* Philox stream tags (third counter word) */
#define ORC_STREAM_INIT  0x494E4954u /* 'INIT' */
#define ORC_STREAM_SWEEP 0x53574550u /* 'SWEP' */
#define ORC_STREAM_INFER 0x494E4652u /* 'INFR' */

/* ---- special functions (reference float LUTs) -------------------------- */
float orc_lgammaT(float x);
float orc_digammaT(float x);
float orc_digammaf(float x);
float orc_digammaApprox(float x);

/* ---- sampling primitives ----------------------------------------------- */
void   orc_prefix_sum_sse(float* arr, int n);
size_t orc_sample_acc(const float* cum, size_t K, float u01);
/* forShuffled: writes the visiting order of N items for `seed` */
void   orc_shuffled_order(size_t N, size_t seed, uint64_t* out);

/* ---- corpus preparation ------------------------------------------------ */
/* removeStopwords: sorts (cf, df) pairs descending with the min_cf/min_df
 * rule and the rm_top rotation.  order[old_id] = new_id.  Returns realV. */
uint64_t orc_remove_stopwords(uint64_t nv, uint64_t* cf, uint64_t* df,
                              uint64_t min_cf, uint64_t min_df, uint64_t rm_top,
                              uint32_t* order);
/* sortAndWriteOrder on one doc: stable sort of words, w_order[old] = new */
void orc_sort_doc(uint32_t* words, size_t n, uint32_t* w_order);

/* z0 ~ Discrete(alpha) per doc-major token i (Philox stream INIT); tokens
 * with word >= V get 0xFFFF (tomotopy's non_topic_id). */
void orc_init_z(uint64_t N, const uint32_t* words, uint32_t V, uint32_t K,
                const float* alpha, uint64_t seed, uint16_t* z);

/* counts from assignments (doc-major CSR) */
void orc_counts_from_z(uint64_t D, const uint64_t* doc_off, const uint32_t* words,
                       const uint16_t* z, uint32_t V, uint32_t K,
                       int32_t* ndk /*D*K*/, int32_t* nkw /*V*K: column v is K ints*/,
                       int32_t* nk /*K*/);

/* word-major layout: stable counting sort of the doc-major tokens by word.
 * w_off[V+1]; tok_doc[Nv]; tok_pos[Nv] = doc-major position. Returns Nv. */
uint64_t orc_word_major(uint64_t D, const uint64_t* doc_off, const uint32_t* words,
                        uint32_t V, uint64_t* w_off, uint32_t* tok_doc, uint64_t* tok_pos);

/* ---- the device sampler's semantics (snapshot sweep) ------------------- */
/* z_old/z_new are word-major.  `iter` is the global step.  Reads only the
 * start-of-sweep counts; does not modify them. */
void orc_sweep_snapshot(uint32_t K, uint32_t V, const float* alpha, float eta,
                        uint64_t seed, uint32_t iter,
                        const uint64_t* w_off, const uint32_t* tok_doc,
                        const int32_t* ndk, const int32_t* nkw, const int32_t* nk,
                        const uint16_t* z_old, uint16_t* z_new);
/* the conditional of one token as FP64 probabilities (normalised), own
 * assignment removed.  For the 1e-5 relative check. */
void orc_conditional_f64(uint32_t K, uint32_t V, const float* alpha, float eta,
                         const int32_t* ndk_row, const int32_t* nkw_col, const int32_t* nk,
                         uint16_t z_own, double* p);
/* apply the deltas of a sweep (word-major z) to the counts, then z_old = z_new */
void orc_apply_sweep(uint32_t K, uint32_t V, const uint64_t* w_off, const uint32_t* tok_doc,
                     int32_t* ndk, int32_t* nkw, int32_t* nk,
                     uint16_t* z_old, const uint16_t* z_new);

/* doc-major sweep: live n_dk; n_kw / n_k read from the start-of-sweep
 * snapshot (own assignment removed) and deltas written to *_next, which the
 * caller initialises as copies of the snapshot.  z is doc-major. */
void orc_sweep_doc_live(uint32_t K, uint32_t V, const float* alpha, float eta,
                        uint64_t seed, uint32_t iter, uint64_t D, const uint64_t* doc_off,
                        const uint32_t* words, int32_t* ndk,
                        const int32_t* nkw, const int32_t* nk,
                        int32_t* nkw_next, int32_t* nk_next, uint16_t* z);
/* the same over a subset of documents (docs[0..n_docs), in that order); the
 * device splits a sweep into G groups of documents this way */
void orc_sweep_doc_live_subset(uint32_t K, uint32_t V, const float* alpha, float eta,
                               uint64_t seed, uint32_t iter, uint64_t D, const uint64_t* doc_off,
                               const uint32_t* words, int32_t* ndk,
                               const int32_t* nkw, const int32_t* nk,
                               int32_t* nkw_next, int32_t* nk_next, uint16_t* z,
                               const uint64_t* docs, uint64_t n_docs);

/* ---- the reference's sequential sampler (ParallelScheme::NONE) ---------- */
/* Doc-major; live counts; forShuffled doc order; SSE prefix sum; strict
 * search.  rng_state is a splitmix64 state (tomotopy's EigenRand stream is
 * not restated). */
void orc_gibbs_none(uint64_t D, const uint64_t* doc_off, const uint32_t* words,
                    uint32_t V, uint32_t K, const float* alpha, float eta,
                    uint16_t* z, int32_t* ndk, int32_t* nkw, int32_t* nk,
                    uint64_t* rng_state);

/* ---- the reference's PARTITION scheme on nthreads host threads ---------- */
/* vocab chunks by cumulative cf; W rounds per sweep; shared nkw (disjoint
 * columns), private nk copies merged by rowsum.  This is the CPU baseline. */
typedef struct orc_partition orc_partition;
orc_partition* orc_partition_create(uint64_t D, const uint64_t* doc_off, const uint32_t* words,
                                    uint32_t V, uint32_t K, const float* alpha, float eta,
                                    uint16_t* z, int32_t* ndk, int32_t* nkw, int32_t* nk,
                                    const uint64_t* vocab_cf, uint32_t nthreads, uint64_t seed);
void orc_partition_train(orc_partition* p, uint32_t iters);
void orc_partition_destroy(orc_partition* p);

/* ---- log-likelihood ---------------------------------------------------- */
/* reference style: float LUT lgamma, double accumulation (LDAModel.hpp:616-668) */
double orc_ll_docs_lut(uint64_t D, uint32_t K, const int32_t* ndk, const int32_t* doc_len,
                       const float* alpha);
double orc_ll_rest_lut(uint32_t K, uint32_t V, const int32_t* nkw, const int32_t* nk, float eta);
/* FP64: lgamma() in double, same terms */
double orc_ll_docs_f64(uint64_t D, uint32_t K, const int32_t* ndk, const int32_t* doc_len,
                       const float* alpha);
double orc_ll_rest_f64(uint32_t K, uint32_t V, const int32_t* nkw, const int32_t* nk, float eta);

/* ---- alpha optimisation (Minka fixed point, 10 inner iterations) -------- */
void orc_optimize_alpha(uint64_t D, uint32_t K, const int32_t* ndk, const int32_t* doc_len,
                        float* alpha);

/* ---- per-document infer (together=False) -------------------------------- */
/* The device infer semantics for one prepared (vid-sorted) document against
 * a frozen model (LDAModel.hpp:920-953, _getTopicsByDoc :1145-1159): writes
 * z, the doc's topic counts and theta (may be NULL); returns the FP64 ll =
 * LLRest(model + doc) - LLRest(model) + LLDocs(doc). */
double orc_infer_doc(uint32_t K, uint32_t V, const float* alpha, float eta,
                     const int32_t* nkw, const int32_t* nk,
                     const uint32_t* words, uint32_t len, uint32_t iters,
                     uint64_t seed, uint64_t doc_key, uint16_t* z, int32_t* ndk_out, float* theta);

/* ---- weighted counts: TermWeight IDF / PMI ----------------------------- */
/* Tokens carry float weights (LDAModel.hpp:795-809, 1093-1122); counts are
 * float sums and decrements clamp at 0 (Utils.hpp:132-155).  Device
 * semantics: n_dk rows change in float in token order; n_kw / n_k are float
 * states folded between document groups from integer deltas in units of
 * 2^-24 (orc_wq), so the fold does not depend on the order of the adds. */
int64_t orc_wq(float w);                 /* llrintf(w * 2^24) */
float   orc_fold(float n, int64_t q);    /* max(n + (float)q * 2^-24, 0) */
void orc_fold_w(uint32_t K, uint32_t V, float* nkw, float* nk, int64_t* dkw, int64_t* dk);
/* counts from z: n_dk and the document weight sums in token order (the
 * reference's accumulation), n_kw / n_k folded from zero */
void orc_counts_from_z_w(uint64_t D, const uint64_t* doc_off, const uint32_t* words,
                         const uint16_t* z, const float* wt, uint32_t V, uint32_t K,
                         float* ndk, float* doc_wlen, float* nkw, float* nk);
/* one document group of a weighted sweep: reads the folded state, writes
 * deltas to dkw / dk */
void orc_sweep_doc_live_w_subset(uint32_t K, uint32_t V, const float* alpha, float eta,
                                 uint64_t seed, uint32_t iter, const uint64_t* doc_off,
                                 const uint32_t* words, const float* wt, float* ndk,
                                 const float* nkw, const float* nk, int64_t* dkw, int64_t* dk,
                                 uint16_t* z, const uint64_t* docs, uint64_t n_docs);
double orc_ll_docs_w_f64(uint64_t D, uint32_t K, const float* ndk, const float* doc_wlen,
                         const float* alpha);
double orc_ll_rest_w_f64(uint32_t K, uint32_t V, const float* nkw, const float* nk, float eta);
void orc_optimize_alpha_w(uint64_t D, uint32_t K, const float* ndk, const float* doc_wlen, float* alpha);
/* per-document infer against a frozen weighted model; words sorted by id,
 * every token of one word carrying the same weight */
double orc_infer_doc_w(uint32_t K, uint32_t V, const float* alpha, float eta,
                       const float* nkw, const float* nk,
                       const uint32_t* words, const float* wt, uint32_t len, uint32_t iters,
                       uint64_t seed, uint64_t doc_key, uint16_t* z, float* ndk, float* theta);

/* ---- word priors (set_word_prior; LDAModel.hpp:99-117, 636-651, 724-737, 765-779) --- */
/* pidx[v] >= 0: word v's eta column is row pidx[v] of prior (K floats), else
 * eta everywhere; esum[k] = the rows' sums rounded once from double. */
void orc_prior_esum(uint32_t K, uint32_t V, const int32_t* pidx, const float* prior, float eta, float* esum);
void orc_init_z_p(uint64_t N, const uint32_t* words, uint32_t V, uint32_t K, const int32_t* pidx,
                  const float* prior, float eta, uint64_t seed, uint16_t* z);
void orc_sweep_doc_live_p_subset(uint32_t K, uint32_t V, const float* alpha, float eta,
                                 const int32_t* pidx, const float* prior, const float* esum,
                                 uint64_t seed, uint32_t iter, const uint64_t* doc_off,
                                 const uint32_t* words, int32_t* ndk,
                                 const int32_t* nkw, const int32_t* nk,
                                 int32_t* nkw_next, int32_t* nk_next, uint16_t* z,
                                 const uint64_t* docs, uint64_t n_docs);
double orc_ll_rest_p_f64(uint32_t K, uint32_t V, const int32_t* nkw, const int32_t* nk, float eta,
                         const int32_t* pidx, const float* prior, const float* esum);
double orc_infer_doc_p(uint32_t K, uint32_t V, const float* alpha, float eta,
                       const int32_t* pidx, const float* prior, const float* esum,
                       const int32_t* nkw, const int32_t* nk,
                       const uint32_t* words, uint32_t len, uint32_t iters,
                       uint64_t seed, uint64_t doc_key, uint16_t* z, int32_t* ndk, float* theta);

/* ---- per-document topic masks and alphas (LLDA / PLDA / DMR conditionals) -- */
/* A_k = ((float)n_dk + alpha_dk) * m_dk; mask: D rows of ceil(K/32) words or
 * NULL; arow: per-document rows of alpha_rows (M x K) or NULL */
void orc_sweep_doc_live_m_subset(uint32_t K, uint32_t V, const float* alpha, const float* alpha_rows,
                                 const uint32_t* arow, const uint32_t* mask, float eta,
                                 uint64_t seed, uint32_t iter, const uint64_t* doc_off,
                                 const uint32_t* words, int32_t* ndk,
                                 const int32_t* nkw, const int32_t* nk,
                                 int32_t* nkw_next, int32_t* nk_next, uint16_t* z,
                                 const uint64_t* docs, uint64_t n_docs);
double orc_ll_docs_m_f64(uint64_t D, uint32_t K, const int32_t* ndk, const int32_t* doc_len,
                         const float* alpha_rows, const uint32_t* arow);

/* ---- the device sweep with every option and the long-document split ----- */
typedef struct {
    uint32_t K, V;
    const float* alpha; float eta;
    const int32_t* pidx; const float* prior; const float* esum;   /* word priors or NULL */
    const float* alpha_rows; const uint32_t* arow;                /* per-document alphas or NULL */
    const uint32_t* mask;                                         /* D x ceil(K/32) or NULL */
    uint64_t seed; uint32_t iter;
    const uint64_t* doc_off; const uint32_t* words;
    int32_t* ndk; const int32_t* nkw; const int32_t* nk;
    int32_t* nkw_next; int32_t* nk_next; uint16_t* z;
    uint64_t split_len; uint32_t slices, step;   /* split_len 0: no document is split */
    /* shared rows (PT's pseudo-documents): docs[] then lists rows; row r's
     * documents are unit_docs[unit_off[r] .. unit_off[r+1]), sampled one after
     * another with the row live; NULL: every document is its own row */
    const uint64_t* unit_off; const uint32_t* unit_docs;
} orc_sweep_spec;
/* the documents docs[0 .. n_docs) of one group (see tmt_oracle.c) */
void orc_sweep_docs(const orc_sweep_spec* sp, const uint64_t* docs, uint64_t n_docs);

/* ---- the conditional a draw implies (gate: 1e-5 of FP64) ---------------- */
/* width[k]: the length of the r-interval (r = u * total) mapped to topic k by
 * the device's blocked draw (A with the token removed, phi the word's table
 * column, phi_own the own topic's weight); returns total. */
float orc_draw_intervals(const float* A, const float* phi, uint32_t K, uint32_t zo, float phi_own,
                         double* width, double* start);
uint32_t orc_blocked_draw(const float* A, const float* phi, uint32_t K, uint32_t zo, float phi_own, float u);
/* the same for tomotopy's draw over dist_k = (A_k * B_k) / C_k (SSE prefix sum) */
float orc_ref_draw_intervals(const float* A, const float* B, const float* C, uint32_t K, double* width);

/* ---- the reference's sequential sampler with weights / word priors ------- */
void orc_gibbs_none_w(uint64_t D, const uint64_t* doc_off, const uint32_t* words, const float* wt,
                      uint32_t V, uint32_t K, const float* alpha, float eta,
                      uint16_t* z, float* ndk, float* nkw, float* nk, uint64_t* rng_state);
void orc_gibbs_none_p(uint64_t D, const uint64_t* doc_off, const uint32_t* words,
                      uint32_t V, uint32_t K, const float* alpha, float eta,
                      const int32_t* pidx, const float* prior, const float* esum,
                      uint16_t* z, int32_t* ndk, int32_t* nkw, int32_t* nk, uint64_t* rng_state);

/* ---- the benchmark workload without the engine (CPU baseline) ------------ */
typedef struct {
    uint32_t V, T;           /* vocabulary, true topics */
    uint64_t D;              /* documents */
    int32_t len_kind;        /* 0 Poisson, 1 lognormal */
    double len_a, len_b;     /* Poisson mean | lognormal mu, sigma */
    uint32_t len_min, len_max;
    double doc_alpha, topic_beta, zipf_s;
    uint64_t seed, doc_offset;
} orc_synth_spec;
/* the seeded synthetic corpus (tomotopy_b200/csrc/synth.cpp restated): words
 * NULL fills doc_off[D+1] and *n_tokens only; 0 on success */
int orc_synth_corpus(const orc_synth_spec* s, uint64_t* doc_off, uint32_t* words, uint64_t capacity,
                     uint64_t* n_tokens, uint32_t threads);
/* removeStopwords + prepareDoc of a whole corpus in place; returns realV */
uint64_t orc_prepare_corpus(uint64_t D, const uint64_t* doc_off, uint32_t* words, uint64_t nv,
                            uint64_t min_cf, uint64_t min_df, uint64_t rm_top, uint32_t* order, uint32_t threads);

#ifdef __cplusplus
}
#endif
#endif
