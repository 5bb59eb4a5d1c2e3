/*
 * tomotopy_b200.h -- C ABI of the B200 collapsed-Gibbs LDA engine.
 *
 * This is the drop-in boundary for tomotopy's plain LDAModel hot path.  Each
 * entry point names the tomotopy interface it replaces (paths relative to
 * the tomotopy source tree).  Conventions:
 *   - status codes only (tmt_status); no C++ exception crosses this ABI;
 *     tmt_last_error() returns the message of a handle's last failure;
 *   - the caller owns every host buffer; a handle owns its device buffers;
 *   - calls on one handle are serialised by the caller (tomotopy holds the
 *     GIL across train/infer, py_LDA.cpp:277-411); the server functions are
 *     internally thread-safe;
 *   - word ids >= V (tomotopy's realV, the vocabulary after stop-word
 *     removal) are carried but never sampled, as in LDAModel.hpp:339;
 *   - topic ids are uint16 (tomotopy's Tid, Dictionary.h:16), so 1 <= K <= 32767
 *     (models.py:84);  count matrices are int32 (TermWeight::one);
 *   - n_kw is K x V column-major: column v holds K contiguous int32, the
 *     layout of ModelStateLDA::numByTopicWord (LDAModel.hpp:61-67, LDA.h:80-95);
 *   - n_dk is D x K row-major: row d holds K contiguous int32, one
 *     DocumentLDA::numByTopic per document (LDA.h:146).
 */
#ifndef TOMOTOPY_B200_H
#define TOMOTOPY_B200_H
#include <stdint.h>
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum tmt_status {
    TMT_OK = 0,
    TMT_ERR_INVALID_ARGUMENT = -1,  /* tomotopy: exc::InvalidArgument -> ValueError */
    TMT_ERR_CUDA = -2,
    TMT_ERR_OUT_OF_MEMORY = -3,     /* device allocation or HBM budget exceeded */
    TMT_ERR_STATE = -4,             /* call out of order (e.g. train before upload) */
    TMT_ERR_UNSUPPORTED = -5,
    TMT_ERR_CANCELLED = -6,
    TMT_ERR_TIMEOUT = -7,
    TMT_ERR_INTERNAL = -8           /* tomotopy: train() < 0 -> RuntimeError("Train failed") */
} tmt_status;

typedef struct tmt_handle tmt_handle;

/* Sampler kernels for the training sweep. */
typedef enum tmt_sampler {
    TMT_SAMPLER_AUTO = 0,   /* the engine's choice: the dense sampler */
    TMT_SAMPLER_DENSE = 1,  /* full K-vector conditional per token */
    TMT_SAMPLER_SPARSE = 2  /* not built: tmt_create returns TMT_ERR_UNSUPPORTED.  The exact bucket
                               decomposition of the conditional pays when documents and words hold
                               few nonzero topics; documents of the benchmark corpora keep ~160
                               nonzero topics at K = 1000 and their frequent words' columns are
                               dense, so the buckets would gather more per token than the dense
                               pass loads */
} tmt_sampler;

/* Model hyper-parameters.  Mirrors LDAArgs (LDA.h:170-176) plus the
 * optimiser settings of LDAModel (LDAModel.hpp:210). */
typedef struct tmt_config {
    uint32_t K;              /* topics, 1..32767 */
    uint32_t V;              /* realV: word ids >= V are skipped */
    const float* alpha;      /* K Dirichlet doc-topic priors, or NULL to use alpha_scalar */
    float alpha_scalar;
    float eta;               /* symmetric topic-word prior, > 0 */
    uint64_t seed;
    uint32_t optim_interval; /* re-fit alpha every n sweeps after burn_in; 0 = never (tomotopy default 10) */
    uint32_t burn_in;
    int32_t device;          /* CUDA device ordinal */
    int32_t sampler;         /* tmt_sampler */
    uint64_t hbm_budget;     /* bytes this handle may allocate; 0 = unlimited */
    uint32_t sweep_groups;   /* documents per sweep are sampled in this many groups, the
                                n_kw / n_k snapshot refreshed between groups; 0 = 1 */
} tmt_config;

/* Read-only facts about a handle. */
typedef struct tmt_info {
    uint64_t D;              /* documents */
    uint64_t N_all;          /* tokens uploaded (all word ids) */
    uint64_t N;              /* tokens sampled (word id < V) */
    uint64_t global_step;    /* sweeps done (TopicModel::globalStep) */
    uint64_t device_bytes;   /* device memory held by the handle */
    uint32_t K, V;
    int32_t sampler;         /* the sampler the last sweep used */
    float last_sweep_ms;     /* device time of the last sweep (CUDA events) */
    uint64_t kernel_launches;/* kernels launched by this handle so far */
    double sweep_kernel_ms;  /* device time of the sweep kernels of the last tmt_train call */
    uint32_t sweeps_timed;   /* sweeps in that sum */
    uint32_t sweep_groups;   /* document groups per sweep in use */
    double train_ms;         /* device time of the last tmt_train call, first sweep to last (CUDA events) */
    uint32_t rank, world;    /* this handle's shard of a corpus split across ranks (0, 1: unsharded) */
} tmt_info;

/* Replaces ILDAModel::create (LDAModel.cpp:10-13) + the LDAModel ctor checks
 * (LDAModel.hpp:962-983): K in 1..32767, alpha > 0, eta > 0. */
tmt_status tmt_create(const tmt_config* cfg, tmt_handle** out);

/* Replaces LDAModel::prepare's device-relevant part (LDAModel.hpp:1073-1138):
 * uploads the doc-major corpus (words already vocab-reordered and sorted by
 * id inside each document, as prepareDoc does, LDAModel.hpp:716-722), draws
 * z0 ~ Discrete(alpha) (initializeDocState, LDAModel.hpp:781-813) unless z0
 * is given, and builds n_dk, n_kw and n_k.
 * wid[doc_off[D]], doc_off[D+1]; z0 is doc-major or NULL. */
tmt_status tmt_upload_corpus(tmt_handle* h, const uint32_t* wid, const uint64_t* doc_off,
                             uint64_t D, const uint16_t* z0);

/* tmt_upload_corpus with weighted counts: the LDAModel<TermWeight::idf|pmi>
 * instantiations (LDAModel.hpp:287-299 addWordTo with doc.wordWeights, the
 * weights set in initializeDocState, :795-809).  weights[i] is token i's
 * weight (the caller computes tomotopy's IDF / PMI weights; entries of
 * words >= V are ignored), finite, in [0, 65536], all together below 2^38.
 * n_dk, n_kw and n_k are then float sums of weights; a removal clamps at 0
 * (updateCnt<true>, Utils.hpp:132-155); each document's length is its weight
 * sum (SumWordWeight, LDA.h:104-117), used by the log-likelihood and the
 * alpha optimiser.  n_dk rows change in float in token order; n_kw / n_k are
 * float states that change between document groups by integer deltas in
 * units of 2^-24, so results do not depend on the order of atomic adds.
 * Single GPU only (a sharded corpus is rejected). */
tmt_status tmt_upload_corpus_weighted(tmt_handle* h, const uint32_t* wid, const uint64_t* doc_off,
                                      uint64_t D, const uint16_t* z0, const float* weights);

/* Documents sharded across GPUs: tomotopy's COPY_MERGE scheme
 * (LDAModel.hpp:555-570) with the workers on different devices.  Rank r holds
 * the contiguous global documents [doc_begin, doc_begin + D) and a replica of
 * n_kw / n_k.  The document groups are cut over the GLOBAL longest-first order,
 * so every group's snapshot is the same on every rank; after each group the
 * ranks' integer count deltas (n_kw then n_k, K*V + K int32) are summed by
 * `allreduce`, and the next group starts from the summed state.  Draws use the
 * global token index, so z and every count equal those of one GPU holding the
 * whole corpus, bit for bit (with the alpha optimisation the digamma sums are
 * reduced in another order: equal up to FP64 rounding).
 *
 * allreduce(user, buf, count, dtype, stream): an in-place SUM over all ranks of
 * `count` elements (dtype TMT_I32 or TMT_F64) of DEVICE memory, ordered on the
 * CUDA stream `stream` (a cudaStream_t); returns 0 on success.  Every rank makes
 * the same calls in the same order. */
enum { TMT_I32 = 0, TMT_F64 = 1 };
typedef int32_t (*tmt_allreduce_fn)(void* user, void* buf, uint64_t count, int32_t dtype, void* stream);
typedef struct tmt_shard {
    uint32_t rank, world;
    uint64_t D_global;                /* documents over all ranks */
    uint64_t doc_begin;               /* global index of this rank's first document */
    const uint64_t* doc_len_global;   /* D_global document lengths (all words), rank order */
    tmt_allreduce_fn allreduce;
    void* user;
} tmt_shard;

/* The plan behind tmt_upload_shard (host only): the global longest-first order
 * cut into `groups` equal-token ranges, as tmt_upload_corpus cuts one corpus.
 * local_order[D_local] = this rank's documents (local indices) in global order;
 * local_bounds[groups + 1]: group g is local_order[local_bounds[g] ..
 * local_bounds[g+1]); global_bounds[groups + 1] (nullable): the groups'
 * document counts over all ranks, as prefix bounds; *token_offset (nullable) =
 * the global index of this rank's first token. */
tmt_status tmt_plan_shard(const uint64_t* doc_len_global, uint64_t D_global, uint32_t groups, uint64_t doc_begin,
                          uint64_t D_local, uint32_t* local_order, uint64_t* local_bounds, uint64_t* global_bounds,
                          uint64_t* token_offset);

/* tmt_upload_corpus for one rank of a sharded corpus (see tmt_shard); the
 * counts after z0 are summed over the ranks. */
tmt_status tmt_upload_shard(tmt_handle* h, const uint32_t* wid, const uint64_t* doc_off, uint64_t D,
                            const uint16_t* z0, const tmt_shard* shard);

/* Replaces TopicModel::train (TopicModel.hpp:684-755) -> LDAModel::trainOne
 * (LDAModel.hpp:505-539): `iters` sweeps, each = sampling (performSampling /
 * sampleDocument, :326-428) + count merge (mergeState, :552-580) + alpha
 * optimisation when due (:529-532).  When ll_every > 0 and ll_out != NULL,
 * writes the FP64 log-likelihood after every ll_every-th sweep
 * (iters / ll_every values). */
tmt_status tmt_train(tmt_handle* h, uint32_t iters, uint32_t ll_every, double* ll_out);

/* Replaces getLLDocs / getLLRest (LDAModel.hpp:616-668) in FP64:
 * ll_docs over n_dk, ll_rest over n_kw and n_k.  ll_per_word =
 * (ll_docs + ll_rest) / N (TopicModel.hpp:757-760). */
tmt_status tmt_ll(tmt_handle* h, double* ll_docs, double* ll_rest);

/* Downloads the model state (any pointer may be NULL): z doc-major
 * (N_all uint16, 0xFFFF for skipped words; DocumentLDA::Zs), n_kw (K x V
 * column-major), n_k (K), alpha (K, after optimisation).  Synchronous.  This
 * and the other downloads copy directly into memory CUDA knows (pinned host
 * memory, or device or managed memory); a plain pageable destination above
 * 32 MB is filled through two 32 MB pinned staging buffers by up to 16 host
 * threads.  The staging buffers are shared by all handles of the process
 * (one staged transfer at a time) and kept until the process exits. */
tmt_status tmt_download_state(tmt_handle* h, uint16_t* z, int32_t* n_kw, int32_t* n_k, float* alpha);

/* Replaces the topic-word state with host arrays n_kw (K x V column-major)
 * and n_k (K): the state a model loaded without its documents carries
 * (TopicModel::_loadModel, TopicModel.hpp:361-395).  Later sweeps and
 * inference use it. */
tmt_status tmt_set_counts(tmt_handle* h, const int32_t* n_kw, const int32_t* n_k);
/* Per-document topic masks: the label masks of LLDAModel (getZLikelihoods
 * multiplies the conditional by doc.labelMask, LLDAModel.hpp:37-48) and
 * PLDAModel (PLDAModel.hpp:39).  mask_bits holds D rows of ceil(K/32) words;
 * bit k of row d allows topic k in document d.  A masked topic's weight is
 * exactly 0; unmasked topics are unchanged.  After the upload (pass z0 drawn
 * inside the masks to the upload); NULL clears.  Single GPU. */
tmt_status tmt_set_doc_topic_mask(tmt_handle* h, const uint32_t* mask_bits);
/* Per-document alphas: DMRModel's getCachedAlpha (DMRModel.hpp:193-206).
 * alpha_rows is M x K (> 0); document d uses row doc_row[d] in the
 * conditional and in the log-likelihood (DMR's getLLDocTopic, :208-224); the
 * alpha optimiser is skipped (DMR fits its own lambda).  After the upload;
 * alpha_rows == NULL clears.  Single GPU. */
tmt_status tmt_set_doc_alpha(tmt_handle* h, uint32_t M, const float* alpha_rows, const uint32_t* doc_row);
/* Shared document rows: PTModel's pseudo-documents (PTModel.hpp:13-24, 72-114).
 * Document d's tokens count in row row_of_doc[d] of an R x K n_dk (the
 * pseudo-document's numByTopicPDoc column) instead of its own row: the
 * conditional's document factor is (n_row,k + alpha_k), a sweep samples each
 * row's documents one after another (ascending document index) with the row
 * live -- as PT's PARTITION keeps a pseudo-document's documents on one worker
 * (PTModel.hpp:206-235) -- and the rows are scheduled like documents (longest
 * first, equal-token groups).  The rows are recounted from z on every call,
 * so a caller that re-assigns pseudo-documents (PTModel::samplePseudoDoc,
 * every pseudoDocSamplingInterval sweeps; it stays on the host) calls this
 * again.  tmt_ll's ll_docs and the alpha optimiser then run over the R rows
 * (PTModel::getLLRest's pseudo-document terms, without the lambda term over
 * numDocsByPDoc, which the caller adds; PTModel::optimizeParameters);
 * tmt_download_doc_topic returns the R rows.  Documents are not split.
 * After the upload; integer counts, one GPU, no per-document masks or alphas;
 * row_of_doc == NULL returns to one row per document (recounted from z). */
tmt_status tmt_set_doc_rows(tmt_handle* h, uint64_t R, const uint32_t* row_of_doc);
/* Word priors: LDAModel::setWordPrior (LDAModel.hpp:1031-1045) as applied by
 * prepareWordPriors (:724-737).  Word word_ids[p] (< V, each once) gets the
 * K-vector priors[p*K .. p*K+K-1] (finite, >= 0) as its eta column; every
 * other word keeps the scalar eta.  The conditional uses eta_kv and the
 * per-topic sums of eta over the words (getZLikelihoods<true>, :273-285),
 * z0 of every token is drawn from its word's eta column (updateStateWithDoc,
 * :765-779), and the log-likelihood and inference use the same table
 * (getLLRest, :636-651).  Call before the upload; P = 0 clears. */
tmt_status tmt_set_word_priors(tmt_handle* h, uint32_t P, const uint32_t* word_ids, const float* priors);
/* tmt_set_counts for weighted counts (tmt_upload_corpus_weighted): n_kw (V x K
 * floats, column v = K values) and n_k (K); values finite and >= 0. */
tmt_status tmt_set_counts_f32(tmt_handle* h, const float* n_kw, const float* n_k);
/* Replaces alpha (K values > 0), e.g. the optimised alphas of a loaded model. */
tmt_status tmt_set_alpha(tmt_handle* h, const float* alpha);
/* Sets the sweep counter (TopicModel::globalStep), e.g. after a load; it keys
 * the draws and the alpha-optimisation schedule. */
tmt_status tmt_set_global_step(tmt_handle* h, uint64_t step);
/* Sets the seed that keys the sweep draws (the model's random generator, which
 * tomotopy's copy() carries over: LDAModel.hpp copy constructor via TopicModel's rg). */
tmt_status tmt_set_seed(tmt_handle* h, uint64_t seed);
/* Sets the alpha-optimisation schedule between train() calls
 * (LDAModel::optimInterval / burnIn, python setters py_LDA.cpp). */
tmt_status tmt_set_optim(tmt_handle* h, uint32_t optim_interval, uint32_t burn_in);
/* Long documents.  A document of at least split_len tokens (all ids counted)
 * is sampled by one block as 8 slices of contiguous positions side by side,
 * each with a private copy of the document's n_dk row that takes in the other
 * slices' changes every `step` positions -- the within-document counterpart of
 * tomotopy's PARTITION chunks (LDAModel.hpp:436-489: a document's tokens split
 * by vocabulary range; its sorted tokens make each slice a vocabulary range).
 * Without it one warp samples a document in order and the document's length
 * bounds its group's time.  Default (min_tokens = 0): per document group,
 * split_len = max(8 * 7 * step, ceil(group tokens / 4096)) -- a split
 * document is at least 8 times the 7 * step tokens a draw may see stale --
 * for integer counts with K <= 512; min_tokens >= 2^32 - 1: never; step 0: 16.  The split
 * depends only on the corpus and these settings (never on timing or the
 * device), so results stay bit-reproducible. */
tmt_status tmt_set_doc_split(tmt_handle* h, uint64_t min_tokens, uint32_t step);
/* Per document group, how many documents are split (*n = groups). */
tmt_status tmt_get_doc_split(const tmt_handle* h, uint32_t* n_long, uint32_t cap, uint32_t* n);
/* Single GPU: after the autotuner's first sweeps, each sweep is one launch of
 * a CUDA graph holding the sweep's kernels (default on).  0 launches every
 * kernel from the host instead; results are identical either way.  Replaces
 * nothing in tomotopy: the loop it captures is TopicModel::train's
 * (TopicModel.hpp:684-755) iteration over trainOne. */
tmt_status tmt_set_graphs(tmt_handle* h, int32_t enable);
/* The sweep-kernel variant the autotuner chose for each document group
 * (-1 while tuning); *n = the number of groups.  Diagnostics only. */
tmt_status tmt_get_sweep_variants(const tmt_handle* h, int32_t* out, uint32_t cap, uint32_t* n);
/* The autotuner's measurements: out[g * n_variants + v] = milliseconds of
 * group g's launches under variant v, summed over the tuning sweeps that ran
 * it (0 where none has); *n_groups, *n_variants.  Diagnostics only. */
tmt_status tmt_get_sweep_timings(const tmt_handle* h, float* out, uint32_t cap, uint32_t* n_groups,
                                 uint32_t* n_variants);

/* Weighted counts (tmt_upload_corpus_weighted): n_dk (D x K row-major),
 * n_kw (V x K, column v = K floats: numByTopicWord of ModelStateLDA<float>),
 * n_k (K) and the document weight sums (D); any pointer may be NULL.
 * Integer-count corpora return TMT_ERR_STATE (use tmt_download_state). */
tmt_status tmt_download_counts_f32(tmt_handle* h, float* n_dk, float* n_kw, float* n_k, float* doc_wlen);

/* Downloads n_dk (D x K row-major int32; DocumentLDA::numByTopic). */
tmt_status tmt_download_doc_topic(tmt_handle* h, int32_t* n_dk);

/* Replaces LDAModel::_infer<together = false> (LDAModel.hpp:920-953) behind
 * TopicModel::infer (TopicModel.hpp:842-875): each of the D documents
 * (doc-major ids in the model's vocabulary; ids >= V are carried but not
 * sampled) gets a private copy of the handle's current model with its own
 * tokens added, z0 ~ Discrete(alpha), then `iters` sequential Gibbs sweeps.
 * Outputs (host, may be NULL): theta[D x K] = (n_dk + alpha) / (N_d +
 * sum(alpha)) (_getTopicsByDoc, LDAModel.hpp:1145-1159) and ll[D] =
 * LLRest(model + doc) - LLRest(model) + LLDocs(doc) in FP64.  Documents are
 * sorted by id internally, as prepareDoc does.  Draws are keyed by seed and
 * doc_keys[d] (NULL: key 0 for every document, as tomotopy starts every
 * document's chain from a freshly seeded generator), so a document's result
 * does not depend on the other documents of the call.  The model is not
 * changed. */
tmt_status tmt_infer_batch(tmt_handle* h, const uint32_t* wid, const uint64_t* doc_off, uint64_t D,
                           uint32_t iters, uint64_t seed, const uint64_t* doc_keys, float* theta, double* ll);
/* tmt_infer_batch for a model with weighted counts (tmt_upload_corpus_weighted):
 * weights[i] is token i's weight, computed by the caller as tomotopy does for
 * new documents (IDF: the word's vocabWeights entry; PMI: from the word's
 * count in the document, LDAModel.hpp:795-809); every token of one word in a
 * document must carry the same weight.  n_dk is a float sum of weights, theta
 * divides by the document's weight sum (_getTopicsByDoc, LDAModel.hpp:1145-1159). */
tmt_status tmt_infer_batch_weighted(tmt_handle* h, const uint32_t* wid, const uint64_t* doc_off, uint64_t D,
                                    const float* weights, uint32_t iters, uint64_t seed, const uint64_t* doc_keys,
                                    float* theta, double* ll);

/* ---- served inference: continuous batching over resident frozen models ----
 * No single tomotopy counterpart: it serves tomotopy's infer() (models.py:354,
 * LDAModel.hpp:920-953) as a request loop.  A worker thread admits submitted
 * documents into free slots of their model and into free space of the token
 * arena (token_budget tokens: the HBM budget for documents in flight), and
 * each step advances every active document by ceil(step_token_sweeps /
 * length) sweeps on the device; requests that arrive while others run join
 * at the next step.  A finished document's theta and ll are those of
 * tmt_infer_batch for the same model, words, iters, seed and key, whatever
 * else shares the GPU.  All functions are thread-safe. */
typedef struct tmt_server tmt_server;
typedef struct tmt_server_config {
    int32_t device;
    uint32_t max_slots;          /* documents in flight per model */
    uint64_t token_budget;       /* tokens in flight over all models */
    uint32_t step_token_sweeps;  /* work per document per step, in token-sweeps (0: 4096) */
    uint32_t max_doc_len;        /* longer documents are rejected */
} tmt_server_config;
typedef struct tmt_server_stats {
    uint64_t steps, completed, queued;
    double mean_active;          /* documents per step, averaged over steps */
    uint64_t tokens_in_flight_max;
    uint64_t token_sweeps;       /* token-sweeps advanced (document length x sweeps) */
    double alg_bytes;            /* token-sweeps x (4K + 8): the frozen n_kw column per draw + z */
    double kernel_ms;            /* device time of the inference launches (CUDA events) */
    double busy_ms;              /* wall time of the steps */
} tmt_server_stats;

tmt_status tmt_server_start(const tmt_server_config* cfg, tmt_server** out);
/* Makes a frozen model resident: host arrays n_kw (K x V column-major), n_k,
 * alpha; returns its id.  Call before submitting to it. */
tmt_status tmt_server_add_model(tmt_server* s, uint32_t K, uint32_t V, const float* alpha, float eta,
                                const int32_t* n_kw, const int32_t* n_k, uint32_t* model_id);
/* Queues one document (ids in the model's vocabulary); returns at once. */
/* tmt_server_add_model for a model with weighted counts (TermWeight IDF /
 * PMI: n_kw V x K and n_k K as floats); its requests come through
 * tmt_server_submit_weighted / tmt_server_submit_batch_weighted, which carry
 * each token's weight (the same weight for every token of one word in a
 * document, as the weights of tmt_infer_batch_weighted). */
tmt_status tmt_server_add_model_f32(tmt_server* s, uint32_t K, uint32_t V, const float* alpha, float eta,
                                    const float* n_kw, const float* n_k, uint32_t* model_id);
tmt_status tmt_server_submit_weighted(tmt_server* s, uint32_t model_id, const uint32_t* wid, const float* weights,
                                      uint32_t len, uint32_t iters, uint64_t seed, uint64_t key, uint64_t* request_id);
tmt_status tmt_server_submit_batch_weighted(tmt_server* s, const uint32_t* model_ids, const uint32_t* wid,
                                            const float* weights, const uint64_t* doc_off, uint64_t n, uint32_t iters,
                                            uint64_t seed, const uint64_t* keys, uint64_t* request_ids);
/* Word priors of a resident model (tmt_set_word_priors' table: word_ids[p] < V
 * gets the K-vector priors[p*K ..] as its eta column); only before the model's
 * first request (TMT_ERR_STATE after). */
tmt_status tmt_server_set_model_priors(tmt_server* s, uint32_t model_id, uint32_t P, const uint32_t* word_ids,
                                       const float* priors);
tmt_status tmt_server_submit(tmt_server* s, uint32_t model_id, const uint32_t* wid, uint32_t len, uint32_t iters,
                             uint64_t seed, uint64_t key, uint64_t* request_id);
/* Waits up to wait_ms for a finished document; TMT_ERR_TIMEOUT when none.
 * theta gets the model's K values (theta_cap >= K); latency_ms is submit to
 * completion. */
tmt_status tmt_server_poll(tmt_server* s, uint32_t wait_ms, uint64_t* request_id, uint32_t* model_id,
                           float* theta, uint32_t theta_cap, double* ll, double* latency_ms);
/* Queues n documents (document d = wid[doc_off[d] .. doc_off[d+1]), model
 * model_ids[d], key keys[d] or 0) under one lock; request_ids[d] gets each id. */
tmt_status tmt_server_submit_batch(tmt_server* s, const uint32_t* model_ids, const uint32_t* wid,
                                   const uint64_t* doc_off, uint64_t n, uint32_t iters, uint64_t seed,
                                   const uint64_t* keys, uint64_t* request_ids);
/* Waits up to wait_ms for finished documents and returns up to max_n of them
 * (*n_out); result i has theta at theta + i * theta_stride (theta_stride >= K). */
tmt_status tmt_server_poll_batch(tmt_server* s, uint32_t wait_ms, uint64_t max_n, uint64_t* request_ids,
                                 uint32_t* model_ids, float* theta, uint32_t theta_stride, double* ll,
                                 double* latency_ms, uint64_t* n_out);
tmt_status tmt_server_get_stats(tmt_server* s, tmt_server_stats* out);
const char* tmt_server_last_error(const tmt_server* s);
/* Stops the worker (queued and running documents are dropped) and frees the server. */
tmt_status tmt_server_stop(tmt_server* s);

/* Host-side preparation of an integer-id corpus, replacing the vocabulary
 * part of LDAModel::prepare (LDAModel.hpp:1073-1138): removeStopwords
 * (TopicModel.hpp:526-571) reorders ids by (cf, df) descending with the
 * min_cf / min_df / rm_top rules and yields realV; prepareDoc
 * (LDAModel.hpp:716-722) sorts every document by the new ids.  Outputs:
 * words_out[N] (doc-major, re-numbered, sorted per doc), w_order[N]
 * (w_order[original position] = sorted position within the doc; may be NULL),
 * vocab_order[n_vocab] (old id -> new id), vocab_cf / vocab_df (by new id;
 * may be NULL), *real_v. */
tmt_status tmt_prepare_corpus(uint64_t D, const uint64_t* doc_off, const uint32_t* words,
                              uint32_t n_vocab, uint64_t min_cf, uint64_t min_df, uint64_t rm_top,
                              uint32_t* words_out, uint32_t* w_order, uint32_t* vocab_order,
                              uint64_t* vocab_cf, uint64_t* vocab_df, uint32_t* real_v);

/* tmt_prepare_corpus on GPU `device`, for large corpora: the same outputs, bit
 * for bit (the per-document sorts run on the device, the vocabulary order on
 * the host).  Every document holds at most 16384 tokens; a longer one returns
 * TMT_ERR_INVALID_ARGUMENT with a message in err (use tmt_prepare_corpus).
 * Allocates and frees its own device memory. */
tmt_status tmt_prepare_corpus_device(int32_t device, uint64_t D, const uint64_t* doc_off, const uint32_t* words,
                                     uint32_t n_vocab, uint64_t min_cf, uint64_t min_df, uint64_t rm_top,
                                     uint32_t* words_out, uint32_t* w_order, uint32_t* vocab_order,
                                     uint64_t* vocab_cf, uint64_t* vocab_df, uint32_t* real_v, char* err,
                                     uint64_t err_len);

/* tmt_prepare_corpus in two halves, for a corpus split across processes:
 * the (cf, df) of one shard's words (by old id), and the preparation of one
 * shard from the counts summed over all shards, so that every shard gets the
 * same vocabulary order. */
tmt_status tmt_corpus_counts(uint64_t D, const uint64_t* doc_off, const uint32_t* words, uint32_t n_vocab,
                             uint64_t* vocab_cf, uint64_t* vocab_df);
tmt_status tmt_prepare_corpus_counted(uint64_t D, const uint64_t* doc_off, const uint32_t* words,
                                      uint32_t n_vocab, const uint64_t* cf, const uint64_t* df,
                                      uint64_t min_cf, uint64_t min_df, uint64_t rm_top,
                                      uint32_t* words_out, uint32_t* w_order, uint32_t* vocab_order,
                                      uint32_t* real_v);

/* No counterpart in tomotopy.  The FP64 log-likelihood of tmt_ll computed
 * from caller-owned DEVICE arrays -- n_dk (D x K), doc_len (D valid-token
 * counts), alpha (K), n_kw (K x V column-major), n_k (K) -- into ll_out (2
 * doubles on the device: ll_docs, ll_rest), on `stream` (a cudaStream_t;
 * NULL = the legacy default stream), without allocating any memory.  For
 * callers that may not call cudaMalloc: a serving process whose device
 * memory is handed out up front by its own pool, a plug-in inside a host
 * framework that owns every device allocation, or a pipelined stream that
 * must not pick up the implicit device synchronisation cudaMalloc/cudaFree
 * can cause.  Its scratch is one static device array of 281 KB, held by
 * every GPU that loads this library until the process exits; it supports
 * K <= 32767 and rejects larger K with TMT_ERR_INVALID_ARGUMENT.  Every
 * array must be device or managed memory (anything else is rejected before
 * a launch).  The first call on a device -- and the first after its context
 * changes, e.g. after cudaDeviceReset, which also replaces the array --
 * looks up that array's device address (with the device current) and
 * caches it; make that first call before any stream capture.  All calls on
 * a device share the scratch: calls that overlap on the GPU race and give
 * wrong sums -- serialise them (one stream, or events).  Each call
 * overwrites every scratch slot it reads, so no clearing is needed.  The
 * grid is tmt_ll's, so the result equals tmt_ll's bit for bit on the same
 * counts.  A CUDA error already pending on the calling thread is reported
 * (TMT_ERR_CUDA) and left pending, and nothing is launched.  The launches
 * are asynchronous on `stream`.  A message for a non-OK status is written
 * to err (err_len bytes, may be NULL). */
tmt_status tmt_ll_counts_noalloc(const int32_t* n_dk, uint64_t D, uint32_t K, const int32_t* doc_len,
                                 const float* alpha, const int32_t* n_kw, uint32_t V, const int32_t* n_k,
                                 float eta, double* ll_out, void* stream, char* err, size_t err_len);

tmt_status tmt_get_info(const tmt_handle* h, tmt_info* out);
const char* tmt_last_error(const tmt_handle* h);
void tmt_destroy(tmt_handle* h);

/* ---- the host model: tomotopy's LDAModel over the engine ----------------
 * One object per model (tomotopy's LDAModelObject -> ILDAModel,
 * py_LDA.cpp:151-611, LDAModel.hpp): dictionary and documents on the host,
 * sampling state on the device.  Word lists cross the ABI as NUL-separated
 * UTF-8 strings.  Only TermWeight.ONE and symmetric eta. */
typedef struct tmt_model tmt_model;
typedef struct tmt_model_args {
    uint32_t K;
    const float* alpha;      /* n_alpha == 1 (symmetric) or n_alpha == K */
    uint32_t n_alpha;
    float eta;
    uint64_t seed;
    uint64_t min_cf, min_df, rm_top;
    int32_t device;
    uint32_t sweep_groups;   /* 0: engine default */
    int32_t tw;              /* TermWeight (tomotopy/__init__.py:10-33): 0 ONE, 1 IDF, 2 PMI */
} tmt_model_args;
typedef struct tmt_model_info {
    uint32_t K, V, n_vocab;  /* V = realV (used vocabulary); n_vocab = all words seen */
    uint64_t n_docs, N, global_step;
    int32_t prepared;
    float alpha, eta;
    uint32_t optim_interval, burn_in;
    uint64_t seed, min_cf, min_df, rm_top;
    int32_t tw;              /* TermWeight: 0 ONE, 1 IDF, 2 PMI */
    double weighted_n;       /* TopicModel::weightedN, ll_per_word's denominator */
} tmt_model_info;

/* LDAModel ctor checks (LDAModel.hpp:962-983). */
tmt_status tmt_model_create(const tmt_model_args* args, tmt_model** out);
/* add_doc (TopicModel.hpp:397-449): *doc_id = -1 for an empty document. */
tmt_status tmt_model_add_doc(tmt_model* m, const char* words, uint32_t n_words, int64_t* doc_id);
/* set_word_prior (LDAModel.hpp:1031-1045, py_LDA.cpp:241-269): n == K priors >= 0
 * for `word` (added to the dictionary); before train() only; a second call for
 * the same word is ignored, as etaByWord.emplace ignores it. */
tmt_status tmt_model_set_word_prior(tmt_model* m, const char* word, const float* prior, uint32_t n);
/* get_word_prior (LDAModel.hpp:1047-1062): *n = K and the priors (the word's
 * eta column once prepared with priors), or *n = 0 for none; out may be NULL. */
tmt_status tmt_model_get_word_prior(tmt_model* m, const char* word, float* out, uint32_t* n);
/* LDAModel::prepare (LDAModel.hpp:1073-1138); train() calls it when needed. */
tmt_status tmt_model_prepare(tmt_model* m);
/* TopicModel::train (TopicModel.hpp:684-755) for `iters` sweeps. */
tmt_status tmt_model_train(tmt_model* m, uint32_t iters);
/* optim_interval / burn_in properties (LDAModel.hpp:1000-1010); any time between train() calls. */
tmt_status tmt_model_set_optim(tmt_model* m, uint32_t optim_interval, uint32_t burn_in);
/* Sets the seed of the model's sweep draws (copy() keeps the original's). */
tmt_status tmt_model_set_seed(tmt_model* m, uint64_t seed);
tmt_status tmt_model_get_info(tmt_model* m, tmt_model_info* out);
/* getLLDocs + getLLRest in FP64 (LDAModel.hpp:616-674). */
tmt_status tmt_model_ll(tmt_model* m, double* ll_docs, double* ll_rest);
/* current alphas (K). */
tmt_status tmt_model_alpha(tmt_model* m, float* out);
/* _getWidsByTopic (LDAModel.hpp:828-841): V floats. */
tmt_status tmt_model_topic_word_dist(tmt_model* m, uint32_t topic, int normalize, float* out);
/* _getTopicsCount (LDAModel.hpp:815-826): K counts. */
tmt_status tmt_model_count_by_topics(tmt_model* m, uint64_t* out);
/* the vocabulary as NUL-separated words (used_only: the first V); *need = bytes. */
tmt_status tmt_model_vocab(tmt_model* m, uint32_t used_only, char* buf, uint64_t cap, uint64_t* need);
/* vocabCf / vocabDf over all words (may be NULL). */
tmt_status tmt_model_vocab_freq(tmt_model* m, uint64_t* cf, uint64_t* df);
/* a document's word ids and topics in its original word order (py_LDA.cpp:613-619). */
tmt_status tmt_model_doc(tmt_model* m, uint64_t doc, uint32_t* words, uint16_t* topics, uint32_t* len);
/* _getTopicsByDoc (LDAModel.hpp:1145-1159) and the document's FP64 getLLDocs. */
tmt_status tmt_model_doc_topic_dist(tmt_model* m, uint64_t doc, int normalize, float* out, double* ll);
/* infer (together=False) of D string documents: words joined NUL-separated,
 * doc_nwords[d] words each; unknown words are dropped (makeDoc). */
tmt_status tmt_model_infer(tmt_model* m, const char* words, const uint64_t* doc_nwords, uint64_t D, uint32_t iters,
                           uint64_t seed, float* theta, double* ll);
/* infer with together=True (LDAModel.hpp:852-893): the D documents are
 * sampled jointly against the model's counts plus their own; one ll. */
tmt_status tmt_model_infer_together(tmt_model* m, const char* words, const uint64_t* doc_nwords, uint64_t D,
                                    uint32_t iters, uint64_t seed, float* theta, double* ll);
/* tomotopy's model layout (TopicModel.hpp:335-359): *out is malloc'ed; free
 * it with tmt_model_free_buffer. */
tmt_status tmt_model_save(tmt_model* m, const uint8_t* extra, uint64_t extra_len, int full, uint8_t** out,
                          uint64_t* out_len);
void tmt_model_free_buffer(uint8_t* buf);
/* _loadModel (TopicModel.hpp:361-395) + prepare(false): *extra is malloc'ed.
 * device < 0 parses only: queries and save work from the host copy, no GPU
 * is touched, and training / inference are unavailable. */
tmt_status tmt_model_load(const uint8_t* data, uint64_t len, int32_t device, uint32_t sweep_groups, tmt_model** out,
                          uint8_t** extra, uint64_t* extra_len);
const char* tmt_model_last_error(const tmt_model* m);
void tmt_model_destroy(tmt_model* m);

/* ---- synthetic corpus (workload generator; not a tomotopy interface) ---- */
typedef enum tmt_len_kind { TMT_LEN_POISSON = 0, TMT_LEN_LOGNORMAL = 1 } tmt_len_kind;
typedef struct tmt_synth_spec {
    uint32_t V, T;           /* vocabulary, true topics */
    uint64_t D;              /* documents */
    int32_t len_kind;        /* tmt_len_kind */
    double len_a, len_b;     /* Poisson mean | lognormal mu, sigma */
    uint32_t len_min, len_max;
    double doc_alpha;        /* theta_d ~ Dirichlet(doc_alpha) */
    double topic_beta;       /* phi_t ~ Dirichlet(topic_beta * V * Zipf(zipf_s)) */
    double zipf_s;
    uint64_t seed;
    uint32_t threads;        /* 0 = all hardware threads */
    uint64_t doc_offset;     /* documents are drawn as numbers doc_offset .. doc_offset+D-1: with the
                                same seed, a different offset gives new documents of the same topics */
} tmt_synth_spec;

/* Two calls: with words == NULL fills doc_off[D+1] and *n_tokens; then with
 * words of capacity >= *n_tokens fills the word ids (doc-major). */
tmt_status tmt_synth_corpus(const tmt_synth_spec* spec, uint64_t* doc_off,
                            uint32_t* words, uint64_t capacity, uint64_t* n_tokens);

#ifdef __cplusplus
}
#endif
#endif
