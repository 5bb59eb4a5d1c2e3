"""ctypes binding of the CPU oracle (oracle/liboracle.so) and of the
reference-primitive shim (oracle/_ref/libtmtref.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and
the CPU-baseline arm of bench.py, as the checker.  The product package never
imports it.  See tmt_oracle.h for what each function restates (tomotopy
file:line) and for the parity status.
"""
import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
# TMT_ORACLE_LIB selects another build of the same source (e.g. the -O3
# -march=native build of `make -C oracle native`; results are bit-identical:
# no fast-math, no FMA contraction)
_LIB = os.environ.get("TMT_ORACLE_LIB") or os.path.join(HERE, "liboracle.so")
_REF = os.path.join(HERE, "_ref", "libtmtref.so")

_u8p = C.POINTER(C.c_uint8)


def build(ref_tree=None):
    """Compile liboracle.so (and _ref when the tomotopy tree is present)."""
    cmd = ["make", "-s", "-C", HERE]
    if ref_tree:
        cmd.append("REF=" + ref_tree)
    subprocess.run(cmd, check=True)


def _ptr(a):
    return a.ctypes.data_as(C.c_void_p) if a is not None else None


def _load():
    if not os.path.exists(_LIB):
        build()
    lib = C.CDLL(_LIB)
    V = C.c_void_p
    sig = {
        "orc_philox4x32_10": (None, [V, V, V]),
        "orc_u01": (C.c_float, [C.c_uint32]),
        "orc_lgammaT": (C.c_float, [C.c_float]),
        "orc_digammaT": (C.c_float, [C.c_float]),
        "orc_digammaf": (C.c_float, [C.c_float]),
        "orc_digammaApprox": (C.c_float, [C.c_float]),
        "orc_prefix_sum_sse": (None, [V, C.c_int]),
        "orc_sample_acc": (C.c_size_t, [V, C.c_size_t, C.c_float]),
        "orc_shuffled_order": (None, [C.c_size_t, C.c_size_t, V]),
        "orc_remove_stopwords": (C.c_uint64, [C.c_uint64, V, V, C.c_uint64, C.c_uint64, C.c_uint64, V]),
        "orc_sort_doc": (None, [V, C.c_size_t, V]),
        "orc_init_z": (None, [C.c_uint64, V, C.c_uint32, C.c_uint32, V, C.c_uint64, V]),
        "orc_counts_from_z": (None, [C.c_uint64, V, V, V, C.c_uint32, C.c_uint32, V, V, V]),
        "orc_word_major": (C.c_uint64, [C.c_uint64, V, V, C.c_uint32, V, V, V]),
        "orc_sweep_snapshot": (None, [C.c_uint32, C.c_uint32, V, C.c_float, C.c_uint64, C.c_uint32,
                                      V, V, V, V, V, V, V]),
        "orc_conditional_f64": (None, [C.c_uint32, C.c_uint32, V, C.c_float, V, V, V, C.c_uint16, V]),
        "orc_sweep_doc_live": (None, [C.c_uint32, C.c_uint32, V, C.c_float, C.c_uint64, C.c_uint32,
                                      C.c_uint64, V, V, V, V, V, V, V, V]),
        "orc_sweep_doc_live_subset": (None, [C.c_uint32, C.c_uint32, V, C.c_float, C.c_uint64, C.c_uint32,
                                             C.c_uint64] + [V] * 9 + [C.c_uint64]),
        "orc_apply_sweep": (None, [C.c_uint32, C.c_uint32, V, V, V, V, V, V, V]),
        "orc_gibbs_none": (None, [C.c_uint64, V, V, C.c_uint32, C.c_uint32, V, C.c_float, V, V, V, V, V]),
        "orc_partition_create": (V, [C.c_uint64, V, V, C.c_uint32, C.c_uint32, V, C.c_float,
                                     V, V, V, V, V, C.c_uint32, C.c_uint64]),
        "orc_partition_train": (None, [V, C.c_uint32]),
        "orc_partition_destroy": (None, [V]),
        "orc_ll_docs_lut": (C.c_double, [C.c_uint64, C.c_uint32, V, V, V]),
        "orc_ll_rest_lut": (C.c_double, [C.c_uint32, C.c_uint32, V, V, C.c_float]),
        "orc_ll_docs_f64": (C.c_double, [C.c_uint64, C.c_uint32, V, V, V]),
        "orc_ll_rest_f64": (C.c_double, [C.c_uint32, C.c_uint32, V, V, C.c_float]),
        "orc_optimize_alpha": (None, [C.c_uint64, C.c_uint32, V, V, V]),
        "orc_infer_doc": (C.c_double, [C.c_uint32, C.c_uint32, V, C.c_float, V, V, V, C.c_uint32,
                                       C.c_uint32, C.c_uint64, C.c_uint64, V, V, V]),
        "orc_wq": (C.c_int64, [C.c_float]),
        "orc_fold": (C.c_float, [C.c_float, C.c_int64]),
        "orc_fold_w": (None, [C.c_uint32, C.c_uint32, V, V, V, V]),
        "orc_counts_from_z_w": (None, [C.c_uint64, V, V, V, V, C.c_uint32, C.c_uint32, V, V, V, V]),
        "orc_sweep_doc_live_w_subset": (None, [C.c_uint32, C.c_uint32, V, C.c_float, C.c_uint64, C.c_uint32]
                                        + [V] * 10 + [C.c_uint64]),
        "orc_ll_docs_w_f64": (C.c_double, [C.c_uint64, C.c_uint32, V, V, V]),
        "orc_ll_rest_w_f64": (C.c_double, [C.c_uint32, C.c_uint32, V, V, C.c_float]),
        "orc_optimize_alpha_w": (None, [C.c_uint64, C.c_uint32, V, V, V]),
        "orc_prior_esum": (None, [C.c_uint32, C.c_uint32, V, V, C.c_float, V]),
        "orc_init_z_p": (None, [C.c_uint64, V, C.c_uint32, C.c_uint32, V, V, C.c_float, C.c_uint64, V]),
        "orc_sweep_doc_live_p_subset": (None, [C.c_uint32, C.c_uint32, V, C.c_float, V, V, V, C.c_uint64,
                                               C.c_uint32] + [V] * 9 + [C.c_uint64]),
        "orc_ll_rest_p_f64": (C.c_double, [C.c_uint32, C.c_uint32, V, V, C.c_float, V, V, V]),
        "orc_infer_doc_p": (C.c_double, [C.c_uint32, C.c_uint32, V, C.c_float, V, V, V, V, V, V, C.c_uint32,
                                         C.c_uint32, C.c_uint64, C.c_uint64, V, V, V]),
        "orc_sweep_doc_live_m_subset": (None, [C.c_uint32, C.c_uint32, V, V, V, V, C.c_float, C.c_uint64,
                                               C.c_uint32] + [V] * 9 + [C.c_uint64]),
        "orc_ll_docs_m_f64": (C.c_double, [C.c_uint64, C.c_uint32, V, V, V, V]),
        "orc_gibbs_none_w": (None, [C.c_uint64, V, V, V, C.c_uint32, C.c_uint32, V, C.c_float, V, V, V, V, V]),
        "orc_gibbs_none_p": (None, [C.c_uint64, V, V, C.c_uint32, C.c_uint32, V, C.c_float, V, V, V, V, V, V, V,
                                    V]),
        "orc_infer_doc_w": (C.c_double, [C.c_uint32, C.c_uint32, V, C.c_float, V, V, V, V, C.c_uint32,
                                         C.c_uint32, C.c_uint64, C.c_uint64, V, V, V]),
    }
    for name, (res, args) in sig.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    return lib


lib = _load()


def load_ref():
    """The reference-primitive shim, or None when it was not built here."""
    if not os.path.exists(_REF):
        return None
    r = C.CDLL(_REF)
    V = C.c_void_p
    for name, res, args in [
        ("ref_lgammaT", C.c_float, [C.c_float]),
        ("ref_digammaT", C.c_float, [C.c_float]),
        ("ref_digammaf", C.c_float, [C.c_float]),
        ("ref_digammaApprox", C.c_double, [C.c_float]),
        ("ref_prefix_sum", None, [V, C.c_int]),
        ("ref_sample_acc", C.c_size_t, [V, C.c_size_t, C.c_float]),
        ("ref_shuffled_order", None, [C.c_size_t, C.c_size_t, V]),
        ("ref_sort_and_write_order", None, [V, C.c_size_t, V]),
        ("ref_remove_stopwords", C.c_uint64, [C.c_uint64, V, V, C.c_uint64, C.c_uint64, C.c_uint64, V]),
    ]:
        f = getattr(r, name)
        f.restype = res
        f.argtypes = args
    return r


# ---------------------------------------------------------------------------
# numpy-level helpers
# ---------------------------------------------------------------------------
def f32(a):
    return np.ascontiguousarray(a, dtype=np.float32)


def philox(ctr, key):
    c = np.asarray(ctr, dtype=np.uint32)
    k = np.asarray(key, dtype=np.uint32)
    out = np.zeros(4, dtype=np.uint32)
    lib.orc_philox4x32_10(_ptr(c), _ptr(k), _ptr(out))
    return out


class Corpus:
    """A prepared doc-major corpus: words already vocab-reordered and sorted
    by id inside each document (LDAModel.hpp:716-722)."""

    def __init__(self, doc_off, words, V):
        self.doc_off = np.ascontiguousarray(doc_off, dtype=np.uint64)
        self.words = np.ascontiguousarray(words, dtype=np.uint32)
        self.V = int(V)
        self.D = len(self.doc_off) - 1
        self.doc_len = np.zeros(self.D, dtype=np.int32)
        valid = self.words < self.V
        lens = np.diff(self.doc_off.astype(np.int64))
        if self.D:
            self.doc_len[:] = np.add.reduceat(valid.astype(np.int32), self.doc_off[:-1].astype(np.int64)) \
                if len(self.words) else 0
            self.doc_len[lens == 0] = 0
        self.N = int(valid.sum())

    def sort_docs(self):
        for d in range(self.D):
            b, e = int(self.doc_off[d]), int(self.doc_off[d + 1])
            self.words[b:e] = np.sort(self.words[b:e], kind="stable")
        return self

    def word_major(self):
        w_off = np.zeros(self.V + 1, dtype=np.uint64)
        tok_doc = np.zeros(max(self.N, 1), dtype=np.uint32)
        tok_pos = np.zeros(max(self.N, 1), dtype=np.uint64)
        lib.orc_word_major(self.D, _ptr(self.doc_off), _ptr(self.words), self.V,
                           _ptr(w_off), _ptr(tok_doc), _ptr(tok_pos))
        return w_off, tok_doc[:self.N], tok_pos[:self.N]


class State:
    """Counts + assignments for the oracle samplers."""

    def __init__(self, corpus, K, alpha, eta, seed, z0=None):
        self.c = corpus
        self.K = int(K)
        self.alpha = f32(np.broadcast_to(np.asarray(alpha, dtype=np.float32), (self.K,)).copy())
        self.eta = float(np.float32(eta))
        self.seed = int(seed)
        n_all = len(corpus.words)
        if z0 is None:
            self.z = np.zeros(max(n_all, 1), dtype=np.uint16)
            lib.orc_init_z(n_all, _ptr(corpus.words), corpus.V, self.K, _ptr(self.alpha), self.seed,
                           _ptr(self.z))
            self.z = self.z[:n_all]
        else:
            self.z = np.ascontiguousarray(z0, dtype=np.uint16).copy()
        self.recount()

    def recount(self):
        c = self.c
        self.ndk = np.zeros((c.D, self.K), dtype=np.int32)
        self.nkw = np.zeros((c.V, self.K), dtype=np.int32)   # column v = K ints
        self.nk = np.zeros(self.K, dtype=np.int32)
        lib.orc_counts_from_z(c.D, _ptr(c.doc_off), _ptr(c.words), _ptr(self.z), c.V, self.K,
                              _ptr(self.ndk), _ptr(self.nkw), _ptr(self.nk))

    # --- samplers -----------------------------------------------------------
    def gibbs_none(self, iters, rng_state):
        st = np.array([rng_state], dtype=np.uint64)
        c = self.c
        for _ in range(iters):
            lib.orc_gibbs_none(c.D, _ptr(c.doc_off), _ptr(c.words), c.V, self.K, _ptr(self.alpha),
                               self.eta, _ptr(self.z), _ptr(self.ndk), _ptr(self.nkw), _ptr(self.nk),
                               _ptr(st))
        return int(st[0])

    def snapshot_sweeps(self, iters, start_step=0):
        """The device sampler's semantics, `iters` sweeps from global step start_step."""
        c = self.c
        w_off, tok_doc, tok_pos = c.word_major()
        zw = np.ascontiguousarray(self.z[tok_pos.astype(np.int64)], dtype=np.uint16) if c.N else \
            np.zeros(1, np.uint16)
        zn = np.zeros_like(zw)
        for it in range(iters):
            lib.orc_sweep_snapshot(self.K, c.V, _ptr(self.alpha), self.eta, self.seed, start_step + it,
                                   _ptr(w_off), _ptr(tok_doc), _ptr(self.ndk), _ptr(self.nkw),
                                   _ptr(self.nk), _ptr(zw), _ptr(zn))
            lib.orc_apply_sweep(self.K, c.V, _ptr(w_off), _ptr(tok_doc), _ptr(self.ndk), _ptr(self.nkw),
                                _ptr(self.nk), _ptr(zw), _ptr(zn))
        if c.N:
            self.z[tok_pos.astype(np.int64)] = zw[:c.N]

    def group_bounds(self, groups):
        """Document groups of a sweep: the documents ordered longest first
        (stable), cut into `groups` contiguous ranges holding equal shares of
        the tokens -- position p is in group g when prefix(p) * G lies in
        [g * total, (g + 1) * total)."""
        c = self.c
        lens = np.diff(c.doc_off.astype(np.int64))
        order = np.argsort(-lens, kind="stable").astype(np.uint64)
        total = int(lens.sum())
        prefix = np.concatenate([[0], np.cumsum(lens[order.astype(np.int64)])[:-1]]) if c.D else np.zeros(0)
        bounds = [0]
        for g in range(1, groups):
            bounds.append(int(np.sum(prefix * groups < g * total)))
        bounds.append(c.D)
        return order, bounds

    def doc_live_sweeps(self, iters, start_step=0, groups=1):
        """The device sweep: doc-major, live n_dk, snapshot n_kw / n_k,
        sampled group by group (see group_bounds), the snapshot refreshed
        between groups."""
        c = self.c
        order, b = self.group_bounds(groups)
        parts = [np.ascontiguousarray(order[b[g]:b[g + 1]]) for g in range(groups)]
        for it in range(iters):
            for part in parts:
                if len(part) == 0:
                    continue
                nkw2 = self.nkw.copy()
                nk2 = self.nk.copy()
                lib.orc_sweep_doc_live_subset(self.K, c.V, _ptr(self.alpha), self.eta, self.seed, start_step + it,
                                              c.D, _ptr(c.doc_off), _ptr(c.words), _ptr(self.ndk), _ptr(self.nkw),
                                              _ptr(self.nk), _ptr(nkw2), _ptr(nk2), _ptr(self.z), _ptr(part),
                                              len(part))
                self.nkw = nkw2
                self.nk = nk2

    def optimize_alpha(self):
        lib.orc_optimize_alpha(self.c.D, self.K, _ptr(self.ndk), _ptr(self.c.doc_len), _ptr(self.alpha))

    # --- log-likelihood -------------------------------------------------------
    def ll_f64(self):
        c = self.c
        a = lib.orc_ll_docs_f64(c.D, self.K, _ptr(self.ndk), _ptr(c.doc_len), _ptr(self.alpha))
        b = lib.orc_ll_rest_f64(self.K, c.V, _ptr(self.nkw), _ptr(self.nk), self.eta)
        return a, b

    def ll_lut(self):
        c = self.c
        a = lib.orc_ll_docs_lut(c.D, self.K, _ptr(self.ndk), _ptr(c.doc_len), _ptr(self.alpha))
        b = lib.orc_ll_rest_lut(self.K, c.V, _ptr(self.nkw), _ptr(self.nk), self.eta)
        return a, b

    def ll_per_word(self, lut=False):
        a, b = self.ll_lut() if lut else self.ll_f64()
        return (a + b) / max(self.c.N, 1)


def weights_idf(corpus):
    """TermWeight.IDF token weights: vocabWeights[v] = (float)log(D / (double)df[v])
    (LDAModel.hpp:1093-1113, df over documents' distinct in-vocabulary words),
    token weight = vocabWeights[word] (:801-803); 0 for out-of-vocabulary tokens."""
    c = corpus
    df = np.zeros(c.V, dtype=np.int64)
    for d in range(c.D):
        ws = c.words[c.doc_off[d]:c.doc_off[d + 1]]
        df[np.unique(ws[ws < c.V])] += 1
    with np.errstate(divide="ignore"):
        vw = np.log(c.D / df.astype(np.float64)).astype(np.float32)
    wt = np.zeros(len(c.words), dtype=np.float32)
    m = c.words < c.V
    wt[m] = vw[c.words[m]]
    return wt, vw


def weights_pmi(corpus):
    """TermWeight.PMI token weights: vocabWeights[v] = (float)(cf[v] / (double)totCf)
    (LDAModel.hpp:1114-1121; cf over every token of the corpus), token weight
    max((float)log(tf / vocabWeights[v] / len), 0) with tf the word's count in
    the document and len the document's token count, in float (:804-807)."""
    c = corpus
    nv = int(c.words.max()) + 1 if len(c.words) else 0
    cf = np.bincount(c.words.astype(np.int64), minlength=max(nv, c.V)).astype(np.float64)
    tot = float(len(c.words))
    vw = (cf[:c.V] / tot).astype(np.float32)
    wt = np.zeros(len(c.words), dtype=np.float32)
    for d in range(c.D):
        b, e = int(c.doc_off[d]), int(c.doc_off[d + 1])
        ws = c.words[b:e]
        m = ws < c.V
        tf = np.bincount(ws[m].astype(np.int64), minlength=c.V)
        q = (tf[ws[m]].astype(np.float32) / vw[ws[m]]) / np.float32(e - b)
        wt[b:e][m] = np.maximum(np.log(q.astype(np.float64)).astype(np.float32), np.float32(0))
    return wt, vw


class StateW:
    """Weighted counts (TermWeight IDF / PMI) for the device sweep's semantics:
    float n_dk rows updated in token order, float n_kw / n_k folded between
    document groups from integer deltas in units of 2^-24."""

    def __init__(self, corpus, K, alpha, eta, seed, weights, z0=None):
        self.c = corpus
        self.K = int(K)
        self.alpha = f32(np.broadcast_to(np.asarray(alpha, dtype=np.float32), (self.K,)).copy())
        self.eta = float(np.float32(eta))
        self.seed = int(seed)
        self.wt = np.ascontiguousarray(weights, dtype=np.float32)
        n_all = len(corpus.words)
        if z0 is None:
            self.z = np.zeros(max(n_all, 1), dtype=np.uint16)
            lib.orc_init_z(n_all, _ptr(corpus.words), corpus.V, self.K, _ptr(self.alpha), self.seed,
                           _ptr(self.z))
            self.z = self.z[:n_all]
        else:
            self.z = np.ascontiguousarray(z0, dtype=np.uint16).copy()
        self.recount()

    def recount(self):
        c = self.c
        self.ndk = np.zeros((c.D, self.K), dtype=np.float32)
        self.doc_wlen = np.zeros(max(c.D, 1), dtype=np.float32)
        self.nkw = np.zeros((c.V, self.K), dtype=np.float32)
        self.nk = np.zeros(self.K, dtype=np.float32)
        lib.orc_counts_from_z_w(c.D, _ptr(c.doc_off), _ptr(c.words), _ptr(self.z), _ptr(self.wt), c.V, self.K,
                                _ptr(self.ndk), _ptr(self.doc_wlen), _ptr(self.nkw), _ptr(self.nk))

    group_bounds = State.group_bounds

    def doc_live_sweeps(self, iters, start_step=0, groups=1):
        c = self.c
        order, b = self.group_bounds(groups)
        parts = [np.ascontiguousarray(order[b[g]:b[g + 1]]) for g in range(groups)]
        dkw = np.zeros((c.V, self.K), dtype=np.int64)
        dk = np.zeros(self.K, dtype=np.int64)
        for it in range(iters):
            for part in parts:
                if len(part) == 0:
                    continue
                lib.orc_fold_w(self.K, c.V, _ptr(self.nkw), _ptr(self.nk), _ptr(dkw), _ptr(dk))
                lib.orc_sweep_doc_live_w_subset(self.K, c.V, _ptr(self.alpha), self.eta, self.seed,
                                                start_step + it, _ptr(c.doc_off), _ptr(c.words), _ptr(self.wt),
                                                _ptr(self.ndk), _ptr(self.nkw), _ptr(self.nk), _ptr(dkw), _ptr(dk),
                                                _ptr(self.z), _ptr(part), len(part))
            lib.orc_fold_w(self.K, c.V, _ptr(self.nkw), _ptr(self.nk), _ptr(dkw), _ptr(dk))

    def gibbs_none(self, iters, rng_state):
        """tomotopy's sequential sampler with these weights (live float counts)."""
        st = np.array([rng_state], dtype=np.uint64)
        c = self.c
        for _ in range(iters):
            lib.orc_gibbs_none_w(c.D, _ptr(c.doc_off), _ptr(c.words), _ptr(self.wt), c.V, self.K, _ptr(self.alpha),
                                 self.eta, _ptr(self.z), _ptr(self.ndk), _ptr(self.nkw), _ptr(self.nk), _ptr(st))
        return int(st[0])

    def optimize_alpha(self):
        lib.orc_optimize_alpha_w(self.c.D, self.K, _ptr(self.ndk), _ptr(self.doc_wlen), _ptr(self.alpha))

    def ll_f64(self):
        c = self.c
        a = lib.orc_ll_docs_w_f64(c.D, self.K, _ptr(self.ndk), _ptr(self.doc_wlen), _ptr(self.alpha))
        b = lib.orc_ll_rest_w_f64(self.K, c.V, _ptr(self.nkw), _ptr(self.nk), self.eta)
        return a, b

    def ll_per_word(self):
        """ll / realN: tomotopy counts weightedN in prepare() before the
        weights exist (TopicModel.hpp:507-523, 652-655), so a freshly trained
        weighted model divides by the token count."""
        a, b = self.ll_f64()
        return (a + b) / self.c.N


class StateP(State):
    """Integer counts with word priors (etaByTopicWord): prior_ids[p] gets
    priors[p] (K floats) as its eta column."""

    def __init__(self, corpus, K, alpha, eta, seed, prior_ids, priors, z0=None):
        self.c = corpus
        self.K = int(K)
        self.alpha = f32(np.broadcast_to(np.asarray(alpha, dtype=np.float32), (self.K,)).copy())
        self.eta = float(np.float32(eta))
        self.seed = int(seed)
        self.pidx = np.full(corpus.V, -1, dtype=np.int32)
        self.pidx[np.asarray(prior_ids, dtype=np.int64)] = np.arange(len(prior_ids), dtype=np.int32)
        self.prior = np.ascontiguousarray(priors, dtype=np.float32).reshape(len(prior_ids), self.K) \
            if len(prior_ids) else np.zeros((1, self.K), np.float32)
        self.esum = np.zeros(self.K, dtype=np.float32)
        lib.orc_prior_esum(self.K, corpus.V, _ptr(self.pidx), _ptr(self.prior), self.eta, _ptr(self.esum))
        n_all = len(corpus.words)
        if z0 is None:
            self.z = np.zeros(max(n_all, 1), dtype=np.uint16)
            lib.orc_init_z_p(n_all, _ptr(corpus.words), corpus.V, self.K, _ptr(self.pidx), _ptr(self.prior),
                             self.eta, self.seed, _ptr(self.z))
            self.z = self.z[:n_all]
        else:
            self.z = np.ascontiguousarray(z0, dtype=np.uint16).copy()
        self.recount()

    def doc_live_sweeps(self, iters, start_step=0, groups=1):
        c = self.c
        order, b = self.group_bounds(groups)
        parts = [np.ascontiguousarray(order[b[g]:b[g + 1]]) for g in range(groups)]
        for it in range(iters):
            for part in parts:
                if len(part) == 0:
                    continue
                nkw2 = self.nkw.copy()
                nk2 = self.nk.copy()
                lib.orc_sweep_doc_live_p_subset(self.K, c.V, _ptr(self.alpha), self.eta, _ptr(self.pidx),
                                                _ptr(self.prior), _ptr(self.esum), self.seed, start_step + it,
                                                _ptr(c.doc_off), _ptr(c.words), _ptr(self.ndk), _ptr(self.nkw),
                                                _ptr(self.nk), _ptr(nkw2), _ptr(nk2), _ptr(self.z), _ptr(part),
                                                len(part))
                self.nkw = nkw2
                self.nk = nk2

    def ll_f64(self):
        c = self.c
        a = lib.orc_ll_docs_f64(c.D, self.K, _ptr(self.ndk), _ptr(c.doc_len), _ptr(self.alpha))
        b = lib.orc_ll_rest_p_f64(self.K, c.V, _ptr(self.nkw), _ptr(self.nk), self.eta, _ptr(self.pidx),
                                  _ptr(self.prior), _ptr(self.esum))
        return a, b

    def gibbs_none(self, iters, rng_state):
        """tomotopy's sequential sampler with these word priors."""
        st = np.array([rng_state], dtype=np.uint64)
        c = self.c
        for _ in range(iters):
            lib.orc_gibbs_none_p(c.D, _ptr(c.doc_off), _ptr(c.words), c.V, self.K, _ptr(self.alpha), self.eta,
                                 _ptr(self.pidx), _ptr(self.prior), _ptr(self.esum), _ptr(self.z), _ptr(self.ndk),
                                 _ptr(self.nkw), _ptr(self.nk), _ptr(st))
        return int(st[0])

    def infer_doc(self, nkw, nk, alpha, words, iters, seed, doc_key):
        words = np.ascontiguousarray(words, dtype=np.uint32)
        z = np.zeros(max(len(words), 1), dtype=np.uint16)
        ndk = np.zeros(self.K, dtype=np.int32)
        theta = np.zeros(self.K, dtype=np.float32)
        a = f32(np.asarray(alpha, dtype=np.float32).copy())
        ll = lib.orc_infer_doc_p(self.K, self.c.V, _ptr(a), self.eta, _ptr(self.pidx), _ptr(self.prior),
                                 _ptr(self.esum), _ptr(np.ascontiguousarray(nkw, np.int32)),
                                 _ptr(np.ascontiguousarray(nk, np.int32)), _ptr(words), len(words), iters, seed,
                                 doc_key, _ptr(z), _ptr(ndk), _ptr(theta))
        return ll, z[:len(words)], ndk, theta


class StateM(State):
    """Per-document topic masks (LLDA / PLDA) and alphas (DMR) on top of the
    doc-major sweep: A_k = ((float)n_dk + alpha_dk) * m_dk.  mask: D x K bool
    or None; alpha_rows (M x K) with doc_row (D) or None.  z0 is the caller's."""

    def __init__(self, corpus, K, alpha, eta, seed, z0, mask=None, alpha_rows=None, doc_row=None):
        super().__init__(corpus, K, alpha, eta, seed, z0=z0)
        self.mask_bits = None
        if mask is not None:
            mw = (self.K + 31) // 32
            bits = np.zeros((corpus.D, mw * 32), dtype=bool)
            bits[:, :self.K] = np.asarray(mask, dtype=bool)
            w = np.packbits(bits.reshape(corpus.D, mw, 32)[:, :, ::-1], axis=2, bitorder="big")
            self.mask_bits = np.ascontiguousarray(w.view(">u4").reshape(corpus.D, mw).astype(np.uint32))
        self.alpha_rows = None if alpha_rows is None else np.ascontiguousarray(alpha_rows, np.float32)
        self.doc_row = None if doc_row is None else np.ascontiguousarray(doc_row, np.uint32)

    def doc_live_sweeps(self, iters, start_step=0, groups=1):
        c = self.c
        order, b = self.group_bounds(groups)
        parts = [np.ascontiguousarray(order[b[g]:b[g + 1]]) for g in range(groups)]
        for it in range(iters):
            for part in parts:
                if len(part) == 0:
                    continue
                nkw2 = self.nkw.copy()
                nk2 = self.nk.copy()
                lib.orc_sweep_doc_live_m_subset(self.K, c.V, _ptr(self.alpha), _ptr(self.alpha_rows),
                                                _ptr(self.doc_row), _ptr(self.mask_bits), self.eta, self.seed,
                                                start_step + it, _ptr(c.doc_off), _ptr(c.words), _ptr(self.ndk),
                                                _ptr(self.nkw), _ptr(self.nk), _ptr(nkw2), _ptr(nk2), _ptr(self.z),
                                                _ptr(part), len(part))
                self.nkw = nkw2
                self.nk = nk2

    def ll_f64(self):
        a, b = super().ll_f64()
        if self.alpha_rows is not None:
            c = self.c
            a = lib.orc_ll_docs_m_f64(c.D, self.K, _ptr(self.ndk), _ptr(c.doc_len), _ptr(self.alpha_rows),
                                      _ptr(self.doc_row))
        return a, b


class Partition:
    """tomotopy's PARTITION scheme on host threads (the CPU baseline)."""

    def __init__(self, state, nthreads, vocab_cf=None, seed=1):
        c = state.c
        if vocab_cf is None:
            vocab_cf = np.bincount(c.words[c.words < c.V], minlength=c.V).astype(np.uint64)
        self.cf = np.ascontiguousarray(vocab_cf, dtype=np.uint64)
        self.s = state
        self.h = lib.orc_partition_create(c.D, _ptr(c.doc_off), _ptr(c.words), c.V, state.K,
                                          _ptr(state.alpha), state.eta, _ptr(state.z), _ptr(state.ndk),
                                          _ptr(state.nkw), _ptr(state.nk), _ptr(self.cf), nthreads, seed)

    def train(self, iters):
        lib.orc_partition_train(self.h, iters)

    def close(self):
        if self.h:
            lib.orc_partition_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()


def infer_doc(K, V, alpha, eta, nkw, nk, words, iters, seed, doc_key):
    """Infer one document (ids sorted ascending) against a frozen model."""
    words = np.ascontiguousarray(words, dtype=np.uint32)
    z = np.zeros(max(len(words), 1), dtype=np.uint16)
    ndk = np.zeros(K, dtype=np.int32)
    theta = np.zeros(K, dtype=np.float32)
    a = f32(np.broadcast_to(np.asarray(alpha, dtype=np.float32), (K,)).copy())
    ll = lib.orc_infer_doc(K, V, _ptr(a), float(np.float32(eta)), _ptr(np.ascontiguousarray(nkw, np.int32)),
                           _ptr(np.ascontiguousarray(nk, np.int32)), _ptr(words), len(words), iters, seed,
                           doc_key, _ptr(z), _ptr(ndk), _ptr(theta))
    return ll, z[:len(words)], ndk, theta


def infer_doc_w(K, V, alpha, eta, nkw, nk, words, weights, iters, seed, doc_key):
    """Infer one document (ids sorted ascending, one weight per word within
    the document) against a frozen model with weighted counts."""
    words = np.ascontiguousarray(words, dtype=np.uint32)
    wt = np.ascontiguousarray(weights, dtype=np.float32)
    z = np.zeros(max(len(words), 1), dtype=np.uint16)
    ndk = np.zeros(K, dtype=np.float32)
    theta = np.zeros(K, dtype=np.float32)
    a = f32(np.broadcast_to(np.asarray(alpha, dtype=np.float32), (K,)).copy())
    ll = lib.orc_infer_doc_w(K, V, _ptr(a), float(np.float32(eta)), _ptr(np.ascontiguousarray(nkw, np.float32)),
                             _ptr(np.ascontiguousarray(nk, np.float32)), _ptr(words), _ptr(wt), len(words), iters,
                             seed, doc_key, _ptr(z), _ptr(ndk), _ptr(theta))
    return ll, z[:len(words)], ndk, theta
