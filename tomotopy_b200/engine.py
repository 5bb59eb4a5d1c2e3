"""Thin Python wrapper over the engine's C ABI (tmt_create / tmt_upload_corpus /
tmt_train / tmt_ll / tmt_download_state ...).  Host buffers are numpy arrays;
the handle owns the device buffers."""
import ctypes as C

import numpy as np

from ._lib import (lib, check, TmtConfig, TmtInfo, TmtSynthSpec, TmtServerConfig, TmtServerStats, TmtError,
                   SAMPLER_AUTO, LEN_POISSON, LEN_LOGNORMAL)


def _p(a):
    return a.ctypes.data_as(C.c_void_p) if a is not None else None


class Engine:
    """One model state on one GPU (tmt_handle)."""

    def __init__(self, K, V, alpha=0.1, eta=0.01, seed=0, optim_interval=10, burn_in=0, device=0,
                 sampler=SAMPLER_AUTO, hbm_budget=0, sweep_groups=0):
        self.K, self.V = int(K), int(V)
        self._eta = float(np.float32(eta))
        a = np.broadcast_to(np.asarray(alpha, dtype=np.float32), (self.K,)).copy() \
            if np.ndim(alpha) else None
        self._alpha_buf = a
        cfg = TmtConfig(K=self.K, V=self.V,
                        alpha=a.ctypes.data_as(C.POINTER(C.c_float)) if a is not None else None,
                        alpha_scalar=float(alpha) if a is None else 0.0, eta=float(eta), seed=int(seed),
                        optim_interval=int(optim_interval), burn_in=int(burn_in), device=int(device),
                        sampler=int(sampler), hbm_budget=int(hbm_budget), sweep_groups=int(sweep_groups))
        h = C.c_void_p()
        st = lib.tmt_create(C.byref(cfg), C.byref(h))
        self.h = h
        if st != 0:
            msg = lib.tmt_last_error(h).decode() if h.value else "tmt_create failed"
            self.close()
            check(st, None, msg)
        self.D = 0
        self.n_all = 0

    def close(self):
        if getattr(self, "h", None) is not None and self.h.value:
            lib.tmt_destroy(self.h)
        self.h = None

    def __del__(self):
        self.close()

    def upload(self, doc_off, words, z0=None, weights=None):
        """tmt_upload_corpus, or tmt_upload_corpus_weighted when per-token
        weights (TermWeight IDF / PMI) are given."""
        self._doc_off = np.ascontiguousarray(doc_off, dtype=np.uint64)
        self._words = np.ascontiguousarray(words, dtype=np.uint32)
        self._n_rows = None
        zz = np.ascontiguousarray(z0, dtype=np.uint16) if z0 is not None else None
        self.D = len(self._doc_off) - 1
        self.n_all = int(self._doc_off[-1]) if self.D >= 0 else 0
        if weights is None:
            self.weighted = False
            check(lib.tmt_upload_corpus(self.h, _p(self._words), _p(self._doc_off), self.D, _p(zz)), self.h)
        else:
            self._wt = np.ascontiguousarray(weights, dtype=np.float32)
            if len(self._wt) != self.n_all:
                raise ValueError("weights must hold one value per token")
            self.weighted = True
            check(lib.tmt_upload_corpus_weighted(self.h, _p(self._words), _p(self._doc_off), self.D, _p(zz),
                                                 _p(self._wt)), self.h)

    def train(self, iters, ll_every=0):
        n = iters // ll_every if ll_every else 0
        out = np.zeros(max(n, 1), dtype=np.float64)
        check(lib.tmt_train(self.h, int(iters), int(ll_every), _p(out) if n else None), self.h)
        return out[:n]

    def set_word_priors(self, word_ids, priors):
        """tmt_set_word_priors: word_ids[p] gets priors[p] (K floats) as its eta
        column; call before upload()."""
        ids = np.ascontiguousarray(word_ids, dtype=np.uint32)
        pr = np.ascontiguousarray(priors, dtype=np.float32).reshape(len(ids), self.K) if len(ids) else \
            np.zeros((0, self.K), np.float32)
        self._prior_ids, self._prior = ids, pr
        check(lib.tmt_set_word_priors(self.h, len(ids), _p(ids), _p(pr)), self.h)

    def set_doc_topic_mask(self, mask):
        """tmt_set_doc_topic_mask from a boolean D x K array (None clears):
        topic k is allowed in document d where mask[d, k]."""
        if mask is None:
            check(lib.tmt_set_doc_topic_mask(self.h, None), self.h)
            return
        self._mask = pack_topic_mask(mask, self.K)
        if self._mask.shape[0] != self.D:
            raise ValueError("the mask needs one row per document")
        check(lib.tmt_set_doc_topic_mask(self.h, _p(self._mask)), self.h)

    def set_doc_alpha(self, rows, doc_row):
        """tmt_set_doc_alpha: alpha rows (M x K) and each document's row (None clears)."""
        if rows is None:
            check(lib.tmt_set_doc_alpha(self.h, 0, None, None), self.h)
            return
        self._arows = np.ascontiguousarray(rows, dtype=np.float32).reshape(-1, self.K)
        self._arow = np.ascontiguousarray(doc_row, dtype=np.uint32)
        check(lib.tmt_set_doc_alpha(self.h, len(self._arows), _p(self._arows), _p(self._arow)), self.h)

    def sweep_variants(self):
        """The autotuner's sweep-kernel variant per document group (-1 while tuning)."""
        n = C.c_uint32()
        check(lib.tmt_get_sweep_variants(self.h, None, 0, C.byref(n)), self.h)
        out = np.zeros(max(n.value, 1), dtype=np.int32)
        check(lib.tmt_get_sweep_variants(self.h, _p(out), n.value, C.byref(n)), self.h)
        return out[:n.value].tolist()

    def sweep_timings(self):
        """The autotuner's milliseconds per document group and variant (G x n_variants)."""
        g, v = C.c_uint32(), C.c_uint32()
        check(lib.tmt_get_sweep_timings(self.h, None, 0, C.byref(g), C.byref(v)), self.h)
        out = np.zeros(max(g.value * v.value, 1), dtype=np.float32)
        check(lib.tmt_get_sweep_timings(self.h, _p(out), out.size, C.byref(g), C.byref(v)), self.h)
        return out[:g.value * v.value].reshape(g.value, v.value)

    def set_doc_rows(self, row_of_doc, R=None):
        """tmt_set_doc_rows: document d counts in row row_of_doc[d] of R shared
        rows (PT's pseudo-documents); None returns to one row per document."""
        if row_of_doc is None:
            check(lib.tmt_set_doc_rows(self.h, 0, None), self.h)
            self._n_rows = None
            return
        rows = np.ascontiguousarray(row_of_doc, dtype=np.uint32)
        if len(rows) != self.D:
            raise ValueError("row_of_doc needs one entry per document")
        R = int(rows.max()) + 1 if R is None else int(R)
        check(lib.tmt_set_doc_rows(self.h, R, _p(rows)), self.h)
        self._n_rows = R

    def set_doc_split(self, min_tokens=0, step=0):
        """tmt_set_doc_split: documents of at least min_tokens tokens are
        sampled as 8 slices merging every `step` positions (0: the engine's
        rule / step; 2**32 - 1: never split)."""
        check(lib.tmt_set_doc_split(self.h, int(min_tokens), int(step)), self.h)

    def doc_split(self):
        """Per document group, how many documents are split."""
        n = C.c_uint32()
        check(lib.tmt_get_doc_split(self.h, None, 0, C.byref(n)), self.h)
        out = np.zeros(max(n.value, 1), dtype=np.uint32)
        check(lib.tmt_get_doc_split(self.h, _p(out), n.value, C.byref(n)), self.h)
        return out[:n.value].tolist()

    def set_graphs(self, enable):
        """Sweeps as CUDA graph launches after the autotuner's first sweeps
        (default) or as separate kernel launches; results are identical."""
        check(lib.tmt_set_graphs(self.h, int(bool(enable))), self.h)

    def infer(self, doc_off, words, iters=100, seed=0, doc_keys=None, weights=None):
        """tmt_infer_batch (tmt_infer_batch_weighted with per-token weights):
        returns (theta [D x K] float32, ll [D] float64)."""
        doc_off = np.ascontiguousarray(doc_off, dtype=np.uint64)
        words = np.ascontiguousarray(words, dtype=np.uint32)
        D = len(doc_off) - 1
        theta = np.zeros((max(D, 1), self.K), dtype=np.float32)
        ll = np.zeros(max(D, 1), dtype=np.float64)
        keys = np.ascontiguousarray(doc_keys, dtype=np.uint64) if doc_keys is not None else None
        if weights is None:
            check(lib.tmt_infer_batch(self.h, _p(words), _p(doc_off), D, int(iters), int(seed), _p(keys),
                                      _p(theta), _p(ll)), self.h)
        else:
            wt = np.ascontiguousarray(weights, dtype=np.float32)
            check(lib.tmt_infer_batch_weighted(self.h, _p(words), _p(doc_off), D, _p(wt), int(iters), int(seed),
                                               _p(keys), _p(theta), _p(ll)), self.h)
        return theta[:D], ll[:D]

    @property
    def eta(self):
        return self._eta

    def ll(self):
        a, b = C.c_double(), C.c_double()
        check(lib.tmt_ll(self.h, C.byref(a), C.byref(b)), self.h)
        return a.value, b.value

    def ll_per_word(self):
        a, b = self.ll()
        n = self.info().N
        return (a + b) / n if n else 0.0

    def state(self):
        """(z, n_kw [V x K], n_k, alpha); float counts when weighted."""
        z = np.zeros(max(self.n_all, 1), dtype=np.uint16)
        alpha = np.zeros(self.K, dtype=np.float32)
        if getattr(self, "weighted", False):
            nkw = np.zeros((self.V, self.K), dtype=np.float32)
            nk = np.zeros(self.K, dtype=np.float32)
            check(lib.tmt_download_state(self.h, _p(z), None, None, _p(alpha)), self.h)
            check(lib.tmt_download_counts_f32(self.h, None, _p(nkw), _p(nk), None), self.h)
        else:
            nkw = np.zeros((self.V, self.K), dtype=np.int32)
            nk = np.zeros(self.K, dtype=np.int32)
            check(lib.tmt_download_state(self.h, _p(z), _p(nkw), _p(nk), _p(alpha)), self.h)
        return z[:self.n_all], nkw, nk, alpha

    def doc_topic(self):
        """n_dk [D x K] (the R shared rows after set_doc_rows); float when weighted."""
        if getattr(self, "weighted", False):
            ndk = np.zeros((max(self.D, 1), self.K), dtype=np.float32)
            check(lib.tmt_download_counts_f32(self.h, _p(ndk), None, None, None), self.h)
            return ndk[:self.D]
        n = getattr(self, "_n_rows", None) or self.D
        ndk = np.zeros((max(n, 1), self.K), dtype=np.int32)
        check(lib.tmt_download_doc_topic(self.h, _p(ndk)), self.h)
        return ndk[:n]

    def doc_weight_sums(self):
        """Per-document weight sums of a weighted corpus."""
        out = np.zeros(max(self.D, 1), dtype=np.float32)
        check(lib.tmt_download_counts_f32(self.h, None, None, None, _p(out)), self.h)
        return out[:self.D]

    def info(self):
        i = TmtInfo()
        check(lib.tmt_get_info(self.h, C.byref(i)), self.h)
        return i


def pack_topic_mask(mask, K):
    """A boolean D x K topic mask as the C ABI's bit rows: D rows of ceil(K/32)
    uint32 words, bit (k % 32) of word k // 32 set where topic k is allowed."""
    m = np.asarray(mask, dtype=bool).reshape(-1, K)
    D = m.shape[0]
    mw = (K + 31) // 32
    bits = np.zeros((D, mw * 32), dtype=bool)
    bits[:, :K] = m
    words = np.packbits(bits.reshape(D, mw, 32)[:, :, ::-1], axis=2, bitorder="big")
    return np.ascontiguousarray(words.view(">u4").reshape(D, mw).astype(np.uint32))


def synth_corpus(V, T, D, length, seed, doc_alpha=0.1, topic_beta=0.01, zipf_s=1.07, threads=0, doc_offset=0):
    """Seeded synthetic corpus (tmt_synth_corpus).  length = ("poisson", mean, lo, hi)
    or ("lognormal", mu, sigma, lo, hi).  Returns (doc_off uint64[D+1], words uint32[N])."""
    if length[0] == "poisson":
        kind, a, b, lo, hi = LEN_POISSON, float(length[1]), 0.0, int(length[2]), int(length[3])
    else:
        kind, a, b, lo, hi = LEN_LOGNORMAL, float(length[1]), float(length[2]), int(length[3]), int(length[4])
    spec = TmtSynthSpec(V=V, T=T, D=D, len_kind=kind, len_a=a, len_b=b, len_min=lo, len_max=hi,
                        doc_alpha=doc_alpha, topic_beta=topic_beta, zipf_s=zipf_s, seed=seed, threads=threads,
                        doc_offset=doc_offset)
    off = np.zeros(D + 1, dtype=np.uint64)
    n = C.c_uint64()
    check(lib.tmt_synth_corpus(C.byref(spec), _p(off), None, 0, C.byref(n)), None, "synth lengths")
    words = np.zeros(max(n.value, 1), dtype=np.uint32)
    check(lib.tmt_synth_corpus(C.byref(spec), _p(off), _p(words), n.value, C.byref(n)), None, "synth words")
    return off, words[:n.value]


def prepare_ids(doc_off, words, min_cf=0, min_df=0, rm_top=0):
    """Integer-id corpus preparation as tomotopy's prepare() does it: vocab
    reorder by (cf, df) descending with the stop-word rules (removeStopwords,
    TopicModel.hpp:526-571), then each document sorted by id (prepareDoc,
    LDAModel.hpp:716-722).  Returns (doc_off, words, realV, order)."""
    doc_off = np.ascontiguousarray(doc_off, dtype=np.uint64)
    words = np.ascontiguousarray(words, dtype=np.uint32)
    D = len(doc_off) - 1
    nv = int(words.max()) + 1 if len(words) else 0
    out = np.zeros(max(len(words), 1), dtype=np.uint32)
    order = np.zeros(max(nv, 1), dtype=np.uint32)
    rv = C.c_uint32()
    check(lib.tmt_prepare_corpus(D, _p(doc_off), _p(words), nv, min_cf, min_df, rm_top, _p(out), None,
                                 _p(order), None, None, C.byref(rv)), None, "tmt_prepare_corpus")
    return doc_off, out[:len(words)], int(rv.value), order[:nv]


class Server:
    """Continuous-batching inference over resident frozen models (tmt_server_*)."""

    def __init__(self, max_slots=4096, token_budget=1 << 24, step_token_sweeps=4096, max_doc_len=1 << 16, device=0):
        cfg = TmtServerConfig(device=int(device), max_slots=int(max_slots), token_budget=int(token_budget),
                              step_token_sweeps=int(step_token_sweeps), max_doc_len=int(max_doc_len))
        h = C.c_void_p()
        check(lib.tmt_server_start(C.byref(cfg), C.byref(h)), None, "tmt_server_start")
        self.h = h
        self.K = {}

    def add_model(self, K, V, alpha, eta, n_kw, n_k):
        """A frozen model: int32 counts, or float counts (weighted: its requests
        then carry token weights)."""
        a = np.ascontiguousarray(np.broadcast_to(np.asarray(alpha, np.float32), (K,)))
        mid = C.c_uint32()
        if np.asarray(n_kw).dtype == np.float32:
            nkw = np.ascontiguousarray(n_kw, dtype=np.float32)
            nk = np.ascontiguousarray(n_k, dtype=np.float32)
            check(lib.tmt_server_add_model_f32(self.h, K, V, _p(a), float(eta), _p(nkw), _p(nk), C.byref(mid)),
                  None, "tmt_server_add_model_f32")
        else:
            nkw = np.ascontiguousarray(n_kw, dtype=np.int32)
            nk = np.ascontiguousarray(n_k, dtype=np.int32)
            check(lib.tmt_server_add_model(self.h, K, V, _p(a), float(eta), _p(nkw), _p(nk), C.byref(mid)), None,
                  "tmt_server_add_model")
        self.K[mid.value] = int(K)
        return mid.value

    def add_engine_model(self, eng):
        """A trained engine's frozen state, with its word priors; float counts
        for a weighted engine."""
        _, nkw, nk, alpha = eng.state()
        mid = self.add_model(eng.K, eng.V, alpha, eng.eta, nkw, nk)
        ids = getattr(eng, "_prior_ids", None)
        if ids is not None and len(ids):
            self.set_model_priors(mid, ids, eng._prior)
        return mid

    def set_model_priors(self, model_id, word_ids, priors):
        """tmt_server_set_model_priors, before the model's first request."""
        ids = np.ascontiguousarray(word_ids, dtype=np.uint32)
        pr = np.ascontiguousarray(priors, dtype=np.float32)
        check(lib.tmt_server_set_model_priors(self.h, int(model_id), len(ids), _p(ids), _p(pr)), None,
              "tmt_server_set_model_priors")

    def submit(self, model_id, words, iters=100, seed=0, key=0, weights=None):
        w = np.ascontiguousarray(words, dtype=np.uint32)
        rid = C.c_uint64()
        if weights is None:
            check(lib.tmt_server_submit(self.h, int(model_id), _p(w), len(w), int(iters), int(seed), int(key),
                                        C.byref(rid)), None, "tmt_server_submit")
        else:
            wt = np.ascontiguousarray(weights, dtype=np.float32)
            check(lib.tmt_server_submit_weighted(self.h, int(model_id), _p(w), _p(wt), len(w), int(iters),
                                                 int(seed), int(key), C.byref(rid)), None,
                  "tmt_server_submit_weighted")
        return rid.value

    def poll(self, wait_ms=1000):
        """(request_id, model_id, theta, ll, latency_ms) or None on timeout."""
        rid, mid = C.c_uint64(), C.c_uint32()
        cap = max(self.K.values()) if self.K else 1
        theta = np.zeros(cap, dtype=np.float32)
        ll, lat = C.c_double(), C.c_double()
        st = lib.tmt_server_poll(self.h, int(wait_ms), C.byref(rid), C.byref(mid), _p(theta), cap, C.byref(ll),
                                 C.byref(lat))
        if st == -7:
            return None
        if st != 0:
            raise TmtError(st, lib.tmt_server_last_error(self.h).decode())
        return rid.value, mid.value, theta[:self.K[mid.value]].copy(), ll.value, lat.value

    def submit_batch(self, model_ids, doc_off, words, iters=100, seed=0, keys=None, weights=None):
        """Queues len(doc_off) - 1 documents at once; returns their request ids."""
        off = np.ascontiguousarray(doc_off, dtype=np.uint64)
        w = np.ascontiguousarray(words, dtype=np.uint32)
        n = len(off) - 1
        mids = np.ascontiguousarray(np.broadcast_to(np.asarray(model_ids, np.uint32), (n,)))
        k = np.ascontiguousarray(keys, dtype=np.uint64) if keys is not None else None
        rids = np.zeros(max(n, 1), dtype=np.uint64)
        wt = np.ascontiguousarray(weights, dtype=np.float32) if weights is not None else None
        check(lib.tmt_server_submit_batch_weighted(self.h, _p(mids), _p(w), _p(wt), _p(off), n, int(iters),
                                                   int(seed), _p(k), _p(rids)), None, "tmt_server_submit_batch")
        return rids[:n]

    def poll_batch(self, max_n=4096, wait_ms=1000):
        """Up to max_n finished documents as arrays (request_id, model_id,
        theta [n x max K], ll, latency_ms), or None on timeout."""
        cap = max(self.K.values()) if self.K else 1
        rid = np.zeros(max_n, np.uint64)
        mid = np.zeros(max_n, np.uint32)
        theta = np.zeros((max_n, cap), np.float32)
        ll = np.zeros(max_n, np.float64)
        lat = np.zeros(max_n, np.float64)
        n = C.c_uint64()
        st = lib.tmt_server_poll_batch(self.h, int(wait_ms), int(max_n), _p(rid), _p(mid), _p(theta), cap, _p(ll),
                                       _p(lat), C.byref(n))
        if st == -7:
            return None
        if st != 0:
            raise TmtError(st, lib.tmt_server_last_error(self.h).decode())
        k = n.value
        return rid[:k], mid[:k], theta[:k], ll[:k], lat[:k]

    def stats(self):
        s = TmtServerStats()
        check(lib.tmt_server_get_stats(self.h, C.byref(s)), None, "tmt_server_get_stats")
        return s

    def close(self):
        if getattr(self, "h", None) is not None and self.h.value:
            lib.tmt_server_stop(self.h)
        self.h = None

    def __del__(self):
        self.close()
