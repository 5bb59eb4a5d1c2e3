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


class SweepSpec(C.Structure):
    """orc_sweep_spec (tmt_oracle.h)."""
    _fields_ = [("K", C.c_uint32), ("V", C.c_uint32), ("alpha", C.c_void_p), ("eta", C.c_float),
                ("pidx", C.c_void_p), ("prior", C.c_void_p), ("esum", C.c_void_p),
                ("alpha_rows", C.c_void_p), ("arow", C.c_void_p), ("mask", C.c_void_p),
                ("seed", C.c_uint64), ("iter", C.c_uint32),
                ("doc_off", C.c_void_p), ("words", C.c_void_p),
                ("ndk", C.c_void_p), ("nkw", C.c_void_p), ("nk", C.c_void_p),
                ("nkw_next", C.c_void_p), ("nk_next", C.c_void_p), ("z", C.c_void_p),
                ("split_len", C.c_uint64), ("slices", C.c_uint32), ("step", C.c_uint32),
                ("unit_off", C.c_void_p), ("unit_docs", C.c_void_p)]


# The long-document split of the device sweep (engine.cu, split_len_of): a
# document of at least split_len tokens is sampled as SPLIT_SLICES slices side
# by side, merging their n_dk changes every `step` positions.  split_len per
# document group: max(8 * (SPLIT_SLICES - 1) * step, ceil(group tokens / 4096)),
# for integer counts with K <= SPLIT_MAX_K.
SPLIT_SLICES, SPLIT_STEP, SPLIT_MAX_K = 8, 16, 512


def split_len_of(group_tokens, K, min_len=0, step=SPLIT_STEP):
    """The split threshold of a document group (0: no document is split).
    min_len: the engine's override (0: the rule; >= 2^32 - 1: never)."""
    if K > SPLIT_MAX_K or min_len >= 0xFFFFFFFF:
        return 0
    if min_len:
        return int(min_len)
    return max(8 * (SPLIT_SLICES - 1) * int(step), (int(group_tokens) + 4095) // 4096)


class SynthSpec(C.Structure):
    """orc_synth_spec (tmt_oracle.h)."""
    _fields_ = [("V", C.c_uint32), ("T", C.c_uint32), ("D", C.c_uint64), ("len_kind", C.c_int32),
                ("len_a", C.c_double), ("len_b", C.c_double), ("len_min", C.c_uint32), ("len_max", C.c_uint32),
                ("doc_alpha", C.c_double), ("topic_beta", C.c_double), ("zipf_s", C.c_double),
                ("seed", C.c_uint64), ("doc_offset", C.c_uint64)]


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
        "orc_draw_intervals": (C.c_float, [V, V, C.c_uint32, C.c_uint32, C.c_float, V, V]),
        "orc_sweep_docs": (None, [C.POINTER(SweepSpec), V, C.c_uint64]),
        "orc_synth_corpus": (C.c_int, [C.POINTER(SynthSpec), V, V, C.c_uint64, V, C.c_uint32]),
        "orc_prepare_corpus": (C.c_uint64, [C.c_uint64, V, V, C.c_uint64, C.c_uint64, C.c_uint64, C.c_uint64, V,
                                            C.c_uint32]),
        "orc_blocked_draw": (C.c_uint32, [V, V, C.c_uint32, C.c_uint32, C.c_float, C.c_float]),
        "orc_ref_draw_intervals": (C.c_float, [V, V, V, C.c_uint32, V]),
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


def synth_corpus(V, T, D, length, seed, doc_alpha=0.1, topic_beta=0.01, zipf_s=1.07, threads=0, doc_offset=0):
    """The benchmark's seeded synthetic corpus, generated without the engine
    (orc_synth_corpus): length = ("poisson", mean, lo, hi) or ("lognormal",
    mu, sigma, lo, hi).  Returns (doc_off uint64[D+1], words uint32[N])."""
    if length[0] == "poisson":
        kind, a, b, lo, hi = 0, float(length[1]), 0.0, int(length[2]), int(length[3])
    else:
        kind, a, b, lo, hi = 1, float(length[1]), float(length[2]), int(length[3]), int(length[4])
    spec = SynthSpec(V=V, T=T, D=D, len_kind=kind, len_a=a, len_b=b, len_min=lo, len_max=hi, doc_alpha=doc_alpha,
                     topic_beta=topic_beta, zipf_s=zipf_s, seed=seed, doc_offset=doc_offset)
    th = threads or os.cpu_count() or 1
    off = np.zeros(D + 1, dtype=np.uint64)
    n = np.zeros(1, dtype=np.uint64)
    if lib.orc_synth_corpus(C.byref(spec), _ptr(off), None, 0, _ptr(n), th) != 0:
        raise ValueError("bad synthetic corpus spec")
    words = np.zeros(max(int(n[0]), 1), dtype=np.uint32)
    lib.orc_synth_corpus(C.byref(spec), _ptr(off), _ptr(words), int(n[0]), _ptr(n), th)
    return off, words[:int(n[0])]


def prepare_ids(doc_off, words, min_cf=0, min_df=0, rm_top=0, threads=0):
    """removeStopwords + prepareDoc of a corpus (orc_prepare_corpus):
    returns (doc_off, words renumbered and sorted per document, realV, order)."""
    doc_off = np.ascontiguousarray(doc_off, dtype=np.uint64)
    out = np.ascontiguousarray(words, dtype=np.uint32).copy()
    nv = int(out.max()) + 1 if len(out) else 0
    order = np.zeros(max(nv, 1), dtype=np.uint32)
    rv = lib.orc_prepare_corpus(len(doc_off) - 1, _ptr(doc_off), _ptr(out), nv, min_cf, min_df, rm_top,
                                _ptr(order), threads or os.cpu_count() or 1)
    return doc_off, out, int(rv), order[:nv]


def token_factors(ndk_row, nkw_col, nk, alpha, eta, V, zo):
    """The float operands of one token's draw with the token removed: the
    device's (A, phi, phi_own) and tomotopy's (A, B, C) of getZLikelihoods
    (LDAModel.hpp:273-285), each rounded as the code rounds it."""
    K = len(nk)
    veta = np.float32(eta) * np.float32(V)
    own = (np.arange(K) == zo).astype(np.int32)
    A = f32((np.asarray(ndk_row) - own).astype(np.float32) + f32(alpha))
    R = f32(np.float32(1) / (np.asarray(nk).astype(np.float32) + veta))
    phi = f32((np.asarray(nkw_col).astype(np.float32) + np.float32(eta)) * R)
    phi_own = np.float32((np.float32(nkw_col[zo] - 1) + np.float32(eta)) *
                         (np.float32(1) / (np.float32(nk[zo] - 1) + veta)))
    B = f32((np.asarray(nkw_col) - own).astype(np.float32) + np.float32(eta))
    Cc = f32((np.asarray(nk) - own).astype(np.float32) + veta)
    return A, phi, phi_own, B, Cc


def implied_conditionals(ndk_row, nkw_col, nk, alpha, eta, V, zo):
    """(p_device, p_tomotopy, p_f64): the topic probabilities the device's
    blocked draw and tomotopy's prefix-sum draw imply for one token (interval
    widths over the total), and the FP64 conditional."""
    K = len(nk)
    A, phi, phi_own, B, Cc = token_factors(ndk_row, nkw_col, nk, alpha, eta, V, zo)
    w = np.zeros(K)
    t = lib.orc_draw_intervals(_ptr(A), _ptr(phi), K, int(zo), float(phi_own), _ptr(w), None)
    wr = np.zeros(K)
    tr = lib.orc_ref_draw_intervals(_ptr(A), _ptr(B), _ptr(Cc), K, _ptr(wr))
    p64 = np.zeros(K)
    lib.orc_conditional_f64(K, V, _ptr(f32(alpha)), float(eta), _ptr(np.ascontiguousarray(ndk_row, np.int32)),
                            _ptr(np.ascontiguousarray(nkw_col, np.int32)), _ptr(np.ascontiguousarray(nk, np.int32)),
                            int(zo), _ptr(p64))
    return w / t, wr / tr, p64


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

    def _spec_extra(self):
        """orc_sweep_spec fields of the conditional's options (priors, masks)."""
        return {}

    def doc_live_sweeps(self, iters, start_step=0, groups=1, split_min=0, split_step=SPLIT_STEP):
        """The device sweep: doc-major, live n_dk, snapshot n_kw / n_k,
        sampled group by group (see group_bounds), the snapshot refreshed
        between groups; long documents split as the engine splits them
        (split_min / split_step: the engine's tmt_set_doc_split)."""
        c = self.c
        order, b = self.group_bounds(groups)
        lens = np.diff(c.doc_off.astype(np.int64))
        parts = [np.ascontiguousarray(order[b[g]:b[g + 1]]) for g in range(groups)]
        splits = [split_len_of(lens[p.astype(np.int64)].sum(), self.K, split_min, split_step) for p in parts]
        extra = self._spec_extra()
        for it in range(iters):
            for part, sl in zip(parts, splits):
                if len(part) == 0:
                    continue
                nkw2 = self.nkw.copy()
                nk2 = self.nk.copy()
                sp = SweepSpec(K=self.K, V=c.V, alpha=self.alpha.ctypes.data, eta=self.eta, seed=self.seed,
                               iter=start_step + it, doc_off=c.doc_off.ctypes.data, words=c.words.ctypes.data,
                               ndk=self.ndk.ctypes.data, nkw=self.nkw.ctypes.data, nk=self.nk.ctypes.data,
                               nkw_next=nkw2.ctypes.data, nk_next=nk2.ctypes.data, z=self.z.ctypes.data,
                               split_len=sl, slices=SPLIT_SLICES, step=int(split_step), **extra)
                lib.orc_sweep_docs(C.byref(sp), _ptr(part), len(part))
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

    def _spec_extra(self):
        return dict(pidx=self.pidx.ctypes.data, prior=self.prior.ctypes.data, esum=self.esum.ctypes.data)

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

    def _spec_extra(self):
        e = {}
        if self.mask_bits is not None:
            e["mask"] = self.mask_bits.ctypes.data
        if self.alpha_rows is not None:
            e["alpha_rows"] = self.alpha_rows.ctypes.data
            e["arow"] = self.doc_row.ctypes.data
        return e

    def ll_f64(self):
        a, b = super().ll_f64()
        if self.alpha_rows is not None:
            c = self.c
            a = lib.orc_ll_docs_m_f64(c.D, self.K, _ptr(self.ndk), _ptr(c.doc_len), _ptr(self.alpha_rows),
                                      _ptr(self.doc_row))
        return a, b


class StateR(State):
    """Shared document rows (PT's pseudo-documents, PTModel.hpp:13-24): document
    d counts in row row_of[d] of R rows of n_dk; a sweep samples each row's
    documents one after another (ascending index) with the row live, the rows
    ordered and grouped as documents are (by their total length).  ll_docs and
    the alpha optimiser run over the rows."""

    def __init__(self, corpus, K, alpha, eta, seed, row_of, R, z0=None):
        self.row_of = np.ascontiguousarray(row_of, dtype=np.uint32)
        self.R = int(R)
        super().__init__(corpus, K, alpha, eta, seed, z0=z0)

    def set_rows(self, row_of, R):
        self.row_of = np.ascontiguousarray(row_of, dtype=np.uint32)
        self.R = int(R)
        self.recount()

    def recount(self):
        super().recount()              # n_kw, n_k (and per-document rows, replaced below)
        c = self.c
        self.ndk = np.zeros((self.R, self.K), dtype=np.int32)
        ok = c.words < c.V
        doc = np.repeat(np.arange(c.D), np.diff(c.doc_off.astype(np.int64)))
        np.add.at(self.ndk, (self.row_of[doc[ok]].astype(np.int64), self.z[ok].astype(np.int64)), 1)
        self.row_len = np.zeros(self.R, dtype=np.int32)
        np.add.at(self.row_len, self.row_of.astype(np.int64), c.doc_len)
        lens = np.diff(c.doc_off.astype(np.int64))
        self.unit_len = np.zeros(self.R, dtype=np.int64)
        np.add.at(self.unit_len, self.row_of.astype(np.int64), lens)
        self.unit_docs = np.argsort(self.row_of, kind="stable").astype(np.uint32)
        self.unit_off = np.concatenate([[0], np.cumsum(np.bincount(self.row_of, minlength=self.R))]).astype(np.uint64)

    def group_bounds(self, groups):
        order = np.argsort(-self.unit_len, kind="stable").astype(np.uint64)
        total = int(self.unit_len.sum())
        prefix = np.concatenate([[0], np.cumsum(self.unit_len[order.astype(np.int64)])[:-1]]) if self.R else \
            np.zeros(0)
        bounds = [0] + [int(np.sum(prefix * groups < g * total)) for g in range(1, groups)] + [self.R]
        return order, bounds

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
                sp = SweepSpec(K=self.K, V=c.V, alpha=self.alpha.ctypes.data, eta=self.eta, seed=self.seed,
                               iter=start_step + it, doc_off=c.doc_off.ctypes.data, words=c.words.ctypes.data,
                               ndk=self.ndk.ctypes.data, nkw=self.nkw.ctypes.data, nk=self.nk.ctypes.data,
                               nkw_next=nkw2.ctypes.data, nk_next=nk2.ctypes.data, z=self.z.ctypes.data,
                               split_len=0, slices=SPLIT_SLICES, step=SPLIT_STEP,
                               unit_off=self.unit_off.ctypes.data, unit_docs=self.unit_docs.ctypes.data)
                lib.orc_sweep_docs(C.byref(sp), _ptr(part), len(part))
                self.nkw = nkw2
                self.nk = nk2

    def optimize_alpha(self):
        lib.orc_optimize_alpha(self.R, self.K, _ptr(self.ndk), _ptr(self.row_len), _ptr(self.alpha))

    def ll_f64(self):
        a = lib.orc_ll_docs_f64(self.R, self.K, _ptr(self.ndk), _ptr(self.row_len), _ptr(self.alpha))
        b = lib.orc_ll_rest_f64(self.K, self.c.V, _ptr(self.nkw), _ptr(self.nk), self.eta)
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
