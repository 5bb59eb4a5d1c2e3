"""tomotopy's LDAModel API over the B200 engine.

The same constructor, methods and properties as tomotopy.LDAModel
(tomotopy/models.py:48-660 in the tomotopy tree), with the dictionary and
documents held by the C++ host model (tmt_model_*) and the sampling state on
the GPU.  Differences that a caller can see:
  - `workers` and `parallel` are accepted and ignored: the sweep runs on the
    device with its own parallel scheme (one worker per document, document
    groups; see the design notes);
  - TermWeight ONE, IDF and PMI, and word priors (set_word_prior), all on the
    device path;
  - log-likelihoods are computed in FP64 with exact lgamma (tomotopy uses a
    float lookup table; the two agree to ~1e-5 relative).
"""
import ctypes as C
import os
import pickle
from copy import deepcopy
from enum import IntEnum
from typing import List, Optional, Tuple, Union

import numpy as np

from . import __version__ as _version
from ._lib import lib, TmtModelArgs, TmtModelInfo, TmtError

isa = "cuda-sm_100a"


class TermWeight(IntEnum):
    """tomotopy.TermWeight (__init__.py:10-33)."""
    ONE = 0
    IDF = 1
    PMI = 2


class ParallelScheme(IntEnum):
    """tomotopy.ParallelScheme (__init__.py:35-64); accepted, not used."""
    DEFAULT = 0
    NONE = 1
    COPY_MERGE = 2
    PARTITION = 3


def _check(st, m=None, what=""):
    if st == 0:
        return
    msg = lib.tmt_model_last_error(m).decode() if m is not None else what
    if st == -1:
        raise ValueError(msg)
    raise RuntimeError(msg or what or f"status {st}")


def _joined(words):
    ws = [str(w) for w in words]
    for w in ws:
        if "\0" in w:
            raise ValueError("words must not contain NUL characters")
    return ("\0".join(ws) + "\0").encode("utf-8") if ws else b"", len(ws)


def _p(a):
    return a.ctypes.data_as(C.c_void_p) if a is not None else None


class Document:
    """A document of a model (tomotopy.utils.Document, the LDA part)."""

    def __init__(self, model, index=None, words=None):
        self._model = model
        self._index = index
        self._words = words          # unbound documents (make_doc) keep their words
        self._theta = None
        self._ll = None

    def _bound(self):
        return self._index is not None

    @property
    def words(self):
        """word ids in the model's vocabulary, original order"""
        if not self._bound():
            return [self._model._word_id(w) for w in self._words if self._model._word_id(w) is not None]
        w, _ = self._model._doc_arrays(self._index)
        return w.tolist()

    @property
    def topics(self):
        """topic of every word, original order (0xFFFF-removed words as -1)"""
        if not self._bound():
            raise RuntimeError("topics of an unbound document are not kept")
        _, z = self._model._doc_arrays(self._index)
        return np.where(z == 0xFFFF, -1, z.astype(np.int32)).astype(np.int16)

    def __len__(self):
        return len(self.words)

    def get_topic_dist(self, normalize=True):
        """theta of the document (_getTopicsByDoc, LDAModel.hpp:1145-1159)"""
        if not self._bound():
            if self._theta is None:
                raise RuntimeError("call infer() first")
            return self._theta
        out = np.zeros(self._model.k, dtype=np.float32)
        _check(lib.tmt_model_doc_topic_dist(self._model._h, self._index, int(bool(normalize)), _p(out), None),
               self._model._h)
        return out

    def get_topics(self, top_n=10):
        d = self.get_topic_dist()
        idx = np.argsort(-d, kind="stable")[:top_n]
        return [(int(i), float(d[i])) for i in idx]

    def get_ll(self):
        """log-likelihood of the document's topic assignments (FP64)"""
        if not self._bound():
            return self._ll
        out = np.zeros(self._model.k, dtype=np.float32)
        ll = C.c_double()
        _check(lib.tmt_model_doc_topic_dist(self._model._h, self._index, 1, _p(out), C.byref(ll)), self._model._h)
        return ll.value


class LDAModel:
    """Latent Dirichlet Allocation (tomotopy.LDAModel) trained by collapsed Gibbs sampling on a B200."""

    def __init__(self, tw: Union[int, str] = "one", min_cf: int = 0, min_df: int = 0, rm_top: int = 0, k: int = 1,
                 alpha: Union[float, List[float]] = 0.1, eta: float = 0.01, seed: Optional[int] = None,
                 corpus=None, transform=None, device: int = 0, sweep_groups: int = 0):
        self.init_params = deepcopy({k_: v for k_, v in locals().items() if k_ != "self" and not k_.startswith("_")})
        self.init_params["version"] = _version
        if isinstance(tw, str):
            try:
                tw = TermWeight[tw.upper()]
            except KeyError:
                raise ValueError(f"Unknown term weight: {tw}")
        if int(tw) not in (TermWeight.ONE, TermWeight.IDF, TermWeight.PMI):
            raise ValueError(f"Unknown term weight: {tw}")
        if corpus is not None:
            raise NotImplementedError("tomotopy.utils.Corpus ingestion is out of scope; use add_doc")
        if not 1 <= int(k) <= 32767:
            raise ValueError(f"wrong K value (K = {k})")
        al = np.atleast_1d(np.asarray(alpha, dtype=np.float32))
        if seed is None:
            seed = int.from_bytes(os.urandom(4), "little")
        args = TmtModelArgs(K=int(k), alpha=al.ctypes.data_as(C.POINTER(C.c_float)), n_alpha=len(al), eta=float(eta),
                            seed=int(seed), min_cf=int(min_cf), min_df=int(min_df), rm_top=int(rm_top),
                            device=int(device), sweep_groups=int(sweep_groups), tw=int(tw))
        h = C.c_void_p()
        st = lib.tmt_model_create(C.byref(args), C.byref(h))
        self._h = h
        if st != 0:
            msg = lib.tmt_model_last_error(h).decode()
            self._close()
            raise ValueError(msg)
        self._word_index = None

    # -- lifetime ------------------------------------------------------------
    def _close(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            lib.tmt_model_destroy(self._h)
        self._h = None

    def __del__(self):
        self._close()

    def _info(self):
        i = TmtModelInfo()
        _check(lib.tmt_model_get_info(self._h, C.byref(i)), self._h)
        return i

    # -- documents -----------------------------------------------------------
    def add_doc(self, words, ignore_empty_words=True) -> Optional[int]:
        """Adds a document (an iterable of str); returns its index, or None for an empty one."""
        if isinstance(words, str):
            raise ValueError("`words` must be an iterable of str")
        buf, n = _joined(words)
        if n == 0 and not ignore_empty_words:
            raise ValueError("A document should have at least one word")
        did = C.c_int64()
        _check(lib.tmt_model_add_doc(self._h, buf, n, C.byref(did)), self._h)
        self._word_index = None
        return None if did.value < 0 else did.value

    def make_doc(self, words) -> Document:
        """An unseen document for infer(); words outside the vocabulary are dropped at inference."""
        if isinstance(words, str):
            raise ValueError("`words` must be an iterable of str")
        return Document(self, None, [str(w) for w in words])

    @property
    def docs(self):
        """the documents of the model (read-only)"""
        return [Document(self, i) for i in range(self._info().n_docs)]

    def _doc_arrays(self, i):
        n = C.c_uint32()
        _check(lib.tmt_model_doc(self._h, int(i), None, None, C.byref(n)), self._h)
        w = np.zeros(max(1, n.value), dtype=np.uint32)
        z = np.zeros(max(1, n.value), dtype=np.uint16)
        _check(lib.tmt_model_doc(self._h, int(i), _p(w), _p(z), C.byref(n)), self._h)
        return w[:n.value], z[:n.value]

    def _vocab_list(self, used_only):
        need = C.c_uint64()
        _check(lib.tmt_model_vocab(self._h, int(used_only), None, 0, C.byref(need)), self._h)
        buf = C.create_string_buffer(max(1, need.value))
        _check(lib.tmt_model_vocab(self._h, int(used_only), buf, need.value, C.byref(need)), self._h)
        raw = buf.raw[:need.value]
        return [w.decode("utf-8") for w in raw.split(b"\0")[:-1]] if need.value else []

    def _word_id(self, w):
        if self._word_index is None:
            self._word_index = {x: i for i, x in enumerate(self._vocab_list(False))}
        return self._word_index.get(w)

    # -- training --------------------------------------------------------------
    def train(self, iterations=10, workers=0, parallel=0, freeze_topics=False, callback_interval=10, callback=None,
              show_progress=False) -> None:
        """Runs `iterations` Gibbs sweeps on the GPU (workers / parallel are accepted and ignored)."""
        if show_progress:
            inner = callback

            def callback(mdl, cur, tot):
                if inner is not None:
                    inner(mdl, cur, tot)
                print(f"iteration {cur}/{tot}  ll_per_word {mdl.ll_per_word:.5f}", flush=True)
        _check(lib.tmt_model_prepare(self._h), self._h)
        self._word_index = None
        if callback is None or callback_interval <= 0:
            if callback is not None:
                callback(self, 0, iterations)
            _check(lib.tmt_model_train(self._h, int(iterations)), self._h)
            if callback is not None:
                callback(self, iterations, iterations)
            return
        done = 0
        callback(self, 0, iterations)
        while done < iterations:
            n = min(callback_interval, iterations - done)
            _check(lib.tmt_model_train(self._h, int(n)), self._h)
            done += n
            callback(self, done, iterations)

    # -- inference ---------------------------------------------------------------
    def infer(self, doc, iterations=100, tolerance=-1, workers=0, parallel=0, together=False,
              transform=None) -> Tuple:
        """Topic distributions of unseen documents (LDAModel.hpp:843-954).

        One Document -> (topic_dist, ll); a list -> (list of topic_dist, list of ll), or a
        single ll when together=True."""
        if not self._info().prepared:
            raise RuntimeError("cannot infer with untrained model")
        single = isinstance(doc, Document)
        docs = [doc] if single else list(doc)
        for d in docs:
            if not isinstance(d, Document):
                raise ValueError("`doc` must be tomotopy.Document type or list of tomotopy.Document")
            if d._model is not self:
                raise ValueError("`doc` was from another model, not fit to this model")
        words = [d._words if not d._bound() else [self.vocabs[i] for i in d.words] for d in docs]
        counts = np.array([len(w) for w in words], dtype=np.uint64)
        buf = b"".join((("\0".join(map(str, w)) + "\0").encode("utf-8") if len(w) else b"") for w in words)
        K = self.k
        theta = np.zeros((max(1, len(docs)), K), dtype=np.float32)
        if together:
            ll = C.c_double()
            _check(lib.tmt_model_infer_together(self._h, buf, _p(counts), len(docs), int(iterations), 0,
                                                _p(theta), C.byref(ll)), self._h)
            lls = ll.value
        else:
            lla = np.zeros(max(1, len(docs)), dtype=np.float64)
            _check(lib.tmt_model_infer(self._h, buf, _p(counts), len(docs), int(iterations), 0, _p(theta),
                                       _p(lla)), self._h)
            lls = lla[:len(docs)].tolist()
        dists = [theta[i].copy() for i in range(len(docs))]
        for d, t, l_ in zip(docs, dists, lls if not together else [lls] * len(docs)):
            if not d._bound():
                d._theta, d._ll = t, l_
        if single:
            return dists[0], (lls[0] if not together else lls)
        return dists, lls

    # -- queries ---------------------------------------------------------------
    def get_topic_word_dist(self, topic_id, normalize=True) -> np.ndarray:
        """p(word | topic) over the used vocabulary (_getWidsByTopic, LDAModel.hpp:828-841)."""
        V = self._info().V
        out = np.zeros(max(1, V), dtype=np.float32)
        _check(lib.tmt_model_topic_word_dist(self._h, int(topic_id), int(bool(normalize)), _p(out)), self._h)
        return out[:V]

    def get_topic_words(self, topic_id, top_n=10, return_id=False):
        """The top_n words of a topic with their probabilities (ties by word id)."""
        dist = self.get_topic_word_dist(topic_id)
        idx = np.argsort(-dist, kind="stable")[:top_n]
        vocab = self._vocab_list(True)
        if return_id:
            return [(vocab[i], int(i), float(dist[i])) for i in idx]
        return [(vocab[i], float(dist[i])) for i in idx]

    def get_count_by_topics(self) -> np.ndarray:
        out = np.zeros(self.k, dtype=np.uint64)
        _check(lib.tmt_model_count_by_topics(self._h, _p(out)), self._h)
        return out

    def get_word_prior(self, word) -> List[float]:
        """The topic distribution prior of `word` (tomotopy's get_word_prior):
        its K priors, or [] when it has none."""
        n = C.c_uint32()
        _check(lib.tmt_model_get_word_prior(self._h, word.encode(), None, C.byref(n)), self._h)
        out = np.zeros(max(n.value, 1), dtype=np.float32)
        _check(lib.tmt_model_get_word_prior(self._h, word.encode(), _p(out), C.byref(n)), self._h)
        return [float(x) for x in out[:n.value]]

    def set_word_prior(self, word, prior):
        """Sets the topic distribution prior of `word` (tomotopy's set_word_prior,
        py_LDA.cpp:241-269): a list of K floats, or a dict {topic_id: float}
        whose missing topics keep eta.  Before train() only."""
        if self._info().prepared:
            raise RuntimeError("cannot set_word_prior() after train()")
        k = self.k
        if isinstance(prior, dict):
            vals = np.full(k, self.eta, dtype=np.float32)
            for t, v in prior.items():
                t = int(t)
                if t < 0 or t >= k:
                    raise ValueError("`prior` must be a dict of {topic_id: float}")
                vals[t] = float(v)
        else:
            try:
                vals = np.asarray([float(x) for x in prior], dtype=np.float32)
            except (TypeError, ValueError):
                raise ValueError("`prior` must be a list of floats with len = k")
        _check(lib.tmt_model_set_word_prior(self._h, str(word).encode(), _p(vals), len(vals)), self._h)

    def summary(self, initial_hp=True, params=True, topic_word_top_n=5, file=None, flush=False):
        import sys
        file = file or sys.stdout
        i = self._info()
        print(f"<Basic Info>\n| LDAModel (current version: {_version})\n| {i.n_docs} docs, {i.N} words\n"
              f"| Total Vocabs: {i.n_vocab}, Used Vocabs: {i.V}\n| Term Weighting: {TermWeight(i.tw).name}",
              file=file)
        print(f"<Training Info>\n| Iterations: {i.global_step}", file=file)
        if i.prepared:
            print(f"| Log-likelihood per word: {self.ll_per_word:.5f}", file=file)
        if params:
            print(f"<Parameters>\n| alpha: {self.alpha}\n| eta: {self.eta}", file=file)
        if i.prepared and topic_word_top_n > 0:
            print("<Topics>", file=file)
            cnt = self.get_count_by_topics()
            for kk in range(self.k):
                ws = " ".join(w for w, _ in self.get_topic_words(kk, top_n=topic_word_top_n))
                print(f"| #{kk} ({int(cnt[kk])}) : {ws}", file=file)
        if flush:
            file.flush()

    # -- persistence -------------------------------------------------------------
    def saves(self, full=True) -> bytes:
        """tomotopy's binary model layout (TopicModel.hpp:335-359), init_params pickled as extra data."""
        extra = pickle.dumps(self.init_params)
        eb = np.frombuffer(extra, dtype=np.uint8).copy()
        out = C.POINTER(C.c_uint8)()
        n = C.c_uint64()
        _check(lib.tmt_model_save(self._h, _p(eb), len(eb), int(bool(full)), C.byref(out), C.byref(n)), self._h)
        try:
            return C.string_at(out, n.value)
        finally:
            lib.tmt_model_free_buffer(out)

    def save(self, filename: str, full=True) -> None:
        data = self.saves(full)
        with open(filename, "wb") as f:
            f.write(data)

    @classmethod
    def loads(cls, data: bytes, device: int = 0, sweep_groups: int = 0) -> "LDAModel":
        buf = np.frombuffer(bytes(data), dtype=np.uint8).copy()
        h = C.c_void_p()
        ex = C.POINTER(C.c_uint8)()
        exn = C.c_uint64()
        st = lib.tmt_model_load(_p(buf), len(buf), int(device), int(sweep_groups), C.byref(h), C.byref(ex),
                                C.byref(exn))
        try:
            extra = C.string_at(ex, exn.value) if exn.value else b""
        finally:
            if ex:
                lib.tmt_model_free_buffer(ex)
        if st != 0:
            msg = lib.tmt_model_last_error(h).decode() if h.value else "load failed"
            if h.value:
                lib.tmt_model_destroy(h)
            raise ValueError(msg)
        inst = cls.__new__(cls)
        inst._h = h
        inst._word_index = None
        try:
            inst.init_params = pickle.loads(extra) if extra else {}
        except Exception:
            inst.init_params = {}
        seed = inst.init_params.get("seed") if isinstance(inst.init_params, dict) else None
        if isinstance(seed, int):
            _check(lib.tmt_model_set_seed(h, seed & 0xFFFFFFFFFFFFFFFF), h)
        return inst

    @classmethod
    def load(cls, filename: str, device: int = 0, sweep_groups: int = 0) -> "LDAModel":
        with open(filename, "rb") as f:
            return cls.loads(f.read(), device, sweep_groups)

    def copy(self) -> "LDAModel":
        """A deep copy (through the binary layout)."""
        c = type(self).loads(self.saves(full=True), device=int(self.init_params.get("device", 0)))
        c.init_params = deepcopy(self.init_params)
        _check(lib.tmt_model_set_seed(c._h, self._info().seed), c._h)
        return c

    # -- properties --------------------------------------------------------------
    @property
    def k(self) -> int:
        return self._info().K

    @property
    def alpha(self) -> np.ndarray:
        """the per-topic Dirichlet prior (after optimisation)"""
        out = np.zeros(self.k, dtype=np.float32)
        if self._info().prepared:
            _check(lib.tmt_model_alpha(self._h, _p(out)), self._h)
        else:
            a = np.atleast_1d(np.asarray(self.init_params.get("alpha", 0.1), dtype=np.float32))
            out[:] = np.broadcast_to(a, out.shape)
        return out

    @property
    def eta(self) -> float:
        return float(self._info().eta)

    @property
    def tw(self) -> int:
        return int(self._info().tw)

    @property
    def global_step(self) -> int:
        return int(self._info().global_step)

    @property
    def ll_per_word(self) -> float:
        i = self._info()
        if not i.prepared or i.N == 0:
            return 0.0
        a, b = C.c_double(), C.c_double()
        _check(lib.tmt_model_ll(self._h, C.byref(a), C.byref(b)), self._h)
        # TopicModel::getLLPerWord divides by weightedN (TopicModel.hpp:757-760)
        return (a.value + b.value) / (i.weighted_n or i.N)

    @property
    def perplexity(self) -> float:
        return float(np.exp(-self.ll_per_word))

    @property
    def num_vocabs(self) -> int:
        return int(self._info().V)

    @property
    def num_words(self) -> int:
        return int(self._info().N)

    @property
    def optim_interval(self) -> int:
        return int(self._info().optim_interval)

    @optim_interval.setter
    def optim_interval(self, value: int):
        i = self._info()
        _check(lib.tmt_model_set_optim(self._h, int(value), int(i.burn_in)), self._h)

    @property
    def burn_in(self) -> int:
        return int(self._info().burn_in)

    @burn_in.setter
    def burn_in(self, value: int):
        i = self._info()
        _check(lib.tmt_model_set_optim(self._h, int(i.optim_interval), int(value)), self._h)

    @property
    def vocabs(self) -> List[str]:
        return self._vocab_list(False)

    @property
    def used_vocabs(self) -> List[str]:
        return self._vocab_list(True)

    def _freqs(self):
        n = self._info().n_vocab
        cf = np.zeros(max(1, n), dtype=np.uint64)
        df = np.zeros(max(1, n), dtype=np.uint64)
        _check(lib.tmt_model_vocab_freq(self._h, _p(cf), _p(df)), self._h)
        return cf[:n], df[:n]

    @property
    def vocab_freq(self) -> List[int]:
        return self._freqs()[0].tolist()

    @property
    def vocab_df(self) -> List[int]:
        return self._freqs()[1].tolist()

    @property
    def used_vocab_freq(self) -> List[int]:
        return self._freqs()[0][:self.num_vocabs].tolist()

    @property
    def used_vocab_df(self) -> List[int]:
        return self._freqs()[1][:self.num_vocabs].tolist()

    @property
    def removed_top_words(self) -> List[str]:
        i = self._info()
        if not i.prepared or not i.rm_top:
            return []
        return self._vocab_list(False)[i.n_vocab - i.rm_top:]
