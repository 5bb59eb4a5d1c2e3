"""tomotopy's binary model layout: files written by tomotopy's own serializer
(tests/golden/lda_*.bin, from oracle/_ref/libtmtserial.so: serializer.hpp,
Dictionary.cpp, SharedString.cpp, tvector.hpp of the tomotopy tree) are read
by the host model and written back byte for byte.  Parse-only loads
(device -1), no GPU."""
import ctypes as C
import os

import numpy as np
import pytest

import tomotopy_b200 as tp
from tomotopy_b200._lib import lib, TmtModelInfo

G = os.path.join(os.path.dirname(__file__), "golden")
F = np.load(os.path.join(G, "lda_fields.npz"))


def _load(name):
    data = np.frombuffer(open(os.path.join(G, name), "rb").read(), np.uint8).copy()
    h = C.c_void_p()
    ex = C.POINTER(C.c_uint8)()
    exn = C.c_uint64()
    st = lib.tmt_model_load(data.ctypes.data_as(C.c_void_p), len(data), -1, 0, C.byref(h), C.byref(ex), C.byref(exn))
    assert st == 0, lib.tmt_model_last_error(h)
    extra = C.string_at(ex, exn.value)
    lib.tmt_model_free_buffer(ex)
    return h, extra, data.tobytes()


def _save(h, extra, full):
    eb = np.frombuffer(extra, np.uint8).copy()
    out = C.POINTER(C.c_uint8)()
    n = C.c_uint64()
    assert lib.tmt_model_save(h, eb.ctypes.data_as(C.c_void_p), len(eb), full, C.byref(out), C.byref(n)) == 0, \
        lib.tmt_model_last_error(h)
    b = C.string_at(out, n.value)
    lib.tmt_model_free_buffer(out)
    return b


@pytest.mark.parametrize("name,full", [("lda_full.bin", 1), ("lda_model_only.bin", 0)])
def test_golden_round_trip_bytes(name, full):
    h, extra, raw = _load(name)
    assert extra == bytes(range(37))
    assert _save(h, extra, full) == raw
    if full:
        # the full file also gives the model-only file
        assert _save(h, extra, 0) == open(os.path.join(G, "lda_model_only.bin"), "rb").read()
    lib.tmt_model_destroy(h)


def test_golden_fields():
    h, extra, raw = _load("lda_full.bin")
    i = TmtModelInfo()
    assert lib.tmt_model_get_info(h, C.byref(i)) == 0
    assert (i.K, i.V, i.n_vocab, i.n_docs, i.global_step) == (int(F["K"]), int(F["realV"]), int(F["nv"]), 12, 123)
    assert (i.burn_in, i.optim_interval) == (5, 10)
    assert i.eta == pytest.approx(0.02)
    K, V = int(F["K"]), int(F["realV"])
    a = np.zeros(K, np.float32)
    assert lib.tmt_model_alpha(h, a.ctypes.data_as(C.c_void_p)) == 0
    np.testing.assert_array_equal(a, F["alphas"])
    cnt = np.zeros(K, np.uint64)
    assert lib.tmt_model_count_by_topics(h, cnt.ctypes.data_as(C.c_void_p)) == 0
    np.testing.assert_array_equal(cnt, F["nk"])
    dist = np.zeros(V, np.float32)
    assert lib.tmt_model_topic_word_dist(h, 2, 1, dist.ctypes.data_as(C.c_void_p)) == 0
    ref = (F["nkw"][:, 2].astype(np.float32) + np.float32(0.02)) / (np.float32(F["nk"][2]) + np.float32(V) * np.float32(0.02))
    np.testing.assert_allclose(dist, ref, rtol=1e-6)
    need = C.c_uint64()
    lib.tmt_model_vocab(h, 0, None, 0, C.byref(need))
    buf = C.create_string_buffer(need.value)
    lib.tmt_model_vocab(h, 0, buf, need.value, C.byref(need))
    assert [w.decode() for w in buf.raw.split(b"\0")[:-1]] == list(F["vocab"])
    off, words, order, zs = F["doc_off"], F["words"], F["w_order"], F["zs"]
    for d in range(12):
        b, e = int(off[d]), int(off[d + 1])
        n = C.c_uint32()
        w = np.zeros(max(1, e - b), np.uint32)
        z = np.zeros(max(1, e - b), np.uint16)
        assert lib.tmt_model_doc(h, d, w.ctypes.data_as(C.c_void_p), z.ctypes.data_as(C.c_void_p), C.byref(n)) == 0
        assert n.value == e - b
        np.testing.assert_array_equal(w[:n.value], words[b:e][order[b:e]])
        np.testing.assert_array_equal(z[:n.value], zs[b:e][order[b:e]])
    lib.tmt_model_destroy(h)


def test_python_loads_parse_only():
    data = open(os.path.join(G, "lda_full.bin"), "rb").read()
    m = tp.LDAModel.loads(data, device=-1)
    assert m.k == int(F["K"]) and m.num_vocabs == int(F["realV"]) and m.global_step == 123
    assert len(m.docs) == 12
    np.testing.assert_array_equal(m.get_count_by_topics(), F["nk"])
    top = m.get_topic_words(0, top_n=3)
    assert len(top) == 3 and all(isinstance(w, str) for w, _ in top)


def test_corrupt_input_is_rejected():
    data = bytearray(open(os.path.join(G, "lda_full.bin"), "rb").read())
    for cut in (3, 40, 200, len(data) - 5):
        with pytest.raises(ValueError):
            tp.LDAModel.loads(bytes(data[:cut]), device=-1)
    bad = bytearray(data)
    bad[0:3] = b"HDP"
    with pytest.raises(ValueError):
        tp.LDAModel.loads(bytes(bad), device=-1)
