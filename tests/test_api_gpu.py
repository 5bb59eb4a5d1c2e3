"""tomotopy's LDA API on the device path: the LDA cases of tomotopy's own
test/unit_test.py (train with several worker counts, a corpus whose every
word is removed, save/load as file and bytes with continued training, copy,
infer, infer together, uninitialised documents, reproducibility, asymmetric
alpha), on synthetic text documents."""
import numpy as np
import pytest

import tomotopy_b200 as tp

pytestmark = pytest.mark.gpu


def text_docs(n=200, V=1500, seed=4, mean=80):
    off, w = tp.synth_corpus(V, 12, n, ("poisson", mean, 1, 10 * mean), seed=seed)
    return [[f"w{x}" for x in w[off[d]:off[d + 1]]] for d in range(n)]


DOCS = text_docs()


def build(k=40, **kw):
    mdl = tp.LDAModel(k=k, seed=kw.pop("seed", 42), **kw)
    for d in DOCS:
        mdl.add_doc(d)
    return mdl


@pytest.mark.parametrize("workers,parallel", [(1, 0), (4, tp.ParallelScheme.PARTITION), (0, tp.ParallelScheme.COPY_MERGE)])
def test_train(workers, parallel):
    mdl = build()
    mdl.train(200, workers=workers, parallel=parallel)
    assert mdl.global_step == 200
    assert np.isfinite(mdl.ll_per_word) and mdl.ll_per_word < 0
    assert mdl.num_words == sum(len(d) for d in DOCS)
    assert mdl.get_count_by_topics().sum() == mdl.num_words
    assert len(mdl.get_topic_words(0, top_n=10)) == 10
    dist = mdl.get_topic_word_dist(3)
    assert dist.shape == (mdl.num_vocabs,) and abs(dist.sum() - 1) < 1e-4


def test_train_callback_and_optim():
    mdl = build(k=20)
    seen = []
    mdl.optim_interval = 5
    mdl.burn_in = 10
    mdl.train(40, callback_interval=10, callback=lambda m, c, t: seen.append((c, t)))
    assert seen == [(0, 40), (10, 40), (20, 40), (30, 40), (40, 40)]
    assert not np.allclose(mdl.alpha, 0.1)            # alpha was re-fitted


def test_null_doc():
    mdl = tp.LDAModel(k=10, min_df=200, rm_top=200, seed=1)
    for d in DOCS[:50]:
        mdl.add_doc(d)
    mdl.train(20)
    assert mdl.num_vocabs == 0 and mdl.num_words == 0
    assert mdl.ll_per_word == 0.0


def test_empty_document_is_ignored():
    mdl = tp.LDAModel(k=3, seed=1)
    assert mdl.add_doc([]) is None
    with pytest.raises(ValueError):
        mdl.add_doc([], ignore_empty_words=False)
    assert mdl.add_doc(["a", "b"]) == 0


def test_save_and_load(tmp_path):
    mdl = build(k=30)
    mdl.train(100)
    words0 = mdl.get_topic_words(5)
    ll0 = mdl.ll_per_word
    path = str(tmp_path / "model.bin")
    mdl.save(path)
    m2 = tp.LDAModel.load(path)
    assert m2.get_topic_words(5) == words0
    assert m2.ll_per_word == pytest.approx(ll0, rel=1e-12)
    assert m2.global_step == 100 and m2.init_params["k"] == 30
    np.testing.assert_array_equal(m2.docs[7].topics, mdl.docs[7].topics)
    m3 = tp.LDAModel.loads(mdl.saves(full=True))
    saved = mdl.saves(full=False)
    t2, ll2 = mdl.infer(mdl.make_doc(DOCS[0]))     # inference leaves the training state alone
    m2.train(20)
    m3.train(20)                        # same state, same seed: the same continuation
    mdl.train(20)                       # the seed travels in init_params
    np.testing.assert_array_equal(m2.docs[3].topics, m3.docs[3].topics)
    np.testing.assert_array_equal(m2.docs[3].topics, mdl.docs[3].topics)
    assert m2.global_step == 120
    # a model saved without its documents still infers
    m4 = tp.LDAModel.loads(saved)
    assert len(m4.docs) == 0
    t, ll = m4.infer(m4.make_doc(DOCS[0]))
    np.testing.assert_array_equal(t, t2)
    assert ll == ll2


def test_copy_train():
    mdl = build(k=20)
    mdl.train(50)
    cp = mdl.copy()
    assert cp.get_topic_words(2) == mdl.get_topic_words(2)
    mdl.train(20)
    cp.train(20)
    np.testing.assert_array_equal(cp.docs[0].topics, mdl.docs[0].topics)


def test_infer():
    mdl = build(k=25)
    mdl.train(100)
    unseen = text_docs(n=10, seed=99)
    docs = [mdl.make_doc(d) for d in unseen]
    dists, lls = mdl.infer(docs, iterations=50)
    assert len(dists) == 10 and len(lls) == 10
    for t in dists:
        assert t.shape == (25,) and abs(t.sum() - 1) < 1e-4
    t1, l1 = mdl.infer(docs[3], iterations=50)
    np.testing.assert_array_equal(t1, dists[3])
    assert l1 == lls[3]
    np.testing.assert_array_equal(docs[3].get_topic_dist(), dists[3])


def test_infer_together():
    mdl = build(k=25)
    mdl.train(100)
    docs = [mdl.make_doc(d) for d in text_docs(n=10, seed=98)]
    dists, ll = mdl.infer(docs, iterations=50, together=True)
    assert len(dists) == 10 and isinstance(ll, float) and np.isfinite(ll)
    for t in dists:
        assert abs(t.sum() - 1) < 1e-4


def test_uninit_doc():
    mdl = build(k=10)
    mdl.train(10)
    d = mdl.make_doc(DOCS[1])
    with pytest.raises(RuntimeError):
        d.get_topic_dist()
    mdl.infer(d)
    assert d.get_topic_dist().shape == (10,)


def test_reproducibility():
    tops = []
    for _ in range(3):
        mdl = build(k=20, seed=42)
        mdl.train(100, workers=1)
        tops.append([mdl.get_topic_words(k) for k in range(20)])
    assert tops[0] == tops[1] == tops[2]


def test_asymmetric_alpha():
    mdl = build(k=20, alpha=[0.1 * (i + 1) for i in range(20)])
    mdl.optim_interval = 0
    mdl.train(50)
    np.testing.assert_allclose(mdl.alpha, [0.1 * (i + 1) for i in range(20)], rtol=1e-6)
    with pytest.raises(ValueError):
        tp.LDAModel(k=5, alpha=[0.1, 0.2])


def test_document_views():
    mdl = build(k=15)
    mdl.train(30)
    d = mdl.docs[11]
    assert [mdl.vocabs[i] for i in d.words] == DOCS[11]           # original word order
    assert len(d.topics) == len(DOCS[11])
    assert abs(d.get_topic_dist().sum() - 1) < 1e-4
    assert np.isfinite(d.get_ll())
    assert mdl.used_vocabs == mdl.vocabs[:mdl.num_vocabs]
    assert sum(mdl.used_vocab_freq) == mdl.num_words
