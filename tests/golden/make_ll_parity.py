"""Generates tests/golden/ll_partition.json: the ll_per_word curve of
tomotopy's own train() on the benchmark corpora, for the ll-parity gate.

tomotopy's train() runs ParallelScheme::PARTITION on all host threads
(TopicModel.hpp:684-755, LDAModel.hpp:356-428, 436-489) with the model's
defaults optim_interval=10, burn_in=0 (LDAModel.hpp:210, 529-532).  tomotopy
itself cannot be built here (its CMake fetches Eigen and EigenRand), so the
oracle's C restatement of that scheme (oracle/tmt_oracle.c, orc_partition_*)
stands in; it is deterministic for a given thread count, so its curve is
computed once, here, and committed.  Every 10 iterations the FP64
ll_per_word (getLL / realN, TopicModel.hpp:757-760) of the state after that
iteration (after the alpha update when one is due) is recorded, for seeds
1..5.

Corpora (the seeded synthetic stand-ins of the benchmark configurations,
generated and prepared as bench.py does, identified by a SHA-1 of the
prepared ids):
  c1   V=10k, 20 true topics, D=1,000, Poisson(1500) lengths; k=20, 200 iterations
  c2   V=50k, 100 true topics, D=100,000, lognormal(ln 200, 0.8); k=100, 500 iterations
  c3s  the k=1000 configuration's generator, first 100,000 documents
       (lognormal(ln 100, 1.2)); k=1000, 50 iterations

    make -C oracle native
    TMT_ORACLE_LIB=oracle/liboracle_native.so python tests/golden/make_ll_parity.py c1:10 c1:0 c3s:10 c2:10
(arguments: run:optim_interval; results are merged into the JSON file.)
"""
import hashlib
import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))
OUT = os.path.join(HERE, "ll_partition.json")

RUNS = {
    "c1": dict(config="c1", docs=0, iters=200),
    "c2": dict(config="c2", docs=0, iters=500),
    "c3s": dict(config="c3", docs=100000, iters=50),
}
SEEDS = (1, 2, 3, 4, 5)
ALPHA, ETA = 0.1, 0.01


def corpus_of(run):
    """The prepared corpus of a parity run: (doc_off, words, realV, K, sha1)."""
    import bench
    r = RUNS[run]
    w = dict(bench.WORKLOADS[r["config"]])
    if r["docs"]:
        w["D"] = r["docs"]
    off, words, V = bench.make_corpus(w)
    h = hashlib.sha1()
    h.update(np.ascontiguousarray(off, np.uint64).tobytes())
    h.update(np.ascontiguousarray(words, np.uint32).tobytes())
    return off, words, V, w["K"], h.hexdigest()


def run_partition(run, optim):
    import oracle as O
    off, words, V, K, sha = corpus_of(run)
    iters = RUNS[run]["iters"]
    c = O.Corpus(off, words, V)
    cf = np.bincount(words[words < V], minlength=V).astype(np.uint64)
    threads = os.cpu_count() or 1
    curves = {}
    t0 = time.time()
    for seed in SEEDS:
        st = O.State(c, K, ALPHA, ETA, seed)
        p = O.Partition(st, threads, vocab_cf=cf, seed=seed)
        curve = []
        for it in range(iters):
            p.train(1)
            if optim and (it + 1) % optim == 0:
                st.optimize_alpha()       # trainOne: after the merge, (globalStep + 1) % optimInterval == 0
            if (it + 1) % 10 == 0:
                curve.append(st.ll_per_word())
        p.close()
        curves[str(seed)] = curve
        print(f"{run} optim={optim} seed={seed}: ll_per_word after {iters} = {curve[-1]:.6f} "
              f"({time.time() - t0:.0f} s)", flush=True)
    return {"config": RUNS[run]["config"], "docs": RUNS[run]["docs"] or None, "K": K, "V": int(V),
            "D": int(c.D), "N": int(c.N), "corpus_sha1": sha, "alpha": ALPHA, "eta": ETA, "iters": iters,
            "optim_interval": optim, "burn_in": 0, "ll_every": 10, "threads": threads,
            "scheme": "PARTITION (oracle restatement)", "seconds": round(time.time() - t0, 1),
            "ll_per_word": curves}


def main(args):
    data = {"about": "ll_per_word every 10 iterations of tomotopy's PARTITION train() restated in the "
                     "oracle; generated by tests/golden/make_ll_parity.py", "runs": {}}
    if os.path.exists(OUT):
        with open(OUT) as f:
            data = json.load(f)
    for a in args:
        run, optim = a.split(":")
        res = run_partition(run, int(optim))
        data["runs"][f"{run}/optim{int(optim)}"] = res
        with open(OUT + ".tmp", "w") as f:
            json.dump(data, f, indent=1)
        os.replace(OUT + ".tmp", OUT)


if __name__ == "__main__":
    main(sys.argv[1:] or ["c1:10", "c1:0", "c3s:10", "c2:10"])
