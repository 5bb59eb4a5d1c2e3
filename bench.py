"""Benchmark of the LDA collapsed-Gibbs training sweep on B200.

Default workload: LDA k=1000 over the ~204M-token synthetic corpus
(V=100,000 Zipf(1.07) words, 1,000 true topics, D=1,000,000 documents with
lognormal(ln 100, 1.2) lengths clipped to [5, 5000]); alpha=0.1, eta=0.01.
A step is one training sweep over every token (tomotopy's trainOne).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--config c1|c2|c3] [--impl ours|reference]

Prints one JSON line (rank 0).  `value` is sampled tokens/s over all ranks
with the corpus resident in HBM; `e2e` is the same metric through the C ABI
from host buffers (corpus upload, the sweeps, the log-likelihood read and the
z / n_kw download inside the timed region).  The reference arm
(--impl reference) times the CPU restatement of tomotopy's PARTITION scheme
(oracle/) with all host threads on a bounded sample of the same corpus.
"""
import argparse
import ctypes as C
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

WORKLOADS = {
    # configs of the tomotopy LDA benchmark shapes (synthetic stand-ins)
    "c1": dict(V=10000, T=20, D=1000, length=("poisson", 1500, 1, 100000), K=20, seed=20261204),
    "c2": dict(V=50000, T=100, D=100000, length=("lognormal", float(np.log(200)), 0.8, 10, 10000), K=100,
               seed=20261205),
    "c3": dict(V=100000, T=1000, D=1000000, length=("lognormal", float(np.log(100)), 1.2, 5, 5000), K=1000,
               seed=20261206),
}
ALPHA, ETA = 0.1, 0.01
METRIC = "Gibbs sampled tokens/s (LDA train sweep)"


def bytes_per_sweep(N, K, V):
    """Algorithmic bytes of one sweep, dense-conditional operand model:
    per token one K-vector of int32 counts (4K) + doc id / word id / z
    traffic (16 B); per word its n_kw column read and written (8K); the
    offsets and n_k."""
    return N * (4 * K + 16) + 8 * K * V + 4 * (V + 1) + 8 * K


# DRAM bytes of one sweep measured by ncu outside the bench (dram__bytes_read.sum +
# dram__bytes_write.sum), keyed by config: shown beside the roofline as the
# capture it came from; the bench itself measures no DRAM traffic, so its
# roofline.traffic stays null.
NCU_TRAFFIC = {"c3": {"bytes_per_sweep": 108.3e9 + 9.6e9,
                      "source": "profiles/k_sweep_doc_c3_traffic.md (100k-document capture scaled by tokens, "
                                "plus k_phi_copy)"}}


# ll-parity runs: the benchmark corpora at the configurations' iteration
# counts (the k=1000 one on its first 100,000 documents), against tomotopy's
# PARTITION train() restated in the oracle (tests/golden/ll_partition.json,
# written by tests/golden/make_ll_parity.py)
PARITY = {
    "c1": dict(config="c1", docs=0, iters=200),
    "c2": dict(config="c2", docs=0, iters=500),
    "c3s": dict(config="c3", docs=100000, iters=50),
}
PARITY_SEEDS = (1, 2, 3, 4, 5)
PARITY_FILE = os.path.join(ROOT, "tests", "golden", "ll_partition.json")


def parity_corpus(run):
    """The prepared corpus of a parity run: (doc_off, words, realV, K, sha1 of the ids)."""
    import hashlib
    r = PARITY[run]
    w = dict(WORKLOADS[r["config"]])
    if r["docs"]:
        w["D"] = r["docs"]
    off, words, V = make_corpus(w)
    h = hashlib.sha1()
    h.update(np.ascontiguousarray(off, np.uint64).tobytes())
    h.update(np.ascontiguousarray(words, np.uint32).tobytes())
    return off, words, V, w["K"], h.hexdigest()


def gpu_parity(run, optim, seeds=PARITY_SEEDS, corpus=None):
    """ll_per_word every 10 sweeps of the device sampler on a parity run's
    corpus, per seed (tomotopy's defaults: alpha 0.1, eta 0.01, burn_in 0)."""
    import tomotopy_b200 as T
    off, words, V, K, sha = corpus or parity_corpus(run)
    iters = PARITY[run]["iters"]
    curves, ms = {}, []
    for seed in seeds:
        eng = T.Engine(K, V, alpha=ALPHA, eta=ETA, seed=seed, optim_interval=optim)
        eng.upload(off, words)
        ll = eng.train(iters, ll_every=10)
        info = eng.info()
        curves[str(seed)] = (ll / info.N).tolist()
        ms.append(info.train_ms / iters)
        eng.close()
    return {"corpus_sha1": sha, "ll_per_word": curves, "ms_per_sweep": ms}


def parity_compare(ref, gpu):
    """Mean over seeds of the final ll_per_word, and the relative gap."""
    r = float(np.mean([c[-1] for c in ref["ll_per_word"].values()]))
    g = float(np.mean([c[-1] for c in gpu["ll_per_word"].values()]))
    return {"ref_mean": r, "gpu_mean": g, "rel_gap": abs(g - r) / abs(r),
            "ref_final": [c[-1] for c in ref["ll_per_word"].values()],
            "gpu_final": [c[-1] for c in gpu["ll_per_word"].values()]}


def run_parity(args):
    """One JSON line per parity run in the fixture: the device sampler's
    ll_per_word against tomotopy's PARTITION train() (oracle restatement) at
    the same iteration count, 5 seeds."""
    import torch
    torch.cuda.set_device(0)
    with open(PARITY_FILE) as f:
        ref = json.load(f)["runs"]
    corpora = {}
    for key, r in sorted(ref.items()):
        run = key.split("/")[0]
        if args.config in PARITY and run != args.config:
            continue
        if run not in corpora:
            corpora[run] = parity_corpus(run)
        g = gpu_parity(run, r["optim_interval"], corpus=corpora[run])
        cmp = parity_compare(r, g)
        print(json.dumps({"metric": "ll_per_word at the same iteration count (device vs PARTITION)", "run": key,
                          "K": r["K"], "V": r["V"], "D": r["D"], "N": r["N"], "iters": r["iters"],
                          "optim_interval": r["optim_interval"], "same_corpus": g["corpus_sha1"] == r["corpus_sha1"],
                          "ref_threads": r["threads"], "gpu_ms_per_sweep": float(np.mean(g["ms_per_sweep"])),
                          **cmp}), flush=True)


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons, sampled every 200 ms."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device=0):
        self.device = device
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax.append(float(parts[2]))
            except ValueError:
                continue
            for n, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def load_oracle(native=True):
    """The oracle (test infrastructure: the CPU baseline's restatement of
    tomotopy's PARTITION train()), built for this host at -O3 -march=native
    (bit-identical to the -O2 build: no fast-math, no FMA contraction)."""
    odir = os.path.join(ROOT, "oracle")
    if native and "oracle" not in sys.modules:
        # always rebuilt (-B): a -march=native build from another machine may
        # use instructions this host lacks
        r = subprocess.run(["make", "-s", "-B", "-C", odir, "native"], capture_output=True, text=True)
        if r.returncode == 0:
            os.environ["TMT_ORACLE_LIB"] = os.path.join(odir, "liboracle_native.so")
    sys.path.insert(0, odir)
    import oracle as O
    return O


def host_cpu():
    """CPU model and hardware threads of this host."""
    model = "unknown"
    try:
        with open("/proc/cpuinfo") as f:
            for ln in f:
                if ln.startswith("model name"):
                    model = ln.split(":", 1)[1].strip()
                    break
    except OSError:
        pass
    return {"model": model, "threads": os.cpu_count() or 1}


def tomotopy_probe():
    """tomotopy itself, when importable here (its version and tp.isa); it is
    not installable offline, so the CPU leg falls back to the oracle port."""
    try:
        import tomotopy as tp
        return {"importable": True, "version": tp.__version__, "isa": tp.isa}
    except Exception as e:
        return {"importable": False, "why": type(e).__name__ + ": " + str(e)[:80]}


def l2_statement(n_tokens, K, V):
    """Whether the inputs exceed the 126 MB L2 between timed sweeps."""
    mb_c, mb_kw = 4 * n_tokens / 1e6, 4 * K * V / 1e6
    big = mb_c + mb_kw > 126
    return (f"inputs {'larger' if big else 'smaller'} than L2 (corpus {mb_c:.0f} MB per GPU, n_kw {mb_kw:.0f} MB)"
            + ("" if big else ": the state stays in L2 across sweeps, as it does in training"))


def workload_config(cfg, w, world):
    """The workload definition both arms print as `config`: the
    configuration, its sizes and the model's hyper-parameters."""
    return {"workload": workload_name(cfg, w), "K": w["K"], "V": w["V"], "D": w["D"] * world,
            "alpha": ALPHA, "eta": ETA, "true_topics": w["T"], "length": list(w["length"]),
            "generator_seed": w["seed"],
            "parallelism": (f"dp{world}: documents sharded, n_kw deltas summed over NCCL per group"
                            if world > 1 else "dp1")}


def oracle_corpus(w):
    """The workload's prepared corpus built by the oracle (no engine code)."""
    O = load_oracle()
    off, words = O.synth_corpus(w["V"], w["T"], w["D"], w["length"], seed=w["seed"])
    off, words, realV, _ = O.prepare_ids(off, words)
    return off, words, realV


def make_corpus(w, threads=0):
    import tomotopy_b200 as T
    off, words = T.synth_corpus(w["V"], w["T"], w["D"], w["length"], seed=w["seed"], threads=threads)
    off, words, realV, _ = T.prepare_ids(off, words)
    return off, words, realV


def idf_weights(off, words, V):
    """TermWeight IDF per token (LDAModel.hpp:1093-1122): (float)log(D / df(w)),
    df counted over documents; the prepared corpus holds each document's
    words sorted, so a document's distinct words start its runs."""
    D = len(off) - 1
    o = off.astype(np.int64)
    first = np.ones(len(words), bool)
    first[1:] = words[1:] != words[:-1]
    first[o[:-1][np.diff(o) > 0]] = True
    ok = words < V
    df = np.bincount(words[first & ok], minlength=V)[:V]
    idf = np.log(D / np.maximum(df, 1).astype(np.float64)).astype(np.float32)
    return np.where(ok, idf[np.minimum(words, V - 1)], np.float32(0)).astype(np.float32)


def make_shard(w, rank, world):
    """Rank r's part of one corpus split across ranks: the documents
    [r*D, (r+1)*D) of the seeded generator, prepared with the vocabulary order
    of the whole corpus (the ranks' (cf, df) summed), and every rank's
    document lengths."""
    import torch
    import torch.distributed as dist
    import tomotopy_b200 as T
    from tomotopy_b200 import shard as S
    off, words = T.synth_corpus(w["V"], w["T"], w["D"], w["length"], seed=w["seed"], doc_offset=rank * w["D"])

    def sum_counts(cf, df):
        t = torch.from_numpy(np.concatenate([cf, df]).astype(np.int64)).cuda()
        dist.all_reduce(t)
        a = t.cpu().numpy().astype(np.uint64)
        cf[:] = a[:len(cf)]
        df[:] = a[len(cf):]

    off, words, V, _ = S.prepare_ids(off, words, w["V"], sum_counts)
    lens = torch.from_numpy(np.diff(off.astype(np.int64))).cuda()
    allg = torch.empty(world * len(lens), dtype=torch.int64, device="cuda")
    dist.all_gather_into_tensor(allg, lens)
    return off, words, V, allg.cpu().numpy().astype(np.uint64)


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


# tokens of the CPU arm's sample per sweep, by K: about a second of PARTITION
# work per sweep on a host of a few dozen cores
REF_SAMPLE_TOKENS = {20: 1_500_000, 100: 8_000_000, 1000: 3_000_000}


def run_reference(args, w):
    """The reference arm: tomotopy's train() -- ParallelScheme::PARTITION on
    every host thread (TopicModel.hpp:684-755, LDAModel.hpp:356-489) -- on the
    host cores.  tomotopy cannot be built offline (its CMake fetches Eigen and
    EigenRand), so the oracle's C restatement of PARTITION stands in, compiled
    here at -O3 -march=native.  The corpus is the workload's, generated and
    prepared by the oracle (no engine code is loaded); each step is one
    PARTITION sweep over a bounded sample -- the workload's first documents --
    so the run ends within minutes.  Rank 0 only."""
    rank, world, _ = dist_env()
    if rank != 0:
        return
    probe = tomotopy_probe()
    O = load_oracle()
    off, words, V = oracle_corpus(w)
    cores = os.cpu_count() or 1
    target = REF_SAMPLE_TOKENS.get(w["K"], 2_000_000)
    D = int(np.searchsorted(off.astype(np.int64), target))
    D = max(1, min(D, len(off) - 1))
    soff = off[:D + 1].copy()
    swords = words[:int(soff[-1])].copy()
    c = O.Corpus(soff, swords, V)
    st = O.State(c, w["K"], ALPHA, ETA, seed=1)
    cf = np.bincount(swords[swords < V], minlength=V).astype(np.uint64)
    part = O.Partition(st, cores, vocab_cf=cf, seed=1)
    for _ in range(args.warmup):
        part.train(1)
    times = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        part.train(1)
        times.append(time.perf_counter() - t0)
    part.close()
    t = float(np.sum(times))
    value = c.N * args.steps / t
    native = os.environ.get("TMT_ORACLE_LIB", "").endswith("liboracle_native.so")
    sample = (f"the workload's first {D} documents ({c.N} tokens of {len(words)}), one PARTITION sweep per "
              f"step, {cores} host threads")
    line = {
        "metric": METRIC, "value": value, "unit": "tokens/s", "n_gpus": args.gpus, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1000 * t / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded LDA generative process)",
        "impl": "reference",
        "config": dict(workload_config(args.config, w, world), l2=l2_statement(len(words), w["K"], w["V"])),
        "corpus": {"realV": int(V), "tokens_all_ids": int(len(words)), "built_by": "oracle (synth + prepare restated)"},
        "sample": {"docs": D, "tokens": int(c.N)},
        "ll_per_word": st.ll_per_word(),
        "ll_after_sweeps": args.warmup + args.steps,
        "cpu_baseline": {"value": value, "unit": "tokens/s", "cores": cores, "kind": "port", "sample": sample,
                         "cpu": host_cpu(),
                         "build": ("gcc -O3 -march=native -ffp-contract=off" if native
                                   else "gcc -O2 -ffp-contract=off (native build failed)"),
                         "tomotopy": probe},
        "e2e": {"value": value, "unit": "tokens/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def workload_name(cfg, w):
    return (f"LDA k={w['K']} V={w['V']} D={w['D']} ({cfg}: synthetic LDA corpus, {w['T']} true topics, "
            f"Zipf(1.07), lengths {w['length'][0]})")


def cpu_baseline_sample(w, off, words, V, seconds=10.0):
    """The oracle's PARTITION port on the host (-O3 -march=native), bounded to ~`seconds`."""
    O = load_oracle()
    cores = os.cpu_count() or 1
    target = {20: 3_000_000, 100: 1_000_000, 1000: 300_000}.get(w["K"], 500_000)
    D = int(np.searchsorted(off.astype(np.int64), target))
    D = max(1, min(D, len(off) - 1))
    soff = off[:D + 1].copy()
    swords = words[:int(soff[-1])].copy()
    c = O.Corpus(soff, swords, V)
    st = O.State(c, w["K"], ALPHA, ETA, seed=1)
    cf = np.bincount(swords[swords < V], minlength=V).astype(np.uint64)
    part = O.Partition(st, cores, vocab_cf=cf, seed=1)
    part.train(1)
    n, t = 0, 0.0
    while t < seconds and n < 20:
        t0 = time.perf_counter()
        part.train(1)
        t += time.perf_counter() - t0
        n += 1
    part.close()
    return {"value": c.N * n / t, "unit": "tokens/s", "cores": cores, "kind": "port",
            "sample": f"first {D} docs ({c.N} tokens), {n} PARTITION sweeps on {cores} host threads",
            "cpu": host_cpu(), "tomotopy": tomotopy_probe()}


INFER = {
    # served infer(), single model: k=100 trained on config 1's corpus; requests lognormal(ln 150, 1.0)
    "c4": dict(models=[dict(K=100, V=10000, T=20, D=1000, length=("poisson", 1500, 1, 100000),
                            seed=20261204, sweeps=200)],
               mix=[1.0], length=("lognormal", float(np.log(150)), 1.0, 10, 5000), iters=50,
               rates=[1000, 5000, 20000, 50000, 100000]),
    # served infer(), three resident models, traffic 60/30/10, 100 sweeps each
    "c5": dict(models=[dict(K=50, V=20000, T=50, D=40000, length=("lognormal", float(np.log(100)), 1.2, 5, 10000),
                            seed=20261207, sweeps=50),
                       dict(K=200, V=50000, T=200, D=40000, length=("lognormal", float(np.log(100)), 1.2, 5, 10000),
                            seed=20261208, sweeps=50),
                       dict(K=1000, V=100000, T=1000, D=40000, length=("lognormal", float(np.log(100)), 1.2, 5, 10000),
                            seed=20261209, sweeps=50)],
               mix=[0.6, 0.3, 0.1], length=("lognormal", float(np.log(100)), 1.2, 5, 10000), iters=100,
               rates=[1000, 5000, 20000, 50000]),
}


def infer_requests(mc, order, n, length, seed_off):
    """n unseen documents from the model's generative process; words outside
    the model's dictionary are dropped, as tomotopy's makeDoc does."""
    import tomotopy_b200 as T
    off, w = T.synth_corpus(mc["V"], mc["T"], n, length, seed=mc["seed"], doc_offset=10_000_000 + seed_off)
    docs = []
    for d in range(n):
        ids = w[off[d]:off[d + 1]]
        ids = ids[ids < len(order)]
        docs.append(order[ids].astype(np.uint32))
    return docs


def run_infer(args):
    import threading as th
    import torch
    import tomotopy_b200 as T
    cfg = INFER[args.config]
    torch.cuda.set_device(0)
    engines, orders = [], []
    for mc in cfg["models"]:
        off, w = T.synth_corpus(mc["V"], mc["T"], mc["D"], mc["length"], seed=mc["seed"])
        off, w, V, order = T.prepare_ids(off, w)
        eng = T.Engine(mc["K"], V, alpha=ALPHA, eta=ETA, seed=1, optim_interval=0)
        eng.upload(off, w)
        eng.train(mc["sweeps"])
        engines.append(eng)
        orders.append(order)
    rng = np.random.default_rng(7)
    n_req = args.requests
    which = rng.choice(len(engines), size=n_req, p=cfg["mix"])
    docs = [None] * n_req
    for m in range(len(engines)):
        idx = np.nonzero(which == m)[0]
        ds = infer_requests(cfg["models"][m], orders[m], len(idx), cfg["length"], seed_off=m * 1_000_000)
        for i, d in zip(idx, ds):
            docs[i] = d
    iters = cfg["iters"]
    ntok = sum(len(d) for d in docs)

    # plain per-document GPU infer: one tmt_infer_batch call per document
    n_plain = min(200, n_req)
    t0 = time.perf_counter()
    plain_ll = []
    for i in range(n_plain):
        d = docs[i]
        th_, ll_ = engines[which[i]].infer(np.array([0, len(d)], np.uint64), d, iters=iters, seed=0)
        plain_ll.append(ll_[0])
    plain_dps = n_plain / (time.perf_counter() - t0)

    # one tmt_infer_batch call per model over all of its requests: the kernel alone
    t0 = time.perf_counter()
    for m, e in enumerate(engines):
        idx = np.nonzero(which == m)[0]
        if not len(idx):
            continue
        lens = np.array([len(docs[i]) for i in idx], np.uint64)
        boff = np.concatenate([[0], np.cumsum(lens)]).astype(np.uint64)
        bw = np.concatenate([docs[i] for i in idx]).astype(np.uint32)
        e.infer(boff, bw, iters=iters, seed=0)
    batched_dps = n_req / (time.perf_counter() - t0)

    srv = T.Server(max_slots=args.slots, token_budget=1 << 25, step_token_sweeps=args.step_tokens,
                   max_doc_len=1 << 16)
    mids = [srv.add_engine_model(e) for e in engines]

    # request i as one CSR batch, so that a run submits any range of it in one call
    all_off = np.concatenate([[0], np.cumsum([len(d) for d in docs])]).astype(np.uint64)
    all_w = np.concatenate(docs).astype(np.uint32)
    all_mid = np.array([mids[m] for m in which], np.uint32)

    def submit_range(a, b):
        off = all_off[a:b + 1] - all_off[a]
        return srv.submit_batch(all_mid[a:b], off, all_w[int(all_off[a]):int(all_off[b])], iters=iters, seed=0)

    def serve(rate):
        n = n_req if rate is None else int(min(n_req, max(200, 2.0 * rate)))
        lat, got = [], {}
        done = th.Event()

        def collect():
            while len(got) < n:
                r = srv.poll_batch(max_n=8192, wait_ms=500)
                if r is None:
                    if done.is_set():
                        break
                    continue
                rid, mid, _, ll, la = r
                for j in range(len(rid)):
                    got[int(rid[j])] = (int(rid[j]), int(mid[j]), None, float(ll[j]), float(la[j]))
                lat.extend(la.tolist())
        c = th.Thread(target=collect, daemon=True)
        c.start()
        ids = {}
        t0 = time.perf_counter()
        if rate is None:
            for a in range(0, n, 4096):
                b = min(n, a + 4096)
                for i, r in zip(range(a, b), submit_range(a, b)):
                    ids[int(r)] = i
        else:
            gaps = np.random.default_rng(11).exponential(1.0 / rate, n)
            arrive = np.cumsum(gaps)
            i = 0
            while i < n:
                now = time.perf_counter() - t0
                b = int(np.searchsorted(arrive, now, side="right"))
                if b > i:
                    for q, r in zip(range(i, b), submit_range(i, b)):
                        ids[int(r)] = q
                    i = b
                if i < n:
                    time.sleep(max(0.0, min(arrive[i] - (time.perf_counter() - t0), 0.002)))
        c.join(timeout=600)
        wall = time.perf_counter() - t0
        done.set()
        c.join(timeout=5)
        lat_a = np.array(lat)
        return {"offered_docs_per_s": rate, "docs_per_s": len(got) / wall, "p50_ms": float(np.percentile(lat_a, 50)),
                "p99_ms": float(np.percentile(lat_a, 99)), "completed": len(got)}, got, ids

    st0 = srv.stats()
    sat, got, ids = serve(None)
    st1 = srv.stats()
    # same results as plain per-document infer (same seeds, keys 0)
    served_ll = {ids[k]: v[3] for k, v in got.items()}
    agree = all(served_ll[i] == plain_ll[i] for i in range(n_plain))
    sweeps = [serve(r)[0] for r in cfg["rates"]]
    st = srv.stats()
    srv.close()
    tok_per_doc = ntok / n_req
    line = {
        "metric": f"served infer docs/s ({args.config})", "value": sat["docs_per_s"], "unit": "docs/s",
        "n_gpus": 1, "higher_is_better": True, "dtype": "f32", "data": "synthetic (seeded LDA generative process)",
        "config": {"workload": f"{args.config}: " + ", ".join(f"k={m['K']} V={m['V']}" for m in cfg["models"]) +
                   f"; mix {cfg['mix']}; {iters} sweeps per document; {n_req} requests, {tok_per_doc:.1f} tokens/doc",
                   "slots": args.slots, "step_token_sweeps": args.step_tokens},
        "saturation": sat, "rate_sweep": sweeps,
        "plain_per_document_docs_per_s": plain_dps, "speedup_vs_plain": sat["docs_per_s"] / plain_dps,
        "token_sweeps_per_s": sat["docs_per_s"] * tok_per_doc * iters,
        "results_identical_to_plain": bool(agree),
        "mean_ll_per_word_plain": float(np.sum(plain_ll) / max(1, sum(len(docs[i]) for i in range(n_plain)))),
        "server": {"steps": int(st.steps), "mean_active": st.mean_active,
                   "saturation_steps": int(st1.steps - st0.steps),
                   "saturation_mean_active": ((st1.mean_active * st1.steps - st0.mean_active * st0.steps)
                                              / max(1, st1.steps - st0.steps))},
        "batched_docs_per_s": batched_dps,
    }
    # the saturation run: device time of the inference launches against the
    # per-draw bytes (the frozen n_kw column, 4K, plus z, 8 B per token-sweep)
    k_ms = st1.kernel_ms - st0.kernel_ms
    alg = st1.alg_bytes - st0.alg_bytes
    peak, peak_kind = peaks()
    if k_ms > 0:
        achieved = alg / (k_ms / 1000.0) / 1e9
        line["roofline"] = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                            "frac": achieved / peak, "traffic": None, "kernel": "k_infer_slots",
                            "kernel_ms": k_ms, "alg_bytes": alg, "peak_source": peak_kind,
                            "step_busy_ms": st1.busy_ms - st0.busy_ms, "steps": int(st1.steps - st0.steps),
                            "token_sweeps": int(st1.token_sweeps - st0.token_sweeps)}
    if not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_infer_baseline(engines, which, docs, iters)
    print(json.dumps(line), flush=True)


def cpu_infer_baseline(engines, which, docs, iters, seconds=10.0):
    """tomotopy's per-document infer (LDAModel.hpp:920-953) restated in the
    oracle, one document per host thread."""
    from concurrent.futures import ThreadPoolExecutor
    O = load_oracle()
    models = []
    for e in engines:
        _, nkw, nk, alpha = e.state()
        models.append((e.K, e.V, alpha, e.eta, nkw, nk))
    cores = os.cpu_count() or 1
    n = 0
    t0 = time.perf_counter()

    def one(i):
        K, V, alpha, eta, nkw, nk = models[which[i]]
        O.infer_doc(K, V, alpha, eta, nkw, nk, np.sort(docs[i]), iters, 0, 0)

    with ThreadPoolExecutor(cores) as ex:
        while time.perf_counter() - t0 < seconds and n < len(docs):
            batch = list(range(n, min(len(docs), n + 4 * cores)))
            list(ex.map(one, batch))
            n += len(batch)
    t = time.perf_counter() - t0
    return {"value": n / t, "unit": "docs/s", "cores": cores, "kind": "port",
            "sample": f"{n} request documents, per-document infer on {cores} host threads"}


def run_prepare(args, w):
    """Corpus preparation (tomotopy's removeStopwords + prepareDoc) of the
    workload's raw ids: tmt_prepare_corpus_device against the host
    tmt_prepare_corpus on all host threads, host buffers in and out, outputs
    compared bit for bit.  One JSON line (tokens/s of the device path)."""
    import torch
    import tomotopy_b200 as T
    from tomotopy_b200._lib import lib
    torch.cuda.set_device(0)
    off, words = T.synth_corpus(w["V"], w["T"], w["D"], w["length"], seed=w["seed"], threads=os.cpu_count())
    nv = int(words.max()) + 1
    D, N = len(off) - 1, len(words)

    def p(a):
        return a.ctypes.data_as(C.c_void_p)

    def once(device):
        out = np.zeros(N, np.uint32)
        wo = np.zeros(N, np.uint32)
        order = np.zeros(nv, np.uint32)
        cf = np.zeros(nv, np.uint64)
        df = np.zeros(nv, np.uint64)
        rv = C.c_uint32()
        t0 = time.perf_counter()
        if device:
            err = C.create_string_buffer(512)
            st = lib.tmt_prepare_corpus_device(0, D, p(off), p(words), nv, 0, 0, 0, p(out), p(wo), p(order), p(cf),
                                               p(df), C.byref(rv), err, len(err))
        else:
            st = lib.tmt_prepare_corpus(D, p(off), p(words), nv, 0, 0, 0, p(out), p(wo), p(order), p(cf), p(df),
                                        C.byref(rv))
        dt = time.perf_counter() - t0
        if st != 0:
            raise RuntimeError("preparation failed: %d" % st)
        return dt, (out, wo, order, cf, df, rv.value)

    for _ in range(args.warmup):
        once(True)
    td = min(once(True)[0] for _ in range(max(args.steps, 1)))
    th = min(once(False)[0] for _ in range(2))
    a, b = once(True)[1], once(False)[1]
    same = all(np.array_equal(x, y) for x, y in zip(a[:5], b[:5])) and a[5] == b[5]
    print(json.dumps({
        "metric": "corpus preparation tokens/s (vocab reorder + per-document sort)", "value": N / td,
        "unit": "tokens/s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "ms_per_step": td * 1e3,
        "higher_is_better": True, "dtype": "u32", "data": "synthetic (seeded LDA generative process)",
        "config": {"workload": args.config, "D": D, "tokens": N, "n_vocab": nv,
                   "timing": "wall clock around one call, host buffers in and out, best of the timed calls"},
        "host": {"value": N / th, "ms": th * 1e3, "threads": os.cpu_count(), "kind": "tmt_prepare_corpus"},
        "identical": bool(same)}), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--config", default="c3", choices=sorted(set(WORKLOADS) | set(INFER) | set(PARITY)))
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true", help="skip the end-to-end C-ABI pass")
    ap.add_argument("--docs", type=int, default=0, help="override the document count (smaller case)")
    ap.add_argument("--groups", type=int, default=0, help="document groups per sweep (0: engine default)")
    ap.add_argument("--split", type=int, default=0,
                    help="train mode: split documents of at least this many tokens (0: the engine's rule)")
    ap.add_argument("--split-step", type=int, default=0, help="train mode: positions per slice between merges")
    ap.add_argument("--mode", default="train", choices=["train", "infer", "prepare", "parity"])
    ap.add_argument("--tw", default="one", choices=["one", "idf"],
                    help="train mode: term weighting of the corpus (idf: weighted counts, one GPU)")
    ap.add_argument("--requests", type=int, default=20000, help="infer mode: documents per run")
    ap.add_argument("--slots", type=int, default=8192, help="infer mode: server slots per model")
    ap.add_argument("--step-tokens", type=int, default=4096, help="infer mode: token-sweeps per document per step")
    args = ap.parse_args()
    if args.mode == "infer":
        if args.config not in INFER:
            args.config = "c4"
        return run_infer(args)
    if args.mode == "parity":
        return run_parity(args)
    args.warmup = max(args.warmup, 3)
    w = dict(WORKLOADS[args.config])
    if args.docs:
        w["D"] = args.docs
    if args.mode == "prepare":
        return run_prepare(args, w)
    if args.impl == "reference":
        return run_reference(args, w)

    rank, world, local = dist_env()
    import torch
    torch.cuda.set_device(local)
    if world > 1:
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=600))
    import tomotopy_b200 as T

    K = w["K"]
    if world > 1:
        # one corpus split across the ranks (weak scaling: every rank holds a
        # full-size share); one chain, n_kw deltas summed per group over NCCL
        from tomotopy_b200 import shard as S
        off, words, V, lens_global = make_shard(w, rank, world)

        def new_engine():
            return S.ShardedEngine(K, V, alpha=ALPHA, eta=ETA, seed=1, optim_interval=0, device=local,
                                   sweep_groups=args.groups)

        def upload(e, o, ws):
            e.upload_shard(o, ws, lens_global, rank * w["D"], rank, world)
    else:
        off, words, V = make_corpus(w)
    wts = None
    if args.tw != "one":
        if world > 1:
            raise SystemExit("--tw idf runs on one GPU (weighted counts are not sharded)")
        wts = idf_weights(off, words, V)
    if world == 1:

        def new_engine():
            return T.Engine(K, V, alpha=ALPHA, eta=ETA, seed=1, optim_interval=0, device=local,
                            sweep_groups=args.groups)

        def upload(e, o, ws, wt=None):
            e.upload(o, ws, weights=wt)

    def total(x, op="sum"):
        t = torch.tensor([float(x)], dtype=torch.float64, device="cuda")
        if world > 1:
            torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX if op == "max"
                                         else torch.distributed.ReduceOp.SUM)
        return float(t.item())

    def configure(e):
        if args.split or args.split_step:
            e.set_doc_split(args.split, args.split_step)

    eng = new_engine()
    configure(eng)
    if wts is not None:
        upload(eng, off, words, wts)
    else:
        upload(eng, off, words)
    info0 = eng.info()
    N = info0.N
    N_all_ranks = int(total(N))
    # the engine's autotuner: the first sweeps after an upload time each
    # sweep-kernel variant per document group (identical results); they run
    # here, before the warm-up, and are reported as tuning_sweeps
    tuning = 0
    while -1 in eng.sweep_variants():
        eng.train(1)
        tuning += 1
    eng.train(args.warmup)
    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    clocks = ClockSampler(local)
    clocks.start()
    launches0 = eng.info().kernel_launches
    t0 = time.perf_counter()
    eng.train(args.steps)
    wall = time.perf_counter() - t0
    info = eng.info()
    variants = eng.sweep_variants()
    tuning_ms = [[round(float(x), 3) for x in row] for row in eng.sweep_timings()]
    split = eng.doc_split()
    launches = info.kernel_launches - launches0
    clk = clocks.stop()
    kernel_ms = info.sweep_kernel_ms / max(info.sweeps_timed, 1)
    # device time of the K sweeps (CUDA events on the engine's stream around the
    # whole train call), the max over ranks
    step_ms = total(info.train_ms / args.steps, "max")
    wall_ms = total(wall * 1000 / args.steps, "max")
    value = N_all_ranks * 1000.0 / step_ms
    ll = eng.ll()
    ll_sweeps = tuning + args.warmup + args.steps

    # e2e through the C ABI from the caller's pageable numpy arrays (tomotopy's
    # own buffers are pageable std::vectors): engine creation, corpus upload
    # (staged through pinned buffers), z0 and counts, the autotuner's sweeps and
    # the K sweeps of one train() call, the log-likelihood, and the z / n_kw /
    # n_k download into fresh pageable arrays
    if args.no_e2e:
        e2e_obj = None
    else:
        eng.close()
        e_words = np.ascontiguousarray(words).copy()
        e_off = np.ascontiguousarray(off).copy()
        e_wts = np.ascontiguousarray(wts).copy() if wts is not None else None
        if world > 1:
            torch.distributed.barrier()
        torch.cuda.synchronize()
        te0 = time.perf_counter()
        e2e = new_engine()
        configure(e2e)
        if e_wts is not None:
            upload(e2e, e_off, e_words, e_wts)
        else:
            upload(e2e, e_off, e_words)
        e2e.train(args.steps)
        e2e.ll()
        z, nkw, nk, _ = e2e.state()
        te = total(time.perf_counter() - te0, "max")
        h2d = e_words.nbytes + e_off.nbytes + (e_wts.nbytes if e_wts is not None else 0)
        d2h = z.nbytes + nkw.nbytes + nk.nbytes + 16
        e2e_obj = {"value": N_all_ranks * args.steps / te, "unit": "tokens/s",
                   "h2d_bytes_per_step": h2d / args.steps, "d2h_bytes_per_step": d2h / args.steps,
                   "includes": "engine creation, corpus upload from pageable arrays (staged), z0 init + counts, "
                               "one train() call of K sweeps (its first sweeps tune the kernel variants), ll, "
                               "z/n_kw/n_k download into fresh pageable arrays"}
        e2e.close()
        eng = None

    peak, peak_kind = peaks()
    alg = bytes_per_sweep(N, K, V)
    achieved = alg / (kernel_ms / 1000.0) / 1e9
    if rank == 0:
        cfgd = workload_config(args.config, w, world)
        cfgd["l2"] = l2_statement(len(words), K, w["V"])
        line = {
            "metric": METRIC, "value": value, "unit": "tokens/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": step_ms, "wall_ms_per_step": wall_ms,
            "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded LDA generative process)",
            "config": cfgd,
            "corpus": {"realV": int(V), "tokens": N_all_ranks, "tokens_all_ids": int(len(words)) * world},
            "engine": {"sweep_groups": int(info.sweep_groups), "sweep_variants": variants,
                       "tuning_ms": tuning_ms, "split_docs_per_group": split, "tuning_sweeps": tuning, "term_weight": args.tw,
                       "optim_interval": 0},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": None,
                         "kernel": "k_sweep_doc", "kernel_ms": kernel_ms, "alg_bytes_per_launch": alg,
                         "per": "one sweep = all k_sweep_doc + k_phi_copy launches of the document groups",
                         "traffic_ncu": NCU_TRAFFIC.get(args.config) if args.tw == "one" else None,
                         "peak_source": peak_kind},
            "e2e": e2e_obj,
            "gpu_launches": int(launches),
            "clocks": clk,
            "ll_per_word": (ll[0] + ll[1]) / N_all_ranks if N_all_ranks else 0.0,
            "ll_after_sweeps": ll_sweeps,
        }
        if not args.no_cpu_baseline and world == 1 and args.tw == "one":
            line["cpu_baseline"] = cpu_baseline_sample(w, off, words, V)
        print(json.dumps(line), flush=True)
    if eng is not None:
        eng.close()
    if world > 1:
        torch.distributed.barrier()
        torch.distributed.destroy_process_group()


if __name__ == "__main__":
    main()
