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


def make_corpus(w, threads=0):
    import tomotopy_b200 as T
    off, words = T.synth_corpus(w["V"], w["T"], w["D"], w["length"], seed=w["seed"], threads=threads)
    off, words, realV, _ = T.prepare_ids(off, words)
    return off, words, realV


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


def run_reference(args, w):
    """tomotopy's PARTITION scheme restated on the host (oracle), all threads,
    on a bounded sample of the workload's documents."""
    rank, world, _ = dist_env()
    if rank != 0:
        return
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    off, words, V = make_corpus(w)
    cores = os.cpu_count() or 1
    # bounded sample: a prefix of the documents, ~tokens so one sweep is ~1 s of host work
    target = {20: 6_000_000, 100: 2_000_000, 1000: 600_000}.get(w["K"], 1_000_000)
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
    line = {
        "metric": METRIC, "value": value, "unit": "tokens/s", "n_gpus": args.gpus, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1000 * t / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "impl": "reference",
        "config": {"workload": workload_name(args.config, w), "K": w["K"], "docs_sampled": D,
                   "tokens_sampled": c.N},
        "cpu_baseline": {"value": value, "unit": "tokens/s", "cores": cores, "kind": "port",
                         "sample": f"first {D} docs ({c.N} tokens) of the workload, PARTITION scheme, "
                                   f"{cores} host threads, one sweep per step"},
        "e2e": {"value": value, "unit": "tokens/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def workload_name(cfg, w):
    return (f"LDA k={w['K']} V={w['V']} D={w['D']} ({cfg}: synthetic LDA corpus, {w['T']} true topics, "
            f"Zipf(1.07), lengths {w['length'][0]})")


def cpu_baseline_sample(w, off, words, V, seconds=10.0):
    """The oracle's PARTITION port on the host, bounded to ~`seconds`."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
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
            "sample": f"first {D} docs ({c.N} tokens), {n} PARTITION sweeps on {cores} host threads"}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--config", default="c3", choices=sorted(WORKLOADS))
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true", help="skip the end-to-end C-ABI pass")
    ap.add_argument("--docs", type=int, default=0, help="override the document count (smaller case)")
    ap.add_argument("--groups", type=int, default=0, help="document groups per sweep (0: engine default)")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    w = dict(WORKLOADS[args.config])
    if args.docs:
        w["D"] = args.docs
    if args.impl == "reference":
        return run_reference(args, w)

    rank, world, local = dist_env()
    import torch
    torch.cuda.set_device(local)
    if world > 1:
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=600))
    import tomotopy_b200 as T

    off, words, V = make_corpus(w)
    K = w["K"]
    # documents sharded across ranks (weak scaling: every rank holds a full-size corpus
    # of its own documents; ranks are independent chains)
    eng = T.Engine(K, V, alpha=ALPHA, eta=ETA, seed=1 + rank, optim_interval=0, device=local,
                   sweep_groups=args.groups)
    eng.upload(off, words)
    info0 = eng.info()
    N = info0.N
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
    launches = info.kernel_launches - launches0
    clk = clocks.stop()
    kernel_ms = info.sweep_kernel_ms / max(info.sweeps_timed, 1)
    # device time of the K sweeps: sum of per-sweep events (kernel + the n_kw copy)
    step_ms = wall * 1000 / args.steps
    t_dev = torch.tensor([step_ms], dtype=torch.float64, device="cuda")
    if world > 1:
        torch.distributed.all_reduce(t_dev, op=torch.distributed.ReduceOp.MAX)
    step_ms = float(t_dev.item())
    value = N * world * 1000.0 / step_ms

    # e2e through the C ABI from host buffers: upload + steps + ll + download
    if args.no_e2e:
        ll = eng.ll()
        e2e_obj = None
    else:
        eng.close()
        pin_words = torch.from_numpy(words).pin_memory().numpy()
        pin_off = torch.from_numpy(off).pin_memory().numpy()
        e2e = T.Engine(K, V, alpha=ALPHA, eta=ETA, seed=1 + rank, optim_interval=0, device=local,
                       sweep_groups=args.groups)
        torch.cuda.synchronize()
        te0 = time.perf_counter()
        e2e.upload(pin_off, pin_words)
        e2e.train(args.steps)
        ll = e2e.ll()
        z, nkw, nk, _ = e2e.state()
        te = time.perf_counter() - te0
        h2d = pin_words.nbytes + pin_off.nbytes
        d2h = z.nbytes + nkw.nbytes + nk.nbytes + 16
        e2e_obj = {"value": N * world * args.steps / te, "unit": "tokens/s", "h2d_bytes_per_step": h2d / args.steps,
                   "d2h_bytes_per_step": d2h / args.steps,
                   "includes": "corpus upload (pinned), z0 init + counts, the sweeps, ll, z/n_kw/n_k download"}
        e2e.close()

    peak, peak_kind = peaks()
    alg = bytes_per_sweep(N, K, V)
    achieved = alg / (kernel_ms / 1000.0) / 1e9
    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "tokens/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": step_ms, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded LDA generative process)",
            "config": {"workload": workload_name(args.config, w), "K": K, "V": V, "D": int(len(off) - 1),
                       "tokens": int(N), "alpha": ALPHA, "eta": ETA, "sweep_groups": int(info.sweep_groups), "parallelism": f"dp{world} (independent chains)",
                       "l2": "inputs larger than L2 (corpus %.0f MB, n_kw %.0f MB)" % (words.nbytes / 1e6, 4 * K * V / 1e6)},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": None,
                         "kernel": "k_sweep_doc", "kernel_ms": kernel_ms, "alg_bytes_per_launch": alg,
                         "peak_source": peak_kind},
            "e2e": e2e_obj,
            "gpu_launches": int(launches),
            "clocks": clk,
            "ll_per_word": (ll[0] + ll[1]) / N if N else 0.0,
        }
        if not args.no_cpu_baseline:
            line["cpu_baseline"] = cpu_baseline_sample(w, off, words, V)
        print(json.dumps(line), flush=True)
    eng.close()
    if world > 1:
        torch.distributed.barrier()
        torch.distributed.destroy_process_group()


if __name__ == "__main__":
    main()
