#!/usr/bin/env python
"""bench.py -- throughput of the GPU multi-vector search path on B200.

One step = one search pass over the workload's query set (10,000 queries x 32
tokens for the default "medium" workload: 1M synthetic docs / ~70M tokens,
65,536 centroids, nbits 2, nprobe 8, k 10).  The index is built on the GPU
from the seeded synthetic corpus before anything is timed.

  value : queries/s with queries resident in HBM (mvr_search_device), device
          time by CUDA events on the launching stream, L2 flushed between
          steps, max over ranks
  e2e   : queries/s through mvr_search with pinned HOST query/result buffers
          (copies inside the timed region), wall clock around each call
  roofline : the dominant stage's algorithmic work / its CUDA-event time
  cpu_baseline : the oracle's multi-threaded CPU port of the same path on a
          bounded query sample (rank 0, N=1)

--impl reference times that CPU port alone (all host threads) as the
reference arm.  N>1 (torchrun): each rank serves its own query set against its
own replica of the index (weak scaling, no data-path collective).
"""
import argparse
import hashlib
import json
import math
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "multi-vector-retrieval-gpu_b200"))

METRIC = ("QPS & p99 ms at recall@10>=0.99 vs exact MaxSim: learned+BF16/FP8 vs plain, "
          "1 B200")
CACHE_VERSION = "mvr-index-v1"
# ncu: dram__bytes_read + dram__bytes_write of the FP8 MaxSim kernel
# (rerank_ws_kernel) per reranked token on the 200,000-doc profiling case
# (--profile-case, 20,842,514 reranked tokens), by nbits: 695.07 MB at
# nbits 2, 1365.26 MB at nbits 4
RERANK_DRAM_BYTES_PER_TOKEN = {2: 33.35, 4: 65.50}

WORKLOADS = {
    # medium: 1M docs, 65,536 centroids, nbits 2, 10,000 queries (the headline workload)
    # probe_topk: the shortlist tuner's pick for recall@10 >= 0.99 against
    # exhaustive MaxSim over the index's decoded vectors (300 tuning queries)
    "medium": dict(n_doc=1_000_000, n_centroid=65536, n_bit=2, n_query=10_000, n_tok=32,
                   nprobe=8, topk=10, probe_topk=1500, kmeans_iter=4, seed=0, n_gt=100,
                   n_tune=300),
    # small: 10k docs, 8,192 centroids, nbits 2, 1,000 queries (CPU-runnable scale)
    # heavy: 4-bit codes, docs up to 300 tokens, queries of 32 or 64 tokens
    # (the corpus of the 1M-doc workload's size)
    "heavy": dict(n_doc=1_000_000, n_centroid=65536, n_bit=4, n_query=10_000, n_tok=[32, 64],
                  nprobe=8, topk=10, probe_topk=1500, kmeans_iter=4, seed=0, n_gt=100,
                  n_tune=300, len_hi=300),
    "small": dict(n_doc=10_000, n_centroid=8192, n_bit=2, n_query=1000, n_tok=32, nprobe=4,
                  topk=10, probe_topk=200, kmeans_iter=8, seed=0, n_gt=200, n_tune=300),
    # corpora larger than the device holds as raw tokens, built by streaming
    # (block-keyed generator, tensor-core assignment) and scanned piecewise for
    # the ground truths; probe_topk: starting point, the tuner reports its pick
    # large: 4M docs, 262,144 centroids, nbits 2, ragged 8..32-token queries in
    # batches of 4,096
    "large": dict(n_doc=4_000_000, n_centroid=262_144, n_bit=2, n_query=16_384, n_tok=(8, 32),
                  nprobe=8, topk=10, probe_topk=1500, kmeans_iter=4, seed=0, n_gt=100,
                  n_tune=200, stream=True, batch=4096),
    # xl: 8M docs up to 300 tokens, 262,144 centroids, nbits 4, 32- or 64-token
    # queries in batches of 1,024
    "xl": dict(n_doc=8_000_000, n_centroid=262_144, n_bit=4, n_query=10_240, n_tok=[32, 64],
               nprobe=8, topk=10, probe_topk=1500, kmeans_iter=4, seed=0, n_gt=100, n_tune=200,
               len_hi=300, stream=True, batch=1024),
}


def peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        p = json.load(open(path))
        return dict(hbm=p["hbm_gbs"], tc=p["bf16_tflops"], tc_sus=p["bf16_tflops_sustained"],
                    src="measured")
    return dict(hbm=6650.0, tc=1590.0, tc_sus=1400.0, src="fallback")


class ClockSampler:
    """nvidia-smi samples during the timed region."""

    def __init__(self, gpu):
        self.gpu = gpu
        self.proc = None
        self.lines = []

    def __enter__(self):
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={q}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


def cache_dir(w):
    key = json.dumps({k: w.get(k) for k in ("n_doc", "n_centroid", "n_bit", "kmeans_iter", "seed",
                                             "len_hi")}, sort_keys=True) + CACHE_VERSION
    return os.path.join("/tmp", "mvr_bench_cache", hashlib.sha1(key.encode()).hexdigest()[:16])


def get_index(w, device, rank, want_tokens):
    """GPU-built index (cached on local disk so both bench arms build once)."""
    import torch
    from mvr import build, formats, synth
    spec = synth.CorpusSpec(w["n_doc"], seed=w["seed"], len_hi=w.get("len_hi", 180))
    cdir = cache_dir(w)
    tok = None
    t0 = time.time()
    if os.path.exists(os.path.join(cdir, "DONE")):
        host = formats.read_index_dir(cdir)
        host["n_bit"] = w["n_bit"]
        built_s = None
    else:
        tok = synth.tokens(spec, device)
        ix = build.build_index(tok, spec.item_n_vec, w["n_centroid"], w["n_bit"],
                               kmeans_iter=w["kmeans_iter"], seed=123 + w["seed"])
        host = build.to_host(ix)
        del ix
        built_s = time.time() - t0
        if rank == 0:
            tmp = cdir + f".tmp{os.getpid()}"
            try:
                formats.write_index_dir(tmp, host["item_n_vec"], host["centroid"],
                                        host["vq_code"], host["weight"], host["residual"],
                                        host["ivf_off"], host["ivf_size"], host["ivf_ids"])
                open(os.path.join(tmp, "DONE"), "w").close()
                os.replace(tmp, cdir)
            except OSError:
                pass
    if want_tokens and tok is None:
        tok = synth.tokens(spec, device)
    torch.cuda.empty_cache()
    return spec, host, tok, built_s


def get_index_stream(w, device):
    """Index of a streamed workload, built on the device one doc range at a
    time (the raw corpus is never resident); returns (spec, device arrays,
    build seconds)."""
    import torch
    from mvr import build, synth
    spec = synth.CorpusSpec(w["n_doc"], seed=w["seed"], len_hi=w.get("len_hi", 180))
    t0 = time.time()
    ix = build.build_index_stream(spec, w["n_centroid"], w["n_bit"], kmeans_iter=w["kmeans_iter"],
                                  seed=123 + w["seed"], device=device)
    torch.cuda.synchronize()
    return spec, ix, time.time() - t0


def gt_chunks(spec, tokens_of, n_q_tok):
    """(d0, lens, tokens) pieces of the corpus for exhaustive_topk_stream:
    generator blocks (or index ranges) of synth.BLOCK_DOCS docs, cut into
    pieces whose FP64 score matrix stays under ~8 GB."""
    from mvr import synth
    lens = spec.item_n_vec.astype(np.int64)
    max_tok = int(max(1 << 14, min(1 << 18, 8e9 / (8.0 * max(1, n_q_tok)))))
    for b0 in range(0, spec.n_doc, synth.BLOCK_DOCS):
        b1 = min(spec.n_doc, b0 + synth.BLOCK_DOCS)
        x = tokens_of(b0, b1)
        toff = np.zeros(b1 - b0 + 1, np.int64)
        toff[1:] = np.cumsum(lens[b0:b1])
        d0 = 0
        while d0 < b1 - b0:
            d1 = int(np.searchsorted(toff, toff[d0] + max_tok, side="right")) - 1
            d1 = min(max(d1, d0 + 1), b1 - b0)
            yield b0 + d0, lens[b0 + d0:b0 + d1], x[toff[d0]:toff[d1]]
            d0 = d1
        del x


def load_gpu_index(host, device_idx):
    from mvr import Index
    return Index.from_arrays(host["item_n_vec"], host["centroid"], host["vq_code"],
                             host["ivf_off"], host["ivf_size"], host["ivf_ids"], host["weight"],
                             host["n_bit"], host["residual"], device=device_idx)


def cpu_port_qps(host, q_np, off, w, n_threads, probe_topk, budget_s=15.0):
    """The oracle's CPU port of the path (test infrastructure) on a bounded
    query sample; returns (qps, sample size, seconds)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pyoracle
    o = pyoracle.Oracle(host["item_n_vec"], host["centroid"], host["vq_code"], host["residual"],
                        host["weight"], host["ivf_off"], host["ivf_size"], host["ivf_ids"],
                        host["n_bit"])
    probe_n = min(len(off) - 1, max(2 * n_threads, 8))
    t = time.perf_counter()
    o.search(q_np[: off[probe_n]], off[: probe_n + 1], w["topk"], w["nprobe"], probe_topk,
             n_threads=n_threads)
    per_q = (time.perf_counter() - t) / probe_n
    n = int(min(len(off) - 1, max(probe_n, budget_s / max(per_q, 1e-6))))
    t = time.perf_counter()
    o.search(q_np[: off[n]], off[: n + 1], w["topk"], w["nprobe"], probe_topk,
             n_threads=n_threads)
    dt = time.perf_counter() - t
    return n / dt, n, dt, o


def score_error_f64(q, off, ids, scores, arrays, n_bit, n_check):
    """Relative error of the returned FP32 scores against FP64 MaxSim of the
    same docs over the index's decoded vectors (GPUComputeScore.hpp:193-282
    semantics, applied to x = centroid + weight[bucket]): max and mean over
    the first n_check queries' returned docs.  arrays: the index's arrays, as
    numpy (host) or torch tensors on the GPU."""
    import torch
    from mvr import exhaustive
    dev = q.device

    def t(a):
        return a if isinstance(a, torch.Tensor) else torch.from_numpy(np.ascontiguousarray(a))
    lens = t(arrays["item_n_vec"]).cpu().numpy().view(np.uint32).astype(np.int64)
    start = np.concatenate([[0], np.cumsum(lens)])
    bpv = 128 * n_bit // 8
    cen = t(arrays["centroid"]).to(dev)
    code_all, res_all = t(arrays["vq_code"]), t(arrays["residual"]).view(-1)
    errs = []
    for i in range(n_check):
        docs = [int(d) for d in ids[i] if d != 0xFFFFFFFF]
        if not docs:
            continue
        tok = np.concatenate([np.arange(start[d], start[d + 1]) for d in docs])
        ti = torch.from_numpy(tok).to(code_all.device)
        code = code_all[ti].to(dev)
        res = res_all.view(-1, bpv)[ti].to(dev)
        x = exhaustive.decode_tokens(cen, code, res, t(arrays["weight"]), n_bit).double()
        s = q[int(off[i]):int(off[i + 1])].double() @ x.T
        seg = torch.repeat_interleave(torch.arange(len(docs), device=dev),
                                      torch.from_numpy(lens[docs]).to(dev))
        m = torch.full((s.shape[0], len(docs)), -torch.inf, dtype=torch.float64, device=dev)
        m.scatter_reduce_(1, seg.expand(s.shape[0], -1), s, reduce="amax")
        ref = m.sum(0).cpu().numpy()
        got = np.asarray([float(sc) for d, sc in zip(ids[i], scores[i]) if d != 0xFFFFFFFF])
        errs.append(np.abs(got - ref) / np.maximum(np.abs(ref), 1e-12))
    e = np.concatenate(errs) if errs else np.zeros(0)
    return {"max_rel": float(e.max()) if len(e) else None,
            "mean_rel": float(e.mean()) if len(e) else None, "results": int(len(e))}


def plain_parity(g, o, q_np, off, w, probe_topk, n_check, gpu_ids, gpu_scores, n_threads):
    """Part of the CPU-baseline leg: the first n_check workload queries traced
    stage by stage through the GPU's plain FP32 path (mvr_search_trace) and
    searched by the oracle's CPU port, with the timed plain-path top-k of the
    same queries; counts the queries whose probe lists, candidate sets with
    approximate scores, shortlists with exact scores, and final top-k are
    bit-identical."""
    from concurrent.futures import ThreadPoolExecutor
    k, nprobe = w["topk"], w["nprobe"]
    qs = [np.ascontiguousarray(q_np[off[i]:off[i + 1]]) for i in range(n_check)]
    with ThreadPoolExecutor(n_threads) as ex:  # the oracle's C calls release the GIL
        refs = list(ex.map(lambda qi: o.search_one(qi, k, nprobe, probe_topk), qs))
    cnt = dict(probe=0, candidates=0, shortlist=0, topk=0, topk_timed=0)
    for i, (qi, r) in enumerate(zip(qs, refs)):
        t = g.trace(qi, k, nprobe, probe_topk)
        cnt["probe"] += bool(np.array_equal(t["probe_id"], r["probe_id"]) and
                             np.array_equal(t["probe_score"], r["probe_score"]))
        cnt["candidates"] += bool(np.array_equal(t["cand_id"], r["cand_id"]) and
                                  np.array_equal(t["cand_score"], r["cand_score"]))
        o_ = np.argsort(r["short_id"])
        cnt["shortlist"] += bool(np.array_equal(t["short_id"], r["short_id"][o_]) and
                                 np.array_equal(t["short_approx"], r["short_approx"][o_]) and
                                 np.array_equal(t["short_exact"], r["short_exact"][o_]))
        cnt["topk"] += bool(np.array_equal(t["id"], r["id"]) and np.array_equal(t["score"], r["score"]))
        cnt["topk_timed"] += bool(np.array_equal(gpu_ids[i], r["id"]) and
                                  np.array_equal(gpu_scores[i], r["score"]))
    exact = min(cnt.values())
    return {"queries": n_check, "bit_exact": exact, "per_stage": cnt,
            "path": "plain FP32 GPU path vs the oracle's CPU port, same index and queries",
            "checked": "probe ids+scores, candidate ids+approximate scores, shortlist ids+"
                       "approximate+exact scores, top-k ids+scores (traced and timed runs)"}


def plaid_cpu_baseline(host, q_np, off, k, n_threads, gi_eval, gi_raw, budget_s=10.0,
                       sweep_q=30):
    """The reference's own PLAID CPU search (its compiled extensions, oracle/
    plaid_cpu.py) over this index re-laid in PLAID's layout, at PLAID's
    defaults for k, on a bounded sample of the workload's queries; recall@k
    on the first len(gi_eval) queries."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import plaid_cpu
    if not plaid_cpu.available():
        return {"value": None, "sample": "not run: reference PLAID extensions not built"}
    p = plaid_cpu.PlaidCPU(host["item_n_vec"], host["centroid"], host["vq_code"],
                           host["residual"], host["weight"], host["ivf_off"], host["ivf_size"],
                           host["ivf_ids"], host["n_bit"], n_threads=n_threads)
    n_q = len(off) - 1
    est, t, n = [], time.perf_counter(), 0
    while n < n_q and (n < len(gi_eval) or time.perf_counter() - t < budget_s):
        est.append(p.search_one(q_np[off[n]:off[n + 1]], k)[0])
        n += 1
    dt = time.perf_counter() - t
    m = min(len(gi_eval), len(est))
    # wider settings (PLAID's k=100 defaults, then 4x its candidate budget)
    # on the first sweep_q queries: how far PLAID's recall goes and at what rate
    sweep = []
    for prm in (dict(ncells=2, centroid_score_threshold=0.45, ndocs=1024),
                dict(ncells=4, centroid_score_threshold=0.4, ndocs=4096)):
        ns_ = min(sweep_q, n_q, len(gi_eval))
        t0 = time.perf_counter()
        e2 = [p.search_one(q_np[off[i]:off[i + 1]], k, **prm)[0] for i in range(ns_)]
        d2 = time.perf_counter() - t0
        sweep.append({"params": prm, "queries": ns_, "queries/s": ns_ / d2,
                      "recall@10": float(formats_recall(gi_eval[:ns_], e2, k)),
                      "recall@10_vs_raw": float(formats_recall(gi_raw[:ns_], e2, k))})
    return {"value": n / dt, "unit": "queries/s", "cores": n_threads, "kind": "reference",
            "sample": f"first {n} of the {n_q} queries ({dt:.1f} s)",
            "params": plaid_cpu.defaults(k),
            "recall@10": float(formats_recall(gi_eval[:m], est[:m], k)),
            "recall@10_vs_raw": float(formats_recall(gi_raw[:m], est[:m], k)),
            "sweep": sweep}


def formats_recall(gnd, est, k):
    from mvr import formats
    return formats.recall_at_k(gnd, est, k).mean()


def run_reference(args, w):
    import torch
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    if w.get("stream"):
        print(json.dumps({"impl": "reference", "unavailable": "streamed workload: the CPU port "
                          "needs the whole index in host memory; timed on the default workloads"}))
        return
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    from mvr import formats, synth
    # the index is built (once, cached on local disk) by a child process, so
    # this process maps no library of the GPU engine: it reads the cached
    # index files and runs only the CPU port
    cdir = cache_dir(w)
    if not os.path.exists(os.path.join(cdir, "DONE")):
        cmd = [sys.executable, os.path.abspath(__file__), "--build-index-only",
               "--workload", args.workload]
        if args.n_doc:
            cmd += ["--n-doc", str(args.n_doc)]
        if args.n_centroid:
            cmd += ["--n-centroid", str(args.n_centroid)]
        subprocess.run(cmd, check=True, env=dict(os.environ, CUDA_VISIBLE_DEVICES=str(local)))
    host = formats.read_index_dir(cdir)
    host["n_bit"] = w["n_bit"]
    spec = synth.CorpusSpec(w["n_doc"], seed=w["seed"], len_hi=w.get("len_hi", 180))
    q, off = synth.queries(spec, w["n_query"], w["n_tok"], f"cuda:{local}", seed=100)
    q_np = q.cpu().numpy()
    del q
    n_threads = os.cpu_count()
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pyoracle
    o = pyoracle.Oracle(host["item_n_vec"], host["centroid"], host["vq_code"], host["residual"],
                        host["weight"], host["ivf_off"], host["ivf_size"], host["ivf_ids"],
                        host["n_bit"])
    # size each step to a bounded sample (~8 s of CPU work)
    t = time.perf_counter()
    m = min(w["n_query"], 2 * n_threads)
    o.search(q_np[: off[m]], off[: m + 1], w["topk"], w["nprobe"], w["probe_topk"],
             n_threads=n_threads)
    per_q = (time.perf_counter() - t) / m
    n = int(max(m, min(w["n_query"], 8.0 / max(per_q, 1e-6))))
    for _ in range(args.warmup):
        o.search(q_np[: off[m]], off[: m + 1], w["topk"], w["nprobe"], w["probe_topk"],
                 n_threads=n_threads)
    t = time.perf_counter()
    for s in range(args.steps):
        a = (s * n) % max(1, w["n_query"] - n + 1)
        o.search(q_np[off[a]: off[a + n]], off[a: a + n + 1] - off[a], w["topk"], w["nprobe"],
                 w["probe_topk"], n_threads=n_threads)
    dt = time.perf_counter() - t
    qps = args.steps * n / dt
    line = {
        "impl": "reference", "metric": METRIC, "value": qps, "unit": "queries/s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": dt / args.steps * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": dict(workload_config(w, w["probe_topk"]),
                       path="the oracle's CPU port of the reference's IGP GPU search path "
                            "(same index files and queries as the GPU arm)"),
        "cpu_baseline": {"value": qps, "unit": "queries/s", "cores": n_threads, "kind": "port",
                         "sample": f"{n} queries per step of the {w['n_query']}-query workload"},
        "e2e": {"value": qps, "unit": "queries/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))


def workload_config(w, probe_topk):
    """The workload's description, the same for both arms."""
    return {"workload": (f"{w['n_doc']:,} synthetic docs (lognormal 70/35, clipped "
                         f"8..{w.get('len_hi', 180)}), "
                         f"{w['n_centroid']:,} centroids, nbits {w['n_bit']}, "
                         f"{w['n_query']:,} queries x {w['n_tok']} tok, nprobe {w['nprobe']}, "
                         f"k {w['topk']}, probe_topk {probe_topk}"),
            "n_doc": w["n_doc"], "n_centroid": w["n_centroid"], "n_bit": w["n_bit"],
            "queries_per_step": w["n_query"], "query_tokens": w["n_tok"], "nprobe": w["nprobe"],
            "topk": w["topk"], "probe_topk": probe_topk, "kmeans_iter": w["kmeans_iter"],
            "l2": "flushed (256 MiB write) between timed steps"}


def run_profile_case(fast_flag, n_bit=2):
    """A case small enough for ncu (a few GB on the device, one batch per
    search, inputs larger than L2): the raw tokens are freed before searching,
    so only the compressed index (~0.5 GB at nbits 2, ~1 GB at 4) and the
    working set are resident.  296 queries = 2 filter CTAs per SM."""
    import torch
    from mvr import build, synth
    spec = synth.CorpusSpec(200_000, seed=0)
    tok = synth.tokens(spec, "cuda")
    ix = build.build_index(tok, spec.item_n_vec, 16384, n_bit, kmeans_iter=2)
    del tok
    g = build.load_built(ix)
    del ix
    torch.cuda.empty_cache()
    n = 296
    g.set_batch(n)
    q, _ = synth.queries(spec, n, 32, "cuda", seed=5)
    out_s = torch.empty((n, 10), dtype=torch.float32, device="cuda")
    out_i = torch.empty((n, 10), dtype=torch.int32, device="cuda")
    for fl in (fast_flag, 0):
        st = g.search_device(q.data_ptr(), None, n, 32, 10, 8, 1000, out_s.data_ptr(),
                             out_i.data_ptr(), 0, semantics=fl)
        print("flags", fl, "device_ms", round(st.device_ms, 4), "stages_ms",
              [round(x, 4) for x in st.stage_ms], "reranked_tokens", st.n_rerank_tok, flush=True)
    print("max_mem_GB", round(torch.cuda.max_memory_allocated() / 1e9, 2))
    g.close()
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["mvr", "reference"], default="mvr")
    ap.add_argument("--workload", choices=sorted(WORKLOADS), default="medium")
    ap.add_argument("--probe-topk", type=int, default=None)
    ap.add_argument("--n-doc", type=int, default=None, help="override the workload's corpus size")
    ap.add_argument("--n-centroid", type=int, default=None,
                    help="override the workload's centroid count")
    ap.add_argument("--rescore", type=int, default=0, help="FP32 re-score width (0: 4*k)")
    ap.add_argument("--no-graphs", action="store_true",
                    help="launch every kernel from the host instead of replaying the recorded "
                         "CUDA graph of the (repeated) device-buffer search")
    ap.add_argument("--batch", type=int, default=0,
                    help="queries per device batch (0: the library's default)")
    ap.add_argument("--impute", action="store_true",
                    help="headline path: approximate scores impute unmatched query tokens "
                         "(MVR_CAND_IMPUTE); the plain path keeps the reference's scores")
    ap.add_argument("--precision", choices=["bf16", "fp8"], default="fp8",
                    help="tensor-core MaxSim precision of the headline path")
    ap.add_argument("--build-index-only", action="store_true", help=argparse.SUPPRESS)
    ap.add_argument("--prune", action="store_true",
                    help="also train the learned candidate pruner on plain-path traces of this "
                         "corpus and time the pruned FP8 search (MVR_PRUNE)")
    ap.add_argument("--prune-queries", type=int, default=50000,
                    help="training queries traced through the plain path (40 traces each)")
    ap.add_argument("--prune-keep", type=int, default=400,
                    help="shortlisted docs the pruned search scores per confident query")
    ap.add_argument("--prune-epochs", type=int, default=3)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--parity-queries", type=int, default=50,
                    help="queries of the workload checked stage by stage against the oracle's "
                         "CPU port inside the CPU-baseline leg (0: none)")
    ap.add_argument("--no-plaid-baseline", action="store_true",
                    help="skip the reference's PLAID CPU search (cpu_baseline_plaid; run by "
                         "default at N=1 on the resident workloads)")
    ap.add_argument("--profile-case", action="store_true",
                    help="small profiling target instead of the bench: 200,000 docs, 16,384 "
                         "centroids, one mixed-precision and one plain search of 296 queries")
    ap.add_argument("--profile-bits", type=int, choices=[1, 2, 4, 8], default=2,
                    help="residual code width of the profiling case")
    ap.add_argument("--no-tune", action="store_true",
                    help="skip the shortlist tuner (it only reports unless --use-tuned)")
    ap.add_argument("--gt-dtype", choices=["f64", "f32"], default="f64",
                    help="streamed workloads: arithmetic of the exhaustive ground truths "
                         "(f32 adds an FP64 spot check of 8 queries)")
    ap.add_argument("--tune-batch", action="store_true",
                    help="also time the headline search at several queries-per-batch sizes "
                         "(with --use-tuned, run at the fastest)")
    ap.add_argument("--use-tuned", action="store_true",
                    help="time this run's tuned shortlist sizes instead of the workload's")
    ap.add_argument("--target", type=float, default=0.99,
                    help="recall@k target of the shortlist tuner (vs exhaustive MaxSim over "
                         "the index's decoded vectors)")
    args = ap.parse_args()
    w = dict(WORKLOADS[args.workload])
    if args.probe_topk:
        w["probe_topk"] = w["probe_topk_fast"] = args.probe_topk
    if args.n_doc:
        w["n_doc"] = args.n_doc
    if args.n_centroid:
        w["n_centroid"] = args.n_centroid
    if args.build_index_only:  # child of the reference arm: build and cache the index
        import torch
        get_index(w, "cuda:0", 0, want_tokens=False)
        return
    if args.impl == "reference":
        return run_reference(args, w)
    if args.profile_case:
        from mvr import PREC_BF16, PREC_FP8
        return run_profile_case(PREC_FP8 if args.precision == "fp8" else PREC_BF16,
                                args.profile_bits)

    import torch
    import torch.distributed as dist
    from mvr import CAND_IMPUTE, PREC_BF16, PREC_FP8, exhaustive, formats, synth, tune
    from mvr import dist as mdist
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dev = f"cuda:{local}"
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(minutes=20))

    streamed = bool(w.get("stream"))
    if streamed:
        from mvr import build
        spec, dix, built_s = get_index_stream(w, dev)
        host, tok = None, None
        g = build.load_built(dix, local)
    else:
        spec, host, tok, built_s = get_index(w, dev, rank, want_tokens=(rank == 0))
        g = load_gpu_index(host, local)
    g.set_rescore(args.rescore)
    if args.batch or w.get("batch"):
        g.set_batch(args.batch or w["batch"])
    g.set_graphs(not args.no_graphs)
    q, off = synth.queries(spec, w["n_query"], w["n_tok"], dev, seed=100 + rank)
    n_query, T = w["n_query"], q.shape[0]
    k, nprobe = w["topk"], w["nprobe"]
    stream = torch.cuda.current_stream()
    out_s = torch.empty((n_query, k), dtype=torch.float32, device=dev)
    out_i = torch.empty((n_query, k), dtype=torch.int32, device=dev)
    FAST, PLAIN = (PREC_FP8 if args.precision == "fp8" else PREC_BF16), 0
    if args.impute:
        FAST |= CAND_IMPUTE
    # shortlist sizes: the workload's fixed values (the tuner's picks for this
    # corpus at the default target, so the reference arm times the same
    # configuration); --use-tuned times this run's own picks instead
    ptk = {FAST: w.get("probe_topk_fast", w["probe_topk"]), PLAIN: w["probe_topk"]}

    ragged = isinstance(w["n_tok"], (list, tuple))
    q_off = off if ragged else None      # token offsets passed only for ragged queries
    n_vec = 0 if ragged else w["n_tok"]
    nq_avg = T / n_query                 # query tokens per query

    def step(flags):
        return g.search_device(q.data_ptr(), q_off, n_query, n_vec, k, nprobe, ptk[flags],
                               out_s.data_ptr(), out_i.data_ptr(), stream.cuda_stream,
                               semantics=flags)

    # ground truths (rank 0): exhaustive FP64 MaxSim over the raw tokens, and
    # over the index's own decoded tokens (what candidate generation can
    # reach); the shortlist sizes are tuned on a separate query sample against
    # the latter, then recall is measured on the first n_gt workload queries
    recall, tuning, score_err = {}, {}, {}
    # the other tensor-core precision (timed beside the headline path)
    other = (FAST ^ PREC_FP8 ^ PREC_BF16) if FAST & (PREC_FP8 | PREC_BF16) else PREC_BF16
    ptk[other] = ptk[FAST]
    if rank == 0:
        n_gt, n_tune = w["n_gt"], w["n_tune"]
        qg = q[: int(off[n_gt])]
        qt, offt = synth.queries(spec, n_tune, w["n_tok"], dev, seed=900)
        both = torch.cat([qg, qt])
        both_off = np.concatenate([off[: n_gt + 1], off[n_gt] + offt[1:]]).astype(np.uint64)
        if streamed:  # raw tokens regenerated and index vectors decoded piece by piece
            bpv = 128 * w["n_bit"] // 8
            toff = np.zeros(spec.n_doc + 1, np.int64)
            toff[1:] = np.cumsum(spec.item_n_vec.astype(np.int64))
            gdt = torch.float32 if args.gt_dtype == "f32" else torch.float64

            def raw(a, b):
                return synth.tokens_range(spec, a, b, dev)
            _, gi_raw = exhaustive.exhaustive_topk_stream(
                qg, off[: n_gt + 1], gt_chunks(spec, raw, qg.shape[0]), k, dtype=gdt)
            res2 = dix["residual"].view(-1, bpv)

            def decoded(a, b):
                return exhaustive.decode_tokens(dix["centroid"], dix["vq_code"][toff[a]:toff[b]],
                                                res2[toff[a]:toff[b]], dix["weight"], w["n_bit"])
            _, gi_idx = exhaustive.exhaustive_topk_stream(
                both, both_off, gt_chunks(spec, decoded, both.shape[0]), k, dtype=gdt)
            if gdt == torch.float32:  # FP64 spot check of the FP32 ground truths
                m = min(8, n_gt)
                qs = qg[: int(off[m])]
                _, c_raw = exhaustive.exhaustive_topk_stream(
                    qs, off[: m + 1], gt_chunks(spec, raw, qs.shape[0]), k)
                _, c_dec = exhaustive.exhaustive_topk_stream(
                    qs, off[: m + 1], gt_chunks(spec, decoded, qs.shape[0]), k)
                recall["gt_f32_spot_check"] = float(
                    (np.mean(np.all(c_raw == gi_raw[:m], axis=1)) +
                     np.mean(np.all(c_dec == gi_idx[:m], axis=1))) / 2)
            del res2
        else:
            _, gi_raw = exhaustive.exhaustive_topk(qg, off[: n_gt + 1], tok, spec.item_n_vec, k)
            del tok
            torch.cuda.empty_cache()
            dec = exhaustive.decode_tokens(torch.from_numpy(host["centroid"]).to(dev),
                                           torch.from_numpy(host["vq_code"].view(np.int32)).to(dev),
                                           torch.from_numpy(host["residual"]).to(dev).view(-1, 128 * host["n_bit"] // 8),
                                           torch.from_numpy(host["weight"]), host["n_bit"])
            _, gi_idx = exhaustive.exhaustive_topk(both, both_off, dec, spec.item_n_vec, k)
            del dec
        torch.cuda.empty_cache()
        gi_eval, gi_tune = gi_idx[:n_gt], gi_idx[n_gt:]
        qt_np = qt.cpu().numpy() if ragged else qt.cpu().numpy().reshape(n_tune, w["n_tok"], 128)
        if not args.no_tune:
            for name, fl in (("fast", FAST), ("plain", PLAIN)):
                t = tune.tune(g, qt_np, gi_tune, k, nprobe, args.target, fl,
                              tok_off=offt if ragged else None)
                tuning[name] = dict(probe_topk=t["probe_topk"], recall_tune=t["recall"],
                                    reached=t["reached"], fixed=ptk[fl],
                                    table=[(x["probe_topk"], round(x["recall"], 4),
                                            round(x["ms"], 3)) for x in t["table"]])
                if args.use_tuned:
                    ptk[fl] = t["probe_topk"]
            if args.tune_batch:  # queries per device batch of the headline path (all queries)
                qh = q.cpu().numpy() if ragged else q.cpu().numpy().reshape(n_query, w["n_tok"], 128)
                tb = tune.tune_batch(g, qh, k, nprobe, ptk[FAST], FAST,
                                     tok_off=off if ragged else None)
                tuning["batch"] = dict(batch=tb["batch"], table=[(x["batch"], round(x["ms"], 3))
                                                                 for x in tb["table"]])
                g.set_batch(tb["batch"] if args.use_tuned else (args.batch or w.get("batch", 0)))
        arrays = dix if streamed else host
        ptk[other] = ptk[FAST]
        for name, fl in (("fast", FAST), ("plain", PLAIN), ("other", other)):
            step(fl)
            est = out_i[:n_gt].cpu().numpy().view(np.uint32)
            recall[name] = float(formats.recall_at_k(gi_eval, est, k).mean())
            recall[name + "_raw"] = float(formats.recall_at_k(gi_raw, est, k).mean())
            score_err[name] = score_error_f64(q, off, est, out_s[:n_gt].cpu().numpy(), arrays,
                                              w["n_bit"], n_gt)
        if streamed:
            del dix, arrays
        torch.cuda.empty_cache()
    if world > 1:  # every rank serves at rank 0's tuned shortlist sizes
        pt = torch.tensor([ptk[FAST], ptk[PLAIN]], dtype=torch.int64, device=dev)
        dist.broadcast(pt, 0)
        ptk[FAST], ptk[PLAIN] = int(pt[0]), int(pt[1])
        ptk[other] = ptk[FAST]

    # tile shape of the FP8 MaxSim kernel (docs per CTA): tuned on this rank's
    # own workload queries; results do not depend on it, only the time
    if FAST & PREC_FP8 and not args.no_tune and w["n_bit"] in (2, 4):
        qh = q.cpu().numpy() if ragged else q.cpu().numpy().reshape(n_query, w["n_tok"], 128)
        tt = tune.tune_tile(g, qh, k, nprobe, ptk[FAST], FAST, tok_off=off if ragged else None)
        tuning["tile"] = dict(docs_per_cta=tt["docs"],
                              table=[(x["docs"], round(x["ms"], 3)) for x in tt["table"]])

    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)

    def measure(flags, profile=False):
        for _ in range(args.warmup):
            step(flags)
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()
        if profile:  # ncu --profile-from-start off captures exactly the timed steps
            torch.cuda.profiler.start()
        ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
              for _ in range(args.steps)]
        acc = dict(stage=np.zeros(6), launches=0, n_cand=0, n_tok=0, n_ent=0, n_batch=0,
                   fallback=0)
        for s in range(args.steps):
            flush.fill_(s & 0xFF)
            ev[s][0].record(stream)
            st = step(flags)
            ev[s][1].record(stream)
            acc["stage"] += np.asarray(list(st.stage_ms))
            acc["launches"] += st.gpu_launches
            acc["n_cand"] += st.n_cand_total
            acc["n_tok"] += st.n_rerank_tok
            acc["n_ent"] += st.n_list_ent
            acc["n_batch"] += st.n_batch
            acc["fallback"] += st.n_prune_fallback
        torch.cuda.synchronize()
        if profile:
            torch.cuda.profiler.stop()
        total_ms = mdist.max_over_ranks(sum(a.elapsed_time(b) for a, b in ev), dev)
        if world > 1:
            dist.barrier()
        acc["total_ms"] = total_ms
        acc["qps"] = world * n_query * args.steps / (total_ms / 1e3)
        return acc

    plain = measure(PLAIN)
    alt = measure(other)
    with ClockSampler(local) as clk:
        fast = measure(FAST, profile=True)
    value = fast["qps"]
    # stage events inside a replayed graph that could not be timed: take the
    # per-stage breakdown from host-launched steps of the same search (the
    # decision is collective, so every rank runs the same barriers)
    untimed = mdist.max_over_ranks(float(not args.no_graphs and fast["stage"].sum() == 0.0), dev)
    if untimed > 0.0:
        g.set_graphs(False)
        fast["stage"] = measure(FAST)["stage"]
        g.set_graphs(True)

    # learned candidate pruner (config-4 protocol): traces of the plain path
    # on this corpus, training with libmvr's kernels, then two pruned
    # searches timed and their recall measured like the headline path's
    prune_rec = None
    if args.prune and rank == 0 and world == 1 and not streamed and not ragged:
        from mvr import PRUNE
        from mvr import prune as mprune
        t0 = time.time()
        qtr, offtr = synth.queries(spec, args.prune_queries, w["n_tok"], dev, seed=700)
        X, y, qid = mprune.traces(g, qtr.cpu().numpy(), offtr, nprobe, ptk[PLAIN],
                                  per_query=40, seed=1)
        t_trace = time.time() - t0
        hold = qid >= int(0.95 * args.prune_queries)
        t0 = time.time()
        params, hist = mprune.train(X[~hold], y[~hold], epochs=args.prune_epochs)
        t_train = time.time() - t0
        margin = mprune.margin_for(X[hold], y[hold], params)
        keep = min(args.prune_keep, ptk[FAST])
        g.set_pruner(params, keep, margin)

        def pruned(fl):
            """One pruned path: recall, error against FP64, timing."""
            ptk[fl] = ptk[FAST] if fl & FAST else ptk[PLAIN]
            step(fl)
            est = out_i[:w["n_gt"]].cpu().numpy().view(np.uint32)
            rec = float(formats.recall_at_k(gi_eval, est, k).mean())
            rec_raw = float(formats.recall_at_k(gi_raw, est, k).mean())
            err = score_error_f64(q, off, est, out_s[:w["n_gt"]].cpu().numpy(), host, w["n_bit"],
                                  w["n_gt"])
            m = measure(fl)
            return {"qps": m["qps"], "ms_per_step": m["total_ms"] / args.steps,
                    "shortlist": ptk[fl], "fallback_frac": m["fallback"] / (args.steps * n_query),
                    "recall@10": rec, "recall@10_vs_raw": rec_raw,
                    "recall@10_loss_vs_plain": recall.get("plain", 0.0) - rec,
                    "score_error_vs_f64": err,
                    "rerank_tok_per_query": m["n_tok"] / (args.steps * n_query),
                    "stage_ms_per_step": [float(x / args.steps) for x in m["stage"]]}

        # the configuration's protocol: the kept docs decompressed and scored
        # by the exact FP32 MaxSim (against the plain path) ...
        ex = pruned(PLAIN | PRUNE)
        ex["speedup_vs_plain"] = ex["qps"] / plain["qps"]
        # ... and the kept docs through the FP8 MaxSim + FP32 re-score
        # (against the headline path)
        f8 = pruned(FAST | PRUNE)
        f8["speedup_vs_headline"] = f8["qps"] / fast["qps"]
        f8["recall@10_loss_vs_headline"] = recall.get("fast", 0.0) - f8["recall@10"]
        prune_rec = {"exact": ex, "fp8": f8, "keep": keep, "margin": margin,
                     "traces": int(len(y)), "train_queries": args.prune_queries,
                     "trace_s": t_trace, "train_s": t_train, "train_loss": hist,
                     "heldout_rmse": margin / 3.0,
                     "features": "per query token the best E4M3 centroid score among the doc's "
                                 "tokens' centroids, and log(doc length)",
                     "model": "MLP 33-256-256-1, GELU, BF16 weights, FP32 accumulation; "
                              "trained by libmvr's kernels (Adam, MSE on exact MaxSim / nq)"}
        g.set_pruner(None, 0, 0.0)

    # end to end: pinned host buffers, copies inside every step
    hq = q.cpu().pin_memory()
    hs = torch.empty((n_query, k), dtype=torch.float32).pin_memory()
    hi = torch.empty((n_query, k), dtype=torch.int32).pin_memory()
    qtime = np.zeros(n_query)
    e2e_dt = []
    for s in range(args.warmup + args.steps):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        st_e = g.search_host_ptr(hq.data_ptr(), q_off, n_query, n_vec, k, nprobe, ptk[FAST],
                                 hs.data_ptr(), hi.data_ptr(), semantics=FAST, qtime=qtime)
        if s >= args.warmup:
            e2e_dt.append(time.perf_counter() - t0)
    e2e_s = mdist.max_over_ranks(sum(e2e_dt), dev)
    e2e = world * n_query * args.steps / e2e_s
    p50, p99 = (float(np.percentile(qtime, p)) * 1e3 for p in (50, 99))

    if rank != 0:
        dist.destroy_process_group()
        return

    # roofline of the dominant stage of the headline (mixed-precision) path;
    # stage_ms: 0 query copy, 1 probe, 2 filter, 3 rerank, 4 re-score+top-k, 5 copy
    pk = peaks()
    S = args.steps
    C, D = w["n_centroid"], 128
    bpv = D * w["n_bit"] // 8
    stage = fast["stage"]
    n_launch = max(1, fast["n_batch"])  # batches = launches of each stage's kernel, all steps
    tok_launch = fast["n_tok"] / n_launch
    probe_flop = 2.0 * T * C * D * S
    rerank_bytes = (4.0 + bpv) * fast["n_tok"]           # vq code + residual bytes per token
    filter_bytes = 4.0 * fast["n_ent"] + 16.0 * fast["n_cand"]  # list entries; keys out + in
    fp8_ran = bool(FAST & PREC_FP8) and w["n_bit"] in (2, 4)  # FP8 MaxSim: 2- and 4-bit codes
    rk = ("rerank_ws_kernel (FP8)" if fp8_ran else
          "rerank_tmem_kernel (BF16)" if w["n_bit"] <= 2 else "rerank_tc_kernel (BF16)")
    kern = {1: ("probe_tc_kernel + probe_rescore_kernel", "tensor", probe_flop / 1e12,
                pk["tc_sus"], "TFLOP/s"),
            2: ("filter_hash_kernel + filter_select_kernel", "hbm", filter_bytes / 1e9, pk["hbm"],
                "GB/s"),
            3: (rk, "hbm", rerank_bytes / 1e9, pk["hbm"], "GB/s")}
    dom = max((1, 2, 3), key=lambda i: stage[i])
    name, bound, work, peak, unit = kern[dom]
    achieved = work / (stage[dom] / 1e3)
    names = ("query_copy", "probe", "filter", "rerank", "rescore_topk", "result_copy")
    # DRAM bytes per reranked token of the FP8 rerank kernel, measured by ncu
    # on the 200,000-doc profiling case, scaled to a launch of this workload
    # by its reranked tokens
    per_tok = RERANK_DRAM_BYTES_PER_TOKEN.get(w["n_bit"])
    traffic = per_tok * tok_launch if (dom == 3 and fp8_ran and per_tok) else None
    roof = {"kernel": name, "bound": bound, "achieved": achieved, "peak": peak, "unit": unit,
            "frac": achieved / peak, "traffic": traffic,
            "algorithmic_bytes_per_launch": rerank_bytes / n_launch if dom == 3 else None,
            "peak_source": f"{pk['src']} ({'bf16 sustained' if bound == 'tensor' else 'HBM copy'})",
            "stage_share": {n: float(stage[i] / stage.sum()) for i, n in enumerate(names)},
            "per_stage": {kern[i][0]: {"ms_per_step": float(stage[i] / S), "bound": kern[i][1],
                                       "achieved": kern[i][2] / (stage[i] / 1e3),
                                       "frac": kern[i][2] / (stage[i] / 1e3) / kern[i][3],
                                       "unit": kern[i][4]} for i in (1, 2, 3)},
            "rerank_tflops": 2.0 * nq_avg * D * fast["n_tok"] / 1e12 / (stage[3] / 1e3),
            "rescore_topk_ms_per_step": float(stage[4] / S)}

    cpu, parity = None, None
    if streamed:
        cpu = {"value": None, "unit": "queries/s", "cores": 0, "kind": "port",
               "sample": "not run: the streamed index lives on the device only (the CPU port "
                         "is timed on the default workloads)"}
    elif world == 1 and not args.no_cpu_baseline:
        qps_cpu, n_s, dt_s, orc = cpu_port_qps(host, hq.numpy(), off, w, os.cpu_count(),
                                               ptk[PLAIN])
        cpu = {"value": qps_cpu, "unit": "queries/s", "cores": os.cpu_count(), "kind": "port",
               "sample": f"first {n_s} of the {n_query} queries ({dt_s:.1f} s)"}
        if args.parity_queries > 0:  # the oracle as the checker of the plain GPU path
            n_chk = min(args.parity_queries, n_query)
            step(PLAIN)
            torch.cuda.synchronize()
            parity = plain_parity(g, orc, hq.numpy(), off, w, ptk[PLAIN], n_chk,
                                  out_i[:n_chk].cpu().numpy().view(np.uint32),
                                  out_s[:n_chk].cpu().numpy(), os.cpu_count())
    plaid = None
    if not args.no_plaid_baseline and not streamed and world == 1:
        plaid = plaid_cpu_baseline(host, hq.numpy(), off, k, os.cpu_count(), gi_eval, gi_raw)

    R = args.rescore or 4 * k
    gt_dt = args.gt_dtype if streamed else "f64"
    gt_name = ("FP32 (FP64 spot check: gt_f32_spot_check)" if gt_dt == "f32" else "FP64")
    line = {
        "metric": METRIC, "value": value, "unit": "queries/s", "n_gpus": world, "steps": S,
        "warmup": args.warmup, "ms_per_step": fast["total_ms"] / S, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "fp8" if fp8_ran else "bf16",
        "data": "synthetic",
        "config": dict(workload_config(w, ptk[FAST]),
                       **{"path": f"{'FP8' if fp8_ran else 'BF16'} tensor-core MaxSim + FP32 "
                                  "re-score", "rescore": R, "probe_topk": ptk[FAST], "probe_topk_plain": ptk[PLAIN],
                          "recall@10": recall.get("fast"), "recall@10_plain": recall.get("plain"),
                          "recall@10_vs_raw": recall.get("fast_raw"),
                          "recall@10_plain_vs_raw": recall.get("plain_raw"),
                          "recall_ground_truth": f"exhaustive {gt_name} MaxSim over the index's "
                          "decoded vectors (recall@10); over the raw synthetic tokens (..._vs_raw)",
                          "recall_queries": w["n_gt"], "tuning": tuning,
                          "ground_truth_dtype": gt_dt,
                          "gt_f32_spot_check": recall.get("gt_f32_spot_check"),
                          ("recall@10_bf16" if other & PREC_BF16 else "recall@10_fp8"):
                              recall.get("other"),
                          "score_error_vs_f64": {
                              "what": "returned FP32 scores vs FP64 MaxSim of the same docs over "
                                      "the decoded index vectors, over the recall queries' "
                                      "top-k",
                              "headline": score_err.get("fast"), "plain": score_err.get("plain"),
                              ("bf16" if other & PREC_BF16 else "fp8"): score_err.get("other")},
                          "plain_fp32_qps": plain["qps"],
                          ("bf16_qps" if other & PREC_BF16 else "fp8_qps"): alt["qps"],
                          "candidate_scores": "imputed (MVR_CAND_IMPUTE)" if args.impute
                          else "reference (0 for unmatched tokens)",
                          "speedup_vs_plain": value / plain["qps"],
                          "plain_stage_ms_per_step": [float(x / S) for x in plain["stage"]],
                          "p50_ms": p50, "p99_ms": p99, "latency": "per query = its batch's "
                          "device latency incl. copies (e2e run)",
                          "parallelism": f"replica x{world}, queries split by rank",
                          "launch": "host launches" if args.no_graphs else
                          "one recorded CUDA graph per step (replayed)",
                          "index_build_s": built_s,
                          "index_build": "streamed: block-keyed generator, tensor-core assignment"
                          if streamed else "resident corpus, FP32 assignment",
                          "queries_per_batch": args.batch or w.get("batch") or "8 per SM",
                          "cand_per_query": fast["n_cand"] / (S * n_query),
                          "rerank_tok_per_query": fast["n_tok"] / (S * n_query)}),
        "e2e": {"value": e2e, "unit": "queries/s",
                "h2d_bytes_per_step": int(st_e.h2d_bytes), "d2h_bytes_per_step": int(st_e.d2h_bytes)},
        "roofline": roof,
        "cpu_baseline": cpu,
        **({"cpu_baseline_plaid": plaid} if plaid is not None else {}),
        **({"parity": parity} if parity is not None else {}),
        **({"pruner": prune_rec} if prune_rec is not None else {}),
        "clocks": clk.summary(),
        "gpu_launches": int(fast["launches"]),
        "p99_ms": p99,
    }
    print(json.dumps(line))
    if world > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
