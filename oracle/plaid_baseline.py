"""CPU baselines on one host, no GPU: the reference's PLAID CPU search
(plaid_cpu.py, the reference's compiled extensions) and the oracle's C port
of the IGP search path, over the same synthetic index (built on the CPU with
the oracle's codec and IVF functions), with recall@10 against exhaustive
FP64 MaxSim over the index's decoded vectors and over the raw tokens.
Baseline infrastructure; prints one JSON line.

    python oracle/plaid_baseline.py [--n-doc 10000 --n-centroid 8192 ...]
"""
import argparse
import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
sys.path.insert(0, os.path.join(os.path.dirname(HERE), "multi-vector-retrieval-gpu_b200"))


def recall(gt, est, k):
    return float(np.mean([len(set(gt[i][:k]) & set(est[i][:k])) / k for i in range(len(gt))]))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--n-doc", type=int, default=10_000)
    ap.add_argument("--n-centroid", type=int, default=8192)
    ap.add_argument("--n-bit", type=int, default=2)
    ap.add_argument("--n-query", type=int, default=200)
    ap.add_argument("--nprobe", type=int, default=4)
    ap.add_argument("--probe-topk", type=int, default=200)
    ap.add_argument("--threads", type=int, default=os.cpu_count())
    ap.add_argument("--kmeans-iter", type=int, default=4)
    a = ap.parse_args()
    import torch
    import plaid_cpu
    import pyoracle
    from mvr import synth
    torch.set_num_threads(a.threads)
    k = 10
    spec = synth.CorpusSpec(a.n_doc, seed=0)
    tok = synth.tokens(spec, "cpu").numpy()
    # spherical k-means on the reference's k-means sample of docs (the GPU
    # builder's method, vq.py:15-30 sample rule), max-inner-product assignment
    n_s = min(1 + int(8 * np.sqrt(120 * a.n_doc)), a.n_doc)
    rng = np.random.default_rng(12345)
    docs = np.sort(rng.choice(a.n_doc, n_s, replace=False))
    toff = np.concatenate([[0], np.cumsum(spec.item_n_vec.astype(np.int64))])
    sample = tok[np.concatenate([np.arange(toff[d], toff[d + 1]) for d in docs])]
    cen = sample[rng.choice(len(sample), a.n_centroid, replace=False)].copy()
    for _ in range(a.kmeans_iter):
        c = pyoracle.assign(sample, cen).astype(np.int64)
        sums = np.stack([np.bincount(c, weights=sample[:, d], minlength=a.n_centroid)
                         for d in range(sample.shape[1])], axis=1)
        nz = np.bincount(c, minlength=a.n_centroid) > 0
        cen[nz] = (sums[nz] / np.linalg.norm(sums[nz], axis=1, keepdims=True)).astype(np.float32)
    code = pyoracle.assign(tok, cen)
    cut, w = pyoracle.quantize(tok, cen, code, a.n_bit)
    res = pyoracle.pack_residual(tok, cen, code, cut, a.n_bit)
    off_i, size_i, ids_i = pyoracle.ivf_build(code, spec.item_n_vec, a.n_centroid)
    o = pyoracle.Oracle(spec.item_n_vec, cen, code, res, w, off_i, size_i, ids_i, a.n_bit)
    q, off = synth.queries(spec, a.n_query, 32, "cpu", seed=100)
    q = q.numpy()
    _, gt_dec = pyoracle.exhaustive_f64(q, off, o.decompress_all(), spec.item_n_vec, k)
    _, gt_raw = pyoracle.exhaustive_f64(q, off, tok, spec.item_n_vec, k)

    p = plaid_cpu.PlaidCPU(spec.item_n_vec, cen, code, res, w, off_i, size_i, ids_i, a.n_bit,
                           n_threads=a.threads)
    p.search_one(q[off[0]:off[1]], k)  # warm-up
    t = time.perf_counter()
    est = [p.search_one(q[off[i]:off[i + 1]], k)[0] for i in range(a.n_query)]
    plaid_s = time.perf_counter() - t
    est = [np.pad(e, (0, k - len(e)), constant_values=-1) for e in est]

    o.search(q[:off[8]], off[:9], k, a.nprobe, a.probe_topk, n_threads=a.threads)  # warm-up
    t = time.perf_counter()
    _, ig = o.search(q, off, k, a.nprobe, a.probe_topk, n_threads=a.threads)
    igp_s = time.perf_counter() - t
    print(json.dumps({
        "corpus": f"{a.n_doc:,} synthetic docs, {a.n_centroid:,} centroids, nbits {a.n_bit}, "
                  f"{a.n_query} queries x 32 tokens, k {k}",
        "threads": a.threads,
        "plaid_cpu_reference": {"qps": a.n_query / plaid_s, "params": plaid_cpu.defaults(k),
                                "recall@10_vs_decoded": recall(gt_dec, est, k),
                                "recall@10_vs_raw": recall(gt_raw, est, k)},
        "igp_cpu_port": {"qps": a.n_query / igp_s, "nprobe": a.nprobe,
                         "probe_topk": a.probe_topk,
                         "recall@10_vs_decoded": recall(gt_dec, ig.astype(np.int64), k),
                         "recall@10_vs_raw": recall(gt_raw, ig.astype(np.int64), k)},
    }))


if __name__ == "__main__":
    main()
