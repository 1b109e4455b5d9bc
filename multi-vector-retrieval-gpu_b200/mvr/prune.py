"""Learned candidate pruner (MVR_PRUNE; no counterpart in the reference).

An MLP 33 -> 256 -> 256 -> 1 (GELU, BF16 weights, FP32 accumulation)
predicts, from a shortlisted doc's features -- per query token the best
centroid score among the doc's tokens' centroids, and log(doc length) --
the doc's exact MaxSim divided by the query's token count.  The search then
scores with the FP8 MaxSim only the `keep` docs with the best predictions,
falling back to the whole shortlist when the prediction of the query's R-th
best doc does not lead its keep-th best by `margin`; the exact FP32 re-score
still decides the final top-k.

traces() runs the plain path (mvr_search_trace) and keeps, per query, the
exact MaxSim and the features of a sample of its shortlist; train() fits
the MLP with libmvr's hand-written kernels (mvr_mlp_train_step: forward,
backward and Adam on the GPU); margin_for() calibrates the confidence
margin on held-out traces.
"""
import ctypes as C
import math

import numpy as np

from . import _lib

NUM_PARAMS = 74753


def traces(g, queries, tok_off, nprobe, probe_topk, per_query=40, seed=0):
    """(X [N, 33] float32, y [N] float32, qid [N] int64): for each query,
    the exact top-(per_query // 2) of its shortlist and per_query // 2 more
    drawn at random from the rest, with y = exact MaxSim / query tokens."""
    rng = np.random.default_rng(seed)
    xs, ys, qs = [], [], []
    n_query = len(tok_off) - 1
    for i in range(n_query):
        qi = queries[tok_off[i]:tok_off[i + 1]]
        t = g.trace(qi, 10, nprobe, probe_topk, features=True, cand=False)
        ex, f = t["short_exact"], t["short_feat"]
        if len(ex) == 0:
            continue
        order = np.argsort(-ex, kind="stable")
        top = order[: per_query // 2]
        rest = order[per_query // 2:]
        pick = np.concatenate([top, rng.choice(rest, min(len(rest), per_query - len(top)),
                                                replace=False)]) if len(rest) else top
        xs.append(f[pick])
        ys.append(ex[pick] / qi.shape[0])
        qs.append(np.full(len(pick), i, np.int64))
    return (np.concatenate(xs).astype(np.float32), np.concatenate(ys).astype(np.float32),
            np.concatenate(qs))


def init_params(seed=0):
    """Scaled normal initialisation of the parameter vector (float32), biases 0."""
    rng = np.random.default_rng(seed)
    p = np.zeros(NUM_PARAMS, np.float32)
    o = 0
    for shape, scale in (((256, 33), 1 / math.sqrt(33)), ((256,), 0.0),
                         ((256, 256), 1 / math.sqrt(256)), ((256,), 0.0),
                         ((256,), 1 / math.sqrt(256)), ((1,), 0.0)):
        n = int(np.prod(shape))
        p[o:o + n] = rng.standard_normal(n).astype(np.float32) * scale
        o += n
    return p


def train(X, y, epochs=3, batch=4096, lr=1e-3, seed=0, device="cuda", log=None):
    """Fits the MLP to (X, y) with libmvr's training kernels (Adam on the
    mean squared error, one shuffled pass per epoch).  Returns (params float32
    [NUM_PARAMS], per-epoch mean losses)."""
    import torch
    L = _lib.lib()
    Xd = torch.from_numpy(np.ascontiguousarray(X, np.float32)).to(device)
    yd = torch.from_numpy(np.ascontiguousarray(y, np.float32)).to(device)
    p = torch.from_numpy(init_params(seed)).to(device)
    m = torch.zeros_like(p)
    v = torch.zeros_like(p)
    n = Xd.shape[0]
    batch = min(batch, n)
    work = torch.zeros(L.mvr_mlp_work_floats(batch), device=device)
    loss = torch.zeros(1, device=device)
    gen = torch.Generator(device="cpu").manual_seed(seed)
    step, hist = 0, []
    for ep in range(epochs):
        perm = torch.randperm(n, generator=gen).to(device)
        tot, cnt = 0.0, 0
        for a in range(0, n - batch + 1, batch):
            idx = perm[a:a + batch]
            xb, yb = Xd[idx].contiguous(), yd[idx].contiguous()
            step += 1
            _lib.check(L.mvr_mlp_train_step(
                C.c_void_p(xb.data_ptr()), C.c_void_p(yb.data_ptr()), batch,
                C.c_void_p(p.data_ptr()), C.c_void_p(m.data_ptr()), C.c_void_p(v.data_ptr()),
                C.c_void_p(work.data_ptr()), lr, step, C.c_void_p(loss.data_ptr()), None))
            tot += float(loss[0])
            cnt += 1
        hist.append(tot / max(cnt, 1))
        if log:
            log(f"epoch {ep}: loss {hist[-1]:.6f}")
    return p.cpu().numpy(), hist


def predict(X, params, device="cuda"):
    """The MLP on CUDA cores (the training kernels' forward pass)."""
    import torch
    L = _lib.lib()
    n = X.shape[0]
    Xd = torch.from_numpy(np.ascontiguousarray(X, np.float32)).to(device)
    p = torch.from_numpy(np.ascontiguousarray(params, np.float32)).to(device)
    work = torch.zeros(L.mvr_mlp_work_floats(n), device=device)
    out = torch.zeros(n, device=device)
    _lib.check(L.mvr_mlp_forward(C.c_void_p(Xd.data_ptr()), n, C.c_void_p(p.data_ptr()),
                                 C.c_void_p(work.data_ptr()), C.c_void_p(out.data_ptr()), None))
    return out.cpu().numpy()


def margin_for(X, y, params, k_sigma=3.0):
    """Confidence margin: k_sigma times the RMS prediction error on held-out
    traces (prediction units)."""
    err = predict(X, params) - y
    return float(k_sigma * np.sqrt(np.mean(err.astype(np.float64) ** 2)))
