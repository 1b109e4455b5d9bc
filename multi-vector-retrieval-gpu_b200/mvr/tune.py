"""Shortlist-size autotuner.

The search path's cost grows with the shortlist (probe_topk docs are
decompressed and scored per query) and, on the mixed-precision path, with the
FP32 re-score width R.  `tune` measures, on a sample of queries with a known
ground truth, the recall@k and the device time of every candidate setting and
returns the cheapest one whose recall reaches the target: the smallest
shortlist (then the smallest re-score width), a deterministic choice since
the work per query grows with both.  The ground truth is
whatever the caller wants the search to reproduce: the exhaustive MaxSim over
the index's own decoded vectors measures the loss of candidate generation
alone (the quantity a shortlist size can change), the exhaustive MaxSim over
raw embeddings adds the loss of the residual codes.
"""
import numpy as np

from .formats import recall_at_k


def tune(index, queries, gnd_ids, k, nprobe, target, semantics,
         probe_topks=(100, 150, 200, 300, 400, 600, 800, 1000, 1500, 2000, 3000, 4000,
                     6000, 8000),
         rescores=(0,), repeats=3, tok_off=None):
    """queries: float32 [n_query, n_tok, 128] (host), or [total_tokens, 128]
    with tok_off (uint64 [n_query + 1]) for ragged queries; gnd_ids:
    [n_query, >= k].
    Returns dict(probe_topk, rescore, recall, ms, table, reached) for the
    smallest setting with mean recall@k >= target (the most accurate one if
    none reaches it); the ascending grid is measured up to the first setting
    that reaches the target, and `table` lists every setting measured."""
    table = []
    for ptk in probe_topks:
        if ptk < k:
            continue
        if table and any(t["recall"] >= target for t in table):
            break  # the grid ascends: the smallest setting reaching the target is known
        for r in rescores:
            if r and (r < k or r > ptk):
                continue
            index.set_rescore(r)
            best_ms = None
            for _ in range(repeats):
                if tok_off is None:
                    s, i, st = index.search(queries, k, nprobe, ptk, semantics=semantics,
                                            with_stats=True)
                else:
                    s, i, st = index.search(queries, k, nprobe, ptk, tok_off=tok_off,
                                            semantics=semantics, with_stats=True)
                best_ms = st["device_ms"] if best_ms is None else min(best_ms, st["device_ms"])
            rec = float(recall_at_k(gnd_ids, i, k).mean())
            table.append(dict(probe_topk=ptk, rescore=r, recall=rec, ms=best_ms))
    index.set_rescore(0)
    ok = [t for t in table if t["recall"] >= target]
    pick = (min(ok, key=lambda t: (t["probe_topk"], t["rescore"])) if ok
            else max(table, key=lambda t: (t["recall"], -t["probe_topk"])))
    return dict(pick, table=table, reached=bool(ok))


def tune_batch(index, queries, k, nprobe, probe_topk, semantics,
               batches=(296, 592, 1184, 2368, 4096), repeats=3, tok_off=None):
    """Queries per device batch: every candidate size is set on the index
    (set_batch) and the same search timed (best device time of `repeats`);
    returns dict(batch, ms, qps, table) for the fastest, then restores the
    library default (set_batch(0)).  Results do not depend on the batch
    size, only the time does (larger batches fill the tensor-core tiles and
    amortise launches; smaller ones shorten each batch's latency)."""
    n_query = len(tok_off) - 1 if tok_off is not None else len(queries)
    table = []
    for b in batches:
        index.set_batch(b)
        best = None
        for _ in range(repeats):
            if tok_off is None:
                st = index.search(queries, k, nprobe, probe_topk, semantics=semantics,
                                  with_stats=True)[2]
            else:
                st = index.search(queries, k, nprobe, probe_topk, tok_off=tok_off,
                                  semantics=semantics, with_stats=True)[2]
            best = st["device_ms"] if best is None else min(best, st["device_ms"])
        table.append(dict(batch=b, ms=best, qps=n_query / (best / 1e3) if best else None))
    index.set_batch(0)
    pick = min(table, key=lambda t: (t["ms"], t["batch"]))
    return dict(pick, table=table)


def tune_tile(index, queries, k, nprobe, probe_topk, semantics, tiles=(32, 64, 128, 256), repeats=3,
              tok_off=None, stage=3):
    """Tile shape of the FP8 MaxSim kernel (shortlisted docs per CTA): every
    candidate is set on the index (set_rerank_tile) and the same search timed
    (best of `repeats` of the rerank stage's device time, stage_ms[stage]);
    returns dict(docs, ms, table) for the fastest and leaves it set.  Results
    do not depend on the tile shape, only the time does (more docs per CTA
    amortise its set-up, fewer spread a short shortlist over more SMs)."""
    table = []
    for d in tiles:
        index.set_rerank_tile(d)
        best = None
        for _ in range(repeats):
            if tok_off is None:
                st = index.search(queries, k, nprobe, probe_topk, semantics=semantics,
                                  with_stats=True)[2]
            else:
                st = index.search(queries, k, nprobe, probe_topk, tok_off=tok_off,
                                  semantics=semantics, with_stats=True)[2]
            ms = st["stage_ms"][stage] or st["device_ms"]
            best = ms if best is None else min(best, ms)
        table.append(dict(docs=d, ms=best))
    pick = min(table, key=lambda t: (t["ms"], t["docs"]))
    index.set_rerank_tile(pick["docs"])
    return dict(pick, table=table)
