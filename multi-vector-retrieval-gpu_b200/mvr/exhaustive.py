"""Exhaustive MaxSim ground truth on the GPU (the reference's
BruteForceProgressive semantics, GPUComputeScore.hpp:193-282: score(q, d) =
sum over query tokens of the max over doc tokens of <q_t, d_j>), in FP64 by
default, streamed over token chunks cut at doc boundaries.  Used to measure
recall; the search path does not call it."""
import numpy as np
import torch


def _doc_ranges(lens, chunk_tokens):
    """[d0, d1) ranges of ~chunk_tokens tokens, cut at doc boundaries."""
    n_doc = len(lens)
    doc_start = np.zeros(n_doc + 1, np.int64)
    doc_start[1:] = np.cumsum(lens)
    out, d0 = [], 0
    while d0 < n_doc:
        d1 = int(np.searchsorted(doc_start, doc_start[d0] + chunk_tokens, side="right")) - 1
        d1 = min(max(d1, d0 + 1), n_doc)
        out.append((d0, d1, int(doc_start[d0]), int(doc_start[d1])))
        d0 = d1
    return out


def exhaustive_topk_stream(q, tok_off, chunks, k, dtype=torch.float64):
    """Exhaustive top-k over docs delivered in pieces.  chunks: iterable of
    (d0, lens, tokens): consecutive doc ranges in ascending order, lens the
    docs' token counts (numpy), tokens their [sum(lens), 128] vectors on the
    device of q.  Each piece's doc scores are computed in full, its top-k
    merged into the running top-k; ties keep the lower doc id throughout.
    Returns (scores float64 [n_query, k], ids int64 [n_query, k]) sorted by
    (score desc, id asc)."""
    dev = q.device
    n_query = len(tok_off) - 1
    qd = q.to(dtype)
    tok_q = torch.repeat_interleave(torch.arange(n_query, device=dev),
                                    torch.from_numpy(np.diff(np.asarray(tok_off, np.int64))).to(dev))
    best_s = torch.empty((n_query, 0), dtype=dtype, device=dev)
    best_i = torch.empty((n_query, 0), dtype=torch.int64, device=dev)
    for d0, lens, x in chunks:
        nd = len(lens)
        s = qd @ x.to(dev, dtype).T                                   # [Tq, tok]
        doc_of = torch.repeat_interleave(torch.arange(nd, device=dev),
                                         torch.from_numpy(np.asarray(lens, np.int64)).to(dev))
        m = torch.full((qd.shape[0], nd), -torch.inf, dtype=dtype, device=dev)
        m.scatter_reduce_(1, doc_of.expand(qd.shape[0], -1), s, reduce="amax")
        per_q = torch.zeros((n_query, nd), dtype=dtype, device=dev)
        per_q.index_add_(0, tok_q, m)
        top = torch.sort(per_q, dim=1, descending=True, stable=True)
        kk = min(k, nd)
        cat_s = torch.cat([best_s, top.values[:, :kk]], 1)
        cat_i = torch.cat([best_i, top.indices[:, :kk] + d0], 1)
        o = torch.sort(cat_s, dim=1, descending=True, stable=True).indices[:, :k]
        best_s, best_i = torch.gather(cat_s, 1, o), torch.gather(cat_i, 1, o)
    return best_s.cpu().numpy(), best_i.cpu().numpy()


def exhaustive_topk(q, tok_off, doc_tokens, item_n_vec, k, dtype=torch.float64,
                    chunk_tokens=1 << 18):
    """q: [total_q_tok, 128] (CUDA), tok_off: uint64 [n_query+1],
    doc_tokens: [n_vec, 128] (CUDA), item_n_vec: uint32 [n_doc].
    Returns (scores float64 [n_query, k], ids int64 [n_query, k]) sorted by
    (score desc, id asc)."""
    lens = np.asarray(item_n_vec, np.int64)
    q = q.to(doc_tokens.device)
    chunks = ((d0, lens[d0:d1], doc_tokens[t0:t1])
              for d0, d1, t0, t1 in _doc_ranges(lens, chunk_tokens))
    return exhaustive_topk_stream(q, tok_off, chunks, k, dtype)


def decode_tokens(centroid, vq_code, residual, weight, n_bit, chunk=1 << 22):
    """Every token of an index decoded the way the FP32 search path decodes
    it: x = centroid[code] + weight[bucket] (one FP32 add per value), buckets
    unpacked MSB-first, dim j = byte * (8 / n_bit) + i (RerankPP.hpp:100-111).
    Inputs are torch tensors on the GPU (residual uint8 [n_vec, 128*n_bit/8]);
    returns float32 [n_vec, 128] on the same device."""
    dev = centroid.device
    n = vq_code.shape[0]
    vpb = 8 // n_bit
    shifts = torch.tensor([8 - n_bit * (i + 1) for i in range(vpb)], device=dev,
                          dtype=torch.int32)
    w = weight.to(dev, torch.float32)
    code = vq_code.to(torch.int64)
    out = torch.empty((n, 128), dtype=torch.float32, device=dev)
    for a in range(0, n, chunk):
        b = min(n, a + chunk)
        r = residual[a:b].to(torch.int32).unsqueeze(-1)            # [m, bytes, 1]
        bucket = ((r >> shifts) & ((1 << n_bit) - 1)).reshape(b - a, 128)
        out[a:b] = centroid[code[a:b]] + w[bucket.to(torch.int64)]
    return out
