"""Exhaustive MaxSim ground truth on the GPU (the reference's
BruteForceProgressive semantics, GPUComputeScore.hpp:193-282: score(q, d) =
sum over query tokens of the max over doc tokens of <q_t, d_j>), in FP64 by
default, streamed over token chunks cut at doc boundaries.  Used to measure
recall; the search path does not call it."""
import numpy as np
import torch


def exhaustive_topk(q, tok_off, doc_tokens, item_n_vec, k, dtype=torch.float64,
                    chunk_tokens=1 << 18):
    """q: [total_q_tok, 128] (CUDA), tok_off: uint64 [n_query+1],
    doc_tokens: [n_vec, 128] (CUDA), item_n_vec: uint32 [n_doc].
    Returns (scores float64 [n_query, k], ids int64 [n_query, k]) sorted by
    (score desc, id asc)."""
    dev = doc_tokens.device
    n_query = len(tok_off) - 1
    n_doc = len(item_n_vec)
    lens = np.asarray(item_n_vec, np.int64)
    doc_start = np.zeros(n_doc + 1, np.int64)
    doc_start[1:] = np.cumsum(lens)
    qd = q.to(dev, dtype)
    tok_q = torch.repeat_interleave(torch.arange(n_query, device=dev),
                                    torch.from_numpy(np.diff(tok_off.astype(np.int64))).to(dev))
    scores = torch.empty((n_query, n_doc), dtype=dtype, device=dev)
    d0 = 0
    while d0 < n_doc:
        d1 = int(np.searchsorted(doc_start, doc_start[d0] + chunk_tokens, side="right")) - 1
        d1 = max(d1, d0 + 1)
        d1 = min(d1, n_doc)
        t0, t1 = int(doc_start[d0]), int(doc_start[d1])
        x = doc_tokens[t0:t1].to(dtype)
        s = qd @ x.T                                            # [Tq, tok]
        doc_of = torch.repeat_interleave(torch.arange(d1 - d0, device=dev),
                                         torch.from_numpy(lens[d0:d1]).to(dev))
        m = torch.full((qd.shape[0], d1 - d0), -torch.inf, dtype=dtype, device=dev)
        m.scatter_reduce_(1, doc_of.expand(qd.shape[0], -1), s, reduce="amax")
        per_q = torch.zeros((n_query, d1 - d0), dtype=dtype, device=dev)
        per_q.index_add_(0, tok_q, m)
        scores[:, d0:d1] = per_q
        d0 = d1
    # (score desc, id asc): stable sort of ids by descending score
    order = torch.sort(scores, dim=1, descending=True, stable=True)
    return order.values[:, :k].cpu().numpy(), order.indices[:, :k].cpu().numpy()


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
