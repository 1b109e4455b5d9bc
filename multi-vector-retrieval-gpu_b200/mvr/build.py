"""GPU index builder producing the reference's index layout (the pipeline of
vq_sq_pack.vq_sq_ivf, script/evaluation/technique/vq_sq_pack.py:91-109):

 1. k-means sample: min(1 + int(8*sqrt(120*n_item)), n_item) docs drawn with
    Python's random.seed(12345); random.sample (vq.py:15-30);
 2. spherical k-means on the sample: max-inner-product assignment (libmvr's
    FP32 scoring kernel), FP64 centroid sums (libmvr kernel), L2-normalised
    centroids; empty clusters keep their previous centroid.  (The reference
    uses faiss-gpu k-means, which is not available; centroids therefore match
    the reference's only in distribution.)
 3. quantile cutoffs / weights: exact order statistics of all sample residual
    coordinates, ranks floor(q * N) (ResidualScalarQuantizationPack.hpp:
    17-99), found by bisection on the float bit patterns;
 4. assignment of every token + residual packing (libmvr kernels);
 5. doc -> unique-centroid IVF lists, ascending doc ids (IVFIndex.hpp:92-166).
Returns CUDA tensors; `to_host` gives numpy arrays for formats.write_index_dir.
`build_index_stream` runs the same pipeline over a corpus generated (or read)
one doc range at a time, with the tensor-core assignment by default.
"""
import ctypes as C
import math
import random

import numpy as np
import torch

from ._lib import check, lib


def n_centroid_default(n_vec):
    """2^floor(log2(16 * sqrt(n_vec))) (eval_igp_gpu_basic.py:205)."""
    return int(2 ** math.floor(math.log2(16 * math.sqrt(n_vec))))


def sample_items(n_item):
    n = min(1 + int(8 * np.sqrt(120 * n_item)), n_item)
    random.seed(12345)
    return sorted(random.sample(range(n_item), n))


def _p(t):
    return C.c_void_p(t.data_ptr())


def assign(vec, centroid, stream=None):
    code = torch.empty(vec.shape[0], dtype=torch.int32, device=vec.device)
    score = torch.empty(vec.shape[0], dtype=torch.float32, device=vec.device)
    st = C.c_void_p(stream.cuda_stream if stream is not None else torch.cuda.current_stream().cuda_stream)
    check(lib().mvr_assign_device(_p(vec), vec.shape[0], _p(centroid), centroid.shape[0],
                                  centroid.shape[1], _p(code), _p(score), st))
    return code, score


def assign_tc(vec, centroid, stream=None):
    """assign() on the tensor cores (mvr_assign_tc_device): BF16 candidates,
    exact FP32 re-score; for builds over hundreds of millions of vectors."""
    code = torch.empty(vec.shape[0], dtype=torch.int32, device=vec.device)
    score = torch.empty(vec.shape[0], dtype=torch.float32, device=vec.device)
    st = C.c_void_p(stream.cuda_stream if stream is not None else torch.cuda.current_stream().cuda_stream)
    check(lib().mvr_assign_tc_device(_p(vec), vec.shape[0], _p(centroid), centroid.shape[0],
                                     centroid.shape[1], _p(code), _p(score), st))
    return code, score


def _ord_keys(x):
    b = x.contiguous().view(torch.int32).to(torch.int64)
    return torch.where(b < 0, -(b & 0x7FFFFFFF) - 1, b)  # signed-order of floats


def _key_to_float(k):
    k = int(k)
    bits = k if k >= 0 else (-(k + 1)) | 0x80000000
    return np.array([bits & 0xFFFFFFFF], np.uint32).view(np.float32)[0]


def order_statistic(keys, rank):
    """rank-th smallest (0-based) of the signed-order keys, by bisection."""
    lo, hi = int(keys.min()), int(keys.max())
    while lo < hi:
        mid = (lo + hi) // 2
        if int((keys <= mid).sum()) >= rank + 1:
            hi = mid
        else:
            lo = mid + 1
    return _key_to_float(lo)


def quantize_params(err_flat, n_bit):
    keys = _ord_keys(err_flat)
    n = err_flat.numel()
    nq = 1 << n_bit
    cut = [order_statistic(keys, int(math.floor((1.0 * (i + 1) / nq) * n))) for i in range(nq - 1)]
    w = [order_statistic(keys, int(math.floor((1.0 * i / nq + 0.5 / nq) * n))) for i in range(nq)]
    return np.asarray(cut, np.float32), np.asarray(w, np.float32)


def kmeans(sample, n_centroid, n_iter=20, seed=123, assign_fn=assign):
    dev = sample.device
    g = torch.Generator(device=dev).manual_seed(seed)
    idx = torch.randperm(sample.shape[0], device=dev, generator=g)[:n_centroid]
    cen = torch.nn.functional.normalize(sample[idx].clone(), dim=1)
    sums = torch.empty((n_centroid, sample.shape[1]), dtype=torch.float64, device=dev)
    cnt = torch.empty(n_centroid, dtype=torch.int64, device=dev)
    st = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    for _ in range(n_iter):
        code, _ = assign_fn(sample, cen)
        sums.zero_()
        cnt.zero_()
        check(lib().mvr_kmeans_accumulate_device(_p(sample), sample.shape[0], sample.shape[1],
                                                 _p(code), _p(sums), _p(cnt), st))
        nz = cnt > 0
        mean = (sums[nz] / cnt[nz].unsqueeze(1).to(torch.float64)).to(torch.float32)
        cen[nz] = torch.nn.functional.normalize(mean, dim=1)
    return cen.contiguous()


def ivf_build(code, item_n_vec, n_centroid):
    dev = code.device
    n_item = len(item_n_vec)
    doc = torch.repeat_interleave(torch.arange(n_item, device=dev, dtype=torch.int64),
                                  torch.from_numpy(np.asarray(item_n_vec, np.int64)).to(dev))
    key = torch.unique(code.to(torch.int64) * n_item + doc)   # sorted by (centroid, doc)
    cid = key // n_item
    ids = (key % n_item).to(torch.int32)
    size = torch.bincount(cid, minlength=n_centroid).to(torch.int32)
    off = torch.zeros(n_centroid, dtype=torch.int64, device=dev)
    off[1:] = torch.cumsum(size.to(torch.int64), 0)[:-1]
    return off, size, ids


def _doc_offsets(item_n_vec):
    off = np.zeros(len(item_n_vec) + 1, np.int64)
    off[1:] = np.cumsum(np.asarray(item_n_vec, np.int64))
    return off


def train(sample, n_centroid, n_bit, kmeans_iter=20, seed=123, assign_fn=assign):
    """Centroids, quantile cutoffs and bucket weights from the k-means sample."""
    cen = kmeans(sample, n_centroid, kmeans_iter, seed, assign_fn)
    s_code, _ = assign_fn(sample, cen)
    err = (sample - cen[s_code.long()]).reshape(-1)
    cutoff, weight = quantize_params(err, n_bit)
    return cen, cutoff, weight


def encode(tokens, cen, cutoff, n_bit, code_out, residual_out, assign_fn=assign):
    """Codes and packed residuals of `tokens` into the given slices
    (int32 [n], uint8 [n * 128 * n_bit / 8])."""
    code, _ = assign_fn(tokens, cen)
    code_out.copy_(code)
    st = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    cut = np.ascontiguousarray(cutoff, np.float32)
    check(lib().mvr_pack_residual_device(_p(tokens), tokens.shape[0], _p(cen), 128, _p(code_out),
                                         C.c_void_p(cut.ctypes.data), n_bit, _p(residual_out), st))


def _finish(item_n_vec, cen, code, weight, residual, cutoff, n_bit, n_centroid):
    ivf_off, ivf_size, ivf_ids = ivf_build(code, item_n_vec, n_centroid)
    dev = code.device
    return dict(item_n_vec=torch.from_numpy(item_n_vec.view(np.int32)).to(dev),
                centroid=cen, vq_code=code, weight=torch.from_numpy(weight).to(dev),
                residual=residual, ivf_off=ivf_off, ivf_size=ivf_size, ivf_ids=ivf_ids,
                cutoff=cutoff, n_bit=n_bit)


def build_index(tokens, item_n_vec, n_centroid, n_bit, kmeans_iter=20, seed=123,
                assign_fn=assign):
    """tokens: CUDA float32 [n_vec, 128]; item_n_vec: numpy uint32 [n_item]."""
    assert tokens.is_cuda and tokens.dtype == torch.float32 and tokens.shape[1] == 128
    item_n_vec = np.asarray(item_n_vec, np.uint32)
    off = _doc_offsets(item_n_vec)
    pids = np.asarray(sample_items(len(item_n_vec)), np.int64)
    tok_idx = np.concatenate([np.arange(off[p], off[p + 1]) for p in pids])
    sample = tokens[torch.from_numpy(tok_idx).to(tokens.device)].contiguous()
    cen, cutoff, weight = train(sample, n_centroid, n_bit, kmeans_iter, seed, assign_fn)
    del sample
    n = tokens.shape[0]
    code = torch.empty(n, dtype=torch.int32, device=tokens.device)
    residual = torch.empty(n * (128 * n_bit // 8), dtype=torch.uint8, device=tokens.device)
    encode(tokens, cen, cutoff, n_bit, code, residual, assign_fn)
    return _finish(item_n_vec, cen, code, weight, residual, cutoff, n_bit, n_centroid)


def build_index_stream(spec, n_centroid, n_bit, kmeans_iter=20, seed=123, device="cuda",
                       chunk_docs=1 << 17, assign_fn=assign_tc, tokens_fn=None):
    """build_index over a corpus that is never resident as a whole: the
    tokens of doc range [d0, d1) come from tokens_fn(spec, d0, d1, device)
    (default: synth.tokens_range, the block-keyed synthetic stream), one
    range of chunk_docs docs at a time -- once to gather the k-means sample,
    once to encode.  Only the compressed index and the sample stay on the
    device, so corpora of hundreds of millions of tokens fit.  With the same
    tokens and assign_fn the result equals build_index's."""
    from . import synth
    if tokens_fn is None:
        tokens_fn = synth.tokens_range
    item_n_vec = np.asarray(spec.item_n_vec, np.uint32)
    n_item = len(item_n_vec)
    off = _doc_offsets(item_n_vec)
    pids = np.asarray(sample_items(n_item), np.int64)
    ranges = [(d0, min(n_item, d0 + chunk_docs)) for d0 in range(0, n_item, chunk_docs)]
    parts = []
    for d0, d1 in ranges:
        p = pids[(pids >= d0) & (pids < d1)]
        if len(p) == 0:
            continue
        tok = tokens_fn(spec, d0, d1, device)
        idx = np.concatenate([np.arange(off[i], off[i + 1]) for i in p]) - off[d0]
        parts.append(tok[torch.from_numpy(idx).to(tok.device)])
        del tok
    sample = torch.cat(parts).contiguous()
    del parts
    cen, cutoff, weight = train(sample, n_centroid, n_bit, kmeans_iter, seed, assign_fn)
    del sample
    torch.cuda.empty_cache()
    n = int(off[-1])
    bpv = 128 * n_bit // 8
    code = torch.empty(n, dtype=torch.int32, device=device)
    residual = torch.empty(n * bpv, dtype=torch.uint8, device=device)
    for d0, d1 in ranges:
        t0, t1 = int(off[d0]), int(off[d1])
        tok = tokens_fn(spec, d0, d1, device)
        encode(tok, cen, cutoff, n_bit, code[t0:t1], residual[t0 * bpv:t1 * bpv], assign_fn)
        del tok
    return _finish(item_n_vec, cen, code, weight, residual, cutoff, n_bit, n_centroid)


def to_host(ix):
    return dict(item_n_vec=ix["item_n_vec"].cpu().numpy().view(np.uint32),
                centroid=ix["centroid"].cpu().numpy(),
                vq_code=ix["vq_code"].cpu().numpy().view(np.uint32),
                weight=ix["weight"].cpu().numpy(), residual=ix["residual"].cpu().numpy(),
                ivf_off=ix["ivf_off"].cpu().numpy().view(np.uint64),
                ivf_size=ix["ivf_size"].cpu().numpy().view(np.uint32),
                ivf_ids=ix["ivf_ids"].cpu().numpy().view(np.uint32), n_bit=ix["n_bit"])


def load_built(ix, device=0):
    """Index handle from a build_index result (device-to-device copy)."""
    from .index import Index
    return Index.from_device_arrays(ix["item_n_vec"], ix["centroid"], ix["vq_code"], ix["ivf_off"],
                                    ix["ivf_size"], ix["ivf_ids"], ix["weight"], ix["n_bit"],
                                    ix["residual"], device)
