"""Seeded synthetic clustered ColBERT-like corpora (stand-in for the
reference's LoTTE / MS MARCO / HotpotQA / Wikipedia embeddings, which are not
available here).

Generator: n_latent cluster means uniform on the unit sphere S^127; each doc
draws 5..15 of them; doc lengths ~ lognormal with mean 70 / sd 35, rounded and
clipped to [8, 180]; token = normalize(mu_c + 0.45 * N(0, I)) with c one of the
doc's clusters; a query token = normalize(mu_c + 0.55 * N(0, I)) with c one of
a random doc's clusters.  The noise vector is N(0, I/128) scaled by 0.45
(0.55): its expected norm is 0.45 (0.55), so a token keeps cos ~0.91 (~0.87)
with its cluster mean.  (Per-dimension unit variance would give a noise norm
of ~5.1 and cos ~0.19 with the mean, under which exact-MaxSim rankings are
noise-dominated and no IVF method reaches meaningful recall.)  torch RNG on
the requested device (CPU and CUDA streams differ but each is deterministic
for a seed).
"""
import math

import numpy as np
import torch

DIM = 128
LEN_MEAN, LEN_SD = 70.0, 35.0
LN_SIGMA = math.sqrt(math.log(1.0 + (LEN_SD / LEN_MEAN) ** 2))
LN_MU = math.log(LEN_MEAN) - LN_SIGMA ** 2 / 2


class CorpusSpec:
    def __init__(self, n_doc, seed=0, n_latent=20000, len_lo=8, len_hi=180, k_lo=5, k_hi=15):
        g = np.random.default_rng(seed)
        self.n_doc = n_doc
        self.seed = seed
        lens = np.rint(g.lognormal(LN_MU, LN_SIGMA, n_doc))
        self.item_n_vec = np.clip(lens, len_lo, len_hi).astype(np.uint32)
        self.doc_k = g.integers(k_lo, k_hi + 1, n_doc).astype(np.int64)
        self.doc_clusters = g.integers(0, n_latent, (n_doc, k_hi)).astype(np.int64)
        mu = g.standard_normal((n_latent, DIM)).astype(np.float32)
        self.latent = mu / np.linalg.norm(mu, axis=1, keepdims=True)
        self.item_off = np.zeros(n_doc, np.uint64)
        self.item_off[1:] = np.cumsum(self.item_n_vec[:-1], dtype=np.uint64)

    @property
    def n_vec(self):
        return int(self.item_n_vec.sum())


def _normalize_(x):
    x /= torch.linalg.vector_norm(x, dim=1, keepdim=True)
    return x


def tokens(spec, device="cpu", noise=0.45, chunk=1 << 22, out=None):
    """All doc tokens, float32 [n_vec, 128] on `device`, generated in chunks."""
    dev = torch.device(device)
    gen = torch.Generator(device=dev).manual_seed(spec.seed * 1000003 + 17)
    n_vec = spec.n_vec
    if out is None:
        out = torch.empty((n_vec, DIM), dtype=torch.float32, device=dev)
    latent = torch.from_numpy(spec.latent).to(dev)
    doc_k = torch.from_numpy(spec.doc_k).to(dev)
    clusters = torch.from_numpy(spec.doc_clusters).to(dev)
    lens = torch.from_numpy(spec.item_n_vec.astype(np.int64)).to(dev)
    doc_of = torch.repeat_interleave(torch.arange(spec.n_doc, device=dev), lens)
    for s in range(0, n_vec, chunk):
        e = min(n_vec, s + chunk)
        d = doc_of[s:e]
        slot = (torch.rand(e - s, device=dev, generator=gen) * doc_k[d]).long().clamp_max_(14)
        c = clusters[d, slot]
        x = latent[c] + (noise / math.sqrt(DIM)) * torch.randn((e - s, DIM), device=dev,
                                                              generator=gen)
        out[s:e] = _normalize_(x)
    return out


BLOCK_DOCS = 1 << 15  # docs per generator block of the block-keyed token stream


def n_vec_range(spec, d0, d1):
    return int(spec.item_n_vec[d0:d1].sum(dtype=np.int64))


def _block_tokens(spec, k, dev, noise):
    """Tokens of doc block k (docs [k * BLOCK_DOCS, (k + 1) * BLOCK_DOCS)) from
    the block's own generator."""
    d0 = k * BLOCK_DOCS
    d1 = min(spec.n_doc, d0 + BLOCK_DOCS)
    gen = torch.Generator(device=dev).manual_seed(spec.seed * 1000003 + 104729 * (k + 1))
    lens = torch.from_numpy(spec.item_n_vec[d0:d1].astype(np.int64)).to(dev)
    doc_of = torch.repeat_interleave(torch.arange(d1 - d0, device=dev), lens)
    n = doc_of.shape[0]
    doc_k = torch.from_numpy(spec.doc_k[d0:d1]).to(dev)
    clusters = torch.from_numpy(spec.doc_clusters[d0:d1]).to(dev)
    k_max = spec.doc_clusters.shape[1] - 1
    slot = (torch.rand(n, device=dev, generator=gen) * doc_k[doc_of]).long().clamp_max_(k_max)
    latent = torch.from_numpy(spec.latent).to(dev)
    x = latent[clusters[doc_of, slot]]
    x += (noise / math.sqrt(DIM)) * torch.randn((n, DIM), device=dev, generator=gen)
    return _normalize_(x)


def tokens_range(spec, d0, d1, device="cpu", noise=0.45):
    """Tokens of docs [d0, d1), float32 [n_vec_range(spec, d0, d1), 128], from
    the block-keyed stream: every block of BLOCK_DOCS docs draws from its own
    generator, so any doc range is generated without the docs before it and
    corpora far larger than device memory can be built and scanned in
    pieces.  (A different stream from `tokens`, which draws the whole corpus
    from one generator; same distribution.)"""
    dev = torch.device(device)
    parts = []
    k_end = (d1 + BLOCK_DOCS - 1) // BLOCK_DOCS if d1 > d0 else 0
    for k in range(d0 // BLOCK_DOCS, k_end):
        b0 = k * BLOCK_DOCS
        x = _block_tokens(spec, k, dev, noise)
        s = n_vec_range(spec, b0, max(d0, b0))
        e = n_vec_range(spec, b0, min(d1, b0 + BLOCK_DOCS))
        parts.append(x[s:e])
    if not parts:
        return torch.empty((0, DIM), dtype=torch.float32, device=dev)
    return parts[0] if len(parts) == 1 else torch.cat(parts)


def doc_chunks(spec, max_tokens):
    """[d0, d1) ranges covering the corpus, each <= max_tokens tokens (one
    doc may exceed it alone)."""
    off = np.zeros(spec.n_doc + 1, np.int64)
    off[1:] = np.cumsum(spec.item_n_vec, dtype=np.int64)
    out, d0 = [], 0
    while d0 < spec.n_doc:
        d1 = int(np.searchsorted(off, off[d0] + max_tokens, side="right")) - 1
        d1 = min(spec.n_doc, max(d1, d0 + 1))
        out.append((d0, d1))
        d0 = d1
    return out


def queries(spec, n_query, n_tok=32, device="cpu", noise=0.55, seed=1):
    """Queries built from random docs' clusters.  n_tok: int; a tuple (lo, hi)
    for ragged queries (token counts uniform in [lo, hi]); or a list of token
    counts drawn with equal probability.  Returns (float32 [total_tokens, 128]
    tensor, uint64 token offsets [n_query+1])."""
    g = np.random.default_rng(seed + 7919 * spec.seed)
    if isinstance(n_tok, list):
        counts = g.choice(np.asarray(n_tok), n_query)
    elif isinstance(n_tok, tuple):
        counts = g.integers(n_tok[0], n_tok[1] + 1, n_query)
    else:
        counts = np.full(n_query, n_tok)
    off = np.zeros(n_query + 1, np.uint64)
    off[1:] = np.cumsum(counts)
    docs = g.integers(0, spec.n_doc, n_query)
    cl = []
    for i in range(n_query):
        k = spec.doc_k[docs[i]]
        cl.append(spec.doc_clusters[docs[i], g.integers(0, k, counts[i])])
    cl = np.concatenate(cl)
    dev = torch.device(device)
    gen = torch.Generator(device=dev).manual_seed(seed * 7 + spec.seed)
    x = torch.from_numpy(spec.latent[cl]).to(dev)
    x = x + (noise / math.sqrt(DIM)) * torch.randn(x.shape, device=dev, generator=gen)
    return _normalize_(x).contiguous(), off
