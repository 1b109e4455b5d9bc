"""Shared test fixtures: tiny indexes built on the CPU with the oracle's
codec functions (the reference's build semantics), and comparison helpers."""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (os.path.join(ROOT, "oracle"), os.path.join(ROOT, "multi-vector-retrieval-gpu_b200")):
    if p not in sys.path:
        sys.path.insert(0, p)

import pyoracle  # noqa: E402
from mvr import synth  # noqa: E402


def tiny_index(n_doc=300, n_centroid=64, n_bit=2, seed=0, len_hi=180, n_latent=200, lengths=None):
    spec = synth.CorpusSpec(n_doc, seed=seed, n_latent=n_latent, len_hi=len_hi)
    if lengths is not None:  # explicit doc lengths (edge cases)
        spec.item_n_vec = np.asarray(lengths, np.uint32)
        spec.item_off = np.zeros(n_doc, np.uint64)
        spec.item_off[1:] = np.cumsum(spec.item_n_vec[:-1], dtype=np.uint64)
    tok = synth.tokens(spec, "cpu").numpy()
    rng = np.random.default_rng(seed + 5)
    cen = tok[rng.choice(len(tok), n_centroid, replace=False)]
    cen = cen + 0.05 * rng.standard_normal(cen.shape).astype(np.float32)
    cen = (cen / np.linalg.norm(cen, axis=1, keepdims=True)).astype(np.float32)
    code = pyoracle.assign(tok, cen)
    cut, w = pyoracle.quantize(tok, cen, code, n_bit)
    res = pyoracle.pack_residual(tok, cen, code, cut, n_bit)
    off, size, ids = pyoracle.ivf_build(code, spec.item_n_vec, n_centroid)
    return dict(spec=spec, tokens=tok, item_n_vec=spec.item_n_vec, centroid=cen, vq_code=code,
                cutoff=cut, weight=w, residual=res, ivf_off=off, ivf_size=size, ivf_ids=ids,
                n_bit=n_bit)


def oracle_of(ix):
    return pyoracle.Oracle(ix["item_n_vec"], ix["centroid"], ix["vq_code"], ix["residual"],
                           ix["weight"], ix["ivf_off"], ix["ivf_size"], ix["ivf_ids"], ix["n_bit"])


def make_queries(ix, n_query, n_tok=32, seed=1):
    q, off = synth.queries(ix["spec"], n_query, n_tok, "cpu", seed=seed)
    return q.numpy(), off


def assert_same_topk(a_ids, a_s, b_ids, b_s):
    np.testing.assert_array_equal(a_ids, b_ids)
    np.testing.assert_array_equal(a_s, b_s)
