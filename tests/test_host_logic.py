"""Host-side logic on the CPU: synthetic generator statistics, the GPU
builder's pure-host helpers (sample selection, centroid-count formula, exact
order statistics by bisection, IVF build), and the exhaustive ground truth
(torch, CPU tensors here) against the oracle's FP64 exhaustive MaxSim."""
import numpy as np
import torch

import pyoracle
from helpers import tiny_index
from mvr import build, exhaustive, synth


def test_generator_shapes_and_stats():
    spec = synth.CorpusSpec(2000, seed=3)
    assert spec.item_n_vec.min() >= 8 and spec.item_n_vec.max() <= 180
    assert 60 < spec.item_n_vec.mean() < 80
    tok = synth.tokens(spec, "cpu")
    assert tok.shape == (spec.n_vec, 128)
    np.testing.assert_allclose(torch.linalg.vector_norm(tok, dim=1).numpy(), 1.0, atol=1e-5)
    q, off = synth.queries(spec, 10, (8, 32), "cpu", seed=2)
    assert len(off) == 11 and q.shape[0] == off[-1]
    assert all(8 <= d <= 32 for d in np.diff(off))
    tok2 = synth.tokens(spec, "cpu")
    assert torch.equal(tok, tok2)  # deterministic


def test_sample_and_centroid_formula():
    assert build.n_centroid_default(700_000) == 8192
    assert build.n_centroid_default(70_000_000) == 131072
    s = build.sample_items(10_000)
    assert len(s) == min(1 + int(8 * np.sqrt(120 * 10_000)), 10_000)
    assert s == sorted(set(s))


def test_order_statistics_exact():
    rng = np.random.default_rng(0)
    x = rng.standard_normal(100_001).astype(np.float32)
    x[::7] = 0.25  # ties
    x[::11] = -0.0
    keys = build._ord_keys(torch.from_numpy(x))
    srt = np.sort(x)
    for r in (0, 1, 500, 50_000, 99_999, 100_000):
        assert build.order_statistic(keys, r) == srt[r]
    cut, w = build.quantize_params(torch.from_numpy(x), 2)
    nq = 4
    np.testing.assert_array_equal(cut, [srt[int(np.floor((i + 1) / nq * len(x)))] for i in range(3)])


def test_ivf_build_torch_matches_oracle():
    ix = tiny_index(n_doc=150, n_centroid=50, seed=2)
    off, size, ids = build.ivf_build(torch.from_numpy(ix["vq_code"].astype(np.int32)),
                                     ix["item_n_vec"], 50)
    np.testing.assert_array_equal(off.numpy(), ix["ivf_off"])
    np.testing.assert_array_equal(size.numpy(), ix["ivf_size"])
    np.testing.assert_array_equal(ids.numpy().view(np.uint32), ix["ivf_ids"])


def test_exhaustive_topk_matches_oracle_f64():
    ix = tiny_index(n_doc=120, n_centroid=16, seed=4)
    q, off = synth.queries(ix["spec"], 3, 12, "cpu", seed=9)
    s, i = exhaustive.exhaustive_topk(q, off, torch.from_numpy(ix["tokens"]), ix["item_n_vec"], 7,
                                      chunk_tokens=300)
    rs, ri = pyoracle.exhaustive_f64(q.numpy(), off, ix["tokens"], ix["item_n_vec"], 7)
    np.testing.assert_array_equal(i, ri)
    np.testing.assert_allclose(s, rs, rtol=1e-12)


def test_block_keyed_tokens_any_range():
    """tokens_range: any doc range equals the matching slice of the whole
    corpus (each block of docs has its own generator), across block edges."""
    old = synth.BLOCK_DOCS
    synth.BLOCK_DOCS = 500
    try:
        spec = synth.CorpusSpec(1700, seed=6, n_latent=300)
        full = synth.tokens_range(spec, 0, spec.n_doc)
        assert full.shape == (spec.n_vec, 128)
        assert torch.allclose(torch.linalg.vector_norm(full, dim=1), torch.ones(spec.n_vec))
        for d0, d1 in ((0, 1), (499, 501), (500, 1000), (1234, 1700), (1699, 1700), (7, 7)):
            t0, t1 = synth.n_vec_range(spec, 0, d0), synth.n_vec_range(spec, 0, d1)
            assert torch.equal(synth.tokens_range(spec, d0, d1), full[t0:t1])
        ch = synth.doc_chunks(spec, 10_000)
        assert ch[0][0] == 0 and ch[-1][1] == spec.n_doc
        assert all(a[1] == b[0] for a, b in zip(ch, ch[1:]))
        assert all(synth.n_vec_range(spec, a, b) <= 10_000 for a, b in ch)
    finally:
        synth.BLOCK_DOCS = old


def test_exhaustive_stream_equals_whole_corpus():
    """exhaustive_topk_stream over doc pieces (the way corpora larger than the
    device are scanned) gives the whole-corpus top-k, ties by lower id."""
    ix = tiny_index(n_doc=300, n_centroid=16, seed=8)
    q, off = synth.queries(ix["spec"], 4, (3, 20), "cpu", seed=2)
    tok = torch.from_numpy(ix["tokens"])
    lens = ix["item_n_vec"].astype(np.int64)
    s, i = exhaustive.exhaustive_topk(q, off, tok, ix["item_n_vec"], 9)
    toff = np.concatenate([[0], np.cumsum(lens)])
    for cut in ((0, 300), (0, 1, 150, 151, 300), (0, 97, 203, 300)):
        chunks = ((a, lens[a:b], tok[toff[a]:toff[b]]) for a, b in zip(cut, cut[1:]))
        s2, i2 = exhaustive.exhaustive_topk_stream(q, off, chunks, 9)
        np.testing.assert_array_equal(i2, i)
        np.testing.assert_allclose(s2, s, rtol=1e-12)
    # duplicated docs: equal scores keep the lower id across pieces
    dup = torch.cat([tok[toff[5]:toff[6]], tok[toff[5]:toff[6]]])
    l2 = np.array([lens[5], lens[5]])
    _, idup = exhaustive.exhaustive_topk_stream(q, off, [(0, l2[:1], dup[:lens[5]]),
                                                         (1, l2[1:], dup[lens[5]:])], 2)
    assert (idup == np.array([0, 1])).all()



def test_bench_ground_truth_pieces_cover_the_corpus():
    """bench.gt_chunks: consecutive doc pieces, each within its generator
    block and the score-matrix budget, whose tokens are the corpus's."""
    import importlib.util
    import os
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    spec_b = importlib.util.spec_from_file_location("bench_mod", os.path.join(root, "bench.py"))
    bench = importlib.util.module_from_spec(spec_b)
    spec_b.loader.exec_module(bench)
    old = synth.BLOCK_DOCS
    synth.BLOCK_DOCS = 400
    try:
        spec = synth.CorpusSpec(1000, seed=2, n_latent=100)
        full = synth.tokens_range(spec, 0, spec.n_doc)
        pieces = list(bench.gt_chunks(spec, lambda a, b: synth.tokens_range(spec, a, b),
                                      n_q_tok=2_000_000))  # budget -> 16,384-token floor
        d, t = 0, 0
        for d0, lens, x in pieces:
            assert d0 == d and x.shape[0] == int(lens.sum())
            assert d0 // 400 == (d0 + len(lens) - 1) // 400      # within one block
            assert x.shape[0] <= 16_384 or len(lens) == 1
            assert torch.equal(x, full[t:t + x.shape[0]])
            d += len(lens)
            t += x.shape[0]
        assert d == spec.n_doc and t == spec.n_vec
    finally:
        synth.BLOCK_DOCS = old


def test_bench_reference_arm_declines_streamed_workloads():
    """bench.py --impl reference on a streamed workload prints its
    `unavailable` line (the CPU port needs the whole index in host memory)
    without touching a GPU."""
    import json
    import os
    import subprocess
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    for wl in ("large", "xl"):
        out = subprocess.run([sys.executable, os.path.join(root, "bench.py"), "--impl",
                              "reference", "--workload", wl], capture_output=True, text=True,
                             timeout=120, check=True).stdout.strip().splitlines()[-1]
        line = json.loads(out)
        assert line["impl"] == "reference" and "unavailable" in line


def test_exhaustive_stream_fp32_screen_matches_fp64():
    """The FP32 variant of the piecewise ground truth (bench --gt-dtype f32)
    ranks like FP64 on a corpus without near-ties."""
    ix = tiny_index(n_doc=250, n_centroid=16, seed=12)
    q, off = synth.queries(ix["spec"], 5, 24, "cpu", seed=3)
    tok = torch.from_numpy(ix["tokens"])
    lens = ix["item_n_vec"].astype(np.int64)
    toff = np.concatenate([[0], np.cumsum(lens)])
    cuts = (0, 90, 250)

    def pieces():
        return ((a, lens[a:b], tok[toff[a]:toff[b]]) for a, b in zip(cuts, cuts[1:]))
    s64, i64 = exhaustive.exhaustive_topk_stream(q, off, pieces(), 10)
    s32, i32 = exhaustive.exhaustive_topk_stream(q, off, pieces(), 10, dtype=torch.float32)
    np.testing.assert_array_equal(i32, i64)
    np.testing.assert_allclose(s32, s64, rtol=1e-5)

