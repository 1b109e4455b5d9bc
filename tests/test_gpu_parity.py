"""CUDA path vs the oracle, through the C ABI: probed centroid ids, candidate
sets, approximate scores, shortlists, decompressed vectors / bucket indices,
exact MaxSim scores and final top-k are all compared bit-for-bit (the path's
canonical FP32 arithmetic is specified in oracle/mvr_oracle.h); FP32 exact
scores are additionally checked within 1e-5 relative of FP64."""
import glob
import os

import numpy as np
import pytest

import pyoracle
from helpers import make_queries, oracle_of, tiny_index
from mvr import SEM_BASIC, SEM_PP, Index, MvrError, _lib

pytestmark = pytest.mark.gpu
TOL = 1e-5
GOLDEN = sorted(glob.glob(os.path.join(os.path.dirname(__file__), "golden", "codec_*d128.npz")))


def with_orphan_centroids(ix, n_orphan):
    """Appends centroids that no token is closest to (negated copies), so
    their IVF lists are empty, and rebuilds codes / residuals / lists."""
    cen = np.concatenate([ix["centroid"], -ix["centroid"][np.arange(n_orphan) % len(ix["centroid"])]])
    code = pyoracle.assign(ix["tokens"], cen)
    cut, w = pyoracle.quantize(ix["tokens"], cen, code, ix["n_bit"])
    res = pyoracle.pack_residual(ix["tokens"], cen, code, cut, ix["n_bit"])
    off, size, ids = pyoracle.ivf_build(code, ix["item_n_vec"], len(cen))
    return dict(ix, centroid=cen, vq_code=code, weight=w, residual=res, ivf_off=off,
                ivf_size=size, ivf_ids=ids)


def gpu_index(ix):
    return Index.from_arrays(ix["item_n_vec"], ix["centroid"], ix["vq_code"], ix["ivf_off"],
                             ix["ivf_size"], ix["ivf_ids"], ix["weight"], ix["n_bit"],
                             ix["residual"])


@pytest.fixture(scope="module", params=[1, 2, 4, 8], ids=lambda b: f"b{b}")
def pair(request):
    ix = tiny_index(n_doc=400, n_centroid=96, n_bit=request.param, seed=request.param)
    g = gpu_index(ix)
    yield ix, g, oracle_of(ix)
    g.close()


@pytest.mark.parametrize("path", GOLDEN, ids=[os.path.basename(p)[6:-4] for p in GOLDEN])
def test_decode_matches_reference_golden(path):
    c = np.load(path)
    g = Index.from_arrays(c["item_n_vec"], c["centroid"], c["code"], c["ivf_off"], c["ivf_size"],
                          c["ivf_ids"], c["weight"], int(c["n_bit"]), c["residual"])
    ids = np.arange(len(c["code"]), dtype=np.uint64)
    np.testing.assert_array_equal(g.decompress(ids), c["decoded"])
    np.testing.assert_array_equal(
        g.unpack_buckets(ids),
        pyoracle.unpack_buckets(c["residual"], len(c["code"]), 128, int(c["n_bit"])))
    g.close()


def compare_trace(t, r):
    np.testing.assert_array_equal(t["probe_id"], r["probe_id"])
    np.testing.assert_array_equal(t["probe_score"], r["probe_score"])
    np.testing.assert_array_equal(t["cand_id"], r["cand_id"])
    np.testing.assert_array_equal(t["cand_score"], r["cand_score"])
    o = np.argsort(r["short_id"])
    np.testing.assert_array_equal(t["short_id"], r["short_id"][o])
    np.testing.assert_array_equal(t["short_approx"], r["short_approx"][o])
    np.testing.assert_array_equal(t["short_exact"], r["short_exact"][o])
    np.testing.assert_array_equal(t["id"], r["id"])
    np.testing.assert_array_equal(t["score"], r["score"])


@pytest.mark.parametrize("sem", [SEM_PP, SEM_BASIC], ids=["pp", "basic"])
def test_stage_trace_bit_exact(pair, sem):
    ix, g, o = pair
    q, off = make_queries(ix, 4, 32, seed=21)
    for i in range(4):
        qi = q[off[i]:off[i + 1]]
        for nprobe, ptk, k in ((4, 100, 10), (8, 300, 100)):
            compare_trace(g.trace(qi, k, nprobe, ptk, sem), o.search_one(qi, k, nprobe, ptk, sem))


def test_batched_ragged_search_bit_exact(pair):
    ix, g, o = pair
    q, off = make_queries(ix, 37, (1, 64), seed=5)
    g.set_batch(8)  # several batches incl. a partial one
    s, i, st = g.search(q, 10, 6, 120, tok_off=off, with_stats=True)
    g.set_batch(0)
    rs, ri = o.search(q, off, 10, 6, 120)
    np.testing.assert_array_equal(i, ri)
    np.testing.assert_array_equal(s, rs)
    assert st["n_batch"] == 5 and st["gpu_launches"] >= 4 * 5


def test_uniform_and_device_entry_points_agree(pair):
    import torch
    ix, g, o = pair
    q, off = make_queries(ix, 12, 32, seed=8)
    s1, i1 = g.search(q.reshape(12, 32, 128), 10, 4, 100)
    dq = torch.from_numpy(q).cuda()
    ds = torch.empty((12, 10), dtype=torch.float32, device="cuda")
    di = torch.empty((12, 10), dtype=torch.int32, device="cuda")
    st = g.search_device(dq.data_ptr(), None, 12, 32, 10, 4, 100, ds.data_ptr(), di.data_ptr())
    np.testing.assert_array_equal(ds.cpu().numpy(), s1)
    np.testing.assert_array_equal(di.cpu().numpy().view(np.uint32), i1)
    assert st.h2d_bytes < 4096 and st.d2h_bytes == 0


def test_exact_scores_within_fp64_tolerance(pair):
    ix, g, o = pair
    q, off = make_queries(ix, 3, 32, seed=9)
    dec = o.decompress_all().astype(np.float64)
    toff = np.concatenate([[0], np.cumsum(ix["item_n_vec"].astype(np.int64))])
    for k in range(3):
        qi = q[off[k]:off[k + 1]]
        t = g.trace(qi, 10, 4, 100)
        for d, s in zip(t["short_id"], t["short_exact"]):
            ref = (qi.astype(np.float64) @ dec[toff[d]:toff[d + 1]].T).max(1).sum()
            assert abs(s - ref) <= TOL * abs(ref), (d, s, ref)


def test_edge_cases():
    lens = np.random.default_rng(3).integers(1, 13, 60)
    lens[:3] = 1  # single-token docs
    ix = tiny_index(n_doc=60, n_centroid=40, n_bit=2, seed=7, lengths=lens)
    g, o = gpu_index(ix), oracle_of(ix)
    assert ix["item_n_vec"].min() == 1
    q, off = make_queries(ix, 3, 64, seed=3)
    cases = [dict(k=5, nprobe=32, ptk=5),       # nprobe = max, topk = probe_topk
             dict(k=10, nprobe=1, ptk=8000),    # shortlist larger than candidate set
             dict(k=60, nprobe=2, ptk=60)]      # topk beyond candidates -> padded tail
    for c in cases:
        for i in range(3):
            qi = q[off[i]:off[i + 1]]
            for nq in (1, 7, 64):
                compare_trace(g.trace(qi[:nq], c["k"], c["nprobe"], c["ptk"]),
                              o.search_one(qi[:nq], c["k"], c["nprobe"], c["ptk"]))
    r = g.trace(q[:4], 60, 1, 60)
    pad = r["id"] == 0xFFFFFFFF
    assert np.all(np.isneginf(r["score"][pad]))
    g.close()
    # 80 orphan centroids own no token: empty IVF lists get probed
    ix2 = with_orphan_centroids(tiny_index(n_doc=60, n_centroid=20, n_bit=4, seed=8,
                                           lengths=lens), 80)
    assert (ix2["ivf_size"] == 0).sum() >= 40
    g2, o2 = gpu_index(ix2), oracle_of(ix2)
    for i in range(3):
        qi = q[off[i]:off[i + 1]]
        compare_trace(g2.trace(qi, 10, 32, 40), o2.search_one(qi, 10, 32, 40))
    g2.close()


def test_invalid_arguments_rejected(pair):
    ix, g, o = pair
    q = np.zeros((1, 32, 128), np.float32)
    bad = [dict(k=10, nprobe=4, ptk=5), dict(k=10, nprobe=0, ptk=50),
           dict(k=10, nprobe=10_000, ptk=50), dict(k=2000, nprobe=4, ptk=4000),
           dict(k=10, nprobe=4, ptk=9000)]
    for b in bad:
        with pytest.raises(MvrError) as e:
            g.search(q, b["k"], b["nprobe"], b["ptk"])
        assert e.value.code in (_lib.MVR_ERR_INVALID_ARG, _lib.MVR_ERR_UNSUPPORTED)
    with pytest.raises(MvrError):
        g.search(np.zeros((1, 65, 128), np.float32), 10, 4, 50)
    with pytest.raises(MvrError):
        g.search(np.zeros((2, 128), np.float32), 10, 4, 50, tok_off=np.array([0, 2, 1], np.uint64))


def test_gpu_builder_matches_oracle_codec():
    import torch
    from mvr import build, synth
    spec = synth.CorpusSpec(800, seed=4, n_latent=300)
    tok = synth.tokens(spec, "cuda")
    ix = build.build_index(tok, spec.item_n_vec, 128, 2, kmeans_iter=3)
    h = build.to_host(ix)
    tn = tok.cpu().numpy()
    np.testing.assert_array_equal(h["vq_code"], pyoracle.assign(tn, h["centroid"]))
    np.testing.assert_array_equal(
        h["residual"], pyoracle.pack_residual(tn, h["centroid"], h["vq_code"], ix["cutoff"], 2))
    off, size, ids = pyoracle.ivf_build(h["vq_code"], spec.item_n_vec, 128)
    np.testing.assert_array_equal(h["ivf_off"], off)
    np.testing.assert_array_equal(h["ivf_size"], size)
    np.testing.assert_array_equal(h["ivf_ids"], ids)
    # quantile parameters: exact order statistics of the k-means sample residuals
    pids = build.sample_items(len(spec.item_n_vec))
    toff = np.concatenate([[0], np.cumsum(spec.item_n_vec.astype(np.int64))])
    sidx = np.concatenate([np.arange(toff[p], toff[p + 1]) for p in pids])
    samp = tn[sidx]
    cut, w = pyoracle.quantize(samp, h["centroid"], pyoracle.assign(samp, h["centroid"]), 2)
    np.testing.assert_array_equal(ix["cutoff"], cut)
    np.testing.assert_array_equal(h["weight"], w)
    g = build.load_built(ix)
    assert g.info()["n_vec"] == len(tn)
    g.close()
    del tok
    torch.cuda.empty_cache()


def test_streaming_builder_and_tensor_core_assignment():
    """build_index_stream generates and encodes the corpus one doc range at a
    time (ranges not aligned with the generator's blocks); with the same
    tokens and the FP32 assignment it equals build_index over the resident
    corpus, array for array.  The tensor-core assignment
    (mvr_assign_tc_device) returns the FP32 argmax for nearly every vector
    and the exact FP32 score wherever the codes agree; an index streamed with
    it searches bit-exactly like the oracle on the same arrays."""
    import torch
    from mvr import build, synth
    old = synth.BLOCK_DOCS
    synth.BLOCK_DOCS = 1000
    try:
        spec = synth.CorpusSpec(5000, seed=5, n_latent=400)
        tok = synth.tokens_range(spec, 0, spec.n_doc, "cuda")
        a = build.build_index(tok, spec.item_n_vec, 256, 2, kmeans_iter=2)
        b = build.build_index_stream(spec, 256, 2, kmeans_iter=2, chunk_docs=1500,
                                     assign_fn=build.assign)
        for key in ("centroid", "vq_code", "weight", "residual", "ivf_off", "ivf_size", "ivf_ids"):
            assert torch.equal(a[key], b[key]), key
        np.testing.assert_array_equal(a["cutoff"], b["cutoff"])
        c32, s32 = build.assign(tok, a["centroid"])
        ctc, stc = build.assign_tc(tok, a["centroid"])
        agree = c32 == ctc
        assert agree.float().mean().item() > 0.999
        assert torch.equal(s32[agree], stc[agree])
        assert bool((stc[~agree] <= s32[~agree]).all())
        del tok
        c = build.build_index_stream(spec, 256, 2, kmeans_iter=2, chunk_docs=1500)
        g, h = build.load_built(c), build.to_host(c)
        o = pyoracle.Oracle(h["item_n_vec"], h["centroid"], h["vq_code"], h["residual"],
                            h["weight"], h["ivf_off"], h["ivf_size"], h["ivf_ids"], 2)
        q, off = synth.queries(spec, 6, 32, "cpu", seed=4)
        q = q.numpy()
        s, i = g.search(q.reshape(6, 32, 128), 10, 4, 150)
        rs, ri = o.search(q, off, 10, 4, 150)
        np.testing.assert_array_equal(i, ri)
        np.testing.assert_array_equal(s, rs)
        g.close()
    finally:
        synth.BLOCK_DOCS = old
        torch.cuda.empty_cache()


def test_config1_scale_gpu_built_index_bit_exact():
    """10,000 docs / 8,192 centroids / nbits 2 (the small synthetic config),
    built on the GPU; 16 queries x (nprobe 4, k 10 and 100) vs the oracle."""
    import torch
    from mvr import build, synth
    spec = synth.CorpusSpec(10_000, seed=1)
    tok = synth.tokens(spec, "cuda")
    ix = build.build_index(tok, spec.item_n_vec, 8192, 2, kmeans_iter=2)
    g = build.load_built(ix)
    h = build.to_host(ix)
    o = pyoracle.Oracle(h["item_n_vec"], h["centroid"], h["vq_code"], h["residual"], h["weight"],
                        h["ivf_off"], h["ivf_size"], h["ivf_ids"], 2)
    q, off = synth.queries(spec, 16, 32, "cpu", seed=3)
    q = q.numpy()
    for k, ptk in ((10, 200), (100, 1000)):
        s, i = g.search(q.reshape(16, 32, 128), k, 4, ptk)
        rs, ri = o.search(q, off, k, 4, ptk)
        np.testing.assert_array_equal(i, ri)
        np.testing.assert_array_equal(s, rs)
    g.close()
    del tok
    torch.cuda.empty_cache()


def test_hash_filter_sixteen_ranges_bit_exact():
    """A query that probes more than 256 lists (tokens x nprobe) spreads its
    hash tables over 16 doc ranges instead of 8 (at most 7,168 candidates per
    range).  With 80,000 short docs, 32 tokens at nprobe 16 give more
    candidates than 8 ranges hold but fewer than 16 do: no overflow, and the
    result matches the oracle bit for bit; so do 64-token queries at nprobe 4
    (8 ranges) and 8 (16 ranges), and a ragged batch mixing both kinds."""
    lens = np.random.default_rng(11).integers(6, 12, 80_000)
    ix = tiny_index(n_doc=80_000, n_centroid=32, n_bit=2, seed=12, lengths=lens, n_latent=64)
    g, o = gpu_index(ix), oracle_of(ix)
    q, off = make_queries(ix, 2, 32, seed=13)
    qi = q[off[0]:off[1]]
    t = g.trace(qi, 10, 16, 1000)
    compare_trace(t, o.search_one(qi, 10, 16, 1000))
    assert 8 * 7168 < len(t["cand_id"]) <= 16 * 7168
    q64, off64 = make_queries(ix, 2, 64, seed=14)
    for nprobe in (4, 8):
        qi = q64[off64[1]:off64[2]]
        compare_trace(g.trace(qi, 10, nprobe, 800), o.search_one(qi, 10, nprobe, 800))
    qr, offr = make_queries(ix, 6, (4, 64), seed=15)
    s, i = g.search(qr, 10, 8, 800, tok_off=offr)
    rs, ri = o.search(qr, offr, 10, 8, 800)
    np.testing.assert_array_equal(i, ri)
    np.testing.assert_array_equal(s, rs)
    g.close()


def test_hash_filter_overflow_falls_back_bit_exact():
    """With 130,000 short docs and half the centroids probed, a query has more
    candidates than even 16 hash-table ranges hold (16 x 7,168): the rank-table
    filter redoes it; with one probe nothing overflows.  Both must match the
    oracle bit for bit, and queries of the two kinds mixed in one batch must
    not disturb each other."""
    lens = np.random.default_rng(11).integers(6, 12, 130_000)
    ix = tiny_index(n_doc=130_000, n_centroid=32, n_bit=2, seed=12, lengths=lens, n_latent=64)
    g, o = gpu_index(ix), oracle_of(ix)
    q, off = make_queries(ix, 4, 32, seed=13)
    for nprobe in (16, 1):
        qi = q[off[0]:off[1]]
        t = g.trace(qi, 10, nprobe, 1000)
        compare_trace(t, o.search_one(qi, 10, nprobe, 1000))
        if nprobe == 16:
            assert len(t["cand_id"]) > 16 * 7168
    # mixed batch: the same queries at nprobe 16 in one call
    s, i = g.search(q, 10, 16, 1000, tok_off=off)
    rs, ri = o.search(q, off, 10, 16, 1000)
    np.testing.assert_array_equal(i, ri)
    np.testing.assert_array_equal(s, rs)
    # imputed candidate scores through the fallback
    from mvr import CAND_IMPUTE
    qi = q[off[1]:off[2]]
    compare_trace(g.trace(qi, 10, 16, 1000, CAND_IMPUTE),
                  o.search_one(qi, 10, 16, 1000, CAND_IMPUTE))
    # the fallback's stamp epochs advance on the device: replays of one
    # recorded graph (two fallback chunks per batch) stay exact
    import torch
    dq = torch.from_numpy(q).cuda()
    g.set_graphs(True)
    for _ in range(3):
        ds = torch.empty((4, 10), dtype=torch.float32, device="cuda")
        di = torch.empty((4, 10), dtype=torch.int32, device="cuda")
        g.search_device(dq.data_ptr(), off, 4, 0, 10, 16, 1000, ds.data_ptr(), di.data_ptr(), 0)
        torch.cuda.synchronize()
        np.testing.assert_array_equal(di.cpu().numpy().view(np.uint32), ri)
        np.testing.assert_array_equal(ds.cpu().numpy(), rs)
    g.set_graphs(False)
    g.close()


@pytest.mark.parametrize("sem", [SEM_PP, SEM_BASIC], ids=["pp", "basic"])
def test_imputed_candidate_scores_bit_exact(pair, sem):
    """MVR_CAND_IMPUTE: an unmatched query token contributes its lowest probed
    score to the approximate score; candidates, scores, shortlist and top-k
    match the oracle's (the same option) bit for bit, through the hash filter
    and through the rank-table fallback (80,000-doc case below)."""
    from mvr import CAND_IMPUTE
    ix, g, o = pair
    q, off = make_queries(ix, 3, 32, seed=23)
    for i in range(3):
        qi = q[off[i]:off[i + 1]]
        for nprobe, ptk, k in ((4, 100, 10), (8, 300, 100)):
            compare_trace(g.trace(qi, k, nprobe, ptk, sem | CAND_IMPUTE),
                          o.search_one(qi, k, nprobe, ptk, sem | CAND_IMPUTE))


def test_graph_replay_matches_direct_calls(pair):
    """mvr_index_set_graphs: repeated mvr_search_device calls replay one
    recorded CUDA graph; results equal the direct launches' and the oracle's,
    for ragged queries across several batches, on every replay."""
    import torch
    from mvr import PREC_FP8
    ix, g, o = pair
    q, off = make_queries(ix, 12, (1, 64), seed=29)
    rs, ri = o.search(q, off, 10, 6, 120)
    dq = torch.from_numpy(q).cuda()
    for flags in (SEM_PP, PREC_FP8):
        outs = []
        g.set_batch(5)
        for graphs in (False, True, True, True):
            g.set_graphs(graphs)
            s = torch.empty((12, 10), dtype=torch.float32, device="cuda")
            i = torch.empty((12, 10), dtype=torch.int32, device="cuda")
            st = g.search_device(dq.data_ptr(), off, 12, 0, 10, 6, 120, s.data_ptr(), i.data_ptr(),
                                 0, semantics=flags)
            assert st.n_batch == 3
            torch.cuda.synchronize()
            outs.append((s.cpu().numpy(), i.cpu().numpy().view(np.uint32)))
        g.set_graphs(False)
        g.set_batch(0)
        for s_, i_ in outs[1:]:
            np.testing.assert_array_equal(i_, outs[0][1])
            np.testing.assert_array_equal(s_, outs[0][0])
        if flags == SEM_PP:
            np.testing.assert_array_equal(outs[0][1], ri)
            np.testing.assert_array_equal(outs[0][0], rs)
