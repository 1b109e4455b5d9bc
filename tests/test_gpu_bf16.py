"""Mixed-precision paths (MVR_PREC_BF16, MVR_PREC_FP8): the BF16 or FP8
(E4M3) tensor-core (tcgen05) MaxSim over the shortlist followed by the exact
FP32 re-score of its best R docs.  Checked against the oracle: the
approximate scores lie within BF16 (FP8) rounding of the exact FP32 MaxSim,
every returned score is bit-identical to the oracle's FP32 MaxSim of that
doc, and the top-k equals the plain path's wherever the plain path's exact
ranking survives the approximate pre-selection."""
import numpy as np
import pytest

import pyoracle
from helpers import make_queries, oracle_of, tiny_index
from mvr import PREC_BF16, PREC_FP8, SEM_BASIC, SEM_PP, Index

pytestmark = pytest.mark.gpu


def gpu_index(ix):
    return Index.from_arrays(ix["item_n_vec"], ix["centroid"], ix["vq_code"], ix["ivf_off"],
                             ix["ivf_size"], ix["ivf_ids"], ix["weight"], ix["n_bit"],
                             ix["residual"])


@pytest.fixture(scope="module", params=[1, 2, 4, 8], ids=lambda b: f"b{b}")
def pair(request):
    ix = tiny_index(n_doc=500, n_centroid=96, n_bit=request.param, seed=10 + request.param)
    g = gpu_index(ix)
    yield ix, g, oracle_of(ix)
    g.close()


@pytest.mark.parametrize("sem", [SEM_PP, SEM_BASIC], ids=["pp", "basic"])
def test_bf16_scores_close_to_exact(pair, sem):
    ix, g, o = pair
    q, off = make_queries(ix, 4, (8, 64), seed=31)
    rel = []
    for i in range(4):
        qi = q[off[i]:off[i + 1]]
        t = g.trace(qi, 10, 6, 200, sem | PREC_BF16)
        r = o.search_one(qi, 10, 6, 200, sem)
        np.testing.assert_array_equal(t["short_id"], np.sort(r["short_id"]))
        exact = np.array([o.maxsim_item(qi, d, sem) for d in t["short_id"]])
        err = np.abs(t["short_exact"] - exact) / np.maximum(np.abs(exact), 1e-3)
        rel.append(err)
        assert err.max() < 3e-2, err.max()
    assert np.concatenate(rel).mean() < 5e-3


@pytest.mark.parametrize("sem", [SEM_PP, SEM_BASIC], ids=["pp", "basic"])
def test_bf16_topk_scores_are_exact_fp32(pair, sem):
    ix, g, o = pair
    q, off = make_queries(ix, 24, 32, seed=33)
    s_bf, i_bf = g.search(q.reshape(24, 32, 128), 10, 6, 200, semantics=sem | PREC_BF16)
    s_pl, i_pl = g.search(q.reshape(24, 32, 128), 10, 6, 200, semantics=sem)
    same = 0
    for k in range(24):
        qk = q[off[k]:off[k + 1]]
        for d, s in zip(i_bf[k], s_bf[k]):
            if d != 0xFFFFFFFF:
                assert s == o.maxsim_item(qk, d, sem)  # bit-exact FP32 re-score
        same += np.array_equal(i_bf[k], i_pl[k])
        # order is by exact score: (score desc, id asc)
        assert all((s_bf[k][j] > s_bf[k][j + 1]) or
                   (s_bf[k][j] == s_bf[k][j + 1] and i_bf[k][j] < i_bf[k][j + 1])
                   for j in range(9))
    assert same >= 22, same


def test_bf16_rescore_width_and_batches(pair):
    ix, g, o = pair
    q, off = make_queries(ix, 30, (1, 64), seed=35)
    ref_s, ref_i = g.search(q, 10, 4, 150, tok_off=off)
    g.set_rescore(150)  # re-score the whole shortlist: identical to the plain path
    g.set_batch(7)
    s, i = g.search(q, 10, 4, 150, tok_off=off, semantics=PREC_BF16)
    g.set_rescore(0)
    g.set_batch(0)
    np.testing.assert_array_equal(i, ref_i)
    np.testing.assert_array_equal(s, ref_s)


def test_bf16_small_shortlists():
    lens = np.random.default_rng(1).integers(1, 20, 80)
    ix = tiny_index(n_doc=80, n_centroid=30, n_bit=2, seed=5, lengths=lens)
    g, o = gpu_index(ix), oracle_of(ix)
    q, off = make_queries(ix, 5, 32, seed=2)
    for i in range(5):
        qi = q[off[i]:off[i + 1]]
        for nq in (1, 32):
            t = g.trace(qi[:nq], 10, 1, 12, PREC_BF16)
            r = o.search_one(qi[:nq], 10, 1, 12)
            assert len(t["short_id"]) == len(r["short_id"])
            ok = t["id"] != 0xFFFFFFFF
            assert ok.sum() == min(10, len(r["short_id"]))
    g.close()


@pytest.mark.parametrize("n_centroid", [96, 700])
def test_tensor_core_probe_matches_exact(n_centroid):
    """nprobe <= 16 under MVR_PREC_BF16 scores centroids on the tensor cores
    and re-scores the candidates in exact FP32: probe ids and scores must be
    the plain path's, bit for bit."""
    ix = tiny_index(n_doc=700, n_centroid=n_centroid, n_bit=2, seed=n_centroid)
    g, o = gpu_index(ix), oracle_of(ix)
    q, off = make_queries(ix, 6, (1, 64), seed=41)
    for i in range(6):
        qi = q[off[i]:off[i + 1]]
        for nprobe in (1, 8, 16):
            t = g.trace(qi, 10, nprobe, 100, PREC_BF16)
            r = o.search_one(qi, 10, nprobe, 100)
            np.testing.assert_array_equal(t["probe_id"], r["probe_id"])
            np.testing.assert_array_equal(t["probe_score"], r["probe_score"])
            np.testing.assert_array_equal(t["cand_id"], r["cand_id"])
    # a multi-batch run exercises several token tiles and centroid splits
    s, i = g.search(q, 10, 8, 100, tok_off=off, semantics=PREC_BF16)
    s2, i2 = g.search(q, 10, 8, 100, tok_off=off)
    assert (i == i2).all(axis=1).sum() >= 5
    g.close()


@pytest.fixture(scope="module", params=["b2", "b4", "b4mixed"])
def pair2(request):
    """2- and 4-bit indexes for the FP8 kernel; b4mixed permutes the 16 bucket
    weights so that both halves of the code range hold weights of both signs
    (the 4-bit decode's sign table)."""
    n_bit = 2 if request.param == "b2" else 4
    ix = tiny_index(n_doc=600, n_centroid=96, n_bit=n_bit, seed=77 if n_bit == 2 else 81)
    if request.param == "b4mixed":
        w = np.asarray(ix["weight"], np.float32)
        perm = np.random.default_rng(3).permutation(len(w))
        while (np.sign(w[perm[:8]]).min() >= 0 or np.sign(w[perm[:8]]).max() <= 0 or
               np.sign(w[perm[8:]]).min() >= 0 or np.sign(w[perm[8:]]).max() <= 0):
            perm = np.random.default_rng(int(perm[0]) + 11).permutation(len(w))
        ix["weight"] = w[perm].copy()
    g = gpu_index(ix)
    yield ix, g, oracle_of(ix)
    g.close()


@pytest.mark.parametrize("sem", [SEM_PP, SEM_BASIC], ids=["pp", "basic"])
def test_fp8_scores_close_to_exact(pair2, sem):
    """E4M3 operands (3 mantissa bits) with FP32 accumulation: per-doc MaxSim
    within 6e-2 relative of the exact FP32 value, 1.5e-2 on average."""
    ix, g, o = pair2
    q, off = make_queries(ix, 4, (8, 64), seed=51)
    rel = []
    for i in range(4):
        qi = q[off[i]:off[i + 1]]
        t = g.trace(qi, 10, 6, 200, sem | PREC_FP8)
        r = o.search_one(qi, 10, 6, 200, sem)
        np.testing.assert_array_equal(t["short_id"], np.sort(r["short_id"]))
        exact = np.array([o.maxsim_item(qi, d, sem) for d in t["short_id"]])
        err = np.abs(t["short_exact"] - exact) / np.maximum(np.abs(exact), 1e-3)
        rel.append(err)
        assert err.max() < 6e-2, err.max()
    assert np.concatenate(rel).mean() < 1.5e-2


@pytest.mark.parametrize("sem", [SEM_PP, SEM_BASIC], ids=["pp", "basic"])
def test_fp8_topk_scores_are_exact_fp32(pair2, sem):
    ix, g, o = pair2
    q, off = make_queries(ix, 24, 32, seed=53)
    s8, i8 = g.search(q.reshape(24, 32, 128), 10, 6, 200, semantics=sem | PREC_FP8)
    s_pl, i_pl = g.search(q.reshape(24, 32, 128), 10, 6, 200, semantics=sem)
    same = 0
    for k in range(24):
        qk = q[off[k]:off[k + 1]]
        for d, s in zip(i8[k], s8[k]):
            if d != 0xFFFFFFFF:
                assert s == o.maxsim_item(qk, d, sem)  # bit-exact FP32 re-score
        same += np.array_equal(i8[k], i_pl[k])
    assert same >= 20, same


def test_fp8_rescore_all_equals_plain_and_other_widths_run(pair2):
    ix, g, o = pair2
    q, off = make_queries(ix, 30, (1, 64), seed=55)
    ref_s, ref_i = g.search(q, 10, 4, 150, tok_off=off)
    g.set_rescore(150)
    g.set_batch(7)
    s, i = g.search(q, 10, 4, 150, tok_off=off, semantics=PREC_FP8)
    g.set_rescore(0)
    g.set_batch(0)
    np.testing.assert_array_equal(i, ref_i)
    np.testing.assert_array_equal(s, ref_s)
    # 1- and 8-bit indexes take the BF16 kernels under MVR_PREC_FP8
    for n_bit in (1, 8):
        ixb = tiny_index(n_doc=200, n_centroid=40, n_bit=n_bit, seed=78)
        gb, ob = gpu_index(ixb), oracle_of(ixb)
        qb, offb = make_queries(ixb, 3, 32, seed=56)
        sb, ib = gb.search(qb.reshape(3, 32, 128), 10, 4, 60, semantics=PREC_FP8)
        for k in range(3):
            for d, sc in zip(ib[k], sb[k]):
                if d != 0xFFFFFFFF:
                    assert sc == ob.maxsim_item(qb[offb[k]:offb[k + 1]], d, SEM_PP)
        gb.close()


@pytest.mark.parametrize("n_bit", [2, 4])
def test_fp8_doc_group_boundaries(n_bit):
    """The FP8 kernel packs the tokens of a CTA's docs densely into 128-row
    MMA tiles, and each epilogue warp takes 32 of those rows: docs of 1, 31,
    32, 33, 63, 64, 65, 96 and 97 tokens (and random lengths up to 200) start
    and end at every offset of a 32-row group, fill one exactly or cross into
    the next, and cross tile boundaries; shortlists of 333 docs span several
    CTAs and end in partial tiles.  Approximate scores stay within FP8
    rounding of the exact MaxSim and the returned scores are exact, for
    20..32-token and 33..64-token queries in one batch, at every tile shape
    (256 -- the default; 128 for queries of more than 32 tokens --, 64, 32
    and 128 docs per CTA)."""
    rng = np.random.default_rng(91 + n_bit)
    edge = [1, 31, 32, 33, 63, 64, 65, 96, 97]
    lens = np.concatenate([np.tile(edge, 12), rng.integers(1, 201, 300)]).astype(np.uint32)
    rng.shuffle(lens)
    ix = tiny_index(n_doc=len(lens), n_centroid=64, n_bit=n_bit, seed=92 + n_bit, lengths=lens)
    g, o = gpu_index(ix), oracle_of(ix)
    q, off = make_queries(ix, 6, (20, 64), seed=93)
    for docs in (256, 64, 32, 128):
        g.set_rerank_tile(docs)
        rel = []
        for i in range(6):
            qi = q[off[i]:off[i + 1]]
            t = g.trace(qi, 10, 6, 333, PREC_FP8)
            r = o.search_one(qi, 10, 6, 333)
            np.testing.assert_array_equal(t["short_id"], np.sort(r["short_id"]))
            exact = np.array([o.maxsim_item(qi, d) for d in t["short_id"]])
            err = np.abs(t["short_exact"] - exact) / np.maximum(np.abs(exact), 1e-3)
            assert err.max() < 6e-2, (docs, i, err.max())
            rel.append(err)
        assert np.concatenate(rel).mean() < 1.5e-2, docs
        s8, i8 = g.search(q, 10, 6, 333, tok_off=off, semantics=PREC_FP8)
        for k in range(6):
            for d, sc in zip(i8[k], s8[k]):
                if d != 0xFFFFFFFF:
                    assert sc == o.maxsim_item(q[off[k]:off[k + 1]], d)
    g.close()
