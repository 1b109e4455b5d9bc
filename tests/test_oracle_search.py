"""The oracle's search pipeline against an independent numpy restatement of
the reference's PP semantics (FilterPP.hpp:99-142,366-394, RerankPP.hpp:
115-161,458-471) on tiny seeded indexes, plus its stated canonical
arithmetic (sequential fmaf dot products)."""
import numpy as np
import pytest

import pyoracle
from helpers import make_queries, oracle_of, tiny_index

TOL = 1e-5  # relative tolerance of FP32 scores against FP64


@pytest.fixture(scope="module")
def ix():
    return tiny_index(n_doc=250, n_centroid=48, n_bit=2, seed=3)


def np_reference(ix, q, topk, nprobe, probe_topk, basic=False):
    cen = ix["centroid"].astype(np.float64)
    S = q.astype(np.float64) @ cen.T + 1.0
    probe = np.argsort(-S, axis=1, kind="stable")[:, :nprobe]
    n_item = len(ix["item_n_vec"])
    M = np.zeros((n_item, q.shape[0]))
    hit = np.zeros(n_item, bool)
    for t in range(q.shape[0]):
        for c in probe[t]:
            lst = ix["ivf_ids"][ix["ivf_off"][c]: ix["ivf_off"][c] + ix["ivf_size"][c]]
            M[lst, t] = np.maximum(M[lst, t], S[t, c])
            hit[lst] = True
    cand = np.nonzero(hit)[0]
    approx = M[cand].sum(1)
    order = np.lexsort((cand, -approx))[:probe_topk]
    short = cand[order]
    o = oracle_of(ix)
    dec = o.decompress_all().astype(np.float64)
    off = np.concatenate([[0], np.cumsum(ix["item_n_vec"].astype(np.int64))])
    mx = ix["item_n_vec"].max()
    exact = []
    for d in short:
        x = dec[off[d]:off[d + 1]]
        m = (q.astype(np.float64) @ x.T).max(1)
        if basic and ix["item_n_vec"][d] < mx:
            m = np.maximum(m, 0)
        exact.append(m.sum())
    exact = np.asarray(exact)
    fin = np.lexsort((short, -exact))[:topk]
    return dict(probe=probe, S=S, cand=cand, approx=approx, short=short, exact=exact,
                top_ids=short[fin], top_s=exact[fin])


def gap_ok(sorted_desc, n, tol=1e-5):
    return n >= len(sorted_desc) or sorted_desc[n - 1] - sorted_desc[n] > tol * abs(sorted_desc[n - 1])


@pytest.mark.parametrize("semantics", [pyoracle.SEM_PP, pyoracle.SEM_BASIC])
def test_oracle_matches_numpy_fp64(ix, semantics):
    q, off = make_queries(ix, 6, 32, seed=11)
    o = oracle_of(ix)
    for i in range(6):
        qi = q[off[i]:off[i + 1]]
        r = o.search_one(qi, 10, 4, 60, semantics)
        ref = np_reference(ix, qi, 10, 4, 60, basic=semantics == pyoracle.SEM_BASIC)
        # probes: identical wherever the nprobe-th / (nprobe+1)-th gap clears the tolerance
        for t in range(qi.shape[0]):
            srt = np.sort(ref["S"][t])[::-1]
            if gap_ok(srt, 4):
                assert set(r["probe_id"][t]) == set(ref["probe"][t])
        if all(gap_ok(np.sort(ref["S"][t])[::-1], 4) for t in range(qi.shape[0])):
            np.testing.assert_array_equal(r["cand_id"], ref["cand"])
            np.testing.assert_allclose(r["cand_score"], ref["approx"], rtol=TOL)
        np.testing.assert_allclose(np.sort(r["short_exact"]),
                                   np.sort(np.asarray([o.maxsim_item(qi, d, semantics)
                                                       for d in r["short_id"]])), rtol=0)
        # exact scores of the shortlisted docs: FP32 within 1e-5 of FP64
        ref_ex = {d: s for d, s in zip(ref["short"], ref["exact"])}
        for d, s in zip(r["short_id"], r["short_exact"]):
            if d in ref_ex:
                assert abs(s - ref_ex[d]) <= TOL * abs(ref_ex[d]) + 1e-6


def test_probe_sorted_and_tie_break():
    S = np.array([[1.0, 2.0, 2.0, 0.5, 2.0]], np.float32)
    ids = np.zeros(3, np.uint32)
    sc = np.zeros(3, np.float32)
    import ctypes as C
    pyoracle.lib().orc_probe(C.c_void_p(S.ctypes.data), 1, 5, 3, C.c_void_p(ids.ctypes.data),
                             C.c_void_p(sc.ctypes.data))
    np.testing.assert_array_equal(ids, [1, 2, 4])


def test_canonical_dot_is_sequential_fma():
    rng = np.random.default_rng(0)
    q = rng.standard_normal((3, 128)).astype(np.float32)
    c = rng.standard_normal((5, 128)).astype(np.float32)
    S = pyoracle.centroid_scores(q, c)
    for i in range(3):
        for j in range(5):
            acc = np.float32(0)
            for d in range(128):  # fma in float64 then round == correctly rounded fmaf
                acc = np.float32(np.float64(q[i, d]) * np.float64(c[j, d]) + np.float64(acc))
            assert S[i, j] == np.float32(acc + np.float32(1.0))


def test_few_candidates_and_padding(ix):
    o = oracle_of(ix)
    q, off = make_queries(ix, 1, 4, seed=2)
    r = o.search_one(q, 5, 1, 5000, pyoracle.SEM_PP)
    assert len(r["short_id"]) == len(r["cand_id"]) < 5000
    assert np.all(np.diff(r["score"][np.isfinite(r["score"])]) <= 0)


def test_batch_equals_single(ix):
    q, off = make_queries(ix, 5, (8, 32), seed=4)
    o = oracle_of(ix)
    s, i = o.search(q, off, 10, 4, 80, n_threads=3)
    for k in range(5):
        r = o.search_one(q[off[k]:off[k + 1]], 10, 4, 80)
        np.testing.assert_array_equal(i[k], r["id"])
        np.testing.assert_array_equal(s[k], r["score"])


def test_exhaustive_f64_matches_numpy(ix):
    q, off = make_queries(ix, 2, 8, seed=5)
    s, i = pyoracle.exhaustive_f64(q, off, ix["tokens"], ix["item_n_vec"], 5)
    toff = np.concatenate([[0], np.cumsum(ix["item_n_vec"].astype(np.int64))])
    for k in range(2):
        qk = q[off[k]:off[k + 1]].astype(np.float64)
        sc = np.array([(qk @ ix["tokens"][toff[d]:toff[d + 1]].astype(np.float64).T).max(1).sum()
                       for d in range(len(ix["item_n_vec"]))])
        o = np.lexsort((np.arange(len(sc)), -sc))[:5]
        np.testing.assert_array_equal(i[k], o)
        np.testing.assert_allclose(s[k], sc[o], rtol=1e-12)
