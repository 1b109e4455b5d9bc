"""mvr_filter_noalloc -- the candidate filter with its scratch in a fixed
array inside libmvr, for callers that cannot allocate device memory while
serving queries (a plugin in a host whose GPU memory is all reserved by the
host's own pool allocator, or a latency-critical caller that cannot take
cudaMalloc's implicit synchronisation).

Checked through the C ABI against the regular filter stage of mvr_search
(via mvr_search_trace) on two calls in a row, and against the oracle's filter
(fed the oracle's own probe lists) at a small size and at the largest size the
array accepts (262,144 docs, 32 query tokens): same shortlist, same
approximate scores, bit for bit (the tolerance of every other filter test).
This file is collected last on purpose."""
import ctypes as C

import numpy as np
import pytest

from helpers import make_queries, oracle_of, tiny_index
from mvr import Index, _lib

pytestmark = pytest.mark.gpu


def _index(ix):
    return Index.from_arrays(ix["item_n_vec"], ix["centroid"], ix["vq_code"], ix["ivf_off"],
                             ix["ivf_size"], ix["ivf_ids"], ix["weight"], ix["n_bit"],
                             ix["residual"])


def _noalloc(g, probe_id, probe_score, nprobe, ptk):
    import torch
    dev = "cuda"
    pid = torch.from_numpy(probe_id.astype(np.int32).reshape(-1)).to(dev)
    ps = torch.from_numpy(probe_score.reshape(-1)).to(dev)
    sid = torch.full((ptk,), -1, dtype=torch.int32, device=dev)
    sap = torch.zeros(ptk, dtype=torch.float32, device=dev)
    ns = torch.zeros(1, dtype=torch.int32, device=dev)
    nq = probe_id.shape[0]
    rc = _lib.lib().mvr_filter_noalloc(g._h, C.c_void_p(pid.data_ptr()), C.c_void_p(ps.data_ptr()),
                                       nq, nprobe, ptk, C.c_void_p(sid.data_ptr()),
                                       C.c_void_p(sap.data_ptr()), C.c_void_p(ns.data_ptr()), None)
    _lib.check(rc)
    torch.cuda.synchronize()
    n = int(ns.item())
    ids = sid[:n].cpu().numpy().view(np.uint32)
    o = np.argsort(ids)
    return ids[o], sap[:n].cpu().numpy()[o]


def test_noalloc_filter_matches_search_filter_two_calls():
    ix = tiny_index(n_doc=600, n_centroid=80, n_bit=2, seed=21)
    g = _index(ix)
    q, off = make_queries(ix, 2, 32, seed=22)
    for i in range(2):  # two calls in a row share (and must reset) the scratch array
        qi = q[off[i]:off[i + 1]]
        t = g.trace(qi, 10, 6, 150)
        ids, approx = _noalloc(g, t["probe_id"], t["probe_score"], 6, 150)
        np.testing.assert_array_equal(ids, t["short_id"])
        np.testing.assert_array_equal(approx, t["short_approx"])
    g.close()


def _vs_oracle(ix, n_query, nprobe, ptk, seed):
    g, o = _index(ix), oracle_of(ix)
    q, off = make_queries(ix, n_query, 32, seed=seed)
    for i in range(n_query):
        qi = q[off[i]:off[i + 1]]
        r = o.search_one(qi, 10, nprobe, ptk)
        ids, approx = _noalloc(g, r["probe_id"], r["probe_score"], nprobe, ptk)
        order = np.argsort(r["short_id"])
        np.testing.assert_array_equal(ids, r["short_id"][order])
        np.testing.assert_array_equal(approx, r["short_approx"][order])
        t = g.trace(qi, 10, nprobe, ptk)
        np.testing.assert_array_equal(ids, t["short_id"])
    g.close()


def test_noalloc_filter_matches_oracle_filter():
    _vs_oracle(tiny_index(n_doc=900, n_centroid=96, n_bit=2, seed=31), 2, 5, 200, 32)


def test_noalloc_filter_at_the_size_limit():
    """Exactly 262,144 one-token docs (the array's doc limit) and 32 query
    tokens (its token limit); every doc of a probed list ties with the others
    of that list, so the shortlist's cut exercises the (score desc, id asc)
    order."""
    n = 1 << 18
    ix = tiny_index(n_doc=n, n_centroid=64, n_bit=2, seed=33, lengths=np.ones(n, np.uint32))
    _vs_oracle(ix, 2, 4, 3000, 34)


def test_noalloc_filter_rejects_oversize():
    ix = tiny_index(n_doc=40, n_centroid=16, n_bit=2, seed=3)
    g = _index(ix)
    pid = np.zeros((33, 4), np.uint32)
    with pytest.raises(_lib.MvrError) as e:
        _noalloc(g, pid, np.zeros((33, 4), np.float32), 4, 50)
    assert e.value.code == _lib.MVR_ERR_INVALID_ARG and "[1, 32]" in str(e.value)
    g.close()
    big = tiny_index(n_doc=(1 << 18) + 1, n_centroid=16, n_bit=2, seed=4,
                     lengths=np.ones((1 << 18) + 1, np.uint32))
    gb = _index(big)
    with pytest.raises(_lib.MvrError) as e:
        _noalloc(gb, np.zeros((4, 4), np.uint32), np.zeros((4, 4), np.float32), 4, 50)
    assert e.value.code == _lib.MVR_ERR_INVALID_ARG and "262144" in str(e.value)
    gb.close()
