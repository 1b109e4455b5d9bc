"""The reference's own PLAID CPU search extensions (compiled from its sources
by oracle/build_plaid.py) over this project's index re-laid in PLAID's
layout: the reference's decompress_residuals reproduces the oracle's decode
bit for bit for every code width (so the re-laying is exact), and the PLAID
search returns its top-k by the MaxSim of the normalized decompressed
vectors."""
import numpy as np
import pytest

import plaid_cpu
from helpers import make_queries, oracle_of, tiny_index

pytestmark = pytest.mark.skipif(not plaid_cpu.available(),
                                reason="reference PLAID extensions not built (oracle/build_plaid.py)")


def plaid_of(ix):
    return plaid_cpu.PlaidCPU(ix["item_n_vec"], ix["centroid"], ix["vq_code"], ix["residual"],
                              ix["weight"], ix["ivf_off"], ix["ivf_size"], ix["ivf_ids"],
                              ix["n_bit"], n_threads=4)


def test_reversed_bit_map_is_an_involution():
    for b in (1, 2, 4, 8):
        m = plaid_cpu.reversed_bit_map(b)
        assert np.array_equal(m[m], np.arange(256))
    assert plaid_cpu.reversed_bit_map(2)[0b01101100] == 0b10011100
    assert np.array_equal(plaid_cpu.reversed_bit_map(8), np.array(
        [int(f"{x:08b}"[::-1], 2) for x in range(256)], np.uint8))


@pytest.mark.parametrize("n_bit", [1, 2, 4, 8])
def test_reference_decompress_equals_oracle_decode(n_bit):
    ix = tiny_index(n_doc=300, n_centroid=48, n_bit=n_bit, seed=30 + n_bit)
    o, p = oracle_of(ix), plaid_of(ix)
    pids = np.array([0, 7, 150, 299, 7])
    d = p.decompress_pids(pids).numpy()
    ref = np.concatenate([o.decompress_item(i) for i in pids])
    np.testing.assert_array_equal(d, ref)


def test_plaid_search_ranks_by_normalized_maxsim():
    ix = tiny_index(n_doc=500, n_centroid=64, n_bit=2, seed=41)
    o, p = oracle_of(ix), plaid_of(ix)
    q, off = make_queries(ix, 3, 32, seed=42)
    for i in range(3):
        qi = q[off[i]:off[i + 1]]
        ids, sc = p.search_one(qi, 10)
        assert len(ids) == 10 and len(set(ids.tolist())) == 10
        assert np.all(np.diff(sc) <= 0)
        for d, s in zip(ids, sc):
            x = o.decompress_item(int(d)).astype(np.float64)
            x /= np.linalg.norm(x, axis=1, keepdims=True)
            ref = (qi.astype(np.float64) @ x.T).max(1).sum()
            assert abs(s - ref) < 1e-4 * max(1.0, abs(ref))


def test_bench_plaid_baseline_line():
    """bench.py --plaid-baseline: the reported object (QPS on a bounded sample,
    recall against the given ground truths)."""
    import importlib.util
    import os
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sb = importlib.util.spec_from_file_location("bench_mod2", os.path.join(root, "bench.py"))
    bench = importlib.util.module_from_spec(sb)
    sb.loader.exec_module(bench)
    ix = tiny_index(n_doc=300, n_centroid=48, n_bit=2, seed=71)
    q, off = make_queries(ix, 6, 32, seed=72)
    o = oracle_of(ix)
    _, gt = o.search(q, off, 10, 48, 300)  # every list probed: the exact top-10
    r = bench.plaid_cpu_baseline(dict(ix), q, off, 10, 2, gt, gt, budget_s=0.5)
    assert r["kind"] == "reference" and r["value"] > 0 and 0.0 <= r["recall@10"] <= 1.0
    assert r["params"] == {"ncells": 1, "centroid_score_threshold": 0.5, "ndocs": 256}
