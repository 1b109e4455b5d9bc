"""mvr.plaid_adapter.Searcher: the reference's PLAID Searcher call site
(search_all_embedding_by_vector) answered by this package's engine over a
PLAID index directory.  CPU: the adapter's logic over an oracle-backed
engine; GPU: the default engine (libmvr) over a synthetic index written as a
PLAID directory, equal to the oracle's search bit for bit."""
import os
import tempfile

import numpy as np
import pytest

from helpers import make_queries, oracle_of, tiny_index
from mvr import formats
from mvr.plaid_adapter import Searcher


class OracleEngine:
    def __init__(self, o):
        self.o = o

    def search(self, q, k, nprobe, probe_topk, with_stats=True, with_stages=True):
        n, nv, d = q.shape
        off = np.arange(n + 1, dtype=np.uint64) * nv
        s, i = self.o.search(q.reshape(-1, d), off, k, nprobe, probe_topk)
        return s, i, {"query_time_s": np.zeros(n), "stage_time_s": np.zeros((n, 6))}


def write_plaid(ix, path):
    formats.write_plaid_index(path, ix["item_n_vec"], ix["centroid"], ix["vq_code"], ix["weight"],
                              ix["residual"], ix["ivf_off"], ix["ivf_size"], ix["ivf_ids"],
                              ix["n_bit"])


def test_adapter_call_site_and_ranking_file():
    ix = tiny_index(n_doc=400, n_centroid=48, n_bit=2, seed=61)
    o = oracle_of(ix)
    q, off = make_queries(ix, 5, 32, seed=62)
    q = q.reshape(5, 32, 128)
    qids = [3, 14, 15, 92, 65]
    with tempfile.TemporaryDirectory() as td:
        write_plaid(ix, os.path.join(td, "plaid"))
        s = Searcher(index=os.path.join(td, "plaid"), engine=OracleEngine(o))
        s.configure(ncells=3, ndocs=120)
        res = s.search_all_embedding_by_vector(q, "query_embedding.npy", qids, k=10)
        ranking, times = res[0], res[1:]
        assert len(times) == 7 and all(len(t) == 5 for t in times)
        rs, ri = o.search(q.reshape(-1, 128), off, 10, 3, 120)
        for j, qid in enumerate(qids):
            assert [p for p, r, sc in ranking.data[qid]] == ri[j].tolist()
            assert [r for p, r, sc in ranking.data[qid]] == list(range(1, 11))
        path = ranking.save_absolute_path(os.path.join(td, "answer.tsv"))
        back = formats.read_answer_tsv(path)
        assert sorted(back) == sorted(qids) and back[3][0][0] == int(ri[0][0])
    # PLAID's defaults for k = 10 fill the unset settings
    s2 = Searcher(index=None, engine=OracleEngine(o))
    s2.search_all_embedding_by_vector(q, "", qids, k=10)
    assert (s2.config.ncells, s2.config.ndocs, s2.config.centroid_score_threshold) == (1, 256, 0.5)


@pytest.mark.gpu
def test_adapter_default_engine_on_gpu_equals_oracle():
    ix = tiny_index(n_doc=500, n_centroid=64, n_bit=2, seed=63)
    q, off = make_queries(ix, 6, 32, seed=64)
    with tempfile.TemporaryDirectory() as td:
        write_plaid(ix, td)
        back = formats.read_plaid_index(td)  # PLAID stores fp16 centroids and weights
        o = oracle_of(dict(back))
        s = Searcher(index=td)
        s.configure(ncells=4, ndocs=150)
        ranking = s.search_all_embedding_by_vector(q.reshape(6, 32, 128), "", list(range(6)),
                                                   k=10)[0]
        s.engine.close()
    rs, ri = o.search(q, off, 10, 4, 150)
    for j in range(6):
        assert [p for p, r, sc in ranking.data[j]] == ri[j].tolist()
        assert [sc for p, r, sc in ranking.data[j]] == [float(x) for x in rs[j]]
