"""Real ColBERT data shipped with the reference: the 500-doc LoTTE PLAID
index (multi-vector-retrieval-data/Index/lotte-500-gnd/plaid), its 100 encoded
queries and the reference's exhaustive top-10 over the raw embeddings (which
are not shipped).  Read where the reference tree is present (skipped
elsewhere; nothing of it is copied here):

* read_plaid_index / write_plaid_index round-trip the index exactly and write
  the same file set;
* the IGP search (the oracle, which the FP32 CUDA path matches bit for bit)
  over the PLAID index's centroids, codes and weights reaches recall@10 0.99
  against exhaustive MaxSim over the index's decoded vectors and the
  quantization ceiling (the decoded-index exhaustive search's own recall)
  against the shipped raw-embedding ground truth;
* the reference's own PLAID CPU search runs on its own index."""
import os
import tempfile

import numpy as np
import pytest

import pyoracle
from mvr import formats
from refroot import ref_path

DATA = ref_path("multi-vector-retrieval-data")
IDX = os.path.join(DATA, "Index", "lotte-500-gnd", "plaid")
pytestmark = pytest.mark.skipif(not os.path.isdir(IDX), reason="reference data tree absent")


@pytest.fixture(scope="module")
def lotte():
    ix = formats.read_plaid_index(IDX)
    q = np.load(os.path.join(DATA, "Embedding", "lotte-500-gnd", "query_embedding.npy"))
    qids = [int(line.split("\t")[0]) for line in
            open(os.path.join(DATA, "RawData", "lotte-500-gnd", "document", "queries.dev.tsv"))]
    gt = formats.read_answer_tsv(os.path.join(DATA, "Embedding", "lotte-500-gnd",
                                              "lotte-500-gnd-groundtruth-top10--.tsv"))
    gt10 = [[p for p, r, s in sorted(gt[qq], key=lambda t: t[1])] for qq in qids]
    o = pyoracle.Oracle(ix["item_n_vec"], ix["centroid"], ix["vq_code"], ix["residual"],
                        ix["weight"], ix["ivf_off"], ix["ivf_size"], ix["ivf_ids"], ix["n_bit"])
    return ix, np.ascontiguousarray(q, np.float32), gt10, o


def test_plaid_index_round_trip(lotte):
    ix = lotte[0]
    assert ix["n_bit"] == 2 and ix["centroid"].shape == (2048, 128)
    assert int(ix["item_n_vec"].sum()) == len(ix["vq_code"])
    with tempfile.TemporaryDirectory() as td:
        formats.write_plaid_index(td, ix["item_n_vec"], ix["centroid"], ix["vq_code"],
                                  ix["weight"], ix["residual"], ix["ivf_off"], ix["ivf_size"],
                                  ix["ivf_ids"], ix["n_bit"], cutoff=ix["cutoff"])
        assert sorted(os.listdir(td)) == sorted(os.listdir(IDX))
        back = formats.read_plaid_index(td)
    for k, v in ix.items():
        np.testing.assert_array_equal(np.asarray(back[k]), np.asarray(v), err_msg=k)


def test_igp_search_recall_on_real_queries(lotte):
    ix, q, gt10, o = lotte
    off = np.arange(len(q) + 1, dtype=np.uint64) * q.shape[1]
    qf = q.reshape(-1, q.shape[2])
    _, gdec = pyoracle.exhaustive_f64(qf, off, o.decompress_all(), ix["item_n_vec"], 10)
    ceiling = formats.recall_at_k(gt10, gdec, 10).mean()
    _, ids = o.search(qf, off, 10, 8, 300)
    assert formats.recall_at_k(gdec, ids, 10).mean() >= 0.99
    assert formats.recall_at_k(gt10, ids, 10).mean() >= ceiling - 0.01
    assert ceiling > 0.7


def test_reference_plaid_search_on_its_own_index(lotte):
    import plaid_cpu
    if not plaid_cpu.available():
        pytest.skip("reference PLAID extensions not built")
    ix, q, gt10, _ = lotte
    p = plaid_cpu.PlaidCPU(ix["item_n_vec"], ix["centroid"], ix["vq_code"], ix["residual"],
                           ix["weight"], ix["ivf_off"], ix["ivf_size"], ix["ivf_ids"],
                           ix["n_bit"], n_threads=4)
    est = [p.search_one(q[j], 10)[0] for j in range(len(q))]
    # PLAID keeps ndocs / 4 of its candidates: short (even empty) lists where
    # few docs share a query's cells (ncells 1)
    assert all(len(e) <= 10 for e in est) and sum(len(e) == 10 for e in est) >= 80
    assert formats.recall_at_k(gt10, est, 10).mean() > 0.6
