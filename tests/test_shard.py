"""Document-sharded search (mvr.shard): index partition by doc range, merge
of per-shard top-k lists, and a 2-rank gloo job.  The oracle stands in for
the GPU engine on each shard (the GPU version is in test_gpu_shard.py).
With every shard's shortlist holding all of its candidates the merged top-k
equals the single-index top-k bit for bit."""
import os
import socket
import sys

import numpy as np
import pytest
import torch
import torch.multiprocessing as mp

from helpers import make_queries, oracle_of, tiny_index
from mvr import shard

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def oracle_shard(h):
    import pyoracle
    return pyoracle.Oracle(h["item_n_vec"], h["centroid"], h["vq_code"], h["residual"],
                           h["weight"], h["ivf_off"], h["ivf_size"], h["ivf_ids"], h["n_bit"])


def test_split_index_keeps_docs_and_lists():
    ix = tiny_index(n_doc=150, n_centroid=24, n_bit=2, seed=3)
    parts = [shard.split_index(ix, a, b) for a, b in shard.doc_ranges(150, 4)]
    assert sum(len(p["item_n_vec"]) for p in parts) == 150
    assert sum(len(p["vq_code"]) for p in parts) == len(ix["vq_code"])
    assert sum(len(p["ivf_ids"]) for p in parts) == len(ix["ivf_ids"])
    np.testing.assert_array_equal(np.concatenate([p["residual"] for p in parts]),
                                  ix["residual"].reshape(-1))
    for (a, b), p in zip(shard.doc_ranges(150, 4), parts):
        for c in range(24):
            lst = p["ivf_ids"][int(p["ivf_off"][c]):int(p["ivf_off"][c]) + int(p["ivf_size"][c])]
            full = ix["ivf_ids"][int(ix["ivf_off"][c]):int(ix["ivf_off"][c]) + int(ix["ivf_size"][c])]
            np.testing.assert_array_equal(lst + a, full[(full >= a) & (full < b)])


@pytest.mark.parametrize("n_shards", [2, 3])
def test_sharded_search_equals_single_index(n_shards):
    ix = tiny_index(n_doc=180, n_centroid=32, n_bit=2, seed=4)
    q, off = make_queries(ix, 6, 32, seed=5)
    s_ref, i_ref = oracle_of(ix).search(q, off, 10, 6, 180)  # shortlist = every candidate
    ss, ii = [], []
    for a, b in shard.doc_ranges(180, n_shards):
        s, i = oracle_shard(shard.split_index(ix, a, b)).search(q, off, 10, 6, 180)
        ss.append(s)
        ii.append(np.where(i == 0xFFFFFFFF, i, i + a).astype(np.uint32))
    ms, mi = shard.merge_topk(np.stack(ss), np.stack(ii), 10)
    np.testing.assert_array_equal(mi, i_ref)
    np.testing.assert_array_equal(ms, s_ref)
    ts, ti = shard.merge_topk(torch.from_numpy(np.stack(ss)), torch.from_numpy(np.stack(ii).astype(np.int64)), 10)
    np.testing.assert_array_equal(ti.numpy().astype(np.uint32), i_ref)
    np.testing.assert_array_equal(ts.numpy(), s_ref)


def test_merge_breaks_ties_by_id():
    s = np.array([[[1.0, 0.5]], [[1.0, 0.5]]], np.float32)
    i = np.array([[[7, 3]], [[2, 9]]], np.uint32)
    ms, mi = shard.merge_topk(s, i, 3)
    np.testing.assert_array_equal(mi, [[2, 7, 3]])
    np.testing.assert_array_equal(ms, [[1.0, 1.0, 0.5]])


def _free_port():
    so = socket.socket()
    so.bind(("127.0.0.1", 0))
    p = so.getsockname()[1]
    so.close()
    return p


def _worker(rank, world, port, out_dir):
    for p in (os.path.join(ROOT, "tests"), os.path.join(ROOT, "oracle"),
              os.path.join(ROOT, "multi-vector-retrieval-gpu_b200")):
        sys.path.insert(0, p)
    from datetime import timedelta

    import torch.distributed as dist
    from helpers import make_queries, tiny_index
    from mvr import shard as sh
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    ix = tiny_index(n_doc=160, n_centroid=32, n_bit=2, seed=9)
    q, off = make_queries(ix, 5, 32, seed=10)
    d0, d1 = sh.doc_ranges(160, world)[rank]
    o = oracle_shard(sh.split_index(ix, d0, d1))

    def local():
        s, i = o.search(q, off, 10, 6, 160)
        return torch.from_numpy(s), torch.from_numpy(i.astype(np.int64))

    s, i = sh.search_sharded(local, d0, 10)
    if rank == 0:
        np.save(os.path.join(out_dir, "s.npy"), s.numpy())
        np.save(os.path.join(out_dir, "i.npy"), i.numpy())
    dist.barrier()
    dist.destroy_process_group()


def test_two_rank_gloo_sharded_search(tmp_path):
    mp.spawn(_worker, args=(2, _free_port(), str(tmp_path)), nprocs=2, join=True)
    ix = tiny_index(n_doc=160, n_centroid=32, n_bit=2, seed=9)
    q, off = make_queries(ix, 5, 32, seed=10)
    s_ref, i_ref = oracle_of(ix).search(q, off, 10, 6, 160)
    np.testing.assert_array_equal(np.load(tmp_path / "i.npy").astype(np.uint32), i_ref)
    np.testing.assert_array_equal(np.load(tmp_path / "s.npy"), s_ref)
