"""Query-parallel multi-rank search on CPU with gloo (world size 2): each rank
searches its shard of the queries (the oracle stands in for the GPU engine),
the slowest rank's time is the job's, and the gathered top-k lists equal a
single-process run."""
import os
import socket
import sys

import numpy as np
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, out_dir):
    for p in (os.path.join(ROOT, "tests"), os.path.join(ROOT, "oracle"),
              os.path.join(ROOT, "multi-vector-retrieval-gpu_b200")):
        sys.path.insert(0, p)
    import torch.distributed as dist
    from helpers import make_queries, oracle_of, tiny_index
    from mvr import dist as mdist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    from datetime import timedelta
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    ix = tiny_index(n_doc=200, n_centroid=32, seed=6)
    o = oracle_of(ix)
    q, off = make_queries(ix, 9, 32, seed=8)
    a, b = mdist.shard(9, rank, world)
    s, i = o.search(q[off[a]:off[b]], off[a:b + 1] - off[a], 10, 4, 60, n_threads=1)
    gi, gs = mdist.gather_topk(i, s)
    t = mdist.max_over_ranks(float(rank + 1))
    if rank == 0:
        np.savez(os.path.join(out_dir, "r.npz"), ids=gi, scores=gs, t=t)
    dist.barrier()
    dist.destroy_process_group()


def test_shard_partition():
    from mvr import dist as mdist
    for n in (0, 1, 7, 10):
        for w in (1, 2, 3):
            parts = [mdist.shard(n, r, w) for r in range(w)]
            assert parts[0][0] == 0 and parts[-1][1] == n
            assert all(parts[r][1] == parts[r + 1][0] for r in range(w - 1))


def test_two_rank_query_parallel_search(tmp_path):
    import pyoracle  # noqa: F401
    from helpers import make_queries, oracle_of, tiny_index
    mp.start_processes(_worker, args=(2, _free_port(), str(tmp_path)), nprocs=2, join=True,
                       start_method="spawn")
    r = np.load(tmp_path / "r.npz")
    ix = tiny_index(n_doc=200, n_centroid=32, seed=6)
    q, off = make_queries(ix, 9, 32, seed=8)
    s, i = oracle_of(ix).search(q, off, 10, 4, 60, n_threads=1)
    np.testing.assert_array_equal(r["ids"], i)
    np.testing.assert_array_equal(r["scores"].astype(np.float32), s)
    assert float(r["t"]) == 2.0
