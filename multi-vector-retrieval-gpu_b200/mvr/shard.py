"""Document-sharded search across GPUs.

The path shards naturally by document: rank r holds a contiguous doc range
[d0, d1) of the index -- those docs' lengths, codes and residuals and the
sub-lists of every IVF list that fall in the range (ids made local by
subtracting d0) -- plus the full centroid table and bucket weights.  Every
rank scores all queries against its shard and keeps its local top-k; one
all-gather of k (score, id) pairs per query per rank and a merge by (score
desc, id asc) give the global top-k.  Each shard draws its shortlist from its
own candidates, so the merged result equals the single-GPU result exactly
whenever every shard's shortlist holds all of its candidates, and otherwise
differs only where a global top-k doc missed its shard's shortlist.

`split_index` partitions host index arrays (the reference's on-disk layout),
`merge_topk` merges per-shard results (numpy or torch, CPU or GPU), and
`search_sharded` runs one rank's part of a torch.distributed job (NCCL on
GPUs, gloo in the CPU tests).
"""
import numpy as np


def doc_ranges(n_item, n_shards):
    """[d0, d1) of every shard: contiguous, sizes differing by <= 1."""
    base, extra = divmod(n_item, n_shards)
    out, d = [], 0
    for r in range(n_shards):
        n = base + (1 if r < extra else 0)
        out.append((d, d + n))
        d += n
    return out


def split_index(host, d0, d1):
    """The shard of host index arrays (item_n_vec, centroid, vq_code,
    residual, weight, ivf_off, ivf_size, ivf_ids, n_bit) holding docs
    [d0, d1), with doc ids renumbered from 0."""
    lens = np.asarray(host["item_n_vec"], np.uint32)
    tok_off = np.zeros(len(lens) + 1, np.int64)
    tok_off[1:] = np.cumsum(lens, dtype=np.int64)
    t0, t1 = int(tok_off[d0]), int(tok_off[d1])
    bpv = 128 * int(host["n_bit"]) // 8
    n_cent = len(host["ivf_size"])
    ids = np.asarray(host["ivf_ids"], np.uint32)
    size = np.asarray(host["ivf_size"], np.int64)
    cid = np.repeat(np.arange(n_cent, dtype=np.int64), size)
    keep = (ids >= d0) & (ids < d1)
    new_size = np.bincount(cid[keep], minlength=n_cent).astype(np.uint32)
    new_off = np.zeros(n_cent, np.uint64)
    new_off[1:] = np.cumsum(new_size[:-1], dtype=np.uint64)
    residual = np.asarray(host["residual"]).reshape(-1)
    return dict(item_n_vec=lens[d0:d1].copy(), centroid=host["centroid"],
                vq_code=np.asarray(host["vq_code"])[t0:t1].copy(),
                residual=residual[t0 * bpv:t1 * bpv].copy(), weight=host["weight"],
                ivf_off=new_off, ivf_size=new_size, ivf_ids=(ids[keep] - d0).astype(np.uint32),
                n_bit=host["n_bit"])


def merge_topk(scores, ids, k):
    """Global top-k of per-shard results.  scores / ids: [n_shards, n_query,
    k_shard] (numpy arrays or torch tensors; ids already global, 0xFFFFFFFF /
    -inf for empty slots).  Order (score desc, id asc), as every top-k of the
    search path.  Returns (scores, ids) [n_query, k] of the input's kind."""
    try:
        import torch
        is_torch = isinstance(scores, torch.Tensor)
    except ImportError:  # pragma: no cover
        is_torch = False
    if is_torch:
        import torch
        s = scores.permute(1, 0, 2).reshape(scores.shape[1], -1)
        i = ids.permute(1, 0, 2).reshape(ids.shape[1], -1).to(torch.int64) & 0xFFFFFFFF
        o = torch.sort(i, dim=1, stable=True).indices             # id asc
        s, i = torch.gather(s, 1, o), torch.gather(i, 1, o)
        o = torch.sort(s, dim=1, descending=True, stable=True).indices  # score desc
        return torch.gather(s, 1, o)[:, :k], torch.gather(i, 1, o)[:, :k]
    s = np.transpose(np.asarray(scores), (1, 0, 2)).reshape(np.shape(scores)[1], -1)
    i = np.transpose(np.asarray(ids, np.uint32), (1, 0, 2)).reshape(np.shape(ids)[1], -1)
    out_s = np.empty((s.shape[0], k), np.float32)
    out_i = np.empty((s.shape[0], k), np.uint32)
    for r in range(s.shape[0]):
        o = np.lexsort((i[r], -s[r].astype(np.float64)))[:k]
        out_s[r], out_i[r] = s[r][o], i[r][o]
    return out_s, out_i


def search_sharded(search_local, d0, k, device="cpu"):
    """One rank's part of a doc-sharded search job.  search_local() returns
    this shard's (scores [n_query, k], local ids [n_query, k]) as torch
    tensors on `device`; the ids are made global with d0, all ranks'
    results are all-gathered and merged.  Returns the global (scores, ids)
    on every rank."""
    import torch
    import torch.distributed as dist
    s, i = search_local()
    i = i.to(torch.int64) & 0xFFFFFFFF
    valid = i != 0xFFFFFFFF
    i = torch.where(valid, i + d0, i)
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return merge_topk(s.unsqueeze(0), i.unsqueeze(0), k)
    world = dist.get_world_size()
    gs = [torch.empty_like(s) for _ in range(world)]
    gi = [torch.empty_like(i) for _ in range(world)]
    dist.all_gather(gs, s.contiguous())
    dist.all_gather(gi, i.contiguous())
    return merge_topk(torch.stack(gs), torch.stack(gi), k)
