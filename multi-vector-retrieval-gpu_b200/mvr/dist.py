"""Multi-GPU plumbing for query-parallel search (one index replica per GPU,
queries split by rank): the only cross-rank traffic is the timing reduction
and, when a caller wants all answers on one rank, a gather of the per-rank
top-k lists.  No collective sits on the search data path.

Works with any torch.distributed backend (NCCL on GPUs, gloo in the CPU
tests)."""
import numpy as np
import torch
import torch.distributed as dist


def shard(n, rank, world):
    """[start, end) of rank's contiguous share of n items (sizes differ by <= 1)."""
    base, extra = divmod(n, world)
    start = rank * base + min(rank, extra)
    return start, start + base + (1 if rank < extra else 0)


def max_over_ranks(value, device="cpu"):
    """Max of a float over all ranks (the timing rule: slowest rank wins)."""
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def gather_topk(ids, scores, device="cpu"):
    """Concatenates every rank's (ids [n_r, k], scores [n_r, k]) in rank order
    on all ranks; ranks may hold different n_r."""
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return ids, scores
    world = dist.get_world_size()
    n = torch.tensor([ids.shape[0]], dtype=torch.int64, device=device)
    ns = [torch.zeros_like(n) for _ in range(world)]
    dist.all_gather(ns, n)
    ns = [int(x.item()) for x in ns]
    mx = max(ns)
    k = ids.shape[1]
    pi = torch.zeros((mx, k), dtype=torch.int64, device=device)
    ps = torch.zeros((mx, k), dtype=torch.float64, device=device)
    pi[: ids.shape[0]] = torch.as_tensor(np.asarray(ids, np.int64), device=device)
    ps[: ids.shape[0]] = torch.as_tensor(np.asarray(scores, np.float64), device=device)
    gi = [torch.zeros_like(pi) for _ in range(world)]
    gs = [torch.zeros_like(ps) for _ in range(world)]
    dist.all_gather(gi, pi)
    dist.all_gather(gs, ps)
    out_i = np.concatenate([g[:m].cpu().numpy() for g, m in zip(gi, ns)])
    out_s = np.concatenate([g[:m].cpu().numpy() for g, m in zip(gs, ns)])
    return out_i, out_s
