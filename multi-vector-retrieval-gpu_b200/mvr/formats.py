"""Reference on-disk index format: the five .npy arrays and ivf.index
(IVFIndex::save, IVFIndex.hpp:168-183: uint32 n_centroid; uint64 n_ele;
uint64 offset[C]; uint32 size[C]; uint32 ids[n_ele], little endian), plus the
query/answer files of the reference's CLI (IGPGPUBasic.cpp:32-73,150-171),
and the PLAID index directory of the reference's ColBERT baseline (read and
write, see read_plaid_index)."""
import json
import os
import struct

import numpy as np

INDEX_FILES = ("item_n_vec_l.npy", "centroid_l.npy", "vq_code_l.npy", "weight_l.npy",
               "residual_code_l.npy", "ivf.index")


def write_ivf(path, offset, size, ids):
    offset = np.ascontiguousarray(offset, np.uint64)
    size = np.ascontiguousarray(size, np.uint32)
    ids = np.ascontiguousarray(ids, np.uint32)
    with open(path, "wb") as f:
        f.write(struct.pack("<IQ", len(size), len(ids)))
        f.write(offset.tobytes())
        f.write(size.tobytes())
        f.write(ids.tobytes())


def read_ivf(path):
    with open(path, "rb") as f:
        n_c, n_ele = struct.unpack("<IQ", f.read(12))
        offset = np.frombuffer(f.read(8 * n_c), np.uint64)
        size = np.frombuffer(f.read(4 * n_c), np.uint32)
        ids = np.frombuffer(f.read(4 * n_ele), np.uint32)
    if len(ids) != n_ele or len(size) != n_c:
        raise ValueError(f"truncated ivf.index: {path}")
    return offset, size, ids


def write_index_dir(path, item_n_vec, centroid, vq_code, weight, residual, ivf_off, ivf_size,
                    ivf_ids):
    """Writes an index directory exactly as the reference's build script does
    (eval_igp_gpu_basic.py:106-113: vq_code saved as int32)."""
    os.makedirs(path, exist_ok=True)
    np.save(os.path.join(path, "item_n_vec_l.npy"), np.asarray(item_n_vec, np.uint32))
    np.save(os.path.join(path, "centroid_l.npy"), np.asarray(centroid, np.float32))
    np.save(os.path.join(path, "vq_code_l.npy"), np.asarray(vq_code, np.int32))
    np.save(os.path.join(path, "weight_l.npy"), np.asarray(weight, np.float32))
    np.save(os.path.join(path, "residual_code_l.npy"), np.asarray(residual, np.uint8).reshape(-1))
    write_ivf(os.path.join(path, "ivf.index"), ivf_off, ivf_size, ivf_ids)


def read_index_dir(path):
    off, size, ids = read_ivf(os.path.join(path, "ivf.index"))
    return dict(
        item_n_vec=np.load(os.path.join(path, "item_n_vec_l.npy")).astype(np.uint32),
        centroid=np.load(os.path.join(path, "centroid_l.npy")).astype(np.float32),
        vq_code=np.load(os.path.join(path, "vq_code_l.npy")).astype(np.uint32),
        weight=np.load(os.path.join(path, "weight_l.npy")).astype(np.float32),
        residual=np.load(os.path.join(path, "residual_code_l.npy")).astype(np.uint8),
        ivf_off=off, ivf_size=size, ivf_ids=ids)


def write_answer_tsv(path, qid, ids, scores):
    """qid \\t pid \\t rank(1-based) \\t score rows (IGPGPUBasic.cpp:164-171)."""
    with open(path, "w") as f:
        for i, q in enumerate(qid):
            for r in range(ids.shape[1]):
                f.write(f"{q}\t{ids[i, r]}\t{r + 1}\t{scores[i, r]:g}\n")


def read_answer_tsv(path):
    out = {}
    with open(path) as f:
        for line in f:
            q, p, r, s = line.rstrip("\n").split("\t")
            out.setdefault(int(q), []).append((int(p), int(r), float(s)))
    return out


def recall_at_k(gnd_ids, est_ids, k):
    """|gnd top-k  intersect  est top-k| / k per query (count_recall,
    performance_metric.py:259-272)."""
    r = []
    for g, e in zip(gnd_ids, est_ids):
        r.append(len(np.intersect1d(np.asarray(g)[:k], np.asarray(e)[:k])) / k)
    return np.asarray(r)


# ----------------------------------------------------------------------
# PLAID index directory (the reference's ColBERT baseline): centroids.pt
# (fp16 [C, dim]), buckets.pt ((cutoffs f32 [2^b - 1], weights f16 [2^b])),
# avg_residual.pt, ivf.pid.pt ((pids i32, list lengths i64); each list the
# ascending unique pids of a centroid, utils.py:8-53), per chunk i:
# i.codes.pt (i32 [n]), i.residuals.pt (u8 [n, dim * b / 8]),
# i.metadata.json, doclens.i.json; metadata.json / plan.json (config with
# dim and nbits, num_chunks, num_partitions, num_embeddings).  PLAID packs a
# dim's bucket least-significant bit first (ResidualCodec.binarize,
# residual.py:189-205), the IGP layout most-significant bit first in the same
# byte slots: the two differ by reversing the bits of every b-wide group.
# ----------------------------------------------------------------------
def group_bit_reverse(n_bit):
    """Byte table reversing the bits of every n_bit-wide group (an
    involution: PLAID <-> IGP residual bytes)."""
    out = np.zeros(256, np.uint8)
    for x in range(256):
        z = 0
        for g in range(8 // n_bit):
            v = (x >> (g * n_bit)) & ((1 << n_bit) - 1)
            r = 0
            for i in range(n_bit):
                r |= ((v >> i) & 1) << (n_bit - 1 - i)
            z |= r << (g * n_bit)
        out[x] = z
    return out


def read_plaid_index(path):
    """A PLAID index directory as the IGP arrays of this package (residual
    bytes re-laid to the IGP bit order, centroids and weights widened to
    float32), plus its cutoffs."""
    import torch
    meta = json.load(open(os.path.join(path, "metadata.json")))
    n_bit = int(meta["config"]["nbits"])
    cen = torch.load(os.path.join(path, "centroids.pt"), map_location="cpu")
    cut, w = torch.load(os.path.join(path, "buckets.pt"), map_location="cpu")
    ivf, lens = torch.load(os.path.join(path, "ivf.pid.pt"), map_location="cpu")
    codes, res, doclens = [], [], []
    for i in range(int(meta["num_chunks"])):
        codes.append(torch.load(os.path.join(path, f"{i}.codes.pt"), map_location="cpu").numpy())
        res.append(torch.load(os.path.join(path, f"{i}.residuals.pt"), map_location="cpu").numpy())
        doclens += json.load(open(os.path.join(path, f"doclens.{i}.json")))
    size = lens.numpy().astype(np.uint32)
    off = np.zeros(len(size), np.uint64)
    off[1:] = np.cumsum(size[:-1], dtype=np.uint64)
    rev = group_bit_reverse(n_bit)
    return dict(item_n_vec=np.asarray(doclens, np.uint32),
                centroid=cen.float().numpy(),
                vq_code=np.concatenate(codes).astype(np.int32).view(np.uint32),
                weight=w.float().numpy(), cutoff=cut.float().numpy(),
                residual=rev[np.concatenate(res)].reshape(-1),
                ivf_off=off, ivf_size=size, ivf_ids=ivf.numpy().astype(np.int32).view(np.uint32),
                n_bit=n_bit)


def write_plaid_index(path, item_n_vec, centroid, vq_code, weight, residual, ivf_off, ivf_size,
                      ivf_ids, n_bit, cutoff=None):
    """Writes an index of this package as a one-chunk PLAID index directory
    that read_plaid_index (and the reference's IndexLoader) reads: centroids
    stored in fp16 and weights in fp16 as PLAID stores them.  The IGP index
    keeps no cutoffs; without them the midpoints of adjacent weights are
    written (PLAID's search does not read them), and avg_residual (unused
    by PLAID's search) is the mean |weight|."""
    import torch
    os.makedirs(path, exist_ok=True)
    item_n_vec = np.asarray(item_n_vec, np.int64)
    centroid = np.asarray(centroid, np.float32)
    weight = np.asarray(weight, np.float32)
    n, dim = len(vq_code), centroid.shape[1]
    if cutoff is None:
        cutoff = (weight[1:] + weight[:-1]) / 2
    torch.save(torch.from_numpy(centroid).half(), os.path.join(path, "centroids.pt"))
    torch.save((torch.from_numpy(np.asarray(cutoff, np.float32)),
                torch.from_numpy(weight).half()), os.path.join(path, "buckets.pt"))
    torch.save(torch.tensor(float(np.abs(weight).mean())).half(),
               os.path.join(path, "avg_residual.pt"))
    size = np.asarray(ivf_size, np.int64)
    ids = np.asarray(ivf_ids, np.uint32).view(np.int32)
    off = np.asarray(ivf_off, np.int64)
    ivf = np.concatenate([ids[o:o + z] for o, z in zip(off, size)]) if len(size) else ids[:0]
    torch.save((torch.from_numpy(np.ascontiguousarray(ivf)), torch.from_numpy(size)),
               os.path.join(path, "ivf.pid.pt"))
    torch.save(torch.from_numpy(np.asarray(vq_code, np.uint32).view(np.int32).copy()),
               os.path.join(path, "0.codes.pt"))
    bpv = dim * n_bit // 8
    rev = group_bit_reverse(n_bit)
    torch.save(torch.from_numpy(rev[np.asarray(residual, np.uint8).reshape(n, bpv)]),
               os.path.join(path, "0.residuals.pt"))
    json.dump({"passage_offset": 0, "num_passages": len(item_n_vec), "num_embeddings": n,
               "embedding_offset": 0}, open(os.path.join(path, "0.metadata.json"), "w"), indent=4)
    json.dump(item_n_vec.tolist(), open(os.path.join(path, "doclens.0.json"), "w"))
    config = {"dim": dim, "nbits": int(n_bit), "similarity": "cosine", "interaction": "colbert",
              "ncells": None, "centroid_score_threshold": None, "ndocs": None}
    avg = float(item_n_vec.mean()) if len(item_n_vec) else 0.0
    json.dump({"config": config, "num_chunks": 1, "num_partitions": len(size),
               "num_embeddings": n, "avg_doclen": avg},
              open(os.path.join(path, "metadata.json"), "w"), indent=4)
    json.dump({"config": config, "num_chunks": 1, "num_partitions": len(size),
               "num_embeddings_est": float(n), "avg_doclen_est": avg},
              open(os.path.join(path, "plan.json"), "w"), indent=4)
