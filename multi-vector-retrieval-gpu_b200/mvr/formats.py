"""Reference on-disk index format: the five .npy arrays and ivf.index
(IVFIndex::save, IVFIndex.hpp:168-183: uint32 n_centroid; uint64 n_ele;
uint64 offset[C]; uint32 size[C]; uint32 ids[n_ele], little endian), plus the
query/answer files of the reference's CLI (IGPGPUBasic.cpp:32-73,150-171)."""
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
