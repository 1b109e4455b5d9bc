"""Generates the golden fixtures in this folder from the REFERENCE's own code.

Runs only where the reference sources exist: it imports the module that
oracle/Makefile (target `ref`) compiles from the reference's unmodified
ResidualScalarQuantizationPack.hpp, IVFIndex.hpp and Distance.hpp.  The codec
fixtures freeze, per case, the reference's quantile cutoffs/weights, packed
residual codes, decode table, decoded vectors, IVF lists and ivf.index bytes
for seeded synthetic inputs; the MaxSim fixtures freeze the reference's
vectorSetDistance of seeded query sets against every item, over the decoded
vectors (the rerank's MaxSim) and over the raw vectors (the exhaustive
ground truth's).  The oracle and the CUDA path are checked against them where
the reference itself cannot travel.

    make -C oracle ref && python tests/golden/make_golden.py [codec|maxsim]
"""
import glob
import os
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))

# (name, n_bit, dim, n_item, max_len, n_centroid, seed, coarse)
CASES = [
    ("b1_d128", 1, 128, 20, 10, 16, 101, False),
    ("b2_d128", 2, 128, 20, 10, 16, 102, False),
    ("b4_d128", 4, 128, 20, 10, 16, 103, False),
    ("b8_d128", 8, 128, 20, 10, 16, 104, False),
    ("b1_d36", 1, 36, 24, 8, 8, 105, False),
    ("b2_d36_ties", 2, 36, 24, 8, 8, 106, True),
]


def make_inputs(n_bit, dim, n_item, max_len, n_centroid, seed, coarse):
    rng = np.random.default_rng(seed)
    item_n_vec = rng.integers(1, max_len + 1, n_item).astype(np.uint32)
    n_vec = int(item_n_vec.sum())
    vec = rng.standard_normal((n_vec, dim)).astype(np.float32)
    vec /= np.linalg.norm(vec, axis=1, keepdims=True)
    cen = rng.standard_normal((n_centroid, dim)).astype(np.float32)
    cen /= np.linalg.norm(cen, axis=1, keepdims=True)
    if coarse:  # many exactly tied residual values
        vec = np.round(vec * 8) / 8
        cen = np.round(cen * 8) / 8
    vec = vec.astype(np.float32)
    cen = cen.astype(np.float32)
    code = np.argmax(vec @ cen.T, axis=1).astype(np.uint32)
    return item_n_vec, vec, cen, code


def make_maxsim(mvr_ref):
    """maxsim_<case>.npz: 3 seeded query sets (32 vectors at dim 128, 8 at
    dim 36) and the reference's vectorSetDistance of each against every item's
    decoded vectors and raw vectors of the codec case."""
    for name, n_bit, dim, n_item, max_len, n_cent, seed, coarse in CASES:
        z = np.load(os.path.join(HERE, f"codec_{name}.npz"))
        rng = np.random.default_rng(seed + 1000)
        nq = 32 if dim == 128 else 8
        q = rng.standard_normal((3, nq, dim)).astype(np.float32)
        q /= np.linalg.norm(q, axis=2, keepdims=True)
        q = q.astype(np.float32)
        off = np.concatenate([[0], np.cumsum(z["item_n_vec"].astype(np.int64))])
        dec, raw = z["decoded"], z["vec"]
        ms_dec = np.array([[mvr_ref.vector_set_distance(q[i], dec[off[j]:off[j + 1]])
                            for j in range(n_item)] for i in range(3)], np.float32)
        ms_raw = np.array([[mvr_ref.vector_set_distance(q[i], raw[off[j]:off[j + 1]])
                            for j in range(n_item)] for i in range(3)], np.float32)
        np.savez_compressed(os.path.join(HERE, f"maxsim_{name}.npz"), query=q,
                            maxsim_decoded=ms_dec, maxsim_raw=ms_raw)
        print(name, "maxsim", ms_dec[0, :4])


def main():
    sys.path.insert(0, os.path.join(ROOT, "oracle", "_ref"))
    import mvr_ref  # noqa: E402  (reference code, compiled from its sources)

    what = sys.argv[1] if len(sys.argv) > 1 else "all"
    if what in ("all", "codec"):
        make_codec(mvr_ref)
    if what in ("all", "maxsim"):
        make_maxsim(mvr_ref)
    print("fixtures:", sorted(os.path.basename(p) for p in glob.glob(os.path.join(HERE, "*.npz"))))


def make_codec(mvr_ref):
    for name, n_bit, dim, n_item, max_len, n_cent, seed, coarse in CASES:
        item_n_vec, vec, cen, code = make_inputs(n_bit, dim, n_item, max_len, n_cent,
                                                 seed, coarse)
        cutoff, weight = mvr_ref.compute_quantized_scalar(vec, cen, code, n_bit)
        cutoff = np.asarray(cutoff, np.float32)
        weight = np.asarray(weight, np.float32)
        comp = mvr_ref.CompressResidualCode(cen, cutoff, weight, n_bit)
        residual = np.asarray(comp.compute_residual_code(vec, code)[0], np.uint8)
        table = mvr_ref.decode_table(n_bit, weight)
        decoded = mvr_ref.decode_all(residual, weight, item_n_vec, cen, code, n_bit)
        with tempfile.TemporaryDirectory() as td:
            path = os.path.join(td, "ivf.index")
            off, size, ids = mvr_ref.ivf_build(code.tolist(), item_n_vec.tolist(),
                                               len(code), n_item, n_cent, path)
            ivf_bytes = np.frombuffer(open(path, "rb").read(), np.uint8)
            lists = mvr_ref.read_ivf_index(path)
        assert sum(len(x) for x in lists) == len(ids)
        np.savez_compressed(
            os.path.join(HERE, f"codec_{name}.npz"),
            n_bit=n_bit, item_n_vec=item_n_vec, vec=vec, centroid=cen, code=code,
            cutoff=cutoff, weight=weight, residual=residual, table=table,
            decoded=decoded, ivf_off=np.asarray(off, np.uint64),
            ivf_size=np.asarray(size, np.uint32), ivf_ids=np.asarray(ids, np.uint32),
            ivf_bytes=ivf_bytes)
        print(name, "n_vec", len(code), "cutoff", cutoff, "weight", weight)


if __name__ == "__main__":
    main()
