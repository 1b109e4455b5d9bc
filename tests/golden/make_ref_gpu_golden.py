"""Generates tests/golden/refgpu_*.npz from the REFERENCE's own GPU search
kernels, run on a GPU through oracle/_ref/libref_gpu.so (oracle/ref_gpu.cu,
built by `make -C oracle ref`): the reference's cuBLAS centroid scores, its
filter kernels' candidate sets and per-(candidate, query token) maxima, and
its rerank kernels' decoded vectors and per-(query token, doc) MaxSim maxima.

Each case stores its whole input (a small seeded index built with the
oracle's codec, its queries, and the oracle's probe lists and shortlist that
were fed to the reference filter and rerank) beside the reference outputs,
so the fixtures need no regeneration to be checked.  Run on a machine with a
GPU:

    python tests/golden/make_ref_gpu_golden.py <out dir>
"""
import ctypes as C
import hashlib
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.dirname(HERE))
from helpers import make_queries, oracle_of, tiny_index  # noqa: E402

# (name, n_bit, n_doc, doc length range, n_centroid, seed, n_query, query tokens, nprobe, P)
# query tokens * P is a multiple of 256 (the reference reduceMax's blocks)
CASES = [
    ("b2", 2, 400, (4, 12), 128, 71, 2, 32, 4, 120),
    ("b4", 4, 240, (4, 12), 96, 72, 2, 16, 4, 48),
    ("b1", 1, 240, (4, 12), 96, 73, 2, 8, 3, 64),
]


def _p(a):
    return C.c_void_p(a.ctypes.data)


def lib():
    so = os.path.join(ROOT, "oracle", "_ref", "libref_gpu.so")
    L = C.CDLL(so)
    for f in ("ref_centroid_scores", "ref_filter", "ref_rerank"):
        getattr(L, f).restype = C.c_int
    return L


def run_case(L, name, n_bit, n_doc, lrange, n_cent, seed, n_query, n_tok, nprobe, P):
    rng = np.random.default_rng(seed)
    lengths = rng.integers(lrange[0], lrange[1] + 1, n_doc).astype(np.uint32)
    ix = tiny_index(n_doc=n_doc, n_centroid=n_cent, n_bit=n_bit, seed=seed, lengths=lengths)
    o = oracle_of(ix)
    q, off = make_queries(ix, n_query, n_tok, seed=seed + 1)
    item_off = np.zeros(n_doc, np.uint64)
    item_off[1:] = np.cumsum(lengths[:-1], dtype=np.uint64)
    out = dict(n_bit=np.uint32(n_bit), nprobe=np.uint32(nprobe), P=np.uint32(P),
               item_n_vec=lengths, centroid=ix["centroid"], vq_code=ix["vq_code"],
               residual=ix["residual"], weight=ix["weight"], ivf_off=ix["ivf_off"],
               ivf_size=ix["ivf_size"], ivf_ids=ix["ivf_ids"], query=q, q_off=off)
    S, probe_id, probe_score, cand_off, cand, qmax, short_id, vmax = [], [], [], [0], [], [], [], []
    vec_digest = []
    for i in range(n_query):
        qi = np.ascontiguousarray(q[off[i]:off[i + 1]])
        nq = qi.shape[0]
        r = o.search_one(qi, 10, nprobe, P)
        s = np.zeros((nq, n_cent), np.float32)
        assert L.ref_centroid_scores(_p(qi), nq, _p(ix["centroid"]), n_cent, 128, _p(s)) == 0
        pid = np.ascontiguousarray(r["probe_id"], np.uint32)
        psc = np.ascontiguousarray(r["probe_score"], np.float32)
        c_out = np.zeros(n_doc, np.uint32)
        n_c = np.zeros(1, np.uint32)
        qm = np.zeros((n_doc, nq), np.float32)
        assert L.ref_filter(n_doc, n_cent, _p(ix["ivf_off"]), _p(ix["ivf_size"]),
                            _p(ix["ivf_ids"]), C.c_uint64(len(ix["ivf_ids"])), _p(pid),
                            _p(psc), nq, nprobe, _p(c_out), _p(n_c), _p(qm)) == 0
        nc = int(n_c[0])
        sid = np.ascontiguousarray(r["short_id"], np.uint32)
        assert len(sid) == P, f"{name}: shortlist {len(sid)} < P {P}"
        ntok = int(lengths[sid].sum())
        vec = np.zeros((ntok, 128), np.float32)
        mx = np.zeros((nq, P), np.float32)
        assert L.ref_rerank(n_doc, _p(lengths), _p(item_off), C.c_uint64(int(lengths.sum())),
                            _p(ix["centroid"]), n_cent, 128, _p(ix["vq_code"]),
                            _p(ix["residual"]), _p(ix["weight"]), n_bit, _p(qi), nq, _p(sid),
                            P, _p(vec), _p(mx)) == 0
        S.append(s)
        probe_id.append(pid)
        probe_score.append(psc)
        cand.append(c_out[:nc])
        qmax.append(qm[:nc])
        cand_off.append(cand_off[-1] + nc)
        short_id.append(sid)
        vmax.append(mx)
        vec_digest.append(hashlib.sha256(vec.tobytes()).hexdigest())
        if i == 0:
            out["vec_first_doc"] = vec[: int(lengths[sid[0]])]
    out.update(ref_S=np.concatenate(S), probe_id=np.concatenate(probe_id),
               probe_score=np.concatenate(probe_score), ref_cand=np.concatenate(cand),
               ref_cand_off=np.asarray(cand_off, np.uint64), ref_qmax=np.concatenate(qmax),
               short_id=np.stack(short_id), ref_max=np.stack(vmax),
               ref_vec_sha256=np.asarray(vec_digest))
    return out


def main(out_dir=HERE):
    L = lib()
    os.makedirs(out_dir, exist_ok=True)
    for case in CASES:
        d = run_case(L, *case)
        path = os.path.join(out_dir, f"refgpu_{case[0]}.npz")
        np.savez_compressed(path, **d)
        print("wrote", path, os.path.getsize(path), "bytes")


if __name__ == "__main__":
    main(*sys.argv[1:])
