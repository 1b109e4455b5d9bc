"""The search stages pinned to REFERENCE output: fixtures made by the
reference's own GPU kernels (FilterPP.hpp gather_ivf_data /
find_candidate_item / max_qvec_doc_score, RerankPP.hpp gather_vq_data /
decompressAndAddResidual / reduceMax, MatrixMulCUBLAS.hpp MatrixMultiply),
compiled unmodified and run on a GPU by tests/golden/make_ref_gpu_golden.py.

Each fixture holds a small index, its queries, the probe lists and shortlist
the oracle chose for them (the reference filter and rerank were fed exactly
those), and the reference's outputs.  Checked here:

* centroid scores: the canonical FP32 chain is within 2e-6 (a few ulps) of
  the reference's cuBLAS S = Q.C^T + 1, and the probe ids equal the
  reference-score top-nprobe wherever the ranking gap exceeds 1e-5;
* candidate sets: integer-exact;
* approximate scores: the exact (2^-32 fixed-point) sum of the reference's
  per-(candidate, query token) maxima equals the oracle's / CUDA path's
  approximate score bit for bit -- the maxima themselves are equal because the
  FP32 inputs are;
* decoded doc tokens: bit-exact (sha256 of every shortlisted token);
* MaxSim: per (query token, doc) maxima within 1e-5 of FP64 over the decoded
  tokens, and the exact FP32 doc scores within 1e-5 relative of the sum of the
  reference's maxima (cuBLAS sums in another order than the canonical chain).
"""
import glob
import hashlib
import os

import numpy as np
import pytest

import pyoracle

HERE = os.path.dirname(os.path.abspath(__file__))
FILES = sorted(glob.glob(os.path.join(HERE, "golden", "refgpu_*.npz")))
TOL = 1e-5


def fixed_sum(rows):
    """The canonical approximate score of each row: every term v as
    round(v * 2^32) in int64, the integer sum rounded once to FP32, scaled by
    2^-32 (oracle/mvr_oracle.c orc_fixed / orc_unfixed)."""
    t = np.rint(rows.astype(np.float64) * 4294967296.0).astype(np.int64)
    return t.sum(axis=1).astype(np.float32) * np.float32(1.0 / 4294967296.0)


def load(path):
    f = dict(np.load(path))
    f["name"] = os.path.basename(path)
    return f


def queries(f):
    off = f["q_off"]
    return [np.ascontiguousarray(f["query"][off[i]:off[i + 1]]) for i in range(len(off) - 1)]


def per_query(f, i):
    """Reference outputs of query i."""
    co = f["ref_cand_off"]
    nq = int(f["q_off"][i + 1] - f["q_off"][i])
    sl = slice(int(co[i]), int(co[i + 1]))
    s0 = int(f["q_off"][i])
    return dict(S=f["ref_S"][s0:s0 + nq], probe_id=f["probe_id"][s0:s0 + nq],
                probe_score=f["probe_score"][s0:s0 + nq], cand=f["ref_cand"][sl],
                qmax=f["ref_qmax"][sl], short_id=f["short_id"][i], vmax=f["ref_max"][i],
                vec_sha=str(f["ref_vec_sha256"][i]))


def oracle(f):
    return pyoracle.Oracle(f["item_n_vec"], f["centroid"], f["vq_code"], f["residual"],
                           f["weight"], f["ivf_off"], f["ivf_size"], f["ivf_ids"], int(f["n_bit"]))


def ref_probe(S, nprobe):
    """Top-nprobe per token of the reference scores by (score desc, id asc),
    with a flag per token: True where the nprobe-th and (nprobe+1)-th scores
    are more than TOL apart (the selection cannot flip under rounding)."""
    order = np.lexsort((np.broadcast_to(np.arange(S.shape[1]), S.shape), -S.astype(np.float64)))
    top = order[:, :nprobe]
    srt = np.take_along_axis(S, order, axis=1)
    safe = (srt[:, nprobe - 1] - srt[:, nprobe]) > TOL if S.shape[1] > nprobe else \
        np.ones(S.shape[0], bool)
    return top, safe


def check_probe(f, r, pid):
    top, safe = ref_probe(r["S"], int(f["nprobe"]))
    assert safe.any()
    for t in np.flatnonzero(safe):
        assert set(pid[t]) == set(top[t]), (f["name"], t)


pytestmark = pytest.mark.skipif(not FILES, reason="reference GPU fixtures absent")


@pytest.mark.parametrize("path", FILES, ids=[os.path.basename(p) for p in FILES])
def test_oracle_pinned_to_reference_gpu_kernels(path):
    f = load(path)
    o = oracle(f)
    nprobe, P = int(f["nprobe"]), int(f["P"])
    for i, qi in enumerate(queries(f)):
        r = per_query(f, i)
        got = o.search_one(qi, 10, nprobe, P)
        # the fixture's inputs are the oracle's own choices
        np.testing.assert_array_equal(got["probe_id"], r["probe_id"])
        np.testing.assert_array_equal(got["short_id"], r["short_id"])
        # centroid scores and probes vs the reference's cuBLAS scores
        S = pyoracle.centroid_scores(qi, f["centroid"])
        np.testing.assert_allclose(S, r["S"], rtol=0, atol=2e-6)
        check_probe(f, r, got["probe_id"])
        # candidate set and approximate scores vs the reference filter kernels
        np.testing.assert_array_equal(got["cand_id"], r["cand"])
        np.testing.assert_array_equal(got["cand_score"], fixed_sum(r["qmax"]))
        # decoded tokens vs decompressAndAddResidual
        dec = np.concatenate([o.decompress_item(int(d)) for d in r["short_id"]])
        assert hashlib.sha256(dec.tobytes()).hexdigest() == r["vec_sha"]
        if i == 0:
            np.testing.assert_array_equal(o.decompress_item(int(r["short_id"][0])),
                                          f["vec_first_doc"])
        # MaxSim: reference per-(token, doc) maxima vs FP64, doc scores vs exact FP32
        q64 = qi.astype(np.float64)
        for j, d in enumerate(r["short_id"]):
            x = o.decompress_item(int(d)).astype(np.float64)
            m64 = (q64 @ x.T).max(axis=1)
            np.testing.assert_allclose(r["vmax"][:, j], m64, rtol=0, atol=TOL)
            ref_score = float(r["vmax"][:, j].astype(np.float64).sum())
            ex = got["short_exact"][j]
            assert abs(ex - ref_score) <= TOL * max(1.0, abs(ref_score)), (d, ex, ref_score)


@pytest.mark.gpu
@pytest.mark.parametrize("path", FILES, ids=[os.path.basename(p) for p in FILES])
def test_cuda_path_pinned_to_reference_gpu_kernels(path):
    from mvr import Index
    f = load(path)
    nprobe, P = int(f["nprobe"]), int(f["P"])
    with Index.from_arrays(f["item_n_vec"], f["centroid"], f["vq_code"], f["ivf_off"],
                           f["ivf_size"], f["ivf_ids"], f["weight"], int(f["n_bit"]),
                           f["residual"]) as g:
        for i, qi in enumerate(queries(f)):
            r = per_query(f, i)
            t = g.trace(qi, 10, nprobe, P)
            np.testing.assert_array_equal(t["probe_id"], r["probe_id"])
            np.testing.assert_array_equal(t["probe_score"], r["probe_score"])
            check_probe(f, r, t["probe_id"])
            np.testing.assert_array_equal(t["cand_id"], r["cand"])
            np.testing.assert_array_equal(t["cand_score"], fixed_sum(r["qmax"]))
            np.testing.assert_array_equal(t["short_id"], np.sort(r["short_id"]))
            order = np.argsort(r["short_id"])
            ref_scores = r["vmax"].astype(np.float64).sum(axis=0)[order]
            np.testing.assert_allclose(t["short_exact"], ref_scores, rtol=TOL, atol=TOL)
            vid = np.concatenate([np.arange(int(s), int(s) + int(n), dtype=np.uint64) for s, n in
                                  zip(np.concatenate([[0], np.cumsum(f["item_n_vec"].astype(
                                      np.uint64))])[r["short_id"]], f["item_n_vec"][r["short_id"]])])
            dec = g.decompress(vid)
            assert hashlib.sha256(dec.tobytes()).hexdigest() == r["vec_sha"]
