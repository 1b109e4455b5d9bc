"""The oracle against the reference's own codec / IVF / MaxSim outputs
(golden fixtures produced by tests/golden/make_golden.py from the reference
code)."""
import glob
import os

import numpy as np
import pytest

import pyoracle

GOLDEN = sorted(glob.glob(os.path.join(os.path.dirname(__file__), "golden", "codec_*.npz")))


@pytest.fixture(params=GOLDEN, ids=[os.path.basename(p)[6:-4] for p in GOLDEN])
def case(request):
    return dict(np.load(request.param))


def test_fixtures_present():
    assert len(GOLDEN) >= 6
    for p in GOLDEN:
        assert os.path.exists(p.replace("codec_", "maxsim_"))


def test_quantile_cutoffs_and_weights(case):
    cut, w = pyoracle.quantize(case["vec"], case["centroid"], case["code"], int(case["n_bit"]))
    np.testing.assert_array_equal(cut, case["cutoff"])
    np.testing.assert_array_equal(w, case["weight"])


def test_residual_pack_bit_exact(case):
    res = pyoracle.pack_residual(case["vec"], case["centroid"], case["code"], case["cutoff"],
                                 int(case["n_bit"]))
    np.testing.assert_array_equal(res, case["residual"])


def test_decode_table_bit_exact(case):
    t = pyoracle.decode_table(int(case["n_bit"]), case["weight"])
    np.testing.assert_array_equal(t, case["table"])


def test_decode_bit_exact(case):
    o = pyoracle.Oracle(case["item_n_vec"], case["centroid"], case["code"], case["residual"],
                        case["weight"], case["ivf_off"], case["ivf_size"], case["ivf_ids"],
                        int(case["n_bit"]))
    np.testing.assert_array_equal(o.decompress_all(), case["decoded"])


def test_bucket_indices_reconstruct_decode(case):
    n_bit = int(case["n_bit"])
    n_vec, dim = case["vec"].shape
    b = pyoracle.unpack_buckets(case["residual"], n_vec, dim, n_bit)
    assert b.max() < (1 << n_bit)
    rec = case["centroid"][case["code"]] + case["weight"][b]
    np.testing.assert_array_equal(rec.astype(np.float32), case["decoded"])


def test_ivf_lists_bit_exact(case):
    off, size, ids = pyoracle.ivf_build(case["code"], case["item_n_vec"], len(case["centroid"]))
    np.testing.assert_array_equal(off, case["ivf_off"])
    np.testing.assert_array_equal(size, case["ivf_size"])
    np.testing.assert_array_equal(ids, case["ivf_ids"])


def test_maxsim_matches_reference_distance(case, request):
    """The oracle's MaxSim of a query set against a doc's decoded vectors
    (PP semantics: sum over query vectors of the max over the doc's true
    length; the FP32 rerank's arithmetic) against the reference's own
    vectorSetDistance (Distance.hpp) over the reference's decoded vectors,
    and the oracle's FP64 exhaustive MaxSim over the raw vectors against the
    same reference function over the raw vectors.  The reference accumulates
    each dot with separate FP32 multiplies and adds, the oracle with fused
    multiply-adds (FP64 for the exhaustive one): equal to FP32 rounding."""
    path = request.node.callspec.params["case"]
    z = np.load(path.replace("codec_", "maxsim_"))
    o = pyoracle.Oracle(case["item_n_vec"], case["centroid"], case["code"], case["residual"],
                        case["weight"], case["ivf_off"], case["ivf_size"], case["ivf_ids"],
                        int(case["n_bit"]))
    n_item = len(case["item_n_vec"])
    q = z["query"]
    ours = np.array([[o.maxsim_item(q[i], j, pyoracle.SEM_PP) for j in range(n_item)]
                     for i in range(len(q))], np.float32)
    np.testing.assert_allclose(ours, z["maxsim_decoded"], rtol=2e-6, atol=2e-6)
    nq = q.shape[1]
    off = np.arange(len(q) + 1, dtype=np.uint64) * nq
    s, ids = pyoracle.exhaustive_f64(q.reshape(-1, q.shape[2]), off, case["vec"],
                                     case["item_n_vec"], n_item)
    raw = np.zeros((len(q), n_item))
    np.put_along_axis(raw, ids.astype(np.int64), s, axis=1)
    np.testing.assert_allclose(raw, z["maxsim_raw"], rtol=2e-6, atol=2e-6)

