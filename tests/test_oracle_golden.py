"""The oracle against the reference's own codec / IVF outputs (golden
fixtures produced by tests/golden/make_golden.py from the reference code)."""
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
