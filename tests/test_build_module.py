"""GPGPUBuildIndexPackGPU, the pybind11 module with the reference build
module's names and arguments (src/app/build_index/GPGPUBuildIndexPackGPU.cpp:
14-44), against the oracle's restatement of the reference codec and IVF
builder (itself checked against the reference's compiled code and golden
vectors): the IVF build and its file bytes on the CPU; the quantizer's
cutoffs / weights and the packed residual codes on the GPU."""
import os
import sys

import numpy as np
import pytest

import pyoracle

LIB = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))),
                   "multi-vector-retrieval-gpu_b200", "lib")


def module():
    if LIB not in sys.path:
        sys.path.insert(0, LIB)
    import GPGPUBuildIndexPackGPU
    return GPGPUBuildIndexPackGPU


def corpus(seed, n_item=300, n_cent=40):
    rng = np.random.default_rng(seed)
    item_n_vec = rng.integers(1, 30, n_item).astype(np.uint32)
    n_vec = int(item_n_vec.sum())
    vec = rng.standard_normal((n_vec, 128)).astype(np.float32)
    vec /= np.linalg.norm(vec, axis=1, keepdims=True)
    cen = rng.standard_normal((n_cent, 128)).astype(np.float32)
    cen /= np.linalg.norm(cen, axis=1, keepdims=True)
    code = pyoracle.assign(vec, cen)
    return vec, cen, np.asarray(code, np.uint32), item_n_vec


def test_module_names_match_the_reference_module():
    m = module()
    assert callable(m.compute_quantized_scalar)
    for name in ("compute_residual_code",):
        assert hasattr(m.CompressResidualCode, name)
    for name in ("build", "save"):
        assert hasattr(m.IVFIndex, name)


@pytest.mark.parametrize("seed", [1, 2])
def test_ivf_index_build_and_save_match_the_oracle(tmp_path, seed):
    from mvr import formats
    m = module()
    vec, cen, code, item_n_vec = corpus(seed)
    ivf = m.IVFIndex(vq_code_l=code, item_n_vec_l=item_n_vec, n_vec=len(code),
                     n_item=len(item_n_vec), n_centroid=len(cen))
    ivf.build()
    ivf.save(location=str(tmp_path / "a.index"))
    off, size, ids = pyoracle.ivf_build(code, item_n_vec, len(cen))
    formats.write_ivf(str(tmp_path / "b.index"), off, size, ids)
    assert (tmp_path / "a.index").read_bytes() == (tmp_path / "b.index").read_bytes()


def test_ivf_index_rejects_inconsistent_sizes():
    m = module()
    with pytest.raises(ValueError):
        m.IVFIndex(vq_code_l=np.zeros(10, np.uint32), item_n_vec_l=np.array([3, 4], np.uint32),
                   n_vec=10, n_item=2, n_centroid=4)


@pytest.mark.gpu
@pytest.mark.parametrize("n_bit", [1, 2, 4, 8])
def test_quantizer_and_residual_codes_match_the_oracle(n_bit):
    m = module()
    vec, cen, code, _ = corpus(10 + n_bit, n_item=400)
    cut, w = m.compute_quantized_scalar(item_vec_l=vec, centroid_l=cen, code_l=code, n_bit=n_bit)
    rcut, rw = pyoracle.quantize(vec, cen, code, n_bit)
    np.testing.assert_array_equal(np.asarray(cut, np.float32), rcut)
    np.testing.assert_array_equal(np.asarray(w, np.float32), rw)
    sq = m.CompressResidualCode(centroid_l=cen, cutoff_l=cut, weight_l=w, n_bit=n_bit)
    assert sq.n_val_per_vec == 128 * n_bit // 8
    # the reference script calls it chunk by chunk and unpacks a 1-tuple
    got = []
    for s in range(0, len(vec), 1000):
        chunk, = sq.compute_residual_code(vec_l=vec[s:s + 1000], code_l=code[s:s + 1000])
        got.append(np.array(chunk, dtype=np.uint8))
    np.testing.assert_array_equal(np.concatenate(got),
                                  pyoracle.pack_residual(vec, cen, code, rcut, n_bit))
