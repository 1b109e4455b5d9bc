"""Reference on-disk formats: ivf.index bytes equal the reference's own
IVFIndex::save output (golden), index directories round-trip, libmvr's loader
rejects malformed inputs before touching a device."""
import glob
import os

import numpy as np
import pytest

from mvr import _lib, formats

GOLDEN = sorted(glob.glob(os.path.join(os.path.dirname(__file__), "golden", "codec_*.npz")))


@pytest.mark.parametrize("path", GOLDEN, ids=[os.path.basename(p)[6:-4] for p in GOLDEN])
def test_ivf_bytes_match_reference(path, tmp_path):
    g = np.load(path)
    out = tmp_path / "ivf.index"
    formats.write_ivf(out, g["ivf_off"], g["ivf_size"], g["ivf_ids"])
    assert out.read_bytes() == g["ivf_bytes"].tobytes()
    off, size, ids = formats.read_ivf(out)
    np.testing.assert_array_equal(ids, g["ivf_ids"])


def test_index_dir_round_trip(tmp_path):
    g = np.load(GOLDEN[1])
    formats.write_index_dir(tmp_path, g["item_n_vec"], g["centroid"], g["code"], g["weight"],
                            g["residual"], g["ivf_off"], g["ivf_size"], g["ivf_ids"])
    assert np.load(tmp_path / "vq_code_l.npy").dtype == np.int32  # as the reference saves it
    r = formats.read_index_dir(tmp_path)
    np.testing.assert_array_equal(r["vq_code"], g["code"])
    np.testing.assert_array_equal(r["residual"], g["residual"])


def test_truncated_ivf_rejected(tmp_path):
    g = np.load(GOLDEN[0])
    formats.write_index_dir(tmp_path, g["item_n_vec"], g["centroid"], g["code"], g["weight"],
                            g["residual"], g["ivf_off"], g["ivf_size"], g["ivf_ids"])
    data = (tmp_path / "ivf.index").read_bytes()
    (tmp_path / "ivf.index").write_bytes(data[:-4])
    with pytest.raises(ValueError):
        formats.read_ivf(tmp_path / "ivf.index")
    import ctypes as C
    h = C.c_void_p()
    rc = _lib.lib().mvr_index_load(str(tmp_path).encode(), len(g["centroid"]), int(g["n_bit"]), 0,
                                   C.byref(h))
    assert rc == _lib.MVR_ERR_IO
    assert b"truncated" in _lib.lib().mvr_last_error()


def test_recall_metric():
    gnd = [np.array([1, 2, 3]), np.array([4, 5, 6])]
    est = [np.array([3, 2, 9]), np.array([7, 8, 9])]
    np.testing.assert_allclose(formats.recall_at_k(gnd, est, 3), [2 / 3, 0.0])
