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


def test_plaid_igp_conversion_round_trip_and_chunks(tmp_path):
    """mvr.convert: IGP dir -> PLAID dir -> IGP dir keeps codes, residual
    bytes and lists exactly (centroids and weights pass through fp16); a
    PLAID directory split into two chunks reads back the same."""
    import json
    import torch
    from mvr import convert, formats
    from helpers import tiny_index
    ix = tiny_index(n_doc=120, n_centroid=16, n_bit=4, seed=9)
    a, p, b = tmp_path / "igp", tmp_path / "plaid", tmp_path / "igp2"
    formats.write_index_dir(str(a), ix["item_n_vec"], ix["centroid"], ix["vq_code"],
                            ix["weight"], ix["residual"], ix["ivf_off"], ix["ivf_size"],
                            ix["ivf_ids"])
    assert convert.main(["igp2plaid", str(a), str(p), "4"]) == 0
    assert convert.main(["plaid2igp", str(p), str(b)]) == 0
    x, y = formats.read_index_dir(str(a)), formats.read_index_dir(str(b))
    for k in ("item_n_vec", "vq_code", "residual", "ivf_off", "ivf_size", "ivf_ids"):
        np.testing.assert_array_equal(x[k], y[k], err_msg=k)
    np.testing.assert_array_equal(y["centroid"], x["centroid"].astype(np.float16).astype(np.float32))
    np.testing.assert_array_equal(y["weight"], x["weight"].astype(np.float16).astype(np.float32))
    # two chunks: docs [0, 50) and [50, 120)
    one = formats.read_plaid_index(str(p))
    n0 = int(ix["item_n_vec"][:50].sum())
    codes = torch.load(p / "0.codes.pt")
    res = torch.load(p / "0.residuals.pt")
    dl = json.load(open(p / "doclens.0.json"))
    torch.save(codes[:n0].clone(), p / "0.codes.pt")
    torch.save(res[:n0].clone(), p / "0.residuals.pt")
    json.dump(dl[:50], open(p / "doclens.0.json", "w"))
    torch.save(codes[n0:].clone(), p / "1.codes.pt")
    torch.save(res[n0:].clone(), p / "1.residuals.pt")
    json.dump(dl[50:], open(p / "doclens.1.json", "w"))
    meta = json.load(open(p / "metadata.json"))
    meta["num_chunks"] = 2
    json.dump(meta, open(p / "metadata.json", "w"))
    two = formats.read_plaid_index(str(p))
    for k, v in one.items():
        np.testing.assert_array_equal(np.asarray(two[k]), np.asarray(v), err_msg=k)
    assert convert.main(["bogus"]) == 2
