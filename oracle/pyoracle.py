"""ctypes binding of the CPU oracle (oracle/liboracle.so).

Test infrastructure only: imported by tests/, by __graft_entry__.smoke() as the
checker, and by bench.py's cpu_baseline / --impl reference leg.  The product
(libmvr) never calls it.
"""
import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None

SEM_PP = 0
SEM_BASIC = 1


class OrcIndex(C.Structure):
    _fields_ = [
        ("n_item", C.c_uint32), ("n_centroid", C.c_uint32), ("dim", C.c_uint32),
        ("n_bit", C.c_uint32), ("n_vec", C.c_uint64), ("n_ele_ivf", C.c_uint64),
        ("item_n_vec", C.c_void_p), ("item_off", C.c_void_p),
        ("centroid", C.c_void_p), ("vq_code", C.c_void_p),
        ("residual", C.c_void_p), ("weight", C.c_void_p),
        ("ivf_off", C.c_void_p), ("ivf_size", C.c_void_p),
        ("ivf_ids", C.c_void_p), ("max_item_n_vec", C.c_uint32),
    ]


class OrcTrace(C.Structure):
    _fields_ = [
        ("probe_id", C.c_void_p), ("probe_score", C.c_void_p),
        ("cand_cap", C.c_uint32), ("n_cand", C.c_uint32),
        ("cand_id", C.c_void_p), ("cand_score", C.c_void_p),
        ("n_short", C.c_uint32), ("short_id", C.c_void_p),
        ("short_approx", C.c_void_p), ("short_exact", C.c_void_p),
    ]


def lib():
    global _LIB
    if _LIB is None:
        path = os.path.join(_HERE, "liboracle.so")
        if not os.path.exists(path):
            raise RuntimeError(f"oracle library missing: {path} (run make -C oracle)")
        _LIB = C.CDLL(path)
    return _LIB


def _p(a):
    return C.c_void_p(a.ctypes.data) if a is not None else None


def _c(a, dtype):
    return np.ascontiguousarray(a, dtype=dtype)


class Oracle:
    """Holds contiguous copies of an index's arrays and an OrcIndex view."""

    def __init__(self, item_n_vec, centroid, vq_code, residual, weight,
                 ivf_off, ivf_size, ivf_ids, n_bit):
        self.item_n_vec = _c(item_n_vec, np.uint32)
        self.item_off = np.zeros(len(self.item_n_vec), np.uint64)
        if len(self.item_n_vec) > 1:
            self.item_off[1:] = np.cumsum(self.item_n_vec[:-1], dtype=np.uint64)
        self.centroid = _c(centroid, np.float32)
        self.vq_code = _c(vq_code, np.uint32)
        self.residual = _c(residual, np.uint8)
        self.weight = _c(weight, np.float32)
        self.ivf_off = _c(ivf_off, np.uint64)
        self.ivf_size = _c(ivf_size, np.uint32)
        self.ivf_ids = _c(ivf_ids, np.uint32)
        self.n_bit = int(n_bit)
        ix = OrcIndex()
        ix.n_item = len(self.item_n_vec)
        ix.n_centroid, ix.dim = self.centroid.shape
        ix.n_bit = self.n_bit
        ix.n_vec = len(self.vq_code)
        ix.n_ele_ivf = len(self.ivf_ids)
        for name in ("item_n_vec", "item_off", "centroid", "vq_code", "residual",
                     "weight", "ivf_off", "ivf_size", "ivf_ids"):
            setattr(ix, name, getattr(self, name).ctypes.data)
        ix.max_item_n_vec = int(self.item_n_vec.max()) if ix.n_item else 0
        self.ix = ix

    @property
    def dim(self):
        return self.centroid.shape[1]

    def search_one(self, q, topk, nprobe, probe_topk, semantics=SEM_PP,
                   trace=True):
        q = _c(q, np.float32)
        nq = q.shape[0]
        out_s = np.zeros(topk, np.float32)
        out_i = np.zeros(topk, np.uint32)
        tr = None
        arrs = {}
        if trace:
            cap = self.ix.n_item
            arrs = dict(
                probe_id=np.zeros(nq * nprobe, np.uint32),
                probe_score=np.zeros(nq * nprobe, np.float32),
                cand_id=np.zeros(cap, np.uint32),
                cand_score=np.zeros(cap, np.float32),
                short_id=np.zeros(probe_topk, np.uint32),
                short_approx=np.zeros(probe_topk, np.float32),
                short_exact=np.zeros(probe_topk, np.float32),
            )
            tr = OrcTrace()
            tr.cand_cap = cap
            for k, v in arrs.items():
                setattr(tr, k, v.ctypes.data)
        rc = lib().orc_search_one(C.byref(self.ix), _p(q), C.c_uint32(nq),
                                  C.c_uint32(topk), C.c_uint32(nprobe),
                                  C.c_uint32(probe_topk), C.c_int(semantics),
                                  C.byref(tr) if tr is not None else None,
                                  _p(out_s), _p(out_i))
        if rc != 0:
            raise ValueError(f"orc_search_one failed rc={rc}")
        res = {"score": out_s, "id": out_i}
        if trace:
            n_cand, n_short = tr.n_cand, tr.n_short
            res.update(
                probe_id=arrs["probe_id"].reshape(nq, nprobe),
                probe_score=arrs["probe_score"].reshape(nq, nprobe),
                cand_id=arrs["cand_id"][:n_cand], cand_score=arrs["cand_score"][:n_cand],
                short_id=arrs["short_id"][:n_short],
                short_approx=arrs["short_approx"][:n_short],
                short_exact=arrs["short_exact"][:n_short])
        return res

    def search(self, q, q_tok_off, topk, nprobe, probe_topk, semantics=SEM_PP,
               n_threads=None):
        q = _c(q, np.float32)
        off = _c(q_tok_off, np.uint64)
        n_query = len(off) - 1
        out_s = np.zeros((n_query, topk), np.float32)
        out_i = np.zeros((n_query, topk), np.uint32)
        rc = lib().orc_search(C.byref(self.ix), _p(q), _p(off), C.c_uint32(n_query),
                              C.c_uint32(topk), C.c_uint32(nprobe),
                              C.c_uint32(probe_topk), C.c_int(semantics),
                              C.c_int(n_threads or os.cpu_count()), _p(out_s), _p(out_i))
        if rc != 0:
            raise ValueError(f"orc_search failed rc={rc}")
        return out_s, out_i

    def maxsim_item(self, q, item, semantics=SEM_PP):
        q = _c(q, np.float32)
        f = lib().orc_maxsim_item
        f.restype = C.c_float
        return f(C.byref(self.ix), _p(q), C.c_uint32(q.shape[0]), C.c_uint32(item),
                 C.c_int(semantics))

    def decompress_item(self, item):
        out = np.zeros((int(self.item_n_vec[item]), self.dim), np.float32)
        lib().orc_decompress_item(C.byref(self.ix), C.c_uint32(item), _p(out))
        return out

    def decompress_all(self):
        ids = np.arange(len(self.vq_code), dtype=np.uint64)
        out = np.zeros((len(ids), self.dim), np.float32)
        lib().orc_decompress(C.byref(self.ix), _p(ids), C.c_uint64(len(ids)), _p(out))
        return out


def decode_table(n_bit, weight):
    weight = _c(weight, np.float32)
    vpb = 8 // n_bit
    out = np.zeros((256, vpb), np.float32)
    lib().orc_decode_table(C.c_uint32(n_bit), _p(weight), _p(out))
    return out


def unpack_buckets(residual, n_vec, dim, n_bit):
    residual = _c(residual, np.uint8)
    out = np.zeros((n_vec, dim), np.uint8)
    lib().orc_unpack_buckets(_p(residual), C.c_uint64(n_vec), C.c_uint32(dim),
                             C.c_uint32(n_bit), _p(out))
    return out


def quantize(vec, centroid, code, n_bit):
    vec = _c(vec, np.float32)
    centroid = _c(centroid, np.float32)
    code = _c(code, np.uint32)
    cut = np.zeros((1 << n_bit) - 1, np.float32)
    w = np.zeros(1 << n_bit, np.float32)
    rc = lib().orc_quantize(_p(vec), C.c_uint64(vec.shape[0]), C.c_uint32(vec.shape[1]),
                            _p(centroid), _p(code), C.c_uint32(n_bit), _p(cut), _p(w))
    if rc:
        raise MemoryError("orc_quantize")
    return cut, w


def pack_residual(vec, centroid, code, cutoff, n_bit):
    vec = _c(vec, np.float32)
    centroid = _c(centroid, np.float32)
    code = _c(code, np.uint32)
    cutoff = _c(cutoff, np.float32)
    n, dim = vec.shape
    vpb = 8 // n_bit
    bpv = (dim + vpb - 1) // vpb
    out = np.zeros(n * bpv, np.uint8)
    lib().orc_pack_residual(_p(vec), C.c_uint64(n), C.c_uint32(dim), _p(centroid),
                            _p(code), _p(cutoff), C.c_uint32(n_bit), _p(out))
    return out


def ivf_build(code, item_n_vec, n_centroid):
    code = _c(code, np.uint32)
    item_n_vec = _c(item_n_vec, np.uint32)
    f = lib().orc_ivf_build
    f.restype = C.c_uint64
    n_ele = f(_p(code), _p(item_n_vec), C.c_uint32(len(item_n_vec)),
              C.c_uint32(n_centroid), None, None, None)
    off = np.zeros(n_centroid, np.uint64)
    size = np.zeros(n_centroid, np.uint32)
    ids = np.zeros(n_ele, np.uint32)
    f(_p(code), _p(item_n_vec), C.c_uint32(len(item_n_vec)), C.c_uint32(n_centroid),
      _p(off), _p(size), _p(ids))
    return off, size, ids


def assign(vec, centroid, n_threads=None):
    vec = _c(vec, np.float32)
    centroid = _c(centroid, np.float32)
    code = np.zeros(vec.shape[0], np.uint32)
    lib().orc_assign(_p(vec), C.c_uint64(vec.shape[0]), _p(centroid),
                     C.c_uint32(centroid.shape[0]), C.c_uint32(centroid.shape[1]),
                     C.c_int(n_threads or os.cpu_count()), _p(code))
    return code


def centroid_scores(q, centroid):
    q = _c(q, np.float32)
    centroid = _c(centroid, np.float32)
    S = np.zeros((q.shape[0], centroid.shape[0]), np.float32)
    lib().orc_centroid_scores(_p(q), C.c_uint32(q.shape[0]), _p(centroid),
                              C.c_uint32(centroid.shape[0]), C.c_uint32(centroid.shape[1]),
                              _p(S))
    return S


def exhaustive_f64(q, q_tok_off, tok, item_n_vec, topk, n_threads=None):
    q = _c(q, np.float32)
    off = _c(q_tok_off, np.uint64)
    tok = _c(tok, np.float32)
    item_n_vec = _c(item_n_vec, np.uint32)
    item_off = np.zeros(len(item_n_vec), np.uint64)
    if len(item_n_vec) > 1:
        item_off[1:] = np.cumsum(item_n_vec[:-1], dtype=np.uint64)
    n_query = len(off) - 1
    out_s = np.zeros((n_query, topk), np.float64)
    out_i = np.zeros((n_query, topk), np.uint32)
    lib().orc_exhaustive_f64(_p(q), _p(off), C.c_uint32(n_query), _p(tok),
                             _p(item_n_vec), _p(item_off), C.c_uint32(len(item_n_vec)),
                             C.c_uint32(tok.shape[1]), C.c_uint32(topk),
                             C.c_int(n_threads or os.cpu_count()), _p(out_s), _p(out_i))
    return out_s, out_i
