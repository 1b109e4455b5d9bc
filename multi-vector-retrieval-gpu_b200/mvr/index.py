"""Python surface of libmvr: load an index, search(queries, k).

The search entry points mirror the reference's method facades
(IGPGPUPP::search, src/impl/IGPGPUPP.hpp:253-331): queries are float32
[n_query, n_vec, 128] (or ragged rows + token offsets), results are
(scores float32 [n_query, k], ids uint32 [n_query, k]).
"""
import ctypes as C

import numpy as np

from . import _lib
from ._lib import check, lib

SEM_PP = _lib.MVR_SEM_PP
SEM_BASIC = _lib.MVR_SEM_BASIC
PREC_BF16 = _lib.MVR_PREC_BF16
PREC_FP8 = _lib.MVR_PREC_FP8
CAND_IMPUTE = _lib.MVR_CAND_IMPUTE
PRUNE = _lib.MVR_PRUNE


def _ptr(a):
    return C.c_void_p(a.ctypes.data) if a is not None else None


def _c(a, dtype):
    return np.ascontiguousarray(a, dtype=dtype)


def _flatten_queries(queries, tok_off):
    q = np.asarray(queries)
    if tok_off is None:
        if q.ndim != 3:
            raise ValueError("queries must be [n_query, n_vec, dim] when tok_off is None")
        return _c(q, np.float32), None, q.shape[0], q.shape[1]
    off = _c(tok_off, np.uint64)
    if q.ndim != 2:
        raise ValueError("ragged queries must be [total_tokens, dim]")
    return _c(q, np.float32), off, len(off) - 1, 0


class Index:
    def __init__(self, handle):
        self._h = handle

    # -- construction ------------------------------------------------------
    @classmethod
    def load(cls, index_dir, n_centroid, n_bit, device=0):
        h = C.c_void_p()
        check(lib().mvr_index_load(str(index_dir).encode(), n_centroid, n_bit, device, C.byref(h)))
        return cls(h)

    @classmethod
    def load_files(cls, item_n_vec_l, centroid_l, vq_code_l, ivf_index, weight_l, residual_code_l,
                   n_centroid, n_bit, device=0):
        h = C.c_void_p()
        names = [str(x).encode() for x in (item_n_vec_l, centroid_l, vq_code_l, ivf_index,
                                            weight_l, residual_code_l)]
        check(lib().mvr_index_load_files(*names, n_centroid, n_bit, device, C.byref(h)))
        return cls(h)

    @classmethod
    def from_arrays(cls, item_n_vec, centroid, vq_code, ivf_off, ivf_size, ivf_ids, weight, n_bit,
                    residual, device=0):
        arrs = [_c(item_n_vec, np.uint32), _c(centroid, np.float32), _c(vq_code, np.uint32),
                _c(ivf_off, np.uint64), _c(ivf_size, np.uint32), _c(ivf_ids, np.uint32),
                _c(weight, np.float32), _c(residual, np.uint8)]
        inv, cen, code, off, size, ids, w, res = arrs
        h = C.c_void_p()
        check(lib().mvr_index_from_arrays(_ptr(inv), len(inv), _ptr(cen), cen.shape[0],
                                          cen.shape[1], _ptr(code), len(code), _ptr(off),
                                          _ptr(size), _ptr(ids), len(ids), _ptr(w), n_bit,
                                          _ptr(res), device, C.byref(h)))
        return cls(h)

    @classmethod
    def from_plaid_dir(cls, path, device=0):
        """A PLAID index directory (the reference's ColBERT baseline) loaded
        as an IGP index: its centroids, codes, bucket weights and IVF lists,
        residual bits re-laid (formats.read_plaid_index)."""
        from . import formats
        ix = formats.read_plaid_index(path)
        return cls.from_arrays(ix["item_n_vec"], ix["centroid"], ix["vq_code"], ix["ivf_off"],
                               ix["ivf_size"], ix["ivf_ids"], ix["weight"], ix["n_bit"],
                               ix["residual"], device=device)

    @classmethod
    def from_device_arrays(cls, item_n_vec, centroid, vq_code, ivf_off, ivf_size, ivf_ids, weight,
                           n_bit, residual, device=0):
        """Arguments are CUDA tensors (uint32 as int32 storage is accepted)."""
        for t in (item_n_vec, centroid, vq_code, ivf_off, ivf_size, ivf_ids, weight, residual):
            assert t.is_cuda and t.is_contiguous()
        h = C.c_void_p()
        check(lib().mvr_index_from_device_arrays(
            C.c_void_p(item_n_vec.data_ptr()), item_n_vec.numel(),
            C.c_void_p(centroid.data_ptr()), centroid.shape[0], centroid.shape[1],
            C.c_void_p(vq_code.data_ptr()), vq_code.numel(), C.c_void_p(ivf_off.data_ptr()),
            C.c_void_p(ivf_size.data_ptr()), C.c_void_p(ivf_ids.data_ptr()), ivf_ids.numel(),
            C.c_void_p(weight.data_ptr()), n_bit, C.c_void_p(residual.data_ptr()), device,
            C.byref(h)))
        return cls(h)

    def close(self):
        if self._h:
            lib().mvr_index_free(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # -- info ------------------------------------------------------------
    def info(self):
        inf = _lib.IndexInfo()
        check(lib().mvr_index_get_info(self._h, C.byref(inf)))
        return {k: getattr(inf, k) for k, _ in inf._fields_}

    def set_batch(self, max_batch_queries):
        check(lib().mvr_index_set_batch(self._h, max_batch_queries))

    def set_rescore(self, n_rescore):
        check(lib().mvr_index_set_rescore(self._h, n_rescore))

    def set_pruner(self, params, keep, margin):
        """Learned pruner of MVR_PRUNE searches: params float32 [74753]
        (None removes it), keep docs per query, confidence margin."""
        if params is None:
            check(lib().mvr_index_set_pruner(self._h, None, 0, 0.0))
            return
        p = _c(params, np.float32)
        check(lib().mvr_index_set_pruner(self._h, _ptr(p), int(keep), float(margin)))

    def set_rerank_tile(self, docs_per_cta=0):
        """Shortlisted docs per CTA of the FP8 MaxSim kernel: 32, 64, 128 or
        256 (0: the default, 256; queries of more than 32 tokens use at most
        128)."""
        check(lib().mvr_index_set_rerank_tile(self._h, int(docs_per_cta)))

    def set_wait_limit(self, wait_ns=0):
        """Time bound (ns) of the pipeline waits of the FP8 and the exact FP32
        MaxSim kernels; 0 restores the default (1 s).  A failure-detection
        test hook."""
        check(lib().mvr_index_set_wait_limit(self._h, int(wait_ns)))

    def set_graphs(self, enable=True):
        """Replay repeated search_device calls as one recorded CUDA graph."""
        check(lib().mvr_index_set_graphs(self._h, 1 if enable else 0))

    # -- search ----------------------------------------------------------
    def search(self, queries, k, nprobe, probe_topk, tok_off=None, semantics=SEM_PP,
               with_stats=False, with_stages=False):
        q, off, n_query, n_vec = _flatten_queries(queries, tok_off)
        scores = np.zeros((n_query, k), np.float32)
        ids = np.zeros((n_query, k), np.uint32)
        qtime = np.zeros(n_query, np.float64)
        st = _lib.Stats()
        if with_stages:
            stages = np.zeros((n_query, 6), np.float64)
            check(lib().mvr_search_staged(self._h, _ptr(q), _ptr(off), n_query, n_vec, k, nprobe,
                                          probe_topk, semantics, _ptr(scores), _ptr(ids),
                                          _ptr(qtime), _ptr(stages), C.byref(st)))
        else:
            stages = None
            check(lib().mvr_search(self._h, _ptr(q), _ptr(off), n_query, n_vec, k, nprobe,
                                   probe_topk, semantics, _ptr(scores), _ptr(ids), _ptr(qtime),
                                   C.byref(st)))
        if not with_stats:
            return scores, ids
        out = dict(st.as_dict(), query_time_s=qtime)
        if stages is not None:
            out["stage_time_s"] = stages
        return scores, ids, out

    def search_host_ptr(self, q_ptr, off, n_query, n_vec, k, nprobe, probe_topk, scores_ptr,
                        ids_ptr, semantics=SEM_PP, qtime=None):
        """Raw-pointer host search (e.g. pinned torch tensors); returns Stats.
        qtime (float64 [n_query], optional) receives per-query batch latency."""
        st = _lib.Stats()
        off = _c(off, np.uint64) if off is not None else None
        check(lib().mvr_search(self._h, C.c_void_p(q_ptr), _ptr(off), n_query, n_vec, k, nprobe,
                               probe_topk, semantics, C.c_void_p(scores_ptr),
                               C.c_void_p(ids_ptr), _ptr(qtime), C.byref(st)))
        return st

    def search_device(self, q_ptr, off, n_query, n_vec, k, nprobe, probe_topk, scores_ptr,
                      ids_ptr, stream_ptr=0, semantics=SEM_PP):
        """Device-pointer search; off is a host uint64 array or None."""
        st = _lib.Stats()
        off = _c(off, np.uint64) if off is not None else None
        check(lib().mvr_search_device(self._h, C.c_void_p(q_ptr), _ptr(off), n_query, n_vec, k,
                                      nprobe, probe_topk, semantics, C.c_void_p(scores_ptr),
                                      C.c_void_p(ids_ptr), C.c_void_p(stream_ptr or None),
                                      C.byref(st)))
        return st

    def trace(self, query, k, nprobe, probe_topk, semantics=SEM_PP, features=False, pred=False,
              cand=True):
        """One query through every stage; with features / pred also the
        learned pruner's features [n_short, 33] / predictions of the
        shortlist (short_feat / short_pred); cand=False skips the candidate
        set (n_item-sized buffers)."""
        q = _c(query, np.float32)
        nq = q.shape[0]
        n_item = self.info()["n_item"] if cand else 0
        arrs = dict(
            probe_id=np.zeros(nq * nprobe, np.uint32), probe_score=np.zeros(nq * nprobe, np.float32),
            short_id=np.zeros(probe_topk, np.uint32), short_approx=np.zeros(probe_topk, np.float32),
            short_exact=np.zeros(probe_topk, np.float32), topk_score=np.zeros(k, np.float32),
            topk_id=np.zeros(k, np.uint32))
        if features:
            arrs["short_feat"] = np.zeros(probe_topk * 33, np.float32)
        if pred:
            arrs["short_pred"] = np.zeros(probe_topk, np.float32)
        if cand:
            arrs["cand_id"] = np.zeros(n_item, np.uint32)
            arrs["cand_score"] = np.zeros(n_item, np.float32)
        tr = _lib.Trace()
        tr.cand_cap = n_item
        for name, a in arrs.items():
            setattr(tr, name, a.ctypes.data)
        check(lib().mvr_search_trace(self._h, _ptr(q), nq, k, nprobe, probe_topk, semantics,
                                     C.byref(tr)))
        nc, ns = tr.n_cand, tr.n_short
        return dict(probe_id=arrs["probe_id"].reshape(nq, nprobe),
                    probe_score=arrs["probe_score"].reshape(nq, nprobe), n_cand=nc,
                    **({"cand_id": arrs["cand_id"][:nc], "cand_score": arrs["cand_score"][:nc]}
                       if cand else {}),
                    short_id=arrs["short_id"][:ns], short_approx=arrs["short_approx"][:ns],
                    short_exact=arrs["short_exact"][:ns], score=arrs["topk_score"],
                    id=arrs["topk_id"],
                    **({"short_feat": arrs["short_feat"][:ns * 33].reshape(ns, 33)}
                       if features else {}),
                    **({"short_pred": arrs["short_pred"][:ns]} if pred else {}))

    def decompress(self, vec_ids):
        ids = _c(vec_ids, np.uint64)
        out = np.zeros((len(ids), 128), np.float32)
        check(lib().mvr_decompress(self._h, _ptr(ids), len(ids), _ptr(out)))
        return out

    def unpack_buckets(self, vec_ids):
        ids = _c(vec_ids, np.uint64)
        out = np.zeros((len(ids), 128), np.uint8)
        check(lib().mvr_unpack_buckets(self._h, _ptr(ids), len(ids), _ptr(out)))
        return out
