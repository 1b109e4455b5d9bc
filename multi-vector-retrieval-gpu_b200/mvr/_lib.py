"""ctypes binding of libmvr (include/mvr.h).

The library is built in-tree (multi-vector-retrieval-gpu_b200/lib/libmvr.so).
There is no fallback: if it is missing, importing this module raises.
"""
import ctypes as C
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_DIR = os.path.join(os.path.dirname(_HERE), "lib")
LIB_PATH = os.path.join(LIB_DIR, "libmvr.so")

MVR_OK = 0
MVR_ERR_INVALID_ARG = 1
MVR_ERR_IO = 2
MVR_ERR_CUDA = 3
MVR_ERR_OOM = 4
MVR_ERR_UNSUPPORTED = 5
MVR_SEM_PP = 0
MVR_SEM_BASIC = 1
MVR_PREC_BF16 = 2
MVR_PREC_FP8 = 4
MVR_CAND_IMPUTE = 8
MVR_PRUNE = 16

# every symbol include/mvr.h declares
EXPORTS = (
    "mvr_last_error", "mvr_device_count", "mvr_index_load", "mvr_index_load_files",
    "mvr_index_from_arrays", "mvr_index_from_device_arrays", "mvr_index_free",
    "mvr_index_get_info", "mvr_index_set_batch", "mvr_index_set_rescore", "mvr_index_set_graphs",
    "mvr_search", "mvr_search_staged",
    "mvr_search_device", "mvr_search_trace", "mvr_decompress", "mvr_unpack_buckets",
    "mvr_assign_device", "mvr_assign_tc_device", "mvr_pack_residual_device",
    "mvr_kmeans_accumulate_device", "mvr_residual_quantiles_device",
    "mvr_filter_noalloc", "mvr_index_set_wait_limit",
    "mvr_mlp_work_floats", "mvr_mlp_train_step", "mvr_mlp_forward", "mvr_index_set_pruner",
    "mvr_index_set_rerank_tile",
)


class MvrError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"[mvr status {code}] {msg}")
        self.code = code


class IndexInfo(C.Structure):
    _fields_ = [("n_item", C.c_uint32), ("n_centroid", C.c_uint32), ("dim", C.c_uint32),
                ("n_bit", C.c_uint32), ("n_vec", C.c_uint64), ("n_ele_ivf", C.c_uint64),
                ("max_item_n_vec", C.c_uint32), ("max_ivf_list", C.c_uint32),
                ("device_bytes", C.c_uint64), ("device", C.c_int)]


class Stats(C.Structure):
    _fields_ = [("wall_s", C.c_double), ("device_ms", C.c_double), ("batch_ms_max", C.c_double),
                ("n_batch", C.c_uint32), ("gpu_launches", C.c_uint32),
                ("h2d_bytes", C.c_uint64), ("d2h_bytes", C.c_uint64),
                ("n_cand_total", C.c_uint64), ("n_rerank_tok", C.c_uint64),
                ("n_list_ent", C.c_uint64), ("stage_ms", C.c_double * 6),
                ("n_prune_fallback", C.c_uint64)]

    def as_dict(self):
        d = {k: getattr(self, k) for k, _ in self._fields_}
        d["stage_ms"] = list(self.stage_ms)
        return d


class Trace(C.Structure):
    _fields_ = [("probe_id", C.c_void_p), ("probe_score", C.c_void_p),
                ("cand_cap", C.c_uint32), ("n_cand", C.c_uint32),
                ("cand_id", C.c_void_p), ("cand_score", C.c_void_p),
                ("n_short", C.c_uint32), ("short_id", C.c_void_p),
                ("short_approx", C.c_void_p), ("short_exact", C.c_void_p),
                ("topk_score", C.c_void_p), ("topk_id", C.c_void_p),
                ("short_feat", C.c_void_p), ("short_pred", C.c_void_p)]


_lib = None


def lib():
    """Load libmvr.so (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(f"libmvr.so is not built ({LIB_PATH}); run __graft_entry__.build()")
    L = C.CDLL(LIB_PATH)
    vp, u32, u64, i32 = C.c_void_p, C.c_uint32, C.c_uint64, C.c_int
    L.mvr_last_error.restype = C.c_char_p
    L.mvr_device_count.restype = i32
    sig = {
        "mvr_index_load": [C.c_char_p, u32, u32, i32, C.POINTER(vp)],
        "mvr_index_load_files": [C.c_char_p] * 6 + [u32, u32, i32, C.POINTER(vp)],
        "mvr_index_from_arrays": [vp, u32, vp, u32, u32, vp, u64, vp, vp, vp, u64, vp, u32, vp,
                                  i32, C.POINTER(vp)],
        "mvr_index_from_device_arrays": [vp, u32, vp, u32, u32, vp, u64, vp, vp, vp, u64, vp, u32,
                                         vp, i32, C.POINTER(vp)],
        "mvr_index_free": [vp],
        "mvr_index_get_info": [vp, C.POINTER(IndexInfo)],
        "mvr_index_set_batch": [vp, u32],
        "mvr_index_set_rescore": [vp, u32],
        "mvr_index_set_graphs": [vp, i32],
        "mvr_search": [vp, vp, vp, u32, u32, u32, u32, u32, u32, vp, vp, vp, C.POINTER(Stats)],
        "mvr_search_staged": [vp, vp, vp, u32, u32, u32, u32, u32, u32, vp, vp, vp, vp,
                              C.POINTER(Stats)],
        "mvr_search_device": [vp, vp, vp, u32, u32, u32, u32, u32, u32, vp, vp, vp,
                              C.POINTER(Stats)],
        "mvr_search_trace": [vp, vp, u32, u32, u32, u32, u32, C.POINTER(Trace)],
        "mvr_decompress": [vp, vp, u64, vp],
        "mvr_unpack_buckets": [vp, vp, u64, vp],
        "mvr_assign_device": [vp, u64, vp, u32, u32, vp, vp, vp],
        "mvr_assign_tc_device": [vp, u64, vp, u32, u32, vp, vp, vp],
        "mvr_pack_residual_device": [vp, u64, vp, u32, vp, vp, u32, vp, vp],
        "mvr_kmeans_accumulate_device": [vp, u64, u32, vp, vp, vp, vp],
        "mvr_residual_quantiles_device": [vp, u64, vp, u32, vp, u32, vp, vp, vp],
        "mvr_filter_noalloc": [vp, vp, vp, u32, u32, u32, vp, vp, vp, vp],
        "mvr_index_set_wait_limit": [vp, u64],
        "mvr_mlp_train_step": [vp, vp, u32, vp, vp, vp, vp, C.c_float, u32, vp, vp],
        "mvr_mlp_forward": [vp, u32, vp, vp, vp, vp],
        "mvr_index_set_pruner": [vp, vp, u32, C.c_float],
        "mvr_index_set_rerank_tile": [vp, u32],
    }
    for name, args in sig.items():
        f = getattr(L, name)
        f.argtypes = args
        f.restype = i32
    L.mvr_mlp_work_floats.argtypes = [u32]
    L.mvr_mlp_work_floats.restype = C.c_size_t
    _lib = L
    return L


def check(rc):
    if rc != MVR_OK:
        raise MvrError(rc, lib().mvr_last_error().decode(errors="replace"))
    return rc
