"""Python mirror of the reference's method facades IGPGPUBasic
(src/impl/IGPGPUBasic.hpp:38-313) and IGPGPUPP (src/impl/IGPGPUPP.hpp:
36-335): constructor(item_n_vec_l_fname[, n_cpu_thread]),
buildIndex(centroid_l, vq_code_l, ivf_index, weight_l, residual_code_l,
n_centroid, n_bit) -> bool, search(query_l, n_query, query_n_vec, topk,
nprobe, probe_topk) -> result with result_score_l / result_ID_l /
compute_time_l (+ batch_query_time for PP).  Errors raise ValueError where
the reference exits; the index stays usable after search()."""
from types import SimpleNamespace

import numpy as np

from ._lib import MvrError
from .index import SEM_BASIC, SEM_PP, Index


class _Base:
    _sem = SEM_PP

    def __init__(self, item_n_vec_l_fname, device=0):
        self.item_n_vec_l_fname = item_n_vec_l_fname
        self.device = device
        self.index = None
        self.last_error = ""

    def buildIndex(self, centroid_l_fname, vq_code_l_fname, ivf_index_fname, weight_l_fname,
                   residual_code_l_fname, n_centroid, n_bit):
        try:
            self.index = Index.load_files(self.item_n_vec_l_fname, centroid_l_fname,
                                          vq_code_l_fname, ivf_index_fname, weight_l_fname,
                                          residual_code_l_fname, n_centroid, n_bit, self.device)
        except MvrError as e:
            self.last_error = str(e)
            self.index = None
            return False
        return True

    def _run(self, query_l, n_query, query_n_vec, topk, nprobe, probe_topk):
        if self.index is None:
            raise RuntimeError("search before a successful buildIndex")
        if probe_topk < topk:
            raise ValueError("the number of refined topk is smaller than the number of returned topk")
        q = np.ascontiguousarray(query_l, np.float32).reshape(n_query, query_n_vec, -1)
        n_warm = min(n_query, 10)
        if n_warm:
            self.index.search(q[:n_warm], topk, nprobe, probe_topk, semantics=self._sem)
        return self.index.search(q, topk, nprobe, probe_topk, semantics=self._sem,
                                 with_stats=True, with_stages=True)


class IGPGPUBasic(_Base):
    _sem = SEM_BASIC

    def search(self, query_l, n_query, query_n_vec, topk, nprobe, probe_topk):
        s, i, st = self._run(query_l, n_query, query_n_vec, topk, nprobe, probe_topk)
        stg = st["stage_time_s"]
        zero = np.zeros(n_query)
        return SimpleNamespace(
            result_score_l=s.reshape(-1), result_ID_l=i.reshape(-1),
            compute_time_l=st["query_time_s"], reset_time_l=zero,
            transmit_query_time_l=stg[:, 0], cand_gen_time_l=stg[:, 1], filter_time_l=stg[:, 2],
            filter_transmit_time_l=zero, filter_compute_time_l=stg[:, 2],
            rerank_time_l=stg[:, 3] + stg[:, 4] + stg[:, 5], rerank_transmit_time_l=stg[:, 5],
            rerank_compute_time_l=stg[:, 3] + stg[:, 4], n_query=n_query, topk=topk)


class IGPGPUPP(_Base):
    _sem = SEM_PP

    def __init__(self, item_n_vec_l_fname, n_cpu_thread=1, device=0):
        super().__init__(item_n_vec_l_fname, device)
        self.n_cpu_thread = n_cpu_thread  # accepted; queries run in device batches

    def search(self, query_l, n_query, query_n_vec, topk, nprobe, probe_topk):
        s, i, st = self._run(query_l, n_query, query_n_vec, topk, nprobe, probe_topk)
        return SimpleNamespace(result_score_l=s.reshape(-1), result_ID_l=i.reshape(-1),
                               compute_time_l=st["query_time_s"], batch_query_time=st["wall_s"],
                               n_query=n_query, topk=topk)
