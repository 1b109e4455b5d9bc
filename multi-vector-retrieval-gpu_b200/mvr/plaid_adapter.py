"""Drop-in for the reference's PLAID call site: a Searcher whose
search_all_embedding_by_vector (colbert/searcher.py:181-236) answers from
this package's GPU engine over a PLAID index directory, so a driver written
against ColBERT's Searcher (run.py:305-340: configure(...), then
search_all_embedding_by_vector(query_emb, query_embd_filename, qid_l, k)
returning the ranking and the per-query time lists) runs unchanged.

The PLAID directory's centroids, codes, bucket weights and IVF lists are
loaded as an IGP index (formats.read_plaid_index); the search is the IGP
path: PLAID's ncells (cells probed per query vector) is taken as nprobe and
its ndocs (docs kept by the approximate filter) as probe_topk; PLAID's
centroid_score_threshold has no counterpart in the IGP scoring and is kept
only as a setting.  Scores are the IGP path's exact MaxSim over the
un-normalized decoded vectors, not PLAID's normalized ones.
"""
import numpy as np

# PLAID's defaults by k (searcher.py:291-312)
_DEFAULTS = ((10, (1, 0.5, 256)), (100, (2, 0.45, 1024)))


class Ranking:
    """The part of ColBERT's Ranking (colbert/data/ranking.py:26-97) that the
    evaluation drivers use: qid -> [(pid, rank, score)], flattened rows,
    save_absolute_path writing qid \\t pid \\t rank \\t score lines."""

    def __init__(self, data):
        self.data = data
        self.flat_ranking = [(qid, *rest) for qid, sub in data.items() for rest in sub]

    def todict(self):
        return dict(self.data)

    def tolist(self):
        return list(self.flat_ranking)

    def items(self):
        return self.data.items()

    def save_absolute_path(self, new_path):
        with open(new_path, "w") as f:
            for items in self.flat_ranking:
                f.write("\t".join(str(x) for x in items) + "\n")
        return new_path


class SearchConfig:
    def __init__(self):
        self.ncells = None
        self.centroid_score_threshold = None
        self.ndocs = None

    def export(self):
        return dict(ncells=self.ncells, centroid_score_threshold=self.centroid_score_threshold,
                    ndocs=self.ndocs)


class Searcher:
    """Searcher(index=<PLAID index dir>) on the GPU (device), or on an
    `engine` with the same search(queries, k, nprobe, probe_topk,
    with_stats=True, with_stages=True) contract as mvr.Index."""

    def __init__(self, index, checkpoint=None, config=None, device=0, engine=None):
        self.checkpoint = checkpoint
        self.config = SearchConfig()
        if engine is None:
            from .index import Index
            engine = Index.from_plaid_dir(index, device=device)
        self.engine = engine

    def configure(self, **kw):
        for key, val in kw.items():
            setattr(self.config, key, val)

    def _params(self, k):
        ncells, thr, ndocs = next((d for kmax, d in _DEFAULTS if k <= kmax),
                                  (4, 0.4, max(k * 4, 4096)))
        c = self.config
        if c.ncells is None:
            c.ncells = ncells
        if c.centroid_score_threshold is None:
            c.centroid_score_threshold = thr
        if c.ndocs is None:
            c.ndocs = ndocs
        return int(c.ncells), max(int(c.ndocs), k)

    def search_all_embedding_by_vector(self, query_emb, query_embd_filename, qid_l, k=10,
                                       filter_fn=None):
        """Returns (ranking, time_l, time_ivf_l, time_filter_l, time_refine_l,
        n_refine_ivf_l, n_refine_filter_l, n_vec_score_refine_l) like the
        reference (times in ms per query: its batch's device latency and
        stage times; the candidate counts are not tracked per query: -1)."""
        if filter_fn is not None:
            raise NotImplementedError("filter_fn is not supported by the GPU engine")
        q = np.ascontiguousarray(query_emb, np.float32)
        if q.ndim != 3 or len(qid_l) != q.shape[0]:
            raise ValueError("query_emb must be [n_query, n_vec, dim] with one qid per query")
        nprobe, probe_topk = self._params(k)
        scores, ids, st = self.engine.search(q, k, nprobe, probe_topk, with_stats=True,
                                             with_stages=True)
        data = {}
        for qi, qid in enumerate(qid_l):
            rows = [(int(p), r + 1, float(s)) for r, (p, s) in enumerate(zip(ids[qi], scores[qi]))
                    if p != 0xFFFFFFFF]
            data[qid] = rows
        stage = np.asarray(st["stage_time_s"]) * 1e3
        n = q.shape[0]
        return (Ranking(data), list(np.asarray(st["query_time_s"]) * 1e3), list(stage[:, 1]),
                list(stage[:, 2]), list(stage[:, 3] + stage[:, 4]), [-1] * n, [-1] * n, [-1] * n)
