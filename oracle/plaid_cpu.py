"""CPU PLAID search of the reference, over an index of this project re-laid
in PLAID's layout -- baseline and test infrastructure, not the product.

The reference ships, next to its GPU IGP method, the PLAID CPU search of its
ColBERT baseline: IndexScorer.rank, CPU branch (colbert/search/
index_storage.py:80-198) with candidate generation (search/
candidate_generation.py:13-66).  This module restates that orchestration
(the ColBERT package itself does not import on Python 3.12) and runs the
reference's own compiled extensions for the heavy steps: filter_pids_cpp
(approximate centroid scores, two-stage top-ndocs), decompress_residuals_cpp
and segmented_maxsim_cpp, built from the reference sources by
oracle/build_plaid.py into oracle/_ref/plaid/.

Re-laying an IGP index for PLAID keeps the centroids, codes, bucket weights
and IVF lists; only the residual bytes change: IGP packs each dim's bucket
most-significant-bit first, PLAID (ResidualCodec.binarize, residual.py:
189-205) least-significant-bit first within the same byte slots, so a PLAID
byte is the IGP byte with the bits of every nbits-wide group reversed --
the reference's own reversed_bit_map (residual.py:48-67), an involution.
PLAID then scores normalized decompressed vectors (residual.py:274-276), the
IGP path does not.
"""
import importlib.machinery
import importlib.util
import os
from itertools import product

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
PLAID_DIR = os.path.join(HERE, "_ref", "plaid")
NAMES = ("filter_pids_cpp", "decompress_residuals_cpp", "segmented_maxsim_cpp")

# PLAID's defaults by k (searcher.py:291-312)
DEFAULTS = ((10, dict(ncells=1, centroid_score_threshold=0.5, ndocs=256)),
            (100, dict(ncells=2, centroid_score_threshold=0.45, ndocs=1024)))


def available():
    return all(os.path.exists(os.path.join(PLAID_DIR, n, n + ".so")) for n in NAMES)


def _load(name):
    import torch  # noqa: F401  (the extensions link against libtorch)
    path = os.path.join(PLAID_DIR, name, name + ".so")
    loader = importlib.machinery.ExtensionFileLoader(name, path)
    spec = importlib.util.spec_from_file_location(name, path, loader=loader)
    mod = importlib.util.module_from_spec(spec)
    loader.exec_module(mod)
    return getattr(mod, name)


def reversed_bit_map(n_bit):
    """Byte -> byte with the bits of every n_bit-wide group reversed."""
    out = np.zeros(256, np.uint8)
    for x in range(256):
        z = 0
        for g in range(8 // n_bit):
            v = (x >> (g * n_bit)) & ((1 << n_bit) - 1)
            r = 0
            for i in range(n_bit):
                r |= ((v >> i) & 1) << (n_bit - 1 - i)
            z |= r << (g * n_bit)
        out[x] = z
    return out


def defaults(k):
    for kmax, d in DEFAULTS:
        if k <= kmax:
            return dict(d)
    return dict(ncells=4, centroid_score_threshold=0.4, ndocs=max(k * 4, 4096))


class PlaidCPU:
    """One index re-laid for PLAID; search_one(q, k) follows IndexScorer.rank."""

    def __init__(self, item_n_vec, centroid, vq_code, residual, weight, ivf_off, ivf_size,
                 ivf_ids, n_bit, n_threads=None):
        import torch
        if n_threads:
            torch.set_num_threads(n_threads)
        self.filter_pids = _load("filter_pids_cpp")
        self.decompress = _load("decompress_residuals_cpp")
        self.segmented_maxsim = _load("segmented_maxsim_cpp")
        self.n_bit = int(n_bit)
        vpb = 8 // self.n_bit
        self.centroids = torch.from_numpy(np.ascontiguousarray(centroid, np.float32))
        self.dim = self.centroids.shape[1]
        self.codes = torch.from_numpy(np.ascontiguousarray(vq_code).view(np.int32))
        self.doclens = torch.from_numpy(np.asarray(item_n_vec, np.int64))
        self.offsets = torch.cat([torch.zeros(1, dtype=torch.int64), torch.cumsum(self.doclens, 0)])
        rbm = reversed_bit_map(self.n_bit)
        self.rbm = torch.from_numpy(rbm)
        bpv = self.dim * self.n_bit // 8
        res = np.asarray(residual, np.uint8).reshape(-1, bpv)
        self.residuals = torch.from_numpy(rbm[res])          # PLAID bit order
        nb = len(weight)
        self.lookup = torch.tensor(list(product(range(nb), repeat=vpb)), dtype=torch.uint8)
        self.bucket_weights = torch.from_numpy(np.ascontiguousarray(weight, np.float32))
        self.ivf_off = np.asarray(ivf_off, np.int64)
        self.ivf_size = np.asarray(ivf_size, np.int64)
        self.ivf_ids = torch.from_numpy(np.asarray(ivf_ids, np.uint32).view(np.int32))

    def decompress_pids(self, pids):
        """decompress_residuals_cpp of the given docs (unnormalized)."""
        import torch
        return self.decompress(torch.as_tensor(pids, dtype=torch.int32), self.doclens,
                               self.offsets, self.bucket_weights, self.rbm, self.lookup,
                               self.residuals, self.codes, self.centroids, self.dim, self.n_bit)

    def search_one(self, q, k, ncells=None, centroid_score_threshold=None, ndocs=None):
        """Top-k (pids, scores) of one query [nq, dim] (float32, normalized)."""
        import torch
        d = defaults(k)
        ncells = ncells or d["ncells"]
        thr = d["centroid_score_threshold"] if centroid_score_threshold is None else centroid_score_threshold
        ndocs = ndocs or d["ndocs"]
        with torch.inference_mode():
            Q = torch.from_numpy(np.ascontiguousarray(q, np.float32))
            scores = self.centroids @ Q.T                                   # [C, nq]
            if ncells == 1:
                cells = scores.argmax(dim=0, keepdim=True).permute(1, 0)
            else:
                cells = scores.topk(ncells, dim=0, sorted=False).indices.permute(1, 0)
            cells = cells.flatten().unique().numpy()
            pids = torch.cat([self.ivf_ids[self.ivf_off[c]:self.ivf_off[c] + self.ivf_size[c]]
                              for c in cells])
            pids = torch.unique_consecutive(pids.sort().values)
            idx = scores.max(-1).values >= thr
            # filter_pids pops ndocs entries from its queue: never ask for more
            # than there are candidates
            nf = min(ndocs, int(pids.numel()))
            if nf < 4:
                return np.zeros(0, np.int64), np.zeros(0, np.float32)
            pids, _ = self.filter_pids(pids.to(torch.int32), scores.contiguous(), self.codes,
                                       self.doclens, self.offsets, idx, nf)
            D = self.decompress_pids(pids)
            D = torch.nn.functional.normalize(D.to(torch.float32), p=2, dim=-1)
            s = self.segmented_maxsim(D @ Q.T, self.doclens[pids.long()])
            o = s.sort(descending=True)
            top = o.indices[:k]
            return pids[top].numpy().astype(np.int64), o.values[:k].numpy()
