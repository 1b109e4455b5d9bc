"""Document-sharded search on the GPU (mvr.shard): the index split into doc
ranges, one handle per shard (here all on cuda:0), each shard's top-k made
global and merged.  With every shard's shortlist holding all of its
candidates the merged top-k equals the single-index GPU top-k and the
oracle's, bit for bit (PP semantics: BASIC's zero padding depends on the
index-wide longest doc)."""
import numpy as np
import pytest
import torch

from helpers import make_queries, oracle_of, tiny_index
from mvr import Index, shard

pytestmark = pytest.mark.gpu


def gpu_index(h):
    return Index.from_arrays(h["item_n_vec"], h["centroid"], h["vq_code"], h["ivf_off"],
                             h["ivf_size"], h["ivf_ids"], h["weight"], h["n_bit"], h["residual"])


@pytest.mark.parametrize("n_shards", [2, 3])
def test_gpu_sharded_search_equals_single_index(n_shards):
    ix = tiny_index(n_doc=400, n_centroid=64, n_bit=2, seed=21)
    q, off = make_queries(ix, 8, (4, 64), seed=22)
    full = gpu_index(ix)
    s_ref, i_ref = full.search(q, 10, 8, 400, tok_off=off)
    full.close()
    rs, ri = oracle_of(ix).search(q, off, 10, 8, 400)
    np.testing.assert_array_equal(i_ref, ri)
    ss, ii = [], []
    for a, b in shard.doc_ranges(400, n_shards):
        g = gpu_index(shard.split_index(ix, a, b))
        s, i = g.search(q, 10, 8, 400, tok_off=off)
        g.close()
        ss.append(torch.from_numpy(s).cuda())
        i64 = torch.from_numpy(i.astype(np.int64)).cuda()
        ii.append(torch.where(i64 == 0xFFFFFFFF, i64, i64 + a))
    ms, mi = shard.merge_topk(torch.stack(ss), torch.stack(ii), 10)
    np.testing.assert_array_equal(mi.cpu().numpy().astype(np.uint32), i_ref)
    np.testing.assert_array_equal(ms.cpu().numpy(), s_ref)
