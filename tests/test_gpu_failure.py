"""Failure detection on the GPU without a fault: the FP8 MaxSim kernel's
pipeline waits are bounded, and a wait that runs out stops the kernel (which
still lets its copies and MMAs finish and frees its tensor memory), sets the
handle's error flag, and makes the search fail with MVR_ERR_CUDA.  The test
shrinks the bound to a single timer tick so that waits run out, then checks
the error, restores the bound, and checks that the same handle searches
exactly as before (every returned score the oracle's exact FP32 MaxSim)."""
import numpy as np
import pytest

from helpers import make_queries, oracle_of, tiny_index
from mvr import PREC_FP8, Index, _lib

pytestmark = pytest.mark.gpu


def test_fp8_wait_timeout_reports_error_and_handle_recovers():
    ix = tiny_index(n_doc=700, n_centroid=96, n_bit=2, seed=61)
    o = oracle_of(ix)
    q, off = make_queries(ix, 8, 32, seed=62)
    with Index.from_arrays(ix["item_n_vec"], ix["centroid"], ix["vq_code"], ix["ivf_off"],
                           ix["ivf_size"], ix["ivf_ids"], ix["weight"], ix["n_bit"],
                           ix["residual"]) as g:
        s0, i0 = g.search(q.reshape(8, 32, 128), 10, 6, 300, semantics=PREC_FP8)
        g.set_wait_limit(1)
        with pytest.raises(_lib.MvrError) as e:
            g.search(q.reshape(8, 32, 128), 10, 6, 300, semantics=PREC_FP8)
        assert e.value.code == _lib.MVR_ERR_CUDA and "timed out" in str(e.value)
        g.set_wait_limit(0)
        for _ in range(2):
            s1, i1 = g.search(q.reshape(8, 32, 128), 10, 6, 300, semantics=PREC_FP8)
            np.testing.assert_array_equal(i1, i0)
            np.testing.assert_array_equal(s1, s0)
        for k in range(8):
            for d, sc in zip(i1[k], s1[k]):
                if d != 0xFFFFFFFF:
                    assert sc == o.maxsim_item(q[off[k]:off[k + 1]], int(d))
