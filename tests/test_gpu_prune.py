"""The learned candidate pruner: its MLP kernels (33 -> 256 -> 256 -> 1,
GELU, BF16-rounded weights, FP32 accumulation) against a plain PyTorch FP32
reference of the same arithmetic -- the forward pass, one Adam step (loss,
gradients and updated parameters through torch autograd), and a short
training run that fits a synthetic target -- then the pruner in the search
path: its features, the tensor-core MLP against the CUDA-core one, and the
keep / fallback behaviour of MVR_PRUNE."""
import ctypes as C
import math

import numpy as np
import pytest

from mvr import _lib

pytestmark = pytest.mark.gpu
NP = 74753


def split(p):
    o = 0
    out = []
    for shape in ((256, 33), (256,), (256, 256), (256,), (256,), (1,)):
        n = int(np.prod(shape))
        out.append(p[o:o + n].view(*shape))
        o += n
    assert o == NP
    return out


def torch_forward(x, p):
    import torch
    W1, b1, W2, b2, w3, b3 = split(p)

    def bf(t):  # BF16 rounding with a straight-through gradient
        return t + (t.to(torch.bfloat16).to(torch.float32) - t).detach()

    def gelu(z):
        return 0.5 * z * (1.0 + torch.tanh(0.7978845608 * (z + 0.044715 * z ** 3)))
    h1 = bf(gelu(x @ bf(W1).T + b1))
    h2 = bf(gelu(h1 @ bf(W2).T + b2))
    return h2 @ bf(w3) + b3


def init_params(seed):
    import torch
    g = torch.Generator().manual_seed(seed)
    p = torch.zeros(NP)
    W1, b1, W2, b2, w3, b3 = split(p)
    W1.copy_(torch.randn(256, 33, generator=g) / math.sqrt(33))
    W2.copy_(torch.randn(256, 256, generator=g) / math.sqrt(256))
    w3.copy_(torch.randn(256, generator=g) / math.sqrt(256))
    b1.copy_(0.1 * torch.randn(256, generator=g))
    b2.copy_(0.1 * torch.randn(256, generator=g))
    return p


def lib_forward(x, p):
    import torch
    n = x.shape[0]
    work = torch.zeros(_lib.lib().mvr_mlp_work_floats(n), device="cuda")
    out = torch.zeros(n, device="cuda")
    _lib.check(_lib.lib().mvr_mlp_forward(C.c_void_p(x.data_ptr()), n, C.c_void_p(p.data_ptr()),
                                          C.c_void_p(work.data_ptr()),
                                          C.c_void_p(out.data_ptr()), None))
    return out


def train_steps(x, y, p, m, v, steps, lr, loss):
    import torch
    n = x.shape[0]
    work = torch.zeros(_lib.lib().mvr_mlp_work_floats(n), device="cuda")
    for step in steps:
        _lib.check(_lib.lib().mvr_mlp_train_step(
            C.c_void_p(x.data_ptr()), C.c_void_p(y.data_ptr()), n, C.c_void_p(p.data_ptr()),
            C.c_void_p(m.data_ptr()), C.c_void_p(v.data_ptr()), C.c_void_p(work.data_ptr()), lr,
            step, C.c_void_p(loss.data_ptr()), None))


def test_mlp_forward_matches_torch():
    import torch
    x = torch.randn(1000, 33, generator=torch.Generator().manual_seed(1)).cuda()
    p = init_params(2).cuda()
    got = lib_forward(x, p)
    ref = torch_forward(x, p)
    torch.testing.assert_close(got, ref, rtol=2e-4, atol=2e-4)


def test_mlp_adam_step_matches_torch():
    import torch
    n = 777
    g = torch.Generator().manual_seed(3)
    x = torch.randn(n, 33, generator=g).cuda()
    y = torch.randn(n, generator=g).cuda()
    p = init_params(4).cuda()
    m = torch.zeros(NP, device="cuda")
    v = torch.zeros(NP, device="cuda")
    loss = torch.zeros(1, device="cuda")
    p_ref = p.clone().requires_grad_(True)
    lr = 1e-3
    train_steps(x, y, p, m, v, (1, 2), lr, loss)
    opt = torch.optim.Adam([p_ref], lr=lr, betas=(0.9, 0.999), eps=1e-8)
    for _ in (1, 2):
        opt.zero_grad()
        ref_loss = 0.5 * ((torch_forward(x, p_ref) - y) ** 2).mean()
        ref_loss.backward()
        opt.step()
    torch.testing.assert_close(loss[0], ref_loss.detach(), rtol=1e-4, atol=1e-6)
    torch.testing.assert_close(p, p_ref.detach(), rtol=1e-4, atol=2e-6)


def test_mlp_training_fits_a_target():
    import torch
    n = 4096
    g = torch.Generator().manual_seed(5)
    x = torch.rand(n, 33, generator=g).cuda()
    y = (x[:, :32].max(1).values + 0.3 * x[:, 32]).contiguous()
    p = init_params(6).cuda()
    p[-257:] = 0.0
    m = torch.zeros(NP, device="cuda")
    v = torch.zeros(NP, device="cuda")
    loss = torch.zeros(1, device="cuda")
    train_steps(x, y, p, m, v, (1,), 1e-3, loss)
    first = float(loss[0])
    train_steps(x, y, p, m, v, range(2, 301), 1e-3, loss)
    assert float(loss[0]) < 0.05 * first, (first, float(loss[0]))


# ---- the pruner in the search path (MVR_PRUNE) ----

def _index(n_bit=2, seed=81):
    from helpers import tiny_index
    from mvr import Index
    ix = tiny_index(n_doc=600, n_centroid=80, n_bit=n_bit, seed=seed)
    g = Index.from_arrays(ix["item_n_vec"], ix["centroid"], ix["vq_code"], ix["ivf_off"],
                          ix["ivf_size"], ix["ivf_ids"], ix["weight"], ix["n_bit"],
                          ix["residual"])
    return ix, g


@pytest.mark.parametrize("n_bit", [2, 4])
def test_prune_features_are_centroid_interaction_scores(n_bit):
    """Features = per query token the best (E4M3) centroid score over the
    doc's tokens, within FP8 rounding of the FP32 value, and log(length)."""
    from helpers import make_queries
    ix, g = _index(n_bit)
    q, off = make_queries(ix, 3, (20, 32), seed=82)
    start = np.concatenate([[0], np.cumsum(ix["item_n_vec"].astype(np.int64))])
    for i in range(3):
        qi = q[off[i]:off[i + 1]]
        t = g.trace(qi, 10, 5, 150, features=True)
        f = t["short_feat"]
        for j, d in enumerate(t["short_id"]):
            codes = ix["vq_code"][start[d]:start[d + 1]]
            ci = (qi.astype(np.float64) @ ix["centroid"][codes].T.astype(np.float64)).max(1)
            np.testing.assert_allclose(f[j, :len(qi)], ci, rtol=0, atol=0.06)
            assert np.all(f[j, len(qi):32] == 0.0)
            assert abs(f[j, 32] - math.log(ix["item_n_vec"][d])) < 1e-5
    g.close()


def test_prune_mlp_tensor_cores_match_cuda_core_reference():
    """The tensor-core MLP (BF16 features, hardware tanh) against the CUDA-core
    forward pass on the same features."""
    from helpers import make_queries
    from mvr import prune
    ix, g = _index()
    q, off = make_queries(ix, 3, 32, seed=83)
    params = prune.init_params(7)
    g.set_pruner(params, 50, 0.0)
    for i in range(3):
        t = g.trace(q[off[i]:off[i + 1]], 10, 5, 150, features=True, pred=True)
        ref = prune.predict(t["short_feat"], params)
        np.testing.assert_allclose(t["short_pred"], ref, rtol=3e-2, atol=3e-2)
    g.close()


def test_prune_search_keep_and_fallback():
    """keep >= shortlist: the FP8 path's results; a margin no prediction gap
    reaches: every query falls back, same results; margin -inf: every query
    scores only its `keep` best predictions, and every returned score is the
    exact FP32 MaxSim."""
    from helpers import make_queries, oracle_of
    from mvr import PREC_FP8, PRUNE, prune
    ix, g = _index()
    o = oracle_of(ix)
    q, off = make_queries(ix, 12, 32, seed=84)
    X, y, _ = prune.traces(g, q, off, 5, 150, per_query=40, seed=1)
    params, hist = prune.train(X, y, epochs=20, batch=256, lr=2e-3)
    assert hist[-1] < hist[0]
    s8, i8 = g.search(q.reshape(12, 32, 128), 10, 5, 150, semantics=PREC_FP8)
    g.set_pruner(params, 150, 0.0)
    s, i, st = g.search(q.reshape(12, 32, 128), 10, 5, 150, semantics=PREC_FP8 | PRUNE,
                        with_stats=True)
    np.testing.assert_array_equal(i, i8)
    np.testing.assert_array_equal(s, s8)
    g.set_pruner(params, 60, 1e9)
    s, i, st = g.search(q.reshape(12, 32, 128), 10, 5, 150, semantics=PREC_FP8 | PRUNE,
                        with_stats=True)
    np.testing.assert_array_equal(i, i8)
    assert st["n_prune_fallback"] == 12
    g.set_pruner(params, 60, -1e9)
    s, i, st = g.search(q.reshape(12, 32, 128), 10, 5, 150, semantics=PREC_FP8 | PRUNE,
                        with_stats=True)
    assert st["n_prune_fallback"] == 0
    for k in range(12):
        for d, sc in zip(i[k], s[k]):
            if d != 0xFFFFFFFF:
                assert sc == o.maxsim_item(q[off[k]:off[k + 1]], int(d))
    g.close()


def test_prune_plain_path_keep_and_fallback():
    """MVR_PRUNE without a precision flag (the pruned docs go straight to the
    exact FP32 MaxSim): keep >= shortlist gives the plain path's results bit
    for bit; a margin no gap reaches falls back on every query, same results;
    margin -inf scores only the kept docs, and every returned score is the
    exact FP32 MaxSim of its doc (the oracle's canonical arithmetic)."""
    from helpers import make_queries, oracle_of
    from mvr import PRUNE, prune
    ix, g = _index(4, seed=85)
    o = oracle_of(ix)
    q, off = make_queries(ix, 12, 32, seed=86)
    X, y, _ = prune.traces(g, q, off, 5, 150, per_query=40, seed=2)
    params, _ = prune.train(X, y, epochs=20, batch=256, lr=2e-3)
    s0, i0 = g.search(q.reshape(12, 32, 128), 10, 5, 150, semantics=0)
    g.set_pruner(params, 150, 0.0)
    s, i = g.search(q.reshape(12, 32, 128), 10, 5, 150, semantics=PRUNE)
    np.testing.assert_array_equal(i, i0)
    np.testing.assert_array_equal(s, s0)
    g.set_pruner(params, 60, 1e9)
    s, i, st = g.search(q.reshape(12, 32, 128), 10, 5, 150, semantics=PRUNE, with_stats=True)
    np.testing.assert_array_equal(i, i0)
    np.testing.assert_array_equal(s, s0)
    assert st["n_prune_fallback"] == 12
    g.set_pruner(params, 60, -1e9)
    s, i, st = g.search(q.reshape(12, 32, 128), 10, 5, 150, semantics=PRUNE, with_stats=True)
    assert st["n_prune_fallback"] == 0
    assert st["n_rerank_tok"] < sum(
        int(ix["item_n_vec"][int(d)]) for k in range(12) for d in
        g.trace(q[off[k]:off[k + 1]], 10, 5, 150)["short_id"])
    for k in range(12):
        for d, sc in zip(i[k], s[k]):
            if d != 0xFFFFFFFF:
                assert sc == o.maxsim_item(q[off[k]:off[k + 1]], int(d))
    g.close()
