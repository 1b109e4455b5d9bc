"""Shortlist tuner (mvr.tune): picks the smallest probe_topk whose recall@k
reaches the target, the most accurate one when none does, and measures the
ascending grid up to the first setting that reaches the target.  A stand-in index answers with the ground truth's first
r(probe_topk) ids plus filler, so recall grows with the shortlist."""
import numpy as np

from mvr import tune


class FakeIndex:
    def __init__(self, gnd, hits):
        self.gnd, self.hits, self.rescore, self.calls = gnd, hits, 0, []

    def set_rescore(self, r):
        self.rescore = r

    def search(self, queries, k, nprobe, probe_topk, semantics=0, with_stats=False):
        self.calls.append((probe_topk, self.rescore, semantics))
        h = self.hits(probe_topk)
        ids = np.full((len(self.gnd), k), 10_000, np.uint32)
        ids[:, :h] = self.gnd[:, :h]
        ids[:, h:] += np.arange(k - h, dtype=np.uint32)
        st = dict(device_ms=float(probe_topk) / 100.0)
        return np.zeros((len(self.gnd), k), np.float32), ids, st


def test_picks_smallest_shortlist_reaching_target():
    gnd = np.arange(40, dtype=np.uint32).reshape(4, 10)
    idx = FakeIndex(gnd, lambda p: min(10, p // 100))
    t = tune.tune(idx, np.zeros((4, 32, 128), np.float32), gnd, 10, 8, 0.9, semantics=2,
                  probe_topks=(100, 300, 900, 1000, 2000), repeats=2)
    assert t["reached"] and t["probe_topk"] == 900 and abs(t["recall"] - 0.9) < 1e-9
    assert [x["probe_topk"] for x in t["table"]] == [100, 300, 900]
    assert all(c[2] == 2 for c in idx.calls) and len(idx.calls) == 6
    assert idx.rescore == 0


def test_most_accurate_when_target_unreachable():
    gnd = np.arange(20, dtype=np.uint32).reshape(2, 10)
    idx = FakeIndex(gnd, lambda p: 3 if p < 500 else 5)
    t = tune.tune(idx, np.zeros((2, 8, 128), np.float32), gnd, 10, 4, 0.99, semantics=0,
                  probe_topks=(5, 100, 600, 800), repeats=1)
    assert not t["reached"] and t["probe_topk"] == 600 and t["recall"] == 0.5
    assert 5 not in [x["probe_topk"] for x in t["table"]]  # below k: skipped


def test_batch_tuner_picks_the_fastest_and_restores_the_default():
    class BatchIndex:
        def __init__(self):
            self.batch, self.sets = 0, []

        def set_batch(self, b):
            self.batch = b
            self.sets.append(b)

        def search(self, queries, k, nprobe, probe_topk, semantics=0, with_stats=False,
                   tok_off=None):
            ms = {296: 9.0, 592: 7.0, 1184: 5.0, 2368: 5.0, 4096: 6.0}[self.batch]
            return None, None, dict(device_ms=ms)

    idx = BatchIndex()
    t = tune.tune_batch(idx, np.zeros((100, 32, 128), np.float32), 10, 8, 1500, 4, repeats=2)
    assert t["batch"] == 1184 and t["ms"] == 5.0 and abs(t["qps"] - 100 / 5e-3) < 1e-6
    assert [x["batch"] for x in t["table"]] == [296, 592, 1184, 2368, 4096]
    assert idx.sets[-1] == 0

