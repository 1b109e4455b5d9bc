"""The IGPGPUBasic / IGPGPUPP executables and the Python mirror classes run
the reference's command line on the reference's directory layout and write
its answer / performance files; answers equal the oracle's."""
import os
import subprocess

import numpy as np
import pandas as pd
import pytest

from helpers import make_queries, oracle_of, tiny_index
from mvr import IGPGPUBasic, IGPGPUPP, _lib, formats
import pyoracle

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def dataset(tmp_path_factory):
    root = tmp_path_factory.mktemp("home")
    base = root / "Dataset" / "multi-vector-retrieval-GPU"
    ix = tiny_index(n_doc=300, n_centroid=64, n_bit=2, seed=12)
    idx_dir = base / "Index" / "synth" / "igp-n_centroid_64-n_bit_2"
    formats.write_index_dir(idx_dir, ix["item_n_vec"], ix["centroid"], ix["vq_code"],
                            ix["weight"], ix["residual"], ix["ivf_off"], ix["ivf_size"],
                            ix["ivf_ids"])
    q, off = make_queries(ix, 20, 32, seed=13)
    (base / "Embedding" / "synth").mkdir(parents=True)
    np.save(base / "Embedding" / "synth" / "query_embedding.npy", q.reshape(20, 32, 128))
    (base / "RawData" / "synth" / "document").mkdir(parents=True)
    qid = [1000 + 3 * i for i in range(20)]
    with open(base / "RawData" / "synth" / "document" / "queries.dev.tsv", "w") as f:
        for x in qid:
            f.write(f"{x}\tquery text {x}\n")
    (base / "Result" / "answer").mkdir(parents=True)
    return dict(root=root, base=base, ix=ix, q=q, off=off, qid=qid, idx_dir=idx_dir)


def run_cli(ds, exe, extra):
    args = [os.path.join(_lib.LIB_DIR, exe), "-username", "u", "-dataset", "synth", "-method-name",
            "igp", "-num-centroid", "64", "-num-bit", "2", "-topk", "10", "-nprobe", "4",
            "-probe_topk", "100", "-is_profile", "false"] + extra
    env = dict(os.environ, MVR_DATASET_ROOT=str(ds["root"]))
    r = subprocess.run(args, env=env, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr


@pytest.mark.parametrize("exe,sem", [("IGPGPUPP", pyoracle.SEM_PP),
                                     ("IGPGPUBasic", pyoracle.SEM_BASIC)])
def test_cli_answers_match_oracle(dataset, exe, sem):
    extra = ["-n_thread", "2"] if exe == "IGPGPUPP" else []
    run_cli(dataset, exe, extra)
    ans = dataset["base"] / "Result" / "answer"
    suffix = "nprobe_4-probe_topk_100" + ("-n_thread_2" if exe == "IGPGPUPP" else "")
    fn = ans / f"synth-igp-top10-n_centroid_64-n_bit_2-{suffix}.tsv"
    got = formats.read_answer_tsv(fn)
    o = oracle_of(dataset["ix"])
    s, i = o.search(dataset["q"], dataset["off"], 10, 4, 100, semantics=sem)
    for k, q in enumerate(dataset["qid"]):
        rows = got[q]
        assert [r[0] for r in rows] == list(i[k])
        assert [r[1] for r in rows] == list(range(1, 11))
        np.testing.assert_allclose([r[2] for r in rows], s[k], rtol=1e-5)
    perf = pd.read_csv(ans / f"synth-igp-performance-top10-n_centroid_64-n_bit_2-{suffix}.tsv",
                       delimiter="\t")
    assert len(perf) == 20 and (perf["search_time"] > 0).all()
    if exe == "IGPGPUBasic":
        for col in ("reset_time", "cand_gen_time", "filter_time", "rerank_time",
                    "rerank_compute_time"):
            assert col in perf.columns
    else:
        txt = open(ans / f"synth-igp-performance-top10-n_centroid_64-n_bit_2-{suffix}.txt").read()
        assert "batch_query_time(s)\t" in txt and "n_query\t20" in txt


def test_cli_reports_bad_index(dataset, tmp_path):
    env = dict(os.environ, MVR_DATASET_ROOT=str(tmp_path))
    r = subprocess.run([os.path.join(_lib.LIB_DIR, "IGPGPUPP"), "-username", "u", "-dataset", "x",
                        "-method-name", "igp", "-num-centroid", "64", "-num-bit", "2", "-topk",
                        "10", "-nprobe", "4", "-probe_topk", "100", "-n_thread", "1",
                        "-is_profile", "false"], env=env, capture_output=True, text=True)
    assert r.returncode != 0 and "buildIndex failed" in r.stderr


def test_python_mirror_classes(dataset):
    d = dataset["idx_dir"]
    files = [str(d / f) for f in ("centroid_l.npy", "vq_code_l.npy", "ivf.index", "weight_l.npy",
                                  "residual_code_l.npy")]
    o = oracle_of(dataset["ix"])
    for cls, sem in ((IGPGPUPP, pyoracle.SEM_PP), (IGPGPUBasic, pyoracle.SEM_BASIC)):
        m = cls(str(d / "item_n_vec_l.npy"))
        assert m.buildIndex(*files, 64, 2)
        r = m.search(dataset["q"], 20, 32, 10, 4, 100)
        s, i = o.search(dataset["q"], dataset["off"], 10, 4, 100, semantics=sem)
        np.testing.assert_array_equal(r.result_ID_l, i.reshape(-1))
        np.testing.assert_array_equal(r.result_score_l, s.reshape(-1))
        assert len(r.compute_time_l) == 20
        with pytest.raises(ValueError):
            m.search(dataset["q"], 20, 32, 10, 4, 5)
    bad = IGPGPUPP(str(d / "item_n_vec_l.npy"))
    assert not bad.buildIndex(*files, 63, 2)
