"""The shipped SpMM kernel selectors on the held-out part of their corpus
(CPU: the numpy restatement of the network over the stored features and the
stored forced-kernel SpMM times, each measured on a B200). For each k band
(k = 8, 32, 128 in the corpus) the kernel the library would run from the
prediction (the most probable one that applies) must cost at most 10% more
than the library's measured choice on average (regret <= 10%), and less
than always running the row-group kernel."""
import gzip
import json
import os

import numpy as np
import pytest

import perf_libs_sparse_b200 as pls
from perf_libs_sparse_b200 import selector as S

HERE = os.path.dirname(os.path.abspath(pls.__file__))
CORPUS = os.path.join(HERE, "selector_data", "spmm_corpus.jsonl.gz")


@pytest.fixture(scope="module")
def corpus():
    if not (os.path.exists(S.SHIPPED_SPMM) and os.path.exists(CORPUS)):
        pytest.skip("no shipped SpMM selector")
    with gzip.open(CORPUS, "rt") as f:
        rows = [json.loads(line) for line in f]
    rows.sort(key=lambda d: d["idx"])
    return rows


def test_shipped_spmm_selector_regret(corpus):
    from oracle import selector_ref

    n_train = int(round(0.8 * len(corpus)))
    held = corpus[n_train:]
    X = np.array([d["features"] for d in held], np.float64)
    params = np.load(S.SHIPPED_SPMM)
    for b, k in enumerate(S.SPMM_KS):
        T = S.spmm_library_times(np.array([d["ms"][str(k)] for d in held], np.float64))
        best = np.min(np.where(np.isfinite(T), T, np.inf), axis=1)
        probs = selector_ref.mlp_predict(params[f"b{b}"], len(S.SPMM_CLASSES), X)
        pick = S.spmm_pick(probs, T)
        regret = T[np.arange(len(T)), pick] / best - 1.0
        assert regret.mean() <= 0.10, (k, regret.mean(), np.percentile(regret, 90))
        assert (T[:, 0] / best - 1.0).mean() > regret.mean(), k
