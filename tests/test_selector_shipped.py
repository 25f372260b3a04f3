"""The shipped selector on the held-out part of the corpus it was trained on
(CPU: the numpy restatement of the network over the stored features and the
exhaustive tuner's stored timings). The corpus is 3,000 generated matrices,
2,400 train / 600 held out; every timing in it was measured on a B200 by the
library's exhaustive tuner."""
import gzip
import json
import os

import numpy as np
import pytest

import perf_libs_sparse_b200 as pls
from perf_libs_sparse_b200 import selector as S

HERE = os.path.dirname(os.path.abspath(pls.__file__))
CORPUS = os.path.join(HERE, "selector_data", "corpus.jsonl.gz")


@pytest.fixture(scope="module")
def heldout():
    if not (os.path.exists(S.SHIPPED) and os.path.exists(CORPUS)):
        pytest.skip("no shipped selector")
    with gzip.open(CORPUS, "rt") as f:
        corpus = [json.loads(line) for line in f]
    corpus.sort(key=lambda d: d["idx"])
    assert len(corpus) == 3000
    return corpus[2400:]


def test_shipped_selector_regret_and_gain_over_rule(heldout):
    from oracle import selector_ref

    cands = S.candidates()
    params = np.load(S.SHIPPED)
    X = np.array([d["features"] for d in heldout], np.float64)
    T = np.array([d["ms"] for d in heldout], np.float64)
    cls = selector_ref.mlp_predict(params, len(cands), X).argmax(1)
    best = T.min(1)
    chosen = T[np.arange(len(T)), cls]
    regret = chosen / best - 1
    # the method without the network: the reference's padding-efficiency rule
    betas = np.array([d["beta"] for d in heldout])
    nnz = np.array([d["nnz"] for d in heldout], np.float64)
    m = np.array([d["m"] for d in heldout], np.float64)
    tpr = np.clip(2 ** np.floor(np.log2(np.maximum(nnz / np.maximum(m, 1), 1))), 1, 32).astype(int)
    plain_idx = [int(np.flatnonzero((cands[:, 0] == pls.KIND_CSR) & (cands[:, 3] == t))[0]) for t in tpr]
    rule_idx = np.array([S.reference_rule(cands, betas[i], plain_idx[i]) for i in range(len(T))])
    rule = T[np.arange(len(T)), rule_idx]
    plain = T[np.arange(len(T)), plain_idx]
    assert regret.mean() <= 0.10 and np.percentile(regret, 90) <= 0.10
    assert (rule / best - 1).mean() > 3 * regret.mean()
    assert np.exp(np.log(rule / chosen).mean()) > 1.1
    assert np.exp(np.log(plain / chosen).mean()) > 1.1
