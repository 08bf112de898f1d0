"""The learned schedule choices (zkwasm-prover_b200/choices.py) on their
committed data and parameters, on the CPU: the models' held-out picks,
recomputed with a NumPy restatement of the MLP's forward pass, give the
regrets recorded when they were trained, and for the table-or-plain MSM
choice and the extended-domain layout the learned pick has less regret than
the library's fixed rule."""
import importlib
import json
import os

import numpy as np
import pytest


@pytest.fixture(scope="module")
def C():
    return importlib.import_module("zkwasm-prover_b200.choices")


def _data(C):
    with open(os.path.join(C.HERE, "choices_data.json")) as f:
        return json.load(f)


@pytest.mark.parametrize("name", ["ntt_split", "msm_table", "extend"])
def test_recorded_regret_reproduces(C, name):
    S = importlib.import_module("zkwasm-prover_b200.schedule")
    data = _data(C)[name]
    params = np.load(C.model_path(name))["params"]
    meta = json.loads(str(np.load(C.model_path(name))["meta"]))
    test = [r for r in data if C.size_of(name, r) % 2 == 1]

    def pick(r):
        cands = C.candidates(r)
        X = np.array([C.encode(name, r, c) for c in cands], np.float32)
        return cands[int(np.argmin(S.mlp_forward_numpy(params, X)))]

    learned, _ = C.regret(test, pick)
    assert abs(learned - meta["regret_learned_ms"]) < 1e-3 * max(1.0, meta["regret_learned_ms"]) + 1e-6
    if name in ("msm_table", "extend"):
        fixed = meta["regret_fixed_rule_ms"]
        assert learned < fixed


def test_encodings_have_the_model_width(C):
    assert len(C.enc_ntt(22, 8, [11, 11])) == C.DIM
    assert len(C.enc_msm_table(1 << 22, 8, [0.1] * 7, 1)) == C.DIM
    assert len(C.enc_extend(22, 3, 8, "pairs", 8)) == C.DIM
