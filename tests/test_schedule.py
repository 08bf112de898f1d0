"""What the learned schedule gains over the methods without it, on the
timings the exhaustive autotuner recorded on a B200
(zkwasm-prover_b200/msm_schedule_data.json) and the model trained on them
(msm_schedule_model.npz).  The model is evaluated with the NumPy restatement
of the forward kernel, so this runs without a GPU."""
import json
import math
import os

import numpy as np


def _load(zkp):
    d = os.path.dirname(zkp.LIB_PATH)
    with open(os.path.join(d, "msm_schedule_data.json")) as f:
        records = json.load(f)
    params = np.load(os.path.join(d, "msm_schedule_model.npz"))["params"].astype(np.float64)
    return records, params


def _learned_picker(S, params):
    def pick(r):
        f = S.shape_features(r["n"], r["batch"], r["hist"])
        cands = list(range(S.C_MIN, S.C_MAX + 1))
        X = np.array([S.model_input(f, c) for c in cands], np.float64)
        return cands[int(np.argmin(S.mlp_forward_numpy(params, X)))]

    return pick


def test_learned_schedule_beats_formulas_on_unseen_sizes(zkp):
    S = zkp.schedule
    records, params = _load(zkp)
    held_out = [r for r in records if (r["n"].bit_length() - 1) % 2 == 1]
    assert len(held_out) >= 16
    learned, _ = S.regret(held_out, _learned_picker(S, params))
    default, _ = S.regret(held_out, lambda r: S.default_window(r["n"]))
    reference, _ = S.regret(held_out, lambda r: S.reference_window(r["n"]))
    best = sum(min(r["times_ms"].values()) for r in held_out)
    # regret in ms summed over the unseen shapes
    assert learned < default and learned < reference
    assert learned < 0.05 * best


def test_dataset_is_consistent(zkp):
    records, params = _load(zkp)
    assert params.shape[0] == zkp.load_library().zkp_mlp_param_count()
    for r in records:
        assert abs(sum(r["hist"]) - 1.0) < 1e-6
        times = {int(c): v for c, v in r["times_ms"].items()}
        assert r["best"] == min(times, key=times.get)
        assert all(v > 0 and math.isfinite(v) for v in times.values())


def test_ntt_splits_enumeration(zkp):
    # the radix autotuner's candidates: ordered splits into 2-3 passes of 2^6..2^12
    S = zkp.schedule
    for log_n in (13, 16, 20, 24, 25):
        splits = S.ntt_splits(log_n)
        assert splits and len({tuple(x) for x in splits}) == len(splits)
        for sp in splits:
            assert sum(sp) == log_n and 2 <= len(sp) <= 3 and all(6 <= r <= 12 for r in sp)
    assert sorted(map(tuple, S.ntt_splits(13))) == [(6, 7), (7, 6)]
    assert [8, 8, 8] in S.ntt_splits(24) and [12, 12] in S.ntt_splits(24)
