"""Learned schedule choices beyond the MSM window.

The schedule module's MLP (10 inputs, two hidden layers of 64, one output;
forward, gradient and Adam in csrc/schedule.cu) predicts the log-time of a
candidate from the shape's features and the candidate's encoding; a pick is
the argmin over the candidates.  Three more choices are learned the same way,
each with its own parameters, from the exhaustive tuners' timings on this GPU:

* ``ntt_split``: the pass radices of a batched NTT of ncols columns of 2^k
  points (every split into 2-3 passes of 2^6..2^12; the library's default is
  the split its tuner found fastest for one column);
* ``msm_table``: an MSM pipeline over the SRS table (zkp_msm_batch_table, at
  the library's batch-table width) or over the plain bases
  (zkp_msm_batch, the library's windows), for a batch of same-size MSMs with
  a given scalar distribution (the table is built once per SRS, so its build
  time is not part of the choice);
* ``extend``: the extended-domain phase's multiplier-table layout
  (Montgomery or (w, w') pairs) and columns per launch.

Every model is trained on the even log-sizes and judged on the odd ones:
regret (ms) = time of the pick - time of the tuner's best, summed over the
held-out shapes, against the library's fixed rule for the same choice.  A
choice only changes the schedule, never a value: the results are identical
whatever is picked (the parity tests run every split, layout and table
option).
"""
from __future__ import annotations

import ctypes
import json
import math
import os

import numpy as np
import torch

from . import abi
from . import host as H
from . import schedule as S

HERE = os.path.dirname(os.path.abspath(__file__))
DIM = 10


def model_path(name: str) -> str:
    return os.path.join(HERE, f"choice_{name}_model.npz")


# ------------------------------------------------------------------ encodings


def enc_ntt(log_n: int, ncols: int, split) -> list:
    r = list(split) + [0] * (3 - len(split))
    return [log_n / 25.0, math.log2(max(1, ncols)) / 6.0, r[0] / 12.0, r[1] / 12.0, r[2] / 12.0,
            len(split) / 3.0, max(split) / 12.0, min(split) / 12.0, 0.0, 0.0]


def enc_msm_table(n: int, batch: int, hist, table: int) -> list:
    return [math.log2(max(1, n)) / 24.0, math.log2(max(1, batch)) / 6.0] + [float(x) for x in hist] + [float(table)]


def enc_extend(log_n: int, ext_bits: int, ncols: int, layout: str, chunk: int) -> list:
    return [log_n / 24.0, ext_bits / 4.0, math.log2(max(1, ncols)) / 6.0, 1.0 if layout == "pairs" else 0.0,
            math.log2(chunk) / 6.0, math.log2(max(1, ncols // chunk)) / 6.0, 0.0, 0.0, 0.0, 0.0]


def key_str(k) -> str:
    return json.dumps(k)


def candidates(record) -> list:
    return [json.loads(k) for k in record["times_ms"]]


def encode(name: str, record, cand) -> list:
    if name == "ntt_split":
        return enc_ntt(record["log_n"], record["ncols"], cand)
    if name == "msm_table":
        return enc_msm_table(record["n"], record["batch"], record["hist"], cand)
    return enc_extend(record["log_n"], record["ext_bits"], record["ncols"], cand[0], cand[1])


def size_of(name: str, record) -> int:
    return record["n"].bit_length() - 1 if name == "msm_table" else record["log_n"]


# ------------------------------------------------------------------ exhaustive data


def collect_ntt(log_ns, ncols_list=(1, 8, 32), reps=2, max_elems=1 << 30):
    """One record per (log_n, ncols): the time of every split."""
    out = []
    for log_n in log_ns:
        for ncols in ncols_list:
            if (ncols << log_n) > max_elems:
                continue
            best, times = S.autotune_ntt(log_n, ncols, reps)
            out.append({"log_n": log_n, "ncols": ncols, "best": best,
                        "times_ms": {key_str(list(k)): v for k, v in times.items()}})
            torch.cuda.empty_cache()
    return out


def collect_msm_table(sizes, batches=(1, 4, 8), mixes=S.MIXES, reps=2, seed=300):
    """One record per (n, batch, mix): the whole batch's time through a table
    pipeline (1) and through a plain pipeline (0)."""
    out = []
    L = S.lib()
    nmax = max(sizes)
    bases, _ = S.bases_with_known_logs(nmax, seed)
    for n in sizes:
        cw = L.zkp_msm_batch_table_default_window((ctypes.c_uint32 * 1)(n), 1)
        table, c = H.msm_table_build(bases, n, cw)
        for batch in batches:
            for mi, mix in enumerate(mixes):
                cols = [S.scalars(n, mix, seed + 31 * n.bit_length() + 1000 * j + mi) for j in range(batch)]
                hist = S.histogram(cols[0])
                ns = [n] * batch
                times = {}
                for tab in (0, 1):
                    def run():
                        if tab:
                            return H.msm_batch_table(table, n, c, cols, ns)
                        return H.msm_batch(bases, cols, ns)
                    run()
                    torch.cuda.synchronize()
                    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                    a.record()
                    for _ in range(reps):
                        run()
                    b.record()
                    b.synchronize()
                    times[key_str(tab)] = a.elapsed_time(b) / reps
                out.append({"n": n, "batch": batch, "mix": mix, "hist": hist, "table_window": c,
                            "best": min(times, key=times.get), "times_ms": times})
                del cols
        del table
        torch.cuda.empty_cache()
    return out


def collect_extend(shapes, reps=2):
    """shapes: (log_n, ext_bits, ncols); one record each with the time of every
    (layout, columns per launch)."""
    out = []
    for log_n, ext_bits, ncols in shapes:
        chunks = tuple(c for c in (1, 2, 4, 8, 16, 32) if c <= ncols and ncols % c == 0)
        best, times = S.autotune_extend(log_n, ext_bits, ncols, chunks=chunks, reps=reps)
        out.append({"log_n": log_n, "ext_bits": ext_bits, "ncols": ncols, "best": list(best),
                    "times_ms": {key_str(list(k)): v for k, v in times.items()}})
        torch.cuda.empty_cache()
    return out


# ------------------------------------------------------------------ training, picking, regret


def training_set(name: str, records):
    """Inputs, per-shape centred log-time targets and sqrt(best ms) weights
    (as the MSM window model)."""
    X, y, w = [], [], []
    for r in records:
        logs = {k: math.log(v) for k, v in r["times_ms"].items()}
        mean = sum(logs.values()) / len(logs)
        wt = math.sqrt(min(r["times_ms"].values()))
        for k, lt in logs.items():
            X.append(encode(name, r, json.loads(k)))
            y.append(lt - mean)
            w.append(wt)
    w = np.array(w, np.float32)
    return np.array(X, np.float32), np.array(y, np.float32), w / w.mean()


class ChoiceModel:
    def __init__(self, name: str, model: S.Model):
        self.name, self.m = name, model

    @classmethod
    def load(cls, name: str, path=None):
        return cls(name, S.Model.load(path or model_path(name)))

    @classmethod
    def train(cls, name: str, records, steps=4000, seed=1):
        m = S.Model.fresh(seed)
        X, y, w = training_set(name, records)
        hist = m.train(X, y, steps=steps, weights=w)
        return cls(name, m), hist

    def save(self, path=None, meta=None):
        self.m.save(path or model_path(self.name), meta)

    def pick(self, record, cands=None):
        """The candidate with the smallest predicted time (record carries the
        shape; cands defaults to the record's measured candidates)."""
        cands = cands if cands is not None else candidates(record)
        X = np.array([encode(self.name, record, c) for c in cands], np.float32)
        return cands[int(np.argmin(self.m.predict(X)))]

    def pick_many(self, records, cands):
        """pick() for many records over the same candidates, in one forward
        pass of the model."""
        if not records:
            return []
        X = np.array([encode(self.name, r, c) for r in records for c in cands], np.float32)
        y = self.m.predict(X).reshape(len(records), len(cands))
        return [cands[int(i)] for i in np.argmin(y, axis=1)]


def default_pick(name: str, record):
    """The library's fixed rule for the choice."""
    if name == "ntt_split":
        return H.ntt_default_plan(record["log_n"])
    if name == "msm_table":
        return 1
    # the extend phase: Montgomery tables at 2^22 and above, pairs below; 8 columns per launch
    chunk = 8 if record["ncols"] >= 8 else record["ncols"]
    return ["montgomery" if record["log_n"] >= 22 else "pairs", chunk]


def regret(records, picker):
    total, rows = 0.0, []
    for r in records:
        best = min(r["times_ms"].values())
        k = key_str(picker(r))
        t = r["times_ms"].get(k)
        if t is None:  # a pick that was not measured (should not happen): charge the worst
            t = max(r["times_ms"].values())
        rows.append({"shape": {kk: r[kk] for kk in r if kk not in ("times_ms", "best", "hist")},
                     "picked": json.loads(k), "regret_ms": t - best})
        total += t - best
    return total, rows


def evaluate(name: str, records, steps=4000):
    """Train on even sizes, judge on odd ones; returns (model, report)."""
    train = [r for r in records if size_of(name, r) % 2 == 0]
    test = [r for r in records if size_of(name, r) % 2 == 1]
    model, hist = ChoiceModel.train(name, train, steps=steps)
    learned, rows_l = regret(test, model.pick)
    fixed, rows_f = regret(test, lambda r: default_pick(name, r))
    best_total = sum(min(r["times_ms"].values()) for r in test)
    return model, {"choice": name, "train_shapes": len(train), "test_shapes": len(test),
                   "best_total_ms": best_total, "regret_learned_ms": learned, "regret_fixed_rule_ms": fixed,
                   "loss": hist, "rows_learned": rows_l, "rows_fixed_rule": rows_f}
