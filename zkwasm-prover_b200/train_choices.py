"""Train the three learned schedule choices on this GPU (choices.py).

    python zkwasm-prover_b200/train_choices.py OUT_DIR [DATA.json]

With DATA.json (a choices_data.json written earlier) the timings are read
from it instead of measured again.

1. times every candidate of every shape with the exhaustive tuners:
   NTT pass splits (2^13..2^25, 1 / 8 / 32 columns), MSM table or plain
   pipeline (2^12..2^22, batches of 1 / 4 / 8, four scalar distributions),
   extended-domain layout and columns per launch (2^16..2^22, e = 1..3,
   8 and 16 columns);
2. trains one MLP per choice with the library's kernels on the even sizes;
3. reports the held-out regret (odd sizes, ms against the tuner's best) of
   the learned pick and of the library's fixed rule;
4. writes OUT_DIR/choice_<name>_model.npz, OUT_DIR/choices_data.json and
   OUT_DIR/choices_eval.json.
"""
import importlib
import json
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))


def main(out_dir, data_path=None):
    C = importlib.import_module("zkwasm-prover_b200.choices")
    os.makedirs(out_dir, exist_ok=True)
    if data_path:
        with open(data_path) as f:
            data = json.load(f)
    else:
        data = {}
        data["ntt_split"] = C.collect_ntt(range(13, 26))
        data["msm_table"] = C.collect_msm_table([1 << k for k in range(12, 23)])
        data["extend"] = C.collect_extend([(k, e, c) for k in range(16, 23) for e in (1, 2, 3) for c in (8, 16)])
        with open(os.path.join(out_dir, "choices_data.json"), "w") as f:
            json.dump(data, f)
    report = {}
    for name, records in data.items():
        model, rep = C.evaluate(name, records)
        model.save(os.path.join(out_dir, f"choice_{name}_model.npz"),
                   meta={"choice": name, "regret_learned_ms": rep["regret_learned_ms"],
                         "regret_fixed_rule_ms": rep["regret_fixed_rule_ms"]})
        report[name] = rep
        print(name, {k: v for k, v in rep.items() if not k.startswith("rows") and k != "loss"}, flush=True)
    with open(os.path.join(out_dir, "choices_eval.json"), "w") as f:
        json.dump(report, f, indent=1)


if __name__ == "__main__":
    main(sys.argv[1], sys.argv[2] if len(sys.argv) > 2 else None)
