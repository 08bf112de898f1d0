"""Train the MSM schedule model on this GPU.

    python zkwasm-prover_b200/train_schedule.py OUT_DIR [RECORDS.json]

With RECORDS.json (a msm_schedule_data.json written earlier) the timings are
read from it instead of measured again.

1. autotunes every (size, batch, scalar mix) shape for sizes 2^12..2^22,
   batches of 1, 4, 16 and 32 same-size MSMs in one zkp_msm_batch pipeline
   (at most 2^26 scalars per batch) and four scalar distributions (uniform,
   small < 2^20, 90%-sparse, mixed);
2. trains the MLP with the library's kernels on the even sizes (weighted
   mean squared error of per-shape centred log times);
3. evaluates the window picked by the model, by the library's default
   formula and by the reference's formula (src/cuda/msm.rs:105) on the
   held-out odd sizes, as regret in ms against the autotuner's best;
4. writes OUT_DIR/msm_schedule_model.npz, OUT_DIR/msm_schedule_data.json and
   OUT_DIR/msm_schedule_eval.json.
"""
import importlib
import json
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))


def main(out_dir, records_path=None):
    zkp = importlib.import_module("zkwasm-prover_b200")
    S = zkp.schedule
    os.makedirs(out_dir, exist_ok=True)
    sizes = [1 << k for k in range(12, 23)]
    if records_path:
        with open(records_path) as f:
            records = json.load(f)
    else:
        records = S.collect(sizes, batches=(1, 4, 16, 32), max_points=1 << 26)
    train = [r for r in records if (r["n"].bit_length() - 1) % 2 == 0]
    test = [r for r in records if (r["n"].bit_length() - 1) % 2 == 1]
    X, y, w = S.training_set(train)
    model = S.Model.fresh(seed=7)
    loss_hist = model.train(X, y, steps=10000, lr=3e-3, weights=w)

    def learned(r):
        return model.pick(S.shape_features(r["n"], r["batch"], r["hist"]))

    out = {"loss_history": loss_hist, "train_shapes": len(train), "test_shapes": len(test),
           "candidates": [S.C_MIN, S.C_MAX]}
    for name, recs in (("train", train), ("test", test)):
        res = {}
        for pname, picker in (("learned", learned), ("default", lambda r: S.default_window(r["n"])),
                              ("reference_formula", lambda r: S.reference_window(r["n"], r["batch"]))):
            tot, rows = S.regret(recs, picker)
            res[pname] = {"total_regret_ms": tot, "rows": rows}
        res["best_total_ms"] = sum(min(r["times_ms"].values()) for r in recs)
        out[name] = res
    model.save(os.path.join(out_dir, "msm_schedule_model.npz"),
               meta={"trained_on": "even log2 sizes 12..22, batches 1/4/16/32"})
    with open(os.path.join(out_dir, "msm_schedule_data.json"), "w") as f:
        json.dump(records, f)
    with open(os.path.join(out_dir, "msm_schedule_eval.json"), "w") as f:
        json.dump(out, f, indent=1)
    print(json.dumps({k: {p: v[p]["total_regret_ms"] for p in ("learned", "default", "reference_formula")}
                      for k, v in out.items() if k in ("train", "test")}))


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else "schedule_out", sys.argv[2] if len(sys.argv) > 2 else None)
