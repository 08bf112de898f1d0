"""Host-side pieces of bench.py that need no GPU: the roofline traffic figure
is taken from the committed ncu capture only for the captured size and only
while the transform's source is the one that capture ran."""
import hashlib
import json
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

import bench  # noqa: E402


def test_coset_traffic_follows_the_capture(tmp_path, monkeypatch):
    prof = os.path.join(ROOT, "profiles", "coset_ntt_traffic.json")
    with open(prof) as f:
        d = json.load(f)
    src = os.path.join(ROOT, "zkwasm-prover_b200", "csrc", "ntt.cu")
    with open(src, "rb") as f:
        current = hashlib.sha256(f.read()).hexdigest() == d["source_sha256"]
    got = bench.coset_traffic(8, d["log_n"])
    if current:
        assert got == d["bytes_per_column"] * 8
        # per column: at least the algorithmic read and write of 2^log_n elements
        assert d["bytes_per_column"] >= 2 * (1 << d["log_n"]) * 32
    else:
        assert got is None
    # another size has no capture
    assert bench.coset_traffic(8, d["log_n"] - 1) is None
    # a changed source reads as stale
    fake = tmp_path / "repo"
    (fake / "profiles").mkdir(parents=True)
    (fake / "zkwasm-prover_b200" / "csrc").mkdir(parents=True)
    (fake / "profiles" / "coset_ntt_traffic.json").write_text(json.dumps(d))
    (fake / "zkwasm-prover_b200" / "csrc" / "ntt.cu").write_text("// changed\n")
    monkeypatch.setattr(bench, "ROOT", str(fake))
    assert bench.coset_traffic(8, d["log_n"]) is None


def test_kernel_counts_cover_multi_kernel_entry_points():
    calls = {"zkp_msm_batch_table": 2, "zkp_scan_scratch_elems": 5, "field_op": 3}
    # scratch queries launch nothing; every other call at least one kernel
    assert bench._launch_count(calls, None) == 2 * bench.KERNELS_PER_CALL["zkp_msm_batch_table"] + 3
