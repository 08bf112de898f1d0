"""The C-ABI library loads without a GPU and exports every symbol that
include/*.h declares: the reference's 27 (src/cuda/bn254_c.rs:4-309) and the
batched zkp_* entry points."""
import ctypes
import os
import subprocess

REF_SYMBOLS = [
    "ntt", "field_op", "extended_prepare", "permutation_eval_h_p1", "permutation_eval_h_p2",
    "permutation_eval_h_l", "field_sum", "field_op_batch_mul_sum", "lookup_eval_h", "logup_eval_h",
    "logup_eval_h_extra_inputs", "logup_eval_h_z_set", "logup_sum_input_inv",
    "logup_eval_h_inputs_product_sum", "shuffle_eval_h", "shuffle_eval_h_v2", "expand_omega_buffer",
    "field_mul_zip", "poly_eval", "shplonk_h_x_merge", "shplonk_h_x_div_points", "eval_logup_z_compose",
    "eval_logup_z_pure", "batch_msm_collect", "msm", "prepare_table_lookup", "calc_m",
]


def test_header_declares_reference_symbols(zkp):
    declared = zkp.abi.declared_symbols()
    assert len(REF_SYMBOLS) == 27
    for s in REF_SYMBOLS:
        assert s in declared, s
    assert len(set(declared)) == len(declared)


def test_library_exports_declared_symbols(zkp):
    lib = zkp.load_library()
    for s in zkp.abi.declared_symbols():
        assert hasattr(lib, s), s
        assert s in zkp.abi.SIGNATURES, s
    # the shared object exports them as plain C symbols (no C++ mangling)
    out = subprocess.check_output(["nm", "-D", "--defined-only", zkp.LIB_PATH], text=True)
    exported = {line.split()[-1] for line in out.splitlines() if " T " in line}
    for s in zkp.abi.declared_symbols():
        assert s in exported, s


def test_static_archive_for_rust_link(zkp):
    # build.rs:10 links `zkwasm_prover_kernel` statically
    a = os.path.join(os.path.dirname(zkp.LIB_PATH), "libzkwasm_prover_kernel.a")
    assert os.path.exists(a)
    out = subprocess.check_output(["nm", "--defined-only", a], text=True)
    for s in REF_SYMBOLS:
        assert f" T {s}\n" in out + "\n", s


def test_scratch_queries_without_gpu(zkp):
    lib = zkp.load_library()
    for n in (1, 1 << 10, 1 << 18, 1 << 22):
        c = lib.zkp_msm_default_window(n)
        assert 4 <= c <= 22
        assert lib.zkp_msm_scratch_bytes(n, 0) > 0
    assert lib.zkp_scan_scratch_elems(1 << 22) >= (1 << 22) // 2048
