"""Host-side argument checks of every entry point: null pointers, undersized
scratch, out-of-range sizes, window widths and pass splits, and a drop-in
`msm()` region that fits no window plan.  Each call must return
cudaErrorInvalidValue (1) before it enqueues anything.

These run where no GPU is present, on fake (never dereferenced) non-null
addresses: a check that failed to catch its argument would try to launch, and
without a device that returns a different error code, so the exact value 1
shows the call stopped at its argument check.  With a GPU present the module
is skipped, since a missed check would launch on the fake addresses there."""
import ctypes

import pytest

F = 0x10000  # a fake device address (never dereferenced)
INVALID = 1  # cudaErrorInvalidValue


@pytest.fixture(scope="module")
def L(zkp):
    import torch

    if torch.cuda.is_available():
        pytest.skip("argument checks are exercised on fake addresses, only where no GPU is present")
    return zkp.load_library()


def _nulls(fn, args, ptr_idx, expect=INVALID):
    """Call fn with each pointer argument of ptr_idx set to NULL in turn."""
    for i in ptr_idx:
        a = list(args)
        a[i] = None
        assert fn(*a) == expect, f"{fn.__name__}: NULL argument {i} accepted"


N = 1 << 12


def test_reference_symbols_reject_null_pointers(L):
    sw = ctypes.c_bool(False)
    sa = ctypes.addressof(sw)
    _nulls(L.ntt, [F, F, F, F, F, 13, 8, sa, None], [0, 1, 3, 7])
    _nulls(L.permutation_eval_h_p1, [F, F, F, F, F, F, N], range(6))
    _nulls(L.permutation_eval_h_p2, [F, F, F, F, F, 4, -3, N], [0, 1, 2, 4])
    _nulls(L.permutation_eval_h_l, [F, F, F, F, N, None], range(4))
    _nulls(L.field_sum, [F, F, F, F, F, 3, N], range(5))
    _nulls(L.field_op_batch_mul_sum, [F, F, F, 4, N, None], range(3))
    _nulls(L.lookup_eval_h, [F] * 12 + [1, N, None], range(12))
    _nulls(L.logup_eval_h, [F] * 11 + [1, N, None], range(11))
    _nulls(L.logup_eval_h_extra_inputs, [F] * 6 + [1, N, None], range(6))
    _nulls(L.logup_eval_h_z_set, [F, F, F, F, F, 3, -2, N, None], [0, 1, 2, 4])
    _nulls(L.logup_sum_input_inv, [F, F, F, F, 0, N, None], [0, 1, 3])
    _nulls(L.logup_eval_h_inputs_product_sum, [F, F, F, 2, N, None], range(3))
    _nulls(L.shuffle_eval_h, [F] * 8 + [1, N], range(8))
    _nulls(L.shuffle_eval_h_v2, [F, F, F, F, 2, F, F, F, F, F, 1, N], [0, 1, 2, 3, 5, 6, 7, 8, 9])
    _nulls(L.expand_omega_buffer, [F, 12, 0], [0])
    _nulls(L.field_mul_zip, [F, F, 3, N], [0, 1])
    _nulls(L.poly_eval, [F, F, F, N, None], range(3))
    _nulls(L.shplonk_h_x_merge, [F, F, F, F, F, 3, N], range(5))
    _nulls(L.shplonk_h_x_div_points, [F, F, F, 4, N], range(3))
    _nulls(L.eval_logup_z_compose, [F, F, F, F, F, F, 5, N, None], range(6))
    _nulls(L.eval_logup_z_pure, [F, F, F, F, 5, N, None], [0, 2, 3])
    _nulls(L.batch_msm_collect, [F, F, F, F, F, 64, 20, 13, 2, None], [4])
    _nulls(L.msm, [F, F, F, F, F, F, F, F, F, N, 20, 13, 64, 64, 4 * N, 1, None], [0, 1, 2, 7])
    _nulls(L.prepare_table_lookup, [F] * 7 + [N * 32, 12, N - 9, None], [0, 5])
    _nulls(L.calc_m, [F] * 8 + [N * 32, 12, N - 9, None], [0, 1, 2, 4, 5])


def test_field_op_operand_rules(L):
    # op 0 (add) with no R operand at all, an unknown op, no L operand
    assert L.field_op(F, F, 0, None, None, 0, None, N, 0, None) == INVALID
    assert L.field_op(F, F, 0, None, F, 0, None, N, 4, None) == INVALID
    assert L.field_op(F, None, 0, None, F, 0, None, N, 1, None) == INVALID
    assert L.field_op(None, F, 0, None, F, 0, None, N, 0, None) == INVALID
    assert L.field_op(F, F, 0, None, F, 0, None, -1, 0, None) == INVALID


def test_reference_symbols_reject_bad_sizes(L):
    sw = ctypes.c_bool(False)
    sa = ctypes.addressof(sw)
    assert L.ntt(F, F, F, F, None, 29, 8, sa, None) == INVALID
    assert L.ntt(F, None, F, F, None, 13, 8, sa, None) == INVALID  # a multi-pass size needs tmp
    assert L.extended_prepare(F, F, 3, 2 * N, N, 0, None) == INVALID  # size beyond the extended size
    assert L.extended_prepare(F, None, 3, N, 4 * N, 0, None) == INVALID
    assert L.extended_prepare(F, F, 0, N, 4 * N, 0, None) == INVALID
    assert L.expand_omega_buffer(F, 31, 0) == INVALID
    assert L.field_mul_zip(F, F, 0, N) == INVALID
    assert L.poly_eval(F, F, F, 3 * 64, None) == INVALID  # not a power of two
    assert L.poly_eval(F, F, F, 0, None) == INVALID
    assert L.logup_eval_h_inputs_product_sum(F, F, F, 0, N, None) == INVALID
    assert L.shuffle_eval_h_v2(F, F, F, F, 0, F, F, F, F, F, 1, N) == INVALID
    assert L.eval_logup_z_compose(F, F, F, F, F, F, N, N, None) == INVALID  # last_z_index out of range
    assert L.eval_logup_z_pure(F, F, F, F, -1, N, None) == INVALID
    assert L.prepare_table_lookup(F, F, F, F, F, F, F, N * 32, 28, 0, None) == INVALID
    assert L.prepare_table_lookup(F, F, F, F, F, F, F, N * 32, 12, N + 1, None) == INVALID
    assert L.calc_m(F, F, F, F, F, F, F, F, N * 32, 12, N + 1, None) == INVALID


def test_dropin_msm_region_that_fits_no_plan(L):
    # windows << c plus 2 * workers Jacobian points no larger than the region's
    # 256-byte head
    assert L.msm(F, F, F, F, F, F, F, F, F, N, 1, 1, 64, 0, 4 * N, 1, None) == INVALID
    # a region of 8 points (768 bytes) and a sort buffer of 3 * n * 2 words:
    # no window from 4 to 22 bits fits both
    assert L.msm(F, F, F, F, F, F, F, F, F, 1 << 20, 2, 2, 64, 0, 6 << 22, 1, None) == INVALID
    # window widths outside what the reference host can ask for
    assert L.msm(F, F, F, F, F, F, F, F, F, N, 20, 0, 64, 64, 4 * N, 1, None) == INVALID
    assert L.msm(F, F, F, F, F, F, F, F, F, N, 20, 25, 64, 64, 4 * N, 1, None) == INVALID


def test_batched_entry_points_reject_bad_arguments(L):
    U32 = ctypes.c_uint32
    I32 = ctypes.c_int
    # MSM: undersized scratch, missing buffers, more points than the table holds
    need = L.zkp_msm_scratch_bytes(N, 0)
    assert need > 0
    assert L.zkp_msm(F, F, F, N, 0, F, need - 1, None) == INVALID
    _nulls(L.zkp_msm, [F, F, F, N, 0, F, need, None], [0, 1, 2, 5])
    assert L.zkp_msm_table_build(F, F, N, 30, None) == INVALID
    assert L.zkp_msm_table(F, F, N, 16, F, N + 1, F, 1 << 30, None) == INVALID
    ns = (U32 * 3)(N, N // 2, 64)
    need_b = L.zkp_msm_batch_scratch_bytes(ctypes.addressof(ns), None, 3)
    assert need_b > 0
    assert L.zkp_msm_batch(F, F, F, ctypes.addressof(ns), None, 3, F, need_b - 1, None) == INVALID
    _nulls(L.zkp_msm_batch, [F, F, F, ctypes.addressof(ns), None, 3, F, need_b, None], [0, 1, 2, 3, 6])
    assert L.zkp_msm_batch_table(F, F, 0, 16, F, ctypes.addressof(ns), 3, F, 1 << 40, None) == INVALID
    # an MSM longer than the table's bases
    assert L.zkp_msm_batch_table(F, F, N // 2, 16, F, ctypes.addressof(ns), 3, F, 1 << 40, None) == INVALID
    assert L.zkp_msm_static(None, F, F, 16, None) == INVALID
    assert L.zkp_msm_static(F, F, F, (1 << 14) + 1, None) == INVALID
    # NTT: sizes, column counts, pass splits
    res = I32(0)
    ra = ctypes.addressof(res)
    assert L.zkp_ntt_batch(F, F, F, None, 0, 1, N, ra, None) == INVALID
    assert L.zkp_ntt_batch(F, F, F, None, 29, 1, N, ra, None) == INVALID
    assert L.zkp_ntt_batch(F, F, F, None, 12, 0, N, ra, None) == INVALID
    assert L.zkp_ntt_batch(F, None, F, None, 13, 1, N, ra, None) == INVALID
    _nulls(L.zkp_ntt_batch, [F, F, F, None, 12, 1, N, ra, None], [0, 2, 7])
    for rad in ([7, 7], [6, 5, 5], [13, 3], [4, 4, 4, 2, 2]):
        r = (I32 * len(rad))(*rad)
        assert L.zkp_ntt_batch_plan(F, F, F, None, 16, 1, N, ctypes.addressof(r), len(rad), ra, None) == INVALID
    # coset tables and the extension phase
    assert L.zkp_coset_twist_tables(F, F, F, 12, 7, F, None) == INVALID
    assert L.zkp_coset_twist_tables(None, F, F, 12, 3, F, None) == INVALID
    assert L.zkp_extend_table_elems(25, 3) == 0
    assert L.zkp_extend_batch_tables(F, F, F, 1, 12, 3, None, F, None, None) == INVALID
    assert L.zkp_extend_batch_tables(F, F, F, 1, 25, 3, F, F, None, None) == INVALID
    _nulls(L.zkp_extend_batch, [F, F, F, 1, 12, 3, F, F, F, F, F, None, None], [0, 2, 6, 7, 8, 9, 10])
    assert L.zkp_powers(None, F, F, N, None) == INVALID
    # scans, inversions, grand products
    _nulls(L.zkp_batch_inverse, [F, F, F, N, 0, F, None], [0, 1])
    _nulls(L.zkp_grand_product, [F, F, N, F, F, None], [0, 1, 4])
    _nulls(L.zkp_grand_sum, [F, F, N, F, F, None], [0, 1, 4])
    _nulls(L.zkp_permutation_z, [F, F, F, 4, F, F, F, F, F, N, F, None], [0, 1, 2, 4, 5, 6, 7, 10])
    assert L.zkp_permutation_z(F, F, F, 0, F, F, F, F, F, N, F, None) == INVALID
    _nulls(L.zkp_shuffle_z, [F, F, F, F, 2, N, F, None], [0, 1, 2, 3, 6])
    assert L.zkp_shuffle_z(F, F, F, F, 0, N, F, None) == INVALID
    _nulls(L.zkp_fr_to_mont, [F, F, N, None], [0, 1])
    _nulls(L.zkp_g1_multiples, [F, F, N, None], [0, 1])
    # learned schedule and staging
    assert L.zkp_mlp_init(None, 1, None) == INVALID
    assert L.zkp_mlp_forward(None, F, 4, F, None) == INVALID
    assert L.zkp_scalar_histogram(None, N, F, None) == INVALID
    assert L.zkp_copy_queue_push(None, F, F, 64, 1, None) == INVALID
    assert L.zkp_copy_queue_sync(None) == INVALID
