"""ctypes binding of libzkwasm_prover_kernel.so (include/zkwasm_prover_kernel.h).

This is the binding a Python caller (or the parity tests) uses; the Rust host
binds the same symbols through src/cuda/bn254_c.rs.  Pointers are passed as
integers (``tensor.data_ptr()``), streams as ``torch.cuda.Stream.cuda_stream``.
"""
from __future__ import annotations

import ctypes
import os
import re

from . import LIB_PATH, HERE

P = ctypes.c_void_p
I = ctypes.c_int
U = ctypes.c_uint32
SZ = ctypes.c_size_t
S = ctypes.c_void_p  # cudaStream_t
E = ctypes.c_int     # cudaError_t

SIGNATURES = {
    # Part 1: reference-compatible (src/cuda/bn254_c.rs:4-309)
    "ntt": [P, P, P, P, P, I, I, P, S],
    "field_op": [P, P, I, P, P, I, P, I, I, S],
    "extended_prepare": [P, P, I, I, I, I, S],
    "permutation_eval_h_p1": [P, P, P, P, P, P, I],
    "permutation_eval_h_p2": [P, P, P, P, P, I, I, I],
    "permutation_eval_h_l": [P, P, P, P, I, S],
    "field_sum": [P, P, P, P, P, I, I],
    "field_op_batch_mul_sum": [P, P, P, I, I, S],
    "lookup_eval_h": [P, P, P, P, P, P, P, P, P, P, P, P, I, I, S],
    "logup_eval_h": [P, P, P, P, P, P, P, P, P, P, P, I, I, S],
    "logup_eval_h_extra_inputs": [P, P, P, P, P, P, I, I, S],
    "logup_eval_h_z_set": [P, P, P, P, P, I, I, I, S],
    "logup_sum_input_inv": [P, P, P, P, I, I, S],
    "logup_eval_h_inputs_product_sum": [P, P, P, I, I, S],
    "shuffle_eval_h": [P, P, P, P, P, P, P, P, I, I],
    "shuffle_eval_h_v2": [P, P, P, P, I, P, P, P, P, P, I, I],
    "expand_omega_buffer": [P, I, I],
    "field_mul_zip": [P, P, I, I],
    "poly_eval": [P, P, P, I, S],
    "shplonk_h_x_merge": [P, P, P, P, P, I, I],
    "shplonk_h_x_div_points": [P, P, P, I, I],
    "eval_logup_z_compose": [P, P, P, P, P, P, I, I, S],
    "eval_logup_z_pure": [P, P, P, P, I, I, S],
    "batch_msm_collect": [P, P, P, P, P, U, U, U, U, S],
    "msm": [P, P, P, P, P, P, P, P, P, I, I, I, I, I, I, I, S],
    "prepare_table_lookup": [P, P, P, P, P, P, P, U, U, U, S],
    "calc_m": [P, P, P, P, P, P, P, P, U, U, U, S],
    # Part 2: batched, allocation-free
    "zkp_msm_scratch_bytes": ([U, I], SZ),
    "zkp_msm_default_window": ([U], I),
    "zkp_msm": [P, P, P, U, I, P, SZ, S],
    "zkp_msm_table_bytes": ([U, I], SZ),
    "zkp_msm_table_default_window": ([U], I),
    "zkp_msm_table_build": [P, P, U, I, S],
    "zkp_msm_table_scratch_bytes": ([U, I], SZ),
    "zkp_msm_table": [P, P, U, I, P, U, P, SZ, S],
    "zkp_msm_batch_table_default_window": ([P, U], I),
    "zkp_msm_batch_table_scratch_bytes": ([P, U, U, I], SZ),
    "zkp_msm_batch_table": [P, P, U, I, P, P, U, P, SZ, S],
    "zkp_msm_batch_scratch_bytes": ([P, P, U], SZ),
    "zkp_msm_batch": [P, P, P, P, P, U, P, SZ, S],
    "zkp_ntt_batch": [P, P, P, P, I, U, SZ, P, S],
    "zkp_ntt_default_plan": ([I, P], I),
    "zkp_ntt_batch_plan": [P, P, P, P, I, U, SZ, P, I, P, S],
    "zkp_powers": [P, P, P, U, S],
    "zkp_coset_table_elems": ([I, I], SZ),
    "zkp_coset_twist_tables": [P, P, P, I, I, P, S],
    "zkp_extend_batch": [P, P, P, U, I, I, P, P, P, P, P, P, S],
    "zkp_extend_table_elems": ([I, I], SZ),
    "zkp_extend_tables": [P, P, P, P, P, P, I, I, S],
    "zkp_extend_batch_tables": [P, P, P, U, I, I, P, P, P, S],
    "zkp_batch_inverse": [P, P, P, U, I, P, S],
    "zkp_scan_scratch_elems": ([U], SZ),
    "zkp_scan_timeouts": ([], U),
    "zkp_g1_multiples": [P, P, U, S],
    "zkp_fr_to_mont": [P, P, U, S],
    "zkp_grand_product": [P, P, U, P, P, S],
    "zkp_grand_sum": [P, P, U, P, P, S],
    "zkp_permutation_z": [P, P, P, I, P, P, P, P, P, U, P, S],
    "zkp_shuffle_z": [P, P, P, P, I, U, P, S],
    "zkp_msm_static": [P, P, P, U, S],
    "zkp_scalar_histogram": [P, U, P, S],
    "zkp_msm_autotune": ([P, P, U, I, I, I, P, SZ, P, P, S], I),
    "zkp_mlp_input_dim": ([], I),
    "zkp_mlp_param_count": ([], SZ),
    "zkp_mlp_scratch_floats": ([U], SZ),
    "zkp_mlp_init": [P, ctypes.c_uint64, S],
    "zkp_mlp_forward": [P, P, U, P, S],
    "zkp_mlp_grad": [P, P, P, P, U, P, P, P, S],
    "zkp_mlp_train_step": [P, P, P, P, P, P, P, U, ctypes.c_float, I, P, P, S],
    "zkp_msm_schedule_predict": ([P, P, I, I, P, S], I),
    "zkp_ntt_batch_twisted": [P, P, P, P, P, P, I, U, SZ, SZ, I, S],
    "zkp_shoup_pairs": [P, P, U, S],
    "zkp_eval_h_fused": [P, P, S],
    "zkp_coset_combine": [P, P, SZ, P, P, I, I, S],
    "zkp_poly_divide_scratch_elems": ([U], SZ),
    "zkp_poly_divide_linear": [P, P, P, U, P, S],
    "zkp_poly_eval_batch_scratch_elems": ([U], SZ),
    "zkp_poly_eval_batch": [P, P, U, P, U, P, S],
    "zkp_calib_mont_rate": [P, U, U, S],
    "zkp_calib_shoup_rate": [P, P, U, U, S],
    # Part 4: host staging (csrc/staging.cu)
    "zkp_host_pool_create": ([SZ, I, I], P),
    "zkp_host_pool_alloc": ([P, SZ], P),
    "zkp_host_pool_free": ([P, P], I),
    "zkp_host_pool_stats": ([P, P, P], None),
    "zkp_host_pool_destroy": ([P], None),
    "zkp_copy_queue_create": ([I, I], P),
    "zkp_copy_queue_push": [P, P, P, SZ, I, S],
    "zkp_copy_queue_sync": [P],
    "zkp_copy_queue_destroy": ([P], None),
}

_lib = None


class CudaError(RuntimeError):
    pass


class _Strict:
    """The CDLL with every declared function wrapped in an exact-arity check:
    ctypes otherwise passes surplus arguments as varargs, which silently
    shifts every later argument (a stream handle becomes garbage)."""

    def __init__(self, cdll):
        self._cdll = cdll
        # per-entry-point call counts while counting is on (benchmark
        # instrumentation: each call of a compute entry point launches one or
        # more kernels)
        self.calls = None
        for name, sig in SIGNATURES.items():
            fn = getattr(cdll, name)
            argtypes, restype = sig if isinstance(sig, tuple) else (sig, E)
            fn.argtypes, fn.restype = argtypes, restype
            setattr(self, name, self._wrap(name, fn, len(argtypes)))

    def _wrap(self, name, fn, arity):
        def call(*args):
            if len(args) != arity:
                raise TypeError(f"{name} takes {arity} arguments, got {len(args)}")
            if self.calls is not None:
                self.calls[name] = self.calls.get(name, 0) + 1
            return fn(*args)

        call.__name__ = name
        return call

    def __getattr__(self, name):
        return getattr(self._cdll, name)


def load_library(path: str = LIB_PATH):
    """Load the kernel library; raises if it has not been built."""
    global _lib
    if _lib is not None and path == LIB_PATH:
        return _lib
    if not os.path.exists(path):
        raise ImportError(f"{path} is missing: run __graft_entry__.build() (make -C csrc)")
    lib = _Strict(ctypes.CDLL(path, mode=ctypes.RTLD_GLOBAL))
    if path == LIB_PATH:
        _lib = lib
    return lib


def check(err: int, what: str = ""):
    if err != 0:
        raise CudaError(f"{what} failed with cudaError {err}")


def declared_symbols(header_dir: str | None = None) -> list:
    """Function names declared in include/*.h (for the export test)."""
    header_dir = header_dir or os.path.join(os.path.dirname(HERE), "include")
    names = []
    for fn in sorted(os.listdir(header_dir)):
        if not fn.endswith(".h"):
            continue
        text = open(os.path.join(header_dir, fn)).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        for m in re.finditer(r"^\s*(?:cudaError_t|size_t|int)\s+([A-Za-z_]\w*)\s*\(", text, flags=re.M):
            names.append(m.group(1))
    return names
