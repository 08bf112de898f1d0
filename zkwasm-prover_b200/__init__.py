"""B200 (sm_100a) KZG proving hot path for BN254, behind the reference's C ABI.

The product is the in-tree shared library ``libzkwasm_prover_kernel.so``
(built from ``csrc/`` by ``build()``), exporting the 27 symbols the reference's
Rust host links against (src/cuda/bn254_c.rs:4-309) plus batched ``zkp_*``
entry points; see ``include/zkwasm_prover_kernel.h``.

``host`` mirrors the reference's host-side wrappers for this path
(src/cuda/ntt.rs, src/cuda/msm.rs, src/cuda/bn254.rs) over torch device
memory, so callers and tests read like the reference's own.  There is no CPU
fallback: every entry point goes through the CUDA library and raises if it is
missing.
"""
from __future__ import annotations

import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libzkwasm_prover_kernel.so")
CSRC = os.path.join(HERE, "csrc")


def build(jobs: int = 8) -> str:
    """Compile csrc/*.cu for sm_100a into the in-tree library (make -C csrc)."""
    subprocess.check_call(["make", "-s", "-C", CSRC, f"-j{jobs}"])
    return LIB_PATH


from . import abi  # noqa: E402
from . import host  # noqa: E402
from . import schedule  # noqa: E402
from .abi import load_library  # noqa: E402

__all__ = ["build", "load_library", "abi", "host", "schedule", "LIB_PATH"]
