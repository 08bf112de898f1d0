"""zkp_msm_static: the MSM entry point for callers that cannot allocate device
memory (a host whose device memory is all owned by its own pool, or a
latency-critical path that cannot take cudaMalloc's implicit
synchronisation).  Its scratch is a fixed array inside the library,
so this file checks, through the C ABI, that two calls in a row (the second
sees the first call's leftovers in that array) return the same points as the
existing zkp_msm entry point, and that oversized inputs are refused.

The file name sorts last so that a run stopping at the first failure has run
every other test already; it also passes alone in a fresh process.
"""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

MAX_N = 1 << 14


def _aff(O, t):
    torch.cuda.synchronize()
    return O.g1_jac_to_aff(t.detach().cpu().numpy().view(np.uint64).reshape(1, 12))


def test_static_msm_matches_zkp_msm_twice(O, gpu):
    H = gpu.host
    L = gpu.load_library()
    st = H.stream_handle()
    for n, seed in ((MAX_N, 1), (1000, 2)):
        d = O.rand_fr(n, 300 + seed)
        bases = H.to_device(O.g1_gen_bases(d))
        ref = H.msm(bases, H.to_device(O.rand_fr(n, 400 + seed)), n=n)
        exp = _aff(O, ref)
        scalars = H.to_device(O.rand_fr(n, 400 + seed))
        for _ in range(2):
            out = torch.zeros(12, dtype=torch.int64, device="cuda")
            gpu.abi.check(L.zkp_msm_static(out.data_ptr(), bases.data_ptr(), scalars.data_ptr(), n, st),
                          "zkp_msm_static")
            assert (_aff(O, out) == exp).all()


def test_static_msm_rejects_oversize(O, gpu):
    H = gpu.host
    L = gpu.load_library()
    out = torch.zeros(12, dtype=torch.int64, device="cuda")
    bases = torch.zeros((MAX_N + 1, 8), dtype=torch.int64, device="cuda")
    scalars = torch.zeros((MAX_N + 1, 4), dtype=torch.int64, device="cuda")
    err = L.zkp_msm_static(out.data_ptr(), bases.data_ptr(), scalars.data_ptr(), MAX_N + 1, H.stream_handle())
    assert err == 1  # cudaErrorInvalidValue, nothing launched
    torch.cuda.synchronize()
    assert int(out.abs().sum()) == 0
