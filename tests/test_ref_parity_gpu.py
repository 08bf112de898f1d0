"""This library against the reference's own CUDA kernels (cuda/bn254.cu and
cuda/msm.cu rebuilt for sm_100a into oracle/_ref/ by `make -C oracle ref`), on
identical seeded inputs, bit for bit.

* every quotient, multi-open, coset and lookup symbol of tests/ref_cases.py at
  n = 2^12 and 2^16, plus the outputs against the hashes the reference's own
  kernels produced (tests/golden/reference_kernels.json);
* the drop-in `ntt` at every size 2^13..2^25 (every built-in pass split of
  the default plan, radix-2^11 and three-pass ones included), forward and
  inverse, against the reference's `ntt`, and against the oracle's DFT up to
  2^24;
* the drop-in `msm` + `batch_msm_collect` for 8 columns of 2^22 points with
  the reference host's c = 13 sizing (src/cuda/msm.rs:275-317), against the
  reference's kernels and the known-discrete-log identity;
* the coset extension of the k = 22 proof's size (2^22 -> 2^25, e = 3) against
  the reference's iNTT -> extended_prepare -> NTT sequence
  (src/eval_h.rs:255-265)."""
import ctypes
import json
import os

import numpy as np
import pytest
import torch

import ref_cases as RC

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "reference_kernels.json")


@pytest.fixture(scope="module")
def libs(gpu):
    if not os.path.exists(RC.REF_LIB):
        pytest.skip("reference kernels not built (make -C oracle ref)")
    return gpu.load_library(), RC.load_ref()


def _cmp(a, b, what):
    assert set(a) == set(b), what
    for k in a:
        assert a[k].shape == b[k].shape, f"{what}: {k} shape"
        bad = np.nonzero((a[k] != b[k]).any(axis=-1) if a[k].ndim > 1 else a[k] != b[k])[0]
        assert bad.size == 0, f"{what}: {k} differs at {bad.size} rows, first {bad[:5].tolist()}"


@pytest.mark.parametrize("n", [1 << 12, 1 << 16])
@pytest.mark.parametrize("name", [c.name for c in RC.CASES])
def test_symbol_matches_reference_kernels(libs, name, n):
    ours, ref = libs
    case = next(c for c in RC.CASES if c.name == name)
    if n < case.min_n:
        pytest.skip(f"the reference needs n >= {case.min_n}")
    got = case.run(ours, RC.Dev(), n)
    exp = case.run(ref, RC.Dev(), n)
    _cmp(got, exp, f"{name} n={n}")
    golden = json.load(open(GOLDEN)).get("kernels", {}).get(f"{name}@{n}")
    if golden is not None:
        assert {k: RC.sha(v) for k, v in exp.items()} == golden, "reference output differs from the recorded one"


def _ref_ntt_tables(O, log_n, inverse):
    """The reference host's table set (src/cuda/ntt.rs:15-59): omegas built by
    the library's expand_omega_buffer (bit-reversed half table at 2^22 and
    2^24), and the pq radix table of 2^(max_deg - 1) entries."""
    n = 1 << log_n
    w = O.omega(log_n)
    if inverse:
        w = pow(w, -1, O.R_MOD)
    max_deg = min(8, log_n)
    tw = pow(w, n >> max_deg, O.R_MOD)
    pq = O.fr_vec([pow(tw, i, O.R_MOD) for i in range((1 << max_deg) >> 1)])
    return w, pq


def _ntt(L, O, data, log_n, inverse):
    """The reference host's ntt_raw sequence through library L on a device copy
    of `data`; returns the device tensor holding the result."""
    n = 1 << log_n
    w, pq = _ref_ntt_tables(O, log_n, inverse)
    om = torch.zeros((n, 4), dtype=torch.int64, device="cuda")
    om[:2] = RC.Dev().put(O.fr_vec([1, w]))
    torch.cuda.synchronize()
    assert L.expand_omega_buffer(om.data_ptr(), log_n, 1) == 0
    buf = data.clone()
    tmp = torch.empty_like(buf)
    ninv = RC.Dev().put(O.fr(pow(n, -1, O.R_MOD)))
    pqd = RC.Dev().put(pq)
    swap = ctypes.c_bool(False)
    assert L.ntt(buf.data_ptr(), tmp.data_ptr(), pqd.data_ptr(), om.data_ptr(), ninv.data_ptr() if inverse else 0,
                 log_n, 8, ctypes.addressof(swap), 0) == 0
    torch.cuda.synchronize()
    del om, pqd, ninv
    return tmp if swap.value else buf


@pytest.mark.parametrize("log_n", list(range(13, 26)))
def test_dropin_ntt_every_default_plan(O, libs, log_n):
    ours, ref = libs
    n = 1 << log_n
    a = O.rand_fr(n, 31000 + log_n)
    dev = RC.Dev().put(a)
    for inverse in (False, True):
        got = _ntt(ours, O, dev, log_n, inverse)
        exp = _ntt(ref, O, dev, log_n, inverse)
        assert torch.equal(got, exp), f"2^{log_n} inverse={inverse} differs from the reference kernels"
        if log_n <= 24:
            host = got.cpu().numpy().view(np.uint64)
            want = O.intt(a, log_n) if inverse else O.ntt(a, log_n)
            assert (host == want).all(), f"2^{log_n} inverse={inverse} differs from the oracle DFT"
        del got, exp


def _ref_msm_batch(L, bases_dev, scalar_devs, n):
    """src/cuda/msm.rs:239-455 with the reference host's sizing through library
    L: msm per column, then batch_msm_collect; Jacobian results (count, 12)."""
    count = len(scalar_devs)
    threads, bits = 64, 254
    c = min((count - 1).bit_length(), 3) + 10 + max((n - 1).bit_length(), 22) - 22
    windows = (bits + c - 1) // c
    bucket = windows << c
    worker = (n + threads - 1) // threads * threads if n < 128 * 512 else 128 * 512
    region = bucket + 2 * worker
    curve = torch.empty((count * region, 12), dtype=torch.int64, device="cuda")
    single = n * windows
    idx = [torch.empty(single, dtype=torch.int32, device="cuda") for _ in range(4)]
    sort = torch.empty(3 * single, dtype=torch.int32, device="cuda")
    acc = [torch.empty(2 * worker, dtype=torch.int32, device="cuda") for _ in range(count)]
    base = curve.data_ptr()
    for i, s in enumerate(scalar_devs):
        assert L.msm(base + i * region * 96, bases_dev.data_ptr(), s.data_ptr(), idx[0].data_ptr(),
                     idx[1].data_ptr(), idx[2].data_ptr(), idx[3].data_ptr(), sort.data_ptr(), acc[i].data_ptr(), n,
                     windows, c, threads, worker, 3 * single * 4, 1, 0) == 0
    torch.cuda.synchronize()
    dp = lambda xs: torch.tensor(xs, dtype=torch.int64, device="cuda")  # noqa: E731
    ri = dp([a.data_ptr() for a in acc])
    nri = dp([a.data_ptr() + worker * 4 for a in acc])
    ra = dp([base + (i * region + bucket) * 96 for i in range(count)])
    nra = dp([base + (i * region + bucket + worker) * 96 for i in range(count)])
    bk = dp([base + i * region * 96 for i in range(count)])
    assert L.batch_msm_collect(ri.data_ptr(), ra.data_ptr(), nri.data_ptr(), nra.data_ptr(), bk.data_ptr(), worker,
                               windows, c, count, 0) == 0
    torch.cuda.synchronize()
    out = torch.stack([curve[i * region] for i in range(count)]).cpu().numpy().view(np.uint64)
    assert c == 13 or count < 8
    return out


def test_dropin_msm_8x2p22_reference_sizing(O, libs, gpu):
    ours, ref = libs
    H = gpu.host
    n, count = 1 << 22, 8
    d = O.rand_fr(n, 5151)
    bases = H.to_device(O.g1_gen_bases(d))
    scal = [O.rand_fr(n, 7700 + i) for i in range(count)]
    sdev = [H.to_device(s) for s in scal]
    b = H.ReferenceMsmBatch(bases, sdev, n)
    assert b.c == 13
    b.enqueue()
    got = b.results()
    exp_ref = _ref_msm_batch(ref, bases, sdev, n)
    for i in range(count):
        want = O.msm_known_dlog(d, scal[i])
        assert (O.g1_jac_to_aff(got[i].reshape(1, 12)) == want).all(), f"column {i} vs known dlog"
        assert (O.g1_jac_to_aff(exp_ref[i].reshape(1, 12)) == want).all(), f"reference column {i}"


def test_coset_extension_2p22_to_2p25(O, libs, gpu):
    """zkp_extend_batch (one column, shift zeta) against the reference host's
    sequence: ntt_raw (iNTT 2^22) -> extended_prepare(zeta coset, zero pad) ->
    ntt_raw at 2^25 (src/eval_h.rs:255-265, 324-337)."""
    ours, ref = libs
    H = gpu.host
    log_n, e = 22, 3
    n, N = 1 << log_n, 1 << (log_n + e)
    lag = O.rand_fr(n, 9090)
    lag_dev = RC.Dev().put(lag)
    # reference sequence
    coeff_ref = _ntt(ref, O, lag_dev, log_n, True)
    big = torch.zeros((N, 4), dtype=torch.int64, device="cuda")
    big[:n].copy_(coeff_ref)
    del coeff_ref
    zeta = RC.ZETA
    cp = RC.Dev().put(O.fr_vec([zeta, pow(zeta, -1, O.R_MOD)]))
    assert ref.extended_prepare(big.data_ptr(), cp.data_ptr(), 3, n, N, 0, 0) == 0
    torch.cuda.synchronize()
    ext_ref = _ntt(ref, O, big, log_n + e, False)
    del big
    # this library's fused phase
    tw_inv = H.generate_omega_buffers(O.fr(pow(O.omega(log_n), -1, O.R_MOD)), log_n)
    tw = H.generate_omega_buffers(O.fr(O.omega(log_n)), log_n)
    n_inv = H.to_device(O.fr(pow(n, -1, O.R_MOD)))
    twist = H.twist_tables(O.fr(zeta), O.fr(O.omega(log_n + e)), log_n, e, tw)
    ext = H.empty_fr(N)
    coeff = H.empty_fr(n)
    scratch = H.empty_fr(N)
    H.extend_batch(ext, coeff, lag_dev, 1, log_n, e, tw_inv, n_inv, tw, twist, scratch)
    torch.cuda.synchronize()
    assert (coeff.cpu().numpy().view(np.uint64) == O.intt(lag, log_n)).all()
    assert torch.equal(ext, ext_ref), "extended column differs from the reference sequence"
    del scratch, twist
    tables = H.extend_tables(tw, tw_inv, n_inv, O.fr(zeta), O.fr(O.omega(log_n + e)), log_n, e)
    ext.zero_()
    H.extend_batch_tables(ext, coeff, lag_dev, 1, log_n, e, tables, H.empty_fr(N))
    torch.cuda.synchronize()
    assert torch.equal(ext, ext_ref), "extended column over the pair tables differs"
