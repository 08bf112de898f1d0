"""NTT parity on the GPU through the C ABI (ntt / expand_omega_buffer /
extended_prepare as the reference's host calls them, src/cuda/ntt.rs), and the
batched zkp_* transforms, against the oracle DFT bit for bit."""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _omega_mont(O, log_n, inverse=False):
    w = O.omega(log_n)
    if inverse:
        w = pow(w, -1, O.R_MOD)
    return O.fr(w)


@pytest.mark.parametrize("log_n", [1, 2, 3, 4, 5, 6, 7, 9, 10, 11, 12, 13, 15, 17, 20])
def test_ntt_forward_and_inverse(O, gpu, log_n):
    H = gpu.host
    n = 1 << log_n
    a = O.rand_fr(n, 1000 + log_n)
    omegas, pq = H.generate_ntt_buffers(_omega_mont(O, log_n), log_n)
    iomegas, ipq = H.generate_ntt_buffers(_omega_mont(O, log_n, True), log_n)
    div = H.to_device(O.fr(pow(n, -1, O.R_MOD)))
    s = H.to_device(a)
    t = H.empty_fr(n)
    s, t = H.ntt_raw(s, t, pq, omegas, log_n)
    torch.cuda.synchronize()
    assert (H.to_host(s) == O.ntt(a, log_n)).all()
    s, t = H.ntt_raw(s, t, ipq, iomegas, log_n, intt_divisor=div)
    torch.cuda.synchronize()
    assert (H.to_host(s) == a).all()


def test_ntt_reference_test_input(O, gpu):
    # src/profile.rs:198-205: s_0 random, s_i = s_{i-1} + i, k = 22 in the reference
    H = gpu.host
    log_n = 16
    s0 = O.fr_ints(O.rand_fr(1, 77))[0]
    xs = [s0]
    for i in range(1, 1 << log_n):
        xs.append((xs[-1] + i) % O.R_MOD)
    a = O.fr_vec(xs)
    omegas, pq = H.generate_ntt_buffers(_omega_mont(O, log_n), log_n)
    s, t = H.ntt_raw(H.to_device(a), H.empty_fr(1 << log_n), pq, omegas, log_n)
    torch.cuda.synchronize()
    assert (H.to_host(s) == O.ntt(a, log_n)).all()


def test_expand_omega_buffer_natural(O, gpu):
    H = gpu.host
    # 2^13: every entry (two coarse threads of 64 runs of 64)
    buf = H.generate_omega_buffers(_omega_mont(O, 13), 13, True)
    assert (H.to_host(buf) == O.expand_omega(O.omega(13), 13)).all()
    for log_n in (1, 2, 5, 6, 7, 11, 12, 22):
        buf = H.generate_omega_buffers(_omega_mont(O, log_n), log_n, True)
        got = H.to_host(buf)
        n = 1 << log_n
        # spot check against w^i, run and coarse-thread boundaries included
        idx = sorted({i for i in (0, 1, 2, 3, 63, 64, 65, 4095, 4096, 4097, n // 2, n - 1) if i < n}
                     | set(np.random.default_rng(1).integers(0, n, 50).tolist()))
        w = O.omega(log_n)
        for i in idx:
            assert O.fr_ints(got[i])[0] == pow(w, i, O.R_MOD)


def test_extended_prepare(O, gpu):
    H = gpu.host
    n, N = 1 << 10, 1 << 13
    z = O.cube_roots_of_unity()[1]
    cp = O.fr_vec([z, pow(z, 2, O.R_MOD)])
    s = np.concatenate([O.rand_fr(n, 3), O.rand_fr(N - n, 4)])
    d = H.to_device(s)
    H.extended_prepare(d, H.to_device(cp), 3, n, N, False)
    torch.cuda.synchronize()
    assert (H.to_host(d) == O.extended_prepare(s, cp, 3, n, N, False)).all()
    H.extended_prepare(d, H.to_device(cp), 3, n, N, True)
    torch.cuda.synchronize()
    exp = O.extended_prepare(O.extended_prepare(s, cp, 3, n, N, False), cp, 3, n, N, True)
    assert (H.to_host(d) == exp).all()


@pytest.mark.parametrize("log_n,ncols", [(6, 5), (12, 3), (14, 4), (18, 2)])
def test_ntt_batch_columns(O, gpu, log_n, ncols):
    H = gpu.host
    n = 1 << log_n
    a = O.rand_fr(n * ncols, 500 + log_n)
    omegas = H.generate_omega_buffers(_omega_mont(O, log_n), log_n)
    buf = H.to_device(a)
    tmp = H.empty_fr(n * ncols)
    out = H.ntt_batch(buf, tmp, omegas, log_n, ncols)
    torch.cuda.synchronize()
    got = H.to_host(out)
    for c in range(ncols):
        assert (got[c * n:(c + 1) * n] == O.ntt(a[c * n:(c + 1) * n], log_n)).all()


# fused stage radices: 2^18 -> 2^9, 2^19 -> 2^9, 2^20 and 2^21 -> 2^10, 2^22 -> 2^11
@pytest.mark.parametrize("pairs", [False, True])
@pytest.mark.parametrize("log_n,ext_bits,ncols", [(4, 3, 2), (10, 3, 3), (13, 3, 2), (16, 2, 2),
                                                  (18, 3, 2), (19, 2, 1), (20, 3, 1), (22, 1, 1)])
def test_extend_batch_matches_coset_ntt(O, gpu, log_n, ext_bits, ncols, pairs):
    # pairs: the same phase over (w, w') tables and products by known factors
    H = gpu.host
    n = 1 << log_n
    shift = 7  # the field's multiplicative generator
    lag = O.rand_fr(n * ncols, 900 + log_n)
    tw_inv = H.generate_omega_buffers(_omega_mont(O, log_n, True), log_n)
    tw = H.generate_omega_buffers(_omega_mont(O, log_n), log_n)
    n_inv = H.to_device(O.fr(pow(n, -1, O.R_MOD)))
    twist = H.twist_tables(O.fr(shift), O.fr(O.omega(log_n + ext_bits)), log_n, ext_bits, tw)
    E = 1 << ext_bits
    ext = H.empty_fr(ncols * E * n)
    coeff = H.empty_fr(ncols * n)
    scratch = H.empty_fr(ncols * E * n)
    if pairs:
        tables = H.extend_tables(tw, tw_inv, n_inv, O.fr(shift), O.fr(O.omega(log_n + ext_bits)), log_n, ext_bits)
        H.extend_batch_tables(ext, coeff, H.to_device(lag), ncols, log_n, ext_bits, tables, scratch)
    else:
        H.extend_batch(ext, coeff, H.to_device(lag), ncols, log_n, ext_bits, tw_inv, n_inv, tw, twist, scratch)
    torch.cuda.synchronize()
    ge, gc = H.to_host(ext), H.to_host(coeff)
    for c in range(ncols):
        co = O.intt(lag[c * n:(c + 1) * n], log_n)
        assert (gc[c * n:(c + 1) * n] == co).all()
        assert (ge[c * E * n:(c + 1) * E * n] == O.coset_ntt(co, log_n, log_n + ext_bits, shift)).all()


@pytest.mark.parametrize("n", [1, 2, 63, 64, 65, 4097, 5000, 70000])
def test_powers(O, gpu, n):
    # zkp_powers: out[i] = base * w^i for every i < n
    H = gpu.host
    base, w = 0x1234567 * 7 % O.R_MOD, O.omega(20)
    out = H.empty_fr(n)
    b_dev, w_dev = H.to_device(O.fr(base)), H.to_device(O.fr(w))
    gpu.abi.check(gpu.load_library().zkp_powers(out.data_ptr(), b_dev.data_ptr(), w_dev.data_ptr(), n,
                                                H.stream_handle()))
    torch.cuda.synchronize()
    got = O.fr_ints(H.to_host(out))
    exp, v = [], base
    for _ in range(n):
        exp.append(v)
        v = v * w % O.R_MOD
    assert got == exp


def test_ntt_every_pass_split_same_result(O, gpu):
    # every split the radix autotuner may pick gives the same transform
    H, S = gpu.host, gpu.schedule
    log_n, ncols = 16, 2
    n = 1 << log_n
    a = O.rand_fr(n * ncols, 1401)
    om = H.generate_omega_buffers(_omega_mont(O, log_n), log_n, False)
    exp = np.concatenate([O.ntt(a[c * n:(c + 1) * n], log_n) for c in range(ncols)])
    splits = S.ntt_splits(log_n)
    assert [10, 6] in splits and [6, 10] in splits and H.ntt_default_plan(log_n) in splits
    for split in splits:
        buf, tmp = H.to_device(a), H.empty_fr(n * ncols)
        out = H.ntt_batch_plan(buf, tmp, om, log_n, ncols, split)
        torch.cuda.synchronize()
        assert (H.to_host(out) == exp).all(), split


def test_ntt_plan_rejects_bad_splits(gpu):
    H = gpu.host
    buf, tmp = H.empty_fr(1 << 16), H.empty_fr(1 << 16)
    om = H.empty_fr(1 << 16)
    for bad in ([10, 5], [13, 3], [8, 8, 1], [9, 9]):
        with pytest.raises(gpu.abi.CudaError):
            H.ntt_batch_plan(buf, tmp, om, 16, 1, bad)


def test_autotune_ntt_picks_a_split(gpu):
    best, times = gpu.schedule.autotune_ntt(14, ncols=4, reps=1)
    assert tuple(best) in times and sum(best) == 14 and len(times) == len(gpu.schedule.ntt_splits(14))
