"""The benchmark's own sizes, checked against the oracle: the 64-column phase
(2^20 Lagrange columns -> iNTT -> coset NTT on 2^23, shift 7) and single MSMs
of 2^22 points, plain and over a base table.

The phase is run as the benchmark runs it (chunks of 8 columns over the (w, w')
multiplier tables); every column's coefficient form is compared with the
oracle's inverse DFT, and the whole extended output of the first column of the
first chunk and the last column of the last chunk with the oracle's coset DFT.
The MSMs use the reference's known-discrete-log identity
(src/cuda/msm.rs:501-512): with bases P_i = [d_i]G, sum_i [s_i] P_i equals
[sum_i s_i d_i] G, which the oracle evaluates in O(n) at any size."""
import ctypes

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _omega_mont(O, log_n, inverse=False):
    w = O.omega(log_n)
    return O.fr(pow(w, -1, O.R_MOD) if inverse else w)


def test_extend_phase_64_columns_2p20_to_2p23(O, gpu):
    H = gpu.host
    log_n, ext_bits, ncols, chunk, shift = 20, 3, 64, 8, 7
    n, E = 1 << log_n, 1 << ext_bits
    lag = O.rand_fr(n * ncols, 4242)
    tw_inv = H.generate_omega_buffers(_omega_mont(O, log_n, True), log_n)
    tw = H.generate_omega_buffers(_omega_mont(O, log_n), log_n)
    n_inv = H.to_device(O.fr(pow(n, -1, O.R_MOD)))
    tables = H.extend_tables(tw, tw_inv, n_inv, O.fr(shift), O.fr(O.omega(log_n + ext_bits)), log_n, ext_bits)
    ext = H.empty_fr(chunk * E * n)
    coeff = H.empty_fr(chunk * n)
    scratch = H.empty_fr(chunk * E * n)
    lag_dev = H.to_device(lag)
    checked_ext = 0
    for c0 in range(0, ncols, chunk):
        H.extend_batch_tables(ext, coeff, lag_dev[c0 * n:(c0 + chunk) * n], chunk, log_n, ext_bits, tables, scratch)
        torch.cuda.synchronize()
        gc = H.to_host(coeff)
        for c in range(chunk):
            col = c0 + c
            co = O.intt(lag[col * n:(col + 1) * n], log_n)
            assert (gc[c * n:(c + 1) * n] == co).all(), f"coefficients of column {col}"
            if col in (0, ncols - 1):
                ge = H.to_host(ext[c * E * n:(c + 1) * E * n])
                assert (ge == O.coset_ntt(co, log_n, log_n + ext_bits, shift)).all(), f"extension of column {col}"
                checked_ext += 1
    assert checked_ext == 2


@pytest.fixture(scope="module")
def msm_2p22(O):
    n = 1 << 22
    d = O.rand_fr(n, 5151)
    s = O.rand_fr(n, 5152)
    return n, O.g1_gen_bases(d), s, O.msm_known_dlog(d, s), d


def test_msm_2p22_known_dlog(O, gpu, msm_2p22):
    H = gpu.host
    n, bases, s, exp, _ = msm_2p22
    out = H.msm(H.to_device(bases), H.to_device(s), n=n)
    torch.cuda.synchronize()
    assert (O.g1_jac_to_aff(H.to_host(out).reshape(1, 12)) == exp).all()


def test_msm_table_2p22_known_dlog(O, gpu, msm_2p22):
    H = gpu.host
    n, bases, s, exp, _ = msm_2p22
    table, c = H.msm_table_build(H.to_device(bases), n)
    for _ in range(2):  # the second call runs on the first call's scratch contents
        out = H.msm_table(table, n, c, H.to_device(s), n=n)
        torch.cuda.synchronize()
        assert (O.g1_jac_to_aff(H.to_host(out).reshape(1, 12)) == exp).all()


def test_msm_batch_uneven_over_one_srs(O, gpu, msm_2p22):
    """24 MSMs over prefixes of one 2^22-point SRS, sizes 2^14..2^22 (one of
    each end), uniform, witness-like (< 2^20), sparse and mixed scalars: one
    pipeline with the library's windows, one with the learned windows, and one
    over a table of the SRS, each against the known-discrete-log identity."""
    import importlib

    H = gpu.host
    S = importlib.import_module("zkwasm-prover_b200.schedule")
    nsrs, bases, _, _, d = msm_2p22
    rng = np.random.default_rng(77)
    logs = [14, 22] + [int(x) for x in rng.integers(14, 23, 22)]
    mixes = ["uniform", "small", "sparse", "mixed"]
    ns = [1 << lg for lg in logs]
    cols = [S.scalars(n, mixes[i % 4], 600 + i) for i, n in enumerate(ns)]
    exp = [O.msm_known_dlog(d[:n], H.to_host(c)) for n, c in zip(ns, cols)]
    bases_dev = H.to_device(bases)

    def check(out):
        torch.cuda.synchronize()
        got = H.to_host(out)
        for i in range(len(ns)):
            assert (O.g1_jac_to_aff(got[i].reshape(1, 12)) == exp[i]).all(), f"MSM {i} (2^{logs[i]})"

    check(H.msm_batch(bases_dev, cols, ns))
    model = S.Model.load()
    learned = [model.pick(S.shape_features(n, len(ns), S.histogram(c))) for n, c in zip(ns, cols)]
    check(H.msm_batch(bases_dev, cols, ns, learned))
    n_arr = (ctypes.c_uint32 * len(ns))(*ns)
    c = gpu.load_library().zkp_msm_batch_table_default_window(ctypes.addressof(n_arr), len(ns))
    table, c = H.msm_table_build(bases_dev, nsrs, c)
    check(H.msm_batch_table(table, nsrs, c, cols, ns))
