"""Device scans against the oracle: batch inversion, grand products / sums,
the logup z (eval_logup_z_compose / _pure, logup_sum_input_inv as the
reference's host calls them, src/lib.rs:589-744) and the permutation and
shuffle grand products that the reference computes on the CPU
(src/permutation.rs:16-150, src/shuffle.rs:143-212)."""
import ctypes

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


# (1 << 22) + 5: 2049 block products, so the three-phase form recurses twice
@pytest.mark.parametrize("n", [1, 5, 2048, 2049, 100000, 1 << 20, (1 << 22) + 5])
@pytest.mark.parametrize("with_scratch", [False, True])
def test_batch_inverse(O, gpu, n, with_scratch):
    H = gpu.host
    a = O.rand_fr(n, 100 + n)
    if n > 10:
        a[7] = 0
        a[n - 1] = 0
    c = O.rand_fr(1, 3)
    out = H.empty_fr(n)
    scratch = H.scan_scratch(n) if with_scratch else None
    H.batch_inverse(out, H.to_device(a), H.to_device(c), scratch=scratch)
    torch.cuda.synchronize()
    exp = O.inv(O.add(a, c))
    assert (H.to_host(out) == exp).all()
    # plain inverse with zero -> zero, in place
    d = H.to_device(a)
    H.batch_inverse(d, d, scratch=scratch)
    torch.cuda.synchronize()
    assert (H.to_host(d) == O.batch_inv(a)).all()


# 2049 and 4097: a last tile of one element; (1 << 22) + 3: 2049 tiles, so the
# look-back windows of 32 tiles wrap many times
@pytest.mark.parametrize("n", [1, 7, 2048, 2049, 4097, 300000, 1 << 22, (1 << 22) + 3])
def test_grand_product_and_sum(O, gpu, n):
    H = gpu.host
    a = O.rand_fr(n, 200 + n)
    init = O.rand_fr(1, 9)
    out = H.empty_fr(n)
    H.grand_product(out, H.to_device(a), H.to_device(init))
    torch.cuda.synchronize()
    assert (H.to_host(out) == O.prefix_product_excl(a, init)).all()
    H.grand_sum(out, H.to_device(a), None)
    torch.cuda.synchronize()
    assert (H.to_host(out) == O.prefix_sum_excl(a)).all()
    # in place, with an initial value, and no look-back wait ran out
    d = H.to_device(a)
    H.grand_sum(d, d, H.to_device(init))
    torch.cuda.synchronize()
    assert (H.to_host(d) == O.prefix_sum_excl(a, init)).all()
    assert gpu.load_library().zkp_scan_timeouts() == 0


def test_logup_reference_abi(O, gpu):
    """logup_sum_input_inv over two inputs, then eval_logup_z_compose for the
    first set and eval_logup_z_pure for a second set, chained through last_z."""
    H = gpu.host
    L = gpu.load_library()
    n = 1 << 16
    u = n - 17
    beta = O.rand_fr(1, 11)
    bint = O.fr_ints(beta)[0]
    inp0, inp1 = O.rand_fr(n, 12), O.rand_fr(n, 13)
    table = O.rand_fr(n, 14)
    m = O.fr_vec([i % 5 for i in range(n)])
    d_beta = H.to_device(beta)
    s = H.zeros_fr(n)
    tmp = H.empty_fr(n)
    st = H.stream_handle()
    d0, d1 = H.to_device(inp0), H.to_device(inp1)
    gpu.abi.check(L.logup_sum_input_inv(s.data_ptr(), d0.data_ptr(), tmp.data_ptr(), d_beta.data_ptr(), 0, n, st))
    gpu.abi.check(L.logup_sum_input_inv(s.data_ptr(), d1.data_ptr(), tmp.data_ptr(), d_beta.data_ptr(), 1, n, st))
    torch.cuda.synchronize()
    exp_sum = O.logup_sum_input_inv(O.logup_sum_input_inv(None, inp0, bint, 0), inp1, bint, 1)
    assert (H.to_host(s) == exp_sum).all()
    z = H.empty_fr(n)
    last = H.zeros_fr(1)
    dt, dm = H.to_device(table), H.to_device(m)
    gpu.abi.check(L.eval_logup_z_compose(z.data_ptr(), s.data_ptr(), dt.data_ptr(), dm.data_ptr(),
                                         d_beta.data_ptr(), last.data_ptr(), u, n, st))
    torch.cuda.synchronize()
    exp_z, exp_last = O.eval_logup_z_compose(exp_sum, table, m, bint, u)
    assert (H.to_host(z) == exp_z).all()
    assert (H.to_host(last) == exp_last).all()
    # second set: z2 = last_z + prefix sum of its input sums
    z2 = H.to_device(exp_sum)
    gpu.abi.check(L.eval_logup_z_pure(z2.data_ptr(), s.data_ptr(), dt.data_ptr(), last.data_ptr(), u, n, st))
    torch.cuda.synchronize()
    exp_z2, exp_last2 = O.eval_logup_z_pure(exp_sum, u, exp_last)
    assert (H.to_host(z2) == exp_z2).all()
    assert (H.to_host(last) == exp_last2).all()


def test_permutation_z_device(O, gpu):
    H = gpu.host
    L = gpu.load_library()
    log_n, ncols, chunk, u = 12, 5, 2, (1 << 12) - 10
    n = 1 << log_n
    cols = [O.rand_fr(n, 300 + i) for i in range(ncols)]
    sigs = [O.rand_fr(n, 400 + i) for i in range(ncols)]
    beta, gamma = 987654321, 123456789
    exp = O.permutation_product(cols, sigs, beta, gamma, log_n, chunk, u)
    omegas = H.generate_omega_buffers(O.fr(O.omega(log_n)), log_n)
    dcols = [H.to_device(c) for c in cols]
    dsigs = [H.to_device(s) for s in sigs]
    db, dg = H.to_device(O.fr(beta)), H.to_device(O.fr(gamma))
    dlt = O.delta()
    scratch = H.scan_scratch(n)
    zs = []
    init = H.to_device(O.fr(1))
    st = H.stream_handle()
    for k, c0 in enumerate(range(0, ncols, chunk)):
        cc = dcols[c0:c0 + chunk]
        ss = dsigs[c0:c0 + chunk]
        dbeta = H.to_device(O.fr_vec([beta * pow(dlt, c0 + j, O.R_MOD) % O.R_MOD for j in range(len(cc))]))
        pc, ps = H.ptr_array(cc), H.ptr_array(ss)
        z = H.empty_fr(n)
        gpu.abi.check(L.zkp_permutation_z(z.data_ptr(), pc.data_ptr(), ps.data_ptr(), len(cc), db.data_ptr(),
                                          dg.data_ptr(), dbeta.data_ptr(), omegas.data_ptr(), init.data_ptr(), n,
                                          scratch.data_ptr(), st))
        torch.cuda.synchronize()
        zs.append(z)
        init = z[u:u + 1].clone()
    for z, e in zip(zs, exp):
        assert (H.to_host(z) == e).all()


def test_shuffle_z_device(O, gpu):
    H = gpu.host
    L = gpu.load_library()
    n = 1 << 13
    ins = [O.rand_fr(n, 500 + i) for i in range(3)]
    tabs = [O.rand_fr(n, 600 + i) for i in range(3)]
    beta = 55555
    exp = O.shuffle_product(ins, tabs, beta)
    di, dt = [H.to_device(x) for x in ins], [H.to_device(x) for x in tabs]
    betas = H.to_device(O.fr_vec([pow(beta, g + 1, O.R_MOD) for g in range(3)]))
    pi, pt = H.ptr_array(di), H.ptr_array(dt)
    z = H.empty_fr(n)
    scratch = H.empty_fr(n + gpu.load_library().zkp_scan_scratch_elems(n))
    gpu.abi.check(L.zkp_shuffle_z(z.data_ptr(), pi.data_ptr(), pt.data_ptr(), betas.data_ptr(), 3, n,
                                  scratch.data_ptr(), H.stream_handle()))
    torch.cuda.synchronize()
    assert (H.to_host(z) == exp).all()
