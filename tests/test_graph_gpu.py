"""CUDA-graph capture of the batched phases: each entry point is captured
once and replayed (no host work, no host memory read at replay), and the
replayed results equal the oracle's."""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _jac_to_aff(O, j):
    return O.g1_jac_to_aff(np.asarray(j, np.uint64).reshape(-1, 12))


def _capture(fn):
    fn()  # warm-up outside capture (one-time function attributes)
    torch.cuda.synchronize()
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g):
        fn()
    return g


def test_graph_msm_batch(O, gpu):
    H = gpu.host
    nmax = 1 << 12
    d = O.rand_fr(nmax, 501)
    bases = H.to_device(O.g1_gen_bases(d))
    ns = [nmax, 1000, 1, 4096, 77] * 20  # 100 MSMs: two descriptor launches
    cols = [O.rand_fr(n, 600 + i) for i, n in enumerate(ns)]
    dev = [H.to_device(c) for c in cols]
    out = torch.empty((len(ns), 12), dtype=torch.int64, device="cuda")
    ws = [0] * len(ns)
    import ctypes
    n_arr = (ctypes.c_uint32 * len(ns))(*ns)
    scratch = torch.empty(gpu.load_library().zkp_msm_batch_scratch_bytes(ctypes.addressof(n_arr), None, len(ns)),
                          dtype=torch.uint8, device="cuda")
    ptrs = H.ptr_array(dev)
    g = _capture(lambda: H.msm_batch(bases, dev, ns, ws, scratch=scratch, out=out, ptrs=ptrs))
    out.zero_()
    g.replay()
    torch.cuda.synchronize()
    got = _jac_to_aff(O, H.to_host(out))
    for i in (0, 1, 2, 3, 4, 57, 99):
        assert (got[i] == O.msm_known_dlog(d[:ns[i]], cols[i])).all(), i
    # new scalars in the same buffers: the replay reads them
    for i in (0, 3):
        cols[i] = O.rand_fr(ns[i], 700 + i)
        dev[i].copy_(H.to_device(cols[i]))
    g.replay()
    torch.cuda.synchronize()
    got = _jac_to_aff(O, H.to_host(out))
    for i in (0, 3):
        assert (got[i] == O.msm_known_dlog(d[:ns[i]], cols[i])).all(), i


def test_graph_msm_and_table(O, gpu):
    H = gpu.host
    n = 3000
    d = O.rand_fr(n, 511)
    bases = H.to_device(O.g1_gen_bases(d))
    s = O.rand_fr(n, 512)
    sd = H.to_device(s)
    table, c = H.msm_table_build(bases, n, 0)
    scr1 = H.msm_scratch(n)
    scr2 = torch.empty(gpu.load_library().zkp_msm_table_scratch_bytes(n, c), dtype=torch.uint8, device="cuda")
    o1 = torch.empty(12, dtype=torch.int64, device="cuda")
    o2 = torch.empty(12, dtype=torch.int64, device="cuda")

    def both():
        H.msm(bases, sd, n=n, scratch=scr1, out=o1)
        H.msm_table(table, n, c, sd, n=n, scratch=scr2, out=o2)

    g = _capture(both)
    o1.zero_()
    o2.zero_()
    g.replay()
    torch.cuda.synchronize()
    exp = O.msm_known_dlog(d, s)
    assert (_jac_to_aff(O, H.to_host(o1)) == exp).all()
    assert (_jac_to_aff(O, H.to_host(o2)) == exp).all()


def _omega_mont(O, log_n, inverse=False):
    w = O.omega(log_n)
    return O.fr(pow(w, -1, O.R_MOD) if inverse else w)


def test_graph_extend_phase(O, gpu):
    # a two-chunk extend phase (fused stage) over pair tables, as one graph
    H = gpu.host
    log_n, ext_bits, ncols, chunk = 18, 3, 4, 2
    n, E = 1 << log_n, 1 << ext_bits
    shift = 7
    lag = O.rand_fr(n * ncols, 521)
    tw_inv = H.generate_omega_buffers(_omega_mont(O, log_n, True), log_n)
    tw = H.generate_omega_buffers(_omega_mont(O, log_n), log_n)
    n_inv = H.to_device(O.fr(pow(n, -1, O.R_MOD)))
    tables = H.extend_tables(tw, tw_inv, n_inv, O.fr(shift), O.fr(O.omega(log_n + ext_bits)), log_n, ext_bits)
    lag_d = H.to_device(lag)
    ext = H.empty_fr(ncols * E * n)
    coeff = H.empty_fr(ncols * n)
    scratch = H.empty_fr(chunk * E * n)

    def phase():
        for c0 in range(0, ncols, chunk):
            H.extend_batch_tables(ext[c0 * E * n:], coeff[c0 * n:], lag_d[c0 * n:], chunk, log_n, ext_bits, tables,
                                  scratch)

    g = _capture(phase)
    ext.zero_()
    g.replay()
    torch.cuda.synchronize()
    ge = H.to_host(ext)
    for c in (0, 3):
        co = O.intt(lag[c * n:(c + 1) * n], log_n)
        assert (ge[c * E * n:(c + 1) * E * n] == O.coset_ntt(co, log_n, log_n + ext_bits, shift)).all()
