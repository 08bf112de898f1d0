"""The per-coset quotient and multi-open entry points against the oracle, bit
for bit: zkp_eval_h_fused (every constraint family, rotations of both signs),
zkp_ntt_batch_twisted + zkp_coset_combine (against the reference host's
field_mul_zip -> iNTT of 2^(k+e) -> extended_prepare(to_coset) sequence,
restated by the oracle), zkp_poly_divide_linear (against the reference's own
host recurrence, src/multiopen.rs:145-159) and zkp_poly_eval_batch."""
import ctypes
import importlib

import numpy as np
import pytest
import torch

import ref_cases as RC

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def P(gpu):
    return importlib.import_module("zkwasm-prover_b200.prover")


def _h(t):
    torch.cuda.synchronize()
    return t.detach().cpu().contiguous().numpy().view(np.uint64).reshape(-1, 4)


@pytest.mark.parametrize("log_n", [4, 12, 20])
def test_poly_divide_linear(O, gpu, P, log_n):
    L = gpu.load_library()
    n = 1 << log_n
    a = O.rand_fr(n, 70 + log_n)
    ad = RC.Dev().put(a)
    for z in (O.fr_ints(O.rand_fr(1, 71))[0], 0, 1, O.R_MOD - 1):
        q = torch.empty_like(ad)
        scratch = torch.empty((L.zkp_poly_divide_scratch_elems(n), 4), dtype=torch.int64, device="cuda")
        zh = np.array(P.limbs(z), dtype=np.uint64)
        assert L.zkp_poly_divide_linear(q.data_ptr(), ad.data_ptr(), zh.ctypes.data, n, scratch.data_ptr(), 0) == 0
        assert (_h(q) == O.poly_divide_linear(a, z)).all(), f"z={z}"


def test_poly_eval_batch(O, gpu, P):
    L = gpu.load_library()
    for log_n in (1, 10, 16):
        n = 1 << log_n
        polys = [O.rand_fr(n, 80 + i) for i in range(5)]
        x = O.fr_ints(O.rand_fr(1, 81))[0]
        d = RC.Dev()
        dp = d.ptrs([d.put(p) for p in polys])
        pw = P.powers(1, x, n)
        out = torch.empty((5, 4), dtype=torch.int64, device="cuda")
        scratch = torch.empty((L.zkp_poly_eval_batch_scratch_elems(5), 4), dtype=torch.int64, device="cuda")
        assert L.zkp_poly_eval_batch(out.data_ptr(), dp.data_ptr(), 5, pw.data_ptr(), n, scratch.data_ptr(), 0) == 0
        assert O.fr_ints(_h(out)) == [O.poly_eval(p, x) for p in polys]


@pytest.mark.parametrize("ext_bits", [1, 2, 3])
@pytest.mark.parametrize("pairs", [False, True])
def test_cosets_and_combine(O, gpu, P, ext_bits, pairs):
    """Coset values from coefficients (zkp_ntt_batch_twisted) and back
    (zkp_coset_combine) against the oracle's whole-domain restatement."""
    L = gpu.load_library()
    k = 12
    n, E = 1 << k, 1 << ext_bits
    N = n * E
    coeff = O.rand_fr(n, 90 + ext_bits)
    # forward: coset j of the zeta-coset extension of the coefficients
    ext = O.coset_ntt(coeff, k, k + ext_bits, RC.ZETA)
    tab = P.Tables(k)
    wN = O.omega(k + ext_bits)
    src = RC.Dev().put(coeff)
    tmp = torch.empty((n, 4), dtype=torch.int64, device="cuda")
    if pairs:
        twp = torch.empty((2 * n, 4), dtype=torch.int64, device="cuda")
        assert L.zkp_shoup_pairs(twp.data_ptr(), tab.tw.data_ptr(), n, 0) == 0
    for j in range(E):
        sj = RC.ZETA * pow(wN, j, O.R_MOD) % O.R_MOD
        twist = P.powers(1, sj, n)
        out = torch.empty((n, 4), dtype=torch.int64, device="cuda")
        if pairs:
            tp = torch.empty((2 * n, 4), dtype=torch.int64, device="cuda")
            assert L.zkp_shoup_pairs(tp.data_ptr(), twist.data_ptr(), n, 0) == 0
            assert L.zkp_ntt_batch_twisted(out.data_ptr(), src.data_ptr(), tmp.data_ptr(), twp.data_ptr(),
                                           tp.data_ptr(), 0, k, 1, n, n, 1, 0) == 0
        else:
            assert L.zkp_ntt_batch_twisted(out.data_ptr(), src.data_ptr(), tmp.data_ptr(), tab.tw.data_ptr(),
                                           twist.data_ptr(), 0, k, 1, n, n, 0, 0) == 0
        assert (_h(out) == ext[j::E]).all(), f"coset {j}"
    # backward: arbitrary values h on the extended domain, divided by Z_H per
    # coset, to coefficients with the coset undone
    hv = O.rand_fr(N, 95)
    t = [pow((pow(RC.ZETA * pow(wN, j, O.R_MOD), n, O.R_MOD) - 1) % O.R_MOD, -1, O.R_MOD) for j in range(E)]
    exp = O.field_mul_zip(hv, O.fr_vec(t))
    exp = O.intt(exp, k + ext_bits)
    exp = O.extended_prepare(exp, O.fr_vec([pow(RC.ZETA, -1, O.R_MOD), RC.ZETA]), 3, n, N, True)
    hc = RC.Dev().put(np.concatenate([O.mul(hv[j::E], O.fr_vec([t[j]])) for j in range(E)]))
    g = torch.empty_like(hc)
    tmpE = torch.empty_like(hc)
    assert L.zkp_ntt_batch_twisted(g.data_ptr(), hc.data_ptr(), tmpE.data_ptr(), tab.tw_inv.data_ptr(), 0,
                                   tab.n_inv.data_ptr(), k, E, n, n, 0, 0) == 0
    winv = P.powers(1, pow(wN, -1, O.R_MOD), n)
    wE = pow(wN, n, O.R_MOD)
    consts = P.fr_tensor([1] * E + [pow(wE, -kk, O.R_MOD) for kk in range(E)] +
                         [pow(RC.ZETA, -kk, O.R_MOD) * pow(E, -1, O.R_MOD) % O.R_MOD for kk in range(3)])
    out = torch.empty((N, 4), dtype=torch.int64, device="cuda")
    assert L.zkp_coset_combine(out.data_ptr(), g.data_ptr(), n, winv.data_ptr(), consts.data_ptr(), k, ext_bits,
                               0) == 0
    assert (_h(out) == exp).all()


def test_eval_h_fused_matches_restatement(O, gpu, P):
    """Every family of zkp_eval_h_fused on random columns (rotation scale 2,
    as on a whole extended domain of E = 2) against the oracle's restatement of
    the reference's kernels in their chain order."""
    L = gpu.load_library()
    n, rs = 1 << 10, 2
    R = O.R_MOD
    rnd = iter(range(300, 10_000))
    col = lambda: O.rand_fr(n, next(rnd))  # noqa: E731
    y, beta, gamma = [O.fr_ints(O.rand_fr(1, s))[0] for s in (1, 2, 3)]
    yv, bv, gv = O.fr_vec([y]), O.fr_vec([beta]), O.fr_vec([gamma])
    l0, ll, la, X = col(), col(), col(), col()
    d = RC.Dev()
    # gates: two terms with rotations of both signs
    gcols = [col() for _ in range(4)]
    gco = O.rand_fr(2, 9)
    terms = [(gco[0:1], [(gcols[0], 0), (gcols[1], 1)]), (gco[1:2], [(gcols[2], -1), (gcols[3], 2)])]
    v, rots = [], []
    for c_, fs in terms:
        v.append(d.put(c_))
        for cc, r in fs:
            v.append(d.put(cc))
            rots.append(r)
        v.append(None)
    # permutation: 5 columns in chunks of 2
    pc = [col() for _ in range(5)]
    ps = [col() for _ in range(5)]
    pz = [col() for _ in range(3)]
    db = [beta * pow(P.DELTA, c, R) % R for c in range(5)]
    last = -3
    # lookups and shuffles
    lk = [[col() for _ in range(4)] for _ in range(2)]
    sh = [[col() for _ in range(5)]]  # z, (in, tab) x 2
    sbetas = [pow(beta, i + 1, R) for i in range(2)]
    scale = O.rand_fr(1, 11)
    a = P._EvalHArgs()
    a.n, a.rot_scale = n, rs
    keep = [d.put(yv), d.ptrs(v), d.i32(rots), d.put(l0), d.put(ll), d.put(la), d.put(X), d.put(bv), d.put(gv),
            d.ptrs([d.put(z) for z in pz]), d.ptrs([d.put(c_) for c_ in pc]), d.ptrs([d.put(c_) for c_ in ps]),
            d.put(O.fr_vec(db)), d.ptrs([d.put(c_) for q in lk for c_ in q]),
            d.ptrs([d.put(c_) for q in sh for c_ in q]), d.i32([2]), d.put(O.fr_vec(sbetas)), d.put(scale)]
    (a.y, a.gate_terms, a.gate_rots, a.l0, a.l_last, a.l_active, a.x, a.beta, a.gamma, a.perm_z, a.perm_cols,
     a.perm_sigmas, a.perm_dbeta, a.lookup_cols, a.shuffle_cols, a.shuffle_group_len, a.shuffle_betas,
     a.scale) = [t.data_ptr() for t in keep]
    a.gate_terms_n = len(v)
    a.perm_chunks, a.perm_chunk_len, a.perm_cols_n, a.perm_last_rot = 3, 2, 5, last
    a.lookups, a.shuffles = 2, 1
    h = torch.empty((n, 4), dtype=torch.int64, device="cuda")
    assert L.zkp_eval_h_fused(h.data_ptr(), ctypes.byref(a), 0) == 0
    # restatement in the chain order of src/eval_h.rs (rotations scaled by rs)
    sc_terms = [(c_, [(cc, r * rs) for cc, r in fs]) for c_, fs in terms]
    t = O.field_op_batch_mul_sum(O.zeros(n), sc_terms, n)
    t = O.permutation_eval_h_p1(t, pz[0], pz[-1], l0, ll, yv)
    t = O.permutation_eval_h_p2(t, pz, l0, ll, yv, last * rs)
    for j in range(3):
        Lp, Rp = O._rot(pz[j], rs), pz[j]
        for c in range(2 * j, min(5, 2 * j + 2)):
            Lp = O.mul(Lp, O.add(O.add(pc[c], O.mul(ps[c], bv)), gv))
            Rp = O.mul(Rp, O.add(O.add(pc[c], O.mul(X, O.fr_vec([db[c]]))), gv))
        t = O.add(O.mul(t, yv), O.mul(la, O.sub(Lp, Rp)))
    for q in lk:
        fb, tb = O.add(q[0], bv), O.add(q[1], bv)
        t = O.logup_eval_h(t, fb, O.one(n), tb, q[2], q[3], q[3], l0, ll, la, yv, rs)
    for q in sh:
        t = O.shuffle_eval_h_v2(t, [q[1], q[3]], [q[2], q[4]], O.fr_vec(sbetas), q[0], l0, ll, la, yv, rs)
    t = O.mul(t, scale)
    assert (_h(h) == t).all()
