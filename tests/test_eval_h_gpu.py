"""Quotient (eval_h) kernels, multi-open helpers and lookup multiplicities
through the reference-compatible C symbols, against the oracle's restatement
of cuda/bn254.cu."""
import random

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

N = 1 << 12


@pytest.fixture(scope="module")
def env(O, gpu):
    H = gpu.host
    L = gpu.load_library()

    class E:
        pass

    e = E()
    e.H, e.L, e.O = H, L, O
    e.st = H.stream_handle()
    e.keep = []

    def dev(a):
        t = H.to_device(a)
        e.keep.append(t)
        return t

    def arr(ts):
        t = H.ptr_array(ts)
        e.keep.append(t)
        return t

    e.dev, e.arr = dev, arr
    e.cols = [O.rand_fr(N, 1000 + i) for i in range(8)]
    e.y, e.beta, e.gamma = O.rand_fr(1, 1), O.rand_fr(1, 2), O.rand_fr(1, 3)
    return e


def _res(e, seed=77):
    r = e.O.rand_fr(N, seed)
    return r, e.dev(r)


def _get(e, t):
    torch.cuda.synchronize()
    return e.H.to_host(t)


def P(t):
    return 0 if t is None else t.data_ptr()


@pytest.mark.parametrize("op", [0, 1, 2, 3])
@pytest.mark.parametrize("l_rot,r_rot", [(0, 0), (1, -1), (-3, 5)])
def test_field_op(env, op, l_rot, r_rot):
    e, O = env, env.O
    l, r = e.cols[0], e.cols[1]
    lc, rc = e.cols[2][:1], e.cols[3][:1]
    for use_lc, use_rc in ((False, False), (True, False), (False, True), (True, True)):
        res = e.H.empty_fr(N)
        err = e.L.field_op(P(res), P(e.dev(l)), l_rot, P(e.dev(lc)) if use_lc else 0, P(e.dev(r)), r_rot,
                           P(e.dev(rc)) if use_rc else 0, N, op, e.st)
        e.H.abi.check(err) if hasattr(e.H, "abi") else None
        assert err == 0
        exp = O.field_op(l, l_rot, lc if use_lc else None, r, r_rot, rc if use_rc else None, N, op)
        assert (_get(e, res) == exp).all()
    # the size-2 in-place "add [gamma, delta]" use (src/eval_h.rs:757-765)
    a2 = e.cols[4][:2].copy()
    res = e.dev(a2)
    assert e.L.field_op(P(res), P(res), 0, 0, P(e.dev(e.cols[5][:2])), 0, 0, 2, 0, e.st) == 0
    assert (_get(e, res) == O.add(a2, e.cols[5][:2])).all()


def test_field_op_batch_mul_sum(env):
    e, O = env, env.O
    res0, res = _res(e)
    coeffs = O.rand_fr(3, 5)
    terms = [(coeffs[0:1], [(e.cols[0], 0), (e.cols[1], 1)]),
             (coeffs[1:2], [(e.cols[2], -1)]),
             (coeffs[2:3], [(e.cols[3], 2), (e.cols[4], 0), (e.cols[5], -2)])]
    v, rot = [], []
    dc = [e.dev(coeffs[i:i + 1]) for i in range(3)]
    for (c, fs), d in zip(terms, dc):
        v.append(d.data_ptr())
        for col, r in fs:
            v.append(e.dev(col).data_ptr())
            rot.append(r)
        v.append(0)
    vd = torch.tensor(v, dtype=torch.int64, device="cuda")
    rd = torch.tensor(rot, dtype=torch.int32, device="cuda")
    assert e.L.field_op_batch_mul_sum(P(res), P(vd), P(rd), len(v), N, e.st) == 0
    assert (_get(e, res) == O.field_op_batch_mul_sum(res0, terms, N)).all()


def test_field_op_batch_mul_sum_many_groups(env):
    # the term lists of many gate groups in one call: 75 terms of two columns,
    # 300 list entries, more than the kernel stages in shared memory
    e, O = env, env.O
    res0, res = _res(e, 6)
    coeffs = O.rand_fr(75, 6)
    rng = np.random.default_rng(7)
    terms, v, rot = [], [], []
    for t in range(75):
        cs = [(e.cols[int(rng.integers(0, 8))], int(rng.integers(-3, 4))) for _ in range(2)]
        terms.append((coeffs[t:t + 1], cs))
        v.append(e.dev(coeffs[t:t + 1]).data_ptr())
        for col, r in cs:
            v.append(e.dev(col).data_ptr())
            rot.append(r)
        v.append(0)
    assert len(v) == 300
    vd = torch.tensor(v, dtype=torch.int64, device="cuda")
    rd = torch.tensor(rot, dtype=torch.int32, device="cuda")
    assert e.L.field_op_batch_mul_sum(P(res), P(vd), P(rd), len(v), N, e.st) == 0
    assert (_get(e, res) == O.field_op_batch_mul_sum(res0, terms, N)).all()


@pytest.mark.parametrize("yv", [0, 1, "m-1"])
def test_known_factor_edges(env, yv):
    # the challenge (y, beta) and the gate coefficients enter the products as
    # known factors: 0, 1 and m - 1, against columns that hold 0 and m - 1
    e, O = env, env.O
    yv = O.R_MOD - 1 if yv == "m-1" else yv
    y = O.fr_vec([yv])
    c = [x.copy() for x in e.cols]
    for k in range(8):
        c[k][k] = O.fr_vec([0])[0]
        c[k][k + 1] = O.fr_vec([O.R_MOD - 1])[0]
    res0, res = _res(e, 40)
    assert e.L.permutation_eval_h_p1(P(res), P(e.dev(c[0])), P(e.dev(c[1])), P(e.dev(c[6])), P(e.dev(c[7])),
                                     P(e.dev(y)), N) == 0
    assert (_get(e, res) == O.permutation_eval_h_p1(res0, c[0], c[1], c[6], c[7], y)).all()
    res0, res = _res(e, 41)
    assert e.L.permutation_eval_h_p2(P(res), P(e.arr([e.dev(s) for s in c[:4]])), P(e.dev(c[6])), P(e.dev(c[7])),
                                     P(e.dev(y)), 4, 3, N) == 0
    assert (_get(e, res) == O.permutation_eval_h_p2(res0, c[:4], c[6], c[7], y, 3)).all()
    res0, res = _res(e, 42)
    assert e.L.permutation_eval_h_l(P(res), P(e.dev(y)), P(e.dev(e.gamma)), P(e.dev(c[2])), N, e.st) == 0
    assert (_get(e, res) == O.permutation_eval_h_l(res0, y, e.gamma, c[2])).all()
    res0, res = _res(e, 43)
    assert e.L.logup_eval_h(P(res), *[P(e.dev(x)) for x in c[:8]], P(e.dev(c[0])), P(e.dev(y)), -2, N,
                            e.st) == 0
    exp = O.logup_eval_h(res0, c[0], c[1], c[2], c[3], c[4], c[5], c[6], c[7], c[0], y, -2)
    assert (_get(e, res) == exp).all()
    res0, res = _res(e, 44)
    assert e.L.logup_eval_h_extra_inputs(P(res), P(e.dev(c[1])), P(e.dev(c[2])), P(e.dev(c[3])), P(e.dev(c[4])),
                                         P(e.dev(y)), 1, N, e.st) == 0
    assert (_get(e, res) == O.logup_eval_h_extra_inputs(res0, c[1], c[2], c[3], c[4], y, 1)).all()
    res0, res = _res(e, 45)
    assert e.L.shuffle_eval_h(P(res), *[P(e.dev(x)) for x in c[:6]], P(e.dev(y)), 1, N) == 0
    assert (_get(e, res) == O.shuffle_eval_h(res0, c[0], c[1], c[2], c[3], c[4], c[5], y, 1)).all()
    res0, res = _res(e, 46)
    betas = O.fr_vec([yv, 5, O.R_MOD - 1])
    assert e.L.shuffle_eval_h_v2(P(res), P(e.arr([e.dev(x) for x in c[:3]])), P(e.arr([e.dev(x) for x in c[3:6]])),
                                 P(e.dev(betas)), 3, P(e.dev(c[6])), P(e.dev(c[7])), P(e.dev(c[0])),
                                 P(e.dev(c[1])), P(e.dev(y)), 1, N) == 0
    exp = O.shuffle_eval_h_v2(res0, c[:3], c[3:6], betas, c[6], c[7], c[0], c[1], y, 1)
    assert (_get(e, res) == exp).all()
    # gate terms whose coefficients are the edge value, with a term of no
    # columns (its coefficient alone) in the middle of the list
    res0, res = _res(e, 47)
    coeffs = O.fr_vec([yv, O.R_MOD - 1, yv, 7])
    terms = [(coeffs[0:1], [(c[0], 0), (c[1], 1)]), (coeffs[1:2], []), (coeffs[2:3], [(c[2], -1)]),
             (coeffs[3:4], [(c[3], 2), (c[4], 0), (c[5], -2)])]
    v, rot = [], []
    for cf, fs in terms:
        v.append(e.dev(cf).data_ptr())
        for col, r in fs:
            v.append(e.dev(col).data_ptr())
            rot.append(r)
        v.append(0)
    vd = torch.tensor(v, dtype=torch.int64, device="cuda")
    rd = torch.tensor(rot, dtype=torch.int32, device="cuda")
    assert e.L.field_op_batch_mul_sum(P(res), P(vd), P(rd), len(v), N, e.st) == 0
    assert (_get(e, res) == O.field_op_batch_mul_sum(res0, terms, N)).all()


def test_permutation_eval_h(env):
    e, O = env, env.O
    l0, ll = e.cols[6], e.cols[7]
    res0, res = _res(e, 1)
    assert e.L.permutation_eval_h_p1(P(res), P(e.dev(e.cols[0])), P(e.dev(e.cols[1])), P(e.dev(l0)), P(e.dev(ll)),
                                     P(e.dev(e.y)), N) == 0
    assert (_get(e, res) == O.permutation_eval_h_p1(res0, e.cols[0], e.cols[1], l0, ll, e.y)).all()
    res0, res = _res(e, 2)
    sets = e.cols[:4]
    rot = -7
    assert e.L.permutation_eval_h_p2(P(res), P(e.arr([e.dev(s) for s in sets])), P(e.dev(l0)), P(e.dev(ll)),
                                     P(e.dev(e.y)), len(sets), rot, N) == 0
    assert (_get(e, res) == O.permutation_eval_h_p2(res0, sets, l0, ll, e.y, rot)).all()
    res0, res = _res(e, 3)
    assert e.L.logup_eval_h_z_set(P(res), P(e.arr([e.dev(s) for s in sets])), P(e.dev(l0)), P(e.dev(ll)),
                                  P(e.dev(e.y)), len(sets), rot, N, e.st) == 0
    assert (_get(e, res) == O.permutation_eval_h_p2(res0, sets, l0, ll, e.y, rot)).all()
    res0, res = _res(e, 4)
    assert e.L.permutation_eval_h_l(P(res), P(e.dev(e.beta)), P(e.dev(e.gamma)), P(e.dev(e.cols[2])), N,
                                    e.st) == 0
    assert (_get(e, res) == O.permutation_eval_h_l(res0, e.beta, e.gamma, e.cols[2])).all()


def test_logup_eval_h(env):
    e, O = env, env.O
    c = e.cols
    res0, res = _res(e, 5)
    assert e.L.logup_eval_h(P(res), *[P(e.dev(x)) for x in c[:8]], P(e.dev(c[0])), P(e.dev(e.y)), 1, N,
                            e.st) == 0
    exp = O.logup_eval_h(res0, c[0], c[1], c[2], c[3], c[4], c[5], c[6], c[7], c[0], e.y, 1)
    assert (_get(e, res) == exp).all()
    res0, res = _res(e, 6)
    assert e.L.logup_eval_h_extra_inputs(P(res), P(e.dev(c[1])), P(e.dev(c[2])), P(e.dev(c[3])), P(e.dev(c[4])),
                                         P(e.dev(e.y)), 1, N, e.st) == 0
    exp = O.logup_eval_h_extra_inputs(res0, c[1], c[2], c[3], c[4], e.y, 1)
    assert (_get(e, res) == exp).all()
    for k in (1, 2, 5):
        prod, psum = e.H.empty_fr(N), e.H.empty_fr(N)
        assert e.L.logup_eval_h_inputs_product_sum(P(prod), P(psum), P(e.arr([e.dev(x) for x in c[:k]])), k, N,
                                                   e.st) == 0
        ep, es = O.logup_eval_h_inputs_product_sum(c[:k])
        assert (_get(e, prod) == ep).all() and (_get(e, psum) == es).all()


def test_lookup_eval_h(env):
    e, O = env, env.O
    c = e.cols
    res0, res = _res(e, 7)
    # res, input, table, permuted_input, permuted_table, z, l0, l_last, l_active_row, y, beta, gamma
    assert e.L.lookup_eval_h(P(res), *[P(e.dev(x)) for x in c[:8]], P(e.dev(e.y)),
                             P(e.dev(e.beta)), P(e.dev(e.gamma)), 1, N, e.st) == 0
    # restated from cuda/bn254.cu:798-865
    inp, tab, pin, ptab, z, l0, ll, la = c[0], c[1], c[2], c[3], c[4], c[5], c[6], c[7]
    t = O.mul(res0, e.y)
    t = O.add(t, O.mul(l0, O.sub(O.one(1), z)))
    t = O.mul(t, e.y)
    t = O.add(t, O.mul(ll, O.sub(O.sqr(z), z)))
    t = O.mul(t, e.y)
    u = O.mul(O.mul(O.add(pin, e.beta), O.add(ptab, e.gamma)), O._rot(z, 1))
    u = O.sub(u, O.mul(z, O.mul(inp, tab)))
    t = O.add(t, O.mul(u, la))
    t = O.mul(t, e.y)
    p = O.sub(pin, ptab)
    t = O.add(t, O.mul(l0, p))
    t = O.mul(t, e.y)
    u = O.mul(O.sub(pin, O._rot(pin, -1)), p)
    t = O.add(t, O.mul(u, la))
    assert (_get(e, res) == t).all()


def test_shuffle_eval_h(env):
    e, O = env, env.O
    c = e.cols
    res0, res = _res(e, 8)
    assert e.L.shuffle_eval_h(P(res), *[P(e.dev(x)) for x in c[:6]], P(e.dev(e.y)), 1, N) == 0
    exp = O.shuffle_eval_h(res0, c[0], c[1], c[2], c[3], c[4], c[5], e.y, 1)
    assert (_get(e, res) == exp).all()
    res0, res = _res(e, 9)
    betas = O.rand_fr(3, 10)
    assert e.L.shuffle_eval_h_v2(P(res), P(e.arr([e.dev(x) for x in c[:3]])), P(e.arr([e.dev(x) for x in c[3:6]])),
                                 P(e.dev(betas)), 3, P(e.dev(c[6])), P(e.dev(c[7])), P(e.dev(c[0])),
                                 P(e.dev(c[1])), P(e.dev(e.y)), 1, N) == 0
    exp = O.shuffle_eval_h_v2(res0, c[:3], c[3:6], betas, c[6], c[7], c[0], c[1], e.y, 1)
    assert (_get(e, res) == exp).all()


def test_small_maps(env):
    e, O = env, env.O
    c = e.cols
    buf = e.dev(c[0].copy())
    coeff = c[1][:5].copy()
    assert e.L.field_mul_zip(P(buf), P(e.dev(coeff)), 5, N) == 0
    assert (_get(e, buf) == O.field_mul_zip(c[0], coeff)).all()
    # field_sum: res = sum_j v_j[i] * omegas[((n + rot_j) * i) mod n] * c_j
    log_n = 12
    om = O.expand_omega(O.omega(log_n), log_n)
    res = e.H.empty_fr(N)
    vs = [e.dev(x) for x in c[:3]]
    vc = [e.dev(c[3][:1]), None, e.dev(c[4][:1])]
    rots = [0, 1, -1]
    vcd = torch.tensor([0 if x is None else x.data_ptr() for x in vc], dtype=torch.int64, device="cuda")
    rd = torch.tensor(rots, dtype=torch.int32, device="cuda")
    assert e.L.field_sum(P(res), P(e.arr(vs)), P(vcd), P(rd), P(e.dev(om)), 3, N) == 0
    exp = O.field_sum(c[:3], [c[3][:1], None, c[4][:1]], rots, om, N)
    assert (_get(e, res) == exp).all()
    # shplonk helpers
    res0, res = _res(e, 11)
    diffs = O.rand_fr(3, 12)
    assert e.L.shplonk_h_x_merge(P(res), P(e.dev(e.y)), P(e.dev(c[2])), P(e.dev(om)), P(e.dev(diffs)), 3, N) == 0
    assert (_get(e, res) == O.shplonk_h_x_merge(res0, e.y, c[2], om, diffs)).all()
    vals = e.dev(c[5].copy())
    pts = O.rand_fr(4, 13)
    assert e.L.shplonk_h_x_div_points(P(vals), P(e.dev(om)), P(e.dev(pts)), 4, N) == 0
    assert (_get(e, vals) == O.shplonk_h_x_div_points(c[5], om, pts)).all()


@pytest.mark.parametrize("log_n", [1, 4, 12, 16])
def test_poly_eval(env, log_n):
    e, O = env, env.O
    n = 1 << log_n
    p = O.rand_fr(n, 20 + log_n)
    x = O.fr_ints(O.rand_fr(1, 21))[0]
    xt = O.fr_vec([pow(x, 1 << d, O.R_MOD) for d in range(max(1, log_n))])
    res = e.H.empty_fr(n)
    assert e.L.poly_eval(P(e.dev(p)), P(res), P(e.dev(xt)), n, e.st) == 0
    assert O.fr_ints(_get(e, res)[:1])[0] == O.poly_eval(p, x)


def test_lookup_multiplicity(env):
    e, O = env, env.O
    k = 12
    n = 1 << k
    u = n - 9
    rng = random.Random(3)
    table = [rng.randrange(300) for _ in range(n)]  # duplicates on purpose
    present = sorted(set(table[:u]))
    inputs = [[rng.choice(present) for _ in range(n)] for _ in range(2)]
    m = [0] * n
    last = {}
    for i in range(u):
        last[table[i]] = i  # largest usable row holding each value
    for inp in inputs:
        for x in inp[:u]:
            m[last[x]] += 1
    dt = e.dev(O.fr_vec(table))
    words = [torch.empty(n * 8, dtype=torch.int32, device="cuda") for _ in range(6)]
    mm = e.H.zeros_fr(n)
    assert e.L.prepare_table_lookup(P(dt), P(words[0]), P(words[1]), P(words[2]), P(words[3]), P(words[4]),
                                    P(words[5]), n * 32, k, u, e.st) == 0
    for inp in inputs:
        assert e.L.calc_m(P(mm), P(dt), P(e.dev(O.fr_vec(inp))), P(words[3]), P(words[4]), P(words[0]),
                          P(words[1]), P(words[5]), n * 32, k, u, e.st) == 0
    assert O.fr_ints(_get(e, mm)) == m
