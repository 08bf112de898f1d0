"""Runs the device field and curve code on the CPU (host emulation of the PTX
carry chains, tests/host_check.cpp) against the oracle.  This checks the exact
operation sequence of csrc/field.cuh and csrc/curve.cuh without a GPU."""
import ctypes
import os
import random
import subprocess
import tempfile

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))


@pytest.fixture(scope="module")
def hc():
    out = os.path.join(tempfile.mkdtemp(prefix="zk_hc_"), "hc.so")
    subprocess.check_call(["g++", "-O2", "-std=c++17", "-shared", "-fPIC", "-o", out,
                           os.path.join(HERE, "host_check.cpp")])
    L = ctypes.CDLL(out)
    P = ctypes.c_void_p
    for name, args in {
        "hc_mul": [ctypes.c_int, P, P, P, ctypes.c_long],
        "hc_add": [ctypes.c_int, P, P, P, ctypes.c_long],
        "hc_sub": [ctypes.c_int, P, P, P, ctypes.c_long],
        "hc_inv": [P, P, ctypes.c_long],
        "hc_from_mont": [P, P, ctypes.c_long],
        "hc_pow": [P, P, ctypes.c_uint32],
        "hc_xyzz_from_aff": [P, P],
        "hc_xyzz_add_aff": [P, P, P],
        "hc_xyzz_add": [P, P, P],
        "hc_xyzz_dbl": [P, P],
        "hc_xyzz_mul_u32": [P, P, ctypes.c_uint32],
        "hc_xyzz_to_jac": [P, P],
        "hc_glv_split": [P, P, P, P, ctypes.c_long],
        "hc_lazy": [ctypes.c_int, P, P, P, ctypes.c_long],
        "hc_madd_lazy_chain": [P, P, P, ctypes.c_long],
        "hc_mul_shoup": [P, P, P, P, ctypes.c_long],
        "hc_glv_phi": [P, P, ctypes.c_long],
    }.items():
        getattr(L, name).argtypes = args
    L.hc_bits_at.argtypes = [P, ctypes.c_uint32, ctypes.c_uint32]
    L.hc_bits_at.restype = ctypes.c_uint32
    L.hc_signed_digit.argtypes = [P, ctypes.c_int, ctypes.c_int, P]
    L.hc_signed_digit.restype = ctypes.c_int
    return L


def _p(a):
    return a.ctypes.data


def _edge(O, mod, conv):
    rng = random.Random(5)
    vals = [0, 1, 2, mod - 1, mod - 2, (mod - 1) // 2, 1 << 200, (1 << 254) % mod]
    vals += [rng.randrange(mod) for _ in range(300)]
    return vals, np.concatenate([conv(v) for v in vals])


@pytest.mark.parametrize("which", [0, 1])
def test_field_ops_match_oracle(O, hc, which):
    mod = O.R_MOD if which == 0 else O.Q_MOD
    conv = O.fr if which == 0 else O.fq
    xs, a = _edge(O, mod, conv)
    ys = xs[::-1]
    b = a[::-1].copy()
    for name, ref in (("hc_mul", O.mul), ("hc_add", O.add), ("hc_sub", O.sub)):
        out = np.empty_like(a)
        getattr(hc, name)(which, _p(out), _p(a), _p(b), a.shape[0])
        assert (out == ref(a, b, which)).all(), name


def test_lazy_inputs_below_2m(O, hc):
    # fe_mul accepts inputs below 2m: feed raw limbs of x + m
    rng = random.Random(9)
    for which, mod in ((0, O.R_MOD), (1, O.Q_MOD)):
        xs = [rng.randrange(mod) for _ in range(100)]
        ys = [rng.randrange(mod) for _ in range(100)]
        a = np.stack([O.int_to_limbs((x * O.MONT_R % mod) + mod) for x in xs])
        b = np.stack([O.int_to_limbs(y * O.MONT_R % mod) for y in ys])
        out = np.empty_like(a)
        hc.hc_mul(which, _p(out), _p(a), _p(b), a.shape[0])
        ints = O.fr_ints if which == 0 else O.fq_ints
        assert ints(out) == [x * y % mod for x, y in zip(xs, ys)]
        assert all(O.limbs_to_int(out[i]) < mod for i in range(out.shape[0]))


def test_inverse_pow_from_mont(O, hc):
    xs, a = _edge(O, O.R_MOD, O.fr)
    out = np.empty_like(a)
    hc.hc_inv(_p(out), _p(a), a.shape[0])
    assert (out == O.inv(a)).all()
    hc.hc_from_mont(_p(out), _p(a), a.shape[0])
    assert [O.limbs_to_int(out[i]) for i in range(len(xs))] == [x % O.R_MOD for x in xs]
    o1 = np.empty((1, 4), np.uint64)
    hc.hc_pow(_p(o1), _p(O.fr(3)), 1000003)
    assert O.fr_ints(o1)[0] == pow(3, 1000003, O.R_MOD)


def test_signed_digits_recompose(O, hc):
    rng = random.Random(17)
    ks = [0, 1, O.R_MOD - 1, (1 << 253) + 12345] + [rng.randrange(O.R_MOD) for _ in range(200)]
    for c in (4, 7, 10, 13, 15, 16, 17, 20, 22):
        W = (254 + c - 1) // c
        for k in ks:
            limbs = O.int_to_limbs(k)
            carry = ctypes.c_uint32(0)
            tot = 0
            for w in range(W):
                d = hc.hc_signed_digit(_p(limbs), w, c, ctypes.addressof(carry))
                assert -(1 << (c - 1)) < d <= (1 << (c - 1))
                tot += d << (c * w)
            assert carry.value == 0 and tot == k, (c, k)


def _x_of_aff(O, p):
    x = np.empty(16, np.uint64)
    return x


def _xyzz(hc, aff):
    out = np.empty(16, np.uint64)
    hc.hc_xyzz_from_aff(_p(out), _p(np.ascontiguousarray(aff.reshape(8))))
    return out


def _to_aff(O, hc, x):
    j = np.empty(12, np.uint64)
    hc.hc_xyzz_to_jac(_p(j), _p(x))
    return O.g1_jac_to_aff(j)[0]


def test_xyzz_formulas(O, hc):
    ks = O.rand_fr(6, 23)
    pts = O.g1_gen_bases(ks)
    kk = O.fr_ints(ks)
    P0 = O.aff_to_pyint(pts[0])
    # chain of mixed additions equals the sum
    acc = np.zeros(16, np.uint64)  # identity (ZZ = 0)
    exp = None
    for p in pts:
        out = np.empty(16, np.uint64)
        hc.hc_xyzz_add_aff(_p(out), _p(acc), _p(np.ascontiguousarray(p)))
        acc = out
        exp = O.pyint_ec_add(exp, O.aff_to_pyint(p))
    assert O.aff_to_pyint(_to_aff(O, hc, acc)) == exp
    # P + P through the mixed-addition doubling branch
    x0 = _xyzz(hc, pts[0])
    out = np.empty(16, np.uint64)
    hc.hc_xyzz_add_aff(_p(out), _p(x0), _p(np.ascontiguousarray(pts[0])))
    assert O.aff_to_pyint(_to_aff(O, hc, out)) == O.pyint_ec_add(P0, P0)
    # P + (-P) = identity
    negp = pts[0].copy()
    negp[4:] = O.neg(pts[0][4:], 1)
    hc.hc_xyzz_add_aff(_p(out), _p(x0), _p(np.ascontiguousarray(negp)))
    assert O.aff_to_pyint(_to_aff(O, hc, out)) is None
    # general addition, doubling, and the equal-points branch of add
    x1 = _xyzz(hc, pts[1])
    hc.hc_xyzz_add(_p(out), _p(x0), _p(x1))
    assert O.aff_to_pyint(_to_aff(O, hc, out)) == O.pyint_ec_add(P0, O.aff_to_pyint(pts[1]))
    d = np.empty(16, np.uint64)
    hc.hc_xyzz_dbl(_p(d), _p(out))
    s01 = O.pyint_ec_add(P0, O.aff_to_pyint(pts[1]))
    assert O.aff_to_pyint(_to_aff(O, hc, d)) == O.pyint_ec_add(s01, s01)
    hc.hc_xyzz_add(_p(d), _p(out), _p(out))
    assert O.aff_to_pyint(_to_aff(O, hc, d)) == O.pyint_ec_add(s01, s01)
    # small scalar multiplication
    for k in (1, 2, 3, 255, 16384, 65535):
        hc.hc_xyzz_mul_u32(_p(d), _p(x0), k)
        assert O.aff_to_pyint(_to_aff(O, hc, d)) == O.pyint_ec_mul(P0, k)
    # identity conversions
    zero = np.zeros(16, np.uint64)
    j = np.empty(12, np.uint64)
    hc.hc_xyzz_to_jac(_p(j), _p(zero))
    assert O.fq_ints(j[8:])[0] == 0 and O.fq_ints(j[4:8])[0] == 1


def test_glv_split_matches_restatement(O, hc):
    rng = random.Random(17)
    ks = [0, 1, 2, O.R_MOD - 1, O.R_MOD // 2, O.GLV_LAMBDA, (O.R_MOD - 1) // 3, (1 << 253) - 1]
    ks += [rng.randrange(O.R_MOD) for _ in range(3000)]
    k = np.array([[(x >> (64 * j)) & (2 ** 64 - 1) for j in range(4)] for x in ks], np.uint64)
    m1, m2 = np.zeros_like(k), np.zeros_like(k)
    neg = np.zeros(2 * len(ks), np.int32)
    hc.hc_glv_split(_p(k), _p(m1), _p(m2), _p(neg), len(ks))
    for i, x in enumerate(ks):
        a = sum(int(m1[i, j]) << (64 * j) for j in range(4)) * (-1 if neg[2 * i] else 1)
        b = sum(int(m2[i, j]) << (64 * j) for j in range(4)) * (-1 if neg[2 * i + 1] else 1)
        assert (a, b) == O.glv_split(x)
        assert (a + b * O.GLV_LAMBDA - x) % O.R_MOD == 0
        assert abs(a) < 2 ** 127 and abs(b) < 2 ** 127


def test_glv_phi_is_lambda_multiple(O, hc):
    d = O.rand_fr(64, 18)
    pts = O.g1_gen_bases(d)
    out = np.zeros_like(pts)
    hc.hc_glv_phi(_p(out), _p(pts), pts.shape[0])
    lam = O.fr_vec([x * O.GLV_LAMBDA % O.R_MOD for x in O.fr_ints(d)])
    assert (out == O.g1_gen_bases(lam)).all()


@pytest.mark.parametrize("op", [0, 1, 2, 3, 4, 5])
def test_lazy_fr_ops(O, hc, op):
    # representatives in [0, 2m): results stay below 2m and are congruent to
    # the exact Montgomery product / sum / difference (ops 3-5: over Fq)
    r = O.R_MOD if op < 3 else O.Q_MOD
    rng = random.Random(40 + op)
    xs = [0, 1, r - 1, r, r + 1, 2 * r - 1] + [rng.randrange(2 * r) for _ in range(2000)]
    ys = [2 * r - 1, r, 1, 0, r - 1, 2 * r - 1] + [rng.randrange(2 * r) for _ in range(2000)]
    lim = lambda v: np.array([[(v >> (64 * j)) & (2 ** 64 - 1) for j in range(4)]], np.uint64)
    a = np.concatenate([lim(x) for x in xs])
    b = np.concatenate([lim(y) for y in ys])
    out = np.zeros_like(a)
    hc.hc_lazy(op, _p(out), _p(a), _p(b), a.shape[0])
    rinv = pow(1 << 256, -1, r)
    for i, (x, y) in enumerate(zip(xs, ys)):
        got = sum(int(out[i, j]) << (64 * j) for j in range(4))
        exp = x * y * rinv if op % 3 == 0 else x + y if op % 3 == 1 else x - y
        assert got < 2 * r and (got - exp) % r == 0


def test_madd_lazy_chain(O, hc):
    # mixed additions on [0, 2p) coordinates (the accumulation loop's form)
    # equal the canonical chain, including the doubling and P + (-P) branches
    ks = O.rand_fr(40, 47)
    pts = O.g1_gen_bases(ks)
    pts[7] = pts[6]                            # equal points: doubling branch
    pts[9] = pts[8]
    pts[9, 4:] = O.neg(pts[8][4:], 1)          # P + (-P) after the run so far
    acc = np.zeros(16, np.uint64)
    for p in pts:
        out = np.empty(16, np.uint64)
        hc.hc_xyzz_add_aff(_p(out), _p(acc), _p(np.ascontiguousarray(p)))
        acc = out
    got = np.empty(16, np.uint64)
    hc.hc_madd_lazy_chain(_p(got), _p(np.zeros(16, np.uint64)), _p(np.ascontiguousarray(pts)), pts.shape[0])
    assert (got == acc).all()
    # a start point whose coordinates are lifted to [p, 2p)
    start = _xyzz(hc, pts[0])
    lifted = start.copy()
    for k in range(4):
        v = sum(int(start[4 * k + j]) << (64 * j) for j in range(4)) + O.Q_MOD
        lifted[4 * k: 4 * k + 4] = [(v >> (64 * j)) & (2 ** 64 - 1) for j in range(4)]
    ref = start
    for p in pts[1:20]:
        out = np.empty(16, np.uint64)
        hc.hc_xyzz_add_aff(_p(out), _p(ref), _p(np.ascontiguousarray(p)))
        ref = out
    hc.hc_madd_lazy_chain(_p(got), _p(lifted), _p(np.ascontiguousarray(pts[1:20])), 19)
    assert (got == ref).all()


def test_mul_by_known_factor(O, hc):
    # a * w mod r from w and w' = floor(w 2^256 / r) for any a < 2^256:
    # result below 2r and congruent; extreme a and w included
    r = O.R_MOD
    rng = random.Random(61)
    A = [0, 1, 2 ** 256 - 1, 2 * r - 1, r] + [rng.randrange(2 ** 256) for _ in range(3000)]
    Wv = [r - 1, 1, 0, r - 1, (r - 1) // 2] + [rng.randrange(r) for _ in range(3000)]
    lim = lambda v: [(v >> (64 * j)) & (2 ** 64 - 1) for j in range(4)]
    a = np.array([lim(x) for x in A], np.uint64)
    w = np.array([lim(x) for x in Wv], np.uint64)
    wp = np.array([lim((x << 256) // r) for x in Wv], np.uint64)
    out = np.zeros_like(a)
    hc.hc_mul_shoup(_p(out), _p(a), _p(w), _p(wp), a.shape[0])
    for i, (x, y) in enumerate(zip(A, Wv)):
        got = sum(int(out[i, j]) << (64 * j) for j in range(4))
        assert got < 2 * r and (got - x * y) % r == 0, i
