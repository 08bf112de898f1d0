"""Cases that run one reference-ABI symbol on seeded inputs, shared by the
parity tests against the reference's own kernels (tests/test_ref_parity_gpu.py)
and by the golden-vector generator (tests/golden/make_golden.py).

Each case builds its inputs from the oracle's seeded generator, calls the
symbol through a ctypes library (this project's libzkwasm_prover_kernel.so or
the reference's cuda/bn254.cu rebuilt for sm_100a in oracle/_ref/), and
returns its outputs as numpy uint64 arrays; ``expect`` restates the same
outputs with the oracle on the CPU.  Every case stays inside the reference's
own preconditions (cuda/bn254.cu):
  * sizes are multiples of 64 (one 64-thread block per 64 rows, no tail);
  * field_op rotations are >= 0: the reference indexes l[(i + rot) % n] with
    signed ints, which reads before the buffer for a negative rot;
  * logup_sum_input_inv needs n >= 32768 (cuda/bn254.cu:1914-1934) and the
    logup z scans n a multiple of 16384 (cuda/bn254.cu:1936-1993);
  * calc_m's inputs are all present in the table (the reference asserts,
    cuda/bn254.cu:1694);
  * shplonk points lie outside the domain (no zero denominators).
Test infrastructure only: nothing in the product imports it.
"""
from __future__ import annotations

import ctypes
import hashlib
import importlib
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for _p in (ROOT, os.path.join(ROOT, "oracle")):
    if _p not in sys.path:
        sys.path.insert(0, _p)

import oracle as O  # noqa: E402

REF_LIB = os.path.join(ROOT, "oracle", "_ref", "libzkwasm_prover_kernel_ref.so")
# halo2curves' ZETA for BN254 Fr: the cube root of unity that is also G1's GLV lambda
ZETA = O.GLV_LAMBDA


def sha(a) -> str:
    return hashlib.sha256(np.ascontiguousarray(a, np.uint64).tobytes()).hexdigest()


def load_ref():
    """The reference kernels rebuilt for sm_100a, with the argument types of
    the reference FFI (src/cuda/bn254_c.rs:4-309) set on each symbol."""
    pkg = importlib.import_module("zkwasm-prover_b200")
    lib = ctypes.CDLL(REF_LIB)
    for name, sig in pkg.abi.SIGNATURES.items():
        if name.startswith("zkp_"):
            continue
        fn = getattr(lib, name)
        fn.argtypes, fn.restype = sig, ctypes.c_int
    return lib


class Dev:
    """Device buffers of one case run (kept alive until the case synchronises)."""

    def __init__(self):
        import torch

        self.torch = torch
        self.keep = []

    def put(self, a):
        t = self.torch.from_numpy(np.ascontiguousarray(a, np.uint64).view(np.int64)).cuda()
        self.keep.append(t)
        return t

    def empty(self, n, words=4):
        t = self.torch.empty((n, words), dtype=self.torch.int64, device="cuda")
        self.keep.append(t)
        return t

    def zeros(self, n, words=4):
        t = self.torch.zeros((n, words), dtype=self.torch.int64, device="cuda")
        self.keep.append(t)
        return t

    def ptrs(self, ts):
        t = self.torch.tensor([0 if x is None else x.data_ptr() for x in ts], dtype=self.torch.int64, device="cuda")
        self.keep.append(t)
        return t

    def i32(self, xs):
        t = self.torch.tensor(list(xs), dtype=self.torch.int32, device="cuda")
        self.keep.append(t)
        return t

    def get(self, t):
        self.torch.cuda.synchronize()
        return t.detach().cpu().contiguous().numpy().view(np.uint64)


def P(t):
    return 0 if t is None else t.data_ptr()


def inputs(n: int, seed: int):
    """Eight seeded columns and three seeded challenges."""
    cols = [O.rand_fr(n, seed + i) for i in range(8)]
    y, beta, gamma = O.rand_fr(1, seed + 100), O.rand_fr(1, seed + 101), O.rand_fr(1, seed + 102)
    return cols, y, beta, gamma


class Case:
    """One symbol call: run(L, d, n) -> {name: array}; expect(n) -> the same
    from the oracle; min_n: the smallest n the reference accepts."""

    def __init__(self, name, run, expect, min_n=64):
        self.name, self.run, self.expect, self.min_n = name, run, expect, min_n


CASES = []


def case(name, min_n=64):
    def deco(pair):
        run, expect = pair()
        CASES.append(Case(name, run, expect, min_n))
        return pair
    return deco


SEED = 4242

# ---------------------------------------------------------------- field_op

_FIELD_OP_VARIANTS = [(0, 0, False, False), (1, 3, True, False), (5, 0, False, True), (2, 1, True, True),
                      (0, 7, "only", False)]


def _field_op_case(op, l_rot, r_rot, lc, rc):
    def run(L, d, n):
        cols, *_ = inputs(n, SEED)
        l = None if lc == "only" else d.put(cols[0])
        lcd = d.put(cols[2][:1]) if lc else None
        rcd = d.put(cols[3][:1]) if rc else None
        res = d.empty(n)
        assert L.field_op(P(res), P(l), l_rot, P(lcd), P(d.put(cols[1])), r_rot, P(rcd), n, op, None) == 0
        return {"res": d.get(res)}

    def expect(n):
        cols, *_ = inputs(n, SEED)
        l = None if lc == "only" else cols[0]
        return {"res": O.field_op(l, l_rot, cols[2][:1] if lc else None, cols[1], r_rot,
                                  cols[3][:1] if rc else None, n, op)}
    return run, expect


for _op in range(4):
    for _v in _FIELD_OP_VARIANTS:
        _run, _exp = _field_op_case(_op, *_v)
        CASES.append(Case(f"field_op_op{_op}_rot{_v[0]}_{_v[1]}_c{_v[2]}{_v[3]}", _run, _exp))


def _terms(n, cols, coeffs):
    """Gate-like term list: coefficient, columns with rotations (both signs),
    and a term of the coefficient alone."""
    spec = [[(0, 0), (1, 1)], [], [(2, -1)], [(3, 2), (4, 0), (5, -2)], [(6, 8), (6, 0)]]
    return [(coeffs[i:i + 1], [(cols[c], r) for c, r in s]) for i, s in enumerate(spec)]


@case("field_op_batch_mul_sum")
def _():
    def run(L, d, n):
        cols, *_ = inputs(n, SEED)
        coeffs = O.rand_fr(5, SEED + 7)
        res = d.put(O.rand_fr(n, SEED + 8))
        v, rot = [], []
        for c, fs in _terms(n, cols, coeffs):
            v.append(d.put(c))
            for col, r in fs:
                v.append(d.put(col))
                rot.append(r)
            v.append(None)
        vd = d.ptrs(v)
        assert L.field_op_batch_mul_sum(P(res), P(vd), P(d.i32(rot)), len(v), n, None) == 0
        return {"res": d.get(res)}

    def expect(n):
        cols, *_ = inputs(n, SEED)
        return {"res": O.field_op_batch_mul_sum(O.rand_fr(n, SEED + 8), _terms(n, cols, O.rand_fr(5, SEED + 7)), n)}
    return run, expect


# ---------------------------------------------------------------- permutation


@case("permutation_eval_h_p1")
def _():
    def run(L, d, n):
        c, y, *_ = inputs(n, SEED)
        res = d.put(c[7])
        assert L.permutation_eval_h_p1(P(res), P(d.put(c[0])), P(d.put(c[1])), P(d.put(c[2])), P(d.put(c[3])),
                                       P(d.put(y)), n) == 0
        return {"res": d.get(res)}

    def expect(n):
        c, y, *_ = inputs(n, SEED)
        return {"res": O.permutation_eval_h_p1(c[7], c[0], c[1], c[2], c[3], y)}
    return run, expect


def _p2_case(rot, sym):
    def run(L, d, n):
        c, y, *_ = inputs(n, SEED)
        res = d.put(c[7])
        sets = d.ptrs([d.put(s) for s in c[:4]])
        if sym == "p2":
            assert L.permutation_eval_h_p2(P(res), P(sets), P(d.put(c[4])), P(d.put(c[5])), P(d.put(y)), 4, rot,
                                           n) == 0
        else:
            assert L.logup_eval_h_z_set(P(res), P(sets), P(d.put(c[4])), P(d.put(c[5])), P(d.put(y)), 4, rot, n,
                                        None) == 0
        return {"res": d.get(res)}

    def expect(n):
        c, y, *_ = inputs(n, SEED)
        return {"res": O.permutation_eval_h_p2(c[7], c[:4], c[4], c[5], y, rot)}
    return run, expect


for _rot in (-40, 24):
    for _sym in ("p2", "z_set"):
        _run, _exp = _p2_case(_rot, _sym)
        CASES.append(Case(f"{'permutation_eval_h_p2' if _sym == 'p2' else 'logup_eval_h_z_set'}_rot{_rot}",
                          _run, _exp))


@case("permutation_eval_h_l")
def _():
    def run(L, d, n):
        c, y, beta, gamma = inputs(n, SEED)
        res = d.put(c[7])
        assert L.permutation_eval_h_l(P(res), P(d.put(beta)), P(d.put(gamma)), P(d.put(c[0])), n, None) == 0
        return {"res": d.get(res)}

    def expect(n):
        c, y, beta, gamma = inputs(n, SEED)
        return {"res": O.permutation_eval_h_l(c[7], beta, gamma, c[0])}
    return run, expect


# ---------------------------------------------------------------- lookups and shuffles


def _logup_case(rot):
    def run(L, d, n):
        c, y, *_ = inputs(n, SEED)
        res = d.put(O.rand_fr(n, SEED + 9))
        assert L.logup_eval_h(P(res), *[P(d.put(x)) for x in c[:8]], P(d.put(c[0])), P(d.put(y)), rot, n,
                              None) == 0
        return {"res": d.get(res)}

    def expect(n):
        c, y, *_ = inputs(n, SEED)
        return {"res": O.logup_eval_h(O.rand_fr(n, SEED + 9), c[0], c[1], c[2], c[3], c[4], c[5], c[6], c[7], c[0],
                                      y, rot)}
    return run, expect


for _rot in (1, 8):
    _run, _exp = _logup_case(_rot)
    CASES.append(Case(f"logup_eval_h_rot{_rot}", _run, _exp))


@case("logup_eval_h_extra_inputs")
def _():
    def run(L, d, n):
        c, y, *_ = inputs(n, SEED)
        res = d.put(c[7])
        assert L.logup_eval_h_extra_inputs(P(res), P(d.put(c[1])), P(d.put(c[2])), P(d.put(c[3])), P(d.put(c[4])),
                                           P(d.put(y)), 8, n, None) == 0
        return {"res": d.get(res)}

    def expect(n):
        c, y, *_ = inputs(n, SEED)
        return {"res": O.logup_eval_h_extra_inputs(c[7], c[1], c[2], c[3], c[4], y, 8)}
    return run, expect


def _ips_case(k):
    def run(L, d, n):
        c, *_ = inputs(n, SEED)
        prod, psum = d.empty(n), d.empty(n)
        assert L.logup_eval_h_inputs_product_sum(P(prod), P(psum), P(d.ptrs([d.put(x) for x in c[:k]])), k, n,
                                                 None) == 0
        return {"product": d.get(prod), "product_sum": d.get(psum)}

    def expect(n):
        c, *_ = inputs(n, SEED)
        p, s = O.logup_eval_h_inputs_product_sum(c[:k])
        return {"product": p, "product_sum": s}
    return run, expect


for _k in (1, 2, 3):
    _run, _exp = _ips_case(_k)
    CASES.append(Case(f"logup_eval_h_inputs_product_sum_{_k}", _run, _exp))


@case("shuffle_eval_h")
def _():
    def run(L, d, n):
        c, y, *_ = inputs(n, SEED)
        res = d.put(c[7])
        assert L.shuffle_eval_h(P(res), *[P(d.put(x)) for x in c[:6]], P(d.put(y)), 8, n) == 0
        return {"res": d.get(res)}

    def expect(n):
        c, y, *_ = inputs(n, SEED)
        return {"res": O.shuffle_eval_h(c[7], c[0], c[1], c[2], c[3], c[4], c[5], y, 8)}
    return run, expect


@case("shuffle_eval_h_v2")
def _():
    def run(L, d, n):
        c, y, beta, _ = inputs(n, SEED)
        res = d.put(c[7])
        betas = O.rand_fr(3, SEED + 10)
        assert L.shuffle_eval_h_v2(P(res), P(d.ptrs([d.put(x) for x in c[:3]])), P(d.ptrs([d.put(x) for x in c[3:6]])),
                                   P(d.put(betas)), 3, P(d.put(c[6])), P(d.put(c[0])), P(d.put(c[1])),
                                   P(d.put(c[2])), P(d.put(y)), 1, n) == 0
        return {"res": d.get(res)}

    def expect(n):
        c, y, beta, _ = inputs(n, SEED)
        return {"res": O.shuffle_eval_h_v2(c[7], c[:3], c[3:6], O.rand_fr(3, SEED + 10), c[6], c[0], c[1], c[2], y,
                                           1)}
    return run, expect


def _lookup_expect(res0, c, y, beta, gamma):
    """cuda/bn254.cu:798-865, restated step by step."""
    inp, tab, pin, ptab, z, l0, ll, la = c[0], c[1], c[2], c[3], c[4], c[5], c[6], c[7]
    t = O.mul(res0, y)
    t = O.add(t, O.mul(l0, O.sub(O.one(1), z)))
    t = O.mul(t, y)
    t = O.add(t, O.mul(ll, O.sub(O.sqr(z), z)))
    t = O.mul(t, y)
    u = O.mul(O.mul(O.add(pin, beta), O.add(ptab, gamma)), O._rot(z, 1))
    u = O.sub(u, O.mul(z, O.mul(inp, tab)))
    t = O.add(t, O.mul(u, la))
    t = O.mul(t, y)
    p = O.sub(pin, ptab)
    t = O.add(t, O.mul(l0, p))
    t = O.mul(t, y)
    u = O.mul(O.sub(pin, O._rot(pin, -1)), p)
    return O.add(t, O.mul(u, la))


@case("lookup_eval_h")
def _():
    def run(L, d, n):
        c, y, beta, gamma = inputs(n, SEED)
        res = d.put(O.rand_fr(n, SEED + 11))
        assert L.lookup_eval_h(P(res), *[P(d.put(x)) for x in c[:8]], P(d.put(y)), P(d.put(beta)),
                               P(d.put(gamma)), 1, n, None) == 0
        return {"res": d.get(res)}

    def expect(n):
        c, y, beta, gamma = inputs(n, SEED)
        return {"res": _lookup_expect(O.rand_fr(n, SEED + 11), c, y, beta, gamma)}
    return run, expect


# ---------------------------------------------------------------- small maps


def _zip_case(k):
    def run(L, d, n):
        c, *_ = inputs(n, SEED)
        buf = d.put(c[0])
        assert L.field_mul_zip(P(buf), P(d.put(c[1][:k])), k, n) == 0
        return {"buf": d.get(buf)}

    def expect(n):
        c, *_ = inputs(n, SEED)
        return {"buf": O.field_mul_zip(c[0], c[1][:k])}
    return run, expect


for _k in (3, 8):
    _run, _exp = _zip_case(_k)
    CASES.append(Case(f"field_mul_zip_{_k}", _run, _exp))


def _omegas(n):
    log_n = n.bit_length() - 1
    return O.expand_omega(O.omega(log_n), log_n)


@case("field_sum")
def _():
    rots = [0, 1, -1]

    def run(L, d, n):
        c, *_ = inputs(n, SEED)
        res = d.empty(n)
        vc = d.ptrs([d.put(c[3][:1]), None, d.put(c[4][:1])])
        assert L.field_sum(P(res), P(d.ptrs([d.put(x) for x in c[:3]])), P(vc), P(d.i32(rots)),
                           P(d.put(_omegas(n))), 3, n) == 0
        return {"res": d.get(res)}

    def expect(n):
        c, *_ = inputs(n, SEED)
        return {"res": O.field_sum(c[:3], [c[3][:1], None, c[4][:1]], rots, _omegas(n), n)}
    return run, expect


@case("shplonk_h_x_merge")
def _():
    def run(L, d, n):
        c, y, *_ = inputs(n, SEED)
        res = d.put(c[7])
        diffs = O.rand_fr(3, SEED + 12)
        assert L.shplonk_h_x_merge(P(res), P(d.put(y)), P(d.put(c[2])), P(d.put(_omegas(n))), P(d.put(diffs)), 3,
                                   n) == 0
        return {"res": d.get(res)}

    def expect(n):
        c, y, *_ = inputs(n, SEED)
        return {"res": O.shplonk_h_x_merge(c[7], y, c[2], _omegas(n), O.rand_fr(3, SEED + 12))}
    return run, expect


@case("shplonk_h_x_div_points")
def _():
    def run(L, d, n):
        c, *_ = inputs(n, SEED)
        vals = d.put(c[5])
        assert L.shplonk_h_x_div_points(P(vals), P(d.put(_omegas(n))), P(d.put(O.rand_fr(4, SEED + 13))), 4, n) == 0
        return {"values": d.get(vals)}

    def expect(n):
        c, *_ = inputs(n, SEED)
        return {"values": O.shplonk_h_x_div_points(c[5], _omegas(n), O.rand_fr(4, SEED + 13))}
    return run, expect


@case("poly_eval")
def _():
    def xt(n):
        x = O.fr_ints(O.rand_fr(1, SEED + 14))[0]
        return x, O.fr_vec([pow(x, 1 << dd, O.R_MOD) for dd in range(max(1, n.bit_length() - 1))])

    def run(L, d, n):
        c, *_ = inputs(n, SEED)
        res = d.empty(n)
        assert L.poly_eval(P(d.put(c[0])), P(res), P(d.put(xt(n)[1])), n, None) == 0
        return {"eval": d.get(res)[:1]}

    def expect(n):
        c, *_ = inputs(n, SEED)
        return {"eval": O.fr_vec([O.poly_eval(c[0], xt(n)[0])])}
    return run, expect


def _coset_powers(to_coset):
    z = ZETA
    zi = pow(ZETA, -1, O.R_MOD)
    # src/eval_h.rs:620-623 ([g_coset, g_coset_inv]) and :507-510 ([g_coset_inv, g_coset])
    return O.fr_vec([zi, z] if to_coset else [z, zi])


def _prep_case(to_coset):
    def run(L, d, n):
        s = d.put(O.rand_fr(4 * n, SEED + 15))
        assert L.extended_prepare(P(s), P(d.put(_coset_powers(to_coset))), 3, n, 4 * n, int(to_coset), None) == 0
        return {"s": d.get(s)}

    def expect(n):
        return {"s": O.extended_prepare(O.rand_fr(4 * n, SEED + 15), _coset_powers(to_coset), 3, n, 4 * n,
                                        to_coset)}
    return run, expect


for _tc in (False, True):
    _run, _exp = _prep_case(_tc)
    CASES.append(Case(f"extended_prepare_to_coset{int(_tc)}", _run, _exp))


@case("expand_omega_buffer")
def _():
    def run(L, d, n):
        log_n = n.bit_length() - 1
        buf = d.zeros(n)
        buf[:2].copy_(d.put(O.fr_vec([1, O.omega(log_n)])))
        d.torch.cuda.synchronize()
        assert L.expand_omega_buffer(P(buf), log_n, 0) == 0
        return {"buf": d.get(buf)}

    def expect(n):
        return {"buf": _omegas(n)}
    return run, expect


# ---------------------------------------------------------------- lookup multiplicity, logup scans


def _m_inputs(n):
    rng = np.random.default_rng(SEED + 16)
    u = n - 9
    table = rng.integers(0, 300, n)  # duplicates on purpose
    present = np.unique(table[:u])
    inp = [rng.choice(present, n) for _ in range(2)]
    return table, inp, u


@case("calc_m")
def _():
    def run(L, d, n):
        import torch

        table, inp, u = _m_inputs(n)
        k = n.bit_length() - 1
        dt = d.put(O.fr_vec(table.tolist()))
        words = [torch.empty(n * 8, dtype=torch.int32, device="cuda") for _ in range(6)]
        d.keep.extend(words)
        m = d.zeros(n)
        assert L.prepare_table_lookup(P(dt), P(words[0]), P(words[1]), P(words[2]), P(words[3]), P(words[4]),
                                      P(words[5]), n * 32, k, u, None) == 0
        for x in inp:
            assert L.calc_m(P(m), P(dt), P(d.put(O.fr_vec(x.tolist()))), P(words[3]), P(words[4]), P(words[0]),
                            P(words[1]), P(words[5]), n * 32, k, u, None) == 0
        return {"m": d.get(m)}

    def expect(n):
        # each input row counts once at the largest usable table row holding its value
        table, inp, u = _m_inputs(n)
        last = {}
        for i in range(u):
            last[int(table[i])] = i
        m = [0] * n
        for x in inp:
            for v in x[:u]:
                m[last[int(v)]] += 1
        return {"m": O.fr_vec(m)}
    return run, expect


@case("logup_sum_input_inv", min_n=1 << 15)
def _():
    def run(L, d, n):
        c, _, beta, _ = inputs(n, SEED)
        s = d.zeros(n)
        tmp = d.empty(n)
        assert L.logup_sum_input_inv(P(s), P(d.put(c[0])), P(tmp), P(d.put(beta)), 0, n, None) == 0
        assert L.logup_sum_input_inv(P(s), P(d.put(c[1])), P(tmp), P(d.put(beta)), 1, n, None) == 0
        return {"sum": d.get(s)}

    def expect(n):
        c, _, beta, _ = inputs(n, SEED)
        b = O.fr_ints(beta)[0]
        s = O.logup_sum_input_inv(None, c[0], b, 0)
        return {"sum": O.logup_sum_input_inv(s, c[1], b, 1)}
    return run, expect


@case("eval_logup_z_compose_then_pure", min_n=1 << 14)
def _():
    def run(L, d, n):
        c, _, beta, _ = inputs(n, SEED)
        m = O.fr_vec([i % 5 for i in range(n)])
        z, z2 = d.empty(n), d.empty(n)
        last = d.zeros(1)
        s1 = d.put(c[0])
        assert L.eval_logup_z_compose(P(z), P(s1), P(d.put(c[1])), P(d.put(m)), P(d.put(beta)), P(last), n - 17, n,
                                      None) == 0
        z2.copy_(d.put(c[2]))
        assert L.eval_logup_z_pure(P(z2), P(d.empty(n)), P(d.empty(n)), P(last), n - 17, n, None) == 0
        return {"z": d.get(z), "z_pure": d.get(z2), "last_z": d.get(last)}

    def expect(n):
        c, _, beta, _ = inputs(n, SEED)
        m = O.fr_vec([i % 5 for i in range(n)])
        z, last = O.eval_logup_z_compose(c[0], c[1], m, O.fr_ints(beta)[0], n - 17)
        z2, last2 = O.eval_logup_z_pure(c[2], n - 17, last)
        return {"z": z, "z_pure": z2, "last_z": last2}
    return run, expect


def cases_for(n):
    return [c for c in CASES if n >= c.min_n]
