"""CPU oracle for the BN254 KZG proving hot path (test infrastructure only).

Only ``tests/``, ``__graft_entry__.smoke()`` and the ``cpu_baseline`` leg of
``bench.py`` import this module.  The product library never does.

Layout conventions (identical to halo2 / the reference's device buffers):

* an Fr or Fq element is 4 little-endian u64 limbs in Montgomery form
  (R = 2^256); arrays are numpy ``uint64`` of shape ``(n, 4)``;
* a G1 affine point is ``(x, y)``, 8 limbs, identity ``(0, 0)``;
* a G1 Jacobian point is ``(X, Y, Z)``, 12 limbs, identity ``Z = 0``
  (reference: cuda/zprize/ec.cuh:142, read back as ``C::Curve`` at
  src/cuda/msm.rs:441-452).

Every formula below cites the reference line it restates.  The field and
group primitives come from ``bn254_oracle.c`` (built by ``oracle/Makefile``);
``pyint_*`` helpers restate the same maths with Python integers and pin the C
code on small cases.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle_bn254.so")

# Public BN254 parameters.
R_MOD = 0x30644E72E131A029B85045B68181585D2833E84879B9709143E1F593F0000001
Q_MOD = 0x30644E72E131A029B85045B68181585D97816A916871CA8D3C208C16D87CFD47
TWO_ADICITY = 28
GENERATOR = 7
MONT_R = 1 << 256

_lib = None


def lib():
    """Load (building if needed) the C oracle."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        subprocess.check_call(["make", "-s", "-C", HERE])
    L = ctypes.CDLL(LIB_PATH)
    P = ctypes.c_void_p
    i64 = ctypes.c_long
    ci = ctypes.c_int
    sig = {
        "or_init": [],
        "or_field_consts": [ci, P, P, P, P],
        "or_vec_add": [ci, P, P, P, i64],
        "or_vec_sub": [ci, P, P, P, i64],
        "or_vec_mul": [ci, P, P, P, i64],
        "or_vec_mul_scalar": [ci, P, P, P, i64],
        "or_vec_neg": [ci, P, P, i64],
        "or_vec_to_mont": [ci, P, P, i64],
        "or_vec_from_mont": [ci, P, P, i64],
        "or_vec_inv": [ci, P, P, i64],
        "or_pow": [ci, P, P, P],
        "or_batch_inv": [P, P, i64],
        "or_prefix_product_excl": [P, P, P, i64],
        "or_prefix_sum_excl": [P, P, P, i64],
        "or_ntt": [P, ci, P],
        "or_intt": [P, ci, P],
        "or_dft_naive": [P, P, ci, P],
        "or_powers": [P, P, i64],
        "or_poly_divide_linear": [P, P, i64],
        "or_coset_extend": [P, P, ci, ci, P, P],
        "or_g1_generator": [P],
        "or_g1_is_on_curve": [P],
        "or_g1_jac_to_aff": [P, P, i64],
        "or_g1_add_jac": [P, P, P],
        "or_g1_dbl_jac": [P, P],
        "or_g1_mul_aff": [P, P, P],
        "or_g1_gen_bases": [P, P, i64],
        "or_msm": [P, P, P, i64, ci],
        "or_inner_product": [P, P, P, i64],
        "or_rand_fr": [P, i64, ctypes.c_uint64],
    }
    for name, args in sig.items():
        fn = getattr(L, name)
        fn.argtypes = args
        fn.restype = ctypes.c_int if name == "or_g1_is_on_curve" else None
    L.or_init()
    _lib = L
    return L


def _p(a: np.ndarray):
    assert a.dtype == np.uint64 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data


def _arr(a) -> np.ndarray:
    return np.ascontiguousarray(np.asarray(a, dtype=np.uint64).reshape(-1, 4))


# ----------------------------------------------------------------------------
# integer <-> limb conversion

def int_to_limbs(x: int) -> np.ndarray:
    return np.array([(x >> (64 * i)) & 0xFFFFFFFFFFFFFFFF for i in range(4)], dtype=np.uint64)


def limbs_to_int(a) -> int:
    a = np.asarray(a, dtype=np.uint64).reshape(-1)
    return sum(int(a[i]) << (64 * i) for i in range(4))


def fr(x: int) -> np.ndarray:
    """Python int -> Montgomery-form Fr element, shape (1, 4)."""
    return int_to_limbs((x % R_MOD) * MONT_R % R_MOD).reshape(1, 4)


def fq(x: int) -> np.ndarray:
    return int_to_limbs((x % Q_MOD) * MONT_R % Q_MOD).reshape(1, 4)


def fr_vec(xs) -> np.ndarray:
    return np.concatenate([fr(int(x)) for x in xs], axis=0) if len(xs) else np.zeros((0, 4), np.uint64)


def fr_ints(a) -> list:
    """Montgomery-form array -> list of canonical ints."""
    a = _arr(a)
    rinv = pow(MONT_R, -1, R_MOD)
    return [limbs_to_int(a[i]) * rinv % R_MOD for i in range(a.shape[0])]


def fq_ints(a) -> list:
    a = _arr(a)
    rinv = pow(MONT_R, -1, Q_MOD)
    return [limbs_to_int(a[i]) * rinv % Q_MOD for i in range(a.shape[0])]


# ----------------------------------------------------------------------------
# field constants derived from the public parameters

def root_of_unity() -> int:
    """GENERATOR^((r-1)/2^S): the 2^28-th root of unity halo2 uses for Fr."""
    return pow(GENERATOR, (R_MOD - 1) >> TWO_ADICITY, R_MOD)


def omega(log_n: int) -> int:
    """Primitive 2^log_n-th root of unity, as the reference derives it
    (src/profile.rs:193-196: square ROOT_OF_UNITY (S - k) times)."""
    w = root_of_unity()
    for _ in range(log_n, TWO_ADICITY):
        w = w * w % R_MOD
    return w


# GLV endomorphism of G1 (Gallant, Lambert, Vanstone, CRYPTO 2001), used by
# the library's MSM; the reference has no counterpart (its MSM runs on the
# full 254-bit scalars), so this restates the published method: beta and
# lambda are the cube roots of unity mod p and mod r with
# (beta x, y) = [lambda] (x, y), the short lattice basis comes from the
# extended Euclidean algorithm on (r, lambda) stopped at sqrt(r), and
# c_i = floor(k g_i / 2^256) with g1 = round(b2 2^256 / r), g2 = round(-b1 2^256 / r).
GLV_LAMBDA = 0x30644E72E131A029048B6E193FD84104CC37A73FEC2BC5E9B8CA0B2D36636F23
GLV_BETA = 0x30644E72E131A0295E6DD9E7E0ACCCB0C28F069FBB966E3DE4BD44E5607CFD48


def _glv_basis():
    import math

    r0, t0, r1, t1 = R_MOD, 0, GLV_LAMBDA, 1
    seq = [(r0, t0), (r1, t1)]
    while r1:
        q = r0 // r1
        r0, r1 = r1, r0 - q * r1
        t0, t1 = t1, t0 - q * t1
        seq.append((r1, t1))
    i = max(j for j, (rj, _) in enumerate(seq) if rj >= math.isqrt(R_MOD))
    v1 = (seq[i + 1][0], -seq[i + 1][1])
    v2 = min([(seq[i][0], -seq[i][1]), (seq[i + 2][0], -seq[i + 2][1])], key=lambda v: v[0] ** 2 + v[1] ** 2)
    return v1 + v2


GLV_A1, GLV_B1, GLV_A2, GLV_B2 = _glv_basis()
GLV_G1 = ((GLV_B2 << 256) + R_MOD // 2) // R_MOD
GLV_G2 = ((-GLV_B1 << 256) + R_MOD // 2) // R_MOD


def glv_split(k: int):
    """(k1, k2) with k = k1 + k2 lambda (mod r), |k1|, |k2| < 2^127."""
    c1 = (k * GLV_G1) >> 256
    c2 = (k * GLV_G2) >> 256
    return k - c1 * GLV_A1 - c2 * GLV_A2, -c1 * GLV_B1 - c2 * GLV_B2


def delta() -> int:
    """GENERATOR^(2^S), the permutation column-coset generator halo2 uses
    (src/permutation.rs:51, 94)."""
    return pow(GENERATOR, 1 << TWO_ADICITY, R_MOD)


def cube_roots_of_unity() -> tuple:
    """The two primitive cube roots of unity in Fr (halo2's ZETA is one of them;
    src/eval_h.rs:620-623 passes [zeta, zeta^-1] as coset powers)."""
    g = pow(GENERATOR, (R_MOD - 1) // 3, R_MOD)
    return tuple(sorted([g, g * g % R_MOD]))


# ----------------------------------------------------------------------------
# vector field arithmetic (Fr unless noted); scalars broadcast from shape (1, 4)

def _binop(name, a, b, which=0):
    a, b = _arr(a), _arr(b)
    n = max(a.shape[0], b.shape[0])
    out = np.empty((n, 4), np.uint64)
    if b.shape[0] == 1 and n > 1 and name == "or_vec_mul":
        lib().or_vec_mul_scalar(which, _p(out), _p(a), _p(b), n)
        return out
    if a.shape[0] == 1 and n > 1:
        a = np.ascontiguousarray(np.repeat(a, n, axis=0))
    if b.shape[0] == 1 and n > 1:
        b = np.ascontiguousarray(np.repeat(b, n, axis=0))
    getattr(lib(), name)(which, _p(out), _p(a), _p(b), n)
    return out


def add(a, b, which=0):
    return _binop("or_vec_add", a, b, which)


def sub(a, b, which=0):
    return _binop("or_vec_sub", a, b, which)


def mul(a, b, which=0):
    return _binop("or_vec_mul", a, b, which)


def sqr(a, which=0):
    return mul(a, a, which)


def neg(a, which=0):
    a = _arr(a)
    out = np.empty_like(a)
    lib().or_vec_neg(which, _p(out), _p(a), a.shape[0])
    return out


def inv(a, which=0):
    a = _arr(a)
    out = np.empty_like(a)
    lib().or_vec_inv(which, _p(out), _p(a), a.shape[0])
    return out


def to_mont(a_canonical, which=0):
    a = _arr(a_canonical)
    out = np.empty_like(a)
    lib().or_vec_to_mont(which, _p(out), _p(a), a.shape[0])
    return out


def from_mont(a, which=0):
    a = _arr(a)
    out = np.empty_like(a)
    lib().or_vec_from_mont(which, _p(out), _p(a), a.shape[0])
    return out


def one(n=1):
    return np.repeat(fr(1), n, axis=0)


def zeros(n):
    return np.zeros((n, 4), np.uint64)


def rand_fr(n: int, seed: int) -> np.ndarray:
    """Seeded uniform Fr elements (Montgomery form): splitmix64 + rejection."""
    out = np.empty((n, 4), np.uint64)
    lib().or_rand_fr(_p(out), n, seed & 0xFFFFFFFFFFFFFFFF)
    return out


def batch_inv(a):
    """Montgomery batch inversion; zero maps to zero."""
    a = _arr(a)
    out = np.empty_like(a)
    lib().or_batch_inv(_p(out), _p(a), a.shape[0])
    return out


def prefix_product_excl(a, init=None):
    a = _arr(a)
    out = np.empty_like(a)
    init = fr(1) if init is None else _arr(init)
    lib().or_prefix_product_excl(_p(out), _p(a), _p(init), a.shape[0])
    return out


def prefix_sum_excl(a, init=None):
    a = _arr(a)
    out = np.empty_like(a)
    init = zeros(1) if init is None else _arr(init)
    lib().or_prefix_sum_excl(_p(out), _p(a), _p(init), a.shape[0])
    return out


def pow_fr(a_int: int, e: int) -> int:
    return pow(a_int, e, R_MOD)


# ----------------------------------------------------------------------------
# NTT (reference: src/cuda/ntt.rs:36-93 -> cuda/bn254.cu:1357-1428)

def ntt(a, log_n: int, w: int | None = None):
    """Natural-order forward NTT by w (default omega(log_n)): X_j = sum x_i w^ij."""
    a = np.array(_arr(a), copy=True)
    assert a.shape[0] == 1 << log_n
    w = omega(log_n) if w is None else w
    wm = fr(w)  # keep the buffer alive across the call
    lib().or_ntt(_p(a), log_n, _p(wm))
    return a


def intt(a, log_n: int, w: int | None = None):
    """Inverse NTT: NTT by w^-1 then scale by n^-1 (the ``n_inv`` argument)."""
    a = np.array(_arr(a), copy=True)
    w = omega(log_n) if w is None else w
    wm = fr(w)
    lib().or_intt(_p(a), log_n, _p(wm))
    return a


def dft_naive(a, log_n: int, w: int):
    a = _arr(a)
    out = np.empty_like(a)
    wm = fr(w)
    lib().or_dft_naive(_p(out), _p(a), log_n, _p(wm))
    return out


def expand_omega(w: int, log_n: int):
    """Natural twiddle table w^i, i < 2^log_n (cuda/bn254.cu:1073-1093)."""
    n = 1 << log_n
    out = [1] * n
    for i in range(1, n):
        out[i] = out[i - 1] * w % R_MOD
    return fr_vec(out)


def extended_prepare(s, coset_powers, coset_powers_n: int, size: int, extended_size: int, to_coset: bool):
    """cuda/bn254.cu:1232-1253 with kernel 641-662.

    to_coset == False: zero s[size:extended_size], then s[i] *= coset_powers[i % cpn - 1]
    for i < size with i % cpn != 0.  to_coset == True: the same multiply over
    i < extended_size (used to undo the coset shift, src/eval_h.rs:507-510)."""
    s = np.array(_arr(s), copy=True)
    cp = _arr(coset_powers)
    if not to_coset:
        s[size:extended_size] = 0
        lim = size
    else:
        lim = extended_size
    idx = np.arange(lim)
    k = idx % coset_powers_n
    for j in range(1, coset_powers_n):
        sel = idx[k == j]
        if len(sel):
            s[sel] = mul(s[sel], cp[j - 1:j])
    return s


def coset_powers_table(shift: int, n: int):
    """shift^i for i < n (Montgomery)."""
    out = np.empty((n, 4), np.uint64)
    sm = fr(shift)
    lib().or_powers(_p(out), _p(sm), n)
    return out


def coset_ntt(coeffs, log_n: int, ext_log: int, shift: int):
    """Extended-domain evaluation: c_i * shift^i, zero pad to 2^ext_log, NTT.
    Output j is p(shift * w_N^j) with w_N = omega(ext_log)."""
    c = _arr(coeffs)
    n = 1 << log_n
    assert c.shape[0] == n
    out = np.empty((1 << ext_log, 4), np.uint64)
    sm, wm = fr(shift), fr(omega(ext_log))
    lib().or_coset_extend(_p(out), _p(c), log_n, ext_log - log_n, _p(sm), _p(wm))
    return out


# ----------------------------------------------------------------------------
# G1

def g1_generator():
    out = np.empty((1, 8), np.uint64)
    lib().or_g1_generator(out.ctypes.data)
    return out


def g1_gen_bases(dlogs):
    """P_i = [dlog_i] G as affine points (n, 8)."""
    d = _arr(dlogs)
    out = np.empty((d.shape[0], 8), np.uint64)
    lib().or_g1_gen_bases(out.ctypes.data, _p(d), d.shape[0])
    return out


def g1_mul(p_aff, k_mont):
    p = np.ascontiguousarray(np.asarray(p_aff, np.uint64).reshape(8))
    out = np.empty(8, np.uint64)
    k = _arr(k_mont)
    lib().or_g1_mul_aff(out.ctypes.data, p.ctypes.data, _p(k))
    return out.reshape(1, 8)


def g1_jac_to_aff(p_jac):
    p = np.ascontiguousarray(np.asarray(p_jac, np.uint64).reshape(-1, 12))
    out = np.empty((p.shape[0], 8), np.uint64)
    lib().or_g1_jac_to_aff(out.ctypes.data, p.ctypes.data, p.shape[0])
    return out


def g1_is_on_curve(p_aff) -> bool:
    p = np.ascontiguousarray(np.asarray(p_aff, np.uint64).reshape(8))
    return bool(lib().or_g1_is_on_curve(p.ctypes.data))


def msm(bases_aff, scalars, c: int = 0):
    """Pippenger MSM, affine result (1, 8)."""
    b = np.ascontiguousarray(np.asarray(bases_aff, np.uint64).reshape(-1, 8))
    s = _arr(scalars)
    assert b.shape[0] == s.shape[0]
    out = np.empty((1, 8), np.uint64)
    lib().or_msm(out.ctypes.data, b.ctypes.data, _p(s), s.shape[0], c)
    return out


def inner_product(a, b):
    a, b = _arr(a), _arr(b)
    out = np.empty((1, 4), np.uint64)
    lib().or_inner_product(_p(out), _p(a), _p(b), a.shape[0])
    return out


def msm_known_dlog(dlogs, scalars):
    """Known-discrete-log identity of src/cuda/msm.rs:501-512: with P_i = [d_i]G,
    MSM(P, a) = [sum a_i d_i] G.  O(n) and exact at any size."""
    return g1_mul(g1_generator(), inner_product(dlogs, scalars))


# ----------------------------------------------------------------------------
# pure-Python restatements for pinning the C oracle on small inputs

def pyint_ec_add(P, Q):
    """Affine addition over Fq with None as the identity."""
    if P is None:
        return Q
    if Q is None:
        return P
    (x1, y1), (x2, y2) = P, Q
    if x1 == x2:
        if (y1 + y2) % Q_MOD == 0:
            return None
        lam = 3 * x1 * x1 * pow(2 * y1, -1, Q_MOD) % Q_MOD
    else:
        lam = (y2 - y1) * pow(x2 - x1, -1, Q_MOD) % Q_MOD
    x3 = (lam * lam - x1 - x2) % Q_MOD
    return (x3, (lam * (x1 - x3) - y1) % Q_MOD)


def pyint_ec_mul(P, k):
    R = None
    while k:
        if k & 1:
            R = pyint_ec_add(R, P)
        P = pyint_ec_add(P, P)
        k >>= 1
    return R


def aff_to_pyint(p_aff):
    p = np.asarray(p_aff, np.uint64).reshape(8)
    x, y = fq_ints(p[:4])[0], fq_ints(p[4:])[0]
    return None if (x == 0 and y == 0) else (x, y)


def pyint_dft(xs, w):
    n = len(xs)
    return [sum(xs[i] * pow(w, i * j, R_MOD) for i in range(n)) % R_MOD for j in range(n)]


# ----------------------------------------------------------------------------
# grand products / sums (device scans in the product; CPU in the reference)

def permutation_product(columns, sigmas, beta: int, gamma: int, log_n: int,
                        chunk_len: int, unusable_rows_start: int):
    """src/permutation.rs:16-150 without the random tail: for each chunk of
    ``chunk_len`` permutation columns, z_j[0] = previous chunk's z at
    ``unusable_rows_start`` (1 for the first), and
    z_j[i+1] = z_j[i] * prod_c (v_c[i] + beta*delta^c*w^i + gamma) / (v_c[i] + beta*sigma_c[i] + gamma).
    Returns one (n, 4) array per chunk; rows after ``unusable_rows_start`` are
    left as the running product (the reference overwrites them with randomness)."""
    n = 1 << log_n
    w = omega(log_n)
    dlt = delta()
    ws = coset_powers_table(w, n)
    zs = []
    carry = fr(1)
    for ci in range(0, len(columns), chunk_len):
        cols = columns[ci:ci + chunk_len]
        sig = sigmas[ci:ci + chunk_len]
        den = None
        for v, s in zip(cols, sig):
            t = add(add(mul(_arr(s), fr(beta)), fr(gamma)), _arr(v))
            den = t if den is None else mul(den, t)
        den = batch_inv(den)
        dpow = pow(dlt, ci, R_MOD)
        num = den
        for v in cols:
            t = add(add(mul(ws, fr(dpow * beta % R_MOD)), fr(gamma)), _arr(v))
            num = mul(num, t)
            dpow = dpow * dlt % R_MOD
        z = prefix_product_excl(num, carry)
        zs.append(z)
        carry = z[unusable_rows_start:unusable_rows_start + 1].copy()
    return zs


def shuffle_product(inputs, tables, beta: int):
    """src/shuffle.rs:143-212 without the random tail: with beta_i = beta^(i+1),
    z[0] = 1, z[i+1] = z[i] * prod_g (input_g[i] + beta_g) / (table_g[i] + beta_g)."""
    n = _arr(inputs[0]).shape[0]
    den = None
    num = None
    for g, (a, s) in enumerate(zip(inputs, tables)):
        bg = fr(pow(beta, g + 1, R_MOD))
        t = add(_arr(s), bg)
        den = t if den is None else mul(den, t)
        u = add(_arr(a), bg)
        num = u if num is None else mul(num, u)
    return prefix_product_excl(mul(batch_inv(den), num), fr(1))


def logup_sum_input_inv(sum_prev, inp, beta: int, init: int):
    """cuda/bn254.cu:19-61 / 1914-1934: sum[i] (+)= 1 / (input[i] + beta)."""
    t = batch_inv(add(_arr(inp), fr(beta)))
    return t if init == 0 else add(sum_prev, t)


def eval_logup_z_compose(input_sum, table, multiplicity, beta: int,
                         last_z_index: int, init_z=None):
    """cuda/bn254.cu:1968-1993 -> 63-90, 212-220, 1936-1966.

    Returns (z, table_inv_tail, last_z): z = exclusive prefix sum of
    input_sum[i] - m[i] / (table[i] + beta) (z[0] = init_z, 0 when absent),
    last_z = z[last_z_index]."""
    tinv = batch_inv(add(_arr(table), fr(beta)))
    d = sub(_arr(input_sum), mul(tinv, _arr(multiplicity)))
    z = prefix_sum_excl(d, init_z)
    return z, z[last_z_index:last_z_index + 1].copy()


def eval_logup_z_pure(input_sum, last_z_index: int, init_z):
    """cuda/bn254.cu:1936-1966: z = exclusive prefix sum of input starting at
    init_z (the previous set's z at last_z_index); returns (z, last_z)."""
    z = prefix_sum_excl(_arr(input_sum), init_z)
    return z, z[last_z_index:last_z_index + 1].copy()


# ----------------------------------------------------------------------------
# quotient (eval_h) elementwise formulas, restated from cuda/bn254.cu

def _rot(a, r):
    """a[(i + r) mod n]"""
    return np.ascontiguousarray(np.roll(_arr(a), -r, axis=0))


def field_op(l, l_rot, l_c, r, r_rot, r_c, n, op):
    """cuda/bn254.cu:585-639: op 0 add, 1 mul, 2 copy of the left, 3 sub."""
    if l is not None:
        fl = _rot(l, l_rot)
        if l_c is not None:
            fl = mul(fl, l_c)
    else:
        fl = np.repeat(_arr(l_c), n, axis=0)
    fr_ = None
    if r is not None:
        fr_ = _rot(r, r_rot)
        if r_c is not None:
            fr_ = mul(fr_, r_c)
    elif r_c is not None:
        fr_ = np.repeat(_arr(r_c), n, axis=0)
    if op == 0:
        return add(fl, fr_)
    if op == 1:
        return mul(fl, fr_)
    if op == 2:
        return fl
    if op == 3:
        return sub(fl, fr_)
    raise ValueError("bad op")


def field_op_batch_mul_sum(res, terms, n):
    """cuda/bn254.cu:542-572: res[i] += sum_t coeff_t * prod_j v_tj[(i + rot_tj) mod n].
    ``terms`` is a list of (coeff (1,4), [(column, rot), ...])."""
    acc = zeros(n)
    for coeff, factors in terms:
        t = np.repeat(_arr(coeff), n, axis=0)
        for col, rot in factors:
            t = mul(t, _rot(col, rot))
        acc = add(acc, t)
    return add(res, acc)


def permutation_eval_h_p1(res, first_set, last_set, l0, l_last, y):
    """cuda/bn254.cu:664-699."""
    t1 = mul(res, y)
    t1 = add(t1, mul(sub(one(1), first_set), l0))
    t1 = mul(t1, y)
    t2 = mul(sub(sqr(last_set), last_set), l_last)
    return add(t1, t2)


def permutation_eval_h_p2(res, sets, l0, l_last, y, rot):
    """cuda/bn254.cu:701-733 (also logup_eval_h_z_set, 1518-1541)."""
    t1 = _arr(res)
    for j in range(1, len(sets)):
        t1 = mul(t1, y)
        t1 = add(t1, mul(sub(sets[j], _rot(sets[j - 1], rot)), l0))
    return t1


def permutation_eval_h_l(res, beta, gamma, p):
    """cuda/bn254.cu:735-765: res[i] += p[i]*beta (+ gamma at i == 0)."""
    t = mul(p, beta)
    t[0:1] = add(t[0:1], gamma)
    return add(res, t)


def logup_eval_h(res, input_product, input_product_sum, table, multiplicity,
                 z_first, z_last, l0, l_last, l_active_row, y, rot):
    """cuda/bn254.cu:867-921."""
    t = mul(res, y)
    t = add(t, mul(l0, z_first))
    t = mul(t, y)
    t = add(t, mul(l_last, z_last))
    t = mul(t, y)
    u = sub(_rot(z_first, rot), z_first)
    u = mul(u, table)
    u = add(u, multiplicity)
    u = mul(u, input_product)
    p = mul(table, input_product_sum)
    u = sub(u, p)
    u = mul(u, l_active_row)
    return add(t, u)


def logup_eval_h_extra_inputs(res, input_product, input_product_sum, z, l_active_row, y, rot):
    """cuda/bn254.cu:924-948."""
    t = mul(res, y)
    u = sub(_rot(z, rot), z)
    u = mul(u, input_product)
    u = sub(u, input_product_sum)
    u = mul(u, l_active_row)
    return add(t, u)


def logup_eval_h_inputs_product_sum(sets):
    """cuda/bn254.cu:1172-1213: product and leave-one-out sum of products."""
    k = len(sets)
    n = _arr(sets[0]).shape[0]
    prod = one(n)
    for s in sets:
        prod = mul(prod, s)
    tot = zeros(n)
    for j in range(k):
        u = one(n)
        for kk in range(k):
            if kk != j:
                u = mul(u, sets[kk])
        tot = add(tot, u)
    return prod, tot


def shuffle_eval_h(res, inp, table, z, l0, l_last, l_active_row, y, rot):
    """cuda/bn254.cu:975-1015."""
    t = mul(res, y)
    t = add(t, mul(l0, sub(one(1), z)))
    t = mul(t, y)
    t = add(t, mul(l_last, sub(sqr(z), z)))
    t = mul(t, y)
    u = sub(mul(table, _rot(z, rot)), mul(inp, z))
    return add(t, mul(u, l_active_row))


def shuffle_eval_h_v2(res, inputs, tables, betas, z, l0, l_last, l_active_row, y, rot):
    """cuda/bn254.cu:1017-1071: l = prod (input_j + beta_j), r = prod (table_j + beta_j)."""
    betas = _arr(betas)
    l = add(inputs[0], betas[0:1])
    r = add(tables[0], betas[0:1])
    for j in range(1, len(inputs)):
        l = mul(l, add(inputs[j], betas[j:j + 1]))
        r = mul(r, add(tables[j], betas[j:j + 1]))
    t = mul(res, y)
    t = add(t, mul(l0, sub(one(1), z)))
    t = mul(t, y)
    t = add(t, mul(l_last, sub(sqr(z), z)))
    t = mul(t, y)
    u = sub(mul(r, _rot(z, rot)), mul(l, z))
    return add(t, mul(u, l_active_row))


def field_mul_zip(buf, coeff):
    """cuda/bn254.cu:1121-1131: buf[i] *= coeff[i mod len(coeff)]."""
    b = _arr(buf)
    c = _arr(coeff)
    idx = np.arange(b.shape[0]) % c.shape[0]
    return mul(b, np.ascontiguousarray(c[idx]))


def field_sum(vs, v_cs, v_rots, omegas, n):
    """cuda/bn254.cu:496-540: res[i] = sum_j v_j[i] * omegas[((n + rot_j) * i) & (n-1)] (* c_j)."""
    om = _arr(omegas)
    i = np.arange(n)
    acc = None
    for v, c, rot in zip(vs, v_cs, v_rots):
        e = ((n + rot) * i) & (n - 1)
        t = mul(v, np.ascontiguousarray(om[e]))
        if c is not None:
            t = mul(t, c)
        acc = t if acc is None else add(acc, t)
    return acc


def poly_divide_linear(a, z: int):
    """src/multiopen.rs:145-159: the quotient of a(X) - a(z) by X - z with the
    reference's layout (last coefficient 0), by its own recurrence."""
    out = np.array(_arr(a), copy=True)
    lib().or_poly_divide_linear(_p(out), _p(fr(z)), out.shape[0])
    return out


def poly_eval(p, x: int):
    """Horner evaluation of the coefficient vector p at x (cuda/bn254.cu:1608-1634
    leaves the value at res[0])."""
    vals = fr_ints(p)
    acc = 0
    for c in reversed(vals):
        acc = (acc * x + c) % R_MOD
    return acc


def shplonk_h_x_merge(res, v, values, omegas, diff_points):
    """cuda/bn254.cu:1133-1149: res[i] = res[i]*v + values[i] * prod_j (omegas[i] - d_j)."""
    t = _arr(values)
    for j in range(_arr(diff_points).shape[0]):
        t = mul(t, sub(omegas, _arr(diff_points)[j:j + 1]))
    return add(mul(res, v), t)


def shplonk_h_x_div_points(values, omegas, points):
    """cuda/bn254.cu:1151-1170: values[i] /= prod_j (omegas[i] - p_j)."""
    pts = _arr(points)
    t = sub(omegas, pts[0:1])
    for j in range(1, pts.shape[0]):
        t = mul(t, sub(omegas, pts[j:j + 1]))
    return mul(values, batch_inv(t))
