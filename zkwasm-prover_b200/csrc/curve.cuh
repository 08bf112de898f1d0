// BN254 G1 (y^2 = x^3 + 3 over Fq) for the MSM.
//
// Storage formats shared with the Rust host (reference: src/cuda/msm.rs:441-452,
// cuda/zprize/ec.cuh:142):
//   affine   (x, y)      64 B, identity encoded as (0, 0)
//   Jacobian (X, Y, Z)   96 B, x = X/Z^2, y = Y/Z^3, identity Z = 0
// Bucket arithmetic uses extended Jacobian "XYZZ" coordinates
// (X, Y, ZZ, ZZZ) with x = X/ZZ, y = Y/ZZZ, ZZ^3 = ZZZ^2, identity ZZ = 0.
// Formulas follow the Explicit-Formulas Database for short Weierstrass a = 0:
//   madd-2008-s   XYZZ + affine       8M + 2S
//   mdbl-2008-s-1 2 * affine          2M + 3S (as the equal-points case)
//   add-2008-s    XYZZ + XYZZ        12M + 2S
//   dbl-2008-s-1  2 * XYZZ            6M + 3S
#pragma once
#include "field.cuh"

namespace zk {

// Fq product used by the point formulas.  On the device it is one
// out-of-line function: a mixed addition alone is ten products of ~350
// instructions each, and inlining every product of the accumulation loop
// overflows the instruction cache.
// cmul_lazy leaves out the final subtraction: for inputs below 2p the result
// is below 2p and congruent to the product (4p < 2^256).
#if defined(__CUDA_ARCH__)
#if defined(ZK_CURVE_INLINE_MUL)
__device__ __forceinline__ Fq cmul(const Fq& a, const Fq& b) { return fe_mul<FqCfg>(a, b); }
__device__ __forceinline__ Fq cmul_lazy(const Fq& a, const Fq& b) { return fe_mul_lazy<FqCfg>(a, b); }
#else
__device__ __noinline__ Fq cmul(const Fq a, const Fq b) { return fe_mul<FqCfg>(a, b); }
__device__ __noinline__ Fq cmul_lazy(const Fq a, const Fq b) { return fe_mul_lazy<FqCfg>(a, b); }
#endif
#else
inline Fq cmul(const Fq& a, const Fq& b) { return fe_mul<FqCfg>(a, b); }
inline Fq cmul_lazy(const Fq& a, const Fq& b) { return fe_mul_lazy<FqCfg>(a, b); }
#endif

struct Aff {
    Fq x, y;
};

struct Xyzz {
    Fq x, y, zz, zzz;
};

struct Jac {
    Fq x, y, z;
};

ZK_HD Xyzz xyzz_identity() {
    Xyzz r;
    r.x = fe_zero<FqCfg>();
    r.y = fe_zero<FqCfg>();
    r.zz = fe_zero<FqCfg>();
    r.zzz = fe_zero<FqCfg>();
    return r;
}

ZK_HD bool xyzz_is_id(const Xyzz& p) { return fe_is_zero<FqCfg>(p.zz); }
ZK_HD bool aff_is_id(const Aff& p) { return fe_is_zero<FqCfg>(p.x) && fe_is_zero<FqCfg>(p.y); }

ZK_HD Xyzz xyzz_from_aff(const Aff& a) {
    if (aff_is_id(a)) return xyzz_identity();
    Xyzz r;
    r.x = a.x;
    r.y = a.y;
    r.zz = fe_one<FqCfg>();
    r.zzz = fe_one<FqCfg>();
    return r;
}

// Product policies for the point formulas: CurveMul calls cmul (out of line
// on the device), CurveMulInline expands every product in place, for
// single-thread latency-bound code where the compiler should overlap the
// independent products of one formula.
struct CurveMul {
    static ZK_HD Fq mul(const Fq& a, const Fq& b) { return cmul(a, b); }
    static ZK_HD Fq mul_lazy(const Fq& a, const Fq& b) { return cmul_lazy(a, b); }
};
struct CurveMulInline {
    static ZK_HD Fq mul(const Fq& a, const Fq& b) { return fe_mul<FqCfg>(a, b); }
    static ZK_HD Fq mul_lazy(const Fq& a, const Fq& b) { return fe_mul_lazy<FqCfg>(a, b); }
};

// 2 * (x, y) for affine (x, y), as XYZZ (mdbl-2008-s-1)
template <class M = CurveMul>
ZK_HD Xyzz aff_dbl(const Fq& x, const Fq& y) {
    Fq u = fe_dbl<FqCfg>(y);
    Fq v = M::mul(u, u);
    Fq w = M::mul(u, v);
    Fq s = M::mul(x, v);
    Fq xx = M::mul(x, x);
    Fq mm = fe_add<FqCfg>(fe_dbl<FqCfg>(xx), xx);
    Xyzz r;
    r.x = fe_sub<FqCfg>(fe_sub<FqCfg>(M::mul(mm, mm), s), s);
    r.y = fe_sub<FqCfg>(M::mul(mm, fe_sub<FqCfg>(s, r.x)), M::mul(w, y));
    r.zz = v;
    r.zzz = w;
    return r;
}

// 2 * p (dbl-2008-s-1)
template <class M = CurveMul>
ZK_HD Xyzz xyzz_dbl(const Xyzz& p) {
    if (xyzz_is_id(p)) return p;
    Fq u = fe_dbl<FqCfg>(p.y);
    Fq v = M::mul(u, u);
    Fq w = M::mul(u, v);
    Fq s = M::mul(p.x, v);
    Fq xx = M::mul(p.x, p.x);
    Fq mm = fe_add<FqCfg>(fe_dbl<FqCfg>(xx), xx);
    Xyzz r;
    r.x = fe_sub<FqCfg>(fe_sub<FqCfg>(M::mul(mm, mm), s), s);
    r.y = fe_sub<FqCfg>(M::mul(mm, fe_sub<FqCfg>(s, r.x)), M::mul(w, p.y));
    r.zz = M::mul(v, p.zz);
    r.zzz = M::mul(w, p.zzz);
    return r;
}

// p + (x2, y2) with (x2, y2) affine and not the identity (madd-2008-s)
template <class M = CurveMul>
ZK_HD Xyzz xyzz_add_aff(const Xyzz& p, const Fq& x2, const Fq& y2) {
    if (xyzz_is_id(p)) {
        Xyzz r;
        r.x = x2;
        r.y = y2;
        r.zz = fe_one<FqCfg>();
        r.zzz = fe_one<FqCfg>();
        return r;
    }
    Fq u2 = M::mul(x2, p.zz);
    Fq s2 = M::mul(y2, p.zzz);
    Fq pp_ = fe_sub<FqCfg>(u2, p.x);
    Fq rr = fe_sub<FqCfg>(s2, p.y);
    if (fe_is_zero<FqCfg>(pp_)) {
        if (fe_is_zero<FqCfg>(rr)) return aff_dbl<M>(x2, y2);
        return xyzz_identity();
    }
    Fq pp = M::mul(pp_, pp_);
    Fq ppp = M::mul(pp_, pp);
    Fq q = M::mul(p.x, pp);
    Xyzz r;
    r.x = fe_sub<FqCfg>(fe_sub<FqCfg>(fe_sub<FqCfg>(M::mul(rr, rr), ppp), q), q);
    r.y = fe_sub<FqCfg>(M::mul(rr, fe_sub<FqCfg>(q, r.x)), M::mul(p.y, ppp));
    r.zz = M::mul(p.zz, pp);
    r.zzz = M::mul(p.zzz, ppp);
    return r;
}

// madd-2008-s on lazily reduced coordinates: p's coordinates lie in [0, 2p)
// (congruent to the exact ones), (x2, y2) is canonical and not the identity,
// and so are the result's coordinates.  Products skip their final subtraction
// and sums and differences work modulo 2p; the equal-x test reduces first.
// A non-identity p never has zz = 0 mod p, so the identity stays zz = 0.
template <class M = CurveMul>
ZK_HD Xyzz xyzz_add_aff_lazy(const Xyzz& p, const Fq& x2, const Fq& y2) {
    if (xyzz_is_id(p)) {
        Xyzz r;
        r.x = x2;
        r.y = y2;
        r.zz = fe_one<FqCfg>();
        r.zzz = fe_one<FqCfg>();
        return r;
    }
    Fq u2 = M::mul_lazy(x2, p.zz);
    Fq s2 = M::mul_lazy(y2, p.zzz);
    Fq pp_ = fe_sub_lazy<FqCfg>(u2, p.x);
    Fq rr = fe_sub_lazy<FqCfg>(s2, p.y);
    if (fe_is_zero<FqCfg>(fe_canon<FqCfg>(pp_))) {
        if (fe_is_zero<FqCfg>(fe_canon<FqCfg>(rr))) return aff_dbl<M>(x2, y2);
        return xyzz_identity();
    }
    Fq pp = M::mul_lazy(pp_, pp_);
    Fq ppp = M::mul_lazy(pp_, pp);
    Fq q = M::mul_lazy(p.x, pp);
    Xyzz r;
    r.x = fe_sub_lazy<FqCfg>(fe_sub_lazy<FqCfg>(fe_sub_lazy<FqCfg>(M::mul_lazy(rr, rr), ppp), q), q);
    r.y = fe_sub_lazy<FqCfg>(M::mul_lazy(rr, fe_sub_lazy<FqCfg>(q, r.x)), M::mul_lazy(p.y, ppp));
    r.zz = M::mul_lazy(p.zz, pp);
    r.zzz = M::mul_lazy(p.zzz, ppp);
    return r;
}

// canonical coordinates of a lazily reduced point
ZK_HD Xyzz xyzz_canon(const Xyzz& p) {
    Xyzz r;
    r.x = fe_canon<FqCfg>(p.x);
    r.y = fe_canon<FqCfg>(p.y);
    r.zz = fe_canon<FqCfg>(p.zz);
    r.zzz = fe_canon<FqCfg>(p.zzz);
    return r;
}

// p + q (add-2008-s)
template <class M = CurveMul>
ZK_HD Xyzz xyzz_add(const Xyzz& p, const Xyzz& q) {
    if (xyzz_is_id(p)) return q;
    if (xyzz_is_id(q)) return p;
    Fq u1 = M::mul(p.x, q.zz);
    Fq u2 = M::mul(q.x, p.zz);
    Fq s1 = M::mul(p.y, q.zzz);
    Fq s2 = M::mul(q.y, p.zzz);
    Fq pp_ = fe_sub<FqCfg>(u2, u1);
    Fq rr = fe_sub<FqCfg>(s2, s1);
    if (fe_is_zero<FqCfg>(pp_)) {
        if (fe_is_zero<FqCfg>(rr)) return xyzz_dbl<M>(p);
        return xyzz_identity();
    }
    Fq pp = M::mul(pp_, pp_);
    Fq ppp = M::mul(pp_, pp);
    Fq qq = M::mul(u1, pp);
    Xyzz r;
    r.x = fe_sub<FqCfg>(fe_sub<FqCfg>(fe_sub<FqCfg>(M::mul(rr, rr), ppp), qq), qq);
    r.y = fe_sub<FqCfg>(M::mul(rr, fe_sub<FqCfg>(qq, r.x)), M::mul(s1, ppp));
    r.zz = M::mul(M::mul(p.zz, q.zz), pp);
    r.zzz = M::mul(M::mul(p.zzz, q.zzz), ppp);
    return r;
}

// [k] p for a small unsigned k (double-and-add from the top bit)
template <class M = CurveMul>
ZK_HD Xyzz xyzz_mul_u32(const Xyzz& p, uint32_t k) {
    Xyzz r = xyzz_identity();
    if (k == 0 || xyzz_is_id(p)) return r;
    int top = 31;
    while (!((k >> top) & 1)) top--;
    r = p;
    for (int b = top - 1; b >= 0; b--) {
        r = xyzz_dbl<M>(r);
        if ((k >> b) & 1) r = xyzz_add<M>(r, p);
    }
    return r;
}

// XYZZ -> Jacobian without an inversion: with ZZ = z^2, ZZZ = z^3 the point
// (X * ZZ^2, Y * ZZ^3, ZZZ) has X'/Z'^2 = X/ZZ and Y'/Z'^3 = Y/ZZZ.
// The identity becomes (0, 1, 0), halo2's Jacobian identity.
template <class M = CurveMul>
ZK_HD Jac xyzz_to_jac(const Xyzz& p) {
    Jac r;
    if (xyzz_is_id(p)) {
        r.x = fe_zero<FqCfg>();
        r.y = fe_one<FqCfg>();
        r.z = fe_zero<FqCfg>();
        return r;
    }
    Fq zz2 = M::mul(p.zz, p.zz);
    Fq zz3 = M::mul(zz2, p.zz);
    r.x = M::mul(p.x, zz2);
    r.y = M::mul(p.y, zz3);
    r.z = p.zzz;
    return r;
}

// Signed c-bit window digit of a canonical scalar, least significant window
// first: d = bits + carry, and digits above 2^(c-1) become d - 2^c with a carry
// into the next window.  Digits lie in [-(2^(c-1)-1), 2^(c-1)], so a window
// needs 2^(c-1) buckets; for scalars below 2^254 and 4 <= c <= 22 the
// ceil(254/c) windows absorb the final carry.
ZK_HD int msm_signed_digit(const uint32_t k[8], int w, int c, uint32_t& carry) {
    uint32_t d = bits_at(k, (uint32_t)(w * c), (uint32_t)c) + carry;
    const uint32_t half = 1u << (c - 1);
    if (d > half) {
        carry = 1;
        return (int)d - (int)(1u << c);
    }
    carry = 0;
    return (int)d;
}

}  // namespace zk
