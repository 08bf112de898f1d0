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

// Independent products of one formula step in one call, so the scheduler
// interleaves their carry chains: the point-formula kernels run at 16 warps
// per SM or fewer and are bound by instruction latency, and a call per product
// serialises them (3.6% of a 2^22 MSM).  LAZY: results in [0, 2p) without the
// final subtraction, else canonical.
struct Fq2 {
    Fq a, b;
};
struct Fq3 {
    Fq a, b, c;
};
struct Fq4 {
    Fq a, b, c, d;
};
template <bool LAZY>
ZK_HD Fq fmul(const Fq& a, const Fq& b) {
    return LAZY ? fe_mul_lazy<FqCfg>(a, b) : fe_mul<FqCfg>(a, b);
}
#if defined(__CUDA_ARCH__) && !defined(ZK_CURVE_INLINE_MUL)
#define ZK_CMUL __device__ __noinline__
#else
#define ZK_CMUL ZK_HD
#endif
template <bool LAZY>
ZK_CMUL Fq2 cmul2(const Fq a0, const Fq b0, const Fq a1, const Fq b1) {
    return {fmul<LAZY>(a0, b0), fmul<LAZY>(a1, b1)};
}
template <bool LAZY>
ZK_CMUL Fq3 cmul3(const Fq a0, const Fq b0, const Fq a1, const Fq b1, const Fq a2, const Fq b2) {
    return {fmul<LAZY>(a0, b0), fmul<LAZY>(a1, b1), fmul<LAZY>(a2, b2)};
}
template <bool LAZY>
ZK_CMUL Fq4 cmul4(const Fq a0, const Fq b0, const Fq a1, const Fq b1, const Fq a2, const Fq b2, const Fq a3,
                  const Fq b3) {
    return {fmul<LAZY>(a0, b0), fmul<LAZY>(a1, b1), fmul<LAZY>(a2, b2), fmul<LAZY>(a3, b3)};
}
#undef ZK_CMUL

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

// 2 * p (dbl-2008-s-1), its nine products in three grouped calls
ZK_HD Xyzz xyzz_dbl(const Xyzz& p) {
    if (xyzz_is_id(p)) return p;
    const Fq u = fe_dbl<FqCfg>(p.y);
    const Fq2 vx = cmul2<false>(u, u, p.x, p.x);  // V = U^2, X^2
    const Fq mm = fe_add<FqCfg>(fe_dbl<FqCfg>(vx.b), vx.b);
    const Fq4 ws = cmul4<false>(u, vx.a, p.x, vx.a, vx.a, p.zz, mm, mm);  // W, S, ZZ3, M^2
    Xyzz r;
    r.x = fe_sub<FqCfg>(fe_sub<FqCfg>(ws.d, ws.b), ws.b);
    const Fq3 t = cmul3<false>(mm, fe_sub<FqCfg>(ws.b, r.x), ws.a, p.y, ws.a, p.zzz);
    r.y = fe_sub<FqCfg>(t.a, t.b);
    r.zz = ws.c;
    r.zzz = t.c;
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
ZK_HD Xyzz xyzz_add_aff_lazy(const Xyzz& p, const Fq& x2, const Fq& y2) {
    if (xyzz_is_id(p)) {
        Xyzz r;
        r.x = x2;
        r.y = y2;
        r.zz = fe_one<FqCfg>();
        r.zzz = fe_one<FqCfg>();
        return r;
    }
    const Fq2 us = cmul2<true>(x2, p.zz, y2, p.zzz);  // U2, S2
    const Fq pp_ = fe_sub_lazy<FqCfg>(us.a, p.x);
    const Fq rr = fe_sub_lazy<FqCfg>(us.b, p.y);
    if (fe_is_zero<FqCfg>(fe_canon<FqCfg>(pp_))) {
        if (fe_is_zero<FqCfg>(fe_canon<FqCfg>(rr))) return aff_dbl(x2, y2);
        return xyzz_identity();
    }
    const Fq2 sq = cmul2<true>(pp_, pp_, rr, rr);      // PP, R^2
    const Fq2 pq = cmul2<true>(pp_, sq.a, p.x, sq.a);  // PPP, Q
    Xyzz r;
    r.x = fe_sub_lazy<FqCfg>(fe_sub_lazy<FqCfg>(fe_sub_lazy<FqCfg>(sq.b, pq.a), pq.b), pq.b);
    const Fq4 f = cmul4<true>(rr, fe_sub_lazy<FqCfg>(pq.b, r.x), p.y, pq.a, p.zz, sq.a, p.zzz, pq.a);
    r.y = fe_sub_lazy<FqCfg>(f.a, f.b);
    r.zz = f.c;
    r.zzz = f.d;
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

// p + q (add-2008-s), its fourteen products in four grouped calls
ZK_HD Xyzz xyzz_add(const Xyzz& p, const Xyzz& q) {
    if (xyzz_is_id(p)) return q;
    if (xyzz_is_id(q)) return p;
    const Fq4 us = cmul4<false>(p.x, q.zz, q.x, p.zz, p.y, q.zzz, q.y, p.zzz);  // U1, U2, S1, S2
    const Fq pp_ = fe_sub<FqCfg>(us.b, us.a);
    const Fq rr = fe_sub<FqCfg>(us.d, us.c);
    if (fe_is_zero<FqCfg>(pp_)) {
        if (fe_is_zero<FqCfg>(rr)) return xyzz_dbl(p);
        return xyzz_identity();
    }
    const Fq4 sq = cmul4<false>(pp_, pp_, rr, rr, p.zz, q.zz, p.zzz, q.zzz);  // PP, R^2, ZZ1 ZZ2, ZZZ1 ZZZ2
    const Fq2 pq = cmul2<false>(pp_, sq.a, us.a, sq.a);                       // PPP, Q
    Xyzz r;
    r.x = fe_sub<FqCfg>(fe_sub<FqCfg>(fe_sub<FqCfg>(sq.b, pq.a), pq.b), pq.b);
    const Fq4 f = cmul4<false>(rr, fe_sub<FqCfg>(pq.b, r.x), us.c, pq.a, sq.c, sq.a, sq.d, pq.a);
    r.y = fe_sub<FqCfg>(f.a, f.b);
    r.zz = f.c;
    r.zzz = f.d;
    return r;
}

// [k] p for a small unsigned k (double-and-add from the top bit)
ZK_HD Xyzz xyzz_mul_u32(const Xyzz& p, uint32_t k) {
    Xyzz r = xyzz_identity();
    if (k == 0 || xyzz_is_id(p)) return r;
    int top = 31;
    while (!((k >> top) & 1)) top--;
    r = p;
    for (int b = top - 1; b >= 0; b--) {
        r = xyzz_dbl(r);
        if ((k >> b) & 1) r = xyzz_add(r, p);
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
