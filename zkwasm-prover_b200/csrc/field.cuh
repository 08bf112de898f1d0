// BN254 prime-field arithmetic for sm_100a: 8 x 32-bit limbs, Montgomery form
// with R = 2^256.  In memory an element is 32 bytes, little-endian, which is
// byte-identical to halo2's 4 x u64 layout (reference: cuda/zprize/ff_storage.cuh,
// src/cuda/msm.rs:441-452), so device buffers are shared with the Rust host
// unchanged.
//
// Multiplication is operand-scanning Montgomery multiplication (Montgomery,
// "Modular multiplication without trial division", 1985) with the reduction
// interleaved row by row.  Each row is two carry chains of mad.lo / mad.hi on
// the integer multiply-add pipe; every chain is one inline-PTX block so the
// carry flag never crosses an asm statement.  On the host the same chains are
// emulated in plain C, which lets the CPU test-suite run the exact operation
// sequence of the device code against the oracle.
//
// Bounds: with m < 2^254, inputs a, b < 2m give a 9-word accumulator that never
// overflows (intermediates stay below 4m * 2^32 < 2^288) and a pre-subtraction
// result below 2m; one conditional subtraction then returns a value below m.
#pragma once
#include <stdint.h>

#if defined(__CUDACC__)
#define ZK_HD __host__ __device__ __forceinline__
#else
#define ZK_HD inline
#endif

namespace zk {

// pick j-th of eight constants; folds to an immediate when j is a compile-time constant
ZK_HD constexpr uint32_t pick8(int j, uint32_t a0, uint32_t a1, uint32_t a2, uint32_t a3, uint32_t a4, uint32_t a5,
                               uint32_t a6, uint32_t a7) {
    return j == 0 ? a0 : j == 1 ? a1 : j == 2 ? a2 : j == 3 ? a3 : j == 4 ? a4 : j == 5 ? a5 : j == 6 ? a6 : a7;
}

struct FrCfg {
    // r = 0x30644e72e131a029b85045b68181585d2833e84879b9709143e1f593f0000001
    static ZK_HD constexpr uint32_t M(int j) {
        return pick8(j, 0xf0000001u, 0x43e1f593u, 0x79b97091u, 0x2833e848u, 0x8181585du, 0xb85045b6u, 0xe131a029u,
                     0x30644e72u);
    }
    static constexpr uint32_t INV = 0xefffffffu;  // -r^-1 mod 2^32
    static ZK_HD constexpr uint32_t ONE(int j) {  // 2^256 mod r
        return pick8(j, 0x4ffffffbu, 0xac96341cu, 0x9f60cd29u, 0x36fc7695u, 0x7879462eu, 0x666ea36fu, 0x9a07df2fu,
                     0x0e0a77c1u);
    }
    static ZK_HD constexpr uint32_t R2(int j) {  // 2^512 mod r
        return pick8(j, 0xae216da7u, 0x1bb8e645u, 0xe35c59e3u, 0x53fe3ab1u, 0x53bb8085u, 0x8c49833du, 0x7f4e44a5u,
                     0x0216d0b1u);
    }
    static ZK_HD constexpr uint32_t R3(int j) {  // 2^768 mod r
        return pick8(j, 0xb4bf0040u, 0x5e94d8e1u, 0x1cfbb6b8u, 0x2a489cbeu, 0xa19fcfedu, 0x893cc664u, 0x7fcc657cu,
                     0x0cf8594bu);
    }
    static ZK_HD constexpr uint32_t PINV(int j) {  // r^-1 mod 2^256
        return pick8(j, 0x10000001u, 0x3d1e0a6cu, 0xb396ee4cu, 0x9a7979b4u, 0x66f9dc6eu, 0x1c6567d7u, 0xf27cbe4du,
                     0x8c07d0e2u);
    }
};

struct FqCfg {
    // p = 0x30644e72e131a029b85045b68181585d97816a916871ca8d3c208c16d87cfd47
    static ZK_HD constexpr uint32_t M(int j) {
        return pick8(j, 0xd87cfd47u, 0x3c208c16u, 0x6871ca8du, 0x97816a91u, 0x8181585du, 0xb85045b6u, 0xe131a029u,
                     0x30644e72u);
    }
    static constexpr uint32_t INV = 0xe4866389u;  // -p^-1 mod 2^32
    static ZK_HD constexpr uint32_t ONE(int j) {
        return pick8(j, 0xc58f0d9du, 0xd35d438du, 0xf5c70b3du, 0x0a78eb28u, 0x7879462cu, 0x666ea36fu, 0x9a07df2fu,
                     0x0e0a77c1u);
    }
    static ZK_HD constexpr uint32_t R2(int j) {
        return pick8(j, 0x538afa89u, 0xf32cfc5bu, 0xd44501fbu, 0xb5e71911u, 0x0a417ff6u, 0x47ab1effu, 0xcab8351fu,
                     0x06d89f71u);
    }
    static ZK_HD constexpr uint32_t R3(int j) {  // 2^768 mod p
        return pick8(j, 0xda1530dfu, 0xb1cd6dafu, 0xa7283db6u, 0x62f210e6u, 0x0ada0afbu, 0xef7f0b0cu, 0x2d592544u,
                     0x20fd6e90u);
    }
};

template <class C>
struct alignas(16) Fe {
    uint32_t v[8];
};

typedef Fe<FrCfg> Fr;
typedef Fe<FqCfg> Fq;

// ---------------------------------------------------------------------------
// carry-chain building blocks (device: PTX; host: C emulation of the same ops)

// t[0..8] += a[0..7] * b   (lo chain then hi chain; t[8] absorbs the carries)
ZK_HD void row_mad(uint32_t t[9], const uint32_t a[8], uint32_t b) {
#if defined(__CUDA_ARCH__)
    asm("mad.lo.cc.u32  %0, %9,  %17, %0;\n\t"
        "madc.lo.cc.u32 %1, %10, %17, %1;\n\t"
        "madc.lo.cc.u32 %2, %11, %17, %2;\n\t"
        "madc.lo.cc.u32 %3, %12, %17, %3;\n\t"
        "madc.lo.cc.u32 %4, %13, %17, %4;\n\t"
        "madc.lo.cc.u32 %5, %14, %17, %5;\n\t"
        "madc.lo.cc.u32 %6, %15, %17, %6;\n\t"
        "madc.lo.cc.u32 %7, %16, %17, %7;\n\t"
        "addc.u32       %8, %8, 0;\n\t"
        "mad.hi.cc.u32  %1, %9,  %17, %1;\n\t"
        "madc.hi.cc.u32 %2, %10, %17, %2;\n\t"
        "madc.hi.cc.u32 %3, %11, %17, %3;\n\t"
        "madc.hi.cc.u32 %4, %12, %17, %4;\n\t"
        "madc.hi.cc.u32 %5, %13, %17, %5;\n\t"
        "madc.hi.cc.u32 %6, %14, %17, %6;\n\t"
        "madc.hi.cc.u32 %7, %15, %17, %7;\n\t"
        "madc.hi.u32    %8, %16, %17, %8;"
        : "+r"(t[0]), "+r"(t[1]), "+r"(t[2]), "+r"(t[3]), "+r"(t[4]), "+r"(t[5]), "+r"(t[6]),
          "+r"(t[7]), "+r"(t[8])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(a[4]), "r"(a[5]), "r"(a[6]), "r"(a[7]),
          "r"(b));
#else
    uint64_t c = 0;
    for (int j = 0; j < 8; j++) {
        uint64_t s = (uint64_t)(uint32_t)((uint64_t)a[j] * b) + t[j] + c;
        t[j] = (uint32_t)s;
        c = s >> 32;
    }
    t[8] = (uint32_t)(t[8] + c);
    c = 0;
    for (int j = 0; j < 8; j++) {
        uint64_t s = (uint64_t)(uint32_t)(((uint64_t)a[j] * b) >> 32) + t[j + 1] + c;
        t[j + 1] = (uint32_t)s;
        c = s >> 32;
    }
#endif
}

// r = t - m (8 words) and returns the borrow mask (0 or 0xffffffff)
ZK_HD uint32_t sub8_borrow(uint32_t r[8], const uint32_t t[8], const uint32_t m[8]) {
#if defined(__CUDA_ARCH__)
    uint32_t br;
    asm("sub.cc.u32  %0, %9,  %17;\n\t"
        "subc.cc.u32 %1, %10, %18;\n\t"
        "subc.cc.u32 %2, %11, %19;\n\t"
        "subc.cc.u32 %3, %12, %20;\n\t"
        "subc.cc.u32 %4, %13, %21;\n\t"
        "subc.cc.u32 %5, %14, %22;\n\t"
        "subc.cc.u32 %6, %15, %23;\n\t"
        "subc.cc.u32 %7, %16, %24;\n\t"
        "subc.u32    %8, 0, 0;"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
          "=r"(r[7]), "=r"(br)
        : "r"(t[0]), "r"(t[1]), "r"(t[2]), "r"(t[3]), "r"(t[4]), "r"(t[5]), "r"(t[6]), "r"(t[7]),
          "r"(m[0]), "r"(m[1]), "r"(m[2]), "r"(m[3]), "r"(m[4]), "r"(m[5]), "r"(m[6]), "r"(m[7]));
    return br;
#else
    uint64_t b = 0;
    for (int j = 0; j < 8; j++) {
        uint64_t d = (uint64_t)t[j] - m[j] - b;
        r[j] = (uint32_t)d;
        b = (d >> 63) & 1;
    }
    return b ? 0xffffffffu : 0u;
#endif
}

// r = a + b (8 words), returns carry (0/1)
ZK_HD uint32_t add8_carry(uint32_t r[8], const uint32_t a[8], const uint32_t b[8]) {
#if defined(__CUDA_ARCH__)
    uint32_t c;
    asm("add.cc.u32  %0, %9,  %17;\n\t"
        "addc.cc.u32 %1, %10, %18;\n\t"
        "addc.cc.u32 %2, %11, %19;\n\t"
        "addc.cc.u32 %3, %12, %20;\n\t"
        "addc.cc.u32 %4, %13, %21;\n\t"
        "addc.cc.u32 %5, %14, %22;\n\t"
        "addc.cc.u32 %6, %15, %23;\n\t"
        "addc.cc.u32 %7, %16, %24;\n\t"
        "addc.u32    %8, 0, 0;"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
          "=r"(r[7]), "=r"(c)
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(a[4]), "r"(a[5]), "r"(a[6]), "r"(a[7]),
          "r"(b[0]), "r"(b[1]), "r"(b[2]), "r"(b[3]), "r"(b[4]), "r"(b[5]), "r"(b[6]), "r"(b[7]));
    return c;
#else
    uint64_t c = 0;
    for (int j = 0; j < 8; j++) {
        uint64_t s = (uint64_t)a[j] + b[j] + c;
        r[j] = (uint32_t)s;
        c = s >> 32;
    }
    return (uint32_t)c;
#endif
}

// r = mask ? a : b  (mask is 0 or all ones)
ZK_HD void select8(uint32_t r[8], uint32_t mask, const uint32_t a[8], const uint32_t b[8]) {
#pragma unroll
    for (int j = 0; j < 8; j++) r[j] = b[j] ^ ((a[j] ^ b[j]) & mask);
}

// ---------------------------------------------------------------------------
// field operations

template <class C>
ZK_HD Fe<C> fe_zero() {
    Fe<C> r;
#pragma unroll
    for (int j = 0; j < 8; j++) r.v[j] = 0;
    return r;
}

template <class C>
ZK_HD Fe<C> fe_one() {
    Fe<C> r;
#pragma unroll
    for (int j = 0; j < 8; j++) r.v[j] = C::ONE(j);
    return r;
}

template <class C>
ZK_HD Fe<C> fe_modulus() {
    Fe<C> r;
#pragma unroll
    for (int j = 0; j < 8; j++) r.v[j] = C::M(j);
    return r;
}

// Conditional subtraction of m: input < 2m, output < m.
template <class C>
ZK_HD void fe_reduce_once(uint32_t t[8]) {
    uint32_t u[8], m[8];
#pragma unroll
    for (int j = 0; j < 8; j++) m[j] = C::M(j);
    uint32_t br = sub8_borrow(u, t, m);
    select8(t, br, t, u);
}

// acc[0..8] += a[P] * b, a[P+2] * b, a[P+4] * b, a[P+6] * b with the four
// 64-bit products laid side by side (lo at word 2k, hi at word 2k+1): one
// carry chain.  P = 0 gives the even-limb products (positions 0..7 of the
// running sum), P = 1 the odd-limb ones (positions 1..8, stored from word 0).
template <int P>
ZK_HD void chain4(uint32_t acc[9], const uint32_t a[8], uint32_t b) {
#if defined(__CUDA_ARCH__)
    asm("mad.lo.cc.u32  %0, %9,  %13, %0;\n\t"
        "madc.hi.cc.u32 %1, %9,  %13, %1;\n\t"
        "madc.lo.cc.u32 %2, %10, %13, %2;\n\t"
        "madc.hi.cc.u32 %3, %10, %13, %3;\n\t"
        "madc.lo.cc.u32 %4, %11, %13, %4;\n\t"
        "madc.hi.cc.u32 %5, %11, %13, %5;\n\t"
        "madc.lo.cc.u32 %6, %12, %13, %6;\n\t"
        "madc.hi.cc.u32 %7, %12, %13, %7;\n\t"
        "addc.u32       %8, %8, 0;"
        : "+r"(acc[0]), "+r"(acc[1]), "+r"(acc[2]), "+r"(acc[3]), "+r"(acc[4]), "+r"(acc[5]), "+r"(acc[6]),
          "+r"(acc[7]), "+r"(acc[8])
        : "r"(a[P]), "r"(a[P + 2]), "r"(a[P + 4]), "r"(a[P + 6]), "r"(b));
#else
    uint64_t c = 0;
    for (int k = 0; k < 4; k++) {
        const uint64_t p = (uint64_t)a[P + 2 * k] * b;
        uint64_t s = (uint64_t)acc[2 * k] + (uint32_t)p + c;
        acc[2 * k] = (uint32_t)s;
        c = s >> 32;
        s = (uint64_t)acc[2 * k + 1] + (uint32_t)(p >> 32) + c;
        acc[2 * k + 1] = (uint32_t)s;
        c = s >> 32;
    }
    acc[8] = (uint32_t)(acc[8] + c);
#endif
}

// o[0..7] += e[1..8], carry into o[8]
ZK_HD void merge_shift(uint32_t o[9], const uint32_t e[9]) {
#if defined(__CUDA_ARCH__)
    asm("add.cc.u32  %0, %0, %9;\n\t"
        "addc.cc.u32 %1, %1, %10;\n\t"
        "addc.cc.u32 %2, %2, %11;\n\t"
        "addc.cc.u32 %3, %3, %12;\n\t"
        "addc.cc.u32 %4, %4, %13;\n\t"
        "addc.cc.u32 %5, %5, %14;\n\t"
        "addc.cc.u32 %6, %6, %15;\n\t"
        "addc.cc.u32 %7, %7, %16;\n\t"
        "addc.u32    %8, %8, 0;"
        : "+r"(o[0]), "+r"(o[1]), "+r"(o[2]), "+r"(o[3]), "+r"(o[4]), "+r"(o[5]), "+r"(o[6]), "+r"(o[7]),
          "+r"(o[8])
        : "r"(e[1]), "r"(e[2]), "r"(e[3]), "r"(e[4]), "r"(e[5]), "r"(e[6]), "r"(e[7]), "r"(e[8]));
#else
    uint64_t c = 0;
    for (int j = 0; j < 8; j++) {
        uint64_t s = (uint64_t)o[j] + e[j + 1] + c;
        o[j] = (uint32_t)s;
        c = s >> 32;
    }
    o[8] = (uint32_t)(o[8] + c);
#endif
}

// Montgomery product a * b * 2^-256 mod m without the final subtraction:
// for a, b < 2m (and m < 2^254) the result is below (4m^2 + m 2^256) / 2^256
// < 2m.
//
// Operand scanning with the running sum T split into an even accumulator E
// (products of even limbs of a) and an odd accumulator O (odd limbs, one word
// up): T = E + 2^32 O.  Each row adds a * b_i and q * m (q = E_0 * -m^-1) as
// four independent carry chains of alternating mad.lo / mad.hi over the same
// operands, then folds E >> 32 into O, which becomes the next row's E.  This
// measured about 1.5x the rate of the lo-chain / hi-chain row form on B200.
template <class C>
ZK_HD Fe<C> fe_mul_lazy(const Fe<C>& a, const Fe<C>& b) {
    uint32_t m[8];
#pragma unroll
    for (int j = 0; j < 8; j++) m[j] = C::M(j);
    uint32_t e[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    uint32_t o[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
#pragma unroll
    for (int i = 0; i < 8; i++) {
        chain4<0>(e, a.v, b.v[i]);
        chain4<1>(o, a.v, b.v[i]);
        const uint32_t q = e[0] * C::INV;
        chain4<0>(e, m, q);
        chain4<1>(o, m, q);
        // e[0] is now zero: T / 2^32 = (E >> 32) + O
        merge_shift(o, e);
#pragma unroll
        for (int j = 0; j < 9; j++) {
            e[j] = o[j];
            o[j] = 0;
        }
    }
    Fe<C> r;
#pragma unroll
    for (int j = 0; j < 8; j++) r.v[j] = e[j];
    return r;
}

// ---------------------------------------------------------------------------
// Products by a known factor (Shoup): for a canonical w and its companion
// w' = floor(w 2^256 / m), a * w mod m for any a < 2^256 from q = the high
// half of a w' (truncated below column 7: short by at most one) and
// a w - q m, which then lies in [0, 3m); one conditional subtraction of m
// leaves [0, 2m).  With a in Montgomery form and w canonical the result is
// the Montgomery form of the product, as fe_mul_lazy(a, w R mod m) would give,
// for 207 multiply-adds instead of 264.

// (c0, c1, c2) += x * y (product scanning, one column)
ZK_HD void mac3(uint32_t& c0, uint32_t& c1, uint32_t& c2, uint32_t x, uint32_t y) {
#if defined(__CUDA_ARCH__)
    asm("mad.lo.cc.u32  %0, %3, %4, %0;\n\t"
        "madc.hi.cc.u32 %1, %3, %4, %1;\n\t"
        "addc.u32       %2, %2, 0;"
        : "+r"(c0), "+r"(c1), "+r"(c2)
        : "r"(x), "r"(y));
#else
    const uint64_t p = (uint64_t)x * y;
    uint64_t s = (uint64_t)c0 + (uint32_t)p;
    c0 = (uint32_t)s;
    s = (uint64_t)c1 + (uint32_t)(p >> 32) + (s >> 32);
    c1 = (uint32_t)s;
    c2 += (uint32_t)(s >> 32);
#endif
}

// (c1, c2) += high word of x * y
ZK_HD void machi2(uint32_t& c1, uint32_t& c2, uint32_t x, uint32_t y) {
#if defined(__CUDA_ARCH__)
    asm("mad.hi.cc.u32 %0, %2, %3, %0;\n\t"
        "addc.u32      %1, %1, 0;"
        : "+r"(c1), "+r"(c2)
        : "r"(x), "r"(y));
#else
    const uint64_t s = (uint64_t)c1 + (uint32_t)(((uint64_t)x * y) >> 32);
    c1 = (uint32_t)s;
    c2 += (uint32_t)(s >> 32);
#endif
}

// r = a * b mod 2^256
ZK_HD void mul_lo8(uint32_t r[8], const uint32_t a[8], const uint32_t b[8]) {
    uint32_t c0 = 0, c1 = 0, c2 = 0;
#pragma unroll
    for (int k = 0; k < 7; k++) {
#pragma unroll
        for (int i = 0; i <= k; i++) mac3(c0, c1, c2, a[i], b[k - i]);
        r[k] = c0;
        c0 = c1;
        c1 = c2;
        c2 = 0;
    }
#pragma unroll
    for (int i = 0; i < 8; i++) c0 += a[i] * b[7 - i];
    r[7] = c0;
}

// q = floor(S / 2^256) for S the sum of the partial products of a * b from
// column 7 up and the high words of column 6: floor(a b / 2^256) or one less
// (the terms left out sum to less than 2^229)
ZK_HD void mul_hi8_trunc(uint32_t q[8], const uint32_t a[8], const uint32_t b[8]) {
    uint32_t c1 = 0, c2 = 0;
#pragma unroll
    for (int i = 0; i <= 6; i++) machi2(c1, c2, a[i], b[6 - i]);
    uint32_t c0 = c1;
    c1 = c2;
    c2 = 0;
#pragma unroll
    for (int i = 0; i <= 7; i++) mac3(c0, c1, c2, a[i], b[7 - i]);
#pragma unroll
    for (int k = 8; k < 15; k++) {
        c0 = c1;
        c1 = c2;
        c2 = 0;
#pragma unroll
        for (int i = k - 7; i <= 7; i++) mac3(c0, c1, c2, a[i], b[k - i]);
        q[k - 8] = c0;
    }
    q[7] = c1;
}

template <class C>
ZK_HD Fe<C> fe_mul_shoup(const Fe<C>& a, const Fe<C>& w, const Fe<C>& wp) {
    uint32_t m[8], q[8], x[8], y[8], r[8], u[8];
#pragma unroll
    for (int j = 0; j < 8; j++) m[j] = C::M(j);
    mul_hi8_trunc(q, a.v, wp.v);
    mul_lo8(x, a.v, w.v);
    mul_lo8(y, q, m);
    sub8_borrow(r, x, y);
    const uint32_t br = sub8_borrow(u, r, m);
    Fe<C> o;
    select8(o.v, br, r, u);
    return o;
}

// The companion w' = floor(w 2^256 / m) of w from its Montgomery form
// wm = w 2^256 mod m: w 2^256 = w' m + wm, so w' = -wm m^-1 mod 2^256 (exact,
// as w' < 2^256).  Needs C::PINV = m^-1 mod 2^256.
template <class C>
ZK_HD Fe<C> fe_shoup_companion(const Fe<C>& wm) {
    uint32_t neg[8], zero[8], pinv[8];
#pragma unroll
    for (int j = 0; j < 8; j++) {
        zero[j] = 0;
        pinv[j] = C::PINV(j);
    }
    sub8_borrow(neg, zero, wm.v);
    Fe<C> r;
    mul_lo8(r.v, neg, pinv);
    return r;
}

// Montgomery product a * b * 2^-256 mod m; a, b < 2m, result < m.
template <class C>
ZK_HD Fe<C> fe_mul(const Fe<C>& a, const Fe<C>& b) {
    Fe<C> r = fe_mul_lazy<C>(a, b);
    fe_reduce_once<C>(r.v);
    return r;
}

// 2m, limb j
template <class C>
ZK_HD constexpr uint32_t twice_m(int j) {
    return (C::M(j) << 1) | (j ? C::M(j - 1) >> 31 : 0u);
}

// Lazily reduced representatives in [0, 2m) (m < 2^254, so sums of two stay
// below 2^256): a + b and a - b for a, b < 2m, results < 2m; fe_canon maps
// [0, 2m) to the canonical [0, m).
template <class C>
ZK_HD Fe<C> fe_add_lazy(const Fe<C>& a, const Fe<C>& b) {
    uint32_t t[8], u[8], m2[8];
#pragma unroll
    for (int j = 0; j < 8; j++) m2[j] = twice_m<C>(j);
    add8_carry(t, a.v, b.v);
    const uint32_t br = sub8_borrow(u, t, m2);
    Fe<C> r;
    select8(r.v, br, t, u);
    return r;
}

template <class C>
ZK_HD Fe<C> fe_sub_lazy(const Fe<C>& a, const Fe<C>& b) {
    uint32_t t[8], u[8], m2[8];
#pragma unroll
    for (int j = 0; j < 8; j++) m2[j] = twice_m<C>(j);
    const uint32_t br = sub8_borrow(t, a.v, b.v);
    add8_carry(u, t, m2);
    Fe<C> r;
    select8(r.v, br, u, t);
    return r;
}

template <class C>
ZK_HD Fe<C> fe_canon(const Fe<C>& a) {
    Fe<C> r = a;
    fe_reduce_once<C>(r.v);
    return r;
}

template <class C>
ZK_HD Fe<C> fe_sqr(const Fe<C>& a) {
    return fe_mul<C>(a, a);
}

// Montgomery reduction only: a * 2^-256 mod m (leaves Montgomery form).
template <class C>
ZK_HD Fe<C> fe_from_mont(const Fe<C>& a) {
    uint32_t t[9];
    uint32_t m[8];
#pragma unroll
    for (int j = 0; j < 8; j++) {
        m[j] = C::M(j);
        t[j] = a.v[j];
    }
    t[8] = 0;
#pragma unroll
    for (int i = 0; i < 8; i++) {
        uint32_t q = t[0] * C::INV;
        row_mad(t, m, q);
#pragma unroll
        for (int j = 0; j < 8; j++) t[j] = t[j + 1];
        t[8] = 0;
    }
    fe_reduce_once<C>(t);
    Fe<C> r;
#pragma unroll
    for (int j = 0; j < 8; j++) r.v[j] = t[j];
    return r;
}

template <class C>
ZK_HD Fe<C> fe_to_mont(const Fe<C>& a) {
    Fe<C> r2;
#pragma unroll
    for (int j = 0; j < 8; j++) r2.v[j] = C::R2(j);
    return fe_mul<C>(a, r2);
}

// a + b mod m for a, b < m
template <class C>
ZK_HD Fe<C> fe_add(const Fe<C>& a, const Fe<C>& b) {
    Fe<C> r;
    add8_carry(r.v, a.v, b.v);
    fe_reduce_once<C>(r.v);
    return r;
}

// a - b mod m for a, b < m
template <class C>
ZK_HD Fe<C> fe_sub(const Fe<C>& a, const Fe<C>& b) {
    uint32_t t[8], u[8], m[8];
#pragma unroll
    for (int j = 0; j < 8; j++) m[j] = C::M(j);
    uint32_t br = sub8_borrow(t, a.v, b.v);
    add8_carry(u, t, m);
    Fe<C> r;
    select8(r.v, br, u, t);
    return r;
}

template <class C>
ZK_HD Fe<C> fe_dbl(const Fe<C>& a) {
    return fe_add<C>(a, a);
}

template <class C>
ZK_HD bool fe_is_zero(const Fe<C>& a) {
    uint32_t x = 0;
#pragma unroll
    for (int j = 0; j < 8; j++) x |= a.v[j];
    return x == 0;
}

template <class C>
ZK_HD bool fe_eq(const Fe<C>& a, const Fe<C>& b) {
    uint32_t x = 0;
#pragma unroll
    for (int j = 0; j < 8; j++) x |= a.v[j] ^ b.v[j];
    return x == 0;
}

template <class C>
ZK_HD Fe<C> fe_neg(const Fe<C>& a) {
    return fe_sub<C>(fe_zero<C>(), a);
}

// a^e for a 32-bit exponent
template <class C>
ZK_HD Fe<C> fe_pow_u32(Fe<C> a, uint32_t e) {
    Fe<C> r = fe_one<C>();
    while (e) {
        if (e & 1) r = fe_mul<C>(r, a);
        e >>= 1;
        if (e) a = fe_sqr<C>(a);
    }
    return r;
}

// a^(m-2): multiplicative inverse by Fermat's little theorem (0 maps to 0).
// 8-limb helpers of the binary inversion
ZK_HD bool limbs_is_one(const uint32_t x[8]) {
    uint32_t o = x[0] ^ 1u;
#pragma unroll
    for (int j = 1; j < 8; j++) o |= x[j];
    return o == 0;
}

ZK_HD bool limbs_geq(const uint32_t a[8], const uint32_t b[8]) {
    uint32_t t[8];
    return sub8_borrow(t, a, b) == 0;
}

ZK_HD void limbs_shr1(uint32_t x[8]) {
#pragma unroll
    for (int j = 0; j < 7; j++) x[j] = (x[j] >> 1) | (x[j + 1] << 31);
    x[7] >>= 1;
}

// x / 2 mod m for x < m (x + m < 2^255 fits)
template <class C>
ZK_HD void limbs_half_mod(uint32_t x[8]) {
    if (x[0] & 1u) {
        uint32_t m[8];
#pragma unroll
        for (int j = 0; j < 8; j++) m[j] = C::M(j);
        add8_carry(x, x, m);
    }
    limbs_shr1(x);
}

// x - y mod m for x, y < m
template <class C>
ZK_HD void limbs_sub_mod(uint32_t x[8], const uint32_t y[8]) {
    uint32_t t[8], u[8], m[8];
#pragma unroll
    for (int j = 0; j < 8; j++) m[j] = C::M(j);
    const uint32_t br = sub8_borrow(t, x, y);
    add8_carry(u, t, m);
    select8(x, br, u, t);
}

// Inverse of a Montgomery-form element (zero maps to zero).  Binary extended
// Euclid (variable time) on the representative A = a R: u, v start at A and
// m with u = x1 A, v = x2 A (mod m) kept invariant; halving and subtracting
// until u or v is 1 gives A^-1, and the Montgomery product with R^3 turns it
// into a^-1 R.  Each step is a few short 8-limb chains, so one thread takes
// a fraction of the latency of the ~380 dependent products of a^(m-2).
template <class C>
ZK_HD Fe<C> fe_inv(const Fe<C>& a) {
    if (fe_is_zero<C>(a)) return a;
    uint32_t u[8], v[8], x1[8], x2[8];
#pragma unroll
    for (int j = 0; j < 8; j++) {
        u[j] = a.v[j];
        v[j] = C::M(j);
        x1[j] = j == 0 ? 1u : 0u;
        x2[j] = 0u;
    }
    bool first = true;
    for (;;) {
        while (!(u[0] & 1u)) {
            limbs_shr1(u);
            limbs_half_mod<C>(x1);
        }
        while (!(v[0] & 1u)) {
            limbs_shr1(v);
            limbs_half_mod<C>(x2);
        }
        if (limbs_is_one(u)) break;
        if (limbs_is_one(v)) {
            first = false;
            break;
        }
        if (limbs_geq(u, v)) {
            sub8_borrow(u, u, v);
            limbs_sub_mod<C>(x1, x2);
        } else {
            sub8_borrow(v, v, u);
            limbs_sub_mod<C>(x2, x1);
        }
    }
    Fe<C> x, r3;
#pragma unroll
    for (int j = 0; j < 8; j++) {
        x.v[j] = first ? x1[j] : x2[j];
        r3.v[j] = C::R3(j);
    }
    return fe_mul<C>(x, r3);
}

// n-bit field of a canonical (non-Montgomery) 256-bit value starting at bit `start`
ZK_HD uint32_t bits_at(const uint32_t v[8], uint32_t start, uint32_t nbits) {
    uint32_t w = start >> 5, off = start & 31;
    uint64_t lo = v[w];
    uint64_t hi = (w + 1 < 8) ? v[w + 1] : 0;
    uint64_t x = (lo | (hi << 32)) >> off;
    return (uint32_t)(x & ((nbits >= 32) ? 0xffffffffull : ((1ull << nbits) - 1)));
}

}  // namespace zk
