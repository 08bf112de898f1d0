// GLV endomorphism of BN254 G1 for the MSM.
//
// beta = 0x30644e72e131a0295e6dd9e7e0acccb0c28f069fbb966e3de4bd44e5607cfd48 is
// a primitive cube root of unity mod p, so phi(x, y) = (beta x, y) maps the
// curve y^2 = x^3 + 3 to itself, and phi(P) = [lambda] P for the cube root of
// unity mod r lambda = 0x30644e72e131a029048b6e193fd84104cc37a73fec2bc5e9b8ca0b2d36636f23
// (the pairing of the two roots checked on the generator (1, 2)).
//
// A scalar k < r splits as k = k1 + k2 lambda (mod r) with |k1|, |k2| < 2^127
// (Gallant-Lambert-Vanstone): with the short basis (a1, b1), (a2, b2) of the
// lattice {(x, y) : x + y lambda = 0 mod r} from the extended Euclidean
// algorithm on (r, lambda),
//   a1 = 147946756881789319000765030803803410728   b1 = -9931322734385697763
//   a2 = 9931322734385697763                      b2 = 147946756881789319010696353538189108491
// c1 = floor(k g1 / 2^256), c2 = floor(k g2 / 2^256) with g1 = round(b2 2^256 / r),
// g2 = round(-b1 2^256 / r), and
//   k1 = k - c1 a1 - c2 a2,   k2 = -c1 b1 - c2 b2.
// An MSM over n points with 254-bit scalars becomes one over 2n points (P_i
// and phi(P_i)) with 127-bit scalars: half the windows, half the buckets and
// half the doublings of the final combination.
#pragma once
#include "curve.cuh"

namespace zk {

// beta * 2^256 mod p (Montgomery form)
ZK_HD constexpr uint32_t glv_beta(int j) {
    return pick8(j, 0x13e80b9cu, 0x3350c88eu, 0xdb5e56b9u, 0x7dce557cu, 0xb615564au, 0x6001b4b8u, 0x020217e0u,
                 0x2682e617u);
}

// t[0..nt) += a[0..na) * b[0..nb), dropping what falls beyond nt limbs
ZK_HD void glv_mac(uint32_t* t, int nt, const uint32_t* a, int na, const uint32_t* b, int nb) {
    for (int i = 0; i < na; i++) {
        uint64_t c = 0;
        for (int j = 0; j < nb && i + j < nt; j++) {
            const uint64_t s = (uint64_t)a[i] * b[j] + t[i + j] + c;
            t[i + j] = (uint32_t)s;
            c = s >> 32;
        }
        for (int j = i + nb; j < nt && c; j++) {
            const uint64_t s = (uint64_t)t[j] + c;
            t[j] = (uint32_t)s;
            c = s >> 32;
        }
    }
}

// two's complement of x[0..n): returns the sign, leaves the magnitude in x
ZK_HD bool glv_abs(uint32_t* x, int n) {
    const bool neg = x[n - 1] >> 31;
    if (neg) {
        uint32_t c = 1;
        for (int j = 0; j < n; j++) {
            const uint64_t s = (uint64_t)(~x[j]) + c;
            x[j] = (uint32_t)s;
            c = (uint32_t)(s >> 32);
        }
    }
    return neg;
}

// k (canonical, < r) -> magnitudes m1, m2 (< 2^127, 8 limbs, upper four zero)
// and signs with k = (-1)^neg1 m1 + (-1)^neg2 m2 lambda (mod r)
ZK_HD void glv_split(const uint32_t k[8], uint32_t m1[8], uint32_t m2[8], bool& neg1, bool& neg2) {
    const uint32_t g1[5] = {0x00ff6565u, 0x5398fd03u, 0xa773d2d2u, 0x4ccef014u, 0x00000002u};
    const uint32_t g2[3] = {0xc7e0b3d7u, 0xd91d232eu, 0x00000002u};
    const uint32_t a1[4] = {0x7d4f1128u, 0x8211bbebu, 0xeeb859fcu, 0x6f4d8248u};
    const uint32_t b1abs[2] = {0x94d213e3u, 0x89d32568u};  // -b1 = a2
    const uint32_t b2[4] = {0x1221250bu, 0x0be4e154u, 0xeeb859fdu, 0x6f4d8248u};
    uint32_t t[13];
    for (int j = 0; j < 13; j++) t[j] = 0;
    glv_mac(t, 13, k, 8, g1, 5);
    uint32_t c1[5];
    for (int j = 0; j < 5; j++) c1[j] = t[8 + j];
    for (int j = 0; j < 11; j++) t[j] = 0;
    glv_mac(t, 11, k, 8, g2, 3);
    uint32_t c2[3];
    for (int j = 0; j < 3; j++) c2[j] = t[8 + j];
    // k1 = k - (c1 a1 + c2 a2), in 9 limbs
    uint32_t s[9];
    for (int j = 0; j < 9; j++) s[j] = 0;
    glv_mac(s, 9, c1, 5, a1, 4);
    glv_mac(s, 9, c2, 3, b1abs, 2);
    uint32_t x[9];
    uint64_t br = 0;
    for (int j = 0; j < 9; j++) {
        const uint64_t d = (uint64_t)(j < 8 ? k[j] : 0u) - s[j] - br;
        x[j] = (uint32_t)d;
        br = (d >> 32) & 1;
    }
    neg1 = glv_abs(x, 9);
    for (int j = 0; j < 8; j++) m1[j] = j < 4 ? x[j] : 0u;
    // k2 = c1 |b1| - c2 b2, in 8 limbs
    uint32_t u[8], v[8];
    for (int j = 0; j < 8; j++) u[j] = v[j] = 0;
    glv_mac(u, 8, c1, 5, b1abs, 2);
    glv_mac(v, 8, c2, 3, b2, 4);
    br = 0;
    for (int j = 0; j < 8; j++) {
        const uint64_t d = (uint64_t)u[j] - v[j] - br;
        x[j] = (uint32_t)d;
        br = (d >> 32) & 1;
    }
    neg2 = glv_abs(x, 8);
    for (int j = 0; j < 8; j++) m2[j] = j < 4 ? x[j] : 0u;
}

// phi(P) = (beta x, y); the identity (0, 0) stays itself
ZK_HD Aff glv_phi(const Aff& a) {
    Fq b;
#pragma unroll
    for (int j = 0; j < 8; j++) b.v[j] = glv_beta(j);
    Aff r;
    r.x = fe_mul<FqCfg>(a.x, b);
    r.y = a.y;
    return r;
}

}  // namespace zk
