/*
 * CPU oracle for the BN254 KZG proving hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  Nothing in the product library links, loads or
 * calls this file: it is the checker that the CUDA path is compared against
 * (tests/, __graft_entry__.smoke() and the cpu_baseline leg of bench.py).
 *
 * It restates, in plain C with unsigned __int128, the arithmetic that the
 * reference computes:
 *   - Fr / Fq Montgomery arithmetic with R = 2^256 and 4 x u64 little-endian
 *     limbs, byte-identical to halo2's field layout (reference:
 *     cuda/zprize/ff_storage.cuh, src/cuda/msm.rs:441-452);
 *   - G1 over y^2 = x^3 + 3 in Jacobian coordinates, affine identity (0, 0),
 *     Jacobian identity Z = 0 (reference: cuda/zprize/ec.cuh:142);
 *   - natural-order radix-2 NTT, i.e. the DFT that halo2's best_fft computes
 *     (reference call sites: src/profile.rs:212, src/cuda/ntt.rs:61-93);
 *   - Pippenger MSM whose affine result equals best_multiexp's
 *     (reference test: src/cuda/msm.rs:457-537);
 *   - Montgomery batch inversion, grand products and grand sums
 *     (reference: src/permutation.rs:16-150, src/shuffle.rs:143-212,
 *     cuda/bn254.cu:19-220).
 * Elementwise quotient formulas are composed in oracle.py from the vector
 * primitives exported here.
 *
 * Multithreading (OpenMP) is used for the MSM, the NTT and point generation so
 * that the same code doubles as the timed CPU baseline.
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <omp.h>

typedef uint64_t u64;
typedef unsigned __int128 u128;

typedef struct {
    u64 m[4];    /* modulus */
    u64 inv;     /* -m^-1 mod 2^64 */
    u64 one[4];  /* R mod m */
    u64 r2[4];   /* R^2 mod m */
} fdesc;

/* Public BN254 parameters. */
static fdesc FR = {{0x43e1f593f0000001ULL, 0x2833e84879b97091ULL, 0xb85045b68181585dULL, 0x30644e72e131a029ULL}, 0, {0}, {0}};
static fdesc FQ = {{0x3c208c16d87cfd47ULL, 0x97816a916871ca8dULL, 0xb85045b68181585dULL, 0x30644e72e131a029ULL}, 0, {0}, {0}};
static int g_init = 0;

static inline const fdesc *F(int which) { return which ? &FQ : &FR; }

static inline int geq(const u64 a[4], const u64 b[4]) {
    for (int i = 3; i >= 0; i--) {
        if (a[i] > b[i]) return 1;
        if (a[i] < b[i]) return 0;
    }
    return 1;
}

static inline u64 sub4(u64 r[4], const u64 a[4], const u64 b[4]) {
    u64 br = 0;
    for (int i = 0; i < 4; i++) {
        u128 d = (u128)a[i] - b[i] - br;
        r[i] = (u64)d;
        br = (u64)(d >> 127) & 1;
    }
    return br;
}

static inline u64 add4(u64 r[4], const u64 a[4], const u64 b[4]) {
    u64 c = 0;
    for (int i = 0; i < 4; i++) {
        u128 s = (u128)a[i] + b[i] + c;
        r[i] = (u64)s;
        c = (u64)(s >> 64);
    }
    return c;
}

static inline void f_add(const fdesc *f, u64 r[4], const u64 a[4], const u64 b[4]) {
    u64 t[4];
    u64 c = add4(t, a, b);
    if (c || geq(t, f->m)) sub4(t, t, f->m);
    memcpy(r, t, 32);
}

static inline void f_sub(const fdesc *f, u64 r[4], const u64 a[4], const u64 b[4]) {
    u64 t[4];
    if (sub4(t, a, b)) add4(t, t, f->m);
    memcpy(r, t, 32);
}

static inline int f_is_zero(const u64 a[4]) { return (a[0] | a[1] | a[2] | a[3]) == 0; }

static inline void f_neg(const fdesc *f, u64 r[4], const u64 a[4]) {
    if (f_is_zero(a)) { memset(r, 0, 32); return; }
    sub4(r, f->m, a);
}

/* CIOS Montgomery multiplication: r = a * b * 2^-256 mod m, inputs < m. */
static inline void f_mul(const fdesc *f, u64 r[4], const u64 a[4], const u64 b[4]) {
    u64 t[6] = {0, 0, 0, 0, 0, 0};
    for (int i = 0; i < 4; i++) {
        u128 c = 0;
        for (int j = 0; j < 4; j++) {
            c = (u128)a[j] * b[i] + t[j] + (u64)(c >> 64);
            t[j] = (u64)c;
        }
        c = (u128)t[4] + (u64)(c >> 64);
        t[4] = (u64)c;
        t[5] = (u64)(c >> 64);
        u64 q = t[0] * f->inv;
        c = (u128)q * f->m[0] + t[0];
        for (int j = 1; j < 4; j++) {
            c = (u128)q * f->m[j] + t[j] + (u64)(c >> 64);
            t[j - 1] = (u64)c;
        }
        c = (u128)t[4] + (u64)(c >> 64);
        t[3] = (u64)c;
        t[4] = t[5] + (u64)(c >> 64);
    }
    u64 o[4] = {t[0], t[1], t[2], t[3]};
    if (t[4] || geq(o, f->m)) sub4(o, o, f->m);
    memcpy(r, o, 32);
}

static inline void f_sqr(const fdesc *f, u64 r[4], const u64 a[4]) { f_mul(f, r, a, a); }

static void f_pow_u64(const fdesc *f, u64 r[4], const u64 a[4], const u64 e[4]) {
    u64 acc[4], base[4];
    memcpy(acc, f->one, 32);
    memcpy(base, a, 32);
    for (int i = 0; i < 4; i++) {
        for (int b = 0; b < 64; b++) {
            if ((e[i] >> b) & 1) f_mul(f, acc, acc, base);
            f_sqr(f, base, base);
        }
    }
    memcpy(r, acc, 32);
}

/* Inverse by Fermat's little theorem; inverse of 0 is 0. */
static void f_inv(const fdesc *f, u64 r[4], const u64 a[4]) {
    u64 e[4], two[4] = {2, 0, 0, 0};
    sub4(e, f->m, two);
    f_pow_u64(f, r, a, e);
}

static void f_to_mont(const fdesc *f, u64 r[4], const u64 a[4]) { f_mul(f, r, a, f->r2); }
static void f_from_mont(const fdesc *f, u64 r[4], const u64 a[4]) {
    u64 one[4] = {1, 0, 0, 0};
    f_mul(f, r, a, one);
}

static void init_field(fdesc *f) {
    /* inv = -m^-1 mod 2^64 by Newton iteration */
    u64 x = 1;
    for (int i = 0; i < 7; i++) x *= 2 - f->m[0] * x;
    f->inv = (u64)0 - x;
    /* one = 2^256 mod m by doubling 1 two hundred fifty-six times */
    u64 t[4] = {1, 0, 0, 0};
    for (int i = 0; i < 256; i++) f_add(f, t, t, t);
    memcpy(f->one, t, 32);
    /* r2 = 2^512 mod m: keep doubling */
    for (int i = 0; i < 256; i++) f_add(f, t, t, t);
    memcpy(f->r2, t, 32);
}

void or_init(void) {
    if (g_init) return;
    init_field(&FR);
    init_field(&FQ);
    g_init = 1;
}

/* ------------------------------------------------------------------ */
/* exported scalar and vector field primitives (which: 0 = Fr, 1 = Fq) */

void or_field_consts(int which, u64 *m, u64 *one, u64 *r2, u64 *inv) {
    or_init();
    const fdesc *f = F(which);
    memcpy(m, f->m, 32);
    memcpy(one, f->one, 32);
    memcpy(r2, f->r2, 32);
    *inv = f->inv;
}

void or_vec_add(int which, u64 *r, const u64 *a, const u64 *b, long n) {
    or_init();
    const fdesc *f = F(which);
#pragma omp parallel for if (n > 65536)
    for (long i = 0; i < n; i++) f_add(f, r + 4 * i, a + 4 * i, b + 4 * i);
}
void or_vec_sub(int which, u64 *r, const u64 *a, const u64 *b, long n) {
    or_init();
    const fdesc *f = F(which);
#pragma omp parallel for if (n > 65536)
    for (long i = 0; i < n; i++) f_sub(f, r + 4 * i, a + 4 * i, b + 4 * i);
}
void or_vec_mul(int which, u64 *r, const u64 *a, const u64 *b, long n) {
    or_init();
    const fdesc *f = F(which);
#pragma omp parallel for if (n > 16384)
    for (long i = 0; i < n; i++) f_mul(f, r + 4 * i, a + 4 * i, b + 4 * i);
}
/* r[i] = a[i] * b[0] */
void or_vec_mul_scalar(int which, u64 *r, const u64 *a, const u64 *b, long n) {
    or_init();
    const fdesc *f = F(which);
    u64 s[4];
    memcpy(s, b, 32);
#pragma omp parallel for if (n > 16384)
    for (long i = 0; i < n; i++) f_mul(f, r + 4 * i, a + 4 * i, s);
}
void or_vec_neg(int which, u64 *r, const u64 *a, long n) {
    or_init();
    const fdesc *f = F(which);
    for (long i = 0; i < n; i++) f_neg(f, r + 4 * i, a + 4 * i);
}
void or_vec_to_mont(int which, u64 *r, const u64 *a, long n) {
    or_init();
    const fdesc *f = F(which);
#pragma omp parallel for if (n > 16384)
    for (long i = 0; i < n; i++) f_to_mont(f, r + 4 * i, a + 4 * i);
}
void or_vec_from_mont(int which, u64 *r, const u64 *a, long n) {
    or_init();
    const fdesc *f = F(which);
#pragma omp parallel for if (n > 16384)
    for (long i = 0; i < n; i++) f_from_mont(f, r + 4 * i, a + 4 * i);
}
void or_vec_inv(int which, u64 *r, const u64 *a, long n) {
    or_init();
    const fdesc *f = F(which);
#pragma omp parallel for if (n > 64)
    for (long i = 0; i < n; i++) f_inv(f, r + 4 * i, a + 4 * i);
}
/* r = a^e with e a canonical 256-bit exponent (4 x u64) */
void or_pow(int which, u64 *r, const u64 *a, const u64 *e) {
    or_init();
    f_pow_u64(F(which), r, a, e);
}

/* Montgomery batch inversion (zeros stay zero), sequential: the reference's
 * batch_invert semantics (src/permutation.rs:73-75, cuda/bn254.cu:92-115). */
void or_batch_inv(u64 *r, const u64 *a, long n) {
    or_init();
    const fdesc *f = &FR;
    u64 *pre = (u64 *)malloc(sizeof(u64) * 4 * (n + 1));
    u64 acc[4];
    memcpy(acc, f->one, 32);
    for (long i = 0; i < n; i++) {
        memcpy(pre + 4 * i, acc, 32);
        if (!f_is_zero(a + 4 * i)) f_mul(f, acc, acc, a + 4 * i);
    }
    u64 inv[4];
    f_inv(f, inv, acc);
    for (long i = n - 1; i >= 0; i--) {
        if (f_is_zero(a + 4 * i)) {
            memset(r + 4 * i, 0, 32);
            continue;
        }
        u64 ai[4];
        memcpy(ai, a + 4 * i, 32);
        f_mul(f, r + 4 * i, inv, pre + 4 * i);
        f_mul(f, inv, inv, ai);
    }
    free(pre);
}

/* Exclusive prefix product: r[0] = init, r[i] = init * a[0] * ... * a[i-1]. */
void or_prefix_product_excl(u64 *r, const u64 *a, const u64 *init, long n) {
    or_init();
    u64 acc[4];
    memcpy(acc, init, 32);
    for (long i = 0; i < n; i++) {
        u64 ai[4];
        memcpy(ai, a + 4 * i, 32);
        memcpy(r + 4 * i, acc, 32);
        f_mul(&FR, acc, acc, ai);
    }
}

/* Exclusive prefix sum: r[0] = init, r[i] = init + a[0] + ... + a[i-1]. */
void or_prefix_sum_excl(u64 *r, const u64 *a, const u64 *init, long n) {
    or_init();
    u64 acc[4];
    memcpy(acc, init, 32);
    for (long i = 0; i < n; i++) {
        u64 ai[4];
        memcpy(ai, a + 4 * i, 32);
        memcpy(r + 4 * i, acc, 32);
        f_add(&FR, acc, acc, ai);
    }
}

/* ------------------------------------------------------------------ */
/* NTT: natural order in and out, X[j] = sum_i x[i] omega^(ij).       */

static void bit_reverse_perm(u64 *a, int log_n) {
    long n = 1L << log_n;
    for (long i = 0; i < n; i++) {
        long j = 0;
        for (int b = 0; b < log_n; b++) j |= ((i >> b) & 1) << (log_n - 1 - b);
        if (j > i) {
            u64 t[4];
            memcpy(t, a + 4 * i, 32);
            memcpy(a + 4 * i, a + 4 * j, 32);
            memcpy(a + 4 * j, t, 32);
        }
    }
}

/* In-place NTT by omega (Montgomery form, a primitive 2^log_n-th root). */
void or_ntt(u64 *a, int log_n, const u64 *omega) {
    or_init();
    const fdesc *f = &FR;
    long n = 1L << log_n;
    if (log_n == 0) return;
    bit_reverse_perm(a, log_n);
    /* twiddle table w^i for i < n/2 */
    u64 *tw = (u64 *)malloc(sizeof(u64) * 4 * (n / 2));
    memcpy(tw, f->one, 32);
    for (long i = 1; i < n / 2; i++) f_mul(f, tw + 4 * i, tw + 4 * (i - 1), omega);
    for (int s = 1; s <= log_n; s++) {
        long m = 1L << s, half = m >> 1, step = n / m;
#pragma omp parallel for if (n >= 4096)
        for (long idx = 0; idx < n / 2; idx++) {
            long blk = idx / half, j = idx % half;
            long i0 = blk * m + j, i1 = i0 + half;
            u64 t[4], u[4];
            f_mul(f, t, a + 4 * i1, tw + 4 * (j * step));
            memcpy(u, a + 4 * i0, 32);
            f_add(f, a + 4 * i0, u, t);
            f_sub(f, a + 4 * i1, u, t);
        }
    }
    free(tw);
}

/* In-place inverse NTT: NTT by omega^-1 then scale by n^-1. */
void or_intt(u64 *a, int log_n, const u64 *omega) {
    or_init();
    const fdesc *f = &FR;
    long n = 1L << log_n;
    u64 winv[4], ninv[4], nn[4] = {(u64)n, 0, 0, 0};
    f_inv(f, winv, omega);
    or_ntt(a, log_n, winv);
    f_to_mont(f, nn, nn);
    f_inv(f, ninv, nn);
#pragma omp parallel for if (n >= 16384)
    for (long i = 0; i < n; i++) f_mul(f, a + 4 * i, a + 4 * i, ninv);
}

/* out[i] = base^i for i < n (Montgomery in and out) */
/* The division the reference runs on the host after the multi-open batching
 * (src/multiopen.rs:145-159 GWC, 543-553 SHPLONK), step by step: tmp = a[n-1],
 * a[n-1] = 0, then for i = n-2 .. 1: p = a[i] + tmp z, a[i] = tmp, tmp = p;
 * a[0] = tmp.  In place on n Montgomery-form coefficients (n >= 2). */
void or_poly_divide_linear(u64 *a, const u64 *z, long n) {
    u64 tmp[4], p[4], t[4];
    memcpy(tmp, a + 4 * (n - 1), 32);
    memset(a + 4 * (n - 1), 0, 32);
    for (long i = n - 2; i >= 1; i--) {
        f_mul(&FR, t, tmp, z);
        f_add(&FR, p, a + 4 * i, t);
        memcpy(a + 4 * i, tmp, 32);
        memcpy(tmp, p, 32);
    }
    memcpy(a, tmp, 32);
}

void or_powers(u64 *out, const u64 *base, long n) {
    or_init();
    const fdesc *f = &FR;
    if (n <= 0) return;
    memcpy(out, f->one, 32);
    for (long i = 1; i < n; i++) f_mul(f, out + 4 * i, out + 4 * (i - 1), base);
}

/* Coset extension of one column: out[j] = sum_i c_i (shift * wN^j)^i for
 * j < 2^(log_n + ext_bits); c_i scaled by shift^i, zero padded, one NTT. */
void or_coset_extend(u64 *out, const u64 *coeffs, int log_n, int ext_bits, const u64 *shift, const u64 *w_ext) {
    or_init();
    const fdesc *f = &FR;
    long n = 1L << log_n, N = n << ext_bits;
    u64 *pw = (u64 *)malloc(sizeof(u64) * 4 * n);
    or_powers(pw, shift, n);
#pragma omp parallel for if (n >= 16384)
    for (long i = 0; i < n; i++) f_mul(f, out + 4 * i, coeffs + 4 * i, pw + 4 * i);
    memset(out + 4 * n, 0, sizeof(u64) * 4 * (N - n));
    free(pw);
    or_ntt(out, log_n + ext_bits, w_ext);
}

/* Naive O(n^2) DFT, used to pin or_ntt on small sizes. */
void or_dft_naive(u64 *out, const u64 *a, int log_n, const u64 *omega) {
    or_init();
    const fdesc *f = &FR;
    long n = 1L << log_n;
    for (long j = 0; j < n; j++) {
        u64 acc[4] = {0, 0, 0, 0}, wj[4], w[4];
        /* wj = omega^j */
        memcpy(wj, f->one, 32);
        for (long k = 0; k < j; k++) f_mul(f, wj, wj, omega);
        memcpy(w, f->one, 32);
        for (long i = 0; i < n; i++) {
            u64 t[4];
            f_mul(f, t, a + 4 * i, w);
            f_add(f, acc, acc, t);
            f_mul(f, w, w, wj);
        }
        memcpy(out + 4 * j, acc, 32);
    }
}

/* ------------------------------------------------------------------ */
/* G1: y^2 = x^3 + 3 over Fq.  Jacobian (X, Y, Z): x = X/Z^2, y = Y/Z^3. */

typedef struct { u64 x[4], y[4], z[4]; } jac;
typedef struct { u64 x[4], y[4]; } aff;

static inline int aff_is_id(const aff *p) { return f_is_zero(p->x) && f_is_zero(p->y); }
static inline int jac_is_id(const jac *p) { return f_is_zero(p->z); }
static inline void jac_set_id(jac *p) {
    memset(p->x, 0, 32);
    memcpy(p->y, FQ.one, 32);
    memset(p->z, 0, 32);
}

/* dbl-2009-l (a = 0) */
static void jac_dbl(jac *r, const jac *p) {
    const fdesc *f = &FQ;
    if (jac_is_id(p)) { *r = *p; return; }
    u64 A[4], B[4], C[4], D[4], E[4], Fv[4], t[4], z3[4];
    f_sqr(f, A, p->x);
    f_sqr(f, B, p->y);
    f_sqr(f, C, B);
    f_add(f, t, p->x, B);
    f_sqr(f, t, t);
    f_sub(f, t, t, A);
    f_sub(f, t, t, C);
    f_add(f, D, t, t);
    f_add(f, E, A, A);
    f_add(f, E, E, A);
    f_sqr(f, Fv, E);
    f_mul(f, z3, p->y, p->z);
    f_add(f, z3, z3, z3);
    u64 x3[4], y3[4];
    f_sub(f, x3, Fv, D);
    f_sub(f, x3, x3, D);
    f_sub(f, t, D, x3);
    f_mul(f, y3, E, t);
    f_add(f, C, C, C);
    f_add(f, C, C, C);
    f_add(f, C, C, C);
    f_sub(f, y3, y3, C);
    memcpy(r->x, x3, 32);
    memcpy(r->y, y3, 32);
    memcpy(r->z, z3, 32);
}

/* General Jacobian addition (add-2007-bl shape, with the doubling case). */
static void jac_add(jac *r, const jac *p, const jac *q) {
    const fdesc *f = &FQ;
    if (jac_is_id(p)) { *r = *q; return; }
    if (jac_is_id(q)) { *r = *p; return; }
    u64 z1z1[4], z2z2[4], u1[4], u2[4], s1[4], s2[4], t[4];
    f_sqr(f, z1z1, p->z);
    f_sqr(f, z2z2, q->z);
    f_mul(f, u1, p->x, z2z2);
    f_mul(f, u2, q->x, z1z1);
    f_mul(f, t, q->z, z2z2);
    f_mul(f, s1, p->y, t);
    f_mul(f, t, p->z, z1z1);
    f_mul(f, s2, q->y, t);
    if (memcmp(u1, u2, 32) == 0) {
        if (memcmp(s1, s2, 32) == 0) { jac_dbl(r, p); return; }
        jac_set_id(r);
        return;
    }
    u64 h[4], i[4], j[4], rr[4], v[4], x3[4], y3[4], z3[4];
    f_sub(f, h, u2, u1);
    f_add(f, i, h, h);
    f_sqr(f, i, i);
    f_mul(f, j, h, i);
    f_sub(f, rr, s2, s1);
    f_add(f, rr, rr, rr);
    f_mul(f, v, u1, i);
    f_sqr(f, x3, rr);
    f_sub(f, x3, x3, j);
    f_sub(f, x3, x3, v);
    f_sub(f, x3, x3, v);
    f_sub(f, t, v, x3);
    f_mul(f, y3, rr, t);
    f_mul(f, t, s1, j);
    f_add(f, t, t, t);
    f_sub(f, y3, y3, t);
    f_add(f, z3, p->z, q->z);
    f_sqr(f, z3, z3);
    f_sub(f, z3, z3, z1z1);
    f_sub(f, z3, z3, z2z2);
    f_mul(f, z3, z3, h);
    memcpy(r->x, x3, 32);
    memcpy(r->y, y3, 32);
    memcpy(r->z, z3, 32);
}

static void jac_add_aff(jac *r, const jac *p, const aff *q) {
    if (aff_is_id(q)) { *r = *p; return; }
    jac t;
    memcpy(t.x, q->x, 32);
    memcpy(t.y, q->y, 32);
    memcpy(t.z, FQ.one, 32);
    jac_add(r, p, &t);
}

static void jac_to_aff(aff *r, const jac *p) {
    const fdesc *f = &FQ;
    if (jac_is_id(p)) { memset(r, 0, sizeof(*r)); return; }
    u64 zi[4], zi2[4], zi3[4];
    f_inv(f, zi, p->z);
    f_sqr(f, zi2, zi);
    f_mul(f, zi3, zi2, zi);
    f_mul(f, r->x, p->x, zi2);
    f_mul(f, r->y, p->y, zi3);
}

/* scalar given canonical (not Montgomery), 4 x u64 */
static void jac_scalar_mul(jac *r, const jac *p, const u64 k[4]) {
    jac acc;
    jac_set_id(&acc);
    for (int i = 255; i >= 0; i--) {
        jac_dbl(&acc, &acc);
        if ((k[i / 64] >> (i % 64)) & 1) jac_add(&acc, &acc, p);
    }
    *r = acc;
}

/* ---- exported G1 helpers; points are arrays of u64 (affine: 8, jacobian: 12) ---- */

void or_g1_generator(u64 *out_aff) {
    or_init();
    u64 one[4] = {1, 0, 0, 0}, two[4] = {2, 0, 0, 0};
    f_to_mont(&FQ, out_aff, one);
    f_to_mont(&FQ, out_aff + 4, two);
}

int or_g1_is_on_curve(const u64 *p_aff) {
    or_init();
    const aff *p = (const aff *)p_aff;
    if (aff_is_id(p)) return 1;
    u64 y2[4], x3[4], three[4] = {3, 0, 0, 0}, b[4];
    f_sqr(&FQ, y2, p->y);
    f_sqr(&FQ, x3, p->x);
    f_mul(&FQ, x3, x3, p->x);
    f_to_mont(&FQ, b, three);
    f_add(&FQ, x3, x3, b);
    return memcmp(x3, y2, 32) == 0;
}

void or_g1_jac_to_aff(u64 *out_aff, const u64 *p_jac, long n) {
    or_init();
#pragma omp parallel for if (n > 64)
    for (long i = 0; i < n; i++) jac_to_aff((aff *)(out_aff + 8 * i), (const jac *)(p_jac + 12 * i));
}

void or_g1_add_jac(u64 *r, const u64 *p, const u64 *q) {
    or_init();
    jac t;
    jac_add(&t, (const jac *)p, (const jac *)q);
    memcpy(r, &t, sizeof(t));
}

void or_g1_dbl_jac(u64 *r, const u64 *p) {
    or_init();
    jac t;
    jac_dbl(&t, (const jac *)p);
    memcpy(r, &t, sizeof(t));
}

/* [k]P for affine P and Montgomery-form scalar k; result affine. */
void or_g1_mul_aff(u64 *out_aff, const u64 *p_aff, const u64 *k_mont) {
    or_init();
    jac p, r;
    const aff *a = (const aff *)p_aff;
    if (aff_is_id(a)) { memset(out_aff, 0, 64); return; }
    memcpy(p.x, a->x, 32);
    memcpy(p.y, a->y, 32);
    memcpy(p.z, FQ.one, 32);
    u64 k[4];
    f_from_mont(&FR, k, k_mont);
    jac_scalar_mul(&r, &p, k);
    jac_to_aff((aff *)out_aff, &r);
}

/* Fixed-base generation: out[i] = [k_i]G (affine), k_i Montgomery-form Fr.
 * Comb of 8-bit windows: table[w][d] = [d * 2^(8w)]G. */
void or_g1_gen_bases(u64 *out_aff, const u64 *k_mont, long n) {
    or_init();
    jac *tab = (jac *)malloc(sizeof(jac) * 32 * 256);
    jac g;
    u64 ga[8];
    or_g1_generator(ga);
    memcpy(g.x, ga, 32);
    memcpy(g.y, ga + 4, 32);
    memcpy(g.z, FQ.one, 32);
    jac base = g;
    for (int w = 0; w < 32; w++) {
        jac_set_id(&tab[w * 256]);
        for (int d = 1; d < 256; d++) jac_add(&tab[w * 256 + d], &tab[w * 256 + d - 1], &base);
        for (int b = 0; b < 8; b++) jac_dbl(&base, &base);
    }
    jac *tmp = (jac *)malloc(sizeof(jac) * n);
#pragma omp parallel for schedule(static)
    for (long i = 0; i < n; i++) {
        u64 k[4];
        f_from_mont(&FR, k, k_mont + 4 * i);
        jac acc;
        jac_set_id(&acc);
        for (int w = 0; w < 32; w++) {
            int d = (int)((k[w / 8] >> ((w % 8) * 8)) & 0xff);
            if (d) jac_add(&acc, &acc, &tab[w * 256 + d]);
        }
        tmp[i] = acc;
    }
    /* batch normalisation with Montgomery's trick, in chunks per thread */
#pragma omp parallel
    {
        int nt = omp_get_num_threads(), id = omp_get_thread_num();
        long chunk = (n + nt - 1) / nt, s = id * chunk, e = s + chunk > n ? n : s + chunk;
        if (s < e) {
            u64 *pre = (u64 *)malloc(sizeof(u64) * 4 * (e - s));
            u64 acc[4];
            memcpy(acc, FQ.one, 32);
            for (long i = s; i < e; i++) {
                memcpy(pre + 4 * (i - s), acc, 32);
                if (!jac_is_id(&tmp[i])) f_mul(&FQ, acc, acc, tmp[i].z);
            }
            u64 inv[4];
            f_inv(&FQ, inv, acc);
            for (long i = e - 1; i >= s; i--) {
                aff *o = (aff *)(out_aff + 8 * i);
                if (jac_is_id(&tmp[i])) { memset(o, 0, 64); continue; }
                u64 zi[4], zi2[4], zi3[4];
                f_mul(&FQ, zi, inv, pre + 4 * (i - s));
                f_mul(&FQ, inv, inv, tmp[i].z);
                f_sqr(&FQ, zi2, zi);
                f_mul(&FQ, zi3, zi2, zi);
                f_mul(&FQ, o->x, tmp[i].x, zi2);
                f_mul(&FQ, o->y, tmp[i].y, zi3);
            }
            free(pre);
        }
    }
    free(tmp);
    free(tab);
}

/* Pippenger MSM: out = sum_i [k_i] P_i, as an affine point.
 * Windows are split across threads; each thread accumulates its windows'
 * buckets with mixed additions and reduces them by running sums.
 * c is the window width in bits (0: pick from n). */
void or_msm(u64 *out_aff, const u64 *bases_aff, const u64 *k_mont, long n, int c) {
    or_init();
    if (c <= 0) {
        c = 1;
        while ((1L << (c + 1)) * (c + 1) < n * 2 && c < 16) c++;
        if (c < 4) c = 4;
    }
    int W = (254 + c - 1) / c;
    u64 *ks = (u64 *)malloc(sizeof(u64) * 4 * n);
#pragma omp parallel for if (n > 16384)
    for (long i = 0; i < n; i++) f_from_mont(&FR, ks + 4 * i, k_mont + 4 * i);
    jac *wsum = (jac *)malloc(sizeof(jac) * W);
    long nb = 1L << c;
#pragma omp parallel for schedule(dynamic, 1)
    for (int w = 0; w < W; w++) {
        jac *b = (jac *)malloc(sizeof(jac) * nb);
        for (long j = 0; j < nb; j++) jac_set_id(&b[j]);
        int sb = w * c;
        for (long i = 0; i < n; i++) {
            const u64 *k = ks + 4 * i;
            int limb = sb / 64, off = sb % 64;
            u64 d = k[limb] >> off;
            if (off + c > 64 && limb < 3) d |= k[limb + 1] << (64 - off);
            d &= (u64)(nb - 1);
            if (d) jac_add_aff(&b[d], &b[d], (const aff *)(bases_aff + 8 * i));
        }
        jac run, acc;
        jac_set_id(&run);
        jac_set_id(&acc);
        for (long j = nb - 1; j >= 1; j--) {
            jac_add(&run, &run, &b[j]);
            jac_add(&acc, &acc, &run);
        }
        wsum[w] = acc;
        free(b);
    }
    jac r;
    jac_set_id(&r);
    for (int w = W - 1; w >= 0; w--) {
        for (int i = 0; i < c; i++) jac_dbl(&r, &r);
        jac_add(&r, &r, &wsum[w]);
    }
    jac_to_aff((aff *)out_aff, &r);
    free(wsum);
    free(ks);
}

/* sum_i a_i * b_i over Fr (Montgomery in/out), used by the known-discrete-log
 * MSM identity: if P_i = [b_i]G then MSM(P, a) = [sum a_i b_i]G. */
void or_inner_product(u64 *out, const u64 *a, const u64 *b, long n) {
    or_init();
    int nt = omp_get_max_threads();
    u64 *part = (u64 *)calloc((size_t)nt * 4, sizeof(u64));
#pragma omp parallel
    {
        int id = omp_get_thread_num(), T = omp_get_num_threads();
        u64 acc[4] = {0, 0, 0, 0};
        for (long i = id; i < n; i += T) {
            u64 t[4];
            f_mul(&FR, t, a + 4 * i, b + 4 * i);
            f_add(&FR, acc, acc, t);
        }
        memcpy(part + 4 * id, acc, 32);
    }
    u64 acc[4] = {0, 0, 0, 0};
    for (int i = 0; i < nt; i++) f_add(&FR, acc, acc, part + 4 * i);
    memcpy(out, acc, 32);
    free(part);
}

/* Deterministic seeded uniform Fr generation (splitmix64 + rejection below r),
 * returned in Montgomery form. */
static inline u64 splitmix64(u64 *s) {
    u64 z = (*s += 0x9e3779b97f4a7c15ULL);
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
    return z ^ (z >> 31);
}

void or_rand_fr(u64 *out, long n, u64 seed) {
    or_init();
#pragma omp parallel for if (n > 65536)
    for (long blk = 0; blk < (n + 4095) / 4096; blk++) {
        u64 s = seed ^ (0xd1b54a32d192ed03ULL * (u64)(blk + 1));
        long e = (blk + 1) * 4096 > n ? n : (blk + 1) * 4096;
        for (long i = blk * 4096; i < e; i++) {
            u64 v[4];
            do {
                for (int j = 0; j < 4; j++) v[j] = splitmix64(&s);
                v[3] &= 0x3fffffffffffffffULL;
            } while (geq(v, FR.m));
            f_to_mont(&FR, out + 4 * i, v);
        }
    }
}
