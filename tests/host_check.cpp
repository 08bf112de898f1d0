// Host build of the device field and curve code (csrc/field.cuh, csrc/curve.cuh)
// for the CPU test-suite: without __CUDA_ARCH__ the PTX carry chains fall back
// to a C emulation of the same instruction sequence, so these entry points run
// the device algorithms on the CPU against the oracle.
#include <string.h>
#include "../zkwasm-prover_b200/csrc/curve.cuh"

using namespace zk;

template <class C>
static Fe<C> ld(const uint64_t* p) {
    Fe<C> r;
    memcpy(r.v, p, 32);
    return r;
}
template <class C>
static void st(uint64_t* p, const Fe<C>& v) {
    memcpy(p, v.v, 32);
}

extern "C" {

void hc_mul(int which, uint64_t* out, const uint64_t* a, const uint64_t* b, long n) {
    for (long i = 0; i < n; i++) {
        if (which == 0)
            st(out + 4 * i, fe_mul<FrCfg>(ld<FrCfg>(a + 4 * i), ld<FrCfg>(b + 4 * i)));
        else
            st(out + 4 * i, fe_mul<FqCfg>(ld<FqCfg>(a + 4 * i), ld<FqCfg>(b + 4 * i)));
    }
}

void hc_add(int which, uint64_t* out, const uint64_t* a, const uint64_t* b, long n) {
    for (long i = 0; i < n; i++) {
        if (which == 0)
            st(out + 4 * i, fe_add<FrCfg>(ld<FrCfg>(a + 4 * i), ld<FrCfg>(b + 4 * i)));
        else
            st(out + 4 * i, fe_add<FqCfg>(ld<FqCfg>(a + 4 * i), ld<FqCfg>(b + 4 * i)));
    }
}

void hc_sub(int which, uint64_t* out, const uint64_t* a, const uint64_t* b, long n) {
    for (long i = 0; i < n; i++) {
        if (which == 0)
            st(out + 4 * i, fe_sub<FrCfg>(ld<FrCfg>(a + 4 * i), ld<FrCfg>(b + 4 * i)));
        else
            st(out + 4 * i, fe_sub<FqCfg>(ld<FqCfg>(a + 4 * i), ld<FqCfg>(b + 4 * i)));
    }
}

void hc_inv(uint64_t* out, const uint64_t* a, long n) {
    for (long i = 0; i < n; i++) st(out + 4 * i, fe_inv<FrCfg>(ld<FrCfg>(a + 4 * i)));
}

void hc_from_mont(uint64_t* out, const uint64_t* a, long n) {
    for (long i = 0; i < n; i++) st(out + 4 * i, fe_from_mont<FrCfg>(ld<FrCfg>(a + 4 * i)));
}

void hc_pow(uint64_t* out, const uint64_t* a, uint32_t e) { st(out, fe_pow_u32<FrCfg>(ld<FrCfg>(a), e)); }

uint32_t hc_bits_at(const uint64_t* k, uint32_t start, uint32_t nbits) {
    uint32_t v[8];
    memcpy(v, k, 32);
    return bits_at(v, start, nbits);
}

// XYZZ points as 16 u64; affine as 8; Jacobian as 12
static Xyzz ldx(const uint64_t* p) {
    Xyzz r;
    r.x = ld<FqCfg>(p);
    r.y = ld<FqCfg>(p + 4);
    r.zz = ld<FqCfg>(p + 8);
    r.zzz = ld<FqCfg>(p + 12);
    return r;
}
static void stx(uint64_t* p, const Xyzz& v) {
    st(p, v.x);
    st(p + 4, v.y);
    st(p + 8, v.zz);
    st(p + 12, v.zzz);
}

void hc_xyzz_from_aff(uint64_t* out, const uint64_t* a) {
    Aff q;
    q.x = ld<FqCfg>(a);
    q.y = ld<FqCfg>(a + 4);
    stx(out, xyzz_from_aff(q));
}

void hc_xyzz_add_aff(uint64_t* out, const uint64_t* p, const uint64_t* a) {
    stx(out, xyzz_add_aff(ldx(p), ld<FqCfg>(a), ld<FqCfg>(a + 4)));
}

void hc_xyzz_add(uint64_t* out, const uint64_t* p, const uint64_t* q) { stx(out, xyzz_add(ldx(p), ldx(q))); }

void hc_xyzz_dbl(uint64_t* out, const uint64_t* p) { stx(out, xyzz_dbl(ldx(p))); }

void hc_xyzz_mul_u32(uint64_t* out, const uint64_t* p, uint32_t k) { stx(out, xyzz_mul_u32(ldx(p), k)); }

void hc_xyzz_to_jac(uint64_t* out, const uint64_t* p) {
    Jac j = xyzz_to_jac(ldx(p));
    st(out, j.x);
    st(out + 4, j.y);
    st(out + 8, j.z);
}

}  // extern "C"

extern "C" int hc_signed_digit(const uint64_t* k, int w, int c, uint32_t* carry) {
    uint32_t v[8];
    memcpy(v, k, 32);
    return msm_signed_digit(v, w, c, *carry);
}

#include "../zkwasm-prover_b200/csrc/glv.cuh"

// k: canonical scalars (4 x u64); m1, m2: magnitudes; neg: two flags per scalar
extern "C" void hc_glv_split(const uint64_t* k, uint64_t* m1, uint64_t* m2, int* neg, long n) {
    for (long i = 0; i < n; i++) {
        uint32_t kv[8], a[8], b[8];
        memcpy(kv, k + 4 * i, 32);
        bool n1, n2;
        glv_split(kv, a, b, n1, n2);
        memcpy(m1 + 4 * i, a, 32);
        memcpy(m2 + 4 * i, b, 32);
        neg[2 * i] = n1;
        neg[2 * i + 1] = n2;
    }
}

// affine points (8 x u64 each, Montgomery) -> phi(points)
extern "C" void hc_glv_phi(uint64_t* out, const uint64_t* pts, long n) {
    for (long i = 0; i < n; i++) {
        Aff a;
        memcpy(a.x.v, pts + 8 * i, 32);
        memcpy(a.y.v, pts + 8 * i + 4, 32);
        const Aff r = glv_phi(a);
        memcpy(out + 8 * i, r.x.v, 32);
        memcpy(out + 8 * i + 4, r.y.v, 32);
    }
}

// lazily reduced operations on inputs in [0, 2m): op 0 mul, 1 add, 2 sub over
// Fr; 3, 4, 5 the same over Fq
template <class C>
static Fe<C> lazy_op(int op, const Fe<C>& x, const Fe<C>& y) {
    return op == 0 ? fe_mul_lazy<C>(x, y) : op == 1 ? fe_add_lazy<C>(x, y) : fe_sub_lazy<C>(x, y);
}

extern "C" void hc_lazy(int op, uint64_t* out, const uint64_t* a, const uint64_t* b, long n) {
    for (long i = 0; i < n; i++) {
        if (op < 3)
            st(out + 4 * i, lazy_op<FrCfg>(op, ld<FrCfg>(a + 4 * i), ld<FrCfg>(b + 4 * i)));
        else
            st(out + 4 * i, lazy_op<FqCfg>(op - 3, ld<FqCfg>(a + 4 * i), ld<FqCfg>(b + 4 * i)));
    }
}

// a chain of n lazily reduced mixed additions onto acc (16 words, coordinates
// in [0, 2p)), canonical result
extern "C" void hc_madd_lazy_chain(uint64_t* out, const uint64_t* acc, const uint64_t* pts, long n) {
    Xyzz a;
    a.x = ld<FqCfg>(acc);
    a.y = ld<FqCfg>(acc + 4);
    a.zz = ld<FqCfg>(acc + 8);
    a.zzz = ld<FqCfg>(acc + 12);
    for (long i = 0; i < n; i++) a = xyzz_add_aff_lazy(a, ld<FqCfg>(pts + 8 * i), ld<FqCfg>(pts + 8 * i + 4));
    a = xyzz_canon(a);
    st(out, a.x);
    st(out + 4, a.y);
    st(out + 8, a.zz);
    st(out + 12, a.zzz);
}

// Fr products by a known factor: out = fe_mul_shoup(a, w, wp)
extern "C" void hc_mul_shoup(uint64_t* out, const uint64_t* a, const uint64_t* w, const uint64_t* wp, long n) {
    for (long i = 0; i < n; i++)
        st(out + 4 * i, fe_mul_shoup<FrCfg>(ld<FrCfg>(a + 4 * i), ld<FrCfg>(w + 4 * i), ld<FrCfg>(wp + 4 * i)));
}
