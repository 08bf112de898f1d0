// Device helpers shared by the single and the batched MSM pipelines: point
// loads / stores and the final window combination.
#pragma once
#include "common.cuh"

namespace zk {

__device__ __forceinline__ Aff ld_aff(const Aff* p) {
    Aff a;
    a.x = ldg_elem<FqCfg>(&p->x);
    a.y = ldg_elem<FqCfg>(&p->y);
    return a;
}

__device__ __forceinline__ Xyzz ld_xyzz(const Xyzz* p) {
    Xyzz r;
    r.x = ld_elem<FqCfg>(&p->x);
    r.y = ld_elem<FqCfg>(&p->y);
    r.zz = ld_elem<FqCfg>(&p->zz);
    r.zzz = ld_elem<FqCfg>(&p->zzz);
    return r;
}

__device__ __forceinline__ void st_xyzz(Xyzz* p, const Xyzz& v) {
    st_elem<FqCfg>(&p->x, v.x);
    st_elem<FqCfg>(&p->y, v.y);
    st_elem<FqCfg>(&p->zz, v.zz);
    st_elem<FqCfg>(&p->zzz, v.zzz);
}

// ---------------------------------------------------------------------------
// Final combination  sum_w 2^(c w) S_w  (Horner, (W - 1) c doublings).
//
// It is one dependent chain, so its time is the latency of the products on
// the chain.  One warp's Fq product is bound by the multiply pipe of its SM
// sub-partition, so a thread cannot overlap two products; instead a CTA of
// four warps (one per sub-partition) evaluates up to four independent products
// of a formula at once: lane 0 of warp k computes product k, the results meet
// in shared memory, and every thread keeps the whole point in registers and
// does the additions itself.  A doubling (6M + 3S) becomes three product
// levels, an addition (12M + 2S) four.

static constexpr int COOP_THREADS = 128;

struct Coop {
    Fq* buf;  // shared, 2 x 4 elements (double-buffered result slots)
    int par;
};

// r_k = a_k * b_k for k < cnt, all threads receive every result
template <int CNT>
__device__ __forceinline__ void coop_mul(Coop& co, const Fq& a0, const Fq& b0, const Fq& a1, const Fq& b1,
                                         const Fq& a2, const Fq& b2, const Fq& a3, const Fq& b3, Fq& r0, Fq& r1,
                                         Fq& r2, Fq& r3) {
    const int wp = threadIdx.x >> 5;
    Fq* slot = co.buf + 4 * co.par;
    if ((threadIdx.x & 31) == 0 && wp < CNT) {
        const Fq a = wp == 0 ? a0 : wp == 1 ? a1 : wp == 2 ? a2 : a3;
        const Fq b = wp == 0 ? b0 : wp == 1 ? b1 : wp == 2 ? b2 : b3;
        slot[wp] = fe_mul<FqCfg>(a, b);
    }
    __syncthreads();
    r0 = slot[0];
    if (CNT > 1) r1 = slot[1];
    if (CNT > 2) r2 = slot[2];
    if (CNT > 3) r3 = slot[3];
    // the next call writes the other slot set; this one is rewritten only
    // after every thread has passed the next barrier, i.e. read these results
    co.par ^= 1;
}

// 2 * p, dbl-2008-s-1 in three product levels
__device__ __forceinline__ Xyzz coop_dbl(Coop& co, const Xyzz& p) {
    if (xyzz_is_id(p)) return p;
    Fq d = fe_zero<FqCfg>();
    const Fq u = fe_dbl<FqCfg>(p.y);
    Fq v, xx;
    coop_mul<2>(co, u, u, p.x, p.x, d, d, d, d, v, xx, d, d);
    const Fq mm = fe_add<FqCfg>(fe_dbl<FqCfg>(xx), xx);
    Fq w, s, m2, zz;
    coop_mul<4>(co, u, v, p.x, v, mm, mm, v, p.zz, w, s, m2, zz);
    Xyzz r;
    r.x = fe_sub<FqCfg>(fe_sub<FqCfg>(m2, s), s);
    const Fq t = fe_sub<FqCfg>(s, r.x);
    Fq zzz, wy, mt;
    coop_mul<3>(co, w, p.zzz, w, p.y, mm, t, d, d, zzz, wy, mt, d);
    r.y = fe_sub<FqCfg>(mt, wy);
    r.zz = zz;
    r.zzz = zzz;
    return r;
}

// p + q, add-2008-s in four product levels
__device__ __forceinline__ Xyzz coop_add(Coop& co, const Xyzz& p, const Xyzz& q) {
    if (xyzz_is_id(p)) return q;
    if (xyzz_is_id(q)) return p;
    Fq d = fe_zero<FqCfg>();
    Fq u1, u2, s1, s2;
    coop_mul<4>(co, p.x, q.zz, q.x, p.zz, p.y, q.zzz, q.y, p.zzz, u1, u2, s1, s2);
    const Fq P = fe_sub<FqCfg>(u2, u1);
    const Fq R = fe_sub<FqCfg>(s2, s1);
    if (fe_is_zero<FqCfg>(P)) {
        if (fe_is_zero<FqCfg>(R)) return coop_dbl(co, p);
        return xyzz_identity();
    }
    Fq pp, zzp, zzzp, rr;
    coop_mul<4>(co, P, P, p.zz, q.zz, p.zzz, q.zzz, R, R, pp, zzp, zzzp, rr);
    Fq ppp, qq, zz;
    coop_mul<3>(co, P, pp, u1, pp, zzp, pp, d, d, ppp, qq, zz, d);
    Xyzz r;
    r.x = fe_sub<FqCfg>(fe_sub<FqCfg>(fe_sub<FqCfg>(rr, ppp), qq), qq);
    const Fq t = fe_sub<FqCfg>(qq, r.x);
    Fq zzz, sp, rt;
    coop_mul<3>(co, zzzp, ppp, s1, ppp, R, t, d, d, zzz, sp, rt, d);
    r.y = fe_sub<FqCfg>(rt, sp);
    r.zz = zz;
    r.zzz = zzz;
    return r;
}

// XYZZ -> Jacobian (X ZZ^2, Y ZZ^3, ZZZ); identity -> (0, 1, 0)
__device__ __forceinline__ Jac coop_to_jac(Coop& co, const Xyzz& p) {
    Jac r;
    if (xyzz_is_id(p)) {
        r.x = fe_zero<FqCfg>();
        r.y = fe_one<FqCfg>();
        r.z = fe_zero<FqCfg>();
        return r;
    }
    Fq d = fe_zero<FqCfg>(), zz2, zz3;
    coop_mul<1>(co, p.zz, p.zz, d, d, d, d, d, d, zz2, d, d, d);
    coop_mul<2>(co, zz2, p.zz, p.x, zz2, d, d, d, d, zz3, r.x, d, d);
    coop_mul<1>(co, p.y, zz3, d, d, d, d, d, d, r.y, d, d, d);
    r.z = p.zzz;
    return r;
}

// Horner over the W window sums win[0..W) of one MSM by the whole CTA
// (COOP_THREADS threads); every thread returns the Jacobian result.
__device__ __forceinline__ Jac coop_horner(Fq* sh_buf, const Xyzz* win, int W, int c) {
    Coop co{sh_buf, 0};
    Xyzz acc = W > 0 ? ld_xyzz(win + W - 1) : xyzz_identity();
    for (int w = W - 2; w >= 0; w--) {
        for (int i = 0; i < c; i++) acc = coop_dbl(co, acc);
        acc = coop_add(co, acc, ld_xyzz(win + w));
    }
    return coop_to_jac(co, acc);
}

}  // namespace zk
