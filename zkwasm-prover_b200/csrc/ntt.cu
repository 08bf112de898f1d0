// Radix-2^k NTT for BN254 Fr on sm_100a.
//
// A transform of size n = 2^log_n is a sequence of global passes (Stockham
// autosort, natural order in and out).  Pass t has radix R_t = 2^LOGR and
// P_t = R_1 * ... * R_{t-1}.  Work item q in [0, n/R_t) with J = q mod P_t and
// Q = q / P_t:
//     reads   x[q + (n/R_t) * i]                       i < R_t
//     y_j   = sum_i x_i w_{R_t}^{ij}                   (in shared memory)
//     writes  dst[J + P_t*j + P_t*R_t*Q] = y_j * w_n^{P_t*Q*j}
// so the final pass leaves X[j] = sum_i x_i w_n^{ij} in natural order.  Inside a
// CTA the radix-R_t DFT is itself a Stockham sequence of radix-8 (then 4 or 2)
// sub-stages held in registers, exchanging through shared memory.
//
// Twiddles come from the natural table w^i (i < n) that expand_omega_buffer
// builds; a sub-stage twiddle w_R^e is entry e * (n/R).
//
// The same pass kernel serves the coset extension: an optional per-input
// multiplier table (the coset twist s^k, applied on load in the first pass),
// an optional output scale (n^-1 for the inverse transform) and an output
// index map pos -> (pos << out_shift) + z * out_off_z that interleaves the
// 2^e sub-transforms of an extended domain.
//
// Reference behaviour replaced: cuda/bn254.cu:1357-1428 (ntt), 294-418
// (merge_ntt_kernel), 421-494 (_ntt_core).
#include "common.cuh"
#include "kernels.h"

namespace zk {

// Every Fr product of the pass kernels goes through one out-of-line function:
// inlined, the ~30 product sites of a pass (each ~350 instructions) overflow
// the instruction cache and warps stall on instruction fetch.
//
// Inside a pass, values are kept lazily reduced in [0, 2r): the products skip
// their final conditional subtraction (nt_mulz) and the butterflies add and
// subtract modulo 2r; every value leaves a pass canonical (fe_canon at the
// last sub-stage), so buffers in global memory always hold canonical values.
#if defined(ZK_NTT_INLINE_MUL)
__device__ __forceinline__ Fr nt_mul(const Fr& a, const Fr& b) { return fe_mul<FrCfg>(a, b); }
__device__ __forceinline__ Fr nt_mulz(const Fr& a, const Fr& b) { return fe_mul_lazy<FrCfg>(a, b); }
__device__ __forceinline__ Fr nt_shoup(const Fr& a, const Fr& w, const Fr& wp) {
    return fe_mul_shoup<FrCfg>(a, w, wp);
}
#else
__device__ __noinline__ Fr nt_mul(const Fr a, const Fr b) { return fe_mul<FrCfg>(a, b); }
__device__ __noinline__ Fr nt_mulz(const Fr a, const Fr b) { return fe_mul_lazy<FrCfg>(a, b); }
__device__ __noinline__ Fr nt_shoup(const Fr a, const Fr w, const Fr wp) { return fe_mul_shoup<FrCfg>(a, w, wp); }
#endif

// Two or three independent products in one call, so the scheduler can
// interleave their carry chains.
struct Fr2 {
    Fr a, b;
};
struct Fr3 {
    Fr a, b, c;
};
#if defined(ZK_NTT_INLINE_MUL)
#define ZK_NTMUL __device__ __forceinline__
#else
#define ZK_NTMUL __device__ __noinline__
#endif
ZK_NTMUL Fr2 nt_mulz2(const Fr a0, const Fr w0, const Fr a1, const Fr w1) {
    return {fe_mul_lazy<FrCfg>(a0, w0), fe_mul_lazy<FrCfg>(a1, w1)};
}
ZK_NTMUL Fr3 nt_mulz3(const Fr a0, const Fr w0, const Fr a1, const Fr w1, const Fr a2, const Fr w2) {
    return {fe_mul_lazy<FrCfg>(a0, w0), fe_mul_lazy<FrCfg>(a1, w1), fe_mul_lazy<FrCfg>(a2, w2)};
}
ZK_NTMUL Fr2 nt_shoup2(const Fr a0, const Fr w0, const Fr p0, const Fr a1, const Fr w1, const Fr p1) {
    return {fe_mul_shoup<FrCfg>(a0, w0, p0), fe_mul_shoup<FrCfg>(a1, w1, p1)};
}
ZK_NTMUL Fr3 nt_shoup3(const Fr a0, const Fr w0, const Fr p0, const Fr a1, const Fr w1, const Fr p1, const Fr a2,
                       const Fr w2, const Fr p2) {
    return {fe_mul_shoup<FrCfg>(a0, w0, p0), fe_mul_shoup<FrCfg>(a1, w1, p1), fe_mul_shoup<FrCfg>(a2, w2, p2)};
}
#undef ZK_NTMUL

// Multiplier tables (twiddles, twists, scales) come in two layouts.
// TwM: one Montgomery-form element per entry, multiplied with nt_mulz.
// TwS: the pair (w, w') per entry, w canonical and w' = floor(w 2^256 / r),
// multiplied with nt_shoup (207 multiply-adds instead of 264; both results
// lie in [0, 2r)).  Every product of the pass kernels is by a table entry.
struct TwM {
    struct K {
        Fr w;
    };
    static __device__ __forceinline__ K ld(const Fr* t, size_t i) { return {ldg_elem<FrCfg>(t + i)}; }
    static __device__ __forceinline__ Fr mul(const Fr& v, const K& k) { return nt_mulz(v, k.w); }
    static __device__ __forceinline__ Fr2 mul2(const Fr& v0, const K& k0, const Fr& v1, const K& k1) {
        return nt_mulz2(v0, k0.w, v1, k1.w);
    }
    static __device__ __forceinline__ Fr3 mul3(const Fr& v0, const K& k0, const Fr& v1, const K& k1, const Fr& v2,
                                               const K& k2) {
        return nt_mulz3(v0, k0.w, v1, k1.w, v2, k2.w);
    }
    static __host__ __device__ __forceinline__ const Fr* off(const Fr* t, size_t i) { return t + i; }
};
struct TwS {
    struct K {
        Fr w, wp;
    };
    static __device__ __forceinline__ K ld(const Fr* t, size_t i) {
        return {ldg_elem<FrCfg>(t + 2 * i), ldg_elem<FrCfg>(t + 2 * i + 1)};
    }
    static __device__ __forceinline__ Fr mul(const Fr& v, const K& k) { return nt_shoup(v, k.w, k.wp); }
    static __device__ __forceinline__ Fr2 mul2(const Fr& v0, const K& k0, const Fr& v1, const K& k1) {
        return nt_shoup2(v0, k0.w, k0.wp, v1, k1.w, k1.wp);
    }
    static __device__ __forceinline__ Fr3 mul3(const Fr& v0, const K& k0, const Fr& v1, const K& k1, const Fr& v2,
                                               const K& k2) {
        return nt_shoup3(v0, k0.w, k0.wp, v1, k1.w, k1.wp, v2, k2.w, k2.wp);
    }
    static __host__ __device__ __forceinline__ const Fr* off(const Fr* t, size_t i) { return t + 2 * i; }
};


// ---------------------------------------------------------------- small DFTs
// Decimation in frequency, natural input; outputs land bit-reversed and are
// relabelled by the caller.

__device__ __forceinline__ void dft2(Fr& a, Fr& b) {
    Fr t = fe_add_lazy<FrCfg>(a, b);
    b = fe_sub_lazy<FrCfg>(a, b);
    a = t;
}

// v[0..3] -> y[k] at position rev2(k): y0=v0, y1=v2, y2=v1, y3=v3
template <class TW>
__device__ __forceinline__ void dft4_dif(Fr& v0, Fr& v1, Fr& v2, Fr& v3, const typename TW::K& w4) {
    dft2(v0, v2);
    dft2(v1, v3);
    v3 = TW::mul(v3, w4);
    dft2(v0, v1);
    dft2(v2, v3);
}

// v[0..7] -> y[j] at position rev3(j)
template <class TW>
__device__ __forceinline__ void dft8_dif(Fr v[8], const typename TW::K& w8, const typename TW::K& w4,
                                         const typename TW::K& w83) {
    dft2(v[0], v[4]);
    dft2(v[1], v[5]);
    dft2(v[2], v[6]);
    dft2(v[3], v[7]);
    const Fr3 m = TW::mul3(v[5], w8, v[6], w4, v[7], w83);
    v[5] = m.a;
    v[6] = m.b;
    v[7] = m.c;
    // the two radix-4 DFTs side by side
    dft2(v[0], v[2]);
    dft2(v[1], v[3]);
    dft2(v[4], v[6]);
    dft2(v[5], v[7]);
    const Fr2 m4 = TW::mul2(v[3], w4, v[7], w4);
    v[3] = m4.a;
    v[7] = m4.b;
    dft2(v[0], v[1]);
    dft2(v[2], v[3]);
    dft2(v[4], v[5]);
    dft2(v[6], v[7]);
}


// output-side work of the last sub-stage: the inter-pass twiddle w_n^{P*Q*y}
// and the optional scale
struct PassOut {
    const Fr* tw;
    int log_p;       // global P
    uint32_t qhi;    // Q = q >> log_p for this thread's DFT
    const Fr* scale;
    const Fr* wrow;  // when set: output y is multiplied by wrow[y] instead
};

// (the result is canonical: it leaves the pass)
template <class TW>
__device__ __forceinline__ Fr finish_out(const PassOut& o, Fr v, uint32_t y) {
    if (o.wrow) return fe_canon<FrCfg>(TW::mul(v, TW::ld(o.wrow, y)));
    if (o.qhi != 0 && y != 0) v = TW::mul(v, TW::ld(o.tw, (size_t)(o.qhi * y) << o.log_p));
    if (o.scale) v = TW::mul(v, TW::ld(o.scale, 0));
    return fe_canon<FrCfg>(v);
}

// radix-8 sub-stage over one DFT of size R in shared memory
template <int LOGR, class TW>
__device__ __forceinline__ void stage8(Fr* x, int u, int log_ps, bool last, const Fr* tw, int log_n,
                                       const Fr* in_mul, size_t in_base, int log_items,
                                       const PassOut& po) {
    constexpr int R = 1 << LOGR;
    constexpr int S = R / 8;
    Fr v[8];
#pragma unroll
    for (int i = 0; i < 8; i++) v[i] = sm_ld(x, u + S * i);
    __syncthreads();
    if (in_mul) {
#pragma unroll
        for (int i = 0; i < 8; i++)
            v[i] = TW::mul(v[i], TW::ld(in_mul, in_base + ((size_t)(u + S * i) << log_items)));
    }
    const int sh = log_n - LOGR;  // w_R^e = tw[e << sh]
    {
        const typename TW::K w8 = TW::ld(tw, (size_t)(S * 1) << sh);
        const typename TW::K w4 = TW::ld(tw, (size_t)(S * 2) << sh);
        const typename TW::K w83 = TW::ld(tw, (size_t)(S * 3) << sh);
        dft8_dif<TW>(v, w8, w4, w83);
    }
    const int J = u & ((1 << log_ps) - 1);
    const int ilo = u >> log_ps;
    // y[j] sits in v[rev3(j)]
    const int rev[8] = {0, 4, 2, 6, 1, 5, 3, 7};
    if (ilo != 0) {
#pragma unroll
        for (int j = 1; j < 7; j += 2) {
            const Fr2 t = TW::mul2(v[rev[j]], TW::ld(tw, (size_t)((ilo * j) << log_ps) << sh), v[rev[j + 1]],
                                   TW::ld(tw, (size_t)((ilo * (j + 1)) << log_ps) << sh));
            v[rev[j]] = t.a;
            v[rev[j + 1]] = t.b;
        }
        v[rev[7]] = TW::mul(v[rev[7]], TW::ld(tw, (size_t)((ilo * 7) << log_ps) << sh));
    }
#pragma unroll
    for (int j = 0; j < 8; j++) {
        Fr y = v[rev[j]];
        const int pos = J + (j << log_ps) + (ilo << (log_ps + 3));
        if (last) y = finish_out<TW>(po, y, (uint32_t)pos);
        sm_st(x, pos, y);
    }
    __syncthreads();
}

// final radix-4 sub-stage (two items per thread); P_s = R/4 so no sub-stage twiddle
template <int LOGR, class TW>
__device__ __forceinline__ void stage4_last(Fr* x, int lt, const Fr* tw, int log_n, const PassOut& po,
                                            const Fr* in_mul, size_t in_base, int log_items) {
    constexpr int R = 1 << LOGR;
    constexpr int S = R / 4;  // items and read stride
    constexpr int TH = (R >= 8) ? R / 8 : 1;
    Fr v[8];
#pragma unroll
    for (int k = 0; k < 2; k++) {
        int u = lt + k * TH;
#pragma unroll
        for (int i = 0; i < 4; i++) v[4 * k + i] = sm_ld(x, u + S * i);
    }
    __syncthreads();
    const int sh = log_n - LOGR;
    const typename TW::K w4 = TW::ld(tw, (size_t)S << sh);
#pragma unroll
    for (int k = 0; k < 2; k++) {
        int u = lt + k * TH;
        if (in_mul) {
#pragma unroll
            for (int i = 0; i < 4; i++)
                v[4 * k + i] = TW::mul(v[4 * k + i], TW::ld(in_mul, in_base + ((size_t)(u + S * i) << log_items)));
        }
        dft4_dif<TW>(v[4 * k], v[4 * k + 1], v[4 * k + 2], v[4 * k + 3], w4);
        const int rev[4] = {0, 2, 1, 3};
#pragma unroll
        for (int j = 0; j < 4; j++) {
            const int pos = u + S * j;  // J = u, P_s = S, ilo = 0
            sm_st(x, pos, finish_out<TW>(po, v[4 * k + rev[j]], (uint32_t)pos));
        }
    }
    __syncthreads();
}

// final radix-2 sub-stage (four items per thread)
template <int LOGR, class TW>
__device__ __forceinline__ void stage2_last(Fr* x, int lt, const PassOut& po) {
    constexpr int R = 1 << LOGR;
    constexpr int S = R / 2;
    constexpr int TH = R / 8;
    // each thread reads and rewrites only its own slots u and u + S, so a
    // pair is finished before the next is loaded (two elements live at a time)
#pragma unroll 1
    for (int k = 0; k < 4; k++) {
        const int u = lt + k * TH;
        Fr v0 = sm_ld(x, u), v1 = sm_ld(x, u + S);
        dft2(v0, v1);
        sm_st(x, u, finish_out<TW>(po, v0, (uint32_t)u));
        sm_st(x, u + S, finish_out<TW>(po, v1, (uint32_t)(u + S)));
    }
    __syncthreads();
}

#ifndef ZK_PASS10_MIN_BLOCKS
#define ZK_PASS10_MIN_BLOCKS 4
#endif

// resident CTAs per SM the register budget of a pass kernel is sized for:
// 16 warps per SM (128 registers a thread) for most shapes
__host__ __device__ constexpr int pass_min_blocks(int logr, int g) {
    return ((g << logr) / 8) >= 512 ? 1
           : (logr == 10 && g == 1) ? ZK_PASS10_MIN_BLOCKS
           : ((g << logr) / 8 >= 32 ? 512 / ((g << logr) / 8) : 16);
}

template <int LOGR, int G, class TW>
__global__ void __launch_bounds__((G << LOGR) / 8, pass_min_blocks(LOGR, G))
ntt_pass_kernel(NttPassArgs a) {
    constexpr int R = 1 << LOGR;
    constexpr int TR = R / 8;  // threads per DFT
    constexpr int T = G * TR;
    extern __shared__ uint4 smem_u4[];
    Fr* sm = reinterpret_cast<Fr*>(smem_u4);
    const int tid = threadIdx.x;
    const int log_items = a.log_n - LOGR;
    // Blocks run column-fastest: the CTAs of one item across the batch's
    // columns are resident together, so the twiddle and twist values they
    // share are read from DRAM once and from L2 by the other columns (in grid
    // order every column would stream both tables again, 3.5x the pass's
    // algorithmic reads at 8 columns of 2^22).
    const uint64_t lin = (uint64_t)blockIdx.y * gridDim.x + blockIdx.x;
    const uint32_t bx = (uint32_t)(lin / gridDim.y), by = (uint32_t)(lin % gridDim.y);
    const uint32_t q0 = bx * G;
    const Fr* src = a.src + by * a.src_ys + blockIdx.z * a.src_zs;
    Fr* dst = a.dst + by * a.dst_ys + blockIdx.z * a.dst_zs;

    // coalesced load: chunk c -> (i, g, h); global x[q0 + g + (i << log_items)]
    for (int c = tid; c < G * R * 2; c += T) {
        const int h = c & 1, e = c >> 1;
        const int g = e % G, i = e / G;
        const size_t gi = (size_t)(q0 + g) + ((size_t)i << log_items);
        *sm_slot(sm + g * R, i, h) = reinterpret_cast<const uint4*>(src + gi)[h];
    }
    __syncthreads();

    const int g = tid / TR, lt = tid % TR;
    Fr* x = sm + g * R;
    const uint32_t q = q0 + g;
    PassOut po;
    po.tw = a.tw;
    po.log_p = a.log_p;
    po.qhi = q >> a.log_p;
    po.scale = a.scale;
    po.wrow = nullptr;
    const Fr* in_mul = a.in_mul ? TW::off(a.in_mul, blockIdx.z * a.in_mul_zs) : nullptr;
    const size_t in_base = q;  // natural input position = q + (i << log_items)

    constexpr int NS8 = LOGR / 3;
    constexpr int REM = LOGR % 3;
    int log_ps = 0;
#pragma unroll 1
    for (int s = 0; s < NS8; s++) {
        const bool last = (s == NS8 - 1) && (REM == 0);
        stage8<LOGR, TW>(x, lt, log_ps, last, a.tw, a.log_n, s == 0 ? in_mul : nullptr, in_base, log_items, po);
        log_ps += 3;
    }
    if (REM == 2)
        stage4_last<LOGR, TW>(x, lt, a.tw, a.log_n, po, NS8 == 0 ? in_mul : nullptr, in_base, log_items);
    if (REM == 1) stage2_last<LOGR, TW>(x, lt, po);

    // coalesced store: dst[(J + P*j + P*R*Q) << out_shift + z*out_off_z]
    const uint32_t pm = (1u << a.log_p) - 1;
    const size_t zoff = (size_t)blockIdx.z * a.out_off_z;
    for (int c = tid; c < G * R * 2; c += T) {
        const int h = c & 1, e = c >> 1;
        int gg, j;
        if (a.log_p == 0) {
            gg = e >> LOGR;
            j = e & (R - 1);
        } else {
            gg = e % G;
            j = e / G;
        }
        const uint32_t qq = q0 + gg;
        const size_t pos = (size_t)(qq & pm) + ((size_t)j << a.log_p) + ((size_t)(qq >> a.log_p) << (a.log_p + LOGR));
        const size_t o = (pos << a.out_shift) + zoff;
        reinterpret_cast<uint4*>(dst + o)[h] = *sm_slot(sm + gg * R, j, h);
    }
}

// in-CTA DFT of size 2^LOGR on tile x (natural order in and out)
template <int LOGR, class TW>
__device__ __forceinline__ void dft_tile(Fr* x, int lt, const Fr* tw, int log_n, const PassOut& po) {
    constexpr int NS8 = LOGR / 3;
    constexpr int REM = LOGR % 3;
    int log_ps = 0;
#pragma unroll 1
    for (int s = 0; s < NS8; s++) {
        stage8<LOGR, TW>(x, lt, log_ps, (s == NS8 - 1) && (REM == 0), tw, log_n, nullptr, 0, 0, po);
        log_ps += 3;
    }
    if (REM == 2) stage4_last<LOGR, TW>(x, lt, tw, log_n, po, nullptr, 0, 0);
    if (REM == 1) stage2_last<LOGR, TW>(x, lt, po);
}

// Fused extended-domain stage.  For one column and work item q it runs
//   (1) the last pass of the inverse transform: radix R = 2^LOGR, P = n/R,
//       input tmp[q + (n/R) i], output the coefficients c[q + (n/R) j] * n^-1,
//       written to coeff;
//   (2) for each coset z, the first pass of that coset's forward transform in
//       the reversed radix order (radix R first, P = 1), whose item q reads
//       exactly the same coefficients c[q + (n/R) i], twisted by
//       t_z^(q + (n/R) i) = t_z^q * S_z[i]: the tile is multiplied by S_z,
//       transformed, and output y is multiplied by W_z[q R + y] = w^(q y) t_z^q
//       (inter-pass twiddle and the item's twist constant), then written to
//       sub[z n + y + R q].
// The coefficients stay in shared memory across the 2^e cosets, so they are
// read once instead of 2^e times with a strided pattern.
#ifndef ZK_FUSED_ONE_TILE
#define ZK_FUSED_ONE_TILE 1
#endif

// resident CTAs per SM the register budget is sized for: two tiles of 2^LOGR
// elements in shared memory allow 7 CTAs of 2^9, 3 of 2^10 and 1 of 2^11; one
// tile (the coefficients re-read from L2 for each coset) allows 4 of 2^10 and,
// at 128 registers a thread, 2 of 2^11 (the 2^22 -> 2^25 extension: 82.1 ->
// 73.0 ms per 8 columns on B200 against one CTA of 255 registers)
#ifndef ZK_FUSED11_MIN_BLOCKS
#define ZK_FUSED11_MIN_BLOCKS 2
#endif
__host__ __device__ constexpr int fused_min_blocks(int logr) {
    return logr <= 9 ? 7 : logr == 10 ? (ZK_FUSED_ONE_TILE ? 4 : 3) : ZK_FUSED11_MIN_BLOCKS;
}

template <int LOGR, class TW>
__global__ void __launch_bounds__((1 << LOGR) / 8, fused_min_blocks(LOGR))
ntt_fused_extend_kernel(FusedExtendArgs a) {
    constexpr int R = 1 << LOGR;
    constexpr int T = R / 8;
    extern __shared__ uint4 smem_u4[];
    Fr* A = reinterpret_cast<Fr*>(smem_u4);
    Fr* B = ZK_FUSED_ONE_TILE ? A : A + R;
    const int tid = threadIdx.x;
    const int log_items = a.log_n - LOGR;
    // column-fastest block order, as in ntt_pass_kernel: the per-coset tables
    // an item reads are shared by every column of the launch
    const uint64_t lin = (uint64_t)blockIdx.y * gridDim.x + blockIdx.x;
    const uint32_t q = (uint32_t)(lin / gridDim.y), col = (uint32_t)(lin % gridDim.y);
    const size_t n = (size_t)1 << a.log_n;
    const Fr* src = a.src + col * a.src_ys;
    Fr* coeff = a.coeff + col * a.coeff_ys;
    Fr* sub = a.sub + col * a.sub_ys;

    for (int c = tid; c < R * 2; c += T) {
        const int h = c & 1, i = c >> 1;
        *sm_slot(A, i, h) = reinterpret_cast<const uint4*>(src + q + ((size_t)i << log_items))[h];
    }
    __syncthreads();
    PassOut po;
    po.tw = a.tw_inv;
    po.log_p = log_items;
    po.qhi = 0;
    po.scale = a.n_inv;
    po.wrow = nullptr;
    dft_tile<LOGR, TW>(A, tid, a.tw_inv, a.log_n, po);
    for (int c = tid; c < R * 2; c += T) {
        const int h = c & 1, j = c >> 1;
        reinterpret_cast<uint4*>(coeff + q + ((size_t)j << log_items))[h] = *sm_slot(A, j, h);
    }
    for (int z = 0; z < a.E; z++) {
        const Fr* S = TW::off(a.stab, (size_t)z * R);
        if (ZK_FUSED_ONE_TILE) {
            // the tile is the workspace: coset 0 twists it in place, later
            // cosets re-read the coefficients this CTA wrote (L2-resident)
            __syncthreads();
            for (int i = tid; i < R; i += T) {
                const Fr cf = z == 0 ? sm_ld(A, i) : ld_elem<FrCfg>(coeff + q + ((size_t)i << log_items));
                sm_st(B, i, TW::mul(cf, TW::ld(S, i)));
            }
        } else {
            for (int i = tid; i < R; i += T) sm_st(B, i, TW::mul(sm_ld(A, i), TW::ld(S, i)));
        }
        __syncthreads();
        PassOut pf;
        pf.tw = a.tw;
        pf.log_p = 0;
        pf.qhi = 0;
        pf.scale = nullptr;
        pf.wrow = TW::off(a.wtab, (size_t)z * n + (size_t)q * R);
        dft_tile<LOGR, TW>(B, tid, a.tw, a.log_n, pf);
        Fr* out = sub + (size_t)z * n + (size_t)q * R;
        for (int c = tid; c < R * 2; c += T) {
            const int h = c & 1, y = c >> 1;
            reinterpret_cast<uint4*>(out + y)[h] = *sm_slot(B, y, h);
        }
        __syncthreads();
    }
}

template <int LOGR, class TW>
static cudaError_t launch_fused(const FusedExtendArgs& a, unsigned ncols, cudaStream_t s) {
    constexpr int R = 1 << LOGR;
    const size_t smem = (size_t)(ZK_FUSED_ONE_TILE ? 1 : 2) * R * sizeof(Fr);
    static SmemOptIn opt;
    ZK_CHECK(opt.ensure(ntt_fused_extend_kernel<LOGR, TW>, (int)smem));
    dim3 grid(1u << (a.log_n - LOGR), ncols, 1);
    ntt_fused_extend_kernel<LOGR, TW><<<grid, R / 8, smem, s>>>(a);
    return cudaGetLastError();
}

template <class TW>
static cudaError_t fused_dispatch(const FusedExtendArgs& a, int log_r, unsigned ncols, cudaStream_t s) {
    switch (log_r) {
        case 9: return launch_fused<9, TW>(a, ncols, s);
        case 10: return launch_fused<10, TW>(a, ncols, s);
        case 11: return launch_fused<11, TW>(a, ncols, s);
        default: return cudaErrorInvalidValue;
    }
}

cudaError_t ntt_fused_extend(const FusedExtendArgs& a, int log_r, unsigned ncols, cudaStream_t s) {
    return a.pairs ? fused_dispatch<TwS>(a, log_r, ncols, s) : fused_dispatch<TwM>(a, log_r, ncols, s);
}

// Tables of the fused stage for radix R = 2^log_r: wtab[z n + q R + y] =
// w^(q y) t_z^q (q < n/R, y < R) and stab[z R + i] = (t_z^(n/R))^i, with
// t_z = shift * w_ext^z and w^k read from the natural table tw.
template <bool PAIRS>
__global__ void fused_tables_kernel(Fr* wtab, Fr* stab, const Fr* tw, const Fr* shift, const Fr* w_ext, int log_n,
                                    int log_r) {
    const uint32_t z = blockIdx.y;
    const uint32_t R = 1u << log_r;
    const uint32_t items = 1u << (log_n - log_r);
    const size_t n = (size_t)1 << log_n;
    const Fr tz = nt_mul(ld_elem<FrCfg>(shift), fe_pow_u32<FrCfg>(ld_elem<FrCfg>(w_ext), z));
    for (uint32_t q = blockIdx.x; q < items; q += gridDim.x) {
        const Fr tq = fe_pow_u32<FrCfg>(tz, q);
        for (uint32_t y = threadIdx.x; y < R; y += blockDim.x) {
            const Fr w = ld_elem<FrCfg>(tw + (size_t)q * y);
            st_factor<PAIRS>(wtab, (size_t)z * n + (size_t)q * R + y, y == 0 ? tq : nt_mul(w, tq));
        }
    }
    if (blockIdx.x == 0) {
        const Fr s = fe_pow_u32<FrCfg>(tz, items);
        for (uint32_t i = threadIdx.x; i < R; i += blockDim.x)
            st_factor<PAIRS>(stab, (size_t)z * R + i, fe_pow_u32<FrCfg>(s, i));
    }
}

cudaError_t ntt_fused_tables(Fr* wtab, Fr* stab, const Fr* tw, const Fr* shift, const Fr* w_ext, int log_n, int log_r,
                             int ext_bits, cudaStream_t s, bool pairs) {
    const uint32_t items = 1u << (log_n - log_r);
    dim3 grid(items < 4096 ? items : 4096, 1u << ext_bits);
    if (pairs)
        fused_tables_kernel<true><<<grid, 256, 0, s>>>(wtab, stab, tw, shift, w_ext, log_n, log_r);
    else
        fused_tables_kernel<false><<<grid, 256, 0, s>>>(wtab, stab, tw, shift, w_ext, log_n, log_r);
    return cudaGetLastError();
}

// out[i] = (w, w') for the Montgomery-form factors in[i], i < n
__global__ void shoup_pairs_kernel(Fr* out, const Fr* in, size_t n) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        st_factor<true>(out, i, ld_elem<FrCfg>(in + i));
}

cudaError_t shoup_pairs(Fr* out, const Fr* in, size_t n, cudaStream_t s) {
    if (n == 0) return cudaSuccess;
    const size_t blocks = (n + 255) / 256;
    shoup_pairs_kernel<<<(unsigned)(blocks < 148 * 32 ? blocks : 148 * 32), 256, 0, s>>>(out, in, n);
    return cudaGetLastError();
}

// tiny transforms (n <= 4): direct O(n^2) evaluation by one thread per column
__global__ void ntt_tiny_kernel(NttPassArgs a) {
    const int n = 1 << a.log_n;
    const Fr* src = a.src + blockIdx.y * a.src_ys;
    Fr* dst = a.dst + blockIdx.y * a.dst_ys;
    if (threadIdx.x != 0) return;
    Fr x[4], y[4];
    for (int i = 0; i < n; i++) {
        x[i] = ld_elem<FrCfg>(src + i);
        if (a.in_mul) x[i] = nt_mul(x[i], ld_elem<FrCfg>(a.in_mul + i));
    }
    for (int j = 0; j < n; j++) {
        Fr acc = fe_zero<FrCfg>();
        for (int i = 0; i < n; i++) {
            Fr t = x[i];
            int e = (i * j) & (n - 1);
            if (e) t = nt_mul(t, ld_elem<FrCfg>(a.tw + e));
            acc = fe_add<FrCfg>(acc, t);
        }
        if (a.scale) acc = nt_mul(acc, ld_elem<FrCfg>(a.scale));
        y[j] = acc;
    }
    for (int j = 0; j < n; j++) st_elem<FrCfg>(dst + ((size_t)j << a.out_shift), y[j]);
}

// ---------------------------------------------------------------- launchers

template <int LOGR, int G, class TW>
static cudaError_t launch_pass(const NttPassArgs& a, unsigned ny, unsigned nz, cudaStream_t s) {
    constexpr int R = 1 << LOGR;
    constexpr int T = (G * R) / 8;
    const size_t smem = (size_t)G * R * sizeof(Fr);
    static SmemOptIn opt;
    ZK_CHECK(opt.ensure(ntt_pass_kernel<LOGR, G, TW>, (int)smem));
    const unsigned items = 1u << (a.log_n - LOGR);
    dim3 grid(items / G, ny, nz);
    ntt_pass_kernel<LOGR, G, TW><<<grid, T, smem, s>>>(a);
    return cudaGetLastError();
}

// preferred items per CTA so that a CTA holds about 1024 elements
static int pass_group(int log_r, int log_n) {
    int g = 1;
    if (log_r <= 9) g = 1 << (10 - log_r);
    if (g > 16) g = 16;
    const int items = 1 << (log_n - log_r);
    if (g > items) g = items;
    return g;
}

template <class TW>
static cudaError_t pass_dispatch(const NttPassArgs& a, int log_r, unsigned ny, unsigned nz, cudaStream_t s) {
    const int g = pass_group(log_r, a.log_n);
#define ZK_PASS(LR, GG) \
    if (log_r == LR && g == GG) return launch_pass<LR, GG, TW>(a, ny, nz, s);
    ZK_PASS(3, 1) ZK_PASS(4, 1) ZK_PASS(5, 1) ZK_PASS(6, 1) ZK_PASS(7, 1) ZK_PASS(8, 1)
    ZK_PASS(9, 1) ZK_PASS(10, 1) ZK_PASS(11, 1) ZK_PASS(12, 1)
    ZK_PASS(6, 2) ZK_PASS(6, 4) ZK_PASS(6, 8) ZK_PASS(6, 16)
    ZK_PASS(7, 2) ZK_PASS(7, 4) ZK_PASS(7, 8)
    ZK_PASS(8, 2) ZK_PASS(8, 4)
    ZK_PASS(9, 2)
#undef ZK_PASS
    return cudaErrorInvalidValue;
}

cudaError_t ntt_pass(const NttPassArgs& a, int log_r, unsigned ny, unsigned nz, cudaStream_t s) {
    if (a.log_n <= 2) {
        if (a.pairs) return cudaErrorInvalidValue;  // the direct kernel reads Montgomery tables
        ntt_tiny_kernel<<<dim3(1, ny, nz), 32, 0, s>>>(a);
        return cudaGetLastError();
    }
    return a.pairs ? pass_dispatch<TwS>(a, log_r, ny, nz, s) : pass_dispatch<TwM>(a, log_r, ny, nz, s);
}

// split log_n into pass radices (at most ZK_NTT_MAX_PASS_BITS bits per pass,
// as even as possible).  11: 2^24 runs as three passes of 2^8 (4.25 ms on
// B200) rather than two of 2^12 (4.78 ms; one 512-thread CTA of 128 KB per
// SM); 10 would slow 2^21 and 2^22.
#ifndef ZK_NTT_MAX_PASS_BITS
#define ZK_NTT_MAX_PASS_BITS 11
#endif
// The splits the radix autotuner (zkp_ntt_batch_plan over every split into
// 2-3 passes of 2^6..2^12, one column) measured fastest on B200 for 2^13..2^25;
// other sizes use the even split below.
static const int8_t TUNED_SPLIT[13][3] = {{7, 6, 0},  {6, 8, 0},  {6, 9, 0},   {8, 8, 0},  {8, 9, 0},
                                          {9, 9, 0},  {11, 8, 0}, {10, 10, 0}, {11, 10, 0}, {11, 11, 0},
                                          {11, 6, 6}, {9, 9, 6},  {9, 10, 6}};

int ntt_plan(int log_n, int radices[4]) {
    if (log_n <= 12) {
        radices[0] = log_n;
        return 1;
    }
    if (log_n <= 25) {
        const int8_t* t = TUNED_SPLIT[log_n - 13];
        const int np = t[2] ? 3 : 2;
        for (int i = 0; i < np; i++) radices[i] = t[i];
        return np;
    }
    int np = (log_n + ZK_NTT_MAX_PASS_BITS - 1) / ZK_NTT_MAX_PASS_BITS;
    if (np < 2) np = 2;
    for (int i = 0; i < np; i++) radices[i] = log_n / np + (i < log_n % np ? 1 : 0);
    return np;
}

cudaError_t ntt_run(Fr* buf, Fr* tmp, const Fr* tw, const Fr* scale, int log_n, unsigned ncols,
                    size_t col_stride, bool* result_in_tmp, cudaStream_t s) {
    int rad[4];
    const int np = ntt_plan(log_n, rad);
    return ntt_run_plan(buf, tmp, tw, scale, log_n, ncols, col_stride, rad, np, result_in_tmp, s);
}

cudaError_t ntt_run_plan(Fr* buf, Fr* tmp, const Fr* tw, const Fr* scale, int log_n, unsigned ncols,
                         size_t col_stride, const int* rad, int np, bool* result_in_tmp, cudaStream_t s) {
    int log_p = 0;
    for (int p = 0; p < np; p++) {
        // one pass runs in place; otherwise ping-pong buf -> tmp -> buf ...
        Fr* src = (np == 1 || p % 2 == 0) ? buf : tmp;
        Fr* dst = (np == 1) ? buf : (p % 2 == 0 ? tmp : buf);
        NttPassArgs a = {};
        a.src = src;
        a.dst = dst;
        a.tw = tw;
        a.log_n = log_n;
        a.log_p = log_p;
        a.scale = (p == np - 1) ? scale : nullptr;
        a.src_ys = col_stride;
        a.dst_ys = col_stride;
        ZK_CHECK(ntt_pass(a, rad[p], ncols, 1, s));
        log_p += rad[p];
    }
    *result_in_tmp = (np > 1) && (np % 2 == 1);
    return cudaSuccess;
}

// ---------------------------------------------------------------- tables

// Geometric sequences out[i] = base * w^i for i0 <= i < n (base null: 1) in
// two launches, one product per element instead of a power per thread:
//   coarse  out[k C] for every k: a thread takes GEO_C2 consecutive k, starts
//           from one power and steps by w^C;
//   fine    the run out[k C + 1 .. k C + C - 1] from out[k C] by steps of w.
// Each run is C dependent products on one thread, and the thread count stays
// n / C.
static constexpr uint32_t GEO_C = 64;
static constexpr uint32_t GEO_C2 = 64;

__device__ __forceinline__ Fr geo_base(const Fr* base) { return base ? ld_elem<FrCfg>(base) : fe_one<FrCfg>(); }

__global__ void geo_coarse_kernel(Fr* out, const Fr* base, const Fr* w, uint32_t n, uint32_t i0) {
    const uint64_t k0 = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) * GEO_C2;
    if (k0 * GEO_C >= n) return;
    const Fr r = fe_pow_u32<FrCfg>(ld_elem<FrCfg>(w), GEO_C);
    Fr cur = nt_mul(geo_base(base), fe_pow_u32<FrCfg>(r, (uint32_t)k0));
    for (uint64_t k = k0; k < k0 + GEO_C2 && k * GEO_C < n; k++) {
        if (k * GEO_C >= i0) st_elem<FrCfg>(out + k * GEO_C, cur);
        cur = nt_mul(cur, r);
    }
}

__global__ void geo_fine_kernel(Fr* out, const Fr* base, const Fr* w, uint32_t n, uint32_t i0) {
    const uint64_t s = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) * GEO_C;
    if (s >= n) return;
    const Fr ww = ld_elem<FrCfg>(w);
    // a run start below i0 was not written by the coarse pass
    Fr cur = s >= i0 ? ld_elem<FrCfg>(out + s) : nt_mul(geo_base(base), fe_pow_u32<FrCfg>(ww, (uint32_t)s));
    for (uint64_t i = s + 1; i < s + GEO_C && i < n; i++) {
        cur = nt_mul(cur, ww);
        if (i >= i0) st_elem<FrCfg>(out + i, cur);
    }
}

static cudaError_t geometric_from(Fr* out, const Fr* base, const Fr* w, uint32_t n, uint32_t i0, cudaStream_t s) {
    if (n <= i0) return cudaSuccess;
    const uint64_t runs = (n + GEO_C - 1) / GEO_C;
    const uint64_t coarse = (runs + GEO_C2 - 1) / GEO_C2;
    geo_coarse_kernel<<<(unsigned)((coarse + 127) / 128), 128, 0, s>>>(out, base, w, n, i0);
    ZK_CHECK(cudaGetLastError());
    geo_fine_kernel<<<(unsigned)((runs + 127) / 128), 128, 0, s>>>(out, base, w, n, i0);
    return cudaGetLastError();
}

// buf[i] = w^i for 2 <= i < n, with w = buf[1] (entries 0 and 1 written by the
// host and left as they are)
cudaError_t expand_powers(Fr* buf, uint32_t n, cudaStream_t s) { return geometric_from(buf, nullptr, buf + 1, n, 2, s); }

// out[i] = base * w^i for i < n, w and base given by value in device memory
cudaError_t geometric(Fr* out, const Fr* base, const Fr* w, uint32_t n, cudaStream_t s) {
    return geometric_from(out, base, w, n, 0, s);
}

}  // namespace zk
