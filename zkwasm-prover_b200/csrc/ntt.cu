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

// ---------------------------------------------------------------- small DFTs
// Decimation in frequency, natural input; outputs land bit-reversed and are
// relabelled by the caller.

__device__ __forceinline__ void dft2(Fr& a, Fr& b) {
    Fr t = fe_add<FrCfg>(a, b);
    b = fe_sub<FrCfg>(a, b);
    a = t;
}

// v[0..3] -> y[k] at position rev2(k): y0=v0, y1=v2, y2=v1, y3=v3
__device__ __forceinline__ void dft4_dif(Fr& v0, Fr& v1, Fr& v2, Fr& v3, const Fr& w4) {
    dft2(v0, v2);
    dft2(v1, v3);
    v3 = fe_mul<FrCfg>(v3, w4);
    dft2(v0, v1);
    dft2(v2, v3);
}

// v[0..7] -> y[j] at position rev3(j)
__device__ __forceinline__ void dft8_dif(Fr v[8], const Fr& w8, const Fr& w4, const Fr& w83) {
    dft2(v[0], v[4]);
    dft2(v[1], v[5]);
    dft2(v[2], v[6]);
    dft2(v[3], v[7]);
    v[5] = fe_mul<FrCfg>(v[5], w8);
    v[6] = fe_mul<FrCfg>(v[6], w4);
    v[7] = fe_mul<FrCfg>(v[7], w83);
    dft4_dif(v[0], v[1], v[2], v[3], w4);
    dft4_dif(v[4], v[5], v[6], v[7], w4);
}

// Shared-memory tiles hold 32-byte elements as two 16-byte halves.  Element
// p, half h lives at 16-byte slot 2 * (p ^ ((p >> 3) & 3)) + (h ^ (((p >> 2) ^
// (p >> 5)) & 1)): a bijection on each tile that gives the eight threads of a
// quarter-warp eight distinct bank groups both for runs of consecutive elements
// and for the stride-8 writes of the first radix-8 sub-stage.
__device__ __forceinline__ uint4* sm_slot(Fr* x, uint32_t p, uint32_t h) {
    const uint32_t pp = p ^ ((p >> 3) & 3u);
    const uint32_t hh = h ^ (((p >> 2) ^ (p >> 5)) & 1u);
    return reinterpret_cast<uint4*>(x) + 2 * pp + hh;
}
__device__ __forceinline__ Fr sm_ld(Fr* x, uint32_t p) {
    const uint4 a = *sm_slot(x, p, 0), b = *sm_slot(x, p, 1);
    Fr r;
    r.v[0] = a.x; r.v[1] = a.y; r.v[2] = a.z; r.v[3] = a.w;
    r.v[4] = b.x; r.v[5] = b.y; r.v[6] = b.z; r.v[7] = b.w;
    return r;
}
__device__ __forceinline__ void sm_st(Fr* x, uint32_t p, const Fr& v) {
    *sm_slot(x, p, 0) = make_uint4(v.v[0], v.v[1], v.v[2], v.v[3]);
    *sm_slot(x, p, 1) = make_uint4(v.v[4], v.v[5], v.v[6], v.v[7]);
}

// output-side work of the last sub-stage: the inter-pass twiddle w_n^{P*Q*y}
// and the optional scale
struct PassOut {
    const Fr* tw;
    int log_p;       // global P
    uint32_t qhi;    // Q = q >> log_p for this thread's DFT
    const Fr* scale;
};

__device__ __forceinline__ Fr finish_out(const PassOut& o, Fr v, uint32_t y) {
    if (o.qhi != 0 && y != 0) v = fe_mul<FrCfg>(v, ldg_elem<FrCfg>(o.tw + ((size_t)(o.qhi * y) << o.log_p)));
    if (o.scale) v = fe_mul<FrCfg>(v, ldg_elem<FrCfg>(o.scale));
    return v;
}

// radix-8 sub-stage over one DFT of size R in shared memory
template <int LOGR>
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
            v[i] = fe_mul<FrCfg>(v[i], ldg_elem<FrCfg>(in_mul + in_base + ((size_t)(u + S * i) << log_items)));
    }
    const int sh = log_n - LOGR;  // w_R^e = tw[e << sh]
    {
        Fr w8 = ldg_elem<FrCfg>(tw + ((size_t)(S * 1) << sh));
        Fr w4 = ldg_elem<FrCfg>(tw + ((size_t)(S * 2) << sh));
        Fr w83 = ldg_elem<FrCfg>(tw + ((size_t)(S * 3) << sh));
        dft8_dif(v, w8, w4, w83);
    }
    const int J = u & ((1 << log_ps) - 1);
    const int ilo = u >> log_ps;
    // y[j] sits in v[rev3(j)]
    const int rev[8] = {0, 4, 2, 6, 1, 5, 3, 7};
#pragma unroll
    for (int j = 0; j < 8; j++) {
        Fr y = v[rev[j]];
        if (j != 0 && ilo != 0)
            y = fe_mul<FrCfg>(y, ldg_elem<FrCfg>(tw + ((size_t)((ilo * j) << log_ps) << sh)));
        const int pos = J + (j << log_ps) + (ilo << (log_ps + 3));
        if (last) y = finish_out(po, y, (uint32_t)pos);
        sm_st(x, pos, y);
    }
    __syncthreads();
}

// final radix-4 sub-stage (two items per thread); P_s = R/4 so no sub-stage twiddle
template <int LOGR>
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
    Fr w4 = ldg_elem<FrCfg>(tw + ((size_t)S << sh));
#pragma unroll
    for (int k = 0; k < 2; k++) {
        int u = lt + k * TH;
        if (in_mul) {
#pragma unroll
            for (int i = 0; i < 4; i++)
                v[4 * k + i] = fe_mul<FrCfg>(
                    v[4 * k + i], ldg_elem<FrCfg>(in_mul + in_base + ((size_t)(u + S * i) << log_items)));
        }
        dft4_dif(v[4 * k], v[4 * k + 1], v[4 * k + 2], v[4 * k + 3], w4);
        const int rev[4] = {0, 2, 1, 3};
#pragma unroll
        for (int j = 0; j < 4; j++) {
            const int pos = u + S * j;  // J = u, P_s = S, ilo = 0
            sm_st(x, pos, finish_out(po, v[4 * k + rev[j]], (uint32_t)pos));
        }
    }
    __syncthreads();
}

// final radix-2 sub-stage (four items per thread)
template <int LOGR>
__device__ __forceinline__ void stage2_last(Fr* x, int lt, const PassOut& po) {
    constexpr int R = 1 << LOGR;
    constexpr int S = R / 2;
    constexpr int TH = R / 8;
    Fr v[8];
#pragma unroll
    for (int k = 0; k < 4; k++) {
        int u = lt + k * TH;
        v[2 * k] = sm_ld(x, u);
        v[2 * k + 1] = sm_ld(x, u + S);
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < 4; k++) {
        int u = lt + k * TH;
        dft2(v[2 * k], v[2 * k + 1]);
        sm_st(x, u, finish_out(po, v[2 * k], (uint32_t)u));
        sm_st(x, u + S, finish_out(po, v[2 * k + 1], (uint32_t)(u + S)));
    }
    __syncthreads();
}

template <int LOGR, int G>
__global__ void __launch_bounds__((G << LOGR) / 8, ((G << LOGR) / 8) >= 512 ? 1 : ((G << LOGR) / 8 >= 32 ? 512 / ((G << LOGR) / 8) : 16))
ntt_pass_kernel(NttPassArgs a) {
    constexpr int R = 1 << LOGR;
    constexpr int TR = R / 8;  // threads per DFT
    constexpr int T = G * TR;
    extern __shared__ uint4 smem_u4[];
    Fr* sm = reinterpret_cast<Fr*>(smem_u4);
    const int tid = threadIdx.x;
    const int log_items = a.log_n - LOGR;
    const uint32_t q0 = blockIdx.x * G;
    const Fr* src = a.src + blockIdx.y * a.src_ys + blockIdx.z * a.src_zs;
    Fr* dst = a.dst + blockIdx.y * a.dst_ys + blockIdx.z * a.dst_zs;

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
    const Fr* in_mul = a.in_mul ? a.in_mul + blockIdx.z * a.in_mul_zs : nullptr;
    const size_t in_base = q;  // natural input position = q + (i << log_items)

    constexpr int NS8 = LOGR / 3;
    constexpr int REM = LOGR % 3;
    int log_ps = 0;
#pragma unroll 1
    for (int s = 0; s < NS8; s++) {
        const bool last = (s == NS8 - 1) && (REM == 0);
        stage8<LOGR>(x, lt, log_ps, last, a.tw, a.log_n, s == 0 ? in_mul : nullptr, in_base, log_items, po);
        log_ps += 3;
    }
    if (REM == 2) stage4_last<LOGR>(x, lt, a.tw, a.log_n, po, NS8 == 0 ? in_mul : nullptr, in_base, log_items);
    if (REM == 1) stage2_last<LOGR>(x, lt, po);

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

// tiny transforms (n <= 4): direct O(n^2) evaluation by one thread per column
__global__ void ntt_tiny_kernel(NttPassArgs a) {
    const int n = 1 << a.log_n;
    const Fr* src = a.src + blockIdx.y * a.src_ys;
    Fr* dst = a.dst + blockIdx.y * a.dst_ys;
    if (threadIdx.x != 0) return;
    Fr x[4], y[4];
    for (int i = 0; i < n; i++) {
        x[i] = ld_elem<FrCfg>(src + i);
        if (a.in_mul) x[i] = fe_mul<FrCfg>(x[i], ld_elem<FrCfg>(a.in_mul + i));
    }
    for (int j = 0; j < n; j++) {
        Fr acc = fe_zero<FrCfg>();
        for (int i = 0; i < n; i++) {
            Fr t = x[i];
            int e = (i * j) & (n - 1);
            if (e) t = fe_mul<FrCfg>(t, ld_elem<FrCfg>(a.tw + e));
            acc = fe_add<FrCfg>(acc, t);
        }
        if (a.scale) acc = fe_mul<FrCfg>(acc, ld_elem<FrCfg>(a.scale));
        y[j] = acc;
    }
    for (int j = 0; j < n; j++) st_elem<FrCfg>(dst + ((size_t)j << a.out_shift), y[j]);
}

// ---------------------------------------------------------------- launchers

template <int LOGR, int G>
static cudaError_t launch_pass(const NttPassArgs& a, unsigned ny, unsigned nz, cudaStream_t s) {
    constexpr int R = 1 << LOGR;
    constexpr int T = (G * R) / 8;
    const size_t smem = (size_t)G * R * sizeof(Fr);
    static bool attr_set = false;
    if (!attr_set) {
        ZK_CHECK(cudaFuncSetAttribute(ntt_pass_kernel<LOGR, G>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)smem));
        attr_set = true;
    }
    const unsigned items = 1u << (a.log_n - LOGR);
    dim3 grid(items / G, ny, nz);
    ntt_pass_kernel<LOGR, G><<<grid, T, smem, s>>>(a);
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

cudaError_t ntt_pass(const NttPassArgs& a, int log_r, unsigned ny, unsigned nz, cudaStream_t s) {
    if (a.log_n <= 2) {
        ntt_tiny_kernel<<<dim3(1, ny, nz), 32, 0, s>>>(a);
        return cudaGetLastError();
    }
    const int g = pass_group(log_r, a.log_n);
#define ZK_PASS(LR, GG) \
    if (log_r == LR && g == GG) return launch_pass<LR, GG>(a, ny, nz, s);
    ZK_PASS(3, 1) ZK_PASS(4, 1) ZK_PASS(5, 1) ZK_PASS(6, 1) ZK_PASS(7, 1) ZK_PASS(8, 1)
    ZK_PASS(9, 1) ZK_PASS(10, 1) ZK_PASS(11, 1) ZK_PASS(12, 1)
    ZK_PASS(6, 2) ZK_PASS(6, 4) ZK_PASS(6, 8) ZK_PASS(6, 16)
    ZK_PASS(7, 2) ZK_PASS(7, 4) ZK_PASS(7, 8)
    ZK_PASS(8, 2) ZK_PASS(8, 4)
    ZK_PASS(9, 2)
#undef ZK_PASS
    return cudaErrorInvalidValue;
}

// split log_n into pass radices (at most 12 bits per pass, as even as possible)
int ntt_plan(int log_n, int radices[4]) {
    if (log_n <= 12) {
        radices[0] = log_n;
        return 1;
    }
    int np = (log_n + 11) / 12;
    if (np < 2) np = 2;
    for (int i = 0; i < np; i++) radices[i] = log_n / np + (i < log_n % np ? 1 : 0);
    return np;
}

cudaError_t ntt_run(Fr* buf, Fr* tmp, const Fr* tw, const Fr* scale, int log_n, unsigned ncols,
                    size_t col_stride, bool* result_in_tmp, cudaStream_t s) {
    int rad[4];
    const int np = ntt_plan(log_n, rad);
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

// buf[i] = w^i for 2 <= i < n, with w = buf[1] (entries 0 and 1 written by the host)
__global__ void expand_powers_kernel(Fr* buf, uint32_t n, uint32_t chunk) {
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    uint32_t s = t * chunk, e = s + chunk;
    if (s < 2) s = 2;
    if (e > n) e = n;
    if (s >= e) return;
    Fr w = ld_elem<FrCfg>(buf + 1);
    Fr cur = fe_pow_u32<FrCfg>(w, s);
    for (uint32_t i = s; i < e; i++) {
        st_elem<FrCfg>(buf + i, cur);
        cur = fe_mul<FrCfg>(cur, w);
    }
}

cudaError_t expand_powers(Fr* buf, uint32_t n, cudaStream_t s) {
    if (n <= 2) return cudaSuccess;
    const uint32_t chunk = 16;
    const uint32_t threads = (n + chunk - 1) / chunk;
    expand_powers_kernel<<<(threads + 127) / 128, 128, 0, s>>>(buf, n, chunk);
    return cudaGetLastError();
}

// out[i] = base * w^i for i < n, w and base given by value in device memory
__global__ void geometric_kernel(Fr* out, const Fr* base, const Fr* w, uint32_t n, uint32_t chunk) {
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    uint32_t s = t * chunk, e = s + chunk;
    if (e > n) e = n;
    if (s >= e) return;
    Fr ww = ld_elem<FrCfg>(w);
    Fr cur = fe_mul<FrCfg>(ld_elem<FrCfg>(base), fe_pow_u32<FrCfg>(ww, s));
    for (uint32_t i = s; i < e; i++) {
        st_elem<FrCfg>(out + i, cur);
        cur = fe_mul<FrCfg>(cur, ww);
    }
}

cudaError_t geometric(Fr* out, const Fr* base, const Fr* w, uint32_t n, cudaStream_t s) {
    const uint32_t chunk = 16;
    const uint32_t threads = (n + chunk - 1) / chunk;
    geometric_kernel<<<(threads + 127) / 128, 128, 0, s>>>(out, base, w, n, chunk);
    return cudaGetLastError();
}

}  // namespace zk
