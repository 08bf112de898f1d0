// Device scans over BN254 Fr: batch inversion (Montgomery's trick), exclusive
// prefix products and sums with a carried-in initial value, and the grand
// products / sums of the permutation, shuffle and logup arguments built on them.
//
// Reference behaviour replaced:
//   logup_sum_input_inv        cuda/bn254.cu:19-61, 1914-1934 (one serial chunk
//                              and one inversion per thread)
//   eval_logup_z_compose/pure  cuda/bn254.cu:63-220, 1936-1993 (5 launches, a
//                              single-thread middle level)
//   permutation product        src/permutation.rs:16-150 (CPU, rayon)
//   shuffle product            src/shuffle.rs:143-212 (CPU, rayon)
#include "common.cuh"
#include "kernels.h"

namespace zk {

static constexpr int ST = 256;  // threads per block
static constexpr int SK = 8;    // elements per thread
static constexpr int SBLK = ST * SK;

enum { OP_ADD = 0, OP_MUL = 1 };

__device__ __forceinline__ Fr op_apply(int op, const Fr& a, const Fr& b) {
    return op == OP_MUL ? fe_mul<FrCfg>(a, b) : fe_add<FrCfg>(a, b);
}
__device__ __forceinline__ Fr op_ident(int op) { return op == OP_MUL ? fe_one<FrCfg>() : fe_zero<FrCfg>(); }

__device__ __forceinline__ Fr shfl_up_fr(const Fr& v, int o) {
    Fr r;
#pragma unroll
    for (int j = 0; j < 8; j++) r.v[j] = __shfl_up_sync(0xffffffffu, v.v[j], o);
    return r;
}

// block-wide exclusive scan of one value per thread (thread order);
// wsm holds at least 32 elements
__device__ Fr block_excl_scan_fr(int op, const Fr& v, Fr* wsm, Fr& total) {
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
    Fr x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        Fr y = shfl_up_fr(x, o);
        if (lane >= o) x = op_apply(op, y, x);
    }
    Fr e = shfl_up_fr(x, 1);
    if (lane == 0) e = op_ident(op);
    if (lane == 31) wsm[wid] = x;
    __syncthreads();
    if (wid == 0) {
        Fr w = lane < nw ? wsm[lane] : op_ident(op);
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            Fr y = shfl_up_fr(w, o);
            if (lane >= o) w = op_apply(op, y, w);
        }
        if (lane < nw) wsm[lane] = w;
    }
    __syncthreads();
    total = wsm[nw - 1];
    Fr r = wid ? op_apply(op, wsm[wid - 1], e) : e;
    __syncthreads();
    return r;
}

// ------------------------------------------------------------ batch inverse
// Montgomery's trick over a block of ST * SK elements: one field inversion per
// block.  Thread t owns elements base + t + ST*k (coalesced); its chunk
// product is combined with the exclusive prefix E_t and suffix S_t of the
// other threads' products, so inv(chunk_t) = inv(total) * S_t * E_t, and the
// chunk is unwound locally.  The element value comes from a functor that is
// evaluated twice (forward and backward) instead of being stored, so the
// kernel needs no scratch memory.  Zero elements invert to zero.

struct SrcPlus {  // in[i] + c  (c optional)
    const Fr* in;
    const Fr* c;
    __device__ __forceinline__ Fr operator()(uint32_t i) const {
        Fr a = ld_elem<FrCfg>(in + i);
        return c ? fe_add<FrCfg>(a, ld_elem<FrCfg>(c)) : a;
    }
};

struct SrcPointDiff {  // prod_j (omegas[i] - points[j])
    const Fr* omegas;
    const Fr* points;
    int np;
    __device__ __forceinline__ Fr operator()(uint32_t i) const {
        const Fr w = ld_elem<FrCfg>(omegas + i);
        Fr t = fe_sub<FrCfg>(w, ld_elem<FrCfg>(points));
        for (int j = 1; j < np; j++) t = fe_mul<FrCfg>(t, fe_sub<FrCfg>(w, ld_elem<FrCfg>(points + j)));
        return t;
    }
};

struct DstStore {  // out[i] = (acc ? out[i] : 0) + inv
    Fr* out;
    int acc;
    __device__ __forceinline__ void operator()(uint32_t i, const Fr& v) const {
        st_elem<FrCfg>(out + i, acc ? fe_add<FrCfg>(v, ld_elem<FrCfg>(out + i)) : v);
    }
};

struct DstScale {  // out[i] *= inv
    Fr* out;
    __device__ __forceinline__ void operator()(uint32_t i, const Fr& v) const {
        st_elem<FrCfg>(out + i, fe_mul<FrCfg>(ld_elem<FrCfg>(out + i), v));
    }
};

// product of each block's SBLK elements (zeros count as one), for the
// three-phase form below
template <class Src>
__global__ void __launch_bounds__(ST) batch_prod_kernel(Src src, uint32_t n, Fr* tot) {
    __shared__ Fr wsm[32];
    const size_t base = (size_t)blockIdx.x * SBLK;
    const int t = threadIdx.x;
    const Fr one = fe_one<FrCfg>();
    Fr run = one;
#pragma unroll
    for (int k = 0; k < SK; k++) {
        const size_t i = base + t + (size_t)ST * k;
        if (i < n) {
            Fr a = src((uint32_t)i);
            if (!fe_is_zero<FrCfg>(a)) run = fe_mul<FrCfg>(run, a);
        }
    }
    Fr total;
    block_excl_scan_fr(OP_MUL, run, wsm, total);
    if (t == 0) st_elem<FrCfg>(tot + blockIdx.x, total);
}

// inv_tots: the inverses of the block products (three-phase form), or null
// to invert each block's product in the block (one Fermat inversion per block)
// The per-thread prefix products live in shared memory (SK x ST elements,
// 64 KB), not registers: at about 80 registers three blocks fit an SM, so
// while one block waits on its inversion (about 36 us on one thread) two
// others compute.
static constexpr size_t BATCH_INV_SMEM = (size_t)SK * ST * sizeof(Fr);

template <class Src, class Dst>
__global__ void __launch_bounds__(ST, 3) batch_inv_kernel(Src src, Dst dst, uint32_t n, const Fr* inv_tots) {
    __shared__ Fr wsm[32];
    __shared__ Fr rev[ST];
    __shared__ Fr inv_tot;
    extern __shared__ uint4 smem_u4[];
    Fr* pre_sm = reinterpret_cast<Fr*>(smem_u4);  // [k][t]
    const size_t base = (size_t)blockIdx.x * SBLK;
    const int t = threadIdx.x;
    const Fr one = fe_one<FrCfg>();
    Fr run = one;
#pragma unroll
    for (int k = 0; k < SK; k++) {
        const size_t i = base + t + (size_t)ST * k;
        Fr a = one;
        if (i < n) {
            a = src((uint32_t)i);
            if (fe_is_zero<FrCfg>(a)) a = one;
        }
        run = fe_mul<FrCfg>(run, a);
        pre_sm[k * ST + t] = run;
    }
    Fr tot;
    Fr E = block_excl_scan_fr(OP_MUL, run, wsm, tot);
    rev[ST - 1 - t] = run;
    __syncthreads();
    Fr rv = rev[t];
    __syncthreads();
    Fr tot2;
    Fr Srev = block_excl_scan_fr(OP_MUL, rv, wsm, tot2);
    rev[ST - 1 - t] = Srev;
    __syncthreads();
    Fr S = rev[t];
    if (t == 0) inv_tot = inv_tots ? ld_elem<FrCfg>(inv_tots + blockIdx.x) : fe_inv<FrCfg>(tot);
    __syncthreads();
    Fr cur = fe_mul<FrCfg>(fe_mul<FrCfg>(inv_tot, S), E);
#pragma unroll
    for (int k = SK - 1; k >= 0; k--) {
        const size_t i = base + t + (size_t)ST * k;
        Fr a = one;
        bool zero = true;
        if (i < n) {
            a = src((uint32_t)i);
            zero = fe_is_zero<FrCfg>(a);
            if (zero) a = one;
        }
        Fr inv_k = k ? fe_mul<FrCfg>(cur, pre_sm[(k - 1) * ST + t]) : cur;
        cur = fe_mul<FrCfg>(cur, a);
        if (i < n) dst((uint32_t)i, zero ? fe_zero<FrCfg>() : inv_k);
    }
}

// Scratch elements of the three-phase form for n elements: the block
// products and their inverses, then the same for the blocks of those.
size_t batch_inv_scratch_elems(uint32_t n) {
    const uint32_t nb = (n + SBLK - 1) / SBLK;
    return nb <= 1 ? 0 : 2 * (size_t)nb + batch_inv_scratch_elems(nb);
}

// With scratch of batch_inv_scratch_elems(n) and n above 2^22: (1) block
// products, (2) their inverses by the same routine (recursively, one field
// inversion at the top), (3) every block unwound with its product's inverse.
// Otherwise each block inverts its own product (binary extended Euclid, about
// 30 us of one thread while the block waits): measured on B200 this is the
// faster form up to 2^22 elements (0.078 against 0.136 ms at 2^16, 0.57
// against 0.64 ms at 2^22), the extra pass of the three-phase form costing
// more than the inversion stalls that other resident blocks partly hide.
static constexpr uint32_t BATCH_INV_THREE_PHASE_ABOVE = 1u << 22;

template <class Src, class Dst>
static cudaError_t launch_batch_inv(Src src, Dst dst, uint32_t n, Fr* scratch, size_t scratch_elems, cudaStream_t s) {
    if (n == 0) return cudaSuccess;
    static SmemOptIn opt;
    ZK_CHECK(opt.ensure(batch_inv_kernel<Src, Dst>, (int)BATCH_INV_SMEM));
    const uint32_t nb = (n + SBLK - 1) / SBLK;
    if (n > BATCH_INV_THREE_PHASE_ABOVE && scratch && scratch_elems >= batch_inv_scratch_elems(n)) {
        Fr* tot = scratch;
        Fr* inv = scratch + nb;
        batch_prod_kernel<Src><<<nb, ST, 0, s>>>(src, n, tot);
        ZK_CHECK(cudaGetLastError());
        ZK_CHECK(launch_batch_inv(SrcPlus{tot, nullptr}, DstStore{inv, 0}, nb, scratch + 2 * (size_t)nb,
                                  scratch_elems - 2 * (size_t)nb, s));
        batch_inv_kernel<Src, Dst><<<nb, ST, BATCH_INV_SMEM, s>>>(src, dst, n, inv);
        return cudaGetLastError();
    }
    batch_inv_kernel<Src, Dst><<<nb, ST, BATCH_INV_SMEM, s>>>(src, dst, n, nullptr);
    return cudaGetLastError();
}

cudaError_t batch_inverse(Fr* out, const Fr* in, const Fr* c, uint32_t n, int accumulate, Fr* scratch,
                          size_t scratch_elems, cudaStream_t s) {
    return launch_batch_inv(SrcPlus{in, c}, DstStore{out, accumulate}, n, scratch, scratch_elems, s);
}

// values[i] /= prod_j (omegas[i] - points[j])
cudaError_t div_by_point_diffs(Fr* values, const Fr* omegas, const Fr* points, int np, uint32_t n, Fr* scratch,
                               size_t scratch_elems, cudaStream_t s) {
    if (np <= 0) return cudaSuccess;
    return launch_batch_inv(SrcPointDiff{omegas, points, np}, DstScale{values}, n, scratch, scratch_elems, s);
}

// ------------------------------------------------------------ exclusive scan

// single block: exclusive scan of m <= SBLK values with init, in place; optional total
__global__ void __launch_bounds__(ST) scan_small_kernel(Fr* x, uint32_t m, int op, const Fr* init) {
    __shared__ Fr wsm[32];
    const size_t base = (size_t)threadIdx.x * SK;
    Fr v[SK];
    Fr run = op_ident(op);
#pragma unroll
    for (int k = 0; k < SK; k++) {
        Fr a = (base + k < m) ? ld_elem<FrCfg>(x + base + k) : op_ident(op);
        v[k] = run;
        run = op_apply(op, run, a);
    }
    Fr tot;
    Fr e = block_excl_scan_fr(op, run, wsm, tot);
    const Fr i0 = init ? ld_elem<FrCfg>(init) : op_ident(op);
    e = op_apply(op, i0, e);
#pragma unroll
    for (int k = 0; k < SK; k++)
        if (base + k < m) st_elem<FrCfg>(x + base + k, op_apply(op, e, v[k]));
}

// ------------------------------------------------------------ single-pass scan
// One launch over tiles of SBLK elements (decoupled look-back).  A block takes
// the next tile number from an atomic ticket, so every tile it waits on
// belongs to a block that started before it and is running; it scans its tile
// locally, publishes the tile's aggregate (state 1), then one warp looks back
// over the preceding tiles 32 at a time, combining aggregates until it meets a
// published inclusive prefix (state 2), and publishes its own inclusive
// prefix.  The elements are read once and written once.  The prefix product
// uses it: there the two products per element hide the waits.  The prefix
// sum, bound by HBM, runs as reduce-then-scan (further below).
//
// Every wait polls at most SCAN_POLL_LIMIT times.  A wait that runs out adds
// one to the device counter g_scan_timeouts (zkp_scan_timeouts reads it), takes
// the missing tile as the identity and carries on, so a launch always ends.

static constexpr uint32_t SCAN_POLL_LIMIT = 1u << 22;
__device__ uint32_t g_scan_timeouts;

struct ScanTiles {
    uint32_t* words;  // [0] the ticket, [1 .. 1 + nb) tile states
    Fr* agg;          // nb tile aggregates
    Fr* incl;         // nb inclusive prefixes
};

__device__ __forceinline__ uint32_t ld_acquire_u32(const uint32_t* p) {
    uint32_t v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_release_u32(uint32_t* p, uint32_t v) {
    asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
// a value another block published: read past L1
__device__ __forceinline__ Fr ldcg_fr(const Fr* p) {
    const uint4* q = reinterpret_cast<const uint4*>(p);
    const uint4 a = __ldcg(q), b = __ldcg(q + 1);
    Fr r;
    r.v[0] = a.x; r.v[1] = a.y; r.v[2] = a.z; r.v[3] = a.w;
    r.v[4] = b.x; r.v[5] = b.y; r.v[6] = b.z; r.v[7] = b.w;
    return r;
}
__device__ __forceinline__ Fr shfl_xor_fr(const Fr& v, int m) {
    Fr r;
#pragma unroll
    for (int j = 0; j < 8; j++) r.v[j] = __shfl_xor_sync(0xffffffffu, v.v[j], m);
    return r;
}

// The tile passes through shared memory (swizzled 32-byte slots, sm_slot) so
// that global loads and stores are coalesced 16-byte accesses while each
// thread scans SK consecutive elements.
static constexpr size_t SCAN_TILE_SMEM = (size_t)SBLK * sizeof(Fr);

// OPK: the operation, fixed at compile time (OP_MUL: the sum uses the
// reduce-then-scan form below).
template <int OPK>
__global__ void __launch_bounds__(ST, 2) scan_onepass_kernel(Fr* out, const Fr* in, uint32_t n, const Fr* init,
                                                              ScanTiles tiles) {
    constexpr int op = OPK;
    __shared__ Fr wsm[32];
    __shared__ uint32_t s_tile;
    __shared__ Fr s_prefix;
    extern __shared__ uint4 smem_u4[];
    Fr* sm = reinterpret_cast<Fr*>(smem_u4);
    if (threadIdx.x == 0) s_tile = atomicAdd(tiles.words, 1u);
    __syncthreads();
    const uint32_t tile = s_tile;
    const size_t t0 = (size_t)tile * SBLK;
    const uint32_t cnt = n - t0 < (size_t)SBLK ? (uint32_t)(n - t0) : (uint32_t)SBLK;
    {
        const Fr id = op_ident(op);
        const uint4* src = reinterpret_cast<const uint4*>(in + t0);
        for (uint32_t c = threadIdx.x; c < 2u * SBLK; c += ST) {
            const uint32_t e = c >> 1, h = c & 1;
            *sm_slot(sm, e, h) = e < cnt ? src[c]
                                         : (h ? make_uint4(id.v[4], id.v[5], id.v[6], id.v[7])
                                              : make_uint4(id.v[0], id.v[1], id.v[2], id.v[3]));
        }
    }
    __syncthreads();
    const uint32_t lbase = threadIdx.x * SK;
    Fr v[SK];
    Fr run = op_ident(op);
#pragma unroll
    for (int k = 0; k < SK; k++) {
        const Fr a = sm_ld(sm, lbase + k);
        v[k] = run;
        run = op_apply(op, run, a);
    }
    Fr tot;
    const Fr e = block_excl_scan_fr(op, run, wsm, tot);
    uint32_t* state = tiles.words + 1;
    if (threadIdx.x < 32) {
        const int lane = threadIdx.x;
        Fr prefix = op_ident(op);
        if (tile == 0) {
            if (init) prefix = ld_elem<FrCfg>(init);
        } else {
            if (lane == 0) {
                st_elem<FrCfg>(tiles.agg + tile, tot);
                st_release_u32(state + tile, 1u);
            }
            // window of the 32 tiles p, p - 1, ..., p - 31 (lane order)
            int64_t p = (int64_t)tile - 1;
            for (;;) {
                const int64_t idx = p - lane;
                uint32_t f = 2;  // before tile 0: never reached, tile 0 is inclusive
                Fr val = op_ident(op);
                if (idx >= 0) {
                    f = ld_acquire_u32(state + idx);
                    uint32_t polls = 0;
                    while (f == 0 && ++polls < SCAN_POLL_LIMIT) {
                        __nanosleep(64);
                        f = ld_acquire_u32(state + idx);
                    }
                    if (f == 0) {
                        atomicAdd(&g_scan_timeouts, 1u);
                        f = 1;
                    } else {
                        val = ldcg_fr(f == 2 ? tiles.incl + idx : tiles.agg + idx);
                    }
                }
                // the nearest inclusive prefix ends the walk: lanes up to it count
                const unsigned incl_mask = __ballot_sync(0xffffffffu, f == 2);
                const int last = incl_mask ? __ffs(incl_mask) - 1 : 31;
                Fr c = lane <= last ? val : op_ident(op);
#pragma unroll
                for (int m = 16; m > 0; m >>= 1) c = op_apply(op, c, shfl_xor_fr(c, m));
                prefix = op_apply(op, c, prefix);
                if (incl_mask) break;
                p -= 32;
            }
        }
        if (lane == 0) {
            st_elem<FrCfg>(tiles.incl + tile, op_apply(op, prefix, tot));
            st_release_u32(state + tile, 2u);
            s_prefix = prefix;
        }
    }
    __syncthreads();
    const Fr pre = op_apply(op, s_prefix, e);
#pragma unroll
    for (int k = 0; k < SK; k++) sm_st(sm, lbase + k, op_apply(op, pre, v[k]));
    __syncthreads();
    uint4* dst = reinterpret_cast<uint4*>(out + t0);
    for (uint32_t c = threadIdx.x; c < 2u * cnt; c += ST) dst[c] = *sm_slot(sm, c >> 1, c & 1);
}

// Reduce-then-scan, for the sum (bound by HBM, where the look-back's waits
// cost more than they save), over segments of 256 elements, one warp each,
// read row by row (32 consecutive elements an instruction): (1) every
// segment's sum, (2) their exclusive scan with the initial value (this routine
// again above 2048 segments), (3) every segment scanned from its prefix, each
// row by shuffles with the carry of the rows before it.  No shared tile and no
// block barrier, so few registers and many warps per SM hide the loads; the
// elements are read twice and written once.
static constexpr uint32_t WSEG = 256;

__global__ void __launch_bounds__(256) seg_sum_kernel(const Fr* in, uint32_t n, Fr* agg) {
    const uint32_t w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    const size_t base = (size_t)w * WSEG;
    if (base >= n) return;  // the whole warp: w is uniform across it
    Fr acc = fe_zero<FrCfg>();
#pragma unroll
    for (uint32_t k = 0; k < WSEG / 32; k++) {
        const size_t i = base + k * 32 + lane;
        if (i < n) acc = fe_add<FrCfg>(acc, ld_elem<FrCfg>(in + i));
    }
#pragma unroll
    for (int m = 16; m > 0; m >>= 1) acc = fe_add<FrCfg>(acc, shfl_xor_fr(acc, m));
    if (lane == 0) st_elem<FrCfg>(agg + w, acc);
}

// out may alias in: a warp reads each row before it writes it, and segments
// belong to one warp each
__global__ void __launch_bounds__(256) seg_scan_kernel(Fr* out, const Fr* in, uint32_t n, const Fr* pre) {
    const uint32_t w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    const size_t base = (size_t)w * WSEG;
    if (base >= n) return;
    Fr carry = ld_elem<FrCfg>(pre + w);
#pragma unroll 1
    for (uint32_t k = 0; k < WSEG / 32; k++) {
        const size_t i = base + k * 32 + lane;
        const Fr x = i < n ? ld_elem<FrCfg>(in + i) : fe_zero<FrCfg>();
        Fr v = x;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const Fr y = shfl_up_fr(v, o);
            if ((int)lane >= o) v = fe_add<FrCfg>(y, v);
        }
        Fr e = shfl_up_fr(v, 1);
        if (lane == 0) e = fe_zero<FrCfg>();
        if (i < n) st_elem<FrCfg>(out + i, fe_add<FrCfg>(carry, e));
        Fr tot;
#pragma unroll
        for (int j = 0; j < 8; j++) tot.v[j] = __shfl_sync(0xffffffffu, v.v[j], 31);
        carry = fe_add<FrCfg>(carry, tot);
    }
}

// scratch of the sum's reduce-then-scan: the segment sums, then the same for
// the segment sums' own scan
static size_t seg_scan_elems(uint32_t n) {
    if (n <= (uint32_t)SBLK) return 0;
    const uint32_t ns = (n + WSEG - 1) / WSEG;
    return ns + seg_scan_elems(ns);
}

// tile states after the aggregates and prefixes, in Fr elements
static size_t onepass_elems(uint32_t nb) { return 2 * (size_t)nb + ((size_t)nb + 1 + 7) / 8; }

// scratch of the scans, also enough for the three-phase batch inversion
// (the callers below use it for both, one after the other)
size_t fr_scan_tmp_elems(uint32_t n) {
    const uint32_t nb = (n + SBLK - 1) / SBLK;
    size_t one = n > (uint32_t)SBLK ? onepass_elems(nb) : 1;
    if (seg_scan_elems(n) > one) one = seg_scan_elems(n);
    const size_t inv = batch_inv_scratch_elems(n);
    return one > inv ? one : inv;
}

uint32_t fr_scan_timeouts() {
    uint32_t v = 0;
    if (cudaMemcpyFromSymbol(&v, g_scan_timeouts, sizeof(v)) != cudaSuccess) return 0xffffffffu;
    return v;
}

// out[i] = init op x_0 op ... op x_{i-1}; out may alias in (each tile is read
// whole before it is written, and no block reads another's elements)
cudaError_t fr_scan_excl(Fr* out, const Fr* in, uint32_t n, const Fr* init, int op, Fr* tmp, cudaStream_t s) {
    if (n == 0) return cudaSuccess;
    if (n <= (uint32_t)SBLK) {
        if (out != in) ZK_CHECK(cudaMemcpyAsync(out, in, (size_t)n * sizeof(Fr), cudaMemcpyDeviceToDevice, s));
        scan_small_kernel<<<1, ST, 0, s>>>(out, n, op, init);
        return cudaGetLastError();
    }
    if (!tmp) return cudaErrorInvalidValue;
    if (op == OP_ADD) {
        const uint32_t ns = (n + WSEG - 1) / WSEG;
        const unsigned blocks = (unsigned)(((uint64_t)ns * 32 + 255) / 256);
        seg_sum_kernel<<<blocks, 256, 0, s>>>(in, n, tmp);
        ZK_CHECK(cudaGetLastError());
        ZK_CHECK(fr_scan_excl(tmp, tmp, ns, init, op, tmp + ns, s));
        seg_scan_kernel<<<blocks, 256, 0, s>>>(out, in, n, tmp);
        return cudaGetLastError();
    }
    if (op != OP_MUL) return cudaErrorInvalidValue;
    const uint32_t nb = (n + SBLK - 1) / SBLK;
    ScanTiles tiles;
    tiles.agg = tmp;
    tiles.incl = tmp + nb;
    tiles.words = reinterpret_cast<uint32_t*>(tmp + 2 * (size_t)nb);
    static SmemOptIn opt;
    ZK_CHECK(opt.ensure(scan_onepass_kernel<OP_MUL>, (int)SCAN_TILE_SMEM));
    ZK_CHECK(cudaMemsetAsync(tiles.words, 0, ((size_t)nb + 1) * sizeof(uint32_t), s));
    scan_onepass_kernel<OP_MUL><<<nb, ST, SCAN_TILE_SMEM, s>>>(out, in, n, init, tiles);
    return cudaGetLastError();
}

// ------------------------------------------------------------------- logup

__global__ void logup_step2_kernel(Fr* z, const Fr* sum, const Fr* m, uint32_t n) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        st_elem<FrCfg>(z + i, fe_sub<FrCfg>(ld_elem<FrCfg>(sum + i), fe_mul<FrCfg>(ld_elem<FrCfg>(m + i), ld_elem<FrCfg>(z + i))));
}

__global__ void copy_elem_kernel(Fr* dst, const Fr* src) {
    if (threadIdx.x == 0) st_elem<FrCfg>(dst, ld_elem<FrCfg>(src));
}

// z = exclusive prefix sum of z starting at *last_z; then *last_z = z[last_index]
cudaError_t logup_z_scan(Fr* z, Fr* last_z, int last_index, uint32_t n, Fr* tmp, cudaStream_t s) {
    ZK_CHECK(fr_scan_excl(z, z, n, last_z, OP_ADD, tmp, s));
    if (last_index >= 0 && (uint32_t)last_index < n) {
        copy_elem_kernel<<<1, 32, 0, s>>>(last_z, z + last_index);
        ZK_CHECK(cudaGetLastError());
    }
    return cudaSuccess;
}

cudaError_t logup_z_compose(Fr* z, const Fr* sum, const Fr* table, const Fr* m, const Fr* beta, Fr* last_z,
                            int last_index, uint32_t n, Fr* tmp, cudaStream_t s) {
    // tmp may be the table itself (the reference-ABI entry reuses it once the
    // inverses are taken); then the inversion runs without scratch
    Fr* inv_scratch = tmp == table ? nullptr : tmp;
    ZK_CHECK(batch_inverse(z, table, beta, n, 0, inv_scratch, fr_scan_tmp_elems(n), s));
    unsigned nb = (n + 255) / 256;
    if (nb > 148 * 32) nb = 148 * 32;
    logup_step2_kernel<<<nb, 256, 0, s>>>(z, sum, m, n);
    ZK_CHECK(cudaGetLastError());
    return logup_z_scan(z, last_z, last_index, n, tmp, s);
}

// ------------------------------------------------ permutation / shuffle ratio
// d[i] = prod_c (v_c[i] + beta*delta^c*w^i + gamma) / prod_c (v_c[i] + beta*sigma_c[i] + gamma)
// with delta^c for the chunk's columns given as dpow[c] (c < ncols).

__global__ void perm_den_kernel(Fr* den, const Fr* const* cols, const Fr* const* sig, int ncols, const Fr* beta,
                                const Fr* gamma, uint32_t n) {
    // beta is a known factor; the product stays lazily reduced until the store
    const KnownFr kb = block_known(beta);
    const Fr g = ld_elem<FrCfg>(gamma);
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        Fr acc = fe_one<FrCfg>();
        for (int c = 0; c < ncols; c++) {
            const Fr t = fe_add_lazy<FrCfg>(fe_add_lazy<FrCfg>(mul_known(ld_elem<FrCfg>(sig[c] + i), kb), g),
                                            ld_elem<FrCfg>(cols[c] + i));
            acc = c ? fe_mul_lazy<FrCfg>(acc, t) : t;
        }
        st_elem<FrCfg>(den + i, fe_canon<FrCfg>(acc));
    }
}

// d[i] = inv_den[i] * prod_c (v_c[i] + beta*delta^c*w^i + gamma); omega table
// w^i.  The beta delta^c of up to PERM_KNOWN columns are staged per block as
// known factors; the product stays lazily reduced until the store.
static constexpr int PERM_KNOWN = 64;

__global__ void perm_num_kernel(Fr* d, const Fr* const* cols, const Fr* dbeta, int ncols, const Fr* gamma,
                                const Fr* omegas, uint32_t n) {
    __shared__ KnownFr sk[PERM_KNOWN];
    const bool staged = ncols <= PERM_KNOWN;
    if (staged) {
        for (int c = threadIdx.x; c < ncols; c += blockDim.x) sk[c] = known_fr(ld_elem<FrCfg>(dbeta + c));
        __syncthreads();
    }
    const Fr g = ld_elem<FrCfg>(gamma);
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const Fr w = ld_elem<FrCfg>(omegas + i);
        Fr acc = ld_elem<FrCfg>(d + i);
        for (int c = 0; c < ncols; c++) {
            const Fr wb = staged ? mul_known(w, sk[c]) : fe_mul_lazy<FrCfg>(w, ld_elem<FrCfg>(dbeta + c));
            const Fr t = fe_add_lazy<FrCfg>(fe_add_lazy<FrCfg>(wb, g), ld_elem<FrCfg>(cols[c] + i));
            acc = fe_mul_lazy<FrCfg>(acc, t);
        }
        st_elem<FrCfg>(d + i, fe_canon<FrCfg>(acc));
    }
}

static unsigned grid_n(uint32_t n) {
    unsigned nb = (n + 255) / 256;
    if (nb > 148 * 32) nb = 148 * 32;
    return nb ? nb : 1;
}

// one chunk of the permutation argument: z = exclusive prefix product of the
// ratio, starting at *init (1 for the first chunk, the previous chunk's z at
// the last usable row otherwise).  dbeta[c] = beta * delta^(chunk_offset + c).
cudaError_t permutation_chunk_z(Fr* z, const Fr* const* cols, const Fr* const* sig, int ncols, const Fr* beta,
                                const Fr* gamma, const Fr* dbeta, const Fr* omegas, const Fr* init, uint32_t n,
                                Fr* tmp, cudaStream_t s) {
    perm_den_kernel<<<grid_n(n), 256, 0, s>>>(z, cols, sig, ncols, beta, gamma, n);
    ZK_CHECK(cudaGetLastError());
    ZK_CHECK(batch_inverse(z, z, nullptr, n, 0, tmp, fr_scan_tmp_elems(n), s));
    perm_num_kernel<<<grid_n(n), 256, 0, s>>>(z, cols, dbeta, ncols, gamma, omegas, n);
    ZK_CHECK(cudaGetLastError());
    return fr_scan_excl(z, z, n, init, OP_MUL, tmp, s);
}

// shuffle: z = exclusive prefix product of prod_g (input_g + beta_g) / prod_g (table_g + beta_g)
__global__ void shuffle_terms_kernel(Fr* den, Fr* num, const Fr* const* inputs, const Fr* const* tables,
                                     const Fr* betas, int groups, uint32_t n) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        // lazily reduced until the stores
        Fr a = fe_one<FrCfg>(), b = fe_one<FrCfg>();
        for (int g = 0; g < groups; g++) {
            const Fr bg = ld_elem<FrCfg>(betas + g);
            a = fe_mul_lazy<FrCfg>(a, fe_add_lazy<FrCfg>(ld_elem<FrCfg>(inputs[g] + i), bg));
            b = fe_mul_lazy<FrCfg>(b, fe_add_lazy<FrCfg>(ld_elem<FrCfg>(tables[g] + i), bg));
        }
        st_elem<FrCfg>(num + i, fe_canon<FrCfg>(a));
        st_elem<FrCfg>(den + i, fe_canon<FrCfg>(b));
    }
}

__global__ void mul_inplace_kernel(Fr* a, const Fr* b, uint32_t n) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        st_elem<FrCfg>(a + i, fe_mul<FrCfg>(ld_elem<FrCfg>(a + i), ld_elem<FrCfg>(b + i)));
}

cudaError_t shuffle_z(Fr* z, const Fr* const* inputs, const Fr* const* tables, const Fr* betas, int groups,
                      uint32_t n, Fr* num_tmp, Fr* tmp, cudaStream_t s) {
    shuffle_terms_kernel<<<grid_n(n), 256, 0, s>>>(z, num_tmp, inputs, tables, betas, groups, n);
    ZK_CHECK(cudaGetLastError());
    ZK_CHECK(batch_inverse(z, z, nullptr, n, 0, tmp, fr_scan_tmp_elems(n), s));
    mul_inplace_kernel<<<grid_n(n), 256, 0, s>>>(z, num_tmp, n);
    ZK_CHECK(cudaGetLastError());
    return fr_scan_excl(z, z, n, nullptr, OP_MUL, tmp, s);
}

}  // namespace zk
