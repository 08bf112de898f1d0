// A batch of MSMs of different sizes over one base array (an SRS prefix per
// MSM) in one pipeline: one key space for every bucket of every MSM, one
// counting sort, one accumulation pass, and the per-MSM window reductions and
// final combinations running side by side.  Each MSM keeps its own window
// width, so a schedule (autotuned or predicted) can pick it per size and scalar
// distribution.
//
// Reference behaviour replaced: the per-column msm() loop of
// src/cuda/msm.rs:319-350 followed by batch_msm_collect
// (cuda/msm.cu:434-467), which sorts and reduces one MSM at a time and combines
// windows on one thread per MSM.
#include <vector>

#include "common.cuh"
#include "kernels.h"
#include "glv.cuh"
#include "msm_common.cuh"

namespace zk {

struct BatchDesc {
    uint32_t n, c, W, B;
    uint32_t Wb;       // bucket sets: W, or 1 over a table of pre-multiplied bases
    uint32_t kw;       // key stride per window: B, or 0 over a table
    uint32_t key_off;  // first bucket key of this MSM
    uint32_t sc_off;   // first global scalar index of this MSM
    uint32_t G, seg;   // reduction segments per window and buckets per segment
    uint32_t red_off;  // first reduction thread
    uint32_t win_off;  // first window slot
};

// largest i in [0, count) with d[i].*field <= x
template <uint32_t BatchDesc::*F>
__device__ __forceinline__ uint32_t find_desc(const BatchDesc* d, uint32_t count, uint32_t x) {
    uint32_t lo = 0, hi = count;
    while (hi - lo > 1) {
        const uint32_t mid = (lo + hi) >> 1;
        if (d[mid].*F <= x)
            lo = mid;
        else
            hi = mid;
    }
    return lo;
}

// Every MSM of the batch runs on GLV halves: scalar j of an MSM becomes
// |k1| on base j and |k2| on phi(base j), stored at point phi_off + j
// (phi_off = nmax, the longest MSM's base prefix, whose images are computed
// once; or nsrs over a table, whose window j entry of point p sits at
// p + j pw).

__device__ __forceinline__ void batch_count_half(const uint32_t v[8], const BatchDesc& q, uint32_t* cnt) {
    uint32_t carry = 0;
    for (uint32_t w = 0; w < q.W; w++) {
        const int dg = msm_signed_digit(v, (int)w, (int)q.c, carry);
        if (dg != 0) {
            const uint32_t mag = dg > 0 ? (uint32_t)dg : (uint32_t)(-dg);
            atomicAdd(&cnt[q.key_off + w * q.kw + mag - 1], 1u);
        }
    }
}

__global__ void batch_count_kernel(const BatchDesc* d, uint32_t count, const Fr* const* scalars, uint32_t total,
                                   uint32_t* cnt) {
    for (uint32_t s = blockIdx.x * blockDim.x + threadIdx.x; s < total; s += gridDim.x * blockDim.x) {
        const uint32_t i = find_desc<&BatchDesc::sc_off>(d, count, s);
        const BatchDesc q = d[i];
        const Fr k = fe_from_mont<FrCfg>(ldg_elem<FrCfg>(scalars[i] + (s - q.sc_off)));
        uint32_t m1[8], m2[8];
        bool n1, n2;
        glv_split(k.v, m1, m2, n1, n2);
        batch_count_half(m1, q, cnt);
        batch_count_half(m2, q, cnt);
    }
}

// as scatter_digits of the single MSM: eight slot claims in flight together
__device__ __forceinline__ void batch_scatter_half(const uint32_t v[8], const BatchDesc& q, uint32_t point,
                                                   uint32_t pw, bool negate, const uint32_t* offset, uint32_t* cnt,
                                                   uint32_t* entries) {
    const uint32_t nbit = negate ? 0x80000000u : 0u;
    uint32_t carry = 0;
    for (uint32_t w0 = 0; w0 < q.W; w0 += 8) {
        uint32_t key[8], neg[8], base[8], slot[8];
#pragma unroll
        for (uint32_t u = 0; u < 8; u++) {
            key[u] = 0xffffffffu;
            neg[u] = 0;
            if (w0 + u < q.W) {
                const int dg = msm_signed_digit(v, (int)(w0 + u), (int)q.c, carry);
                if (dg != 0) {
                    const uint32_t mag = dg > 0 ? (uint32_t)dg : (uint32_t)(-dg);
                    key[u] = q.key_off + (w0 + u) * q.kw + mag - 1;
                    neg[u] = (dg < 0 ? 0x80000000u : 0u) ^ nbit;
                }
            }
        }
#pragma unroll
        for (uint32_t u = 0; u < 8; u++) {
            if (key[u] != 0xffffffffu) {
                slot[u] = atomicSub(&cnt[key[u]], 1u) - 1u;
                base[u] = offset[key[u]];
            }
        }
#pragma unroll
        for (uint32_t u = 0; u < 8; u++)
            if (key[u] != 0xffffffffu) entries[base[u] + slot[u]] = (point + (w0 + u) * pw) | neg[u];
    }
}

__global__ void batch_scatter_kernel(const BatchDesc* d, uint32_t count, const Fr* const* scalars, uint32_t total,
                                     uint32_t phi_off, uint32_t pw, const uint32_t* offset, uint32_t* cnt,
                                     uint32_t* entries) {
    for (uint32_t s = blockIdx.x * blockDim.x + threadIdx.x; s < total; s += gridDim.x * blockDim.x) {
        const uint32_t i = find_desc<&BatchDesc::sc_off>(d, count, s);
        const BatchDesc q = d[i];
        const uint32_t j = s - q.sc_off;
        const Fr k = fe_from_mont<FrCfg>(ldg_elem<FrCfg>(scalars[i] + j));
        uint32_t m1[8], m2[8];
        bool n1, n2;
        glv_split(k.v, m1, m2, n1, n2);
        batch_scatter_half(m1, q, j, pw, n1, offset, cnt, entries);
        batch_scatter_half(m2, q, phi_off + j, pw, n2, offset, cnt, entries);
    }
}

// as msm_reduce_kernel, over every MSM's (window, segment) threads; each
// MSM's threads start on a 128-thread boundary, so a CTA serves one MSM and
// its group trees (GS = min(G, 128) threads, one window) stay inside the CTA
__global__ void __launch_bounds__(128) batch_reduce_kernel(const BatchDesc* d, uint32_t count, uint32_t total,
                                                           const Xyzz* buckets, const uint32_t* offset,
                                                           Xyzz* segsum) {
    __shared__ Xyzz sm[128];
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t i = find_desc<&BatchDesc::red_off>(d, count, blockIdx.x * blockDim.x);
    const BatchDesc q = d[i];
    const uint32_t lt = t - q.red_off;
    Xyzz S = xyzz_identity();
    if (t < total && lt < q.Wb * q.G) {
        const uint32_t w = lt / q.G, g = lt % q.G;
        const uint32_t lo = g * q.seg;
        Xyzz T = xyzz_identity();
        for (uint32_t j = 0; j < q.seg; j++) {
            const uint32_t key = q.key_off + w * q.B + lo + q.seg - 1 - j;
            if (offset[key + 1] != offset[key]) T = xyzz_add(T, ld_xyzz(buckets + key));
            S = xyzz_add(S, T);
        }
        if (lo) S = xyzz_add(S, xyzz_mul_u32(T, lo));
    }
    const uint32_t GS = q.G < 128 ? q.G : 128;
    const uint32_t k = threadIdx.x;
    sm[k] = S;
    __syncthreads();
    for (uint32_t h = GS >> 1; h > 0; h >>= 1) {
        if ((k & (GS - 1)) < h) sm[k] = xyzz_add(sm[k], sm[k + h]);
        __syncthreads();
    }
    if ((k & (GS - 1)) == 0 && t < total && lt < q.Wb * q.G) st_xyzz(segsum + q.red_off + lt / GS, sm[k]);
}

// one CTA per (MSM, bucket set): adds the set's G / min(G, 128) group sums,
// each thread a strided subset first, then a tree (blockDim a power of two)
__global__ void __launch_bounds__(256) batch_window_kernel(const BatchDesc* d, uint32_t count, const Xyzz* segsum, Xyzz* winsum) {
    extern __shared__ uint4 smem_u4[];
    Xyzz* sm = reinterpret_cast<Xyzz*>(smem_u4);
    const uint32_t b = blockIdx.x, k = threadIdx.x;
    const uint32_t i = find_desc<&BatchDesc::win_off>(d, count, b);
    const BatchDesc q = d[i];
    const uint32_t w = b - q.win_off;
    const uint32_t parts = q.G < 128 ? 1u : q.G / 128u;
    Xyzz acc = xyzz_identity();
    for (uint32_t g = k; g < parts; g += blockDim.x) acc = xyzz_add(acc, ld_xyzz(segsum + q.red_off + w * parts + g));
    sm[k] = acc;
    __syncthreads();
    for (uint32_t h = blockDim.x >> 1; h > 0; h >>= 1) {
        if (k < h) sm[k] = xyzz_add(sm[k], sm[k + h]);
        __syncthreads();
    }
    if (k == 0) st_xyzz(winsum + b, sm[0]);
}

// one CTA of COOP_THREADS threads per MSM
__global__ void __launch_bounds__(COOP_THREADS) batch_final_kernel(const BatchDesc* d, const Xyzz* winsum,
                                                                    Jac* out) {
    __shared__ Fq buf[8];
    const uint32_t i = blockIdx.x;
    const BatchDesc q = d[i];
    const Jac j = coop_horner(buf, winsum + q.win_off, q.n ? (int)q.Wb : 0, (int)q.c);
    if (threadIdx.x == 0) {
        st_elem<FqCfg>(&out[i].x, j.x);
        st_elem<FqCfg>(&out[i].y, j.y);
        st_elem<FqCfg>(&out[i].z, j.z);
    }
}

// The descriptor table reaches the device through kernel parameters, DESC_CHUNK
// descriptors per launch (under the 4 KB classic parameter limit): a graph
// that captures the pipeline keeps them by value, where a copy from host
// memory would read a host buffer long gone at replay.
static constexpr uint32_t DESC_CHUNK = 64;
struct DescChunk {
    uint32_t count;
    BatchDesc d[DESC_CHUNK];
};

__global__ void batch_desc_kernel(BatchDesc* out, DescChunk c) {
    for (uint32_t i = threadIdx.x; i < c.count; i += blockDim.x) out[i] = c.d[i];
}

// ------------------------------------------------------------------ planning

struct BatchLayout {
    std::vector<BatchDesc> desc;
    uint32_t NB = 0, total = 0, red_total = 0, win_total = 0, L = 8, nacc = 1, maxG = 1, nmax = 0;
    uint64_t entries = 0;
    size_t off_desc = 0, off_cnt = 0, off_offset = 0, off_scan = 0, off_entries = 0, off_pkey = 0, off_ppt = 0,
           off_buckets = 0, off_segsum = 0, off_winsum = 0, off_phi = 0, bytes = 0;
};

static size_t al(size_t x) { return (x + 255) / 256 * 256; }

#ifndef ZK_MSM_BATCH_REDUCE_THREADS
#define ZK_MSM_BATCH_REDUCE_THREADS 131072
#endif
static constexpr uint64_t BATCH_REDUCE_THREADS = ZK_MSM_BATCH_REDUCE_THREADS;

// nsrs > 0: every MSM runs over one table of pre-multiplied bases of width
// c[0] (one bucket set per MSM); otherwise per-MSM widths c[i] (0 or a null c:
// the library's choice) over the bases and their images
static bool batch_plan(const uint32_t* n, const int* c, uint32_t count, uint32_t nsrs, BatchLayout& L) {
    L.desc.resize(count);
    std::vector<MsmPlan> plans(count);
    uint64_t all_buckets = 0;
    for (uint32_t i = 0; i < count; i++) {
        if (nsrs && n[i] > nsrs) return false;
        plans[i] = nsrs ? msm_make_table_plan(n[i], c[0], nsrs) : msm_make_plan(n[i], c ? c[i] : 0, true);
        all_buckets += (uint64_t)plans[i].Wb * plans[i].B;
    }
    // The reduction threads of the whole batch share one budget, in
    // proportion to each MSM's buckets: a segment's closing product lo * T
    // costs about 1.5 c additions, so many MSMs with the single-MSM thread
    // counts would spend more on those than on the running sums themselves.
    for (uint32_t i = 0; i < count; i++) {
        MsmPlan& p = plans[i];
        const uint64_t share = BATCH_REDUCE_THREADS * (uint64_t)p.Wb * p.B / (all_buckets ? all_buckets : 1);
        uint32_t G = 1;
        while ((uint64_t)G * 2 * p.Wb <= share && G * 2 <= p.G) G *= 2;
        p.G = G;
        p.seg = p.B / G;
    }
    uint64_t key = 0, sc = 0, red = 0, win = 0, ent = 0;
    for (uint32_t i = 0; i < count; i++) {
        const MsmPlan& p = plans[i];
        BatchDesc& q = L.desc[i];
        q.n = n[i];
        q.c = (uint32_t)p.c;
        q.W = (uint32_t)p.W;
        q.B = p.B;
        q.Wb = (uint32_t)p.Wb;
        q.kw = nsrs ? 0u : p.B;
        q.key_off = (uint32_t)key;
        q.sc_off = (uint32_t)sc;
        q.G = p.G;
        q.seg = p.seg;
        red = (red + 127) / 128 * 128;  // each MSM's reduction threads start a CTA
        q.red_off = (uint32_t)red;
        q.win_off = (uint32_t)win;
        key += (uint64_t)p.Wb * p.B;
        sc += n[i];
        red += (uint64_t)p.Wb * p.G;
        red = (red + 127) / 128 * 128;
        win += p.Wb;
        ent += msm_entry_count(p);
        if (p.G > L.maxG) L.maxG = p.G;
        if (n[i] > L.nmax) L.nmax = n[i];
    }
    if (key >= 0xffffffffull || sc >= 0x7fffffffull || ent >= 0xffffffffull || red >= 0xffffffffull ||
        L.nmax >= 0x40000000u)
        return false;
    L.NB = (uint32_t)key;
    L.total = (uint32_t)sc;
    L.red_total = (uint32_t)red;
    L.win_total = (uint32_t)win;
    L.entries = ent;
    const uint64_t target = 148ull * 4 * 128;
    uint64_t Lp = (ent + target - 1) / target;
    if (Lp < 8) Lp = 8;
    L.L = (uint32_t)Lp;
    L.nacc = (uint32_t)((ent + Lp - 1) / Lp);
    if (L.nacc == 0) L.nacc = 1;
    size_t o = 0;
    L.off_desc = o;
    o = al(o + count * sizeof(BatchDesc));
    L.off_cnt = o;
    o = al(o + (size_t)L.NB * 4);
    L.off_offset = o;
    o = al(o + ((size_t)L.NB + 1) * 4);
    L.off_scan = o;
    o = al(o + scan_tmp_words(L.NB) * 4);
    L.off_entries = o;
    o = al(o + ent * 4);
    L.off_pkey = o;
    o = al(o + ((size_t)2 * L.nacc + msm_merge_extra(L.nacc)) * 4);
    L.off_ppt = o;
    o = al(o + ((size_t)2 * L.nacc + msm_merge_extra(L.nacc)) * sizeof(Xyzz));
    L.off_buckets = o;
    o = al(o + (size_t)L.NB * sizeof(Xyzz));
    L.off_segsum = o;
    o = al(o + (size_t)L.red_total * sizeof(Xyzz));
    L.off_winsum = o;
    o = al(o + (size_t)L.win_total * sizeof(Xyzz));
    L.off_phi = o;
    o = al(o + (nsrs ? 0 : (size_t)L.nmax * sizeof(Aff)));
    L.bytes = o;
    return true;
}

size_t msm_batch_scratch_bytes(const uint32_t* n, const int* c, uint32_t count, uint32_t nsrs) {
    BatchLayout L;
    if (count == 0 || !batch_plan(n, c, count, nsrs, L)) return 0;
    return L.bytes;
}

cudaError_t msm_batch_run(Jac* out, const Aff* bases, const Fr* const* scalars, const uint32_t* n, const int* c,
                          uint32_t count, void* scratch, size_t scratch_bytes, cudaStream_t st, uint32_t nsrs) {
    if (count == 0) return cudaSuccess;
    BatchLayout L;
    if (!batch_plan(n, c, count, nsrs, L)) return cudaErrorInvalidValue;
    if (L.bytes > scratch_bytes) return cudaErrorInvalidValue;
    char* base = reinterpret_cast<char*>(scratch);
    BatchDesc* d = reinterpret_cast<BatchDesc*>(base + L.off_desc);
    uint32_t* cnt = reinterpret_cast<uint32_t*>(base + L.off_cnt);
    uint32_t* offset = reinterpret_cast<uint32_t*>(base + L.off_offset);
    uint32_t* scan = reinterpret_cast<uint32_t*>(base + L.off_scan);
    uint32_t* entries = reinterpret_cast<uint32_t*>(base + L.off_entries);
    uint32_t* pkey = reinterpret_cast<uint32_t*>(base + L.off_pkey);
    Xyzz* ppt = reinterpret_cast<Xyzz*>(base + L.off_ppt);
    Xyzz* buckets = reinterpret_cast<Xyzz*>(base + L.off_buckets);
    Xyzz* segsum = reinterpret_cast<Xyzz*>(base + L.off_segsum);
    Xyzz* winsum = reinterpret_cast<Xyzz*>(base + L.off_winsum);
    Aff* phi = reinterpret_cast<Aff*>(base + L.off_phi);
    for (uint32_t i0 = 0; i0 < count; i0 += DESC_CHUNK) {
        DescChunk ch;
        ch.count = count - i0 < DESC_CHUNK ? count - i0 : DESC_CHUNK;
        for (uint32_t i = 0; i < ch.count; i++) ch.d[i] = L.desc[i0 + i];
        batch_desc_kernel<<<1, DESC_CHUNK, 0, st>>>(d + i0, ch);
        ZK_CHECK(cudaGetLastError());
    }
    ZK_CHECK(cudaMemsetAsync(cnt, 0, (size_t)L.NB * 4, st));
    unsigned g1 = (L.total + 255) / 256;
    if (g1 > 148u * 64u) g1 = 148u * 64u;
    if (g1 == 0) g1 = 1;
    batch_count_kernel<<<g1, 256, 0, st>>>(d, count, scalars, L.total, cnt);
    ZK_CHECK(cudaGetLastError());
    ZK_CHECK(scan_u32(cnt, offset, L.NB, scan, st));
    batch_scatter_kernel<<<g1, 256, 0, st>>>(d, count, scalars, L.total, nsrs ? nsrs : L.nmax, 2 * nsrs, offset,
                                             cnt, entries);
    ZK_CHECK(cudaGetLastError());
    if (nsrs) {
        // bases is the table: every entry indexes it directly
        ZK_CHECK(msm_accumulate_merge(entries, offset, L.NB, bases, nullptr, 0xffffffffu, L.L, L.nacc, buckets, pkey,
                                      ppt, st));
    } else {
        ZK_CHECK(msm_phi(bases, L.nmax, phi, st));
        ZK_CHECK(
            msm_accumulate_merge(entries, offset, L.NB, bases, phi, L.nmax, L.L, L.nacc, buckets, pkey, ppt, st));
    }
    batch_reduce_kernel<<<(L.red_total + 127) / 128, 128, 0, st>>>(d, count, L.red_total, buckets, offset, segsum);
    ZK_CHECK(cudaGetLastError());
    const uint32_t max_parts = L.maxG < 128 ? 1u : L.maxG / 128u;
    uint32_t bd = 1;
    while (bd < max_parts && bd < 256) bd <<= 1;
    static SmemOptIn opt;
    ZK_CHECK(opt.ensure(batch_window_kernel, 512 * (int)sizeof(Xyzz)));
    batch_window_kernel<<<L.win_total, bd, (size_t)bd * sizeof(Xyzz), st>>>(d, count, segsum, winsum);
    ZK_CHECK(cudaGetLastError());
    batch_final_kernel<<<count, COOP_THREADS, 0, st>>>(d, winsum, out);
    return cudaGetLastError();
}

}  // namespace zk
