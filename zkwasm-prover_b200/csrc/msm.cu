// Pippenger multi-scalar multiplication over BN254 G1 for sm_100a.
//
// Pipeline (all on one stream, no host synchronisation, no allocation):
//   1. count    one thread per scalar: Montgomery -> canonical, signed c-bit
//               digits, atomic histogram of bucket keys (window * B + |d| - 1)
//   2. scan     exclusive prefix sum of the histogram -> bucket offsets
//   3. scatter  digits again; each non-zero digit claims a slot in its bucket
//               and stores (point index | sign << 31): a device counting sort
//   4. accumulate  every thread owns a fixed-length slice of the sorted entries
//               and sums runs of equal key with XYZZ + affine additions; runs
//               that cross a slice boundary are left as head / tail partials
//   5. merge    partials of buckets split across slices: a reduction by key,
//               warp-segmented scans level by level (log-depth in the split)
//   6. reduce   per window, segments of buckets by running sums:
//               sum_b (b+1) B_b = S_seg + lo * T_seg
//   7. window   tree sum of the segment results per window
//   8. final    Horner over windows (c doublings each) -> Jacobian output,
//               four warps evaluating the independent products of each formula
//
// Reference behaviour replaced: cuda/msm.cu:9-467 (unsigned digits, CUB radix
// sort, Jacobian accumulation, one-thread window combine) behind the C entry
// points msm / batch_msm_collect.
#include "common.cuh"
#include "kernels.h"
#include "glv.cuh"
#include "msm_common.cuh"

namespace zk {

static constexpr uint32_t KEY_NONE = 0xffffffffu;

#ifndef ZK_MSM_REDUCE_THREADS
#define ZK_MSM_REDUCE_THREADS 32768
#endif

// Lanes of a warp that hit the same bucket key share one atomic: the lowest
// lane of each group of equal keys adds the group's size.  Skewed digits
// (narrow top windows, repeated or small scalars) would otherwise serialise
// thousands of atomics on a handful of addresses.  Whole warps only.
__device__ __forceinline__ uint32_t key_group(uint32_t key, int& leader, uint32_t& rank) {
    const uint32_t peers = __match_any_sync(0xffffffffu, key);
    const uint32_t lane = threadIdx.x & 31;
    leader = __ffs(peers) - 1;
    rank = __popc(peers & ((1u << lane) - 1u));
    return peers;
}

// histogram of the nonzero signed digits of one scalar magnitude v (whole
// warps: lanes without a scalar pass zero)
// Bucket key of digit d of window w: w * kw + |d| - 1 (kw = 2^(c-1) gives
// every window its own buckets; kw = 0 puts all windows into one set, for
// tables of the bases pre-multiplied by 2^(c w)).
__device__ __forceinline__ void count_digits(const uint32_t v[8], int c, int W, uint32_t kw,
                                             uint32_t* __restrict__ count) {
    uint32_t carry = 0;
    for (int w = 0; w < W; w++) {
        const int d = msm_signed_digit(v, w, c, carry);
        const uint32_t key = d != 0 ? (uint32_t)w * kw + (uint32_t)(d > 0 ? d : -d) - 1 : KEY_NONE;
        int leader;
        uint32_t rank;
        const uint32_t peers = key_group(key, leader, rank);
        if (key != KEY_NONE && rank == 0) atomicAdd(&count[key], (uint32_t)__popc(peers));
    }
}

// entries (point + w pw | sign << 31) of the nonzero digits of one scalar
// magnitude v whose point is `point`, negated when `neg` (pw = 0, or the
// window stride of a table of pre-multiplied bases).  Windows go in groups of
// eight: the digits, then eight independent slot claims (atomics with a
// return value) in flight together, then the stores.
__device__ __forceinline__ void scatter_digits(const uint32_t v[8], int c, int W, uint32_t kw, uint32_t point,
                                               uint32_t pw, bool neg, const uint32_t* __restrict__ offset,
                                               uint32_t* __restrict__ count, uint32_t* __restrict__ entries) {
    const uint32_t nbit = neg ? 0x80000000u : 0u;
    uint32_t carry = 0;
    for (int w0 = 0; w0 < W; w0 += 8) {
        uint32_t key[8], base[8], slot[8];
#pragma unroll
        for (int u = 0; u < 8; u++) {
            key[u] = KEY_NONE;
            if (w0 + u < W) {
                const int d = msm_signed_digit(v, w0 + u, c, carry);
                if (d != 0) {
                    const uint32_t mag = d > 0 ? (uint32_t)d : (uint32_t)(-d);
                    key[u] = ((uint32_t)(w0 + u) * kw + mag - 1) | ((d < 0 ? 0x80000000u : 0u) ^ nbit);
                }
            }
        }
#pragma unroll
        for (int u = 0; u < 8; u++) {
            const uint32_t kk = key[u] == KEY_NONE ? KEY_NONE : key[u] & 0x7fffffffu;
            int leader;
            uint32_t rank;
            const uint32_t peers = key_group(kk, leader, rank);
            if (kk != KEY_NONE) {
                uint32_t top = 0;
                if (rank == 0) top = atomicSub(&count[kk], (uint32_t)__popc(peers));
                top = __shfl_sync(peers, top, leader);
                slot[u] = top - 1u - rank;
                base[u] = offset[kk];
            }
        }
#pragma unroll
        for (int u = 0; u < 8; u++)
            if (key[u] != KEY_NONE)
                entries[base[u] + slot[u]] = (point + (uint32_t)(w0 + u) * pw) | (key[u] & 0x80000000u);
    }
}

// one thread per scalar: Montgomery -> canonical, then the digits of the
// scalar (GLV = false) or of its two GLV halves |k1| (point i) and |k2|
// (point phi_off + i, the image of base i under the endomorphism)
template <bool GLV>
__global__ void msm_count_kernel(const Fr* __restrict__ scalars, uint32_t n, int c, int W, uint32_t kw,
                                 uint32_t* __restrict__ count) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i - (threadIdx.x & 31) >= n) return;  // whole warps past the end
    const Fr k = i < n ? fe_from_mont<FrCfg>(ldg_elem<FrCfg>(scalars + i)) : fe_zero<FrCfg>();
    if (GLV) {
        uint32_t m1[8], m2[8];
        bool n1, n2;
        glv_split(k.v, m1, m2, n1, n2);
        count_digits(m1, c, W, kw, count);
        count_digits(m2, c, W, kw, count);
    } else {
        count_digits(k.v, c, W, kw, count);
    }
}

template <bool GLV>
__global__ void msm_scatter_kernel(const Fr* __restrict__ scalars, uint32_t n, int c, int W, uint32_t kw,
                                   uint32_t pw, uint32_t phi_off, const uint32_t* __restrict__ offset,
                                   uint32_t* __restrict__ count, uint32_t* __restrict__ entries) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i - (threadIdx.x & 31) >= n) return;  // whole warps past the end
    const Fr k = i < n ? fe_from_mont<FrCfg>(ldg_elem<FrCfg>(scalars + i)) : fe_zero<FrCfg>();
    if (GLV) {
        uint32_t m1[8], m2[8];
        bool n1, n2;
        glv_split(k.v, m1, m2, n1, n2);
        scatter_digits(m1, c, W, kw, i, pw, n1, offset, count, entries);
        scatter_digits(m2, c, W, kw, phi_off + i, pw, n2, offset, count, entries);
    } else {
        scatter_digits(k.v, c, W, kw, i, pw, false, offset, count, entries);
    }
}

// phi[i] = (beta x_i, y_i), the endomorphism images of the bases
__global__ void msm_phi_kernel(const Aff* __restrict__ bases, uint32_t n, Aff* __restrict__ phi) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const Aff r = glv_phi(ld_aff(bases + i));
    st_elem<FqCfg>(&phi[i].x, r.x);
    st_elem<FqCfg>(&phi[i].y, r.y);
}

__device__ __forceinline__ void prefetch_l1(const void* p) { asm volatile("prefetch.global.L1 [%0];" ::"l"(p)); }

// largest k in [lo, hi) with off[k] <= pos
__device__ __forceinline__ uint32_t find_bucket(const uint32_t* off, uint32_t lo, uint32_t hi, uint32_t pos) {
    while (hi - lo > 1) {
        uint32_t mid = (lo + hi) >> 1;
        if (off[mid] <= pos)
            lo = mid;
        else
            hi = mid;
    }
    return lo;
}

// point idx of the sorted entries: bases[idx] below nbase, else the
// endomorphism image phi[idx - nbase] (GLV halves)
__device__ __forceinline__ const Aff* entry_point(const Aff* bases, const Aff* phi, uint32_t nbase, uint32_t idx) {
    return idx < nbase ? bases + idx : phi + (idx - nbase);
}

// resident CTAs per SM the accumulation's register budget is sized for: 4
// (126 registers, no spill); on B200, 5 (102 registers, 152 bytes of spill)
// made a 2^22 MSM 2.5% slower and 6 (85 registers) 4% slower
#ifndef ZK_ACC_MIN_BLOCKS
#define ZK_ACC_MIN_BLOCKS 4
#endif

__global__ void __launch_bounds__(128, ZK_ACC_MIN_BLOCKS) msm_accumulate_kernel(const uint32_t* __restrict__ entries,
                                                             const uint32_t* __restrict__ offset, uint32_t NB,
                                                             const Aff* __restrict__ bases,
                                                             const Aff* __restrict__ phi, uint32_t nbase, uint32_t L,
                                                             uint32_t nacc, Xyzz* __restrict__ buckets,
                                                             uint32_t* __restrict__ part_key,
                                                             Xyzz* __restrict__ part_pt) {
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= nacc) return;
    const uint32_t total = offset[NB];
    // L covers the plan's largest entry count; zero digits (sparse or small
    // scalars) leave fewer entries, which are spread over all nacc threads
    // instead of the first total / L of them
    const uint32_t fair = (total + nacc - 1) / nacc;
    L = min(L, max(fair, 8u));
    const uint32_t s = t * L;
    uint32_t head_key = KEY_NONE, tail_key = KEY_NONE;
    if (s < total) {
        const uint32_t e = min(s + L, total);
        uint32_t key = find_bucket(offset, 0, NB, s);
        uint32_t kbeg = offset[key], kend = offset[key + 1];
        // One flat loop over the slice: every lane adds one entry per
        // iteration, so the lanes of a warp stay in step across bucket
        // boundaries (a loop per bucket run would idle the lanes whose runs
        // end first).  The base of the next entry is prefetched into L1 while
        // the current one is added (a register copy would cost occupancy).
        Xyzz acc = xyzz_identity();
        uint32_t ent_next = entries[s];
        prefetch_l1(entry_point(bases, phi, nbase, ent_next & 0x7fffffffu));
        for (uint32_t p = s; p < e; p++) {
            const uint32_t ent = ent_next;
            if (p + 1 < e) {
                ent_next = entries[p + 1];
                prefetch_l1(entry_point(bases, phi, nbase, ent_next & 0x7fffffffu));
            }
            Aff a = ld_aff(entry_point(bases, phi, nbase, ent & 0x7fffffffu));
            if (!aff_is_id(a)) {
                if (ent >> 31) a.y = fe_neg<FqCfg>(a.y);
                acc = xyzz_add_aff_lazy(acc, a.x, a.y);
            }
            if (p + 1 == kend || p + 1 == e) {  // the run of this bucket ends here
                const bool before = kbeg < s;
                const bool after = kend > e;
                acc = xyzz_canon(acc);
                if (!before && !after) {
                    st_xyzz(buckets + key, acc);
                } else if (before) {
                    head_key = key;
                    st_xyzz(part_pt + 2 * t, acc);
                } else {
                    tail_key = key;
                    st_xyzz(part_pt + 2 * t + 1, acc);
                }
                acc = xyzz_identity();
                if (p + 1 < e) {
                    // the next non-empty bucket is usually within a few keys
                    const uint32_t pos = p + 1;
                    uint32_t k = key + 1, tries = 0;
                    while (tries < 8 && offset[k + 1] <= pos) {
                        k++;
                        tries++;
                    }
                    key = (offset[k + 1] > pos) ? k : find_bucket(offset, k, NB, pos);
                    kbeg = offset[key];
                    kend = offset[key + 1];
                }
            }
        }
    }
    part_key[2 * t] = head_key;
    part_key[2 * t + 1] = tail_key;
}

// ---------------------------------------------------------------- merge
// Buckets split across accumulation slices are summed from the partials by a
// reduction by key.  Level 0 has one item per slice t: key part_key[2t] (the
// bucket its slice starts inside, or none) and the head partial, to which the
// tail partial of slice t-1 is added (a tail is always continued by the next
// slice's head).  Keys are sorted and an empty item never sits inside a run of
// one key, so each warp does a segmented inclusive scan of 32 items with
// shuffles; a run that starts and ends inside the warp is a finished bucket,
// and the run that enters the warp from the left (slot 2w) or leaves it to the
// right (slot 2w+1) is passed to the next level, which repeats the same on
// 2 ceil(M / 32) items.  A bucket over m slices therefore costs O(log m)
// dependent additions instead of m.

__device__ __forceinline__ Xyzz shfl_up_xyzz(const Xyzz& p, unsigned d) {
    Xyzz r;
#pragma unroll
    for (int i = 0; i < 8; i++) {
        r.x.v[i] = __shfl_up_sync(0xffffffffu, p.x.v[i], d);
        r.y.v[i] = __shfl_up_sync(0xffffffffu, p.y.v[i], d);
        r.zz.v[i] = __shfl_up_sync(0xffffffffu, p.zz.v[i], d);
        r.zzz.v[i] = __shfl_up_sync(0xffffffffu, p.zzz.v[i], d);
    }
    return r;
}

template <bool LEVEL0>
__device__ __forceinline__ uint32_t merge_key(const uint32_t* ikey, uint32_t i) {
    return LEVEL0 ? ikey[2 * i] : ikey[i];
}

template <bool LEVEL0>
__global__ void __launch_bounds__(128) msm_merge_level_kernel(const uint32_t* __restrict__ ikey,
                                                              const Xyzz* __restrict__ ipt, uint32_t M,
                                                              uint32_t* __restrict__ okey, Xyzz* __restrict__ opt,
                                                              Xyzz* __restrict__ buckets) {
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t lane = threadIdx.x & 31;
    const uint32_t base = t - lane;
    if (base >= M) return;  // whole warps only
    uint32_t k = t < M ? merge_key<LEVEL0>(ikey, t) : KEY_NONE;
    Xyzz P = xyzz_identity();
    if (k != KEY_NONE) {
        P = ld_xyzz(ipt + (LEVEL0 ? 2 * t : t));
        if (LEVEL0 && t > 0 && ikey[2 * t - 1] == k) P = xyzz_add(ld_xyzz(ipt + 2 * t - 1), P);
    }
    for (unsigned d = 1; d < 32; d <<= 1) {
        const uint32_t kj = __shfl_up_sync(0xffffffffu, k, d);
        const Xyzz Q = shfl_up_xyzz(P, d);
        if (lane >= d && kj == k && k != KEY_NONE) P = xyzz_add(Q, P);
    }
    const uint32_t last = (M - base < 32u ? M - base : 32u) - 1;  // last valid lane
    const uint32_t prev = base > 0 ? merge_key<LEVEL0>(ikey, base - 1) : KEY_NONE;
    const uint32_t next = base + 32 < M ? merge_key<LEVEL0>(ikey, base + 32) : KEY_NONE;
    const uint32_t k0 = __shfl_sync(0xffffffffu, k, 0);
    const uint32_t kl = __shfl_sync(0xffffffffu, k, last);
    const uint32_t kn = __shfl_down_sync(0xffffffffu, k, 1);
    const bool from_left = k0 != KEY_NONE && prev == k0;  // the first run started in an earlier warp
    const bool to_right = kl != KEY_NONE && next == kl;   // the last run continues in a later warp
    const uint32_t w2 = 2 * (base >> 5);
    const bool run_end = lane == last || (lane < last && kn != k);
    if (lane <= last && run_end && k != KEY_NONE) {
        const bool first = from_left && k == k0, lastrun = to_right && k == kl;
        if (first && lastrun) {  // the run spans the whole warp
            okey[w2] = k;
            st_xyzz(opt + w2, xyzz_identity());
            okey[w2 + 1] = k;
            st_xyzz(opt + w2 + 1, P);
        } else if (first) {
            okey[w2] = k;
            st_xyzz(opt + w2, P);
        } else if (lastrun) {
            okey[w2 + 1] = k;
            st_xyzz(opt + w2 + 1, P);
        } else {
            st_xyzz(buckets + k, P);
        }
    }
    if (lane == 0 && okey) {
        if (!from_left) okey[w2] = KEY_NONE;
        if (!to_right) okey[w2 + 1] = KEY_NONE;
    }
}

// items of the merge levels above level 0 (stored after the 2 * nacc partials)
size_t msm_merge_extra(uint32_t nacc) {
    size_t total = 0;
    for (uint32_t M = nacc; M > 32;) {
        M = 2 * ((M + 31) / 32);
        total += M;
    }
    return total;
}

static cudaError_t msm_merge(uint32_t* part_key, Xyzz* part_pt, uint32_t nacc, Xyzz* buckets, cudaStream_t st) {
    const uint32_t* ik = part_key;
    const Xyzz* ip = part_pt;
    uint32_t* ok = part_key + 2 * (size_t)nacc;
    Xyzz* op = part_pt + 2 * (size_t)nacc;
    uint32_t M = nacc;
    for (bool level0 = true;; level0 = false) {
        const bool top = M <= 32;  // one warp: every run ends inside it
        const uint32_t blocks = (M + 127) / 128;
        if (level0)
            msm_merge_level_kernel<true><<<blocks, 128, 0, st>>>(ik, ip, M, top ? nullptr : ok, top ? nullptr : op,
                                                                 buckets);
        else
            msm_merge_level_kernel<false><<<blocks, 128, 0, st>>>(ik, ip, M, top ? nullptr : ok,
                                                                  top ? nullptr : op, buckets);
        ZK_CHECK(cudaGetLastError());
        if (top) break;
        const uint32_t M2 = 2 * ((M + 31) / 32);
        ik = ok;
        ip = op;
        ok += M2;
        op += M2;
        M = M2;
    }
    return cudaSuccess;
}

// Thread t = w G + g sums segment g of window w by running sums; then each
// group of GS = min(G, 128) consecutive threads (one window) adds its results
// as a tree, and the group's sum goes to segsum[t / GS], so the window
// kernel is left with G / GS partial sums per window.
__global__ void __launch_bounds__(128) msm_reduce_kernel(const Xyzz* __restrict__ buckets,
                                                         const uint32_t* __restrict__ offset, int W, uint32_t B,
                                                         uint32_t seg, uint32_t G, Xyzz* __restrict__ segsum) {
    __shared__ Xyzz sm[128];
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    Xyzz S = xyzz_identity();
    if (t < (uint32_t)W * G) {
        const uint32_t w = t / G, g = t % G;
        const uint32_t lo = g * seg;
        Xyzz T = xyzz_identity();
        for (uint32_t j = 0; j < seg; j++) {
            const uint32_t b = lo + seg - 1 - j;
            const uint32_t key = w * B + b;
            if (offset[key + 1] != offset[key]) T = xyzz_add(T, ld_xyzz(buckets + key));
            S = xyzz_add(S, T);
        }
        if (lo) S = xyzz_add(S, xyzz_mul_u32(T, lo));
    }
    const uint32_t GS = G < 128 ? G : 128;
    const uint32_t k = threadIdx.x;
    sm[k] = S;
    __syncthreads();
    for (uint32_t h = GS >> 1; h > 0; h >>= 1) {
        if ((k & (GS - 1)) < h) sm[k] = xyzz_add(sm[k], sm[k + h]);
        __syncthreads();
    }
    if ((k & (GS - 1)) == 0 && t < (uint32_t)W * G) st_xyzz(segsum + t / GS, sm[k]);
}

// one CTA per window; blockDim (a power of two, <= G) threads first add
// G / blockDim segment results each, then reduce as a tree
__global__ void __launch_bounds__(256) msm_window_kernel(const Xyzz* __restrict__ segsum, uint32_t G, Xyzz* __restrict__ winsum) {
    extern __shared__ uint4 smem_u4[];
    Xyzz* sm = reinterpret_cast<Xyzz*>(smem_u4);
    const uint32_t w = blockIdx.x, i = threadIdx.x, T = blockDim.x;
    Xyzz acc = ld_xyzz(segsum + (size_t)w * G + i);
    for (uint32_t k = i + T; k < G; k += T) acc = xyzz_add(acc, ld_xyzz(segsum + (size_t)w * G + k));
    sm[i] = acc;
    __syncthreads();
    for (uint32_t h = T >> 1; h > 0; h >>= 1) {
        if (i < h) sm[i] = xyzz_add(sm[i], sm[i + h]);
        __syncthreads();
    }
    if (i == 0) st_xyzz(winsum + w, sm[0]);
}

// one CTA of COOP_THREADS threads
__global__ void __launch_bounds__(COOP_THREADS) msm_final_kernel(const Xyzz* __restrict__ winsum, int W, int c,
                                                                  Jac* __restrict__ out) {
    __shared__ Fq buf[8];
    const Jac j = coop_horner(buf, winsum, W, c);
    if (threadIdx.x == 0) {
        st_elem<FqCfg>(&out->x, j.x);
        st_elem<FqCfg>(&out->y, j.y);
        st_elem<FqCfg>(&out->z, j.z);
    }
}

// windows of c bits for 254-bit scalars, or for the < 2^127 GLV halves
static int windows_for(int c, bool glv) { return glv ? (128 + c - 1) / c : (254 + c - 1) / c; }

// ------------------------------------------------------------ base tables
// For bases that stay resident across many MSMs (the SRS of a proving key),
// entry j 2 nsrs + i = [2^(c j)] base_i and entry j 2 nsrs + nsrs + i its
// endomorphism image.  Digit d of window j of a scalar then adds table entry
// j directly into the one bucket set of |d|: the sum over windows needs no
// doublings, and the bucket reduction runs once instead of once per window.

__device__ __forceinline__ void st_aff(Aff* p, const Aff& a) {
    st_elem<FqCfg>(&p->x, a.x);
    st_elem<FqCfg>(&p->y, a.y);
}

// One thread per base: W windows of c doublings each.  The W - 1 affine
// conversions share one field inversion (Montgomery's trick over the base's
// own windows): window j's XYZZ form is parked in its two table slots (X, Y in
// the base's slot, ZZ, ZZZ in the image's), the product of the ZZ ZZZ is
// inverted once, and the windows are converted from the last back.  An
// inversion is about 36 us of one thread, so W - 1 of them dominated the build.
__global__ void __launch_bounds__(128) msm_table_kernel(Aff* __restrict__ table, const Aff* __restrict__ bases,
                                                        uint32_t nsrs, int c, int W) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nsrs) return;
    const size_t stride = 2 * (size_t)nsrs;
    Aff a = ld_aff(bases + i);
    st_aff(table + i, a);
    st_aff(table + nsrs + i, glv_phi(a));
    Xyzz acc = xyzz_from_aff(a);
    Fq pre[32];  // pre[j] = product of d_1 .. d_{j-1}, d_j = ZZ_j ZZZ_j (1 for the identity); W <= 32
    Fq run = fe_one<FqCfg>();
    for (int j = 1; j < W; j++) {
        for (int k = 0; k < c; k++) acc = xyzz_dbl(acc);
        Aff* slot = table + j * stride + i;
        Aff* islot = table + j * stride + nsrs + i;
        st_elem<FqCfg>(&slot->x, acc.x);
        st_elem<FqCfg>(&slot->y, acc.y);
        st_elem<FqCfg>(&islot->x, acc.zz);
        st_elem<FqCfg>(&islot->y, acc.zzz);
        pre[j] = run;
        if (!xyzz_is_id(acc)) run = cmul(run, cmul(acc.zz, acc.zzz));
    }
    Fq inv = fe_inv<FqCfg>(run);  // 1 / (d_1 ... d_{W-1})
    for (int j = W - 1; j >= 1; j--) {
        Aff* slot = table + j * stride + i;
        Aff* islot = table + j * stride + nsrs + i;
        Xyzz p;
        p.x = ld_elem<FqCfg>(&slot->x);
        p.y = ld_elem<FqCfg>(&slot->y);
        p.zz = ld_elem<FqCfg>(&islot->x);
        p.zzz = ld_elem<FqCfg>(&islot->y);
        Aff r;
        if (xyzz_is_id(p)) {
            r.x = fe_zero<FqCfg>();
            r.y = fe_zero<FqCfg>();
        } else {
            const Fq dj = cmul(p.zz, p.zzz);
            const Fq inv_dj = cmul(inv, pre[j]);  // 1 / d_j
            inv = cmul(inv, dj);                  // 1 / (d_1 ... d_{j-1})
            r.x = cmul(p.x, cmul(inv_dj, p.zzz));  // X / ZZ
            r.y = cmul(p.y, cmul(inv_dj, p.zz));   // Y / ZZZ
        }
        st_aff(slot, r);
        st_aff(islot, glv_phi(r));
    }
}

cudaError_t msm_table_build(Aff* table, const Aff* bases, uint32_t nsrs, int c, cudaStream_t st) {
    if (nsrs == 0) return cudaSuccess;
    msm_table_kernel<<<(nsrs + 127) / 128, 128, 0, st>>>(table, bases, nsrs, c, windows_for(c, true));
    return cudaGetLastError();
}

// ------------------------------------------------------------------ planning


static size_t align_up(size_t x, size_t a) { return (x + a - 1) / a * a; }

static int pick_c(uint32_t n, bool glv) {
    int best = 4;
    double best_cost = 1e300;
    for (int c = 4; c <= 20; c++) {
        const double W = windows_for(c, glv);
        const double pts = glv ? 2.0 * n : (double)n;
        const double cost = 10.0 * pts * W + 28.0 * W * (double)(1u << (c - 1)) + 9.0 * 150.0 * (W - 1) * c;
        if (cost < best_cost) {
            best_cost = cost;
            best = c;
        }
    }
    return best;
}

// over a table: every window's digits go into one bucket set, so the
// reduction is paid once and there is no Horner chain.  A bucket costs about
// five sorted entries (its reduction and the shorter runs of a wider key
// space), fitted to B200 timings at 2^14..2^22 points.
static int pick_c_table(uint32_t n) {
    int best = 4;
    double best_cost = 1e300;
    for (int c = 4; c <= 22; c++) {
        const double cost = 2.0 * n * windows_for(c, true) + 5.0 * (double)(1u << (c - 1));
        if (cost < best_cost) {
            best_cost = cost;
            best = c;
        }
    }
    return best;
}

int msm_table_default_window(uint32_t n) { return pick_c_table(n); }

// one width for a batch over one table: each MSM has its own bucket set, and
// with many sets in one pipeline a bucket costs about 25 sorted entries (their
// reductions share one thread budget), fitted to 256 MSMs of 2^14..2^22
// points on B200 (c = 13..17: 456, 450, 431, 413, 429 ms; 19: 525 ms)
int msm_batch_table_default_window(const uint32_t* n, uint32_t count) {
    double pts = 0;
    for (uint32_t i = 0; i < count; i++) pts += 2.0 * n[i];
    const double per_bucket = count > 1 ? 25.0 : 5.0;
    int best = 4;
    double best_cost = 1e300;
    for (int c = 4; c <= 22; c++) {
        const double cost = pts * windows_for(c, true) + per_bucket * count * (double)(1u << (c - 1));
        if (cost < best_cost) {
            best_cost = cost;
            best = c;
        }
    }
    return best;
}

static void plan_finish(MsmPlan& p) {
    p.B = 1u << (p.c - 1);
    p.NB = (uint32_t)p.Wb * p.B;
    const uint64_t max_entries = msm_entry_count(p);
    const uint64_t target_threads = 148ull * 4 * 128;
    uint64_t L = (max_entries + target_threads - 1) / target_threads;
    if (L < 8) L = 8;
    p.L = (uint32_t)L;
    p.nacc = (uint32_t)((max_entries + L - 1) / L);
    if (p.nacc == 0) p.nacc = 1;
    // up to ZK_MSM_REDUCE_THREADS reduction threads in total (the running-sum
    // segments are latency bound, so they need many threads), at most 4096 per
    // window when there is one bucket set per window
    const uint32_t gcap = p.Wb == 1 ? ZK_MSM_REDUCE_THREADS : 4096;
    uint32_t G = 1;
    while (G < gcap && (uint64_t)G * 2 * p.Wb <= ZK_MSM_REDUCE_THREADS && G * 2 <= p.B) G *= 2;
    p.G = G;
    p.seg = p.B / G;
}

MsmPlan msm_make_plan(uint32_t n, int c, bool glv) {
    MsmPlan p;
    p.n = n;
    p.glv = glv ? 1 : 0;
    p.c = (c >= 4 && c <= 22) ? c : pick_c(n, glv);
    p.W = windows_for(p.c, glv);
    p.Wb = p.W;
    p.nsrs = 0;
    plan_finish(p);
    return p;
}

MsmPlan msm_make_table_plan(uint32_t n, int c, uint32_t nsrs) {
    MsmPlan p;
    p.n = n;
    p.glv = 1;
    p.c = (c >= 4 && c <= 22) ? c : pick_c_table(n);
    p.W = windows_for(p.c, true);
    p.Wb = 1;
    p.nsrs = nsrs;
    plan_finish(p);
    return p;
}

size_t msm_table_points(uint32_t nsrs, int c) {
    if (c < 4 || c > 22) return 0;
    return (size_t)windows_for(c, true) * 2 * nsrs;
}

size_t msm_u32_words(const MsmPlan& p) {
    size_t w = 0;
    w += align_up(p.NB, 64);
    w += align_up(p.NB + 1, 64);
    w += align_up(scan_tmp_words(p.NB), 64);
    w += align_up(msm_entry_count(p), 64);
    w += align_up((size_t)2 * p.nacc + msm_merge_extra(p.nacc), 64);
    return w;
}

size_t msm_point_count(const MsmPlan& p) {
    return (size_t)2 * p.nacc + msm_merge_extra(p.nacc) + p.NB + (size_t)p.Wb * p.G + p.Wb;
}

// endomorphism images are made per call unless a table holds them
static bool needs_phi(const MsmPlan& p) { return p.glv && !p.nsrs; }

size_t msm_scratch_bytes(const MsmPlan& p) {
    return align_up(msm_u32_words(p) * 4, 256) + msm_point_count(p) * sizeof(Xyzz) +
           (needs_phi(p) ? (size_t)p.n * sizeof(Aff) : 0);
}

void msm_layout_split(const MsmPlan& p, uint32_t* words, Xyzz* points, MsmScratch* s) {
    uint32_t* w = words;
    s->count = w;
    w += align_up(p.NB, 64);
    s->offset = w;
    w += align_up(p.NB + 1, 64);
    s->scan_tmp = w;
    w += align_up(scan_tmp_words(p.NB), 64);
    s->entries = w;
    w += align_up(msm_entry_count(p), 64);
    s->part_key = w;
    Xyzz* q = points;
    s->part_pt = q;
    q += (size_t)2 * p.nacc + msm_merge_extra(p.nacc);
    s->buckets = q;
    q += p.NB;
    s->segsum = q;
    q += (size_t)p.Wb * p.G;
    s->winsum = q;
    q += p.Wb;
    s->phi = needs_phi(p) ? reinterpret_cast<Aff*>(q) : nullptr;
}

bool msm_layout_arenas(const MsmPlan& p, void* const* arena, const size_t* arena_bytes, int n_arenas,
                       MsmScratch* s, int winsum_arena) {
    // the plan's buffers, largest first, each into the first arena with room
    const size_t parts = (size_t)2 * p.nacc + msm_merge_extra(p.nacc);
    void** slot[10] = {reinterpret_cast<void**>(&s->count),    reinterpret_cast<void**>(&s->offset),
                       reinterpret_cast<void**>(&s->scan_tmp), reinterpret_cast<void**>(&s->entries),
                       reinterpret_cast<void**>(&s->part_key), reinterpret_cast<void**>(&s->part_pt),
                       reinterpret_cast<void**>(&s->buckets),  reinterpret_cast<void**>(&s->segsum),
                       reinterpret_cast<void**>(&s->winsum),   reinterpret_cast<void**>(&s->phi)};
    size_t bytes[10] = {(size_t)p.NB * 4,
                        ((size_t)p.NB + 1) * 4,
                        scan_tmp_words(p.NB) * 4,
                        msm_entry_count(p) * 4,
                        parts * 4,
                        parts * sizeof(Xyzz),
                        (size_t)p.NB * sizeof(Xyzz),
                        (size_t)p.Wb * p.G * sizeof(Xyzz),
                        (size_t)p.Wb * sizeof(Xyzz),
                        needs_phi(p) ? (size_t)p.n * sizeof(Aff) : 0};
    int order[10];
    for (int i = 0; i < 10; i++) order[i] = i;
    for (int i = 1; i < 10; i++)
        for (int j = i; j > 0 && bytes[order[j]] > bytes[order[j - 1]]; j--) {
            const int t = order[j];
            order[j] = order[j - 1];
            order[j - 1] = t;
        }
    size_t used[8] = {};
    if (n_arenas > 8) n_arenas = 8;
    for (int k = 0; k < 10; k++) {
        const int b = order[k];
        int a = 0;
        for (; a < n_arenas; a++) {
            if (b == 8 && winsum_arena >= 0 && a != winsum_arena) continue;
            const uintptr_t base = reinterpret_cast<uintptr_t>(arena[a]);
            const size_t start = align_up(base + used[a], 256) - base;
            if (start + bytes[b] <= arena_bytes[a]) {
                *slot[b] = reinterpret_cast<char*>(arena[a]) + start;
                used[a] = start + bytes[b];
                break;
            }
        }
        if (a == n_arenas) return false;
    }
    if (!needs_phi(p)) s->phi = nullptr;
    return true;
}

void msm_layout(const MsmPlan& p, void* base, MsmScratch* s) {
    uint32_t* words = reinterpret_cast<uint32_t*>(base);
    Xyzz* pts = reinterpret_cast<Xyzz*>(reinterpret_cast<char*>(base) + align_up(msm_u32_words(p) * 4, 256));
    msm_layout_split(p, words, pts, s);
}

// stages 4 and 5 over any sorted key space (shared by the batched MSM)
cudaError_t msm_phi(const Aff* bases, uint32_t n, Aff* phi, cudaStream_t st) {
    if (n == 0) return cudaSuccess;
    msm_phi_kernel<<<(n + 255) / 256, 256, 0, st>>>(bases, n, phi);
    return cudaGetLastError();
}

cudaError_t msm_accumulate_merge(const uint32_t* entries, const uint32_t* offset, uint32_t NB, const Aff* bases,
                                 const Aff* phi, uint32_t nbase, uint32_t L, uint32_t nacc, Xyzz* buckets,
                                 uint32_t* part_key, Xyzz* part_pt, cudaStream_t st) {
    msm_accumulate_kernel<<<(nacc + 127) / 128, 128, 0, st>>>(entries, offset, NB, bases, phi, nbase, L,
                                                              nacc, buckets, part_key,
                                                              part_pt);
    ZK_CHECK(cudaGetLastError());
    return msm_merge(part_key, part_pt, nacc, buckets, st);
}

// ------------------------------------------------------------ parked finals
// The reference host runs msm() once per column and then batch_msm_collect
// over all of them.  msm() can stop after the window sums and leave a note
// of where they are; batch_msm_collect then runs every MSM's final Horner
// chain at once, one CTA each, instead of one latency-bound chain per call.

struct MsmParked {
    uint32_t magic, W, c, pad;
    const Xyzz* winsum;  // device address of the window sums
};
static constexpr uint32_t PARK_MAGIC = 0x4d534d50u;

__global__ void msm_park_kernel(MsmParked* note, uint32_t W, uint32_t c, const Xyzz* winsum) {
    note->magic = PARK_MAGIC;
    note->W = W;
    note->c = c;
    note->pad = 0;
    note->winsum = winsum;
}

// one CTA per region: regions[i] + note_off holds the note, the Jacobian
// result goes to regions[i][0]
__global__ void __launch_bounds__(COOP_THREADS) msm_collect_kernel(char* const* regions, uint32_t note_off) {
    __shared__ Fq buf[8];
    char* base = regions[blockIdx.x];
    const MsmParked note = *reinterpret_cast<const MsmParked*>(base + note_off);
    if (note.magic != PARK_MAGIC) return;  // uniform: no msm() result parked here
    const Jac j = coop_horner(buf, note.winsum, (int)note.W, (int)note.c);
    if (threadIdx.x == 0) {
        Jac* out = reinterpret_cast<Jac*>(base);
        st_elem<FqCfg>(&out->x, j.x);
        st_elem<FqCfg>(&out->y, j.y);
        st_elem<FqCfg>(&out->z, j.z);
    }
}

cudaError_t msm_collect(char* const* regions, uint32_t count, uint32_t note_off, cudaStream_t st) {
    if (count == 0) return cudaSuccess;
    msm_collect_kernel<<<count, COOP_THREADS, 0, st>>>(regions, note_off);
    return cudaGetLastError();
}

cudaError_t msm_run(Jac* out, const Aff* bases, const Fr* scalars, const MsmPlan& p, const MsmScratch& s,
                    cudaStream_t st, void* park_note) {
    if (p.n == 0) {
        // empty sum: the identity
        if (park_note) {
            msm_park_kernel<<<1, 1, 0, st>>>(reinterpret_cast<MsmParked*>(park_note), 0, (uint32_t)p.c, nullptr);
            return cudaGetLastError();
        }
        msm_final_kernel<<<1, COOP_THREADS, 0, st>>>(nullptr, 0, p.c, out);
        return cudaGetLastError();
    }
    const uint32_t tb = 256;
    const uint32_t nblk = (p.n + tb - 1) / tb;
    // over a table all windows share one bucket set and entry j 2 nsrs + i
    // is base i times 2^(c j)
    const uint32_t kw = p.nsrs ? 0u : p.B;
    const uint32_t pw = p.nsrs ? 2 * p.nsrs : 0u;
    const uint32_t phi_off = p.nsrs ? p.nsrs : p.n;
    ZK_CHECK(cudaMemsetAsync(s.count, 0, sizeof(uint32_t) * p.NB, st));
    if (p.glv)
        msm_count_kernel<true><<<nblk, tb, 0, st>>>(scalars, p.n, p.c, p.W, kw, s.count);
    else
        msm_count_kernel<false><<<nblk, tb, 0, st>>>(scalars, p.n, p.c, p.W, kw, s.count);
    ZK_CHECK(cudaGetLastError());
    ZK_CHECK(scan_u32(s.count, s.offset, p.NB, s.scan_tmp, st));
    if (p.glv) {
        msm_scatter_kernel<true><<<nblk, tb, 0, st>>>(scalars, p.n, p.c, p.W, kw, pw, phi_off, s.offset, s.count,
                                                      s.entries);
        ZK_CHECK(cudaGetLastError());
        if (needs_phi(p)) msm_phi_kernel<<<nblk, tb, 0, st>>>(bases, p.n, s.phi);
    } else {
        msm_scatter_kernel<false><<<nblk, tb, 0, st>>>(scalars, p.n, p.c, p.W, kw, pw, phi_off, s.offset, s.count,
                                                       s.entries);
    }
    ZK_CHECK(cudaGetLastError());
    msm_accumulate_kernel<<<(p.nacc + 127) / 128, 128, 0, st>>>(s.entries, s.offset, p.NB, bases, s.phi,
                                                                needs_phi(p) ? p.n : 0xffffffffu, p.L, p.nacc,
                                                                s.buckets, s.part_key, s.part_pt);
    ZK_CHECK(cudaGetLastError());
    ZK_CHECK(msm_merge(s.part_key, s.part_pt, p.nacc, s.buckets, st));
    const uint32_t nred = (uint32_t)p.Wb * p.G;
    msm_reduce_kernel<<<(nred + 127) / 128, 128, 0, st>>>(s.buckets, s.offset, p.Wb, p.B, p.seg, p.G, s.segsum);
    ZK_CHECK(cudaGetLastError());
    // partial sums per window left by the reduce kernel's group trees
    const uint32_t parts = p.G < 128 ? 1u : p.G / 128u;
    const uint32_t wt = parts < 256 ? parts : 256;
    msm_window_kernel<<<p.Wb, wt, (size_t)wt * sizeof(Xyzz), st>>>(s.segsum, parts, s.winsum);
    ZK_CHECK(cudaGetLastError());
    if (park_note) {
        msm_park_kernel<<<1, 1, 0, st>>>(reinterpret_cast<MsmParked*>(park_note), (uint32_t)p.Wb, (uint32_t)p.c,
                                          s.winsum);
        return cudaGetLastError();
    }
    msm_final_kernel<<<1, COOP_THREADS, 0, st>>>(s.winsum, p.Wb, p.c, out);
    return cudaGetLastError();
}

}  // namespace zk
