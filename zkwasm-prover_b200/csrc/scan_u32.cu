// Exclusive prefix sum of u32 counts (bucket offsets for the MSM counting sort).
// Three launches: per-block scan of 4096 values, scan of the block totals,
// and the add-back.
#include "common.cuh"
#include "kernels.h"

namespace zk {

static constexpr int SCAN_T = 1024;
static constexpr int SCAN_V = 4;
static constexpr int SCAN_BLK = SCAN_T * SCAN_V;

size_t scan_tmp_words(uint32_t n) { return (n + SCAN_BLK - 1) / SCAN_BLK + 1; }

// block-wide exclusive scan of one value per thread; returns the block total
__device__ __forceinline__ uint32_t block_excl_scan(uint32_t v, uint32_t* warp_tot, uint32_t& total) {
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    uint32_t x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) warp_tot[wid] = x;
    __syncthreads();
    if (wid == 0) {
        uint32_t w = (lane < (int)(blockDim.x >> 5)) ? warp_tot[lane] : 0;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            uint32_t y = __shfl_up_sync(0xffffffffu, w, o);
            if (lane >= o) w += y;
        }
        warp_tot[lane] = w;  // inclusive
    }
    __syncthreads();
    total = warp_tot[(blockDim.x >> 5) - 1];
    uint32_t before = wid ? warp_tot[wid - 1] : 0;
    uint32_t r = before + x - v;
    __syncthreads();
    return r;
}

__global__ void __launch_bounds__(SCAN_T) scan_block_kernel(const uint32_t* in, uint32_t* out, uint32_t n,
                                                            uint32_t* bsum) {
    __shared__ uint32_t wt[32];
    const size_t base = (size_t)blockIdx.x * SCAN_BLK + (size_t)threadIdx.x * SCAN_V;
    uint32_t v[SCAN_V];
    uint32_t s = 0;
#pragma unroll
    for (int i = 0; i < SCAN_V; i++) {
        v[i] = (base + i < n) ? in[base + i] : 0;
        s += v[i];
    }
    uint32_t tot;
    uint32_t pre = block_excl_scan(s, wt, tot);
#pragma unroll
    for (int i = 0; i < SCAN_V; i++) {
        if (base + i < n) out[base + i] = pre;
        pre += v[i];
    }
    if (threadIdx.x == 0) bsum[blockIdx.x] = tot;
}

// one CTA scans the block totals in chunks of SCAN_BLK, carrying the sum
__global__ void __launch_bounds__(SCAN_T) scan_top_kernel(uint32_t* bsum, uint32_t nb, uint32_t* total_out) {
    __shared__ uint32_t wt[32];
    uint32_t carry = 0;
    for (uint32_t chunk = 0; chunk < nb; chunk += SCAN_BLK) {
        const uint32_t base = chunk + threadIdx.x * SCAN_V;
        uint32_t v[SCAN_V];
        uint32_t s = 0;
#pragma unroll
        for (int i = 0; i < SCAN_V; i++) {
            v[i] = (base + i < nb) ? bsum[base + i] : 0;
            s += v[i];
        }
        uint32_t tot;
        uint32_t pre = carry + block_excl_scan(s, wt, tot);
#pragma unroll
        for (int i = 0; i < SCAN_V; i++) {
            if (base + i < nb) bsum[base + i] = pre;
            pre += v[i];
        }
        carry += tot;
    }
    if (threadIdx.x == 0) *total_out = carry;
}

__global__ void __launch_bounds__(SCAN_T) scan_add_kernel(uint32_t* out, uint32_t n, const uint32_t* bsum) {
    const uint32_t add = bsum[blockIdx.x];
    if (add == 0) return;
    const size_t base = (size_t)blockIdx.x * SCAN_BLK + (size_t)threadIdx.x * SCAN_V;
#pragma unroll
    for (int i = 0; i < SCAN_V; i++)
        if (base + i < n) out[base + i] += add;
}

cudaError_t scan_u32(const uint32_t* in, uint32_t* out, uint32_t n, uint32_t* tmp, cudaStream_t s) {
    const uint32_t nb = (n + SCAN_BLK - 1) / SCAN_BLK;
    if (nb == 0) return cudaMemsetAsync(out, 0, sizeof(uint32_t), s);
    scan_block_kernel<<<nb, SCAN_T, 0, s>>>(in, out, n, tmp);
    scan_top_kernel<<<1, SCAN_T, 0, s>>>(tmp, nb, out + n);
    if (nb > 1) scan_add_kernel<<<nb, SCAN_T, 0, s>>>(out, n, tmp);
    return cudaGetLastError();
}

}  // namespace zk
