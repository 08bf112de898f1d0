// Lookup multiplicities without sorting, and polynomial evaluation.
//
// prepare_table_lookup / calc_m (reference: cuda/bn254.cu:1637-1912, which
// radix-sorts the table by its low k+2 bits and then radix-sorts and merges
// the matches): here the usable table rows go into an open-addressing hash
// table keyed by the full 32-byte value.  Among equal values the slot keeps
// the largest row index, which is the row the reference's downward scan over
// the stably sorted table credits.  calc_m then probes once per input row and
// counts hits per table row; m[row] += count (Montgomery form), so m
// accumulates over the inputs of a lookup exactly as in the reference.
// Inputs absent from the table are skipped (the reference asserts).
//
// poly_eval (reference: cuda/bn254.cu:238-258, 1608-1634): levels of Horner
// over chunks of 16 coefficients, using the table x^(2^d); level values stay
// in place at stride 16^level, and the value lands in res[0].
#include "common.cuh"
#include "kernels.h"

namespace zk {

static constexpr uint32_t SLOT_EMPTY = 0xffffffffu;

__device__ __forceinline__ uint32_t hash_fr(const Fr& v) {
    uint32_t h = v.v[0] * 0x9e3779b1u ^ v.v[1] * 0x85ebca77u ^ v.v[2] * 0xc2b2ae3du ^ v.v[3];
    h ^= h >> 15;
    h *= 0x2c1b3c6du;
    h ^= h >> 12;
    return h;
}

__global__ void table_insert_kernel(const Fr* table, uint32_t usable, uint32_t* slots, uint32_t mask) {
    for (uint32_t r = blockIdx.x * blockDim.x + threadIdx.x; r < usable; r += gridDim.x * blockDim.x) {
        const Fr v = ld_elem<FrCfg>(table + r);
        uint32_t h = hash_fr(v) & mask;
        for (uint32_t probe = 0; probe <= mask; probe++) {
            uint32_t cur = atomicCAS(&slots[h], SLOT_EMPTY, r);
            if (cur == SLOT_EMPTY) break;
            if (fe_eq<FrCfg>(ld_elem<FrCfg>(table + cur), v)) {
                atomicMax(&slots[h], r);
                break;
            }
            h = (h + 1) & mask;
        }
    }
}

__global__ void input_count_kernel(const Fr* table, const Fr* input, uint32_t usable, const uint32_t* slots,
                                   uint32_t mask, uint32_t* cnt) {
    for (uint32_t r = blockIdx.x * blockDim.x + threadIdx.x; r < usable; r += gridDim.x * blockDim.x) {
        const Fr v = ld_elem<FrCfg>(input + r);
        uint32_t h = hash_fr(v) & mask;
        for (uint32_t probe = 0; probe <= mask; probe++) {
            const uint32_t cur = slots[h];
            if (cur == SLOT_EMPTY) break;
            if (fe_eq<FrCfg>(ld_elem<FrCfg>(table + cur), v)) {
                atomicAdd(&cnt[cur], 1u);
                break;
            }
            h = (h + 1) & mask;
        }
    }
}

__global__ void add_counts_kernel(Fr* m, const uint32_t* cnt, uint32_t n) {
    for (uint32_t r = blockIdx.x * blockDim.x + threadIdx.x; r < n; r += gridDim.x * blockDim.x) {
        const uint32_t c = cnt[r];
        if (c == 0) continue;
        Fr x = fe_zero<FrCfg>();
        x.v[0] = c;
        x = fe_to_mont<FrCfg>(x);
        st_elem<FrCfg>(m + r, fe_add<FrCfg>(ld_elem<FrCfg>(m + r), x));
    }
}

static unsigned grid_rows(uint32_t n) {
    unsigned nb = (n + 255) / 256;
    if (nb > 148 * 32) nb = 148 * 32;
    return nb ? nb : 1;
}

cudaError_t lookup_table_build(const Fr* table, uint32_t usable, uint32_t* slots, uint32_t log_slots,
                               cudaStream_t s) {
    const uint32_t nslots = 1u << log_slots;
    if (usable > nslots / 2) return cudaErrorInvalidValue;
    ZK_CHECK(cudaMemsetAsync(slots, 0xff, (size_t)nslots * sizeof(uint32_t), s));
    table_insert_kernel<<<grid_rows(usable), 256, 0, s>>>(table, usable, slots, nslots - 1);
    return cudaGetLastError();
}

cudaError_t lookup_count(Fr* m, const Fr* table, const Fr* input, uint32_t n, uint32_t usable, const uint32_t* slots,
                         uint32_t log_slots, uint32_t* cnt, cudaStream_t s) {
    ZK_CHECK(cudaMemsetAsync(cnt, 0, (size_t)n * sizeof(uint32_t), s));
    input_count_kernel<<<grid_rows(usable), 256, 0, s>>>(table, input, usable, slots, (1u << log_slots) - 1, cnt);
    ZK_CHECK(cudaGetLastError());
    add_counts_kernel<<<grid_rows(n), 256, 0, s>>>(m, cnt, n);
    return cudaGetLastError();
}

// ------------------------------------------------------------------ poly_eval

// values of this level sit at positions j * stride; chunk j of C values is
// reduced by Horner with x and written back at position j * C * stride
__global__ void horner_level_kernel(const Fr* in, Fr* out, const Fr* x, uint32_t count, uint32_t C, uint32_t stride) {
    for (uint32_t j = blockIdx.x * blockDim.x + threadIdx.x; j < count; j += gridDim.x * blockDim.x) {
        const Fr xx = ld_elem<FrCfg>(x);
        const size_t base = (size_t)j * C * stride;
        // lazily reduced in [0, 2r) until the store
        Fr acc = ld_elem<FrCfg>(in + base + (size_t)(C - 1) * stride);
        for (int i = (int)C - 2; i >= 0; i--)
            acc = fe_add_lazy<FrCfg>(fe_mul_lazy<FrCfg>(acc, xx), ld_elem<FrCfg>(in + base + (size_t)i * stride));
        st_elem<FrCfg>(out + base, fe_canon<FrCfg>(acc));
    }
}

#ifndef POLY_EVAL_LOG_CHUNK
#define POLY_EVAL_LOG_CHUNK 4  // Horner chunks of 16 coefficients
#endif

cudaError_t poly_eval(const Fr* p, Fr* res, const Fr* x_table, uint32_t n, cudaStream_t s) {
    if (n == 0) return cudaErrorInvalidValue;
    if (n == 1) return cudaMemcpyAsync(res, p, sizeof(Fr), cudaMemcpyDeviceToDevice, s);
    if (n & (n - 1)) return cudaErrorInvalidValue;
    int log_n = 0;
    while ((1u << log_n) < n) log_n++;
    int done = 0;  // log2 of the current stride
    uint32_t remain = n;
    const Fr* src = p;
    while (remain > 1) {
        int d = log_n - done;
        if (d > POLY_EVAL_LOG_CHUNK) d = POLY_EVAL_LOG_CHUNK;
        const uint32_t C = 1u << d;
        const uint32_t count = remain / C;
        horner_level_kernel<<<grid_rows(count), 256, 0, s>>>(src, res, x_table + done, count, C, 1u << done);
        ZK_CHECK(cudaGetLastError());
        src = res;
        done += d;
        remain = count;
    }
    return cudaSuccess;
}

}  // namespace zk
