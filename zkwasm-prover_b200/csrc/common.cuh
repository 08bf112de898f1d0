// Shared device helpers: 32-byte element loads/stores and launch checks.
#pragma once
#include <cuda_runtime.h>
#include <stddef.h>
#include <stdint.h>

#include <mutex>

#include "field.cuh"

namespace zk {

template <class C>
__device__ __forceinline__ Fe<C> ld_elem(const Fe<C>* p) {
    const uint4* q = reinterpret_cast<const uint4*>(p);
    uint4 a = q[0], b = q[1];
    Fe<C> r;
    r.v[0] = a.x; r.v[1] = a.y; r.v[2] = a.z; r.v[3] = a.w;
    r.v[4] = b.x; r.v[5] = b.y; r.v[6] = b.z; r.v[7] = b.w;
    return r;
}

// read-only path (input buffers that the kernel does not write)
template <class C>
__device__ __forceinline__ Fe<C> ldg_elem(const Fe<C>* p) {
    const uint4* q = reinterpret_cast<const uint4*>(p);
    uint4 a = __ldg(q), b = __ldg(q + 1);
    Fe<C> r;
    r.v[0] = a.x; r.v[1] = a.y; r.v[2] = a.z; r.v[3] = a.w;
    r.v[4] = b.x; r.v[5] = b.y; r.v[6] = b.z; r.v[7] = b.w;
    return r;
}

template <class C>
__device__ __forceinline__ void st_elem(Fe<C>* p, const Fe<C>& v) {
    uint4* q = reinterpret_cast<uint4*>(p);
    q[0] = make_uint4(v.v[0], v.v[1], v.v[2], v.v[3]);
    q[1] = make_uint4(v.v[4], v.v[5], v.v[6], v.v[7]);
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

// entry i of a multiplier table from the Montgomery form wm of its factor:
// wm itself, or the pair (w, w' = floor(w 2^256 / r)) of fe_mul_shoup at
// elements 2i and 2i + 1
template <bool PAIRS>
__device__ __forceinline__ void st_factor(Fr* t, size_t i, const Fr& wm) {
    if (PAIRS) {
        st_elem<FrCfg>(t + 2 * i, fe_from_mont<FrCfg>(wm));
        st_elem<FrCfg>(t + 2 * i + 1, fe_shoup_companion<FrCfg>(wm));
    } else {
        st_elem<FrCfg>(t + i, wm);
    }
}

// A factor fixed for a whole launch (a challenge such as y or beta, a gate
// coefficient) in the pair form of fe_mul_shoup, built once from its
// Montgomery form: every product by it then costs 207 multiply-adds instead of
// 264 and lands in [0, 2r) like fe_mul_lazy.
struct KnownFr {
    Fr w, wp;
};

__device__ __forceinline__ KnownFr known_fr(const Fr& wm) {
    const Fr c = fe_canon<FrCfg>(wm);
    return {fe_from_mont<FrCfg>(c), fe_shoup_companion<FrCfg>(c)};
}

__device__ __forceinline__ Fr mul_known(const Fr& a, const KnownFr& k) { return fe_mul_shoup<FrCfg>(a, k.w, k.wp); }

// known_fr of the factor at p, built once per block by thread 0 (every thread
// of the block must call it); the second barrier lets a kernel call it again
// without thread 0 overwriting the slot before every thread has read it
__device__ __forceinline__ KnownFr block_known(const Fr* p) {
    __shared__ KnownFr k;
    if (threadIdx.x == 0) k = known_fr(ld_elem<FrCfg>(p));
    __syncthreads();
    const KnownFr r = k;
    __syncthreads();
    return r;
}

}  // namespace zk

#define ZK_CHECK(x)                           \
    do {                                      \
        cudaError_t err__ = (x);              \
        if (err__ != cudaSuccess) return err__; \
    } while (0)

namespace zk {

// Raises a kernel's dynamic shared-memory limit once per device: the
// attribute belongs to the device that is current when it is set, so a flag
// shared by all devices would leave a second GPU without it.  One instance per
// launch site (a function-local static), safe to call from several threads.
struct SmemOptIn {
    std::mutex mu;
    uint64_t done = 0;  // bit d: set on device d

    template <class K>
    cudaError_t ensure(K kernel, int bytes) {
        int dev = 0;
        ZK_CHECK(cudaGetDevice(&dev));
        if (dev < 0 || dev >= 64) return cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
        std::lock_guard<std::mutex> lock(mu);
        if ((done >> dev) & 1u) return cudaSuccess;
        ZK_CHECK(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
        done |= uint64_t(1) << dev;
        return cudaSuccess;
    }
};

}  // namespace zk
