// MSM entry point that allocates nothing, for callers that cannot call
// cudaMalloc: a host whose device memory is entirely owned by its own pool
// (the prover reserves one pool up front and a stray allocation either fails
// or fragments it), and latency-critical paths that must not pay cudaMalloc's
// implicit device synchronisation.  Such callers cannot size and hand over the scratch
// that zkp_msm takes either, so this variant keeps its scratch in a fixed
// device array inside the library.
//
// Limits and sharing rules:
//   - at most ZKP_MSM_STATIC_MAX_N points per call; larger n is rejected with
//     cudaErrorInvalidValue before anything is launched;
//   - the scratch is one 9 MiB __device__ array per GPU that loads the
//     library, held until the process exits;
//   - every call on a device shares it and it keeps the previous call's
//     contents; the bucket histogram, the only part read before it is
//     written, is cleared on the stream at the start of each call;
//   - calls whose work overlaps on the GPU (different streams, or host
//     threads without ordering) race on the scratch and give wrong results;
//     serialise them on one stream;
//   - the first call on a device looks up the array's device address with
//     cudaGetSymbolAddress (with that device current); make that first call
//     before any stream capture begins.
#include <mutex>

#include "common.cuh"
#include "kernels.h"

#define ZKP_MSM_STATIC_MAX_N (1u << 14)
#define ZKP_MSM_STATIC_BYTES (9u << 20)
#define ZKP_MSM_STATIC_WINDOW 10
#define ZKP_MAX_DEVICES 64

static __device__ __align__(256) unsigned char g_msm_static_scratch[ZKP_MSM_STATIC_BYTES];

static void* g_static_addr[ZKP_MAX_DEVICES];
static std::mutex g_static_mu;

// fixed window and at least 32 sorted entries per accumulation thread, so the
// scratch of every n <= ZKP_MSM_STATIC_MAX_N fits the array
static zk::MsmPlan static_plan(uint32_t n) {
    zk::MsmPlan p = zk::msm_make_plan(n, ZKP_MSM_STATIC_WINDOW, false);
    const uint64_t entries = (uint64_t)n * p.W;
    if (p.L < 32) {
        p.L = 32;
        p.nacc = (uint32_t)((entries + p.L - 1) / p.L);
        if (p.nacc == 0) p.nacc = 1;
    }
    return p;
}

extern "C" cudaError_t zkp_msm_static(void* out, const void* bases, const void* scalars, uint32_t n,
                                      cudaStream_t stream) {
    if (!out || (n && (!bases || !scalars))) return cudaErrorInvalidValue;
    if (n > ZKP_MSM_STATIC_MAX_N) return cudaErrorInvalidValue;
    int dev = 0;
    cudaError_t err = cudaGetDevice(&dev);
    if (err != cudaSuccess) return err;
    if (dev < 0 || dev >= ZKP_MAX_DEVICES) return cudaErrorInvalidDevice;
    void* base = nullptr;
    {
        std::lock_guard<std::mutex> lock(g_static_mu);
        if (!g_static_addr[dev]) {
            void* p = nullptr;
            err = cudaGetSymbolAddress(&p, g_msm_static_scratch);
            if (err != cudaSuccess) return err;
            g_static_addr[dev] = p;
        }
        base = g_static_addr[dev];
    }
    zk::MsmPlan plan = static_plan(n);
    if (zk::msm_scratch_bytes(plan) > ZKP_MSM_STATIC_BYTES) return cudaErrorInvalidValue;
    zk::MsmScratch sc = {};
    if (n) zk::msm_layout(plan, base, &sc);
    return zk::msm_run(reinterpret_cast<zk::Jac*>(out), reinterpret_cast<const zk::Aff*>(bases),
                       reinterpret_cast<const zk::Fr*>(scalars), plan, sc, stream);
}
