// Host staging for column transfers (host code of the library).
//
// Reference behaviour replaced: the pinned huge-page host allocator
// (src/hugetlb.rs: 256 MiB mmap(MAP_HUGETLB) blocks split into 128 MiB chunks,
// registered with the CUDA driver) and the bounded asynchronous copy queue
// (src/async_copy_queue.rs: at most `max` device-to-host copies in flight,
// each on its own stream, the oldest waited for before a new one is issued),
// which keep the column copies of a proof off the critical path.
//
// * HostPool: blocks of `chunks_per_block` chunks of `chunk_bytes`, mapped
//   with huge pages when asked and available (else transparent huge pages are
//   requested with madvise), page-locked with cudaHostRegister when asked.
//   Allocation hands out whole chunks from a free list; blocks are kept until
//   the pool is destroyed.  Thread-safe.
// * CopyQueue: a ring of streams; a push orders its copy after the work
//   already queued on the caller's stream (an event), issues one
//   cudaMemcpyAsync and records a completion event; with `max` copies in
//   flight the oldest is waited for first.  Not thread-safe (one owner).
#include <sys/mman.h>

#include <deque>
#include <mutex>
#include <new>
#include <vector>

#include "common.cuh"

namespace {

struct HostBlock {
    char* base;
    size_t bytes;   // length of the mapping (a whole number of huge pages for MAP_HUGETLB)
    bool mapped;    // mmap'ed (else operator new)
    bool pinned;    // cudaHostRegister'ed
};

// MAP_HUGETLB mappings are made in whole huge pages; munmap must be given the
// rounded length or it fails with EINVAL and the block leaks.  2 MiB is the
// default huge-page size on x86-64 and aarch64 hosts.
constexpr size_t HUGE_PAGE_BYTES = size_t(2) << 20;

void release_block(const HostBlock& b) {
    if (b.pinned) cudaHostUnregister(b.base);
    if (b.mapped) {
        // a failed munmap leaves the mapping in place; there is nothing more to do here than not crash
        (void)munmap(b.base, b.bytes);
    } else {
        ::operator delete(b.base, std::align_val_t(4096));
    }
}

struct HostPool {
    size_t chunk = 0;
    int per_block = 0;
    int flags = 0;
    std::mutex mu;
    std::vector<HostBlock> blocks;
    std::vector<char*> free_chunks;
    size_t used = 0;
};

constexpr int POOL_PIN = 1;
constexpr int POOL_HUGE = 2;

bool pool_grow(HostPool* p) {
    const size_t bytes = p->chunk * (size_t)p->per_block;
    HostBlock b{nullptr, bytes, false, false};
    if (p->flags & POOL_HUGE) {
#ifdef MAP_HUGETLB
        const size_t huge_bytes = (bytes + HUGE_PAGE_BYTES - 1) / HUGE_PAGE_BYTES * HUGE_PAGE_BYTES;
        void* m = mmap(nullptr, huge_bytes, PROT_READ | PROT_WRITE, MAP_PRIVATE | MAP_ANONYMOUS | MAP_HUGETLB, -1, 0);
        if (m != MAP_FAILED) {
            b.base = static_cast<char*>(m);
            b.bytes = huge_bytes;
            b.mapped = true;
        }
#endif
        if (!b.base) {
            void* m = mmap(nullptr, bytes, PROT_READ | PROT_WRITE, MAP_PRIVATE | MAP_ANONYMOUS, -1, 0);
            if (m == MAP_FAILED) return false;
#ifdef MADV_HUGEPAGE
            madvise(m, bytes, MADV_HUGEPAGE);
#endif
            b.base = static_cast<char*>(m);
            b.mapped = true;
        }
    } else {
        b.base = static_cast<char*>(::operator new(bytes, std::align_val_t(4096), std::nothrow));
        if (!b.base) return false;
    }
    if (p->flags & POOL_PIN) {
        if (cudaHostRegister(b.base, b.bytes, cudaHostRegisterDefault) != cudaSuccess) {
            cudaGetLastError();
            release_block(b);
            return false;
        }
        b.pinned = true;
    }
    p->blocks.push_back(b);
    for (int i = p->per_block - 1; i >= 0; i--) p->free_chunks.push_back(b.base + (size_t)i * p->chunk);
    return true;
}

struct CopyQueue {
    int max = 1;
    int device = 0;
    std::vector<cudaStream_t> streams;
    std::vector<cudaEvent_t> done;    // one completion event per stream slot
    std::deque<int> in_flight;        // stream slots, oldest first
    cudaEvent_t order = nullptr;      // "after" marker on the caller's stream
    int next = 0;
};

}  // namespace

extern "C" {

void* zkp_host_pool_create(size_t chunk_bytes, int chunks_per_block, int flags) {
    if (chunk_bytes == 0 || chunks_per_block <= 0) return nullptr;
    HostPool* p = new (std::nothrow) HostPool;
    if (!p) return nullptr;
    p->chunk = (chunk_bytes + 4095) / 4096 * 4096;
    p->per_block = chunks_per_block;
    p->flags = flags;
    return p;
}

void* zkp_host_pool_alloc(void* pool, size_t bytes) {
    HostPool* p = static_cast<HostPool*>(pool);
    if (!p || bytes == 0 || bytes > p->chunk) return nullptr;
    std::lock_guard<std::mutex> lock(p->mu);
    if (p->free_chunks.empty() && !pool_grow(p)) return nullptr;
    char* c = p->free_chunks.back();
    p->free_chunks.pop_back();
    p->used++;
    return c;
}

int zkp_host_pool_free(void* pool, void* ptr) {
    HostPool* p = static_cast<HostPool*>(pool);
    if (!p || !ptr) return -1;
    char* c = static_cast<char*>(ptr);
    std::lock_guard<std::mutex> lock(p->mu);
    for (const HostBlock& b : p->blocks) {
        if (c >= b.base && c < b.base + p->chunk * (size_t)p->per_block) {
            if ((size_t)(c - b.base) % p->chunk != 0) return -1;
            for (char* f : p->free_chunks)
                if (f == c) return -1;  // double free
            p->free_chunks.push_back(c);
            p->used--;
            return 0;
        }
    }
    return -1;
}

// blocks mapped so far and chunks handed out
void zkp_host_pool_stats(void* pool, size_t* blocks, size_t* used_chunks) {
    HostPool* p = static_cast<HostPool*>(pool);
    if (!p) return;
    std::lock_guard<std::mutex> lock(p->mu);
    if (blocks) *blocks = p->blocks.size();
    if (used_chunks) *used_chunks = p->used;
}

void zkp_host_pool_destroy(void* pool) {
    HostPool* p = static_cast<HostPool*>(pool);
    if (!p) return;
    for (const HostBlock& b : p->blocks) release_block(b);
    delete p;
}

void* zkp_copy_queue_create(int max_in_flight, int device) {
    if (max_in_flight <= 0) return nullptr;
    CopyQueue* q = new (std::nothrow) CopyQueue;
    if (!q) return nullptr;
    q->max = max_in_flight;
    q->device = device;
    // the streams and events belong to `device`; the caller's current device
    // is put back before returning, on success and on failure
    int prev_device = 0;
    if (cudaGetDevice(&prev_device) != cudaSuccess || cudaSetDevice(device) != cudaSuccess) {
        cudaGetLastError();
        delete q;
        return nullptr;
    }
    bool ok = cudaEventCreateWithFlags(&q->order, cudaEventDisableTiming) == cudaSuccess;
    for (int i = 0; ok && i < max_in_flight; i++) {
        cudaStream_t s;
        cudaEvent_t e;
        ok = cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking) == cudaSuccess;
        if (!ok) break;
        q->streams.push_back(s);
        ok = cudaEventCreateWithFlags(&e, cudaEventDisableTiming) == cudaSuccess;
        if (ok) q->done.push_back(e);
    }
    if (!ok) {
        for (cudaStream_t s : q->streams) cudaStreamDestroy(s);
        for (cudaEvent_t e : q->done) cudaEventDestroy(e);
        if (q->order) cudaEventDestroy(q->order);
        delete q;
        cudaSetDevice(prev_device);
        return nullptr;
    }
    cudaSetDevice(prev_device);
    return q;
}

// one copy of `bytes` (kind: a cudaMemcpyKind), ordered after the work queued
// on `after` so far; waits for the oldest copy when `max` are in flight
cudaError_t zkp_copy_queue_push(void* queue, void* dst, const void* src, size_t bytes, int kind,
                                cudaStream_t after) {
    CopyQueue* q = static_cast<CopyQueue*>(queue);
    if (!q || (bytes && (!dst || !src))) return cudaErrorInvalidValue;
    if ((int)q->in_flight.size() == q->max) {
        const int old = q->in_flight.front();
        q->in_flight.pop_front();
        ZK_CHECK(cudaEventSynchronize(q->done[old]));
    }
    const int slot = q->next;
    q->next = (q->next + 1) % q->max;
    cudaStream_t s = q->streams[slot];
    ZK_CHECK(cudaEventRecord(q->order, after));
    ZK_CHECK(cudaStreamWaitEvent(s, q->order, 0));
    if (bytes) ZK_CHECK(cudaMemcpyAsync(dst, src, bytes, (cudaMemcpyKind)kind, s));
    ZK_CHECK(cudaEventRecord(q->done[slot], s));
    q->in_flight.push_back(slot);
    return cudaSuccess;
}

// waits for every copy in flight
cudaError_t zkp_copy_queue_sync(void* queue) {
    CopyQueue* q = static_cast<CopyQueue*>(queue);
    if (!q) return cudaErrorInvalidValue;
    while (!q->in_flight.empty()) {
        const int old = q->in_flight.front();
        q->in_flight.pop_front();
        ZK_CHECK(cudaEventSynchronize(q->done[old]));
    }
    return cudaSuccess;
}

void zkp_copy_queue_destroy(void* queue) {
    CopyQueue* q = static_cast<CopyQueue*>(queue);
    if (!q) return;
    zkp_copy_queue_sync(q);
    for (cudaStream_t s : q->streams) cudaStreamDestroy(s);
    for (cudaEvent_t e : q->done) cudaEventDestroy(e);
    if (q->order) cudaEventDestroy(q->order);
    delete q;
}

}  // extern "C"
