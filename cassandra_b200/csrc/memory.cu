// Memory of the library's objects (layouts, solvers, batches, the one-shot
// fits): a per-device cache of device blocks and a cache of pinned host
// blocks.  The training loop fits the same shapes again and again (one fit
// per empty-count stage, per epoch), and every fit used to map and unmap
// gigabytes through cudaMalloc/cudaFree, whose cost varies from call to call.
// Freed blocks now stay with the library and are handed out again to
// requests of about their size.
//
// cudaFree waits for the device before it frees; the cache keeps that
// guarantee lazily: a block freed since the device was last synchronised is
// handed out again only after one cudaDeviceSynchronize, so work still using
// it has finished.  Cached bytes are capped (a quarter of the device's
// memory); cas_release_cached_memory() returns them all.  The cache is never
// torn down at exit (the CUDA runtime may be gone by then).
#include <map>
#include <mutex>
#include <unordered_map>
#include <vector>

#include "common.cuh"

namespace cas {
namespace {

constexpr int kHostDevice = -1;  // pool key of pinned host blocks

struct Block {
    size_t size;
    int pool;           // device ordinal or kHostDevice
    unsigned long long epoch;  // sync epoch of the pool when the block was freed
};

struct Pool {
    std::multimap<size_t, void*> free_blocks;
    size_t cached = 0;
    size_t cap = 0;
    unsigned long long epoch = 1;  // bumped by every synchronisation
};

struct Cache {
    std::mutex mu;
    std::unordered_map<void*, Block> live;   // handed out
    std::unordered_map<void*, Block> idle;   // in a free list
    std::map<int, Pool> pools;
};

Cache& cache()
{
    static Cache* c = new Cache;  // never destroyed: see the header comment
    return *c;
}

size_t round_size(size_t n)
{
    if (n >= (size_t(1) << 20)) return (n + (size_t(2) << 20) - 1) & ~((size_t(2) << 20) - 1);
    return (n + 511) & ~size_t(511);
}

Pool& pool_of(Cache& c, int key)
{
    Pool& p = c.pools[key];
    if (p.cap == 0) {
        if (key == kHostDevice) {
            p.cap = size_t(8) << 30;
        } else {
            size_t free_b = 0, total_b = 0;
            if (cudaMemGetInfo(&free_b, &total_b) != cudaSuccess) total_b = size_t(16) << 30;
            p.cap = total_b / 4;
        }
    }
    return p;
}

void release_pool(Cache& c, int key, Pool& p)
{
    if (p.free_blocks.empty()) return;
    int prev = -1;
    if (key != kHostDevice) {
        cudaGetDevice(&prev);
        cudaSetDevice(key);
        cudaDeviceSynchronize();
    }
    for (auto& fb : p.free_blocks) {
        if (key == kHostDevice)
            cudaFreeHost(fb.second);
        else
            cudaFree(fb.second);
        c.idle.erase(fb.second);
    }
    p.free_blocks.clear();
    p.cached = 0;
    if (key != kHostDevice && prev >= 0) cudaSetDevice(prev);
}

cudaError_t cached_alloc(void** out, size_t bytes, bool host)
{
    *out = nullptr;
    if (bytes == 0) bytes = 1;
    int key = kHostDevice;
    if (!host) {
        const cudaError_t e = cudaGetDevice(&key);
        if (e != cudaSuccess) return e;
    }
    const size_t want = round_size(bytes);
    Cache& c = cache();
    std::lock_guard<std::mutex> lk(c.mu);
    Pool& p = pool_of(c, key);
    auto it = p.free_blocks.lower_bound(want);
    if (it != p.free_blocks.end() && it->first <= want + want / 4) {
        void* ptr = it->second;
        Block blk = c.idle[ptr];
        if (blk.epoch >= p.epoch) {
            // freed since the last synchronisation: wait for its last users
            const cudaError_t e = cudaDeviceSynchronize();
            if (e != cudaSuccess) return e;
            p.epoch++;
        }
        p.free_blocks.erase(it);
        c.idle.erase(ptr);
        p.cached -= blk.size;
        c.live[ptr] = Block{blk.size, key, 0};
        *out = ptr;
        return cudaSuccess;
    }
    cudaError_t e = host ? cudaMallocHost(out, want) : cudaMalloc(out, want);
    if (e == cudaErrorMemoryAllocation && p.cached > 0) {
        cudaGetLastError();  // clear the sticky-free allocation error
        release_pool(c, key, p);
        e = host ? cudaMallocHost(out, want) : cudaMalloc(out, want);
    }
    if (e != cudaSuccess) {
        *out = nullptr;
        return e;
    }
    c.live[*out] = Block{want, key, 0};
    return cudaSuccess;
}

void cached_free(void* ptr)
{
    if (!ptr) return;
    Cache& c = cache();
    std::lock_guard<std::mutex> lk(c.mu);
    auto it = c.live.find(ptr);
    if (it == c.live.end()) return;  // not ours (never happens for library objects)
    Block blk = it->second;
    c.live.erase(it);
    Pool& p = pool_of(c, blk.pool);
    if (p.cached + blk.size > p.cap) {
        // over the cap: really free it (cudaFree / cudaFreeHost wait as usual)
        if (blk.pool == kHostDevice) {
            cudaFreeHost(ptr);
        } else {
            int prev = -1;
            cudaGetDevice(&prev);
            if (prev != blk.pool) cudaSetDevice(blk.pool);
            cudaFree(ptr);
            if (prev != blk.pool && prev >= 0) cudaSetDevice(prev);
        }
        return;
    }
    blk.epoch = p.epoch;
    c.idle[ptr] = blk;
    p.free_blocks.emplace(blk.size, ptr);
    p.cached += blk.size;
}

}  // namespace

cudaError_t dmalloc_bytes(void** p, size_t bytes) { return cached_alloc(p, bytes, false); }
void dfree(const void* p) { cached_free(const_cast<void*>(p)); }
cudaError_t hmalloc_bytes(void** p, size_t bytes) { return cached_alloc(p, bytes, true); }
void hfree(const void* p) { cached_free(const_cast<void*>(p)); }

size_t cached_bytes()
{
    Cache& c = cache();
    std::lock_guard<std::mutex> lk(c.mu);
    size_t n = 0;
    for (auto& kv : c.pools) n += kv.second.cached;
    return n;
}

}  // namespace cas

extern "C" {

CAS_API size_t cas_cached_memory(void) { return cas::cached_bytes(); }

CAS_API void cas_release_cached_memory(void)
{
    cas::Cache& c = cas::cache();
    std::lock_guard<std::mutex> lk(c.mu);
    for (auto& kv : c.pools) cas::release_pool(c, kv.first, kv.second);
}

}  // extern "C"
