// Status/error plumbing, pattern-set handles and the indexer kernel.
#include <atomic>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "common.cuh"
#include "internal.cuh"
#include "indexer.cuh"
#include "patterns.h"

namespace cas {

namespace {
thread_local std::string g_last_error;
std::atomic<long long> g_launches{0};
}  // namespace

void count_launch(long long n) { g_launches.fetch_add(n, std::memory_order_relaxed); }
long long launch_count() { return g_launches.load(std::memory_order_relaxed); }

void set_error(const std::string& msg) { g_last_error = msg; }
const std::string& last_error() { return g_last_error; }

int sm_count()
{
    static std::mutex mu;
    static std::vector<int> cache;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return 148;
    std::lock_guard<std::mutex> lock(mu);
    if (static_cast<int>(cache.size()) <= dev) cache.resize(dev + 1, 0);
    if (cache[dev] == 0) {
        int n = 0;
        if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || n <= 0) n = 148;
        cache[dev] = n;
    }
    return cache[dev];
}

cas_status require_device()
{
    int n = 0;
    cudaError_t e = cudaGetDeviceCount(&n);
    if (e != cudaSuccess || n == 0) {
        cudaGetLastError();
        set_error("no usable CUDA device (cassandra_b200 has no CPU fallback)");
        return CAS_ERR_NO_DEVICE;
    }
    return CAS_OK;
}

// ---------------------------------------------------------------------------
// Indexer kernel.
//
// A warp indexes 32 positions per step: every lane loads one 16-byte
// position record, then the warp walks the 32 positions (broadcast by
// shuffles) and lane j evaluates slots j, j + 32, ... of the current
// position, so each CSR row is written as contiguous 128-byte segments.
// The slot recipes live in shared memory, and so does the current
// position's digit board (64 cells, one byte each, written by lanes 0-15 as
// one word of four cells each), from which every square costs a byte load.
// ---------------------------------------------------------------------------

// Cells of squares 4j .. 4j+3 as four bytes: each of the four bits of the
// player's and the opponent's nibble spread to bit 0 of its byte.
__device__ __forceinline__ uint32_t cell_word(uint32_t p_nib, uint32_t o_nib)
{
    const uint32_t sp = (p_nib * 0x00204081u) & 0x01010101u;  // bit i -> bit 8i
    const uint32_t so = (o_nib * 0x00204081u) & 0x01010101u;
    return sp | (so << 1);
}

constexpr int kRowIndexThreads = 256;

__global__ void __launch_bounds__(kRowIndexThreads) index_kernel(const Instance* __restrict__ g_inst, int k,
                                                                 const uint32_t* __restrict__ tables,
                                                                 const ulonglong2* __restrict__ pos, int64_t n,
                                                                 uint32_t* __restrict__ out)
{
    __shared__ __align__(16) uint32_t s_board[kRowIndexThreads / 32][16];
    extern __shared__ Instance s_inst[];
    for (int i = threadIdx.x; i < k; i += blockDim.x) s_inst[i] = g_inst[i];
    __syncthreads();

    const int lane = threadIdx.x & 31;
    uint32_t* wboard = s_board[threadIdx.x >> 5];
    const uint8_t* board = reinterpret_cast<const uint8_t*>(wboard);
    const int64_t warps = static_cast<int64_t>(gridDim.x) * (blockDim.x >> 5);
    for (int64_t base = (static_cast<int64_t>(blockIdx.x) * (blockDim.x >> 5) + (threadIdx.x >> 5)) * 32; base < n;
         base += warps * 32) {
        ulonglong2 mine = make_ulonglong2(0, 0);
        if (base + lane < n) mine = pos[base + lane];
        const int cnt = n - base < 32 ? static_cast<int>(n - base) : 32;
        for (int i = 0; i < cnt; i++) {
            const uint64_t p = __shfl_sync(0xffffffffu, mine.x, i);
            const uint64_t o = __shfl_sync(0xffffffffu, mine.y, i);
            __syncwarp();  // the previous position's board is read
            if (lane < 16)
                wboard[lane] = cell_word(static_cast<uint32_t>(p >> (4 * lane)) & 0xFu,
                                         static_cast<uint32_t>(o >> (4 * lane)) & 0xFu);
            __syncwarp();
            uint32_t* row = out + (base + i) * k;
            for (int j = lane; j < k; j += 32) row[j] = eval_slot_board_all<1>(s_inst[j], tables, board);
        }
    }
}

cas_status launch_index(const DevicePatterns& dp, const uint64_t* d_pos, int64_t n, uint32_t* d_out,
                        cudaStream_t stream)
{
    if (n == 0) return CAS_OK;
    const int threads = kRowIndexThreads;
    const int64_t warps_needed = (n + 31) / 32;
    const int64_t blocks = std::min<int64_t>((warps_needed + 7) / 8, static_cast<int64_t>(sm_count()) * 8);
    const size_t smem = sizeof(Instance) * dp.k;
    { index_kernel<<<static_cast<unsigned>(blocks), threads, smem, stream>>>(
        dp.instances, dp.k, dp.tables, reinterpret_cast<const ulonglong2*>(d_pos), n, d_out); cas::count_launch(); }
    CAS_CHECK_LAUNCH();
    return CAS_OK;
}

}  // namespace cas

using namespace cas;

struct cas_patterns {
    PatternSet set;
    DevicePatterns dev;  // uploaded lazily, per device
    int device = -1;
    std::mutex mu;
};

namespace cas {
cas_status patterns_on_device(const cas_patterns* cp, const DevicePatterns** out)
{
    auto* p = const_cast<cas_patterns*>(cp);
    CAS_TRY(require_device());
    int dev = 0;
    CAS_CUDA(cudaGetDevice(&dev));
    std::lock_guard<std::mutex> lock(p->mu);
    if (p->device != dev) {
        if (p->device >= 0) {
            int cur = dev;
            cudaSetDevice(p->device);
            dfree(p->dev.instances);
            dfree(p->dev.tables);
            cudaSetDevice(cur);
            p->dev = DevicePatterns{};
        }
        const PatternSet& s = p->set;
        CAS_CUDA(dmalloc(&p->dev.instances, sizeof(Instance) * s.instances.size()));
        CAS_CUDA(cudaMemcpy(p->dev.instances, s.instances.data(), sizeof(Instance) * s.instances.size(),
                            cudaMemcpyHostToDevice));
        const size_t tb = std::max<size_t>(1, s.tables.size());
        CAS_CUDA(dmalloc(&p->dev.tables, sizeof(uint32_t) * tb));
        if (!s.tables.empty())
            CAS_CUDA(cudaMemcpy(p->dev.tables, s.tables.data(), sizeof(uint32_t) * s.tables.size(),
                                cudaMemcpyHostToDevice));
        p->dev.k = static_cast<int>(s.instances.size());
        p->dev.cols = s.cols;
        p->device = dev;
    }
    *out = &p->dev;
    return CAS_OK;
}

const PatternSet& pattern_set(const cas_patterns* p) { return p->set; }
}  // namespace cas

extern "C" {

CAS_API const char* cas_status_name(cas_status s)
{
    switch (s) {
        case CAS_OK: return "CAS_OK";
        case CAS_ERR_SIZE_MISMATCH: return "CAS_ERR_SIZE_MISMATCH";
        case CAS_ERR_INVALID_ARGUMENT: return "CAS_ERR_INVALID_ARGUMENT";
        case CAS_ERR_PATTERN: return "CAS_ERR_PATTERN";
        case CAS_ERR_CUDA: return "CAS_ERR_CUDA";
        case CAS_ERR_OUT_OF_MEMORY: return "CAS_ERR_OUT_OF_MEMORY";
        case CAS_ERR_NO_DEVICE: return "CAS_ERR_NO_DEVICE";
        case CAS_ERR_BREAKDOWN: return "CAS_ERR_BREAKDOWN";
        case CAS_ERR_NOT_CONVERGED: return "CAS_ERR_NOT_CONVERGED";
    }
    return "CAS_ERR_UNKNOWN";
}

CAS_API size_t cas_last_error(char* buf, size_t cap)
{
    const std::string& m = last_error();
    if (buf && cap) {
        const size_t n = std::min(cap - 1, m.size());
        std::memcpy(buf, m.data(), n);
        buf[n] = 0;
    }
    return m.size();
}

CAS_API int cas_version(void) { return 20100; }  // 2.1.0: solver checkpoints (cas_solver_*_state)

CAS_API long long cas_kernel_launches(void) { return launch_count(); }

CAS_API cas_status cas_patterns_create(const uint64_t* masks, int n, cas_index_mode mode, cas_patterns** out)
{
    CAS_REQUIRE(out && masks && n > 0, CAS_ERR_INVALID_ARGUMENT, "cas_patterns_create: null argument or n <= 0");
    CAS_REQUIRE(mode == CAS_INDEX_REFERENCE || mode == CAS_INDEX_EXPANDED, CAS_ERR_INVALID_ARGUMENT,
                "cas_patterns_create: unknown index mode");
    *out = nullptr;
    auto* p = new (std::nothrow) cas_patterns;
    CAS_REQUIRE(p, CAS_ERR_OUT_OF_MEMORY, "cas_patterns_create: out of host memory");
    std::string err;
    if (!build_pattern_set(masks, n, mode, p->set, err)) {
        delete p;
        set_error("cas_patterns_create: " + err);
        return CAS_ERR_PATTERN;
    }
    *out = p;
    return CAS_OK;
}

CAS_API void cas_patterns_destroy(cas_patterns* p)
{
    if (!p) return;
    if (p->device >= 0) {
        int cur = 0;
        cudaGetDevice(&cur);
        cudaSetDevice(p->device);
        dfree(p->dev.instances);
        dfree(p->dev.tables);
        cudaSetDevice(cur);
    }
    delete p;
}

CAS_API int64_t cas_patterns_cols(const cas_patterns* p) { return p ? p->set.cols : -1; }

CAS_API int cas_patterns_nnz_per_row(const cas_patterns* p)
{
    return p ? static_cast<int>(p->set.instances.size()) : -1;
}

CAS_API cas_status cas_patterns_variations(const cas_patterns* p, uint64_t* h_out)
{
    CAS_REQUIRE(p && h_out, CAS_ERR_INVALID_ARGUMENT, "cas_patterns_variations: null argument");
    std::memcpy(h_out, p->set.variations.data(), sizeof(uint64_t) * p->set.variations.size());
    return CAS_OK;
}

CAS_API cas_status cas_patterns_indexer(const cas_patterns* p, int i, uint64_t* stored_pattern, int* order,
                                        int64_t* space, int64_t* offset)
{
    CAS_REQUIRE(p && i >= 0 && i < static_cast<int>(p->set.indexers.size()), CAS_ERR_INVALID_ARGUMENT,
                "cas_patterns_indexer: bad handle or index");
    const IndexerInfo& in = p->set.indexers[i];
    if (stored_pattern) *stored_pattern = in.stored_pattern;
    if (order) *order = in.order;
    if (space) *space = in.space;
    if (offset) *offset = in.offset;
    return CAS_OK;
}

CAS_API cas_status cas_index(const cas_patterns* p, const uint64_t* d_positions, int64_t n, uint32_t* d_out,
                             void* stream)
{
    cas::NvtxRange nvtx_range("cas_index");
    CAS_REQUIRE(p && n >= 0, CAS_ERR_INVALID_ARGUMENT, "cas_index: null handle or negative count");
    CAS_REQUIRE(n == 0 || (d_positions && d_out), CAS_ERR_INVALID_ARGUMENT, "cas_index: null buffer");
    CAS_REQUIRE((reinterpret_cast<uintptr_t>(d_positions) & 15) == 0, CAS_ERR_INVALID_ARGUMENT,
                "cas_index: position records must be 16-byte aligned");
    const DevicePatterns* dp = nullptr;
    CAS_TRY(patterns_on_device(p, &dp));
    return launch_index(*dp, d_positions, n, d_out, static_cast<cudaStream_t>(stream));
}

}  // extern "C"
