// Shared helpers for the cassandra_b200 CUDA library: status handling, the
// thread-local error message behind cas_last_error(), launch helpers and the
// deterministic block reductions used by every kernel.
#pragma once
#include <cuda_runtime.h>
#include <cstdint>
#include <cstdio>
#include <string>

#include <nvtx3/nvToolsExt.h>

#include "../../include/cassandra_b200.h"

namespace cas {

// An NVTX range over a scope: the library's long host calls (fits, layout
// builds, solves) show as named ranges in a profiler timeline.  Header-only
// NVTX 3: without a profiler attached a push/pop is a few instructions.
struct NvtxRange {
    explicit NvtxRange(const char* name) { nvtxRangePushA(name); }
    ~NvtxRange() { nvtxRangePop(); }
    NvtxRange(const NvtxRange&) = delete;
    NvtxRange& operator=(const NvtxRange&) = delete;
};

// Thread-local message of the last failing call (read by cas_last_error).
void set_error(const std::string& msg);
const std::string& last_error();

// Number of SMs of the current device (cached per device).
int sm_count();

// Process-wide count of kernels this library has launched (kernels inside a
// replayed CUDA graph are counted at each replay).  Read by
// cas_kernel_launches().
void count_launch(long long n = 1);
long long launch_count();

struct Error {
    cas_status status;
    std::string msg;
};

// Device and pinned-host memory of the library's objects, from a cache that
// keeps freed blocks for reuse (memory.cu).  dfree/hfree keep cudaFree's
// guarantee that work still using the block finishes before it is reused.
cudaError_t dmalloc_bytes(void** p, size_t bytes);
void dfree(const void* p);
cudaError_t hmalloc_bytes(void** p, size_t bytes);
void hfree(const void* p);
template <typename T>
cudaError_t dmalloc(T** p, size_t bytes)
{
    return dmalloc_bytes(reinterpret_cast<void**>(p), bytes);
}
template <typename T>
cudaError_t hmalloc(T** p, size_t bytes)
{
    return hmalloc_bytes(reinterpret_cast<void**>(p), bytes);
}

}  // namespace cas

// Returns from the enclosing cas_status function on a CUDA error.
#define CAS_CUDA(call)                                                                         \
    do {                                                                                       \
        cudaError_t e_ = (call);                                                               \
        if (e_ != cudaSuccess) {                                                               \
            cas::set_error(std::string(#call) + ": " + cudaGetErrorString(e_));                \
            return e_ == cudaErrorMemoryAllocation ? CAS_ERR_OUT_OF_MEMORY : CAS_ERR_CUDA;     \
        }                                                                                      \
    } while (0)

#define CAS_CHECK_LAUNCH() CAS_CUDA(cudaGetLastError())

#define CAS_TRY(call)                               \
    do {                                            \
        cas_status s_ = (call);                     \
        if (s_ != CAS_OK) return s_;                \
    } while (0)

#define CAS_REQUIRE(cond, code, msg)                \
    do {                                            \
        if (!(cond)) {                              \
            cas::set_error(msg);                    \
            return (code);                          \
        }                                           \
    } while (0)

namespace cas {

inline unsigned ceil_div(int64_t a, int64_t b) { return static_cast<unsigned>((a + b - 1) / b); }

// Neumaier's compensated sum: (s, c) accumulates x with the rounding error of
// each addition kept in c.  Used for the FP64 reductions of the mixed solver.
struct Comp {
    double s = 0, c = 0;
    __host__ __device__ void add(double x)
    {
        double t = s + x;
        if (fabs(s) >= fabs(x))
            c += (s - t) + x;
        else
            c += (x - t) + s;
        s = t;
    }
    __host__ __device__ void add(const Comp& o)
    {
        add(o.s);
        add(o.c);
    }
    __host__ __device__ double value() const { return s + c; }
};

// Deterministic block-wide sum of one double per thread: warp shuffles in a
// fixed tree, then warp 0 combines the warp totals in lane order.  All
// threads of the block must call it; the result is valid in thread 0.
template <int BLOCK>
__device__ inline double block_sum(double v, double* smem)
{
    static_assert(BLOCK % 32 == 0 && BLOCK <= 1024, "block size");
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    if (lane == 0) smem[warp] = v;
    __syncthreads();
    double r = 0;
    if (warp == 0) {
        r = lane < BLOCK / 32 ? smem[lane] : 0.0;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) r += __shfl_down_sync(0xffffffffu, r, o);
    }
    __syncthreads();
    return r;
}

// Compensated variant: each thread contributes a Comp; the tree combines
// (s, c) pairs with Neumaier steps so the FP64 result keeps ~2x precision.
template <int BLOCK>
__device__ inline Comp block_sum_comp(Comp v, double* smem)
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        Comp w;
        w.s = __shfl_down_sync(0xffffffffu, v.s, o);
        w.c = __shfl_down_sync(0xffffffffu, v.c, o);
        v.add(w);
    }
    if (lane == 0) {
        smem[2 * warp] = v.s;
        smem[2 * warp + 1] = v.c;
    }
    __syncthreads();
    Comp r;
    if (warp == 0) {
        if (lane < BLOCK / 32) {
            r.s = smem[2 * lane];
            r.c = smem[2 * lane + 1];
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            Comp w;
            w.s = __shfl_down_sync(0xffffffffu, r.s, o);
            w.c = __shfl_down_sync(0xffffffffu, r.c, o);
            r.add(w);
        }
    }
    __syncthreads();
    return r;
}

}  // namespace cas
