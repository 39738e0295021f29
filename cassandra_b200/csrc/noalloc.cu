// An allocation-free entry point: y = A x and ||y||^2 over caller-owned
// row-major indices.
//
// Some callers cannot let this library allocate device memory: code whose
// device memory belongs to another allocator (a framework's caching pool, or a
// budget reserved at start-up that must not grow), and code on a path where
// cudaMalloc / cudaFree are unacceptable because they synchronise the device
// or may not be called there.  The regular products keep their per-CTA
// partial sums in memory the library allocates; this variant keeps them in a
// fixed, file-scope device array instead, so a call allocates nothing.
//
// The scratch array below is part of the library's device image: every GPU
// that loads the library holds its 128 KB until the process exits.  Host code
// cannot pass the array's name to a kernel (on the host it is only a
// stand-in for the device symbol), so the device address is looked up with
// cudaGetSymbolAddress once per device, on that device's first call; make that
// first call before any stream capture.  The lookup is cached per device
// ordinal for the life of the process: it assumes the device's primary
// context (the one the CUDA runtime uses), and does not survive
// cudaDeviceReset, after which the library's device image may load elsewhere.
// All calls share the array and it keeps the last call's contents; each call
// overwrites every partial it reads, so nothing has to start at zero, but
// calls that overlap on the GPU (other streams or threads) race on the array
// and must be serialised by the caller.  A column index >= cols is never
// read through: it makes its row's y and the norm NaN.
#include <mutex>

#include "common.cuh"
#include "internal.cuh"

namespace cas {
namespace {

constexpr int kNoAllocThreads = 256;                  // 8 warps, one row per warp at a time
constexpr int64_t kNoAllocRowsPerCta = 2048;          // fixed: partials depend on rows only
constexpr int kNoAllocMaxCtas = 8192;                 // scratch capacity in CTAs
constexpr int64_t kNoAllocMaxRows = kNoAllocRowsPerCta * kNoAllocMaxCtas;  // 16,777,216

// Per-CTA (sum, compensation) pairs of ||y||^2.
static __device__ __align__(256) double g_noalloc_partials[2 * kNoAllocMaxCtas];

// An index >= cols is never read through: it contributes NaN, so that row's
// y and the norm come out NaN instead of the kernel reading outside x (the
// call is asynchronous and cannot report the bad index as a status).
__global__ void __launch_bounds__(kNoAllocThreads) noalloc_spmv_norm_kernel(const uint32_t* __restrict__ idx, int k,
                                                                            int64_t rows, int64_t cols,
                                                                            const double* __restrict__ x,
                                                                            double* __restrict__ y,
                                                                            double* __restrict__ partials)
{
    const double kNaN = __longlong_as_double(0x7FF8000000000000LL);
    __shared__ double smem[64];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int64_t r0 = static_cast<int64_t>(blockIdx.x) * kNoAllocRowsPerCta;
    const int64_t r1 = min(rows, r0 + kNoAllocRowsPerCta);
    Comp mine;
    for (int64_t r = r0 + warp; r < r1; r += kNoAllocThreads / 32) {
        const uint32_t* row = idx + r * k;
        double acc = 0;
        for (int j = lane; j < k; j += 32) {
            const uint32_t c = __ldg(row + j);
            acc += c < cols ? __ldg(x + c) : kNaN;
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
        if (lane == 0) {
            y[r] = acc;
            mine.add(acc * acc);
        }
    }
    const Comp total = block_sum_comp<kNoAllocThreads>(mine, smem);
    if (threadIdx.x == 0) {
        partials[2 * blockIdx.x] = total.s;
        partials[2 * blockIdx.x + 1] = total.c;
    }
}

__global__ void __launch_bounds__(1024) noalloc_norm_finish_kernel(const double* __restrict__ partials, int n,
                                                                   double* __restrict__ out)
{
    __shared__ double smem[64];
    Comp acc;
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        acc.add(partials[2 * i]);
        acc.add(partials[2 * i + 1]);
    }
    const Comp total = block_sum_comp<1024>(acc, smem);
    if (threadIdx.x == 0) *out = total.value();
}

// Device address of the scratch array, looked up once per device.
std::mutex g_noalloc_mu;
double* g_noalloc_ptr[64] = {};

cas_status noalloc_scratch(double** out)
{
    int dev = 0;
    CAS_CUDA(cudaGetDevice(&dev));
    CAS_REQUIRE(dev >= 0 && dev < 64, CAS_ERR_INVALID_ARGUMENT, "cas_spmv_norm_noalloc: device index above 63");
    std::lock_guard<std::mutex> lock(g_noalloc_mu);
    if (!g_noalloc_ptr[dev]) {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_partials);
        if (e != cudaSuccess || !p) {
            set_error(std::string("cas_spmv_norm_noalloc: cudaGetSymbolAddress failed: ") + cudaGetErrorString(e));
            return CAS_ERR_CUDA;
        }
        g_noalloc_ptr[dev] = static_cast<double*>(p);
    }
    *out = g_noalloc_ptr[dev];
    return CAS_OK;
}

}  // namespace
}  // namespace cas

using namespace cas;

extern "C" {

CAS_API int64_t cas_spmv_norm_noalloc_max_rows(void) { return kNoAllocMaxRows; }

CAS_API cas_status cas_spmv_norm_noalloc(const uint32_t* d_indices, int nnz_per_row, int64_t rows, int64_t cols,
                                         const double* d_x, double* d_y, double* d_norm2, void* stream)
{
    CAS_REQUIRE(nnz_per_row > 0 && rows >= 0 && cols >= 0, CAS_ERR_INVALID_ARGUMENT,
                "cas_spmv_norm_noalloc: negative size or nnz_per_row <= 0");
    CAS_REQUIRE(rows <= kNoAllocMaxRows, CAS_ERR_INVALID_ARGUMENT,
                "cas_spmv_norm_noalloc: rows exceeds the fixed scratch capacity of 16,777,216 rows "
                "(2048 rows per CTA x 8192 CTAs); use cas_spmv for larger matrices");
    CAS_REQUIRE(d_norm2 && (rows == 0 || (d_indices && d_x && d_y)), CAS_ERR_INVALID_ARGUMENT,
                "cas_spmv_norm_noalloc: null pointer");
    CAS_TRY(require_device());
    double* scratch = nullptr;
    CAS_TRY(noalloc_scratch(&scratch));
    auto s = static_cast<cudaStream_t>(stream);
    const int ctas = static_cast<int>((rows + kNoAllocRowsPerCta - 1) / kNoAllocRowsPerCta);
    if (ctas > 0) {
        { noalloc_spmv_norm_kernel<<<ctas, kNoAllocThreads, 0, s>>>(d_indices, nnz_per_row, rows, cols, d_x, d_y,
                                                                   scratch); cas::count_launch(); }
        CAS_CHECK_LAUNCH();
    }
    { noalloc_norm_finish_kernel<<<1, 1024, 0, s>>>(scratch, ctas, d_norm2); cas::count_launch(); }
    CAS_CHECK_LAUNCH();
    return CAS_OK;
}

}  // extern "C"
