// The device-resident CSR: construction (indexing, the sort-built transposed
// copy, column statistics) and the products A x, A' y and the Jacobi diagonal.
//
// Layout in HBM for rows R, K entries per row, cols C, nnz = R K:
//   idx       R*K  uint32   row-major column indices (the reference's MatrixCSR)
//   row_idx   nnz  uint32   rows of each entry, sorted by (column, row)
//   col_ptr   C+1  int64    start of each column in row_idx
//   unit_*                  A' y work units (<= kUnit entries of one column)
//   diag_int  C    uint64   diag(A'A), exact integers
#include <algorithm>
#include <vector>

#include "common.cuh"
#include "fast.cuh"
#include "internal.cuh"

namespace cas {

namespace {

// ---------------------------------------------------------------------------
// Exclusive scan of uint32 (totals must stay below 2^32).
// ---------------------------------------------------------------------------
constexpr int kScanThreads = 256;
constexpr int kScanItems = 16;
constexpr int kScanTile = kScanThreads * kScanItems;

__global__ void scan_reduce_kernel(const uint32_t* __restrict__ in, int64_t n, uint32_t* __restrict__ sums)
{
    __shared__ uint32_t s[kScanThreads / 32];
    const int64_t base = static_cast<int64_t>(blockIdx.x) * kScanTile;
    uint32_t acc = 0;
    for (int i = threadIdx.x; i < kScanTile; i += kScanThreads)
        if (base + i < n) acc += in[base + i];
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
    if ((threadIdx.x & 31) == 0) s[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        uint32_t t = 0;
        for (int w = 0; w < kScanThreads / 32; w++) t += s[w];
        sums[blockIdx.x] = t;
    }
}

// Exclusive scan of one tile, plus a per-tile carry-in.
__global__ void scan_tile_kernel(const uint32_t* __restrict__ in, int64_t n, const uint32_t* __restrict__ carry,
                                 uint32_t* __restrict__ out)
{
    __shared__ uint32_t s[kScanThreads];
    const int64_t base = static_cast<int64_t>(blockIdx.x) * kScanTile + static_cast<int64_t>(threadIdx.x) * kScanItems;
    uint32_t v[kScanItems];
    uint32_t local = 0;
#pragma unroll
    for (int i = 0; i < kScanItems; i++) {
        v[i] = base + i < n ? in[base + i] : 0;
        local += v[i];
    }
    s[threadIdx.x] = local;
    __syncthreads();
    for (int o = 1; o < kScanThreads; o <<= 1) {
        uint32_t t = threadIdx.x >= o ? s[threadIdx.x - o] : 0;
        __syncthreads();
        s[threadIdx.x] += t;
        __syncthreads();
    }
    uint32_t run = s[threadIdx.x] - local + (carry ? carry[blockIdx.x] : 0);
#pragma unroll
    for (int i = 0; i < kScanItems; i++) {
        if (base + i < n) out[base + i] = run;
        run += v[i];
    }
}

// Exclusive scan of n uint32 values into out (may alias in).  Returns the
// total through *total_d (device, may be null).
cas_status exclusive_scan(const uint32_t* in, uint32_t* out, int64_t n, cudaStream_t s)
{
    if (n <= 0) return CAS_OK;
    const int64_t tiles = (n + kScanTile - 1) / kScanTile;
    if (tiles == 1) {
        { scan_tile_kernel<<<1, kScanThreads, 0, s>>>(in, n, nullptr, out); cas::count_launch(); }
        CAS_CHECK_LAUNCH();
        return CAS_OK;
    }
    uint32_t* sums = nullptr;
    CAS_CUDA(cudaMallocAsync(&sums, sizeof(uint32_t) * tiles, s));
    { scan_reduce_kernel<<<static_cast<unsigned>(tiles), kScanThreads, 0, s>>>(in, n, sums); cas::count_launch(); }
    CAS_CHECK_LAUNCH();
    cas_status st = exclusive_scan(sums, sums, tiles, s);
    if (st == CAS_OK) {
        { scan_tile_kernel<<<static_cast<unsigned>(tiles), kScanThreads, 0, s>>>(in, n, sums, out); cas::count_launch(); }
        if (cudaGetLastError() != cudaSuccess) st = CAS_ERR_CUDA;
    }
    cudaFreeAsync(sums, s);
    return st;
}

// ---------------------------------------------------------------------------
// Stable LSD radix sort of (key, value) uint32 pairs, 8 bits per pass.
// Pass 0 may take its values implicitly as entry / k (the CSR row), which is
// how the transposed copy is built straight from the row-major indices.
// ---------------------------------------------------------------------------
constexpr int kSortThreads = 256;
constexpr int kSortRounds = 16;
constexpr int kSortTile = kSortThreads * kSortRounds;
constexpr int kRadix = 256;

__global__ void __launch_bounds__(kSortThreads) radix_hist_kernel(const uint32_t* __restrict__ keys, int64_t n,
                                                                  int shift, int64_t tiles,
                                                                  uint32_t* __restrict__ counts)
{
    __shared__ uint32_t h[kRadix];
    for (int64_t tile = blockIdx.x; tile < tiles; tile += gridDim.x) {
        h[threadIdx.x] = 0;
        __syncthreads();
        const int64_t base = tile * kSortTile;
        for (int r = 0; r < kSortRounds; r++) {
            const int64_t i = base + r * kSortThreads + threadIdx.x;
            if (i < n) atomicAdd(&h[(keys[i] >> shift) & (kRadix - 1)], 1u);
        }
        __syncthreads();
        counts[static_cast<int64_t>(threadIdx.x) * tiles + tile] = h[threadIdx.x];
        __syncthreads();
    }
}

__global__ void __launch_bounds__(kSortThreads) radix_scatter_kernel(
    const uint32_t* __restrict__ keys_in, const uint32_t* __restrict__ vals_in, int implicit_k, int64_t n, int shift,
    int64_t tiles, const uint32_t* __restrict__ offsets, uint32_t* __restrict__ keys_out,
    uint32_t* __restrict__ vals_out)
{
    constexpr int kWarps = kSortThreads / 32;
    __shared__ uint32_t base[kRadix], running[kRadix], total[kRadix];
    __shared__ uint32_t wcount[kWarps][kRadix];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const unsigned lt_mask = (1u << lane) - 1;
    for (int64_t tile = blockIdx.x; tile < tiles; tile += gridDim.x) {
        base[threadIdx.x] = offsets[static_cast<int64_t>(threadIdx.x) * tiles + tile];
        running[threadIdx.x] = 0;
        for (int w = 0; w < kWarps; w++) wcount[w][threadIdx.x] = 0;
        __syncthreads();
        for (int r = 0; r < kSortRounds; r++) {
            const int64_t i = tile * kSortTile + r * kSortThreads + threadIdx.x;
            const bool valid = i < n;
            uint32_t key = 0, val = 0;
            if (valid) {
                key = keys_in[i];
                val = vals_in ? vals_in[i] : static_cast<uint32_t>(i / implicit_k);
            }
            const uint32_t d = valid ? (key >> shift) & (kRadix - 1) : 0xFFFFu;
            const unsigned peers = __match_any_sync(0xffffffffu, d);
            const int rank = __popc(peers & lt_mask);
            if (valid && rank == 0) wcount[warp][d] = __popc(peers);
            __syncthreads();
            {
                uint32_t acc = 0;
                for (int w = 0; w < kWarps; w++) {
                    const uint32_t c = wcount[w][threadIdx.x];
                    wcount[w][threadIdx.x] = acc;
                    acc += c;
                }
                total[threadIdx.x] = acc;
            }
            __syncthreads();
            if (valid) {
                const uint32_t pos = base[d] + running[d] + wcount[warp][d] + rank;
                keys_out[pos] = key;
                vals_out[pos] = val;
            }
            __syncthreads();
            running[threadIdx.x] += total[threadIdx.x];
            for (int w = 0; w < kWarps; w++) wcount[w][threadIdx.x] = 0;
            __syncthreads();
        }
    }
}

// Sorts keys/values stably by the low `bits` bits of the key.  keys_in is not
// modified.  The result ends in (*keys_res, *vals_res), which point into
// bufA/bufB.
cas_status radix_sort_pairs(const uint32_t* keys_in, const uint32_t* vals_in, int implicit_k, int64_t n, int bits,
                            uint32_t* keysA, uint32_t* valsA, uint32_t* keysB, uint32_t* valsB,
                            uint32_t** keys_res, uint32_t** vals_res, cudaStream_t s)
{
    const int64_t tiles = (n + kSortTile - 1) / kSortTile;
    const int passes = std::max(1, (bits + 7) / 8);
    uint32_t* counts = nullptr;
    CAS_CUDA(cudaMallocAsync(&counts, sizeof(uint32_t) * kRadix * std::max<int64_t>(tiles, 1), s));
    const unsigned grid = static_cast<unsigned>(std::min<int64_t>(tiles, static_cast<int64_t>(sm_count()) * 8));
    const uint32_t* kin = keys_in;
    const uint32_t* vin = vals_in;
    cas_status st = CAS_OK;
    for (int pass = 0; pass < passes && st == CAS_OK && n > 0; pass++) {
        uint32_t* kout = (pass % 2 == 0) ? keysA : keysB;
        uint32_t* vout = (pass % 2 == 0) ? valsA : valsB;
        { radix_hist_kernel<<<grid, kSortThreads, 0, s>>>(kin, n, pass * 8, tiles, counts); cas::count_launch(); }
        if (cudaGetLastError() != cudaSuccess) {
            st = CAS_ERR_CUDA;
            break;
        }
        st = exclusive_scan(counts, counts, kRadix * tiles, s);
        if (st != CAS_OK) break;
        { radix_scatter_kernel<<<grid, kSortThreads, 0, s>>>(kin, vin, implicit_k, n, pass * 8, tiles, counts, kout,
                                                          vout); cas::count_launch(); }
        if (cudaGetLastError() != cudaSuccess) st = CAS_ERR_CUDA;
        kin = kout;
        vin = vout;
        *keys_res = kout;
        *vals_res = vout;
    }
    cudaFreeAsync(counts, s);
    if (st != CAS_OK) set_error("radix sort: kernel launch failed");
    return st;
}

// ---------------------------------------------------------------------------
// Column structure from the sorted keys.
// ---------------------------------------------------------------------------
__global__ void col_ptr_kernel(const uint32_t* __restrict__ keys, int64_t nnz, int64_t cols,
                               int64_t* __restrict__ col_ptr)
{
    for (int64_t e = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; e <= nnz;
         e += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        const int64_t prev = e > 0 ? static_cast<int64_t>(keys[e - 1]) : -1;
        const int64_t cur = e < nnz ? static_cast<int64_t>(keys[e]) : cols;
        for (int64_t c = prev + 1; c <= cur && c <= cols; c++) col_ptr[c] = e;
    }
}

// diag(A'A)_c = sum over rows of m^2 (m = multiplicity of c in the row),
// accumulated as sum over entries of 2j+1 where j is the entry's position in
// its (column, row) run.  Integer sums: any order gives the same result.
__global__ void diag_kernel(const uint32_t* __restrict__ keys, const uint32_t* __restrict__ rows, int64_t nnz,
                            uint64_t* __restrict__ diag)
{
    const int lane = threadIdx.x & 31;
    for (int64_t e0 = static_cast<int64_t>(blockIdx.x) * blockDim.x; e0 < nnz;
         e0 += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        const int64_t e = e0 + threadIdx.x;
        const bool valid = e < nnz;
        uint32_t c = 0xFFFFFFFFu, contrib = 0;
        if (valid) {
            c = keys[e];
            const uint32_t r = rows[e];
            int64_t j = 0;
            while (e - j - 1 >= 0 && keys[e - j - 1] == c && rows[e - j - 1] == r) j++;
            contrib = static_cast<uint32_t>(2 * j + 1);
        }
        const unsigned peers = __match_any_sync(0xffffffffu, c);
        const uint32_t sum = __reduce_add_sync(peers, contrib);
        if (valid && lane == __ffs(peers) - 1) atomicAdd(reinterpret_cast<unsigned long long*>(diag + c), sum);
    }
}

__global__ void unit_count_kernel(const int64_t* __restrict__ col_ptr, int64_t cols, uint32_t* __restrict__ cnt)
{
    for (int64_t c = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; c < cols;
         c += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        const int64_t len = col_ptr[c + 1] - col_ptr[c];
        cnt[c] = static_cast<uint32_t>(len == 0 ? 1 : (len + kUnit - 1) / kUnit);
    }
}

__global__ void unit_fill_kernel(const uint32_t* __restrict__ unit_ptr, int64_t cols, int32_t* __restrict__ unit_col)
{
    for (int64_t c = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; c < cols;
         c += static_cast<int64_t>(gridDim.x) * blockDim.x)
        for (uint32_t u = unit_ptr[c]; u < unit_ptr[c + 1]; u++) unit_col[u] = static_cast<int32_t>(c);
}

__global__ void bound_check_kernel(const uint32_t* __restrict__ idx, int64_t n, uint32_t cols,
                                   unsigned int* __restrict__ bad)
{
    for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
         i += static_cast<int64_t>(gridDim.x) * blockDim.x)
        if (idx[i] >= cols) atomicOr(bad, 1u);
}

// ---------------------------------------------------------------------------
// Products.
// ---------------------------------------------------------------------------

// y = A x: one warp per row, lanes stride over the row's K indices (a
// coalesced 4K-byte stream), gathers of x summed in FP64, warp-shuffle tree.
template <typename T>
__global__ void __launch_bounds__(256) spmv_kernel(const uint32_t* __restrict__ idx, int64_t rows, int k,
                                                   const T* __restrict__ x, T* __restrict__ y)
{
    const int lane = threadIdx.x & 31;
    const int64_t warps = static_cast<int64_t>(gridDim.x) * (blockDim.x >> 5);
    for (int64_t r = static_cast<int64_t>(blockIdx.x) * (blockDim.x >> 5) + (threadIdx.x >> 5); r < rows;
         r += warps) {
        const uint32_t* row = idx + r * k;
        double acc = 0;
        for (int j = lane; j < k; j += 32) acc += static_cast<double>(__ldg(x + __ldg(row + j)));
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
        if (lane == 0) y[r] = static_cast<T>(acc);
    }
}

// Partial sums of A' y: one warp per work unit.
template <typename T>
__global__ void __launch_bounds__(256) spmv_t_units_kernel(CsrView a, const T* __restrict__ y,
                                                           double* __restrict__ partial)
{
    const int lane = threadIdx.x & 31;
    const int64_t warps = static_cast<int64_t>(gridDim.x) * (blockDim.x >> 5);
    for (int64_t u = static_cast<int64_t>(blockIdx.x) * (blockDim.x >> 5) + (threadIdx.x >> 5); u < a.units;
         u += warps) {
        const int32_t c = a.unit_col[u];
        const int64_t begin = a.col_ptr[c] + static_cast<int64_t>(u - a.unit_ptr[c]) * kUnit;
        const int64_t end = min(a.col_ptr[c + 1], begin + kUnit);
        double acc = 0;
        for (int64_t e = begin + lane; e < end; e += 32) acc += static_cast<double>(__ldg(y + __ldg(a.row_idx + e)));
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
        if (lane == 0) partial[u] = acc;
    }
}

template <typename T>
__global__ void spmv_t_finalize_kernel(CsrView a, const double* __restrict__ partial, T* __restrict__ x)
{
    for (int64_t c = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; c < a.cols;
         c += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        double acc = 0;
        for (uint32_t u = a.unit_ptr[c]; u < a.unit_ptr[c + 1]; u++) acc += partial[u];
        x[c] = static_cast<T>(acc);
    }
}

template <typename T>
__global__ void jacobi_kernel(const uint64_t* __restrict__ diag, int64_t cols, T* __restrict__ out)
{
    for (int64_t c = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; c < cols;
         c += static_cast<int64_t>(gridDim.x) * blockDim.x)
        out[c] = static_cast<T>(1) / static_cast<T>(diag[c]);
}

unsigned grid_for(int64_t work, int per_block)
{
    const int64_t want = (work + per_block - 1) / per_block;
    return static_cast<unsigned>(std::max<int64_t>(1, std::min<int64_t>(want, static_cast<int64_t>(sm_count()) * 16)));
}

}  // namespace

template <typename T>
cas_status spmv(const CsrView& a, const T* x, T* y, cudaStream_t s)
{
    if (a.rows == 0) return CAS_OK;
    { spmv_kernel<T><<<grid_for(a.rows, 8), 256, 0, s>>>(a.idx, a.rows, a.k, x, y); cas::count_launch(); }
    CAS_CHECK_LAUNCH();
    return CAS_OK;
}

template <typename T>
cas_status spmv_t(const CsrView& a, const T* y, double* unit_partial, T* x, cudaStream_t s)
{
    if (a.cols == 0) return CAS_OK;
    { spmv_t_units_kernel<T><<<grid_for(a.units, 8), 256, 0, s>>>(a, y, unit_partial); cas::count_launch(); }
    CAS_CHECK_LAUNCH();
    { spmv_t_finalize_kernel<T><<<grid_for(a.cols, 256), 256, 0, s>>>(a, unit_partial, x); cas::count_launch(); }
    CAS_CHECK_LAUNCH();
    return CAS_OK;
}

template <typename T>
cas_status jacobi(const CsrView& a, T* out, cudaStream_t s)
{
    if (a.cols == 0) return CAS_OK;
    { jacobi_kernel<T><<<grid_for(a.cols, 256), 256, 0, s>>>(a.diag_int, a.cols, out); cas::count_launch(); }
    CAS_CHECK_LAUNCH();
    return CAS_OK;
}

template cas_status spmv<float>(const CsrView&, const float*, float*, cudaStream_t);
template cas_status spmv<double>(const CsrView&, const double*, double*, cudaStream_t);
template cas_status spmv_t<float>(const CsrView&, const float*, double*, float*, cudaStream_t);
template cas_status spmv_t<double>(const CsrView&, const double*, double*, double*, cudaStream_t);
template cas_status jacobi<float>(const CsrView&, float*, cudaStream_t);
template cas_status jacobi<double>(const CsrView&, double*, cudaStream_t);

// Builds the transposed copy, column pointers, work units and diag(A'A) for a
// CSR whose idx array is in place.
cas_status build_structure(cas_csr* a, cudaStream_t s)
{
    const int64_t nnz = a->rows * a->k;
    CAS_REQUIRE(nnz < 0xFFFFFFFFLL, CAS_ERR_INVALID_ARGUMENT,
                "CSR with 2^32 or more entries is not supported (uint32 entry offsets)");
    CAS_REQUIRE(a->rows < 0xFFFFFFFFLL, CAS_ERR_INVALID_ARGUMENT, "rows must fit uint32");
    const int64_t cols = a->cols;
    CAS_CUDA(dmalloc(&a->col_ptr, sizeof(int64_t) * (cols + 1)));
    if (!a->diag_int) {
        CAS_CUDA(dmalloc(&a->diag_int, sizeof(uint64_t) * std::max<int64_t>(cols, 1)));
        CAS_CUDA(cudaMemsetAsync(a->diag_int, 0, sizeof(uint64_t) * std::max<int64_t>(cols, 1), s));
    }

    if (nnz > 0) {
        unsigned int* bad = nullptr;
        CAS_CUDA(cudaMallocAsync(&bad, sizeof(unsigned int), s));
        CAS_CUDA(cudaMemsetAsync(bad, 0, sizeof(unsigned int), s));
        { bound_check_kernel<<<grid_for(nnz, 1024), 256, 0, s>>>(a->idx, nnz, static_cast<uint32_t>(cols), bad); cas::count_launch(); }
        CAS_CHECK_LAUNCH();
        unsigned int hbad = 0;
        CAS_CUDA(cudaMemcpyAsync(&hbad, bad, sizeof hbad, cudaMemcpyDeviceToHost, s));
        CAS_CUDA(cudaStreamSynchronize(s));
        cudaFreeAsync(bad, s);
        CAS_REQUIRE(hbad == 0, CAS_ERR_INVALID_ARGUMENT, "column index >= cols in CSR indices");
    }

    int bits = 1;
    while (bits < 32 && (1LL << bits) < cols) bits++;
    uint32_t *kA = nullptr, *vA = nullptr, *kB = nullptr, *vB = nullptr;
    const size_t bytes = sizeof(uint32_t) * std::max<int64_t>(nnz, 1);
    CAS_CUDA(dmalloc(&kA, bytes));
    CAS_CUDA(dmalloc(&vA, bytes));
    CAS_CUDA(dmalloc(&kB, bytes));
    CAS_CUDA(dmalloc(&vB, bytes));
    uint32_t *keys = kA, *vals = vA;
    cas_status st = CAS_OK;
    if (nnz > 0) st = radix_sort_pairs(a->idx, nullptr, a->k, nnz, bits, kA, vA, kB, vB, &keys, &vals, s);
    if (st == CAS_OK) {
        { col_ptr_kernel<<<grid_for(nnz + 1, 256), 256, 0, s>>>(keys, nnz, cols, a->col_ptr); cas::count_launch(); }
        if (nnz > 0) { diag_kernel<<<grid_for(nnz, 256), 256, 0, s>>>(keys, vals, nnz, a->diag_int); cas::count_launch(); }
        if (cudaGetLastError() != cudaSuccess) st = CAS_ERR_CUDA;
    }
    // keep the sorted rows, release the rest
    a->row_idx = vals;
    for (uint32_t* p : {kA, vA, kB, vB})
        if (p != vals) dfree(p);
    if (st != CAS_OK) return st;

    // A'y work units
    CAS_CUDA(dmalloc(&a->unit_ptr, sizeof(uint32_t) * (cols + 1)));
    if (cols > 0) {
        { unit_count_kernel<<<grid_for(cols, 256), 256, 0, s>>>(a->col_ptr, cols, a->unit_ptr); cas::count_launch(); }
        CAS_CHECK_LAUNCH();
    }
    CAS_CUDA(cudaMemsetAsync(a->unit_ptr + cols, 0, sizeof(uint32_t), s));
    CAS_TRY(exclusive_scan(a->unit_ptr, a->unit_ptr, cols + 1, s));
    uint32_t units = 0;
    CAS_CUDA(cudaMemcpyAsync(&units, a->unit_ptr + cols, sizeof units, cudaMemcpyDeviceToHost, s));
    CAS_CUDA(cudaStreamSynchronize(s));
    a->units = units;
    CAS_CUDA(dmalloc(&a->unit_col, sizeof(int32_t) * std::max<int64_t>(units, 1)));
    CAS_CUDA(dmalloc(&a->unit_partial, sizeof(double) * std::max<int64_t>(units, 1)));
    if (cols > 0) {
        { unit_fill_kernel<<<grid_for(cols, 256), 256, 0, s>>>(a->unit_ptr, cols, a->unit_col); cas::count_launch(); }
        CAS_CHECK_LAUNCH();
    }
    return CAS_OK;
}

}  // namespace cas

using namespace cas;

namespace {
void free_csr(cas_csr* a)
{
    if (!a) return;
    int cur = 0;
    cudaGetDevice(&cur);
    if (a->device >= 0) cudaSetDevice(a->device);
    dfree(a->idx);
    dfree(a->col_ptr);
    dfree(a->row_idx);
    dfree(a->unit_col);
    dfree(a->unit_ptr);
    dfree(a->diag_int);
    dfree(a->unit_partial);
    if (a->fast) {
        fast_free(*a->fast);
        delete a->fast;
    }
    cudaSetDevice(cur);
    delete a;
}

cas_status finish_create(cas_csr* a, cudaStream_t s, cas_csr** out)
{
    cas_status st = build_structure(a, s);
    if (st == CAS_OK) {
        cudaError_t e = cudaStreamSynchronize(s);
        if (e != cudaSuccess) {
            set_error(std::string("CSR build: ") + cudaGetErrorString(e));
            st = CAS_ERR_CUDA;
        }
    }
    if (st != CAS_OK) {
        free_csr(a);
        return st;
    }
    *out = a;
    return CAS_OK;
}
}  // namespace

extern "C" {

CAS_API cas_status cas_csr_from_positions_layout(const cas_patterns* p, const uint64_t* d_positions, int64_t rows,
                                                 int layouts, void* stream, cas_csr** out)
{
    return cas::csr_from_positions(p, d_positions, rows, layouts, static_cast<cudaStream_t>(stream), out, nullptr);
}
}  // extern "C"

cas_status cas::csr_from_positions(const cas_patterns* p, const uint64_t* d_positions, int64_t rows, int layouts,
                                   cudaStream_t s, cas_csr** out, const PositionChunks* chunks)
{
    cas::NvtxRange nvtx_range("cas_csr_from_positions");
    CAS_REQUIRE(p && out && rows >= 0, CAS_ERR_INVALID_ARGUMENT, "cas_csr_from_positions: bad argument");
    CAS_REQUIRE(rows == 0 || d_positions, CAS_ERR_INVALID_ARGUMENT, "cas_csr_from_positions: null positions");
    CAS_REQUIRE((reinterpret_cast<uintptr_t>(d_positions) & 15) == 0, CAS_ERR_INVALID_ARGUMENT,
                "cas_csr_from_positions: position records must be 16-byte aligned");
    CAS_REQUIRE(layouts > 0 && (layouts & ~(CAS_LAYOUT_ROWS | CAS_LAYOUT_BLOCKED)) == 0, CAS_ERR_INVALID_ARGUMENT,
                "cas_csr_from_positions: layouts must be a non-empty mask of cas_layout");
    CAS_REQUIRE(!(layouts & CAS_LAYOUT_BLOCKED) || fast_supported(pattern_set(p)), CAS_ERR_INVALID_ARGUMENT,
                "cas_csr_from_positions: the blocked layout needs index spaces <= 65536 per pattern");
    CAS_REQUIRE(rows * static_cast<int64_t>(cas_patterns_nnz_per_row(p)) < 0xFFFFFFFFLL, CAS_ERR_INVALID_ARGUMENT,
                "cas_csr_from_positions: 2^32 or more entries are not supported");
    *out = nullptr;
    const DevicePatterns* dp = nullptr;
    CAS_TRY(patterns_on_device(p, &dp));
    auto* a = new cas_csr;
    CAS_CUDA(cudaGetDevice(&a->device));
    a->rows = rows;
    a->cols = dp->cols;
    a->k = dp->k;
    a->layouts = layouts;
    cudaError_t e = dmalloc(&a->diag_int, sizeof(uint64_t) * std::max<int64_t>(a->cols, 1));
    if (e == cudaSuccess) e = cudaMemsetAsync(a->diag_int, 0, sizeof(uint64_t) * std::max<int64_t>(a->cols, 1), s);
    if (e != cudaSuccess) {
        free_csr(a);
        set_error("cas_csr_from_positions: cannot allocate the column statistics");
        return CAS_ERR_OUT_OF_MEMORY;
    }
    cas_status st = CAS_OK;
    if (layouts & CAS_LAYOUT_BLOCKED) {
        a->fast = new FastLayout;
        // diag(A'A) comes from the blocked copy unless the row layout builds it
        st = fast_build(*dp, pattern_set(p), d_positions, rows, nullptr, 1,
                        (layouts & CAS_LAYOUT_ROWS) ? nullptr : a->diag_int, *a->fast, s, chunks);
        if (st != CAS_OK) {
            free_csr(a);
            return st;
        }
    }
    if (layouts & CAS_LAYOUT_ROWS) {
        e = dmalloc(&a->idx, sizeof(uint32_t) * std::max<int64_t>(rows * a->k, 1));
        if (e != cudaSuccess) {
            free_csr(a);
            set_error("cas_csr_from_positions: cannot allocate the index array");
            return CAS_ERR_OUT_OF_MEMORY;
        }
        if (chunks && !(layouts & CAS_LAYOUT_BLOCKED))  // the row layout indexes all rows at once
            for (int c = 0; c < chunks->n; c++) CAS_CUDA(cudaStreamWaitEvent(s, chunks->ready[c], 0));
        st = launch_index(*dp, d_positions, rows, a->idx, s);
        if (st != CAS_OK) {
            free_csr(a);
            return st;
        }
        return finish_create(a, s, out);
    }
    e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) {
        free_csr(a);
        set_error(std::string("CSR build: ") + cudaGetErrorString(e));
        return CAS_ERR_CUDA;
    }
    *out = a;
    return CAS_OK;
}

extern "C" {

CAS_API cas_status cas_csr_from_positions_batched(const cas_patterns* p, const uint64_t* d_positions,
                                                  const int64_t* h_problem_rows, int problems, void* stream,
                                                  cas_csr** out)
{
    cas::NvtxRange nvtx_range("cas_csr_from_positions_batched");
    CAS_REQUIRE(p && out && h_problem_rows && problems >= 1 && problems <= kMaxProblems, CAS_ERR_INVALID_ARGUMENT,
                "cas_csr_from_positions_batched: bad argument (1 to 64 problems)");
    CAS_REQUIRE(fast_supported(pattern_set(p)), CAS_ERR_INVALID_ARGUMENT,
                "cas_csr_from_positions_batched: the blocked layout needs index spaces <= 65536 per pattern");
    int64_t rows = 0;
    for (int q = 0; q < problems; q++) {
        CAS_REQUIRE(h_problem_rows[q] >= 0, CAS_ERR_INVALID_ARGUMENT,
                    "cas_csr_from_positions_batched: negative problem size");
        rows += h_problem_rows[q];
    }
    CAS_REQUIRE(rows == 0 || d_positions, CAS_ERR_INVALID_ARGUMENT, "cas_csr_from_positions_batched: null positions");
    CAS_REQUIRE((reinterpret_cast<uintptr_t>(d_positions) & 15) == 0, CAS_ERR_INVALID_ARGUMENT,
                "cas_csr_from_positions_batched: position records must be 16-byte aligned");
    *out = nullptr;
    const DevicePatterns* dp = nullptr;
    CAS_TRY(patterns_on_device(p, &dp));
    auto s = static_cast<cudaStream_t>(stream);
    auto* a = new cas_csr;
    CAS_CUDA(cudaGetDevice(&a->device));
    a->rows = rows;
    a->cols = dp->cols * problems;
    a->k = dp->k;
    a->layouts = CAS_LAYOUT_BLOCKED;
    cudaError_t e = dmalloc(&a->diag_int, sizeof(uint64_t) * std::max<int64_t>(a->cols, 1));
    if (e == cudaSuccess) e = cudaMemsetAsync(a->diag_int, 0, sizeof(uint64_t) * std::max<int64_t>(a->cols, 1), s);
    if (e != cudaSuccess) {
        free_csr(a);
        set_error("cas_csr_from_positions_batched: cannot allocate the column statistics");
        return CAS_ERR_OUT_OF_MEMORY;
    }
    a->fast = new FastLayout;
    cas_status st = fast_build(*dp, pattern_set(p), d_positions, rows, h_problem_rows, problems, a->diag_int,
                               *a->fast, s);
    if (st == CAS_OK) {
        e = cudaStreamSynchronize(s);
        if (e != cudaSuccess) {
            set_error(std::string("batched CSR build: ") + cudaGetErrorString(e));
            st = CAS_ERR_CUDA;
        }
    }
    if (st != CAS_OK) {
        free_csr(a);
        return st;
    }
    *out = a;
    return CAS_OK;
}

CAS_API int cas_csr_problems(const cas_csr* a, int64_t* h_row0)
{
    if (!a) return -1;
    if (!a->fast) {
        if (h_row0) {
            h_row0[0] = 0;
            h_row0[1] = a->rows;
        }
        return 1;
    }
    const FastGeometry& g = a->fast->g;
    if (h_row0)
        for (int q = 0; q <= g.nprob; q++) h_row0[q] = g.prow0[q];
    return g.nprob;
}

CAS_API cas_status cas_csr_from_positions(const cas_patterns* p, const uint64_t* d_positions, int64_t rows,
                                          void* stream, cas_csr** out)
{
    CAS_REQUIRE(p, CAS_ERR_INVALID_ARGUMENT, "cas_csr_from_positions: null pattern set");
    const int layouts = CAS_LAYOUT_ROWS | (fast_supported(pattern_set(p)) ? CAS_LAYOUT_BLOCKED : 0);
    return cas_csr_from_positions_layout(p, d_positions, rows, layouts, stream, out);
}

CAS_API int cas_csr_layouts(const cas_csr* a) { return a ? a->layouts : 0; }

CAS_API int64_t cas_block_rows(void) { return kBlockRows; }

CAS_API int cas_csr_schedules(const cas_csr* a, cas_schedule* out, int max, cas_schedule* in_use)
{
    if (!a || !a->fast) return -1;
    const FastLayout& f = *a->fast;
    if (in_use) {
        in_use->chunks_per_item = f.t32.per_sc;
        in_use->range_major = f.t32.range_major ? 1 : 0;
        in_use->items_per_sm = f.t32.items_per_sm;
        in_use->pack = f.t32.pack ? 1 : 0;
        in_use->persistent = f.t32.persistent ? 1 : 0;
        in_use->ms = 0;
        for (int i = 0; i < f.ntune; i++)
            if (f.tune[i].per_sc == f.t32.per_sc && f.tune[i].range_major == in_use->range_major &&
                f.tune[i].items_per_sm == f.t32.items_per_sm && f.tune[i].pack == in_use->pack &&
                f.tune[i].persistent == in_use->persistent)
                in_use->ms = f.tune[i].ms;
    }
    int n = 0;
    for (int i = 0; i < f.ntune && out && n < max; i++, n++)
        out[n] = cas_schedule{f.tune[i].per_sc, f.tune[i].range_major, f.tune[i].items_per_sm, f.tune[i].pack,
                              f.tune[i].persistent, f.tune[i].ms};
    return n;
}

CAS_API cas_status cas_eval_forward(const cas_csr* a, int64_t row0, int64_t row1, const float* d_w, float* d_score,
                                    void* stream)
{
    CAS_REQUIRE(a && a->fast, CAS_ERR_INVALID_ARGUMENT, "cas_eval_forward: the CSR needs the blocked layout");
    CAS_REQUIRE(0 <= row0 && row0 <= row1 && row1 <= a->rows, CAS_ERR_SIZE_MISMATCH,
                "cas_eval_forward: row range outside the matrix");
    CAS_REQUIRE(row1 == row0 || (d_w && d_score), CAS_ERR_INVALID_ARGUMENT, "cas_eval_forward: null buffer");
    return fast_eval_forward(*a->fast, row0, row1, d_w, d_score, static_cast<cudaStream_t>(stream));
}

CAS_API cas_status cas_eval_backward(const cas_csr* a, int64_t row0, int64_t row1, const float* d_g, float* d_grad,
                                     void* stream)
{
    CAS_REQUIRE(a && a->fast, CAS_ERR_INVALID_ARGUMENT, "cas_eval_backward: the CSR needs the blocked layout");
    CAS_REQUIRE(a->fast->g.nprob == 1, CAS_ERR_INVALID_ARGUMENT,
                "cas_eval_backward: needs the layout of a single fit, not a batch");
    CAS_REQUIRE(0 <= row0 && row0 <= row1 && row1 <= a->rows, CAS_ERR_SIZE_MISMATCH,
                "cas_eval_backward: row range outside the matrix");
    CAS_REQUIRE(row0 % kBlockRows == 0 && (row1 % kBlockRows == 0 || row1 == a->rows), CAS_ERR_INVALID_ARGUMENT,
                "cas_eval_backward: the row range must start and end on block boundaries (cas_block_rows())");
    CAS_REQUIRE(d_grad && (row1 == row0 || d_g), CAS_ERR_INVALID_ARGUMENT, "cas_eval_backward: null buffer");
    const int64_t b0 = row0 / kBlockRows, b1 = (row1 + kBlockRows - 1) / kBlockRows;
    return fast_eval_backward(*a->fast, b0, b1, d_g, d_grad, static_cast<cudaStream_t>(stream));
}

CAS_API cas_status cas_eval_adam_step(const cas_csr* a, int64_t row0, int64_t row1, const float* d_target,
                                      float* d_w, float* d_m, float* d_v, int64_t* d_step, double* d_loss_sum,
                                      const cas_adam_opts* opts, void* stream)
{
    CAS_REQUIRE(a && a->fast, CAS_ERR_INVALID_ARGUMENT, "cas_eval_adam_step: the CSR needs the blocked layout");
    CAS_REQUIRE(a->fast->g.nprob == 1, CAS_ERR_INVALID_ARGUMENT,
                "cas_eval_adam_step: needs the layout of a single fit, not a batch");
    CAS_REQUIRE(0 <= row0 && row0 <= row1 && row1 <= a->rows, CAS_ERR_SIZE_MISMATCH,
                "cas_eval_adam_step: row range outside the matrix");
    CAS_REQUIRE(row0 % kBlockRows == 0 && (row1 % kBlockRows == 0 || row1 == a->rows), CAS_ERR_INVALID_ARGUMENT,
                "cas_eval_adam_step: the row range must start and end on block boundaries (cas_block_rows())");
    CAS_REQUIRE(opts, CAS_ERR_INVALID_ARGUMENT, "cas_eval_adam_step: null options");
    CAS_REQUIRE(row1 == row0 || (d_target && d_w && d_m && d_v && d_step && d_loss_sum), CAS_ERR_INVALID_ARGUMENT,
                "cas_eval_adam_step: null buffer");
    CAS_REQUIRE(opts->lr >= 0 && opts->beta1 >= 0 && opts->beta1 < 1 && opts->beta2 >= 0 && opts->beta2 < 1 &&
                    opts->eps > 0 && opts->l2 >= 0 && opts->delta > 0,
                CAS_ERR_INVALID_ARGUMENT, "cas_eval_adam_step: bad options");
    const EvalAdam o{opts->lr, opts->beta1, opts->beta2, opts->eps, opts->l2, opts->delta};
    return fast_eval_adam_step(*a->fast, row0, row1, d_target, d_w, d_m, d_v, d_step, d_loss_sum, o,
                               static_cast<cudaStream_t>(stream));
}

CAS_API cas_status cas_csr_from_indices(const uint32_t* d_indices, int nnz_per_row, int64_t rows, int64_t cols,
                                        void* stream, cas_csr** out)
{
    CAS_REQUIRE(out && nnz_per_row > 0 && rows >= 0 && cols >= 0, CAS_ERR_INVALID_ARGUMENT,
                "cas_csr_from_indices: bad argument");
    CAS_REQUIRE(rows == 0 || d_indices, CAS_ERR_INVALID_ARGUMENT, "cas_csr_from_indices: null indices");
    CAS_REQUIRE(cols < 0xFFFFFFFFLL, CAS_ERR_INVALID_ARGUMENT, "cas_csr_from_indices: cols must fit uint32");
    *out = nullptr;
    CAS_TRY(require_device());
    auto s = static_cast<cudaStream_t>(stream);
    auto* a = new cas_csr;
    CAS_CUDA(cudaGetDevice(&a->device));
    a->rows = rows;
    a->cols = cols;
    a->k = nnz_per_row;
    a->layouts = CAS_LAYOUT_ROWS;
    const size_t bytes = sizeof(uint32_t) * rows * nnz_per_row;
    cudaError_t e = dmalloc(&a->idx, std::max<size_t>(bytes, 4));
    if (e == cudaSuccess && bytes) e = cudaMemcpyAsync(a->idx, d_indices, bytes, cudaMemcpyDefault, s);
    if (e != cudaSuccess) {
        free_csr(a);
        set_error(std::string("cas_csr_from_indices: ") + cudaGetErrorString(e));
        return e == cudaErrorMemoryAllocation ? CAS_ERR_OUT_OF_MEMORY : CAS_ERR_CUDA;
    }
    return finish_create(a, s, out);
}

CAS_API void cas_csr_destroy(cas_csr* a) { free_csr(a); }
CAS_API int64_t cas_csr_rows(const cas_csr* a) { return a ? a->rows : -1; }
CAS_API int64_t cas_csr_cols(const cas_csr* a) { return a ? a->cols : -1; }
CAS_API int cas_csr_nnz_per_row(const cas_csr* a) { return a ? a->k : -1; }
CAS_API const uint32_t* cas_csr_indices(const cas_csr* a) { return a ? a->idx : nullptr; }

CAS_API cas_status cas_csr_transposed(const cas_csr* a, const int64_t** d_col_ptr, const uint32_t** d_row_idx)
{
    CAS_REQUIRE(a, CAS_ERR_INVALID_ARGUMENT, "cas_csr_transposed: null handle");
    if (d_col_ptr) *d_col_ptr = a->col_ptr;
    if (d_row_idx) *d_row_idx = a->row_idx;
    return CAS_OK;
}

CAS_API cas_status cas_spmv(const cas_csr* a, cas_dtype dtype, const void* d_x, void* d_y, void* stream)
{
    CAS_REQUIRE(a, CAS_ERR_INVALID_ARGUMENT, "cas_spmv: null handle");
    CAS_REQUIRE((d_x || a->cols == 0) && (d_y || a->rows == 0), CAS_ERR_INVALID_ARGUMENT, "cas_spmv: null vector");
    auto s = static_cast<cudaStream_t>(stream);
    if (a->fast && (dtype == CAS_F32 || dtype == CAS_F64)) {
        if (dtype == CAS_F32)
            return fast_spmv<float, float>(*a->fast, static_cast<const float*>(d_x), static_cast<float*>(d_y), nullptr,
                                           nullptr, nullptr, nullptr, 0, s, nullptr);
        return fast_spmv<double, double>(*a->fast, static_cast<const double*>(d_x), static_cast<double*>(d_y), nullptr,
                                         nullptr, nullptr, nullptr, 0, s, nullptr);
    }
    if (dtype == CAS_F32) return spmv<float>(a->view(), static_cast<const float*>(d_x), static_cast<float*>(d_y), s);
    if (dtype == CAS_F64)
        return spmv<double>(a->view(), static_cast<const double*>(d_x), static_cast<double*>(d_y), s);
    set_error("cas_spmv: unknown dtype");
    return CAS_ERR_INVALID_ARGUMENT;
}

CAS_API cas_status cas_spmv_t(const cas_csr* a, cas_dtype dtype, const void* d_y, void* d_x, void* stream)
{
    CAS_REQUIRE(a, CAS_ERR_INVALID_ARGUMENT, "cas_spmv_t: null handle");
    CAS_REQUIRE((d_y || a->rows == 0) && (d_x || a->cols == 0), CAS_ERR_INVALID_ARGUMENT, "cas_spmv_t: null vector");
    auto s = static_cast<cudaStream_t>(stream);
    if (a->fast && dtype == CAS_F32)
        return fast_spmv_t<float>(*a->fast, static_cast<const float*>(d_y), static_cast<float*>(d_x), s);
    if (a->fast && dtype == CAS_F64)
        return fast_spmv_t<double>(*a->fast, static_cast<const double*>(d_y), static_cast<double*>(d_x), s);
    if (dtype == CAS_F32)
        return spmv_t<float>(a->view(), static_cast<const float*>(d_y), a->unit_partial, static_cast<float*>(d_x), s);
    if (dtype == CAS_F64)
        return spmv_t<double>(a->view(), static_cast<const double*>(d_y), a->unit_partial, static_cast<double*>(d_x),
                              s);
    set_error("cas_spmv_t: unknown dtype");
    return CAS_ERR_INVALID_ARGUMENT;
}

CAS_API cas_status cas_jacobi(const cas_csr* a, cas_dtype dtype, void* d_out, void* stream)
{
    CAS_REQUIRE(a && (d_out || a->cols == 0), CAS_ERR_INVALID_ARGUMENT, "cas_jacobi: null argument");
    auto s = static_cast<cudaStream_t>(stream);
    if (dtype == CAS_F32) return jacobi<float>(a->view(), static_cast<float*>(d_out), s);
    if (dtype == CAS_F64) return jacobi<double>(a->view(), static_cast<double*>(d_out), s);
    set_error("cas_jacobi: unknown dtype");
    return CAS_ERR_INVALID_ARGUMENT;
}

}  // extern "C"
