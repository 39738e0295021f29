// Blocked pattern layout: build (indexing straight into the layout, a
// per-block column sort for the transposed copy, chunk pointers, diag(A'A))
// and the two products.  See fast.cuh for the layout.
//
// A x   one CTA per row block (1024 threads, 16 rows each).  For every pattern
//       the CTA copies that pattern's slice of x (up to 224 KB) into shared
//       memory and every thread gathers its rows' entries from there; the
//       uint16 index stream is read once, coalesced (16 B per row and
//       pattern).  HBM traffic: 2 B per entry + the output.
// A'y   one CTA per work item (a column chunk of one pattern x a range of row
//       blocks).  Per block the CTA stages y's block slice in shared memory,
//       streams the chunk's column-sorted entries (4 B each, coalesced),
//       gathers y from shared memory and reduces each run of equal columns
//       with a deterministic segmented scan into a shared-memory accumulator
//       of the chunk.  Items write partial column sums that the caller adds
//       in a fixed order: no atomics anywhere, bitwise reproducible.
#include <algorithm>
#include <vector>

#include "common.cuh"
#include "fast.cuh"
#include "indexer.cuh"

namespace cas {

namespace {

constexpr int kSortThreads = 1024;
constexpr int kSortWarps = kSortThreads / 32;
constexpr int kItemsPerThread = 16;  // A'y entries per thread and round (a multiple of 8)

unsigned fgrid(int64_t work, int per)
{
    const int64_t want = (work + per - 1) / per;
    return static_cast<unsigned>(std::max<int64_t>(1, std::min<int64_t>(want, static_cast<int64_t>(sm_count()) * 4)));
}

// ---------------------------------------------------------------------------
// Indexing into the blocked layout: one thread per row, all patterns.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256) fast_index_kernel(const Instance* __restrict__ g_inst, int k,
                                                         const uint32_t* __restrict__ tables,
                                                         const ulonglong2* __restrict__ pos, FastGeometry g,
                                                         uint16_t* __restrict__ a16)
{
    extern __shared__ Instance s_inst[];
    for (int i = threadIdx.x; i < k; i += blockDim.x) s_inst[i] = g_inst[i];
    __syncthreads();
    for (int64_t r = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; r < g.rows;
         r += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        const ulonglong2 ps = pos[r];
        const uint32_t plo = static_cast<uint32_t>(ps.x), phi = static_cast<uint32_t>(ps.x >> 32);
        const uint32_t olo = static_cast<uint32_t>(ps.y), ohi = static_cast<uint32_t>(ps.y >> 32);
        const int64_t b = r / kBlockRows, rb = r - b * kBlockRows;
        for (int p = 0; p < g.npat; p++) {
            const int s0 = g.slot0[p], ns = g.slots[p];
            const uint32_t off = static_cast<uint32_t>(g.off[p]);
            uint32_t v[8];
#pragma unroll
            for (int s = 0; s < 8; s++)
                v[s] = s < ns ? eval_slot(s_inst[s0 + s], tables, plo, phi, olo, ohi) - off : 0u;
            uint16_t* dst = a16 + g.seg(b, p) + rb * ns;
            if (ns == 8) {
                *reinterpret_cast<uint4*>(dst) =
                    make_uint4(v[0] | (v[1] << 16), v[2] | (v[3] << 16), v[4] | (v[5] << 16), v[6] | (v[7] << 16));
            } else if (ns == 4) {
                *reinterpret_cast<uint2*>(dst) = make_uint2(v[0] | (v[1] << 16), v[2] | (v[3] << 16));
            } else if (ns == 2) {
                *reinterpret_cast<uint32_t*>(dst) = v[0] | (v[1] << 16);
            } else {
                *dst = static_cast<uint16_t>(v[0]);
            }
        }
    }
}

// ---------------------------------------------------------------------------
// Per-(block, pattern) stable sort of entries by local column: two 8-bit LSD
// passes inside one CTA, through a per-CTA scratch slice (L2 resident).
// Items are (column << 16) | row-in-block; the input order is row-major
// (row, slot), so equal columns keep ascending rows.
// ---------------------------------------------------------------------------
struct SortSmem {
    uint32_t hist[256];
    uint32_t base[256];
    uint32_t running[256];
    uint32_t total[256];
    uint32_t wcount[kSortWarps][256];
};

__device__ void block_exclusive_scan_256(uint32_t* hist, uint32_t* out)
{
    // 256 values scanned by the first 8 warps; others idle.
    __shared__ uint32_t warp_tot[8];
    const int t = threadIdx.x;
    uint32_t v = 0, incl = 0;
    if (t < 256) {
        v = hist[t];
        incl = v;
        const int lane = t & 31;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t u = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += u;
        }
        if (lane == 31) warp_tot[t >> 5] = incl;
    }
    __syncthreads();
    if (t < 256) {
        uint32_t pre = 0;
        for (int w = 0; w < (t >> 5); w++) pre += warp_tot[w];
        out[t] = pre + incl - v;
    }
    __syncthreads();
}

template <bool FROM_A16>
__device__ void sort_pass(const uint16_t* __restrict__ a16_in, const uint32_t* __restrict__ in, int n, int slots,
                          int shift, uint32_t* __restrict__ out, SortSmem& sm)
{
    const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
    const unsigned lt_mask = (1u << lane) - 1;
    auto item_at = [&](int e) -> uint32_t {
        if (FROM_A16) return (static_cast<uint32_t>(a16_in[e]) << 16) | static_cast<uint32_t>(e / slots);
        return in[e];
    };
    if (t < 256) sm.hist[t] = 0;
    for (int w = 0; w < kSortWarps; w++)
        if (t < 256) sm.wcount[w][t] = 0;
    __syncthreads();
    for (int e = t; e < n; e += kSortThreads) atomicAdd(&sm.hist[(item_at(e) >> shift) & 255u], 1u);
    __syncthreads();
    block_exclusive_scan_256(sm.hist, sm.base);
    if (t < 256) sm.running[t] = 0;
    __syncthreads();
    for (int r0 = 0; r0 < n; r0 += kSortThreads) {
        const int e = r0 + t;
        const bool valid = e < n;
        const uint32_t item = valid ? item_at(e) : 0u;
        const uint32_t d = valid ? (item >> shift) & 255u : 0xFFFFu;
        const unsigned peers = __match_any_sync(0xffffffffu, d);
        const int rank = __popc(peers & lt_mask);
        if (valid && rank == 0) sm.wcount[warp][d] = __popc(peers);
        __syncthreads();
        if (t < 256) {
            uint32_t acc = 0;
            for (int w = 0; w < kSortWarps; w++) {
                const uint32_t c = sm.wcount[w][t];
                sm.wcount[w][t] = acc;
                acc += c;
            }
            sm.total[t] = acc;
        }
        __syncthreads();
        if (valid) out[sm.base[d] + sm.running[d] + sm.wcount[warp][d] + rank] = item;
        __syncthreads();
        if (t < 256) {
            sm.running[t] += sm.total[t];
            for (int w = 0; w < kSortWarps; w++) sm.wcount[w][t] = 0;
        }
        __syncthreads();
    }
}

__global__ void __launch_bounds__(kSortThreads, 1) fast_sort_kernel(FastGeometry g, const uint16_t* __restrict__ a16,
                                                                   uint32_t* __restrict__ g32,
                                                                   uint32_t* __restrict__ scratch)
{
    __shared__ SortSmem sm;
    uint32_t* mine = scratch + static_cast<int64_t>(blockIdx.x) * kBlockRows * 8;
    const int64_t groups = g.nblocks * g.npat;
    for (int64_t grp = blockIdx.x; grp < groups; grp += gridDim.x) {
        const int64_t b = grp / g.npat;
        const int p = static_cast<int>(grp - b * g.npat);
        const int n = static_cast<int>(g.seg_len(b, p));
        const int64_t seg = g.seg(b, p);
        sort_pass<true>(a16 + seg, nullptr, n, g.slots[p], 16, mine, sm);
        sort_pass<false>(nullptr, mine, n, g.slots[p], 24, g32 + seg, sm);
    }
}

// First entry of every (block, chunk) in G32: lower bound of the chunk's
// first column in the sorted group.
__global__ void fast_chunk_kernel(FastGeometry g, const uint32_t* __restrict__ g32, uint32_t* __restrict__ chunk_start)
{
    const int64_t total = g.nblocks * g.nchunks;
    for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < total;
         i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        const int64_t b = i / g.nchunks;
        const int ch = static_cast<int>(i - b * g.nchunks);
        int p = 0;
        while (p + 1 < g.npat && g.chunk0[p + 1] <= ch) p++;
        const uint32_t c0 = static_cast<uint32_t>(ch - g.chunk0[p]) * kChunkCols;
        const int64_t seg = g.seg(b, p);
        int64_t lo = 0, hi = g.seg_len(b, p);
        while (lo < hi) {
            const int64_t mid = (lo + hi) >> 1;
            if ((g32[seg + mid] >> 16) < c0)
                lo = mid + 1;
            else
                hi = mid;
        }
        chunk_start[i] = static_cast<uint32_t>(seg + lo);
    }
}

// diag(A'A)_c = sum over rows of m^2: inside a sorted group equal
// (column, row) pairs are adjacent, so the j-th copy contributes 2j+1.
__global__ void fast_diag_kernel(FastGeometry g, const uint32_t* __restrict__ g32, uint64_t* __restrict__ diag)
{
    const int lane = threadIdx.x & 31;
    const int64_t groups = g.nblocks * g.npat;
    for (int64_t grp = blockIdx.x; grp < groups; grp += gridDim.x) {
        const int64_t b = grp / g.npat;
        const int p = static_cast<int>(grp - b * g.npat);
        const int64_t seg = g.seg(b, p), n = g.seg_len(b, p);
        for (int64_t e0 = 0; e0 < n; e0 += blockDim.x) {
            const int64_t e = e0 + threadIdx.x;
            uint32_t col = 0xFFFFFFFFu, contrib = 0;
            if (e < n) {
                const uint32_t v = g32[seg + e];
                int64_t j = 0;
                while (e - j - 1 >= 0 && g32[seg + e - j - 1] == v) j++;
                col = v >> 16;
                contrib = static_cast<uint32_t>(2 * j + 1);
            }
            const unsigned peers = __match_any_sync(0xffffffffu, col);
            const uint32_t sum = __reduce_add_sync(peers, contrib);
            if (e < n && lane == __ffs(peers) - 1)
                atomicAdd(reinterpret_cast<unsigned long long*>(diag + g.off[p] + col), sum);
        }
    }
}

// ---------------------------------------------------------------------------
// A x on the blocked layout.
// ---------------------------------------------------------------------------
template <typename T>
struct AccOf {
    using type = float;
};
template <>
struct AccOf<double> {
    using type = double;
};

template <typename T>
__device__ __forceinline__ void gather_row(const uint16_t* __restrict__ src, int ns, const T* __restrict__ table,
                                           const T* __restrict__ xg, int cap, bool all_in_table,
                                           typename AccOf<T>::type& acc)
{
    uint32_t w[4];
    if (ns == 8) {
        const uint4 u = *reinterpret_cast<const uint4*>(src);
        w[0] = u.x, w[1] = u.y, w[2] = u.z, w[3] = u.w;
    } else if (ns == 4) {
        const uint2 u = *reinterpret_cast<const uint2*>(src);
        w[0] = u.x, w[1] = u.y;
    } else if (ns == 2) {
        w[0] = *reinterpret_cast<const uint32_t*>(src);
    } else {
        w[0] = *src;
    }
#pragma unroll
    for (int s = 0; s < 8; s++) {
        if (s < ns) {
            const uint32_t c = (w[s >> 1] >> ((s & 1) * 16)) & 0xFFFFu;
            acc += static_cast<typename AccOf<T>::type>(all_in_table || static_cast<int>(c) < cap ? table[c]
                                                                                               : __ldg(xg + c));
        }
    }
}

// One index word (two 16-bit columns) of a row gathered into acc.
template <typename T, bool ALL_IN>
__device__ __forceinline__ void gather_word(uint32_t wd, const T* __restrict__ table, const T* __restrict__ xg,
                                            int cap, typename AccOf<T>::type& acc)
{
    using Acc = typename AccOf<T>::type;
    const int c0 = static_cast<int>(wd & 0xFFFFu), c1 = static_cast<int>(wd >> 16);
    acc += static_cast<Acc>(ALL_IN || c0 < cap ? table[c0] : __ldg(xg + c0));
    acc += static_cast<Acc>(ALL_IN || c1 < cap ? table[c1] : __ldg(xg + c1));
}

// Scalar stores of one 16-byte vector (the destination need not be aligned).
__device__ __forceinline__ void store_vec(float* d, uint4 u)
{
    d[0] = __uint_as_float(u.x);
    d[1] = __uint_as_float(u.y);
    d[2] = __uint_as_float(u.z);
    d[3] = __uint_as_float(u.w);
}
__device__ __forceinline__ void store_vec(double* d, uint4 u)
{
    d[0] = __hiloint2double(static_cast<int>(u.y), static_cast<int>(u.x));
    d[1] = __hiloint2double(static_cast<int>(u.w), static_cast<int>(u.z));
}

// Copies a pattern's slice of x (cap entries) into shared memory with
// 16-byte loads, several in flight per thread.
template <typename T>
__device__ __forceinline__ void load_table(T* __restrict__ table, const T* __restrict__ xg, int cap)
{
    constexpr int kPer = 16 / sizeof(T);
    const int mis = static_cast<int>((reinterpret_cast<uintptr_t>(xg) & 15) / sizeof(T));
    const int head = min(cap, mis ? kPer - mis : 0);
    if (static_cast<int>(threadIdx.x) < head) table[threadIdx.x] = xg[threadIdx.x];
    const int nvec = (cap - head) / kPer;
    const uint4* src = reinterpret_cast<const uint4*>(xg + head);
    T* dst = table + head;
    for (int v0 = threadIdx.x; v0 < nvec; v0 += 4 * blockDim.x) {
        uint4 u[4];
#pragma unroll
        for (int k = 0; k < 4; k++) {
            const int v = v0 + k * blockDim.x;
            if (v < nvec) u[k] = __ldg(src + v);
        }
#pragma unroll
        for (int k = 0; k < 4; k++) {
            const int v = v0 + k * blockDim.x;
            if (v < nvec) store_vec(dst + v * kPer, u[k]);
        }
    }
    const int done = head + nvec * kPer;
    for (int i = done + threadIdx.x; i < cap; i += blockDim.x) table[i] = xg[i];
}

// Rows of one 8-slot pattern segment (the expanded layout): each thread owns
// kAxRows rows (stride kAxThreads); the 16-byte index word of row j+kAxAhead
// is loaded while row j is gathered, so kAxAhead loads per thread stay in
// flight.
template <typename T, bool ALL_IN>
__device__ __forceinline__ void gather_segment8(const uint16_t* __restrict__ base, int nb,
                                                const T* __restrict__ table, const T* __restrict__ xg, int cap,
                                                typename AccOf<T>::type (&acc)[kAxRows])
{
    uint4 w[kAxAhead];
#pragma unroll
    for (int j = 0; j < kAxAhead; j++) {
        const int r = threadIdx.x + j * kAxThreads;
        w[j] = r < nb ? *reinterpret_cast<const uint4*>(base + static_cast<int64_t>(r) * 8) : make_uint4(0, 0, 0, 0);
    }
#pragma unroll
    for (int j = 0; j < kAxRows; j++) {
        const uint4 cur = w[j % kAxAhead];
        if (j + kAxAhead < kAxRows) {
            const int rn = threadIdx.x + (j + kAxAhead) * kAxThreads;
            w[j % kAxAhead] = rn < nb ? *reinterpret_cast<const uint4*>(base + static_cast<int64_t>(rn) * 8)
                                      : make_uint4(0, 0, 0, 0);
        }
        const int r = threadIdx.x + j * kAxThreads;
        if (r < nb) {
            gather_word<T, ALL_IN>(cur.x, table, xg, cap, acc[j]);
            gather_word<T, ALL_IN>(cur.y, table, xg, cap, acc[j]);
            gather_word<T, ALL_IN>(cur.z, table, xg, cap, acc[j]);
            gather_word<T, ALL_IN>(cur.w, table, xg, cap, acc[j]);
        }
    }
}

// ALL8: every pattern has 8 slots (the expanded layout), so only the
// pipelined 8-slot path is compiled in.
template <typename T, typename Y, int MODE, bool ALL8>
__global__ void __launch_bounds__(kAxThreads, 1) fast_spmv_kernel(FastGeometry g, const uint16_t* __restrict__ a16,
                                                                   const T* __restrict__ x, Y* __restrict__ y,
                                                                   const double* __restrict__ b,
                                                                   const double* __restrict__ coef,
                                                                   double* __restrict__ part,
                                                                   const int* __restrict__ done)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T* table = reinterpret_cast<T*>(smem_raw);
    __shared__ double red[64];
    if (done && *(volatile const int*)done) return;
    constexpr int kCap = sizeof(T) == 4 ? kTable32 : kTable64;
    using Acc = typename AccOf<T>::type;
    const double c = MODE == 1 ? *coef : 0.0;
    Comp mine;
    for (int64_t blk = blockIdx.x; blk < g.nblocks; blk += gridDim.x) {
        const int nb = static_cast<int>(g.block_rows(blk));
        Acc acc[kAxRows];
#pragma unroll
        for (int j = 0; j < kAxRows; j++) acc[j] = 0;
        for (int p = 0; p < g.npat; p++) {
            const int cap = min(g.space[p], kCap);
            const T* xg = x + g.off[p];
            __syncthreads();
            load_table<T>(table, xg, cap);
            __syncthreads();
            const uint16_t* base = a16 + g.seg(blk, p);
            const bool all_in = g.space[p] <= kCap;
            const int ns = g.slots[p];
            if (ALL8 || ns == 8) {
                if (all_in)
                    gather_segment8<T, true>(base, nb, table, xg, cap, acc);
                else
                    gather_segment8<T, false>(base, nb, table, xg, cap, acc);
            } else if (!ALL8) {
#pragma unroll
                for (int j = 0; j < kAxRows; j++) {
                    const int r = threadIdx.x + j * kAxThreads;
                    if (r < nb) gather_row<T>(base + static_cast<int64_t>(r) * ns, ns, table, xg, cap, all_in, acc[j]);
                }
            }
        }
#pragma unroll
        for (int j = 0; j < kAxRows; j++) {
            const int r = threadIdx.x + j * kAxThreads;
            if (r < nb) {
                const int64_t row = blk * kBlockRows + r;
                double v = static_cast<double>(acc[j]);
                if (MODE == 1) v = static_cast<double>(y[row]) * -c + v;
                if (MODE == 2) v = (b ? b[row] : 0.0) - v;
                const Y yv = static_cast<Y>(v);
                y[row] = yv;
                mine.add(static_cast<double>(yv) * static_cast<double>(yv));
            }
        }
    }
    if (part) {
        const Comp r = block_sum_comp<kAxThreads>(mine, red);
        if (threadIdx.x == 0) {
            part[2 * blockIdx.x] = r.s;
            part[2 * blockIdx.x + 1] = r.c;
        }
    }
}

// ---------------------------------------------------------------------------
// A'y on the blocked layout.
// ---------------------------------------------------------------------------
struct TView {
    int per_sc;
    const int* item_sc;
    const int* item_b0;
    const int* item_b1;
    const int64_t* item_part;
    int sc_base[kMaxFastPatterns + 1];
};

template <typename T>
struct SegSmem {
    T warp_v[32];
    int warp_f[32];
    T warp_excl[32];
    T carry;
};

// Segmented reduction of one round of column-sorted entries into acc.
// Each thread owns kItemsPerThread consecutive entries of [e_lo, e_hi); runs
// of equal columns are summed and added to acc[col] exactly once, in an
// order fixed by the data, so the result is bitwise reproducible:
//   1. each thread sums its runs; runs wholly inside the thread are added to
//      acc directly (no other thread touches that column in this tile);
//   2. the partial runs at thread boundaries are combined by a segmented
//      scan: shuffles inside each warp, then warp 0 scans the 32 warp
//      aggregates; the chain entering the round (an open run of the previous
//      round) is ss.carry;
//   3. the thread where a boundary run ends adds the combined sum.
// round_start is a multiple of 4 entries, so every thread reads its
// entries with 16-byte loads.
template <typename T>
__device__ __forceinline__ void run_step(uint32_t e, uint32_t c0, const T* __restrict__ ytile, T* __restrict__ acc,
                                         int& hc, int& tc, T& hs, T& sum, bool& single, bool& any)
{
    const int col = static_cast<int>((e >> 16) - c0);
    const T v = ytile[e & 0xFFFFu];
    if (!any) {
        any = true;
        hc = tc = col;
        sum = v;
    } else if (col == tc) {
        sum += v;
    } else {
        if (single) {
            hs = sum;  // the head run closes inside this thread
            single = false;
        } else {
            acc[tc] += sum;  // interior run: only this thread touches tc
        }
        tc = col;
        sum = v;
    }
}

template <typename T>
__device__ void seg_round(const uint32_t* __restrict__ g32, uint32_t round_start, uint32_t e_lo, uint32_t e_hi,
                          uint32_t c0, const T* __restrict__ ytile, T* __restrict__ acc, SegSmem<T>& ss)
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const uint32_t e_first = round_start + threadIdx.x * kItemsPerThread;
    int hc = -1, tc = -1;
    T hs = 0, sum = 0;
    bool single = true, any = false;
    const bool full = e_first >= e_lo && e_first + kItemsPerThread <= e_hi;
    uint32_t first_ent = 0, last_ent = 0;
    if (full) {
        // every entry valid: 16-byte loads, no per-entry checks
#pragma unroll
        for (int q = 0; q < kItemsPerThread / 4; q++) {
            const uint4 u = *reinterpret_cast<const uint4*>(g32 + e_first + 4 * q);
            if (q == 0) first_ent = u.x;
            if (q == kItemsPerThread / 4 - 1) last_ent = u.w;
            run_step<T>(u.x, c0, ytile, acc, hc, tc, hs, sum, single, any);
            run_step<T>(u.y, c0, ytile, acc, hc, tc, hs, sum, single, any);
            run_step<T>(u.z, c0, ytile, acc, hc, tc, hs, sum, single, any);
            run_step<T>(u.w, c0, ytile, acc, hc, tc, hs, sum, single, any);
        }
    } else if (e_first + kItemsPerThread > e_lo && e_first < e_hi) {
        const uint32_t lo = max(e_first, e_lo), hi = min(e_first + kItemsPerThread, e_hi);
        first_ent = g32[lo];
        last_ent = g32[hi - 1];
        for (uint32_t e = lo; e < hi; e++) run_step<T>(g32[e], c0, ytile, acc, hc, tc, hs, sum, single, any);
    }
    const T ts = sum;
    if (single) hs = sum;
    // neighbours: the previous thread's last entry and the next thread's
    // first entry, by shuffle inside the warp, from memory at warp edges
    const uint32_t first_valid = max(e_first, e_lo);
    const uint32_t last_valid = min(e_first + kItemsPerThread, e_hi) - 1;
    const uint32_t prev_ent_sh = __shfl_up_sync(0xffffffffu, last_ent, 1);
    const uint32_t next_ent_sh = __shfl_down_sync(0xffffffffu, first_ent, 1);
    const bool prev_any = __shfl_up_sync(0xffffffffu, any, 1);
    const bool next_any = __shfl_down_sync(0xffffffffu, any, 1);
    bool cont_prev = false, cont_next = false;
    if (any) {
        if (first_valid > e_lo) {
            const uint32_t pe = (lane > 0 && prev_any) ? prev_ent_sh : g32[first_valid - 1];
            cont_prev = static_cast<int>((pe >> 16) - c0) == hc;
        }
        if (last_valid + 1 < e_hi) {
            const uint32_t ne = (lane < 31 && next_any) ? next_ent_sh : g32[last_valid + 1];
            cont_next = static_cast<int>((ne >> 16) - c0) == tc;
        }
    }
    // segmented inclusive scan of tail partials over threads: a thread joins
    // the previous chain when its whole range is one run that continues it.
    T v = any ? ts : T(0);
    bool f = !(any && single && cont_prev);
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        const T vu = __shfl_up_sync(0xffffffffu, v, d);
        const bool fu = __shfl_up_sync(0xffffffffu, f, d);
        if (lane >= d) {
            if (!f) v += vu;
            f = f || fu;
        }
    }
    if (lane == 31) {
        ss.warp_v[warp] = v;
        ss.warp_f[warp] = f;
    }
    __syncthreads();
    if (warp == 0) {
        // same scan over the warp aggregates, seeded with the round's carry
        constexpr int kWarps = kFastThreads / 32;
        T wv = lane < kWarps ? ss.warp_v[lane] : T(0);
        bool wf = lane < kWarps ? ss.warp_f[lane] != 0 : true;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            const T vu = __shfl_up_sync(0xffffffffu, wv, d);
            const bool fu = __shfl_up_sync(0xffffffffu, wf, d);
            if (lane >= d) {
                if (!wf) wv += vu;
                wf = wf || fu;
            }
        }
        const T carry = ss.carry;
        const T incl = wf ? wv : wv + carry;  // chain value at the end of warp `lane`
        T excl = __shfl_up_sync(0xffffffffu, incl, 1);
        if (lane == 0) excl = carry;
        if (lane < kWarps) ss.warp_excl[lane] = excl;
        if (lane == kWarps - 1) ss.carry = incl;  // open chain leaving the round
    }
    __syncthreads();
    const T excl_w = ss.warp_excl[warp];
    const T X = f ? v : v + excl_w;  // chain value ending at this thread
    T Xprev = __shfl_up_sync(0xffffffffu, X, 1);
    if (lane == 0) Xprev = excl_w;
    if (any) {
        if (single) {
            if (!cont_next) acc[hc] += X;
        } else {
            acc[hc] += cont_prev ? Xprev + hs : hs;
            if (!cont_next) acc[tc] += ts;
        }
    }
    __syncthreads();
}

template <typename T>
__global__ void __launch_bounds__(kFastThreads, 1) fast_spmv_t_kernel(FastGeometry g, TView tv,
                                                                       const uint32_t* __restrict__ g32,
                                                                       const uint32_t* __restrict__ chunk_start,
                                                                       const T* __restrict__ y,
                                                                       T* __restrict__ partial,
                                                                       const int* __restrict__ done, int item_base,
                                                                       int64_t y_block0)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ SegSmem<T> ss;
    if (done && *(volatile const int*)done) return;
    const int width_max = kChunkCols * tv.per_sc;
    T* acc = reinterpret_cast<T*>(smem_raw);
    T* ytile = acc + width_max;
    const int item = blockIdx.x + item_base;
    const int sc = tv.item_sc[item];
    int p = 0;
    while (p + 1 < g.npat && tv.sc_base[p + 1] <= sc) p++;
    const int pat_chunks = (p + 1 < g.npat ? g.chunk0[p + 1] : g.nchunks) - g.chunk0[p];
    const int ch0_local = (sc - tv.sc_base[p]) * tv.per_sc;
    const int ch1_local = min(ch0_local + tv.per_sc, pat_chunks);
    const int ch0 = g.chunk0[p] + ch0_local;
    const uint32_t c0 = static_cast<uint32_t>(ch0_local) * kChunkCols;
    const int width = min(g.space[p], ch1_local * kChunkCols) - static_cast<int>(c0);
    for (int i = threadIdx.x; i < width; i += kFastThreads) acc[i] = 0;
    for (int64_t blk = tv.item_b0[item]; blk < tv.item_b1[item]; blk++) {
        const int nb = static_cast<int>(g.block_rows(blk));
        __syncthreads();
        const T* yb = y + (blk - y_block0) * kBlockRows;
        for (int i = threadIdx.x; i < nb; i += kFastThreads) ytile[i] = yb[i];
        if (threadIdx.x == 0) ss.carry = 0;
        __syncthreads();
        const uint32_t e_lo = chunk_start[blk * g.nchunks + ch0];
        const uint32_t e_hi = ch1_local < pat_chunks
                                  ? chunk_start[blk * g.nchunks + g.chunk0[p] + ch1_local]
                                  : static_cast<uint32_t>(g.seg(blk, p) + g.seg_len(blk, p));
        for (uint32_t rs = e_lo & ~3u; rs < e_hi; rs += kFastThreads * kItemsPerThread)
            seg_round<T>(g32, rs, e_lo, e_hi, c0, ytile, acc, ss);
    }
    __syncthreads();
    T* out = partial + (tv.item_part[item] - tv.item_part[item_base]);
    for (int i = threadIdx.x; i < width; i += kFastThreads) out[i] = acc[i];
}

// Evaluator forward on a row range: score[r - row0] = sum_j w[col_rj], one
// thread per row, 16-byte index loads, gathers of w through L1/L2 (the range
// is a minibatch, too short to amortise staging w in shared memory).
__global__ void __launch_bounds__(256) fast_rows_forward_kernel(FastGeometry g, const uint16_t* __restrict__ a16,
                                                                const float* __restrict__ w, int64_t row0,
                                                                int64_t row1, float* __restrict__ out)
{
    for (int64_t r = row0 + static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; r < row1;
         r += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        const int64_t b = r / kBlockRows, rb = r - b * kBlockRows;
        float acc = 0;
        for (int p = 0; p < g.npat; p++)
            gather_row<float>(a16 + g.seg(b, p) + rb * g.slots[p], g.slots[p], w + g.off[p], w + g.off[p], 0, false,
                              acc);
        out[r - row0] = acc;
    }
}

// Dense column sums of per-block partials laid out [block][cols].
__global__ void block_partial_sum_kernel(const float* __restrict__ partial, int nb, int64_t cols,
                                         float* __restrict__ out)
{
    for (int64_t c = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; c < cols;
         c += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        float acc = 0;
        for (int j = 0; j < nb; j++) acc += partial[static_cast<int64_t>(j) * cols + c];
        out[c] = acc;
    }
}

template <typename T>
__global__ void fast_col_sum_kernel(FastCols fc, const T* __restrict__ partial, T* __restrict__ x)
{
    for (int64_t c = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; c < fc.g.cols;
         c += static_cast<int64_t>(gridDim.x) * blockDim.x)
        x[c] = static_cast<T>(fast_col_sum<T>(fc, partial, c));
}

// Builds the work list of one A'y variant from the entry counts per (block,
// chunk): super-chunks of per_sc chunks, each split into block ranges so that
// items carry about equal numbers of entries.
cas_status build_items(const FastGeometry& g, const std::vector<int64_t>& entries_bc, int per_sc, size_t elem,
                       FastTranspose& t)
{
    t.per_sc = per_sc;
    std::vector<int> sc_pat;
    int nsc = 0;
    for (int p = 0; p < g.npat; p++) {
        t.sc_base[p] = nsc;
        const int pch = (p + 1 < g.npat ? g.chunk0[p + 1] : g.nchunks) - g.chunk0[p];
        const int n = (pch + per_sc - 1) / per_sc;
        for (int i = 0; i < n; i++) sc_pat.push_back(p);
        nsc += n;
    }
    t.sc_base[g.npat] = nsc;
    t.nsc = nsc;
    // entries per super-chunk
    std::vector<int64_t> sc_entries(nsc, 0);
    int64_t total = 0;
    for (int64_t b = 0; b < g.nblocks; b++)
        for (int ch = 0; ch < g.nchunks; ch++) {
            int p = 0;
            while (p + 1 < g.npat && g.chunk0[p + 1] <= ch) p++;
            const int sc = t.sc_base[p] + (ch - g.chunk0[p]) / per_sc;
            sc_entries[sc] += entries_bc[b * g.nchunks + ch];
            total += entries_bc[b * g.nchunks + ch];
        }
    const int64_t target_items = static_cast<int64_t>(sm_count()) * 2;
    const double per_item = std::max<double>(1.0, static_cast<double>(total) / target_items);
    std::vector<int> item_sc, item_b0, item_b1, sc_item0;
    std::vector<int64_t> item_part;
    int64_t part_elems = 0;
    for (int sc = 0; sc < nsc; sc++) {
        sc_item0.push_back(static_cast<int>(item_sc.size()));
        const int p = sc_pat[sc];
        const int pch = (p + 1 < g.npat ? g.chunk0[p + 1] : g.nchunks) - g.chunk0[p];
        const int c0l = (sc - t.sc_base[p]) * per_sc;
        const int width = std::min<int>(g.space[p], std::min(c0l + per_sc, pch) * kChunkCols) - c0l * kChunkCols;
        int64_t n = static_cast<int64_t>(std::llround(sc_entries[sc] / per_item));
        n = std::max<int64_t>(1, std::min<int64_t>(n, g.nblocks));
        for (int64_t i = 0; i < n; i++) {
            item_sc.push_back(sc);
            item_b0.push_back(static_cast<int>(g.nblocks * i / n));
            item_b1.push_back(static_cast<int>(g.nblocks * (i + 1) / n));
            item_part.push_back(part_elems);
            part_elems += width;
        }
    }
    sc_item0.push_back(static_cast<int>(item_sc.size()));
    t.nitems = static_cast<int>(item_sc.size());
    CAS_CUDA(cudaMalloc(&t.item_sc, sizeof(int) * t.nitems));
    CAS_CUDA(cudaMalloc(&t.item_b0, sizeof(int) * t.nitems));
    CAS_CUDA(cudaMalloc(&t.item_b1, sizeof(int) * t.nitems));
    CAS_CUDA(cudaMalloc(&t.item_part, sizeof(int64_t) * t.nitems));
    CAS_CUDA(cudaMalloc(&t.sc_item0, sizeof(int) * (nsc + 1)));
    CAS_CUDA(cudaMalloc(&t.partial, elem * std::max<int64_t>(part_elems, 1)));
    CAS_CUDA(cudaMemcpy(t.item_sc, item_sc.data(), sizeof(int) * t.nitems, cudaMemcpyHostToDevice));
    CAS_CUDA(cudaMemcpy(t.item_b0, item_b0.data(), sizeof(int) * t.nitems, cudaMemcpyHostToDevice));
    CAS_CUDA(cudaMemcpy(t.item_b1, item_b1.data(), sizeof(int) * t.nitems, cudaMemcpyHostToDevice));
    CAS_CUDA(cudaMemcpy(t.item_part, item_part.data(), sizeof(int64_t) * t.nitems, cudaMemcpyHostToDevice));
    CAS_CUDA(cudaMemcpy(t.sc_item0, sc_item0.data(), sizeof(int) * (nsc + 1), cudaMemcpyHostToDevice));
    return CAS_OK;
}

// Work list of one item per (block, chunk), block-major, for adjoints over a
// block range (minibatches): item b * nchunks + ch; partial offsets give the
// layout [block][global column] relative to the first item of the range.
cas_status build_block_items(const FastGeometry& g, FastTranspose& t)
{
    t.per_sc = 1;
    for (int p = 0; p < g.npat; p++) t.sc_base[p] = g.chunk0[p];
    t.sc_base[g.npat] = g.nchunks;
    t.nsc = g.nchunks;
    const int64_t n = g.nblocks * g.nchunks;
    t.nitems = static_cast<int>(n);
    std::vector<int> isc(n), ib0(n), ib1(n);
    std::vector<int64_t> ipart(n);
    for (int64_t b = 0; b < g.nblocks; b++)
        for (int ch = 0; ch < g.nchunks; ch++) {
            int p = 0;
            while (p + 1 < g.npat && g.chunk0[p + 1] <= ch) p++;
            const int64_t i = b * g.nchunks + ch;
            isc[i] = ch;
            ib0[i] = static_cast<int>(b);
            ib1[i] = static_cast<int>(b + 1);
            ipart[i] = b * g.cols + g.off[p] + static_cast<int64_t>(ch - g.chunk0[p]) * kChunkCols;
        }
    CAS_CUDA(cudaMalloc(&t.item_sc, sizeof(int) * n));
    CAS_CUDA(cudaMalloc(&t.item_b0, sizeof(int) * n));
    CAS_CUDA(cudaMalloc(&t.item_b1, sizeof(int) * n));
    CAS_CUDA(cudaMalloc(&t.item_part, sizeof(int64_t) * n));
    CAS_CUDA(cudaMemcpy(t.item_sc, isc.data(), sizeof(int) * n, cudaMemcpyHostToDevice));
    CAS_CUDA(cudaMemcpy(t.item_b0, ib0.data(), sizeof(int) * n, cudaMemcpyHostToDevice));
    CAS_CUDA(cudaMemcpy(t.item_b1, ib1.data(), sizeof(int) * n, cudaMemcpyHostToDevice));
    CAS_CUDA(cudaMemcpy(t.item_part, ipart.data(), sizeof(int64_t) * n, cudaMemcpyHostToDevice));
    return CAS_OK;
}

TView tview(const FastTranspose& t)
{
    TView v;
    v.per_sc = t.per_sc;
    v.item_sc = t.item_sc;
    v.item_b0 = t.item_b0;
    v.item_b1 = t.item_b1;
    v.item_part = t.item_part;
    for (int i = 0; i <= kMaxFastPatterns; i++) v.sc_base[i] = t.sc_base[i];
    return v;
}

template <typename T>
const FastTranspose& transpose_of(const FastLayout& f)
{
    return sizeof(T) == 4 ? f.t32 : f.t64;
}

template <typename T>
size_t spmv_t_smem(const FastTranspose& t)
{
    return sizeof(T) * (static_cast<size_t>(kChunkCols) * t.per_sc + kBlockRows);
}

void free_transpose(FastTranspose& t)
{
    cudaFree(t.item_sc);
    cudaFree(t.item_b0);
    cudaFree(t.item_b1);
    cudaFree(t.item_part);
    cudaFree(t.sc_item0);
    cudaFree(t.partial);
    t = FastTranspose{};
}

// Opt-in shared memory for every product kernel (set outside any stream
// capture, at build time).
cas_status fast_set_attributes()
{
    const int s32 = static_cast<int>(sizeof(float) * kTable32), s64 = static_cast<int>(sizeof(double) * kTable64);
    const int t32 = static_cast<int>(sizeof(float) * (static_cast<size_t>(kChunkCols) * 4 + kBlockRows));
    const int t64 = static_cast<int>(sizeof(double) * (static_cast<size_t>(kChunkCols) * 1 + kBlockRows));
    const auto attr = cudaFuncAttributeMaxDynamicSharedMemorySize;
    CAS_CUDA(cudaFuncSetAttribute(fast_spmv_kernel<float, float, 0, true>, attr, s32));
    CAS_CUDA(cudaFuncSetAttribute(fast_spmv_kernel<float, float, 0, false>, attr, s32));
    CAS_CUDA(cudaFuncSetAttribute(fast_spmv_kernel<float, float, 1, true>, attr, s32));
    CAS_CUDA(cudaFuncSetAttribute(fast_spmv_kernel<float, float, 1, false>, attr, s32));
    CAS_CUDA(cudaFuncSetAttribute(fast_spmv_kernel<float, float, 2, true>, attr, s32));
    CAS_CUDA(cudaFuncSetAttribute(fast_spmv_kernel<float, float, 2, false>, attr, s32));
    CAS_CUDA(cudaFuncSetAttribute(fast_spmv_kernel<double, double, 0, true>, attr, s64));
    CAS_CUDA(cudaFuncSetAttribute(fast_spmv_kernel<double, double, 0, false>, attr, s64));
    CAS_CUDA(cudaFuncSetAttribute(fast_spmv_kernel<double, double, 1, true>, attr, s64));
    CAS_CUDA(cudaFuncSetAttribute(fast_spmv_kernel<double, double, 1, false>, attr, s64));
    CAS_CUDA(cudaFuncSetAttribute(fast_spmv_kernel<double, double, 2, true>, attr, s64));
    CAS_CUDA(cudaFuncSetAttribute(fast_spmv_kernel<double, double, 2, false>, attr, s64));
    CAS_CUDA(cudaFuncSetAttribute(fast_spmv_kernel<double, float, 0, true>, attr, s64));
    CAS_CUDA(cudaFuncSetAttribute(fast_spmv_kernel<double, float, 0, false>, attr, s64));
    CAS_CUDA(cudaFuncSetAttribute(fast_spmv_kernel<double, float, 1, true>, attr, s64));
    CAS_CUDA(cudaFuncSetAttribute(fast_spmv_kernel<double, float, 1, false>, attr, s64));
    CAS_CUDA(cudaFuncSetAttribute(fast_spmv_kernel<double, float, 2, true>, attr, s64));
    CAS_CUDA(cudaFuncSetAttribute(fast_spmv_kernel<double, float, 2, false>, attr, s64));
    CAS_CUDA(cudaFuncSetAttribute(fast_spmv_t_kernel<float>, attr, t32));
    CAS_CUDA(cudaFuncSetAttribute(fast_spmv_t_kernel<double>, attr, t64));
    return CAS_OK;
}

}  // namespace

bool fast_supported(const PatternSet& ps)
{
    if (ps.indexers.empty() || static_cast<int>(ps.indexers.size()) > kMaxFastPatterns) return false;
    for (const IndexerInfo& in : ps.indexers) {
        if (in.space > 65536) return false;
        if (in.order != 1 && in.order != 2 && in.order != 4 && in.order != 8) return false;
    }
    return true;
}

void fast_free(FastLayout& f)
{
    cudaFree(f.a16);
    cudaFree(f.g32);
    cudaFree(f.chunk_start);
    free_transpose(f.t32);
    free_transpose(f.t64);
    free_transpose(f.tb);
    cudaFree(f.eval_partial);
    f = FastLayout{};
}

cas_status fast_build(const DevicePatterns& dp, const PatternSet& ps, const uint64_t* d_pos, int64_t rows,
                      uint64_t* diag_int, FastLayout& f, cudaStream_t s)
{
    CAS_REQUIRE(fast_supported(ps), CAS_ERR_INVALID_ARGUMENT, "pattern set does not fit the blocked layout");
    FastGeometry& g = f.g;
    g = FastGeometry{};
    g.npat = static_cast<int>(ps.indexers.size());
    g.k = dp.k;
    g.rows = rows;
    g.cols = ps.cols;
    g.nblocks = (rows + kBlockRows - 1) / kBlockRows;
    int slot = 0, chunk = 0;
    for (int p = 0; p < g.npat; p++) {
        g.slot0[p] = slot;
        g.slots[p] = ps.indexers[p].order;
        g.off[p] = ps.indexers[p].offset;
        g.space[p] = static_cast<int>(ps.indexers[p].space);
        g.chunk0[p] = chunk;
        slot += g.slots[p];
        chunk += (g.space[p] + kChunkCols - 1) / kChunkCols;
    }
    g.nchunks = chunk;
    const int64_t elems = std::max<int64_t>(g.total_elems(), 8);
    CAS_CUDA(cudaMalloc(&f.a16, sizeof(uint16_t) * elems));
    CAS_CUDA(cudaMalloc(&f.g32, sizeof(uint32_t) * elems));
    CAS_CUDA(cudaMalloc(&f.chunk_start, sizeof(uint32_t) * std::max<int64_t>(g.nblocks * g.nchunks, 1)));
    if (rows > 0) {
        const int threads = 256;
        const unsigned grid = fgrid(rows, threads);
        { fast_index_kernel<<<grid * 4, threads, sizeof(Instance) * dp.k, s>>>(
            dp.instances, dp.k, dp.tables, reinterpret_cast<const ulonglong2*>(d_pos), g, f.a16); cas::count_launch(); }
        CAS_CHECK_LAUNCH();
        const int64_t groups = g.nblocks * g.npat;
        const unsigned sgrid = static_cast<unsigned>(std::min<int64_t>(groups, static_cast<int64_t>(sm_count())));
        uint32_t* scratch = nullptr;
        CAS_CUDA(cudaMallocAsync(&scratch, sizeof(uint32_t) * kBlockRows * 8 * sgrid, s));
        { fast_sort_kernel<<<sgrid, kSortThreads, 0, s>>>(g, f.a16, f.g32, scratch); cas::count_launch(); }
        CAS_CHECK_LAUNCH();
        cudaFreeAsync(scratch, s);
        { fast_chunk_kernel<<<fgrid(g.nblocks * g.nchunks, 256), 256, 0, s>>>(g, f.g32, f.chunk_start); cas::count_launch(); }
        CAS_CHECK_LAUNCH();
        if (diag_int) {
            { fast_diag_kernel<<<std::min<unsigned>(static_cast<unsigned>(groups), sm_count() * 8), 256, 0, s>>>(
                g, f.g32, diag_int); cas::count_launch(); }
            CAS_CHECK_LAUNCH();
        }
    }
    // entries per (block, chunk) -> work items
    std::vector<uint32_t> cs(static_cast<size_t>(g.nblocks * g.nchunks));
    if (!cs.empty()) {
        CAS_CUDA(cudaMemcpyAsync(cs.data(), f.chunk_start, sizeof(uint32_t) * cs.size(), cudaMemcpyDeviceToHost, s));
        CAS_CUDA(cudaStreamSynchronize(s));
    }
    std::vector<int64_t> entries(cs.size(), 0);
    for (int64_t b = 0; b < g.nblocks; b++)
        for (int p = 0; p < g.npat; p++) {
            const int c_end = p + 1 < g.npat ? g.chunk0[p + 1] : g.nchunks;
            for (int ch = g.chunk0[p]; ch < c_end; ch++) {
                const int64_t lo = cs[b * g.nchunks + ch];
                const int64_t hi = ch + 1 < c_end ? static_cast<int64_t>(cs[b * g.nchunks + ch + 1])
                                                  : g.seg(b, p) + g.seg_len(b, p);
                entries[b * g.nchunks + ch] = hi - lo;
            }
        }
    if (g.nblocks > 0) {
        CAS_TRY(build_items(g, entries, 4, sizeof(float), f.t32));
        CAS_TRY(build_items(g, entries, 1, sizeof(double), f.t64));
        CAS_TRY(build_block_items(g, f.tb));
    }
    return fast_set_attributes();
}

cas_status fast_diag(const FastLayout& f, uint64_t* diag, cudaStream_t s)
{
    const int64_t groups = f.g.nblocks * f.g.npat;
    if (groups == 0) return CAS_OK;
    { fast_diag_kernel<<<std::min<unsigned>(static_cast<unsigned>(groups), sm_count() * 8), 256, 0, s>>>(f.g, f.g32, diag); cas::count_launch(); }
    CAS_CHECK_LAUNCH();
    return CAS_OK;
}

template <typename T, typename Y>
cas_status fast_spmv(const FastLayout& f, const T* x, Y* y, const double* b, const double* coef, double* part,
                     int* done_flag, int mode, cudaStream_t s, int* n_parts)
{
    const unsigned grid = static_cast<unsigned>(std::max<int64_t>(1, std::min<int64_t>(f.g.nblocks, sm_count())));
    if (n_parts) *n_parts = static_cast<int>(grid);
    if (f.g.nblocks == 0) return CAS_OK;
    const size_t smem = sizeof(T) * (sizeof(T) == 4 ? kTable32 : kTable64);
    auto launch = [&](auto kern) -> cas_status {
        { kern<<<grid, kAxThreads, smem, s>>>(f.g, f.a16, x, y, b, coef, part, done_flag); cas::count_launch(); }
        CAS_CHECK_LAUNCH();
        return CAS_OK;
    };
    bool all8 = true;
    for (int p = 0; p < f.g.npat; p++) all8 = all8 && f.g.slots[p] == 8;
    if (all8) {
        if (mode == 0) return launch(fast_spmv_kernel<T, Y, 0, true>);
        if (mode == 1) return launch(fast_spmv_kernel<T, Y, 1, true>);
        return launch(fast_spmv_kernel<T, Y, 2, true>);
    }
    if (mode == 0) return launch(fast_spmv_kernel<T, Y, 0, false>);
    if (mode == 1) return launch(fast_spmv_kernel<T, Y, 1, false>);
    return launch(fast_spmv_kernel<T, Y, 2, false>);
}

template <typename T>
cas_status fast_spmv_t_partials(const FastLayout& f, const T* y, int* done_flag, cudaStream_t s)
{
    const FastTranspose& t = transpose_of<T>(f);
    if (t.nitems == 0) return CAS_OK;
    const size_t smem = spmv_t_smem<T>(t);
    { fast_spmv_t_kernel<T><<<t.nitems, kFastThreads, smem, s>>>(f.g, tview(t), f.g32, f.chunk_start, y,
                                                                static_cast<T*>(t.partial), done_flag, 0, 0); cas::count_launch(); }
    CAS_CHECK_LAUNCH();
    return CAS_OK;
}

template <typename T>
FastCols fast_cols(const FastLayout& f)
{
    const FastTranspose& t = transpose_of<T>(f);
    FastCols c;
    c.g = f.g;
    c.per_sc = t.per_sc;
    c.sc_item0 = t.sc_item0;
    c.item_part = t.item_part;
    for (int i = 0; i <= kMaxFastPatterns; i++) c.sc_base[i] = t.sc_base[i];
    return c;
}

template <typename T>
cas_status fast_spmv_t(const FastLayout& f, const T* y, T* x, cudaStream_t s)
{
    CAS_TRY(fast_spmv_t_partials<T>(f, y, nullptr, s));
    const FastTranspose& t = transpose_of<T>(f);
    if (f.g.cols == 0) return CAS_OK;
    if (t.nitems == 0) {
        CAS_CUDA(cudaMemsetAsync(x, 0, sizeof(T) * f.g.cols, s));
        return CAS_OK;
    }
    { fast_col_sum_kernel<T><<<fgrid(f.g.cols, 256), 256, 0, s>>>(fast_cols<T>(f), static_cast<const T*>(t.partial), x); cas::count_launch(); }
    CAS_CHECK_LAUNCH();
    return CAS_OK;
}

cas_status fast_eval_forward(const FastLayout& f, int64_t row0, int64_t row1, const float* w, float* score,
                             cudaStream_t s)
{
    if (row1 <= row0) return CAS_OK;
    { fast_rows_forward_kernel<<<fgrid(row1 - row0, 256) * 4, 256, 0, s>>>(f.g, f.a16, w, row0, row1, score); cas::count_launch(); }
    CAS_CHECK_LAUNCH();
    return CAS_OK;
}

cas_status fast_eval_backward(FastLayout& f, int64_t b0, int64_t b1, const float* g, float* grad, cudaStream_t s)
{
    const int64_t nb = b1 - b0;
    if (f.g.cols == 0) return CAS_OK;
    if (nb <= 0) {
        CAS_CUDA(cudaMemsetAsync(grad, 0, sizeof(float) * f.g.cols, s));
        return CAS_OK;
    }
    if (nb > f.eval_blocks) {
        if (f.eval_partial) {
            CAS_CUDA(cudaStreamSynchronize(s));
            cudaFree(f.eval_partial);
            f.eval_partial = nullptr;
        }
        CAS_CUDA(cudaMalloc(&f.eval_partial, sizeof(float) * nb * f.g.cols));
        f.eval_blocks = nb;
    }
    const size_t smem = sizeof(float) * (static_cast<size_t>(kChunkCols) + kBlockRows);
    const int items = static_cast<int>(nb * f.g.nchunks);
    { fast_spmv_t_kernel<float><<<items, kFastThreads, smem, s>>>(f.g, tview(f.tb), f.g32, f.chunk_start, g,
                                                                 f.eval_partial, nullptr,
                                                                 static_cast<int>(b0 * f.g.nchunks), b0); cas::count_launch(); }
    CAS_CHECK_LAUNCH();
    { block_partial_sum_kernel<<<fgrid(f.g.cols, 256), 256, 0, s>>>(f.eval_partial, static_cast<int>(nb), f.g.cols,
                                                                  grad); cas::count_launch(); }
    CAS_CHECK_LAUNCH();
    return CAS_OK;
}

template cas_status fast_spmv<float, float>(const FastLayout&, const float*, float*, const double*, const double*,
                                            double*, int*, int, cudaStream_t, int*);
template cas_status fast_spmv<double, double>(const FastLayout&, const double*, double*, const double*,
                                              const double*, double*, int*, int, cudaStream_t, int*);
template cas_status fast_spmv<double, float>(const FastLayout&, const double*, float*, const double*, const double*,
                                             double*, int*, int, cudaStream_t, int*);
template cas_status fast_spmv_t_partials<float>(const FastLayout&, const float*, int*, cudaStream_t);
template cas_status fast_spmv_t_partials<double>(const FastLayout&, const double*, int*, cudaStream_t);
template FastCols fast_cols<float>(const FastLayout&);
template FastCols fast_cols<double>(const FastLayout&);
template cas_status fast_spmv_t<float>(const FastLayout&, const float*, float*, cudaStream_t);
template cas_status fast_spmv_t<double>(const FastLayout&, const double*, double*, cudaStream_t);

}  // namespace cas
