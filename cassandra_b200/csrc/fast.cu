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
#include <cstring>
#include <cstdio>
#include <cstdlib>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "common.cuh"
#include "fast.cuh"
#include "indexer.cuh"

namespace cas {

namespace {

constexpr int kSortThreads = 256;  // a sort pass's round is kSortThreads items (at least 256: one thread per digit)
constexpr int kSortWarps = kSortThreads / 32;
constexpr int kSortCtasPerSm = 4;  // groups sorted at once per SM: their barriers and scans overlap
// The A'y accumulator of a work item holds at most kMaxSc column chunks
// (with the y tile, the FP32 kernel's dynamic shared memory: 192 KB).  The
// build-time autotuner picks the schedule (accumulator width, items per SM,
// packing of narrow patterns, persistent CTAs).
constexpr int kMaxSc = 4;
constexpr int64_t kBatchItemBlocks = 4;  // most row blocks of one A'y work item in a batched layout
constexpr int64_t kBatchSmallBlocks = 8;  // batched problems this small get one block per A'y item

unsigned fgrid(int64_t work, int per)
{
    const int64_t want = (work + per - 1) / per;
    return static_cast<unsigned>(std::max<int64_t>(1, std::min<int64_t>(want, static_cast<int64_t>(sm_count()) * 4)));
}

// ---------------------------------------------------------------------------
// Indexing into the blocked layout: one thread per row, all patterns.
// ---------------------------------------------------------------------------
constexpr int kIndexThreads = 256;
constexpr int kIndexBoardBytes = 64 * kIndexThreads;  // one digit board per thread

// A16 of rows [r_begin, r_end): one thread per row, whose 64 cells go to a
// digit board first, so that every square of every instance costs one
// shared-memory byte load and a multiply-add.
__global__ void __launch_bounds__(kIndexThreads) fast_index_kernel(const Instance* __restrict__ g_inst, int k,
                                                         const uint32_t* __restrict__ tables,
                                                         const ulonglong2* __restrict__ pos, FastGeometry g,
                                                         uint16_t* __restrict__ a16, int64_t r_begin, int64_t r_end)
{
    extern __shared__ __align__(16) unsigned char s_raw[];
    // the digit boards of the CTA's rows, then the instances
    uint8_t* board = s_raw + threadIdx.x;
    Instance* s_inst = reinterpret_cast<Instance*>(s_raw + kIndexBoardBytes);
    for (int i = threadIdx.x; i < k; i += blockDim.x) s_inst[i] = g_inst[i];
    __syncthreads();
    for (int64_t r = r_begin + static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; r < r_end;
         r += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        const ulonglong2 ps = pos[r];
        fill_board<kIndexThreads>(board, static_cast<uint32_t>(ps.x), static_cast<uint32_t>(ps.x >> 32),
                                  static_cast<uint32_t>(ps.y), static_cast<uint32_t>(ps.y >> 32));
        int64_t b, rb;
        g.locate_row(r, b, rb);
        for (int p = 0; p < g.npat; p++) {
            const int s0 = g.slot0[p], ns = g.slots[p];
            const uint32_t off = static_cast<uint32_t>(g.off[p]);
            uint32_t v[8];
#pragma unroll
            for (int s = 0; s < 8; s++)
                v[s] = s < ns ? eval_slot_board<kIndexThreads>(s_inst[s0 + s], tables, board) - off : 0u;
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
// passes inside one CTA, the first into a per-CTA scratch slice.  Items are
// (column << 16) | (row-in-block << 2) | end, end (bit 0) set on the last
// entry of each column; the input order is row-major (row, slot), so equal
// columns keep ascending rows.
//
// A pass moves its items in tiles of kSortTile: each warp ranks its 512
// items by digit (peers from ballots, in item order, counts per digit in shared
// memory), one scan per tile turns the warps' counts into offsets, the tile
// is scattered digit by digit into a shared buffer and written out from
// there, so that consecutive threads write the consecutive output positions
// of a digit's run.  The final pass writes G32's round order and the end
// flags: an entry ends its run when the next entry of its digit in the tile
// has another column; the last entry of a digit in a tile waits (position
// and column kept per digit) for the digit's first entry in a later tile,
// or for the pass's end (the next entry then has another digit).
// ---------------------------------------------------------------------------
constexpr int kSortPerThread = 16;                           // items per thread and tile
constexpr int kSortTile = kSortThreads * kSortPerThread;     // items per tile
constexpr int kSortWarpItems = 32 * kSortPerThread;          // items a warp ranks per tile
constexpr uint32_t kNoPend = 0xFFFFFFFFu;
constexpr int kSortPrefetchPieces = kSortTile * 4 / 4096;  // 4 KB pieces of a tile of 4-byte items

struct SortSmem {
    uint32_t hist[256];     // digit counts of the first pass (counted from the input)
    uint32_t hist2[256];    // digit counts of the final pass (counted by the first pass's write-out)
    uint32_t base[256];     // first output position of each digit
    uint32_t running[256];  // entries of each digit written by earlier tiles
    uint32_t tcount[256];   // the tile's entries of each digit
    uint32_t tbase[256];    // the digit's first slot in the tile buffer
    uint32_t pend_pos[256]; // final pass: the digit's last entry so far (kNoPend: none)
    uint32_t pend_col[256]; //   and its column
    uint32_t dst[256];      // output position of the tile buffer's slot 0 for the digit (mod 2^32)
    uint32_t tend[256];     // end of the digit's slots in the tile buffer
    uint32_t wcnt[kSortWarps][256];
    uint32_t buf[kSortTile];
};

__device__ void block_exclusive_scan_256(const uint32_t* hist, uint32_t* out)
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

// The lanes of the warp whose valid 8-bit digit equals this lane's (from
// eight ballots: no match instruction, which costs far more here).  Only
// meaningful on valid lanes.
__device__ __forceinline__ unsigned digit_peers(uint32_t d, bool valid)
{
    unsigned peers = __ballot_sync(0xffffffffu, valid);
#pragma unroll
    for (int b = 0; b < 8; b++) {
        const bool bit = (d >> b) & 1u;
        const unsigned m = __ballot_sync(0xffffffffu, bit);
        peers &= bit ? m : ~m;
    }
    return peers;
}

// One stable 8-bit counting-sort pass of a group's n items by the digit at
// `shift`.  FROM_A16: the first pass, items made from the A16 segment
// (local column << 16 | row << 2), written to out in sorted order while the
// final pass's digit counts are gathered.  !FROM_A16: the final pass, items
// read from `in`, written in G32's round order (round_phys of the sorted
// position; out starts on a round boundary) with their end flags.
template <bool FROM_A16>
__device__ void sort_pass(const uint16_t* __restrict__ a16_in, const uint32_t* __restrict__ in, int n, int slots,
                          int shift, uint32_t* __restrict__ out, SortSmem& sm)
{
    constexpr bool FINAL = !FROM_A16;
    const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
    const unsigned lt_mask = (1u << lane) - 1;
    auto item_at = [&](int e) -> uint32_t {
        if (FROM_A16) return (static_cast<uint32_t>(a16_in[e]) << 16) | (static_cast<uint32_t>(e / slots) << 2);
        return in[e];
    };
    if (FROM_A16) {
        // the digits (low column bytes) of the group, 8 columns per 16-byte
        // load (segments start on 1024-entry rounds), the last n % 8 one by
        // one
        if (t < 256) sm.hist[t] = 0;
        __syncthreads();
        const uint4* v = reinterpret_cast<const uint4*>(a16_in);
        for (int e = (n & ~7) + t; e < n; e += kSortThreads) atomicAdd(&sm.hist[a16_in[e] & 255u], 1u);
        for (int i = t; i < n / 8; i += kSortThreads) {
            const uint4 u = __ldcs(v + i);
            const uint32_t w[4] = {u.x, u.y, u.z, u.w};
#pragma unroll
            for (int q = 0; q < 8; q++) atomicAdd(&sm.hist[(w[q >> 1] >> (16 * (q & 1))) & 255u], 1u);
        }
        __syncthreads();
    }
    block_exclusive_scan_256(FROM_A16 ? sm.hist : sm.hist2, sm.base);
    if (t < 256) {
        sm.running[t] = 0;
        if (FROM_A16) sm.hist2[t] = 0;
        sm.pend_pos[t] = kNoPend;
    }
    for (int t0 = 0; t0 < n; t0 += kSortTile) {
        // the next tile's input into L2 while this one is ranked, in 4 KB
        // pieces rounded up to 16 bytes (inside the group's room: whole
        // rounds of A16, whole tiles of the scratch slice)
        if (t < kSortPrefetchPieces) {
            const int nt = t0 + kSortTile;
            const int64_t bytes = static_cast<int64_t>(min(kSortTile, n - nt)) * (FROM_A16 ? 2 : 4);
            const int64_t lo = static_cast<int64_t>(t) * 4096;
            if (nt < n && lo < bytes) {
                const char* src = FROM_A16 ? reinterpret_cast<const char*>(a16_in + nt)
                                           : reinterpret_cast<const char*>(in + nt);
                const int64_t piece = bytes - lo < 4096 ? bytes - lo : 4096;
                const unsigned len = static_cast<unsigned>((piece + 15) & ~int64_t(15));
                asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(src + lo), "r"(len) : "memory");
            }
        }
        // 1. rank: the warp's items t0 + warp * 512 + 32 k + lane, in item order
        for (int i = lane; i < 256; i += 32) sm.wcnt[warp][i] = 0;
        __syncwarp();
        uint32_t item[kSortPerThread];
        uint32_t rk[kSortPerThread];  // rank among the warp's items of the same digit
#pragma unroll
        for (int k = 0; k < kSortPerThread; k++) {  // all loads first: one memory latency per tile
            const int e = t0 + warp * kSortWarpItems + k * 32 + lane;
            item[k] = e < n ? item_at(e) : 0u;
        }
#pragma unroll
        for (int k = 0; k < kSortPerThread; k++) {
            const int e = t0 + warp * kSortWarpItems + k * 32 + lane;
            const bool valid = e < n;
            const uint32_t d = (item[k] >> shift) & 255u;
            const unsigned peers = digit_peers(d, valid);
            const int leader = __ffs(peers) - 1;
            uint32_t before = 0;
            if (valid && lane == leader) {
                before = sm.wcnt[warp][d];
                sm.wcnt[warp][d] = before + __popc(peers);
            }
            before = __shfl_sync(0xffffffffu, before, leader);
            rk[k] = before + __popc(peers & lt_mask);
            __syncwarp();
        }
        __syncthreads();
        // 2. per digit: each warp's offset inside the tile's run of the digit
        if (t < 256) {
            uint32_t acc = 0;
            for (int w = 0; w < kSortWarps; w++) {
                const uint32_t c = sm.wcnt[w][t];
                sm.wcnt[w][t] = acc;
                acc += c;
            }
            sm.tcount[t] = acc;
        }
        __syncthreads();
        block_exclusive_scan_256(sm.tcount, sm.tbase);
        // 3. the tile into the buffer, digit by digit; per digit, the output
        // position of buffer slot 0 and the end of its slots
        if (t < 256) {
            sm.dst[t] = sm.base[t] + sm.running[t] - sm.tbase[t];
            sm.tend[t] = sm.tbase[t] + sm.tcount[t];
        }
#pragma unroll
        for (int k = 0; k < kSortPerThread; k++) {
            const int e = t0 + warp * kSortWarpItems + k * 32 + lane;
            if (e < n) {
                const uint32_t d = (item[k] >> shift) & 255u;
                sm.buf[sm.tbase[d] + sm.wcnt[warp][d] + rk[k]] = item[k];
            }
        }
        __syncthreads();
        // 4. out: consecutive buffer slots of a digit are consecutive positions
        const int tn = min(kSortTile, n - t0);
        for (int j = t; j < tn; j += kSortThreads) {
            uint32_t it = sm.buf[j];
            const uint32_t d = (it >> shift) & 255u;
            const uint32_t pos = sm.dst[d] + static_cast<uint32_t>(j);
            if (FINAL) {
                const bool last_in_tile = static_cast<uint32_t>(j) + 1 == sm.tend[d];
                if (!last_in_tile && (sm.buf[j + 1] >> 16) != (it >> 16)) it |= 1u;
                out[round_phys(pos)] = it;
            } else {
                out[pos] = it;
                atomicAdd(&sm.hist2[it >> 24], 1u);
            }
        }
        if (FINAL && t < 256 && sm.tcount[t] > 0) {
            // the digit's entry waiting from an earlier tile ends its run
            // unless this tile's first entry of the digit continues its column
            const uint32_t first = sm.buf[sm.tbase[t]];
            if (sm.pend_pos[t] != kNoPend && (first >> 16) != sm.pend_col[t]) out[round_phys(sm.pend_pos[t])] |= 1u;
            sm.pend_pos[t] = sm.base[t] + sm.running[t] + sm.tcount[t] - 1;
            sm.pend_col[t] = sm.buf[sm.tbase[t] + sm.tcount[t] - 1] >> 16;
        }
        __syncthreads();
        if (t < 256) sm.running[t] += sm.tcount[t];
    }
    // the last entry of every digit ends its run (the next has another digit)
    if (FINAL && t < 256 && sm.pend_pos[t] != kNoPend) out[round_phys(sm.pend_pos[t])] |= 1u;
    __syncthreads();
}

__global__ void __launch_bounds__(kSortThreads, kSortCtasPerSm) fast_sort_kernel(FastGeometry g,
                                                                                const uint16_t* __restrict__ a16,
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

// First entry of every (block, column sub-chunk) in G32: lower bound of the
// sub-chunk's first column in the sorted group (sub-chunks past the end of
// a pattern's columns get the group's end).
__global__ void fast_sub_kernel(FastGeometry g, const uint32_t* __restrict__ g32, uint32_t* __restrict__ sub_start)
{
    const int nsub = g.nchunks * kSubPerChunk;
    const int64_t total = g.nblocks * nsub;
    for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < total;
         i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        const int64_t b = i / nsub;
        const int j = static_cast<int>(i - b * nsub);
        const int ch = j / kSubPerChunk;
        int p = 0;
        while (p + 1 < g.npat && g.chunk0[p + 1] <= ch) p++;
        const uint32_t c0 = static_cast<uint32_t>(j - g.chunk0[p] * kSubPerChunk) * kSubCols;
        const int64_t seg = g.seg(b, p);
        int64_t lo = 0, hi = g.seg_len(b, p);
        while (lo < hi) {
            const int64_t mid = (lo + hi) >> 1;
            if ((g32[seg + round_phys(static_cast<uint32_t>(mid))] >> 16) < c0)
                lo = mid + 1;
            else
                hi = mid;
        }
        sub_start[i] = static_cast<uint32_t>(seg + lo);
    }
}

// Entries of every (block, chunk): the distance between the chunk's first
// sub-chunk start and the next chunk's (or the group's end).
__global__ void fast_chunk_entries_kernel(FastGeometry g, const uint32_t* __restrict__ sub_start,
                                          uint32_t* __restrict__ out)
{
    const int64_t total = g.nblocks * g.nchunks;
    for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < total;
         i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        const int64_t b = i / g.nchunks;
        const int ch = static_cast<int>(i - b * g.nchunks);
        int p = 0;
        while (p + 1 < g.npat && g.chunk0[p + 1] <= ch) p++;
        const int c_end = p + 1 < g.npat ? g.chunk0[p + 1] : g.nchunks;
        const int64_t lo = sub_start[i * kSubPerChunk];
        const int64_t hi = ch + 1 < c_end ? static_cast<int64_t>(sub_start[(i + 1) * kSubPerChunk])
                                          : g.seg(b, p) + g.seg_len(b, p);
        out[i] = static_cast<uint32_t>(hi - lo);
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
                const uint32_t v = g32[seg + round_phys(static_cast<uint32_t>(e))];
                int64_t j = 0;
                while (e - j - 1 >= 0 &&
                       (g32[seg + round_phys(static_cast<uint32_t>(e - j - 1))] >> 2) == (v >> 2))
                    j++;  // same (column, row)
                col = v >> 16;
                contrib = static_cast<uint32_t>(2 * j + 1);
            }
            const unsigned peers = __match_any_sync(0xffffffffu, col);
            const uint32_t sum = __reduce_add_sync(peers, contrib);
            if (e < n && lane == __ffs(peers) - 1)
                atomicAdd(reinterpret_cast<unsigned long long*>(diag + g.col_base(b) + g.off[p] + col), sum);
        }
    }
}

// The column counts A'1 from the FP32 A'y partials of a vector of ones:
// every partial (and every sum the A'y kernel forms on the way) counts
// entries of one column inside one item, so it is an exact float integer
// while the item holds fewer than 2^24 entries; the column sums add the
// partials in FP64.
__global__ void fast_count_kernel(FastCols fc, const float* __restrict__ partial, uint64_t* __restrict__ diag)
{
    for (int64_t c = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; c < fc.g.cols;
         c += static_cast<int64_t>(gridDim.x) * blockDim.x)
        diag[c] = static_cast<uint64_t>(fast_col_sum<float>(fc, partial, c));
}

constexpr int kRepeatRounds = 16;  // G32 rounds of one warp's stretch

// One G32 round (4 KB, on a 16-byte boundary) into L2.
__device__ __forceinline__ void prefetch_round(const uint32_t* round)
{
    asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(round),
                 "r"(static_cast<unsigned>(kRound * sizeof(uint32_t)))
                 : "memory");
}

// The repeats' share of diag(A'A): a row holding a column m times adds
// m^2 = m + 2 (1 + 2 + ... + (m - 1)), and the count A'1 holds the m.
// Equal (column, row) pairs are adjacent in a sorted group and number at
// most the pattern's slots (<= 8).  A warp takes a stretch of kRepeatRounds
// rounds of one group; per round each lane holds its 32 consecutive sorted
// entries (the lane run of the round: eight 16-byte words 512 bytes apart)
// and counts copies along them, starting from the entry before its run and
// the number of equal entries that end there (the previous lane's, carried
// from lane 31 across rounds, and walked back in G32 at the stretch's
// start).  A lane adds a column's repeats once per run of that column.
__global__ void __launch_bounds__(256, 4) fast_repeat_kernel(FastGeometry g, const uint32_t* __restrict__ g32,
                                                             uint64_t* __restrict__ diag, int stretches)
{
    const int lane = threadIdx.x & 31;
    const int64_t nwarps = (static_cast<int64_t>(gridDim.x) * blockDim.x) >> 5;
    const int64_t units = g.nblocks * g.npat * stretches;
    for (int64_t u = (static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5; u < units; u += nwarps) {
        const int64_t grp = u / stretches;
        const int st = static_cast<int>(u - grp * stretches);
        const int64_t b = grp / g.npat;
        const int p = static_cast<int>(grp - b * g.npat);
        const int64_t seg = g.seg(b, p), n = g.seg_len(b, p);
        const int64_t r_begin = static_cast<int64_t>(st) * kRepeatRounds * kRound;
        if (r_begin >= n) continue;  // uniform over the warp
        const int64_t r_end = n < r_begin + kRepeatRounds * kRound ? n : r_begin + kRepeatRounds * kRound;
        uint64_t* dcol = diag + g.col_base(b) + g.off[p];
        if (lane == 0 && r_begin + kRound < r_end) prefetch_round(g32 + seg + r_begin + kRound);
        // the entry before the stretch and the equal entries ending there
        uint32_t carry_last = 0;
        int carry_tail = 0;  // 0: none before
        if (r_begin > 0) {
            carry_last = g32[seg + round_phys(static_cast<uint32_t>(r_begin - 1))];
            carry_tail = 1;
            while (carry_tail < r_begin &&
                   (g32[seg + round_phys(static_cast<uint32_t>(r_begin - 1 - carry_tail))] >> 2) == (carry_last >> 2))
                carry_tail++;
        }
        for (int64_t r0 = r_begin; r0 < r_end; r0 += kRound) {
            // the round after next into L2 (whole rounds: the segment's room
            // ends on a round)
            if (lane == 0 && r0 + 2 * kRound < r_end) prefetch_round(g32 + seg + r0 + 2 * kRound);
            const int64_t lb = r0 + kLaneRun * lane;  // the lane's first sorted position
            const int64_t rem = r_end - lb;
            const int cnt = rem <= 0 ? 0 : (rem >= kLaneRun ? kLaneRun : static_cast<int>(rem));
            uint32_t e[kLaneRun];
            const uint4* src = reinterpret_cast<const uint4*>(g32 + seg + r0) + lane;
#pragma unroll
            for (int q = 0; q < kLaneRun / 4; q++) {
                uint4 w = make_uint4(0, 0, 0, 0);
                if (4 * q < cnt) w = src[32 * q];
                e[4 * q] = w.x, e[4 * q + 1] = w.y, e[4 * q + 2] = w.z, e[4 * q + 3] = w.w;
            }
            // the run's last entry and the equal entries ending it (a full
            // run holds more than 8 entries, so this needs nothing before it)
            int tail = 0;
            uint32_t last = 0;
#pragma unroll
            for (int k = 0; k < kLaneRun; k++) {
                if (k < cnt) {
                    tail = (k > 0 && (e[k] >> 2) == (e[k - 1] >> 2)) ? tail + 1 : 1;
                    last = e[k];
                }
            }
            uint32_t before = __shfl_up_sync(0xffffffffu, last, 1);
            int m = __shfl_up_sync(0xffffffffu, tail, 1);
            if (lane == 0) before = carry_last, m = carry_tail;
            carry_last = __shfl_sync(0xffffffffu, last, 31);
            carry_tail = __shfl_sync(0xffffffffu, tail, 31);
            uint64_t acc = 0;
            uint32_t acc_col = cnt > 0 ? e[0] >> 16 : 0;
#pragma unroll
            for (int k = 0; k < kLaneRun; k++) {
                if (k < cnt) {
                    const uint32_t col = e[k] >> 16;
                    if (col != acc_col) {
                        if (acc) atomicAdd(reinterpret_cast<unsigned long long*>(dcol + acc_col), acc);
                        acc = 0;
                        acc_col = col;
                    }
                    if (m > 0 && (e[k] >> 2) == (before >> 2)) {  // copy number m (from 0) of (column, row)
                        acc += 2 * static_cast<uint64_t>(m);
                        m++;
                    } else {
                        m = 1;
                    }
                    before = e[k];
                }
            }
            if (acc) atomicAdd(reinterpret_cast<unsigned long long*>(dcol + acc_col), acc);
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

// Asks L2 to fetch [p, p + bytes) (the 16-byte words wholly inside it), in
// 4 KB bulk prefetches spread over the CTA's threads.  A hint: the data is
// read later with ordinary loads.
__device__ __forceinline__ void prefetch_l2(const void* p, int64_t bytes)
{
    if (bytes <= 0) return;
    const uintptr_t a = (reinterpret_cast<uintptr_t>(p) + 15) & ~uintptr_t(15);
    const uintptr_t e = (reinterpret_cast<uintptr_t>(p) + static_cast<uintptr_t>(bytes)) & ~uintptr_t(15);
    for (uintptr_t c = a + static_cast<uintptr_t>(threadIdx.x) * 4096; c < e;
         c += static_cast<uintptr_t>(blockDim.x) * 4096) {
        const unsigned n = static_cast<unsigned>(min(static_cast<uint64_t>(e - c), static_cast<uint64_t>(4096)));
        asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(c), "r"(n) : "memory");
    }
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
// ROWS rows (stride kAxThreads); the 16-byte index word of row j+AHEAD is
// loaded while row j is gathered, so AHEAD loads per thread stay in flight.
template <typename T, bool ALL_IN, int ROWS, int AHEAD>
__device__ __forceinline__ void gather_segment8(const uint16_t* __restrict__ base, int nb,
                                                const T* __restrict__ table, const T* __restrict__ xg, int cap,
                                                typename AccOf<T>::type (&acc)[ROWS])
{
    uint4 w[AHEAD];
#pragma unroll
    for (int j = 0; j < AHEAD; j++) {
        const int r = threadIdx.x + j * kAxThreads;
        w[j] = r < nb ? *reinterpret_cast<const uint4*>(base + static_cast<int64_t>(r) * 8) : make_uint4(0, 0, 0, 0);
    }
#pragma unroll
    for (int j = 0; j < ROWS; j++) {
        const uint4 cur = w[j % AHEAD];
        if (j + AHEAD < ROWS) {
            const int rn = threadIdx.x + (j + AHEAD) * kAxThreads;
            w[j % AHEAD] = rn < nb ? *reinterpret_cast<const uint4*>(base + static_cast<int64_t>(rn) * 8)
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

// Prefix sums over an active list of a per-problem count (cnt(q)) into
// pref[0..n] in shared memory, by warp 0; every thread returns the total.
template <typename F>
__device__ __forceinline__ int active_prefix(const FastActive* __restrict__ act, int* pref, F cnt)
{
    const int n = act->n;
    if (threadIdx.x < 32) {
        const int lane = threadIdx.x;
        int carry = 0;
        for (int base = 0; base < n; base += 32) {
            const int t = base + lane;
            int v = t < n ? cnt(act->list[t]) : 0;
#pragma unroll
            for (int d = 1; d < 32; d <<= 1) {
                const int u = __shfl_up_sync(0xffffffffu, v, d);
                if (lane >= d) v += u;
            }
            if (t < n) pref[t + 1] = carry + v;
            carry += __shfl_sync(0xffffffffu, v, 31);
        }
        if (lane == 0) pref[0] = 0;
    }
    __syncthreads();
    return pref[n];
}

// Slot k of the active list with pref[k] <= i < pref[k + 1] (0 <= i < pref[n]).
__device__ __forceinline__ int active_slot(const int* pref, int n, int i)
{
    int lo = 0, hi = n - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (pref[mid] <= i)
            lo = mid;
        else
            hi = mid - 1;
    }
    return lo;
}

// Splits of a work unit when `units` units of a product are to fill `ctas`
// CTAs: as many as keep every split unit in one wave, at most cap.  A few
// units' time is set by their chains of dependent loads, not by their
// bytes, so one wave of larger units beats two of smaller ones.
__host__ __device__ __forceinline__ int unit_splits(int64_t units, int64_t ctas, int cap)
{
    if (units <= 0) return 1;
    const int64_t k = ctas / units;
    return static_cast<int>(k < 1 ? 1 : (k > cap ? cap : k));
}

// ALL8: every pattern has 8 slots (the expanded layout), so only the
// pipelined 8-slot path is compiled in.
// A work unit is one of a block's row splits (a CTA stages x's pattern
// slices once per unit, so splits pay only when units are few).  part
// (optional) receives one compensated partial of ||y||^2 per unit, so that
// the norms of the problems of a batched layout can be summed apart.
// Blocks of problems whose pdone flag is set are skipped (partials 0).
// Without act: units (block, split) for every block, `split` splits each,
// partials [block][split].  With act: the listed problems' blocks only,
// split for `ctas` CTAs, partials [block][kAxSplitMax] (splits past the one
// in use written 0); a split of kAxSplitMax is left to
// fast_spmv_direct_kernel.
// ROWS: rows per thread (a unit holds at most kAxThreads * ROWS rows: a
// whole block), AHEAD: index loads in flight per thread.
template <typename T, typename Y, int MODE, bool ALL8, int ROWS = kAxRows, int AHEAD = kAxAhead>
__global__ void __launch_bounds__(kAxThreads, 1) fast_spmv_kernel(FastGeometry g, const uint16_t* __restrict__ a16,
                                                                   const T* __restrict__ x, Y* __restrict__ y,
                                                                   const double* __restrict__ b,
                                                                   const double* __restrict__ coef,
                                                                   double* __restrict__ part,
                                                                   const int* __restrict__ done,
                                                                   const int* __restrict__ pdone,
                                                                   const FastActive* __restrict__ act, int split,
                                                                   int ctas)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T* table = reinterpret_cast<T*>(smem_raw);
    __shared__ double red[64];
    __shared__ int pref[kMaxProblems + 1];
    if (done && *(volatile const int*)done) return;
    constexpr int kCap = sizeof(T) == 4 ? kTable32 : kTable64;
    using Acc = typename AccOf<T>::type;
    const double c = MODE == 1 ? *coef : 0.0;
    int S = split, stride = split;
    int64_t units = g.nblocks * split;
    if (act) {
        const int nblk = active_prefix(act, pref, [&](int q) { return g.pblk0[q + 1] - g.pblk0[q]; });
        S = unit_splits(nblk, ctas, kAxSplitMax);
        stride = kAxSplitMax;
        units = static_cast<int64_t>(nblk) * S;
    }
    if (act && S == kAxSplitMax) return;  // few rows per unit: fast_spmv_direct_kernel's launch
    for (int64_t u = blockIdx.x; u < units; u += gridDim.x) {
        const int sp = static_cast<int>(u % S);
        int64_t blk = u / S;
        if (act) {
            const int i = static_cast<int>(blk);
            const int slot = active_slot(pref, act->n, i);
            blk = g.pblk0[act->list[slot]] + (i - pref[slot]);
        }
        const int q = g.prob_of_block(blk);
        double* pu = part ? part + 2 * (blk * stride + sp) : nullptr;
        if (pu && sp == 0 && static_cast<int>(threadIdx.x) < 2 * (stride - S)) pu[2 * S + threadIdx.x] = 0;
        if (pdone && pdone[q]) {
            if (pu && threadIdx.x == 0) {
                pu[0] = 0;
                pu[1] = 0;
            }
            continue;
        }
        const int rows_b = static_cast<int>(g.block_rows(blk));
        const int r0 = static_cast<int>(static_cast<int64_t>(rows_b) * sp / S);
        const int nb = static_cast<int>(static_cast<int64_t>(rows_b) * (sp + 1) / S) - r0;
        const int64_t row0 = g.block_row0(blk) + r0;
        const T* xq = x + q * g.pcols;
        Comp mine;
        Acc acc[ROWS];
#pragma unroll
        for (int j = 0; j < ROWS; j++) acc[j] = 0;
        // the index stream of a pattern is fetched into L2 one phase ahead,
        // so that HBM keeps streaming while x's next slice is staged
        prefetch_l2(a16 + g.seg(blk, 0) + static_cast<int64_t>(r0) * g.slots[0],
                    static_cast<int64_t>(nb) * g.slots[0] * 2);
        for (int p = 0; p < g.npat; p++) {
            const int cap = min(g.space[p], kCap);
            const T* xg = xq + g.off[p];
            __syncthreads();
            load_table<T>(table, xg, cap);
            __syncthreads();
            if (p + 1 < g.npat)
                prefetch_l2(a16 + g.seg(blk, p + 1) + static_cast<int64_t>(r0) * g.slots[p + 1],
                            static_cast<int64_t>(nb) * g.slots[p + 1] * 2);
            const int ns = g.slots[p];
            const uint16_t* base = a16 + g.seg(blk, p) + static_cast<int64_t>(r0) * ns;
            const bool all_in = g.space[p] <= kCap;
            if (ALL8 || ns == 8) {
                if (all_in)
                    gather_segment8<T, true, ROWS, AHEAD>(base, nb, table, xg, cap, acc);
                else
                    gather_segment8<T, false, ROWS, AHEAD>(base, nb, table, xg, cap, acc);
            } else if (!ALL8) {
#pragma unroll
                for (int j = 0; j < ROWS; j++) {
                    const int r = threadIdx.x + j * kAxThreads;
                    if (r < nb) gather_row<T>(base + static_cast<int64_t>(r) * ns, ns, table, xg, cap, all_in, acc[j]);
                }
            }
        }
#pragma unroll
        for (int j = 0; j < ROWS; j++) {
            const int r = threadIdx.x + j * kAxThreads;
            if (r < nb) {
                const int64_t row = row0 + r;
                double v = static_cast<double>(acc[j]);
                if (MODE == 1) v = static_cast<double>(y[row]) * -c + v;
                if (MODE == 2) v = (b ? b[row] : 0.0) - v;
                const Y yv = static_cast<Y>(v);
                y[row] = yv;
                mine.add(static_cast<double>(yv) * static_cast<double>(yv));
            }
        }
        if (pu) {
            const Comp r = block_sum_comp<kAxThreads>(mine, red);
            if (threadIdx.x == 0) {
                pu[0] = r.s;
                pu[1] = r.c;
            }
        }
    }
}

constexpr int kDirectPatterns = 8;  // most 8-slot patterns of the direct A x's unrolled path

// A x over units of at most kAxDirectRows rows (a block split kAxSplitMax
// ways) without staging x: one thread per row gathers its entries through
// L1/L2 in pattern and slot order, the order of the staged kernel, so both
// give the same values.  Few remaining rows (the last small problems of a
// batch, a small fit) are not worth staging every x slice per CTA.  Without
// act it runs when the host chose kAxSplitMax splits; with act it decides on
// the device, as the staged kernel (launched beside it) does with the same
// `ctas`, and exactly one of the two does the work.  Partials as the staged
// kernel's with stride kAxSplitMax.
template <typename T, typename Y, int MODE, bool ALL8>
__global__ void __launch_bounds__(kAxDirectRows) fast_spmv_direct_kernel(FastGeometry g,
                                                                         const uint16_t* __restrict__ a16,
                                                                         const T* __restrict__ x, Y* __restrict__ y,
                                                                         const double* __restrict__ b,
                                                                         const double* __restrict__ coef,
                                                                         double* __restrict__ part,
                                                                         const int* __restrict__ done,
                                                                         const int* __restrict__ pdone,
                                                                         const FastActive* __restrict__ act, int ctas)
{
    __shared__ double red[64];
    __shared__ int pref[kMaxProblems + 1];
    if (done && *(volatile const int*)done) return;
    using Acc = typename AccOf<T>::type;
    const double c = MODE == 1 ? *coef : 0.0;
    int64_t nblk = g.nblocks;
    if (act) {
        nblk = active_prefix(act, pref, [&](int q) { return g.pblk0[q + 1] - g.pblk0[q]; });
        if (unit_splits(nblk, ctas, kAxSplitMax) != kAxSplitMax) return;  // the staged kernel's work
    }
    const int64_t units = nblk * kAxSplitMax;
    for (int64_t u = blockIdx.x; u < units; u += gridDim.x) {
        const int sp = static_cast<int>(u % kAxSplitMax);
        int64_t blk = u / kAxSplitMax;
        if (act) {
            const int i = static_cast<int>(blk);
            const int slot = active_slot(pref, act->n, i);
            blk = g.pblk0[act->list[slot]] + (i - pref[slot]);
        }
        const int q = g.prob_of_block(blk);
        double* pu = part ? part + 2 * (blk * kAxSplitMax + sp) : nullptr;
        if (pdone && pdone[q]) {
            if (pu && threadIdx.x == 0) {
                pu[0] = 0;
                pu[1] = 0;
            }
            continue;
        }
        const int rows_b = static_cast<int>(g.block_rows(blk));
        const int r0 = static_cast<int>(static_cast<int64_t>(rows_b) * sp / kAxSplitMax);
        const int nb = static_cast<int>(static_cast<int64_t>(rows_b) * (sp + 1) / kAxSplitMax) - r0;
        const T* xq = x + q * g.pcols;
        Comp mine;
        const int r = threadIdx.x;
        if (r < nb) {
            Acc acc = 0;
            if (ALL8) {
                // up to kDirectPatterns patterns of 8 slots: every index word
                // first, then all gathers, so that they are in flight together
                uint4 w[kDirectPatterns];
#pragma unroll
                for (int p = 0; p < kDirectPatterns; p++)
                    if (p < g.npat)
                        w[p] = *reinterpret_cast<const uint4*>(a16 + g.seg(blk, p) + static_cast<int64_t>(r0 + r) * 8);
#pragma unroll
                for (int p = 0; p < kDirectPatterns; p++) {
                    if (p < g.npat) {
                        const T* xg = xq + g.off[p];
                        gather_word<T, true>(w[p].x, xg, xg, 0, acc);
                        gather_word<T, true>(w[p].y, xg, xg, 0, acc);
                        gather_word<T, true>(w[p].z, xg, xg, 0, acc);
                        gather_word<T, true>(w[p].w, xg, xg, 0, acc);
                    }
                }
            } else {
                for (int p = 0; p < g.npat; p++) {
                    const int ns = g.slots[p];
                    gather_row<T>(a16 + g.seg(blk, p) + static_cast<int64_t>(r0 + r) * ns, ns, xq, xq + g.off[p], 0,
                                  false, acc);
                }
            }
            const int64_t row = g.block_row0(blk) + r0 + r;
            double v = static_cast<double>(acc);
            if (MODE == 1) v = static_cast<double>(y[row]) * -c + v;
            if (MODE == 2) v = (b ? b[row] : 0.0) - v;
            const Y yv = static_cast<Y>(v);
            y[row] = yv;
            mine.add(static_cast<double>(yv) * static_cast<double>(yv));
        }
        if (pu) {
            const Comp rs = block_sum_comp<kAxDirectRows>(mine, red);
            if (threadIdx.x == 0) {
                pu[0] = rs.s;
                pu[1] = rs.c;
            }
        }
    }
}

// ---------------------------------------------------------------------------
// A'y on the blocked layout.
// ---------------------------------------------------------------------------
struct TView {
    const int* item_sc;
    const int* item_b0;
    const int* item_b1;
    const int64_t* item_part;
    const int* sc_piece0;
    const int* sc_width;
    const int* piece_pat;
    const int* piece_ch0;
    const int* piece_ch1;
    const int* piece_acc;
    const int* sc_item0;  // [nprob * nsc + 1]: items of problem q are [sc_item0[q * nsc], sc_item0[(q + 1) * nsc])
    int nsc;
    int per_sc;
    int nitems;
};

// Column-sorted entries are reduced lane by lane.  For one block of an item,
// the entry ranges of all the item's pieces (their shares of columns) are
// cut into G32 rounds: piece k covers the rounds that overlap its range
// [lo_k, hi_k), and the pieces' round lists, one after another, form the
// block's list of virtual rounds, which the 32 warps split into contiguous
// stretches of nearly equal length.  In a round each lane owns 32
// consecutive entries (one round is read with 8 coalesced 16-byte loads per
// lane; entries outside the piece's range are masked).  An entry's bit 0
// marks the last entry of its column, so a lane sums y over its entries and
// closes a run at every flagged entry, with no column comparisons.  A
// column's entries of a block are one run, so only the lane where a run ends
// touches its column, and the order of the adds is fixed by the data: the
// result is bitwise reproducible.
//   1. at every run end the lane adds its own part of the run to acc[col];
//   2. the parts of a run in the lanes before (their open tails) are combined
//      by a segmented scan over the warp's lanes (shuffles; the run still
//      open at the end of the warp's previous round enters as `carry`) and
//      added by the lane where the run ends;
//   3. the run still open at the end of a warp's stretch goes to the warp's
//      record;
//   4. after the block, warp 0 combines the 32 records with the same
//      segmented scan (one lane per warp) and adds each chain to the column
//      where it ends.
// A run never crosses pieces (a piece holds whole columns), so the chain is
// reset where a warp's stretch moves on to the next piece.

constexpr int kMaxPieces = kMaxFastPatterns;  // pieces of one super-chunk: at most one per pattern

// The pieces of one (item, block): logical entry ranges, the accumulator
// index of column field 0, and the first virtual round of each piece.
struct BlockPieces {
    uint32_t lo[kMaxPieces];
    uint32_t hi[kMaxPieces];
    int acc_off[kMaxPieces];
    int round0[kMaxPieces + 1];
    int n;
};

// What a warp leaves for the runs that cross warp boundaries.
template <typename T>
struct WarpRec {
    T ls;        // open sum of the warp's last run (0 when that run ends in the warp)
    int fc;      // accumulator index of the warp's first entry's column
    int valid;   // the warp's stretch is non-empty
    int cp;      // the first run continues the previous warp's last run
    int single;  // no run ends in the warp's stretch
};

// y of an entry: its row, already scaled by 4, sits in bits 2..15.
template <typename T>
__device__ __forceinline__ T y_of(const T* __restrict__ ytile, uint32_t e)
{
    if constexpr (sizeof(T) == 4)
        return *reinterpret_cast<const T*>(reinterpret_cast<const char*>(ytile) + (e & 0xFFFCu));
    else
        return ytile[(e & 0xFFFCu) >> 2];
}

// Segmented inclusive scan over the 32 lanes of the open run sums ts.  A
// chain starts at a lane that ends a run (its tail) or whose first entry
// starts a column; a lane with no run end that continues the run from its
// left (single && cont_prev) extends the chain.  The lane whose first run
// continues from the left and ends in it gets the chain of the lanes before
// it (carry before lane 0) through `sink`.  Lanes without entries pass the
// chain through.  Returns the chain leaving lane 31.
template <typename T, typename Sink>
__device__ __forceinline__ T lane_chain(bool any, bool single, bool cont_prev, int hc, T ts, T carry, Sink&& sink)
{
    const int lane = threadIdx.x & 31;
    T v = any ? ts : T(0);
    bool f = any && !(single && cont_prev);
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        const T vu = __shfl_up_sync(0xffffffffu, v, d);
        const bool fu = __shfl_up_sync(0xffffffffu, f, d);
        if (lane >= d) {
            if (!f) v += vu;
            f = f || fu;
        }
    }
    const T X = f ? v : v + carry;  // chain value ending at this lane
    T Xprev = __shfl_up_sync(0xffffffffu, X, 1);
    if (lane == 0) Xprev = carry;
    if (any && !single && cont_prev) sink(hc, Xprev);
    return __shfl_sync(0xffffffffu, X, 31);
}

__device__ __forceinline__ uint32_t word_of(const uint4& u, int j)
{
    return j == 0 ? u.x : (j == 1 ? u.y : (j == 2 ? u.z : u.w));
}

// A lane's entries of one round: slots [k0, k1) of its 32 (all of them when
// FULL), read from src (the lane's first 16-byte word of the round) in two
// halves of 16.  Runs that end here are added to accc (indexed by an entry's
// column field); returns the open tail, the OR of the entries (bit 0: some
// run ended) and the first and last entries in range.
template <typename T, bool FULL>
__device__ __forceinline__ T lane_entries(const uint4* __restrict__ src, int k0, int k1, const T* __restrict__ ytile,
                                          T* __restrict__ accc, uint32_t& eor, uint32_t& first_e, uint32_t& last_e)
{
    T sum = 0;
    uint32_t o = 0, fe = 1u, le = 1u;
#pragma unroll
    for (int h = 0; h < 2; h++) {
        uint4 u[4];
#pragma unroll
        for (int q = 0; q < 4; q++) u[q] = __ldcs(src + 32 * (4 * h + q));
#pragma unroll
        for (int t = 0; t < kLaneRun / 2; t++) {
            const int s = (kLaneRun / 2) * h + t;
            const uint32_t e = word_of(u[t >> 2], t & 3);
            if (FULL || (s >= k0 && s < k1)) {
                sum += y_of<T>(ytile, e);
                o |= e;
                if (e & 1u) {  // the run ends here: this lane's part of it
                    accc[e >> 16] += sum;
                    sum = T(0);
                }
                if (FULL) {
                    if (s == 0) fe = e;
                } else if (s == k0) {
                    fe = e;
                }
                le = e;
            }
        }
    }
    eor = o;
    first_e = fe;
    last_e = le;
    return sum;
}

// Lane 0 of each warp asks L2 for the first round of the warp's stretch in
// the block whose table is bp (issued a block ahead, before its barrier).
__device__ __forceinline__ void prefetch_first_round(const uint32_t* __restrict__ g32, const BlockPieces& bp)
{
    constexpr int kWarps = kFastThreads / 32;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane != 0) return;
    const int nrounds = bp.round0[bp.n];
    const int v = nrounds * warp / kWarps;
    if (v >= nrounds * (warp + 1) / kWarps) return;  // no stretch
    int k = 0;
    while (bp.round0[k + 1] <= v) k++;
    const uint32_t rbase = ((bp.lo[k] / kRound) + static_cast<uint32_t>(v - bp.round0[k])) * kRound;
    asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(g32 + rbase),
                 "r"(static_cast<unsigned>(kRound * sizeof(uint32_t)))
                 : "memory");
}

// The reduction of one block's entries of every piece in `bp` into acc.
// Ends with a block barrier and warp 0's record combination; the next block
// may restage ytile after the next barrier.
template <typename T>
__device__ __forceinline__ void reduce_block(const uint32_t* __restrict__ g32, const BlockPieces& bp,
                                             const BlockPieces* next, const T* __restrict__ ytile,
                                             T* __restrict__ acc, WarpRec<T>* recs)
{
    constexpr int kWarps = kFastThreads / 32;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int nrounds = bp.round0[bp.n];
    const int vr0 = nrounds * warp / kWarps, vr1 = nrounds * (warp + 1) / kWarps;
    T carry = 0;
    bool prev_end = true;
    bool w_end = false, w_cp = false;
    int w_fc = 0;
    int k = 0;
    while (k < bp.n && bp.round0[k + 1] <= vr0) k++;
    for (int vr = vr0; vr < vr1; vr++) {
        if (vr >= bp.round0[k + 1]) {  // the stretch moves on to the next piece
            do {
                k++;
            } while (vr >= bp.round0[k + 1]);
            carry = T(0);
            prev_end = true;
        }
        const uint32_t lo = bp.lo[k], hi = bp.hi[k];
        const uint32_t rbase = ((lo / kRound) + static_cast<uint32_t>(vr - bp.round0[k])) * kRound;
        T* accc = acc + bp.acc_off[k];
        if (lane == 0 && vr + 1 < bp.round0[k + 1]) {
            // the next round of this piece into L2 while this one is reduced
            asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(g32 + rbase + kRound),
                         "r"(static_cast<unsigned>(kRound * sizeof(uint32_t)))
                         : "memory");
        }
        const uint4* src = reinterpret_cast<const uint4*>(g32 + rbase) + lane;
        const uint32_t lb = rbase + kLaneRun * lane;  // the lane's first slot
        const int k0 = lo > lb ? static_cast<int>(min(lo - lb, static_cast<uint32_t>(kLaneRun))) : 0;
        const int k1 = hi > lb ? static_cast<int>(min(hi - lb, static_cast<uint32_t>(kLaneRun))) : 0;
        const bool any = k0 < k1;
        uint32_t eor, first_e, last_e;
        T sum;
        if (__all_sync(0xffffffffu, k0 == 0 && k1 == kLaneRun))
            sum = lane_entries<T, true>(src, 0, kLaneRun, ytile, accc, eor, first_e, last_e);
        else
            sum = lane_entries<T, false>(src, k0, k1, ytile, accc, eor, first_e, last_e);
        // no run ends in the lane: one column, its last entry not flagged
        const bool single = any && !(eor & 1u);
        const int hc = static_cast<int>(first_e >> 16);  // the lane's first run
        // the lane continues the run of the entry before it unless that entry
        // ended its run (previous lane's last entry; at lane 0 the warp's
        // previous round, and none in the warp's first round: the record
        // chain joins runs across warps)
        const uint32_t f = lb + static_cast<uint32_t>(k0);
        const uint32_t prev_last = __shfl_up_sync(0xffffffffu, last_e, 1);
        const bool cont_prev = any && f > lo && (lane == 0 ? (vr != vr0 && !prev_end) : !(prev_last & 1u));
        auto sink = [&](int col, T val) { accc[col] += val; };
        const unsigned anyb = __ballot_sync(0xffffffffu, any);
        const int lastl = 31 - __clz(anyb);  // a round holds at least one entry of its piece
        if (__ballot_sync(0xffffffffu, single && cont_prev) == 0) {
            // no lane extends a run from its left: a chain is one lane's tail
            T prev_ts = __shfl_up_sync(0xffffffffu, sum, 1);
            if (lane == 0) prev_ts = carry;
            if (any && !single && cont_prev) sink(hc, prev_ts);
            carry = __shfl_sync(0xffffffffu, sum, lastl);
        } else {
            carry = lane_chain<T>(any, single, cont_prev, hc, sum, carry, sink);
        }
        prev_end = (__shfl_sync(0xffffffffu, last_e, lastl) & 1u) != 0;
        if (vr == vr0) {
            // the stretch's first entry: its column, and whether it continues
            // the run that ends the previous warp's stretch
            const int fl = __ffs(anyb) - 1;
            const uint32_t f0 = __shfl_sync(0xffffffffu, f, fl);
            w_fc = bp.acc_off[k] + static_cast<int>(__shfl_sync(0xffffffffu, first_e, fl) >> 16);
            w_cp = f0 > lo && !(g32[round_phys(f0 - 1)] & 1u);
        }
        const bool ended = __ballot_sync(0xffffffffu, any && !single) != 0;  // every lane votes, every round
        w_end = w_end || ended;
    }
    if (next) prefetch_first_round(g32, *next);  // while the other warps finish this block
    if (lane == 0) {
        WarpRec<T>& rec = recs[warp];
        rec.valid = vr0 < vr1;
        rec.ls = carry;  // the chain still open at the stretch's end (0 if its last run ended)
        rec.fc = w_fc;
        rec.cp = w_cp;
        rec.single = !w_end;
    }
    __syncthreads();
    if (warp == 0) {
        WarpRec<T> r{};  // lanes past the CTA's warps carry no stretch
        if (lane < kWarps) r = recs[lane];
        lane_chain<T>(r.valid != 0, r.single != 0, r.cp != 0, r.fc, r.ls, T(0),
                      [&](int col, T val) { acc[col] += val; });
    }
}

// ---------------------------------------------------------------------------
// The same reduction for items whose blocks hold few rounds (the FP64
// products, whose accumulator holds one chunk): each (block, piece) entry
// range is cut into 32 nearly equal stretches of whole 4-entry words, one
// per warp, so every warp works whatever the number of rounds; a warp's
// stretch is reduced in steps of kStretchRun entries per lane (consecutive
// in the sorted order, two 16-byte words of G32 each), with the same lane
// chain and warp records.
// ---------------------------------------------------------------------------
constexpr int kStretchRun = 16;                 // entries per lane and step
constexpr int kStretchVecs = kStretchRun / 4;   // 16-byte words per lane and step

// The 16-byte word of G32 that holds sorted positions e .. e+3 (e a
// multiple of 4).
__device__ __forceinline__ uint4 word_at(const uint32_t* __restrict__ g32, uint32_t e)
{
    return __ldcs(reinterpret_cast<const uint4*>(g32 + round_phys(e)));
}

// A lane's entries of a step are all inside the warp's stretch.
__device__ __forceinline__ bool lane_full(uint32_t e_first, uint32_t w_lo, uint32_t w_hi)
{
    return e_first >= w_lo && e_first + kStretchRun <= w_hi;
}

__device__ __forceinline__ void load_lane(const uint32_t* __restrict__ g32, uint32_t e_first,
                                          uint4 (&u)[kStretchVecs])
{
#pragma unroll
    for (int q = 0; q < kStretchVecs; q++) u[q] = word_at(g32, e_first + 4 * q);
}

// One step of a warp over [w_lo, w_hi): lanes take kStretchRun entries
// each from step_start (a multiple of 4).  A lane whose entries are all in
// range gets them in `cur` (loaded ahead by the caller); edge lanes load
// theirs one by one.  accc: the accumulator shifted so that an entry's
// column field indexes it.  carry: the run open before the step (updated);
// prev_end: the last entry before this step ended its run (updated).
template <typename T>
__device__ __forceinline__ void stretch_step(const uint32_t* __restrict__ g32, uint32_t step_start, uint32_t w_lo,
                                             uint32_t w_hi, const T* __restrict__ ytile, T* __restrict__ accc,
                                             T& carry, bool& prev_end, const uint4 (&cur)[kStretchVecs], bool full)
{
    const int lane = threadIdx.x & 31;
    const uint32_t e_first = step_start + lane * kStretchRun;
    T sum = 0;
    uint32_t ends = 0;
    auto step = [&](uint32_t e) {
        sum += y_of<T>(ytile, e);
        ends |= e;
        if (e & 1u) {  // the run ends here: this lane's part of it
            accc[e >> 16] += sum;
            sum = T(0);
        }
    };
    bool any = false;
    uint32_t first_ent = 1u, last_ent = 1u;  // an empty lane looks like a closed run
    if (full) {
        first_ent = cur[0].x;
#pragma unroll
        for (int q = 0; q < kStretchVecs; q++) {
            step(cur[q].x);
            step(cur[q].y);
            step(cur[q].z);
            step(cur[q].w);
        }
        any = true;
        last_ent = cur[kStretchVecs - 1].w;
    } else {
        const uint32_t lo = max(e_first, w_lo), hi = min(e_first + kStretchRun, w_hi);
        if (lo < hi) {
            for (uint32_t e = lo; e < hi; e++) step(g32[round_phys(e)]);
            any = true;
            first_ent = g32[round_phys(lo)];
            last_ent = g32[round_phys(hi - 1)];
        }
    }
    const bool single = any && !(ends & 1u);
    const int hc = static_cast<int>(first_ent >> 16);
    const uint32_t first_valid = max(e_first, w_lo);
    const uint32_t prev_last = __shfl_up_sync(0xffffffffu, last_ent, 1);
    const bool cont_prev = any && first_valid > w_lo && (lane == 0 ? !prev_end : !(prev_last & 1u));
    auto sink = [&](int col, T val) { accc[col] += val; };
    if (__ballot_sync(0xffffffffu, single && cont_prev) == 0) {
        T prev_ts = __shfl_up_sync(0xffffffffu, sum, 1);
        if (lane == 0) prev_ts = carry;
        if (any && !single && cont_prev) sink(hc, prev_ts);
        const int last = min(31, static_cast<int>((w_hi - 1 - step_start) / kStretchRun));  // last lane with entries
        carry = __shfl_sync(0xffffffffu, sum, last);
    } else {
        carry = lane_chain<T>(any, single, cont_prev, hc, sum, carry, sink);
    }
    prev_end = (__shfl_sync(0xffffffffu, last_ent, 31) & 1u) != 0;
}

// The stretch reduction of one block's entries [e_lo, e_hi) of one piece
// into accc (indexed by column field).  Ends with a block barrier; warp 0
// then combines the records (recs: the set of this piece; the caller
// alternates two sets so that the next piece may start meanwhile).
template <typename T>
__device__ __forceinline__ void reduce_stretch(const uint32_t* __restrict__ g32, uint32_t e_lo, uint32_t e_hi,
                                               const T* __restrict__ ytile, T* __restrict__ accc, WarpRec<T>* recs)
{
    constexpr int kWarps = kFastThreads / 32;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const uint64_t n = e_hi - e_lo;
    auto cut = [&](int w) -> uint32_t {
        if (w == 0) return e_lo;
        if (w == kWarps) return e_hi;
        return max(e_lo, (e_lo + static_cast<uint32_t>(n * w / kWarps)) & ~3u);
    };
    const uint32_t w_lo = cut(warp), w_hi = cut(warp + 1);
    T carry = 0;
    bool prev_end = true;
    const uint32_t step_len = 32 * kStretchRun;
    const uint32_t rs0 = w_lo & ~3u;
    if (w_lo < w_hi) {
        // two register buffers that swap roles every step: the next step's
        // entries load while this one is reduced
        uint4 ba[kStretchVecs], bb[kStretchVecs];
        uint32_t rs = rs0;
        bool fa = rs < w_hi && lane_full(rs + lane * kStretchRun, w_lo, w_hi);
        if (fa) load_lane(g32, rs + lane * kStretchRun, ba);
        while (rs < w_hi) {
            uint32_t rn = rs + step_len;
            const bool fb = rn < w_hi && lane_full(rn + lane * kStretchRun, w_lo, w_hi);
            if (fb) load_lane(g32, rn + lane * kStretchRun, bb);
            stretch_step<T>(g32, rs, w_lo, w_hi, ytile, accc, carry, prev_end, ba, fa);
            rs = rn;
            if (rs >= w_hi) break;
            rn = rs + step_len;
            fa = rn < w_hi && lane_full(rn + lane * kStretchRun, w_lo, w_hi);
            if (fa) load_lane(g32, rn + lane * kStretchRun, ba);
            stretch_step<T>(g32, rs, w_lo, w_hi, ytile, accc, carry, prev_end, bb, fb);
            rs = rn;
        }
    }
    if (lane == 0) {
        WarpRec<T>& rec = recs[warp];
        rec.valid = w_lo < w_hi;
        rec.ls = carry;  // the chain still open at the stretch's end (0 if its last run ended)
        rec.fc = rec.cp = rec.single = 0;
        if (w_lo < w_hi) {
            const uint32_t ef = g32[round_phys(w_lo)], el = g32[round_phys(w_hi - 1)];
            rec.fc = static_cast<int>(ef >> 16);
            rec.cp = w_lo > e_lo && !(g32[round_phys(w_lo - 1)] & 1u);
            rec.single = ((ef ^ el) >> 16) == 0 && !(el & 1u);
        }
    }
    __syncthreads();
    if (warp == 0) {
        WarpRec<T> r{};  // lanes past the CTA's warps carry no stretch
        if (lane < kWarps) r = recs[lane];
        lane_chain<T>(r.valid != 0, r.single != 0, r.cp != 0, r.fc, r.ls, T(0),
                      [&](int col, T val) { accc[col] += val; });
    }
}

// Accumulator columns [a0, a1) of piece pc that split `split` of `nsplit`
// covers: its share of the piece's column sub-chunks.
__device__ __forceinline__ void piece_share(const FastGeometry& g, const TView& tv, int pc, int split, int nsplit,
                                            int& a0, int& a1)
{
    const int p = tv.piece_pat[pc];
    const int cl0 = (tv.piece_ch0[pc] - g.chunk0[p]) * kChunkCols;
    const int w = min(g.space[p], (tv.piece_ch1[pc] - g.chunk0[p]) * kChunkCols) - cl0;
    const int ns = (w + kSubCols - 1) / kSubCols;
    a0 = min(w, ns * split / nsplit * kSubCols);
    a1 = min(w, ns * (split + 1) / nsplit * kSubCols);
}

// The table of one block's pieces (entry ranges of their shares, the
// accumulator offsets, the virtual rounds), by one warp.
__device__ __forceinline__ void fill_pieces(const FastGeometry& g, const TView& tv, const uint32_t* __restrict__ sub_start,
                                            int pc0, int pc1, int split, int nsplit, int64_t blk, BlockPieces& bp)
{
    const int lane = threadIdx.x & 31;
    const int nsub = g.nchunks * kSubPerChunk;
    const int npc = pc1 - pc0;
    uint32_t lo = 0, hi = 0;
    int off = 0, nr = 0;
    if (lane < npc) {
        const int pc = pc0 + lane;
        int a0, a1;
        piece_share(g, tv, pc, split, nsplit, a0, a1);
        if (a0 < a1) {
            const int p = tv.piece_pat[pc];
            const int ch0 = tv.piece_ch0[pc];
            const int pat_sub_end = (p + 1 < g.npat ? g.chunk0[p + 1] : g.nchunks) * kSubPerChunk;
            const int j0 = ch0 * kSubPerChunk + a0 / kSubCols;
            const int j1 = ch0 * kSubPerChunk + (a1 + kSubCols - 1) / kSubCols;
            lo = sub_start[blk * nsub + j0];
            hi = j1 < pat_sub_end ? sub_start[blk * nsub + j1]
                                  : static_cast<uint32_t>(g.seg(blk, p) + g.seg_len(blk, p));
            off = tv.piece_acc[pc] - (ch0 - g.chunk0[p]) * kChunkCols;
            if (lo < hi) nr = static_cast<int>((hi - 1) / kRound - lo / kRound) + 1;
        }
    }
    int incl = nr;  // inclusive scan of the rounds over the pieces
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        const int v = __shfl_up_sync(0xffffffffu, incl, d);
        if (lane >= d) incl += v;
    }
    if (lane < npc) {
        bp.lo[lane] = lo;
        bp.hi[lane] = hi;
        bp.acc_off[lane] = off;
        bp.round0[lane + 1] = incl;
    }
    if (lane == 0) {
        bp.round0[0] = 0;
        bp.n = npc;
    }
}

// One work unit: split `split` of `nsplit` of item `item`, i.e. the partial
// column sums of its share of super-chunk item_sc[item]'s columns (a share
// of every piece's column sub-chunks) over the blocks [item_b0, item_b1),
// written to those columns of partial + item_part[item] -
// item_part[item_base].  A column's entries of a block are one run of the
// sorted group, so splitting at sub-chunk bounds splits no run.
// STRETCH: each (block, piece) range is reduced on its own by the stretch
// reduction (the FP64 items); else the block's pieces share one round list.
template <typename T, bool STRETCH>
__device__ __forceinline__ void aty_item(const FastGeometry& g, const TView& tv, const uint32_t* __restrict__ g32,
                                         const uint32_t* __restrict__ sub_start, const T* __restrict__ y,
                                         T* __restrict__ partial, int item, int item_base, int64_t y_block0,
                                         int split, int nsplit, T* __restrict__ acc, T* __restrict__ ytile,
                                         WarpRec<T> (*recs)[kFastThreads / 32], BlockPieces* bp,
                                         const int* __restrict__ pdone)
{
    if (pdone && pdone[g.prob_of_block(tv.item_b0[item])]) return;  // retired problem: partials unused
    const int sc = tv.item_sc[item];
    const int pc0 = tv.sc_piece0[sc], pc1 = tv.sc_piece0[sc + 1];
    const int nsub = g.nchunks * kSubPerChunk;
    bool any = false;
    for (int pc = pc0; pc < pc1; pc++) {
        int a0, a1;
        piece_share(g, tv, pc, split, nsplit, a0, a1);
        any = any || a0 < a1;
        T* ap = acc + tv.piece_acc[pc];
        for (int i = a0 + threadIdx.x; i < a1; i += kFastThreads) ap[i] = 0;
    }
    if (!any) return;  // more splits than sub-chunks: nothing here
    const int warp = threadIdx.x >> 5;
    const int64_t b0 = tv.item_b0[item], b1 = tv.item_b1[item];
    if (!STRETCH && warp == 0) fill_pieces(g, tv, sub_start, pc0, pc1, split, nsplit, b0, bp[0]);
    for (int64_t blk = b0; blk < b1; blk++) {
        const int nb = static_cast<int>(g.block_rows(blk));
        const int i = static_cast<int>(blk - b0);
        __syncthreads();
        if (!STRETCH && i == 0) prefetch_first_round(g32, bp[0]);
        const T* yb = y ? y + (g.block_row0(blk) - g.block_row0(y_block0)) : nullptr;
        if (!yb) {  // no y: a vector of ones (the column counts A'1)
            for (int i = threadIdx.x; i < nb; i += kFastThreads) ytile[i] = T(1);
        } else if ((reinterpret_cast<uintptr_t>(yb) & 15) == 0) {
            // 16-byte loads, kInFlight per thread issued before their stores
            // (FP32: the whole tile in two rounds; FP64 keeps its registers)
            constexpr int kPer = 16 / sizeof(T);
            constexpr int kInFlight = sizeof(T) == 4 ? 2 : 1;
            const int nvec = nb / kPer;
            const uint4* srcv = reinterpret_cast<const uint4*>(yb);
            uint4* dst = reinterpret_cast<uint4*>(ytile);
            for (int i0 = threadIdx.x; i0 < nvec; i0 += kInFlight * kFastThreads) {
                uint4 v[kInFlight];
#pragma unroll
                for (int kk = 0; kk < kInFlight; kk++)
                    if (i0 + kk * kFastThreads < nvec) v[kk] = __ldg(srcv + i0 + kk * kFastThreads);
#pragma unroll
                for (int kk = 0; kk < kInFlight; kk++)
                    if (i0 + kk * kFastThreads < nvec) dst[i0 + kk * kFastThreads] = v[kk];
            }
            for (int i = nvec * kPer + threadIdx.x; i < nb; i += kFastThreads) ytile[i] = yb[i];
        } else {
            for (int i = threadIdx.x; i < nb; i += kFastThreads) ytile[i] = yb[i];
        }
        if (y && blk + 1 < tv.item_b1[item])  // the next block's y slice into L2
            prefetch_l2(y + (g.block_row0(blk + 1) - g.block_row0(y_block0)),
                        static_cast<int64_t>(g.block_rows(blk + 1)) * static_cast<int64_t>(sizeof(T)));
        if constexpr (STRETCH) {
            __syncthreads();
            int flip = 0;
            for (int pc = pc0; pc < pc1; pc++) {
                int a0, a1;
                piece_share(g, tv, pc, split, nsplit, a0, a1);
                if (a0 >= a1) continue;
                const int p = tv.piece_pat[pc];
                const int ch0 = tv.piece_ch0[pc];
                const int pat_sub_end = (p + 1 < g.npat ? g.chunk0[p + 1] : g.nchunks) * kSubPerChunk;
                const int j0 = ch0 * kSubPerChunk + a0 / kSubCols;
                const int j1 = ch0 * kSubPerChunk + (a1 + kSubCols - 1) / kSubCols;
                const uint32_t e_lo = sub_start[blk * nsub + j0];
                const uint32_t e_hi = j1 < pat_sub_end ? sub_start[blk * nsub + j1]
                                                       : static_cast<uint32_t>(g.seg(blk, p) + g.seg_len(blk, p));
                T* accc = acc + tv.piece_acc[pc] - (ch0 - g.chunk0[p]) * kChunkCols;
                reduce_stretch<T>(g32, e_lo, e_hi, ytile, accc, recs[flip]);
                flip ^= 1;
            }
            continue;
        }
        if (warp == 0 && blk + 1 < b1)  // the next block's table, a block ahead
            fill_pieces(g, tv, sub_start, pc0, pc1, split, nsplit, blk + 1, bp[(i + 1) & 1]);
        __syncthreads();
        reduce_block<T>(g32, bp[i & 1], blk + 1 < b1 ? &bp[(i + 1) & 1] : nullptr, ytile, acc, recs[0]);
    }
    __syncthreads();
    T* out = partial + (tv.item_part[item] - tv.item_part[item_base]);
    for (int pc = pc0; pc < pc1; pc++) {
        int a0, a1;
        piece_share(g, tv, pc, split, nsplit, a0, a1);
        const int o = tv.piece_acc[pc];
        for (int i = a0 + threadIdx.x; i < a1; i += kFastThreads) out[o + i] = acc[o + i];
    }
}

// A'y over a work list; a unit is one of the nsplit column splits of an
// item.  With ctr (persistent schedule: one CTA per SM) the CTAs take units
// in order from the counter ctr[0] until the list is done, so no SM idles
// while units of uneven duration remain; which CTA runs a unit does not
// change its output, so results stay bitwise reproducible.  The last CTA to
// finish resets the counters for the next launch (launches on one work list
// must therefore be stream-ordered).  Without ctr, CTA i runs unit i of the
// items from item_base on.  With act (and ctr) the units are those of the
// listed problems' items, split by a factor derived from their number.
template <typename T>
__global__ void __launch_bounds__(kFastThreads, 1) fast_spmv_t_kernel(FastGeometry g, TView tv,
                                                                       const uint32_t* __restrict__ g32,
                                                                       const uint32_t* __restrict__ sub_start,
                                                                       const T* __restrict__ y,
                                                                       T* __restrict__ partial,
                                                                       const int* __restrict__ done, int item_base,
                                                                       int64_t y_block0, int* __restrict__ ctr,
                                                                       const int* __restrict__ pdone,
                                                                       const FastActive* __restrict__ act, int nsplit)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    // two record sets: the stretch reduction alternates them per piece, so
    // that warp 0 may still combine one piece's records while the other
    // warps start on the next piece
    __shared__ WarpRec<T> recs[2][kFastThreads / 32];
    __shared__ BlockPieces bp[2];  // this block's piece table and the next one's
    constexpr bool kStretch = sizeof(T) == 8;  // FP64 items hold one chunk: few rounds per block
    __shared__ int s_item;
    __shared__ int pref[kMaxProblems + 1];
    if (done && *(volatile const int*)done) return;
    T* ytile = reinterpret_cast<T*>(smem_raw);  // first: its entries' byte offsets address it directly
    T* acc = ytile + kBlockRows;
    if (!ctr) {
        const int u = static_cast<int>(blockIdx.x);
        aty_item<T, kStretch>(g, tv, g32, sub_start, y, partial, u / nsplit + item_base, item_base, y_block0,
                              u % nsplit, nsplit, acc, ytile, recs, bp, pdone);
        return;
    }
    int K = nsplit, units = tv.nitems * nsplit;
    if (act) {
        const int nit = active_prefix(act, pref, [&](int q) {
            return tv.sc_item0[(q + 1) * tv.nsc] - tv.sc_item0[q * tv.nsc];
        });
        K = unit_splits(nit, gridDim.x, kAtySplitMax);
        units = nit * K;
    }
    while (true) {
        __syncthreads();
        if (threadIdx.x == 0) s_item = atomicAdd(ctr, 1);
        __syncthreads();
        const int u = s_item;
        if (u >= units) break;
        int item = u / K;
        if (act) {
            const int slot = active_slot(pref, act->n, item);
            item = tv.sc_item0[act->list[slot] * tv.nsc] + (item - pref[slot]);
        }
        aty_item<T, kStretch>(g, tv, g32, sub_start, y, partial, item, 0, 0, u % K, K, acc, ytile, recs, bp, pdone);
    }
    if (threadIdx.x == 0) {
        __threadfence();
        if (atomicAdd(ctr + 1, 1) == static_cast<int>(gridDim.x) - 1) {
            ctr[0] = 0;
            ctr[1] = 0;
            __threadfence();
        }
    }
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
        int64_t b, rb;
        g.locate_row(r, b, rb);
        const float* wq = w + g.col_base(b);
        float acc = 0;
        for (int p = 0; p < g.npat; p++)
            gather_row<float>(a16 + g.seg(b, p) + rb * g.slots[p], g.slots[p], wq + g.off[p], wq + g.off[p], 0, false,
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

// Forward of a training step fused with its loss: per row the score (as in
// fast_rows_forward_kernel), d = score - target, the Huber loss of d summed
// per CTA into red[blockIdx.x] (FP64, deterministic tree), and the loss
// gradient dscore = clamp(d, -delta, delta) / n for the adjoint.
__global__ void __launch_bounds__(256) eval_loss_grad_kernel(FastGeometry g, const uint16_t* __restrict__ a16,
                                                             const float* __restrict__ w,
                                                             const float* __restrict__ target, int64_t row0,
                                                             int64_t row1, float delta, float inv_n,
                                                             float* __restrict__ dscore, double* __restrict__ red)
{
    __shared__ double smem[32];
    double hs = 0;
    for (int64_t r = row0 + static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; r < row1;
         r += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        int64_t b, rb;
        g.locate_row(r, b, rb);
        const float* wq = w + g.col_base(b);
        float acc = 0;
        for (int p = 0; p < g.npat; p++)
            gather_row<float>(a16 + g.seg(b, p) + rb * g.slots[p], g.slots[p], wq + g.off[p], wq + g.off[p], 0, false,
                              acc);
        const float d = acc - target[r - row0];
        const float ad = fabsf(d);
        hs += ad < delta ? 0.5f * d * d : delta * (ad - 0.5f * delta);
        dscore[r - row0] = fminf(fmaxf(d, -delta), delta) * inv_n;
    }
    const double t = block_sum<256>(hs, smem);
    if (threadIdx.x == 0) red[blockIdx.x] = t;
}

// Epilogue of a training step, per column c: the gradient g = sum of the
// adjoint's block partials (block order) + 2 l2 w, then Adam on w, m, v with
// the step t = *step + 1 (torch.optim.Adam's update: m += (1 - b1)(g - m),
// v = b2 v + (1 - b2) g^2, w -= lr / (1 - b1^t) * m / (sqrt(v) / sqrt(1 -
// b2^t) + eps)).  ||w||^2 before the update is summed per CTA; the last CTA
// (integer counter) adds the step's loss, sum(Huber)/n + l2 ||w||^2, to
// *loss_sum, stores t and resets the counter.
__global__ void __launch_bounds__(256) eval_adam_kernel(const float* __restrict__ partial, int nb, int64_t cols,
                                                        float* __restrict__ w, float* __restrict__ m,
                                                        float* __restrict__ v, int64_t* __restrict__ step,
                                                        double* __restrict__ loss_sum, double* __restrict__ red,
                                                        int nred, int* __restrict__ ctr, EvalAdam o, double inv_n)
{
    __shared__ double smem[32];
    __shared__ int last;
    const int64_t t = *step + 1;  // read by every CTA before the last one stores t
    const float step_size = static_cast<float>(o.lr / (1.0 - pow(static_cast<double>(o.beta1), static_cast<double>(t))));
    const float bc2_sqrt = static_cast<float>(sqrt(1.0 - pow(static_cast<double>(o.beta2), static_cast<double>(t))));
    double wsq = 0;
    for (int64_t c = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; c < cols;
         c += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        float gc = 0;
        for (int j = 0; j < nb; j++) gc += partial[static_cast<int64_t>(j) * cols + c];
        const float wc = w[c];
        wsq += static_cast<double>(wc) * wc;
        gc += (2.0f * o.l2) * wc;
        float mc = m[c];
        mc += (1.0f - o.beta1) * (gc - mc);
        const float vc = o.beta2 * v[c] + (1.0f - o.beta2) * gc * gc;
        const float denom = sqrtf(vc) / bc2_sqrt + o.eps;
        w[c] = wc - step_size * (mc / denom);
        m[c] = mc;
        v[c] = vc;
    }
    const double s = block_sum<256>(wsq, smem);
    if (threadIdx.x == 0) {
        red[kEvalRedMax + blockIdx.x] = s;
        __threadfence();
        last = atomicAdd(ctr, 1) == static_cast<int>(gridDim.x) - 1;
    }
    __syncthreads();
    if (last) {  // the whole last CTA: strided sums, then the fixed block tree
        __threadfence();
        double h = 0, q = 0;
        for (int i = threadIdx.x; i < nred; i += blockDim.x) h += __ldcg(red + i);
        for (int i = threadIdx.x; i < static_cast<int>(gridDim.x); i += blockDim.x) q += __ldcg(red + kEvalRedMax + i);
        h = block_sum<256>(h, smem);
        q = block_sum<256>(q, smem);
        if (threadIdx.x == 0) {
            *loss_sum += h * inv_n + static_cast<double>(o.l2) * q;
            *step = t;
            *ctr = 0;
            __threadfence();
        }
    }
}

template <typename T>
__global__ void fast_col_sum_kernel(FastCols fc, const T* __restrict__ partial, T* __restrict__ x)
{
    for (int64_t c = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; c < fc.g.cols;
         c += static_cast<int64_t>(gridDim.x) * blockDim.x)
        x[c] = static_cast<T>(fast_col_sum<T>(fc, partial, c));
}

// The small arrays of a work list, gathered on the host and sent to the
// device as one block: one allocation and one copy instead of one each, so
// that building a layout makes few driver calls.
struct MetaPack {
    std::vector<unsigned char> host;
    std::vector<std::pair<size_t, void**>> fields;

    template <typename V>
    void add(const std::vector<V>& v, V** field)
    {
        const size_t off = (host.size() + 15) & ~size_t(15);
        host.resize(off + sizeof(V) * std::max<size_t>(v.size(), 1), 0);
        if (!v.empty()) std::memcpy(host.data() + off, v.data(), sizeof(V) * v.size());
        fields.emplace_back(off, reinterpret_cast<void**>(field));
    }
    // Uploads the block into *base and points every field into it.
    cas_status upload(void** base)
    {
        CAS_CUDA(dmalloc(base, std::max<size_t>(host.size(), 16)));
        if (!host.empty()) CAS_CUDA(cudaMemcpy(*base, host.data(), host.size(), cudaMemcpyHostToDevice));
        for (auto& f : fields) *f.second = static_cast<unsigned char*>(*base) + f.first;
        return CAS_OK;
    }
};

// Columns of a global chunk (the last chunk of a pattern may be partial).
int chunk_width(const FastGeometry& g, int ch)
{
    int p = 0;
    while (p + 1 < g.npat && g.chunk0[p + 1] <= ch) p++;
    return std::min(kChunkCols, g.space[p] - (ch - g.chunk0[p]) * kChunkCols);
}

int pattern_of_chunk(const FastGeometry& g, int ch)
{
    int p = 0;
    while (p + 1 < g.npat && g.chunk0[p + 1] <= ch) p++;
    return p;
}

// Super-chunk pieces, host side.
struct Pieces {
    std::vector<int> sc_piece0, sc_width, pat, ch0, ch1, acc, chunk_sc, chunk_acc;
};

// Packs the chunks, in pattern order, into accumulators of cap columns: a
// chunk joins the current super-chunk while it fits, and consecutive chunks
// of one pattern in one super-chunk form one piece.
Pieces pack_chunks(const FastGeometry& g, int cap, bool across_patterns)
{
    Pieces pc;
    pc.chunk_sc.resize(g.nchunks);
    pc.chunk_acc.resize(g.nchunks);
    int w = 0;
    for (int ch = 0; ch < g.nchunks; ch++) {
        const int p = pattern_of_chunk(g, ch);
        const int cw = chunk_width(g, ch);
        const bool new_pattern = !pc.pat.empty() && pc.pat.back() != p;
        if (pc.sc_piece0.empty() || w + cw > cap || (new_pattern && !across_patterns)) {
            if (!pc.sc_piece0.empty()) pc.sc_width.push_back(w);
            pc.sc_piece0.push_back(static_cast<int>(pc.pat.size()));
            w = 0;
        }
        const bool extend = !pc.pat.empty() && pc.sc_piece0.back() < static_cast<int>(pc.pat.size()) &&
                            pc.pat.back() == p && pc.ch1.back() == ch;
        if (extend) {
            pc.ch1.back() = ch + 1;
        } else {
            pc.pat.push_back(p);
            pc.ch0.push_back(ch);
            pc.ch1.push_back(ch + 1);
            pc.acc.push_back(w);
        }
        pc.chunk_sc[ch] = static_cast<int>(pc.sc_piece0.size()) - 1;
        pc.chunk_acc[ch] = w;
        w += cw;
    }
    if (!pc.sc_piece0.empty()) pc.sc_width.push_back(w);
    pc.sc_piece0.push_back(static_cast<int>(pc.pat.size()));
    return pc;
}

void pack_pieces(const Pieces& pc, FastTranspose& t, MetaPack& mp)
{
    t.nsc = static_cast<int>(pc.sc_width.size());
    t.npieces = static_cast<int>(pc.pat.size());
    mp.add(pc.sc_piece0, &t.sc_piece0);
    mp.add(pc.sc_width, &t.sc_width);
    mp.add(pc.pat, &t.piece_pat);
    mp.add(pc.ch0, &t.piece_ch0);
    mp.add(pc.ch1, &t.piece_ch1);
    mp.add(pc.acc, &t.piece_acc);
    mp.add(pc.chunk_sc, &t.chunk_sc);
    mp.add(pc.chunk_acc, &t.chunk_acc);
}

// Builds the work list of one A'y variant from the entry counts per (block,
// chunk): super-chunks of at most per_sc chunks of columns, each split into
// block ranges so that items carry about equal numbers of entries.
// The most G32 entries of any item: its super-chunk's chunks over its blocks.
int64_t max_item_entries(const FastGeometry& g, const std::vector<int64_t>& entries_bc, const Pieces& pc,
                         const std::vector<int>& item_sc, const std::vector<int>& item_b0,
                         const std::vector<int>& item_b1)
{
    const int nsc = pc.sc_width.empty() ? 0 : static_cast<int>(pc.sc_width.size());
    // prefix over blocks of every super-chunk's entries
    std::vector<int64_t> pre(static_cast<size_t>(g.nblocks + 1) * nsc, 0);
    for (int64_t b = 0; b < g.nblocks; b++) {
        for (int sc = 0; sc < nsc; sc++) pre[(b + 1) * nsc + sc] = pre[b * nsc + sc];
        for (int ch = 0; ch < g.nchunks; ch++) pre[(b + 1) * nsc + pc.chunk_sc[ch]] += entries_bc[b * g.nchunks + ch];
    }
    int64_t most = 0;
    for (size_t i = 0; i < item_sc.size(); i++)
        most = std::max(most, pre[static_cast<size_t>(item_b1[i]) * nsc + item_sc[i]] -
                                  pre[static_cast<size_t>(item_b0[i]) * nsc + item_sc[i]]);
    return most;
}

cas_status build_items(const FastGeometry& g, const std::vector<int64_t>& entries_bc, int per_sc, int items_per_sm,
                       bool range_major, bool pack, bool persistent, size_t elem, FastTranspose& t)
{
    t.per_sc = per_sc;
    t.range_major = range_major;
    t.items_per_sm = items_per_sm;
    t.pack = pack;
    t.persistent = persistent;
    const Pieces pc = pack_chunks(g, per_sc * kChunkCols, pack);
    MetaPack mp;
    pack_pieces(pc, t, mp);
    const int nsc = t.nsc;
    // entries per (problem, super-chunk); items never span problems
    std::vector<int64_t> sc_entries(static_cast<size_t>(g.nprob) * nsc, 0);
    int64_t total = 0;
    for (int q = 0; q < g.nprob; q++)
        for (int64_t b = g.pblk0[q]; b < g.pblk0[q + 1]; b++)
            for (int ch = 0; ch < g.nchunks; ch++) {
                sc_entries[static_cast<size_t>(q) * nsc + pc.chunk_sc[ch]] += entries_bc[b * g.nchunks + ch];
                total += entries_bc[b * g.nchunks + ch];
            }
    const int64_t target_items = static_cast<int64_t>(sm_count()) * items_per_sm;
    const double per_item = std::max<double>(1.0, static_cast<double>(total) / target_items);
    std::vector<int> item_sc, item_b0, item_b1, sc_item0;
    std::vector<int64_t> item_part;
    int64_t part_elems = 0;
    if (range_major && g.nprob == 1 && nsc > 1) {
        // One fit: every super-chunk shares one partition of the blocks into
        // ranges, and the items run range by range (within a range the
        // heaviest super-chunks first), so that the CTAs at work at one time
        // stage the y slices of the same few blocks: a slice comes from HBM
        // once and from L2 for the other super-chunks.  Items of one
        // super-chunk stay contiguous in the partial buffer, in range order,
        // which is the order its column sums add them in.
        const int64_t nb = g.pblk0[1] - g.pblk0[0];
        const int64_t nr = std::max<int64_t>(1, std::min<int64_t>(nb, (target_items + nsc - 1) / nsc));
        std::vector<int> order(nsc);
        for (int sc = 0; sc < nsc; sc++) order[sc] = sc;
        std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return sc_entries[a] > sc_entries[b]; });
        // partials in item order; each super-chunk's items listed for the
        // column sums in range order
        std::vector<std::vector<int64_t>> by_sc(nsc);
        for (int64_t r = 0; r < nr; r++)
            for (int sc : order) {
                item_sc.push_back(sc);
                item_b0.push_back(static_cast<int>(g.pblk0[0] + nb * r / nr));
                item_b1.push_back(static_cast<int>(g.pblk0[0] + nb * (r + 1) / nr));
                item_part.push_back(part_elems);
                by_sc[sc].push_back(part_elems);
                part_elems += pc.sc_width[sc];
            }
        std::vector<int64_t> part_by_sc;
        part_by_sc.reserve(item_sc.size());
        for (int sc = 0; sc < nsc; sc++) {
            sc_item0.push_back(static_cast<int>(part_by_sc.size()));
            part_by_sc.insert(part_by_sc.end(), by_sc[sc].begin(), by_sc[sc].end());
        }
        sc_item0.push_back(static_cast<int>(part_by_sc.size()));
        t.nitems = static_cast<int>(item_sc.size());
        t.max_item_entries = max_item_entries(g, entries_bc, pc, item_sc, item_b0, item_b1);
        mp.add(item_sc, &t.item_sc);
        mp.add(item_b0, &t.item_b0);
        mp.add(item_b1, &t.item_b1);
        mp.add(item_part, &t.item_part);
        mp.add(sc_item0, &t.sc_item0);
        mp.add(part_by_sc, &t.sc_part);
        mp.add(std::vector<int>{0, 0}, &t.ctr);
        CAS_TRY(mp.upload(&t.meta));
        CAS_CUDA(dmalloc(&t.partial, elem * std::max<int64_t>(part_elems, 1)));
        return CAS_OK;
    }
    for (int q = 0; q < g.nprob; q++) {
        const int64_t qb0 = g.pblk0[q], qnb = g.pblk0[q + 1] - g.pblk0[q];
        for (int sc = 0; sc < nsc; sc++) {
            sc_item0.push_back(static_cast<int>(item_sc.size()));
            if (qnb == 0) continue;
            int64_t n = static_cast<int64_t>(std::llround(sc_entries[static_cast<size_t>(q) * nsc + sc] / per_item));
            // batched layouts: at most kBatchItemBlocks blocks per item, and
            // one block per item for problems of at most kBatchSmallBlocks
            // blocks (the small stages that iterate longest), so that a
            // problem left alone (or with few others) still has short units:
            // a unit's blocks run one after another in one CTA
            if (g.nprob > 1)
                n = std::max<int64_t>(n, qnb <= kBatchSmallBlocks ? qnb
                                                                  : (qnb + kBatchItemBlocks - 1) / kBatchItemBlocks);
            n = std::max<int64_t>(1, std::min<int64_t>(n, qnb));
            for (int64_t i = 0; i < n; i++) {
                item_sc.push_back(sc);
                item_b0.push_back(static_cast<int>(qb0 + qnb * i / n));
                item_b1.push_back(static_cast<int>(qb0 + qnb * (i + 1) / n));
                item_part.push_back(part_elems);
                part_elems += pc.sc_width[sc];
            }
        }
    }
    sc_item0.push_back(static_cast<int>(item_sc.size()));
    t.nitems = static_cast<int>(item_sc.size());
    t.max_item_entries = max_item_entries(g, entries_bc, pc, item_sc, item_b0, item_b1);
    mp.add(item_sc, &t.item_sc);
    mp.add(item_b0, &t.item_b0);
    mp.add(item_b1, &t.item_b1);
    mp.add(item_part, &t.item_part);
    mp.add(sc_item0, &t.sc_item0);
    mp.add(item_part, &t.sc_part);  // items are listed super-chunk by super-chunk already
    mp.add(std::vector<int>{0, 0}, &t.ctr);
    CAS_TRY(mp.upload(&t.meta));
    CAS_CUDA(dmalloc(&t.partial, elem * std::max<int64_t>(part_elems, 1)));
    return CAS_OK;
}

// Work list of one item per (block, chunk), block-major, for adjoints over a
// block range (minibatches): item b * nchunks + ch, one piece per chunk;
// partial offsets give the layout [block][global column] relative to the
// first item of the range.
cas_status build_block_items(const FastGeometry& g, FastTranspose& t)
{
    t.per_sc = 1;
    Pieces pc;
    for (int ch = 0; ch < g.nchunks; ch++) {
        pc.sc_piece0.push_back(ch);
        pc.sc_width.push_back(chunk_width(g, ch));
        pc.pat.push_back(pattern_of_chunk(g, ch));
        pc.ch0.push_back(ch);
        pc.ch1.push_back(ch + 1);
        pc.acc.push_back(0);
        pc.chunk_sc.push_back(ch);
        pc.chunk_acc.push_back(0);
    }
    pc.sc_piece0.push_back(g.nchunks);
    MetaPack mp;
    pack_pieces(pc, t, mp);
    const int64_t n = g.nblocks * g.nchunks;
    t.nitems = static_cast<int>(n);
    std::vector<int> isc(n), ib0(n), ib1(n);
    std::vector<int64_t> ipart(n);
    for (int64_t b = 0; b < g.nblocks; b++)
        for (int ch = 0; ch < g.nchunks; ch++) {
            const int p = pattern_of_chunk(g, ch);
            const int64_t i = b * g.nchunks + ch;
            isc[i] = ch;
            ib0[i] = static_cast<int>(b);
            ib1[i] = static_cast<int>(b + 1);
            ipart[i] = b * g.cols + g.off[p] + static_cast<int64_t>(ch - g.chunk0[p]) * kChunkCols;
        }
    mp.add(isc, &t.item_sc);
    mp.add(ib0, &t.item_b0);
    mp.add(ib1, &t.item_b1);
    mp.add(ipart, &t.item_part);
    return mp.upload(&t.meta);
}

TView tview(const FastTranspose& t)
{
    TView v;
    v.per_sc = t.per_sc;
    v.item_sc = t.item_sc;
    v.item_b0 = t.item_b0;
    v.item_b1 = t.item_b1;
    v.item_part = t.item_part;
    v.sc_piece0 = t.sc_piece0;
    v.sc_width = t.sc_width;
    v.piece_pat = t.piece_pat;
    v.piece_ch0 = t.piece_ch0;
    v.piece_ch1 = t.piece_ch1;
    v.piece_acc = t.piece_acc;
    v.sc_item0 = t.sc_item0;
    v.nsc = t.nsc;
    v.nitems = t.nitems;
    return v;
}

template <typename T>
const FastTranspose& transpose_of(const FastLayout& f)
{
    return sizeof(T) == 4 ? f.t32 : f.t64;
}

template <typename T>
size_t spmv_t_smem(int per_sc)
{
    return sizeof(T) * (static_cast<size_t>(kChunkCols) * per_sc + kBlockRows);
}

void free_transpose(FastTranspose& t)
{
    dfree(t.meta);
    dfree(t.partial);
    t = FastTranspose{};
}

// Opt-in shared memory for every product kernel (set outside any stream
// capture, at the first build on each device).
cas_status fast_set_attributes_now();
cas_status fast_set_attributes()
{
    static std::mutex mu;
    static std::vector<char> done;
    int dev = 0;
    CAS_CUDA(cudaGetDevice(&dev));
    std::lock_guard<std::mutex> lk(mu);
    if (static_cast<int>(done.size()) <= dev) done.resize(dev + 1, 0);
    if (done[dev]) return CAS_OK;
    CAS_TRY(fast_set_attributes_now());
    done[dev] = 1;
    return CAS_OK;
}
cas_status fast_set_attributes_now()
{
    const int s32 = static_cast<int>(sizeof(float) * kTable32), s64 = static_cast<int>(sizeof(double) * kTable64);
    const int t32 = static_cast<int>(spmv_t_smem<float>(kMaxSc));
    const int t64 = static_cast<int>(spmv_t_smem<double>(1));
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

// ---------------------------------------------------------------------------
// Build-time autotuner of the FP32 A'y schedule.  Every candidate work list
// is built and timed (partials + column sums, CUDA events, one warm-up
// launch) on this layout; the fastest is kept and remembered per geometry
// for the rest of the process, so later builds of the same shape skip the
// timing.  CAS_ATY_SCHEDULE="chunks,range_major,items_per_sm,pack,persistent"
// forces a schedule.
// ---------------------------------------------------------------------------
struct Sched {
    int per_sc;
    bool range_major;
    int ips;
    bool pack;
    bool persistent;
};
constexpr Sched kSchedDefault = {4, false, 2, false, false};
constexpr Sched kSchedCandidates[] = {
    {4, false, 2, false, false}, {4, false, 3, false, false}, {4, false, 2, true, true}, {4, false, 4, true, true},
    {4, false, 4, false, true},  {2, false, 4, true, true},   {4, false, 6, false, true}, {4, true, 2, false, false},
    {4, true, 4, false, true},   {4, true, 6, false, true},   {4, true, 4, true, true},   {2, true, 4, true, true}};
static_assert(sizeof(kSchedCandidates) / sizeof(Sched) <= kMaxTune, "tune table");
constexpr int64_t kTuneMinBlocks = 64;  // smaller layouts take the default schedule

std::mutex g_tune_mu;
std::map<std::string, Sched> g_tune_cache;

std::string tune_key(const FastGeometry& g)
{
    std::string k = std::to_string(g.k) + "/" + std::to_string(g.nblocks) + "/" + std::to_string(g.rows);
    for (int p = 0; p < g.npat; p++) k += "/" + std::to_string(g.space[p]) + "x" + std::to_string(g.slots[p]);
    for (int q = 0; q <= g.nprob; q++) k += ":" + std::to_string(g.pblk0[q]);
    return k;
}

bool valid_sched(const Sched& c)
{
    return c.per_sc >= 1 && c.per_sc <= kMaxSc && c.ips >= 1 && c.ips <= 16;
}

cas_status tune_transpose(FastLayout& f, const std::vector<int64_t>& entries, cudaStream_t s)
{
    const FastGeometry& g = f.g;
    f.ntune = 0;
    f.tune_cached = 0;
    auto build = [&](const Sched& c) {
        return build_items(g, entries, c.per_sc, c.ips, c.range_major, c.pack, c.persistent, sizeof(float), f.t32);
    };
    if (const char* env = std::getenv("CAS_ATY_SCHEDULE")) {
        int a = 0, b = 0, c = 0, d = 0, e = 0;
        const int n = std::sscanf(env, "%d,%d,%d,%d,%d", &a, &b, &c, &d, &e);
        const Sched forced{a, b != 0, c, d != 0, e != 0};
        CAS_REQUIRE(n == 5 && valid_sched(forced), CAS_ERR_INVALID_ARGUMENT,
                    "CAS_ATY_SCHEDULE must be \"chunks,range_major,items_per_sm,pack,persistent\" within limits");
        return build(forced);
    }
    if (g.nblocks < kTuneMinBlocks) return build(kSchedDefault);
    const std::string key = tune_key(g);
    {
        std::lock_guard<std::mutex> lk(g_tune_mu);
        auto it = g_tune_cache.find(key);
        if (it != g_tune_cache.end()) {
            f.tune_cached = 1;
            return build(it->second);
        }
    }
    float* y = nullptr;
    float* x = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    cas_status st = CAS_OK;
    auto fail = [&](cudaError_t e) {
        if (e != cudaSuccess && st == CAS_OK) {
            set_error(std::string("autotuner: ") + cudaGetErrorString(e));
            st = CAS_ERR_CUDA;
        }
    };
    fail(dmalloc(&y, sizeof(float) * g.rows));
    fail(dmalloc(&x, sizeof(float) * std::max<int64_t>(g.cols, 1)));
    fail(cudaEventCreate(&e0));
    fail(cudaEventCreate(&e1));
    if (st == CAS_OK) fail(cudaMemsetAsync(y, 0, sizeof(float) * g.rows, s));
    Sched best = kSchedDefault;
    float best_ms = 1e30f;
    for (const Sched& c : kSchedCandidates) {
        if (st != CAS_OK) break;
        st = build(c);
        if (st == CAS_OK) st = fast_spmv_t<float>(f, y, x, s);  // warm-up
        if (st == CAS_OK) fail(cudaEventRecord(e0, s));
        for (int r = 0; r < 2 && st == CAS_OK; r++) st = fast_spmv_t<float>(f, y, x, s);
        if (st == CAS_OK) fail(cudaEventRecord(e1, s));
        if (st == CAS_OK) fail(cudaEventSynchronize(e1));
        float ms = 0;
        if (st == CAS_OK) fail(cudaEventElapsedTime(&ms, e0, e1));
        free_transpose(f.t32);
        if (st != CAS_OK) break;
        ms *= 0.5f;
        f.tune[f.ntune++] =
            FastTuneEntry{c.per_sc, c.range_major ? 1 : 0, c.ips, c.pack ? 1 : 0, c.persistent ? 1 : 0, ms};
        if (ms < best_ms) {
            best_ms = ms;
            best = c;
        }
    }
    dfree(y);
    dfree(x);
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    if (st != CAS_OK) return st;
    {
        std::lock_guard<std::mutex> lk(g_tune_mu);
        g_tune_cache[key] = best;
    }
    return build(best);
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
    dfree(f.a16);
    dfree(f.g32);
    dfree(f.sub_start);
    free_transpose(f.t32);
    free_transpose(f.t64);
    free_transpose(f.tb);
    dfree(f.eval_partial);
    dfree(f.eval_dscore);
    dfree(f.eval_red);
    dfree(f.eval_ctr);
    f = FastLayout{};
}

cas_status fast_build(const DevicePatterns& dp, const PatternSet& ps, const uint64_t* d_pos, int64_t rows,
                      const int64_t* prob_rows, int nprob, uint64_t* diag_int, FastLayout& f, cudaStream_t s,
                      const PositionChunks* chunks)
{
    cas::NvtxRange nvtx_range("blocked layout build");
    CAS_REQUIRE(fast_supported(ps), CAS_ERR_INVALID_ARGUMENT, "pattern set does not fit the blocked layout");
    CAS_REQUIRE(nprob >= 1 && nprob <= kMaxProblems, CAS_ERR_INVALID_ARGUMENT,
                "blocked layout: 1 to 64 problems per batch");
    CAS_TRY(fast_set_attributes());
    FastGeometry& g = f.g;
    g = FastGeometry{};
    g.npat = static_cast<int>(ps.indexers.size());
    g.k = dp.k;
    g.rows = rows;
    g.nprob = nprob;
    g.pcols = ps.cols;
    g.cols = ps.cols * nprob;
    // problem table: rows and whole blocks of each problem
    int64_t r0 = 0, b0 = 0;
    for (int q = 0; q < nprob; q++) {
        const int64_t rq = prob_rows ? prob_rows[q] : rows;
        CAS_REQUIRE(rq >= 0, CAS_ERR_INVALID_ARGUMENT, "blocked layout: negative problem size");
        g.prow0[q] = r0;
        g.pblk0[q] = static_cast<int>(b0);
        r0 += rq;
        b0 += (rq + kBlockRows - 1) / kBlockRows;
    }
    g.prow0[nprob] = r0;
    g.pblk0[nprob] = static_cast<int>(b0);
    CAS_REQUIRE(r0 == rows, CAS_ERR_SIZE_MISMATCH, "blocked layout: problem sizes do not add up to the rows");
    g.nblocks = b0;
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
    CAS_REQUIRE(g.total_elems() < 0xFFFFFFFFLL, CAS_ERR_INVALID_ARGUMENT,
                "blocked layout: 2^32 or more entries (with block padding) are not supported");
    const int64_t elems = std::max<int64_t>(g.total_elems(), 8);
    CAS_CUDA(dmalloc(&f.a16, sizeof(uint16_t) * elems));
    CAS_CUDA(dmalloc(&f.g32, sizeof(uint32_t) * elems));
    const int64_t nsub = g.nblocks * g.nchunks * kSubPerChunk;
    CAS_CUDA(dmalloc(&f.sub_start, sizeof(uint32_t) * std::max<int64_t>(nsub, 1)));
    if (rows > 0) {
        const int threads = 256;
        // one launch over all rows, or one per arriving chunk behind its copy
        const int nch = chunks ? chunks->n : 1;
        int64_t r0 = 0;
        for (int c = 0; c < nch; c++) {
            const int64_t r1 = chunks ? std::min(chunks->row_end[c], rows) : rows;
            if (chunks) CAS_CUDA(cudaStreamWaitEvent(s, chunks->ready[c], 0));
            if (r1 > r0) {
                const unsigned grid = fgrid(r1 - r0, threads);
                { fast_index_kernel<<<grid * 4, kIndexThreads, kIndexBoardBytes + sizeof(Instance) * dp.k, s>>>(
                    dp.instances, dp.k, dp.tables, reinterpret_cast<const ulonglong2*>(d_pos), g, f.a16, r0, r1);
                  cas::count_launch(); }
                CAS_CHECK_LAUNCH();
            }
            r0 = std::max(r0, r1);
        }
        if (r0 < rows) {  // rows past the last chunk (all chunks are waited for above)
            { fast_index_kernel<<<fgrid(rows - r0, kIndexThreads) * 4, kIndexThreads, kIndexBoardBytes + sizeof(Instance) * dp.k, s>>>(
                dp.instances, dp.k, dp.tables, reinterpret_cast<const ulonglong2*>(d_pos), g, f.a16, r0, rows);
              cas::count_launch(); }
            CAS_CHECK_LAUNCH();
        }
        const int64_t groups = g.nblocks * g.npat;
        const unsigned sgrid =
            static_cast<unsigned>(std::min<int64_t>(groups, static_cast<int64_t>(sm_count()) * kSortCtasPerSm));
        uint32_t* scratch = nullptr;
        CAS_CUDA(dmalloc(&scratch, sizeof(uint32_t) * kBlockRows * 8 * sgrid));
        { fast_sort_kernel<<<sgrid, kSortThreads, 0, s>>>(g, f.a16, f.g32, scratch); cas::count_launch(); }
        CAS_CHECK_LAUNCH();
        dfree(scratch);
        { fast_sub_kernel<<<fgrid(nsub, 256), 256, 0, s>>>(g, f.g32, f.sub_start); cas::count_launch(); }
        CAS_CHECK_LAUNCH();
    }
    // entries per (block, chunk) -> work items
    std::vector<int64_t> entries(static_cast<size_t>(g.nblocks * g.nchunks), 0);
    if (!entries.empty() && rows > 0) {
        std::vector<uint32_t> ce(entries.size());
        uint32_t* d_ce = nullptr;
        CAS_CUDA(dmalloc(&d_ce, sizeof(uint32_t) * ce.size()));
        { fast_chunk_entries_kernel<<<fgrid(static_cast<int64_t>(ce.size()), 256), 256, 0, s>>>(g, f.sub_start, d_ce); cas::count_launch(); }
        CAS_CHECK_LAUNCH();
        CAS_CUDA(cudaMemcpyAsync(ce.data(), d_ce, sizeof(uint32_t) * ce.size(), cudaMemcpyDeviceToHost, s));
        CAS_CUDA(cudaStreamSynchronize(s));
        dfree(d_ce);
        for (size_t i = 0; i < ce.size(); i++) entries[i] = ce[i];
    }
    if (g.nblocks > 0) {
        CAS_TRY(tune_transpose(f, entries, s));
        // FP64 items hold one chunk, so the y slices would be read once per
        // chunk: always range by range
        CAS_TRY(build_items(g, entries, 1, 2, true, true, false, sizeof(double), f.t64));
        if (g.nprob == 1) CAS_TRY(build_block_items(g, f.tb));  // evaluator minibatches: single fits only
        if (diag_int && rows > 0) CAS_TRY(fast_diag(f, diag_int, s));
    }
    return CAS_OK;
}

cas_status fast_diag(const FastLayout& f, uint64_t* diag, cudaStream_t s)
{
    const int64_t groups = f.g.nblocks * f.g.npat;
    if (f.g.cols == 0) return CAS_OK;
    if (groups == 0) {
        CAS_CUDA(cudaMemsetAsync(diag, 0, sizeof(uint64_t) * f.g.cols, s));
        return CAS_OK;
    }
    const unsigned grid = std::min<unsigned>(static_cast<unsigned>(groups), sm_count() * 8);
    int max_slots = 0;
    for (int p = 0; p < f.g.npat; p++) max_slots = std::max(max_slots, f.g.slots[p]);
    // a column's count inside an item is at most the item's entries;
    // CAS_DIAG_FROM_G32=1 takes the direct count whatever the items
    const char* direct = std::getenv("CAS_DIAG_FROM_G32");
    const bool exact32 = f.t32.nitems > 0 && f.t32.partial && !(direct && std::strcmp(direct, "1") == 0) &&
                         f.t32.max_item_entries < (int64_t(1) << 24);
    if (!exact32) {
        CAS_CUDA(cudaMemsetAsync(diag, 0, sizeof(uint64_t) * f.g.cols, s));
        { fast_diag_kernel<<<grid, 256, 0, s>>>(f.g, f.g32, diag); cas::count_launch(); }
        CAS_CHECK_LAUNCH();
        return CAS_OK;
    }
    CAS_TRY(fast_spmv_t_partials<float>(f, nullptr, nullptr, s));  // no y: ones
    { fast_count_kernel<<<fgrid(f.g.cols, 256), 256, 0, s>>>(fast_cols<float>(f), static_cast<const float*>(f.t32.partial), diag); cas::count_launch(); }
    CAS_CHECK_LAUNCH();
    const int stretches = (kBlockRows * max_slots + kRepeatRounds * kRound - 1) / (kRepeatRounds * kRound);
    const int64_t warps = groups * stretches;
    const unsigned rgrid = static_cast<unsigned>(std::max<int64_t>(1, std::min<int64_t>((warps + 7) / 8, sm_count() * 8)));
    { fast_repeat_kernel<<<rgrid, 256, 0, s>>>(f.g, f.g32, diag, stretches); cas::count_launch(); }
    CAS_CHECK_LAUNCH();
    return CAS_OK;
}

int fast_ax_splits(int64_t nblocks) { return unit_splits(nblocks, sm_count(), kAxSplitMax); }

template <typename T, typename Y>
cas_status fast_spmv(const FastLayout& f, const T* x, Y* y, const double* b, const double* coef, double* part,
                     int* done_flag, int mode, cudaStream_t s, int* n_parts, const int* pdone, const FastActive* act)
{
    const int split = act ? 1 : fast_ax_splits(f.g.nblocks);
    const int64_t units = f.g.nblocks * (act ? kAxSplitMax : split);
    const int ctas = static_cast<int>(std::max<int64_t>(1, std::min<int64_t>(units, sm_count())));
    if (n_parts) *n_parts = static_cast<int>(units);  // one norm partial per (block, split)
    if (f.g.nblocks == 0) return CAS_OK;
    const size_t smem = sizeof(T) * (sizeof(T) == 4 ? kTable32 : kTable64);
    const bool direct = act || split == kAxSplitMax;
    const bool staged = act || split != kAxSplitMax;
    auto launch = [&](auto kern) -> cas_status {
        { kern<<<ctas, kAxThreads, smem, s>>>(f.g, f.a16, x, y, b, coef, part, done_flag, pdone, act, split, ctas); cas::count_launch(); }
        CAS_CHECK_LAUNCH();
        return CAS_OK;
    };
    bool all8 = true;
    for (int p = 0; p < f.g.npat; p++) all8 = all8 && f.g.slots[p] == 8;
    if (direct) {
        const unsigned dgrid = static_cast<unsigned>(
            std::max<int64_t>(1, std::min<int64_t>(f.g.nblocks * kAxSplitMax, 4LL * sm_count())));
        const bool d8 = all8 && f.g.npat <= kDirectPatterns;
        auto kd = d8 ? (mode == 0 ? fast_spmv_direct_kernel<T, Y, 0, true>
                                  : (mode == 1 ? fast_spmv_direct_kernel<T, Y, 1, true>
                                               : fast_spmv_direct_kernel<T, Y, 2, true>))
                     : (mode == 0 ? fast_spmv_direct_kernel<T, Y, 0, false>
                                  : (mode == 1 ? fast_spmv_direct_kernel<T, Y, 1, false>
                                               : fast_spmv_direct_kernel<T, Y, 2, false>));
        { kd<<<dgrid, kAxDirectRows, 0, s>>>(f.g, f.a16, x, y, b, coef, part, done_flag, pdone, act, ctas); cas::count_launch(); }
        CAS_CHECK_LAUNCH();
    }
    if (!staged) return CAS_OK;
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
cas_status fast_spmv_t_partials(const FastLayout& f, const T* y, int* done_flag, cudaStream_t s, const int* pdone,
                                const FastActive* act)
{
    const FastTranspose& t = transpose_of<T>(f);
    if (t.nitems == 0) return CAS_OK;
    const size_t smem = spmv_t_smem<T>(t.per_sc);
    // with an active list the kernel splits the units itself (persistent);
    // else the items are split so that a short list still fills the GPU
    const int nsplit = act ? 1 : unit_splits(t.nitems, sm_count(), kAtySplitMax);
    const int units = t.nitems * nsplit;
    const bool persistent = t.persistent || act;
    const unsigned grid = static_cast<unsigned>(persistent ? std::min(units, sm_count()) : units);
    const unsigned pgrid = act ? static_cast<unsigned>(sm_count()) : grid;
    int* ctr = persistent ? t.ctr : nullptr;
    { fast_spmv_t_kernel<T><<<pgrid, kFastThreads, smem, s>>>(f.g, tview(t), f.g32, f.sub_start, y,
                                                                  static_cast<T*>(t.partial), done_flag, 0, 0,
                                                                  ctr, pdone, act, nsplit); cas::count_launch(); }
    CAS_CHECK_LAUNCH();
    return CAS_OK;
}

template <typename T>
FastCols fast_cols(const FastLayout& f)
{
    const FastTranspose& t = transpose_of<T>(f);
    FastCols c;
    c.g = f.g;
    c.nsc = t.nsc;
    c.chunk_sc = t.chunk_sc;
    c.chunk_acc = t.chunk_acc;
    c.sc_item0 = t.sc_item0;
    c.sc_part = t.sc_part;
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

// The evaluator's per-call buffers for adjoints over nb blocks (grown, never
// shrunk).  A call made while `s` is capturing marks them as held by a CUDA
// graph: from then on a call that would grow them (and so free the buffers
// the graph's kernels use) is refused, captured or not, and so is growing
// during a capture.  Growing waits for the whole device, since eager work
// on other streams may still use the old buffers.
static cas_status eval_buffers(FastLayout& f, int64_t nb, cudaStream_t s)
{
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    CAS_CUDA(cudaStreamIsCapturing(s, &cap));
    const bool capturing = cap != cudaStreamCaptureStatusNone;
    if (nb > f.eval_blocks) {
        CAS_REQUIRE(!capturing, CAS_ERR_INVALID_ARGUMENT,
                    "evaluator step: a captured call may not grow the matrix's evaluator scratch; make one call of "
                    "the largest minibatch before capturing");
        CAS_REQUIRE(!f.eval_captured, CAS_ERR_INVALID_ARGUMENT,
                    "evaluator step: the matrix's evaluator scratch is held by captured CUDA graphs; a call over "
                    "more blocks than they were captured with would reallocate it (use a new matrix)");
        if (f.eval_partial || f.eval_dscore) {
            CAS_CUDA(cudaDeviceSynchronize());
            dfree(f.eval_partial);
            dfree(f.eval_dscore);
            f.eval_partial = nullptr;
            f.eval_dscore = nullptr;
            f.eval_blocks = 0;
        }
        CAS_CUDA(dmalloc(&f.eval_partial, sizeof(float) * nb * f.g.cols));
        CAS_CUDA(dmalloc(&f.eval_dscore, sizeof(float) * nb * kBlockRows));
        f.eval_blocks = nb;
    }
    if (!f.eval_red) {
        CAS_REQUIRE(!capturing, CAS_ERR_INVALID_ARGUMENT,
                    "evaluator step: make one call of the largest minibatch before capturing");
        CAS_CUDA(dmalloc(&f.eval_red, sizeof(double) * 2 * kEvalRedMax));
        CAS_CUDA(dmalloc(&f.eval_ctr, sizeof(int)));
        CAS_CUDA(cudaMemsetAsync(f.eval_ctr, 0, sizeof(int), s));
    }
    if (capturing) f.eval_captured = true;
    return CAS_OK;
}

// The adjoint's per-block partials of blocks [b0, b1) on g into eval_partial.
// One CTA per (block, chunk) item: splitting a minibatch's items over more
// CTAs re-stages y per split and was measured slower (8.6 against 6.8 ms
// per epoch of the 8M-row evaluator workload).
static cas_status eval_adjoint_partials(FastLayout& f, int64_t b0, int64_t b1, const float* g, cudaStream_t s)
{
    const size_t smem = spmv_t_smem<float>(1);
    const int items = static_cast<int>((b1 - b0) * f.g.nchunks);
    { fast_spmv_t_kernel<float><<<items, kFastThreads, smem, s>>>(f.g, tview(f.tb), f.g32, f.sub_start, g,
                                                                 f.eval_partial, nullptr,
                                                                 static_cast<int>(b0 * f.g.nchunks), b0, nullptr,
                                                                 nullptr, nullptr, 1); cas::count_launch(); }
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
    CAS_TRY(eval_buffers(f, nb, s));
    CAS_TRY(eval_adjoint_partials(f, b0, b1, g, s));
    { block_partial_sum_kernel<<<fgrid(f.g.cols, 256), 256, 0, s>>>(f.eval_partial, static_cast<int>(nb), f.g.cols,
                                                                  grad); cas::count_launch(); }
    CAS_CHECK_LAUNCH();
    return CAS_OK;
}

cas_status fast_eval_adam_step(FastLayout& f, int64_t row0, int64_t row1, const float* target, float* w, float* m,
                               float* v, int64_t* step, double* loss_sum, const EvalAdam& o, cudaStream_t s)
{
    const int64_t n = row1 - row0;
    const int64_t b0 = row0 / kBlockRows, b1 = (row1 + kBlockRows - 1) / kBlockRows;
    if (f.g.cols == 0 || n <= 0) return CAS_OK;
    CAS_TRY(eval_buffers(f, b1 - b0, s));
    const unsigned g1 = std::min<unsigned>(fgrid(n, 256), kEvalRedMax);  // one thread per row up to 4 CTAs per SM
    { eval_loss_grad_kernel<<<g1, 256, 0, s>>>(f.g, f.a16, w, target, row0, row1, o.delta, 1.0f / static_cast<float>(n),
                                               f.eval_dscore, f.eval_red); cas::count_launch(); }
    CAS_CHECK_LAUNCH();
    CAS_TRY(eval_adjoint_partials(f, b0, b1, f.eval_dscore, s));
    const unsigned g3 = std::min<unsigned>(fgrid(f.g.cols, 256), kEvalRedMax);
    { eval_adam_kernel<<<g3, 256, 0, s>>>(f.eval_partial, static_cast<int>(b1 - b0), f.g.cols, w, m, v, step,
                                          loss_sum, f.eval_red, static_cast<int>(g1), f.eval_ctr, o,
                                          1.0 / static_cast<double>(n)); cas::count_launch(); }
    CAS_CHECK_LAUNCH();
    return CAS_OK;
}

template cas_status fast_spmv<float, float>(const FastLayout&, const float*, float*, const double*, const double*,
                                            double*, int*, int, cudaStream_t, int*, const int*, const FastActive*);
template cas_status fast_spmv<double, double>(const FastLayout&, const double*, double*, const double*,
                                              const double*, double*, int*, int, cudaStream_t, int*, const int*,
                                              const FastActive*);
template cas_status fast_spmv<double, float>(const FastLayout&, const double*, float*, const double*, const double*,
                                             double*, int*, int, cudaStream_t, int*, const int*, const FastActive*);
template cas_status fast_spmv_t_partials<float>(const FastLayout&, const float*, int*, cudaStream_t, const int*,
                                                const FastActive*);
template cas_status fast_spmv_t_partials<double>(const FastLayout&, const double*, int*, cudaStream_t, const int*,
                                                 const FastActive*);
template FastCols fast_cols<float>(const FastLayout&);
template FastCols fast_cols<double>(const FastLayout&);
template cas_status fast_spmv_t<float>(const FastLayout&, const float*, float*, cudaStream_t);
template cas_status fast_spmv_t<double>(const FastLayout&, const double*, double*, cudaStream_t);

}  // namespace cas
