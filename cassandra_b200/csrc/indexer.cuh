// Device evaluation of the indexer recipes built by patterns.cpp: the
// ternary digits of a square list and the per-kind combination of
// Pattern/Indexer.cpp:17-317.
#pragma once
#include <cstdint>

#include "patterns.h"

namespace cas {

__device__ __forceinline__ uint32_t digits(const uint8_t* sq, int n, uint32_t plo, uint32_t phi, uint32_t olo,
                                           uint32_t ohi)
{
    uint32_t idx = 0;
    for (int i = n - 1; i >= 0; i--) {
        const int t = sq[i];
        const uint32_t pw = t < 32 ? plo : phi, ow = t < 32 ? olo : ohi;
        const int sh = t & 31;
        idx = idx * 3 + ((pw >> sh) & 1u) + (((ow >> sh) & 1u) << 1);
    }
    return idx;
}

// A row's cells as a digit board in shared memory: board[t * STRIDE] =
// cell(pos, t) for the 64 squares, one byte each.  With STRIDE the CTA's
// thread count and board = base + threadIdx.x, a warp's 32 rows sit in 32
// consecutive bytes of every square's line: reads and writes of one square
// by a warp touch 8 words, without bank conflicts.
template <int STRIDE>
__device__ __forceinline__ void fill_board(uint8_t* board, uint32_t plo, uint32_t phi, uint32_t olo, uint32_t ohi)
{
#pragma unroll
    for (int t = 0; t < 32; t++) {
        board[t * STRIDE] = static_cast<uint8_t>(((plo >> t) & 1u) | (((olo >> t) & 1u) << 1));
        board[(t + 32) * STRIDE] = static_cast<uint8_t>(((phi >> t) & 1u) | (((ohi >> t) & 1u) << 1));
    }
}

template <int STRIDE>
__device__ __forceinline__ uint32_t board_digits(const uint8_t* sq, int n, const uint8_t* board)
{
    uint32_t idx = 0;
    for (int i = n - 1; i >= 0; i--) idx = idx * 3 + board[sq[i] * STRIDE];
    return idx;
}

// The per-kind combination of an instance's square lists; dig(list, n)
// gives the digits of one list.
template <typename Digits>
__device__ __forceinline__ uint32_t combine_slot(const Instance& in, const uint32_t* __restrict__ tables, Digits&& dig)
{
    uint32_t r;
    if (in.kind == kDirect) {
        r = dig(in.sq[0], in.n0);
    } else if (in.kind == kTable) {
        r = __ldg(tables + in.table_offset + dig(in.sq[0], in.n0));
    } else {
        uint32_t a = dig(in.sq[0], in.n0);
        uint32_t b = dig(in.sq[1], in.n1);
        const uint32_t lo = min(a, b), hi = max(a, b);
        r = lo * in.half_size + hi - (lo * (lo + 1) / 2);
        if (in.kind == kDiagPair) r = r * in.diag_size + dig(in.sq[2], in.n2);
    }
    return in.offset + r;
}

__device__ __forceinline__ uint32_t eval_slot(const Instance& in, const uint32_t* __restrict__ tables, uint32_t plo,
                                              uint32_t phi, uint32_t olo, uint32_t ohi)
{
    return combine_slot(in, tables,
                        [&](const uint8_t* sq, int n) { return digits(sq, n, plo, phi, olo, ohi); });
}

// eval_slot from the row's digit board (fill_board), every kind inlined.
template <int STRIDE>
__device__ __forceinline__ uint32_t eval_slot_board_all(const Instance& in, const uint32_t* __restrict__ tables,
                                                        const uint8_t* board)
{
    return combine_slot(in, tables, [&](const uint8_t* sq, int n) { return board_digits<STRIDE>(sq, n, board); });
}

template <int STRIDE>
__device__ __noinline__ uint32_t eval_slot_board_other(const Instance& in, const uint32_t* __restrict__ tables,
                                                       const uint8_t* board)
{
    return eval_slot_board_all<STRIDE>(in, tables, board);
}

// The same for callers that unroll it over a pattern's slots: only the
// direct kind (every instance of the expanded mode) is inlined, as the other
// kinds' code would not fit the instruction cache beside it.
template <int STRIDE>
__device__ __forceinline__ uint32_t eval_slot_board(const Instance& in, const uint32_t* __restrict__ tables,
                                                    const uint8_t* board)
{
    if (in.kind == kDirect) return in.offset + board_digits<STRIDE>(in.sq[0], in.n0, board);
    return eval_slot_board_other<STRIDE>(in, tables, board);
}

}  // namespace cas
